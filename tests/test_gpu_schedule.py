"""GPU: dependency-ordered plan assembly (all colours in one persistent launch).

The fragment kernel's plan path runs its colours as one launch whose tiles wait,
in the kernel, for the groups (one colour within one band of element ids) whose
elements share nodes with theirs in earlier colours.  Checked here:
* the schedule tables: tiles cover every list position once, dependencies point
  to earlier groups, and every earlier-colour element that shares a node with an
  element is in a group that the element's group reaches through its
  dependencies (so each block still receives its contributions in colour order);
* results equal the colour-by-colour launches bit for bit (orders 2-4, LINEAR,
  NONLINEAR, MIXED, residual-only and Jacobian-only, structured, periodic and
  scrambled numbering, bands from 2 elements up), and the oracle within 1e-12;
* the bounded waits: a group that never completes (failure injection) makes its
  dependants' waits run out after the limit; the launch still ends, the call
  reports FEM_ERR_TIMEOUT, and the next assembly on the same context is correct."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12


def _scrambled(fem, m, seed):
    """The same mesh with node and element numbering permuted."""
    rng = np.random.default_rng(seed)
    perm = rng.permutation(m.num_nodes)
    inv = np.empty_like(perm)
    inv[perm] = np.arange(perm.size)
    n = m.nodes_per_element
    conn = inv[m.conn.reshape(-1, n)][rng.permutation(m.num_elements)].reshape(-1).astype(np.int32)
    return fem.Mesh(m.order, np.ascontiguousarray(m.coords[perm]), m.conn_ptr.copy(), conn,
                    np.ascontiguousarray(m.states[perm]), m.E, m.nu, m.t, m.name + "_scrambled")


MESHES = {
    "sq24x20_p2": lambda f: f.square_mesh(24, 20, 2, 2.0, 1.0, 0.2, seed=0x650),
    "sq17x13_p3": lambda f: f.square_mesh(17, 13, 3, 10.0, 10.0, 0.2, seed=0x651),
    "sq9x11_p4": lambda f: f.square_mesh(9, 11, 4, 1.0, 1.5, 0.15, seed=0x652),
    "ann6x40_p2": lambda f: f.annulus_mesh(6, 40, 2, seed=0x653),
    "ann5x17_p3": lambda f: f.annulus_mesh(5, 17, 3, seed=0x654),
    "scr_sq15x12_p3": lambda f: _scrambled(f, f.square_mesh(15, 12, 3, 1.0, 1.0, 0.2, seed=0x655), 0x656),
}


def _check_tables(fem, m, plan):
    nE = m.num_elements
    colour, nc = fem.colour_elements(m.num_nodes, m.conn_ptr, m.conn)
    listed = np.concatenate([np.nonzero(colour == c)[0] for c in range(nc)])
    tb = plan.schedule_tables()
    begin, count, group = tb["tile_begin"], tb["tile_count"], tb["tile_group"]
    G = tb["group_tiles"].size
    cover = np.zeros(nE, np.int64)
    grp = np.full(nE, -1)
    for b, c, g in zip(begin, count, group):
        cover[b:b + c] += 1
        grp[listed[b:b + c]] = g
    assert np.all(cover == 1)
    assert np.all(np.bincount(group, minlength=G) == tb["group_tiles"])
    # tiles in dispatch order: groups never decrease; even lengths except a group's last tile
    assert np.all(np.diff(group) >= 0)
    last = np.r_[group[1:] != group[:-1], True]
    assert np.all((count % 2 == 0) | last)
    gcol = np.full(G, -1)
    for e in range(nE):
        assert gcol[grp[e]] in (-1, colour[e])
        gcol[grp[e]] = colour[e]
    ptr, deps = tb["dep_ptr"], tb["deps"]
    reach = []
    for g in range(G):
        r = set()
        for d in deps[ptr[g]:ptr[g + 1]]:
            assert d < g
            r.add(int(d))
            r |= reach[d]
        reach.append(r)
    n = m.nodes_per_element
    conn = m.conn.reshape(-1, n)
    by_node = {}
    for e in range(nE):
        for a in conn[e]:
            by_node.setdefault(int(a), []).append(e)
    for els in by_node.values():
        for e1 in els:
            for e2 in els:
                if colour[e1] < colour[e2]:
                    assert grp[e1] in reach[grp[e2]], (e1, e2)


def _outputs(fem, cuda, m, plan, prec="fp64", strain="linear", res_on=True, mat_on=True):
    import torch
    d = fem.DeviceMesh(m, cuda)
    res = torch.full((m.num_nodes * 2,), 3.0, dtype=torch.float64, device=cuda) if res_on else None
    mat = torch.full((plan.nnzb * 4,), 3.0, dtype=torch.float64, device=cuda) if mat_on else None
    plan.assemble(d.states, d.coords, m.E, m.nu, m.t, res, mat, precision=prec, strain=strain)
    torch.cuda.synchronize()
    return (res.cpu().numpy() if res_on else None), (mat.cpu().numpy() if mat_on else None)


@pytest.mark.parametrize("name", list(MESHES))
@pytest.mark.parametrize("band", [0, 2, 6, 64])
def test_schedule_equals_colour_launches(fem, orc, cuda, name, band):
    m = MESHES[name](fem)
    plan = fem.Plan(m.order, m.num_nodes, m.conn_ptr, m.conn)
    try:
        assert plan.schedule()["groups"] == 0  # plans start with the colour launches
        modes = [("fp64", "linear", True, True), ("fp64", "linear", True, False), ("fp64", "linear", False, True)]
        if m.order in (2, 3):
            modes.append(("fp64", "nonlinear", True, True))
        if m.order == 3:
            modes.append(("mixed", "linear", True, True))
        plan.set_schedule(0)
        plan.set_layout("colours")  # the schedule orders the colour layout's groups
        ref = {k: _outputs(fem, cuda, m, plan, *k) for k in modes}
        if band:
            plan.set_schedule(band, 2 if band <= 6 else 0)
        else:
            plan.set_schedule(10**9)  # one band: the colours in sequence inside one launch
        _check_tables(fem, m, plan)
        for k in modes:
            assert plan.scheduled(k[1], k[0])
            got = _outputs(fem, cuda, m, plan, *k)
            for x, y in zip(got, ref[k]):
                assert (x is None and y is None) or np.array_equal(x, y), (k, band)
        assert plan.wait_status() == 0
        rowp, cols = plan.pattern()
        R0, A0 = orc.assemble(m, orc.element_bsr_map(m.conn_ptr, m.conn, m.nodes_per_element, rowp, cols), cols.size)
        R, A = ref[("fp64", "linear", True, True)]
        assert np.abs(R - R0).max() <= FP64_TOL * np.abs(R0).max()
        assert np.abs(A - A0).max() <= FP64_TOL * np.abs(A0).max()
    finally:
        plan.close()


def test_schedule_bounded_wait_runs_out_and_context_survives(fem, orc, cuda):
    import torch
    m = fem.square_mesh(20, 16, 3, 1.0, 1.0, 0.2, seed=0x657)
    plan = fem.Plan(m.order, m.num_nodes, m.conn_ptr, m.conn)
    try:
        plan.set_schedule(40, 2)
        tb = plan.schedule_tables()
        ptr = tb["dep_ptr"]
        # a group that others wait for
        waited = np.unique(tb["deps"])
        assert waited.size > 0
        plan.set_schedule_waits(wait_limit_ns=20_000_000, stall_group=int(waited[0]))
        d = fem.DeviceMesh(m, cuda)
        res = torch.empty(m.num_nodes * 2, dtype=torch.float64, device=cuda)
        mat = torch.empty(plan.nnzb * 4, dtype=torch.float64, device=cuda)
        with pytest.raises(fem.FemError) as ei:
            plan.assemble(d.states, d.coords, m.E, m.nu, m.t, res, mat, timed=True)
        assert ei.value.status == fem.FEM_ERR_TIMEOUT
        # asynchronous form: the count is read (and cleared) by schedule_status
        plan.assemble(d.states, d.coords, m.E, m.nu, m.t, res, mat)
        assert plan.wait_status() >= 1
        assert plan.wait_status() == 0
        # normal waits again: the same context assembles correctly
        plan.set_schedule_waits(stall_group=-1)
        plan.assemble(d.states, d.coords, m.E, m.nu, m.t, res, mat, timed=True)
        rowp, cols = plan.pattern()
        R0, A0 = orc.assemble(m, orc.element_bsr_map(m.conn_ptr, m.conn, m.nodes_per_element, rowp, cols), cols.size)
        assert np.abs(res.cpu().numpy() - R0).max() <= FP64_TOL * np.abs(R0).max()
        assert np.abs(mat.cpu().numpy() - A0).max() <= FP64_TOL * np.abs(A0).max()
        assert int(ptr[-1]) == tb["deps"].size
    finally:
        plan.close()


def test_schedule_rejects_order1_and_bad_stall_group(fem, cuda):
    m1 = fem.square_mesh(4, 4, 1, seed=0x658)
    p1 = fem.Plan(1, m1.num_nodes, m1.conn_ptr, m1.conn)
    try:
        with pytest.raises(fem.FemError) as ei:
            p1.set_schedule(64)
        assert ei.value.status == fem.FEM_ERR_UNSUPPORTED
    finally:
        p1.close()
    m = fem.square_mesh(4, 4, 2, seed=0x659)
    p = fem.Plan(2, m.num_nodes, m.conn_ptr, m.conn)
    try:
        with pytest.raises(fem.FemError) as ei:
            p.set_schedule_waits(stall_group=10**6)
        assert ei.value.status == fem.FEM_ERR_INVALID_ARGUMENT
    finally:
        p.close()
