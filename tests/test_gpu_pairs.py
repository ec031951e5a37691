"""GPU: the pair layout of the fragment kernel's single-mesh plan launches (orders
2-4; a warp assembles an element and its right neighbour in one step).  Against
the FP64 oracle at 1e-12; against the colour layout to rounding (a block's
contributions are added in another order only where more than two elements share
it); deterministic (the second element's reductions land after the first's);
every mode the fragment kernel serves: residual + Jacobian, residual only,
Jacobian only, NONLINEAR (orders 2, 3), MIXED (order 3); layout switching."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12


def _scramble(fem, m, seed):
    rng = np.random.default_rng(seed)
    nn = (m.order + 1) ** 2
    pe = rng.permutation(m.num_elements)
    pn = rng.permutation(m.num_nodes)
    inv = np.empty_like(pn)
    inv[pn] = np.arange(pn.size)
    conn = pn[m.conn.reshape(-1, nn)[pe]].reshape(-1).astype(np.int32)
    return fem.Mesh(m.order, m.coords[inv], np.arange(0, conn.size + 1, nn, dtype=np.int32), conn, m.states[inv],
                    m.E, m.nu, m.t)


MESHES = {
    "square_p2": lambda f: f.square_mesh(13, 9, 2, 1.0, 1.0, 0.15, seed=71),
    "square_p3": lambda f: f.square_mesh(11, 8, 3, 1.0, 1.0, 0.15, seed=72),
    "square_p4": lambda f: f.square_mesh(7, 6, 4, 1.0, 1.0, 0.15, seed=73),
    "annulus_p2": lambda f: f.annulus_mesh(5, 36, 2, seed=74),
    "scrambled_p3": lambda f: _scramble(f, f.square_mesh(9, 7, 3, 1.0, 1.0, 0.15, seed=75), 75),
}


def _run(fem, cuda, m, plan, d, prec="fp64", strain="linear", res_on=True, mat_on=True):
    import torch
    res = torch.full((m.num_nodes * 2,), float("nan"), dtype=torch.float64, device=cuda) if res_on else None
    mat = torch.full((plan.nnzb * 4,), float("nan"), dtype=torch.float64, device=cuda) if mat_on else None
    plan.assemble(d.states, d.coords, m.E, m.nu, m.t, res, mat, precision=prec, strain=strain)
    torch.cuda.synchronize()
    return (res.cpu().numpy() if res_on else None), (mat.cpu().numpy() if mat_on else None)


@pytest.mark.parametrize("name", list(MESHES))
def test_pair_layout_matches_oracle_and_colours(fem, orc, cuda, name):
    m = MESHES[name](fem)
    plan = fem.Plan(m.order, m.num_nodes, m.conn_ptr, m.conn)
    d = fem.DeviceMesh(m, cuda)
    try:
        lay, npairs, ncol = plan.layout()
        assert lay == "pairs" and npairs > 0 and ncol >= 4
        modes = [("fp64", "linear", True, True), ("fp64", "linear", True, False), ("fp64", "linear", False, True)]
        if m.order in (2, 3):
            modes.append(("fp64", "nonlinear", True, True))
        if m.order == 3:
            modes.append(("mixed", "linear", True, True))
        got = {k: _run(fem, cuda, m, plan, d, *k) for k in modes}
        again = _run(fem, cuda, m, plan, d, *modes[0])
        assert all(np.array_equal(x, y) for x, y in zip(again, got[modes[0]]))  # deterministic
        plan.set_layout("colours")
        assert plan.layout()[0] == "colours"
        ref = {k: _run(fem, cuda, m, plan, d, *k) for k in modes}
        for k in modes:
            for x, y in zip(got[k], ref[k]):
                if x is None:
                    continue
                assert not np.isnan(x).any(), k
                tol = 1e-6 if k[0] == "mixed" else 1e-14
                assert np.abs(x - y).max() <= tol * np.abs(y).max(), k
        rowp, cols = plan.pattern()
        R0, A0 = orc.assemble(m, orc.element_bsr_map(m.conn_ptr, m.conn, m.nodes_per_element, rowp, cols), cols.size)
        R, A = got[modes[0]]
        assert np.abs(R - R0).max() <= FP64_TOL * np.abs(R0).max()
        assert np.abs(A - A0).max() <= FP64_TOL * np.abs(A0).max()
        plan.set_layout("pairs")
        assert plan.layout()[0] == "pairs"
    finally:
        plan.close()


def test_layout_errors(fem, cuda):
    m = fem.square_mesh(4, 4, 1)
    plan = fem.Plan(m.order, m.num_nodes, m.conn_ptr, m.conn)
    try:
        assert plan.layout() == ("colours", 0, 0)
        with pytest.raises(fem.FemError) as ei:
            plan.set_layout("pairs")
        assert ei.value.status == fem.FEM_ERR_UNSUPPORTED
        plan.set_layout("colours")
    finally:
        plan.close()


def test_chained_launches_see_the_callers_writes(fem, cuda):
    """The later colour launches of an assembly overlap the previous launch's tail
    (programmatic dependent launch); the first one follows the caller's work in
    stream order, so states a caller kernel writes just before the call are the
    states assembled -- on a stream, for several back-to-back calls."""
    import torch
    m = fem.square_mesh(24, 20, 3, 1.0, 1.0, 0.15, seed=77)
    plan = fem.Plan(m.order, m.num_nodes, m.conn_ptr, m.conn)
    d = fem.DeviceMesh(m, cuda)
    stream = torch.cuda.Stream(device=cuda)
    res = torch.empty(m.num_nodes * 2, dtype=torch.float64, device=cuda)
    mat = torch.empty(plan.nnzb * 4, dtype=torch.float64, device=cuda)
    base = d.states.clone()
    refs = []
    for k in range(3):  # reference results, one call at a time
        d.states.copy_(base * (1.0 + 0.5 * k))
        torch.cuda.synchronize()
        plan.assemble(d.states, d.coords, m.E, m.nu, m.t, res, mat)
        torch.cuda.synchronize()
        refs.append((res.clone(), mat.clone()))
    outs = []
    with torch.cuda.stream(stream):
        for k in range(3):
            d.states.copy_(base)
            d.states.mul_(1.0 + 0.5 * k)  # a kernel on the same stream right before the call
            plan.assemble(d.states, d.coords, m.E, m.nu, m.t, res, mat, stream=stream.cuda_stream)
            outs.append((res.clone(), mat.clone()))
    stream.synchronize()
    for (r, a), (r0, a0) in zip(outs, refs):
        assert torch.equal(r, r0) and torch.equal(a, a0)
    plan.close()
