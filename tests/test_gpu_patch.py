"""GPU parity of the order-3 patch layout (fem_plan_create_ex with FEM_PLAN_PATCHES).

The patch kernel sums strips of neighbouring elements in shared memory and writes
row segments with bulk copies; it must give the oracle's residual and Jacobian
within 1e-12 relative (normwise, max|diff| / max|oracle|), overwrite the outputs
completely, and agree with the colour-ordered plan path to rounding.  Meshes: strips
that fill grid rows, strips that wrap to the next row, a periodic annulus, scrambled
numbering (patches of unrelated elements) and a single element."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _scramble(fem, m, seed):
    rng = np.random.default_rng(seed)
    perm = rng.permutation(m.num_nodes)
    inv = np.argsort(perm)
    conn = perm[m.conn.reshape(-1, m.nodes_per_element)][rng.permutation(m.num_elements)]
    return fem.Mesh(m.order, np.ascontiguousarray(m.coords[inv]), m.conn_ptr.copy(),
                    np.ascontiguousarray(conn.reshape(-1)).astype(np.int32), np.ascontiguousarray(m.states[inv]),
                    m.E, m.nu, m.t, m.name + "_scrambled", m.seed)


MESHES = {
    "strips_32x6": lambda f: f.square_mesh(32, 6, 3, 10.0, 2.0, 0.2, seed=51),
    "wrap_13x7": lambda f: f.square_mesh(13, 7, 3, 2.0, 1.0, 0.15, seed=52),
    "annulus_5x24": lambda f: f.annulus_mesh(5, 24, 3, seed=53),
    "scrambled_9x8": lambda f: _scramble(f, f.square_mesh(9, 8, 3, 1.0, 1.0, 0.15, seed=54), 54),
    "one_el": lambda f: f.square_mesh(1, 1, 3, seed=55),
}


@pytest.mark.parametrize("name", list(MESHES))
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_patch_plan_vs_oracle(fem, orc, cuda, name, precision):
    import torch
    m = MESHES[name](fem)
    plan = fem.Plan(3, m.num_nodes, m.conn_ptr, m.conn, patches=True)
    assert (m.num_elements + 7) // 8 <= plan.num_patches <= m.num_elements
    assert plan.launches() == plan.patch_colours
    rowp, cols = plan.pattern()
    r2, c2 = orc.bsr_pattern(m.num_nodes, m.conn_ptr, m.conn)
    assert np.array_equal(rowp, r2) and np.array_equal(cols, c2)
    mp = orc.element_bsr_map(m.conn_ptr, m.conn, 16, rowp, cols)
    R0, A0 = orc.assemble(m, mp, cols.size)
    d = fem.DeviceMesh(m, cuda)
    res = torch.full((m.num_nodes * 2,), 7.0, dtype=torch.float64, device=cuda)
    mat = torch.full((cols.size * 4,), float("nan"), dtype=torch.float64, device=cuda)
    for _ in range(2):  # complete overwrite, repeatable
        plan.assemble(d.states, d.coords, m.E, m.nu, m.t, res, mat, precision=precision)
    torch.cuda.synchronize()
    assert _rel(res.cpu().numpy(), R0) <= FP64_TOL
    assert _rel(mat.cpu().numpy(), A0) <= FP64_TOL
    # matrix only (patch kernel without the residual), residual only (colour path)
    mat.fill_(3.0)
    plan.assemble(d.states, d.coords, m.E, m.nu, m.t, None, mat, precision=precision)
    res.fill_(3.0)
    plan.assemble(d.states, d.coords, m.E, m.nu, m.t, res, None, precision=precision)
    torch.cuda.synchronize()
    assert _rel(mat.cpu().numpy(), A0) <= FP64_TOL
    assert _rel(res.cpu().numpy(), R0) <= FP64_TOL
    plan.close()


def test_patch_and_colour_paths_agree(fem, cuda):
    """Same mesh, both layouts: identical pattern, results equal to rounding, and the
    patch result is deterministic (bit-identical on a second run)."""
    import torch
    m = fem.square_mesh(64, 40, 3, 10.0, 10.0, 0.2, seed=56)
    d = fem.DeviceMesh(m, cuda)
    pp = fem.Plan(3, m.num_nodes, m.conn_ptr, m.conn, patches=True)
    pc = fem.Plan(3, m.num_nodes, m.conn_ptr, m.conn)
    assert pp.num_colours == pc.num_colours and pp.nnzb == pc.nnzb
    outs = []
    for plan in (pp, pc, pp):
        res = torch.empty(m.num_nodes * 2, dtype=torch.float64, device=cuda)
        mat = torch.empty(plan.nnzb * 4, dtype=torch.float64, device=cuda)
        plan.assemble(d.states, d.coords, m.E, m.nu, m.t, res, mat)
        outs.append((res, mat))
    torch.cuda.synchronize()
    (r0, a0), (r1, a1), (r2, a2) = outs
    assert torch.equal(r0, r2) and torch.equal(a0, a2)
    assert float((r0 - r1).abs().max() / r1.abs().max()) <= 1e-13
    assert float((a0 - a1).abs().max() / a1.abs().max()) <= 1e-13
    pp.close()
    pc.close()


def test_patch_flag_at_other_orders(fem, cuda):
    """FEM_PLAN_PATCHES is ignored at orders other than 3 (no patches, colour path)."""
    m = fem.square_mesh(6, 5, 2, seed=57)
    plan = fem.Plan(2, m.num_nodes, m.conn_ptr, m.conn, patches=True)
    assert plan.num_patches == 0 and plan.patch_colours == 0
    plan.close()
