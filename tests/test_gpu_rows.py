"""GPU, order-1 row assembly (plans of order-1 meshes write each block row once):
which plans take it, launch counts, and oracle parity on meshes whose rows stress
the chunking — fans whose centre rows hold 81 and 127 blocks (a long row inside a
chunk; 127 is the longest row a plan accepts), a fan of 70 elements around one
node (rejected by plan creation: more than 64 colours and a 141-block row), and a
scrambled node numbering (rows of a chunk refer to elements all over the mesh).
Tolerance 1e-12 relative, as for the other FP64 paths."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _fan(fem, k, seed=0):
    """k kite-shaped quads around the origin: (centre, r_i, m_i, r_(i+1)) in the
    tensor order (0,0), (1,0), (0,1), (1,1) = centre, r_i, r_(i+1), m_i."""
    th = 2 * np.pi * np.arange(k) / k
    ring = np.stack([np.cos(th), np.sin(th)], 1)
    mid = 1.5 * np.stack([np.cos(th + np.pi / k), np.sin(th + np.pi / k)], 1)
    coords = np.concatenate([[[0.0, 0.0]], ring, mid])
    conn = []
    for i in range(k):
        conn += [0, 1 + i, 1 + (i + 1) % k, 1 + k + i]
    rng = np.random.default_rng(seed)
    states = rng.uniform(-1e-3, 1e-3, coords.shape)
    return fem.Mesh(1, np.ascontiguousarray(coords), np.arange(k + 1, dtype=np.int32) * 4,
                    np.array(conn, dtype=np.int32), states, 70e9, 0.3, 1.0, f"fan{k}")


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _plan_vs_oracle(fem, orc, cuda, m, precision="fp64"):
    import torch
    plan = fem.Plan(m.order, m.num_nodes, m.conn_ptr, m.conn)
    rowp, cols = plan.pattern()
    mp = orc.element_bsr_map(m.conn_ptr, m.conn, m.nodes_per_element, rowp, cols)
    R0, A0 = orc.assemble(m, mp, cols.size)
    d = fem.DeviceMesh(m, cuda)
    res = torch.full((m.num_nodes * 2,), float("nan"), dtype=torch.float64, device=cuda)
    mat = torch.full((plan.nnzb * 4,), float("nan"), dtype=torch.float64, device=cuda)
    plan.assemble(d.states, d.coords, m.E, m.nu, m.t, res, mat, precision=precision)
    assert _rel(res.cpu().numpy(), R0) <= TOL
    assert _rel(mat.cpu().numpy(), A0) <= TOL
    # residual only and matrix only give the same values
    res2 = torch.full_like(res, float("nan"))
    plan.assemble(d.states, d.coords, m.E, m.nu, m.t, res2, None, precision=precision)
    mat2 = torch.full_like(mat, float("nan"))
    plan.assemble(d.states, d.coords, m.E, m.nu, m.t, None, mat2, precision=precision)
    assert torch.equal(res2, res) and torch.equal(mat2, mat)
    return plan


def test_row_assembly_selection(fem, cuda):
    m1 = fem.square_mesh(9, 7, 1, 1.0, 1.0, 0.1, seed=3)
    p1 = fem.Plan(1, m1.num_nodes, m1.conn_ptr, m1.conn)
    assert p1.row_chunks == (m1.num_nodes + 31) // 32
    assert p1.launches() == 1 and p1.launches("nonlinear") == p1.num_colours
    m2 = fem.square_mesh(5, 5, 2, 1.0, 1.0, 0.1, seed=3)
    p2 = fem.Plan(2, m2.num_nodes, m2.conn_ptr, m2.conn)
    # order 2: no row tables; one launch per colour, or one dependency-ordered launch
    assert p2.row_chunks == 0 and p2.launches() == p2.num_colours
    p2.set_schedule(-1)
    assert p2.launches() == 1
    p1.close()
    p2.close()


@pytest.mark.parametrize("k", [40, 63])
def test_fan_long_rows(fem, orc, cuda, k):
    m = _fan(fem, k, seed=k)
    plan = _plan_vs_oracle(fem, orc, cuda, m)
    assert plan.row_chunks > 0
    plan.close()


def test_fan_beyond_plan_limits(fem, cuda):
    m = _fan(fem, 70)
    with pytest.raises(fem.FemError):
        fem.Plan(m.order, m.num_nodes, m.conn_ptr, m.conn)


def test_scrambled_numbering_rows(fem, orc, cuda):
    m = fem.square_mesh(23, 17, 1, 2.0, 1.0, 0.15, seed=8)
    perm = np.random.default_rng(8).permutation(m.num_nodes)
    inv = np.argsort(perm)
    m.coords = np.ascontiguousarray(m.coords[perm])
    m.states = np.ascontiguousarray(m.states[perm])
    m.conn = inv[m.conn].astype(np.int32)
    plan = _plan_vs_oracle(fem, orc, cuda, m, precision="mixed")
    assert plan.row_chunks > 0
    plan.close()
