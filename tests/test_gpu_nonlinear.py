"""GPU parity of the GreenStrainType::NONLINEAR kernels (FEM_STRAIN_NONLINEAR,
the reference kernels' strainType template option, element/FEKernels.h:286,317,
379,589,786) through the C ABI against the FP64 oracle, plus size-independent
properties: a finite rigid rotation is stress free (R = 0) and its rotation
increment lies in the null space of K.

Tolerance: 1e-12 relative (max|diff| / max|oracle|) per output, as for the
linear FP64 path.  States are scaled to displacement gradients of a few percent
so the Green-strain terms are a visible fraction of the result."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12

MESHES = {
    "sq8_p1": lambda f: f.square_mesh(8, 8, 1, 1.0, 1.0, 0.1, seed=31),
    "sq6x5_p2": lambda f: f.square_mesh(6, 5, 2, 2.0, 1.0, 0.2, seed=32),
    "sq5x4_p3": lambda f: f.square_mesh(5, 4, 3, 10.0, 10.0, 0.2, seed=33),
    "sq3x4_p4": lambda f: f.square_mesh(3, 4, 4, 1.0, 1.5, 0.15, seed=34),
    "sq37x23_p2": lambda f: f.square_mesh(37, 23, 2, 1.0, 1.0, 0.15, seed=35),
    "ann5x17_p3": lambda f: f.annulus_mesh(5, 17, 3, seed=36),
    "one_p1": lambda f: f.square_mesh(1, 1, 1, seed=37),
    "one_p4": lambda f: f.square_mesh(1, 1, 4, seed=38),
}


def _large_states(m, amp=0.05, seed=0):
    """Smooth field plus noise with displacement gradients of about `amp`."""
    rng = np.random.default_rng(seed)
    X = m.coords
    L = max(np.ptp(X[:, 0]), np.ptp(X[:, 1]), 1e-30)
    u = amp * L * np.stack([np.sin(2.1 * X[:, 1] / L) + 0.3 * X[:, 0] / L, np.cos(1.7 * X[:, 0] / L)], 1)
    u += rng.uniform(-0.05, 0.05, u.shape) * amp * L / 10
    m.states = np.ascontiguousarray(u)
    return m


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _setup(fem, m, cuda):
    import torch
    d = fem.DeviceMesh(m, cuda)
    rowp, cols = fem.build_bsr_pattern(m.num_nodes, m.conn_ptr, m.conn)
    mp = fem.build_element_bsr_map(m.conn_ptr, m.conn, m.nodes_per_element, rowp, cols)
    return d, rowp, cols, mp, torch.from_numpy(mp).to(cuda)


@pytest.mark.parametrize("name", list(MESHES))
def test_dropin_nonlinear_fp64(fem, orc, cuda, name):
    import torch
    m = _large_states(MESHES[name](fem), seed=len(name))
    d, rowp, cols, mp, dmap = _setup(fem, m, cuda)
    R0, A0 = orc.assemble(m, mp, cols.size, strain="nonlinear")
    Rl, _ = orc.assemble(m, mp, cols.size)
    assert _rel(Rl, R0) > 1e-4  # the nonlinear terms matter at this amplitude
    res = torch.zeros(m.num_nodes * 2, dtype=torch.float64, device=cuda)
    mat = torch.zeros(cols.size * 4, dtype=torch.float64, device=cuda)
    fem.run_jacobian_kernel(m.order, d.conn_ptr, d.conn, m.num_elements, d.states, d.coords, m.E, m.nu, m.t, dmap,
                            res, mat, strain="nonlinear")
    assert _rel(res.cpu().numpy(), R0) <= TOL
    assert _rel(mat.cpu().numpy(), A0) <= TOL
    res2 = torch.zeros_like(res)
    fem.run_residual_kernel(m.order, d.conn_ptr, d.conn, m.num_elements, d.states, d.coords, m.E, m.nu, m.t, res2,
                            strain="nonlinear")
    assert _rel(res2.cpu().numpy(), R0) <= TOL
    mat2 = torch.zeros_like(mat)
    fem.run_jacobian_kernel(m.order, d.conn_ptr, d.conn, m.num_elements, d.states, d.coords, m.E, m.nu, m.t, dmap,
                            None, mat2, strain="nonlinear")
    assert _rel(mat2.cpu().numpy(), A0) <= TOL


@pytest.mark.parametrize("name", list(MESHES))
def test_plan_nonlinear_fp64(fem, orc, cuda, name):
    import torch
    m = _large_states(MESHES[name](fem), seed=3 + len(name))
    plan = fem.Plan(m.order, m.num_nodes, m.conn_ptr, m.conn)
    rowp, cols = plan.pattern()
    mp = orc.element_bsr_map(m.conn_ptr, m.conn, m.nodes_per_element, rowp, cols)
    R0, A0 = orc.assemble(m, mp, cols.size, strain="nonlinear")
    d = fem.DeviceMesh(m, cuda)
    res = torch.full((m.num_nodes * 2,), float("nan"), dtype=torch.float64, device=cuda)
    mat = torch.full((plan.nnzb * 4,), float("nan"), dtype=torch.float64, device=cuda)
    plan.assemble(d.states, d.coords, m.E, m.nu, m.t, res, mat, strain="nonlinear")
    assert _rel(res.cpu().numpy(), R0) <= TOL
    assert _rel(mat.cpu().numpy(), A0) <= TOL
    res2 = torch.full_like(res, float("nan"))
    plan.assemble(d.states, d.coords, m.E, m.nu, m.t, res2, None, strain="nonlinear")
    assert _rel(res2.cpu().numpy(), R0) <= TOL
    mat2 = torch.full_like(mat, float("nan"))
    plan.assemble(d.states, d.coords, m.E, m.nu, m.t, None, mat2, strain="nonlinear")
    assert torch.equal(mat2, mat)
    plan.close()


def test_nonlinear_rejects_mixed_and_unknown_strain(fem, cuda):
    import torch
    m = MESHES["sq8_p1"](fem)
    d, rowp, cols, mp, dmap = _setup(fem, m, cuda)
    res = torch.zeros(m.num_nodes * 2, dtype=torch.float64, device=cuda)
    mat = torch.zeros(cols.size * 4, dtype=torch.float64, device=cuda)
    with pytest.raises(fem.FemError, match="FP64"):
        fem.run_jacobian_kernel(m.order, d.conn_ptr, d.conn, m.num_elements, d.states, d.coords, m.E, m.nu, m.t, dmap,
                                res, mat, strain="nonlinear", precision="mixed")
    with pytest.raises(fem.FemError, match="strain type"):
        fem.run_residual_kernel(m.order, d.conn_ptr, d.conn, m.num_elements, d.states, d.coords, m.E, m.nu, m.t, res,
                                strain=7)
    plan = fem.Plan(m.order, m.num_nodes, m.conn_ptr, m.conn)
    with pytest.raises(fem.FemError, match="FP64"):
        plan.assemble(d.states, d.coords, m.E, m.nu, m.t, res, None, strain="nonlinear", precision="mixed")
    plan.close()


@pytest.mark.parametrize("order,n", [(1, 256), (2, 96), (3, 64), (4, 40)])
def test_finite_rotation_properties(fem, cuda, order, n):
    """u = (Q - I) x for a 0.3 rad rotation on a distorted mesh: the nonlinear
    residual vanishes to rounding, K is exactly symmetric, and K W (x + u) = 0."""
    import torch
    m = fem.square_mesh(n, n, order, 1.0, 1.0, 0.15, seed=40 + order)
    th = 0.3
    Q = np.array([[np.cos(th), -np.sin(th)], [np.sin(th), np.cos(th)]])
    m.states = np.ascontiguousarray(m.coords @ Q.T - m.coords)
    plan = fem.Plan(m.order, m.num_nodes, m.conn_ptr, m.conn)
    d = fem.DeviceMesh(m, cuda)
    res = torch.empty(m.num_nodes * 2, dtype=torch.float64, device=cuda)
    mat = torch.empty(plan.nnzb * 4, dtype=torch.float64, device=cuda)
    plan.assemble(d.states, d.coords, m.E, m.nu, m.t, res, mat, strain="nonlinear")
    rowp_d, cols_d = plan.device_pattern()
    # scale: |K| |u|
    x = d.states.reshape(-1)
    Kscale = float(mat.abs().max()) * float(x.abs().max())
    assert float(res.abs().max()) <= 1e-11 * Kscale
    W = np.array([[0.0, -1.0], [1.0, 0.0]])
    inc = torch.from_numpy(np.ascontiguousarray(((m.coords + m.states) @ W.T).reshape(-1))).to(cuda)
    y = torch.empty_like(inc)
    fem.lib.fem_bsr_spmv(m.num_nodes, rowp_d, cols_d, mat.data_ptr(), inc.data_ptr(), y.data_ptr(),
                         torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert float(y.abs().max()) <= 1e-11 * float(mat.abs().max()) * float(inc.abs().max())
    rowp, cols = plan.pattern()
    A = mat.reshape(-1, 2, 2).cpu().numpy()
    rng = np.random.default_rng(order)
    amax = np.abs(A).max()
    for r in rng.integers(0, m.num_nodes, size=100):
        for j in range(rowp[r], rowp[r + 1]):
            c = cols[j]
            jt = rowp[c] + np.searchsorted(cols[rowp[c]:rowp[c + 1]], r)
            if c != r:  # off-diagonal pairs are written as one block and its transpose
                assert np.array_equal(A[j], A[jt].T)
            else:
                assert abs(A[j][0, 1] - A[j][1, 0]) <= 1e-13 * amax
    plan.close()
