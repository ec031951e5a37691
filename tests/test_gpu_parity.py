"""GPU parity: the CUDA path through the C ABI against the FP64 oracle.

Tolerances: plain FP64 results must match within 1e-12 relative (normwise,
max|diff| / max|oracle|, per output); the mixed-precision path (FP32 element
products, FP64 J/detJ/J^-1 and FP64 accumulate) within 1e-6 relative Frobenius.
Integer topology is compared bit for bit in tests/test_host.py.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
MIXED_TOL = 1e-6


def _dev(fem, m, cuda):
    import torch
    d = fem.DeviceMesh(m, cuda)
    rowp, cols = fem.build_bsr_pattern(m.num_nodes, m.conn_ptr, m.conn)
    mp = fem.build_element_bsr_map(m.conn_ptr, m.conn, m.nodes_per_element, rowp, cols)
    d.rowp_h, d.cols_h, d.map_h = rowp, cols, mp
    d.map = torch.from_numpy(mp).to(cuda)
    d.rowp = torch.from_numpy(rowp).to(cuda)
    d.cols = torch.from_numpy(cols).to(cuda)
    d.nnzb = int(cols.size)
    return d


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def _frob(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


MESHES = {
    "sq8_p1": lambda f: f.square_mesh(8, 8, 1, 1.0, 1.0, 0.1, seed=11),
    "sq6x5_p2": lambda f: f.square_mesh(6, 5, 2, 2.0, 1.0, 0.2, seed=12),
    "sq5x4_p3": lambda f: f.square_mesh(5, 4, 3, 10.0, 10.0, 0.2, seed=13),
    "sq3x4_p4": lambda f: f.square_mesh(3, 4, 4, 1.0, 1.5, 0.15, seed=14),
    "sq37x23_p2": lambda f: f.square_mesh(37, 23, 2, 1.0, 1.0, 0.15, seed=15),
    "sq41x9_p4": lambda f: f.square_mesh(41, 9, 4, 4.0, 1.0, 0.15, seed=16),
    "ann8x32_p2": lambda f: f.annulus_mesh(8, 32, 2, seed=17),
    "ann5x17_p3": lambda f: f.annulus_mesh(5, 17, 3, seed=18),
    "one_p1": lambda f: f.square_mesh(1, 1, 1, seed=19),
    "one_p4": lambda f: f.square_mesh(1, 1, 4, seed=20),
}


@pytest.mark.parametrize("name", list(MESHES))
def test_dropin_jacobian_and_residual_fp64(fem, orc, cuda, name):
    import torch
    m = MESHES[name](fem)
    d = _dev(fem, m, cuda)
    R0, A0 = orc.assemble(m, d.map_h, d.nnzb)
    res = torch.zeros(m.num_nodes * 2, dtype=torch.float64, device=cuda)
    mat = torch.zeros(d.nnzb * 4, dtype=torch.float64, device=cuda)
    secs = fem.run_jacobian_kernel(m.order, d.conn_ptr, d.conn, m.num_elements, d.states, d.coords, m.E, m.nu, m.t,
                                   d.map, res, mat)
    assert secs > 0
    assert _rel(res.cpu().numpy(), R0) <= FP64_TOL
    assert _rel(mat.cpu().numpy(), A0) <= FP64_TOL
    # residual-only kernel (runResidualKernel)
    res2 = torch.zeros_like(res)
    fem.run_residual_kernel(m.order, d.conn_ptr, d.conn, m.num_elements, d.states, d.coords, m.E, m.nu, m.t, res2)
    assert _rel(res2.cpu().numpy(), R0) <= FP64_TOL
    # Jacobian without residual (residual == nullptr, FEKernels.h:996)
    mat2 = torch.zeros_like(mat)
    fem.run_jacobian_kernel(m.order, d.conn_ptr, d.conn, m.num_elements, d.states, d.coords, m.E, m.nu, m.t, d.map,
                            None, mat2)
    assert _rel(mat2.cpu().numpy(), A0) <= FP64_TOL


def test_dropin_accumulates_into_outputs(fem, orc, cuda):
    """Accumulate-into contract: a second call adds the same values again."""
    import torch
    m = MESHES["sq6x5_p2"](fem)
    d = _dev(fem, m, cuda)
    R0, A0 = orc.assemble(m, d.map_h, d.nnzb)
    res = torch.full((m.num_nodes * 2,), 0.5, dtype=torch.float64, device=cuda)
    mat = torch.full((d.nnzb * 4,), -1.0, dtype=torch.float64, device=cuda)
    for _ in range(2):
        fem.run_jacobian_kernel(m.order, d.conn_ptr, d.conn, m.num_elements, d.states, d.coords, m.E, m.nu, m.t,
                                d.map, res, mat, timed=False)
    assert _rel(res.cpu().numpy() - 0.5, 2 * R0) <= FP64_TOL
    assert _rel(mat.cpu().numpy() + 1.0, 2 * A0) <= 4 * FP64_TOL


@pytest.mark.parametrize("name,precision", [("sq6x5_p2", "fp64"), ("sq5x4_p3", "fp64"), ("sq3x4_p4", "fp64"),
                                            ("sq5x4_p3", "mixed"), ("ann5x17_p3", "mixed")])
def test_dropin_unaligned_matrix_and_map(fem, orc, cuda, name, precision):
    """The drop-in contract asks only 8-byte alignment of matEntries and 4-byte of
    the element map: a matrix one double and a map one int past a 16-byte boundary
    take the atomic and 4-byte staging paths and give the same result (MIXED at
    order 3: the BF16x6 stiffness through the same write paths)."""
    import torch
    m = MESHES[name](fem)
    d = _dev(fem, m, cuda)
    R0, A0 = orc.assemble(m, d.map_h, d.nnzb)
    res = torch.zeros(m.num_nodes * 2, dtype=torch.float64, device=cuda)
    mat_buf = torch.zeros(d.nnzb * 4 + 1, dtype=torch.float64, device=cuda)
    map_buf = torch.zeros(d.map.numel() + 1, dtype=torch.int32, device=cuda)
    map_buf[1:] = d.map
    mat, dmap = mat_buf[1:], map_buf[1:]
    assert mat.data_ptr() % 16 == 8 and dmap.data_ptr() % 16 == 4
    fem.run_jacobian_kernel(m.order, d.conn_ptr, d.conn, m.num_elements, d.states, d.coords, m.E, m.nu, m.t, dmap,
                            res, mat, precision=precision)
    assert _rel(res.cpu().numpy(), R0) <= FP64_TOL
    if precision == "fp64":
        assert _rel(mat.cpu().numpy(), A0) <= FP64_TOL
    else:
        assert _frob(mat.cpu().numpy(), A0) <= MIXED_TOL


@pytest.mark.parametrize("name", ["sq8_p1", "sq6x5_p2", "sq5x4_p3", "sq3x4_p4", "ann8x32_p2", "sq41x9_p4"])
def test_mixed_precision_error(fem, orc, cuda, name):
    import torch
    m = MESHES[name](fem)
    d = _dev(fem, m, cuda)
    R0, A0 = orc.assemble(m, d.map_h, d.nnzb)
    res = torch.zeros(m.num_nodes * 2, dtype=torch.float64, device=cuda)
    mat = torch.zeros(d.nnzb * 4, dtype=torch.float64, device=cuda)
    fem.run_jacobian_kernel(m.order, d.conn_ptr, d.conn, m.num_elements, d.states, d.coords, m.E, m.nu, m.t, d.map,
                            res, mat, precision="mixed")
    assert _frob(res.cpu().numpy(), R0) <= MIXED_TOL
    assert _frob(mat.cpu().numpy(), A0) <= MIXED_TOL


@pytest.mark.parametrize("name,reduced", [("sq5x4_p3", True), ("ann5x17_p3", True), ("sq37x23_p2", False)])
def test_mixed_order3_runs_reduced_precision(fem, orc, cuda, name, reduced):
    """MIXED at order 3 runs its element stiffness as BF16x6 tensor-core products:
    the Jacobian differs from the FP64 oracle by FP32-level rounding (well inside
    1e-6, well above FP64 rounding) while the residual stays FP64; order 2 runs the
    FP64 kernel and matches at 1e-12."""
    import torch
    m = MESHES[name](fem)
    d = _dev(fem, m, cuda)
    R0, A0 = orc.assemble(m, d.map_h, d.nnzb)
    plan = fem.Plan(m.order, m.num_nodes, m.conn_ptr, m.conn)
    res = torch.empty(m.num_nodes * 2, dtype=torch.float64, device=cuda)
    mat = torch.empty(d.nnzb * 4, dtype=torch.float64, device=cuda)
    plan.assemble(d.states, d.coords, m.E, m.nu, m.t, res, mat, precision="mixed")
    torch.cuda.synchronize()
    err = _frob(mat.cpu().numpy(), A0)
    assert _rel(res.cpu().numpy(), R0) <= FP64_TOL
    if reduced:
        assert 1e-10 < err <= 1e-6, err
    else:
        assert _rel(mat.cpu().numpy(), A0) <= FP64_TOL
    plan.close()


@pytest.mark.parametrize("name", ["sq8_p1", "sq37x23_p2", "sq5x4_p3", "sq41x9_p4", "ann5x17_p3", "one_p4"])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_plan_overwrites_complete_result(fem, orc, cuda, name, precision):
    """Plan path: output is fully written (no zeroing needed), pattern bit-exact."""
    import torch
    m = MESHES[name](fem)
    plan = fem.Plan(m.order, m.num_nodes, m.conn_ptr, m.conn)
    rowp, cols = plan.pattern()
    r2, c2 = orc.bsr_pattern(m.num_nodes, m.conn_ptr, m.conn)
    assert np.array_equal(rowp, r2) and np.array_equal(cols, c2)
    mp = orc.element_bsr_map(m.conn_ptr, m.conn, m.nodes_per_element, rowp, cols)
    R0, A0 = orc.assemble(m, mp, cols.size)
    d = fem.DeviceMesh(m, cuda)
    res = torch.full((m.num_nodes * 2,), 7.0, dtype=torch.float64, device=cuda)
    mat = torch.full((cols.size * 4,), float("nan"), dtype=torch.float64, device=cuda)
    for _ in range(2):
        plan.assemble(d.states, d.coords, m.E, m.nu, m.t, res, mat, precision=precision)
    tol, err = (FP64_TOL, _rel) if precision == "fp64" else (MIXED_TOL, _frob)
    assert err(res.cpu().numpy(), R0) <= tol
    assert err(mat.cpu().numpy(), A0) <= tol
    # residual only / matrix only
    res.fill_(3.0)
    plan.assemble(d.states, d.coords, m.E, m.nu, m.t, res, None, precision=precision)
    assert err(res.cpu().numpy(), R0) <= tol
    mat.fill_(3.0)
    plan.assemble(d.states, d.coords, m.E, m.nu, m.t, None, mat, precision=precision)
    assert err(mat.cpu().numpy(), A0) <= tol
    plan.close()


def test_config1_square64_p1_exact(fem, orc, cuda):
    """64x64 order-1 unit square (+-0.1h, u in [-1e-3,1e-3], E=70e9, nu=0.3)."""
    import torch
    m = fem.square64_p1()
    d = _dev(fem, m, cuda)
    assert d.nnzb == 37249
    R0, A0 = orc.assemble(m, d.map_h, d.nnzb)
    res = torch.zeros(m.num_nodes * 2, dtype=torch.float64, device=cuda)
    mat = torch.zeros(d.nnzb * 4, dtype=torch.float64, device=cuda)
    fem.run_jacobian_kernel(1, d.conn_ptr, d.conn, m.num_elements, d.states, d.coords, m.E, m.nu, m.t, d.map, res, mat)
    assert _rel(res.cpu().numpy(), R0) <= FP64_TOL
    assert _rel(mat.cpu().numpy(), A0) <= FP64_TOL


def test_spmv_and_R_equals_Ku(fem, orc, cuda):
    import torch
    m = MESHES["sq37x23_p2"](fem)
    d = _dev(fem, m, cuda)
    res = torch.zeros(m.num_nodes * 2, dtype=torch.float64, device=cuda)
    mat = torch.zeros(d.nnzb * 4, dtype=torch.float64, device=cuda)
    fem.run_jacobian_kernel(m.order, d.conn_ptr, d.conn, m.num_elements, d.states, d.coords, m.E, m.nu, m.t, d.map,
                            res, mat)
    y = torch.zeros_like(res)
    fem.bsr_spmv(d.rowp, d.cols, mat, d.states.reshape(-1), y)
    y_ref = orc.bsr_spmv(d.rowp_h, d.cols_h, mat.cpu().numpy(), m.states.reshape(-1))
    assert _rel(y.cpu().numpy(), y_ref) <= 1e-13
    assert _rel(y.cpu().numpy(), res.cpu().numpy()) <= 1e-11


def test_error_statuses(fem, cuda):
    import torch
    m = MESHES["sq8_p1"](fem)
    d = _dev(fem, m, cuda)
    res = torch.zeros(m.num_nodes * 2, dtype=torch.float64, device=cuda)
    mat = torch.zeros(d.nnzb * 4, dtype=torch.float64, device=cuda)
    args = (d.conn_ptr, d.conn, m.num_elements, d.states, d.coords, m.E, m.nu, m.t)
    with pytest.raises(fem.FemError) as ei:
        fem.run_residual_kernel(5, *args, res)
    assert ei.value.status == fem.FEM_ERR_INVALID_ORDER
    with pytest.raises(fem.FemError) as ei:
        fem.run_jacobian_kernel(0, *args, d.map, res, mat)
    assert ei.value.status == fem.FEM_ERR_INVALID_ORDER
    with pytest.raises(fem.FemError) as ei:
        fem.run_residual_kernel(1, d.conn_ptr, d.conn, m.num_elements, d.states.data_ptr() + 8, d.coords, m.E, m.nu,
                                m.t, res)
    assert ei.value.status == fem.FEM_ERR_MISALIGNED
    with pytest.raises(fem.FemError) as ei:
        fem.run_jacobian_kernel(1, *args, None, res, mat)
    assert ei.value.status == fem.FEM_ERR_INVALID_ARGUMENT
    # zero elements: no work, success
    assert fem.run_jacobian_kernel(1, d.conn_ptr, d.conn, 0, d.states, d.coords, m.E, m.nu, m.t, d.map, res,
                                   mat) == 0.0
    assert float(res.abs().max()) == 0.0 and float(mat.abs().max()) == 0.0


def _scramble(fem, m, seed):
    """Same mesh with node ids and element order permuted (unstructured numbering)."""
    rng = np.random.default_rng(seed)
    perm = rng.permutation(m.num_nodes)          # new id of old node
    inv = np.argsort(perm)
    n = m.nodes_per_element
    conn = perm[m.conn.reshape(-1, n)]
    order = rng.permutation(m.num_elements)
    conn = np.ascontiguousarray(conn[order].reshape(-1)).astype(np.int32)
    return fem.Mesh(m.order, np.ascontiguousarray(m.coords[inv]), m.conn_ptr.copy(), conn,
                    np.ascontiguousarray(m.states[inv]), m.E, m.nu, m.t, m.name + "_scrambled", m.seed)


@pytest.mark.parametrize("p", [1, 2, 3, 4])
def test_scrambled_numbering(fem, orc, cuda, p):
    """Unstructured node numbering and element order: more colours, scattered rows."""
    import torch
    m = _scramble(fem, fem.square_mesh(9, 7, p, 1.0, 1.0, 0.15, seed=40 + p), seed=p)
    d = _dev(fem, m, cuda)
    R0, A0 = orc.assemble(m, d.map_h, d.nnzb)
    res = torch.zeros(m.num_nodes * 2, dtype=torch.float64, device=cuda)
    mat = torch.zeros(d.nnzb * 4, dtype=torch.float64, device=cuda)
    fem.run_jacobian_kernel(m.order, d.conn_ptr, d.conn, m.num_elements, d.states, d.coords, m.E, m.nu, m.t, d.map,
                            res, mat)
    assert _rel(res.cpu().numpy(), R0) <= FP64_TOL
    assert _rel(mat.cpu().numpy(), A0) <= FP64_TOL
    plan = fem.Plan(m.order, m.num_nodes, m.conn_ptr, m.conn)
    assert plan.num_colours >= 4
    res.fill_(9.0)
    mat.fill_(9.0)
    plan.assemble(d.states, d.coords, m.E, m.nu, m.t, res, mat)
    torch.cuda.synchronize()
    assert _rel(res.cpu().numpy(), R0) <= FP64_TOL
    assert _rel(mat.cpu().numpy(), A0) <= FP64_TOL
    plan.close()


def test_connptr_offsets_are_honoured(fem, orc, cuda):
    """The drop-in path reads conn[connPtr[e] + a]: a conn array with unused gaps
    between elements gives the same result."""
    import torch
    m = fem.square_mesh(5, 4, 2, seed=51)
    d = _dev(fem, m, cuda)
    R0, A0 = orc.assemble(m, d.map_h, d.nnzb)
    n = m.nodes_per_element
    gap = 3
    conn_g = np.full(m.num_elements * (n + gap), -1, np.int32)
    ptr_g = (np.arange(m.num_elements + 1) * (n + gap)).astype(np.int32)
    for e in range(m.num_elements):
        conn_g[ptr_g[e]:ptr_g[e] + n] = m.conn[e * n:(e + 1) * n]
    res = torch.zeros(m.num_nodes * 2, dtype=torch.float64, device=cuda)
    mat = torch.zeros(d.nnzb * 4, dtype=torch.float64, device=cuda)
    fem.run_jacobian_kernel(m.order, torch.from_numpy(ptr_g).to(cuda), torch.from_numpy(conn_g).to(cuda),
                            m.num_elements, d.states, d.coords, m.E, m.nu, m.t, d.map, res, mat)
    assert _rel(res.cpu().numpy(), R0) <= FP64_TOL
    assert _rel(mat.cpu().numpy(), A0) <= FP64_TOL
