"""GPU: fem_run_jacobian_batched_static, the batched drop-in assembly for callers
that cannot allocate device memory (its scratch is a file-scope device array).

Called through the C ABI on meshes of all four orders (plus an empty mesh given
with NULL arrays), twice in a row, and compared with fem_run_jacobian called once
per mesh and with the FP64 CPU oracle, within the FP64 tolerance of the other
parity tests (1e-12 relative, normwise).  Collected last so that a run stopping
at the first failure has run every other test before it."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12


class DropinMesh(C.Structure):
    _fields_ = [("elementOrder", C.c_int), ("numElements", C.c_int), ("connPtr", C.c_void_p), ("conn", C.c_void_p),
                ("states", C.c_void_p), ("nodeCoords", C.c_void_p), ("E", C.c_double), ("nu", C.c_double),
                ("t", C.c_double), ("elementBCSRMap", C.c_void_p), ("residual", C.c_void_p),
                ("matEntries", C.c_void_p)]


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def test_static_batched_matches_per_mesh_calls(fem, orc, cuda):
    import torch
    lib = fem.lib
    fn = lib.fem_run_jacobian_batched_static
    fn.restype = C.c_int
    fn.argtypes = [C.c_int, C.POINTER(DropinMesh), C.c_void_p]
    meshes = [fem.square_mesh(9, 7, 1, 1.0, 1.0, 0.1, seed=31), fem.square_mesh(6, 5, 2, 2.0, 1.0, 0.2, seed=32),
              fem.annulus_mesh(3, 11, 3, seed=33), fem.square_mesh(4, 3, 4, 1.0, 1.5, 0.15, seed=34),
              fem.square_mesh(40, 30, 2, 1.0, 1.0, 0.15, seed=35), fem.square_mesh(2, 2, 1, seed=36)]
    keep, descs, refs, oracle = [], [], [], []
    for m in meshes:
        d = fem.DeviceMesh(m, cuda)
        rowp, cols = fem.build_bsr_pattern(m.num_nodes, m.conn_ptr, m.conn)
        mp = torch.from_numpy(fem.build_element_bsr_map(m.conn_ptr, m.conn, m.nodes_per_element, rowp, cols)).to(cuda)
        res = torch.zeros(m.num_nodes * 2, dtype=torch.float64, device=cuda)
        mat = torch.zeros(cols.size * 4, dtype=torch.float64, device=cuda)
        fem.run_jacobian_kernel(m.order, d.conn_ptr, d.conn, m.num_elements, d.states, d.coords, m.E, m.nu, m.t, mp,
                                res, mat)
        refs.append((res.cpu().numpy(), mat.cpu().numpy()))
        oracle.append(orc.assemble(m, fem.build_element_bsr_map(m.conn_ptr, m.conn, m.nodes_per_element, rowp, cols),
                                   cols.size))
        out_r, out_m = torch.zeros_like(res), torch.zeros_like(mat)
        keep.append((d, mp, out_r, out_m))
        descs.append(DropinMesh(m.order, m.num_elements, d.conn_ptr.data_ptr(), d.conn.data_ptr(),
                                d.states.data_ptr(), d.coords.data_ptr(), m.E, m.nu, m.t, mp.data_ptr(),
                                out_r.data_ptr(), out_m.data_ptr()))
    # an empty mesh with NULL arrays sits between the others: it must be skipped
    descs.insert(2, DropinMesh(2, 0, None, None, None, None, 70e9, 0.3, 1.0, None, None, None))
    table = (DropinMesh * len(descs))(*descs)
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):  # two calls in a row: the scratch keeps the previous call's contents
        for _, _, r, a in keep:
            r.zero_()
            a.zero_()
        st = fn(len(descs), table, stream)
        assert st == 0, lib.fem_last_error().decode()
        torch.cuda.synchronize()
        for (_, _, r, a), (R0, A0), (R1, A1) in zip(keep, refs, oracle):
            rh, ah = r.cpu().numpy(), a.cpu().numpy()
            assert _rel(rh, R0) <= FP64_TOL and _rel(ah, A0) <= FP64_TOL
            assert _rel(rh, R1) <= FP64_TOL and _rel(ah, A1) <= FP64_TOL


def test_static_batched_rejects_oversized_requests(fem, cuda):
    lib = fem.lib
    fn = lib.fem_run_jacobian_batched_static
    fn.restype = C.c_int
    fn.argtypes = [C.c_int, C.POINTER(DropinMesh), C.c_void_p]
    table = (DropinMesh * 257)()
    for d in table:
        d.elementOrder, d.numElements = 1, 0
    assert fn(257, table, None) == fem.FEM_ERR_UNSUPPORTED
    assert b"256" in lib.fem_last_error()
    table[0].elementOrder = 7
    assert fn(1, table, None) == fem.FEM_ERR_INVALID_ORDER


def test_static_batched_refuses_stream_capture(fem, cuda):
    """The mesh table is staged in host memory at call time, so a capturing stream
    is refused (a captured copy would re-read the staging at every replay)."""
    import torch
    lib = fem.lib
    fn = lib.fem_run_jacobian_batched_static
    fn.restype = C.c_int
    fn.argtypes = [C.c_int, C.POINTER(DropinMesh), C.c_void_p]
    m = fem.square_mesh(3, 3, 1, seed=37)
    d = fem.DeviceMesh(m, cuda)
    rowp, cols = fem.build_bsr_pattern(m.num_nodes, m.conn_ptr, m.conn)
    mp = torch.from_numpy(fem.build_element_bsr_map(m.conn_ptr, m.conn, m.nodes_per_element, rowp, cols)).to(cuda)
    res = torch.zeros(m.num_nodes * 2, dtype=torch.float64, device=cuda)
    mat = torch.zeros(cols.size * 4, dtype=torch.float64, device=cuda)
    table = (DropinMesh * 1)(DropinMesh(1, m.num_elements, d.conn_ptr.data_ptr(), d.conn.data_ptr(),
                                        d.states.data_ptr(), d.coords.data_ptr(), m.E, m.nu, m.t, mp.data_ptr(),
                                        res.data_ptr(), mat.data_ptr()))
    assert fn(1, table, torch.cuda.current_stream().cuda_stream) == 0  # first call: address lookup
    torch.cuda.synchronize()
    side = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=side):
        res.mul_(1.0)  # keeps the captured graph non-empty
        st = fn(1, table, side.cuda_stream)
    assert st == fem.FEM_ERR_UNSUPPORTED
    assert b"capturing" in lib.fem_last_error()
    del g
