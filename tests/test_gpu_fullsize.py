"""GPU, full workload sizes: properties that do not need the oracle at scale.

1024x1024 order-3 square (18.9 M DOF, 236 M blocks) and the 512x2048 order-2
annulus: R = K u through the device SpMV (linear strain), exact symmetry of K
(blocks (i, j) and (j, i)^T), the plan and drop-in paths agreeing, and the mixed
path within 1e-6 relative Frobenius of FP64.  A sampled slice of elements is
checked against the oracle directly."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _full(fem, orc, cuda, m):
    import torch
    plan = fem.Plan(m.order, m.num_nodes, m.conn_ptr, m.conn)
    d = fem.DeviceMesh(m, cuda)
    res = torch.empty(m.num_nodes * 2, dtype=torch.float64, device=cuda)
    mat = torch.empty(plan.nnzb * 4, dtype=torch.float64, device=cuda)
    plan.assemble(d.states, d.coords, m.E, m.nu, m.t, res, mat)
    rowp_d, cols_d = plan.device_pattern()
    x = d.states.reshape(-1)
    y = torch.empty_like(res)
    fem.lib.fem_bsr_spmv(m.num_nodes, rowp_d, cols_d, mat.data_ptr(), x.data_ptr(), y.data_ptr(),
                         torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    # R = K u
    assert float((y - res).abs().max() / res.abs().max()) <= 1e-11
    # symmetry on sampled rows: block (r, c) equals block (c, r) transposed
    rowp, cols = plan.pattern()
    rng = np.random.default_rng(3)
    rows = rng.integers(0, m.num_nodes, size=200)
    A = mat.reshape(-1, 2, 2)
    scale = float(A.abs().max())
    for r in rows:
        for j in range(rowp[r], rowp[r + 1]):
            c = cols[j]
            jt = rowp[c] + np.searchsorted(cols[rowp[c]:rowp[c + 1]], r)
            assert float((A[j] - A[jt].T).abs().max()) <= 1e-13 * scale
    # mixed precision against FP64 at full size
    res64, mat64 = res.clone(), mat.clone()
    plan.assemble(d.states, d.coords, m.E, m.nu, m.t, res, mat, precision="mixed")
    torch.cuda.synchronize()
    assert float(torch.linalg.vector_norm(res - res64) / torch.linalg.vector_norm(res64)) <= 1e-6
    assert float(torch.linalg.vector_norm(mat - mat64) / torch.linalg.vector_norm(mat64)) <= 1e-6
    # drop-in path (reference contract) on the same mesh
    mp = torch.from_numpy(fem.build_element_bsr_map(m.conn_ptr, m.conn, m.nodes_per_element, rowp, cols)).to(cuda)
    res.zero_()
    mat.zero_()
    fem.run_jacobian_kernel(m.order, d.conn_ptr, d.conn, m.num_elements, d.states, d.coords, m.E, m.nu, m.t, mp, res,
                            mat)
    assert float((res - res64).abs().max() / res64.abs().max()) <= 1e-12
    assert float((mat - mat64).abs().max() / mat64.abs().max()) <= 1e-12
    del mp, mat, mat64
    # a slice of elements against the oracle: the first 512 elements' own contributions
    sub = fem.submesh(m, 0, 512)
    srow, scol = fem.build_bsr_pattern(sub.num_nodes, sub.conn_ptr, sub.conn)
    smap = orc.element_bsr_map(sub.conn_ptr, sub.conn, sub.nodes_per_element, srow, scol)
    R0, A0 = orc.assemble(sub, smap, scol.size)
    sd = fem.DeviceMesh(sub, cuda)
    sr = torch.zeros(sub.num_nodes * 2, dtype=torch.float64, device=cuda)
    sa = torch.zeros(scol.size * 4, dtype=torch.float64, device=cuda)
    fem.run_jacobian_kernel(sub.order, sd.conn_ptr, sd.conn, sub.num_elements, sd.states, sd.coords, sub.E, sub.nu,
                            sub.t, torch.from_numpy(smap).to(cuda), sr, sa)
    assert np.abs(sr.cpu().numpy() - R0).max() <= 1e-12 * np.abs(R0).max()
    assert np.abs(sa.cpu().numpy() - A0).max() <= 1e-12 * np.abs(A0).max()
    plan.close()


def test_square1024_p3_full_size(fem, orc, cuda):
    _full(fem, orc, cuda, fem.square1024_p3())


def test_annulus512x2048_p2_full_size(fem, orc, cuda):
    _full(fem, orc, cuda, fem.annulus512x2048_p2())
