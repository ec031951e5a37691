"""GPU parity against the reference's own outputs.

tests/golden/ref_assembly.npz holds the residual and BSR matrix that the
reference's CPU assembly (element/FEKernels.h, compiled from the header as
oracle/_ref/libfemref.so; tests/golden/make_golden.py) produced on small meshes
of orders 1 to 4, and its residual and matrix-vector fingerprint on the 64x64
order-1 mesh.  The CUDA paths (drop-in Jacobian and residual entry points, plan
assembly, NONLINEAR residual) must reproduce them within the FP64 tolerance,
1e-12 relative (normwise).  This checks the library against the reference
directly, not only through the oracle."""
import numpy as np
import pytest

import golden_fixtures as gf

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12


def _outputs(fem, cuda, m):
    import torch
    d = fem.DeviceMesh(m, cuda)
    rowp, cols = fem.build_bsr_pattern(m.num_nodes, m.conn_ptr, m.conn)
    mp = torch.from_numpy(fem.build_element_bsr_map(m.conn_ptr, m.conn, m.nodes_per_element, rowp, cols)).to(cuda)
    z = lambda n: torch.zeros(n, dtype=torch.float64, device=cuda)  # noqa: E731
    res, mat = z(m.num_nodes * 2), z(cols.size * 4)
    fem.run_jacobian_kernel(m.order, d.conn_ptr, d.conn, m.num_elements, d.states, d.coords, m.E, m.nu, m.t, mp, res,
                            mat)
    res_only = z(m.num_nodes * 2)
    fem.run_residual_kernel(m.order, d.conn_ptr, d.conn, m.num_elements, d.states, d.coords, m.E, m.nu, m.t, res_only)
    res_nl = z(m.num_nodes * 2)
    fem.run_residual_kernel(m.order, d.conn_ptr, d.conn, m.num_elements, d.states, d.coords, m.E, m.nu, m.t, res_nl,
                            strain="nonlinear")
    plan = fem.Plan(m.order, m.num_nodes, m.conn_ptr, m.conn)
    pres, pmat = torch.full_like(res, 7.0), torch.full_like(mat, 7.0)
    plan.assemble(d.states, d.coords, m.E, m.nu, m.t, pres, pmat)
    torch.cuda.synchronize()
    plan.close()
    out = {k: v.cpu().numpy() for k, v in
           dict(res=res, mat=mat, res_only=res_only, res_nl=res_nl, plan_res=pres, plan_mat=pmat).items()}
    return out, rowp, cols


@pytest.mark.parametrize("name", gf.SMALL)
def test_cuda_reproduces_reference_outputs(fem, cuda, name):
    z = gf.load()
    m = gf.mesh(z, name)
    out, rowp, cols = _outputs(fem, cuda, m)
    assert np.array_equal(rowp, z[f"{name}/rowp"]) and np.array_equal(cols, z[f"{name}/cols"])
    R, A, Rn = z[f"{name}/residual"], z[f"{name}/matrix"], z[f"{name}/residual_nonlinear"]
    for key in ("res", "res_only", "plan_res"):
        assert gf.rel(out[key], R) <= FP64_TOL, key
    for key in ("mat", "plan_mat"):
        assert gf.rel(out[key], A) <= FP64_TOL, key
    assert gf.rel(out["res_nl"], Rn) <= FP64_TOL


def test_cuda_reproduces_reference_config1(fem, orc, cuda):
    z = gf.load()
    m = fem.mesh.square64_p1()
    out, rowp, cols = _outputs(fem, cuda, m)
    v = np.random.default_rng(0x60A).uniform(-1.0, 1.0, m.num_nodes * 2)
    for rk, mk in (("res", "mat"), ("plan_res", "plan_mat")):
        assert gf.rel(out[rk], z["config1/residual"]) <= FP64_TOL
        assert gf.rel(orc.bsr_spmv(rowp, cols, out[mk], v), z["config1/matvec"]) <= FP64_TOL
        assert abs(np.linalg.norm(out[mk]) / z["config1/matrix_fro"][0] - 1.0) <= FP64_TOL
