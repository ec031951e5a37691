"""GPU: a mesh read from a BDF file (small-field GRID / CQUADn cards, element nodes
in gmsh order, the order the reference's meshes come from gmsh through
fixGmshBDF, meshes/GmshUtils.py:118-196) assembles through a plan to the same
residual and Jacobian as the mesh it was written from, and to the FP64 oracle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("p", [1, 2, 3, 4])
def test_bdf_ingest_assembles(fem, orc, cuda, tmp_path, p):
    import torch
    m = fem.square_mesh(6, 5, p, 2.0, 1.0, 0.15, seed=80 + p)
    path = str(tmp_path / f"ingest_p{p}.bdf")
    fem.write_bdf(m, path, node_order="gmsh")
    r = fem.read_bdf(path, node_order="gmsh", E=m.E, nu=m.nu, t=m.t, states=m.states)
    # the file's gmsh element order comes back in tensor order, node for node
    assert np.array_equal(r.conn, m.conn) and np.allclose(r.coords, m.coords, rtol=0, atol=1e-12)
    out = []
    for mesh in (m, r):
        plan = fem.Plan(mesh.order, mesh.num_nodes, mesh.conn_ptr, mesh.conn)
        d = fem.DeviceMesh(mesh, cuda)
        res = torch.empty(mesh.num_nodes * 2, dtype=torch.float64, device=cuda)
        mat = torch.empty(plan.nnzb * 4, dtype=torch.float64, device=cuda)
        plan.assemble(d.states, d.coords, mesh.E, mesh.nu, mesh.t, res, mat)
        torch.cuda.synchronize()
        rowp, cols = plan.pattern()
        out.append((res.cpu().numpy(), mat.cpu().numpy(), rowp, cols))
        plan.close()
    (R0, A0, rp0, c0), (R1, A1, rp1, c1) = out
    assert np.array_equal(rp0, rp1) and np.array_equal(c0, c1)
    # coordinates pass through 8-character fields: equal to the file's rounding
    scale_r, scale_a = np.abs(R0).max(), np.abs(A0).max()
    assert np.abs(R1 - R0).max() <= 1e-9 * scale_r
    assert np.abs(A1 - A0).max() <= 1e-9 * scale_a
    Ro, Ao = orc.assemble(r, orc.element_bsr_map(r.conn_ptr, r.conn, r.nodes_per_element, rp1, c1), c1.size)
    assert np.abs(R1 - Ro).max() <= 1e-12 * np.abs(Ro).max()
    assert np.abs(A1 - Ao).max() <= 1e-12 * np.abs(Ao).max()
