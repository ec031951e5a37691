"""The oracle against the reference's own code (CPU).

The reference's CPU assembly (element/FEKernels.h:317-508 through its dispatchers
runResidualKernel / runJacobianKernel, :1030-1225) is compiled from the header
where it lies, with the A2D interface restated in oracle/a2d_shim/, as
oracle/_ref/libfemref.so.  Its outputs on small meshes of every order and on the
64x64 order-1 mesh are committed (tests/golden/ref_assembly.npz, made by
tests/golden/make_golden.py); the oracle must reproduce them within 1e-13
(normwise; measured ~4e-16: the oracle states the AD stack in closed form and
stores Ke untransposed), and the patterns bit for bit.  Where the reference
build is present (this checkout, after `make -C oracle ref`), the same
comparison also runs live on further meshes."""
import numpy as np
import pytest

import golden_fixtures as gf

TOL = 1e-13


@pytest.mark.parametrize("name", gf.SMALL)
def test_oracle_reproduces_reference_outputs(orc, fem, name):
    z = gf.load()
    m = gf.mesh(z, name)
    rowp, cols = orc.bsr_pattern(m.num_nodes, m.conn_ptr, m.conn)
    assert np.array_equal(rowp, z[f"{name}/rowp"]) and np.array_equal(cols, z[f"{name}/cols"])
    rowp2, cols2 = fem.build_bsr_pattern(m.num_nodes, m.conn_ptr, m.conn)
    assert np.array_equal(rowp2, rowp) and np.array_equal(cols2, cols)
    mp = orc.element_bsr_map(m.conn_ptr, m.conn, m.nodes_per_element, rowp, cols)
    R, A = orc.assemble(m, mp, cols.size)
    assert gf.rel(R, z[f"{name}/residual"]) <= TOL
    assert gf.rel(A, z[f"{name}/matrix"]) <= TOL
    Rn, _ = orc.assemble(m, jacobian=False, strain="nonlinear")
    assert gf.rel(Rn, z[f"{name}/residual_nonlinear"]) <= TOL


def test_oracle_reproduces_reference_config1(orc, fem):
    """64x64 order-1 mesh (the CPU-runnable configuration): residual, the matrix
    applied to a seeded vector, and the matrix norm."""
    z = gf.load()
    m = fem.mesh.square64_p1()
    rowp, cols = orc.bsr_pattern(m.num_nodes, m.conn_ptr, m.conn)
    mp = orc.element_bsr_map(m.conn_ptr, m.conn, m.nodes_per_element, rowp, cols)
    R, A = orc.assemble(m, mp, cols.size)
    assert gf.rel(R, z["config1/residual"]) <= TOL
    v = np.random.default_rng(0x60A).uniform(-1.0, 1.0, m.num_nodes * 2)
    assert gf.rel(orc.bsr_spmv(rowp, cols, A, v), z["config1/matvec"]) <= TOL
    assert abs(np.linalg.norm(A) / z["config1/matrix_fro"][0] - 1.0) <= TOL


@pytest.mark.skipif(not __import__("oracle").ref_available(), reason="reference build (oracle/_ref) not present")
@pytest.mark.parametrize("order", [1, 2, 3, 4])
def test_oracle_matches_reference_build_live(orc, fem, order):
    for m in (fem.square_mesh(6, 5, order, 3.0, 2.0, 0.15, seed=0x610 + order),
              fem.annulus_mesh(2, 7, order, seed=0x620 + order)):
        rowp, cols = orc.bsr_pattern(m.num_nodes, m.conn_ptr, m.conn)
        mp = orc.element_bsr_map(m.conn_ptr, m.conn, m.nodes_per_element, rowp, cols)
        R0, A0 = orc.assemble(m, mp, cols.size)
        R1, A1 = orc.ref_assemble(m, mp, cols.size)
        assert gf.rel(R1, R0) <= TOL and gf.rel(A1, A0) <= TOL
        R2, _ = orc.ref_assemble(m, jacobian=False)
        assert gf.rel(R2, R0) <= TOL
        Rn0, An0 = orc.assemble(m, mp, cols.size, strain="nonlinear")
        Rn1, An1 = orc.ref_assemble(m, mp, cols.size, strain="nonlinear")
        assert gf.rel(Rn1, Rn0) <= TOL
        # The reference's CPU Jacobian loop clears its forward seed matrix, values
        # included, before each column (FEKernels.h:467), so its NONLINEAR Jacobian
        # is the tangent at zero displacement: the LINEAR matrix.  Its GPU kernel
        # keeps the values (FEKernels.h:926-936); the oracle and the library follow
        # the GPU kernel (consistent tangent at the current state).
        assert gf.rel(An1, A0) <= TOL
        assert gf.rel(An0, A0) > 1e-6
