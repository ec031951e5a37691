"""CPU checks of the FP64 oracle: pinned against tables computed by the
reference's own headers, plus known-answer physics tests (the reference ships
no fixtures and its A2D/TACS dependencies are absent)."""
import pathlib

import numpy as np
import pytest

GOLDEN = pathlib.Path(__file__).resolve().parent / "golden" / "ref_tables.txt"


def _golden():
    g = {"gauss": {}, "dN": {}, "N1d": {}}
    for line in GOLDEN.read_text().splitlines():
        f = line.split()
        if f[0] == "gauss":
            g["gauss"][(int(f[1]), int(f[2]))] = (float.fromhex(f[3]), float.fromhex(f[4]))
        elif f[0] == "dN":
            g["dN"][(int(f[1]), int(f[2]), int(f[3]))] = (float.fromhex(f[4]), float.fromhex(f[5]))
        else:
            g["N1d"][(int(f[1]), int(f[2]), int(f[3]))] = tuple(float.fromhex(v) for v in f[4:7])
    return g


@pytest.mark.parametrize("p", [1, 2, 3, 4])
def test_tables_bit_exact_vs_reference_headers(orc, p):
    """Gauss points/weights and the 2D derivative table equal, bit for bit, what
    element/GaussQuadrature.h and element/LagrangeShapeFuncs.h compute."""
    g = _golden()
    xi, w, dN = orc.tables(p)
    for i in range(p + 1):
        assert (xi[i], w[i]) == g["gauss"][(p, i)]
    n = (p + 1) ** 2
    for q in range(n):
        for a in range(n):
            assert tuple(dN[q, a]) == g["dN"][(p, q, a)], (p, q, a)
    pts = sorted({k[1] for k in g["N1d"] if k[0] == p})
    for i in pts:
        x = g["N1d"][(p, i, 0)][0]
        N, dNx = orc.lagrange1d(p, [x])
        for k in range(p + 1):
            assert (N[0, k], dNx[0, k]) == g["N1d"][(p, i, k)][1:]


@pytest.mark.parametrize("p", [1, 2, 3, 4])
def test_partition_of_unity(orc, p):
    x = np.linspace(-1, 1, 17)
    N, dN = orc.lagrange1d(p, x)
    assert np.allclose(N.sum(1), 1.0, atol=1e-13)
    assert np.allclose(dN.sum(1), 0.0, atol=1e-12)
    _, _, d2 = orc.tables(p)
    assert np.allclose(d2.sum(1), 0.0, atol=1e-12)


def test_q4_unit_square_matches_closed_form(orc):
    """Undistorted unit-square Q4: the exact integral of B^T D B (sympy)."""
    sp = pytest.importorskip("sympy")
    x, y = sp.symbols("x y")
    E, nu = 70e9, 0.3
    N = [(1 - x) * (1 - y), x * (1 - y), (1 - x) * y, x * y]
    B = sp.zeros(3, 8)
    for a, Na in enumerate(N):
        B[0, 2 * a] = sp.diff(Na, x)
        B[1, 2 * a + 1] = sp.diff(Na, y)
        B[2, 2 * a] = sp.diff(Na, y)
        B[2, 2 * a + 1] = sp.diff(Na, x)
    D = sp.Rational(1) * E / (1 - nu ** 2) * sp.Matrix([[1, nu, 0], [nu, 1, 0], [0, 0, (1 - nu) / 2]])
    K = np.array(sp.integrate(sp.integrate(B.T * D * B, (x, 0, 1)), (y, 0, 1)).evalf(), dtype=float)
    X = np.array([[0, 0], [1, 0], [0, 1], [1, 1]], float)
    _, Ke = orc.element(1, X, np.zeros((4, 2)), E, nu, 1.0)
    assert np.abs(Ke - K).max() <= 1e-13 * np.abs(K).max()


def _distorted_element(fem, p, seed=7):
    m = fem.square_mesh(1, 1, p, 1.0, 1.0, 0.0, seed=seed)
    rng = np.random.default_rng(seed)
    X = m.coords + rng.uniform(-0.05, 0.05, m.coords.shape) / p
    return X


@pytest.mark.parametrize("p", [1, 2, 3, 4])
def test_element_properties(fem, orc, p):
    """Symmetry, rigid-body null space, R = K u (linear strain) and finite differences."""
    X = _distorted_element(fem, p)
    n = (p + 1) ** 2
    rng = np.random.default_rng(p)
    U = rng.uniform(-1e-3, 1e-3, (n, 2))
    E, nu, t = 70e9, 0.3, 0.5
    Re, Ke = orc.element(p, X, U, E, nu, t)
    scale = np.abs(Ke).max()
    assert np.abs(Ke - Ke.T).max() <= 1e-13 * scale
    rot = np.stack([-X[:, 1], X[:, 0]], 1).reshape(-1)
    for r in (np.tile([1.0, 0.0], n), np.tile([0.0, 1.0], n), rot):
        assert np.abs(Ke @ r).max() <= 1e-12 * scale * np.abs(r).max()
        Rr, _ = orc.element(p, X, r.reshape(n, 2), E, nu, t)
        assert np.abs(Rr).max() <= 1e-12 * scale * np.abs(r).max()
    assert np.abs(Ke @ U.reshape(-1) - Re).max() <= 1e-12 * np.abs(Re).max()
    h = 1e-7
    for c in (0, 3, 2 * n - 1):
        Up, Um = U.copy().reshape(-1), U.copy().reshape(-1)
        Up[c] += h
        Um[c] -= h
        Rp, _ = orc.element(p, X, Up.reshape(n, 2), E, nu, t)
        Rm, _ = orc.element(p, X, Um.reshape(n, 2), E, nu, t)
        fd = (Rp - Rm) / (2 * h)
        assert np.abs(fd - Ke[:, c]).max() <= 1e-6 * scale


@pytest.mark.parametrize("p", [1, 2, 3, 4])
def test_patch_test_uniform_strain(fem, orc, p):
    """u = A x (uniform strain) on a distorted mesh: interior-node residual is 0
    (p+1 Gauss points integrate grad(N)*adj(J), of degree 2p, exactly)."""
    m = fem.square_mesh(4, 3, p, 2.0, 1.5, 0.2, seed=11)
    A = np.array([[1e-3, 4e-4], [-2e-4, 7e-4]])
    m.states = m.coords @ A.T
    rowp, cols = fem.build_bsr_pattern(m.num_nodes, m.conn_ptr, m.conn)
    R, _ = orc.assemble(m, jacobian=False)
    X = m.coords
    boundary = (np.isclose(X[:, 0], 0) | np.isclose(X[:, 0], 2.0) | np.isclose(X[:, 1], 0) | np.isclose(X[:, 1], 1.5))
    Rn = R.reshape(-1, 2)
    assert np.abs(Rn[~boundary]).max() <= 1e-9 * np.abs(Rn[boundary]).max()


@pytest.mark.parametrize("p", [1, 2, 3, 4])
def test_global_R_equals_K_u(fem, orc, p):
    m = fem.square_mesh(5, 4, p, 1.3, 1.1, 0.2, seed=3)
    rowp, cols = fem.build_bsr_pattern(m.num_nodes, m.conn_ptr, m.conn)
    mp = fem.build_element_bsr_map(m.conn_ptr, m.conn, (p + 1) ** 2, rowp, cols)
    R, A = orc.assemble(m, mp, cols.size)
    Ku = orc.bsr_spmv(rowp, cols, A, m.states.reshape(-1))
    assert np.abs(Ku - R).max() <= 1e-12 * np.abs(R).max()


def test_reference_analytic_field_fixture(fem, orc):
    """The reference driver's analytic displacement field (verification/TACSHelpers.h:192-196)
    on an annulus: R = K u and a symmetric K."""
    m = fem.annulus_mesh(3, 12, 2, seed=1)
    x, y = m.coords[:, 0], m.coords[:, 1]
    m.states = 1e-2 * np.stack([np.sin(2 * np.pi * x) + np.sin(2 * np.pi * y),
                                np.cos(2 * np.pi * x) + np.cos(2 * np.pi * y)], 1)
    rowp, cols = fem.build_bsr_pattern(m.num_nodes, m.conn_ptr, m.conn)
    mp = fem.build_element_bsr_map(m.conn_ptr, m.conn, 9, rowp, cols)
    R, A = orc.assemble(m, mp, cols.size)
    Ku = orc.bsr_spmv(rowp, cols, A, m.states.reshape(-1))
    assert np.abs(Ku - R).max() <= 1e-12 * np.abs(R).max()
    dense = np.zeros((m.num_dof, m.num_dof))
    for r in range(m.num_nodes):
        for j in range(rowp[r], rowp[r + 1]):
            dense[2 * r:2 * r + 2, 2 * cols[j]:2 * cols[j] + 2] = A[4 * j:4 * j + 4].reshape(2, 2)
    assert np.abs(dense - dense.T).max() <= 1e-12 * np.abs(dense).max()


def test_parallel_oracle_agrees(fem, orc):
    m = fem.square_mesh(16, 16, 2, perturb=0.1, seed=5)
    rowp, cols = fem.build_bsr_pattern(m.num_nodes, m.conn_ptr, m.conn)
    mp = fem.build_element_bsr_map(m.conn_ptr, m.conn, 9, rowp, cols)
    R0, A0 = orc.assemble(m, mp, cols.size)
    R1, A1 = orc.assemble(m, mp, cols.size, parallel=True)
    assert np.abs(R1 - R0).max() <= 1e-13 * np.abs(R0).max()
    assert np.abs(A1 - A0).max() <= 1e-13 * np.abs(A0).max()
