"""CPU checks of the oracle's GreenStrainType::NONLINEAR element (the reference's
planeStressWeakRes<NONLINEAR>, element/FEKernels.h:286-315, which its kernels take
as a template option, :317,379,589,786): the weak residual is the gradient of
the strain energy, the Jacobian is the derivative of the residual, finite rigid
rotations are stress free, and the small-strain limit is the linear element."""
import numpy as np
import pytest

E, NU, T = 70e9, 0.3, 0.5


def _element_data(fem, p, amp, seed=7):
    m = fem.square_mesh(1, 1, p, 1.0, 1.0, 0.0, seed=seed)
    rng = np.random.default_rng(seed + p)
    X = m.coords + rng.uniform(-0.05, 0.05, m.coords.shape) / p
    U = rng.uniform(-amp, amp, X.shape)
    return X, U


@pytest.mark.parametrize("p", [1, 2, 3, 4])
def test_residual_is_energy_gradient(fem, orc, p):
    X, U = _element_data(fem, p, 5e-2)
    n = X.shape[0]
    Re, _ = orc.element(p, X, U, E, NU, T, strain="nonlinear")
    h = 1e-6
    for c in (0, 1, n, 2 * n - 1):
        Up, Um = U.copy().reshape(-1), U.copy().reshape(-1)
        Up[c] += h
        Um[c] -= h
        fd = (orc.element_energy(p, X, Up.reshape(n, 2), E, NU, T, "nonlinear") -
              orc.element_energy(p, X, Um.reshape(n, 2), E, NU, T, "nonlinear")) / (2 * h)
        assert abs(fd - Re[c]) <= 1e-6 * np.abs(Re).max()


@pytest.mark.parametrize("p", [1, 2, 3, 4])
def test_jacobian_is_residual_derivative_and_symmetric(fem, orc, p):
    X, U = _element_data(fem, p, 5e-2)
    n = X.shape[0]
    _, Ke = orc.element(p, X, U, E, NU, T, strain="nonlinear")
    scale = np.abs(Ke).max()
    assert np.abs(Ke - Ke.T).max() <= 1e-13 * scale
    h = 1e-7
    for c in range(0, 2 * n, max(1, n // 3)):
        Up, Um = U.copy().reshape(-1), U.copy().reshape(-1)
        Up[c] += h
        Um[c] -= h
        Rp, _ = orc.element(p, X, Up.reshape(n, 2), E, NU, T, strain="nonlinear")
        Rm, _ = orc.element(p, X, Um.reshape(n, 2), E, NU, T, strain="nonlinear")
        assert np.abs((Rp - Rm) / (2 * h) - Ke[:, c]).max() <= 1e-6 * scale


@pytest.mark.parametrize("p", [1, 2, 3, 4])
def test_finite_rigid_rotation(fem, orc, p):
    """u = (Q - I) x: Green strain vanishes, so R = 0, and K annihilates the
    rotation increment W (x + u); the linear element is not rotation invariant."""
    X, _ = _element_data(fem, p, 0.0)
    n = X.shape[0]
    th = 0.4
    Q = np.array([[np.cos(th), -np.sin(th)], [np.sin(th), np.cos(th)]])
    U = X @ Q.T - X
    _, K0 = orc.element(p, X, np.zeros_like(U), E, NU, T)
    scale = np.abs(K0).max() * np.abs(U).max()
    Rn, Kn = orc.element(p, X, U, E, NU, T, strain="nonlinear")
    assert np.abs(Rn).max() <= 1e-12 * scale
    Rl, _ = orc.element(p, X, U, E, NU, T, strain="linear")
    assert np.abs(Rl).max() >= 1e-2 * scale
    W = np.array([[0.0, -1.0], [1.0, 0.0]])
    inc = ((X + U) @ W.T).reshape(-1)
    assert np.abs(Kn @ inc).max() <= 1e-12 * np.abs(Kn).max() * np.abs(inc).max()


@pytest.mark.parametrize("p", [1, 3])
def test_small_strain_limit(fem, orc, p):
    """At u = 0 both strains give the same K and R = 0; for small u the
    difference is second order in u."""
    X, U = _element_data(fem, p, 1e-3)
    R0l, K0l = orc.element(p, X, np.zeros_like(U), E, NU, T)
    R0n, K0n = orc.element(p, X, np.zeros_like(U), E, NU, T, strain="nonlinear")
    assert np.abs(R0n).max() == 0.0 and np.abs(R0l).max() == 0.0
    assert np.abs(K0n - K0l).max() <= 1e-14 * np.abs(K0l).max()
    d = []
    for s in (1.0, 0.5):
        Rl, _ = orc.element(p, X, s * U, E, NU, T)
        Rn, _ = orc.element(p, X, s * U, E, NU, T, strain="nonlinear")
        d.append(np.abs(Rn - Rl).max())
    assert 3.5 <= d[0] / d[1] <= 4.5
