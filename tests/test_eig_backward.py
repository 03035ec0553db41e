"""Eigen-derivatives of the symmetric tridiagonal T_n used by the gradient path (host code,
no GPU): dL/dalpha and dL/dbeta from dL/dE and dL/dI (I_i = s_{1,i}^2) against central finite
differences of a LAPACK eigensolve."""
import numpy as np
import pytest

from nadvibs_b200.autograd import tridiag_eig_backward, tridiag_eigh


@pytest.mark.parametrize("n,seed", [(6, 1), (15, 2), (40, 3)])
def test_tridiag_eig_backward_matches_fd(n, seed):
    rng = np.random.default_rng(seed)
    a = rng.normal(size=n)
    b = rng.uniform(0.2, 1.0, size=n - 1)
    gE = rng.normal(size=n)
    gI = rng.normal(size=n)

    def loss(a_, b_):
        E, S = tridiag_eigh(a_, b_)
        return float(gE @ E + gI @ (S[0, :] ** 2))

    E, S = tridiag_eigh(a, b)
    abar, bbar = tridiag_eig_backward(E, S, gE, gI)
    h = 1e-6
    fa = np.array([(loss(a + h * np.eye(n)[i], b) - loss(a - h * np.eye(n)[i], b)) / (2 * h) for i in range(n)])
    fb = np.array([(loss(a, b + h * np.eye(n - 1)[i]) - loss(a, b - h * np.eye(n - 1)[i])) / (2 * h)
                   for i in range(n - 1)])
    scale = max(np.abs(fa).max(), np.abs(fb).max())
    assert np.abs(abar - fa).max() <= 1e-6 * scale
    assert np.abs(bbar - fb).max() <= 1e-6 * scale


def test_energies_only_gradient_is_the_eigenvector_outer_product():
    rng = np.random.default_rng(9)
    n = 10
    a, b = rng.normal(size=n), rng.uniform(0.3, 1.0, size=n - 1)
    E, S = tridiag_eigh(a, b)
    gE = np.zeros(n)
    gE[0] = 1.0
    abar, bbar = tridiag_eig_backward(E, S, gE, None)
    assert np.allclose(abar, S[:, 0] ** 2, atol=1e-14)
    assert np.allclose(bbar, 2 * S[:-1, 0] * S[1:, 0], atol=1e-14)
