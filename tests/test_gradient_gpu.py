"""Gradient path: the adjoint contraction d<u|H|v>/dtheta (nvb_hv_adjoint_coeffs) against
central finite differences of the oracle's H.v, and Hellmann-Feynman gradients of converged
Ritz energies (nvb_hellmann_feynman) against finite differences of the dense lowest
eigenvalue.  theta = (nadvibs.in expansion coefficients, block constants, frequencies)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from nadvibs_b200 import _lib as L
from nadvibs_b200 import synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _params(nstates, basis, ordr, niter=30):
    p = L.default_params()
    p.nstates, p.nmodes, p.ordr, p.niter = nstates, len(basis), ordr, niter
    for i, b in enumerate(basis):
        p.basis[i] = b
    return p


def _split(theta, npot, nb, M):
    return theta[npot + nb:], theta[npot:npot + nb], theta[:npot]


def _unflatten(pot_flat, nb, ordr, M):
    out, off = [], 0
    for _ in range(nb):
        per = []
        for d in range(1, ordr + 1):
            n = synth.numut(M, d)
            per.append(pot_flat[off:off + n])
            off += n
        out.append(per)
    return out


# ordr 3 runs the cubic Gram path (every P_m an entry of (X u, x^2 u)^T (v, X v, x^2 v, x^3 v,
# X X v)): cases with several distinct triples of modes, 1- and 2-function modes, up to 4 states
# and both settings of the x^3 quirk
@pytest.mark.parametrize("seed,nstates,basis,ordr,qc", [(41, 2, [4, 3, 3], 2, 1), (42, 3, [3, 3, 2], 3, 1),
                                                        (43, 1, [5, 4], 4, 1), (44, 2, [4, 4, 3], 2, 1),
                                                        (45, 2, [4, 3, 2, 3], 3, 1), (45, 2, [4, 3, 2, 3], 3, 0),
                                                        (46, 1, [5, 3, 4, 2, 3], 3, 1), (47, 4, [2, 3, 2, 2], 3, 0),
                                                        (48, 2, [3, 1, 4, 3], 3, 1)])
@pytest.mark.parametrize("dt", [torch.float64, torch.float32])
def test_adjoint_matches_finite_differences(seed, nstates, basis, ordr, qc, dt):
    cfg = synth.random_small(seed, nstates, basis, ordr)
    om, cc, pot = synth.draw_small(cfg)
    M = len(basis)
    nb = nstates * (nstates + 1) // 2
    potf = synth.flatten_pot(pot)
    npot = len(potf)
    theta = np.concatenate([potf, cc, om])
    S = O.system_from_arrays(basis, nstates, ordr, om, cc, pot, quirk_lower=False, quirk_cubic=bool(qc))
    rng = np.random.default_rng(seed)
    u = rng.normal(size=S.ntotal)
    v = rng.normal(size=S.ntotal)
    with L.Handle.from_arrays(_params(nstates, basis, ordr), om, cc, potf, quirk_lower=0, quirk_cubic=qc) as h:
        ut = torch.from_numpy(u).to("cuda", dtype=dt)
        vt = torch.from_numpy(v).to("cuda", dtype=dt)
        torch.cuda.synchronize()
        g = h.adjoint_ptr(ut.data_ptr(), vt.data_ptr(), L.DTYPE_F64 if dt == torch.float64 else L.DTYPE_F32)
    if dt == torch.float32:
        u = ut.double().cpu().numpy()
        v = vt.double().cpu().numpy()

    def f(th):
        w, c, p = _split(th, npot, nb, M)
        Sx = O.system_from_arrays(basis, nstates, ordr, w, c, _unflatten(p, nb, ordr, M), quirk_lower=False,
                                  quirk_cubic=bool(qc), ztoler=0.0)
        return float(u @ Sx.hv(v))

    fd = np.zeros_like(theta)
    for i in range(len(theta)):
        h_i = 1e-6 * max(abs(theta[i]), 1e-3)
        tp, tm = theta.copy(), theta.copy()
        tp[i] += h_i
        tm[i] -= h_i
        fd[i] = (f(tp) - f(tm)) / (2 * h_i)
    scale = np.abs(fd).max()
    tol = 1e-6 if dt == torch.float64 else 1e-4
    assert np.abs(g - fd).max() <= tol * scale, np.abs(g - fd).argmax()


def test_hellmann_feynman_matches_dense_eigenvalue_derivative():
    nstates, basis, ordr = 2, [4, 4, 3], 2
    cfg = synth.random_small(51, nstates, basis, ordr, offdiag_even=False)
    om, cc, pot = synth.draw_small(cfg)
    potf = synth.flatten_pot(pot)
    M, nb, npot = len(basis), 3, len(potf)
    dim = nstates * int(np.prod(basis))
    with L.Handle.from_arrays(_params(nstates, basis, ordr), om, cc, potf, quirk_lower=0, archive_max=dim) as h:
        h.set_reorthog(2, 50)
        h.seed()
        h.lanczos(dim)
        E, G = h.hellmann_feynman(2)
    theta = np.concatenate([potf, cc, om])

    def lowest(th):
        w, c, p = _split(th, npot, nb, M)
        Sx = O.system_from_arrays(basis, nstates, ordr, w, c, _unflatten(p, nb, ordr, M), quirk_lower=False,
                                  ztoler=0.0)
        return np.linalg.eigvalsh(Sx.dense())[0]

    assert E[0] == pytest.approx(lowest(theta), abs=1e-10)
    for i in list(range(0, len(theta), 3)) + [len(theta) - 1]:
        h_i = 1e-5 * max(abs(theta[i]), 1e-3)
        tp, tm = theta.copy(), theta.copy()
        tp[i] += h_i
        tm[i] -= h_i
        fd = (lowest(tp) - lowest(tm)) / (2 * h_i)
        assert G[0, i] == pytest.approx(fd, rel=1e-5, abs=1e-9 * max(1.0, abs(fd)))


def test_adjoint_cubic_eleven_modes_single_buffered_tile():
    """3 states and 11 modes give 384 Gram columns: too many for two column tiles in shared
    memory, so the cubic Gram path runs its single-buffered tile.  Checked against central
    differences of the oracle on every frequency and block constant and a spread of expansion
    coefficients of each degree."""
    nstates, basis, ordr, seed = 3, [2, 2, 3, 2, 2, 2, 2, 2, 2, 3, 2], 3, 49
    cfg = synth.random_small(seed, nstates, basis, ordr)
    om, cc, pot = synth.draw_small(cfg)
    M = len(basis)
    nb = nstates * (nstates + 1) // 2
    potf = synth.flatten_pot(pot)
    npot = len(potf)
    theta = np.concatenate([potf, cc, om])
    S = O.system_from_arrays(basis, nstates, ordr, om, cc, pot, quirk_lower=False, quirk_cubic=True)
    rng = np.random.default_rng(seed)
    u = rng.normal(size=S.ntotal)
    v = rng.normal(size=S.ntotal)
    with L.Handle.from_arrays(_params(nstates, basis, ordr), om, cc, potf, quirk_lower=0, quirk_cubic=1) as h:
        ut = torch.from_numpy(u).to("cuda")
        vt = torch.from_numpy(v).to("cuda")
        torch.cuda.synchronize()
        g = h.adjoint_ptr(ut.data_ptr(), vt.data_ptr(), L.DTYPE_F64)

    def f(th):
        w, c, p = _split(th, npot, nb, M)
        Sx = O.system_from_arrays(basis, nstates, ordr, w, c, _unflatten(p, nb, ordr, M), quirk_lower=False,
                                  quirk_cubic=True, ztoler=0.0)
        return float(u @ Sx.hv(v))

    idx = list(range(0, npot, 23)) + list(range(npot, len(theta)))
    fd = np.zeros(len(idx))
    for j, i in enumerate(idx):
        h_i = 1e-6 * max(abs(theta[i]), 1e-3)
        tp, tm = theta.copy(), theta.copy()
        tp[i] += h_i
        tm[i] -= h_i
        fd[j] = (f(tp) - f(tm)) / (2 * h_i)
    assert np.abs(g[idx] - fd).max() <= 1e-6 * np.abs(fd).max()
