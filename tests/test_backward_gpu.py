"""Reverse sweep through the Lanczos recurrence (nvb_lanczos_backward) and the differentiable
Ritz energies / intensities / convolved spectrum (nadvibs_b200.autograd), against central
finite differences of the GPU forward, against Hellmann-Feynman for a converged root, and for
consistency across checkpoint intervals and precisions."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from nadvibs_b200 import _lib as L
from nadvibs_b200 import synth
from nadvibs_b200.autograd import (converged_mask, converged_spectrum, convolved_spectrum, ritz, split_theta,
                                   tridiag_eig_backward, tridiag_eigh)

pytestmark = pytest.mark.gpu


def _params(nstates, basis, ordr):
    p = L.default_params()
    p.nstates, p.nmodes, p.ordr, p.niter = nstates, len(basis), ordr, 30
    for i, b in enumerate(basis):
        p.basis[i] = b
    return p


def _system(seed, nstates, basis, ordr=2, **kw):
    cfg = synth.random_small(seed, nstates, basis, ordr, offdiag_even=False, **kw)
    om, cc, pot = synth.draw_small(cfg)
    return _params(nstates, basis, ordr), np.concatenate([synth.flatten_pot(pot), cc, om])


def _forward(p, theta, n, **opts):
    pot, cc, om = split_theta(theta, p.nstates, p.nmodes)
    with L.Handle.from_arrays(p, om, cc, pot, **opts) as h:
        h.seed()
        a, b = h.lanczos(n)
    E, S = tridiag_eigh(a[:n], b[1:n])
    return E, S[0, :] ** 2


def _gradient(p, theta, n, gE, gI, k, record=True, **opts):
    pot, cc, om = split_theta(theta, p.nstates, p.nmodes)
    with L.Handle.from_arrays(p, om, cc, pot, **opts) as h:
        if record:
            h.set_checkpoints(k)
        h.seed()
        a, b = h.lanczos(n)
        E, S = tridiag_eigh(a[:n], b[1:n])
        abar, bbar_off = tridiag_eig_backward(E, S, gE, gI)
        bbar = np.zeros(n)
        bbar[: n - 1] = bbar_off
        return h.lanczos_backward(n, abar, bbar, k)


def _fd(f, theta, idx, rel=1e-5):
    out = []
    for i in idx:
        h = rel * max(abs(theta[i]), 1e-4)
        tp, tm = theta.copy(), theta.copy()
        tp[i] += h
        tm[i] -= h
        out.append((f(tp) - f(tm)) / (2 * h))
    return np.array(out)


@pytest.mark.parametrize("seed,nstates,basis,n", [(71, 2, [4, 4, 3], 10), (72, 3, [3, 3, 2, 2], 12),
                                                  (73, 1, [6, 5], 14)])
def test_backward_matches_finite_differences(seed, nstates, basis, n):
    p, theta = _system(seed, nstates, basis)
    rng = np.random.default_rng(seed)
    gE, gI = rng.normal(size=n), rng.normal(size=n)
    g = _gradient(p, theta, n, gE, gI, k=4, quirk_lower=0)

    def f(th):
        E, I = _forward(p, th, n, quirk_lower=0)
        return float(gE @ E + gI @ I)

    idx = sorted(set(rng.choice(theta.size, size=min(12, theta.size), replace=False).tolist()) | {theta.size - 1})
    fd = _fd(f, theta, idx)
    scale = np.abs(fd).max()
    assert np.abs(g[idx] - fd).max() <= 2e-6 * scale, (g[idx], fd)


def test_cubic_system_gradient_matches_finite_differences():
    """ordr 3: the reverse sweep takes the per-coefficient adjoint (no Gram path) at every step;
    central differences of the GPU forward, and the automatic plan against one level."""
    p, theta = _system(81, 2, [4, 3, 3], ordr=3)
    n = 10
    rng = np.random.default_rng(81)
    gE, gI = rng.normal(size=n), rng.normal(size=n)
    g = _gradient(p, theta, n, gE, gI, k=0, record=False, quirk_lower=0)
    g1 = _gradient(p, theta, n, gE, gI, k=3, record=False, quirk_lower=0)
    assert np.abs(g - g1).max() <= 1e-12 * np.abs(g1).max()

    def f(th):
        E, I = _forward(p, th, n, quirk_lower=0)
        return float(gE @ E + gI @ I)

    idx = sorted(set(rng.choice(theta.size, size=min(14, theta.size), replace=False).tolist()) | {theta.size - 1})
    # the cubic coefficients are small, so the relative step is tiny and the differences carry
    # rounding noise: estimate it from two step sizes and allow the gradient that much beyond
    # the 2e-6 bound of the quadratic tests
    fd = _fd(f, theta, idx)
    fd2 = _fd(f, theta, idx, rel=3e-5)
    tol = 2e-6 * np.abs(fd).max() + 3.0 * np.abs(fd - fd2)
    assert (np.abs(g[idx] - fd) <= tol).all(), (g[idx], fd, fd2)


def test_eig_backward_on_the_gpu_matches_the_host():
    rng = np.random.default_rng(82)
    n = 60
    E, S = tridiag_eigh(rng.normal(size=n), rng.uniform(0.2, 1.0, size=n - 1))
    gE, gI = rng.normal(size=n), rng.normal(size=n)
    a0, b0 = tridiag_eig_backward(E, S, gE, gI)
    a1, b1 = tridiag_eig_backward(E, S, gE, gI, device="cuda:0")
    scale = max(np.abs(a0).max(), np.abs(b0).max())
    assert np.abs(a1 - a0).max() <= 1e-12 * scale and np.abs(b1 - b0).max() <= 1e-12 * scale


def test_checkpoint_interval_and_recording_do_not_change_the_gradient():
    p, theta = _system(74, 2, [4, 3, 3])
    n = 13
    rng = np.random.default_rng(74)
    gE, gI = rng.normal(size=n), rng.normal(size=n)
    ref = _gradient(p, theta, n, gE, gI, k=n, quirk_lower=0)
    scale = np.abs(ref).max()
    for k, rec in [(1, True), (3, True), (5, False), (13, False)]:
        g = _gradient(p, theta, n, gE, gI, k=k, record=rec, quirk_lower=0)
        assert np.abs(g - ref).max() <= 1e-12 * scale, (k, rec)


def _gradient_with_budget(p, theta, n, gE, gI, vectors, record_k=0, precision=None):
    """Automatic plan (k = 0) under a budget of `vectors` vectors beyond the fixed work set."""
    pot, cc, om = split_theta(theta, p.nstates, p.nmodes)
    opts = {"quirk_lower": 0}
    if precision is not None:
        opts["precision"] = precision
    with L.Handle.from_arrays(p, om, cc, pot, **opts) as h:
        if record_k:
            h.set_checkpoints(record_k)
        h.seed()
        a, b = h.lanczos(n)
        E, S = tridiag_eigh(a[:n], b[1:n])
        abar, bbar_off = tridiag_eig_backward(E, S, gE, gI)
        bbar = np.zeros(n)
        bbar[: n - 1] = bbar_off
        N = p.nstates * int(np.prod([p.basis[i] for i in range(p.nmodes)]))
        per = N * (4 if precision == L.NVB_MIXED else 8)
        if vectors is not None:
            h.set_backward_memory(int(5 * per + 10 * N * 8 + vectors * per))
        g = h.lanczos_backward(n, abar, bbar, 0)
        return g, h.backward_plan()


@pytest.mark.parametrize("precision", [None, L.NVB_MIXED])
def test_recursive_checkpointing_matches_single_level(precision):
    """Depths 0, 1 and 2 of the automatic plan replay the same vectors as one level of interval
    n, so the gradients agree to FP64 rounding; the plan follows the budget."""
    p, theta = _system(80, 2, [4, 3, 3])
    n = 40
    rng = np.random.default_rng(80)
    gE, gI = rng.normal(size=n), rng.normal(size=n)
    opts = {"quirk_lower": 0}
    if precision is not None:
        opts["precision"] = precision
    ref = _gradient(p, theta, n, gE, gI, k=n, record=False, **opts)
    scale = np.abs(ref).max()
    # vectors needed (2 L B + B + 2): L = 0: 42, L = 1 (B = 7): 23, L = 2 (B = 4): 22
    for vectors, branching, stored in [(None, n, n), (42, n, n), (23, 7, 7), (22, 4, 4)]:
        g, plan = _gradient_with_budget(p, theta, n, gE, gI, vectors, precision=precision)
        assert plan["top_interval"] == 0 and plan["stored_range"] == stored, (vectors, plan)
        assert plan["branching"] == branching, (vectors, plan)
        assert np.abs(g - ref).max() <= 1e-12 * scale, (vectors, plan)
    # replays: depth 0 one pass (n - 1 H.v), depth 2 about three passes
    _, p0 = _gradient_with_budget(p, theta, n, gE, gI, 42, precision=precision)
    _, p2 = _gradient_with_budget(p, theta, n, gE, gI, 22, precision=precision)
    assert p0["replayed_hv"] == n and 2 * n < p2["replayed_hv"] <= 3 * n, (p0, p2)
    # the forward's recorded pairs become the top level
    g, plan = _gradient_with_budget(p, theta, n, gE, gI, 32, record_k=10, precision=precision)
    assert plan["top_interval"] == 10, plan
    assert np.abs(g - ref).max() <= 1e-12 * scale
    # below the deepest plan's need the sweep refuses instead of allocating
    with pytest.raises(L.NvbError):
        _gradient_with_budget(p, theta, n, gE, gI, 10, precision=precision)


def test_converged_root_matches_hellmann_feynman():
    nstates, basis = 2, [5, 5, 3]
    p, theta = _system(75, nstates, basis)
    n = 60
    pot, cc, om = split_theta(theta, nstates, len(basis))
    with L.Handle.from_arrays(p, om, cc, pot, quirk_lower=0) as h:
        h.set_checkpoints(10)
        h.seed()
        a, b = h.lanczos(n)
        E, S = tridiag_eigh(a[:n], b[1:n])
        assert abs(b[n] * S[-1, 0]) < 1e-9  # the lowest root has converged
        gE = np.zeros(n)
        gE[0] = 1.0
        abar, bbar_off = tridiag_eig_backward(E, S, gE, None)
        bbar = np.zeros(n)
        bbar[: n - 1] = bbar_off
        g = h.lanczos_backward(n, abar, bbar, 10)
        e_hf, g_hf = h.hellmann_feynman(1)
    assert e_hf[0] == pytest.approx(E[0], abs=1e-12)
    assert np.abs(g - g_hf[0]).max() <= 1e-6 * np.abs(g_hf[0]).max()


def test_spectrum_gradient_through_autograd_matches_finite_differences():
    p, theta = _system(76, 2, [4, 4, 3])
    n = 10
    grid = torch.linspace(-500.0, 6000.0, 256, dtype=torch.float64)
    w = torch.from_numpy(np.random.default_rng(76).normal(size=256))

    def loss_t(th):
        E, I = ritz(th, p, n, k=3, quirk_lower=0)
        return (w * convolved_spectrum(E, I, grid, 20.0)).sum()

    th = torch.from_numpy(theta.copy()).requires_grad_(True)
    loss_t(th).backward()
    g = th.grad.numpy()

    def f(x):
        E, I = _forward(p, x, n, quirk_lower=0)
        return float((w * convolved_spectrum(torch.from_numpy(E), torch.from_numpy(I), grid, 20.0)).sum())

    rng = np.random.default_rng(77)
    idx = sorted(rng.choice(theta.size, size=10, replace=False).tolist())
    fd = _fd(f, theta, idx)
    assert np.abs(g[idx] - fd).max() <= 1e-5 * np.abs(fd).max()


def test_mixed_precision_gradient_close_to_fp64():
    p, theta = _system(78, 2, [4, 4, 3])
    n = 10
    rng = np.random.default_rng(78)
    gE, gI = rng.normal(size=n), rng.normal(size=n)
    g64 = _gradient(p, theta, n, gE, gI, k=4, quirk_lower=0)
    g32 = _gradient(p, theta, n, gE, gI, k=4, quirk_lower=0, precision=L.NVB_MIXED)
    assert np.abs(g32 - g64).max() <= 1e-3 * np.abs(g64).max()


def test_backward_refuses_one_sided_couplings():
    cfg = synth.random_small(79, 2, [3, 3], 2, offdiag_even=True, zero_frac=0.0)
    om, cc, pot = synth.draw_small(cfg)
    p = _params(2, [3, 3], 2)
    with L.Handle.from_arrays(p, om, cc, synth.flatten_pot(pot), quirk_lower=1) as h:
        h.seed()
        h.lanczos(5)
        with pytest.raises(L.NvbError):
            h.lanczos_backward(5, np.ones(5), None, 2)


def _config4():
    cfg = synth.config(4)
    om, cc, pot = synth.draw(cfg)
    p = _params(cfg.nstates, cfg.basis, cfg.ordr)
    return p, np.concatenate([synth.flatten_pot(pot), cc, om])


@pytest.mark.parametrize("prec", [L.NVB_FP64, L.NVB_MIXED])
def test_full_forward_record_matches_replayed_plans(prec):
    """Checkpoint interval -1: the forward records every v_j and H v_j, the reverse sweep replays
    nothing, and the gradient equals the automatic (replaying) plan's and one level of interval
    7 to 1e-12 relative.  A budget too small for the record leaves it out and the same call
    falls back to the automatic plan."""
    p, theta = _system(21, 2, [4, 3, 4, 3], 2)
    n = 40
    rng = np.random.default_rng(8)
    gE = rng.normal(size=n)
    gI = rng.normal(size=n)
    g_auto = _gradient(p, theta, n, gE, gI, 0, record=False, precision=prec)
    g_k7 = _gradient(p, theta, n, gE, gI, 7, precision=prec)
    pot, cc, om = split_theta(theta, p.nstates, p.nmodes)
    with L.Handle.from_arrays(p, om, cc, pot, precision=prec) as h:
        h.set_checkpoints(-1)
        h.seed()
        a, b = h.lanczos(n)
        E, S = tridiag_eigh(a[:n], b[1:n])
        abar, bbar_off = tridiag_eig_backward(E, S, gE, gI)
        bbar = np.zeros(n)
        bbar[: n - 1] = bbar_off
        g_rec = h.lanczos_backward(n, abar, bbar, -1)
        assert h.backward_plan()["replayed_hv"] == 0
    scale = np.abs(g_auto).max()
    assert np.abs(g_rec - g_auto).max() <= 1e-12 * scale
    assert np.abs(g_rec - g_k7).max() <= 1e-12 * scale
    with L.Handle.from_arrays(p, om, cc, pot, precision=prec) as h:
        h.set_backward_memory(1)  # nothing fits: no record, and the sweep must then replay
        h.set_checkpoints(-1)
        h.seed()
        h.lanczos(n)
        h.set_backward_memory(0)
        g_fb = h.lanczos_backward(n, abar, bbar, -1)
        assert h.backward_plan()["replayed_hv"] > 0
    assert np.abs(g_fb - g_auto).max() <= 1e-12 * scale


def test_config4_converged_roots_match_hellmann_feynman():
    """Gradient system (2 states, basis [14,12,10,8,8,6], 400 iterations, checkpoints every 50):
    the reverse sweep for a random combination of the converged roots among the lowest 20
    equals the Hellmann-Feynman combination.  (Unconverged Ritz values of a long plain-Lanczos
    run are chaotic functions of theta at the scale of rounding; finite differences of them do
    not converge as h shrinks, so converged roots carry the exact check.)"""
    p, theta = _config4()
    n, k = 400, 50
    pot, cc, om = split_theta(theta, p.nstates, p.nmodes)
    with L.Handle.from_arrays(p, om, cc, pot) as h:
        h.set_checkpoints(k)
        h.seed()
        a, b = h.lanczos(n)
        E, S = tridiag_eigh(a[:n], b[1:n])
        res = np.abs(b[n] * S[-1, :20])
        gap = np.minimum(E[1:21] - E[:20], np.concatenate([[np.inf], E[1:20] - E[:19]]))
        ok = (res < 1e-9) & (gap > 1e-6)  # converged, no ghost copy next to it
        assert ok.sum() >= 5
        c = np.where(ok, np.random.default_rng(4).normal(size=20), 0.0)
        gE = np.zeros(n)
        gE[:20] = c
        abar, bbar_off = tridiag_eig_backward(E, S, gE, None)
        bbar = np.zeros(n)
        bbar[: n - 1] = bbar_off
        g = h.lanczos_backward(n, abar, bbar, k)
        _, ghf = h.hellmann_feynman(20)
    ref = c @ ghf
    assert np.abs(g - ref).max() <= 1e-6 * np.abs(ref).max()


def test_config4_converged_spectrum_gradient_meets_1e5_against_finite_differences():
    """Gradient system (2 states, basis [14,12,10,8,8,6], 400 plain iterations, automatic
    checkpoint plan): the Gaussian-convolved spectrum (sigma 20 cm^-1, 2048 points) of the
    converged Ritz values (bji < 1e-9 hartree in the unperturbed run, ghost copies included,
    the mask kept fixed) against central differences with h = 1e-3 cm^-1 on expansion
    coefficients, block constants and frequencies: 1e-5 relative to max |fd|."""
    p, theta = _config4()
    n = 400
    grid = torch.linspace(-200.0, 8000.0, 2048, dtype=torch.float64)
    w = torch.from_numpy(np.random.default_rng(4).normal(size=2048))
    th = torch.from_numpy(theta.copy()).requires_grad_(True)
    E, I, bji = ritz(th, p, n, residuals=True)
    mask = converged_mask(bji, 1e-9)
    assert int(mask.sum()) >= 10
    (w * converged_spectrum(E, I, mask, grid, 20.0)).sum().backward()
    g = th.grad.numpy()
    npot = theta.size - 3 - p.nmodes

    def f(x):
        E2, I2 = _forward(p, x, n)
        return float((w * converged_spectrum(torch.from_numpy(E2), torch.from_numpy(I2), mask, grid, 20.0)).sum())

    idx = [0, 3, 10, 40, 77, npot, npot + 2, theta.size - 1, theta.size - 4]
    fd = []
    for i in idx:
        hs = 1e-3 / 219474.6313705 * (0.05 if i < npot else 1.0)
        tp, tm = theta.copy(), theta.copy()
        tp[i] += hs
        tm[i] -= hs
        fd.append((f(tp) - f(tm)) / (2 * hs))
    fd = np.array(fd)
    assert np.abs(g[idx] - fd).max() <= 1e-5 * np.abs(fd).max()


def test_config4_spectrum_gradient_against_finite_differences():
    """Gaussian-convolved spectrum (sigma 20 cm^-1, 2048 points) after 100 iterations against
    central differences with h = 1e-3 cm^-1: within 2 % (the finite differences themselves
    vary by that much with h, see the converged-root test for the exact check)."""
    p, theta = _config4()
    n = 100
    grid = torch.linspace(-200.0, 8000.0, 2048, dtype=torch.float64)
    w = torch.from_numpy(np.random.default_rng(4).normal(size=2048))
    th = torch.from_numpy(theta.copy()).requires_grad_(True)
    E, I = ritz(th, p, n)  # automatic checkpoint plan
    (w * convolved_spectrum(E, I, grid, 20.0)).sum().backward()
    g = th.grad.numpy()
    npot = theta.size - 3 - p.nmodes

    def f(x):
        E, I = _forward(p, x, n)
        return float((w * convolved_spectrum(torch.from_numpy(E), torch.from_numpy(I), grid, 20.0)).sum())

    idx = [0, 3, 10, 40, npot, npot + 2, theta.size - 1, theta.size - 4]
    fd = []
    for i in idx:
        hs = 1e-3 / 219474.6313705 * (0.05 if i < npot else 1.0)
        tp, tm = theta.copy(), theta.copy()
        tp[i] += hs
        tm[i] -= hs
        fd.append((f(tp) - f(tm)) / (2 * hs))
    fd = np.array(fd)
    assert np.abs(g[idx] - fd).max() <= 2e-2 * np.abs(fd).max()
