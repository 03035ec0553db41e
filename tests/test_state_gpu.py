"""Restart state (restart.log + nadvibs.35.0), the device archive and lead contributors
(identify_roots, Source/top.f90:1124-1230) through the C ABI, against the oracle."""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from nadvibs_b200 import _lib as L
from nadvibs_b200 import synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _setup(n=1, **opts):
    cfg = synth.config(n)
    om, cc, pot = synth.draw(cfg)
    p = L.default_params()
    p.nstates, p.nmodes, p.ordr = cfg.nstates, cfg.nmodes, cfg.ordr
    for i, b in enumerate(cfg.basis):
        p.basis[i] = b
    h = L.Handle.from_arrays(p, om, cc, synth.flatten_pot(pot), **opts)
    S = O.system_from_arrays(cfg.basis, cfg.nstates, cfg.ordr, om, cc, pot)
    return cfg, h, S


@pytest.mark.parametrize("prec", [L.NVB_FP64, L.NVB_MIXED])
def test_restart_roundtrip_continues_the_recurrence(tmp_path, prec):
    cfg, h, S = _setup(1, precision=prec)
    with h:
        h.seed()
        h.lanczos(40)
        h.save_restart(str(tmp_path))
        a_all, b_all = h.lanczos(10)
    log = (tmp_path / "restart.log").read_text().splitlines()
    assert log[0].strip() == "TOTAL NUMBER OF ITERATIONS IN FILE" and int(log[1]) == 40
    assert os.path.getsize(tmp_path / "nadvibs.35.0") == 3 * cfg.dimen * cfg.nstates * 8
    # the q vectors are v(n-1), v(n) and the unnormalised residual
    q = np.fromfile(tmp_path / "nadvibs.35.0").reshape(3, -1)
    assert np.linalg.norm(q[1]) == pytest.approx(1.0, rel=1e-6)
    assert np.linalg.norm(q[2]) == pytest.approx(b_all[40], rel=1e-6)
    _, h2, _ = _setup(1, precision=prec)
    with h2:
        h2.load_restart(str(tmp_path))
        assert h2.sizes()["iters"] == 40
        a2, b2 = h2.lanczos(10)
    assert (tmp_path / "restart.log.old").exists() and not (tmp_path / "nadvibs.35.0").exists()
    np.testing.assert_array_equal(a2[:40], a_all[:40])
    tol = 1e-10 if prec == L.NVB_FP64 else 1e-5
    np.testing.assert_allclose(a2[40:], a_all[40:], rtol=tol)
    np.testing.assert_allclose(b2[40:], b_all[40:], rtol=tol)


def test_restart_rejects_damaged_files(tmp_path):
    cfg, h, S = _setup(1)
    with h:
        h.seed()
        h.lanczos(5)
        h.save_restart(str(tmp_path))
    good_log = (tmp_path / "restart.log").read_text()
    vec = (tmp_path / "nadvibs.35.0").read_bytes()
    # truncated log
    (tmp_path / "restart.log").write_text("\n".join(good_log.splitlines()[:5]) + "\n")
    _, h2, _ = _setup(1)
    with h2:
        with pytest.raises(L.NvbError) as e:
            h2.load_restart(str(tmp_path))
        assert e.value.code == -2
    # short vector file
    (tmp_path / "restart.log").write_text(good_log)
    (tmp_path / "nadvibs.35.0").write_bytes(vec[: len(vec) // 2])
    _, h3, _ = _setup(1)
    with h3:
        with pytest.raises(L.NvbError) as e:
            h3.load_restart(str(tmp_path))
        assert e.value.code == -2
    # non-finite coefficient
    (tmp_path / "nadvibs.35.0").write_bytes(vec)
    lines = good_log.splitlines()
    lines[5] = " NaN" + lines[5][4:]
    (tmp_path / "restart.log").write_text("\n".join(lines) + "\n")
    _, h4, _ = _setup(1)
    with h4:
        with pytest.raises(L.NvbError):
            h4.load_restart(str(tmp_path))


def _oracle_leads(S, niter, nroots, k):
    a, b, V, _ = S.lanczos(niter, keep_vectors=True)
    E, bji, inten, sign, T = O.ritz(a, b)
    out = []
    for r in range(nroots):
        psi = T[:, r] @ V
        sq = psi ** 2
        order = np.argsort(-sq, kind="stable")[:k]
        out.append((order, sq[order], np.sign(psi[order]), psi))
    return E, out


@pytest.mark.parametrize("archive", [0, 200])
def test_lead_contributors_match_oracle(tmp_path, archive):
    """50 iterations stay inside the rounding horizon of config 1 (no ghost copies yet), so the
    GPU's and the oracle's Lanczos bases agree and so must their Ritz vectors."""
    niter, nroots, k = 50, 4, 5
    cfg, h, S = _setup(1, archive_max=archive)
    N = cfg.dimen
    with h:
        h.seed()
        h.lanczos(niter)
        res = h.lead_contributors(nroots, k, str(tmp_path / "rootinfo.dat"))
    E, ref = _oracle_leads(S, niter, nroots, k)
    for r in range(nroots):
        order, sq, sgn, psi = ref[r]
        lin = (res["state"][r] - 1) * N + (res["index"][r] - 1)
        np.testing.assert_allclose(res["c2"][r], sq, rtol=1e-8, atol=1e-12)
        # indices agree where the magnitudes are distinct
        distinct = np.abs(np.diff(np.concatenate([sq, [0.0]]))) > 1e-9
        assert np.array_equal(lin[distinct], order[distinct])
        np.testing.assert_array_equal(res["phase"][r][distinct], sgn[distinct])
        w = np.array([np.sum(psi[s * N:(s + 1) * N] ** 2) for s in range(cfg.nstates)])
        np.testing.assert_allclose(res["pct"][r], 100 * w / w.sum(), rtol=1e-8, atol=1e-10)
    text = (tmp_path / "rootinfo.dat").read_text().splitlines()
    assert text[0].startswith(" Summary for computing    4 eigenvectors")
    assert text[-1] == "------------ FINISHED EXECUTION ------------"
    assert sum(1 for t in text if t.startswith(" State vector:")) == nroots * k
    assert sum(1 for t in text if t.startswith(" Percent State (1,2):")) == nroots


@pytest.mark.parametrize("sys_id", [1, 3])
def test_spin_orbit_matches_oracle(tmp_path, sys_id):
    """Spin-orbit parameters of the lowest soroots roots and sodata.in (identify_roots,
    Source/top.f90:1153-1175, 1231-1252) against the oracle's Ritz vectors and its own
    formatting, inside the rounding horizon (40 iterations)."""
    niter, soroots, nroots = 40, 4, 6
    if sys_id == 1:
        cfg, h, S = _setup(1, archive_max=200)
    else:
        cfg = synth.random_small(91, 3, [4, 4, 3], 2, offdiag_even=False)
        om, cc, pot = synth.draw_small(cfg)
        p = L.default_params()
        p.nstates, p.nmodes, p.ordr, p.niter = 3, 3, 2, niter
        for i, b in enumerate(cfg.basis):
            p.basis[i] = b
        h = L.Handle.from_arrays(p, om, cc, synth.flatten_pot(pot))
        S = O.system_from_arrays(cfg.basis, 3, 2, om, cc, pot)
    with h:
        h.seed()
        h.lanczos(niter)
        res = h.spin_orbit(soroots, nroots, str(tmp_path / "sodata.in"))
    a, b, V, _ = S.lanczos(niter, keep_vectors=True)
    E, bji, inten, sign, T = O.ritz(a, b)
    psi = [T[:, r] @ V for r in range(soroots)]
    fac = inten[:nroots].max()
    np.testing.assert_allclose(res["energy_ev"], E[:soroots] * O.AU2EV, rtol=1e-12)
    np.testing.assert_allclose(res["amp"], np.sqrt(inten[:soroots] / fac) * sign[:soroots], rtol=1e-8, atol=1e-12)
    ns = cfg.nstates
    for i in range(1, soroots):
        for j in range(i):
            bi, bj = psi[i].reshape(ns, -1), psi[j].reshape(ns, -1)
            ref = bi @ bj.T
            np.testing.assert_allclose(res["overlap"][i, j], ref, rtol=1e-7, atol=1e-10)
    assert not res["overlap"][np.triu_indices(soroots)].any()
    text = (tmp_path / "sodata.in").read_text().splitlines()
    want = O.sodata_lines(E, inten, sign, psi, soroots, nroots, ns)
    assert len(text) == len(want)
    # the root lines are exact; overlap lines agree to the printed digits where the values are
    # not at the rounding noise of a cancellation
    assert text[: 2 + soroots + (ns - 1)] == want[: 2 + soroots + (ns - 1)]
    for t, w in zip(text[2 + soroots + (ns - 1):], want[2 + soroots + (ns - 1):]):
        assert t[:13] == w[:13]
        np.testing.assert_allclose([float(x) for x in t[13:].split()], [float(x) for x in w[13:].split()],
                                   rtol=1e-5, atol=1e-9)
