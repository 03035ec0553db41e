"""Displaced / Duschinsky Franck-Condon seed (Source/secondary.f90:372-726): the oracle's
restatement of the reference's recursions against direct numerical quadrature of
<m_b(T x + d)|n_a(x)> for one and two modes (rotated, displaced, frequency-changed, with the
initial state excited), and the GPU seed against the oracle."""
import math

import numpy as np
import pytest

from oracle import displaced as D


@pytest.mark.parametrize("a,b,d,m", [(1.0, 1.0, 0.7, 0), (1.0, 1.6, -0.4, 0), (0.8, 1.3, 0.5, 1),
                                     (1.2, 0.7, 0.3, 2)])
def test_oracle_recursion_matches_quadrature_1d(a, b, d, m):
    o = D.overlaps([8], [a], [b], [d], [1.0], [m])
    q = D.quadrature_overlaps([8], [a], [b], [d], [1.0], [m], npts=4000, half_width=12)
    assert np.abs(o - q).max() < 1e-12


@pytest.mark.parametrize("m", [[0, 0], [1, 0], [0, 2]])
def test_oracle_recursion_matches_quadrature_2d_rotated(m):
    th = 0.3
    T = np.array([[np.cos(th), -np.sin(th)], [np.sin(th), np.cos(th)]])
    tmat = T.T.reshape(-1)  # tmat[i*n + k] = T[k, i]
    o = D.overlaps([5, 4], [1.0, 1.4], [1.2, 0.9], [0.4, -0.3], tmat, m)
    q = D.quadrature_overlaps([5, 4], [1.0, 1.4], [1.2, 0.9], [0.4, -0.3], tmat, m, npts=300, half_width=10)
    assert np.abs(o - q).max() < 1e-12


def test_only_the_first_excited_mode_counts():
    o1 = D.overlaps([4, 4], [1.0, 1.1], [1.2, 0.9], [0.2, 0.1], np.eye(2).reshape(-1), [1, 2])
    o2 = D.overlaps([4, 4], [1.0, 1.1], [1.2, 0.9], [0.2, 0.1], np.eye(2).reshape(-1), [1, 0])
    assert np.array_equal(o1, o2)


def _gpu_case(seed, nstates, basis, istate):
    from nadvibs_b200 import _lib as L
    from nadvibs_b200 import synth
    from oracle import oracle as O
    cfg = synth.random_small(seed, nstates, basis, 2, offdiag_even=False)
    om, cc, pot = synth.draw_small(cfg)
    rng = np.random.default_rng(seed)
    M = len(basis)
    Q, _ = np.linalg.qr(rng.normal(size=(M, M)))
    tmat = Q.T.reshape(-1)                      # T = Q, column-major
    bom = om * rng.uniform(0.8, 1.2, size=M)
    dvec = rng.normal(0.0, 4.0, size=M)
    p = L.default_params()
    p.nstates, p.nmodes, p.ordr, p.niter = nstates, M, 2, 20
    for i, b in enumerate(basis):
        p.basis[i] = b
    for i, v in enumerate(istate):
        p.initstate[i] = v
    S = O.system_from_arrays(basis, nstates, 2, om, cc, pot, quirk_lower=False)
    ov = D.overlaps(basis, om, bom, dvec, tmat, istate)
    return L, p, om, cc, synth.flatten_pot(pot), (bom, dvec, tmat), S, ov, cfg


def _numpy_lanczos(S, v1, n):
    a, b = [], [float(np.linalg.norm(v1))]
    vp, v, bp = np.zeros_like(v1), v1 / b[0], 0.0
    for _ in range(n):
        w = S.hv(v)
        al = float(v @ w)
        r = w - al * v - bp * vp
        be = float(np.linalg.norm(r))
        a.append(al)
        b.append(be)
        vp, v, bp = v, r / be, be
    return np.array(a), np.array(b)


@pytest.mark.gpu
@pytest.mark.parametrize("istate", [[0, 0, 0], [0, 2, 0]])
@pytest.mark.parametrize("prec", [0, 1])
def test_gpu_displaced_seed_drives_the_recurrence(istate, prec):
    L, p, om, cc, potf, disp, S, ov, cfg = _gpu_case(81, 2, [5, 4, 3], istate)
    n = 12
    w = np.array([1.0, 0.5])
    q = (w / w.sum()) / np.linalg.norm(w / w.sum())
    v1 = np.concatenate([q[s] * ov / np.linalg.norm(ov) for s in range(2)])
    a_ref, b_ref = _numpy_lanczos(S, v1, n)
    with L.Handle.from_arrays(p, om, cc, potf, quirk_lower=0, precision=prec) as h:
        h.set_displaced_seed(*disp)
        assert h.seed_overlap() == pytest.approx(np.linalg.norm(ov), rel=1e-12)
        h.seed(w)
        a, b = h.lanczos(n)
    tol = 1e-10 if prec == 0 else 2e-5
    scale = np.abs(a_ref).max()
    assert np.abs(a - a_ref).max() <= tol * scale
    assert np.abs(b[1:] - b_ref[1:]).max() <= tol * scale


@pytest.mark.gpu
def test_gpu_displaced_seed_from_files_and_replay(tmp_path):
    from nadvibs_b200 import synth
    L, p, om, cc, potf, disp, S, ov, cfg = _gpu_case(82, 2, [4, 4, 3], [1, 0, 0])
    b_in, n_in = str(tmp_path / "basis.in"), str(tmp_path / "nadvibs.in")
    synth.write_basis_in(b_in, cfg, niter=20, initstate=[1, 0, 0], shiftref=1)
    _, _, pot = synth.draw_small(cfg)
    synth.write_nadvibs_in(n_in, 3, om, cc, pot, displaced=disp)
    with L.Handle.from_files(b_in, n_in, quirk_lower=0) as h:
        assert h.seed_overlap() == pytest.approx(np.linalg.norm(ov), rel=1e-12)
        h.seed()
        h.lanczos(15)
        two_pass = h.lead_contributors(3, 4)
    with L.Handle.from_files(b_in, n_in, quirk_lower=0, archive_max=50) as h:
        h.seed()
        h.lanczos(15)
        archived = h.lead_contributors(3, 4)
    np.testing.assert_allclose(two_pass["c2"], archived["c2"], rtol=1e-10, atol=1e-14)


def _report_lines(path):
    with open(path) as f:
        return f.read().splitlines()


@pytest.mark.gpu
@pytest.mark.parametrize("istate", [[0, 0, 0], [0, 2, 0]])
def test_gpu_seed_report_of_the_displaced_seed(istate, tmp_path):
    """The seed section of output.dat (Source/secondary.f90:351-802) for a displaced seed: one
    line per quanta-sum level whose counts add up to the basis size, the <m| levels built, the
    overlap with the initial state, the dominant basis functions in the reference's format
    ('  NN. q,q,q,: value') equal to the oracle's 40 largest <m|n>^2, and the normalisation by
    the state weights."""
    L, p, om, cc, potf, disp, S, ov, cfg = _gpu_case(82, 2, [5, 4, 3], istate)
    out = str(tmp_path / "output.dat")
    w = np.array([1.0, 0.5])
    with L.Handle.from_arrays(p, om, cc, potf, quirk_lower=0) as h:
        h.set_displaced_seed(*disp)
        h.seed(w)
        h.write_seed_report(out)
    lines = _report_lines(out)
    assert "  Generating seed vector by computing ANION/ORIGIN overlap..." in lines
    levels = [ln for ln in lines if ln.startswith("  LEVEL ")]
    assert len(levels) == (5 - 1) + (4 - 1) + (3 - 1) + 1
    assert sum(int(ln.split()[-1]) for ln in levels) == 5 * 4 * 3
    assert [ln for ln in lines if ln.startswith("  Building <m|")] == \
        [f"  Building <m| = <{i:2d}|" for i in range(1, max(istate) + 1)]
    ovl = [ln for ln in lines if ln.startswith("  Overlap with the initial state:")]
    assert float(ovl[0].split(":")[1]) == pytest.approx(np.linalg.norm(ov), abs=1e-6)
    dom = [ln for ln in lines if len(ln) > 5 and ln[4] == "." and ln[:4].strip().isdigit()]
    order = np.argsort(-ov ** 2, kind="stable")[:40]
    assert len(dom) == min(40, int((ov != 0).sum()))
    for k, (ln, row) in enumerate(zip(dom, order)):
        head, val = ln.rsplit(":", 1)
        assert head.startswith(f"  {k + 1:2d}. ")
        quanta = [int(t) for t in head[6:].split(",") if t.strip()]
        assert quanta == [row // 12, (row // 3) % 4, row % 3]
        assert float(val) == pytest.approx(ov[row] ** 2, abs=1e-6)
    norms = [ln for ln in lines if ln.startswith("  ||STATE")]
    q = w / w.sum()
    for s, ln in enumerate(norms):
        assert float(ln.split("=")[1].split("--")[0]) == pytest.approx(q[s], abs=1e-4)
    assert lines.count("  Normalizing Initial Lanczos Vector...") == 1


@pytest.mark.gpu
def test_gpu_seed_report_of_the_origin_seed(tmp_path):
    """shiftref = 0: the report of the reference's simple seed (the ground state of every
    electronic state): overlap 1, one dominant contribution (all quanta 0, weight 1)."""
    from nadvibs_b200 import _lib as L
    from nadvibs_b200 import synth
    cfg = synth.config(1)
    om, cc, pot = synth.draw(cfg)
    p = L.default_params()
    p.nstates, p.nmodes, p.ordr = cfg.nstates, cfg.nmodes, cfg.ordr
    for i, b in enumerate(cfg.basis):
        p.basis[i] = b
    out = str(tmp_path / "output.dat")
    with L.Handle.from_arrays(p, om, cc, synth.flatten_pot(pot)) as h:
        h.seed()
        h.write_seed_report(out)
    lines = _report_lines(out)
    assert "  Generating seed vector using ANION basis..." in lines
    assert "  Overlap with the initial state:       1.000000" in lines
    assert "   1.  0, 0, 0, 0,:     1.000000" in lines
    assert "  || TOTAL || = 1.0000 -- (|| TOTAL ||)^2 = 1.0000" in lines
