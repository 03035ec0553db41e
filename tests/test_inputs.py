"""Input stage (no GPU): basis.in namelist, nadvibs.in reader and the term compiler of the
product library against the oracle's restatement of Source/top.f90:88-246."""
import math
import os

import numpy as np
import pytest

from nadvibs_b200 import _lib as L
from nadvibs_b200 import synth
from oracle import oracle as O
from oracle import termcomp as tc


def _host_handle(b, n):
    return L.Handle.from_files(b, n, device=-1)


def _compare_terms(h, tt):
    got = h.terms()
    assert len(got) == tt.nterms
    for t, g in enumerate(got):
        assert [int(m) for m in g["modes"]] == tt.modes[t]
        assert [int(p) for p in g["pows"]] == tt.pows[t]
        assert g["pairs"] == tt.pairs[t]
        np.testing.assert_allclose(g["coefs"], tt.coefs[t], rtol=1e-15, atol=0)


@pytest.mark.parametrize("n", [1, 2, 4, 5])
def test_term_table_matches_oracle_for_benchmark_systems(tmp_path, n):
    cfg = synth.config(n)
    b, f = synth.write_inputs(str(tmp_path), cfg)
    kv, S = O.system_from_files(b, f)
    with _host_handle(b, f) as h:
        sz = h.sizes()
        assert sz["dimen"] == cfg.dimen and sz["nstates"] == cfg.nstates
        _compare_terms(h, S.tt)


@pytest.mark.parametrize("seed,nstates,basis,ordr", [(1, 2, [3, 4, 2], 2), (2, 3, [2, 2, 3, 2], 3),
                                                     (3, 4, [3, 1, 2], 4), (4, 1, [6], 4), (5, 10, [2, 2], 1)])
def test_term_table_matches_oracle_random(tmp_path, seed, nstates, basis, ordr):
    cfg = synth.random_small(seed, nstates, basis, ordr)
    om, cc, pot = synth.draw_small(cfg)
    synth.write_nadvibs_in(str(tmp_path / "nadvibs.in"), len(basis), om, cc, pot)
    synth.write_basis_in(str(tmp_path / "basis.in"), cfg)
    kv, S = O.system_from_files(str(tmp_path / "basis.in"), str(tmp_path / "nadvibs.in"))
    with _host_handle(str(tmp_path / "basis.in"), str(tmp_path / "nadvibs.in")) as h:
        _compare_terms(h, S.tt)
    # in-memory path gives the same table
    p = L.read_basis(str(tmp_path / "basis.in"))
    with L.Handle.from_arrays(p, om, cc, synth.flatten_pot(pot), device=-1) as h2:
        _compare_terms(h2, S.tt)


def test_ztoler_drops_small_coefficients(tmp_path):
    cfg = synth.random_small(11, 2, [3, 3], 2, zero_frac=0.0)
    om, cc, pot = synth.draw_small(cfg)
    pot[0][0][0] = 1e-9
    synth.write_nadvibs_in(str(tmp_path / "nadvibs.in"), 2, om, cc, pot)
    synth.write_basis_in(str(tmp_path / "basis.in"), cfg, ztoler="1.0d-8")
    kv, S = O.system_from_files(str(tmp_path / "basis.in"), str(tmp_path / "nadvibs.in"))
    assert kv["ztoler"] == 1e-8
    with _host_handle(str(tmp_path / "basis.in"), str(tmp_path / "nadvibs.in")) as h:
        _compare_terms(h, S.tt)


NAMELISTS = [
    "&NADVIBS niter=500, nmodes=4, nstates=2, basis=8,8,6,6, ordr=2 /\n",
    " &nadvibs\n  niter = 500 ! comment\n  nmodes=3 nstates=3\n  basis = 3*4\n  weights = 1.0d0, 0.5D0 2e0\n"
    "  ztoler = 1.0d-12, bconv = 4, idroots = -3, reorthog = 2, chkorthog = 50\n /\n",
    "&NADVIBS\n nmodes=5, basis(1)=10, basis(3)=7, npirr=3,2, nirreps=2, initstate=0,1,1,0,0 /",
    "$NADVIBS nmodes=2 basis=5 6 restart=0 $END",
]


@pytest.mark.parametrize("text", NAMELISTS)
def test_namelist_parse_matches_oracle(tmp_path, text):
    path = tmp_path / "basis.in"
    path.write_text(text)
    kv = tc.read_namelist(text.replace("$NADVIBS", "&NADVIBS").replace("$END", "/"))
    p = L.read_basis(str(path))
    for key in ["niter", "nmodes", "nstates", "ordr", "bconv", "idroots", "reorthog", "chkorthog", "nirreps"]:
        assert getattr(p, key) == kv[key], key
    assert list(p.basis[: p.nmodes]) == kv["nfunc"]
    assert list(p.initstate[: p.nmodes]) == kv["istate"]
    assert list(p.npirr[: p.nirreps]) == kv["npirr"][: kv["nirreps"]]
    assert list(p.weights[:3]) == kv["weights"][:3]
    assert p.ztoler == kv["ztoler"]


def test_list_directed_variants(tmp_path):
    """Values may span records, carry D exponents and r*c repeats; leftovers on a record are
    discarded (Fortran list-directed input)."""
    cfg = synth.random_small(21, 2, [3, 2, 2], 2, zero_frac=0.0)
    om, cc, pot = synth.draw_small(cfg)
    lines = [" freq", " " + " ".join(f"{v:.17e}".replace("e", "D") for v in om) + " 99 99"]
    for b in range(3):
        lines += [" const", f" {cc[b]:.17e}, extra"]
        lines += [" order1"] + [f" {v:.17e}" for v in pot[b][0]]
        vals = pot[b][1].copy()
        vals[1] = vals[2] = 0.0
        pot[b][1] = vals
        lines += [" order2", f" {vals[0]:.17e} 2*0.0", " " + " ".join(f"{v:.17e}" for v in vals[3:])]
    (tmp_path / "nadvibs.in").write_text("\n".join(lines) + "\n")
    synth.write_basis_in(str(tmp_path / "basis.in"), cfg)
    kv, S = O.system_from_files(str(tmp_path / "basis.in"), str(tmp_path / "nadvibs.in"))
    np.testing.assert_array_equal(S.omega, om)
    with _host_handle(str(tmp_path / "basis.in"), str(tmp_path / "nadvibs.in")) as h:
        _compare_terms(h, S.tt)


def test_bad_inputs_fail_with_codes(tmp_path):
    cfg = synth.config(1)
    b, f = synth.write_inputs(str(tmp_path), cfg)
    text = open(f).read().splitlines()
    (tmp_path / "short.in").write_text("\n".join(text[:-3]) + "\n")
    with pytest.raises(L.NvbError) as e:
        _host_handle(b, str(tmp_path / "short.in"))
    assert e.value.code == -2
    bad = text[:]
    bad[1] = bad[1].replace(bad[1].split()[0], "NaN", 1)
    (tmp_path / "nan.in").write_text("\n".join(bad) + "\n")
    with pytest.raises(L.NvbError) as e:
        _host_handle(b, str(tmp_path / "nan.in"))
    assert e.value.code in (-1, -2)
    with pytest.raises(L.NvbError) as e:
        _host_handle(str(tmp_path / "missing.in"), f)
    assert e.value.code == -2
    (tmp_path / "unk.in").write_text("&NADVIBS nmodes=4, bogus=3 /\n")
    with pytest.raises(L.NvbError):
        L.read_basis(str(tmp_path / "unk.in"))
    (tmp_path / "big.in").write_text("&NADVIBS nmodes=1, nstates=2, ordr=5, basis=4 /\n")
    p = L.read_basis(str(tmp_path / "big.in"))
    with pytest.raises(L.NvbError) as e:
        L.Handle.from_arrays(p, [0.01], [0, 0, 0], np.zeros(15), device=-1)
    assert e.value.code == -1
