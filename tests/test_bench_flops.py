"""The bench's reference-equivalent flop count of one H.v (bench.hv_flops) against the oracle's
restatement of the reference's term compiler and step enumeration (CPU only)."""
import importlib.util
import math
import os

import pytest

from nadvibs_b200 import synth
from oracle import termcomp as TC

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_module", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


@pytest.mark.parametrize("n", [1, 2, 4])
def test_hv_flops_matches_the_term_table(n):
    cfg = synth.config(n)
    om, cc, pot = synth.draw(cfg)
    tt = TC.compile_terms(cfg.nmodes, cfg.nstates, cfg.ordr, om, cc, pot)
    nfunc = list(cfg.basis)
    count = cfg.nstates  # harmonic energy + constants per state
    for t in range(tt.nterms):
        steps = TC.term_steps(tt.modes[t], tt.pows[t], nfunc)
        nonzero = sum(1 for s in steps if any(s))
        count += nonzero * len(tt.pairs[t])
        if TC.is_diag_term(tt.pows[t], tt.modes[t], nfunc):
            count += len(tt.pairs[t])
    expected = 2.0 * math.prod(cfg.basis) * count
    assert _bench().hv_flops(cfg) == pytest.approx(expected, rel=1e-12)


def test_config2_flops_per_hv():
    # 468 shift contributions + 27 diagonal-section terms per row position, 2 flops each
    assert _bench().hv_flops(synth.config(2)) == pytest.approx(2.0 * 88_473_600 * 495, rel=1e-12)
