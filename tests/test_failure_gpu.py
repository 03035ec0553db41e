"""Failure detection without a GPU fault: with nvb_set_fault_test(1) the factorised quadratic
H.v kernel issues none of its shared-memory copies, so every bounded wait of its consumer warps
runs out.  The kernel must finish (no hang), report through its error word (NVB_ERR_CUDA at the
next synchronising call), and leave the handle usable: the same Lanczos run afterwards matches
a handle that never failed."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from nadvibs_b200 import _lib as L
from nadvibs_b200 import synth

pytestmark = pytest.mark.gpu


def _handle():
    cfg = synth.random_small(61, 1, [4, 3, 5, 4, 8, 8], 2, offdiag_bilinear=False)
    om, cc, pot = synth.draw_small(cfg)
    p = L.default_params()
    p.nstates, p.nmodes, p.ordr, p.niter = 1, 6, 2, 20
    for i, b in enumerate(cfg.basis):
        p.basis[i] = b
    return L.Handle.from_arrays(p, om, cc, synth.flatten_pot(pot), hv_kernel=3)


def test_waits_that_run_out_are_reported_and_the_handle_recovers():
    with _handle() as ref:
        ref.seed()
        a_ref, b_ref = ref.lanczos(8)
    with _handle() as h:
        assert h.hv_kernel() == "quad"
        h.set_fault_test(1)
        h.seed()
        with pytest.raises(L.NvbError) as e:
            h.lanczos(3)
        assert e.value.code == -3  # NVB_ERR_CUDA
        assert "gave up waiting" in str(e.value)
        h.set_fault_test(0)
        h.synchronize()          # the error was reported once
        h.seed()
        a, b = h.lanczos(8)
    np.testing.assert_array_equal(a, a_ref)
    np.testing.assert_array_equal(b, b_ref)
