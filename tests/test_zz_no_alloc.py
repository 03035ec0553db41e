"""The allocation-free inner product, nvb_dot_noalloc, through the C ABI.

Callers that cannot allocate device memory (their GPU memory is owned by their own pool
allocator, or their loop must not call cudaMalloc/cudaFree, which may synchronise the device)
use nvb_dot_noalloc: its block partials live in a static device array of the library.  Here
it runs twice in a row, on different inputs, and each result is compared with nvb_dot (the
handle-based product, whose partials are in cudaMalloc'd scratch) within the FP64 tolerance
used by the other dot-product tests (1e-12 relative).  This file is collected last so that a
failure here stops a -x run only after every other test has run.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from nadvibs_b200 import _lib as L
from nadvibs_b200 import synth

pytestmark = pytest.mark.gpu


def _handle():
    cfg = synth.config(4)
    om, cc, pot = synth.draw(cfg)
    p = L.default_params()
    p.nstates, p.nmodes, p.ordr = cfg.nstates, cfg.nmodes, cfg.ordr
    for i, b in enumerate(cfg.basis):
        p.basis[i] = b
    return L.Handle.from_arrays(p, om, cc, synth.flatten_pot(pot)), cfg.dimen * cfg.nstates


@pytest.mark.parametrize("dt", [torch.float64, torch.float32])
def test_dot_noalloc_matches_dot_on_two_calls(dt):
    h, n = _handle()
    code = L.DTYPE_F64 if dt == torch.float64 else L.DTYPE_F32
    with h:
        g = torch.Generator(device="cuda").manual_seed(11)
        a, b, c = (torch.randn(n, generator=g, device="cuda", dtype=dt) for _ in range(3))
        res = torch.zeros(2, device="cuda", dtype=torch.float64)
        stream = torch.cuda.current_stream().cuda_stream
        torch.cuda.synchronize()
        L.dot_noalloc(a.data_ptr(), b.data_ptr(), n, code, res[0:1].data_ptr(), stream, 0.5, 2.0)
        L.dot_noalloc(b.data_ptr(), c.data_ptr(), n, code, res[1:2].data_ptr(), stream, 1.0, 1.0)
        torch.cuda.synchronize()
        got = res.cpu().numpy()
        ref1 = h.dot_ptr(a.data_ptr(), b.data_ptr(), code, 0.5, 2.0)
        ref2 = h.dot_ptr(b.data_ptr(), c.data_ptr(), code, 1.0, 1.0)
        assert got[0] == pytest.approx(ref1, rel=1e-12, abs=1e-9)
        assert got[1] == pytest.approx(ref2, rel=1e-12, abs=1e-9)


def test_dot_noalloc_rejects_more_than_its_maximum():
    # rejected on the host before any launch; the pointers are never dereferenced
    dummy = torch.zeros(4, device="cuda", dtype=torch.float64)
    with pytest.raises(L.NvbError) as e:
        L.dot_noalloc(dummy.data_ptr(), dummy.data_ptr(), (1 << 32) + 1, L.DTYPE_F64, dummy.data_ptr())
    assert e.value.code == -1 and "maximum" in str(e.value)
