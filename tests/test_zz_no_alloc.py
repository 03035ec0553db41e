"""The allocation-free inner product, nvb_dot_noalloc, through the C ABI.

Callers that cannot allocate device memory (their GPU memory is owned by their own pool
allocator, or their loop must not call cudaMalloc/cudaFree, which may synchronise the device)
use nvb_dot_noalloc: its block partials live in a static device array of the library.  Here
it runs twice in a row, on different inputs, and each result is compared with nvb_dot (the
handle-based product, whose partials are in cudaMalloc'd scratch) within the FP64 tolerance
used by the other dot-product tests (1e-12 relative); further cases cover n = 0, sizes just
around the grid's block boundaries, a vector spread over every partial of the static array,
a non-default stream, and its bandwidth against torch.dot on the same vectors.  This file is collected
last so that a failure here stops a -x run only after every other test has run.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from nadvibs_b200 import _lib as L
from nadvibs_b200 import synth

pytestmark = pytest.mark.gpu


def _handle(n_cfg=4):
    cfg = synth.config(n_cfg)
    om, cc, pot = synth.draw(cfg)
    p = L.default_params()
    p.nstates, p.nmodes, p.ordr = cfg.nstates, cfg.nmodes, cfg.ordr
    for i, b in enumerate(cfg.basis):
        p.basis[i] = b
    return L.Handle.from_arrays(p, om, cc, synth.flatten_pot(pot)), cfg.dimen * cfg.nstates


def _code(dt):
    return L.DTYPE_F64 if dt == torch.float64 else L.DTYPE_F32


@pytest.mark.parametrize("dt", [torch.float64, torch.float32])
def test_dot_noalloc_matches_dot_on_two_calls(dt):
    h, n = _handle()
    code = _code(dt)
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


# n = 0 (only the final reduction runs, writing 0), sizes around the block boundaries of the
# grid (1,024 elements per block at the smallest grain, 1,184 blocks at most on 148
# multiprocessors) and a size that uses every block many times over
SIZES = [0, 1, 1023, 1024, 1025, 1024 * 1184 - 1, 1024 * 1184 + 1, 37_000_003]


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("dt", [torch.float64, torch.float32])
def test_dot_noalloc_sizes_against_float64(n, dt):
    g = torch.Generator(device="cuda").manual_seed(n % 1000 + 3)
    a = torch.randn(max(n, 1), generator=g, device="cuda", dtype=dt)
    b = torch.randn(max(n, 1), generator=g, device="cuda", dtype=dt)
    res = torch.full((2,), 123.0, device="cuda", dtype=torch.float64)
    s = torch.cuda.Stream()  # a non-default stream
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        for i in range(2):  # two calls in a row: the second reuses what the first left in the array
            L.dot_noalloc(a.data_ptr(), b.data_ptr(), n, _code(dt), res[i:i + 1].data_ptr(), s.cuda_stream,
                          1.0, 0.25)
    s.synchronize()
    ref = 0.25 * torch.dot(a[:n].double(), b[:n].double()).item() if n else 0.0
    tol = 1e-12 * max(1.0, float(torch.linalg.vector_norm(a[:n].double()) * torch.linalg.vector_norm(b[:n].double())))
    got = res.cpu().numpy()
    assert abs(got[0] - ref) <= tol and got[1] == got[0]


def test_dot_noalloc_bandwidth_close_to_dot():
    """Device time per call within a factor 1.5 of torch.dot's on the same vectors, large
    enough to stream from HBM (64 Mi FP64 elements, 1 GiB for both inputs)."""
    n = 1 << 26
    g = torch.Generator(device="cuda").manual_seed(5)
    a = torch.randn(n, generator=g, device="cuda", dtype=torch.float64)
    b = torch.randn(n, generator=g, device="cuda", dtype=torch.float64)
    res = torch.zeros(1, device="cuda", dtype=torch.float64)
    st = torch.cuda.current_stream()
    for _ in range(3):
        L.dot_noalloc(a.data_ptr(), b.data_ptr(), n, L.DTYPE_F64, res.data_ptr(), st.cuda_stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(10):
        L.dot_noalloc(a.data_ptr(), b.data_ptr(), n, L.DTYPE_F64, res.data_ptr(), st.cuda_stream)
    e1.record(st)
    torch.cuda.synchronize()
    t_na = e0.elapsed_time(e1) / 10
    e0.record(st)
    for _ in range(10):
        torch.dot(a, b)
    e1.record(st)
    torch.cuda.synchronize()
    t_lib = e0.elapsed_time(e1) / 10
    gbs = 2 * 8 * n / (t_na * 1e-3) / 1e9
    assert t_na <= 1.5 * t_lib, f"noalloc {t_na:.3f} ms ({gbs:.0f} GB/s) vs torch.dot {t_lib:.3f} ms"


def test_dot_noalloc_rejects_more_than_its_maximum():
    # rejected on the host before any launch; the pointers are never dereferenced
    dummy = torch.zeros(4, device="cuda", dtype=torch.float64)
    with pytest.raises(L.NvbError) as e:
        L.dot_noalloc(dummy.data_ptr(), dummy.data_ptr(), (1 << 32) + 1, L.DTYPE_F64, dummy.data_ptr())
    assert e.value.code == -1 and "maximum" in str(e.value)
