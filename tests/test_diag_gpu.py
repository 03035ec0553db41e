"""Measured ceilings (FMA throughput, neighbour-tile stream) and the factorised kernels'
tile-stream accounting."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from nadvibs_b200 import _lib as L
from nadvibs_b200 import synth

pytestmark = pytest.mark.gpu


def _params(cfg):
    p = L.default_params()
    p.nstates, p.nmodes, p.ordr = cfg.nstates, cfg.nmodes, cfg.ordr
    for i, b in enumerate(cfg.basis):
        p.basis[i] = b
    p.niter = cfg.niter
    return p


def test_measured_ceilings_are_plausible():
    f64 = L.measure_fma(L.DTYPE_F64, 0.2)
    f32 = L.measure_fma(L.DTYPE_F32, 0.2)
    assert 1e12 < f64 < f32 < 1e15
    ts = L.measure_tile_stream(18432, 8, 1, 0.2)
    assert 1e12 < ts < 1e14  # bytes/s: between 1 and 100 TB/s
    with pytest.raises(L.NvbError):
        L.measure_tile_stream(18433, 8, 1, 0.1)  # not a multiple of 16


@pytest.mark.parametrize("kind", ["quad", "cubic"])
def test_hv_tile_stream_counts_items_inside_the_basis(kind):
    """Bytes per product = sum over items of the tiles whose neighbour lies inside the basis:
    at least the own tiles of every state, at most every item on every tile."""
    if kind == "quad":
        cfg = synth.random_small(63, 3, [6, 5, 4, 8, 8], 2, offdiag_bilinear=False)
    else:
        cfg = synth.random_small(72, 3, [6, 9, 8, 8, 8], 3, offdiag_max_order=1)
    om, cc, pot = synth.draw_small(cfg)
    with L.Handle.from_arrays(_params(cfg), om, cc, synth.flatten_pot(pot)) as h:
        assert h.hv_kernel(L.DTYPE_F64) == kind
        n = int(np.prod(cfg.basis)) * cfg.nstates
        x = torch.randn(n, device="cuda", dtype=torch.float64)
        y = torch.empty_like(x)
        h.set_stream(torch.cuda.current_stream().cuda_stream)
        h.hv_ptr(x.data_ptr(), y.data_ptr(), L.DTYPE_F64)
        torch.cuda.synchronize()
        ts = h.hv_tile_stream(L.DTYPE_F64)
    tiles = n // (ts["tile_bytes"] // 8)  # state-tiles
    assert ts["tile_bytes"] % 16 == 0 and ts["slots"] >= 3 and ts["ctas_per_sm"] >= 1
    assert ts["bytes_per_hv"] >= tiles * ts["tile_bytes"]
    assert ts["bytes_per_hv"] <= tiles * ts["tile_bytes"] * 4096
