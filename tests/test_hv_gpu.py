"""H.v parity through the C ABI on the GPU against the CPU oracle (Source/top.f90:672-818).

FP64: max |y_gpu - y_oracle| <= 1e-12 * max |y| (same summation order per element; only
FMA contraction and the rounding of the element products differ).
FP32: max |y_gpu - y_oracle| <= 2e-5 * max |y| (single-precision evaluation).
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from nadvibs_b200 import _lib as L
from nadvibs_b200 import synth
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL64 = 1e-12
TOL32 = 2e-5


def _handle(p_or_cfg, om, cc, pot, **opts):
    return L.Handle.from_arrays(p_or_cfg, om, cc, synth.flatten_pot(pot), **opts)


def _params(cfg):
    p = L.default_params()
    p.nstates, p.nmodes, p.ordr = cfg.nstates, cfg.nmodes, cfg.ordr
    for i, b in enumerate(cfg.basis):
        p.basis[i] = b
    p.niter = cfg.niter
    return p


def _hv_gpu(h, x: np.ndarray, dtype=torch.float64):
    xt = torch.from_numpy(x).to(device="cuda", dtype=dtype)
    yt = torch.empty_like(xt)
    h.set_stream(torch.cuda.current_stream().cuda_stream)
    h.hv_ptr(xt.data_ptr(), yt.data_ptr(), L.DTYPE_F64 if dtype == torch.float64 else L.DTYPE_F32)
    torch.cuda.synchronize()
    return yt.double().cpu().numpy()


SMALL = [(7, 2, [3, 4], 2), (8, 3, [2, 3, 2], 3), (9, 2, [4, 1, 3], 4), (10, 1, [5, 4], 4),
         (12, 4, [3, 3, 2, 2], 2), (13, 2, [1, 1], 2), (14, 10, [2, 3], 2), (15, 3, [6, 5, 4], 4),
         (16, 5, [2, 2, 2, 2, 2, 2], 3)]


@pytest.mark.parametrize("seed,nstates,basis,ordr", SMALL)
@pytest.mark.parametrize("quirks", [(1, 1), (0, 0)])
def test_hv_small_systems_fp64_and_fp32(seed, nstates, basis, ordr, quirks):
    cfg = synth.random_small(seed, nstates, basis, ordr)
    om, cc, pot = synth.draw_small(cfg)
    S = O.system_from_arrays(basis, nstates, ordr, om, cc, pot, quirk_cubic=bool(quirks[0]),
                             quirk_lower=bool(quirks[1]))
    x = np.random.default_rng(seed).normal(size=S.ntotal)
    y_ref = S.hv(x)
    with _handle(_params(cfg), om, cc, pot, quirk_cubic=quirks[0], quirk_lower=quirks[1]) as h:
        y64 = _hv_gpu(h, x)
        y32 = _hv_gpu(h, x, torch.float32)
    scale = np.abs(y_ref).max()
    assert np.abs(y64 - y_ref).max() <= TOL64 * scale
    assert np.abs(y32 - y_ref).max() <= TOL32 * scale


MEDIUM = [(31, 1, [8, 8, 6, 6, 6, 4], 2), (32, 2, [8, 6, 8, 6, 6, 4], 3), (33, 3, [10, 8, 6, 4, 4, 4], 2),
          (34, 4, [10, 8, 4, 4, 4, 4], 4), (35, 3, [12, 10, 8, 8, 6, 6], 2)]


@pytest.mark.parametrize("seed,nstates,basis,ordr", MEDIUM)
@pytest.mark.parametrize("quirks", [(1, 1), (0, 0)])
def test_hv_slab_kernel_matches_oracle(seed, nstates, basis, ordr, quirks):
    """Systems large enough for the slab-tiled kernel (hv_kernel=2 forces it; creation fails
    if the system does not suit it), against the oracle and the gather kernel."""
    cfg = synth.random_small(seed, nstates, basis, ordr)
    om, cc, pot = synth.draw_small(cfg)
    S = O.system_from_arrays(basis, nstates, ordr, om, cc, pot, quirk_cubic=bool(quirks[0]),
                             quirk_lower=bool(quirks[1]))
    x = np.random.default_rng(seed).normal(size=S.ntotal)
    y_ref = S.hv(x, nthreads=8)
    scale = np.abs(y_ref).max()
    with _handle(_params(cfg), om, cc, pot, quirk_cubic=quirks[0], quirk_lower=quirks[1], hv_kernel=2) as h:
        y64 = _hv_gpu(h, x)
        y32 = _hv_gpu(h, x, torch.float32)
    with _handle(_params(cfg), om, cc, pot, quirk_cubic=quirks[0], quirk_lower=quirks[1], hv_kernel=1) as hg:
        g64 = _hv_gpu(hg, x)
    assert np.abs(g64 - y_ref).max() <= TOL64 * scale
    assert np.abs(y64 - y_ref).max() <= TOL64 * scale
    assert np.abs(y32 - y_ref).max() <= TOL32 * scale


QUAD = [(61, 1, [4, 3, 5, 4, 8, 8]), (62, 2, [3, 3, 3, 2, 4, 8, 4]), (63, 3, [6, 5, 4, 8, 8]),
        (64, 4, [5, 4, 4, 2, 8, 4]), (65, 3, [5, 4, 8, 8, 4, 2])]


@pytest.mark.parametrize("seed,nstates,basis", QUAD)
@pytest.mark.parametrize("quirks", [(1, 1), (0, 0)])
def test_hv_quadratic_kernel_matches_oracle(seed, nstates, basis, quirks):
    """Quadratic systems with state-diagonal bilinear terms (off-diagonal blocks: constants,
    linear terms and squares) through the factorised kernel (hv_kernel=3 forces it; creation
    fails if the system does not suit it), against the oracle and the gather kernel.  The
    bases put 1-3 modes on the slow side, pencils of 2-8 rows and 2-level modes."""
    cfg = synth.random_small(seed, nstates, basis, 2, offdiag_bilinear=False)
    om, cc, pot = synth.draw_small(cfg)
    S = O.system_from_arrays(basis, nstates, 2, om, cc, pot, quirk_cubic=bool(quirks[0]),
                             quirk_lower=bool(quirks[1]))
    x = np.random.default_rng(seed).normal(size=S.ntotal)
    y_ref = S.hv(x, nthreads=8)
    scale = np.abs(y_ref).max()
    with _handle(_params(cfg), om, cc, pot, quirk_cubic=quirks[0], quirk_lower=quirks[1], hv_kernel=3) as h:
        y64 = _hv_gpu(h, x)
        y32 = _hv_gpu(h, x, torch.float32)
    with _handle(_params(cfg), om, cc, pot, quirk_cubic=quirks[0], quirk_lower=quirks[1], hv_kernel=1) as hg:
        g64 = _hv_gpu(hg, x)
    assert np.abs(g64 - y_ref).max() <= TOL64 * scale
    assert np.abs(y64 - y_ref).max() <= TOL64 * scale
    assert np.abs(y32 - y_ref).max() <= TOL32 * scale


def test_hv_quadratic_kernel_rejects_unsuited_systems():
    """Bilinear inter-state couplings, cubic terms or a basis without a 32-aligned pencil
    stride cannot use the factorised kernel: forcing it fails at creation."""
    for basis, ordr, bil in [([4, 3, 5, 4, 8, 8], 2, True), ([4, 3, 5, 4, 8, 8], 3, False),
                             ([8, 8, 6, 6], 2, False)]:
        cfg = synth.random_small(66, 2, basis, ordr, offdiag_bilinear=bil, zero_frac=0.0)
        om, cc, pot = synth.draw_small(cfg)
        with pytest.raises(L.NvbError):
            _handle(_params(cfg), om, cc, pot, hv_kernel=3).close()


@pytest.mark.parametrize("n", [1, 4])
def test_hv_benchmark_systems_full(n):
    cfg = synth.config(n)
    om, cc, pot = synth.draw(cfg)
    S = O.system_from_arrays(cfg.basis, cfg.nstates, cfg.ordr, om, cc, pot)
    x = np.random.default_rng(n).normal(size=S.ntotal)
    y_ref = S.hv(x, nthreads=8)
    with _handle(_params(cfg), om, cc, pot) as h:
        y64 = _hv_gpu(h, x)
        y32 = _hv_gpu(h, x, torch.float32)
    scale = np.abs(y_ref).max()
    assert np.abs(y64 - y_ref).max() <= TOL64 * scale
    assert np.abs(y32 - y_ref).max() <= TOL32 * scale


@pytest.mark.parametrize("n", [2])
@pytest.mark.parametrize("dt", [torch.float64, torch.float32])
def test_hv_drop_in_size_rows_and_symmetry(n, dt):
    """Full-size systems through the benchmark's kernel in both precisions: oracle rows at 2000
    random positions (plus the first/last rows and the truncation corners) of H x for the
    same (FP32-rounded, for FP32) x, and <u,Hv> = <Hu,v> over the whole vector."""
    cfg = synth.config(n)
    om, cc, pot = synth.draw(cfg)
    S = O.system_from_arrays(cfg.basis, cfg.nstates, cfg.ordr, om, cc, pot)
    N = S.dimen
    code = L.DTYPE_F64 if dt == torch.float64 else L.DTYPE_F32
    tol = TOL64 if dt == torch.float64 else TOL32
    g = torch.Generator(device="cuda").manual_seed(n)
    x = torch.randn(S.ntotal, generator=g, device="cuda", dtype=dt)
    u = torch.randn(S.ntotal, generator=g, device="cuda", dtype=dt)
    with _handle(_params(cfg), om, cc, pot) as h:
        assert h.hv_kernel(code) == "quad"
        h.set_stream(torch.cuda.current_stream().cuda_stream)
        y = torch.empty_like(x)
        h.hv_ptr(x.data_ptr(), y.data_ptr(), code)
        hu = torch.empty_like(u)
        h.hv_ptr(u.data_ptr(), hu.data_ptr(), code)
        torch.cuda.synchronize()
        lhs = torch.dot(u.double(), y.double()).item()
        rhs = torch.dot(hu.double(), x.double()).item()
        sym_tol = 1e-10 if dt == torch.float64 else 1e-5
        assert abs(lhs - rhs) <= sym_tol * torch.linalg.vector_norm(y.double()).item() * \
            torch.linalg.vector_norm(u.double()).item()
        rng = np.random.default_rng(n)
        rows = np.concatenate([[0, 1, N - 2, N - 1], rng.integers(0, N, size=2000)])
        xh = x.double().cpu().numpy()
        yr = S.hv_rows(xh, rows)
        yg = y.view(cfg.nstates, N).double().cpu().numpy()[:, rows].T
        assert np.abs(yg - yr).max() <= tol * np.abs(yr).max()
