"""The factorised cubic H.v kernel (hv_kernel=4) against the CPU oracle (Source/top.f90:672-818,
elements Source/function.f90:186-250 with both settings of the x^3 quirk).

Systems of order 3 whose couplings between different states are constants and linear terms
(the form of the large benchmark system).  The bases put 1-3 modes on the slow side, 2-5 fast
modes, pencils of 2-9 rows, 1- and 2-function modes, and pencils of 64..576 threads (above 288
threads the kernel runs FP32 only and FP64 falls back to another kernel).
FP64: max |y - y_oracle| <= 1e-12 max |y|; FP32: <= 2e-5 max |y|.
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

# (seed, states, basis): fast modes / slow modes / pencil threads in the comments
CUBIC = [(71, 2, [10, 8, 64]),                 # 2 fast, 1 slow, 64 threads
         (72, 3, [6, 9, 8, 8, 8]),             # 3 fast, 2 slow
         (73, 1, [5, 4, 9, 8, 4, 4, 4]),       # 4 fast, 3 slow
         (74, 4, [4, 3, 3, 2, 8, 4, 2, 2]),    # 5 fast, 3 slow, 4 states, 2-function modes
         (75, 2, [5, 3, 4, 2, 2, 8, 2, 2]),    # 5 fast, 3 slow, 64 threads
         (76, 3, [6, 5, 4, 4, 4, 2, 2]),       # 5 fast, 2 slow
         (77, 2, [2, 1, 9, 8, 8, 8])]          # 3 fast, slow modes of 2, 1 and 9 functions
WIDE = [(78, 2, [5, 4, 4, 8, 4, 3, 4]),        # 384 threads: FP32 only
        (79, 3, [3, 2, 4, 3, 8, 6, 6, 4, 4])]  # 576 threads, 3 states, 5 fast: the benchmark shape


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


def _system(seed, nstates, basis, quirks):
    cfg = synth.random_small(seed, nstates, basis, 3, offdiag_max_order=1)
    om, cc, pot = synth.draw_small(cfg)
    S = O.system_from_arrays(basis, nstates, 3, om, cc, pot, quirk_cubic=bool(quirks[0]),
                             quirk_lower=bool(quirks[1]))
    return cfg, om, cc, pot, S


@pytest.mark.parametrize("seed,nstates,basis", CUBIC)
@pytest.mark.parametrize("quirks", [(1, 1), (0, 0)])
def test_hv_cubic_kernel_matches_oracle(seed, nstates, basis, quirks):
    cfg, om, cc, pot, S = _system(seed, nstates, basis, quirks)
    x = np.random.default_rng(seed).normal(size=S.ntotal)
    y_ref = S.hv(x, nthreads=8)
    scale = np.abs(y_ref).max()
    with L.Handle.from_arrays(_params(cfg), om, cc, synth.flatten_pot(pot), quirk_cubic=quirks[0],
                              quirk_lower=quirks[1], hv_kernel=4) as h:
        assert h.hv_kernel(L.DTYPE_F64) == "cubic" and h.hv_kernel(L.DTYPE_F32) == "cubic"
        y64 = _hv_gpu(h, x)
        y32 = _hv_gpu(h, x, torch.float32)
    assert np.abs(y64 - y_ref).max() <= TOL64 * scale
    assert np.abs(y32 - y_ref).max() <= TOL32 * scale


@pytest.mark.parametrize("seed,nstates,basis", WIDE)
@pytest.mark.parametrize("quirks", [(1, 1), (0, 0)])
def test_hv_cubic_kernel_wide_pencils_fp32(seed, nstates, basis, quirks):
    cfg, om, cc, pot, S = _system(seed, nstates, basis, quirks)
    x = np.random.default_rng(seed).normal(size=S.ntotal)
    y_ref = S.hv(x, nthreads=8)
    scale = np.abs(y_ref).max()
    with L.Handle.from_arrays(_params(cfg), om, cc, synth.flatten_pot(pot), quirk_cubic=quirks[0],
                              quirk_lower=quirks[1]) as h:
        assert h.hv_kernel(L.DTYPE_F32) == "cubic"
        assert h.hv_kernel(L.DTYPE_F64) != "cubic"
        y32 = _hv_gpu(h, x, torch.float32)
        y64 = _hv_gpu(h, x)
    assert np.abs(y32 - y_ref).max() <= TOL32 * scale
    assert np.abs(y64 - y_ref).max() <= TOL64 * scale


def test_hv_cubic_kernel_rejects_unsuited_systems():
    """Quadratic couplings between different states, or a basis without a 32-aligned pencil
    stride, cannot use the cubic kernel: forcing it fails at creation."""
    for basis, omax in [([6, 9, 8, 8, 8], 2), ([8, 8, 6, 6], 1)]:
        cfg = synth.random_small(80, 2, basis, 3, offdiag_max_order=omax, zero_frac=0.0)
        om, cc, pot = synth.draw_small(cfg)
        with pytest.raises(L.NvbError):
            L.Handle.from_arrays(_params(cfg), om, cc, synth.flatten_pot(pot), hv_kernel=4).close()


def test_hv_cubic_lanczos_matches_oracle():
    """Twenty FP64 Lanczos steps through the cubic kernel (alpha fused into its epilogue)."""
    cfg, om, cc, pot, S = _system(74, 4, [4, 3, 3, 2, 8, 4, 2, 2], (1, 1))
    with L.Handle.from_arrays(_params(cfg), om, cc, synth.flatten_pot(pot), hv_kernel=4) as h:
        h.seed()
        a, b = h.lanczos(20)
    ao, bo, _, _ = S.lanczos(20)
    np.testing.assert_allclose(a, ao, rtol=1e-10, atol=0)
    np.testing.assert_allclose(b, bo[:21], rtol=1e-10, atol=0)


@pytest.mark.parametrize("basis", [[4, 4, 6, 5, 8, 8, 6, 6, 4, 4], None])
def test_hv_cubic_benchmark_system_rows_and_symmetry(basis):
    """Config 5's Hamiltonian through the cubic kernel in FP32, on a reduced basis and at the
    literal size (2.97e9 elements, 11.9 GB per vector): oracle rows at 1000 random positions
    (plus the first and last rows) of H x for the same FP32-rounded x, and <u,Hx> = <Hu,x>
    over the whole vector."""
    cfg = synth.config(5)
    if basis is not None:
        cfg.basis = basis
    om, cc, pot = synth.draw(cfg)
    S = O.system_from_arrays(cfg.basis, cfg.nstates, cfg.ordr, om, cc, pot)
    N = S.dimen
    g = torch.Generator(device="cuda").manual_seed(5)
    x = torch.randn(S.ntotal, generator=g, device="cuda", dtype=torch.float32)
    u = torch.randn(S.ntotal, generator=g, device="cuda", dtype=torch.float32)
    with L.Handle.from_arrays(_params(cfg), om, cc, synth.flatten_pot(pot), precision=L.NVB_MIXED) as h:
        assert h.hv_kernel(L.DTYPE_F32) == "cubic"
        h.set_stream(torch.cuda.current_stream().cuda_stream)
        y = torch.empty_like(x)
        h.hv_ptr(x.data_ptr(), y.data_ptr(), L.DTYPE_F32)
        hu = torch.empty_like(u)
        h.hv_ptr(u.data_ptr(), hu.data_ptr(), L.DTYPE_F32)
        torch.cuda.synchronize()
    def dot(a, b):  # FP64 dot product in chunks (one torch.dot takes at most 2^31 elements)
        c = 1 << 28
        return sum(torch.dot(a[i:i + c].double(), b[i:i + c].double()).item() for i in range(0, a.numel(), c))

    lhs, rhs = dot(u, y), dot(hu, x)
    assert abs(lhs - rhs) <= 1e-5 * np.sqrt(dot(y, y) * dot(u, u))
    del hu, u
    rng = np.random.default_rng(5)
    rows = np.concatenate([[0, N - 1], rng.integers(0, N, size=1000)])
    xh = x.cpu().numpy().astype(np.float64)
    yr = S.hv_rows(xh, rows)
    idx = torch.from_numpy(rows).to("cuda")
    yg = y.view(cfg.nstates, N)[:, idx].double().cpu().numpy().T
    assert np.abs(yg - yr).max() <= TOL32 * np.abs(yr).max()
