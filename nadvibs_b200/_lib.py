"""ctypes binding of libnadvibs_gpu.so (the C ABI of include/nadvibs.h).

The library is built in-tree (``nadvibs_b200/libnadvibs_gpu.so``, see ``build.py``).  There is
no CPU fallback: if the library is missing, or no CUDA device is usable when a handle is
created, the call raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libnadvibs_gpu.so")

NVB_FP64, NVB_MIXED = 0, 1
DTYPE_F64, DTYPE_F32 = 0, 1

ERRORS = {-1: "NVB_ERR_ARG", -2: "NVB_ERR_IO", -3: "NVB_ERR_CUDA", -4: "NVB_ERR_STATE",
          -5: "NVB_ERR_NOMEM", -6: "NVB_ERR_BREAKDOWN"}


class NvbError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class Params(C.Structure):
    _fields_ = [(n, C.c_int64) for n in ("niter", "natoms", "nmodes", "nstates", "ordr", "restart", "bconv",
                                          "idroots", "soroots", "reorthog", "chkorthog", "nseg", "shiftref",
                                          "nirreps")] + \
               [("ztoler", C.c_double), ("maxdisk", C.c_double), ("basis", C.c_int64 * 100),
                ("initstate", C.c_int64 * 100), ("npirr", C.c_int64 * 10), ("weights", C.c_double * 10)]


class Options(C.Structure):
    _fields_ = [(n, C.c_int64) for n in ("precision", "device", "quirk_cubic", "quirk_lower", "archive_max",
                                          "hv_kernel", "seed")]


_lib = None

# (name, restype, argtypes); every entry point returns int status unless stated
_SIGS = {
    "nvb_params_default": [C.c_void_p],
    "nvb_options_default": [C.c_void_p],
    "nvb_read_basis": [C.c_char_p, C.c_void_p],
    "nvb_create_from_files": [C.c_char_p, C.c_char_p, C.c_void_p, C.c_void_p],
    "nvb_create": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p],
    "nvb_destroy": [C.c_void_p],
    "nvb_get_sizes": [C.c_void_p] + [C.c_void_p] * 6,
    "nvb_hv_kernel_in_use": [C.c_void_p, C.c_int64, C.c_void_p],
    "nvb_set_checkpoints": [C.c_void_p, C.c_int64],
    "nvb_set_archive": [C.c_void_p, C.c_int64, C.c_int64, C.c_char_p],
    "nvb_reorth_log": [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p],
    "nvb_reorth_omega": [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p],
    "nvb_measure_fma": [C.c_int64, C.c_double, C.c_void_p],
    "nvb_measure_tile_stream": [C.c_int64, C.c_int64, C.c_int64, C.c_double, C.c_void_p],
    "nvb_hv_tile_stream": [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p],
    "nvb_write_seed_report": [C.c_void_p, C.c_char_p],
    "nvb_set_fault_test": [C.c_void_p, C.c_int64],
    "nvb_set_displaced_seed": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p],
    "nvb_seed_overlap": [C.c_void_p, C.c_void_p],
    "nvb_convolve": [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_int64, C.c_double, C.c_int64, C.c_void_p],
    "nvb_spin_orbit": [C.c_void_p, C.c_int64, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, C.c_char_p],
    "nvb_lanczos_backward": [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p],
    "nvb_set_backward_memory": [C.c_void_p, C.c_int64],
    "nvb_backward_plan": [C.c_void_p, C.c_void_p],
    "nvb_get_terms": [C.c_void_p] + [C.c_void_p] * 7,
    "nvb_set_precision": [C.c_void_p, C.c_int64],
    "nvb_set_stream": [C.c_void_p, C.c_void_p],
    "nvb_synchronize": [C.c_void_p],
    "nvb_hv": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64],
    "nvb_seed": [C.c_void_p, C.c_void_p],
    "nvb_lanczos": [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p],
    "nvb_ritz": [C.c_void_p, C.c_int64] + [C.c_void_p] * 5,
    "nvb_write_eigenvalues": [C.c_void_p, C.c_char_p],
    "nvb_write_header": [C.c_void_p, C.c_char_p],
    "nvb_lanczos_vectors": [C.c_void_p] + [C.c_void_p] * 6,
    "nvb_set_timing": [C.c_void_p, C.c_int64],
    "nvb_save_restart": [C.c_void_p, C.c_char_p, C.c_char_p],
    "nvb_set_reorthog": [C.c_void_p, C.c_int64, C.c_int64],
    "nvb_hv_adjoint_coeffs": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p],
    "nvb_hellmann_feynman": [C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p],
    "nvb_load_restart": [C.c_void_p, C.c_char_p, C.c_char_p],
    "nvb_lead_contributors": [C.c_void_p, C.c_int64, C.c_int64] + [C.c_void_p] * 6,
    "nvb_dot": [C.c_void_p, C.c_void_p, C.c_double, C.c_void_p, C.c_double, C.c_int64, C.c_void_p],
    "nvb_dot_noalloc": [C.c_void_p, C.c_double, C.c_void_p, C.c_double, C.c_int64, C.c_int64, C.c_void_p, C.c_void_p],
    "nvb_get_timing": [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p],
}


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is not built: run `python -m nadvibs_b200.build` "
                              "(there is no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, args in _SIGS.items():
            fn = getattr(L, name, None)
            if fn is None:
                continue
            fn.restype = C.c_int
            fn.argtypes = args
        L.nvb_last_error.restype = C.c_char_p
        L.nvb_last_error.argtypes = []
        _lib = L
    return _lib


def check(rc: int) -> None:
    if rc != 0:
        raise NvbError(rc, lib().nvb_last_error().decode(errors="replace"))


def _p(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def dot_noalloc(a_ptr: int, b_ptr: int, n: int, dtype: int, result_ptr: int, stream_ptr: int = 0,
                sa: float = 1.0, sb: float = 1.0) -> None:
    """nvb_dot_noalloc: <sa*a, sb*b> written to the device double at result_ptr (no allocation)."""
    check(lib().nvb_dot_noalloc(C.c_void_p(a_ptr), sa, C.c_void_p(b_ptr), sb, n, dtype, C.c_void_p(result_ptr),
                                C.c_void_p(stream_ptr) if stream_ptr else None))


def measure_fma(dtype: int, seconds: float = 2.0) -> float:
    """nvb_measure_fma: FMA throughput of the current device (flop/s, 2 per FMA)."""
    r = C.c_double()
    check(lib().nvb_measure_fma(dtype, seconds, C.byref(r)))
    return r.value


def measure_tile_stream(tile_bytes: int, slots: int = 8, ctas_per_sm: int = 1, seconds: float = 1.0) -> float:
    """nvb_measure_tile_stream: bytes/s of whole tiles streamed from L2 into a shared-memory ring."""
    r = C.c_double()
    check(lib().nvb_measure_tile_stream(tile_bytes, slots, ctas_per_sm, seconds, C.byref(r)))
    return r.value


SHAPE_FWHM_GAUSSIAN, SHAPE_GAUSSIAN, SHAPE_LORENTZIAN = 0, 1, 2


def convolve(center, height, grid, width: float, shape: int = SHAPE_FWHM_GAUSSIAN) -> np.ndarray:
    """nvb_convolve: broadened line spectrum on grid (GPU, FP64)."""
    c = np.ascontiguousarray(center, dtype=np.float64)
    h = np.ascontiguousarray(height, dtype=np.float64)
    g = np.ascontiguousarray(grid, dtype=np.float64)
    if c.shape != h.shape:
        raise ValueError("center and height differ in length")
    out = np.zeros(g.size)
    check(lib().nvb_convolve(_p(c), _p(h), c.size, _p(g), g.size, float(width), int(shape), _p(out)))
    return out


def default_params() -> Params:
    p = Params()
    check(lib().nvb_params_default(C.byref(p)))
    return p


def default_options(**kw) -> Options:
    o = Options()
    check(lib().nvb_options_default(C.byref(o)))
    for k, v in kw.items():
        setattr(o, k, int(v))
    return o


def read_basis(path: str) -> Params:
    p = Params()
    check(lib().nvb_read_basis(path.encode(), C.byref(p)))
    return p


class Handle:
    """Owns one nvb_handle."""

    def __init__(self, ptr):
        self.ptr = ptr

    @classmethod
    def from_files(cls, basis: str, nadvibs: str, **opts) -> "Handle":
        o = default_options(**opts)
        h = C.c_void_p()
        check(lib().nvb_create_from_files(basis.encode(), nadvibs.encode(), C.byref(o), C.byref(h)))
        return cls(h)

    @classmethod
    def from_arrays(cls, params: Params, omega, concoef, potterms, **opts) -> "Handle":
        o = default_options(**opts)
        om = np.ascontiguousarray(omega, dtype=np.float64)
        cc = np.ascontiguousarray(concoef, dtype=np.float64)
        pt = np.ascontiguousarray(potterms, dtype=np.float64)
        h = C.c_void_p()
        check(lib().nvb_create(C.byref(params), _p(om), _p(cc), _p(pt), C.byref(o), C.byref(h)))
        return cls(h)

    def close(self):
        if self.ptr:
            lib().nvb_destroy(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def sizes(self) -> dict:
        v = [C.c_int64() for _ in range(6)]
        check(lib().nvb_get_sizes(self.ptr, *[C.byref(x) for x in v]))
        return dict(zip(("dimen", "nstates", "nmodes", "nterms", "npot", "iters"), [x.value for x in v]))

    def hv_tile_stream(self, dtype: int = DTYPE_F64) -> dict:
        """nvb_hv_tile_stream: the factorised H.v's neighbour-tile stream (bytes per product,
        tile bytes, ring slots, CTAs per multiprocessor); zeros for the slab / gather kernels."""
        b = C.c_double()
        v = [C.c_int64() for _ in range(3)]
        check(lib().nvb_hv_tile_stream(self.ptr, dtype, C.byref(b), *[C.byref(x) for x in v]))
        return {"bytes_per_hv": b.value, "tile_bytes": v[0].value, "slots": v[1].value, "ctas_per_sm": v[2].value}

    def hv_kernel(self, dtype: int = DTYPE_F64) -> str:
        """Name of the H.v kernel products of this dtype run: gather, slab, quad or cubic."""
        k = C.c_int64()
        check(lib().nvb_hv_kernel_in_use(self.ptr, dtype, C.byref(k)))
        return {1: "gather", 2: "slab", 3: "quad", 4: "cubic"}[k.value]

    def terms(self):
        sz = self.sizes()
        nt, S = sz["nterms"], sz["nstates"]
        tcnt = np.zeros(max(nt, 1), np.int64)
        tmode = np.zeros((max(nt, 1), 4), np.int64)
        tpow = np.zeros((max(nt, 1), 4), np.int64)
        tnp = np.zeros(max(nt, 1), np.int64)
        tpa = np.zeros((max(nt, 1), S * S), np.int64)
        tpb = np.zeros((max(nt, 1), S * S), np.int64)
        tco = np.zeros((max(nt, 1), S * S))
        check(lib().nvb_get_terms(self.ptr, _p(tcnt), _p(tmode), _p(tpow), _p(tnp), _p(tpa), _p(tpb), _p(tco)))
        out = []
        for t in range(nt):
            c = int(tcnt[t])
            out.append(dict(modes=list(tmode[t, :c]), pows=list(tpow[t, :c]),
                            pairs=[(int(tpa[t, q]), int(tpb[t, q])) for q in range(tnp[t])],
                            coefs=list(tco[t, : tnp[t]])))
        return out

    def set_precision(self, prec: int):
        check(lib().nvb_set_precision(self.ptr, prec))

    def set_stream(self, stream_ptr: int | None):
        """Run on a caller stream (a cudaStream_t as int).  0 means the legacy default stream
        (passed as cudaStreamLegacy); None restores the handle's own stream."""
        if stream_ptr is None:
            check(lib().nvb_set_stream(self.ptr, None))
        else:
            check(lib().nvb_set_stream(self.ptr, C.c_void_p(stream_ptr if stream_ptr else 1)))

    def synchronize(self):
        check(lib().nvb_synchronize(self.ptr))

    def hv_ptr(self, x_ptr: int, y_ptr: int, dtype: int):
        check(lib().nvb_hv(self.ptr, C.c_void_p(x_ptr), C.c_void_p(y_ptr), dtype))

    def seed(self, weights=None):
        w = None if weights is None else np.ascontiguousarray(weights, dtype=np.float64)
        check(lib().nvb_seed(self.ptr, _p(w)))

    def lanczos(self, niter: int):
        it = self.sizes()["iters"] + niter
        a = np.zeros(max(it, 1))
        b = np.zeros(it + 1)
        rc = lib().nvb_lanczos(self.ptr, niter, _p(a), _p(b))
        check(rc)
        return a[:it], b

    def ritz(self, n: int, vectors: bool = False):
        E = np.zeros(n); bji = np.zeros(n); inten = np.zeros(n)
        sign = np.zeros(n, np.int64)
        V = np.zeros((n, n)) if vectors else None
        check(lib().nvb_ritz(self.ptr, n, _p(E), _p(bji), _p(inten), _p(sign), _p(V)))
        return E, bji, inten, sign, (V.T.copy() if vectors else None)

    def write_header(self, path: str):
        check(lib().nvb_write_header(self.ptr, path.encode()))

    def write_eigenvalues(self, path: str):
        check(lib().nvb_write_eigenvalues(self.ptr, path.encode()))

    def lanczos_vectors(self):
        p = [C.c_void_p() for _ in range(3)]
        s = [C.c_double() for _ in range(3)]
        check(lib().nvb_lanczos_vectors(self.ptr, C.byref(p[0]), C.byref(s[0]), C.byref(p[1]), C.byref(s[1]),
                                        C.byref(p[2]), C.byref(s[2])))
        return [(p[i].value, s[i].value) for i in range(3)]

    def set_timing(self, enable: bool = True):
        check(lib().nvb_set_timing(self.ptr, int(enable)))

    def timing(self):
        a, b, n = C.c_double(), C.c_double(), C.c_int64()
        check(lib().nvb_get_timing(self.ptr, C.byref(a), C.byref(b), C.byref(n)))
        return a.value, b.value, n.value

    def dot_ptr(self, a_ptr: int, b_ptr: int, dtype: int, sa: float = 1.0, sb: float = 1.0) -> float:
        r = C.c_double()
        check(lib().nvb_dot(self.ptr, C.c_void_p(a_ptr), sa, C.c_void_p(b_ptr), sb, dtype, C.byref(r)))
        return r.value

    def save_restart(self, directory: str, vecdir: str | None = None):
        check(lib().nvb_save_restart(self.ptr, directory.encode(), vecdir.encode() if vecdir else None))

    def load_restart(self, directory: str, vecdir: str | None = None):
        check(lib().nvb_load_restart(self.ptr, directory.encode(), vecdir.encode() if vecdir else None))

    def lead_contributors(self, nroots: int, k: int, rootinfo: str | None = None):
        S = self.sizes()["nstates"]
        st = np.zeros(max(nroots * k, 1), np.int64); ix = np.zeros(max(nroots * k, 1), np.int64)
        c2 = np.zeros(max(nroots * k, 1)); ph = np.zeros(max(nroots * k, 1), np.int64)
        pct = np.zeros(nroots * S)
        check(lib().nvb_lead_contributors(self.ptr, nroots, k, _p(st), _p(ix), _p(c2), _p(ph), _p(pct),
                                          rootinfo.encode() if rootinfo else None))
        n = nroots * k
        return dict(state=st[:n].reshape(nroots, k), index=ix[:n].reshape(nroots, k),
                    c2=c2[:n].reshape(nroots, k), phase=ph[:n].reshape(nroots, k), pct=pct.reshape(nroots, S))

    def write_seed_report(self, path: str):
        """Append the seed section of output.dat (nvb_write_seed_report)."""
        check(lib().nvb_write_seed_report(self.ptr, path.encode()))

    def set_reorthog(self, reorthog: int, chkorthog: int = 100):
        check(lib().nvb_set_reorthog(self.ptr, reorthog, chkorthog))

    ARCHIVE_DEVICE, ARCHIVE_HOST, ARCHIVE_FILE = 0, 1, 2

    def set_archive(self, kind: int, max_vectors: int, path: str | None = None):
        """Where the Lanczos-vector archive lives from the next seed (nvb_set_archive): 0 device
        memory, 1 pinned host memory, 2 a file at path in the reference's nadvibs.34 layout."""
        check(lib().nvb_set_archive(self.ptr, kind, max_vectors, path.encode() if path else None))

    def reorth_omega(self, n: int):
        """(omega1[0..n], omega2[0..n], omega2 of the last step before its resets) (nvb_reorth_omega)."""
        w1, w2, w3 = (np.zeros(n + 1) for _ in range(3))
        check(lib().nvb_reorth_omega(self.ptr, n, _p(w1), _p(w2), _p(w3)))
        return w1, w2, w3

    def reorth_log(self) -> np.ndarray:
        """(iteration, lo, hi) of every interval partial re-orthogonalisation used (nvb_reorth_log)."""
        n = C.c_int64()
        check(lib().nvb_reorth_log(self.ptr, 0, None, None, None, C.byref(n)))
        it, lo, hi = (np.zeros(max(n.value, 1), dtype=np.int64) for _ in range(3))
        check(lib().nvb_reorth_log(self.ptr, n.value, _p(it), _p(lo), _p(hi), C.byref(n)))
        return np.stack([it[:n.value], lo[:n.value], hi[:n.value]], axis=1)

    def ncoef(self) -> int:
        sz = self.sizes()
        S = sz["nstates"]
        return sz["npot"] + S * (S + 1) // 2 + sz["nmodes"]

    def adjoint_ptr(self, u_ptr: int, v_ptr: int, dtype: int) -> np.ndarray:
        g = np.zeros(self.ncoef())
        check(lib().nvb_hv_adjoint_coeffs(self.ptr, C.c_void_p(u_ptr), C.c_void_p(v_ptr), dtype, _p(g)))
        return g

    def spin_orbit(self, soroots: int, nroots: int | None = None, path: str | None = None) -> dict:
        """nvb_spin_orbit: energies (eV), sqrt(I/Imax)*sign and state-block overlaps of the lowest
        soroots Ritz vectors; writes sodata.in to path when given."""
        nroots = soroots if nroots is None else nroots
        S = self.sizes()["nstates"]
        e, amp = np.zeros(soroots), np.zeros(soroots)
        ov = np.zeros((soroots, soroots, S, S))
        check(lib().nvb_spin_orbit(self.ptr, soroots, nroots, _p(e), _p(amp), _p(ov),
                                   None if path is None else path.encode()))
        return dict(energy_ev=e, amp=amp, overlap=ov)

    def set_displaced_seed(self, bomega, dvec, tmat):
        """nvb_set_displaced_seed: initial-state frequencies, displacement, Duschinsky matrix
        (column-major flat, tmat[i*nmodes + k] = T[k, i])."""
        b = np.ascontiguousarray(bomega, dtype=np.float64)
        d = np.ascontiguousarray(dvec, dtype=np.float64)
        t = np.ascontiguousarray(tmat, dtype=np.float64).reshape(-1)
        check(lib().nvb_set_displaced_seed(self.ptr, _p(b), _p(d), _p(t)))

    def seed_overlap(self) -> float:
        v = C.c_double()
        check(lib().nvb_seed_overlap(self.ptr, C.byref(v)))
        return v.value

    def set_fault_test(self, mode: int):
        """nvb_set_fault_test: 1 = the quadratic H.v kernel issues no copies (its waits run out)."""
        check(lib().nvb_set_fault_test(self.ptr, mode))

    def set_checkpoints(self, k: int):
        """Record (v_{c-1}, v_c) every k iterations from the next seed (nvb_set_checkpoints);
        k = -1 records the whole forward when it fits the backward budget."""
        check(lib().nvb_set_checkpoints(self.ptr, k))

    def set_backward_memory(self, nbytes: int):
        """Device-memory budget of the automatic (k = 0) reverse sweep; 0 = 85% of free memory."""
        check(lib().nvb_set_backward_memory(self.ptr, int(nbytes)))

    def backward_plan(self) -> dict:
        """The last reverse sweep's plan (nvb_backward_plan)."""
        a = np.zeros(4, dtype=np.int64)
        check(lib().nvb_backward_plan(self.ptr, _p(a)))
        return {"top_interval": int(a[0]), "branching": int(a[1]), "stored_range": int(a[2]),
                "replayed_hv": int(a[3])}

    def lanczos_backward(self, n: int, alpha_bar, beta_bar=None, k: int = 0) -> np.ndarray:
        """dL/dtheta from dL/dalpha_1..n and dL/dbeta_1..n (nvb_lanczos_backward); k = 0 picks
        the checkpoint recursion from the memory budget, k > 0 is one level of interval k."""
        ab = np.ascontiguousarray(alpha_bar, dtype=np.float64)
        if ab.shape != (n,):
            raise ValueError("alpha_bar must have n entries")
        bb = None if beta_bar is None else np.ascontiguousarray(beta_bar, dtype=np.float64)
        if bb is not None and bb.shape != (n,):
            raise ValueError("beta_bar must have n entries")
        g = np.zeros(self.ncoef())
        check(lib().nvb_lanczos_backward(self.ptr, n, _p(ab), None if bb is None else _p(bb), k, _p(g)))
        return g

    def hellmann_feynman(self, nroots: int):
        g = np.zeros((nroots, self.ncoef()))
        e = np.zeros(nroots)
        check(lib().nvb_hellmann_feynman(self.ptr, nroots, _p(g), _p(e)))
        return e, g
