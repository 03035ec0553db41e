"""ORACLE (test infrastructure only) -- Python side of the CPU restatement.

Loads ``oracle/_build/liboracle.so`` (built from ``nvb_oracle.c`` by :func:`build`) and
exposes the reference-semantics H.v, Lanczos recurrence, GIVENS tridiagonal solve and the
output-table formatting.  Used only by tests/, ``__graft_entry__.smoke()`` and
``bench.py``'s CPU baseline / reference arm, as the checker.  Parity status: UNPINNED
against the reference (no Fortran toolchain here, no reference outputs for this path);
see the header of ``nvb_oracle.c``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from . import termcomp as tc

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")
SRC = os.path.join(HERE, "nvb_oracle.c")

AU2WAVE = 219474.6313705  # Source/progdata.f90:7
AU2EV = 27.211384523      # Source/progdata.f90:8


def build(force: bool = False) -> str:
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(SRC):
        subprocess.check_call(["gcc", "-O2", "-fopenmp", "-fPIC", "-shared", "-std=c11",
                               "-ffp-contract=off", SRC, "-o", LIB, "-lm"])
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        _lib = C.CDLL(LIB)
        _lib.orc_hoelem.restype = C.c_double
        _lib.orc_hoelem.argtypes = [C.c_int64] * 4
        _lib.orc_dimen.restype = C.c_int64
    return _lib


class _Sys(C.Structure):
    _fields_ = [("nstates", C.c_int64), ("nmodes", C.c_int64), ("ordr", C.c_int64),
                ("nterms", C.c_int64), ("maxpairs", C.c_int64),
                ("nfunc", C.c_void_p), ("omega", C.c_void_p), ("concoef", C.c_void_p),
                ("tcnt", C.c_void_p), ("tmode", C.c_void_p), ("tpow", C.c_void_p),
                ("tnpair", C.c_void_p), ("tpa", C.c_void_p), ("tpb", C.c_void_p),
                ("tcoef", C.c_void_p), ("quirk_cubic", C.c_int64), ("quirk_lower", C.c_int64)]


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


class OracleSystem:
    """A compiled term table held in the reference's representation."""

    def __init__(self, nfunc, omega, concoef, tt: tc.TermTable, nstates: int, ordr: int,
                 quirk_cubic: bool = True, quirk_lower: bool = True):
        self.nfunc = np.ascontiguousarray(nfunc, dtype=np.int64)
        self.omega = np.ascontiguousarray(omega, dtype=np.float64)
        self.concoef = np.ascontiguousarray(concoef, dtype=np.float64)
        self.tt = tt
        self.nstates, self.ordr = nstates, ordr
        nt = tt.nterms
        mp = max(1, nstates * nstates)
        self.tcnt = np.array([len(m) for m in tt.modes] or [0], dtype=np.int64)
        self.tmode = np.zeros((max(nt, 1), ordr), dtype=np.int64)
        self.tpow = np.zeros((max(nt, 1), ordr), dtype=np.int64)
        self.tnpair = np.zeros(max(nt, 1), dtype=np.int64)
        self.tpa = np.zeros((max(nt, 1), mp), dtype=np.int64)
        self.tpb = np.zeros((max(nt, 1), mp), dtype=np.int64)
        self.tcoef = np.zeros((max(nt, 1), mp), dtype=np.float64)
        for t in range(nt):
            for l, (m, p) in enumerate(zip(tt.modes[t], tt.pows[t])):
                self.tmode[t, l] = m
                self.tpow[t, l] = p
            self.tnpair[t] = len(tt.pairs[t])
            for q, ((a, b), c) in enumerate(zip(tt.pairs[t], tt.coefs[t])):
                self.tpa[t, q], self.tpb[t, q], self.tcoef[t, q] = a, b, c
        self.s = _Sys(nstates, len(self.nfunc), ordr, nt, mp, _p(self.nfunc), _p(self.omega),
                      _p(self.concoef), _p(self.tcnt), _p(self.tmode), _p(self.tpow),
                      _p(self.tnpair), _p(self.tpa), _p(self.tpb), _p(self.tcoef),
                      int(quirk_cubic), int(quirk_lower))

    @property
    def dimen(self) -> int:
        return int(np.prod(self.nfunc, dtype=np.int64))

    @property
    def ntotal(self) -> int:
        return self.dimen * self.nstates

    def hv(self, x: np.ndarray, nthreads: int = 1, rowdiv: bool = False) -> np.ndarray:
        """y = H x.  rowdiv=True decodes every row's digits by division in every pass instead
        of walking them with the incremental counter (same result, bit for bit)."""
        x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1)
        assert x.size == self.ntotal
        y = np.empty_like(x)
        fn = lib().orc_hv_rowdiv if rowdiv else lib().orc_hv
        rc = fn(C.byref(self.s), _p(x), _p(y), C.c_int(nthreads))
        if rc:
            raise RuntimeError(f"orc_hv failed {rc}")
        return y

    def hv_rows(self, x: np.ndarray, rows) -> np.ndarray:
        """(H x) at the given rows for all states: array [len(rows), nstates]."""
        x = np.ascontiguousarray(x, dtype=np.float64).reshape(-1)
        assert x.size == self.ntotal
        r = np.ascontiguousarray(rows, dtype=np.int64)
        y = np.zeros((len(r), self.nstates))
        rc = lib().orc_hv_rows(C.byref(self.s), _p(x), _p(r), C.c_int64(len(r)), _p(y))
        if rc:
            raise RuntimeError(f"orc_hv_rows failed {rc}")
        return y

    def lanczos(self, niter: int, weights=None, keep_vectors: bool = False, nthreads: int = 1):
        w = np.ascontiguousarray(weights if weights is not None else np.ones(self.nstates), dtype=np.float64)
        alpha = np.zeros(niter)
        beta = np.zeros(niter + 1)
        vecs = np.zeros((niter, self.ntotal)) if keep_vectors else None
        qf = np.zeros(3 * self.ntotal)
        rc = lib().orc_lanczos(C.byref(self.s), _p(w), C.c_int64(niter), _p(alpha), _p(beta),
                               _p(vecs) if vecs is not None else None, _p(qf), C.c_int(nthreads))
        if rc:
            raise RuntimeError(f"orc_lanczos failed {rc}")
        return alpha, beta, vecs, qf.reshape(3, -1)

    def dense(self) -> np.ndarray:
        """Dense H (columns H e_j), small systems only."""
        n = self.ntotal
        H = np.zeros((n, n))
        e = np.zeros(n)
        for j in range(n):
            e[:] = 0.0
            e[j] = 1.0
            H[:, j] = self.hv(e)
        return H


def system_from_files(basis_path: str, nadvibs_path: str, quirk_cubic=True, quirk_lower=True):
    with open(basis_path) as f:
        kv = tc.read_namelist(f.read())
    with open(nadvibs_path) as f:
        om, cc, pot, _ = tc.read_nadvibs(f.read(), kv["nmodes"], kv["nstates"], kv["ordr"], kv["neworigin"])
    tt = tc.compile_terms(kv["nmodes"], kv["nstates"], kv["ordr"], om, cc, pot, kv["ztoler"])
    return kv, OracleSystem(kv["nfunc"], om, cc, tt, kv["nstates"], kv["ordr"], quirk_cubic, quirk_lower)


def system_from_arrays(nfunc, nstates, ordr, omega, concoef, pot, ztoler=1e-20, quirk_cubic=True,
                       quirk_lower=True) -> OracleSystem:
    tt = tc.compile_terms(len(nfunc), nstates, ordr, omega, concoef, pot, ztoler)
    return OracleSystem(nfunc, omega, concoef, tt, nstates, ordr, quirk_cubic, quirk_lower)


def hoelem(p: int, a: int, b: int, quirk_cubic: bool = True) -> float:
    return lib().orc_hoelem(p, a, b, int(quirk_cubic))


def givens_tridiag(alpha: np.ndarray, beta_codiag: np.ndarray, nroot: int | None = None):
    n = len(alpha)
    nroot = n if nroot is None else nroot
    a = np.ascontiguousarray(alpha, dtype=np.float64)
    b = np.ascontiguousarray(beta_codiag, dtype=np.float64)
    if b.size == 0:
        b = np.zeros(1)
    root = np.zeros(nroot)
    vect = np.zeros((nroot, n))
    rc = lib().orc_givens_tridiag(C.c_int64(n), _p(a), _p(b), C.c_int64(nroot), _p(root), _p(vect))
    if rc:
        raise RuntimeError("givens failed")
    return root, vect.T.copy()   # vect[:, i] eigenvector i


def ritz(alpha: np.ndarray, beta: np.ndarray):
    """compute_ritzsystem (Source/secondary.f90:240-257): (E, bji, intensity, sign, vectors)."""
    n = len(alpha)
    E = np.zeros(n); bji = np.zeros(n); inten = np.zeros(n)
    sign = np.zeros(n, dtype=np.int64)
    vect = np.zeros((n, n))
    a = np.ascontiguousarray(alpha, dtype=np.float64)
    b = np.ascontiguousarray(beta[: n + 1], dtype=np.float64)
    rc = lib().orc_ritz(C.c_int64(n), _p(a), _p(b), _p(E), _p(bji), _p(inten), _p(sign), _p(vect))
    if rc:
        raise RuntimeError("ritz failed")
    return E, bji, inten, sign, vect.T.copy()


def eigen_table(alpha, beta, omega, bjiconv: float):
    """The root filter and table of compute_eigenvalues (Source/top.f90:1051-1113).
    Returns (zpve_cm, first_cm, intensity_factor, rows) with rows of
    (root, index, bji, E_cm_rel, E_eV_rel, I_rel)."""
    E, bji, inten, sign, _ = ritz(alpha, beta)
    n = len(E)
    good = [1]
    thresh = 0.0
    for i in range(2, n + 1):
        if bji[i - 1] < bjiconv:
            g = good[-1]
            if AU2WAVE * abs(E[i - 1] - E[g - 1]) < thresh:  # never true with thresh=0
                inten[g - 1] += inten[i - 1]
                if bji[i - 1] < bji[g - 1]:
                    inten[i - 1] = inten[g - 1]
                    good[-1] = i
            else:
                good.append(i)
    zpve = sum(0.5 * w for w in omega) * AU2WAVE
    first = E[good[0] - 1] * AU2WAVE
    fac = 0.0
    for g in good:
        if inten[g - 1] > fac:
            fac = inten[g - 1]
    rows = []
    for k, g in enumerate(good, start=1):
        rows.append((k, g, bji[g - 1], (E[g - 1] - E[good[0] - 1]) * AU2WAVE, (E[g - 1] - E[0]) * AU2EV,
                     inten[g - 1] / fac))
    return zpve, first, fac, rows


def _real4(v: float) -> float:
    """A default-REAL Fortran literal assigned to a real*8 variable keeps single precision."""
    return float(np.float32(v))


def convolve_fwhm(c, h, xstart=_real4(-0.1), xend=_real4(0.4), nt=2000, fwhm=5e-3, eshift=_real4(2.7807)):
    """convolve/main.f90:24-43: xstart, xend and eshift are default-REAL literals there
    (single precision), fwhm=5.d-3 is double."""
    c = np.ascontiguousarray(c, dtype=np.float64)
    h = np.ascontiguousarray(h, dtype=np.float64)
    xo = np.zeros(nt + 2)
    yo = np.zeros(nt + 2)
    lib().orc_convolve_fwhm(C.c_int64(len(c)), _p(c), _p(h), C.c_double(xstart), C.c_double(xend),
                            C.c_int64(nt), C.c_double(fwhm), C.c_double(eshift), _p(xo), _p(yo))
    return xo, yo


def convolve_sigma(x, y, sigma, grid, aperture="Gaussian"):
    """convolve.py:28-48: Gaussian exp(-((g-x)/sigma)^2/2) or Lorentzian, normalised to max."""
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    env = np.zeros(len(grid))
    for i, g in enumerate(grid):
        t = (g - x) / sigma
        if aperture == "Gaussian":
            env[i] = np.sum(y * np.exp(-0.5 * t * t))
        else:
            env[i] = np.sum(y * (1.0 / sigma / (1.0 + t * t)))
    return env / np.max(env)


# ---------------------------------------------------------------- output.dat text
def _I(v: int, w: int) -> str:
    s = str(int(v))
    return "*" * w if len(s) > w else s.rjust(w)


def _F(v: float, w: int, d: int) -> str:
    s = f"{v:.{d}f}"
    return "*" * w if len(s) > w else s.rjust(w)


def _ES(v: float, w: int, d: int) -> str:
    m, e = f"{v:.{d}E}".split("E")
    ex = int(e)
    s = f"{m}E{ex:+03d}" if abs(ex) < 100 else f"{m}{ex:+04d}"
    return "*" * w if len(s) > w else s.rjust(w)


def eigen_table_lines(alpha, beta, omega, bjiconv: float):
    """The text of compute_eigenvalues (Source/top.f90:1095-1112) from ZPVE to the last row."""
    zpve, first, fac, rows = eigen_table(alpha, beta, omega, bjiconv)
    out = [f"  ZPVE from nadvibs.in (reference state): {_F(zpve, 12, 4)} cm-1",
           f"  FIRST eigenvalue:                       {_F(first, 12, 4)} cm-1",
           f"  Intensity Factor (MAX Intensity):       {_F(fac, 12, 8)}",
           "  Root  Index  Convergence     E(cm-1)        E(eV)     Intensity"]
    for k, g, b, ecm, eev, it in rows:
        out.append(_I(k, 6) + _I(g, 7) + _ES(b, 13, 4) + _F(ecm, 15, 5) + _F(eev, 12, 5) + _F(it, 12, 7))
    return out


def sodata_lines(E, inten, sign, psi, soroots: int, nroots: int, nstates: int):
    """The text of sodata.in (Source/top.f90:1153-1175, 1231-1252, formats 1001-1005 and
    1013-1014) from the Ritz values/intensities/signs of T_n and the Ritz vectors psi[i]
    (flat, state blocks of equal length): root lines, then for i > j the overlaps of state
    block k of psi_i with state block l of psi_j, k != l, k outer."""
    fac = max(inten[:nroots])
    out = [_I(soroots, 5), " Root   Energy (eV)      Sqrt(Int.)*sign"]
    for i in range(soroots):
        out.append(_I(i + 1, 5) + "  " + _ES(E[i] * AU2EV, 15, 8) + "  " + _ES(np.sqrt(inten[i] / fac) * sign[i], 15, 8))
    if nstates == 2:
        out.append(" R(i)  R(j)   [S1(i)S2(j)]   [S2(i)S1(j)]")
    if nstates == 3:
        out += [" R(i)  R(j)   [S1(i)S2(j)]   [S1(i)S3(j)]  [S2(i)S1(j)]",
                " R(i)  R(j)   [S2(i)S3(j)]   [S3(i)S1(j)]  [S3(i)S2(j)]"]
    if nstates in (2, 3):
        for i in range(1, soroots):
            blk_i = np.asarray(psi[i]).reshape(nstates, -1)
            for j in range(i):
                blk_j = np.asarray(psi[j]).reshape(nstates, -1)
                dp = [float(blk_i[k] @ blk_j[l]) for k in range(nstates) for l in range(nstates) if k != l]
                head = _I(i + 1, 5) + " " + _I(j + 1, 5) + "  "
                if nstates == 2:
                    out.append(head + _ES(dp[0], 14, 6) + " " + _ES(dp[1], 14, 6))
                else:
                    out.append(head + " ".join(_ES(x, 14, 6) for x in dp[:3]))
                    out.append(head + " ".join(_ES(x, 14, 6) for x in dp[3:]))
    return out


def extract_spectrum(path: str, threshold: float = 1e-15):
    """extract.py:22-50: (E_eV, I, convergence) rows of output.dat's table with convergence <
    threshold and I != 0, in table order."""
    with open(path) as f:
        lines = f.readlines()
    start = stop = None
    for i, l in enumerate(lines):
        if "Root  Index  Convergence     E(cm-1)        E(eV)     Intensity" in l:
            start = i + 1
        if "All requested eigenvalues computed." in l:
            stop = i - 1
            break
    out = []
    for l in lines[start:stop]:
        t = l.split()
        c, x, y = float(t[2]), float(t[4]), float(t[5])
        if c < threshold and y != 0:
            out.append((x, y, c))
    return out
