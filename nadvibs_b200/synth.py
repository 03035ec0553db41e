"""Seeded synthetic ``basis.in`` / ``nadvibs.in`` generator for the benchmark systems.

The reference ships no example input (its only example archive is missing), so every
benchmark and parity case is a seeded synthetic vibronic Hamiltonian written in the
reference's own file formats:

* ``basis.in`` is the ``&NADVIBS`` namelist read by ``get_keywords``
  (Source/secondary.f90:826-870).
* ``nadvibs.in`` is the list-directed coefficient file read by ``read_constants``
  (Source/top.f90:122-135): a comment line, the frequencies (hartree), then for every
  state block k=i(i-1)/2+j (i>=j, Source/top.f90:79-85) a comment, the constant, and per
  expansion order a comment and ``C(nmodes+d-1, d)`` coefficients in the monomial order of
  Source/top.f90:153-168 (k1>=k2>=...>=kd, first digit fastest).

Coefficients are drawn in dimensionless normal coordinates and cm^-1, then written in the
file convention ``c_file = c_dimless/AU2WAVE * prod(omega_k^(p_k/2))`` (omega in hartree),
which inverts the ``1/prod(omega^(p/2))`` scaling of Source/top.f90:216.

Choices recorded here (the benchmark descriptions leave them open):
* quadratic (and cubic) diagonal-block terms are drawn on ALL monomials of that degree;
* off-diagonal blocks carry only linear terms on the listed modes, constants and
  higher-order off-diagonal terms are 0 (so the lower-triangle-only constant coupling of
  the reference never fires for these systems);
* "gaps" are the diagonal constants of states 2.. relative to state 1;
* the random stream is ``numpy.random.default_rng(1000 + config_number)``.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field

import numpy as np

AU2WAVE = 219474.6313705  # Source/progdata.f90:7


def numut(n: int, d: int) -> int:
    """Number of degree-d monomials in n variables, C(n+d-1, d) (Source/function.f90:253-258)."""
    return math.comb(n + d - 1, d)


def monomials(nmodes: int, order: int) -> list[tuple[int, ...]]:
    """Monomials of one order in the file order of Source/top.f90:153-168.

    Returns tuples (k1, k2, ..., kd), 1-based, with k1 >= k2 >= ... >= kd.  The first digit
    runs fastest; when a digit passes ``nmodes`` it resets and carries, then every digit is
    raised to at least the value of the digit after it.
    """
    otab = [1] * order
    otab[0] = 0
    out = []
    for _ in range(numut(nmodes, order)):
        otab[0] += 1
        for l in range(order - 1):
            if otab[l] > nmodes:
                otab[l] = 1
                otab[l + 1] += 1
        for l in range(order - 2, -1, -1):
            if otab[l] < otab[l + 1]:
                otab[l] = otab[l + 1]
        out.append(tuple(otab))
    return out


@dataclass
class SynthConfig:
    name: str
    nstates: int
    basis: list[int]
    ordr: int
    gaps: list[float]                       # cm^-1, diagonal constants of states 1..nstates
    couplings: dict[tuple[int, int], list[int]]  # (i, j) i>j -> 1-based modes with linear coupling
    niter: int
    seed: int
    reorthog: int = 0
    chkorthog: int = 100
    lin_sigma: float = 200.0
    quad_sigma: float = 50.0
    cub_sigma: float = 10.0
    coup_sigma: float = 300.0
    omega_range: tuple[float, float] = (500.0, 3000.0)
    idroots: int = 0
    bconv: int = 0
    weights: list[float] | None = None
    extra: dict = field(default_factory=dict)

    @property
    def nmodes(self) -> int:
        return len(self.basis)

    @property
    def dimen(self) -> int:
        return int(np.prod(self.basis, dtype=np.int64))


def _cfg(n: int) -> SynthConfig:
    if n == 1:
        return SynthConfig("config1", 2, [8, 8, 6, 6], 2, [0.0, 1000.0], {(2, 1): [3, 4]}, 500, 1001)
    if n in (2, 3):
        return SynthConfig(f"config{n}", 3, [20, 16, 12, 10, 8, 8, 6, 6], 2, [0.0, 800.0, 1500.0],
                           {(2, 1): [1, 2, 3], (3, 1): [4, 5, 6], (3, 2): [6, 7, 8]},
                           2000, 1000 + n, reorthog=2 if n == 3 else 0, chkorthog=100)
    if n == 4:
        return SynthConfig("config4", 2, [14, 12, 10, 8, 8, 6], 2, [0.0, 1000.0], {(2, 1): [5, 6]},
                           400, 1004)
    if n == 5:
        return SynthConfig("config5", 3, [16, 14, 12, 10, 8, 8, 6, 6, 4, 4], 3, [0.0, 800.0, 1500.0],
                           {(2, 1): [1, 2, 3], (3, 1): [4, 5, 6], (3, 2): [6, 7, 8]}, 3000, 1005)
    raise ValueError(f"unknown benchmark system {n}")


def config(n: int) -> SynthConfig:
    """The five benchmark systems (1: CPU-size, 2/3: drop-in size, 4: gradient, 5: large cubic)."""
    return _cfg(n)


def draw(cfg: SynthConfig):
    """Draw (omega_hartree[M], concoef_file[nstblks], potterms_file[nstblks][ordr][numut]).

    Random draws happen in a fixed order: frequencies, then blocks in file order, then
    orders, then monomials in file order; a draw is made only where a coefficient is
    nonzero by construction.
    """
    rng = np.random.default_rng(cfg.seed)
    M, S = cfg.nmodes, cfg.nstates
    om_cm = rng.uniform(cfg.omega_range[0], cfg.omega_range[1], size=M)
    omega = om_cm / AU2WAVE
    nstblks = S * (S + 1) // 2
    concoef = np.zeros(nstblks)
    pot = []
    sig = {1: cfg.lin_sigma, 2: cfg.quad_sigma, 3: cfg.cub_sigma, 4: cfg.cub_sigma}
    for i in range(1, S + 1):
        for j in range(1, i + 1):
            k = i * (i - 1) // 2 + j
            diag = i == j
            concoef[k - 1] = (cfg.gaps[i - 1] / AU2WAVE) if diag else 0.0
            per_order = []
            for d in range(1, cfg.ordr + 1):
                mons = monomials(M, d)
                vals = np.zeros(len(mons))
                for t, mono in enumerate(mons):
                    if diag:
                        c = rng.normal(0.0, sig[d])
                    elif d == 1 and mono[0] in cfg.couplings.get((i, j), []):
                        c = rng.normal(0.0, cfg.coup_sigma)
                    else:
                        continue
                    scale = 1.0
                    for m in mono:
                        scale *= math.sqrt(omega[m - 1])
                    vals[t] = c / AU2WAVE * scale
                per_order.append(vals)
            pot.append(per_order)
    return omega, concoef, pot


def _fmt_vals(vals, per_line=4) -> str:
    lines = []
    for s in range(0, len(vals), per_line):
        lines.append(" " + " ".join(f"{float(v): .16E}" for v in vals[s:s + per_line]))
    if not lines:
        lines.append("")
    return "\n".join(lines) + "\n"


def write_nadvibs_in(path: str, nmodes: int, omega, concoef, pot, displaced=None) -> None:
    """Write ``nadvibs.in`` in the layout read by Source/top.f90:122-135; ``displaced`` =
    (bomega, dvec, tmat) appends the initial-state blocks read when shiftref != 0
    (Source/top.f90:130-134; tmat column-major, tmat[i*nmodes + k] = T[k, i])."""
    S_blocks = len(concoef)
    with open(path, "w") as f:
        f.write(" FREQUENCIES (hartree)\n")
        f.write(_fmt_vals(omega))
        for b in range(S_blocks):
            f.write(f" BLOCK {b + 1} CONSTANT\n")
            f.write(_fmt_vals([concoef[b]]))
            for d, vals in enumerate(pot[b], start=1):
                f.write(f" BLOCK {b + 1} ORDER {d}\n")
                f.write(_fmt_vals(vals))
        if displaced is not None:
            bomega, dvec, tmat = displaced
            f.write(" INITIAL-STATE FREQUENCIES (hartree)\n")
            f.write(_fmt_vals(bomega))
            f.write(" DISPLACEMENT\n")
            f.write(_fmt_vals(dvec))
            f.write(" DUSCHINSKY MATRIX (column-major)\n")
            f.write(_fmt_vals(tmat))


def write_basis_in(path: str, cfg: SynthConfig, niter: int | None = None, initstate=None, **over) -> None:
    """Write the ``&NADVIBS`` namelist (keys of Source/secondary.f90:844-845)."""
    kv = dict(niter=cfg.niter if niter is None else niter, natoms=max(2, (cfg.nmodes + 6) // 3),
              nmodes=cfg.nmodes, nstates=cfg.nstates, ordr=cfg.ordr, restart=0,
              bconv=cfg.bconv, idroots=cfg.idroots, soroots=0, reorthog=cfg.reorthog,
              chkorthog=cfg.chkorthog, nseg=1, shiftref=0, nirreps=1)
    kv.update(over)
    weights = cfg.weights if cfg.weights is not None else [1.0] * cfg.nstates
    with open(path, "w") as f:
        f.write(" &NADVIBS\n")
        for k, v in kv.items():
            f.write(f"  {k} = {v},\n")
        f.write("  basis = " + ", ".join(str(b) for b in cfg.basis) + ",\n")
        f.write("  npirr = " + str(cfg.nmodes) + ",\n")
        ist = [0] * cfg.nmodes if initstate is None else list(initstate)
        f.write("  initstate = " + ", ".join(str(int(v)) for v in ist) + ",\n")
        f.write("  weights = " + ", ".join(f"{w:.6f}" for w in weights) + "\n")
        f.write(" /\n")


def write_inputs(directory: str, cfg: SynthConfig, niter: int | None = None, **over) -> tuple[str, str]:
    """Write ``basis.in`` and ``nadvibs.in`` for ``cfg`` into ``directory``."""
    os.makedirs(directory, exist_ok=True)
    omega, concoef, pot = draw(cfg)
    b = os.path.join(directory, "basis.in")
    n = os.path.join(directory, "nadvibs.in")
    write_basis_in(b, cfg, niter=niter, **over)
    write_nadvibs_in(n, cfg.nmodes, omega, concoef, pot)
    return b, n


def random_small(seed: int, nstates: int, basis: list[int], ordr: int, dense: bool = True,
                 offdiag_even: bool = True, zero_frac: float = 0.3,
                 offdiag_bilinear: bool = True, offdiag_max_order: int | None = None) -> SynthConfig:
    """A tiny system for edge cases: every block may carry every order (incl. off-diagonal
    constants and even powers when ``offdiag_even``), with a fraction of exact zeros.
    ``offdiag_bilinear=False`` drops the off-diagonal monomials of two or more distinct modes
    (the vibronic-coupling form the factorised quadratic kernel accepts);
    ``offdiag_max_order=1`` keeps only constants and linear terms between different states
    (the form the factorised cubic kernel accepts)."""
    cfg = SynthConfig(f"small{seed}", nstates, list(basis), ordr, [0.0] * nstates, {}, 30, seed)
    cfg.extra = dict(dense=dense, offdiag_even=offdiag_even, zero_frac=zero_frac,
                     offdiag_bilinear=offdiag_bilinear, offdiag_max_order=offdiag_max_order)
    return cfg


def draw_small(cfg: SynthConfig):
    rng = np.random.default_rng(cfg.seed)
    M, S = cfg.nmodes, cfg.nstates
    omega = rng.uniform(500.0, 3000.0, size=M) / AU2WAVE
    nstblks = S * (S + 1) // 2
    concoef = np.zeros(nstblks)
    pot = []
    for i in range(1, S + 1):
        for j in range(1, i + 1):
            k = i * (i - 1) // 2 + j
            diag = i == j
            if diag or cfg.extra.get("offdiag_even", True):
                concoef[k - 1] = rng.normal(0.0, 500.0) / AU2WAVE
            per_order = []
            for d in range(1, cfg.ordr + 1):
                mons = monomials(M, d)
                vals = rng.normal(0.0, 200.0 / d, size=len(mons)) / AU2WAVE
                keep = rng.uniform(size=len(mons)) >= cfg.extra.get("zero_frac", 0.3)
                if not diag and not cfg.extra.get("offdiag_even", True) and d % 2 == 0:
                    keep[:] = False
                if not diag and not cfg.extra.get("offdiag_bilinear", True) and d >= 2:
                    keep &= np.array([len(set(mo)) == 1 for mo in mons])
                omax = cfg.extra.get("offdiag_max_order")
                if not diag and omax is not None and d > omax:
                    keep[:] = False
                vals = np.where(keep, vals, 0.0)
                for t, mono in enumerate(mons):
                    for m in mono:
                        vals[t] *= math.sqrt(omega[m - 1])
                per_order.append(vals)
            pot.append(per_order)
    return omega, concoef, pot


def flatten_pot(pot) -> np.ndarray:
    """Concatenate potterms as [block][order][monomial] (the in-memory layout of the C ABI)."""
    return np.concatenate([np.asarray(v, dtype=np.float64) for blk in pot for v in blk])
