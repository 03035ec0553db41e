"""Spectrum post-step of the Lanczos stage: the line spectrum of ``output.dat`` and its
broadening, in place of the reference's helper programs.

* :func:`extract` -- the filter of ``extract.py`` (lines 22-50): rows of the eigenvalue table
  whose convergence is below a threshold and whose intensity is non-zero, as (E/eV, I).
* :func:`convolve_fwhm` -- ``convolve/main.f90`` (lines 24-43): Gaussians of FWHM 5e-3 eV on
  2002 points from -0.1 to 0.4 eV, shifted by 2.7807 eV (its default-REAL literals kept as
  single-precision values), computed on the GPU (``nvb_convolve``).
* :func:`convolve` -- ``convolve.py`` (lines 28-48): Gaussian or Lorentzian of width sigma on a
  given grid, normalised to its maximum, on the GPU.
The differentiable broadening used by the gradient path is
``nadvibs_b200.autograd.convolved_spectrum``.
"""
from __future__ import annotations

import numpy as np

from . import _lib as L

TABLE_HEAD = "Root  Index  Convergence     E(cm-1)        E(eV)     Intensity"
TABLE_END = "All requested eigenvalues computed."


def _fortran_float(s: str) -> float:
    """A number as Fortran prints it, including ES fields whose three-digit exponent drops the
    letter (1.0227-321); extract.py's float() fails on those."""
    try:
        return float(s)
    except ValueError:
        for i in range(len(s) - 1, 0, -1):
            if s[i] in "+-" and s[i - 1] not in "eEdD":
                return float(s[:i] + "E" + s[i:])
        raise


def extract(output_dat: str, threshold: float = 1e-15, invert: bool = False,
            shift_maximum: float | None = None):
    """(E_eV, intensity, convergence) arrays of the table rows that pass the filter."""
    with open(output_dat) as f:
        lines = f.readlines()
    first = last = None
    for i, line in enumerate(lines):
        if TABLE_HEAD in line:
            first = i + 1
        if TABLE_END in line:
            last = i - 1  # the table ends one line above the closing message
            break
    if first is None or last is None:
        raise ValueError(f"{output_dat}: no eigenvalue table")
    rows = [line.split() for line in lines[first:last]]
    conv = np.array([_fortran_float(r[2]) for r in rows])
    x = np.array([float(r[4]) for r in rows])
    y = np.array([float(r[5]) for r in rows])
    if invert:
        x = -x
    if shift_maximum is not None and len(y):
        x = x + (shift_maximum - x[np.argmax(y)])
    keep = (conv < threshold) & (y != 0)
    return x[keep], y[keep], conv[keep]


def write_lines(path: str, x, y) -> None:
    """spectrum.txt in extract.py's format ("%12.5f%12.7f")."""
    with open(path, "w") as f:
        for a, b in zip(x, y):
            f.write("%12.5f%12.7f\n" % (a, b))


def fortran_grid(xstart: float = float(np.float32(-0.1)), xend: float = float(np.float32(0.4)), nt: int = 2000):
    """The grid of convolve/main.f90: x_i = xstart + i (xend - xstart)/(nt + 1), i = 0..nt+1."""
    dx = (xend - xstart) / float(nt + 1)
    return xstart + np.arange(nt + 2, dtype=np.float64) * dx


def convolve_fwhm(center, height, fwhm: float = 5e-3, grid=None, eshift: float = float(np.float32(2.7807))):
    """(x + eshift, y) of convolve/main.f90 for lines (center, height) in eV."""
    g = fortran_grid() if grid is None else np.asarray(grid, dtype=np.float64)
    y = L.convolve(center, height, g, fwhm, L.SHAPE_FWHM_GAUSSIAN)
    return g + eshift, y


def convolve(center, height, grid, sigma: float, aperture: str = "Gaussian"):
    """convolve.py's envelope: Gaussian or Lorentzian of width sigma, divided by its maximum."""
    shape = {"Gaussian": L.SHAPE_GAUSSIAN, "Lorentzian": L.SHAPE_LORENTZIAN}[aperture]
    env = L.convolve(center, height, grid, sigma, shape)
    return env / env.max()
