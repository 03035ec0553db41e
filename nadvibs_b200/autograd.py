"""Gradients of Lanczos Ritz energies, Franck-Condon intensities and convolved spectra with
respect to the Hamiltonian's inputs (no counterpart in the reference, which has no derivative
code).

``theta`` is the flat vector of ``nadvibs.in`` inputs in the layout of
``nvb_hv_adjoint_coeffs``: the expansion coefficients (file layout [block][order][monomial],
file units), the block constants, then the frequencies (hartree).

Forward: a handle is built from ``theta`` (``nvb_create``), seeded as the reference seeds
(``Source/secondary.f90:727-783``), run for ``niter`` plain Lanczos iterations (recording
checkpoint pairs every ``k`` iterations when k > 0), and T_n = tridiag(beta, alpha, beta) is
diagonalised:
Ritz energies E_i (hartree) and intensities I_i = s_{1,i}^2 (the squared first component of
eigenvector i, the Franck-Condon weight of the seed, ``Source/secondary.f90:240-257``).

Backward: the eigen-derivatives of the symmetric tridiagonal give dL/dalpha_i and
dL/dbeta_i,
    Tbar = S (diag(Ebar) + F o (S^T Sbar)) S^T,   F_ij = 1/(E_j - E_i) (i != j),
with Sbar = e_1 (2 s_1 Ibar)^T; pairs of nearly equal Ritz values (ghost copies of a
converged root) are damped, F_ij = d/(d^2 + eps^2).  Then ``nvb_lanczos_backward`` runs the
reverse sweep through the recurrence on the GPU and contracts the adjoint vectors with
dH/dtheta.  The primal vectors come from the forward: with k = -1 (the default) the forward
records every v_j and H v_j when they fit the device-memory budget
(``Handle.set_backward_memory``) and the sweep replays nothing; otherwise they are recomputed
from checkpoint pairs: with k > 0 one level every k iterations; with k = 0 (or -1 without the
record) the shallowest recursive checkpointing that fits the budget.

Losses: after a long plain-Lanczos run the unconverged Ritz values are chaotic functions of
theta at the scale of rounding (ghost copies form as roots converge), so a loss over all Ritz
values has no finite-difference limit.  ``ritz(..., residuals=True)`` also returns the
residual estimates bji; ``converged_mask`` / ``converged_spectrum`` restrict a loss to the
converged roots (ghost copies included), a smooth function of theta whose reverse-sweep
gradient agrees with central differences.
"""
from __future__ import annotations

import numpy as np
import torch
from scipy.linalg import eigh_tridiagonal

from . import _lib as L

AU2WAVE = 219474.6313705  # Source/progdata.f90:7


def split_theta(theta: np.ndarray, nstates: int, nmodes: int):
    """(potterms, concoef, omega) views of a flat theta."""
    nb = nstates * (nstates + 1) // 2
    npot = theta.size - nb - nmodes
    if npot < 0:
        raise ValueError("theta is shorter than concoef + omega")
    return theta[:npot], theta[npot:npot + nb], theta[npot + nb:]


def tridiag_eigh(alpha: np.ndarray, beta_off: np.ndarray):
    """All eigenpairs of the symmetric tridiagonal T (ascending), LAPACK."""
    return eigh_tridiagonal(alpha, beta_off)


def tridiag_eig_backward(E: np.ndarray, S: np.ndarray, gE: np.ndarray | None, gI: np.ndarray | None,
                         eps_rel: float = 1e-10, device=None):
    """dL/dalpha (n) and dL/dbeta_1..n-1 (n-1) from dL/dE and dL/dI, I_i = S[0, i]^2.

    Only the diagonal and the first off-diagonal of Tbar = S M S^T are formed (one n^3 product,
    S M, then row-wise dot products with S).  With `device` a CUDA device the product runs there
    in FP64 (torch); the results come back as numpy arrays either way."""
    n = E.size
    inner = np.zeros((n, n))
    if gE is not None:
        inner[np.diag_indices(n)] += gE
    if gI is not None:
        sbar0 = 2.0 * S[0, :] * gI                     # Sbar[0, i]; other rows of Sbar are zero
        ssb = np.outer(S[0, :], sbar0)                 # (S^T Sbar)[j, i] = S[0, j] Sbar[0, i]
        d = E[None, :] - E[:, None]                    # d[i, j] = E_j - E_i
        eps = eps_rel * max(1.0, float(np.abs(E).max()))
        F = d / (d * d + eps * eps)
        np.fill_diagonal(F, 0.0)
        inner += F * ssb
    if device is not None and torch.device(device).type == "cuda":
        St = torch.from_numpy(np.ascontiguousarray(S)).to(device)
        SM = St @ torch.from_numpy(inner).to(device)
        diag = (SM * St).sum(dim=1)
        up = (SM[:-1] * St[1:]).sum(dim=1)             # Tbar[i, i+1]
        lo = (SM[1:] * St[:-1]).sum(dim=1)             # Tbar[i+1, i]
        abar = diag.cpu().numpy()
        bbar = (up + lo).cpu().numpy()                 # 2 * symmetrised off-diagonal
        return abar, bbar
    SM = S @ inner
    abar = np.einsum("ij,ij->i", SM, S)
    bbar = np.einsum("ij,ij->i", SM[:-1], S[1:]) + np.einsum("ij,ij->i", SM[1:], S[:-1])
    return abar, bbar


class LanczosRitz(torch.autograd.Function):
    """(E, I, bji) = Ritz energies, intensities and residual estimates |beta_n s_{n,i}| of niter
    Lanczos steps on H(theta); bji is not differentiable (it selects converged roots)."""

    @staticmethod
    def forward(ctx, theta: torch.Tensor, params, niter: int, k: int, opts: dict):
        th = theta.detach().to("cpu", torch.float64).numpy().copy()
        pot, cc, om = split_theta(th, int(params.nstates), int(params.nmodes))
        h = L.Handle.from_arrays(params, om, cc, pot, **opts)
        try:
            h.set_checkpoints(k)
            h.seed()
            a, b = h.lanczos(niter)
        except Exception:
            h.close()
            raise
        E, S = tridiag_eigh(a[:niter], b[1:niter])
        ctx.h, ctx.niter, ctx.k = h, niter, k
        ctx.E, ctx.S = E, S
        ctx.dev = theta.device
        out_E = torch.from_numpy(E.copy()).to(theta.device)
        out_I = torch.from_numpy((S[0, :] ** 2).copy()).to(theta.device)
        out_r = torch.from_numpy(np.abs(b[niter] * S[-1, :])).to(theta.device)
        ctx.mark_non_differentiable(out_r)
        return out_E, out_I, out_r

    @staticmethod
    def backward(ctx, gE, gI, gR=None):
        gEn = None if gE is None else gE.detach().to("cpu", torch.float64).numpy()
        gIn = None if gI is None else gI.detach().to("cpu", torch.float64).numpy()
        dev = ctx.dev if torch.device(ctx.dev).type == "cuda" else None
        abar, bbar_off = tridiag_eig_backward(ctx.E, ctx.S, gEn, gIn, device=dev)
        n = ctx.niter
        bbar = np.zeros(n)
        bbar[: n - 1] = bbar_off  # beta_n does not enter T_n
        try:
            g = ctx.h.lanczos_backward(n, abar, bbar, ctx.k)
        finally:
            ctx.h.close()
            ctx.h = None
        return torch.from_numpy(g).to(ctx.dev), None, None, None, None


def ritz(theta: torch.Tensor, params, niter: int, k: int = -1, residuals: bool = False, **opts):
    """Differentiable Ritz energies (hartree) and intensities of niter Lanczos steps (k: the
    checkpoint interval of nvb_set_checkpoints; the default -1 records the whole forward when
    it fits the backward budget, so the reverse sweep replays nothing, and otherwise takes the
    automatic recursive plan); with
    residuals=True also the residual estimates bji = |beta_n s_{n,i}| (hartree, constant
    w.r.t. theta), the convergence test of the reference's eigenvalue table
    (Source/top.f90:1074)."""
    E, I, r = LanczosRitz.apply(theta, params, niter, k, opts)
    return (E, I, r) if residuals else (E, I)


def converged_mask(bji: torch.Tensor, tol: float = 1e-9) -> torch.Tensor:
    """Ritz values converged to tol (bji < tol, hartree), ghost copies of converged roots
    included.  A spectrum or loss restricted to them is a smooth function of theta: after a
    long plain-Lanczos run the unconverged Ritz values are chaotic at the scale of rounding
    (finite differences of them do not converge as the step shrinks), while a converged root,
    summed over its ghost copies, has a well-defined energy and Franck-Condon weight.  Use the
    mask of the unperturbed run as a constant when comparing with finite differences."""
    return bji < tol


def converged_spectrum(E: torch.Tensor, I: torch.Tensor, mask: torch.Tensor, grid_cm: torch.Tensor,
                       sigma_cm: float = 20.0) -> torch.Tensor:
    """Gaussian-broadened spectrum of the converged Ritz values (mask from converged_mask),
    energies relative to the lowest of them (cm^-1)."""
    return convolved_spectrum(E[mask], I[mask], grid_cm, sigma_cm)


def convolved_spectrum(E: torch.Tensor, I: torch.Tensor, grid_cm: torch.Tensor, sigma_cm: float = 20.0,
                       origin: str = "lowest") -> torch.Tensor:
    """Gaussian-broadened stick spectrum on grid_cm (cm^-1): sum_i I_i exp(-(x - e_i)^2 / 2 sigma^2),
    e_i = (E_i - E_0) in cm^-1 with E_0 the lowest Ritz energy (origin "lowest") or 0 ("absolute")."""
    e = E * AU2WAVE
    if origin == "lowest":
        e = e - e.min()
    x = grid_cm[:, None] - e[None, :]
    return (I[None, :] * torch.exp(-0.5 * (x / sigma_cm) ** 2)).sum(dim=1)
