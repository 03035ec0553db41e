"""ORACLE (test infrastructure only) -- Lanczos with exact-overlap partial re-orthogonalisation.

Restates, for reorthog=2, update_lanczos / Hv / lanczos_step (Source/top.f90:646-842),
set_omega's exact branch (Source/top.f90:855-861: omega(2,i) = <q3, v_i>, not divided by beta)
and partial_orthog (Source/top.f90:910-1005): intervals around |omega| >= sqrt(eps) widened to
|omega| >= eps^(3/4), classical Gram-Schmidt of q3 against the archived vectors of the
intervals, repeated on the next step, beta recomputed.  The eps-sized random resets of
omega after a re-orthogonalisation are set to 0 here (they cannot cross either threshold).
Numpy + the C oracle's H.v; small systems only.  Parity status: unpinned (see oracle.py).
"""
from __future__ import annotations

import numpy as np


def choose_intervals(om2, it: int, eps: float = 2.0 ** -53):
    """partial_orthog's intervals (Source/top.f90:915-968) from omega(2, 0:it): around every i with
    |omega| >= sqrt(eps), widened while |omega| >= eps^(3/4), duplicates of the previous interval's
    ends dropped, and (1, 1) added when no interval starts at 1."""
    eta = eps ** 0.75
    oi = [i for i in range(1, it + 1) if abs(om2[i]) >= np.sqrt(eps)]
    ranges = []
    if oi:
        lid, rid = [], []
        for o in oi:
            j = o
            while j >= 1 and not abs(om2[j]) < eta:
                j -= 1
            lid.append(max(j, 1))
            k = o
            while k <= it and not abs(om2[k]) < eta:
                k += 1
            rid.append(min(k, it))
        ranges = [(lid[0], rid[0])]
        for a, b in zip(lid[1:], rid[1:]):
            if a != ranges[-1][0] and b != ranges[-1][1]:
                ranges.append((a, b))
        if min(r[0] for r in ranges) > 1:
            ranges.append((1, 1))
    return ranges


def lanczos_reorth_exact(S, niter: int, weights=None, log=None):
    """alpha[1..n], beta[0..n] and the Lanczos vectors; with a list `log`, every interval
    partial_orthog orthogonalises against is appended as (iteration, lo, hi), 1-based."""
    eps = 2.0 ** -53
    eta = eps ** 0.75
    N = S.ntotal
    ns = S.nstates
    w = np.ones(ns) if weights is None else np.asarray(weights, float)
    wsum = w.sum() or 1.0
    q3 = np.zeros(N)
    for s in range(ns):
        q3[s * S.dimen] = w[s] / wsum
    q3 /= np.sqrt(np.sum(q3 ** 2))
    q1 = np.zeros(N)
    q2 = np.zeros(N)
    alpha = np.zeros(niter + 1)
    beta = np.zeros(niter + 1)
    beta[0] = np.sqrt(q3 @ q3)
    V = []
    om2 = np.zeros(niter + 2)
    firststep = True
    ranges = []
    for it in range(1, niter + 1):
        q1 = q2.copy()
        q3 = q3 * (1.0 / beta[it - 1])
        q2 = q3.copy()
        V.append(q2.copy())
        q3 = S.hv(q2)
        alpha[it] = q2 @ q3
        q3 = q3 - alpha[it] * q2
        if it > 1:
            q3 = q3 - beta[it - 1] * q1
        beta[it] = np.sqrt(q3 @ q3)
        if it <= 1:
            continue
        om2[: it + 1] = 0.0
        for i in range(1, it + 1):
            om2[i] = q3 @ V[i - 1]
        if firststep:
            ranges = choose_intervals(om2, it, eps)
        if ranges:
            if log is not None:
                log.extend((it, a, b) for a, b in ranges)
            dots = [[q3 @ V[j - 1] for j in range(a, b + 1)] for a, b in ranges]
            for (a, b), d in zip(ranges, dots):
                for j, c in zip(range(a, b + 1), d):
                    q3 = q3 - c * V[j - 1]
                    om2[j] = 0.0
            firststep = not firststep
            beta[it] = np.sqrt(q3 @ q3)
    return alpha[1:], beta, np.array(V)
