"""ORACLE (test infrastructure only) -- the displaced / Duschinsky Franck-Condon seed of
``generate_initialvec`` (Source/secondary.f90:372-726, the ``neworigin`` branch).

The seed is the overlap <m|n> of an initial vibrational state |m> (frequencies bomega, in the
coordinates y = T x + d of the Hamiltonian's basis modes x, one mode excited by istate) with
every product basis function |n> (frequencies aomega) of the Hamiltonian.  Restated from the
reference:

* matrices (secondary.f90:407-478): A = (a + T^T b T)/2, A1 = sqrt(a) A^-1 sqrt(a) - 1,
  A2 = sqrt(a) A^-1 T^T sqrt(b), A3 = sqrt(b) T A^-1 T^T sqrt(b),
  A2d_i = sum_j A2_ij d_j sqrt(b_j), A3d_i = sum_j (A3_ji - 2 delta_ij) d_j sqrt(b_j);
* level recursion (secondary.f90:486-581): C(0) = 1,
  C(n + e_j) = 2 sum_{k in irrep(j)} A1_jk n_k C(n - e_k) - A2d_j C(n);
* initial-state recursion (secondary.f90:590-682), mode i = the excited mode, level m:
  C_m(n) = 2 (m-1) (A3_ii - 1) C_{m-2}(n) - A3d_i C_{m-1}(n) + 2 sum_k A2_ki n_k C_{m-1}(n - e_k);
* scale (secondary.f90:683-725): <m|n> = d2 C(n) / sqrt(prod_j 2^{n_j} n_j! 2^{m_j} m_j!),
  d2 = sqrt(sqrt(prod_j a_j b_j) |det T| / det A) exp(-sum_j b_j d_j^2 / 2 + (sqrt(b) d)^T A3 (sqrt(b) d) / 4).

This restatement builds each C(n) from n - e_j with j the LAST mode having n_j > 0 (the GPU
code uses the first), so the two agree only because the recursion is consistent; both are
checked against direct quadrature in the tests.
"""
from __future__ import annotations

import math

import numpy as np


def gauss_elim_det(t: np.ndarray) -> float:
    """|det T| as the product of |pivots| of elimination with row pivoting (secondary.f90:309-347)."""
    m = np.array(t, dtype=np.float64)
    n = m.shape[0]
    for i in range(n - 1):
        r = i + int(np.argmax(np.abs(m[i:, i])))
        if r != i:
            m[[i, r]] = m[[r, i]]
        for j in range(i + 1, n):
            if m[j, i] != 0:
                m[j] += (-m[j, i] / m[i, i]) * m[i]
    return float(np.prod(np.abs(np.diag(m))))


def matrices(aomega, bomega, dvec, tmat):
    a = np.asarray(aomega, dtype=np.float64)
    b = np.asarray(bomega, dtype=np.float64)
    d = np.asarray(dvec, dtype=np.float64)
    n = a.size
    T = np.asarray(tmat, dtype=np.float64).reshape(n, n).T  # T[k, i] = tmat[i*n + k] (column-major)
    detT = gauss_elim_det(T)
    A = 0.5 * (T.T @ np.diag(b) @ T) + 0.5 * np.diag(a)
    w = np.linalg.eigvalsh(A)
    detA = float(np.prod(np.abs(w)))
    Ainv = np.linalg.inv(A)
    sa, sb = np.sqrt(a), np.sqrt(b)
    A1 = Ainv * np.outer(sa, sa) - np.eye(n)
    A2 = (Ainv @ T.T) * np.outer(sa, sb)
    A3 = (T @ Ainv @ T.T) * np.outer(sb, sb)
    A2d = A2 @ (d * sb)
    A3d = (A3 - 2 * np.eye(n)).T @ (d * sb)
    d1 = -0.5 * np.sum(b * d * d) + 0.25 * (d * sb) @ A3 @ (d * sb)
    d2 = math.sqrt(math.sqrt(float(np.prod(b * a))) * detT / detA) * math.exp(d1)
    return dict(T=T, A1=A1, A2=A2, A3=A3, A2d=A2d, A3d=A3d, d2=d2, detT=detT, detA=detA)


def overlaps(nfunc, aomega, bomega, dvec, tmat, istate=None, npirr=None) -> np.ndarray:
    """<m|n> for every product function n (flat, last mode fastest)."""
    nfunc = [int(v) for v in nfunc]
    M = len(nfunc)
    istate = [0] * M if istate is None else [int(v) for v in istate]
    # only one mode may be excited: the first positive entry (Source/top.f90:326-334)
    seen = False
    for i in range(M):
        if istate[i] > 0 and not seen:
            seen = True
        else:
            istate[i] = 0
    npirr = [M] if npirr is None else list(npirr)
    irrep = []
    for l, c in enumerate(npirr):
        irrep += [l] * c
    mx = matrices(aomega, bomega, dvec, tmat)
    A1, A2, A3, A2d, A3d = mx["A1"], mx["A2"], mx["A3"], mx["A2d"], mx["A3d"]
    shape = tuple(nfunc)
    idx = list(np.ndindex(*shape))
    level = {}
    for n in idx:
        level.setdefault(sum(n), []).append(n)
    C = np.zeros(shape)
    C[(0,) * M] = 1.0
    for L in range(1, sum(v - 1 for v in nfunc) + 1):
        for n in level.get(L, []):
            j = max(q for q in range(M) if n[q] > 0)
            p = list(n)
            p[j] -= 1
            s = 0.0
            for k in range(M):
                if irrep[k] != irrep[j] or p[k] == 0:
                    continue
                pk = list(p)
                pk[k] -= 1
                s += A1[j, k] * p[k] * C[tuple(pk)]
            C[n] = 2.0 * s - A2d[j] * C[tuple(p)]
    imode = next((i for i in range(M) if istate[i] > 0), M - 1)
    ninit = istate[imode]
    cm2, cm1 = np.zeros(shape), C
    for m in range(1, ninit + 1):
        cm = 2.0 * (m - 1) * (A3[imode, imode] - 1.0) * cm2 - A3d[imode] * cm1
        for n in idx:
            for k in range(M):
                if n[k] > 0:
                    nk = list(n)
                    nk[k] -= 1
                    cm[n] += 2.0 * A2[k, imode] * n[k] * cm1[tuple(nk)]
        cm2, cm1 = cm1, cm
    C = cm1
    out = np.empty(shape)
    for n in idx:
        den = 1.0
        for j in range(M):
            den *= 2.0 ** n[j] * math.factorial(n[j]) * 2.0 ** istate[j] * math.factorial(istate[j])
        out[n] = mx["d2"] * C[n] / math.sqrt(den)
    return out.reshape(-1)


def quadrature_overlaps(nfunc, aomega, bomega, dvec, tmat, istate=None, npts=400, half_width=9.0):
    """Independent check for 1-2 modes: sqrt|det T| * integral of chi_m(T x + d) phi_n(x) dx on a
    grid, phi_n / chi_m harmonic-oscillator eigenfunctions of frequencies aomega / bomega
    (mass-weighted coordinates, hbar = 1)."""
    from numpy.polynomial.hermite import hermval

    a = np.asarray(aomega, dtype=np.float64)
    b = np.asarray(bomega, dtype=np.float64)
    d = np.asarray(dvec, dtype=np.float64)
    M = a.size
    T = np.asarray(tmat, dtype=np.float64).reshape(M, M).T
    istate = [0] * M if istate is None else list(istate)

    def ho(n, w, x):
        c = np.zeros(n + 1)
        c[n] = 1.0
        return (w / np.pi) ** 0.25 / math.sqrt(2.0 ** n * math.factorial(n)) * hermval(np.sqrt(w) * x, c) \
            * np.exp(-0.5 * w * x * x)

    axes = [np.linspace(-half_width / math.sqrt(a[i]), half_width / math.sqrt(a[i]), npts) for i in range(M)]
    grids = np.meshgrid(*axes, indexing="ij")
    X = np.stack([g.reshape(-1) for g in grids])  # [M, P]
    Y = T @ X + d[:, None]
    chi = np.ones(X.shape[1])
    for k in range(M):
        chi *= ho(istate[k], b[k], Y[k])
    dv = np.prod([ax[1] - ax[0] for ax in axes])
    out = []
    for n in np.ndindex(*[int(v) for v in nfunc]):
        phi = np.ones(X.shape[1])
        for i in range(M):
            phi *= ho(n[i], a[i], X[i])
        out.append(math.sqrt(abs(np.linalg.det(T))) * float(np.sum(chi * phi)) * dv)
    return np.array(out)
