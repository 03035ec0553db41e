// All eigenpairs of the Lanczos tridiagonal matrix T_n (FP64, host).
//
// Eigenvalues: Sturm-sequence bisection on T scaled to unit Euclidean norm, every root
// bisected independently (OpenMP over roots) until the midpoint equals an end of the
// bracket.  Eigenvectors: two sweeps of inverse iteration with row pivoting, a
// pseudo-random start for roots that repeat to 100*eps, Gram-Schmidt among such roots, and
// normalisation with components below eps/100 set to zero.  The eigenvector steps are kept
// alike to GIVENS (Source/yarkony.f90:385-478) -- start vector, pivot rule, random
// generator, and the multiplier it applies to pivoted rows in the second sweep -- because
// the reference reports the sign of each eigenvector's first component (Tsign, written to
// sodata.in) and the phases of lead contributors, and those depend on these steps.
#include <cfloat>
#include <cmath>
#include <vector>

#include "nvb_internal.h"

namespace nvb {

static double machine_eps() {
    // determine_epsilon (Source/secondary.f90:260-271): first power of two that no longer
    // changes 1 when added.
    volatile double e = 1.0;
    for (;;) {
        e = e / 2.0;
        volatile double e1 = e + 1.0;
        if (e1 == 1.0) break;
    }
    return e;
}

// Number of eigenvalues of the scaled T below x (pivots < 0), tiny pivots skip one row.
static int64_t sturm_below(int64_t n, const double *d, const double *e2, double x, double tiny) {
    int64_t below = 0;
    int64_t j = 0;
    double f = d[0] - x;
    for (;;) {
        if (std::fabs(f) < tiny) {
            j += 2;
            below += 1;
            if (j < n) { f = d[j] - x; continue; }
            break;
        }
        if (f < 0.0) below += 1;
        j += 1;
        if (j >= n) break;
        f = d[j] - x - e2[j - 1] / f;
    }
    return below;
}

void tridiag_eigen(int64_t n, const double *diag, const double *codiag, double *eig, double *vect) {
    if (n <= 0) return;
    if (n == 1) {
        eig[0] = diag[0];
        if (vect) vect[0] = 1.0;
        return;
    }
    const double ETA = machine_eps();
    const double DEL1 = ETA / 100.0, DELTA = ETA * ETA * 100.0;
    const double DELBIG = DBL_MAX * DELTA / 1000.0, THETA1 = 1000.0 / DBL_MAX;
    const double TOLER = ETA * 100.0;
    double factor = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        if (i > 0) factor = std::fmax(factor, std::fabs(codiag[i - 1]));
        factor = std::fmax(factor, std::fabs(diag[i]));
    }
    if (factor == 0.0) {
        for (int64_t i = 0; i < n; ++i) {
            eig[i] = 0.0;
            if (vect) {
                for (int64_t j = 0; j < n; ++j) vect[i * n + j] = 0.0;
                vect[i * n + i] = 1.0;
            }
        }
        return;
    }
    double anorm = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        if (i > 0) anorm += (codiag[i - 1] / factor) * (codiag[i - 1] / factor);
        anorm += (diag[i] / factor) * (diag[i] / factor) / 2.0;
    }
    anorm = std::sqrt(anorm * 2.0) * factor;
    std::vector<double> d(n), e(n + 1, 0.0), e2(n, 0.0);
    for (int64_t i = 0; i < n; ++i) d[i] = diag[i] / anorm;
    for (int64_t i = 0; i + 1 < n; ++i) {
        e[i] = codiag[i] / anorm;
        e2[i] = e[i] * e[i];
    }
    std::vector<double> root(n);
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t I = 1; I <= n; ++I) {
        double lo = -1.0, hi = 1.0;
        for (;;) {
            const double t = (lo + hi) * 0.5;
            if (t == lo || t == hi) break;
            if (sturm_below(n, d.data(), e2.data(), t, THETA1) >= I) hi = t;
            else lo = t;
        }
        root[I - 1] = hi;
    }
    for (int64_t i = 0; i < n; ++i) eig[i] = root[i] * anorm;
    if (!vect) return;
    // inverse iteration
    std::vector<double> B2(n + 1), B3(n + 1), B4(n + 1), B5(n + 1);
    const double RPOWER = 8388608.0, RPOW1 = RPOWER / 2.0;
    double rnd = RPOWER - 3.0;
    int64_t ia = 0;
    double temp = 0.0;
    auto E1 = [&](int64_t j) { return e[j - 1]; };  // 1-based codiagonal, E1(n) = 0
    for (int64_t I = 1; I <= n; ++I) {
        double *v = vect + (I - 1) * n;
        for (int64_t j = 0; j < n; ++j) v[j] = 1.0;
        const double ar = root[I - 1];
        if (I == 1 || !(std::fabs(root[I - 2] - ar) < TOLER)) ia = -1;
        ia += 1;
        double el1 = d[0] - ar, el2 = E1(1);
        for (int64_t J = 1; J <= n - 1; ++J) {
            if (std::fabs(el1) <= std::fabs(E1(J))) {
                B2[J] = E1(J);
                B3[J] = d[J] - ar;
                B4[J] = E1(J + 1);
                temp = 1.0;
                if (std::fabs(E1(J)) > THETA1) temp = el1 / E1(J);
                el1 = el2 - temp * B3[J];
                el2 = -temp * E1(J + 1);
            } else {
                B2[J] = el1;
                B3[J] = el2;
                B4[J] = 0.0;
                temp = E1(J) / el1;
                el1 = d[J] - ar - temp * el2;
                el2 = E1(J + 1);
            }
            B5[J] = temp;
        }
        B2[n] = el1;
        B3[n] = 0.0;
        B4[n] = 0.0;
        B4[n - 1] = 0.0;
        if (ia != 0)
            for (int64_t j = 0; j < n; ++j) {
                rnd = std::fmod(4099.0 * rnd, RPOWER);
                v[j] = rnd / RPOW1 - 1.0;
            }
        for (int sweep = 1; sweep <= 2; ++sweep) {
            for (int64_t L = n; L >= 1; --L) {
                for (;;) {
                    const double v1 = L + 1 <= n ? v[L] : 0.0, v2 = L + 2 <= n ? v[L + 1] : 0.0;
                    const double x = v[L - 1] - v1 * B3[L] - v2 * B4[L];
                    if (std::fabs(x) > DELBIG) {
                        for (int64_t k = 0; k < n; ++k) v[k] = v[k] / DELBIG;
                        continue;
                    }
                    temp = B2[L];
                    if (std::fabs(B2[L]) < DELTA) temp = DELTA;
                    v[L - 1] = x / temp;
                    break;
                }
            }
            if (sweep == 2) break;
            double x = v[0];
            for (int64_t J = 1; J <= n - 1; ++J) {
                if (B2[J] == E1(J)) {
                    v[J - 1] = v[J];
                    x = x - v[J] * temp;  // multiplier as applied by GIVENS (see header)
                } else {
                    v[J - 1] = x;
                    x = v[J] - x * B5[J];
                }
            }
            v[n - 1] = x;
        }
        for (int64_t j1 = 1; j1 <= ia; ++j1) {
            const double *w = vect + (I - j1 - 1) * n;
            double s = 0.0;
            for (int64_t j = 0; j < n; ++j) s += v[j] * w[j];
            for (int64_t j = 0; j < n; ++j) v[j] -= s * w[j];
        }
        double mx = 0.0;
        for (int64_t j = 0; j < n; ++j) mx = std::fmax(std::fabs(v[j]), mx);
        double ss = 0.0;
        for (int64_t j = 0; j < n; ++j) {
            const double q = v[j] / mx;
            ss += q * q;
        }
        const double f = 1.0 / (std::sqrt(ss) * mx);
        for (int64_t j = 0; j < n; ++j) {
            v[j] = v[j] * f;
            if (std::fabs(v[j]) < DEL1) v[j] = 0.0;
        }
    }
}

}  // namespace nvb
