/*
 * ORACLE -- test infrastructure only.  CPU (FP64, optional OpenMP) restatement of the
 * NadVibS Lanczos stage.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline / reference arm load this library, as the checker and the timed CPU
 * baseline.  The product library never links or calls it.
 *
 * Parity status: UNPINNED against the reference.  The reference (Fortran 90 + MPI +
 * Global Arrays) cannot be compiled in this image (no Fortran compiler, no MPI, no GA),
 * and it ships no example input/output for this path.  Every function below restates
 * the reference's algorithm from its source and is checked by known-answer tests
 * (dense Hamiltonian, displaced oscillator, analytic <m|x^p|n>, scipy tridiagonal).
 *
 * Deviations from the reference's arithmetic, all at the rounding level:
 *  - the reference forms the harmonic energy (dkin) and the matrix-element product d1
 *    incrementally along its row sweep (Source/top.f90:721-730, 794-796); here dkin is
 *    formed directly per row, and d1 is recomputed from scratch whenever the row walk
 *    changes one of the term's digits (the walk itself is incremental, as the reference's);
 *  - GA_DDOT's reduction order is rank dependent; here dots are summed in row order
 *    (single thread) or per-thread blocks combined in thread order (OpenMP).
 * The per-element accumulation order of H.v follows the reference: diagonal part first,
 * then terms / shift steps / block pairs in table order.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_MAXM 64
#define ORC_MAXS 16

typedef struct orc_system {
    int64_t nstates, nmodes, ordr, nterms, maxpairs;
    const int64_t *nfunc;   /* [nmodes] */
    const double *omega;    /* [nmodes] hartree */
    const double *concoef;  /* [nstates(nstates+1)/2] block order of cpindx */
    const int64_t *tcnt;    /* [nterms] distinct modes of term t */
    const int64_t *tmode;   /* [nterms*ordr] 1-based modes (decreasing) */
    const int64_t *tpow;    /* [nterms*ordr] powers */
    const int64_t *tnpair;  /* [nterms] */
    const int64_t *tpa;     /* [nterms*maxpairs] row state (1-based) */
    const int64_t *tpb;     /* [nterms*maxpairs] column state (1-based) */
    const double *tcoef;    /* [nterms*maxpairs] scaled coefficients */
    int64_t quirk_cubic;    /* 1: reference <m|x^3|m+1> (missing factor 3); 0: exact */
    int64_t quirk_lower;    /* 1: reference lower-triangle-only diagonal coupling; 0: symmetric */
} orc_system;

/* hoelem: Source/function.f90:186-250.  a, b are 1-based basis indices. */
double orc_hoelem(int64_t p, int64_t a, int64_t b, int64_t quirk_cubic)
{
    double m = (double)a - 1.0;
    double r = 0.0;
    switch (p) {
    case 0: r = (b == a) ? 1.0 : 0.0; break;
    case 1:
        if (b == a + 1) r = sqrt((m + 1) / 2);
        else if (b == a - 1) r = sqrt(m / 2);
        break;
    case 2:
        if (b == a + 2) r = sqrt((m + 1) * (m + 2) / 4);
        else if (b == a) r = ((2 * m + 1) / 2);
        else if (b == a - 2) r = sqrt(m * (m - 1) / 4);
        break;
    case 3:
        if (b == a + 3) r = sqrt((m + 1) * (m + 2) * (m + 3) / 8);
        else if (b == a + 1) r = sqrt(((m + 1) * (m + 1) * (m + 1)) / 8) * (quirk_cubic ? 1.0 : 3.0);
        else if (b == a - 1) r = sqrt((m * m * m) / 8) * (quirk_cubic ? 1.0 : 3.0);
        else if (b == a - 3) r = sqrt(m * (m - 1) * (m - 2) / 8);
        break;
    case 4:
        if (b == a + 4) r = sqrt((m + 1) * (m + 2) * (m + 3) * (m + 4)) / 4;
        else if (b == a + 2) r = (2 * m + 3) * sqrt((m + 1) * (m + 2)) / 2;
        else if (b == a) r = 3 * (2 * m * m + 2 * m + 1) / 4;
        else if (b == a - 2) r = (2 * m - 1) * sqrt(m * (m - 1)) / 2;
        else if (b == a - 4) r = sqrt(m * (m - 1) * (m - 2) * (m - 3)) / 4;
        break;
    default: r = 0.0;
    }
    return r;
}

/* element used by Hv: homatel(iordr(|s|/2+1,p) + min(n,n+s) + 1) = <lo|x^p|lo+|s|> with
 * lo = min(n, n+s) (0-based), Source/top.f90:772,800 with the table of :501-527. */
static double elem(const orc_system *S, int64_t p, int64_t n, int64_t s)
{
    int64_t lo = s < 0 ? n + s : n;
    int64_t j = s < 0 ? -s : s;
    return orc_hoelem(p, lo + 1, lo + 1 + j, S->quirk_cubic);
}

static int64_t smax_of(int64_t p, int64_t nf)
{
    int64_t s = p;
    while (s > nf - 1) s -= 2;   /* Source/secondary.f90:33-37 */
    return s;
}

int64_t orc_dimen(const orc_system *S)
{
    int64_t d = 1;
    for (int64_t k = 0; k < S->nmodes; ++k) d *= S->nfunc[k];
    return d;
}

static void shifts_of(const orc_system *S, int64_t *shft)
{
    /* shft(k) = prod_{j>k} nfunc(j), Source/top.f90:379-386 */
    for (int64_t k = 0; k < S->nmodes; ++k) {
        shft[k] = 1;
        for (int64_t j = k + 1; j < S->nmodes; ++j) shft[k] *= S->nfunc[j];
    }
}

static int is_diag_term(const orc_system *S, int64_t t)
{
    for (int64_t l = 0; l < S->tcnt[t]; ++l) {
        int64_t m = S->tmode[t * S->ordr + l] - 1;
        if (smax_of(S->tpow[t * S->ordr + l], S->nfunc[m]) % 2 != 0) return 0;
    }
    return 1;
}

/* y = H x, layout x[s*dimen + r] (column-major q(dimen,nstates)).  Source/top.f90:672-818.
 * walk = 1: each (term, shift) pass walks its rows with an incremental mixed-radix counter of
 * the digits (Source/top.f90:781-803: a per-row increment of the fastest digit with carries;
 * the element product of the term is recomputed only when one of the term's digits changed);
 * walk = 0: the digits of every row are decoded by division in every pass.  Both give the same
 * bits (same products in the same order per element); walk = 1 is the timed CPU baseline. */
static int orc_hv_impl(const orc_system *S, const double *x, double *y, int nthreads, int walk)
{
    const int64_t N = orc_dimen(S), NS = S->nstates, M = S->nmodes;
    int64_t shft[ORC_MAXM];
    if (M > ORC_MAXM || NS > ORC_MAXS) return -1;
    shifts_of(S, shft);
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    /* dblks (Source/top.f90:528-553): state pairs i>j with a constant or even-power term */
    int dchk[ORC_MAXS][ORC_MAXS];
    memset(dchk, 0, sizeof dchk);
    for (int64_t i = 1, k = 0; i <= NS; ++i)
        for (int64_t j = 1; j <= i; ++j, ++k)
            if (fabs(S->concoef[k]) > 1e-16) { dchk[i - 1][j - 1] = 1; dchk[j - 1][i - 1] = 1; }
    for (int64_t t = 0; t < S->nterms; ++t)
        if (is_diag_term(S, t))
            for (int64_t q = 0; q < S->tnpair[t]; ++q)
                dchk[S->tpa[t * S->maxpairs + q] - 1][S->tpb[t * S->maxpairs + q] - 1] = 1;

    /* ---- diagonal part, Source/top.f90:712-756 ---- */
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < N; ++r) {
        int64_t n[ORC_MAXM];
        int64_t rem = r;
        double dkin = 0.0;
        for (int64_t k = 0; k < M; ++k) { n[k] = rem / shft[k]; rem -= n[k] * shft[k]; }
        for (int64_t k = 0; k < M; ++k) dkin += ((double)n[k] + 0.5) * S->omega[k];
        double dv[ORC_MAXS][ORC_MAXS];
        for (int64_t i = 1, k = 0; i <= NS; ++i)
            for (int64_t j = 1; j <= i; ++j, ++k) { dv[i - 1][j - 1] = S->concoef[k]; dv[j - 1][i - 1] = S->concoef[k]; }
        for (int64_t t = 0; t < S->nterms; ++t) {
            if (!is_diag_term(S, t)) continue;
            double d1 = 1.0;
            for (int64_t l = 0; l < S->tcnt[t]; ++l) {
                int64_t m = S->tmode[t * S->ordr + l] - 1;
                d1 = d1 * elem(S, S->tpow[t * S->ordr + l], n[m], 0);
            }
            for (int64_t q = 0; q < S->tnpair[t]; ++q) {
                int64_t a = S->tpa[t * S->maxpairs + q] - 1, b = S->tpb[t * S->maxpairs + q] - 1;
                dv[a][b] = dv[a][b] + S->tcoef[t * S->maxpairs + q] * d1;
            }
        }
        for (int64_t s = 0; s < NS; ++s) y[s * N + r] = 0.0 + (dv[s][s] + dkin) * x[s * N + r];
        for (int64_t i = 0; i < NS; ++i)
            for (int64_t j = 0; j < i; ++j)
                if (dchk[i][j]) {
                    y[i * N + r] = y[i * N + r] + dv[i][j] * x[j * N + r];
                    if (!S->quirk_lower) y[j * N + r] = y[j * N + r] + dv[j][i] * x[i * N + r];
                }
    }

    /* ---- shift part: one streaming pass per (term, nonzero shift), Source/top.f90:758-808,
     * shifts enumerated as in Source/secondary.f90:27-64,98-124 ---- */
    for (int64_t t = 0; t < S->nterms; ++t) {
        int64_t d = S->tcnt[t];
        int64_t md[8], pw[8], sm[8], sdir[8];
        int64_t nsteps = 1;
        int bad = 0;
        for (int64_t l = 0; l < d; ++l) {
            md[l] = S->tmode[t * S->ordr + l] - 1;
            pw[l] = S->tpow[t * S->ordr + l];
            sm[l] = smax_of(pw[l], S->nfunc[md[l]]);
            if (sm[l] < 0) bad = 1;
            nsteps *= sm[l] + 1;
            sdir[l] = -sm[l];
        }
        if (bad) continue;
        sdir[d - 1] -= 2;
        for (int64_t st = 0; st < nsteps; ++st) {
            int64_t l = d - 1;
            while (sdir[l] >= sm[l]) { sdir[l] = -sm[l]; --l; }
            sdir[l] += 2;
            int64_t stride = 0;
            for (int64_t q = 0; q < d; ++q) stride += sdir[q] * shft[md[q]];
            if (stride == 0) continue;
            const int64_t np = S->tnpair[t];
            const int64_t *pa = S->tpa + t * S->maxpairs, *pb = S->tpb + t * S->maxpairs;
            const double *pc = S->tcoef + t * S->maxpairs;
            int64_t sd[8];
            for (int64_t q = 0; q < d; ++q) sd[q] = sdir[q];
            if (walk) {
                int64_t mdmax = 0;
                for (int64_t q = 0; q < d; ++q) mdmax = md[q] > mdmax ? md[q] : mdmax;
#pragma omp parallel
                {
                    int nth = 1, tid = 0;
#ifdef _OPENMP
                    nth = omp_get_num_threads();
                    tid = omp_get_thread_num();
#endif
                    const int64_t r0 = N * tid / nth, r1 = N * (tid + 1) / nth;
                    int64_t n[ORC_MAXM];
                    int64_t rem = r0;
                    for (int64_t k = 0; k < M; ++k) { n[k] = rem / shft[k]; rem -= n[k] * shft[k]; }
                    int dirty = 1, ok = 0;
                    double d1 = 1.0;
                    for (int64_t r = r0; r < r1; ++r) {
                        if (dirty) {
                            d1 = 1.0;
                            ok = 1;
                            for (int64_t q = 0; q < d; ++q) {
                                int64_t nc = n[md[q]] + sd[q];
                                if (nc < 0 || nc >= S->nfunc[md[q]]) { ok = 0; break; }
                                d1 = d1 * elem(S, pw[q], n[md[q]], sd[q]);
                            }
                            dirty = 0;
                        }
                        if (ok) {
                            int64_t c = r + stride;
                            for (int64_t q = 0; q < np; ++q)
                                y[(pa[q] - 1) * N + r] = y[(pa[q] - 1) * N + r] + x[(pb[q] - 1) * N + c] * pc[q] * d1;
                        }
                        /* next row: increment the fastest digit, carrying into slower ones */
                        int64_t k = M - 1;
                        while (k >= 0 && ++n[k] == S->nfunc[k]) { n[k] = 0; --k; }
                        if (k <= mdmax) dirty = 1;
                    }
                }
                continue;
            }
#pragma omp parallel for schedule(static)
            for (int64_t r = 0; r < N; ++r) {
                double d1 = 1.0;
                int ok = 1;
                for (int64_t q = 0; q < d; ++q) {
                    int64_t nq = (r / shft[md[q]]) % S->nfunc[md[q]];
                    int64_t nc = nq + sd[q];
                    if (nc < 0 || nc >= S->nfunc[md[q]]) { ok = 0; break; }
                    d1 = d1 * elem(S, pw[q], nq, sd[q]);
                }
                if (!ok) continue;
                int64_t c = r + stride;
                for (int64_t q = 0; q < np; ++q)
                    y[(pa[q] - 1) * N + r] = y[(pa[q] - 1) * N + r] + x[(pb[q] - 1) * N + c] * pc[q] * d1;
            }
        }
    }
    return 0;
}

int orc_hv(const orc_system *S, const double *x, double *y, int nthreads)
{
    return orc_hv_impl(S, x, y, nthreads, 1);
}

/* the same product with the digits of every row decoded by division in every pass */
int orc_hv_rowdiv(const orc_system *S, const double *x, double *y, int nthreads)
{
    return orc_hv_impl(S, x, y, nthreads, 0);
}

/* y at selected rows only (all states), same terms as orc_hv, for full-size spot checks:
 * yrow[k*nstates + s] = (H x)[s*dimen + rows[k]]. */
int orc_hv_rows(const orc_system *S, const double *x, const int64_t *rows, int64_t nrows, double *yrow)
{
    const int64_t N = orc_dimen(S), NS = S->nstates, M = S->nmodes;
    int64_t shft[ORC_MAXM];
    if (M > ORC_MAXM || NS > ORC_MAXS) return -1;
    shifts_of(S, shft);
    int dchk[ORC_MAXS][ORC_MAXS];
    memset(dchk, 0, sizeof dchk);
    for (int64_t i = 1, k = 0; i <= NS; ++i)
        for (int64_t j = 1; j <= i; ++j, ++k)
            if (fabs(S->concoef[k]) > 1e-16) { dchk[i - 1][j - 1] = 1; dchk[j - 1][i - 1] = 1; }
    for (int64_t t = 0; t < S->nterms; ++t)
        if (is_diag_term(S, t))
            for (int64_t q = 0; q < S->tnpair[t]; ++q)
                dchk[S->tpa[t * S->maxpairs + q] - 1][S->tpb[t * S->maxpairs + q] - 1] = 1;
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t k = 0; k < nrows; ++k) {
        const int64_t r = rows[k];
        double *y = yrow + k * NS;
        int64_t n[ORC_MAXM];
        int64_t rem = r;
        double dkin = 0.0;
        for (int64_t m = 0; m < M; ++m) { n[m] = rem / shft[m]; rem -= n[m] * shft[m]; }
        for (int64_t m = 0; m < M; ++m) dkin += ((double)n[m] + 0.5) * S->omega[m];
        double dv[ORC_MAXS][ORC_MAXS];
        for (int64_t i = 1, q = 0; i <= NS; ++i)
            for (int64_t j = 1; j <= i; ++j, ++q) { dv[i - 1][j - 1] = S->concoef[q]; dv[j - 1][i - 1] = S->concoef[q]; }
        for (int64_t t = 0; t < S->nterms; ++t) {
            if (!is_diag_term(S, t)) continue;
            double d1 = 1.0;
            for (int64_t l = 0; l < S->tcnt[t]; ++l)
                d1 = d1 * elem(S, S->tpow[t * S->ordr + l], n[S->tmode[t * S->ordr + l] - 1], 0);
            for (int64_t q = 0; q < S->tnpair[t]; ++q) {
                int64_t a = S->tpa[t * S->maxpairs + q] - 1, b = S->tpb[t * S->maxpairs + q] - 1;
                dv[a][b] = dv[a][b] + S->tcoef[t * S->maxpairs + q] * d1;
            }
        }
        for (int64_t s = 0; s < NS; ++s) y[s] = (dv[s][s] + dkin) * x[s * N + r];
        for (int64_t i = 0; i < NS; ++i)
            for (int64_t j = 0; j < i; ++j)
                if (dchk[i][j]) {
                    y[i] = y[i] + dv[i][j] * x[j * N + r];
                    if (!S->quirk_lower) y[j] = y[j] + dv[j][i] * x[i * N + r];
                }
        for (int64_t t = 0; t < S->nterms; ++t) {
            int64_t d = S->tcnt[t], md[8], pw[8], sm[8], sdir[8], nsteps = 1;
            int bad = 0;
            for (int64_t l = 0; l < d; ++l) {
                md[l] = S->tmode[t * S->ordr + l] - 1;
                pw[l] = S->tpow[t * S->ordr + l];
                sm[l] = smax_of(pw[l], S->nfunc[md[l]]);
                if (sm[l] < 0) bad = 1;
                nsteps *= sm[l] + 1;
                sdir[l] = -sm[l];
            }
            if (bad) continue;
            sdir[d - 1] -= 2;
            for (int64_t st = 0; st < nsteps; ++st) {
                int64_t l = d - 1;
                while (sdir[l] >= sm[l]) { sdir[l] = -sm[l]; --l; }
                sdir[l] += 2;
                int64_t stride = 0, ok = 1;
                double d1 = 1.0;
                for (int64_t q = 0; q < d; ++q) stride += sdir[q] * shft[md[q]];
                if (stride == 0) continue;
                for (int64_t q = 0; q < d; ++q) {
                    int64_t nc = n[md[q]] + sdir[q];
                    if (nc < 0 || nc >= S->nfunc[md[q]]) { ok = 0; break; }
                    d1 = d1 * elem(S, pw[q], n[md[q]], sdir[q]);
                }
                if (!ok) continue;
                for (int64_t q = 0; q < S->tnpair[t]; ++q) {
                    int64_t a = S->tpa[t * S->maxpairs + q] - 1, b = S->tpb[t * S->maxpairs + q] - 1;
                    y[a] = y[a] + x[b * N + r + stride] * S->tcoef[t * S->maxpairs + q] * d1;
                }
            }
        }
    }
    return 0;
}

/* Deterministic dot product: per-thread contiguous blocks combined in thread order. */
static double ddot(const double *a, const double *b, int64_t n, int nthreads)
{
    if (nthreads <= 1) {
        double s = 0.0;
        for (int64_t i = 0; i < n; ++i) s += a[i] * b[i];
        return s;
    }
    double part[512];
    int nt = nthreads > 512 ? 512 : nthreads;
#pragma omp parallel num_threads(nt)
    {
#ifdef _OPENMP
        int tid = omp_get_thread_num(), tn = omp_get_num_threads();
#else
        int tid = 0, tn = 1;
#endif
        int64_t lo = n * tid / tn, hi = n * (tid + 1) / tn;
        double s = 0.0;
        for (int64_t i = lo; i < hi; ++i) s += a[i] * b[i];
        part[tid] = s;
        if (tid == 0) nt = tn;
    }
    double s = 0.0;
    for (int t = 0; t < nt; ++t) s += part[t];
    return s;
}

/* Plain Lanczos (reorthog=0) in the reference's operation order:
 *   seed  Source/secondary.f90:727-783 (|0..0> x weights, normalised), beta(0)=||q3||
 *   update_lanczos Source/top.f90:646-670: q1=q2; q3=q3*(1/beta(i-1)); q2=q3
 *   Hv, lanczos_step Source/top.f90:820-842: alpha=<q2,q3>; q3-=alpha q2; q3-=beta(i-1) q1;
 *   beta(i)=sqrt(<q3,q3>).
 * alpha[1..niter] -> alpha[0..niter-1]; beta[0..niter].  vecs (optional) receives the
 * normalised q2 of every iteration (niter*N), qfinal (optional) q1,q2,q3 at the end. */
int orc_lanczos(const orc_system *S, const double *weights, int64_t niter, double *alpha, double *beta,
                double *vecs, double *qfinal, int nthreads)
{
    const int64_t N = orc_dimen(S), NS = S->nstates, NT = N * NS;
    double *q1 = calloc((size_t)NT, sizeof(double));
    double *q2 = calloc((size_t)NT, sizeof(double));
    double *q3 = calloc((size_t)NT, sizeof(double));
    if (!q1 || !q2 || !q3) { free(q1); free(q2); free(q3); return -2; }
    /* seed: row 1 of every state = 1, d1=sqrt(<q3,q3>/nstates)=1, state i scaled by
     * statew(i)/(sum statew * d1), then the whole vector normalised */
    double wsum = 0.0;
    for (int64_t s = 0; s < NS; ++s) wsum += weights[s];
    if (wsum == 0.0) wsum = 1.0;
    for (int64_t s = 0; s < NS; ++s) q3[s * N] = 1.0;
    double d1 = sqrt(ddot(q3, q3, NT, 1) / (double)NS);
    for (int64_t s = 0; s < NS; ++s) q3[s * N] = q3[s * N] * (weights[s] / (wsum * d1));
    double d2 = 0.0;
    for (int64_t s = 0; s < NS; ++s) { double e = sqrt(q3[s * N] * q3[s * N]); d2 += e * e; }
    double sc = 1.0 / sqrt(d2);
    for (int64_t s = 0; s < NS; ++s) q3[s * N] *= sc;
    beta[0] = sqrt(ddot(q3, q3, NT, nthreads));
    for (int64_t it = 1; it <= niter; ++it) {
        double inv = 1. / beta[it - 1];
        memcpy(q1, q2, (size_t)NT * sizeof(double));
#pragma omp parallel for schedule(static) num_threads(nthreads > 0 ? nthreads : 1)
        for (int64_t i = 0; i < NT; ++i) q3[i] = q3[i] * inv;
        memcpy(q2, q3, (size_t)NT * sizeof(double));
        if (vecs) memcpy(vecs + (it - 1) * NT, q2, (size_t)NT * sizeof(double));
        orc_hv(S, q2, q3, nthreads);
        double a = ddot(q2, q3, NT, nthreads);
        alpha[it - 1] = a;
#pragma omp parallel for schedule(static) num_threads(nthreads > 0 ? nthreads : 1)
        for (int64_t i = 0; i < NT; ++i) q3[i] = 1.0 * q3[i] + (-a) * q2[i];
        if (it > 1) {
            double b = beta[it - 1];
#pragma omp parallel for schedule(static) num_threads(nthreads > 0 ? nthreads : 1)
            for (int64_t i = 0; i < NT; ++i) q3[i] = 1.0 * q3[i] + (-b) * q1[i];
        }
        beta[it] = sqrt(ddot(q3, q3, NT, nthreads));
    }
    if (qfinal) {
        memcpy(qfinal, q1, (size_t)NT * sizeof(double));
        memcpy(qfinal + NT, q2, (size_t)NT * sizeof(double));
        memcpy(qfinal + 2 * NT, q3, (size_t)NT * sizeof(double));
    }
    free(q1); free(q2); free(q3);
    return 0;
}

/* GIVENS (Source/yarkony.f90:91-543) restated for the only matrices it receives here:
 * tridiagonal T packed by make_tmatrix (Source/secondary.f90:898-919).  For such input
 * the Householder section stores zero transformation vectors, so the final back-rotation
 * (SIMVEC) leaves the vectors unchanged; both are omitted.  Kept as written: Euclidean
 * norm scaling, Sturm bisection to the last bit, two-sweep inverse iteration with
 * pivoting, pseudo-random start for repeated roots, Gram-Schmidt among close roots,
 * normalisation with the DEL1 cut-off, and the stale multiplier used for "case two" rows
 * in the second sweep (Source/yarkony.f90:840-841 uses TEMP, not B(J,5)).
 * alpha[0..n-1] diagonal, beta[0..n-2] codiagonal (reference beta(1..n-1)).
 * root[nroot] ascending, vect column-major n x nroot. */
int orc_givens_tridiag(int64_t n, const double *alpha, const double *beta, int64_t nroot,
                       double *root, double *vect)
{
    double eps = 1.0;
    for (;;) { eps = eps / 2.0; double e1 = eps + 1.0; if (e1 == 1.0) break; }  /* determine_epsilon */
    const double ETA = eps, THETA = DBL_MAX;
    const double DEL1 = ETA / 100.0, DELTA = ETA * ETA * 100.0;
    const double DELBIG = THETA * DELTA / 1000.0, THETA1 = 1000.0 / THETA;
    const double TOLER = ETA * 100.0;
    const double RPOWER = 8388608.0, RPOW1 = RPOWER / 2.0;
    double RAND1 = RPOWER - 3.0;
    if (nroot <= 0) return 0;
    if (n == 1) { root[0] = alpha[0]; vect[0] = 1.0; return 0; }
    /* scale to the Euclidean norm, summing over the packed array in column order */
    double factor = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        if (i > 0) factor = fmax(factor, fabs(beta[i - 1]));
        factor = fmax(factor, fabs(alpha[i]));
    }
    if (factor == 0.0) {
        for (int64_t i = 0; i < nroot; ++i) {
            for (int64_t j = 0; j < n; ++j) vect[i * n + j] = 0.0;
            vect[i * n + i] = 1.0;
            root[i] = 0.0;
        }
        return 0;
    }
    double anorm = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        if (i > 0) anorm = anorm + (beta[i - 1] / factor) * (beta[i - 1] / factor);
        anorm = anorm + (alpha[i] / factor) * (alpha[i] / factor) / 2.0;
    }
    anorm = sqrt(anorm * 2.0) * factor;
    double *d = malloc((size_t)n * sizeof(double));
    double *B1 = calloc((size_t)(n + 1), sizeof(double)), *B2 = calloc((size_t)(n + 1), sizeof(double));
    double *B3 = calloc((size_t)(n + 1), sizeof(double)), *B4 = calloc((size_t)(n + 1), sizeof(double));
    double *B5 = calloc((size_t)(n + 1), sizeof(double));
    double *V = calloc((size_t)(n + 2), sizeof(double));
    if (!d || !B1 || !B2 || !B3 || !B4 || !B5 || !V) return -2;
    /* 1-based views: d[j] = A(diag j), B1[j] = codiagonal j (j=1..n-1), B1[n] unused (0) */
    for (int64_t j = 1; j <= n; ++j) d[j - 1] = alpha[j - 1] / anorm;
    for (int64_t j = 1; j < n; ++j) B1[j] = beta[j - 1] / anorm;
    B1[n] = 0.0;
#define D(j) d[(j) - 1]
    /* STURM section */
    for (int64_t j = 1; j <= n; ++j) { B2[j] = D(j); B3[j] = B1[j] * B1[j]; }
    double *R = malloc((size_t)(nroot + 1) * sizeof(double));
    for (int64_t i = 1; i <= nroot; ++i) R[i] = 1.0;
    double rootl = -1.0;
    for (int64_t I = 1; I <= nroot; ++I) {
        double rootx = 1.0;
        for (int64_t J = I; J <= nroot; ++J) rootx = fmin(rootx, R[J]);
        R[I] = rootx;
        for (;;) {
            double trial = (rootl + R[I]) * 0.5;
            if (trial == rootl || trial == R[I]) break;
            int64_t nomtch = n, J = 1;
            double f0 = B2[J] - trial;
            for (;;) {
                if (fabs(f0) < THETA1) {
                    J += 2; nomtch -= 1;
                    if (J <= n) { f0 = B2[J] - trial; continue; }
                    break;
                }
                if (f0 >= 0.0) nomtch -= 1;
                J += 1;
                if (J > n) break;
                f0 = B2[J] - trial - B3[J - 1] / f0;
            }
            if (nomtch >= I) {
                R[I] = trial;
                int64_t nom = nroot < nomtch ? nroot : nomtch;
                R[nom] = trial;
            } else {
                rootl = trial;
            }
        }
    }
    /* TRIVEC section */
    for (int64_t i = 0; i < nroot * n; ++i) vect[i] = 1.0;
    int64_t IA = 0;
    double temp = 0.0;
    for (int64_t I = 1; I <= nroot; ++I) {
        double aroot = R[I];
        double *VI = vect + (I - 1) * n;  /* VI[j-1] = VECT(j,I) */
        if (I == 1 || !(fabs(R[I - 1] - aroot) < TOLER)) IA = -1;
        IA = IA + 1;
        double elim1 = D(1) - aroot, elim2 = B1[1];
        for (int64_t J = 1; J <= n - 1; ++J) {
            if (fabs(elim1) <= fabs(B1[J])) {
                B2[J] = B1[J]; B3[J] = D(J + 1) - aroot; B4[J] = B1[J + 1];
                temp = 1.0;
                if (fabs(B1[J]) > THETA1) temp = elim1 / B1[J];
                elim1 = elim2 - temp * B3[J];
                elim2 = -temp * B1[J + 1];
            } else {
                B2[J] = elim1; B3[J] = elim2; B4[J] = 0.0;
                temp = B1[J] / elim1;
                elim1 = D(J + 1) - aroot - temp * elim2;
                elim2 = B1[J + 1];
            }
            B5[J] = temp;
        }
        B2[n] = elim1; B3[n] = 0.0; B4[n] = 0.0; B4[n - 1] = 0.0;
        int iter = 1;
        if (IA != 0) {
            for (int64_t J = 1; J <= n; ++J) {
                RAND1 = fmod(4099.0 * RAND1, RPOWER);
                VI[J - 1] = RAND1 / RPOW1 - 1.0;
            }
        }
        for (;;) {
            /* back substitution (label 790); VECT(n+1), VECT(n+2) enter only times zero */
            for (int64_t L = n; L >= 1; --L) {
                for (;;) {
                    double v1 = (L + 1 <= n) ? VI[L] : 0.0, v2 = (L + 2 <= n) ? VI[L + 1] : 0.0;
                    double e = VI[L - 1] - v1 * B3[L] - v2 * B4[L];
                    if (fabs(e) > DELBIG) {
                        for (int64_t K = 0; K < n; ++K) VI[K] = VI[K] / DELBIG;
                        continue;
                    }
                    temp = B2[L];
                    if (fabs(B2[L]) < DELTA) temp = DELTA;
                    VI[L - 1] = e / temp;
                    break;
                }
            }
            if (iter == 1) {
                iter = 2;
                /* label 890: apply the elimination to the vector */
                double e = VI[0];
                for (int64_t J = 1; J <= n - 1; ++J) {
                    if (B2[J] == B1[J]) {
                        VI[J - 1] = VI[J];
                        e = e - VI[J] * temp;
                    } else {
                        VI[J - 1] = e;
                        e = VI[J] - e * B5[J];
                    }
                }
                VI[n - 1] = e;
                continue;
            }
            break;
        }
        /* label 800: orthogonalise a repeated-root vector to the previous IA vectors */
        for (int64_t J1 = 1; J1 <= IA; ++J1) {
            double *VK = vect + (I - J1 - 1) * n;
            temp = 0.0;
            for (int64_t J = 0; J < n; ++J) temp = temp + VI[J] * VK[J];
            for (int64_t J = 0; J < n; ++J) VI[J] = VI[J] - temp * VK[J];
        }
        /* label 900: normalise */
        double e = 0.0;
        for (int64_t J = 0; J < n; ++J) e = fmax(fabs(VI[J]), e);
        temp = 0.0;
        for (int64_t J = 0; J < n; ++J) { double e2 = VI[J] / e; temp = temp + e2 * e2; }
        temp = 1.0 / (sqrt(temp) * e);
        for (int64_t J = 0; J < n; ++J) {
            VI[J] = VI[J] * temp;
            if (fabs(VI[J]) < DEL1) VI[J] = 0.0;
        }
    }
    for (int64_t I = 1; I <= nroot; ++I) root[I - 1] = R[I] * anorm;
#undef D
    free(d); free(B1); free(B2); free(B3); free(B4); free(B5); free(V); free(R);
    return 0;
}

/* compute_ritzsystem, Source/secondary.f90:240-257: bji=|beta(n)*vect(n,i)|, intensity
 * vect(1,i)^2, sign of vect(1,i). */
int orc_ritz(int64_t n, const double *alpha, const double *beta /* beta[0..n] */,
             double *eig, double *bji, double *inten, int64_t *sign, double *vect)
{
    int rc = orc_givens_tridiag(n, alpha, beta + 1, n, eig, vect);
    if (rc) return rc;
    for (int64_t i = 0; i < n; ++i) {
        bji[i] = fabs(beta[n] * vect[i * n + (n - 1)]);
        sign[i] = vect[i * n] < 0 ? -1 : 1;
        inten[i] = vect[i * n] * vect[i * n];
    }
    return 0;
}

/* Gaussian broadening of convolve/main.f90:24-43 with convolve/sub.f90:1-11 (FWHM). */
void orc_convolve_fwhm(int64_t nlines, const double *c, const double *h, double xstart, double xend,
                       int64_t nt, double fwhm, double eshift, double *xo, double *yo)
{
    double dx = (xend - xstart) / (double)(nt + 1);
    double sigma = fwhm / (2.0 * sqrt(2.0 * log(2.0)));
    for (int64_t i = 0; i <= nt + 1; ++i) {
        double xx = xstart + (double)i * dx, y = 0.0;
        for (int64_t j = 0; j < nlines; ++j) y += h[j] * exp(-(xx - c[j]) * (xx - c[j]) / (2.0 * sigma * sigma));
        xo[i] = xx + eshift;
        yo[i] = y;
    }
}
