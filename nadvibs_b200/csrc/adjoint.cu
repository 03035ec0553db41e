// Adjoint of H.v with respect to the Hamiltonian's input coefficients (no counterpart in the
// reference, which has no derivative code).
//
// theta = (potterms in the nadvibs.in layout, concoef, omega).  With P_m[a][b] = <u_a|M_m|v_b>
// for every monomial m of the file (zero coefficients included), C[a][b] = <u_a|v_b> and
// K_k = sum_a <u_a|(n_k+1/2)|v_a>:
//   d<u|H|v>/d c(block (i,j), m) = s_m (P_m[i][j] + [i!=j] P_m[j][i]),  s_m = prod omega^(-p/2)
//   d<u|H|v>/d concoef(i,j)      = C[i][j] + [i!=j] C[j][i]
//   d<u|H|v>/d omega_k           = K_k + sum_terms sum_pairs (-p_k/(2 omega_k)) coef_ab P_m[a][b]
// M_m is the monomial's operator exactly as H.v applies it (analytic <m|x^p|n>, cubic quirk
// per the handle's option); couplings between different states are taken symmetric.
// One kernel pass per chunk of monomials: each thread walks rows (grid-stride) and keeps
// TB*S*S FP64 accumulators; block partials are summed on the host in a fixed order.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "handle.h"

namespace nvb {

#define CK(x)                                                                                    \
    do {                                                                                         \
        cudaError_t e_ = (x);                                                                    \
        if (e_ != cudaSuccess) fail(NVB_ERR_CUDA, std::string(#x ": ") + cudaGetErrorString(e_)); \
    } while (0)

struct AdjStep {  // one shift of one monomial
    int mono;      // chunk-local monomial index
    int nm;
    int mode[MAX_ORDER];
    int sig[MAX_ORDER];
    int etab[MAX_ORDER];
    long long stride;
};

constexpr int ADJ_THREADS = 256;

template <typename T, int S, int TB>
__global__ void __launch_bounds__(ADJ_THREADS) k_adjoint(const AdjStep *__restrict__ steps, int nsteps,
                                                        const double *__restrict__ etab, int etab_len,
                                                        const int *__restrict__ nfunc,
                                                        const long long *__restrict__ shft, int M, long long dimen,
                                                        const T *__restrict__ u, const T *__restrict__ v,
                                                        double *__restrict__ part) {
    extern __shared__ double s_etab[];
    for (int i = threadIdx.x; i < etab_len; i += blockDim.x) s_etab[i] = etab[i];
    __syncthreads();
    double acc[TB][S][S];
#pragma unroll
    for (int t = 0; t < TB; ++t)
#pragma unroll
        for (int a = 0; a < S; ++a)
#pragma unroll
            for (int b = 0; b < S; ++b) acc[t][a][b] = 0.0;
    const long long gstride = (long long)gridDim.x * blockDim.x;
    for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < dimen; r += gstride) {
        int dig[64];
        long long rem = r;
        for (int k = 0; k < M; ++k) {
            const long long d = rem / shft[k];
            rem -= d * shft[k];
            dig[k] = (int)d;
        }
        double ua[S];
#pragma unroll
        for (int a = 0; a < S; ++a) ua[a] = (double)u[a * dimen + r];
        for (int i = 0; i < nsteps; ++i) {
            const AdjStep *st = steps + i;
            double e = 1.0;
            bool ok = true;
            const int nm = st->nm;
            for (int l = 0; l < nm; ++l) {
                const int md = st->mode[l];
                const int n = dig[md], nc = n + st->sig[l];
                if (nc < 0 || nc >= nfunc[md]) { ok = false; break; }
                e *= s_etab[st->etab[l] + (nc < n ? nc : n)];
            }
            if (!ok) continue;
            const long long c = r + st->stride;
            double vb[S];
#pragma unroll
            for (int b = 0; b < S; ++b) vb[b] = (double)v[b * dimen + c] * e;
            const int t = st->mono;
#pragma unroll
            for (int tt = 0; tt < TB; ++tt)
                if (tt == t)
#pragma unroll
                    for (int a = 0; a < S; ++a)
#pragma unroll
                        for (int b = 0; b < S; ++b) acc[tt][a][b] += ua[a] * vb[b];
        }
    }
    __shared__ double red[ADJ_THREADS];
#pragma unroll
    for (int t = 0; t < TB; ++t)
#pragma unroll
        for (int a = 0; a < S; ++a)
#pragma unroll
            for (int b = 0; b < S; ++b) {
                red[threadIdx.x] = acc[t][a][b];
                __syncthreads();
                for (int o = blockDim.x / 2; o > 0; o >>= 1) {
                    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
                    __syncthreads();
                }
                if (threadIdx.x == 0) part[(long long)blockIdx.x * TB * S * S + (t * S + a) * S + b] = red[0];
                __syncthreads();
            }
}

// overlaps C[a][b] = <u_a|v_b> and harmonic K_k = sum_a <u_a|(n_k+1/2)|v_a>
template <typename T, int S>
__global__ void __launch_bounds__(ADJ_THREADS) k_adj_diag(const long long *__restrict__ shft, int M, long long dimen,
                                                         const T *__restrict__ u, const T *__restrict__ v,
                                                         double *__restrict__ part) {
    double c[S][S];
    double kin[64];
#pragma unroll
    for (int a = 0; a < S; ++a)
#pragma unroll
        for (int b = 0; b < S; ++b) c[a][b] = 0.0;
    for (int k = 0; k < M; ++k) kin[k] = 0.0;
    const long long gstride = (long long)gridDim.x * blockDim.x;
    for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < dimen; r += gstride) {
        double ua[S], vb[S], uv = 0.0;
#pragma unroll
        for (int a = 0; a < S; ++a) {
            ua[a] = (double)u[a * dimen + r];
            vb[a] = (double)v[a * dimen + r];
            uv += ua[a] * vb[a];
        }
#pragma unroll
        for (int a = 0; a < S; ++a)
#pragma unroll
            for (int b = 0; b < S; ++b) c[a][b] += ua[a] * vb[b];
        long long rem = r;
        for (int k = 0; k < M; ++k) {
            const long long d = rem / shft[k];
            rem -= d * shft[k];
            kin[k] += ((double)d + 0.5) * uv;
        }
    }
    __shared__ double red[ADJ_THREADS];
    const int nout = S * S + M;
    for (int q = 0; q < nout; ++q) {
        double val = 0.0;
#pragma unroll
        for (int a = 0; a < S; ++a)
#pragma unroll
            for (int b = 0; b < S; ++b)
                if (q == a * S + b) val = c[a][b];
        if (q >= S * S) val = kin[q - S * S];
        red[threadIdx.x] = val;
        __syncthreads();
        for (int o = blockDim.x / 2; o > 0; o >>= 1) {
            if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
            __syncthreads();
        }
        if (threadIdx.x == 0) part[(long long)blockIdx.x * nout + q] = red[0];
        __syncthreads();
    }
}

// ---- ordr <= 2: every P_m is an entry of a Gram matrix G = A^T B over the rows of a state,
//   A = [u_a, X_k u_a],  B = [v_b, X_k v_b, x_k^2 v_b, (n_k + 1/2) v_b]
// (X_k the ladder part <n|x|n+-1> along mode k, x_k^2 the analytic square, both truncated to
// the basis exactly as H.v applies them):
//   <u_a|v_b> = G[u_a][v_b],  <u_a|x_k|v_b> = G[u_a][X_k v_b],  <u_a|x_k^2|v_b> = G[u_a][x_k^2 v_b],
//   <u_a|x_k x_l|v_b> = G[X_k u_a][X_l v_b] (X_k symmetric),  K_k = sum_a G[u_a][(n_k+1/2) v_a].
// Only G1 = u^T B and G2 = (X u)^T (X v) are needed.  One kernel expands the columns of a
// tile of rows into shared memory and accumulates both; block partials are summed in a fixed
// order.

constexpr int GRAM_TR = 64;      // rows per shared-memory tile (a multiple of 4)
static_assert(GRAM_TR % 4 == 0, "the Gram sums are unrolled by 4 rows");
constexpr int GRAM_MAXPER = 8;   // Gram outputs: S*(3M+1)*S + (MS)^2 <= 8*256 (4-output tasks <= 256 threads)

// Per block: for each tile of GRAM_TR rows, the expanded columns of those rows go to shared
// memory (one thread per (row, state)), then every thread accumulates its Gram outputs over
// the tile.  Outputs o < n1: G1[a][j] = <u_a, B_j>; o >= n1: G2[(k,a)][(l,b)] = <X_k u_a, X_l v_b>.
template <typename T>
__global__ void __launch_bounds__(256, 4) k_adj_gram(const T *__restrict__ u, const T *__restrict__ v,
                                                 const double *__restrict__ etab, int nmax,
                                                 const int *__restrict__ nfunc, const long long *__restrict__ shft,
                                                 int M, int S, long long dimen, int accumulate,
                                                 double *__restrict__ part) {
    extern __shared__ double sm[];
    const int MS = M * S, nA = S + MS, nB = S + 3 * MS;
    const int n1 = S * nB, n2 = MS * MS, nout = n1 + n2;
    double *sA = sm, *sB = sm + GRAM_TR * nA;  // [row][col]
    const double *E1 = etab + (0 * ETAB_J + 1) * nmax;  // <m|x|m+1>
    const double *E2 = etab + (1 * ETAB_J + 2) * nmax;  // <m|x^2|m+2>
    const double *D2 = etab + (1 * ETAB_J + 0) * nmax;  // <m|x^2|m>
    const int tid = threadIdx.x, nth = blockDim.x;
    const bool small = dimen <= 0xFFFFFFFFll;
    // this thread's task: 4 outputs of one row ia of G1 or G2, and its row group
    const int K1 = (nB + 3) / 4, K2 = (MS + 3) / 4;
    const int ntask = S * K1 + MS * K2;
    const int ngrp = nth / ntask > 0 ? nth / ntask : 1;  // row groups splitting the tile
    const int task = tid % ntask, rg = tid / ntask;
    int ia, jb0, kst, nq, obase;
    if (task < S * K1) {
        ia = task / K1;
        const int k = task - ia * K1;
        jb0 = k;
        kst = K1;
        nq = k + 3 * K1 < nB ? 4 : (nB - k + K1 - 1) / K1;
        obase = ia * nB + k;
    } else {
        const int t2 = task - S * K1;
        const int i2 = t2 / K2, k = t2 - i2 * K2;
        ia = S + i2;
        jb0 = S + k;
        kst = K2;
        nq = k + 3 * K2 < MS ? 4 : (MS - k + K2 - 1) / K2;
        obase = n1 + i2 * MS + k;
    }
    const int active_rg = rg < ngrp;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (long long t0 = (long long)blockIdx.x * GRAM_TR; t0 < dimen; t0 += (long long)gridDim.x * GRAM_TR) {
        for (int e = tid; e < GRAM_TR * S; e += nth) {
            const int rl = e % GRAM_TR, s = e / GRAM_TR;
            const long long r = t0 + rl;
            double *a = sA + rl * nA, *b = sB + rl * nB;
            if (r >= dimen) {
                a[s] = 0.0;
                b[s] = 0.0;
                for (int k = 0; k < M; ++k) {
                    a[S + k * S + s] = 0.0;
                    b[S + k * S + s] = b[S + MS + k * S + s] = b[S + 2 * MS + k * S + s] = 0.0;
                }
                continue;
            }
            const T *us = u + s * dimen, *vs = v + s * dimen;
            const double u0 = (double)us[r], v0 = (double)vs[r];
            a[s] = u0;
            b[s] = v0;
            long long rem = r;
            for (int k = 0; k < M; ++k) {
                const long long sh = shft[k];
                // digit of mode k (32-bit division when the state block has < 2^32 rows)
                const int d = small ? (int)((unsigned)rem / (unsigned)sh) : (int)(rem / sh);
                rem -= (long long)d * sh;
                const int nf = nfunc[k];
                double xu = 0.0, xv = 0.0, tv = D2[d] * v0;
                if (d + 1 < nf) {
                    const double e = E1[d];
                    xu += e * (double)us[r + sh];
                    xv += e * (double)vs[r + sh];
                }
                if (d >= 1) {
                    const double e = E1[d - 1];
                    xu += e * (double)us[r - sh];
                    xv += e * (double)vs[r - sh];
                }
                if (d + 2 < nf) tv += E2[d] * (double)vs[r + 2 * sh];
                if (d >= 2) tv += E2[d - 2] * (double)vs[r - 2 * sh];
                a[S + k * S + s] = xu;
                b[S + k * S + s] = xv;
                b[S + MS + k * S + s] = tv;
                b[S + 2 * MS + k * S + s] = ((double)d + 0.5) * v0;
            }
        }
        __syncthreads();
        // G1 row ia < S: tasks k < K1, outputs jb = k + q K1 (q < 4) of the nB columns of B;
        // G2 row ia >= S: tasks k < K2, outputs jb = S + k + q K2 of the MS columns X v.  Lanes
        // of a task row read consecutive words of sB; the row groups split the tile's rows.
        if (task < ntask && active_rg) {
            const double *pa = sA + ia;
            const double *pb = sB + jb0;
            for (int r = rg; r < GRAM_TR; r += ngrp) {
                const double a = pa[r * nA];
                const double *b = pb + r * nB;
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    if (q < nq) acc[q] += a * b[q * kst];
            }
        }
        __syncthreads();
    }
    // sum the row groups' partials (in group order) and update the block's partials:
    // overwritten, or (accumulate) summed over the calls of a reverse sweep by the block that
    // owns them, so one reduction over blocks serves all its steps
    double *red = sm;  // reuses the tile: [ngrp][ntask][4]
    if (task < ntask && active_rg)
#pragma unroll
        for (int q = 0; q < 4; ++q) red[(rg * ntask + task) * 4 + q] = acc[q];
    __syncthreads();
    if (task < ntask && rg == 0) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            if (q >= nq) break;
            double v = 0.0;
            for (int g2 = 0; g2 < ngrp; ++g2) v += red[(g2 * ntask + task) * 4 + q];
            double *pp = part + (long long)blockIdx.x * nout + obase + q * kst;
            *pp = accumulate ? *pp + v : v;
        }
    }
}

// shared memory of one Gram block: the expanded tile, or the row groups' partials at the end
static size_t gram_smem(int S, int M) {
    const int MS = M * S, nA = S + MS, nB = S + 3 * MS;
    return std::max<size_t>((size_t)GRAM_TR * (nA + nB), 4 * 256) * sizeof(double);
}

static bool gram_fits(int S, int M) {
    const int MS = M * S, nB = S + 3 * MS;
    const int ntask = S * ((nB + 3) / 4) + MS * ((MS + 3) / 4);  // one thread per 4-output task
    return S * nB + MS * MS <= GRAM_MAXPER * 256 && ntask <= 256 && gram_smem(S, M) <= 200 * 1024;
}

// out[o] (+)= sum over blocks g = 0..ng-1 of part[g][o]: one warp per output, lane l summing
// blocks l, l + 32, ... in order, then a fixed butterfly (the same order on every call)
__global__ void k_gram_reduce(const double *__restrict__ part, int ng, int nout, int accumulate,
                              double *__restrict__ out) {
    const int o = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (o >= nout) return;
    double s = 0.0;
    for (int g = lane; g < ng; g += 32) s += part[(long long)g * nout + o];
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) s += __shfl_xor_sync(0xffffffffu, s, d);
    if (lane == 0) out[o] = accumulate ? out[o] + s : s;
}

// ---- ordr 3: P_m for every monomial of degree <= 3 is an entry of G = A^T B with
//   A = [u_a, X_k u_a, x_k^2 u_a],
//   B = [v_b, X_k v_b, x_k^2 v_b, (n_k + 1/2) v_b, x_k^3 v_b, X_l X_m v_b (l < m)]
// (x_k^p with the analytic truncated elements H.v applies, the cubic quirk included; all
// operators symmetric and operators on different modes commuting):
//   x_k: <u_a, X_k v_b>   x_k^2: <u_a, x_k^2 v_b>   x_k^3: <u_a, x_k^3 v_b>
//   x_k x_l: <X_k u_a, X_l v_b>   x_k^2 x_l: <x_k^2 u_a, X_l v_b>
//   x_k x_l x_m (k < l < m): <X_k u_a, X_l X_m v_b>,   C = <u_a, v_b>,   K_k = sum_a <u_a, (n_k+1/2) v_a>.
// Only those entries are formed: a task list of (A column, up to 4 B columns).  Per tile of
// G3_TR = 32 rows the columns are expanded into shared memory (digits decoded once per row;
// a warp per (state, mode) or (state, pair of modes) family and a lane per row, so each gather
// reads consecutive rows), then every thread accumulates its tasks over the tile's rows.
// Block partials are summed in a fixed order.

constexpr int G3_TR = 64;  // rows per tile: two per lane
constexpr int G3_THREADS = 512;
struct G3Task {
    short ia, nq;
    short jb[4];
};

template <typename T, int TPT>
__global__ void __launch_bounds__(G3_THREADS, 1) k_adj_gram3(const T *__restrict__ u, const T *__restrict__ v,
                                                          const double *__restrict__ etab, int nmax,
                                                          const int *__restrict__ nfunc,
                                                          const long long *__restrict__ shft, int M, int S,
                                                          long long dimen, const G3Task *__restrict__ tasks,
                                                          int ntask, int accumulate, double *__restrict__ part) {
    extern __shared__ double sm[];
    const int MS = M * S, P2 = M * (M - 1) / 2, nA = S + 2 * MS, nB = S + 4 * MS + P2 * S;
    const int nB1 = nB + 1;  // column nB stays zero: the padding of tasks with fewer than 4 outputs
    const int nout = 4 * ntask;
    double *sA = sm, *sB = sm + G3_TR * nA;             // [row][col]
    double *stab = sB + G3_TR * nB1;                     // element rows E1, E2, D2, E31, E33 [nmax]
    long long *ssh = reinterpret_cast<long long *>(stab + 5 * nmax);  // [M] strides
    int *sdig = reinterpret_cast<int *>(ssh + M);        // [row][mode]
    int *spair = sdig + G3_TR * M;                       // pair p: l | m << 8
    int *snf = spair + P2;                               // [M] nfunc
    const int tid = threadIdx.x, nth = blockDim.x;
    const bool small = dimen <= 0xFFFFFFFFll;
    for (int i = tid; i < nmax; i += nth) {
        stab[0 * nmax + i] = etab[(0 * ETAB_J + 1) * nmax + i];  // <n|x|n+1>
        stab[1 * nmax + i] = etab[(1 * ETAB_J + 2) * nmax + i];  // <n|x^2|n+2>
        stab[2 * nmax + i] = etab[(1 * ETAB_J + 0) * nmax + i];  // <n|x^2|n>
        stab[3 * nmax + i] = etab[(2 * ETAB_J + 1) * nmax + i];  // <n|x^3|n+1>
        stab[4 * nmax + i] = etab[(2 * ETAB_J + 3) * nmax + i];  // <n|x^3|n+3>
    }
    for (int k = tid; k < M; k += nth) {
        ssh[k] = shft[k];
        snf[k] = nfunc[k];
    }
    for (int e = tid; e < G3_TR; e += nth) sB[e * nB1 + nB] = 0.0;
    if (tid == 0) {
        int q = 0;
        for (int l = 0; l < M; ++l)
            for (int m = l + 1; m < M; ++m) spair[q++] = l | (m << 8);
    }
    const double *E1 = stab, *E2 = stab + nmax, *D2 = stab + 2 * nmax, *E31 = stab + 3 * nmax, *E33 = stab + 4 * nmax;
    // this thread's tasks: A column and 4 B columns (padded with the zero column)
    int ia[TPT], jb[TPT][4], nq[TPT];
    double acc[TPT][4];
#pragma unroll
    for (int j = 0; j < TPT; ++j) {
        const int t = tid + j * nth;
        G3Task tk = t < ntask ? tasks[t] : G3Task{0, 0, {0, 0, 0, 0}};
        ia[j] = tk.ia;
        nq[j] = tk.nq;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            jb[j][q] = q < tk.nq ? tk.jb[q] : nB;
            acc[j][q] = 0.0;
        }
    }
    __syncthreads();
    static_assert(G3_TR % 32 == 0, "whole warps of rows");
    const int lane = tid & 31, wid = tid >> 5, nwarp = nth >> 5;
    for (long long t0 = (long long)blockIdx.x * G3_TR; t0 < dimen; t0 += (long long)gridDim.x * G3_TR) {
        // digits of the tile's rows (one thread per row)
        for (int e = tid; e < G3_TR; e += nth) {
            const long long r = t0 + e;
            if (r >= dimen) continue;
            long long rem = r;
            for (int k = 0; k < M; ++k) {
                const long long sh = ssh[k];
                const int d = small ? (int)((unsigned)rem / (unsigned)sh) : (int)(rem / sh);
                rem -= (long long)d * sh;
                sdig[e * M + k] = d;
            }
        }
        __syncthreads();
        // column families: a warp per (state, mode) or (state, pair of modes), a lane per row
        // (G3_TR / 32 rows per lane), so each gather of a warp reads consecutive rows
        if (wid < S) {
            const int s = wid;
#pragma unroll
            for (int hr = 0; hr < G3_TR / 32; ++hr) {
                const int e = lane + 32 * hr;
                const long long r = t0 + e;
                sA[e * nA + s] = r < dimen ? (double)u[(long long)s * dimen + r] : 0.0;
                sB[e * nB1 + s] = r < dimen ? (double)v[(long long)s * dimen + r] : 0.0;
            }
        }
        for (int f = wid; f < S * M; f += nwarp)
#pragma unroll
        for (int hr = 0; hr < G3_TR / 32; ++hr) {
            const int e = lane + 32 * hr;
            const long long r = t0 + e;
            const bool in = r < dimen;
            double *a = sA + e * nA, *b = sB + e * nB1;
            const int s = f / M, k = f - s * M;
            double xu = 0.0, xv = 0.0, x2u = 0.0, x2v = 0.0, x3v = 0.0, hv = 0.0;
            if (in) {
                const T *ur = u + (long long)s * dimen + r, *vr = v + (long long)s * dimen + r;
                const int d = sdig[e * M + k], nf = snf[k];
                const long long sh = ssh[k];
                const double u0 = (double)ur[0], v0 = (double)vr[0];
                x2u = D2[d] * u0;
                x2v = D2[d] * v0;
                hv = ((double)d + 0.5) * v0;
                if (d + 1 < nf) {
                    const double up = (double)ur[sh], vp = (double)vr[sh];
                    xu += E1[d] * up;
                    xv += E1[d] * vp;
                    x3v += E31[d] * vp;
                }
                if (d >= 1) {
                    const double um = (double)ur[-sh], vm = (double)vr[-sh];
                    xu += E1[d - 1] * um;
                    xv += E1[d - 1] * vm;
                    x3v += E31[d - 1] * vm;
                }
                if (d + 2 < nf) {
                    x2u += E2[d] * (double)ur[2 * sh];
                    x2v += E2[d] * (double)vr[2 * sh];
                }
                if (d >= 2) {
                    x2u += E2[d - 2] * (double)ur[-2 * sh];
                    x2v += E2[d - 2] * (double)vr[-2 * sh];
                }
                if (d + 3 < nf) x3v += E33[d] * (double)vr[3 * sh];
                if (d >= 3) x3v += E33[d - 3] * (double)vr[-3 * sh];
            }
            a[S + k * S + s] = xu;
            a[S + MS + k * S + s] = x2u;
            b[S + k * S + s] = xv;
            b[S + MS + k * S + s] = x2v;
            b[S + 2 * MS + k * S + s] = hv;
            b[S + 3 * MS + k * S + s] = x3v;
        }
        for (int f = wid; f < S * P2; f += nwarp)
#pragma unroll
        for (int hr = 0; hr < G3_TR / 32; ++hr) {
            const int e = lane + 32 * hr;
            const long long r = t0 + e;
            const bool in = r < dimen;
            double *b = sB + e * nB1;
            const int s = f / P2, p = f - s * P2, l = spair[p] & 255, m = spair[p] >> 8;
            double xx = 0.0;
            if (in) {
                const T *vr = v + (long long)s * dimen + r;
                const int dl = sdig[e * M + l], dm = sdig[e * M + m], nl = snf[l], nm = snf[m];
                const long long shl = ssh[l], shm = ssh[m];
                const bool lp = dl + 1 < nl, lm = dl >= 1, mp = dm + 1 < nm, mm = dm >= 1;
                const double elp = lp ? E1[dl] : 0.0, elm = lm ? E1[dl - 1] : 0.0;
                const double emp = mp ? E1[dm] : 0.0, emm = mm ? E1[dm - 1] : 0.0;
                if (lp && mp) xx += elp * emp * (double)vr[shl + shm];
                if (lp && mm) xx += elp * emm * (double)vr[shl - shm];
                if (lm && mp) xx += elm * emp * (double)vr[shm - shl];
                if (lm && mm) xx += elm * emm * (double)vr[-shl - shm];
            }
            b[S + 4 * MS + p * S + s] = xx;
        }
        __syncthreads();
        // Gram sums over the tile's rows: 4 outputs per task, no branches
#pragma unroll
        for (int j = 0; j < TPT; ++j) {
            const double *pa = sA + ia[j];
            const double *p0 = sB + jb[j][0], *p1 = sB + jb[j][1], *p2 = sB + jb[j][2], *p3 = sB + jb[j][3];
            double c0 = acc[j][0], c1 = acc[j][1], c2 = acc[j][2], c3 = acc[j][3];
#pragma unroll 8
            for (int rr = 0; rr < G3_TR; ++rr) {
                const double av = pa[rr * nA];
                c0 += av * p0[rr * nB1];
                c1 += av * p1[rr * nB1];
                c2 += av * p2[rr * nB1];
                c3 += av * p3[rr * nB1];
            }
            acc[j][0] = c0;
            acc[j][1] = c1;
            acc[j][2] = c2;
            acc[j][3] = c3;
        }
        __syncthreads();
    }
#pragma unroll
    for (int j = 0; j < TPT; ++j) {
        const int t = tid + j * nth;
        if (t >= ntask) continue;
#pragma unroll
        for (int q = 0; q < 4; ++q)
            if (q < nq[j]) {
                double *pp = part + (long long)blockIdx.x * nout + 4 * t + q;
                *pp = accumulate ? *pp + acc[j][q] : acc[j][q];
            }
    }
}

// Column indices of the ordr-3 Gram (host side; the kernel lays them out identically).
struct G3Cols {
    int S, M, MS, P2, nA, nB;
    G3Cols(int S_, int M_) : S(S_), M(M_), MS(M_ * S_), P2(M_ * (M_ - 1) / 2) {
        nA = S + 2 * MS;
        nB = S + 4 * MS + P2 * S;
    }
    int u(int a) const { return a; }
    int Xu(int k, int a) const { return S + k * S + a; }
    int x2u(int k, int a) const { return S + MS + k * S + a; }
    int v(int b) const { return b; }
    int Xv(int k, int b) const { return S + k * S + b; }
    int x2v(int k, int b) const { return S + MS + k * S + b; }
    int hv(int k, int b) const { return S + 2 * MS + k * S + b; }
    int x3v(int k, int b) const { return S + 3 * MS + k * S + b; }
    int pair(int l, int m) const { return l * M - l * (l + 1) / 2 + (m - l - 1); }  // l < m
    int XXv(int l, int m, int b) const { return S + 4 * MS + pair(l, m) * S + b; }
};

// The task list (A column, up to 4 B columns) and the output index of every needed (A, B) pair.
static void gram3_tasks(int S, int M, std::vector<G3Task> &tasks, std::vector<int> &index) {
    const G3Cols c(S, M);
    tasks.clear();
    index.assign((size_t)c.nA * c.nB, -1);
    // the row's B columns in ascending order, dealt to its K tasks round-robin (task k takes
    // columns k, k + K, k + 2K, k + 3K): neighbouring threads read neighbouring words of a
    // shared-memory row (no bank conflicts from a 4-column stride)
    auto row = [&](int ia, std::vector<int> jbs) {
        std::sort(jbs.begin(), jbs.end());
        const int n = (int)jbs.size(), K = (n + 3) / 4, t0 = (int)tasks.size();
        for (int k = 0; k < K; ++k) {
            G3Task t{};
            t.ia = (short)ia;
            for (int q = 0; q < 4 && k + q * K < n; ++q) {
                t.jb[q] = (short)jbs[k + q * K];
                index[(size_t)ia * c.nB + jbs[k + q * K]] = 4 * (t0 + k) + q;
                t.nq = (short)(q + 1);
            }
            tasks.push_back(t);
        }
    };
    for (int a = 0; a < S; ++a) {
        std::vector<int> j;
        for (int b = 0; b < S; ++b) j.push_back(c.v(b));
        for (int k = 0; k < M; ++k)
            for (int b = 0; b < S; ++b) {
                j.push_back(c.Xv(k, b));
                j.push_back(c.x2v(k, b));
                j.push_back(c.hv(k, b));
                j.push_back(c.x3v(k, b));
            }
        row(c.u(a), j);
    }
    for (int k = 0; k < M; ++k)
        for (int a = 0; a < S; ++a) {
            std::vector<int> j;
            for (int l = 0; l < M; ++l)
                if (l != k)
                    for (int b = 0; b < S; ++b) j.push_back(c.Xv(l, b));
            for (int l = k + 1; l < M; ++l)
                for (int m = l + 1; m < M; ++m)
                    for (int b = 0; b < S; ++b) j.push_back(c.XXv(l, m, b));
            row(c.Xu(k, a), j);
            std::vector<int> j2;
            for (int l = 0; l < M; ++l)
                if (l != k)
                    for (int b = 0; b < S; ++b) j2.push_back(c.Xv(l, b));
            row(c.x2u(k, a), j2);
        }
}

static size_t gram3_smem(int S, int M, int nmax) {
    const G3Cols c(S, M);
    return (size_t)(G3_TR * (c.nA + c.nB + 1) + 5 * nmax) * sizeof(double) + (size_t)M * sizeof(long long) +
           (size_t)(G3_TR * M + c.P2 + M) * sizeof(int);
}

static bool gram3_fits(int S, int M) {
    if (M > 255) return false;
    const G3Cols c(S, M);
    std::vector<G3Task> t;
    std::vector<int> idx;
    if (c.nB > 32767 || c.nA > 32767) return false;
    gram3_tasks(S, M, t, idx);
    return gram3_smem(S, M, 64) <= 200 * 1024 && t.size() <= (size_t)4 * G3_THREADS;
}

static int gram3_len(int S, int M) {
    std::vector<G3Task> t;
    std::vector<int> idx;
    gram3_tasks(S, M, t, idx);
    return 4 * (int)t.size();
}

// the task table on the device and the grid, once per handle
static void gram3_setup(nvb_handle *h) {
    if (h->d_g3task) return;
    std::vector<G3Task> t;
    std::vector<int> idx;
    gram3_tasks(h->sys.S, h->sys.M, t, idx);
    CK(cudaMalloc(&h->d_g3task, t.size() * sizeof(G3Task)));
    CK(cudaMemcpy(h->d_g3task, t.data(), t.size() * sizeof(G3Task), cudaMemcpyHostToDevice));
    h->g3_ntask = (int)t.size();
    int nsm = 0;
    CK(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->device));
    h->g3_grid = (int)std::min<long long>((h->sys.dimen + G3_TR - 1) / G3_TR, (long long)nsm * 2);
}

static int gram3_grid(const nvb_handle *h) {
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->device);
    return (int)std::min<long long>((h->sys.dimen + G3_TR - 1) / G3_TR, (long long)nsm * 2);
}

template <typename T, int TPT>
static void gram3_kernel(nvb_handle *h, const T *u, const T *v, int accumulate, double *part, size_t shm) {
    auto k = k_adj_gram3<T, TPT>;
    if (shm > 48 * 1024) CK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm));
    const Plan &pl = h->plan;
    k<<<h->g3_grid, G3_THREADS, shm, h->stream>>>(u, v, pl.d_etab, pl.nmax, pl.d_nfunc, pl.d_shft, h->sys.M, h->sys.S,
                                                   h->sys.dimen, (const G3Task *)h->d_g3task, h->g3_ntask,
                                                   accumulate, part);
}

// G (+)= the ordr-3 Gram entries of (u, v) through block partials part[g3_grid * gram3_len];
// G == nullptr: only the partials (accumulate: added to those already there).
template <typename T>
static void gram3_launch(nvb_handle *h, const T *u, const T *v, double *G, int accumulate, double *part) {
    const int S = h->sys.S, M = h->sys.M;
    if (!gram3_fits(S, M)) fail(NVB_ERR_ARG, "adjoint: too many modes x states for the ordr-3 Gram path");
    gram3_setup(h);
    const size_t shm = gram3_smem(S, M, h->plan.nmax);
    if (shm > 227 * 1024) fail(NVB_ERR_ARG, "adjoint: the ordr-3 Gram tile does not fit in shared memory");
    const int tpt = (h->g3_ntask + G3_THREADS - 1) / G3_THREADS;
    const int acc = G ? 0 : accumulate;
    switch (tpt) {
    case 1: gram3_kernel<T, 1>(h, u, v, acc, part, shm); break;
    case 2: gram3_kernel<T, 2>(h, u, v, acc, part, shm); break;
    case 3: gram3_kernel<T, 3>(h, u, v, acc, part, shm); break;
    default: gram3_kernel<T, 4>(h, u, v, acc, part, shm); break;
    }
    const int nout = 4 * h->g3_ntask;
    if (G) k_gram_reduce<<<(nout * 32 + 255) / 256, 256, 0, h->stream>>>(part, h->g3_grid, nout, accumulate, G);
    CK(cudaGetLastError());
}

static int smax_of(int p, int64_t nf) {
    int s = p;
    while (s > nf - 1) s -= 2;
    return s;
}

struct Mono {
    std::vector<int> modes, pows;
};

static std::vector<Mono> all_monomials(const System &sys) {
    std::vector<Mono> out;
    for (int d = 1; d <= sys.ordr; ++d)
        for (auto &dig : monomials(sys.M, d)) {
            Mono m;
            for (int x : dig) {
                auto it = std::find(m.modes.begin(), m.modes.end(), x - 1);
                if (it == m.modes.end()) {
                    m.modes.push_back(x - 1);
                    m.pows.push_back(1);
                } else m.pows[it - m.modes.begin()] += 1;
            }
            out.push_back(m);
        }
    return out;
}

template <typename T, int S, int TB>
static void launch_chunk(nvb_handle *h, const std::vector<AdjStep> &steps, const T *u, const T *v, double *part,
                         int grid) {
    AdjStep *d = nullptr;
    CK(cudaMalloc((void **)&d, std::max<size_t>(1, steps.size()) * sizeof(AdjStep)));
    CK(cudaMemcpyAsync(d, steps.data(), steps.size() * sizeof(AdjStep), cudaMemcpyHostToDevice, h->stream));
    const Plan &pl = h->plan;
    k_adjoint<T, S, TB><<<grid, ADJ_THREADS, pl.h_etab.size() * sizeof(double), h->stream>>>(
        d, (int)steps.size(), pl.d_etab, (int)pl.h_etab.size(), pl.d_nfunc, pl.d_shft, pl.M, pl.dimen, u, v, part);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(h->stream));
    cudaFree(d);
}

// Length of the raw Gram output of the ordr <= 2 path: G1 = u^T B (S x nB), G2 = (X u)^T (X v)
// (MS x MS), with A = [u (S), X u (M S)] and B = [v (S), X v (M S), x^2 v (M S), (n+1/2) v (M S)].
static int gram_len(int S, int M) {
    const int MS = M * S, nB = S + 3 * MS;
    return S * nB + MS * MS;
}

static int gram_grid(const nvb_handle *h) {
    return (int)std::min<long long>((h->sys.dimen + GRAM_TR - 1) / GRAM_TR, 148 * 4);
}

// G (+)= the Gram matrices of (u, v) on the device, through block partials part[gram_grid *
// gram_len] (no host synchronisation).  G == nullptr: only the block partials are formed
// (accumulate: added to the partials already there); adjoint_gram_reduce sums them later.
template <typename T>
static void gram_launch(nvb_handle *h, const T *u, const T *v, double *G, int accumulate, double *part) {
    const System &sys = h->sys;
    const Plan &pl = h->plan;
    const int S = sys.S, M = sys.M;
    const int nout = gram_len(S, M);
    if (!gram_fits(S, M)) fail(NVB_ERR_ARG, "adjoint: too many modes x states for the Gram path");
    const long long Ns = sys.dimen;
    const int grid = gram_grid(h);
    const size_t shm = gram_smem(S, M);
    if (shm > 48 * 1024) CK(cudaFuncSetAttribute(k_adj_gram<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm));
    k_adj_gram<T><<<grid, 256, shm, h->stream>>>(u, v, pl.d_etab, pl.nmax, pl.d_nfunc, pl.d_shft, M, S, Ns,
                                                 G ? 0 : accumulate, part);
    if (G) k_gram_reduce<<<(nout * 32 + 255) / 256, 256, 0, h->stream>>>(part, grid, nout, accumulate, G);
    CK(cudaGetLastError());
}

// P[m][a][b] for the monomials of an ordr <= 2 system and Cq = (C[a][b], K_k) from the Gram
// matrices (host copy Gh of length gram_len).
static void gram_pc(const nvb_handle *h, const std::vector<double> &Gh, const std::vector<Mono> &monos,
                    std::vector<double> &P, std::vector<double> &Cq) {
    const System &sys = h->sys;
    const int S = sys.S, M = sys.M;
    const int MS = M * S, nB = S + 3 * MS;
    const int n1 = S * nB;
    auto g = [&](int a, int j) { return Gh[(size_t)a * nB + j]; };            // <u_a, B_j>
    auto g2 = [&](int k, int a, int l, int b) { return Gh[n1 + (size_t)(k * S + a) * MS + l * S + b]; };
    const int nm = (int)monos.size();
    P.assign((size_t)nm * S * S, 0.0);
    for (int t = 0; t < nm; ++t) {
        const Mono &mo = monos[t];
        for (int a = 0; a < S; ++a)
            for (int b = 0; b < S; ++b) {
                double val = 0.0;
                if (mo.modes.size() == 1 && mo.pows[0] == 1) val = g(a, S + mo.modes[0] * S + b);
                else if (mo.modes.size() == 1) val = g(a, S + M * S + mo.modes[0] * S + b);
                else val = g2(mo.modes[0], a, mo.modes[1], b);
                P[(size_t)t * S * S + a * S + b] = val;
            }
    }
    Cq.assign((size_t)S * S + M, 0.0);
    for (int a = 0; a < S; ++a)
        for (int b = 0; b < S; ++b) Cq[a * S + b] = g(a, b);
    for (int k = 0; k < M; ++k)
        for (int a = 0; a < S; ++a) Cq[S * S + k] += g(a, S + 2 * M * S + k * S + a);
}

// P[m][a][b] for the monomials of an ordr-3 system and Cq = (C[a][b], K_k) from the Gram
// entries (host copy Gh of length gram3_len, laid out by gram3_tasks)
static void gram3_pc(const nvb_handle *h, const std::vector<double> &Gh, const std::vector<Mono> &monos,
                     std::vector<double> &P, std::vector<double> &Cq) {
    const int S = h->sys.S, M = h->sys.M;
    const G3Cols c(S, M);
    std::vector<G3Task> tasks;
    std::vector<int> index;
    gram3_tasks(S, M, tasks, index);
    auto G = [&](int ia, int jb) {
        const int o = index[(size_t)ia * c.nB + jb];
        if (o < 0) fail(NVB_ERR_STATE, "adjoint: Gram entry not formed");
        return Gh[(size_t)o];
    };
    const int nm = (int)monos.size();
    P.assign((size_t)nm * S * S, 0.0);
    for (int t = 0; t < nm; ++t) {
        const Mono &mo = monos[t];
        int deg = 0;
        for (int pw : mo.pows) deg += pw;
        for (int a = 0; a < S; ++a)
            for (int b = 0; b < S; ++b) {
                double val = 0.0;
                if (mo.modes.size() == 1) {
                    const int k = mo.modes[0];
                    if (deg == 1) val = G(c.u(a), c.Xv(k, b));
                    else if (deg == 2) val = G(c.u(a), c.x2v(k, b));
                    else val = G(c.u(a), c.x3v(k, b));
                } else if (mo.modes.size() == 2) {
                    const int k0 = mo.modes[0], k1 = mo.modes[1];
                    if (deg == 2) val = G(c.Xu(k0, a), c.Xv(k1, b));
                    else if (mo.pows[0] == 2) val = G(c.x2u(k0, a), c.Xv(k1, b));  // x_k0^2 x_k1
                    else val = G(c.x2u(k1, a), c.Xv(k0, b));                      // x_k0 x_k1^2
                } else {
                    int k[3] = {mo.modes[0], mo.modes[1], mo.modes[2]};
                    std::sort(k, k + 3);
                    val = G(c.Xu(k[0], a), c.XXv(k[1], k[2], b));
                }
                P[(size_t)t * S * S + a * S + b] = val;
            }
    }
    Cq.assign((size_t)S * S + M, 0.0);
    for (int a = 0; a < S; ++a)
        for (int b = 0; b < S; ++b) Cq[a * S + b] = G(c.u(a), c.v(b));
    for (int k = 0; k < M; ++k)
        for (int a = 0; a < S; ++a) Cq[S * S + k] += G(c.u(a), c.hv(k, a));
}

template <typename T>
static void gram3_adjoint(nvb_handle *h, const T *u, const T *v, const std::vector<Mono> &monos, std::vector<double> &P,
                          std::vector<double> &Cq) {
    gram3_setup(h);
    const int nout = 4 * h->g3_ntask, grid = h->g3_grid;
    double *part = (double *)scratch_vector(h, ((size_t)grid + 1) * nout * sizeof(double));
    double *G = part + (size_t)grid * nout;
    gram3_launch<T>(h, u, v, G, 0, part);
    std::vector<double> Gh(nout);
    CK(cudaMemcpyAsync(Gh.data(), G, nout * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    gram3_pc(h, Gh, monos, P, Cq);
}

template <typename T>
static void gram_adjoint(nvb_handle *h, const T *u, const T *v, const std::vector<Mono> &monos, std::vector<double> &P,
                         std::vector<double> &Cq) {
    const int nout = gram_len(h->sys.S, h->sys.M), grid = gram_grid(h);
    double *part = (double *)scratch_vector(h, ((size_t)grid + 1) * nout * sizeof(double));
    double *G = part + (size_t)grid * nout;
    gram_launch<T>(h, u, v, G, 0, part);
    std::vector<double> Gh(nout);
    CK(cudaMemcpyAsync(Gh.data(), G, nout * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    gram_pc(h, Gh, monos, P, Cq);
}

// dL/dtheta in the layout of nvb_hv_adjoint_coeffs from P[m][a][b] = <u_a| monomial m |v_b> and
// Cq = (C[a][b] = <u_a|v_b>, K_k = sum_a <u_a|(n_k+1/2)|v_a>); linear in (P, Cq).
static void assemble_grad(const nvb_handle *h, const std::vector<Mono> &monos, const std::vector<double> &P,
                          const std::vector<double> &Cq, double *grad) {
    const System &sys = h->sys;
    const int S = sys.S, M = sys.M;
    const int nm = (int)monos.size();
    const int nb = sys.nstblks();
    const int64_t npot = (int64_t)sys.potterms.size();
    std::vector<std::pair<int, int>> cp(nb);
    for (int i = 1; i <= S; ++i)
        for (int j = 1; j <= i; ++j) cp[i * (i - 1) / 2 + j - 1] = {i - 1, j - 1};
    // monomial id of (order d, index k)
    std::vector<int> mono_base(sys.ordr + 1, 0);
    for (int d = 1; d <= sys.ordr; ++d) mono_base[d] = (d == 1 ? 0 : mono_base[d - 1] + (int)numut(M, d - 1));
    std::vector<double> scale(nm, 1.0);
    for (int t = 0; t < nm; ++t)
        for (size_t l = 0; l < monos[t].modes.size(); ++l)
            scale[t] /= std::sqrt(std::pow(sys.omega[monos[t].modes[l]], (double)monos[t].pows[l]));
    for (int b = 0; b < nb; ++b) {
        auto [i, j] = cp[b];
        for (int d = 1; d <= sys.ordr; ++d) {
            const int64_t off = sys.pot_offset[(size_t)b * sys.ordr + d - 1];
            const int64_t cnt = numut(M, d);
            for (int64_t k = 0; k < cnt; ++k) {
                const int t = mono_base[d] + (int)k;
                double g = P[(size_t)t * S * S + i * S + j];
                if (i != j) g += P[(size_t)t * S * S + j * S + i];
                grad[off + k] = scale[t] * g;
            }
        }
        double gc = Cq[i * S + j];
        if (i != j) gc += Cq[j * S + i];
        grad[npot + b] = gc;
    }
    // frequencies: harmonic part plus the omega dependence of every scaled coefficient
    for (int k = 0; k < M; ++k) grad[npot + nb + k] = Cq[S * S + k];
    for (int b = 0; b < nb; ++b) {
        auto [i, j] = cp[b];
        for (int d = 1; d <= sys.ordr; ++d) {
            const int64_t off = sys.pot_offset[(size_t)b * sys.ordr + d - 1];
            const int64_t cnt = numut(M, d);
            for (int64_t k = 0; k < cnt; ++k) {
                const double c = sys.potterms[off + k];
                if (c == 0.0) continue;
                const int t = mono_base[d] + (int)k;
                double g = P[(size_t)t * S * S + i * S + j];
                if (i != j) g += P[(size_t)t * S * S + j * S + i];
                for (size_t l = 0; l < monos[t].modes.size(); ++l) {
                    const int md = monos[t].modes[l];
                    grad[npot + nb + md] += -(double)monos[t].pows[l] / (2.0 * sys.omega[md]) * c * scale[t] * g;
                }
            }
        }
    }
}

template <typename T, int S>
static void adjoint_s(nvb_handle *h, const T *u, const T *v, double *grad) {
    constexpr int TB = S * S <= 4 ? 8 : (S * S <= 9 ? 3 : 2);
    const System &sys = h->sys;
    const Plan &pl = h->plan;
    const int M = sys.M;
    const auto monos = all_monomials(sys);
    const int nm = (int)monos.size();
    const int grid = 148 * 4;
    // P[m][a][b]
    std::vector<double> P((size_t)nm * S * S, 0.0);
    std::vector<double> Cq;
    if (sys.ordr <= 2 && gram_fits(S, M)) {
        gram_adjoint<T>(h, u, v, monos, P, Cq);
    } else if (sys.ordr == 3 && gram3_fits(S, M)) {
        gram3_adjoint<T>(h, u, v, monos, P, Cq);
    } else {
    double *part = nullptr;
    CK(cudaMalloc((void **)&part, (size_t)grid * std::max(TB * S * S, S * S + M) * sizeof(double)));
    for (int m0 = 0; m0 < nm; m0 += TB) {
        std::vector<AdjStep> steps;
        for (int t = m0; t < std::min(nm, m0 + TB); ++t) {
            const Mono &mo = monos[t];
            const int d = (int)mo.modes.size();
            int sm[MAX_ORDER], sd[MAX_ORDER];
            bool bad = false;
            long long ns = 1;
            for (int l = 0; l < d; ++l) {
                sm[l] = smax_of(mo.pows[l], sys.nfunc[mo.modes[l]]);
                if (sm[l] < 0) bad = true;
                ns *= sm[l] + 1;
                sd[l] = -sm[l];
            }
            if (bad) continue;
            sd[d - 1] -= 2;
            for (long long k = 0; k < ns; ++k) {
                int l = d - 1;
                while (sd[l] >= sm[l]) { sd[l] = -sm[l]; --l; }
                sd[l] += 2;
                AdjStep st{};
                st.mono = t - m0;
                st.nm = d;
                long long stride = 0;
                for (int q = 0; q < d; ++q) {
                    st.mode[q] = mo.modes[q];
                    st.sig[q] = sd[q];
                    st.etab[q] = ((mo.pows[q] - 1) * ETAB_J + std::abs(sd[q])) * pl.nmax;
                    stride += (long long)sd[q] * sys.shft[mo.modes[q]];
                }
                st.stride = stride;
                steps.push_back(st);  // the zero shift of an all-even monomial included
            }
        }
        launch_chunk<T, S, TB>(h, steps, u, v, part, grid);
        std::vector<double> hp((size_t)grid * TB * S * S);
        CK(cudaMemcpy(hp.data(), part, hp.size() * sizeof(double), cudaMemcpyDeviceToHost));
        for (int t = m0; t < std::min(nm, m0 + TB); ++t)
            for (int ab = 0; ab < S * S; ++ab) {
                double s = 0.0;
                for (int g = 0; g < grid; ++g) s += hp[(size_t)g * TB * S * S + (t - m0) * S * S + ab];
                P[(size_t)t * S * S + ab] = s;
            }
    }
    // overlaps and harmonic part
    k_adj_diag<T, S><<<grid, ADJ_THREADS, 0, h->stream>>>(pl.d_shft, M, pl.dimen, u, v, part);
    CK(cudaGetLastError());
    const int nout = S * S + M;
    std::vector<double> hq((size_t)grid * nout);
    CK(cudaMemcpyAsync(hq.data(), part, hq.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    cudaFree(part);
    Cq.assign(nout, 0.0);
    for (int q = 0; q < nout; ++q)
        for (int g = 0; g < grid; ++g) Cq[q] += hq[(size_t)g * nout + q];
    }
    assemble_grad(h, monos, P, Cq, grad);
}

void hv_adjoint(nvb_handle *h, const void *u, const void *v, int dtype, double *grad) {
    const bool f32 = dtype == NVB_DTYPE_F32;
#define ADJ_CASE(SS)                                                                  \
    case SS:                                                                          \
        if (f32) adjoint_s<float, SS>(h, (const float *)u, (const float *)v, grad);   \
        else adjoint_s<double, SS>(h, (const double *)u, (const double *)v, grad);    \
        break;
    switch (h->sys.S) {
        ADJ_CASE(1)
        ADJ_CASE(2)
        ADJ_CASE(3)
        ADJ_CASE(4)
    default: fail(NVB_ERR_ARG, "the adjoint supports up to 4 states");
    }
#undef ADJ_CASE
}

// Accumulated adjoint for the reverse sweep (ordr <= 2 systems whose Gram matrices fit): the
// gradient is linear in the Gram matrices, so the sweep sums them on the device over all
// steps and assembles the gradient once.
static bool gram3_path(const nvb_handle *h) { return h->sys.ordr == 3 && gram3_fits(h->sys.S, h->sys.M); }

int64_t adjoint_gram_len(const nvb_handle *h) {
    if (h->sys.ordr <= 2 && gram_fits(h->sys.S, h->sys.M)) return gram_len(h->sys.S, h->sys.M);
    if (gram3_path(h)) return gram3_len(h->sys.S, h->sys.M);
    return 0;
}
int64_t adjoint_gram_part_len(const nvb_handle *h) {
    return (int64_t)(gram3_path(h) ? gram3_grid(h) : gram_grid(h)) * adjoint_gram_len(h);
}

void adjoint_gram_add(nvb_handle *h, const void *u, const void *v, int dtype, double *G, int accumulate, double *part) {
    if (gram3_path(h)) {
        if (dtype == NVB_DTYPE_F32) gram3_launch<float>(h, (const float *)u, (const float *)v, G, accumulate, part);
        else gram3_launch<double>(h, (const double *)u, (const double *)v, G, accumulate, part);
        return;
    }
    if (dtype == NVB_DTYPE_F32) gram_launch<float>(h, (const float *)u, (const float *)v, G, accumulate, part);
    else gram_launch<double>(h, (const double *)u, (const double *)v, G, accumulate, part);
}

void adjoint_gram_reduce(nvb_handle *h, const double *part, double *G) {
    const int nout = (int)adjoint_gram_len(h);
    const int grid = gram3_path(h) ? gram3_grid(h) : gram_grid(h);
    k_gram_reduce<<<(nout * 32 + 255) / 256, 256, 0, h->stream>>>(part, grid, nout, 0, G);
    CK(cudaGetLastError());
}

void adjoint_gram_grad(nvb_handle *h, const double *G, double *grad) {
    const int64_t nout = adjoint_gram_len(h);
    if (nout == 0) fail(NVB_ERR_STATE, "adjoint: no Gram path for this system");
    std::vector<double> Gh((size_t)nout);
    CK(cudaMemcpyAsync(Gh.data(), G, nout * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    const auto monos = all_monomials(h->sys);
    std::vector<double> P, Cq;
    if (gram3_path(h)) gram3_pc(h, Gh, monos, P, Cq);
    else gram_pc(h, Gh, monos, P, Cq);
    assemble_grad(h, monos, P, Cq, grad);
}

int64_t ncoef_of(const nvb_handle *h) { return (int64_t)h->sys.potterms.size() + h->sys.nstblks() + h->sys.M; }

// Ritz vectors, declared in state.cu
void ritz_vectors_public(nvb_handle *h, int64_t nroots, const std::vector<double> &V, double *psi);

// Hellmann-Feynman: grad[r*ncoef + i] = <psi_r| dH/dtheta_i |psi_r> for the lowest nroots Ritz
// vectors of T_n (normalised in FP64).
void hellmann_feynman(nvb_handle *h, int64_t nroots, double *grad, double *energies) {
    const int64_t n = h->iters;
    if (n < 1) fail(NVB_ERR_STATE, "no Lanczos iterations");
    if (nroots < 1 || nroots > n) fail(NVB_ERR_ARG, "nroots must be in 1..iterations");
    const long long N = h->ntotal();
    std::vector<double> E(n), V((size_t)n * n);
    tridiag_eigen(n, h->alpha.data() + 1, h->beta.data() + 1, E.data(), V.data());
    double *psi = nullptr;
    CK(cudaMalloc((void **)&psi, (size_t)nroots * N * sizeof(double)));
    try {
        ritz_vectors_public(h, nroots, V, psi);
        const int64_t nc = ncoef_of(h);
        for (int64_t r = 0; r < nroots; ++r) {
            double *p = psi + (size_t)r * N;
            const double nrm2 = device_dot(h, p, 1.0, p, 1.0, NVB_DTYPE_F64);
            hv_adjoint(h, p, p, NVB_DTYPE_F64, grad + r * nc);
            for (int64_t i = 0; i < nc; ++i) grad[r * nc + i] /= nrm2;
            if (energies) energies[r] = E[r];
        }
    } catch (...) {
        cudaFree(psi);
        throw;
    }
    cudaFree(psi);
}

}  // namespace nvb
