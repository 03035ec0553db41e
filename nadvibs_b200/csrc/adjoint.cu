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
// The sums over rows run on the FP64 tensor cores (mma m8n8k4): G is cut into 8 x 8 blocks
// (8 A columns x 8 B columns) and only the blocks holding a needed entry are formed.  The
// columns are ordered so that the needed entries cluster: A = [X u, x^2 u, u]; B = X v first,
// then v, x^2 v, (n+1/2) v, x^3 v, then X_l X_m v by descending l (an A column X_k u needs
// exactly the pairs with l > k, a prefix).  Per tile of TR rows the columns are expanded into
// shared memory (column-major, a warp per (mode, state) or per pair of modes over all states, a
// lane per row, element tables in shared memory), and each warp runs its blocks' MMAs over the
// tile (over the previous tile, interleaved with its gathers, when two tiles fit).  Block
// partials are summed in a fixed order.

constexpr int G3_THREADS = 640;
constexpr int G3_NBW = 8;  // most MMA blocks per warp
constexpr int G3_SMAX = 4; // most electronic states

// Shared-memory column positions of the ordr-3 Gram columns: A = [X u, x^2 u, u] padded to 8;
// B regrouped.
struct G3Pos {
    int nA8, XO, PO, nB8;
    __host__ __device__ G3Pos(int S, int M) {
        const int MS = M * S, P2 = M * (M - 1) / 2;
        nA8 = (S + 2 * MS + 7) & ~7;
        XO = (MS + 7) & ~7;                   // v, x^2 v, (n+1/2) v, x^3 v
        PO = (XO + S + 3 * MS + 7) & ~7;      // X_l X_m v
        nB8 = (PO + P2 * S + 7) & ~7;
    }
};

__device__ __forceinline__ void mma_f64_884(double (&c)[2], double a, double b) {
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
        : "+d"(c[0]), "+d"(c[1])
        : "d"(a), "d"(b));
}

// TR rows per tile (a multiple of 32); column pitch TR + 4 doubles, so the 4 x 4 fragment of
// each half-warp (4 rows of 4 columns) covers all 32 banks; NBW: most MMA blocks per warp.
// NBUF = 2: two column tiles, so one barrier per tile separates the expansion of tile i (and the
// digits of tile i+1) from the MMAs of tile i-1, and warps in either phase overlap; NBUF = 1:
// one tile, expansion and MMAs separated by barriers.
template <typename T, int TR, int NBW, int NBUF, int S>
__global__ void __launch_bounds__(G3_THREADS, 1)
    k_adj_gram3(const T *__restrict__ u, const T *__restrict__ v, const double *__restrict__ etab, int nmax,
                const int *__restrict__ nfunc, const long long *__restrict__ shft, int M, long long dimen,
                const int *__restrict__ blocks, int nblk, int nbw, int accumulate, double *__restrict__ part) {
    constexpr int PT = TR + 4, RPL = TR / 32;
    static_assert(TR % 32 == 0, "whole warps of rows");
    static_assert(S >= 1 && S <= G3_SMAX, "states");
    const int dimi = (int)dimen;  // <= INT_MAX (checked on the host)
    extern __shared__ double sm[];
    const int MS = M * S, P2 = M * (M - 1) / 2;
    const G3Pos ps(S, M);
    const int tcols = (ps.nA8 + ps.nB8) * PT;                  // one column tile: A then B, [column][row]
    double *stab = sm + NBUF * tcols;                          // element rows E1, E2, D2, E31, E33 [nmax]
    int *ssh = reinterpret_cast<int *>(stab + 5 * nmax);       // [M] strides
    int *snf = ssh + M;                                        // [M] nfunc
    int *spair = snf + M;                                      // pair p (descending l): l | m << 8
    int *sdig0 = spair + P2;                                   // [NBUF][mode][row]
    const int tid = threadIdx.x, nth = blockDim.x, lane = tid & 31, wid = tid >> 5, nwarp = nth >> 5;
    for (int i = tid; i < NBUF * tcols; i += nth) sm[i] = 0.0;  // padding columns stay zero
    for (int i = tid; i < nmax; i += nth) {
        stab[0 * nmax + i] = etab[(0 * ETAB_J + 1) * nmax + i];  // <n|x|n+1>
        stab[1 * nmax + i] = etab[(1 * ETAB_J + 2) * nmax + i];  // <n|x^2|n+2>
        stab[2 * nmax + i] = etab[(1 * ETAB_J + 0) * nmax + i];  // <n|x^2|n>
        stab[3 * nmax + i] = etab[(2 * ETAB_J + 1) * nmax + i];  // <n|x^3|n+1>
        stab[4 * nmax + i] = etab[(2 * ETAB_J + 3) * nmax + i];  // <n|x^3|n+3>
    }
    for (int k = tid; k < M; k += nth) {
        ssh[k] = (int)shft[k];
        snf[k] = nfunc[k];
    }
    if (tid == 0) {
        int q = 0;
        for (int l = M - 2; l >= 0; --l)
            for (int m = l + 1; m < M; ++m) spair[q++] = l | (m << 8);
    }
    const double *E1 = stab, *E2 = stab + nmax, *D2 = stab + 2 * nmax, *E31 = stab + 3 * nmax, *E33 = stab + 4 * nmax;
    // this warp's blocks [wid * nbw, +nq) (nbw <= NBW): fragment offsets of A (column ib*8 + lane/4)
    // and B (column jb*8 + lane/4) within a column tile, row lane%4 of each 4-row step
    const int nq = max(0, min(nbw, nblk - wid * nbw));
    int aoff[NBW], boff[NBW];
    double acc[NBW][2];
#pragma unroll
    for (int q = 0; q < NBW; ++q) {
        const int w = q < nq ? blocks[wid * nbw + q] : 0;
        aoff[q] = ((w & 0xffff) * 8 + (lane >> 2)) * PT + (lane & 3);
        boff[q] = (ps.nA8 + (w >> 16) * 8 + (lane >> 2)) * PT + (lane & 3);
        acc[q][0] = acc[q][1] = 0.0;
    }
    const long long tstride = (long long)gridDim.x * TR, first = (long long)blockIdx.x * TR;
    const int ntl = first < dimen ? (int)((dimen - first + tstride - 1) / tstride) : 0;  // this block's tiles
    // digits of tile t's rows: a thread per (mode, row)
    auto digits = [&](int t, int *sdig) {
        const long long t0 = first + (long long)t * tstride;
        for (int i = tid; i < M * TR; i += nth) {
            const int k = i / TR, e = i - k * TR;
            const long long r = t0 + e;
            sdig[i] = r < dimen ? (int)((unsigned)r / (unsigned)ssh[k] % (unsigned)snf[k]) : 0;
        }
    };
    // The columns of tile t, one family at a time: families f < MS the (mode, state) pairs, then
    // the pairs of modes over all states (each about twelve gathers per row), a lane per row.
    // `between()` runs while the family's loads are in flight (the double-buffered schedule puts
    // a slice of the previous tile's MMAs there).  Offsets of neighbours outside the basis are
    // clamped to the row itself and their coefficients are zero, so the loads are unconditional.
    auto family = [&](int f, int t, const int *sdig, double *sA, auto &&between) {
        double *sB = sA + ps.nA8 * PT;
        const int t0 = (int)(first + (long long)t * tstride);  // < dimen <= INT_MAX: the tile exists
        if (f < MS) {
            const int k = f / S, s = f - k * S, nf = snf[k], sh = ssh[k];
            double g[RPL][12];
#pragma unroll
            for (int hr = 0; hr < RPL; ++hr) {
                const int e = lane + 32 * hr;
                const int r = t0 + e;
                const bool in = r < dimi;
                const int d = sdig[k * TR + e];
                const int o1p = in && d + 1 < nf ? sh : 0, o1m = in && d >= 1 ? -sh : 0;
                const int o2p = in && d + 2 < nf ? 2 * sh : 0, o2m = in && d >= 2 ? -2 * sh : 0;
                const int o3p = in && d + 3 < nf ? 3 * sh : 0, o3m = in && d >= 3 ? -3 * sh : 0;
                const int rr = in ? r : t0;
                const T *ur = u + (long long)s * dimen + rr, *vr = v + (long long)s * dimen + rr;
                g[hr][0] = (double)ur[0];
                g[hr][1] = (double)vr[0];
                g[hr][2] = (double)ur[o1p];
                g[hr][3] = (double)vr[o1p];
                g[hr][4] = (double)ur[o1m];
                g[hr][5] = (double)vr[o1m];
                g[hr][6] = (double)ur[o2p];
                g[hr][7] = (double)vr[o2p];
                g[hr][8] = (double)ur[o2m];
                g[hr][9] = (double)vr[o2m];
                g[hr][10] = (double)vr[o3p];
                g[hr][11] = (double)vr[o3m];
            }
            between();
#pragma unroll
            for (int hr = 0; hr < RPL; ++hr) {
                const int e = lane + 32 * hr;
                const bool in = t0 + e < dimi;
                const int d = sdig[k * TR + e];
                const bool p1 = in && d + 1 < nf, m1 = in && d >= 1, p2 = in && d + 2 < nf, m2 = in && d >= 2;
                const bool p3 = in && d + 3 < nf, m3 = in && d >= 3;
                const double u0 = in ? g[hr][0] : 0.0, v0 = in ? g[hr][1] : 0.0;
                const double e1p = p1 ? E1[d] : 0.0, e1m = m1 ? E1[d - 1] : 0.0;
                const double e31p = p1 ? E31[d] : 0.0, e31m = m1 ? E31[d - 1] : 0.0;
                const double e2p = p2 ? E2[d] : 0.0, e2m = m2 ? E2[d - 2] : 0.0, ed2 = in ? D2[d] : 0.0;
                const double e33p = p3 ? E33[d] : 0.0, e33m = m3 ? E33[d - 3] : 0.0;
                const double xu = e1p * g[hr][2] + e1m * g[hr][4];
                const double xv = e1p * g[hr][3] + e1m * g[hr][5];
                const double x2u = ed2 * u0 + e2p * g[hr][6] + e2m * g[hr][8];
                const double x2v = ed2 * v0 + e2p * g[hr][7] + e2m * g[hr][9];
                const double x3v = e31p * g[hr][3] + e31m * g[hr][5] + e33p * g[hr][10] + e33m * g[hr][11];
                const int c = k * S + s;
                if (k == 0) {
                    sA[(2 * MS + s) * PT + e] = u0;
                    sB[(ps.XO + s) * PT + e] = v0;
                }
                sA[c * PT + e] = xu;
                sA[(MS + c) * PT + e] = x2u;
                sB[c * PT + e] = xv;
                sB[(ps.XO + S + c) * PT + e] = x2v;
                sB[(ps.XO + S + MS + c) * PT + e] = ((double)d + 0.5) * v0;
                sB[(ps.XO + S + 2 * MS + c) * PT + e] = x3v;
            }
        } else {
            const int pd = f - MS, pw = spair[pd], l = pw & 255, m = pw >> 8;
            const int nl = snf[l], nm = snf[m], shl = ssh[l], shm = ssh[m];
            double g[RPL][4 * G3_SMAX];
#pragma unroll
            for (int hr = 0; hr < RPL; ++hr) {
                const int e = lane + 32 * hr;
                const int r = t0 + e;
                const bool in = r < dimi;
                const int dl = sdig[l * TR + e], dm = sdig[m * TR + e];
                const bool lp = in && dl + 1 < nl, lm = in && dl >= 1, mp = dm + 1 < nm, mm = dm >= 1;
                const int opp = lp && mp ? shl + shm : 0, opm = lp && mm ? shl - shm : 0;
                const int omp = lm && mp ? shm - shl : 0, omm = lm && mm ? -shl - shm : 0;
                const int rr = in ? r : t0;
#pragma unroll
                for (int s = 0; s < G3_SMAX; ++s)
                    if (s < S) {
                        const T *vr = v + (long long)s * dimen + rr;
                        g[hr][4 * s + 0] = (double)vr[opp];
                        g[hr][4 * s + 1] = (double)vr[opm];
                        g[hr][4 * s + 2] = (double)vr[omp];
                        g[hr][4 * s + 3] = (double)vr[omm];
                    }
            }
            between();
#pragma unroll
            for (int hr = 0; hr < RPL; ++hr) {
                const int e = lane + 32 * hr;
                const bool in = t0 + e < dimi;
                const int dl = sdig[l * TR + e], dm = sdig[m * TR + e];
                const bool lp = in && dl + 1 < nl, lm = in && dl >= 1, mp = dm + 1 < nm, mm = dm >= 1;
                const double elp = lp ? E1[dl] : 0.0, elm = lm ? E1[dl - 1] : 0.0;
                const double emp = mp ? E1[dm] : 0.0, emm = mm ? E1[dm - 1] : 0.0;
                const double cpp = elp * emp, cpm = elp * emm, cmp = elm * emp, cmm = elm * emm;
#pragma unroll
                for (int s = 0; s < G3_SMAX; ++s)
                    if (s < S)
                        sB[(ps.PO + pd * S + s) * PT + e] =
                            cpp * g[hr][4 * s] + cpm * g[hr][4 * s + 1] + cmp * g[hr][4 * s + 2] + cmm * g[hr][4 * s + 3];
            }
        }
    };
    // MMA steps [k0, k1) (four rows each) of a column tile
    // (a warp's blocks run A-block major: a block with the same A block as the one before it
    // reuses its A fragment)
    auto mma = [&](const double *cols, int k0, int k1) {
        if (nq == 0) return;
        for (int kk = k0; kk < k1; ++kk) {
            double a = 0.0;
#pragma unroll
            for (int q = 0; q < NBW; ++q)
                if (q < nq) {
                    if (q == 0 || aoff[q] != aoff[q - 1]) a = cols[aoff[q] + 4 * kk];
                    mma_f64_884(acc[q], a, cols[boff[q] + 4 * kk]);
                }
        }
    };
    __syncthreads();  // tables and strides
    if (ntl > 0) digits(0, sdig0);
    __syncthreads();
    if constexpr (NBUF == 2) {
        // tile i: this warp's families, each followed (while its loads are in flight) by a slice
        // of the MMA steps of tile i-1; then the digits of tile i+1
        const int nfam = MS + P2;
        for (int i = 0; i <= ntl; ++i) {
            const int nfw = i < ntl && wid < nfam ? (nfam - wid + nwarp - 1) / nwarp : 0;
            const int nk = i >= 1 ? TR / 4 : 0;
            const int kc = nfw > 0 ? (nk + nfw - 1) / nfw : nk;
            const double *mcols = sm + ((i - 1) & 1) * tcols;
            int kdone = 0;
            for (int j = 0; j < nfw; ++j)
                family(wid + j * nwarp, i, sdig0 + (i & 1) * M * TR, sm + (i & 1) * tcols, [&] {
                    const int k1 = min(nk, kdone + kc);
                    mma(mcols, kdone, k1);
                    kdone = k1;
                });
            mma(mcols, kdone, nk);
            if (i + 1 < ntl) digits(i + 1, sdig0 + ((i + 1) & 1) * M * TR);
            __syncthreads();
        }
    } else {
        for (int i = 0; i < ntl; ++i) {
            for (int f = wid; f < MS + P2; f += nwarp) family(f, i, sdig0, sm, [] {});
            __syncthreads();
            mma(sm, 0, TR / 4);
            if (i + 1 < ntl) digits(i + 1, sdig0);
            __syncthreads();
        }
    }
    // block q's entry (row lane/4, columns 2 (lane%4) + i) at 64 q + 8 row + column
    double *pb = part + (long long)blockIdx.x * 64 * nblk;
#pragma unroll
    for (int q = 0; q < NBW; ++q)
        if (q < nq)
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                double *pp = pb + (wid * nbw + q) * 64 + (lane >> 2) * 8 + 2 * (lane & 3) + i;
                *pp = accumulate ? *pp + acc[q][i] : acc[q][i];
            }
}

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
    // shared-memory positions (G3Pos) of an A column (X u, x^2 u, then u: the u columns, which
    // alone need v, x^2 v, (n+1/2) v and x^3 v, share one 8-column block) and of a B column
    int posA(int ia) const { return ia < S ? 2 * MS + ia : ia - S; }
    int posB(int jb) const {
        const G3Pos p(S, M);
        if (jb < S) return p.XO + jb;                                  // v
        if (jb < S + MS) return jb - S;                                // X v
        if (jb < S + 4 * MS) return p.XO + S + (jb - S - MS);          // x^2 v, (n+1/2) v, x^3 v
        const int q = jb - S - 4 * MS, pr = q / S, b = q - pr * S;     // X_l X_m v: descending l
        int l = 0;
        while (pair(l, M - 1) < pr) ++l;
        const int m = pr - pair(l, l + 1) + l + 1;
        const int pd = (M - 1 - l) * (M - 2 - l) / 2 + (m - l - 1);
        return p.PO + pd * S + b;
    }
};

// The needed (A, B) entries of the ordr-3 Gram, the 8 x 8 MMA blocks that hold them (A block
// | B block << 16, A-block major) and the output index of every needed entry (64 block + 8 row
// + column; -1 where not formed).
static void gram3_blocks(int S, int M, std::vector<int> &blocks, std::vector<int> &index) {
    const G3Cols c(S, M);
    const G3Pos p(S, M);
    std::vector<std::pair<int, int>> need;
    for (int a = 0; a < S; ++a) {
        for (int b = 0; b < S; ++b) need.push_back({c.u(a), c.v(b)});
        for (int k = 0; k < M; ++k)
            for (int b = 0; b < S; ++b) {
                need.push_back({c.u(a), c.Xv(k, b)});
                need.push_back({c.u(a), c.x2v(k, b)});
                need.push_back({c.u(a), c.hv(k, b)});
                need.push_back({c.u(a), c.x3v(k, b)});
            }
    }
    for (int k = 0; k < M; ++k)
        for (int a = 0; a < S; ++a) {
            for (int l = 0; l < M; ++l)
                if (l != k)
                    for (int b = 0; b < S; ++b) {
                        need.push_back({c.Xu(k, a), c.Xv(l, b)});
                        need.push_back({c.x2u(k, a), c.Xv(l, b)});
                    }
            for (int l = k + 1; l < M; ++l)
                for (int m = l + 1; m < M; ++m)
                    for (int b = 0; b < S; ++b) need.push_back({c.Xu(k, a), c.XXv(l, m, b)});
        }
    const int nbA = p.nA8 / 8, nbB = p.nB8 / 8;
    std::vector<int> bno((size_t)nbA * nbB, -1);
    for (auto &e : need) bno[(size_t)(c.posA(e.first) / 8) * nbB + c.posB(e.second) / 8] = 0;
    blocks.clear();
    for (int i = 0; i < nbA; ++i)
        for (int j = 0; j < nbB; ++j)
            if (bno[(size_t)i * nbB + j] == 0) {
                bno[(size_t)i * nbB + j] = (int)blocks.size();
                blocks.push_back(i | (j << 16));
            }
    index.assign((size_t)c.nA * c.nB, -1);
    for (auto &e : need) {
        const int pa = c.posA(e.first), pb = c.posB(e.second);
        index[(size_t)e.first * c.nB + e.second] = 64 * bno[(size_t)(pa / 8) * nbB + pb / 8] + 8 * (pa % 8) + pb % 8;
    }
}

// Tile shapes in order of preference: TR rows per tile, NBUF column tiles.
struct G3Shape {
    int tr, nbuf;
};
constexpr G3Shape G3_SHAPES[2] = {{32, 2}, {32, 1}};
constexpr size_t G3_SMEM_MAX = 200 * 1024;

static size_t gram3_smem(int S, int M, int nmax, G3Shape sh) {
    const G3Pos p(S, M);
    const int P2 = M * (M - 1) / 2;
    return (size_t)(sh.nbuf * (p.nA8 + p.nB8) * (sh.tr + 4) + 5 * nmax) * sizeof(double) +
           (size_t)(2 * M + P2 + sh.nbuf * sh.tr * M) * sizeof(int);
}

// the first tile shape whose shared memory fits (tr = 0: none)
static G3Shape gram3_shape(const nvb_handle *h) {
    for (const G3Shape &sh : G3_SHAPES)
        if (gram3_smem(h->sys.S, h->sys.M, h->plan.nmax, sh) <= G3_SMEM_MAX) return sh;
    return {0, 0};
}

static bool gram3_fits(const nvb_handle *h) {
    const int S = h->sys.S, M = h->sys.M;
    if (M > 255 || M < 1 || S > G3_SMAX || h->sys.dimen > 0x7fffffffll) return false;
    if (gram3_shape(h).tr == 0) return false;
    std::vector<int> b, idx;
    gram3_blocks(S, M, b, idx);
    return b.size() <= (size_t)G3_NBW * (G3_THREADS / 32);
}

static int gram3_len(int S, int M) {
    std::vector<int> b, idx;
    gram3_blocks(S, M, b, idx);
    return 64 * (int)b.size();
}

static int gram3_grid(const nvb_handle *h) {
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->device);
    const int tr = gram3_shape(h).tr;
    return (int)std::min<long long>((h->sys.dimen + tr - 1) / tr, (long long)nsm * 2);
}

// the block list on the device and the grid, once per handle
static void gram3_setup(nvb_handle *h) {
    if (h->d_g3blk) return;
    std::vector<int> b, idx;
    gram3_blocks(h->sys.S, h->sys.M, b, idx);
    CK(cudaMalloc(&h->d_g3blk, b.size() * sizeof(int)));
    CK(cudaMemcpy(h->d_g3blk, b.data(), b.size() * sizeof(int), cudaMemcpyHostToDevice));
    h->g3_nblk = (int)b.size();
    h->g3_grid = gram3_grid(h);
}

template <typename T, int TR, int NBW, int NBUF, int S>
static void gram3_kernel(nvb_handle *h, const T *u, const T *v, int nbw, int accumulate, double *part, size_t shm) {
    auto k = k_adj_gram3<T, TR, NBW, NBUF, S>;
    if (shm > 48 * 1024) CK(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)shm));
    const Plan &pl = h->plan;
    k<<<h->g3_grid, G3_THREADS, shm, h->stream>>>(u, v, pl.d_etab, pl.nmax, pl.d_nfunc, pl.d_shft, h->sys.M,
                                                   h->sys.dimen, (const int *)h->d_g3blk, h->g3_nblk, nbw,
                                                   accumulate, part);
}

template <typename T, int TR, int NBUF, int S>
static void gram3_kernel_nbw(nvb_handle *h, const T *u, const T *v, int nbw, int accumulate, double *part,
                             size_t shm) {
    if (nbw <= 2) gram3_kernel<T, TR, 2, NBUF, S>(h, u, v, nbw, accumulate, part, shm);
    else if (nbw <= 4) gram3_kernel<T, TR, 4, NBUF, S>(h, u, v, nbw, accumulate, part, shm);
    else if (nbw <= 6) gram3_kernel<T, TR, 6, NBUF, S>(h, u, v, nbw, accumulate, part, shm);
    else gram3_kernel<T, TR, 8, NBUF, S>(h, u, v, nbw, accumulate, part, shm);
}

template <typename T, int S>
static void gram3_kernel_s(nvb_handle *h, const T *u, const T *v, int nbuf, int nbw, int accumulate, double *part,
                           size_t shm) {
    if (nbuf == 2) gram3_kernel_nbw<T, 32, 2, S>(h, u, v, nbw, accumulate, part, shm);
    else gram3_kernel_nbw<T, 32, 1, S>(h, u, v, nbw, accumulate, part, shm);
}

// G (+)= the ordr-3 Gram entries of (u, v) through block partials part[g3_grid * gram3_len];
// G == nullptr: only the partials (accumulate: added to those already there).
template <typename T>
static void gram3_launch(nvb_handle *h, const T *u, const T *v, double *G, int accumulate, double *part) {
    const int S = h->sys.S, M = h->sys.M;
    if (!gram3_fits(h)) fail(NVB_ERR_ARG, "adjoint: too many modes x states for the ordr-3 Gram path");
    gram3_setup(h);
    const G3Shape sh = gram3_shape(h);
    const size_t shm = gram3_smem(S, M, h->plan.nmax, sh);
    const int nwarp = G3_THREADS / 32, nbw = (h->g3_nblk + nwarp - 1) / nwarp;
    const int acc = G ? 0 : accumulate;
    switch (S) {
    case 1: gram3_kernel_s<T, 1>(h, u, v, sh.nbuf, nbw, acc, part, shm); break;
    case 2: gram3_kernel_s<T, 2>(h, u, v, sh.nbuf, nbw, acc, part, shm); break;
    case 3: gram3_kernel_s<T, 3>(h, u, v, sh.nbuf, nbw, acc, part, shm); break;
    default: gram3_kernel_s<T, 4>(h, u, v, sh.nbuf, nbw, acc, part, shm); break;
    }
    const int nout = 64 * h->g3_nblk;
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
// entries (host copy Gh of length gram3_len, laid out by gram3_blocks)
static void gram3_pc(const nvb_handle *h, const std::vector<double> &Gh, const std::vector<Mono> &monos,
                     std::vector<double> &P, std::vector<double> &Cq) {
    const int S = h->sys.S, M = h->sys.M;
    const G3Cols c(S, M);
    std::vector<int> blocks;
    std::vector<int> index;
    gram3_blocks(S, M, blocks, index);
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
    const int nout = 64 * h->g3_nblk, grid = h->g3_grid;
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
    } else if (sys.ordr == 3 && gram3_fits(h)) {
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
static bool gram3_path(const nvb_handle *h) { return h->sys.ordr == 3 && gram3_fits(h); }

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
