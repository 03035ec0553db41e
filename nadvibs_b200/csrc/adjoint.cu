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
int64_t adjoint_gram_len(const nvb_handle *h) {
    return (h->sys.ordr <= 2 && gram_fits(h->sys.S, h->sys.M)) ? gram_len(h->sys.S, h->sys.M) : 0;
}
int64_t adjoint_gram_part_len(const nvb_handle *h) { return (int64_t)gram_grid(h) * adjoint_gram_len(h); }

void adjoint_gram_add(nvb_handle *h, const void *u, const void *v, int dtype, double *G, int accumulate, double *part) {
    if (dtype == NVB_DTYPE_F32) gram_launch<float>(h, (const float *)u, (const float *)v, G, accumulate, part);
    else gram_launch<double>(h, (const double *)u, (const double *)v, G, accumulate, part);
}

void adjoint_gram_reduce(nvb_handle *h, const double *part, double *G) {
    const int nout = (int)adjoint_gram_len(h);
    k_gram_reduce<<<(nout * 32 + 255) / 256, 256, 0, h->stream>>>(part, gram_grid(h), nout, 0, G);
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
    gram_pc(h, Gh, monos, P, Cq);
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
