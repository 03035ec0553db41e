// H.v, gather form: one thread per row (basis function index within a state), all states of
// that row accumulated in registers.  General: any number of states (<=10), modes, and
// expansion order (<=4).  It evaluates, for output row n,
//
//   y_a(n) = (sum_k w_k (n_k+1/2) + D_aa(n)) x_a(n) + sum_{b != a, applied} D_ab(n) x_b(n)
//          + sum_{steps (t, s != 0) valid at n} sum_b C^t_ab * prod_l E(p_l, n_l, s_l) * x_b(n + s)
//
// which is the matrix-free product of Hv (Source/top.f90:672-818): D is the diagonal block of
// Source/top.f90:731-751 (constants + even-power terms at zero shift), the steps are the
// (term, shift) passes of Source/top.f90:758-808 with the shift ranges of
// Source/secondary.f90:27-64, and per output element the contributions are accumulated in
// the reference's order (diagonal, then terms / steps / pairs in table order).
#include <cuda_runtime.h>

#include "plan.h"

namespace nvb {

template <typename T>
struct KArgs {
    const DevStep *steps;
    int nsteps;
    const DevDiag *diag;
    int ndiag;
    const T *coef;                   // [nterms][S][S]
    const unsigned long long *mask;  // [nterms][2]
    const T *cst;                    // [S][S]
    const int *dpair;                // [S][S]
    const T *etab;
    int etab_len;
    const int *nfunc;
    const long long *shft;
    const T *omega;
    int M;
    long long dimen;
};

template <typename T, int S>
__global__ void __launch_bounds__(256) k_hv_gather(KArgs<T> A, const T *__restrict__ x, T *__restrict__ y,
                                                  const double *__restrict__ scale_dev,
                                                  double *__restrict__ alpha_part) {
    extern __shared__ __align__(16) unsigned char smem[];
    T *s_etab = reinterpret_cast<T *>(smem);
    unsigned char *s_dig = smem + ((A.etab_len * sizeof(T) + 15) / 16) * 16;
    const int tid = threadIdx.x;
    for (int i = tid; i < A.etab_len; i += blockDim.x) s_etab[i] = A.etab[i];
    const long long r = (long long)blockIdx.x * blockDim.x + tid;
    const bool active = r < A.dimen;
    const long long N = A.dimen;
    T ekin = 0;
    if (active) {
        long long rem = r;
        for (int k = 0; k < A.M; ++k) {
            const long long sh = A.shft[k];
            const int d = (int)(rem / sh);
            rem -= (long long)d * sh;
            s_dig[k * blockDim.x + tid] = (unsigned char)d;
            ekin += A.omega[k] * ((T)d + (T)0.5);
        }
    }
    __syncthreads();
    double part = 0.0;
    if (active) {
        const unsigned char *dig = s_dig + tid;
        T xc[S], acc[S], D[S][S];
#pragma unroll
        for (int a = 0; a < S; ++a) xc[a] = x[a * N + r];
#pragma unroll
        for (int a = 0; a < S; ++a)
#pragma unroll
            for (int b = 0; b < S; ++b) D[a][b] = A.cst[a * S + b];
        for (int i = 0; i < A.ndiag; ++i) {
            const DevDiag *dg = A.diag + i;
            T d1 = 1;
            const int nm = dg->nm, term = dg->term;
            for (int l = 0; l < nm; ++l) d1 = d1 * s_etab[dg->etab[l] + dig[dg->mode[l] * blockDim.x]];
            const unsigned long long m0 = A.mask[2 * term], m1 = A.mask[2 * term + 1];
            const T *cf = A.coef + (size_t)term * S * S;
#pragma unroll
            for (int a = 0; a < S; ++a)
#pragma unroll
                for (int b = 0; b < S; ++b) {
                    const int bit = a * S + b;
                    const bool on = bit < 64 ? ((m0 >> bit) & 1ull) : ((m1 >> (bit - 64)) & 1ull);
                    if (on && A.dpair[a * S + b]) D[a][b] = D[a][b] + cf[a * S + b] * d1;
                }
        }
#pragma unroll
        for (int a = 0; a < S; ++a) {
            acc[a] = (D[a][a] + ekin) * xc[a];
#pragma unroll
            for (int b = 0; b < S; ++b)
                if (b != a && A.dpair[a * S + b]) acc[a] = acc[a] + D[a][b] * xc[b];
        }
        for (int i = 0; i < A.nsteps; ++i) {
            const DevStep *st = A.steps + i;
            T e = 1;
            bool ok = true;
            const int nm = st->nm;
            for (int l = 0; l < nm; ++l) {
                const int md = st->mode[l];
                const int n = dig[md * blockDim.x];
                const int nc = n + st->sig[l];
                if (nc < 0 || nc >= A.nfunc[md]) { ok = false; break; }
                e = e * s_etab[st->etab[l] + (nc < n ? nc : n)];
            }
            if (!ok) continue;
            const int term = st->term;
            const unsigned long long m0 = A.mask[2 * term], m1 = A.mask[2 * term + 1];
            const T *cf = A.coef + (size_t)term * S * S;
            const T *xs = x + r + st->stride;
            T xb[S];
#pragma unroll
            for (int b = 0; b < S; ++b) {
                bool need = false;
#pragma unroll
                for (int a = 0; a < S; ++a) {
                    const int bit = a * S + b;
                    need |= bit < 64 ? ((m0 >> bit) & 1ull) : ((m1 >> (bit - 64)) & 1ull);
                }
                xb[b] = need ? xs[b * N] : (T)0;
            }
#pragma unroll
            for (int a = 0; a < S; ++a)
#pragma unroll
                for (int b = 0; b < S; ++b) {
                    const int bit = a * S + b;
                    const bool on = bit < 64 ? ((m0 >> bit) & 1ull) : ((m1 >> (bit - 64)) & 1ull);
                    if (on) acc[a] = acc[a] + xb[b] * cf[a * S + b] * e;
                }
        }
        const T sc = scale_dev ? (T)(*scale_dev) : (T)1;
#pragma unroll
        for (int a = 0; a < S; ++a) {
            const T v = acc[a] * sc;
            y[a * N + r] = v;
            part += ((double)xc[a] * (double)sc) * (double)v;
        }
    }
    if (alpha_part) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
        __shared__ double red[32];
        if ((tid & 31) == 0) red[tid >> 5] = part;
        __syncthreads();
        if (tid < 32) {
            double v = tid < (int)(blockDim.x >> 5) ? red[tid] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (tid == 0) alpha_part[blockIdx.x] = v;
        }
    }
}

template <typename T>
static KArgs<T> make_args(const Plan &pl);

template <>
KArgs<double> make_args<double>(const Plan &pl) {
    return KArgs<double>{pl.d_steps, pl.nsteps, pl.d_diag,  pl.ndiag,  pl.d_coef,  pl.d_mask,  pl.d_const, pl.d_dpair,
                         pl.d_etab,  (int)pl.h_etab.size(), pl.d_nfunc, pl.d_shft, pl.d_omega, pl.M, pl.dimen};
}
template <>
KArgs<float> make_args<float>(const Plan &pl) {
    return KArgs<float>{pl.d_steps,  pl.nsteps, pl.d_diag,   pl.ndiag,   pl.d_coef_f, pl.d_mask,  pl.d_const_f, pl.d_dpair,
                        pl.d_etab_f, (int)pl.h_etab.size(), pl.d_nfunc, pl.d_shft, pl.d_omega_f, pl.M, pl.dimen};
}

template <typename T, int S>
static void launch_s(const Plan &pl, const T *x, T *y, const double *sc, double *ap, cudaStream_t st) {
    KArgs<T> a = make_args<T>(pl);
    const int threads = 256;
    const long long blocks = (pl.dimen + threads - 1) / threads;
    size_t smem = ((a.etab_len * sizeof(T) + 15) / 16) * 16 + (size_t)pl.M * threads;
    static bool attr = false;
    if (!attr && smem > 48 * 1024) {
        cudaFuncSetAttribute(k_hv_gather<T, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr = true;
    }
    k_hv_gather<T, S><<<(unsigned)blocks, threads, smem, st>>>(a, x, y, sc, ap);
}

int hv_gather_blocks(const Plan &pl) { return (int)((pl.dimen + 255) / 256); }

template <typename T>
void hv_gather_launch(const Plan &pl, const T *x, T *y, const double *sc, double *ap, cudaStream_t st) {
    switch (pl.S) {
    case 1: launch_s<T, 1>(pl, x, y, sc, ap, st); break;
    case 2: launch_s<T, 2>(pl, x, y, sc, ap, st); break;
    case 3: launch_s<T, 3>(pl, x, y, sc, ap, st); break;
    case 4: launch_s<T, 4>(pl, x, y, sc, ap, st); break;
    case 5: launch_s<T, 5>(pl, x, y, sc, ap, st); break;
    case 6: launch_s<T, 6>(pl, x, y, sc, ap, st); break;
    case 7: launch_s<T, 7>(pl, x, y, sc, ap, st); break;
    case 8: launch_s<T, 8>(pl, x, y, sc, ap, st); break;
    case 9: launch_s<T, 9>(pl, x, y, sc, ap, st); break;
    case 10: launch_s<T, 10>(pl, x, y, sc, ap, st); break;
    default: fail(NVB_ERR_ARG, "nstates out of range");
    }
}

template void hv_gather_launch<double>(const Plan &, const double *, double *, const double *, double *, cudaStream_t);
template void hv_gather_launch<float>(const Plan &, const float *, float *, const double *, double *, cudaStream_t);

}  // namespace nvb
