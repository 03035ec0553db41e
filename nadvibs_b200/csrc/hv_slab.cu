// Slab-tiled H.v (see slab.h for the decomposition).  One CTA per tile of T_F rows (fixed
// slow digits), SLAB_RPT rows per thread.
//
// Prologue: the CTA computes, for every step, the slow element factor of its tile (uniform
// over the CTA) into shared memory; the step's packed fast part (shift, fast table rows,
// state masks) and its term's S x S coupling block are tile-independent tables in global
// memory, read through L1 (this keeps the CTA's shared memory small, so that several CTAs
// share a multiprocessor on systems with thousands of steps).
// Staged groups (steps with fast shifts, and the own tile): the neighbour tile x(p + sigma_S)
// is copied to shared memory by TMA bulk copies (cp.async.bulk, one per source state) that
// complete on an mbarrier; two buffers alternate so the copy of the next staged group
// overlaps the arithmetic of the current one.  Fast shifts read the staged tile at
// row + stride; a zero halo and element factors that vanish outside the basis make
// out-of-range fast shifts contribute exactly zero.
// Direct groups (pure slow shifts): y_a += sum_b C_ab x_b(p + sigma_S) with C uniform; their
// loads go straight to global memory while a staged copy is in flight.
// Epilogue: scale, store y, and the per-block partial of <scale*x, y>.
#include <cuda_runtime.h>

#include <cstdint>

#include "slab.h"

namespace nvb {

template <typename T>
struct SlabArgs {
    const SlabStep *steps;
    const int4 *info;  // [nsteps] packed fast part of each step
    const T *scoef;    // [nsteps][S][S] coupling block of each step's term
    int nsteps;
    const SlabGroup *groups;
    int ngroups;
    int nstaged;
    const SlabDiag *diag;
    int ndiag;
    const T *ftab;
    int ftab_len;
    const T *etab;
    int etab_len;
    const T *coef;                   // [nterms][S][S]
    const unsigned long long *mask;  // [nterms][2]
    const T *cst;                    // [S][S]
    const int *dpair;                // [S][S]
    const long long *slow_tshft;
    const int *slow_nfunc;
    const T *slow_omega;
    const long long *fast_shft;
    const T *fast_omega;
    int m, nF, pad, cols;
    long long TF, dimen;
    long long sstate;  // elements per state in a buffer: pad + TF + pad + tail
    int *err;
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// Bounded wait on an mbarrier phase: returns false after ~2^22 polls (the copy never landed).
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned phase) {
    const uint32_t a = smem_u32(bar);
    for (int i = 0; i < (1 << 22); ++i) {
        uint32_t ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(ok)
            : "r"(a), "r"(phase)
            : "memory");
        if (ok) return true;
    }
    return false;
}

__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

template <typename T>
struct SlabMaxThreads {
    static constexpr int value = sizeof(T) == 8 ? 384 : 512;
};

// packed step word: nfast (3 bits) | fast fields (4 x 2 bits) << 3 | column mask (4) << 11 |
// pair mask (16) << 15
__device__ __forceinline__ int info_nfast(unsigned w) { return (int)(w & 7u); }
__device__ __forceinline__ int info_field(unsigned w, int q) { return (int)((w >> (3 + 2 * q)) & 3u); }
__device__ __forceinline__ unsigned info_cols(unsigned w) { return (w >> 11) & 15u; }
__device__ __forceinline__ unsigned info_pairs(unsigned w) { return w >> 15; }

template <typename T, int S>
__global__ void __launch_bounds__(SlabMaxThreads<T>::value) k_hv_slab(SlabArgs<T> A, const T *__restrict__ x,
                                                                      T *__restrict__ y,
                                                                      const double *__restrict__ scale_dev,
                                                                      double *__restrict__ alpha_part) {
    extern __shared__ __align__(128) unsigned char smem[];
    const SlabLayout Lo =
        slab_layout(A.ftab_len, A.etab_len, A.nsteps, A.ngroups - A.nstaged, S, A.m, A.sstate, (int)sizeof(T));
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem);
    T *s_ftab = reinterpret_cast<T *>(smem + Lo.ftab);
    T *s_etab = reinterpret_cast<T *>(smem + Lo.etab);
    T *s_sf = reinterpret_cast<T *>(smem + Lo.sf);  // [nsteps] slow element factor of each step
    T *s_cg = reinterpret_cast<T *>(smem + Lo.cg);
    int *s_sd = reinterpret_cast<int *>(smem + Lo.sd);
    T *s_buf = reinterpret_cast<T *>(smem + Lo.buf);
    const int stride_state = (int)A.sstate;  // shared-memory offsets fit in 32 bits
    const int stride_buf = stride_state * S;
    const int TF = (int)A.TF;
    constexpr int S2 = S * S;

    const int tid = threadIdx.x, nth = blockDim.x;
    const long long tile = blockIdx.x;
    for (int i = tid; i < A.ftab_len; i += nth) s_ftab[i] = A.ftab[i];
    for (int i = tid; i < A.etab_len; i += nth) s_etab[i] = A.etab[i];
    if (tid == 0) {
        long long rem = tile;
        for (int l = 0; l < A.m; ++l) {
            const long long d = rem / A.slow_tshft[l];
            rem -= d * A.slow_tshft[l];
            s_sd[l] = (int)d;
        }
        for (int b = 0; b < SLAB_NBUF; ++b) mbar_init(&bar[b], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int b = 0; b < SLAB_NBUF; ++b)
        for (int s = 0; s < S; ++s) {
            T *base = s_buf + b * stride_buf + s * stride_state;
            for (int i = tid; i < A.pad; i += nth) base[i] = (T)0;
            for (int i = A.pad + TF + tid; i < stride_state; i += nth) base[i] = (T)0;
        }
    __syncthreads();
    // per-CTA slow element factor of every step (zero where the slow neighbour leaves the
    // basis); the step's fast part and coupling block are tile-independent (A.info, A.scoef)
    for (int i = tid; i < A.nsteps; i += nth) {
        const SlabStep *st = A.steps + i;
        T sf = 1;
        const int nsl = st->nslow;
        for (int q = 0; q < nsl; ++q) {
            const int md = st->slow_mode[q];
            const int n = s_sd[md];
            const int nc = n + st->slow_sig[q];
            if (nc < 0 || nc >= A.slow_nfunc[md]) {
                sf = 0;
                break;
            }
            sf = sf * s_etab[st->slow_etab[q] + (nc < n ? nc : n)];
        }
        s_sf[i] = sf;
    }
    __syncthreads();
    // direct groups: the sum of their steps' blocks (uniform over the tile)
    for (int q = A.nstaged + tid; q < A.ngroups; q += nth) {
        const SlabGroup *G = A.groups + q;
        T C[S2];
#pragma unroll
        for (int ab = 0; ab < S2; ++ab) C[ab] = 0;
        for (int i = G->step_begin; i < G->step_end; ++i) {
            const T sf = s_sf[i];
#pragma unroll
            for (int ab = 0; ab < S2; ++ab) C[ab] += __ldg(A.scoef + (size_t)i * S2 + ab) * sf;
        }
#pragma unroll
        for (int ab = 0; ab < S2; ++ab) s_cg[(q - A.nstaged) * S2 + ab] = C[ab];
    }

    auto group_valid = [&](int g) {
        const SlabGroup *G = A.groups + g;
        for (int l = 0; l < A.m; ++l) {
            const int n = s_sd[l] + G->sig[l];
            if (n < 0 || n >= A.slow_nfunc[l]) return false;
        }
        return true;
    };
    auto next_valid = [&](int g) {
        for (int q = g + 1; q < A.nstaged; ++q)
            if (group_valid(q)) return q;
        return -1;
    };
    const unsigned tile_bytes = (unsigned)(A.TF * sizeof(T));
    auto issue = [&](int g, int b) {  // thread 0 only
        const SlabGroup *G = A.groups + g;
        const unsigned msk = G->state_mask;
        fence_proxy_async();
        mbar_expect_tx(&bar[b], (unsigned)__popc(msk) * tile_bytes);
        const long long src_tile = tile + G->tile_shift;
#pragma unroll
        for (int s = 0; s < S; ++s)
            if (msk & (1u << s))
                bulk_g2s(s_buf + b * stride_buf + s * stride_state + A.pad, x + s * A.dimen + src_tile * A.TF,
                         tile_bytes, &bar[b]);
    };

    // per-row fast digits (8 bits per fast mode)
    uint32_t pk[SLAB_RPT];
#pragma unroll
    for (int k = 0; k < SLAB_RPT; ++k) {
        const long long r = (long long)k * nth + tid;
        uint32_t p = 0;
        if (r < A.TF) {
            long long rem = r;
            for (int j = 0; j < A.nF; ++j) {
                const long long d = rem / A.fast_shft[j];
                rem -= d * A.fast_shft[j];
                p |= (uint32_t)d << (8 * j);
            }
        }
        pk[k] = p;
    }
    // digits of the fast fields other than the slowest one, identical for every k in the
    // column mapping
    const uint32_t pkt = pk[0] & ~0xFFu;
    T acc[S][SLAB_RPT];
#pragma unroll
    for (int a = 0; a < S; ++a)
#pragma unroll
        for (int k = 0; k < SLAB_RPT; ++k) acc[a][k] = 0;

    unsigned phase_bits = 0;  // bit b = parity of the next completion of buffer b
    int g = 0, bi = 0;
    int nxt = next_valid(0);
    __syncthreads();  // step tables complete
    if (tid == 0) {
        issue(0, 0);
        if (nxt >= 0) issue(nxt, 1);
    }

    int dnext = A.nstaged;
    const int ndirect = A.ngroups - A.nstaged;
    const int quota = A.nstaged > 0 ? (ndirect + A.nstaged - 1) / A.nstaged : ndirect;
    auto do_direct = [&](int count) {
        while (count > 0 && dnext < A.ngroups) {
            const int q = dnext++;
            if (!group_valid(q)) continue;
            --count;
            const SlabGroup *G = A.groups + q;
            T C[S2];
#pragma unroll
            for (int ab = 0; ab < S2; ++ab) C[ab] = s_cg[(q - A.nstaged) * S2 + ab];
            const long long base = (tile + G->tile_shift) * A.TF;
            const unsigned smask = G->state_mask;
#pragma unroll
            for (int b = 0; b < S; ++b) {
                if (!(smask & (1u << b))) continue;
                T xb[SLAB_RPT];
                const T *src = x + b * A.dimen + base + tid;
#pragma unroll
                for (int k = 0; k < SLAB_RPT; ++k) xb[k] = (k * nth + tid < TF) ? __ldcg(src + k * nth) : (T)0;
#pragma unroll
                for (int a = 0; a < S; ++a)
                    if (C[a * S + b] != (T)0) {
#pragma unroll
                        for (int k = 0; k < SLAB_RPT; ++k) acc[a][k] = acc[a][k] + C[a * S + b] * xb[k];
                    }
            }
        }
    };

    bool failed = false;
    while (g >= 0) {
        do_direct(quota);
        // the decision to give up is block-wide: every thread leaves the loop together (its
        // barriers stay uniform), and the copies still in flight are drained below
        const bool landed = mbar_wait(&bar[bi], (phase_bits >> bi) & 1u);
        if (__syncthreads_or(!landed)) {
            failed = true;
            break;
        }
        phase_bits ^= 1u << bi;
        const T *buf = s_buf + bi * stride_buf + A.pad;
        if (g == 0) {
            // diagonal section: harmonic energy, constants and zero-shift even terms
            T xown[S][SLAB_RPT];
#pragma unroll
            for (int a = 0; a < S; ++a)
#pragma unroll
                for (int k = 0; k < SLAB_RPT; ++k) xown[a][k] = buf[a * stride_state + k * nth + tid];
            T ekin[SLAB_RPT];
            {
                T slow_ekin = 0;
                for (int l = 0; l < A.m; ++l) slow_ekin += A.slow_omega[l] * ((T)s_sd[l] + (T)0.5);
#pragma unroll
                for (int k = 0; k < SLAB_RPT; ++k) {
                    T e = slow_ekin;
                    for (int j = 0; j < A.nF; ++j) e += A.fast_omega[j] * ((T)((pk[k] >> (8 * j)) & 0xFFu) + (T)0.5);
                    ekin[k] = e;
                }
            }
#pragma unroll
            for (int a = 0; a < S; ++a)
#pragma unroll
                for (int k = 0; k < SLAB_RPT; ++k) {
                    T v = (A.cst[a * S + a] + ekin[k]) * xown[a][k];
#pragma unroll
                    for (int b = 0; b < S; ++b)
                        if (b != a && A.dpair[a * S + b]) v = v + A.cst[a * S + b] * xown[b][k];
                    acc[a][k] += v;
                }
            for (int i = 0; i < A.ndiag; ++i) {
                const SlabDiag *dg = A.diag + i;
                T sf = 1;
                const int nsl = dg->nslow, nfa = dg->nfast;
                for (int q = 0; q < nsl; ++q) sf = sf * s_etab[dg->slow_etab[q] + s_sd[dg->slow_mode[q]]];
                T e[SLAB_RPT];
#pragma unroll
                for (int k = 0; k < SLAB_RPT; ++k) e[k] = sf;
                for (int q = 0; q < nfa; ++q) {
                    const int sh = 8 * dg->fast_field[q];
                    const T *row = s_ftab + dg->fast_row[q];
#pragma unroll
                    for (int k = 0; k < SLAB_RPT; ++k) e[k] = e[k] * row[(int)((pk[k] >> sh) & 0xFFu)];
                }
                const int dterm = dg->term;
                const unsigned pm = (unsigned)(A.mask[2 * dterm] & 0xFFFFull);
#pragma unroll
                for (int a = 0; a < S; ++a)
#pragma unroll
                    for (int b = 0; b < S; ++b)
                        if (((pm >> (a * S + b)) & 1u) && A.dpair[a * S + b]) {
                            const T c = A.coef[(size_t)dterm * S2 + a * S + b];
#pragma unroll
                            for (int k = 0; k < SLAB_RPT; ++k) acc[a][k] = acc[a][k] + c * e[k] * xown[b][k];
                        }
            }
        }
        const int sbeg = A.groups[g].step_begin, send = A.groups[g].step_end;
        for (int i = sbeg; i < send; ++i) {
            const int4 inf = __ldg(A.info + i);
            const unsigned w = (unsigned)inf.y;
            const int nfa = info_nfast(w);
            T e[SLAB_RPT];
#pragma unroll
            for (int k = 0; k < SLAB_RPT; ++k) e[k] = 1;
            if (nfa >= 1 && A.cols) {
                // the slowest fast mode's digit is k (uniform table reads), the others are fixed
                T et = 1;
                int mrow = -1;
                for (int q = 0; q < nfa; ++q) {
                    const int f = info_field(w, q);
                    const int off = q == 0 ? (inf.z & 0xFFFF)
                                           : q == 1 ? (int)((unsigned)inf.z >> 16)
                                                    : q == 2 ? (inf.w & 0xFFFF) : (int)((unsigned)inf.w >> 16);
                    if (f == 0) mrow = off;
                    else et *= s_ftab[off + (int)((pkt >> (8 * f)) & 0xFFu)];
                }
                if (mrow >= 0) {
#pragma unroll
                    for (int k = 0; k < SLAB_RPT; ++k) e[k] = et * s_ftab[mrow + k];
                } else {
#pragma unroll
                    for (int k = 0; k < SLAB_RPT; ++k) e[k] = et;
                }
            } else if (nfa >= 1) {
                const T *row = s_ftab + (inf.z & 0xFFFF);
                const int sh = 8 * info_field(w, 0);
#pragma unroll
                for (int k = 0; k < SLAB_RPT; ++k) e[k] = row[(int)((pk[k] >> sh) & 0xFFu)];
                if (nfa >= 2) {
                    const T *row2 = s_ftab + ((unsigned)inf.z >> 16);
                    const int sh2 = 8 * info_field(w, 1);
#pragma unroll
                    for (int k = 0; k < SLAB_RPT; ++k) e[k] *= row2[(int)((pk[k] >> sh2) & 0xFFu)];
                    for (int q = 2; q < nfa; ++q) {
                        const T *rq = s_ftab + (q == 2 ? (inf.w & 0xFFFF) : ((unsigned)inf.w >> 16));
                        const int shq = 8 * info_field(w, q);
#pragma unroll
                        for (int k = 0; k < SLAB_RPT; ++k) e[k] *= rq[(int)((pk[k] >> shq) & 0xFFu)];
                    }
                }
            }
            const unsigned cols = info_cols(w), pairs = info_pairs(w);
            const T sfi = s_sf[i];
            const T *cm = A.scoef + (size_t)i * S2;
#pragma unroll
            for (int b = 0; b < S; ++b) {
                if (!((cols >> b) & 1u)) continue;
                T xb[SLAB_RPT];
                const T *src = buf + (b * stride_state + inf.x + tid);
#pragma unroll
                for (int k = 0; k < SLAB_RPT; ++k) xb[k] = src[k * nth];
                if (nfa >= 1) {
#pragma unroll
                    for (int k = 0; k < SLAB_RPT; ++k) xb[k] *= e[k];
                }
#pragma unroll
                for (int a = 0; a < S; ++a)
                    if ((pairs >> (a * S + b)) & 1u) {
                        const T c = __ldg(cm + a * S + b) * sfi;
#pragma unroll
                        for (int k = 0; k < SLAB_RPT; ++k) acc[a][k] = acc[a][k] + c * xb[k];
                    }
            }
        }
        __syncthreads();  // every thread is done with buffer bi
        const int n2 = nxt >= 0 ? next_valid(nxt) : -1;
        if (tid == 0 && n2 >= 0) issue(n2, bi);
        g = nxt;
        nxt = n2;
        bi ^= 1;
    }
    if (failed) {
        if (tid == 0) {
            // buffer bi holds the copy that was awaited, buffer bi^1 the next group's copy
            // (issued when there is one): wait for both (bounded) before the CTA leaves, so
            // that no bulk copy completes into the shared memory of an exited CTA
            mbar_wait(&bar[bi], (phase_bits >> bi) & 1u);
            if (nxt >= 0) mbar_wait(&bar[bi ^ 1], (phase_bits >> (bi ^ 1)) & 1u);
            atomicExch(A.err, 1);
        }
        return;
    }
    do_direct(A.ngroups);
    const T sc = scale_dev ? (T)(*scale_dev) : (T)1;
    double part = 0.0;
#pragma unroll
    for (int a = 0; a < S; ++a)
#pragma unroll
        for (int k = 0; k < SLAB_RPT; ++k) {
            const long long r = (long long)k * nth + tid;
            if (r < A.TF) {
                const T v = acc[a][k] * sc;
                const long long gi = a * A.dimen + tile * A.TF + r;
                y[gi] = v;
                if (alpha_part) part += ((double)__ldcg(x + gi) * (double)sc) * (double)v;
            }
        }
    if (alpha_part) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
        __shared__ double red[32];
        if ((tid & 31) == 0) red[tid >> 5] = part;
        __syncthreads();
        if (tid < 32) {
            double v = tid < (nth >> 5) ? red[tid] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (tid == 0) alpha_part[blockIdx.x] = v;
        }
    }
}

template <typename T>
static SlabArgs<T> slab_args(const SlabPlan &sp, const Plan &pl) {
    SlabArgs<T> a{};
    a.steps = sp.d_steps;
    a.info = sp.d_info;
    a.nsteps = (int)sp.steps.size();
    a.groups = sp.d_groups;
    a.ngroups = (int)sp.groups.size();
    a.nstaged = sp.nstaged;
    a.diag = sp.d_diag;
    a.ndiag = (int)sp.diag.size();
    a.ftab_len = (int)sp.ftab.size();
    a.etab_len = (int)pl.h_etab.size();
    a.mask = pl.d_mask;
    a.dpair = pl.d_dpair;
    a.slow_tshft = sp.d_slow_tshft;
    a.slow_nfunc = sp.d_slow_nfunc;
    a.fast_shft = sp.d_fast_shft;
    a.m = sp.m;
    a.cols = sp.cols;
    a.nF = sp.nF;
    a.pad = sp.pad;
    a.TF = sp.TF;
    a.dimen = pl.dimen;
    a.sstate = sp.sstate;
    a.err = sp.d_err;
    if constexpr (sizeof(T) == 8) {
        a.ftab = (const T *)sp.d_ftab;
        a.etab = (const T *)pl.d_etab;
        a.coef = (const T *)pl.d_coef;
        a.scoef = (const T *)sp.d_scoef;
        a.cst = (const T *)pl.d_const;
        a.slow_omega = (const T *)sp.d_slow_omega;
        a.fast_omega = (const T *)sp.d_fast_omega;
    } else {
        a.ftab = (const T *)sp.d_ftab_f;
        a.etab = (const T *)pl.d_etab_f;
        a.coef = (const T *)pl.d_coef_f;
        a.scoef = (const T *)sp.d_scoef_f;
        a.cst = (const T *)pl.d_const_f;
        a.slow_omega = (const T *)sp.d_slow_omega_f;
        a.fast_omega = (const T *)sp.d_fast_omega_f;
    }
    return a;
}

template <typename T, int S>
static void launch_slab_s(const SlabPlan &sp, const Plan &pl, const T *x, T *y, const double *sc, double *ap,
                          cudaStream_t st) {
    const size_t smem = sp.smem_bytes[sizeof(T) == 8 ? 0 : 1];
    cudaFuncSetAttribute(k_hv_slab<T, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_hv_slab<T, S><<<(unsigned)sp.ntiles, sp.threads, smem, st>>>(slab_args<T>(sp, pl), x, y, sc, ap);
}

template <typename T>
void slab_launch(const SlabPlan &sp, const Plan &pl, const T *x, T *y, const double *scale, double *alpha_part,
                 cudaStream_t st) {
    switch (pl.S) {
    case 1: launch_slab_s<T, 1>(sp, pl, x, y, scale, alpha_part, st); break;
    case 2: launch_slab_s<T, 2>(sp, pl, x, y, scale, alpha_part, st); break;
    case 3: launch_slab_s<T, 3>(sp, pl, x, y, scale, alpha_part, st); break;
    case 4: launch_slab_s<T, 4>(sp, pl, x, y, scale, alpha_part, st); break;
    default: fail(NVB_ERR_ARG, "slab kernel supports up to 4 states");
    }
}

template void slab_launch<double>(const SlabPlan &, const Plan &, const double *, double *, const double *, double *,
                                  cudaStream_t);
template void slab_launch<float>(const SlabPlan &, const Plan &, const float *, float *, const double *, double *,
                                 cudaStream_t);

}  // namespace nvb
