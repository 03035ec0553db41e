// Factorised quadratic H.v kernel (see quad.h for the algebra).
//
// Warp-specialised persistent CTAs walk the tiles (fixed slow digits) with a stride of the
// grid.  The last warp is the producer: it lists each tile's valid items one tile ahead, and
// one lane walks the same item sequence as the consumers (per tile, per target state a: the
// own tile x_a, the other states' own tiles, the slow +-1 / +-2 / bilinear neighbour tiles),
// copying each item into the next slot of a ring of shared-memory buffers with a TMA bulk
// copy completing on the slot's "full" mbarrier, after the consumers released the slot on its
// "empty" mbarrier.  The other warps are the consumers; a thread owns the pencil of mode m
// (rows r*shft(m) + tid) and folds each item into registers:
//   own x_a:      diagonal section, Z_l += G^aa_l x_a + Q^a_kl X_k x_a (fast k < l), squares;
//   own x_b:      off-diagonal diagonal-section entries, Z_l += G^ab_l x_b, squares of x_b;
//   slow +-1:     y_a += G^ab_k e x_b(p+-e_k), Z_l += Q^a_kl e x_a(p+-e_k);
//   slow +-2:     y_a += R^ab_k e x_b(p+-2e_k);
//   slow pairs:   y_a += Q^a_kl e x_a(p+-e_k+-e_l);
// with e the tile's slow element factor.  Finally y_a += X_l Z_l: by register shifts for
// l = m, and for each other fast mode through one shared-memory buffer (one mode at a time,
// so that the buffer costs one ring slot, not NF - 1).  Out-of-basis neighbours have element
// factor 0 (the item is skipped by producer and consumers alike) and zero-filled halos.
// Every wait is bounded: a wait that runs out raises a CTA abort flag, after which no thread
// waits again and the kernel reports the failure through its error word.
#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>

#include "quad.h"

namespace nvb {

namespace {

template <typename T>
struct QuadArgs {
    const T *blk;  // tab | G | R | Q | cst | omega
    const int *slow;
    const QuadItem *items;
    const int *item_beg;
    int *err;
    int M, m, nmax, nv, pad, sstate, TF, ntiles, nslot, nitems;
    int nocopy;      // failure test: the producer issues no copy, so every consumer wait runs out
    int wait_limit;  // polls before a wait gives up
    long long dimen;
    unsigned dpm;
    unsigned ownmask;  // bit a*S+b: the other state's own tile x_b is an item of target a
    QuadFast<T> F;
};

// consumers (<= 288 = 9 warps) + the producer warp: 10 warps keep <= 3 warps per SM sub-partition,
// so a thread may hold up to 168 registers
constexpr int QUAD_MAXTH = 288 + 32;
constexpr int R = QUAD_RPT;
constexpr int WAIT_LIMIT = 1 << 22;

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// arrive on bar when pred holds (a predicated instruction, no branch)
__device__ __forceinline__ void mbar_arrive_if(uint64_t *bar, bool pred) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.u32 p, %1, 0;\n @p mbarrier.arrive.shared::cta.b64 _, [%0];\n}\n" ::"r"(
            smem_u32(bar)),
        "r"((unsigned)pred)
        : "memory");
}

__device__ __forceinline__ bool mbar_try(uint64_t *bar, unsigned parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait on a phase; gives up (and raises the abort flag) after `limit` polls, or early
// once another thread raised it.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity, volatile int *abort_flag,
                                          int limit = WAIT_LIMIT) {
    for (int i = 0; i < limit; ++i) {
        if (mbar_try(bar, parity)) return true;
        if ((i & 255) == 255 && *abort_flag) return false;
    }
    *abort_flag = 1;
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

// barrier 1 among the consumer warps only (the producer never joins it)
__device__ __forceinline__ void consumer_sync(int n) { asm volatile("bar.sync 1, %0;" ::"r"(n) : "memory"); }

// element-table row of an item's (first or second) slow factor
__device__ __forceinline__ int item_row(int kind, int s) {
    return kind == QI_SLOW2 ? (s > 0 ? 2 : 3) : (s > 0 ? 0 : 1);
}

// NC > 0: the number of consumer threads (= shft(m)) as a compile-time constant, so that the
// rows of a thread's pencil are immediate offsets; NC = 0 reads it from the launch.
template <typename T, int S, int NF, int NC>
__global__ void __launch_bounds__(QUAD_MAXTH, sizeof(T) == 4 ? 2 : 1)
    k_hv_quad(const QuadArgs<T> A, const T *__restrict__ x, T *__restrict__ y, const double *__restrict__ scale_dev,
              double *__restrict__ alpha_part) {
    extern __shared__ __align__(128) unsigned char smem[];
    const int M = A.M, m = A.m, nmax = A.nmax, sst = A.sstate, TF = A.TF, NS = A.nslot, pad = A.pad;
    const QuadLayout Lo = quad_layout(M, S, nmax, m, NF, sst, (int)sizeof(T), NS, A.nitems);
    uint64_t *full = reinterpret_cast<uint64_t *>(smem);
    uint64_t *empty = full + QUAD_MAXSLOT;
    volatile int *abort_flag = reinterpret_cast<volatile int *>(smem + 2 * QUAD_MAXSLOT * 8);
    T *s_tab = reinterpret_cast<T *>(smem + Lo.tab);
    T *s_G = reinterpret_cast<T *>(smem + Lo.G);
    T *s_R = reinterpret_cast<T *>(smem + Lo.R);
    T *s_Q = reinterpret_cast<T *>(smem + Lo.Q);
    T *s_cst = reinterpret_cast<T *>(smem + Lo.cst);
    T *s_om = reinterpret_cast<T *>(smem + Lo.om);
    int *s_sl = reinterpret_cast<int *>(smem + Lo.sd);  // slow tile strides [MAXSL], nfunc [MAXSL]
    T *s_se = reinterpret_cast<T *>(smem + Lo.se);      // [2][MAXSL][5] slow element factors of a tile
    T *s_dt = reinterpret_cast<T *>(smem + Lo.dt);      // [2][S*S+1] slow diagonal block, energy
    QuadItem *s_it = reinterpret_cast<QuadItem *>(smem + Lo.items);
    int *s_cnt = reinterpret_cast<int *>(smem + Lo.cnt);  // [2][MAXS][2]
    T *s_rec = reinterpret_cast<T *>(smem + Lo.rec);      // [2][nitems][NF+1]
    int *s_ib = reinterpret_cast<int *>(smem + Lo.items + A.nitems * (int)sizeof(QuadItem));
    T *s_ring = reinterpret_cast<T *>(smem + Lo.ring);  // [NS][sst]
    T *s_z = reinterpret_cast<T *>(smem + Lo.z);        // [sst] Z_l of one fast mode l > m
    const int tid = threadIdx.x;
    const int nc = NC > 0 ? NC : (int)blockDim.x - 32;  // consumer threads = shft(m)
    const long long N = A.dimen;
    const QuadFast<T> &F = A.F;
    constexpr int SS = S * S;
    const int *tsh = s_sl, *snf = s_sl + QUAD_MAXSL;

    {
        const int ntab = M * 5 * nmax, nG = M * SS, nQ = M * M * S;
        const T *src = A.blk;
        for (int i = tid; i < ntab; i += blockDim.x) s_tab[i] = src[i];
        src += ntab;
        for (int i = tid; i < nG; i += blockDim.x) s_G[i] = src[i];
        src += nG;
        for (int i = tid; i < nG; i += blockDim.x) s_R[i] = src[i];
        src += nG;
        for (int i = tid; i < nQ; i += blockDim.x) s_Q[i] = src[i];
        src += nQ;
        for (int i = tid; i < SS; i += blockDim.x) s_cst[i] = src[i];
        src += SS;
        for (int i = tid; i < M; i += blockDim.x) s_om[i] = src[i];
        for (int i = tid; i < m; i += blockDim.x) {
            s_sl[i] = A.slow[i];
            s_sl[QUAD_MAXSL + i] = A.slow[m + i];
        }
        for (int i = tid; i < A.nitems; i += blockDim.x) s_it[i] = A.items[i];
        for (int i = tid; i <= 3 * S; i += blockDim.x) s_ib[i] = A.item_beg[i];
        const int nz = (NS + 1) * sst;  // ring and Z are contiguous
        for (int i = tid; i < nz; i += blockDim.x) s_ring[i] = (T)0;
    }
    if (tid == 0) {
        for (int i = 0; i < NS; ++i) {
            mbar_init(&full[i], 1);
            mbar_init(&empty[i], (unsigned)(nc >> 5));
        }
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    fence_proxy_async();
    __syncthreads();

    if (tid >= nc) {
        // ---------------- producer ----------------
        // One tile ahead of the copies the warp lists the tile's present items (ballot per 32
        // items, compacted into s_pl[q] for tile parity q: the count, then each item's source
        // offset in x relative to the tile); lane 0 then issues the tile's copies from the list
        // in consumption order, each after its slot was released, reading the next offset
        // before it waits.  (The producer lane is on the critical path: listing ahead keeps the
        // ballots out of the gap between two tiles' copies, and the precomputed offsets keep
        // the item records and their address arithmetic out of the issue loop; one issuing lane
        // keeps the copies in the order the consumers take them.)
        const int lane = tid - nc;
        const unsigned bytes = (unsigned)TF * (unsigned)sizeof(T);
        const int nit = s_ib[S];
        long long *s_pl = reinterpret_cast<long long *>(smem + Lo.plist);  // [2][nitems + 1]
        auto list = [&](int tile, int q) {
            long long *pl = s_pl + q * (nit + 1);
            int base = 0;
            for (int i0 = 0; i0 < nit; i0 += 32) {
                const int it = i0 + lane;
                bool ok = false;
                if (it < nit) {
                    const QuadItem qi = s_it[it];
                    ok = true;
                    if (qi.kind != QI_OWN) {
                        const int dk = (tile / tsh[qi.k]) % snf[qi.k];
                        ok = s_tab[(qi.k * 5 + item_row(qi.kind, qi.sk)) * nmax + dk] != (T)0;
                        if (qi.kind == QI_PAIR) {
                            const int dl = (tile / tsh[qi.l]) % snf[qi.l];
                            ok = ok && s_tab[(qi.l * 5 + item_row(qi.kind, qi.sl)) * nmax + dl] != (T)0;
                        }
                    }
                }
                const unsigned bal = __ballot_sync(0xffffffffu, ok);
                if (ok) {
                    const QuadItem &qi = s_it[it];
                    pl[1 + base + __popc(bal & ((1u << lane) - 1u))] =
                        (long long)qi.b * N + (long long)qi.tshift * TF;
                }
                base += __popc(bal);
            }
            if (lane == 0) pl[0] = base;
            __syncwarp();
        };
        // Issuing lanes: lane L < IL issues the items with global index g = L, L + IL, ... into
        // slot g % NS (phase (g / NS) & 1), so every slot is still filled in item order and
        // guarded by its own empty / full phases.  FP32 streams twice as many (half-size) tiles
        // per byte and issues from two lanes (5 % faster on config 2); FP64 from one.
        constexpr int IL = sizeof(T) == 4 ? 2 : 1;
        int slot = lane % NS;
        unsigned ph = 0;
        long long issued = 0, g0 = 0;  // g0: global index of the tile's first item
        int stop = A.nocopy;
        if (blockIdx.x < A.ntiles) list(blockIdx.x, 0);
        int q = 0;
        for (int tile = blockIdx.x; tile < A.ntiles && !stop; tile += gridDim.x, q ^= 1) {
            if (tile + (int)gridDim.x < A.ntiles) list(tile + gridDim.x, q ^ 1);
            const long long *pl = s_pl + q * (nit + 1);
            const int cnt = (int)pl[0];
            if (lane < IL) {
                const T *xt = x + (long long)tile * TF;
                int i = 0;
                if constexpr (IL > 1) i = (int)(((lane - g0) % IL + IL) % IL);
                long long nxt = i < cnt ? pl[1 + i] : 0;
                for (; i < cnt && !stop; i += IL) {
                    const long long off = nxt;
                    if (i + IL < cnt) nxt = pl[1 + i + IL];
                    // No slot whose copy may still be in flight is ever free here: a consumer
                    // whose wait gave up does not release its slot, so the producer's wait for
                    // that slot runs out (or sees the abort flag) and it stops.  (Reading the
                    // abort flag before every copy as well costs ~20 % of the kernel time: the
                    // producer lanes are on the critical path.)
                    if (mbar_wait(&empty[slot], ph ^ 1u, abort_flag, A.wait_limit)) {
                        mbar_expect_tx(&full[slot], bytes);
                        bulk_g2s(s_ring + slot * sst + pad, xt + off, bytes, &full[slot]);
                        ++issued;
                    } else {
                        stop = 1;
                    }
                    if constexpr (IL == 1) {
                        if (++slot == NS) {
                            slot = 0;
                            ph ^= 1u;
                        }
                    } else {
                        slot += IL;
                        if (slot >= NS) {
                            slot -= NS;
                            ph ^= 1u;
                        }
                    }
                }
            }
            if constexpr (IL > 1) {
                g0 += cnt;
                stop = __any_sync(0xffffffffu, stop);
            } else {
                stop = __shfl_sync(0xffffffffu, stop, 0);
            }
        }
        if (lane < IL && stop) {
            // each issuing lane waits (bounded) for its own copies still in flight (its k-th
            // copy went to slot (L + IL k) % NS) before the CTA leaves
            const long long per = (NS + IL - 1) / IL;
            const long long n = issued < per ? issued : per;
            for (long long k = issued - n; k < issued; ++k) {
                const long long g = lane + (long long)IL * k;
                const int s2 = (int)(g % NS);
                const unsigned p = (unsigned)((g / NS) & 1);
                for (int w = 0; w < WAIT_LIMIT && !mbar_try(&full[s2], p); ++w) {
                }
            }
            atomicExch(A.err, 1);
        }
        return;
    }

    // ---------------- consumers ----------------
    // the thread's digits and ladder factors along the fast modes j >= 1; FP64 reads the factors
    // from the element table when used (registers are its limit: 168 per thread at 10 warps)
    int dj[NF];
    T e1pa[NF], e1ma[NF];
#pragma unroll
    for (int j = 0; j < NF; ++j) {
        dj[j] = 0;
        e1pa[j] = e1ma[j] = (T)0;
        if (j >= 1) {
            dj[j] = (tid / F.sh[j]) % F.nf[j];
            if constexpr (sizeof(T) == 4) {
                e1pa[j] = s_tab[((m + j) * 5 + 0) * nmax + dj[j]];
                e1ma[j] = s_tab[((m + j) * 5 + 1) * nmax + dj[j]];
            }
        }
    }
    auto e1p = [&](int j) -> T {
        if constexpr (sizeof(T) == 8) return s_tab[((m + j) * 5 + 0) * nmax + dj[j]];
        else return e1pa[j];
    };
    auto e1m = [&](int j) -> T {
        if constexpr (sizeof(T) == 8) return s_tab[((m + j) * 5 + 1) * nmax + dj[j]];
        else return e1ma[j];
    };
    const T sc = scale_dev ? (T)(*scale_dev) : (T)1;
    const int nv = A.nv;
    const int lane = tid & 31, wid = tid >> 5;
    // FP32: items are folded without testing their wait's outcome (after an abort the results
    // are discarded by the host) and slots are released by a predicated arrive, both without
    // branches; measured 3 % faster in FP32 and 4 % slower in FP64, so FP64 keeps the branches
    constexpr bool kNoBranch = sizeof(T) == 4;
    constexpr bool kSpreadXZ = sizeof(T) == 8;
    double part = 0.0;
    int slot = 0;
    unsigned ph = 0;
    int tp = 0;
    bool ok = true;
    // the next ring slot: wait for its copy (bounded), return this thread's column in it
    auto take = [&]() -> const T * {
        ok = mbar_try(&full[slot], ph) || mbar_wait(&full[slot], ph, abort_flag, A.wait_limit);
        return s_ring + slot * sst + pad + tid;
    };
    // hand the slot back to the producer (one arrival per warp, by lane 0) and step to the
    // next one.  Only a lane 0 that saw the slot's copy land releases it: a slot whose wait
    // gave up may still be the target of a copy in flight, so it is never handed back (the
    // producer then stops on the abort flag and drains its copies before the CTA exits).
    auto release = [&]() {
        __syncwarp();
        if constexpr (kNoBranch) mbar_arrive_if(&empty[slot], lane == 0 && ok);
        else if (lane == 0 && ok) mbar_arrive(&empty[slot]);
        if (++slot == NS) {
            slot = 0;
            ph ^= 1u;
        }
    };
    for (int tile = blockIdx.x; tile < A.ntiles; tile += gridDim.x, tp ^= 1) {
        // the tile's slow element factors and the slow part of the diagonal block
        if (tid < m) {
            const int l = tid;
            const int d = (tile / tsh[l]) % snf[l];
#pragma unroll
            for (int q = 0; q < 5; ++q) s_se[(tp * QUAD_MAXSL + l) * 5 + q] = s_tab[(l * 5 + q) * nmax + d];
        } else if (tid >= 32 && tid < 32 + SS + 1) {
            const int ab = tid - 32;
            T v = 0;
            if (ab < SS) {
                v = s_cst[ab];
                if ((A.dpm >> ab) & 1u)
                    for (int l = 0; l < m; ++l) {
                        const int d = (tile / tsh[l]) % snf[l];
                        v += s_R[l * SS + ab] * s_tab[(l * 5 + 4) * nmax + d];
                    }
            } else {
                for (int l = 0; l < m; ++l) {
                    const int d = (tile / tsh[l]) % snf[l];
                    v += s_om[l] * ((T)d + (T)0.5);
                }
            }
            s_dt[tp * (SS + 1) + ab] = v;
        }
        consumer_sync(nc);
        const T *se = s_se + tp * QUAD_MAXSL * 5;
        const T *dt = s_dt + tp * (SS + 1);
        // records of the tile's present slow items, compacted per target state a by one
        // consumer warp (warp a mod the consumer warps) in the producer's order: coefficient c and z[j] with the slow element factors folded in
        // (z only for the Z items, which come first); the counts go to s_cnt
        for (int a = wid; a < S; a += nc >> 5) {  // nc >= 64: at least two consumer warps
            const int beg = s_ib[S + 1 + a], zend = s_ib[2 * S + 1 + a], end = s_ib[a + 1];
            T *rc = s_rec + (tp * A.nitems + s_ib[a]) * (NF + 1);
            int base = 0, nzp = 0;
            for (int i0 = beg; i0 < end; i0 += 32) {
                const int i = i0 + lane;
                bool present = false;
                T c = (T)0, z[NF];
#pragma unroll
                for (int j = 0; j < NF; ++j) z[j] = (T)0;
                if (i < end) {
                    const QuadItem q = s_it[i];
                    const int b = q.b;
                    T e = se[q.k * 5 + item_row(q.kind, q.sk)];
                    if (q.kind == QI_PAIR) e *= se[q.l * 5 + item_row(q.kind, q.sl)];
                    present = e != (T)0;
                    if (q.kind == QI_SLOW1) {
                        c = s_G[q.k * SS + a * S + b] * e;
                        if (i < zend) {
#pragma unroll
                            for (int j = 0; j < NF; ++j) z[j] = s_Q[(q.k * M + m + j) * S + a] * e;
                        }
                    } else if (q.kind == QI_SLOW2) {
                        c = s_R[q.k * SS + a * S + b] * e;
                    } else {
                        c = s_Q[(q.k * M + q.l) * S + a] * e;
                    }
                }
                const unsigned bal = __ballot_sync(0xffffffffu, present);
                const unsigned balz = __ballot_sync(0xffffffffu, present && i < zend);
                if (present) {
                    const int pos = base + __popc(bal & ((1u << lane) - 1u));
                    rc[pos * (NF + 1)] = c;
#pragma unroll
                    for (int j = 0; j < NF; ++j) rc[pos * (NF + 1) + 1 + j] = z[j];
                }
                base += __popc(bal);
                nzp += __popc(balz);
            }
            if (lane == 0) {
                s_cnt[(tp * QUAD_MAXS + a) * 2] = nzp;
                s_cnt[(tp * QUAD_MAXS + a) * 2 + 1] = base;
            }
        }
        consumer_sync(nc);
        const long long tbase = (long long)tile * TF;
#pragma unroll
        for (int a = 0; a < S; ++a) {
            T xr[R], acc[R], Z[NF][R];
#pragma unroll
            for (int r = 0; r < R; ++r) {
                xr[r] = acc[r] = (T)0;
#pragma unroll
                for (int j = 0; j < NF; ++j) Z[j][r] = (T)0;
            }
            auto hj = [&](int j) -> T { return (T)dj[j] + (T)0.5; };  // <n|x^2|n> of the fast digit j >= 1
            // own tile x_a: diagonal section, fast linear and bilinear into Z, fast squares
            {
                const T *buf = take();
                if (kNoBranch || ok) {
#pragma unroll
                    for (int r = 0; r < R; ++r) xr[r] = buf[r * nc];
                    T ek = dt[SS], daa = dt[a * S + a];
#pragma unroll
                    for (int j = 1; j < NF; ++j) {
                        ek += F.om[j] * hj(j);
                        daa += F.R[j][a][a] * hj(j);
                    }
#pragma unroll
                    for (int r = 0; r < R; ++r) {
                        const T h = (T)r + (T)0.5;
                        acc[r] += (daa + F.R[0][a][a] * h + ek + F.om[0] * h) * xr[r];
                    }
#pragma unroll
                    for (int j = 0; j < NF; ++j) {
                        const T g = F.G[j][a][a];
                        if (g != (T)0) {
#pragma unroll
                            for (int r = 0; r < R; ++r) Z[j][r] += g * xr[r];
                        }
                    }
                    // Z_l += Q^a_il X_i x_a (fast i < l)
#pragma unroll
                    for (int i = 0; i + 1 < NF; ++i) {
                        bool any = false;
#pragma unroll
                        for (int j = i + 1; j < NF; ++j) any |= F.Q[i][j][a] != (T)0;
                        if (!any) continue;
                        T V[R];
#pragma unroll
                        for (int r = 0; r < R; ++r) {
                            if (i == 0) {
                                T v = (T)0;
                                if (r + 1 < R) v += F.em[0][r] * xr[r + 1];
                                if (r >= 1) v += F.em[1][r] * xr[r - 1];
                                V[r] = v;
                            } else {
                                const T *p = buf + r * nc;
                                V[r] = e1p(i) * p[F.sh[i]] + e1m(i) * p[-F.sh[i]];
                            }
                        }
#pragma unroll
                        for (int j = i + 1; j < NF; ++j) {
                            const T qq = F.Q[i][j][a];
                            if (qq == (T)0) continue;
#pragma unroll
                            for (int r = 0; r < R; ++r) Z[j][r] += qq * V[r];
                        }
                    }
#pragma unroll
                    for (int j = 0; j < NF; ++j) {
                        const T rr = F.R[j][a][a];
                        if (rr == (T)0) continue;
                        T e2p = (T)0, e2m = (T)0;
                        if (j >= 1) {
                            e2p = s_tab[((m + j) * 5 + 2) * nmax + dj[j]];
                            e2m = s_tab[((m + j) * 5 + 3) * nmax + dj[j]];
                        }
#pragma unroll
                        for (int r = 0; r < R; ++r) {
                            T v = (T)0;
                            if (j == 0) {
                                if (r + 2 < R) v += F.em[2][r] * xr[r + 2];
                                if (r >= 2) v += F.em[3][r] * xr[r - 2];
                            } else {
                                const T *p = buf + r * nc;
                                v = e2p * p[2 * F.sh[j]] + e2m * p[-2 * F.sh[j]];
                            }
                            acc[r] += rr * v;
                        }
                    }
                }
                release();
            }
            // the other states' own tiles x_b: diagonal-section entries, fast linear into Z,
            // fast squares
#pragma unroll
            for (int b = 0; b < S; ++b) {
                if (b == a || !((A.ownmask >> (a * S + b)) & 1u)) continue;
                const T *buf = take();
                if (kNoBranch || ok) {
                    T xb[R];
#pragma unroll
                    for (int r = 0; r < R; ++r) xb[r] = buf[r * nc];
                    if ((A.dpm >> (a * S + b)) & 1u) {
                        T dab = dt[a * S + b];
#pragma unroll
                        for (int j = 1; j < NF; ++j) dab += F.R[j][a][b] * hj(j);
                        const T r0 = F.R[0][a][b];
#pragma unroll
                        for (int r = 0; r < R; ++r) acc[r] += (dab + r0 * ((T)r + (T)0.5)) * xb[r];
                    }
#pragma unroll
                    for (int j = 0; j < NF; ++j) {
                        const T g = F.G[j][a][b];
                        if (g != (T)0) {
#pragma unroll
                            for (int r = 0; r < R; ++r) Z[j][r] += g * xb[r];
                        }
                        const T rr = F.R[j][a][b];
                        if (rr != (T)0) {
                            T e2p = (T)0, e2m = (T)0;
                            if (j >= 1) {
                                e2p = s_tab[((m + j) * 5 + 2) * nmax + dj[j]];
                                e2m = s_tab[((m + j) * 5 + 3) * nmax + dj[j]];
                            }
#pragma unroll
                            for (int r = 0; r < R; ++r) {
                                T v = (T)0;
                                const T *p = buf + r * nc;
                                if (j == 0) {
                                    if (r + 2 < R) v += F.em[2][r] * p[2 * nc];
                                    if (r >= 2) v += F.em[3][r] * p[-2 * nc];
                                } else {
                                    v = e2p * p[2 * F.sh[j]] + e2m * p[-2 * F.sh[j]];
                                }
                                acc[r] += rr * v;
                            }
                        }
                    }
                }
                release();
            }
            // present slow items: the Z items (y_a += c x, Z_l += z_l x), then the
            // coefficient-only items two at a time.  Z is final once the Z items are in, so
            // y_a += X_l Z_l is applied in between the coefficient-only items: mode m at once by
            // register shifts, every other fast mode at its own evenly spaced point, through
            // the shared Z buffer between two consumer barriers.  (Applied in one block at the
            // end, these steps stalled the consumers for long enough to fill the ring and idle
            // the copies; spread out, the ring keeps streaming through each step: 3.5 % faster
            // in FP64 on the 265M-element system, neutral to slightly slower in FP32, which
            // therefore applies them after the last item.)
            {
                const int nzp = s_cnt[(tp * QUAD_MAXS + a) * 2], nsp = s_cnt[(tp * QUAD_MAXS + a) * 2 + 1];
                const T *rc = s_rec + (tp * A.nitems + s_ib[a]) * (NF + 1);
                int j = 0;
                for (; j < nzp; ++j) {
                    const T *buf = take();
                    if (kNoBranch || ok) {
                        T v[R];
#pragma unroll
                        for (int r = 0; r < R; ++r) v[r] = buf[r * nc];
                        const T c = rc[j * (NF + 1)];
#pragma unroll
                        for (int r = 0; r < R; ++r) acc[r] += c * v[r];
#pragma unroll
                        for (int q = 0; q < NF; ++q) {
                            const T zq = rc[j * (NF + 1) + 1 + q];
#pragma unroll
                            for (int r = 0; r < R; ++r) Z[q][r] += zq * v[r];
                        }
                    }
                    release();
                }
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    T v = acc[r];
                    if (r + 1 < R) v += F.em[0][r] * Z[0][r + 1];
                    if (r >= 1) v += F.em[1][r] * Z[0][r - 1];
                    acc[r] = v;
                }
                // fast mode jj >= 1: Z_jj through s_z (every consumer thread takes part)
                auto xz = [&](auto jc) {
                    constexpr int jj = decltype(jc)::value;
#pragma unroll
                    for (int r = 0; r < R; ++r) s_z[pad + r * nc + tid] = r < nv ? Z[jj][r] : (T)0;
                    consumer_sync(nc);
#pragma unroll
                    for (int r = 0; r < R; ++r) {
                        const T *p = s_z + pad + r * nc + tid;
                        acc[r] += e1p(jj) * p[F.sh[jj]] + e1m(jj) * p[-F.sh[jj]];
                    }
                    consumer_sync(nc);  // s_z is rewritten next
                };
                int done = 1;  // fast modes applied
                auto xz_next = [&]() {
                    if constexpr (NF > 1) {
                        if (done == 1) xz(std::integral_constant<int, 1>{});
                    }
                    if constexpr (NF > 2) {
                        if (done == 2) xz(std::integral_constant<int, 2>{});
                    }
                    if constexpr (NF > 3) {
                        if (done == 3) xz(std::integral_constant<int, 3>{});
                    }
                    ++done;
                };
                const int nco = nsp - nzp;  // the same in every consumer thread
                for (; j + 1 < nsp; j += 2) {
                    if (kSpreadXZ && done < NF && (j - nzp) * NF >= done * nco) xz_next();
                    // two consecutive slots: the first is held (not released) while the second
                    // is awaited; the ring has at least three slots
                    const T *b0 = take();
                    const bool ok0 = ok;
                    const int s0 = slot;
                    if (++slot == NS) {
                        slot = 0;
                        ph ^= 1u;
                    }
                    const T *b1 = take();
                    if (kNoBranch || (ok0 && ok)) {
                        T v0[R], v1[R];
#pragma unroll
                        for (int r = 0; r < R; ++r) {
                            v0[r] = b0[r * nc];
                            v1[r] = b1[r * nc];
                        }
                        const T c0 = rc[j * (NF + 1)], c1 = rc[(j + 1) * (NF + 1)];
#pragma unroll
                        for (int r = 0; r < R; ++r) acc[r] = fma(c1, v1[r], fma(c0, v0[r], acc[r]));
                    }
                    __syncwarp();
                    if constexpr (kNoBranch) mbar_arrive_if(&empty[s0], lane == 0 && ok0);
                    else if (lane == 0 && ok0) mbar_arrive(&empty[s0]);
                    release();
                }
                if (j < nsp) {
                    const T *buf = take();
                    if (kNoBranch || ok) {
                        const T c = rc[j * (NF + 1)];
#pragma unroll
                        for (int r = 0; r < R; ++r) acc[r] += c * buf[r * nc];
                    }
                    release();
                }
                while (done < NF) xz_next();
            }
#pragma unroll
            for (int r = 0; r < R; ++r)
                if (r < nv) {
                    const T v = acc[r] * sc;
                    y[a * N + tbase + r * nc + tid] = v;
                    if (alpha_part) part += ((double)xr[r] * (double)sc) * (double)v;
                }
        }
    }
    if (*abort_flag && tid == 0) atomicExch(A.err, 1);
    if (alpha_part) {
        __shared__ double red[32];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
        if ((tid & 31) == 0) red[tid >> 5] = part;
        consumer_sync(nc);
        if (tid < 32) {
            double v = tid < (nc >> 5) ? red[tid] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (tid == 0) alpha_part[blockIdx.x] = v;
        }
    }
}

template <typename T>
QuadArgs<T> quad_args(const QuadPlan &qp) {
    QuadArgs<T> a{};
    a.slow = qp.d_slow;
    a.items = qp.d_items;
    a.item_beg = qp.d_item_beg;
    a.err = qp.d_err;
    a.nocopy = qp.test_nocopy;
    a.wait_limit = qp.test_nocopy ? (1 << 14) : WAIT_LIMIT;
    a.M = qp.M;
    a.m = qp.m;
    a.nmax = qp.nmax;
    a.nv = qp.nv;
    a.pad = qp.pad;
    a.sstate = qp.sstate;
    a.TF = qp.TF;
    a.ntiles = qp.ntiles;
    a.nitems = (int)qp.items.size();
    a.dimen = qp.dimen;
    a.dpm = qp.dpm;
    a.ownmask = qp.ownmask;
    if constexpr (sizeof(T) == 8) {
        a.blk = (const T *)qp.d_blk;
        a.F = qp.fast_d;
        a.nslot = qp.nslot[0];
    } else {
        a.blk = (const T *)qp.d_blk_f;
        a.F = qp.fast_f;
        a.nslot = qp.nslot[1];
    }
    return a;
}

template <typename T, int S, int NF, int NC>
int launch_q(QuadPlan &qp, const T *x, T *y, const double *sc, double *ap, cudaStream_t st) {
    const int idx = sizeof(T) == 8 ? 0 : 1;
    const size_t smem = qp.smem[idx];
    const int threads = qp.threads + 32;
    auto kern = k_hv_quad<T, S, NF, NC>;
    if (qp.grid[idx] == 0) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        int dev = 0, nsm = 0, per = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, threads, smem);
        if (per < 1) fail(NVB_ERR_CUDA, "quadratic H.v kernel does not fit on a multiprocessor");
        long long g = (long long)nsm * per;
        if (g > qp.ntiles) g = qp.ntiles;
        qp.grid[idx] = (int)g;
    }
    kern<<<qp.grid[idx], threads, smem, st>>>(quad_args<T>(qp), x, y, sc, ap);
    return qp.grid[idx];
}

template <typename T, int S>
int launch_qs(QuadPlan &qp, const T *x, T *y, const double *sc, double *ap, cudaStream_t st) {
    const bool n288 = qp.threads == 288;
    switch (qp.nF) {
    case 2: return n288 ? launch_q<T, S, 2, 288>(qp, x, y, sc, ap, st) : launch_q<T, S, 2, 0>(qp, x, y, sc, ap, st);
    case 3: return n288 ? launch_q<T, S, 3, 288>(qp, x, y, sc, ap, st) : launch_q<T, S, 3, 0>(qp, x, y, sc, ap, st);
    case 4: return n288 ? launch_q<T, S, 4, 288>(qp, x, y, sc, ap, st) : launch_q<T, S, 4, 0>(qp, x, y, sc, ap, st);
    default: fail(NVB_ERR_ARG, "quadratic kernel: unsupported number of fast modes");
    }
}

}  // namespace

template <typename T>
int quad_launch(QuadPlan &qp, const T *x, T *y, const double *scale, double *alpha_part, cudaStream_t st) {
    switch (qp.S) {
    case 1: return launch_qs<T, 1>(qp, x, y, scale, alpha_part, st);
    case 2: return launch_qs<T, 2>(qp, x, y, scale, alpha_part, st);
    case 3: return launch_qs<T, 3>(qp, x, y, scale, alpha_part, st);
    case 4: return launch_qs<T, 4>(qp, x, y, scale, alpha_part, st);
    default: fail(NVB_ERR_ARG, "quadratic kernel supports up to 4 states");
    }
}

template int quad_launch<double>(QuadPlan &, const double *, double *, const double *, double *, cudaStream_t);
template int quad_launch<float>(QuadPlan &, const float *, float *, const double *, double *, cudaStream_t);

}  // namespace nvb
