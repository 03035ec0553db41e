// Factorised cubic H.v kernel (see cubic.h for the algebra); included by the per-precision
// instantiation files.
//
// Warp-specialised persistent CTAs walk the tiles with a stride of the grid.  The last warp is
// the producer: it lists each tile's items whose neighbour tile lies inside the basis, one tile
// ahead, and one lane streams them in consumption order into a ring of shared-memory slots with
// TMA bulk copies (full/empty mbarriers, bounded waits, an abort flag and an error word), as in
// the quadratic kernel.  The other warps are the consumers; a thread owns the pencil of mode m.
// Per tile the consumers evaluate every item's coefficient program for the tile's slow digits
// (presence and the record c, e, z_f), compact each target's present items in order, then per
// target state a fold:
//   own x_a:    c x + X_f-coefficients z_f into Z, the fast diagonal (harmonic + x_f^2 zero
//               shift), x_f^2 (+-2), X_f X_g into Z_g, x_f x_g x_h = X_h (X_f X_g), x_f^2 x_h =
//               X_h (x_f^2) into Z_h, x_f^3 directly;
//   own x_b:    c x_b, z_f x_b into Z (constants and linear couplings);
//   +-1 items of fast-quadratic terms (x_s x_f x_g, x_s x_f^2): c, z_f, and e times the tabled
//               fast quadratic (X_f X_g into Z_g, x_f^2 directly);
//   Z items:    c x, z_f x into Z;
//   C items:    c x, two at a time, with y_a += X_f Z_f applied in between (mode m by register
//               shifts, the other fast modes through one shared-memory buffer).
// Fast shifts read the staged tile at row +- strides (a zero halo of 3 strides of the slowest
// fast mode after m; element rows vanish outside the basis); shifts along mode m are register
// moves within the pencil.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>

#include "cubic.h"
#include "ring.h"

namespace nvb {
namespace cubk {

using namespace ring;

template <typename T>
struct CubArgs {
    const T *blk;  // tab | cs
    const T *tcoef;
    const CubTerm *tinfo;
    const int *slow;
    const CubItem *items;
    const int *seg;
    int *err;
    int M, m, nmax, nv, pad, sstate, TF, ntiles, nslot, nitems, nterms;
    int nocopy;      // failure test: the producer issues no copy, so every consumer wait runs out
    int wait_limit;  // polls before a wait gives up
    long long dimen;
    CubFast<T> F;
};

constexpr int R = CUB_RPT;

template <typename T, int S, int NF, int NC, int MAXT, int MINB>
__global__ void __launch_bounds__(MAXT, MINB)
    k_hv_cubic(const CubArgs<T> A, const T *__restrict__ x, T *__restrict__ y, const double *__restrict__ scale_dev,
               double *__restrict__ alpha_part) {
    extern __shared__ __align__(128) unsigned char smem[];
    const int M = A.M, m = A.m, nmax = A.nmax, sst = A.sstate, TF = A.TF, NS = A.nslot, pad = A.pad;
    const int nit = A.nitems;
    const int nterm = A.nterms;
    const CubLayout Lo = cub_layout(M, S, nmax, m, NF, sst, (int)sizeof(T), NS, nit, nterm);
    uint64_t *full = reinterpret_cast<uint64_t *>(smem);
    uint64_t *empty = full + CUB_MAXSLOT;
    volatile int *abort_flag = reinterpret_cast<volatile int *>(smem + 2 * CUB_MAXSLOT * 8);
    T *s_tab = reinterpret_cast<T *>(smem + Lo.tab);
    T *s_cs = reinterpret_cast<T *>(smem + Lo.cs);
    int *s_sl = reinterpret_cast<int *>(smem + Lo.sd);    // slow tile strides [MAXSL], nfunc [MAXSL]
    int *s_dig = reinterpret_cast<int *>(smem + Lo.dig);  // [2][MAXSL] slow digits of a tile
    CubItem *s_it = reinterpret_cast<CubItem *>(smem + Lo.items);
    int *s_seg = reinterpret_cast<int *>(smem + Lo.seg);
    long long *s_pl = reinterpret_cast<long long *>(smem + Lo.plist);
    unsigned char *s_pres = smem + Lo.pres;
    short *s_cl = reinterpret_cast<short *>(smem + Lo.cl);
    int *s_cnt = reinterpret_cast<int *>(smem + Lo.cnt);
    T *s_rec = reinterpret_cast<T *>(smem + Lo.rec);
    T *s_ring = reinterpret_cast<T *>(smem + Lo.ring);  // [NS][sst]
    T *s_z = reinterpret_cast<T *>(smem + Lo.z);        // [sst] Z_f of one fast mode f >= 1
    // at the start of a tile s_z holds the term products [nterm] and their record slots [nterm]
    T *s_prod = s_z;
    signed char *s_pslot = reinterpret_cast<signed char *>(s_z + nterm);
    const int tid = threadIdx.x;
    const int nc = NC > 0 ? NC : (int)blockDim.x - 32;  // consumer threads = shft(m)
    const long long N = A.dimen;
    const CubFast<T> &F = A.F;
    const int *tsh = s_sl, *snf = s_sl + CUB_MAXSL;
    constexpr int NREC = NF + 2;

    {
        const int ntab = M * CUB_ROWS * nmax, ncs = S * m * NF * NF;
        for (int i = tid; i < ntab; i += blockDim.x) s_tab[i] = A.blk[i];
        for (int i = tid; i < ncs; i += blockDim.x) s_cs[i] = A.blk[ntab + i];
        for (int i = tid; i < m; i += blockDim.x) {
            s_sl[i] = A.slow[i];
            s_sl[CUB_MAXSL + i] = A.slow[m + i];
        }
        for (int i = tid; i < nit; i += blockDim.x) s_it[i] = A.items[i];
        for (int i = tid; i <= 4 * S; i += blockDim.x) s_seg[i] = A.seg[i];
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
        // The warp lists each tile's present items one tile ahead (ballot per 32 items, compacted
        // into s_pl[q] for tile parity q: the count, then each item's source offset in x relative
        // to the tile); lane 0 issues the tile's copies in consumption order, each after its slot
        // was released, reading the next offset before it waits (the producer lane is on the
        // critical path).
        const int lane = tid - nc;
        const unsigned bytes = (unsigned)TF * (unsigned)sizeof(T);
        auto list = [&](int tile, int q) {
            long long *pl = s_pl + q * (nit + 1);
            int base = 0;
            for (int i0 = 0; i0 < nit; i0 += 32) {
                const int it = i0 + lane;
                bool ok = false;
                if (it < nit) {
                    const CubItem &ci = s_it[it];
                    ok = true;
                    for (int k = 0; k < ci.nsh; ++k) {
                        const int l = ci.md[k];
                        const int d = (tile / tsh[l]) % snf[l] + ci.sv[k];
                        ok = ok && d >= 0 && d < snf[l];
                    }
                }
                const unsigned bal = __ballot_sync(0xffffffffu, ok);
                if (ok) {
                    const CubItem &ci = s_it[it];
                    pl[1 + base + __popc(bal & ((1u << lane) - 1u))] = (long long)ci.b * N + (long long)ci.tshift * TF;
                }
                base += __popc(bal);
            }
            if (lane == 0) pl[0] = base;
            __syncwarp();
        };
        int slot = 0;
        unsigned ph = 0;
        long long issued = 0;
        int stop = A.nocopy;
        if (blockIdx.x < A.ntiles) list(blockIdx.x, 0);
        int q = 0;
        for (int tile = blockIdx.x; tile < A.ntiles && !stop; tile += gridDim.x, q ^= 1) {
            if (tile + (int)gridDim.x < A.ntiles) list(tile + gridDim.x, q ^ 1);
            const long long *pl = s_pl + q * (nit + 1);
            const int cnt = (int)pl[0];
            if (lane == 0) {
                const T *xt = x + (long long)tile * TF;
                long long nxt = cnt > 0 ? pl[1] : 0;
                for (int i = 0; i < cnt && !stop; ++i) {
                    const long long off = nxt;
                    if (i + 1 < cnt) nxt = pl[2 + i];
                    // a consumer whose wait gave up never releases its slot, so no slot with a
                    // copy in flight is reissued: the producer's wait for it runs out and it stops
                    if (mbar_wait(&empty[slot], ph ^ 1u, abort_flag, A.wait_limit)) {
                        mbar_expect_tx(&full[slot], bytes);
                        bulk_g2s(s_ring + slot * sst + pad, xt + off, bytes, &full[slot]);
                        ++issued;
                    } else {
                        stop = 1;
                    }
                    if (++slot == NS) {
                        slot = 0;
                        ph ^= 1u;
                    }
                }
            }
            stop = __shfl_sync(0xffffffffu, stop, 0);
        }
        if (lane == 0 && stop) {
            // copies still in flight complete on their full barriers: wait for them (bounded)
            const long long n = issued < NS ? issued : NS;
            for (long long i = issued - n; i < issued; ++i) {
                const int s2 = (int)(i % NS);
                const unsigned p = (unsigned)((i / NS) & 1);
                for (int w = 0; w < WAIT_LIMIT && !mbar_try(&full[s2], p); ++w) {
                }
            }
            atomicExch(A.err, 1);
        }
        return;
    }

    // ---------------- consumers ----------------
    int dj[NF];
#pragma unroll
    for (int j = 0; j < NF; ++j) dj[j] = j >= 1 ? (tid / F.sh[j]) % F.nf[j] : 0;
    // element row `row` of fast mode j >= 1 at this thread's digit
    auto tv = [&](int j, int row) -> T { return s_tab[((m + j) * CUB_ROWS + row) * nmax + dj[j]]; };
    const T sc = scale_dev ? (T)(*scale_dev) : (T)1;
    const int nv = A.nv;
    const int lane = tid & 31, wid = tid >> 5, nwarp = nc >> 5;
    constexpr bool kNoBranch = sizeof(T) == 4;  // FP32: fold without testing the wait (results discarded on abort)
    double part = 0.0;
    int slot = 0;
    unsigned ph = 0;
    int tp = 0;
    bool ok = true;
    auto take = [&]() -> const T * {
        ok = mbar_try(&full[slot], ph) || mbar_wait(&full[slot], ph, abort_flag, A.wait_limit);
        return s_ring + slot * sst + pad + tid;
    };
    // only a lane 0 that saw the slot's copy land releases it (a slot whose wait gave up may still
    // be the target of a copy in flight)
    auto release = [&]() {
        __syncwarp();
        if constexpr (kNoBranch) mbar_arrive_if(&empty[slot], lane == 0 && ok);
        else if (lane == 0 && ok) mbar_arrive(&empty[slot]);
        if (++slot == NS) {
            slot = 0;
            ph ^= 1u;
        }
    };
    // X_f of a column at the thread's rows: mode m by register shifts of v, the others from the
    // staged tile p (= slot column of this thread)
    auto Xf = [&](auto fc, const T *v, const T *p, T *out) {
        constexpr int f = decltype(fc)::value;
        if constexpr (f == 0) {
#pragma unroll
            for (int r = 0; r < R; ++r) {
                T s = (T)0;
                if (r + 1 < R) s += F.em[ER_1P][r] * v[r + 1];
                if (r >= 1) s += F.em[ER_1M][r] * v[r - 1];
                out[r] = s;
            }
        } else {
            const T ep = tv(f, ER_1P), em = tv(f, ER_1M);
            const int sh = F.sh[f];
#pragma unroll
            for (int r = 0; r < R; ++r) out[r] = ep * p[r * nc + sh] + em * p[r * nc - sh];
        }
    };
    // x_f^2 of a column (the +-2 part in out, the zero shift separately by the caller)
    auto T2f = [&](auto fc, const T *v, const T *p, T *out) {
        constexpr int f = decltype(fc)::value;
        if constexpr (f == 0) {
#pragma unroll
            for (int r = 0; r < R; ++r) {
                T s = (T)0;
                if (r + 2 < R) s += F.em[ER_2P][r] * v[r + 2];
                if (r >= 2) s += F.em[ER_2M][r] * v[r - 2];
                out[r] = s;
            }
        } else {
            const T ep = tv(f, ER_2P), em = tv(f, ER_2M);
            const int sh = 2 * F.sh[f];
#pragma unroll
            for (int r = 0; r < R; ++r) out[r] = ep * p[r * nc + sh] + em * p[r * nc - sh];
        }
    };
    auto Df = [&](auto fc, int r) -> T {
        constexpr int f = decltype(fc)::value;
        if constexpr (f == 0) return F.em[ER_D2][r];
        else return tv(f, ER_D2);
    };
    for (int tile = blockIdx.x; tile < A.ntiles; tile += gridDim.x, tp ^= 1) {
        if (tid < m) s_dig[tp * CUB_MAXSL + tid] = (tile / tsh[tid]) % snf[tid];
        consumer_sync(nc);
        const int *dig = s_dig + tp * CUB_MAXSL;
        // every term's product for this tile, all terms in parallel (their element factors are
        // table entries at the tile's own digits, valid whether or not the item is present);
        // then every item's presence and record, summing its products in program order
        for (int t = tid; t < nterm; t += nc) {
            const CubTerm ti = A.tinfo[t];
            T v = A.tcoef[t];
            for (int q = 0; q < ti.nf; ++q) v *= s_tab[(ti.md[q] * CUB_ROWS + ti.rw[q]) * nmax + dig[ti.md[q]]];
            s_prod[t] = v;
            s_pslot[t] = ti.slot;
        }
        consumer_sync(nc);
        for (int i = tid; i < nit; i += nc) {
            const CubItem &ci = s_it[i];
            bool pres = true;
            for (int k = 0; k < ci.nsh; ++k) {
                const int d = dig[ci.md[k]] + ci.sv[k];
                pres = pres && d >= 0 && d < snf[ci.md[k]];
            }
            T *rc = s_rec + i * NREC;
#pragma unroll
            for (int q = 0; q < NREC; ++q) rc[q] = (T)0;
            if (pres)
                for (int t = ci.tb; t < ci.te; ++t) rc[s_pslot[t]] += s_prod[t];
            s_pres[i] = pres ? 1 : 0;
        }
        consumer_sync(nc);
        // each target's present Q / Z / C items in order (warp a mod the consumer warps)
        for (int a = wid; a < S; a += nwarp) {
            const int q0 = s_seg[4 * a + 1], z0 = s_seg[4 * a + 2], c0 = s_seg[4 * a + 3], end = s_seg[4 * a + 4];
            int base = 0, nq = 0, nz = 0;
            for (int i0 = q0; i0 < end; i0 += 32) {
                const int i = i0 + lane;
                const bool p = i < end && s_pres[i] != 0;
                const unsigned bal = __ballot_sync(0xffffffffu, p);
                if (p) s_cl[q0 + base + __popc(bal & ((1u << lane) - 1u))] = (short)i;
                base += __popc(bal);
                nq += __popc(__ballot_sync(0xffffffffu, p && i < z0));
                nz += __popc(__ballot_sync(0xffffffffu, p && i >= z0 && i < c0));
            }
            if (lane == 0) {
                s_cnt[a * 4 + 0] = nq;
                s_cnt[a * 4 + 1] = nz;
                s_cnt[a * 4 + 2] = base - nq - nz;
            }
        }
        consumer_sync(nc);
        const long long tbase = (long long)tile * TF;
#pragma unroll
        for (int a = 0; a < S; ++a) {
            T acc[R], Z[NF][R];
#pragma unroll
            for (int r = 0; r < R; ++r) {
                acc[r] = (T)0;
#pragma unroll
                for (int j = 0; j < NF; ++j) Z[j][r] = (T)0;
            }
            // ---- own tile x_a (its column lives only here; the alpha partial re-reads x from L2)
            {
                const T *rc = s_rec + s_seg[4 * a] * NREC;
                const T *buf = take();
                if (kNoBranch || ok) {
                    T xr[R];
#pragma unroll
                    for (int r = 0; r < R; ++r) xr[r] = buf[r * nc];
                    T dfast = (T)0;
#pragma unroll
                    for (int j = 1; j < NF; ++j) dfast += (F.om[j] + F.R2[j][a]) * tv(j, ER_D2);
                    const T c0 = rc[0] + dfast, d0 = F.om[0] + F.R2[0][a];
#pragma unroll
                    for (int r = 0; r < R; ++r) acc[r] += (c0 + d0 * F.em[ER_D2][r]) * xr[r];
#pragma unroll
                    for (int f = 0; f < NF; ++f) {
                        const T zf = rc[2 + f];
#pragma unroll
                        for (int r = 0; r < R; ++r) Z[f][r] += zf * xr[r];
                    }
                    auto per_mode = [&](auto fc) {
                        constexpr int f = decltype(fc)::value;
                        // X_f x: X_g X_f into Z_g (g > f); for f >= 1 also X_m X_f into Z_h via C3[0][f][h]
                        bool needV = false;
#pragma unroll
                        for (int g = f + 1; g < NF; ++g) needV |= F.Q2[f][g][a] != (T)0;
                        if constexpr (f >= 1) {
#pragma unroll
                            for (int h = f + 1; h < NF; ++h) needV |= F.C3[0][f][h][a] != (T)0;
                        }
                        if (needV) {
                            T V[R];
                            Xf(fc, xr, buf, V);
#pragma unroll
                            for (int g = f + 1; g < NF; ++g) {
                                const T q = F.Q2[f][g][a];
                                if (q != (T)0) {
#pragma unroll
                                    for (int r = 0; r < R; ++r) Z[g][r] += q * V[r];
                                }
                            }
                            if constexpr (f >= 1) {
                                bool anyP = false;
#pragma unroll
                                for (int h = f + 1; h < NF; ++h) anyP |= F.C3[0][f][h][a] != (T)0;
                                if (anyP) {
                                    T P[R];
                                    Xf(std::integral_constant<int, 0>{}, V, nullptr, P);
#pragma unroll
                                    for (int h = f + 1; h < NF; ++h) {
                                        const T c = F.C3[0][f][h][a];
                                        if (c != (T)0) {
#pragma unroll
                                            for (int r = 0; r < R; ++r) Z[h][r] += c * P[r];
                                        }
                                    }
                                }
                            }
                        }
                        // x_f^2 x: the +-2 part of the square term, and x_f^2 x_h = X_h (x_f^2 x) into Z_h
                        bool needS = F.R2[f][a] != (T)0;
#pragma unroll
                        for (int h = 0; h < NF; ++h)
                            if (h != f) needS |= (h > f ? F.C3[f][f][h][a] : F.C3[h][f][f][a]) != (T)0;
                        if (needS) {
                            T Tt[R];
                            T2f(fc, xr, buf, Tt);
                            const T r2 = F.R2[f][a];
                            if (r2 != (T)0) {
#pragma unroll
                                for (int r = 0; r < R; ++r) acc[r] += r2 * Tt[r];
                            }
#pragma unroll
                            for (int h = 0; h < NF; ++h) {
                                if (h == f) continue;
                                const T c = h > f ? F.C3[f][f][h][a] : F.C3[h][f][f][a];
                                if (c != (T)0) {
#pragma unroll
                                    for (int r = 0; r < R; ++r) Z[h][r] += c * (Tt[r] + Df(fc, r) * xr[r]);
                                }
                            }
                        }
                        // x_f^3
                        const T c3 = F.C3[f][f][f][a];
                        if (c3 != (T)0) {
                            if constexpr (f == 0) {
#pragma unroll
                                for (int r = 0; r < R; ++r) {
                                    T s = (T)0;
                                    if (r + 3 < R) s += F.em[ER_3P3][r] * xr[r + 3];
                                    if (r >= 3) s += F.em[ER_3M3][r] * xr[r - 3];
                                    if (r + 1 < R) s += F.em[ER_3P1][r] * xr[r + 1];
                                    if (r >= 1) s += F.em[ER_3M1][r] * xr[r - 1];
                                    acc[r] += c3 * s;
                                }
                            } else {
                                const T p3 = tv(f, ER_3P3), m3 = tv(f, ER_3M3), p1 = tv(f, ER_3P1), m1 = tv(f, ER_3M1);
                                const int sh = F.sh[f];
#pragma unroll
                                for (int r = 0; r < R; ++r) {
                                    const T *p = buf + r * nc;
                                    acc[r] += c3 * (p3 * p[3 * sh] + m3 * p[-3 * sh] + p1 * p[sh] + m1 * p[-sh]);
                                }
                            }
                        }
                    };
                    per_mode(std::integral_constant<int, 0>{});
                    if constexpr (NF > 1) per_mode(std::integral_constant<int, 1>{});
                    if constexpr (NF > 2) per_mode(std::integral_constant<int, 2>{});
                    if constexpr (NF > 3) per_mode(std::integral_constant<int, 3>{});
                    if constexpr (NF > 4) per_mode(std::integral_constant<int, 4>{});
                    // x_f x_g x_h = X_h (X_f X_g x) over fast modes 1 <= f < g < h
#pragma unroll
                    for (int f = 1; f < NF; ++f)
#pragma unroll
                        for (int g = f + 1; g < NF; ++g) {
                            bool any = false;
#pragma unroll
                            for (int h = g + 1; h < NF; ++h) any |= F.C3[f][g][h][a] != (T)0;
                            if (!any) continue;
                            const T fp = tv(f, ER_1P), fm = tv(f, ER_1M), gp = tv(g, ER_1P), gm = tv(g, ER_1M);
                            const T pp = fp * gp, pm = fp * gm, mp = fm * gp, mm = fm * gm;
                            const int sf = F.sh[f], sg = F.sh[g];
                            T P[R];
#pragma unroll
                            for (int r = 0; r < R; ++r) {
                                const T *p = buf + r * nc;
                                P[r] = pp * p[sf + sg] + pm * p[sf - sg] + mp * p[sg - sf] + mm * p[-sf - sg];
                            }
#pragma unroll
                            for (int h = g + 1; h < NF; ++h) {
                                const T c = F.C3[f][g][h][a];
                                if (c != (T)0) {
#pragma unroll
                                    for (int r = 0; r < R; ++r) Z[h][r] += c * P[r];
                                }
                            }
                        }
                }
                release();
            }
            // ---- the other states' own tiles: constants and linear couplings
            const int qbase = s_seg[4 * a + 1];
            for (int i = s_seg[4 * a] + 1; i < qbase; ++i) {
                const T *rc = s_rec + i * NREC;
                const T *buf = take();
                if (kNoBranch || ok) {
                    T v[R];
#pragma unroll
                    for (int r = 0; r < R; ++r) v[r] = buf[r * nc];
                    const T c = rc[0];
#pragma unroll
                    for (int r = 0; r < R; ++r) acc[r] += c * v[r];
#pragma unroll
                    for (int f = 0; f < NF; ++f) {
                        const T zf = rc[2 + f];
#pragma unroll
                        for (int r = 0; r < R; ++r) Z[f][r] += zf * v[r];
                    }
                }
                release();
            }
            const int nq = s_cnt[a * 4 + 0], nz = s_cnt[a * 4 + 1], ncc = s_cnt[a * 4 + 2];
            // ---- +-1 items of the fast-quadratic terms x_s x_f x_g, x_s x_f^2
            for (int k = 0; k < nq; ++k) {
                const int idx = s_cl[qbase + k];
                const T *rc = s_rec + idx * NREC;
                const T *cs = s_cs + (a * m + s_it[idx].qs) * NF * NF;
                const T *buf = take();
                if (kNoBranch || ok) {
                    T v[R];
#pragma unroll
                    for (int r = 0; r < R; ++r) v[r] = buf[r * nc];
                    const T c = rc[0], e = rc[1];
#pragma unroll
                    for (int r = 0; r < R; ++r) acc[r] += c * v[r];
#pragma unroll
                    for (int f = 0; f < NF; ++f) {
                        const T zf = rc[2 + f];
#pragma unroll
                        for (int r = 0; r < R; ++r) Z[f][r] += zf * v[r];
                    }
                    T dq = (T)0;  // sum over f >= 1 of e cs_ff <n_f|x_f^2|n_f> (the zero shift of x_f^2)
                    auto per_mode = [&](auto fc) {
                        constexpr int f = decltype(fc)::value;
                        bool any = false;
#pragma unroll
                        for (int g = f + 1; g < NF; ++g) any |= cs[f * NF + g] != (T)0;
                        if (any) {
                            T V[R];
                            Xf(fc, v, buf, V);
#pragma unroll
                            for (int g = f + 1; g < NF; ++g) {
                                const T q = e * cs[f * NF + g];
#pragma unroll
                                for (int r = 0; r < R; ++r) Z[g][r] += q * V[r];
                            }
                        }
                        const T cff = cs[f * NF + f];
                        if (cff != (T)0) {
                            T Tt[R];
                            T2f(fc, v, buf, Tt);
                            const T q = e * cff;
                            if constexpr (f == 0) {
#pragma unroll
                                for (int r = 0; r < R; ++r) acc[r] += q * (Tt[r] + F.em[ER_D2][r] * v[r]);
                            } else {
#pragma unroll
                                for (int r = 0; r < R; ++r) acc[r] += q * Tt[r];
                                dq += q * tv(f, ER_D2);
                            }
                        }
                    };
                    per_mode(std::integral_constant<int, 0>{});
                    if constexpr (NF > 1) per_mode(std::integral_constant<int, 1>{});
                    if constexpr (NF > 2) per_mode(std::integral_constant<int, 2>{});
                    if constexpr (NF > 3) per_mode(std::integral_constant<int, 3>{});
                    if constexpr (NF > 4) per_mode(std::integral_constant<int, 4>{});
#pragma unroll
                    for (int r = 0; r < R; ++r) acc[r] += dq * v[r];
                }
                release();
            }
            // ---- items with fast linear parts
            for (int k = 0; k < nz; ++k) {
                const T *rc = s_rec + s_cl[qbase + nq + k] * NREC;
                const T *buf = take();
                if (kNoBranch || ok) {
                    T v[R];
#pragma unroll
                    for (int r = 0; r < R; ++r) v[r] = buf[r * nc];
                    const T c = rc[0];
#pragma unroll
                    for (int r = 0; r < R; ++r) acc[r] += c * v[r];
#pragma unroll
                    for (int f = 0; f < NF; ++f) {
                        const T zf = rc[2 + f];
#pragma unroll
                        for (int r = 0; r < R; ++r) Z[f][r] += zf * v[r];
                    }
                }
                release();
            }
            // ---- Z is final: mode m by register shifts now, the other fast modes in between the
            // coefficient-only items (each through s_z between two consumer barriers)
            {
                T P[R];
                Xf(std::integral_constant<int, 0>{}, Z[0], nullptr, P);
#pragma unroll
                for (int r = 0; r < R; ++r) acc[r] += P[r];
            }
            auto xz = [&](auto jc) {
                constexpr int jj = decltype(jc)::value;
#pragma unroll
                for (int r = 0; r < R; ++r) s_z[pad + r * nc + tid] = r < nv ? Z[jj][r] : (T)0;
                consumer_sync(nc);
                const T ep = tv(jj, ER_1P), em = tv(jj, ER_1M);
                const int sh = F.sh[jj];
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const T *p = s_z + pad + r * nc + tid;
                    acc[r] += ep * p[sh] + em * p[-sh];
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
                if constexpr (NF > 4) {
                    if (done == 4) xz(std::integral_constant<int, 4>{});
                }
                ++done;
            };
            // ---- coefficient-only items, two at a time
            {
                const short *cl = s_cl + qbase + nq + nz;
                int j = 0;
                for (; j + 1 < ncc; j += 2) {
                    if (done < NF && j * NF >= done * ncc) xz_next();
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
                        const T c0 = s_rec[cl[j] * NREC], c1 = s_rec[cl[j + 1] * NREC];
#pragma unroll
                        for (int r = 0; r < R; ++r) acc[r] = fma(c1, v1[r], fma(c0, v0[r], acc[r]));
                    }
                    __syncwarp();
                    if constexpr (kNoBranch) mbar_arrive_if(&empty[s0], lane == 0 && ok0);
                    else if (lane == 0 && ok0) mbar_arrive(&empty[s0]);
                    release();
                }
                if (j < ncc) {
                    const T *buf = take();
                    if (kNoBranch || ok) {
                        const T c = s_rec[cl[j] * NREC];
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
                    const long long o = a * N + tbase + r * nc + tid;
                    const T v = acc[r] * sc;
                    y[o] = v;
                    if (alpha_part) part += ((double)x[o] * (double)sc) * (double)v;
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
CubArgs<T> cub_args(const CubPlan &cp) {
    CubArgs<T> a{};
    a.tinfo = cp.d_tinfo;
    a.slow = cp.d_slow;
    a.items = cp.d_items;
    a.seg = cp.d_seg;
    a.err = cp.d_err;
    a.nocopy = cp.test_nocopy;
    a.wait_limit = cp.test_nocopy ? (1 << 14) : WAIT_LIMIT;
    a.M = cp.M;
    a.m = cp.m;
    a.nmax = cp.nmax;
    a.nv = cp.nv;
    a.pad = cp.pad;
    a.sstate = cp.sstate;
    a.TF = cp.TF;
    a.ntiles = cp.ntiles;
    a.nitems = (int)cp.items.size();
    a.nterms = (int)cp.tinfo.size();
    a.dimen = cp.dimen;
    if constexpr (sizeof(T) == 8) {
        a.blk = (const T *)cp.d_blk;
        a.tcoef = (const T *)cp.d_tcoef;
        a.F = cp.fast_d;
        a.nslot = cp.nslot[0];
    } else {
        a.blk = (const T *)cp.d_blk_f;
        a.tcoef = (const T *)cp.d_tcoef_f;
        a.F = cp.fast_f;
        a.nslot = cp.nslot[1];
    }
    return a;
}

template <typename T, int S, int NF, int NC, int MAXT, int MINB>
int launch_c(CubPlan &cp, const T *x, T *y, const double *sc, double *ap, cudaStream_t st) {
    const int idx = sizeof(T) == 8 ? 0 : 1;
    const size_t smem = cp.smem[idx];
    const int threads = cp.threads + 32;
    auto kern = k_hv_cubic<T, S, NF, NC, MAXT, MINB>;
    if (cp.grid[idx] == 0) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        int dev = 0, nsm = 0, per = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, threads, smem);
        if (per < 1) fail(NVB_ERR_CUDA, "cubic H.v kernel does not fit on a multiprocessor");
        long long g = (long long)nsm * per;
        if (g > cp.ntiles) g = cp.ntiles;
        cp.grid[idx] = (int)g;
    }
    kern<<<cp.grid[idx], threads, smem, st>>>(cub_args<T>(cp), x, y, sc, ap);
    return cp.grid[idx];
}

// the launch of one precision and launch shape over the supported (states, fast modes)
template <typename T, int NC, int MAXT, int MINB>
int launch_shape(CubPlan &cp, const T *x, T *y, const double *sc, double *ap, cudaStream_t st) {
#define NVB_CUB_NF(S_)                                                                      \
    switch (cp.nF) {                                                                        \
    case 2: return launch_c<T, S_, 2, NC, MAXT, MINB>(cp, x, y, sc, ap, st);                \
    case 3: return launch_c<T, S_, 3, NC, MAXT, MINB>(cp, x, y, sc, ap, st);                \
    case 4: return launch_c<T, S_, 4, NC, MAXT, MINB>(cp, x, y, sc, ap, st);                \
    case 5: return launch_c<T, S_, 5, NC, MAXT, MINB>(cp, x, y, sc, ap, st);                \
    default: fail(NVB_ERR_ARG, "cubic kernel: unsupported number of fast modes");           \
    }
    switch (cp.S) {
    case 1: NVB_CUB_NF(1)
    case 2: NVB_CUB_NF(2)
    case 3: NVB_CUB_NF(3)
    case 4: NVB_CUB_NF(4)
    default: fail(NVB_ERR_ARG, "cubic kernel supports up to 4 states");
    }
#undef NVB_CUB_NF
    return 0;
}

}  // namespace cubk
}  // namespace nvb
