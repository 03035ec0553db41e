// Host planner for the slab-tiled H.v kernel (see slab.h).
#include <algorithm>
#include <cmath>
#include <map>

#include "slab.h"

namespace nvb {

static int smax_of(int p, int64_t nf) {
    int s = p;
    while (s > nf - 1) s -= 2;  // Source/secondary.f90:33-37
    return s;
}

static int slab_max_threads(int eb) { return eb == 8 ? 384 : 512; }  // matches the kernel's launch bounds

static int slab_threads(long long TF) {
    long long t = (TF + SLAB_RPT - 1) / SLAB_RPT;
    t = (t + 31) / 32 * 32;
    return (int)t;
}

size_t slab_smem(const SlabPlan &sp, const Plan &pl, int eb) {
    return slab_layout((long long)sp.ftab.size(), (long long)pl.h_etab.size(), (long long)sp.steps.size(),
                       (long long)(sp.groups.size() - sp.nstaged), pl.S, sp.m, sp.sstate, eb)
        .total;
}

bool slab_build(SlabPlan &sp, const Plan &pl, const System &sys, int quirk_cubic, int eb) {
    sp = SlabPlan{};
    const int S = sys.S, M = sys.M;
    if (S > 4) return false;
    // Choose the tile: the largest suffix of modes (fast modes) whose double-buffered tile
    // plus halo fits 220 KB of shared memory, that needs <= 1024 threads, and that leaves at
    // least two tiles per SM.
    const size_t smem_cap = 220 * 1024;
    int best_m = -1;
    for (int m = M - 1; m >= 1; --m) {
        long long TF = 1;
        for (int k = m; k < M; ++k) TF *= sys.nfunc[k];
        const int nF = M - m;
        if (nF > SLAB_MAXF || m > SLAB_MAXSL) break;
        if (slab_threads(TF) > slab_max_threads(eb)) break;
        const long long pad_est = std::min<long long>(TF, (long long)sys.ordr * sys.shft[m]);
        const size_t need = (size_t)(TF + 2 * pad_est) * S * eb * SLAB_NBUF + 16 * 1024;
        if (need > smem_cap) break;
        if (sys.dimen / TF < 2 * 148) break;
        if (TF % 4 == 0) best_m = m;
    }
    if (best_m < 1) return false;
    const int m = best_m;
    sp.m = m;
    sp.nF = M - m;
    sp.TF = 1;
    for (int k = m; k < M; ++k) sp.TF *= sys.nfunc[k];
    sp.ntiles = sys.dimen / sp.TF;
    if (sp.TF < 64) return false;                             // too little work per CTA
    if (sp.TF % 4 != 0 || sys.dimen % 4 != 0) return false;  // 16-byte TMA alignment
    sp.threads = slab_threads(sp.TF);
    {
        const long long sm = sys.shft[m];  // rows per value of the slowest fast mode
        if (sm % 32 == 0 && sm <= slab_max_threads(eb) && sys.nfunc[m] <= SLAB_RPT) {
            sp.threads = (int)sm;
            sp.cols = 1;
        }
    }
    sp.frow_len = std::max(pl.nmax, SLAB_RPT);
    for (int l = 0; l < m; ++l) {
        sp.slow_tshft.push_back(sys.shft[l] / sp.TF);
        sp.slow_nfunc.push_back((int)sys.nfunc[l]);
        sp.slow_omega.push_back(sys.omega[l]);
    }
    for (int k = m; k < M; ++k) {
        sp.fast_nfunc.push_back((int)sys.nfunc[k]);
        sp.fast_shft.push_back(sys.shft[k]);
        sp.fast_omega.push_back(sys.omega[k]);
    }
    // fast element table rows, keyed by (fast field, power, shift)
    std::map<std::tuple<int, int, int>, int> frow;
    auto fast_row = [&](int j, int p, int s) {
        auto key = std::make_tuple(j, p, s);
        auto it = frow.find(key);
        if (it != frow.end()) return it->second;
        const int r = (int)frow.size() * sp.frow_len;  // element offset of the row
        frow[key] = r;
        const int nf = sp.fast_nfunc[j];
        for (int n = 0; n < sp.frow_len; ++n) {
            double v = 0.0;
            if (n < nf && n + s >= 0 && n + s < nf) {
                const int lo = std::min(n, n + s);
                v = hoelem(p, lo + 1, lo + 1 + std::abs(s), quirk_cubic);
            }
            sp.ftab.push_back(v);
        }
        return r;
    };
    auto etab_row = [&](int p, int j) { return ((p - 1) * ETAB_J + j) * pl.nmax; };
    std::map<std::vector<int>, int> gidx;
    std::vector<std::vector<SlabStep>> gsteps;
    std::vector<unsigned> gmask;
    std::vector<std::vector<int>> gkeys;
    auto group_of = [&](const std::vector<int> &key) {
        auto it = gidx.find(key);
        if (it != gidx.end()) return it->second;
        const int g = (int)gsteps.size();
        gidx[key] = g;
        gsteps.emplace_back();
        gmask.push_back(0u);
        gkeys.push_back(key);
        return g;
    };
    group_of(std::vector<int>(m, 0));  // own tile first
    const int nt = (int)sys.terms.size();
    for (int t = 0; t < nt; ++t) {
        const Term &T = sys.terms[t];
        unsigned cols = 0;
        for (auto &pr : T.pairs) cols |= 1u << pr.b;
        int sm[MAX_ORDER], sd[MAX_ORDER];
        bool bad = false, diag = true;
        long long nsteps = 1;
        for (int l = 0; l < T.nm; ++l) {
            sm[l] = smax_of(T.pow[l], sys.nfunc[T.mode[l]]);
            if (sm[l] < 0) bad = true;
            if (sm[l] % 2 != 0) diag = false;
            nsteps *= sm[l] + 1;
            sd[l] = -sm[l];
        }
        if (bad) continue;
        if (diag) {
            SlabDiag dg{};
            dg.term = t;
            for (int l = 0; l < T.nm; ++l) {
                if (T.mode[l] < m) {
                    dg.slow_mode[dg.nslow] = (short)T.mode[l];
                    dg.slow_etab[dg.nslow] = etab_row(T.pow[l], 0);
                    dg.nslow++;
                } else {
                    const int j = T.mode[l] - m;
                    dg.fast_field[dg.nfast] = (short)j;
                    dg.fast_row[dg.nfast] = fast_row(j, T.pow[l], 0);
                    dg.nfast++;
                }
            }
            sp.diag.push_back(dg);
        }
        sd[T.nm - 1] -= 2;
        for (long long k = 0; k < nsteps; ++k) {
            int l = T.nm - 1;
            while (sd[l] >= sm[l]) { sd[l] = -sm[l]; --l; }
            sd[l] += 2;
            bool zero = true;
            for (int q = 0; q < T.nm; ++q) zero &= sd[q] == 0;
            if (zero) continue;
            std::vector<int> key(m, 0);
            SlabStep st{};
            st.term = t;
            long long stride = 0;
            for (int q = 0; q < T.nm; ++q) {
                const int md = T.mode[q];
                if (md < m) {
                    key[md] = sd[q];
                    st.slow_mode[st.nslow] = (short)md;
                    st.slow_sig[st.nslow] = (short)sd[q];
                    st.slow_etab[st.nslow] = etab_row(T.pow[q], std::abs(sd[q]));
                    st.nslow++;
                } else {
                    const int j = md - m;
                    st.fast_field[st.nfast] = (short)j;
                    st.fast_row[st.nfast] = fast_row(j, T.pow[q], sd[q]);
                    st.nfast++;
                    stride += (long long)sd[q] * sys.shft[md];
                }
            }
            st.stride = (int)stride;
            sp.pad = std::max<int>(sp.pad, (int)std::llabs(stride));
            const int g = group_of(key);
            gsteps[g].push_back(st);
            gmask[g] |= cols;
        }
    }
    sp.pad = (sp.pad + 3) / 4 * 4;
    // rows RPT*threads-1 >= TF read zeros from a tail after the halo
    sp.sstate = sp.pad + sp.TF + sp.pad + ((long long)SLAB_RPT * sp.threads - sp.TF);
    gmask[0] = (1u << S) - 1;  // the own tile feeds the diagonal part of every state
    std::vector<size_t> order;
    for (int pass = 0; pass < 2; ++pass)
        for (size_t g = 0; g < gsteps.size(); ++g) {
            bool direct = g != 0;
            for (auto &st : gsteps[g]) direct &= st.nfast == 0;
            if ((pass == 0) != direct) order.push_back(g);
        }
    for (size_t g : order) {
        SlabGroup G{};
        G.direct = 0;
        if (g != 0) {
            G.direct = 1;
            for (auto &st : gsteps[g]) G.direct &= st.nfast == 0 ? 1 : 0;
        }
        if (!G.direct) sp.nstaged++;
        long long ts = 0;
        for (int l = 0; l < m; ++l) {
            G.sig[l] = (short)gkeys[g][l];
            ts += (long long)gkeys[g][l] * sp.slow_tshft[l];
        }
        G.tile_shift = ts;
        G.step_begin = (int)sp.steps.size();
        sp.steps.insert(sp.steps.end(), gsteps[g].begin(), gsteps[g].end());
        G.step_end = (int)sp.steps.size();
        G.state_mask = gmask[g];
        sp.groups.push_back(G);
    }
    sp.nfrows = (int)frow.size();
    if (sp.ftab.empty()) sp.ftab.assign(sp.frow_len, 0.0);
    if (sp.ftab.size() > 65535) return false;  // fast row offsets are packed in 16 bits
    // per-step constants: word = nfast (3 bits) | fast fields (4 x 2 bits) << 3 | column mask
    // (4) << 11 | pair mask (16) << 15, and the term's coupling block on its state pairs
    sp.info.resize(sp.steps.size());
    sp.scoef.assign(sp.steps.size() * (size_t)S * S, 0.0);
    for (size_t i = 0; i < sp.steps.size(); ++i) {
        const SlabStep &st = sp.steps[i];
        const unsigned pm = (unsigned)(pl.h_mask[2 * (size_t)st.term] & 0xFFFFull);
        unsigned cols = 0;
        for (int ab = 0; ab < S * S; ++ab)
            if ((pm >> ab) & 1u) {
                cols |= 1u << (ab % S);
                sp.scoef[i * S * S + ab] = pl.h_coef[(size_t)st.term * S * S + ab];
            }
        unsigned w = (unsigned)st.nfast | (cols << 11) | (pm << 15);
        int fr[4] = {0, 0, 0, 0};
        for (int q = 0; q < st.nfast; ++q) {
            w |= (unsigned)st.fast_field[q] << (3 + 2 * q);
            fr[q] = st.fast_row[q];
        }
        sp.info[i] = make_int4(st.stride, (int)w, fr[0] | (fr[1] << 16), fr[2] | (fr[3] << 16));
    }
    sp.smem_bytes[0] = slab_smem(sp, pl, 8);
    sp.smem_bytes[1] = slab_smem(sp, pl, 4);
    if (sp.smem_bytes[eb == 8 ? 0 : 1] > 227 * 1024) return false;
    sp.ok = true;
    return true;
}

#define CK(x)                                                                                    \
    do {                                                                                         \
        cudaError_t e_ = (x);                                                                    \
        if (e_ != cudaSuccess) fail(NVB_ERR_CUDA, std::string(#x ": ") + cudaGetErrorString(e_)); \
    } while (0)

template <typename T>
static void up(T *&d, const std::vector<T> &h) {
    size_t n = std::max<size_t>(h.size(), 1);
    CK(cudaMalloc((void **)&d, n * sizeof(T)));
    if (!h.empty()) CK(cudaMemcpy(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
}

void slab_upload(SlabPlan &sp) {
    if (!sp.ok) return;
    up(sp.d_steps, sp.steps);
    up(sp.d_groups, sp.groups);
    up(sp.d_diag, sp.diag);
    up(sp.d_ftab, sp.ftab);
    up(sp.d_ftab_f, std::vector<float>(sp.ftab.begin(), sp.ftab.end()));
    up(sp.d_slow_tshft, sp.slow_tshft);
    up(sp.d_slow_nfunc, sp.slow_nfunc);
    up(sp.d_slow_omega, sp.slow_omega);
    up(sp.d_slow_omega_f, std::vector<float>(sp.slow_omega.begin(), sp.slow_omega.end()));
    up(sp.d_fast_nfunc, sp.fast_nfunc);
    up(sp.d_fast_shft, sp.fast_shft);
    up(sp.d_fast_omega, sp.fast_omega);
    up(sp.d_fast_omega_f, std::vector<float>(sp.fast_omega.begin(), sp.fast_omega.end()));
    up(sp.d_info, sp.info);
    up(sp.d_scoef, sp.scoef);
    up(sp.d_scoef_f, std::vector<float>(sp.scoef.begin(), sp.scoef.end()));
    CK(cudaMalloc((void **)&sp.d_err, sizeof(int)));
    CK(cudaMemset(sp.d_err, 0, sizeof(int)));
}

void slab_free(SlabPlan &sp) {
    void *ps[] = {sp.d_steps, sp.d_groups, sp.d_diag, sp.d_ftab, sp.d_ftab_f, sp.d_slow_tshft, sp.d_slow_nfunc,
                  sp.d_slow_omega, sp.d_slow_omega_f, sp.d_fast_nfunc, sp.d_fast_shft, sp.d_fast_omega,
                  sp.d_fast_omega_f, sp.d_err, sp.d_info, sp.d_scoef, sp.d_scoef_f};
    for (void *p : ps)
        if (p) cudaFree(p);
    sp.d_steps = nullptr; sp.d_groups = nullptr; sp.d_diag = nullptr; sp.d_ftab = nullptr; sp.d_ftab_f = nullptr;
    sp.d_slow_tshft = nullptr; sp.d_slow_nfunc = nullptr; sp.d_slow_omega = nullptr; sp.d_slow_omega_f = nullptr;
    sp.d_fast_nfunc = nullptr; sp.d_fast_shft = nullptr; sp.d_fast_omega = nullptr; sp.d_fast_omega_f = nullptr;
    sp.d_err = nullptr;
    sp.d_info = nullptr; sp.d_scoef = nullptr; sp.d_scoef_f = nullptr;
}

}  // namespace nvb
