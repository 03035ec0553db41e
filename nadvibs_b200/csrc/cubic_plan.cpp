// Host planner of the factorised cubic H.v kernel (see cubic.h).
#include <algorithm>
#include <array>
#include <cmath>
#include <map>
#include <string>
#include <type_traits>

#include "cubic.h"

namespace nvb {

namespace {

// Shift range of x^p on a mode with nf functions (Source/secondary.f90:33-37): -1 = no element.
int smax_of(int p, long long nf) {
    int s = p;
    while (s > nf - 1) s -= 2;
    return s;
}

// element row of x^p at shift s
int row_of(int p, int s) {
    if (p == 1) return s > 0 ? ER_1P : ER_1M;
    if (p == 2) return s > 0 ? ER_2P : (s < 0 ? ER_2M : ER_D2);
    // p == 3
    if (s == 3) return ER_3P3;
    if (s == -3) return ER_3M3;
    return s > 0 ? ER_3P1 : ER_3M1;
}

struct Build {
    int kind = CK_C;  // CK_OWN for sigma = 0
    int qs = -1;
    std::vector<CubTerm> info;
    std::vector<double> coef;
};

}  // namespace

bool cubic_build(CubPlan &cp, const Plan &pl, const System &sys, int quirk_cubic) {
    cp = CubPlan{};
    const int S = sys.S, M = sys.M;
    if (S > CUB_MAXS || sys.ordr > 3 || M < 3) return false;
    for (const Term &t : sys.terms) {
        int order = 0;
        for (int l = 0; l < t.nm; ++l) order += t.pow[l];
        if (order > 3) return false;
        for (auto &pr : t.pairs)
            if (pr.a != pr.b && order != 1) return false;  // couplings between states: linear only
    }
    // tile: the slowest mode m whose pencil stride is a multiple of 32 threads (64..576) with <= 8
    // rows, at most CUB_MAXF fast modes and at least one slow mode
    int best = -1;
    for (int m = M - 1; m >= 1; --m) {
        const long long th = sys.shft[m];
        if (th > 576) break;
        if (M - m > CUB_MAXF) break;
        if (m > CUB_MAXSL) continue;
        if (th % 32 == 0 && th >= 64 && sys.nfunc[m] <= CUB_RPT && M - m >= 2) best = m;
    }
    if (best < 1) return false;
    const int m = best, NF = M - m;
    cp.S = S;
    cp.M = M;
    cp.m = m;
    cp.nF = NF;
    cp.nmax = pl.nmax;
    cp.threads = (int)sys.shft[m];
    cp.nv = (int)sys.nfunc[m];
    cp.TF = cp.threads * cp.nv;
    if (sys.dimen / cp.TF > (1LL << 30)) return false;
    cp.ntiles = (int)(sys.dimen / cp.TF);
    cp.dimen = sys.dimen;
    // halo: fast shifts up to +-3 strides of the slowest fast mode after m
    long long pad = 0;
    for (int k = m + 1; k < M; ++k) pad = std::max<long long>(pad, 3 * sys.shft[k]);
    cp.pad = (int)((pad + 3) / 4 * 4);
    cp.sstate = cp.pad + cp.threads * CUB_RPT + cp.pad;
    for (int l = 0; l < m; ++l) {
        cp.slow_tshft.push_back((int)(sys.shft[l] / cp.TF));
        cp.slow_nfunc.push_back((int)sys.nfunc[l]);
    }
    // element rows, zero where the partner function is outside the basis
    const int nmax = pl.nmax;
    cp.tab.assign((size_t)M * CUB_ROWS * nmax, 0.0);
    for (int j = 0; j < M; ++j) {
        const int nf = (int)sys.nfunc[j];
        double *t = cp.tab.data() + (size_t)j * CUB_ROWS * nmax;
        for (int n = 0; n < nf; ++n) {
            if (n + 1 < nf) t[ER_1P * nmax + n] = hoelem(1, n + 1, n + 2, quirk_cubic);
            if (n >= 1) t[ER_1M * nmax + n] = hoelem(1, n, n + 1, quirk_cubic);
            if (n + 2 < nf) t[ER_2P * nmax + n] = hoelem(2, n + 1, n + 3, quirk_cubic);
            if (n >= 2) t[ER_2M * nmax + n] = hoelem(2, n - 1, n + 1, quirk_cubic);
            t[ER_D2 * nmax + n] = hoelem(2, n + 1, n + 1, quirk_cubic);
            if (n + 3 < nf) t[ER_3P3 * nmax + n] = hoelem(3, n + 1, n + 4, quirk_cubic);
            if (n >= 3) t[ER_3M3 * nmax + n] = hoelem(3, n - 2, n + 1, quirk_cubic);
            if (n + 1 < nf) t[ER_3P1 * nmax + n] = hoelem(3, n + 1, n + 2, quirk_cubic);
            if (n >= 1) t[ER_3M1 * nmax + n] = hoelem(3, n, n + 1, quirk_cubic);
        }
    }
    // x^2 with nf < 3 and x^3 with nf < 4 keep only the shifts the reference applies (rows of the
    // dropped shifts are already zero: their partners are outside the basis)
    CubFast<double> &F = cp.fast_d;
    F = CubFast<double>{};
    for (int j = 0; j < NF; ++j) {
        F.sh[j] = (int)sys.shft[m + j];
        F.nf[j] = (int)sys.nfunc[m + j];
        F.om[j] = sys.omega[m + j];
    }
    for (int q = 0; q < CUB_ROWS; ++q)
        for (int r = 0; r < CUB_RPT; ++r) F.em[q][r] = r < nmax ? cp.tab[((size_t)m * CUB_ROWS + q) * nmax + r] : 0.0;
    cp.cs.assign((size_t)S * m * NF * NF, 0.0);

    // items keyed by (target a, source b, slow shift vector)
    using Key = std::array<int, 2 + CUB_MAXSL>;
    std::map<Key, Build> byk;
    auto key_of = [&](int a, int b, const int *sig) {
        Key k{};
        k[0] = a;
        k[1] = b;
        for (int l = 0; l < m; ++l) k[2 + l] = sig[l];
        return k;
    };
    auto add_term = [&](int a, int b, const int *sig, int slot, double coef, int nfac, const int *fm, const int *fr) {
        Build &B = byk[key_of(a, b, sig)];
        CubTerm t{};
        t.slot = (signed char)slot;
        t.nf = (signed char)nfac;
        for (int q = 0; q < nfac; ++q) {
            t.md[q] = (signed char)fm[q];
            t.rw[q] = (signed char)fr[q];
        }
        B.info.push_back(t);
        B.coef.push_back(coef);
    };
    int zero[CUB_MAXSL] = {0};
    // own tiles of every target exist; harmonic energy of the slow modes and the constants
    for (int a = 0; a < S; ++a) {
        byk[key_of(a, a, zero)].kind = CK_OWN;
        for (int l = 0; l < m; ++l) {
            int fm[1] = {l}, fr[1] = {ER_D2};
            add_term(a, a, zero, 0, sys.omega[l], 1, fm, fr);  // omega (n + 1/2)
        }
        for (int b = 0; b < S; ++b) {
            const double c = pl.h_const[a * S + b];
            if (pl.h_dpair[a * S + b] && c != 0.0) add_term(a, b, zero, 0, c, 0, nullptr, nullptr);
        }
    }
    for (const Term &t : sys.terms) {
        bool bad = false;
        int sm[MAX_ORDER];
        for (int l = 0; l < t.nm; ++l) {
            sm[l] = smax_of(t.pow[l], sys.nfunc[t.mode[l]]);
            if (sm[l] < 0) bad = true;
        }
        if (bad) continue;  // odd power on a single-function mode: no elements
        // slow and fast factors
        int ns = 0, smode[MAX_ORDER], spow[MAX_ORDER], smx[MAX_ORDER];
        int nfst = 0, fmode[3], fpow[3];
        int df = 0;
        for (int l = 0; l < t.nm; ++l) {
            if (t.mode[l] < m) {
                smode[ns] = t.mode[l];
                spow[ns] = t.pow[l];
                smx[ns] = sm[l];
                ++ns;
            } else {
                fmode[nfst] = t.mode[l] - m;
                fpow[nfst] = t.pow[l];
                ++nfst;
                df += t.pow[l];
            }
        }
        for (auto &pr : t.pairs) {
            const int a = pr.a, b = pr.b;
            const double c = pr.coef;
            if (ns == 0) {
                // pure fast monomial on the own tile
                if (df == 1) {
                    add_term(a, b, zero, 2 + fmode[0], c, 0, nullptr, nullptr);
                } else if (df == 2) {
                    if (nfst == 1) F.R2[fmode[0]][a] += c;
                    else F.Q2[std::min(fmode[0], fmode[1])][std::max(fmode[0], fmode[1])][a] += c;
                } else {
                    int f3[3], k = 0;
                    for (int q = 0; q < nfst; ++q)
                        for (int r = 0; r < fpow[q]; ++r) f3[k++] = fmode[q];
                    std::sort(f3, f3 + 3);
                    F.C3[f3[0]][f3[1]][f3[2]][a] += c;
                }
                continue;
            }
            // slow shift combinations (last factor fastest, as Source/secondary.f90:98-124)
            int sd[MAX_ORDER];
            for (int q = 0; q < ns; ++q) sd[q] = -smx[q];
            while (true) {
                int sig[CUB_MAXSL] = {0};
                int fm[3], fr[3];
                bool allzero = true;
                for (int q = 0; q < ns; ++q) {
                    sig[smode[q]] = sd[q];
                    fm[q] = smode[q];
                    fr[q] = row_of(spow[q], sd[q]);
                    if (sd[q] != 0) allzero = false;
                }
                if (allzero) {
                    // zero slow shift: the own tile of b; fast degree 0 is the diagonal section
                    // (all slow powers even), fast degree 1 a tile-dependent X_f coefficient
                    if (df == 0) add_term(a, b, zero, 0, c, ns, fm, fr);
                    else if (df == 1) add_term(a, b, zero, 2 + fmode[0], c, ns, fm, fr);
                    else return false;  // degree >= 4
                } else if (df == 0) {
                    add_term(a, b, sig, 0, c, ns, fm, fr);
                } else if (df == 1) {
                    add_term(a, b, sig, 2 + fmode[0], c, ns, fm, fr);
                } else {
                    // df == 2: slow part is x_s; the fast quadratic goes to the s table, the item
                    // carries e = <n|x_s|n+-1>
                    if (ns != 1 || spow[0] != 1 || a != b) return false;
                    const int s = smode[0];
                    Build &B = byk[key_of(a, b, sig)];
                    if (B.qs < 0) {
                        B.qs = s;
                        add_term(a, b, sig, 1, 1.0, 1, fm, fr);
                    }
                    B.kind = CK_Q;
                    // the table is shared by the +e_s and -e_s items: add the coefficient once
                    if (sd[0] > 0) {
                        int f = fmode[0], g = nfst == 2 ? fmode[1] : fmode[0];
                        if (f > g) std::swap(f, g);
                        cp.cs[(((size_t)a * m + s) * NF + f) * NF + g] += c;
                    }
                }
                // next combination
                int q = ns - 1;
                while (q >= 0 && sd[q] + 2 > smx[q]) {
                    sd[q] = -smx[q];
                    --q;
                }
                if (q < 0) break;
                sd[q] += 2;
            }
        }
    }
    // kinds: own (sigma = 0), Q (fast quadratic), Z (fast linear), C (coefficients only)
    for (auto &kv : byk) {
        Build &B = kv.second;
        bool own = true;
        for (int l = 0; l < m; ++l) own = own && kv.first[2 + l] == 0;
        if (own) {
            B.kind = CK_OWN;
            continue;
        }
        if (B.kind == CK_Q) continue;
        B.kind = CK_C;
        for (auto &t : B.info)
            if (t.slot >= 2) B.kind = CK_Z;
    }
    // item list per target in kernel order
    cp.items.clear();
    cp.seg.assign(4 * S + 1, 0);
    cp.tinfo.clear();
    cp.tcoef.clear();
    for (int a = 0; a < S; ++a) {
        std::vector<std::pair<Key, Build *>> lists[4];
        for (auto &kv : byk)
            if (kv.first[0] == a) lists[kv.second.kind].push_back({kv.first, &kv.second});
        // own a first, then the other states' own tiles
        std::stable_sort(lists[CK_OWN].begin(), lists[CK_OWN].end(),
                         [&](auto &x, auto &y) { return (x.first[1] != a) < (y.first[1] != a); });
        for (int k = 0; k < 4; ++k) {
            cp.seg[4 * a + k] = (int)cp.items.size();
            for (auto &e : lists[k]) {
                const Key &ky = e.first;
                Build &B = *e.second;
                CubItem it{};
                it.kind = (signed char)B.kind;
                it.b = (signed char)ky[1];
                it.qs = (signed char)std::max(B.qs, 0);
                int n = 0;
                long long ts = 0;
                for (int l = 0; l < m; ++l)
                    if (ky[2 + l] != 0) {
                        if (n == 3) return false;
                        it.md[n] = (signed char)l;
                        it.sv[n] = (signed char)ky[2 + l];
                        ts += (long long)ky[2 + l] * cp.slow_tshft[l];
                        ++n;
                    }
                it.nsh = (signed char)n;
                it.tshift = (int)ts;
                it.tb = (int)cp.tinfo.size();
                for (size_t q = 0; q < B.info.size(); ++q) {
                    cp.tinfo.push_back(B.info[q]);
                    cp.tcoef.push_back(B.coef[q]);
                }
                it.te = (int)cp.tinfo.size();
                cp.items.push_back(it);
            }
        }
    }
    cp.seg[4 * S] = (int)cp.items.size();
    if (cp.items.size() > 4096) return false;
    // fast tables in single precision
    CubFast<float> &Ff = cp.fast_f;
    Ff = CubFast<float>{};
    for (int j = 0; j < CUB_MAXF; ++j) {
        Ff.sh[j] = F.sh[j];
        Ff.nf[j] = F.nf[j];
        Ff.om[j] = (float)F.om[j];
        for (int a = 0; a < CUB_MAXS; ++a) {
            Ff.R2[j][a] = (float)F.R2[j][a];
            for (int k = 0; k < CUB_MAXF; ++k) {
                Ff.Q2[j][k][a] = (float)F.Q2[j][k][a];
                for (int l = 0; l < CUB_MAXF; ++l) Ff.C3[j][k][l][a] = (float)F.C3[j][k][l][a];
            }
        }
    }
    for (int q = 0; q < CUB_ROWS; ++q)
        for (int r = 0; r < CUB_RPT; ++r) Ff.em[q][r] = (float)F.em[q][r];
    // ring depth per precision; FP64 runs at most 288 consumer threads (register file)
    for (int eb : {8, 4}) {
        const int i = eb == 8 ? 0 : 1;
        if (eb == 8 && cp.threads > 288) continue;
        const int nit = (int)cp.items.size(), nterm = (int)cp.tinfo.size();
        const size_t fixed = (size_t)cub_layout(M, S, nmax, m, NF, cp.sstate, eb, 0, nit, nterm).total;
        const size_t slot = (size_t)cp.sstate * eb;
        size_t budget = 226 * 1024;
        int per = 1;
        if (eb == 4 && cp.threads <= 288 && fixed + 4 * slot <= 112 * 1024) {
            budget = 112 * 1024;
            per = 2;
        }
        if (fixed + 3 * slot > budget) continue;
        cp.nslot[i] = (int)std::min<size_t>(CUB_MAXSLOT, (budget - fixed) / slot);
        cp.smem[i] = (size_t)cub_layout(M, S, nmax, m, NF, cp.sstate, eb, cp.nslot[i], nit, nterm).total;
        cp.per_sm[i] = per;
        cp.prec_ok[i] = true;
    }
    cp.ok = cp.prec_ok[0] || cp.prec_ok[1];
    return cp.ok;
}

#define CK(x)                                                                                    \
    do {                                                                                         \
        cudaError_t e_ = (x);                                                                    \
        if (e_ != cudaSuccess) fail(NVB_ERR_CUDA, std::string(#x ": ") + cudaGetErrorString(e_)); \
    } while (0)

void cubic_upload(CubPlan &cp) {
    cubic_free(cp);
    std::vector<double> blk = cp.tab;
    blk.insert(blk.end(), cp.cs.begin(), cp.cs.end());
    std::vector<float> blkf(blk.begin(), blk.end());
    std::vector<float> tcf(cp.tcoef.begin(), cp.tcoef.end());
    std::vector<int> slow;
    for (int v : cp.slow_tshft) slow.push_back(v);
    for (int v : cp.slow_nfunc) slow.push_back(v);
    auto up = [](auto *&d, const auto &h) {
        using E = typename std::decay_t<decltype(h)>::value_type;
        const size_t n = std::max<size_t>(h.size(), 1);
        CK(cudaMalloc((void **)&d, n * sizeof(E)));
        if (!h.empty()) CK(cudaMemcpy(d, h.data(), h.size() * sizeof(E), cudaMemcpyHostToDevice));
    };
    up(cp.d_blk, blk);
    up(cp.d_blk_f, blkf);
    up(cp.d_tcoef, cp.tcoef);
    up(cp.d_tcoef_f, tcf);
    up(cp.d_tinfo, cp.tinfo);
    up(cp.d_slow, slow);
    up(cp.d_items, cp.items);
    up(cp.d_seg, cp.seg);
    CK(cudaMalloc((void **)&cp.d_err, sizeof(int)));
    CK(cudaMemset(cp.d_err, 0, sizeof(int)));
}

void cubic_free(CubPlan &cp) {
    void *ps[] = {cp.d_blk, cp.d_blk_f, cp.d_tcoef, cp.d_tcoef_f, cp.d_tinfo, cp.d_slow, cp.d_items, cp.d_seg, cp.d_err};
    for (void *p : ps)
        if (p) cudaFree(p);
    cp.d_blk = nullptr;
    cp.d_blk_f = nullptr;
    cp.d_tcoef = nullptr;
    cp.d_tcoef_f = nullptr;
    cp.d_tinfo = nullptr;
    cp.d_slow = nullptr;
    cp.d_items = nullptr;
    cp.d_seg = nullptr;
    cp.d_err = nullptr;
}

}  // namespace nvb
