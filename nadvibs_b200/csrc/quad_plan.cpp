// Host planner of the factorised quadratic H.v kernel (see quad.h).
#include <algorithm>
#include <cmath>

#include "quad.h"

namespace nvb {

bool quad_build(QuadPlan &qp, const Plan &pl, const System &sys) {
    qp = QuadPlan{};
    const int S = sys.S, M = sys.M;
    if (S > QUAD_MAXS || sys.ordr > 2 || M < 2) return false;
    for (const Term &t : sys.terms) {
        int order = 0;
        for (int l = 0; l < t.nm; ++l) order += t.pow[l];
        if (order > 2) return false;
        if (t.nm == 2)
            for (auto &pr : t.pairs)
                if (pr.a != pr.b) return false;  // bilinear inter-state coupling: not factorisable here
    }
    // tile: the slowest fast mode m whose pencil stride shft(m) is a multiple of 32 threads
    // (64..288 consumer threads) and whose pencil has <= 8 rows
    int best = -1;
    for (int m = M - 1; m >= 1; --m) {
        const long long th = sys.shft[m];
        if (th > 288) break;
        if (M - m > QUAD_MAXF) break;
        if (m > QUAD_MAXSL) continue;
        if (th % 32 == 0 && th >= 64 && sys.nfunc[m] <= QUAD_RPT && M - m >= 2) best = m;
    }
    if (best < 1) return false;
    const int m = best;
    qp.S = S;
    qp.M = M;
    qp.m = m;
    qp.nF = M - m;
    qp.nmax = pl.nmax;
    qp.threads = (int)sys.shft[m];
    qp.nv = (int)sys.nfunc[m];
    qp.TF = qp.threads * qp.nv;
    if (sys.dimen / qp.TF > (1LL << 30)) return false;
    qp.ntiles = (int)(sys.dimen / qp.TF);
    qp.dimen = sys.dimen;
    long long pad = 0;
    for (int k = m + 1; k < M; ++k) pad = std::max<long long>(pad, 2 * sys.shft[k]);
    qp.pad = (int)((pad + 3) / 4 * 4);
    qp.sstate = qp.pad + qp.threads * QUAD_RPT + qp.pad;
    for (int l = 0; l < m; ++l) {
        qp.slow_tshft.push_back((int)(sys.shft[l] / qp.TF));
        qp.slow_nfunc.push_back((int)sys.nfunc[l]);
    }
    // couplings by shape
    qp.G.assign((size_t)M * S * S, 0.0);
    qp.R.assign((size_t)M * S * S, 0.0);
    qp.Q.assign((size_t)M * M * S, 0.0);
    for (const Term &t : sys.terms) {
        if (t.nm == 1 && t.pow[0] == 1)
            for (auto &pr : t.pairs) qp.G[((size_t)t.mode[0] * S + pr.a) * S + pr.b] += pr.coef;
        else if (t.nm == 1 && t.pow[0] == 2)
            for (auto &pr : t.pairs) qp.R[((size_t)t.mode[0] * S + pr.a) * S + pr.b] += pr.coef;
        else if (t.nm == 2) {
            const int k = std::min(t.mode[0], t.mode[1]), l = std::max(t.mode[0], t.mode[1]);
            for (auto &pr : t.pairs) qp.Q[((size_t)k * M + l) * S + pr.a] += pr.coef;
        }
    }
    qp.cst = pl.h_const;
    qp.dpm = 0;
    for (int ab = 0; ab < S * S; ++ab)
        if (pl.h_dpair[ab]) qp.dpm |= 1u << ab;
    qp.omega = sys.omega;
    // element tables E1+[n] = <n|x|n+1>, E1-[n] = <n|x|n-1>, E2+[n] = <n|x^2|n+2>,
    // E2-[n] = <n|x^2|n-2>, D2[n] = <n|x^2|n>, zero where the partner row is outside the basis
    const int nmax = pl.nmax;
    qp.tab.assign((size_t)M * 5 * nmax, 0.0);
    for (int j = 0; j < M; ++j) {
        const int nf = (int)sys.nfunc[j];
        double *t = qp.tab.data() + (size_t)j * 5 * nmax;
        for (int n = 0; n < nf; ++n) {
            if (n + 1 < nf) t[0 * nmax + n] = hoelem(1, n + 1, n + 2, 1);
            if (n >= 1) t[1 * nmax + n] = hoelem(1, n, n + 1, 1);
            if (n + 2 < nf) t[2 * nmax + n] = hoelem(2, n + 1, n + 3, 1);
            if (n >= 2) t[3 * nmax + n] = hoelem(2, n - 1, n + 1, 1);
            t[4 * nmax + n] = hoelem(2, n + 1, n + 1, 1);
        }
    }
    // fast-mode parameter block
    QuadFast<double> &F = qp.fast_d;
    F = QuadFast<double>{};
    for (int j = 0; j < qp.nF; ++j) {
        const int l = m + j;
        F.sh[j] = (int)sys.shft[l];
        F.nf[j] = (int)sys.nfunc[l];
        F.om[j] = sys.omega[l];
        for (int a = 0; a < S; ++a)
            for (int b = 0; b < S; ++b) {
                F.G[j][a][b] = qp.G[((size_t)l * S + a) * S + b];
                F.R[j][a][b] = qp.R[((size_t)l * S + a) * S + b];
            }
        for (int i = 0; i < j; ++i)
            for (int a = 0; a < S; ++a) F.Q[i][j][a] = qp.Q[((size_t)(m + i) * M + l) * S + a];
    }
    for (int q = 0; q < 5; ++q)
        for (int r = 0; r < QUAD_RPT; ++r) F.em[q][r] = r < nmax ? qp.tab[((size_t)m * 5 + q) * nmax + r] : 0.0;
    QuadFast<float> &Ff = qp.fast_f;
    Ff = QuadFast<float>{};
    for (int j = 0; j < QUAD_MAXF; ++j) {
        Ff.sh[j] = F.sh[j];
        Ff.nf[j] = F.nf[j];
        Ff.om[j] = (float)F.om[j];
        for (int a = 0; a < QUAD_MAXS; ++a) {
            for (int b = 0; b < QUAD_MAXS; ++b) {
                Ff.G[j][a][b] = (float)F.G[j][a][b];
                Ff.R[j][a][b] = (float)F.R[j][a][b];
            }
            for (int i = 0; i < QUAD_MAXF; ++i) Ff.Q[i][j][a] = (float)F.Q[i][j][a];
        }
    }
    for (int q = 0; q < 5; ++q)
        for (int r = 0; r < QUAD_RPT; ++r) Ff.em[q][r] = (float)F.em[q][r];
    // ring items per target state: own tiles, slow +-1, slow +-2, slow bilinear
    qp.items.clear();
    qp.item_beg.assign(S + 1, 0);
    qp.slow_beg.assign(S, 0);
    qp.z_end.assign(S, 0);
    qp.ownmask = 0;
    for (int a = 0; a < S; ++a) {
        qp.item_beg[a] = (int)qp.items.size();
        auto push = [&](int kind, int b, int k, int sk, int l, int sl) {
            QuadItem it{};
            it.kind = (signed char)kind;
            it.a = (signed char)a;
            it.b = (signed char)b;
            it.k = (signed char)k;
            it.sk = (signed char)sk;
            it.l = (signed char)l;
            it.sl = (signed char)sl;
            it.tshift = kind == QI_OWN ? 0 : sk * qp.slow_tshft[k] + (kind == QI_PAIR ? sl * qp.slow_tshft[l] : 0);
            qp.items.push_back(it);
        };
        push(QI_OWN, a, 0, 0, 0, 0);
        for (int b = 0; b < S; ++b) {
            if (b == a) continue;
            bool need = false;
            if (pl.h_dpair[a * S + b]) {
                need |= qp.cst[a * S + b] != 0.0;
                for (int k = 0; k < M; ++k) need |= qp.R[((size_t)k * S + a) * S + b] != 0.0;
            }
            for (int j = 0; j < qp.nF; ++j)
                need |= qp.G[((size_t)(m + j) * S + a) * S + b] != 0.0 || qp.R[((size_t)(m + j) * S + a) * S + b] != 0.0;
            if (need) {
                push(QI_OWN, b, 0, 0, 0, 0);
                qp.ownmask |= 1u << (a * S + b);
            }
        }
        // slow +-1: first the own state's tiles that feed Z (slow-fast bilinear), then the
        // coefficient-only ones, so that the kernel's per-tile records keep the Z items first
        qp.slow_beg[a] = (int)qp.items.size();
        auto feeds_z = [&](int k) {
            for (int j = 0; j < qp.nF; ++j)
                if (qp.Q[((size_t)k * M + m + j) * S + a] != 0.0) return true;
            return false;
        };
        for (int k = 0; k < m; ++k)
            if (sys.nfunc[k] >= 2 && feeds_z(k)) {
                push(QI_SLOW1, a, k, +1, 0, 0);
                push(QI_SLOW1, a, k, -1, 0, 0);
            }
        qp.z_end[a] = (int)qp.items.size();
        for (int k = 0; k < m; ++k) {
            if (sys.nfunc[k] < 2) continue;
            for (int b = 0; b < S; ++b) {
                if (b == a && feeds_z(k)) continue;
                if (qp.G[((size_t)k * S + a) * S + b] == 0.0) continue;
                push(QI_SLOW1, b, k, +1, 0, 0);
                push(QI_SLOW1, b, k, -1, 0, 0);
            }
        }
        for (int k = 0; k < m; ++k) {
            if (sys.nfunc[k] < 3) continue;
            for (int b = 0; b < S; ++b)
                if (qp.R[((size_t)k * S + a) * S + b] != 0.0) {
                    push(QI_SLOW2, b, k, +2, 0, 0);
                    push(QI_SLOW2, b, k, -2, 0, 0);
                }
        }
        for (int k = 0; k < m; ++k)
            for (int l = k + 1; l < m; ++l)
                if (sys.nfunc[k] > 1 && sys.nfunc[l] > 1 && qp.Q[((size_t)k * M + l) * S + a] != 0.0)
                    for (int sk : {+1, -1})
                        for (int sl : {+1, -1}) push(QI_PAIR, a, k, sk, l, sl);
    }
    qp.item_beg[S] = (int)qp.items.size();
    if (qp.items.size() > 1024) return false;  // the producer keeps one validity bit per item in a warp
    // ring depth: as many slots as fit next to the tables and Z (<= QUAD_MAXSLOT)
    for (int eb : {8, 4}) {
        const int i = eb == 8 ? 0 : 1;
        const size_t fixed = (size_t)quad_layout(M, S, nmax, m, qp.nF, qp.sstate, eb, 0, (int)qp.items.size()).total;
        const size_t slot = (size_t)qp.sstate * eb;
        // FP64: one CTA per multiprocessor; FP32: two where they fit (more warps to hide latency)
        size_t budget = eb == 8 ? 226 * 1024 : 112 * 1024;
        if (fixed + 4 * slot > budget) budget = 226 * 1024;
        if (fixed + 3 * slot > budget) return false;
        qp.nslot[i] = (int)std::min<size_t>(QUAD_MAXSLOT, (budget - fixed) / slot);
        qp.smem[i] = (size_t)quad_layout(M, S, nmax, m, qp.nF, qp.sstate, eb, qp.nslot[i], (int)qp.items.size()).total;
    }
    qp.ok = true;
    return true;
}

#define CK(x)                                                                                    \
    do {                                                                                         \
        cudaError_t e_ = (x);                                                                    \
        if (e_ != cudaSuccess) fail(NVB_ERR_CUDA, std::string(#x ": ") + cudaGetErrorString(e_)); \
    } while (0)

void quad_upload(QuadPlan &qp) {
    if (!qp.ok) return;
    std::vector<double> blk;
    for (auto *v : {&qp.tab, &qp.G, &qp.R, &qp.Q, &qp.cst, &qp.omega}) blk.insert(blk.end(), v->begin(), v->end());
    std::vector<float> blkf(blk.begin(), blk.end());
    std::vector<int> slow(qp.slow_tshft);
    slow.insert(slow.end(), qp.slow_nfunc.begin(), qp.slow_nfunc.end());
    slow.push_back(0);
    CK(cudaMalloc((void **)&qp.d_blk, blk.size() * sizeof(double)));
    CK(cudaMemcpy(qp.d_blk, blk.data(), blk.size() * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMalloc((void **)&qp.d_blk_f, blkf.size() * sizeof(float)));
    CK(cudaMemcpy(qp.d_blk_f, blkf.data(), blkf.size() * sizeof(float), cudaMemcpyHostToDevice));
    CK(cudaMalloc((void **)&qp.d_slow, slow.size() * sizeof(int)));
    CK(cudaMemcpy(qp.d_slow, slow.data(), slow.size() * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMalloc((void **)&qp.d_items, qp.items.size() * sizeof(QuadItem)));
    CK(cudaMemcpy(qp.d_items, qp.items.data(), qp.items.size() * sizeof(QuadItem), cudaMemcpyHostToDevice));
    // item_beg[0..S], slow_beg[0..S-1], z_end[0..S-1]
    std::vector<int> beg(qp.item_beg);
    beg.insert(beg.end(), qp.slow_beg.begin(), qp.slow_beg.end());
    beg.insert(beg.end(), qp.z_end.begin(), qp.z_end.end());
    CK(cudaMalloc((void **)&qp.d_item_beg, beg.size() * sizeof(int)));
    CK(cudaMemcpy(qp.d_item_beg, beg.data(), beg.size() * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMalloc((void **)&qp.d_err, sizeof(int)));
    CK(cudaMemset(qp.d_err, 0, sizeof(int)));
}

void quad_free(QuadPlan &qp) {
    void *ps[] = {qp.d_blk, qp.d_blk_f, qp.d_slow, qp.d_items, qp.d_item_beg, qp.d_err};
    for (void *p : ps)
        if (p) cudaFree(p);
    qp.d_blk = nullptr;
    qp.d_blk_f = nullptr;
    qp.d_slow = nullptr;
    qp.d_items = nullptr;
    qp.d_item_beg = nullptr;
    qp.d_err = nullptr;
}

}  // namespace nvb
