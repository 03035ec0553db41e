// Host-side construction of the device plan from the merged term table.
#include "plan.h"

#include <cmath>
#include <cstring>

namespace nvb {

// <a-1| x^p |b-1> in the infinite harmonic-oscillator basis, x = (a + a^+)/sqrt(2).
// The table has to equal the reference's (Source/function.f90:186-250) because it defines
// the Hamiltonian; quirk_cubic keeps its <m|x^3|m+-1>, which lacks the factor 3 of the exact
// value 3*sqrt((m+1)^3/8).
double hoelem(int p, int a, int b, int quirk_cubic) {
    const double m = (double)a - 1.0;
    switch (p) {
    case 0: return b == a ? 1.0 : 0.0;
    case 1:
        if (b == a + 1) return std::sqrt((m + 1) / 2);
        if (b == a - 1) return std::sqrt(m / 2);
        return 0.0;
    case 2:
        if (b == a + 2) return std::sqrt((m + 1) * (m + 2) / 4);
        if (b == a) return (2 * m + 1) / 2;
        if (b == a - 2) return std::sqrt(m * (m - 1) / 4);
        return 0.0;
    case 3: {
        const double f = quirk_cubic ? 1.0 : 3.0;
        if (b == a + 3) return std::sqrt((m + 1) * (m + 2) * (m + 3) / 8);
        if (b == a + 1) return std::sqrt(((m + 1) * (m + 1) * (m + 1)) / 8) * f;
        if (b == a - 1) return std::sqrt((m * m * m) / 8) * f;
        if (b == a - 3) return std::sqrt(m * (m - 1) * (m - 2) / 8);
        return 0.0;
    }
    case 4:
        if (b == a + 4) return std::sqrt((m + 1) * (m + 2) * (m + 3) * (m + 4)) / 4;
        if (b == a + 2) return (2 * m + 3) * std::sqrt((m + 1) * (m + 2)) / 2;
        if (b == a) return 3 * (2 * m * m + 2 * m + 1) / 4;
        if (b == a - 2) return (2 * m - 1) * std::sqrt(m * (m - 1)) / 2;
        if (b == a - 4) return std::sqrt(m * (m - 1) * (m - 2) * (m - 3)) / 4;
        return 0.0;
    default: return 0.0;
    }
}

static int smax_of(int p, int64_t nf) {
    int s = p;
    while (s > nf - 1) s -= 2;  // Source/secondary.f90:33-37
    return s;
}

void plan_build(Plan &pl, const System &sys, int quirk_cubic, int quirk_lower) {
    const int S = sys.S, M = sys.M;
    pl.S = S;
    pl.M = M;
    pl.dimen = sys.dimen;
    pl.nmax = 1;
    for (auto nf : sys.nfunc) pl.nmax = std::max<int>(pl.nmax, (int)nf);
    pl.h_nfunc.assign(sys.nfunc.begin(), sys.nfunc.end());
    pl.h_shft.assign(sys.shft.begin(), sys.shft.end());
    pl.h_omega = sys.omega;
    // element table
    pl.h_etab.assign((size_t)4 * ETAB_J * pl.nmax, 0.0);
    for (int p = 1; p <= 4; ++p)
        for (int j = 0; j < ETAB_J; ++j)
            for (int m = 0; m < pl.nmax; ++m)
                pl.h_etab[((size_t)(p - 1) * ETAB_J + j) * pl.nmax + m] = hoelem(p, m + 1, m + 1 + j, quirk_cubic);
    auto etab_row = [&](int p, int j) { return ((p - 1) * ETAB_J + j) * pl.nmax; };
    // per-term dense coupling blocks
    const int nt = (int)sys.terms.size();
    pl.nterms = nt;
    pl.h_coef.assign((size_t)std::max(nt, 1) * S * S, 0.0);
    pl.h_mask.assign((size_t)std::max(nt, 1) * 2, 0ull);
    for (int t = 0; t < nt; ++t)
        for (auto &pr : sys.terms[t].pairs) {
            pl.h_coef[((size_t)t * S + pr.a) * S + pr.b] = pr.coef;
            int bit = pr.a * S + pr.b;
            pl.h_mask[(size_t)t * 2 + (bit >> 6)] |= 1ull << (bit & 63);
        }
    // diagonal-section bookkeeping (Source/top.f90:528-553 and :717-755)
    std::vector<int> dchk((size_t)S * S, 0);
    for (int i = 0; i < S; ++i)
        for (int j = 0; j <= i; ++j) {
            double c = sys.concoef[(size_t)(i + 1) * i / 2 + j];
            if (std::fabs(c) > 1e-16) dchk[i * S + j] = dchk[j * S + i] = 1;
        }
    pl.h_steps.clear();
    pl.h_diag.clear();
    for (int t = 0; t < nt; ++t) {
        const Term &T = sys.terms[t];
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
        if (bad) continue;  // odd power on a single-function mode: no elements
        if (diag) {
            DevDiag dg{};
            dg.nm = T.nm;
            dg.term = t;
            for (int l = 0; l < T.nm; ++l) {
                dg.mode[l] = T.mode[l];
                dg.etab[l] = etab_row(T.pow[l], 0);
            }
            pl.h_diag.push_back(dg);
            for (auto &pr : T.pairs) dchk[pr.a * S + pr.b] = 1;
        }
        // shift enumeration of Source/secondary.f90:98-124 (last digit fastest)
        sd[T.nm - 1] -= 2;
        for (long long k = 0; k < nsteps; ++k) {
            int l = T.nm - 1;
            while (sd[l] >= sm[l]) { sd[l] = -sm[l]; --l; }
            sd[l] += 2;
            long long stride = 0;
            for (int q = 0; q < T.nm; ++q) stride += (long long)sd[q] * sys.shft[T.mode[q]];
            if (stride == 0) continue;
            DevStep st{};
            st.nm = T.nm;
            st.term = t;
            st.stride = stride;
            for (int q = 0; q < T.nm; ++q) {
                st.mode[q] = T.mode[q];
                st.sig[q] = sd[q];
                st.etab[q] = etab_row(T.pow[q], std::abs(sd[q]));
            }
            pl.h_steps.push_back(st);
        }
    }
    pl.nsteps = (int)pl.h_steps.size();
    pl.ndiag = (int)pl.h_diag.size();
    // which entries of the diagonal block are applied, and their constants
    pl.h_const.assign((size_t)S * S, 0.0);
    pl.h_dpair.assign((size_t)S * S, 0);
    for (int a = 0; a < S; ++a)
        for (int b = 0; b < S; ++b) {
            const int hi = std::max(a, b), lo = std::min(a, b);
            const double c = sys.concoef[(size_t)(hi + 1) * hi / 2 + lo];
            bool applied;
            if (a == b) applied = true;
            else if (a > b) applied = dchk[a * S + b] != 0;
            else applied = !quirk_lower && dchk[a * S + b] != 0;
            pl.h_dpair[a * S + b] = applied ? 1 : 0;
            pl.h_const[a * S + b] = applied ? c : 0.0;
        }
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

static std::vector<float> tof(const std::vector<double> &v) { return std::vector<float>(v.begin(), v.end()); }

void plan_upload(Plan &pl) {
    plan_free(pl);
    up(pl.d_steps, pl.h_steps);
    up(pl.d_diag, pl.h_diag);
    up(pl.d_coef, pl.h_coef);
    up(pl.d_coef_f, tof(pl.h_coef));
    up(pl.d_mask, pl.h_mask);
    up(pl.d_const, pl.h_const);
    up(pl.d_const_f, tof(pl.h_const));
    up(pl.d_dpair, pl.h_dpair);
    up(pl.d_etab, pl.h_etab);
    up(pl.d_etab_f, tof(pl.h_etab));
    up(pl.d_nfunc, pl.h_nfunc);
    up(pl.d_shft, pl.h_shft);
    up(pl.d_omega, pl.h_omega);
    up(pl.d_omega_f, tof(pl.h_omega));
}

void plan_free(Plan &pl) {
    void *ps[] = {pl.d_steps, pl.d_diag, pl.d_coef, pl.d_coef_f, pl.d_mask, pl.d_const, pl.d_const_f,
                  pl.d_dpair, pl.d_etab, pl.d_etab_f, pl.d_nfunc, pl.d_shft, pl.d_omega, pl.d_omega_f};
    for (void *p : ps)
        if (p) cudaFree(p);
    pl.d_steps = nullptr; pl.d_diag = nullptr; pl.d_coef = nullptr; pl.d_coef_f = nullptr;
    pl.d_mask = nullptr; pl.d_const = nullptr; pl.d_const_f = nullptr; pl.d_dpair = nullptr;
    pl.d_etab = nullptr; pl.d_etab_f = nullptr; pl.d_nfunc = nullptr; pl.d_shft = nullptr;
    pl.d_omega = nullptr; pl.d_omega_f = nullptr;
}

}  // namespace nvb
