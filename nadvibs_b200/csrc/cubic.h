// Factorised H.v for cubic Hamiltonians (ordr <= 3) whose couplings between different states
// are constants and linear terms: the form of the large mixed-precision benchmark system
// (diagonal blocks with every monomial up to degree 3, off-diagonal blocks linear).
//
// The modes split as in the quadratic kernel: slow modes 0..m-1, fast modes m..M-1, one tile =
// the rows with fixed slow digits, one thread per pencil of mode m (rows r*shft(m) + tid).  Every
// monomial factors into a slow part and a fast part.  The slow part's shift combinations
// (Source/top.f90:757-806 with the shift rules of Source/secondary.f90:33-37,98-124) select a
// neighbour state-tile x_b(p + sigma) -- an "item", streamed through the shared-memory ring by
// TMA bulk copies -- and give an element factor that depends only on the tile's slow digits.
// The fast part is an operator on the item's rows, of degree 0 (a coefficient), 1 (X_f) or 2
// (only on the +-1 neighbours of a slow mode s: x_s x_f x_g and x_s x_f^2), or of degree 3 on the
// own tile (x_f x_g x_h over fast modes).  All fast operators are folded into
//   y_a = c x + sum_f X_f Z_f,   Z_f = sum (coefficient) * (fast operator of degree <= 2) x,
// using that operators on different modes commute: x_f x_g x_h = X_h (X_f X_g), x_f^2 x_h =
// X_h (x_f^2), x_f x_g = X_g X_f; only x_f^2, x_f^3 and the degree-2 parts of the +-1 items are
// applied directly.  Per item the tile-dependent coefficients (c, z_f and, for the +-1 items of
// fast-quadratic terms, the slow element factor e) are evaluated once per tile from a short
// program of (coefficient, slow element factors) terms.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "plan.h"

namespace nvb {

constexpr int CUB_RPT = 8;      // rows per thread (the pencil of mode m), nfunc(m) <= 8
constexpr int CUB_MAXF = 5;     // fast modes
constexpr int CUB_MAXSL = 12;   // slow modes
constexpr int CUB_MAXS = 4;     // electronic states
constexpr int CUB_MAXSLOT = 16;
constexpr int CUB_ROWS = 9;     // element rows per mode (below)
// element rows: <n|x|n+-1>, <n|x^2|n+-2>, <n|x^2|n>, <n|x^3|n+-3>, <n|x^3|n+-1>; zero where the
// partner function is outside the basis
enum CubRow { ER_1P = 0, ER_1M = 1, ER_2P = 2, ER_2M = 3, ER_D2 = 4, ER_3P3 = 5, ER_3M3 = 6, ER_3P1 = 7, ER_3M1 = 8 };

// Fast-mode data passed by value (constant-bank operands inside the kernel).
template <typename T>
struct CubFast {
    int sh[CUB_MAXF];                                   // shft of fast mode m+j (sh[0] = threads)
    int nf[CUB_MAXF];                                   // nfunc of fast mode m+j
    T em[CUB_ROWS][CUB_RPT];                            // mode m element rows by digit
    T om[CUB_MAXF];                                     // frequencies
    T R2[CUB_MAXF][CUB_MAXS];                           // x_f^2, state-diagonal
    T Q2[CUB_MAXF][CUB_MAXF][CUB_MAXS];                 // x_f x_g, f < g, state-diagonal
    T C3[CUB_MAXF][CUB_MAXF][CUB_MAXF][CUB_MAXS];       // x_f x_g x_h, f <= g <= h, state-diagonal
};

enum CubKind { CK_OWN = 0, CK_Q = 1, CK_Z = 2, CK_C = 3 };
// One state-tile streamed through the ring: x_b(p + sigma) for the tile p and target state a.
struct CubItem {
    signed char kind;    // CubKind
    signed char b;       // source state
    signed char nsh;     // number of slow modes sigma shifts (0..3)
    signed char qs;      // CK_Q: the slow mode s of x_s (fast quadratic table row)
    signed char md[3];   // slow modes of sigma
    signed char sv[3];   // their shifts
    signed char pad0[2];
    int tshift;          // sigma in tiles
    int tb, te;          // its coefficient program: terms [tb, te)
};
// record[slot] += coef * prod_q tab[md[q]][rw[q]][slow digit of md[q]]; slot 0 = c, 1 = e, 2+f = z_f
struct CubTerm {
    signed char slot, nf;
    signed char md[3], rw[3];
};

struct CubPlan {
    bool ok = false;
    bool prec_ok[2] = {false, false};  // FP64, FP32
    int S = 0, m = 0, nF = 0, M = 0, nmax = 0;
    int TF = 0, ntiles = 0;
    long long dimen = 0;
    int threads = 0, pad = 0, nv = 0, sstate = 0;
    std::vector<int> slow_tshft, slow_nfunc;
    std::vector<double> tab;  // [M][CUB_ROWS][nmax]
    // per target state a: items[seg[4a] ..) = own a, the other states' own tiles, then from seg[4a+1]
    // the +-1 items with fast quadratic parts, from seg[4a+2] the items with fast linear parts,
    // from seg[4a+3] the coefficient-only items; seg[4S] = total
    std::vector<CubItem> items;
    std::vector<int> seg;
    std::vector<CubTerm> tinfo;
    std::vector<double> tcoef;
    std::vector<double> cs;  // [S][m][nF][nF] fast quadratic of the x_s items: x_s x_f x_g (f < g), x_s x_f^2 (f = g)
    CubFast<double> fast_d{};
    CubFast<float> fast_f{};
    int nslot[2] = {0, 0};
    size_t smem[2] = {0, 0};
    int grid[2] = {0, 0};
    int per_sm[2] = {1, 1};
    // device
    double *d_blk = nullptr;  // tab | cs
    float *d_blk_f = nullptr;
    double *d_tcoef = nullptr;
    float *d_tcoef_f = nullptr;
    CubTerm *d_tinfo = nullptr;
    int *d_slow = nullptr;  // [2][m]: tile shifts, nfunc
    CubItem *d_items = nullptr;
    int *d_seg = nullptr;
    int *d_err = nullptr;
    int test_nocopy = 0;
};

// Shared-memory layout (byte offsets), identical on host and device.
struct CubLayout {
    int tab, cs, sd, dig, items, seg, plist, pres, cl, cnt, rec, ring, z, total;
};
__host__ __device__ inline CubLayout cub_layout(int M, int S, int nmax, int m, int nF, int sstate, int eb, int nslot,
                                                int nitems, int nterms) {
    CubLayout L{};
    int o = 2 * CUB_MAXSLOT * 8 + 16;  // full / empty mbarriers, abort flag
    auto take = [&](int bytes) {
        int r = o;
        o += (bytes + 15) / 16 * 16;
        return r;
    };
    L.tab = take(M * CUB_ROWS * nmax * eb);
    L.cs = take(S * (m > 0 ? m : 1) * nF * nF * eb);
    L.sd = take(2 * CUB_MAXSL * 4);        // slow tile strides, nfunc
    L.dig = take(2 * CUB_MAXSL * 4);       // per tile parity: slow digits
    L.items = take(nitems * (int)sizeof(CubItem));
    L.seg = take((4 * CUB_MAXS + 1) * 4);
    L.plist = take(2 * (nitems + 1) * 8);  // producer: per tile parity, count and present items' source offsets
    L.pres = take(nitems);                 // consumers: presence of every item in the tile
    L.cl = take(nitems * 2);               // consumers: present items of each target, in order (< 4096)
    L.cnt = take(CUB_MAXS * 4 * 4);        // per target: Q, Z, C items present
    L.rec = take(nitems * (nF + 2) * eb);  // per item: c, e, z[nF]
    o = (o + 127) / 128 * 128;
    L.ring = take(nslot * sstate * eb);
    // Z exchange buffer; at the start of a tile it holds the term products and their slots
    const int zb = sstate * eb, pb = nterms * (eb + 1);
    L.z = take(zb > pb ? zb : pb);
    L.total = o;
    return L;
}

bool cubic_build(CubPlan &cp, const Plan &pl, const System &sys, int quirk_cubic);
void cubic_upload(CubPlan &cp);
void cubic_free(CubPlan &cp);
// Launches by precision (hv_cubic_f64.cu, hv_cubic_f32.cu; FP32 pencils of more than 288
// threads in hv_cubic_f32w.cu).  Each returns the number of blocks (= partials written to
// alpha_part).
int cubic_launch_f64(CubPlan &cp, const double *x, double *y, const double *scale, double *alpha_part, cudaStream_t st);
int cubic_launch_f32(CubPlan &cp, const float *x, float *y, const double *scale, double *alpha_part, cudaStream_t st);
int cubic_launch_f32_wide(CubPlan &cp, const float *x, float *y, const double *scale, double *alpha_part,
                          cudaStream_t st);
template <typename T>
inline int cubic_launch(CubPlan &cp, const T *x, T *y, const double *scale, double *alpha_part, cudaStream_t st) {
    if constexpr (sizeof(T) == 8) return cubic_launch_f64(cp, x, y, scale, alpha_part, st);
    else return cubic_launch_f32(cp, x, y, scale, alpha_part, st);
}

}  // namespace nvb
