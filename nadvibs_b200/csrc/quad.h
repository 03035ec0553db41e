// Factorised H.v for quadratic Hamiltonians (ordr <= 2) whose bilinear couplings x_k x_l are
// diagonal in the electronic states: the linear vibronic-coupling form with quadratic
// diagonal blocks, which is the structure of the drop-in benchmark systems.
//
// With X_k the ladder part <n|x|n+-1> along mode k and T_k the +-2 part of x_k^2,
//   y_a = D_ab(p) x_b + sum_k G^ab_k X_k x_b + sum_k R^ab_k T_k x_b + sum_{k<l} Q^a_kl X_k X_l x_a
// where D is the diagonal section of the reference's product (constants, harmonic energy and
// the zero-shift part of the squares; Source/top.f90:717-755) and the rest are its shifted
// steps (Source/top.f90:757-806).  The modes split as in the slab kernel: slow modes 0..m-1,
// fast modes m..M-1, one tile = the rows with fixed slow digits.  A thread owns the whole
// pencil of mode m (rows r*shft(m) + tid, r = digit of mode m), so shifts along m are
// register moves.  The bilinear part is factorised over the fast modes,
//   sum_{k<l} Q_kl X_k X_l x = sum_{l fast} X_l Z_l + sum_{k<l slow} Q_kl X_k X_l x,
//   Z_l = sum_b G^ab_l x_b + sum_{k<l} Q^a_kl X_k x_a,
// so a row costs O(M) arithmetic instead of O(M^2).  Z_m stays in registers, Z_l (l > m) goes
// through shared memory for the fast shifts.  Everything a tile reads besides its own rows is
// a whole neighbour state-tile x_b(p + sigma) with a slow shift sigma (X_k x for slow k from
// the +-1 tiles, the +-2 tiles of the squares, the +-e_k +- e_l tiles of the slow bilinear
// terms, and the other states' own tiles): the kernel streams these "items" through a ring
// of shared-memory slots filled by TMA bulk copies from a producer warp, so that many tiles
// are in flight per multiprocessor.
#pragma once
#include <cstdint>
#include <vector>

#include "plan.h"

namespace nvb {

constexpr int QUAD_RPT = 8;     // rows per thread (the pencil of mode m), nfunc(m) <= 8
constexpr int QUAD_MAXF = 4;    // fast modes
constexpr int QUAD_MAXSL = 12;  // slow modes
constexpr int QUAD_MAXS = 4;    // electronic states

// Fast-mode data passed by value: indexed by compile-time constants inside the kernel, so the
// coefficients are constant-bank operands.
template <typename T>
struct QuadFast {
    int sh[QUAD_MAXF];                       // shft of fast mode m+j (sh[0] = threads)
    int nf[QUAD_MAXF];                       // nfunc of fast mode m+j
    T em[5][QUAD_RPT];                       // mode m rows E1+, E1-, E2+, E2-, D2 by digit
    T G[QUAD_MAXF][QUAD_MAXS][QUAD_MAXS];    // linear blocks of the fast modes
    T R[QUAD_MAXF][QUAD_MAXS][QUAD_MAXS];    // square blocks
    T Q[QUAD_MAXF][QUAD_MAXF][QUAD_MAXS];    // [i][j][a], i < j, bilinear fast-fast
    T om[QUAD_MAXF];                         // frequencies
};

// One state-tile streamed through the shared-memory ring: x_b(p + shift) for the tile p.
enum QuadItemKind { QI_OWN = 0, QI_SLOW1 = 1, QI_SLOW2 = 2, QI_PAIR = 3 };
struct QuadItem {
    signed char kind;   // QuadItemKind
    signed char b;      // source state
    signed char k, sk;  // slow mode and its shift (+-1 or +-2); unused for QI_OWN
    signed char l, sl;  // second slow mode of a bilinear neighbour (QI_PAIR)
    signed char a;      // target state whose list holds the item
    signed char pad0;
    int tshift;         // sum of the shifts times the slow tile strides
};

struct QuadPlan {
    bool ok = false;
    int S = 0, m = 0, nF = 0, M = 0, nmax = 0;
    int TF = 0, ntiles = 0;
    long long dimen = 0;
    int threads = 0, pad = 0, nv = 0;  // nv = nfunc(m)
    int sstate = 0;                    // elements per state in a shared-memory array
    unsigned dpm = 0;                  // bit a*S+b: entry (a,b) of the diagonal block applied
    // host copies, S x S blocks in the scaled (dimensionless) coefficients
    std::vector<double> G;    // [M][S][S] linear
    std::vector<double> R;    // [M][S][S] squares
    std::vector<double> Q;    // [M][M][S] bilinear, state-diagonal, k < l stored at [k][l]
    std::vector<double> cst;  // [S][S] diagonal-section constants (applied entries only)
    std::vector<double> tab;  // per mode j: rows E1+, E1-, E2+, E2-, D2, each of nmax
    std::vector<double> omega;
    std::vector<int> slow_tshft, slow_nfunc;
    // per target state a: items[item_beg[a] .. item_beg[a+1]) in the order own a, the other
    // states' own tiles (bit a*S+b of ownmask), from slow_beg[a] the slow +-1 tiles of state a
    // that feed Z (up to z_end[a]), then the coefficient-only slow items
    std::vector<QuadItem> items;
    std::vector<int> item_beg, slow_beg, z_end;
    unsigned ownmask = 0;
    int nslot[2] = {0, 0};        // ring slots, FP64 / FP32
    QuadFast<double> fast_d{};
    QuadFast<float> fast_f{};
    // device: one block of doubles and one of floats: tab | G | R | Q | cst | omega
    double *d_blk = nullptr;
    float *d_blk_f = nullptr;
    int *d_slow = nullptr;  // [2][m]: tile shifts, nfunc
    QuadItem *d_items = nullptr;
    int *d_item_beg = nullptr;
    int *d_err = nullptr;
    size_t smem[2] = {0, 0};  // FP64, FP32
    int grid[2] = {0, 0};
    int test_nocopy = 0;      // failure test (nvb_set_fault_test): no copies, waits run out
};

// Shared-memory layout (byte offsets), identical on host and device.
struct QuadLayout {
    int tab, G, R, Q, cst, om, sd, se, dt, items, cnt, plist, rec, ring, z, total;
};
constexpr int QUAD_MAXSLOT = 16;
__host__ __device__ inline QuadLayout quad_layout(int M, int S, int nmax, int m, int nF, int sstate, int eb,
                                                  int nslot, int nitems) {
    QuadLayout L{};
    int o = 2 * QUAD_MAXSLOT * 8 + 16;  // full / empty mbarriers of the ring, abort flag
    auto take = [&](int bytes) {
        int r = o;
        o += (bytes + 15) / 16 * 16;
        return r;
    };
    L.tab = take(M * 5 * nmax * eb);
    L.G = take(M * S * S * eb);
    L.R = take(M * S * S * eb);
    L.Q = take(M * M * S * eb);
    L.cst = take(S * S * eb);
    L.om = take(M * eb);
    L.sd = take(2 * QUAD_MAXSL * 4);
    L.se = take(2 * QUAD_MAXSL * 5 * eb);
    L.dt = take(2 * (S * S + 1) * eb);
    L.items = take(nitems * (int)sizeof(QuadItem) + (3 * QUAD_MAXS + 1) * 4);
    L.cnt = take(2 * QUAD_MAXS * 2 * 4);            // per tile parity and target: Z items, slow items present
    L.plist = take(2 * (nitems + 1) * 8);           // producer: per tile parity, count and the present items' source offsets
    L.rec = take(2 * nitems * (nF + 1) * eb);       // per tile parity: c, z[nF] of the present slow items
    o = (o + 127) / 128 * 128;
    L.ring = take(nslot * sstate * eb);
    L.z = take(sstate * eb);
    L.total = o;
    return L;
}

bool quad_build(QuadPlan &qp, const Plan &pl, const System &sys);
void quad_upload(QuadPlan &qp);
void quad_free(QuadPlan &qp);
// Returns the number of blocks (= partials written to alpha_part).
template <typename T>
int quad_launch(QuadPlan &qp, const T *x, T *y, const double *scale, double *alpha_part, cudaStream_t st);

}  // namespace nvb
