// Slab-tiled H.v: plan structures shared by the host planner and the kernel.
//
// The modes are split into slow modes 0..m-1 and fast modes m..M-1.  A tile is the set of
// rows with fixed slow digits p: T_F = prod(nfunc[m..M-1]) consecutive rows per state.  Every
// (term, nonzero shift) step is filed under its slow shift sigma_S; for each group the CTA
// stages the neighbour tile x(p + sigma_S) (all states it needs) in shared memory with TMA
// bulk copies and applies the group's steps, whose fast parts are shifts inside the tile.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "plan.h"

namespace nvb {

constexpr int SLAB_MAXF = 4;      // fast modes (8-bit digits packed in a uint32 per row)
constexpr int SLAB_MAXSL = 16;    // slow modes
constexpr int SLAB_RPT = 8;       // rows per thread
constexpr int SLAB_NBUF = 2;      // tile buffers (double buffering)

struct SlabStep {
    int term;                   // coefficient block
    int nslow;                  // slow factors: etab row + slow mode + shift
    short slow_mode[MAX_ORDER];
    short slow_sig[MAX_ORDER];
    int slow_etab[MAX_ORDER];   // row in the plain element table (etab) for (p, |s|)
    int nfast;
    short fast_field[MAX_ORDER];  // fast mode index j (digit field)
    int fast_row[MAX_ORDER];      // row in the fast table (zero where n+s leaves the basis)
    int stride;                   // fast shift in rows inside the tile
};

struct SlabGroup {
    short sig[SLAB_MAXSL];   // slow shift per slow mode
    long long tile_shift;    // sum sig_l * (shft_l / T_F)
    int step_begin, step_end;
    unsigned int state_mask; // source states b read by the group's steps
    int direct;              // 1: every step is a pure slow shift (no fast shift): read the
                             // neighbour tile straight from global memory, no staging
};

struct SlabDiag {            // zero-shift part of an all-even term
    int term;
    int nslow;
    short slow_mode[MAX_ORDER];
    int slow_etab[MAX_ORDER];
    int nfast;
    short fast_field[MAX_ORDER];
    int fast_row[MAX_ORDER];
};

struct SlabPlan {
    bool ok = false;
    int m = 0;                 // number of slow modes
    int nF = 0;                // number of fast modes
    long long TF = 0;          // rows per tile
    long long ntiles = 0;
    int threads = 0;
    int cols = 0;              // 1: threads = shft(m), row r = k*threads + tid, so the digit of the
                               // slowest fast mode is k and the other fast digits depend on tid only
    int frow_len = 0;          // entries per fast-table row (>= SLAB_RPT)
    int pad = 0;               // zero halo (elements) before/after each staged state tile
    long long sstate = 0;      // elements per state in a buffer: pad + TF + pad + tail
    int nfrows = 0;            // fast table rows
    std::vector<SlabStep> steps;
    std::vector<SlabGroup> groups;   // staged groups first (own tile first), then direct ones
    int nstaged = 0;
    std::vector<SlabDiag> diag;
    std::vector<double> ftab;  // [nfrows][nmax]
    std::vector<long long> slow_tshft;  // [m] shft_l / T_F
    std::vector<int> slow_nfunc;        // [m]
    std::vector<double> slow_omega;     // [m]
    std::vector<int> fast_nfunc;        // [nF]
    std::vector<long long> fast_shft;   // [nF]
    std::vector<double> fast_omega;     // [nF]
    // per-step constants (the same for every tile), read through L1 by the kernel: packed fast
    // part (stride, nfast | fields | column mask | pair mask, fast table rows) and the S x S
    // coupling block of the step's term (zero outside its state pairs)
    std::vector<int4> info;             // [nsteps]
    std::vector<double> scoef;          // [nsteps][S][S]
    // device copies
    int4 *d_info = nullptr;
    double *d_scoef = nullptr;
    float *d_scoef_f = nullptr;
    SlabStep *d_steps = nullptr;
    SlabGroup *d_groups = nullptr;
    SlabDiag *d_diag = nullptr;
    double *d_ftab = nullptr;
    float *d_ftab_f = nullptr;
    long long *d_slow_tshft = nullptr;
    int *d_slow_nfunc = nullptr;
    double *d_slow_omega = nullptr;
    float *d_slow_omega_f = nullptr;
    int *d_fast_nfunc = nullptr;
    long long *d_fast_shft = nullptr;
    double *d_fast_omega = nullptr;
    float *d_fast_omega_f = nullptr;
    int *d_err = nullptr;
    size_t smem_bytes[2] = {0, 0};  // per precision (0 = FP64, 1 = FP32)
};

// Dynamic shared-memory layout of the slab kernel (byte offsets), shared by host and device.
struct SlabLayout {
    size_t ftab, etab, sf, cg, sd, buf, total;
};
__host__ __device__ inline SlabLayout slab_layout(long long ftab_len, long long etab_len, long long nsteps,
                                                  long long ndirect, int S, int m, long long sstate, int eb) {
    SlabLayout L;
    size_t off = 64;  // mbarriers
    L.ftab = off;
    off += (size_t)ftab_len * eb;
    L.etab = off;
    off += (size_t)etab_len * eb;
    L.sf = off;
    off += (size_t)nsteps * eb;
    L.cg = off;
    off += (size_t)ndirect * S * S * eb;
    off = (off + 15) / 16 * 16;
    L.sd = off;
    off += (size_t)m * 4 + 16;
    off = (off + 127) / 128 * 128;
    L.buf = off;
    off += (size_t)SLAB_NBUF * S * sstate * eb;
    L.total = off;
    return L;
}

// Builds the slab plan; returns false (and leaves ok=false) when the system does not suit
// it (too few tiles, misaligned tiles, too many states/modes).
bool slab_build(SlabPlan &sp, const Plan &pl, const System &sys, int quirk_cubic, int elem_bytes);
void slab_upload(SlabPlan &sp);
void slab_free(SlabPlan &sp);
template <typename T>
void slab_launch(const SlabPlan &sp, const Plan &pl, const T *x, T *y, const double *scale, double *alpha_part,
                 cudaStream_t st);
size_t slab_smem(const SlabPlan &sp, const Plan &pl, int elem_bytes);

}  // namespace nvb
