// The opaque nvb_handle: term table, device plan, Lanczos state and scratch.
#pragma once
#include <cuda_runtime.h>

#include <array>
#include <cstdio>
#include <functional>
#include <memory>
#include <string>
#include <vector>

#include "cubic.h"
#include "plan.h"
#include "quad.h"
#include "slab.h"

struct nvb_handle {
    nvb::System sys;
    nvb_options opt{};
    nvb::Plan plan;
    nvb::SlabPlan slab[2];  // slab-tiled H.v plans for FP64 (0) and FP32 (1) vectors
    nvb::QuadPlan quad;     // factorised quadratic H.v plan (both precisions)
    nvb::CubPlan cubic;     // factorised cubic H.v plan (both precisions)
    // ordr-3 Gram adjoint (adjoint.cu): its 8 x 8 MMA block list on the device, block count and grid
    void *d_g3blk = nullptr;
    int g3_nblk = 0, g3_grid = 0;
    int device = 0;
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    int precision = NVB_FP64;
    // Lanczos state.  Three device buffers hold unnormalised vectors; v = scale[i] * buf[i].
    void *buf[3] = {nullptr, nullptr, nullptr};
    int cur = 0, prev = 1, work = 2;
    int64_t iters = 0;      // completed iterations
    bool seeded = false;
    std::vector<double> seed_w;  // weights the seed was built from (replayed for Ritz vectors)
    int64_t cap = 0;        // capacity of d_alpha / d_beta (iterations)
    double *d_alpha = nullptr;  // [cap+1], alpha(i) at index i
    double *d_beta = nullptr;   // [cap+1], beta(i) at index i
    double *d_scale = nullptr;  // [3]
    int *d_status = nullptr;    // [2]: breakdown flag, iteration
    double *d_part = nullptr;   // reduction partials
    int64_t part_len = 0;
    std::vector<double> alpha, beta;  // host copies: alpha[1..iters] (alpha[0] unused), beta[0..iters]
    // archive of normalised Lanczos vectors v_1..v_k (archive.cu): device memory (arch, the
    // handle's precision), pinned host blocks, or a file in the reference's FP64 layout
    int arch_kind = 0;  // ARCH_DEVICE, ARCH_HOST, ARCH_FILE
    void *arch = nullptr;
    int64_t arch_cap = 0, arch_n = 0;
    int64_t harch_max = 0;              // capacity of the host kinds (vectors)
    std::vector<void *> harch_blocks;   // pinned blocks of whole vectors (ARCH_HOST)
    std::string arch_path;              // ARCH_FILE
    FILE *arch_file = nullptr;
    void *arch_stage[2] = {nullptr, nullptr};  // device staging ring of the streamed chunks
    void *arch_stage64 = nullptr;              // FP64 staging of the file's records
    void *arch_bounce = nullptr;               // pinned bounce buffer of the file
    cudaStream_t arch_stream = nullptr;        // copy stream of the staging ring
    cudaEvent_t arch_ready[2] = {nullptr, nullptr}, arch_free[2] = {nullptr, nullptr};
    // re-orthogonalisation
    int64_t reorthog = 0, chkorthog = 100;
    std::vector<double> omega1, omega2;  // omega(1,0:n), omega(2,0:n)
    bool firststep = true;
    std::vector<std::pair<int64_t, int64_t>> orth_ranges;
    std::vector<std::array<int64_t, 3>> orth_log;  // (iteration, lo, hi) of every Gram-Schmidt interval
    std::vector<double> omega_pre;                 // omega(2, 0:it) of the last step, before its resets
    uint64_t rng_state = 0;
    // per-phase device timing (CUDA events on the handle's stream)
    bool timing = false;
    std::vector<cudaEvent_t> ev;  // 3 per iteration of a chunk: start, after H.v, end
    double t_hv_ms = 0.0, t_iter_ms = 0.0;
    int64_t n_timed = 0;
    // checkpoints of the forward for the reverse sweep: (v_{c-1}, v_c) at iterations
    // c = 1, 1+k, 1+2k, ... in the handle's precision, and their scales
    int64_t ck_k = 0, ck_count = 0, ck_cap = 0;
    void *ck_buf = nullptr;
    double *ck_scale = nullptr;
    // full record of the forward (ck_k = -1), when it fits the backward budget: v_0 = 0,
    // v_1..v_{n+1} in native precision with their scales, so that the reverse sweep replays
    // nothing (it rebuilds w_j = H v_j from the recurrence)
    void *rec_v = nullptr;
    double *rec_vs = nullptr;
    int64_t rec_cap = 0, rec_n = 0;
    bool rec_ok = false;
    // the reverse sweep: device-memory budget for k = 0 (bytes, 0 = 85% of free memory) and
    // the last sweep's plan (top-level interval, branching, longest stored range, replayed H.v)
    int64_t grad_budget = 0;
    int64_t bw_plan[4] = {0, 0, 0, 0};
    // displaced / Duschinsky seed: <m|n> over one state block (FP64) and its norm
    double *seed_vec = nullptr;
    double seed_norm = 0.0;
    double seed_secs = 0.0;  // wall time of the last nvb_seed (the seed report's "Time Required")
    // cached scratch for ad-hoc vectors
    void *tmp = nullptr;
    size_t tmp_bytes = 0;

    size_t elem_size() const { return precision == NVB_MIXED ? sizeof(float) : sizeof(double); }
    int64_t ntotal() const { return sys.dimen * sys.S; }
};

namespace nvb {
void ensure_device(nvb_handle *h);
void lanczos_alloc(nvb_handle *h);
void lanczos_free(nvb_handle *h);
void lanczos_seed(nvb_handle *h, const double *weights);
void lanczos_run(nvb_handle *h, int64_t niter);
void hv_any(nvb_handle *h, const void *x, void *y, int dtype, const double *scale_dev, double *alpha_part,
            int *nblocks_out);
void ensure_partials(nvb_handle *h, int64_t n);
void check_kernel_flags(nvb_handle *h);
double device_dot(nvb_handle *h, const void *a, double sa, const void *b, double sb, int dtype);
// the same inner product (same kernels, same summation order) written to device memory, no
// host synchronisation
void device_dot_async(nvb_handle *h, const void *a, double sa, const void *b, double sb, int dtype, double *out_dev);
void *scratch_vector(nvb_handle *h, size_t bytes);
void grow_scalars_public(nvb_handle *h, int64_t need);
constexpr int ARCH_DEVICE = 0, ARCH_HOST = 1, ARCH_FILE = 2;
void archive_configure(nvb_handle *h, int kind, int64_t max_vectors, const char *path);
int64_t archive_capacity(const nvb_handle *h);
bool archive_holds(const nvb_handle *h, int64_t n);
void archive_free(nvb_handle *h);
void archive_ensure(nvb_handle *h, int64_t need);
void archive_push(nvb_handle *h, int64_t it);
// fn(base, first, count) over chunks of archive entries lo..hi (1-based), base = the device
// address of entry `first` (native precision) for kernels on the handle's stream
void archive_for_chunks(nvb_handle *h, int64_t lo, int64_t hi,
                        const std::function<void(const void *, int64_t, int64_t)> &fn);
void save_restart(nvb_handle *h, const char *dir, const char *vdir);
void load_restart(nvb_handle *h, const char *dir, const char *vdir);
void hv_adjoint(nvb_handle *h, const void *u, const void *v, int dtype, double *grad);
// reverse-sweep adjoint: Gram matrices accumulated on the device (length adjoint_gram_len, 0
// when the system has no Gram path), partials buffer of adjoint_gram_part_len doubles
int64_t adjoint_gram_len(const nvb_handle *h);
int64_t adjoint_gram_part_len(const nvb_handle *h);
void adjoint_gram_add(nvb_handle *h, const void *u, const void *v, int dtype, double *G, int accumulate, double *part);
// G = sum over blocks of the partials that adjoint_gram_add(..., G = nullptr, ...) accumulated
void adjoint_gram_reduce(nvb_handle *h, const double *part, double *G);
void adjoint_gram_grad(nvb_handle *h, const double *G, double *grad);
void hellmann_feynman(nvb_handle *h, int64_t nroots, double *grad, double *energies);
void displaced_seed(nvb_handle *h);
double seed_fill(nvb_handle *h, void *buf, const std::vector<double> &w);
std::vector<double> seed_weights(const nvb_handle *h);
void ckpt_reserve(nvb_handle *h, int64_t total_iters);
void ckpt_save(nvb_handle *h, int64_t it);
void rec_save_v(nvb_handle *h, int64_t it);  // the full record (checkpoint interval -1)
void rec_done(nvb_handle *h, int64_t it);
void ckpt_free(nvb_handle *h);
void lanczos_backward(nvb_handle *h, int64_t n, const double *abar, const double *bbar, int64_t k, double *grad);
int64_t ncoef_of(const nvb_handle *h);
void lead_contributors(nvb_handle *h, int64_t nroots, int64_t k, int64_t *state, int64_t *index, double *c2,
                       int64_t *phase, double *pct, const char *rootinfo);
void spin_orbit(nvb_handle *h, int64_t soroots, int64_t nroots, double *e_ev, double *amp, double *ov,
                const char *path);
void write_seed_report(nvb_handle *h, const char *path);
}  // namespace nvb
