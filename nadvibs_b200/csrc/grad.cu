// Reverse-mode derivative of the Lanczos recurrence with respect to the Hamiltonian's input
// coefficients (no counterpart in the reference, which has no derivative code).
//
// Forward (Source/top.f90:646-670,820-842, as nvb_lanczos runs it, re-orthogonalisation off):
//   w_i = H v_i,  alpha_i = <v_i, w_i>,  r_i = w_i - alpha_i v_i - beta_{i-1} v_{i-1},
//   beta_i = ||r_i||,  v_{i+1} = r_i / beta_i,   v_1 = the seed (independent of theta).
// Given the adjoints abar_i = dL/dalpha_i and bbar_i = dL/dbeta_i of a loss of T_n, the
// reverse sweep i = n..1 carries vbar_{i+1}, vbar_i, vbar_{i-1}:
//   btot = bbar_i - <vbar_{i+1}, v_{i+1}> / beta_i
//   rbar = vbar_{i+1} / beta_i + btot v_{i+1}
//   atot = abar_i - <rbar, v_i>
//   bbar_{i-1} -= <rbar, v_{i-1}>,   vbar_{i-1} -= beta_{i-1} rbar
//   wbar = rbar + atot v_i,   vbar_i += -alpha_i rbar + atot w_i + H^T wbar
//   thetabar += d<wbar|H|v_i>/dtheta                                  (nvb_hv_adjoint_coeffs)
// H^T = H: the reverse sweep refuses handles whose diagonal-section couplings are applied to
// one triangle only (quirk_lower with constant or even-power inter-state couplings).
//
// The primal vectors come back range by range, last range first, by replaying the recurrence
// with the stored alpha/beta in the handle's precision (the way the two-pass Ritz vectors are
// rebuilt) from checkpoint pairs (v_{c-1}, v_c).  A range of at most bmax iterations is
// replayed into storage (v_{c-1}..v_{e+1}, native precision) and reversed; a longer range is
// split into up to B sub-ranges, one replay records their starting pairs, and they are reversed
// last-first (recursive checkpointing).  With an explicit interval k there is one level: pairs
// every k iterations (the forward's, nvb_set_checkpoints) and bmax = k.  With k = 0 the
// shallowest depth L that fits the memory budget is used (B = bmax ~ n^(1/(L+1)),
// 2 L B + bmax + 2 native vectors, L + 1 replays of the run).  No w_j = H v_j is stored: the
// step rebuilds it from the recurrence, w_j = beta_j v_{j+1} + alpha_j v_j + beta_{j-1} v_{j-1},
// from the same stored vectors in every plan (so every plan gives the same gradient).  The
// adjoint vectors and every dot product are FP64 (10 FP64 work vectors).
//
// A reverse step does not synchronise with the host: its dot products and bbar stay in device
// memory and feed the step kernels directly, and for systems with the Gram path (ordr <= 2)
// the adjoint's Gram matrices are summed on the device over all steps, the gradient being
// assembled once at the end (it is linear in them).  Cubic and quartic systems contract
// d<wbar|H|v_i>/dtheta per step on the host side of nvb_hv_adjoint_coeffs.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "handle.h"

namespace nvb {

#define CK(x)                                                                                    \
    do {                                                                                         \
        cudaError_t e_ = (x);                                                                    \
        if (e_ != cudaSuccess) fail(NVB_ERR_CUDA, std::string(#x ": ") + cudaGetErrorString(e_)); \
    } while (0)

namespace {

int grid_g(long long n) {
    long long b = (n + 1023) / 1024;
    if (b > 148 * 16) b = 148 * 16;
    return (int)std::max<long long>(b, 1);
}

__global__ void k_to_f32(float *__restrict__ dst, const double *__restrict__ src, long long n) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) dst[i] = (float)src[i];
}

// A mixed-precision handle whose FP64 products have no factorised kernel (a pencil too wide for
// the FP64 register state) while its FP32 products have one: the reverse sweep forms H wbar in
// FP32 through the factorised kernel (the forward's own precision; ~1e-7 relative per product)
// instead of the general FP64 kernel, at the cost of two FP32 work vectors.
static bool sweep_hv_f32(const nvb_handle *h) {
    if (h->precision != NVB_MIXED) return false;
    const bool f64 = h->quad.ok || (h->cubic.ok && h->cubic.prec_ok[0]);
    const bool f32 = h->quad.ok || (h->cubic.ok && h->cubic.prec_ok[1]);
    return !f64 && f32;
}

template <typename T>
__global__ void k_to_f64(double *__restrict__ dst, const T *__restrict__ src, double sc, long long n) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        dst[i] = sc * (double)src[i];
}

// out = a1 x1 + a2 x2 (acc = 0) or out += a1 x1 + a2 x2 (acc = 1); x2 may be null
__global__ void k_lin(double *__restrict__ out, double a1, const double *__restrict__ x1, double a2,
                      const double *__restrict__ x2, int acc, long long n) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        double v = a1 * x1[i];
        if (x2) v += a2 * x2[i];
        out[i] = acc ? out[i] + v : v;
    }
}

// w_i = H v_i rebuilt from the recurrence: r_i = w_i - alpha_i v_i - beta_{i-1} v_{i-1} and
// v_{i+1} = r_i / beta_i give w_i = beta_i v_{i+1} + alpha_i v_i + beta_{i-1} v_{i-1}
// (cn, cp carry the scales of the stored vectors; vp null for i = 1, where v_0 = 0)
__global__ void k_wrec(double *__restrict__ w, double cn, const double *__restrict__ vn, double al,
                       const double *__restrict__ vi, double cp, const double *__restrict__ vp, long long n) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        double v = cn * vn[i] + al * vi[i];
        if (vp) v += cp * vp[i];
        w[i] = v;
    }
}

// the replay step of the two-pass Ritz vectors: w = w - alpha sc c - beta_prev sp p
template <typename T>
__global__ void k_replay(T *__restrict__ w, const T *__restrict__ c, const T *__restrict__ p, double sc, double sp,
                         double alpha, double beta_prev, long long n) {
    const double a = alpha * sc, b = beta_prev * sp;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        double r = (double)w[i] - a * (double)c[i];
        r = r - b * (double)p[i];
        w[i] = (T)r;
    }
}

// rbar = vb_next / beta_i + btot v_{i+1},  btot = bbar_i - <vb_next, v_{i+1}> / beta_i  (bbar_i and
// the dot product read from device memory; v_{i+1} = sn * vn)
__global__ void k_rbar(double *__restrict__ rbar, const double *__restrict__ vbn, const double *__restrict__ vn,
                       double sn, double inv_be, const double *__restrict__ bbar_i, const double *__restrict__ dot1,
                       long long n) {
    const double btot = (*bbar_i - *dot1 * inv_be) * sn;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        rbar[i] = inv_be * vbn[i] + btot * vn[i];
}

// atot = abar_i - <rbar, v_i>;  vb_cur += -alpha_i rbar + atot w_i;  wbar = rbar + atot v_i;
// vb_prev += -beta_{i-1} rbar (when i > 1)
__global__ void k_step(double *__restrict__ vbc, double *__restrict__ wbar, double *__restrict__ vbp,
                       const double *__restrict__ rbar, const double *__restrict__ w, const double *__restrict__ vi,
                       double al, double abar_i, const double *__restrict__ dot2, double bprev, int has_prev,
                       long long n) {
    const double atot = abar_i - *dot2;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const double r = rbar[i];
        vbc[i] = vbc[i] + (-al * r + atot * w[i]);
        wbar[i] = 1.0 * r + atot * vi[i];
        if (has_prev) vbp[i] = vbp[i] + (-bprev * r);
    }
}

// bbar_{i-1} -= <rbar, v_{i-1}>
__global__ void k_bbar_sub(double *__restrict__ bbar, const double *__restrict__ dot3) { *bbar -= *dot3; }

struct DevBuf {
    void *p = nullptr;
    DevBuf() = default;
    explicit DevBuf(size_t bytes) {
        if (bytes) CK(cudaMalloc(&p, bytes));
    }
    ~DevBuf() {
        if (p) cudaFree(p);
    }
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
};

}  // namespace

// ---------------------------------------------------------------- checkpoints of the forward

static void rec_free(nvb_handle *h) {
    if (h->rec_v) cudaFree(h->rec_v);
    if (h->rec_vs) cudaFree(h->rec_vs);
    h->rec_v = nullptr;
    h->rec_vs = nullptr;
    h->rec_cap = h->rec_n = 0;
    h->rec_ok = false;
}

// The full record (ck_k = -1) of v_0..v_{total_iters+1}, from the seed (w_j = H v_j is rebuilt
// from them in the sweep): kept only when it and the sweep's FP64 work vectors fit the backward
// budget (nvb_set_backward_memory, default
// 85 % of the free device memory); otherwise nothing is recorded and the sweep replays.
static void rec_reserve(nvb_handle *h, int64_t total_iters) {
    if (h->iters == 0) h->rec_n = 0;
    if (h->rec_n != h->iters) {  // a record must run contiguously from the seed
        h->rec_ok = false;
        return;
    }
    if (h->rec_ok && total_iters <= h->rec_cap) return;
    const size_t per = (size_t)h->ntotal() * h->elem_size(), per64 = (size_t)h->ntotal() * sizeof(double);
    const size_t keep = h->rec_ok ? (size_t)h->rec_n : 0;
    size_t freeb = 0, totalb = 0;
    CK(cudaMemGetInfo(&freeb, &totalb));
    const double held = h->rec_ok ? (double)(h->rec_cap + 2) * (double)per : 0.0;
    const double budget = h->grad_budget > 0 ? (double)h->grad_budget : 0.85 * ((double)freeb + held);
    const double need = (double)(total_iters + 2) * (double)per + (sweep_hv_f32(h) ? 7.0 : 5.0) * (double)per +
                        10.0 * (double)per64;
    if (need > budget) {
        rec_free(h);
        return;
    }
    void *nv = nullptr;
    double *ns = nullptr;
    bool ok = cudaMalloc(&nv, (size_t)(total_iters + 2) * per) == cudaSuccess &&
              cudaMalloc((void **)&ns, (size_t)(total_iters + 2) * sizeof(double)) == cudaSuccess;
    if (!ok) {
        (void)cudaGetLastError();  // an out-of-memory return is not sticky: clear it, record nothing
        if (nv) cudaFree(nv);
        if (ns) cudaFree(ns);
        rec_free(h);
        return;
    }
    CK(cudaMemsetAsync(nv, 0, per, h->stream));  // v_0 = 0
    CK(cudaMemsetAsync(ns, 0, sizeof(double), h->stream));
    if (keep > 0) {
        CK(cudaMemcpyAsync((char *)nv + per, (char *)h->rec_v + per, (keep + 1) * per, cudaMemcpyDeviceToDevice,
                           h->stream));
        CK(cudaMemcpyAsync(ns + 1, h->rec_vs + 1, (keep + 1) * sizeof(double), cudaMemcpyDeviceToDevice,
                           h->stream));
        CK(cudaStreamSynchronize(h->stream));
    }
    const int64_t n_keep = (int64_t)keep;
    rec_free(h);
    h->rec_v = nv;
    h->rec_vs = ns;
    h->rec_cap = total_iters;
    h->rec_n = n_keep;
    h->rec_ok = true;
}

// At the start of iteration it (buffer cur = v_it with its scale): the full record's copy; after
// its H.v the record counts iteration it as done.  At the end of a run, v_{it+1}.
void rec_save_v(nvb_handle *h, int64_t it) {
    if (h->ck_k != -1 || !h->rec_ok || it > h->rec_cap + 1 || h->rec_n < it - 1) return;
    const size_t per = (size_t)h->ntotal() * h->elem_size();
    CK(cudaMemcpyAsync((char *)h->rec_v + (size_t)it * per, h->buf[h->cur], per, cudaMemcpyDeviceToDevice, h->stream));
    CK(cudaMemcpyAsync(h->rec_vs + it, h->d_scale + h->cur, sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
}

void rec_done(nvb_handle *h, int64_t it) {
    if (h->ck_k != -1 || !h->rec_ok || it > h->rec_cap || h->rec_n != it - 1) return;
    h->rec_n = it;
}

void ckpt_reserve(nvb_handle *h, int64_t total_iters) {
    if (h->ck_k == -1) {
        rec_reserve(h, total_iters);
        return;
    }
    if (h->ck_k <= 0) return;
    const int64_t need = (total_iters + h->ck_k - 1) / h->ck_k;
    if (need <= h->ck_cap) return;
    const size_t per = (size_t)h->ntotal() * h->elem_size();
    void *nb = nullptr;
    double *ns = nullptr;
    CK(cudaMalloc(&nb, 2 * (size_t)need * per));
    CK(cudaMalloc((void **)&ns, 2 * (size_t)need * sizeof(double)));
    if (h->ck_buf && h->ck_count > 0) {
        CK(cudaMemcpyAsync(nb, h->ck_buf, 2 * (size_t)h->ck_count * per, cudaMemcpyDeviceToDevice, h->stream));
        CK(cudaMemcpyAsync(ns, h->ck_scale, 2 * (size_t)h->ck_count * sizeof(double), cudaMemcpyDeviceToDevice,
                           h->stream));
        CK(cudaStreamSynchronize(h->stream));
    }
    if (h->ck_buf) cudaFree(h->ck_buf);
    if (h->ck_scale) cudaFree(h->ck_scale);
    h->ck_buf = nb;
    h->ck_scale = ns;
    h->ck_cap = need;
}

// At the start of iteration it: buffers cur = v_it, prev = v_{it-1} (scaled by d_scale).
void ckpt_save(nvb_handle *h, int64_t it) {
    if (h->ck_k <= 0 || (it - 1) % h->ck_k != 0) return;
    const int64_t c = (it - 1) / h->ck_k;
    if (c != h->ck_count || c >= h->ck_cap) return;  // only a contiguous record from the seed
    const size_t per = (size_t)h->ntotal() * h->elem_size();
    char *dst = (char *)h->ck_buf + 2 * (size_t)c * per;
    CK(cudaMemcpyAsync(dst, h->buf[h->prev], per, cudaMemcpyDeviceToDevice, h->stream));
    CK(cudaMemcpyAsync(dst + per, h->buf[h->cur], per, cudaMemcpyDeviceToDevice, h->stream));
    CK(cudaMemcpyAsync(h->ck_scale + 2 * c, h->d_scale + h->prev, sizeof(double), cudaMemcpyDeviceToDevice,
                       h->stream));
    CK(cudaMemcpyAsync(h->ck_scale + 2 * c + 1, h->d_scale + h->cur, sizeof(double), cudaMemcpyDeviceToDevice,
                       h->stream));
    h->ck_count = c + 1;
}

void ckpt_free(nvb_handle *h) {
    if (h->ck_buf) cudaFree(h->ck_buf);
    if (h->ck_scale) cudaFree(h->ck_scale);
    h->ck_buf = nullptr;
    h->ck_scale = nullptr;
    h->ck_cap = h->ck_count = 0;
    rec_free(h);
}

// ---------------------------------------------------------------- replay

// The seed vector in native precision into buf (as lanczos_seed builds it); returns its scale.
static double seed_native(nvb_handle *h, void *buf) {
    seed_fill(h, buf, seed_weights(h));
    return 1.0 / h->beta[0];
}

// Builds the checkpoints of iterations 1, 1+k, ... <= n by replaying from the seed (when the
// forward did not record them).
static void ckpt_by_replay(nvb_handle *h, int64_t k, int64_t n) {
    if (h->ck_k != k) ckpt_free(h);
    h->ck_k = k;
    h->ck_count = 0;
    ckpt_reserve(h, n);
    const long long N = h->ntotal();
    const size_t per = (size_t)N * h->elem_size();
    const bool mixed = h->precision == NVB_MIXED;
    const int dt = mixed ? NVB_DTYPE_F32 : NVB_DTYPE_F64;
    DevBuf b0(per), b1(per), b2(per), dscb(sizeof(double));
    void *b3[3] = {b0.p, b1.p, b2.p};
    double *dsc = (double *)dscb.p;
    int prev = 0, cur = 1, work = 2;
    CK(cudaMemsetAsync(b3[prev], 0, per, h->stream));
    double sprev = 0.0, scur = seed_native(h, b3[cur]);
    for (int64_t j = 1; j <= n; ++j) {
        if ((j - 1) % k == 0) {
            const int64_t c = (j - 1) / k;
            char *dst = (char *)h->ck_buf + 2 * (size_t)c * per;
            CK(cudaMemcpyAsync(dst, b3[prev], per, cudaMemcpyDeviceToDevice, h->stream));
            CK(cudaMemcpyAsync(dst + per, b3[cur], per, cudaMemcpyDeviceToDevice, h->stream));
            const double sc2[2] = {sprev, scur};
            CK(cudaMemcpyAsync(h->ck_scale + 2 * c, sc2, sizeof sc2, cudaMemcpyHostToDevice, h->stream));
            CK(cudaStreamSynchronize(h->stream));
            h->ck_count = c + 1;
        }
        if (j == n) break;
        CK(cudaMemcpyAsync(dsc, &scur, sizeof(double), cudaMemcpyHostToDevice, h->stream));
        hv_any(h, b3[cur], b3[work], dt, dsc, nullptr, nullptr);
        if (mixed)
            k_replay<float><<<grid_g(N), 256, 0, h->stream>>>((float *)b3[work], (const float *)b3[cur],
                                                              (const float *)b3[prev], scur, sprev, h->alpha[j],
                                                              h->beta[j - 1], N);
        else
            k_replay<double><<<grid_g(N), 256, 0, h->stream>>>((double *)b3[work], (const double *)b3[cur],
                                                               (const double *)b3[prev], scur, sprev, h->alpha[j],
                                                               h->beta[j - 1], N);
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(h->stream));
        const int op = prev;
        prev = cur;
        cur = work;
        work = op;
        sprev = scur;
        scur = 1.0 / h->beta[j];
    }
}

// ---------------------------------------------------------------- the reverse sweep

namespace {

// A checkpoint pair (v_{c-1}, v_c) in native buffers with their scales.
struct CkPair {
    const void *prev, *cur;
    double sprev, scur;
};

struct Sweep {
    nvb_handle *h = nullptr;
    long long N = 0;
    size_t per = 0, per64 = 0;
    bool mixed = false;
    int dt = NVB_DTYPE_F64, g = 1;
    int64_t n = 0, B = 2, bmax = 1;  // branching of a level, longest range reversed from storage
    void *b3[3] = {nullptr, nullptr, nullptr};
    void *segv = nullptr;                    // native v_{c-1}..v_{e+1} of a base range
    std::vector<double> segs;                // their scales
    double *vb_next = nullptr, *vb_cur = nullptr, *vb_prev = nullptr, *rbar = nullptr, *wbar = nullptr,
           *wv = nullptr, *v64[3] = {nullptr, nullptr, nullptr}, *w64 = nullptr;
    float *w32a = nullptr, *w32b = nullptr;  // H wbar in FP32 (sweep_hv_f32)
    std::vector<double> abar, bbar, gstep;
    double *grad = nullptr;
    int64_t nc = 0, replayed = 0;  // H.v applications of the replays
    // device-side scalars of the reverse step (no host synchronisation inside a step): bbar,
    // the step's three dot products, the replay's scales; the accumulated adjoint Gram
    // matrices when the system has the Gram path (else the per-step host adjoint)
    double *d_bbar = nullptr, *d_dots = nullptr, *d_rscal = nullptr, *G = nullptr, *gpart = nullptr;
    bool gram_started = false;

    void to64(double *dst, const void *src, double sc) {
        if (mixed) k_to_f64<float><<<g, 256, 0, h->stream>>>(dst, (const float *)src, sc, N);
        else k_to_f64<double><<<g, 256, 0, h->stream>>>(dst, (const double *)src, sc, N);
    }
    void *nat(void *base, int64_t i) { return (char *)base + (size_t)i * per; }

    // Replays iterations c..last from P: on_v(j, prev, sprev, cur, scur) at every j, and
    // on_w(j, w) with w = H v_j (native) for j < last.
    template <typename FV, typename FW>
    void replay(const CkPair &P, int64_t c, int64_t last, FV on_v, FW on_w) {
        // the scale of the current vector at each step, uploaded once
        std::vector<double> scal((size_t)(last - c + 1));
        scal[0] = P.scur;
        for (int64_t j = c + 1; j <= last; ++j) scal[(size_t)(j - c)] = 1.0 / h->beta[j - 1];
        // stream-ordered: the previous replay's H.v launches read the old scales first
        CK(cudaMemcpyAsync(d_rscal, scal.data(), scal.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        CK(cudaMemcpyAsync(b3[0], P.prev, per, cudaMemcpyDeviceToDevice, h->stream));
        CK(cudaMemcpyAsync(b3[1], P.cur, per, cudaMemcpyDeviceToDevice, h->stream));
        int prev = 0, cur = 1, work = 2;
        double sprev = P.sprev, scur = P.scur;
        for (int64_t j = c; j <= last; ++j) {
            on_v(j, b3[prev], sprev, b3[cur], scur);
            if (j == last) break;
            hv_any(h, b3[cur], b3[work], dt, d_rscal + (j - c), nullptr, nullptr);
            ++replayed;
            on_w(j, b3[work]);
            if (mixed)
                k_replay<float><<<g, 256, 0, h->stream>>>((float *)b3[work], (const float *)b3[cur],
                                                          (const float *)b3[prev], scur, sprev, h->alpha[j],
                                                          h->beta[j - 1], N);
            else
                k_replay<double><<<g, 256, 0, h->stream>>>((double *)b3[work], (const double *)b3[cur],
                                                           (const double *)b3[prev], scur, sprev, h->alpha[j],
                                                           h->beta[j - 1], N);
            CK(cudaGetLastError());
            const int op = prev;
            prev = cur;
            cur = work;
            work = op;
            sprev = scur;
            scur = 1.0 / h->beta[j];
        }
    }

    // reverse steps e..c of a range whose v_{c-1}..v_{e+1} are in segv (w_i rebuilt from them)
    void reverse_steps(int64_t c, int64_t e) {
        auto V = [&](int64_t j, double *dst) { to64(dst, nat(segv, j - (c - 1)), segs[j - (c - 1)]); };
        for (int64_t i = e; i >= c; --i) {
            const double al = h->alpha[i], be = h->beta[i], bprev = h->beta[i - 1];
            // v_{i+1} and v_{i-1} are read where they are stored (FP64 handles: the stored vector
            // and its scale, no copy); v_i, which the adjoint contraction also reads, and
            // everything of a mixed handle are widened to FP64 first
            const double *vn = v64[0], *vp = v64[2], *wi = w64, *vi = v64[1];
            double sn = 1.0, sp = 1.0;
            if (mixed) {
                V(i + 1, v64[0]);
                if (i > 1) V(i - 1, v64[2]);
            } else {
                vn = (const double *)nat(segv, i + 1 - (c - 1));
                sn = segs[i + 1 - (c - 1)];
                if (i > 1) {
                    vp = (const double *)nat(segv, i - 1 - (c - 1));
                    sp = segs[i - 1 - (c - 1)];
                }
            }
            V(i, v64[1]);
            k_wrec<<<g, 256, 0, h->stream>>>(w64, be * sn, vn, al, vi, bprev * sp, i > 1 ? vp : nullptr, N);
            device_dot_async(h, vb_next, 1.0, vn, sn, NVB_DTYPE_F64, d_dots);
            k_rbar<<<g, 256, 0, h->stream>>>(rbar, vb_next, vn, sn, 1.0 / be, d_bbar + i, d_dots, N);
            device_dot_async(h, rbar, 1.0, vi, 1.0, NVB_DTYPE_F64, d_dots + 1);
            if (i > 1) {
                device_dot_async(h, rbar, 1.0, vp, sp, NVB_DTYPE_F64, d_dots + 2);
                k_bbar_sub<<<1, 1, 0, h->stream>>>(d_bbar + i - 1, d_dots + 2);
            }
            k_step<<<g, 256, 0, h->stream>>>(vb_cur, wbar, vb_prev, rbar, wi, vi, al, abar[i - 1], d_dots + 1, bprev,
                                             i > 1 ? 1 : 0, N);
            if (w32a) {  // H wbar through the FP32 factorised kernel
                k_to_f32<<<g, 256, 0, h->stream>>>(w32a, wbar, N);
                hv_any(h, w32a, w32b, NVB_DTYPE_F32, nullptr, nullptr, nullptr);
                k_to_f64<float><<<g, 256, 0, h->stream>>>(wv, w32b, 1.0, N);
            } else {
                hv_any(h, wbar, wv, NVB_DTYPE_F64, nullptr, nullptr, nullptr);  // H wbar
            }
            k_lin<<<g, 256, 0, h->stream>>>(vb_cur, 1.0, wv, 0.0, nullptr, 1, N);
            CK(cudaGetLastError());
            if (G) {
                // per-block partials summed over the sweep; one reduction at the end
                adjoint_gram_add(h, wbar, vi, NVB_DTYPE_F64, nullptr, gram_started ? 1 : 0, gpart);
                gram_started = true;
            } else {
                hv_adjoint(h, wbar, vi, NVB_DTYPE_F64, gstep.data());
                for (int64_t q = 0; q < nc; ++q) grad[q] += gstep[q];
            }
            // rotate: vbar_{i+1} <- vbar_i, vbar_i <- vbar_{i-1}, vbar_{i-1} <- 0
            double *t = vb_next;
            vb_next = vb_cur;
            vb_cur = vb_prev;
            vb_prev = t;
            CK(cudaMemsetAsync(vb_prev, 0, per64, h->stream));
        }
    }

    // Reverses iterations c..e given the pair at c.  Ranges up to bmax are replayed into the
    // base storage; longer ones are split into up to B sub-ranges whose starting pairs one
    // replay records, and reversed last-first.
    void reverse_range(const CkPair &P, int64_t c, int64_t e) {
        const int64_t len = e - c + 1;
        if (len <= bmax) {
            replay(
                P, c, e + 1,
                [&](int64_t j, const void *pv, double sp, const void *cv, double sc) {
                    if (j == c) {
                        CK(cudaMemcpyAsync(nat(segv, 0), pv, per, cudaMemcpyDeviceToDevice, h->stream));
                        segs[0] = sp;
                    }
                    CK(cudaMemcpyAsync(nat(segv, j - c + 1), cv, per, cudaMemcpyDeviceToDevice, h->stream));
                    segs[j - c + 1] = sc;
                },
                [&](int64_t, const void *) {});
            reverse_steps(c, e);
            return;
        }
        const int64_t sub = (len + B - 1) / B, nsub = (len + sub - 1) / sub;
        DevBuf store(2 * (size_t)nsub * per);
        std::vector<double> sc(2 * (size_t)nsub);
        replay(
            P, c, c + (nsub - 1) * sub,
            [&](int64_t j, const void *pv, double sp, const void *cv, double scv) {
                if ((j - c) % sub) return;
                const int64_t t = (j - c) / sub;
                CK(cudaMemcpyAsync(nat(store.p, 2 * t), pv, per, cudaMemcpyDeviceToDevice, h->stream));
                CK(cudaMemcpyAsync(nat(store.p, 2 * t + 1), cv, per, cudaMemcpyDeviceToDevice, h->stream));
                sc[2 * t] = sp;
                sc[2 * t + 1] = scv;
            },
            [&](int64_t, const void *) {});
        for (int64_t t = nsub - 1; t >= 0; --t) {
            const CkPair Q{nat(store.p, 2 * t), nat(store.p, 2 * t + 1), sc[2 * t], sc[2 * t + 1]};
            reverse_range(Q, c + t * sub, std::min(c + (t + 1) * sub - 1, e));
        }
    }
};

}  // namespace

// Levels of the recursion for n iterations when `vectors` native vectors are available for
// the pair stores and the base range: depth L (0 = one base range), branching B, base bmax.
static bool plan_levels(int64_t n, double vectors, int64_t *L, int64_t *B, int64_t *bmax) {
    for (int64_t l = 0; l <= 12; ++l) {
        int64_t b = (int64_t)std::ceil(std::pow((double)n, 1.0 / (double)(l + 1)) - 1e-9);
        b = std::max<int64_t>(b, 2);
        while (b > 2) {  // the smallest b with b^(l+1) >= n
            double p = 1.0;
            for (int64_t q = 0; q <= l; ++q) p *= (double)(b - 1);
            if (p >= (double)n) --b;
            else break;
        }
        const int64_t base = l == 0 ? n : b;
        const double need = 2.0 * (double)l * (double)b + (double)base + 2.0;
        if (need <= vectors) {
            *L = l;
            *B = b;
            *bmax = base;
            return true;
        }
    }
    return false;
}

void lanczos_backward(nvb_handle *h, int64_t n, const double *abar_in, const double *bbar_in, int64_t k,
                      double *grad) {
    if (n < 1 || n > h->iters) fail(NVB_ERR_ARG, "n must be in 1..iterations done");
    if (k < -1) fail(NVB_ERR_ARG, "checkpoint interval must be >= -1 (0 = automatic, -1 = the forward's full record)");
    // the forward's full record, when it was kept and covers n: nothing is replayed
    const bool from_record = k == -1 && h->ck_k == -1 && h->rec_ok && h->rec_n >= n;
    if (k == -1 && !from_record) k = 0;  // no record (it did not fit): the automatic plan
    if (h->reorthog > 0) fail(NVB_ERR_STATE, "the reverse sweep differentiates plain Lanczos (reorthog = 0)");
    if (!(h->beta[n] > 0.0)) fail(NVB_ERR_STATE, "beta_n is zero: v_{n+1} does not exist");
    {
        const int S = h->sys.S;
        for (int a = 0; a < S; ++a)
            for (int b = 0; b < S; ++b)
                if (h->plan.h_dpair[a * S + b] != h->plan.h_dpair[b * S + a])
                    fail(NVB_ERR_STATE, "H is not symmetric (quirk_lower with inter-state constant or even-power "
                                        "couplings): the reverse sweep needs H^T = H");
    }
    Sweep W;
    W.h = h;
    W.n = n;
    W.N = h->ntotal();
    W.per = (size_t)W.N * h->elem_size();
    W.per64 = (size_t)W.N * sizeof(double);
    W.mixed = h->precision == NVB_MIXED;
    W.dt = W.mixed ? NVB_DTYPE_F32 : NVB_DTYPE_F64;
    W.g = grid_g(W.N);
    W.nc = ncoef_of(h);
    // the plan.  An explicit k is one level: pairs every k iterations (the forward's record, else
    // one replay from the seed) and bmax = k.  k = 0 picks the shallowest recursion that fits the
    // memory budget, over the forward's pairs when they were recorded, else from the seed.
    int64_t top = 0;  // interval of the top-level pairs in h->ck_buf, 0 = start from the seed pair
    if (from_record) {
        W.B = 1;
        W.bmax = n;
    } else if (k > 0) {
        W.bmax = std::min(k, n);
        W.B = (n + W.bmax - 1) / W.bmax;  // ranges of the one level
        top = n > k ? k : 0;
        if (top && !(h->ck_k == top && h->ck_count >= (n + top - 1) / top && h->ck_buf)) {
            ckpt_by_replay(h, top, n);
            W.replayed += n - 1;
        }
    } else {
        const bool fwd = h->ck_k > 0 && h->ck_k < n && h->ck_buf && h->ck_count >= (n + h->ck_k - 1) / h->ck_k;
        const int64_t span = fwd ? h->ck_k : n;
        size_t freeb = 0, totalb = 0;
        CK(cudaMemGetInfo(&freeb, &totalb));
        const double budget = h->grad_budget > 0 ? (double)h->grad_budget : 0.85 * (double)freeb;
        const double fixed = (sweep_hv_f32(h) ? 7.0 : 5.0) * (double)W.per + 10.0 * (double)W.per64;
        int64_t L = 0;
        if (!plan_levels(span, (budget - fixed) / (double)W.per, &L, &W.B, &W.bmax))
            fail(NVB_ERR_NOMEM, "the reverse sweep does not fit the device-memory budget");
        top = fwd ? h->ck_k : 0;
    }
    h->bw_plan[0] = top;
    h->bw_plan[1] = W.B;
    h->bw_plan[2] = W.bmax;
    // base storage and work vectors (no base storage when the forward's record is the base range)
    const size_t nbase = from_record ? 0 : 1;
    DevBuf segv(nbase * (size_t)(W.bmax + 2) * W.per), b0(nbase * W.per), b1(nbase * W.per), b2(nbase * W.per);
    DevBuf vbn(W.per64), vbc(W.per64), vbp(W.per64), rb(W.per64), wb(W.per64), wvb(W.per64), c0(W.per64),
        c1(W.per64), c2(W.per64), cw(W.per64);
    const bool h32 = sweep_hv_f32(h);
    DevBuf w32a(h32 ? W.per : 0), w32b(h32 ? W.per : 0);
    W.w32a = (float *)w32a.p;
    W.w32b = (float *)w32b.p;
    W.segv = segv.p;
    W.segs.assign(W.bmax + 2, 0.0);
    W.b3[0] = b0.p;
    W.b3[1] = b1.p;
    W.b3[2] = b2.p;
    W.vb_next = (double *)vbn.p;
    W.vb_cur = (double *)vbc.p;
    W.vb_prev = (double *)vbp.p;
    W.rbar = (double *)rb.p;
    W.wbar = (double *)wb.p;
    W.wv = (double *)wvb.p;
    W.v64[0] = (double *)c0.p;
    W.v64[1] = (double *)c1.p;
    W.v64[2] = (double *)c2.p;
    W.w64 = (double *)cw.p;
    CK(cudaMemsetAsync(W.vb_next, 0, W.per64, h->stream));
    CK(cudaMemsetAsync(W.vb_cur, 0, W.per64, h->stream));
    CK(cudaMemsetAsync(W.vb_prev, 0, W.per64, h->stream));
    W.abar.assign(abar_in, abar_in + n);
    W.bbar.assign(n + 1, 0.0);  // bbar[i] for beta_i, i = 0..n
    for (int64_t i = 1; i <= n; ++i) W.bbar[i] = bbar_in ? bbar_in[i - 1] : 0.0;
    const int64_t glen = adjoint_gram_len(h), gplen = adjoint_gram_part_len(h);
    DevBuf dscal((size_t)(2 * (n + 1) + 3) * sizeof(double)), gbuf((size_t)std::max<int64_t>(1, glen + gplen) * sizeof(double));
    W.d_bbar = (double *)dscal.p;
    W.d_rscal = W.d_bbar + (n + 1);
    W.d_dots = W.d_rscal + (n + 1);
    CK(cudaMemcpyAsync(W.d_bbar, W.bbar.data(), (n + 1) * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    if (glen > 0) {
        W.G = (double *)gbuf.p;
        W.gpart = W.G + glen;
        CK(cudaMemsetAsync(W.gpart, 0, (size_t)gplen * sizeof(double), h->stream));
    }
    W.grad = grad;
    std::fill(grad, grad + W.nc, 0.0);
    W.gstep.assign(W.nc, 0.0);
    if (from_record) {
        // the base range 1..n straight from the record: v_j in slot j
        W.segv = h->rec_v;
        CK(cudaMemcpyAsync(W.segs.data(), h->rec_vs, (size_t)(n + 2) * sizeof(double), cudaMemcpyDeviceToHost,
                           h->stream));
        CK(cudaStreamSynchronize(h->stream));
        W.segs[0] = 0.0;
        W.reverse_steps(1, n);
    } else if (top == 0) {
        // from the seed pair (v_0 = 0, v_1 = the seed)
        DevBuf zero(W.per), seed(W.per);
        CK(cudaMemsetAsync(zero.p, 0, W.per, h->stream));
        seed_fill(h, seed.p, seed_weights(h));
        W.reverse_range(CkPair{zero.p, seed.p, 0.0, 1.0 / h->beta[0]}, 1, n);
    } else {
        const int64_t nseg = (n + top - 1) / top;
        std::vector<double> cks(2 * (size_t)nseg);
        CK(cudaMemcpy(cks.data(), h->ck_scale, cks.size() * sizeof(double), cudaMemcpyDeviceToHost));
        for (int64_t s2 = nseg - 1; s2 >= 0; --s2) {
            const CkPair P{(char *)h->ck_buf + 2 * (size_t)s2 * W.per, (char *)h->ck_buf + (2 * (size_t)s2 + 1) * W.per,
                         cks[2 * s2], cks[2 * s2 + 1]};
            W.reverse_range(P, 1 + s2 * top, std::min((s2 + 1) * top, n));
        }
    }
    if (W.G) {
        adjoint_gram_reduce(h, W.gpart, W.G);  // the Gram matrices summed over all steps
        adjoint_gram_grad(h, W.G, grad);       // and the gradient they give (linear in them)
    }
    CK(cudaStreamSynchronize(h->stream));
    h->bw_plan[3] = W.replayed;
    check_kernel_flags(h);
}

}  // namespace nvb
