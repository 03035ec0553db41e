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
// The primal vectors come back segment by segment, last segment first: the forward saves
// (v_{c-1}, v_c) every k iterations (nvb_set_checkpoints), and each segment of k iterations
// is replayed from its checkpoint with the stored alpha/beta in the handle's precision, the
// same way the two-pass Ritz vectors are rebuilt; the replay keeps v_j and w_j = H v_j of the
// segment in FP64.  The adjoint vectors and every dot product are FP64.  Device memory:
// 2 ceil(n/k) checkpoint vectors (handle precision) + (2k + 3) FP64 segment vectors + 6 FP64
// work vectors.
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

struct DevBuf {
    void *p = nullptr;
    DevBuf() = default;
    explicit DevBuf(size_t bytes) { CK(cudaMalloc(&p, bytes)); }
    ~DevBuf() {
        if (p) cudaFree(p);
    }
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
};

}  // namespace

// ---------------------------------------------------------------- checkpoints of the forward

void ckpt_reserve(nvb_handle *h, int64_t total_iters) {
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
}

// ---------------------------------------------------------------- replay

// Replays iterations from (prev = v_{c-1}, cur = v_c) in the handle's precision, writing the
// FP64 vectors v_{c-1} .. v_{last} to seg[0 .. last-c+1] and w_j = H v_j (j = c .. last-1) to
// wseg[0 .. last-c-1].  The three native buffers are scratch; the scales are host values.
static void replay_segment(nvb_handle *h, void *b3[3], double sprev, double scur, int64_t c, int64_t last,
                           double *seg, double *wseg, double *dsc) {
    const long long N = h->ntotal();
    const bool mixed = h->precision == NVB_MIXED;
    const int dt = mixed ? NVB_DTYPE_F32 : NVB_DTYPE_F64;
    int prev = 0, cur = 1, work = 2;
    auto to64 = [&](double *dst, const void *src, double sc) {
        if (mixed) k_to_f64<float><<<grid_g(N), 256, 0, h->stream>>>(dst, (const float *)src, sc, N);
        else k_to_f64<double><<<grid_g(N), 256, 0, h->stream>>>(dst, (const double *)src, sc, N);
    };
    to64(seg, b3[prev], sprev);
    for (int64_t j = c; j <= last; ++j) {
        to64(seg + (size_t)(j - c + 1) * N, b3[cur], scur);
        if (j == last) break;
        CK(cudaMemcpyAsync(dsc, &scur, sizeof(double), cudaMemcpyHostToDevice, h->stream));
        hv_any(h, b3[cur], b3[work], dt, dsc, nullptr, nullptr);
        to64(wseg + (size_t)(j - c) * N, b3[work], 1.0);  // w_j = H v_j, kept for the sweep
        if (mixed)
            k_replay<float><<<grid_g(N), 256, 0, h->stream>>>((float *)b3[work], (const float *)b3[cur],
                                                              (const float *)b3[prev], scur, sprev, h->alpha[j],
                                                              h->beta[j - 1], N);
        else
            k_replay<double><<<grid_g(N), 256, 0, h->stream>>>((double *)b3[work], (const double *)b3[cur],
                                                               (const double *)b3[prev], scur, sprev, h->alpha[j],
                                                               h->beta[j - 1], N);
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(h->stream));  // dsc is rewritten next step
        const int op = prev;
        prev = cur;
        cur = work;
        work = op;
        sprev = scur;
        scur = 1.0 / h->beta[j];
    }
    CK(cudaStreamSynchronize(h->stream));
}

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

void lanczos_backward(nvb_handle *h, int64_t n, const double *abar_in, const double *bbar_in, int64_t k,
                      double *grad) {
    if (n < 1 || n > h->iters) fail(NVB_ERR_ARG, "n must be in 1..iterations done");
    if (k < 1) fail(NVB_ERR_ARG, "checkpoint interval must be >= 1");
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
    const long long N = h->ntotal();
    const size_t per64 = (size_t)N * sizeof(double);
    const size_t per = (size_t)N * h->elem_size();
    const int64_t nc = ncoef_of(h);
    // checkpoints: the forward's when they cover iterations 1..n with interval k, else replay
    if (!(h->ck_k == k && h->ck_count >= (n + k - 1) / k && h->ck_buf)) ckpt_by_replay(h, k, n);
    const int64_t nseg = (n + k - 1) / k;
    std::vector<double> cks(2 * (size_t)nseg);
    CK(cudaMemcpy(cks.data(), h->ck_scale, cks.size() * sizeof(double), cudaMemcpyDeviceToHost));

    DevBuf segb((size_t)(k + 2) * per64), wsegb((size_t)(k + 1) * per64), b0(per), b1(per), b2(per),
        dscb(sizeof(double));
    DevBuf vbn(per64), vbc(per64), vbp(per64), rb(per64), wb(per64), w(per64);
    double *seg = (double *)segb.p, *wseg = (double *)wsegb.p;
    void *b3[3] = {b0.p, b1.p, b2.p};
    double *vb_next = (double *)vbn.p, *vb_cur = (double *)vbc.p, *vb_prev = (double *)vbp.p;
    double *rbar = (double *)rb.p, *wbar = (double *)wb.p, *wv = (double *)w.p;
    CK(cudaMemsetAsync(vb_next, 0, per64, h->stream));
    CK(cudaMemsetAsync(vb_cur, 0, per64, h->stream));
    CK(cudaMemsetAsync(vb_prev, 0, per64, h->stream));
    std::vector<double> abar(abar_in, abar_in + n), bbar(n + 1, 0.0);  // bbar[i] for beta_i, i = 0..n
    for (int64_t i = 1; i <= n; ++i) bbar[i] = bbar_in ? bbar_in[i - 1] : 0.0;
    std::fill(grad, grad + nc, 0.0);
    std::vector<double> gstep(nc);
    const int g = grid_g(N);
    auto dot = [&](const double *a, const double *b) { return device_dot(h, a, 1.0, b, 1.0, NVB_DTYPE_F64); };

    for (int64_t s = nseg - 1; s >= 0; --s) {
        const int64_t c = 1 + s * k, e = std::min(c + k - 1, n);
        // replay v_{c-1} .. v_{e+1} into seg[0 .. e-c+2]
        CK(cudaMemcpyAsync(b3[0], (char *)h->ck_buf + 2 * (size_t)s * per, per, cudaMemcpyDeviceToDevice, h->stream));
        CK(cudaMemcpyAsync(b3[1], (char *)h->ck_buf + (2 * (size_t)s + 1) * per, per, cudaMemcpyDeviceToDevice,
                           h->stream));
        replay_segment(h, b3, cks[2 * s], cks[2 * s + 1], c, e + 1, seg, wseg, (double *)dscb.p);
        auto V = [&](int64_t j) { return seg + (size_t)(j - (c - 1)) * N; };  // v_j, c-1 <= j <= e+1
        for (int64_t i = e; i >= c; --i) {
            const double al = h->alpha[i], be = h->beta[i], bprev = h->beta[i - 1];
            const double *wi = wseg + (size_t)(i - c) * N;  // w_i = H v_i from the replay
            const double btot = bbar[i] - dot(vb_next, V(i + 1)) / be;
            k_lin<<<g, 256, 0, h->stream>>>(rbar, 1.0 / be, vb_next, btot, V(i + 1), 0, N);
            const double atot = abar[i - 1] - dot(rbar, V(i));
            if (i > 1) bbar[i - 1] -= dot(rbar, V(i - 1));
            k_lin<<<g, 256, 0, h->stream>>>(vb_cur, -al, rbar, atot, wi, 1, N);
            k_lin<<<g, 256, 0, h->stream>>>(wbar, 1.0, rbar, atot, V(i), 0, N);
            if (i > 1) k_lin<<<g, 256, 0, h->stream>>>(vb_prev, -bprev, rbar, 0.0, nullptr, 1, N);
            hv_any(h, wbar, wv, NVB_DTYPE_F64, nullptr, nullptr, nullptr);  // H wbar
            k_lin<<<g, 256, 0, h->stream>>>(vb_cur, 1.0, wv, 0.0, nullptr, 1, N);
            CK(cudaGetLastError());
            hv_adjoint(h, wbar, V(i), NVB_DTYPE_F64, gstep.data());
            for (int64_t q = 0; q < nc; ++q) grad[q] += gstep[q];
            // rotate: vbar_{i+1} <- vbar_i, vbar_i <- vbar_{i-1}, vbar_{i-1} <- 0
            double *t = vb_next;
            vb_next = vb_cur;
            vb_cur = vb_prev;
            vb_prev = t;
            CK(cudaMemsetAsync(vb_prev, 0, per64, h->stream));
        }
    }
    CK(cudaStreamSynchronize(h->stream));
    check_kernel_flags(h);
}

}  // namespace nvb
