// The Lanczos recurrence on the device.
//
// Per iteration i (reference: update_lanczos + Hv + lanczos_step, Source/top.f90:646-670,
// 672-818, 820-842), with v = scale * buffer so no normalisation pass is needed:
//   pass A  w = H v_i, with the partial sums of alpha_i = <v_i, w> fused in the H.v kernel;
//   reduce  alpha_i (fixed-order FP64 sum of the block partials);
//   pass B  r = w - alpha_i v_i - beta_{i-1} v_{i-1}, with partial sums of ||r||^2;
//   reduce  beta_i = sqrt(sum), scale(r) = 1/beta_i, breakdown check.
// The three buffers rotate (current, previous, work).  All reductions accumulate in FP64;
// in the mixed precision mode the buffers are FP32 and pass B computes in FP64 before
// rounding r to FP32 (its norm is taken from the rounded values).
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>

#include "handle.h"

namespace nvb {

#define CK(x)                                                                                    \
    do {                                                                                         \
        cudaError_t e_ = (x);                                                                    \
        if (e_ != cudaSuccess) fail(NVB_ERR_CUDA, std::string(#x ": ") + cudaGetErrorString(e_)); \
    } while (0)

template <typename T>
void hv_gather_launch(const Plan &pl, const T *x, T *y, const double *sc, double *ap, cudaStream_t st);
int hv_gather_blocks(const Plan &pl);

constexpr int RED_THREADS = 256;
constexpr int FIN_THREADS = 1024;

__device__ __forceinline__ double block_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __shared__ double red[32];
    const int tid = threadIdx.x;
    __syncthreads();
    if ((tid & 31) == 0) red[tid >> 5] = v;
    __syncthreads();
    double s = 0.0;
    if (tid < 32) {
        s = tid < (int)(blockDim.x >> 5) ? red[tid] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    }
    return s;  // valid in thread 0
}

// Fixed-order sum of partials: thread t sums t, t+1024, ..., then a tree reduction.
// mode 0: out[0] = sum.  mode 1: out[0] = sqrt(sum); scale[0] = 1/out[0]; breakdown flags.
__global__ void k_finalize(const double *__restrict__ part, int n, double *out, int mode, double *scale, int *status,
                           int iter) {
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s += part[i];
    s = block_sum(s);
    if (threadIdx.x == 0) {
        if (mode == 0) {
            out[0] = s;
            if (!isfinite(s) && status && status[0] == 0) { status[0] = 2; status[1] = iter; }
        } else {
            const double b = sqrt(s);
            out[0] = b;
            const bool bad = !(b > 1e-300) || !isfinite(b);
            if (bad && status && status[0] == 0) { status[0] = 1; status[1] = iter; }
            if (scale) scale[0] = bad ? 0.0 : 1.0 / b;
        }
    }
}

// Pass B, r = w - alpha v_i - beta_{i-1} v_{i-1} in place of w with partial sums of ||r||^2
// (FP64 arithmetic, r rounded to the buffers' type and the norm taken from the rounded values),
// with W-element vector accesses (float4 / double2: 16 bytes per load and store, so that enough
// bytes are in flight to stream at the HBM copy rate); elements beyond the last whole vector
// are done one by one.
template <typename T, typename V, int W>
__global__ void k_passB_vec(T *__restrict__ w, const T *__restrict__ c, const T *__restrict__ p,
                            const double *__restrict__ sc, const double *__restrict__ sp,
                            const double *__restrict__ alpha, const double *__restrict__ beta_prev, long long n,
                            double *__restrict__ part) {
    const double a = *alpha * *sc;
    const double b = *beta_prev * *sp;
    double acc = 0.0;
    const long long nvec = n / W;
    const long long stride = (long long)gridDim.x * blockDim.x;
    V *wv = reinterpret_cast<V *>(w);
    const V *cv = reinterpret_cast<const V *>(c);
    const V *pv = reinterpret_cast<const V *>(p);
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < nvec; i += stride) {
        V x = wv[i];
        const V y = cv[i], z = pv[i];
        T *xs = reinterpret_cast<T *>(&x);
        const T *ys = reinterpret_cast<const T *>(&y);
        const T *zs = reinterpret_cast<const T *>(&z);
#pragma unroll
        for (int q = 0; q < W; ++q) {
            double r = (double)xs[q] - a * (double)ys[q];
            r = r - b * (double)zs[q];
            const T rt = (T)r;
            xs[q] = rt;
            acc += (double)rt * (double)rt;
        }
        wv[i] = x;
    }
    for (long long i = nvec * W + (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        double r = (double)w[i] - a * (double)c[i];
        r = r - b * (double)p[i];
        const T rt = (T)r;
        w[i] = rt;
        acc += (double)rt * (double)rt;
    }
    acc = block_sum(acc);
    if (threadIdx.x == 0) part[blockIdx.x] = acc;
}

// <sa*a, sb*b> partials
template <typename T>
__global__ void k_dot(const T *__restrict__ a, const T *__restrict__ b, double sa, double sb, long long n,
                      double *__restrict__ part) {
    double acc = 0.0;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        acc += ((double)a[i] * sa) * ((double)b[i] * sb);
    acc = block_sum(acc);
    if (threadIdx.x == 0) part[blockIdx.x] = acc;
}

template <typename T>
__global__ void k_seed(T *__restrict__ v, long long dimen, int S, const double *__restrict__ w) {
    const long long n = dimen * S;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const long long s = i / dimen, r = i - s * dimen;
        v[i] = r == 0 ? (T)w[s] : (T)0;
    }
}

static int grid_for(long long n) {
    long long b = (n + RED_THREADS * 4 - 1) / (RED_THREADS * 4);
    if (b > 148 * 16) b = 148 * 16;
    if (b < 1) b = 1;
    return (int)b;
}

void ensure_partials(nvb_handle *h, int64_t n) {
    if (n <= h->part_len) return;
    if (h->d_part) cudaFree(h->d_part);
    h->d_part = nullptr;
    CK(cudaMalloc((void **)&h->d_part, (size_t)n * sizeof(double)));
    h->part_len = n;
}

void *scratch_vector(nvb_handle *h, size_t bytes) {
    if (bytes > h->tmp_bytes) {
        if (h->tmp) cudaFree(h->tmp);
        h->tmp = nullptr;
        CK(cudaMalloc(&h->tmp, bytes));
        h->tmp_bytes = bytes;
    }
    return h->tmp;
}

void hv_any(nvb_handle *h, const void *x, void *y, int dtype, const double *scale_dev, double *alpha_part,
            int *nblocks_out) {
    if (alpha_part == nullptr && nblocks_out) *nblocks_out = 0;
    const SlabPlan &sp = h->slab[dtype == NVB_DTYPE_F32 ? 1 : 0];
    const bool aligned = ((uintptr_t)x % 16) == 0;
    if (h->quad.ok && aligned) {
        int nb;
        if (dtype == NVB_DTYPE_F64)
            nb = quad_launch<double>(h->quad, (const double *)x, (double *)y, scale_dev, alpha_part, h->stream);
        else
            nb = quad_launch<float>(h->quad, (const float *)x, (float *)y, scale_dev, alpha_part, h->stream);
        CK(cudaGetLastError());
        if (nblocks_out) *nblocks_out = nb;
        return;
    }
    if (h->cubic.ok && h->cubic.prec_ok[dtype == NVB_DTYPE_F32 ? 1 : 0] && aligned) {
        int nb;
        if (dtype == NVB_DTYPE_F64)
            nb = cubic_launch<double>(h->cubic, (const double *)x, (double *)y, scale_dev, alpha_part, h->stream);
        else
            nb = cubic_launch<float>(h->cubic, (const float *)x, (float *)y, scale_dev, alpha_part, h->stream);
        CK(cudaGetLastError());
        if (nblocks_out) *nblocks_out = nb;
        return;
    }
    if (sp.ok && aligned && h->opt.hv_kernel != 1) {
        if (dtype == NVB_DTYPE_F64)
            slab_launch<double>(sp, h->plan, (const double *)x, (double *)y, scale_dev, alpha_part, h->stream);
        else
            slab_launch<float>(sp, h->plan, (const float *)x, (float *)y, scale_dev, alpha_part, h->stream);
        CK(cudaGetLastError());
        if (nblocks_out) *nblocks_out = (int)sp.ntiles;
        return;
    }
    if (dtype == NVB_DTYPE_F64)
        hv_gather_launch<double>(h->plan, (const double *)x, (double *)y, scale_dev, alpha_part, h->stream);
    else
        hv_gather_launch<float>(h->plan, (const float *)x, (float *)y, scale_dev, alpha_part, h->stream);
    CK(cudaGetLastError());
    if (nblocks_out) *nblocks_out = hv_gather_blocks(h->plan);
}

// A tiled kernel whose tile copy never completed sets its error flag and stops early.
void check_kernel_flags(nvb_handle *h) {
    if (h->quad.ok && h->quad.d_err) {
        int e = 0;
        CK(cudaMemcpy(&e, h->quad.d_err, sizeof(int), cudaMemcpyDeviceToHost));
        if (e) {
            CK(cudaMemset(h->quad.d_err, 0, sizeof(int)));  // reported once; the handle stays usable
            fail(NVB_ERR_CUDA, "quadratic H.v: a shared-memory tile copy did not complete (kernel gave up waiting)");
        }
    }
    if (h->cubic.ok && h->cubic.d_err) {
        int e = 0;
        CK(cudaMemcpy(&e, h->cubic.d_err, sizeof(int), cudaMemcpyDeviceToHost));
        if (e) {
            CK(cudaMemset(h->cubic.d_err, 0, sizeof(int)));
            fail(NVB_ERR_CUDA, "cubic H.v: a shared-memory tile copy did not complete (kernel gave up waiting)");
        }
    }
    for (int i = 0; i < 2; ++i)
        if (h->slab[i].ok && h->slab[i].d_err) {
            int e = 0;
            CK(cudaMemcpy(&e, h->slab[i].d_err, sizeof(int), cudaMemcpyDeviceToHost));
            if (e) {
                CK(cudaMemset(h->slab[i].d_err, 0, sizeof(int)));
                fail(NVB_ERR_CUDA, "slab H.v: a shared-memory tile copy did not complete (kernel gave up waiting)");
            }
        }
}

static void grow_scalars(nvb_handle *h, int64_t need) {
    if (need <= h->cap) return;
    int64_t nc = std::max<int64_t>(need, 2 * h->cap);
    double *na = nullptr, *nb = nullptr;
    CK(cudaMalloc((void **)&na, (size_t)(nc + 1) * sizeof(double)));
    CK(cudaMalloc((void **)&nb, (size_t)(nc + 1) * sizeof(double)));
    CK(cudaMemsetAsync(na, 0, (size_t)(nc + 1) * sizeof(double), h->stream));
    CK(cudaMemsetAsync(nb, 0, (size_t)(nc + 1) * sizeof(double), h->stream));
    if (h->d_alpha) {
        CK(cudaMemcpyAsync(na, h->d_alpha, (size_t)(h->cap + 1) * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
        CK(cudaMemcpyAsync(nb, h->d_beta, (size_t)(h->cap + 1) * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        cudaFree(h->d_alpha);
        cudaFree(h->d_beta);
    }
    h->d_alpha = na;
    h->d_beta = nb;
    h->cap = nc;
}

void grow_scalars_public(nvb_handle *h, int64_t need) { grow_scalars(h, need); }

void lanczos_alloc(nvb_handle *h) {
    const size_t bytes = (size_t)h->ntotal() * h->elem_size();
    for (int i = 0; i < 3; ++i) {
        if (h->buf[i]) cudaFree(h->buf[i]);
        h->buf[i] = nullptr;
        CK(cudaMalloc(&h->buf[i], bytes));
    }
    if (!h->d_scale) CK(cudaMalloc((void **)&h->d_scale, 3 * sizeof(double)));
    if (!h->d_status) CK(cudaMalloc((void **)&h->d_status, 2 * sizeof(int)));
    grow_scalars(h, 16);
    ensure_partials(h, std::max<int64_t>(hv_gather_blocks(h->plan), 148 * 16));
}

void lanczos_free(nvb_handle *h) {
    for (auto e : h->ev) cudaEventDestroy(e);
    h->ev.clear();
    for (int i = 0; i < 3; ++i)
        if (h->buf[i]) { cudaFree(h->buf[i]); h->buf[i] = nullptr; }
    if (h->d_alpha) cudaFree(h->d_alpha);
    if (h->d_beta) cudaFree(h->d_beta);
    if (h->d_scale) cudaFree(h->d_scale);
    if (h->d_status) cudaFree(h->d_status);
    if (h->d_part) cudaFree(h->d_part);
    archive_free(h);
    if (h->tmp) cudaFree(h->tmp);
    h->d_alpha = h->d_beta = h->d_scale = h->d_part = nullptr;
    h->d_status = nullptr;
    h->tmp = nullptr;
    h->cap = h->part_len = 0;
    h->tmp_bytes = 0;
}

template <typename T>
__global__ void k_seed_vec(T *__restrict__ v, const double *__restrict__ o, long long dimen, int S,
                           const double *__restrict__ q, double inv) {
    const long long n = dimen * S;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const long long s = i / dimen, r = i - s * dimen;
        v[i] = (T)(q[s] * (o[r] * inv));
    }
}

std::vector<double> seed_weights(const nvb_handle *h) {
    const int S = h->sys.S;
    if ((int)h->seed_w.size() == S) return h->seed_w;
    return std::vector<double>(h->sys.prm.weights, h->sys.prm.weights + S);
}

// The seed of generate_initialvec (Source/secondary.f90:351-783) in the handle's precision
// into buf; returns beta(0), the norm of the stored vector.  Simple branch: q3 = 0 except row 1
// of every state = 1, so d1 = sqrt(<q3,q3>/nstates) = 1.  Displaced branch (shiftref != 0):
// every state block holds <m|n> (seed.cu), d1 = sqrt(sum_n <m|n>^2).  Then state i is scaled
// by statew(i)/(sum(statew)*d1) and the vector normalised.
double seed_fill(nvb_handle *h, void *buf, const std::vector<double> &w) {
    const int S = h->sys.S;
    double wsum = 0.0;
    for (double v : w) wsum += v;
    if (wsum == 0.0) wsum = 1.0;
    std::vector<double> q(S);
    double d2 = 0.0;
    for (int s = 0; s < S; ++s) {
        q[s] = 1.0 * (w[s] / (wsum * 1.0));
        const double e = std::sqrt(q[s] * q[s]);
        d2 += e * e;
    }
    if (!(d2 > 0.0)) fail(NVB_ERR_ARG, "seed weights are all zero");
    const double scl = 1.0 / std::sqrt(d2);
    double nrm = 0.0;
    for (int s = 0; s < S; ++s) {
        q[s] *= scl;
        nrm += q[s] * q[s];
    }
    const bool mixed = h->precision == NVB_MIXED;
    if (mixed) {
        nrm = 0.0;
        for (int s = 0; s < S; ++s) nrm += (double)(float)q[s] * (double)(float)q[s];
    }
    double *dw = nullptr;
    CK(cudaMalloc((void **)&dw, S * sizeof(double)));
    CK(cudaMemcpyAsync(dw, q.data(), S * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    const long long n = h->ntotal();
    double beta0 = std::sqrt(nrm);
    if (!h->sys.neworigin) {
        if (mixed) k_seed<float><<<grid_for(n), RED_THREADS, 0, h->stream>>>((float *)buf, h->sys.dimen, S, dw);
        else k_seed<double><<<grid_for(n), RED_THREADS, 0, h->stream>>>((double *)buf, h->sys.dimen, S, dw);
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(h->stream));
    } else {
        if (!h->seed_vec) displaced_seed(h);
        if (!(h->seed_norm > 0.0)) fail(NVB_ERR_ARG, "displaced seed: the initial state has no overlap with the basis");
        const double inv = 1.0 / h->seed_norm;
        if (mixed)
            k_seed_vec<float><<<grid_for(n), RED_THREADS, 0, h->stream>>>((float *)buf, h->seed_vec, h->sys.dimen, S,
                                                                         dw, inv);
        else
            k_seed_vec<double><<<grid_for(n), RED_THREADS, 0, h->stream>>>((double *)buf, h->seed_vec, h->sys.dimen,
                                                                          S, dw, inv);
        CK(cudaGetLastError());
        beta0 = std::sqrt(device_dot(h, buf, 1.0, buf, 1.0, mixed ? NVB_DTYPE_F32 : NVB_DTYPE_F64));
    }
    cudaFree(dw);
    return beta0;
}

// generate_initialvec (Source/secondary.f90:351-783): the seed (seed_fill), v(0) = 0,
// beta(0) = ||seed||.
void lanczos_seed(nvb_handle *h, const double *weights) {
    const int S = h->sys.S;
    if (!h->buf[0]) lanczos_alloc(h);
    std::vector<double> w(S);
    for (int s = 0; s < S; ++s) w[s] = weights ? weights[s] : h->sys.prm.weights[s];
    h->seed_w = w;
    h->cur = 0; h->prev = 1; h->work = 2;
    const long long n = h->ntotal();
    const double beta0 = seed_fill(h, h->buf[h->cur], w);
    CK(cudaMemsetAsync(h->buf[h->prev], 0, (size_t)n * h->elem_size(), h->stream));
    double sc[3] = {0, 0, 0};
    sc[h->cur] = 1.0 / beta0;
    CK(cudaMemcpyAsync(h->d_scale, sc, sizeof sc, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemsetAsync(h->d_status, 0, 2 * sizeof(int), h->stream));
    CK(cudaMemsetAsync(h->d_beta, 0, sizeof(double), h->stream));
    CK(cudaMemcpyAsync(h->d_beta, &beta0, sizeof(double), cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    h->alpha.assign(1, 0.0);
    h->beta.assign(1, beta0);
    h->iters = 0;
    h->ck_count = 0;
    h->seeded = true;
    h->arch_n = 0;
    h->firststep = true;
    h->omega1.assign(1, 0.0);
    h->omega2.assign(1, 0.0);
}

template <typename T>
static void passB_launch(nvb_handle *h, int64_t it, int *blocks) {
    const long long n = h->ntotal();
    const int g = grid_for(n);
    // the three buffers are cudaMalloc'd (256-byte aligned): 16-byte vector accesses
    if constexpr (sizeof(T) == 4)
        k_passB_vec<float, float4, 4><<<g, RED_THREADS, 0, h->stream>>>(
            (float *)h->buf[h->work], (const float *)h->buf[h->cur], (const float *)h->buf[h->prev],
            h->d_scale + h->cur, h->d_scale + h->prev, h->d_alpha + it, h->d_beta + it - 1, n, h->d_part);
    else
        k_passB_vec<double, double2, 2><<<g, RED_THREADS, 0, h->stream>>>(
            (double *)h->buf[h->work], (const double *)h->buf[h->cur], (const double *)h->buf[h->prev],
            h->d_scale + h->cur, h->d_scale + h->prev, h->d_alpha + it, h->d_beta + it - 1, n, h->d_part);
    *blocks = g;
}

// One Lanczos iteration, stream-ordered, no host synchronisation.
static void lanczos_iter(nvb_handle *h, int64_t it, int slot) {
    const int dt = h->precision == NVB_MIXED ? NVB_DTYPE_F32 : NVB_DTYPE_F64;
    int nb = 0;
    ckpt_save(h, it);
    rec_save_v(h, it);
    archive_push(h, it);
    if (h->timing) CK(cudaEventRecord(h->ev[3 * slot], h->stream));
    hv_any(h, h->buf[h->cur], h->buf[h->work], dt, h->d_scale + h->cur, h->d_part, &nb);
    rec_done(h, it);  // the record holds v_it; w_it is rebuilt from the v's in the reverse sweep
    if (h->timing) CK(cudaEventRecord(h->ev[3 * slot + 1], h->stream));
    k_finalize<<<1, FIN_THREADS, 0, h->stream>>>(h->d_part, nb, h->d_alpha + it, 0, nullptr, h->d_status, (int)it);
    if (dt == NVB_DTYPE_F32) passB_launch<float>(h, it, &nb);
    else passB_launch<double>(h, it, &nb);
    k_finalize<<<1, FIN_THREADS, 0, h->stream>>>(h->d_part, nb, h->d_beta + it, 1, h->d_scale + h->work,
                                                 h->d_status, (int)it);
    CK(cudaGetLastError());
    if (h->timing) CK(cudaEventRecord(h->ev[3 * slot + 2], h->stream));
    const int old_prev = h->prev;
    h->prev = h->cur;
    h->cur = h->work;
    h->work = old_prev;
}

void reorth_after_iter(nvb_handle *h, int64_t it, int64_t niter_total);
void reorth_init(nvb_handle *h, int64_t niter_total);

// Iteration-by-iteration path of nvb_lanczos with re-orthogonalisation (set_omega +
// partial_orthog after every iteration from the second, Source/main.f90:66-69).
static void reorth_run(nvb_handle *h, int64_t niter) {
    const int64_t total = h->iters + niter;
    if (h->iters == 0) reorth_init(h, total);
    if (h->timing && h->ev.size() < 3) {
        for (auto e : h->ev) cudaEventDestroy(e);
        h->ev.assign(3, nullptr);
        for (auto &e : h->ev) CK(cudaEventCreate(&e));
    }
    for (int64_t k = 0; k < niter; ++k) {
        const int64_t it = h->iters + 1;
        lanczos_iter(h, it, 0);
        int st[2] = {0, 0};
        CK(cudaMemcpyAsync(st, h->d_status, sizeof st, cudaMemcpyDeviceToHost, h->stream));
        double ab[2];
        CK(cudaMemcpyAsync(&ab[0], h->d_alpha + it, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaMemcpyAsync(&ab[1], h->d_beta + it, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        check_kernel_flags(h);
        if (h->timing) {
            float a = 0.f, b = 0.f;
            CK(cudaEventElapsedTime(&a, h->ev[0], h->ev[1]));
            CK(cudaEventElapsedTime(&b, h->ev[0], h->ev[2]));
            h->t_hv_ms += a;
            h->t_iter_ms += b;
            h->n_timed += 1;
        }
        h->alpha.resize(it + 1);
        h->beta.resize(it + 1);
        h->alpha[it] = ab[0];
        h->beta[it] = ab[1];
        if (st[0] != 0) fail(NVB_ERR_BREAKDOWN, "Lanczos breakdown at iteration " + std::to_string(st[1]));
        h->iters = it;
        if (it > 1) reorth_after_iter(h, it, total);
    }
}

void lanczos_run(nvb_handle *h, int64_t niter) {
    if (!h->seeded) fail(NVB_ERR_STATE, "nvb_lanczos called before nvb_seed / nvb_load_restart");
    if (niter < 0) fail(NVB_ERR_ARG, "niter < 0");
    grow_scalars(h, h->iters + niter + 1);
    archive_ensure(h, h->iters + niter);
    ckpt_reserve(h, h->iters + niter);
    if (h->reorthog > 0) {
        if (archive_capacity(h) < h->iters + niter)
            fail(NVB_ERR_ARG, "re-orthogonalisation needs every Lanczos vector: give the archive room for >= " +
                                  std::to_string(h->iters + niter) +
                                  " vectors (options archive_max for device memory, or nvb_set_archive)");
        if (h->arch_n != h->iters)
            fail(NVB_ERR_STATE, "re-orthogonalisation cannot resume: the archive does not hold the earlier Lanczos "
                                "vectors (after a restart only a file archive with every earlier vector does)");
        reorth_run(h, niter);
        return;
    }
    const int64_t chunk = 64;
    int64_t done = 0;
    while (done < niter) {
        const int64_t n = std::min(chunk, niter - done);
        if (h->timing && h->ev.size() < (size_t)(3 * chunk)) {
            for (auto e : h->ev) cudaEventDestroy(e);
            h->ev.assign(3 * chunk, nullptr);
            for (auto &e : h->ev) CK(cudaEventCreate(&e));
        }
        for (int64_t k = 0; k < n; ++k) lanczos_iter(h, h->iters + done + k + 1, (int)k);
        int st[2] = {0, 0};
        CK(cudaMemcpyAsync(st, h->d_status, sizeof st, cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        check_kernel_flags(h);
        if (h->timing)
            for (int64_t k = 0; k < n; ++k) {
                float a = 0.f, b = 0.f;
                CK(cudaEventElapsedTime(&a, h->ev[3 * k], h->ev[3 * k + 1]));
                CK(cudaEventElapsedTime(&b, h->ev[3 * k], h->ev[3 * k + 2]));
                h->t_hv_ms += a;
                h->t_iter_ms += b;
                h->n_timed += 1;
            }
        done += n;
        if (st[0] != 0) {
            const int64_t total = h->iters + done;
            h->alpha.resize(total + 1);
            h->beta.resize(total + 1);
            CK(cudaMemcpy(h->alpha.data() + 1, h->d_alpha + 1, total * sizeof(double), cudaMemcpyDeviceToHost));
            CK(cudaMemcpy(h->beta.data(), h->d_beta, (total + 1) * sizeof(double), cudaMemcpyDeviceToHost));
            h->iters = st[1];
            h->alpha.resize(h->iters + 1);
            h->beta.resize(h->iters + 1);
            fail(NVB_ERR_BREAKDOWN, std::string("Lanczos breakdown at iteration ") + std::to_string(st[1]) +
                                        (st[0] == 1 ? ": beta not positive/finite" : ": alpha not finite"));
        }
    }
    h->iters += niter;
    rec_save_v(h, h->iters + 1);  // v_{n+1} of the full record
    h->alpha.resize(h->iters + 1);
    h->beta.resize(h->iters + 1);
    if (h->iters > 0) {
        CK(cudaMemcpy(h->alpha.data() + 1, h->d_alpha + 1, h->iters * sizeof(double), cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(h->beta.data(), h->d_beta, (h->iters + 1) * sizeof(double), cudaMemcpyDeviceToHost));
    }
}

void device_dot_async(nvb_handle *h, const void *a, double sa, const void *b, double sb, int dtype, double *out_dev) {
    const long long n = h->ntotal();
    const int g = grid_for(n);
    ensure_partials(h, g + 1);
    if (dtype == NVB_DTYPE_F32)
        k_dot<float><<<g, RED_THREADS, 0, h->stream>>>((const float *)a, (const float *)b, sa, sb, n, h->d_part);
    else
        k_dot<double><<<g, RED_THREADS, 0, h->stream>>>((const double *)a, (const double *)b, sa, sb, n, h->d_part);
    k_finalize<<<1, FIN_THREADS, 0, h->stream>>>(h->d_part, g, out_dev, 0, nullptr, nullptr, 0);
    CK(cudaGetLastError());
}

double device_dot(nvb_handle *h, const void *a, double sa, const void *b, double sb, int dtype) {
    const long long n = h->ntotal();
    const int g = grid_for(n);
    ensure_partials(h, g + 1);
    if (dtype == NVB_DTYPE_F32)
        k_dot<float><<<g, RED_THREADS, 0, h->stream>>>((const float *)a, (const float *)b, sa, sb, n, h->d_part);
    else
        k_dot<double><<<g, RED_THREADS, 0, h->stream>>>((const double *)a, (const double *)b, sa, sb, n, h->d_part);
    k_finalize<<<1, FIN_THREADS, 0, h->stream>>>(h->d_part, g, h->d_part + g, 0, nullptr, nullptr, 0);
    CK(cudaGetLastError());
    double r = 0.0;
    CK(cudaMemcpyAsync(&r, h->d_part + g, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return r;
}

}  // namespace nvb
