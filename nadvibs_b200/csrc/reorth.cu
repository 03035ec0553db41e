// Lanczos-vector orthogonality monitoring and partial re-orthogonalisation.
//
// Restates set_omega (Source/top.f90:844-908) and partial_orthog (Source/top.f90:910-1005),
// the partial re-orthogonalisation of H. Simon (Math. Comp. 42, 115-142, 1984):
//  * reorthog=2: omega(2,i) = <r_n, v_i> for every archived v_i (exact, not divided by beta);
//  * reorthog=1: the omega recurrence with random perturbations, and every chkorthog
//    iterations the exact overlaps replacing estimates that are smaller in magnitude;
//  * partial_orthog: intervals around |omega| >= sqrt(eps) widened to |omega| >= eps^(3/4);
//    classical Gram-Schmidt of r_n against the archived vectors of the intervals, repeated on
//    the next step, and beta(n) recomputed.
// The random draws (gauss_random, Source/function.f90:260-267) come from a seeded generator
// (the reference's random_seed() is unseeded).  The host keeps omega; overlaps and updates run
// on the device against the archive (archive.cu: device memory, or pinned host memory / a file
// streamed to the device in chunks), which must hold every Lanczos vector.
#include <cuda_runtime.h>

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

constexpr int MD_THREADS = 256;
constexpr int MD_MAXV = 16;  // archived vectors per pass

static int md_grid(long long n) {
    long long b = (n + 4 * MD_THREADS - 1) / (4 * MD_THREADS);
    if (b > 148 * 4) b = 148 * 4;
    return (int)std::max<long long>(b, 1);
}

// part[blk * nv + j] = sum_i (sq*q_i) * v_{first+j, i}
template <typename T>
__global__ void k_multi_dot(const T *__restrict__ q, double sq, const T *__restrict__ arch, long long first, int nv,
                            long long n, double *__restrict__ part) {
    double acc[MD_MAXV];
#pragma unroll
    for (int j = 0; j < MD_MAXV; ++j) acc[j] = 0.0;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const double x = (double)q[i] * sq;
#pragma unroll
        for (int j = 0; j < MD_MAXV; ++j)
            if (j < nv) acc[j] += x * (double)arch[(first + j) * n + i];
    }
    __shared__ double red[MD_THREADS];
    for (int j = 0; j < nv; ++j) {
        red[threadIdx.x] = acc[j];
        __syncthreads();
        for (int o = blockDim.x / 2; o > 0; o >>= 1) {
            if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
            __syncthreads();
        }
        if (threadIdx.x == 0) part[(long long)blockIdx.x * nv + j] = red[0];
        __syncthreads();
    }
}

// q -= sum_j c_j v_{first+j}  (q unscaled storage)
template <typename T>
__global__ void k_multi_axpy(T *__restrict__ q, const T *__restrict__ arch, long long first, int nv,
                             const double *__restrict__ c, long long n) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        double x = (double)q[i];
        for (int j = 0; j < nv; ++j) x -= c[j] * (double)arch[(first + j) * n + i];
        q[i] = (T)x;
    }
}

template <typename T>
__global__ void k_norm2(const T *__restrict__ q, long long n, double *__restrict__ part) {
    double acc = 0.0;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const double x = (double)q[i];
        acc += x * x;
    }
    __shared__ double red[MD_THREADS];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

static double uniform01(nvb_handle *h) {
    // xorshift64*, values in (0, 1]
    uint64_t x = h->rng_state ? h->rng_state : 0x9E3779B97F4A7C15ull;
    x ^= x >> 12;
    x ^= x << 25;
    x ^= x >> 27;
    h->rng_state = x;
    const uint64_t r = x * 2685821657736338717ull;
    return ((double)(r >> 11) + 1.0) / 9007199254740992.0;
}

// gauss_random (Source/function.f90:260-267): Box-Muller with the reference's formula
static double gauss(nvb_handle *h, double mean, double sigma) {
    const double r1 = uniform01(h), r2 = uniform01(h);
    return mean + sigma * std::sqrt(-2.0 * std::log(r1)) * std::cos(6.283185307179586 * r2);
}

// overlaps <s*q, v_j> for j in [lo, hi] (1-based archive indices), host result.  The archive
// is read chunk by chunk (streamed from the host or the file for those kinds); the block
// partials of every vector stay on the device until one copy at the end.
static std::vector<double> overlaps(nvb_handle *h, const void *q, double sq, int64_t lo, int64_t hi) {
    std::vector<double> out;
    if (hi < lo) return out;
    const long long n = h->ntotal();
    const int g = md_grid(n);
    const int64_t cnt = hi - lo + 1;
    ensure_partials(h, (int64_t)g * cnt);
    std::vector<std::pair<int64_t, int>> groups;  // (offset from lo, vectors) of each kernel call
    archive_for_chunks(h, lo, hi, [&](const void *base, int64_t first, int64_t count) {
        for (int64_t off = 0; off < count; off += MD_MAXV) {
            const int nv = (int)std::min<int64_t>(MD_MAXV, count - off);
            const int64_t o = first - lo + off;
            double *part = h->d_part + (size_t)o * g;
            if (h->precision == NVB_MIXED)
                k_multi_dot<float><<<g, MD_THREADS, 0, h->stream>>>((const float *)q, sq, (const float *)base, off, nv,
                                                                    n, part);
            else
                k_multi_dot<double><<<g, MD_THREADS, 0, h->stream>>>((const double *)q, sq, (const double *)base, off,
                                                                     nv, n, part);
            CK(cudaGetLastError());
            groups.push_back({o, nv});
        }
    });
    std::vector<double> part((size_t)g * cnt);
    CK(cudaMemcpyAsync(part.data(), h->d_part, part.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    out.assign(cnt, 0.0);
    for (auto &gr : groups) {
        const double *pp = part.data() + (size_t)gr.first * g;
        for (int jv = 0; jv < gr.second; ++jv) {
            double acc = 0.0;
            for (int b = 0; b < g; ++b) acc += pp[(size_t)b * gr.second + jv];
            out[gr.first + jv] = acc;
        }
    }
    return out;
}

// q -= sum_j c_j v_{lo+j}, the archive read chunk by chunk
static void subtract(nvb_handle *h, void *q, int64_t lo, const std::vector<double> &c) {
    if (c.empty()) return;
    const long long n = h->ntotal();
    ensure_partials(h, (int64_t)c.size());
    double *dc = h->d_part;  // the coefficients ride in the reduction scratch (not in use here)
    CK(cudaMemcpyAsync(dc, c.data(), c.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    archive_for_chunks(h, lo, lo + (int64_t)c.size() - 1, [&](const void *base, int64_t first, int64_t count) {
        for (int64_t off = 0; off < count; off += MD_MAXV) {
            const int nv = (int)std::min<int64_t>(MD_MAXV, count - off);
            const double *cc = dc + (first - lo) + off;
            if (h->precision == NVB_MIXED)
                k_multi_axpy<float><<<md_grid(n), MD_THREADS, 0, h->stream>>>((float *)q, (const float *)base, off, nv,
                                                                               cc, n);
            else
                k_multi_axpy<double><<<md_grid(n), MD_THREADS, 0, h->stream>>>((double *)q, (const double *)base, off,
                                                                                nv, cc, n);
            CK(cudaGetLastError());
        }
    });
    CK(cudaStreamSynchronize(h->stream));
}

static double norm_of(nvb_handle *h, const void *q) {
    const long long n = h->ntotal();
    const int g = md_grid(n);
    ensure_partials(h, g);
    if (h->precision == NVB_MIXED)
        k_norm2<float><<<g, MD_THREADS, 0, h->stream>>>((const float *)q, n, h->d_part);
    else
        k_norm2<double><<<g, MD_THREADS, 0, h->stream>>>((const double *)q, n, h->d_part);
    std::vector<double> part(g);
    CK(cudaMemcpyAsync(part.data(), h->d_part, g * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    double s = 0.0;
    for (double v : part) s += v;
    return std::sqrt(s);
}

double machine_eps_public() {
    volatile double e = 1.0;
    for (;;) {
        e = e / 2.0;
        volatile double e1 = e + 1.0;
        if (e1 == 1.0) break;
    }
    return e;
}

// omega initial values (Source/top.f90:590-594): omega(1,0)=0, omega(1,1)=1, omega(2,0)=0,
// omega(2,1) = gauss(0,0.6)*eps*nstates*dimen, omega(2,2)=1.
void reorth_init(nvb_handle *h, int64_t niter_total) {
    const double eps = machine_eps_public();
    h->omega1.assign(niter_total + 2, 0.0);
    h->omega2.assign(niter_total + 2, 0.0);
    h->omega1[1] = 1.0;
    h->omega2[1] = gauss(h, 0.0, 0.6) * eps * (double)h->sys.S * (double)h->sys.dimen;
    if (niter_total + 2 > 2) h->omega2[2] = 1.0;
    h->firststep = true;
    h->orth_ranges.clear();
    h->orth_log.clear();
}

// Called after iteration `it` (>= 2) when reorthog > 0.  State: buf[cur] = r_it (raw),
// buf[prev]*s_prev = v_it.  Updates omega, possibly r_it and beta(it) (host and device).
void reorth_after_iter(nvb_handle *h, int64_t it, int64_t niter_total) {
    const double eps = machine_eps_public();
    const double eta = std::pow(eps, 0.75);
    auto &a = h->alpha;
    auto &b = h->beta;
    auto &w1 = h->omega1;
    auto &w2 = h->omega2;
    if ((int64_t)w1.size() < niter_total + 2) w1.resize(niter_total + 2, 0.0);
    if ((int64_t)w2.size() < niter_total + 2) w2.resize(niter_total + 2, 0.0);
    const double dimtot = (double)h->sys.S * (double)h->sys.dimen;
    double sc[3];
    CK(cudaMemcpyAsync(sc, h->d_scale, sizeof sc, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    void *r = h->buf[h->cur];
    // ---- set_omega
    if (h->reorthog > 1) {
        for (int64_t i = 0; i <= it; ++i) w2[i] = 0.0;
        std::vector<double> ov = overlaps(h, r, 1.0, 1, it);
        for (int64_t i = 1; i <= it; ++i) w2[i] = ov[i - 1];
    } else {
        if (it < niter_total) w2[it + 1] = 1.0;
        w1[it] = gauss(h, 0.0, 0.6) * eps * dimtot * b[1] / b[it];
        for (int64_t k = 1; k <= it - 1; ++k)
            w1[k] = (1 / b[it]) * (b[k] * w2[k + 1] + (a[k] - a[it]) * w2[k] + b[k - 1] * w2[k - 1] - b[it - 1] * w1[k]) +
                    eps * (b[k] + b[it]) * gauss(h, 0.0, 0.3);
        for (int64_t i = 1; i <= it; ++i) std::swap(w1[i], w2[i]);
        if (it % h->chkorthog == 0 && it > 1) {
            std::vector<double> oq2 = overlaps(h, h->buf[h->prev], sc[h->prev], 1, it - 1);
            std::vector<double> oq3 = overlaps(h, r, 1.0, 1, it - 1);
            for (int64_t i = 1; i <= it - 1; ++i) {
                const double c1 = oq2[i - 1], c2 = oq3[i - 1] / b[it];
                if (std::fabs(w1[i]) < std::fabs(c1)) w1[i] = c1;
                if (std::fabs(w2[i]) < std::fabs(c2)) w2[i] = c2;
            }
        }
    }
    h->omega_pre.assign(w2.begin(), w2.begin() + it + 1);
    // ---- partial_orthog
    if (h->firststep) {
        std::vector<int64_t> oi;
        for (int64_t i = 1; i <= it; ++i)
            if (std::fabs(w2[i]) >= std::sqrt(eps)) oi.push_back(i);
        h->orth_ranges.clear();
        if (!oi.empty()) {
            std::vector<int64_t> lidx, ridx;
            for (int64_t o : oi) {
                int64_t j = o;
                for (; j >= 1; --j)
                    if (std::fabs(w2[j]) < eta) break;
                if (j < 1) j = 1;
                lidx.push_back(j);
                int64_t k = o;
                for (; k <= it; ++k)
                    if (std::fabs(w2[k]) < eta) break;
                if (k > it) k = it;
                ridx.push_back(k);
            }
            h->orth_ranges.push_back({lidx[0], ridx[0]});
            for (size_t i = 1; i < oi.size(); ++i)
                if (lidx[i] != h->orth_ranges.back().first && ridx[i] != h->orth_ranges.back().second)
                    h->orth_ranges.push_back({lidx[i], ridx[i]});
            int64_t mn = INT64_MAX;
            for (auto &pr : h->orth_ranges)
                if (pr.first > 0) mn = std::min(mn, pr.first);
            if (mn > 1) h->orth_ranges.push_back({1, 1});
        }
    }
    if (!h->orth_ranges.empty()) {
        std::vector<std::vector<double>> dots;
        for (auto &pr : h->orth_ranges) dots.push_back(overlaps(h, r, 1.0, pr.first, pr.second));
        for (size_t i = 0; i < h->orth_ranges.size(); ++i) {
            h->orth_log.push_back({it, h->orth_ranges[i].first, h->orth_ranges[i].second});
            subtract(h, r, h->orth_ranges[i].first, dots[i]);
            for (int64_t j = h->orth_ranges[i].first; j <= h->orth_ranges[i].second; ++j) w2[j] = eps * gauss(h, 0.0, 2.0);
        }
        h->firststep = !h->firststep;
        const double nb = norm_of(h, r);
        b[it] = nb;
        const double inv = nb > 0 ? 1.0 / nb : 0.0;
        CK(cudaMemcpyAsync(h->d_beta + it, &b[it], sizeof(double), cudaMemcpyHostToDevice, h->stream));
        CK(cudaMemcpyAsync(h->d_scale + h->cur, &inv, sizeof(double), cudaMemcpyHostToDevice, h->stream));
        CK(cudaStreamSynchronize(h->stream));
    }
}

}  // namespace nvb
