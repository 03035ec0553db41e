// Spectrum post-step: broadening of a line spectrum (centres, heights) on a grid.  Replaces the
// reference's stand-alone broadening programs: convolve/main.f90:24-43 with sub.f90's
// gaussian (FWHM), and convolve.py:28-48 (Gaussian / Lorentzian of width sigma).
// One thread per grid point sums the lines in input order in FP64.
#include <cuda_runtime.h>

#include <cmath>
#include <string>

#include "nvb_internal.h"

namespace nvb {

#define CK(x)                                                                                    \
    do {                                                                                         \
        cudaError_t e_ = (x);                                                                    \
        if (e_ != cudaSuccess) fail(NVB_ERR_CUDA, std::string(#x ": ") + cudaGetErrorString(e_)); \
    } while (0)

constexpr int CONV_CHUNK = 1024;  // lines staged in shared memory at a time

__global__ void k_convolve(const double *__restrict__ c, const double *__restrict__ h, long long n,
                           const double *__restrict__ grid, long long ng, double width, int shape,
                           double *__restrict__ out) {
    __shared__ double sc[CONV_CHUNK], sh[CONV_CHUNK];
    const long long g = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const double x = g < ng ? grid[g] : 0.0;
    // shape 0: sub.f90's gaussian with FWHM width: sigma = fwhm / (2 sqrt(2 ln 2)),
    //          h exp(-(x-c)^2 / (2 sigma^2));
    // shape 1: convolve.py's Gaussian, h exp(-((x-c)/sigma)^2 / 2);
    // shape 2: convolve.py's Lorentzian, h / sigma / (1 + ((x-c)/sigma)^2)
    const double sigma = shape == 0 ? width / (2.0 * sqrt(2.0 * log(2.0))) : width;
    double y = 0.0;
    for (long long j0 = 0; j0 < n; j0 += CONV_CHUNK) {
        const int m = (int)(n - j0 < CONV_CHUNK ? n - j0 : CONV_CHUNK);
        __syncthreads();
        for (int i = threadIdx.x; i < m; i += blockDim.x) {
            sc[i] = c[j0 + i];
            sh[i] = h[j0 + i];
        }
        __syncthreads();
        if (g < ng) {
            if (shape == 0) {
                for (int i = 0; i < m; ++i) {
                    const double d = x - sc[i];
                    y += sh[i] * exp(-d * d / (2.0 * sigma * sigma));
                }
            } else if (shape == 1) {
                for (int i = 0; i < m; ++i) {
                    const double t = (x - sc[i]) / sigma;
                    y += sh[i] * exp(-0.5 * t * t);
                }
            } else {
                for (int i = 0; i < m; ++i) {
                    const double t = (x - sc[i]) / sigma;
                    y += sh[i] * (1.0 / sigma / (1.0 + t * t));
                }
            }
        }
    }
    if (g < ng) out[g] = y;
}

void convolve_lines(const double *c, const double *h, int64_t n, const double *grid, int64_t ng, double width,
                    int64_t shape, double *out) {
    if (n < 0 || ng < 0) fail(NVB_ERR_ARG, "negative length");
    if (shape < 0 || shape > 2) fail(NVB_ERR_ARG, "shape must be 0 (FWHM Gaussian), 1 (Gaussian) or 2 (Lorentzian)");
    if (!(width > 0.0)) fail(NVB_ERR_ARG, "width must be positive");
    if (ng == 0) return;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) fail(NVB_ERR_CUDA, "no CUDA device available");
    double *d = nullptr;
    const size_t bytes = (size_t)(2 * std::max<int64_t>(n, 1) + 2 * ng) * sizeof(double);
    CK(cudaMalloc((void **)&d, bytes));
    double *dc = d, *dh = d + std::max<int64_t>(n, 1), *dg = dh + std::max<int64_t>(n, 1), *dout = dg + ng;
    cudaError_t e = cudaSuccess;
    if (n > 0) {
        e = cudaMemcpy(dc, c, n * sizeof(double), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(dh, h, n * sizeof(double), cudaMemcpyHostToDevice);
    }
    if (e == cudaSuccess) e = cudaMemcpy(dg, grid, ng * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        k_convolve<<<(unsigned)((ng + 255) / 256), 256>>>(dc, dh, n, dg, ng, width, (int)shape, dout);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(out, dout, ng * sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) fail(NVB_ERR_CUDA, std::string("convolve: ") + cudaGetErrorString(e));
}

}  // namespace nvb
