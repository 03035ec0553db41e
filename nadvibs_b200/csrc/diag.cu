// Measured arithmetic ceiling of the CUDA cores (nvb_measure_fma): the FMA throughput of this
// GPU in FP64 and FP32, so that the H.v kernels' arithmetic side is compared with a
// measurement rather than a datasheet figure.  Each thread runs 8 independent FMA chains in
// registers (no memory traffic inside the loop); the grid fills every multiprocessor several
// times over; kernels are repeated until about `seconds` of device time have passed, timed
// with CUDA events on the handle-free default stream.
#include <cuda_runtime.h>

#include <string>

#include "../../include/nadvibs.h"
#include "nvb_internal.h"

namespace {

constexpr int FMA_CHAINS = 8;
constexpr int FMA_THREADS = 256;

template <typename T>
__global__ void __launch_bounds__(FMA_THREADS) k_fma_loop(T *__restrict__ sink, int iters, T b, T c) {
    T a[FMA_CHAINS];
#pragma unroll
    for (int q = 0; q < FMA_CHAINS; ++q) a[q] = (T)(threadIdx.x + q) * (T)1e-3;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int q = 0; q < FMA_CHAINS; ++q) a[q] = fma(a[q], b, c);
    }
    T s = 0;
#pragma unroll
    for (int q = 0; q < FMA_CHAINS; ++q) s += a[q];
    if (s == (T)12345.678) sink[0] = s;  // keeps the chains live; never taken for these inputs
}

#define CKD(x)                                                                                        \
    do {                                                                                              \
        cudaError_t e_ = (x);                                                                         \
        if (e_ != cudaSuccess) nvb::fail(NVB_ERR_CUDA, std::string(#x ": ") + cudaGetErrorString(e_)); \
    } while (0)

template <typename T>
double measure(double seconds) {
    int dev = 0, nsm = 0;
    CKD(cudaGetDevice(&dev));
    CKD(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    const int blocks = nsm * 8, iters = 1 << 14;
    T *sink = nullptr;
    CKD(cudaMalloc((void **)&sink, sizeof(T)));
    cudaEvent_t e0, e1;
    CKD(cudaEventCreate(&e0));
    CKD(cudaEventCreate(&e1));
    const T b = (T)0.999999, c = (T)1e-7;
    k_fma_loop<T><<<blocks, FMA_THREADS>>>(sink, iters, b, c);  // warm-up
    CKD(cudaGetLastError());
    CKD(cudaDeviceSynchronize());
    // one launch's time, then enough launches for the requested duration
    CKD(cudaEventRecord(e0));
    k_fma_loop<T><<<blocks, FMA_THREADS>>>(sink, iters, b, c);
    CKD(cudaEventRecord(e1));
    CKD(cudaEventSynchronize(e1));
    float ms1 = 0.f;
    CKD(cudaEventElapsedTime(&ms1, e0, e1));
    int reps = (int)(seconds * 1e3 / (ms1 > 1e-3f ? ms1 : 1e-3f));
    if (reps < 1) reps = 1;
    if (reps > 100000) reps = 100000;
    CKD(cudaEventRecord(e0));
    for (int r = 0; r < reps; ++r) k_fma_loop<T><<<blocks, FMA_THREADS>>>(sink, iters, b, c);
    CKD(cudaEventRecord(e1));
    CKD(cudaEventSynchronize(e1));
    float ms = 0.f;
    CKD(cudaEventElapsedTime(&ms, e0, e1));
    CKD(cudaGetLastError());
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    const double flops = 2.0 * FMA_CHAINS * (double)iters * (double)blocks * FMA_THREADS * (double)reps;
    return flops / (ms * 1e-3);
}

}  // namespace

extern "C" int nvb_measure_fma(int64_t dtype, double seconds, double *flops_per_s) {
    try {
        if (!flops_per_s) nvb::fail(NVB_ERR_ARG, "null argument");
        if (seconds <= 0.0) nvb::fail(NVB_ERR_ARG, "seconds <= 0");
        if (dtype == NVB_DTYPE_F64) *flops_per_s = measure<double>(seconds);
        else if (dtype == NVB_DTYPE_F32) *flops_per_s = measure<float>(seconds);
        else nvb::fail(NVB_ERR_ARG, "bad dtype");
        return NVB_OK;
    } catch (const nvb::Error &e) {
        nvb::set_error(e.msg);
        return e.code;
    }
}
