// Measured ceilings of this GPU.
//
// Arithmetic (nvb_measure_fma): the FMA throughput of this
// GPU in FP64 and FP32, so that the H.v kernels' arithmetic side is compared with a
// measurement rather than a datasheet figure.  Each thread runs 8 independent FMA chains in
// registers (no memory traffic inside the loop); the grid fills every multiprocessor several
// times over; kernels are repeated until about `seconds` of device time have passed, timed
// with CUDA events on the handle-free default stream.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>

#include "../../include/nadvibs.h"
#include "nvb_internal.h"
#include "ring.h"

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

// Measured delivery rate of the tiled H.v kernels' data path (nvb_measure_tile_stream):
// `ctas` CTAs per multiprocessor, each a producer warp and 9 consumer warps as in the H.v kernels,
// with a ring of `slots` shared-memory slots that lane 0 of the producer fills by TMA bulk copies
// (cp.async.bulk, no multicast) of `tile_bytes` from pseudo-random tile positions of a 64 MB
// buffer (L2-resident); every consumer thread reads its share of a slot before its warp releases
// it.  No arithmetic: the rate at which whole neighbour tiles can be streamed from L2 into shared
// memory, the ceiling of the H.v kernels' item stream.  Every wait is bounded (error word).
namespace {

constexpr int TS_CONSUMERS = 288;

__global__ void __launch_bounds__(TS_CONSUMERS + 32) k_tile_stream(const unsigned char *__restrict__ src,
                                                                     unsigned ntile, int tb, int slots, int items,
                                                                     int *err, float *sink) {
    using namespace nvb::ring;
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t *full = reinterpret_cast<uint64_t *>(smem);
    uint64_t *empty = full + 16;
    volatile int *abort_flag = reinterpret_cast<volatile int *>(smem + 256);
    unsigned char *ring = smem + 512;
    const int tid = threadIdx.x, nc = TS_CONSUMERS;
    if (tid == 0) {
        for (int i = 0; i < slots; ++i) {
            mbar_init(&full[i], 1);
            mbar_init(&empty[i], (unsigned)(nc >> 5));
        }
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    fence_proxy_async();
    __syncthreads();
    const unsigned salt = blockIdx.x * 7919u + 12345u;
    if (tid >= nc) {
        if (tid == nc) {
            int slot = 0;
            unsigned ph = 0;
            long long issued = 0;
            bool stop = false;
            for (int i = 0; i < items && !stop; ++i) {
                unsigned h = salt + (unsigned)i * 104729u;  // integer hash (xorshift-multiply)
                h ^= h >> 16;
                h *= 0x7feb352du;
                h ^= h >> 15;
                h *= 0x846ca68bu;
                h ^= h >> 16;
                const unsigned t = h % ntile;
                if (mbar_wait(&empty[slot], ph ^ 1u, abort_flag)) {
                    mbar_expect_tx(&full[slot], (unsigned)tb);
                    bulk_g2s(ring + (size_t)slot * tb, src + (size_t)t * tb, (unsigned)tb, &full[slot]);
                    ++issued;
                } else {
                    stop = true;
                }
                if (++slot == slots) {
                    slot = 0;
                    ph ^= 1u;
                }
            }
            if (stop) {
                const long long n = issued < slots ? issued : slots;
                for (long long i = issued - n; i < issued; ++i) {
                    const int s2 = (int)(i % slots);
                    const unsigned p = (unsigned)((i / slots) & 1);
                    for (int w = 0; w < WAIT_LIMIT && !mbar_try(&full[s2], p); ++w) {
                    }
                }
                atomicExch(err, 1);
            }
        }
        return;
    }
    const int lane = tid & 31, nvec = tb / 16;
    float acc = 0.f;
    int slot = 0;
    unsigned ph = 0;
    for (int i = 0; i < items; ++i) {
        const bool ok = mbar_try(&full[slot], ph) || mbar_wait(&full[slot], ph, abort_flag);
        if (ok) {
            const float4 *p = reinterpret_cast<const float4 *>(ring + (size_t)slot * tb);
            for (int v = tid; v < nvec; v += nc) {
                const float4 q = p[v];
                acc += q.x + q.y + q.z + q.w;
            }
        }
        __syncwarp();
        if (lane == 0 && ok) mbar_arrive(&empty[slot]);
        if (++slot == slots) {
            slot = 0;
            ph ^= 1u;
        }
    }
    if (acc == 1234.5f) sink[blockIdx.x] = acc;  // keeps the reads live; never taken for zero data
    if (*abort_flag && tid == 0) atomicExch(err, 1);
}

}  // namespace

extern "C" int nvb_measure_tile_stream(int64_t tile_bytes, int64_t slots, int64_t ctas_per_sm, double seconds,
                                       double *bytes_per_s) {
    unsigned char *src = nullptr;
    float *sink = nullptr;
    int *err = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    auto release = [&]() {
        if (src) cudaFree(src);
        if (sink) cudaFree(sink);
        if (err) cudaFree(err);
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
    };
    try {
        if (!bytes_per_s) nvb::fail(NVB_ERR_ARG, "null argument");
        if (seconds <= 0.0) nvb::fail(NVB_ERR_ARG, "seconds <= 0");
        if (tile_bytes < 16 || tile_bytes % 16 != 0 || tile_bytes > 64 * 1024)
            nvb::fail(NVB_ERR_ARG, "tile_bytes must be a multiple of 16 in [16, 65536]");
        if (slots < 2 || slots > 16) nvb::fail(NVB_ERR_ARG, "slots must be in [2, 16]");
        if (ctas_per_sm < 1 || ctas_per_sm > 4) nvb::fail(NVB_ERR_ARG, "ctas_per_sm must be in [1, 4]");
        const size_t smem = 512 + (size_t)slots * (size_t)tile_bytes;
        if (smem * (size_t)ctas_per_sm > 227 * 1024) nvb::fail(NVB_ERR_ARG, "ring does not fit in shared memory");
        int dev = 0, nsm = 0;
        CKD(cudaGetDevice(&dev));
        CKD(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        const size_t buf = 64u << 20;
        const unsigned ntile = (unsigned)(buf / (size_t)tile_bytes);
        CKD(cudaMalloc((void **)&src, buf));
        CKD(cudaMemset(src, 0, buf));
        CKD(cudaMalloc((void **)&sink, (size_t)nsm * ctas_per_sm * sizeof(float)));
        CKD(cudaMalloc((void **)&err, sizeof(int)));
        CKD(cudaMemset(err, 0, sizeof(int)));
        CKD(cudaFuncSetAttribute(k_tile_stream, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        int per = 0;
        CKD(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_tile_stream, TS_CONSUMERS + 32, smem));
        if (per < ctas_per_sm) nvb::fail(NVB_ERR_ARG, "the requested CTAs per multiprocessor do not fit");
        const int grid = nsm * (int)ctas_per_sm;
        CKD(cudaEventCreate(&e0));
        CKD(cudaEventCreate(&e1));
        int items = 256;
        k_tile_stream<<<grid, TS_CONSUMERS + 32, smem>>>(src, ntile, (int)tile_bytes, (int)slots, items, err, sink);
        CKD(cudaGetLastError());
        CKD(cudaDeviceSynchronize());
        // size the timed launch from a short one
        CKD(cudaEventRecord(e0));
        k_tile_stream<<<grid, TS_CONSUMERS + 32, smem>>>(src, ntile, (int)tile_bytes, (int)slots, items, err, sink);
        CKD(cudaEventRecord(e1));
        CKD(cudaEventSynchronize(e1));
        float ms = 0.f;
        CKD(cudaEventElapsedTime(&ms, e0, e1));
        const double scale = seconds * 1e3 / (ms > 1e-3f ? ms : 1e-3f);
        items = (int)std::min<double>(1 << 24, std::max<double>(items, items * scale));
        CKD(cudaEventRecord(e0));
        k_tile_stream<<<grid, TS_CONSUMERS + 32, smem>>>(src, ntile, (int)tile_bytes, (int)slots, items, err, sink);
        CKD(cudaEventRecord(e1));
        CKD(cudaEventSynchronize(e1));
        CKD(cudaGetLastError());
        CKD(cudaEventElapsedTime(&ms, e0, e1));
        int e = 0;
        CKD(cudaMemcpy(&e, err, sizeof(int), cudaMemcpyDeviceToHost));
        if (e) nvb::fail(NVB_ERR_CUDA, "tile stream: a copy did not complete (the kernel gave up waiting)");
        *bytes_per_s = (double)grid * items * (double)tile_bytes / (ms * 1e-3);
        release();
        return NVB_OK;
    } catch (const nvb::Error &e) {
        release();
        nvb::set_error(e.msg);
        return e.code;
    }
}
