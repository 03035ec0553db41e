// Allocation-free inner product (nvb_dot_noalloc).
//
// Some callers cannot allocate device memory: a host program whose GPU memory is owned by
// its own pool allocator (it reserved the device's memory up front and hands out slices),
// or a driver loop that must not call cudaMalloc/cudaFree because those may synchronise the
// device.  For them this entry point computes <sa*a, sb*b> with its block partials in a
// static device array compiled into this library instead of cudaMalloc'd scratch.  The
// caller passes the inputs and a device pointer for the result; nothing is allocated.
//
// Limits and sharing:
//  * one partial per block of 2^20 elements, at most 4096 blocks: n <= 2^32 elements
//    (the array is 4097 doubles, about 32 KiB, held by every GPU that loads the library
//    until the process exits);
//  * every call, on every stream, uses the same array; each call overwrites the partials it
//    uses before reading them, so no clearing is needed, but calls that overlap on the GPU
//    race with each other and must be ordered by the caller (same stream or events);
//  * the first call on a device looks up the array's device address with
//    cudaGetSymbolAddress (once per device, with that device current); make that first
//    call before any stream capture.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/nadvibs.h"
#include "nvb_internal.h"

namespace {

constexpr long long NOALLOC_CHUNK = 1ll << 20;  // elements per block
constexpr int NOALLOC_MAX_BLOCKS = 4096;        // => n <= 2^32
constexpr int NOALLOC_THREADS = 256;
constexpr int NOALLOC_MAX_DEVICES = 64;

// Partials [0, nblocks) of the current call.  Host code never touches this symbol directly:
// in host code the name is only a stand-in, so kernels get its address from
// cudaGetSymbolAddress.
static __device__ __align__(256) double g_noalloc_partials[NOALLOC_MAX_BLOCKS + 1];

double *g_scratch_dev[NOALLOC_MAX_DEVICES] = {};
std::mutex g_mu;

double *scratch_for_current_device() {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) nvb::fail(NVB_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) nvb::fail(NVB_ERR_ARG, "device ordinal beyond 63");
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_dev[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_partials);
        if (e != cudaSuccess || !p)
            nvb::fail(NVB_ERR_CUDA, std::string("cudaGetSymbolAddress of the static scratch array: ") +
                                        cudaGetErrorString(e));
        g_scratch_dev[dev] = static_cast<double *>(p);
    }
    return g_scratch_dev[dev];
}

__device__ __forceinline__ double block_sum_na(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __shared__ double red[32];
    const int tid = threadIdx.x;
    if ((tid & 31) == 0) red[tid >> 5] = v;
    __syncthreads();
    double s = 0.0;
    if (tid < 32) {
        s = tid < (int)(blockDim.x >> 5) ? red[tid] : 0.0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    }
    return s;
}

template <typename T>
__global__ void k_dot_chunks(const T *__restrict__ a, const T *__restrict__ b, double sa, double sb, long long n,
                             double *__restrict__ partials) {
    const long long beg = (long long)blockIdx.x * NOALLOC_CHUNK;
    const long long end = beg + NOALLOC_CHUNK < n ? beg + NOALLOC_CHUNK : n;
    double acc = 0.0;
    for (long long i = beg + threadIdx.x; i < end; i += blockDim.x) acc += ((double)a[i] * sa) * ((double)b[i] * sb);
    acc = block_sum_na(acc);
    if (threadIdx.x == 0) partials[blockIdx.x] = acc;
}

__global__ void k_dot_final(const double *__restrict__ partials, int nb, double *__restrict__ out) {
    double s = 0.0;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) s += partials[i];
    s = block_sum_na(s);
    if (threadIdx.x == 0) *out = s;
}

}  // namespace

extern "C" int nvb_dot_noalloc(const void *a, double sa, const void *b, double sb, int64_t n, int64_t dtype,
                               double *result_dev, void *stream) {
    try {
        if (!a || !b || !result_dev) nvb::fail(NVB_ERR_ARG, "null argument");
        if (dtype != NVB_DTYPE_F64 && dtype != NVB_DTYPE_F32) nvb::fail(NVB_ERR_ARG, "bad dtype");
        if (n < 0) nvb::fail(NVB_ERR_ARG, "n < 0");
        if (n > (long long)NOALLOC_MAX_BLOCKS * NOALLOC_CHUNK)
            nvb::fail(NVB_ERR_ARG, "n = " + std::to_string(n) +
                                       " exceeds the maximum of the allocation-free dot product, 2^32 elements "
                                       "(4096 blocks of 2^20 elements in its static scratch array)");
        double *part = scratch_for_current_device();
        cudaStream_t st = (cudaStream_t)stream;
        const int nb = (int)((n + NOALLOC_CHUNK - 1) / NOALLOC_CHUNK);
        if (nb > 0) {
            if (dtype == NVB_DTYPE_F64)
                k_dot_chunks<double><<<nb, NOALLOC_THREADS, 0, st>>>((const double *)a, (const double *)b, sa, sb, n,
                                                                     part);
            else
                k_dot_chunks<float><<<nb, NOALLOC_THREADS, 0, st>>>((const float *)a, (const float *)b, sa, sb, n,
                                                                    part);
        }
        k_dot_final<<<1, 1024, 0, st>>>(part, nb, result_dev);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) nvb::fail(NVB_ERR_CUDA, std::string("nvb_dot_noalloc launch: ") + cudaGetErrorString(e));
        return NVB_OK;
    } catch (const nvb::Error &e) {
        nvb::set_error(e.msg);
        return e.code;
    }
}
