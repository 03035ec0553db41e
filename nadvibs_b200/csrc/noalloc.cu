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
//  * at most 4096 block partials (the array is 4097 doubles, about 32 KiB, held by every GPU
//    that loads the library until the process exits); the grid is sized from n, about eight
//    blocks per multiprocessor for large n, each block striding over the whole vector, and
//    a call takes n <= 2^32 elements;
//  * every call, on every stream, uses the same array; each call overwrites the partials it
//    uses before reading them, so no clearing is needed, but calls that overlap on the GPU
//    race with each other and must be ordered by the caller (same stream or events);
//  * the array's device address is looked up with cudaGetSymbolAddress on the first call in
//    each CUDA context (once per device, with that device current, and again if the
//    device's context was reset); make that first call before any stream capture.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <string>

#include "../../include/nadvibs.h"
#include "nvb_internal.h"

namespace {

constexpr long long NOALLOC_MAX_N = 1ll << 32;  // elements per call
constexpr int NOALLOC_MAX_BLOCKS = 4096;        // partials in the static array
constexpr int NOALLOC_THREADS = 256;
constexpr int NOALLOC_MIN_PER_THREAD = 4;       // a grid never has blocks with less work than this
constexpr int NOALLOC_MAX_DEVICES = 64;

// Partials [0, nblocks) of the current call.  Host code never touches this symbol directly:
// in host code the name is only a stand-in, so kernels get its address from
// cudaGetSymbolAddress.
static __device__ __align__(256) double g_noalloc_partials[NOALLOC_MAX_BLOCKS + 1];

// per device: the context the address was looked up in, and the address
struct ScratchAddr {
    unsigned long long ctx_id = 0;
    double *ptr = nullptr;
};
ScratchAddr g_scratch_dev[NOALLOC_MAX_DEVICES];
std::mutex g_mu;

typedef int (*CtxGetCurrentFn)(void **);
typedef int (*CtxGetIdFn)(void *, unsigned long long *);

// Identifier of the current CUDA context (0 if the driver does not report one): a
// cudaDeviceReset gives the device a new primary context, in which the static array has a
// new address.
unsigned long long current_context_id() {
    static CtxGetCurrentFn get_current = nullptr;
    static CtxGetIdFn get_id = nullptr;
    static bool looked_up = false;
    if (!looked_up) {
        void *f1 = nullptr, *f2 = nullptr;
        cudaDriverEntryPointQueryResult q1, q2;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1) == cudaSuccess &&
            q1 == cudaDriverEntryPointSuccess)
            get_current = (CtxGetCurrentFn)f1;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2) == cudaSuccess &&
            q2 == cudaDriverEntryPointSuccess)
            get_id = (CtxGetIdFn)f2;
        looked_up = true;
    }
    if (!get_current || !get_id) return 0;
    void *ctx = nullptr;
    unsigned long long id = 0;
    if (get_current(&ctx) != 0 || !ctx || get_id(ctx, &id) != 0) return 0;
    return id;
}

double *scratch_for_current_device() {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) nvb::fail(NVB_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) nvb::fail(NVB_ERR_ARG, "device ordinal beyond 63");
    // make the device's primary context current (cudaSetDevice initialises it) before asking
    // for its identifier
    e = cudaSetDevice(dev);
    if (e != cudaSuccess) nvb::fail(NVB_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    const unsigned long long id = current_context_id();
    std::lock_guard<std::mutex> lk(g_mu);
    ScratchAddr &sa = g_scratch_dev[dev];
    if (!sa.ptr || sa.ctx_id != id) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_partials);
        if (e != cudaSuccess || !p)
            nvb::fail(NVB_ERR_CUDA, std::string("cudaGetSymbolAddress of the static scratch array: ") +
                                        cudaGetErrorString(e));
        sa.ptr = static_cast<double *>(p);
        sa.ctx_id = id;
    }
    return sa.ptr;
}

// blocks of a call over n elements: enough for every multiprocessor several times over, at
// most the array's 4096 partials, and none with fewer than 4 elements per thread
int blocks_for(long long n, int nsm) {
    if (n <= 0) return 0;
    long long nb = (n + (long long)NOALLOC_THREADS * NOALLOC_MIN_PER_THREAD - 1) /
                   ((long long)NOALLOC_THREADS * NOALLOC_MIN_PER_THREAD);
    const long long cap = std::min<long long>(NOALLOC_MAX_BLOCKS, 8ll * std::max(nsm, 1));
    return (int)std::max<long long>(1, std::min(nb, cap));
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

// block b sums elements b*256 + t, (b + nb)*256 + t, ... (coalesced, grid-stride)
template <typename T>
__global__ void k_dot_chunks(const T *__restrict__ a, const T *__restrict__ b, double sa, double sb, long long n,
                             double *__restrict__ partials) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    double acc = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        acc += ((double)a[i] * sa) * ((double)b[i] * sb);
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
        if (n > NOALLOC_MAX_N)
            nvb::fail(NVB_ERR_ARG, "n = " + std::to_string(n) +
                                       " exceeds the maximum of the allocation-free dot product, 2^32 elements");
        double *part = scratch_for_current_device();
        cudaStream_t st = (cudaStream_t)stream;
        int dev = 0, nsm = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) nsm = 1;
        const int nb = blocks_for(n, nsm);
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
