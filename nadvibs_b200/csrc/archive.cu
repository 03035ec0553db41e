// Archive of the normalised Lanczos vectors v_1..v_k, for re-orthogonalisation and one-pass
// Ritz vectors.  The reference keeps it on disk (nadvibs.34.<rank>, Source/top.f90:570-571,
// 595-598, written by write_ga and read back by read_ga, Source/secondary.f90:273-308): a
// direct-access file whose records are the nstates columns of dimen FP64 values of each
// vector, vector after vector.  Here it lives
//   * in device memory (ARCH_DEVICE, the options' archive_max): consumers read it in place;
//   * in pinned host memory (ARCH_HOST), in blocks of vectors allocated as the run grows; or
//   * in a file in the reference's layout (ARCH_FILE, FP64 whatever the handle's precision),
// and the host-side kinds are streamed to the device in chunks of whole vectors: one
// cudaMemcpyAsync per chunk on a copy stream into a two-slot staging ring, the consumer
// kernels of chunk c running on the handle's stream while chunk c + 1 is copied.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <functional>
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

constexpr size_t ARCH_CHUNK_BYTES = 256ull << 20;  // target size of one streamed chunk

int grid_a(long long n) {
    long long b = (n + 1023) / 1024;
    if (b > 148 * 8) b = 148 * 8;
    return (int)std::max<long long>(b, 1);
}

template <typename T>
__global__ void k_scale_copy_a(const T *__restrict__ src, const double *__restrict__ scale, T *__restrict__ dst,
                               long long n) {
    const double s = *scale;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        dst[i] = (T)((double)src[i] * s);
}

// the file's FP64 record of v = scale * src
template <typename T>
__global__ void k_scale_widen(const T *__restrict__ src, const double *__restrict__ scale, double *__restrict__ dst,
                              long long n) {
    const double s = *scale;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        dst[i] = (double)src[i] * s;
}

__global__ void k_narrow(const double *__restrict__ src, float *__restrict__ dst, long long n) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) dst[i] = (float)src[i];
}

size_t native_bytes(const nvb_handle *h) { return (size_t)h->ntotal() * h->elem_size(); }
size_t file_bytes(const nvb_handle *h) { return (size_t)h->ntotal() * sizeof(double); }

// vectors per streamed chunk (and per pinned block of the host kind)
int64_t chunk_vectors(const nvb_handle *h) {
    const size_t per = h->arch_kind == ARCH_FILE ? file_bytes(h) : native_bytes(h);
    return std::max<int64_t>(1, std::min<int64_t>(16, (int64_t)(ARCH_CHUNK_BYTES / std::max<size_t>(per, 1))));
}

void staging_ensure(nvb_handle *h) {
    if (h->arch_stage[0]) return;
    const int64_t cv = chunk_vectors(h);
    for (int s = 0; s < 2; ++s) CK(cudaMalloc(&h->arch_stage[s], (size_t)cv * native_bytes(h)));
    if (h->arch_kind == ARCH_FILE) {
        CK(cudaMalloc(&h->arch_stage64, (size_t)cv * file_bytes(h)));
        CK(cudaHostAlloc(&h->arch_bounce, (size_t)cv * file_bytes(h), cudaHostAllocDefault));
    }
    CK(cudaStreamCreateWithFlags(&h->arch_stream, cudaStreamNonBlocking));
    for (int s = 0; s < 2; ++s) {
        CK(cudaEventCreateWithFlags(&h->arch_ready[s], cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&h->arch_free[s], cudaEventDisableTiming));
    }
}

void file_open(nvb_handle *h) {
    if (h->arch_file) return;
    h->arch_file = std::fopen(h->arch_path.c_str(), "r+b");
    if (!h->arch_file) h->arch_file = std::fopen(h->arch_path.c_str(), "w+b");
    if (!h->arch_file) fail(NVB_ERR_IO, "cannot open the Lanczos-vector archive " + h->arch_path);
}

void file_rw(nvb_handle *h, bool write, int64_t first, int64_t count, void *buf) {
    file_open(h);
    const size_t per = file_bytes(h);
    if (fseeko(h->arch_file, (off_t)((size_t)first * per), SEEK_SET) != 0)
        fail(NVB_ERR_IO, "seek in the Lanczos-vector archive " + h->arch_path);
    const size_t n = (size_t)count * per;
    const size_t done = write ? std::fwrite(buf, 1, n, h->arch_file) : std::fread(buf, 1, n, h->arch_file);
    if (done != n)
        fail(NVB_ERR_IO, std::string(write ? "write to" : "read from") + " the Lanczos-vector archive " + h->arch_path +
                             " (record " + std::to_string(first + 1) + ")");
    if (write) std::fflush(h->arch_file);
}

// H2D of vectors [first, first + count) (0-based) into staging slot s, on the copy stream
void stage_chunk(nvb_handle *h, int s, int64_t first, int64_t count) {
    const size_t per = native_bytes(h);
    CK(cudaStreamWaitEvent(h->arch_stream, h->arch_free[s], 0));
    if (h->arch_kind == ARCH_HOST) {
        const int64_t cv = chunk_vectors(h);
        const int64_t blk = first / cv, off = first - blk * cv;  // a chunk never spans two blocks
        CK(cudaMemcpyAsync(h->arch_stage[s], (const char *)h->harch_blocks[(size_t)blk] + (size_t)off * per,
                           (size_t)count * per, cudaMemcpyHostToDevice, h->arch_stream));
    } else {
        // the copy stream must be done with the bounce buffer before it is refilled
        CK(cudaStreamSynchronize(h->arch_stream));
        file_rw(h, false, first, count, h->arch_bounce);
        const size_t per64 = file_bytes(h);
        if (h->precision == NVB_MIXED) {
            CK(cudaMemcpyAsync(h->arch_stage64, h->arch_bounce, (size_t)count * per64, cudaMemcpyHostToDevice,
                               h->arch_stream));
            k_narrow<<<grid_a((long long)count * h->ntotal()), 256, 0, h->arch_stream>>>(
                (const double *)h->arch_stage64, (float *)h->arch_stage[s], (long long)count * h->ntotal());
            CK(cudaGetLastError());
        } else {
            CK(cudaMemcpyAsync(h->arch_stage[s], h->arch_bounce, (size_t)count * per64, cudaMemcpyHostToDevice,
                               h->arch_stream));
        }
    }
    CK(cudaEventRecord(h->arch_ready[s], h->arch_stream));
}

}  // namespace

void archive_configure(nvb_handle *h, int kind, int64_t max_vectors, const char *path) {
    if (kind < ARCH_DEVICE || kind > ARCH_FILE) fail(NVB_ERR_ARG, "archive kind must be 0 (device), 1 (host), 2 (file)");
    if (max_vectors < 0) fail(NVB_ERR_ARG, "archive size < 0");
    if (kind == ARCH_FILE && (!path || !*path)) fail(NVB_ERR_ARG, "the file archive needs a path");
    archive_free(h);
    h->arch_kind = kind;
    if (kind == ARCH_DEVICE) {
        h->opt.archive_max = max_vectors;
        h->harch_max = 0;
    } else {
        h->opt.archive_max = 0;
        h->harch_max = max_vectors;
        if (kind == ARCH_FILE) h->arch_path = path;
    }
}

int64_t archive_capacity(const nvb_handle *h) {
    return h->arch_kind == ARCH_DEVICE ? h->opt.archive_max : h->harch_max;
}

bool archive_holds(const nvb_handle *h, int64_t n) {
    if (h->arch_kind == ARCH_DEVICE) return h->arch && h->arch_n >= n;
    return h->harch_max > 0 && h->arch_n >= n;
}

void archive_free(nvb_handle *h) {
    if (h->arch) cudaFree(h->arch);
    h->arch = nullptr;
    h->arch_cap = h->arch_n = 0;
    for (void *b : h->harch_blocks) cudaFreeHost(b);
    h->harch_blocks.clear();
    for (int s = 0; s < 2; ++s) {
        if (h->arch_stage[s]) cudaFree(h->arch_stage[s]);
        h->arch_stage[s] = nullptr;
        if (h->arch_ready[s]) cudaEventDestroy(h->arch_ready[s]);
        if (h->arch_free[s]) cudaEventDestroy(h->arch_free[s]);
        h->arch_ready[s] = h->arch_free[s] = nullptr;
    }
    if (h->arch_stage64) cudaFree(h->arch_stage64);
    h->arch_stage64 = nullptr;
    if (h->arch_bounce) cudaFreeHost(h->arch_bounce);
    h->arch_bounce = nullptr;
    if (h->arch_stream) cudaStreamDestroy(h->arch_stream);
    h->arch_stream = nullptr;
    if (h->arch_file) std::fclose(h->arch_file);
    h->arch_file = nullptr;
}

void archive_ensure(nvb_handle *h, int64_t need) {
    if (h->arch_kind != ARCH_DEVICE) {
        if (h->harch_max <= 0) return;
        staging_ensure(h);
        if (h->arch_kind == ARCH_HOST) {
            const int64_t cv = chunk_vectors(h), cap = std::min<int64_t>(need, h->harch_max);
            while ((int64_t)h->harch_blocks.size() * cv < cap) {
                void *b = nullptr;
                const cudaError_t e = cudaHostAlloc(&b, (size_t)cv * native_bytes(h), cudaHostAllocDefault);
                if (e != cudaSuccess) {
                    (void)cudaGetLastError();
                    fail(NVB_ERR_NOMEM, "pinned host memory for the Lanczos-vector archive: " +
                                            std::to_string(h->harch_blocks.size() * cv) + " vectors allocated, " +
                                            std::to_string(cap) + " needed (" + cudaGetErrorString(e) + ")");
                }
                h->harch_blocks.push_back(b);
            }
            h->arch_cap = (int64_t)h->harch_blocks.size() * cv;
        } else {
            file_open(h);
            h->arch_cap = h->harch_max;
        }
        return;
    }
    if (h->opt.archive_max <= 0) return;
    const int64_t cap = std::min<int64_t>(need, h->opt.archive_max);
    if (cap <= h->arch_cap) return;
    void *na = nullptr;
    const size_t per = native_bytes(h);
    CK(cudaMalloc(&na, per * cap));
    if (h->arch && h->arch_n > 0) CK(cudaMemcpyAsync(na, h->arch, per * h->arch_n, cudaMemcpyDeviceToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (h->arch) cudaFree(h->arch);
    h->arch = na;
    h->arch_cap = cap;
}

// stores v_it = scale[cur] * buf[cur] as archive entry it - 1 (at the start of iteration it)
void archive_push(nvb_handle *h, int64_t it) {
    if (it - 1 != h->arch_n || h->arch_n >= h->arch_cap) return;
    const long long n = h->ntotal();
    const bool mixed = h->precision == NVB_MIXED;
    if (h->arch_kind == ARCH_DEVICE) {
        if (!h->arch) return;
        void *dst = (char *)h->arch + native_bytes(h) * (size_t)(it - 1);
        if (mixed)
            k_scale_copy_a<float><<<grid_a(n), 256, 0, h->stream>>>((const float *)h->buf[h->cur], h->d_scale + h->cur,
                                                                    (float *)dst, n);
        else
            k_scale_copy_a<double><<<grid_a(n), 256, 0, h->stream>>>((const double *)h->buf[h->cur],
                                                                     h->d_scale + h->cur, (double *)dst, n);
        CK(cudaGetLastError());
    } else if (h->arch_kind == ARCH_HOST) {
        // the scaled vector into staging slot 0 (after its last reader), then to the host block
        const int64_t cv = chunk_vectors(h), blk = (it - 1) / cv, off = (it - 1) - blk * cv;
        CK(cudaStreamWaitEvent(h->stream, h->arch_ready[0], 0));
        if (mixed)
            k_scale_copy_a<float><<<grid_a(n), 256, 0, h->stream>>>((const float *)h->buf[h->cur], h->d_scale + h->cur,
                                                                    (float *)h->arch_stage[0], n);
        else
            k_scale_copy_a<double><<<grid_a(n), 256, 0, h->stream>>>((const double *)h->buf[h->cur],
                                                                     h->d_scale + h->cur, (double *)h->arch_stage[0], n);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync((char *)h->harch_blocks[(size_t)blk] + (size_t)off * native_bytes(h), h->arch_stage[0],
                           native_bytes(h), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaEventRecord(h->arch_free[0], h->stream));
    } else {
        // the FP64 record of the reference's layout, written before the next iteration starts
        if (mixed)
            k_scale_widen<float><<<grid_a(n), 256, 0, h->stream>>>((const float *)h->buf[h->cur], h->d_scale + h->cur,
                                                                   (double *)h->arch_stage64, n);
        else
            k_scale_widen<double><<<grid_a(n), 256, 0, h->stream>>>((const double *)h->buf[h->cur],
                                                                    h->d_scale + h->cur, (double *)h->arch_stage64, n);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(h->arch_bounce, h->arch_stage64, file_bytes(h), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        file_rw(h, true, it - 1, 1, h->arch_bounce);
    }
    h->arch_n = it;
}

// fn(base, first, count) for consecutive chunks covering archive entries [lo, hi] (1-based):
// base = device address of entry `first` in native precision, valid for the call (the
// consumer's kernels run on the handle's stream).
void archive_for_chunks(nvb_handle *h, int64_t lo, int64_t hi,
                        const std::function<void(const void *, int64_t, int64_t)> &fn) {
    if (hi < lo) return;
    if (!archive_holds(h, hi)) fail(NVB_ERR_STATE, "the Lanczos-vector archive does not hold the vectors needed");
    if (h->arch_kind == ARCH_DEVICE) {
        fn((const char *)h->arch + native_bytes(h) * (size_t)(lo - 1), lo, hi - lo + 1);
        return;
    }
    const int64_t cv = chunk_vectors(h);
    // chunks aligned to blocks of cv entries (0-based)
    std::vector<std::pair<int64_t, int64_t>> ch;
    for (int64_t f = lo - 1; f <= hi - 1;) {
        const int64_t end = std::min(hi - 1, (f / cv + 1) * cv - 1);
        ch.push_back({f, end - f + 1});
        f = end + 1;
    }
    // the copy stream may only overwrite a slot after the handle's stream is done with it
    for (int s = 0; s < 2; ++s) CK(cudaEventRecord(h->arch_free[s], h->stream));
    stage_chunk(h, 0, ch[0].first, ch[0].second);
    for (size_t c = 0; c < ch.size(); ++c) {
        const int s = (int)(c & 1);
        if (c + 1 < ch.size()) stage_chunk(h, s ^ 1, ch[c + 1].first, ch[c + 1].second);
        CK(cudaStreamWaitEvent(h->stream, h->arch_ready[s], 0));
        fn(h->arch_stage[s], ch[c].first + 1, ch[c].second);
        CK(cudaEventRecord(h->arch_free[s], h->stream));
    }
}

}  // namespace nvb
