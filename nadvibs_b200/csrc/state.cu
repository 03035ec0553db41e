// Lanczos state on disk and Ritz vectors.
//
//  * restart.log + nadvibs.35.0: make_restart (Source/top.f90:1007-1049), load_restartinfo
//    (Source/secondary.f90:872-892) and the restore of Source/top.f90:557-588.  The vector
//    file is the single-rank form of the reference's direct-access file (recl = 8*dimen
//    bytes, no record markers): records 1..3*nstates hold q1, q2, q3 state by state, FP64.
//  * archive of normalised Lanczos vectors on the device (Source/secondary.f90:273-308 keeps
//    them on disk): filled during nvb_lanczos when archive_max allows.
//  * Ritz vectors psi_i = sum_k s(k,i) v_k (Source/top.f90:1181-1187) from the archive or, when
//    the archive does not hold every vector, by replaying the recurrence from the seed with
//    the stored alpha/beta (two-pass Lanczos), and the lead basis functions of each
//    (Source/top.f90:1188-1230, rootinfo.dat formats :1264-1282).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "handle.h"

namespace nvb {

#define CK(x)                                                                                    \
    do {                                                                                         \
        cudaError_t e_ = (x);                                                                    \
        if (e_ != cudaSuccess) fail(NVB_ERR_CUDA, std::string(#x ": ") + cudaGetErrorString(e_)); \
    } while (0)

std::string fstr(const char *fmt, ...);
std::string fI(int64_t v, int w);
std::string fF(double v, int w, int d);
std::string fES(double v, int w, int d);

template <typename T>
__global__ void k_to_f64(const T *__restrict__ src, double scale, double *__restrict__ dst, long long n) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        dst[i] = (double)src[i] * scale;
}

template <typename T>
__global__ void k_from_f64(const double *__restrict__ src, T *__restrict__ dst, long long n) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) dst[i] = (T)src[i];
}

template <typename T>
__global__ void k_scale_copy(const T *__restrict__ src, const double *__restrict__ scale, T *__restrict__ dst,
                             long long n) {
    const double s = *scale;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        dst[i] = (T)((double)src[i] * s);
}

// psi[j] += c[j] * v for a block of roots (c in device memory), FP64 accumulators
template <typename T>
__global__ void k_ritz_accum(const T *__restrict__ v, double vs, const double *__restrict__ c, int nroots,
                             double *__restrict__ psi, long long n) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const double x = (double)v[i] * vs;
        for (int j = 0; j < nroots; ++j) psi[(long long)j * n + i] += c[j] * x;
    }
}

// block-wise max of psi^2 (value, first index) for the lead-contributor search
__global__ void k_argmax_sq(const double *__restrict__ psi, const unsigned char *__restrict__ taken, long long n,
                            double *__restrict__ bval, long long *__restrict__ bidx) {
    double best = -1.0;
    long long bi = -1;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const double v = taken[i] ? 0.0 : psi[i] * psi[i];
        if (v > best || (v == best && i < bi)) { best = v; bi = i; }
    }
    __shared__ double sv[256];
    __shared__ long long si[256];
    sv[threadIdx.x] = best;
    si[threadIdx.x] = bi;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            const double v2 = sv[threadIdx.x + o];
            const long long i2 = si[threadIdx.x + o];
            if (v2 > sv[threadIdx.x] || (v2 == sv[threadIdx.x] && i2 >= 0 && (si[threadIdx.x] < 0 || i2 < si[threadIdx.x]))) {
                sv[threadIdx.x] = v2;
                si[threadIdx.x] = i2;
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        bval[blockIdx.x] = sv[0];
        bidx[blockIdx.x] = si[0];
    }
}

__global__ void k_state_norms(const double *__restrict__ psi, long long dimen, int S, double *__restrict__ part) {
    // part[blockIdx.x * S + s] = partial sum of psi^2 over state s
    for (int s = 0; s < S; ++s) {
        double acc = 0.0;
        const long long stride = (long long)gridDim.x * blockDim.x;
        for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < dimen; i += stride) {
            const double v = psi[(long long)s * dimen + i];
            acc += v * v;
        }
        __shared__ double red[256];
        red[threadIdx.x] = acc;
        __syncthreads();
        for (int o = blockDim.x / 2; o > 0; o >>= 1) {
            if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
            __syncthreads();
        }
        if (threadIdx.x == 0) part[(long long)blockIdx.x * S + s] = red[0];
        __syncthreads();
    }
}

// part[blockIdx.x * S*S + k*S + l] = partial sum of a[k][r] * b[l][r] (state blocks of length dimen)
__global__ void k_state_cross(const double *__restrict__ a, const double *__restrict__ b, long long dimen, int S,
                              double *__restrict__ part) {
    __shared__ double red[256];
    for (int k = 0; k < S; ++k)
        for (int l = 0; l < S; ++l) {
            double acc = 0.0;
            const long long stride = (long long)gridDim.x * blockDim.x;
            for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < dimen; i += stride)
                acc += a[(long long)k * dimen + i] * b[(long long)l * dimen + i];
            red[threadIdx.x] = acc;
            __syncthreads();
            for (int o = blockDim.x / 2; o > 0; o >>= 1) {
                if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
                __syncthreads();
            }
            if (threadIdx.x == 0) part[(long long)blockIdx.x * S * S + k * S + l] = red[0];
            __syncthreads();
        }
}

static int grid_n(long long n) {
    long long b = (n + 1023) / 1024;
    if (b > 148 * 8) b = 148 * 8;
    if (b < 1) b = 1;
    return (int)b;
}

// ---------------------------------------------------------------- vector export / import
static void export_vector(nvb_handle *h, const void *buf, double scale, FILE *f) {
    const long long n = h->ntotal();
    const long long chunk = 1ll << 23;  // 64 MiB of FP64 per transfer
    double *dtmp = (double *)scratch_vector(h, (size_t)std::min(n, chunk) * sizeof(double));
    std::vector<double> host((size_t)std::min(n, chunk));
    for (long long off = 0; off < n; off += chunk) {
        const long long m = std::min(chunk, n - off);
        if (h->precision == NVB_MIXED)
            k_to_f64<float><<<grid_n(m), 256, 0, h->stream>>>((const float *)buf + off, scale, dtmp, m);
        else
            k_to_f64<double><<<grid_n(m), 256, 0, h->stream>>>((const double *)buf + off, scale, dtmp, m);
        CK(cudaGetLastError());
        CK(cudaMemcpyAsync(host.data(), dtmp, (size_t)m * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        if (std::fwrite(host.data(), sizeof(double), (size_t)m, f) != (size_t)m)
            fail(NVB_ERR_IO, "short write of a restart vector");
    }
}

static void import_vector(nvb_handle *h, void *buf, FILE *f) {
    const long long n = h->ntotal();
    const long long chunk = 1ll << 23;
    double *dtmp = (double *)scratch_vector(h, (size_t)std::min(n, chunk) * sizeof(double));
    std::vector<double> host((size_t)std::min(n, chunk));
    for (long long off = 0; off < n; off += chunk) {
        const long long m = std::min(chunk, n - off);
        if (std::fread(host.data(), sizeof(double), (size_t)m, f) != (size_t)m)
            fail(NVB_ERR_IO, "restart vector file is shorter than 3*nstates*dimen doubles");
        for (long long i = 0; i < m; ++i)
            if (!std::isfinite(host[i])) fail(NVB_ERR_IO, "non-finite value in the restart vector file");
        CK(cudaMemcpyAsync(dtmp, host.data(), (size_t)m * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        if (h->precision == NVB_MIXED)
            k_from_f64<float><<<grid_n(m), 256, 0, h->stream>>>(dtmp, (float *)buf + off, m);
        else
            k_from_f64<double><<<grid_n(m), 256, 0, h->stream>>>(dtmp, (double *)buf + off, m);
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(h->stream));
    }
}

static std::string join(const char *dir, const char *name) {
    std::string d = dir && *dir ? dir : ".";
    if (d.back() != '/') d += '/';
    return d + name;
}

static void write_reals(FILE *f, const double *v, int64_t n) {
    for (int64_t i = 0; i < n; ++i) {
        std::fprintf(f, " %24.16E", v[i]);
        if (i % 4 == 3 || i == n - 1) std::fprintf(f, "\n");
    }
    if (n == 0) std::fprintf(f, "\n");
}

void save_restart(nvb_handle *h, const char *dir, const char *vdir) {
    if (!h->seeded || h->iters < 1) fail(NVB_ERR_STATE, "no Lanczos iterations to save");
    if (!vdir) vdir = dir;
    const int64_t n = h->iters;
    const std::string rl = join(dir, "restart.log");
    FILE *f = std::fopen(rl.c_str(), "w");
    if (!f) fail(NVB_ERR_IO, "cannot write " + rl);
    std::fprintf(f, " TOTAL NUMBER OF ITERATIONS IN FILE\n %11lld\n", (long long)n);
    std::fprintf(f, " ITERATION NUMBER TO RESTART FROM\n %11lld\n", (long long)n);
    std::fprintf(f, " ALPHA COEFFICIENTS -- diagonal T matrix elements\n");
    write_reals(f, h->alpha.data() + 1, n);
    std::fprintf(f, " BETA COEFFICIENTS -- off-diagonal T matrix elements\n");
    write_reals(f, h->beta.data(), n + 1);
    if (h->reorthog > 0) {
        std::vector<double> o1(n + 1, 0.0), o2(n + 1, 0.0);
        for (int64_t i = 0; i <= n && i < (int64_t)h->omega1.size(); ++i) o1[i] = h->omega1[i];
        for (int64_t i = 0; i <= n && i < (int64_t)h->omega2.size(); ++i) o2[i] = h->omega2[i];
        std::fprintf(f, " OMEGA(1) -- ORTHOGONALITY INFORMATION\n");
        write_reals(f, o1.data(), n + 1);
        std::fprintf(f, " OMEGA(2) -- ORTHOGONALITY INFORMATION\n");
        write_reals(f, o2.data(), n + 1);
    }
    std::fclose(f);
    // q1 = v_{n-1} (work buffer), q2 = v_n (prev buffer), q3 = r_n (cur buffer, unscaled)
    double sc[3];
    CK(cudaMemcpyAsync(sc, h->d_scale, sizeof sc, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    const std::string vf = join(vdir, "nadvibs.35.0");
    FILE *g = std::fopen(vf.c_str(), "wb");
    if (!g) fail(NVB_ERR_IO, "cannot write " + vf);
    export_vector(h, h->buf[h->work], sc[h->work], g);
    export_vector(h, h->buf[h->prev], sc[h->prev], g);
    export_vector(h, h->buf[h->cur], 1.0, g);
    if (std::fclose(g) != 0) fail(NVB_ERR_IO, "error closing " + vf);
}

// list-directed reader for restart.log (values may span records)
namespace {
struct Tok {
    std::vector<std::string> lines;
    size_t pos = 0;
    void skip() {
        if (pos >= lines.size()) fail(NVB_ERR_IO, "restart.log: truncated");
        ++pos;
    }
    std::vector<double> vals(int64_t n) {
        std::vector<double> out;
        while ((int64_t)out.size() < n) {
            if (pos >= lines.size()) fail(NVB_ERR_IO, "restart.log: truncated value list");
            std::string l = lines[pos++];
            for (auto &c : l)
                if (c == ',' || c == 'd' || c == 'D') c = (c == ',') ? ' ' : 'E';
            const char *p = l.c_str();
            char *e = nullptr;
            while ((int64_t)out.size() < n) {
                double v = std::strtod(p, &e);
                if (e == p) break;
                out.push_back(v);
                p = e;
            }
            while (*p == ' ' || *p == '\t' || *p == '\r') ++p;
            if (*p && (int64_t)out.size() < n) fail(NVB_ERR_IO, std::string("restart.log: bad number near '") + p + "'");
        }
        for (double v : out)
            if (!std::isfinite(v)) fail(NVB_ERR_IO, "restart.log: non-finite coefficient");
        return out;
    }
};
}  // namespace

std::string read_file(const std::string &path);
void lanczos_alloc(nvb_handle *h);
void grow_scalars_public(nvb_handle *h, int64_t need);

void load_restart(nvb_handle *h, const char *dir, const char *vdir) {
    if (!vdir) vdir = dir;
    const std::string rl = join(dir, "restart.log");
    Tok t;
    {
        std::string text = read_file(rl);
        size_t s = 0;
        while (s <= text.size()) {
            size_t e = text.find('\n', s);
            if (e == std::string::npos) e = text.size();
            t.lines.push_back(text.substr(s, e - s));
            s = e + 1;
        }
    }
    t.skip();
    const int64_t total = (int64_t)t.vals(1)[0];
    t.skip();
    const int64_t nload = (int64_t)t.vals(1)[0];
    if (nload < 1 || total < nload) fail(NVB_ERR_IO, "restart.log: bad iteration counts");
    if (total != nload) fail(NVB_ERR_IO, "restart.log: restarting before the last iteration needs the disk archive (not kept)");
    t.skip();
    std::vector<double> a = t.vals(nload);
    t.skip();
    std::vector<double> b = t.vals(nload + 1);
    std::vector<double> o1, o2;
    if (h->reorthog > 0) {
        t.skip();
        o1 = t.vals(nload + 1);
        t.skip();
        o2 = t.vals(nload + 1);
    }
    if (!(b[nload] > 0.0)) fail(NVB_ERR_IO, "restart.log: beta(n) must be positive");
    const std::string vf = join(vdir, "nadvibs.35.0");
    FILE *g = std::fopen(vf.c_str(), "rb");
    if (!g) fail(NVB_ERR_IO, "cannot open " + vf);
    if (!h->buf[0]) lanczos_alloc(h);
    h->cur = 0;
    h->prev = 1;
    h->work = 2;
    try {
        import_vector(h, h->buf[h->work], g);  // q1 = v_{n-1}
        import_vector(h, h->buf[h->prev], g);  // q2 = v_n
        import_vector(h, h->buf[h->cur], g);   // q3 = r_n
    } catch (...) {
        std::fclose(g);
        throw;
    }
    std::fclose(g);
    h->alpha.assign(nload + 1, 0.0);
    for (int64_t i = 0; i < nload; ++i) h->alpha[i + 1] = a[i];
    h->beta = b;
    h->iters = nload;
    h->seed_w.assign(h->sys.prm.weights, h->sys.prm.weights + h->sys.S);
    h->omega1 = o1;
    h->omega2 = o2;
    h->seeded = true;
    h->arch_n = 0;
    h->firststep = true;
    h->orth_ranges.clear();
    // a file archive that already holds v_1..v_nload (the reference's nadvibs.34.0 of the run
    // being restarted) lets re-orthogonalisation resume (Source/top.f90:572-575,582-587)
    if (h->arch_kind == ARCH_FILE && h->harch_max >= nload) {
        archive_ensure(h, nload);
        if (FILE *f = std::fopen(h->arch_path.c_str(), "rb")) {
            std::fseek(f, 0, SEEK_END);
            const long long bytes = (long long)ftello(f);
            std::fclose(f);
            if (bytes >= (long long)nload * (long long)h->ntotal() * (long long)sizeof(double)) h->arch_n = nload;
        }
    }
    // device copies of the recurrence coefficients and the buffer scales
    grow_scalars_public(h, nload + 1);
    CK(cudaMemcpyAsync(h->d_alpha, h->alpha.data(), (nload + 1) * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemcpyAsync(h->d_beta, h->beta.data(), (nload + 1) * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    double sc[3];
    sc[h->work] = 1.0;
    sc[h->prev] = 1.0;
    sc[h->cur] = 1.0 / b[nload];
    CK(cudaMemcpyAsync(h->d_scale, sc, sizeof sc, cudaMemcpyHostToDevice, h->stream));
    CK(cudaMemsetAsync(h->d_status, 0, 2 * sizeof(int), h->stream));
    CK(cudaStreamSynchronize(h->stream));
    // as the reference: the log is kept as restart.log.old, the vector file is consumed
    const std::string old = rl + ".old";
    std::rename(rl.c_str(), old.c_str());
    std::remove(vf.c_str());
}

// ---------------------------------------------------------------- Ritz vectors
void lanczos_seed(nvb_handle *h, const double *weights);
void hv_any(nvb_handle *h, const void *x, void *y, int dtype, const double *scale_dev, double *alpha_part,
            int *nblocks_out);

template <typename T>
__global__ void k_replay_step(T *__restrict__ w, const T *__restrict__ c, const T *__restrict__ p, double sc, double sp,
                              double alpha, double beta_prev, long long n) {
    const double a = alpha * sc, b = beta_prev * sp;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        double r = (double)w[i] - a * (double)c[i];
        r = r - b * (double)p[i];
        w[i] = (T)r;
    }
}

// psi (device, nroots * N FP64) = sum_k V(k, j) v_k, j < nroots, V column-major niter x niter
static void ritz_vectors(nvb_handle *h, int64_t nroots, const std::vector<double> &V, double *psi) {
    const int64_t n = h->iters;
    const long long N = h->ntotal();
    CK(cudaMemsetAsync(psi, 0, (size_t)nroots * N * sizeof(double), h->stream));
    double *dc = nullptr;
    CK(cudaMalloc((void **)&dc, (size_t)n * nroots * sizeof(double)));
    std::vector<double> coef((size_t)n * nroots);
    for (int64_t k = 0; k < n; ++k)
        for (int64_t j = 0; j < nroots; ++j) coef[(size_t)k * nroots + j] = V[(size_t)j * n + k];
    CK(cudaMemcpyAsync(dc, coef.data(), coef.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    const bool mixed = h->precision == NVB_MIXED;
    if (archive_holds(h, n)) {
        const size_t per = (size_t)N * h->elem_size();
        archive_for_chunks(h, 1, n, [&](const void *base, int64_t first, int64_t count) {
            for (int64_t q = 0; q < count; ++q) {
                const int64_t k = first - 1 + q;
                const void *vk = (const char *)base + per * q;
                if (mixed)
                    k_ritz_accum<float><<<grid_n(N), 256, 0, h->stream>>>((const float *)vk, 1.0, dc + k * nroots,
                                                                          (int)nroots, psi, N);
                else
                    k_ritz_accum<double><<<grid_n(N), 256, 0, h->stream>>>((const double *)vk, 1.0, dc + k * nroots,
                                                                           (int)nroots, psi, N);
            }
        });
    } else {
        // replay v_1..v_n from the seed with the stored alpha/beta in three scratch buffers
        const size_t per = (size_t)N * h->elem_size();
        void *b3[3] = {nullptr, nullptr, nullptr};
        for (int i = 0; i < 3; ++i) CK(cudaMalloc(&b3[i], per));
        // the seed lanczos_seed built (the weights nvb_seed used, or basis.in's after a restart)
        seed_fill(h, b3[0], seed_weights(h));
        CK(cudaMemsetAsync(b3[1], 0, per, h->stream));
        int cur = 0, prev = 1, work = 2;
        double scur = 1.0 / h->beta[0], sprev = 0.0;
        const int dt = mixed ? NVB_DTYPE_F32 : NVB_DTYPE_F64;
        double *dsc = nullptr;
        CK(cudaMalloc((void **)&dsc, sizeof(double)));
        for (int64_t k = 1; k <= n; ++k) {
            if (mixed)
                k_ritz_accum<float><<<grid_n(N), 256, 0, h->stream>>>((const float *)b3[cur], scur, dc + (k - 1) * nroots,
                                                                      (int)nroots, psi, N);
            else
                k_ritz_accum<double><<<grid_n(N), 256, 0, h->stream>>>((const double *)b3[cur], scur,
                                                                       dc + (k - 1) * nroots, (int)nroots, psi, N);
            if (k == n) break;
            // w = H (scur * cur); r = w - alpha_k v_k - beta_{k-1} v_{k-1}
            CK(cudaMemcpyAsync(dsc, &scur, sizeof(double), cudaMemcpyHostToDevice, h->stream));
            hv_any(h, b3[cur], b3[work], dt, dsc, nullptr, nullptr);
            if (mixed)
                k_replay_step<float><<<grid_n(N), 256, 0, h->stream>>>((float *)b3[work], (const float *)b3[cur],
                                                                       (const float *)b3[prev], scur, sprev, h->alpha[k],
                                                                       h->beta[k - 1], N);
            else
                k_replay_step<double><<<grid_n(N), 256, 0, h->stream>>>((double *)b3[work], (const double *)b3[cur],
                                                                        (const double *)b3[prev], scur, sprev,
                                                                        h->alpha[k], h->beta[k - 1], N);
            CK(cudaStreamSynchronize(h->stream));
            const int op = prev;
            prev = cur;
            cur = work;
            work = op;
            sprev = scur;
            scur = 1.0 / h->beta[k];
        }
        CK(cudaStreamSynchronize(h->stream));
        cudaFree(dsc);
        for (int i = 0; i < 3; ++i) cudaFree(b3[i]);
    }
    CK(cudaStreamSynchronize(h->stream));
    cudaFree(dc);
}

void ritz_vectors_public(nvb_handle *h, int64_t nroots, const std::vector<double> &V, double *psi) {
    ritz_vectors(h, nroots, V, psi);
}

void lead_contributors(nvb_handle *h, int64_t nroots, int64_t k, int64_t *state, int64_t *index, double *c2,
                       int64_t *phase, double *pct, const char *rootinfo) {
    const int64_t n = h->iters;
    if (n < 1) fail(NVB_ERR_STATE, "no Lanczos iterations");
    if (nroots < 1 || nroots > n) fail(NVB_ERR_ARG, "nroots must be in 1..iterations");
    if (k < 0) fail(NVB_ERR_ARG, "k < 0");
    const long long N = h->ntotal();
    const int S = h->sys.S;
    std::vector<double> E(n), V((size_t)n * n);
    tridiag_eigen(n, h->alpha.data() + 1, h->beta.data() + 1, E.data(), V.data());
    double intfactor = 0.0;
    for (int64_t i = 0; i < nroots; ++i) intfactor = std::max(intfactor, V[(size_t)i * n] * V[(size_t)i * n]);
    double *psi = nullptr;
    CK(cudaMalloc((void **)&psi, (size_t)nroots * N * sizeof(double)));
    unsigned char *taken = nullptr;
    const int nb = grid_n(N) > 1024 ? 1024 : grid_n(N);
    double *bval = nullptr;
    long long *bidx = nullptr;
    double *spart = nullptr;
    try {
        ritz_vectors(h, nroots, V, psi);
        CK(cudaMalloc((void **)&taken, (size_t)N));
        CK(cudaMalloc((void **)&bval, nb * sizeof(double)));
        CK(cudaMalloc((void **)&bidx, nb * sizeof(long long)));
        CK(cudaMalloc((void **)&spart, (size_t)nb * S * sizeof(double)));
    } catch (...) {
        cudaFree(psi);
        if (taken) cudaFree(taken);
        throw;
    }
    FILE *f = nullptr;
    if (rootinfo && *rootinfo) {
        f = std::fopen(rootinfo, "w");
        if (!f) fail(NVB_ERR_IO, std::string("cannot write ") + rootinfo);
        std::fprintf(f, " Summary for computing %s eigenvectors corresponding to the lowest eigenvalues\n",
                     fI(nroots, 4).c_str());
    }
    std::vector<double> hv(nb), hs((size_t)nb * S);
    std::vector<long long> hi(nb);
    for (int64_t r = 0; r < nroots; ++r) {
        const double *p = psi + (size_t)r * N;
        CK(cudaMemsetAsync(taken, 0, (size_t)N, h->stream));
        if (f) {
            std::fprintf(f, " Eigenvector %s has been computed...\n", fI(r + 1, 4).c_str());
            std::fprintf(f, " \n ************ ROOT %s *************\n", fI(r + 1, 4).c_str());
            std::fprintf(f, " Energy: %s cm-1, %s eV   Intensity: %s\n\n", fF(E[r] * AU2WAVE, 9, 2).c_str(),
                         fF(E[r] * AU2EV, 9, 5).c_str(),
                         fF(intfactor > 0 ? V[(size_t)r * n] * V[(size_t)r * n] / intfactor : 0.0, 6, 4).c_str());
        }
        for (int64_t j = 0; j < k; ++j) {
            k_argmax_sq<<<nb, 256, 0, h->stream>>>(p, taken, N, bval, bidx);
            CK(cudaMemcpyAsync(hv.data(), bval, nb * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
            CK(cudaMemcpyAsync(hi.data(), bidx, nb * sizeof(long long), cudaMemcpyDeviceToHost, h->stream));
            CK(cudaStreamSynchronize(h->stream));
            double best = -1.0;
            long long bi = -1;
            for (int q = 0; q < nb; ++q)
                if (hi[q] >= 0 && (hv[q] > best || (hv[q] == best && hi[q] < bi))) {
                    best = hv[q];
                    bi = hi[q];
                }
            double val = 0.0;
            CK(cudaMemcpy(&val, p + bi, sizeof(double), cudaMemcpyDeviceToHost));
            const unsigned char one = 1;
            CK(cudaMemcpy(taken + bi, &one, 1, cudaMemcpyHostToDevice));
            const int64_t st = bi / h->sys.dimen, row = bi % h->sys.dimen;
            const int64_t ph = val < 0 ? -1 : 1;
            if (state) state[r * k + j] = st + 1;
            if (index) index[r * k + j] = row + 1;
            if (c2) c2[r * k + j] = best;
            if (phase) phase[r * k + j] = ph;
            if (f) {
                std::fprintf(f, " State vector: %s | Index: %s Phase: %s | Magnitude^2: %s\n", fI(st + 1, 2).c_str(),
                             fI(row + 1, 12).c_str(), fI(ph, 2).c_str(), fF(best, 8, 6).c_str());
                // quanta of each mode (get_barray - 1), 25 per record
                std::string line = " v(i): ";
                int64_t rem = row;
                for (int m = 0; m < h->sys.M; ++m) {
                    const int64_t d = rem / h->sys.shft[m];
                    rem -= d * h->sys.shft[m];
                    if (m > 0 && m % 25 == 0) {
                        std::fprintf(f, "%s\n", line.c_str());
                        line.clear();
                    }
                    line += fI(d, 3);
                }
                std::fprintf(f, "%s\n", line.c_str());
            }
        }
        k_state_norms<<<nb, 256, 0, h->stream>>>(p, h->sys.dimen, S, spart);
        CK(cudaMemcpyAsync(hs.data(), spart, hs.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        std::vector<double> dp(S, 0.0);
        double tot = 0.0;
        for (int s = 0; s < S; ++s) {
            for (int q = 0; q < nb; ++q) dp[s] += hs[(size_t)q * S + s];
            tot += dp[s];
        }
        for (int s = 0; s < S; ++s) {
            dp[s] = 100.0 * std::fabs(dp[s] / tot);
            if (pct) pct[r * S + s] = dp[s];
        }
        if (f) {
            std::fprintf(f, " \n");
            if (S >= 2 && S <= 5) {
                std::string lab, vals;
                for (int s = 0; s < S; ++s) lab += (s ? "," : "") + std::to_string(s + 1);
                for (int s = 0; s < S; ++s) vals += (s ? " %, " : "") + fF(dp[s], 6, 2);
                std::fprintf(f, " Percent State (%s): (%s %%)\n", lab.c_str(), vals.c_str());
            }
            std::fprintf(f, " --------------------------------------------------------------\n");
        }
    }
    if (f) {
        std::fprintf(f, " \n------------ FINISHED EXECUTION ------------\n");
        std::fclose(f);
    }
    cudaFree(psi);
    cudaFree(taken);
    cudaFree(bval);
    cudaFree(bidx);
    cudaFree(spart);
}

// Spin-orbit parameters of identify_roots (Source/top.f90:1153-1175,1231-1252): for the lowest
// soroots Ritz pairs, E_i in eV and sqrt(I_i / I_max) * sign_i (I_max over the lowest nroots,
// sign_i the sign of the first eigenvector component), and for j < i the overlaps of the state
// blocks of the Ritz vectors, ov[i][j][k][l] = sum_r psi_i[k][r] psi_j[l][r].  sodata.in gets
// the reference's text: the overlaps with k != l, in the order (k outer, l inner), for 2 or 3
// states (the reference writes no overlap rows for other state counts).
void spin_orbit(nvb_handle *h, int64_t soroots, int64_t nroots, double *e_ev, double *amp, double *ov,
                const char *path) {
    const int64_t n = h->iters;
    if (n < 1) fail(NVB_ERR_STATE, "no Lanczos iterations");
    if (soroots < 1 || soroots > n) fail(NVB_ERR_ARG, "soroots must be in 1..iterations");
    if (nroots < soroots || nroots > n) fail(NVB_ERR_ARG, "nroots must be in soroots..iterations");
    const long long N = h->ntotal();
    const int S = h->sys.S;
    std::vector<double> E(n), V((size_t)n * n);
    tridiag_eigen(n, h->alpha.data() + 1, h->beta.data() + 1, E.data(), V.data());
    double intfactor = 0.0;
    for (int64_t i = 0; i < nroots; ++i) intfactor = std::max(intfactor, V[(size_t)i * n] * V[(size_t)i * n]);
    std::vector<double> ee(soroots), aa(soroots), oo((size_t)soroots * soroots * S * S, 0.0);
    for (int64_t i = 0; i < soroots; ++i) {
        const double v1 = V[(size_t)i * n];
        ee[i] = E[i] * AU2EV;
        aa[i] = (intfactor > 0 ? std::sqrt(v1 * v1 / intfactor) : 0.0) * (v1 < 0 ? -1.0 : 1.0);
    }
    double *psi = nullptr, *part = nullptr;
    const int nb = grid_n(h->sys.dimen) > 1024 ? 1024 : grid_n(h->sys.dimen);
    CK(cudaMalloc((void **)&psi, (size_t)soroots * N * sizeof(double)));
    try {
        CK(cudaMalloc((void **)&part, (size_t)nb * S * S * sizeof(double)));
        ritz_vectors(h, soroots, V, psi);
        std::vector<double> hp((size_t)nb * S * S);
        for (int64_t i = 1; i < soroots; ++i)
            for (int64_t j = 0; j < i; ++j) {
                k_state_cross<<<nb, 256, 0, h->stream>>>(psi + (size_t)i * N, psi + (size_t)j * N, h->sys.dimen, S,
                                                         part);
                CK(cudaGetLastError());
                CK(cudaMemcpyAsync(hp.data(), part, hp.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
                CK(cudaStreamSynchronize(h->stream));
                double *dst = oo.data() + ((size_t)i * soroots + j) * S * S;
                for (int q = 0; q < nb; ++q)
                    for (int kl = 0; kl < S * S; ++kl) dst[kl] += hp[(size_t)q * S * S + kl];
            }
    } catch (...) {
        cudaFree(psi);
        if (part) cudaFree(part);
        throw;
    }
    cudaFree(psi);
    cudaFree(part);
    if (e_ev) std::copy(ee.begin(), ee.end(), e_ev);
    if (amp) std::copy(aa.begin(), aa.end(), amp);
    if (ov) std::copy(oo.begin(), oo.end(), ov);
    if (path && *path) {
        FILE *f = std::fopen(path, "w");
        if (!f) fail(NVB_ERR_IO, std::string("cannot write ") + path);
        std::fprintf(f, "%s\n", fI(soroots, 5).c_str());
        std::fprintf(f, " Root   Energy (eV)      Sqrt(Int.)*sign\n");
        for (int64_t i = 0; i < soroots; ++i)
            std::fprintf(f, "%s  %s  %s\n", fI(i + 1, 5).c_str(), fES(ee[i], 15, 8).c_str(), fES(aa[i], 15, 8).c_str());
        if (S == 2) std::fprintf(f, " R(i)  R(j)   [S1(i)S2(j)]   [S2(i)S1(j)]\n");
        if (S == 3)
            std::fprintf(f, " R(i)  R(j)   [S1(i)S2(j)]   [S1(i)S3(j)]  [S2(i)S1(j)]\n"
                            " R(i)  R(j)   [S2(i)S3(j)]   [S3(i)S1(j)]  [S3(i)S2(j)]\n");
        if (S == 2 || S == 3)
            for (int64_t i = 1; i < soroots; ++i)
                for (int64_t j = 0; j < i; ++j) {
                    const double *o = oo.data() + ((size_t)i * soroots + j) * S * S;
                    std::vector<double> dp;
                    for (int k = 0; k < S; ++k)
                        for (int l = 0; l < S; ++l)
                            if (k != l) dp.push_back(o[k * S + l]);
                    const std::string ij = fI(i + 1, 5) + " " + fI(j + 1, 5) + "  ";
                    if (S == 2) std::fprintf(f, "%s%s %s\n", ij.c_str(), fES(dp[0], 14, 6).c_str(), fES(dp[1], 14, 6).c_str());
                    else
                        std::fprintf(f, "%s%s %s %s\n%s%s %s %s\n", ij.c_str(), fES(dp[0], 14, 6).c_str(),
                                     fES(dp[1], 14, 6).c_str(), fES(dp[2], 14, 6).c_str(), ij.c_str(),
                                     fES(dp[3], 14, 6).c_str(), fES(dp[4], 14, 6).c_str(), fES(dp[5], 14, 6).c_str());
                }
        std::fclose(f);
    }
}

}  // namespace nvb

namespace nvb {

// The seed section of output.dat (generate_initialvec's report, Source/secondary.f90:351-802,
// formats 1000-1011 and 1022-1025): for the displaced seed the number of basis functions of
// every quanta sum ("level") and the <m| levels built, for either seed the overlap with the
// initial state, its 40 dominant basis functions (repeated argmax of q^2 with the row zeroed in
// every state), and the normalisation of the initial Lanczos vector by the state weights.
void write_seed_report(nvb_handle *h, const char *path) {
    if (!h->seeded) fail(NVB_ERR_STATE, "nvb_write_seed_report needs nvb_seed first");
    const System &sys = h->sys;
    const int S = sys.S, M = sys.M;
    const long long N = sys.dimen;
    FILE *f = std::fopen(path, "a");
    if (!f) fail(NVB_ERR_IO, std::string("cannot open ") + path);
    const std::string stars(70, '*');
    double d1 = 1.0;  // sqrt(<q3,q3>/nstates) of the unscaled seed
    if (sys.neworigin) {
        std::fprintf(f, "\n  %s\n  Generating seed vector by computing ANION/ORIGIN overlap...\n", stars.c_str());
        // basis functions per quanta sum (level-synchronous recursion over sum_k n_k)
        std::vector<long long> cnt(1, 1);
        for (int k = 0; k < M; ++k) {
            const int nf = (int)sys.nfunc[k];
            std::vector<long long> nx(cnt.size() + nf - 1, 0);
            for (size_t l = 0; l < cnt.size(); ++l)
                for (int q = 0; q < nf; ++q) nx[l + q] += cnt[l];
            cnt.swap(nx);
        }
        const int nlev = (int)cnt.size() - 1;
        long long tcount = 0;
        for (int j = 0; j < nlev; ++j) {
            std::fprintf(f, "  LEVEL %s, Number of terms:     %s\n", fI(j, 5).c_str(), fI(cnt[(size_t)j], 12).c_str());
            tcount += cnt[(size_t)j];
        }
        std::fprintf(f, "  LEVEL %s, Number of terms:     %s\n", fI(nlev, 5).c_str(), fI(1, 12).c_str());
        tcount += 1;
        std::fprintf(f, "\n  Sum over levels:                  %s\n  Size of direct product basis:     %s\n\n",
                     fI(tcount, 12).c_str(), fI(N, 12).c_str());
        int imode = M - 1;
        for (int i = 0; i < M; ++i)
            if (sys.istate[(size_t)i] > 0) {
                imode = i;
                break;
            }
        for (int64_t i = 1; i <= sys.istate[(size_t)imode]; ++i)
            std::fprintf(f, "  Building <m| = <%s|\n", fI(i, 2).c_str());
        d1 = h->seed_norm;
    } else {
        std::fprintf(f, "\n  %s\n  Generating seed vector using ANION basis...\n", stars.c_str());
    }
    std::fprintf(f, "\n  Overlap with the initial state:   %s\n", fF(d1, 12, 6).c_str());
    std::fprintf(f, "\n  Dominant Contributions to Overlap\n  ---------------------------------\n");
    // every state holds the same unscaled seed: the simple one is 1 at the first row, the
    // displaced one <m|n>
    auto quanta = [&](long long row) {
        std::string s;
        long long rem = row;
        for (int k = 0; k < M; ++k) {
            const long long d = rem / sys.shft[(size_t)k];
            rem -= d * sys.shft[(size_t)k];
            s += fI(d, 2) + ",";
        }
        return s;
    };
    if (sys.neworigin && h->seed_vec) {
        const int nb = (int)std::min<long long>((N + 255) / 256, 1024);
        unsigned char *taken = nullptr;
        double *bval = nullptr;
        long long *bidx = nullptr;
        CK(cudaMalloc((void **)&taken, (size_t)N));
        CK(cudaMalloc((void **)&bval, nb * sizeof(double)));
        CK(cudaMalloc((void **)&bidx, nb * sizeof(long long)));
        CK(cudaMemsetAsync(taken, 0, (size_t)N, h->stream));
        std::vector<double> hv(nb);
        std::vector<long long> hi(nb);
        for (int sidx = 1; sidx <= 40; ++sidx) {
            k_argmax_sq<<<nb, 256, 0, h->stream>>>(h->seed_vec, taken, N, bval, bidx);
            CK(cudaMemcpyAsync(hv.data(), bval, nb * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
            CK(cudaMemcpyAsync(hi.data(), bidx, nb * sizeof(long long), cudaMemcpyDeviceToHost, h->stream));
            CK(cudaStreamSynchronize(h->stream));
            double best = -1.0;
            long long bi = -1;
            for (int q = 0; q < nb; ++q)
                if (hi[q] >= 0 && (hv[q] > best || (hv[q] == best && hi[q] < bi))) {
                    best = hv[q];
                    bi = hi[q];
                }
            if (bi < 0 || best == 0.0) break;
            const unsigned char one = 1;
            CK(cudaMemcpy(taken + bi, &one, 1, cudaMemcpyHostToDevice));
            std::fprintf(f, "  %s. %s: %s\n", fI(sidx, 2).c_str(), quanta(bi).c_str(), fF(best, 12, 6).c_str());
        }
        cudaFree(taken);
        cudaFree(bval);
        cudaFree(bidx);
    } else {
        std::fprintf(f, "  %s. %s: %s\n", fI(1, 2).c_str(), quanta(0).c_str(), fF(1.0, 12, 6).c_str());
    }
    // the state weights scale the blocks, then the vector is normalised
    double wsum = 0.0;
    for (double w : h->seed_w) wsum += w;
    if (wsum == 0.0) wsum = 1.0;
    std::fprintf(f, "\n  Normalization of Initial Lanczos Vector\n");
    double tot = 0.0;
    for (int s = 0; s < S; ++s) {
        const double n = std::fabs(h->seed_w[(size_t)s] / wsum);
        tot += n * n;
        std::fprintf(f, "  ||STATE%s|| = %s -- (||STATE%s||)^2 = %s\n", fI(s + 1, 2).c_str(), fF(n, 6, 4).c_str(),
                     fI(s + 1, 2).c_str(), fF(n * n, 6, 4).c_str());
    }
    std::fprintf(f, "  || TOTAL || = %s -- (|| TOTAL ||)^2 = %s\n", fF(std::sqrt(tot), 6, 4).c_str(),
                 fF(tot, 6, 4).c_str());
    std::fprintf(f, "  Normalizing Initial Lanczos Vector...\n");
    std::fprintf(f, "  || TOTAL || = %s -- (|| TOTAL ||)^2 = %s\n", fF(1.0, 6, 4).c_str(), fF(1.0, 6, 4).c_str());
    std::fprintf(f, "\n  Time Required: %s secs.\n  %s\n\n", fF(h->seed_secs, 14, 3).c_str(), stars.c_str());
    std::fclose(f);
}

}  // namespace nvb
