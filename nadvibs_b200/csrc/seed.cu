// Displaced / Duschinsky Franck-Condon seed (generate_initialvec, neworigin branch,
// Source/secondary.f90:372-726): <m|n> between the initial vibrational state |m> (frequencies
// bomega in the coordinates y = T x + d of the Hamiltonian's modes x, at most one mode
// excited) and every product basis function |n> (frequencies omega).
//
// Host: the matrices of Source/secondary.f90:407-478,
//   A = (a + T^T b T)/2,  A1 = sqrt(a) A^-1 sqrt(a) - 1,  A2 = sqrt(a) A^-1 T^T sqrt(b),
//   A3 = sqrt(b) T A^-1 T^T sqrt(b),  A2d = A2 sqrt(b) d,  A3d = (A3 - 2)^T sqrt(b) d,
//   d2 = sqrt(sqrt(prod a b) |det T| / det A) exp(-b.d^2/2 + (sqrt(b) d)^T A3 (sqrt(b) d)/4).
// Device, level by level in the total quanta L (one launch per level, every element checks its
// level): C(0) = 1 and, with j the first mode of n with n_j > 0 and p = n - e_j,
//   C(n) = 2 sum_{k in irrep(j)} A1_jk p_k C(p - e_k) - A2d_j C(p)
// (the reference writes each C(n) from whichever (p, j) its traversal visits last; the
// recursion is consistent, so the choice only moves the last bits).  Then the initial-state
// levels m = 1..istate(i) (Source/secondary.f90:590-682):
//   C_m(n) = 2 (m-1) (A3_ii - 1) C_{m-2}(n) - A3d_i C_{m-1}(n) + 2 sum_k A2_ki n_k C_{m-1}(n - e_k),
// and the scale <m|n> = d2 C(n) / sqrt(prod_j 2^{n_j} n_j! 2^{m_j} m_j!) (:683-725).
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

constexpr int SEED_MAXM = MAX_MODES;

struct SeedArgs {
    int M;
    long long dimen;
    long long shft[SEED_MAXM];
    int nfunc[SEED_MAXM];
    int irrep[SEED_MAXM];
};

int seed_grid(long long n) { return (int)std::max<long long>(1, std::min<long long>((n + 255) / 256, 148 * 16)); }

// C(n) for the elements at total quanta L
__global__ void k_fc_level(SeedArgs a, const double *__restrict__ A1, const double *__restrict__ A2d, int L,
                           double *__restrict__ C) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < a.dimen; r += stride) {
        int dig[SEED_MAXM];
        long long rem = r;
        int lev = 0, j = -1;
        for (int k = 0; k < a.M; ++k) {
            dig[k] = (int)(rem / a.shft[k]);
            rem -= (long long)dig[k] * a.shft[k];
            lev += dig[k];
            if (j < 0 && dig[k] > 0) j = k;
        }
        if (lev != L || j < 0) continue;
        const long long p = r - a.shft[j];
        dig[j] -= 1;
        double s = 0.0;
        for (int k = 0; k < a.M; ++k)
            if (a.irrep[k] == a.irrep[j] && dig[k] > 0) s += A1[j * a.M + k] * dig[k] * C[p - a.shft[k]];
        C[r] = 2.0 * s - A2d[j] * C[p];
    }
}

// one initial-state level m in mode i
__global__ void k_fc_mstep(SeedArgs a, const double *__restrict__ A2, double c2, double c1, int i,
                           const double *__restrict__ cm2, const double *__restrict__ cm1, double *__restrict__ cm) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < a.dimen; r += stride) {
        double v = c2 * cm2[r] + c1 * cm1[r];
        long long rem = r;
        for (int k = 0; k < a.M; ++k) {
            const int d = (int)(rem / a.shft[k]);
            rem -= (long long)d * a.shft[k];
            if (d > 0) v += 2.0 * A2[k * a.M + i] * d * cm1[r - a.shft[k]];
        }
        cm[r] = v;
    }
}

// <m|n> = d2 C(n) / sqrt(prod_j 2^{n_j} n_j!) / sqrt(prod_j 2^{m_j} m_j!); pw[j*64+n] = 2^n n!
__global__ void k_fc_scale(SeedArgs a, const double *__restrict__ pw, double d2m, double *__restrict__ C) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < a.dimen; r += stride) {
        double den = 1.0;
        long long rem = r;
        for (int k = 0; k < a.M; ++k) {
            const int d = (int)(rem / a.shft[k]);
            rem -= (long long)d * a.shft[k];
            den *= pw[k * 256 + d];
        }
        C[r] = d2m * C[r] / sqrt(den);
    }
}

// per-block partial sums of x^2
__global__ void k_sumsq(const double *__restrict__ x, long long n, double *__restrict__ part) {
    __shared__ double red[256];
    double acc = 0.0;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) acc += x[i] * x[i];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// |det| by elimination with row pivoting (gauss_elim, Source/secondary.f90:309-347)
double abs_det(std::vector<double> m, int n) {
    for (int i = 0; i < n - 1; ++i) {
        int mr = i;
        double v = std::fabs(m[(size_t)i * n + i]);
        for (int j = i + 1; j < n; ++j)
            if (std::fabs(m[(size_t)j * n + i]) > v) {
                v = std::fabs(m[(size_t)j * n + i]);
                mr = j;
            }
        if (mr != i)
            for (int c = 0; c < n; ++c) std::swap(m[(size_t)mr * n + c], m[(size_t)i * n + c]);
        for (int j = i + 1; j < n; ++j)
            if (m[(size_t)j * n + i] != 0.0) {
                const double f = -m[(size_t)j * n + i] / m[(size_t)i * n + i];
                for (int c = 0; c < n; ++c) m[(size_t)j * n + c] += f * m[(size_t)i * n + c];
            }
    }
    double d = 1.0;
    for (int i = 0; i < n; ++i) d *= std::fabs(m[(size_t)i * n + i]);
    return d;
}

// inverse (Gauss-Jordan, partial pivoting) and |det| of a row-major n x n matrix
std::vector<double> inverse(std::vector<double> m, int n, double *absdet) {
    std::vector<double> inv((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i) inv[(size_t)i * n + i] = 1.0;
    double det = 1.0;
    for (int c = 0; c < n; ++c) {
        int pr = c;
        for (int r = c + 1; r < n; ++r)
            if (std::fabs(m[(size_t)r * n + c]) > std::fabs(m[(size_t)pr * n + c])) pr = r;
        if (m[(size_t)pr * n + c] == 0.0) fail(NVB_ERR_ARG, "displaced seed: singular A matrix");
        if (pr != c)
            for (int q = 0; q < n; ++q) {
                std::swap(m[(size_t)pr * n + q], m[(size_t)c * n + q]);
                std::swap(inv[(size_t)pr * n + q], inv[(size_t)c * n + q]);
            }
        const double piv = m[(size_t)c * n + c];
        det *= std::fabs(piv);
        for (int q = 0; q < n; ++q) {
            m[(size_t)c * n + q] /= piv;
            inv[(size_t)c * n + q] /= piv;
        }
        for (int r = 0; r < n; ++r)
            if (r != c && m[(size_t)r * n + c] != 0.0) {
                const double f = m[(size_t)r * n + c];
                for (int q = 0; q < n; ++q) {
                    m[(size_t)r * n + q] -= f * m[(size_t)c * n + q];
                    inv[(size_t)r * n + q] -= f * inv[(size_t)c * n + q];
                }
            }
    }
    *absdet = det;
    return inv;
}

}  // namespace

// Builds h->seed_vec = <m|n> (FP64, dimen values) and h->seed_norm = sqrt(sum <m|n>^2).
void displaced_seed(nvb_handle *h) {
    const System &sys = h->sys;
    if (!sys.neworigin) fail(NVB_ERR_STATE, "no displaced-seed data (shiftref = 0)");
    const int M = sys.M;
    if (M > SEED_MAXM) fail(NVB_ERR_ARG, "too many modes for the displaced seed");
    const std::vector<double> &a = sys.omega, &b = sys.bomega, &d = sys.dvec;
    auto T = [&](int k, int i) { return sys.tmat[(size_t)i * M + k]; };  // tmat column-major
    std::vector<double> Tm((size_t)M * M);
    for (int k = 0; k < M; ++k)
        for (int i = 0; i < M; ++i) Tm[(size_t)k * M + i] = T(k, i);
    const double detT = abs_det(Tm, M);
    std::vector<double> A((size_t)M * M, 0.0);
    for (int i = 0; i < M; ++i)
        for (int j = 0; j < M; ++j) {
            double v = 0.0;
            for (int k = 0; k < M; ++k) v += 0.5 * b[k] * T(k, i) * T(k, j);
            if (i == j) v += 0.5 * a[i];
            A[(size_t)i * M + j] = v;
        }
    double detA = 0.0;
    const std::vector<double> Ai = inverse(A, M, &detA);
    auto ai = [&](int i, int j) { return Ai[(size_t)i * M + j]; };
    std::vector<double> A1((size_t)M * M), A2((size_t)M * M), A3((size_t)M * M), A2d(M, 0.0), A3d(M, 0.0);
    for (int i = 0; i < M; ++i)
        for (int j = 0; j < M; ++j) {
            A1[(size_t)i * M + j] = ai(i, j) * std::sqrt(a[i]) * std::sqrt(a[j]) - (i == j ? 1.0 : 0.0);
            double s2 = 0.0, s3 = 0.0;
            for (int k = 0; k < M; ++k) {
                s2 += ai(i, k) * T(j, k);
                for (int l = 0; l < M; ++l) s3 += T(i, k) * ai(k, l) * T(j, l);
            }
            A2[(size_t)i * M + j] = s2 * std::sqrt(a[i]) * std::sqrt(b[j]);
            A3[(size_t)i * M + j] = s3 * std::sqrt(b[i]) * std::sqrt(b[j]);
        }
    for (int i = 0; i < M; ++i)
        for (int j = 0; j < M; ++j) {
            A2d[i] += A2[(size_t)i * M + j] * d[j] * std::sqrt(b[j]);
            A3d[i] += (A3[(size_t)j * M + i] - (i == j ? 2.0 : 0.0)) * d[j] * std::sqrt(b[j]);
        }
    double d1 = 0.0, pab = 1.0;
    for (int i = 0; i < M; ++i) d1 -= 0.5 * b[i] * d[i] * d[i];
    for (int i = 0; i < M; ++i)
        for (int j = 0; j < M; ++j) d1 += 0.25 * std::sqrt(b[i]) * d[i] * A3[(size_t)i * M + j] * d[j] * std::sqrt(b[j]);
    for (int i = 0; i < M; ++i) pab *= b[i] * a[i];
    const double d2 = std::sqrt(std::sqrt(pab) * detT / detA) * std::exp(d1);
    // initial state: the first excited mode (or the last mode, unexcited)
    int imode = M - 1;
    for (int i = 0; i < M; ++i)
        if (sys.istate[i] > 0) {
            imode = i;
            break;
        }
    const int ninit = (int)sys.istate[imode];
    double mfac = 1.0;  // prod_j 2^{m_j} m_j!
    for (int q = 1; q <= ninit; ++q) mfac *= 2.0 * q;
    // device
    SeedArgs sa{};
    sa.M = M;
    sa.dimen = sys.dimen;
    int nlev = 0;
    for (int k = 0; k < M; ++k) {
        sa.shft[k] = sys.shft[k];
        sa.nfunc[k] = (int)sys.nfunc[k];
        sa.irrep[k] = sys.irrep[k];
        nlev += (int)sys.nfunc[k] - 1;
    }
    std::vector<double> pw((size_t)M * 256, 1.0);
    for (int k = 0; k < M; ++k)
        for (int n = 1; n < 256; ++n) pw[(size_t)k * 256 + n] = pw[(size_t)k * 256 + n - 1] * 2.0 * n;
    const long long N = sys.dimen;
    const size_t mats = (size_t)3 * M * M + 2 * M + pw.size();
    std::vector<double> hm;
    hm.insert(hm.end(), A1.begin(), A1.end());
    hm.insert(hm.end(), A2.begin(), A2.end());
    hm.insert(hm.end(), A3.begin(), A3.end());
    hm.insert(hm.end(), A2d.begin(), A2d.end());
    hm.insert(hm.end(), A3d.begin(), A3d.end());
    hm.insert(hm.end(), pw.begin(), pw.end());
    double *dm = nullptr, *c0 = nullptr, *c1 = nullptr, *c2 = nullptr;
    CK(cudaMalloc((void **)&dm, mats * sizeof(double)));
    const size_t vb = (size_t)N * sizeof(double);
    try {
        CK(cudaMemcpy(dm, hm.data(), mats * sizeof(double), cudaMemcpyHostToDevice));
        const double *dA1 = dm, *dA2 = dm + (size_t)M * M, *dA2d = dm + (size_t)3 * M * M,
                     *dpw = dm + (size_t)3 * M * M + 2 * M;
        CK(cudaMalloc((void **)&c0, vb));
        CK(cudaMemsetAsync(c0, 0, vb, h->stream));
        const double one = 1.0;
        CK(cudaMemcpyAsync(c0, &one, sizeof(double), cudaMemcpyHostToDevice, h->stream));
        for (int L = 1; L <= nlev; ++L) k_fc_level<<<seed_grid(N), 256, 0, h->stream>>>(sa, dA1, dA2d, L, c0);
        CK(cudaGetLastError());
        double *res = c0;
        if (ninit > 0) {
            CK(cudaMalloc((void **)&c1, vb));
            CK(cudaMalloc((void **)&c2, vb));
            CK(cudaMemsetAsync(c1, 0, vb, h->stream));
            double *cm2 = c1, *cm1 = c0, *cm = c2;  // C_{m-2} = 0 for m = 1
            const double a3ii = A3[(size_t)imode * M + imode];
            for (int m = 1; m <= ninit; ++m) {
                k_fc_mstep<<<seed_grid(N), 256, 0, h->stream>>>(sa, dA2, 2.0 * (m - 1) * (a3ii - 1.0), -A3d[imode],
                                                                imode, cm2, cm1, cm);
                double *t = cm2;
                cm2 = cm1;
                cm1 = cm;
                cm = t;
            }
            CK(cudaGetLastError());
            res = cm1;
        }
        k_fc_scale<<<seed_grid(N), 256, 0, h->stream>>>(sa, dpw, d2 / std::sqrt(mfac), res);
        CK(cudaGetLastError());
        if (h->seed_vec) cudaFree(h->seed_vec);
        h->seed_vec = res;
        for (double *p : {c0, c1, c2})
            if (p && p != res) cudaFree(p);
        c0 = c1 = c2 = nullptr;
        const int g = seed_grid(N);
        double *part = nullptr;
        CK(cudaMalloc((void **)&part, g * sizeof(double)));
        k_sumsq<<<g, 256, 0, h->stream>>>(h->seed_vec, N, part);
        std::vector<double> hp(g);
        cudaError_t e = cudaMemcpyAsync(hp.data(), part, g * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
        cudaFree(part);
        if (e != cudaSuccess) fail(NVB_ERR_CUDA, std::string("displaced seed: ") + cudaGetErrorString(e));
        double ss = 0.0;
        for (double v : hp) ss += v;
        h->seed_norm = std::sqrt(ss);
    } catch (...) {
        cudaFree(dm);
        for (double *p : {c0, c1, c2})
            if (p && p != h->seed_vec) cudaFree(p);
        throw;
    }
    cudaFree(dm);
}

}  // namespace nvb
