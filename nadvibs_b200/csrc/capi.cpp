// extern "C" entry points of libnadvibs_gpu.so (declared in include/nadvibs.h).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <string>

#include "handle.h"

namespace nvb {
void write_header(nvb_handle *h, const char *path);
void write_eigenvalues(nvb_handle *h, const char *path, double seconds);

static thread_local std::string g_err;

void set_error(const std::string &m) { g_err = m; }
[[noreturn]] void fail(int code, const std::string &msg) { throw Error{code, msg}; }

void ensure_device(nvb_handle *h) {
    if (h->device < 0) fail(NVB_ERR_CUDA, "host-only handle (device = -1): no device work possible");
    cudaError_t e = cudaSetDevice(h->device);
    if (e != cudaSuccess) fail(NVB_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
}
}  // namespace nvb

using namespace nvb;

template <typename F>
static int guarded(F &&f) {
    try {
        f();
        return NVB_OK;
    } catch (const Error &e) {
        set_error(e.msg);
        return e.code;
    } catch (const std::bad_alloc &) {
        set_error("host allocation failed");
        return NVB_ERR_NOMEM;
    } catch (const std::exception &e) {
        set_error(e.what());
        return NVB_ERR_ARG;
    }
}

#define CKA(x)                                                                                   \
    do {                                                                                         \
        cudaError_t e_ = (x);                                                                    \
        if (e_ != cudaSuccess) fail(NVB_ERR_CUDA, std::string(#x ": ") + cudaGetErrorString(e_)); \
    } while (0)

extern "C" {

int nvb_params_default(nvb_params *p) {
    return guarded([&] {
        if (!p) fail(NVB_ERR_ARG, "null params");
        std::memset(p, 0, sizeof *p);
        // Source/secondary.f90:835-843
        p->restart = 0; p->niter = 1;
        for (int i = 0; i < 100; ++i) { p->basis[i] = 1; p->initstate[i] = 0; }
        p->nstates = 1; p->ordr = 2; p->natoms = 2; p->nmodes = 1;
        p->nirreps = 1;
        for (int i = 0; i < 10; ++i) p->npirr[i] = 0;
        p->npirr[0] = p->nmodes;
        p->shiftref = 0; p->bconv = 0; p->idroots = 0; p->soroots = 0;
        p->reorthog = 0; p->chkorthog = 100; p->nseg = 1; p->ztoler = 1e-20;
        p->maxdisk = 1000;
        for (int i = 0; i < 10; ++i) p->weights[i] = 1.0;
    });
}

int nvb_options_default(nvb_options *o) {
    return guarded([&] {
        if (!o) fail(NVB_ERR_ARG, "null options");
        std::memset(o, 0, sizeof *o);
        o->precision = NVB_FP64;
        o->device = 0;
        o->quirk_cubic = 1;
        o->quirk_lower = 1;
        o->archive_max = 0;
        o->hv_kernel = 0;
        o->seed = 12345;
    });
}

int nvb_read_basis(const char *path, nvb_params *p) {
    return guarded([&] {
        if (!path || !p) fail(NVB_ERR_ARG, "null argument");
        nvb_params q;
        nvb_params_default(&q);
        parse_basis_text(read_file(path), q);
        *p = q;
    });
}

static void create_common(nvb_handle *h, const nvb_params &p, const double *omega, const double *concoef,
                          const double *pot, const nvb_options *opt) {
    if (opt) h->opt = *opt;
    else nvb_options_default(&h->opt);
    if (h->opt.precision != NVB_FP64 && h->opt.precision != NVB_MIXED) fail(NVB_ERR_ARG, "bad precision");
    build_system(h->sys, p, omega, concoef, pot);
    h->reorthog = p.reorthog;
    h->chkorthog = p.chkorthog > 0 ? p.chkorthog : 100;
    if (h->opt.device == -1) {  // host-only handle: term table and text outputs, no device work
        h->device = -1;
        return;
    }
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0)
        fail(NVB_ERR_CUDA, std::string("no CUDA device available (") + cudaGetErrorString(e) + "); there is no CPU path");
    if (h->opt.device < 0 || h->opt.device >= ndev) fail(NVB_ERR_ARG, "device ordinal out of range");
    h->device = (int)h->opt.device;
    ensure_device(h);
    CKA(cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking));
    h->stream = h->own_stream;
    h->precision = (int)h->opt.precision;
    plan_build(h->plan, h->sys, (int)h->opt.quirk_cubic, (int)h->opt.quirk_lower);
    plan_upload(h->plan);
    if (h->opt.hv_kernel == 0 || h->opt.hv_kernel == 3) {
        if (nvb::quad_build(h->quad, h->plan, h->sys)) nvb::quad_upload(h->quad);
        if (h->opt.hv_kernel == 3 && !h->quad.ok)
            fail(NVB_ERR_ARG, "factorised quadratic kernel requested but the system does not suit it");
    }
    if ((h->opt.hv_kernel == 0 && !h->quad.ok) || h->opt.hv_kernel == 4) {
        if (nvb::cubic_build(h->cubic, h->plan, h->sys, (int)h->opt.quirk_cubic)) nvb::cubic_upload(h->cubic);
        if (h->opt.hv_kernel == 4 && !h->cubic.ok)
            fail(NVB_ERR_ARG, "factorised cubic kernel requested but the system does not suit it");
    }
    if (h->opt.hv_kernel == 0 || h->opt.hv_kernel == 2) {
        for (int i = 0; i < 2; ++i)
            if (slab_build(h->slab[i], h->plan, h->sys, (int)h->opt.quirk_cubic, i == 0 ? 8 : 4)) slab_upload(h->slab[i]);
        if (h->opt.hv_kernel == 2 && !h->slab[0].ok && !h->slab[1].ok)
            fail(NVB_ERR_ARG, "slab kernel requested but the system does not suit it");
    }
    h->reorthog = p.reorthog;
    h->chkorthog = p.chkorthog > 0 ? p.chkorthog : 100;
    h->rng_state = (uint64_t)h->opt.seed * 6364136223846793005ull + 1442695040888963407ull;
}

int nvb_create(const nvb_params *p, const double *omega, const double *concoef, const double *potterms,
               const nvb_options *opt, nvb_handle **out) {
    nvb_handle *h = nullptr;
    int rc = guarded([&] {
        if (!p || !omega || !concoef || !potterms || !out) fail(NVB_ERR_ARG, "null argument");
        h = new nvb_handle();
        create_common(h, *p, omega, concoef, potterms, opt);
    });
    if (rc != NVB_OK) {
        if (h) nvb_destroy(h);
        if (out) *out = nullptr;
        return rc;
    }
    *out = h;
    return NVB_OK;
}

int nvb_create_from_files(const char *basis_path, const char *nadvibs_path, const nvb_options *opt,
                          nvb_handle **out) {
    nvb_handle *h = nullptr;
    int rc = guarded([&] {
        if (!basis_path || !nadvibs_path || !out) fail(NVB_ERR_ARG, "null argument");
        nvb_params p;
        nvb_params_default(&p);
        parse_basis_text(read_file(basis_path), p);
        std::vector<double> om, cc, pot, disp;
        parse_nadvibs_text(read_file(nadvibs_path), p, om, cc, pot, &disp);
        h = new nvb_handle();
        create_common(h, p, om.data(), cc.data(), pot.data(), opt);
        if (p.shiftref != 0) {
            const int64_t M = p.nmodes;
            set_displaced(h->sys, disp.data(), disp.data() + M, disp.data() + 2 * M);
        }
    });
    if (rc != NVB_OK) {
        if (h) nvb_destroy(h);
        if (out) *out = nullptr;
        return rc;
    }
    *out = h;
    return NVB_OK;
}

int nvb_destroy(nvb_handle *h) {
    if (!h) return NVB_OK;
    int rc = guarded([&] {
        if (h->device >= 0) {
            cudaSetDevice(h->device);
            if (h->stream) cudaStreamSynchronize(h->stream);
            lanczos_free(h);
            plan_free(h->plan);
            slab_free(h->slab[0]);
            slab_free(h->slab[1]);
            quad_free(h->quad);
            if (h->d_g3blk) cudaFree(h->d_g3blk);
            cubic_free(h->cubic);
            ckpt_free(h);
            if (h->seed_vec) cudaFree(h->seed_vec);
            if (h->own_stream) cudaStreamDestroy(h->own_stream);
        }
    });
    delete h;
    return rc;
}

const char *nvb_last_error(void) { return g_err.c_str(); }

int nvb_hv_tile_stream(nvb_handle *h, int64_t dtype, double *bytes_per_hv, int64_t *tile_bytes, int64_t *slots,
                       int64_t *ctas_per_sm) {
    return guarded([&] {
        if (!h || !bytes_per_hv || !tile_bytes || !slots || !ctas_per_sm) fail(NVB_ERR_ARG, "null argument");
        if (dtype != NVB_DTYPE_F64 && dtype != NVB_DTYPE_F32) fail(NVB_ERR_ARG, "dtype must be NVB_DTYPE_F64 or NVB_DTYPE_F32");
        if (h->device < 0) fail(NVB_ERR_STATE, "host-only handle");
        const int idx = dtype == NVB_DTYPE_F32 ? 1 : 0, eb = idx ? 4 : 8;
        *bytes_per_hv = 0.0;
        *tile_bytes = *slots = *ctas_per_sm = 0;
        int nsm = 0;
        CKA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, h->device));
        // fraction of tiles whose neighbour along slow mode k at shift s lies inside the basis
        auto inside = [](int nf, int s) { return (double)std::max(nf - std::abs(s), 0) / (double)nf; };
        if (h->quad.ok) {
            const nvb::QuadPlan &q = h->quad;
            double items = 0.0;
            for (const nvb::QuadItem &it : q.items) {
                double f = 1.0;
                if (it.kind != nvb::QI_OWN) f *= inside(q.slow_nfunc[it.k], it.sk);
                if (it.kind == nvb::QI_PAIR) f *= inside(q.slow_nfunc[it.l], it.sl);
                items += f;
            }
            *bytes_per_hv = items * (double)q.ntiles * (double)q.TF * eb;
            *tile_bytes = (int64_t)q.TF * eb;
            *slots = q.nslot[idx];
            *ctas_per_sm = q.grid[idx] > 0 ? std::max<int64_t>(1, q.grid[idx] / nsm) : 1;
        } else if (h->cubic.ok && h->cubic.prec_ok[idx]) {
            const nvb::CubPlan &c = h->cubic;
            double items = 0.0;
            for (const nvb::CubItem &it : c.items) {
                double f = 1.0;
                for (int k = 0; k < it.nsh; ++k) f *= inside(c.slow_nfunc[it.md[k]], it.sv[k]);
                items += f;
            }
            *bytes_per_hv = items * (double)c.ntiles * (double)c.TF * eb;
            *tile_bytes = (int64_t)c.TF * eb;
            *slots = c.nslot[idx];
            *ctas_per_sm = c.grid[idx] > 0 ? std::max<int64_t>(1, c.grid[idx] / nsm) : c.per_sm[idx];
        }
    });
}

int nvb_hv_kernel_in_use(nvb_handle *h, int64_t dtype, int64_t *kernel) {
    return guarded([&] {
        if (!h || !kernel) fail(NVB_ERR_ARG, "null argument");
        if (dtype != NVB_DTYPE_F64 && dtype != NVB_DTYPE_F32) fail(NVB_ERR_ARG, "dtype must be NVB_DTYPE_F64 or NVB_DTYPE_F32");
        if (h->device < 0) fail(NVB_ERR_STATE, "host-only handle");
        if (h->quad.ok) *kernel = 3;
        else if (h->cubic.ok && h->cubic.prec_ok[dtype == NVB_DTYPE_F32 ? 1 : 0]) *kernel = 4;
        else if (h->slab[dtype == NVB_DTYPE_F32 ? 1 : 0].ok) *kernel = 2;
        else *kernel = 1;
    });
}

int nvb_get_sizes(nvb_handle *h, int64_t *dimen, int64_t *nstates, int64_t *nmodes, int64_t *nterms, int64_t *npot,
                  int64_t *iters) {
    return guarded([&] {
        if (!h) fail(NVB_ERR_ARG, "null handle");
        if (dimen) *dimen = h->sys.dimen;
        if (nstates) *nstates = h->sys.S;
        if (nmodes) *nmodes = h->sys.M;
        if (nterms) *nterms = (int64_t)h->sys.terms.size();
        if (npot) *npot = (int64_t)h->sys.potterms.size();
        if (iters) *iters = h->iters;
    });
}

int nvb_get_terms(nvb_handle *h, int64_t *tcnt, int64_t *tmode, int64_t *tpow, int64_t *tnpair, int64_t *tpa,
                  int64_t *tpb, double *tcoef) {
    return guarded([&] {
        if (!h) fail(NVB_ERR_ARG, "null handle");
        const int S = h->sys.S;
        for (size_t t = 0; t < h->sys.terms.size(); ++t) {
            const Term &T = h->sys.terms[t];
            if (tcnt) tcnt[t] = T.nm;
            for (int l = 0; l < 4; ++l) {
                if (tmode) tmode[t * 4 + l] = l < T.nm ? T.mode[l] + 1 : 0;
                if (tpow) tpow[t * 4 + l] = l < T.nm ? T.pow[l] : 0;
            }
            if (tnpair) tnpair[t] = (int64_t)T.pairs.size();
            for (int q = 0; q < S * S; ++q) {
                const bool on = q < (int)T.pairs.size();
                if (tpa) tpa[t * S * S + q] = on ? T.pairs[q].a + 1 : 0;
                if (tpb) tpb[t * S * S + q] = on ? T.pairs[q].b + 1 : 0;
                if (tcoef) tcoef[t * S * S + q] = on ? T.pairs[q].coef : 0.0;
            }
        }
    });
}

int nvb_set_precision(nvb_handle *h, int64_t precision) {
    return guarded([&] {
        if (!h) fail(NVB_ERR_ARG, "null handle");
        if (precision != NVB_FP64 && precision != NVB_MIXED) fail(NVB_ERR_ARG, "bad precision");
        ensure_device(h);
        if (precision != h->precision) {
            CKA(cudaStreamSynchronize(h->stream));
            for (int i = 0; i < 3; ++i)
                if (h->buf[i]) { cudaFree(h->buf[i]); h->buf[i] = nullptr; }
            {
                const int kind = h->arch_kind;
                const int64_t cap = archive_capacity(h);
                const std::string path = h->arch_path;
                archive_free(h);  // the archive's vectors are in the old precision: start afresh
                archive_configure(h, kind, cap, path.c_str());
            }
            h->precision = (int)precision;
        }
        h->seeded = false;
        h->iters = 0;
    });
}

int nvb_set_stream(nvb_handle *h, void *stream) {
    return guarded([&] {
        if (!h) fail(NVB_ERR_ARG, "null handle");
        h->stream = stream ? (cudaStream_t)stream : h->own_stream;
    });
}

int nvb_synchronize(nvb_handle *h) {
    return guarded([&] {
        if (!h) fail(NVB_ERR_ARG, "null handle");
        ensure_device(h);
        CKA(cudaStreamSynchronize(h->stream));
        check_kernel_flags(h);
    });
}

int nvb_set_fault_test(nvb_handle *h, int64_t mode) {
    return guarded([&] {
        if (!h) fail(NVB_ERR_ARG, "null handle");
        if (mode != 0 && mode != 1) fail(NVB_ERR_ARG, "fault-test mode must be 0 or 1");
        h->quad.test_nocopy = (int)mode;
        h->cubic.test_nocopy = (int)mode;
    });
}

int nvb_hv(nvb_handle *h, const void *x, void *y, int64_t dtype) {
    return guarded([&] {
        if (!h || !x || !y) fail(NVB_ERR_ARG, "null argument");
        if (dtype != NVB_DTYPE_F64 && dtype != NVB_DTYPE_F32) fail(NVB_ERR_ARG, "bad dtype");
        if (x == y) fail(NVB_ERR_ARG, "x and y must not alias");
        ensure_device(h);
        hv_any(h, x, y, (int)dtype, nullptr, nullptr, nullptr);
    });
}

int nvb_seed(nvb_handle *h, const double *weights) {
    return guarded([&] {
        if (!h) fail(NVB_ERR_ARG, "null handle");
        ensure_device(h);
        const auto t0 = std::chrono::steady_clock::now();
        lanczos_seed(h, weights);
        h->seed_secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    });
}

int nvb_write_seed_report(nvb_handle *h, const char *path) {
    return guarded([&] {
        if (!h || !path) fail(NVB_ERR_ARG, "null argument");
        ensure_device(h);
        write_seed_report(h, path);
    });
}

int nvb_lanczos(nvb_handle *h, int64_t niter, double *alpha, double *beta) {
    return guarded([&] {
        if (!h) fail(NVB_ERR_ARG, "null handle");
        ensure_device(h);
        try {
            lanczos_run(h, niter);
        } catch (const Error &e) {
            if (alpha) std::memcpy(alpha, h->alpha.data() + 1, h->iters * sizeof(double));
            if (beta) std::memcpy(beta, h->beta.data(), (h->iters + 1) * sizeof(double));
            throw;
        }
        if (alpha) std::memcpy(alpha, h->alpha.data() + 1, h->iters * sizeof(double));
        if (beta) std::memcpy(beta, h->beta.data(), (h->iters + 1) * sizeof(double));
    });
}

int nvb_ritz(nvb_handle *h, int64_t n, double *E, double *bji, double *inten, int64_t *sign, double *vect) {
    return guarded([&] {
        if (!h || !E) fail(NVB_ERR_ARG, "null argument");
        if (n < 1 || n > h->iters) fail(NVB_ERR_STATE, "n must be in 1..iterations done");
        std::vector<double> V((size_t)n * n);
        tridiag_eigen(n, h->alpha.data() + 1, h->beta.data() + 1, E, V.data());
        for (int64_t i = 0; i < n; ++i) {
            const double s1 = V[(size_t)i * n], sn = V[(size_t)i * n + n - 1];
            if (bji) bji[i] = std::fabs(h->beta[n] * sn);
            if (inten) inten[i] = s1 * s1;
            if (sign) sign[i] = s1 < 0 ? -1 : 1;
        }
        if (vect) std::memcpy(vect, V.data(), V.size() * sizeof(double));
    });
}

int nvb_write_eigenvalues(nvb_handle *h, const char *path) {
    return guarded([&] {
        if (!h || !path) fail(NVB_ERR_ARG, "null argument");
        auto t0 = std::chrono::steady_clock::now();
        // timing printed is that of the eigen-solve itself
        write_eigenvalues(h, path, 0.0);
        (void)t0;
    });
}

int nvb_write_header(nvb_handle *h, const char *path) {
    return guarded([&] {
        if (!h || !path) fail(NVB_ERR_ARG, "null argument");
        write_header(h, path);
    });
}

int nvb_lanczos_vectors(nvb_handle *h, void **cur, double *scur, void **prev, double *sprev, void **res,
                        double *sres) {
    return guarded([&] {
        if (!h) fail(NVB_ERR_ARG, "null handle");
        if (!h->seeded) fail(NVB_ERR_STATE, "no Lanczos state");
        ensure_device(h);
        double sc[3];
        CKA(cudaMemcpyAsync(sc, h->d_scale, sizeof sc, cudaMemcpyDeviceToHost, h->stream));
        CKA(cudaStreamSynchronize(h->stream));
        if (cur) *cur = h->buf[h->cur];
        if (scur) *scur = sc[h->cur];
        if (prev) *prev = h->buf[h->prev];
        if (sprev) *sprev = sc[h->prev];
        if (res) *res = h->buf[h->work];
        if (sres) *sres = sc[h->work];
    });
}

int nvb_set_timing(nvb_handle *h, int64_t enable) {
    return guarded([&] {
        if (!h) fail(NVB_ERR_ARG, "null handle");
        h->timing = enable != 0;
        h->t_hv_ms = h->t_iter_ms = 0.0;
        h->n_timed = 0;
    });
}

int nvb_get_timing(nvb_handle *h, double *hv_ms, double *iter_ms, int64_t *n) {
    return guarded([&] {
        if (!h) fail(NVB_ERR_ARG, "null handle");
        if (hv_ms) *hv_ms = h->t_hv_ms;
        if (iter_ms) *iter_ms = h->t_iter_ms;
        if (n) *n = h->n_timed;
    });
}

int nvb_dot(nvb_handle *h, const void *a, double sa, const void *b, double sb, int64_t dtype, double *result) {
    return guarded([&] {
        if (!h || !a || !b || !result) fail(NVB_ERR_ARG, "null argument");
        if (dtype != NVB_DTYPE_F64 && dtype != NVB_DTYPE_F32) fail(NVB_ERR_ARG, "bad dtype");
        ensure_device(h);
        *result = device_dot(h, a, sa, b, sb, (int)dtype);
    });
}

int nvb_save_restart(nvb_handle *h, const char *dir, const char *vecdir) {
    return guarded([&] {
        if (!h) fail(NVB_ERR_ARG, "null handle");
        ensure_device(h);
        save_restart(h, dir, vecdir);
    });
}

int nvb_load_restart(nvb_handle *h, const char *dir, const char *vecdir) {
    return guarded([&] {
        if (!h) fail(NVB_ERR_ARG, "null handle");
        ensure_device(h);
        load_restart(h, dir, vecdir);
    });
}

int nvb_lead_contributors(nvb_handle *h, int64_t nroots, int64_t k, int64_t *state, int64_t *index, double *c2,
                          int64_t *phase, double *pct, const char *rootinfo_path) {
    return guarded([&] {
        if (!h) fail(NVB_ERR_ARG, "null handle");
        ensure_device(h);
        lead_contributors(h, nroots, k, state, index, c2, phase, pct, rootinfo_path);
    });
}

int nvb_set_archive(nvb_handle *h, int64_t kind, int64_t max_vectors, const char *path) {
    return guarded([&] {
        if (!h) fail(NVB_ERR_ARG, "null handle");
        ensure_device(h);
        if (h->stream) CKA(cudaStreamSynchronize(h->stream));
        archive_configure(h, (int)kind, max_vectors, path);  // filled from the next nvb_seed on
    });
}

int nvb_reorth_log(nvb_handle *h, int64_t max_entries, int64_t *iteration, int64_t *lo, int64_t *hi, int64_t *count) {
    return guarded([&] {
        if (!h || !count) fail(NVB_ERR_ARG, "null argument");
        const int64_t n = (int64_t)h->orth_log.size();
        *count = n;
        for (int64_t i = 0; i < std::min(n, max_entries); ++i) {
            if (iteration) iteration[i] = h->orth_log[(size_t)i][0];
            if (lo) lo[i] = h->orth_log[(size_t)i][1];
            if (hi) hi[i] = h->orth_log[(size_t)i][2];
        }
    });
}

int nvb_reorth_omega(nvb_handle *h, int64_t n, double *omega1, double *omega2, double *omega2_step) {
    return guarded([&] {
        if (!h) fail(NVB_ERR_ARG, "null handle");
        if (n < 0) fail(NVB_ERR_ARG, "n < 0");
        for (int64_t i = 0; i <= n; ++i) {
            if (omega1) omega1[i] = i < (int64_t)h->omega1.size() ? h->omega1[(size_t)i] : 0.0;
            if (omega2) omega2[i] = i < (int64_t)h->omega2.size() ? h->omega2[(size_t)i] : 0.0;
            if (omega2_step) omega2_step[i] = i < (int64_t)h->omega_pre.size() ? h->omega_pre[(size_t)i] : 0.0;
        }
    });
}

int nvb_set_reorthog(nvb_handle *h, int64_t reorthog, int64_t chkorthog) {
    return guarded([&] {
        if (!h) fail(NVB_ERR_ARG, "null handle");
        if (reorthog < 0 || chkorthog < 1) fail(NVB_ERR_ARG, "reorthog >= 0 and chkorthog >= 1 required");
        h->reorthog = reorthog;
        h->chkorthog = chkorthog;
    });
}

int nvb_hv_adjoint_coeffs(nvb_handle *h, const void *u, const void *v, int64_t dtype, double *grad) {
    return guarded([&] {
        if (!h || !u || !v || !grad) fail(NVB_ERR_ARG, "null argument");
        if (dtype != NVB_DTYPE_F64 && dtype != NVB_DTYPE_F32) fail(NVB_ERR_ARG, "bad dtype");
        ensure_device(h);
        hv_adjoint(h, u, v, (int)dtype, grad);
    });
}

int nvb_convolve(const double *center, const double *height, int64_t n, const double *grid, int64_t ngrid,
                 double width, int64_t shape, double *out) {
    return guarded([&] {
        if ((n > 0 && (!center || !height)) || (ngrid > 0 && (!grid || !out))) fail(NVB_ERR_ARG, "null argument");
        convolve_lines(center, height, n, grid, ngrid, width, shape, out);
    });
}

int nvb_spin_orbit(nvb_handle *h, int64_t soroots, int64_t nroots, double *energy_ev, double *amp, double *overlap,
                   const char *sodata_path) {
    return guarded([&] {
        if (!h) fail(NVB_ERR_ARG, "null handle");
        ensure_device(h);
        spin_orbit(h, soroots, nroots, energy_ev, amp, overlap, sodata_path);
    });
}

int nvb_set_displaced_seed(nvb_handle *h, const double *bomega, const double *dvec, const double *tmat) {
    return guarded([&] {
        if (!h || !bomega || !dvec || !tmat) fail(NVB_ERR_ARG, "null argument");
        set_displaced(h->sys, bomega, dvec, tmat);
        if (h->seed_vec) cudaFree(h->seed_vec);
        h->seed_vec = nullptr;
        h->seed_norm = 0.0;
    });
}

int nvb_seed_overlap(nvb_handle *h, double *overlap) {
    return guarded([&] {
        if (!h || !overlap) fail(NVB_ERR_ARG, "null argument");
        if (!h->sys.neworigin) {
            *overlap = 1.0;
            return;
        }
        ensure_device(h);
        if (!h->seed_vec) displaced_seed(h);
        *overlap = h->seed_norm;
    });
}

int nvb_set_checkpoints(nvb_handle *h, int64_t k) {
    return guarded([&] {
        if (!h) fail(NVB_ERR_ARG, "null handle");
        if (k < -1) fail(NVB_ERR_ARG, "checkpoint interval < -1");
        ensure_device(h);
        if (k != h->ck_k) ckpt_free(h);
        h->ck_k = k;
        h->ck_count = 0;
    });
}

int nvb_set_backward_memory(nvb_handle *h, int64_t bytes) {
    return guarded([&] {
        if (!h) fail(NVB_ERR_ARG, "null handle");
        if (bytes < 0) fail(NVB_ERR_ARG, "memory budget < 0");
        h->grad_budget = bytes;
    });
}

int nvb_backward_plan(nvb_handle *h, int64_t *plan) {
    return guarded([&] {
        if (!h || !plan) fail(NVB_ERR_ARG, "null argument");
        for (int i = 0; i < 4; ++i) plan[i] = h->bw_plan[i];
    });
}

int nvb_lanczos_backward(nvb_handle *h, int64_t n, const double *alpha_bar, const double *beta_bar, int64_t k,
                         double *grad) {
    return guarded([&] {
        if (!h || !alpha_bar || !grad) fail(NVB_ERR_ARG, "null argument");
        ensure_device(h);
        lanczos_backward(h, n, alpha_bar, beta_bar, k, grad);
    });
}

int nvb_hellmann_feynman(nvb_handle *h, int64_t nroots, double *grad, double *energies) {
    return guarded([&] {
        if (!h || !grad) fail(NVB_ERR_ARG, "null argument");
        ensure_device(h);
        hellmann_feynman(h, nroots, grad, energies);
    });
}

}  // extern "C"
