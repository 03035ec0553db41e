/*
 * nadvibs.h -- C ABI of the B200 Lanczos stage of NadVibS (libnadvibs_gpu.so).
 *
 * Drop-in boundary for the Lanczos stage of the reference program
 * (Source/main.f90:61-79): a Fortran driver binds these entry points through
 * ISO_C_BINDING (all integers int64_t, reals double, strings NUL-terminated), a C driver
 * calls them directly, and the Python package binds them with ctypes.
 *
 * Conventions
 *  - Every entry point returns 0 on success and a negative NVB_ERR_* code on failure;
 *    nvb_last_error() returns a thread-local message for the last failure.  The
 *    reference prints and continues on errors (Source/top.f90:396,1303-1308); here
 *    failures are reported to the caller instead.
 *  - A handle owns its device memory and a CUDA stream; caller-owned host arrays are
 *    never retained.  One host thread per handle.
 *  - Vectors passed by device pointer use the reference layout q(dimen, nstates),
 *    column-major: element (row r, state s) at s*dimen + r, rows ordered with the last
 *    mode fastest (shft(k) = prod_{j>k} nfunc(j), Source/top.f90:379-386).
 *  - Energies are hartree unless stated otherwise; AU2WAVE = 219474.6313705.
 *  - There is no CPU fallback: without a usable CUDA device nvb_create* fails.
 */
#ifndef NADVIBS_H
#define NADVIBS_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NVB_OK 0
#define NVB_ERR_ARG (-1)       /* invalid argument or size */
#define NVB_ERR_IO (-2)        /* file missing, unreadable or malformed */
#define NVB_ERR_CUDA (-3)      /* CUDA runtime error or no device */
#define NVB_ERR_STATE (-4)     /* call out of order (e.g. ritz before lanczos) */
#define NVB_ERR_NOMEM (-5)     /* device or host allocation failed */
#define NVB_ERR_BREAKDOWN (-6) /* Lanczos breakdown: beta below threshold or not finite */

#define NVB_FP64 0  /* vectors and H.v in FP64 */
#define NVB_MIXED 1 /* vectors and H.v in FP32, recurrence/dots/eigensolve in FP64 */

#define NVB_DTYPE_F64 0
#define NVB_DTYPE_F32 1

typedef struct nvb_handle nvb_handle;

/* The &NADVIBS namelist of basis.in, with the reference's defaults and array bounds
 * (get_keywords, Source/secondary.f90:826-870). */
typedef struct nvb_params {
    int64_t niter, natoms, nmodes, nstates, ordr, restart, bconv, idroots, soroots;
    int64_t reorthog, chkorthog, nseg, shiftref, nirreps;
    double ztoler, maxdisk;
    int64_t basis[100];
    int64_t initstate[100];
    int64_t npirr[10];
    double weights[10];
} nvb_params;

/* Build options (not part of the reference input). */
typedef struct nvb_options {
    int64_t precision;     /* NVB_FP64 or NVB_MIXED */
    int64_t device;        /* CUDA device ordinal; -1 = host-only handle (term table and
                              text outputs only, every device entry point fails) */
    int64_t quirk_cubic;   /* 1 (default): <m|x^3|m+-1> as the reference tabulates it
                              (Source/function.f90:225-227, a factor 3 short); 0: exact */
    int64_t quirk_lower;   /* 1 (default): constant / even-power couplings between different
                              states applied to the lower triangle only, as the reference
                              does (Source/top.f90:752-754); 0: symmetric */
    int64_t archive_max;   /* max Lanczos vectors kept on the device for Ritz vectors /
                              re-orthogonalisation; 0 = none (two-pass Ritz vectors) */
    int64_t hv_kernel;     /* 0 = automatic choice (factorised quadratic kernel where the
                              system suits it, else the factorised cubic kernel, else the
                              slab-tiled kernel, else gather); 1 = gather kernel; 2 = slab-tiled
                              kernel; 3 = factorised quadratic kernel (ordr <= 2, state-diagonal
                              bilinear terms); 4 = factorised cubic kernel (ordr <= 3, couplings
                              between different states constant or linear) */
    int64_t seed;          /* seed of the omega-recurrence noise (the reference is unseeded) */
} nvb_options;

/* Defaults of both structures.  Replaces the assignments of Source/secondary.f90:835-843. */
int nvb_params_default(nvb_params *p);
int nvb_options_default(nvb_options *o);

/* Parse basis.in (the &NADVIBS group).  Replaces get_keywords (Source/secondary.f90:826-870)
 * without the restart bookkeeping, which nvb_load_restart performs. */
int nvb_read_basis(const char *path, nvb_params *p);

/* Read basis.in + nadvibs.in and build the device plan.  Replaces read_basis +
 * read_constants + initialize_elements (Source/top.f90:32-246,344-634).  Only
 * shiftref=0 inputs are accepted (the Duschinsky seed is not built). */
int nvb_create_from_files(const char *basis_path, const char *nadvibs_path, const nvb_options *opt,
                          nvb_handle **out);

/* Same, from memory.  omega[nmodes] (hartree), concoef[nstates(nstates+1)/2] in block order
 * k = i(i-1)/2 + j (i >= j), potterms = for each block, for each order d = 1..ordr, the
 * C(nmodes+d-1, d) coefficients in the nadvibs.in monomial order (Source/top.f90:122-168),
 * concatenated without padding. */
int nvb_create(const nvb_params *p, const double *omega, const double *concoef, const double *potterms,
               const nvb_options *opt, nvb_handle **out);

int nvb_destroy(nvb_handle *h);
const char *nvb_last_error(void);

/* Sizes: dimen = prod(nfunc) (rows per state), total = dimen*nstates, nterms = distinct
 * monomials after the merge, npot = number of potterms values, iters = completed Lanczos
 * iterations. */
int nvb_get_sizes(nvb_handle *h, int64_t *dimen, int64_t *nstates, int64_t *nmodes, int64_t *nterms,
                  int64_t *npot, int64_t *iters);

/* Which H.v kernel a product with vectors of this dtype runs (16-byte aligned vectors):
 * 1 = gather, 2 = slab-tiled, 3 = factorised quadratic, 4 = factorised cubic.  No reference
 * counterpart (the
 * reference has one product routine, Source/top.f90:672-818). */
int nvb_hv_kernel_in_use(nvb_handle *h, int64_t dtype, int64_t *kernel);

/* The merged term table in the reference's representation (nzindx/nzblks/nzcoef of
 * Source/top.f90:199-231): for term t, tcnt[t] distinct modes, tmode[t*4+l] (1-based) and
 * tpow[t*4+l]; tnpair[t] state pairs tpa/tpb[t*nstates^2+q] (1-based) with coefficient
 * tcoef[t*nstates^2+q] (scaled by 1/prod omega^(p/2)). */
int nvb_get_terms(nvb_handle *h, int64_t *tcnt, int64_t *tmode, int64_t *tpow, int64_t *tnpair,
                  int64_t *tpa, int64_t *tpb, double *tcoef);

/* Precision of subsequent Lanczos runs (resets the Lanczos state). */
int nvb_set_precision(nvb_handle *h, int64_t precision);

/* Run the handle's work on a caller stream (cudaStream_t passed as void*, e.g.
 * cudaStreamLegacy for the legacy default stream); NULL restores the handle-owned stream,
 * which does not synchronise with the legacy default stream. */
int nvb_set_stream(nvb_handle *h, void *stream);
/* Waits for the handle's stream and reports a tiled H.v kernel that gave up waiting for a
 * shared-memory copy (NVB_ERR_CUDA; the error is reported once and the handle stays usable). */
int nvb_synchronize(nvb_handle *h);

/* Failure-detection test hook (no reference counterpart): mode 1 makes the factorised
 * quadratic and cubic H.v kernels issue none of their copies, so every wait of its consumer warps runs out
 * (after a short poll limit in this mode); the kernel raises its abort flag, finishes without
 * touching the missing data and sets its error word, which the next nvb_synchronize /
 * nvb_lanczos reports as NVB_ERR_CUDA.  Mode 0 (default) restores normal operation. */
int nvb_set_fault_test(nvb_handle *h, int64_t mode);

/* y = H x on device pointers of dtype NVB_DTYPE_F64 or NVB_DTYPE_F32 (both vectors the same
 * dtype).  Replaces Hv (Source/top.f90:672-818).  Stream-ordered, asynchronous. */
int nvb_hv(nvb_handle *h, const void *x, void *y, int64_t dtype);

/* Generate the seed vector: |0...0> in every state weighted by weights[nstates] and
 * normalised (generate_initialvec, simple branch, Source/secondary.f90:727-783).
 * weights may be NULL (basis.in weights).  Resets the Lanczos state; beta(0)=||seed||. */
int nvb_seed(nvb_handle *h, const double *weights);

/* Run niter further Lanczos iterations (update_lanczos + Hv + lanczos_step [+ set_omega +
 * partial_orthog], Source/main.f90:63-71, Source/top.f90:646-1005) with the handle's
 * reorthogonalisation settings.  alpha receives alpha(1..iters), beta beta(0..iters) for
 * ALL iterations done so far (iters = previous + niter); either may be NULL. */
int nvb_lanczos(nvb_handle *h, int64_t niter, double *alpha, double *beta);

/* Re-orthogonalisation mode as in basis.in (Source/secondary.f90:847-848): reorthog 0 none,
 * 1 omega recurrence with exact checks every chkorthog iterations, 2 exact overlaps;
 * partial re-orthogonalisation (set_omega + partial_orthog, Source/top.f90:844-1005) runs after
 * every iteration from the second.  It needs every Lanczos vector in the archive (options
 * archive_max, or nvb_set_archive, >= total iterations), else nvb_lanczos fails with
 * NVB_ERR_ARG.  The
 * omega recurrence's random draws use the options' seed (the reference is unseeded). */
int nvb_set_reorthog(nvb_handle *h, int64_t reorthog, int64_t chkorthog);

/* Where the archive of Lanczos vectors lives, from the next nvb_seed on (the reference's disk
 * archive nadvibs.34.<rank>, Source/top.f90:570-571,595-598, written and read by write_ga /
 * read_ga, Source/secondary.f90:273-308): kind 0 device memory (the same as the options'
 * archive_max = max_vectors), 1 pinned host memory (allocated in blocks as the run grows), 2
 * the file at path in the reference's layout (each vector as nstates records of dimen FP64
 * values, vector after vector, whatever the handle's precision).  Host memory and the file are
 * streamed to the device in chunks of whole vectors for re-orthogonalisation and Ritz vectors.
 * With a file archive that holds every earlier vector, re-orthogonalisation resumes after
 * nvb_load_restart. */
int nvb_set_archive(nvb_handle *h, int64_t kind, int64_t max_vectors, const char *path);

/* The intervals of Lanczos vectors that partial re-orthogonalisation (partial_orthog,
 * Source/top.f90:910-1005) orthogonalised against since the seed, in order: entry i =
 * (iteration[i], lo[i], hi[i]), 1-based, at most max_entries written (arrays may be NULL);
 * *count = the number of entries.  No reference counterpart (the reference does not report
 * them). */
int nvb_reorth_log(nvb_handle *h, int64_t max_entries, int64_t *iteration, int64_t *lo, int64_t *hi,
                   int64_t *count);

/* The orthogonality estimates of re-orthogonalisation (set_omega, Source/top.f90:844-908),
 * entries 0..n: omega1 = omega(1,:) and omega2 = omega(2,:) as they stand (the reference writes
 * both to restart.log), omega2_step = omega(2,:) of the last iteration as partial_orthog saw
 * it, before the resets of the orthogonalised intervals.  Arrays may be NULL.  No reference
 * counterpart as an entry point. */
int nvb_reorth_omega(nvb_handle *h, int64_t n, double *omega1, double *omega2, double *omega2_step);

/* Ritz system of T_n, n <= iters (compute_ritzsystem, Source/secondary.f90:240-257):
 * E[n] ascending (hartree), bji[n] = |beta(n) s(n,i)|, inten[n] = s(1,i)^2, sign[n] of
 * s(1,i); vect (optional, n*n column-major) the eigenvectors of T_n. */
int nvb_ritz(nvb_handle *h, int64_t n, double *E, double *bji, double *inten, int64_t *sign, double *vect);

/* Write output.dat's eigenvalue section (compute_eigenvalues, Source/top.f90:1051-1113)
 * for T_n, n = iters, with bjiconv = 10^-bconv from basis.in, appending to path. */
int nvb_write_eigenvalues(nvb_handle *h, const char *path);

/* Append the seed section of output.dat after nvb_seed (generate_initialvec's report,
 * Source/secondary.f90:351-802): for a displaced seed (shiftref != 0) the number of basis
 * functions per quanta-sum level and the <m| levels built; for either seed the overlap with the
 * initial state, its (up to) 40 dominant basis functions with their quanta, the normalisation
 * of the initial Lanczos vector by the state weights and the time nvb_seed took. */
int nvb_write_seed_report(nvb_handle *h, const char *path);

/* Write the output.dat header for the job (print_basis, Source/top.f90:248-342), replacing
 * path. */
int nvb_write_header(nvb_handle *h, const char *path);

/* Device pointer to the current Lanczos vector v_i, v_{i-1} and the residual (dtype of the
 * handle's precision) with their scale factors (v = scale * buffer). */
int nvb_lanczos_vectors(nvb_handle *h, void **cur, double *scur, void **prev, double *sprev, void **res,
                        double *sres);

/* Restart state (make_restart / load_restartinfo + restore, Source/top.f90:1007-1049,
 * Source/secondary.f90:872-892, Source/top.f90:557-588): restart.log (text: iteration counts,
 * alpha(1:n), beta(0:n), and omega(1,0:n), omega(2,0:n) when re-orthogonalising) in dir
 * (NULL = current directory, where the reference keeps it) and nadvibs.35.0 (q1 = v(n-1),
 * q2 = v(n), q3 = the unnormalised residual, each as nstates records of dimen FP64 values) in
 * vecdir (the reference's -o scratch directory; NULL = dir).  nvb_load_restart resumes the
 * handle at iteration n; as the reference, it renames restart.log to restart.log.old and
 * deletes nadvibs.35.0 once loaded.  Restarting from an iteration before the last one (which
 * needs the reference's disk archive) is rejected. */
int nvb_save_restart(nvb_handle *h, const char *dir, const char *vecdir);
int nvb_load_restart(nvb_handle *h, const char *dir, const char *vecdir);

/* Ritz vectors of the lowest nroots roots of T_n (n = iterations done) and their lead basis
 * functions (identify_roots, Source/top.f90:1124-1230): for root r and j < k, the j-th
 * largest |psi|^2 entry: state[r*k+j] (1-based), index[r*k+j] (1-based row),
 * c2[r*k+j] = |psi|^2, phase[r*k+j] = sign of psi; pct[r*nstates+s] = percent weight of state
 * s.  Vectors come from the device archive when it holds every iteration (options
 * archive_max), otherwise the recurrence is replayed from the seed with the stored
 * alpha/beta (two-pass Lanczos).  rootinfo_path (optional) receives rootinfo.dat in the
 * reference's format.  Any output array may be NULL. */
int nvb_lead_contributors(nvb_handle *h, int64_t nroots, int64_t k, int64_t *state, int64_t *index, double *c2,
                          int64_t *phase, double *pct, const char *rootinfo_path);

/* Spin-orbit parameters of the lowest soroots Ritz pairs (Source/top.f90:1153-1175 and
 * 1231-1252, the soroots branch of identify_roots): energy_ev[i] = E_i in eV,
 * amp[i] = sqrt(I_i / I_max) * sign_i with I_max the largest intensity among the lowest nroots
 * roots (the reference uses nroots = max(idroots, soroots)) and sign_i the sign of the first
 * eigenvector component, and overlap[((i*soroots + j)*nstates + k)*nstates + l] =
 * <psi_i restricted to state k | psi_j restricted to state l> for j < i (zero for j >= i),
 * from the Ritz vectors (archive or two-pass replay).  sodata_path (optional) receives
 * sodata.in in the reference's format (its overlap rows only for 2 or 3 states, as the
 * reference writes them).  Any output array may be NULL. */
int nvb_spin_orbit(nvb_handle *h, int64_t soroots, int64_t nroots, double *energy_ev, double *amp, double *overlap,
                   const char *sodata_path);

/* Broadening of a line spectrum on the GPU (the post-step programs of the reference):
 * out[g] = sum_j height[j] f(grid[g] - center[j]) over host arrays, lines summed in order in
 * FP64, on the current CUDA device.  shape 0: Gaussian of full width at half maximum `width`
 * (convolve/main.f90:24-43 with convolve/sub.f90's gaussian); shape 1: exp(-t^2/2), t =
 * (x-c)/width (convolve.py's Gaussian); shape 2: 1/width/(1+t^2) (convolve.py's Lorentzian).
 * No normalisation (convolve.py divides by the maximum afterwards). */
int nvb_convolve(const double *center, const double *height, int64_t n, const double *grid, int64_t ngrid,
                 double width, int64_t shape, double *out);

/* Adjoint contraction of the gradient path (no counterpart in the reference):
 * grad[npot + nstblks + nmodes] = d<u|H(theta)|v>/d theta for theta = (the potterms of
 * nvb_create's layout -- every nadvibs.in expansion coefficient, zero ones included --, the
 * block constants concoef, the frequencies omega).  u, v are device vectors of dtype in the
 * reference layout.  Couplings between different states are differentiated in their
 * symmetric form (the lower-triangle-only constant coupling of the reference is a quirk of
 * the forward product; see nvb_options.quirk_lower). */
int nvb_hv_adjoint_coeffs(nvb_handle *h, const void *u, const void *v, int64_t dtype, double *grad);

/* Hellmann-Feynman gradients of the lowest nroots Ritz energies of T_n (n = iterations
 * done): grad[r*ncoef + i] = <psi_r|dH/dtheta_i|psi_r>/<psi_r|psi_r> with the Ritz vectors
 * psi_r (archive or two-pass replay, as nvb_lead_contributors), ncoef = npot + nstblks +
 * nmodes in the layout of nvb_hv_adjoint_coeffs; energies[nroots] (optional) the Ritz values.
 * Exact derivatives for converged roots. */
int nvb_hellmann_feynman(nvb_handle *h, int64_t nroots, double *grad, double *energies);

/* Displaced / Duschinsky Franck-Condon seed (shiftref != 0; generate_initialvec's neworigin
 * branch, Source/secondary.f90:372-726): the seed's state blocks hold <m|n>, the overlap of the
 * initial vibrational state |m> -- frequencies bomega[nmodes] (hartree) in the coordinates
 * y = T x + dvec of the Hamiltonian's modes x, T[k][i] = tmat[i*nmodes + k] (column-major, as
 * nadvibs.in lists it), excited in the first mode with initstate > 0 -- with every product
 * function |n>.  nvb_create_from_files reads the three blocks from nadvibs.in when basis.in
 * sets shiftref != 0 (Source/top.f90:130-134); nvb_set_displaced_seed supplies them for a
 * handle made with nvb_create (before nvb_seed).  nvb_seed_overlap returns
 * sqrt(sum_n <m|n>^2), the part of the initial state inside the basis (the reference prints
 * it as "Overlap with the initial state"; 1 for the simple seed). */
int nvb_set_displaced_seed(nvb_handle *h, const double *bomega, const double *dvec, const double *tmat);
int nvb_seed_overlap(nvb_handle *h, double *overlap);

/* Record checkpoints of the forward for nvb_lanczos_backward: from the next nvb_seed on,
 * nvb_lanczos saves (v_{c-1}, v_c) at iterations c = 1, 1+k, 1+2k, ... in device memory
 * (2 ceil(niter/k) vectors of the handle's precision).  k = -1 records the whole forward
 * (every v_j, niter + 2 vectors) when that and the sweep's work vectors fit
 * the budget of nvb_set_backward_memory, and nothing otherwise; a sweep with k = -1 then
 * replays nothing (or, without the record, takes the automatic plan of k = 0).  k = 0 stops
 * recording and frees them.  No reference counterpart. */
int nvb_set_checkpoints(nvb_handle *h, int64_t k);

/* Reverse sweep through the first n Lanczos iterations (plain Lanczos, reorthog = 0): given
 * alpha_bar[i-1] = dL/dalpha_i and beta_bar[i-1] = dL/dbeta_i (i = 1..n; beta_bar may be NULL
 * for zeros) of a loss L of T_n, returns grad[ncoef] = dL/dtheta in the layout of
 * nvb_hv_adjoint_coeffs.  Primal vectors are recomputed range by range, last range first, by
 * replaying the recurrence from checkpoint pairs (v_{c-1}, v_c):
 *   k > 0: one level, pairs every k iterations (the forward's, when nvb_set_checkpoints(h, k)
 *          preceded nvb_seed; else one replay from the seed records them), each range of k
 *          iterations replayed into storage (k + 2 vectors of the handle's precision);
 *   k = -1: the forward's full record (nvb_set_checkpoints(h, -1)), nothing replayed; the
 *          automatic plan when the record was not kept;
 *   k = 0: automatic.  The shallowest recursion that fits the budget of
 *          nvb_set_backward_memory (default 85% of free device memory): with depth L, each
 *          level splits its range into B ~ n^(1/(L+1)) sub-ranges whose starting pairs one
 *          replay records, down to ranges of at most B iterations replayed into storage
 *          (2 L B + B + 2 vectors; L + 1 replays of the run).  L = 0 (everything stored,
 *          n + 2 vectors) when it fits.  The forward's pairs, when recorded, are the top level.
 * No plan stores w_j = H v_j: each step rebuilds it from the recurrence,
 * w_j = beta_j v_{j+1} + alpha_j v_j + beta_{j-1} v_{j-1}, from the same stored vectors.
 * Adjoint vectors and dot products are FP64 in every plan; the gradient does not depend on the
 * plan beyond rounding of FP64 sums.  Needs H^T = H (fails with NVB_ERR_STATE under
 * quirk_lower with inter-state constant or even-power couplings).  No reference counterpart
 * (the reference has no derivative code). */
int nvb_lanczos_backward(nvb_handle *h, int64_t n, const double *alpha_bar, const double *beta_bar, int64_t k,
                         double *grad);

/* Device-memory budget (bytes) of the automatic plan of nvb_lanczos_backward (k = 0); 0 = 85%
 * of the free device memory at the call.  The sweep fails with NVB_ERR_NOMEM when even the
 * deepest recursion does not fit.  No reference counterpart. */
int nvb_set_backward_memory(nvb_handle *h, int64_t bytes);

/* The last nvb_lanczos_backward's plan: plan[0] = interval of the top-level pairs (0 = the
 * sweep started from the seed pair), plan[1] = branching B of a level, plan[2] = longest range
 * replayed into storage, plan[3] = H.v applications spent in replays.  No reference
 * counterpart. */
int nvb_backward_plan(nvb_handle *h, int64_t *plan);

/* <sa*a, sb*b> over the handle's total vector length (dimen*nstates) of two device vectors of
 * dtype, summed in FP64 in a fixed order (block partials in the handle's scratch, then one
 * block); the result is returned in host memory (the call synchronises the stream).
 * Replaces GA_DDOT on the Lanczos vectors (e.g. Source/top.f90:829,833). */
int nvb_dot(nvb_handle *h, const void *a, double sa, const void *b, double sb, int64_t dtype, double *result);

/* Allocation-free variant of nvb_dot (no counterpart in the reference).  For callers that
 * cannot allocate device memory -- a host program whose GPU memory is owned by its own pool
 * allocator, or a loop that must not call cudaMalloc/cudaFree because they may synchronise
 * the device.  Computes <sa*a, sb*b> for n elements of dtype and writes it to the device
 * double *result_dev, asynchronously on stream (a cudaStream_t, NULL = default stream).
 * No handle and no allocation: the block partials live in a static device array of this
 * library (4097 doubles, ~32 KiB per GPU that loads it, kept until exit), so n <= 2^32
 * (larger n fails with NVB_ERR_ARG).  All calls share that array and each overwrites the
 * partials it reads; calls that overlap on the GPU race, so order them (one stream or
 * events).  The grid is sized from n (up to eight blocks per multiprocessor).  The first call
 * on each device looks up the array's address (cudaGetSymbolAddress, once per device and
 * again after a reset of the device's context) and should come before any stream capture. */
int nvb_dot_noalloc(const void *a, double sa, const void *b, double sb, int64_t n, int64_t dtype, double *result_dev,
                    void *stream);

/* Measured FMA throughput of the current device's CUDA cores (no reference counterpart): a
 * register-only kernel of independent FMA chains, repeated for about `seconds` of device time
 * and timed with CUDA events; *flops_per_s = 2 x FMAs / s for dtype NVB_DTYPE_F64 or
 * NVB_DTYPE_F32.  The arithmetic ceiling the H.v kernels' flops are compared with. */
int nvb_measure_fma(int64_t dtype, double seconds, double *flops_per_s);

/* Measured rate (bytes/s) at which whole tiles of tile_bytes can be streamed from L2 into
 * shared memory on the current device by the tiled H.v kernels' data path (no reference
 * counterpart): ctas_per_sm CTAs per multiprocessor, each a producer warp issuing TMA bulk
 * copies of pseudo-random tiles of a 64 MB buffer into a ring of `slots` slots and 9 consumer
 * warps that read each slot before releasing it, no arithmetic, about `seconds` of device time
 * timed with CUDA events.  The ceiling of the factorised kernels' neighbour-tile stream. */
int nvb_measure_tile_stream(int64_t tile_bytes, int64_t slots, int64_t ctas_per_sm, double seconds,
                            double *bytes_per_s);

/* The neighbour-tile stream of a factorised H.v (quadratic or cubic kernel) for vectors of
 * dtype: bytes copied from L2 into shared memory per product (every item whose neighbour tile
 * lies inside the basis, once per tile), the tile size, and the ring's slots and CTAs per
 * multiprocessor (after a first product; 1 before).  All zero when the dtype's products use the
 * slab or gather kernel.  No reference counterpart. */
int nvb_hv_tile_stream(nvb_handle *h, int64_t dtype, double *bytes_per_hv, int64_t *tile_bytes, int64_t *slots,
                       int64_t *ctas_per_sm);

/* Per-phase device timing of nvb_lanczos (the reference writes per-phase wall times to
 * output.dat, Source/top.f90:663-667,814-817,834-841): when enabled, CUDA events on the
 * handle's stream bracket the H.v launch and the whole iteration; nvb_get_timing returns
 * the accumulated milliseconds and the number of timed iterations.  Enabling resets them. */
int nvb_set_timing(nvb_handle *h, int64_t enable);
int nvb_get_timing(nvb_handle *h, double *hv_ms, double *iter_ms, int64_t *n);

#ifdef __cplusplus
}
#endif
#endif
