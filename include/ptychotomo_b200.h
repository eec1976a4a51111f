/*
 * ptychotomo_b200 — C ABI of the B200-native ptycho-tomography operators.
 *
 * The entry points replace the two native classes that the reference exposes
 * to Python through SWIG (nikitinvv/ptychotomo):
 *
 *   class radonusfft   src/cuda/radonusfft.i:15-46, src/include/radonusfft.cuh:3-36
 *   class ptychofft    src/cuda/ptychofft.i:14-48,  src/include/ptychofft.cuh:3-35
 *
 * Conventions (the same as the SWIG layer, where pointers travel as size_t):
 *   - every array argument is a DEVICE pointer; complex arrays are
 *     interleaved complex64 (float2); the caller owns inputs and outputs;
 *   - the handle owns its scratch memory, allocated once at creation;
 *     fwd/adj allocate nothing and do not synchronise the host;
 *   - `stream` is a cudaStream_t (NULL = legacy default stream);
 *   - every function returns PT_OK (0) or a negative PT_ERR_* code, and
 *     pt_last_error() then describes the failure (the reference returns
 *     void and checks nothing).
 * Layouts are the reference's: tomography object f [Nz][n][n], projections
 * g [Ntheta][Nz][n]; ptycho object psi [Ntheta][Nz][n], data
 * g [Ntheta][Nscan][detx][dety], scan [2][Ntheta][Nscan] (x then y),
 * probe [Nprb][Nprb].
 */
#ifndef PTYCHOTOMO_B200_H
#define PTYCHOTOMO_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PT_OK 0
#define PT_ERR_ARG (-1)          /* invalid argument (null pointer, bad size, scan outside object) */
#define PT_ERR_UNSUPPORTED (-2)  /* size outside the compiled FFT sizes */
#define PT_ERR_CUDA (-3)         /* CUDA runtime error (launch, copy) */
#define PT_ERR_ALLOC (-4)        /* device allocation failed at creation */
#define PT_ERR_STATE (-5)        /* operator used before setobj */

typedef struct pt_radon pt_radon;
typedef struct pt_ptycho pt_ptycho;

/* Last error message of the calling thread ("" if none). */
const char *pt_last_error(void);
/* Library version string. */
const char *pt_version(void);

/* ---- USFFT Radon transform (tomography operator) ------------------------ */

/* radonusfft::radonusfft(Ntheta, Nz, N)  — src/cuda/radonusfft.cu:5-39.
 * n is the object width; internal N = 3n/2, oversampled grid 2N, Gaussian
 * kernel half-width M and parameter mu as in radonusfft.cu:7-12. */
int pt_radon_create(size_t ntheta, size_t nz, size_t n, pt_radon **out);
/* Same, with the kernel half-width forced to m_override (0 = reference M).
 * A smaller M is a precision variant, not the reference operator. */
int pt_radon_create_ex(size_t ntheta, size_t nz, size_t n, int m_override, pt_radon **out);
/* radonusfft::~radonusfft — src/cuda/radonusfft.cu:41-52. NULL is accepted. */
int pt_radon_destroy(pt_radon *h);
/* radonusfft::setobj(theta) — src/cuda/radonusfft.cu:141-144.
 * theta: device float[Ntheta].  Also builds the polar coordinate tables
 * (takexy, kernels.cuh:84-95) and the adjoint's tile bins; blocks the host. */
int pt_radon_setobj(pt_radon *h, const float *theta, void *stream);
/* radonusfft::fwd(g, f) — src/cuda/radonusfft.cu:54-92.  g = R f. */
int pt_radon_fwd(pt_radon *h, void *g, const void *f, void *stream);
/* radonusfft::adj(f, g) — src/cuda/radonusfft.cu:94-139.  f = R* g. */
int pt_radon_adj(pt_radon *h, void *f, const void *g, void *stream);
/* fwd/adj with the output multiplied by `scale` inside the last kernel
 * (Solver.fwd_tomo/adj_tomo apply coeftomo this way, solver.py:67-80). */
int pt_radon_fwd_scaled(pt_radon *h, void *g, const void *f, float scale, void *stream);
int pt_radon_adj_scaled(pt_radon *h, void *f, const void *g, float scale, void *stream);
/* The exact adjoint of pt_radon_fwd, f = scale * R^T g (no counterpart in the
 * reference).  The reference's adjoint replicates the edge samples of each
 * detector line and crops the padded slice, so it equals R^T only where g
 * and the result vanish on their borders (radonusfft.cu:94-139,
 * kernels.cuh:189-216); here the lines are zero-padded (the adjoint of the
 * forward's crop) and the padded slice is folded onto its edge pixels (the
 * adjoint of the forward's edge replication).  Used by the preconditioned
 * tomography CG, which needs the true gradient of its quadratic. */
int pt_radon_adj_exact(pt_radon *h, void *f, const void *g, float scale, void *stream);
/* Autotuner (no counterpart in the reference): times the forward with its
 * 8-slice chunks on the caller's stream alone and pipelined on two and on
 * four streams (one chunk's FFTs under another chunk's gather), each with the
 * Gaussian gather reading the grid through L1, from shared-memory tiles
 * (16 x 16 window origins per tile) copied by the threads, and from the same
 * tiles loaded by the Tensor Memory Accelerator (one 3-D box per block,
 * completed on an mbarrier; offered when the tensor maps encode), `trials`
 * runs each after a warm-up, and keeps the fastest for this handle
 * (*out = streams + 8 * gather).  g, f: caller buffers of the forward's
 * shapes (overwritten).  Blocks the host.  Every variant gives
 * bit-identical results.  Fails, and withdraws the TMA variant, if a TMA
 * tile load timed out. */
int pt_radon_autotune(pt_radon *h, void *g, const void *f, int trials, int *out, void *stream);
/* Sets the forward's variant directly: streams 1, 2 or 4, gather 0 (L1),
 * 1 (tiles) or 2 (TMA tiles; PT_ERR_UNSUPPORTED if unavailable). */
int pt_radon_set_variant(pt_radon *h, int streams, int gather);
/* Reads (and clears) the TMA gather's failure code (0 none; 1 a tile load's
 * bounded wait ran out; 2 a misaligned staging buffer: the block then skips
 * its points without issuing or waiting) and whether the TMA gather is
 * available.  Blocks the host. */
int pt_radon_status(pt_radon *h, int *tma_timeouts, int *tma_available);
/* Tests the TMA gather's bounded wait: one launch over the first slice
 * chunk's grid whose blocks wait, with a short spin limit, on an mbarrier
 * that nothing arrives at, so every wait runs out and records the failure
 * instead of hanging; each block then waits for its real tile copy before
 * returning.  *code receives the recorded code (1 expected) and the flag is
 * cleared.  Writes no output.  Blocks the host. */
int pt_radon_check_tma_wait(pt_radon *h, int *code, void *stream);
/* Internal parameters: N, kernel half-width M, mu. */
int pt_radon_get_params(const pt_radon *h, int *N, int *M, float *mu);
/* Copies the polar coordinate tables x, y (device float[Ntheta][N] each). */
int pt_radon_get_xy(const pt_radon *h, float *x, float *y, void *stream);

/* ---- ptychography operator --------------------------------------------- */

/* ptychofft::ptychofft(Ntheta, Nz, N, Ntheta0, Nscan, detx, dety, Nprb)
 * — src/cuda/ptychofft.cu:5-33.  ntheta0 is accepted and unused, as in the
 * reference. */
int pt_ptycho_create(size_t ntheta, size_t nz, size_t n, size_t ntheta0, size_t nscan,
                     size_t detx, size_t dety, size_t nprb, pt_ptycho **out);
/* ptychofft::~ptychofft — src/cuda/ptychofft.cu:35-46. NULL is accepted. */
int pt_ptycho_destroy(pt_ptycho *h);
/* ptychofft::setobj(scan, prb) — src/cuda/ptychofft.cu:48-56.
 * scan: device float[2][Ntheta][Nscan]; prb: device complex64[Nprb][Nprb].
 * Scans with roundf(x)<0 or roundf(y)<0 are skipped (the reference's
 * sentinel, kernels.cuh:256); a patch reaching past the object is rejected
 * with PT_ERR_ARG (the reference reads out of bounds).  Blocks the host. */
int pt_ptycho_setobj(pt_ptycho *h, const float *scan, const void *prb, void *stream);
/* ptychofft::fwd(g, f) — src/cuda/ptychofft.cu:58-76.  g = F Q f. */
int pt_ptycho_fwd(pt_ptycho *h, void *g, const void *f, void *stream);
/* ptychofft::adj(f, g) — src/cuda/ptychofft.cu:78-93.  f = Q* F* g. */
int pt_ptycho_adj(pt_ptycho *h, void *f, const void *g, void *stream);
/* fwd/adj with the output multiplied by `scale` (Solver.fwd_ptycho /
 * adj_ptycho apply coefptycho this way, solver.py:100-125). */
int pt_ptycho_fwd_scaled(pt_ptycho *h, void *g, const void *f, float scale, void *stream);
int pt_ptycho_adj_scaled(pt_ptycho *h, void *f, const void *g, float scale, void *stream);
/* Gradient of the ptycho data term, solver.py:219-224: f = scale * Q* F* r
 * with the residual r = fpsi - D fpsi / (|fpsi|^2 + 1e-32) (model 0, Poisson)
 * or fpsi - sqrt(D) exp(i angle fpsi) (model 1, Gaussian), D = dscale * data,
 * formed while the adjoint loads its frames (no residual array).  fpsi is
 * not modified. */
int pt_ptycho_adj_resid(pt_ptycho *h, void *f, const void *fpsi, const float *data, float dscale, int model,
                        float scale, void *stream);
/* Probe retrieval: the operator as a linear map of the probe.  No counterpart
 * in the reference, which keeps the probe fixed.
 *   pt_ptycho_adj_probe:       gprb[P][P] = scale * c * sum over frames of
 *       conj(psi patch) * (inverse 2-D DFT of conj(phase) * g), the adjoint of
 *       fwd with respect to the probe for the object psi [Ntheta][Nz][N];
 *   pt_ptycho_adj_probe_resid: the same with g = the data-term residual of
 *       fpsi (as pt_ptycho_adj_resid): the data term's probe gradient;
 *   pt_ptycho_fwd_probe:       fwd(g, psi) with the probe prb [P][P] instead
 *       of the one given to setobj (which stays in place).
 * Deterministic (fixed-order sum of per-block partials).  Detectors 16..128;
 * PT_ERR_UNSUPPORTED for 8. */
int pt_ptycho_adj_probe(pt_ptycho *h, void *gprb, const void *g, const void *psi, float scale, void *stream);
int pt_ptycho_adj_probe_resid(pt_ptycho *h, void *gprb, const void *psi, const void *fpsi, const float *data,
                              float dscale, int model, float scale, void *stream);
int pt_ptycho_fwd_probe(pt_ptycho *h, void *g, const void *psi, const void *prb, float scale, void *stream);
/* Autotuner (no counterpart in the reference): the adjoint splits each
 * angle's scans over `parts` blocks (own slabs, then a fixed-order sum);
 * times the adjoint for parts in {1, 2, 3, 4, 6, 8, 12, 16} (<= Nscan),
 * `trials` runs each after a warm-up, and keeps the fastest (default: a
 * wave-count model).  f, g: caller buffers of the adjoint's shapes (f is
 * overwritten).  Allocates the slabs; blocks the host. */
int pt_ptycho_autotune(pt_ptycho *h, void *f, const void *g, int trials, int *parts_out, void *stream);
/* Sets the adjoint's split (1 <= parts <= Nscan; detectors below 16 keep
 * their one split) and allocates its slabs. */
int pt_ptycho_set_parts(pt_ptycho *h, int parts);
/* The adjoint's current split. */
int pt_ptycho_get_parts(const pt_ptycho *h, int *parts);
/* Sub-pixel scan model (no counterpart in the reference, which rounds each
 * scan position to the grid and applies a constant per-scan phase,
 * kernels.cuh:306-336 / ptychofft.cu:58-93).  quant > 0: the frame of scan
 * s is F(P(r - d) psi(c + r)) with c = round(s), d = s - c quantised to
 * multiples of 1/quant pixel, P(r - d) the band-limited (Dirichlet-kernel)
 * interpolation of the probe, and no per-scan phase; fwd, adj and the fused
 * residual adjoints all follow it.  quant = 0 restores the reference model.
 * Builds one shifted probe table per distinct offset pair (at most 2 GiB;
 * rebuilt by every later setobj, which switches the model off if that
 * fails), needs setobj first and a detector of 16 or
 * more; probe retrieval is refused while it is on.  Set-up: allocates,
 * blocks the host. */
int pt_ptycho_set_subpixel(pt_ptycho *h, int quant, void *stream);
/* The sub-pixel model's quantisation (0: off) and its number of tables. */
int pt_ptycho_get_subpixel(const pt_ptycho *h, int *quant, int *ntables);


/* ---- Solver arithmetic (src/ptychotomo/solver.py:48-336) -----------------
 * Building blocks of the drop-in Solver; complex arrays are complex64.
 * Reductions accumulate in FP64 into `out` (device doubles) through a caller
 * workspace of pt_reduce_workspace_bytes() bytes; results are deterministic
 * (fixed grid, fixed summation order). */
size_t pt_reduce_workspace_bytes(void);
/* op 0: ||a||^2; 1: sum conj(a)*b (re, im); 2: ||a||^2, Re<a,b>, ||b||^2;
 * 3: max|a|; 4: sum angle(a) over columns [c0, c1) of rows of length ncol
 * (takexi's background phase, solver.py:151-156); 5: ||a - b||^2;
 * 6: sum_i sqrt(|a_i|^2 + |a_{i+n}|^2 + |a_{i+2n}|^2) (TV term of take_lagr,
 * solver.py:299); 7: max|angle(a)| (phase-wrap check, solver.py:238). */
int pt_reduce_c64(int op, const void *a, const void *b, size_t n, int c0, int c1, int ncol, void *work,
                  void *out, void *stream);
/* Ptycho data-term decrease of the CG line search for J step lengths
 * (solver.py:208-214, :171-177), with D = dscale * data and t(x) =
 * |x|^2 - 2 D log max(|x|, 1e-32) (model 0, Poisson) or (|x| - sqrt D)^2
 * (model 1, Gaussian):  out[j] = sum over frames of t(f) - t(f + gammas[j] d),
 * formed per element without cancellation (log1p of the relative change)
 * and summed in FP64.  gammas: device double[J], J <= 16. */
int pt_ls_frames(const void *f, const void *d, const float *data, float dscale, size_t n, int model,
                 const double *gammas, int J, void *work, void *out, void *stream);
/* pt_ls_frames, and then f <- f + gammas[0] * d in place.  With f = F Q psi
 * and d = F Q dir, f becomes F Q (psi + gammas[0] dir) by linearity: the
 * frames of the next CG iterate when the line search keeps its first step
 * (solver.py:219 recomputes them with fwd_ptycho).  The returned sums are
 * those of the unmodified f. */
int pt_ls_frames_advance(void *f, const void *d, const float *data, float dscale, size_t n, int model,
                         const double *gammas, int J, void *work, void *out, void *stream);
/* pt_ls_frames without allocating anything and without a workspace argument.
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory at call time: a host application whose memory pool owns the device
 * memory, or a latency-bound loop that must not call cudaMalloc (which can
 * synchronise the device) after start-up.  The scratch (148 KiB: 1184
 * blocks x 16 FP64 partials) is a static device array of the library, held
 * on every GPU that loads it until the process exits.  The array's device
 * address belongs to a CUDA context: the first call in each context (the
 * runtime's primary context of a device, a caller's own driver-API context,
 * or the new primary context after cudaDeviceReset) looks it up with
 * cudaGetSymbolAddress and caches it with that context's id; make that first
 * call before any stream capture.  J > 16 is rejected with PT_ERR_ARG.
 * All calls share the scratch: calls that overlap on the GPU (different
 * streams, or concurrent host threads) race and give wrong sums. */
int pt_ls_frames_noalloc(const void *f, const void *d, const float *data, float dscale, size_t n, int model,
                         const double *gammas, int J, void *out, void *stream);
/* Lagrangian data term, solver.py:294-298 (D = dscale * data). */
int pt_lagr_frames(const void *f, const float *data, float dscale, size_t n, int model, void *work, void *out,
                   void *stream);
/* Gradient residual of the data term (solver.py:220-224), D = dscale * data:
 * Poisson f - D f / (|f|^2 + 1e-32); Gaussian f - sqrt(D) exp(i angle f). */
int pt_residual_c64(void *out, const void *f, const float *data, float dscale, size_t n, int model, void *stream);
/* out = scale * |x|^2 (float32), the intensities of fwd_ptycho_batch (solver.py:115). */
int pt_abs2_c64(float *out, const void *x, size_t n, float scale, void *stream);
/* out = sum_{j<k} coef[j] * x[j]  (k <= 4, coef as (re, im) float pairs). */
int pt_lincomb_c64(void *out, size_t n, int k, const void *const *x, const float *coef, void *stream);
/* mode 0: out = a*b; 1: out = conj(a)*(b - c); 2: out = conj(a)*b. */
int pt_cmul_c64(void *out, const void *a, const void *b, const void *c, size_t n, int mode, void *stream);
/* out = exp(i s x) exp(i phi)  (exptomo, solver.py:59-60, and the h update, :322). */
int pt_expmap_c64(void *out, const void *x, size_t n, float s, float phi, void *stream);
/* out = (cre + i cim) * mlog(x)  (mlog/logtomo, solver.py:48-64). */
int pt_logmap_c64(void *out, const void *x, size_t n, float cre, float cim, void *stream);
/* takexi, solver.py:163-166, from t = (psi - lamd/rho) exp(-i pshift):
 * K = i t * inv_tmax, xi0 = K * (-i mlog(t)) * cxi. */
int pt_takexi_c64(void *K, void *xi0, const void *t, size_t n, float inv_tmax, float cxi, void *stream);
/* TV operator J (fwd_reg, solver.py:128-134) and J* (adj_reg, :137-146),
 * u [nz][ny][nx], res/g [3][nz][ny][nx], scaled by s (2/sqrt(3), -2/sqrt(3)). */
int pt_reg_fwd_c64(void *res, const void *u, int nz, int ny, int nx, float s, void *stream);
int pt_reg_adj_c64(void *res, const void *g, int nz, int ny, int nx, float s, void *stream);
/* Zeroes the components of g [3][nz][ny][nx] that no forward difference of J
 * produces (x = nx-1 in component 0, y = ny-1 in 1, z = nz-1 in 2), so that
 * pt_reg_adj_c64 of the result is the exact adjoint J^T (no counterpart in
 * the reference: its adj_reg also reads those entries, solver.py:137-146). */
int pt_reg_mask_c64(void *g, int nz, int ny, int nx, void *stream);
/* solve_reg, solver.py:257-264: z = soft(J u + mu/tau, thr), isotropic over the 3 components. */
int pt_solve_reg_c64(void *z, const void *u, const void *mu, int nz, int ny, int nx, float s, float inv_tau,
                     float thr, void *stream);

/* ---- learned Fourier preconditioner of the tomography CG -----------------
 * No counterpart in the reference: its tomography CG (solver.py:180-203) is
 * unpreconditioned.  A 3 -> 64 -> 64 -> 1 MLP with SiLU activations maps the
 * features of a Fourier frequency to the log of a positive filter value.
 * Parameters: one FP32 vector of pt_mlp_param_count() values, W1 [64][3],
 * b1 [64], W2 [64][64], b2 [64], W3 [64], b3.  bf16 != 0: the kernels round
 * the weights (not the biases) to bfloat16, round-to-nearest-even, before
 * their FP32 arithmetic. */
int pt_mlp_param_count(void);
/* Bytes of the workspace pt_mlp_grad needs. */
size_t pt_mlp_workspace_bytes(void);
/* z[p] = MLP(x[p][0..2]) for p < npts. */
int pt_mlp_forward(const float *params, int bf16, const float *x, float *z, size_t npts, void *stream);
/* The same forward with the 64 x 64 layer on the tensor cores: per tile of
 * 128 points one chain of tcgen05.mma (kind::f16, bf16 A = h1 rounded from
 * FP32, bf16 B = W2, FP32 accumulators in tensor memory), read back with
 * tcgen05.ld; layer 1 and the epilogue in FP32 with bf16 weights.  *err (a
 * device int) is set nonzero if a tile's bounded wait for its MMAs ran out
 * (that tile's z is then not written). */
int pt_mlp_forward_tc(const float *params, const float *x, float *z, size_t npts, int *err, void *stream);
/* Tests that kernel's bounded wait: one tile of 128 points (x: 128 x 3,
 * z: 128) whose threads first wait, with a short spin limit, on an mbarrier
 * that nothing arrives at; the wait runs out, *err is set to 1, the MMAs'
 * own barrier is awaited before the tensor memory is released, and z is not
 * written. */
int pt_mlp_check_tc_wait(const float *params, const float *x, float *z, int *err, void *stream);
/* Least-squares loss inv_wsum * sum_p w[p] (z[p] - y[p])^2 into *loss (device
 * double) and its gradient with respect to the parameters into grad
 * (device float[param_count]).  Deterministic: fixed per-block tiles, fixed
 * block order. */
int pt_mlp_grad(const float *params, int bf16, const float *x, const float *y, const float *w, size_t npts,
                float inv_wsum, float *grad, double *loss, void *work, void *stream);
/* One Adam step (bias-corrected, step >= 1) on the FP32 parameters. */
int pt_mlp_adam(float *params, float *m, float *v, const float *grad, int step, float lr, float beta1, float beta2,
                float eps, void *stream);

/* The preconditioner P = D^-1/2 F2^-1 diag(p) F2 D^-1/2 of the tomography CG
 * on volumes [nz][n][n] (F2: the 2-D DFT of each slice), with D the diagonal
 * of rho kbar R^T R + tau J^T J and, in the interior,
 * p(w) = (rho kbar dI + tau dJI) / (rho kbar a(w) + tau j(w)): a(w) the
 * (learned) symbol of R^T R, j(w) the TV symbol.  n in {16 .. 512}, powers
 * of two.  The handle owns its scratch (two volumes); apply allocates
 * nothing. */
typedef struct pt_precond pt_precond;
int pt_precond_create(size_t nz, size_t n, pt_precond **out);
int pt_precond_destroy(pt_precond *h);
/* Features of every frequency of an n x n slice, x[(ky n + kx)][3] in DFT
 * order: |w| / (n/2); the angular sampling density at the direction of w
 * (measured Fourier lines within +-3 degrees over the count for ntheta
 * uniform angles); the angle to the nearest measured line over pi/2 (the
 * missing-wedge extent).  theta: device float[ntheta]. */
int pt_precond_features(const float *theta, int ntheta, int n, float *x, void *stream);
/* log_a: device float[n][n], the log of the symbol of R^T R in DFT order
 * (the network's output); the handle keeps a = exp(log_a). */
int pt_precond_set_log_symbol(pt_precond *h, const float *log_a, void *stream);
/* Copies the symbol a (device float[n][n]). */
int pt_precond_get_symbol(const pt_precond *h, float *a, void *stream);
/* The diagonal of (scale R)^T (scale R) from the radon operator r (same n):
 * exact for the edge pixels and one interior pixel (every other pixel takes
 * its value).  Runs forwards of unit pixels; allocates; blocks the host. */
int pt_precond_set_diag(pt_precond *h, pt_radon *r, float scale, void *stream);
/* Copies the diagonal (device float[n][n]) and its interior value (host). */
int pt_precond_get_diag(const pt_precond *h, float *dR, float *dI, void *stream);
/* out = P in (out may alias in); rho_kbar = rho * mean |K|^2 > 0, tau >= 0. */
int pt_precond_apply(pt_precond *h, void *out, const void *in, float rho_kbar, float tau, void *stream);
/* num[k] += sum over slices of Re(conj(Z[k]) AZ[k]), den[k] += |Z[k]|^2 with
 * Z = F2 z, AZ = F2 az (device double[n][n] each): the statistics of the
 * per-frequency Rayleigh quotients that train the network. */
int pt_precond_spectrum(pt_precond *h, double *num, double *den, const void *z, const void *az, void *stream);
/* Training targets from the accumulated statistics: y = log(num / den) and
 * w = 1 where num / den > 0 and den > den_max_rel * max(den), else 0 (device
 * float[nn] each).  Reads den back to the host (blocks). */
int pt_precond_targets(const double *num, const double *den, int nn, double den_max_rel, float *y, float *w,
                       void *stream);
/* x *= W: a radial window about each slice's centre, 1 within r0 pixels,
 * falling linearly to 0 at r1 (in place). */
int pt_precond_window(pt_precond *h, void *x, float r0, float r1, void *stream);
/* dst = F2 src (unnormalised forward 2-D DFT of every slice). */
int pt_precond_dft2(pt_precond *h, void *dst, const void *src, void *stream);
/* dst = F2^-1(sqrt(|F2 src|^2 + floor^2) exp(2 pi i u)) with u uniform from
 * a hash of (seed, index): a probe with src's modulus spectrum (floored) and
 * random phases; src = NULL: a white probe (unit modulus everywhere). */
int pt_precond_phase_probe(pt_precond *h, void *dst, const void *src, unsigned seed, float floor, void *stream);

/* ---- device-resident scalars: one ADMM iteration as a CUDA graph ---------
 * No counterpart in the reference, whose Solver (solver.py:171-336) decides
 * every step length, Dai-Yuan beta and penalty on the host.  Scalars live in
 * device doubles; reductions (pt_reduce_c64, pt_ls_frames) write into them,
 * the pt_scalar_* one-thread kernels apply the reference's rules there, and
 * the *_dev kernels read them.  Coefficient arrays are (re, im) pairs. */
/* out = sum_{j<k} coef_j x_j with coef (device double[2k]); does nothing when
 * skip_zero is not NULL and *skip_zero == 0. */
int pt_lincomb_dev_c64(void *out, size_t n, int k, const void *const *x, const double *coef, const double *skip_zero,
                       void *stream);
/* Dai-Yuan beta = g2 / (dg - dg0) (solver.py:194-197; 0 for a zero
 * denominator or first != 0); coef = (-1, 0, beta) for d <- -g + beta d. */
int pt_scalar_dy_beta(const double *g2, const double *dg, const double *dg0, int first, double *coef, void *stream);
/* The tomography line search (solver.py:171-177, minf of :181-184) on the
 * closed form: c1 = rho q1[1] + tau q2[1], c2 = rho q1[2] + tau q2[2]
 * (q = quad3 triples), rt = (rho, tau); gamma (in/out) halves while
 * -(2 gamma c1 + gamma^2 c2) < 0 and gamma > 1e-12; coef = (1, 0, gamma). */
int pt_scalar_tomo_gamma(const double *q1, const double *q2, const double *rt, double *gamma, double *coef,
                         void *stream);
/* The ptycho line search (solver.py:171-177 with minf of :208-214) in passes,
 * as Solver.cg_ptycho takes it: state = (accepted, step, gamma, the step by
 * which the frames are currently advanced).
 * ls_begin clears accepted and keeps gamma0 = gamma; ls_candidates writes
 * gam[j] = gamma 2^-j, j < J; ls_pass takes the first j with !(data[j] + rho
 * (2 g_j q[1] - g_j^2 q[2]) < 0 and g_j > 1e-12) (step 0 for g_j <= 1e-12) or
 * sets gamma <- g_{J-1}/2, and does nothing once a step was accepted; ls_end
 * writes coef = (1, 0, step) (0 if no pass accepted one) and corr = (1, 0,
 * step - gamma0), the correction of frames that the first pass advanced by
 * gamma0 (pt_ls_frames_advance). */
int pt_scalar_ls_begin(double *state, void *stream);
int pt_scalar_ls_candidates(const double *state, int J, double *gam, void *stream);
int pt_scalar_ls_pass(const double *data, const double *gam, int J, const double *quad, const double *rt,
                      double *state, void *stream);
int pt_scalar_ls_end(const double *state, double *coef, double *corr, void *stream);
/* After the first pass: if it accepted no step, coef = (1, 0, -gamma0) undoes
 * its advance of the frames (and the state records it); else coef = (1, 0, 0),
 * for a pass that skips itself (pt_lincomb_dev_c64 with skip_zero = &coef[2]). */
int pt_scalar_ls_unadvance(double *state, double *coef, void *stream);
/* pt_ls_frames that does nothing when skip[0] != 0 (a device-side decision
 * made the pass unnecessary); out is then left as it was. */
int pt_ls_frames_dev(const void *f, const void *d, const float *data, float dscale, size_t n, int model,
                     const double *gammas, int J, void *work, void *out, const double *skip, void *stream);
/* takexi's scalars (solver.py:151-166): pshift = (band1 + band2) / (2 cnt),
 * coef = (e, -e / rho) with e = exp(-i pshift). */
int pt_scalar_takexi(const double *band1, const double *band2, double cnt, const double *rt, double *pshift,
                     double *coef, void *stream);
/* The multiplier updates' coefficients (solver.py:326-327): (1, rho, -rho) and (1, tau, -tau). */
int pt_scalar_multipliers(const double *rt, double *coef_l, double *coef_m, void *stream);
/* The penalty update (solver.py:267-282) of rt = (rho, tau) in place from
 * r1 = ||psi - h||^2, s1 = ||h - h0||^2, r2 = ||phi - e||^2, s2 = ||e - e0||^2. */
int pt_scalar_penalty(const double *r1, const double *s1, const double *r2, const double *s2, double *rt,
                      void *stream);
/* The preconditioned CG's scalars: beta = gz / gz0 (0 on the first
 * iteration or after a restart), coef = (-1, 0, beta); the exact step
 * gamma = -c1 / c2 when it descends (else 0 and a restart), coef = (1, 0,
 * gamma); rk_tau = (rho |K|^2 / count, tau). */
int pt_scalar_pcg_beta(const double *gz, double *gz0, double *restart, int first, double *coef, void *stream);
int pt_scalar_pcg_step(const double *q1, const double *q2, const double *rt, double *restart, double *coef,
                       void *stream);
int pt_scalar_pcg_rk(const double *k2, double count, const double *rt, double *rk_tau, void *stream);
/* coef = (a0 [* s0[0]], 0, a1 [* s1[0]], 0) (a null s multiplies by 1). */
int pt_scalar_coef2(const double *s0, double a0, const double *s1, double a1, double *coef, void *stream);
/* out = (a / x[0], 0). */
int pt_scalar_inv(const double *x, double a, double *out, void *stream);
/* pt_expmap_c64, pt_takexi_c64, pt_solve_reg_c64 and pt_precond_apply with
 * their scalars read from device memory (phi; max|t|; rt = (rho, tau);
 * rk_tau). */
int pt_expmap_dev_c64(void *out, const void *x, size_t n, float s, const double *phi, void *stream);
int pt_takexi_dev_c64(void *K, void *xi0, const void *t, size_t n, const double *tmax, float cxi, void *stream);
int pt_solve_reg_dev_c64(void *z, const void *u, const void *mu, int nz, int ny, int nx, float s, const double *rt,
                         float alpha, void *stream);
int pt_precond_apply_dev(pt_precond *h, void *out, const void *in, const double *rk_tau, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* PTYCHOTOMO_B200_H */
