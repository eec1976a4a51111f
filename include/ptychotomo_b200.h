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
/* solve_reg, solver.py:257-264: z = soft(J u + mu/tau, thr), isotropic over the 3 components. */
int pt_solve_reg_c64(void *z, const void *u, const void *mu, int nz, int ny, int nx, float s, float inv_tau,
                     float thr, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* PTYCHOTOMO_B200_H */
