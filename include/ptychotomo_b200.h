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

#ifdef __cplusplus
}
#endif

#endif /* PTYCHOTOMO_B200_H */
