// Shared helpers: complex arithmetic on float2, error reporting, launch checks.
#pragma once

#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>

#include "../../include/ptychotomo_b200.h"

// ---- complex64 arithmetic ---------------------------------------------------
__host__ __device__ __forceinline__ float2 operator+(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ float2 operator-(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ float2 operator*(float s, float2 a) { return make_float2(s * a.x, s * a.y); }
__host__ __device__ __forceinline__ float2 operator*(float2 a, float s) { return make_float2(s * a.x, s * a.y); }
__host__ __device__ __forceinline__ float2 cmul(float2 a, float2 b)
{
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// conj(a) * b
__host__ __device__ __forceinline__ float2 cmulc(float2 a, float2 b)
{
    return make_float2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
__host__ __device__ __forceinline__ float2 czero() { return make_float2(0.f, 0.f); }

// ---- data-term residual of the ptycho gradient (solver.py:220-224) ----------
// D = measured intensity (already scaled).  Poisson: x - D x / (|x|^2 + 1e-32),
// the quotient as D times the correctly rounded reciprocal of the divisor (a
// normal number >= 1e-32), so zero counts, which are common, take the same
// path as the rest.  Gaussian: x - sqrt(D) exp(i angle(x)), formed as
// x (1 - sqrt(D) / |x|) with rsqrtf for 1/|x| (within 2 ulp; the reference's
// angle/exp pair is itself a few ulp from exact); for |x|^2 < 1e-30 (and
// x = 0, where angle is 0) through atan2 as written.
__device__ __forceinline__ float2 pt_residual_poisson(float2 x, float D)
{
    const float q = D * __frcp_rn(x.x * x.x + x.y * x.y + 1e-32f);
    return make_float2(x.x - q * x.x, x.y - q * x.y);
}
// the rare |x|^2 < 1e-30 case, kept out of line so that unrolled callers stay small
static __device__ __noinline__ float2 pt_residual_gaussian_tiny(float2 x, float sq)
{
    float sn, cs;
    sincosf(atan2f(x.y, x.x), &sn, &cs);
    return make_float2(x.x - sq * cs, x.y - sq * sn);
}
__device__ __forceinline__ float2 pt_residual_gaussian(float2 x, float D)
{
    const float sq = sqrtf(D);
    const float a2 = x.x * x.x + x.y * x.y;
    if (a2 >= 1e-30f) {
        const float r = sq * rsqrtf(a2);
        return make_float2(x.x - r * x.x, x.y - r * x.y);
    }
    return pt_residual_gaussian_tiny(x, sq);
}

namespace pt {

// Thread-local last-error text (defined in pt_capi.cu).
void set_error(const char *fmt, ...);
void clear_error();
// Slice count and angle count of a radon operator (pt_radon.cu).
int radon_dims(const pt_radon *h, int *nz, int *ntheta);

}  // namespace pt

#define PT_CHECK_ARG(cond, ...)            \
    do {                                   \
        if (!(cond)) {                     \
            pt::set_error(__VA_ARGS__);    \
            return PT_ERR_ARG;             \
        }                                  \
    } while (0)

#define PT_CUDA(call)                                                                       \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess) {                                                            \
            pt::set_error("%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, \
                          __LINE__);                                                        \
            return PT_ERR_CUDA;                                                             \
        }                                                                                   \
    } while (0)

// After a kernel launch: report configuration errors without synchronising.
#define PT_LAUNCHED(name)                                                                      \
    do {                                                                                       \
        cudaError_t e_ = cudaGetLastError();                                                   \
        if (e_ != cudaSuccess) {                                                               \
            pt::set_error("launch of %s failed: %s (%s:%d)", name, cudaGetErrorString(e_),     \
                          __FILE__, __LINE__);                                                 \
            return PT_ERR_CUDA;                                                                \
        }                                                                                      \
    } while (0)
