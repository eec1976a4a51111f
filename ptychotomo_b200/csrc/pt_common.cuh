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

namespace pt {

// Thread-local last-error text (defined in pt_capi.cu).
void set_error(const char *fmt, ...);
void clear_error();

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
