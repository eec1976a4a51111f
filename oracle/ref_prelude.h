/* Force-included ahead of the reference's src/cuda/radonusfft.cu when the
 * oracle build compiles it (oracle/Makefile).  TEST INFRASTRUCTURE.
 *
 * radonusfft::adj (radonusfft.cu:110) clears the buffer `fde` with
 * (2N+2M)^2*Nz elements although the constructor (radonusfft.cu:16)
 * allocated only (2N)^2*Nz.  To run the unmodified reference without an
 * out-of-bounds device write, every cudaMalloc of that translation unit is
 * over-allocated (3x + 1 MiB, enough for every n >= 8 where
 * (2N+2M)^2 / (2N)^2 <= 2.5).  The algorithm itself is untouched. */
#pragma once
#include <cuda_runtime.h>
static inline cudaError_t oracle_padded_cuda_malloc(void **p, size_t bytes)
{
    return cudaMalloc(p, 3 * bytes + (1u << 20));
}
#define cudaMalloc oracle_padded_cuda_malloc
