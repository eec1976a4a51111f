/* extern "C" shim over the reference's C++ operator classes, standing in
 * for the SWIG modules of src/cuda/radonusfft.i and src/cuda/ptychofft.i
 * (SWIG is absent here).  TEST INFRASTRUCTURE: built by oracle/Makefile
 * into oracle/_ref and loaded only by tests and the CPU/reference legs of
 * bench.py.  Pointers travel as size_t exactly as in the SWIG interface. */
#include <cuda_runtime.h>
#include <cstddef>
#if defined(ORACLE_SHIM_RADON)
#include "radonusfft.cuh"
extern "C" {
void *ref_radon_create(size_t ntheta, size_t nz, size_t n) { return new radonusfft(ntheta, nz, n); }
void ref_radon_setobj(void *h, size_t theta) { static_cast<radonusfft *>(h)->setobj(theta); }
void ref_radon_fwd(void *h, size_t g, size_t f) { static_cast<radonusfft *>(h)->fwd(g, f); }
void ref_radon_adj(void *h, size_t f, size_t g) { static_cast<radonusfft *>(h)->adj(f, g); }
void ref_radon_destroy(void *h) { delete static_cast<radonusfft *>(h); }
}
#endif
#if defined(ORACLE_SHIM_PTYCHO)
#include "ptychofft.cuh"
extern "C" {
void *ref_ptycho_create(size_t ntheta, size_t nz, size_t n, size_t ntheta0, size_t nscan,
                        size_t detx, size_t dety, size_t nprb)
{
    return new ptychofft(ntheta, nz, n, ntheta0, nscan, detx, dety, nprb);
}
void ref_ptycho_setobj(void *h, size_t scan, size_t prb) { static_cast<ptychofft *>(h)->setobj(scan, prb); }
void ref_ptycho_fwd(void *h, size_t g, size_t f) { static_cast<ptychofft *>(h)->fwd(g, f); }
void ref_ptycho_adj(void *h, size_t f, size_t g) { static_cast<ptychofft *>(h)->adj(f, g); }
void ref_ptycho_destroy(void *h) { delete static_cast<ptychofft *>(h); }
}
#endif
extern "C" int ref_sync_status(void)
{
    cudaError_t e = cudaDeviceSynchronize();
    if (e == cudaSuccess) e = cudaGetLastError();
    return (int)e;
}
