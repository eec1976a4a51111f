"""ctypes access to the reference's own CUDA operators (oracle/_ref).

TEST INFRASTRUCTURE.  ``oracle/Makefile`` compiles the reference's
src/cuda/radonusfft.cu and src/cuda/ptychofft.cu unmodified (plus an
extern "C" shim standing in for the SWIG modules) into
``oracle/_ref/libref_radon.so`` and ``oracle/_ref/libref_ptycho.so``.
Pointers are passed as size_t, like the reference's SWIG interface.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

REF_DIR = Path(__file__).resolve().parents[1] / "oracle" / "_ref"
_sz = ctypes.c_size_t
_vp = ctypes.c_void_p


def available() -> bool:
    return (REF_DIR / "libref_radon.so").exists() and (REF_DIR / "libref_ptycho.so").exists()


_libs = {}


def _load(name):
    if name not in _libs:
        lib = ctypes.CDLL(str(REF_DIR / name))
        lib.ref_sync_status.restype = ctypes.c_int
        if "radon" in name:
            lib.ref_radon_create.restype = _vp
            lib.ref_radon_create.argtypes = [_sz, _sz, _sz]
            for f in ("setobj",):
                getattr(lib, "ref_radon_" + f).argtypes = [_vp, _sz]
            lib.ref_radon_fwd.argtypes = [_vp, _sz, _sz]
            lib.ref_radon_adj.argtypes = [_vp, _sz, _sz]
            lib.ref_radon_destroy.argtypes = [_vp]
        else:
            lib.ref_ptycho_create.restype = _vp
            lib.ref_ptycho_create.argtypes = [_sz] * 8
            lib.ref_ptycho_setobj.argtypes = [_vp, _sz, _sz]
            lib.ref_ptycho_fwd.argtypes = [_vp, _sz, _sz]
            lib.ref_ptycho_adj.argtypes = [_vp, _sz, _sz]
            lib.ref_ptycho_destroy.argtypes = [_vp]
        _libs[name] = lib
    return _libs[name]


def _sync(lib):
    rc = lib.ref_sync_status()
    if rc != 0:
        raise RuntimeError(f"reference CUDA operator failed with cudaError {rc}")


class RefRadon:
    """The reference radonusfft(Ntheta, Nz, N)."""

    def __init__(self, ntheta, nz, n):
        self.lib = _load("libref_radon.so")
        self.h = self.lib.ref_radon_create(ntheta, nz, n)
        _sync(self.lib)

    def setobj(self, theta_ptr):
        self.lib.ref_radon_setobj(self.h, theta_ptr)
        _sync(self.lib)

    def fwd(self, g_ptr, f_ptr, sync=True):
        self.lib.ref_radon_fwd(self.h, g_ptr, f_ptr)
        if sync:
            _sync(self.lib)

    def adj(self, f_ptr, g_ptr, sync=True):
        self.lib.ref_radon_adj(self.h, f_ptr, g_ptr)
        if sync:
            _sync(self.lib)

    def free(self):
        if self.h:
            self.lib.ref_radon_destroy(self.h)
            self.h = None


class RefPtycho:
    """The reference ptychofft(Ntheta, Nz, N, Ntheta0, Nscan, detx, dety, Nprb)."""

    def __init__(self, ntheta, nz, n, nscan, det, nprb):
        self.lib = _load("libref_ptycho.so")
        self.h = self.lib.ref_ptycho_create(ntheta, nz, n, ntheta, nscan, det, det, nprb)
        _sync(self.lib)

    def setobj(self, scan_ptr, prb_ptr):
        self.lib.ref_ptycho_setobj(self.h, scan_ptr, prb_ptr)
        _sync(self.lib)

    def fwd(self, g_ptr, f_ptr, sync=True):
        self.lib.ref_ptycho_fwd(self.h, g_ptr, f_ptr)
        if sync:
            _sync(self.lib)

    def adj(self, f_ptr, g_ptr, sync=True):
        self.lib.ref_ptycho_adj(self.h, f_ptr, g_ptr)
        if sync:
            _sync(self.lib)

    def free(self):
        if self.h:
            self.lib.ref_ptycho_destroy(self.h)
            self.h = None
