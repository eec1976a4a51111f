"""ctypes binding of ``libptychotomo_b200.so`` (declared in include/ptychotomo_b200.h).

The library is the only compute path: if it is missing or fails to load,
every operator raises instead of falling back to anything else.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

LIB_PATH = Path(__file__).resolve().with_name("libptychotomo_b200.so")

PT_OK = 0
PT_ERR_ARG = -1
PT_ERR_UNSUPPORTED = -2
PT_ERR_CUDA = -3
PT_ERR_ALLOC = -4
PT_ERR_STATE = -5

_CODES = {PT_ERR_ARG: "invalid argument", PT_ERR_UNSUPPORTED: "unsupported size",
          PT_ERR_CUDA: "CUDA error", PT_ERR_ALLOC: "allocation failed", PT_ERR_STATE: "bad state"}


class PtychotomoError(RuntimeError):
    """A C-ABI call returned a negative status; ``code`` holds it."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"{msg} [{_CODES.get(code, 'error')} {code}]")
        self.code = code


class PtychotomoArgError(PtychotomoError, ValueError):
    """Status PT_ERR_ARG: the arguments are invalid."""


_vp = ctypes.c_void_p
_sz = ctypes.c_size_t
_int = ctypes.c_int
_f = ctypes.c_float

# name -> (restype, argtypes); every entry point declared in the public header
SIGNATURES = {
    "pt_last_error": (ctypes.c_char_p, []),
    "pt_version": (ctypes.c_char_p, []),
    "pt_radon_create": (_int, [_sz, _sz, _sz, ctypes.POINTER(_vp)]),
    "pt_radon_create_ex": (_int, [_sz, _sz, _sz, _int, ctypes.POINTER(_vp)]),
    "pt_radon_destroy": (_int, [_vp]),
    "pt_radon_setobj": (_int, [_vp, _vp, _vp]),
    "pt_radon_fwd": (_int, [_vp, _vp, _vp, _vp]),
    "pt_radon_adj": (_int, [_vp, _vp, _vp, _vp]),
    "pt_radon_fwd_scaled": (_int, [_vp, _vp, _vp, _f, _vp]),
    "pt_radon_adj_scaled": (_int, [_vp, _vp, _vp, _f, _vp]),
    "pt_radon_adj_exact": (_int, [_vp, _vp, _vp, _f, _vp]),
    "pt_radon_get_params": (_int, [_vp, ctypes.POINTER(_int), ctypes.POINTER(_int), ctypes.POINTER(_f)]),
    "pt_radon_get_xy": (_int, [_vp, _vp, _vp, _vp]),
    "pt_ptycho_create": (_int, [_sz, _sz, _sz, _sz, _sz, _sz, _sz, _sz, ctypes.POINTER(_vp)]),
    "pt_ptycho_destroy": (_int, [_vp]),
    "pt_ptycho_setobj": (_int, [_vp, _vp, _vp, _vp]),
    "pt_ptycho_fwd": (_int, [_vp, _vp, _vp, _vp]),
    "pt_ptycho_adj": (_int, [_vp, _vp, _vp, _vp]),
    "pt_ptycho_fwd_scaled": (_int, [_vp, _vp, _vp, _f, _vp]),
    "pt_ptycho_adj_scaled": (_int, [_vp, _vp, _vp, _f, _vp]),
    "pt_ptycho_adj_resid": (_int, [_vp, _vp, _vp, _vp, _f, _int, _f, _vp]),
    "pt_ptycho_adj_probe": (_int, [_vp, _vp, _vp, _vp, _f, _vp]),
    "pt_ptycho_adj_probe_resid": (_int, [_vp, _vp, _vp, _vp, _vp, _f, _int, _f, _vp]),
    "pt_ptycho_fwd_probe": (_int, [_vp, _vp, _vp, _vp, _f, _vp]),
    "pt_ptycho_autotune": (_int, [_vp, _vp, _vp, _int, ctypes.POINTER(_int), _vp]),
    "pt_ptycho_get_parts": (_int, [_vp, ctypes.POINTER(_int)]),
    "pt_ptycho_set_parts": (_int, [_vp, _int]),
    "pt_ptycho_set_subpixel": (_int, [_vp, _int, _vp]),
    "pt_ptycho_get_subpixel": (_int, [_vp, ctypes.POINTER(_int), ctypes.POINTER(_int)]),
    "pt_radon_autotune": (_int, [_vp, _vp, _vp, _int, ctypes.POINTER(_int), _vp]),
    "pt_radon_set_variant": (_int, [_vp, _int, _int]),
    "pt_radon_status": (_int, [_vp, ctypes.POINTER(_int), ctypes.POINTER(_int)]),
    "pt_radon_check_tma_wait": (_int, [_vp, ctypes.POINTER(_int), _vp]),
    "pt_reduce_workspace_bytes": (_sz, []),
    "pt_reduce_c64": (_int, [_int, _vp, _vp, _sz, _int, _int, _int, _vp, _vp, _vp]),
    "pt_ls_frames": (_int, [_vp, _vp, _vp, _f, _sz, _int, _vp, _int, _vp, _vp, _vp]),
    "pt_ls_frames_advance": (_int, [_vp, _vp, _vp, _f, _sz, _int, _vp, _int, _vp, _vp, _vp]),
    "pt_lagr_frames": (_int, [_vp, _vp, _f, _sz, _int, _vp, _vp, _vp]),
    "pt_ls_frames_noalloc": (_int, [_vp, _vp, _vp, _f, _sz, _int, _vp, _int, _vp, _vp]),
    "pt_residual_c64": (_int, [_vp, _vp, _vp, _f, _sz, _int, _vp]),
    "pt_abs2_c64": (_int, [_vp, _vp, _sz, _f, _vp]),
    "pt_lincomb_c64": (_int, [_vp, _sz, _int, ctypes.POINTER(_vp), ctypes.POINTER(_f), _vp]),
    "pt_cmul_c64": (_int, [_vp, _vp, _vp, _vp, _sz, _int, _vp]),
    "pt_expmap_c64": (_int, [_vp, _vp, _sz, _f, _f, _vp]),
    "pt_logmap_c64": (_int, [_vp, _vp, _sz, _f, _f, _vp]),
    "pt_takexi_c64": (_int, [_vp, _vp, _vp, _sz, _f, _f, _vp]),
    "pt_reg_fwd_c64": (_int, [_vp, _vp, _int, _int, _int, _f, _vp]),
    "pt_reg_adj_c64": (_int, [_vp, _vp, _int, _int, _int, _f, _vp]),
    "pt_reg_mask_c64": (_int, [_vp, _int, _int, _int, _vp]),
    "pt_solve_reg_c64": (_int, [_vp, _vp, _vp, _int, _int, _int, _f, _f, _f, _vp]),
    "pt_precond_create": (_int, [_sz, _sz, ctypes.POINTER(_vp)]),
    "pt_precond_destroy": (_int, [_vp]),
    "pt_precond_features": (_int, [_vp, _int, _int, _vp, _vp]),
    "pt_precond_set_log_symbol": (_int, [_vp, _vp, _vp]),
    "pt_precond_get_symbol": (_int, [_vp, _vp, _vp]),
    "pt_precond_set_diag": (_int, [_vp, _vp, _f, _vp]),
    "pt_precond_get_diag": (_int, [_vp, _vp, ctypes.POINTER(_f), _vp]),
    "pt_precond_apply": (_int, [_vp, _vp, _vp, _f, _f, _vp]),
    "pt_precond_spectrum": (_int, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "pt_precond_dft2": (_int, [_vp, _vp, _vp, _vp]),
    "pt_precond_targets": (_int, [_vp, _vp, _int, ctypes.c_double, _vp, _vp, _vp]),
    "pt_precond_window": (_int, [_vp, _vp, _f, _f, _vp]),
    "pt_precond_phase_probe": (_int, [_vp, _vp, _vp, ctypes.c_uint, _f, _vp]),
    "pt_precond_apply_dev": (_int, [_vp, _vp, _vp, _vp, _vp]),
    "pt_lincomb_dev_c64": (_int, [_vp, _sz, _int, ctypes.POINTER(_vp), _vp, _vp, _vp]),
    "pt_scalar_dy_beta": (_int, [_vp, _vp, _vp, _int, _vp, _vp]),
    "pt_scalar_tomo_gamma": (_int, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "pt_scalar_ls_begin": (_int, [_vp, _vp]),
    "pt_scalar_ls_candidates": (_int, [_vp, _int, _vp, _vp]),
    "pt_scalar_ls_pass": (_int, [_vp, _vp, _int, _vp, _vp, _vp, _vp]),
    "pt_scalar_ls_end": (_int, [_vp, _vp, _vp, _vp]),
    "pt_scalar_ls_unadvance": (_int, [_vp, _vp, _vp]),
    "pt_ls_frames_dev": (_int, [_vp, _vp, _vp, _f, _sz, _int, _vp, _int, _vp, _vp, _vp, _vp]),
    "pt_scalar_takexi": (_int, [_vp, _vp, ctypes.c_double, _vp, _vp, _vp, _vp]),
    "pt_scalar_multipliers": (_int, [_vp, _vp, _vp, _vp]),
    "pt_scalar_penalty": (_int, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "pt_scalar_pcg_beta": (_int, [_vp, _vp, _vp, _int, _vp, _vp]),
    "pt_scalar_pcg_step": (_int, [_vp, _vp, _vp, _vp, _vp, _vp]),
    "pt_scalar_pcg_rk": (_int, [_vp, ctypes.c_double, _vp, _vp, _vp]),
    "pt_scalar_coef2": (_int, [_vp, ctypes.c_double, _vp, ctypes.c_double, _vp, _vp]),
    "pt_scalar_inv": (_int, [_vp, ctypes.c_double, _vp, _vp]),
    "pt_expmap_dev_c64": (_int, [_vp, _vp, _sz, _f, _vp, _vp]),
    "pt_takexi_dev_c64": (_int, [_vp, _vp, _vp, _sz, _vp, _f, _vp]),
    "pt_solve_reg_dev_c64": (_int, [_vp, _vp, _vp, _int, _int, _int, _f, _vp, _f, _vp]),
    "pt_mlp_param_count": (_int, []),
    "pt_mlp_workspace_bytes": (_sz, []),
    "pt_mlp_forward": (_int, [_vp, _int, _vp, _vp, _sz, _vp]),
    "pt_mlp_forward_tc": (_int, [_vp, _vp, _vp, _sz, _vp, _vp]),
    "pt_mlp_check_tc_wait": (_int, [_vp, _vp, _vp, _vp, _vp]),
    "pt_mlp_grad": (_int, [_vp, _int, _vp, _vp, _vp, _sz, _f, _vp, _vp, _vp, _vp]),
    "pt_mlp_adam": (_int, [_vp, _vp, _vp, _vp, _int, _f, _f, _f, _f, _vp]),
}

_lib = None


def lib() -> ctypes.CDLL:
    """Load the CUDA library once; raise if it has not been built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise ImportError(f"{LIB_PATH.name} is not built; run `python -m ptychotomo_b200.build`")
        handle = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


def last_error() -> str:
    return lib().pt_last_error().decode(errors="replace")


def check(rc: int, what: str = "") -> None:
    if rc != PT_OK:
        msg = last_error() or what
        cls = PtychotomoArgError if rc == PT_ERR_ARG else PtychotomoError
        raise cls(rc, msg)


def current_stream() -> int:
    """The calling thread's current torch CUDA stream handle (0 without torch)."""
    try:
        import torch
    except ImportError:  # pragma: no cover - torch is a dependency of the solver only
        return 0
    if not torch.cuda.is_available():
        return 0
    return torch.cuda.current_stream().cuda_stream


def as_ptr(x) -> int:
    """Device address of an int (as in the reference's SWIG calls) or a tensor."""
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        if not x.is_cuda:
            raise ValueError("operator arrays must be CUDA tensors")
        if not x.is_contiguous():
            raise ValueError("operator arrays must be contiguous")
        return x.data_ptr()
    raise TypeError(f"expected a device pointer (int) or a CUDA tensor, got {type(x).__name__}")
