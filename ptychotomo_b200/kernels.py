"""Thin Python wrappers of the Solver kernels of libptychotomo_b200.so.

Every function queues work on the current torch CUDA stream.  Arrays are
torch CUDA tensors (complex64 unless noted); reductions return Python
numbers accumulated in FP64 on the GPU.
"""
from __future__ import annotations

import ctypes
import math

import torch

from ._lib import check, current_stream, lib


def _p(t: torch.Tensor) -> int:
    if not t.is_cuda or not t.is_contiguous():
        raise ValueError("kernel arrays must be contiguous CUDA tensors")
    return t.data_ptr()


def _c64(t: torch.Tensor, name: str = "array"):
    if t.dtype != torch.complex64:
        raise TypeError(f"{name} must be complex64, got {t.dtype}")
    return _p(t)


class Reducer:
    """FP64 reductions with a persistent device workspace (deterministic)."""

    OPS = {"norm2": 0, "dot": 1, "quad3": 2, "maxabs": 3, "angle_band": 4, "norm2_diff": 5, "tv": 6,
           "maxangle": 7}

    # values per op (many() packs them in this order)
    _NVALS = {"norm2": 1, "dot": 2, "quad3": 3, "maxabs": 1, "norm2_diff": 1, "tv": 1, "maxangle": 1}

    def __init__(self, device):
        nbytes = lib().pt_reduce_workspace_bytes()
        self.work = torch.empty(nbytes // 8, dtype=torch.float64, device=device)
        self.out = torch.empty(16, dtype=torch.float64, device=device)
        self.gam = torch.empty(16, dtype=torch.float64, device=device)
        self.outm = torch.empty(64, dtype=torch.float64, device=device)

    def _run(self, op, a, b=None, n=None, c0=0, c1=0, ncol=1, k=1):
        n = a.numel() if n is None else n
        check(lib().pt_reduce_c64(op, _c64(a), _c64(b) if b is not None else None, n, c0, c1, ncol,
                                  _p(self.work), _p(self.out), current_stream()), "reduce")
        return self.out[:k].tolist()

    def many(self, ops):
        """Several reductions with one read-back: ops = [(name, a[, b]), ...]
        with name in norm2, dot, quad3, norm2_diff; returns their results in
        order, as the single methods return them."""
        off = 0
        base = self.outm.data_ptr()
        for name, *arrs in ops:
            a = arrs[0]
            b = arrs[1] if len(arrs) > 1 else None
            check(lib().pt_reduce_c64(self.OPS[name], _c64(a), _c64(b) if b is not None else None, a.numel(), 0, 0, 1,
                                      _p(self.work), base + 8 * off, current_stream()), "reduce")
            off += self._NVALS[name]
        return self.unpack(ops, self.outm[:off].tolist())

    @classmethod
    def unpack(cls, ops, flat):
        out, off = [], 0
        for name, *_ in ops:
            k = cls._NVALS[name]
            v = flat[off:off + k]
            off += k
            out.append(complex(v[0], v[1]) if name == "dot" else tuple(v) if name == "quad3" else v[0])
        return out

    def norm2(self, a):
        """||a||^2 (cp.linalg.norm(a)**2 in the reference)."""
        return self._run(0, a)[0]

    def dot(self, a, b):
        """sum(conj(a) * b)."""
        re, im = self._run(1, a, b, k=2)
        return complex(re, im)

    def quad3(self, a, b):
        """(||a||^2, Re<a, b>, ||b||^2)."""
        return tuple(self._run(2, a, b, k=3))

    def maxabs(self, a):
        return self._run(3, a)[0]

    def angle_band_sum(self, a, c0, c1):
        """Sum of angle(a) over columns [c0, c1) of the last axis."""
        return self._run(4, a, c0=c0, c1=c1, ncol=a.shape[-1])[0]

    def norm2_diff(self, a, b):
        """||a - b||^2."""
        return self._run(5, a, b)[0]

    def tv(self, phi):
        """sum over voxels of sqrt(sum_c |phi_c|^2) for phi [3, ...]."""
        return self._run(6, phi, n=phi.numel() // 3)[0]

    def maxangle(self, a):
        return self._run(7, a)[0]

    def ls_frames(self, f, d, data, dscale, model, gammas, advance=False):
        """Ptycho data term for each step length in `gammas` (<= 16).

        ``advance``: afterwards f <- f + gammas[0] d in place (pt_ls_frames_advance).
        """
        J = len(gammas)
        self.gam[:J].copy_(torch.tensor(gammas, dtype=torch.float64), non_blocking=False)
        fn = lib().pt_ls_frames_advance if advance else lib().pt_ls_frames
        check(fn(_c64(f), _c64(d) if d is not None else None, _p(data), float(dscale),
                 f.numel(), model, _p(self.gam), J, _p(self.work), _p(self.out),
                 current_stream()), "ls_frames")
        return self.out[:J].tolist()

    def lagr_frames(self, f, data, dscale, model):
        check(lib().pt_lagr_frames(_c64(f), _p(data), float(dscale), f.numel(), model, _p(self.work),
                                   _p(self.out), current_stream()), "lagr_frames")
        return self.out[0].item()


def lincomb(out, terms):
    """out = sum c_i x_i for terms [(c_i, x_i)], up to 4 (out may alias an x_i)."""
    k = len(terms)
    xs = (ctypes.c_void_p * 4)(*[_c64(x) for _, x in terms] + [None] * (4 - k))
    cs = (ctypes.c_float * 8)()
    for j, (c, _) in enumerate(terms):
        c = complex(c)
        cs[2 * j], cs[2 * j + 1] = c.real, c.imag
    check(lib().pt_lincomb_c64(_c64(out), out.numel(), k, xs, cs, current_stream()), "lincomb")
    return out


def cmul(out, a, b, c=None, mode=0):
    """mode 0: a*b; 1: conj(a)*(b - c); 2: conj(a)*b."""
    check(lib().pt_cmul_c64(_c64(out), _c64(a), _c64(b), _c64(c) if c is not None else None, out.numel(), mode,
                            current_stream()), "cmul")
    return out


def expmap(out, x, s, phi=0.0):
    """out = exp(i s x) * exp(i phi)."""
    check(lib().pt_expmap_c64(_c64(out), _c64(x), out.numel(), float(s), float(phi), current_stream()), "expmap")
    return out


def logmap(out, x, c=1.0):
    """out = c * mlog(x)."""
    c = complex(c)
    check(lib().pt_logmap_c64(_c64(out), _c64(x), out.numel(), c.real, c.imag, current_stream()), "logmap")
    return out


def takexi(K, xi0, t, tmax, cxi):
    check(lib().pt_takexi_c64(_c64(K), _c64(xi0), _c64(t), t.numel(), 1.0 / tmax, float(cxi), current_stream()),
          "takexi")


def reg_fwd(res, u, s):
    nz, ny, nx = u.shape
    check(lib().pt_reg_fwd_c64(_c64(res), _c64(u), nz, ny, nx, float(s), current_stream()), "reg_fwd")
    return res


def reg_adj(res, g, s):
    nz, ny, nx = res.shape
    check(lib().pt_reg_adj_c64(_c64(res), _c64(g), nz, ny, nx, float(s), current_stream()), "reg_adj")
    return res


def reg_mask(g):
    """Zero the entries of g [3, nz, ny, nx] outside the range of J (in place)."""
    _, nz, ny, nx = g.shape
    check(lib().pt_reg_mask_c64(_c64(g), nz, ny, nx, current_stream()), "reg_mask")
    return g


def solve_reg(z, u, mu, s, inv_tau, thr):
    nz, ny, nx = u.shape
    check(lib().pt_solve_reg_c64(_c64(z), _c64(u), _c64(mu), nz, ny, nx, float(s), float(inv_tau), float(thr),
                                 current_stream()), "solve_reg")
    return z


def residual(out, f, data, dscale, model):
    check(lib().pt_residual_c64(_c64(out), _c64(f), _p(data), float(dscale), f.numel(), model, current_stream()),
          "residual")
    return out


def abs2(out, x, scale):
    if out.dtype != torch.float32:
        raise TypeError("abs2 output must be float32")
    check(lib().pt_abs2_c64(_p(out), _c64(x), x.numel(), float(scale), current_stream()), "abs2")
    return out


SQRT3_INV2 = float(2 / math.sqrt(3))
