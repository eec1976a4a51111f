"""Drop-in Python classes ``radonusfft`` and ``ptychofft``.

Same constructor arguments and methods as the reference's SWIG classes
(src/cuda/radonusfft.i:15-46, src/cuda/ptychofft.i:14-48): arrays are
passed as device addresses (ints, as CuPy's ``.data.ptr``), or as CUDA
tensors for convenience.  Work is queued on the caller's current torch
stream (or on ``stream=`` when given).  Failures raise
:class:`~ptychotomo_b200._lib.PtychotomoError` instead of silently
producing garbage.
"""
from __future__ import annotations

import ctypes

from ._lib import as_ptr, check, current_stream, lib


class radonusfft:  # noqa: N801 - reference class name
    """USFFT Radon transform; ``radonusfft(Ntheta, Nz, N)`` as radonusfft.cu:5."""

    def __init__(self, Ntheta, Nz, N, m_override: int = 0):
        h = ctypes.c_void_p()
        check(lib().pt_radon_create_ex(int(Ntheta), int(Nz), int(N), int(m_override), ctypes.byref(h)),
              "radonusfft create")
        self._h = h
        self.Ntheta, self.Nz, self.n = int(Ntheta), int(Nz), int(N)
        Np, M, mu = ctypes.c_int(), ctypes.c_int(), ctypes.c_float()
        check(lib().pt_radon_get_params(h, ctypes.byref(Np), ctypes.byref(M), ctypes.byref(mu)))
        self.N, self.M, self.mu = Np.value, M.value, mu.value

    def setobj(self, theta, stream=None):
        """radonusfft::setobj(theta), radonusfft.cu:141."""
        check(lib().pt_radon_setobj(self._h, as_ptr(theta), _s(stream)), "radonusfft.setobj")

    def fwd(self, g, f, stream=None, scale: float | None = None):
        """radonusfft::fwd(g, f), radonusfft.cu:54: g[Ntheta,Nz,n] = R f[Nz,n,n]."""
        if scale is None:
            check(lib().pt_radon_fwd(self._h, as_ptr(g), as_ptr(f), _s(stream)), "radonusfft.fwd")
        else:
            check(lib().pt_radon_fwd_scaled(self._h, as_ptr(g), as_ptr(f), float(scale), _s(stream)),
                  "radonusfft.fwd")

    def adj(self, f, g, stream=None, scale: float | None = None):
        """radonusfft::adj(f, g), radonusfft.cu:94: f[Nz,n,n] = R* g[Ntheta,Nz,n]."""
        if scale is None:
            check(lib().pt_radon_adj(self._h, as_ptr(f), as_ptr(g), _s(stream)), "radonusfft.adj")
        else:
            check(lib().pt_radon_adj_scaled(self._h, as_ptr(f), as_ptr(g), float(scale), _s(stream)),
                  "radonusfft.adj")

    def adj_exact(self, f, g, scale=1.0, stream=None):
        """f = scale * R^T g, the exact adjoint of fwd (zero-padded detector
        lines, margins of the padded slice folded onto the edge pixels); adj
        is the reference's, exact only for border-vanishing g and f."""
        check(lib().pt_radon_adj_exact(self._h, as_ptr(f), as_ptr(g), float(scale), _s(stream)),
              "radonusfft.adj_exact")

    def autotune(self, g, f, trials=3, stream=None):
        """Time the forward with its slice chunks on one stream and pipelined
        on two and on four, each with the gather through L1, from
        shared-memory tiles and from TMA-staged tiles; keep the fastest for
        this operator.  g, f: buffers of fwd's shapes (g is overwritten).
        Returns (streams, gather), gather 0 (L1), 1 (tiles) or 2 (TMA tiles)."""
        out = ctypes.c_int()
        check(lib().pt_radon_autotune(self._h, as_ptr(g), as_ptr(f), int(trials), ctypes.byref(out), _s(stream)),
              "radonusfft.autotune")
        return out.value % 8, out.value // 8

    def set_variant(self, streams=2, gather=0):
        """The forward's variant without timing (results are identical):
        gather 0 (L1), 1 or True (shared-memory tiles), 2 (TMA-staged tiles)."""
        check(lib().pt_radon_set_variant(self._h, int(streams), int(gather)), "radonusfft.set_variant")

    def check_tma_wait(self, stream=None):
        """Run the TMA gather with a barrier that cannot complete and a short
        wait limit; returns the failure code the blocks recorded (1)."""
        code = ctypes.c_int()
        check(lib().pt_radon_check_tma_wait(self._h, ctypes.byref(code), _s(stream)), "radonusfft.check_tma_wait")
        return code.value

    def status(self):
        """(TMA gather failure code since the last call: 0 none, 1 a tile load
        timed out, 2 a misaligned staging buffer; TMA gather available)."""
        a, b = ctypes.c_int(), ctypes.c_int()
        check(lib().pt_radon_status(self._h, ctypes.byref(a), ctypes.byref(b)), "radonusfft.status")
        return a.value, bool(b.value)

    def get_xy(self, x, y, stream=None):
        """Copy the polar coordinate tables (each float32 [Ntheta, N])."""
        check(lib().pt_radon_get_xy(self._h, as_ptr(x), as_ptr(y), _s(stream)), "radonusfft.get_xy")

    def free(self):
        if getattr(self, "_h", None):
            lib().pt_radon_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:  # interpreter shutdown
            pass


class ptychofft:  # noqa: N801 - reference class name
    """Ptychography operator; ``ptychofft(Ntheta, Nz, N, Ntheta0, Nscan, detx, dety, Nprb)``."""

    def __init__(self, Ntheta, Nz, N, Ntheta0, Nscan, detx, dety, Nprb):
        h = ctypes.c_void_p()
        check(lib().pt_ptycho_create(int(Ntheta), int(Nz), int(N), int(Ntheta0), int(Nscan), int(detx),
                                     int(dety), int(Nprb), ctypes.byref(h)), "ptychofft create")
        self._h = h
        self.Ntheta, self.Nz, self.N = int(Ntheta), int(Nz), int(N)
        self.Nscan, self.detx, self.dety, self.Nprb = int(Nscan), int(detx), int(dety), int(Nprb)

    def setobj(self, scan, prb, stream=None):
        """ptychofft::setobj(scan, prb), ptychofft.cu:48."""
        check(lib().pt_ptycho_setobj(self._h, as_ptr(scan), as_ptr(prb), _s(stream)), "ptychofft.setobj")

    def fwd(self, g, f, stream=None, scale: float | None = None):
        """ptychofft::fwd(g, f), ptychofft.cu:58."""
        if scale is None:
            check(lib().pt_ptycho_fwd(self._h, as_ptr(g), as_ptr(f), _s(stream)), "ptychofft.fwd")
        else:
            check(lib().pt_ptycho_fwd_scaled(self._h, as_ptr(g), as_ptr(f), float(scale), _s(stream)),
                  "ptychofft.fwd")

    def adj(self, f, g, stream=None, scale: float | None = None):
        """ptychofft::adj(f, g), ptychofft.cu:78."""
        if scale is None:
            check(lib().pt_ptycho_adj(self._h, as_ptr(f), as_ptr(g), _s(stream)), "ptychofft.adj")
        else:
            check(lib().pt_ptycho_adj_scaled(self._h, as_ptr(f), as_ptr(g), float(scale), _s(stream)),
                  "ptychofft.adj")

    def autotune(self, f, g, trials=3, stream=None):
        """Time the adjoint for each split of an angle's scans over blocks and
        keep the fastest.  f, g: buffers of adj's shapes (f is overwritten).
        Returns the chosen number of parts."""
        out = ctypes.c_int()
        check(lib().pt_ptycho_autotune(self._h, as_ptr(f), as_ptr(g), int(trials), ctypes.byref(out), _s(stream)),
              "ptychofft.autotune")
        return out.value

    @property
    def parts(self):
        out = ctypes.c_int()
        check(lib().pt_ptycho_get_parts(self._h, ctypes.byref(out)), "ptychofft.parts")
        return out.value

    @parts.setter
    def parts(self, value):
        check(lib().pt_ptycho_set_parts(self._h, int(value)), "ptychofft.parts")

    # ---- sub-pixel scan model (no counterpart in the reference) -------------
    def set_subpixel(self, quant, stream=None):
        """quant > 0: frames F(P(r - d) psi(c + r)), c = round(scan), d the
        offset quantised to 1/quant pixel, P(r - d) the band-limited
        interpolation of the probe, no per-scan phase; 0: the reference's
        rounded positions with its constant phase.  Call after setobj (later
        setobj calls rebuild the shifted probes)."""
        check(lib().pt_ptycho_set_subpixel(self._h, int(quant), _s(stream)), "ptychofft.set_subpixel")

    @property
    def subpixel(self):
        """(quant, number of shifted probe tables); quant 0: off."""
        q, k = ctypes.c_int(), ctypes.c_int()
        check(lib().pt_ptycho_get_subpixel(self._h, ctypes.byref(q), ctypes.byref(k)), "ptychofft.subpixel")
        return q.value, k.value

    def adj_resid(self, f, fpsi, data, dscale, model, scale=1.0, stream=None):
        """Gradient of the data term: f = scale * Q* F* residual(fpsi, dscale * data)."""
        check(lib().pt_ptycho_adj_resid(self._h, as_ptr(f), as_ptr(fpsi), as_ptr(data), float(dscale), int(model),
                                        float(scale), _s(stream)), "ptychofft.adj_resid")

    # ---- probe retrieval (no counterpart in the reference) -----------------
    def adj_probe(self, gprb, g, psi, scale=1.0, stream=None):
        """gprb [Nprb, Nprb] = adjoint of fwd as a map of the probe, for the object psi."""
        check(lib().pt_ptycho_adj_probe(self._h, as_ptr(gprb), as_ptr(g), as_ptr(psi), float(scale), _s(stream)),
              "ptychofft.adj_probe")

    def adj_probe_resid(self, gprb, psi, fpsi, data, dscale, model, scale=1.0, stream=None):
        """Probe gradient of the data term: adj_probe of residual(fpsi, dscale * data)."""
        check(lib().pt_ptycho_adj_probe_resid(self._h, as_ptr(gprb), as_ptr(psi), as_ptr(fpsi), as_ptr(data),
                                              float(dscale), int(model), float(scale), _s(stream)),
              "ptychofft.adj_probe_resid")

    def fwd_probe(self, g, psi, prb, scale=1.0, stream=None):
        """fwd(g, psi) with the probe prb instead of the one given to setobj."""
        check(lib().pt_ptycho_fwd_probe(self._h, as_ptr(g), as_ptr(psi), as_ptr(prb), float(scale), _s(stream)),
              "ptychofft.fwd_probe")

    def free(self):
        if getattr(self, "_h", None):
            lib().pt_ptycho_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def _s(stream):
    if stream is None:
        return current_stream()
    if hasattr(stream, "cuda_stream"):
        return stream.cuda_stream
    return int(stream)
