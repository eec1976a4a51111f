"""NumPy restatement of the reference ptychography operator.

TEST INFRASTRUCTURE (the oracle).  Follows:

* constructor        src/cuda/ptychofft.cu:5-33
* setobj             src/cuda/ptychofft.cu:48-56 + takeshifts (kernels.cuh:306-317)
* fwd                src/cuda/ptychofft.cu:58-76 + mul (kernels.cuh:243-265), shifts (:319-336)
* adj                src/cuda/ptychofft.cu:78-93 + shiftsa (kernels.cuh:338-355), mula (:267-288)

* sub-pixel model   no counterpart in the reference (set_subpixel): the probe
                     evaluated at the scan's offset by the Fourier shift
                     theorem (numpy FFTs), no per-scan phase

Layouts: object psi is [Ntheta, Nz, N]; data g is [Ntheta, Nscan, detx, dety];
scan is [2, Ntheta, Nscan] float32 (x then y); prb is [Nprb, Nprb].
Frame element (ix, iy) multiplies prb[ix, iy] with psi[sty+iy, stx+ix]
(kernels.cuh:257-263): the detector row runs along the object column.
"""
from __future__ import annotations

import numpy as np
import scipy.fft as sfft

from ._threads import WORKERS

PI_REF = 3.1415926535  # kernels.cuh:1


def roundf(v):
    """C roundf: half away from zero (evaluated in float64, exact for float32)."""
    v = np.asarray(v, np.float64)
    return np.sign(v) * np.floor(np.abs(v) + 0.5)


def scan_corners(scan):
    """Integer patch corners (stx, sty) = roundf(scan), kernels.cuh:255-256."""
    scan = np.asarray(scan, np.float32)
    return roundf(scan[0]).astype(np.int64), roundf(scan[1]).astype(np.int64)


def scan_phases(scan):
    """takeshifts, kernels.cuh:306-317: exp(2*pi*i*(scan - roundf(scan)))."""
    scan = np.asarray(scan, np.float32)
    out = []
    for v in (scan[0], scan[1]):
        frac = (v - roundf(v).astype(np.float32)).astype(np.float32)
        arg = np.float32(2 * PI_REF * frac.astype(np.float64)).astype(np.float64)
        out.append(np.cos(arg) + 1j * np.sin(arg))
    return out[0], out[1]


def shift_probe(prb, dx, dy):
    """The probe evaluated at (ix - dx, iy - dy) by band-limited
    (trigonometric) interpolation of its samples: the DFT of prb times
    exp(-2 pi i k d / P) per axis, with the Nyquist bin of an even size
    multiplied by cos(pi d) (the real, symmetric choice).  prb is [ix, iy]."""
    prb = np.asarray(prb, np.complex128)
    out = np.fft.fft2(prb)
    for ax, d in ((0, dx), (1, dy)):
        P = prb.shape[ax]
        k = np.fft.fftfreq(P) * P
        ramp = np.exp(-2j * np.pi * k * d / P)
        if P % 2 == 0:
            ramp[P // 2] = np.cos(np.pi * d)
        out = out * (ramp[:, None] if ax == 0 else ramp[None, :])
    return np.fft.ifft2(out)


class PtychoFFT:
    """Oracle twin of class ptychofft (ptychofft.cuh, ptychofft.cu)."""

    def __init__(self, ntheta, nz, n, ntheta0, nscan, detx, dety, nprb):
        self.ntheta, self.nz, self.n = ntheta, nz, n
        self.nscan, self.detx, self.dety, self.nprb = nscan, detx, dety, nprb
        self.c = 1.0 / np.sqrt(np.float32(detx * dety))   # kernels.cuh:260
        self.quant = 0

    def set_subpixel(self, quant):
        """Sub-pixel scan model: offsets d = scan - roundf(scan) (float32, as
        the device computes them) rounded half-to-even to multiples of
        1/quant; each frame's probe is shift_probe(prb, dx, dy) and the
        per-scan phase is dropped.  quant 0: the reference model."""
        self.quant = int(quant)

    def _offsets(self):
        out = []
        for v, c in ((self.scan[0], self.stx), (self.scan[1], self.sty)):
            frac = (v - c.astype(np.float32)).astype(np.float32).astype(np.float64)
            out.append(np.rint(frac * self.quant) / self.quant)
        return out

    def _frame_probes(self):
        """{(t, s): probe} under the sub-pixel model, one FFT shift per distinct offset."""
        dx, dy = self._offsets()
        cache, out = {}, {}
        for t in range(self.ntheta):
            for s in range(self.nscan):
                key = (dx[t, s], dy[t, s])
                if key not in cache:
                    cache[key] = shift_probe(self.prb, *key)
                out[t, s] = cache[key]
        return out

    def setobj(self, scan, prb):
        scan = np.asarray(scan, np.float32).reshape(2, self.ntheta, self.nscan)
        self.scan = scan
        self.stx, self.sty = scan_corners(scan)
        sx, sy = scan_phases(scan)
        self.phase = sx * sy
        self.prb = np.asarray(prb).astype(np.complex128).reshape(self.nprb, self.nprb)
        P = self.nprb
        ok = (self.stx >= 0) & (self.sty >= 0)
        if np.any(ok & ((self.stx + P > self.n) | (self.sty + P > self.nz))):
            raise ValueError("scan patch exceeds the object (reference has no upper bound check)")

    def fwd(self, f):
        P, dx, dy = self.nprb, self.detx, self.dety
        f = np.asarray(f).reshape(self.ntheta, self.nz, self.n)
        rs, cs = (dx - P) // 2, (dy - P) // 2
        g = np.zeros((self.ntheta, self.nscan, dx, dy), np.complex128)
        probes = self._frame_probes() if self.quant else None
        for t in range(self.ntheta):
            for s in range(self.nscan):
                x0, y0 = self.stx[t, s], self.sty[t, s]
                if x0 < 0 or y0 < 0:
                    continue
                patch = f[t, y0:y0 + P, x0:x0 + P].astype(np.complex128).T   # [ix, iy]
                g[t, s, rs:rs + P, cs:cs + P] = self.c * (probes[t, s] if probes else self.prb) * patch
        g = sfft.fft2(g, axes=(-2, -1), workers=WORKERS)
        if not self.quant:
            g *= self.phase[:, :, None, None]
        return g

    def adj(self, g):
        P, dx, dy = self.nprb, self.detx, self.dety
        g = np.asarray(g).reshape(self.ntheta, self.nscan, dx, dy).astype(np.complex128)
        rs, cs = (dx - P) // 2, (dy - P) // 2
        if not self.quant:
            g = g * np.conj(self.phase)[:, :, None, None]
        g = sfft.ifft2(g, axes=(-2, -1), workers=WORKERS) * (dx * dy)
        f = np.zeros((self.ntheta, self.nz, self.n), np.complex128)
        probes = self._frame_probes() if self.quant else None
        cp = self.c * np.conj(self.prb)
        for t in range(self.ntheta):
            for s in range(self.nscan):
                x0, y0 = self.stx[t, s], self.sty[t, s]
                if x0 < 0 or y0 < 0:
                    continue
                cps = self.c * np.conj(probes[t, s]) if probes else cp
                f[t, y0:y0 + P, x0:x0 + P] += (cps * g[t, s, rs:rs + P, cs:cs + P]).T
        return f

    # ---- adjoint with respect to the probe (no counterpart in the reference) --
    def adj_probe(self, g, f):
        """gprb[ix, iy] = c sum_frames conj(f[t, y0 + iy, x0 + ix]) G[t, s, rs + ix, cs + iy],
        G = unnormalised inverse DFT of conj(phase) g: the adjoint of fwd as a
        linear map of the probe, for the object f."""
        P, dx, dy = self.nprb, self.detx, self.dety
        g = np.asarray(g).reshape(self.ntheta, self.nscan, dx, dy).astype(np.complex128)
        f = np.asarray(f).reshape(self.ntheta, self.nz, self.n)
        rs, cs = (dx - P) // 2, (dy - P) // 2
        G = sfft.ifft2(g * np.conj(self.phase)[:, :, None, None], axes=(-2, -1), workers=WORKERS) * (dx * dy)
        gp = np.zeros((P, P), np.complex128)
        for t in range(self.ntheta):
            for s in range(self.nscan):
                x0, y0 = self.stx[t, s], self.sty[t, s]
                if x0 < 0 or y0 < 0:
                    continue
                patch = f[t, y0:y0 + P, x0:x0 + P].astype(np.complex128).T   # [ix, iy]
                gp += np.conj(patch) * G[t, s, rs:rs + P, cs:cs + P]
        return self.c * gp

    def fwd_probe(self, f, prb):
        """fwd with the probe prb instead of the one given to setobj."""
        own = self.prb
        self.prb = np.asarray(prb).astype(np.complex128).reshape(self.nprb, self.nprb)
        try:
            return self.fwd(f)
        finally:
            self.prb = own
