"""Seeded synthetic inputs with the shapes and value ranges of the workloads.

No public dataset is used (the reference's chip phantoms are not
distributed); these generators stand in for them:

* :func:`phantom`  complex refractive index u = -delta + i*beta on [nz, n, n]
  from random ellipsoids, delta in [0, delta_max], beta in [0, beta_max]
  (sign convention of the reference driver test.py:46-48);
* :func:`probe`    Gaussian amplitude with a smooth seeded random phase;
* :func:`raster_scan`, :func:`jittered_spiral_scan`  scan positions in the
  reference layout [2, ntheta, nscan] (x then y), float32, with -1 marking
  an unused slot (the reference's sentinel, kernels.cuh:256).
"""
from __future__ import annotations

import numpy as np


def phantom(n: int, nz: int | None = None, seed: int = 0, n_ellipsoids: int = 20,
            delta_max: float = 1e-5, beta_max: float = 1e-6) -> np.ndarray:
    nz = n if nz is None else nz
    rng = np.random.default_rng(seed)
    z, y, x = np.meshgrid(np.linspace(-1, 1, nz), np.linspace(-1, 1, n), np.linspace(-1, 1, n), indexing="ij")
    delta = np.zeros((nz, n, n))
    beta = np.zeros((nz, n, n))
    for _ in range(n_ellipsoids):
        c = rng.uniform(-0.45, 0.45, 3)
        r = rng.uniform(0.05, 0.3, 3)
        a = rng.uniform(0, np.pi)
        xr = (x - c[0]) * np.cos(a) + (y - c[1]) * np.sin(a)
        yr = -(x - c[0]) * np.sin(a) + (y - c[1]) * np.cos(a)
        inside = (xr / r[0]) ** 2 + (yr / r[1]) ** 2 + ((z - c[2]) / r[2]) ** 2 <= 1
        delta[inside] += rng.uniform(0.1, 1.0)
        beta[inside] += rng.uniform(0.1, 1.0)
    delta *= delta_max / max(delta.max(), 1e-30)
    beta *= beta_max / max(beta.max(), 1e-30)
    return (-delta + 1j * beta).astype(np.complex64)


def _smooth_noise(shape, rng, width):
    f = rng.standard_normal(shape)
    k = np.fft.fftfreq(shape[0])[:, None] ** 2 + np.fft.fftfreq(shape[1])[None, :] ** 2
    f = np.real(np.fft.ifft2(np.fft.fft2(f) * np.exp(-k * (np.pi * width) ** 2 * 2)))
    return f / max(np.abs(f).max(), 1e-30)


def probe(size: int, sigma: float | None = None, seed: int = 0, phase_amp: float = 0.5,
          maxint: float = 1.0) -> np.ndarray:
    """Gaussian amplitude (sigma in pixels, default size*12/64) times exp(i*phase)."""
    sigma = size * 12.0 / 64.0 if sigma is None else sigma
    rng = np.random.default_rng(seed)
    t = np.arange(size) - (size - 1) / 2
    amp = np.exp(-(t[:, None] ** 2 + t[None, :] ** 2) / (2 * sigma ** 2))
    ph = phase_amp * _smooth_noise((size, size), rng, size / 8)
    return (np.sqrt(maxint) * amp * np.exp(1j * ph)).astype(np.complex64)


def raster_scan(ntheta: int, nside: int, n: int, nz: int, nprb: int, step: float | None = None) -> np.ndarray:
    """nside x nside raster per angle; positions clamped so every patch fits.

    With ``step=None`` the positions are ``linspace(0, n - nprb, nside)``.
    """
    if step is None:
        px = np.linspace(0, n - nprb, nside)
        py = np.linspace(0, nz - nprb, nside)
    else:
        px = np.minimum(np.arange(nside) * step, n - nprb)
        py = np.minimum(np.arange(nside) * step, nz - nprb)
    gx, gy = np.meshgrid(px, py)
    scan = np.empty((2, ntheta, nside * nside), np.float32)
    scan[0] = gx.ravel()[None, :]
    scan[1] = gy.ravel()[None, :]
    return scan


def jittered_spiral_scan(ntheta: int, n: int, nz: int, nprb: int, counts, jitter: float = 3.0,
                         seed: int = 0) -> np.ndarray:
    """Per-angle spiral scans with uneven counts, padded with -1 to max(counts)."""
    rng = np.random.default_rng(seed)
    counts = np.asarray(counts, int)
    nmax = int(counts.max())
    scan = -np.ones((2, ntheta, nmax), np.float32)
    cx, cy = (n - nprb) / 2, (nz - nprb) / 2
    for t in range(ntheta):
        k = np.arange(counts[t])
        r = np.sqrt(k / max(counts[t] - 1, 1))
        a = k * 2.39996323 + rng.uniform(0, 2 * np.pi)
        x = cx + r * cx * np.cos(a) + rng.uniform(-jitter, jitter, counts[t])
        y = cy + r * cy * np.sin(a) + rng.uniform(-jitter, jitter, counts[t])
        scan[0, t, :counts[t]] = np.clip(x, 0, n - nprb - 0.5)
        scan[1, t, :counts[t]] = np.clip(y, 0, nz - nprb - 0.5)
    return scan


def angles(ntheta: int, lo: float = 0.0, hi: float = np.pi) -> np.ndarray:
    """ntheta angles uniform on [lo, hi), float32."""
    return (lo + (hi - lo) * np.arange(ntheta) / ntheta).astype(np.float32)
