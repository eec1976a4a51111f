"""NumPy restatement of the reference USFFT Radon operator.

TEST INFRASTRUCTURE (the oracle).  Follows, step by step:

* constructor / parameters     src/cuda/radonusfft.cu:5-12
* fwd                          src/cuda/radonusfft.cu:54-92
* adj                          src/cuda/radonusfft.cu:94-139
* setobj                       src/cuda/radonusfft.cu:141-144
* kernels                      src/include/kernels.cuh:5-216

Arithmetic is complex128, except where the reference takes a discrete
decision from a float32 value (polar coordinates, floor() of the grid
position, the circular mask, the kernel parameter mu); those are evaluated
in float32 exactly as the reference writes them.  cuFFT's C2C transforms
are unnormalised with FORWARD = exp(-2*pi*i...), which scipy.fft matches
(inverse = ifft * length); the FFTs run on all host cores (``workers``).
The gridding is one sparse matrix (taps x weights) applied to every slice
at once, its columns split over threads.

The reference computes the polar coordinates with the fast intrinsics
``__cosf``/``__sinf`` (kernels.cuh:91-92).  Their results cannot be
reproduced on the CPU, so :func:`takexy` uses float32 ``cos``/``sin`` and
every entry point accepts explicit coordinate tables (``xy=``) so that a
test can hand the oracle the exact tables a GPU computed.
"""
from __future__ import annotations

import math
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import scipy.fft as sfft
import scipy.sparse as sparse

from ._threads import WORKERS

PI_REF = 3.1415926535  # kernels.cuh:1 (#define PI 3.1415926535)


def usfft_params(n: int):
    """Internal size N, kernel half-width M and Gaussian parameter mu.

    radonusfft.cu:7-12: N = n*3/2; eps = 1e-6 (float);
    mu = -log(eps)/(2*N*N) in float; M = ceil(2N/PI*sqrt(-mu*log(eps)+(mu*N)^2/4)).
    """
    N = n * 3 // 2
    eps = np.float32(1e-6)
    mu = np.float32(-np.log(eps)) / np.float32(2 * N * N)
    inner = np.float32(-mu * np.log(eps)) + np.float32((mu * np.float32(N)) ** 2 / 4)
    M = int(math.ceil(2 * N / PI_REF * math.sqrt(float(inner))))
    return N, M, np.float32(mu)


def takexy(theta, N: int):
    """Polar sample coordinates, kernels.cuh:84-95, layout [ntheta, N].

    x = (k-N/2)/N*cos(theta), y = -(k-N/2)/N*sin(theta) in float32, each
    clamped to 0.5-1e-5 when >= 0.5.
    """
    theta = np.asarray(theta, dtype=np.float32)
    k = np.arange(N)
    s = (k - N // 2).astype(np.float32) / np.float32(N)
    sn = (-(k - N // 2)).astype(np.float32) / np.float32(N)
    x = (s[None, :] * np.cos(theta).astype(np.float32)[:, None]).astype(np.float32)
    y = (sn[None, :] * np.sin(theta).astype(np.float32)[:, None]).astype(np.float32)
    clamp = np.float32(0.5 - 1e-5)
    x[x >= np.float32(0.5)] = clamp
    y[y >= np.float32(0.5)] = clamp
    return x, y


def circ_mask(N: int):
    """kernels.cuh:160-172 with r = 1.0f/N: (4x^2+4y^2) < 1-r in float32."""
    t = (np.arange(N) - N // 2).astype(np.float32) / np.float32(N)
    x = t[None, :]
    y = t[:, None]
    lhs = np.float32(4) * x * x + np.float32(4) * y * y
    rhs = np.float32(1) - np.float32(1.0) / np.float32(N)
    return (lhs < rhs).astype(np.float64)


def deapod(N: int, mu):
    """phi(tx,ty) = exp(-mu(tx-N/2)^2 - mu(ty-N/2)^2), kernels.cuh:12,23."""
    t = (np.arange(N) - N // 2).astype(np.float64)
    mu = float(mu)
    return np.exp(-mu * t[None, :] ** 2 - mu * t[:, None] ** 2)


def checker(L: int):
    """fftshiftc sign (-1)^(x+y), kernels.cuh:28-37."""
    s = 1.0 - 2.0 * ((np.arange(L) + 1) % 2)
    return s[:, None] * s[None, :]


def checker1(L: int):
    """fftshift1c sign (1-2((k+1)%2)), kernels.cuh:39-48."""
    return 1.0 - 2.0 * ((np.arange(L) + 1) % 2)


class GridTaps:
    """Tap indices and weights of the Gaussian gridding, kernels.cuh:97-158.

    For point p = (theta, k): ell0 = floor(2N*x0) - M + i0,
    w0 = ell0/(2N) - x0 (float32), w = PI/mu*exp(-PI^2/mu*(w0^2+w1^2)).
    The haloed grid index N+M+ell of the reference is, after the halo
    wrap/fold (kernels.cuh:50-82), the periodic FFT index (N+ell) mod 2N.
    """

    def __init__(self, x, y, N: int, M: int, mu):
        G = 2 * N
        x = np.asarray(x, np.float32).ravel()
        y = np.asarray(y, np.float32).ravel()
        fx = np.floor(np.float32(G) * x).astype(np.int64)
        fy = np.floor(np.float32(G) * y).astype(np.int64)
        i = np.arange(2 * M + 1)
        ell0 = fx[:, None] - M + i[None, :]
        ell1 = fy[:, None] - M + i[None, :]
        w0 = (ell0.astype(np.float32) / np.float32(G) - x[:, None]).astype(np.float32)
        w1 = (ell1.astype(np.float32) / np.float32(G) - y[:, None]).astype(np.float32)
        mu = float(mu)
        a = PI_REF * PI_REF / mu
        wx = np.exp(-a * w0.astype(np.float64) ** 2)
        wy = np.exp(-a * w1.astype(np.float64) ** 2)
        self.w = (PI_REF / abs(mu)) * wy[:, :, None] * wx[:, None, :]
        cx = np.mod(N + ell0, G)
        cy = np.mod(N + ell1, G)
        self.idx = (cy[:, :, None] * G + cx[:, None, :])
        self.npts = x.size
        self.G = G
        taps = (2 * M + 1) ** 2
        self.S = sparse.csr_matrix((self.w.ravel(), self.idx.ravel(), np.arange(0, self.npts * taps + 1, taps)),
                                   shape=(self.npts, G * G))
        self.ST = self.S.T.tocsr()

    @staticmethod
    def _apply(A, X):
        """A @ X for X [cols, k] complex, the k columns split over threads."""
        k = X.shape[1]
        if k < 2 or WORKERS < 2:
            return A @ X
        parts = np.array_split(np.arange(k), min(k, WORKERS))
        with ThreadPoolExecutor(len(parts)) as ex:
            cols = list(ex.map(lambda c: A @ X[:, c], parts))
        return np.concatenate(cols, axis=1)

    def gather(self, F):
        """F: [G, G] or [nz, G, G] complex -> samples [npts] or [npts, nz]."""
        if F.ndim == 2:
            return self.S @ F.ravel()
        return self._apply(self.S, np.ascontiguousarray(F.reshape(F.shape[0], -1).T))

    def scatter(self, g):
        """g: [npts] or [npts, nz] complex -> grid [G, G] or [G*G, nz] (transpose of gather)."""
        if g.ndim == 1:
            return (self.ST @ g).reshape(self.G, self.G)
        return self._apply(self.ST, np.ascontiguousarray(g))


class RadonUSFFT:
    """Oracle twin of class radonusfft (radonusfft.cuh, radonusfft.cu).

    Shapes follow the reference: f is [Nz, n, n], g is [Ntheta, Nz, n]
    (complex).  ``xy`` optionally supplies the polar coordinate tables
    (each [Ntheta, N] float32) instead of :func:`takexy`; ``params``
    optionally supplies (N, M, mu).
    """

    def __init__(self, ntheta: int, nz: int, n: int, params=None):
        self.ntheta, self.nz, self.n = ntheta, nz, n
        N, M, mu = params if params is not None else usfft_params(n)
        self.N, self.M, self.mu = N, M, np.float32(mu)
        self.G = 2 * N
        self.theta = None
        self._taps = None
        self._mask = circ_mask(N)
        self._phi = deapod(N, self.mu)

    def setobj(self, theta, xy=None):
        """radonusfft.cu:141-144 (plus the takexy of :76/:116)."""
        self.theta = np.asarray(theta, np.float32)
        x, y = takexy(self.theta, self.N) if xy is None else xy
        self.x = np.asarray(x, np.float32).reshape(self.ntheta, self.N)
        self.y = np.asarray(y, np.float32).reshape(self.ntheta, self.N)
        self._taps = GridTaps(self.x, self.y, self.N, self.M, self.mu)

    # ---- forward: radonusfft.cu:54-92 -------------------------------------
    def fwd(self, f):
        n, N, G, nz = self.n, self.N, self.G, self.nz
        f = np.asarray(f).reshape(nz, n, n)
        c0 = N // 6
        # memcpy2D into the centre of N x N, then pad2 edge replication
        idx = np.clip(np.arange(N), c0, 5 * N // 6 - 1) - c0
        fp = f.astype(np.complex128)[:, idx][:, :, idx]
        fp = fp * self._mask                                  # circ
        fde = np.zeros((nz, G, G), np.complex128)
        fde[:, N // 2:N // 2 + N, N // 2:N // 2 + N] = fp / self._phi / (4 * N * N)  # divphi
        chk = checker(G)
        fde *= chk                                            # fftshiftc
        F = sfft.fft2(fde, axes=(-2, -1), workers=WORKERS)    # cufft fwd 2-D
        F *= chk                                              # fftshiftc on the haloed grid
        g = (self._taps.gather(F) / N).reshape(self.ntheta, N, nz).transpose(0, 2, 1)
        s1 = checker1(N)
        g = sfft.ifft(g * s1, axis=-1, workers=WORKERS) * N * s1   # fftshift1c, 1-D inverse, fftshift1c
        return g[:, :, c0:c0 + n]

    # ---- adjoint: radonusfft.cu:94-139 ------------------------------------
    def adj(self, g):
        n, N, G, nz = self.n, self.N, self.G, self.nz
        g = np.asarray(g).reshape(self.ntheta, nz, n)
        c0 = N // 6
        idx = np.clip(np.arange(N), c0, 5 * N // 6 - 1) - c0   # pad (kernels.cuh:189)
        gl = g.astype(np.complex128)[:, :, idx]
        s1 = checker1(N)
        gl = sfft.fft(gl * s1, axis=-1, workers=WORKERS) * s1  # fftshift1c, 1-D fwd, fftshift1c
        chk = checker(G)
        pts = np.ascontiguousarray(gl.transpose(0, 2, 1).reshape(self.ntheta * N, nz)) / N
        F = self._taps.scatter(pts).T.reshape(nz, G, G)         # scatter + wrapadj
        F *= chk                                               # fftshiftc on haloed grid
        fde = sfft.ifft2(F, axes=(-2, -1), workers=WORKERS) * (G * G)   # cufft inverse 2-D
        fde *= chk                                             # fftshiftc
        fc = fde[:, N // 2:N // 2 + N, N // 2:N // 2 + N] / self._phi / (4 * N * N)
        fc = fc * self._mask                                   # circ
        return fc[:, c0:c0 + n, c0:c0 + n]

    # ---- exact adjoint of fwd (no counterpart in the reference) ---------------
    def adj_exact(self, g):
        """The exact adjoint of fwd: adj with the edge-replicating pad of the
        detector lines replaced by the zero padding that is the adjoint of
        fwd's crop, and the final crop replaced by the fold that is the adjoint
        of pad2 (every margin pixel of the N x N slice added onto the edge
        pixel it copies).  Equals adj where g and the result's border vanish."""
        n, N, G, nz = self.n, self.N, self.G, self.nz
        g = np.asarray(g).reshape(self.ntheta, nz, n)
        c0 = N // 6
        gl = np.zeros((self.ntheta, nz, N), np.complex128)
        gl[:, :, c0:c0 + n] = g
        s1 = checker1(N)
        gl = sfft.fft(gl * s1, axis=-1, workers=WORKERS) * s1
        chk = checker(G)
        pts = np.ascontiguousarray(gl.transpose(0, 2, 1).reshape(self.ntheta * N, nz)) / N
        F = self._taps.scatter(pts).T.reshape(nz, G, G)
        F *= chk
        fde = sfft.ifft2(F, axes=(-2, -1), workers=WORKERS) * (G * G)
        fde *= chk
        fc = fde[:, N // 2:N // 2 + N, N // 2:N // 2 + N] / self._phi / (4 * N * N)
        fc = fc * self._mask
        idx = np.clip(np.arange(N), c0, c0 + n - 1) - c0            # pad2's source index
        fold = np.zeros((n, N))
        fold[idx, np.arange(N)] = 1.0                                # fold[i, t] = 1 where t copies i
        return np.einsum("it,ztu,ju->zij", fold, fc, fold)

