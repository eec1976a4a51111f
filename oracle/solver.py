"""NumPy restatement of the reference ADMM Solver.

TEST INFRASTRUCTURE (the oracle).  Mirrors src/ptychotomo/solver.py:19-336
method by method with CuPy replaced by NumPy.  Arrays are complex64 like the
reference; every reduction (norms, dot products, sums of the likelihood)
is accumulated in float64, which is the precision choice the GPU engine
makes too.  Documented fixes: ``takexi`` uses ``r = prb.shape[0] // 2``
(solver.py:151 divides with ``/`` and then slices with the float); the CG
loops stop once the line search returns gamma = 0 (gamma only halves, so the
iterate cannot change any more; the reference would go on to divide by an
exactly-zero Dai-Yuan denominator and return NaN), and a zero Dai-Yuan
denominator gives beta = 0.
"""
from __future__ import annotations

from concurrent.futures import ThreadPoolExecutor

import numpy as np

from ._threads import WORKERS
from .ptycho import PtychoFFT
from .usfft import RadonUSFFT

PLANCK_CONSTANT = 6.58211928e-19  # [keV*s]   solver.py:15
SPEED_OF_LIGHT = 299792458e+2    # [cm/s]    solver.py:16


def _norm2(a):
    """||a||^2 accumulated in float64."""
    a = np.asarray(a)
    return float(np.sum(a.real.astype(np.float64) ** 2 + a.imag.astype(np.float64) ** 2))


def _vdot(a, b):
    """sum(conj(a)*b) accumulated in complex128."""
    return complex(np.vdot(np.asarray(a).astype(np.complex128).ravel(),
                           np.asarray(b).astype(np.complex128).ravel()))


def _par_sum(fn, *arrays):
    """sum of fn(chunk...) over chunks of the arrays' first axis, in threads
    (NumPy releases the GIL inside its elementwise loops)."""
    k = min(WORKERS, arrays[0].shape[0])
    if k < 2:
        return fn(*arrays)
    bounds = np.linspace(0, arrays[0].shape[0], k + 1).astype(int)
    with ThreadPoolExecutor(k) as ex:
        parts = ex.map(lambda i: fn(*(a[bounds[i]:bounds[i + 1]] for a in arrays)), range(k))
        return sum(parts)


class Solver:
    """solver.py:19-46 constructor; operators as in solver.py:48-146."""

    def __init__(self, prb, scan, theta, det, voxelsize, energy, ntheta, nz, n, ptheta, pnz, xy=None):
        self.voxelsize = voxelsize
        self.energy = energy
        self.scan = np.asarray(scan, np.float32)
        self.prb = np.asarray(prb).astype(np.complex64)
        self.ntheta, self.nz, self.n = ntheta, nz, n
        self.nscan = self.scan.shape[2]
        self.ndety, self.ndetx = det[0], det[1]
        self.nprb = self.prb.shape[0]
        self.ptheta, self.pnz = ptheta, pnz
        self.cl_ptycho = PtychoFFT(ptheta, nz, n, ptheta, self.nscan, self.ndety, self.ndetx, self.nprb)
        self.cl_tomo = RadonUSFFT(ntheta, pnz, n)
        self.cl_tomo.setobj(np.asarray(theta, np.float32), xy=xy)
        self.coeftomo = np.float32(1 / np.sqrt(ntheta * n / 2))
        self.coefptycho = np.float32(1 / np.abs(self.prb).max())
        self.coefdata = np.float32(1 / (self.ndetx * self.ndety * (np.abs(self.prb) ** 2).max()))

    # ---- elementwise maps, solver.py:48-64 -------------------------------
    def mlog(self, psi):
        res = psi.copy()
        res[np.abs(psi) < 1e-32] = 1e-32
        return np.log(res)

    def wavenumber(self):
        return 2 * np.pi / (2 * np.pi * PLANCK_CONSTANT * SPEED_OF_LIGHT / self.energy)

    def exptomo(self, psi):
        return np.exp(1j * psi * self.voxelsize * self.wavenumber() / self.coeftomo).astype(np.complex64)

    def logtomo(self, psi):
        return (-1j / self.wavenumber() * self.mlog(psi) / self.voxelsize * self.coeftomo).astype(np.complex64)

    # ---- tomography, solver.py:67-97 ---------------------------------------
    def fwd_tomo(self, u):
        return (self.cl_tomo.fwd(u) * self.coeftomo).astype(np.complex64)

    def adj_tomo(self, data):
        return (self.cl_tomo.adj(data) * self.coeftomo).astype(np.complex64)

    def fwd_tomo_batch(self, u):
        res = np.zeros([self.ntheta, self.nz, self.n], np.complex64)
        for k in range(self.nz // self.pnz):
            ids = slice(k * self.pnz, (k + 1) * self.pnz)
            res[:, ids] = self.fwd_tomo(u[ids])
        return res

    def adj_tomo_batch(self, data):
        res = np.zeros([self.nz, self.n, self.n], np.complex64)
        for k in range(self.nz // self.pnz):
            ids = slice(k * self.pnz, (k + 1) * self.pnz)
            res[ids] = self.adj_tomo(data[:, ids])
        return res

    # ---- ptychography, solver.py:100-125 -----------------------------------
    def _setobj(self, ids):
        self.cl_ptycho.setobj(self.scan[:, ids], self.prb)

    def fwd_ptycho(self, psi):
        return (self.cl_ptycho.fwd(psi) * self.coefptycho).astype(np.complex64)

    def fwd_ptycho_batch(self, psi):
        data = np.zeros([self.ntheta, self.nscan, self.ndety, self.ndetx], np.float32)
        for k in range(self.ntheta // self.ptheta):
            ids = slice(k * self.ptheta, (k + 1) * self.ptheta)
            self._setobj(ids)
            data[ids] = (np.abs(self.fwd_ptycho(psi[ids])) ** 2 / self.coefdata).astype(np.float32)
        return data

    def adj_ptycho(self, data):
        return (self.cl_ptycho.adj(data) * self.coefptycho).astype(np.complex64)

    # ---- TV regulariser, solver.py:128-146 ---------------------------------
    def fwd_reg(self, u):
        res = np.zeros([3, *u.shape], np.complex64)
        res[0, :, :, :-1] = u[:, :, 1:] - u[:, :, :-1]
        res[1, :, :-1, :] = u[:, 1:, :] - u[:, :-1, :]
        res[2, :-1, :, :] = u[1:, :, :] - u[:-1, :, :]
        res *= np.float32(2 / np.sqrt(3))
        return res

    def adj_reg(self, gr):
        res = np.zeros(gr.shape[1:], np.complex64)
        res[:, :, 1:] = gr[0, :, :, 1:] - gr[0, :, :, :-1]
        res[:, :, 0] = gr[0, :, :, 0]
        res[:, 1:, :] += gr[1, :, 1:, :] - gr[1, :, :-1, :]
        res[:, 0, :] += gr[1, :, 0, :]
        res[1:, :, :] += gr[2, 1:, :, :] - gr[2, :-1, :, :]
        res[0, :, :] += gr[2, 0, :, :]
        res *= np.float32(-2 / np.sqrt(3))
        return res

    # ---- linearisation, solver.py:149-168 ----------------------------------
    def takexi(self, psi, phi, lamd, mu, rho, tau):
        r = self.prb.shape[0] // 2
        m1 = np.mean(np.angle(psi[:, :, r:2 * r]).astype(np.float64))
        m2 = np.mean(np.angle(psi[:, :, psi.shape[2] - 2 * r:psi.shape[2] - r]).astype(np.float64))
        pshift = (m1 + m2) / 2
        t = (psi - lamd / np.float32(rho)).astype(np.complex64)
        t = (t * np.exp(-1j * pshift)).astype(np.complex64)
        logt = self.mlog(t)
        K = (1j * self.voxelsize * self.wavenumber() * t / self.coeftomo).astype(np.complex64)
        K = (K / np.abs(K).max()).astype(np.complex64)
        xi0 = (K * (-1j * logt / (self.voxelsize * self.wavenumber())) * self.coeftomo).astype(np.complex64)
        xi1 = (phi - mu / np.float32(tau)).astype(np.complex64)
        return xi0, xi1, K, pshift

    # ---- line search, solver.py:171-177 ------------------------------------
    trace = None   # list: records (kind, gamma) of every line search when set

    def line_search(self, minf, gamma, u, fu, d, fd, kind=""):
        while minf(u, fu) - minf(u + gamma * d, fu + gamma * fd) < 0 and gamma > 1e-12:
            gamma *= 0.5
        if gamma <= 1e-12:
            gamma = 0
        if self.trace is not None:
            self.trace.append((kind, gamma))
        return gamma

    # ---- CG tomography, solver.py:180-203 ----------------------------------
    def cg_tomo(self, xi0, xi1, K, init, rho, tau, titer):
        def minf(KRu, gu):
            return rho * _norm2(KRu - xi0) + tau * _norm2(gu - xi1)

        u = init.copy()
        gamma = 2
        for i in range(titer):
            KRu = (K * self.fwd_tomo_batch(u)).astype(np.complex64)
            gu = self.fwd_reg(u)
            grad = (rho * self.adj_tomo_batch(np.conj(K) * (KRu - xi0))
                    + tau * self.adj_reg(gu - xi1)).astype(np.complex64)
            if i == 0:
                d = -grad
            else:
                den = _vdot(d, grad - grad0)
                beta = _norm2(grad) / den if den != 0 else 0.0
                d = (-grad + beta * d).astype(np.complex64)
            grad0 = grad
            gamma = self.line_search(minf, gamma, KRu, gu,
                                     (K * self.fwd_tomo_batch(d)).astype(np.complex64), self.fwd_reg(d), "tomo")
            u = (u + gamma * d).astype(np.complex64)
            if gamma == 0:
                break   # gamma only halves: u can no longer change in this call
        return u

    # ---- CG ptychography, solver.py:206-254 --------------------------------
    def cg_ptycho(self, data, init, h, lamd, rho, piter, model):
        def data_term(fpsi, data):
            if model == 'gaussian':
                return _norm2(np.abs(fpsi) - np.sqrt(data))
            a = np.abs(fpsi).astype(np.float64)
            return float(np.sum(a ** 2 - 2 * data.astype(np.float64) * self.mlog(a)))

        def minf(psi, fpsi):
            f = _par_sum(data_term, fpsi, data)
            f += rho * _norm2(h - psi + lamd / rho)
            return f

        psi = init.copy()
        gamma = 2
        for i in range(piter):
            fpsi = self.fwd_ptycho(psi)
            if model == 'gaussian':
                grad = self.adj_ptycho(fpsi - np.sqrt(data) * np.exp(1j * np.angle(fpsi)))
            else:
                grad = self.adj_ptycho(fpsi - data * fpsi / (np.abs(fpsi) ** 2 + 1e-32))
            grad = (grad - rho * (h - psi + lamd / rho)).astype(np.complex64)
            if i == 0:
                d = -grad
            else:
                den = _vdot(d, grad - grad0)
                beta = _norm2(grad) / den if den != 0 else 0.0
                d = (-grad + beta * d).astype(np.complex64)
            grad0 = grad
            fd = self.fwd_ptycho(d)
            gamma = self.line_search(minf, gamma, psi, fpsi, d, fd, "ptycho")
            psi = (psi + gamma * d).astype(np.complex64)
            if gamma == 0:
                break   # gamma only halves: psi can no longer change in this call
        return psi

    def cg_ptycho_batch(self, data, init, h, lamd, rho, piter, model):
        psi = init.copy()
        for k in range(self.ntheta // self.ptheta):
            ids = slice(k * self.ptheta, (k + 1) * self.ptheta)
            self._setobj(ids)
            datap = (data[ids] * self.coefdata).astype(np.float32)
            psi[ids] = self.cg_ptycho(datap, psi[ids], h[ids], lamd[ids], rho, piter, model)
        return psi

    # ---- regulariser / penalties / monitor, solver.py:257-305 --------------
    def solve_reg(self, u, mu, tau, alpha):
        z = (self.fwd_reg(u) + mu / np.float32(tau)).astype(np.complex64)
        za = np.sqrt(np.real(np.sum(z * np.conj(z), 0)))
        thr = alpha / tau
        z[:, za <= thr] = 0
        m = za > thr
        z[:, m] -= (thr * z[:, m] / za[m]).astype(np.complex64)
        return z

    def update_penalty(self, psi, h, h0, phi, e, e0, rho, tau):
        r = _norm2(psi - h)
        s = _norm2(rho * (h - h0))
        if r > 10 * s:
            rho *= 2
        elif s > 10 * r:
            rho *= 0.5
        r = _norm2(phi - e)
        s = _norm2(tau * (e - e0))
        if r > 10 * s:
            tau *= 2
        elif s > 10 * r:
            tau *= 0.5
        return rho, tau

    def take_lagr(self, psi, phi, data, h, e, lamd, mu, alpha, rho, tau, model):
        lagr = np.zeros(7, np.float64)
        for k in range(self.ntheta // self.ptheta):
            ids = slice(k * self.ptheta, (k + 1) * self.ptheta)
            self._setobj(ids)
            fpsi = self.fwd_ptycho(psi[ids])
            datap = (data[ids] * self.coefdata).astype(np.float64)
            a = np.abs(fpsi).astype(np.float64)
            if model == 'poisson':
                lagr[0] += np.sum(a ** 2 - 2 * datap * self.mlog(a)
                                  - (datap - 2 * datap * self.mlog(np.sqrt(datap))))
            else:
                lagr[0] += _norm2(a - np.sqrt(datap))
        lagr[1] = alpha * np.sum(np.sqrt(np.real(np.sum(phi * np.conj(phi), 0)).astype(np.float64)))
        lagr[2] = 2 * np.real(_vdot(lamd, h - psi))
        lagr[3] = rho * _norm2(h - psi)
        lagr[4] = 2 * np.real(_vdot(mu, e - phi))
        lagr[5] = tau * _norm2(e - phi)
        lagr[6] = np.sum(lagr[0:5])   # solver.py:304 sums terms 0..4 only
        return lagr

    # ---- ADMM, solver.py:308-336 -------------------------------------------
    STATE = ("u", "psi", "h", "e", "phi", "lamd", "mu")

    def admm_step(self, m, st, rho, tau, data, alpha, piter, titer, model):
        """One iteration of the loop body solver.py:311-329 from the state st
        (a dict of u, psi, h, e, phi, lamd, mu); returns (new state, rho, tau)."""
        u, psi, h, e, phi, lamd, mu = (st[k] for k in self.STATE)
        h0, e0 = h, e
        psi = self.cg_ptycho_batch(data, psi, h, lamd, rho, piter + (m < 2) * 32, model)
        xi0, xi1, K, pshift = self.takexi(psi, phi, lamd, mu, rho, tau)
        u = self.cg_tomo(xi0, xi1, K, u, rho, tau, titer)
        phi = self.solve_reg(u, mu, tau, alpha)
        h = (self.exptomo(self.fwd_tomo_batch(u)) * np.exp(1j * pshift)).astype(np.complex64)
        e = self.fwd_reg(u)
        lamd = (lamd + rho * (h - psi)).astype(np.complex64)
        mu = (mu + tau * (e - phi)).astype(np.complex64)
        rho, tau = self.update_penalty(psi, h, h0, phi, e, e0, rho, tau)
        return dict(u=u, psi=psi, h=h, e=e, phi=phi, lamd=lamd, mu=mu), rho, tau

    def admm(self, data, h, e, psi, phi, lamd, mu, u, alpha, piter, titer, niter, model,
             lagr_every=10, history=None):
        rho, tau = 0.5, 0.5
        st = dict(u=u, psi=psi, h=h, e=e, phi=phi, lamd=lamd, mu=mu)
        for m in range(niter):
            st, rho, tau = self.admm_step(m, st, rho, tau, data, alpha, piter, titer, model)
            if history is not None:
                history.append(dict(m=m, rho=rho, tau=tau))
            if lagr_every and m % lagr_every == 0 and history is not None:
                history[-1]["lagr"] = self.take_lagr(st["psi"], st["phi"], data, st["h"], st["e"], st["lamd"],
                                                     st["mu"], alpha, rho, tau, model)
        return st["u"], st["psi"]
