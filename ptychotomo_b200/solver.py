"""Drop-in ADMM ptycho-tomography Solver on torch CUDA tensors.

Same constructor and methods as the reference Solver
(src/ptychotomo/solver.py:19-336); arrays are torch CUDA tensors
(complex64 / float32) instead of CuPy arrays.  Every arithmetic step runs in
libptychotomo_b200.so: the USFFT and ptycho operators, and the Solver
kernels (linear combinations, TV, exp/log maps, FP64 reductions).  torch
only allocates memory.

Differences from the reference, all deliberate:
* reductions (norms, inner products, the Poisson log-likelihood, the
  Lagrangian) accumulate in FP64;
* the line searches evaluate the decrease minf(x) - minf(x + g d) directly:
  quadratic terms in closed form (||w + g d||^2 - ||w||^2 = 2 g Re<w, d> +
  g^2 ||d||^2) and the Poisson / Gaussian term per element without
  cancellation (log1p of the relative change), summed in FP64, for 2, then
  8, then 16 step lengths per pass.  They take the halving decisions of
  solver.py:171-177 exactly, except where the decrease is within FP32
  rounding of zero (near convergence), where the reference's own float
  atomics make it differ from run to run;
* takexi uses r = prb.shape[0] // 2 (solver.py:151 slices with a float);
* cg_tomo evaluates K R u - xi0 and J u - xi1 once per call and then advances
  them with each step (+ gamma K R d, + gamma J d, which the line search has
  formed already) instead of re-evaluating the Radon transform of the new
  iterate (solver.py:189-190): the same quantities up to FP32 rounding, one
  USFFT forward and one TV pass fewer per CG iteration; admm takes R u for
  h (solver.py:325) from the same running sum instead of a new transform;
* likewise cg_ptycho takes F Q psi of the next iterate as F Q psi + gamma
  F Q d, stored by the line-search kernel for its first candidate step,
  whenever that step is the one taken (solver.py:219 recomputes it); the
  forward is recomputed otherwise;
* a CG loop stops once its line search returns gamma = 0 (gamma only
  halves, so the iterate cannot change any more; the reference would divide
  by an exactly-zero Dai-Yuan denominator next and return NaN), and a zero
  Dai-Yuan denominator gives beta = 0;
* fwd_ptycho_batch returns a device tensor; admm accepts data on the host
  or the device and keeps it resident on the device;
* all angles / slices of a *_batch call go through one operator launch
  (the reference loops over ptheta / pnz chunks; results are identical).
"""
from __future__ import annotations

import math
import os

import numpy as np
import torch

from . import kernels as K
from .operators import ptychofft, radonusfft

PLANCK_CONSTANT = 6.58211928e-19  # [keV*s]  solver.py:15
SPEED_OF_LIGHT = 299792458e+2    # [cm/s]   solver.py:16

_MODELS = {"poisson": 0, "gaussian": 1}


def _as_tuple(x):
    return tuple(x) if isinstance(x, (list, tuple)) else x


def _dev_tensor(x, dtype, device):
    if isinstance(x, torch.Tensor):
        return x.to(device=device, dtype=dtype).contiguous()
    return torch.as_tensor(np.asarray(x), dtype=dtype, device=device).contiguous()


class Solver:
    def __init__(self, prb, scan, theta, det, voxelsize, energy, ntheta, nz, n, ptheta, pnz, device=None,
                 subpixel=0, _held=None):
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        dev = self.device
        self.voxelsize = voxelsize
        self.energy = energy
        self.prb = _dev_tensor(prb, torch.complex64, dev)
        self.theta = _dev_tensor(theta, torch.float32, dev)
        self.ntheta, self.nz, self.n = ntheta, nz, n
        # the angles [th0, th1) and slices [z0, z1) this process holds: all of
        # them here, one shard of each under ShardedSolver (angle-major arrays
        # psi, h, lamd, data hold the angles; slice-major u, e, phi, mu the slices)
        th0, th1, z0, z1 = _held if _held is not None else (0, ntheta, 0, nz)
        self.theta_range, self.z_range = (th0, th1), (z0, z1)
        self.ntheta_held, self.nz_held = th1 - th0, z1 - z0
        self.scan = _dev_tensor(scan, torch.float32, dev)[:, th0:th1].contiguous()
        self.nscan = self.scan.shape[2]
        self.ndety, self.ndetx = det[0], det[1]
        self.nprb = self.prb.shape[0]
        self.ptheta, self.pnz = ptheta, pnz
        if self.ntheta_held % ptheta or self.nz_held % pnz:
            raise ValueError("ptheta must divide ntheta and pnz must divide nz (solver.py:86,111)")
        # tomography: the pnz-chunk operator of fwd_tomo/adj_tomo and one for whole batches
        self.cl_tomo = radonusfft(ntheta, pnz, n)
        self.cl_tomo.setobj(self.theta)
        if pnz == self.nz_held:
            self._tomo_all = self.cl_tomo
        else:
            self._tomo_all = radonusfft(ntheta, self.nz_held, n)
            self._tomo_all.setobj(self.theta)
        # ptychography: one operator per angle chunk, its scans set once
        self._ptycho = []
        for k in range(self.ntheta_held // ptheta):
            op = ptychofft(ptheta, nz, n, ptheta, self.nscan, self.ndety, self.ndetx, self.nprb)
            op.setobj(self.scan[:, k * ptheta:(k + 1) * ptheta].contiguous(), self.prb)
            self._ptycho.append(op)
        self.cl_ptycho = self._ptycho[0]
        if ptheta != self.ntheta_held:
            self._ptycho_all = ptychofft(self.ntheta_held, nz, n, self.ntheta_held, self.nscan, self.ndety,
                                         self.ndetx, self.nprb)
            self._ptycho_all.setobj(self.scan, self.prb)
        else:
            self._ptycho_all = self.cl_ptycho
        # sub-pixel scan model (not in the reference): subpixel = quantisation
        # of the scan offsets in 1/pixel; 0 keeps the reference's rounded scans
        self.subpixel = int(subpixel)
        if self.subpixel:
            for op in {id(o): o for o in self._ptycho + [self._ptycho_all]}.values():
                op.set_subpixel(self.subpixel)
        # normalization coefficients, solver.py:43-46 (float32 like the reference)
        self._red_local = K.Reducer(dev)   # for quantities every process holds whole (the probe)
        self.red = self._reducer(K.Reducer(dev))
        amax = self.red.maxabs(self.prb)
        self.coeftomo = float(np.float32(1 / np.float32(np.sqrt(ntheta * n / 2))))
        self.coefptycho = float(np.float32(1 / np.float32(amax)))
        self.coefdata = float(np.float32(1 / (self.ndetx * self.ndety * np.float32(amax) ** 2)))

    # ---- helpers ----------------------------------------------------------
    # Hooks for ShardedSolver: global reductions, angle <-> slice re-sharding.
    # One process holds everything, so they are identities here.
    def _reducer(self, red):
        return red

    def _sum_probe(self, g):
        """Sum of per-process probe gradients (one process: itself)."""
        return g

    def _theta_to_z(self, x):
        """[angles held, nz, n] -> [ntheta, slices held, n]."""
        return x

    def _z_to_theta(self, x):
        """[ntheta, slices held, n] -> [angles held, nz, n]."""
        return x

    def _empty(self, shape, dtype=torch.complex64):
        return torch.empty(shape, dtype=dtype, device=self.device)

    def _ids(self, k):
        return slice(k * self.ptheta, (k + 1) * self.ptheta)

    # ---- maps, solver.py:48-64 --------------------------------------------
    def mlog(self, psi):
        return K.logmap(torch.empty_like(psi), psi, 1.0)

    def wavenumber(self):
        return 2 * np.pi / (2 * np.pi * PLANCK_CONSTANT * SPEED_OF_LIGHT / self.energy)

    def exptomo(self, psi):
        return K.expmap(torch.empty_like(psi), psi, self.voxelsize * self.wavenumber() / self.coeftomo)

    def logtomo(self, psi):
        c = -1j / self.wavenumber() / self.voxelsize * self.coeftomo
        return K.logmap(torch.empty_like(psi), psi, c)

    # ---- tomography, solver.py:67-97 --------------------------------------
    def fwd_tomo(self, u):
        res = self._empty([self.ntheta, self.pnz, self.n])
        self.cl_tomo.fwd(res, u, scale=self.coeftomo)
        return res

    def adj_tomo(self, data):
        res = self._empty([self.pnz, self.n, self.n])
        self.cl_tomo.adj(res, data, scale=self.coeftomo)
        return res

    def fwd_tomo_batch(self, u):
        res = self._empty([self.ntheta, self.nz_held, self.n])
        self._tomo_all.fwd(res, u, scale=self.coeftomo)
        return res

    def adj_tomo_batch(self, data):
        res = self._empty([self.nz_held, self.n, self.n])
        self._tomo_all.adj(res, data, scale=self.coeftomo)
        return res

    # ---- ptychography, solver.py:100-125 ----------------------------------
    def fwd_ptycho(self, psi):
        """FQ psi on the current angle chunk (self.cl_ptycho)."""
        res = self._empty([self.ptheta, self.nscan, self.ndety, self.ndetx])
        self.cl_ptycho.fwd(res, psi, scale=self.coefptycho)
        return res

    def fwd_ptycho_batch(self, psi):
        """|FQ psi|^2 / coefdata for all angles (a device float32 tensor)."""
        frames = self._empty([self.ntheta_held, self.nscan, self.ndety, self.ndetx])
        self._ptycho_all.fwd(frames, psi, scale=self.coefptycho)
        data = self._empty(frames.shape, torch.float32)
        return K.abs2(data, frames, 1.0 / self.coefdata)

    def adj_ptycho(self, data):
        res = self._empty([self.ptheta, self.nz, self.n])
        self.cl_ptycho.adj(res, data, scale=self.coefptycho)
        return res

    # ---- TV, solver.py:128-146 --------------------------------------------
    def fwd_reg(self, u):
        return K.reg_fwd(self._empty([3, *u.shape]), u, np.float32(2 / np.sqrt(3)))

    def adj_reg(self, gr):
        return K.reg_adj(self._empty(gr.shape[1:]), gr, np.float32(-2 / np.sqrt(3)))

    # ---- linearisation, solver.py:149-168 ---------------------------------
    def takexi(self, psi, phi, lamd, mu, rho, tau):
        r = self.prb.shape[0] // 2
        ncols = psi.shape[2]
        cnt = self.ntheta * self.nz * r   # elements in each column band over all angles
        m1 = self.red.angle_band_sum(psi, r, 2 * r) / cnt
        m2 = self.red.angle_band_sum(psi, ncols - 2 * r, ncols - r) / cnt
        pshift = (m1 + m2) / 2
        e = complex(math.cos(-pshift), math.sin(-pshift))
        t = K.lincomb(torch.empty_like(psi), [(e, psi), (-e / rho, lamd)])
        tmax = self.red.maxabs(t)
        Kt, xi0 = torch.empty_like(psi), torch.empty_like(psi)
        K.takexi(Kt, xi0, t, tmax, self.coeftomo / (self.voxelsize * self.wavenumber()))
        xi1 = K.lincomb(torch.empty_like(phi), [(1.0, phi), (-1.0 / tau, mu)])
        return xi0, xi1, Kt, pshift

    # ---- line search, solver.py:171-177 -----------------------------------
    def line_search(self, minf, gamma, u, fu, d, fd):
        """Generic backtracking with a user functional, as in the reference."""
        while minf(u, fu) - minf(u + gamma * d, fu + gamma * fd) < 0 and gamma > 1e-12:
            gamma *= 0.5
        if gamma <= 1e-12:
            gamma = 0
        return gamma

    trace = None   # list: records (kind, gamma) of every CG line search when set
    # ptycho CG: the line search also advances the frames by its first step, and
    # the next iteration reuses them instead of a new forward when that step is taken
    advance_frames = True

    @staticmethod
    def _halve_until(gamma, decrease):
        """Same decisions as solver.py:172-177 given decrease(g) = minf(0) - minf(g)."""
        while decrease(gamma) < 0 and gamma > 1e-12:
            gamma *= 0.5
        return 0 if gamma <= 1e-12 else gamma

    # ---- CG tomography, solver.py:180-203 ---------------------------------
    precond = None   # a learned.FourierPreconditioner: cg_tomo then runs the preconditioned CG

    def set_preconditioner(self, pre):
        """Use the preconditioned CG (``pcg_tomo``) with ``pre`` in cg_tomo and
        admm from now on; None restores the reference's CG."""
        self.precond = pre

    def cg_tomo(self, xi0, xi1, Kt, init, rho, tau, titer):
        return self._cg_tomo(xi0, xi1, Kt, init, rho, tau, titer)[0]

    def pcg_tomo(self, xi0, xi1, Kt, init, rho, tau, titer, precond=None, tol=0.0, history=None):
        """Preconditioned CG on the tomography subproblem of cg_tomo
        (solver.py:180-203), rho ||K R u - xi0||^2 + tau ||J u - xi1||^2, a
        quadratic in u: the exact gradient rho R^T conj(K) (K R u - xi0) +
        tau J^T (J u - xi1) (R^T: radonusfft.adj_exact; J^T: adj_reg on the
        range of J), z = P g, Fletcher-Reeves directions and the exact step
        along each.  P is ``precond`` (SPD, so the minimiser is that of the
        subproblem); None is the identity: plain CG with exact steps, the
        fallback and the judge of the preconditioner's error.  Stops after
        titer iterations or once ||g|| <= tol ||g_0||; ``history`` receives
        ||g_k|| / ||g_0||.  Returns (u, R u)."""
        return self._pcg_tomo(xi0, xi1, Kt, init, rho, tau, titer, precond, tol, history)

    def _pcg_tomo(self, xi0, xi1, Kt, init, rho, tau, titer, precond, tol=0.0, history=None):
        red = self.red
        u = init.clone()
        Ru = self.fwd_tomo_batch(u)
        a = K.cmul(torch.empty_like(xi0), Kt, Ru)
        K.lincomb(a, [(1.0, a), (-1.0, xi0)])
        xi1m = K.reg_mask(xi1.clone())       # entries of xi1 outside the range of J are constant in u
        b = self.fwd_reg(u)
        K.lincomb(b, [(1.0, b), (-1.0, xi1m)])
        rk = rho * red.norm2(Kt) / Kt.numel() if precond is not None else 0.0
        ka = torch.empty_like(a)
        g = torch.empty_like(u)
        z = torch.empty_like(u) if precond is not None else g
        d = None
        gz0 = g0n = None
        for _ in range(titer):
            K.cmul(ka, Kt, a, mode=2)
            self._tomo_all.adj_exact(g, ka, scale=self.coeftomo)
            K.lincomb(g, [(rho, g), (tau, self.adj_reg(b))])
            if precond is not None:
                precond.apply(z, g, rk, tau)
                gz = red.dot(g, z).real
                gn = red.norm2(g) if (tol > 0 or history is not None) else None
            else:
                gz = red.norm2(g)
                gn = gz
            if gn is not None:
                g0n = gn if g0n is None else g0n
                if history is not None:
                    history.append(math.sqrt(gn / g0n) if g0n > 0 else 0.0)
                if tol > 0 and gn <= tol * tol * g0n:
                    break
            steepest = d is None or gz0 is None or gz0 <= 0
            if steepest:
                d = K.lincomb(torch.empty_like(z), [(-1.0, z)])
            else:
                K.lincomb(d, [(-1.0, z), (gz / gz0, d)])
            gz0 = gz
            Rd = self.fwd_tomo_batch(d)
            fd = K.cmul(torch.empty_like(xi0), Kt, Rd)
            gd = self.fwd_reg(d)
            _, a_fd, fd2 = red.quad3(a, fd)
            _, b_gd, gd2 = red.quad3(b, gd)
            c1 = rho * a_fd + tau * b_gd
            c2 = rho * fd2 + tau * gd2
            if not (c1 < 0 and c2 > 0):
                if not steepest:
                    gz0 = None          # a conjugate direction that does not descend: retry along -z
                    continue
                break                   # -z does not descend either: converged to rounding
            gamma = -c1 / c2
            if self.trace is not None:
                self.trace.append(("pcg", gamma))
            K.lincomb(u, [(1.0, u), (gamma, d)])
            K.lincomb(Ru, [(1.0, Ru), (gamma, Rd)])
            K.lincomb(a, [(1.0, a), (gamma, fd)])
            K.lincomb(b, [(1.0, b), (gamma, gd)])
        return u, Ru

    def _cg_tomo(self, xi0, xi1, Kt, init, rho, tau, titer):
        """cg_tomo, also returning R u of the final iterate (for h in admm)."""
        if self.precond is not None:
            return self._pcg_tomo(xi0, xi1, Kt, init, rho, tau, titer, self.precond)
        red = self.red
        u = init.clone()
        gamma = 2
        grad0 = d = None
        # R u, a = K R u - xi0 and b = J u - xi1: evaluated for the first
        # iterate, then advanced with the step (u + g d gives R u + g R d,
        # a + g K R d and b + g J d, all formed already for the line search)
        Ru = self.fwd_tomo_batch(u)
        a = K.cmul(torch.empty_like(xi0), Kt, Ru)
        K.lincomb(a, [(1.0, a), (-1.0, xi0)])
        b = self.fwd_reg(u)
        K.lincomb(b, [(1.0, b), (-1.0, xi1)])
        for i in range(titer):
            ga = self.adj_tomo_batch(K.cmul(torch.empty_like(a), Kt, a, mode=2))
            grad = K.lincomb(ga, [(rho, ga), (tau, self.adj_reg(b))])
            if i == 0:
                d = K.lincomb(torch.empty_like(grad), [(-1.0, grad)])
            else:
                dg, dg0, g2 = red.many([("dot", d, grad), ("dot", d, grad0), ("norm2", grad)])
                den = dg - dg0
                beta = g2 / den if den != 0 else 0.0
                K.lincomb(d, [(-1.0, grad), (beta, d)])
            grad0 = grad
            Rd = self.fwd_tomo_batch(d)
            fd = K.cmul(torch.empty_like(xi0), Kt, Rd)
            gd = self.fwd_reg(d)
            (_, a_fd, fd2), (_, b_gd, gd2) = red.many([("quad3", a, fd), ("quad3", b, gd)])
            c1 = rho * a_fd + tau * b_gd
            c2 = rho * fd2 + tau * gd2
            gamma = self._halve_until(gamma, lambda g: -(2 * g * c1 + g * g * c2))
            if self.trace is not None:
                self.trace.append(("tomo", gamma))
            K.lincomb(u, [(1.0, u), (gamma, d)])
            if gamma == 0:
                break   # gamma only halves: u can no longer change in this call
            K.lincomb(Ru, [(1.0, Ru), (gamma, Rd)])
            if i + 1 < titer:
                K.lincomb(a, [(1.0, a), (gamma, fd)])
                K.lincomb(b, [(1.0, b), (gamma, gd)])
        return u, Ru

    # ---- CG ptychography, solver.py:206-254 -------------------------------
    def cg_ptycho(self, data, init, h, lamd, rho, piter, model, dscale=1.0):
        """CG on the current angle chunk; data are raw counts times dscale."""
        red = self.red
        mdl = _MODELS[model]
        psi = init.clone()
        gamma = 2
        grad0 = d = None
        w = torch.empty_like(psi)
        fpsi = None
        for i in range(piter):
            if fpsi is None:
                fpsi = self.fwd_ptycho(psi)
            grad = self._empty([self.ptheta, self.nz, self.n])   # Q*F*(residual), residual formed on load
            self.cl_ptycho.adj_resid(grad, fpsi, data, dscale, mdl, scale=self.coefptycho)
            K.lincomb(w, [(1.0, h), (-1.0, psi), (1.0 / rho, lamd)])     # h - psi + lamd/rho
            K.lincomb(grad, [(1.0, grad), (-rho, w)])
            if i == 0:
                d = K.lincomb(torch.empty_like(grad), [(-1.0, grad)])
            else:
                dg, dg0, g2 = red.many([("dot", d, grad), ("dot", d, grad0), ("norm2", grad)])
                den = dg - dg0
                beta = g2 / den if den != 0 else 0.0
                K.lincomb(d, [(-1.0, grad), (beta, d)])
            grad0 = grad
            fd = self.fwd_ptycho(d)
            _, w_d, d2 = red.quad3(w, d)
            # minf(psi) - minf(psi + g d) = data-term decrease (per element, FP64)
            #   + rho (2 g Re<w, d> - g^2 ||d||^2)  for the penalty rho ||w - g d||^2
            npass = 0
            advanced = None   # the step by which the first pass advanced fpsi
            while True:
                # gamma usually survives: try (g, g/2) first, then 8, then 16 halvings per pass
                J = (2, 8, 16)[min(npass, 2)]
                gs = [gamma * 0.5 ** j for j in range(J)]
                adv = self.advance_frames and npass == 0 and i + 1 < piter
                if advanced is not None:   # a later pass needs the frames of psi itself
                    fpsi = self.fwd_ptycho(psi)
                    advanced = None
                npass += 1
                vals = red.ls_frames(fpsi, fd, data, dscale, mdl, gs, advance=adv)
                if adv:
                    advanced = gs[0]
                chosen = None
                for g, dec_data in zip(gs, vals):
                    dec = dec_data + rho * (2 * g * w_d - g * g * d2)
                    if not (dec < 0 and g > 1e-12):
                        chosen = g
                        break
                if chosen is not None:
                    gamma = 0 if chosen <= 1e-12 else chosen
                    break
                gamma = gs[-1] * 0.5
            if self.trace is not None:
                self.trace.append(("ptycho", gamma))
            K.lincomb(psi, [(1.0, psi), (gamma, d)])
            # fpsi + gamma fd = F Q (psi + gamma d): kept when the step taken is
            # the one the line search advanced the frames by
            if advanced is None or gamma != advanced:
                fpsi = None
            del fd
            if gamma == 0:
                break   # gamma only halves: psi can no longer change in this call
        if red.maxangle(psi) > 3.14:
            print("possible phase wrap, max computed angle", red.maxangle(psi))
        return psi

    # ---- probe retrieval (no counterpart in the reference) -----------------
    def set_probe(self, prb):
        """Use the probe prb [Nprb, Nprb] in every ptycho operator from now on
        (coefptycho and coefdata keep the values of the first probe)."""
        self.prb = _dev_tensor(prb, torch.complex64, self.device)
        for k, op in enumerate(self._ptycho):
            op.setobj(self.scan[:, k * self.ptheta:(k + 1) * self.ptheta].contiguous(), self.prb)
        if self._ptycho_all is not self.cl_ptycho:
            self._ptycho_all.setobj(self.scan, self.prb)

    def cg_probe(self, data, psi, prb, piter, model):
        """Dai-Yuan CG on the probe with psi fixed: minimises the ptycho data
        term of solver.py:208-214 over the probe, with the line search of
        cg_ptycho.  data [angles held, Nscan, det, det] raw counts, psi
        [angles held, Nz, N]; returns the new probe [Nprb, Nprb]."""
        data = self._as_data(data)
        red, loc = self.red, self._red_local
        mdl = _MODELS[model]
        p = _dev_tensor(prb, torch.complex64, self.device).clone()
        chunks = [(self._ids(k), op) for k, op in enumerate(self._ptycho)]
        frames = [self.ptheta, self.nscan, self.ndety, self.ndetx]

        def fwd(q, ids, op):
            out = self._empty(frames)
            op.fwd_probe(out, psi[ids].contiguous(), q, scale=self.coefptycho)
            return out

        gamma = 2
        grad0 = d = None
        for i in range(piter):
            fp = [fwd(p, ids, op) for ids, op in chunks]
            grad = torch.zeros_like(p)
            gk = torch.empty_like(p)
            for (ids, op), f in zip(chunks, fp):
                op.adj_probe_resid(gk, psi[ids].contiguous(), f, data[ids], self.coefdata, mdl, scale=self.coefptycho)
                K.lincomb(grad, [(1.0, grad), (1.0, gk)])
            grad = self._sum_probe(grad)
            if i == 0:
                d = K.lincomb(torch.empty_like(grad), [(-1.0, grad)])
            else:
                den = loc.dot(d, grad) - loc.dot(d, grad0)
                beta = loc.norm2(grad) / den if den != 0 else 0.0
                K.lincomb(d, [(-1.0, grad), (beta, d)])
            grad0 = grad
            fd = [fwd(d, ids, op) for ids, op in chunks]
            npass = 0
            while True:
                J = (2, 8, 16)[min(npass, 2)]
                npass += 1
                gs = [gamma * 0.5 ** j for j in range(J)]
                vals = np.zeros(J)
                for (ids, _), f, fdk in zip(chunks, fp, fd):
                    vals += np.asarray(red.ls_frames(f, fdk, data[ids], self.coefdata, mdl, gs))
                chosen = next((g for g, dec in zip(gs, vals) if not (dec < 0 and g > 1e-12)), None)
                if chosen is not None:
                    gamma = 0 if chosen <= 1e-12 else chosen
                    break
                gamma = gs[-1] * 0.5
            if self.trace is not None:
                self.trace.append(("probe", gamma))
            K.lincomb(p, [(1.0, p), (gamma, d)])
            del fp, fd
            if gamma == 0:
                break
        return p

    def cg_ptycho_batch(self, data, init, h, lamd, rho, piter, model):
        data = self._as_data(data)
        if self.ptheta == self.ntheta_held:
            self.cl_ptycho = self._ptycho[0]
            return self.cg_ptycho(data, init, h, lamd, rho, piter, model, dscale=self.coefdata)
        psi = init.clone()
        for k in range(self.ntheta_held // self.ptheta):
            ids = self._ids(k)
            self.cl_ptycho = self._ptycho[k]
            psi[ids] = self.cg_ptycho(data[ids], psi[ids].contiguous(), h[ids].contiguous(),
                                      lamd[ids].contiguous(), rho, piter, model, dscale=self.coefdata)
        return psi

    def _as_data(self, data):
        if isinstance(data, torch.Tensor) and data.is_cuda and data.dtype == torch.float32 and data.is_contiguous():
            return data
        return _dev_tensor(data, torch.float32, self.device)

    # ---- regulariser, penalties, monitor, solver.py:257-305 ---------------
    def solve_reg(self, u, mu, tau, alpha):
        z = self._empty([3, *u.shape])
        return K.solve_reg(z, u, mu, np.float32(2 / np.sqrt(3)), 1.0 / tau, alpha / tau)

    def update_penalty(self, psi, h, h0, phi, e, e0, rho, tau):
        r = self.red.norm2_diff(psi, h)
        s = rho * rho * self.red.norm2_diff(h, h0)
        if r > 10 * s:
            rho *= 2
        elif s > 10 * r:
            rho *= 0.5
        r = self.red.norm2_diff(phi, e)
        s = tau * tau * self.red.norm2_diff(e, e0)
        if r > 10 * s:
            tau *= 2
        elif s > 10 * r:
            tau *= 0.5
        return rho, tau

    def take_lagr(self, psi, phi, data, h, e, lamd, mu, alpha, rho, tau, model):
        data = self._as_data(data)
        red = self.red
        lagr = np.zeros(7)
        for k in range(self.ntheta_held // self.ptheta):
            ids = self._ids(k)
            self.cl_ptycho = self._ptycho[k]
            fpsi = self.fwd_ptycho(psi[ids].contiguous())
            lagr[0] += red.lagr_frames(fpsi, data[ids], self.coefdata, _MODELS[model])
        lagr[1] = alpha * red.tv(phi)
        lagr[2] = 2 * (red.dot(lamd, h) - red.dot(lamd, psi)).real
        lagr[3] = rho * red.norm2_diff(h, psi)
        lagr[4] = 2 * (red.dot(mu, e) - red.dot(mu, phi)).real
        lagr[5] = tau * red.norm2_diff(e, phi)
        lagr[6] = np.sum(lagr[0:5])  # the reference sums terms 0..4 (solver.py:304)
        return lagr

    # ---- checkpoint / resume (no counterpart in the reference) ------------
    _STATE = ("u", "psi", "h", "e", "phi", "lamd", "mu")

    def _checkpoint_file(self, path):
        return str(path)

    def save_state(self, path, m, rho, tau, **arrays):
        """Write the ADMM state after iteration m (atomically: a temporary file, then rename)."""
        path = self._checkpoint_file(path)
        state = {"m": int(m), "rho": float(rho), "tau": float(tau),
                 "held": (self.theta_range, self.z_range, self.ntheta, self.nz, self.n)}
        state.update({k: arrays[k].detach().cpu() for k in self._STATE})
        state["prb"] = self.prb.detach().cpu()
        tmp = path + ".tmp"
        torch.save(state, tmp)
        os.replace(tmp, path)

    def load_state(self, path):
        """The state written by save_state, arrays on this Solver's device."""
        state = torch.load(self._checkpoint_file(path), map_location="cpu", weights_only=True)
        if tuple(map(_as_tuple, state["held"])) != tuple(map(_as_tuple, (
                self.theta_range, self.z_range, self.ntheta, self.nz, self.n))):
            raise ValueError("checkpoint %s was written for another problem or shard" % path)
        for k in self._STATE:
            state[k] = state[k].to(self.device)
        return state

    # ---- ADMM, solver.py:308-336 ------------------------------------------
    def admm_step(self, m, st, rho, tau, data, alpha, piter, titer, model, probe_iter=0):
        """One ADMM iteration, the loop body of solver.py:311-329, from the state
        st (a dict of u, psi, h, e, phi, lamd, mu; device tensors, data as
        _as_data gives it); returns (new state, rho, tau).  With probe_iter > 0
        the probe is refined after the ptycho subproblem (no counterpart in
        the reference)."""
        u, psi, h, e, phi, lamd, mu = (st[k] for k in self._STATE)
        h0, e0 = h, e
        psi = self.cg_ptycho_batch(data, psi, h, lamd, rho, piter + (m < 2) * 32, model)
        if probe_iter > 0:
            self.set_probe(self.cg_probe(data, psi, self.prb, probe_iter, model))
        xi0, xi1, Kt, pshift = self.takexi(psi, phi, lamd, mu, rho, tau)
        u, Ru = self._cg_tomo(self._theta_to_z(xi0), xi1, self._theta_to_z(Kt), u, rho, tau, titer)
        phi = self.solve_reg(u, mu, tau, alpha)
        h = K.expmap(torch.empty_like(psi), self._z_to_theta(Ru),
                     self.voxelsize * self.wavenumber() / self.coeftomo, pshift)
        e = self.fwd_reg(u)
        lamd = K.lincomb(torch.empty_like(lamd), [(1.0, lamd), (rho, h), (-rho, psi)])
        mu = K.lincomb(torch.empty_like(mu), [(1.0, mu), (tau, e), (-tau, phi)])
        rho, tau = self.update_penalty(psi, h, h0, phi, e, e0, rho, tau)
        return dict(u=u, psi=psi, h=h, e=e, phi=phi, lamd=lamd, mu=mu), rho, tau

    def admm(self, data, h, e, psi, phi, lamd, mu, u, alpha, piter, titer, niter, model, verbose=True,
             history=None, checkpoint=None, checkpoint_every=1, resume=False, probe_iter=0):
        """ADMM as solver.py:308-336.  With ``checkpoint`` (a file path) the state
        is saved every ``checkpoint_every`` iterations and after the last one;
        with ``resume`` a run continues from that file (iteration m + 1 of the
        same schedule) instead of from the arrays passed in.  With ``probe_iter``
        > 0 the probe is retrieved too: after each ptycho subproblem, that many
        cg_probe iterations update it (``self.prb`` holds the result)."""
        data = self._as_data(data)
        rho, tau = 0.5, 0.5
        m0 = 0
        if resume and checkpoint is not None and os.path.exists(self._checkpoint_file(checkpoint)):
            st = self.load_state(checkpoint)
            m0, rho, tau = st["m"] + 1, st["rho"], st["tau"]
            u, psi, h, e, phi, lamd, mu = (st[k] for k in self._STATE)
            if "prb" in st and not torch.equal(st["prb"], self.prb.cpu()):
                self.set_probe(st["prb"])
        st = dict(u=u, psi=psi, h=h, e=e, phi=phi, lamd=lamd, mu=mu)
        for m in range(m0, niter):
            st, rho, tau = self.admm_step(m, st, rho, tau, data, alpha, piter, titer, model, probe_iter)
            u, psi, h, e, phi, lamd, mu = (st[k] for k in self._STATE)
            if history is not None:
                history.append(dict(m=m, rho=rho, tau=tau))
            if np.mod(m, 10) == 0 and (verbose or history is not None):
                lagr = self.take_lagr(psi, phi, data, h, e, lamd, mu, alpha, rho, tau, model)
                if history is not None:
                    history[-1]["lagr"] = lagr
                if verbose:
                    print("%d/%d) rho=%.2e, tau=%.2e, Lagrangian terms:  %.2e %.2e %.2e %.2e %.2e %.2e, Sum: %.2e" %
                          (m, niter, rho, tau, *lagr))
            if checkpoint is not None and ((m + 1) % checkpoint_every == 0 or m == niter - 1):
                self.save_state(checkpoint, m, rho, tau, u=u, psi=psi, h=h, e=e, phi=phi, lamd=lamd, mu=mu)
        return u, psi
