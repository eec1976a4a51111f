"""One ADMM iteration captured as a CUDA graph (no counterpart in the reference).

The reference's Solver (src/ptychotomo/solver.py:171-336) takes every step
length, Dai-Yuan beta and penalty decision on the host, so every CG
iteration waits for the GPU several times.  :class:`GraphedADMM` runs the
same iteration (solver.py:311-329) with every scalar in a device array (the
"arena"): reductions write into its slots, one-thread kernels
(pt_scalar_*) apply the reference's rules there, and linear combinations read
their coefficients from it.  The launch sequence is then fixed, so iteration
m >= 2 (piter ptycho and titer tomography CG iterations) is captured once
with torch.cuda.graph and replayed; the first two iterations (piter + 32
ptycho CG iterations, solver.py:315) run the same sequence eagerly.

Differences from Solver.admm, all by construction of a fixed sequence:
* the ptycho line search runs the host Solver's passes of 2, 8 and 16 step
  lengths (a pass skips itself on the device once an earlier one accepted a
  step); if none of the 26 candidates passes, that iteration steps by 0 and
  the next starts from gamma 2^-26 of the first candidate (the host Solver
  would keep halving along the same direction);
* F Q psi advances by linearity (F Q (psi + g d) = F Q psi + g F Q d): by
  the first candidate step inside the first line-search pass, as the host's,
  and by a correction pass (which skips itself when the first candidate was
  taken) otherwise, where the host computes a new forward; it is recomputed
  once per CG call;
* a CG whose step is 0 keeps iterating with zero steps (the host Solver
  breaks out of the loop; the iterate is the same).
With ``precond`` the tomography subproblem runs the preconditioned CG of
Solver.pcg_tomo instead.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import kernels as K
from ._lib import check, current_stream, lib
from .solver import _MODELS


def _p(t):
    return t.data_ptr()


class _Arena:
    """Named slots of one device float64 array."""

    def __init__(self, device, size=512):
        self.buf = torch.zeros(size, dtype=torch.float64, device=device)
        self.base = self.buf.data_ptr()
        self.used = 0
        self.names = {}

    def __call__(self, name, count=1):
        if name not in self.names:
            if self.used + count > self.buf.numel():
                raise RuntimeError("scalar arena full")
            self.names[name] = (self.used, count)
            self.used += count
        return self.base + 8 * self.names[name][0]

    def view(self, name):
        o, c = self.names[name]
        return self.buf[o:o + c]


class GraphedADMM:
    """ADMM iterations of ``slv`` (a Solver holding all angles and slices)
    with device-resident scalars.

    ``data``: the counts (device float32, as Solver.admm takes them);
    alpha, piter, titer, model: as Solver.admm.  ``precond``: a
    FourierPreconditioner for the tomography subproblem (None: the
    reference's CG)."""

    def __init__(self, slv, data, alpha, piter, titer, model, precond=None):
        if slv.ptheta != slv.ntheta_held or slv.nz_held != slv.nz:
            raise ValueError("GraphedADMM needs a Solver with ptheta = ntheta and pnz = nz")
        self.slv, self.alpha, self.piter, self.titer = slv, float(alpha), int(piter), int(titer)
        self.model = _MODELS[model]
        self.precond = precond
        self.data = slv._as_data(data)
        dev = slv.device
        self.dev = dev
        nt, nz, n = slv.ntheta_held, slv.nz, slv.n
        c = dict(dtype=torch.complex64, device=dev)
        frames = (nt, slv.nscan, slv.ndety, slv.ndetx)
        self.A = _Arena(dev)
        # state (fixed addresses: the graph reads and writes them in place)
        self.u = torch.zeros((nz, n, n), **c)
        self.psi = torch.zeros((nt, nz, n), **c)
        self.h, self.h0, self.lamd = (torch.zeros((nt, nz, n), **c) for _ in range(3))
        self.e, self.e0, self.phi, self.mu = (torch.zeros((3, nz, n, n), **c) for _ in range(4))
        # work
        self.fpsi = torch.empty(frames, **c)
        self.fd = torch.empty(frames, **c)
        self.pg = [torch.empty((nt, nz, n), **c) for _ in range(2)]     # ptycho gradients (this, previous)
        self.pd = torch.empty((nt, nz, n), **c)
        self.pw = torch.empty((nt, nz, n), **c)
        self.t = torch.empty((nt, nz, n), **c)
        self.Kt = torch.empty((nt, nz, n), **c)
        self.xi0 = torch.empty((nt, nz, n), **c)
        self.xi1 = torch.empty((3, nz, n, n), **c)
        self.Ru = torch.empty((nt, nz, n), **c)
        self.ta = torch.empty((nt, nz, n), **c)
        self.tka = torch.empty((nt, nz, n), **c)
        self.tRd = torch.empty((nt, nz, n), **c)
        self.tfd = torch.empty((nt, nz, n), **c)
        self.tb = torch.empty((3, nz, n, n), **c)
        self.tgd = torch.empty((3, nz, n, n), **c)
        self.tjb = torch.empty((nz, n, n), **c)
        self.tg = [torch.empty((nz, n, n), **c) for _ in range(2)]
        self.tz = torch.empty((nz, n, n), **c) if precond is not None else None
        self.td = torch.empty((nz, n, n), **c)
        self.work = torch.empty(lib().pt_reduce_workspace_bytes() // 8, dtype=torch.float64, device=dev)
        self.graph = None
        self.trace = None   # a list: (kind, step) of every CG step of eager iterations (reads back each one)

    # ---- state in / out ---------------------------------------------------
    def load(self, st, rho, tau):
        """Copy a Solver.admm_step state (dict) and the penalties in."""
        for k in ("u", "psi", "h", "e", "phi", "lamd", "mu"):
            getattr(self, k).copy_(st[k])
        self.A("rt", 2)
        self.A.view("rt").copy_(torch.tensor([rho, tau], dtype=torch.float64))

    def state(self):
        """(state dict of views, rho, tau); reading rho and tau synchronises."""
        rho, tau = self.A.view("rt").tolist()
        return {k: getattr(self, k) for k in ("u", "psi", "h", "e", "phi", "lamd", "mu")}, rho, tau

    # ---- launch helpers ---------------------------------------------------
    def _st(self):
        return current_stream()

    def _red(self, op, slot, a, b=None, n=None, c0=0, c1=0, ncol=1):
        n = a.numel() if n is None else n
        check(lib().pt_reduce_c64(op, _p(a), _p(b) if b is not None else None, n, c0, c1, ncol, _p(self.work),
                                  slot, self._st()), "reduce")

    def _lin(self, out, xs, coef, skip_zero=None):
        arr = (ctypes.c_void_p * 4)(*[_p(x) for x in xs] + [None] * (4 - len(xs)))
        check(lib().pt_lincomb_dev_c64(_p(out), out.numel(), len(xs), arr, coef, skip_zero, self._st()),
              "lincomb_dev")

    def _coef(self, name, a0, s0=None, a1=0.0, s1=None):
        """coef slot = (a0 * [s0], 0, a1 * [s1], 0) (s0, s1: slot addresses or None)."""
        slot = self.A(name, 4)
        check(lib().pt_scalar_coef2(s0, float(a0), s1, float(a1), slot, self._st()), "coef2")
        return slot

    def _coef_const(self, name, vals):
        """A slot with one or two constant real coefficients, written by a
        kernel (inside a capture, a host write would not be replayed)."""
        slot = self.A(name, 4)
        v1 = float(vals[1]) if len(vals) > 1 else 0.0
        check(lib().pt_scalar_coef2(None, float(vals[0]), None, v1, slot, self._st()), "coef2")
        return slot

    # ---- the iteration ----------------------------------------------------
    def _ptycho_cg(self, piter):
        slv, A = self.slv, self.A
        rt = A("rt", 2)
        op = slv._ptycho_all
        dscale = slv.coefdata
        check(lib().pt_scalar_coef2(None, 0.0, None, 2.0, A("pls", 4), self._st()), "coef2")   # gamma = 2
        op.fwd(self.fpsi, self.psi, scale=slv.coefptycho)
        # w = h - psi + lamd / rho: coefficients (1, -1, 1/rho)
        w = A("wcoef", 6)
        check(lib().pt_scalar_coef2(None, 1.0, None, -1.0, w, self._st()), "coef2")
        check(lib().pt_scalar_inv(rt, 1.0, w + 32, self._st()), "scalar_inv")
        for i in range(piter):
            g, g0 = self.pg[i % 2], self.pg[(i + 1) % 2]
            op.adj_resid(g, self.fpsi, self.data, dscale, self.model, scale=slv.coefptycho)
            self._lin(self.pw, [self.h, self.psi, self.lamd], w)
            self._lin(g, [g, self.pw], self._coef("gr", 1.0, None, -1.0, rt))
            if i == 0:
                self._lin(self.pd, [g], self._coef_const("m1", [-1.0]))
            else:
                self._red(1, A("dg", 2), self.pd, g)
                self._red(1, A("dg0", 2), self.pd, g0)
                self._red(0, A("g2"), g)
                check(lib().pt_scalar_dy_beta(A("g2"), A("dg", 2), A("dg0", 2), 0, A("pbeta", 4), self._st()),
                      "dy_beta")
                self._lin(self.pd, [g, self.pd], A("pbeta", 4))
            op.fwd(self.fd, self.pd, scale=slv.coefptycho)
            self._red(2, A("pq", 3), self.pw, self.pd)
            # the host's passes of 2, 8 and 16 step lengths; later passes skip
            # themselves on the device once one accepted a step
            state = A("pls", 3)
            check(lib().pt_scalar_ls_begin(state, self._st()), "ls_begin")
            for J in (2, 8, 16):
                check(lib().pt_scalar_ls_candidates(state, J, A("gams", 16), self._st()), "ls_candidates")
                if J == 2:   # the first pass also advances the frames by its first step (as the host's)
                    check(lib().pt_ls_frames_advance(_p(self.fpsi), _p(self.fd), _p(self.data), float(dscale),
                                                     self.fpsi.numel(), self.model, A("gams", 16), J,
                                                     _p(self.work), A("lsv", 16), self._st()), "ls_frames_advance")
                else:
                    check(lib().pt_ls_frames_dev(_p(self.fpsi), _p(self.fd), _p(self.data), float(dscale),
                                                 self.fpsi.numel(), self.model, A("gams", 16), J, _p(self.work),
                                                 A("lsv", 16), state, self._st()), "ls_frames_dev")
                check(lib().pt_scalar_ls_pass(A("lsv", 16), A("gams", 16), J, A("pq", 3), rt, state, self._st()),
                      "ls_pass")
                if J == 2:   # rejected: the later passes need the frames of psi itself
                    ua = A("punadv", 4)
                    check(lib().pt_scalar_ls_unadvance(state, ua, self._st()), "ls_unadvance")
                    self._lin(self.fpsi, [self.fpsi, self.fd], ua, skip_zero=ua + 16)
            check(lib().pt_scalar_ls_end(state, A("pstep", 4), A("pcorr", 4), self._st()), "ls_end")
            if self.trace is not None:
                self.trace.append(("ptycho", float(A.view("pstep")[2])))
            self._lin(self.psi, [self.psi, self.pd], A("pstep", 4))
            # frames of the new iterate: already there when the first candidate was taken
            corr = A("pcorr", 4)
            self._lin(self.fpsi, [self.fpsi, self.fd], corr, skip_zero=corr + 16)

    def _takexi(self):
        slv, A = self.slv, self.A
        rt = A("rt", 2)
        r = slv.prb.shape[0] // 2
        ncols = self.psi.shape[2]
        cnt = slv.ntheta * slv.nz * r
        self._red(4, A("band1"), self.psi, c0=r, c1=2 * r, ncol=ncols)
        self._red(4, A("band2"), self.psi, c0=ncols - 2 * r, c1=ncols - r, ncol=ncols)
        check(lib().pt_scalar_takexi(A("band1"), A("band2"), float(cnt), rt, A("pshift"), A("tcoef", 4),
                                     self._st()), "takexi scalars")
        self._lin(self.t, [self.psi, self.lamd], A("tcoef", 4))
        self._red(3, A("tmax"), self.t)
        cxi = slv.coeftomo / (slv.voxelsize * slv.wavenumber())
        check(lib().pt_takexi_dev_c64(_p(self.Kt), _p(self.xi0), _p(self.t), self.t.numel(), A("tmax"), float(cxi),
                                      self._st()), "takexi_dev")
        # xi1 = phi - mu / tau
        x1 = A("x1coef", 4)
        check(lib().pt_scalar_coef2(None, 1.0, None, 0.0, x1, self._st()), "coef2")
        check(lib().pt_scalar_inv(A("rt", 2) + 8, -1.0, x1 + 16, self._st()), "scalar_inv")
        self._lin(self.xi1, [self.phi, self.mu], x1)

    def _tomo_cg(self):
        slv, A = self.slv, self.A
        rt = A("rt", 2)
        tau_slot = rt + 8
        u, Ru, a, b = self.u, self.Ru, self.ta, self.tb
        slv._tomo_all.fwd(Ru, u, scale=slv.coeftomo)
        K.cmul(a, self.Kt, Ru)
        K.lincomb(a, [(1.0, a), (-1.0, self.xi0)])
        xi1 = self.xi1
        if self.precond is not None:
            K.reg_mask(xi1)
        slv_fwd_reg(b, u)
        K.lincomb(b, [(1.0, b), (-1.0, xi1)])
        pcg = self.precond is not None
        if pcg:
            self._red(0, A("k2"), self.Kt)
            check(lib().pt_scalar_pcg_rk(A("k2"), float(self.Kt.numel()), rt, A("rk_tau", 2), self._st()), "pcg_rk")
            check(lib().pt_scalar_coef2(None, 0.0, None, 0.0, A("restart", 4), self._st()), "coef2")
        else:
            check(lib().pt_scalar_coef2(None, 2.0, None, 0.0, A("tgam", 4), self._st()), "coef2")
        for i in range(self.titer):
            g, g0 = self.tg[i % 2], self.tg[(i + 1) % 2]
            K.cmul(self.tka, self.Kt, a, mode=2)
            if pcg:
                slv._tomo_all.adj_exact(g, self.tka, scale=slv.coeftomo)
            else:
                slv._tomo_all.adj(g, self.tka, scale=slv.coeftomo)
            K.reg_adj(self.tjb, b, np.float32(-2 / np.sqrt(3)))
            self._lin(g, [g, self.tjb], self._coef("tgr", 1.0, rt, 1.0, tau_slot))
            if pcg:
                z = self.tz
                check(lib().pt_precond_apply_dev(self.precond._h, _p(z), _p(g), A("rk_tau", 2), self._st()),
                      "precond apply_dev")
                self._red(1, A("gz", 2), g, z)
                check(lib().pt_scalar_pcg_beta(A("gz", 2), A("gz0"), A("restart", 4), int(i == 0), A("tbeta", 4),
                                               self._st()), "pcg_beta")
                self._lin(self.td, [z, self.td] if i > 0 else [z], A("tbeta", 4) if i > 0 else
                          self._coef_const("m1", [-1.0]))
            else:
                if i == 0:
                    self._lin(self.td, [g], self._coef_const("m1", [-1.0]))
                else:
                    self._red(1, A("tdg", 2), self.td, g)
                    self._red(1, A("tdg0", 2), self.td, g0)
                    self._red(0, A("tg2"), g)
                    check(lib().pt_scalar_dy_beta(A("tg2"), A("tdg", 2), A("tdg0", 2), 0, A("tbeta", 4), self._st()),
                          "dy_beta")
                    self._lin(self.td, [g, self.td], A("tbeta", 4))
            slv._tomo_all.fwd(self.tRd, self.td, scale=slv.coeftomo)
            K.cmul(self.tfd, self.Kt, self.tRd)
            slv_fwd_reg(self.tgd, self.td)
            self._red(2, A("q1", 3), a, self.tfd)
            self._red(2, A("q2", 3), b, self.tgd)
            if pcg:
                check(lib().pt_scalar_pcg_step(A("q1", 3), A("q2", 3), rt, A("restart", 4), A("tstep", 4),
                                               self._st()), "pcg_step")
            else:
                check(lib().pt_scalar_tomo_gamma(A("q1", 3), A("q2", 3), rt, A("tgam", 4), A("tstep", 4),
                                                 self._st()), "tomo_gamma")
            st = A("tstep", 4)
            if self.trace is not None:
                self.trace.append(("pcg" if pcg else "tomo", float(A.view("tstep")[2])))
            self._lin(u, [u, self.td], st)
            self._lin(Ru, [Ru, self.tRd], st)
            self._lin(a, [a, self.tfd], st)
            self._lin(b, [b, self.tgd], st)

    def _launch(self, piter):
        slv, A = self.slv, self.A
        rt = A("rt", 2)
        self.h0.copy_(self.h)
        self.e0.copy_(self.e)
        self._ptycho_cg(piter)
        self._takexi()
        self._tomo_cg()
        # phi = solve_reg(u, mu, tau, alpha)
        nz, n = slv.nz, slv.n
        check(lib().pt_solve_reg_dev_c64(_p(self.phi), _p(self.u), _p(self.mu), nz, n, n,
                                         float(np.float32(2 / np.sqrt(3))), rt, self.alpha, self._st()), "solve_reg")
        check(lib().pt_expmap_dev_c64(_p(self.h), _p(self.Ru), self.h.numel(),
                                      float(slv.voxelsize * slv.wavenumber() / slv.coeftomo), A("pshift"),
                                      self._st()), "expmap")
        slv_fwd_reg(self.e, self.u)
        check(lib().pt_scalar_multipliers(rt, A("lcoef", 6), A("mcoef", 6), self._st()), "multipliers")
        self._lin(self.lamd, [self.lamd, self.h, self.psi], A("lcoef", 6))
        self._lin(self.mu, [self.mu, self.e, self.phi], A("mcoef", 6))
        self._red(5, A("r1"), self.psi, self.h)
        self._red(5, A("s1"), self.h, self.h0)
        self._red(5, A("r2"), self.phi, self.e)
        self._red(5, A("s2"), self.e, self.e0)
        check(lib().pt_scalar_penalty(A("r1"), A("s1"), A("r2"), A("s2"), rt, self._st()), "penalty")

    # ---- public -----------------------------------------------------------
    def step(self, m):
        """Iteration m, eagerly (the same launches the graph holds)."""
        self._launch(self.piter + (m < 2) * 32)

    def capture(self):
        """Capture the steady iteration (piter ptycho CG iterations) once.
        The state buffers keep their contents: capture runs nothing."""
        torch.cuda.synchronize(self.dev)
        # a warm-up on a side stream initialises lazily created library state
        # (attributes, occupancy queries) outside the capture
        self.graph = torch.cuda.CUDAGraph()
        saved = {k: getattr(self, k).clone() for k in ("u", "psi", "h", "e", "phi", "lamd", "mu")}
        rt = self.A.view("rt").clone()
        trace, self.trace = self.trace, None
        s = torch.cuda.Stream(self.dev)
        s.wait_stream(torch.cuda.current_stream(self.dev))
        with torch.cuda.stream(s):
            self._launch(self.piter)
        torch.cuda.current_stream(self.dev).wait_stream(s)
        with torch.cuda.graph(self.graph):
            self._launch(self.piter)
        for k, v in saved.items():
            getattr(self, k).copy_(v)
        self.A.view("rt").copy_(rt)
        self.trace = trace
        torch.cuda.synchronize(self.dev)

    def replay(self):
        self.graph.replay()

    def run(self, m0, niter, graph=True):
        """Iterations m0 .. niter-1.  Iterations 0 and 1 (36-step ptycho CGs
        from psi = 1, whose last steps are decided within FP32 rounding) run
        through the host Solver's admm_step, so they are those of Solver.admm;
        later ones replay the graph (graph=True) or run its launch sequence
        eagerly."""
        for m in range(m0, niter):
            if m < 2:
                st, rho, tau = self.state()
                st, rho, tau = self.slv.admm_step(m, {k: v.clone() for k, v in st.items()}, rho, tau, self.data,
                                                  self.alpha, self.piter, self.titer,
                                                  ("poisson", "gaussian")[self.model])
                self.load(st, rho, tau)
            elif not graph:
                self.step(m)
            else:
                if self.graph is None:
                    self.capture()
                self.replay()


def slv_fwd_reg(res, u):
    K.reg_fwd(res, u, np.float32(2 / np.sqrt(3)))
    return res
