"""The learned Fourier preconditioner of the tomography CG.

No counterpart in the reference, whose tomography CG
(src/ptychotomo/solver.py:180-203) is unpreconditioned.  This module holds
the network part: a 3 -> 64 -> 64 -> 1 MLP (SiLU) whose forward pass,
gradient and Adam update are the library's own kernels (pt_mlp_*); the
weights are bfloat16 in the arithmetic (FP32 master copy, FP32
accumulation).
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from ._lib import check, current_stream, lib


def _p(t):
    if not t.is_cuda or not t.is_contiguous():
        raise ValueError("network arrays must be contiguous CUDA tensors")
    return t.data_ptr()


class MLP:
    """The preconditioner network with its optimiser state on one device."""

    H = 64

    def __init__(self, device, seed=0, bf16=True, params=None):
        self.device = torch.device(device)
        self.bf16 = bool(bf16)
        self.npar = lib().pt_mlp_param_count()
        if params is None:
            params = self.init_params(seed)
        self.params = torch.as_tensor(np.asarray(params, np.float32), device=self.device).contiguous()
        if self.params.numel() != self.npar:
            raise ValueError(f"expected {self.npar} parameters, got {self.params.numel()}")
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.grad = torch.zeros_like(self.params)
        self.loss = torch.zeros(1, dtype=torch.float64, device=self.device)
        self.work = torch.empty(lib().pt_mlp_workspace_bytes() // 4, dtype=torch.float32, device=self.device)
        self.step = 0
        self._tc_err = None

    @classmethod
    def init_params(cls, seed=0):
        """He-style uniform initialisation (seeded), biases zero."""
        H = cls.H
        rng = np.random.default_rng(seed)
        W1 = rng.uniform(-1, 1, (H, 3)) * np.sqrt(6.0 / 3)
        W2 = rng.uniform(-1, 1, (H, H)) * np.sqrt(6.0 / H)
        W3 = rng.uniform(-1, 1, H) * np.sqrt(3.0 / H)
        return np.concatenate([W1.ravel(), np.zeros(H), W2.ravel(), np.zeros(H), W3, np.zeros(1)]).astype(np.float32)

    def forward(self, x, out=None):
        """x [npts, 3] float32 (device) -> z [npts]."""
        n = x.shape[0]
        out = torch.empty(n, dtype=torch.float32, device=self.device) if out is None else out
        check(lib().pt_mlp_forward(_p(self.params), int(self.bf16), _p(x), _p(out), n, current_stream()),
              "mlp_forward")
        return out

    def forward_tc(self, x, out=None):
        """The same network on the tensor cores: the 64 x 64 layer as tcgen05
        MMAs (bf16 weights and bf16-rounded h1, FP32 accumulation in tensor
        memory), layer 1 and the rest in FP32.  Raises if a tile's MMA did not
        complete within its bounded wait."""
        n = x.shape[0]
        out = torch.empty(n, dtype=torch.float32, device=self.device) if out is None else out
        if self._tc_err is None:
            self._tc_err = torch.zeros(1, dtype=torch.int32, device=self.device)
        check(lib().pt_mlp_forward_tc(_p(self.params), _p(x), _p(out), n, _p(self._tc_err), current_stream()),
              "mlp_forward_tc")
        return out

    def check_tc_wait(self):
        """Run one tile of the tensor-core forward whose wait cannot complete
        (a barrier nothing arrives at, short limit); returns the recorded
        failure code (1) and clears it."""
        x = torch.zeros((128, 3), dtype=torch.float32, device=self.device)
        z = torch.zeros(128, dtype=torch.float32, device=self.device)
        if self._tc_err is None:
            self._tc_err = torch.zeros(1, dtype=torch.int32, device=self.device)
        check(lib().pt_mlp_check_tc_wait(_p(self.params), _p(x), _p(z), _p(self._tc_err), current_stream()),
              "mlp_check_tc_wait")
        return self.tc_status()

    def tc_status(self):
        """Nonzero if a tensor-core forward's MMA wait ran out (then cleared)."""
        if self._tc_err is None:
            return 0
        v = int(self._tc_err.item())
        self._tc_err.zero_()
        return v

    def loss_grad(self, x, y, w, inv_wsum):
        """Loss (device double, kept in self.loss) and gradient (self.grad)."""
        check(lib().pt_mlp_grad(_p(self.params), int(self.bf16), _p(x), _p(y), _p(w), x.shape[0], float(inv_wsum),
                                _p(self.grad), _p(self.loss), _p(self.work), current_stream()), "mlp_grad")
        return self.loss

    def adam(self, lr, beta1=0.9, beta2=0.999, eps=1e-8):
        self.step += 1
        check(lib().pt_mlp_adam(_p(self.params), _p(self.m), _p(self.v), _p(self.grad), self.step, float(lr),
                                float(beta1), float(beta2), float(eps), current_stream()), "mlp_adam")

    def fit(self, x, y, w, steps, lr=3e-3, lr_final=3e-4, log_every=0):
        """Full-batch Adam on the weighted least-squares loss, the step size
        decaying geometrically from lr to lr_final.  Returns the loss history
        (every log_every steps, and the last) as floats."""
        inv = 1.0 / float(w.double().sum())
        hist = []
        for k in range(steps):
            self.loss_grad(x, y, w, inv)
            if log_every and (k % log_every == 0):
                hist.append((k, float(self.loss.item())))
            self.adam(lr * (lr_final / lr) ** (k / max(steps - 1, 1)))
        self.loss_grad(x, y, w, inv)
        hist.append((steps, float(self.loss.item())))
        return hist

    def state(self):
        return self.params.detach().cpu().numpy().copy()


class FourierPreconditioner:
    """P = D^-1/2 F2^-1 diag(p) F2 D^-1/2 for the tomography CG of one
    radon operator (pt_precond_*): D the diagonal of rho kbar R^T R + tau J^T J
    (exact for the edge pixels, from unit-pixel forwards), p from the symbol
    a(w) of R^T R, which the network predicts from the features of w.

    ``radon``: the operator the CG applies (its n and slice count), ``theta``
    its angles (device float32), ``scale`` the factor the CG applies to it
    (Solver.coeftomo)."""

    def __init__(self, radon, theta, scale, device):
        self.device = torch.device(device)
        self.n, self.nz = radon.n, radon.Nz
        self.scale = float(scale)
        h = ctypes.c_void_p()
        check(lib().pt_precond_create(self.nz, self.n, ctypes.byref(h)), "precond create")
        self._h = h
        check(lib().pt_precond_set_diag(h, radon._h, self.scale, current_stream()), "precond set_diag")
        self.theta = theta.to(device=self.device, dtype=torch.float32).contiguous()
        self.x = torch.empty((self.n * self.n, 3), dtype=torch.float32, device=self.device)
        check(lib().pt_precond_features(_p(self.theta), self.theta.numel(), self.n, _p(self.x), current_stream()),
              "precond features")
        self.net = None

    def set_network(self, net, tensor_cores=True):
        """Symbol a = exp(net(features)) for every frequency, evaluated on the
        tensor cores (MLP.forward_tc) when the network has bf16 weights and
        tensor_cores is set, else on the CUDA cores (MLP.forward)."""
        if tensor_cores and net.bf16:
            z = net.forward_tc(self.x)
            if net.tc_status():
                raise RuntimeError("precond: a tensor-core MMA wait ran out while evaluating the symbol")
        else:
            z = net.forward(self.x)
        check(lib().pt_precond_set_log_symbol(self._h, _p(z), current_stream()), "precond set_log_symbol")
        self.net = net

    def set_log_symbol(self, log_a):
        check(lib().pt_precond_set_log_symbol(self._h, _p(log_a), current_stream()), "precond set_log_symbol")

    def symbol(self):
        a = torch.empty((self.n, self.n), dtype=torch.float32, device=self.device)
        check(lib().pt_precond_get_symbol(self._h, _p(a), current_stream()), "precond get_symbol")
        return a

    def diag(self):
        d = torch.empty((self.n, self.n), dtype=torch.float32, device=self.device)
        dI = ctypes.c_float()
        check(lib().pt_precond_get_diag(self._h, _p(d), ctypes.byref(dI), current_stream()), "precond get_diag")
        return d, dI.value

    def apply(self, out, g, rho_kbar, tau):
        check(lib().pt_precond_apply(self._h, _p(out), _p(g), float(rho_kbar), float(tau), current_stream()),
              "precond apply")
        return out

    def spectrum(self, num, den, z, az):
        check(lib().pt_precond_spectrum(self._h, _p(num), _p(den), _p(z), _p(az), current_stream()),
              "precond spectrum")

    def phase_probe(self, dst, src, seed, floor=0.0):
        check(lib().pt_precond_phase_probe(self._h, _p(dst), _p(src), int(seed) & 0xFFFFFFFF, float(floor),
                                           current_stream()), "precond phase_probe")
        return dst

    def free(self):
        if getattr(self, "_h", None):
            lib().pt_precond_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.free()
        except Exception:  # interpreter shutdown
            pass


def harvest_targets(radon, pre, seeds, probes=4, window=(0.30, 0.42)):
    """Training targets: per-frequency Rayleigh quotients of the interior
    part of R^T R.

    For each seed, ``probes`` white probes (unit modulus at every 2-D
    frequency of every slice, random phases from the seed), windowed to the
    slice interior (radial window W, 1 within window[0] n, 0 beyond
    window[1] n), give z = W z0 and A z = W s^2 R^T R z (s = pre.scale; the
    exact adjoint), and
        a*(w) = sum Re(conj(Z) AZ) / sum |Z|^2   (Z = F2 z, AZ = F2 A z),
    the symbol of the operator away from the border, where the forward's
    edge replication makes the diagonal 8-54 times larger (the diagonal D of
    the preconditioner handles the border; unwindowed probes spread that
    border weight over every frequency, a white bias that swamps the small
    high-frequency symbol).  The slices and probes of a seed average its
    noise.  Returns [(log a*, weight)] per seed, float32 [n * n] each; the
    weight is 1 where the quotient is positive.  (Probes with the modulus
    spectrum of CG residuals were tried first: where a residual has little
    energy the quotient is dominated by leakage from strong frequencies, and
    the network fit to them slowed the CG down.)"""
    s = pre.scale
    n, nz = pre.n, pre.nz
    out = []
    cplx = dict(dtype=torch.complex64, device=pre.device)
    z, az = torch.empty((nz, n, n), **cplx), torch.empty((nz, n, n), **cplx)
    rz = torch.empty((radon.Ntheta, nz, n), **cplx)
    for seed in seeds:
        num = torch.zeros((n, n), dtype=torch.float64, device=pre.device)
        den = torch.zeros_like(num)
        for k in range(probes):
            check(lib().pt_precond_phase_probe(pre._h, _p(z), None, (int(seed) * 7919 + k) & 0xFFFFFFFF, 1.0,
                                               current_stream()), "precond phase_probe")
            if window is not None:
                check(lib().pt_precond_window(pre._h, _p(z), window[0] * n, window[1] * n, current_stream()),
                      "precond window")
            radon.fwd(rz, z, scale=s)
            radon.adj_exact(az, rz, scale=s)
            if window is not None:
                check(lib().pt_precond_window(pre._h, _p(az), window[0] * n, window[1] * n, current_stream()),
                      "precond window")
            pre.spectrum(num, den, z, az)
        y = torch.empty(n * n, dtype=torch.float32, device=pre.device)
        w = torch.empty_like(y)
        check(lib().pt_precond_targets(_p(num), _p(den), n * n, 1e-12, _p(y), _p(w), current_stream()),
              "precond targets")
        out.append((y, w))
    return out


def train_network(x, train, held_out, steps=1500, lr=3e-3, lr_final=3e-4, seed=0, bf16=True, log_every=250):
    """Fit the network to the targets of the training volumes (full batch,
    the project's Adam kernel); returns (net, history, train loss, held-out
    loss).  x: the features [n*n, 3]; train / held_out: lists of (y, w)."""
    X = x.repeat(len(train), 1).contiguous()
    Y = torch.cat([y for y, _ in train]).contiguous()
    W = torch.cat([w for _, w in train]).contiguous()
    net = MLP(x.device, seed=seed, bf16=bf16)
    hist = net.fit(X, Y, W, steps, lr=lr, lr_final=lr_final, log_every=log_every)
    train_loss = hist[-1][1]
    held = None
    if held_out:
        Xh = x.repeat(len(held_out), 1).contiguous()
        Yh = torch.cat([y for y, _ in held_out]).contiguous()
        Wh = torch.cat([w for _, w in held_out]).contiguous()
        held = float(net.loss_grad(Xh, Yh, Wh, 1.0 / float(Wh.double().sum())).item())
    return net, hist, train_loss, held
