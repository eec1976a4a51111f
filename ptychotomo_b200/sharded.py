"""ADMM across GPUs: angles and slices sharded over the ranks of a process group.

One process per GPU.  The reference's Solver (src/ptychotomo/solver.py:19-336)
splits the work into angle chunks (ptycho) and slice chunks (tomography) on
one device; here each rank holds one block of angles and one block of slices:

* ptychography is independent per angle: psi, h, lamd, the measured data and
  the scans are split by angle;
* the USFFT Radon transform is independent per slice: u, e, phi, mu are split
  by slice, and each rank's Radon operator sees every angle of its slices;
* two re-shards per ADMM iteration (solver.py:320-326): xi0 and K go from
  angle shards to slice shards after takexi, R u comes back from slice shards
  to angle shards for h (one all-to-all each);
* the TV operator J and its adjoint (solver.py:128-146) take the neighbouring
  rank's boundary slice (a one-slice halo);
* every norm, inner product, line-search sum and maximum is reduced over the
  ranks in FP64, so all ranks take the same step lengths.  A sharded run is
  the single-process Solver with ptheta = ntheta and pnz = nz, up to the
  order of the FP64 sums.

``ShardComm`` carries the collectives: NCCL on the GPUs' own memory, or gloo
with the collective buffers staged through host memory (CPU process groups).
"""
from __future__ import annotations

import torch
import torch.distributed as dist

from .solver import Solver


def block_ranges(total: int, parts: int):
    """Contiguous split of range(total) into `parts` blocks, the first total % parts one longer."""
    base, extra = divmod(total, parts)
    out, start = [], 0
    for r in range(parts):
        size = base + (r < extra)
        out.append((start, start + size))
        start += size
    return out


class ShardComm:
    """Collectives of a sharded ADMM over a torch.distributed process group.

    ``stage_on_host`` copies collective buffers to host memory and back, for
    gloo process groups whose ranks compute on GPUs; NCCL groups use device
    buffers directly.
    """

    def __init__(self, ntheta: int, nz: int, group=None, stage_on_host: bool | None = None):
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.ntheta, self.nz = ntheta, nz
        if self.world > min(ntheta, nz):
            raise ValueError("every rank needs at least one angle and one slice (%d ranks, %d angles, %d slices)"
                             % (self.world, ntheta, nz))
        self.theta_ranges = block_ranges(ntheta, self.world)
        self.z_ranges = block_ranges(nz, self.world)
        backend = dist.get_backend(group)
        self.stage_on_host = (backend != "nccl") if stage_on_host is None else stage_on_host

    # ---- helpers ----------------------------------------------------------
    def _out(self, t):
        return t.cpu() if self.stage_on_host and t.is_cuda else t

    def _back(self, t, like):
        return t.to(like.device) if t.device != like.device else t

    def _peer(self, r):
        """Global rank of group rank r (P2P calls take global ranks)."""
        return r if self.group is None else dist.get_global_rank(self.group, r)

    # ---- FP64 scalar reductions ------------------------------------------
    def allreduce(self, values, op="sum", device=None):
        """Sum (or max) of a list of floats over the ranks, in FP64."""
        dev = torch.device("cpu") if self.stage_on_host or device is None else device
        t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.SUM if op == "sum" else dist.ReduceOp.MAX, group=self.group)
        return t.tolist()

    def allreduce_tensor(self, x):
        """Sum of a (complex) tensor over the ranks; every rank receives it."""
        if self.world == 1:
            return x
        xr = torch.view_as_real(x) if x.is_complex() else x
        buf = self._out(xr.contiguous())
        dist.all_reduce(buf, op=dist.ReduceOp.SUM, group=self.group)
        buf = self._back(buf, x)
        return torch.view_as_complex(buf.contiguous()) if x.is_complex() else buf

    # ---- angle <-> slice re-sharding --------------------------------------
    def theta_to_z(self, x):
        """[angles held, nz, n] -> [ntheta, slices held, n] (complex64)."""
        th0, th1 = self.theta_ranges[self.rank]
        z0, z1 = self.z_ranges[self.rank]
        if self.world == 1:
            return x
        n = x.shape[-1]
        xr = torch.view_as_real(x)
        send = torch.cat([xr[:, a:b].reshape(-1) for a, b in self.z_ranges])
        in_splits = [(th1 - th0) * (b - a) * n * 2 for a, b in self.z_ranges]
        out_splits = [(b - a) * (z1 - z0) * n * 2 for a, b in self.theta_ranges]
        send = self._out(send)
        recv = torch.empty(sum(out_splits), dtype=send.dtype, device=send.device)
        dist.all_to_all_single(recv, send, out_splits, in_splits, group=self.group)
        recv = self._back(recv, x)
        # blocks arrive in rank order = angle order: [ntheta][slices held][n][2]
        return torch.view_as_complex(recv.view(self.ntheta, z1 - z0, n, 2))

    def z_to_theta(self, x):
        """[ntheta, slices held, n] -> [angles held, nz, n] (complex64)."""
        th0, th1 = self.theta_ranges[self.rank]
        z0, z1 = self.z_ranges[self.rank]
        if self.world == 1:
            return x
        n = x.shape[-1]
        xr = torch.view_as_real(x)
        send = torch.cat([xr[a:b].reshape(-1) for a, b in self.theta_ranges])
        in_splits = [(b - a) * (z1 - z0) * n * 2 for a, b in self.theta_ranges]
        out_splits = [(th1 - th0) * (b - a) * n * 2 for a, b in self.z_ranges]
        send = self._out(send)
        recv = torch.empty(sum(out_splits), dtype=send.dtype, device=send.device)
        dist.all_to_all_single(recv, send, out_splits, in_splits, group=self.group)
        recv = self._back(recv, x)
        parts, off = [], 0
        for (a, b), size in zip(self.z_ranges, out_splits):
            parts.append(recv[off:off + size].view(th1 - th0, b - a, n, 2))
            off += size
        return torch.view_as_complex(torch.cat(parts, dim=1).contiguous())

    # ---- one-slice halos --------------------------------------------------
    def _exchange(self, send_to, send_buf, recv_from, recv_like):
        ops, recv = [], None
        if send_to is not None:
            ops.append(dist.P2POp(dist.isend, self._out(send_buf.contiguous()), self._peer(send_to), self.group))
        if recv_from is not None:
            recv = torch.empty_like(self._out(recv_like))
            ops.append(dist.P2POp(dist.irecv, recv, self._peer(recv_from), self.group))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        return None if recv is None else self._back(recv, recv_like)

    def halo_from_next(self, x, axis=0):
        """First slice (along `axis`) of the next rank's block; None on the last rank."""
        r = self.rank
        first = x.narrow(axis, 0, 1)
        return self._exchange(r - 1 if r > 0 else None, first, r + 1 if r + 1 < self.world else None, first)

    def halo_from_prev(self, x, axis=0):
        """Last slice (along `axis`) of the previous rank's block; None on rank 0."""
        r = self.rank
        last = x.narrow(axis, x.shape[axis] - 1, 1)
        return self._exchange(r + 1 if r + 1 < self.world else None, last, r - 1 if r > 0 else None, last)

    # ---- assembling sharded arrays (tests, output) -----------------------
    def gather(self, x, axis, ranges):
        """Concatenate every rank's block along `axis` (all ranks receive the whole array)."""
        if self.world == 1:
            return x
        xr = torch.view_as_real(x) if x.is_complex() else x
        parts = []
        for r, (a, b) in enumerate(ranges):
            shape = list(xr.shape)
            shape[axis] = b - a
            buf = self._out(xr.contiguous()) if r == self.rank else torch.empty(
                shape, dtype=xr.dtype, device=self._out(xr).device)
            dist.broadcast(buf, self._peer(r), group=self.group)
            parts.append(self._back(buf, x))
        out = torch.cat(parts, dim=axis)
        return torch.view_as_complex(out.contiguous()) if x.is_complex() else out


class _GlobalReducer:
    """A Reducer whose results are reduced over the ranks (FP64 sums, maxima)."""

    _MAX = ("maxabs", "maxangle")

    def __init__(self, red, comm: ShardComm, device):
        self._red, self._comm, self._dev = red, comm, device

    def many(self, ops):
        """The local reductions of Reducer.many, then one all-reduce of all
        their values (sums only)."""
        if any(name in self._MAX for name, *_ in ops):
            raise ValueError("many() batches sums only")
        local = self._red.many(ops)
        flat = []
        for v in local:
            flat += [v.real, v.imag] if isinstance(v, complex) else list(v) if isinstance(v, tuple) else [v]
        from .kernels import Reducer
        return Reducer.unpack(ops, self._comm.allreduce(flat, "sum", self._dev))

    def __getattr__(self, name):
        fn = getattr(self._red, name)
        if not callable(fn) or name.startswith("_"):
            return fn

        def reduced(*args, **kw):
            v = fn(*args, **kw)
            op = "max" if name in self._MAX else "sum"
            if isinstance(v, complex):
                re, im = self._comm.allreduce([v.real, v.imag], op, self._dev)
                return complex(re, im)
            if isinstance(v, (list, tuple)):
                out = self._comm.allreduce(list(v), op, self._dev)
                return tuple(out) if isinstance(v, tuple) else out
            return self._comm.allreduce([v], op, self._dev)[0]

        return reduced


class ShardedSolver(Solver):
    """The drop-in Solver on one shard of a multi-GPU ADMM.

    Construct on every rank with the global arguments of ``Solver`` (prb, all
    scans, all angles, ...) and a ``ShardComm``.  Method arguments and results
    are this rank's shards: angle-major arrays (psi, h, lamd, data) hold the
    angles ``comm.theta_ranges[rank]``, slice-major arrays (u, e, phi, mu) the
    slices ``comm.z_ranges[rank]``.
    """

    def __init__(self, prb, scan, theta, det, voxelsize, energy, ntheta, nz, n, comm: ShardComm, device=None):
        self.comm = comm
        th0, th1 = comm.theta_ranges[comm.rank]
        z0, z1 = comm.z_ranges[comm.rank]
        super().__init__(prb, scan, theta, det, voxelsize, energy, ntheta, nz, n, th1 - th0, z1 - z0,
                         device=device, _held=(th0, th1, z0, z1))

    def _reducer(self, red):
        return _GlobalReducer(red, self.comm, self.device)

    def _theta_to_z(self, x):
        return self.comm.theta_to_z(x)

    def _sum_probe(self, g):
        return self.comm.allreduce_tensor(g)

    def _z_to_theta(self, x):
        return self.comm.z_to_theta(x)

    # J and J* along z need the neighbouring rank's boundary slice
    def fwd_reg(self, u):
        nxt = self.comm.halo_from_next(u)
        if nxt is None:
            return super().fwd_reg(u)
        ext = torch.cat([u, nxt])
        return super().fwd_reg(ext)[:, :-1].contiguous()

    def adj_reg(self, gr):
        prv = self.comm.halo_from_prev(gr, axis=1)
        if prv is None:
            return super().adj_reg(gr)
        ext = torch.cat([prv, gr], dim=1)
        return super().adj_reg(ext)[1:].contiguous()

    def solve_reg(self, u, mu, tau, alpha):
        nxt = self.comm.halo_from_next(u)
        if nxt is None:
            return super().solve_reg(u, mu, tau, alpha)
        ext = torch.cat([u, nxt])
        mu_ext = torch.cat([mu, torch.zeros_like(mu[:, :1])], dim=1)
        return super().solve_reg(ext, mu_ext, tau, alpha)[:, :-1].contiguous()

    def _checkpoint_file(self, path):
        """Each rank keeps its own shards: <path>.rank<r>of<world>."""
        return "%s.rank%dof%d" % (path, self.comm.rank, self.comm.world)

    # ---- shard helpers ----------------------------------------------------
    def theta_shard(self, x):
        """This rank's angles of a global angle-major array."""
        a, b = self.comm.theta_ranges[self.comm.rank]
        return x[a:b]

    def z_shard(self, x, axis=0):
        """This rank's slices of a global slice-major array (axis 0, or 1 for [3, nz, n, n])."""
        a, b = self.comm.z_ranges[self.comm.rank]
        return x[a:b] if axis == 0 else x[:, a:b]

    def gather_theta(self, x):
        return self.comm.gather(x, 0, self.comm.theta_ranges)

    def gather_z(self, x, axis=0):
        return self.comm.gather(x, axis, self.comm.z_ranges)
