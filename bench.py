"""Operator throughput benchmark (one JSON line on rank 0).

Workload (one step): the four hot-path operators at 256^3 —
radonusfft fwd + adj (n = nz = 256, 384 angles on [0, pi), M = 7) and
ptychofft fwd + adj (384 angles x 13x13 raster scans, 128x128 probe and
detector), on seeded synthetic inputs.  Metric: algorithmic HBM bytes of the
four operators (pass model below) per second of device time, summed over
ranks (each rank runs the full workload: weak scaling, no data-path
collective).

Pass-model algorithmic bytes per call (complex64 = 8 B):
  USFFT fwd/adj   8 * nz * (n^2 + 4 G^2 + theta * n),  G = 3n
                  (read the object, write the 2N-oversampled grid, column-FFT
                  read + write, gather read, write the projections)
  ptycho fwd/adj  8 * S * (nprb^2 + det^2),  S = total scans
                  (read the probe-sized patch, write the detector frame)

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
    python bench.py --admm        # ADMM wall time (128^3 run, 256^3 iterations); under torchrun with
                                  # --gpus N: the sharded ADMM's iteration time and its all-to-alls
    python bench.py --cg-kernels  # the ptycho CG's frame kernels at the operator workload
    python bench.py --precision   # operator errors vs direct sums, reconstruction errors
    python bench.py --uneven      # uneven scans: one launch for all angles vs one per angle
    python bench.py --precond     # learned preconditioner of the tomography CG (360 angles, missing wedge)
    python bench.py --time-to-target   # time to the plain ADMM's reconstruction: plain vs graph-captured variants
    python bench.py --pcie        # pinned host<->device copy rates (the bound of the e2e leg)
    python bench.py --radon-variants   # radon forward time by chunk pipeline count and gather

``--impl reference`` times the reference's operators: by default the CPU
restatement of the reference (oracle/, all host cores, a bounded sample of
the same workload); ``--ref-backend cuda`` instead times the reference's own
CUDA operators compiled from its sources (oracle/_ref) on the same GPU.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

CFG = dict(n=256, nz=256, ntheta=384, nprb=128, det=128, nside=13, M=7)


def usfft_bytes(n, nz, ntheta):
    G = 3 * n
    return 8 * nz * (n * n + 4 * G * G + ntheta * n)


def ptycho_bytes(S, nprb, det):
    return 8 * S * (nprb * nprb + det * det)


GATHER_NAMES = {0: "L1", 1: "smem tiles", 2: "TMA smem tiles"}


def workload_bytes(c):
    S = c["ntheta"] * c["nside"] ** 2
    ub = usfft_bytes(c["n"], c["nz"], c["ntheta"])
    pb = ptycho_bytes(S, c["nprb"], c["det"])
    return {"radon_fwd": ub, "radon_adj": ub, "ptycho_fwd": pb, "ptycho_adj": pb}


def config_dict(c, extra=None):
    d = {"workload": "radonusfft fwd+adj (n=nz={n}, {ntheta} angles, M={M}) + ptychofft fwd+adj "
                     "({ntheta} angles x {nside}x{nside} scans, {nprb}^2 probe, {det}^2 detector)".format(**c),
         "n": c["n"], "nz": c["nz"], "ntheta": c["ntheta"], "nprb": c["nprb"], "det": c["det"],
         "scans_per_angle": c["nside"] ** 2, "kernel_half_width": c["M"],
         "l2": "inputs larger than L2 (8.5 GB of detector frames per step), no flush",
         "parallelism": "one replica per GPU (angles/slices shard with no exchange)"}
    if extra:
        d.update(extra)
    return d


# DRAM bytes (read + write) of the ptycho adjoint kernel k_ptycho_adj128 per
# 128^2 detector frame at 256^3, by the adjoint's angle split (parts), each
# from one ncu capture (dram__bytes_read.sum + dram__bytes_write.sum, one
# launch, --clock-control none) of
#   python bench.py --ntheta 148 [--no-autotune --ptycho-parts P] --steps 1 --warmup 1 --no-e2e --no-cpu-baseline
# parts 1: 3,691,507,712 + 500,559,104 bytes for 148 x 169 = 25,012 frames;
# parts 3: 3,956,107,008 + 983,063,552 bytes for the same frames.
# 148 angles are one wave of one-slab angle blocks (parts x 148 blocks for a
# split), the per-wave layout of the 384-angle workload, so the figure is
# scaled by the frame count of the run.
PTYCHO_ADJ128_DRAM_PER_FRAME = {1: (3675596800 + 500556032) / 25012, 3: (3934423552 + 988413184) / 25012}


def traffic_source(parts):
    return ("ncu dram__bytes_read.sum + dram__bytes_write.sum of one k_ptycho_adj128 launch (parts %d) at 148 "
            "angles (25,012 frames of 128^2, 256^3 object): %.0f B per frame, scaled by this run's frames"
            % (parts, PTYCHO_ADJ128_DRAM_PER_FRAME[parts]))


def dram_traffic(c, parts):
    """DRAM bytes per ptycho-adjoint kernel launch, scaled from the per-frame
    capture of the same split; None where no capture applies (other detector,
    probe or object sizes, fewer angles than SMs, or an uncaptured split)."""
    if ((c["det"], c["nprb"], c["n"], c["nz"]) != (128, 128, 256, 256) or c["ntheta"] < 148
            or parts not in PTYCHO_ADJ128_DRAM_PER_FRAME):
        return None
    return int(round(PTYCHO_ADJ128_DRAM_PER_FRAME[parts] * c["ntheta"] * c["nside"] ** 2))


# ----------------------------------------------------------------------------
# clocks sampler (nvidia-smi during the timed region)
# ----------------------------------------------------------------------------
class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax = float(p[2])
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


# ----------------------------------------------------------------------------
# our implementation
# ----------------------------------------------------------------------------
def make_inputs(c, seed=0):
    from ptychotomo_b200 import synthetic
    rng = np.random.default_rng(seed)
    n, nz, nt = c["n"], c["nz"], c["ntheta"]
    theta = synthetic.angles(nt)
    u = synthetic.phantom(n, nz, seed=seed)
    prb = synthetic.probe(c["nprb"], seed=seed)
    scan = synthetic.raster_scan(nt, c["nside"], n, nz, c["nprb"])
    proj = (rng.standard_normal((nt, nz, n)) + 1j * rng.standard_normal((nt, nz, n))).astype(np.complex64)
    psi = np.exp(1j * 0.3 * rng.standard_normal((nt, nz, n))).astype(np.complex64)
    return theta, u, prb, scan, proj, psi


class Ops:
    """The four operators with device-resident inputs/outputs."""

    def __init__(self, c, torch, dev):
        from ptychotomo_b200 import ptychofft, radonusfft
        self.c, self.torch, self.dev = c, torch, dev
        theta, u, prb, scan, proj, psi = make_inputs(c)
        n, nz, nt, S = c["n"], c["nz"], c["ntheta"], c["nside"] ** 2
        t = lambda a: torch.from_numpy(a).to(dev)  # noqa: E731
        self.radon = radonusfft(nt, nz, n, m_override=0 if c["M"] == 7 else c["M"])
        self.radon.setobj(t(theta))
        self.ptycho = ptychofft(nt, nz, n, nt, S, c["det"], c["det"], c["nprb"])
        self.ptycho.setobj(t(scan), t(prb))
        self.u, self.proj, self.psi = t(u), t(proj), t(psi)
        cplx = dict(dtype=torch.complex64, device=dev)
        self.proj_out = torch.empty((nt, nz, n), **cplx)
        self.u_out = torch.empty((nz, n, n), **cplx)
        self.frames = torch.empty((nt, S, c["det"], c["det"]), **cplx)
        self.psi_out = torch.empty((nt, nz, n), **cplx)
        self.host = None
        self.tuned = None

    def autotune(self):
        """The operators' autotuners (set-up, untimed): the radon forward's
        streams and gather variant, the ptycho adjoint's angle split."""
        self.ptycho.fwd(self.frames, self.psi)
        streams, gather = self.radon.autotune(self.proj_out, self.u, trials=3)
        parts = self.ptycho.autotune(self.psi_out, self.frames, trials=3)
        self.tuned = {"radon_fwd_streams": streams, "radon_gather": GATHER_NAMES[gather],
                      "ptycho_adj_parts": parts}
        return self.tuned

    def step(self, ev=None):
        r, p = self.radon, self.ptycho
        seq = [("radon_fwd", lambda: r.fwd(self.proj_out, self.u)),
               ("radon_adj", lambda: r.adj(self.u_out, self.proj)),
               ("ptycho_fwd", lambda: p.fwd(self.frames, self.psi)),
               ("ptycho_adj", lambda: p.adj(self.psi_out, self.frames))]
        for name, fn in seq:
            if ev is not None:
                ev[name][0].record()
            fn()
            if ev is not None:
                ev[name][1].record()

    # end to end through the public API: host inputs -> device -> host outputs
    def e2e_setup(self):
        torch = self.torch
        pin = lambda x: torch.empty(x.shape, dtype=x.dtype, pin_memory=True)  # noqa: E731
        self.h_in = {k: pin(getattr(self, k)) for k in ("u", "proj", "psi")}
        for k, v in self.h_in.items():
            v.copy_(getattr(self, k).cpu())
        self.h_frames = pin(self.frames)   # ptycho adj input comes from the host too
        self.h_frames.copy_(self.frames.cpu())
        self.h_out = {k: pin(getattr(self, k)) for k in ("proj_out", "u_out", "frames", "psi_out")}
        self.d_frames_in = torch.empty_like(self.frames)
        # uploads, kernels and downloads on three streams: the 8.5 GB frame
        # download of ptychofft.fwd and the 8.5 GB frame upload of ptychofft.adj
        # use the two PCIe directions at the same time
        self.s_h2d = torch.cuda.Stream(self.dev)
        self.s_d2h = torch.cuda.Stream(self.dev)

    def e2e_step(self):
        torch = self.torch
        r, p = self.radon, self.ptycho
        cs, hs, ds = torch.cuda.current_stream(self.dev), self.s_h2d, self.s_d2h
        cs.wait_stream(ds)   # the previous step's downloads finished before outputs are rewritten
        hs.wait_stream(cs)   # ... and its kernels before inputs are overwritten
        # copy engines serve each direction in issue order: small inputs first,
        # ptychofft.fwd first so that its 8.5 GB download overlaps the 8.5 GB
        # frame upload of ptychofft.adj
        up = {}
        with torch.cuda.stream(hs):
            for k, dst, src in (("psi", self.psi, self.h_in["psi"]), ("u", self.u, self.h_in["u"]),
                                ("proj", self.proj, self.h_in["proj"]), ("frames", self.d_frames_in, self.h_frames)):
                dst.copy_(src, non_blocking=True)
                up[k] = torch.cuda.Event()
                up[k].record(hs)
        for k, call, out in (("psi", lambda: p.fwd(self.frames, self.psi), "frames"),
                             ("u", lambda: r.fwd(self.proj_out, self.u), "proj_out"),
                             ("proj", lambda: r.adj(self.u_out, self.proj), "u_out"),
                             ("frames", lambda: p.adj(self.psi_out, self.d_frames_in), "psi_out")):
            cs.wait_event(up[k])
            call()
            done = torch.cuda.Event()
            done.record(cs)
            ds.wait_event(done)
            with torch.cuda.stream(ds):
                self.h_out[out].copy_(getattr(self, out), non_blocking=True)
        cs.wait_stream(ds)   # the step ends when its results are on the host

    def e2e_bytes(self):
        bi = sum(v.numel() * v.element_size() for v in self.h_in.values()) + self.h_frames.numel() * 8
        bo = sum(v.numel() * v.element_size() for v in self.h_out.values())
        return bi, bo

    def launches_per_step(self):
        """Kernel launches of one step: radon fwd 4 per 8-slice chunk, radon adj 3,
        ptycho fwd 1, ptycho adj 1 plus the slab reduction when the angles are
        split into parts (the operator's current split)."""
        zc = -(-self.c["nz"] // 8)
        return 4 * zc + 3 + 1 + 1 + (self.ptycho.parts > 1)


def run_ours(args, rank, world, local):
    import torch
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    dist = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
    c = dict(CFG)
    ops = Ops(c, torch, dev)
    if not args.no_autotune:
        ops.autotune()
    if args.ptycho_parts:
        ops.ptycho.parts = args.ptycho_parts
        ops.tuned = dict(ops.tuned or {}, ptycho_adj_parts=args.ptycho_parts, parts_source="--ptycho-parts")
    if args.radon_variant:
        streams, gather = (int(v) for v in args.radon_variant.split(","))
        ops.radon.set_variant(streams, gather)
        ops.tuned = dict(ops.tuned or {}, radon_fwd_streams=streams, radon_gather=GATHER_NAMES[gather],
                         radon_source="--radon-variant")
    bytes_op = workload_bytes(c)
    step_bytes = sum(bytes_op.values())

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        ops.step()
    names = list(bytes_op)
    ev = {k: [[torch.cuda.Event(enable_timing=True) for _ in range(2)] for _ in range(args.steps)] for k in names}
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    with Clocks(local) as clk:
        t0.record()
        for i in range(args.steps):
            ops.step({k: ev[k][i] for k in names})
        t1.record()
        barrier()
    ms = t0.elapsed_time(t1)
    per_op = {k: float(np.mean([e[0].elapsed_time(e[1]) for e in ev[k]])) for k in names}
    ms_max = ms
    if dist is not None:
        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_max = float(t.item())
    ms_step = ms_max / args.steps
    value = world * step_bytes / (ms_step * 1e-3) / 1e9

    # end to end through the public API with host buffers
    if args.no_e2e:
        ops.e2e_setup = lambda: None
        ops.e2e_step = lambda: None
        ops.e2e_bytes = lambda: (0, 0)
    ops.e2e_setup()
    for _ in range(2):
        ops.e2e_step()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e_steps = max(1, min(args.steps, 5))
    e0.record()
    for _ in range(e_steps):
        ops.e2e_step()
    e1.record()
    barrier()
    e_ms = e0.elapsed_time(e1) / e_steps
    if dist is not None:
        t = torch.tensor([e_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e_ms = float(t.item())
    bi, bo = ops.e2e_bytes()

    peaks = {}
    pf = ROOT / "MEASURED_PEAKS.json"
    if pf.exists():
        peaks = json.loads(pf.read_text())
    peak = peaks.get("hbm_gbs")
    peak_src = "measured" if peak else "fallback"
    peak = peak or 6650.0
    # the roofline entry is for the step's largest single kernel: the ptycho
    # operators are one launch each (k_ptycho_fwd128, k_ptycho_adj128 plus a
    # short slab reduction); the radon operators are sequences of short
    # launches (4 per 8-slice chunk forward), each far below either ptycho
    # kernel, so their rates are in per_op_gbs only
    # the ptycho adjoint (k_ptycho_adj128): the largest single kernel of the step
    dom = "ptycho_adj"
    achieved = bytes_op[dom] / (per_op[dom] * 1e-3) / 1e9
    traffic = dram_traffic(c, ops.ptycho.parts)

    line = {"metric": "operator HBM GB/s (radonusfft fwd+adj + ptychofft fwd+adj, 256^3)",
            "value": round(value, 2), "unit": "GB/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_step, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c64 (fp32 complex)", "data": "synthetic",
            "config": config_dict(c, {"autotuned": ops.tuned} if ops.tuned else None),
            "per_op_ms": {k: round(v, 4) for k, v in per_op.items()},
            "per_op_gbs": {k: round(bytes_op[k] / (per_op[k] * 1e-3) / 1e9, 1) for k in names},
            "e2e": None if args.no_e2e else {
                "value": round(world * step_bytes / (e_ms * 1e-3) / 1e9, 2), "unit": "GB/s",
                "ms_per_step": round(e_ms, 3), "h2d_bytes_per_step": bi, "d2h_bytes_per_step": bo},
            "gpu_launches": ops.launches_per_step() * args.steps,
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1), "peak": peak,
                         "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": traffic,
                         "traffic_source": traffic_source(ops.ptycho.parts) if traffic is not None else None,
                         "peak_source": peak_src + " hbm_gbs (copy, burst)"},
            "clocks": clk.summary()}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(c, workers=1)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return line


# ----------------------------------------------------------------------------
# CPU restatement of the reference (oracle) on a bounded sample
# ----------------------------------------------------------------------------
def _cpu_sample_job(job):
    """One slice of the USFFT (fwd + adj) or one angle of the ptycho op (fwd + adj)."""
    kind, c, seed = job
    sys.path.insert(0, str(ROOT))
    from oracle.ptycho import PtychoFFT
    from oracle.usfft import RadonUSFFT
    from ptychotomo_b200 import synthetic
    rng = np.random.default_rng(seed)
    n, nt = c["n"], c["ntheta"]
    t = time.perf_counter()
    if kind == "radon":
        op = RadonUSFFT(nt, 1, n)
        op.setobj(synthetic.angles(nt))
        u = rng.standard_normal((1, n, n)) + 1j * rng.standard_normal((1, n, n))
        g = op.fwd(u)
        op.adj(g)
        b = 2 * usfft_bytes(n, 1, nt)
    else:
        S = c["nside"] ** 2
        op = PtychoFFT(1, c["nz"], n, 1, S, c["det"], c["det"], c["nprb"])
        op.setobj(synthetic.raster_scan(1, c["nside"], n, c["nz"], c["nprb"]), synthetic.probe(c["nprb"]))
        psi = np.exp(1j * rng.standard_normal((1, c["nz"], n)))
        op.adj(op.fwd(psi))
        b = 2 * ptycho_bytes(S, c["nprb"], c["det"])
    return b, time.perf_counter() - t


def cpu_baseline(c, workers=1, slices_per_worker=2, angles_per_worker=8):
    """Oracle port timed on a bounded sample, extrapolated to the full workload.

    Each of ``workers`` processes runs USFFT fwd+adj on ``slices_per_worker``
    slices and ptycho fwd+adj on ``angles_per_worker`` angles (the same sizes
    as the workload).  The measured time per slice and per angle (all workers
    busy at once) gives the time of the full workload: its nz slices and
    ntheta angles split across the workers.
    """
    jobs = []
    for w in range(workers):
        jobs += [("radon", c, 100 * w + i) for i in range(slices_per_worker)]
        jobs += [("ptycho", c, 100 * w + i) for i in range(angles_per_worker)]
    t = time.perf_counter()
    if workers == 1:
        res = [_cpu_sample_job(j) for j in jobs]
    else:
        import multiprocessing as mp
        with mp.get_context("spawn").Pool(workers) as pool:
            res = pool.map(_cpu_sample_job, jobs)
    wall = time.perf_counter() - t
    t_slice = np.mean([r[1] for j, r in zip(jobs, res) if j[0] == "radon"])
    t_angle = np.mean([r[1] for j, r in zip(jobs, res) if j[0] == "ptycho"])
    t_full = (t_slice * c["nz"] + t_angle * c["ntheta"]) / workers
    value = sum(workload_bytes(c).values()) / t_full / 1e9
    return {"value": round(value, 4), "unit": "GB/s", "cores": workers, "kind": "port",
            "sample": f"{workers} process(es) x ({slices_per_worker} of {c['nz']} slices radonusfft fwd+adj + "
                      f"{angles_per_worker} of {c['ntheta']} angles ptychofft fwd+adj), NumPy oracle; "
                      f"extrapolated: {t_slice:.2f} s/slice, {t_angle:.3f} s/angle",
            "seconds": round(wall, 2), "est_full_step_s": round(t_full, 1),
            "est_per_operator_s": {"radonusfft_fwd_adj": round(t_slice * c["nz"] / workers, 2),
                                   "ptychofft_fwd_adj": round(t_angle * c["ntheta"] / workers, 2)}}


def run_reference_cpu(args):
    c = dict(CFG)
    workers = max(1, min(os.cpu_count() or 1, 32))
    vals = []
    for _ in range(args.warmup):
        cpu_baseline(c, workers)  # warm imports / page cache
        break
    t0 = time.perf_counter()
    for _ in range(args.steps):
        vals.append(cpu_baseline(c, workers))
    wall = time.perf_counter() - t0
    value = float(np.mean([v["value"] for v in vals]))
    cb = dict(vals[-1])
    cb["value"] = round(value, 4)
    return {"impl": "reference", "metric": "operator HBM GB/s (radonusfft fwd+adj + ptychofft fwd+adj, 256^3)",
            "value": round(value, 4), "unit": "GB/s", "n_gpus": 0, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(1e3 * wall / max(args.steps, 1), 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c128 (NumPy oracle)", "data": "synthetic",
            "config": config_dict(c, {"backend": "CPU restatement of the reference (oracle/), all host cores"}),
            "cpu_baseline": cb,
            "e2e": {"value": round(value, 4), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def run_reference_cuda(args, local):
    """The reference's own CUDA operators (oracle/_ref) on the same workload."""
    import torch
    sys.path.insert(0, str(ROOT / "tests"))
    import refcuda
    if not refcuda.available():
        return {"impl": "reference", "unavailable": "oracle/_ref not built (make -C oracle)"}
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    c = dict(CFG)
    theta, u, prb, scan, proj, psi = make_inputs(c)
    n, nz, nt, S = c["n"], c["nz"], c["ntheta"], c["nside"] ** 2
    t = lambda a: torch.from_numpy(a).to(dev)  # noqa: E731
    th, u_d, prb_d, scan_d, proj_d, psi_d = map(t, (theta, u, prb, scan, proj, psi))
    cplx = dict(dtype=torch.complex64, device=dev)
    proj_out = torch.empty((nt, nz, n), **cplx)
    u_out = torch.empty((nz, n, n), **cplx)
    frames = torch.empty((nt, S, c["det"], c["det"]), **cplx)
    psi_out = torch.empty((nt, nz, n), **cplx)
    r = refcuda.RefRadon(nt, nz, n)
    r.setobj(th.data_ptr())
    p = refcuda.RefPtycho(nt, nz, n, S, c["det"], c["nprb"])
    p.setobj(scan_d.data_ptr(), prb_d.data_ptr())

    def step():
        r.fwd(proj_out.data_ptr(), u_d.data_ptr(), sync=False)
        r.adj(u_out.data_ptr(), proj_d.data_ptr(), sync=False)
        p.fwd(frames.data_ptr(), psi_d.data_ptr(), sync=False)
        p.adj(psi_out.data_ptr(), frames.data_ptr(), sync=False)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / args.steps
    value = sum(workload_bytes(c).values()) / (ms * 1e-3) / 1e9
    return {"impl": "reference", "metric": "operator HBM GB/s (radonusfft fwd+adj + ptychofft fwd+adj, 256^3)",
            "value": round(value, 2), "unit": "GB/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms, 3), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "c64 (fp32 complex)", "data": "synthetic",
            "config": config_dict(c, {"backend": "reference CUDA operators compiled from its sources (oracle/_ref)"}),
            "e2e": {"value": round(value, 2), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


# ---- ADMM wall time ----------------------------------------------------------
# Small plain-ADMM problem: 128^3, 128 angles on [0, pi), 64^2 probe (sigma 12)
# and detector, 7x7 raster with step 10 px, 5 keV, voxel 1e-6 cm, Poisson
# counts at 1e3 mean photons per pixel, 4 ADMM iterations x 4 CG iterations
# (the first two ADMM iterations run 4 + 32 ptycho CG iterations), TV 1e-3.
ADMM_SMALL = dict(n=128, nz=128, ntheta=128, nprb=64, det=64, nside=7, step=10.0, photons=1e3, niter=4,
                  piter=4, titer=4, alpha=1e-3, voxel=1e-6, energy=5.0)


def synthetic_phantom(c, seed=0):
    from ptychotomo_b200 import synthetic
    return synthetic.phantom(c["n"], c["nz"], seed=seed + 2)


def _admm_problem(c, torch, dev, seed=0):
    """Solver, device counts and the true object for an ADMM config."""
    from ptychotomo_b200 import Solver, synthetic
    n, nz, nt = c["n"], c["nz"], c["ntheta"]
    theta = synthetic.angles(nt)
    prb = synthetic.probe(c["nprb"], seed=seed + 1)
    scan = synthetic.raster_scan(nt, c["nside"], n, nz, c["nprb"], step=c.get("step"))
    obj = synthetic.phantom(n, nz, seed=seed + 2)
    slv = Solver(prb, scan, theta, [c["det"], c["det"]], c["voxel"], c["energy"], nt, nz, n, nt, nz, device=dev)
    u = torch.from_numpy(obj).to(dev)
    inten = slv.fwd_ptycho_batch(slv.exptomo(slv.fwd_tomo_batch(u)))
    scale = c["photons"] / float(inten.mean())
    g = torch.Generator(device=dev).manual_seed(seed + 3)
    data = torch.poisson(inten * scale, generator=g) / scale
    return slv, data, u


def _admm_run(slv, data, c, torch, dev, niter, history=None):
    cplx = dict(dtype=torch.complex64, device=dev)
    nt, nz, n = c["ntheta"], c["nz"], c["n"]
    psi = torch.ones((nt, nz, n), **cplx)
    z3 = lambda: torch.zeros((3, nz, n, n), **cplx)  # noqa: E731
    return slv.admm(data, psi.clone(), z3(), psi, z3(), torch.zeros_like(psi), z3(), torch.zeros((nz, n, n), **cplx),
                    c["alpha"], c["piter"], c["titer"], niter, "poisson", verbose=False, history=history)


def _admm_cpu_estimate(c, data, psi_t):
    """NumPy oracle on a bounded sample of the small ADMM, extrapolated to the full run.

    Sample: 2 ptycho CG iterations at full size, one radonusfft fwd + adj on 2 of
    the slices (per-slice cost x nz), and the elementwise ADMM steps once.  Full
    run = sum over ADMM iterations of (piter_m / 2) x CG-ptycho(2) + titer x
    (2 fwd + 1 adj) tomography passes + 1 fwd for h + the elementwise steps.
    """
    from oracle.solver import Solver as OSolver
    from oracle.usfft import RadonUSFFT
    from ptychotomo_b200 import synthetic
    n, nz, nt = c["n"], c["nz"], c["ntheta"]
    theta = synthetic.angles(nt)
    prb = synthetic.probe(c["nprb"], seed=1)
    scan = synthetic.raster_scan(nt, c["nside"], n, nz, c["nprb"], step=c.get("step"))
    obj = synthetic.phantom(n, nz, seed=2)
    osl = OSolver(prb, scan, theta, [c["det"], c["det"]], c["voxel"], c["energy"], nt, nz, n, nt, nz)
    psi = np.ones((nt, nz, n), np.complex64)
    t0 = time.perf_counter()
    osl.cg_ptycho_batch(data, psi, psi.copy(), np.zeros_like(psi), 0.5, 2, "poisson")
    t_cgp2 = time.perf_counter() - t0
    r = RadonUSFFT(nt, 2, n)
    r.setobj(theta)
    f2 = obj[:2].astype(np.complex64)
    t0 = time.perf_counter()
    g2 = r.fwd(f2)
    t_fwd = (time.perf_counter() - t0) / 2 * nz
    t0 = time.perf_counter()
    r.adj(g2)
    t_adj = (time.perf_counter() - t0) / 2 * nz
    z3 = np.zeros((3, nz, n, n), np.complex64)
    t0 = time.perf_counter()
    xi0, xi1, K, ps = osl.takexi(psi_t, z3, np.zeros_like(psi_t), z3, 0.5, 0.5)
    osl.solve_reg(np.zeros((nz, n, n), np.complex64), z3, 0.5, c["alpha"])
    osl.fwd_reg(np.zeros((nz, n, n), np.complex64))
    osl.update_penalty(psi_t, psi_t, psi_t, z3, z3, z3, 0.5, 0.5)
    t_rest = time.perf_counter() - t0
    total = 0.0
    for m in range(c["niter"]):
        piter = c["piter"] + (m < 2) * 32
        total += piter / 2 * t_cgp2 + c["titer"] * (2 * t_fwd + t_adj) + t_fwd + t_rest
    sample = ("NumPy oracle, 1 process: 2 CG-ptycho iterations at full size (%.1f s), radonusfft fwd/adj on "
              "2 of %d slices (%.2f / %.2f s per full call), elementwise ADMM steps (%.1f s); extrapolated to "
              "%d ADMM iterations" % (t_cgp2, nz, t_fwd, t_adj, t_rest, c["niter"]))
    return total, sample


def run_admm(args, local):
    """ADMM wall time on one GPU: the small plain-ADMM problem end to end, and the
    steady-state ADMM iteration (piter = titer = 4) at 256^3 with 384 angles."""
    import torch
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    c = dict(ADMM_SMALL)
    slv, data, u_true = _admm_problem(c, torch, dev)
    cpu_inputs = None
    if not args.no_cpu_baseline:   # the same counts and true psi for the oracle sample
        cpu_inputs = (data.cpu().numpy(), slv.exptomo(slv.fwd_tomo_batch(u_true)).cpu().numpy())
    _admm_run(slv, data, c, torch, dev, 1)   # warm-up (allocator, tables)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    u, _ = _admm_run(slv, data, c, torch, dev, c["niter"])
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    err = float(torch.linalg.vector_norm(u - u_true) / torch.linalg.vector_norm(u_true))
    del slv, data, u_true, u

    class Stamps(list):
        def append(self, x):
            torch.cuda.synchronize()
            x["t"] = time.perf_counter()
            super().append(x)

    big = dict(ADMM_SMALL, n=256, nz=256, ntheta=384, nprb=128, det=128, nside=13, step=None)
    slv, data, _ = _admm_problem(big, torch, dev)
    hist = Stamps()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    _admm_run(slv, data, big, torch, dev, 4, history=hist)
    it_ms = [1e3 * (b["t"] - a) for a, b in zip([t0] + [h["t"] for h in hist[:-1]], hist)]
    # probe retrieval at the same size: 4 CG iterations on the probe for the current psi
    psi_b = slv.exptomo(slv.fwd_tomo_batch(torch.from_numpy(synthetic_phantom(big)).to(dev)))
    torch.cuda.synchronize()
    tp = time.perf_counter()
    slv.cg_probe(data, psi_b, slv.prb, 4, "poisson")
    torch.cuda.synchronize()
    probe_ms = 1e3 * (time.perf_counter() - tp)
    line = {"metric": "plain Poisson ADMM wall time, 128^3 (4 ADMM x 4 CG iterations)", "value": round(wall, 3),
            "unit": "s", "n_gpus": 1, "higher_is_better": False, "dtype": "c64 (fp32 complex), FP64 reductions",
            "data": "synthetic", "config": {"workload": "plain ADMM: " + json.dumps(c)},
            "recon_rel_err_vs_phantom": round(err, 4),
            "iteration_ms_256cubed": {"workload": "384 angles, 13x13 scans, 128^2 probe/detector; iterations 0-1 "
                                                  "run 36 ptycho CG iterations, 2-3 run 4",
                                      "ms": [round(x, 1) for x in it_ms]},
            "probe_cg_4iter_ms_256cubed": round(probe_ms, 1)}
    if not args.no_cpu_baseline:
        est, sample = _admm_cpu_estimate(c, *cpu_inputs)
        line["cpu_baseline"] = {"value": round(est, 1), "unit": "s", "cores": 1, "kind": "port", "sample": sample}
    return line


def run_admm_sharded(args, rank, world, local):
    """ADMM iterations of the sharded Solver on `world` GPUs (one process
    each, NCCL): 256^3, 384 angles, 13x13 scans, 128^2 probe, Poisson 1e3
    photons; every rank holds a block of angles and a block of slices.
    Times 4 steady iterations (4 + 4 CG) as the maximum over ranks of CUDA
    events, and the angle <-> slice all-to-alls inside them separately."""
    import datetime

    import torch
    import torch.distributed as dist
    from ptychotomo_b200 import synthetic
    from ptychotomo_b200.sharded import ShardComm, ShardedSolver
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    if not dist.is_initialized():
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)
    c = dict(ADMM_SMALL, n=256, nz=256, ntheta=384, nprb=128, det=128, nside=13, step=None)
    n, nz, nt = c["n"], c["nz"], c["ntheta"]
    comm = ShardComm(nt, nz)
    theta = synthetic.angles(nt)
    prb = synthetic.probe(c["nprb"], seed=1)
    scan = synthetic.raster_scan(nt, c["nside"], n, nz, c["nprb"])
    obj = synthetic.phantom(n, nz, seed=2)
    slv = ShardedSolver(prb, scan, theta, [c["det"], c["det"]], c["voxel"], c["energy"], nt, nz, n, comm, device=dev)
    u_r = torch.from_numpy(slv.z_shard(obj)).to(dev)
    inten = slv.fwd_ptycho_batch(slv.exptomo(slv._z_to_theta(slv.fwd_tomo_batch(u_r))))
    scale = c["photons"] / float(inten.mean())
    g = torch.Generator(device=dev).manual_seed(3 + rank)
    data = torch.poisson(inten * scale, generator=g) / scale
    del inten
    th0, th1 = comm.theta_ranges[rank]
    z0, z1 = comm.z_ranges[rank]
    cx = dict(dtype=torch.complex64, device=dev)
    one = torch.ones((th1 - th0, nz, n), **cx)
    z3 = torch.zeros((3, z1 - z0, n, n), **cx)
    st = dict(u=torch.zeros((z1 - z0, n, n), **cx), psi=one.clone(), h=one.clone(), e=z3.clone(), phi=z3.clone(),
              lamd=torch.zeros_like(one), mu=z3.clone())
    # time the all-to-alls inside the iterations with events around each call
    xfer = []
    orig_t2z, orig_z2t = comm.theta_to_z, comm.z_to_theta

    def timed(fn):
        def run(x):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            y = fn(x)
            e1.record()
            xfer.append((e0, e1))
            return y
        return run
    comm.theta_to_z, comm.z_to_theta = timed(orig_t2z), timed(orig_z2t)
    rho = tau = 0.5
    st, rho, tau = slv.admm_step(2, st, rho, tau, data, c["alpha"], 4, 4, "poisson")    # warm-up
    xfer.clear()
    dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    K = max(1, args.steps if args.steps < 10 else 4)
    for m in range(K):
        st, rho, tau = slv.admm_step(2 + m, st, rho, tau, data, c["alpha"], 4, 4, "poisson")
    e1.record()
    dist.barrier()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / K
    xms = sum(a.elapsed_time(b) for a, b in xfer) / K
    t = torch.tensor([ms, xms], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms, xms = t.tolist()
    line = {"metric": "sharded ADMM ms per iteration (256^3, 384 angles)", "value": round(ms, 2), "unit": "ms",
            "n_gpus": world, "steps": K, "higher_is_better": False, "scaling": "strong", "data": "synthetic",
            "dtype": "c64 (fp32 complex), FP64 reductions",
            "config": {"workload": "ShardedSolver, angle and slice blocks per rank, NCCL all-to-alls, 4 + 4 CG "
                                   "iterations per ADMM iteration", "parallelism": "angles/slices over %d ranks" % world},
            "all_to_all_ms_per_iteration": round(xms, 3)}
    dist.barrier()
    dist.destroy_process_group()
    return line


def run_cg_kernels(args, local):
    """Device time of the ptycho CG's frame-sized kernels at the operator workload:
    the gradient adjoint with the residual formed on load (Poisson, Gaussian) and
    the line-search reduction for 2, 8 and 16 step lengths."""
    import torch
    from ptychotomo_b200 import kernels as K
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    c = dict(CFG)
    ops = Ops(c, torch, dev)
    p = ops.ptycho
    g = torch.Generator(device=dev).manual_seed(5)
    p.fwd(ops.frames, ops.psi)
    data = (ops.frames.abs() ** 2 * (1 + 0.1 * torch.rand(ops.frames.shape, device=dev, generator=g))).float()
    fd = 0.1 * ops.frames.roll(1, dims=-1)
    red = K.Reducer(dev)
    P = c["nprb"]
    gprb = torch.empty((P, P), dtype=torch.complex64, device=dev)
    prb2 = torch.randn((P, P), dtype=torch.complex64, device=dev, generator=g)
    cases = {"adj_resid_poisson": lambda: p.adj_resid(ops.psi_out, ops.frames, data, 1.0, 0),
             "adj_resid_gaussian": lambda: p.adj_resid(ops.psi_out, ops.frames, data, 1.0, 1),
             "ptycho_adj": lambda: p.adj(ops.psi_out, ops.frames),
             "ls_frames_J2": lambda: red.ls_frames(ops.frames, fd, data, 1.0, 0, [1.0, 0.5]),
             "ls_frames_J8": lambda: red.ls_frames(ops.frames, fd, data, 1.0, 0, [0.5 ** j for j in range(8)]),
             "ls_frames_J16": lambda: red.ls_frames(ops.frames, fd, data, 1.0, 0, [0.5 ** j for j in range(16)]),
             "adj_probe_resid_poisson": lambda: p.adj_probe_resid(gprb, ops.psi, ops.frames, data, 1.0, 0),
             "fwd_probe": lambda: p.fwd_probe(fd, ops.psi, prb2)}
    out = {}
    for name, fn in cases.items():
        for _ in range(args.warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        out[name] = round(e0.elapsed_time(e1) / args.steps, 3)
    S = c["ntheta"] * c["nside"] ** 2
    frame = 8 * S * c["det"] ** 2
    return {"metric": "ptycho CG frame kernels (and the probe-retrieval ones), ms per call", "unit": "ms",
            "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": False, "data": "synthetic",
            "config": config_dict(c), "ms": out,
            "bytes_per_call": {"adj_resid": frame + frame // 2, "ls_frames": 2 * frame + frame // 2}}


def run_precision(args, local):
    """Precision of the FP32 operators and reconstructions (one GPU + host cores).

    Operators at 256^3 with 512 angles on [0, pi): the USFFT forward (M = 7 and
    the M = 4 variant) on 2 slices x 16 angles against the complex128 direct
    sum (oracle/nudft.py), beside the complex128 gridding of the oracle on the
    same sample; the USFFT adjoint identity over the whole volume (FP64 dots);
    the ptycho forward of 2 angles (169 frames each, 128^2) against dense
    complex128 DFTs.  Reconstructions: 32^3, 16 angles, 4 ADMM iterations at
    1e2, 1e3 and 1e4 mean photons per pixel, against the oracle Solver on the
    same counts and against the phantom.
    """
    import torch
    from oracle.nudft import ptycho_fwd_exact, radon_fwd_exact
    from oracle.ptycho import PtychoFFT
    from oracle.solver import Solver as OSolver
    from oracle.usfft import RadonUSFFT
    from ptychotomo_b200 import Solver, ptychofft, radonusfft, synthetic
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))  # noqa: E731
    out = {}
    n = nz = 256
    nt = 512
    theta = synthetic.angles(nt)
    obj = synthetic.phantom(n, nz, seed=4).astype(np.complex64)
    rng = np.random.default_rng(5)
    ang = np.sort(rng.choice(nt, 16, replace=False))
    zs = [nz // 3, 2 * nz // 3]
    for M in (7, 4):
        op = radonusfft(nt, nz, n, m_override=0 if M == 7 else M)
        op.setobj(torch.from_numpy(theta).to(dev))
        f = torch.from_numpy(obj).to(dev)
        g = torch.empty((nt, nz, n), dtype=torch.complex64, device=dev)
        op.fwd(g, f)
        x = torch.empty((nt, op.N), dtype=torch.float32, device=dev)
        y = torch.empty_like(x)
        op.get_xy(x, y)
        xs, ys = x.cpu().numpy()[ang], y.cpu().numpy()[ang]
        exact = radon_fwd_exact(obj[zs], theta[ang], n, xy=(xs, ys))
        gpu = g.cpu().numpy()[ang][:, zs]
        row = {"gpu_vs_direct_sum": rel(gpu, exact)}
        if M == 7:
            orc = RadonUSFFT(len(ang), len(zs), n)
            orc.setobj(theta[ang], xy=(xs, ys))
            row["oracle_c128_gridding_vs_direct_sum"] = rel(orc.fwd(obj[zs]), exact)
            gg = torch.randn((nt, nz, n), dtype=torch.complex64, device=dev, generator=torch.Generator(
                device=dev).manual_seed(6))
            fa = torch.empty((nz, n, n), dtype=torch.complex64, device=dev)
            op.adj(fa, gg)
            a = torch.vdot(g.flatten().cdouble(), gg.flatten().cdouble()).item()
            b = torch.vdot(f.flatten().cdouble(), fa.flatten().cdouble()).item()
            row["adjoint_identity_mismatch"] = abs(a - b) / abs(a)
        out["radon_fwd_M%d" % M] = row
        del op, g
    prb = synthetic.probe(128, seed=1)
    scan = synthetic.raster_scan(2, 13, n, nz, 128)
    psi = np.exp(1j * 0.3 * rng.standard_normal((2, nz, n))).astype(np.complex64)
    pop = ptychofft(2, nz, n, 2, scan.shape[2], 128, 128, 128)
    pop.setobj(torch.from_numpy(scan).to(dev), torch.from_numpy(prb).to(dev))
    fr = torch.empty((2, scan.shape[2], 128, 128), dtype=torch.complex64, device=dev)
    pop.fwd(fr, torch.from_numpy(psi).to(dev))
    orc = PtychoFFT(2, nz, n, 2, scan.shape[2], 128, 128, 128)
    orc.setobj(scan, prb)
    out["ptycho_fwd_det128"] = {"gpu_vs_dense_dft": rel(fr.cpu().numpy(), ptycho_fwd_exact(orc, psi))}
    # reconstructions
    n, nz, nt = 32, 32, 16
    theta = synthetic.angles(nt)
    prb = synthetic.probe(16, seed=1)
    scan = synthetic.raster_scan(nt, 3, n, nz, 16)
    scan[0] += np.float32(0.3)
    obj = synthetic.phantom(n, nz, seed=2)
    args_ = (prb, scan, theta, [16, 16], 1e-6, 5.0, nt, nz, n, nt, nz)
    gs = Solver(*args_, device=dev)
    x = torch.empty((nt, gs.cl_tomo.N), dtype=torch.float32, device=dev)
    y = torch.empty_like(x)
    gs._tomo_all.get_xy(x, y)
    os_ = OSolver(*args_, xy=(x.cpu().numpy(), y.cpu().numpy()))
    inten = os_.fwd_ptycho_batch(os_.exptomo(os_.fwd_tomo_batch(obj)))
    rec = {}
    for photons in (1e2, 1e3, 1e4):
        sc = photons / float(inten.mean())
        data = (np.random.default_rng(7).poisson(inten * sc) / sc).astype(np.float32)
        psi0 = np.ones((nt, nz, n), np.complex64)
        z3 = np.zeros((3, nz, n, n), np.complex64)
        u0 = np.zeros((nz, n, n), np.complex64)
        T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)  # noqa: E731
        ug, _ = gs.admm(T(data), T(psi0), T(z3), T(psi0), T(z3), T(np.zeros_like(psi0)), T(z3), T(u0), 1e-3, 4, 4, 4,
                        "poisson", verbose=False)
        uo, _ = os_.admm(data, psi0.copy(), z3.copy(), psi0.copy(), z3.copy(), np.zeros_like(psi0), z3.copy(),
                         u0.copy(), 1e-3, 4, 4, 4, "poisson")
        ug = ug.cpu().numpy()
        rec["photons_%g" % photons] = {"u_vs_oracle_solver": rel(ug, uo), "u_vs_phantom": rel(ug, obj),
                                       "oracle_u_vs_phantom": rel(uo, obj)}
    out["reconstruction_32cubed_4iter"] = rec
    # reconstructions at 256^3: 512 angles on [0, pi), 13 x 13 scans, 128^2
    # probe, Poisson counts at the three photon levels, 4 ADMM x 4 CG (the
    # small configuration's schedule), against the phantom (the oracle Solver
    # at this size would take hours on the host; it is compared at 32^3 above)
    del gs, os_
    torch.cuda.empty_cache()
    c256 = dict(n=256, nz=256, ntheta=512, nprb=128, det=128, nside=13, step=None, voxel=1e-6, energy=5.0)
    rec256 = {}
    for photons in (1e2, 1e3, 1e4):
        slv, data, u_true = _admm_problem(dict(c256, photons=photons), torch, dev, seed=4)
        cx = dict(dtype=torch.complex64, device=dev)
        one = torch.ones((512, 256, 256), **cx)
        z3 = torch.zeros((3, 256, 256, 256), **cx)
        t0 = time.perf_counter()
        ug, _ = slv.admm(data, one.clone(), z3.clone(), one, z3.clone(), torch.zeros_like(one), z3.clone(),
                         torch.zeros((256, 256, 256), **cx), 1e-3, 4, 4, 4, "poisson", verbose=False)
        torch.cuda.synchronize()
        rec256["photons_%g" % photons] = {
            "u_vs_phantom": float(torch.linalg.vector_norm(ug - u_true) / torch.linalg.vector_norm(u_true)),
            "delta_vs_phantom": float(torch.linalg.vector_norm(ug.real - u_true.real) /
                                      torch.linalg.vector_norm(u_true.real)),
            "beta_vs_phantom": float(torch.linalg.vector_norm(ug.imag - u_true.imag) /
                                     torch.linalg.vector_norm(u_true.imag)),
            "seconds": round(time.perf_counter() - t0, 2)}
        del slv, data, u_true, ug, one, z3
        torch.cuda.empty_cache()
    out["reconstruction_256cubed_512angles_4iter"] = rec256
    return {"metric": "precision study (relative L2 errors)", "n_gpus": 1, "data": "synthetic",
            "config": {"workload": "operators 256^3 / 512 angles (sampled 2 slices x 16 angles for the USFFT "
                                   "direct sums, 2 angles x 169 frames for ptycho); reconstructions 32^3, 16 "
                                   "angles, 4 ADMM iterations (against the oracle Solver), and 256^3, 512 angles, "
                                   "4 ADMM iterations (against the phantom)"},
            "errors": out}


def run_uneven(args, local):
    """Batched uneven scans with a graph-captured iteration, against a per-angle
    loop: 256^3, 720 angles, per-angle scan counts drawn from [100, 400] on a
    jittered spiral (+-3 px; padded with the -1 sentinel), 128^2 probe and
    detector, Poisson counts at 1e3 photons.  Times (1) a ptycho CG iteration
    with all angles in one operator launch (ptheta = ntheta) and with one
    launch per angle (ptheta = 1, the reference's chunk loop at its finest),
    and (2) a steady ADMM iteration (4 + 4 CG iterations): all angles batched
    with device-resident scalars, replayed as one CUDA graph, against the
    host-driven Solver with one launch per angle."""
    import torch
    from ptychotomo_b200 import Solver, synthetic
    from ptychotomo_b200.graphed import GraphedADMM
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    n = nz = 256
    nt, P = args.ntheta or 720, 128
    rng = np.random.default_rng(11)
    counts = rng.integers(100, 401, nt)
    scan = synthetic.jittered_spiral_scan(nt, n, nz, P, counts, jitter=3.0, seed=12)
    theta = synthetic.angles(nt)
    prb = synthetic.probe(P, seed=1)
    obj = synthetic.phantom(n, nz, seed=2)
    out, adm = {}, {}
    data = None
    cx = dict(dtype=torch.complex64, device=dev)

    def init():
        one = torch.ones((nt, nz, n), **cx)
        z3 = torch.zeros((3, nz, n, n), **cx)
        return dict(u=torch.zeros((nz, n, n), **cx), psi=one.clone(), h=one.clone(), e=z3.clone(), phi=z3.clone(),
                    lamd=torch.zeros_like(one), mu=z3.clone())

    for label, ptheta in (("batched", nt), ("per_angle", 1)):
        slv = Solver(prb, scan, theta, [P, P], 1e-6, 5.0, nt, nz, n, ptheta, nz, device=dev)
        if data is None:
            inten = slv.fwd_ptycho_batch(slv.exptomo(slv.fwd_tomo_batch(torch.from_numpy(obj).to(dev))))
            scale = 1e3 / float(inten.mean())
            g = torch.Generator(device=dev).manual_seed(13)
            data = torch.poisson(inten * scale, generator=g) / scale
            del inten
            torch.cuda.empty_cache()
        psi = torch.ones((nt, nz, n), **cx)
        slv.cg_ptycho_batch(data, psi, psi.clone(), torch.zeros_like(psi), 0.5, 1, "poisson")   # warm-up
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        slv.cg_ptycho_batch(data, psi, psi.clone(), torch.zeros_like(psi), 0.5, 4, "poisson")
        torch.cuda.synchronize()
        out[label] = round(1e3 * (time.perf_counter() - t0) / 4, 2)
        del psi
        torch.cuda.empty_cache()
        # a steady ADMM iteration (m = 2) from the same start
        if label == "batched":
            gr = GraphedADMM(slv, data, 1e-3, 4, 4, "poisson")
            gr.load(init(), 0.5, 0.5)
            gr.capture()
            gr.replay()                 # warm-up replay
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            gr.replay()
            torch.cuda.synchronize()
            adm["batched_graph"] = round(1e3 * (time.perf_counter() - t0), 1)
            del gr
        else:
            st = init()
            slv.admm_step(2, st, 0.5, 0.5, data, 1e-3, 4, 4, "poisson")     # warm-up
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            slv.admm_step(2, st, 0.5, 0.5, data, 1e-3, 4, 4, "poisson")
            torch.cuda.synchronize()
            adm["per_angle_host"] = round(1e3 * (time.perf_counter() - t0), 1)
            del st
        del slv
        torch.cuda.empty_cache()
    frames = int(counts.sum())
    return {"metric": "ms per ADMM iteration and per ptycho CG iteration, uneven scans: batched (graph-replayed "
                      "ADMM iteration) vs one launch per angle",
            "unit": "ms", "n_gpus": 1, "higher_is_better": False, "data": "synthetic",
            "config": {"workload": "256^3, %d angles, scans per angle in [100, 400] (%d frames, padded to %d), "
                                   "jittered spiral, 128^2 probe/detector, Poisson 1e3 photons, 4 + 4 CG iterations "
                                   "per ADMM iteration" % (nt, frames, nt * int(counts.max()))},
            "ms_per_admm_iteration": adm, "admm_speedup": round(adm["per_angle_host"] / adm["batched_graph"], 2),
            "ms_per_cg_iteration": out, "cg_speedup": round(out["per_angle"] / out["batched"], 2)}


# ---- learned preconditioner of the tomography CG ------------------------------
# 256^3, 360 angles on [-60, 60) degrees (a 60-degree missing wedge): 64
# training and 16 held-out seeds of white random-phase probes on 8-slice
# volumes (the symbol is per slice) give the targets; the 3->64->64->1
# network is trained on the GPU; then the tomography subproblem of cg_tomo
# on a 256^3 phantom (K = 1, xi0 = R u, xi1 = 0, rho = 0.5) is solved to a
# 1e-4 gradient reduction by plain CG and by PCG with: the diagonal alone
# (Jacobi), the analytic ramp symbol, the symbol measured on the training
# probes (no network), and the network's symbol.
PRECOND = dict(n=256, nz=256, ntheta=360, lo=-np.pi / 3, hi=np.pi / 3, train=64, held=16, harvest_nz=8,
               probes=4, steps=1500, tol=1e-4, max_iter=400)


def _precond_setup(c, torch, dev, nz):
    from ptychotomo_b200 import Solver, synthetic
    theta = synthetic.angles(c["ntheta"], c["lo"], c["hi"])
    prb = synthetic.probe(8, seed=1)          # the tomography operator is what is used here
    scan = synthetic.raster_scan(c["ntheta"], 2, c["n"], nz, 8)
    slv = Solver(prb, scan, theta, [8, 8], 1e-6, 5.0, c["ntheta"], nz, c["n"], c["ntheta"], nz, device=dev)
    return slv, torch.from_numpy(theta).to(dev)


def run_precond(args, local):
    import torch
    from ptychotomo_b200 import synthetic
    from ptychotomo_b200.learned import FourierPreconditioner, harvest_targets, train_network
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    c = dict(PRECOND)
    n = c["n"]
    # training targets from plain CG runs on 8-slice volumes
    hs, th = _precond_setup(c, torch, dev, c["harvest_nz"])
    hpre = FourierPreconditioner(hs._tomo_all, th, hs.coeftomo, dev)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    tg = harvest_targets(hs._tomo_all, hpre, range(1000, 1000 + c["train"] + c["held"]), probes=c["probes"])
    torch.cuda.synchronize()
    t_harvest = time.perf_counter() - t0
    t0 = time.perf_counter()
    net, hist, train_loss, held = train_network(hpre.x, tg[:c["train"]], tg[c["train"]:], steps=c["steps"],
                                                lr=1e-2, lr_final=1e-3, seed=0)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    # the measured symbol itself (mean log over the training probe sets), for comparison
    ys = torch.stack([y for y, _ in tg[:c["train"]]])
    ws = torch.stack([w for _, w in tg[:c["train"]]])
    est_log = ((ys * ws).sum(0) / ws.sum(0).clamp(min=1)).contiguous()
    del hs, hpre, tg
    torch.cuda.empty_cache()
    # the network's forward over a 512^2 frequency grid (262,144 points): CUDA
    # cores (FP32 h1) against the tensor cores (tcgen05 64 x 64 layer)
    xq = torch.rand((512 * 512, 3), device=dev)
    fwd_ms = {}
    for label, fn in (("cuda_cores", net.forward), ("tensor_cores", net.forward_tc)):
        for _ in range(3):
            fn(xq)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(20):
            fn(xq)
        e1.record()
        torch.cuda.synchronize()
        fwd_ms[label] = round(e0.elapsed_time(e1) / 20, 4)
    if net.tc_status():
        raise RuntimeError("tensor-core forward: an MMA wait ran out")
    del xq
    # the subproblem at 256^3
    slv, th = _precond_setup(c, torch, dev, c["nz"])
    pre = FourierPreconditioner(slv._tomo_all, th, slv.coeftomo, dev)
    u = torch.from_numpy(synthetic.phantom(n, c["nz"], seed=5000) * 1e5).to(dev)
    xi0 = slv.fwd_tomo_batch(u)
    Kt = torch.ones_like(xi0)
    xi1 = torch.zeros((3, c["nz"], n, n), dtype=torch.complex64, device=dev)
    u0 = torch.zeros_like(u)
    _, dI = pre.diag()
    k = np.fft.fftfreq(n)
    r = np.hypot(k[None, :], k[:, None])
    ramp = 1.0 / np.maximum(r, 1.0 / n)
    ramp_log = torch.from_numpy(np.log(ramp * dI / ramp.mean()).astype(np.float32)).to(dev)
    jac_log = torch.full((n * n,), float(np.log(dI)), dtype=torch.float32, device=dev)
    out = {}
    for tau in (0.5, 0.05):
        row = {}
        for label in ("plain", "jacobi", "ramp", "measured", "learned"):
            if label == "jacobi":
                pre.set_log_symbol(jac_log)
            elif label == "ramp":
                pre.set_log_symbol(ramp_log)
            elif label == "measured":
                pre.set_log_symbol(est_log)
            elif label == "learned":
                pre.set_network(net)
            P = None if label == "plain" else pre
            slv.pcg_tomo(xi0, xi1, Kt, u0, 0.5, tau, 2, P)      # warm-up
            torch.cuda.synchronize()
            hist_g = []
            t0 = time.perf_counter()
            slv.pcg_tomo(xi0, xi1, Kt, u0, 0.5, tau, c["max_iter"], P, tol=c["tol"], history=hist_g)
            torch.cuda.synchronize()
            dt = time.perf_counter() - t0
            reached = hist_g[-1] <= c["tol"]
            row[label] = {"iterations": len(hist_g) - 1 if reached else None, "seconds": round(dt, 3),
                          "final_reduction": float("%.3g" % hist_g[-1]),
                          # the gradient reduction after 4 iterations: the ADMM runs 4 per subproblem
                          "reduction_after_4": float("%.3g" % hist_g[min(4, len(hist_g) - 1)])}
        out["tau_%g" % tau] = row
    return {"metric": "tomography CG iterations and wall time to a 1e-4 gradient reduction, 256^3, 360 angles on "
                      "[-60, 60) degrees", "unit": "iterations / s", "n_gpus": 1, "higher_is_better": False,
            "data": "synthetic", "dtype": "c64 (fp32 complex); network bf16 weights, FP32 accumulation",
            "config": {"workload": json.dumps({k: (round(v, 6) if isinstance(v, float) else v) for k, v in c.items()})},
            "training": {"harvest_s": round(t_harvest, 2), "train_s": round(t_train, 2), "steps": c["steps"],
                         "loss_first": hist[0][1], "train_loss": train_loss, "held_out_loss": held},
            "network_forward_ms_262144_points": fwd_ms,
            "subproblem": out}


# ---- time to the plain method's reconstruction ---------------------------------
# The operator workload's geometry (256^3, 384 angles on [0, pi), 13x13 scans,
# 128^2 probe and detector), Poisson counts.  Plain: the drop-in Solver.admm
# (the reference's algorithm, host-driven, FP32 with FP64 reductions) for
# `iters` iterations; its last iterate is the target.  Variants: the same
# algorithm with device-resident scalars and the steady iteration replayed as
# a CUDA graph, without and with the learned preconditioner in the
# tomography CG.  Each variant's time to rel-L2 <= 1e-3 of the target on
# delta = -Re u and beta = Im u is the wall time of its iterations up to the
# first that gets there (device-synchronised after every iteration).
# Three more figures say how far that target is defined: the plain method run
# again on counts perturbed by a relative 1e-7 (the size of FP32 rounding)
# ends `sensitivity` away from its own reconstruction (its last value is the
# `floor`); each variant's time to within that floor of the plain
# reconstruction; and each variant's time to the plain reconstruction's
# quality (its rel-L2 error against the true object, delta and beta), a
# target that does not depend on the path.
TTT = dict(n=256, nz=256, ntheta=384, nprb=128, det=128, nside=13, step=None, photons=1e3, alpha=1e-3, piter=4,
           titer=4, voxel=1e-6, energy=5.0, iters=60, tol=1e-3)


# The reference driver's own reconstruction problem (test.py:25-62): 3n/2
# angles on linspace(0, pi) (endpoint included), energy 8.8 keV, a 16-pixel
# flat-top probe of peak intensity 0.1 (objects.probe), scanner3 rasters of
# step 8 with its random offsets (NumPy seed 0), 64^2 detector, TV weight
# 3e-7; the phantom stands in for the chip volume the script reads, and the
# counts are Poisson at 1e3 mean photons per pixel (the script's raw counts
# at peak intensity 0.1 are below one photon per pixel).
DRIVER = dict(n=64, prbsize=16, maxint=0.1, shift=8, det=64, voxel=1e-6, energy=8.8, alpha=3e-7, piter=4, titer=4,
              photons=1e3, iters=100, tol=1e-3)


def _driver_problem(c, torch, dev):
    from ptychotomo_b200 import Solver, probe, scanner3, synthetic
    n = c["n"]
    c.update(nz=n, ntheta=3 * n // 2)
    np.random.seed(0)
    theta = np.linspace(0, np.pi, c["ntheta"]).astype("float32")
    prb = probe(c["prbsize"], c["maxint"])
    scan = scanner3(theta, (n, n), c["shift"], c["shift"], c["prbsize"], spiral=0, randscan=True, save=False)
    obj = synthetic.phantom(n, n, seed=2)
    slv = Solver(prb, scan, theta, [c["det"], c["det"]], c["voxel"], c["energy"], c["ntheta"], n, n, c["ntheta"], n,
                 device=dev)
    u = torch.from_numpy(obj).to(dev)
    inten = slv.fwd_ptycho_batch(slv.exptomo(slv.fwd_tomo_batch(u)))
    scale = c["photons"] / float(inten.mean())
    data = torch.poisson(inten * scale, generator=torch.Generator(device=dev).manual_seed(3)) / scale
    return slv, data, u


def _rel_parts(u, ref):
    import torch
    n = torch.linalg.vector_norm
    return float(n(u.real - ref.real) / n(ref.real)), float(n(u.imag - ref.imag) / n(ref.imag))


def run_time_to_target(args, local):
    import torch
    from ptychotomo_b200.graphed import GraphedADMM
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    c = dict(TTT)
    if args.ttt_iters:
        c["iters"] = args.ttt_iters
    if args.ttt_size:
        c.update(n=args.ttt_size, nz=args.ttt_size)
    if args.ttt_alpha is not None:
        c["alpha"] = args.ttt_alpha
    if args.ttt_photons is not None:
        c["photons"] = args.ttt_photons
    if args.ttt_energy is not None:
        c["energy"] = args.ttt_energy
    if args.ttt_driver:
        c = dict(DRIVER, n=args.ttt_size or DRIVER["n"], iters=args.ttt_iters or DRIVER["iters"])
        slv, data, u_true = _driver_problem(c, torch, dev)
    else:
        slv, data, u_true = _admm_problem(c, torch, dev)
    data = slv._as_data(data)
    nt, nz, n = c["ntheta"], c["nz"], c["n"]
    cx = dict(dtype=torch.complex64, device=dev)

    def init():
        one = torch.ones((nt, nz, n), **cx)
        z3 = torch.zeros((3, nz, n, n), **cx)
        return dict(u=torch.zeros((nz, n, n), **cx), psi=one.clone(), h=one.clone(), e=z3.clone(), phi=z3.clone(),
                    lamd=torch.zeros_like(one), mu=z3.clone())

    def plain_run(d=data):
        st, rho, tau = init(), 0.5, 0.5
        us, ts = [], []
        t = 0.0
        for m in range(c["iters"]):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            st, rho, tau = slv.admm_step(m, st, rho, tau, d, c["alpha"], c["piter"], c["titer"], "poisson")
            torch.cuda.synchronize()
            t += time.perf_counter() - t0
            us.append(st["u"].clone())
            ts.append(t)
        return us, ts

    def graphed_run(pre):
        slv.set_preconditioner(pre)
        g = GraphedADMM(slv, data, c["alpha"], c["piter"], c["titer"], "poisson", precond=pre)
        g.load(init(), 0.5, 0.5)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        g.capture()            # set-up, counted in the wall time
        torch.cuda.synchronize()
        t = time.perf_counter() - t0
        graphed_run.capture_s = t
        us, ts = [], []
        for m in range(c["iters"]):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            g.run(m, m + 1)    # iterations 0-1 through the host Solver, then graph replays
            torch.cuda.synchronize()
            t += time.perf_counter() - t0
            us.append(g.u.clone())
            ts.append(t)
        slv.set_preconditioner(None)
        return us, ts

    us_w, _ = plain_run()   # warm-up (library state, allocator); also the run-to-run check
    us_p, ts_p = plain_run()
    ref = us_p[-1]
    repeat_identical = bool(torch.equal(us_w[-1], ref))
    del us_w
    g = torch.Generator(device=dev).manual_seed(99)
    data_pert = data * (1 + 1e-7 * torch.randn(data.shape, generator=g, device=dev, dtype=data.dtype))
    us_s, _ = plain_run(data_pert)
    del data_pert
    sens = [max(_rel_parts(a, b)) for a, b in zip(us_s, us_p)]
    del us_s
    q_ref = _rel_parts(ref, u_true)      # the plain reconstruction's error against the true object
    floor = sens[-1]                     # how far a 1e-7 change of the counts moves plain's own result
    out = {}

    def reach(us, ts):
        r = {}
        for m, (u, t) in enumerate(zip(us, ts)):
            ed, eb = _rel_parts(u, ref)
            if max(ed, eb) <= c["tol"]:
                r = {"iteration": m, "seconds": round(t, 3)}
                break
        if not r:
            ed, eb = _rel_parts(us[-1], ref)
            r = {"iteration": None, "seconds": None, "final_rel_delta": float("%.3g" % ed),
                 "final_rel_beta": float("%.3g" % eb)}
        for m, (u, t) in enumerate(zip(us, ts)):
            qd, qb = _rel_parts(u, u_true)
            if qd <= q_ref[0] and qb <= q_ref[1]:
                r["plain_quality"] = {"iteration": m, "seconds": round(t, 3)}
                break
        else:
            r["plain_quality"] = {"iteration": None, "seconds": None}
        for m, (u, t) in enumerate(zip(us, ts)):
            if max(_rel_parts(u, ref)) <= floor:
                r["within_floor"] = {"iteration": m, "seconds": round(t, 3)}
                break
        else:
            r["within_floor"] = {"iteration": None, "seconds": None}
        qd, qb = _rel_parts(us[-1], u_true)
        r["final_error_vs_truth"] = {"delta": float("%.4g" % qd), "beta": float("%.4g" % qb)}
        return r

    out["plain"] = dict(reach(us_p, ts_p), ms_per_iteration_steady=round(1e3 * (ts_p[-1] - ts_p[2]) / max(len(ts_p) - 3, 1), 2))
    del us_p
    us_g, ts_g = graphed_run(None)
    out["graphed"] = dict(reach(us_g, ts_g), ms_per_iteration_steady=round(1e3 * (ts_g[-1] - ts_g[2]) / max(len(ts_g) - 3, 1), 2),
                          capture_s=round(graphed_run.capture_s, 3),
                          first_iterations_s=[round(v, 3) for v in ts_g[:4]])
    del us_g
    torch.cuda.empty_cache()
    if not args.ttt_no_precond:
        from ptychotomo_b200.learned import FourierPreconditioner, harvest_targets, train_network
        t0 = time.perf_counter()
        pre = FourierPreconditioner(slv._tomo_all, slv.theta, slv.coeftomo, dev)
        hs = _precond_harvest_solver(slv, dev)
        hpre = FourierPreconditioner(hs._tomo_all, slv.theta, hs.coeftomo, dev)
        tg = harvest_targets(hs._tomo_all, hpre, range(2000, 2016), probes=4)
        net, _, _, _ = train_network(hpre.x, tg, [], steps=1000, lr=1e-2, lr_final=1e-3)
        pre.set_network(net)
        torch.cuda.synchronize()
        t_setup = time.perf_counter() - t0
        del hs, hpre, tg
        us_q, ts_q = graphed_run(pre)
        out["graphed_learned_pcg"] = dict(reach(us_q, ts_q), preconditioner_setup_s=round(t_setup, 2),
                                          ms_per_iteration_steady=round(1e3 * (ts_q[-1] - ts_q[2]) / max(len(ts_q) - 3, 1), 2))
    ratios = {k: (round(out["plain"]["seconds"] / v["seconds"], 2) if v.get("seconds") and out["plain"].get("seconds")
                  else None) for k, v in out.items() if k != "plain"}
    pq = out["plain"]["plain_quality"]["seconds"]
    q_ratios = {k: (round(pq / v["plain_quality"]["seconds"], 2) if pq and v["plain_quality"]["seconds"] else None)
                for k, v in out.items() if k != "plain"}
    pf = out["plain"]["within_floor"]["seconds"]
    f_ratios = {k: (round(pf / v["within_floor"]["seconds"], 2) if pf and v["within_floor"]["seconds"] else None)
                for k, v in out.items() if k != "plain"}
    cfg = {k: (v if not isinstance(v, float) else float("%.6g" % v)) for k, v in c.items()}
    return {"metric": "time to rel-L2 <= 1e-3 of the plain FP32 ADMM reconstruction (delta and beta)", "unit": "s",
            "n_gpus": 1, "higher_is_better": False, "data": "synthetic", "dtype": "c64 (fp32 complex), FP64 reductions",
            "config": {"workload": "Poisson ADMM " + json.dumps(cfg)}, "variants": out, "speedup_vs_plain": ratios,
            "plain_repeat_bit_identical": repeat_identical,
            "sensitivity": {"what": "plain ADMM on counts x (1 + 1e-7 N(0,1)) vs on the counts: max rel-L2 (delta, "
                                    "beta) per iteration", "per_iteration": [float("%.3g" % v) for v in sens]},
            "plain_quality_vs_truth": {"delta": float("%.4g" % q_ref[0]), "beta": float("%.4g" % q_ref[1])},
            "speedup_to_plain_quality": q_ratios,
            "floor": {"what": "the plain run's final distance from its 1e-7-perturbed twin: a target no closer than "
                              "this is within the method's own sensitivity", "value": float("%.3g" % floor)},
            "speedup_to_within_floor": f_ratios}


def run_radon_variants(args, local):
    """The radon forward alone (10 calls after 3 warm-ups, CUDA events) for
    every chunk pipeline count and gather at 64^3 / 96, 128^3 / 192 and
    256^3 / 384 angles: the table the autotuner chooses from."""
    import torch
    from ptychotomo_b200 import radonusfft
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    out = {}
    for n, nt in ((64, 96), (128, 192), (256, 384)):
        theta = np.linspace(0, np.pi, nt, endpoint=False).astype(np.float32)
        op = radonusfft(nt, n, n)
        op.setobj(torch.from_numpy(theta).to(dev))
        f = torch.randn((n, n, n), dtype=torch.complex64, device=dev)
        g = torch.empty((nt, n, n), dtype=torch.complex64, device=dev)
        row = {}
        for st in (1, 2, 4):
            for ga in (0, 1, 2):
                op.set_variant(st, ga)
                for _ in range(3):
                    op.fwd(g, f)
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                torch.cuda.synchronize()
                e0.record()
                for _ in range(10):
                    op.fwd(g, f)
                e1.record()
                torch.cuda.synchronize()
                row["streams %d, %s" % (st, GATHER_NAMES[ga])] = round(e0.elapsed_time(e1) / 10, 4)
        out["n%d_%dangles" % (n, nt)] = row
        del op, f, g
    return {"metric": "radonusfft forward ms by variant", "unit": "ms", "n_gpus": 1, "higher_is_better": False,
            "data": "synthetic", "config": {"workload": "n = nz in {64, 128, 256}, 3n/2 angles, M = 7"},
            "variants": out}


def run_pcie(args, local):
    """Host<->device copy rates with pinned buffers (the e2e leg's bound):
    8 GiB each way alone, then both directions at once on two streams."""
    import torch
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    n = 8 * 1024 ** 3 // 8
    h1 = torch.empty(n, dtype=torch.complex64, pin_memory=True)
    h2 = torch.empty(n, dtype=torch.complex64, pin_memory=True)
    d1 = torch.empty(n, dtype=torch.complex64, device=dev)
    d2 = torch.empty(n, dtype=torch.complex64, device=dev)
    s1, s2 = torch.cuda.Stream(dev), torch.cuda.Stream(dev)

    def timed(fn):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        fn()
        torch.cuda.synchronize()
        return time.perf_counter() - t0

    def both():
        with torch.cuda.stream(s1):
            d1.copy_(h1, non_blocking=True)
        with torch.cuda.stream(s2):
            h2.copy_(d2, non_blocking=True)

    B = n * 8
    for _ in range(2):   # the second round is reported
        th = timed(lambda: d1.copy_(h1, non_blocking=True))
        td = timed(lambda: h2.copy_(d2, non_blocking=True))
        tb = timed(both)
    link = subprocess.run(["nvidia-smi", "-i", str(local), "--query-gpu=pcie.link.gen.current,pcie.link.width.current",
                           "--format=csv,noheader"], capture_output=True, text=True).stdout.strip()
    return {"metric": "pinned host<->device copy rate", "unit": "GB/s", "n_gpus": 1, "bytes_each_way": B,
            "h2d": round(B / th / 1e9, 1), "d2h": round(B / td / 1e9, 1), "concurrent_each_way": round(B / tb / 1e9, 1),
            "pcie_link": link}


def _precond_harvest_solver(slv, dev):
    """A Solver with the same angles and width on 8 slices (training targets)."""
    from ptychotomo_b200 import Solver, synthetic
    theta = slv.theta.cpu().numpy()
    nt, n = len(theta), slv.n
    return Solver(synthetic.probe(8, seed=1), synthetic.raster_scan(nt, 2, n, 8, 8), theta, [8, 8], slv.voxelsize,
                  slv.energy, nt, 8, n, nt, 8, device=dev)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--ref-backend", choices=["cpu", "cuda"], default="cpu")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg (profiling runs)")
    ap.add_argument("--no-autotune", action="store_true", help="keep the operators' default variants")
    ap.add_argument("--ptycho-parts", type=int, default=None, help="fix the ptycho adjoint's angle split")
    ap.add_argument("--radon-variant", default=None,
                    help="fix the radon forward: STREAMS,GATHER (gather 0 L1, 1 smem tiles, 2 TMA tiles; e.g. 2,1)")
    ap.add_argument("--ntheta", type=int, default=None, help="override the angle count (small profiling cases)")
    ap.add_argument("--nz", type=int, default=None, help="override the slice count (small profiling cases)")
    ap.add_argument("--admm", action="store_true", help="ADMM wall time instead of operator throughput")
    ap.add_argument("--cg-kernels", action="store_true", help="device time of the ptycho CG's frame kernels")
    ap.add_argument("--precision", action="store_true", help="operator and reconstruction errors")
    ap.add_argument("--uneven", action="store_true", help="uneven scans: batched vs per-angle launches")
    ap.add_argument("--precond", action="store_true", help="learned preconditioner of the tomography CG")
    ap.add_argument("--time-to-target", action="store_true", help="time to the plain ADMM's reconstruction")
    ap.add_argument("--pcie", action="store_true", help="pinned host<->device copy rates (the e2e bound)")
    ap.add_argument("--radon-variants", action="store_true", help="radon forward time by pipeline count and gather")
    ap.add_argument("--ttt-iters", type=int, default=None)
    ap.add_argument("--ttt-size", type=int, default=None)
    ap.add_argument("--ttt-alpha", type=float, default=None)
    ap.add_argument("--ttt-photons", type=float, default=None)
    ap.add_argument("--ttt-energy", type=float, default=None)
    ap.add_argument("--ttt-driver", action="store_true",
                    help="the reference driver script's problem (probe 16, step-8 rasters, TV 3e-7) at --ttt-size")
    ap.add_argument("--ttt-no-precond", action="store_true")
    args = ap.parse_args()
    if args.ntheta:
        CFG["ntheta"] = args.ntheta
    if args.nz:
        CFG["nz"] = args.nz
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    if args.admm and world > 1:
        line = run_admm_sharded(args, rank, world, local)
        if rank == 0:
            print(json.dumps(line), flush=True)
        return 0
    if (args.admm or args.cg_kernels or args.precision or args.uneven or args.precond or args.time_to_target
            or args.pcie or args.radon_variants):
        if rank == 0:
            fn = (run_admm if args.admm else run_cg_kernels if args.cg_kernels else
                  run_precision if args.precision else run_precond if args.precond else
                  run_time_to_target if args.time_to_target else run_pcie if args.pcie else
                  run_radon_variants if args.radon_variants else run_uneven)
            print(json.dumps(fn(args, local)), flush=True)
        return 0
    if args.impl == "reference":
        if rank != 0:
            return 0
        line = run_reference_cuda(args, local) if args.ref_backend == "cuda" else run_reference_cpu(args)
    else:
        line = run_ours(args, rank, world, local)
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
