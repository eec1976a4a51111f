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


def dram_traffic(op):
    """DRAM bytes (read + write) per call of `op` from the committed ncu summary
    profiles/dram_traffic_bench_256cubed.md (rows `| op | bytes | ... |`)."""
    path = ROOT / "profiles" / "dram_traffic_bench_256cubed.md"
    if not path.exists():
        return None
    for line in path.read_text().splitlines():
        cells = [c.strip() for c in line.strip().strip("|").split("|")]
        if len(cells) >= 2 and cells[0] == op:
            try:
                return int(float(cells[1]))
            except ValueError:
                return None
    return None


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

    def e2e_step(self):
        r, p = self.radon, self.ptycho
        self.u.copy_(self.h_in["u"], non_blocking=True)
        r.fwd(self.proj_out, self.u)
        self.h_out["proj_out"].copy_(self.proj_out, non_blocking=True)
        self.proj.copy_(self.h_in["proj"], non_blocking=True)
        r.adj(self.u_out, self.proj)
        self.h_out["u_out"].copy_(self.u_out, non_blocking=True)
        self.psi.copy_(self.h_in["psi"], non_blocking=True)
        p.fwd(self.frames, self.psi)
        self.h_out["frames"].copy_(self.frames, non_blocking=True)
        self.d_frames_in.copy_(self.h_frames, non_blocking=True)
        p.adj(self.psi_out, self.d_frames_in)
        self.h_out["psi_out"].copy_(self.psi_out, non_blocking=True)

    def e2e_bytes(self):
        bi = sum(v.numel() * v.element_size() for v in self.h_in.values()) + self.h_frames.numel() * 8
        bo = sum(v.numel() * v.element_size() for v in self.h_out.values())
        return bi, bo

    def launches_per_step(self):
        zc = -(-self.c["nz"] // 8)
        return 3 * zc + 3 + 2   # radon fwd: 3 per 8-slice chunk; radon adj: 3; ptycho: 1 + 1


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
    dom = max(per_op, key=per_op.get)
    achieved = bytes_op[dom] / (per_op[dom] * 1e-3) / 1e9
    traffic = dram_traffic(dom)

    line = {"metric": "operator HBM GB/s (radonusfft fwd+adj + ptychofft fwd+adj, 256^3)",
            "value": round(value, 2), "unit": "GB/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_step, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "c64 (fp32 complex)", "data": "synthetic",
            "config": config_dict(c),
            "per_op_ms": {k: round(v, 4) for k, v in per_op.items()},
            "per_op_gbs": {k: round(bytes_op[k] / (per_op[k] * 1e-3) / 1e9, 1) for k in names},
            "e2e": None if args.no_e2e else {
                "value": round(world * step_bytes / (e_ms * 1e-3) / 1e9, 2), "unit": "GB/s",
                "ms_per_step": round(e_ms, 3), "h2d_bytes_per_step": bi, "d2h_bytes_per_step": bo},
            "gpu_launches": ops.launches_per_step() * args.steps,
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": round(achieved, 1), "peak": peak,
                         "unit": "GB/s", "frac": round(achieved / peak, 4), "traffic": traffic,
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
            "seconds": round(wall, 2), "est_full_step_s": round(t_full, 1)}


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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--ref-backend", choices=["cpu", "cuda"], default="cpu")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg (profiling runs)")
    ap.add_argument("--ntheta", type=int, default=None, help="override the angle count (small profiling cases)")
    ap.add_argument("--nz", type=int, default=None, help="override the slice count (small profiling cases)")
    args = ap.parse_args()
    if args.ntheta:
        CFG["ntheta"] = args.ntheta
    if args.nz:
        CFG["nz"] = args.nz
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
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
