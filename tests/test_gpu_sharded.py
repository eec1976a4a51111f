"""The sharded ADMM (ptychotomo_b200.sharded.ShardedSolver) against the
single-process Solver with ptheta = ntheta, pnz = nz.

* world size 1: the sharded code path with identity collectives gives the
  same bits as Solver;
* world size 2: two gloo ranks in spawned processes share cuda:0, with the
  collective buffers staged through host memory (the ranks wait for each
  other on the host only; no kernel waits on another process).  Angles and
  slices are split 8 + 8 and 16 + 16.  The ADMM's penalty schedule must
  match exactly, psi and u to 1e-4 (the ptycho adjoint sums its per-angle
  parts in an order that depends on the number of angles per launch, and the
  FP64 reductions add per-rank partials, so the two runs differ in the last
  float bits).
"""
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

N, NZ, NTHETA, NPRB = 32, 32, 16, 16


def _problem():
    from ptychotomo_b200 import synthetic
    theta = synthetic.angles(NTHETA)
    prb = synthetic.probe(NPRB, seed=1)
    scan = synthetic.raster_scan(NTHETA, 3, N, NZ, NPRB)
    scan[0] += np.float32(0.3)
    obj = synthetic.phantom(N, NZ, seed=2)
    return theta, prb, scan, obj


def _data(slv, obj):
    u = torch.from_numpy(obj).cuda()
    d = slv.fwd_ptycho_batch(slv.exptomo(slv.fwd_tomo_batch(u)))
    g = torch.Generator(device="cuda").manual_seed(3)
    return torch.poisson(d * 1e3, generator=g) / 1e3


def _admm(slv, data, niter, th, zs, probe_iter=0):
    c = dict(dtype=torch.complex64, device="cuda")
    psi = torch.ones((th, NZ, N), **c)
    z3 = lambda: torch.zeros((3, zs, N, N), **c)  # noqa: E731
    hist = []
    u, psi = slv.admm(data, psi.clone(), z3(), psi, z3(), torch.zeros_like(psi), z3(),
                      torch.zeros((zs, N, N), **c), 1e-3, 4, 4, niter, "poisson", verbose=False, history=hist,
                      probe_iter=probe_iter)
    return u, psi, [(h["rho"], h["tau"]) for h in hist]


def _reference(niter, probe_iter=0):
    from ptychotomo_b200 import Solver
    theta, prb, scan, obj = _problem()
    slv = Solver(prb, scan, theta, [NPRB, NPRB], 1e-6, 5.0, NTHETA, NZ, N, NTHETA, NZ)
    data = _data(slv, obj)
    out = (data,) + _admm(slv, data, niter, NTHETA, NZ, probe_iter)
    return out + (slv.prb.cpu().numpy(),)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, niter, outdir, data_path, probe_iter):
    import datetime
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    from ptychotomo_b200.sharded import ShardComm, ShardedSolver
    theta, prb, scan, _ = _problem()
    comm = ShardComm(NTHETA, NZ)
    slv = ShardedSolver(prb, scan, theta, [NPRB, NPRB], 1e-6, 5.0, NTHETA, NZ, N, comm)
    data = slv.theta_shard(torch.from_numpy(np.load(data_path)).cuda()).contiguous()
    u, psi, hist = _admm(slv, data, niter, slv.ntheta_held, slv.nz_held, probe_iter)
    u_all, psi_all = slv.gather_z(u), slv.gather_theta(psi)
    if rank == 0:
        np.save(os.path.join(outdir, "u.npy"), u_all.cpu().numpy())
        np.save(os.path.join(outdir, "psi.npy"), psi_all.cpu().numpy())
        np.save(os.path.join(outdir, "hist.npy"), np.array(hist))
        np.save(os.path.join(outdir, "prb.npy"), slv.prb.cpu().numpy())
    dist.barrier()
    dist.destroy_process_group()


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("backend", ["gloo", "nccl"])
def test_sharded_world1_is_the_solver_bitwise(backend):
    import datetime
    import torch.distributed as dist
    from ptychotomo_b200.sharded import ShardComm, ShardedSolver
    data, u_ref, psi_ref, hist_ref, _ = _reference(2)
    store = dist.HashStore()
    kw = {"device_id": torch.device("cuda", 0)} if backend == "nccl" else {}
    dist.init_process_group(backend, store=store, rank=0, world_size=1, timeout=datetime.timedelta(seconds=60), **kw)
    try:
        theta, prb, scan, _ = _problem()
        slv = ShardedSolver(prb, scan, theta, [NPRB, NPRB], 1e-6, 5.0, NTHETA, NZ, N, ShardComm(NTHETA, NZ))
        u, psi, hist = _admm(slv, data, 2, NTHETA, NZ)
    finally:
        dist.destroy_process_group()
    assert hist == hist_ref
    assert torch.equal(u, u_ref) and torch.equal(psi, psi_ref)


@pytest.mark.parametrize("probe_iter", [0, 2])
def test_sharded_two_ranks_on_one_gpu_match_the_solver(tmp_path, probe_iter):
    """probe_iter = 2 also retrieves the probe: its gradient is summed over the ranks."""
    import torch.multiprocessing as mp
    niter = 3
    data, u_ref, psi_ref, hist_ref, prb_ref = _reference(niter, probe_iter)
    data_path = str(tmp_path / "data.npy")
    np.save(data_path, data.cpu().numpy())
    ctx = mp.get_context("spawn")
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, niter, str(tmp_path), data_path, probe_iter))
             for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
    alive = [p for p in procs if p.is_alive()]
    for p in alive:
        p.kill()
    assert not alive, "ranks did not finish"
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    hist = [tuple(h) for h in np.load(tmp_path / "hist.npy").tolist()]
    assert hist == hist_ref
    assert _rel(np.load(tmp_path / "u.npy"), u_ref.cpu().numpy()) < 1e-4
    assert _rel(np.load(tmp_path / "psi.npy"), psi_ref.cpu().numpy()) < 1e-4
    assert _rel(np.load(tmp_path / "prb.npy"), prb_ref) < 1e-4
