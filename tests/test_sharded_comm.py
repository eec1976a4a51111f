"""Collectives of the sharded ADMM (ptychotomo_b200.sharded.ShardComm) on CPU.

Two gloo ranks in spawned processes, ragged shards (5 angles and 7 slices over
2 ranks).  Every rank builds the same seeded global arrays and checks its
shards against them exactly: the angle -> slice and slice -> angle
all-to-alls, the one-slice halos of the TV operator, the FP64 sum / max
reductions (single and batched into one all-reduce) and the gather used to
assemble results.
"""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _crand(g, shape):
    return torch.complex(torch.randn(shape, generator=g), torch.randn(shape, generator=g))


def _worker(rank, world, port, ntheta, nz, n, errq):
    try:
        os.environ["MASTER_ADDR"] = "127.0.0.1"
        os.environ["MASTER_PORT"] = str(port)
        import datetime
        dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
        from ptychotomo_b200.sharded import ShardComm, block_ranges
        comm = ShardComm(ntheta, nz)
        assert comm.theta_ranges == block_ranges(ntheta, world) and comm.z_ranges == block_ranges(nz, world)
        g = torch.Generator().manual_seed(7)
        A = _crand(g, (ntheta, nz, n))            # an angle-major array, e.g. xi0
        U = _crand(g, (3, nz, n, n))              # a slice-major gradient field
        th0, th1 = comm.theta_ranges[rank]
        z0, z1 = comm.z_ranges[rank]
        # angle shard -> slice shard and back
        az = comm.theta_to_z(A[th0:th1].contiguous())
        assert torch.equal(az, A[:, z0:z1])
        assert torch.equal(comm.z_to_theta(A[:, z0:z1].contiguous()), A[th0:th1])
        # halos
        nxt = comm.halo_from_next(U[0, z0:z1].contiguous())
        assert (nxt is None) == (rank == world - 1)
        if nxt is not None:
            assert torch.equal(nxt, U[0, z1:z1 + 1])
        prv = comm.halo_from_prev(U[:, z0:z1].contiguous(), axis=1)
        assert (prv is None) == (rank == 0)
        if prv is not None:
            assert torch.equal(prv, U[:, z0 - 1:z0])
        # FP64 reductions of per-rank partials
        part = float(A[th0:th1].abs().double().pow(2).sum())
        tot, = comm.allreduce([part])
        assert abs(tot - float(A.abs().double().pow(2).sum())) <= 1e-12 * tot
        mx, = comm.allreduce([float(A[th0:th1].abs().max())], op="max")
        assert mx == float(A.abs().max())
        # tensor sum (probe gradients)
        pr = _crand(torch.Generator().manual_seed(rank), (5, 5))
        tot_t = comm.allreduce_tensor(pr.clone())
        want = sum(_crand(torch.Generator().manual_seed(r), (5, 5)) for r in range(world))
        assert torch.allclose(tot_t, want, rtol=1e-6, atol=1e-6)
        # batched reductions: one all-reduce for a CG iteration's Dai-Yuan terms
        from ptychotomo_b200.kernels import Reducer
        from ptychotomo_b200.sharded import _GlobalReducer

        class LocalTerms:     # stands in for the device Reducer: rank-dependent partials
            def many(self, ops):
                r = float(rank + 1)
                return Reducer.unpack(ops, [r, -r, 2 * r, 3 * r, 4 * r, 5 * r])
        red = _GlobalReducer(LocalTerms(), comm, None)
        ops = [("dot", None, None), ("norm2", None), ("quad3", None, None)]
        tot = sum(range(1, world + 1))
        assert red.many(ops) == [complex(tot, -tot), 2.0 * tot, (3.0 * tot, 4.0 * tot, 5.0 * tot)]
        # gather
        assert torch.equal(comm.gather(A[th0:th1].contiguous(), 0, comm.theta_ranges), A)
        assert torch.equal(comm.gather(U[:, z0:z1].contiguous(), 1, comm.z_ranges), U)
        dist.barrier()
        dist.destroy_process_group()
    except Exception as e:  # reported to the parent
        import traceback
        errq.put("rank %d: %s\n%s" % (rank, e, traceback.format_exc()))
        raise


@pytest.mark.parametrize("world,ntheta,nz", [(2, 5, 7), (2, 4, 4), (3, 7, 5)])
def test_shard_comm_gloo(world, ntheta, nz):
    ctx = mp.get_context("spawn")
    errq = ctx.SimpleQueue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, ntheta, nz, 6, errq)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    alive = [p for p in procs if p.is_alive()]
    for p in alive:
        p.kill()
    msgs = []
    while not errq.empty():
        msgs.append(errq.get())
    assert not alive, "ranks did not finish"
    assert not msgs, "\n".join(msgs)
    assert all(p.exitcode == 0 for p in procs)


def test_block_ranges():
    from ptychotomo_b200.sharded import block_ranges
    assert block_ranges(7, 2) == [(0, 4), (4, 7)]
    assert block_ranges(6, 3) == [(0, 2), (2, 4), (4, 6)]
    r = block_ranges(384, 8)
    assert r[0] == (0, 48) and r[-1] == (336, 384)
    assert sum(b - a for a, b in block_ranges(100, 7)) == 100
