"""Generate the golden vectors of tests/golden from the reference itself.

Runs the reference's own CUDA operators (built unmodified by
``make -C oracle`` into oracle/_ref) on small seeded inputs on a GPU and
stores inputs and outputs as .npz fixtures.  The polar coordinate tables
that the GPU computes with ``__cosf``/``__sinf`` are stored too (taken from
ptychotomo_b200, whose takexy kernel evaluates the reference's expression),
so the CPU oracle can be pinned to the reference exactly.

    python tests/golden/make_golden.py OUTDIR
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

import torch  # noqa: E402

import refcuda  # noqa: E402
from ptychotomo_b200 import radonusfft  # noqa: E402

RADON_CASES = [(16, 3, 12, 1), (32, 2, 24, 2), (64, 2, 48, 3)]   # n, nz, ntheta, seed
PTYCHO_CASES = [(2, 32, 32, 6, 16, 16, 4), (2, 24, 40, 5, 32, 16, 5)]  # ntheta,nz,n,nscan,det,nprb,seed


def crand(rng, shape):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)


def radon_case(n, nz, ntheta, seed):
    rng = np.random.default_rng(seed)
    theta = np.sort(rng.uniform(0, np.pi, ntheta)).astype(np.float32)
    f = crand(rng, (nz, n, n))
    g = crand(rng, (ntheta, nz, n))
    dev = torch.device("cuda")
    th_d = torch.from_numpy(theta).to(dev)
    f_d = torch.from_numpy(f).to(dev)
    g_d = torch.from_numpy(g).to(dev)
    ref = refcuda.RefRadon(ntheta, nz, n)
    ref.setobj(th_d.data_ptr())
    out_g = torch.zeros((ntheta, nz, n), dtype=torch.complex64, device=dev)
    out_f = torch.zeros((nz, n, n), dtype=torch.complex64, device=dev)
    ref.fwd(out_g.data_ptr(), f_d.data_ptr())
    ref.adj(out_f.data_ptr(), g_d.data_ptr())
    ref.free()
    op = radonusfft(ntheta, nz, n)
    op.setobj(th_d)
    N = n * 3 // 2
    x = torch.empty((ntheta, N), dtype=torch.float32, device=dev)
    y = torch.empty_like(x)
    op.get_xy(x, y)
    torch.cuda.synchronize()
    return dict(theta=theta, f=f, g=g, fwd=out_g.cpu().numpy(), adj=out_f.cpu().numpy(),
                x=x.cpu().numpy(), y=y.cpu().numpy())


def ptycho_case(ntheta, nz, n, nscan, det, nprb, seed):
    rng = np.random.default_rng(seed)
    scan = np.empty((2, ntheta, nscan), np.float32)
    scan[0] = rng.uniform(0, n - nprb - 0.5, (ntheta, nscan))
    scan[1] = rng.uniform(0, nz - nprb - 0.5, (ntheta, nscan))
    scan[:, 0, 1] = -1  # reference sentinel: this scan is skipped
    prb = crand(rng, (nprb, nprb))
    f = crand(rng, (ntheta, nz, n))
    g = crand(rng, (ntheta, nscan, det, det))
    dev = torch.device("cuda")
    sc_d = torch.from_numpy(scan).to(dev)
    pr_d = torch.from_numpy(prb).to(dev)
    f_d = torch.from_numpy(f).to(dev)
    g_d = torch.from_numpy(g).to(dev)
    ref = refcuda.RefPtycho(ntheta, nz, n, nscan, det, nprb)
    ref.setobj(sc_d.data_ptr(), pr_d.data_ptr())
    out_g = torch.zeros((ntheta, nscan, det, det), dtype=torch.complex64, device=dev)
    out_f = torch.zeros((ntheta, nz, n), dtype=torch.complex64, device=dev)
    ref.fwd(out_g.data_ptr(), f_d.data_ptr())
    ref.adj(out_f.data_ptr(), g_d.data_ptr())
    ref.free()
    return dict(scan=scan, prb=prb, f=f, g=g, fwd=out_g.cpu().numpy(), adj=out_f.cpu().numpy())


def main(outdir):
    out = Path(outdir)
    out.mkdir(parents=True, exist_ok=True)
    for c in RADON_CASES:
        d = radon_case(*c)
        np.savez_compressed(out / "radon_n{}_nz{}_nt{}.npz".format(*c[:3]), **d)
    for c in PTYCHO_CASES:
        d = ptycho_case(*c)
        np.savez_compressed(out / "ptycho_nt{}_nz{}_n{}_ns{}_det{}_p{}.npz".format(*c[:6]), **d)
    print("golden vectors written to", out)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else str(Path(__file__).parent))
