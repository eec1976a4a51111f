"""Probe retrieval: the ptycho operator as a linear map of the probe, and the
probe CG of the Solver (no counterpart in the reference, which keeps the
probe fixed).

* pt_ptycho_adj_probe against the oracle's probe adjoint (rel-L2 <= 1e-5) and
  the adjoint identity <fwd_probe(psi, p), g> = <p, adj_probe(g, psi)>;
* fwd_probe equals setobj(probe) + fwd, bit for bit;
* adj_probe_resid equals adj_probe of the residual;
* Solver.cg_probe lowers the data term and moves a perturbed probe towards
  the true one; admm(probe_iter=0) is the plain ADMM, bit for bit.
"""
import numpy as np
import pytest

from oracle.ptycho import PtychoFFT
from ptychotomo_b200 import synthetic

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def crand(rng, shape):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def make(ntheta, nz, n, nscan, det, nprb, rng):
    from ptychotomo_b200 import ptychofft
    scan = np.empty((2, ntheta, nscan), np.float32)
    scan[0] = rng.uniform(0, max(n - nprb - 0.5, 0), (ntheta, nscan))
    scan[1] = rng.uniform(0, max(nz - nprb - 0.5, 0), (ntheta, nscan))
    scan[:, 0, 1] = -1
    prb = crand(rng, (nprb, nprb))
    op = ptychofft(ntheta, nz, n, ntheta, nscan, det, det, nprb)
    op.setobj(dev(scan), dev(prb))
    orc = PtychoFFT(ntheta, nz, n, ntheta, nscan, det, det, nprb)
    orc.setobj(scan, prb)
    return op, orc, scan, prb


SIZES = [(3, 24, 30, 5, 16, 16), (2, 40, 36, 6, 32, 16), (2, 64, 70, 5, 64, 64), (2, 140, 130, 4, 128, 128),
         (2, 110, 100, 5, 128, 96)]


@pytest.mark.parametrize("ntheta,nz,n,nscan,det,nprb", SIZES)
def test_adj_probe_vs_oracle_and_adjoint(ntheta, nz, n, nscan, det, nprb):
    rng = np.random.default_rng(det + nprb)
    op, orc, _, _ = make(ntheta, nz, n, nscan, det, nprb, rng)
    psi = crand(rng, (ntheta, nz, n))
    g = crand(rng, (ntheta, nscan, det, det))
    gp = torch.zeros((nprb, nprb), dtype=torch.complex64, device="cuda")
    op.adj_probe(gp, dev(g), dev(psi), scale=0.7)
    assert rel(gp.cpu().numpy(), 0.7 * orc.adj_probe(g, psi)) <= 1e-5
    p = dev(crand(rng, (nprb, nprb)))
    fp = torch.zeros((ntheta, nscan, det, det), dtype=torch.complex64, device="cuda")
    op.fwd_probe(fp, dev(psi), p, scale=0.7)
    a = torch.vdot(fp.flatten().cdouble(), dev(g).flatten().cdouble()).item()
    b = torch.vdot(p.flatten().cdouble(), gp.flatten().cdouble()).item()
    assert abs(a - b) / abs(a) <= 1e-5
    gp2 = torch.zeros_like(gp)
    op.adj_probe(gp2, dev(g), dev(psi), scale=0.7)
    assert torch.equal(gp, gp2)   # deterministic


def test_fwd_probe_is_setobj_then_fwd():
    from ptychotomo_b200 import ptychofft
    rng = np.random.default_rng(3)
    op, _, scan, _ = make(2, 140, 130, 4, 128, 96, rng)
    psi = dev(crand(rng, (2, 140, 130)))
    p = crand(rng, (96, 96))
    a = torch.zeros((2, 4, 128, 128), dtype=torch.complex64, device="cuda")
    op.fwd_probe(a, psi, dev(p), scale=0.5)
    op2 = ptychofft(2, 140, 130, 2, 4, 128, 128, 96)
    op2.setobj(dev(scan), dev(p))
    b = torch.zeros_like(a)
    op2.fwd(b, psi, scale=0.5)
    assert torch.equal(a, b)


@pytest.mark.parametrize("model", [0, 1])
def test_adj_probe_resid(model):
    from ptychotomo_b200 import kernels
    rng = np.random.default_rng(8 + model)
    op, _, _, _ = make(2, 64, 70, 5, 64, 64, rng)
    psi = dev(crand(rng, (2, 64, 70)))
    fpsi = dev(crand(rng, (2, 5, 64, 64)))
    data = dev(rng.poisson(2.0, (2, 5, 64, 64)).astype(np.float32))
    res = kernels.residual(torch.empty_like(fpsi), fpsi, data, 0.6, model)
    a = torch.zeros((64, 64), dtype=torch.complex64, device="cuda")
    op.adj_probe(a, res, psi, scale=0.3)
    b = torch.zeros_like(a)
    op.adj_probe_resid(b, psi, fpsi, data, 0.6, model, scale=0.3)
    assert rel(b.cpu().numpy(), a.cpu().numpy()) <= 1e-6


def test_adj_probe_rejects_det8():
    from ptychotomo_b200 import PtychotomoError
    rng = np.random.default_rng(1)
    op, _, _, _ = make(2, 20, 20, 3, 8, 8, rng)
    with pytest.raises(PtychotomoError, match="detector 8"):
        op.adj_probe(torch.zeros((8, 8), dtype=torch.complex64, device="cuda"),
                     torch.zeros((2, 3, 8, 8), dtype=torch.complex64, device="cuda"),
                     torch.zeros((2, 20, 20), dtype=torch.complex64, device="cuda"))


def _problem():
    from ptychotomo_b200 import Solver
    n = nz = 32
    ntheta, nprb = 8, 16
    theta = synthetic.angles(ntheta)
    prb = synthetic.probe(nprb, seed=1)
    scan = synthetic.raster_scan(ntheta, 4, n, nz, nprb)
    scan[0] += np.float32(0.3)
    obj = synthetic.phantom(n, nz, seed=2)
    slv = Solver(prb, scan, theta, [16, 16], 1e-6, 5.0, ntheta, nz, n, ntheta, nz)
    psi = slv.exptomo(slv.fwd_tomo_batch(dev(obj)))
    data = slv.fwd_ptycho_batch(psi)
    return slv, prb, psi, data, obj


@pytest.mark.parametrize("model", ["poisson", "gaussian"])
def test_cg_probe_recovers_perturbed_probe(model):
    slv, prb, psi, data, _ = _problem()
    rng = np.random.default_rng(5)
    p0 = (0.8 * prb * np.exp(0.3j) + 0.02 * crand(rng, prb.shape)).astype(np.complex64)
    slv.set_probe(p0)

    def misfit(p):
        slv.set_probe(p)
        return slv.red.lagr_frames(slv.fwd_ptycho(psi), data, slv.coefdata, 0 if model == "poisson" else 1)

    before = misfit(p0)
    p = slv.cg_probe(data, psi, dev(p0), 12, model)
    after = misfit(p)
    assert np.isfinite(after) and after < 0.5 * before
    # the data constrain the probe up to a global phase
    pc = p.cpu().numpy()
    ph = np.vdot(pc, prb) / abs(np.vdot(pc, prb))
    assert rel(pc * ph, prb) < rel(p0 * np.vdot(p0, prb) / abs(np.vdot(p0, prb)), prb)


def test_admm_probe_iter_zero_is_plain_admm():
    slv, prb, psi, data, obj = _problem()
    c = dict(dtype=torch.complex64, device="cuda")

    def run(**kw):
        slv.set_probe(prb)
        ones = torch.ones((8, 32, 32), **c)
        z3 = torch.zeros((3, 32, 32, 32), **c)
        return slv.admm(data, ones.clone(), z3.clone(), ones.clone(), z3.clone(), torch.zeros_like(ones), z3.clone(),
                        torch.zeros((32, 32, 32), **c), 1e-3, 4, 4, 2, "poisson", verbose=False, **kw)

    u0, p0 = run()
    u1, p1 = run(probe_iter=0)
    assert torch.equal(u0, u1) and torch.equal(p0, p1)
    u2, p2 = run(probe_iter=2)
    assert torch.isfinite(u2).all() and torch.isfinite(slv.prb).all()
    assert not torch.equal(slv.prb, dev(prb))
