"""Sub-pixel scan model of ptychofft (set_subpixel; no counterpart in the
reference, which rounds each scan to the grid and applies a constant phase,
kernels.cuh:306-336).

* fwd and adj with fractional scans against the oracle (probe shifted by the
  Fourier shift theorem in complex128), rel-L2 <= 1e-5, for the det-128
  kernels with a full and a padded probe and for the generic det-64 kernels;
  the adjoint identity to 1e-5.
* Integer scans: the shifted probe tables equal the probe, so the frames are
  bit-identical to the reference model's (whose phase is then 1).
* quant = 0 restores the reference model bit for bit; setobj rebuilds the
  tables; the fused residual adjoint follows the model; probe retrieval is
  refused while it is on.
* The point of the model: moving a scan across the rounding boundary
  (x.49 -> x.51) changes its intensities by a fraction of what the reference
  model's one-pixel jump does.
"""
import numpy as np
import pytest

from oracle.ptycho import PtychoFFT

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def crand(rng, shape):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)


def T(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def gauss_probe(P, sigma, rng):
    y, x = np.mgrid[:P, :P] - (P - 1) / 2
    amp = np.exp(-(x ** 2 + y ** 2) / (2 * sigma ** 2))
    return (amp * np.exp(1j * 0.3 * rng.standard_normal((P, P)))).astype(np.complex64)


def setup(rng, nt, ns, nz, n, det, P, frac=True):
    scan = np.stack([rng.uniform(0.6, n - P - 0.6, (nt, ns)), rng.uniform(0.6, nz - P - 0.6, (nt, ns))])
    if not frac:
        scan = np.round(scan)
    return scan.astype(np.float32), crand(rng, (P, P))


@pytest.mark.parametrize("det,P,quant", [(128, 128, 64), (128, 100, 1024), (64, 48, 16)])
def test_subpixel_matches_oracle(det, P, quant):
    from ptychotomo_b200 import ptychofft
    rng = np.random.default_rng(det + P)
    nt, ns = 3, 7
    nz = n = P + 24
    scan, prb = setup(rng, nt, ns, nz, n, det, P)
    op = ptychofft(nt, nz, n, nt, ns, det, det, P)
    op.setobj(T(scan), T(prb))
    op.set_subpixel(quant)
    q, ntab = op.subpixel
    assert q == quant and 1 <= ntab <= nt * ns
    orc = PtychoFFT(nt, nz, n, nt, ns, det, det, P)
    orc.setobj(scan, prb)
    orc.set_subpixel(quant)
    f = crand(rng, (nt, nz, n))
    g = torch.empty((nt, ns, det, det), dtype=torch.complex64, device="cuda")
    op.fwd(g, T(f))
    assert rel(g.cpu().numpy(), orc.fwd(f)) <= 1e-5
    d = crand(rng, (nt, ns, det, det))
    fa = torch.empty((nt, nz, n), dtype=torch.complex64, device="cuda")
    op.adj(fa, T(d))
    assert rel(fa.cpu().numpy(), orc.adj(d)) <= 1e-5
    # adjoint identity on the device results
    lhs = np.vdot(d.astype(np.complex128), g.cpu().numpy().astype(np.complex128))
    rhs = np.vdot(fa.cpu().numpy().astype(np.complex128), f.astype(np.complex128))
    assert abs(lhs - rhs) / abs(lhs) <= 1e-5


def test_integer_scans_are_the_reference_model():
    from ptychotomo_b200 import ptychofft
    rng = np.random.default_rng(5)
    nt, ns, det, P = 2, 5, 128, 128
    nz = n = 160
    scan, prb = setup(rng, nt, ns, nz, n, det, P, frac=False)
    a = ptychofft(nt, nz, n, nt, ns, det, det, P)
    a.setobj(T(scan), T(prb))
    b = ptychofft(nt, nz, n, nt, ns, det, det, P)
    b.setobj(T(scan), T(prb))
    b.set_subpixel(32)
    assert b.subpixel == (32, 1)
    f = T(crand(rng, (nt, nz, n)))
    ga, gb = (torch.empty((nt, ns, det, det), dtype=torch.complex64, device="cuda") for _ in range(2))
    a.fwd(ga, f)
    b.fwd(gb, f)
    assert torch.equal(ga, gb)


def test_switching_and_rebuilding():
    from ptychotomo_b200 import PtychotomoError, ptychofft
    rng = np.random.default_rng(6)
    nt, ns, det, P = 2, 6, 128, 128
    nz = n = 150
    scan, prb = setup(rng, nt, ns, nz, n, det, P)
    op = ptychofft(nt, nz, n, nt, ns, det, det, P)
    op.setobj(T(scan), T(prb))
    f = T(crand(rng, (nt, nz, n)))
    g0, g1, g2 = (torch.empty((nt, ns, det, det), dtype=torch.complex64, device="cuda") for _ in range(3))
    op.fwd(g0, f)
    op.set_subpixel(64)
    op.fwd(g1, f)
    assert not torch.equal(g0, g1)
    op.set_subpixel(0)
    assert op.subpixel == (0, 0)
    op.fwd(g2, f)
    assert torch.equal(g0, g2)
    # setobj with new scans and probe rebuilds the tables (matches a fresh handle)
    op.set_subpixel(64)
    scan2, prb2 = setup(rng, nt, ns, nz, n, det, P)
    op.setobj(T(scan2), T(prb2))
    fresh = ptychofft(nt, nz, n, nt, ns, det, det, P)
    fresh.setobj(T(scan2), T(prb2))
    fresh.set_subpixel(64)
    op.fwd(g1, f)
    fresh.fwd(g2, f)
    assert torch.equal(g1, g2)
    # the fused residual adjoint follows the model: equals adj of the residual formed in torch
    data = (g1.abs() ** 2 * 0.9).float().contiguous()
    fa, fb = (torch.empty((nt, nz, n), dtype=torch.complex64, device="cuda") for _ in range(2))
    op.adj_resid(fa, g1, data, 1.0, 0)
    resid = g1 - data * g1 / (g1.abs() ** 2 + 1e-32)
    op.adj(fb, resid.contiguous())
    assert float(torch.linalg.vector_norm(fa - fb) / torch.linalg.vector_norm(fb)) <= 1e-5
    gp = torch.empty((P, P), dtype=torch.complex64, device="cuda")
    with pytest.raises(PtychotomoError):
        op.adj_probe(gp, g1, f)


def test_boundary_crossing_is_continuous():
    """A scan moved from x + 0.49 to x + 0.51: the reference model jumps a
    whole pixel (its per-scan phase leaves intensities unchanged); the
    sub-pixel model moves the probe by 0.02 pixel."""
    from ptychotomo_b200 import ptychofft
    rng = np.random.default_rng(7)
    nt, ns, det, P = 1, 2, 64, 64
    nz = n = 96
    prb = gauss_probe(P, 10.0, rng)
    x0, y0 = 15.0, 17.0
    scan = np.array([[[x0 + 0.49, x0 + 0.51]], [[y0, y0]]], np.float32)
    f = np.exp(1j * rng.uniform(-1, 1, (nt, nz, n)) + 0.2 * rng.standard_normal((nt, nz, n))).astype(np.complex64)
    jumps = {}
    for quant in (0, 256):
        op = ptychofft(nt, nz, n, nt, ns, det, det, P)
        op.setobj(T(scan), T(prb))
        if quant:
            op.set_subpixel(quant)
        g = torch.empty((nt, ns, det, det), dtype=torch.complex64, device="cuda")
        op.fwd(g, T(f))
        inten = (g.abs() ** 2).cpu().numpy()[0]
        jumps[quant] = np.linalg.norm(inten[1] - inten[0]) / np.linalg.norm(inten[0])
    print("intensity change across the rounding boundary:", jumps)
    assert jumps[256] < 0.1 * jumps[0]


def test_solver_option():
    from ptychotomo_b200 import Solver, synthetic
    nt, n, P = 4, 64, 16
    theta = synthetic.angles(nt)
    scan = synthetic.raster_scan(nt, 3, n, n, P) + np.float32(0.3)
    slv = Solver(synthetic.probe(P, seed=1), scan, theta, [P, P], 1e-6, 5.0, nt, n, n, nt, n, subpixel=32)
    assert slv.subpixel == 32 and slv.cl_ptycho.subpixel[0] == 32


def test_solver_with_subpixel_scans_matches_oracle():
    """The Solver's ptycho forward and its Poisson CG under the sub-pixel
    model against the oracle Solver whose operator runs the same model
    (the CG to 1e-3, as for the reference model)."""
    from oracle.solver import Solver as OSolver
    from ptychotomo_b200 import Solver, synthetic
    n = nz = 32
    nt, P, quant = 8, 16, 64
    theta = synthetic.angles(nt)
    prb = synthetic.probe(P, seed=1)
    scan = synthetic.raster_scan(nt, 3, n, nz, P)
    scan[0] += np.float32(0.3)
    scan[1] += np.float32(0.45)
    obj = synthetic.phantom(n, nz, seed=2)
    args = (prb, scan, theta, [P, P], 1e-6, 5.0, nt, nz, n, nt, nz)
    gs = Solver(*args, subpixel=quant)
    x = torch.empty((nt, gs.cl_tomo.N), dtype=torch.float32, device="cuda")
    y = torch.empty_like(x)
    gs._tomo_all.get_xy(x, y)
    os_ = OSolver(*args, xy=(x.cpu().numpy(), y.cpu().numpy()))
    os_.cl_ptycho.set_subpixel(quant)
    psi = os_.exptomo(os_.fwd_tomo_batch(obj))
    want = os_.fwd_ptycho_batch(psi)
    got = gs.fwd_ptycho_batch(T(psi))
    assert rel(got.cpu().numpy(), want) <= 1e-5
    data = np.random.default_rng(3).poisson(want * 1e3).astype(np.float32) / np.float32(1e3)
    psi0 = np.ones((nt, nz, n), np.complex64)
    h, lamd = np.ones_like(psi0), np.zeros_like(psi0)
    pg = gs.cg_ptycho_batch(T(data), T(psi0), T(h), T(lamd), 0.5, 4, "poisson")
    po = os_.cg_ptycho_batch(data, psi0, h, lamd, 0.5, 4, "poisson")
    assert rel(pg.cpu().numpy(), po) < 1e-3


def test_subpixel_with_skipped_scans():
    """Sentinel scans (-1, the reference's 'no frame') under the sub-pixel
    model: their frames stay zero and the rest match the oracle."""
    from ptychotomo_b200 import ptychofft
    rng = np.random.default_rng(9)
    nt, ns, det, P = 2, 6, 128, 128
    nz = n = 150
    scan, prb = setup(rng, nt, ns, nz, n, det, P)
    scan[:, 0, 2] = -1
    scan[:, 1, 4] = -1
    op = ptychofft(nt, nz, n, nt, ns, det, det, P)
    op.setobj(T(scan), T(prb))
    op.set_subpixel(32)
    orc = PtychoFFT(nt, nz, n, nt, ns, det, det, P)
    orc.setobj(scan, prb)
    orc.set_subpixel(32)
    f = crand(rng, (nt, nz, n))
    g = torch.empty((nt, ns, det, det), dtype=torch.complex64, device="cuda")
    op.fwd(g, T(f))
    gn = g.cpu().numpy()
    assert not gn[0, 2].any() and not gn[1, 4].any()
    assert rel(gn, orc.fwd(f)) <= 1e-5
    fa = torch.empty((nt, nz, n), dtype=torch.complex64, device="cuda")
    d = crand(rng, (nt, ns, det, det))
    op.adj(fa, T(d))
    assert rel(fa.cpu().numpy(), orc.adj(d)) <= 1e-5
