"""GPU checks of the learned preconditioner's parts and of the preconditioned
tomography CG.

* radonusfft.adj_exact against the oracle's exact adjoint (rel-L2 <= 1e-5)
  and the adjoint identity <R f, g> = <f, R^T g> with inputs that do not
  vanish on their borders (<= 1e-5; the reference's adjoint is off by
  > 1e-2 there);
* the diagonal of R^T R against unit-pixel forwards of the oracle, the
  features against their definition, the filter against a NumPy evaluation
  of D^-1/2 F2^-1 p F2 D^-1/2, the phase probes and spectrum statistics;
* the preconditioned CG keeps the subproblem's minimiser (plain CG, run
  long, judges it: rel-L2 <= 1e-3) and reaches a 1e-4 gradient reduction in
  fewer iterations than plain CG, with a network trained by the library's
  kernels on the symbol measured with random-phase probes (training and
  held-out probe sets).
"""
import numpy as np
import pytest

from oracle.usfft import RadonUSFFT

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def rel(a, b):
    a = a.cpu().numpy() if hasattr(a, "cpu") else np.asarray(a)
    b = b.cpu().numpy() if hasattr(b, "cpu") else np.asarray(b)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def crand(rng, shape):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)


def T(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def radon(n, nz, theta):
    from ptychotomo_b200 import radonusfft
    op = radonusfft(len(theta), nz, n)
    op.setobj(T(theta))
    x = torch.empty((len(theta), op.N), dtype=torch.float32, device="cuda")
    y = torch.empty_like(x)
    op.get_xy(x, y)
    orc = RadonUSFFT(len(theta), nz, n)
    orc.setobj(theta, xy=(x.cpu().numpy(), y.cpu().numpy()))
    return op, orc


@pytest.mark.parametrize("n,nz,nt", [(32, 5, 24), (64, 3, 40), (128, 2, 60)])
def test_exact_adjoint_vs_oracle_and_identity(n, nz, nt):
    rng = np.random.default_rng(n)
    theta = np.sort(rng.uniform(-np.pi / 3, np.pi / 3, nt)).astype(np.float32)
    op, orc = radon(n, nz, theta)
    f, g = crand(rng, (nz, n, n)), crand(rng, (nt, nz, n))
    fa = torch.empty((nz, n, n), dtype=torch.complex64, device="cuda")
    op.adj_exact(fa, T(g), scale=0.5)
    assert rel(fa, 0.5 * orc.adj_exact(g)) <= 1e-5
    gf = torch.empty((nt, nz, n), dtype=torch.complex64, device="cuda")
    op.fwd(gf, T(f))
    op.adj_exact(fa, T(g))
    a = np.vdot(gf.cpu().numpy().astype(np.complex128), g.astype(np.complex128))
    b = np.vdot(f.astype(np.complex128), fa.cpu().numpy().astype(np.complex128))
    assert abs(a - b) / abs(a) <= 1e-5


def _precond(n, nz, theta, scale=0.7):
    from ptychotomo_b200.learned import FourierPreconditioner
    op, orc = radon(n, nz, theta)
    pre = FourierPreconditioner(op, T(theta), scale, "cuda")
    return op, orc, pre


def test_diagonal_matches_unit_pixel_forwards():
    n, nz = 32, 4
    theta = np.linspace(-np.pi / 3, np.pi / 3, 30, endpoint=False).astype(np.float32)
    op, orc, pre = _precond(n, nz, theta, scale=0.7)
    d, dI = pre.diag()
    d = d.cpu().numpy()
    for (y, x) in [(0, 0), (0, 7), (n - 1, 3), (5, 0), (9, n - 1), (n // 2, n // 2)]:
        e = np.zeros((nz, n, n))
        e[0, y, x] = 1
        ref = 0.49 * np.linalg.norm(orc.fwd(e)[:, 0]) ** 2
        assert abs(d[y, x] - ref) <= 1e-5 * ref, (y, x, d[y, x], ref)
    assert d[3, 4] == dI and d[n // 2, n // 2] == dI


def test_features_follow_their_definition():
    n = 32
    theta = np.linspace(-np.pi / 3, np.pi / 3, 60, endpoint=False).astype(np.float32)
    _, _, pre = _precond(n, 2, theta)
    x = pre.x.cpu().numpy()
    k = np.fft.fftfreq(n) * n
    ky, kx = np.meshgrid(k, k, indexing="ij")
    r = np.hypot(kx, ky).ravel() / (n / 2)
    phi = np.mod(np.arctan2(ky, kx), np.pi).ravel()
    phi[0] = 0.0
    psi = np.mod(-theta.astype(np.float64), np.pi)
    dd = np.abs(phi[:, None] - psi[None, :])
    dd = np.minimum(dd, np.pi - dd)
    dens = (dd <= np.pi / 60).sum(1) / (2 * (np.pi / 60) * len(theta) / np.pi)
    gap = dd.min(1) / (np.pi / 2)
    np.testing.assert_allclose(x[:, 0], r, rtol=1e-6, atol=1e-6)
    np.testing.assert_allclose(x[:, 1], dens, rtol=1e-5, atol=1e-5)
    np.testing.assert_allclose(x[:, 2], gap, rtol=1e-5, atol=1e-6)
    assert x[:, 2].max() > 0.3    # a 60-degree missing wedge


def test_filter_matches_numpy():
    n, nz = 64, 3
    theta = np.linspace(0, np.pi, 48, endpoint=False).astype(np.float32)
    _, _, pre = _precond(n, nz, theta)
    rng = np.random.default_rng(1)
    loga = rng.uniform(-3, 0, (n, n)).astype(np.float32)
    pre.set_log_symbol(T(loga))
    g = crand(rng, (nz, n, n))
    rk, tau = 0.37, 0.11
    out = torch.empty((nz, n, n), dtype=torch.complex64, device="cuda")
    pre.apply(out, T(g), rk, tau)
    dR, dI = pre.diag()
    dR = dR.cpu().numpy().astype(np.float64)
    cnt = lambda m: np.array([(i > 0) + (i < m - 1) for i in range(m)], float)  # noqa: E731
    dJ = (4 / 3) * (cnt(nz)[:, None, None] + cnt(n)[None, :, None] + cnt(n)[None, None, :])
    D = rk * dR[None] + tau * dJ
    kf = np.fft.fftfreq(n)
    sy, sx = np.meshgrid(np.sin(np.pi * kf), np.sin(np.pi * kf), indexing="ij")
    j = (4 / 3) * (4 * sx ** 2 + 4 * sy ** 2 + 2)
    p = (rk * dI + tau * (4 / 3) * 6) / (rk * np.exp(loga.astype(np.float64)) + tau * j)
    ref = np.fft.ifft2(np.fft.fft2(g / np.sqrt(D)) * p[None]) / np.sqrt(D)
    assert rel(out, ref) <= 1e-5


def test_phase_probe_keeps_the_modulus_spectrum_and_statistics():
    n, nz = 32, 4
    theta = np.linspace(0, np.pi, 20, endpoint=False).astype(np.float32)
    _, _, pre = _precond(n, nz, theta)
    rng = np.random.default_rng(2)
    r = T(crand(rng, (nz, n, n)))
    z = torch.empty_like(r)
    pre.phase_probe(z, r, 7)
    zn = z.cpu().numpy()
    np.testing.assert_allclose(np.abs(np.fft.fft2(zn)), np.abs(np.fft.fft2(r.cpu().numpy())), rtol=1e-4, atol=1e-4)
    z2 = torch.empty_like(r)
    pre.phase_probe(z2, r, 7)
    assert torch.equal(z, z2)
    az = T(crand(rng, (nz, n, n)))
    num = torch.zeros((n, n), dtype=torch.float64, device="cuda")
    den = torch.zeros_like(num)
    pre.spectrum(num, den, z, az)
    Z, AZ = np.fft.fft2(zn), np.fft.fft2(az.cpu().numpy())
    assert rel(num, np.real(np.conj(Z) * AZ).sum(0)) <= 1e-5
    assert rel(den, (np.abs(Z) ** 2).sum(0)) <= 1e-5


@pytest.fixture(scope="module")
def wedge_problem():
    """A tomography subproblem with a 60-degree missing wedge: 64 wide, 16
    slices, 90 angles on [-60, 60) degrees, K = 1, xi0 = R u of a phantom."""
    from ptychotomo_b200 import Solver, synthetic
    n, nz, nt = 64, 16, 90
    theta = synthetic.angles(nt, -np.pi / 3, np.pi / 3)
    prb = synthetic.probe(16, seed=1)
    scan = synthetic.raster_scan(nt, 2, n, nz, 16)
    slv = Solver(prb, scan, theta, [16, 16], 1e-6, 5.0, nt, nz, n, nt, nz)
    return slv, theta


def _subproblem(slv, seed, tau_data=0.0):
    from ptychotomo_b200 import synthetic
    n, nz, nt = slv.n, slv.nz, slv.ntheta
    u = T(synthetic.phantom(n, nz, seed=seed) * 1e5)
    xi0 = slv.fwd_tomo_batch(u)
    Kt = torch.ones_like(xi0)
    xi1 = torch.zeros((3, nz, n, n), dtype=torch.complex64, device="cuda")
    return xi0, xi1, Kt


def test_pcg_keeps_the_minimiser_and_trained_network_gains(wedge_problem):
    from ptychotomo_b200 import synthetic
    from ptychotomo_b200.learned import FourierPreconditioner, harvest_targets, train_network
    slv, theta = wedge_problem
    n, nz = slv.n, slv.nz
    pre = FourierPreconditioner(slv._tomo_all, T(theta), slv.coeftomo, "cuda")
    tg = harvest_targets(slv._tomo_all, pre, range(100, 112), probes=4)
    net, hist, train_loss, held = train_network(pre.x, tg[:8], tg[8:], steps=800, lr=1e-2, lr_final=1e-3, seed=0)
    print("loss history", hist, "held-out", held)
    assert hist[-1][1] < 0.5 * hist[0][1], hist
    assert held < 1.5 * train_loss, (train_loss, held)
    pre.set_network(net)
    xi0, xi1, Kt = _subproblem(slv, seed=7)
    u0 = torch.zeros((nz, n, n), dtype=torch.complex64, device="cuda")
    rho, tau = 0.5, 0.05
    ustar, _ = slv.pcg_tomo(xi0, xi1, Kt, u0, rho, tau, 600, None, tol=1e-7)
    hp, hq = [], []
    up, _ = slv.pcg_tomo(xi0, xi1, Kt, u0, rho, tau, 400, None, tol=1e-4, history=hp)
    uq, _ = slv.pcg_tomo(xi0, xi1, Kt, u0, rho, tau, 400, pre, tol=1e-4, history=hq)
    print("iterations to 1e-4: plain", len(hp), "learned", len(hq), "train/held-out loss", train_loss, held)
    uq2, _ = slv.pcg_tomo(xi0, xi1, Kt, u0, rho, tau, 200, pre, tol=1e-7)
    assert rel(uq2, ustar) <= 1e-3
    assert len(hq) < len(hp), (len(hq), len(hp))
