"""Parity at the sizes the benchmarks are quoted on.

* radonusfft at n = 256 with the bench's 384 angles on [0, pi) (3 slices, so
  the NumPy oracle stays fast): fwd and adj against the oracle, and the
  adjoint identity, at rel-L2 <= 1e-5;
* ptychofft at the bench geometry: a 256 x 256 object, 13 x 13 scans at
  linspace(0, 256 - 128, 13), 128^2 probe and detector, 3 angles: fwd, adj
  and the Poisson-residual adjoint against the oracle at rel-L2 <= 1e-5;
* the plain ADMM of the small configuration (128 wide, 128 angles on
  [0, pi), 64^2 probe, 7-column raster with step 10, 1e3 photons, TV 1e-3,
  4 CG iterations per subproblem) on a slab of 84 slices (3 scan rows), with
  u and psi compared directly with the oracle Solver after every iteration.
"""
import numpy as np
import pytest

from oracle.ptycho import PtychoFFT
from oracle.solver import Solver as OSolver
from oracle.usfft import RadonUSFFT
from ptychotomo_b200 import synthetic

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TOL = 1e-5


def rel(a, b):
    a = a.cpu().numpy() if hasattr(a, "cpu") else np.asarray(a)
    return float(np.linalg.norm(a - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def crand(rng, shape):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)


def T(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def test_radon_n256_384_angles_vs_oracle():
    from ptychotomo_b200 import radonusfft
    n, nz, nt = 256, 3, 384
    theta = synthetic.angles(nt)
    op = radonusfft(nt, nz, n)
    op.setobj(T(theta))
    x = torch.empty((nt, op.N), dtype=torch.float32, device="cuda")
    y = torch.empty_like(x)
    op.get_xy(x, y)
    orc = RadonUSFFT(nt, nz, n)
    orc.setobj(theta, xy=(x.cpu().numpy(), y.cpu().numpy()))
    rng = np.random.default_rng(256)
    f = crand(rng, (nz, n, n))
    f[:, 0, :] = f[:, -1, :] = f[:, :, 0] = f[:, :, -1] = 0     # border-zero for the adjoint identity
    g = crand(rng, (nt, nz, n))
    g[:, :, 0] = g[:, :, -1] = 0
    gd = torch.empty((nt, nz, n), dtype=torch.complex64, device="cuda")
    fd = torch.empty((nz, n, n), dtype=torch.complex64, device="cuda")
    op.fwd(gd, T(f))
    op.adj(fd, T(g))
    assert rel(gd, orc.fwd(f)) <= TOL
    assert rel(fd, orc.adj(g)) <= TOL
    a = np.vdot(gd.cpu().numpy().astype(np.complex128), g.astype(np.complex128))
    b = np.vdot(f.astype(np.complex128), fd.cpu().numpy().astype(np.complex128))
    assert abs(a - b) / abs(a) <= TOL


def test_ptycho_bench_geometry_vs_oracle():
    from ptychotomo_b200 import ptychofft
    n = nz = 256
    nt, P, nside = 3, 128, 13
    scan = synthetic.raster_scan(nt, nside, n, nz, P)       # linspace(0, 128, 13): 10.67 px steps
    prb = synthetic.probe(P, seed=1)
    rng = np.random.default_rng(13)
    psi = np.exp(1j * 0.3 * rng.standard_normal((nt, nz, n))).astype(np.complex64)
    S = nside * nside
    op = ptychofft(nt, nz, n, nt, S, P, P, P)
    op.setobj(T(scan), T(prb))
    orc = PtychoFFT(nt, nz, n, nt, S, P, P, P)
    orc.setobj(scan, prb)
    frames = torch.empty((nt, S, P, P), dtype=torch.complex64, device="cuda")
    op.fwd(frames, T(psi))
    ref = orc.fwd(psi)
    assert rel(frames, ref) <= TOL
    back = torch.empty((nt, nz, n), dtype=torch.complex64, device="cuda")
    op.adj(back, frames)
    assert rel(back, orc.adj(ref)) <= TOL
    # the CG gradient: Poisson residual formed on load, then the adjoint
    data = (np.abs(ref) ** 2 * rng.uniform(0.5, 1.5, ref.shape)).astype(np.float32)
    op.adj_resid(back, frames, T(data), 1.0, 0)
    resid = ref - data * ref / (np.abs(ref) ** 2 + 1e-32)
    assert rel(back, orc.adj(resid)) <= TOL


CFG1_SLAB = dict(n=128, nz=84, ntheta=128, nprb=64, cols=7, step=10.0, photons=1e3, alpha=1e-3)


def _cfg1_slab():
    c = CFG1_SLAB
    n, nz, nt, P = c["n"], c["nz"], c["ntheta"], c["nprb"]
    rows = (nz - P) // int(c["step"]) + 1                     # rows at y = 0, 10, 20
    scan = synthetic.raster_scan(nt, c["cols"], n, nz, P, step=c["step"])
    scan = scan.reshape(2, nt, c["cols"], c["cols"])[:, :, :rows].reshape(2, nt, -1).copy()
    return synthetic.angles(nt), synthetic.probe(P, seed=1), scan, synthetic.phantom(n, nz, seed=2)


def test_admm_cfg1_slab_lockstep_matches_oracle():
    """Plain Poisson ADMM with 4 CG iterations per subproblem (36 ptycho CG
    steps in iterations 0 and 1, as solver.py:315), both Solvers on the same
    counts and tables, 6 iterations.  Lock-step: each iteration of the oracle
    starts from the GPU Solver's state before that iteration, and u, psi and
    the penalties after it are compared directly.

    Iterations 0 and 1 start from psi = 1: there the Poisson steps are
    ~2^-17 and each CG ends when gamma halves below 1e-12, so where the
    36-step CG stops is decided by data-term decreases within FP32 rounding
    of zero (any two FP32 implementations, and the reference against itself
    with its float atomics, stop at different steps).  psi then agrees to
    2e-3, and u, the tomography response to psi - 1 (itself ~1e-3), is not
    compared.  From iteration 2 on, every line search is decisive: psi
    rel-L2 <= 1e-5 and u <= 1e-4 (measured: ~2e-7 and ~2e-5).  The penalty
    schedule must agree exactly throughout."""
    from ptychotomo_b200 import Solver
    c = CFG1_SLAB
    n, nz, nt, P = c["n"], c["nz"], c["ntheta"], c["nprb"]
    theta, prb, scan, obj = _cfg1_slab()
    args = (prb, scan, theta, [P, P], 1e-6, 5.0, nt, nz, n, nt, nz)
    gs = Solver(*args)
    x = torch.empty((nt, gs.cl_tomo.N), dtype=torch.float32, device="cuda")
    y = torch.empty_like(x)
    gs._tomo_all.get_xy(x, y)
    os_ = OSolver(*args, xy=(x.cpu().numpy(), y.cpu().numpy()))
    inten = os_.fwd_ptycho_batch(os_.exptomo(os_.fwd_tomo_batch(obj)))
    sc = c["photons"] / float(inten.mean())
    data = (np.random.default_rng(3).poisson(inten * sc) / sc).astype(np.float32)
    data_d = T(data)
    one = np.ones((nt, nz, n), np.complex64)
    z3 = np.zeros((3, nz, n, n), np.complex64)
    st = {k: T(v) for k, v in dict(u=np.zeros((nz, n, n), np.complex64), psi=one, h=one, e=z3, phi=z3,
                                   lamd=np.zeros_like(one), mu=z3).items()}
    rho = tau = 0.5
    errs = []
    for m in range(6):
        st_o, ro, to = os_.admm_step(m, {k: v.cpu().numpy() for k, v in st.items()}, rho, tau, data, c["alpha"],
                                     4, 4, "poisson")
        st, rho, tau = gs.admm_step(m, st, rho, tau, data_d, c["alpha"], 4, 4, "poisson")
        errs.append((m, rel(st["psi"], st_o["psi"]), rel(st["u"], st_o["u"]), (rho, tau), (ro, to)))
    print("lock-step (m, psi err, u err, penalties gpu, oracle):", errs)
    for m, ep, eu, pg, po in errs:
        assert pg == po, errs
        if m < 2:
            assert ep <= 2e-3, errs
        else:
            assert ep <= 1e-5, errs
            assert eu <= 1e-4, errs
