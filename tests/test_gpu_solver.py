"""GPU Solver (ptychotomo_b200.Solver) against the oracle Solver (oracle/solver.py,
the NumPy restatement of src/ptychotomo/solver.py) on the same seeded small
problem.  Tolerances: single operators / maps 1e-5 relative L2; CG and ADMM
trajectories 1e-3 (FP32 arithmetic on both paths differs at ~1e-6 per step and
the line-search step lengths are discrete)."""
import numpy as np
import pytest

from oracle.solver import Solver as OSolver
from ptychotomo_b200 import synthetic

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def rel(a, b):
    a = a.cpu().numpy() if hasattr(a, "cpu") else np.asarray(a)
    b = np.asarray(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def T(a, dtype=None):
    t = torch.from_numpy(np.ascontiguousarray(a)).cuda()
    return t if dtype is None else t.to(dtype)


@pytest.fixture(scope="module")
def problem():
    from ptychotomo_b200 import Solver
    n = nz = 32
    ntheta, nprb = 16, 16
    theta = synthetic.angles(ntheta)
    prb = synthetic.probe(nprb, seed=1)
    scan = synthetic.raster_scan(ntheta, 3, n, nz, nprb)          # positions 0, 8, 16
    scan[0] += np.float32(0.3)                                     # sub-pixel phase ramp
    obj = synthetic.phantom(n, nz, seed=2)
    args = (prb, scan, theta, [16, 16], 1e-6, 5.0, ntheta, nz, n, ntheta // 2, nz // 2)
    gs = Solver(*args)
    x = torch.empty((ntheta, gs.cl_tomo.N), dtype=torch.float32, device="cuda")
    y = torch.empty_like(x)
    gs._tomo_all.get_xy(x, y)
    os_ = OSolver(*args, xy=(x.cpu().numpy(), y.cpu().numpy()))
    psi_true = os_.exptomo(os_.fwd_tomo_batch(obj))
    data = os_.fwd_ptycho_batch(psi_true)
    data = np.random.default_rng(3).poisson(data * 1e3).astype(np.float32) / np.float32(1e3)
    return dict(gs=gs, os=os_, obj=obj, data=data, n=n, nz=nz, ntheta=ntheta)


def crand(rng, shape):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)


def test_maps_and_regulariser(problem):
    gs, os_ = problem["gs"], problem["os"]
    rng = np.random.default_rng(0)
    u = crand(rng, (32, 32, 32)) * 1e-3
    assert rel(gs.fwd_reg(T(u)), os_.fwd_reg(u)) < 1e-6
    g3 = crand(rng, (3, 32, 32, 32))
    assert rel(gs.adj_reg(T(g3)), os_.adj_reg(g3)) < 1e-6
    mu = crand(rng, (3, 32, 32, 32)) * 1e-3
    assert rel(gs.solve_reg(T(u), T(mu), 0.7, 1e-3), os_.solve_reg(u, mu, 0.7, 1e-3)) < 1e-5
    p = crand(rng, (16, 32, 32))
    assert rel(gs.mlog(T(p)), os_.mlog(p)) < 1e-6
    assert rel(gs.logtomo(T(p)), os_.logtomo(p)) < 1e-6
    assert rel(gs.exptomo(T(u[:16])), os_.exptomo(u[:16])) < 1e-6


def test_operators_through_solver(problem):
    gs, os_ = problem["gs"], problem["os"]
    rng = np.random.default_rng(1)
    u = crand(rng, (32, 32, 32))
    assert rel(gs.fwd_tomo_batch(T(u)), os_.fwd_tomo_batch(u)) < 1e-5
    g = crand(rng, (16, 32, 32))
    assert rel(gs.adj_tomo_batch(T(g)), os_.adj_tomo_batch(g)) < 1e-5
    assert rel(gs.fwd_tomo(T(u[:16])), os_.fwd_tomo(u[:16])) < 1e-5
    psi = np.exp(1j * crand(rng, (16, 32, 32)).real * 0.3).astype(np.complex64)
    assert rel(gs.fwd_ptycho_batch(T(psi)), os_.fwd_ptycho_batch(psi)) < 1e-5
    gs.cl_ptycho = gs._ptycho[1]
    os_._setobj(slice(8, 16))
    assert rel(gs.fwd_ptycho(T(psi[8:])), os_.fwd_ptycho(psi[8:])) < 1e-5
    fr = crand(rng, (8, 9, 16, 16))
    assert rel(gs.adj_ptycho(T(fr)), os_.adj_ptycho(fr)) < 1e-5


def test_takexi_and_penalties(problem):
    gs, os_ = problem["gs"], problem["os"]
    rng = np.random.default_rng(2)
    psi = np.exp(1j * (0.5 + 0.2 * rng.standard_normal((16, 32, 32)))).astype(np.complex64)
    lamd = crand(rng, (16, 32, 32)) * 1e-2
    phi, mu = crand(rng, (3, 32, 32, 32)), crand(rng, (3, 32, 32, 32))
    a = gs.takexi(T(psi), T(phi), T(lamd), T(mu), 0.5, 0.25)
    b = os_.takexi(psi, phi, lamd, mu, 0.5, 0.25)
    for x, y in zip(a[:3], b[:3]):
        assert rel(x, y) < 1e-5
    assert abs(a[3] - b[3]) < 1e-6
    h, h0 = psi * 1.01, psi
    e, e0 = phi * 0.9, phi
    assert gs.update_penalty(T(psi), T(h), T(h0), T(phi), T(e), T(e0), 0.5, 0.5) == \
        os_.update_penalty(psi, h, h0, phi, e, e0, 0.5, 0.5)


def test_cg_tomo(problem):
    gs, os_ = problem["gs"], problem["os"]
    psi = os_.exptomo(os_.fwd_tomo_batch(problem["obj"]))
    zeros3 = np.zeros((3, 32, 32, 32), np.complex64)
    xi0, xi1, Kt, _ = os_.takexi(psi, zeros3, np.zeros_like(psi), zeros3, 0.5, 0.5)
    u0 = np.zeros((32, 32, 32), np.complex64)
    ug = gs.cg_tomo(T(xi0), T(xi1), T(Kt), T(u0), 0.5, 0.5, 4)
    uo = os_.cg_tomo(xi0, xi1, Kt, u0, 0.5, 0.5, 4)
    assert rel(ug, uo) < 1e-3


@pytest.mark.parametrize("model", ["poisson", "gaussian"])
def test_cg_ptycho_batch(problem, model):
    gs, os_ = problem["gs"], problem["os"]
    data = problem["data"]
    psi0 = np.ones((16, 32, 32), np.complex64)
    h = np.ones_like(psi0)
    lamd = np.zeros_like(psi0)
    pg = gs.cg_ptycho_batch(T(data), T(psi0), T(h), T(lamd), 0.5, 4, model)
    po = os_.cg_ptycho_batch(data, psi0, h, lamd, 0.5, 4, model)
    assert rel(pg, po) < 1e-3


@pytest.mark.parametrize("model", ["poisson", "gaussian"])
def test_admm_matches_oracle(problem, model):
    """Whole ADMM against the oracle.

    Every sub-step matches the oracle to 1e-5 .. 1e-3 (tests above), and the
    line-search step lengths agree exactly until a CG is within FP32 rounding
    of convergence; there, any two FP32 implementations (the reference against
    itself, with its float atomics) break ties differently, and takexi's
    phase subtraction amplifies the tiny psi differences into ~1e-2 in xi0.
    So the end-to-end comparison is on the stable quantities: the penalty
    schedule exactly, the Lagrangian and the reconstruction error vs the
    phantom to 5%."""
    gs, os_ = problem["gs"], problem["os"]
    data = problem["data"]
    nt, nz, n = 16, 32, 32
    init = lambda: (np.ones((nt, nz, n), np.complex64), np.zeros((3, nz, n, n), np.complex64),  # noqa: E731
                    np.ones((nt, nz, n), np.complex64), np.zeros((3, nz, n, n), np.complex64),
                    np.zeros((nt, nz, n), np.complex64), np.zeros((3, nz, n, n), np.complex64),
                    np.zeros((nz, n, n), np.complex64))
    h, e, psi, phi, lamd, mu, u = init()
    hist_g, hist_o = [], []
    ug, psig = gs.admm(T(data), T(h), T(e), T(psi), T(phi), T(lamd), T(mu), T(u), 1e-9, 2, 2, 3, model,
                       verbose=False, history=hist_g)
    h, e, psi, phi, lamd, mu, u = init()
    uo, psio = os_.admm(data, h, e, psi, phi, lamd, mu, u, 1e-9, 2, 2, 3, model, history=hist_o)
    assert [x["rho"] for x in hist_g] == [x["rho"] for x in hist_o]
    assert [x["tau"] for x in hist_g] == [x["tau"] for x in hist_o]
    assert rel(psig, psio) < 1e-3
    lg, lo = hist_g[0]["lagr"], hist_o[0]["lagr"]
    assert abs(lg[0] - lo[0]) <= 5e-2 * abs(lo[0])
    assert abs(lg[6] - lo[6]) <= 5e-2 * abs(lo[6])
    obj = problem["obj"]
    eg = np.linalg.norm(ug.cpu().numpy() - obj) / np.linalg.norm(obj)
    eo = np.linalg.norm(uo - obj) / np.linalg.norm(obj)
    assert abs(eg - eo) <= 5e-2 * eo, (eg, eo)


def _corr(u, obj):
    a, b = u - u.mean(), obj - obj.mean()
    return float(np.corrcoef(a.ravel(), b.ravel())[0, 1])


def test_admm_reconstruction_quality_tracks_oracle(problem):
    """4 ADMM iterations (36+36+4+4 ptycho CG steps): delta = -Re u correlates
    with the phantom (> 0.6) and the GPU's correlation and error track the
    oracle's (the reference algorithm) within 0.03 / 5%."""
    gs, os_ = problem["gs"], problem["os"]
    data = problem["data"]
    nt, nz, n = 16, 32, 32
    c = dict(dtype=torch.complex64, device="cuda")
    ones = torch.ones((nt, nz, n), **c)
    z3 = torch.zeros((3, nz, n, n), **c)
    ug, _ = gs.admm(T(data), ones.clone(), z3.clone(), ones.clone(), z3.clone(), torch.zeros_like(ones), z3.clone(),
                    torch.zeros((nz, n, n), **c), 1e-9, 4, 4, 4, "poisson", verbose=False)
    o1, o3 = np.ones((nt, nz, n), np.complex64), np.zeros((3, nz, n, n), np.complex64)
    uo, _ = os_.admm(data, o1.copy(), o3.copy(), o1.copy(), o3.copy(), np.zeros_like(o1), o3.copy(),
                     np.zeros((nz, n, n), np.complex64), 1e-9, 4, 4, 4, "poisson")
    ug = ug.cpu().numpy()
    obj = problem["obj"]
    cg, co = _corr(ug.real, obj.real), _corr(uo.real, obj.real)
    assert cg > 0.6 and abs(cg - co) < 0.03, (cg, co)
    eg = np.linalg.norm(ug - obj) / np.linalg.norm(obj)
    eo = np.linalg.norm(uo - obj) / np.linalg.norm(obj)
    assert abs(eg - eo) < 5e-2 * eo, (eg, eo)


@pytest.mark.parametrize("model", ["poisson", "gaussian"])
def test_cg_ptycho_det128(model):
    """The CG on 128 detectors (the det-128 operator kernels) tracks the oracle.

    The start is the object at 0.8 times its contrast.  From psi = 1 the Poisson
    step lengths are not determined by FP32 arithmetic: detector pixels where
    |FQ psi| ~ 1e-9 of the frame's peak carry counts, the likelihood is steep
    there, and noise of 3e-8 of the frame RMS in the oracle's own forward moves
    its first step between 2^-11 and 2^-10."""
    from ptychotomo_b200 import Solver
    n = nz = 128
    ntheta, nprb = 4, 96
    theta = synthetic.angles(ntheta)
    prb = synthetic.probe(nprb, seed=4)
    scan = synthetic.raster_scan(ntheta, 3, n, nz, nprb)
    scan[1] += np.float32(0.2)
    obj = synthetic.phantom(n, nz, seed=5)
    args = (prb, scan, theta, [128, 128], 1e-6, 5.0, ntheta, nz, n, ntheta // 2, nz // 2)
    gs = Solver(*args)
    x = torch.empty((ntheta, gs.cl_tomo.N), dtype=torch.float32, device="cuda")
    y = torch.empty_like(x)
    gs._tomo_all.get_xy(x, y)
    os_ = OSolver(*args, xy=(x.cpu().numpy(), y.cpu().numpy()))
    data = os_.fwd_ptycho_batch(os_.exptomo(os_.fwd_tomo_batch(obj)))
    data = np.random.default_rng(6).poisson(data * 1e3).astype(np.float32) / np.float32(1e3)
    psi0 = os_.exptomo(os_.fwd_tomo_batch((0.8 * obj).astype(np.complex64)))
    h, lamd = np.ones_like(psi0), np.zeros_like(psi0)
    gs.trace, os_.trace = [], []
    pg = gs.cg_ptycho_batch(T(data), T(psi0), T(h), T(lamd), 0.5, 4, model)
    po = os_.cg_ptycho_batch(data, psi0, h, lamd, 0.5, 4, model)
    assert [g for _, g in gs.trace] == [g for _, g in os_.trace]
    gs.trace = None
    assert rel(pg, po) < 1e-4


@pytest.mark.parametrize("model", [0, 1])
def test_residual_edge_values(model):
    """The gradient residual (solver.py:220-224) at zeros, tiny and subnormal
    values and zero counts, against numpy's angle / exp form in float64."""
    from ptychotomo_b200 import kernels
    rng = np.random.default_rng(9)
    mags = np.concatenate([np.zeros(4), 10.0 ** rng.uniform(-44, 3, 400)])
    ph = rng.uniform(-np.pi, np.pi, mags.size)
    x = (mags * np.exp(1j * ph)).astype(np.complex64)
    x[1] = np.complex64(1e-45 + 0j)   # subnormal parts
    x[2] = np.complex64(-3e-42 + 2e-43j)
    D = np.where(rng.uniform(size=x.size) < 0.3, 0.0, 10.0 ** rng.uniform(-6, 4, x.size)).astype(np.float32)
    out = kernels.residual(torch.empty(x.size, dtype=torch.complex64, device="cuda"), T(x), T(D), 1.0, model)
    xd = x.astype(np.complex128)
    if model == 0:
        ref = xd - D * xd / (np.abs(xd) ** 2 + 1e-32)
    else:
        ref = xd - np.sqrt(D) * np.exp(1j * np.angle(xd))
    got = out.cpu().numpy().astype(np.complex128)
    scale = np.maximum(np.abs(ref), np.abs(xd)) + np.sqrt(D) + 1e-30
    assert np.all(np.isfinite(got))
    assert np.max(np.abs(got - ref) / scale) < 2e-6


def test_admm_checkpoint_resume_is_bitwise(problem, tmp_path):
    """An ADMM run saved after iteration 2 and resumed gives the same bits as
    an uninterrupted run (deterministic kernels, same penalty schedule); a
    checkpoint of another problem is refused."""
    gs = problem["gs"]
    data = T(problem["data"])
    c = dict(dtype=torch.complex64, device="cuda")

    def init():
        psi = torch.ones((16, 32, 32), **c)
        z3 = torch.zeros((3, 32, 32, 32), **c)
        return dict(h=psi.clone(), e=z3.clone(), psi=psi, phi=z3.clone(), lamd=torch.zeros_like(psi),
                    mu=z3.clone(), u=torch.zeros((32, 32, 32), **c))

    def run(niter, **kw):
        a = init()
        hist = []
        u, psi = gs.admm(data, a["h"], a["e"], a["psi"], a["phi"], a["lamd"], a["mu"], a["u"], 1e-3, 4, 4, niter,
                         "poisson", verbose=False, history=hist, **kw)
        return u, psi, [(x["rho"], x["tau"]) for x in hist]

    u_ref, psi_ref, hist_ref = run(4)
    ck = str(tmp_path / "admm.pt")
    _, _, h1 = run(2, checkpoint=ck)
    u, psi, h2 = run(4, checkpoint=ck, resume=True)
    assert h1 + h2 == hist_ref
    assert torch.equal(u, u_ref) and torch.equal(psi, psi_ref)
    st = torch.load(ck, weights_only=True)
    assert st["m"] == 3
    st["held"] = ((0, 8), (0, 32), 16, 32, 32)
    torch.save(st, ck)
    with pytest.raises(ValueError, match="another problem"):
        run(5, checkpoint=ck, resume=True)


@pytest.mark.parametrize("model", [0, 1])
def test_ls_frames_advance(model):
    """pt_ls_frames_advance returns pt_ls_frames's sums (same kernel and order)
    and leaves f + gammas[0] d in f."""
    from ptychotomo_b200 import kernels
    rng = np.random.default_rng(31 + model)
    n = 5 * 7 * 32 * 32 + 3
    f = T(crand(rng, (n,)))
    d = T(0.1 * crand(rng, (n,)))
    data = T(rng.poisson(3.0, n).astype(np.float32))
    gs = [0.75, 0.375]
    red = kernels.Reducer("cuda")
    ref = red.ls_frames(f, d, data, 0.8, model, gs)
    f2 = f.clone()
    got = red.ls_frames(f2, d, data, 0.8, model, gs, advance=True)
    assert got == ref
    want = f + np.float32(0.75) * d
    assert torch.allclose(f2, want, rtol=1e-6, atol=1e-7)


@pytest.mark.parametrize("model", ["poisson", "gaussian"])
def test_cg_ptycho_advanced_frames_match_recomputed(problem, model):
    """The ptycho CG with frames advanced by the line search takes the same steps
    as the CG that recomputes F Q psi every iteration."""
    gs = problem["gs"]
    data = problem["data"]
    psi0 = np.ones((16, 32, 32), np.complex64)
    h, lamd = np.ones_like(psi0), np.zeros_like(psi0)
    out = []
    for adv in (True, False):
        gs.advance_frames, gs.trace = adv, []
        p = gs.cg_ptycho_batch(T(data), T(psi0), T(h), T(lamd), 0.5, 8, model)
        out.append(([g for _, g in gs.trace], p.cpu().numpy()))
    gs.advance_frames, gs.trace = True, None
    assert out[0][0] == out[1][0]
    assert rel(out[0][1], out[1][1]) < 1e-5


def test_batched_reductions_equal_the_single_ones():
    """Reducer.many (one read-back for the Dai-Yuan terms and the quad3
    triples of a CG iteration) returns exactly what the single calls do."""
    from ptychotomo_b200 import kernels as K
    rng = np.random.default_rng(9)
    a, b = T(crand(rng, (5, 37, 41))), T(crand(rng, (5, 37, 41)))
    red = K.Reducer("cuda")
    many = red.many([("dot", a, b), ("norm2", a), ("quad3", a, b), ("norm2_diff", a, b)])
    assert many == [red.dot(a, b), red.norm2(a), red.quad3(a, b), red.norm2_diff(a, b)]
