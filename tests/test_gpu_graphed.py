"""One ADMM iteration captured as a CUDA graph (ptychotomo_b200.graphed).

* A replay equals the same iterations run eagerly, bit for bit (the graph
  holds exactly the eager launch sequence; every kernel is deterministic).
* The device-scalar iteration tracks the host Solver.admm_step from the same
  state (each iteration from the host's state before it): the same step
  lengths, the same penalty decisions, psi within 1e-5 and u within 1e-3
  (F Q psi advances by linearity instead of the host's occasional new
  forward, so the arithmetic differs at FP32 rounding; u is the tomography
  response to psi's phase and amplifies differences ~100-fold, as in the
  lock-step test against the oracle).
* With the learned preconditioner, the replay equals the eager run too.
"""
import pytest

from ptychotomo_b200 import synthetic

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b))


@pytest.fixture(scope="module")
def problem():
    from ptychotomo_b200 import Solver
    n = nz = 32
    nt, P = 16, 16
    theta = synthetic.angles(nt)
    prb = synthetic.probe(P, seed=1)
    scan = synthetic.raster_scan(nt, 3, n, nz, P)
    obj = synthetic.phantom(n, nz, seed=2)
    slv = Solver(prb, scan, theta, [P, P], 1e-6, 5.0, nt, nz, n, nt, nz)
    u = torch.from_numpy(obj).cuda()
    inten = slv.fwd_ptycho_batch(slv.exptomo(slv.fwd_tomo_batch(u)))
    g = torch.Generator(device="cuda").manual_seed(3)
    data = torch.poisson(inten * 1e3, generator=g) / 1e3
    c = dict(dtype=torch.complex64, device="cuda")
    one = torch.ones((nt, nz, n), **c)
    z3 = torch.zeros((3, nz, n, n), **c)
    st = dict(u=torch.zeros((nz, n, n), **c), psi=one.clone(), h=one.clone(), e=z3.clone(), phi=z3.clone(),
              lamd=torch.zeros_like(one), mu=z3.clone())
    rho = tau = 0.5
    for m in range(2):     # past the 36-step warm-up iterations
        st, rho, tau = slv.admm_step(m, st, rho, tau, slv._as_data(data), 1e-3, 4, 4, "poisson")
    return slv, data, {k: v.clone() for k, v in st.items()}, rho, tau


def _snapshot(g):
    st, rho, tau = g.state()
    return {k: v.clone() for k, v in st.items()}, rho, tau


@pytest.mark.parametrize("use_precond", [False, True])
def test_replay_equals_eager(problem, use_precond):
    from ptychotomo_b200.graphed import GraphedADMM
    slv, data, st0, rho, tau = problem
    pre = None
    if use_precond:
        from ptychotomo_b200.learned import MLP, FourierPreconditioner
        pre = FourierPreconditioner(slv._tomo_all, slv.theta, slv.coeftomo, "cuda")
        pre.set_network(MLP("cuda", seed=0))
    g = GraphedADMM(slv, data, 1e-3, 4, 4, "poisson", precond=pre)
    g.load(st0, rho, tau)
    for m in (2, 3):
        g.step(m)
    eager = _snapshot(g)
    g.load(st0, rho, tau)
    g.capture()
    g.replay()
    g.replay()
    graph = _snapshot(g)
    assert eager[1:] == graph[1:]
    for k in eager[0]:
        assert torch.equal(eager[0][k], graph[0][k]), k


def test_device_scalar_iteration_tracks_host_solver(problem):
    from ptychotomo_b200.graphed import GraphedADMM
    slv, data, st0, rho, tau = problem
    g = GraphedADMM(slv, data, 1e-3, 4, 4, "poisson")
    st, r, t = {k: v.clone() for k, v in st0.items()}, rho, tau
    for m in (2, 3, 4):      # lock-step: both from the host Solver's state before iteration m
        g.load(st, r, t)
        slv.trace, g.trace = [], []
        st, r, t = slv.admm_step(m, st, r, t, slv._as_data(data), 1e-3, 4, 4, "poisson")
        g.step(m)
        gs, gr, gt = g.state()
        print("m", m, "psi", rel(gs["psi"], st["psi"]), "u", rel(gs["u"], st["u"]))
        print("  host steps ", slv.trace)
        print("  graph steps", g.trace)
        for kind in ("ptycho", "tomo"):   # the host stops a CG at a zero step; the graph steps by 0
            hs = [v for k, v in slv.trace if k == kind]
            gs_ = [v for k, v in g.trace if k == kind]
            assert gs_[:len(hs)] == hs and all(v == 0 for v in gs_[len(hs):]), (kind, hs, gs_)
        slv.trace = None
        assert (gr, gt) == (r, t)
        assert rel(gs["psi"], st["psi"]) <= 1e-5
        assert rel(gs["u"], st["u"]) <= 1e-3
