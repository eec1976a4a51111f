"""GPU checks of the preconditioner network kernels (pt_mlp_*) against the
CPU oracle (oracle/mlp.py, float64).

Tolerances: forward values rel-L2 <= 1e-5; parameter gradients rel-L2 <=
1e-5 in FP32 mode (FP32 weights) and with bf16 weights (the oracle rounds the
same weights); one Adam step <= 1e-6; the gradient is bitwise reproducible.
"""
import numpy as np
import pytest

from oracle import mlp as omlp

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def rel(a, b):
    a = a.cpu().numpy() if hasattr(a, "cpu") else np.asarray(a)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _problem(npts, seed):
    rng = np.random.default_rng(seed)
    from ptychotomo_b200.learned import MLP
    params = MLP.init_params(seed) + (rng.standard_normal(omlp.NPAR) * 0.05).astype(np.float32)
    x = rng.uniform(0, 1, (npts, 3)).astype(np.float32)
    y = np.sin(3 * x[:, 0]) + x[:, 1] * x[:, 2]
    w = rng.uniform(0.1, 1, npts).astype(np.float32)
    return params.astype(np.float32), x, y.astype(np.float32), w


@pytest.mark.parametrize("bf16", [False, True])
@pytest.mark.parametrize("npts", [1, 257, 5000])
def test_forward_and_gradient_match_oracle(bf16, npts):
    from ptychotomo_b200.learned import MLP
    params, x, y, w = _problem(npts, 11 + npts)
    net = MLP("cuda", params=params, bf16=bf16)
    X, Y, W = (torch.from_numpy(a).cuda() for a in (x, y, w))
    z = net.forward(X)
    zo = omlp.forward(params, x, bf16=bf16)
    assert rel(z, zo) <= 1e-5
    inv = 1.0 / float(w.astype(np.float64).sum())
    net.loss_grad(X, Y, W, inv)
    lo, go = omlp.loss_and_grad(params, x, y, w, inv, bf16=bf16)
    assert abs(net.loss.item() - lo) <= 1e-5 * abs(lo)
    assert rel(net.grad, go) <= 1e-5


def test_gradient_is_bitwise_reproducible():
    from ptychotomo_b200.learned import MLP
    params, x, y, w = _problem(20000, 5)
    net = MLP("cuda", params=params)
    X, Y, W = (torch.from_numpy(a).cuda() for a in (x, y, w))
    net.loss_grad(X, Y, W, 1e-4)
    g1 = net.grad.clone()
    net.loss_grad(X, Y, W, 1e-4)
    assert torch.equal(g1, net.grad)


def test_adam_step_matches_oracle():
    from ptychotomo_b200.learned import MLP
    params, x, y, w = _problem(3000, 6)
    net = MLP("cuda", params=params)
    X, Y, W = (torch.from_numpy(a).cuda() for a in (x, y, w))
    inv = 1.0 / float(w.astype(np.float64).sum())
    p = params.astype(np.float64)
    m = np.zeros_like(p)
    v = np.zeros_like(p)
    for step in (1, 2, 3):
        net.loss_grad(X, Y, W, inv)
        g = net.grad.cpu().numpy().astype(np.float64)
        net.adam(1e-2)
        p, m, v = omlp.adam(p, m, v, g, step, 1e-2)
        assert rel(net.params, p) <= 1e-6


def test_training_fits_a_smooth_target():
    """Full-batch Adam with the project's kernels reduces the loss of a smooth
    3-feature regression by orders of magnitude."""
    from ptychotomo_b200.learned import MLP
    params, x, y, w = _problem(8192, 7)
    net = MLP("cuda", seed=7)
    X, Y, W = (torch.from_numpy(a).cuda() for a in (x, y, w))
    hist = net.fit(X, Y, W, steps=1500, lr=1e-2, lr_final=1e-3, log_every=500)
    assert hist[-1][1] < 1e-3 * hist[0][1], hist
