"""CPU checks of the preconditioner network's oracle (oracle/mlp.py): its
analytic gradient against central finite differences in float64, and its
bfloat16 rounding against torch's float32 -> bfloat16 conversion."""
import numpy as np

from oracle import mlp


def _problem(seed=0, npts=40):
    rng = np.random.default_rng(seed)
    params = (rng.standard_normal(mlp.NPAR) * 0.3).astype(np.float64)
    x = rng.uniform(-1, 1, (npts, 3))
    y = rng.standard_normal(npts)
    w = rng.uniform(0, 1, npts)
    return params, x, y, w


def test_gradient_matches_finite_differences():
    params, x, y, w = _problem()
    inv = 1.0 / w.sum()
    loss, g = mlp.loss_and_grad(params, x, y, w, inv, bf16=False)
    rng = np.random.default_rng(1)
    idx = rng.choice(mlp.NPAR, 60, replace=False)
    h = 1e-6
    for i in idx:
        e = np.zeros(mlp.NPAR)
        e[i] = h
        lp, _ = mlp.loss_and_grad(params + e, x, y, w, inv, bf16=False)
        lm, _ = mlp.loss_and_grad(params - e, x, y, w, inv, bf16=False)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i])), (i, fd, g[i])


def test_forward_agrees_with_loss_path():
    params, x, y, w = _problem(2)
    z = mlp.forward(params, x, bf16=True)
    loss, _ = mlp.loss_and_grad(params, x, z, w, 1.0, bf16=True)
    assert loss < 1e-20


def test_bf16_rounding_matches_torch():
    import torch
    rng = np.random.default_rng(3)
    a = (rng.standard_normal(10000) * 10.0 ** rng.uniform(-5, 5, 10000)).astype(np.float32)
    ref = torch.from_numpy(a).to(torch.bfloat16).to(torch.float32).numpy()
    assert np.array_equal(mlp.bf16_round(a), ref)
