"""The preconditioner network's forward on the tensor cores (pt_mlp_forward_tc:
the 64 x 64 layer as tcgen05 MMAs with FP32 accumulators in tensor memory)
against the CPU oracle with the same roundings (bf16 weights, h1 rounded to
bf16 before the layer): rel-L2 <= 1e-4 (a float32 h1 and the oracle's
float64 h1 can round to neighbouring bf16 values); within 1e-2 of the
CUDA-core forward, whose h1 stays FP32; bitwise reproducible; no wait ran
out.  Tile sizes cover partial tiles (1, 127, 129 points) and many tiles."""
import numpy as np
import pytest

from oracle import mlp as omlp

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def rel(a, b):
    a = a.cpu().numpy() if hasattr(a, "cpu") else np.asarray(a)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("npts", [1, 127, 128, 129, 5000, 65536])
def test_tensor_core_forward_matches_oracle(npts):
    from ptychotomo_b200.learned import MLP
    rng = np.random.default_rng(npts)
    params = MLP.init_params(3) + (rng.standard_normal(omlp.NPAR) * 0.05).astype(np.float32)
    params = params.astype(np.float32)
    x = rng.uniform(0, 1, (npts, 3)).astype(np.float32)
    net = MLP("cuda", params=params, bf16=True)
    X = torch.from_numpy(x).cuda()
    z = net.forward_tc(X)
    z2 = net.forward_tc(X)
    torch.cuda.synchronize()
    assert net.tc_status() == 0
    assert torch.equal(z, z2)
    zo = omlp.forward(params, x, bf16=True, act_bf16=True)
    assert rel(z, zo) <= 1e-4
    assert rel(z, net.forward(X).cpu().numpy()) <= 1e-2
