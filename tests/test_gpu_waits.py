"""The bounded waits of the kernels that wait on an mbarrier: the TMA-staged
radon gather and the tensor-core network forward.  Each has a status-test
launch whose threads wait on a barrier that nothing arrives at, with a short
limit: the wait must run out, the kernel must record code 1 in its device
flag, wait for its own copies or MMAs, release its resources and return
(no hang, no fault); afterwards the context is usable and the normal paths
give the same results as before."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def test_tma_gather_wait_runs_out_and_reports():
    from ptychotomo_b200 import radonusfft
    rng = np.random.default_rng(0)
    n, nz, nt = 64, 16, 48
    theta = np.linspace(0, np.pi, nt, endpoint=False).astype(np.float32)
    op = radonusfft(nt, nz, n)
    op.setobj(torch.from_numpy(theta).cuda())
    f = torch.from_numpy((rng.standard_normal((nz, n, n)) + 1j * rng.standard_normal((nz, n, n))).astype(np.complex64)).cuda()
    a, b = (torch.empty((nt, nz, n), dtype=torch.complex64, device="cuda") for _ in range(2))
    op.set_variant(1, 2)
    op.fwd(a, f)
    assert op.status() == (0, True)
    assert op.check_tma_wait() == 1
    assert op.status() == (0, True)      # the check clears its flag
    op.fwd(b, f)
    torch.cuda.synchronize()
    assert torch.equal(a, b)


def test_tensor_core_wait_runs_out_and_reports():
    from ptychotomo_b200.learned import MLP
    net = MLP("cuda", seed=1)
    x = torch.rand((1000, 3), device="cuda")
    z0 = net.forward_tc(x)
    assert net.tc_status() == 0
    assert net.check_tc_wait() == 1
    z1 = net.forward_tc(x)
    torch.cuda.synchronize()
    assert net.tc_status() == 0
    assert torch.equal(z0, z1)
