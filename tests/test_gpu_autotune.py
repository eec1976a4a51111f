"""The autotuners: ptychofft.autotune picks the adjoint's angle split and
radonusfft.autotune the forward's stream count and gather variant by timing;
every choice keeps the operators' results (against the oracle, rel-L2 <=
1e-5), and the nine radon forward variants (one, two or four streams; gather
through L1, from shared-memory tiles copied by the threads, or from tiles
loaded by the TMA) give bit-identical projections."""
import numpy as np
import pytest

from oracle.ptycho import PtychoFFT
from oracle.usfft import RadonUSFFT

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def crand(rng, shape):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)


def T(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def test_ptycho_autotune_keeps_the_adjoint():
    from ptychotomo_b200 import ptychofft
    rng = np.random.default_rng(0)
    nt, nz, n, ns, det = 4, 160, 160, 9, 128
    scan = np.stack([rng.uniform(0, n - det - 0.5, (nt, ns)), rng.uniform(0, nz - det - 0.5, (nt, ns))]).astype(np.float32)
    prb = crand(rng, (det, det))
    op = ptychofft(nt, nz, n, nt, ns, det, det, det)
    op.setobj(T(scan), T(prb))
    g = T(crand(rng, (nt, ns, det, det)))
    f = torch.empty((nt, nz, n), dtype=torch.complex64, device="cuda")
    parts = op.autotune(f, g, trials=2)
    assert parts == op.parts and 1 <= parts <= ns
    op.adj(f, g)
    orc = PtychoFFT(nt, nz, n, nt, ns, det, det, det)
    orc.setobj(scan, prb)
    assert rel(f.cpu().numpy(), orc.adj(g.cpu().numpy())) <= 1e-5


def test_radon_autotune_keeps_the_forward():
    from ptychotomo_b200 import radonusfft
    rng = np.random.default_rng(1)
    n, nz, nt = 64, 40, 48
    theta = np.linspace(0, np.pi, nt, endpoint=False).astype(np.float32)
    op = radonusfft(nt, nz, n)
    op.setobj(T(theta))
    f = T(crand(rng, (nz, n, n)))
    g = torch.empty((nt, nz, n), dtype=torch.complex64, device="cuda")
    op.set_variant(1, 0)
    before = torch.empty_like(g)
    op.fwd(before, f)
    timeouts, tma = op.status()
    assert tma and timeouts == 0
    for streams in (1, 2, 4):
        for gather in (0, 1, 2):
            op.set_variant(streams, gather)
            op.fwd(g, f)
            assert torch.equal(g, before), (streams, gather)
    assert op.status() == (0, True)
    streams, gather = op.autotune(g, f, trials=2)
    assert streams in (1, 2, 4) and gather in (0, 1, 2)
    op.fwd(g, f)
    assert torch.equal(g, before)
    x = torch.empty((nt, op.N), dtype=torch.float32, device="cuda")
    y = torch.empty_like(x)
    op.get_xy(x, y)
    orc = RadonUSFFT(nt, nz, n)
    orc.setobj(theta, xy=(x.cpu().numpy(), y.cpu().numpy()))
    assert rel(g.cpu().numpy(), orc.fwd(f.cpu().numpy())) <= 1e-5


@pytest.mark.parametrize("n,nz,nt,m", [(16, 5, 12, 0), (32, 9, 24, 0), (256, 3, 384, 0), (64, 8, 40, 4)])
def test_tiled_gathers_are_bit_identical(n, nz, nt, m):
    """The shared-memory tiled gather and its TMA-staged form against the
    L1 gather at small grids (where the staged region runs past the haloed
    grid: clipped by the threads, zero-filled by the TMA), at the bench's
    width and angle count, and with the M = 4 kernel."""
    from ptychotomo_b200 import radonusfft
    rng = np.random.default_rng(n)
    theta = np.sort(rng.uniform(0, np.pi, nt)).astype(np.float32)
    op = radonusfft(nt, nz, n, m) if m else radonusfft(nt, nz, n)
    op.setobj(T(theta))
    f = T(crand(rng, (nz, n, n)))
    a = torch.empty((nt, nz, n), dtype=torch.complex64, device="cuda")
    b, c = torch.empty_like(a), torch.empty_like(a)
    op.set_variant(1, 0)
    op.fwd(a, f)
    op.set_variant(1, 1)
    op.fwd(b, f)
    op.set_variant(2, 2)
    op.fwd(c, f)
    assert op.status() == (0, True)
    assert torch.equal(a, b) and torch.equal(a, c)
    op.set_variant(4, 2)
    op.fwd(c, f)
    assert torch.equal(a, c)
