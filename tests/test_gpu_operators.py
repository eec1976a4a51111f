"""GPU parity of the radonusfft / ptychofft operators.

Compared with (1) the NumPy oracle on the same seeded inputs and the same
polar coordinate tables, (2) the reference's own CUDA operators
(oracle/_ref) when built, (3) the adjoint identity <A x, y> = <x, A* y>, and
(4) run-to-run bitwise determinism.  Tolerance: relative L2 <= 1e-5 for
fwd/adj (the float32 operators against complex128 / float32 references).
"""
import numpy as np
import pytest

import refcuda
from oracle.ptycho import PtychoFFT
from oracle.usfft import RadonUSFFT, takexy

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

TOL = 1e-5


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(np.asarray(b)))


def crand(rng, shape):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def make_radon(n, nz, ntheta, theta, m_override=0):
    from ptychotomo_b200 import radonusfft
    op = radonusfft(ntheta, nz, n, m_override=m_override)
    op.setobj(dev(theta))
    x = torch.empty((ntheta, op.N), dtype=torch.float32, device="cuda")
    y = torch.empty_like(x)
    op.get_xy(x, y)
    torch.cuda.synchronize()
    orc = RadonUSFFT(ntheta, nz, n)
    orc.setobj(theta, xy=(x.cpu().numpy(), y.cpu().numpy()))
    return op, orc


def radon_fwd(op, f):
    g = torch.zeros((op.Ntheta, op.Nz, op.n), dtype=torch.complex64, device="cuda")
    op.fwd(g, f)
    return g


def radon_adj(op, g):
    f = torch.zeros((op.Nz, op.n, op.n), dtype=torch.complex64, device="cuda")
    op.adj(f, g)
    return f


RADON_SIZES = [(16, 5, 12), (32, 8, 24), (32, 11, 17), (64, 3, 40), (128, 9, 128)]


@pytest.mark.parametrize("n,nz,ntheta", RADON_SIZES)
def test_radon_fwd_adj_vs_oracle(n, nz, ntheta):
    rng = np.random.default_rng(n + nz)
    theta = np.sort(rng.uniform(0, np.pi, ntheta)).astype(np.float32)
    op, orc = make_radon(n, nz, ntheta, theta)
    f = crand(rng, (nz, n, n))
    g = crand(rng, (ntheta, nz, n))
    gf = radon_fwd(op, dev(f)).cpu().numpy()
    fa = radon_adj(op, dev(g)).cpu().numpy()
    assert rel(gf, orc.fwd(f)) <= TOL
    assert rel(fa, orc.adj(g)) <= TOL


def test_radon_polar_tables_match_exact_geometry():
    """Device tables use the reference's __cosf/__sinf; they must lie within
    the documented intrinsic error (|err| <= 2^-21.41 on [-pi, pi]) scaled
    by |k-N/2|/N <= 1/2 of float32 cos/sin tables."""
    n, ntheta = 64, 90
    theta = np.linspace(0, np.pi, ntheta, endpoint=False).astype(np.float32)
    op, orc = make_radon(n, 2, ntheta, theta)
    xe, ye = takexy(theta, op.N)
    assert np.max(np.abs(orc.x - xe)) <= 0.5 * 2 ** -21.41 + 1e-7
    assert np.max(np.abs(orc.y - ye)) <= 0.5 * 2 ** -21.41 + 1e-7


def test_radon_adjoint_identity():
    n, nz, ntheta = 64, 10, 48
    rng = np.random.default_rng(3)
    theta = np.linspace(0, np.pi, ntheta, endpoint=False).astype(np.float32)
    op, _ = make_radon(n, nz, ntheta, theta)
    f = crand(rng, (nz, n, n))
    f[:, 0, :] = f[:, -1, :] = f[:, :, 0] = f[:, :, -1] = 0   # border-zero (pad2 vs crop)
    g = crand(rng, (ntheta, nz, n))
    g[:, :, 0] = g[:, :, -1] = 0
    a = np.vdot(radon_fwd(op, dev(f)).cpu().numpy().astype(np.complex128), g.astype(np.complex128))
    b = np.vdot(f.astype(np.complex128), radon_adj(op, dev(g)).cpu().numpy().astype(np.complex128))
    assert abs(a - b) / abs(a) <= TOL


def test_radon_deterministic():
    n, nz, ntheta = 64, 8, 64
    rng = np.random.default_rng(4)
    theta = np.linspace(0, np.pi, ntheta, endpoint=False).astype(np.float32)
    op, _ = make_radon(n, nz, ntheta, theta)
    g = dev(crand(rng, (ntheta, nz, n)))
    f = dev(crand(rng, (nz, n, n)))
    assert torch.equal(radon_adj(op, g), radon_adj(op, g))
    assert torch.equal(radon_fwd(op, f), radon_fwd(op, f))


def test_radon_scaled_entry_points():
    n, nz, ntheta = 32, 4, 16
    rng = np.random.default_rng(5)
    theta = np.linspace(0, np.pi, ntheta, endpoint=False).astype(np.float32)
    op, _ = make_radon(n, nz, ntheta, theta)
    f = dev(crand(rng, (nz, n, n)))
    g = torch.zeros((ntheta, nz, n), dtype=torch.complex64, device="cuda")
    op.fwd(g, f, scale=0.25)
    assert rel(g.cpu().numpy(), 0.25 * radon_fwd(op, f).cpu().numpy()) <= 1e-6


@pytest.mark.skipif(not refcuda.available(), reason="reference CUDA operators not built (make -C oracle)")
@pytest.mark.parametrize("n,nz,ntheta", [(32, 8, 24), (128, 16, 128)])
def test_radon_vs_reference_cuda(n, nz, ntheta):
    rng = np.random.default_rng(7)
    theta = np.linspace(0, np.pi, ntheta, endpoint=False).astype(np.float32)
    th = dev(theta)
    op, _ = make_radon(n, nz, ntheta, theta)
    f = dev(crand(rng, (nz, n, n)))
    g = dev(crand(rng, (ntheta, nz, n)))
    ref = refcuda.RefRadon(ntheta, nz, n)
    ref.setobj(th.data_ptr())
    gr = torch.zeros((ntheta, nz, n), dtype=torch.complex64, device="cuda")
    fr = torch.zeros((nz, n, n), dtype=torch.complex64, device="cuda")
    ref.fwd(gr.data_ptr(), f.data_ptr())
    ref.adj(fr.data_ptr(), g.data_ptr())
    ref.free()
    assert rel(radon_fwd(op, f).cpu().numpy(), gr.cpu().numpy()) <= TOL
    assert rel(radon_adj(op, g).cpu().numpy(), fr.cpu().numpy()) <= TOL


# ---------------------------------------------------------------------------
# ptychography
# ---------------------------------------------------------------------------
def make_ptycho(ntheta, nz, n, nscan, det, nprb, rng, sentinel=True):
    from ptychotomo_b200 import ptychofft
    scan = np.empty((2, ntheta, nscan), np.float32)
    scan[0] = rng.uniform(0, max(n - nprb - 0.5, 0), (ntheta, nscan))
    scan[1] = rng.uniform(0, max(nz - nprb - 0.5, 0), (ntheta, nscan))
    if sentinel:
        scan[:, 0, 1] = -1
    prb = crand(rng, (nprb, nprb))
    op = ptychofft(ntheta, nz, n, ntheta, nscan, det, det, nprb)
    op.setobj(dev(scan), dev(prb))
    orc = PtychoFFT(ntheta, nz, n, ntheta, nscan, det, det, nprb)
    orc.setobj(scan, prb)
    return op, orc, scan, prb


def p_fwd(op, f):
    g = torch.zeros((op.Ntheta, op.Nscan, op.detx, op.dety), dtype=torch.complex64, device="cuda")
    op.fwd(g, f)
    return g


def p_adj(op, g):
    f = torch.zeros((op.Ntheta, op.Nz, op.N), dtype=torch.complex64, device="cuda")
    op.adj(f, g)
    return f


PTYCHO_SIZES = [(3, 32, 32, 7, 16, 16), (2, 24, 40, 5, 32, 16), (2, 64, 64, 9, 64, 64),
                (2, 130, 140, 6, 128, 128), (3, 100, 110, 5, 128, 96), (4, 20, 20, 3, 8, 8)]


@pytest.mark.parametrize("ntheta,nz,n,nscan,det,nprb", PTYCHO_SIZES)
def test_ptycho_fwd_adj_vs_oracle(ntheta, nz, n, nscan, det, nprb):
    rng = np.random.default_rng(det + nscan)
    op, orc, _, _ = make_ptycho(ntheta, nz, n, nscan, det, nprb, rng)
    f = crand(rng, (ntheta, nz, n))
    g = crand(rng, (ntheta, nscan, det, det))
    assert rel(p_fwd(op, dev(f)).cpu().numpy(), orc.fwd(f)) <= TOL
    assert rel(p_adj(op, dev(g)).cpu().numpy(), orc.adj(g)) <= TOL


def test_ptycho_adjoint_identity_and_determinism():
    rng = np.random.default_rng(11)
    op, _, _, _ = make_ptycho(3, 64, 64, 12, 64, 32, rng)
    f = dev(crand(rng, (3, 64, 64)))
    g = dev(crand(rng, (3, 12, 64, 64)))
    a = torch.vdot(p_fwd(op, f).flatten().cdouble(), g.flatten().cdouble()).item()
    b = torch.vdot(f.flatten().cdouble(), p_adj(op, g).flatten().cdouble()).item()
    assert abs(a - b) / abs(a) <= TOL
    assert torch.equal(p_adj(op, g), p_adj(op, g))


def test_ptycho_rejects_out_of_object_scan():
    from ptychotomo_b200 import PtychotomoArgError, ptychofft
    op = ptychofft(1, 32, 32, 1, 2, 16, 16, 16)
    scan = dev(np.array([[[0.0, 17.0]], [[0.0, 0.0]]], np.float32))
    with pytest.raises(PtychotomoArgError):
        op.setobj(scan, dev(np.ones((16, 16), np.complex64)))


@pytest.mark.skipif(not refcuda.available(), reason="reference CUDA operators not built (make -C oracle)")
@pytest.mark.parametrize("ntheta,nz,n,nscan,det,nprb", [(3, 48, 48, 9, 32, 32), (2, 64, 64, 6, 64, 16)])
def test_ptycho_vs_reference_cuda(ntheta, nz, n, nscan, det, nprb):
    rng = np.random.default_rng(13)
    op, _, scan, prb = make_ptycho(ntheta, nz, n, nscan, det, nprb, rng)
    f = dev(crand(rng, (ntheta, nz, n)))
    g = dev(crand(rng, (ntheta, nscan, det, det)))
    sc, pr = dev(scan), dev(prb)
    ref = refcuda.RefPtycho(ntheta, nz, n, nscan, det, nprb)
    ref.setobj(sc.data_ptr(), pr.data_ptr())
    gr = torch.zeros((ntheta, nscan, det, det), dtype=torch.complex64, device="cuda")
    fr = torch.zeros((ntheta, nz, n), dtype=torch.complex64, device="cuda")
    ref.fwd(gr.data_ptr(), f.data_ptr())
    ref.adj(fr.data_ptr(), g.data_ptr())
    ref.free()
    assert rel(p_fwd(op, f).cpu().numpy(), gr.cpu().numpy()) <= TOL
    assert rel(p_adj(op, g).cpu().numpy(), fr.cpu().numpy()) <= TOL


def test_ptycho_det128_misaligned_output_pointer():
    """A frame buffer that is only 8-byte aligned takes the generic kernel."""
    rng = np.random.default_rng(17)
    op, orc, _, _ = make_ptycho(2, 130, 130, 3, 128, 128, rng)
    f = crand(rng, (2, 130, 130))
    big = torch.zeros(2 * 3 * 128 * 128 + 1, dtype=torch.complex64, device="cuda")
    out = big[1:]
    assert out.data_ptr() % 16 == 8
    op.fwd(out.data_ptr(), dev(f))
    assert rel(out.view(2, 3, 128, 128).cpu().numpy(), orc.fwd(f)) <= TOL


def test_ptycho_det128_misaligned_adjoint_input():
    """An adjoint input that is only 8-byte aligned takes the generic kernel."""
    rng = np.random.default_rng(19)
    op, orc, _, _ = make_ptycho(2, 140, 130, 4, 128, 128, rng)
    g = crand(rng, (2, 4, 128, 128))
    big = torch.zeros(g.size + 1, dtype=torch.complex64, device="cuda")
    big[1:] = dev(g.ravel())
    src = big[1:]
    assert src.data_ptr() % 16 == 8
    out = torch.zeros((2, 140, 130), dtype=torch.complex64, device="cuda")
    op.adj(out, src.data_ptr())
    assert rel(out.cpu().numpy(), orc.adj(g)) <= TOL


@pytest.mark.parametrize("n,shift,parts", [(130, 0, "1"), (131, 0, None), (130, 1, "1")])
def test_ptycho_det128_adjoint_row_alignment(n, shift, parts, monkeypatch):
    """The det-128 adjoint adds a frame into its object rows with 16-byte
    accesses when the frame starts at an even column of an even-width object
    whose output is 16-byte aligned, and with 8-byte accesses otherwise.  Scans
    at both column parities; an odd width; an output that is only 8-byte
    aligned, written directly (one part per angle)."""
    if parts:
        monkeypatch.setenv("PT_PTYCHO_ADJ_PARTS", parts)
    rng = np.random.default_rng(23 + n + shift)
    op, orc, scan, _ = make_ptycho(2, 140, n, 6, 128, 128, rng)
    cols = np.round(scan[0]).astype(int)[scan[0] >= 0]
    assert (cols % 2 == 0).any() and (cols % 2 == 1).any()
    g = crand(rng, (2, 6, 128, 128))
    big = torch.zeros(2 * 140 * n + shift, dtype=torch.complex64, device="cuda")
    out = big[shift:]
    assert out.data_ptr() % 16 == 8 * shift
    op.adj(out.data_ptr(), dev(g))
    assert rel(out.view(2, 140, n).cpu().numpy(), orc.adj(g)) <= TOL


@pytest.mark.parametrize("ntheta,nz,n,nscan,det,nprb", [(2, 130, 140, 6, 128, 128), (2, 100, 110, 4, 128, 96),
                                                       (2, 64, 64, 9, 64, 32), (3, 20, 20, 3, 8, 8)])
@pytest.mark.parametrize("model", [0, 1])
def test_ptycho_adjoint_with_fused_residual(ntheta, nz, n, nscan, det, nprb, model):
    """adj_resid == adj(residual(fpsi, data)), the gradient of solver.py:220-224."""
    from ptychotomo_b200 import kernels
    rng = np.random.default_rng(det + model)
    op, _, _, _ = make_ptycho(ntheta, nz, n, nscan, det, nprb, rng)
    fpsi = dev(crand(rng, (ntheta, nscan, det, det)))
    data = dev(rng.poisson(3.0, (ntheta, nscan, det, det)).astype(np.float32))
    res = kernels.residual(torch.empty_like(fpsi), fpsi, data, 0.7, model)
    ref = torch.zeros((ntheta, nz, n), dtype=torch.complex64, device="cuda")
    op.adj(ref, res, scale=0.5)
    out = torch.zeros_like(ref)
    op.adj_resid(out, fpsi, data, 0.7, model, scale=0.5)
    assert rel(out.cpu().numpy(), ref.cpu().numpy()) <= 1e-6


def test_operators_capture_in_a_cuda_graph():
    """fwd/adj allocate nothing and never synchronise, so one CUDA graph holds a
    whole operator step; replays equal eager calls bit for bit."""
    rng = np.random.default_rng(21)
    n, nz, nt = 64, 16, 24
    theta = np.sort(rng.uniform(0, np.pi, nt)).astype(np.float32)
    rop, _ = make_radon(n, nz, nt, theta)
    pop, _, _, _ = make_ptycho(3, 140, 140, 5, 128, 128, rng)
    f = dev(crand(rng, (nz, n, n)))
    g = dev(crand(rng, (nt, nz, n)))
    psi = dev(crand(rng, (3, 140, 140)))
    frames_in = dev(crand(rng, (3, 5, 128, 128)))
    data = dev(rng.poisson(2.0, (3, 5, 128, 128)).astype(np.float32))
    outs = [torch.zeros((nt, nz, n), dtype=torch.complex64, device="cuda"),
            torch.zeros((nz, n, n), dtype=torch.complex64, device="cuda"),
            torch.zeros((3, 5, 128, 128), dtype=torch.complex64, device="cuda"),
            torch.zeros((3, 140, 140), dtype=torch.complex64, device="cuda"),
            torch.zeros((3, 140, 140), dtype=torch.complex64, device="cuda")]

    def step():
        rop.fwd(outs[0], f)
        rop.adj(outs[1], g)
        pop.fwd(outs[2], psi, scale=0.5)
        pop.adj(outs[3], frames_in)
        pop.adj_resid(outs[4], frames_in, data, 0.3, 0)

    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        step()
    torch.cuda.current_stream().wait_stream(s)
    eager = [o.clone() for o in outs]
    for o in outs:
        o.zero_()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        step()
    for _ in range(2):
        for o in outs:
            o.zero_()
        graph.replay()
        torch.cuda.synchronize()
        for o, e in zip(outs, eager):
            assert torch.equal(o, e)


@pytest.mark.parametrize("det,nprb", [(32, 32), (128, 96), (128, 128)])
def test_ptycho_uneven_scan_counts(det, nprb):
    """Per-angle scan counts drawn from [lo, hi] on a jittered spiral, padded to the
    largest count with the -1 sentinel (kernels.cuh:256,280): every padded scan is
    skipped by both transforms.  The 128 x 128 probe case runs 24 angles, so the
    adjoint's blocks walk runs of valid and skipped frames."""
    from ptychotomo_b200 import ptychofft, synthetic
    rng = np.random.default_rng(det + nprb)
    nt, n, nz = (24 if nprb == 128 else 4), 160, 150
    counts = rng.integers(5, 19, nt)
    scan = synthetic.jittered_spiral_scan(nt, n, nz, nprb, counts, jitter=3.0, seed=det)
    nscan = scan.shape[2]
    assert (scan < 0).any()
    prb = crand(rng, (nprb, nprb))
    op = ptychofft(nt, nz, n, nt, nscan, det, det, nprb)
    op.setobj(dev(scan), dev(prb))
    orc = PtychoFFT(nt, nz, n, nt, nscan, det, det, nprb)
    orc.setobj(scan, prb)
    f = crand(rng, (nt, nz, n))
    g = crand(rng, (nt, nscan, det, det))
    got = p_fwd(op, dev(f)).cpu().numpy()
    assert rel(got, orc.fwd(f)) <= TOL
    for t in range(nt):   # padded scans leave their frames untouched (zero here)
        assert not np.any(got[t, counts[t]:])
    assert rel(p_adj(op, dev(g)).cpu().numpy(), orc.adj(g)) <= TOL


@pytest.mark.parametrize("n,nz,ntheta", [(32, 8, 24), (64, 5, 40)])
def test_radon_m4_variant_vs_oracle(n, nz, ntheta):
    """The M = 4 precision variant (pt_radon_create_ex) against the oracle run with
    the same N, M and mu: the gridding approximation is shared, so the two agree
    to FP32 accuracy; fwd and adj stay adjoint."""
    rng = np.random.default_rng(n + 4)
    theta = np.sort(rng.uniform(0, np.pi, ntheta)).astype(np.float32)
    from ptychotomo_b200 import radonusfft
    op = radonusfft(ntheta, nz, n, m_override=4)
    assert op.M == 4
    op.setobj(dev(theta))
    x = torch.empty((ntheta, op.N), dtype=torch.float32, device="cuda")
    y = torch.empty_like(x)
    op.get_xy(x, y)
    torch.cuda.synchronize()
    orc = RadonUSFFT(ntheta, nz, n, params=(op.N, op.M, op.mu))
    orc.setobj(theta, xy=(x.cpu().numpy(), y.cpu().numpy()))
    f = crand(rng, (nz, n, n))
    g = crand(rng, (ntheta, nz, n))
    assert rel(radon_fwd(op, dev(f)).cpu().numpy(), orc.fwd(f)) <= TOL
    assert rel(radon_adj(op, dev(g)).cpu().numpy(), orc.adj(g)) <= TOL


@pytest.mark.parametrize("det,nprb", [(32, 16), (128, 128)])
def test_ptycho_every_scan_skipped(det, nprb):
    """All scans carry the -1 sentinel (kernels.cuh:256,280): the forward leaves
    zero frames and the adjoint a zero object."""
    from ptychotomo_b200 import ptychofft
    rng = np.random.default_rng(det)
    nt, nz, n, nscan = 3, 130, 140, 4
    scan = -np.ones((2, nt, nscan), np.float32)
    op = ptychofft(nt, nz, n, nt, nscan, det, det, nprb)
    op.setobj(dev(scan), dev(crand(rng, (nprb, nprb))))
    g = torch.full((nt, nscan, det, det), 7.0 + 1j, dtype=torch.complex64, device="cuda")
    op.fwd(g, dev(crand(rng, (nt, nz, n))))
    f = torch.full((nt, nz, n), 7.0 + 1j, dtype=torch.complex64, device="cuda")
    op.adj(f, dev(crand(rng, (nt, nscan, det, det))))
    torch.cuda.synchronize()
    assert not g.abs().any() and not f.abs().any()


def test_radon_largest_width_vs_oracle():
    """n = 512 (the largest compiled width, G = 1536) on a thin case."""
    rng = np.random.default_rng(512)
    n, nz, nt = 512, 3, 12
    theta = np.sort(rng.uniform(0, np.pi, nt)).astype(np.float32)
    op, orc = make_radon(n, nz, nt, theta)
    f = crand(rng, (nz, n, n))
    g = crand(rng, (nt, nz, n))
    assert rel(radon_fwd(op, dev(f)).cpu().numpy(), orc.fwd(f)) <= TOL
    assert rel(radon_adj(op, dev(g)).cpu().numpy(), orc.adj(g)) <= TOL
