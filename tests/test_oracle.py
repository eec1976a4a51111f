"""CPU checks of the oracle itself.

* the gridded USFFT restatement against the complex128 direct-sum NUDFT it
  approximates (Gaussian gridding accuracy ~1e-7 at M = 7);
* adjoint identities of the restated operators (border-zero inputs, since
  the reference's pad2/pad edge replication is not adjoint to its crop);
* the ptycho restatement against dense DFTs;
* pinning: the restatement against the golden vectors that the reference's
  own CUDA operators produced (tests/golden/*.npz, tests/golden/make_golden.py).
"""
from pathlib import Path

import numpy as np
import pytest

from oracle.nudft import ptycho_fwd_exact, radon_fwd_exact
from oracle.ptycho import PtychoFFT, roundf
from oracle.usfft import RadonUSFFT, usfft_params

GOLDEN = Path(__file__).parent / "golden"


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def crand(rng, shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def test_usfft_params_match_reference_formula():
    for n in (8, 16, 128, 256, 512):
        N, M, mu = usfft_params(n)
        assert N == 3 * n // 2 and M == 7
        assert abs(mu - 13.815510557964274 / (2 * N * N)) / mu < 1e-6


@pytest.mark.parametrize("n,nz,ntheta", [(16, 2, 12), (32, 3, 24), (64, 2, 30)])
def test_usfft_vs_direct_nudft(n, nz, ntheta):
    rng = np.random.default_rng(n)
    theta = np.linspace(0, np.pi, ntheta, endpoint=False).astype(np.float32)
    op = RadonUSFFT(ntheta, nz, n)
    op.setobj(theta)
    f = crand(rng, (nz, n, n))
    assert rel(op.fwd(f), radon_fwd_exact(f, theta, n)) < 1e-6


@pytest.mark.parametrize("n,nz,ntheta", [(16, 2, 12), (48 // 3 * 2, 3, 20)])
def test_usfft_adjoint_identity(n, nz, ntheta):
    rng = np.random.default_rng(1)
    theta = np.sort(rng.uniform(0, np.pi, ntheta)).astype(np.float32)
    op = RadonUSFFT(ntheta, nz, n)
    op.setobj(theta)
    f = crand(rng, (nz, n, n))
    f[:, [0, -1], :] = 0
    f[:, :, [0, -1]] = 0
    g = crand(rng, (ntheta, nz, n))
    g[..., [0, -1]] = 0
    a = np.vdot(op.fwd(f), g)
    b = np.vdot(f, op.adj(g))
    assert abs(a - b) / abs(a) < 1e-12


def test_roundf_is_half_away_from_zero():
    v = np.array([0.5, 1.5, 2.5, -0.5, -1.5, 0.49999997, 10.67], np.float32)
    assert roundf(v).tolist() == [1, 2, 3, -1, -2, 0, 11]


@pytest.mark.parametrize("det,nprb", [(16, 16), (32, 16), (64, 16)])
def test_ptycho_vs_dense_dft_and_adjoint(det, nprb):
    rng = np.random.default_rng(det)
    nt, nz, n, ns = 2, 40, 36, 5
    op = PtychoFFT(nt, nz, n, nt, ns, det, det, nprb)
    scan = np.empty((2, nt, ns), np.float32)
    scan[0] = rng.uniform(0, n - nprb - 0.5, (nt, ns))
    scan[1] = rng.uniform(0, nz - nprb - 0.5, (nt, ns))
    scan[:, 1, 2] = -1
    op.setobj(scan, crand(rng, (nprb, nprb)))
    f = crand(rng, (nt, nz, n))
    g = op.fwd(f)
    assert rel(g, ptycho_fwd_exact(op, f)) < 1e-12
    assert np.all(g[1, 2] == 0)                       # sentinel scan stays zero
    y = crand(rng, g.shape)
    assert abs(np.vdot(g, y) - np.vdot(f, op.adj(y))) / abs(np.vdot(g, y)) < 1e-12


def test_ptycho_rejects_patch_outside_object():
    op = PtychoFFT(1, 32, 32, 1, 1, 16, 16, 16)
    with pytest.raises(ValueError):
        op.setobj(np.array([[[17.0]], [[0.0]]], np.float32), np.ones((16, 16)))


GOLDEN_RADON = sorted(GOLDEN.glob("radon_*.npz"))
GOLDEN_PTYCHO = sorted(GOLDEN.glob("ptycho_*.npz"))


@pytest.mark.parametrize("path", GOLDEN_RADON, ids=[p.stem for p in GOLDEN_RADON])
def test_oracle_pinned_to_reference_radon(path):
    d = np.load(path)
    ntheta, nz, n = d["g"].shape
    op = RadonUSFFT(ntheta, nz, n)
    op.setobj(d["theta"], xy=(d["x"], d["y"]))
    assert rel(op.fwd(d["f"]), d["fwd"]) < 2e-6
    assert rel(op.adj(d["g"]), d["adj"]) < 2e-6


@pytest.mark.parametrize("path", GOLDEN_RADON, ids=[p.stem for p in GOLDEN_RADON])
def test_oracle_cpu_geometry_close_to_reference_radon(path):
    """With float32 cos/sin instead of the GPU's __cosf/__sinf tables the
    oracle still agrees with the reference to well inside 1e-5."""
    d = np.load(path)
    ntheta, nz, n = d["g"].shape
    op = RadonUSFFT(ntheta, nz, n)
    op.setobj(d["theta"])
    assert rel(op.fwd(d["f"]), d["fwd"]) < 1e-5
    assert rel(op.adj(d["g"]), d["adj"]) < 1e-5


@pytest.mark.parametrize("path", GOLDEN_PTYCHO, ids=[p.stem for p in GOLDEN_PTYCHO])
def test_oracle_pinned_to_reference_ptycho(path):
    d = np.load(path)
    nt, ns, det, _ = d["g"].shape
    _, nz, n = d["f"].shape
    op = PtychoFFT(nt, nz, n, nt, ns, det, det, d["prb"].shape[0])
    op.setobj(d["scan"], d["prb"])
    assert rel(op.fwd(d["f"]), d["fwd"]) < 2e-6
    assert rel(op.adj(d["g"]), d["adj"]) < 2e-6


def test_golden_vectors_present():
    """The oracle must be pinned: fixtures generated from the reference exist."""
    assert GOLDEN_RADON and GOLDEN_PTYCHO, "run tests/golden/make_golden.py on a GPU"


def test_usfft_exact_adjoint_identity_full_support():
    """adj_exact is the adjoint of fwd for inputs that do not vanish on their
    borders (where the reference's adj is not: it replicates edges)."""
    from oracle.usfft import RadonUSFFT
    n, nz, nt = 32, 2, 20
    rng = np.random.default_rng(9)
    op = RadonUSFFT(nt, nz, n)
    op.setobj(np.linspace(0, np.pi, nt, endpoint=False).astype(np.float32))
    f = rng.standard_normal((nz, n, n)) + 1j * rng.standard_normal((nz, n, n))
    g = rng.standard_normal((nt, nz, n)) + 1j * rng.standard_normal((nt, nz, n))
    a = np.vdot(op.fwd(f), g)
    b = np.vdot(f, op.adj_exact(g))
    assert abs(a - b) / abs(a) < 1e-12
    assert abs(a - np.vdot(f, op.adj(g))) / abs(a) > 1e-2     # the reference's adjoint is not exact here
    f0 = f.copy()
    f0[:, 0, :] = f0[:, -1, :] = f0[:, :, 0] = f0[:, :, -1] = 0
    g0 = g.copy()
    g0[:, :, 0] = g0[:, :, -1] = 0
    inner = (slice(None), slice(1, -1), slice(1, -1))
    assert np.allclose(op.adj_exact(g0)[inner], op.adj(g0)[inner], rtol=0, atol=1e-12 * np.abs(op.adj(g0)).max())
