"""The oracle's sub-pixel scan model (CPU): the Fourier-shift probe equals
the separable Dirichlet-kernel form the device tables use, integer offsets
are exact circular shifts, and integer scans reduce the model to the
reference's (whose per-scan phase is then 1)."""
import numpy as np
import pytest

from oracle.ptycho import PtychoFFT, shift_probe


def dirichlet(t, P):
    t = np.asarray(t, float)
    out = np.where(t == np.floor(t), (np.mod(t, P) == 0).astype(float), 0.0)
    m = t != np.floor(t)
    a = np.pi * t[m] / P
    out[m] = np.sin(np.pi * t[m]) / (P * (np.tan(a) if P % 2 == 0 else np.sin(a)))
    return out


@pytest.mark.parametrize("P", [16, 17, 64])
def test_fourier_shift_is_the_dirichlet_form(P):
    rng = np.random.default_rng(P)
    prb = rng.standard_normal((P, P)) + 1j * rng.standard_normal((P, P))
    i = np.arange(P)
    for dx, dy in ((0.3125, -0.4375), (0.5, -0.5), (-0.0625, 0.0)):
        mx = dirichlet(i[:, None] - dx - i[None, :], P)
        my = dirichlet(i[:, None] - dy - i[None, :], P)
        want = shift_probe(prb, dx, dy)
        assert np.abs(mx @ prb @ my.T - want).max() <= 1e-12 * np.abs(want).max()


def test_integer_offsets_are_rolls():
    rng = np.random.default_rng(1)
    prb = rng.standard_normal((12, 12)) + 1j * rng.standard_normal((12, 12))
    assert np.allclose(shift_probe(prb, 0, 0), prb, atol=1e-13)
    assert np.allclose(shift_probe(prb, 1, -2), np.roll(np.roll(prb, 1, 0), -2, 1), atol=1e-12)


def test_integer_scans_reduce_to_the_reference_model():
    rng = np.random.default_rng(2)
    nt, ns, nz, n, det, P = 2, 3, 24, 24, 16, 12
    scan = np.round(rng.uniform(0, n - P, (2, nt, ns))).astype(np.float32)
    prb = rng.standard_normal((P, P)) + 1j * rng.standard_normal((P, P))
    f = rng.standard_normal((nt, nz, n)) + 1j * rng.standard_normal((nt, nz, n))
    a = PtychoFFT(nt, nz, n, nt, ns, det, det, P)
    a.setobj(scan, prb)
    b = PtychoFFT(nt, nz, n, nt, ns, det, det, P)
    b.setobj(scan, prb)
    b.set_subpixel(16)
    assert np.allclose(a.fwd(f), b.fwd(f), rtol=0, atol=1e-12)
