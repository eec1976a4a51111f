"""ptychotomo_b200.probe / scanner3 against the reference's own generators
(src/ptychotomo/objects.py), through the fixtures that
tests/golden/make_golden_objects.py wrote from it: bit-identical arrays,
including the random scans for a seeded global NumPy generator."""
from pathlib import Path

import numpy as np
import pytest

import ptychotomo_b200 as pt

GOLD = np.load(Path(__file__).parent / "golden" / "objects.npz")
PROBES = [(16, 1.0, 0.8, 1.0), (16, 0.1, 0.8, 1.0), (64, 1.0, 0.6, 1.0), (33, 2.0, 0.8, 0.9)]
SCANS = [(7, (128, 128), 8, 8, 16, 0, False, 0), (5, (64, 96), 6, 5, 16, 2, False, 0),
         (6, (128, 128), 8, 8, 16, 0, True, 3), (4, (80, 100), 7, 9, 20, 3, True, 4)]


@pytest.mark.parametrize("i", range(len(PROBES)))
def test_probe_matches_reference(i):
    p = pt.probe(*PROBES[i])
    assert p.dtype == GOLD["probe%d" % i].dtype
    assert np.array_equal(p, GOLD["probe%d" % i])


@pytest.mark.parametrize("i", range(len(SCANS)))
def test_scanner3_matches_reference(i):
    nt, shape, sx, sy, psize, spiral, rnd, seed = SCANS[i]
    theta = np.linspace(0, np.pi, nt).astype("float32")
    np.random.seed(seed)
    s = pt.scanner3(theta, shape, sx, sy, psize, spiral=spiral, randscan=rnd)
    assert s.dtype == np.float32
    assert np.array_equal(s, GOLD["scan%d" % i])
    # every patch lies inside the object, as the operators require
    corners = np.round(s)
    assert corners.min() >= 0
    assert corners[0].max() <= shape[1] - psize and corners[1].max() <= shape[0] - psize


def test_scanner3_save_warns():
    with pytest.warns(UserWarning, match="not provided"):
        pt.scanner3(np.zeros(2, np.float32), (32, 32), 8, 8, 16, save=True)
