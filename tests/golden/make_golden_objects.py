"""Golden vectors for the scan and probe generators, from the reference itself.

Loads the reference's src/ptychotomo/objects.py (it needs only NumPy) from
the reference source tree given on the command line and stores probe(...) and scanner3(...) outputs for a few
argument sets; the random-scan cases seed NumPy's global generator first,
as a caller of scanner3(randscan=True) would.

    python tests/golden/make_golden_objects.py REFERENCE_ROOT
"""
from __future__ import annotations

import importlib.util
import sys
from pathlib import Path

import numpy as np

OUT = Path(__file__).resolve().parent / "objects.npz"
PROBES = [(16, 1.0, 0.8, 1.0), (16, 0.1, 0.8, 1.0), (64, 1.0, 0.6, 1.0), (33, 2.0, 0.8, 0.9)]
# (ntheta, shape, sx, sy, psize, spiral, randscan, seed)
SCANS = [(7, (128, 128), 8, 8, 16, 0, False, 0), (5, (64, 96), 6, 5, 16, 2, False, 0),
         (6, (128, 128), 8, 8, 16, 0, True, 3), (4, (80, 100), 7, 9, 20, 3, True, 4)]


def main(ref_root):
    spec = importlib.util.spec_from_file_location("ref_objects", Path(ref_root) / "src/ptychotomo/objects.py")
    ref = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(ref)
    out = {}
    for i, (size, maxint, rin, rout) in enumerate(PROBES):
        out["probe%d" % i] = ref.probe(size, maxint, rin, rout)
    for i, (nt, shape, sx, sy, psize, spiral, rnd, seed) in enumerate(SCANS):
        theta = np.linspace(0, np.pi, nt).astype("float32")
        np.random.seed(seed)
        out["scan%d" % i] = ref.scanner3(theta, shape, sx, sy, psize, spiral=spiral, randscan=rnd, save=False)
    np.savez(OUT, **out)
    print("wrote", OUT, {k: (v.shape, v.dtype) for k, v in out.items()})


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(__doc__)
    main(sys.argv[1])
