"""Probe and scan generators of the reference package (host side, NumPy).

``probe`` and ``scanner3`` give the same arrays as the reference's
src/ptychotomo/objects.py:4-16 and :19-65 for the same arguments (and, for
``randscan=True``, the same state of NumPy's global generator), so scripts
written against the reference run unchanged.  The float expressions that
decide a probe pixel's zone and the order of the random draws are the
reference's; the plot that ``scanner3(save=True)`` draws with matplotlib is
not provided.
"""
from __future__ import annotations

import warnings

import numpy as np


def probe(size, maxint=1, rin=0.8, rout=1):
    """Flat-top probe: amplitude 1 inside radius rin, a linear edge out to rout
    (both relative to the corner distance), phase 0.2 x amplitude, peak
    intensity maxint (objects.py:4-16).  complex128 [size, size]."""
    pos = np.arange(size, dtype=np.float64) + 0.5 - size / 2
    rs = np.sqrt(pos[:, None] ** 2 + pos[None, :] ** 2)   # rows, then columns, as objects.py:6
    far = rs.max()
    r_out = np.sqrt(2) * 0.5 * rout * far + 1.0
    r_in = np.sqrt(2) * 0.5 * rin * far
    edge = (rs > r_in) & (rs < r_out)
    amp = np.where(rs < r_in, 1.0, 0.0)
    amp[edge] = (r_out - rs[edge]) / (r_out - r_in)
    amp = amp.astype(np.float32)
    return np.sqrt(maxint) * amp * np.exp(1j * 0.2 * amp)


def scanner3(theta, shape, sx, sy, psize, spiral=0, randscan=False, save=False):
    """Raster scan positions per angle (objects.py:19-65): a grid of step
    (sx, sy) over an object of shape (nz, n) for a psize probe, shifted along
    x by spiral * (angle index + 1) mod sx; with randscan, one random offset
    of up to half a step per angle plus up to a twentieth of a step per
    position (NumPy's global generator).  Positions are then clamped into the
    object.  float32 [2, ntheta, nscan]: x (column) then y (row)."""
    if save:
        warnings.warn("scanner3: the scan plot (save=True) is not provided; positions only")
    xs = np.arange(0, shape[1] - psize + 1, sx)
    ys = np.arange(0, shape[0] - psize + 1, sy)
    grid_x = np.tile(xs, len(ys))      # np.meshgrid(xs, ys) read row by row
    grid_y = np.repeat(ys, len(xs))
    nt, nscan = len(theta), grid_x.size
    scan = np.empty((2, nt, nscan), dtype=np.float32)
    shift = spiral
    for m in range(nt):
        scan[0, m] = grid_x + np.mod(shift, sx)
        scan[1, m] = grid_y
        shift += spiral
        if randscan:   # the reference's draw order: x, y for the angle, then x, y per position
            scan[0, m] += sx * (np.random.random(1) - 0.5) * 1
            scan[1, m] += sy * (np.random.random(1) - 0.5) * 1
            scan[0, m] += sx * (np.random.random(nscan) - 0.5) * 0.1
            scan[1, m] += sy * (np.random.random(nscan) - 0.5) * 0.1
    x, y = scan[0], scan[1]
    x[np.round(x) < 0] = 0
    y[np.round(y) < 0] = 0
    x[np.round(x) > shape[1] - psize] = shape[1] - psize - 1
    y[np.round(y) > shape[0] - psize] = shape[0] - psize - 1
    return scan
