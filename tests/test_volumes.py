"""Volume files (ptychotomo_b200.volumes): the dxchange read_tiff/write_tiff
calls of the reference's driver script (test.py:45-46, 90-93), plus .npy and
.raw.  Round trips for every sample type, the page chain of a stack, a
big-endian multi-strip file built by hand, and files exchanged with Pillow's
TIFF codec where Pillow is installed."""
import os
import struct

import numpy as np
import pytest

from ptychotomo_b200 import volumes


@pytest.mark.parametrize("dtype", [np.float32, np.float64, np.uint8, np.uint16, np.int16, np.int32])
@pytest.mark.parametrize("shape", [(5, 7, 9), (1, 4, 6), (3, 1, 1)])
def test_tiff_round_trip(tmp_path, dtype, shape):
    rng = np.random.default_rng(0)
    a = (rng.standard_normal(shape) * 100).astype(dtype)
    path = volumes.write_tiff(a, str(tmp_path / "sub" / "vol"))
    assert path.endswith("vol.tiff") and os.path.exists(path)
    b = volumes.read_tiff(path)
    want = a[0] if shape[0] == 1 else a
    assert b.dtype == a.dtype and b.shape == want.shape
    assert np.array_equal(b, want)


def test_tiff_2d_and_names(tmp_path):
    a = np.arange(12, dtype=np.float32).reshape(3, 4)
    p1 = volumes.write_tiff(a, str(tmp_path / "x.tif"))
    assert p1.endswith("x.tif")
    assert np.array_equal(volumes.read_tiff(p1), a)
    p2 = volumes.write_tiff(a + 1, str(tmp_path / "x.tif"), overwrite=False)
    p3 = volumes.write_tiff(a + 2, str(tmp_path / "x.tif"), overwrite=False)
    assert p2.endswith("x-1.tif") and p3.endswith("x-2.tif")
    assert np.array_equal(volumes.read_tiff(p1), a) and np.array_equal(volumes.read_tiff(p3), a + 2)
    assert np.array_equal(volumes.read_tiff(volumes.write_tiff(a, str(tmp_path / "x.tif"))), a)


def test_tiff_rejects(tmp_path):
    with pytest.raises(TypeError):
        volumes.write_tiff(np.ones((2, 2), np.complex64), str(tmp_path / "c"))
    with pytest.raises(ValueError):
        volumes.write_tiff(np.ones(4, np.float32), str(tmp_path / "c"))
    bad = tmp_path / "bad.tiff"
    bad.write_bytes(b"not a tiff")
    with pytest.raises(ValueError):
        volumes.read_tiff(str(bad))


def _big_endian_stack(pages, rows_per_strip):
    """A big-endian TIFF stack of int16 pages, several strips per page, with
    the strip offset/count arrays stored out of line."""
    n, h, w = pages.shape
    out = bytearray(b"MM\x00*" + struct.pack(">I", 8))
    nstrips = -(-h // rows_per_strip)
    for p in range(n):
        ifd_at = len(out)
        ntags = 8
        arrays_at = ifd_at + 2 + 12 * ntags + 4
        data_at = arrays_at + 8 * nstrips
        raw = pages[p].astype(">i2").tobytes()
        offs, cnts = [], []
        for s in range(nstrips):
            r0, r1 = s * rows_per_strip, min(h, (s + 1) * rows_per_strip)
            offs.append(data_at + r0 * w * 2)
            cnts.append((r1 - r0) * w * 2)
        nxt = data_at + len(raw)
        nxt += nxt & 1
        tags = [(256, 4, 1, struct.pack(">I", w)), (257, 4, 1, struct.pack(">I", h)),
                (258, 3, 1, struct.pack(">HH", 16, 0)), (259, 3, 1, struct.pack(">HH", 1, 0)),
                (273, 4, nstrips, struct.pack(">I", arrays_at) if nstrips > 1 else struct.pack(">I", offs[0])),
                (277, 3, 1, struct.pack(">HH", 1, 0)),
                (279, 4, nstrips, struct.pack(">I", arrays_at + 4 * nstrips) if nstrips > 1 else struct.pack(">I", cnts[0])),
                (339, 3, 1, struct.pack(">HH", 2, 0))]
        out += struct.pack(">H", ntags)
        for tag, typ, cnt, val in tags:
            out += struct.pack(">HHI", tag, typ, cnt) + val
        out += struct.pack(">I", nxt if p + 1 < n else 0)
        out += struct.pack(">%dI" % nstrips, *offs) + struct.pack(">%dI" % nstrips, *cnts)
        out += raw
        if len(out) & 1:
            out += b"\x00"
    return bytes(out)


def test_tiff_reads_big_endian_multi_strip(tmp_path):
    rng = np.random.default_rng(1)
    a = rng.integers(-3000, 3000, (3, 11, 5)).astype(np.int16)
    f = tmp_path / "be.tiff"
    f.write_bytes(_big_endian_stack(a, rows_per_strip=4))
    b = volumes.read_tiff(str(f))
    assert b.dtype == np.int16 and np.array_equal(b, a)


def test_tiff_against_pillow(tmp_path):
    Image = pytest.importorskip("PIL.Image")
    rng = np.random.default_rng(2)
    a = rng.standard_normal((4, 6, 10)).astype(np.float32)
    path = volumes.write_tiff(a, str(tmp_path / "ours"))
    with Image.open(path) as im:
        got = []
        for k in range(a.shape[0]):
            im.seek(k)
            got.append(np.array(im, dtype=np.float32))
    assert np.array_equal(np.stack(got), a)
    theirs = str(tmp_path / "theirs.tiff")
    imgs = [Image.fromarray(s) for s in a]
    imgs[0].save(theirs, save_all=True, append_images=imgs[1:])
    assert np.array_equal(volumes.read_tiff(theirs), a)


@pytest.mark.parametrize("ext", [".npy", ".tiff", ".raw"])
def test_volume_dispatch(tmp_path, ext):
    rng = np.random.default_rng(3)
    a = rng.standard_normal((3, 4, 5)).astype(np.float32)
    if ext == ".npy":
        a = (a + 1j * a[::-1]).astype(np.complex64)
    path = volumes.write_volume(a, str(tmp_path / ("v" + ext)))
    b = volumes.read_volume(path, shape=a.shape, dtype=a.dtype)
    assert b.dtype == a.dtype and np.array_equal(b, a)
    if ext == ".raw":
        with pytest.raises(ValueError):
            volumes.read_volume(path)
        with pytest.raises(ValueError):
            volumes.read_volume(path, shape=(2, 2), dtype=np.float32)
