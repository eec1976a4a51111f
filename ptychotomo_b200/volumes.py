"""Volume and image-stack files: the reader and writer the reference's driver
script gets from dxchange (test.py:45-46 reads the delta/beta phantoms with
``dxchange.read_tiff``; test.py:90-93 writes delta, beta and the angle and
amplitude of psi with ``dxchange.write_tiff``).

TIFF here is baseline TIFF 6.0 without compression: one page per slice of a
3-D array (a 2-D array is one page), one strip per page, a single sample per
pixel of an integer or IEEE float type (SampleFormat 1, 2 or 3).  The writer
produces little-endian files; the reader takes either byte order and any
strip layout of uncompressed single-sample pages, which covers what tifffile
(dxchange's back end) writes for these arrays.  ``.npy`` and headerless
``.raw`` volumes are handled too.  Host-side only: arrays are NumPy.
"""
from __future__ import annotations

import os
import struct

import numpy as np

__all__ = ["write_tiff", "read_tiff", "write_volume", "read_volume"]

# TIFF tags used
_WIDTH, _LENGTH, _BITS, _COMPRESSION, _PHOTOMETRIC = 256, 257, 258, 259, 262
_STRIP_OFFSETS, _SPP, _ROWS_PER_STRIP, _STRIP_BYTES = 273, 277, 278, 279
_PLANAR, _SAMPLE_FORMAT = 284, 339
_SHORT, _LONG = 3, 4
_TYPE_SIZE = {1: 1, 2: 1, 3: 2, 4: 4, 5: 8, 6: 1, 7: 1, 8: 2, 9: 4, 10: 8, 11: 4, 12: 8, 16: 8}
_TYPE_CODE = {1: "B", 3: "H", 4: "I", 6: "b", 8: "h", 9: "i", 11: "f", 12: "d", 16: "Q"}


def _sample_format(dtype: np.dtype) -> int:
    if dtype.kind == "u":
        return 1
    if dtype.kind == "i":
        return 2
    if dtype.kind == "f":
        return 3
    raise TypeError("TIFF pages hold integer or real samples, not %s" % dtype)


def _tiff_name(fname: str) -> str:
    base = os.path.basename(fname)
    return fname if os.path.splitext(base)[1] else fname + ".tiff"


def write_tiff(data, fname: str, dtype=None, overwrite: bool = True) -> str:
    """Write a 2-D or 3-D real array as a multi-page TIFF (one page per
    leading index); dxchange.write_tiff's call shape.  ``.tiff`` is appended
    when the name has no extension and missing folders are created.  With
    overwrite=False an existing file is kept and the new one is named
    ``<stem>-1``, ``<stem>-2``, ... .  Returns the path written."""
    a = np.asarray(data)
    if dtype is not None:
        a = a.astype(dtype)
    if np.iscomplexobj(a):
        raise TypeError("write_tiff: complex arrays have no TIFF sample type; write .real/.imag")
    if a.dtype == np.bool_:
        a = a.astype(np.uint8)
    if a.ndim == 2:
        a = a[None]
    if a.ndim != 3 or a.shape[1] == 0 or a.shape[2] == 0:
        raise ValueError("write_tiff: expected a 2-D or 3-D array, got shape %s" % (a.shape,))
    a = np.ascontiguousarray(a.astype(a.dtype.newbyteorder("<")))
    fmt = _sample_format(a.dtype)
    path = _tiff_name(fname)
    if not overwrite and os.path.exists(path):
        stem, ext = os.path.splitext(path)
        k = 1
        while os.path.exists("%s-%d%s" % (stem, k, ext)):
            k += 1
        path = "%s-%d%s" % (stem, k, ext)
    folder = os.path.dirname(path)
    if folder:
        os.makedirs(folder, exist_ok=True)
    pages, h, w = a.shape
    bits = 8 * a.dtype.itemsize
    page_bytes = h * w * a.dtype.itemsize
    ntags = 11
    ifd_size = 2 + 12 * ntags + 4
    out = bytearray(b"II*\x00" + struct.pack("<I", 8))
    # layout: header, then for each page its IFD followed by its pixel strip
    pos = 8
    for p in range(pages):
        strip = pos + ifd_size
        nxt = strip + page_bytes
        nxt += nxt & 1                       # IFDs start on a word boundary
        tags = [(_WIDTH, _LONG, w), (_LENGTH, _LONG, h), (_BITS, _SHORT, bits), (_COMPRESSION, _SHORT, 1),
                (_PHOTOMETRIC, _SHORT, 1), (_STRIP_OFFSETS, _LONG, strip), (_SPP, _SHORT, 1),
                (_ROWS_PER_STRIP, _LONG, h), (_STRIP_BYTES, _LONG, page_bytes), (_PLANAR, _SHORT, 1),
                (_SAMPLE_FORMAT, _SHORT, fmt)]
        assert len(tags) == ntags
        ifd = bytearray(struct.pack("<H", ntags))
        for tag, typ, val in tags:           # values fit in the 4-byte field
            ifd += struct.pack("<HHI", tag, typ, 1) + (struct.pack("<HH", val, 0) if typ == _SHORT
                                                        else struct.pack("<I", val))
        ifd += struct.pack("<I", nxt if p + 1 < pages else 0)
        out += ifd + a[p].tobytes()
        if len(out) & 1:
            out += b"\x00"
        pos = len(out)
        if pos >= 1 << 32:
            raise ValueError("write_tiff: the stack exceeds the 4 GiB of a classic TIFF")
    with open(path, "wb") as fh:
        fh.write(bytes(out))
    return path


def _read_ifd(buf: bytes, off: int, e: str):
    n = struct.unpack_from(e + "H", buf, off)[0]
    tags = {}
    for k in range(n):
        tag, typ, cnt = struct.unpack_from(e + "HHI", buf, off + 2 + 12 * k)
        if typ not in _TYPE_SIZE:
            continue
        size = _TYPE_SIZE[typ] * cnt
        voff = off + 2 + 12 * k + 8
        if size > 4:
            voff = struct.unpack_from(e + "I", buf, voff)[0]
        if typ in _TYPE_CODE:
            tags[tag] = list(struct.unpack_from(e + _TYPE_CODE[typ] * cnt, buf, voff))
    nxt = struct.unpack_from(e + "I", buf, off + 2 + 12 * n)[0]
    return tags, nxt


def read_tiff(fname: str) -> np.ndarray:
    """Read a baseline uncompressed TIFF (one sample per pixel) into a NumPy
    array: 2-D for one page, 3-D [page, row, column] for several pages of
    the same size and type (dxchange.read_tiff's result)."""
    with open(fname, "rb") as fh:
        buf = fh.read()
    if buf[:4] == b"II*\x00":
        e = "<"
    elif buf[:4] == b"MM\x00*":
        e = ">"
    else:
        raise ValueError("read_tiff: %s is not a classic TIFF" % fname)
    off = struct.unpack_from(e + "I", buf, 4)[0]
    pages = []
    seen = set()
    while off:
        if off in seen or off + 2 > len(buf):
            raise ValueError("read_tiff: %s has a broken page chain" % fname)
        seen.add(off)
        tags, off = _read_ifd(buf, off, e)
        w, h = tags[_WIDTH][0], tags[_LENGTH][0]
        if tags.get(_COMPRESSION, [1])[0] != 1:
            raise ValueError("read_tiff: compressed pages are not supported")
        if tags.get(_SPP, [1])[0] != 1:
            raise ValueError("read_tiff: only single-sample pages are supported")
        bits = tags.get(_BITS, [1])[0]
        fmt = tags.get(_SAMPLE_FORMAT, [1])[0]
        kind = {1: "u", 2: "i", 3: "f"}.get(fmt)
        if kind is None or bits % 8:
            raise ValueError("read_tiff: unsupported sample format %d / %d bits" % (fmt, bits))
        dt = np.dtype("%s%s%d" % (e, kind, bits // 8))
        data = b"".join(buf[o:o + c] for o, c in zip(tags[_STRIP_OFFSETS], tags[_STRIP_BYTES]))
        if len(data) < w * h * dt.itemsize:
            raise ValueError("read_tiff: %s has a truncated page" % fname)
        pages.append(np.frombuffer(data, dtype=dt, count=w * h).reshape(h, w).astype(dt.newbyteorder("=")))
    if not pages:
        raise ValueError("read_tiff: %s has no pages" % fname)
    if len(pages) == 1:
        return pages[0]
    if any(p.shape != pages[0].shape or p.dtype != pages[0].dtype for p in pages):
        raise ValueError("read_tiff: pages of different sizes or types")
    return np.stack(pages)


def write_volume(data, fname: str) -> str:
    """Write a volume by extension: ``.npy`` (any dtype, complex included),
    ``.tif``/``.tiff`` (real), ``.raw`` (the bytes, C order, native byte
    order; shape and dtype are the caller's to keep)."""
    ext = os.path.splitext(fname)[1].lower()
    folder = os.path.dirname(fname)
    if folder:
        os.makedirs(folder, exist_ok=True)
    a = np.ascontiguousarray(data)
    if ext == ".npy":
        np.save(fname, a)
        return fname
    if ext in (".tif", ".tiff"):
        return write_tiff(a, fname)
    if ext == ".raw":
        a.tofile(fname)
        return fname
    raise ValueError("write_volume: unknown extension %r (.npy, .tif, .tiff, .raw)" % ext)


def read_volume(fname: str, shape=None, dtype=None) -> np.ndarray:
    """Read a volume written by write_volume (or by dxchange/tifffile for
    TIFF); ``.raw`` needs the shape and dtype."""
    ext = os.path.splitext(fname)[1].lower()
    if ext == ".npy":
        return np.load(fname)
    if ext in (".tif", ".tiff"):
        return read_tiff(fname)
    if ext == ".raw":
        if shape is None or dtype is None:
            raise ValueError("read_volume: .raw needs shape and dtype")
        a = np.fromfile(fname, dtype=dtype)
        if a.size != int(np.prod(shape)):
            raise ValueError("read_volume: %s holds %d values, not %s" % (fname, a.size, tuple(shape)))
        return a.reshape(shape)
    raise ValueError("read_volume: unknown extension %r (.npy, .tif, .tiff, .raw)" % ext)
