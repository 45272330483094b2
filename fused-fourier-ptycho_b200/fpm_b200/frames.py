"""Measured frames on disk: the files the reference reads and writes.

The reference's loader reads ``raw_images/<colour>/<k>.tif``, one uint16 TIFF per LED,
k = ``sprintf("%03d", k(i,j))`` with k(i,j) = j + (i-1)·grid over the spiral LED order
(codes_v2/main_run_FPM.m:26-41, codes_v2/func_ware/init_environment_rgb.m:76); its data
generator writes ``imwrite(uint16((2^16-1) * x), "img<n>.tif")`` after a global min / max
normalisation (benchmark/gen_img_batch.m:76-81).  Reading is libfpm's
``read_tiff_stack``; this module names and writes frames (host code, baseline TIFF).
"""
from __future__ import annotations

import struct
from pathlib import Path

import numpy as np

__all__ = ["frame_numbers", "frame_paths", "to_uint16_frames", "write_tiff", "write_frames"]


def frame_numbers(grid_pos, grid: int):
    """File numbers k = j + (i-1)·grid of LEDs given as 1-based (i, j) rows, in LED order
    (``Engine.led_indices`` returns them as its second output)."""
    ij = np.asarray(grid_pos, np.int64).reshape(-1, 2)
    return ij[:, 1] + (ij[:, 0] - 1) * int(grid)


def frame_paths(directory, grid_pos, grid: int, ext: str = ".tif"):
    """``<directory>/<%03d k>.tif`` for each LED in LED order."""
    d = Path(directory)
    return [d / f"{int(k):03d}{ext}" for k in frame_numbers(grid_pos, grid)]


def to_uint16_frames(images):
    """``uint16((2^16-1) * (x - min) / max(x - min))`` over the whole stack, in double;
    MATLAB's uint16() rounds halves away from zero and saturates."""
    x = np.asarray(images, np.float64)
    x = x - x.min()
    mx = x.max()
    if mx > 0:
        x = x / mx
    return np.clip(np.floor(65535.0 * x + 0.5), 0, 65535).astype(np.uint16)


def write_tiff(path, image, rows_per_strip: int | None = None):
    """Baseline little-endian uncompressed TIFF of a (rows, cols) uint8 / uint16 image
    (what MATLAB's imwrite produces for these types)."""
    a = np.ascontiguousarray(image)
    if a.ndim != 2 or a.dtype not in (np.uint8, np.uint16):
        raise ValueError("write_tiff takes a 2-D uint8 or uint16 image")
    rows, cols = a.shape
    bits = a.dtype.itemsize * 8
    row_bytes = cols * a.dtype.itemsize
    rps = rows_per_strip or max(1, min(rows, (1 << 16) // max(1, row_bytes)))
    data = a.astype("<u%d" % a.dtype.itemsize, copy=False).tobytes()
    strips = [(i * row_bytes, min(rows, i + rps) * row_bytes) for i in range(0, rows, rps)]
    n_strips = len(strips)
    n_tags = 9
    ifd = 8
    extra = ifd + 2 + 12 * n_tags + 4                       # out-of-line arrays follow the IFD
    off_arr = extra if n_strips > 1 else None
    cnt_arr = extra + 4 * n_strips if n_strips > 1 else None
    pix = extra + (8 * n_strips if n_strips > 1 else 0)
    offsets = [pix + s for s, _ in strips]
    counts = [e - s for s, e in strips]

    def tag(t, typ, count, value):
        return struct.pack("<HHII", t, typ, count, value)

    tags = [tag(256, 4, 1, cols), tag(257, 4, 1, rows), tag(258, 3, 1, bits), tag(259, 3, 1, 1),
            tag(262, 3, 1, 1),
            tag(273, 4, n_strips, off_arr if n_strips > 1 else offsets[0]),
            tag(277, 3, 1, 1), tag(278, 4, 1, rps),
            tag(279, 4, n_strips, cnt_arr if n_strips > 1 else counts[0])]
    head = b"II*\x00" + struct.pack("<I", ifd) + struct.pack("<H", n_tags) + b"".join(tags) + b"\0" * 4
    if n_strips > 1:
        head += struct.pack("<%dI" % n_strips, *offsets) + struct.pack("<%dI" % n_strips, *counts)
    assert len(head) == pix
    Path(path).write_bytes(head + data)


def write_frames(directory, stack, names=None):
    """Write a MATLAB-order (h, h, L) uint16 stack as L TIFF files; names default to
    ``img<n>.tif`` (n = 1..L, the generator's names).  Returns the paths."""
    d = Path(directory)
    d.mkdir(parents=True, exist_ok=True)
    s = np.asarray(stack)
    L = s.shape[2]
    paths = [d / (names[i] if names else f"img{i + 1}.tif") for i in range(L)]
    for i, p in enumerate(paths):
        write_tiff(p, s[:, :, i])
    return paths
