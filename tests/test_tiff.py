"""Ingest of the measured frames (codes_v2/main_run_FPM.m:26-45): the TIFF reader
of libfpm against Pillow's decoder (the oracle's read_frame) and against the
arrays the files were written from, and the float-stack normalisation on the
device against the oracle.

The reader is host code: everything but the normalisation runs without a GPU.
Files come from two writers: Pillow (the layouts MATLAB's imwrite and camera
software produce: one or a few strips, little-endian) and the small writer
below (big-endian, 16-bit multi-sample pixels, strips that do not divide the
image), so that every branch of the reader meets a file it did not write.
"""
import struct

import numpy as np
import pytest

from conftest import has_gpu

from oracle import fpm_oracle as orc


def write_tiff(path, a, rows_per_strip=None, big=False, bits=None):
    """Baseline uncompressed TIFF of a (rows, cols) or (rows, cols, samples) array."""
    a = np.asarray(a)
    if a.ndim == 2:
        a = a[:, :, None]
    rows, cols, spp = a.shape
    bits = bits or a.dtype.itemsize * 8
    e = ">" if big else "<"
    data = a.astype(e + ("u1" if bits == 8 else "u2")).tobytes()
    row_bytes = cols * spp * bits // 8
    rps = rows_per_strip or rows
    strips = [data[i * row_bytes:min(rows, i + rps) * row_bytes] for i in range(0, rows, rps)]
    # header, then pixel strips, then out-of-line tag values, then the directory
    body = bytearray(b"MM\x00\x2a" if big else b"II\x2a\x00")
    body += b"\x00\x00\x00\x00"
    offsets = []
    for s in strips:
        offsets.append(len(body))
        body += s
        if len(body) % 2:
            body += b"\x00"

    def out_of_line(fmt, vals):
        off = len(body)
        body.extend(struct.pack(e + fmt * len(vals), *vals))
        return off

    entries = []

    def tag(t, typ, vals):
        fmt = {3: "H", 4: "I"}[typ]
        size = struct.calcsize(fmt) * len(vals)
        if size <= 4:
            raw = struct.pack(e + fmt * len(vals), *vals).ljust(4, b"\x00")
        else:
            raw = struct.pack(e + "I", out_of_line(fmt, vals))
        entries.append(struct.pack(e + "HHI", t, typ, len(vals)) + raw)

    tag(256, 4, [cols])
    tag(257, 4, [rows])
    tag(258, 3, [bits] * spp)
    tag(259, 3, [1])
    tag(262, 3, [2 if spp >= 3 else 1])
    tag(273, 4, offsets)
    tag(277, 3, [spp])
    tag(278, 4, [rps])
    tag(279, 4, [len(s) for s in strips])
    tag(284, 3, [1])
    if len(body) % 2:
        body += b"\x00"
    ifd = len(body)
    body += struct.pack(e + "H", len(entries)) + b"".join(entries) + b"\x00\x00\x00\x00"
    body[4:8] = struct.pack(e + "I", ifd)
    path.write_bytes(bytes(body))


def pil_write(path, a, **kw):
    from PIL import Image
    Image.fromarray(a).save(str(path), format="TIFF", **kw)


@pytest.fixture(scope="module")
def lib():
    from fpm_b200 import api
    return api


def rng_frames(seed, n, rows, cols, spp=None, dtype=np.uint16):
    g = np.random.default_rng(seed)
    hi = np.iinfo(dtype).max + 1
    shape = (n, rows, cols) if spp is None else (n, rows, cols, spp)
    return g.integers(0, hi, size=shape, dtype=np.int64).astype(dtype)


def test_u16_frames_from_pillow_match_region(lib, tmp_path):
    frames = rng_frames(0, 5, 40, 56)
    paths = []
    for i, f in enumerate(frames):
        p = tmp_path / f"{i + 1:03d}.tif"
        pil_write(p, f)
        paths.append(p)
    Y = lib.read_tiff_stack(paths, 32, row0=3, col0=17)
    assert Y.dtype == np.uint16 and Y.shape == (32, 32, 5) and Y.flags.f_contiguous
    for i, f in enumerate(frames):
        np.testing.assert_array_equal(Y[:, :, i], f[3:35, 17:49])
        np.testing.assert_array_equal(Y[:, :, i].astype(np.float32),
                                      orc.read_frame(paths[i], 3, 17, 32))


@pytest.mark.parametrize("big", [False, True])
@pytest.mark.parametrize("rps", [None, 1, 7, 64])
def test_strips_and_byte_order(lib, tmp_path, big, rps):
    frames = rng_frames(1, 3, 50, 45)
    paths = []
    for i, f in enumerate(frames):
        p = tmp_path / f"f{i}.tif"
        write_tiff(p, f, rows_per_strip=rps, big=big)
        paths.append(p)
    Y = lib.read_tiff_stack(paths, 24, row0=26, col0=21)
    for i, f in enumerate(frames):
        np.testing.assert_array_equal(Y[:, :, i], f[26:50, 21:45])
        np.testing.assert_array_equal(Y[:, :, i].astype(np.float32),
                                      orc.read_frame(paths[i], 26, 21, 24))


@pytest.mark.parametrize("spp,dtype,writer", [(3, np.uint8, "pil"), (4, np.uint8, "pil"),
                                             (3, np.uint16, "own"), (2, np.uint16, "own")])
def test_multisample_frames_are_averaged(lib, tmp_path, spp, dtype, writer):
    frames = rng_frames(2, 4, 33, 37, spp=spp, dtype=dtype)
    paths = []
    for i, f in enumerate(frames):
        p = tmp_path / f"c{i}.tif"
        (pil_write if writer == "pil" else write_tiff)(p, f)
        paths.append(p)
    Y = lib.read_tiff_stack(paths, 16, row0=9, col0=4, dtype="f32")
    assert Y.dtype == np.float32
    for i, f in enumerate(frames):
        if dtype == np.uint8:
            # Pillow decodes 8-bit multi-sample pixels only (16-bit RGB it reduces to 8 bits)
            np.testing.assert_array_equal(Y[:, :, i], orc.read_frame(paths[i], 9, 4, 16))
        # the float mean of the written samples, one rounding
        exact = f[9:25, 4:20].astype(np.float64).sum(-1) / spp
        np.testing.assert_array_equal(Y[:, :, i], exact.astype(np.float32))


def test_u8_grey_to_u16_and_f32(lib, tmp_path):
    f = rng_frames(3, 1, 20, 20, dtype=np.uint8)[0]
    p = tmp_path / "g.tif"
    pil_write(p, f)
    np.testing.assert_array_equal(lib.read_tiff_stack([p], 20)[:, :, 0], f)
    np.testing.assert_array_equal(lib.read_tiff_stack([p], 20, dtype="f32")[:, :, 0], f)


def test_thread_counts_agree(lib, tmp_path):
    frames = rng_frames(4, 9, 48, 48)
    paths = []
    for i, f in enumerate(frames):
        p = tmp_path / f"{i}.tif"
        write_tiff(p, f, rows_per_strip=5)
        paths.append(p)
    one = lib.read_tiff_stack(paths, 48, threads=1)
    many = lib.read_tiff_stack(paths, 48, threads=4)
    auto = lib.read_tiff_stack(paths, 48)
    np.testing.assert_array_equal(one, many)
    np.testing.assert_array_equal(one, auto)
    np.testing.assert_array_equal(one, np.transpose(frames, (1, 2, 0)))


def _err(lib, *a, **kw):
    with pytest.raises(lib.FpmError) as e:
        lib.read_tiff_stack(*a, **kw)
    assert e.value.status == 1
    return e.value.detail


def test_refusals_name_the_file(lib, tmp_path):
    good = tmp_path / "ok.tif"
    write_tiff(good, rng_frames(5, 1, 16, 16)[0])
    assert "outside" in _err(lib, [good], 16, row0=1)
    assert "outside" in _err(lib, [good], 17)
    missing = tmp_path / "missing.tif"
    assert "cannot open" in _err(lib, [good, missing], 8) and "missing.tif" in _err(lib, [good, missing], 8)
    junk = tmp_path / "junk.tif"
    junk.write_bytes(b"not an image at all")
    assert "not a TIFF" in _err(lib, [junk], 8)
    lzw = tmp_path / "lzw.tif"
    pil_write(lzw, rng_frames(6, 1, 16, 16)[0], compression="tiff_lzw")
    assert "compressed" in _err(lib, [lzw], 8)
    rgb = tmp_path / "rgb.tif"
    pil_write(rgb, rng_frames(7, 1, 16, 16, spp=3, dtype=np.uint8)[0])
    assert "float stack" in _err(lib, [rgb], 8)
    short = tmp_path / "short.tif"
    write_tiff(short, rng_frames(8, 1, 16, 16)[0])
    # a strip byte count smaller than the strip's rows
    a = bytearray(short.read_bytes())
    ifd = struct.unpack("<I", a[4:8])[0]
    n = struct.unpack("<H", a[ifd:ifd + 2])[0]
    for k in range(n):
        e = ifd + 2 + 12 * k
        if struct.unpack("<H", a[e:e + 2])[0] == 279:
            a[e + 8:e + 12] = struct.pack("<I", 100)
    short.write_bytes(bytes(a))
    assert "shorter" in _err(lib, [short], 16)
    # the first failing file in LED order is the one reported
    detail = _err(lib, [good, junk, missing], 8)
    assert "junk.tif" in detail


def test_bad_arguments(lib, tmp_path):
    good = tmp_path / "ok.tif"
    write_tiff(good, rng_frames(9, 1, 16, 16)[0])
    assert "row0" in _err(lib, [good], 8, row0=-1)
    with pytest.raises(KeyError):
        lib.read_tiff_stack([good], 8, dtype="f64")


def test_cli_ingest_writes_the_stack(lib, tmp_path):
    import subprocess
    from conftest import ROOT
    cli = ROOT / "fused-fourier-ptycho_b200" / "fpm_b200" / "_lib" / "fpm_cli"
    frames = rng_frames(10, 4, 30, 30)
    names = []
    for i, f in enumerate(frames):
        p = tmp_path / f"{i + 1:03d}.tif"
        write_tiff(p, f, rows_per_strip=8)
        names.append(str(p))
    lst = tmp_path / "frames.txt"
    lst.write_text("\n".join(names) + "\n\n")
    out = tmp_path / "Y.u16"
    r = subprocess.run([str(cli), "ingest", "--tiff-list", lst, "--h", "16", "--row0", "2",
                        "--col0", "5", "--out", out], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    Y = np.fromfile(out, "<u2").reshape(4, 16, 16)       # page, col, row
    for i, f in enumerate(frames):
        np.testing.assert_array_equal(Y[i].T, f[2:18, 5:21])
    bad = subprocess.run([str(cli), "ingest", "--tiff-list", lst, "--h", "32", "--out", out],
                         capture_output=True, text=True)
    assert bad.returncode == 2 and "outside" in bad.stderr


def test_normalise_f32_oracle_properties():
    x = np.array([[3.5, np.nan], [1.0, 8.0]], np.float32)
    y = orc.normalise_stack_f32(x)
    assert y[0, 0] == np.sqrt(np.float32(2.5) / np.float32(7.0)) and np.isnan(y[0, 1])
    assert y[1, 0] == 0 and y[1, 1] == 1
    np.testing.assert_array_equal(orc.normalise_stack_f32(np.full((2, 2), 5, np.float32)), 0)
    u = rng_frames(11, 2, 8, 8)
    np.testing.assert_array_equal(orc.normalise_stack_f32(u.astype(np.float32)),
                                  orc.normalise_stack_u16(u))


@pytest.mark.gpu
@pytest.mark.skipif(not has_gpu(), reason="needs a CUDA device")
def test_normalise_f32_on_device_bit_exact(engine, tmp_path):
    import torch
    frames = rng_frames(12, 6, 64, 64, spp=3, dtype=np.uint8)
    paths = []
    for i, f in enumerate(frames):
        p = tmp_path / f"{i}.tif"
        pil_write(p, f)
        paths.append(p)
    X = engine.read_stack(paths, 64, dtype="f32")
    ref = orc.normalise_stack_f32(X)
    np.testing.assert_array_equal(engine.normalise_stack(X), ref)
    d = torch.from_numpy(np.ascontiguousarray(X)).cuda()
    np.testing.assert_array_equal(engine.normalise_stack(d).cpu().numpy(), ref)
    # NaN left out of the min / max; a constant stack gives zeros
    Xn = X.copy()
    Xn[1, 2, 3] = np.nan
    got = engine.normalise_stack(np.ascontiguousarray(Xn))
    np.testing.assert_array_equal(got, orc.normalise_stack_f32(Xn))
    np.testing.assert_array_equal(engine.normalise_stack(np.full((8, 8, 2), 7, np.float32)), 0)


@pytest.mark.parametrize("shape,dtype", [((70, 50), np.uint16), ((33, 1000), np.uint16),
                                         ((16, 16), np.uint8)])
def test_package_writer_round_trips(lib, tmp_path, shape, dtype):
    """fpm_b200.frames writes what both libfpm's reader and Pillow read back."""
    from fpm_b200 import frames
    a = rng_frames(13, 1, *shape, dtype=dtype)[0]
    p = tmp_path / "w.tif"
    frames.write_tiff(p, a)
    np.testing.assert_array_equal(orc.read_frame(p, 0, 0, min(shape)), a[:min(shape), :min(shape)])
    h = min(shape)
    np.testing.assert_array_equal(lib.read_tiff_stack([p], h)[:, :, 0], a[:h, :h])


def test_frame_names_and_uint16_conversion(tmp_path):
    from fpm_b200 import frames
    # spiral order of a 3 x 3 grid starts at the centre cell (2, 2): k = 2 + 1*3 = 5
    ij = np.array([[2, 2], [2, 3], [1, 3]])
    assert list(frames.frame_numbers(ij, 3)) == [5, 6, 3]
    assert [p.name for p in frames.frame_paths(tmp_path, ij, 3)] == ["005.tif", "006.tif", "003.tif"]
    x = np.array([[0.0, 0.5], [1.0, 2.0]])
    u = frames.to_uint16_frames(x)
    # (2^16-1) * [0, .25, .5, 1] rounded half away from zero: 16383.75 -> 16384, 32767.5 -> 32768
    np.testing.assert_array_equal(u, [[0, 16384], [32768, 65535]])
    paths = frames.write_frames(tmp_path / "d", np.stack([u, u[::-1]], axis=2))
    assert [p.name for p in paths] == ["img1.tif", "img2.tif"]
