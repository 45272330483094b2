"""fpm_cli, the file-driven front end for hosts without MATLAB.

CPU: usage errors and unreadable inputs are refused before any device work, and
without a device the engine's own status comes back as the exit code.  GPU: a
solve from files equals the same solve through the library call bit for bit
(one engine, one code path; the CLI only moves bytes).
"""
import subprocess

import numpy as np
import pytest

from conftest import ROOT, has_gpu, dataset, led_matlab, to_matlab_stack

CLI = ROOT / "fused-fourier-ptycho_b200" / "fpm_b200" / "_lib" / "fpm_cli"


def run(*args):
    return subprocess.run([str(CLI), *map(str, args)], capture_output=True, text=True)


def _inputs(tmp_path, ds, L):
    """MATLAB-order raw files of the first L LEDs of a data set."""
    f = {
        "stack": tmp_path / "Y.u16", "led": tmp_path / "led.i32", "pupil": tmp_path / "P0c.c64",
        "pupil-amp": tmp_path / "P0.f32",
    }
    f["stack"].write_bytes(np.transpose(ds.raw[:L], (0, 2, 1)).astype("<u2").tobytes())
    f["led"].write_bytes(np.asarray(ds.led_idx[:L], "<i4").tobytes())          # (kl, kt) pairs
    f["pupil"].write_bytes(np.asarray(ds.P0c, np.complex64).T.tobytes())
    f["pupil-amp"].write_bytes(np.asarray(ds.pupil0, np.float32).T.tobytes())
    return f


def test_cli_usage():
    assert CLI.exists(), "fpm_cli is built with libfpm.so"
    r = run()
    assert r.returncode == 2 and "usage" in r.stderr
    r = run("solve", "--h", "64")
    assert r.returncode == 2 and "missing --leds" in r.stderr


def test_cli_refuses_short_files(tmp_path):
    ds = dataset(64, 4, 5, seed=3, aberration=True)
    f = _inputs(tmp_path, ds, 25)
    f["stack"].write_bytes(f["stack"].read_bytes()[:-2])
    r = run("solve", "--h", 64, "--leds", 25, "--pratio", 4, "--batch", 6, "--epochs", 1,
            *sum(([f"--{k}", v] for k, v in f.items()), []))
    assert r.returncode == 2 and "fewer than" in r.stderr


@pytest.mark.skipif(has_gpu(), reason="checks the no-device path")
def test_cli_without_device_reports_engine_status(tmp_path):
    ds = dataset(64, 4, 5, seed=3, aberration=True)
    f = _inputs(tmp_path, ds, 25)
    r = run("solve", "--h", 64, "--leds", 25, "--pratio", 4, "--batch", 6, "--epochs", 1,
            *sum(([f"--{k}", v] for k, v in f.items()), []))
    assert r.returncode == 3 + 6 and "no CUDA device" in r.stderr     # FPM_ERR_NO_DEVICE


@pytest.mark.gpu
def test_cli_solve_equals_library_solve(tmp_path, engine):
    ds = dataset(64, 4, 5, seed=3, aberration=True)
    L, E, B = 25, 2, 6
    f = _inputs(tmp_path, ds, L)
    out = {k: tmp_path / n for k, n in (("out-object", "O.c64"), ("out-pupil", "P.c64"),
                                         ("out-loss", "loss.f64"), ("out-spectrum", "S.c64"))}
    r = run("solve", "--h", 64, "--leds", L, "--pratio", 4, "--batch", B, "--epochs", E,
            "--lr", 2e-3, "--beta", 0.999, "--eps", 1e-4,
            *sum(([f"--{k}", v] for k, v in {**f, **out}.items()), []))
    assert r.returncode == 0, r.stderr
    H = 64 * 4
    O = np.fromfile(out["out-object"], np.complex64).reshape(H, H).T
    P = np.fromfile(out["out-pupil"], np.complex64).reshape(64, 64).T
    S = np.fromfile(out["out-spectrum"], np.complex64).reshape(H, H).T
    loss = np.fromfile(out["out-loss"], np.float64)
    ref = engine.solve(None, ds.P0c, to_matlab_stack(ds.raw[:L]), led_matlab(ds.led_idx[:L]),
                       ds.pupil0, 4, E, B, lr=2e-3, beta=0.999, eps=1e-4)   # bicubic start
    np.testing.assert_array_equal(O, ref["object"])
    np.testing.assert_array_equal(P, ref["pupil"])
    np.testing.assert_array_equal(S, ref["spectrum"])
    np.testing.assert_array_equal(loss, ref["loss"])


@pytest.mark.gpu
def test_cli_solve_from_tiff_frames_equals_library_solve(tmp_path, engine):
    """Frames read from TIFF files (one per LED, region at an offset) give the same
    reconstruction as the library solve of the counts they hold."""
    from PIL import Image
    ds = dataset(64, 4, 5, seed=3, aberration=True)
    L, E, B = 25, 1, 6
    f = _inputs(tmp_path, ds, L)
    del f["stack"]
    names = []
    for l in range(L):
        frame = np.zeros((70, 80), np.uint16)
        frame[5:69, 11:75] = ds.raw[l]                   # [row, col] counts of LED l
        p = tmp_path / f"{l + 1:03d}.tif"
        Image.fromarray(frame).save(str(p), format="TIFF")
        names.append(str(p))
    (tmp_path / "frames.txt").write_text("\n".join(names) + "\n")
    out = tmp_path / "O.c64"
    r = run("solve", "--h", 64, "--leds", L, "--pratio", 4, "--batch", B, "--epochs", E,
            "--tiff-list", tmp_path / "frames.txt", "--row0", 5, "--col0", 11,
            "--out-object", out, *sum(([f"--{k}", v] for k, v in f.items()), []))
    assert r.returncode == 0, r.stderr
    O = np.fromfile(out, np.complex64).reshape(256, 256).T
    ref = engine.solve(None, ds.P0c, to_matlab_stack(ds.raw[:L]), led_matlab(ds.led_idx[:L]),
                       ds.pupil0, 4, E, B)
    np.testing.assert_array_equal(O, ref["object"])


def test_cli_leds_usage_and_no_device(tmp_path):
    r = run("leds", "--grid", 5, "--h", 64)
    assert r.returncode == 2 and "missing --pratio" in r.stderr
    args = ["leds", "--grid", 5, "--h", 64, "--pratio", 4, "--wavelength", 0.532, "--pitch", 4000,
            "--height", 90000, "--pixel", 6.5, "--mag", 4, "--out-led", tmp_path / "l.i32"]
    r = run(*args[:2], 300, *args[3:])
    assert r.returncode == 2 and "--grid" in r.stderr
    if not has_gpu():
        r = run(*args)
        assert r.returncode == 3 + 6                      # FPM_ERR_NO_DEVICE


@pytest.mark.gpu
def test_cli_leds_equals_library_geometry(tmp_path, engine):
    from fpm_b200 import frames
    geo = dict(grid=7, h=256, pratio=4, wavelength_um=0.532, led_pitch_um=4000.0,
               led_height_um=90000.0, camera_pixel_um=6.5, magnification=4.0)
    r = run("leds", "--grid", 7, "--h", 256, "--pratio", 4, "--wavelength", 0.532, "--pitch", 4000,
            "--height", 90000, "--pixel", 6.5, "--mag", 4, "--out-led", tmp_path / "l.i32",
            "--out-frames", tmp_path / "f.txt", "--frames-dir", "raw_images/green")
    assert r.returncode == 0, r.stderr
    led, order = engine.led_indices(geo["grid"], geo["h"], geo["pratio"], geo["wavelength_um"],
                                    geo["led_pitch_um"], geo["led_height_um"],
                                    geo["camera_pixel_um"], geo["magnification"])
    np.testing.assert_array_equal(np.fromfile(tmp_path / "l.i32", "<i4").reshape(-1, 2), led)
    names = (tmp_path / "f.txt").read_text().split()
    assert names == [str(p) for p in frames.frame_paths("raw_images/green", order, 7)]


@pytest.mark.gpu
def test_cli_loss_and_weights_options_equal_library(tmp_path, engine):
    ds = dataset(64, 4, 5, seed=3, aberration=True)
    L = 12
    f = _inputs(tmp_path, ds, L)
    out = tmp_path / "O.c64"
    r = run("solve", "--h", 64, "--leds", L, "--pratio", 4, "--batch", 6, "--epochs", 1,
            "--loss", "isotropic", "--pie", "tPIE", "--out-object", out,
            *sum(([f"--{k}", v] for k, v in f.items()), []))
    assert r.returncode == 0, r.stderr
    O = np.fromfile(out, np.complex64).reshape(256, 256).T
    ref = engine.solve(None, ds.P0c, to_matlab_stack(ds.raw[:L]), led_matlab(ds.led_idx[:L]),
                       ds.pupil0, 4, 1, 6, loss="isotropic", pie="tPIE")
    np.testing.assert_array_equal(O, ref["object"])
    bad = run("solve", "--h", 64, "--leds", L, "--pratio", 4, "--batch", 6, "--epochs", 1,
              "--pie", "rPIE", *sum(([f"--{k}", v] for k, v in f.items()), []))
    assert bad.returncode == 2 and "--pie" in bad.stderr
