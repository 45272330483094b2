"""CPU tests of the C ABI: the library loads, exports every function include/fpm.h
declares, its structs match the ctypes binding byte for byte, and it fails
loudly (never falls back to the CPU) when no CUDA device is present."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import pytest

from conftest import ROOT, has_gpu
import fpm_b200
from fpm_b200 import api

HEADER = ROOT / "include" / "fpm.h"


def header_functions():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[\w ]+?\*?\s*\b(fpm_\w+)\s*\(", text, re.M)))


def test_header_declares_the_bound_entry_points():
    assert set(header_functions()) == set(api.EXPORTED)


def test_library_exports_every_declared_symbol():
    lib = fpm_b200.load_library()
    for name in header_functions():
        assert hasattr(lib, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", str(api._LIB_PATH)], capture_output=True,
                         text=True).stdout
    for name in header_functions():
        assert re.search(rf"\bT {name}\b", out), name


def test_abi_version_and_status_strings():
    lib = fpm_b200.load_library()
    assert lib.fpm_abi_version() == 2
    assert lib.fpm_status_string(0) == b"ok"
    assert lib.fpm_status_string(3) == b"out of device memory"
    assert lib.fpm_status_string(99) == b"unknown status"
    assert lib.fpm_last_error(None) == b""


PROBE = r"""
#include <stdio.h>
#include <stddef.h>
#include "fpm.h"
#define F(T, f) printf(#T "." #f " %zu\n", offsetof(T, f));
int main(void) {
  printf("fpm_problem %zu\nfpm_result %zu\nfpm_device_opts %zu\nfpm_led_geometry %zu\n"
         "fpm_optimizer %zu\n",
         sizeof(fpm_problem), sizeof(fpm_result), sizeof(fpm_device_opts),
         sizeof(fpm_led_geometry), sizeof(fpm_optimizer));
  F(fpm_problem, h) F(fpm_problem, n_leds) F(fpm_problem, pratio) F(fpm_problem, batch)
  F(fpm_problem, epochs) F(fpm_problem, lr) F(fpm_problem, beta) F(fpm_problem, eps)
  F(fpm_problem, pupil_margin) F(fpm_problem, lr_halve_after) F(fpm_problem, lr_decay)
  F(fpm_problem, loss_kind) F(fpm_problem, memory) F(fpm_problem, stack_type)
  F(fpm_problem, stack) F(fpm_problem, led_idx) F(fpm_problem, pupil_init)
  F(fpm_problem, pupil_amp) F(fpm_problem, object_init) F(fpm_problem, pie_weights)
  F(fpm_result, object) F(fpm_result, spectrum) F(fpm_result, pupil) F(fpm_result, loss)
  F(fpm_device_opts, device) F(fpm_device_opts, mem_limit_bytes) F(fpm_device_opts, stream)
  F(fpm_led_geometry, grid) F(fpm_led_geometry, h) F(fpm_led_geometry, pratio)
  F(fpm_led_geometry, wavelength_um) F(fpm_led_geometry, led_pitch_um)
  F(fpm_led_geometry, led_height_um) F(fpm_led_geometry, camera_pixel_um)
  F(fpm_led_geometry, magnification) F(fpm_led_geometry, sample_dx_um)
  F(fpm_led_geometry, sample_dy_um)
  F(fpm_optimizer, kind) F(fpm_optimizer, centered) F(fpm_optimizer, lr) F(fpm_optimizer, beta1)
  F(fpm_optimizer, beta2) F(fpm_optimizer, momentum) F(fpm_optimizer, iter) F(fpm_optimizer, mom1)
  F(fpm_optimizer, mom2) F(fpm_optimizer, buffer) F(fpm_optimizer, clamp_amp)
  F(fpm_optimizer, clamp_margin)
  return 0;
}
"""


def test_struct_layout_matches_c(tmp_path):
    src = tmp_path / "probe.c"
    src.write_text(PROBE)
    exe = tmp_path / "probe"
    subprocess.run(["gcc", "-std=c99", "-I", str(ROOT / "include"), str(src), "-o", str(exe)],
                   check=True)
    lines = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    got = dict(l.rsplit(" ", 1) for l in lines if l)
    assert int(got["fpm_problem"]) == C.sizeof(api.Problem)
    assert int(got["fpm_result"]) == C.sizeof(api.Result)
    assert int(got["fpm_device_opts"]) == C.sizeof(api.DeviceOpts)
    assert int(got["fpm_led_geometry"]) == C.sizeof(api.LedGeometry)
    assert int(got["fpm_optimizer"]) == C.sizeof(api.Optimizer)
    for cname, cls in (("fpm_problem", api.Problem), ("fpm_result", api.Result),
                       ("fpm_device_opts", api.DeviceOpts), ("fpm_led_geometry", api.LedGeometry),
                       ("fpm_optimizer", api.Optimizer)):
        for fname, _ in cls._fields_:
            key = f"{cname}.{fname}"
            if key in got:
                assert int(got[key]) == getattr(cls, fname).offset, key


@pytest.mark.skipif(has_gpu(), reason="checks the behaviour without a CUDA device")
def test_no_device_fails_loudly():
    with pytest.raises(fpm_b200.FpmError) as e:
        fpm_b200.Engine(0)
    assert e.value.status == 6   # FPM_ERR_NO_DEVICE, no CPU fallback


def test_missing_library_raises(tmp_path):
    with pytest.raises(ImportError):
        api.load_library(tmp_path / "absent.so")
