"""Time the reference's own GPU build on the bench workload.

TEST INFRASTRUCTURE.  Loads oracle/_ref/libcufpm_ref.so (the reference's v3
kernels plus cuFFT, driven by the replica of cuFPM_v3/cuFPM_pure_v3.cu:75-207 in
oracle/ref_harness.cu) and times its epoch loop with CUDA events (``ms[0]`` of
``ref_solve``: allocation, cuFFT planning and host copies excluded) on the
workload bench.py times: 19 x 19 LEDs of 2048^2 -> 16384^2, LED batch 26.  The
pixel values do not change the timing of the reference's kernels, so the stack is
the seeded random uint16 stack of ``bench.py --quick-data``, normalised to
amplitudes on the GPU as the reference's driver does before its call.

    python oracle/time_ref.py [--epochs 3] [--h 2048 --pratio 8 --grid 19 --batch 26]

Prints one JSON line: seconds per epoch and per 10-epoch job.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
sys.path.insert(0, str(ROOT / "fused-fourier-ptycho_b200"))
sys.path.insert(0, str(ROOT))


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--epochs", type=int, default=3)
    ap.add_argument("--h", type=int, default=2048)
    ap.add_argument("--pratio", type=int, default=8)
    ap.add_argument("--grid", type=int, default=19)
    ap.add_argument("--batch", type=int, default=26)
    args = ap.parse_args()

    import torch
    import bench

    cfg = bench.Cfg(h=args.h, pratio=args.pratio, grid=args.grid, batch=args.batch)
    dev = torch.device("cuda", 0)
    wl = bench.make_quick_workload_gpu(cfg, dev)
    st = wl["stack"].to(torch.int32)
    mn, mx = float(st.min()), float(st.max())
    # memory [l][c][r]: column-major pages, as the reference's Y
    Y = ((st.float() - mn) / (mx - mn)).sqrt().cpu().numpy()
    del st
    P0 = wl["P0"].cpu().numpy()                       # [c][r] memory
    P0c = wl["P0c"].cpu().numpy()
    led = np.ascontiguousarray(wl["led_np"], np.int32)
    del wl
    torch.cuda.empty_cache()
    H, h = cfg.H, cfg.h
    O0 = np.ones((H, H), np.complex64)
    O = np.empty((H, H), np.complex64)
    P = np.empty((h, h), np.complex64)

    lib = C.CDLL(str(HERE / "_ref" / "libcufpm_ref.so"))
    vp = C.c_void_p
    lib.ref_solve.argtypes = [C.c_int] * 6 + [C.c_float] * 3 + [vp] * 8
    ms = np.zeros(3, np.float32)
    rc = lib.ref_solve(h, H, cfg.L, cfg.pratio, args.epochs, cfg.batch, cfg.lr, cfg.beta, cfg.eps,
                       O0.ctypes.data, P0c.ctypes.data, Y.ctypes.data, led.ctypes.data,
                       P0.ctypes.data, O.ctypes.data, P.ctypes.data, ms.ctypes.data)
    if rc != 0:
        raise SystemExit(f"ref_solve failed: {rc}")
    per_epoch = float(ms[0]) / 1e3 / args.epochs
    print(json.dumps({
        "impl": "reference GPU build (cuFPM_v3 kernels + cuFFT)",
        "workload": cfg.describe()["workload"], "epochs_timed": args.epochs,
        "s_per_epoch": round(per_epoch, 5), "s_per_10_epoch_job": round(10 * per_epoch, 4),
        "s_with_alloc_and_plans": round(float(ms[1]) / 1e3, 4),
        "device": torch.cuda.get_device_name(0),
        "timing": "CUDA events around the epoch loop (ms[0] of ref_solve)"}))


if __name__ == "__main__":
    main()
