"""Benchmark of the FPM reconstruction hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--batch B]

Workload: the full-scale configuration — 19 x 19 LEDs (361 images) of
2048 x 2048 uint16, up-sampling 8 -> 16384 x 16384 complex64 object, LED batch
26, RMSprop lr 5e-4 / beta 0.999 / eps 1e-4, anisotropic feature-domain loss.
Inputs are seeded synthetic data (object, Zernike-aberrated pupil, Poisson
noise at 3e4 peak counts) generated on the GPU before timing.

A step is one epoch (361 LEDs in 14 mini-batches).  ``value`` is the time of
the 10-epoch reconstruction (10 x the measured seconds per epoch) with every
input resident in HBM.  ``e2e`` is the same 10-epoch job through the C ABI with
pinned host buffers (stack in, object + pupil + loss out as the mex returns,
copies inside the timed region): the median of three jobs after one warm-up job,
split into host-to-device copies, device work and device-to-host copies.
``accuracy`` (one GPU) holds the per-epoch relative error of the engine's object
and pupil against an FP64 run of the same job (the torch FP64 checker of
``oracle/torch_ref.py``, outside every timed region) next to the FP32 twin's.
``cpu_baseline`` times the FP32 CPU restatement of the algorithm (numpy /
pocketfft, all host threads) on a bounded sample (two full-size mini-batches)
and projects the 10-epoch job.

``--impl reference`` times the reference's own GPU build on the same workload:
its v3 kernels (``cuFPM_v3/cuda/kernels.cuh``) and cuFFT, compiled from the
reference tree into ``oracle/_ref/libcufpm_ref.so`` and driven by the replica of
``cuFPM_v3/cuFPM_pure_v3.cu:75-207`` in ``oracle/ref_harness.cu`` (the reference
has no CPU implementation of this path; its MATLAB CPU path needs MATLAB).

Multi-GPU: a reconstruction does not shard (every mini-batch reads the object
the previous one updated), so N ranks run N independent replicas
(scaling "weak", no collective); value is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "fused-fourier-ptycho_b200"))
sys.path.insert(0, str(ROOT))

METRIC = ("s per 10-epoch reconstruction at 2048²×361→16384² (LED batch 26); the error "
          "against FP64 per epoch in accuracy; HBM GB/s fraction")
JOB_EPOCHS = 10


# ---------------------------------------------------------------------------
# workload
# ---------------------------------------------------------------------------
class Cfg:
    def __init__(self, h=2048, pratio=8, grid=19, batch=26, seed=0, lr=5e-4, beta=0.999, eps=1e-4):
        self.h, self.pratio, self.grid, self.batch, self.seed = h, pratio, grid, batch, seed
        self.lr, self.beta, self.eps = lr, beta, eps
        self.H = h * pratio
        self.L = grid * grid

    def describe(self):
        return {"workload": f"FPM reconstruction, {self.L} LEDs x {self.h}x{self.h} uint16 -> "
                            f"{self.H}x{self.H} complex64 object, pratio {self.pratio}, "
                            f"LED batch {self.batch}, {JOB_EPOCHS} epochs",
                "h": self.h, "H": self.H, "leds": self.L, "pratio": self.pratio,
                "led_batch": self.batch, "epochs_per_job": JOB_EPOCHS, "lr": self.lr,
                "beta": self.beta, "eps": self.eps, "loss": "anisotropic feature-domain",
                "stack": "uint16 resident (2 B/px), normalised in-kernel",
                "l2": "no flush needed: object 2 GiB, stack 3 GB, both larger than L2"}


def make_quick_workload_gpu(cfg: Cfg, dev):
    """Random uint16 stack with the real optics: for profiler runs, whose per-kernel timing does
    not depend on the pixel values and whose launch list must hold the engine's kernels only."""
    import torch
    from fpm_b200 import synth
    g = torch.Generator(device=dev)
    g.manual_seed(cfg.seed)
    optics = synth.Optics(led_grid=cfg.grid)
    circ = synth.pupil_circle(cfg.h, optics)
    led = synth.led_indices(cfg.h, cfg.pratio, optics)
    stack = torch.randint(0, 30000, (cfg.L, cfg.h, cfg.h), generator=g, device=dev,
                          dtype=torch.int32).to(torch.uint16)
    P0 = torch.from_numpy(np.ascontiguousarray(circ.T)).to(dev)
    torch.cuda.synchronize(dev)
    return {"stack": stack, "P0": P0, "P0c": P0.to(torch.complex64),
            "led": torch.from_numpy(np.ascontiguousarray(led)).to(dev), "led_np": led, "circ": circ}


def make_workload_gpu(cfg: Cfg, dev):
    """Seeded synthetic data set generated with torch on the GPU (same model as fpm_b200.synth)."""
    import torch
    from fpm_b200 import synth
    g = torch.Generator(device=dev)
    g.manual_seed(cfg.seed)
    H, h, p = cfg.H, cfg.h, cfg.pratio

    def smooth(x, sigma):
        f0 = torch.fft.fftfreq(H, device=dev)
        f1 = torch.fft.rfftfreq(H, device=dev)
        X = torch.fft.rfft2(x)
        X *= torch.exp(-2 * (math.pi * sigma) ** 2 * f0 * f0)[:, None]
        X *= torch.exp(-2 * (math.pi * sigma) ** 2 * f1 * f1)[None, :]
        return torch.fft.irfft2(X, s=(H, H))

    def rescale(x, lo, hi):
        mn, mx = x.min(), x.max()
        return (x - mn) / (mx - mn) * (hi - lo) + lo

    amp = rescale(smooth(torch.rand((H, H), generator=g, device=dev), 3.0), 0.5, 1.0)
    ph = rescale(smooth(torch.randn((H, H), generator=g, device=dev), 4.0), -math.pi / 2, math.pi / 2)
    obj = torch.polar(amp, ph)
    del amp, ph
    spec = torch.fft.fftshift(torch.fft.fft2(obj))
    del obj
    optics = synth.Optics(led_grid=cfg.grid)
    circ = synth.pupil_circle(h, optics)
    ptrue = torch.from_numpy((circ * np.exp(1j * synth.pupil_aberration(h, optics, cfg.seed)))
                             .astype(np.complex64)).to(dev)
    led = synth.led_indices(h, p, optics)
    I = torch.empty((cfg.L, h, h), dtype=torch.float32, device=dev)
    ar = torch.arange(h, device=dev)
    for l in range(cfg.L):
        kl, kt = int(led[l, 0]), int(led[l, 1])
        r = (kt - 1 + ar) % H
        c = (kl - 1 + ar) % H
        sub = spec.index_select(0, r).index_select(1, c) * ptrue
        x = torch.fft.ifft2(torch.fft.ifftshift(sub)) / (p * p)
        I[l] = x.real * x.real + x.imag * x.imag
    del spec
    lam = I * (3e4 / float(I.max()))
    del I
    counts = torch.poisson(lam, generator=g).clamp_(max=65535).to(torch.int32)
    del lam
    # column-major pages: memory [l][c][r]
    stack = counts.transpose(1, 2).contiguous().to(torch.uint16)
    del counts
    P0 = torch.from_numpy(np.ascontiguousarray(circ.T)).to(dev)                 # [c][r] memory
    P0c = P0.to(torch.complex64)
    led_t = torch.from_numpy(np.ascontiguousarray(led)).to(dev)               # (kl, kt) pairs
    torch.cuda.synchronize(dev)
    return {"stack": stack, "P0": P0, "P0c": P0c, "led": led_t, "led_np": led, "circ": circ}


# ---------------------------------------------------------------------------
# algorithmic bytes per launch of each stage
# ---------------------------------------------------------------------------
def pupil_support(circ):
    """Rows / columns [lo, hi) of the pupil's non-zero pixels (the engine prunes to them)."""
    rows = np.flatnonzero(np.any(circ != 0, axis=1))
    cols = np.flatnonzero(np.any(circ != 0, axis=0))
    return int(rows[0]), int(rows[-1]) + 1, int(cols[0]), int(cols[-1]) + 1


def _support_of(wl):
    """The support the engine prunes to (none with FPM_PUPIL_SUPPORT=0)."""
    if os.environ.get("FPM_PUPIL_SUPPORT", "1") == "0":
        return None
    return pupil_support(wl["circ"])


def batch_boxes(led, h, H, batch, sup=None):
    """Spectrum box (rspan, cspan) of every mini-batch, as the engine plans them: the union of
    the batch's crops restricted to the pupil support."""
    r_lo, r_hi, c_lo, c_hi = sup if sup is not None else (0, h, 0, h)
    out = []
    L = len(led)
    for cur in range(0, L, batch):
        sl = led[cur:cur + batch]
        kt = sl[:, 1] - 1
        kl = sl[:, 0] - 1
        rspan = min(int((kt + r_hi).max() - (kt + r_lo).min()), H)
        cspan = min(int((kl + c_hi).max() - (kl + c_lo).min()), H)
        out.append((len(sl), rspan, cspan))
    return out


def stage_bytes(cfg: Cfg, led, sup=None):
    """Average algorithmic bytes per launch of each stage over one epoch.

    fr, fc: fractions of crop rows / columns inside the pupil support; the passes read
    and write only what the pruned algorithm needs (zero columns of the first field
    are still written)."""
    H, h = cfg.H, cfg.h
    H2, h2 = H * H, h * h
    sup = sup if sup is not None else (0, h, 0, h)
    fr = (sup[1] - sup[0]) / h
    fc = (sup[3] - sup[2]) / h
    boxes = batch_boxes(led, h, H, cfg.batch, sup)
    nbatch = len(boxes)
    group = max(1, min(cfg.batch, (4 << 30) // (h2 * 16)))
    lr_launches = sum(math.ceil(nb / group) for nb, _, _ in boxes)
    tot = {k: 0.0 for k in ("lr_cols_inverse", "lr_rows_inverse", "lr_rows_forward",
                            "lr_rows_fused", "lr_cols_forward", "pupil_grad", "rows_inverse_stitch",
                            "cols_update", "rows_forward", "rmsprop_pupil", "transpose")}
    for bi, (nb, rspan, cspan) in enumerate(boxes):
        _, rn, cn = boxes[(bi + 1) % nbatch]
        px = h2 * nb
        tot["lr_cols_inverse"] += (8 * fr * fc + 8 * fc) * px   # support crop r8, support columns w8
        tot["lr_rows_inverse"] += 22 * px      # field r8 w8, residual w4, stack r2
        tot["lr_rows_forward"] += 20 * px      # residual r4, field r8 w8
        tot["lr_rows_fused"] += (12 + 8 * fc) * px   # field r8, amplitude rows r4, support columns w8
        tot["lr_cols_forward"] += 16 * fc * px        # support columns r8, gradient spectrum w8
        tot["pupil_grad"] += 16 * fr * fc * px + 8 * h2
        tot["rows_inverse_stitch"] += 8 * fr * fc * px + 8 * H * rspan
        tot["cols_update"] += 8 * H * rspan + 24 * H2 + 8 * H * rn
        tot["rows_forward"] += 8 * H * rn + 8 * rn * cn
        tot["rmsprop_pupil"] += 36 * h2
        # four transposes per batch: pupil, stitch rows, next-box rows, next-box spectrum
        tot["transpose"] += 16 * (h2 + H * rspan + H * rn + rn * cn)
    per = {}
    for k, v in tot.items():
        n = lr_launches if k.startswith("lr_") else (4 * nbatch if k == "transpose" else nbatch)
        per[k] = v / n
    nb0, r0, c0 = boxes[0]
    per["cols_forward"] = 8 * H2 + 8 * H * r0
    per["spectrum_fft2"] = 32 * H2
    # the any-size path's transforms (sides that are not powers of two): a 2-D transform
    # reads and writes its page in each of its four passes (two line passes, two transposes)
    per["any_size_object_fft2"] = 32 * H2
    per["any_size_lr_fft2"] = 32 * h2 * len(led) / max(nbatch, 1)
    per["loss_reduce"] = 8 * 1024
    per["stack_rows"] = 6 * h2 * len(led)    # once per solve: uint16 stack r2, amplitude rows w4
    return per


# ---------------------------------------------------------------------------
def clocks_start(dev_index: int):
    try:
        import torch
        uuid = "GPU-" + str(torch.cuda.get_device_properties(dev_index).uuid)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        f = open(f"/tmp/fpm_clocks_{os.getpid()}.csv", "w")
        proc = subprocess.Popen(["nvidia-smi", "-i", uuid, f"--query-gpu={q}", "--format=csv",
                                 "-lms", "200"], stdout=f, stderr=subprocess.DEVNULL)
        return proc, f
    except Exception:
        return None, None


def clocks_stop(handle):
    proc, f = handle
    if proc is None:
        return None
    time.sleep(0.25)
    proc.terminate()
    try:
        proc.wait(timeout=5)
    except Exception:
        proc.kill()
    f.close()
    try:
        lines = [l.strip() for l in open(f.name) if l.strip()]
        os.unlink(f.name)
    except Exception:
        return None
    rows = [[c.strip() for c in l.split(",")] for l in lines[1:] if not l.startswith("index")]
    sm = [float(r[1].split()[0]) for r in rows if len(r) >= 9 and r[1].split()[0].replace(".", "").isdigit()]
    smax = [float(r[2].split()[0]) for r in rows if len(r) >= 9 and r[2].split()[0].replace(".", "").isdigit()]
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    reasons = sorted({names[i] for r in rows if len(r) >= 9 for i in range(4)
                      if r[5 + i].lower().startswith("active")})
    if not sm:
        return None
    return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(smax) if smax else None,
            "reasons": reasons, "samples": len(sm)}


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ---------------------------------------------------------------------------
# CPU restatement (reference arm / cpu_baseline): bounded sample, projected job
# ---------------------------------------------------------------------------
def cpu_sample(cfg: Cfg, O0, P, Y_b, led_b, steps: int, warmup: int):
    """Times `steps` mini-batches of the FP32 oracle; returns projected job seconds and details."""
    from oracle import fpm_oracle as orc
    workers = orc.default_workers()
    H = cfg.H
    m1 = np.zeros((H, H), np.float32)
    O = O0.copy()
    t_large, t_led = [], []
    for it in range(warmup + steps):
        nled = 1 if it < warmup else len(led_b)        # warm-up: one LED, caches and pools only
        t0 = time.perf_counter()
        S = orc._fft2(O, workers).astype(np.complex64, copy=False)
        t1 = time.perf_counter()
        G, dP, _ = orc.batch_gradients(S, P, Y_b[:nled], led_b[:nled], cfg.pratio, np.float32,
                                       workers)
        del S
        t2 = time.perf_counter()
        g = (orc._ifft2(G, workers) * np.complex64(H * H)).astype(np.complex64, copy=False)
        del G
        O, m1 = orc.rmsprop_step(O, g, m1, cfg.lr, cfg.beta, cfg.eps, np.float32)
        del g
        t3 = time.perf_counter()
        if it >= warmup:
            t_large.append((t1 - t0) + (t3 - t2))
            t_led.append((t2 - t1) / nled)
    batches = JOB_EPOCHS * math.ceil(cfg.L / cfg.batch)
    leds = JOB_EPOCHS * cfg.L
    job = batches * float(np.mean(t_large)) + leds * float(np.mean(t_led))
    per_step = [tl + tg * len(led_b) for tl, tg in zip(t_large, t_led)]
    return job, workers, per_step


def cpu_inputs(cfg: Cfg, wl, nled: int):
    """Host copies of the CPU restatement's inputs, formed without the engine: the
    starting object imresize(Y_1, pratio) (codes_v2/main_run_FPM.m:48) and the amplitudes
    sqrt((I - min)/(max - min)) of the first `nled` frames with the whole stack's (min, max)
    (:43-45), both by the torch restatement of the oracle on the GPU (bit-identical
    single-precision amplitudes, FP64 bicubic), plus the pupil."""
    import torch
    from oracle import torch_ref as tr
    pages = tr.page_normaliser(wl["stack"])                 # memory [l][c][r]
    Y = pages(0, nled).transpose(1, 2).contiguous()         # (nled, h, h) [l, r, c]
    O0 = tr.imresize_bicubic(Y[0], cfg.pratio).to(torch.float32).to(torch.complex64)
    out = (O0.cpu().numpy(), wl["P0c"].T.contiguous().cpu().numpy(), Y.cpu().numpy(),
           wl["led_np"][:nled])
    del O0, Y
    torch.cuda.empty_cache()
    return out


# ---------------------------------------------------------------------------
def replica_max(value: float, world: int, device=None) -> float:
    """The slowest replica's figure: every rank runs its own reconstruction (no shard of
    one reconstruction, no collective on the data path), and a job of N replicas takes
    as long as its slowest rank.  All ranks must call it (one all-reduce)."""
    if world <= 1:
        return float(value)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_ours(args, cfg: Cfg):
    import torch
    import torch.distributed as dist
    import fpm_b200
    from fpm_b200 import api

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    stream = torch.cuda.Stream(device=dev)
    eng = fpm_b200.Engine(local, stream=stream.cuda_stream)
    wl = make_quick_workload_gpu(cfg, dev) if args.quick_data else make_workload_gpu(cfg, dev)
    H, h = cfg.H, cfg.h
    O = torch.empty((H, H), dtype=torch.complex64, device=dev)
    P = torch.empty((h, h), dtype=torch.complex64, device=dev)
    loss = torch.zeros(max(args.steps, args.warmup, JOB_EPOCHS), dtype=torch.float64, device=dev)

    def problem(epochs, memory, stack, led, P0c, P0):
        return api.Problem(h=h, n_leds=cfg.L, pratio=cfg.pratio, batch=cfg.batch, epochs=epochs,
                           lr=cfg.lr, beta=cfg.beta, eps=cfg.eps, pupil_margin=0.2,
                           lr_halve_after=12, lr_decay=0.5, loss_kind=0, memory=memory,
                           stack_type=api.STACK_U16, stack=stack, led_idx=led, pupil_init=P0c,
                           pupil_amp=P0, object_init=None)

    dev_args = (wl["stack"].data_ptr(), wl["led"].data_ptr(), wl["P0c"].data_ptr(),
                wl["P0"].data_ptr())
    res = api.Result(object=O.data_ptr(), spectrum=None, pupil=P.data_ptr(), loss=loss.data_ptr())

    # the autotuner's choice for this shape (one timed epoch per candidate), kept by the
    # context for every solve below
    t_tune = time.perf_counter()
    tune_report = ("skipped (--no-autotune): default launch choices" if args.no_autotune else
                   eng.autotune_raw(problem(1, api.MEM_DEVICE, *dev_args)))
    t_tune = time.perf_counter() - t_tune
    # warm-up epochs
    eng._check(eng.solve_raw(problem(args.warmup, api.MEM_DEVICE, *dev_args), res))
    # timed epochs (device-resident inputs), as a user runs them: epochs after the first
    # replayed from the solve's captured CUDA graph, no stage events
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    ck = clocks_start(local)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    eng._check(eng.solve_raw(problem(args.steps, api.MEM_DEVICE, *dev_args), res))
    e1.record(stream)
    torch.cuda.synchronize(dev)
    clocks = clocks_stop(ck)
    if world > 1:
        dist.barrier()
    ms = e0.elapsed_time(e1)
    # the same epochs again with every stage bracketed by CUDA events on the library's
    # stream (eager launches): the per-kernel times of the roofline
    eng.set_profiling(True)
    eng._check(eng.solve_raw(problem(args.steps, api.MEM_DEVICE, *dev_args), res))
    torch.cuda.synchronize(dev)
    stages = eng.stage_times()
    eng.set_profiling(False)
    ms = replica_max(ms, world, dev)
    ms_step = ms / args.steps
    epoch_loss = loss[: args.steps].cpu().numpy()

    # e2e: the full 10-epoch job through the C ABI with pinned host buffers
    if args.no_e2e:
        return _report(args, cfg, rank, world, ms, ms_step, stages, clocks, epoch_loss, None,
                       wl["led_np"], _support_of(wl)), wl, rank, world
    pin = lambda x: x.cpu().pin_memory()
    hs, hl, hp, ha = pin(wl["stack"]), pin(wl["led"]), pin(wl["P0c"]), pin(wl["P0"])
    # the outputs of the reference's mex call, [O, P] (cuFPM_pure_v3.cu plhs[0..1]), plus
    # the per-epoch loss (80 bytes); the centred spectrum is an extra of this engine
    hO = torch.empty((H, H), dtype=torch.complex64).pin_memory()
    hP = torch.empty((h, h), dtype=torch.complex64).pin_memory()
    hL = torch.empty(JOB_EPOCHS, dtype=torch.float64).pin_memory()
    hres = api.Result(object=hO.data_ptr(), spectrum=None, pupil=hP.data_ptr(),
                      loss=hL.data_ptr())
    hprob = problem(JOB_EPOCHS, api.MEM_HOST, hs.data_ptr(), hl.data_ptr(), hp.data_ptr(),
                    ha.data_ptr())
    def host_job(profile: bool):
        eng.set_profiling(profile)
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)
        w0 = time.perf_counter()
        eng._check(eng.solve_raw(hprob, hres))
        t = time.perf_counter() - w0       # the call returns after its final synchronisation
        st = eng.stage_times() if profile else None
        eng.set_profiling(False)
        return t, st

    host_job(False)                        # warm-up: first-touch of the host-path buffers
    jobs = [host_job(i == 2) for i in range(3)]
    e2e_s = float(np.median([t for t, _ in jobs]))
    e2e_s = replica_max(e2e_s, world, dev)
    split = None
    prof = jobs[2][1]
    if prof:
        h2d_ms = prof.get("copy_inputs_h2d", (0, 0.0, False))[1]
        d2h_ms = prof.get("copy_outputs_d2h", (0, 0.0, False))[1]
        dev_ms = sum(v[1] for k, v in prof.items() if v[2])
        split = {"h2d_ms": round(h2d_ms, 2), "device_ms": round(dev_ms, 2),
                 "d2h_ms": round(d2h_ms, 2), "job_ms": round(jobs[2][0] * 1e3, 2),
                 "host_ms": round(jobs[2][0] * 1e3 - h2d_ms - d2h_ms - dev_ms, 2),
                 "note": "CUDA events around the copies and kernels of the third job; host_ms "
                         "= the rest of the call (validation, planning, launch gaps)"}
    h2d = sum(x.numel() * x.element_size() for x in (hs, hl, hp, ha))
    d2h = sum(x.numel() * x.element_size() for x in (hO, hP, hL))
    e2e = {"value": round(e2e_s, 4), "unit": "s", "h2d_bytes_per_step": h2d,
           "d2h_bytes_per_step": d2h, "jobs_s": [round(t, 4) for t, _ in jobs],
           "split": split,
           "note": "one 10-epoch job per step through fpm_solve with pinned host buffers; "
                   "stack/LEDs/pupil in, object+pupil+loss out (the mex's outputs); median "
                   "of 3 jobs after 1 warm-up job"}
    out = _report(args, cfg, rank, world, ms, ms_step, stages, clocks, epoch_loss, e2e,
                  wl["led_np"], _support_of(wl))
    if out is not None:
        out["autotune"] = {"report": tune_report, "seconds": round(t_tune, 2)}
    eng.close()
    return out, wl, rank, world


# DRAM traffic / algorithmic bytes of a launch, from one ncu capture of the kernel on a
# smaller case (25 LEDs, batch 8: 6.972 GB measured for 7.024 GB algorithmic); the object and moment terms dominate and scale with the units
# processed, so the full-size launch's traffic is this ratio x its algorithmic bytes.
TRAFFIC_RATIO = {"cols_update": 0.993}


def _report(args, cfg, rank, world, ms, ms_step, stages, clocks, epoch_loss, e2e, wl_led,
            sup=None):
    out = None
    if rank == 0:
        peak, peak_kind = measured_peaks()
        sb = stage_bytes(cfg, wl_led, sup)
        st_rep = {}
        prof_ms = sum(v[1] for v in stages.values())
        for name, (n, tms, own) in stages.items():
            avg = tms / n
            gbs = sb.get(name, 0) / (avg * 1e-3) / 1e9 if avg > 0 else 0.0
            st_rep[name] = {"launches": n, "ms_total": round(tms, 3), "ms_avg": round(avg, 4),
                            "share": round(tms / prof_ms, 4), "gbs": round(gbs, 1),
                            "frac_of_measured_hbm": round(gbs / peak, 3), "own_kernel": own}
        own_stages = {k: v for k, v in st_rep.items() if v["own_kernel"]}
        dom = max(st_rep, key=lambda k: st_rep[k]["ms_total"])
        # the roofline's kernel: the longest own stage with an algorithmic byte count
        dom_own = max((k for k in own_stages if k in sb), key=lambda k: own_stages[k]["ms_total"])
        dk = st_rep[dom_own]
        out = {
            "metric": METRIC, "value": round(ms_step * JOB_EPOCHS / 1e3, 4), "unit": "s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms_step, 3), "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 (complex64)",
            "data": "synthetic (seeded, generated on GPU)" if not args.quick_data else "random stack (profiling)",
            "config": dict(cfg.describe(), parallelism=f"replicas x{world}" if world > 1 else "single GPU",
                           step="one epoch (361 LEDs, 14 mini-batches)"),
            "s_per_epoch": round(ms_step / 1e3, 5),
            "led_updates_per_s": round(world * cfg.L / (ms_step / 1e3), 1),
            "loss_per_epoch": [float(x) for x in epoch_loss],
            "gpu_launches": int(sum(v["launches"] for v in own_stages.values())),
            "clocks": clocks,
            "e2e": e2e,
            "roofline": {"bound": "hbm", "kernel": dom_own,
                         "achieved": round(dk["gbs"], 1), "peak": peak, "unit": "GB/s",
                         "frac": round(dk["gbs"] / peak, 3),
                         "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else "fallback 6650 GB/s",
                         "traffic": (round(TRAFFIC_RATIO[dom_own] * sb[dom_own])
                                     if dom_own in TRAFFIC_RATIO else None),
                         "traffic_source": "ncu dram__bytes_read+write on a 25-LED case, scaled"
                                           " by the units processed",
                         "bytes_per_launch": sb[dom_own],
                         "dominant_stage_overall": dom},
            "stages": st_rep,
            "stages_note": "per-stage CUDA-event times of a second run of the same epochs "
                           "with the stages launched eagerly; the timed run replays its "
                           "epochs from a captured graph",
        }
    return out


def cpu_baseline_for(cfg: Cfg, wl, steps=2):
    O0, P, Y, led = cpu_inputs(cfg, wl, cfg.batch)
    job, workers, per_step = cpu_sample(cfg, O0, P, Y, led, steps=steps, warmup=1)
    return {"value": round(job, 2), "unit": "s", "cores": workers, "kind": "port",
            "sample": f"{steps} mini-batches of {cfg.batch} LEDs at full size (FFT2 + IFFT2 + "
                      f"RMSprop on {cfg.H}^2, per-LED pipeline on {cfg.h}^2), FP32 numpy/pocketfft "
                      f"with {workers} threads; projected to {JOB_EPOCHS} epochs x "
                      f"{math.ceil(cfg.L / cfg.batch)} batches"}


def accuracy_for(cfg: Cfg, wl, s_per_epoch: float, epochs: int = JOB_EPOCHS):
    """Per-epoch relative error (||a - b|| / ||b||, complex, no phase alignment) of the
    engine's object and pupil against an FP64 run of the same job from the same start, next
    to the FP32 twin's (torch complex64, cuFFT).  The FP64 run is the torch restatement of
    the oracle (oracle/torch_ref.py) on the GPU, used here as the checker only, outside every
    timed region.  The engine's state after epoch k comes from a k-epoch solve (the solve
    restarts from the same object, pupil and zero moments every time, so these are the
    states of one 10-epoch job).  The spectrum error equals the object error (Parseval)."""
    import torch
    import fpm_b200
    from fpm_b200 import api
    from oracle import torch_ref as tr
    t_start = time.perf_counter()
    dev = wl["stack"].device
    H, h = cfg.H, cfg.h
    opt = (cfg.lr, cfg.beta, cfg.eps)
    eng = fpm_b200.Engine(dev.index or 0)
    O0 = torch.empty((H, H), dtype=torch.complex64, device=dev)       # memory [c][r]
    O = torch.empty_like(O0)
    P = torch.empty((h, h), dtype=torch.complex64, device=dev)

    def solve(k, object_init):
        prob = api.Problem(h=h, n_leds=cfg.L, pratio=cfg.pratio, batch=cfg.batch, epochs=k,
                           lr=cfg.lr, beta=cfg.beta, eps=cfg.eps, pupil_margin=0.2,
                           lr_halve_after=12, lr_decay=0.5, loss_kind=0, memory=api.MEM_DEVICE,
                           stack_type=api.STACK_U16, stack=wl["stack"].data_ptr(),
                           led_idx=wl["led"].data_ptr(), pupil_init=wl["P0c"].data_ptr(),
                           pupil_amp=wl["P0"].data_ptr(), object_init=object_init)
        dst = O0 if k == 0 else O
        eng._check(eng.solve_raw(prob, api.Result(object=dst.data_ptr(), spectrum=None,
                                                  pupil=P.data_ptr(), loss=None)))
        torch.cuda.synchronize(dev)

    solve(0, None)                     # the engine's starting object: imresize(Y_1, pratio)
    pages = tr.page_normaliser(wl["stack"].transpose(1, 2))
    ref = []                           # FP64 states after every epoch, kept in complex64

    def keep(ep, Ok, Pk, loss):
        ref.append((Ok.to(torch.complex64), Pk.to(torch.complex64), float(loss)))

    args = (O0.T, wl["P0c"].T, pages, wl["led_np"], wl["P0"].T, cfg.pratio, epochs, cfg.batch)
    tr.cufpm_pure_v3(*args, opt=opt, on_epoch=keep)
    twin = []
    tr.cufpm_pure_v3(*args, opt=opt, ctype=torch.complex64,
                     on_epoch=lambda ep, Ok, Pk, l: twin.append(
                         (tr.rel_err(Ok, ref[ep][0]), tr.rel_err(Pk, ref[ep][1]))))
    # the storage question: the same FP64 run on amplitudes rounded to FP16 (what an FP16
    # stack would hold), against the FP64 run on the exact single-precision amplitudes
    half = []
    tr.cufpm_pure_v3(O0.T, wl["P0c"].T, lambda a, n: pages(a, n).half().float(), wl["led_np"],
                     wl["P0"].T, cfg.pratio, epochs, cfg.batch, opt=opt,
                     on_epoch=lambda ep, Ok, Pk, l: half.append(tr.rel_err(Ok, ref[ep][0])))
    ours = []
    for k in range(1, epochs + 1):
        solve(k, O0.data_ptr())
        ours.append((tr.rel_err(O.T, ref[k - 1][0]), tr.rel_err(P.T, ref[k - 1][1])))
    spec_err = tr.rel_err(torch.fft.fft2(O.T.to(torch.complex128)),
                          torch.fft.fft2(ref[-1][0].to(torch.complex128)))
    eng.close()
    obj = [o for o, _ in ours]
    within = next((k for k, e in enumerate(obj) if e > 1e-3), len(obj))
    twin_within = next((k for k, (e, _) in enumerate(twin) if e > 1e-3), len(twin))
    out = {"reference": "FP64 run of the same job (torch complex128 restatement of the oracle, "
                        "pinned against the numpy FP64 oracle), same start",
           "epochs": epochs,
           "object_rel_err": [float(f"{e:.3e}") for e in obj],
           "pupil_rel_err": [float(f"{p:.3e}") for _, p in ours],
           "spectrum_rel_err_final": float(f"{spec_err:.3e}"),
           "fp32_twin_object_rel_err": [float(f"{e:.3e}") for e, _ in twin],
           "fp32_twin_pupil_rel_err": [float(f"{p:.3e}") for _, p in twin],
           "fp64_loss": [r[2] for r in ref],
           "fp16_stack_object_rel_err": [float(f"{e:.3e}") for e in half],
           "fp16_stack_note": "FP64 run on amplitudes rounded to FP16 against the FP64 run "
                              "on the exact amplitudes: the cost of holding the stack in "
                              "FP16 instead of the exact uint16 counts (same 2 B/px)",
           "epochs_within_1e-3": within, "fp32_twin_epochs_within_1e-3": twin_within,
           "s_within_1e-3": round(within * s_per_epoch, 4),
           "note": "every FP32 run (this engine, the FP32 twin) sits at the same distance "
                   "from FP64: sign() in the feature-domain loss flips on residual "
                   "differences within an FP32 rounding of zero, whatever the FFT; "
                   "epochs_within_1e-3 counts the leading epochs whose object error stays at "
                   "or below 1e-3",
           "leg_wall_s": round(time.perf_counter() - t_start, 1)}
    del ref, twin, O0, O, P
    torch.cuda.empty_cache()
    return out


def make_instances_gpu(n: int, seed: int, dev):
    """Seeded uneven instances of the batched configuration: low-res side uniform in
    {128, 192, 256, 384, 512}, LED grid in {11, 13, 15, 17, 19} (121-361 LEDs), up-sampling
    uniform in 4..8, each a smooth random object, the circular pupil of the optics, and
    uint16 frames (Poisson at 3e4 peak counts) of its forward model; generated with torch
    on the GPU, arrays in column-major memory as the C ABI takes them."""
    import torch
    from fpm_b200 import synth
    rng = np.random.default_rng(seed)
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    out = []
    for i in range(n):
        h = int(rng.choice([128, 192, 256, 384, 512]))
        grid = int(rng.choice([11, 13, 15, 17, 19]))
        p = int(rng.integers(4, 9))
        H = h * p
        f0 = torch.fft.fftfreq(H, device=dev)
        f1 = torch.fft.rfftfreq(H, device=dev)

        def smooth(x, sigma):
            X = torch.fft.rfft2(x)
            X *= torch.exp(-2 * (math.pi * sigma) ** 2 * f0 * f0)[:, None]
            X *= torch.exp(-2 * (math.pi * sigma) ** 2 * f1 * f1)[None, :]
            y = torch.fft.irfft2(X, s=(H, H))
            return (y - y.min()) / (y.max() - y.min())
        amp = 0.5 + 0.5 * smooth(torch.rand((H, H), generator=g, device=dev), 3.0)
        ph = (smooth(torch.randn((H, H), generator=g, device=dev), 4.0) - 0.5) * math.pi
        spec = torch.fft.fftshift(torch.fft.fft2(torch.polar(amp, ph)))
        del amp, ph
        optics = synth.Optics(led_grid=grid)
        circ = synth.pupil_circle(h, optics)
        P = torch.from_numpy(circ.astype(np.complex64)).to(dev)
        led = synth.led_indices(h, p, optics)
        ar = torch.arange(h, device=dev)
        frames = []
        for kl, kt in led:
            sub = spec.index_select(0, (int(kt) - 1 + ar) % H).index_select(1, (int(kl) - 1 + ar) % H)
            x = torch.fft.ifft2(torch.fft.ifftshift(sub * P)) / (p * p)
            frames.append(x.real ** 2 + x.imag ** 2)
        del spec
        I = torch.stack(frames)
        counts = torch.poisson(I * (3e4 / float(I.max())), generator=g).clamp_(max=65535)
        stack = counts.to(torch.int32).transpose(1, 2).contiguous().to(torch.uint16)   # [l][c][r]
        del I, counts, frames
        P0 = torch.from_numpy(np.ascontiguousarray(circ.T)).to(dev)
        out.append({"h": h, "pratio": p, "L": len(led), "stack": stack, "P0": P0,
                    "P0c": P0.to(torch.complex64),
                    "led": torch.from_numpy(np.ascontiguousarray(led, np.int32)).to(dev)})
    torch.cuda.synchronize(dev)
    return out


def run_instances(args, cfg: Cfg):
    """The batched-instances configuration: 48 independent reconstructions of uneven size
    (low-res side 128-512, 121-361 LEDs, up-sampling 4-8, LED batch 26, 10 epochs), run by
    one fpm_solve_batch call (concurrent instances on a pool of streams, epochs replayed
    from captured graphs) against the same instances solved one by one with fpm_solve;
    aggregate LED-updates/s.  One GPU."""
    import ctypes as C
    import torch
    import fpm_b200
    from fpm_b200 import api
    dev = torch.device("cuda", 0)
    n, E = args.instances, JOB_EPOCHS
    inst = make_instances_gpu(n, 1000 + cfg.seed, dev)
    eng = fpm_b200.Engine(0)
    probs = (api.Problem * n)()
    ress = (api.Result * n)()
    outs = []
    for i, a in enumerate(inst):
        H, h = a["h"] * a["pratio"], a["h"]
        O = torch.empty((H, H), dtype=torch.complex64, device=dev)
        P = torch.empty((h, h), dtype=torch.complex64, device=dev)
        probs[i] = api.Problem(h=h, n_leds=a["L"], pratio=a["pratio"], batch=cfg.batch, epochs=E,
                               lr=cfg.lr, beta=cfg.beta, eps=cfg.eps, pupil_margin=0.2,
                               lr_halve_after=12, lr_decay=0.5, loss_kind=0, memory=api.MEM_DEVICE,
                               stack_type=api.STACK_U16, stack=a["stack"].data_ptr(),
                               led_idx=a["led"].data_ptr(), pupil_init=a["P0c"].data_ptr(),
                               pupil_amp=a["P0"].data_ptr(), object_init=None)
        ress[i] = api.Result(object=O.data_ptr(), spectrum=None, pupil=P.data_ptr(), loss=None)
        outs.append((O, P))
    st = (C.c_int * n)()

    def batch_call(eager=False):
        rc = eng.lib.fpm_solve_batch(eng._ctx, probs, ress, n, 1 if eager else 0, st)
        eng._check(rc)

    def one_by_one():
        for i in range(n):
            eng._check(eng.solve_raw(probs[i], ress[i]))

    led_updates = sum(a["L"] for a in inst) * E
    timings = {}
    for name, fn in (("one_by_one", one_by_one), ("batch_eager", lambda: batch_call(True)),
                     ("batch", batch_call)):
        fn()                                   # warm-up: buffers, tables, kernel attributes
        torch.cuda.synchronize(dev)
        ts = []
        for _ in range(max(1, args.steps)):
            t0 = time.perf_counter()
            fn()                               # each call returns after its results are ready
            ts.append(time.perf_counter() - t0)
        timings[name] = float(np.median(ts))
        if name == "one_by_one":
            ref = [(O.clone(), P.clone()) for O, P in outs]
    same = all(torch.equal(O, r[0]) and torch.equal(P, r[1]) for (O, P), r in zip(outs, ref))
    # where the time goes: each instance solved alone (after the warm-up above)
    per = []
    for i in range(n):
        t0 = time.perf_counter()
        eng._check(eng.solve_raw(probs[i], ress[i]))
        per.append(time.perf_counter() - t0)
    pow2 = lambda v: v & (v - 1) == 0
    any_size = [not (pow2(a["h"]) and pow2(a["h"] * a["pratio"])) for a in inst]
    t_any = sum(t for t, g in zip(per, any_size) if g)
    value = led_updates / timings["batch"]
    line = {"metric": "aggregate LED-updates/s, 48 uneven FPM instances (fpm_solve_batch)",
            "value": round(value, 1), "unit": "LED-updates/s", "n_gpus": 1, "steps": args.steps,
            "warmup": 1, "ms_per_step": round(timings["batch"] * 1e3, 2),
            "higher_is_better": True, "dtype": "f32 (complex64)",
            "data": "synthetic (seeded, generated on GPU)",
            "config": {"workload": f"{n} independent reconstructions, low-res side in "
                                   "{128,192,256,384,512}, 121-361 LEDs, up-sampling 4-8, "
                                   f"LED batch {cfg.batch}, {E} epochs, uint16 frames",
                       "instances": [(a["h"], a["L"], a["pratio"]) for a in inst],
                       "led_updates_per_job": led_updates,
                       "step": "one call solving every instance (10 epochs each)"},
            "one_by_one_led_updates_per_s": round(led_updates / timings["one_by_one"], 1),
            "batch_eager_led_updates_per_s": round(led_updates / timings["batch_eager"], 1),
            "speedup_vs_one_by_one": round(timings["one_by_one"] / timings["batch"], 3),
            "seconds": {k: round(v, 4) for k, v in timings.items()},
            "batch_equals_one_by_one_bitwise": bool(same),
            "instance_seconds": [round(t, 4) for t in per],
            "any_size_instances": int(sum(any_size)),
            "any_size_share_of_time": round(t_any / max(sum(per), 1e-12), 3),
            "timing": "host wall clock around each call (each returns after its final "
                      "synchronisation), median of the steps"}
    eng.close()
    print(json.dumps(line), flush=True)


def run_warmstart(args, cfg: Cfg):
    """The learned warm start.  Training set: `--train-pairs` seeded objects of
    1024^2 seen through 11 x 11 LEDs as 256^2 frames (pratio 4); each pair is the 25
    central amplitudes and the low-pass of the plain method's object after 20 epochs (LED
    batch 8, lr 2e-3).  The network (25 inputs, 32 base channels) is trained with Adam in
    libfpm's own kernels.  Evaluation on held-out seeds at 1024^2 frames from 19 x 19 LEDs
    -> 8192^2 (pratio 8, LED batch 26, lr 5e-4, the headline's settings; the network runs
    on the 1024^2 frames and its output is up-sampled bicubically): per-epoch error of the
    plain start imresize(Y_1, pratio) and of the learned start (falling back to the plain
    start where it raises the first-epoch loss) against the true object and against the
    plain method's converged object (60 epochs), and the epochs each start needs to reach
    the plain start's 20-epoch error.  The object model's smoothing scales with pratio so
    that training and evaluation objects have the same physical statistics.  --ws-small
    runs both halves at 64^2 x 121 -> 256^2."""
    import torch
    import fpm_b200
    from fpm_b200 import warmstart as ws
    small = args.ws_small
    ht, pt, gt, Et, Bt, lrt = (64, 4, 11, 20, 8, 2e-3) if small else (256, 4, 11, 20, 8, 2e-3)
    he, pe, ge, E, B, lr = (64, 4, 11, 20, 8, 2e-3) if small else (1024, 8, 19, 20, 26, 5e-4)
    n_eval, E_ref = (16, 60) if small else (4, 60)
    dev = torch.device("cuda", 0)
    eng = fpm_b200.Engine(0)
    t0 = time.perf_counter()
    x, t = ws.training_pairs(eng, args.train_pairs, ht, pt, gt, Et, Bt, lrt, seed0=10_000,
                             smooth_scale=1.0)
    torch.cuda.synchronize()
    t_pairs = time.perf_counter() - t0
    net = ws.Network(eng, 25, 32, seed=1)
    t0 = time.perf_counter()
    hist = ws.train(net, x, t, args.train_epochs, 32, 1e-3)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    del x, t
    torch.cuda.empty_cache()
    pbs = [ws.make_problem_gpu(he, pe, ge, 90_000 + i, dev, pe / pt) for i in range(n_eval)]
    stacks = [ws.simulate_stack(eng, pb, 31 + i) for i, pb in enumerate(pbs)]
    refs, _ = ws.solve_objects(eng, pbs, stacks, E_ref, B, lr)        # plain, converged
    plain, learned, fallback, plain_r, learned_r = ws.evaluate(eng, net, pbs, stacks, E, B, lr,
                                                               refs)
    # seconds per epoch of one evaluation solve, and of the network's start
    prob = ws.problem_struct(pbs[0], stacks[0], E, B, lr)
    O = torch.empty((he * pe, he * pe), dtype=torch.complex64, device=dev)
    res = fpm_b200.Result(object=O.data_ptr(), spectrum=None, pupil=None, loss=None)
    eng._check(eng.solve_raw(prob, res))
    torch.cuda.synchronize()
    w0 = time.perf_counter()
    eng._check(eng.solve_raw(prob, res))
    s_epoch = (time.perf_counter() - w0) / E
    net.initial_object(ws.problem_struct(pbs[0], stacks[0], 1, B, lr), dev)
    torch.cuda.synchronize()
    w0 = time.perf_counter()
    net.initial_object(ws.problem_struct(pbs[0], stacks[0], 1, B, lr), dev)
    torch.cuda.synchronize()
    s_net = time.perf_counter() - w0
    q = plain[:, E]                                   # the plain start's 20-epoch error

    def epochs_to(curve, target):
        hit = np.nonzero(curve <= target * (1 + 1e-9))[0]
        return int(hit[0]) if len(hit) else None
    ep_plain = [epochs_to(plain[i], q[i]) for i in range(len(pbs))]
    ep_learn = [epochs_to(learned[i], q[i]) for i in range(len(pbs))]
    reached = [e for e in ep_learn if e is not None]
    to_ref = {}
    for thr in (1e-2, 1e-3):
        to_ref[f"{thr:g}"] = {"plain": [epochs_to(plain_r[i], thr) for i in range(len(pbs))],
                              "learned": [epochs_to(learned_r[i], thr) for i in range(len(pbs))]}
    line = {"metric": "epochs to the plain start's 20-epoch error, learned vs plain start",
            "value": round(float(np.mean(ep_plain)) / max(float(np.mean(reached)), 1.0), 3)
                     if len(reached) == len(pbs) else None,
            "value_note": "mean epochs of the plain start / mean epochs of the learned start, "
                          "the latter counted as at least 1 (the network's start costs about "
                          "one solve epoch, s_network_start)",
            "unit": "x fewer epochs", "n_gpus": 1, "higher_is_better": True,
            "dtype": "f32 (complex64) solves; BF16 x BF16 -> FP32 convolutions (tcgen05)",
            "data": "synthetic (seeded objects, simulated frames)",
            "config": {"workload": f"learned warm start: trained on {ht}^2 frames x {gt * gt} LEDs "
                                   f"-> {ht * pt}^2, evaluated on {he}^2 frames x {ge * ge} LEDs "
                                   f"-> {he * pe}^2 (pratio {pe}, LED batch {B}, lr {lr:g})",
                       "train_pairs": args.train_pairs, "train_epochs": args.train_epochs,
                       "pair_solve": f"{Et} epochs, LED batch {Bt}, lr {lrt:g}",
                       "network": "4-level encoder-decoder, 25 inputs, base 32, "
                                  f"{net.n_params} parameters", "held_out": len(pbs),
                       "reference_epochs": E_ref},
            "plain_error_per_epoch": [round(float(v), 5) for v in plain.mean(0)],
            "learned_error_per_epoch": [round(float(v), 5) for v in learned.mean(0)],
            "plain_dist_to_converged_per_epoch": [round(float(v), 5) for v in plain_r.mean(0)],
            "learned_dist_to_converged_per_epoch": [round(float(v), 5) for v in learned_r.mean(0)],
            "error_after_epochs": {"epochs": E, "plain": round(float(plain[:, E].mean()), 5),
                                   "learned": round(float(learned[:, E].mean()), 5)},
            "epochs_plain": ep_plain, "epochs_learned": ep_learn,
            "epochs_to_converged": to_ref,
            "fallbacks": int(sum(fallback)),
            "s_per_epoch": round(s_epoch, 5), "s_network_start": round(s_net, 5),
            "s_to_plain_20_epoch_error": {
                "plain": round(float(np.mean(ep_plain)) * s_epoch, 3),
                "learned": round(float(np.mean(reached)) * s_epoch + s_net, 3) if reached else None},
            "train_loss_first_last": [round(hist[0], 6), round(hist[-1], 6)],
            "seconds": {"pairs": round(t_pairs, 1), "training": round(t_train, 1)}}
    net.close()
    eng.close()
    print(json.dumps(line), flush=True)


def run_simulate(args, cfg: Cfg):
    """Forward model (fpm_simulate): all LED images of a 16384^2 object, device-resident.
    Not the headline metric: a separate line for the simulator row."""
    import torch
    import fpm_b200
    from fpm_b200 import api, synth
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    g = torch.Generator(device=dev)
    g.manual_seed(cfg.seed)
    H, h = cfg.H, cfg.h
    O = torch.polar(0.5 + 0.5 * torch.rand((H, H), generator=g, device=dev),
                    torch.randn((H, H), generator=g, device=dev))
    optics = synth.Optics(led_grid=cfg.grid)
    P = torch.from_numpy(np.ascontiguousarray(synth.pupil_circle(h, optics).T)).to(dev).to(torch.complex64)
    led = torch.from_numpy(np.ascontiguousarray(synth.led_indices(h, cfg.pratio, optics))).to(dev)
    out = torch.empty((cfg.L, h, h), dtype=torch.float32, device=dev)
    stream = torch.cuda.Stream(device=dev)
    eng = fpm_b200.Engine(0, stream=stream.cuda_stream)
    torch.cuda.synchronize(dev)
    call = lambda: eng._check(eng.lib.fpm_simulate(eng._ctx, O.data_ptr(), P.data_ptr(), led.data_ptr(),
                                                   h, cfg.pratio, cfg.L, api.SIM_INTENSITY,
                                                   out.data_ptr(), api.MEM_DEVICE))
    for _ in range(args.warmup):
        call()
    eng.set_profiling(True)
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    stages = {}
    e0.record(stream)
    for _ in range(args.steps):
        call()
        for k, v in eng.stage_times().items():
            n, t, _ = stages.get(k, (0, 0.0, v[2]))
            stages[k] = (n + v[0], t + v[1], v[2])
    e1.record(stream)
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1) / args.steps
    peak, _ = measured_peaks()
    px = h * h * cfg.L
    sb = {"spectrum_fft2": 32 * H * H, "lr_cols_inverse": 16 * px, "sim_rows_inverse": 16 * px,
          "sim_magnitude": 12 * px}
    # bytes per call over the stage's summed time in the timed calls
    st = {k: {"launches": n, "ms_total": round(t, 3),
              "gbs": round(sb.get(k, 0) * args.steps / (t * 1e-3) / 1e9, 1)}
          for k, (n, t, own) in stages.items()}
    dom = max(st, key=lambda k: st[k]["ms_total"])
    line = {"metric": "forward-model LED images per second", "value": round(cfg.L / (ms * 1e-3), 1),
            "unit": "images/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms, 3), "higher_is_better": True, "dtype": "f32 (complex64)",
            "data": "synthetic (seeded random object, circular pupil)",
            "config": {"workload": f"forward model: {H}x{H} object -> {cfg.L} LED images of {h}x{h}",
                       "h": h, "H": H, "leds": cfg.L},
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": st[dom]["gbs"], "peak": peak,
                         "unit": "GB/s", "frac": round(st[dom]["gbs"] / peak, 3)},
            "stages": st}
    eng.close()
    print(json.dumps(line), flush=True)


def _events_ms(stream, fn, steps):
    """Mean device ms of fn() over `steps` calls, CUDA events on the engine's stream."""
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(steps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def run_ingest(args, cfg: Cfg):
    """Ingest row: TIFF frames -> normalised amplitude in HBM (codes_v2/main_run_FPM.m:26-45).
    The host read runs on a bounded sample of frames written to a temporary directory (read
    from the page cache); the device normalisation runs on the full-size stack."""
    import shutil
    import tempfile
    import torch
    import fpm_b200
    from fpm_b200 import api, frames
    from oracle import fpm_oracle as orc
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    h, L, S = cfg.h, cfg.L, min(cfg.L, 32)
    rng = np.random.default_rng(cfg.seed)
    tmp = Path(tempfile.mkdtemp(prefix="fpm_ingest_"))
    try:
        sample = rng.integers(0, 65536, size=(h, h, S), dtype=np.uint16)
        paths = frames.write_frames(tmp, sample)
        stream = torch.cuda.Stream(device=dev)
        eng = fpm_b200.Engine(0, stream=stream.cuda_stream)
        for _ in range(args.warmup):
            Y = api.read_tiff_stack(paths, h)
        t_read = []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            Y = api.read_tiff_stack(paths, h)
            t_read.append(time.perf_counter() - t0)
        assert np.array_equal(Y, sample)
        read_s = float(np.median(t_read))
        # end to end per frame: host read + copy in + normalise on the device + amplitude out
        pin = torch.empty((S, h, h), dtype=torch.uint16).pin_memory()
        out = torch.empty((S, h, h), dtype=torch.float32).pin_memory()
        import ctypes as C
        names = (C.c_char_p * S)(*[os.fsencode(q) for q in paths])
        t_e2e = []
        for k in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            # frames straight into pinned pages (column-major h x h each), then the device
            eng._check(eng.lib.fpm_read_tiff_stack(eng._ctx, names, S, 0, 0, h, api.INGEST_U16,
                                                   pin.data_ptr(), 0))
            eng._check(eng.lib.fpm_normalise_stack(eng._ctx, pin.data_ptr(), pin.numel(),
                                                   out.data_ptr(), api.MEM_HOST))
            if k >= args.warmup:
                t_e2e.append(time.perf_counter() - t0)
        e2e_s = float(np.median(t_e2e))
        assert np.array_equal(pin.numpy().transpose(2, 1, 0), sample)
        # device normalisation of the full stack, inputs resident in HBM
        counts = torch.randint(0, 65536, (L, h, h), dtype=torch.int32, device=dev).to(torch.uint16)
        amp = torch.empty((L, h, h), dtype=torch.float32, device=dev)
        norm = lambda: eng._check(eng.lib.fpm_normalise_stack(
            eng._ctx, counts.data_ptr(), counts.numel(), amp.data_ptr(), api.MEM_DEVICE))
        for _ in range(args.warmup):
            norm()
        ms = _events_ms(stream, norm, args.steps)
        nbytes = 8 * counts.numel()          # min / max read 2, normalise read 2 + write 4 per px
        peak, _ = measured_peaks()
        gbs = nbytes / (ms * 1e-3) / 1e9
        # CPU restatement: Pillow decode + mean + normalise of the same frames
        t0 = time.perf_counter()
        ref = np.stack([orc.read_frame(p, 0, 0, h) for p in paths[:8]], axis=2)
        orc.normalise_stack_f32(ref)
        cpu_frame = (time.perf_counter() - t0) / 8
        line = {"metric": "TIFF frames ingested per second (file -> normalised amplitude)",
                "value": round(S / e2e_s, 1), "unit": "frames/s", "n_gpus": 1,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(e2e_s * 1e3, 3),
                "higher_is_better": True, "dtype": "u16 -> f32", "data": "synthetic (seeded uint16 frames)",
                "config": {"workload": f"ingest: {S} TIFF frames of {h}x{h} uint16 (page cache) per "
                                       f"step; device normalisation on {L} frames", "h": h,
                           "frames_sample": S, "frames_device": L},
                "host_read": {"frames_per_s": round(S / read_s, 1),
                              "gbs": round(S * h * h * 2 / read_s / 1e9, 2),
                              "threads": os.cpu_count()},
                "roofline": {"bound": "hbm", "kernel": "stack_minmax + normalise",
                             "achieved": round(gbs, 1), "peak": peak, "unit": "GB/s",
                             "frac": round(gbs / peak, 3), "traffic": None,
                             "ms_per_launch_pair": round(ms, 4)},
                "cpu_baseline": {"value": round(1.0 / cpu_frame, 2), "unit": "frames/s", "cores": 1,
                                 "kind": "port", "sample": "8 frames: Pillow decode, float mean, "
                                                           "normalise (numpy)"},
                "e2e": {"value": round(S / e2e_s, 1), "unit": "frames/s",
                        "h2d_bytes_per_step": S * h * h * 2, "d2h_bytes_per_step": S * h * h * 4}}
        eng.close()
        print(json.dumps(line), flush=True)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


def run_optimizer(args, cfg: Cfg):
    """Optimiser row: one step of the MATLAB optimiser classes on the H x H object,
    device-resident (the script-level loop's per-batch update)."""
    import torch
    import fpm_b200
    from fpm_b200 import api
    from oracle import fpm_oracle as orc
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    H = cfg.H
    n = H * H
    g = torch.Generator(device=dev)
    g.manual_seed(cfg.seed)
    p = torch.randn((H, H), dtype=torch.complex64, device=dev, generator=g)
    gr = torch.randn((H, H), dtype=torch.complex64, device=dev, generator=g)
    m1 = torch.zeros_like(p)
    m2 = torch.zeros((H, H), dtype=torch.float32, device=dev)
    stream = torch.cuda.Stream(device=dev)
    eng = fpm_b200.Engine(0, stream=stream.cuda_stream)
    peak, _ = measured_peaks()
    kinds = {"rmsprop": (api.Optimizer(kind=api.OPT_RMSPROP, lr=1.5e-3, beta1=0.999), 24),
             "adam": (api.Optimizer(kind=api.OPT_ADAM, lr=1e-3, beta1=0.9, beta2=0.999, iter=1,
                                    mom1=m1.data_ptr(), mom2=m2.data_ptr()), 48),
             "yogi": (api.Optimizer(kind=api.OPT_YOGI, lr=1e-3, beta1=0.9, beta2=0.999,
                                    mom1=m1.data_ptr(), mom2=m2.data_ptr()), 48)}
    res = {}
    for name, (opt, bpe) in kinds.items():
        step = lambda: eng._check(eng.lib.fpm_optimizer_step(eng._ctx, opt, p.data_ptr(), gr.data_ptr(),
                                                             n, api.MEM_DEVICE))
        for _ in range(args.warmup):
            step()
        ms = _events_ms(stream, step, args.steps)
        res[name] = {"ms": round(ms, 4), "gbs": round(bpe * n / (ms * 1e-3) / 1e9, 1),
                     "bytes_per_element": bpe}
    # CPU restatement on a 2048 x 2048 sample, scaled to the object
    rng = np.random.default_rng(cfg.seed)
    ns = 2048 * 2048
    ps = (rng.standard_normal(ns) + 1j * rng.standard_normal(ns)).astype(np.complex64)
    t0 = time.perf_counter()
    orc.adam_class_step(ps, ps, np.zeros_like(ps), np.zeros(ns, np.float32), 0.9, 0.999, 1e-3, 1)
    cpu_ms = (time.perf_counter() - t0) * 1e3 * n / ns
    dom = res["adam"]
    line = {"metric": "optimizer steps per second on the object (Adam)", "value": round(1e3 / dom["ms"], 1),
            "unit": "steps/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": dom["ms"], "higher_is_better": True, "dtype": "f32 (complex64)",
            "data": "synthetic (seeded random parameter and gradient)",
            "config": {"workload": f"optimizer step on a {H}x{H} complex64 object", "H": H,
                       "inputs": "larger than L2 (2 GiB object)"},
            "roofline": {"bound": "hbm", "kernel": "optimizer_step (Adam)", "achieved": dom["gbs"],
                         "peak": peak, "unit": "GB/s", "frac": round(dom["gbs"] / peak, 3),
                         "traffic": None},
            "kinds": res,
            "cpu_baseline": {"value": round(1e3 / cpu_ms, 3), "unit": "steps/s", "cores": 1,
                             "kind": "port", "sample": "Adam step of the oracle on 2048^2 elements, "
                                                       "scaled to the object"}}
    eng.close()
    print(json.dumps(line), flush=True)


def run_reference(args, cfg: Cfg):
    """Reference arm: the reference's own GPU build (its v3 kernels + cuFFT, driven by the
    replica of cuFPM_v3/cuFPM_pure_v3.cu:75-207 in oracle/ref_harness.cu, built from the
    reference tree into oracle/_ref/libcufpm_ref.so), rank 0 only, on the same workload:
    the same seeded frames, normalised to the float amplitudes the mex takes
    (codes_v2/main_run_FPM.m:43-45), the same starting object imresize(Y_1, pratio) (:48),
    pupil and LED corners.  W warm-up epochs in one call, then K epochs in a second call
    timed with CUDA events around its epoch loop (allocation, cuFFT plans and the copies of
    the inputs are outside, as the mex receives gpuArrays already on the device)."""
    import ctypes as C
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if rank != 0:
        return
    lib_path = ROOT / "oracle" / "_ref" / "libcufpm_ref.so"
    import torch
    if not torch.cuda.is_available():
        print(json.dumps({"impl": "reference", "unavailable": "the reference build is GPU code "
                                                              "and no CUDA device is visible"}))
        return
    if not lib_path.exists():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libcufpm_ref.so was "
                                                              "not built (needs the reference tree)"}))
        return
    from oracle import torch_ref as tr
    dev = torch.device("cuda", 0)
    wl = make_quick_workload_gpu(cfg, dev) if args.quick_data else make_workload_gpu(cfg, dev)
    H, h = cfg.H, cfg.h
    pages = tr.page_normaliser(wl["stack"])                  # memory [l][c][r] kept
    Y = torch.empty((cfg.L, h, h), dtype=torch.float32).pin_memory()
    for a in range(0, cfg.L, 32):
        Y[a:a + 32].copy_(pages(a, min(32, cfg.L - a)))
    O0 = tr.imresize_bicubic(pages(0, 1)[0].T, cfg.pratio)   # [r, c]
    O0 = O0.T.to(torch.float32).to(torch.complex64).contiguous().cpu().pin_memory()  # [c][r]
    P0c = wl["P0c"].cpu().pin_memory()
    P0 = wl["P0"].cpu().pin_memory()
    led = torch.from_numpy(np.ascontiguousarray(wl["led_np"], np.int32)).pin_memory()
    del wl
    torch.cuda.empty_cache()
    O = torch.empty((H, H), dtype=torch.complex64).pin_memory()
    P = torch.empty((h, h), dtype=torch.complex64).pin_memory()
    lib = C.CDLL(str(lib_path))
    vp = C.c_void_p
    lib.ref_solve.argtypes = [C.c_int] * 6 + [C.c_float] * 3 + [vp] * 8
    lib.ref_solve.restype = C.c_int
    ms = np.zeros(3, np.float32)

    def call(epochs):
        rc = lib.ref_solve(h, H, cfg.L, cfg.pratio, epochs, cfg.batch, cfg.lr, cfg.beta, cfg.eps,
                           O0.data_ptr(), P0c.data_ptr(), Y.data_ptr(), led.data_ptr(),
                           P0.data_ptr(), O.data_ptr(), P.data_ptr(), ms.ctypes.data)
        if rc != 0:
            raise SystemExit(f"reference build failed: {rc}")

    call(args.warmup)
    ck = clocks_start(0)
    call(args.steps)
    clocks = clocks_stop(ck)
    loop_ms = float(ms[0])
    ms_step = loop_ms / args.steps
    value = round(ms_step * JOB_EPOCHS / 1e3, 4)
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(ms_step, 3), "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 (complex64)",
            "data": "synthetic (seeded, generated on GPU)" if not args.quick_data else "random stack (profiling)",
            "config": dict(cfg.describe(), parallelism=f"replicas x{world}" if world > 1 else "single GPU",
                           step="one epoch (361 LEDs, 14 mini-batches)"),
            "s_per_epoch": round(ms_step / 1e3, 5),
            "led_updates_per_s": round(cfg.L / (ms_step / 1e3), 1),
            "clocks": clocks,
            "reference_build": {
                "library": "oracle/_ref/libcufpm_ref.so (built by oracle/build_ref.py)",
                "kernels": "cuFPM_v3/cuda/kernels.cuh, compiled for sm_100a", "fft": "cuFFT",
                "loop": "replica of cuFPM_v3/cuFPM_pure_v3.cu:75-207 (oracle/ref_harness.cu)",
                "s_call_with_alloc_and_plans": round(float(ms[1]) / 1e3, 4),
                "stack": "float32 amplitude, 4 B/px (the mex input Y)"},
            "cpu_baseline": {"value": value, "unit": "s", "cores": 1, "kind": "reference",
                             "sample": f"{args.steps} epochs of the full workload on the GPU "
                                       f"(the reference has no CPU implementation of this "
                                       f"path); one host thread drives it"},
            "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--batch", type=int, default=26)
    ap.add_argument("--h", type=int, default=2048)
    ap.add_argument("--pratio", type=int, default=8)
    ap.add_argument("--grid", type=int, default=19)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the default launch choices (profiler runs, whose timings would "
                         "mislead the tuner)")
    ap.add_argument("--train-pairs", type=int, default=2000,
                    help="training pairs of the warm-start workload")
    ap.add_argument("--ws-small", action="store_true",
                    help="warm start at 64^2 x 121 -> 256^2 for training and evaluation")
    ap.add_argument("--train-epochs", type=int, default=30,
                    help="passes over the training pairs (--workload warmstart)")
    ap.add_argument("--instances", type=int, default=48,
                    help="instances of the batched workload (--workload instances)")
    ap.add_argument("--no-accuracy", action="store_true",
                    help="skip the per-epoch error against the FP64 run (one GPU only)")
    ap.add_argument("--workload", default="solve",
                    choices=["solve", "simulate", "ingest", "optimizer", "instances",
                             "warmstart"],
                    help="solve: the reconstruction (headline); simulate: the forward model; "
                         "ingest: TIFF frames to normalised amplitude; optimizer: the MATLAB "
                         "optimiser classes' step on the object")
    ap.add_argument("--quick-data", action="store_true",
                    help="random stack instead of the simulated one (profiler runs only)")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        print("warning: fewer than 3 warm-up steps", file=sys.stderr)
    cfg = Cfg(h=args.h, pratio=args.pratio, grid=args.grid, batch=args.batch)
    if args.impl == "reference":
        run_reference(args, cfg)
        return
    if args.workload != "solve":
        {"simulate": run_simulate, "ingest": run_ingest, "optimizer": run_optimizer,
         "instances": run_instances, "warmstart": run_warmstart}[args.workload](args, cfg)
        return
    out, wl, rank, world = run_ours(args, cfg)
    if rank == 0:
        if world == 1 and not args.no_accuracy:
            try:
                out["accuracy"] = accuracy_for(cfg, wl, out["s_per_epoch"])
            except Exception as e:  # the line still prints; the reason is recorded
                out["accuracy"] = {"error": repr(e)[:300]}
        if world == 1 and not args.no_cpu_baseline:
            try:
                out["cpu_baseline"] = cpu_baseline_for(cfg, wl)
            except Exception as e:  # the line still prints; the reason is recorded
                out["cpu_baseline"] = {"value": None, "error": repr(e)[:200]}
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
