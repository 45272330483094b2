"""Learned warm start: the network of libfpm (fpm_cnn_* in include/fpm.h) and its training.

The plain start of the reference is ``imresize(Y_1, pratio)`` with zero phase
(``codes_v2/main_run_FPM.m:48``).  Here a small encoder-decoder maps the central
bright-field frames (the first ``in_channels`` frames of the spiral order: 25 = the
central 5 x 5 LEDs) to the real and imaginary parts of a low-resolution object, which
the library up-samples bicubically into the starting object.  It is trained on pairs
the plain reconstruction itself produces on seeded synthetic objects: the input is the
problem's bright-field amplitudes, the target the low-pass of the plain method's result
after ``epochs`` epochs (the centre h x h of its spectrum, back at the low resolution,
scaled by 1/pratio^2 so that up-sampling restores the object's scale).  Every forward,
backward and update step runs in libfpm's own kernels; torch only holds device buffers.

Arrays follow the library: planes of h x h in the stack's column-major page layout,
batches [n][channels][h*h].
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import api, synth


class Network:
    """One fpm_cnn: the encoder-decoder with its weights, Adam state and buffers."""

    def __init__(self, engine: api.Engine, in_channels: int = 25, base: int = 32, seed: int = 0):
        self.eng = engine
        self.lib = engine.lib
        self.in_channels = in_channels
        self._net = C.c_void_p()
        st = self.lib.fpm_cnn_create(engine._ctx, in_channels, base, seed, C.byref(self._net))
        if st != api.FPM_OK:
            raise api.FpmError(st, "fpm_cnn_create")
        engine._children.add(self)

    def close(self):
        if self._net:
            self.lib.fpm_cnn_destroy(self._net)
            self._net = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st):
        if st != api.FPM_OK:
            raise api.FpmError(st, self.lib.fpm_cnn_last_error(self._net).decode())

    @property
    def n_params(self) -> int:
        return int(self.lib.fpm_cnn_parameter_count(self._net))

    def get_parameters(self) -> np.ndarray:
        out = np.empty(self.n_params, np.float32)
        self._check(self.lib.fpm_cnn_get_parameters(self._net, out.ctypes.data, out.size))
        return out

    def set_parameters(self, p) -> None:
        p = np.ascontiguousarray(p, np.float32)
        self._check(self.lib.fpm_cnn_set_parameters(self._net, p.ctypes.data, p.size))

    def forward(self, x):
        """x: torch CUDA float32 (n, in_channels, h, h) -> (n, 2, h, h)."""
        import torch
        x = x.contiguous()
        n, _, h, _ = x.shape
        y = torch.empty((n, 2, h, h), dtype=torch.float32, device=x.device)
        torch.cuda.current_stream(x.device).synchronize()
        self._check(self.lib.fpm_cnn_forward(self._net, x.data_ptr(), n, h, y.data_ptr()))
        return y

    def gradients(self, x, t):
        """(loss, gradient of every parameter as a host array) of one batch."""
        import torch
        x, t = x.contiguous(), t.contiguous()
        n, _, h, _ = x.shape
        g = np.empty(self.n_params, np.float32)
        loss = C.c_double()
        torch.cuda.current_stream(x.device).synchronize()
        self._check(self.lib.fpm_cnn_gradients(self._net, x.data_ptr(), t.data_ptr(), n, h,
                                               C.byref(loss), g.ctypes.data))
        return float(loss.value), g

    def train_step(self, x, t, lr: float) -> float:
        import torch
        x, t = x.contiguous(), t.contiguous()
        n, _, h, _ = x.shape
        loss = C.c_double()
        torch.cuda.current_stream(x.device).synchronize()
        self._check(self.lib.fpm_cnn_train_step(self._net, x.data_ptr(), t.data_ptr(), n, h,
                                                float(lr), C.byref(loss)))
        return float(loss.value)

    def initial_object(self, prob: api.Problem, device):
        """The starting object of a device-memory problem: (H, H) complex64 in column-major
        memory (the tensor's [c][r] order, as the C ABI takes object_init)."""
        import torch
        H = prob.h * prob.pratio
        O = torch.empty((H, H), dtype=torch.complex64, device=device)
        torch.cuda.current_stream(device).synchronize()
        self._check(self.lib.fpm_cnn_initial_object(self._net, C.byref(prob), O.data_ptr()))
        return O


    def solve(self, prob: api.Problem, res: api.Result) -> bool:
        """fpm_solve_warm: the solve from the learned start, or from the plain start where
        that one's first-epoch loss is lower; True when the network's start was used."""
        import torch
        used = C.c_int32(0)
        torch.cuda.synchronize()
        self._check(self.lib.fpm_solve_warm(self.eng._ctx, self._net, C.byref(prob),
                                            C.byref(res), C.byref(used)))
        return bool(used.value)


# ---------------------------------------------------------------------------
# problems, training pairs, evaluation
# ---------------------------------------------------------------------------
def make_object_gpu(H: int, seed: int, dev, smooth_scale: float = 1.0):
    """The object model of ``synth.make_object`` drawn on the GPU from a seeded torch
    generator (other random values than numpy's for the same seed): amplitude = uniform
    noise smoothed periodically with a Gaussian of sigma 3 smooth_scale pixels, rescaled to
    [0.5, 1]; phase = normal noise smoothed with sigma 4 smooth_scale, rescaled to
    [-pi/2, pi/2].  (H, H) complex64 in [c][r] order."""
    import torch
    g = torch.Generator(device=dev)
    g.manual_seed(int(seed))

    def smooth(x, sigma):
        f0 = torch.fft.fftfreq(H, device=dev)
        f1 = torch.fft.rfftfreq(H, device=dev)
        w0 = torch.exp(-2.0 * (np.pi * sigma) ** 2 * f0 * f0)
        w1 = torch.exp(-2.0 * (np.pi * sigma) ** 2 * f1 * f1)
        return torch.fft.irfft2(torch.fft.rfft2(x) * w0[:, None] * w1[None, :], s=(H, H))

    def rescale(x, lo, hi):
        mn, mx = x.min(), x.max()
        return (x - mn) / torch.clamp(mx - mn, min=1e-30) * (hi - lo) + lo

    amp = rescale(smooth(torch.rand((H, H), generator=g, device=dev), 3.0 * smooth_scale), 0.5, 1.0)
    ph = rescale(smooth(torch.randn((H, H), generator=g, device=dev), 4.0 * smooth_scale),
                 -np.pi / 2, np.pi / 2)
    return torch.polar(amp, ph).to(torch.complex64)


def make_problem_gpu(h: int, pratio: int, grid: int, seed: int, dev, smooth_scale=None):
    """A seeded problem on the GPU: the synthetic object model of ``synth`` (smooth random
    amplitude in [0.5, 1] and phase in [-pi/2, pi/2]; drawn on the GPU by
    ``make_object_gpu`` with that smoothing scale when smooth_scale is given), the circular
    pupil with a seeded aberration, frames of the forward model with Poisson noise at 3e4
    peak counts (engine's simulator), uint16 stack in column-major pages.  Returns tensors
    and the true object."""
    import torch
    optics = synth.Optics(led_grid=grid)
    H = h * pratio
    if smooth_scale is None:
        obj = torch.from_numpy(np.ascontiguousarray(synth.make_object(H, seed).T)).to(dev)   # [c][r]
    else:
        obj = make_object_gpu(H, seed, dev, smooth_scale)
    circ = synth.pupil_circle(h, optics)
    ptrue = circ * np.exp(1j * synth.pupil_aberration(h, optics, seed))
    Pt = torch.from_numpy(np.ascontiguousarray(ptrue.T.astype(np.complex64))).to(dev)
    led = synth.led_indices(h, pratio, optics)
    ledt = torch.from_numpy(np.ascontiguousarray(led, np.int32)).to(dev)
    P0 = torch.from_numpy(np.ascontiguousarray(circ.T)).to(dev)
    return {"h": h, "pratio": pratio, "L": len(led), "object_true": obj, "pupil_true": Pt,
            "led": ledt, "led_np": led, "P0": P0, "P0c": P0.to(torch.complex64), "seed": seed}


def simulate_stack(eng: api.Engine, pb, rng_seed: int):
    """uint16 frames (Poisson at 3e4 peak counts) of a problem from the engine's simulator."""
    import torch
    h, p, L = pb["h"], pb["pratio"], pb["L"]
    I = torch.empty((L, h, h), dtype=torch.float32, device=pb["led"].device)   # [l][c][r]
    eng._check(eng.lib.fpm_simulate(eng._ctx, pb["object_true"].data_ptr(),
                                    pb["pupil_true"].data_ptr(), pb["led"].data_ptr(), h, p, L,
                                    api.SIM_INTENSITY, I.data_ptr(), api.MEM_DEVICE))
    g = torch.Generator(device=I.device)
    g.manual_seed(rng_seed)
    counts = torch.poisson(I * (3e4 / float(I.max())), generator=g).clamp_(max=65535)
    return counts.to(torch.int32).to(torch.uint16)


def problem_struct(pb, stack, epochs, batch, lr, object_init=None, P0c=None):
    P0c = pb["P0c"] if P0c is None else P0c
    return api.Problem(h=pb["h"], n_leds=pb["L"], pratio=pb["pratio"], batch=batch, epochs=epochs,
                       lr=lr, beta=0.999, eps=1e-4, pupil_margin=0.2, lr_halve_after=12,
                       lr_decay=0.5, loss_kind=0, memory=api.MEM_DEVICE, stack_type=api.STACK_U16,
                       stack=stack.data_ptr(), led_idx=pb["led"].data_ptr(),
                       pupil_init=P0c.data_ptr(), pupil_amp=pb["P0"].data_ptr(),
                       object_init=None if object_init is None else object_init.data_ptr())


def amplitudes(stack, count: int):
    """The first `count` frames as the solve normalises them (whole-stack min / max)."""
    import torch
    x = stack.to(torch.int32)
    mn, mx = int(x.min()), int(x.max())
    a = (x[:count].double() - mn) / max(mx - mn, 1)
    return a.to(torch.float32).to(torch.float64).sqrt().to(torch.float32)


def lowpass_target(O, h: int, pratio: int):
    """(2, h, h) real / imaginary planes of the centre h x h of O's spectrum at the low
    resolution, / pratio^2 (so that up-sampling restores O's scale), in O's memory layout."""
    import torch
    H = h * pratio
    F = torch.fft.fftshift(torch.fft.fft2(O.to(torch.complex128)))
    c = H // 2 - h // 2
    lo = torch.fft.ifft2(torch.fft.ifftshift(F[c:c + h, c:c + h])) / (pratio * pratio)
    return torch.stack([lo.real, lo.imag]).to(torch.float32)


def truth_error(O, T) -> float:
    """min over complex scalars a of ||a O - T|| / ||T|| (global phase and scale free)."""
    import torch
    O = O.reshape(-1).to(torch.complex128)
    T = T.reshape(-1).to(torch.complex128)
    a = torch.vdot(O, T) / torch.vdot(O, O)
    return float(torch.linalg.vector_norm(a * O - T) / torch.linalg.vector_norm(T))


def solve_objects(eng: api.Engine, pbs, stacks, epochs: int, batch: int, lr: float, inits=None):
    """Objects after `epochs` epochs of each problem (fpm_solve_batch, concurrent), with the
    bicubic plain start or the given starting objects; returns (objects, first-epoch loss)."""
    import torch
    n = len(pbs)
    probs = (api.Problem * n)()
    ress = (api.Result * n)()
    outs = []
    for i, (pb, st) in enumerate(zip(pbs, stacks)):
        H, h = pb["h"] * pb["pratio"], pb["h"]
        O = torch.empty((H, H), dtype=torch.complex64, device=st.device)
        P = torch.empty((h, h), dtype=torch.complex64, device=st.device)
        lo = torch.zeros(max(epochs, 1), dtype=torch.float64, device=st.device)
        probs[i] = problem_struct(pb, st, epochs, batch, lr, None if inits is None else inits[i])
        ress[i] = api.Result(object=O.data_ptr(), spectrum=None, pupil=P.data_ptr(),
                             loss=lo.data_ptr())
        outs.append((O, lo))
    stv = (C.c_int * n)()
    torch.cuda.synchronize()
    eng._check(eng.lib.fpm_solve_batch(eng._ctx, probs, ress, n, 0, stv))
    return [o for o, _ in outs], [float(l[0]) for _, l in outs]


def training_pairs(eng: api.Engine, n: int, h: int, pratio: int, grid: int, epochs: int,
                   batch: int, lr: float, seed0: int, in_channels: int = 25, chunk: int = 64,
                   smooth_scale=None):
    """(x, t): n inputs (the first in_channels amplitudes of each seeded problem) and targets
    (the low-pass of the plain method's object after `epochs` epochs), on the GPU."""
    import torch
    dev = torch.device("cuda", torch.cuda.current_device())
    xs, ts = [], []
    for c0 in range(0, n, chunk):
        pbs = [make_problem_gpu(h, pratio, grid, seed0 + i, dev, smooth_scale)
               for i in range(c0, min(n, c0 + chunk))]
        stacks = [simulate_stack(eng, pb, 7919 + pb["seed"]) for pb in pbs]
        objs, _ = solve_objects(eng, pbs, stacks, epochs, batch, lr)
        for pb, st, O in zip(pbs, stacks, objs):
            xs.append(amplitudes(st, in_channels))
            ts.append(lowpass_target(O, h, pratio))
        del pbs, stacks, objs
    return torch.stack(xs), torch.stack(ts)


def train(net: Network, x, t, epochs: int, batch_size: int, lr: float, seed: int = 0):
    """Mini-batch Adam over the pairs (a fresh seeded order every epoch); the mean training
    loss of every epoch."""
    import torch
    n = x.shape[0]
    g = torch.Generator()
    g.manual_seed(seed)
    hist = []
    for ep in range(epochs):
        order = torch.randperm(n, generator=g).to(x.device)
        tot, cnt = 0.0, 0
        for b0 in range(0, n - batch_size + 1, batch_size):
            idx = order[b0:b0 + batch_size]
            tot += net.train_step(x.index_select(0, idx), t.index_select(0, idx), lr)
            cnt += 1
        hist.append(tot / max(cnt, 1))
    return hist


def evaluate(eng: api.Engine, net: Network, pbs, stacks, epochs: int, batch: int, lr: float,
             refs=None):
    """Per-epoch error against the true object (global complex scale free) of the plain
    start and of the learned start (falling back to the plain start for a problem whose
    first-epoch loss the network's start raises), for every problem; k-epoch solves for
    k = 1..epochs, each from its start.  With refs (one object per problem, e.g. the plain
    method's converged result) the same distances to those are returned too:
    (plain, learned, fallback) or (plain, learned, fallback, plain_ref, learned_ref)."""
    import torch
    dev = stacks[0].device
    inits = [net.initial_object(problem_struct(pb, st, 1, batch, lr), dev)
             for pb, st in zip(pbs, stacks)]
    plain = np.zeros((len(pbs), epochs + 1))
    learned = np.zeros((len(pbs), epochs + 1))
    plain_r = np.zeros((len(pbs), epochs + 1))
    learned_r = np.zeros((len(pbs), epochs + 1))
    # epoch 0: the starts themselves; first-epoch losses for the fallback rule
    plain0, lp = solve_objects(eng, pbs, stacks, 1, batch, lr)
    _, ll = solve_objects(eng, pbs, stacks, 1, batch, lr, inits)
    fallback = [ll[i] > lp[i] for i in range(len(pbs))]
    starts0, _ = solve_objects(eng, pbs, stacks, 0, batch, lr)       # the bicubic start
    for i, pb in enumerate(pbs):
        T = pb["object_true"]
        plain[i, 0] = truth_error(starts0[i], T)
        learned[i, 0] = truth_error(starts0[i] if fallback[i] else inits[i], T)
        if refs is not None:
            plain_r[i, 0] = truth_error(starts0[i], refs[i])
            learned_r[i, 0] = truth_error(starts0[i] if fallback[i] else inits[i], refs[i])
    chosen = [starts0[i] if fallback[i] else inits[i] for i in range(len(pbs))]
    for k in range(1, epochs + 1):
        op, _ = solve_objects(eng, pbs, stacks, k, batch, lr)
        ol, _ = solve_objects(eng, pbs, stacks, k, batch, lr, chosen)
        for i, pb in enumerate(pbs):
            plain[i, k] = truth_error(op[i], pb["object_true"])
            learned[i, k] = truth_error(ol[i], pb["object_true"])
            if refs is not None:
                plain_r[i, k] = truth_error(op[i], refs[i])
                learned_r[i, k] = truth_error(ol[i], refs[i])
        del op, ol
    if refs is not None:
        return plain, learned, fallback, plain_r, learned_r
    return plain, learned, fallback


def _time_training_steps(h: int, n: int, steps: int, in_channels: int = 25, base: int = 32):
    """Milliseconds per Adam step of the network on seeded random (n, in_channels, h, h)
    inputs and (n, 2, h, h) targets, after one warm-up step."""
    import time
    import torch
    eng = api.Engine(0)
    net = Network(eng, in_channels, base, seed=1)
    g = torch.Generator(device="cuda")
    g.manual_seed(0)
    x = torch.rand((n, in_channels, h, h), device="cuda", generator=g)
    t = 0.1 * torch.randn((n, 2, h, h), device="cuda", generator=g)
    net.train_step(x, t, 1e-3)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        net.train_step(x, t, 1e-3)
    torch.cuda.synchronize()
    ms = (time.perf_counter() - t0) / steps * 1e3
    net.close()
    eng.close()
    return ms


if __name__ == "__main__":
    import argparse
    import json
    ap = argparse.ArgumentParser(description="time Adam steps of the warm-start network")
    ap.add_argument("--h", type=int, default=256)
    ap.add_argument("--n", type=int, default=32)
    ap.add_argument("--steps", type=int, default=3)
    a = ap.parse_args()
    print(json.dumps({"h": a.h, "batch": a.n, "ms_per_step": round(_time_training_steps(a.h, a.n, a.steps), 3)}))
