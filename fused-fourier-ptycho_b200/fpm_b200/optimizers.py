"""The reference's MATLAB optimiser classes, stepping on the device.

The script-level loop of the reference (benchmark/cuFPM_recon_2025_circular.m:108-113,
180-186; codes/main_run_FPM.m:85-86) builds two optimisers and, per mini-batch,

    [dldw1, dldw2] = fullyfusedFPM(wavefront1, wavefront2, Y_batch, ledIdx, pratio);
    wavefront1 = optimizer_w1.step(wavefront1, dldw1);
    wavefront2 = optimizer_w2.step(wavefront2, dldw2);
    wavefront2 = max(min(abs(wavefront2), Pupil0 + ac), Pupil0 - ac) .* sign(wavefront2) .* Pupil0;

Here ``Engine.batch_gradients`` is fullyfusedFPM and these classes keep the MATLAB
constructors, the ``lr`` attribute the loop rescales, and ``step``; each step is one
fused elementwise pass of libfpm (``fpm_optimizer_step``), the clamp included when
``clamp=(Pupil0, ac)`` is given.  Parameters are complex64: numpy arrays (a new array
is returned, as MATLAB's value semantics) or torch tensors on the device (updated in
place and returned).  States start at zero like the classes' constructor arguments
(the reference always passes 0).
"""
from __future__ import annotations

import numpy as np

from .api import (OPT_ADAM, OPT_RMSPROP, OPT_SGD, OPT_YOGI, Optimizer, _engine, _is_torch)

__all__ = ["optimizer_RMSprop", "optimizer_adam", "optimizer_yogi", "optimizer_sgd"]


def _zeros_like(x, complex_: bool):
    if _is_torch(x):
        import torch
        return torch.zeros(x.shape, dtype=torch.complex64 if complex_ else torch.float32,
                           device=x.device)
    return np.zeros(x.shape, np.complex64 if complex_ else np.float32)


def _ptr(x):
    if x is None:
        return None
    return x.data_ptr() if _is_torch(x) else x.ctypes.data


def _same_layout(x, like, dtype):
    """x as a contiguous array / tensor with like's element order."""
    if _is_torch(like):
        import torch
        tdt = {np.complex64: torch.complex64, np.float32: torch.float32}[dtype]
        t = x if _is_torch(x) else torch.as_tensor(np.asarray(x), device=like.device)
        t = t.to(device=like.device, dtype=tdt)
        if t.shape != like.shape:
            raise ValueError(f"shape {tuple(t.shape)} != {tuple(like.shape)}")
        return t.contiguous()
    a = np.asarray(x, dtype)
    if a.shape != like.shape:
        raise ValueError(f"shape {a.shape} != {like.shape}")
    return np.ascontiguousarray(a)


class _Base:
    def __init__(self, lr, engine=None):
        self.lr = lr
        self._engine = engine

    def _prepare(self, para_in, grad):
        if _is_torch(para_in):
            p = para_in.contiguous()
        else:
            p = np.array(para_in, np.complex64, order="C", copy=True)
        g = _same_layout(grad, p, np.complex64)
        return p, g

    def _run(self, p, g, opt: Optimizer, clamp):
        keep = None
        if clamp is not None:
            amp, margin = clamp
            keep = _same_layout(amp, p.real, np.float32)
            opt.clamp_amp = _ptr(keep)
            opt.clamp_margin = float(margin)
        (self._engine or _engine()).optimizer_step(opt, p, g)
        del keep
        return p


class optimizer_sgd(_Base):
    """optimizer_sgd.m: p - lr * grad (the class's own step names an undefined variable)."""

    def __init__(self, lr, engine=None):
        super().__init__(lr, engine)

    def step(self, para_in, grad, clamp=None):
        p, g = self._prepare(para_in, grad)
        return self._run(p, g, Optimizer(kind=OPT_SGD, lr=float(self.lr)), clamp)


class optimizer_RMSprop(_Base):
    """optimizer_RMSprop.m (codes_v2/func_ware/optimizers): constructor
    (squave, buffer, beta1, mum, centered, lr); step(para_in, grad)."""

    def __init__(self, squave=0, buffer=0, beta1=0.9, mum=1, centered=True, lr=1e-2,
                 engine=None):
        super().__init__(lr, engine)
        self.r1 = beta1
        self.mum = mum
        self.centered = bool(centered)
        # squave is recomputed from r1 at every step (optimizer_RMSprop.m:33), so its
        # initial value never matters; buffer and g0 start at zero
        self.buffer = None if np.isscalar(buffer) and buffer == 0 else buffer
        self.g0 = None

    def step(self, para_in, grad, clamp=None):
        p, g = self._prepare(para_in, grad)
        if self.centered and self.g0 is None:
            self.g0 = _zeros_like(p, True)
        if self.mum > 0:
            self.buffer = (_zeros_like(p, True) if self.buffer is None
                           else _same_layout(self.buffer, p, np.complex64))
        opt = Optimizer(kind=OPT_RMSPROP, centered=int(self.centered), lr=float(self.lr),
                        beta1=float(self.r1), momentum=float(self.mum),
                        mom1=_ptr(self.g0) if self.centered else None,
                        buffer=_ptr(self.buffer) if self.mum > 0 else None)
        return self._run(p, g, opt, clamp)


class optimizer_adam(_Base):
    """optimizer_adam.m (codes/func_ware/optimizers): constructor (mom1, mom2, beta1,
    beta2, lr); step(para_in, grad, iter)."""

    def __init__(self, mom1=0, mom2=0, beta1=0.9, beta2=0.999, lr=1e-2, engine=None):
        super().__init__(lr, engine)
        self.r1, self.r2 = beta1, beta2
        self.mom1 = None if np.isscalar(mom1) and mom1 == 0 else mom1
        self.mom2 = None if np.isscalar(mom2) and mom2 == 0 else mom2

    def _moments(self, p):
        self.mom1 = (_zeros_like(p, True) if self.mom1 is None
                     else _same_layout(self.mom1, p, np.complex64))
        self.mom2 = (_zeros_like(p, False) if self.mom2 is None
                     else _same_layout(self.mom2, p.real, np.float32))

    def step(self, para_in, grad, iter=1, clamp=None):
        p, g = self._prepare(para_in, grad)
        self._moments(p)
        opt = Optimizer(kind=OPT_ADAM, lr=float(self.lr), beta1=float(self.r1),
                        beta2=float(self.r2), iter=int(iter), mom1=_ptr(self.mom1),
                        mom2=_ptr(self.mom2))
        return self._run(p, g, opt, clamp)


class optimizer_yogi(optimizer_adam):
    """optimizer_yogi.m (codes_v2/func_ware/optimizers): constructor (mom1, mom2, beta1,
    beta2, lr); step(para_in, grad)."""

    def step(self, para_in, grad, clamp=None):
        p, g = self._prepare(para_in, grad)
        self._moments(p)
        opt = Optimizer(kind=OPT_YOGI, lr=float(self.lr), beta1=float(self.r1),
                        beta2=float(self.r2), mom1=_ptr(self.mom1), mom2=_ptr(self.mom2))
        return self._run(p, g, opt, clamp)
