"""Torch restatement of the oracle, for sizes the numpy oracle cannot reach.

TEST INFRASTRUCTURE ONLY.  The checker of the full-size parity tests and of the
accuracy leg of ``bench.py`` (outside every timed region); the product
(``libfpm.so``) never calls it.

The same algorithm as ``fpm_oracle.batch_gradients`` and ``fpm_oracle.cufpm_pure_v3``
(the reference solver ``cuFPM_v3/cuFPM_pure_v3.cu:128-207`` and its kernels
``cuFPM_v3/cuda/kernels.cuh``; citations per stage there), written in torch so
that it runs on the GPU.  In ``torch.complex128`` it is the FP64 reference at the
bench's full size (a 16384² object in FP64 is 4 GiB: minutes in numpy, seconds on
a B200); in ``torch.complex64`` it is an FP32 twin whose FFTs are cuFFT's.  It is
pinned on the CPU against the numpy oracle (``tests/test_oracle.py``).

Array convention as the numpy oracle: images are tensors indexed ``[row, col]``
(MATLAB order), stacks ``(L, h, h)``, ``led`` an ``(L, 2)`` integer array of rows
``(kl, kt)`` (1-based corner of the LED's crop in the centred spectrum).  A
column-major device buffer of an n x n image is the transpose of such a tensor,
so ``buf.view(n, n).T`` hands engine buffers to these functions without a copy.
"""
from __future__ import annotations

import numpy as np
import torch


def real_dtype(ctype):
    return torch.float64 if ctype == torch.complex128 else torch.float32


def _crop_index(led, h: int, H: int, device):
    """Rows / columns of every LED's crop in the un-shifted spectrum (``kernels.cuh:43-47``)."""
    led = torch.as_tensor(np.asarray(led, np.int64), device=device)
    ar = torch.arange(h, device=device)
    rr = (led[:, 1:2] - 1 + ar[None, :] + H // 2) % H
    cc = (led[:, 0:1] - 1 + ar[None, :] + H // 2) % H
    return rr, cc


def _feature_grad(res, pratio: int, loss_kind: str):
    """Anisotropic (``kernels.cuh:234-263``) or isotropic (``ret_loss.m:7-11``) gradient of
    a stack of residuals (dims 1, 2 = rows, cols), periodic forward differences; returns
    ``(d, loss)`` with the loss summed in float64."""
    rx = torch.roll(res, -1, dims=2) - res
    ry = torch.roll(res, -1, dims=1) - res
    if loss_kind == "anisotropic":
        one = torch.ones((), dtype=res.dtype, device=res.device)
        ox = torch.copysign(one, rx)
        oy = torch.copysign(one, ry)
        loss = float(rx.abs().double().sum() + ry.abs().double().sum())
    elif loss_kind == "isotropic":
        n = torch.sqrt(rx * rx + ry * ry)
        den = n + 1e-5
        ox = rx / den
        oy = ry / den
        loss = float(n.double().sum())
    else:
        raise ValueError(loss_kind)
    d = ((torch.roll(ox, 1, dims=2) - ox) + (torch.roll(oy, 1, dims=1) - oy)) * float(pratio * pratio)
    return d, loss


def batch_gradients(S, P, Y_b, led_b, pratio: int, loss_kind: str = "anisotropic",
                    chunk: int = 8):
    """Gradients of one LED batch at the un-shifted object spectrum ``S``
    (``fpm_oracle.batch_gradients``): ``(G, dP, loss)``, ``G`` the un-shifted gradient
    spectrum already divided by ``H²``, ``dP`` the pupil gradient.  ``Y_b`` (nb, h, h)
    amplitudes (any real dtype; promoted to the working precision).  LEDs are processed
    ``chunk`` at a time to bound the memory of the per-LED fields."""
    ct = S.dtype
    rt = real_dtype(ct)
    H, h = S.shape[0], P.shape[0]
    dev = S.device
    P = P.to(ct)
    G = torch.zeros((H, H), dtype=ct, device=dev)
    Gr = torch.view_as_real(G)
    dP = torch.zeros((h, h), dtype=ct, device=dev)
    loss = 0.0
    led_b = np.asarray(led_b)
    ratio = float(h * h * pratio * pratio)
    for c0 in range(0, len(led_b), chunk):
        leds = led_b[c0:c0 + chunk]
        n = len(leds)
        rr, cc = _crop_index(leds, h, H, dev)
        sub = S[rr[:, :, None], cc[:, None, :]]                          # (n, h, h)
        lat = torch.roll(sub * P, shifts=(h // 2, h // 2), dims=(1, 2))  # K2
        z = torch.fft.ifft2(lat) * float(h * h)                           # K3, unnormalised
        del lat
        res = torch.abs(z) / ratio - torch.as_tensor(Y_b[c0:c0 + n], device=dev).to(rt)
        d, lv = _feature_grad(res, pratio, loss_kind)                     # K4
        loss += lv
        del res
        mag = torch.abs(z)
        rec = torch.where(mag > 0, z / torch.where(mag > 0, mag, 1.0) * d, 0)
        del z, mag, d
        X = torch.roll(torch.fft.fft2(rec), shifts=(h // 2, h // 2), dims=(1, 2))   # K5
        del rec
        w = torch.conj(P)[None] * X / float(H * H)                        # K7, object term
        Gr.index_put_((rr[:, :, None].expand(n, h, h), cc[:, None, :].expand(n, h, h)),
                      torch.view_as_real(w), accumulate=True)
        del w
        dP += (torch.conj(sub) * X).sum(0)                                # pupil term
        del sub, X
    return G, dP, loss


def rmsprop_(w, g, m, lr: float, beta: float, eps: float):
    """In place: ``m = beta m + (1-beta)|g|²``; ``w -= g lr/(sqrt(m)+eps)`` (``kernels.cuh:365-377``)."""
    mu = g.real * g.real + g.imag * g.imag
    m.mul_(beta).add_((1.0 - beta) * mu)
    del mu
    w.sub_(g * (lr / (torch.sqrt(m) + eps)))


def pupil_clamp(w, P0, am: float):
    """``|P| <- P0 clamp(|P|, P0 - am, P0 + am)``, phase kept (``kernels.cuh:396-402``)."""
    ang = torch.atan2(w.imag, w.real)
    a = torch.abs(w)
    a = P0 * torch.maximum(torch.minimum(a, P0 + am), P0 - am)
    return torch.complex(torch.cos(ang) * a, torch.sin(ang) * a)


def cufpm_pure_v3(O0, P0c, Y, led, P0, pratio: int, epochs: int, batch: int,
                  opt=(5e-4, 0.999, 1e-4), am: float = 0.2, lr_halve_after: int = 12,
                  ctype=torch.complex128, loss_kind: str = "anisotropic", chunk: int = 8,
                  on_epoch=None):
    """``[O, P] = cuFPM_pure_v3(O0, P0c, Y, ledIdx, P0, pratio, epochs, B, [lr beta eps])`` in
    torch (``fpm_oracle.cufpm_pure_v3``).  ``Y``: (L, h, h) tensor of amplitudes, or a
    callable ``Y(first, count)`` returning the pages of one batch.  Hyper-parameters are
    rounded to float32 first, as the mex does.  ``on_epoch(ep, O, P, loss)`` is called after
    every epoch.  Returns ``dict(object, pupil, spectrum, loss)`` with the centred spectrum."""
    rt = real_dtype(ctype)
    lr = float(np.float32(opt[0]))
    beta = float(np.float32(opt[1]))
    eps = float(np.float32(opt[2]))
    am = float(np.float32(am))
    O = O0.to(ctype).clone()
    P = P0c.to(ctype).clone()
    P0 = P0.to(rt)
    dev = O.device
    H, h = O.shape[0], P.shape[0]
    L = len(led)
    Y_of = Y if callable(Y) else (lambda a, n: Y[a:a + n])
    m1 = torch.zeros((H, H), dtype=rt, device=dev)
    m2 = torch.zeros((h, h), dtype=rt, device=dev)
    losses = np.zeros(epochs, np.float64)
    led = np.asarray(led)
    for ep in range(epochs):
        cur = 0
        while cur < L:                                   # cuFPM_pure_v3.cu:131-141
            nb = min(batch, L - cur)
            S = torch.fft.fft2(O)
            G, dP, lv = batch_gradients(S, P, Y_of(cur, nb), led[cur:cur + nb], pratio,
                                        loss_kind, chunk)
            del S
            losses[ep] += lv
            g = torch.fft.ifft2(G)                       # K8: the 1/H² is inside G already
            del G
            g.mul_(float(H * H))
            rmsprop_(O, g, m1, lr, beta, eps)            # K9
            del g
            rmsprop_(P, dP, m2, lr, beta, eps)
            P = pupil_clamp(P, P0, am)
            cur += batch
        if ep > lr_halve_after:                          # cuFPM_pure_v3.cu:204-206
            lr = float(np.float32(lr * 0.5))
        if on_epoch is not None:
            on_epoch(ep, O, P, losses[ep])
    spec = torch.fft.fftshift(torch.fft.fft2(O))
    return {"object": O, "pupil": P, "spectrum": spec, "loss": losses}


def normalise_u16(counts):
    """``Y = sqrt((I - min) / max(I - min))`` over the whole stack in single precision
    (``codes_v2/main_run_FPM.m:43-45``; ``fpm_oracle.normalise_stack_u16``): integer
    differences below 2^24 are exact in float32, then one correctly rounded division and
    one correctly rounded square root.  Both are formed in float64 and rounded once to
    float32, which gives the correctly rounded single-precision result (53 >= 2·24 + 2
    bits); torch's own float32 sqrt on the CPU is not correctly rounded."""
    x = counts.to(torch.int32)
    mn = int(x.min())
    mx = int(x.max()) - mn
    y = (x - mn).to(torch.float64)
    if mx > 0:
        y = (y / float(mx)).to(torch.float32).to(torch.float64)
    return torch.sqrt(y).to(torch.float32)


def rel_err(a, b) -> float:
    """``||a-b||₂ / ||b||₂`` in float64, no phase alignment."""
    a = a.to(torch.complex128) if a.is_complex() else a.double()
    b = b.to(torch.complex128) if b.is_complex() else b.double()
    nb = float(torch.linalg.vector_norm(b))
    return float(torch.linalg.vector_norm(a - b)) / (nb if nb > 0 else 1.0)


def page_normaliser(counts):
    """Amplitudes of a uint16 stack (L, h, h) page by page with the whole stack's
    (min, max), as :func:`normalise_u16`: a callable ``Y(first, n)`` for
    :func:`cufpm_pure_v3`, so that the float stack is never formed whole."""
    mn, mx = 1 << 30, -1
    for a in range(0, counts.shape[0], 16):       # int32 copies of a few pages at a time
        c = counts[a:a + 16].to(torch.int32)
        mn, mx = min(mn, int(c.min())), max(mx, int(c.max()))
    mx -= mn

    def pages(first: int, n: int):
        y = (counts[first:first + n].to(torch.int32) - mn).to(torch.float64)
        if mx > 0:
            y = (y / float(mx)).to(torch.float32).to(torch.float64)
        return torch.sqrt(y).to(torch.float32)
    return pages


def imresize_bicubic(img, scale: int, rows_per_chunk: int = 2048):
    """MATLAB ``imresize(img, scale, 'bicubic')`` up-scaling (``codes_v2/main_run_FPM.m:48``)
    in float64 on img's device, with the taps and weights of
    ``fpm_oracle.imresize_bicubic_weights``: rows first, then columns, output rows in
    chunks."""
    from oracle import fpm_oracle as orc
    dev = img.device
    img = img.to(torch.float64)
    ir, wr = orc.imresize_bicubic_weights(img.shape[0], scale)
    ic, wc = orc.imresize_bicubic_weights(img.shape[1], scale)
    ir, wr = torch.from_numpy(ir).to(dev), torch.from_numpy(wr).to(dev)
    ic, wc = torch.from_numpy(ic).to(dev), torch.from_numpy(wc).to(dev)
    t = (img[ir, :] * wr[:, :, None]).sum(dim=1)                 # (n_out_r, n_c)
    out = torch.empty((t.shape[0], ic.shape[0]), dtype=torch.float64, device=dev)
    for r0 in range(0, t.shape[0], rows_per_chunk):
        tc = t[r0:r0 + rows_per_chunk]
        out[r0:r0 + rows_per_chunk] = (tc[:, ic] * wc[None, :, :]).sum(dim=2)
    return out
