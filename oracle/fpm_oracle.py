"""CPU oracle for the cuFPM_pure_v3 reconstruction loop.

TEST INFRASTRUCTURE ONLY.  This module is the checker: only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline / reference arm may
import it.  The product (``libfpm.so``) never calls it and has no CPU path.

It restates, in numpy, the algorithm of the reference solver
``cuFPM_v3/cuFPM_pure_v3.cu:128-207`` and its kernels
``cuFPM_v3/cuda/kernels.cuh``.  The readable MATLAB statement of the same math is
``codes_v2/func_ware/fpm_forward_GPU.m:23-58`` with the loss of
``benchmark/func_ware/ret_loss.m:1-22``; where MATLAB and the v3 CUDA disagree the
v3 CUDA semantics are followed:

* ``sign(0) = +1`` (``copysignf``), ``kernels.cuh:11-15``;
* the phase factor is ``z/|z|`` and 0 where ``|z| = 0``, ``kernels.cuh:265-273``;
* crop indices wrap modulo H, ``kernels.cuh:43-47``;
* RMSprop keeps an exponential moving average and adds ``eps`` outside the
  square root, ``kernels.cuh:368-371``;
* the pupil amplitude clamp goes through atan2/cos/sin with ``am = 0.2``,
  ``kernels.cuh:396-402``, ``cuFPM_pure_v3.cu:198``;
* the learning rate halves after every epoch with index > 12,
  ``cuFPM_pure_v3.cu:204-206``.

Array convention: every image is a numpy array indexed ``A[row, col]`` exactly
like the MATLAB arrays the reference receives (MATLAB dim 1 = rows).  The
column-major memory the C ABI takes is ``np.asfortranarray(A)``.  ``led_idx`` is
``(L, 2)`` int32 rows ``(kl, kt)``: the 1-based column and row of the top-left
corner of LED ``l``'s crop in the *centred* H x H spectrum
(``codes_v2/main_run_FPM.m:53-55``), i.e. MATLAB's ``int32([kl; kt])``.

Two precisions are provided.  ``dtype=np.float64`` is the FP64 transcription
that the relative errors are quoted against.  ``dtype=np.float32`` is an FP32
twin that performs the elementwise arithmetic in single precision with the
same operation order as the CUDA kernels (FFTs by pocketfft in single
precision); it is what the CPU baseline times.

Parity pins: the reference ships no tests, fixtures or golden vectors.  The
oracle's stage functions are pinned by known-answer tests against direct
transcriptions of the MATLAB statements (``ret_loss.m``, ``fft2_ware.m``,
``ifft2_ware.m``, the stitch loop of ``fpm_forward_GPU.m:48-54``) in
``tests/test_oracle.py``.
"""
from __future__ import annotations

import os
from dataclasses import dataclass, field

import numpy as np

try:  # pocketfft with threads; numpy's own FFT is the fallback inside the oracle
    import scipy.fft as _sfft

    def _fft2(a, workers):
        return _sfft.fft2(a, workers=workers)

    def _ifft2(a, workers):
        return _sfft.ifft2(a, workers=workers)
except Exception:  # pragma: no cover
    def _fft2(a, workers):
        return np.fft.fft2(a)

    def _ifft2(a, workers):
        return np.fft.ifft2(a)


def default_workers() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:  # pragma: no cover
        return os.cpu_count() or 1


def sign_copysign(x):
    """``copysignf(1.0f, x)``: +1 for +0, -1 for -0 (``kernels.cuh:11-15``)."""
    return np.copysign(np.ones_like(x), x)


# ---------------------------------------------------------------------------
# stage functions (one per reference kernel)
# ---------------------------------------------------------------------------

def crop_indices(kl: int, kt: int, h: int, H: int):
    """Row / column indices into the *un-shifted* spectrum of LED ``(kl, kt)``.

    ``fused_getSubpupil_shifted``, ``kernels.cuh:43-47``: the centred-spectrum
    position ``kt-1+r`` (row) / ``kl-1+c`` (col) is mapped to the un-shifted FFT
    by adding ``H/2`` modulo ``H``.
    """
    r = (kt - 1 + np.arange(h) + H // 2) % H
    c = (kl - 1 + np.arange(h) + H // 2) % H
    return r, c


def shift_half(a):
    """Swap halves along both axes (fftshift == ifftshift for even sizes).

    ``kernels.cuh:62-63`` (store at ``(i + h/2) % h``) and ``:92-95`` (load at
    the same index).
    """
    return np.roll(np.roll(a, a.shape[0] // 2, axis=0), a.shape[1] // 2, axis=1)


def abs_c(z, dtype):
    """``sqrtf(re*re + im*im)`` in the working precision (``kernels.cuh:5-9``)."""
    re = z.real.astype(dtype, copy=False)
    im = z.imag.astype(dtype, copy=False)
    return np.sqrt(re * re + im * im)


def residual(z, Y_l, h: int, pratio: int, dtype):
    """``|z| / (h*h*pratio^2) - Y`` (``kernels.cuh:223,233``)."""
    ratio = dtype(h * h * pratio * pratio)
    return abs_c(z, dtype) / ratio - Y_l.astype(dtype, copy=False)


def feature_grad(res, pratio: int, dtype, loss: str = "anisotropic"):
    """Feature-domain gradient of the residual; ``loss="isotropic"`` selects
    :func:`feature_grad_isotropic`.

    Anisotropic: gradient of ``Σ|∂c res| + |∂r res|``.

    ``differenceKernel_acc``, ``kernels.cuh:234-263``; MATLAB statement in
    ``benchmark/func_ware/ret_loss.m:3-4,11-12,18-19`` with periodic forward
    differences along columns (``x``) and rows (``y``).
    Returns ``(d, loss)`` with ``d = (ox(c-1)-ox(c) + oy(r-1)-oy(r))·pratio²``
    and ``loss = Σ |Rx| + |Ry|`` (accumulated in float64).
    """
    if loss == "isotropic":
        return feature_grad_isotropic(res, pratio, dtype)
    rx = np.roll(res, -1, axis=1) - res          # res(:, c+1) - res(:, c)
    ry = np.roll(res, -1, axis=0) - res          # res(r+1, :) - res(r, :)
    ox = sign_copysign(rx)
    oy = sign_copysign(ry)
    d = ((np.roll(ox, 1, axis=1) - ox) + (np.roll(oy, 1, axis=0) - oy)) * dtype(pratio * pratio)
    loss = float(np.abs(rx.astype(np.float64)).sum() + np.abs(ry.astype(np.float64)).sum())
    return d.astype(dtype, copy=False), loss


def feature_grad_isotropic(res, pratio: int, dtype):
    """Isotropic feature-domain gradient of ``Σ sqrt(Rx² + Ry²)``.

    ``codes/func_ware/misc/ret_loss.m:7-11,18-19`` ('isotropic', the loss the
    benchmark's ``fpm_forward_GPU.m:38`` selects): ``den = sqrt(Rx² + Ry²) + 1e-5``,
    ``ox = Rx/den``, ``oy = Ry/den``, ``out = ox(c-1) - ox(c) + oy(r-1) - oy(r)``;
    the caller scales by ``pratio²`` as for the anisotropic loss (``:41``).  In the
    working precision, one rounding per operation in this order.
    """
    rx = np.roll(res, -1, axis=1) - res
    ry = np.roll(res, -1, axis=0) - res
    n = np.sqrt(rx * rx + ry * ry)
    den = n + dtype(1e-5)
    ox = rx / den
    oy = ry / den
    d = ((np.roll(ox, 1, axis=1) - ox) + (np.roll(oy, 1, axis=0) - oy)) * dtype(pratio * pratio)
    return d.astype(dtype, copy=False), float(n.astype(np.float64).sum())


def phase_times(z, d, dtype):
    """``d · z/|z|`` with 0 where ``|z| = 0`` (``kernels.cuh:265-273``)."""
    ctype = np.complex64 if dtype == np.float32 else np.complex128
    re = z.real.astype(dtype, copy=False)
    im = z.imag.astype(dtype, copy=False)
    mag = np.sqrt(re * re + im * im)
    nz = mag > 0
    inv = np.zeros_like(mag)
    inv[nz] = dtype(1.0) / mag[nz]
    out = np.empty(z.shape, ctype)
    out.real = np.where(nz, re * inv * d, 0)
    out.imag = np.where(nz, im * inv * d, 0)
    return out


def rmsprop_step(w, g, m, lr, beta, eps, dtype):
    """RMSprop with EMA second moment (``kernels.cuh:365-377``).

    ``mu = beta*m + (1-beta)|g|²``; ``w -= g * lr/(sqrt(mu)+eps)``.
    Returns ``(w_new, mu)``.
    """
    gr = g.real.astype(dtype, copy=False)
    gi = g.imag.astype(dtype, copy=False)
    b = dtype(beta)
    mu = gr * gr + gi * gi
    mu = b * m + (dtype(1.0) - b) * mu
    sq = dtype(lr) / (np.sqrt(mu) + dtype(eps))
    out = np.empty_like(w)
    out.real = w.real - gr * sq
    out.imag = w.imag - gi * sq
    return out, mu


def pupil_clamp(w, P0, am, dtype):
    """``|P| <- P0 · clamp(|P|, P0-am, P0+am)``, phase kept (``kernels.cuh:396-402``)."""
    re = w.real.astype(dtype, copy=False)
    im = w.imag.astype(dtype, copy=False)
    ang = np.arctan2(im, re)
    a = np.sqrt(re * re + im * im)
    p0 = P0.astype(dtype, copy=False)
    a = p0 * np.maximum(np.minimum(a, p0 + dtype(am)), p0 - dtype(am))
    out = np.empty_like(w)
    out.real = np.cos(ang) * a
    out.imag = np.sin(ang) * a
    return out


# ---------------------------------------------------------------------------
# one LED batch (cuFPM_pure_v3.cu:135-199)
# ---------------------------------------------------------------------------

def _deconv_pie(x, ker, pie: str, dtype):
    """``deconv_pie(in, ker, type)`` (benchmark/func_ware/fpm_forward_GPU.m:64-76) for
    'none', 'ePIE' and 'tPIE': ``conj(ker) .* in`` divided by 1, ``max(max(abs(ker).^2))`` or
    ``abs(ker).^2 + 1e-5``."""
    num = np.conj(ker) * x
    if pie == "none":
        return num
    k2 = (ker.real.astype(dtype) ** 2 + ker.imag.astype(dtype) ** 2).astype(dtype)
    if pie == "ePIE":
        return num / k2.max()
    if pie == "tPIE":
        return num / (k2 + dtype(1e-5))
    raise ValueError(pie)


def batch_gradients(S, P, Y_b, leds_b, pratio: int, dtype, workers: int = 1,
                    loss_kind: str = "anisotropic", pie: str = "none"):
    """Gradients of one LED batch at the current object spectrum ``S``.

    ``S`` is the *un-shifted* FFT2 of the object (``cuFPM_pure_v3.cu:135-140``).
    Returns ``(G, dP, loss)`` where ``G`` is the un-shifted gradient spectrum
    already divided by ``H²`` (``kernels.cuh:114-116``), ``dP`` the pupil
    gradient (``kernels.cuh:118-128``, no normalisation) and ``loss`` the
    feature-domain loss of the batch.  ``pie`` weighs the two terms as ``deconv_pie``
    of ``benchmark/func_ware/fpm_forward_GPU.m:64-76`` does ('ePIE': over max|ker|^2 of
    the whole kernel, 'tPIE': over |ker|^2 + 1e-5 per pixel; ker = P for the object term,
    the LED's crop for the pupil term).
    """
    ctype = np.complex64 if dtype == np.float32 else np.complex128
    H = S.shape[0]
    h = P.shape[0]
    G = np.zeros((H, H), ctype)
    dP = np.zeros((h, h), ctype)
    loss = 0.0
    inv_H2 = dtype(1.0) / dtype(H * H)
    for l in range(len(leds_b)):
        kl, kt = int(leds_b[l][0]), int(leds_b[l][1])
        rr, cc = crop_indices(kl, kt, h, H)
        sub = S[np.ix_(rr, cc)]
        # K2: latentZ[ifftshift] = sub·P  (kernels.cuh:49-64)
        lat = shift_half((sub * P).astype(ctype, copy=False))
        # K3: unnormalised inverse FFT (cuFPM_pure_v3.cu:151-156)
        z = (_ifft2(lat, workers) * ctype(h * h)).astype(ctype, copy=False)
        # K4: feature-domain loss gradient (kernels.cuh:197-275)
        res = residual(z, Y_b[l], h, pratio, dtype)
        d, lval = feature_grad(res, pratio, dtype, loss_kind)
        loss += lval
        rec = phase_times(z, d, dtype)
        # K5: unnormalised forward FFT (cuFPM_pure_v3.cu:164-169), read shifted
        X = shift_half(_fft2(rec, workers).astype(ctype, copy=False))
        # K7: G += conj(P)·X / H² at the crop; dP += conj(sub)·X (kernels.cuh:95-128)
        G[np.ix_(rr, cc)] += _deconv_pie(X, P, pie, dtype) * inv_H2
        dP += _deconv_pie(X, sub, pie, dtype)
    return G, dP, loss


# ---------------------------------------------------------------------------
# full solver (cuFPM_pure_v3.cu:44-228)
# ---------------------------------------------------------------------------

@dataclass
class OracleResult:
    object: np.ndarray
    pupil: np.ndarray
    spectrum: np.ndarray
    loss: np.ndarray
    m_object: np.ndarray = field(repr=False, default=None)
    m_pupil: np.ndarray = field(repr=False, default=None)


def cufpm_pure_v3(O0, P0c, Y, led_idx, P0, pratio: int, epochs: int, batch: int,
                  opt=(5e-4, 0.999, 1e-4), am: float = 0.2, lr_halve_after: int = 12,
                  dtype=np.float64, workers: int | None = None,
                  loss_kind: str = "anisotropic", pie: str = "none") -> OracleResult:
    """Oracle of ``[O, P] = cuFPM_pure_v3(O0, P0c, Y, ledIdx, P0, pratio, epochs, B, [lr beta eps])``.

    ``Y`` is ``(L, h, h)`` amplitude (page ``l`` = LED ``l``, the reference's
    ``h x h x L`` MATLAB array with the page axis moved first).  The
    hyper-parameters are rounded to float32 first, as the mex does
    (``cuFPM_pure_v3.cu:63-65``).  Returns the object, pupil, the centred
    spectrum ``fftshift(fft2(O))`` and the per-epoch loss.  ``loss_kind``
    "isotropic" swaps the v3 loss for :func:`feature_grad_isotropic`; ``pie`` weighs
    the gradient terms (:func:`batch_gradients`).
    """
    if workers is None:
        workers = default_workers()
    ctype = np.complex64 if dtype == np.float32 else np.complex128
    lr = float(np.float32(opt[0]))
    beta = float(np.float32(opt[1]))
    eps = float(np.float32(opt[2]))
    am = float(np.float32(am))
    O = np.array(O0, dtype=ctype, copy=True)
    P = np.array(P0c, dtype=ctype, copy=True)
    P0 = np.asarray(P0, dtype=dtype)
    Y = np.asarray(Y)
    L = Y.shape[0]
    H = O.shape[0]
    h = P.shape[0]
    m1 = np.zeros((H, H), dtype)
    m2 = np.zeros((h, h), dtype)
    losses = np.zeros(epochs, np.float64)
    for ep in range(epochs):
        cur = 0
        while cur < L:                       # cuFPM_pure_v3.cu:131-141
            nb = min(batch, L - cur)
            S = _fft2(O, workers).astype(ctype, copy=False)
            G, dP, lv = batch_gradients(S, P, Y[cur:cur + nb], led_idx[cur:cur + nb],
                                        pratio, dtype, workers, loss_kind, pie)
            losses[ep] += lv
            # K8: unnormalised inverse FFT of G (the 1/H² is already inside G)
            g = (_ifft2(G, workers) * ctype(H * H)).astype(ctype, copy=False)
            del G
            # K9: RMSprop on O and P, then the pupil clamp (kernels.cuh:364-410)
            O, m1 = rmsprop_step(O, g, m1, lr, beta, eps, dtype)
            del g
            Pn, m2 = rmsprop_step(P, dP, m2, lr, beta, eps, dtype)
            P = pupil_clamp(Pn, P0, am, dtype)
            cur += batch
        if ep > lr_halve_after:              # cuFPM_pure_v3.cu:204-206
            lr = float(np.float32(lr * 0.5))
    spec = np.fft.fftshift(_fft2(O, workers)).astype(ctype, copy=False)
    return OracleResult(O, P, spec, losses, m1, m2)


def rel_err(a, b) -> float:
    """``||a-b||₂ / ||b||₂`` on complex arrays, no phase alignment."""
    a = np.asarray(a, np.complex128)
    b = np.asarray(b, np.complex128)
    nb = np.linalg.norm(b.ravel())
    return float(np.linalg.norm((a - b).ravel()) / (nb if nb > 0 else 1.0))


# ---------------------------------------------------------------------------
# set-up helpers that the reference runs in MATLAB (restated for checking)
# ---------------------------------------------------------------------------

def normalise_stack_u16(I_u16):
    """``Y = sqrt((I - min) / max(I - min))`` over the whole stack, in single.

    ``codes_v2/main_run_FPM.m:43-45`` (MATLAB ``single`` arithmetic; the
    subtraction of integers below 2^24 is exact, then one correctly rounded
    division and one correctly rounded square root).
    """
    x = np.asarray(I_u16).astype(np.float32)
    x = x - x.min()
    mx = x.max()
    x = x / mx if mx > 0 else x
    return np.sqrt(x).astype(np.float32)


def normalise_stack_f32(x):
    """The same ``sqrt((x - min) / max(x - min))`` over a float stack, in single, with
    NaN left out of the min / max (MATLAB ``min`` / ``max`` omit NaN).  A constant
    stack gives zeros (no division), as ``normalise_stack_u16``."""
    x = np.asarray(x, np.float32)
    mn = np.float32(np.nanmin(x))
    d = x - mn
    mx = np.float32(np.nanmax(x)) - mn
    d = d / mx if mx > 0 else d
    return np.sqrt(d).astype(np.float32)


def read_frame(path, row0: int, col0: int, h: int):
    """One measured frame as ``codes_v2/main_run_FPM.m:37-40`` loads it:
    ``mean(single(imread(name, 'PixelRegion', {rows, cols})), 3)``, the h x h region
    whose top-left pixel is (row0, col0), 0-based.  Decoded by Pillow (an
    independent TIFF decoder standing in for MATLAB's imread); returns float32
    (h, h) in [row, col] order."""
    from PIL import Image
    with Image.open(path) as im:
        a = np.asarray(im)
    a = a[row0:row0 + h, col0:col0 + h]
    if a.shape[:2] != (h, h):
        raise ValueError("pixel region outside the image")
    a = a.astype(np.float32)
    if a.ndim == 3:
        # single-precision sum then one division, as MATLAB's mean of single
        s = np.zeros(a.shape[:2], np.float32)
        for k in range(a.shape[2]):
            s = s + a[:, :, k]
        a = s / np.float32(a.shape[2])
    return a


# ---------------------------------------------------------------------------
# the MATLAB optimiser classes of the script-level loop (single precision, one
# rounding per MATLAB operation, double scalars rounded to single first)
# ---------------------------------------------------------------------------

def abs32(z):
    """MATLAB ``abs`` of a complex single: hypot, correctly rounded (formed in double)."""
    z = np.asarray(z, np.complex64)
    re = z.real.astype(np.float64)
    im = z.imag.astype(np.float64)
    return np.sqrt(re * re + im * im).astype(np.float32)


def _split(z):
    z = np.asarray(z, np.complex64)
    return z.real.astype(np.float32), z.imag.astype(np.float32)


def _join(re, im):
    out = np.empty(re.shape, np.complex64)
    out.real = re
    out.imag = im
    return out


def _f(x):
    return np.float32(x)


def _div_root(g, sq):
    """g ./ (sqrt(sq) + 1e-5) with MATLAB's complex square root where sq < 0."""
    gr, gi = _split(g)
    sq = np.asarray(sq, np.float32)
    neg = sq < 0
    with np.errstate(invalid="ignore"):
        d = np.sqrt(np.where(neg, _f(0), sq)) + _f(1e-5)
    outr, outi = gr / d, gi / d
    if neg.any():
        dr = _f(1e-5)
        di = np.sqrt(-sq[neg])
        den = dr * dr + di * di
        outr[neg] = (gr[neg] * dr + gi[neg] * di) / den
        outi[neg] = (gi[neg] * dr - gr[neg] * di) / den
    return _join(outr, outi)


def rmsprop_class_step(p, g, r1, mum, centered, lr, g0=None, buffer=None):
    """``optimizer_RMSprop.step`` (codes_v2/func_ware/optimizers/optimizer_RMSprop.m:30-47),
    statement by statement as written: ``squave = r1 + (1 - r1) .* abs(grad).^2`` (no running
    average), centred ``g0 = r1 .* g0 + (1 - r1) .* grad; squave = squave - abs(g0).^2``,
    momentum ``buffer = mum .* buffer + grad ./ (sqrt(squave) + 1e-5); p = p - lr .* buffer``,
    else ``p - lr .* (grad ./ (sqrt(squave) + 1e-5))``.  Returns (p, g0, buffer)."""
    a = abs32(g)
    sq = _f(r1) + _f(1.0 - r1) * (a * a)
    if centered:
        g0r, g0i = _split(g0)
        gr, gi = _split(g)
        g0 = _join(_f(r1) * g0r + _f(1.0 - r1) * gr, _f(r1) * g0i + _f(1.0 - r1) * gi)
        b = abs32(g0)
        sq = sq - b * b
    u = _div_root(g, sq)
    pr, pi = _split(p)
    if mum > 0:
        br, bi = _split(buffer)
        ur, ui = _split(u)
        buffer = _join(_f(mum) * br + ur, _f(mum) * bi + ui)
        br, bi = _split(buffer)
        p = _join(pr - _f(lr) * br, pi - _f(lr) * bi)
    else:
        ur, ui = _split(u)
        p = _join(pr - _f(lr) * ur, pi - _f(lr) * ui)
    return p, g0, buffer


def _first_moment(mom1, g, r1):
    mr, mi = _split(mom1)
    gr, gi = _split(g)
    return _join(_f(r1) * mr + _f(1.0 - r1) * gr, _f(r1) * mi + _f(1.0 - r1) * gi)


def adam_class_step(p, g, mom1, mom2, r1, r2, lr, it):
    """``optimizer_adam.step`` (codes/func_ware/optimizers/optimizer_adam.m:25-38); ``bias``
    in double as MATLAB forms it from double scalars.  Returns (p, mom1, mom2)."""
    a = abs32(g)
    mom1 = _first_moment(mom1, g, r1)
    mom2 = _f(r2) * np.asarray(mom2, np.float32) + _f(1.0 - r2) * (a * a)
    bias = _f(np.sqrt(1.0 - r2 ** float(it)) / (1.0 - r1 ** float(it)))
    mr, mi = _split(mom1)
    d = np.sqrt(mom2) + _f(1e-5)
    pr, pi = _split(p)
    p = _join(pr - _f(lr) * ((bias * mr) / d), pi - _f(lr) * ((bias * mi) / d))
    return p, mom1, mom2


def yogi_class_step(p, g, mom1, mom2, r1, r2, lr):
    """``optimizer_yogi.step`` (codes_v2/func_ware/optimizers/optimizer_yogi.m:25-36); MATLAB
    ``sign`` (0 at 0).  Returns (p, mom1, mom2)."""
    a = abs32(g)
    g2 = a * a
    mom1 = _first_moment(mom1, g, r1)
    mom2 = np.asarray(mom2, np.float32)
    mom2 = mom2 - (_f(1.0 - r2) * np.sign(mom2 - g2).astype(np.float32)) * g2
    mr, mi = _split(mom1)
    d = np.sqrt(mom2) + _f(1e-5)
    pr, pi = _split(p)
    p = _join(pr - _f(lr) * (mr / d), pi - _f(lr) * (mi / d))
    return p, mom1, mom2


def sgd_step(p, g, lr):
    """``optimizer_sgd`` (codes/func_ware/optimizers/optimizer_sgd.m:17-22) as intended:
    ``p - lr .* grad`` (the class's statement names an undefined ``update``)."""
    pr, pi = _split(p)
    gr, gi = _split(g)
    return _join(pr - _f(lr) * gr, pi - _f(lr) * gi)


def clamp_pupil_script(p, amp, ac):
    """``max(min(abs(w2), Pupil0 + ac), Pupil0 - ac) .* sign(w2) .* Pupil0``
    (benchmark/cuFPM_recon_2025_circular.m:183-186); sign(z) = z ./ abs(z), 0 at 0."""
    amp = np.asarray(amp, np.float32)
    w = abs32(p)
    t = np.maximum(np.minimum(w, amp + _f(ac)), amp - _f(ac))
    pr, pi = _split(p)
    nz = w > 0
    with np.errstate(invalid="ignore", divide="ignore"):
        sr = np.where(nz, pr / w, _f(0))
        si = np.where(nz, pi / w, _f(0))
    return _join(np.where(nz, (t * sr) * amp, _f(0)), np.where(nz, (t * si) * amp, _f(0)))


def _cubic(x, a=-0.5):
    ax = np.abs(x)
    ax2 = ax * ax
    ax3 = ax2 * ax
    return np.where(ax <= 1, (a + 2) * ax3 - (a + 3) * ax2 + 1,
                    np.where(ax < 2, a * ax3 - 5 * a * ax2 + 8 * a * ax - 4 * a, 0.0))


def imresize_bicubic_weights(n_in: int, scale: int):
    """Tap indices and weights of MATLAB ``imresize(..., scale, 'bicubic')`` (up-scaling).

    Output pixel ``u`` (1-based) samples input ``x = u/scale + 0.5(1-1/scale)``
    with the a=-0.5 cubic, four taps, weights normalised to sum 1 and
    half-sample-symmetric edge handling (``codes_v2/main_run_FPM.m:48``).
    Returns 0-based ``(idx[n_out, 4], w[n_out, 4])``.
    """
    n_out = n_in * scale
    u = np.arange(1, n_out + 1, dtype=np.float64)
    x = u / scale + 0.5 * (1.0 - 1.0 / scale)
    left = np.floor(x - 2.0)
    idx = left[:, None] + np.arange(1, 5)[None, :]      # 1-based taps floor(x-2)+1 .. +4
    w = _cubic(x[:, None] - idx)
    w = w / w.sum(axis=1, keepdims=True)
    aux = np.concatenate([np.arange(1, n_in + 1), np.arange(n_in, 0, -1)])
    idx = aux[np.mod(idx.astype(np.int64) - 1, 2 * n_in)] - 1
    return idx.astype(np.int64), w


def imresize_bicubic(img, scale: int):
    """Separable bicubic up-scaling in float64 (rows first, then columns)."""
    img = np.asarray(img, np.float64)
    ir, wr = imresize_bicubic_weights(img.shape[0], scale)
    ic, wc = imresize_bicubic_weights(img.shape[1], scale)
    t = (img[ir, :] * wr[:, :, None]).sum(axis=1)            # (n_out_r, n_c)
    out = (t[:, ic] * wc[None, :, :]).sum(axis=2)            # (n_out_r, n_out_c)
    return out


# ---------------------------------------------------------------------------
# LED illumination geometry (restated for checking the device helper)
# ---------------------------------------------------------------------------

def spiral_grid_order(n: int):
    """1-based (i, j) grid positions in the centre-out visiting order.

    ``codes_v2/func_ware/init_environment_rgb.m:111-133``: start at the centre
    ((n+1)/2, (n+1)/2); at every step, if the cell one turn further
    (direction + 1, with (sin, cos)(pi/2 * direction) giving (di, dj)) is
    unvisited, take that direction; then step once in the current direction.
    ``n`` must be odd (the centre index is fractional otherwise).
    """
    import math
    seen = np.zeros((n + 1, n + 1), bool)          # 1-based
    i = j = (n + 1) // 2
    seen[i, j] = True
    order = [(i, j)]
    d = 0
    while len(order) < n * n:
        d2 = d + 1
        i2 = int(round(i + math.sin(math.pi / 2 * d2)))
        j2 = int(round(j + math.cos(math.pi / 2 * d2)))
        if not seen[i2, j2]:
            d = d2
        i = int(round(i + math.sin(math.pi / 2 * d)))
        j = int(round(j + math.cos(math.pi / 2 * d)))
        seen[i, j] = True
        order.append((i, j))
    return order


def led_geometry(grid: int, h: int, pratio: int, wavelength_um: float, led_pitch_um: float,
                 led_height_um: float, camera_pixel_um: float, magnification: float,
                 sample_dx_um: float = -0.0, sample_dy_um: float = -0.0):
    """ledIdx (L, 2) int32 rows (kl, kt) in spiral order, plus the (i, j) order.

    Python floats are IEEE doubles and are evaluated one operation at a time in
    MATLAB's left-to-right order (no fused multiply-add):

    * ``init_environment_rgb.m:15-21,31-46``: D_pixel = pixel_size / mag, the
      high-res frequency axis ``(k - NN/2) ./ (N * D_pixel) .* (2*pi)``;
    * ``:64-68,82-90``: per grid cell (i, j), ``a = -vled(i)*D_led + objdx``,
      ``b = -hled(j)*D_led + objdy``, ``den = sqrt(a^2 + b^2 + h^2)``,
      ``v = a/den``, ``u = -b/den``, then u and v swapped;
    * ``:98-106``: uo / vo = first index of the minimum of
      ``|F - k_lamuda * u|`` / ``|F - k_lamuda * v|`` (``find(x == min(x))``,
      first on ties), with ``k_lamuda = 2*pi/lamuda``;
    * ``main_run_FPM.m:21-31,51-55``: LEDs in spiral order,
      ``kl = uo - N/2``, ``kt = vo - M/2``.
    """
    import math
    NN = h * pratio
    D_pixel = camera_pixel_um / magnification
    ND = h * D_pixel
    two_pi = 2 * math.pi
    # elementwise IEEE double operations, one rounding each (numpy does not fuse them)
    F = ((np.arange(NN, dtype=np.int64) - NN // 2) / ND) * two_pi
    k_lamuda = two_pi / wavelength_um
    cen = (grid - 1) / 2

    def nearest(x):
        return int(np.argmin(np.abs(F - x))) + 1        # argmin: first index on ties

    order = spiral_grid_order(grid)
    out = []
    for (i, j) in order:
        vv = (i - 1) - cen
        hh = (j - 1) - cen
        a = (-vv) * led_pitch_um + sample_dx_um
        b = (-hh) * led_pitch_um + sample_dy_um
        den = math.sqrt(a * a + b * b + led_height_um * led_height_um)
        v0 = a / den
        u0 = (-b) / den
        u, v = v0, u0
        uo = nearest(k_lamuda * u)
        vo = nearest(k_lamuda * v)
        out.append((uo - h // 2, vo - h // 2))
    return np.asarray(out, np.int32), np.asarray(order, np.int32)


# ---------------------------------------------------------------------------
# forward model (restated for checking the device simulator)
# ---------------------------------------------------------------------------

def forward_model(O, P, led_idx, pratio: int, amplitude: bool = False, dtype=np.float64):
    """Images of every LED, (L, h, h) [l, r, c]: ``benchmark/gen_img_batch.m:178-201``.

    ``ft = fftshift(fft2(O))`` (:184 with the shift made explicit, as its caller
    passes the centred spectrum), the LED's h x h window with its 1-based
    top-left corner at (kt, kl) taken modulo H like the solver's crop
    (``cuFPM_v3/cuda/kernels.cuh:43-47``), times the pupil, ``x =
    ifft2(ifftshift(.)) / pratio^2`` (:197), and ``|x|^2`` (the intensity the
    data sets hold) or ``abs(x)`` (:199).
    """
    cdt = np.complex128 if dtype == np.float64 else np.complex64
    O = np.asarray(O, cdt)
    P = np.asarray(P, cdt)
    H = O.shape[0]
    h = P.shape[0]
    F = np.fft.fftshift(np.fft.fft2(O))
    out = np.empty((len(led_idx), h, h), dtype)
    ar = np.arange(h)
    for l, (kl, kt) in enumerate(np.asarray(led_idx)):
        sub = F[np.ix_((kt - 1 + ar) % H, (kl - 1 + ar) % H)] * P
        x = np.fft.ifft2(np.fft.ifftshift(sub)) / (pratio * pratio)
        a = np.abs(x)
        out[l] = a if amplitude else a * a
    return out
