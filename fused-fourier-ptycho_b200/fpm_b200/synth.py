"""Seeded synthetic FPM data sets and the optics set-up the reference runs in MATLAB.

The reference's real data set and its source image are not shipped, so every
workload here is generated from a seed:

* object: amplitude = Gaussian-smoothed (sigma 3 px) uniform noise rescaled to
  [0.5, 1]; phase = Gaussian-smoothed (sigma 4 px) normal noise rescaled to
  [-pi/2, pi/2] (periodic smoothing in the Fourier domain);
* optics: lambda 0.532 um, NA 0.1, 6.5 um camera pixel at 4x, LED pitch 4 mm at
  90 mm height, circular pupil (``codes_v2/func_ware/init_environment_rgb.m:1-40``),
  optionally with seeded Zernike defocus / astigmatism;
* LED k-space positions by the nearest-pixel search of
  ``init_environment_rgb.m:83-107`` and the spiral-from-centre order of
  ``init_environment_rgb.m:111-133``; crop corners ``kt = vo - M/2``,
  ``kl = uo - N/2`` (``codes_v2/main_run_FPM.m:23,53-55``);
* images ``|ifft2(ifftshift(crop·P))/pratio²|²`` (the forward model of
  ``benchmark/gen_img_batch.m:194-200``) scaled to a peak of 3e4 counts,
  Poisson noise, uint16;
* amplitudes ``sqrt((I-min)/(max-min))`` over the whole stack
  (``codes_v2/main_run_FPM.m:43-45``) and the initial object
  ``imresize(Y_1, pratio)`` bicubic with zero phase (``main_run_FPM.m:47-48``).

All images are numpy arrays indexed ``[row, col]`` (MATLAB order); stacks are
``(L, h, h)``.  ``led_idx`` is ``(L, 2)`` int32 rows ``(kl, kt)``.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass

import numpy as np

try:
    import scipy.fft as _fft

    def _kw():
        try:
            return {"workers": len(os.sched_getaffinity(0))}
        except Exception:  # pragma: no cover
            return {}
except Exception:  # pragma: no cover
    _fft = np.fft

    def _kw():
        return {}


@dataclass
class Optics:
    wavelength_um: float = 0.532
    na: float = 0.1
    camera_pixel_um: float = 6.5
    magnification: float = 4.0
    led_pitch_mm: float = 4.0
    led_height_mm: float = 90.0
    led_grid: int = 11

    @property
    def dx_um(self) -> float:
        return self.camera_pixel_um / self.magnification


def pupil_circle(h: int, optics: Optics) -> np.ndarray:
    """Circular coherent transfer function ``Fx²+Fy² <= kmax²`` (``init_environment_rgb.m:33-40``)."""
    f = (np.arange(h) - h // 2) / (h * optics.dx_um) * 2.0 * math.pi
    kmax = optics.na * 2.0 * math.pi / optics.wavelength_um
    fy, fx = np.meshgrid(f, f, indexing="ij")
    return ((fx * fx + fy * fy) <= kmax * kmax).astype(np.float32)


def pupil_aberration(h: int, optics: Optics, seed: int, rms_rad: float = 0.5) -> np.ndarray:
    """Seeded defocus + astigmatism phase over the pupil disc, scaled to ``rms_rad`` rms."""
    rng = np.random.default_rng(seed + 7919)
    f = (np.arange(h) - h // 2) / (h * optics.dx_um)
    fy, fx = np.meshgrid(f, f, indexing="ij")
    rad = optics.na / optics.wavelength_um
    rho = np.sqrt(fx * fx + fy * fy) / rad
    th = np.arctan2(fy, fx)
    inside = rho <= 1.0
    c = rng.normal(size=3)
    phi = c[0] * (2 * rho ** 2 - 1) + c[1] * rho ** 2 * np.cos(2 * th) + c[2] * rho ** 2 * np.sin(2 * th)
    phi = np.where(inside, phi, 0.0)
    v = phi[inside]
    v = v - v.mean()
    scale = rms_rad / max(float(np.sqrt((v * v).mean())), 1e-12)
    return np.where(inside, (phi - phi[inside].mean()) * scale, 0.0)


def spiral_order(n: int):
    """1-based (i, j) visiting order of an n x n LED grid, spiralling out from the centre.

    Restates ``init_environment_rgb.m:111-133``: at every step try to turn to
    the next direction (right, down, left, up) if that neighbour is unvisited,
    otherwise keep going.
    """
    steps = [(0, 1), (1, 0), (0, -1), (-1, 0)]
    seen = np.zeros((n + 2, n + 2), bool)
    seen[0, :] = seen[-1, :] = seen[:, 0] = seen[:, -1] = True   # outside counts as visited
    i = j = (n + 1) // 2
    order = [(i, j)]
    seen[i, j] = True
    d = 0
    while len(order) < n * n:
        d2 = d + 1
        di, dj = steps[d2 % 4]
        if not seen[i + di, j + dj]:
            d = d2
        di, dj = steps[d % 4]
        i, j = i + di, j + dj
        order.append((i, j))
        seen[i, j] = True
    return order


def nearest_index(grid: np.ndarray, value: float) -> int:
    """1-based ``find(|grid - value| == min, 1)`` (first index on ties)."""
    d = np.abs(grid - value)
    return int(np.flatnonzero(d == d.min())[0]) + 1


def led_indices(h: int, pratio: int, optics: Optics) -> np.ndarray:
    """Crop corners ``(kl, kt)`` for every LED in spiral order, FP64.

    ``init_environment_rgb.m:83-107`` (angles, swap of u and v, nearest pixel
    on the high-res frequency grid) and ``main_run_FPM.m:23,53-55``.
    """
    n = optics.led_grid
    cen = (n - 1) / 2.0
    vled = np.arange(n) - cen
    hled = np.arange(n) - cen
    D = optics.led_pitch_mm * 1000.0
    h0 = optics.led_height_mm * 1000.0
    k0 = 2.0 * math.pi / optics.wavelength_um
    NN = h * pratio
    fgrid = (np.arange(NN) - NN / 2) / (h * optics.dx_um) * 2.0 * math.pi
    out = []
    for (i, j) in spiral_order(n):
        vv = vled[i - 1]
        hh = hled[j - 1]
        R = math.sqrt((-vv * D) ** 2 + (-hh * D) ** 2 + h0 ** 2)
        v_old = (-vv * D) / R
        u_old = -(-hh * D) / R
        u, v = v_old, u_old                                  # the swap at :193-195
        uo = nearest_index(fgrid, k0 * u)
        vo = nearest_index(fgrid, k0 * v)
        out.append((uo - h // 2, vo - h // 2))               # kl = kc(3)+uo, kt = kc(1)+vo
    return np.asarray(out, np.int32)


def _smooth_periodic(x: np.ndarray, sigma: float) -> np.ndarray:
    """Gaussian smoothing with periodic boundaries via the Fourier domain."""
    n0, n1 = x.shape
    f0 = np.fft.fftfreq(n0).astype(np.float32)
    f1 = np.fft.rfftfreq(n1).astype(np.float32)
    g0 = np.exp(-2.0 * (math.pi * sigma) ** 2 * f0 * f0).astype(np.float32)
    g1 = np.exp(-2.0 * (math.pi * sigma) ** 2 * f1 * f1).astype(np.float32)
    X = _fft.rfft2(x.astype(np.float32), **_kw())
    X *= g0[:, None]
    X *= g1[None, :]
    return _fft.irfft2(X, s=x.shape, **_kw()).astype(np.float32)


def _rescale(x: np.ndarray, lo: float, hi: float) -> np.ndarray:
    mn, mx = float(x.min()), float(x.max())
    return ((x - mn) / (mx - mn if mx > mn else 1.0) * (hi - lo) + lo).astype(np.float32)


def make_object(H: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    amp = _rescale(_smooth_periodic(rng.random((H, H), dtype=np.float32), 3.0), 0.5, 1.0)
    ph = _rescale(_smooth_periodic(rng.standard_normal((H, H), dtype=np.float32), 4.0),
                  -math.pi / 2, math.pi / 2)
    return (amp * np.exp(1j * ph)).astype(np.complex64)


def forward_intensity(spec_centred: np.ndarray, pupil: np.ndarray, led_idx: np.ndarray,
                      pratio: int) -> np.ndarray:
    """``|ifft2(ifftshift(crop·P))/pratio²|²`` per LED (``gen_img_batch.m:194-200``)."""
    h = pupil.shape[0]
    H = spec_centred.shape[0]
    L = led_idx.shape[0]
    out = np.empty((L, h, h), np.float32)
    for l in range(L):
        kl, kt = int(led_idx[l, 0]), int(led_idx[l, 1])
        r = (kt - 1 + np.arange(h)) % H
        c = (kl - 1 + np.arange(h)) % H
        sub = spec_centred[np.ix_(r, c)] * pupil
        x = _fft.ifft2(np.fft.ifftshift(sub), **_kw()) / (pratio * pratio)
        out[l] = (x.real * x.real + x.imag * x.imag).astype(np.float32)
    return out


@dataclass
class Dataset:
    h: int
    pratio: int
    raw: np.ndarray           # (L, h, h) uint16 counts
    Y: np.ndarray             # (L, h, h) float32 amplitude
    led_idx: np.ndarray       # (L, 2) int32 (kl, kt)
    pupil0: np.ndarray        # (h, h) float32 circle
    pupil_true: np.ndarray    # (h, h) complex64
    object_true: np.ndarray   # (H, H) complex64
    O0: np.ndarray            # (H, H) complex64 initial object
    P0c: np.ndarray           # (h, h) complex64 initial pupil


def normalise_u16(raw: np.ndarray) -> np.ndarray:
    """``sqrt((I - min)/max(I - min))`` over the whole stack in single precision."""
    x = raw.astype(np.float32)
    x = x - x.min()
    mx = x.max()
    if mx > 0:
        x = x / mx
    return np.sqrt(x).astype(np.float32)


def bicubic_weights(n_in: int, scale: int):
    """Taps and weights of MATLAB ``imresize`` bicubic up-scaling (a = -0.5, normalised, symmetric edges)."""
    n_out = n_in * scale
    u = np.arange(1, n_out + 1, dtype=np.float64)
    x = u / scale + 0.5 * (1.0 - 1.0 / scale)
    idx = np.floor(x - 2.0)[:, None] + np.arange(1, 5)[None, :]
    t = np.abs(x[:, None] - idx)
    a = -0.5
    w = np.where(t <= 1, (a + 2) * t ** 3 - (a + 3) * t ** 2 + 1,
                 np.where(t < 2, a * t ** 3 - 5 * a * t ** 2 + 8 * a * t - 4 * a, 0.0))
    w = w / w.sum(axis=1, keepdims=True)
    aux = np.concatenate([np.arange(n_in), np.arange(n_in - 1, -1, -1)])
    idx = aux[np.mod(idx.astype(np.int64) - 1, 2 * n_in)]
    return idx, w


def upsample_bicubic(img: np.ndarray, scale: int) -> np.ndarray:
    img = np.asarray(img, np.float64)
    ir, wr = bicubic_weights(img.shape[0], scale)
    ic, wc = bicubic_weights(img.shape[1], scale)
    t = np.einsum("ok,okc->oc", wr, img[ir, :])
    return np.einsum("rok,rok->ro", t[:, ic], np.broadcast_to(wc, (t.shape[0],) + wc.shape))


def make_dataset(h: int, pratio: int, led_grid: int, seed: int = 0, aberration: bool = False,
                 peak_counts: float = 3e4, optics: Optics | None = None) -> Dataset:
    """Generate one seeded data set (see the module docstring for the model)."""
    if optics is None:
        optics = Optics(led_grid=led_grid)
    H = h * pratio
    obj = make_object(H, seed)
    circ = pupil_circle(h, optics)
    if aberration:
        ptrue = (circ * np.exp(1j * pupil_aberration(h, optics, seed))).astype(np.complex64)
    else:
        ptrue = circ.astype(np.complex64)
    led = led_indices(h, pratio, optics)
    spec = np.fft.fftshift(_fft.fft2(obj, **_kw())).astype(np.complex64)
    I = forward_intensity(spec, ptrue, led, pratio)
    del spec
    rng = np.random.default_rng(seed + 104729)
    lam = I * np.float32(peak_counts / float(I.max()))
    raw = np.minimum(rng.poisson(lam), 65535).astype(np.uint16)
    Y = normalise_u16(raw)
    O0 = upsample_bicubic(Y[0], pratio).astype(np.float32).astype(np.complex64)
    return Dataset(h=h, pratio=pratio, raw=raw, Y=Y, led_idx=led, pupil0=circ,
                   pupil_true=ptrue, object_true=obj, O0=O0, P0c=circ.astype(np.complex64))
