"""The allocation-free loss-gradient entry point, through the C ABI.

It is for callers that cannot allocate device memory themselves (a mex inside
MATLAB's GPU memory manager, a framework whose caching allocator owns the
device, an acquisition loop that must not stall on an allocation).  Its loss
must equal the one the existing entry point fpm_batch_gradients reports for
the same batch, on two calls in a row (the fixed scratch array is shared and
keeps the previous call's contents), and its gradient must match the oracle
everywhere except where a residual difference is a near-tie in FP64 (the only
place where two correct FP32 evaluations can take different signs).
This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import led_matlab, to_matlab_stack
from oracle import fpm_oracle as orc
import fpm_b200

pytestmark = pytest.mark.gpu

UNSUPPORTED = 2


def _entry():
    lib = fpm_b200.load_library()
    f = lib.fpm_feature_gradient_noalloc
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_int32, C.c_void_p,
                  C.c_void_p, C.c_void_p]
    f.restype = C.c_int
    return f


def _fields(O, P, led, h, H):
    """z of each LED (column-major pages), as the solver forms it before the loss stage."""
    S = np.fft.fft2(O.astype(np.complex128))
    zs = []
    for kl, kt in led:
        rr, cc = orc.crop_indices(int(kl), int(kt), h, H)
        lat = orc.shift_half(S[np.ix_(rr, cc)] * P)
        zs.append((np.fft.ifft2(lat) * h * h).astype(np.complex64))
    return np.stack(zs)                       # (n, h, h) [l, r, c]


def _run(f, z, Y, pratio):
    import torch
    n, h, _ = z.shape
    dz = torch.from_numpy(np.ascontiguousarray(z.transpose(0, 2, 1))).cuda()      # [l][c][r]
    dy = torch.from_numpy(np.ascontiguousarray(Y.transpose(0, 2, 1).astype(np.float32))).cuda()
    grad = torch.empty_like(dz)
    loss = torch.zeros(1, dtype=torch.float64, device="cuda")
    st = f(dz.data_ptr(), dy.data_ptr(), h, n, pratio, grad.data_ptr(), loss.data_ptr(), None)
    torch.cuda.synchronize()
    assert st == 0, st
    return grad.cpu().numpy().transpose(0, 2, 1), float(loss.item())


def _near_ties(z, Y, h, p, tau=1e-6):
    """Pixels whose gradient depends on a residual difference within tau of zero (FP64):
    the only places where two correct FP32 evaluations may take different signs.  The
    gradient at (r, c) uses the differences at (r, c), (r, c-1) along the columns and
    (r, c), (r-1, c) along the rows."""
    res = orc.residual(z.astype(np.complex128), Y.astype(np.float64), h, p, np.float64)
    rx = np.abs(np.roll(res, -1, axis=1) - res) < tau
    ry = np.abs(np.roll(res, -1, axis=0) - res) < tau
    return rx | np.roll(rx, 1, axis=1) | ry | np.roll(ry, 1, axis=0)


def _check_against_oracle(z, Y, grad, loss, h, p, loss_rtol=1e-6):
    """Gradient equal to the FP32 oracle's on the same fields (relative 2e-6 of the largest
    value) everywhere except at sign near-ties; loss equal to the FP64 loss to loss_rtol."""
    d_or, loss64 = [], 0.0
    for i in range(len(z)):
        d, _ = orc.feature_grad(orc.residual(z[i], Y[i], h, p, np.float32), p, np.float32)
        d_or.append(orc.phase_times(z[i], d, np.float32))
        _, l64 = orc.feature_grad(orc.residual(z[i].astype(np.complex128), Y[i].astype(np.float64),
                                               h, p, np.float64), p, np.float64)
        loss64 += l64
    d_or = np.stack(d_or)
    scale = np.abs(d_or).max()
    bad = np.abs(grad - d_or) > 2e-6 * scale
    ties = np.stack([_near_ties(z[i], Y[i], h, p) for i in range(len(z))])
    assert not (bad & ~ties).any(), int((bad & ~ties).sum())
    assert bad.mean() < 1e-4, bad.mean()
    assert abs(loss - loss64) <= loss_rtol * abs(loss64), (loss, loss64)


def test_noalloc_loss_gradient_matches_existing_entry_point(engine, ds_small):
    ds = ds_small
    f = _entry()
    h, p = ds.h, ds.pratio
    H = h * p
    rng = np.random.default_rng(21)
    O = (ds.O0 * np.exp(1j * 0.2 * rng.standard_normal((H, H)))).astype(np.complex64)
    P = ds.pupil_true
    first = None
    for sl in (slice(0, 9), slice(9, 25)):           # two calls in a row, different sizes
        led = ds.led_idx[sl]
        Y = ds.Y[sl]
        _, _, loss_ref = engine.batch_gradients(O, P, to_matlab_stack(Y), led_matlab(led),
                                                ds.pupil0, p)
        z = _fields(O, P, led, h, H)
        grad, loss = _run(f, z, Y, p)
        assert abs(loss - loss_ref) < 1e-5 * abs(loss_ref)
        _check_against_oracle(z, Y, grad, loss, h, p, loss_rtol=1e-5)
        if first is None:
            first = (z, Y, grad, loss)
    # the shared scratch keeps the last call's contents; repeating call 1 reproduces it exactly
    z, Y, grad, loss = first
    grad2, loss2 = _run(f, z, Y, p)
    np.testing.assert_array_equal(grad2, grad)
    assert loss2 == loss


@pytest.mark.parametrize("h,p,n", [(48, 3, 3), (80, 2, 2), (34, 5, 4)])
def test_noalloc_partial_tiles_and_other_pratios(h, p, n):
    """Sides that are not multiples of the 32 x 32 tile (the partial-tile guards and the
    periodic halo inside a partial tile) and up-sampling ratios other than the data sets',
    against the oracle; two calls in a row."""
    f = _entry()
    rng = np.random.default_rng(h * 10 + p)
    z = ((rng.standard_normal((n, h, h)) + 1j * rng.standard_normal((n, h, h)))
         * (0.5 * h * h * p * p)).astype(np.complex64)
    z[0, 0, 0] = 0                               # |z| = 0: gradient 0 there
    Y = rng.random((n, h, h)).astype(np.float32)
    for _ in range(2):
        grad, loss = _run(f, z, Y, p)
        _check_against_oracle(z, Y, grad, loss, h, p)
        assert grad[0, 0, 0] == 0


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    f = _entry()
    buf = torch.zeros(16, dtype=torch.float64, device="cuda")
    # 17 images of 2048^2 need 17 * 4096 tiles > FPM_NOALLOC_MAX_TILES: refused before any work
    st = f(buf.data_ptr(), buf.data_ptr(), 2048, 17, 8, buf.data_ptr(), buf.data_ptr(), None)
    assert st == UNSUPPORTED
    # sides beyond the stated maximum, including ones whose tile count overflows 32 bits
    for h in (8194, 1_482_882, 2_000_000_000):
        st = f(buf.data_ptr(), buf.data_ptr(), h, 1, 8, buf.data_ptr(), buf.data_ptr(), None)
        assert st == UNSUPPORTED, h
