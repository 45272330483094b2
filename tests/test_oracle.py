"""CPU tests of the oracle: known-answer checks of every stage against direct
transcriptions of the reference's MATLAB statements, plus the golden fixture.

The reference ships no tests or fixtures; these pins are
* the MATLAB forward/backward of ``codes_v2/func_ware/fpm_forward_GPU.m:23-58``
  (with ``fft2_ware``/``ifft2_ware`` of ``codes/func_ware/misc`` and the
  anisotropic ``benchmark/func_ware/ret_loss.m``), written out literally below;
* the golden fixture ``tests/golden/tiny_fp64.npz`` (made by
  ``tests/golden/make_golden.py``);
* when present, outputs of the reference's own CUDA kernels run on a B200
  (``tests/golden/ref_*.npz``, made by ``make_golden.py --ref``).
"""
import math
from pathlib import Path

import numpy as np
import pytest

from oracle import fpm_oracle as orc
from fpm_b200 import synth

GOLDEN = Path(__file__).resolve().parent / "golden"


# ---------------------------------------------------------------------------
# literal transcription of the MATLAB path (1-based ranges -> 0-based slices)
# ---------------------------------------------------------------------------
def m_fft2_ware(x):          # codes/func_ware/misc/fft2_ware.m:3-4
    return np.fft.fftshift(np.fft.fftshift(np.fft.fft2(x, axes=(0, 1)), axes=0), axes=1)


def m_ifft2_ware(x):         # codes/func_ware/misc/ifft2_ware.m:3-4
    return np.fft.ifft2(np.fft.ifftshift(np.fft.ifftshift(x, axes=1), axes=0), axes=(0, 1))


def m_ret_loss(dW):          # benchmark/func_ware/ret_loss.m:3-21, 'anisotropic'
    RxdW = np.concatenate([dW[:, 1:] - dW[:, :-1], dW[:, :1] - dW[:, -1:]], axis=1)
    RydW = np.concatenate([dW[1:, :] - dW[:-1, :], dW[:1, :] - dW[-1:, :]], axis=0)
    loss = np.abs(RxdW) + np.abs(RydW)
    ox = np.sign(RxdW)
    oy = np.sign(RydW)
    out = np.concatenate([ox[:, -1:] - ox[:, :1], ox[:, :-1] - ox[:, 1:]], axis=1)
    out = out + np.concatenate([oy[-1:, :] - oy[:1, :], oy[:-1, :] - oy[1:, :]], axis=0)
    return loss.sum(), out


def m_forward_backward(O, P, Y, led, pratio):
    """fpm_forward_GPU.m:23-58 with deconv 'none'; led rows (kl, kt)."""
    h = P.shape[0]
    F = np.fft.fftshift(np.fft.fft2(O))
    subs = np.empty((h, h, len(led)), complex)
    for l, (kl, kt) in enumerate(led):
        subs[:, :, l] = F[kt - 1:kt - 1 + h, kl - 1:kl - 1 + h]          # :25-31
    x = m_ifft2_ware(subs * P[:, :, None]) / pratio ** 2                # :33
    loss = 0.0
    dm = np.empty(x.shape)
    for l in range(len(led)):                                           # :38
        lv, dm[:, :, l] = m_ret_loss(np.abs(x[:, :, l]) - Y[l])
        loss += lv
    xs = np.where(np.abs(x) > 0, x / np.where(np.abs(x) > 0, np.abs(x), 1), 0)
    x = dm * xs * pratio ** 2                                           # :41
    x_record = m_fft2_ware(x)                                           # :45
    xx = np.conj(P)[:, :, None] * x_record                              # :46
    D = np.zeros(O.shape, complex)
    for l, (kl, kt) in enumerate(led):                                  # :48-54
        D[kt - 1:kt - 1 + h, kl - 1:kl - 1 + h] += xx[:, :, l]
    dldw1 = m_ifft2_ware(D)                                             # :57
    dldw2 = (np.conj(subs) * x_record).sum(axis=2)                      # :58
    return loss, dldw1, dldw2


# ---------------------------------------------------------------------------
def test_shift_half_is_fftshift():
    a = np.random.default_rng(0).random((8, 6))
    np.testing.assert_array_equal(orc.shift_half(a), np.fft.fftshift(a))
    np.testing.assert_array_equal(orc.shift_half(orc.shift_half(a)), a)


def test_crop_indices_are_centred_slice_and_wrap():
    H, h = 32, 8
    S = np.random.default_rng(1).random((H, H)) + 1j
    C = np.fft.fftshift(S)
    kl, kt = 5, 11
    r, c = orc.crop_indices(kl, kt, h, H)
    np.testing.assert_array_equal(S[np.ix_(r, c)], C[kt - 1:kt - 1 + h, kl - 1:kl - 1 + h])
    # a crop running past the edge wraps modulo H (cuFPM_v3/cuda/kernels.cuh:45-46)
    r, c = orc.crop_indices(H - 2, H - 3, h, H)
    rows = [(H - 4 + i) % H for i in range(h)]
    cols = [(H - 3 + i) % H for i in range(h)]
    np.testing.assert_array_equal(S[np.ix_(r, c)], C[np.ix_(rows, cols)])


def test_feature_grad_matches_ret_loss():
    rng = np.random.default_rng(2)
    res = rng.standard_normal((16, 24))
    d, loss = orc.feature_grad(res, 4, np.float64)
    lm, outm = m_ret_loss(res)
    np.testing.assert_allclose(loss, lm, rtol=1e-13)
    np.testing.assert_array_equal(d, outm * 16)


def m_ret_loss_isotropic(dW):  # codes/func_ware/misc/ret_loss.m:3-11,18-21, 'isotropic'
    RxdW = np.concatenate([dW[:, 1:] - dW[:, :-1], dW[:, :1] - dW[:, -1:]], axis=1)
    RydW = np.concatenate([dW[1:, :] - dW[:-1, :], dW[:1, :] - dW[-1:, :]], axis=0)
    den = np.sqrt(RxdW ** 2 + RydW ** 2) + 1e-5
    loss = np.sqrt(RxdW ** 2 + RydW ** 2)
    ox = RxdW / den
    oy = RydW / den
    out = np.concatenate([ox[:, -1:] - ox[:, :1], ox[:, :-1] - ox[:, 1:]], axis=1)
    out = out + np.concatenate([oy[-1:, :] - oy[:1, :], oy[:-1, :] - oy[1:, :]], axis=0)
    return loss.sum(), out


def test_feature_grad_isotropic_matches_ret_loss():
    rng = np.random.default_rng(12)
    res = rng.standard_normal((16, 24))
    d, loss = orc.feature_grad(res, 4, np.float64, "isotropic")
    lm, outm = m_ret_loss_isotropic(res)
    np.testing.assert_allclose(loss, lm, rtol=1e-13)
    np.testing.assert_allclose(d, outm * 16, rtol=1e-12, atol=1e-12)
    # the FP32 twin tracks it to single-precision rounding
    d32, l32 = orc.feature_grad(res.astype(np.float32), 4, np.float32, "isotropic")
    np.testing.assert_allclose(d32, outm * 16, rtol=1e-4, atol=1e-5)


def test_feature_grad_sign_of_zero_is_plus_one():
    # v3 uses copysignf(1, x) (kernels.cuh:11-15): equal neighbours give +1, MATLAB gives 0
    res = np.zeros((4, 4))
    d, loss = orc.feature_grad(res, 1, np.float64)
    assert loss == 0.0
    np.testing.assert_array_equal(d, np.zeros((4, 4)))      # (+1 - +1) + (+1 - +1)
    res = np.zeros((4, 4))
    res[1, 1] = 1.0
    d, _ = orc.feature_grad(res, 1, np.float64)
    # at (1,2): ox(c-1) = sign(0 - 1) = -1, ox(c) = +1 (tie), oy(r-1) = +1, oy(r) = +1 -> -2
    assert d[1, 2] == -2.0
    # at (1,1): ox(c-1) = +1, ox(c) = sign(0-1) = -1, oy(r-1) = +1, oy(r) = -1 -> 4
    assert d[1, 1] == 4.0


def test_phase_times_zero_magnitude():
    z = np.array([[0 + 0j, 3 + 4j]])
    d = np.array([[2.0, 5.0]])
    out = orc.phase_times(z, d, np.float64)
    np.testing.assert_allclose(out, [[0, 3 + 4j]])


def test_batch_gradients_match_matlab_statement(ds_small):
    ds = ds_small
    p = ds.pratio
    H = ds.h * p
    rng = np.random.default_rng(5)
    O = ds.O0.astype(np.complex128) * np.exp(1j * 0.1 * rng.standard_normal((H, H)))
    P = ds.pupil_true.astype(np.complex128)
    led = ds.led_idx[:9]
    Y = ds.Y[:9].astype(np.float64)
    S = np.fft.fft2(O)
    G, dP, loss = orc.batch_gradients(S, P, Y, led, p, np.float64)
    g = np.fft.ifft2(G) * H * H
    lm, d1, d2 = m_forward_backward(O, P, Y, led, p)
    assert abs(loss - lm) <= 1e-10 * abs(lm)
    assert orc.rel_err(g, d1) < 1e-11
    assert orc.rel_err(dP, d2) < 1e-11


def test_rmsprop_and_clamp_known_values():
    w = np.array([1 + 1j], np.complex128)
    g = np.array([3 + 4j], np.complex128)
    m = np.array([0.5])
    wn, mu = orc.rmsprop_step(w, g, m, 0.1, 0.9, 1e-4, np.float64)
    mu_ref = 0.9 * 0.5 + 0.1 * 25.0
    assert mu[0] == pytest.approx(mu_ref)
    s = 0.1 / (math.sqrt(mu_ref) + 1e-4)
    assert wn[0] == pytest.approx((1 - 3 * s) + 1j * (1 - 4 * s))
    P = np.array([2 + 0j, 0.1j, 0.5 + 0j, 0j])
    P0 = np.array([1.0, 1.0, 1.0, 0.0])
    out = orc.pupil_clamp(P, P0, 0.2, np.float64)
    np.testing.assert_allclose(out, [1.2, 0.8j, 0.8, 0.0], atol=1e-15)


def test_fp32_twin_tracks_fp64_on_bright_field(ds_a):
    ds = ds_a
    L = 40   # first five rings of the spiral: no zero-count pixels, no sign ties
    kw = dict(pratio=4, epochs=2, batch=8, opt=(1e-3, 0.999, 1e-4))
    r64 = orc.cufpm_pure_v3(ds.O0, ds.P0c, ds.Y[:L], ds.led_idx[:L], ds.pupil0, dtype=np.float64, **kw)
    r32 = orc.cufpm_pure_v3(ds.O0, ds.P0c, ds.Y[:L], ds.led_idx[:L], ds.pupil0, dtype=np.float32, **kw)
    assert orc.rel_err(r32.object, r64.object) < 1e-5
    assert orc.rel_err(r32.pupil, r64.pupil) < 1e-5
    np.testing.assert_allclose(r32.loss, r64.loss, rtol=1e-5)


def test_spiral_order_visits_every_led_once():
    for n in (3, 5, 11, 19):
        o = synth.spiral_order(n)
        assert len(o) == n * n and len(set(o)) == n * n
        c = (n + 1) // 2
        assert o[0] == (c, c)
        assert o[1] == (c + 1, c)          # first turn: direction 1 (i + 1)
        assert all(abs(a[0] - b[0]) + abs(a[1] - b[1]) == 1 for a, b in zip(o, o[1:]))


def test_led_indices_centre_led():
    opt = synth.Optics(led_grid=11)
    led = synth.led_indices(128, 4, opt)
    H = 512
    # centre LED: u = v = 0 -> nearest frequency index NN/2 + 1 (1-based) -> kl = kt = H/2 + 1 - h/2
    assert tuple(led[0]) == (H // 2 + 1 - 64, H // 2 + 1 - 64)
    assert led.shape == (121, 2)
    assert led.min() >= 1 and (led + 127).max() <= H


def test_geometry_restatements_agree():
    """The oracle's statement-by-statement geometry against the generator's."""
    assert orc.spiral_grid_order(3) == [(2, 2), (3, 2), (3, 1), (2, 1), (1, 1), (1, 2), (1, 3),
                                        (2, 3), (3, 3)]
    for n in (5, 11, 19):
        assert orc.spiral_grid_order(n) == synth.spiral_order(n)
    for grid, h, p in ((5, 64, 2), (11, 128, 4), (19, 256, 8)):
        o = synth.Optics(led_grid=grid)
        led, order = orc.led_geometry(grid, h, p, o.wavelength_um, o.led_pitch_mm * 1000,
                                      o.led_height_mm * 1000, o.camera_pixel_um, o.magnification)
        np.testing.assert_array_equal(led, synth.led_indices(h, p, o))
        assert order.shape == (grid * grid, 2)


def test_geometry_off_axis_sample_area():
    """objdx / objdy shift every illumination angle: the centre LED's crop moves off centre."""
    o = synth.Optics(led_grid=5)
    args = (5, 128, 4, o.wavelength_um, o.led_pitch_mm * 1000, o.led_height_mm * 1000,
            o.camera_pixel_um, o.magnification)
    c, _ = orc.led_geometry(*args)
    s, _ = orc.led_geometry(*args, sample_dx_um=3000.0, sample_dy_um=-2000.0)
    assert tuple(c[0]) == (512 // 2 + 1 - 64, 512 // 2 + 1 - 64)
    assert s[0, 0] > c[0, 0] and s[0, 1] > c[0, 1]   # u <- +dx, v <- -(-dy) after the swap


def test_forward_model_matches_generator_statements():
    """The oracle's forward model against the data generator's (gen_img_batch.m:194-200)
    and a literal slice transcription for crops inside the spectrum."""
    rng = np.random.default_rng(3)
    h, p = 16, 4
    H = h * p
    O = rng.standard_normal((H, H)) + 1j * rng.standard_normal((H, H))
    P = synth.pupil_circle(h, synth.Optics(led_grid=3)) * np.exp(0.2j * rng.standard_normal((h, h)))
    led = np.array([[20, 17], [1, 1], [H - 5, 30], [H, H]], np.int32)
    I = orc.forward_model(O, P, led, p)
    spec = np.fft.fftshift(np.fft.fft2(O)).astype(np.complex64)
    np.testing.assert_allclose(I, synth.forward_intensity(spec, P.astype(np.complex64), led, p),
                               rtol=1e-4, atol=1e-6 * I.max())
    F = np.fft.fftshift(np.fft.fft2(O))
    kl, kt = led[0]
    x = np.fft.ifft2(np.fft.ifftshift(F[kt - 1:kt - 1 + h, kl - 1:kl - 1 + h] * P)) / p ** 2
    np.testing.assert_allclose(I[0], np.abs(x) ** 2, rtol=1e-12)
    np.testing.assert_allclose(orc.forward_model(O, P, led, p, amplitude=True), np.sqrt(I),
                               rtol=1e-12)


def test_torch_forward_model_checker_matches_oracle():
    """The torch complex64 forward model that checks the device simulator at sizes the
    FP64 oracle cannot reach agrees with the oracle (crops inside and past the edge)."""
    import torch
    from conftest import torch_forward_model
    rng = np.random.default_rng(8)
    h, p = 64, 4
    H = h * p
    O = np.exp(1j * 0.3 * rng.standard_normal((H, H)))
    P = synth.pupil_circle(h, synth.Optics(led_grid=3)) * np.exp(0.2j * rng.standard_normal((h, h)))
    led = np.array([[90, 97], [1, 1], [H - 20, 30], [H, H]], np.int32)
    ref = orc.forward_model(O, P, led, p, amplitude=True)
    got = torch_forward_model(torch.from_numpy(O.astype(np.complex64)),
                              torch.from_numpy(P.astype(np.complex64)), led, p).numpy()
    for l in range(len(led)):
        assert orc.rel_err(got[l], ref[l]) < 2e-6, l


def test_bicubic_restatements_agree_and_keep_constants():
    rng = np.random.default_rng(7)
    img = rng.random((12, 12))
    a = orc.imresize_bicubic(img, 4)
    b = synth.upsample_bicubic(img, 4)
    np.testing.assert_allclose(a, b, rtol=0, atol=1e-14)
    np.testing.assert_allclose(orc.imresize_bicubic(np.full((6, 6), 0.7), 3), 0.7, atol=1e-14)


def test_normalise_restatements_agree():
    raw = np.random.default_rng(8).integers(100, 40000, size=(3, 16, 16)).astype(np.uint16)
    np.testing.assert_array_equal(orc.normalise_stack_u16(raw), synth.normalise_u16(raw))


def test_golden_tiny_fixture():
    f = GOLDEN / "tiny_fp64.npz"
    g = np.load(f)
    r = orc.cufpm_pure_v3(g["O0"], g["P0c"], g["Y"], g["led_idx"], g["P0"], int(g["pratio"]),
                          int(g["epochs"]), int(g["batch"]), opt=tuple(g["opt"]), dtype=np.float64,
                          workers=1)
    assert orc.rel_err(r.object, g["object"]) < 1e-12
    assert orc.rel_err(r.pupil, g["pupil"]) < 1e-12
    assert orc.rel_err(r.spectrum, g["spectrum"]) < 1e-12
    np.testing.assert_allclose(r.loss, g["loss"], rtol=1e-12)


@pytest.mark.parametrize("name", sorted(p.name for p in GOLDEN.glob("ref_gradients_*.npz")))
def test_oracle_matches_reference_kernels(name):
    """Pin: gradients of the reference's own CUDA kernels (run on a B200) vs the FP64 oracle."""
    g = np.load(GOLDEN / name)
    S = np.fft.fft2(g["O"].astype(np.complex128))
    G, dP, _ = orc.batch_gradients(S, g["P"].astype(np.complex128), g["Y"].astype(np.float64),
                                   g["led_idx"], int(g["pratio"]), np.float64, workers=1)
    H = S.shape[0]
    dO = np.fft.ifft2(G) * H * H
    assert orc.rel_err(g["ref_dO"], dO) < float(g["tol"])
    assert orc.rel_err(g["ref_dP"], dP) < float(g["tol"])


@pytest.mark.parametrize("name", sorted(p.name for p in GOLDEN.glob("ref_solve_*.npz")))
def test_oracle_tracks_reference_solver(name):
    """Pin: a short reference solve (own kernels + cuFFT on a B200) vs the FP64 oracle."""
    g = np.load(GOLDEN / name)
    r = orc.cufpm_pure_v3(g["O0"], g["P0c"], g["Y"], g["led_idx"], g["P0"], int(g["pratio"]),
                          int(g["epochs"]), int(g["batch"]), opt=tuple(g["opt"]), dtype=np.float64,
                          workers=1)
    assert orc.rel_err(g["ref_object"], r.object) < float(g["tol"])
    assert orc.rel_err(g["ref_pupil"], r.pupil) < float(g["tol"])


def test_deconv_pie_weights_match_the_matlab_statements():
    """deconv_pie (benchmark/func_ware/fpm_forward_GPU.m:64-76) as the oracle restates it."""
    g = np.random.default_rng(12)
    x = (g.standard_normal((3, 8, 8)) + 1j * g.standard_normal((3, 8, 8)))
    ker = (g.standard_normal((3, 8, 8)) + 1j * g.standard_normal((3, 8, 8)))
    for l in range(3):
        np.testing.assert_allclose(orc._deconv_pie(x[l], ker[l], "none", np.float64),
                                   np.conj(ker[l]) * x[l])
        np.testing.assert_allclose(orc._deconv_pie(x[l], ker[l], "ePIE", np.float64),
                                   np.conj(ker[l]) * x[l] / np.max(np.abs(ker[l]) ** 2))
        np.testing.assert_allclose(orc._deconv_pie(x[l], ker[l], "tPIE", np.float64),
                                   np.conj(ker[l]) * x[l] / (np.abs(ker[l]) ** 2 + 1e-5))


# ---------------------------------------------------------------------------
# the torch restatement (the checker at full size, on the GPU) pinned to the oracle
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("loss_kind", ["anisotropic", "isotropic"])
def test_torch_checker_gradients_match_oracle(ds_small, loss_kind):
    """oracle/torch_ref.batch_gradients in complex128 = the FP64 oracle (crops inside and
    past the spectrum edge, LEDs in uneven chunks)."""
    import torch
    from oracle import torch_ref as tr
    ds = ds_small
    H = ds.h * ds.pratio
    rng = np.random.default_rng(9)
    O = (ds.O0 * np.exp(1j * 0.2 * rng.standard_normal((H, H)))).astype(np.complex64)
    led = np.concatenate([ds.led_idx, np.array([[H - 20, 3], [H, H], [1, H - 40]], np.int32)])
    Y = np.concatenate([ds.Y, ds.Y[:3]])
    G, dP, l64 = orc.batch_gradients(np.fft.fft2(O.astype(np.complex128)),
                                     ds.pupil_true.astype(np.complex128), Y.astype(np.float64),
                                     led, ds.pratio, np.float64, loss_kind=loss_kind)
    Gt, dPt, lt = tr.batch_gradients(torch.fft.fft2(torch.from_numpy(O).to(torch.complex128)),
                                     torch.from_numpy(ds.pupil_true), torch.from_numpy(Y), led,
                                     ds.pratio, loss_kind, chunk=7)
    assert orc.rel_err(Gt.numpy(), G) < 1e-13
    assert orc.rel_err(dPt.numpy(), dP) < 1e-13
    assert abs(lt - l64) <= 1e-12 * abs(l64)


def test_torch_checker_solve_matches_oracle(ds_small):
    """oracle/torch_ref.cufpm_pure_v3: complex128 = the FP64 oracle over two epochs with a
    ragged last batch; complex64 stays as close to FP64 as the numpy FP32 twin does."""
    import torch
    from oracle import torch_ref as tr
    ds = ds_small
    opt = (1e-3, 0.999, 1e-4)
    args = (ds.O0, ds.P0c, ds.Y, ds.led_idx, ds.pupil0, ds.pratio, 2, 8)
    r64 = orc.cufpm_pure_v3(*args, opt=opt, workers=1)
    r32 = orc.cufpm_pure_v3(*args, opt=opt, workers=1, dtype=np.float32)
    targs = (torch.from_numpy(ds.O0), torch.from_numpy(ds.P0c), torch.from_numpy(ds.Y),
             ds.led_idx, torch.from_numpy(ds.pupil0), ds.pratio, 2, 8)
    seen = []
    t64 = tr.cufpm_pure_v3(*targs, opt=opt, on_epoch=lambda ep, O, P, l: seen.append(ep))
    t32 = tr.cufpm_pure_v3(*targs, opt=opt, ctype=torch.complex64)
    assert seen == [0, 1]
    for k in ("object", "pupil", "spectrum"):
        assert orc.rel_err(t64[k].numpy(), getattr(r64, k)) < 1e-13, k
        e_t = orc.rel_err(t32[k].numpy(), getattr(r64, k))
        e_n = orc.rel_err(getattr(r32, k), getattr(r64, k))
        assert e_t < max(1e-6, 3 * e_n), (k, e_t, e_n)
    np.testing.assert_allclose(t64["loss"], r64.loss, rtol=1e-12)


def test_torch_checker_normalise_is_bit_exact():
    import torch
    from oracle import torch_ref as tr
    raw = np.random.default_rng(8).integers(100, 60000, size=(4, 32, 32)).astype(np.uint16)
    np.testing.assert_array_equal(tr.normalise_u16(torch.from_numpy(raw)).numpy(),
                                  orc.normalise_stack_u16(raw))
