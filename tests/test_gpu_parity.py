"""GPU parity of the CUDA path (through the C ABI) against the CPU oracle.

Tolerances (relative L2 error, complex, no phase alignment):
* one gradient evaluation, one update, or a few epochs on noiseless
  amplitudes: 2e-5 against FP64, or 3x the FP32 oracle twin's own distance
  to FP64 when that is larger;
* long runs on noisy data: the sign() of the feature-domain loss flips on
  near-tied residual differences, a chaotic process, so every FP32
  implementation (the reference's, the FP32 oracle twin, this engine) drifts
  from FP64 by ~1e-2 after a few epochs of the 128² case.  There the engine must
  stay within max(5x the twin's drift, 3e-2), match the loss curve to 5e-3,
  and reconstruct the true object as well as FP64 does (within 2%);
* integer-exact paths (uint16 ingest, host vs device memory): bit-identical.
"""
import numpy as np
import pytest

from conftest import led_matlab, to_matlab_stack, dataset, torch_forward_model
from oracle import fpm_oracle as orc
import fpm_b200

pytestmark = pytest.mark.gpu

TIGHT = 2e-5


def _solve(engine, ds, L, epochs, batch, opt, raw=False, O0=None):
    Y = ds.raw[:L] if raw else ds.Y[:L]
    return engine.solve(ds.O0 if O0 is None else O0, ds.P0c, to_matlab_stack(Y),
                        led_matlab(ds.led_idx[:L]), ds.pupil0, ds.pratio, epochs, batch,
                        lr=opt[0], beta=opt[1], eps=opt[2])


def test_batch_gradients_vs_oracle(engine, ds_small):
    """The fullyfusedFPM contract, LED by LED and as one batch.

    A residual difference within one FP32 ulp of zero can take the other sign in
    any FP32 implementation (the engine's FFT rounds differently from numpy's),
    which moves that LED's gradient by ~1e-3.  So: every LED's loss must match,
    all but at most two LEDs' gradients must match tightly, none may move more
    than a flip would.
    """
    ds = ds_small
    H = ds.h * ds.pratio
    rng = np.random.default_rng(9)
    O = (ds.O0 * np.exp(1j * 0.2 * rng.standard_normal((H, H)))).astype(np.complex64)
    P = ds.pupil_true
    S64 = np.fft.fft2(O.astype(np.complex128))
    S32 = np.fft.fft2(O)
    errs = []
    for l in range(len(ds.led_idx)):
        sel = slice(l, l + 1)
        dO, dP, loss = engine.batch_gradients(O, P, to_matlab_stack(ds.Y[sel]),
                                              led_matlab(ds.led_idx[sel]), ds.pupil0, ds.pratio)
        G, dP64, l64 = orc.batch_gradients(S64, P.astype(np.complex128),
                                           ds.Y[sel].astype(np.float64), ds.led_idx[sel],
                                           ds.pratio, np.float64)
        G32, dP32, _ = orc.batch_gradients(S32, P, ds.Y[sel], ds.led_idx[sel], ds.pratio,
                                           np.float32)
        dO64 = np.fft.ifft2(G) * H * H
        e32 = orc.rel_err(np.fft.ifft2(G32) * H * H, dO64)
        e = max(orc.rel_err(dO, dO64), orc.rel_err(dP, dP64))
        errs.append(e / max(TIGHT, 3 * e32))
        assert abs(loss - l64) < 1e-5 * abs(l64), l
    errs = np.sort(np.array(errs))
    assert errs[-3] < 1.0, errs[-5:]             # all but two LEDs tight
    assert errs[-1] * TIGHT < 2e-2, errs[-5:]     # the rest within a sign flip
    # one batch of all LEDs: the loss is continuous in the inputs, the gradient within flips
    dO, dP, loss = engine.batch_gradients(O, P, to_matlab_stack(ds.Y), led_matlab(ds.led_idx),
                                          ds.pupil0, ds.pratio)
    G, dP64, l64 = orc.batch_gradients(S64, P.astype(np.complex128), ds.Y.astype(np.float64),
                                       ds.led_idx, ds.pratio, np.float64)
    assert abs(loss - l64) < 1e-5 * abs(l64)
    assert orc.rel_err(dO, np.fft.ifft2(G) * H * H) < 1e-2
    assert orc.rel_err(dP, dP64) < 1e-2


def _noiseless(ds):
    """Amplitudes of the forward model without Poisson noise (no zero counts, no ties)."""
    from fpm_b200 import synth
    spec = np.fft.fftshift(np.fft.fft2(ds.object_true)).astype(np.complex64)
    I = synth.forward_intensity(spec, ds.pupil_true, ds.led_idx, ds.pratio)
    Y = np.sqrt(I / I.max()).astype(np.float32)
    O0 = synth.upsample_bicubic(Y[0], ds.pratio).astype(np.float32).astype(np.complex64)
    return Y, O0


def _tight_vs_oracle(r, ds, Y, O0, L, E, B, opt):
    o64 = orc.cufpm_pure_v3(O0, ds.P0c, Y[:L], ds.led_idx[:L], ds.pupil0, ds.pratio, E, B, opt=opt)
    o32 = orc.cufpm_pure_v3(O0, ds.P0c, Y[:L], ds.led_idx[:L], ds.pupil0, ds.pratio, E, B, opt=opt,
                            dtype=np.float32)
    for k in ("object", "pupil", "spectrum"):
        e = orc.rel_err(r[k], getattr(o64, k))
        e32 = orc.rel_err(getattr(o32, k), getattr(o64, k))
        assert e < max(TIGHT, 3 * e32), (k, e, e32)
    np.testing.assert_allclose(r["loss"], o64.loss, rtol=1e-5)


def test_single_update_vs_oracle(engine, ds_a):
    """One mini-batch, one RMSprop step, noisy data."""
    ds = ds_a
    opt = (1e-3, 0.999, 1e-4)
    r = _solve(engine, ds, 8, 1, 8, opt)
    _tight_vs_oracle(r, ds, ds.Y, ds.O0, 8, 1, 8, opt)


def test_solve_noiseless_vs_oracle(engine, ds_a):
    """Bright-field rings, two epochs (10 updates) on noiseless amplitudes."""
    ds = ds_a
    Y, O0 = _noiseless(ds)
    opt = (1e-3, 0.999, 1e-4)
    r = engine.solve(O0, ds.P0c, to_matlab_stack(Y[:25]), led_matlab(ds.led_idx[:25]), ds.pupil0,
                     ds.pratio, 2, 8, lr=opt[0], beta=opt[1], eps=opt[2])
    _tight_vs_oracle(r, ds, Y, O0, 25, 2, 8, opt)


def _truth_err(O, T):
    """min over complex scalars a of ||a O - T|| / ||T||."""
    O = np.asarray(O, np.complex128).ravel()
    T = np.asarray(T, np.complex128).ravel()
    a = np.vdot(O, T) / np.vdot(O, O)
    return float(np.linalg.norm(a * O - T) / np.linalg.norm(T))


def test_solve_128x121_vs_oracle(engine, ds_a):
    """The 128² case end to end: 121 LEDs, 5 epochs, batch 8, lr 1e-3."""
    ds = ds_a
    opt = (1e-3, 0.999, 1e-4)
    r = _solve(engine, ds, 121, 5, 8, opt)
    o64 = orc.cufpm_pure_v3(ds.O0, ds.P0c, ds.Y, ds.led_idx, ds.pupil0, 4, 5, 8, opt=opt)
    o32 = orc.cufpm_pure_v3(ds.O0, ds.P0c, ds.Y, ds.led_idx, ds.pupil0, 4, 5, 8, opt=opt,
                            dtype=np.float32)
    for k in ("object", "pupil", "spectrum"):
        e = orc.rel_err(r[k], getattr(o64, k))
        e32 = orc.rel_err(getattr(o32, k), getattr(o64, k))
        print(f"128x121 {k}: engine-vs-fp64 {e:.3e}, fp32-oracle-vs-fp64 {e32:.3e}")
        assert e < max(5 * e32, 3e-2), k
    np.testing.assert_allclose(r["loss"], o64.loss, rtol=5e-3)
    assert np.all(np.diff(r["loss"]) < 0)
    q_engine = _truth_err(r["object"], ds.object_true)
    q_fp64 = _truth_err(o64.object, ds.object_true)
    print(f"128x121 error vs true object: engine {q_engine:.4f}, fp64 oracle {q_fp64:.4f}")
    assert abs(q_engine - q_fp64) < 0.02 * q_fp64


def test_uint16_stack_is_bit_identical_to_amplitude(engine, ds_small):
    ds = ds_small
    opt = (2e-3, 0.999, 1e-4)
    a = _solve(engine, ds, 25, 2, 6, opt, raw=False)
    b = _solve(engine, ds, 25, 2, 6, opt, raw=True)
    np.testing.assert_array_equal(a["object"], b["object"])
    np.testing.assert_array_equal(a["pupil"], b["pupil"])
    np.testing.assert_array_equal(a["loss"], b["loss"])


def test_normalise_stack_bit_exact(engine, ds_small):
    amp = engine.normalise_stack(ds_small.raw)
    np.testing.assert_array_equal(amp, orc.normalise_stack_u16(ds_small.raw))


def test_device_memory_matches_host_memory(engine, ds_small):
    import torch
    ds = ds_small
    opt = (2e-3, 0.999, 1e-4)
    host = _solve(engine, ds, 25, 2, 6, opt)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    r = engine.solve(dev(ds.O0), dev(ds.P0c), dev(to_matlab_stack(ds.Y)), dev(led_matlab(ds.led_idx)),
                     dev(ds.pupil0), ds.pratio, 2, 6, lr=opt[0], beta=opt[1], eps=opt[2])
    np.testing.assert_array_equal(r["object"].cpu().numpy(), host["object"])
    np.testing.assert_array_equal(r["pupil"].cpu().numpy(), host["pupil"])
    np.testing.assert_array_equal(r["loss"].cpu().numpy(), host["loss"])


def test_bicubic_initial_object(engine, ds_small):
    ds = ds_small
    r = engine.solve(None, ds.P0c, to_matlab_stack(ds.Y), led_matlab(ds.led_idx), ds.pupil0,
                     ds.pratio, 0, 5)
    ref = orc.imresize_bicubic(ds.Y[0], ds.pratio)
    np.testing.assert_allclose(r["object"].real, ref, rtol=0, atol=2e-7)
    assert np.all(r["object"].imag == 0)


def test_wrapping_crops_and_ragged_batches(engine):
    """LED corners at and past the spectrum edge wrap modulo H; L mod B != 0."""
    from fpm_b200 import synth
    rng = np.random.default_rng(4)
    h, p = 32, 2
    H = h * p
    opt = synth.Optics(led_grid=3)
    O0 = (0.5 + 0.5 * rng.random((H, H)) * np.exp(1j * rng.random((H, H)))).astype(np.complex64)
    P0 = synth.pupil_circle(h, opt)
    led = np.array([[1, 1], [H - 10, 3], [H, H], [20, H - 20], [7, 30], [H // 2, H // 2 + 5],
                    [3, H - 1]], np.int32)
    Y = rng.random((len(led), h, h)).astype(np.float32)
    args = (O0, P0.astype(np.complex64), Y, led, P0)
    for batch in (3, 7, 10):
        r = engine.solve(O0, P0.astype(np.complex64), to_matlab_stack(Y), led_matlab(led), P0, p, 2,
                         batch, lr=1e-3, beta=0.9, eps=1e-4)
        o = orc.cufpm_pure_v3(*args, p, 2, batch, opt=(1e-3, 0.9, 1e-4))
        assert orc.rel_err(r["object"], o.object) < 1e-4, batch
        assert orc.rel_err(r["pupil"], o.pupil) < 1e-4, batch


@pytest.mark.parametrize("n", [16, 32, 64, 128, 256, 512, 1024, 2048, 4096])
def test_fft2_matches_numpy(engine, n):
    rng = np.random.default_rng(n)
    cnt = 3 if n <= 1024 else 1
    x = (rng.standard_normal((n, n, cnt)) + 1j * rng.standard_normal((n, n, cnt))).astype(np.complex64)
    ref = np.fft.fft2(x.astype(np.complex128), axes=(0, 1))
    y = engine.fft2(x, -1)
    assert orc.rel_err(y, ref) < 2e-6 * max(1.0, np.log2(n) / 8)
    yi = engine.fft2(x, +1)
    refi = np.fft.ifft2(x.astype(np.complex128), axes=(0, 1)) * n * n
    assert orc.rel_err(yi, refi) < 2e-6 * max(1.0, np.log2(n) / 8)


def test_fft2_large_lines_device(engine):
    """8192 and 16384-point lines (one line per CTA) on device memory, against numpy."""
    import torch
    for n in (8192, 16384):
        rng = np.random.default_rng(n)
        # a sparse test signal keeps the numpy reference cheap: a few random tones
        x = np.zeros((n, n), np.complex64)
        idx = rng.integers(0, n, size=(64, 2))
        x[idx[:, 0], idx[:, 1]] = (rng.standard_normal(64) + 1j * rng.standard_normal(64))
        y = engine.fft2(torch.from_numpy(x).cuda(), -1).cpu().numpy()
        # check a random sample of output pixels against the direct DFT of the tones
        ks = rng.integers(0, n, size=(256, 2))
        vals = x[idx[:, 0], idx[:, 1]].astype(np.complex128)
        ph = np.exp(-2j * np.pi * (np.outer(ks[:, 0], idx[:, 0]) + np.outer(ks[:, 1], idx[:, 1])) / n)
        ref = ph @ vals
        got = y[ks[:, 0], ks[:, 1]]
        assert np.abs(got - ref).max() < 1e-4 * np.abs(vals).sum(), n


def test_fft2_dense_separable_16384(engine):
    """Every output of a dense 16384 x 16384 transform: a separable input a b^T has the
    separable transform fft(a) fft(b)^T (numpy, FP64), compared on the device."""
    import torch
    n = 16384
    rng = np.random.default_rng(7)
    a = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    b = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    for sign, A, B in ((-1, np.fft.fft(a), np.fft.fft(b)),
                       (+1, np.fft.ifft(a) * n, np.fft.ifft(b) * n)):
        x = torch.outer(torch.from_numpy(a.astype(np.complex64)).cuda(),
                        torch.from_numpy(b.astype(np.complex64)).cuda())
        y = engine.fft2(x, sign)
        del x
        ref = torch.outer(torch.from_numpy(A.astype(np.complex64)).cuda(),
                          torch.from_numpy(B.astype(np.complex64)).cuda())
        err = (torch.linalg.vector_norm(torch.view_as_real(y - ref), dtype=torch.float64)
               / torch.linalg.vector_norm(torch.view_as_real(ref), dtype=torch.float64)).item()
        del y, ref
        torch.cuda.empty_cache()
        assert err < 2e-6 * np.log2(n) / 8, (sign, err)


def test_unsupported_sizes_are_refused(engine):
    """A side with a prime factor above 7 (44 = 4 x 11) has no transform here."""
    rng = np.random.default_rng(1)
    h = 44
    P0 = np.ones((h, h), np.float32)
    with pytest.raises(fpm_b200.FpmError) as e:
        engine.solve(np.ones((88, 88), np.complex64), P0.astype(np.complex64),
                     rng.random((h, h, 2)).astype(np.float32), np.array([[1, 1], [2, 2]], np.int32).T,
                     P0, 2, 1, 2)
    assert e.value.status == 2


def test_lr_schedule_and_single_led(engine, ds_small):
    """One off-centre LED, batch larger than L, lr halving after every epoch."""
    ds = ds_small
    opt = (1e-3, 0.999, 1e-4)
    sel = slice(6, 7)          # off-centre: the gradient is not real-symmetric
    r = engine.solve(ds.O0, ds.P0c, to_matlab_stack(ds.Y[sel]), led_matlab(ds.led_idx[sel]),
                     ds.pupil0, ds.pratio, 3, 4, lr=opt[0], beta=opt[1], eps=opt[2],
                     lr_halve_after=0)
    o64 = orc.cufpm_pure_v3(ds.O0, ds.P0c, ds.Y[sel], ds.led_idx[sel], ds.pupil0, ds.pratio, 3, 4,
                            opt=opt, lr_halve_after=0)
    o32 = orc.cufpm_pure_v3(ds.O0, ds.P0c, ds.Y[sel], ds.led_idx[sel], ds.pupil0, ds.pratio, 3, 4,
                            opt=opt, lr_halve_after=0, dtype=np.float32)
    e32 = orc.rel_err(o32.object, o64.object)
    assert orc.rel_err(r["object"], o64.object) < max(TIGHT, 3 * e32)
    # the schedule itself: without halving the same run moves further
    r2 = engine.solve(ds.O0, ds.P0c, to_matlab_stack(ds.Y[sel]), led_matlab(ds.led_idx[sel]),
                      ds.pupil0, ds.pratio, 3, 4, lr=opt[0], beta=opt[1], eps=opt[2])
    assert orc.rel_err(r2["object"], ds.O0) > orc.rel_err(r["object"], ds.O0)


def test_mirror_of_the_mex_call(ds_small):
    ds = ds_small
    O, P = fpm_b200.cuFPM_pure_v3(ds.O0, ds.P0c, to_matlab_stack(ds.Y), led_matlab(ds.led_idx),
                                  ds.pupil0, ds.pratio, 1, 26, [5e-4, 0.999, 1e-4])
    o = orc.cufpm_pure_v3(ds.O0, ds.P0c, ds.Y, ds.led_idx, ds.pupil0, ds.pratio, 1, 26)
    assert O.shape == (ds.h * ds.pratio,) * 2 and P.shape == (ds.h, ds.h)
    assert orc.rel_err(O, o.object) < 1e-3


# ---- error paths: host-detectable, nothing faults --------------------------
def _bad(engine, ds, **kw):
    args = dict(O0=ds.O0, P0c=ds.P0c, Y=to_matlab_stack(ds.Y[:4]), led_idx=led_matlab(ds.led_idx[:4]),
                P0=ds.pupil0, pratio=ds.pratio, epochs=1, batch=2)
    args.update(kw)
    with pytest.raises(fpm_b200.FpmError) as e:
        engine.solve(**args)
    return e.value.status


def test_invalid_arguments_are_rejected(engine, ds_small):
    ds = ds_small
    assert _bad(engine, ds, batch=0) == 1
    assert _bad(engine, ds, epochs=-1) == 1
    bad_led = led_matlab(ds.led_idx[:4]).copy()
    bad_led[0, 0] = 0
    assert _bad(engine, ds, led_idx=bad_led) == 1
    bad_led[0, 0] = ds.h * ds.pratio + 1
    assert _bad(engine, ds, led_idx=bad_led) == 1
    Yodd = np.zeros((5, 5, 4), np.float32)
    assert _bad(engine, ds, Y=Yodd, P0c=np.zeros((5, 5), np.complex64),
                P0=np.zeros((5, 5), np.float32)) == 1
    assert _bad(engine, ds, beta=1.5) == 1


def test_memory_limit_is_enforced(ds_small):
    ds = ds_small
    e = fpm_b200.Engine(0, mem_limit_bytes=1 << 20)
    with pytest.raises(fpm_b200.FpmError) as ex:
        e.solve(ds.O0, ds.P0c, to_matlab_stack(ds.Y), led_matlab(ds.led_idx), ds.pupil0, ds.pratio,
                1, 4)
    assert ex.value.status == 3
    e.close()


def test_nonfinite_loss_is_reported(engine, ds_small):
    ds = ds_small
    Y = to_matlab_stack(ds.Y[:4]).copy()
    Y[3, 3, 0] = np.nan
    with pytest.raises(fpm_b200.FpmError) as ex:
        engine.solve(ds.O0, ds.P0c, Y, led_matlab(ds.led_idx[:4]), ds.pupil0, ds.pratio, 1, 2)
    assert ex.value.status == 5


@pytest.mark.parametrize("grid,h,p,dx,dy", [(19, 2048, 8, -0.0, -0.0), (11, 128, 4, -0.0, -0.0),
                                           (5, 64, 2, 1625.0, -3250.0), (1, 256, 4, -0.0, -0.0)])
def test_led_indices_on_device_equal_oracle(engine, grid, h, p, dx, dy):
    """FP64 geometry on the device: bit-identical integers to the oracle's IEEE double
    evaluation of init_environment_rgb.m, spiral order included."""
    from fpm_b200 import synth
    o = synth.Optics(led_grid=grid)
    args = (grid, h, p, o.wavelength_um, o.led_pitch_mm * 1000, o.led_height_mm * 1000,
            o.camera_pixel_um, o.magnification)
    led, order = engine.led_indices(*args, sample_dx_um=dx, sample_dy_um=dy)
    ref, ref_order = orc.led_geometry(*args, sample_dx_um=dx, sample_dy_um=dy)
    np.testing.assert_array_equal(order, ref_order)
    np.testing.assert_array_equal(led, ref)


def test_led_indices_rejects_bad_geometry(engine):
    with pytest.raises(fpm_b200.FpmError) as e:
        engine.led_indices(4, 128, 4, 0.532, 4000, 90000, 6.5, 4)     # even grid
    assert e.value.status == 1
    with pytest.raises(fpm_b200.FpmError):
        engine.led_indices(5, 128, 4, 0.0, 4000, 90000, 6.5, 4)       # zero wavelength


def _engine_sized_ref_fixtures():
    """Reference-build fixtures whose sizes the engine supports (powers of two)."""
    from pathlib import Path
    out = []
    for f in sorted((Path(__file__).resolve().parent / "golden").glob("ref_gradients_*.npz")):
        h = int(np.load(f)["P"].shape[0])
        if h & (h - 1) == 0:
            out.append(f.name)
    return out


@pytest.mark.parametrize("name", _engine_sized_ref_fixtures())
def test_gradients_match_reference_build(engine, name):
    """The engine against the reference's own CUDA kernels (+ cuFFT) on the same inputs:
    fixtures of tests/golden made on a B200 by make_golden.py --ref.  The tolerance is the
    fixture's (10x the FP32 twin's distance to FP64, floor 1e-5); a sign of the loss
    stencil taken the other way at a near-tie moves a gradient by ~1e-3, so the engine
    must match within the tolerance or, failing that, the FP64 oracle as tightly as the
    reference build does."""
    from pathlib import Path
    g = np.load(Path(__file__).resolve().parent / "golden" / name)
    h = g["P"].shape[0]
    ones = np.ones((h, h), np.float32)       # pupil amplitude: unused by a gradient call
    dO, dP, loss = engine.batch_gradients(g["O"], g["P"], to_matlab_stack(g["Y"]),
                                          led_matlab(g["led_idx"]), ones, int(g["pratio"]))
    tol = float(g["tol"])
    e_o = orc.rel_err(dO, g["ref_dO"])
    e_p = orc.rel_err(dP, g["ref_dP"])
    print(f"{name}: engine-vs-reference dO {e_o:.3e} dP {e_p:.3e} (tol {tol:.1e})")
    assert e_o < tol and e_p < tol


def test_pupil_support_pruning_is_exact(engine, ds_small):
    """The solve prunes every pass to the pupil's support box; with an off-centre,
    asymmetric support the result must equal the unpruned solve (FPM_PUPIL_SUPPORT=0)
    up to the rounding of the skipped zero terms, and the pupil must stay zero outside."""
    import os
    ds = ds_small
    h = ds.h
    P0 = np.zeros((h, h), np.float32)
    P0[5:41, 20:61] = ds.pupil0[5:41, 20:61] + 0.25          # rows 5..40, cols 20..60
    P0c = (P0 * np.exp(0.3j * np.arange(h)[None, :] / h)).astype(np.complex64)
    args = (ds.O0, P0c, to_matlab_stack(ds.Y[:25]), led_matlab(ds.led_idx[:25]), P0, ds.pratio, 2, 6)
    kw = dict(lr=2e-3, beta=0.999, eps=1e-4)
    pruned = engine.solve(*args, **kw)
    os.environ["FPM_PUPIL_SUPPORT"] = "0"
    try:
        whole = engine.solve(*args, **kw)
    finally:
        del os.environ["FPM_PUPIL_SUPPORT"]
    for k in ("object", "pupil", "spectrum"):
        assert orc.rel_err(pruned[k], whole[k]) < 1e-5, (k, orc.rel_err(pruned[k], whole[k]))
    np.testing.assert_allclose(pruned["loss"], whole["loss"], rtol=1e-6)
    assert np.all(pruned["pupil"][P0 == 0] == 0)
    o64 = orc.cufpm_pure_v3(ds.O0, P0c, ds.Y[:25], ds.led_idx[:25], P0, ds.pratio, 2, 6,
                            opt=(2e-3, 0.999, 1e-4))
    assert orc.rel_err(pruned["object"], o64.object) < 2e-2


@pytest.mark.parametrize("h,p,amplitude", [(64, 4, False), (32, 2, True), (256, 8, False)])
def test_simulate_matches_oracle(engine, h, p, amplitude):
    """Device forward model against the FP64 oracle, crops inside and past the edge."""
    rng = np.random.default_rng(h + p)
    H = h * p
    O = (0.5 + 0.5 * rng.random((H, H))) * np.exp(1j * rng.standard_normal((H, H)))
    from fpm_b200 import synth
    P = synth.pupil_circle(h, synth.Optics(led_grid=5)) * np.exp(0.3j * rng.standard_normal((h, h)))
    led = np.concatenate([rng.integers(1, H + 1, size=(9, 2)),
                          np.array([[1, 1], [H, H], [H - h // 2, 3]])]).astype(np.int32)
    got = engine.simulate(O.astype(np.complex64), P.astype(np.complex64), led_matlab(led), p,
                          amplitude=amplitude)
    ref = orc.forward_model(O, P, led, p, amplitude=amplitude)
    assert got.shape == (h, h, len(led))
    e = orc.rel_err(np.transpose(got, (2, 0, 1)), ref)
    assert e < 2e-6 * max(1.0, np.log2(H) / 8), e


def test_simulate_device_memory_and_bad_input(engine):
    import torch
    rng = np.random.default_rng(5)
    h, p = 64, 2
    H = h * p
    O = (rng.standard_normal((H, H)) + 1j * rng.standard_normal((H, H))).astype(np.complex64)
    P = np.ones((h, h), np.complex64)
    led = led_matlab(np.array([[5, 9], [H, 1]], np.int32))
    host = engine.simulate(O, P, led, p)
    dev = engine.simulate(torch.from_numpy(O).cuda(), torch.from_numpy(P).cuda(),
                          torch.from_numpy(led).cuda(), p).cpu().numpy()
    np.testing.assert_array_equal(host, dev)
    with pytest.raises(fpm_b200.FpmError) as e:
        engine.simulate(O, P, led_matlab(np.array([[0, 1]], np.int32)), p)   # kl = 0
    assert e.value.status == 1


def test_isotropic_loss_gradients_and_solve(engine, ds_small, ds_a):
    """The isotropic loss (ret_loss.m 'isotropic'): no sign decisions, so the FP32 engine
    tracks the FP64 oracle closely; both the separate (h = 64) and fused (h = 128) row
    passes run it."""
    for ds in (ds_small, ds_a):
        H = ds.h * ds.pratio
        rng = np.random.default_rng(21)
        O = (ds.O0 * np.exp(1j * 0.2 * rng.standard_normal((H, H)))).astype(np.complex64)
        P = ds.pupil_true
        sel = slice(0, 9)
        dO, dP, loss = engine.batch_gradients(O, P, to_matlab_stack(ds.Y[sel]),
                                              led_matlab(ds.led_idx[sel]), ds.pupil0, ds.pratio,
                                              loss="isotropic")
        G, dP64, l64 = orc.batch_gradients(np.fft.fft2(O.astype(np.complex128)),
                                           P.astype(np.complex128), ds.Y[sel].astype(np.float64),
                                           ds.led_idx[sel], ds.pratio, np.float64,
                                           loss_kind="isotropic")
        assert abs(loss - l64) < 1e-6 * abs(l64)
        assert orc.rel_err(dO, np.fft.ifft2(G) * H * H) < TIGHT
        assert orc.rel_err(dP, dP64) < TIGHT
        opt = (1e-3, 0.999, 1e-4)
        r = engine.solve(ds.O0, ds.P0c, to_matlab_stack(ds.Y[:16]), led_matlab(ds.led_idx[:16]),
                         ds.pupil0, ds.pratio, 2, 8, lr=opt[0], beta=opt[1], eps=opt[2],
                         loss="isotropic")
        o = orc.cufpm_pure_v3(ds.O0, ds.P0c, ds.Y[:16], ds.led_idx[:16], ds.pupil0, ds.pratio, 2, 8,
                              opt=opt, loss_kind="isotropic")
        assert orc.rel_err(r["object"], o.object) < TIGHT      # the FP32 twin: 2.6e-7
        assert orc.rel_err(r["pupil"], o.pupil) < TIGHT
        np.testing.assert_allclose(r["loss"], o.loss, rtol=1e-6)


def test_16384_columns_32_values_per_thread_match_16(engine):
    """The 16384-point passes run radix-32 stages with 32 values per thread; the 16-value
    variant (FPM_COLS_E16=1) is the same transform with other roundings.  A short solve at
    2048^2 -> 16384^2 and a gradient call must agree to FP32 rounding (isotropic loss: no
    sign decisions that a rounding difference could flip)."""
    import os
    import torch
    from fpm_b200 import synth
    h, p = 2048, 8
    H = h * p
    optics = synth.Optics(led_grid=3)
    circ = synth.pupil_circle(h, optics)
    led = led_matlab(synth.led_indices(h, p, optics)[:3])
    g = torch.Generator(device="cuda")
    g.manual_seed(3)
    Y = (torch.rand((3, h, h), generator=g, device="cuda") * 0.5 + 0.25).permute(1, 2, 0)
    O0 = torch.polar(torch.ones((H, H), device="cuda"),
                     0.1 * torch.randn((H, H), generator=g, device="cuda")).contiguous()
    P0c = torch.from_numpy(circ.astype(np.complex64)).cuda()
    P0 = torch.from_numpy(circ).cuda()
    ledt = torch.from_numpy(led).cuda()
    runs = {}
    for flag in ("0", "1"):
        os.environ["FPM_COLS_E16"] = flag
        try:
            r = engine.solve(O0, P0c, Y, ledt, P0, p, 1, 3, lr=1e-3, spectrum=False,
                             loss="isotropic")
            d = engine.batch_gradients(O0, P0c, Y, ledt, P0, p, loss="isotropic")
            runs[flag] = (r["object"].cpu().numpy(), r["pupil"].cpu().numpy(),
                          d[0].cpu().numpy(), d[1].cpu().numpy())
        finally:
            del os.environ["FPM_COLS_E16"]
    # two FP32 roundings of 16384^2 transforms (each ~5e-6 relative) apart; a wrong
    # transform would be O(1) off
    for a, b in zip(runs["0"], runs["1"]):
        assert orc.rel_err(a, b) < 3e-5, orc.rel_err(a, b)



def test_prefetching_passes_equal_plain_loads(engine):
    """The persistent passes that copy their next input into shared memory during the
    last FFT stage (column update, next-box rows, and at h = 2048 the low-resolution
    forward column pass) compute what their plain-load forms (FPM_COLS_ASYNC=0) compute: a
    2048^2 -> 16384^2 solve over two batches with uint16 frames, whose LED crops sit off
    the box edge, must be bit-identical (the loss to double rounding of its partials)."""
    import os
    import torch
    from fpm_b200 import synth
    h, p = 2048, 8
    H = h * p
    optics = synth.Optics(led_grid=3)
    circ = synth.pupil_circle(h, optics)
    led = led_matlab(synth.led_indices(h, p, optics)[:5])
    g = torch.Generator(device="cuda")
    g.manual_seed(5)
    Y = torch.randint(0, 40000, (5, h, h), generator=g, device="cuda",
                      dtype=torch.int32).to(torch.uint16).permute(1, 2, 0)
    O0 = torch.polar(torch.ones((H, H), device="cuda"),
                     0.1 * torch.randn((H, H), generator=g, device="cuda")).contiguous()
    P0c = torch.from_numpy(circ.astype(np.complex64)).cuda()
    P0 = torch.from_numpy(circ).cuda()
    ledt = torch.from_numpy(led).cuda()
    runs = {}
    for flag in ("1", "0"):
        os.environ["FPM_COLS_ASYNC"] = flag
        try:
            r = engine.solve(O0, P0c, Y, ledt, P0, p, 2, 3, lr=1e-3, spectrum=False)
            runs[flag] = (r["object"].cpu().numpy(), r["pupil"].cpu().numpy(),
                          np.asarray(r["loss"].cpu() if hasattr(r["loss"], "cpu") else r["loss"]))
        finally:
            del os.environ["FPM_COLS_ASYNC"]
    np.testing.assert_array_equal(runs["1"][0], runs["0"][0])
    np.testing.assert_array_equal(runs["1"][1], runs["0"][1])
    np.testing.assert_allclose(runs["1"][2], runs["0"][2], rtol=1e-12)


def test_large_lowres_side_two_pass_rows_vs_oracle(engine):
    """h = 4096 (beyond the fused row pass: the two-pass L2 / L3 form), pratio 2 ->
    8192², one batch of three LEDs with one crop past the spectrum edge, one update,
    against the FP64 oracle."""
    from fpm_b200 import synth
    rng = np.random.default_rng(41)
    h, p = 4096, 2
    H = h * p
    P0 = synth.pupil_circle(h, synth.Optics(led_grid=3)).astype(np.float32)
    O0 = (0.5 + 0.5 * rng.random((H, H)) * np.exp(1j * rng.random((H, H)))).astype(np.complex64)
    led = np.array([[H // 2 - h // 2 + 1, H // 2 - h // 2 + 1], [H - 100, 50], [700, 1900]],
                   np.int32)
    Y = rng.random((3, h, h)).astype(np.float32)
    opt = (1e-3, 0.999, 1e-4)
    r = engine.solve(O0, P0.astype(np.complex64), to_matlab_stack(Y), led_matlab(led), P0, p, 1, 3,
                     lr=opt[0], beta=opt[1], eps=opt[2])
    args = (O0, P0.astype(np.complex64), Y, led, P0, p, 1, 3)
    o = orc.cufpm_pure_v3(*args, opt=opt, workers=orc.default_workers())
    # FP32 rounding of 4096² and 8192² transforms: the bar is the FP32 twin's own distance
    o32 = orc.cufpm_pure_v3(*args, opt=opt, dtype=np.float32, workers=orc.default_workers())
    for k in ("object", "pupil"):
        e, e32 = orc.rel_err(r[k], getattr(o, k)), orc.rel_err(getattr(o32, k), getattr(o, k))
        assert e < max(TIGHT, 3 * e32), (k, e, e32)
    np.testing.assert_allclose(r["loss"], o.loss, rtol=1e-5)


@pytest.mark.parametrize("pie", ["ePIE", "tPIE"])
def test_pie_weights_gradients_and_solve(engine, ds_small, ds_a, pie):
    """The deconv_pie weights of the conventional MATLAB gradient (fpm_forward_GPU.m:64-76)
    on the v3 gradient terms, against the FP64 oracle: gradients of one batch (whole
    crops) and a two-epoch solve (pruned to the pupil support for tPIE, whole crops for
    ePIE), with the isotropic loss so that no sign decision separates the FP32 engine from
    the oracle."""
    for ds in (ds_small, ds_a):
        H = ds.h * ds.pratio
        rng = np.random.default_rng(33)
        O = (ds.O0 * np.exp(1j * 0.2 * rng.standard_normal((H, H)))).astype(np.complex64)
        P = ds.pupil_true
        sel = slice(0, 9)
        dO, dP, loss = engine.batch_gradients(O, P, to_matlab_stack(ds.Y[sel]),
                                              led_matlab(ds.led_idx[sel]), ds.pupil0, ds.pratio,
                                              loss="isotropic", pie=pie)
        G, dP64, l64 = orc.batch_gradients(np.fft.fft2(O.astype(np.complex128)),
                                           P.astype(np.complex128), ds.Y[sel].astype(np.float64),
                                           ds.led_idx[sel], ds.pratio, np.float64,
                                           loss_kind="isotropic", pie=pie)
        # tPIE divides by |ker|^2 + 1e-5 pixel by pixel, which magnifies the rounding of
        # small spectrum values: the bar is the FP32 oracle twin's own distance
        G32, dP32, _ = orc.batch_gradients(np.fft.fft2(O), P.astype(np.complex64),
                                           ds.Y[sel].astype(np.float32), ds.led_idx[sel],
                                           ds.pratio, np.float32, loss_kind="isotropic", pie=pie)
        bar_o = max(TIGHT, 3 * orc.rel_err(np.fft.ifft2(G32.astype(np.complex128)), np.fft.ifft2(G)))
        bar_p = max(TIGHT, 3 * orc.rel_err(dP32, dP64))
        assert abs(loss - l64) < 1e-6 * abs(l64)
        e_o = orc.rel_err(dO, np.fft.ifft2(G) * H * H)
        assert e_o < bar_o, (e_o, bar_o)
        assert orc.rel_err(dP, dP64) < bar_p, (orc.rel_err(dP, dP64), bar_p)
        opt = (1e-3, 0.999, 1e-4)
        r = engine.solve(ds.O0, ds.P0c, to_matlab_stack(ds.Y[:16]), led_matlab(ds.led_idx[:16]),
                         ds.pupil0, ds.pratio, 2, 8, lr=opt[0], beta=opt[1], eps=opt[2],
                         loss="isotropic", pie=pie)
        args = (ds.O0, ds.P0c, ds.Y[:16], ds.led_idx[:16], ds.pupil0, ds.pratio, 2, 8)
        o = orc.cufpm_pure_v3(*args, opt=opt, loss_kind="isotropic", pie=pie)
        o32 = orc.cufpm_pure_v3(*args, opt=opt, loss_kind="isotropic", pie=pie, dtype=np.float32)
        for k in ("object", "pupil"):
            e, e32 = orc.rel_err(r[k], getattr(o, k)), orc.rel_err(getattr(o32, k), getattr(o, k))
            assert e < max(TIGHT, 3 * e32), (k, e, e32)
        np.testing.assert_allclose(r["loss"], o.loss, rtol=1e-6)


def test_full_size_forward_model_and_zero_residual(engine):
    """At the bench's size (2048² frames, pratio 8 -> a 16384² object), where the FP64
    oracle is too slow, two size-independent properties:
    (1) the device forward model (benchmark/gen_img_batch.m:178-201) equals a plain torch
        complex64 restatement of it (cuFFT) to 2e-5 relative L2 per LED, crops inside
        and past the spectrum edge;
    (2) frames simulated from (O, P) are explained by (O, P): the batch loss there is
        below 1e-3 of the loss at the same object with 0.05 rad of phase noise added."""
    import torch
    from fpm_b200 import synth
    h, p = 2048, 8
    H = h * p
    optics = synth.Optics(led_grid=3)
    led = np.concatenate([synth.led_indices(h, p, optics)[:5],
                          np.array([[H - h // 2, 3]])]).astype(np.int32)
    g = torch.Generator(device="cuda")
    g.manual_seed(11)
    O = torch.polar(torch.ones((H, H), device="cuda"),
                    0.2 * torch.randn((H, H), generator=g, device="cuda")).contiguous()
    circ = synth.pupil_circle(h, optics)
    ab = np.exp(0.3j * np.random.default_rng(3).standard_normal((h, h)))
    P = torch.from_numpy((circ * ab).astype(np.complex64)).cuda()
    ledt = torch.from_numpy(led_matlab(led)).cuda()
    Y = engine.simulate(O, P, ledt, p, amplitude=True)            # (h, h, L) on the device
    assert tuple(Y.shape) == (h, h, len(led))

    ref = torch_forward_model(O, P, led, p)                       # (L, h, h), cuFFT
    for l in range(len(led)):
        err = (torch.linalg.vector_norm(Y[:, :, l] - ref[l]) / torch.linalg.vector_norm(ref[l])).item()
        assert err < 2e-5, (l, err)
    del ref

    P0 = torch.from_numpy(circ).cuda()
    scalar = lambda x: float(torch.as_tensor(x).reshape(-1)[0])
    _, _, loss_true = engine.batch_gradients(O, P, Y, ledt, P0, p)
    noise = torch.polar(torch.ones((H, H), device="cuda"),
                        0.05 * torch.randn((H, H), generator=g, device="cuda"))
    _, _, loss_pert = engine.batch_gradients((O * noise).contiguous(), P, Y, ledt, P0, p)
    assert scalar(loss_pert) > 0
    assert scalar(loss_true) < 1e-3 * scalar(loss_pert), (scalar(loss_true), scalar(loss_pert))


def test_bounded_wait_failure_reaches_the_host(engine, ds_small):
    """A device-side wait that runs out (an mbarrier armed for bytes that no copy delivers,
    a bound of 2^20 SM clocks) must come back as FPM_ERR_INTERNAL with its detail, through
    the same device flag the passes use, and leave the context usable for the next solve."""
    st = engine.lib.fpm_selftest_bounded_wait(engine._ctx, 1 << 20)
    assert st == 7, st
    assert "timed out" in engine.lib.fpm_last_error(engine._ctx).decode()
    ds = ds_small
    r = engine.solve(ds.O0, ds.P0c, to_matlab_stack(ds.Y[:8]), led_matlab(ds.led_idx[:8]),
                     ds.pupil0, ds.pratio, 1, 8, lr=1e-3)
    assert np.all(np.isfinite(r["loss"]))
    assert engine.lib.fpm_selftest_bounded_wait(engine._ctx, 0) == 1      # bound out of range
