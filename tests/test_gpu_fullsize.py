"""Parity of the kernels that run at the bench's size, against an FP64 checker.

The bench reconstructs 2048² frames into a 16384² object; several kernels exist only
in their 2048 / 16384 instantiations (the fused row pass with 4-CTA clusters, two CTAs
per SM and TMA tiles at h = 2048, the persistent low-resolution column pass, the 16384-point column
update and row passes with 32 values per thread and bulk-copy prefetch).  The numpy
FP64 oracle takes minutes per update there, so the checker is its torch restatement
(``oracle/torch_ref.py``, pinned on the CPU against the numpy oracle) run on the GPU in
complex128; its complex64 twin (cuFFT) gives the FP32 distance that sets the bars:

* isotropic loss (no sign decisions): within max(2e-5, 3x the twin's distance);
* anisotropic loss (the v3 loss): sign() of residual differences within an FP32
  rounding of zero flips in any FP32 implementation; the same bar then measures the
  engine against the FP64 result exactly as it measures the twin;
* the per-batch loss: 1e-5 relative to FP64 (a sum over 4M pixels per LED, continuous
  in the inputs);
* 361 LEDs of 512² -> 4096² end to end (10 epochs): the criteria of the 128² case
  (within max(5x the twin's drift, 3e-2), loss curve to 5e-3, the true object
  reconstructed as well as FP64 reconstructs it, within 2%).

The reference loop these follow: cuFPM_v3/cuFPM_pure_v3.cu:128-207.
"""
import math

import numpy as np
import pytest

from conftest import led_matlab

pytestmark = pytest.mark.gpu

TIGHT = 2e-5


def _smooth(H, sigma, g, normal):
    import torch
    x = (torch.randn if normal else torch.rand)((H, H), generator=g, device="cuda")
    f0 = torch.fft.fftfreq(H, device="cuda")
    f1 = torch.fft.rfftfreq(H, device="cuda")
    X = torch.fft.rfft2(x)
    X *= torch.exp(-2 * (math.pi * sigma) ** 2 * f0 * f0)[:, None]
    X *= torch.exp(-2 * (math.pi * sigma) ** 2 * f1 * f1)[None, :]
    y = torch.fft.irfft2(X, s=(H, H))
    return (y - y.min()) / (y.max() - y.min())


def _case(h, p, grid, n_leds, seed, shift=(0, 0), past_edge=True):
    """A seeded problem on the GPU in MATLAB index order: true object, aberrated pupil
    (support optionally moved off centre by `shift` pixels), LED corners (the first
    n_leds of the spiral, plus one crop running past the spectrum edge), uint16 frames
    (Poisson at 3e4 peak counts), their amplitudes, and a perturbed starting object."""
    import torch
    from fpm_b200 import synth
    from oracle import torch_ref as tr
    H = h * p
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    amp = 0.5 + 0.5 * _smooth(H, 3.0, g, False)
    ph = (_smooth(H, 4.0, g, True) - 0.5) * math.pi
    O_true = torch.polar(amp, ph)
    del amp, ph
    optics = synth.Optics(led_grid=grid)
    circ = np.roll(synth.pupil_circle(h, optics), shift, axis=(0, 1))
    ab = np.roll(synth.pupil_aberration(h, optics, seed), shift, axis=(0, 1))
    P_true = torch.from_numpy((circ * np.exp(1j * ab)).astype(np.complex64)).cuda()
    P0 = torch.from_numpy(circ.astype(np.float32)).cuda()
    led = synth.led_indices(h, p, optics)[:n_leds]
    if past_edge:
        led = np.concatenate([led, np.array([[H // 2 - h // 3, H - h // 2]], np.int32)])
    led = led.astype(np.int32)
    S = torch.fft.fftshift(torch.fft.fft2(O_true))
    ar = torch.arange(h, device="cuda")
    I = []
    for kl, kt in led:
        sub = S.index_select(0, (int(kt) - 1 + ar) % H).index_select(1, (int(kl) - 1 + ar) % H)
        x = torch.fft.ifft2(torch.fft.ifftshift(sub * P_true)) / (p * p)
        I.append(x.real ** 2 + x.imag ** 2)
    del S
    I = torch.stack(I)
    counts = torch.poisson(I * (3e4 / float(I.max())), generator=g).clamp_(max=65535)
    counts = counts.to(torch.int32).to(torch.uint16)
    del I
    Y = tr.normalise_u16(counts)
    pert = torch.polar(torch.ones((H, H), device="cuda"), 0.3 * (_smooth(H, 6.0, g, True) - 0.5))
    O0 = (O_true * pert).contiguous()
    del pert
    return {"h": h, "p": p, "H": H, "O_true": O_true, "P_true": P_true, "P0": P0,
            "P0c": P0.to(torch.complex64), "led": led, "counts": counts, "Y": Y, "O0": O0}


def _engine_args(c):
    import torch
    stack = c["counts"].permute(1, 2, 0)                   # (h, h, L) MATLAB order
    ledt = torch.from_numpy(led_matlab(c["led"])).cuda()
    return stack, ledt


def _bar(e32):
    return max(TIGHT, 3 * e32)


@pytest.fixture(scope="module")
def full_case():
    import torch
    c = _case(2048, 8, 5, 5, seed=17, shift=(150, -90))
    yield c
    c.clear()
    torch.cuda.empty_cache()


@pytest.mark.parametrize("loss", ["isotropic", "anisotropic"])
def test_bench_size_gradients_vs_fp64(engine, full_case, loss):
    """fpm_batch_gradients at 2048² -> 16384² on uint16 frames (the bench's kernel
    instantiations: L1, the fused row pass <2048, u16>, the persistent column pass
    <2048>, the pupil gradient, stitch pass A, the 16384-point column and row passes),
    one batch of six LEDs with one crop past the spectrum edge, against FP64."""
    import torch
    from oracle import torch_ref as tr
    c = full_case
    H = c["H"]
    stack, ledt = _engine_args(c)
    # the engine normalises the uint16 frames itself; the checker's amplitudes are the
    # bit-identical single-precision values
    assert torch.equal(engine.normalise_stack(c["counts"]), c["Y"])
    dO, dP, loss_e = engine.batch_gradients(c["O0"], c["P_true"], stack, ledt, c["P0"], c["p"],
                                            loss=loss)
    ref = {}
    for ct in (torch.complex128, torch.complex64):
        S = torch.fft.fft2(c["O0"].to(ct))
        G, dPr, lr_ = tr.batch_gradients(S, c["P_true"].to(ct), c["Y"], c["led"], c["p"], loss)
        del S
        dOr = torch.fft.ifft2(G) * float(H * H)
        del G
        ref[ct] = (dOr, dPr, lr_)
    r64, r32 = ref[torch.complex128], ref[torch.complex64]
    e_o, e_p = tr.rel_err(dO, r64[0]), tr.rel_err(dP, r64[1])
    t_o, t_p = tr.rel_err(r32[0], r64[0]), tr.rel_err(r32[1], r64[1])
    print(f"{loss}: dO engine {e_o:.2e} twin {t_o:.2e}; dP engine {e_p:.2e} twin {t_p:.2e}")
    assert e_o < _bar(t_o), (e_o, t_o)
    assert e_p < _bar(t_p), (e_p, t_p)
    assert abs(loss_e - r64[2]) < 1e-5 * abs(r64[2]), (loss_e, r64[2])
    del ref, dO, dP
    torch.cuda.empty_cache()


def test_row_pass_cluster_sizes_are_bit_identical(engine, full_case, monkeypatch):
    """The fused row pass at h = 2048 in clusters of 2, 4 (default) and 8 CTAs: the same
    lines get the same arithmetic whatever the cluster holds (only the halo lines and the
    CTA count differ), so the gradients and the loss agree bit for bit."""
    import torch
    c = full_case
    stack, ledt = _engine_args(c)
    out = {}
    for cl in ("2", "4", "8"):
        monkeypatch.setenv("FPM_L23_CLUSTER", cl)
        out[cl] = engine.batch_gradients(c["O0"], c["P_true"], stack, ledt, c["P0"], c["p"],
                                         loss="anisotropic")
    monkeypatch.delenv("FPM_L23_CLUSTER")
    for cl in ("2", "8"):
        assert torch.equal(out[cl][0], out["4"][0]), cl
        assert torch.equal(out[cl][1], out["4"][1]), cl
        assert out[cl][2] == out["4"][2], cl
    del out
    torch.cuda.empty_cache()


@pytest.mark.parametrize("loss", ["isotropic", "anisotropic"])
def test_h1024_gradients_vs_fp64(engine, loss):
    """fpm_batch_gradients at 1024² -> 4096² (the fused row pass with 8 lines per CTA in
    2-CTA clusters, two CTAs per SM), one batch of six LEDs with one crop past the
    spectrum edge and an off-centre pupil support, against FP64 with the bars above."""
    import torch
    from oracle import torch_ref as tr
    c = _case(1024, 4, 5, 5, seed=23, shift=(-70, 40))
    H = c["H"]
    stack, ledt = _engine_args(c)
    dO, dP, loss_e = engine.batch_gradients(c["O0"], c["P_true"], stack, ledt, c["P0"], c["p"],
                                            loss=loss)
    ref = {}
    for ct in (torch.complex128, torch.complex64):
        S = torch.fft.fft2(c["O0"].to(ct))
        G, dPr, lr_ = tr.batch_gradients(S, c["P_true"].to(ct), c["Y"], c["led"], c["p"], loss)
        ref[ct] = (torch.fft.ifft2(G) * float(H * H), dPr, lr_)
    r64, r32 = ref[torch.complex128], ref[torch.complex64]
    e_o, e_p = tr.rel_err(dO, r64[0]), tr.rel_err(dP, r64[1])
    t_o, t_p = tr.rel_err(r32[0], r64[0]), tr.rel_err(r32[1], r64[1])
    print(f"{loss}: dO engine {e_o:.2e} twin {t_o:.2e}; dP engine {e_p:.2e} twin {t_p:.2e}")
    assert e_o < _bar(t_o), (e_o, t_o)
    assert e_p < _bar(t_p), (e_p, t_p)
    assert abs(loss_e - r64[2]) < 1e-5 * abs(r64[2]), (loss_e, r64[2])
    del ref, dO, dP, c
    torch.cuda.empty_cache()


@pytest.mark.parametrize("loss", ["isotropic", "anisotropic"])
def test_bench_size_solve_vs_fp64(engine, full_case, loss):
    """fpm_solve at 2048² -> 16384² on uint16 frames: two epochs of a 3 + 3 LED batch
    split (the column update pass with RMSprop and its bulk-copy prefetch, the next-box
    row pass, the pupil RMSprop + clamp, the box pruned to an off-centre pupil support,
    the epoch wrap), object / pupil / spectrum / loss against FP64."""
    import torch
    from oracle import torch_ref as tr
    c = full_case
    stack, ledt = _engine_args(c)
    opt = (1e-3, 0.999, 1e-4)
    r = engine.solve(c["O0"], c["P0c"], stack, ledt, c["P0"], c["p"], 2, 3, lr=opt[0],
                     beta=opt[1], eps=opt[2], loss=loss)
    ref = {}
    for ct in (torch.complex128, torch.complex64):
        ref[ct] = tr.cufpm_pure_v3(c["O0"], c["P0c"], c["Y"], c["led"], c["P0"], c["p"], 2, 3,
                                   opt=opt, ctype=ct, loss_kind=loss)
    r64, r32 = ref[torch.complex128], ref[torch.complex64]
    for k in ("object", "pupil", "spectrum"):
        e, t = tr.rel_err(r[k], r64[k]), tr.rel_err(r32[k], r64[k])
        print(f"{loss} {k}: engine {e:.2e} twin {t:.2e}")
        assert e < _bar(t), (k, e, t)
    np.testing.assert_allclose(np.asarray(r["loss"].cpu()), r64["loss"], rtol=1e-5)
    del ref, r
    torch.cuda.empty_cache()


def _truth_err(O, T):
    """min over complex scalars a of ||a O - T|| / ||T|| (torch, float64)."""
    import torch
    O = O.to(torch.complex128).reshape(-1)
    T = T.to(torch.complex128).reshape(-1)
    a = torch.vdot(O, T) / torch.vdot(O, O)
    return float(torch.linalg.vector_norm(a * O - T) / torch.linalg.vector_norm(T))


def test_512x361_end_to_end_vs_fp64(engine):
    """19 x 19 LEDs (361 frames) of 512² uint16 -> 4096², Zernike-aberrated
    pupil, LED batch 26, 10 epochs, lr 1e-3, beta 0.999 (seeded synthetic data with the
    optics of the 128² case scaled to the grid), against FP64 with the 128² case's criteria; the
    recovered pupil's error against the true pupil is reported."""
    import torch
    from fpm_b200 import synth
    from oracle import torch_ref as tr
    ds = synth.make_dataset(512, 8, 19, seed=2, aberration=True)
    opt = (1e-3, 0.999, 1e-4)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
    O0, P0c, P0 = dev(ds.O0), dev(ds.P0c), dev(ds.pupil0)
    raw = dev(ds.raw)                                           # (L, h, h)
    ledt = dev(led_matlab(ds.led_idx))
    r = engine.solve(O0, P0c, raw.permute(1, 2, 0), ledt, P0, 8, 10, 26, lr=opt[0],
                     beta=opt[1], eps=opt[2])
    Y = dev(ds.Y)
    assert torch.equal(tr.normalise_u16(raw), Y)
    r64 = tr.cufpm_pure_v3(O0, P0c, Y, ds.led_idx, P0, 8, 10, 26, opt=opt)
    r32 = tr.cufpm_pure_v3(O0, P0c, Y, ds.led_idx, P0, 8, 10, 26, opt=opt, ctype=torch.complex64)
    for k in ("object", "pupil", "spectrum"):
        e, t = tr.rel_err(r[k], r64[k]), tr.rel_err(r32[k], r64[k])
        print(f"512x361 {k}: engine-vs-fp64 {e:.3e}, fp32-twin-vs-fp64 {t:.3e}")
        assert e < max(5 * t, 3e-2), k
    loss = np.asarray(r["loss"].cpu())
    np.testing.assert_allclose(loss, r64["loss"], rtol=5e-3)
    assert np.all(np.diff(loss) < 0)
    T = dev(ds.object_true)
    q_e, q_64 = _truth_err(r["object"], T), _truth_err(r64["object"], T)
    Pt = dev(ds.pupil_true)
    p_e, p_64 = _truth_err(r["pupil"], Pt), _truth_err(r64["pupil"], Pt)
    print(f"512x361 vs truth: object engine {q_e:.4f} fp64 {q_64:.4f}; "
          f"pupil engine {p_e:.4f} fp64 {p_64:.4f}")
    assert abs(q_e - q_64) < 0.02 * q_64
    assert abs(p_e - p_64) < 0.02 * p_64
    del r, r64, r32
    torch.cuda.empty_cache()
