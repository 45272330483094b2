"""The MATLAB optimiser classes of the reference's script-level loop
(optimizer_RMSprop.m, optimizer_adam.m, optimizer_yogi.m, optimizer_sgd.m) and its
pupil clamp (benchmark/cuFPM_recon_2025_circular.m:180-186).

CPU: the oracle's restatements against literal complex128 transcriptions of the
MATLAB statements (to float32 rounding) and their defining properties.  GPU: every
kind and variant through fpm_optimizer_step over several steps, numpy (host) and
torch (device) memory, bit-exact against the oracle (both do one rounding per MATLAB
operation and the correctly rounded abs); a mini-batch of the script-level loop
(gradients, both steps, clamp) against the oracle's steps on the same gradients.
"""
import numpy as np
import pytest

from conftest import has_gpu, dataset, led_matlab, to_matlab_stack

from oracle import fpm_oracle as orc


def crandn(g, shape, scale=1.0):
    return ((g.standard_normal(shape) + 1j * g.standard_normal(shape)) * scale).astype(np.complex64)


# ---------------------------------------------------------------------------
# oracle (CPU)
# ---------------------------------------------------------------------------

def test_oracle_steps_match_matlab_statements_in_double():
    """The float32 restatements agree with the MATLAB statements evaluated in double."""
    g = np.random.default_rng(0)
    p, gr = crandn(g, (64, 48)), crandn(g, (64, 48), 0.3)
    m1, m2 = crandn(g, (64, 48), 0.1), np.abs(g.standard_normal((64, 48))).astype(np.float32)
    r1, r2, lr, it = 0.9, 0.999, 1.5e-3, 3
    P, M1, M2 = orc.adam_class_step(p, gr, m1, m2, r1, r2, lr, it)
    gd, md1, md2 = gr.astype(complex), r1 * m1 + (1 - r1) * gr, r2 * m2 + (1 - r2) * np.abs(gr) ** 2
    Pd = p - lr * (np.sqrt(1 - r2 ** it) / (1 - r1 ** it)) * md1 / (np.sqrt(md2) + 1e-5)
    np.testing.assert_allclose(M1, md1, rtol=1e-6, atol=1e-7)
    np.testing.assert_allclose(M2, md2, rtol=1e-6)
    np.testing.assert_allclose(P, Pd, rtol=1e-6, atol=1e-6)
    P, M1, M2 = orc.yogi_class_step(p, gr, m1, m2, r1, r2, lr)
    md2 = m2 - (1 - r2) * np.sign(m2 - np.abs(gd) ** 2) * np.abs(gd) ** 2
    np.testing.assert_allclose(M2, md2, rtol=1e-6)
    np.testing.assert_allclose(P, p - lr * md1 / (np.sqrt(md2) + 1e-5), rtol=1e-6, atol=1e-6)
    g0, buf = crandn(g, (64, 48), 1.0), crandn(g, (64, 48), 0.1)   # |g0| ~ 1: squave of both signs
    P, G0, B = orc.rmsprop_class_step(p, gr, 0.999, 0.5, True, lr, g0, buf)
    sq = 0.999 + 0.001 * np.abs(gd) ** 2
    g0d = 0.999 * g0 + 0.001 * gd
    sq = sq - np.abs(g0d) ** 2
    root = np.sqrt(sq.astype(complex))          # MATLAB: complex root of a negative squave
    bd = 0.5 * buf + gd / (root + 1e-5)
    np.testing.assert_allclose(G0, g0d, rtol=1e-6, atol=1e-7)
    ok = np.abs(sq) > 1e-2          # squave = 0.999 + ... - |g0|^2 cancels near 0: ill-conditioned
    np.testing.assert_allclose(B[ok], bd[ok], rtol=1e-5, atol=1e-6)
    np.testing.assert_allclose(P[ok], (p - lr * bd)[ok], rtol=1e-6, atol=1e-6)
    assert (sq < 0).any() and (sq > 0).any()     # both branches of the root
    amp = np.abs(g.standard_normal((64, 48))).astype(np.float32)
    amp[:5] = 0
    Pc = orc.clamp_pupil_script(p, amp, 0.1)
    w = np.abs(p.astype(complex))
    want = np.maximum(np.minimum(w, amp + 0.1), amp - 0.1) * (p / w) * amp
    np.testing.assert_allclose(Pc, want, rtol=1e-6, atol=1e-7)
    assert not Pc[:5].any()


def test_oracle_properties():
    g = np.random.default_rng(1)
    p, gr = crandn(g, (32, 32)), crandn(g, (32, 32))
    # RMSprop as written: squave is rebuilt from r1 each step, so with the same gradient
    # two steps move the parameter by the same amount
    p1, _, _ = orc.rmsprop_class_step(p, gr, 0.999, 0, False, 1e-2)
    p2, _, _ = orc.rmsprop_class_step(p1, gr, 0.999, 0, False, 1e-2)
    np.testing.assert_allclose(p2 - p1, p1 - p, rtol=1e-4, atol=1e-6)
    # Yogi: sign(0) = 0 keeps a zero second moment at zero gradient
    z = np.zeros((4, 4), np.complex64)
    _, _, m2 = orc.yogi_class_step(z, z, z, np.zeros((4, 4), np.float32), 0.9, 0.999, 1e-2)
    assert not m2.any()
    # SGD moves against the gradient
    np.testing.assert_array_equal(orc.sgd_step(p, gr, 0.0), p)


# ---------------------------------------------------------------------------
# device (GPU)
# ---------------------------------------------------------------------------

def _steps_numpy(kind, n_steps, shape, clamp, **kw):
    from fpm_b200 import optimizers as O
    g = np.random.default_rng(7)
    p = crandn(g, shape)
    grads = [crandn(g, shape, 0.2 * (k + 1)) for k in range(n_steps)]
    amp = np.abs(g.standard_normal(shape)).astype(np.float32)
    amp[: shape[0] // 8] = 0
    c = (amp, 0.1) if clamp else None
    dev = {"sgd": lambda: O.optimizer_sgd(kw["lr"]),
           "rmsprop": lambda: O.optimizer_RMSprop(0, 0, kw["r1"], kw["mum"], kw["centered"], kw["lr"]),
           "adam": lambda: O.optimizer_adam(0, 0, kw["r1"], kw["r2"], kw["lr"]),
           "yogi": lambda: O.optimizer_yogi(0, 0, kw["r1"], kw["r2"], kw["lr"])}[kind]()
    ref_p = p.copy()
    z, zr = np.zeros(shape, np.complex64), np.zeros(shape, np.float32)
    s1, s2, s3 = z.copy(), zr.copy(), z.copy()
    got = p
    for k, gk in enumerate(grads):
        got = dev.step(got, gk, iter=k + 1, clamp=c) if kind == "adam" else dev.step(got, gk, clamp=c)
        if kind == "sgd":
            ref_p = orc.sgd_step(ref_p, gk, kw["lr"])
        elif kind == "rmsprop":
            ref_p, s1, s3 = orc.rmsprop_class_step(ref_p, gk, kw["r1"], kw["mum"], kw["centered"],
                                                   kw["lr"], s1, s3)
        elif kind == "adam":
            ref_p, s1, s2 = orc.adam_class_step(ref_p, gk, s1, s2, kw["r1"], kw["r2"], kw["lr"], k + 1)
        else:
            ref_p, s1, s2 = orc.yogi_class_step(ref_p, gk, s1, s2, kw["r1"], kw["r2"], kw["lr"])
        if clamp:
            ref_p = orc.clamp_pupil_script(ref_p, amp, 0.1)
    return got, ref_p


CASES = [("sgd", dict(lr=3e-2)),
         ("rmsprop", dict(r1=0.999, mum=0, centered=False, lr=1.5e-3)),   # the reference's use
         ("rmsprop", dict(r1=0.9, mum=0.5, centered=True, lr=1e-2)),
         ("adam", dict(r1=0.9, r2=0.999, lr=1e-2)),
         ("yogi", dict(r1=0.9, r2=0.999, lr=1e-2))]


@pytest.mark.gpu
@pytest.mark.parametrize("clamp", [False, True])
@pytest.mark.parametrize("kind,kw", CASES)
def test_optimizer_steps_bit_exact(engine, kind, kw, clamp):
    got, ref = _steps_numpy(kind, 3, (96, 80), clamp, **kw)
    np.testing.assert_array_equal(got, ref)


@pytest.mark.gpu
def test_optimizer_device_memory_in_place(engine):
    import torch
    from fpm_b200 import optimizers as O
    g = np.random.default_rng(9)
    p, gr = crandn(g, (128, 64)), crandn(g, (128, 64))
    opt_h, opt_d = O.optimizer_yogi(0, 0, 0.9, 0.999, 1e-2), O.optimizer_yogi(0, 0, 0.9, 0.999, 1e-2)
    ph = p
    pd = torch.from_numpy(p.copy()).cuda()
    for _ in range(2):
        ph = opt_h.step(ph, gr)
        out = opt_d.step(pd, torch.from_numpy(gr).cuda())
        assert out.data_ptr() == pd.data_ptr()            # updated in place
    np.testing.assert_array_equal(pd.cpu().numpy(), ph)
    np.testing.assert_array_equal(opt_d.mom2.cpu().numpy(), opt_h.mom2)


@pytest.mark.gpu
def test_optimizer_refusals(engine):
    from fpm_b200 import api
    p = np.zeros(16, np.complex64)
    for opt, what in ((api.Optimizer(kind=api.OPT_ADAM, lr=1e-2, beta1=0.9, beta2=0.999, iter=1),
                       "mom1 and mom2"),
                      (api.Optimizer(kind=9), "kind"),
                      (api.Optimizer(kind=api.OPT_RMSPROP, centered=1, beta1=0.9), "g0"),
                      (api.Optimizer(kind=api.OPT_SGD, lr=float("nan")), "non-finite")):
        with pytest.raises(api.FpmError) as e:
            engine.optimizer_step(opt, p, p.copy())
        assert e.value.status == 1 and what in e.value.detail
    m1, m2 = np.zeros(16, np.complex64), np.zeros(16, np.float32)
    opt = api.Optimizer(kind=api.OPT_ADAM, lr=1e-2, beta1=0.9, beta2=0.999, iter=0,
                        mom1=m1.ctypes.data, mom2=m2.ctypes.data)
    with pytest.raises(api.FpmError) as e:
        engine.optimizer_step(opt, p, p.copy())
    assert "iter" in e.value.detail


@pytest.mark.gpu
def test_script_loop_minibatch(engine):
    """One mini-batch of the script-level loop (cuFPM_recon_2025_circular.m:165-186):
    fullyfusedFPM gradients, RMSprop steps on object and pupil, pupil clamp; the device
    steps equal the oracle's steps applied to the same gradients."""
    from fpm_b200 import optimizers as O
    ds = dataset(64, 4, 5, seed=3, aberration=True)
    L = 8
    O0 = np.asarray(ds.O0, np.complex64)
    P0c = np.asarray(ds.P0c, np.complex64)
    amp = np.asarray(ds.pupil0, np.float32)
    Y = to_matlab_stack(ds.raw[:L])
    led = led_matlab(ds.led_idx[:L])
    dO, dP, _ = engine.batch_gradients(O0, P0c, Y, led, amp, 4)
    o1 = O.optimizer_RMSprop(0, 0, 0.999, 0, False, 1.5e-3)
    o2 = O.optimizer_RMSprop(0, 0, 0.999, 0, False, 1.5e-3)
    w1 = o1.step(O0, dO)
    w2 = o2.step(P0c, dP, clamp=(amp, 0.1))
    r1, _, _ = orc.rmsprop_class_step(O0, dO, 0.999, 0, False, 1.5e-3)
    r2, _, _ = orc.rmsprop_class_step(P0c, dP, 0.999, 0, False, 1.5e-3)
    r2 = orc.clamp_pupil_script(r2, amp, 0.1)
    np.testing.assert_array_equal(w1, r1)
    np.testing.assert_array_equal(w2, r2)
    assert not w2[amp == 0].any()
