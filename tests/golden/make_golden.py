"""Generate the golden fixtures under tests/golden/.

    python tests/golden/make_golden.py            # tiny_fp64.npz (CPU, FP64 oracle)
    python tests/golden/make_golden.py --ref DIR   # ref_*.npz into DIR (needs a GPU and
                                                   # oracle/_ref/libcufpm_ref.so)

``--ref`` runs the reference's own v3 CUDA kernels (built from the reference
tree by oracle/build_ref.py) on seeded inputs and stores their outputs with a
tolerance: ten times the distance between the FP32 and the FP64 oracle on the
same case (floor 1e-5), i.e. the reference build must sit as close to the FP64
oracle as an FP32 implementation of the oracle does.
"""
from __future__ import annotations

import ctypes as C
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT / "fused-fourier-ptycho_b200"))
sys.path.insert(0, str(ROOT))

from fpm_b200 import synth  # noqa: E402
from oracle import fpm_oracle as orc  # noqa: E402


def tiny():
    ds = synth.make_dataset(32, 2, 3, seed=11, aberration=True)
    opt = (2e-3, 0.999, 1e-4)
    r = orc.cufpm_pure_v3(ds.O0, ds.P0c, ds.Y, ds.led_idx, ds.pupil0, 2, 2, 4, opt=opt,
                          dtype=np.float64, workers=1)
    np.savez_compressed(HERE / "tiny_fp64.npz", O0=ds.O0, P0c=ds.P0c, Y=ds.Y, led_idx=ds.led_idx,
                        P0=ds.pupil0, raw=ds.raw, pratio=2, epochs=2, batch=4, opt=np.array(opt),
                        object=r.object, pupil=r.pupil, spectrum=r.spectrum, loss=r.loss)


def _colmajor(a, dt):
    return np.asfortranarray(np.asarray(a, dt))


def _stack(Y):
    return np.ascontiguousarray(np.transpose(np.asarray(Y, np.float32), (0, 2, 1)))


def ref_lib():
    lib = C.CDLL(str(ROOT / "oracle" / "_ref" / "libcufpm_ref.so"))
    vp = C.c_void_p
    lib.ref_gradients.argtypes = [C.c_int] * 4 + [vp] * 6
    lib.ref_solve.argtypes = [C.c_int] * 6 + [C.c_float] * 3 + [vp] * 8
    return lib


def ref_gradients(lib, O, P, Y, led, pratio):
    h = P.shape[0]
    H = O.shape[0]
    L = Y.shape[0]
    Oc = _colmajor(O, np.complex64)
    Pc = _colmajor(P, np.complex64)
    Ys = _stack(Y)
    ledc = np.ascontiguousarray(np.asarray(led, np.int32))
    dO = np.empty((H, H), np.complex64, order="F")
    dP = np.empty((h, h), np.complex64, order="F")
    rc = lib.ref_gradients(h, H, L, pratio, Oc.ctypes.data, Pc.ctypes.data, Ys.ctypes.data,
                           ledc.ctypes.data, dO.ctypes.data, dP.ctypes.data)
    assert rc == 0, rc
    return dO, dP


def ref_solve(lib, O0, P0c, Y, led, P0, pratio, epochs, batch, opt):
    h = P0c.shape[0]
    H = O0.shape[0]
    L = Y.shape[0]
    O = np.empty((H, H), np.complex64, order="F")
    P = np.empty((h, h), np.complex64, order="F")
    ms = np.zeros(3, np.float32)
    # the converted inputs must stay referenced for the whole call: `.ctypes.data` of a
    # temporary is a dangling address once the temporary is collected
    ins = [_colmajor(O0, np.complex64), _colmajor(P0c, np.complex64), _stack(Y),
           np.ascontiguousarray(led, np.int32), _colmajor(P0, np.float32)]
    rc = lib.ref_solve(h, H, L, pratio, epochs, batch, opt[0], opt[1], opt[2],
                       *[a.ctypes.data for a in ins], O.ctypes.data, P.ctypes.data,
                       ms.ctypes.data)
    del ins
    assert rc == 0, rc
    return O, P, ms


def _wrap_case():
    """h 32, pratio 2, LED corners at and past the spectrum edge (crops wrap modulo H)."""
    rng = np.random.default_rng(4)
    h, p = 32, 2
    H = h * p
    O = (0.5 + 0.5 * rng.random((H, H)) * np.exp(1j * rng.random((H, H)))).astype(np.complex64)
    P = synth.pupil_circle(h, synth.Optics(led_grid=3)).astype(np.complex64)
    led = np.array([[1, 1], [H - 10, 3], [H, H], [40, H - 20], [7, 60], [H // 2, H // 2 + 5]],
                   np.int32)                                     # H = 64
    Y = rng.random((len(led), h, h)).astype(np.float32)
    return O, P, Y, led, p


def refs(outdir: Path):
    outdir.mkdir(parents=True, exist_ok=True)
    lib = ref_lib()
    cases = []
    for name, h, p, grid, seed in (("h32", 32, 4, 5, 5), ("h64", 64, 4, 5, 3)):
        ds = synth.make_dataset(h, p, grid, seed=seed, aberration=True)
        H = h * p
        rng = np.random.default_rng(seed + 1)
        O = (ds.O0 * np.exp(1j * 0.2 * rng.standard_normal((H, H)))).astype(np.complex64)
        cases.append((name, O, ds.pupil_true.astype(np.complex64), ds.Y, ds.led_idx, p))
    cases.append(("wrap",) + _wrap_case())
    for name, O, P, Y, led, p in cases:
        H = O.shape[0]
        dO, dP = ref_gradients(lib, O, P, Y, led, p)
        G64, dP64, _ = orc.batch_gradients(np.fft.fft2(O.astype(np.complex128)),
                                           P.astype(np.complex128), Y.astype(np.float64), led, p,
                                           np.float64, workers=1)
        dO64 = np.fft.ifft2(G64) * H * H
        G32, dP32, _ = orc.batch_gradients(np.fft.fft2(O).astype(np.complex64), P, Y, led, p,
                                           np.float32, workers=1)
        dO32 = np.fft.ifft2(G32).astype(np.complex64) * np.complex64(H * H)
        e32 = max(orc.rel_err(dO32, dO64), orc.rel_err(dP32, dP64))
        tol = max(10 * e32, 1e-5)
        e_ref = max(orc.rel_err(dO, dO64), orc.rel_err(dP, dP64))
        print(f"ref_gradients_{name}: ref-vs-fp64 {e_ref:.3e}  fp32-vs-fp64 {e32:.3e}  tol {tol:.3e}")
        np.savez_compressed(outdir / f"ref_gradients_{name}.npz", O=O, P=P, Y=Y, led_idx=led,
                            pratio=p, ref_dO=dO, ref_dP=dP, tol=tol, err_fp32=e32, err_ref=e_ref)
    # short solves on noiseless amplitudes (no ties: FP32 trajectories stay close to FP64)
    ds = synth.make_dataset(32, 4, 5, seed=5, aberration=True)
    spec = np.fft.fftshift(np.fft.fft2(ds.object_true)).astype(np.complex64)
    I = synth.forward_intensity(spec, ds.pupil_true, ds.led_idx, 4)
    Y = np.sqrt(I / I.max()).astype(np.float32)
    O0 = synth.upsample_bicubic(Y[0], 4).astype(np.float32).astype(np.complex64)
    opt = (1e-3, 0.999, 1e-4)
    for L, E, B in ((8, 1, 8), (16, 1, 8), (25, 2, 8)):
        O, P, ms = ref_solve(lib, O0, ds.P0c, Y[:L], ds.led_idx[:L], ds.pupil0, 4, E, B, opt)
        r64 = orc.cufpm_pure_v3(O0, ds.P0c, Y[:L], ds.led_idx[:L], ds.pupil0, 4, E, B, opt=opt,
                                dtype=np.float64, workers=1)
        r32 = orc.cufpm_pure_v3(O0, ds.P0c, Y[:L], ds.led_idx[:L], ds.pupil0, 4, E, B, opt=opt,
                                dtype=np.float32, workers=1)
        e32 = max(orc.rel_err(r32.object, r64.object), orc.rel_err(r32.pupil, r64.pupil))
        tol = max(10 * e32, 1e-5)
        out = ds.pupil0 == 0
        e_o = orc.rel_err(O, r64.object)
        e_p_in = orc.rel_err(np.where(out, 0, P), np.where(out, 0, r64.pupil))
        print(f"ref_solve L{L} E{E}: object {e_o:.3e} pupil-inside {e_p_in:.3e} "
              f"max|P| outside support {np.abs(P[out]).max():.3e} at {np.unravel_index(np.argmax(np.abs(np.where(out, P, 0))), P.shape)} "
              f"fp32-vs-fp64 {e32:.3e} ms {ms}")
        np.savez_compressed(outdir / f"ref_solve_L{L}.npz", O0=O0, P0c=ds.P0c, Y=Y[:L],
                            led_idx=ds.led_idx[:L], P0=ds.pupil0, pratio=4, epochs=E, batch=B,
                            opt=np.array(opt), ref_object=O, ref_pupil=P, tol=tol, err_fp32=e32)


if __name__ == "__main__":
    if "--ref" in sys.argv:
        refs(Path(sys.argv[sys.argv.index("--ref") + 1]))
    else:
        tiny()
