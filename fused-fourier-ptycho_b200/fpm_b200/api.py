"""ctypes binding of libfpm (include/fpm.h) and the Python mirror of the reference call.

The mirror keeps the reference mex's argument list and MATLAB array shapes:

    O, P = cuFPM_pure_v3(O0, P0c, Y, ledIdx, P0, pratio, epochs, B, [lr, beta, eps])

(``cuFPM_v3/cuFPM_pure_v3.cu:44-66``, call site ``codes_v2/main_run_FPM.m:98-106``)
with ``O0`` complex H x H, ``P0c`` complex h x h, ``Y`` h x h x L (float32
amplitude as the mex takes, or uint16 counts), ``ledIdx`` int32 2 x L
(``[kl; kt]``), ``P0`` real h x h.  Arrays may be numpy arrays (host memory,
copied by the engine) or torch CUDA tensors (device memory, used in place);
their index order is MATLAB's, and they are handed to the C ABI in
column-major memory order (numpy Fortran order; for torch, dimensions
reversed and made contiguous, which is free for tensors already laid out so).

There is no CPU path: without the built library or a CUDA device every compute
call raises.  Only the frame reader (``read_tiff_stack``) is host code by nature.
"""
from __future__ import annotations

import ctypes as C
import os
import weakref
from pathlib import Path

import numpy as np

_LIB_PATH = Path(__file__).resolve().parent / "_lib" / "libfpm.so"

FPM_OK = 0
STATUS_NAMES = {0: "FPM_OK", 1: "FPM_ERR_INVALID_ARGUMENT", 2: "FPM_ERR_UNSUPPORTED",
                3: "FPM_ERR_OUT_OF_MEMORY", 4: "FPM_ERR_CUDA", 5: "FPM_ERR_NONFINITE",
                6: "FPM_ERR_NO_DEVICE", 7: "FPM_ERR_INTERNAL"}
MEM_HOST, MEM_DEVICE = 0, 1
FPM_CTX_AUTOTUNE = 1
STACK_F32, STACK_U16 = 0, 1
LOSS_ANISOTROPIC, LOSS_ISOTROPIC = 0, 1
_LOSS = {"anisotropic": LOSS_ANISOTROPIC, "isotropic": LOSS_ISOTROPIC}
PIE_NONE, PIE_EPIE, PIE_TPIE = 0, 1, 2
_PIE = {"none": PIE_NONE, "ePIE": PIE_EPIE, "tPIE": PIE_TPIE}

# Every symbol include/fpm.h declares.
EXPORTED = ["fpm_create", "fpm_solve", "fpm_batch_gradients", "fpm_normalise_stack",
            "fpm_destroy", "fpm_set_profiling", "fpm_stage_times", "fpm_status_string",
            "fpm_last_error", "fpm_abi_version", "fpm_feature_gradient_noalloc", "fpm_fft2",
            "fpm_led_indices", "fpm_simulate", "fpm_normalise_stack_f32", "fpm_read_tiff_stack",
            "fpm_optimizer_step", "fpm_solve_batch", "fpm_autotune",
            "fpm_selftest_bounded_wait", "fpm_cnn_create", "fpm_cnn_destroy",
            "fpm_cnn_parameter_count", "fpm_cnn_last_error", "fpm_cnn_set_parameters",
            "fpm_cnn_get_parameters", "fpm_cnn_forward", "fpm_cnn_gradients",
            "fpm_cnn_train_step", "fpm_cnn_initial_object", "fpm_solve_warm"]


SIM_INTENSITY, SIM_AMPLITUDE = 0, 1
INGEST_U16, INGEST_F32_MEAN = 0, 1
OPT_RMSPROP, OPT_ADAM, OPT_YOGI, OPT_SGD = 0, 1, 2, 3


class FpmError(RuntimeError):
    def __init__(self, status: int, detail: str):
        self.status = status
        self.detail = detail
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {detail}")


class DeviceOpts(C.Structure):
    _fields_ = [("device", C.c_int32), ("flags", C.c_int32),
                ("mem_limit_bytes", C.c_size_t), ("stream", C.c_void_p)]


class LedGeometry(C.Structure):
    """fpm_led_geometry (include/fpm.h); lengths in micrometres."""
    _fields_ = [("grid", C.c_int32), ("h", C.c_int32), ("pratio", C.c_int32),
                ("reserved0", C.c_int32), ("wavelength_um", C.c_double),
                ("led_pitch_um", C.c_double), ("led_height_um", C.c_double),
                ("camera_pixel_um", C.c_double), ("magnification", C.c_double),
                ("sample_dx_um", C.c_double), ("sample_dy_um", C.c_double)]


class Optimizer(C.Structure):
    """fpm_optimizer (include/fpm.h)."""
    _fields_ = [("kind", C.c_int32), ("centered", C.c_int32), ("lr", C.c_double),
                ("beta1", C.c_double), ("beta2", C.c_double), ("momentum", C.c_double),
                ("iter", C.c_int64), ("mom1", C.c_void_p), ("mom2", C.c_void_p),
                ("buffer", C.c_void_p), ("clamp_amp", C.c_void_p), ("clamp_margin", C.c_double)]


class Problem(C.Structure):
    _fields_ = [("h", C.c_int32), ("n_leds", C.c_int32), ("pratio", C.c_int32),
                ("batch", C.c_int32), ("epochs", C.c_int32),
                ("lr", C.c_float), ("beta", C.c_float), ("eps", C.c_float),
                ("pupil_margin", C.c_float), ("lr_halve_after", C.c_int32),
                ("lr_decay", C.c_float), ("loss_kind", C.c_int32), ("memory", C.c_int32),
                ("stack_type", C.c_int32),
                ("stack", C.c_void_p), ("led_idx", C.c_void_p), ("pupil_init", C.c_void_p),
                ("pupil_amp", C.c_void_p), ("object_init", C.c_void_p),
                ("pie_weights", C.c_int32), ("reserved0", C.c_int32)]


class StageTime(C.Structure):
    _fields_ = [("name", C.c_char_p), ("launches", C.c_int32), ("own_kernel", C.c_int32),
                ("ms", C.c_double)]


class Result(C.Structure):
    _fields_ = [("object", C.c_void_p), ("spectrum", C.c_void_p), ("pupil", C.c_void_p),
                ("loss", C.c_void_p)]


_lib = None


def load_library(path: str | Path | None = None):
    """Load libfpm.so (built in-tree by ``fpm_b200._build.build``); raises if absent."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else _LIB_PATH
    if not p.exists():
        raise ImportError(f"libfpm.so not built at {p}; run __graft_entry__.build()")
    lib = C.CDLL(str(p))
    lib.fpm_create.argtypes = [C.POINTER(C.c_void_p), C.POINTER(DeviceOpts)]
    lib.fpm_create.restype = C.c_int
    lib.fpm_solve.argtypes = [C.c_void_p, C.POINTER(Problem), C.POINTER(Result)]
    lib.fpm_solve.restype = C.c_int
    lib.fpm_solve_batch.argtypes = [C.c_void_p, C.POINTER(Problem), C.POINTER(Result), C.c_int32,
                                    C.c_int32, C.c_void_p]
    lib.fpm_solve_batch.restype = C.c_int
    lib.fpm_autotune.argtypes = [C.c_void_p, C.POINTER(Problem), C.c_char_p, C.c_size_t]
    lib.fpm_autotune.restype = C.c_int
    lib.fpm_selftest_bounded_wait.argtypes = [C.c_void_p, C.c_int64]
    lib.fpm_selftest_bounded_wait.restype = C.c_int
    vp = C.c_void_p
    lib.fpm_cnn_create.argtypes = [vp, C.c_int32, C.c_int32, C.c_uint64, C.POINTER(vp)]
    lib.fpm_cnn_create.restype = C.c_int
    lib.fpm_cnn_destroy.argtypes = [vp]
    lib.fpm_cnn_destroy.restype = None
    lib.fpm_cnn_parameter_count.argtypes = [vp]
    lib.fpm_cnn_parameter_count.restype = C.c_int64
    lib.fpm_cnn_last_error.argtypes = [vp]
    lib.fpm_cnn_last_error.restype = C.c_char_p
    lib.fpm_cnn_set_parameters.argtypes = [vp, vp, C.c_int64]
    lib.fpm_cnn_set_parameters.restype = C.c_int
    lib.fpm_cnn_get_parameters.argtypes = [vp, vp, C.c_int64]
    lib.fpm_cnn_get_parameters.restype = C.c_int
    lib.fpm_cnn_forward.argtypes = [vp, vp, C.c_int32, C.c_int32, vp]
    lib.fpm_cnn_forward.restype = C.c_int
    lib.fpm_cnn_gradients.argtypes = [vp, vp, vp, C.c_int32, C.c_int32, C.POINTER(C.c_double), vp]
    lib.fpm_cnn_gradients.restype = C.c_int
    lib.fpm_cnn_train_step.argtypes = [vp, vp, vp, C.c_int32, C.c_int32, C.c_float,
                                       C.POINTER(C.c_double)]
    lib.fpm_cnn_train_step.restype = C.c_int
    lib.fpm_cnn_initial_object.argtypes = [vp, C.POINTER(Problem), vp]
    lib.fpm_cnn_initial_object.restype = C.c_int
    lib.fpm_solve_warm.argtypes = [vp, vp, C.POINTER(Problem), C.POINTER(Result),
                                   C.POINTER(C.c_int32)]
    lib.fpm_solve_warm.restype = C.c_int
    lib.fpm_batch_gradients.argtypes = [C.c_void_p, C.POINTER(Problem), C.c_void_p, C.c_void_p,
                                        C.c_void_p]
    lib.fpm_batch_gradients.restype = C.c_int
    lib.fpm_normalise_stack.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p, C.c_int32]
    lib.fpm_normalise_stack.restype = C.c_int
    lib.fpm_destroy.argtypes = [C.c_void_p]
    lib.fpm_destroy.restype = None
    lib.fpm_status_string.argtypes = [C.c_int]
    lib.fpm_status_string.restype = C.c_char_p
    lib.fpm_last_error.argtypes = [C.c_void_p]
    lib.fpm_last_error.restype = C.c_char_p
    lib.fpm_set_profiling.argtypes = [C.c_void_p, C.c_int32]
    lib.fpm_set_profiling.restype = C.c_int
    lib.fpm_stage_times.argtypes = [C.c_void_p, C.POINTER(StageTime), C.c_int32]
    lib.fpm_stage_times.restype = C.c_int32
    lib.fpm_fft2.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_int32,
                             C.c_int32]
    lib.fpm_fft2.restype = C.c_int
    lib.fpm_led_indices.argtypes = [C.c_void_p, C.POINTER(LedGeometry), C.c_void_p, C.c_void_p]
    lib.fpm_led_indices.restype = C.c_int
    lib.fpm_simulate.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32,
                                 C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_int32]
    lib.fpm_simulate.restype = C.c_int
    lib.fpm_normalise_stack_f32.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p,
                                            C.c_int32]
    lib.fpm_normalise_stack_f32.restype = C.c_int
    lib.fpm_read_tiff_stack.argtypes = [C.c_void_p, C.POINTER(C.c_char_p), C.c_int32, C.c_int32,
                                        C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_int32]
    lib.fpm_read_tiff_stack.restype = C.c_int
    lib.fpm_optimizer_step.argtypes = [C.c_void_p, C.POINTER(Optimizer), C.c_void_p, C.c_void_p,
                                       C.c_size_t, C.c_int32]
    lib.fpm_optimizer_step.restype = C.c_int
    lib.fpm_abi_version.argtypes = []
    lib.fpm_abi_version.restype = C.c_int32
    if path is None:
        _lib = lib
    return lib


# ---------------------------------------------------------------------------
# array marshalling (MATLAB index order <-> column-major memory)
# ---------------------------------------------------------------------------

def _is_torch(x) -> bool:
    return type(x).__module__.startswith("torch")


def _inputs_ready(*xs):
    """Wait for the torch work that produced CUDA tensor inputs (copies made by the
    layout helpers included): the library runs on its own stream, which orders itself
    after the legacy default stream only, not after a torch side stream."""
    import torch
    for x in xs:
        if _is_torch(x) and x.is_cuda:
            torch.cuda.current_stream(x.device).synchronize()
            return


def _colmajor(x, dtype):
    """(pointer, keep-alive object, memory kind) of x in column-major memory."""
    if _is_torch(x):
        import torch
        tdt = {np.complex64: torch.complex64, np.float32: torch.float32,
               np.uint16: torch.uint16, np.int32: torch.int32}[dtype]
        if x.dtype != tdt:
            raise TypeError(f"expected {tdt}, got {x.dtype}")
        y = x.permute(*reversed(range(x.dim()))).contiguous()
        mem = MEM_DEVICE if y.is_cuda else MEM_HOST
        return y.data_ptr(), y, mem
    a = np.asfortranarray(np.asarray(x, dtype=dtype))
    return a.ctypes.data, a, MEM_HOST


def _empty_like_layout(shape, dtype, device_tensor_like):
    """Output buffer whose MATLAB-order view is returned and whose memory is column-major."""
    if device_tensor_like is not None:
        import torch
        tdt = {np.complex64: torch.complex64, np.float64: torch.float64}[dtype]
        base = torch.empty(tuple(reversed(shape)), dtype=tdt, device=device_tensor_like.device)
        return base.data_ptr(), base.permute(*reversed(range(len(shape))))
    a = np.empty(shape, dtype=dtype, order="F")
    return a.ctypes.data, a


class Engine:
    """One libfpm context (one CUDA device, one stream; not thread-safe)."""

    def __init__(self, device: int = 0, mem_limit_bytes: int = 0, stream: int | None = None,
                 autotune: bool = False):
        self.lib = load_library()
        self._ctx = C.c_void_p()
        opts = DeviceOpts(device, FPM_CTX_AUTOTUNE if autotune else 0, mem_limit_bytes,
                          stream or None)
        # objects that hold library state on this context (warm-start networks), closed
        # before the context is
        self._children = weakref.WeakSet()
        st = self.lib.fpm_create(C.byref(self._ctx), C.byref(opts))
        if st != FPM_OK:
            raise FpmError(st, self.lib.fpm_status_string(st).decode())

    def close(self):
        for ch in list(getattr(self, "_children", ())):
            ch.close()
        if self._ctx:
            self.lib.fpm_destroy(self._ctx)
            self._ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, st: int):
        if st != FPM_OK:
            detail = self.lib.fpm_last_error(self._ctx).decode()
            raise FpmError(st, detail)

    def set_profiling(self, on: bool):
        self._check(self.lib.fpm_set_profiling(self._ctx, 1 if on else 0))

    def stage_times(self):
        """{stage: (launches, summed device ms, own kernel?)} of the last call."""
        n = self.lib.fpm_stage_times(self._ctx, None, 0)
        arr = (StageTime * max(n, 1))()
        n = self.lib.fpm_stage_times(self._ctx, arr, n)
        return {arr[i].name.decode(): (arr[i].launches, arr[i].ms, bool(arr[i].own_kernel))
                for i in range(n)}

    # -- raw entry points (pointers already laid out) --------------------------
    def solve_raw(self, prob: Problem, res: Result) -> int:
        return self.lib.fpm_solve(self._ctx, C.byref(prob), C.byref(res))

    def gradients_raw(self, prob: Problem, d_obj, d_pup, loss) -> int:
        return self.lib.fpm_batch_gradients(self._ctx, C.byref(prob), d_obj, d_pup, loss)

    # -- MATLAB-shaped entry points --------------------------------------------
    def _problem(self, O0, P0c, Y, led_idx, P0, pratio, epochs, batch, lr, beta, eps, am,
                 lr_halve_after, lr_decay, loss="anisotropic", pie="none"):
        keep = []
        y_is_u16 = (str(getattr(Y, "dtype", "")).endswith("uint16"))
        ydt = np.uint16 if y_is_u16 else np.float32
        ys, yk, ymem = _colmajor(Y, ydt)
        keep.append(yk)
        ls, lk, lmem = _colmajor(led_idx, np.int32)
        keep.append(lk)
        ps, pk, pmem = _colmajor(P0c, np.complex64)
        keep.append(pk)
        as_, ak, amem = _colmajor(P0, np.float32)
        keep.append(ak)
        os_ = None
        omem = ymem
        if O0 is not None:
            os_, ok, omem = _colmajor(O0, np.complex64)
            keep.append(ok)
        if len({ymem, lmem, pmem, amem, omem}) != 1:
            raise ValueError("all inputs must live in the same memory (host or one CUDA device)")
        shp = tuple(Y.shape)
        h = int(shp[0])
        L = int(shp[2]) if len(shp) == 3 else 1
        prob = Problem(h=h, n_leds=L, pratio=int(pratio), batch=int(batch), epochs=int(epochs),
                       lr=lr, beta=beta, eps=eps, pupil_margin=am, lr_halve_after=lr_halve_after,
                       lr_decay=lr_decay, loss_kind=_LOSS[loss], memory=ymem,
                       stack_type=STACK_U16 if y_is_u16 else STACK_F32, stack=ys, led_idx=ls,
                       pupil_init=ps, pupil_amp=as_, object_init=os_, pie_weights=_PIE[pie])
        return prob, keep, ymem

    def solve(self, O0, P0c, Y, led_idx, P0, pratio, epochs, batch, lr=5e-4, beta=0.999,
              eps=1e-4, am=0.2, lr_halve_after=12, lr_decay=0.5, spectrum=True,
              loss="anisotropic", pie="none"):
        """Full reconstruction; returns dict(object, pupil, spectrum, loss) in MATLAB order.
        loss: "anisotropic" (the v3 mex) or "isotropic" (ret_loss.m); pie: "none" (the v3
        mex), "ePIE" or "tPIE" (the deconv_pie weights of fpm_forward_GPU.m)."""
        prob, keep, mem = self._problem(O0, P0c, Y, led_idx, P0, pratio, epochs, batch, lr,
                                        beta, eps, am, lr_halve_after, lr_decay, loss, pie)
        h = prob.h
        H = h * prob.pratio
        like = Y if mem == MEM_DEVICE else None
        op, o = _empty_like_layout((H, H), np.complex64, like)
        pp, p = _empty_like_layout((h, h), np.complex64, like)
        sp, s = (None, None)
        if spectrum:
            sp, s = _empty_like_layout((H, H), np.complex64, like)
        lp, loss = _empty_like_layout((max(int(epochs), 1),), np.float64, like)
        res = Result(object=op, spectrum=sp, pupil=pp, loss=lp)
        _inputs_ready(*keep)
        self._check(self.solve_raw(prob, res))
        del keep
        return {"object": o, "pupil": p, "spectrum": s, "loss": loss[: int(epochs)]}

    def solve_batch(self, instances, eager=False, spectrum=False):
        """Many independent reconstructions in one fpm_solve_batch call.  instances: a list
        of dicts with the arguments of solve (O0, P0c, Y, led_idx, P0, pratio, epochs, batch
        and optionally lr, beta, eps, am, lr_halve_after, lr_decay, loss, pie); returns
        (results, statuses) with one solve-style dict per instance."""
        n = len(instances)
        probs = (Problem * n)()
        ress = (Result * n)()
        keep, outs = [], []
        for i, a in enumerate(instances):
            kw = dict(lr=5e-4, beta=0.999, eps=1e-4, am=0.2, lr_halve_after=12, lr_decay=0.5,
                      loss="anisotropic", pie="none")
            kw.update({k: a[k] for k in kw if k in a})
            prob, kp, mem = self._problem(a["O0"], a["P0c"], a["Y"], a["led_idx"], a["P0"],
                                          a["pratio"], a["epochs"], a["batch"], kw["lr"],
                                          kw["beta"], kw["eps"], kw["am"], kw["lr_halve_after"],
                                          kw["lr_decay"], kw["loss"], kw["pie"])
            keep.append(kp)
            h = prob.h
            H = h * prob.pratio
            like = a["Y"] if mem == MEM_DEVICE else None
            op, o = _empty_like_layout((H, H), np.complex64, like)
            pp, pu = _empty_like_layout((h, h), np.complex64, like)
            sp, sv = (None, None)
            if spectrum:
                sp, sv = _empty_like_layout((H, H), np.complex64, like)
            lp, lo = _empty_like_layout((max(int(a["epochs"]), 1),), np.float64, like)
            probs[i] = prob
            ress[i] = Result(object=op, spectrum=sp, pupil=pp, loss=lp)
            outs.append({"object": o, "pupil": pu, "spectrum": sv,
                         "loss": lo[: int(a["epochs"])]})
        st = (C.c_int * n)()
        _inputs_ready(*[x for kp in keep for x in kp])
        rc = self.lib.fpm_solve_batch(self._ctx, probs, ress, n, 1 if eager else 0, st)
        statuses = [int(x) for x in st]
        if rc != FPM_OK and all(x != FPM_OK for x in statuses):
            self._check(rc)
        del keep
        return outs, statuses

    def autotune(self, O0, P0c, Y, led_idx, P0, pratio, batch, loss="anisotropic", pie="none"):
        """fpm_autotune for the shape of this problem; returns the tuner's one-line report."""
        prob, keep, mem = self._problem(O0, P0c, Y, led_idx, P0, pratio, 1, batch, 5e-4, 0.999,
                                        1e-4, 0.2, 12, 0.5, loss, pie)
        buf = C.create_string_buffer(512)
        _inputs_ready(*keep)
        self._check(self.lib.fpm_autotune(self._ctx, C.byref(prob), buf, len(buf)))
        del keep
        return buf.value.decode()

    def autotune_raw(self, prob: Problem) -> str:
        buf = C.create_string_buffer(512)
        self._check(self.lib.fpm_autotune(self._ctx, C.byref(prob), buf, len(buf)))
        return buf.value.decode()

    def batch_gradients(self, O, P, Y, led_idx, P0, pratio, loss="anisotropic", pie="none"):
        """v3 gradients of one LED batch (the fullyfusedFPM contract): (dO, dP, loss)."""
        prob, keep, mem = self._problem(O, P, Y, led_idx, P0, pratio, 0, 1, 0.0, 0.0, 0.0, 0.0,
                                        12, 0.5, loss, pie)
        h = prob.h
        H = h * prob.pratio
        like = Y if mem == MEM_DEVICE else None
        op, o = _empty_like_layout((H, H), np.complex64, like)
        pp, p = _empty_like_layout((h, h), np.complex64, like)
        lp, loss = _empty_like_layout((1,), np.float64, like)
        _inputs_ready(*keep)
        self._check(self.gradients_raw(prob, op, pp, lp))
        del keep
        return o, p, float(loss[0])

    def fft2(self, x, direction=-1):
        """Unnormalised 2-D FFT of a MATLAB-order (n, n) or (n, n, count) complex64 array."""
        if _is_torch(x):
            import torch
            y = x.permute(*reversed(range(x.dim()))).contiguous()
            out = torch.empty_like(y)
            n = int(x.shape[0])
            cnt = int(x.shape[2]) if x.dim() == 3 else 1
            _inputs_ready(y)
            self._check(self.lib.fpm_fft2(self._ctx, y.data_ptr(), out.data_ptr(), n, cnt,
                                          direction, MEM_DEVICE if y.is_cuda else MEM_HOST))
            return out.permute(*reversed(range(x.dim())))
        a = np.asfortranarray(np.asarray(x, np.complex64))
        out = np.empty_like(a, order="F")
        n = a.shape[0]
        cnt = a.shape[2] if a.ndim == 3 else 1
        self._check(self.lib.fpm_fft2(self._ctx, a.ctypes.data, out.ctypes.data, n, cnt,
                                      direction, MEM_HOST))
        return out

    def led_indices(self, grid, h, pratio, wavelength_um, led_pitch_um, led_height_um,
                    camera_pixel_um, magnification, sample_dx_um=-0.0, sample_dy_um=-0.0):
        """ledIdx of a grid x grid LED array in spiral order, computed on the device (FP64).

        Returns (led, order): led (L, 2) int32 rows (kl, kt) -- MATLAB's ledIdx transposed --
        and order (L, 2) int32 rows (i, j), the 1-based grid cell of each LED.
        """
        g = LedGeometry(int(grid), int(h), int(pratio), 0, float(wavelength_um),
                        float(led_pitch_um), float(led_height_um), float(camera_pixel_um),
                        float(magnification), float(sample_dx_um), float(sample_dy_um))
        L = int(grid) * int(grid)
        led = np.empty((L, 2), np.int32)
        order = np.empty((L, 2), np.int32)
        self._check(self.lib.fpm_led_indices(self._ctx, C.byref(g), led.ctypes.data,
                                             order.ctypes.data))
        return led, order

    def simulate(self, obj, pupil, led_idx, pratio, amplitude=False):
        """Forward model (gen_img_batch.m): MATLAB-order (h, h, L) float32 intensities
        |ifft2(ifftshift(crop(fftshift(fft2(obj))) .* pupil)) / pratio^2|^2 (or amplitudes).
        obj (H, H) and pupil (h, h) complex64, led_idx 2 x L int32 (MATLAB ledIdx); numpy
        in host memory or torch tensors on the context's device."""
        os_, ok, om = _colmajor(obj, np.complex64)
        ps, pk, pm = _colmajor(pupil, np.complex64)
        ls, lk, lm = _colmajor(led_idx, np.int32)
        if len({om, pm, lm}) != 1:
            raise ValueError("all inputs must live in the same memory")
        h = int(pupil.shape[0])
        L = int(led_idx.shape[1])
        like = obj if om == MEM_DEVICE else None
        if like is not None:
            import torch
            base = torch.empty((L, h, h), dtype=torch.float32, device=obj.device)
            op, out = base.data_ptr(), base.permute(2, 1, 0)
        else:
            out = np.empty((h, h, L), np.float32, order="F")
            op = out.ctypes.data
        _inputs_ready(ok, pk, lk)
        self._check(self.lib.fpm_simulate(self._ctx, os_, ps, ls, h, int(pratio), L,
                                          SIM_AMPLITUDE if amplitude else SIM_INTENSITY, op, om))
        del ok, pk, lk
        return out

    def normalise_stack(self, counts):
        """Amplitude sqrt((I-min)/(max-min)) over a whole uint16 or float32 stack
        (codes_v2/main_run_FPM.m:43-45), same shape, float32."""
        if _is_torch(counts):
            import torch
            x = counts.contiguous()
            if x.dtype not in (torch.uint16, torch.float32):
                raise TypeError(f"expected uint16 or float32, got {x.dtype}")
            fn = (self.lib.fpm_normalise_stack if x.dtype == torch.uint16
                  else self.lib.fpm_normalise_stack_f32)
            out = torch.empty(x.shape, dtype=torch.float32, device=x.device)
            mem = MEM_DEVICE if x.is_cuda else MEM_HOST
            _inputs_ready(x)
            self._check(fn(self._ctx, x.data_ptr(), x.numel(), out.data_ptr(), mem))
            return out
        x = np.asarray(counts)
        if x.dtype == np.float32:
            fn = self.lib.fpm_normalise_stack_f32
        else:
            x, fn = x.astype(np.uint16, copy=False), self.lib.fpm_normalise_stack
        x = np.ascontiguousarray(x)
        out = np.empty(x.shape, np.float32)
        self._check(fn(self._ctx, x.ctypes.data, x.size, out.ctypes.data, MEM_HOST))
        return out

    def optimizer_step(self, opt: Optimizer, param, grad):
        """One fpm_optimizer_step: param (complex64) updated in place; grad, the states
        named in opt and its clamp amplitude in the same memory (numpy arrays in host
        memory or torch tensors on the context's device, any contiguous layout with the
        same element order)."""
        if _is_torch(param):
            _inputs_ready(param, grad)
            ptr_p, ptr_g, n, mem = param.data_ptr(), grad.data_ptr(), param.numel(), MEM_DEVICE
        else:
            ptr_p, ptr_g, n, mem = param.ctypes.data, grad.ctypes.data, param.size, MEM_HOST
        self._check(self.lib.fpm_optimizer_step(self._ctx, C.byref(opt), ptr_p, ptr_g, n, mem))

    def read_stack(self, paths, h, row0=0, col0=0, dtype="u16", threads=0):
        """read_tiff_stack, failures reported on this context."""
        return read_tiff_stack(paths, h, row0, col0, dtype, threads, _ctx=self)


def read_tiff_stack(paths, h, row0=0, col0=0, dtype="u16", threads=0, _ctx=None):
    """Measured frames, one TIFF per LED in LED order (codes_v2/main_run_FPM.m:26-41):
    the h x h region at 0-based (row0, col0) of each file, as a MATLAB-order (h, h, L)
    array in column-major memory: uint16 counts (dtype "u16", single-sample frames)
    or the float32 mean over each pixel's samples (dtype "f32", mean(single(x), 3)).
    Host-side; needs no GPU.  Raises FpmError naming the file on an unreadable,
    unsupported or too small file."""
    lib = load_library()
    kind = {"u16": INGEST_U16, "f32": INGEST_F32_MEAN}[dtype]
    names = [os.fsencode(p) for p in paths]
    arr = (C.c_char_p * max(1, len(names)))(*names)
    out = np.empty((h, h, len(names)), np.uint16 if kind == INGEST_U16 else np.float32, order="F")
    ctx = _ctx._ctx if _ctx is not None else None
    st = lib.fpm_read_tiff_stack(ctx, arr, len(names), int(row0), int(col0), int(h), kind,
                                 out.ctypes.data, int(threads))
    if st != FPM_OK:
        raise FpmError(st, lib.fpm_last_error(ctx).decode())
    return out


_default_engine = None


def _engine() -> Engine:
    global _default_engine
    if _default_engine is None:
        _default_engine = Engine()
    return _default_engine


def cuFPM_pure_v3(O0, P0c, Y, ledIdx, P0, pratio, epochs, B, opt=(5e-4, 0.999, 1e-4)):
    """Mirror of ``[O, P] = cuFPM_pure_v3(O0, P0c, Y, ledIdx, P0, pratio, epochs, B, [lr beta eps])``."""
    r = _engine().solve(O0, P0c, Y, ledIdx, P0, pratio, epochs, B, lr=float(opt[0]),
                        beta=float(opt[1]), eps=float(opt[2]), spectrum=False)
    return r["object"], r["pupil"]


def fullyfusedFPM(O, P, Y, ledIdx, pratio, P0=None):
    """Mirror of ``[dldw1, dldw2] = fullyfusedFPM(O, P, Y, ledIdx, pratio)`` with the v3 loss."""
    if P0 is None:
        P0 = np.ones(np.asarray(P.shape), np.float32) if not _is_torch(P) else \
            __import__("torch").ones(P.shape, dtype=__import__("torch").float32, device=P.device)
    dO, dP, _ = _engine().batch_gradients(O, P, Y, ledIdx, P0, pratio)
    return dO, dP
