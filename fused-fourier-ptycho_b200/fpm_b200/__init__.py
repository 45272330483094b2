"""B200-native Fourier-ptychographic reconstruction engine (host side).

The compute path is libfpm.so (hand-written sm_100a CUDA behind the C ABI of
include/fpm.h); this package binds it with ctypes and mirrors the reference's
mex calls.  See ``api`` for the entry points and ``synth`` for seeded data sets.
"""
from .api import (EXPORTED, Engine, FpmError, Problem, Result, DeviceOpts, cuFPM_pure_v3,
                  fullyfusedFPM, load_library, read_tiff_stack, MEM_DEVICE, MEM_HOST, STACK_F32,
                  STACK_U16)

__all__ = ["EXPORTED", "Engine", "FpmError", "Problem", "Result", "DeviceOpts", "cuFPM_pure_v3",
           "fullyfusedFPM", "load_library", "read_tiff_stack", "MEM_DEVICE", "MEM_HOST", "STACK_F32",
           "STACK_U16"]
