"""Recipe: build the reference's own v3 kernels into oracle/_ref/libcufpm_ref.so.

TEST INFRASTRUCTURE.  Compiles ``oracle/ref_harness.cu`` (our replica of the
host loop of ``cuFPM_v3/cuFPM_pure_v3.cu:75-207``) against the reference's
``cuFPM_v3/cuda/kernels.cuh`` *where it lies* in the read-only reference tree,
with ``oracle/ref_shim.h`` force-included for the two MATLAB element types.
No reference source is copied into this repository; only the built ``.so``
(git-ignored) is kept under ``oracle/_ref/`` so it travels with the tree.
Runs only where the reference tree exists; elsewhere the prebuilt library is
used as is.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
LIB = OUT / "libcufpm_ref.so"
REF_ROOT = Path(os.environ.get("FPM_REFERENCE_ROOT", "/root/reference"))
REF_KERNELS_DIR = REF_ROOT / "cuFPM_v3" / "cuda"


def build(force: bool = False) -> Path | None:
    if not (REF_KERNELS_DIR / "kernels.cuh").exists():
        return LIB if LIB.exists() else None
    src = HERE / "ref_harness.cu"
    if LIB.exists() and not force and LIB.stat().st_mtime > max(
            src.stat().st_mtime, (HERE / "ref_shim.h").stat().st_mtime):
        return LIB
    OUT.mkdir(exist_ok=True)
    nvcc = os.environ.get("NVCC") or "/usr/local/cuda/bin/nvcc"
    if not Path(nvcc).exists():
        nvcc = shutil.which("nvcc") or nvcc
    cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo",
           "-Xcompiler", "-fPIC", "-shared", "-include", str(HERE / "ref_shim.h"),
           "-I", str(REF_KERNELS_DIR), str(src), "-o", str(LIB), "-lcufft"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"reference build failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
