"""In-tree build of libfpm.so (and the fpm_cli binary) for sm_100a with nvcc.

Objects go to ``fpm_b200/_lib/obj``; the shared library to ``fpm_b200/_lib``.
Rebuilds only what changed (source or header newer than the object).
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = ROOT / "csrc"
INCLUDE = ROOT.parent / "include"
LIBDIR = PKG / "_lib"
OBJDIR = LIBDIR / "obj"
LIB = LIBDIR / "libfpm.so"
CLI = LIBDIR / "fpm_cli"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I", str(INCLUDE),
                  "--expt-relaxed-constexpr"]
LIBS_SOURCES = ["kernels_lowres.cu", "kernels_update.cu", "fft_own.cu", "fpm_api.cpp",
                "noalloc.cu", "pipeline.cu", "geometry.cu", "tiff.cpp",
                "optimizers.cu", "generic.cu", "tuning.cpp", "cnn.cu", "cnn_api.cpp"]
LINK_LIBS = ["-lcudart", "-lpthread"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libfpm")


def _stale(obj: Path, src: Path) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    deps = [src] + list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))
    return any(d.stat().st_mtime > t for d in deps)


def _compile(src: Path, verbose: bool) -> Path:
    obj = OBJDIR / (src.name + ".o")
    if _stale(obj, src):
        cmd = [nvcc()] + NVFLAGS + ["-c", str(src), "-o", str(obj)]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {src.name}:\n{r.stdout}\n{r.stderr}")
    return obj


def build(verbose: bool = False) -> Path:
    OBJDIR.mkdir(parents=True, exist_ok=True)
    srcs = [CSRC / s for s in LIBS_SOURCES]
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    if not LIB.exists() or any(o.stat().st_mtime > LIB.stat().st_mtime for o in objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", str(LIB)] + [str(o) for o in objs] + LINK_LIBS
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link of libfpm.so failed:\n{r.stdout}\n{r.stderr}")
    build_cli(verbose)
    return LIB


def build_cli(verbose: bool = False) -> Path:
    """fpm_cli, the file-driven front end (host C++ over the C ABI), next to libfpm.so."""
    src = CSRC / "fpm_cli.cpp"
    if CLI.exists() and CLI.stat().st_mtime > max(src.stat().st_mtime, LIB.stat().st_mtime,
                                                  (INCLUDE / "fpm.h").stat().st_mtime):
        return CLI
    cxx = os.environ.get("CXX") or shutil.which("g++") or "g++"
    cmd = [cxx, "-O2", "-std=c++17", "-Wall", "-I", str(INCLUDE), str(src), "-o", str(CLI),
           "-L", str(LIBDIR), "-lfpm", "-Wl,-rpath,$ORIGIN"]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"build of fpm_cli failed:\n{r.stdout}\n{r.stderr}")
    return CLI


if __name__ == "__main__":
    print(build(verbose=True))
