import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT / "fused-fourier-ptycho_b200"))
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA path")


def has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def to_matlab_stack(Y):
    """(L, h, h) [l, r, c] -> MATLAB-order (h, h, L)."""
    return np.ascontiguousarray(np.transpose(Y, (1, 2, 0)))


def led_matlab(led):
    """(L, 2) rows (kl, kt) -> MATLAB-order 2 x L int32."""
    return np.ascontiguousarray(np.asarray(led, np.int32).T)


def torch_forward_model(O, P, led, pratio):
    """Checker for sizes the FP64 oracle cannot reach: the forward model of
    benchmark/gen_img_batch.m:178-201 in plain torch complex64 (amplitudes), on
    whatever device O lives.  O (H, H) and P (h, h) complex tensors, led (L, 2) rows
    (kl, kt) 1-based; returns (L, h, h) [l, r, c]."""
    import torch
    H, h = O.shape[0], P.shape[0]
    F = torch.fft.fftshift(torch.fft.fft2(O))
    ar = torch.arange(h, device=O.device)
    out = []
    for kl, kt in np.asarray(led):
        rows, cols = (int(kt) - 1 + ar) % H, (int(kl) - 1 + ar) % H
        sub = F.index_select(0, rows).index_select(1, cols) * P
        out.append(torch.fft.ifft2(torch.fft.ifftshift(sub)).abs() / (pratio * pratio))
    return torch.stack(out)


_CACHE = {}


def dataset(h, pratio, grid, seed=0, aberration=False):
    key = (h, pratio, grid, seed, aberration)
    if key not in _CACHE:
        from fpm_b200 import synth
        _CACHE[key] = synth.make_dataset(h, pratio, grid, seed=seed, aberration=aberration)
    return _CACHE[key]


@pytest.fixture(scope="session")
def ds_a():
    """The 128² case: 11 x 11 LEDs of 128 x 128, pratio 4, seed 0."""
    return dataset(128, 4, 11, seed=0)


@pytest.fixture(scope="session")
def ds_small():
    """A 5 x 5 LED, 64 x 64, pratio 4 case with an aberrated pupil."""
    return dataset(64, 4, 5, seed=3, aberration=True)


@pytest.fixture(scope="session")
def engine():
    if not has_gpu():
        pytest.skip("no CUDA device")
    import fpm_b200
    e = fpm_b200.Engine(0)
    yield e
    e.close()
