"""The autotuner (fpm_autotune, and FPM_CTX_AUTOTUNE for the first solve of a shape).

Its candidates are launch choices that leave the arithmetic alone (LED grouping of the
low-resolution passes, fused or two-pass row transforms, cluster size, the any-size
FFT's lines per block) or change only the rounding of a radix split (the 16384-point
passes' values per thread).  A tuned solve must therefore equal the untuned one: within
2e-5 relative on the object and pupil, the loss to 1e-6.
"""
import numpy as np
import pytest

from conftest import led_matlab, to_matlab_stack, dataset

pytestmark = pytest.mark.gpu


def _close(a, b):
    from oracle import fpm_oracle as orc
    for k in ("object", "pupil"):
        assert orc.rel_err(np.asarray(a[k]), np.asarray(b[k])) < 2e-5, k
    np.testing.assert_allclose(np.asarray(a["loss"]), np.asarray(b["loss"]), rtol=1e-6)


@pytest.mark.parametrize("h,p,B", [(128, 4, 16), (48, 4, 8)])
def test_autotune_report_and_unchanged_results(h, p, B):
    import fpm_b200
    ds = dataset(h, p, 5, seed=9, aberration=True)
    args = (ds.O0, ds.P0c, to_matlab_stack(ds.raw), led_matlab(ds.led_idx), ds.pupil0, p)
    with fpm_b200.Engine(0) as eng:
        plain = eng.solve(*args, 3, B, lr=1e-3)
        rep = eng.autotune(*args, B)
        assert "ms/epoch" in rep and "lr_group=" in rep, rep
        assert "(cached)" in eng.autotune(*args, B)
        tuned = eng.solve(*args, 3, B, lr=1e-3)
    _close(tuned, plain)
    with fpm_b200.Engine(0, autotune=True) as eng:      # tunes inside the first solve
        auto = eng.solve(*args, 3, B, lr=1e-3)
        assert "(cached)" in eng.autotune(*args, B)
    _close(auto, plain)
