"""CPU checks of the warm-start network's oracle (oracle/cnn_oracle.py): its analytic
gradient equals central finite differences of its own loss (FP64, no BF16 rounding), for
every kind of parameter, and its BF16 rounding is round-to-nearest-even."""
import numpy as np

from oracle import cnn_oracle as co


def _case(seed=0, in_ch=3, base=8, n=2, h=16):
    rng = np.random.default_rng(seed)
    sizes = sum(a * b * 9 + b for a, b in co.layers(in_ch, base))
    p = rng.standard_normal(sizes) * 0.2
    x = rng.random((n, in_ch, h, h))
    t = rng.standard_normal((n, 2, h, h)) * 0.1
    return p, x, t, in_ch, base


def test_oracle_gradient_matches_finite_differences():
    p, x, t, in_ch, base = _case()
    loss, g = co.loss_and_gradients(p, x, t, in_ch, base, rounding=False)
    rng = np.random.default_rng(1)
    # a spread of indices: weights and biases of the first, middle and last layers
    offs, idx = 0, []
    for ci, cout in co.layers(in_ch, base):
        nw = ci * cout * 9
        idx += [offs + int(rng.integers(nw)), offs + nw + int(rng.integers(cout))]
        offs += nw + cout
    eps = 1e-6
    for i in idx:
        q = p.copy()
        q[i] += eps
        lp, _ = co.loss_and_gradients(q, x, t, in_ch, base, rounding=False)
        q[i] -= 2 * eps
        lm, _ = co.loss_and_gradients(q, x, t, in_ch, base, rounding=False)
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - g[i]) <= 1e-6 + 1e-4 * abs(fd), (i, fd, g[i])


def test_bf16_rounding_is_nearest_even():
    # exactly representable values stay, halfway cases go to the even neighbour
    assert co.bf16(np.float32(1.0 + 2 ** -7)) == 1.0 + 2 ** -7
    assert co.bf16(np.float32(1.0 + 2 ** -8)) == 1.0            # halfway: even (1.0)
    assert co.bf16(np.float32(1.0 + 3 * 2 ** -8)) == 1.0 + 2 ** -6   # halfway: even
    assert co.bf16(np.float32(-2.5)) == -2.5
