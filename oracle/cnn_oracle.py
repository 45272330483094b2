"""CPU oracle of the warm-start network (fpm_cnn_* of libfpm).

TEST INFRASTRUCTURE ONLY: the checker of tests/test_gpu_cnn.py.  A numpy restatement, in
FP64, of the network that csrc/cnn_api.cpp builds (14 3x3 convolutions with zero padding,
ReLU, 2x2 average pooling, 2x nearest up-sampling, additive skips, a mean-squared loss)
and of its gradients by reverse-mode differentiation, with the convolution operands
rounded to BF16 exactly as the tensor-core kernels stage them (activations, output
gradients and weights round to nearest even; products and sums exact here, FP32 there).
Parameter order as the library's: per layer, weights [Cout][Cin][3][3] then biases.
"""
from __future__ import annotations

import numpy as np


def bf16(x):
    """Round to the nearest BF16 (ties to even), returned as float64."""
    f = np.asarray(x, np.float32)
    b = f.view(np.uint32).astype(np.uint64)
    r = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def layers(in_ch: int, base: int):
    c = base
    return [(in_ch, c), (c, c), (c, 2 * c), (2 * c, 2 * c), (2 * c, 4 * c), (4 * c, 4 * c),
            (4 * c, 8 * c), (8 * c, 4 * c), (4 * c, 4 * c), (4 * c, 2 * c), (2 * c, 2 * c),
            (2 * c, c), (c, c), (c, 2)]


def unpack(params, in_ch: int, base: int):
    out, off = [], 0
    for ci, co in layers(in_ch, base):
        W = params[off:off + co * ci * 9].reshape(co, ci, 3, 3).astype(np.float64)
        off += co * ci * 9
        b = params[off:off + co].astype(np.float64)
        off += co
        out.append((W, b))
    assert off == len(params)
    return out


def _cols(x):
    """(N, C, H, W) -> (N, C*9, H*W) of zero-padded 3x3 neighbourhoods (c, ky, kx)."""
    N, C, H, W = x.shape
    p = np.pad(x, ((0, 0), (0, 0), (1, 1), (1, 1)))
    cols = np.empty((N, C, 9, H, W))
    for t in range(9):
        ky, kx = divmod(t, 3)
        cols[:, :, t] = p[:, :, ky:ky + H, kx:kx + W]
    return cols.reshape(N, C * 9, H * W)


def _r(x, rounding):
    return bf16(x) if rounding else np.asarray(x, np.float64)


def conv(x, W, b, rounding=True):
    N, C, H, Wd = x.shape
    co = W.shape[0]
    y = np.einsum("ok,nkp->nop", _r(W, rounding).reshape(co, -1), _cols(_r(x, rounding)))
    if b is not None:
        y = y + b[None, :, None]
    return y.reshape(N, co, H, Wd)


def conv_back(x, W, gout, rounding=True):
    """(dW, db, dx) of y = conv(x, W, b) given dL/dy, operands rounded as the kernels do
    (rounding=False: the exact derivative, for finite-difference checks)."""
    N, C, H, Wd = x.shape
    co = W.shape[0]
    g = gout.reshape(N, co, H * Wd)
    dW = np.einsum("nop,nkp->ok", _r(g, rounding), _cols(_r(x, rounding))).reshape(W.shape)
    db = gout.sum(axis=(0, 2, 3))
    Wt = np.flip(_r(W, rounding), axis=(2, 3)).transpose(1, 0, 2, 3)   # [ci][co][2-ky][2-kx]
    dx = conv(gout, Wt, None, rounding)
    return dW, db, dx


def pool(x):
    return 0.25 * (x[:, :, 0::2, 0::2] + x[:, :, 0::2, 1::2] + x[:, :, 1::2, 0::2] + x[:, :, 1::2, 1::2])


def pool_back(g):
    return 0.25 * np.repeat(np.repeat(g, 2, axis=2), 2, axis=3)


def up(x):
    return np.repeat(np.repeat(x, 2, axis=2), 2, axis=3)


def up_back(g):
    return g[:, :, 0::2, 0::2] + g[:, :, 0::2, 1::2] + g[:, :, 1::2, 0::2] + g[:, :, 1::2, 1::2]


def relu(x):
    return np.maximum(x, 0.0)


def forward(params, x, in_ch: int, base: int, rounding=True, noise=0.0, seed=0):
    """The output and the activations the backward pass needs.  noise > 0 multiplies every
    convolution's output by (1 + noise * N(0, 1)) (seeded): a twin whose accumulation
    differs from this one's by about the FP32 rounding of the device's sums, so that the
    BF16 rounding of the next layer's operands may flip where the device's may."""
    L = unpack(params, in_ch, base)
    _conv = conv
    rng = np.random.default_rng(seed)

    def conv_(inp, W, b):
        y = _conv(inp, W, b, rounding)
        return y * (1.0 + noise * rng.standard_normal(y.shape)) if noise > 0 else y
    a = {}
    a["r1"] = relu(conv_(x, *L[0]))
    a["e1"] = relu(conv_(a["r1"], *L[1]))
    a["p1"] = pool(a["e1"])
    a["r3"] = relu(conv_(a["p1"], *L[2]))
    a["e2"] = relu(conv_(a["r3"], *L[3]))
    a["p2"] = pool(a["e2"])
    a["r5"] = relu(conv_(a["p2"], *L[4]))
    a["e3"] = relu(conv_(a["r5"], *L[5]))
    a["p3"] = pool(a["e3"])
    a["e4"] = relu(conv_(a["p3"], *L[6]))
    a["u3"] = up(a["e4"])
    a["r8"] = relu(conv_(a["u3"], *L[7]))
    a["s3"] = a["r8"] + a["e3"]
    a["d3"] = relu(conv_(a["s3"], *L[8]))
    a["u2"] = up(a["d3"])
    a["r10"] = relu(conv_(a["u2"], *L[9]))
    a["s2"] = a["r10"] + a["e2"]
    a["d2"] = relu(conv_(a["s2"], *L[10]))
    a["u1"] = up(a["d2"])
    a["r12"] = relu(conv_(a["u1"], *L[11]))
    a["s1"] = a["r12"] + a["e1"]
    a["d1"] = relu(conv_(a["s1"], *L[12]))
    y = conv_(a["d1"], *L[13])
    return y, a, L


def loss_and_gradients(params, x, t, in_ch: int, base: int, rounding=True, noise=0.0, seed=0):
    """mean (y - t)^2 and its gradient with respect to the parameter vector (noise: the
    forward twin of `forward`)."""
    y, a, L = forward(params, x, in_ch, base, rounding, noise, seed)
    n = y.size
    loss = float(((y - t) ** 2).sum() / n)
    dy = 2.0 * (y - t) / n
    grads = [None] * 14

    def back(i, inp, g, need=True):
        dW, db, dx = conv_back(inp, L[i][0], g, rounding)
        grads[i] = (dW, db)
        return dx if need else None

    mask = lambda g, act: np.where(act > 0, g, 0.0)
    g = back(13, a["d1"], dy)
    g = back(12, a["s1"], mask(g, a["d1"]))
    ge1 = g.copy()
    g = back(11, a["u1"], mask(g, a["r12"]))
    g = up_back(g)
    g = back(10, a["s2"], mask(g, a["d2"]))
    ge2 = g.copy()
    g = back(9, a["u2"], mask(g, a["r10"]))
    g = up_back(g)
    g = back(8, a["s3"], mask(g, a["d3"]))
    ge3 = g.copy()
    g = back(7, a["u3"], mask(g, a["r8"]))
    g = up_back(g)
    g = back(6, a["p3"], mask(g, a["e4"]))
    ge3 = ge3 + pool_back(g)
    g = back(5, a["r5"], mask(ge3, a["e3"]))
    g = back(4, a["p2"], mask(g, a["r5"]))
    ge2 = ge2 + pool_back(g)
    g = back(3, a["r3"], mask(ge2, a["e2"]))
    g = back(2, a["p1"], mask(g, a["r3"]))
    ge1 = ge1 + pool_back(g)
    g = back(1, a["r1"], mask(ge1, a["e1"]))
    back(0, x, mask(g, a["r1"]), need=False)
    flat = np.concatenate([np.concatenate([dW.ravel(), db]) for dW, db in grads])
    return loss, flat
