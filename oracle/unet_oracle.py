"""CPU oracle of the warm-start surrogate network (test infrastructure only).

A numpy restatement of every device kernel of
mpi-multi-process-version_b200/csrc/unet_kernels.cu and of the whole U-Net's
forward and backward passes, used by the tests to check the GPU's
activations and gradients.  The reference has no learned component (it always
starts from the conduction state of initial(),
natural-convection_2dim_mono.f90:199-240), so there is no reference code to
pin this file to; it is pinned instead by a finite-difference check of its own
backward pass (tests/test_surrogate.py).

Rounding: with `bf16=True` the oracle rounds to bfloat16 at exactly the points
where the device stores bfloat16 (input image, weights, activations, the
gradients that feed the tensor-core products); everything else is float64.
With `bf16=False` it is plain float64 (used for the finite-difference check).

Layout: images are NHWC arrays (B, H, W, C); 3x3 weights are (Cout, 9, Cin)
with tap = 3*ky + kx; padding 1.
"""
from __future__ import annotations

import numpy as np


def bf16_round(x):
    """Round to the nearest bfloat16 (ties to even), returned as float64."""
    f = np.ascontiguousarray(x, dtype=np.float32)
    b = f.view(np.uint32).astype(np.uint64)
    r = ((b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).astype(np.float64)


def _im2col(x):
    B, H, W, C = x.shape
    xp = np.zeros((B, H + 2, W + 2, C), dtype=np.float64)
    xp[:, 1:-1, 1:-1] = x
    cols = np.empty((B, H, W, 9, C), dtype=np.float64)
    for tap in range(9):
        ky, kx = divmod(tap, 3)
        cols[:, :, :, tap] = xp[:, ky:ky + H, kx:kx + W]
    return cols.reshape(B * H * W, 9 * C)


def conv3x3(x, w, bias=None):
    """z[p, co] = sum_{tap, ci} x[p + offset(tap), ci] w[co, tap, ci] + bias."""
    B, H, W, _ = x.shape
    Cout = w.shape[0]
    z = _im2col(x) @ w.reshape(Cout, -1).T
    if bias is not None:
        z = z + bias
    return z.reshape(B, H, W, Cout)


def conv3x3_dgrad(dz, w):
    """dL/dx of conv3x3 given dL/dz: conv3x3 of dz with w flipped and transposed."""
    wt = flip_weights(w)
    return conv3x3(dz, wt)


def flip_weights(w):
    """wt[ci, tap, co] = w[co, 8 - tap, ci]."""
    return np.ascontiguousarray(w[:, ::-1, :].transpose(2, 1, 0))


def conv3x3_wgrad(dz, x):
    """dw[co, tap, ci] = sum_p dz[p, co] x[p + offset(tap), ci]."""
    Cout = dz.shape[-1]
    Cin = x.shape[-1]
    g = dz.reshape(-1, Cout).T @ _im2col(x)
    return g.reshape(Cout, 9, Cin)


def silu(z):
    return z / (1.0 + np.exp(-z))


def silu_grad(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def pool2(x):
    B, H, W, C = x.shape
    return 0.25 * ((x[:, 0::2, 0::2] + x[:, 0::2, 1::2]) + (x[:, 1::2, 0::2] + x[:, 1::2, 1::2]))


def pool2_backward(dy):
    return 0.25 * np.repeat(np.repeat(dy, 2, axis=1), 2, axis=2)


def up2(x):
    return np.repeat(np.repeat(x, 2, axis=1), 2, axis=2)


def up2_backward(dy):
    return (dy[:, 0::2, 0::2] + dy[:, 0::2, 1::2]) + (dy[:, 1::2, 0::2] + dy[:, 1::2, 1::2])


def head(a, wh, bh):
    return a @ wh.T + bh


def mse(y, t, cw):
    n = y.size
    d = y - t
    loss = float((cw * d * d).sum() / n)
    return loss, 2.0 * cw * d / n


# ---------------------------------------------------------------------------
# the network: layer table shared with the device host code
# ---------------------------------------------------------------------------
IN_CH = 32       # input image channels (the features occupy the first few)
LEVELS = (32, 64, 128, 256)
OUT_CH = 3


def layer_table():
    """[(name, Cin, Cout)] of the 3x3 layers in execution order, then the head."""
    c1, c2, c3, c4 = LEVELS
    return [("e1a", IN_CH, c1), ("e1b", c1, c1), ("e2a", c1, c2), ("e2b", c2, c2),
            ("e3a", c2, c3), ("e3b", c3, c3), ("ba", c3, c4), ("bb", c4, c4),
            ("d3a", c4 + c3, c3), ("d3b", c3, c3), ("d2a", c3 + c2, c2), ("d2b", c2, c2),
            ("d1a", c2 + c1, c1), ("d1b", c1, c1)]


def param_count():
    n = sum(9 * ci * co + co for _, ci, co in layer_table())
    return n + OUT_CH * LEVELS[0] + OUT_CH


def forward(params, x, bf16=True):
    """params: {name: (w, b)} plus 'head': (wh, bh); x: (B, R, R, IN_CH).
    Returns (y, cache)."""
    r = bf16_round if bf16 else (lambda v: np.asarray(v, dtype=np.float64))
    P = {k: (r(w), np.asarray(b, dtype=np.float64) if k != "head" else np.asarray(b, dtype=np.float64))
         for k, (w, b) in params.items()}
    cache = {"x": r(x), "P": P}

    def layer(name, inp):
        w, b = P[name]
        z = conv3x3(inp, w, b)
        if bf16:
            z = z.astype(np.float32).astype(np.float64)
        a = r(silu(z))
        cache[name] = (inp, z, a)
        return a

    a = layer("e1a", cache["x"])
    s1 = layer("e1b", a)
    a = layer("e2a", r(pool2(s1)))
    s2 = layer("e2b", a)
    a = layer("e3a", r(pool2(s2)))
    s3 = layer("e3b", a)
    a = layer("ba", r(pool2(s3)))
    bt = layer("bb", a)
    a = layer("d3a", np.concatenate([up2(bt), s3], axis=-1))
    u3 = layer("d3b", a)
    a = layer("d2a", np.concatenate([up2(u3), s2], axis=-1))
    u2 = layer("d2b", a)
    a = layer("d1a", np.concatenate([up2(u2), s1], axis=-1))
    u1 = layer("d1b", a)
    wh, bh = P["head"]
    y = head(u1, wh, bh)
    cache["u1"] = u1
    return y, cache


def backward(cache, dy, bf16=True):
    """Gradients {name: (dw, db)} of sum(dy * y) through the cached forward."""
    r = bf16_round if bf16 else (lambda v: np.asarray(v, dtype=np.float64))
    f32 = (lambda v: v.astype(np.float32).astype(np.float64)) if bf16 else (lambda v: v)
    P = cache["P"]
    grads = {}
    wh, bh = P["head"]
    u1 = cache["u1"]
    C1 = u1.shape[-1]
    grads["head"] = (dy.reshape(-1, dy.shape[-1]).T @ u1.reshape(-1, C1), dy.reshape(-1, dy.shape[-1]).sum(0))
    da = f32(dy @ wh)

    def back(name, da, need_dx=True):
        inp, z, _ = cache[name]
        dz = r(da * silu_grad(z))
        w, _ = P[name]
        grads[name] = (conv3x3_wgrad(dz, inp), dz.reshape(-1, dz.shape[-1]).sum(0))
        return f32(conv3x3_dgrad(dz, w)) if need_dx else None

    c1, c2, c3, _ = LEVELS
    da = back("d1b", da)
    dcat1 = back("d1a", da)
    da = back("d2b", f32(up2_backward(dcat1[..., :c2])))
    dcat2 = back("d2a", da)
    da = back("d3b", f32(up2_backward(dcat2[..., :c3])))
    dcat3 = back("d3a", da)
    da = back("bb", f32(up2_backward(dcat3[..., :LEVELS[3]])))
    dp3 = back("ba", da)
    ds3 = f32(dcat3[..., LEVELS[3]:] + pool2_backward(dp3))
    da = back("e3b", ds3)
    dp2 = back("e3a", da)
    ds2 = f32(dcat2[..., c3:] + pool2_backward(dp2))
    da = back("e2b", ds2)
    dp1 = back("e2a", da)
    ds1 = f32(dcat1[..., c2:] + pool2_backward(dp1))
    da = back("e1b", ds1)
    back("e1a", da, need_dx=False)
    return grads


def init_params(seed=0):
    """He-style initialisation (the device host code uses the same one)."""
    rng = np.random.default_rng(seed)
    params = {}
    for name, ci, co in layer_table():
        w = rng.normal(0.0, np.sqrt(2.0 / (9 * ci)), size=(co, 9, ci))
        params[name] = (w, np.zeros(co))
    params["head"] = (rng.normal(0.0, np.sqrt(1.0 / LEVELS[0]), size=(OUT_CH, LEVELS[0])), np.zeros(OUT_CH))
    return params
