"""CPU reference of the control-variate network (TEST INFRASTRUCTURE ONLY:
used by tests/ to check the device kernels of nrcps_b200/csrc/cvnet.cu, never
by the product path).

The same network as the device: 3x3x3 periodic cross-correlations
out[s] = b + sum_ci sum_k W[co][ci][k] in[ci][s + d_k] with tanh, mean pool,
tanh hidden layer, linear output; loss 0.5 mean (y - target)^2.  With
bf16=True the weights and activations are rounded to BF16 (round to nearest
even) exactly where the device rounds them and everything else runs in FP64;
with bf16=False the whole computation is FP64 (for finite-difference checks
of the analytic gradients).
"""
from __future__ import annotations

import numpy as np

OFFSETS = [(k // 9 - 1, (k // 3) % 3 - 1, k % 3 - 1) for k in range(27)]


def to_bf16(x) -> np.ndarray:
    """FP32 -> BF16 -> FP64, round to nearest even."""
    b = np.ascontiguousarray(np.asarray(x, dtype=np.float32)).view(np.uint32).astype(np.uint64)
    r = ((b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).astype(np.float64)


def shift(a: np.ndarray, G: int, d) -> np.ndarray:
    """a[..., s] -> a[..., s + d] on the periodic G^3 lattice (s = z + G (y + G x))."""
    sh = a.reshape(a.shape[:-1] + (G, G, G))
    return np.roll(sh, shift=(-d[0], -d[1], -d[2]), axis=(-3, -2, -1)).reshape(a.shape)


def conv(x: np.ndarray, W: np.ndarray, b: np.ndarray, G: int) -> np.ndarray:
    """x [B, Cin, GS], W [Cout, Cin, 27] -> [B, Cout, GS]."""
    out = np.zeros((x.shape[0], W.shape[0], x.shape[2])) + b[None, :, None]
    for k, d in enumerate(OFFSETS):
        out += np.einsum("oc,bcs->bos", W[:, :, k], shift(x, G, d))
    return out


def conv_grads(dZ: np.ndarray, x: np.ndarray, W: np.ndarray, G: int):
    """dW [Cout, Cin, 27], db [Cout], dX [B, Cin, GS] of conv()."""
    dW = np.zeros(W.shape)
    dX = np.zeros(x.shape)
    for k, d in enumerate(OFFSETS):
        xs = shift(x, G, d)
        dW[:, :, k] = np.einsum("bos,bcs->oc", dZ, xs)
        dX += shift(np.einsum("oc,bos->bcs", W[:, :, k], dZ), G, tuple(-v for v in d))
    return dW, dZ.sum(axis=(0, 2)), dX


def forward(params: dict, x: np.ndarray, G: int, bf16: bool = True):
    r = to_bf16 if bf16 else (lambda v: np.asarray(v, dtype=np.float64))
    cache = {"x": np.asarray(x, dtype=np.float64)}
    a = cache["x"]
    for i in (1, 2, 3):
        z = conv(a, r(params[f"w{i}"]), np.asarray(params[f"b{i}"], dtype=np.float64), G)
        a = r(np.tanh(z))
        cache[f"a{i}"] = a
    p = a.mean(axis=2)
    h = np.tanh(p @ np.asarray(params["hw"], dtype=np.float64).T + params["hb"])
    y = h @ np.asarray(params["ow"], dtype=np.float64).T + params["ob"]
    cache.update(p=p, h=h, y=y)
    return y, cache


def loss_and_grads(params: dict, x: np.ndarray, target: np.ndarray, G: int, bf16: bool = True):
    r = to_bf16 if bf16 else (lambda v: np.asarray(v, dtype=np.float64))
    y, c = forward(params, x, G, bf16)
    B, T = y.shape
    d = y - target
    loss = 0.5 * (d ** 2).sum() / (B * T)
    dy = d / (B * T)
    g = {"ow": dy.T @ c["h"], "ob": dy.sum(0)}
    dh = dy @ np.asarray(params["ow"], dtype=np.float64)
    dzh = dh * (1.0 - c["h"] ** 2)
    g["hw"], g["hb"] = dzh.T @ c["p"], dzh.sum(0)
    dp = dzh @ np.asarray(params["hw"], dtype=np.float64)
    GS = x.shape[2]
    dz = (dp[:, :, None] / GS) * (1.0 - c["a3"] ** 2)
    for i in (3, 2, 1):
        inp = c[f"a{i - 1}"] if i > 1 else c["x"]
        dW, db, dX = conv_grads(dz, inp, r(params[f"w{i}"]), G)
        g[f"w{i}"], g[f"b{i}"] = dW, db
        if i > 1:
            dz = dX * (1.0 - c[f"a{i - 1}"] ** 2)
    return loss, y, g
