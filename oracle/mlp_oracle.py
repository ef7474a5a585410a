"""TEST INFRASTRUCTURE ONLY: numpy restatement of the proposal network's
forward and backward pass (64 -> 128 -> 128 -> 192 logits, 191 real
classes), with the same bf16 roundings as the GPU path: weights, the input
features and the stored activations / output gradients are bf16, every
product is accumulated in float64 here (FP32 on the tensor cores).  Used to
check the GPU gradients."""
from __future__ import annotations

import numpy as np

F, H, O, C = 64, 128, 192, 191


def bf16(a: np.ndarray) -> np.ndarray:
    """Round float32 to bfloat16 (round to nearest even), returned as float64."""
    a = np.ascontiguousarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(params: np.ndarray):
    o = 0
    out = {}
    for name, shape in (("w1", (H, F)), ("b1", (H,)), ("w2", (H, H)), ("b2", (H,)),
                        ("w3", (O, H)), ("b3", (O,))):
        n = int(np.prod(shape))
        out[name] = params[o:o + n].reshape(shape).astype(np.float64)
        o += n
    return out


def forward_backward(params: np.ndarray, x_bf16: np.ndarray, labels: np.ndarray):
    """Returns (mean loss, gradient vector in the parameter layout)."""
    p = unpack(params)
    w1, w2, w3 = bf16(p["w1"]), bf16(p["w2"]), bf16(p["w3"])
    x = x_bf16.astype(np.float64)
    n = x.shape[0]
    h1 = bf16(np.maximum(x @ w1.T + p["b1"], 0.0))
    h2 = bf16(np.maximum(h1 @ w2.T + p["b2"], 0.0))
    z = (h2 @ w3.T + p["b3"]).astype(np.float32).astype(np.float64)
    zc = z[:, :C]
    m = zc.max(axis=1, keepdims=True)
    e = np.exp(zc - m)
    s = e.sum(axis=1, keepdims=True)
    prob = e / s
    loss = float(np.mean(-(zc[np.arange(n), labels] - m[:, 0] - np.log(s[:, 0]))))
    dz = np.zeros((n, O))
    dz[:, :C] = prob
    dz[np.arange(n), labels] -= 1.0
    dz = bf16(dz / n)
    gw3 = dz.T @ h2
    gb3 = dz.sum(axis=0)
    dh2 = bf16((dz @ w3) * (h2 > 0))
    gw2 = dh2.T @ h1
    gb2 = dh2.sum(axis=0)
    dh1 = bf16((dh2 @ w2) * (h1 > 0))
    gw1 = dh1.T @ x
    gb1 = dh1.sum(axis=0)
    g = np.concatenate([gw1.ravel(), gb1, gw2.ravel(), gb2, gw3.ravel(), gb3])
    return loss, g
