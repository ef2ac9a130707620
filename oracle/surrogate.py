"""CPU restatement of the learned surrogate (test infrastructure only).

numpy float64 forward and backward of the residual CNN that
mass_hd_b200/surrogate.py trains on the GPU, used to check the GPU
convolutions, epilogues and gradients. The reference has no surrogate: the
network follows the stated design (6 residual blocks of two 3x3
circular-padded convolutions, 64 channels, GELU (tanh form), a linear 5->64 input
convolution and a 64->5 output convolution added to the input fields), and
this restatement is pinned by finite differences (tests/test_surrogate_oracle.py).

With `bf=True` the values the GPU stores in bfloat16 (weights, the padded
activations, the loss gradient and the gradients between layers) are rounded
the same way, so GPU and oracle differ only by FP32 accumulation order and
the hardware tanh estimate.

Layouts: images [B, H, W, C]; weights [cout, 9, cin] with tap = 3*ky + kx
multiplying input pixel (y+ky-1, x+kx-1) (periodic).
"""
from __future__ import annotations

import numpy as np

NBLOCKS = 6
CH = 64
NF = 5


def bf16(a: np.ndarray) -> np.ndarray:
    """Round to bfloat16 (nearest even) and back, as float64."""
    f = np.ascontiguousarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def shift(x: np.ndarray, tap: int) -> np.ndarray:
    """x_tap[b, y, x] = x[b, (y+ky-1) % H, (x+kx-1) % W]."""
    ky, kx = divmod(tap, 3)
    return np.roll(x, shift=(1 - ky, 1 - kx), axis=(1, 2))


def unshift(x: np.ndarray, tap: int) -> np.ndarray:
    ky, kx = divmod(tap, 3)
    return np.roll(x, shift=(ky - 1, kx - 1), axis=(1, 2))


def conv(x: np.ndarray, w: np.ndarray) -> np.ndarray:
    out = 0.0
    for t in range(9):
        out = out + shift(x, t) @ w[:, t, :].T
    return out


def conv_input_grad(dy: np.ndarray, w: np.ndarray) -> np.ndarray:
    dx = 0.0
    for t in range(9):
        dx = dx + unshift(dy @ w[:, t, :], t)
    return dx


def conv_weight_grad(x: np.ndarray, dy: np.ndarray) -> np.ndarray:
    """[cout, 9, cin]"""
    cout, cin = dy.shape[-1], x.shape[-1]
    g = np.empty((cout, 9, cin))
    dyf = dy.reshape(-1, cout)
    for t in range(9):
        g[:, t, :] = dyf.T @ shift(x, t).reshape(-1, cin)
    return g


GELU_C = np.sqrt(2.0 / np.pi)
GELU_A = 0.044715


def gelu(x):
    """GELU in its tanh form (Hendrycks & Gimpel 2016), the form the GPU
    epilogues compute: x/2 (1 + tanh(sqrt(2/pi) (x + 0.044715 x^3)))."""
    return 0.5 * x * (1.0 + np.tanh(GELU_C * (x + GELU_A * x ** 3)))


def gelu_grad(x):
    t = np.tanh(GELU_C * (x + GELU_A * x ** 3))
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * GELU_C * (1.0 + 3.0 * GELU_A * x * x)


def layer_shapes():
    """[(name, cout, cin)] in network order."""
    out = [("in", CH, NF)]
    for i in range(NBLOCKS):
        out += [(f"b{i}c1", CH, CH), (f"b{i}c2", CH, CH)]
    out.append(("out", NF, CH))
    return out


def init_params(seed: int = 0, out_scale: float = 0.1) -> dict:
    """He-style initialisation (std sqrt(2 / fan_in)); the output layer and
    each block's second convolution start scaled by out_scale so the
    untrained network is close to the identity map."""
    rng = np.random.default_rng(seed)
    p = {}
    for name, cout, cin in layer_shapes():
        std = np.sqrt(2.0 / (9 * cin))
        if name == "out" or name.endswith("c2"):
            std *= out_scale
        p[name + ".w"] = rng.normal(0.0, std, (cout, 9, cin))
        p[name + ".b"] = np.zeros(cout)
    return p


def forward(p: dict, x: np.ndarray, bf: bool = False):
    """x: [B, H, W, 5] fields. Returns (prediction [B, H, W, 5], cache)."""
    R = bf16 if bf else (lambda a: a)
    W = {k: (R(v) if k.endswith(".w") else v) for k, v in p.items()}
    xin = R(x)
    h = R(conv(xin, W["in.w"]) + W["in.b"])
    cache = {"xin": xin, "h": [h], "t": [], "u": [], "W": W}
    for i in range(NBLOCKS):
        t = conv(h, W[f"b{i}c1.w"]) + W[f"b{i}c1.b"]
        u = R(gelu(t))
        cache["t"].append(R(t))
        cache["u"].append(u)
        h = R(conv(u, W[f"b{i}c2.w"]) + W[f"b{i}c2.b"] + h)
        cache["h"].append(h)
    pred = conv(h, W["out.w"]) + W["out.b"] + x
    return pred, cache


def loss_and_grads(p: dict, x: np.ndarray, target: np.ndarray, bf: bool = False):
    """Mean squared error over all B*H*W*5 values and its gradients
    {name.w: [cout, 9, cin], name.b: [cout]}."""
    R = bf16 if bf else (lambda a: a)
    pred, c = forward(p, x, bf)
    W = c["W"]
    e = pred - target
    loss = float(np.mean(e * e))
    dout = R(2.0 * e / e.size)
    g = {}
    h6 = c["h"][-1]
    g["out.w"] = conv_weight_grad(h6, dout)
    g["out.b"] = dout.reshape(-1, NF).sum(axis=0)
    dh = R(conv_input_grad(dout, W["out.w"]))
    for i in reversed(range(NBLOCKS)):
        u, t, h = c["u"][i], c["t"][i], c["h"][i]
        g[f"b{i}c2.w"] = conv_weight_grad(u, dh)
        g[f"b{i}c2.b"] = dh.reshape(-1, CH).sum(axis=0)
        dt = R(conv_input_grad(dh, W[f"b{i}c2.w"]) * gelu_grad(t))
        g[f"b{i}c1.w"] = conv_weight_grad(h, dt)
        g[f"b{i}c1.b"] = dt.reshape(-1, CH).sum(axis=0)
        dh = R(conv_input_grad(dt, W[f"b{i}c1.w"]) + dh)
    g["in.w"] = conv_weight_grad(c["xin"], dh)
    g["in.b"] = dh.reshape(-1, CH).sum(axis=0)
    return loss, pred, g


def adamw(p: dict, m: dict, v: dict, g: dict, step: int, lr: float, beta1: float = 0.9,
          beta2: float = 0.999, eps: float = 1e-8, wd: float = 0.01):
    """One AdamW step in place (decoupled weight decay on weights only)."""
    bc1, bc2 = 1 - beta1 ** step, 1 - beta2 ** step
    for k in p:
        m[k] = beta1 * m[k] + (1 - beta1) * g[k]
        v[k] = beta2 * v[k] + (1 - beta2) * g[k] ** 2
        upd = (m[k] / bc1) / (np.sqrt(v[k] / bc2) + eps)
        if k.endswith(".w"):
            upd = upd + wd * p[k]
        p[k] = p[k] - lr * upd
