"""CPU oracle of the learned-densification network (test infrastructure: only tests, the
smoke check and the benchmark's baseline leg use it, as the checker).

The network has no counterpart in the reference: it proposes, per Gaussian, one of
{keep, clone/split, prune} beside the reference's threshold rule (src/densify.rs:125-221).
16 input features -> 64 SiLU -> 64 SiLU -> 3 logits -> softmax. Parameters are one flat
float vector laid out as W1 [16][64], b1 [64], W2 [64][64], b2 [64], W3 [64][3], b3 [3]
(W[in][out]).

`forward` / `backward` evaluate it in float64. With `bf16=True` they round to bfloat16
(round to nearest even) exactly where the tensor-core kernels do: the inputs, the weights,
the hidden activations before each product, and in the backward the logit gradient and
the hidden-layer gradients before each product; sums stay wide. The loss is the weighted
mean cross-entropy  L = sum_s w_s * -log p_s[y_s] / sum_s w_s.
"""
from __future__ import annotations

import numpy as np

IN, HID, OUT = 16, 64, 3
SIZES = [("W1", (IN, HID)), ("b1", (HID,)), ("W2", (HID, HID)), ("b2", (HID,)), ("W3", (HID, OUT)), ("b3", (OUT,))]
NUM_PARAMS = sum(int(np.prod(s)) for _, s in SIZES)


def unpack(theta):
    out, o = {}, 0
    for name, shape in SIZES:
        k = int(np.prod(shape))
        out[name] = np.asarray(theta[o:o + k], np.float64).reshape(shape)
        o += k
    return out


def pack(parts):
    return np.concatenate([np.asarray(parts[name], np.float64).ravel() for name, _ in SIZES])


def bf16(x):
    """Round float64 values to bfloat16 (through float32, round to nearest even)."""
    f = np.asarray(x, np.float32).copy()
    u = f.view(np.uint32)
    rnd = ((u >> 16) & 1) + np.uint32(0x7FFF)
    u = ((u + rnd) & np.uint32(0xFFFF0000)).astype(np.uint32)
    return u.view(np.float32).astype(np.float64)


def silu(z):
    return z / (1.0 + np.exp(-z))


def silu_grad(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def init_params(seed=0):
    """Xavier-uniform weights, zero biases."""
    rng = np.random.default_rng(seed)
    parts = {}
    for name, shape in SIZES:
        if name.startswith("W"):
            lim = np.sqrt(6.0 / (shape[0] + shape[1]))
            parts[name] = rng.uniform(-lim, lim, shape)
        else:
            parts[name] = np.zeros(shape)
    return pack(parts)


def forward(theta, x, bf16_like=False):
    """Returns (probabilities (n,3), cache)."""
    p = unpack(theta)
    r = bf16 if bf16_like else (lambda a: np.asarray(a, np.float64))
    x = r(x)
    z1 = x @ r(p["W1"]) + p["b1"]
    h1 = r(silu(z1))
    z2 = h1 @ r(p["W2"]) + p["b2"]
    h2 = r(silu(z2))
    z3 = h2 @ r(p["W3"]) + p["b3"]
    z = z3 - z3.max(1, keepdims=True)
    e = np.exp(z)
    prob = e / e.sum(1, keepdims=True)
    return prob, dict(x=x, z1=z1, h1=h1, z2=z2, h2=h2, prob=prob, p=p)


def loss(theta, x, y, w, bf16_like=False):
    prob, _ = forward(theta, x, bf16_like)
    n = np.arange(len(y))
    return float(np.sum(w * -np.log(prob[n, y])) / np.sum(w))


def backward(theta, x, y, w, bf16_like=False):
    """Gradient of `loss` with respect to theta (flat, float64)."""
    prob, c = forward(theta, x, bf16_like)
    p = c["p"]
    r = bf16 if bf16_like else (lambda a: np.asarray(a, np.float64))
    n = len(y)
    onehot = np.zeros((n, OUT))
    onehot[np.arange(n), y] = 1.0
    dz3 = (prob - onehot) * (w / np.sum(w))[:, None]
    g = {}
    dz3r = r(dz3)
    g["W3"] = c["h2"].T @ dz3r
    g["b3"] = dz3.sum(0)
    dh2 = dz3r @ r(p["W3"]).T
    dz2 = dh2 * silu_grad(c["z2"])
    dz2r = r(dz2)
    g["W2"] = c["h1"].T @ dz2r
    g["b2"] = dz2.sum(0)
    dh1 = dz2r @ r(p["W2"]).T
    dz1 = dh1 * silu_grad(c["z1"])
    dz1r = r(dz1)
    g["W1"] = c["x"].T @ dz1r
    g["b1"] = dz1.sum(0)
    return pack(g)


def adam(theta, grad, m, v, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    """Adam in float32 arithmetic (the device update), in place; returns theta."""
    t32 = np.asarray(theta, np.float32)
    g = np.asarray(grad, np.float32)
    m[:] = np.float32(b1) * m + np.float32(1 - b1) * g
    v[:] = np.float32(b2) * v + np.float32(1 - b2) * g * g
    mh = m / np.float32(1 - b1 ** step)
    vh = v / np.float32(1 - b2 ** step)
    t32 -= np.float32(lr) * mh / (np.sqrt(vh) + np.float32(eps))
    return t32
