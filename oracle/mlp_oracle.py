"""TEST INFRASTRUCTURE (the checker), not product code.

Float64 CPU restatement of the proposal network of include/mbs_mlp.h
(4 -> 128 -> 128 -> 128 -> 1, erf GELU, mean-squared loss) with its
analytic backward pass.  With ``bf16=True`` it rounds weights, inputs,
activations and back-propagated gradients to BF16 (round to nearest even) at
the points where the CUDA kernels hold them in BF16, so the GPU gradients can
be checked tightly; with ``bf16=False`` it is the exact float64 network.
The MLP has no reference counterpart; this restatement is its oracle.
"""
from __future__ import annotations

import math

import numpy as np

H, IN = 128, 4
_erf = np.vectorize(math.erf)


def split(params: np.ndarray) -> dict:
    p = np.asarray(params, dtype=np.float64)
    o, out = 0, {}
    for name, shape in (("W1", (H, IN)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)),
                        ("W3", (H, H)), ("b3", (H,)), ("w4", (H,)), ("b4", (1,))):
        n = int(np.prod(shape))
        out[name] = p[o:o + n].reshape(shape)
        o += n
    assert o == len(p)
    return out


def flat(d: dict) -> np.ndarray:
    return np.concatenate([d[k].ravel() for k in ("W1", "b1", "W2", "b2", "W3", "b3", "w4", "b4")])


def bf16(x: np.ndarray) -> np.ndarray:
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    f = np.asarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(z):
    return 0.5 * z * (1.0 + _erf(z / math.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + _erf(z / math.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / math.sqrt(2 * math.pi)


def forward(params, q, bf16_round: bool = False):
    P = split(params)
    r = bf16 if bf16_round else (lambda a: np.asarray(a, dtype=np.float64))
    x0 = r(q)
    W1, W2, W3 = r(P["W1"]), r(P["W2"]), r(P["W3"])
    z1 = x0 @ W1.T + P["b1"]
    h1 = r(gelu(z1))
    z2 = h1 @ W2.T + P["b2"]
    h2 = r(gelu(z2))
    z3 = h2 @ W3.T + P["b3"]
    h3 = r(gelu(z3))
    y = h3 @ P["w4"] + P["b4"][0]
    return y, (x0, z1, h1, z2, h2, z3, h3, W1, W2, W3)


def loss_grad(params, q, t, bf16_round: bool = False):
    """Mean-squared loss and its gradient (flat order of include/mbs_mlp.h)."""
    P = split(params)
    r = bf16 if bf16_round else (lambda a: np.asarray(a, dtype=np.float64))
    y, (x0, z1, h1, z2, h2, z3, h3, W1, W2, W3) = forward(params, q, bf16_round)
    n = len(t)
    d = y - t
    loss = float(np.mean(d * d))
    dy = 2.0 * d / n
    g = {"w4": h3.T @ dy, "b4": np.array([dy.sum()])}
    dz3 = r(dy[:, None] * P["w4"][None, :] * gelu_grad(z3))
    g["W3"] = dz3.T @ h2
    g["b3"] = dz3.sum(axis=0)
    dz2 = r((dz3 @ W3) * gelu_grad(z2))
    g["W2"] = dz2.T @ h1
    g["b2"] = dz2.sum(axis=0)
    dz1 = r((dz2 @ W2) * gelu_grad(z1))
    g["W1"] = dz1.T @ x0
    g["b1"] = dz1.sum(axis=0)
    return loss, flat(g)
