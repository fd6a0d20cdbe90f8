"""CPU oracle of the echo surrogate's network -- test infrastructure only.

This file is the checker for the device MLP (spin_systems_b200/csrc/mlp.cu):
tests import it to compare forward outputs, gradients and Adam steps.  The
product never imports it.

The network is the learned-surrogate workload's:
6 -> 256 -> 256 -> 256 -> 128, GELU (erf form) on the three hidden layers, a
linear output layer and a mean-squared-error loss.  Everything here runs in
float64.  With ``bf16=True`` the oracle rounds exactly where the device path
rounds to BF16 -- inputs, weights, hidden activations and the backward
layer gradients fed to the products -- so the only remaining difference is
the device's FP32 accumulation order.  With ``bf16=False`` it is the exact
float64 network, whose analytic gradient is checked against central finite
differences.

The reference (spinsim) has no learned component; there is no reference
file to cite for this oracle.  Parameter layout follows the C ABI:
flat W0[256][6] b0 W1[256][256] b1 W2[256][256] b2 W3[128][256] b3.
"""
from __future__ import annotations

import math

import numpy as np

SIZES = [(6, 256), (256, 256), (256, 256), (256, 128)]
PARAM_COUNT = sum(i * o + o for i, o in SIZES)

_erf = np.vectorize(math.erf, otypes=[np.float64])


def bf16(a: np.ndarray) -> np.ndarray:
    """Round to the nearest BF16 value (ties to even), returned as float64."""
    f = np.ascontiguousarray(a, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def bf16_bits(a: np.ndarray) -> np.ndarray:
    """Raw BF16 bit patterns (uint16) of the rounded values."""
    return (bf16(a).astype(np.float32).view(np.uint32) >> 16).astype(np.uint16)


def gelu(z):
    return 0.5 * z * (1.0 + _erf(z / math.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + _erf(z / math.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / math.sqrt(2.0 * math.pi)


def unpack(params: np.ndarray):
    """Flat parameter vector -> [(W [out][in], b [out])]."""
    p = np.asarray(params, dtype=np.float64)
    out, at = [], 0
    for i, o in SIZES:
        w = p[at:at + i * o].reshape(o, i)
        at += i * o
        b = p[at:at + o]
        at += o
        out.append((w, b))
    assert at == p.size == PARAM_COUNT
    return out


def pack(parts) -> np.ndarray:
    return np.concatenate([np.concatenate([w.ravel(), b.ravel()]) for w, b in parts])


def forward(params, x, bf16_path=True):
    """Returns (y, cache) for inputs x [rows][6]."""
    r = bf16 if bf16_path else (lambda a: np.asarray(a, dtype=np.float64))
    layers = unpack(params)
    a = r(x)
    cache = {"a": [a], "z": []}
    for li, (w, b) in enumerate(layers):
        z = a @ r(w).T + b
        if li < len(layers) - 1:
            cache["z"].append(z)
            a = r(gelu(z))
            cache["a"].append(a)
        else:
            return z, cache
    raise AssertionError


def gradients(params, x, target, bf16_path=True):
    """(loss, flat gradient) of the mean-squared error over rows and outputs."""
    r = bf16 if bf16_path else (lambda a: np.asarray(a, dtype=np.float64))
    layers = unpack(params)
    y, cache = forward(params, x, bf16_path)
    n = y.shape[0]
    d = y - target
    loss = float((d * d).sum() / (n * y.shape[1]))
    g = 2.0 * d / (n * y.shape[1])           # FP32-held layer gradient
    grads = [None] * len(layers)
    for li in range(len(layers) - 1, -1, -1):
        w, _ = layers[li]
        dz = r(g)                            # what the products read
        a_in = cache["a"][li]
        gw = dz.T @ a_in
        gb = g.sum(axis=0)
        grads[li] = (gw, gb)
        if li > 0:
            dh = dz @ r(w)
            g = dh * gelu_grad(cache["z"][li - 1])
    return loss, pack(grads)


def adam_step(params, m, v, grads, lr, step, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam step as the device applies it (bias correction folded into
    the learning rate).  Returns new (params, m, v)."""
    m = b1 * m + (1 - b1) * grads
    v = b2 * v + (1 - b2) * grads * grads
    lr_t = lr * math.sqrt(1 - b2 ** step) / (1 - b1 ** step)
    return params - lr_t * m / (np.sqrt(v) + eps), m, v


def init_params(seed: int = 0) -> np.ndarray:
    """A random parameter vector of the device's initial scale (any values
    do for the checks; this is not the device's initialiser)."""
    rng = np.random.default_rng(seed)
    parts = []
    for li, (i, o) in enumerate(SIZES):
        a = (math.sqrt(6.0) if li < 3 else math.sqrt(3.0)) / math.sqrt(i)
        parts.append((rng.uniform(-a, a, size=(o, i)), rng.normal(0, 0.05, size=o)))
    return pack(parts)
