"""The surrogate network's CPU oracle pinned on its own (no GPU): BF16
rounding against known values, the float64 gradient against central finite
differences, the Adam step against its closed form, and the parameter count
against the C ABI."""
import math

import numpy as np

from oracle import mlp_oracle as mo


def test_bf16_rounding_known_values():
    one = 1.0
    ulp = 2.0 ** -7            # BF16 spacing just above 1
    x = np.array([one, one + ulp / 2, one + 3 * ulp / 2, one + ulp / 4, -2.5, 65504.0])
    got = mo.bf16(x)
    # ties go to even: 1 + ulp/2 -> 1, 1 + 3ulp/2 -> 1 + 2ulp; 65504 rounds up to 2^16
    assert list(got) == [1.0, 1.0, 1.0 + 2 * ulp, 1.0, -2.5, 65536.0]
    bits = mo.bf16_bits(np.array([1.0, -2.0, 0.5]))
    assert list(bits) == [0x3F80, 0xC000, 0x3F00]


def test_pack_roundtrip_and_count(lib):
    p = mo.init_params(3)
    assert p.size == mo.PARAM_COUNT == 166272
    assert np.array_equal(mo.pack(mo.unpack(p)), p)
    lib.ss_mlp_param_count.restype = __import__("ctypes").c_int64
    assert lib.ss_mlp_param_count() == mo.PARAM_COUNT


def test_float64_gradient_matches_finite_differences():
    rng = np.random.default_rng(7)
    p = mo.init_params(1)
    x = rng.uniform(-1, 1, size=(5, 6))
    t = rng.normal(0, 0.5, size=(5, 128))
    loss, g = mo.gradients(p, x, t, bf16_path=False)
    assert loss > 0
    # every tensor: a few random coordinates
    idx = np.concatenate([rng.integers(a, b, 6) for a, b in _segments()])
    h = 1e-6
    for i in idx:
        e = np.zeros_like(p)
        e[i] = h
        lp, _ = mo.gradients(p + e, x, t, bf16_path=False)
        lm, _ = mo.gradients(p - e, x, t, bf16_path=False)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-7 + 1e-5 * abs(fd), (i, fd, g[i])


def test_adam_step_closed_form():
    p = np.array([1.0, -1.0, 0.5])
    g = np.array([0.2, -0.4, 0.0])
    p1, m, v = mo.adam_step(p, np.zeros(3), np.zeros(3), g, lr=0.01, step=1)
    # first step: lr * g / (|g| + eps / sqrt(1 - b2)) per coordinate
    want = p - 0.01 * g / (np.abs(g) + 1e-8 / math.sqrt(1 - 0.999))
    assert np.allclose(p1, want, rtol=0, atol=1e-12)
    assert np.allclose(m, 0.1 * g) and np.allclose(v, 0.001 * g * g)


def _segments():
    at = 0
    for i, o in mo.SIZES:
        yield at, at + i * o
        at += i * o
        yield at, at + o
        at += o
