"""The surrogate network's tensor-core kernels against the CPU oracle
(oracle/mlp_oracle.py), through the C ABI.

Tolerances, written here and derived from where the two paths differ: both
round to BF16 at the same points; the device accumulates in FP32 in its own
order (relative ~1e-6 of each dot product), which occasionally moves a
hidden activation across a BF16 rounding boundary (one BF16 ulp, 2^-8
relative, on that element).
  GEMM              |c - c64| <= 2e-6 * sum_k |a_k b_k| per element
  forward           max |y - y_ref| <= 2e-3, rms <= 2e-4
  gradients         relative L2 error <= 5e-3 per tensor, loss 1e-5
"""
import numpy as np
import pytest

import spin_systems_b200 as ss
from oracle import mlp_oracle as mo

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("M,N,K", [(128, 256, 64), (256, 256, 256), (1024, 128, 256),
                                   (256, 64, 1024), (384, 16, 128), (128, 48, 512)])
def test_gemm_matches_float64(engine, M, N, K):
    rng = np.random.default_rng(M * 7 + N * 3 + K)
    a = mo.bf16(rng.normal(0, 1, size=(M, K)))
    b = mo.bf16(rng.normal(0, 1, size=(N, K)))
    c = ss.mlp_gemm_test(engine, mo.bf16_bits(a), mo.bf16_bits(b))
    ref = a @ b.T
    bound = 2e-6 * (np.abs(a) @ np.abs(b).T) + 1e-30
    err = np.abs(c - ref)
    assert (err <= bound).all(), f"max err {err.max():.3g}, worst ratio {(err / bound).max():.3g}"


def test_gemm_rejects_shapes_outside_the_tiling(engine):
    a = np.zeros((100, 64), dtype=np.uint16)
    b = np.zeros((16, 64), dtype=np.uint16)
    with pytest.raises(ss.InvalidArgumentError):
        ss.mlp_gemm_test(engine, a, b)


@pytest.fixture(scope="module")
def net(engine):
    n = ss.Mlp(engine, batch=256, seed=5)
    yield n
    n._destroy()


def _case(rows, seed):
    rng = np.random.default_rng(seed)
    x = rng.uniform(-1, 1, size=(rows, 6)).astype(np.float32)
    t = (0.5 * np.sin(np.outer(x[:, 0] + 0.5 * x[:, 2], np.linspace(0, 3, 128)))
         * np.exp(-np.abs(x[:, 1:2]))).astype(np.float32)
    return x, t


def test_forward_matches_oracle(net):
    p = mo.init_params(11).astype(np.float32)
    net.set_params(p)
    assert np.array_equal(net.params(), p)
    x, _ = _case(300, 1)          # two device passes, the second one ragged
    y = net.forward(x)
    ref, _ = mo.forward(p.astype(np.float64), x.astype(np.float64))
    err = np.abs(y - ref)
    assert err.max() <= 2e-3 and np.sqrt((err ** 2).mean()) <= 2e-4, (err.max(), np.sqrt((err ** 2).mean()))


def test_gradients_match_oracle(net):
    p = mo.init_params(12).astype(np.float32)
    net.set_params(p)
    x, t = _case(200, 2)          # 200 of 256 rows: the loss masks the padding
    loss, g = net.gradients(x, t)
    ref_loss, ref_g = mo.gradients(p.astype(np.float64), x.astype(np.float64), t.astype(np.float64))
    assert abs(loss - ref_loss) <= 1e-5 * ref_loss
    at = 0
    for i, o in mo.SIZES:
        for size in (i * o, o):
            a, b = g[at:at + size], ref_g[at:at + size]
            rel = np.linalg.norm(a - b) / np.linalg.norm(b)
            assert rel <= 5e-3, (at, size, rel)
            at += size


def test_adam_step_matches_oracle(net):
    p = mo.init_params(13).astype(np.float32)
    net.set_params(p)
    x, t = _case(256, 3)          # the whole set is one batch: any shuffle, same step
    _, g = net.gradients(x, t)
    net.set_params(p)
    net.set_data(x, t)
    lr = 1e-3
    net.train(1, lr, lr, seed=1)
    p1 = net.params().astype(np.float64)
    want, _, _ = mo.adam_step(p.astype(np.float64), 0.0, 0.0, g.astype(np.float64), lr, 1)
    big = np.abs(g) > 1e-5        # below this the step depends on accumulation order
    diff = np.abs(p1 - want)
    assert diff[big].max() <= 2e-3 * lr + 1e-7, diff[big].max()
    assert (diff > 0.05 * lr).mean() < 1e-3


def test_training_reduces_the_loss(engine):
    n = ss.Mlp(engine, batch=256, seed=9)
    x, t = _case(4096, 4)
    n.set_data(x, t)
    losses = n.train(400, 2e-3, 1e-4, seed=3)
    assert np.isfinite(losses).all()
    assert losses[-20:].mean() < 0.1 * losses[:5].mean(), (losses[:5], losses[-20:])
    n._destroy()
