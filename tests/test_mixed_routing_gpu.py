"""Mixed precision's default routing on the device: with the per-size order
limits, every curve of a mixed batch stays within 1e-6 echo error of the
FP64 batch on the same realisations (echo error: max over time of
|corr_x mixed - FP64| / <ref|ref>).  Small sizes are where the FP32
recursion's rounding averages out least; L = 16 (not routed by default) is
checked on 64 realisations of the XY-8 program with finite pulses."""
import numpy as np
import pytest

import spin_systems_b200 as ss
from spin_systems_b200 import abi, workloads
from spin_systems_b200.experiments import corr0

pytestmark = pytest.mark.gpu


def echo_errors(engine, spec, n):
    cfg = spec.config()
    bm = ss.Batch(engine, cfg, 0, n, abi.MIXED)
    _, mixed = bm.run()
    prec, _ = bm.work()
    bm._destroy()
    b64 = ss.Batch(engine, cfg, 0, n, abi.FP64)
    _, fp64 = b64.run()
    b64._destroy()
    scale = corr0(cfg, range(n), 16)
    return np.abs(mixed[:, :, 0] - fp64[:, :, 0]).max(axis=1) / scale, prec


@pytest.mark.parametrize("L,n", [(8, 1024), (10, 512)])
def test_small_sizes_stay_within_budget(engine, L, n):
    spec = workloads.cpmg_uneven(realizations=n)
    spec.spin_choices = (L,)
    err, prec = echo_errors(engine, spec, n)
    assert err.max() <= 1e-6, (err.max(), int((err > 1e-6).sum()))
    assert (prec == abi.FP64).any() and (prec == abi.MIXED).sum() > n // 2


def test_l16_xy8_sixty_four_realisations(engine):
    err, prec = echo_errors(engine, workloads.xy8_finite(nspins=16, realizations=64), 64)
    assert (prec == abi.MIXED).all()
    assert err.max() <= 1e-6, err.max()
