"""The autotuner on the device: it measures every candidate schedule, the
table it installs drives later batches, and every alternative schedule it
can pick computes the same curves as the oracle (FP64 to 1e-10, mixed to
1e-6 in echo error)."""
import numpy as np
import pytest

import spin_systems_b200 as ss
from spin_systems_b200 import abi, workloads

pytestmark = pytest.mark.gpu


def _spec():
    spec = workloads.cpmg_uneven(realizations=8, pulses=2)
    spec.spin_choices = (10, 11, 12, 13)
    spec.nspins = 16
    spec.tau_range = (0.05, 0.2)
    return spec


def test_tuner_fills_the_table_and_writes_the_cache(engine, tmp_path):
    ss.clear_schedule()
    spec = _spec()
    cache = tmp_path / "sched.tsv"
    rows = ss.tune(engine, spec.config(), 0, 8, abi.MIXED, cache)
    keys = {(r["L"], r["precision"]) for r in rows}
    assert keys == {(L, p) for L in (10, 11, 12, 13) for p in ("mixed", "fp64")}
    assert all(r["ns"] > 0 for r in rows)
    ss.clear_schedule()
    ss.load_schedule(cache)
    assert {(r["L"], r["precision"], r["variant"]) for r in ss.schedule()} == {
        (r["L"], r["precision"], r["variant"]) for r in rows}


def test_tuner_times_fp64_only_where_mixed_realisations_can_route(engine):
    # The default limit keeps L = 16 mixed, so a mixed tune there installs
    # no FP64 schedule; an explicit limit routes L = 16 and tunes its FP64
    # (split-cluster) kernel as well.
    spec = _spec()
    spec.spin_choices = (16,)
    for limit, want in ((0, {"mixed"}), (40000, {"mixed", "fp64"})):
        ss.clear_schedule()
        spec.mixed_order_limit = limit
        rows = ss.tune(engine, spec.config(), 0, 4, abi.MIXED)
        assert {r["precision"] for r in rows if r["L"] == 16} == want
    ss.clear_schedule()


@pytest.mark.parametrize("variant", ["L10.R3.f32.smem.c1", "L11.R3.f32.smem.c1",
                                     "L12.R3.f32.smem.c1", "L13.R4.f32.global.c2",
                                     "L11.R4.f64.smem.c1", "L12.R3.f64.global.c2",
                                     "L14.R5.f32.global.c2", "L15.R5.f32.global.c4",
                                     "L16.R5.f32.global.c8", "L12.R4.f64.global.c1",
                                     "L12.R4.f32.reg.c1", "L12.R3.f64.reg.c1",
                                     "L12.R4.f64.reg.c1", "L11.R4.f32.reg.c1",
                                     "L10.R4.f32.reg.c1", "L10.R3.f64.reg.c1",
                                     "L11.R3.f64.reg.c1", "L14.R4.f32.global.c2.split",
                                     "L15.R4.f32.global.c4.split",
                                     "L16.R4.f32.global.c8.split"])
def test_every_alternative_schedule_matches_the_oracle(engine, port, tmp_path, variant):
    ss.clear_schedule()
    spec = _spec()
    cfg = spec.config()
    ss.tune(engine, cfg, 0, 2, abi.FP64)  # learns the device name
    dev = ss.schedule()[0]["device"]
    L = int(variant.split(".")[0][1:])
    prec = "mixed" if ".f32." in variant else "fp64"
    p = tmp_path / "force.tsv"
    p.write_text(f"{dev}\t{L}\t{prec}\t{variant}\t1.0\n")
    ss.clear_schedule()
    ss.load_schedule(p)
    spec.spin_choices = (L,)
    cfg = spec.config()
    want = np.stack([port.run_realization(cfg, i)[1] for i in range(3)])
    _, rows = ss.Batch(engine, cfg, 0, 3, abi.MIXED if prec == "mixed" else abi.FP64).run()
    if prec == "fp64":
        assert np.abs(rows - want).max() < 1e-10
    else:
        scale = []
        for i in range(3):
            s = ss.realization_setup(cfg, i, 16)
            psi = s["psi0"][0::2] + 1j * s["psi0"][1::2]
            k = np.arange(1 << s["L"])
            ref = sum(psi[k ^ (1 << q)] for q in range(s["L"]))
            scale.append(np.vdot(ref, ref).real)
        err = np.abs(rows[:, :, 0] - want[:, :, 0]).max(axis=1) / np.array(scale)
        assert err.max() < 1e-6
    ss.clear_schedule()
