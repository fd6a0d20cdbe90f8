"""The autotuner's host side (no GPU): the compiled schedule list and the
schedule cache format."""
import pytest

import spin_systems_b200 as ss


def test_every_size_has_a_default_and_the_alternatives_are_listed():
    names = [v[0] for v in ss.variants()]
    assert len(names) == len(set(names))
    sizes_mixed = {int(n.split(".")[0][1:]) for n in names if ".f32." in n}
    sizes_fp64 = {int(n.split(".")[0][1:]) for n in names if ".f64." in n}
    assert sizes_mixed == set(range(6, 17)) and sizes_fp64 == set(range(6, 17))
    # sizes with a choice to make
    for L in (10, 11, 12, 13, 14, 15, 16):
        assert sum(n.startswith(f"L{L}.") and ".f32." in n for n in names) >= 2
    assert "L16.R4.f32.global.c8" in names
    # state and reference on clusters of their own at the cluster sizes
    assert {"L14.R4.f32.global.c2.split", "L15.R4.f32.global.c4.split",
            "L16.R4.f32.global.c8.split", "L16.R3.f64.global.c16.split"} <= set(names)
    for name, threads, smem in ss.variants():
        assert 32 <= threads <= 1024 and smem <= 232448


def test_schedule_cache_roundtrip(tmp_path):
    ss.clear_schedule()
    p = tmp_path / "sched.tsv"
    p.write_text("# comment\nNVIDIA B200\t12\tmixed\tL12.R3.f32.smem.c1\t0.025\n"
                 "NVIDIA B200\t12\tfp64\tL12.R3.f64.global.c1\t0.04\n")
    ss.load_schedule(p)
    rows = ss.schedule()
    assert {(r["L"], r["precision"], r["variant"]) for r in rows} == {
        (12, "mixed", "L12.R3.f32.smem.c1"), (12, "fp64", "L12.R3.f64.global.c1")}
    ss.clear_schedule()
    assert ss.schedule() == []


def test_malformed_cache_is_a_config_error(tmp_path):
    p = tmp_path / "bad.tsv"
    p.write_text("NVIDIA B200\ttwelve\tmixed\tL12.R3.f32.smem.c1\t0.1\n")
    with pytest.raises(ss.SpinsimError) as e:
        ss.load_schedule(p)
    assert e.value.kind == "config"
    ss.clear_schedule()
    with pytest.raises(ss.InvalidArgumentError):
        ss.load_schedule(tmp_path / "missing.tsv")


def test_snapshot_budget_is_a_byte_count():
    with pytest.raises(ss.SpinsimError) as e:
        ss.set_snapshot_budget(-1)
    assert e.value.kind == "invalid_argument"
    ss.set_snapshot_budget(0)
    ss.set_snapshot_budget(16 << 30)
