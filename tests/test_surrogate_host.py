"""Host logic of the learned echo surrogate (no GPU): the parameter space,
network features, the pulse programs, the nearest-neighbour baseline and the
fallback's error model."""
import numpy as np

from spin_systems_b200 import surrogate as sg


def test_sample_and_features_cover_the_space():
    p = sg.sample(2000, 3)
    for k, (lo, hi) in sg.RANGES.items():
        assert p[k].min() >= lo and p[k].max() <= hi
    assert set(np.unique(p["nspins"])) == {10, 12, 14}
    assert set(np.unique(p["sequence"])) == {0, 1}
    x = sg.features(p)
    assert x.shape == (2000, 6) and x.dtype == np.float32
    assert x.min() >= -1.0 and x.max() <= 1.0
    assert set(np.unique(x[:, 5])) == {-1.0, 0.0, 1.0}


def test_programs_measure_128_times():
    for seq in (0, 1):
        spec = sg.sweep_spec(seq, 10, [(1.0, 0.5, 0.3, 1.0)], 4)
        assert spec.measurement_count() == sg.POINTS
        cfg = spec.config()
        assert cfg.sweep_points == 1
        assert [cfg.sweep_params[i] for i in range(4)] == [1.0, 0.5, 0.3, 1.0]


def test_nearest_neighbour_returns_the_closest_curve_of_the_same_kind():
    p = sg.sample(50, 1, sizes=(10, 12))
    y = np.arange(50, dtype=float)[:, None] * np.ones((1, sg.POINTS))
    q = p[[7, 21]].copy()
    q["tau"] += 1e-6
    got = sg.nearest_neighbour(p, y, q)
    assert got[0, 0] == 7 and got[1, 0] == 21


def test_error_model_takes_the_worst_near_calibration_point():
    s = object.__new__(sg.Surrogate)
    p = sg.sample(64, 2, sizes=(10,), sequences=(0,))
    s.cal_p, s.cal_x = p, sg.features(p)
    s.cal_err = np.full(64, 1e-4)
    s.cal_err[5] = 5e-3
    q = p[[5]].copy()
    est = s.estimate_error(q, k=4, safety=1.0)
    assert est[0] == 5e-3
    far = p[[5]].copy()
    far["nspins"] = 12
    assert np.isinf(s.estimate_error(far)[0])


def test_vectorised_nearest_matches_brute_force():
    rng = np.random.default_rng(4)
    ref = rng.normal(size=(300, 4))
    q = rng.normal(size=(1000, 4))
    got = sg._nearest(ref, q, 5, chunk=128)
    d = ((q[:, None, :] - ref[None, :, :]) ** 2).sum(axis=2)
    want = np.sort(d, axis=1)[:, :5]
    assert np.allclose(np.sort(np.take_along_axis(d, got, axis=1), axis=1), want)
    one = sg._nearest(ref, q, 1)[:, 0]
    assert np.array_equal(one, d.argmin(axis=1))
    # fewer reference rows than k: every row, padded with the last index
    small = sg._nearest(ref[:3], q[:7], 5)
    assert small.shape == (7, 5) and set(np.unique(small)) <= {0, 1, 2}


def test_split_counts_hold_out_the_requested_points():
    tr, cal, te = sg.split_counts([32768, 8192, 1536], 4096)
    assert sum(te) == 4096
    assert cal == [3276, 819, 153]
    assert [a + b + c for a, b, c in zip(tr, cal, te)] == [32768, 8192, 1536]
    # in proportion to each size's points
    assert te[0] > te[1] > te[2] > 0
    tr, cal, te = sg.split_counts([1000, 500], 0)
    assert te == [100, 50] and cal == [100, 50] and tr == [800, 400]


def test_saved_curves_load_back(tmp_path):
    data = {10: (sg.sample(5, 1, sizes=(10,)), np.linspace(0, 1, 5 * sg.POINTS).reshape(5, -1)),
            12: (sg.sample(3, 2, sizes=(12,)), np.ones((3, sg.POINTS)))}
    path = tmp_path / "curves.npz"
    sg.save_data(str(path), data, 64)
    got, realizations = sg.load_data(str(path))
    assert realizations == 64 and sorted(got) == [10, 12]
    for L in (10, 12):
        assert np.array_equal(got[L][0], data[L][0])
        assert np.allclose(got[L][1], data[L][1], atol=1e-7)


def test_split_programs_keep_the_evolution_and_the_measurements():
    from spin_systems_b200.abi import Evolve, Repeat

    for seq in (0, 1):
        one, four = sg.program(seq), sg.program(seq, substeps=4)

        def evolves(prog):
            out = []
            for st in prog:
                if isinstance(st, Repeat):
                    out += [(e.tau, e.steps) for e in st.body if isinstance(e, Evolve)]
            return out
        a, b = evolves(one), evolves(four)
        assert len(a) == len(b)
        for (t1, n1), (t4, n4) in zip(a, b):
            assert n1 == 1 and n4 == 4 and abs(t1 - t4 * n4) < 1e-15
        spec = sg.sweep_spec(seq, 10, [(1.0, 0.5, 0.3, 1.0)], 4, substeps=4)
        assert spec.measurement_count() == sg.POINTS
