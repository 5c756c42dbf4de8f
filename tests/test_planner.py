"""Learned planner, host side: the CPU oracle's gradient against finite
differences, the feature map, and the model file / install checks."""
import numpy as np
import pytest

import algofft
import mlp as O  # oracle/mlp.py
from algofft import planner as P


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = O.init(1).astype(np.float64) + 0.01 * rng.standard_normal(O.NP)
    X = rng.standard_normal((9, O.D))
    y = rng.standard_normal(9)
    _, g = O.loss_and_grad(p, X, y)
    idx = rng.choice(O.NP, 60, replace=False)
    eps = 1e-6
    for i in idx:
        e = np.zeros(O.NP)
        e[i] = eps
        num = (O.loss_and_grad(p + e, X, y)[0] - O.loss_and_grad(p - e, X, y)[0]) / (2 * eps)
        assert abs(num - g[i]) <= 1e-6 + 1e-5 * abs(g[i]), (i, num, g[i])


def test_sizes_and_feature_map():
    assert P.sizes() == (O.D, O.H, O.NP)
    f = P.features(0, 1000, 0, 1, 0, "gpu-sm100-mixed2-25x40")
    assert f[0] == pytest.approx(np.log2(1000)) and list(f[1:5]) == [3, 0, 3, 0]
    assert f[5] == pytest.approx(np.log2(5))
    assert f[6] == pytest.approx(np.log2((1 << 27) // 8000))  # unknown batch: 128 MB of data
    assert list(f[10:14]) == [0, 0, 1, 0] and f[14] == 1 and f[15] == pytest.approx(np.log2(25))
    f = P.features(1, 4096, 64, 8, 1, "gpu-sm100-tp-64x64-t8192-e16")
    assert list(f[6:10]) == [6, 1, 3, 1] and list(f[10:14]) == [0, 1, 0, 0] and list(f[14:]) == [4, 13]
    f = P.features(0, 1009, 4, 1, 0, "gpu-sm100-bluestein-n1009")
    assert f[5] == pytest.approx(np.log2(1009)) and f[13] == 1 and f[15] == 11
    # compiled mixed-radix families: markers 2 (single pass) and 3 (four-step)
    f = P.features(0, 1000, 4, 1, 0, "gpu-sm100-mixr-n1000")
    assert list(f[10:14]) == [0, 0, 1, 0] and f[14] == 2 and f[15] == 0
    f = P.features(0, 50421, 4, 1, 0, "gpu-sm100-mixc-147x343")
    assert list(f[10:14]) == [0, 0, 1, 0] and f[14] == 3 and f[15] == pytest.approx(np.log2(147))
    # Bluestein on the mixed length (marker 1) against the power of two
    f = P.features(0, 16411, 4, 1, 0, "gpu-sm100-bluestein-n16411-mx")
    assert f[13] == 1 and f[14] == 1 and f[15] == pytest.approx(np.log2(34560))
    f = P.features(0, 16411, 4, 1, 0, "gpu-sm100-bluestein-n16411-p2")
    assert f[13] == 1 and f[14] == 0 and f[15] == 16
    with pytest.raises(algofft.ErrInvalidArgument):
        P.features(0, 64, 1, 1, 0, "no-such-variant")


def test_model_file_round_trip_and_install_checks(tmp_path):
    p = P.init_params(3)
    norm = np.concatenate([np.zeros(O.D), np.ones(O.D), [0.0, 1.0]]).astype(np.float32)
    m = P.Model(p, norm)
    m.save(str(tmp_path / "m.bin"))
    m2 = P.Model.load(str(tmp_path / "m.bin"))
    assert np.array_equal(m2.params, p) and np.array_equal(m2.norm, norm)
    bad = norm.copy()
    bad[O.D] = 0.0
    with pytest.raises(algofft.ErrInvalidArgument):
        P.Model(p, bad).install()
    with pytest.raises(algofft.ErrInvalidArgument):
        algofft.check(algofft.lib().gfft_planner_load_model(str(tmp_path / "missing.bin").encode()))


def test_shapes_are_seeded_and_have_choices():
    a = P.shapes(40, seed=5)
    assert a == P.shapes(40, seed=5)
    for s in a:
        assert len(algofft.Variants(s["n"], s["prec"])) >= 2
        assert s["batch"] >= 1


def test_shipped_model_beats_size_class_rules_on_held_out_shapes():
    # The shipped model against the shipped B200 measurements: on the 500
    # held-out shapes its picks cost less (regret = chosen / fastest) than
    # the size-class rules' picks.  Forward pass: the CPU oracle.
    recs = P.load_records()
    assert len(recs) == P.TRAIN_SHAPES + P.HELD_OUT_SHAPES
    _, held = P.split(recs)
    m = P.Model.load(P.DEFAULT_MODEL)
    ch = P.learned_choices(m, held, predict=lambda X: O.forward(m.params, m.standardize(X)))
    learned = P.regret_stats(held, lambda i, r: ch[i])
    rules = P.regret_stats(held, lambda i, r: r["default"])
    assert learned["missing"] == 0 and rules["missing"] == 0
    assert learned["mean"] < rules["mean"] and learned["p90"] < rules["p90"]
    assert learned["mean"] < 1.05 and learned["optimal"] > 0.6
