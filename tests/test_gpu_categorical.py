"""Categorical features on the device (batched growth): vocabulary codes, the ranked-prefix
split search of best_categorical (cpp/src/histogram.cpp:195-244), routing by the 256-bit
left mask in the partition, the post-tree sweep and predict.

Against the reference's own fit (tests/golden/fit_cat.npz, no PAIR split fired there) and
the oracle restatement: identical structure, split types and left masks; values within
1e-9.  The tie panel gives several categories exactly equal gradient sums, so the ranking's
ties are ordered by std::sort's own algorithm, which the scan replays.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _compare_trees(trees_g, trees_r, atol=1e-9):
    assert len(trees_g) == len(trees_r)
    for t, (a, b) in enumerate(zip(trees_g, trees_r)):
        for fld in ("is_leaf", "feature", "threshold", "left", "right", "missing_left", "n_samples", "depth"):
            assert np.array_equal(getattr(a, fld), getattr(b, fld)), (t, fld)
        assert np.array_equal(a.split_type, b.split_type), (t, "split_type")
        assert np.array_equal(a.cat_left, b.cat_left), (t, "cat_left")
        np.testing.assert_allclose(a.value, b.value, rtol=0, atol=atol)
        np.testing.assert_allclose(a.values, b.values, rtol=0, atol=atol)
        np.testing.assert_allclose(a.prefix, b.prefix, rtol=0, atol=atol)


def test_categorical_fit_matches_reference_fixture(native):
    d = np.load(os.path.join(GOLDEN, "fit_cat.npz"), allow_pickle=True)
    params = dict(eval(str(d["params"])), pair_splits=False)  # no PAIR split fired in the fixture
    b = native.Booster(**params)
    b.fit(d["X"], d["y"], timestamps=d["ts"], entity=d["entity"], is_cat=d["is_cat"])
    trees = b.trees()
    assert len(trees) == int(d["n_trees"])
    assert b.info()["n_bins"] == int(d["n_bins"])
    n_cat = 0
    for t, tr in enumerate(trees):
        for fld in ("is_leaf", "feature", "threshold", "left", "right", "missing_left", "n_samples", "depth"):
            assert np.array_equal(getattr(tr, fld), d[f"t{t}_{fld}"]), (t, fld)
        assert np.array_equal(tr.split_type, d[f"t{t}_split_type"]), t
        assert np.array_equal(tr.cat_left, d[f"t{t}_cat_left"]), t
        np.testing.assert_allclose(tr.values, d[f"t{t}_values"], rtol=0, atol=1e-9)
        np.testing.assert_allclose(tr.prefix, d[f"t{t}_prefix"], rtol=0, atol=1e-9)
        n_cat += int((tr.split_type == 2).sum())
    assert n_cat > 0
    np.testing.assert_allclose(b.raw_predict(d["X"][:500]), d["pred"], rtol=0, atol=1e-9)


def _cat_panel(seed, ties=False):
    rng = np.random.default_rng(seed)
    n, nf = 9000, 7
    X = rng.standard_normal((n, nf))
    X[:, 0] = rng.integers(0, 12, n)
    X[:, 3] = rng.integers(0, 400, n)
    X[:, 5] = np.where(rng.random(n) < 0.02, rng.integers(100, 130, n), rng.integers(0, 6, n))
    X[rng.random((n, nf)) < 0.03] = np.nan
    eff = np.array([0.9, -0.4, 0.1, 1.2, -1.0, 0.0, 0.5, 0.3, -0.7, 0.2, 0.0, -0.2])
    y = eff[np.nan_to_num(X[:, 0], nan=0).astype(int) % 12] + 0.3 * np.nan_to_num(X[:, 1]) + \
        0.5 * rng.standard_normal(n)
    if ties:
        # 24 categories in pairs of identical size and identical targets: their gradient
        # sums tie exactly at every tree's root
        cat = np.repeat(np.arange(24), n // 24)
        rng.shuffle(cat)
        X[:, 0] = cat
        y = np.array([0.5 * (k // 2 % 5) - 1.0 for k in range(24)])[cat]
    ts = np.repeat(np.arange(90), 100).astype(np.int64)
    return X, y, ts, np.array([1, 0, 0, 1, 0, 1, 0], np.int32)


@pytest.mark.parametrize("extra,ties", [(dict(objective="mse"), False),
                                        (dict(objective="mse", cat_min_count=50, cat_smooth=5.0), False),
                                        (dict(objective="mse", goss=1, goss_top=0.3, goss_other=0.2), False),
                                        (dict(objective="pairwise"), False),
                                        (dict(objective="mse", iid_mode=1), False),
                                        (dict(objective="mse"), True)])
def test_categorical_matches_oracle(native, oracle, extra, ties):
    X, y, ts, is_cat = _cat_panel(5, ties)
    params = dict(n_estimators=6, learning_rate=0.1, max_depth=6, max_leaves=20, horizon=1, random_state=1,
                  pair_splits=False, **extra)
    iid = extra.get("iid_mode")
    b = native.Booster(**params)
    b.fit(X, y, timestamps=None if iid else ts, is_cat=is_cat)
    ref, h = oracle.oracle_fit(params, X, y, None if iid else ts, None, is_cat=is_cat)
    try:
        _compare_trees(b.trees(), ref.trees)
        assert any((t.split_type == 2).any() for t in b.trees())
        np.testing.assert_allclose(b.raw_predict(X[:2000]), oracle.oracle_predict(h, X[:2000]), rtol=0, atol=1e-9)
    finally:
        oracle.oracle_free(h)
