"""PAIR splits on the device (cpp/src/tree.cpp:214-281): a leaf whose best axis gain is weak
against its gradient energy also tries the pairs of its top pair_top_k features through
the histogram of the hashed code pair (pair_bin, histogram.hpp:81-85); at most
max_pair_splits_per_tree pair splits per tree, after which every leaf falls back to its
axis split.  The reference turns PAIR on by default below 1M rows, so this is the path a
default TideRegressor takes on device="gpu".

Against the reference's own fit (tests/golden/fit_pairsplit.npz) and the oracle
restatement: identical structure, split types and second features; values within 1e-9.
"""
import os
from types import SimpleNamespace

import numpy as np
import pytest
from missing_bins import empty_missing_nodes

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _compare(trees_g, trees_r, codes=None, n_bins=None, atol=1e-9):
    """Structure, split types and values; missing directions everywhere except at split
    nodes whose missing bin holds no row of the fit (missing_bins.py says why)."""
    assert len(trees_g) == len(trees_r)
    for t, (a, b) in enumerate(zip(trees_g, trees_r)):
        for fld in ("is_leaf", "feature", "threshold", "left", "right", "n_samples", "depth", "split_type",
                    "feature2"):
            assert np.array_equal(getattr(a, fld), getattr(b, fld)), (t, fld)
        _compare_missing(t, a, b, codes, n_bins)
        np.testing.assert_allclose(a.value, b.value, rtol=0, atol=atol)
        np.testing.assert_allclose(a.values, b.values, rtol=0, atol=atol)
        np.testing.assert_allclose(a.prefix, b.prefix, rtol=0, atol=atol)


def _compare_missing(t, a, b, codes, n_bins):
    differ = set(np.flatnonzero(np.asarray(a.missing_left) != np.asarray(b.missing_left)).tolist())
    if not differ:
        return
    assert codes is not None, (t, "missing_left", sorted(differ))
    empty = empty_missing_nodes(b, codes, n_bins)
    assert differ <= empty, (t, "missing_left", sorted(differ - empty))


def test_pair_fit_matches_reference_fixture(native, oracle):
    d = np.load(os.path.join(GOLDEN, "fit_pairsplit.npz"), allow_pickle=True)
    params = eval(str(d["params"]))
    b = native.Booster(**params)
    b.fit(d["X"], d["y"], timestamps=d["ts"], entity=d["entity"])
    trees = b.trees()
    assert len(trees) == int(d["n_trees"])
    codes, nb = oracle.oracle_codes(d["X"], params)
    n_pair = 0
    for t, tr in enumerate(trees):
        for fld in ("is_leaf", "feature", "threshold", "left", "right", "n_samples", "depth", "split_type",
                    "feature2"):
            assert np.array_equal(getattr(tr, fld), d[f"t{t}_{fld}"]), (t, fld)
        ref_tree = SimpleNamespace(**{fld: d[f"t{t}_{fld}"] for fld in (
            "is_leaf", "feature", "threshold", "left", "right", "missing_left", "split_type", "feature2")})
        _compare_missing(t, tr, ref_tree, codes, nb)
        np.testing.assert_allclose(tr.values, d[f"t{t}_values"], rtol=0, atol=1e-9)
        np.testing.assert_allclose(tr.prefix, d[f"t{t}_prefix"], rtol=0, atol=1e-9)
        n_pair += int((tr.split_type == 1).sum())
    assert n_pair > 0
    np.testing.assert_allclose(b.raw_predict(d["X"][:500]), d["pred"], rtol=0, atol=1e-9)


def _interaction_panel():
    rng = np.random.default_rng(7)
    n, nf = 8000, 9
    X = rng.standard_normal((n, nf))
    X[rng.random((n, nf)) < 0.05] = np.nan
    y = np.sign(np.nan_to_num(X[:, 2]) * np.nan_to_num(X[:, 5])) + 0.5 * rng.standard_normal(n)
    ts = np.repeat(np.arange(80), 100).astype(np.int64)
    return X, y, ts


@pytest.mark.parametrize("extra", [dict(objective="mse"), dict(objective="mse", goss=1, goss_top=0.3, goss_other=0.2),
                                   dict(objective="mse", iid_mode=1),
                                   dict(objective="mse", pair_top_k=3, max_pair_splits_per_tree=5, pair_trigger=1.0,
                                        pair_l2=0.5),
                                   dict(objective="pairwise")])
def test_pair_splits_match_oracle(native, oracle, extra):
    X, y, ts = _interaction_panel()
    params = dict(n_estimators=4, learning_rate=0.1, max_depth=6, max_leaves=20, horizon=1, random_state=1,
                  pair_splits=1, **extra)
    ts_arg = None if params.get("iid_mode") else ts
    b = native.Booster(**params)
    b.fit(X, y, timestamps=ts_arg)
    ref, h = oracle.oracle_fit(params, X, y, ts_arg)
    codes, nb = oracle.oracle_codes(X, params)
    try:
        _compare(b.trees(), ref.trees, codes, nb)
        assert sum(int((t.split_type == 1).sum()) for t in b.trees()) > 0
        np.testing.assert_allclose(b.evals_result()["train"], ref.evals_train, rtol=1e-9, atol=1e-9)
        np.testing.assert_allclose(b.raw_predict(X[:1000]), oracle.oracle_predict(h, X[:1000]), rtol=0, atol=1e-9)
    finally:
        oracle.oracle_free(h)


def test_pair_and_categorical_together(native, oracle):
    from test_gpu_categorical import _cat_panel

    rng = np.random.default_rng(3)
    X, y, ts, is_cat = _cat_panel(3)
    y = np.sign(np.nan_to_num(X[:, 1]) * np.nan_to_num(X[:, 2])) + 0.4 * rng.standard_normal(X.shape[0])
    params = dict(n_estimators=4, learning_rate=0.1, max_depth=6, max_leaves=20, horizon=1, random_state=2,
                  objective="mse", pair_splits=1)
    b = native.Booster(**params)
    b.fit(X, y, timestamps=ts, is_cat=is_cat)
    ref, h = oracle.oracle_fit(params, X, y, ts, is_cat=is_cat)
    codes, nb = oracle.oracle_codes(X, params, is_cat)
    try:
        _compare(b.trees(), ref.trees, codes, nb)
        for a, r in zip(b.trees(), ref.trees):
            assert np.array_equal(a.cat_left, r.cat_left)
    finally:
        oracle.oracle_free(h)


def test_default_config_runs_pair_search(native):
    """The reference's defaults (pair_splits on below 1M rows) on device="gpu"."""
    X, y, ts = _interaction_panel()
    b = native.Booster(n_estimators=3, horizon=1)
    b.fit(X, y, timestamps=ts)
    assert sum(int((t.split_type == 1).sum()) for t in b.trees()) > 0
