"""The oracle restatement (oracle/oracle.cpp) against golden fixtures produced by the
reference core itself (tests/golden/make_golden.py).  Everything is bit-exact: the
oracle follows the reference's FP64 statement order and calls the same libstdc++
sampling routines."""
import ctypes as C
import os

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return np.load(os.path.join(GOLD, name), allow_pickle=False)


def test_binner_matches_reference(oracle):
    d = load("binner.npz")
    X = np.ascontiguousarray(d["X"])
    n, nf = X.shape
    edges = np.zeros(nf * 256)
    ne = np.zeros(nf, np.int32)
    nbc = np.zeros(nf, np.int32)
    L = oracle.oracle_lib()
    mb = L.orc_binner_fit(X, n, nf, int(d["max_bin"]), int(d["bin_sample"]), int(d["seed"]), edges, ne, nbc)
    assert mb == int(d["max_bins"])
    assert np.array_equal(ne, d["n_edges"])
    assert np.array_equal(nbc, d["n_bins_col"])
    assert np.array_equal(edges.reshape(nf, 256), d["edges"])
    codes = np.zeros(n * nf, np.uint8)
    L.orc_bin_transform(X, n, nf, edges, ne, codes, nf)
    assert np.array_equal(codes.reshape(n, nf), d["codes"].astype(np.uint8))


def test_histogram_matches_reference(oracle):
    d = load("hist.npz")
    codes = np.ascontiguousarray(d["codes"].astype(np.uint8))
    n, nf = codes.shape
    nb = int(d["n_bins"])
    out = np.zeros(nf * nb * 3)
    oracle.oracle_lib().orc_build_hist(codes, nf, nf, d["idx"], d["idx"].size, d["g"], d["h"], nb, out)
    assert np.array_equal(out.reshape(nf, nb, 3), d["hist"])


def test_split_scan_matches_reference(oracle):
    d = load("hist.npz")
    s = load("split.npz")
    hist = np.ascontiguousarray(d["hist"].reshape(-1))
    nf = d["hist"].shape[0]

    class S(C.Structure):
        _fields_ = [("gain", C.c_double), ("feature", C.c_int), ("threshold_bin", C.c_int),
                    ("missing_go_left", C.c_int)]

    L = oracle.oracle_lib()
    L.orc_best_numeric.restype = S
    L.orc_best_numeric.argtypes = [np.ctypeslib.ndpointer(np.float64, flags="C"), C.c_int, C.c_int, C.c_double,
                                   C.c_double, C.c_int, C.c_double]
    for f in range(nf):
        r = L.orc_best_numeric(hist, int(d["n_bins"]), f, float(s["l2"]), float(s["gamma"]), int(s["min_leaf"]),
                               float(s["min_hess"]))
        assert r.threshold_bin == s["threshold"][f]
        assert r.missing_go_left == s["missing_left"][f]
        assert r.gain == s["gain"][f]


def test_pairwise_gradients_match_reference(oracle):
    d = load("pairwise.npz")
    m = d["y"].size
    g = np.zeros(m)
    h = np.zeros(m)
    grp = np.ascontiguousarray(d["groups"])
    L = oracle.oracle_lib()
    L.orc_grad_hess(5, d["y"], d["pred"], grp.ctypes.data_as(C.c_void_p), m, g, h)
    assert np.array_equal(g, d["g"]) and np.array_equal(h, d["h"])
    assert L.orc_loss(5, d["y"], d["pred"], grp.ctypes.data_as(C.c_void_p), m) == float(d["loss"])


@pytest.mark.parametrize("name", ["fit_mse", "fit_pair", "fit_pairsplit", "fit_cat"])
def test_fit_matches_reference(oracle, name):
    d = load(f"{name}.npz")
    params = eval(str(d["params"]))  # the fixture's own dict literal
    is_cat = d["is_cat"] if "is_cat" in d.files else None
    res, h = oracle.oracle_fit(params, d["X"].astype(np.float64), d["y"], d["ts"], d["entity"], is_cat=is_cat)
    try:
        assert len(res.trees) == int(d["n_trees"])
        assert res.n_bins == int(d["n_bins"]) and res.n_buckets == int(d["n_buckets"])
        assert res.init_score == float(d["init_score"])
        assert np.array_equal(res.init_prefix, d["init_prefix"])
        assert np.array_equal(res.evals_train, d["evals"])
        for t, tr in enumerate(res.trees):
            for fld in ("is_leaf", "feature", "threshold", "left", "right", "missing_left", "n_samples", "depth",
                        "value", "gain", "values", "cover", "prefix", "split_type", "feature2"):
                assert np.array_equal(getattr(tr, fld), d[f"t{t}_{fld}"]), (t, fld)
            if is_cat is not None:
                assert np.array_equal(tr.cat_left, d[f"t{t}_cat_left"]), (t, "cat_left")
        pr = oracle.oracle_predict(h, d["X"][:500].astype(np.float64))
        assert np.array_equal(pr, d["pred"])
    finally:
        oracle.oracle_free(h)


def test_pair_fixture_has_pair_splits():
    """The PAIR fixture exercises the pair search: its trees hold pair nodes."""
    d = load("fit_pairsplit.npz")
    assert sum(int((d[f"t{t}_split_type"] == 1).sum()) for t in range(int(d["n_trees"]))) > 0


@pytest.mark.parametrize("extra", [dict(objective="mse"), dict(objective="mse", goss=1, goss_top=0.3, goss_other=0.2),
                                   dict(objective="mse", iid_mode=1),
                                   dict(objective="mse", pair_top_k=3, max_pair_splits_per_tree=5, pair_trigger=1.0,
                                        pair_l2=0.5),
                                   dict(objective="pairwise")])
def test_pair_splits_match_reference(oracle, extra):
    """PAIR splits (cpp/src/tree.cpp:214-281) in the oracle against the reference core built
    from source, on an interaction target where the axis splits are weak."""
    if not oracle.ref_available():
        pytest.skip("reference core not built (oracle/_ref)")
    rng = np.random.default_rng(7)
    n, nf = 8000, 9
    X = rng.standard_normal((n, nf))
    X[rng.random((n, nf)) < 0.05] = np.nan
    y = np.sign(np.nan_to_num(X[:, 2]) * np.nan_to_num(X[:, 5])) + 0.5 * rng.standard_normal(n)
    ts = np.repeat(np.arange(80), 100).astype(np.int64)
    params = dict(n_estimators=4, learning_rate=0.1, max_depth=6, max_leaves=20, horizon=1, random_state=1,
                  pair_splits=1, **extra)
    ts_arg = None if params.get("iid_mode") else ts
    r, hr = oracle.ref_fit(params, X, y, ts_arg)
    o, ho = oracle.oracle_fit(params, X, y, ts_arg)
    try:
        assert len(r.trees) == len(o.trees)
        assert sum(int((t.split_type == 1).sum()) for t in r.trees) > 0
        for t, (a, b) in enumerate(zip(r.trees, o.trees)):
            for fld in ("is_leaf", "feature", "threshold", "left", "right", "missing_left", "n_samples", "depth",
                        "value", "gain", "values", "cover", "prefix", "split_type", "feature2"):
                assert np.array_equal(getattr(a, fld), getattr(b, fld)), (t, fld)
        assert np.array_equal(r.evals_train, o.evals_train)
        assert np.array_equal(oracle.ref_predict(hr, X[:400]), oracle.oracle_predict(ho, X[:400]))
    finally:
        oracle.ref_free(hr)
        oracle.oracle_free(ho)


def test_cat_fixture_has_categorical_splits():
    d = load("fit_cat.npz")
    assert sum(int((d[f"t{t}_split_type"] == 2).sum()) for t in range(int(d["n_trees"]))) > 0


def _cat_panel(seed, interaction):
    rng = np.random.default_rng(seed)
    n, nf = 9000, 7
    X = rng.standard_normal((n, nf))
    X[:, 0] = rng.integers(0, 12, n)
    X[:, 3] = rng.integers(0, 400, n)
    X[:, 5] = np.where(rng.random(n) < 0.02, rng.integers(100, 130, n), rng.integers(0, 6, n))
    X[rng.random((n, nf)) < 0.03] = np.nan
    if interaction:  # weak single features: PAIR candidates compete with categorical gains
        y = np.sign(np.nan_to_num(X[:, 1]) * np.nan_to_num(X[:, 2])) + 0.4 * rng.standard_normal(n)
    else:
        eff = np.array([0.9, -0.4, 0.1, 1.2, -1.0, 0.0, 0.5, 0.3, -0.7, 0.2, 0.0, -0.2])
        y = eff[np.nan_to_num(X[:, 0], nan=0).astype(int) % 12] + 0.3 * np.nan_to_num(X[:, 1]) + \
            0.5 * rng.standard_normal(n)
    ts = np.repeat(np.arange(90), 100).astype(np.int64)
    return X, y, ts, np.array([1, 0, 0, 1, 0, 1, 0], np.int32)


@pytest.mark.parametrize("extra,interaction", [(dict(objective="mse"), False),
                                               (dict(objective="mse", cat_min_count=50, cat_smooth=5.0), False),
                                               (dict(objective="mse", goss=1, goss_top=0.3, goss_other=0.2), False),
                                               (dict(objective="pairwise"), False),
                                               (dict(objective="mse", iid_mode=1), False),
                                               (dict(objective="mse", pair_splits=1), True)])
def test_categorical_splits_match_reference(oracle, extra, interaction):
    """Categorical features in the oracle (vocabulary binning, binning.cpp:47-84;
    best_categorical, histogram.cpp:195-244; cat_goes_left, tree.hpp:27-30) against the
    reference core built from source: trees with their left masks, losses, predictions."""
    if not oracle.ref_available():
        pytest.skip("reference core not built (oracle/_ref)")
    X, y, ts, is_cat = _cat_panel(3, interaction)
    params = dict(n_estimators=4, learning_rate=0.1, max_depth=6, max_leaves=20, horizon=1, random_state=2, **extra)
    ts_arg = None if params.get("iid_mode") else ts
    r, hr = oracle.ref_fit(params, X, y, ts_arg, is_cat=is_cat)
    o, ho = oracle.oracle_fit(params, X, y, ts_arg, is_cat=is_cat)
    try:
        assert len(r.trees) == len(o.trees) and r.n_bins == o.n_bins
        kinds = {int(k) for t in r.trees for k in t.split_type[t.is_leaf == 0]}
        assert 2 in kinds and (not interaction or 1 in kinds), kinds
        for t, (a, b) in enumerate(zip(r.trees, o.trees)):
            for fld in ("is_leaf", "feature", "threshold", "left", "right", "missing_left", "n_samples", "depth",
                        "value", "gain", "values", "cover", "prefix", "split_type", "feature2", "cat_left"):
                assert np.array_equal(getattr(a, fld), getattr(b, fld)), (t, fld)
        assert np.array_equal(r.evals_train, o.evals_train)
        assert np.array_equal(oracle.ref_predict(hr, X[:500]), oracle.oracle_predict(ho, X[:500]))
    finally:
        oracle.ref_free(hr)
        oracle.oracle_free(ho)


@pytest.mark.parametrize("max_bin,min_count", [(255, 5), (64, 2), (255, 30)])
def test_categorical_binner_matches_reference(oracle, max_bin, min_count):
    """The oracle's Binner::fit + transform with categorical features against the reference
    core: vocabularies, numeric edges, max_bins and the codes."""
    if not oracle.ref_available():
        pytest.skip("reference core not built (oracle/_ref)")
    import ctypes as C
    rng = np.random.default_rng(9)
    n, nf = 15000, 5
    X = rng.standard_normal((n, nf))
    X[:, 0] = rng.integers(0, 12, n)
    X[:, 1] = rng.integers(0, 400, n)
    X[:, 3] = np.where(rng.random(n) < 0.01, rng.integers(100, 160, n), rng.integers(0, 5, n))
    X[:, 4] = rng.integers(0, 3000, n)
    X[rng.random((n, nf)) < 0.03] = np.nan
    is_cat = np.array([1, 1, 0, 1, 1], np.int32)
    R = oracle.ref_lib()
    R.ref_binner_cat.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_uint,
                                 C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    e1 = np.zeros(nf * 256)
    n1 = np.zeros(nf, np.int32)
    mb = np.zeros(1, np.int32)
    codes = np.zeros((n, nf), np.uint16)
    assert R.ref_binner_cat(X.ctypes.data_as(C.c_void_p), n, nf, is_cat.ctypes.data_as(C.c_void_p), max_bin,
                            min_count, 2000, 5, e1.ctypes.data_as(C.c_void_p), n1.ctypes.data_as(C.c_void_p),
                            mb.ctypes.data_as(C.c_void_p), codes.ctypes.data_as(C.c_void_p)) == 0
    L = oracle.oracle_lib()
    L.orc_binner_fit_cat.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_uint32,
                                     C.c_void_p, C.c_void_p, C.c_void_p]
    e2 = np.zeros(nf * 256)
    n2 = np.zeros(nf, np.int32)
    c2 = np.zeros((n, nf), np.uint8)
    nb = L.orc_binner_fit_cat(X.ctypes.data_as(C.c_void_p), n, nf, is_cat.ctypes.data_as(C.c_void_p), max_bin,
                              min_count, 2000, 5, e2.ctypes.data_as(C.c_void_p), n2.ctypes.data_as(C.c_void_p),
                              c2.ctypes.data_as(C.c_void_p))
    assert nb == int(mb[0])
    assert np.array_equal(n1, n2) and np.array_equal(e1, e2)
    assert np.array_equal(codes.astype(np.uint8), c2) and codes.max() <= 255


@pytest.mark.parametrize("max_bin,bin_sample", [(255, 0), (255, 500), (64, 0), (8, 500)])
def test_binner_edge_columns_match_reference(oracle, max_bin, bin_sample):
    """Binner::fit + transform on edge columns (tests/edge_columns.py): the oracle's edges
    bit for bit (NaN edges from infinite ranges included), n_bins_col, max_bins and codes
    against the reference core."""
    from edge_columns import edge_columns

    if not oracle.ref_available():
        pytest.skip("reference core not built (oracle/_ref)")
    X = edge_columns()
    n, nf = X.shape
    e1 = np.zeros(nf * 256)
    n1 = np.zeros(nf, np.int32)
    b1 = np.zeros(nf, np.int32)
    L = oracle.oracle_lib()
    mb1 = L.orc_binner_fit(X, n, nf, max_bin, bin_sample, 7, e1, n1, b1)
    c1 = np.zeros(n * nf, np.uint8)
    L.orc_bin_transform(X, n, nf, e1, n1, c1, nf)
    e2 = np.zeros(nf * 256)
    n2 = np.zeros(nf, np.int32)
    b2 = np.zeros(nf, np.int32)
    mb2 = C.c_int()
    c2 = np.zeros((n, nf), np.uint16)
    assert oracle.ref_lib().ref_binner(X, n, nf, max_bin, bin_sample, 7, e2, n2, b2, C.byref(mb2),
                                       c2.ctypes.data_as(C.c_void_p)) == 0
    assert mb1 == mb2.value
    assert np.array_equal(n1, n2) and np.array_equal(b1, b2)
    assert np.array_equal(e1.view(np.uint64), e2.view(np.uint64))
    assert np.array_equal(c1.reshape(n, nf), c2)


_OPTION_CASES = {
    "embargo3": dict(horizon=1, embargo=3),
    "horizon5_embargo2": dict(horizon=5, embargo=2),
    "buckets7": dict(horizon=1, n_time_buckets=7),
    "finer": dict(horizon=1, finer_torb=1),
    "finer_buckets100": dict(horizon=1, finer_torb=1, n_time_buckets=100),
    "min_cover500": dict(horizon=1, torb_min_cover=500.0),
    "stump": dict(horizon=1, max_leaves=2),
    "depth1": dict(horizon=1, max_depth=1),
    "min_split_gain5": dict(horizon=1, min_split_gain=5.0),
    "min_child_weight50": dict(horizon=1, min_child_weight=50.0),
    "pairwise_goss_h2": dict(horizon=2, objective="pairwise", goss=1, goss_top=0.3, goss_other=0.3),
}


@pytest.mark.parametrize("name", sorted(_OPTION_CASES))
def test_fit_options_match_reference(oracle, name):
    """The oracle's fit against the reference core under the TORB and growth options:
    causal cuts with embargo and horizon (booster.cpp:60-72), bucket counts, the cover
    blend (booster.cpp:604-648) and the growth limits; trees, values, prefixes, losses
    and predictions bit for bit."""
    if not oracle.ref_available():
        pytest.skip("reference core not built (oracle/_ref)")
    from tidegbm_b200 import panels

    p = panels.panel_small(n_dates=70, n_entities=90, n_features=8, seed=4)
    params = {**dict(n_estimators=5, learning_rate=0.1, max_depth=5, objective="mse", random_state=2,
                     pair_splits=False), **_OPTION_CASES[name]}
    X = p.X.astype(np.float64)
    r, hr = oracle.ref_fit(params, X, p.y, p.ts, p.entity, n_jobs=1)
    o, ho = oracle.oracle_fit(params, X, p.y, p.ts, p.entity)
    try:
        assert len(r.trees) == len(o.trees) and r.n_buckets == o.n_buckets
        for t, (a, b) in enumerate(zip(r.trees, o.trees)):
            for fld in ("is_leaf", "feature", "threshold", "left", "right", "missing_left", "n_samples", "depth",
                        "value", "gain", "values", "cover", "prefix"):
                assert np.array_equal(getattr(a, fld), getattr(b, fld)), (t, fld)
        assert np.array_equal(r.evals_train, o.evals_train)
        assert np.array_equal(oracle.ref_predict(hr, X[:500]), oracle.oracle_predict(ho, X[:500]))
    finally:
        oracle.ref_free(hr)
        oracle.oracle_free(ho)


@pytest.mark.parametrize("k", range(8))
def test_small_shapes_match_reference(oracle, k):
    """The oracle's fit against the reference core on small and ragged shapes
    (tests/fit_shapes.py): trees, values, prefixes and predictions bit for bit."""
    from fit_shapes import SHAPES, shape_case

    if not oracle.ref_available():
        pytest.skip("reference core not built (oracle/_ref)")
    X, y, ts, ent, params = shape_case(*SHAPES[k])
    r, hr = oracle.ref_fit(params, X, y, ts, ent, n_jobs=1)
    o, ho = oracle.oracle_fit(params, X, y, ts, ent)
    try:
        assert len(r.trees) == len(o.trees)
        for t, (a, b) in enumerate(zip(r.trees, o.trees)):
            for fld in ("is_leaf", "feature", "threshold", "left", "right", "missing_left", "n_samples", "value",
                        "values", "cover", "prefix"):
                assert np.array_equal(getattr(a, fld), getattr(b, fld)), (t, fld)
        assert np.array_equal(oracle.ref_predict(hr, X), oracle.oracle_predict(ho, X))
    finally:
        oracle.ref_free(hr)
        oracle.oracle_free(ho)


def _pairwise_groups(seed):
    """Dates of 1, 2, 24, 48, 49, 50, 97 and 800 rows (48 is the last size with every pair,
    objective.cpp:179-219), ties in y (pairs of equal labels are skipped), one date whose
    labels are all equal, and predictions far enough apart to reach the exp clamp."""
    rng = np.random.default_rng(seed)
    sizes = [1, 2, 24, 48, 49, 50, 97, 800, 30]
    groups = np.concatenate([np.full(m, k, np.int64) for k, m in enumerate(sizes)])
    n = groups.size
    y = np.round(rng.standard_normal(n), 1)
    y[groups == 8] = 0.5
    pred = rng.standard_normal(n) * np.where(rng.random(n) < 0.05, 40.0, 1.0)
    return np.ascontiguousarray(y), np.ascontiguousarray(pred), np.ascontiguousarray(groups)


@pytest.mark.parametrize("seed", [0, 1])
def test_pairwise_gradient_edges_match_reference(oracle, seed):
    """RankPairwise grad_hess and loss at the edges of its pair sampling, oracle against
    the reference core bit for bit."""
    if not oracle.ref_available():
        pytest.skip("reference core not built (oracle/_ref)")
    y, pred, groups = _pairwise_groups(seed)
    n = y.size
    g1, h1, g2, h2 = np.zeros(n), np.zeros(n), np.zeros(n), np.zeros(n)
    gp = groups.ctypes.data_as(C.c_void_p)
    oracle.oracle_lib().orc_grad_hess(5, y, pred, gp, n, g1, h1)
    oracle.ref_lib().ref_grad_hess(5, y, pred, gp, n, g2, h2)
    assert np.array_equal(g1, g2) and np.array_equal(h1, h2)
    R = oracle.ref_lib()
    R.ref_loss.restype = C.c_double
    R.ref_loss.argtypes = [C.c_int, np.ctypeslib.ndpointer(np.float64, flags="C"),
                           np.ctypeslib.ndpointer(np.float64, flags="C"), C.c_void_p, C.c_int]
    L = oracle.oracle_lib()
    assert L.orc_loss(5, y, pred, gp, n) == R.ref_loss(5, y, pred, gp, n)
