"""A model handed over as the exported arrays (the fields tgb_tree_export, tgb_edges and
tgb_model_info return) rebuilds a reference Booster that predicts exactly as the one it
came from, and survives the reference's .tgbm blob (Booster::save_binary / load_binary,
cpp/src/serialize.cpp:65-255).  Here the source model is the reference's own fit (CPU);
tests/test_gpu_fit.py runs the same hand-over with GPU-grown trees."""
import numpy as np
import pytest


def _ref_or_skip(oracle):
    if not oracle.ref_available():
        pytest.skip("reference core not built (oracle/_ref)")


@pytest.mark.parametrize("iid", [False, True])
def test_exported_arrays_rebuild_reference_model(oracle, iid):
    _ref_or_skip(oracle)
    from tidegbm_b200 import panels

    p = panels.panel_small(n_dates=80, n_entities=120, n_features=10)
    params = dict(n_estimators=6, learning_rate=0.1, max_depth=5, horizon=1, objective="mse", goss=0, random_state=2)
    if iid:
        params["iid_mode"] = 1
    X = p.X.astype(np.float64)
    res, h = oracle.ref_fit(params, X, p.y, None if iid else p.ts, None if iid else p.entity, n_jobs=1)
    try:
        E, ne = oracle.ref_edges_of(h, X.shape[1])
        h2 = oracle.ref_import(X.shape[1], res.n_bins, res.n_buckets, res.init_score, res.init_prefix, E, ne, 255,
                               0.1, "mse", iid, res.trees)
        try:
            want = oracle.ref_predict(h, X)
            np.testing.assert_array_equal(oracle.ref_predict(h2, X), want)
            blob = oracle.ref_save(h2)
            assert blob[:4] == oracle.ref_save(h)[:4]
            h3 = oracle.ref_load(blob)
            try:
                np.testing.assert_array_equal(oracle.ref_predict(h3, X), want)
            finally:
                oracle.ref_free(h3)
        finally:
            oracle.ref_free(h2)
    finally:
        oracle.ref_free(h)
