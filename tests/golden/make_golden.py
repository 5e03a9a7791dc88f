"""Generates the golden fixtures in this folder from the reference TideGBM core,
compiled from its own sources into oracle/_ref/libtgbref.so (make -C oracle ref).

    python tests/golden/make_golden.py

Each fixture is the reference's output on a small seeded input:
  binner.npz    Binner::fit + transform (cpp/src/binning.cpp:34-128): edges, u16 codes
  hist.npz      build_hist_col (cpp/src/histogram.cpp:44-76)
  split.npz     best_numeric_missing per feature (cpp/src/histogram.cpp:144-193)
  pairwise.npz  Objective::grad_hess RankPairwise (cpp/src/objective.cpp:179-219) and loss
  fit_mse.npz   Booster::fit (cpp/src/booster.cpp:231-742): trees, values, TORB prefixes,
                evals, predictions (time mode, mse, GOSS on)
  fit_pair.npz  the same for the pairwise objective
  fit_pairsplit.npz  mse with PAIR splits on (cpp/src/tree.cpp:214-281) over an interaction
                target, where the axis splits are weak; trees carry split_type and feature2
  fit_cat.npz   mse with categorical features (vocabulary binning, binning.cpp:47-84;
                best_categorical, histogram.cpp:195-244): trees carry the left masks
The tests check the oracle restatement (CPU) and the CUDA path (GPU) against them.
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import bind  # noqa: E402
from tidegbm_b200 import panels  # noqa: E402

FIT_MSE = dict(n_estimators=8, learning_rate=0.1, max_depth=5, max_leaves=15, horizon=2, objective="mse", goss=1,
               random_state=4, bin_sample=3000)
FIT_PAIRSPLIT = dict(n_estimators=5, learning_rate=0.1, max_depth=5, max_leaves=15, horizon=1, objective="mse",
                     random_state=3, pair_splits=1)
FIT_PAIR = dict(n_estimators=6, learning_rate=0.08, max_depth=4, max_leaves=12, horizon=1, objective="pairwise",
                random_state=2)


def _X(seed, n, nf, nan=0.03):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((n, nf))
    X[:, 1] = np.round(X[:, 1] * 2)
    X[:, 2] = np.exp(X[:, 2])
    X[rng.random((n, nf)) < nan] = np.nan
    return X


class _Panel:
    def __init__(self, X, y, ts, entity):
        self.X, self.y, self.ts, self.entity = X, y, ts, entity


def interaction_panel(seed=5, n_dates=50, n_entities=100, nf=8):
    """y = sign(x0 * x1) + noise: no single feature separates it, so PAIR splits trigger."""
    rng = np.random.default_rng(seed)
    n = n_dates * n_entities
    X = rng.standard_normal((n, nf)).astype(np.float32)
    X[rng.random((n, nf)) < 0.03] = np.nan
    y = np.sign(np.nan_to_num(X[:, 0]) * np.nan_to_num(X[:, 1])) + 0.3 * rng.standard_normal(n)
    ts = np.repeat(np.arange(n_dates), n_entities).astype(np.int64)
    ent = np.tile(np.arange(n_entities), n_dates).astype(np.int64)
    return _Panel(X, y, ts, ent)


def categorical_panel(seed=3, n_dates=60, n_entities=100, nf=6):
    """Categorical columns 0 (12 values), 3 (400 values: the most frequent 254 are kept) and 5
    (6 common values and rare ones below cat_min_count), with NaNs."""
    rng = np.random.default_rng(seed)
    n = n_dates * n_entities
    X = rng.standard_normal((n, nf))
    X[:, 0] = rng.integers(0, 12, n)
    X[:, 3] = rng.integers(0, 400, n)
    X[:, 5] = np.where(rng.random(n) < 0.02, rng.integers(100, 130, n), rng.integers(0, 6, n))
    X[rng.random((n, nf)) < 0.03] = np.nan
    eff = np.array([0.9, -0.4, 0.1, 1.2, -1.0, 0.0, 0.5, 0.3, -0.7, 0.2, 0.0, -0.2])
    y = eff[np.nan_to_num(X[:, 0], nan=0).astype(int) % 12] + 0.3 * np.nan_to_num(X[:, 1]) + 0.5 * rng.standard_normal(n)
    ts = np.repeat(np.arange(n_dates), n_entities).astype(np.int64)
    ent = np.tile(np.arange(n_entities), n_dates).astype(np.int64)
    p = _Panel(X, y, ts, ent)
    p.is_cat = np.array([1, 0, 0, 1, 0, 1], np.int32)
    return p


FIT_CAT = dict(n_estimators=5, learning_rate=0.1, max_depth=6, max_leaves=20, horizon=1, objective="mse",
               random_state=2)


def main() -> None:
    L = bind.ref_lib()
    # binner
    X = _X(0, 6000, 10)
    n, nf = X.shape
    edges = np.zeros(nf * 256)
    ne = np.zeros(nf, np.int32)
    nbc = np.zeros(nf, np.int32)
    mb = C.c_int()
    codes = np.zeros((n, nf), np.uint16)
    rc = L.ref_binner(np.ascontiguousarray(X), n, nf, 255, 2000, 9, edges, ne, nbc, C.byref(mb),
                      codes.ctypes.data_as(C.c_void_p))
    assert rc == 0
    np.savez_compressed(os.path.join(HERE, "binner.npz"), X=X, max_bin=255, bin_sample=2000, seed=9,
                        edges=edges.reshape(nf, 256), n_edges=ne, n_bins_col=nbc, max_bins=mb.value, codes=codes)
    # histogram over a row subset
    rng = np.random.default_rng(1)
    idx = np.sort(rng.choice(n, 2500, replace=False)).astype(np.int32)
    g = rng.standard_normal(n)
    h = rng.random(n) + 0.5
    col = np.ascontiguousarray(codes.T)
    hist = np.zeros(nf * 255 * 3)
    L.ref_build_hist_col(col, n, nf, idx, idx.size, g, h, 255, 1, hist)
    np.savez_compressed(os.path.join(HERE, "hist.npz"), codes=codes, idx=idx, g=g, h=h, n_bins=255,
                        hist=hist.reshape(nf, 255, 3))
    # split scan on that histogram
    res = np.zeros(nf)
    thr = np.zeros(nf, np.int32)
    ml = np.zeros(nf, np.int32)
    for f in range(nf):
        r = np.zeros(1)
        ir = np.zeros(3, np.int32)
        L.ref_best_numeric(hist, nf, 255, f, 1.0, 0.0, 20, 1e-3, r, ir)
        res[f], thr[f], ml[f] = r[0], ir[1], ir[2]
    np.savez_compressed(os.path.join(HERE, "split.npz"), gain=res, threshold=thr, missing_left=ml, l2=1.0,
                        gamma=0.0, min_leaf=20, min_hess=1e-3)
    # pairwise gradients
    rng = np.random.default_rng(2)
    sizes = np.array([1, 2, 3, 20, 48, 49, 50, 97, 300, 801])
    groups = np.repeat(np.arange(sizes.size, dtype=np.int64), sizes)
    m = groups.size
    y = np.round(rng.standard_normal(m), 2)
    pred = rng.standard_normal(m) * 0.2
    gp = np.zeros(m)
    hp = np.zeros(m)
    L.ref_grad_hess(5, y, pred, groups.ctypes.data_as(C.c_void_p), m, gp, hp)
    loss = L.ref_loss(5, y, pred, groups.ctypes.data_as(C.c_void_p), m)
    np.savez_compressed(os.path.join(HERE, "pairwise.npz"), y=y, pred=pred, groups=groups, g=gp, h=hp, loss=loss)
    # fits
    for name, params, p in (("fit_mse", FIT_MSE, panels.panel_scale(n_dates=40, n_entities=300, n_features=12)),
                            ("fit_pair", FIT_PAIR, panels.panel_pairwise(n_dates=30, n_features=10)),
                            ("fit_pairsplit", FIT_PAIRSPLIT, interaction_panel()),
                            ("fit_cat", FIT_CAT, categorical_panel())):
        Xp = p.X.astype(np.float64)
        is_cat = getattr(p, "is_cat", None)
        res, hnd = bind.ref_fit(params, Xp, p.y, p.ts, p.entity, is_cat=is_cat)
        pr = bind.ref_predict(hnd, Xp[:500])
        bind.ref_free(hnd)
        arrs = {"X": p.X, "y": p.y, "ts": p.ts, "entity": p.entity, "pred": pr, "init_score": res.init_score,
                "init_prefix": res.init_prefix, "evals": res.evals_train, "n_bins": res.n_bins,
                "n_buckets": res.n_buckets, "n_trees": len(res.trees)}
        for t, tr in enumerate(res.trees):
            for fld in ("is_leaf", "feature", "threshold", "left", "right", "missing_left", "n_samples", "depth",
                        "value", "gain", "values", "cover", "prefix", "split_type", "feature2"):
                arrs[f"t{t}_{fld}"] = getattr(tr, fld)
            if is_cat is not None:
                arrs[f"t{t}_cat_left"] = tr.cat_left
        if is_cat is not None:
            arrs["is_cat"] = is_cat
        arrs["params"] = np.array(repr(params))
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **arrs)
    print("fixtures written to", HERE)


if __name__ == "__main__":
    main()
