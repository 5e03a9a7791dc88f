"""Expanding-window walk-forward folds with purge and embargo: the folds of the batched
walk-forward workload, as WalkForwardSplit.split makes them (src/tidegbm/cv.py:35-60)
for integer timestamps (date indices).

The unique timestamps are cut into n_splits + 2 equal chunks (np.linspace); fold i tests
on chunk i (i = 1 .. n_splits) and trains on every row strictly before the test's first
timestamp minus embargo and purge.  Embargo and purge count timestamp steps: they are
multiplied by the median positive gap between consecutive unique timestamps
(parse_horizon, src/tidegbm/utils.py:47-69).  A fold whose training set has fewer than
max(min_train_fraction * n, 10) rows, or whose test set is empty, is skipped.
"""
from __future__ import annotations

import numpy as np


def _median_step(uniq: np.ndarray) -> int:
    if uniq.size < 2:
        return 1
    d = np.diff(uniq)
    d = d[d > 0]
    return max(int(np.median(d)), 1) if d.size else 1


def walk_forward_folds(ts, n_splits: int, embargo: int = 0, purge: int = 0,
                       min_train_fraction: float = 0.3) -> list[tuple[np.ndarray, np.ndarray]]:
    """(train_idx, test_idx) int32 pairs, in fold order."""
    if n_splits < 2:
        raise ValueError("n_splits must be >= 2")
    ts = np.asarray(ts)
    if not np.issubdtype(ts.dtype, np.integer):
        raise ValueError("integer timestamps (date indices) expected")
    ts = ts.astype(np.int64).ravel()
    n = ts.shape[0]
    uniq = np.unique(ts)
    if uniq.size < n_splits + 2:
        raise ValueError("not enough unique timestamps for n_splits")
    step = _median_step(uniq)
    gap = (int(embargo) + int(purge)) * step
    bounds = np.linspace(0, uniq.size, n_splits + 2, dtype=int)
    min_train = int(min_train_fraction * n)
    folds = []
    for i in range(1, n_splits + 1):
        lo, hi = int(bounds[i]), int(bounds[i + 1])
        t0, t1 = uniq[lo], uniq[max(hi - 1, lo)]
        train = np.flatnonzero(ts < t0 - gap)
        test = np.flatnonzero((ts >= t0) & (ts <= t1))
        if train.size < max(min_train, 10) or test.size == 0:
            continue
        folds.append((train.astype(np.int32), test.astype(np.int32)))
    return folds
