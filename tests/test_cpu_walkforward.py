"""The batched walk-forward workload's folds (tidegbm_b200/walkforward.py) against the
reference's WalkForwardSplit (src/tidegbm/cv.py:35-60), through the golden folds that
tests/golden/make_folds.py recorded from it: unit and wider timestamp steps, embargo and
purge, uneven dates, unsorted timestamps, skipped short folds."""
import os

import numpy as np
import pytest

from tidegbm_b200.walkforward import walk_forward_folds

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.parametrize("name", ["walkforward16", "gaps", "uneven", "unsorted"])
def test_folds_match_reference(name):
    d = np.load(os.path.join(HERE, "golden", "folds.npz"))
    n_splits, embargo, purge, mtf = d[f"{name}_params"]
    folds = walk_forward_folds(d[f"{name}_ts"], int(n_splits), int(embargo), int(purge), float(mtf))
    n = int(d[f"{name}_n_folds"])
    assert len(folds) == n
    for k, (train, test) in enumerate(folds):
        assert np.array_equal(train, d[f"{name}_{k}_train"]), (k, "train")
        assert np.array_equal(test, d[f"{name}_{k}_test"]), (k, "test")


def test_expanding_windows_on_sorted_rows():
    """On time-sorted rows every training set is a prefix that grows fold by fold, and no
    training row is within the embargo of its test."""
    ts = np.repeat(np.arange(1000, dtype=np.int64), 7)
    folds = walk_forward_folds(ts, 16, embargo=5, min_train_fraction=0.1)
    sizes = [tr.size for tr, _ in folds]
    assert sizes == sorted(sizes) and len(folds) >= 14
    for tr, te in folds:
        assert np.array_equal(tr, np.arange(tr.size))
        assert ts[tr].max() < ts[te].min() - 5
