"""Golden walk-forward folds from the reference's own WalkForwardSplit
(src/tidegbm/cv.py, with src/tidegbm/utils.py), loaded as standalone modules from the
reference checkout in this container.

    TIDEGBM_REF=<reference checkout> python tests/golden/make_folds.py   # writes tests/golden/folds.npz

Each case stores its timestamps, parameters and, per fold, the train and test indices.
"""
from __future__ import annotations

import importlib.util
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.path.join(os.environ.get("TIDEGBM_REF", ""), "src", "tidegbm")

CASES = [  # (name, timestamps, n_splits, embargo, purge, min_train_fraction)
    ("walkforward16", np.repeat(np.arange(800, dtype=np.int64), 5), 16, 5, None, 0.3),
    ("gaps", np.repeat(np.arange(0, 600, 3, dtype=np.int64), 4), 6, 2, 1, 0.2),
    ("uneven", np.sort(np.random.default_rng(4).integers(0, 300, 2500)).astype(np.int64), 8, 3, None, 0.1),
    ("unsorted", np.random.default_rng(5).integers(0, 120, 900).astype(np.int64), 5, 1, 2, 0.3),
]


def _load(name, path):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def main() -> None:
    pkg = types.ModuleType("tidegbm")
    pkg.__path__ = []
    sys.modules["tidegbm"] = pkg
    _load("tidegbm.utils", os.path.join(REF, "utils.py"))
    cv = _load("tidegbm.cv", os.path.join(REF, "cv.py"))
    out = {}
    for name, ts, n_splits, embargo, purge, mtf in CASES:
        folds = list(cv.WalkForwardSplit(n_splits=n_splits, embargo=embargo, purge=purge,
                                         min_train_fraction=mtf).split(None, timestamp=ts))
        out[f"{name}_ts"] = ts
        out[f"{name}_params"] = np.array([n_splits, embargo or 0, purge or 0, mtf])
        out[f"{name}_n_folds"] = np.array(len(folds))
        for k, (tr, te) in enumerate(folds):
            out[f"{name}_{k}_train"] = tr
            out[f"{name}_{k}_test"] = te
    np.savez_compressed(os.path.join(HERE, "folds.npz"), **out)
    print("wrote", os.path.join(HERE, "folds.npz"))


if __name__ == "__main__":
    main()
