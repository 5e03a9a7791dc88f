"""Parity at the workloads' stated sizes (the bench's configurations), not only at small
ones.

- Pairwise, 2,000 dates x Uniform{50..800} entities (~0.85M rows), 64 features: 20 trees
  against the oracle restatement, structure identical, values within 1e-9.
- Scale, 10M rows x 128 features, GOSS: the codes of the whole panel bit for bit against
  the oracle's transform with the oracle's edges (both computed here), and tree 0 (its
  gradients are identical before the first update, so the GOSS sample is too) identical
  to the oracle's tree 0.  The oracle is single-threaded; its calls run per feature / per
  row chunk in threads (ctypes releases the GIL), so the test takes a few minutes.
"""
import ctypes as C
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest
from missing_bins import empty_missing_nodes

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def _compare(gpu, ref, codes, n_bins, atol=1e-9, n_trees=None):
    """Structure and values; missing directions at every split node whose missing bin holds
    rows (missing_bins.py: an empty missing bin's direction is FP64 residue in the reference)."""
    trees_g = gpu.trees()[:n_trees] if n_trees else gpu.trees()
    trees_r = ref.trees[:n_trees] if n_trees else ref.trees
    assert len(trees_g) == len(trees_r)
    for t, (a, b) in enumerate(zip(trees_g, trees_r)):
        for fld in ("is_leaf", "feature", "threshold", "left", "right", "n_samples", "depth"):
            assert np.array_equal(getattr(a, fld), getattr(b, fld)), (t, fld)
        differ = set(np.flatnonzero(np.asarray(a.missing_left) != np.asarray(b.missing_left)).tolist())
        if differ:
            assert differ <= empty_missing_nodes(b, codes, n_bins), (t, "missing_left", sorted(differ))
        assert np.array_equal(a.cover, b.cover), t
        np.testing.assert_allclose(a.value, b.value, rtol=0, atol=atol)
        np.testing.assert_allclose(a.values, b.values, rtol=0, atol=atol)
        np.testing.assert_allclose(a.prefix, b.prefix, rtol=0, atol=atol)


def test_pairwise_2000_dates_matches_oracle(native, oracle):
    from tidegbm_b200 import panels

    p = panels.panel_pairwise(n_dates=2000)
    assert 800_000 < p.n < 900_000 and p.n_features == 64
    params = dict(n_estimators=20, learning_rate=0.08, max_depth=6, horizon=1, objective="pairwise",
                  random_state=0, pair_splits=False)
    gpu = native.Booster(**params)
    gpu.fit(p.X, p.y, timestamps=p.ts, entity=p.entity)
    ref, h = oracle.oracle_fit(params, p.X.astype(np.float64), p.y, p.ts, p.entity)
    codes, nb = oracle.oracle_codes(p.X, params)
    try:
        _compare(gpu, ref, codes, nb)
        np.testing.assert_allclose(gpu.evals_result()["train"], ref.evals_train, rtol=1e-9, atol=1e-9)
    finally:
        oracle.oracle_free(h)


def test_scale_10m_codes_and_first_tree_match_oracle(native, oracle):
    from tidegbm_b200 import panels

    p = panels.panel_scale()  # 10M x 128, 1% NaN, log-normal columns
    n, nf = p.X.shape
    params = dict(n_estimators=1, learning_rate=0.1, max_depth=8, max_leaves=31, horizon=1, objective="mse",
                  goss=-1, random_state=0, pair_splits=False)
    gpu = native.Booster(**params)
    gpu.fit(p.X, p.y, timestamps=p.ts, entity=p.entity)
    L = oracle.oracle_lib()
    # oracle edges, one feature per call (seed + f * 2654435761 is the seed of column f)
    e_ref = np.zeros((nf, 256))
    n_ref = np.zeros(nf, np.int32)

    def fit_feature(f):
        col = np.ascontiguousarray(p.X[:, f], dtype=np.float64)
        e = np.zeros(256)
        ne = np.zeros(1, np.int32)
        nbc = np.zeros(1, np.int32)
        L.orc_binner_fit(col, n, 1, 255, 262144, (0 + f * 2654435761) & 0xFFFFFFFF, e, ne, nbc)
        e_ref[f] = e
        n_ref[f] = ne[0]

    with ThreadPoolExecutor(16) as ex:
        list(ex.map(fit_feature, range(nf)))
    for f in range(nf):
        assert gpu.edges(f).size == n_ref[f]
        assert np.array_equal(gpu.edges(f).view(np.uint64), e_ref[f, : n_ref[f]].view(np.uint64)), f
    # codes of the whole panel: this library's transform against the oracle's
    from bench import device_codes

    codes = device_codes(native, gpu, p.X)[:, :nf].cpu().numpy()
    flat_e = np.ascontiguousarray(e_ref.reshape(-1))
    chunks = np.array_split(np.arange(n), 64)

    def check_chunk(idx):
        lo, hi = int(idx[0]), int(idx[-1]) + 1
        Xc = np.ascontiguousarray(p.X[lo:hi], dtype=np.float64)
        out = np.zeros((hi - lo) * nf, np.uint8)
        L.orc_bin_transform(Xc, hi - lo, nf, flat_e, n_ref, out, nf)
        return bool(np.array_equal(out.reshape(hi - lo, nf), codes[lo:hi]))

    with ThreadPoolExecutor(16) as ex:
        assert all(ex.map(check_chunk, chunks))
    # tree 0 against the oracle's fit of one tree (GOSS sample of 3M rows)
    ref, h = oracle.oracle_fit(params, p.X.astype(np.float64), p.y, p.ts, p.entity)
    try:
        _compare(gpu, ref, codes, ref.n_bins, n_trees=1)
    finally:
        oracle.oracle_free(h)
