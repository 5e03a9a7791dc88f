"""Batched tree growth (grow = 1, the default): many leaves, and many fits, per launch.

The waves replay the reference's best-first order exactly, so a batched fit must give
the very trees the one-split loop (grow = 0) gives, bit for bit: node ids, splits,
counts, node values, full-data leaf values, TORB prefixes, losses.  Both compute exact
64-bit fixed-point histograms, so the comparison is exact equality, not a tolerance.
Batched fits of several contexts (tgb_fit_batch: walk-forward folds) must each equal the
context's own fit, and the CUDA-graph loop must equal the host-enqueued waves.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _same(a, b):
    ta, tb = a.trees(), b.trees()
    assert len(ta) == len(tb)
    for t, (x, y) in enumerate(zip(ta, tb)):
        for fld in ("is_leaf", "feature", "threshold", "left", "right", "missing_left", "n_samples", "depth",
                    "cover", "value", "gain", "values", "prefix"):
            assert np.array_equal(getattr(x, fld), getattr(y, fld)), (t, fld)
    assert np.array_equal(a.evals_result()["train"], b.evals_result()["train"])
    assert np.array_equal(a.init_prefix(), b.init_prefix())


def _fit(native, p, **params):
    b = native.Booster(**params)
    b.fit(p.X, p.y, timestamps=p.ts, entity=p.entity)
    return b


CASES = {
    "mse": (dict(n_dates=200, n_entities=250, n_features=32),
            dict(n_estimators=12, learning_rate=0.08, max_depth=6, horizon=1, objective="mse", goss=0)),
    "mse_goss_lognormal": ("scale", dict(n_estimators=8, learning_rate=0.1, max_depth=8, horizon=5, objective="mse",
                                         goss=1, random_state=1, bin_sample=20000)),
    "pairwise": ("pairwise", dict(n_estimators=8, learning_rate=0.08, max_depth=6, horizon=1,
                                  objective="pairwise")),
    "leaves40_depth7": ("scale40", dict(n_estimators=5, learning_rate=0.1, max_depth=7, max_leaves=40, horizon=3,
                                        objective="mse", goss=1, random_state=3, bin_sample=30000)),
    "min_leaf_stops": (dict(n_dates=50, n_entities=80, n_features=12),
                       dict(n_estimators=4, learning_rate=0.1, max_depth=6, horizon=1, objective="mse", goss=0,
                            min_samples_leaf=400)),
    "stumps": (dict(n_dates=60, n_entities=100, n_features=8),
               dict(n_estimators=5, learning_rate=0.1, max_depth=1, horizon=1, objective="mse", goss=0)),
    "leaves255": (dict(n_dates=100, n_entities=400, n_features=16),
                  dict(n_estimators=3, learning_rate=0.1, max_depth=12, max_leaves=255, min_samples_leaf=5,
                       horizon=1, objective="mse", goss=0)),
}


def _panel(spec):
    from tidegbm_b200 import panels

    if spec == "scale":
        return panels.panel_scale(n_dates=60, n_entities=1500, n_features=20)
    if spec == "scale40":
        return panels.panel_scale(n_dates=41, n_entities=1333, n_features=40, seed=7)
    if spec == "pairwise":
        return panels.panel_pairwise(n_dates=80)
    return panels.panel_small(**spec)


@pytest.mark.parametrize("name", sorted(CASES))
def test_waves_equal_one_split_loop(native, name):
    spec, params = CASES[name]
    p = _panel(spec)
    params = dict(params, pair_splits=False)
    _same(_fit(native, p, grow=1, **params), _fit(native, p, grow=0, **params))


@pytest.mark.parametrize("cap", [1, 2, 5])
def test_expansion_cap_grows_the_same_trees(native, cap):
    """wave_expand caps the speculative expansions a wave plans (1: only the best leaf,
    the one-split order in waves); every cap grows the same trees, with more waves and
    fewer expansions than the uncapped default."""
    from tidegbm_b200 import panels

    p = panels.panel_scale(n_dates=60, n_entities=1500, n_features=20)
    params = dict(n_estimators=6, learning_rate=0.1, max_depth=8, horizon=1, objective="mse", goss=1,
                  pair_splits=False, grow=1, timing_from=0)
    a = _fit(native, p, wave_expand=cap, **params)
    b = _fit(native, p, **params)
    _same(a, b)
    sa, sb = a.fit_stats(), b.fit_stats()
    assert sa["expansions"] <= sb["expansions"]
    assert sa["timed_selects"] >= sb["timed_selects"]
    if cap == 1:  # one expansion per select: every expansion is committed
        assert sa["expansions"] == sum(int((~t.is_leaf.astype(bool)).sum()) for t in a.trees())


def test_graph_loop_equals_host_waves(native):
    from tidegbm_b200 import panels

    p = panels.panel_scale(n_dates=60, n_entities=1500, n_features=20)
    params = dict(n_estimators=6, learning_rate=0.1, max_depth=8, horizon=1, objective="mse", goss=1,
                  pair_splits=False, grow=1)
    a = _fit(native, p, graph=1, **params)
    b = _fit(native, p, graph=0, **params)
    _same(a, b)
    assert a.fit_stats()["graph_used"] in (0.0, 1.0)


@pytest.mark.parametrize("objective", ["mse", "pairwise"])
def test_batched_folds_equal_own_fits(native, objective):
    """Expanding walk-forward folds (row prefixes of one time-sorted panel) fitted together
    through tgb_fit_batch: each fold's model equals the fold fitted alone."""
    from tidegbm_b200 import panels

    p = panels.panel_pairwise(n_dates=120) if objective == "pairwise" else panels.panel_small(n_dates=240)
    ends = (40, 70, 100, 120) if objective == "pairwise" else (60, 100, 180, 240)
    his = [int(np.searchsorted(p.ts, d)) for d in ends]
    params = dict(n_estimators=6, learning_rate=0.08, max_depth=6, horizon=1, objective=objective, goss=1,
                  random_state=2, pair_splits=False)
    bs = [native.Booster(**params) for _ in his]
    native.Booster.fit_batch(bs, [p.X[:h] for h in his], [p.y[:h] for h in his], [p.ts[:h] for h in his],
                             [p.entity[:h] for h in his])
    for b, h in zip(bs, his):
        own = native.Booster(**params)
        own.fit(p.X[:h], p.y[:h], timestamps=p.ts[:h], entity=p.entity[:h])
        _same(b, own)
        np.testing.assert_array_equal(b.raw_predict(p.X[:500]), own.raw_predict(p.X[:500]))


@pytest.mark.parametrize("bits", [16, 8])
@pytest.mark.parametrize("objective", ["mse", "pairwise"])
def test_quantised_histograms_track_exact(native, bits, objective):
    """hist_bits 16 / 8: stochastically rounded gradients (and hessians) summed exactly; the
    split search is approximate, the leaf values exact.  The fit must stay close to the exact
    one: same training loss within 2% after 20 trees, and a held-out IC within 0.02."""
    from tidegbm_b200 import panels

    if objective == "mse":
        p = panels.panel_small(n_dates=300, n_entities=250, n_features=24)
        ho = panels.panel_small(n_dates=100, n_entities=250, n_features=24, seed=9)
    else:
        p = panels.panel_pairwise(n_dates=200)
        ho = panels.panel_pairwise(n_dates=80, seed=9)
    params = dict(n_estimators=20, learning_rate=0.1, max_depth=6, horizon=1, objective=objective, goss=0,
                  pair_splits=False)
    ex = _fit(native, p, **params)
    q = _fit(native, p, hist_bits=bits, **params)
    le, lq = ex.evals_result()["train"][-1], q.evals_result()["train"][-1]
    assert abs(lq - le) <= 0.02 * abs(le) + 1e-6, (le, lq)

    def ic(pred, panel):
        out = []
        for d in np.unique(panel.ts):
            m = panel.ts == d
            a, b = pred[m] - pred[m].mean(), panel.y[m] - panel.y[m].mean()
            den = np.sqrt((a * a).sum() * (b * b).sum())
            if den > 0:
                out.append((a * b).sum() / den)
        return float(np.mean(out))

    assert abs(ic(q.raw_predict(ho.X), ho) - ic(ex.raw_predict(ho.X), ho)) <= 0.02


@pytest.mark.parametrize("n_features,hist_bits,goss", [(40, 0, 1), (128, 0, 0), (20, 16, 1), (72, 8, 1), (8, 0, 1),
                                                       (33, 16, 1), (256, 0, 0)])
def test_tma_staging_grows_the_same_trees(native, n_features, hist_bits, goss):
    """hist_stage 1 stages the code rows of the constant-hessian histograms in shared
    memory by TMA gathers (32 bytes of each of 4 rows per gather, a feature group past
    the row's last code filled with zeros), 0 loads them lane by lane: the same integer
    sums, so the same trees bit for bit.  40, 72 and 33 features end in a partial group
    (33: one feature in a 48-byte row); 256 features are eight groups; 8 features
    (16-byte rows) cannot be addressed by the gathers and load directly."""
    from tidegbm_b200 import panels

    p = panels.panel_small(n_dates=120, n_entities=300, n_features=n_features, seed=11)
    params = dict(n_estimators=4, learning_rate=0.1, max_depth=7, max_leaves=48, horizon=1, objective="mse",
                  goss=goss, random_state=5, hist_bits=hist_bits, pair_splits=False)
    _same(_fit(native, p, hist_stage=1, **params), _fit(native, p, hist_stage=0, **params))
