"""The serving loop on the GPU (tgb_server_*): fit and predict requests of different
sizes, objectives and precision modes admitted together, running concurrently on their
boosters' own streams.  Each result must be the same as the request run alone, bit for
bit: the fits share no device state (their buffers are their own and are freed in the
order of their own stream) and their arithmetic does not depend on what else runs."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _requests():
    from tidegbm_b200 import panels

    small = panels.panel_small(n_dates=160, n_entities=250, n_features=32, seed=4)
    pair = panels.panel_pairwise(n_dates=90, n_features=32, seed=5)
    big = panels.panel_scale(n_dates=150, n_entities=2000, n_features=64, seed=6)
    base = dict(learning_rate=0.08, horizon=1, pair_splits=False)
    return [
        (small, dict(base, n_estimators=15, max_depth=6, objective="mse", goss=0)),
        (pair, dict(base, n_estimators=8, max_depth=6, objective="pairwise")),
        (big, dict(base, n_estimators=6, max_depth=8, objective="mse", goss=1, hist_bits=8)),
        (small, dict(base, n_estimators=10, max_depth=7, objective="mse", goss=0, hist_bits=16, random_state=3)),
        (big, dict(base, n_estimators=5, max_depth=8, objective="mse", goss=1, grow=0)),
    ]


def _trees(b):
    return [(t.feature.copy(), t.threshold.copy(), t.left.copy(), t.values.copy(), t.prefix.copy()) for t in b.trees()]


def test_results_alone_equal_results_in_the_mix(native):
    reqs = _requests()
    alone = []
    for p, params in reqs:
        b = native.Booster(**params)
        b.fit(p.X, p.y, timestamps=p.ts, entity=p.entity)
        alone.append((_trees(b), b.raw_predict(p.X[:3000])))

    srv = native.Server(device=0, budget_bytes=60e9, slots=8)
    boosters = [native.Booster(**params) for _, params in reqs]
    ids = [srv.submit_fit(b, p.X, p.y, timestamps=p.ts, entity=p.entity) for b, (p, _) in zip(boosters, reqs)]
    # predicts queued behind their model's fit (one request per model at a time)
    preds = [srv.submit_predict(b, p.X[:3000]) for b, (p, _) in zip(boosters, reqs)]
    for rid in ids:
        assert srv.wait(rid) == native.Server.DONE
    for rid, _ in preds:
        assert srv.wait(rid) == native.Server.DONE
    st = srv.stats()
    srv.close()
    assert st["completed"] == 2 * len(reqs) and st["failed"] == 0
    assert st["peak_running"] >= 2  # requests did overlap
    for k, (b, (trees_a, pred_a)) in enumerate(zip(boosters, alone)):
        trees_m = _trees(b)
        assert len(trees_m) == len(trees_a)
        for ta, tm in zip(trees_a, trees_m):
            for x, y in zip(ta, tm):
                assert np.array_equal(x, y), k
        assert np.array_equal(preds[k][1], pred_a), k


def test_oversized_request_is_refused_and_others_run(native):
    from tidegbm_b200 import panels

    p = panels.panel_small(n_dates=40, n_entities=100, n_features=8)
    srv = native.Server(device=0, budget_bytes=2e6, slots=2)
    b = native.Booster(n_estimators=3, horizon=1, pair_splits=False, goss=0)
    with pytest.raises(native.TideError):
        srv.submit_fit(b, np.zeros((200000, 64), np.float32), np.zeros(200000), timestamps=np.arange(200000))
    srv.close()
    srv = native.Server(device=0, budget_bytes=10e9, slots=2)
    rid = srv.submit_fit(b, p.X, p.y, timestamps=p.ts, entity=p.entity)
    assert srv.wait(rid) == native.Server.DONE
    srv.close()
