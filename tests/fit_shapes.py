"""Small and ragged shapes of a fit: one to three features, 17 and 33 features (ragged
feature groups), 64 and 65 rows (GOSS needs more than 64 rows, cpp/src/booster.cpp:558),
and a pairwise fit over dates of 16 rows."""
SHAPES = [
    (20, 5, 1, {}),
    (20, 5, 2, {}),
    (30, 3, 3, {}),
    (8, 8, 4, dict(goss=1)),     # 64 rows: GOSS needs more than 64 (booster.cpp:558)
    (13, 5, 4, dict(goss=1)),    # 65 rows: GOSS on
    (10, 10, 17, dict(goss=1, goss_top=0.5, goss_other=0.2)),
    (40, 25, 33, {}),
    (4, 16, 2, dict(objective="pairwise")),
]


def shape_case(n_dates, n_ent, nf, extra):
    import numpy as np

    rng = np.random.default_rng(nf * 100 + n_dates)
    n = n_dates * n_ent
    X = rng.standard_normal((n, nf))
    X[rng.random((n, nf)) < 0.05] = np.nan
    y = np.nan_to_num(X[:, 0]) + 0.5 * rng.standard_normal(n)
    ts = np.repeat(np.arange(n_dates), n_ent).astype(np.int64)
    ent = np.tile(np.arange(n_ent), n_dates).astype(np.int64)
    params = {**dict(n_estimators=4, learning_rate=0.1, max_depth=4, horizon=1, objective="mse", random_state=1,
                     pair_splits=False, min_samples_leaf=5), **extra}
    return X, y, ts, ent, params
