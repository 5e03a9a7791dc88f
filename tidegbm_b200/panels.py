"""Seeded synthetic panels (dates x entities x features) for the five workloads.

No public dataset is involved: every panel is drawn from a fixed-seed generator
with the shapes and value distributions of the named workloads.  Rows come out
sorted by (date, entity), as TideGBM's Python layer hands them to the core
(src/tidegbm/native.py:96-102).  Generation is chunked by date with one child
seed per chunk, so the result does not depend on the thread count.

    panel_small          400 dates x 250 entities = 100,000 rows, 32 features, mse
    panel_pairwise       2,000 dates, Uniform{50..800} entities (~0.85M rows), 64 features
    panel_scale          5,000 dates x 2,000 entities = 10M rows, 128 features
    panel_walkforward    panel_pairwise's generator at 8,000 dates (~3.4M rows)
"""
from __future__ import annotations

import os
from concurrent.futures import ThreadPoolExecutor
from dataclasses import dataclass

import numpy as np


@dataclass
class Panel:
    X: np.ndarray          # float32, row-major n x F
    y: np.ndarray          # float64, demeaned within date
    ts: np.ndarray         # int64 date index, non-decreasing
    entity: np.ndarray     # int32
    name: str

    @property
    def n(self) -> int:
        return int(self.X.shape[0])

    @property
    def n_features(self) -> int:
        return int(self.X.shape[1])


def _threads() -> int:
    return max(1, min(32, os.cpu_count() or 1))


def _demean_by_date(y: np.ndarray, ts: np.ndarray) -> np.ndarray:
    starts = np.flatnonzero(np.r_[True, ts[1:] != ts[:-1]])
    sums = np.add.reduceat(y, starts)
    counts = np.diff(np.r_[starts, y.size])
    return y - np.repeat(sums / counts, counts)


def _chunked(sizes: np.ndarray, n_features: int, seed: int, fill) -> tuple[np.ndarray, np.ndarray]:
    """Runs fill(rng, m_rows, X_out, lin_out) over date chunks in threads."""
    n = int(sizes.sum())
    X = np.empty((n, n_features), dtype=np.float32)
    lin = np.empty(n, dtype=np.float64)
    n_dates = sizes.size
    n_chunks = max(1, min(256, n_dates))
    bounds = np.linspace(0, n_dates, n_chunks + 1).astype(np.int64)
    row0 = np.r_[0, np.cumsum(sizes)]

    def job(c: int) -> None:
        d0, d1 = int(bounds[c]), int(bounds[c + 1])
        if d1 <= d0:
            return
        r0, r1 = int(row0[d0]), int(row0[d1])
        rng = np.random.default_rng([seed, c])
        fill(rng, sizes[d0:d1], X[r0:r1], lin[r0:r1])

    with ThreadPoolExecutor(_threads()) as ex:
        list(ex.map(job, range(n_chunks)))
    return X, lin


def panel_small(n_dates: int = 400, n_entities: int = 250, n_features: int = 32, seed: int = 0) -> Panel:
    """Plain method, small: N(0,1) features with pairwise correlation 0.3 through a
    shared per-date factor; y = 0.05 (w . x) + N(0,1), demeaned within date."""
    w = np.random.default_rng([seed, 10**6]).standard_normal(n_features)
    sizes = np.full(n_dates, n_entities, dtype=np.int64)
    a, b = np.sqrt(0.3), np.sqrt(0.7)

    def fill(rng, sz, Xo, lo):
        m = int(sz.sum())
        z = np.repeat(rng.standard_normal(sz.size), sz)[:, None]
        Xo[:] = a * z + b * rng.standard_normal((m, n_features))
        lo[:] = 0.05 * (Xo.astype(np.float64) @ w) + rng.standard_normal(m)

    X, lin = _chunked(sizes, n_features, seed, fill)
    ts = np.repeat(np.arange(n_dates, dtype=np.int64), sizes)
    ent = np.concatenate([np.arange(s, dtype=np.int32) for s in sizes])
    return Panel(X, _demean_by_date(lin, ts), ts, ent, "panel_small")


def panel_pairwise(n_dates: int = 2000, n_features: int = 64, seed: int = 1,
                   lo_ent: int = 50, hi_ent: int = 800) -> Panel:
    """Uneven cross-sections: entities per date ~ Uniform{lo_ent..hi_ent}; features
    N(0,1) with 10% of columns Student-t (nu = 3) and 2% NaN; y as panel_small."""
    rng0 = np.random.default_rng([seed, 10**6])
    sizes = rng0.integers(lo_ent, hi_ent + 1, size=n_dates).astype(np.int64)
    w = rng0.standard_normal(n_features)
    heavy = np.zeros(n_features, dtype=bool)
    heavy[rng0.choice(n_features, max(1, n_features // 10), replace=False)] = True
    a, b = np.sqrt(0.3), np.sqrt(0.7)

    def fill(rng, sz, Xo, lo):
        m = int(sz.sum())
        z = np.repeat(rng.standard_normal(sz.size), sz)[:, None]
        V = a * z + b * rng.standard_normal((m, n_features))
        V[:, heavy] = rng.standard_t(3.0, size=(m, int(heavy.sum())))
        lo[:] = 0.05 * (V @ w) + rng.standard_normal(m)
        V[rng.random((m, n_features)) < 0.02] = np.nan
        Xo[:] = V

    X, lin = _chunked(sizes, n_features, seed, fill)
    ts = np.repeat(np.arange(n_dates, dtype=np.int64), sizes)
    ent = np.concatenate([np.arange(s, dtype=np.int32) for s in sizes])
    return Panel(X, _demean_by_date(lin, ts), ts, ent, "panel_pairwise")


def panel_scale(n_dates: int = 5000, n_entities: int = 2000, n_features: int = 128, seed: int = 2,
                sample_seed: int | None = None) -> Panel:
    """Scale: N(0,1) columns mixed with log-normal (sigma = 1) columns (every fourth
    column), 1% NaN; y = 16-sparse linear + 0.1 sin(x_k) + N(0,1), demeaned.  `seed` fixes
    the target function (support, weights), `sample_seed` (default: seed) the rows, so a
    held-out panel of the same function takes another sample_seed."""
    rng0 = np.random.default_rng([seed, 10**6])
    n_support = min(16, n_features)
    support = rng0.choice(n_features, n_support, replace=False)
    w = rng0.standard_normal(n_support)
    k_sin = int(rng0.integers(n_features))
    lognorm = (np.arange(n_features) % 4) == 3
    sizes = np.full(n_dates, n_entities, dtype=np.int64)

    def fill(rng, sz, Xo, lo):
        m = int(sz.sum())
        Xo[:] = rng.standard_normal((m, n_features), dtype=np.float32)
        Xo[:, lognorm] = np.exp(Xo[:, lognorm])
        sig = Xo[:, support].astype(np.float64) @ w + 0.1 * np.sin(Xo[:, k_sin].astype(np.float64))
        lo[:] = sig + rng.standard_normal(m)
        Xo[rng.random((m, n_features), dtype=np.float32) < 0.01] = np.nan

    X, lin = _chunked(sizes, n_features, seed if sample_seed is None else sample_seed, fill)
    ts = np.repeat(np.arange(n_dates, dtype=np.int64), sizes)
    ent = np.tile(np.arange(n_entities, dtype=np.int32), n_dates)
    return Panel(X, _demean_by_date(lin, ts), ts, ent, "panel_scale")


def panel_walkforward(n_dates: int = 8000, n_features: int = 64, seed: int = 3) -> Panel:
    """Batched walk-forward workload: panel_pairwise's generator at 8,000 dates."""
    p = panel_pairwise(n_dates=n_dates, n_features=n_features, seed=seed)
    p.name = "panel_walkforward"
    return p
