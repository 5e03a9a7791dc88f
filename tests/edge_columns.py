"""Columns at the edges of Binner::fit and Binner::transform (cpp/src/binning.cpp:14-134):
all missing, constant, two values, exactly 254 and 255 distinct values (254 uniques give
edges = values and a 256-wide histogram, binning.cpp:130-134; 255 go through the
quantile interpolation), infinities, signed zeros, magnitudes near the ends of the f64
range, 90% missing, heavy ties, and 255 or 64 distinct values of which one is +inf: with
max_bin - 1 = 254 (or 63) bins the interpolation then meets inf * 0 and the reference's
edges hold a NaN (binning.cpp:19-31), which its std::sort and upper_bound carry on."""
import numpy as np


def edge_columns(seed=0, n=6000):
    rng = np.random.default_rng(seed)
    cols = []
    cols.append(np.full(n, np.nan))                                            # all missing
    cols.append(np.full(n, 3.5))                                               # constant
    cols.append(rng.choice([-1.25, 2.0], n))                                   # two values
    cols.append(rng.choice(np.sort(rng.standard_normal(254)), n))              # 254 distinct
    cols.append(rng.choice(np.sort(rng.standard_normal(255)), n))              # 255 distinct
    c = rng.standard_normal(n)
    c[rng.random(n) < 0.05] = np.inf
    c[rng.random(n) < 0.05] = -np.inf
    cols.append(c)                                                             # infinities
    c = rng.choice([-0.0, 0.0, 1.0, -1.0, 0.5], n)
    cols.append(c)                                                             # signed zeros
    c = rng.standard_normal(n) * np.where(rng.random(n) < 0.5, 1e300, 1e-300)
    cols.append(c)                                                             # extreme magnitudes
    c = rng.standard_normal(n)
    c[rng.random(n) < 0.9] = np.nan
    cols.append(c)                                                             # 90% missing
    cols.append(rng.integers(0, 1000, n).astype(float))                        # heavy ties
    cols.append(rng.choice(np.append(np.sort(rng.standard_normal(254)), np.inf), n))  # 255 distinct, +inf
    cols.append(rng.choice(np.append(np.sort(rng.standard_normal(63)), np.inf), n))   # 64 distinct, +inf
    return np.ascontiguousarray(np.column_stack(cols))
