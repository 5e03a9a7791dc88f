"""CPU-only checks: the C-ABI library loads and exports every declared symbol, the
host-side samplers reproduce libstdc++'s std::shuffle, and the host binner's edges
are bit-identical to the oracle's Binner::fit."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared_symbols():
    text = open(os.path.join(ROOT, "include", "tidegbm_b200.h")).read()
    return sorted(set(re.findall(r"TGB_API[^;(]*?\b(tgb_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(native):
    L = C.CDLL(native.LIB_PATH)
    names = _declared_symbols()
    assert len(names) >= 20
    for name in names:
        assert hasattr(L, name), name


def test_no_internal_symbols_exported(native):
    out = os.popen(f"nm -D --defined-only {native.LIB_PATH}").read()
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    assert exported == set(_declared_symbols())


@pytest.mark.parametrize("m,keep,seed", [(1, 1, 0), (10, 3, 1), (1000, 1000, 2), (65535, 100, 3), (65536, 100, 4),
                                         (65537, 65537, 5), (300000, 26214, 6), (1_000_000, 100_000, 7),
                                         (3_000_000, 262_144, 8), (100_000, 0, 9), (2_000_000, 1, 10)])
def test_shuffled_prefix_equals_std_shuffle(native, oracle, m, keep, seed):
    got = np.zeros(keep, np.int32)
    native.check(native.lib().tgb_shuffled_prefix(m, keep, seed, got.ctypes.data_as(C.c_void_p)))
    ref = np.zeros(keep, np.int32)
    L = oracle.oracle_lib()
    L.orc_shuffle_prefix.argtypes = [C.c_int64, C.c_int64, C.c_uint32, C.c_void_p]
    L.orc_shuffle_prefix(m, keep, seed, ref.ctypes.data_as(C.c_void_p))
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("m,keep,seed,n_shuffles", [(1000, 100, 1, 3), (65536, 1000, 2, 4), (300000, 30000, 3, 4),
                                                    (2_000_000, 200_000, 4, 3), (8_000_000, 1_000_000, 5, 2)])
def test_shuffle_sequence_equals_std_shuffle(native, oracle, m, keep, seed, n_shuffles):
    """The GOSS draw sequence: the generator walked between trees without positions (the
    fit's producer) must land exactly where std::shuffle leaves it, tree after tree."""
    got = np.zeros(n_shuffles * keep, np.int32)
    native.check(native.lib().tgb_shuffle_sequence(m, keep, seed, n_shuffles, got.ctypes.data_as(C.c_void_p)))
    ref = np.zeros(n_shuffles * keep, np.int32)
    L = oracle.oracle_lib()
    L.orc_shuffle_sequence.argtypes = [C.c_int64, C.c_int64, C.c_uint32, C.c_int, C.c_void_p]
    L.orc_shuffle_sequence(m, keep, seed, n_shuffles, ref.ctypes.data_as(C.c_void_p))
    assert np.array_equal(got, ref)


@pytest.mark.parametrize("dtype,bin_sample", [(np.float32, 3000), (np.float64, 0), (np.float64, 70000)])
def test_host_binner_matches_oracle(native, oracle, dtype, bin_sample):
    rng = np.random.default_rng(11)
    n, nf = 80000, 12
    X = rng.standard_normal((n, nf)).astype(dtype)
    X[:, 1] = np.round(X[:, 1])  # few uniques: edges = values
    X[:, 2] = np.exp(X[:, 2] * 2)
    X[:, 4] = np.nan  # all missing -> edges {0.0}
    X[rng.random((n, nf)) < 0.02] = np.nan
    e1 = np.zeros(nf * 256)
    n1 = np.zeros(nf, np.int32)
    nb1 = native.lib().tgb_binner_fit(X.ctypes.data_as(C.c_void_p), 0 if dtype == np.float32 else 1, n, nf, 255,
                                      bin_sample, 42, e1.ctypes.data_as(C.c_void_p), n1.ctypes.data_as(C.c_void_p))
    assert nb1 > 0, native.lib().tgb_last_error()
    e2 = np.zeros(nf * 256)
    n2 = np.zeros(nf, np.int32)
    nbc = np.zeros(nf, np.int32)
    nb2 = oracle.oracle_lib().orc_binner_fit(np.ascontiguousarray(X, dtype=np.float64), n, nf, 255, bin_sample, 42,
                                             e2, n2, nbc)
    assert nb1 == nb2
    assert np.array_equal(n1, n2)
    assert np.array_equal(e1, e2)


@pytest.mark.parametrize("dtype,max_bin,bin_sample", [(np.float64, 255, 0), (np.float64, 64, 500),
                                                     (np.float32, 255, 500), (np.float32, 8, 0)])
def test_host_binner_edge_columns_match_oracle(native, oracle, dtype, max_bin, bin_sample):
    """tgb_binner_fit on edge columns (tests/edge_columns.py): edges bit for bit, signed zeros
    included (the kept values reach std::sort in their shuffled order, as in the reference)."""
    from edge_columns import edge_columns

    with np.errstate(over="ignore"):  # float32: the 1e300 values become infinities, 1e-300 signed zeros
        X = np.ascontiguousarray(edge_columns().astype(dtype))
    n, nf = X.shape
    e1 = np.zeros(nf * 256)
    n1 = np.zeros(nf, np.int32)
    nb1 = native.lib().tgb_binner_fit(X.ctypes.data_as(C.c_void_p), 0 if dtype == np.float32 else 1, n, nf,
                                      max_bin, bin_sample, 7, e1.ctypes.data_as(C.c_void_p),
                                      n1.ctypes.data_as(C.c_void_p))
    assert nb1 > 0, native.lib().tgb_last_error()
    e2 = np.zeros(nf * 256)
    n2 = np.zeros(nf, np.int32)
    nbc = np.zeros(nf, np.int32)
    nb2 = oracle.oracle_lib().orc_binner_fit(np.ascontiguousarray(X, dtype=np.float64), n, nf, max_bin, bin_sample,
                                             7, e2, n2, nbc)
    assert nb1 == nb2
    assert np.array_equal(n1, n2)
    assert np.array_equal(e1.view(np.uint64), e2.view(np.uint64))


def test_host_binner_matches_reference_fixture(native):
    """tgb_binner_fit (the host part of binning) against the reference's own edges."""
    import os

    d = np.load(os.path.join(ROOT, "tests", "golden", "binner.npz"))
    X = np.ascontiguousarray(d["X"])
    n, nf = X.shape
    e = np.zeros(nf * 256)
    ne = np.zeros(nf, np.int32)
    nb = native.lib().tgb_binner_fit(X.ctypes.data_as(C.c_void_p), 1, n, nf, int(d["max_bin"]), int(d["bin_sample"]),
                                     int(d["seed"]), e.ctypes.data_as(C.c_void_p), ne.ctypes.data_as(C.c_void_p))
    assert nb == int(d["max_bins"])
    assert np.array_equal(ne, d["n_edges"])
    assert np.array_equal(e.reshape(nf, 256), d["edges"])


def _cat_X(seed, n=20000, nf=6):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((n, nf))
    X[:, 0] = rng.integers(0, 12, n)                                    # few categories
    X[:, 2] = rng.integers(0, 400, n)                                   # more than max_bin - 1: the most frequent kept
    X[:, 3] = np.where(rng.random(n) < 0.01, rng.integers(100, 160, n), rng.integers(0, 5, n))  # rare ones dropped
    X[:, 4] = rng.integers(0, 10**7, n)                                 # nearly all values seen once: all rare
    X[rng.random((n, nf)) < 0.03] = np.nan
    return X, np.array([1, 0, 1, 1, 1, 0], np.int32)


@pytest.mark.parametrize("dtype,max_bin,min_count,bin_sample", [(np.float64, 255, 5, 3000), (np.float32, 255, 5, 0),
                                                                (np.float64, 64, 2, 5000), (np.float64, 255, 20, 0)])
def test_host_categorical_binner_matches_oracle(native, oracle, dtype, max_bin, min_count, bin_sample):
    """tgb_binner_fit_cat's vocabularies and numeric edges against the oracle's
    Binner::fit with categorical features, bit for bit."""
    X, is_cat = _cat_X(4)
    X = X.astype(dtype)
    n, nf = X.shape
    e1 = np.zeros(nf * 256)
    n1 = np.zeros(nf, np.int32)
    nb1 = native.lib().tgb_binner_fit_cat(np.ascontiguousarray(X).ctypes.data_as(C.c_void_p),
                                          0 if dtype == np.float32 else 1, n, nf, is_cat.ctypes.data_as(C.c_void_p),
                                          max_bin, min_count, bin_sample, 7, e1.ctypes.data_as(C.c_void_p),
                                          n1.ctypes.data_as(C.c_void_p))
    assert nb1 > 0, native.lib().tgb_last_error()
    e2 = np.zeros(nf * 256)
    n2 = np.zeros(nf, np.int32)
    L = oracle.oracle_lib()
    L.orc_binner_fit_cat.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_uint32,
                                     C.c_void_p, C.c_void_p, C.c_void_p]
    Xd = np.ascontiguousarray(X, dtype=np.float64)
    nb2 = L.orc_binner_fit_cat(Xd.ctypes.data_as(C.c_void_p), n, nf, is_cat.ctypes.data_as(C.c_void_p), max_bin,
                               min_count, bin_sample, 7, e2.ctypes.data_as(C.c_void_p), n2.ctypes.data_as(C.c_void_p),
                               None)
    assert nb1 == nb2
    assert np.array_equal(n1, n2)
    assert np.array_equal(e1, e2)
    assert n1[2] == max_bin - 1  # the vocabulary cut to the most frequent values
    if min_count >= 5:
        assert n1[4] == 1  # no value is frequent enough: the most frequent one alone
