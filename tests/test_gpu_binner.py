"""Device quantile binning (tgb_binner_fit_device) against the oracle's Binner::fit
and the reference's own edges (tests/golden/binner.npz).  Bit-exact edges.

Cases follow the branches of Binner::fit / quantile_edges (cpp/src/binning.cpp:14-102):
  more non-NaN values than bin_sample (the shuffled sample; both the libstdc++
  pairs path below 2^16 values and the one-draw path above), at most bin_sample
  (every value), a column with no values (edges {0.0}), few distinct values (the
  values are the edges), heavy duplicates, and bin_sample <= 0 (no sampling).
"""
import ctypes as C
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _device_edges(native, X, max_bin, bin_sample, seed):
    n, nf = X.shape
    Xt = torch.from_numpy(np.ascontiguousarray(X)).cuda()
    torch.cuda.synchronize()
    e = np.zeros(nf * 256)
    ne = np.zeros(nf, np.int32)
    nb = native.lib().tgb_binner_fit_device(C.c_void_p(Xt.data_ptr()), 0 if X.dtype == np.float32 else 1, n, nf,
                                            max_bin, bin_sample, seed, e.ctypes.data_as(C.c_void_p),
                                            ne.ctypes.data_as(C.c_void_p), None)
    torch.cuda.synchronize()
    del Xt
    assert nb > 0, native.lib().tgb_last_error()
    return nb, e.reshape(nf, 256), ne


def _oracle_edges(oracle, X, max_bin, bin_sample, seed):
    n, nf = X.shape
    e = np.zeros(nf * 256)
    ne = np.zeros(nf, np.int32)
    nbc = np.zeros(nf, np.int32)
    nb = oracle.oracle_lib().orc_binner_fit(np.ascontiguousarray(X, dtype=np.float64), n, nf, max_bin, bin_sample,
                                            seed, e, ne, nbc)
    return nb, e.reshape(nf, 256), ne


def _panel(n, nf, seed, dtype):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((n, nf)).astype(dtype)
    X[:, 1] = np.round(X[:, 1])            # few distinct values: edges = the values
    X[:, 2] = np.exp(X[:, 2] * 2)          # skewed
    if nf > 4:
        X[:, 4] = np.nan                   # no values: edges {0.0}
    if nf > 5:
        X[:, 5] = np.round(X[:, 5] * 40)   # ~300 distinct values, heavy duplicates
    if nf > 6:
        X[: n // 2, 6] = np.nan            # half missing: fewer values than bin_sample for small n
    X[rng.random((n, nf)) < 0.02] = np.nan
    return X


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
@pytest.mark.parametrize("n,bin_sample", [(80000, 20000), (30000, 12000), (5000, 262144), (120000, 0),
                                          (300000, 262144)])
def test_device_binner_matches_oracle(oracle, native, dtype, n, bin_sample):
    X = _panel(n, 12, 11 + n % 7, dtype)
    nb1, e1, n1 = _device_edges(native, X, 255, bin_sample, 42)
    nb2, e2, n2 = _oracle_edges(oracle, X, 255, bin_sample, 42)
    assert nb1 == nb2
    assert np.array_equal(n1, n2)
    assert np.array_equal(e1, e2)


@pytest.mark.parametrize("max_bin", [8, 64, 256])
def test_device_binner_max_bin(oracle, native, max_bin):
    X = _panel(70000, 7, 3, np.float32)
    nb1, e1, n1 = _device_edges(native, X, max_bin, 50000, 5)
    nb2, e2, n2 = _oracle_edges(oracle, X, max_bin, 50000, 5)
    assert nb1 == nb2
    assert np.array_equal(n1, n2)
    assert np.array_equal(e1, e2)


def test_device_binner_matches_reference_fixture(native):
    d = np.load(os.path.join(ROOT, "tests", "golden", "binner.npz"))
    X = np.ascontiguousarray(d["X"])
    nb, e, ne = _device_edges(native, X, int(d["max_bin"]), int(d["bin_sample"]), int(d["seed"]))
    assert nb == int(d["max_bins"])
    assert np.array_equal(ne, d["n_edges"])
    assert np.array_equal(e, d["edges"])


def test_device_binner_wide_features(oracle, native):
    """More features than one CTA's 128 threads (grid y > 1) and a ragged row count."""
    X = _panel(9001, 300, 8, np.float32)
    nb1, e1, n1 = _device_edges(native, X, 255, 4000, 77)
    nb2, e2, n2 = _oracle_edges(oracle, X, 255, 4000, 77)
    assert nb1 == nb2
    assert np.array_equal(n1, n2)
    assert np.array_equal(e1, e2)


@pytest.mark.parametrize("m,keep,seed", [(1, 1, 0), (10, 3, 1), (65536, 100, 4), (65537, 65537, 5),
                                         (300000, 26214, 6), (1_000_000, 100_000, 7), (3_000_000, 262_144, 8),
                                         (9_900_000, 262_144, 2654435761 * 5 % 2**32), (2_000_000, 1, 10),
                                         (500_000, 500_000, 11), (700_000, 699_999, 12), (65_536, 2, 13)])
def test_device_shuffle_tail_equals_std_shuffle(native, oracle, m, keep, seed):
    """Draws on the device (generator, then the swaps inside the prefix resolved in parallel):
    the same prefix as libstdc++'s std::shuffle.  keep == m and m near 10M included; ranges
    below 2^16 take the host's two-draws path."""
    out = torch.full((keep,), -1, dtype=torch.int32, device="cuda")
    native.check(native.lib().tgb_shuffled_prefix_device(m, keep, seed, C.c_void_p(out.data_ptr()), None))
    ref = np.zeros(keep, np.int32)
    L = oracle.oracle_lib()
    L.orc_shuffle_prefix.argtypes = [C.c_int64, C.c_int64, C.c_uint32, C.c_void_p]
    L.orc_shuffle_prefix(m, keep, seed, ref.ctypes.data_as(C.c_void_p))
    assert np.array_equal(out.cpu().numpy(), ref)


def _ceil_f32(e):
    f = e.astype(np.float32)
    with np.errstate(invalid="ignore"):
        lower = f.astype(np.float64) < e
    f[lower] = np.nextafter(f[lower], np.float32(np.inf))
    return f


@pytest.mark.parametrize("dtype,max_bin,bin_sample,n", [(np.float64, 255, 0, 6000), (np.float64, 64, 500, 6000),
                                                        (np.float32, 255, 500, 6000), (np.float32, 8, 0, 6000),
                                                        (np.float64, 255, 20000, 90000),
                                                        (np.float32, 64, 30000, 90000)])
def test_device_binner_edge_columns_match_oracle(oracle, native, dtype, max_bin, bin_sample, n):
    """The device binner and transform on edge columns (tests/edge_columns.py): all
    missing, constant, 254 / 255 distinct, infinities, signed zeros, extreme magnitudes,
    heavy ties, and +inf with interpolated edges (NaN edges in the reference).  Edges bit
    for bit (the sign of a zero edge and NaN edges included: features whose edges depend on
    std::sort's order of equal values are recomputed in the reference's order), then codes
    bit for bit (the transform runs upper_bound's own bisection, so NaN edges bin as in the
    reference).  90,000 rows take the device shuffle path."""
    from edge_columns import edge_columns

    with np.errstate(over="ignore"):
        X = np.ascontiguousarray(edge_columns(n=n).astype(dtype))
    nrow, nf = X.shape
    nb1, e1, n1 = _device_edges(native, X, max_bin, bin_sample, 7)
    nb2, e2, n2 = _oracle_edges(oracle, X, max_bin, bin_sample, 7)
    assert nb1 == nb2
    assert np.array_equal(n1, n2)
    assert np.array_equal(e1.view(np.uint64), e2.view(np.uint64))
    # codes through the device transform against the oracle's transform
    L = oracle.oracle_lib()
    Xd = np.ascontiguousarray(X, dtype=np.float64)
    ref = np.zeros(nrow * nf, np.uint8)
    L.orc_bin_transform(Xd, nrow, nf, np.ascontiguousarray(e2.reshape(-1)), n2, ref, nf)
    stride = (nf + 15) // 16 * 16
    if dtype == np.float32:
        E = np.full((nf, 256), np.inf, dtype=np.float32)
        for f in range(nf):
            E[f, : n1[f]] = _ceil_f32(e1[f, : n1[f]])
    else:
        E = np.full((nf, 256), np.inf)
        for f in range(nf):
            E[f, : n1[f]] = e1[f, : n1[f]]
    Xt, Et, nt = torch.from_numpy(X).cuda(), torch.from_numpy(E).cuda(), torch.from_numpy(n1).cuda()
    codes = torch.full((nrow, stride), 77, dtype=torch.uint8, device="cuda")
    native.check(native.lib().tgb_bin_transform(C.c_void_p(Xt.data_ptr()), 0 if dtype == np.float32 else 1, nrow, nf,
                                                C.c_void_p(Et.data_ptr()), C.c_void_p(nt.data_ptr()),
                                                C.c_void_p(codes.data_ptr()), stride, None))
    torch.cuda.synchronize()
    assert np.array_equal(codes.cpu().numpy()[:, :nf], ref.reshape(nrow, nf))
