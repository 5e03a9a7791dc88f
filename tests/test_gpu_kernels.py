"""Kernel-level parity: each C-ABI kernel entry point against the oracle restatement
(oracle/oracle.cpp) on the same seeded inputs.

Tolerances: bin codes, counts, partitions and split choices bit-exact; fixed-point
histogram sums within 1e-9 of the FP64 oracle relative to sum(|g|) of the bin
(demeaned gradients make plain relative error meaningless near zero); pairwise
gradients within 1e-12 relative to sum of |pair terms|.
"""
import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def dptr(t):
    return C.c_void_p(t.data_ptr())


def ceil_f32(e):
    f = e.astype(np.float32)
    lower = f.astype(np.float64) < e
    f[lower] = np.nextafter(f[lower], np.float32(np.inf))
    return f


def _binned(oracle, n=20000, nf=40, nan_frac=0.03, seed=0, dtype=np.float32, max_bin=255, bin_sample=5000):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((n, nf)).astype(dtype)
    X[:, 3] = np.round(X[:, 3] * 2)  # few distinct values
    X[:, 5] = np.exp(X[:, 5])
    X[rng.random((n, nf)) < nan_frac] = np.nan
    L = oracle.oracle_lib()
    Xd = np.ascontiguousarray(X, dtype=np.float64)
    edges = np.zeros(nf * 256)
    ne = np.zeros(nf, np.int32)
    nbc = np.zeros(nf, np.int32)
    n_bins = L.orc_binner_fit(Xd, n, nf, max_bin, bin_sample, 7, edges, ne, nbc)
    codes = np.zeros(n * nf, np.uint8)
    L.orc_bin_transform(Xd, n, nf, edges, ne, codes, nf)
    return X, edges.reshape(nf, 256), ne, n_bins, codes.reshape(n, nf)


@pytest.mark.parametrize("dtype", [np.float32, np.float64])
def test_bin_transform_bit_exact(oracle, native, dtype):
    X, edges, ne, n_bins, codes_ref = _binned(oracle, dtype=dtype)
    n, nf = X.shape
    stride = (nf + 15) // 16 * 16
    E = np.full((nf, 256), np.inf)
    for f in range(nf):
        E[f, : ne[f]] = edges[f, : ne[f]]
    if dtype == np.float32:
        E32 = np.full((nf, 256), np.inf, dtype=np.float32)
        for f in range(nf):
            E32[f, : ne[f]] = ceil_f32(edges[f, : ne[f]])
        Ed = torch.from_numpy(E32).cuda()
        Xt = torch.from_numpy(X).cuda()
        dt = 0
    else:
        Ed = torch.from_numpy(E).cuda()
        Xt = torch.from_numpy(np.ascontiguousarray(X, dtype=np.float64)).cuda()
        dt = 1
    net = torch.from_numpy(ne).cuda()
    codes = torch.full((n, stride), 77, dtype=torch.uint8, device="cuda")
    native.check(native.lib().tgb_bin_transform(dptr(Xt), dt, n, nf, dptr(Ed), dptr(net), dptr(codes), stride, None))
    torch.cuda.synchronize()
    got = codes.cpu().numpy()
    assert np.array_equal(got[:, :nf], codes_ref)
    assert (got[:, nf:] == 0).all()


def test_bin_transform_infinities(oracle, native):
    X = np.array([[np.inf], [-np.inf], [np.nan], [0.0], [1e30]], dtype=np.float32)
    X = np.repeat(X, 16, axis=1)
    edges = np.tile(np.array([-1.0, 0.0, 1.0]), (16, 1))
    ne = np.full(16, 3, np.int32)
    E = np.full((16, 256), np.inf, dtype=np.float32)
    E[:, :3] = edges
    codes = torch.zeros((5, 16), dtype=torch.uint8, device="cuda")
    Xt, Et, nt = torch.from_numpy(X).cuda(), torch.from_numpy(E).cuda(), torch.from_numpy(ne).cuda()
    native.check(native.lib().tgb_bin_transform(dptr(Xt), 0, 5, 16, dptr(Et), dptr(nt), dptr(codes), 16, None))
    got = codes.cpu().numpy()[:, 0]
    # upper_bound over {-1, 0, 1} + 1; NaN -> 0 (cpp/src/binning.cpp:112-119)
    assert got.tolist() == [4, 1, 0, 3, 4]


def _hist_case(seed, n=30000, nf=37, n_rows=12345):
    rng = np.random.default_rng(seed)
    codes = rng.integers(0, 256, size=(n, nf), dtype=np.uint8)
    codes[:, 2] = rng.integers(0, 3, size=n)  # heavy collisions
    stride = (nf + 15) // 16 * 16
    padded = np.zeros((n, stride), np.uint8)
    padded[:, :nf] = codes
    rows = np.sort(rng.choice(n, n_rows, replace=False)).astype(np.int32)
    g = rng.standard_normal(n) * 3
    h = rng.random(n) * 2 + 1e-6
    return padded, stride, codes, rows, g, h


def _shift(v, cnt):
    m = np.max(np.abs(v))
    return 61 - (int(np.floor(np.log2(m))) + 1) - int(np.ceil(np.log2(cnt)))


@pytest.mark.parametrize("seed", [0, 1])
def test_hist_build_matches_fp64(oracle, native, seed):
    padded, stride, codes, rows, g, h = _hist_case(seed)
    n, nf = codes.shape
    gs, hs = _shift(g[rows], rows.size), _shift(h[rows], rows.size)
    G = torch.zeros((nf, 256), dtype=torch.int64, device="cuda")
    H = torch.zeros_like(G)
    Cn = torch.zeros((nf, 256), dtype=torch.int32, device="cuda")
    ct, rt = torch.from_numpy(padded).cuda(), torch.from_numpy(rows).cuda()
    gt, ht = torch.from_numpy(g).cuda(), torch.from_numpy(h).cuda()
    native.check(native.lib().tgb_hist_build(dptr(ct), stride, nf, dptr(rt), rows.size, dptr(gt), dptr(ht), gs, hs,
                                             dptr(G), dptr(H), dptr(Cn), None))
    torch.cuda.synchronize()
    ref = np.zeros(nf * 256 * 3)
    oracle.oracle_lib().orc_build_hist(np.ascontiguousarray(codes), nf, nf, rows, rows.size, g, h, 256, ref)
    ref = ref.reshape(nf, 256, 3)
    Gd = G.cpu().numpy() * 2.0 ** -gs
    Hd = H.cpu().numpy() * 2.0 ** -hs
    assert np.array_equal(Cn.cpu().numpy(), ref[:, :, 2].astype(np.int32))
    absg = np.zeros((nf, 256))
    for f in range(nf):
        np.add.at(absg[f], codes[rows, f], np.abs(g[rows]))
    assert np.all(np.abs(Gd - ref[:, :, 0]) <= 1e-9 * absg + 1e-300)
    assert np.allclose(Hd, ref[:, :, 1], rtol=1e-9, atol=0)
    # determinism: a second launch gives identical integers
    G2 = torch.zeros_like(G)
    H2 = torch.zeros_like(H)
    C2 = torch.zeros_like(Cn)
    native.check(native.lib().tgb_hist_build(dptr(ct), stride, nf, dptr(rt), rows.size, dptr(gt), dptr(ht), gs, hs,
                                             dptr(G2), dptr(H2), dptr(C2), None))
    assert torch.equal(G, G2) and torch.equal(H, H2) and torch.equal(Cn, C2)


def test_hist_empty_rows(native):
    G = torch.zeros((16, 256), dtype=torch.int64, device="cuda")
    H = torch.zeros_like(G)
    Cn = torch.zeros((16, 256), dtype=torch.int32, device="cuda")
    codes = torch.zeros((4, 16), dtype=torch.uint8, device="cuda")
    rows = torch.zeros(1, dtype=torch.int32, device="cuda")
    g = torch.zeros(4, dtype=torch.float64, device="cuda")
    native.check(native.lib().tgb_hist_build(dptr(codes), 16, 16, dptr(rows), 0, dptr(g), dptr(g), 0, 0, dptr(G),
                                             dptr(H), dptr(Cn), None))
    assert int(Cn.sum()) == 0


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_split_scan_matches_oracle(oracle, native, seed):
    padded, stride, codes, rows, g, h = _hist_case(seed, n=20000, nf=24, n_rows=9000)
    n, nf = codes.shape
    n_bins = 255
    codes = np.minimum(codes, n_bins - 1)
    padded[:, :nf] = codes
    gs, hs = _shift(g[rows], rows.size), _shift(h[rows], rows.size)
    G = torch.zeros((nf, 256), dtype=torch.int64, device="cuda")
    H = torch.zeros_like(G)
    Cn = torch.zeros((nf, 256), dtype=torch.int32, device="cuda")
    ct, rt = torch.from_numpy(padded).cuda(), torch.from_numpy(rows).cuda()
    gt, ht = torch.from_numpy(g).cuda(), torch.from_numpy(h).cuda()
    L = native.lib()
    native.check(L.tgb_hist_build(dptr(ct), stride, nf, dptr(rt), rows.size, dptr(gt), dptr(ht), gs, hs, dptr(G),
                                  dptr(H), dptr(Cn), None))
    gain = torch.zeros(nf, dtype=torch.float64, device="cuda")
    thr = torch.zeros(nf, dtype=torch.int32, device="cuda")
    ml = torch.zeros(nf, dtype=torch.int32, device="cuda")
    native.check(L.tgb_split_scan(dptr(G), dptr(H), dptr(Cn), nf, n_bins, gs, hs, 1.0, 0.0, 20, 1e-3, dptr(gain),
                                  dptr(thr), dptr(ml), None))
    torch.cuda.synchronize()
    # oracle scan of the device histogram (identical inputs -> identical decisions)
    hist = np.zeros((nf, n_bins, 3))
    hist[:, :, 0] = (G.cpu().numpy() * 2.0 ** -gs)[:, :n_bins]
    hist[:, :, 1] = (H.cpu().numpy() * 2.0 ** -hs)[:, :n_bins]
    hist[:, :, 2] = Cn.cpu().numpy()[:, :n_bins]
    O = oracle.oracle_lib()
    O.orc_best_numeric.restype = None
    import ctypes

    class S(ctypes.Structure):
        _fields_ = [("gain", ctypes.c_double), ("feature", ctypes.c_int), ("threshold_bin", ctypes.c_int),
                    ("missing_go_left", ctypes.c_int)]

    O.orc_best_numeric.restype = S
    O.orc_best_numeric.argtypes = [np.ctypeslib.ndpointer(np.float64, flags="C"), ctypes.c_int, ctypes.c_int,
                                   ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_double]
    flat = np.ascontiguousarray(hist.reshape(-1))
    gd, td, md = gain.cpu().numpy(), thr.cpu().numpy(), ml.cpu().numpy()
    for f in range(nf):
        s = O.orc_best_numeric(flat, n_bins, f, 1.0, 0.0, 20, 1e-3)
        assert td[f] == s.threshold_bin and md[f] == s.missing_go_left, f
        if s.threshold_bin >= 0:
            assert abs(gd[f] - s.gain) <= 1e-12 * max(1.0, abs(s.gain))


@pytest.mark.parametrize("n_rows", [0, 1, 2047, 2048, 2049, 100000])
def test_partition_stable(native, n_rows):
    rng = np.random.default_rng(n_rows)
    n, nf = 120000, 20
    stride = 32
    codes = np.zeros((n, stride), np.uint8)
    codes[:, :nf] = rng.integers(0, 256, size=(n, nf))
    rows = np.sort(rng.choice(n, n_rows, replace=False)).astype(np.int32) if n_rows else np.zeros(1, np.int32)
    feat, thr, mlft = 7, 100, 1
    L = native.lib()
    ct = torch.from_numpy(codes).cuda()
    rt = torch.from_numpy(rows).cuda()
    out = torch.full((max(1, n_rows),), -1, dtype=torch.int32, device="cuda")
    nl = torch.zeros(1, dtype=torch.int32, device="cuda")
    wsb = L.tgb_partition_workspace_bytes(n_rows)
    ws = torch.zeros(wsb, dtype=torch.uint8, device="cuda")
    native.check(L.tgb_partition(dptr(ct), stride, dptr(rt), n_rows, feat, thr, mlft, dptr(out), dptr(nl), dptr(ws),
                                 wsb, None))
    torch.cuda.synchronize()
    r = rows[:n_rows]
    b = codes[r, feat].astype(int)
    left = np.where(b == 0, mlft == 1, b <= thr)
    expect = np.concatenate([r[left], r[~left]])
    assert int(nl.item()) == int(left.sum())
    assert np.array_equal(out.cpu().numpy()[:n_rows], expect)


def test_grad_mse_bit_exact(oracle, native):
    rng = np.random.default_rng(3)
    n = 100001
    y, p = rng.standard_normal(n), rng.standard_normal(n)
    g0, h0 = np.zeros(n), np.zeros(n)
    oracle.oracle_lib().orc_grad_hess(0, y, p, None, n, g0, h0)
    yt, pt = torch.from_numpy(y).cuda(), torch.from_numpy(p).cuda()
    gt, ht = torch.zeros_like(yt), torch.zeros_like(yt)
    native.check(native.lib().tgb_grad_mse(dptr(yt), dptr(pt), n, dptr(gt), dptr(ht), None))
    assert np.array_equal(gt.cpu().numpy(), g0) and np.array_equal(ht.cpu().numpy(), h0)


def test_grad_pairwise_matches_oracle(oracle, native):
    rng = np.random.default_rng(4)
    sizes = np.concatenate([[1, 2, 3, 48, 49, 50, 800, 97], rng.integers(50, 801, size=40)])
    ts = np.repeat(np.arange(sizes.size, dtype=np.int64), sizes)
    n = ts.size
    y = np.round(rng.standard_normal(n), 2)  # ties in y are skipped by the objective
    p = rng.standard_normal(n) * 0.1
    g0, h0 = np.zeros(n), np.zeros(n)
    O = oracle.oracle_lib()
    O.orc_grad_hess(5, y, p, ts.ctypes.data_as(C.c_void_p), n, g0, h0)
    starts = np.r_[0, np.cumsum(sizes)[:-1]].astype(np.int32)
    yt, pt = torch.from_numpy(y).cuda(), torch.from_numpy(p).cuda()
    st, lt = torch.from_numpy(starts).cuda(), torch.from_numpy(sizes.astype(np.int32)).cuda()
    gt, ht = torch.zeros_like(yt), torch.zeros_like(yt)
    native.check(native.lib().tgb_grad_pairwise(dptr(yt), dptr(pt), dptr(st), dptr(lt), None, sizes.size, n, dptr(gt),
                                                dptr(ht), None))
    g1, h1 = gt.cpu().numpy(), ht.cpu().numpy()
    scale = np.abs(g0) + np.abs(h0) + 1e-3
    assert np.all(np.abs(g1 - g0) <= 1e-12 * scale)
    assert np.all(np.abs(h1 - h0) <= 1e-12 * scale)


@pytest.mark.parametrize("seed", [0, 1])
def test_build_hist_gpu_seam_matches_oracle(oracle, native, seed):
    """tgb_build_hist_gpu, the literal drop-in for the reference's build_hist_gpu seam
    (cpp/include/tidegbm/histogram.hpp:57-58): host row-major uint16 codes, host idx/g/h,
    the interleaved FP64 {g, h, c} Hist out.  Against the oracle's build_hist_col: counts
    exact, G within 1e-9 of the per-bin sum of |g| (demeaned gradients make bin totals
    near zero, so the bound is scaled by sum |g|), H within 1e-9 relative.  Called twice,
    with a different row list the second time, on one booster: the resident code matrix is
    reused and the result follows the new rows."""
    _, _, codes, rows, g, h = _hist_case(seed)
    n, nf = codes.shape
    n_bins = 256
    xb = np.ascontiguousarray(codes.astype(np.uint16))
    b = native.Booster(device=0)
    L = native.lib()
    rng = np.random.default_rng(seed + 10)
    for idx in (rows, np.sort(rng.choice(n, 777, replace=False)).astype(np.int32)):
        out = np.zeros(nf * n_bins * 3)
        native.check(L.tgb_build_hist_gpu(b._h, xb.ctypes.data_as(C.c_void_p), nf, idx.ctypes.data_as(C.c_void_p),
                                          idx.size, g.ctypes.data_as(C.c_void_p), h.ctypes.data_as(C.c_void_p),
                                          n_bins, n, out.ctypes.data_as(C.c_void_p)))
        ref = np.zeros(nf * 256 * 3)
        oracle.oracle_lib().orc_build_hist(np.ascontiguousarray(codes), nf, nf, idx, idx.size, g, h, 256, ref)
        out, ref = out.reshape(nf, n_bins, 3), ref.reshape(nf, 256, 3)
        assert np.array_equal(out[:, :, 2], ref[:, :, 2])
        absg = np.zeros((nf, 256))
        for f in range(nf):
            np.add.at(absg[f], codes[idx, f], np.abs(g[idx]))
        assert np.all(np.abs(out[:, :, 0] - ref[:, :, 0]) <= 1e-9 * absg + 1e-300)
        assert np.allclose(out[:, :, 1], ref[:, :, 1], rtol=1e-9, atol=0)


@pytest.mark.parametrize("bits,bound", [(0, 1e-9), (16, 1e-3), (8, 3e-2)])
@pytest.mark.parametrize("var_h", [False, True])
def test_quantized_histogram_error_vs_fp64(oracle, native, bits, bound, var_h):
    """tgb_hist_build_quantized (the fit's payload and wave histogram kernels) against the
    oracle's FP64 build_hist_col: counts exact; max over bins of |G - G_fp64| / sum |g|
    within the mode's bound (exact: 1e-9; int16: 1e-3; int8: 3e-2), and H likewise against
    sum h.  Stochastic rounding keeps the error unbiased, so it shrinks like sqrt(rows)."""
    padded, stride, codes, rows, g, h = _hist_case(3, n=60000, nf=45, n_rows=40000)
    n, nf = codes.shape
    G = torch.zeros((nf, 256), dtype=torch.int64, device="cuda")
    H = torch.zeros_like(G)
    Cn = torch.zeros((nf, 256), dtype=torch.int32, device="cuda")
    ct, rt = torch.from_numpy(padded).cuda(), torch.from_numpy(rows).cuda()
    gt, ht = torch.from_numpy(g).cuda(), torch.from_numpy(h).cuda()
    sc = np.zeros(2)
    native.check(native.lib().tgb_hist_build_quantized(dptr(ct), stride, nf, dptr(rt), rows.size, dptr(gt),
                                                       dptr(ht) if var_h else None, bits, 12345, dptr(G), dptr(H),
                                                       dptr(Cn), sc.ctypes.data_as(C.c_void_p), None))
    torch.cuda.synchronize()
    hh = h if var_h else np.ones(n)
    ref = np.zeros(nf * 256 * 3)
    oracle.oracle_lib().orc_build_hist(np.ascontiguousarray(codes), nf, nf, rows, rows.size, g, hh, 256, ref)
    ref = ref.reshape(nf, 256, 3)
    assert np.array_equal(Cn.cpu().numpy(), ref[:, :, 2].astype(np.int32))
    Gd = G.cpu().numpy() * sc[0]
    Hd = H.cpu().numpy() * sc[1]
    assert np.max(np.abs(Gd - ref[:, :, 0])) <= bound * np.abs(g[rows]).sum()
    assert np.max(np.abs(Hd - ref[:, :, 1])) <= bound * np.abs(hh[rows]).sum()
