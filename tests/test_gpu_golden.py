"""The CUDA path against golden fixtures produced by the reference core itself
(tests/golden/make_golden.py).

Bar: bin codes and histogram counts bit-exact; histogram sums within 1e-9 of the
reference's FP64 sums relative to sum(|g|) of the bin; split choices identical; pairwise
gradients within 1e-12 relative to |g| + |h|; fitted tree structure identical, node and
leaf values, TORB prefix values, losses and predictions within 1e-9 absolute.
"""
import ctypes as C
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return np.load(os.path.join(GOLD, name), allow_pickle=False)


def _p(t):
    return C.c_void_p(t.data_ptr())


def test_bin_transform_matches_reference(native):
    d = load("binner.npz")
    X = np.ascontiguousarray(d["X"])
    n, nf = X.shape
    stride = (nf + 15) // 16 * 16
    E = np.full((nf, 256), np.inf)
    for f in range(nf):
        E[f, : d["n_edges"][f]] = d["edges"][f, : d["n_edges"][f]]
    codes = torch.zeros((n, stride), dtype=torch.uint8, device="cuda")
    Xt, Et = torch.from_numpy(X).cuda(), torch.from_numpy(E).cuda()
    nt = torch.from_numpy(d["n_edges"].astype(np.int32)).cuda()
    native.check(native.lib().tgb_bin_transform(_p(Xt), 1, n, nf, _p(Et), _p(nt), _p(codes), stride, None))
    assert np.array_equal(codes.cpu().numpy()[:, :nf], d["codes"].astype(np.uint8))


def test_histogram_and_split_match_reference(native):
    d = load("hist.npz")
    s = load("split.npz")
    codes = d["codes"].astype(np.uint8)
    n, nf = codes.shape
    stride = 16
    padded = np.zeros((n, stride), np.uint8)
    padded[:, :nf] = codes
    idx, g, h = d["idx"], d["g"], d["h"]
    gs = 61 - (int(np.floor(np.log2(np.abs(g[idx]).max()))) + 1) - int(np.ceil(np.log2(idx.size)))
    hs = 61 - (int(np.floor(np.log2(np.abs(h[idx]).max()))) + 1) - int(np.ceil(np.log2(idx.size)))
    G = torch.zeros((nf, 256), dtype=torch.int64, device="cuda")
    H = torch.zeros_like(G)
    Cn = torch.zeros((nf, 256), dtype=torch.int32, device="cuda")
    L = native.lib()
    # Keep every device tensor referenced until the kernel has finished.
    ct, it = torch.from_numpy(padded).cuda(), torch.from_numpy(idx).cuda()
    gt, ht = torch.from_numpy(g).cuda(), torch.from_numpy(h).cuda()
    native.check(L.tgb_hist_build(_p(ct), stride, nf, _p(it), idx.size, _p(gt), _p(ht), gs, hs, _p(G), _p(H), _p(Cn),
                                  None))
    torch.cuda.synchronize()
    nb = int(d["n_bins"])
    ref = d["hist"]
    assert np.array_equal(Cn.cpu().numpy()[:, :nb], ref[:, :, 2].astype(np.int32))
    absg = np.zeros((nf, nb))
    for f in range(nf):
        np.add.at(absg[f], codes[idx, f], np.abs(g[idx]))
    Gd = G.cpu().numpy()[:, :nb] * 2.0 ** -gs
    Hd = H.cpu().numpy()[:, :nb] * 2.0 ** -hs
    assert np.all(np.abs(Gd - ref[:, :, 0]) <= 1e-9 * absg + 1e-300)
    assert np.allclose(Hd, ref[:, :, 1], rtol=1e-9, atol=0)
    gain = torch.zeros(nf, dtype=torch.float64, device="cuda")
    thr = torch.zeros(nf, dtype=torch.int32, device="cuda")
    ml = torch.zeros(nf, dtype=torch.int32, device="cuda")
    native.check(L.tgb_split_scan(_p(G), _p(H), _p(Cn), nf, nb, gs, hs, float(s["l2"]), float(s["gamma"]),
                                  int(s["min_leaf"]), float(s["min_hess"]), _p(gain), _p(thr), _p(ml), None))
    assert np.array_equal(thr.cpu().numpy(), s["threshold"])
    assert np.array_equal(ml.cpu().numpy(), s["missing_left"])
    ok = s["threshold"] >= 0
    np.testing.assert_allclose(gain.cpu().numpy()[ok], s["gain"][ok], rtol=1e-9)


def test_pairwise_gradients_match_reference(native):
    d = load("pairwise.npz")
    groups = d["groups"]
    starts = np.flatnonzero(np.r_[True, groups[1:] != groups[:-1]]).astype(np.int32)
    lens = np.diff(np.r_[starts, groups.size]).astype(np.int32)
    m = groups.size
    yt, pt = torch.from_numpy(d["y"]).cuda(), torch.from_numpy(d["pred"]).cuda()
    gt, ht = torch.zeros_like(yt), torch.zeros_like(yt)
    st, lt = torch.from_numpy(starts).cuda(), torch.from_numpy(lens).cuda()
    native.check(native.lib().tgb_grad_pairwise(_p(yt), _p(pt), _p(st), _p(lt), None, starts.size, m, _p(gt), _p(ht),
                                                None))
    torch.cuda.synchronize()
    scale = np.abs(d["g"]) + np.abs(d["h"]) + 1e-3
    assert np.all(np.abs(gt.cpu().numpy() - d["g"]) <= 1e-12 * scale)
    assert np.all(np.abs(ht.cpu().numpy() - d["h"]) <= 1e-12 * scale)


@pytest.mark.parametrize("name", ["fit_mse", "fit_pair"])
def test_fit_matches_reference(native, name):
    d = load(f"{name}.npz")
    params = eval(str(d["params"]))  # the fixture's own dict literal
    b = native.Booster(pair_splits=False, **params)
    b.fit(d["X"], d["y"], timestamps=d["ts"], entity=d["entity"])
    trees = b.trees()
    assert len(trees) == int(d["n_trees"])
    info = b.info()
    assert info["n_bins"] == int(d["n_bins"]) and info["n_buckets"] == int(d["n_buckets"])
    for t, tr in enumerate(trees):
        for fld in ("is_leaf", "feature", "threshold", "left", "right", "missing_left", "n_samples", "depth", "cover"):
            assert np.array_equal(getattr(tr, fld), d[f"t{t}_{fld}"]), (t, fld)
        for fld in ("value", "values", "prefix"):
            np.testing.assert_allclose(getattr(tr, fld), d[f"t{t}_{fld}"], rtol=0, atol=1e-9, err_msg=f"{t} {fld}")
        np.testing.assert_allclose(tr.gain, d[f"t{t}_gain"], rtol=1e-9, atol=1e-9)
    np.testing.assert_allclose(b.evals_result()["train"], d["evals"], rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(b.raw_predict(d["X"][:500]), d["pred"], rtol=0, atol=1e-9)
