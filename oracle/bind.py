"""ctypes bindings for the oracle restatement (liboracle.so) and the reference
core compiled from its sources (_ref/libtgbref.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() as the
checker and by bench.py's reference / cpu_baseline legs.  The product never
imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libtgbref.so")
REF_CUDA_SO = os.path.join(HERE, "_ref", "libtgbref_cuda.so")

_P = np.ctypeslib.ndpointer
_f64 = _P(dtype=np.float64, flags="C_CONTIGUOUS")
_i32 = _P(dtype=np.int32, flags="C_CONTIGUOUS")
_i64 = _P(dtype=np.int64, flags="C_CONTIGUOUS")
_u8 = _P(dtype=np.uint8, flags="C_CONTIGUOUS")
_u16 = _P(dtype=np.uint16, flags="C_CONTIGUOUS")

OBJECTIVES = {"mse": 0, "pairwise": 5}


def build_oracle() -> None:
    if not os.path.exists(ORACLE_SO):
        subprocess.check_call(["make", "-s", "-C", HERE, "oracle"])


def ref_available() -> bool:
    return os.path.exists(REF_SO)


class _OrcConfig(C.Structure):
    _fields_ = [
        ("n_estimators", C.c_int), ("learning_rate", C.c_double), ("max_depth", C.c_int),
        ("max_leaves", C.c_int), ("min_samples_leaf", C.c_int), ("min_child_weight", C.c_double),
        ("l2", C.c_double), ("min_split_gain", C.c_double), ("max_bin", C.c_int),
        ("n_time_buckets", C.c_int), ("horizon", C.c_int64), ("embargo", C.c_int64),
        ("iid_mode", C.c_int), ("objective", C.c_int), ("random_state", C.c_int),
        ("goss", C.c_int), ("goss_top", C.c_double), ("goss_other", C.c_double),
        ("bin_sample", C.c_int), ("torb_min_cover", C.c_double), ("finer_torb", C.c_int),
        ("pair_splits", C.c_int), ("pair_trigger", C.c_double), ("pair_top_k", C.c_int),
        ("max_pair_splits_per_tree", C.c_int), ("pair_l2", C.c_double),
        ("cat_smooth", C.c_double), ("cat_min_count", C.c_int),
    ]


_orc = None
_ref = None


def oracle_lib():
    global _orc
    if _orc is None:
        build_oracle()
        L = C.CDLL(ORACLE_SO)
        L.orc_binner_fit.argtypes = [_f64, C.c_int, C.c_int, C.c_int, C.c_int, C.c_uint32, _f64, _i32, _i32]
        L.orc_binner_fit.restype = C.c_int
        L.orc_bin_transform.argtypes = [_f64, C.c_int, C.c_int, _f64, _i32, _u8, C.c_int]
        L.orc_build_hist.argtypes = [_u8, C.c_int, C.c_int, _i32, C.c_int, _f64, _f64, C.c_int, _f64]
        L.orc_grad_hess.argtypes = [C.c_int, _f64, _f64, C.c_void_p, C.c_int, _f64, _f64]
        L.orc_loss.argtypes = [C.c_int, _f64, _f64, C.c_void_p, C.c_int]
        L.orc_loss.restype = C.c_double
        L.orc_config_default.argtypes = [C.POINTER(_OrcConfig)]
        L.orc_fit.argtypes = [C.POINTER(_OrcConfig), _f64, _f64, C.c_int, C.c_int, C.c_void_p, C.c_void_p]
        L.orc_fit.restype = C.c_void_p
        L.orc_last_error.restype = C.c_char_p
        for name in ("orc_n_trees", "orc_n_bins", "orc_n_buckets"):
            getattr(L, name).argtypes = [C.c_void_p]
            getattr(L, name).restype = C.c_int
        L.orc_init_score.argtypes = [C.c_void_p]
        L.orc_init_score.restype = C.c_double
        L.orc_init_prefix.argtypes = [C.c_void_p, _f64]
        L.orc_evals_train.argtypes = [C.c_void_p, _f64]
        L.orc_tree_n_nodes.argtypes = [C.c_void_p, C.c_int]
        L.orc_tree_n_nodes.restype = C.c_int
        L.orc_tree_export.argtypes = [C.c_void_p, C.c_int, _i32, _f64, _f64, _i32, _f64]
        L.orc_predict_raw.argtypes = [C.c_void_p, _f64, C.c_int, _f64]
        L.orc_free.argtypes = [C.c_void_p]
        _orc = L
    return _orc


def ref_lib():
    global _ref
    if _ref is None:
        if not ref_available():
            raise RuntimeError(f"reference core not built ({REF_SO}); run make -C oracle ref")
        L = C.CDLL(REF_SO)
        L.ref_create.restype = C.c_void_p
        L.ref_free.argtypes = [C.c_void_p]
        L.ref_set.argtypes = [C.c_void_p, C.c_char_p, C.c_double]
        L.ref_fit.argtypes = [C.c_void_p, _f64, _f64, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
        L.ref_last_error.restype = C.c_char_p
        L.ref_predict_raw.argtypes = [C.c_void_p, _f64, C.c_int, C.c_int, _f64]
        for name in ("ref_n_trees", "ref_n_bins", "ref_n_time_buckets", "ref_n_evals"):
            getattr(L, name).argtypes = [C.c_void_p]
            getattr(L, name).restype = C.c_int
        L.ref_init_score.argtypes = [C.c_void_p]
        L.ref_init_score.restype = C.c_double
        L.ref_evals_train.argtypes = [C.c_void_p, _f64]
        L.ref_init_prefix.argtypes = [C.c_void_p, _f64]
        L.ref_tree_n_nodes.argtypes = [C.c_void_p, C.c_int]
        L.ref_tree_n_nodes.restype = C.c_int
        L.ref_tree_export.argtypes = [C.c_void_p, C.c_int, _i32, _f64, _f64, _i32, _f64]
        L.ref_edges.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        L.ref_edges.restype = C.c_int
        L.ref_binner.argtypes = [_f64, C.c_int, C.c_int, C.c_int, C.c_int, C.c_uint, _f64, _i32, _i32,
                                 C.POINTER(C.c_int), C.c_void_p]
        L.ref_build_hist_col.argtypes = [_u16, C.c_int, C.c_int, _i32, C.c_int, _f64, _f64, C.c_int,
                                         C.c_int, _f64]
        L.ref_best_numeric.argtypes = [_f64, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int,
                                       C.c_double, _f64, _i32]
        L.ref_grad_hess.argtypes = [C.c_int, _f64, _f64, C.c_void_p, C.c_int, _f64, _f64]
        L.ref_loss.argtypes = [C.c_int, _f64, _f64, C.c_void_p, C.c_int]
        L.ref_loss.restype = C.c_double
        _ref = L
    return _ref


@dataclass
class TreeArrays:
    """One fitted tree as flat arrays (node order = the reference's node ids)."""
    is_leaf: np.ndarray
    feature: np.ndarray
    threshold: np.ndarray
    left: np.ndarray
    right: np.ndarray
    missing_left: np.ndarray
    n_samples: np.ndarray
    depth: np.ndarray
    value: np.ndarray
    gain: np.ndarray
    values: np.ndarray
    cover: np.ndarray
    prefix: np.ndarray
    split_type: np.ndarray | None = None  # SplitType per node (0 axis, 1 pair, 2 categorical), when exported
    feature2: np.ndarray | None = None    # second feature of pair splits (-1 otherwise)
    cat_left: np.ndarray | None = None    # [n_nodes, 4] uint64 left masks of categorical splits

    @classmethod
    def from_raw(cls, inodes: np.ndarray, fnodes: np.ndarray, values, cover, prefix,
                 split: np.ndarray | None = None) -> "TreeArrays":
        I = inodes.reshape(-1, 8)
        F = fnodes.reshape(-1, 2)
        S = None if split is None else split.reshape(-1, 2)
        return cls(I[:, 0].copy(), I[:, 1].copy(), I[:, 2].copy(), I[:, 3].copy(), I[:, 4].copy(),
                   I[:, 5].copy(), I[:, 6].copy(), I[:, 7].copy(), F[:, 0].copy(), F[:, 1].copy(),
                   values, cover, prefix, None if S is None else S[:, 0].copy(), None if S is None else S[:, 1].copy())


@dataclass
class FitResult:
    trees: list = field(default_factory=list)
    init_score: float = 0.0
    init_prefix: np.ndarray | None = None
    evals_train: np.ndarray | None = None
    n_bins: int = 0
    n_buckets: int = 1


def _cfg_struct(params: dict) -> _OrcConfig:
    c = _OrcConfig()
    oracle_lib().orc_config_default(C.byref(c))
    c.pair_splits = 0  # the parity convention ref_fit shares: PAIR only when asked for
    for k, v in params.items():
        if k == "objective":
            v = OBJECTIVES[v] if isinstance(v, str) else int(v)
        if k in ("halo", "n_jobs"):
            continue
        setattr(c, k, int(v) if k == "pair_splits" else v)
    return c


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def oracle_fit(params: dict, X, y, ts=None, entity=None, is_cat=None) -> tuple[FitResult, int]:
    """Runs the oracle restatement's Booster::fit; returns (result, handle).  is_cat marks
    categorical features (one flag per column)."""
    L = oracle_lib()
    c = _cfg_struct(params)
    X = np.ascontiguousarray(X, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    ts = None if ts is None else np.ascontiguousarray(ts, dtype=np.int64)
    ent = None if entity is None else np.ascontiguousarray(entity, dtype=np.int64)
    cat = None if is_cat is None else np.ascontiguousarray(is_cat, dtype=np.int32)
    L.orc_fit_cat.restype = C.c_void_p
    L.orc_fit_cat.argtypes = [C.POINTER(_OrcConfig), _f64, _f64, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                              C.c_void_p]
    h = L.orc_fit_cat(C.byref(c), X, y, X.shape[0], X.shape[1], _ptr(ts), _ptr(ent), _ptr(cat))
    if not h:
        raise ValueError(L.orc_last_error().decode())
    res = FitResult(n_bins=L.orc_n_bins(h), n_buckets=L.orc_n_buckets(h), init_score=L.orc_init_score(h))
    res.init_prefix = np.zeros(res.n_buckets)
    L.orc_init_prefix(h, res.init_prefix)
    nt = L.orc_n_trees(h)
    res.evals_train = np.zeros(nt)
    L.orc_evals_train(h, res.evals_train)
    for t in range(nt):
        nn = L.orc_tree_n_nodes(h, t)
        I = np.zeros(8 * nn, np.int32)
        Fv = np.zeros(2 * nn)
        vals = np.zeros(nn)
        cov = np.zeros(nn, np.int32)
        pre = np.zeros(nn * res.n_buckets)
        L.orc_tree_export(h, t, I, Fv, vals, cov, pre)
        S = np.zeros(2 * nn, np.int32)
        L.orc_tree_export_split(h, t, S.ctypes.data_as(C.c_void_p))
        tr = TreeArrays.from_raw(I, Fv, vals, cov, pre, S)
        tr.cat_left = np.zeros((nn, 4), np.uint64)
        L.orc_tree_export_cat(h, t, tr.cat_left.ctypes.data_as(C.c_void_p))
        res.trees.append(tr)
    return res, h


def oracle_codes(X, params: dict, is_cat=None) -> tuple[np.ndarray, int]:
    """Binner::fit + transform of the oracle (binning.cpp:34-134): row-major uint8 codes of
    X under the fit's binning parameters, and the histogram width max_bins()."""
    L = oracle_lib()
    X = np.ascontiguousarray(X, dtype=np.float64)
    n, nf = X.shape
    cat = np.zeros(nf, np.int32) if is_cat is None else np.ascontiguousarray(is_cat, dtype=np.int32)
    edges = np.zeros(nf * 256)
    n_edges = np.zeros(nf, np.int32)
    codes = np.zeros((n, nf), np.uint8)
    L.orc_binner_fit_cat.restype = C.c_int
    L.orc_binner_fit_cat.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_uint32,
                                     C.c_void_p, C.c_void_p, C.c_void_p]
    nb = L.orc_binner_fit_cat(X.ctypes.data, n, nf, cat.ctypes.data, int(params.get("max_bin", 255)),
                              int(params.get("cat_min_count", 5)), int(params.get("bin_sample", 262144)),
                              int(params.get("random_state", 0)) & 0xFFFFFFFF, edges.ctypes.data, n_edges.ctypes.data,
                              codes.ctypes.data)
    return codes, nb


def oracle_predict(handle, X) -> np.ndarray:
    X = np.ascontiguousarray(X, dtype=np.float64)
    out = np.zeros(X.shape[0])
    oracle_lib().orc_predict_raw(handle, X, X.shape[0], out)
    return out


def oracle_free(handle) -> None:
    oracle_lib().orc_free(handle)


def ref_fit(params: dict, X, y, ts=None, entity=None, n_jobs: int = 0, is_cat=None):
    """Runs the reference core's Booster::fit (rank groups = timestamps, as
    src/tidegbm/native.py:134-137 passes them); returns (FitResult, handle)."""
    L = ref_lib()
    h = L.ref_create()
    settings = {"pair_splits": 0, "halo": 0, "n_jobs": n_jobs}
    settings.update(params)
    for k, v in settings.items():
        if k == "objective":
            v = OBJECTIVES[v] if isinstance(v, str) else int(v)
        if L.ref_set(h, k.encode(), float(v)) != 0:
            raise KeyError(k)
    X = np.ascontiguousarray(X, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    ts = None if ts is None else np.ascontiguousarray(ts, dtype=np.int64)
    ent = None if entity is None else np.ascontiguousarray(entity, dtype=np.int64)
    obj = settings.get("objective", "mse")
    rg = ts if obj in ("pairwise", 5) else None
    if is_cat is None:
        rc = L.ref_fit(h, X, y, X.shape[0], X.shape[1], _ptr(ts), _ptr(rg), _ptr(ent))
    else:
        cat = np.ascontiguousarray(is_cat, dtype=np.int32)
        L.ref_fit_cat.argtypes = [C.c_void_p, _f64, _f64, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                  C.c_void_p]
        rc = L.ref_fit_cat(h, X, y, X.shape[0], X.shape[1], _ptr(ts), _ptr(rg), _ptr(ent), _ptr(cat))
    if rc != 0:
        err = L.ref_last_error().decode()
        L.ref_free(h)
        raise ValueError(err)
    nb = L.ref_n_time_buckets(h)
    res = FitResult(n_bins=L.ref_n_bins(h), n_buckets=nb, init_score=L.ref_init_score(h))
    res.init_prefix = np.zeros(max(nb, 1))
    L.ref_init_prefix(h, res.init_prefix)
    res.evals_train = np.zeros(L.ref_n_evals(h))
    L.ref_evals_train(h, res.evals_train)
    for t in range(L.ref_n_trees(h)):
        nn = L.ref_tree_n_nodes(h, t)
        I = np.zeros(8 * nn, np.int32)
        Fv = np.zeros(2 * nn)
        vals = np.zeros(nn)
        cov = np.zeros(nn, np.int32)
        pre = np.zeros(nn * nb)
        L.ref_tree_export(h, t, I, Fv, vals, cov, pre)
        S = np.zeros(2 * nn, np.int32)
        L.ref_tree_export_split(h, t, S.ctypes.data_as(C.c_void_p))
        tr = TreeArrays.from_raw(I, Fv, vals, cov, pre, S)
        tr.cat_left = np.zeros((nn, 4), np.uint64)
        L.ref_tree_export_cat(h, t, tr.cat_left.ctypes.data_as(C.c_void_p))
        res.trees.append(tr)
    return res, h


def ref_predict(handle, X) -> np.ndarray:
    X = np.ascontiguousarray(X, dtype=np.float64)
    out = np.zeros(X.shape[0])
    if ref_lib().ref_predict_raw(handle, X, X.shape[0], X.shape[1], out) != 0:
        raise ValueError(ref_lib().ref_last_error().decode())
    return out


def ref_free(handle) -> None:
    ref_lib().ref_free(handle)


def ref_import(n_features: int, n_bins: int, n_buckets: int, init_score: float, init_prefix, edges, n_edges,
               max_bin: int, learning_rate: float, objective, iid_mode: bool, trees) -> int:
    """A fitted reference Booster holding a model grown elsewhere (trees as TreeArrays,
    edges F x 256 with n_edges[f] used); returns its handle (free with ref_free)."""
    L = ref_lib()
    obj = OBJECTIVES[objective] if isinstance(objective, str) else int(objective)
    nodes = np.array([t.is_leaf.size for t in trees], np.int32)
    I = np.ascontiguousarray(np.concatenate([np.stack([t.is_leaf, t.feature, t.threshold, t.left, t.right,
                                                       t.missing_left, t.n_samples, t.depth], axis=1).ravel()
                                             for t in trees]).astype(np.int32))
    Fv = np.ascontiguousarray(np.concatenate([np.stack([t.value, t.gain], axis=1).ravel() for t in trees]))
    vals = np.ascontiguousarray(np.concatenate([t.values for t in trees]))
    cov = np.ascontiguousarray(np.concatenate([t.cover for t in trees]).astype(np.int32))
    pre = np.ascontiguousarray(np.concatenate([np.asarray(t.prefix).ravel() for t in trees]))
    ip = np.ascontiguousarray(np.asarray(init_prefix, np.float64))
    E = np.ascontiguousarray(np.asarray(edges, np.float64).reshape(n_features, 256))
    ne = np.ascontiguousarray(np.asarray(n_edges, np.int32))
    h = L.ref_create()
    vp = C.c_void_p
    L.ref_import_model.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_double, vp, C.c_int, vp, vp, C.c_int,
                                   C.c_double, C.c_int, C.c_int, C.c_int, vp, vp, vp, vp, vp, vp]
    rc = L.ref_import_model(h, n_features, n_bins, n_buckets, init_score, _ptr(ip), ip.size, _ptr(E), _ptr(ne),
                            max_bin, learning_rate, obj, int(iid_mode), len(trees), _ptr(nodes), _ptr(I), _ptr(Fv),
                            _ptr(vals), _ptr(cov), _ptr(pre))
    if rc != 0:
        L.ref_free(h)
        raise ValueError(L.ref_last_error().decode())
    return h


def ref_edges_of(handle, n_features: int) -> tuple[np.ndarray, np.ndarray]:
    """Edges (F x 256) and their counts of a fitted reference Booster."""
    L = ref_lib()
    L.ref_edges.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
    L.ref_edges.restype = C.c_int
    E = np.zeros((n_features, 256))
    ne = np.zeros(n_features, np.int32)
    for f in range(n_features):
        ne[f] = L.ref_edges(handle, f, None)
        L.ref_edges(handle, f, E[f].ctypes.data_as(C.c_void_p))
    return E, ne


def ref_save(handle) -> bytes:
    """The reference's .tgbm blob (Booster::save_binary)."""
    L = ref_lib()
    L.ref_save_binary.argtypes = [C.c_void_p, C.c_char_p, C.c_longlong]
    L.ref_save_binary.restype = C.c_longlong
    n = L.ref_save_binary(handle, None, 0)
    if n < 0:
        raise ValueError(L.ref_last_error().decode())
    buf = C.create_string_buffer(int(n))
    L.ref_save_binary(handle, buf, n)
    return buf.raw[: int(n)]


def ref_load(blob: bytes) -> int:
    """A reference Booster from a .tgbm blob (Booster::load_binary)."""
    L = ref_lib()
    L.ref_load_binary.argtypes = [C.c_char_p, C.c_longlong]
    L.ref_load_binary.restype = C.c_void_p
    h = L.ref_load_binary(blob, len(blob))
    if not h:
        raise ValueError(L.ref_last_error().decode())
    return h
