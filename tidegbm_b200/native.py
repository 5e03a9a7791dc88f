"""ctypes binding of libtidegbm_b200.so, shaped like TideGBM's pybind module.

`Booster` mirrors `tidegbm._core.Booster` (cpp/src/bindings.cpp:133-323) for the
GPU path: `set_config(**kwargs)` takes the same keyword names as
`config_from_kwargs` (bindings.cpp:25-127), `fit(X, y, timestamps=..., entity=...)`
runs Booster::fit with device="gpu", `raw_predict` / `evals_result` / `trees()` read
the fitted model back.  Errors raise `TideError` with the library's message, as the
pybind module maps TideError (bindings.cpp:131).

The shared library must be built in-tree (`python -m tidegbm_b200.build`); there is
no CPU fallback: importing this module without the library raises.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtidegbm_b200.so")


class TideError(RuntimeError):
    pass


_lib = None


def lib() -> C.CDLL:
    """Loads libtidegbm_b200.so (building it first if only the sources are present)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        from . import build as _build

        _build.build()
    L = C.CDLL(LIB_PATH)
    vp, i, d, ll, cp = C.c_void_p, C.c_int, C.c_double, C.c_longlong, C.c_char_p
    sig = {
        "tgb_last_error": ([], cp),
        "tgb_kernel_launches": ([], ll),
        "tgb_booster_create": ([i, C.POINTER(vp)], i),
        "tgb_booster_free": ([vp], None),
        "tgb_set_int": ([vp, cp, ll], i),
        "tgb_set_double": ([vp, cp, d], i),
        "tgb_set_str": ([vp, cp, cp], i),
        "tgb_fit": ([vp, vp, i, vp, i, i, vp, vp], i),
        "tgb_fit_batch": ([vp, i, vp, i, vp, vp, i, vp, vp], i),
        "tgb_tree_export_split": ([vp, i, vp, vp, vp], i),
        "tgb_set_categorical": ([vp, vp, i], i),
        "tgb_hist_build_quantized": ([vp, i, i, vp, i, vp, vp, i, C.c_ulonglong, vp, vp, vp, vp, vp], i),
        "tgb_predict_raw": ([vp, vp, i, i, i, vp], i),
        "tgb_model_info": ([vp, vp, vp, vp, vp], i),
        "tgb_init_prefix": ([vp, vp], i),
        "tgb_evals_train": ([vp, vp], i),
        "tgb_tree_n_nodes": ([vp, i], i),
        "tgb_tree_export": ([vp, i, vp, vp, vp, vp, vp], i),
        "tgb_edges": ([vp, i, vp], i),
        "tgb_fit_stats": ([vp, vp], i),
        "tgb_fit_stat": ([vp, cp, vp], i),
        "tgb_binner_fit_device": ([vp, i, i, i, i, i, C.c_uint, vp, vp, vp], i),
        "tgb_binner_fit": ([vp, i, i, i, i, i, C.c_uint, vp, vp], i),
        "tgb_binner_fit_cat": ([vp, i, i, i, vp, i, i, i, C.c_uint, vp, vp], i),
        "tgb_shuffled_prefix": ([ll, ll, C.c_uint, vp], i),
        "tgb_shuffled_prefix_device": ([ll, ll, C.c_uint, vp, vp], i),
        "tgb_shuffle_sequence": ([ll, ll, C.c_uint, i, vp], i),
        "tgb_server_create": ([i, d, i, C.POINTER(vp)], i),
        "tgb_server_free": ([vp], None),
        "tgb_working_set_bytes": ([vp, i, i, i, i], ll),
        "tgb_server_submit_fit": ([vp, vp, vp, i, vp, i, i, vp, vp, C.POINTER(ll)], i),
        "tgb_server_submit_predict": ([vp, vp, vp, i, i, i, vp, C.POINTER(ll)], i),
        "tgb_server_wait": ([vp, ll, d, C.POINTER(i)], i),
        "tgb_server_stats": ([vp, vp], i),
        "tgb_bin_transform": ([vp, i, i, i, vp, vp, vp, i, vp], i),
        "tgb_hist_build": ([vp, i, i, vp, i, vp, vp, i, i, vp, vp, vp, vp], i),
        "tgb_split_scan": ([vp, vp, vp, i, i, i, i, d, d, i, d, vp, vp, vp, vp], i),
        "tgb_partition_workspace_bytes": ([i], C.c_size_t),
        "tgb_partition": ([vp, i, vp, i, i, i, i, vp, vp, vp, C.c_size_t, vp], i),
        "tgb_partition_noalloc": ([vp, i, vp, i, i, i, i, vp, vp, vp], i),
        "tgb_grad_mse": ([vp, vp, i, vp, vp, vp], i),
        "tgb_grad_pairwise": ([vp, vp, vp, vp, vp, i, i, vp, vp, vp], i),
        "tgb_build_hist_gpu": ([vp, vp, i, vp, i, vp, vp, i, i, vp], i),
    }
    for name, (args, res) in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    _lib = L
    return L


def check(rc: int) -> None:
    if rc != 0:
        raise TideError(lib().tgb_last_error().decode())


def _ptr(a) -> C.c_void_p | None:
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return C.c_void_p(a.data_ptr())
    return a.ctypes.data_as(C.c_void_p)


_INT_KEYS = {"n_estimators", "max_depth", "max_leaves", "min_samples_leaf", "max_bin", "n_time_buckets",
             "random_state", "n_jobs", "iid_mode", "halo", "pair_splits", "horizon", "embargo", "goss",
             "bin_sample", "finer_torb", "causal_bins", "causal_structure", "verbose", "col_major_hist",
             "cat_min_count", "timing_from", "timing_to", "profile_hist", "hist_bits", "grow", "graph", "hist_tune", "wave_expand", "hist_stage",
             "pair_top_k", "max_pair_splits_per_tree"}
_DOUBLE_KEYS = {"cat_smooth", "pair_trigger", "pair_l2", "learning_rate", "l2", "l1", "min_child_weight", "min_split_gain", "subsample", "colsample",
                "colsample_bynode", "goss_top", "goss_other", "torb_min_cover", "max_delta_step", "time_decay",
                "structure_frac", "entity_subsample"}
_STR_KEYS = {"objective", "device"}


@dataclass
class Tree:
    """One tree, node order = node ids (the fields .tgbm stores, serialize.cpp:120-143)."""
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
    split_type: np.ndarray | None = None  # 0 axis, 2 categorical
    cat_left: np.ndarray | None = None    # [n_nodes, 4] uint64 left masks of categorical splits
    feature2: np.ndarray | None = None    # second feature of pair splits (-1 otherwise)


class Booster:
    """device="gpu" Booster (cpp/include/tidegbm/booster.hpp:22-72)."""

    def __init__(self, device: int = 0, **params) -> None:
        h = C.c_void_p()
        check(lib().tgb_booster_create(int(device), C.byref(h)))
        self._h = h
        self.params: dict = {}
        self.set_config(device="gpu", **params)

    def __del__(self) -> None:
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            _lib.tgb_booster_free(h)
            self._h = None

    def set_config(self, **kw) -> None:
        L = lib()
        for k, v in kw.items():
            if v is None:
                continue
            if k == "goss" and isinstance(v, bool):
                v = int(v)
            if k in _STR_KEYS:
                check(L.tgb_set_str(self._h, k.encode(), str(v).encode()))
            elif k in _INT_KEYS:
                check(L.tgb_set_int(self._h, k.encode(), int(v)))
            elif k in _DOUBLE_KEYS:
                check(L.tgb_set_double(self._h, k.encode(), float(v)))
            else:
                raise TideError(f"unknown config key: {k}")
            self.params[k] = v

    def fit(self, X, y, timestamps=None, entity=None, is_cat=None, **kw) -> "Booster":
        """is_cat: one flag per feature marking the categorical ones (Booster::fit's is_cat)."""
        if kw:
            self.set_config(**kw)
        ic = None if is_cat is None else np.ascontiguousarray(is_cat, dtype=np.int32)
        check(lib().tgb_set_categorical(self._h, _ptr(ic), 0 if ic is None else ic.size))
        X = np.asarray(X)
        if X.ndim != 2:
            raise TideError("X must be 2d")
        if X.dtype != np.float32:
            X = np.ascontiguousarray(X, dtype=np.float64)
        X = np.ascontiguousarray(X)
        dt = 0 if X.dtype == np.float32 else 1
        y = np.ascontiguousarray(y, dtype=np.float64)
        ts = None if timestamps is None else np.ascontiguousarray(timestamps, dtype=np.int64)
        ent = None if entity is None else np.ascontiguousarray(entity, dtype=np.int64)
        check(lib().tgb_fit(self._h, _ptr(X), dt, _ptr(y), X.shape[0], X.shape[1], _ptr(ts), _ptr(ent)))
        return self

    @staticmethod
    def fit_batch(boosters, Xs, ys, timestamps=None, entities=None) -> None:
        """Fits boosters[k] on (Xs[k], ys[k], timestamps[k], entities[k]) in lockstep
        (tgb_fit_batch): every tree of all of them grows in the same batched launches, and
        each result equals that booster's own fit.  All X share one dtype and feature count."""
        k = len(boosters)
        if not (k == len(Xs) == len(ys)) or k == 0:
            raise TideError("fit_batch: one X and y per booster")
        Xs = [np.ascontiguousarray(X, dtype=np.float32 if np.asarray(X).dtype == np.float32 else np.float64)
              for X in Xs]
        dt = 0 if Xs[0].dtype == np.float32 else 1
        if any((X.dtype == np.float32) != (dt == 0) or X.shape[1] != Xs[0].shape[1] for X in Xs):
            raise TideError("fit_batch: X of one dtype and feature count")
        ys = [np.ascontiguousarray(y, dtype=np.float64) for y in ys]
        tss = None if timestamps is None else [np.ascontiguousarray(t, dtype=np.int64) for t in timestamps]
        ens = None if entities is None else [np.ascontiguousarray(e, dtype=np.int64) for e in entities]
        arr = lambda seq: (C.c_void_p * k)(*[a.ctypes.data for a in seq])
        hs = (C.c_void_p * k)(*[b._h.value for b in boosters])
        ns = (C.c_int * k)(*[X.shape[0] for X in Xs])
        check(lib().tgb_fit_batch(hs, k, arr(Xs), dt, arr(ys), ns, Xs[0].shape[1],
                                  arr(tss) if tss is not None else None, arr(ens) if ens is not None else None))

    def raw_predict(self, X) -> np.ndarray:
        X = np.asarray(X)
        if X.dtype != np.float32:
            X = np.ascontiguousarray(X, dtype=np.float64)
        X = np.ascontiguousarray(X)
        out = np.zeros(X.shape[0])
        check(lib().tgb_predict_raw(self._h, _ptr(X), 0 if X.dtype == np.float32 else 1, X.shape[0], X.shape[1],
                                    _ptr(out)))
        return out

    predict = raw_predict

    def info(self) -> dict:
        nt, nb, nbk = C.c_int(), C.c_int(), C.c_int()
        init = C.c_double()
        check(lib().tgb_model_info(self._h, C.byref(nt), C.byref(nb), C.byref(nbk), C.byref(init)))
        return {"n_trees": nt.value, "n_bins": nb.value, "n_buckets": nbk.value, "init_score": init.value}

    def init_prefix(self) -> np.ndarray:
        out = np.zeros(self.info()["n_buckets"])
        check(lib().tgb_init_prefix(self._h, _ptr(out)))
        return out

    def evals_result(self) -> dict:
        out = np.zeros(self.info()["n_trees"])
        check(lib().tgb_evals_train(self._h, _ptr(out)))
        return {"train": out.tolist(), "valid": []}

    def trees(self) -> list[Tree]:
        info = self.info()
        res = []
        for t in range(info["n_trees"]):
            nn = lib().tgb_tree_n_nodes(self._h, t)
            if nn < 0:
                check(-1)
            I = np.zeros(8 * nn, np.int32)
            F = np.zeros(2 * nn)
            vals = np.zeros(nn)
            cov = np.zeros(nn, np.int32)
            pre = np.zeros(nn * info["n_buckets"])
            check(lib().tgb_tree_export(self._h, t, _ptr(I), _ptr(F), _ptr(vals), _ptr(cov), _ptr(pre)))
            I = I.reshape(-1, 8)
            F = F.reshape(-1, 2)
            ty = np.zeros(nn, np.int32)
            f2 = np.zeros(nn, np.int32)
            cm = np.zeros((nn, 4), np.uint64)
            check(lib().tgb_tree_export_split(self._h, t, _ptr(ty), _ptr(f2), _ptr(cm)))
            res.append(Tree(*(I[:, k].copy() for k in range(8)), F[:, 0].copy(), F[:, 1].copy(), vals, cov, pre,
                            ty, cm, f2))
        return res

    def edges(self, f: int) -> np.ndarray:
        n = lib().tgb_edges(self._h, f, None)
        if n < 0:
            check(-1)
        out = np.zeros(n)
        lib().tgb_edges(self._h, f, _ptr(out))
        return out

    def fit_stats(self) -> dict:
        o = np.zeros(18)
        check(lib().tgb_fit_stats(self._h, _ptr(o)))
        keys = ["total", "sort", "bin_fit", "upload_transform", "trees", "download", "host_rng", "kernel_launches",
                "timed_ms", "timed_trees", "timed_launches", "hist_ms", "hist_launches", "hist_rows", "alloc", "h2d",
                "transpose", "goss_producer"]
        res = dict(zip(keys, o.tolist()))
        for k in ("bin_counts", "bin_draws", "bin_edges", "goss_refits", "pre_upload", "prep", "timed_selects",
                  "graph_used", "hist_cluster", "hist_clusters", "driver", "finish_sync", "driver_free", "release", "expansions"):
            v = C.c_double()
            check(lib().tgb_fit_stat(self._h, k.encode(), C.byref(v)))
            res[k] = v.value
        return res

    def build_hist_gpu(self, xb: np.ndarray, idx: np.ndarray, g: np.ndarray, h: np.ndarray, n_bins: int) -> np.ndarray:
        """Drop-in for build_hist_gpu (cpp/src/histogram_cuda.cu:81-167): returns the
        interleaved FP64 {g, h, c} histogram, shape (n_features, n_bins, 3)."""
        xb = np.ascontiguousarray(xb, dtype=np.uint16)
        idx = np.ascontiguousarray(idx, dtype=np.int32)
        g = np.ascontiguousarray(g, dtype=np.float64)
        h = np.ascontiguousarray(h, dtype=np.float64)
        nf = xb.shape[1]
        out = np.zeros(nf * n_bins * 3)
        check(lib().tgb_build_hist_gpu(self._h, _ptr(xb), nf, _ptr(idx), idx.size, _ptr(g), _ptr(h), n_bins,
                                       xb.shape[0], _ptr(out)))
        return out.reshape(nf, n_bins, 3)


class Server:
    """The serving loop (tgb_server_*): fit and predict requests on one device, admitted in
    arrival order by device-memory budget and free slots, running concurrently on their
    boosters' own streams.  Each request keeps references to its arrays until it is waited
    for, so the host buffers stay alive while the device uses them."""

    QUEUED, RUNNING, DONE, FAILED = 0, 1, 2, 3

    def __init__(self, device: int = 0, budget_bytes: float = 150e9, slots: int = 4) -> None:
        h = C.c_void_p()
        check(lib().tgb_server_create(int(device), float(budget_bytes), int(slots), C.byref(h)))
        self._h = h
        self._keep: dict[int, tuple] = {}

    def close(self) -> None:
        """Waits for every request, then frees the server."""
        if self._h:
            lib().tgb_server_free(self._h)
            self._h = None
            self._keep.clear()

    def __del__(self) -> None:
        if getattr(self, "_h", None) and _lib is not None:
            self.close()

    def submit_fit(self, booster: "Booster", X, y, timestamps=None, entity=None) -> int:
        X = np.asarray(X)
        X = np.ascontiguousarray(X if X.dtype == np.float32 else X.astype(np.float64))
        y = np.ascontiguousarray(y, dtype=np.float64)
        ts = None if timestamps is None else np.ascontiguousarray(timestamps, dtype=np.int64)
        ent = None if entity is None else np.ascontiguousarray(entity, dtype=np.int64)
        rid = C.c_longlong()
        check(lib().tgb_server_submit_fit(self._h, booster._h, _ptr(X), 0 if X.dtype == np.float32 else 1, _ptr(y),
                                          X.shape[0], X.shape[1], _ptr(ts), _ptr(ent), C.byref(rid)))
        self._keep[rid.value] = (booster, X, y, ts, ent)
        return rid.value

    def submit_predict(self, booster: "Booster", X) -> tuple[int, np.ndarray]:
        """Returns (request id, output array filled once the request is done)."""
        X = np.asarray(X)
        X = np.ascontiguousarray(X if X.dtype == np.float32 else X.astype(np.float64))
        out = np.zeros(X.shape[0])
        rid = C.c_longlong()
        check(lib().tgb_server_submit_predict(self._h, booster._h, _ptr(X), 0 if X.dtype == np.float32 else 1,
                                              X.shape[0], X.shape[1], _ptr(out), C.byref(rid)))
        self._keep[rid.value] = (booster, X, out)
        return rid.value, out

    def wait(self, rid: int, timeout_ms: float = -1.0) -> int:
        """Request state; raises TideError with the request's message when it failed."""
        st = C.c_int()
        check(lib().tgb_server_wait(self._h, int(rid), float(timeout_ms), C.byref(st)))
        if st.value in (self.DONE, self.FAILED):
            self._keep.pop(rid, None)
        if st.value == self.FAILED:
            raise TideError(lib().tgb_last_error().decode())
        return st.value

    def stats(self) -> dict:
        o = np.zeros(12)
        check(lib().tgb_server_stats(self._h, _ptr(o)))
        keys = ("completed", "failed", "p50_s", "p99_s", "p50_fit_s", "p99_fit_s", "p50_predict_s", "p99_predict_s",
                "mean_wait_s", "peak_running", "peak_bytes", "busy_s")
        return dict(zip(keys, o.tolist()))


def kernel_launches() -> int:
    return int(lib().tgb_kernel_launches())
