#!/usr/bin/env python
"""Benchmark of the device="gpu" TideGBM training hot path on B200.

Workload (default): the 10M-row panel — 5,000 dates x 2,000 entities, 128 float32
features (N(0,1) and log-normal columns, 1% NaN), 255 bins, objective mse, GOSS auto
(top 20% / other 10%), max_depth 8, max_leaves 31 (reference default), 100 trees,
synthetic seeded data (tidegbm_b200.panels.panel_scale).

A step is one boosting iteration (one tree: gradients, GOSS selection, histograms,
split scans, partitions, post-tree TORB sweep, prediction update, loss).  One fit of
max(100, W+K) trees is run through the C ABI (tgb_fit) from pinned host buffers:
  value     trees/s over trees W..W+K-1, device time from CUDA events on the fit's
            stream (inputs resident in HBM; the 1.28 GB code matrix exceeds L2)
  e2e       trees/s of the whole tgb_fit call (host X/y in, trees out: binning,
            H2D, transform, all trees, D2H) — wall clock, on the second full-size fit of
            the process (a 2-tree fit of the same workload warms it up first; its wall
            time is reported as cold_first_fit)
A second, short fit with per-launch events around every histogram kernel gives the
histogram GB/s (algorithmic bytes: rows x (F code bytes + 16 B of f64 g, h)).
The reference's own CPU fit (oracle/_ref, built from its sources) is timed on a
bounded 1M-row sample of the same workload and scaled to 10M rows; the reference's
only GPU code (build_hist_gpu, compiled for sm_100a) is timed on the same root
histogram as "plain GPU".

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "hist GB/s & trees/s (10M×128, 255 bins) vs plain GPU; serve p50/p99 at same IC"
PARAMS = dict(n_estimators=100, learning_rate=0.1, max_depth=8, max_leaves=31, max_bin=255, horizon=1,
              objective="mse", goss=-1, goss_top=0.2, goss_other=0.1, random_state=0, pair_splits=False)
WORKLOAD = ("panel_scale: 10M rows (5000 dates x 2000 entities) x 128 f32 features, 1% NaN, 255 bins, mse, "
            "GOSS auto (0.2/0.1), max_depth 8, max_leaves 31, 100 trees")


def peaks() -> dict:
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    except Exception:
        return {"hbm_gbs": 6650.0, "source": "fallback"}


class ClockSampler:
    """nvidia-smi clocks + throttle reasons sampled every 200 ms during a region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int) -> None:
        self.gpu = gpu_index
        self.proc = None
        self.path = tempfile.mktemp(suffix=".csv")

    def __enter__(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
        try:
            self.f.close()
        except Exception:
            pass

    def summary(self) -> dict:
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            for ln in open(self.path):
                p = [x.strip() for x in ln.split(",")]
                if len(p) < 9:
                    continue
                try:
                    sm.append(float(p[1]))
                    mx.append(float(p[2]))
                except ValueError:
                    continue
                for nm, v in zip(names, p[5:9]):
                    if v.lower() == "active":
                        reasons.add(nm)
        except Exception:
            pass
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def make_panel(n_dates: int = 5000):
    from tidegbm_b200 import panels

    return panels.panel_scale(n_dates=n_dates)


# ---------------------------------------------------------------- reference CPU
def ref_cpu_trees_per_s(warmup: int, steps: int, n_dates: int = 500) -> dict:
    """The reference's own CPU fit (oracle/_ref, all host cores, n_jobs = 0) on a
    bounded sample of the workload: the first n_dates dates (n_dates x 2000 rows).
    Per-tree time from the reference's per-iteration hook; scaled by rows to 10M."""
    from oracle import bind

    L = bind.ref_lib()
    L.ref_fit_timed.argtypes = [C.c_void_p] + [np.ctypeslib.ndpointer(np.float64, flags="C")] * 2 + \
        [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, np.ctypeslib.ndpointer(np.float64, flags="C")]
    p = make_panel(n_dates)
    X = np.ascontiguousarray(p.X, dtype=np.float64)
    h = L.ref_create()
    n_est = warmup + steps
    cfg = dict(PARAMS, n_estimators=n_est, n_jobs=0, halo=0)
    for k, v in cfg.items():
        if k == "objective":
            v = 0
        if L.ref_set(h, k.encode(), float(v)) != 0:
            raise KeyError(k)
    t_iter = np.zeros(n_est)
    ts = np.ascontiguousarray(p.ts)
    ent = np.ascontiguousarray(p.entity.astype(np.int64))
    devnull = os.open(os.devnull, os.O_WRONLY)
    saved = os.dup(2)
    os.dup2(devnull, 2)  # the reference prints one line per iteration with verbose = 1
    try:
        t0 = time.perf_counter()
        rc = L.ref_fit_timed(h, X, np.ascontiguousarray(p.y), p.n, p.n_features, ts.ctypes.data_as(C.c_void_p),
                             None, ent.ctypes.data_as(C.c_void_p), t_iter)
        wall = time.perf_counter() - t0
    finally:
        os.dup2(saved, 2)
        os.close(devnull)
        os.close(saved)
    L.ref_free(h)
    if rc != 0:
        raise RuntimeError(L.ref_last_error().decode())
    per_tree = (t_iter[n_est - 1] - (t_iter[warmup - 1] if warmup > 0 else 0.0)) / steps
    scale = 10_000_000 / p.n
    return {"value": 1.0 / (per_tree * scale), "unit": "trees/s", "cores": os.cpu_count(), "kind": "reference",
            "sample": f"reference Booster::fit (oracle/_ref, -O3 -fopenmp, n_jobs=0) on {p.n} rows "
                      f"({n_dates} dates x 2000) x 128 of the same generator; {warmup} warm-up + {steps} timed trees "
                      f"via its per-iteration hook ({per_tree:.3f} s/tree), scaled x{scale:g} rows to 10M; "
                      f"fit wall {wall:.1f} s incl. binning",
            "per_tree_s_sample": per_tree}


def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    try:
        from oracle import bind

        if not bind.ref_available():
            raise RuntimeError("reference core not built (oracle/_ref)")
        r = ref_cpu_trees_per_s(max(1, args.warmup), max(1, args.steps))
    except Exception as e:  # pragma: no cover
        print(json.dumps({"impl": "reference", "unavailable": f"{type(e).__name__}: {e}"}))
        return
    line = {"impl": "reference", "metric": METRIC, "value": r["value"], "unit": "trees/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 / r["value"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "parallelism": "host OpenMP"},
            "cpu_baseline": {k: r[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": r["value"], "unit": "trees/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# ---------------------------------------------------------------- plain GPU
def plain_gpu_hist(native, X32, edges, n_edges, idx, g, h, n_bins) -> dict | None:
    """The reference's build_hist_gpu (cpp/src/histogram_cuda.cu:81-167, built for
    sm_100a) on one root histogram, against this library's kernel on the same rows."""
    import torch
    from oracle import bind

    if not os.path.exists(bind.REF_CUDA_SO):
        return None
    R = C.CDLL(bind.REF_CUDA_SO)
    R.refgpu_build_hist.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int,
                                    C.c_int, C.c_void_p]
    n, nf = X32.shape
    stride = (nf + 15) // 16 * 16
    # codes via this library's transform (bit-identical to the reference's Binner::transform)
    E = np.full((nf, 256), np.inf, dtype=np.float32)
    for f in range(nf):
        e = edges[f, : n_edges[f]]
        e32 = e.astype(np.float32)
        low = e32.astype(np.float64) < e
        e32[low] = np.nextafter(e32[low], np.float32(np.inf))
        E[f, : n_edges[f]] = e32
    Xd = torch.from_numpy(X32).cuda()
    Ed = torch.from_numpy(E).cuda()
    ned = torch.from_numpy(n_edges.astype(np.int32)).cuda()
    codes = torch.empty((n, stride), dtype=torch.uint8, device="cuda")
    native.check(native.lib().tgb_bin_transform(C.c_void_p(Xd.data_ptr()), 0, n, nf, C.c_void_p(Ed.data_ptr()),
                                                C.c_void_p(ned.data_ptr()), C.c_void_p(codes.data_ptr()), stride,
                                                None))
    torch.cuda.synchronize()
    del Xd
    xb16 = np.ascontiguousarray(codes[:, :nf].cpu().numpy().astype(np.uint16))
    out = np.zeros(nf * n_bins * 3)
    bytes_alg = idx.size * (nf + 16)
    args = (xb16.ctypes.data_as(C.c_void_p), nf, idx.ctypes.data_as(C.c_void_p), idx.size,
            g.ctypes.data_as(C.c_void_p), h.ctypes.data_as(C.c_void_p), n_bins, n, out.ctypes.data_as(C.c_void_p))
    if R.refgpu_build_hist(*args) != 0:  # first call uploads the code matrix once
        return None
    reps = 3
    t0 = time.perf_counter()
    for _ in range(reps):
        R.refgpu_build_hist(*args)
    ref_s = (time.perf_counter() - t0) / reps
    # this library's kernel on the same rows, inputs resident
    rt = torch.from_numpy(idx).cuda()
    gt, ht = torch.from_numpy(g).cuda(), torch.from_numpy(h).cuda()
    G = torch.zeros((nf, 256), dtype=torch.int64, device="cuda")
    H = torch.zeros_like(G)
    Cn = torch.zeros((nf, 256), dtype=torch.int32, device="cuda")
    gs = 61 - (int(np.floor(np.log2(np.abs(g[idx]).max()))) + 1) - int(np.ceil(np.log2(idx.size)))
    hs = 61 - (int(np.floor(np.log2(np.abs(h[idx]).max()))) + 1) - int(np.ceil(np.log2(idx.size)))
    L = native.lib()
    def ours():
        L.tgb_hist_build(C.c_void_p(codes.data_ptr()), stride, nf, C.c_void_p(rt.data_ptr()), idx.size,
                         C.c_void_p(gt.data_ptr()), C.c_void_p(ht.data_ptr()), gs, hs, C.c_void_p(G.data_ptr()),
                         C.c_void_p(H.data_ptr()), C.c_void_p(Cn.data_ptr()), None)
    for _ in range(3):
        ours()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(torch.cuda.default_stream())  # launches go to the legacy default stream (NULL)
    for _ in range(10):
        ours()
    e1.record(torch.cuda.default_stream())
    torch.cuda.synchronize()
    ours_s = e0.elapsed_time(e1) / 10 / 1e3
    # cross-check: both give the same counts
    cnt = Cn.cpu().numpy()[:, :n_bins] // 13
    same = bool(np.array_equal(cnt, out.reshape(nf, n_bins, 3)[:, :, 2].astype(np.int64)))
    return {"rows": int(idx.size), "features": nf, "plain_gpu_call_s": ref_s,
            "plain_gpu_gbs": bytes_alg / ref_s / 1e9, "ours_kernel_s": ours_s, "ours_gbs": bytes_alg / ours_s / 1e9,
            "counts_match": same,
            "note": "plain GPU = reference build_hist_gpu call as shipped (H2D of g/h/idx, FP64 global atomics "
                    "over u16 row-major codes, D2H); ours = tgb_hist_build kernel on resident inputs"}


# ---------------------------------------------------------------- ours
def held_out_ic(pred, panel) -> float:
    """Mean over dates of the Pearson correlation between prediction and target (rows are
    sorted by date with equal cross-sections)."""
    d = int(panel.ts.max()) + 1
    a = pred.reshape(d, -1)
    b = panel.y.reshape(d, -1)
    a = a - a.mean(axis=1, keepdims=True)
    b = b - b.mean(axis=1, keepdims=True)
    den = np.sqrt((a * a).sum(axis=1) * (b * b).sum(axis=1))
    ok = den > 0
    return float(((a * b).sum(axis=1)[ok] / den[ok]).mean())


SERVING_FEATURES = (32, 64, 128, 256)


def serving_trace(n_requests: int, seed: int = 7, rate: float = 20.0, max_rows: int = 4_000_000) -> list[dict]:
    """The serving workload's request trace: Poisson arrivals (mean `rate` per second),
    70% fit / 30% predict; fits of log-uniform 10k..max_rows rows, features uniform in
    SERVING_FEATURES, 20..200 trees, depth 6..8, mse or pairwise (50/50); predicts of
    log-uniform 1k..1M rows against a model fitted earlier in the trace."""
    rng = np.random.default_rng(seed)
    t = 0.0
    reqs: list[dict] = []
    fits: list[int] = []
    for k in range(n_requests):
        t += float(rng.exponential(1.0 / rate))
        if not fits or rng.random() < 0.7:
            rows = int(np.exp(rng.uniform(np.log(10_000), np.log(max_rows))))
            reqs.append(dict(kind="fit", t=t, rows=rows, features=int(rng.choice(SERVING_FEATURES)),
                             trees=int(rng.integers(20, 201)), depth=int(rng.integers(6, 9)),
                             objective="mse" if rng.random() < 0.5 else "pairwise",
                             offset=int(rng.integers(0, max_rows - rows + 1))))
            fits.append(k)
        else:
            model = int(fits[int(rng.integers(0, len(fits)))])
            rows = int(np.exp(rng.uniform(np.log(1_000), np.log(1_000_000))))
            f = reqs[model]["features"]
            reqs.append(dict(kind="predict", t=t, rows=rows, features=f, model=model,
                             offset=int(rng.integers(0, max_rows - rows + 1))))
    return reqs


def run_serving(native, n_requests: int, local: int, budget_bytes: float = 150e9, slots: int = 8) -> dict:
    """Serves the trace through native.Server (tgb_server_*): requests submitted at their
    arrival times, admitted by the device-memory budget, overlapping on the device; p50/p99
    latency from submission to completion and the aggregate trees/s of the fits.  Request
    data are row ranges of one panel_small-generator panel per feature count (the
    generator of the small workload), prepared before the clock starts."""
    from tidegbm_b200 import panels

    reqs = serving_trace(n_requests)
    max_rows = max(r["rows"] + r["offset"] for r in reqs)
    pools = {}
    for f in sorted({r["features"] for r in reqs}):
        n_dates = (max_rows + 249) // 250
        pools[f] = panels.panel_small(n_dates=n_dates, n_entities=250, n_features=f, seed=100 + f)
    srv = native.Server(device=local, budget_bytes=budget_bytes, slots=slots)
    boosters: dict[int, object] = {}
    ids: list[int] = []
    t0 = time.perf_counter()
    for k, r in enumerate(reqs):
        delay = r["t"] - (time.perf_counter() - t0)
        if delay > 0:
            time.sleep(delay)
        p = pools[r["features"]]
        lo, hi = r["offset"], r["offset"] + r["rows"]
        if r["kind"] == "fit":
            b = native.Booster(device=local, n_estimators=r["trees"], max_depth=r["depth"], learning_rate=0.08,
                               horizon=1, objective=r["objective"], pair_splits=False,
                               hist_bits=8 if r["objective"] == "mse" else 0)
            boosters[k] = b
            ids.append(srv.submit_fit(b, p.X[lo:hi], p.y[lo:hi], timestamps=p.ts[lo:hi], entity=p.entity[lo:hi]))
        else:
            rid, _ = srv.submit_predict(boosters[r["model"]], p.X[lo:hi])
            ids.append(rid)
    failed = []
    for rid in ids:
        try:
            srv.wait(rid)
        except native.TideError as e:
            failed.append(str(e)[:120])
    st = srv.stats()
    srv.close()
    fit_trees = sum(r["trees"] for r in reqs if r["kind"] == "fit")
    return {"requests": n_requests, "fits": sum(r["kind"] == "fit" for r in reqs),
            "predicts": sum(r["kind"] == "predict" for r in reqs), "budget_bytes": budget_bytes, "slots": slots,
            "p50_s": st["p50_s"], "p99_s": st["p99_s"], "p50_fit_s": st["p50_fit_s"], "p99_fit_s": st["p99_fit_s"],
            "p50_predict_s": st["p50_predict_s"], "p99_predict_s": st["p99_predict_s"],
            "mean_wait_s": st["mean_wait_s"], "peak_running": st["peak_running"], "peak_bytes": st["peak_bytes"],
            "trees_per_s": fit_trees / st["busy_s"] if st["busy_s"] > 0 else None, "busy_s": st["busy_s"],
            "failed": failed[:5], "n_failed": len(failed),
            "trace": "Poisson 20 req/s, 70% fit (10k..4M rows, 32..256 features, 20..200 trees, depth 6..8, "
                     "mse int8 / pairwise) / 30% predict (1k..1M rows)"}


def run_walkforward(native, local: int, n_dates: int = 8000, n_splits: int = 16, slots: int = 8) -> dict:
    """The batched walk-forward workload: panel_walkforward (n_dates dates, ~425 rows a
    date, 64 features), n_splits expanding folds with embargo 5 (walkforward.py), horizon 5,
    pairwise, depth 6, 100 trees per fold; every fold submitted at once to the serving
    loop, so the folds train concurrently on the device.  Reports the folds' aggregate
    trees/s from the first submission to the last completion."""
    from tidegbm_b200 import panels
    from tidegbm_b200.walkforward import walk_forward_folds

    p = panels.panel_walkforward(n_dates=n_dates)
    folds = walk_forward_folds(p.ts, n_splits, embargo=5, min_train_fraction=0.1)
    srv = native.Server(device=local, slots=slots)
    boosters, ids = [], []
    for train, _ in folds:
        hi = int(train.size)  # rows are time-sorted: the training set is the prefix [0, hi)
        b = native.Booster(device=local, n_estimators=100, max_depth=6, learning_rate=0.08, horizon=5,
                           objective="pairwise", pair_splits=False)
        boosters.append(b)
        ids.append(srv.submit_fit(b, p.X[:hi], p.y[:hi], timestamps=p.ts[:hi], entity=p.entity[:hi]))
    for rid in ids:
        srv.wait(rid)
    st = srv.stats()
    srv.close()
    trees = 100 * len(folds)
    return {"folds": len(folds), "train_rows": [int(tr.size) for tr, _ in folds], "trees": trees,
            "busy_s": st["busy_s"], "trees_per_s": trees / st["busy_s"] if st["busy_s"] > 0 else None,
            "p50_fold_s": st["p50_fit_s"], "p99_fold_s": st["p99_fit_s"], "peak_running": st["peak_running"],
            "mode": "folds as concurrent requests of the serving loop, one stream each"}


def max_over_ranks(values, device):
    """Element-wise max over the ranks of a list of floats (one process per GPU), after a
    barrier; the values unchanged when no process group of several ranks is running."""
    import torch
    import torch.distributed as dist

    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


def run_ours(args) -> None:
    import torch

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta

        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    from tidegbm_b200 import native

    native.lib()
    W, K = max(3, args.warmup), max(1, args.steps)
    p = make_panel(args.dates)
    n, nf = p.X.shape
    # pinned host buffers for the end-to-end call
    cudart = torch.cuda.cudart()
    for arr in (p.X, p.y):
        cudart.cudaHostRegister(arr.ctypes.data, arr.nbytes, 0)

    # Warm-up fit: the full workload with 2 trees (context, module loading, first-touch
    # device allocations at full size).  Its wall time is reported as the cold fit.
    wb = native.Booster(device=local, **dict(PARAMS, n_estimators=2))
    t0 = time.perf_counter()
    wb.fit(p.X, p.y, timestamps=p.ts, entity=p.entity)
    cold_wall = time.perf_counter() - t0
    cold_stats = wb.fit_stats()
    del wb

    n_est = max(PARAMS["n_estimators"], W + K)
    b = native.Booster(device=local, **dict(PARAMS, n_estimators=n_est, timing_from=W, timing_to=W + K))
    launches0 = native.kernel_launches()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        t0 = time.perf_counter()
        b.fit(p.X, p.y, timestamps=p.ts, entity=p.entity)
        e2e_wall = time.perf_counter() - t0
    st = b.fit_stats()
    timed_ms = st["timed_ms"]
    # timed trees are exactly trees W .. W+K-1 (the bench's K steps)
    assert int(st["timed_trees"]) == K, st
    ms_per_tree = timed_ms / st["timed_trees"]
    # the slowest rank sets both whole-job numbers
    ms_max, e2e_wall = max_over_ranks([ms_per_tree, e2e_wall], "cuda")
    value = world * 1000.0 / ms_max
    info = b.info()
    trees = b.trees()
    d2h = sum(t.is_leaf.size * (8 * 4 + 2 * 8) + t.values.nbytes + t.cover.nbytes + t.prefix.nbytes for t in trees)
    h2d = p.X.nbytes + p.y.nbytes
    e2e = {"value": world * n_est / e2e_wall, "unit": "trees/s", "h2d_bytes_per_step": int(h2d / n_est),
           "d2h_bytes_per_step": int(d2h / n_est), "fit_wall_s": e2e_wall, "trees": n_est,
           "breakdown_s": {k: st[k] for k in ("total", "sort", "pre_upload", "bin_fit", "bin_counts", "bin_draws",
                                              "bin_edges", "upload_transform", "alloc", "h2d", "transpose", "prep",
                                              "trees", "download", "host_rng", "goss_producer", "goss_refits")},
           "cold_first_fit": {"trees": 2, "wall_s": cold_wall,
                              "note": "first full-size fit of the process (warm-up): first-touch device allocations",
                              "breakdown_s": {k: cold_stats[k] for k in ("bin_fit", "alloc", "h2d", "trees")}}}
    # Histogram GB/s: short fit with events around every histogram launch.
    bp = native.Booster(device=local, **dict(PARAMS, n_estimators=W + 2, timing_from=W, timing_to=W + 2,
                                             profile_hist=1))
    bp.fit(p.X, p.y, timestamps=p.ts, entity=p.entity)
    sp = bp.fit_stats()
    del bp
    hist_bytes = sp["hist_rows"] * (nf + 16)
    hist_gbs = hist_bytes / (sp["hist_ms"] / 1e3) / 1e9 if sp["hist_ms"] > 0 else None
    pk = peaks()
    traffic = None
    prof = os.path.join(ROOT, "profiles", "hist_traffic.json")
    rows_per_launch = sp["hist_rows"] / max(1, sp["hist_launches"])
    if os.path.exists(prof):
        try:
            # DRAM bytes per histogrammed row from one ncu capture of the root launch of
            # the 4M-row case, scaled to this run's average rows per launch
            traffic = json.load(open(prof))["dram_bytes_per_row"] * rows_per_launch
        except Exception:
            traffic = None
    roof = {"bound": "hbm", "achieved": hist_gbs, "peak": pk["hbm_gbs"], "unit": "GB/s",
            "frac": (hist_gbs / pk["hbm_gbs"]) if hist_gbs else None, "traffic": traffic,
            "peak_source": pk["source"], "kernel": "hist_node_const_kernel",
            "launches": sp["hist_launches"], "avg_launch_ms": sp["hist_ms"] / max(1, sp["hist_launches"]),
            "rows_per_launch": rows_per_launch,
            "algorithmic_bytes": "rows x (128 code bytes + 16 B f64 g,h) per built node",
            "traffic_note": "DRAM bytes per launch: ncu dram__bytes_read+write of the root launch of the 4M-row case "
                            "per row (profiles/hist_traffic.json) x rows per launch here"}
    # int8 precision mode on the same workload: device trees/s, histogram GB/s, and the
    # held-out IC of both modes on a fresh 1M-row panel of the same target function.
    precision = None
    if rank == 0:
        try:
            bq = native.Booster(device=local, **dict(PARAMS, n_estimators=n_est, timing_from=W, timing_to=W + K,
                                                     hist_bits=8))
            bq.fit(p.X, p.y, timestamps=p.ts, entity=p.entity)
            sq = bq.fit_stats()
            bqp = native.Booster(device=local, **dict(PARAMS, n_estimators=W + 2, timing_from=W, timing_to=W + 2,
                                                      profile_hist=1, hist_bits=8))
            bqp.fit(p.X, p.y, timestamps=p.ts, entity=p.entity)
            sqp = bqp.fit_stats()
            del bqp
            q_gbs = sqp["hist_rows"] * (nf + 16) / (sqp["hist_ms"] / 1e3) / 1e9 if sqp["hist_ms"] > 0 else None
            from tidegbm_b200 import panels

            ho = panels.panel_scale(n_dates=500, seed=2, sample_seed=12)
            ic_e, ic_q = held_out_ic(b.raw_predict(ho.X), ho), held_out_ic(bq.raw_predict(ho.X), ho)
            precision = {"mode": "hist_bits=8 (int8 gradients, stochastic rounding, one shared reduction per code)",
                         "value": 1000.0 / (sq["timed_ms"] / sq["timed_trees"]), "unit": "trees/s",
                         "ms_per_step": sq["timed_ms"] / sq["timed_trees"], "hist_gbs": q_gbs,
                         "hist_roofline_frac": (q_gbs / pk["hbm_gbs"]) if q_gbs else None,
                         "held_out_ic_exact": ic_e, "held_out_ic_int8": ic_q, "ic_change": ic_q - ic_e,
                         "held_out": "1M rows (500 dates x 2000): the training panel's target function, new rows "
                                     "(sample seed 12)"}
            del bq
        except Exception as e:
            precision = {"unavailable": f"{type(e).__name__}: {e}"}
    line = {"metric": METRIC, "value": value, "unit": "trees/s", "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64 (int64 fixed-point histograms)", "data": "synthetic",
            "config": {"workload": WORKLOAD, "n_rows": n, "n_features": nf, "n_bins": info["n_bins"],
                       "timed_trees": int(st["timed_trees"]), "l2": "inputs larger than L2 (1.28 GB codes)",
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
            "hist_gbs": hist_gbs, "roofline": roof, "e2e": e2e,
            "gpu_launches": int(st["timed_launches"]),
            "gpu_launches_note": "this library's kernels per K timed trees (+ CUB radix-sort passes inside GOSS)",
            "clocks": clk.summary(), "precision_int8": precision}
    if rank == 0 and not args.no_baselines:
        try:
            line["cpu_baseline"] = {k: v for k, v in ref_cpu_trees_per_s(1, 3).items() if k != "per_tree_s_sample"}
        except Exception as e:
            line["cpu_baseline"] = {"unavailable": f"{type(e).__name__}: {e}"}
        try:
            edges = np.stack([np.pad(b.edges(f), (0, 256 - b.edges(f).size)) for f in range(nf)])
            n_edges = np.array([b.edges(f).size for f in range(nf)])
            rng = np.random.default_rng(0)
            idx = np.sort(rng.choice(n, 3_000_000, replace=False)).astype(np.int32)
            g = rng.standard_normal(n)
            h = np.ones(n)
            line["plain_gpu"] = plain_gpu_hist(native, p.X, edges, n_edges, idx, g, h, info["n_bins"])
        except Exception as e:
            line["plain_gpu"] = {"unavailable": f"{type(e).__name__}: {e}"}
    if rank == 0 and args.walkforward:
        try:
            line["walkforward"] = run_walkforward(native, local)
        except Exception as e:
            line["walkforward"] = {"unavailable": f"{type(e).__name__}: {e}"}
    if rank == 0 and args.serving > 0:
        try:
            line["serving"] = run_serving(native, args.serving, local)
        except Exception as e:
            line["serving"] = {"unavailable": f"{type(e).__name__}: {e}"}
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--dates", type=int, default=5000, help="panel dates (x 2000 rows); default 10M rows")
    ap.add_argument("--no-baselines", action="store_true")
    ap.add_argument("--walkforward", action="store_true",
                    help="also train the batched walk-forward workload's folds concurrently")
    ap.add_argument("--serving", type=int, default=0, metavar="N",
                    help="also serve an N-request trace of the serving workload (p50/p99 latency)")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
