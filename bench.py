#!/usr/bin/env python
"""Benchmark of the device="gpu" TideGBM training hot path on B200.

Headline workload: the 10M-row panel (5,000 dates x 2,000 entities, 128 float32 features:
N(0,1) and log-normal columns, 1% NaN), 255 bins, objective mse, GOSS auto (top 20% /
other 10%), max_depth 8, max_leaves 31 (the reference default), 100 trees; seeded
synthetic data (tidegbm_b200.panels.panel_scale).  A step is one boosting iteration:
gradients, GOSS selection, the tree's histograms, split scans and partitions (batched
waves), post-tree TORB sweep, prediction update, loss.

  value      trees/s over trees W..W+K-1 of one fit through tgb_fit, device time from CUDA
             events on the fit's stream (inputs resident; the 1.28 GB code matrix exceeds
             L2), exact 64-bit fixed-point histograms, batched growth in a CUDA graph
  e2e        trees/s of the whole tgb_fit call from pinned host X/y (binning, H2D,
             transform, every tree, D2H of the trees)
  roofline   histogram kernel: algorithmic bytes (rows x (128 code bytes + 8 B of g, h))
             over the summed CUDA-event time of every histogram launch of a profiled fit
  plain_gpu  the same fit with one split per launch sequence (grow = 0): the plain GPU
             path the batched and quantised ones stand beside; plus the reference's own
             build_hist_gpu against this library's tgb_build_hist_gpu, both called with
             the same per-call copies, and the resident kernels side by side
  precision  int16 / int8 histograms: trees/s, histogram GB/s, the histogram error
             against an FP64 histogram, the held-out IC change
  pairwise   the pairwise workload (0.85M rows, uneven dates, 64 features, 200 trees)
  walkforward  16 purged expanding folds of the 3.4M-row pairwise panel, batched into one
             fit (tgb_fit_batch) against the folds fitted one at a time on the plain path
  serving    a Poisson trace of fit and predict requests through the serving loop
  cpu_baseline  the reference's CPU Booster::fit (oracle/_ref, built from its sources)
             on the headline panel itself, all host cores
The reference arm (--impl reference) times the reference's CPU fit on the headline panel.

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
PAIR_PARAMS = dict(n_estimators=200, learning_rate=0.08, max_depth=6, max_leaves=31, max_bin=255, horizon=1,
                   objective="pairwise", goss=-1, random_state=0, pair_splits=False)
PAIR_WORKLOAD = ("panel_pairwise: 2000 dates x Uniform{50..800} entities (~0.85M rows) x 64 f32 features "
                 "(10% Student-t nu=3 columns, 2% NaN), pairwise, max_depth 6, 200 trees")
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
def ref_cpu_fit(p, params: dict, warmup: int, steps: int) -> dict:
    """The reference's own CPU Booster::fit (oracle/_ref: its sources compiled with -O3
    -fopenmp), n_jobs = 0 (every host core), on panel p as given, for warmup + steps trees.
    Trees/s from its per-iteration hook over the last `steps` trees; binning and set-up are
    outside that range and reported as setup_s.  The reference picks its own histogram
    path: at 10M x 128 its u16 bins (2.56 GB) exceed ooc_bytes (256 MiB), so it runs the
    mmap'd row-major path it ships (cpp/src/booster.cpp:201-229, 382-390)."""
    from oracle import bind

    L = bind.ref_lib()
    L.ref_fit_timed.argtypes = [C.c_void_p] + [np.ctypeslib.ndpointer(np.float64, flags="C")] * 2 + \
        [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, np.ctypeslib.ndpointer(np.float64, flags="C")]
    X = np.ascontiguousarray(p.X, dtype=np.float64)
    h = L.ref_create()
    n_est = warmup + steps
    cfg = dict(params, n_estimators=n_est, n_jobs=0, halo=0)
    for k, v in cfg.items():
        if k == "objective":
            v = 0 if v == "mse" else 5
        if L.ref_set(h, k.encode(), float(v)) != 0:
            raise KeyError(k)
    t_iter = np.zeros(n_est)
    ts = np.ascontiguousarray(p.ts)
    ent = np.ascontiguousarray(p.entity.astype(np.int64))
    groups = ts if cfg.get("objective") == "pairwise" else None
    devnull = os.open(os.devnull, os.O_WRONLY)
    saved = os.dup(2)
    os.dup2(devnull, 2)  # the reference prints one line per iteration with verbose = 1
    try:
        t0 = time.perf_counter()
        rc = L.ref_fit_timed(h, X, np.ascontiguousarray(p.y), p.n, p.n_features, ts.ctypes.data_as(C.c_void_p),
                             None if groups is None else groups.ctypes.data_as(C.c_void_p),
                             ent.ctypes.data_as(C.c_void_p), t_iter)
        wall = time.perf_counter() - t0
    finally:
        os.dup2(saved, 2)
        os.close(devnull)
        os.close(saved)
    L.ref_free(h)
    if rc != 0:
        raise RuntimeError(L.ref_last_error().decode())
    t_start = t_iter[warmup - 1] if warmup > 0 else 0.0
    per_tree = (t_iter[n_est - 1] - t_start) / steps
    setup = t_iter[0] - (t_iter[1] - t_iter[0] if n_est > 1 else 0.0)
    return {"value": 1.0 / per_tree, "unit": "trees/s", "cores": os.cpu_count(), "kind": "reference",
            "per_tree_s": per_tree, "setup_s": setup, "fit_wall_s": wall, "rows": p.n, "features": p.n_features,
            "trees": n_est}


def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    try:
        from oracle import bind

        if not bind.ref_available():
            raise RuntimeError("reference core not built (oracle/_ref)")
        W, K = max(1, args.warmup), max(1, args.steps)
        p = make_panel(args.dates)
        r = ref_cpu_fit(p, PARAMS, W, K)
    except Exception as e:  # pragma: no cover
        print(json.dumps({"impl": "reference", "unavailable": f"{type(e).__name__}: {e}"}))
        return
    sample = (f"reference Booster::fit (oracle/_ref, -O3 -fopenmp, n_jobs=0, {r['cores']} threads) on the full "
              f"{r['rows']} x {r['features']} panel, {W} warm-up + {K} timed trees via its per-iteration hook "
              f"({r['per_tree_s']:.3f} s/tree; binning and set-up {r['setup_s']:.1f} s outside the range); as "
              f"shipped: mmap'd u16 bins and row-major histograms above ooc_bytes")
    line = {"impl": "reference", "metric": METRIC, "value": r["value"], "unit": "trees/s", "n_gpus": args.gpus,
            "steps": K, "warmup": W, "ms_per_step": 1000.0 / r["value"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "parallelism": "host OpenMP"},
            "cpu_baseline": {"value": r["value"], "unit": "trees/s", "cores": r["cores"], "kind": "reference",
                             "sample": sample},
            "e2e": {"value": r["value"], "unit": "trees/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


# ---------------------------------------------------------------- plain GPU: the seam
def seam_hist(native, b, X32, n_bins) -> dict | None:
    """The reference's build_hist_gpu (cpp/src/histogram_cuda.cu:81-167, built for sm_100a)
    against this library's drop-in for the same seam (tgb_build_hist_gpu), both called as
    the reference calls it: host u16 codes (uploaded once), host idx, g, h copied per call,
    the FP64 {g, h, c} histogram copied back.  Plus the two resident kernels side by side
    (this library's tgb_hist_build against the reference kernel's time without copies is
    not separable: its call is one unit).  Root-sized row set: 3M of the 10M rows."""
    import torch
    from oracle import bind

    if not os.path.exists(bind.REF_CUDA_SO):
        return None
    R = C.CDLL(bind.REF_CUDA_SO)
    R.refgpu_build_hist.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int,
                                    C.c_int, C.c_void_p]
    n, nf = X32.shape
    stride = (nf + 15) // 16 * 16
    codes = device_codes(native, b, X32)
    xb16 = np.ascontiguousarray(codes[:, :nf].cpu().numpy().astype(np.uint16))
    rng = np.random.default_rng(0)
    idx = np.sort(rng.choice(n, 3_000_000, replace=False)).astype(np.int32)
    g = rng.standard_normal(n)
    h = np.ones(n)
    bytes_alg = idx.size * (nf + 8)
    out_ref = np.zeros(nf * n_bins * 3)
    args = (xb16.ctypes.data_as(C.c_void_p), nf, idx.ctypes.data_as(C.c_void_p), idx.size,
            g.ctypes.data_as(C.c_void_p), h.ctypes.data_as(C.c_void_p), n_bins, n, out_ref.ctypes.data_as(C.c_void_p))
    if R.refgpu_build_hist(*args) != 0:  # first call uploads the code matrix once
        return None
    reps = 3
    t0 = time.perf_counter()
    for _ in range(reps):
        R.refgpu_build_hist(*args)
    ref_s = (time.perf_counter() - t0) / reps
    # the same seam through this library (same host buffers, same per-call copies)
    sb = native.Booster(device=0)
    L = native.lib()
    out = np.zeros(nf * n_bins * 3)
    sargs = (sb._h, xb16.ctypes.data_as(C.c_void_p), nf, idx.ctypes.data_as(C.c_void_p), idx.size,
             g.ctypes.data_as(C.c_void_p), h.ctypes.data_as(C.c_void_p), n_bins, n, out.ctypes.data_as(C.c_void_p))
    native.check(L.tgb_build_hist_gpu(*sargs))  # uploads the code matrix once
    t0 = time.perf_counter()
    for _ in range(reps):
        native.check(L.tgb_build_hist_gpu(*sargs))
    seam_s = (time.perf_counter() - t0) / reps
    same = bool(np.array_equal(out.reshape(nf, n_bins, 3)[:, :, 2], out_ref.reshape(nf, n_bins, 3)[:, :, 2]))
    gerr = float(np.max(np.abs(out.reshape(nf, n_bins, 3)[:, :, 0] - out_ref.reshape(nf, n_bins, 3)[:, :, 0])))
    # resident: this library's kernel on device rows, g, h
    rt = torch.from_numpy(idx).cuda()
    gt, ht = torch.from_numpy(g).cuda(), torch.from_numpy(h).cuda()
    G = torch.zeros((nf, 256), dtype=torch.int64, device="cuda")
    H = torch.zeros_like(G)
    Cn = torch.zeros((nf, 256), dtype=torch.int32, device="cuda")
    gs = 61 - (int(np.floor(np.log2(np.abs(g[idx]).max()))) + 1) - int(np.ceil(np.log2(idx.size)))
    hs = 61 - (int(np.floor(np.log2(np.abs(h[idx]).max()))) + 1) - int(np.ceil(np.log2(idx.size)))

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
    return {"rows": int(idx.size), "features": nf,
            "seam": {"reference_build_hist_gpu_s": ref_s, "tgb_build_hist_gpu_s": seam_s,
                     "speedup": ref_s / seam_s, "counts_match": same, "max_abs_g_diff": gerr,
                     "note": "both calls as the reference makes them: H2D of g, h, idx and D2H of the FP64 "
                             "{g, h, c} histogram per call; code matrix uploaded once"},
            "resident_kernel": {"tgb_hist_build_s": ours_s, "gbs": bytes_alg / ours_s / 1e9,
                                "note": "resident inputs, exact 64-bit histogram of the same rows"}}


def device_codes(native, b, X32):
    """Row-major uint8 codes of X32 on the device, with booster b's fitted edges."""
    import torch

    n, nf = X32.shape
    stride = (nf + 15) // 16 * 16
    E = np.full((nf, 256), np.inf, dtype=np.float32)
    ne = np.zeros(nf, np.int32)
    for f in range(nf):
        e = b.edges(f)
        ne[f] = e.size
        e32 = e.astype(np.float32)
        with np.errstate(invalid="ignore"):
            low = e32.astype(np.float64) < e
        e32[low] = np.nextafter(e32[low], np.float32(np.inf))
        E[f, : e.size] = e32
    Xd = torch.from_numpy(X32).cuda()
    Ed = torch.from_numpy(E).cuda()
    ned = torch.from_numpy(ne).cuda()
    codes = torch.empty((n, stride), dtype=torch.uint8, device="cuda")
    native.check(native.lib().tgb_bin_transform(C.c_void_p(Xd.data_ptr()), 0, n, nf, C.c_void_p(Ed.data_ptr()),
                                                C.c_void_p(ned.data_ptr()), C.c_void_p(codes.data_ptr()), stride,
                                                None))
    torch.cuda.synchronize()
    del Xd
    return codes


def hist_error(native, codes, nf, rows, g, h, bits) -> dict:
    """Histogram of `rows` through the fit's payload and histogram kernels in precision mode
    `bits` (tgb_hist_build_quantized) against an FP64 histogram of the same rows (numpy):
    the largest bin error over every (feature, bin), relative to the rows' sum of |g|
    (sum of h for H), the scale a split gain sees."""
    import torch

    stride = codes.shape[1]
    rt = torch.from_numpy(rows).cuda()
    gt = torch.from_numpy(g).cuda()
    ht = None if h is None else torch.from_numpy(h).cuda()
    G = torch.zeros((nf, 256), dtype=torch.int64, device="cuda")
    H = torch.zeros_like(G)
    Cn = torch.zeros((nf, 256), dtype=torch.int32, device="cuda")
    sc = np.zeros(2)
    native.check(native.lib().tgb_hist_build_quantized(
        C.c_void_p(codes.data_ptr()), stride, nf, C.c_void_p(rt.data_ptr()), rows.size, C.c_void_p(gt.data_ptr()),
        None if ht is None else C.c_void_p(ht.data_ptr()), bits, 977, C.c_void_p(G.data_ptr()),
        C.c_void_p(H.data_ptr()), C.c_void_p(Cn.data_ptr()), sc.ctypes.data_as(C.c_void_p), None))
    torch.cuda.synchronize()
    Gq = G.cpu().numpy() * sc[0]
    Hq = H.cpu().numpy() * sc[1]
    cod = codes[:, :nf].cpu().numpy()[rows]
    gr = g[rows]
    hr = np.ones(rows.size) if h is None else h[rows]
    eg = eh = 0.0
    for f in range(nf):
        Gf = np.bincount(cod[:, f], weights=gr, minlength=256)
        Hf = np.bincount(cod[:, f], weights=hr, minlength=256)
        eg = max(eg, float(np.max(np.abs(Gq[f] - Gf))))
        eh = max(eh, float(np.max(np.abs(Hq[f] - Hf))))
    return {"max_bin_err_g_rel": eg / float(np.abs(gr).sum()), "max_bin_err_h_rel": eh / float(hr.sum()),
            "rows": int(rows.size)}


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




def timed_fit(native, local, p, params, W, K):
    """One fit of max(T, W+K) trees with the timed range [W, W+K): trees/s from CUDA events,
    the fit's wall time, its stats; and the booster."""
    n_est = max(params.get("n_estimators", 100), W + K)
    b = native.Booster(device=local, **dict(params, n_estimators=n_est, timing_from=W, timing_to=W + K))
    t0 = time.perf_counter()
    b.fit(p.X, p.y, timestamps=p.ts, entity=p.entity)
    wall = time.perf_counter() - t0
    st = b.fit_stats()
    return b, st, wall, 1000.0 * st["timed_trees"] / st["timed_ms"]


def profiled_hist(native, local, p, params, W, nf, payload_bytes):
    """Histogram GB/s of a short fit with CUDA events around every histogram launch:
    algorithmic bytes = rows histogrammed x (code bytes + g/h payload bytes)."""
    bp = native.Booster(device=local, **dict(params, n_estimators=W + 2, timing_from=W, timing_to=W + 2,
                                             profile_hist=1))
    bp.fit(p.X, p.y, timestamps=p.ts, entity=p.entity)
    sp = bp.fit_stats()
    gbs = sp["hist_rows"] * (nf + payload_bytes) / (sp["hist_ms"] / 1e3) / 1e9 if sp["hist_ms"] > 0 else None
    return {"gbs": gbs, "launches": sp["hist_launches"], "hist_ms": sp["hist_ms"], "rows": sp["hist_rows"],
            "trees": 2, "avg_launch_ms": sp["hist_ms"] / max(1, sp["hist_launches"]),
            "rows_per_launch": sp["hist_rows"] / max(1, sp["hist_launches"])}


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



def run_walkforward(native, local, W: int, n_dates: int = 8000, n_splits: int = 16) -> dict:
    """The batched walk-forward workload: panel_walkforward (8,000 dates, ~425 rows a date,
    64 features), 16 expanding folds with embargo 5 (walkforward.py), horizon 5, pairwise,
    depth 6, 100 trees per fold.  Batched: every fold in one tgb_fit_batch (all folds' trees
    grow in the same wave launches, one CUDA graph per tree round), exact and with int16 /
    int8 histograms.  Plain: the folds one at a time on the plain path (grow = 0).  Trees/s
    over the folds' trees from CUDA events on the fit stream, trees W.. of every fold, and
    the mean held-out IC over the folds' test dates."""
    from tidegbm_b200 import panels
    from tidegbm_b200.walkforward import walk_forward_folds

    p = panels.panel_walkforward(n_dates=n_dates)
    folds = walk_forward_folds(p.ts, n_splits, embargo=5, min_train_fraction=0.1)
    his = [int(tr.size) for tr, _ in folds]  # rows are time-sorted: training set = prefix [0, hi)
    T = 100
    base = dict(n_estimators=T, max_depth=6, learning_rate=0.08, horizon=5, objective="pairwise",
                pair_splits=False, goss=-1)

    def fold_ic(bs):
        ics = []
        for b, (_, te) in zip(bs, folds):
            pr = b.raw_predict(p.X[te])
            ts = p.ts[te]
            for d in np.unique(ts):
                m = ts == d
                a, y = pr[m] - pr[m].mean(), p.y[te][m] - p.y[te][m].mean()
                den = np.sqrt((a * a).sum() * (y * y).sum())
                if den > 0:
                    ics.append((a * y).sum() / den)
        return float(np.mean(ics))

    out = {"folds": len(folds), "train_rows": his, "trees_per_fold": T}

    def batched(extra):
        bs = [native.Booster(device=local, **dict(base, **extra)) for _ in his]
        bs[0].set_config(timing_from=W, timing_to=T)
        t0 = time.perf_counter()
        native.Booster.fit_batch(bs, [p.X[:h] for h in his], [p.y[:h] for h in his], [p.ts[:h] for h in his],
                                 [p.entity[:h] for h in his])
        wall = time.perf_counter() - t0
        st = bs[0].fit_stats()
        return bs, {"trees_per_s": 1000.0 * st["timed_trees"] / st["timed_ms"], "wall_s": wall,
                    "timed_trees": st["timed_trees"], "graph_used": st["graph_used"]}

    bs, r = batched({})
    r["held_out_ic"] = fold_ic(bs)
    out["batched_exact"] = r
    del bs
    for bits in (16, 8):
        bs, r = batched({"hist_bits": bits})
        r["held_out_ic"] = fold_ic(bs)
        out[f"batched_int{bits}"] = r
        del bs
    # plain: one fold at a time, one split per launch sequence
    tot_ms, tot_trees, t0 = 0.0, 0, time.perf_counter()
    pb = []
    for h in his:
        b = native.Booster(device=local, **dict(base, grow=0, timing_from=W, timing_to=T))
        b.fit(p.X[:h], p.y[:h], timestamps=p.ts[:h], entity=p.entity[:h])
        st = b.fit_stats()
        tot_ms += st["timed_ms"]
        tot_trees += st["timed_trees"]
        pb.append(b)
    plain = {"trees_per_s": 1000.0 * tot_trees / tot_ms, "wall_s": time.perf_counter() - t0,
             "held_out_ic": fold_ic(pb)}
    out["plain_one_at_a_time"] = plain
    for k in ("batched_exact", "batched_int16", "batched_int8"):
        out[k]["vs_plain"] = out[k]["trees_per_s"] / plain["trees_per_s"]
        out[k]["ic_change_vs_plain"] = out[k]["held_out_ic"] - plain["held_out_ic"]
    return out


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
    from tidegbm_b200 import native, panels

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

    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        b, st, e2e_wall, _ = timed_fit(native, local, p, PARAMS, W, K)
    n_est = max(PARAMS["n_estimators"], W + K)
    assert int(st["timed_trees"]) == K, st
    ms_per_tree = st["timed_ms"] / st["timed_trees"]
    # the slowest rank sets both whole-job numbers
    ms_max, e2e_wall = max_over_ranks([ms_per_tree, e2e_wall], "cuda")
    value = world * 1000.0 / ms_max
    info = b.info()
    trees = b.trees()
    d2h = sum(t.is_leaf.size * (8 * 4 + 2 * 8) + t.values.nbytes + t.cover.nbytes + t.prefix.nbytes for t in trees)
    h2d = p.X.nbytes + p.y.nbytes
    kernels_per_tree = None
    if st.get("timed_selects"):
        # per tree: gradients, GOSS (keys, 4+1 CUB passes, fix-up, mark, count, scatter), set-up,
        # payload, post-tree sweep: 20 launches; waves: 3 + 5 x (selects - 1) kernels
        kernels_per_tree = 20 + 3 + 5 * (st["timed_selects"] / K - 1)
    e2e = {"value": world * n_est / e2e_wall, "unit": "trees/s", "h2d_bytes_per_step": int(h2d / n_est),
           "d2h_bytes_per_step": int(d2h / n_est), "fit_wall_s": e2e_wall, "trees": n_est,
           "breakdown_s": {k: st[k] for k in ("total", "sort", "pre_upload", "bin_fit", "bin_counts", "bin_draws",
                                              "bin_edges", "upload_transform", "alloc", "h2d", "transpose", "prep",
                                              "driver", "trees", "driver_free", "finish_sync", "download", "release",
                                              "host_rng",
                                              "goss_producer", "goss_refits")},
           "cold_first_fit": {"trees": 2, "wall_s": cold_wall,
                              "note": "first full-size fit of the process (warm-up): first-touch device allocations",
                              "breakdown_s": {k: cold_stats[k] for k in ("bin_fit", "alloc", "h2d", "trees")}}}
    # Histogram GB/s: a short fit with events around every histogram launch.
    hp = profiled_hist(native, local, p, PARAMS, W, nf, 8)
    pk = peaks()
    traffic = None
    prof = os.path.join(ROOT, "profiles", "hist_traffic.json")
    if os.path.exists(prof):
        try:
            # DRAM bytes per histogrammed row from one ncu capture, scaled to this run's rows
            # per launch (traffic grows with the rows a launch histograms)
            traffic = json.load(open(prof))["dram_bytes_per_row"] * hp["rows_per_launch"]
        except Exception:
            traffic = None
    roof = {"bound": "hbm", "achieved": hp["gbs"], "peak": pk["hbm_gbs"], "unit": "GB/s",
            "frac": (hp["gbs"] / pk["hbm_gbs"]) if hp["gbs"] else None, "traffic": traffic,
            "peak_source": pk["source"], "kernel": "wave_hist_kernel (exact, constant hessian)",
            "launches": hp["launches"], "avg_launch_ms": hp["avg_launch_ms"], "rows_per_launch": hp["rows_per_launch"],
            "algorithmic_bytes": "rows x (128 code bytes + 8 B of g, h) per histogrammed node",
            "traffic_note": "DRAM bytes per launch: ncu dram__bytes_read+write per histogrammed row "
                            "(profiles/hist_traffic.json) x rows per launch here"}
    line = {"metric": METRIC, "value": value, "unit": "trees/s", "n_gpus": world, "steps": K, "warmup": W,
            "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64 (int64 fixed-point histograms)", "data": "synthetic",
            "config": {"workload": WORKLOAD, "n_rows": n, "n_features": nf, "n_bins": info["n_bins"],
                       "timed_trees": int(st["timed_trees"]), "l2": "inputs larger than L2 (1.28 GB codes)",
                       "growth": "batched waves in a CUDA graph" if st.get("graph_used") else "batched waves",
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
            "hist_gbs": hp["gbs"], "roofline": roof, "e2e": e2e,
            "gpu_launches": int(round(kernels_per_tree * K)) if kernels_per_tree else int(st["timed_launches"]),
            "gpu_launches_note": "this library's kernels in the K timed trees (the CUB radix-sort passes of GOSS "
                                 "included); the waves of a tree run as one graph launch of 3 + 5 x (selects - 1) "
                                 "kernels, selects counted on the device",
            "clocks": clk.summary()}
    extra_ok = rank == 0 and not args.quick

    def section(name, fn):
        if not extra_ok:
            return
        try:
            line[name] = fn()
        except Exception as e:  # a failing section does not lose the headline line
            line[name] = {"unavailable": f"{type(e).__name__}: {e}"}

    # the plain GPU path: one split per launch sequence, same workload
    def plain():
        pb, pst, pwall, pv = timed_fit(native, local, p, dict(PARAMS, grow=0), W, K)
        php = profiled_hist(native, local, p, dict(PARAMS, grow=0), W, nf, 8)
        same = all(np.array_equal(a.feature, c.feature) and np.array_equal(a.threshold, c.threshold)
                   for a, c in zip(pb.trees(), trees))
        out = {"value": pv, "unit": "trees/s", "ms_per_step": 1000.0 / pv, "hist_gbs": php["gbs"],
               "hist_launches_per_tree": php["launches"] / 2, "trees_identical_to_batched": same,
               "batched_vs_plain": value / pv,
               "path": "grow = 0: one split per launch sequence (scan, partition, smaller-child histogram)"}
        try:
            out.update(seam_hist(native, b, p.X, info["n_bins"]) or {})
        except Exception as e:
            out["seam"] = {"unavailable": f"{type(e).__name__}: {e}"}
        return out

    section("plain_gpu", plain)

    # precision modes on the same workload, the held-out IC of each on a fresh 1M-row panel
    def precision():
        ho = panels.panel_scale(n_dates=500, seed=2, sample_seed=12)
        ic_exact = held_out_ic(b.raw_predict(ho.X), ho)
        codes = device_codes(native, b, p.X)
        rng = np.random.default_rng(5)
        rows = np.sort(rng.choice(n, 3_000_000, replace=False)).astype(np.int32)
        g0 = (np.mean(p.y) - p.y).astype(np.float64)  # tree 0's mse gradient
        out = {"held_out": "1M rows (500 dates x 2000) of the training panel's target function (sample seed 12)",
               "held_out_ic_exact": ic_exact,
               "error_rows": "3M sampled rows (the GOSS root's size) with tree 0's gradient, against an FP64 "
                             "histogram of the same rows",
               "exact": hist_error(native, codes, nf, rows, g0, None, 0)}
        plain_v = line.get("plain_gpu", {}).get("value")
        for bits in (16, 8):
            qb, qst, _, qv = timed_fit(native, local, p, dict(PARAMS, hist_bits=bits), W, K)
            qh = profiled_hist(native, local, p, dict(PARAMS, hist_bits=bits), W, nf, 4 if bits == 16 else 2)
            ic_q = held_out_ic(qb.raw_predict(ho.X), ho)
            out[f"int{bits}"] = {"value": qv, "unit": "trees/s", "ms_per_step": 1000.0 / qv, "hist_gbs": qh["gbs"],
                                 "hist_roofline_frac": qh["gbs"] / pk["hbm_gbs"] if qh["gbs"] else None,
                                 "held_out_ic": ic_q, "ic_change": ic_q - ic_exact,
                                 "hist_error": hist_error(native, codes, nf, rows, g0, None, bits),
                                 "batched_quantised_vs_plain": (qv / plain_v) if plain_v else None,
                                 "algorithmic_bytes": f"rows x (128 code bytes + {4 if bits == 16 else 2} B)"}
            del qb
        del codes
        return out

    section("precision", precision)

    def pairwise():
        pp = panels.panel_pairwise(n_dates=2000)
        pb, pst, pwall, pv = timed_fit(native, local, pp, PAIR_PARAMS, W, K)
        php = profiled_hist(native, local, pp, PAIR_PARAMS, W, pp.n_features, 8)
        lb, lst, lwall, lv = timed_fit(native, local, pp, dict(PAIR_PARAMS, grow=0), W, K)
        out = {"workload": PAIR_WORKLOAD, "rows": pp.n, "value": pv, "unit": "trees/s", "e2e_fit_wall_s": pwall,
               "hist_gbs": php["gbs"], "hist_roofline_frac": php["gbs"] / pk["hbm_gbs"] if php["gbs"] else None,
               "plain_value": lv, "batched_vs_plain": pv / lv}
        # histogram error of the precision modes on tree 0's pairwise gradients (all rows)
        import torch

        codes = device_codes(native, pb, pp.X)
        L = native.lib()
        yt = torch.from_numpy(pp.y).cuda()
        pr = torch.zeros_like(yt)
        gt, ht = torch.zeros_like(yt), torch.zeros_like(yt)
        _, starts, lens = np.unique(pp.ts, return_index=True, return_counts=True)
        rs, rl = torch.from_numpy(starts.astype(np.int32)).cuda(), torch.from_numpy(lens.astype(np.int32)).cuda()
        native.check(L.tgb_grad_pairwise(C.c_void_p(yt.data_ptr()), C.c_void_p(pr.data_ptr()),
                                         C.c_void_p(rs.data_ptr()), C.c_void_p(rl.data_ptr()), None, starts.size,
                                         pp.n, C.c_void_p(gt.data_ptr()), C.c_void_p(ht.data_ptr()), None))
        g0, h0 = gt.cpu().numpy(), ht.cpu().numpy()
        rows = np.arange(pp.n, dtype=np.int32)
        out["hist_error"] = {f"int{bits}" if bits else "exact": hist_error(native, codes, pp.n_features, rows, g0,
                                                                           h0, bits) for bits in (0, 16, 8)}
        for bits in (16, 8):
            qb, _, _, qv = timed_fit(native, local, pp, dict(PAIR_PARAMS, hist_bits=bits), W, K)
            out[f"int{bits}_value"] = qv
            out[f"int{bits}_vs_plain"] = qv / lv
        try:
            r = ref_cpu_fit(pp, PAIR_PARAMS, 1, 2)
            out["cpu_baseline"] = {k: r[k] for k in ("value", "unit", "cores", "kind", "per_tree_s", "setup_s")}
        except Exception as e:
            out["cpu_baseline"] = {"unavailable": f"{type(e).__name__}: {e}"}
        return out

    section("pairwise", pairwise)
    section("walkforward", lambda: run_walkforward(native, local, W))
    if args.serving > 0:
        section("serving", lambda: run_serving(native, args.serving, local))
    if rank == 0 and not args.no_baselines:
        try:
            r = ref_cpu_fit(p, PARAMS, 1, 1)
            line["cpu_baseline"] = {
                "value": r["value"], "unit": "trees/s", "cores": r["cores"], "kind": "reference",
                "sample": f"reference Booster::fit (oracle/_ref, -O3 -fopenmp, n_jobs=0) on the full {r['rows']} x "
                          f"{r['features']} panel, 1 warm-up + 1 timed tree via its per-iteration hook "
                          f"({r['per_tree_s']:.2f} s/tree; binning and set-up {r['setup_s']:.1f} s outside the "
                          f"range); mmap'd u16 bins and row-major histograms, as the reference ships them at "
                          f"this size"}
        except Exception as e:
            line["cpu_baseline"] = {"unavailable": f"{type(e).__name__}: {e}"}
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
    ap.add_argument("--quick", action="store_true", help="headline line only (no side workloads)")
    ap.add_argument("--serving", type=int, default=40, metavar="N",
                    help="serve an N-request trace of the serving workload (p50/p99 latency); 0: skip")
    ap.add_argument("--graph", type=int, default=1, choices=[0, 1],
                    help="0: host-driven waves, every kernel its own launch (for per-kernel launch lists)")
    ap.add_argument("--hist-stage", type=int, default=1, choices=[0, 1],
                    help="0: histogram code rows loaded lane by lane instead of staged by TMA gathers")
    ap.add_argument("--wave-expand", type=int, default=None, metavar="K",
                    help="expansions a wave may plan (the library's default when absent; 0: uncapped)")
    args = ap.parse_args()
    if args.wave_expand is not None:
        PARAMS["wave_expand"] = args.wave_expand
    if args.graph == 0:
        PARAMS["graph"] = 0
    if args.hist_stage == 0:
        PARAMS["hist_stage"] = 0
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
