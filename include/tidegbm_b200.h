/* tidegbm_b200 — C ABI of the B200 (sm_100a) implementation of TideGBM's GBDT
 * training hot path: quantile binning to uint8 codes, per-node gradient/hessian
 * histograms, best-split scan, stable row partitioning, MSE and within-date
 * pairwise gradients, and the per-tree TORB sweep.
 *
 * Conventions (those of the reference C API, cpp/include/tidegbm/c_api.h:9-28 and
 * cpp/src/c_api.cpp:12-18): every function returns 0 on success and -1 on error,
 * with the message in thread-local storage read by tgb_last_error(); no C++
 * exception crosses the ABI; the caller owns every buffer it passes.  Host
 * pointers are plain host memory (pinned memory is faster for the fit upload);
 * "device" pointers are CUDA device memory of the current device and `stream` is
 * a cudaStream_t (NULL = legacy default stream).
 *
 * x_dtype: 0 = float32, 1 = float64, row-major n x n_features.
 */
#ifndef TIDEGBM_B200_H
#define TIDEGBM_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define TGB_API __attribute__((visibility("default")))
#else
#define TGB_API
#endif

typedef struct tgb_booster tgb_booster;

/* Message of the last failed call on this thread (tide_last_error, c_api.cpp:18). */
TGB_API const char* tgb_last_error(void);

/* Number of kernel launches issued by this library in this process (for audits). */
TGB_API long long tgb_kernel_launches(void);

/* ---- Booster level: the device="gpu" Booster (cpp/include/tidegbm/booster.hpp:22-72) ---- */

/* tide_create (c_api.cpp:20-28); one booster owns one CUDA stream and its device
 * buffers on `device` — no process-global state (unlike GpuHistState,
 * cpp/src/histogram_cuda.cu:76-79). */
TGB_API int tgb_booster_create(int device, tgb_booster** out);
/* tide_free (c_api.cpp:30). */
TGB_API void tgb_booster_free(tgb_booster* b);

/* tide_set_int / tide_set_double (c_api.cpp:32-70), extended to every Config key the
 * GPU path reads (cpp/include/tidegbm/config.hpp:12-76).  Unknown keys return -1.
 * Int keys of this library's own: "hist_bits" = 0 (default: exact 64-bit fixed-point
 * histograms, results match the reference), 16 or 8 (gradients and hessians
 * stochastically rounded to int16 / int8 per tree, summed exactly in 32-bit words: fewer
 * shared reductions per code, an approximate split search; leaf values stay exact);
 * "grow" = 1 (default: batched waves, many leaves per launch) or 0 (one split per
 * launch sequence; hist_bits 0, or 8 with objective mse); "graph" = 1 (default: a tree's
 * waves run as one CUDA graph with a device-side loop) or 0 (enqueued by the host);
 * "hist_tune" = 1 (default: the histogram's launch shape is tuned on the first tree and
 * kept for the process) or 0; "wave_expand" = 8 (default: a wave plans the 8 best leaves
 * ranked within the splits left), k > 0 (the k best) or 0 (all of them; the same trees
 * whatever the value); "hist_stage" =
 * 1 (default: the constant-hessian histograms stage code rows in shared memory with TMA
 * gathers) or 0 (each lane loads its rows' codes from global memory; the same results). */
TGB_API int tgb_set_int(tgb_booster* b, const char* key, long long value);
TGB_API int tgb_set_double(tgb_booster* b, const char* key, double value);
/* String keys the reference only sets through pybind (bindings.cpp:78, 115-125):
 * "objective" in {"mse","l2","regression","auto","pairwise","lambdarank"}, "device". */
TGB_API int tgb_set_str(tgb_booster* b, const char* key, const char* value);

/* Booster::fit (cpp/src/booster.cpp:231-742) with device=="gpu", the entry
 * tide_fit (c_api.cpp:72-86) reaches.  X: host, row-major; y: host f64 [n];
 * timestamps: host int64 [n] (required unless iid_mode; rank groups of the pairwise
 * objective); entity: host int64 [n] or NULL (sort key after the timestamp). */
TGB_API int tgb_fit(tgb_booster* b, const void* X, int x_dtype, const double* y, int n, int n_features,
            const long long* timestamps, const long long* entity);

/* Several Booster::fit calls at once (the folds of a walk-forward split, or any set of
 * fits of one feature count on one device): booster k is fitted on (X[k], y[k], n[k],
 * timestamps[k], entity[k]) exactly as tgb_fit would fit it, while the trees of all of
 * them grow in the same batched launches (the boosters' "grow" key must be 1, their
 * "hist_bits" and objective alike, n_estimators equal; at most 64 boosters).  Each
 * result equals the booster's own tgb_fit.  timestamps / entity may be NULL as in tgb_fit. */
TGB_API int tgb_fit_batch(tgb_booster* const* boosters, int n_boosters, const void* const* X, int x_dtype,
                          const double* const* y, const int* n, int n_features, const long long* const* timestamps,
                          const long long* const* entity);

/* Booster::predict_raw (cpp/src/booster.cpp:805-811): init_score + lr * sum of tree
 * values, computed on the device.  X host, out host f64 [n]. */
TGB_API int tgb_predict_raw(tgb_booster* b, const void* X, int x_dtype, int n, int n_features, double* out);

/* Fitted model read-back: the Tree / Node fields the .tgbm format serialises
 * (cpp/src/serialize.cpp:120-143) and the booster fields around them. */
TGB_API int tgb_model_info(tgb_booster* b, int* n_trees, int* n_bins, int* n_buckets, double* init_score);
TGB_API int tgb_init_prefix(tgb_booster* b, double* out);  /* n_buckets values */
TGB_API int tgb_evals_train(tgb_booster* b, double* out);  /* n_trees values (evals.train) */
TGB_API int tgb_tree_n_nodes(tgb_booster* b, int tree);
/* inodes[8k] = {is_leaf, feature, threshold_bin, left, right, missing_go_left, n_samples,
 * depth}; fnodes[2k] = {value, gain}; values/cover per node; prefix n_buckets x n_nodes. */
TGB_API int tgb_tree_export(tgb_booster* b, int tree, int* inodes, double* fnodes, double* values, int* cover,
                    double* prefix);
/* Split type of every node (0 axis, 1 pair, 2 categorical; SplitType,
 * cpp/include/tidegbm/types.hpp:25), the second feature of pair splits (-1 otherwise;
 * Node::feature2) and, per node, the 256-bit left mask of a categorical split
 * (cat_left[4k .. 4k+3], bit b: code b goes left; Node::cat_left,
 * cpp/include/tidegbm/tree.hpp:24).  Any output may be NULL. */
TGB_API int tgb_tree_export_split(tgb_booster* b, int tree, int* types, int* feature2, unsigned long long* cat_left);

/* Categorical features of the next fit (Booster::fit's is_cat, cpp/src/booster.cpp:246-247):
 * is_cat[f] != 0 marks feature f; NULL or n_features 0: every feature numeric.  Their codes
 * come from a vocabulary (binning.cpp:47-84, keys "cat_min_count" and "max_bin"), their
 * splits send a ranked prefix of categories left (histogram.cpp:195-244, key "cat_smooth").
 * Needs "grow" = 1.  The flags stay with the fitted model for predict. */
TGB_API int tgb_set_categorical(tgb_booster* b, const int* is_cat, int n_features);

/* Bin edges of feature f (Binner::edges, cpp/include/tidegbm/binning.hpp:15); returns
 * the count, copies them when out != NULL. */
TGB_API int tgb_edges(tgb_booster* b, int f, double* out);
/* Breakdown of the last fit (18 values): wall seconds {total, sort, bin_fit,
 * upload+transform, trees, download, host_rng}, kernel_launches, then the timed range
 * set by the int keys "timing_from" / "timing_to" (trees [from, to); to < 0: through the
 * last tree) and "profile_hist":
 * {device ms (CUDA events), trees, kernel launches, histogram-kernel ms, histogram
 * launches, rows histogrammed}, then wall seconds {device allocation, X/y H2D,
 * column-major copy, GOSS draw producer}. */
TGB_API int tgb_fit_stats(tgb_booster* b, double* out18);
/* One value of the last fit's breakdown by name (wall seconds): "total", "bin_fit",
 * "bin_counts", "bin_draws", "bin_edges" (the device binner's stages), "h2d", "alloc",
 * "transpose", "trees", "pre_upload" / "prep" (host set-up before the upload / before
 * the tree loop), "goss_refits" (1 when the fit was repeated with the full 64-bit GOSS
 * sort), "timed_selects" (wave selects run in the timed range: with batched growth a tree
 * runs 3 + 5 x (selects - 1) kernels in its waves), "graph_used" (1 when the waves ran as
 * a CUDA graph), "hist_cluster" / "hist_clusters" (the tuned launch shape of the
 * histogram: CTAs per cluster, clusters launched), "driver" (set-up of the batched
 * growth), "driver_free" (its release after the tree loop), "finish_sync" (from the tree
 * loop's end to the GOSS sampler's stop), "release" (the fit's buffers back to the pool),
 * "expansions" (leaves whose children were histogrammed, over all trees; a tree commits
 * max_leaves - 1 of them at most, the rest were speculative).  Unknown names return -1. */
TGB_API int tgb_fit_stat(tgb_booster* b, const char* key, double* out);

/* Host part of Binner::fit (cpp/src/binning.cpp:14-102), numeric features, no mask:
 * quantile edges from the bin_sample values std::shuffle(mt19937(seed + f*2654435761))
 * keeps, bit-identical to the reference.  X host row-major; edges_out [n_features][256],
 * n_edges_out [n_features].  Returns Binner::max_bins() (binning.cpp:130-134) or -1. */
TGB_API int tgb_binner_fit(const void* X, int x_dtype, int n, int n_features, int max_bin, int bin_sample,
                           unsigned seed, double* edges_out, int* n_edges_out);

/* Binner::fit with categorical features (cpp/src/binning.cpp:34-134): for a feature with
 * is_cat[f] != 0, edges_out[f] receives its vocabulary (the distinct values seen at least
 * cat_min_count times, at most max_bin - 1 of them, ascending; code = 1 + index) and
 * n_edges_out[f] its length; numeric features as in tgb_binner_fit.  Host only.
 * Returns max_bins() or -1. */
TGB_API int tgb_binner_fit_cat(const void* X, int x_dtype, int n, int n_features, const int* is_cat, int max_bin,
                               int cat_min_count, int bin_sample, unsigned seed, double* edges_out,
                               int* n_edges_out);

/* Binner::fit on X in device memory (row-major n x n_features of x_dtype, on `stream`):
 * the same edges as tgb_binner_fit, with the non-NaN counts, the value gather, the
 * sample sort, the edge arithmetic and the shuffle draws of features with at least 2^16
 * values as kernels.  edges_out / n_edges_out are host arrays as in tgb_binner_fit.
 * Requires n_features * min(bin_sample, n) < 2^31.  Returns max_bins() or -1. */
TGB_API int tgb_binner_fit_device(const void* X, int x_dtype, int n, int n_features, int max_bin, int bin_sample,
                                  unsigned seed, double* edges_out, int* n_edges_out, void* stream);

/* The first `keep` elements of std::shuffle(iota(m), std::mt19937(seed)) (libstdc++),
 * computed without materialising the range — the GOSS and bin-sample draw
 * (cpp/src/booster.cpp:572, cpp/src/binning.cpp:95). */
TGB_API int tgb_shuffled_prefix(long long m, long long keep, unsigned seed, int* out);

/* The GOSS draw sequence of Booster::fit (cpp/src/booster.cpp:569-588): one
 * std::mt19937(seed) makes n_shuffles std::shuffle's of iota(m), each followed by one
 * draw (grow_tree's seed); out[s*keep ..] receives the first keep of shuffle s.  The
 * generator is walked without producing positions and each prefix restarts from a
 * snapshot, as the fit's GOSS pipeline does.  0 <= keep <= m < 2^31. */
TGB_API int tgb_shuffle_sequence(long long m, long long keep, unsigned seed, int n_shuffles, int* out);

/* tgb_shuffled_prefix's prefix written to device memory out[keep] (on `stream`, synchronised before
 * returning), drawn on the device: the generator runs as one CTA and the swaps inside the
 * prefix are resolved in parallel from the recorded draws.  Ranges below 2^16 (libstdc++'s
 * two-draws path) are drawn on the host and copied.  1 <= keep <= m < 2^31. */
TGB_API int tgb_shuffled_prefix_device(long long m, long long keep, unsigned seed, int* out, void* stream);

/* ---- Serving loop ----
 * Fit and predict requests on one device under a device-memory budget.  Requests start
 * in arrival order, each as soon as a slot is free, its working set
 * (tgb_working_set_bytes) fits beside the running ones, and no other request on the same
 * booster runs.  Each runs on its booster's own stream, so concurrent requests overlap on
 * the device.  The caller keeps the booster and every host buffer of a request untouched
 * until the request has finished.  Latency counts from submission to completion. */
typedef struct tgb_server tgb_server;
TGB_API int tgb_server_create(int device, double budget_bytes, int slots, tgb_server** out);
/* Waits for every queued and running request, then frees the server (not the boosters). */
TGB_API void tgb_server_free(tgb_server* s);
/* Estimated device working set of a fit (kind 0) or predict (kind 1) request of n rows
 * with this booster's configuration, the admission figure; -1 on bad arguments. */
TGB_API long long tgb_working_set_bytes(tgb_booster* b, int kind, int n, int n_features, int x_dtype);
/* Queues tgb_fit(b, ...) / tgb_predict_raw(b, ...); *id_out receives the request id.
 * Fails at submission when the working set exceeds the whole budget. */
TGB_API int tgb_server_submit_fit(tgb_server* s, tgb_booster* b, const void* X, int x_dtype, const double* y, int n,
                                  int n_features, const long long* timestamps, const long long* entity,
                                  long long* id_out);
TGB_API int tgb_server_submit_predict(tgb_server* s, tgb_booster* b, const void* X, int x_dtype, int n,
                                      int n_features, double* out, long long* id_out);
/* Waits up to timeout_ms (< 0: no limit) for request id; *state: 0 queued, 1 running,
 * 2 done, 3 failed (the request's message is then in tgb_last_error).  -1 on a bad id. */
TGB_API int tgb_server_wait(tgb_server* s, long long id, double timeout_ms, int* state);
/* out[12]: completed, failed, latency p50, p99 (s), fit p50, p99, predict p50, p99, mean
 * wait for admission (s), peak requests running, peak admitted bytes, seconds from the
 * first submission to the last completion. */
TGB_API int tgb_server_stats(tgb_server* s, double* out);

/* ---- Kernel level: one reference function each, on device memory ---- */

/* Binner::transform (cpp/src/binning.cpp:104-128): codes[i*stride + f] = 1 + #{edges <= x},
 * NaN -> 0.  edges: device [n_features][256] of x_dtype, padded with +inf; for float32 X
 * pass ceil_f32 of the f64 edges (smallest float >= edge) to reproduce the f64 compare.
 * stride >= n_features, multiple of 16; padding bytes are zeroed. */
TGB_API int tgb_bin_transform(const void* X, int x_dtype, int n, int n_features, const void* edges,
                      const int* n_edges, unsigned char* codes, int stride, void* stream);

/* build_hist_col (cpp/src/histogram.cpp:44-76) and the build_hist_gpu kernel it replaces
 * (cpp/src/histogram_cuda.cu:28-44): for rows[0..n_rows), accumulate
 * G[f][code] += rint(g * 2^gshift), H[f][code] += rint(h * 2^hshift), C[f][code] += 1.
 * G, H: device int64 [n_features][256]; C: device int32 [n_features][256]; all must be
 * zeroed (or hold a partial sum to add to).  Exact integer sums: pick the shifts so
 * that n_rows * max|v| * 2^shift < 2^62. */
TGB_API int tgb_hist_build(const unsigned char* codes, int stride, int n_features, const int* rows, int n_rows,
                   const double* g, const double* h, int gshift, int hshift, long long* G, long long* H,
                   int* C, void* stream);

/* The histogram of tgb_hist_build through the fit's own per-tree payload and histogram
 * kernels: hist_bits 0 (exact 64-bit fixed point) or 16 / 8 (g, and h unless h is NULL,
 * stochastically rounded to int16 / int8 with the fit's scale: the largest |g| of the rows
 * maps to the largest code; `seed` drives the rounding).  h == NULL: unit hessians.
 * G, H: device int64 [n_features][256], C int32, zeroed by the caller; scales_out[2]
 * (host) receives the factors that turn G and H back into gradient units (G * scales_out[0]
 * is the bin's sum of g).  For measuring the quantisation error of the precision modes.
 * rows: device int32, every value < the rows of codes / g / h. */
TGB_API int tgb_hist_build_quantized(const unsigned char* codes, int stride, int n_features, const int* rows,
                                     int n_rows, const double* g, const double* h, int hist_bits,
                                     unsigned long long seed, long long* G, long long* H, int* C, double* scales_out,
                                     void* stream);

/* best_numeric_missing (cpp/src/histogram.cpp:144-193, l1 = 0, no monotone) for every
 * feature of one fixed-point histogram: gain[f], thr[f] (-1 = none), ml[f]. */
TGB_API int tgb_split_scan(const long long* G, const long long* H, const int* C, int n_features, int n_bins,
                   int gshift, int hshift, double l2, double min_split_gain, int min_samples_leaf,
                   double min_child_weight, double* gain, int* thr, int* missing_left, void* stream);

/* split_indices (cpp/src/tree.cpp:68-91): stable partition of rows[0..n_rows) into
 * out[0..n_left) (code == 0 ? missing_left : code <= threshold) and out[n_left..n_rows).
 * n_left_out: device int.  workspace: device scratch of tgb_partition_workspace_bytes(n_rows). */
TGB_API size_t tgb_partition_workspace_bytes(int n_rows);
TGB_API int tgb_partition(const unsigned char* codes, int stride, const int* rows, int n_rows, int feature,
                  int threshold, int missing_left, int* out, int* n_left_out, void* workspace,
                  size_t workspace_bytes, void* stream);

/* tgb_partition for callers that cannot allocate device memory (this entry point has no
 * counterpart in the reference).  Some callers have no way to provide the workspace
 * tgb_partition asks for: a serving process that reserves all device memory at start-up
 * and must not call cudaMalloc later (it can block the device and fail under memory
 * pressure), or a binding that passes only a call's inputs and outputs.  This variant
 * allocates nothing: its scratch (the per-tile counts of left rows) is a fixed device
 * array inside the library (32 KB, held on every GPU that loads the library until the
 * process exits), so n_rows is limited to 16,777,216 (larger calls return -1 with a
 * message).  Every call looks up that array's device address with the device current;
 * the first call on a device may load the library's device code, so make it before any
 * stream capture.  All calls on a device share the array: calls whose kernels may
 * overlap on the GPU (other streams or host threads) race and must be serialised by the
 * caller.  Results equal tgb_partition's. */
TGB_API int tgb_partition_noalloc(const unsigned char* codes, int stride, const int* rows, int n_rows, int feature,
                                  int threshold, int missing_left, int* out, int* n_left_out, void* stream);

/* Objective::grad_hess (cpp/src/objective.cpp:102-219), unit weights, device f64 arrays.
 * MSE: g = pred - y, h = 1.  Pairwise: date groups given as runs of consecutive rows
 * (run_start/run_len device int [n_runs]; rows of a run are order[run_start..] when
 * order != NULL, else consecutive). */
TGB_API int tgb_grad_mse(const double* y, const double* pred, int n, double* g, double* h, void* stream);
TGB_API int tgb_grad_pairwise(const double* y, const double* pred, const int* run_start, const int* run_len,
                      const int* order, int n_runs, int n, double* g, double* h, void* stream);

/* Literal drop-in for the reference seam build_hist_gpu (cpp/include/tidegbm/histogram.hpp:
 * 57-58, cpp/src/histogram_cuda.cu:81-167): host row-major uint16 codes (kept resident
 * on the booster's device across calls with the same pointer), host idx/g/h, result
 * written as the interleaved FP64 {g, h, c} Hist layout (histogram.hpp:14-46),
 * n_features x n_bins. */
TGB_API int tgb_build_hist_gpu(tgb_booster* b, const unsigned short* xb, int n_features, const int* idx, int n_idx,
                       const double* g, const double* h, int n_bins, int n_rows, double* out_ghc);

#ifdef __cplusplus
}
#endif

#endif
