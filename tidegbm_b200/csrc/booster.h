// GPU booster: the device="gpu" implementation of TideGBM's Booster::fit
// (cpp/src/booster.cpp:231-742) for the hot-path subset, plus predict_raw.
#pragma once

#include <cstdint>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

namespace tgb {

struct TideError : std::runtime_error {
    explicit TideError(const std::string& m) : std::runtime_error(m) {}
};

// The Config fields (cpp/include/tidegbm/config.hpp:12-97) the GPU path reads.  Every
// other option keeps its default; options the GPU path does not implement are
// rejected by validate() with a TideError instead of falling back to the CPU.
struct Config {
    int n_estimators = 100;
    double learning_rate = 0.1;
    int max_depth = 6;
    int max_leaves = 31;
    int min_samples_leaf = 20;
    double min_child_weight = 1e-3;
    double l2 = 1.0;
    double min_split_gain = 0.0;
    int max_bin = 255;
    int n_time_buckets = 0;
    int64_t horizon = -1;
    int64_t embargo = 0;
    bool iid_mode = false;
    int objective = 0;  // 0 mse, 5 pairwise (ObjectiveKind, cpp/include/tidegbm/types.hpp:26-35)
    int random_state = 0;
    int goss = -1;
    double goss_top = 0.2;
    double goss_other = 0.1;
    int bin_sample = 262144;
    double torb_min_cover = 0.0;
    double cat_smooth = 1.0;  // config.hpp:70
    int cat_min_count = 5;    // config.hpp:72
    bool finer_torb = true;
    int n_jobs = 0;
    std::string device = "gpu";
    // Options that exist in the reference but are not implemented on the GPU path.
    // pair_splits defaults to true as in the reference (config.hpp:31), off at n >= 1M as
    // the reference turns it off there; PAIR needs batched growth and exact histograms.
    bool pair_splits = true;
    double pair_trigger = 0.25;      // config.hpp:32-35
    int pair_top_k = 6;
    int max_pair_splits_per_tree = 3;
    double pair_l2 = 2.0;
    bool halo = false;
    double subsample = 1.0;
    double colsample = 1.0;
    double colsample_bynode = 1.0;
    double l1 = 0.0;
    double max_delta_step = 0.0;
    double time_decay = 1.0;
    bool causal_bins = false;
    bool causal_structure = false;
    double structure_frac = 1.0;
    double entity_subsample = 1.0;
    // Histogram precision: 0 = exact 64-bit fixed point (results match the reference); 16 / 8
    // = gradients (and hessians) stochastically rounded to int16 / int8 per tree and summed
    // exactly in 32-bit shared words (fewer shared reductions per code; approximate split
    // search, exact leaf values).  With grow = 0 only 8 with a constant hessian (mse).
    int hist_bits = 0;
    // Tree growth: 1 = batched waves (many leaves, and many fits, per launch; wave.h),
    // 0 = one split per iteration.  Both grow the reference's tree.  graph: the waves of a
    // tree run as one CUDA graph with a device-side loop (1) or are enqueued by the host (0).
    int grow = 1;
    int graph = 1;
    // Batched growth: tune the histogram's launch shape on the first tree (1), or use the
    // default (0); the choice is kept per shape of the work for the process.
    int hist_tune = 1;
    // Batched growth: expansions a wave may plan (0: every leaf ranked within the splits
    // left, the widest speculation; k: the k best).  Any value grows the same tree.  8 keeps
    // the waves few while histogramming few children that are never committed (about 32
    // expansions for the 30 splits of a 31-leaf tree, against 37 uncapped).
    int wave_expand = 8;
    // Histogram code rows (constant-hessian modes): staged into shared memory by TMA gathers
    // (1), or loaded by each lane from global memory (0).  Same results either way.
    int hist_stage = 1;
    // Measurement hooks (no effect on results): CUDA events around trees
    // [timing_from, timing_to) (timing_to < 0: through the last tree), and per-launch
    // events around every histogram kernel in that range.
    int timing_from = -1;
    int timing_to = -1;
    bool profile_hist = false;

    void validate() const;
};

struct HostNode {
    int is_leaf, feature, threshold, left, right, missing_left, n_samples, depth;
    double value, gain;
    int type;                    // 0 axis, 1 pair, 2 categorical (SplitType, cpp/include/tidegbm/types.hpp:25)
    unsigned long long cat[4];   // categorical: the codes that go left
    int feature2;                // pair: the second feature
};

struct HostTree {
    std::vector<HostNode> nodes;
    std::vector<double> values;
    std::vector<int> cover;
    std::vector<double> prefix;  // n_buckets x n_nodes
};

struct FitStats {
    double t_total = 0, t_sort = 0, t_binfit = 0, t_upload = 0, t_transform = 0, t_trees = 0, t_download = 0;
    double t_rng = 0;
    double t_alloc = 0, t_h2d = 0, t_transpose = 0, t_producer = 0;
    double t_driver = 0, t_finish_sync = 0;  // wave driver set-up; tree loop's tail to the sampler's stop
    double t_driver_free = 0;                // wave driver release after the tree loop
    double t_release = 0;                    // the fit's working buffers back to the pool
    long long expansions = 0;                // leaves expanded (children histogrammed) over the fit's trees
    double t_bin_counts = 0, t_bin_draws = 0, t_bin_edges = 0;  // stages of the device binner
    int goss_refits = 0;  // 1 when the fit was repeated with the 64-bit GOSS sort
    double t_pre_upload = 0, t_prep = 0;  // host set-up before the upload and before the tree loop
    int gpu_launches = 0;
    // timed range (cfg.timing_from .. last tree), device time from CUDA events
    double timed_ms = 0;
    int timed_trees = 0;
    long long timed_launches = 0;
    double hist_ms = 0;       // sum of histogram-kernel durations in the timed range
    int hist_launches = 0;
    long long hist_rows = 0;  // rows histogrammed in the timed range
    long long timed_selects = 0;  // wave selects run in the timed range (batched growth)
    int graph_used = 0;           // the waves ran as a CUDA graph with a device-side loop
    int hist_cluster = 0, hist_clusters = 0;  // the histogram's launch shape (autotuned)
};

struct DeviceState;  // device buffers of one fit
struct FitRun;

// One fit's inputs (the arguments of GpuBooster::fit).
struct FitInput {
    const void* X;
    int x_dtype;
    const double* y;
    int n, n_f;
    const int64_t* ts;
    const int64_t* entity;
};

class GpuBooster {
public:
    explicit GpuBooster(int device);
    ~GpuBooster();
    GpuBooster(const GpuBooster&) = delete;
    GpuBooster& operator=(const GpuBooster&) = delete;

    Config cfg;
    int device = 0;
    // fitted model
    bool fitted = false;
    int n_features = 0;
    int n_bins = 0;
    int n_buckets = 1;
    double init_score = 0.0;
    std::vector<double> init_prefix;
    std::vector<double> edges;  // n_features x 256 (first n_edges[f] used)
    std::vector<int> n_edges;
    std::vector<HostTree> trees;
    std::vector<double> evals_train;
    FitStats stats;
    // categorical flag per feature for the next fit (Booster::fit's is_cat,
    // cpp/src/booster.cpp:246-247); empty: every feature numeric
    std::vector<int> is_cat;

    void fit(const void* X, int x_dtype, const double* y, int n, int n_f, const int64_t* ts,
             const int64_t* entity);
    void predict_raw(const void* X, int x_dtype, int n, int n_f, double* out);
    // Fits every booster on its input in lockstep on one device: each tree of all of them
    // grows in the same wave launches (batched growth; boosters[0]'s stream and timing
    // hooks).  Each result equals the booster's own fit.
    static void fit_batch(const std::vector<GpuBooster*>& boosters, const std::vector<FitInput>& inputs);

private:
    friend struct FitRun;
    // One fit; exact_goss sorts GOSS keys on all 64 bits.  Returns true when the 32-bit
    // GOSS sort met a tied run too long to fix up (the result must then be recomputed).
    bool fit_once(const void* X, int x_dtype, const double* y, int n, int n_f, const int64_t* ts,
                  const int64_t* entity, bool exact_goss);
    DeviceState* ds_ = nullptr;
};

// Host part of Binner::fit (cpp/src/binning.cpp:14-102) for numeric features: the
// sampled values per feature and their quantile edges.  Returns max_bins().
int binner_fit(const void* X, int x_dtype, int n, int n_f, int max_bin, int bin_sample, uint32_t seed,
               std::vector<double>& edges, std::vector<int>& n_edges, int n_threads);
// Binner::fit with categorical features (is_cat[f] != 0): edges[f] holds the vocabulary of
// a categorical feature (binning.cpp:47-84) and n_edges[f] its length.  Returns max_bins().
int binner_fit_cat(const void* X, int x_dtype, int n, int n_f, const int* is_cat, int max_bin, int cat_min_count,
                   int bin_sample, uint32_t seed, std::vector<double>& edges, std::vector<int>& n_edges,
                   int n_threads);
// The same edges from X in device memory (row-major n x n_f, stream `stream`, a
// cudaStream_t).  binner_fits_device says whether one feature-major sample buffer of
// the sizes involved stays under 2^31 values (else use binner_fit).
struct BinFitTimes {
    double counts = 0, draws = 0, edges = 0;  // wall seconds of the three stages
    int refit_features = 0;  // features whose edges were recomputed on the host
};
bool binner_fits_device(int n, int n_f, int bin_sample);
// binner_fit_device's two stages: binner_plan (per-feature totals, rank bases and the
// kept ranks of the shuffle, from non-NaN counts per 4096-row chunk and feature) and
// binner_fit_from_plan (the device part on X in device memory).
struct BinPlan {
    int n_chunks = 0;
    std::vector<int64_t> m;
    std::vector<long long> base;
    std::vector<uint8_t> take_all;
    std::vector<int> kept;
    int64_t max_sampled = 0;
    long long cap = 1;
    uint32_t seed = 0;
    // sampled features with fewer than 2^16 values (libstdc++'s two-draws shuffle path)
    // and their kept ranks [host_f.size()][bin_sample], drawn on the host; the other
    // sampled features are drawn on the device
    std::vector<int> host_f;
    std::vector<int32_t> keep;
};
void binner_plan(const std::vector<int>& counts, int n, int n_f, int bin_sample, uint32_t seed, int n_threads,
                 BinPlan& plan);
// flagged (optional): features whose edges depend on how std::sort orders equal values
// (both zero signs, or infinities with interpolated edges), to be recomputed on the host.
int binner_fit_from_plan(const BinPlan& plan, const void* Xd, int x_dtype, int n, int n_f, int max_bin,
                         int bin_sample, std::vector<double>& edges, std::vector<int>& n_edges, void* stream,
                         void* arena, size_t arena_bytes, std::vector<int>* flagged = nullptr);
// arena / arena_bytes: device memory the binner may use as scratch (nullptr: allocate).
// X_host (optional): the same X on the host, read when features are recomputed there.
int binner_fit_device(const void* Xd, int x_dtype, int n, int n_f, int max_bin, int bin_sample, uint32_t seed,
                      std::vector<double>& edges, std::vector<int>& n_edges, int n_threads, void* stream,
                      void* arena, size_t arena_bytes, BinFitTimes* tm, const void* X_host = nullptr);

}  // namespace tgb
