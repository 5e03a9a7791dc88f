// extern "C" boundary (include/tidegbm_b200.h).  Every entry catches all exceptions
// and reports -1 + a thread-local message, like the reference C API
// (cpp/src/c_api.cpp:12-18, 20-158).
#include "tidegbm_b200.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <thread>
#include <vector>

#include "booster.h"
#include "sampling.h"
#include "serving.h"
#include "tgb_internal.h"
#include "wave.h"

namespace tgb {
extern std::atomic<long long> g_kernel_launches;
}

struct tgb_booster {
    tgb::GpuBooster* b = nullptr;
    // state of the build_hist_gpu drop-in (per booster, not process-global)
    const unsigned short* host_xb = nullptr;
    int xb_rows = 0, xb_f = 0, xb_stride = 0;
    unsigned char* d_codes = nullptr;
    int* d_idx = nullptr;
    double *d_g = nullptr, *d_h = nullptr;
    long long *d_G = nullptr, *d_H = nullptr;
    int* d_C = nullptr;
    size_t cap_idx = 0, cap_rows = 0, cap_hist = 0;
    ~tgb_booster() {
        cudaFree(d_codes);
        cudaFree(d_idx);
        cudaFree(d_g);
        cudaFree(d_h);
        cudaFree(d_G);
        cudaFree(d_H);
        cudaFree(d_C);
        delete b;
    }
};

struct tgb_server {
    tgb::Scheduler* sched = nullptr;
    int device = 0;
    ~tgb_server() { delete sched; }  // waits for every queued and running request
};

namespace {

thread_local std::string g_err;

// Device working set of a fit or predict request, the serving loop's admission figure:
// the buffers of one fit context (X during binning, row-major and column-major codes,
// per-row f64 state, row lists, GOSS keys, the node histograms) or of one prediction
// (X, codes, output), plus a fixed allowance for scratch and the CUDA context's share.
size_t working_set_bytes(const tgb::Config& c, int kind, long long n, long long n_f, int x_dtype) {
    const long long xsz = x_dtype == 0 ? 4 : 8;
    const long long stride = (n_f + 15) / 16 * 16;
    const long long pitch = (n + 15) / 16 * 16;
    const long long slack = 64ll << 20;
    if (kind == 1) return static_cast<size_t>(n * n_f * xsz + n * stride + 8 * n + slack);
    const long long per_row = 8 * 3              // y, pred, g
                              + (c.objective == 0 ? 16 : 40)  // payloads in both row buffers (+ h)
                              + 8 + 2            // row lists, leaf ids
                              + 26;              // GOSS keys, values and flags
    const long long nodes = 2ll * c.max_leaves - 1;
    const long long hist = n_f * 256 * 20 * nodes;
    return static_cast<size_t>(n * n_f * xsz + n * stride + n_f * pitch + per_row * n + hist + slack);
}

template <class F>
int guard(F&& f) {
    try {
        f();
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    } catch (...) {
        g_err = "unknown error";
        return -1;
    }
}

cudaStream_t as_stream(void* s) { return static_cast<cudaStream_t>(s); }

void need(bool ok, const char* msg) {
    if (!ok) throw tgb::TideError(msg);
}

}  // namespace

extern "C" {

const char* tgb_last_error(void) { return g_err.c_str(); }

long long tgb_kernel_launches(void) { return tgb::g_kernel_launches.load(); }

int tgb_booster_create(int device, tgb_booster** out) {
    return guard([&] {
        need(out != nullptr, "out is NULL");
        auto* h = new tgb_booster();
        try {
            h->b = new tgb::GpuBooster(device);
        } catch (...) {
            delete h;
            throw;
        }
        *out = h;
    });
}

void tgb_booster_free(tgb_booster* b) { delete b; }

int tgb_set_int(tgb_booster* hb, const char* key, long long v) {
    return guard([&] {
        need(hb && key, "NULL argument");
        tgb::Config& c = hb->b->cfg;
        const std::string k(key);
        if (k == "n_estimators") c.n_estimators = static_cast<int>(v);
        else if (k == "max_depth") c.max_depth = static_cast<int>(v);
        else if (k == "max_leaves") c.max_leaves = static_cast<int>(v);
        else if (k == "min_samples_leaf") c.min_samples_leaf = static_cast<int>(v);
        else if (k == "max_bin") c.max_bin = static_cast<int>(v);
        else if (k == "n_time_buckets") c.n_time_buckets = static_cast<int>(v);
        else if (k == "random_state") c.random_state = static_cast<int>(v);
        else if (k == "n_jobs") c.n_jobs = static_cast<int>(v);
        else if (k == "iid_mode") c.iid_mode = v != 0;
        else if (k == "halo") c.halo = v != 0;
        else if (k == "pair_splits") c.pair_splits = v != 0;
        else if (k == "horizon") c.horizon = v;
        else if (k == "embargo") c.embargo = v;
        else if (k == "goss") c.goss = static_cast<int>(v);
        else if (k == "bin_sample") c.bin_sample = static_cast<int>(v);
        else if (k == "finer_torb") c.finer_torb = v != 0;
        else if (k == "objective") c.objective = static_cast<int>(v);
        else if (k == "causal_bins") c.causal_bins = v != 0;
        else if (k == "causal_structure") c.causal_structure = v != 0;
        else if (k == "timing_from") c.timing_from = static_cast<int>(v);
        else if (k == "timing_to") c.timing_to = static_cast<int>(v);
        else if (k == "hist_bits") c.hist_bits = static_cast<int>(v);
        else if (k == "profile_hist") c.profile_hist = v != 0;
        else if (k == "grow") c.grow = static_cast<int>(v);
        else if (k == "graph") c.graph = static_cast<int>(v);
        else if (k == "hist_tune") c.hist_tune = static_cast<int>(v);
        else if (k == "wave_expand") c.wave_expand = static_cast<int>(v);
        else if (k == "hist_stage") c.hist_stage = static_cast<int>(v);
        else if (k == "cat_min_count") c.cat_min_count = static_cast<int>(v);
        else if (k == "pair_top_k") c.pair_top_k = static_cast<int>(v);
        else if (k == "max_pair_splits_per_tree") c.max_pair_splits_per_tree = static_cast<int>(v);
        else if (k == "verbose" || k == "col_major_hist") { /* no effect on GPU path */ }
        else throw tgb::TideError("unknown int key");
    });
}

int tgb_set_double(tgb_booster* hb, const char* key, double v) {
    return guard([&] {
        need(hb && key, "NULL argument");
        tgb::Config& c = hb->b->cfg;
        const std::string k(key);
        if (k == "learning_rate") c.learning_rate = v;
        else if (k == "l2") c.l2 = v;
        else if (k == "l1") c.l1 = v;
        else if (k == "min_child_weight") c.min_child_weight = v;
        else if (k == "min_split_gain") c.min_split_gain = v;
        else if (k == "subsample") c.subsample = v;
        else if (k == "colsample") c.colsample = v;
        else if (k == "colsample_bynode") c.colsample_bynode = v;
        else if (k == "goss_top") c.goss_top = v;
        else if (k == "goss_other") c.goss_other = v;
        else if (k == "torb_min_cover") c.torb_min_cover = v;
        else if (k == "cat_smooth") c.cat_smooth = v;
        else if (k == "pair_trigger") c.pair_trigger = v;
        else if (k == "pair_l2") c.pair_l2 = v;
        else if (k == "max_delta_step") c.max_delta_step = v;
        else if (k == "time_decay") c.time_decay = v;
        else if (k == "structure_frac") c.structure_frac = v;
        else if (k == "entity_subsample") c.entity_subsample = v;
        else throw tgb::TideError("unknown double key");
    });
}

int tgb_set_str(tgb_booster* hb, const char* key, const char* value) {
    return guard([&] {
        need(hb && key && value, "NULL argument");
        tgb::Config& c = hb->b->cfg;
        const std::string k(key), v(value);
        if (k == "objective") {
            // bindings.cpp:115-125 names
            if (v == "mse" || v == "auto" || v == "l2" || v == "regression") c.objective = 0;
            else if (v == "pairwise" || v == "lambdarank") c.objective = 5;
            else if (v == "huber" || v == "quantile" || v == "pinball" || v == "logloss" || v == "binary" ||
                     v == "classification" || v == "rank" || v == "listnet" || v == "multiclass" || v == "custom")
                throw tgb::TideError("GPU path: objective '" + v + "' is not supported (mse or pairwise)");
            else throw tgb::TideError("unknown objective: " + v);
        } else if (k == "device") {
            c.device = v;
        } else {
            throw tgb::TideError("unknown string key");
        }
    });
}

int tgb_fit(tgb_booster* hb, const void* X, int x_dtype, const double* y, int n, int n_features,
            const long long* timestamps, const long long* entity) {
    return guard([&] {
        need(hb && X && y, "NULL argument");
        hb->b->fit(X, x_dtype, y, n, n_features, reinterpret_cast<const int64_t*>(timestamps),
                   reinterpret_cast<const int64_t*>(entity));
    });
}

int tgb_fit_batch(tgb_booster* const* boosters, int n_boosters, const void* const* X, int x_dtype,
                  const double* const* y, const int* n, int n_features, const long long* const* timestamps,
                  const long long* const* entity) {
    return guard([&] {
        need(boosters && X && y && n && n_boosters >= 1, "NULL argument");
        std::vector<tgb::GpuBooster*> bs;
        std::vector<tgb::FitInput> in;
        for (int k = 0; k < n_boosters; ++k) {
            need(boosters[k] && X[k] && y[k], "NULL argument");
            for (int q = 0; q < k; ++q) need(boosters[q] != boosters[k], "a booster appears twice");
            bs.push_back(boosters[k]->b);
            in.push_back(tgb::FitInput{X[k], x_dtype, y[k], n[k], n_features,
                                       timestamps ? reinterpret_cast<const int64_t*>(timestamps[k]) : nullptr,
                                       entity ? reinterpret_cast<const int64_t*>(entity[k]) : nullptr});
        }
        tgb::GpuBooster::fit_batch(bs, in);
    });
}

int tgb_predict_raw(tgb_booster* hb, const void* X, int x_dtype, int n, int n_features, double* out) {
    return guard([&] {
        need(hb && X && out, "NULL argument");
        hb->b->predict_raw(X, x_dtype, n, n_features, out);
    });
}

int tgb_model_info(tgb_booster* hb, int* n_trees, int* n_bins, int* n_buckets, double* init_score) {
    return guard([&] {
        need(hb != nullptr, "NULL booster");
        const auto& b = *hb->b;
        if (n_trees) *n_trees = static_cast<int>(b.trees.size());
        if (n_bins) *n_bins = b.n_bins;
        if (n_buckets) *n_buckets = b.n_buckets;
        if (init_score) *init_score = b.init_score;
    });
}

int tgb_init_prefix(tgb_booster* hb, double* out) {
    return guard([&] {
        need(hb && out, "NULL argument");
        std::copy(hb->b->init_prefix.begin(), hb->b->init_prefix.end(), out);
    });
}

int tgb_evals_train(tgb_booster* hb, double* out) {
    return guard([&] {
        need(hb && out, "NULL argument");
        std::copy(hb->b->evals_train.begin(), hb->b->evals_train.end(), out);
    });
}

int tgb_tree_n_nodes(tgb_booster* hb, int t) {
    if (!hb || t < 0 || t >= static_cast<int>(hb->b->trees.size())) {
        g_err = "tree index out of range";
        return -1;
    }
    return static_cast<int>(hb->b->trees[t].nodes.size());
}

int tgb_tree_export_split(tgb_booster* hb, int t, int* types, int* feature2, unsigned long long* cat_left) {
    return guard([&] {
        need(hb != nullptr, "NULL booster");
        need(t >= 0 && t < static_cast<int>(hb->b->trees.size()), "tree index out of range");
        const tgb::HostTree& tr = hb->b->trees[t];
        for (size_t k = 0; k < tr.nodes.size(); ++k) {
            if (types) types[k] = tr.nodes[k].is_leaf ? 0 : tr.nodes[k].type;
            if (feature2) feature2[k] = tr.nodes[k].is_leaf ? -1 : tr.nodes[k].feature2;
            if (cat_left)
                for (int q = 0; q < 4; ++q) cat_left[4 * k + q] = tr.nodes[k].cat[q];
        }
    });
}

int tgb_set_categorical(tgb_booster* hb, const int* is_cat, int n_features) {
    return guard([&] {
        need(hb != nullptr, "NULL booster");
        need(n_features >= 0, "n_features < 0");
        if (is_cat == nullptr || n_features == 0) hb->b->is_cat.clear();
        else hb->b->is_cat.assign(is_cat, is_cat + n_features);
    });
}

int tgb_tree_export(tgb_booster* hb, int t, int* inodes, double* fnodes, double* values, int* cover, double* prefix) {
    return guard([&] {
        need(hb != nullptr, "NULL booster");
        need(t >= 0 && t < static_cast<int>(hb->b->trees.size()), "tree index out of range");
        const tgb::HostTree& tr = hb->b->trees[t];
        for (size_t k = 0; k < tr.nodes.size(); ++k) {
            const tgb::HostNode& d = tr.nodes[k];
            if (inodes) {
                int* o = inodes + 8 * k;
                o[0] = d.is_leaf;
                o[1] = d.feature;
                o[2] = d.threshold;
                o[3] = d.left;
                o[4] = d.right;
                o[5] = d.missing_left;
                o[6] = d.n_samples;
                o[7] = d.depth;
            }
            if (fnodes) {
                fnodes[2 * k] = d.value;
                fnodes[2 * k + 1] = d.gain;
            }
        }
        if (values) std::copy(tr.values.begin(), tr.values.end(), values);
        if (cover) std::copy(tr.cover.begin(), tr.cover.end(), cover);
        if (prefix) std::copy(tr.prefix.begin(), tr.prefix.end(), prefix);
    });
}

int tgb_edges(tgb_booster* hb, int f, double* out) {
    if (!hb || f < 0 || f >= hb->b->n_features) {
        g_err = "feature index out of range";
        return -1;
    }
    const int ne = hb->b->n_edges[f];
    if (out) std::copy(hb->b->edges.begin() + static_cast<size_t>(f) * 256,
                       hb->b->edges.begin() + static_cast<size_t>(f) * 256 + ne, out);
    return ne;
}

int tgb_fit_stats(tgb_booster* hb, double* o) {
    return guard([&] {
        need(hb && o, "NULL argument");
        const tgb::FitStats& s = hb->b->stats;
        o[0] = s.t_total;
        o[1] = s.t_sort;
        o[2] = s.t_binfit;
        o[3] = s.t_upload;
        o[4] = s.t_trees;
        o[5] = s.t_download;
        o[6] = s.t_rng;
        o[7] = s.gpu_launches;
        o[8] = s.timed_ms;
        o[9] = s.timed_trees;
        o[10] = static_cast<double>(s.timed_launches);
        o[11] = s.hist_ms;
        o[12] = s.hist_launches;
        o[13] = static_cast<double>(s.hist_rows);
        o[14] = s.t_alloc;
        o[15] = s.t_h2d;
        o[16] = s.t_transpose;
        o[17] = s.t_producer;
    });
}

int tgb_binner_fit_cat(const void* X, int x_dtype, int n, int n_features, const int* is_cat, int max_bin,
                       int cat_min_count, int bin_sample, unsigned seed, double* edges_out, int* n_edges_out) {
    int nb = -1;
    const int rc = guard([&] {
        need(X && is_cat && edges_out && n_edges_out, "NULL argument");
        need(x_dtype == 0 || x_dtype == 1, "x_dtype must be 0 or 1");
        need(max_bin >= 8 && max_bin <= 256, "max_bin must be in [8, 256]");
        std::vector<double> e;
        std::vector<int> ne;
        nb = tgb::binner_fit_cat(X, x_dtype, n, n_features, is_cat, max_bin, cat_min_count, bin_sample, seed, e, ne,
                                 static_cast<int>(std::max(1u, std::thread::hardware_concurrency())));
        std::copy(e.begin(), e.end(), edges_out);
        std::copy(ne.begin(), ne.end(), n_edges_out);
    });
    return rc == 0 ? nb : -1;
}

int tgb_binner_fit(const void* X, int x_dtype, int n, int n_features, int max_bin, int bin_sample, unsigned seed,
                   double* edges_out, int* n_edges_out) {
    int nb = -1;
    const int rc = guard([&] {
        need(X && edges_out && n_edges_out, "NULL argument");
        need(x_dtype == 0 || x_dtype == 1, "x_dtype must be 0 or 1");
        need(max_bin >= 8 && max_bin <= 256, "max_bin must be in [8, 256]");
        std::vector<double> e;
        std::vector<int> ne;
        nb = tgb::binner_fit(X, x_dtype, n, n_features, max_bin, bin_sample, seed, e, ne,
                             static_cast<int>(std::max(1u, std::thread::hardware_concurrency())));
        std::copy(e.begin(), e.end(), edges_out);
        std::copy(ne.begin(), ne.end(), n_edges_out);
    });
    return rc == 0 ? nb : -1;
}

int tgb_binner_fit_device(const void* X, int x_dtype, int n, int n_features, int max_bin, int bin_sample,
                          unsigned seed, double* edges_out, int* n_edges_out, void* stream) {
    int nb = -1;
    const int rc = guard([&] {
        need(X && edges_out && n_edges_out, "NULL argument");
        need(n > 0 && n_features > 0, "empty input");
        need(x_dtype == 0 || x_dtype == 1, "x_dtype must be 0 or 1");
        need(max_bin >= 8 && max_bin <= 256, "max_bin must be in [8, 256]");
        need(tgb::binner_fits_device(n, n_features, bin_sample),
             "n_features x min(bin_sample, n) must stay below 2^31 values (use tgb_binner_fit)");
        std::vector<double> e;
        std::vector<int> ne;
        nb = tgb::binner_fit_device(X, x_dtype, n, n_features, max_bin, bin_sample, seed, e, ne,
                                    static_cast<int>(std::max(1u, std::thread::hardware_concurrency())), stream,
                                    nullptr, 0, nullptr);
        std::copy(e.begin(), e.end(), edges_out);
        std::copy(ne.begin(), ne.end(), n_edges_out);
    });
    return rc == 0 ? nb : -1;
}

int tgb_fit_stat(tgb_booster* hb, const char* key, double* out) {
    return guard([&] {
        need(hb && key && out, "NULL argument");
        const tgb::FitStats& s = hb->b->stats;
        const std::string k(key);
        if (k == "bin_counts") *out = s.t_bin_counts;
        else if (k == "bin_draws") *out = s.t_bin_draws;
        else if (k == "bin_edges") *out = s.t_bin_edges;
        else if (k == "bin_fit") *out = s.t_binfit;
        else if (k == "h2d") *out = s.t_h2d;
        else if (k == "alloc") *out = s.t_alloc;
        else if (k == "transpose") *out = s.t_transpose;
        else if (k == "trees") *out = s.t_trees;
        else if (k == "total") *out = s.t_total;
        else if (k == "goss_refits") *out = s.goss_refits;
        else if (k == "timed_selects") *out = static_cast<double>(s.timed_selects);
        else if (k == "graph_used") *out = s.graph_used;
        else if (k == "hist_cluster") *out = s.hist_cluster;
        else if (k == "hist_clusters") *out = s.hist_clusters;
        else if (k == "driver") *out = s.t_driver;
        else if (k == "expansions") *out = static_cast<double>(s.expansions);
        else if (k == "finish_sync") *out = s.t_finish_sync;
        else if (k == "driver_free") *out = s.t_driver_free;
        else if (k == "release") *out = s.t_release;
        else if (k == "pre_upload") *out = s.t_pre_upload;
        else if (k == "prep") *out = s.t_prep;
        else throw tgb::TideError("unknown fit stat: " + k);
    });
}

int tgb_shuffled_prefix(long long m, long long keep, unsigned seed, int* out) {
    return guard([&] {
        need(m >= 0 && m < (1ll << 31) && keep >= 0 && keep <= m, "bad sizes");
        tgb::Mt32 rng(seed);
        tgb::shuffled_prefix(m, keep, rng, out);
    });
}

int tgb_shuffle_sequence(long long m, long long keep, unsigned seed, int n_shuffles, int* out) {
    return guard([&] {
        need(m >= 0 && m < (1ll << 31) && keep >= 0 && keep <= m && n_shuffles >= 0, "bad sizes");
        tgb::Mt32 rng(seed);
        for (int s = 0; s < n_shuffles; ++s) {
            tgb::Mt32 snap = rng;
            tgb::shuffled_prefix(m, keep, snap, out + static_cast<size_t>(s) * keep);
            tgb::skip_shuffle(m, rng);
            (void)rng();
        }
    });
}

int tgb_shuffled_prefix_device(long long m, long long keep, unsigned seed, int* out, void* stream) {
    return guard([&] {
        need(m >= 1 && m < (1ll << 31) && keep >= 1 && keep <= m, "bad sizes");
        need(out != nullptr, "out is null");
        cudaStream_t s = as_stream(stream);
        if (tgb::shuffle_pairs(m)) {  // libstdc++'s two-draws path for short ranges: on the host
            std::vector<int32_t> h(static_cast<size_t>(keep));
            tgb::Mt32 rng(seed);
            tgb::shuffled_prefix(m, keep, rng, h.data());
            tgb::check(cudaMemcpyAsync(out, h.data(), sizeof(int32_t) * h.size(), cudaMemcpyHostToDevice, s),
                       "prefix upload");
            tgb::check(cudaStreamSynchronize(s), "prefix upload");
            return;
        }
        const size_t k = static_cast<size_t>(keep);
        tgb::DBuf<int32_t> scratch;
        scratch.alloc(3 * k + 1, s);  // head [k], items [k], cnt [k + 1]
        int32_t* head = scratch.p;
        int32_t* items = head + k;
        int32_t* cnt = items + k;
        tgb::DBuf<long long> ms_d;
        ms_d.alloc(1, s);
        tgb::DBuf<uint32_t> misc;
        misc.alloc(2, s);  // seed, error flag
        const long long ms = m;
        const uint32_t seed_h = seed;
        int err = 0;
        tgb::check(cudaMemcpyAsync(ms_d.p, &ms, sizeof(ms), cudaMemcpyHostToDevice, s), "size upload");
        tgb::check(cudaMemcpyAsync(misc.p, &seed_h, sizeof(seed_h), cudaMemcpyHostToDevice, s), "seed upload");
        tgb::check(cudaMemsetAsync(misc.p + 1, 0, sizeof(uint32_t), s), "error flag reset");
        tgb::launch_shuffle_prefix(misc.p, ms_d.p, 1, static_cast<int>(keep), out, head, cnt, items,
                                   reinterpret_cast<int*>(misc.p + 1), s);
        tgb::check(cudaMemcpyAsync(&err, misc.p + 1, sizeof(int), cudaMemcpyDeviceToHost, s), "error flag download");
        tgb::check(cudaStreamSynchronize(s), "shuffle draws");
        need(err == 0, "shuffle draws ran past their refill limit");
    });
}

int tgb_bin_transform(const void* X, int x_dtype, int n, int n_features, const void* edges, const int* n_edges,
                      unsigned char* codes, int stride, void* stream) {
    return guard([&] {
        need(stride >= n_features && stride % 16 == 0, "stride must be >= n_features and a multiple of 16");
        need(x_dtype == 0 || x_dtype == 1, "x_dtype must be 0 or 1");
        if (x_dtype == 0)
            tgb::launch_bin_transform_f32(static_cast<const float*>(X), n, n_features, static_cast<const float*>(edges),
                                          n_edges, codes, stride, as_stream(stream));
        else
            tgb::launch_bin_transform_f64(static_cast<const double*>(X), n, n_features,
                                          static_cast<const double*>(edges), n_edges, codes, stride,
                                          as_stream(stream));
    });
}

int tgb_hist_build(const unsigned char* codes, int stride, int n_features, const int* rows, int n_rows,
                   const double* g, const double* h, int gshift, int hshift, long long* G, long long* H, int* C,
                   void* stream) {
    return guard([&] {
        need(stride >= n_features && stride % 16 == 0, "stride must be >= n_features and a multiple of 16");
        tgb::launch_hist_rows(codes, stride, n_features, rows, n_rows, g, h, gshift, hshift, G, H, C,
                              as_stream(stream));
    });
}

int tgb_split_scan(const long long* G, const long long* H, const int* C, int n_features, int n_bins, int gshift,
                   int hshift, double l2, double min_split_gain, int min_samples_leaf, double min_child_weight,
                   double* gain, int* thr, int* missing_left, void* stream) {
    return guard([&] {
        need(n_bins >= 2 && n_bins <= 256, "n_bins must be in [2, 256]");
        tgb::launch_scan_hist(G, H, C, n_features, n_bins, std::ldexp(1.0, -gshift), std::ldexp(1.0, -hshift), l2,
                              min_split_gain, min_samples_leaf, min_child_weight, gain, thr, missing_left,
                              as_stream(stream));
    });
}

size_t tgb_partition_workspace_bytes(int n_rows) {
    const size_t tiles = static_cast<size_t>(std::max(0, n_rows) + tgb::kPartTile - 1) / tgb::kPartTile;
    return 256 + (tiles + 1) * sizeof(int);
}

int tgb_partition(const unsigned char* codes, int stride, const int* rows, int n_rows, int feature, int threshold,
                  int missing_left, int* out, int* n_left_out, void* workspace, size_t workspace_bytes,
                  void* stream) {
    return guard([&] {
        need(workspace_bytes >= tgb_partition_workspace_bytes(n_rows), "workspace too small");
        need(feature >= 0 && feature < stride, "feature out of range");
        char* ws = static_cast<char*>(workspace);  // 256-byte header (reserved), then the tile counts
        tgb::launch_partition_rows(codes, stride, rows, n_rows, feature, threshold, missing_left, out, n_left_out,
                                   reinterpret_cast<int*>(ws + 256), as_stream(stream));
    });
}

int tgb_partition_noalloc(const unsigned char* codes, int stride, const int* rows, int n_rows, int feature,
                          int threshold, int missing_left, int* out, int* n_left_out, void* stream) {
    return guard([&] {
        need(feature >= 0 && feature < stride, "feature out of range");
        tgb::launch_partition_rows_noalloc(codes, stride, rows, n_rows, feature, threshold, missing_left, out,
                                           n_left_out, as_stream(stream));
    });
}

int tgb_grad_mse(const double* y, const double* pred, int n, double* g, double* h, void* stream) {
    return guard([&] { tgb::launch_grad_mse(y, pred, n, g, h, as_stream(stream)); });
}

int tgb_grad_pairwise(const double* y, const double* pred, const int* run_start, const int* run_len, const int* order,
                      int n_runs, int n, double* g, double* h, void* stream) {
    return guard([&] {
        tgb::launch_grad_pairwise(y, pred, run_start, run_len, order, n_runs, n, g, h, as_stream(stream));
    });
}

int tgb_hist_build_quantized(const unsigned char* codes, int stride, int n_features, const int* rows, int n_rows,
                             const double* g, const double* h, int hist_bits, unsigned long long seed, long long* G,
                             long long* H, int* C, double* scales_out, void* stream) {
    return guard([&] {
        need(codes && rows && g && G && H && C && scales_out, "NULL argument");
        need(stride >= n_features && stride % 16 == 0 && n_features > 0, "bad stride");
        need(hist_bits == 0 || hist_bits == 8 || hist_bits == 16, "hist_bits must be 0, 8 or 16");
        need(n_rows >= 0, "n_rows < 0");
        cudaStream_t s = as_stream(stream);
        const bool const_h = h == nullptr;
        const int mode = tgb::hist_mode(hist_bits, const_h);
        // one root job over the caller's rows, through the fit's own quantise and wave
        // histogram kernels (a context whose sample is `rows`)
        tgb::DBuf<tgb::DevTreeState> st;
        tgb::DBuf<tgb::WaveCtl> ctl;
        tgb::DBuf<tgb::WaveCtx> wc;
        tgb::DBuf<unsigned char> gq, hq;
        int n_max = 0;
        {
            std::vector<int> rh(static_cast<size_t>(n_rows));
            if (n_rows > 0)
                tgb::check(cudaMemcpyAsync(rh.data(), rows, sizeof(int) * n_rows, cudaMemcpyDeviceToHost, s), "rows");
            tgb::check(cudaStreamSynchronize(s), "rows");
            for (int r : rh) n_max = std::max(n_max, r + 1);
        }
        st.alloc(1, s);
        ctl.alloc(1, s);
        wc.alloc(1, s);
        const int n_pay = std::max({1, n_max, n_rows});  // payloads by position in the row list
        gq.alloc(static_cast<size_t>(n_pay) * 8, s);
        if (mode == tgb::kHistExactVar) hq.alloc(static_cast<size_t>(n_pay) * 8, s);
        tgb::DevTreeState sh{};
        sh.n_sample = n_rows;
        tgb::check(cudaMemsetAsync(ctl.p, 0, sizeof(tgb::WaveCtl), s), "control reset");
        tgb::check(cudaMemcpyAsync(st.p, &sh, sizeof(sh), cudaMemcpyHostToDevice, s), "state upload");
        const int one = 1;
        tgb::check(cudaMemcpyAsync(&ctl.p->active, &one, sizeof(int), cudaMemcpyHostToDevice, s), "control");
        // sample maxima of |g| and h (the per-tree scales)
        tgb::DBuf<tgb::AllScale> all;
        all.alloc(1, s);
        tgb::check(cudaMemsetAsync(all.p, 0, sizeof(tgb::AllScale), s), "scale reset");
        tgb::launch_rows_max(rows, n_rows, g, h, all.p, s);
        tgb::launch_wave_scales(st.p, all.p, mode, s);
        tgb::launch_wave_quantize(mode, rows, g, h, nullptr, 1.0, st.p, seed, gq.p, hq.p, std::max(1, n_rows), s);
        tgb::WaveCtx w{};
        w.codes = codes;
        w.rows0 = const_cast<int32_t*>(rows);
        w.gq = gq.p;
        w.hq = hq.p;
        w.pay_pitch = n_pay;
        w.pay_bytes = tgb::hist_pay_bytes(mode);
        w.st = st.p;
        w.ctl = ctl.p;
        w.G = G;
        w.H = H;
        w.C = C;
        w.gp.n_features = n_features;
        w.gp.stride = stride;
        w.goss_scale = 1.0;
        w.codes_map_ok = tgb::encode_codes_map(&w.codes_map, codes, n_max, stride) ? 1 : 0;
        tgb::check(cudaMemcpyAsync(wc.p, &w, sizeof(w), cudaMemcpyHostToDevice, s), "context upload");
        tgb::HistTune tune;
        tune.clusters = tgb::wave_hist_clusters(tune.cluster);
        tgb::launch_wave_hist(mode, wc.p, 1, 0, tune, nullptr, s);
        tgb::check(cudaMemcpyAsync(&sh, st.p, sizeof(sh), cudaMemcpyDeviceToHost, s), "state download");
        int err = 0;
        tgb::check(cudaMemcpyAsync(&err, &ctl.p->error, sizeof(int), cudaMemcpyDeviceToHost, s), "error flag");
        tgb::check(cudaStreamSynchronize(s), "quantised histogram");
        if (err != 0) throw tgb::TideError("GPU path: the histogram's TMA staging wait gave up");
        scales_out[0] = sh.inv_gscale;
        scales_out[1] = sh.inv_hscale;
    });
}

int tgb_build_hist_gpu(tgb_booster* hb, const unsigned short* xb, int n_f, const int* idx, int n_idx, const double* g,
                       const double* h, int n_bins, int n_rows, double* out) {
    return guard([&] {
        need(hb && xb && out, "NULL argument");
        need(n_bins >= 1 && n_bins <= 256, "GPU path: n_bins must be <= 256 (uint8 codes)");
        tgb::check(cudaSetDevice(hb->b->device), "cudaSetDevice");
        const size_t hist_sz = static_cast<size_t>(n_f) * n_bins;
        std::fill(out, out + 3 * hist_sz, 0.0);
        if (n_idx <= 0) return;
        if (n_rows <= 0) n_rows = n_idx;  // histogram_cuda.cu:85-88
        const int stride = (n_f + 15) / 16 * 16;
        if (hb->host_xb != xb || hb->xb_rows != n_rows || hb->xb_f != n_f) {
            std::vector<unsigned char> c8(static_cast<size_t>(n_rows) * stride, 0);
            for (size_t i = 0; i < static_cast<size_t>(n_rows); ++i)
                for (int f = 0; f < n_f; ++f) {
                    const unsigned short v = xb[i * n_f + f];
                    if (v > 255) throw tgb::TideError("GPU path: bin code > 255");
                    c8[i * stride + f] = static_cast<unsigned char>(v);
                }
            cudaFree(hb->d_codes);
            hb->d_codes = nullptr;
            tgb::check(cudaMalloc(&hb->d_codes, c8.size()), "cudaMalloc codes");
            tgb::check(cudaMemcpy(hb->d_codes, c8.data(), c8.size(), cudaMemcpyHostToDevice), "H2D codes");
            hb->host_xb = xb;
            hb->xb_rows = n_rows;
            hb->xb_f = n_f;
            hb->xb_stride = stride;
        }
        if (hb->cap_rows < static_cast<size_t>(n_rows)) {
            cudaFree(hb->d_g);
            cudaFree(hb->d_h);
            tgb::check(cudaMalloc(&hb->d_g, sizeof(double) * n_rows), "cudaMalloc g");
            tgb::check(cudaMalloc(&hb->d_h, sizeof(double) * n_rows), "cudaMalloc h");
            hb->cap_rows = n_rows;
        }
        if (hb->cap_idx < static_cast<size_t>(n_idx)) {
            cudaFree(hb->d_idx);
            tgb::check(cudaMalloc(&hb->d_idx, sizeof(int) * n_idx), "cudaMalloc idx");
            hb->cap_idx = n_idx;
        }
        const size_t full = static_cast<size_t>(n_f) * tgb::kBins;
        if (hb->cap_hist < full) {
            cudaFree(hb->d_G);
            cudaFree(hb->d_H);
            cudaFree(hb->d_C);
            tgb::check(cudaMalloc(&hb->d_G, sizeof(long long) * full), "cudaMalloc G");
            tgb::check(cudaMalloc(&hb->d_H, sizeof(long long) * full), "cudaMalloc H");
            tgb::check(cudaMalloc(&hb->d_C, sizeof(int) * full), "cudaMalloc C");
            hb->cap_hist = full;
        }
        tgb::check(cudaMemcpy(hb->d_g, g, sizeof(double) * n_rows, cudaMemcpyHostToDevice), "H2D g");
        tgb::check(cudaMemcpy(hb->d_h, h, sizeof(double) * n_rows, cudaMemcpyHostToDevice), "H2D h");
        tgb::check(cudaMemcpy(hb->d_idx, idx, sizeof(int) * n_idx, cudaMemcpyHostToDevice), "H2D idx");
        tgb::check(cudaMemset(hb->d_G, 0, sizeof(long long) * full), "memset");
        tgb::check(cudaMemset(hb->d_H, 0, sizeof(long long) * full), "memset");
        tgb::check(cudaMemset(hb->d_C, 0, sizeof(int) * full), "memset");
        double mg = 0, mh = 0;
        for (int k = 0; k < n_idx; ++k) {
            mg = std::max(mg, std::fabs(g[idx[k]]));
            mh = std::max(mh, std::fabs(h[idx[k]]));
        }
        auto shift = [&](double mx) {
            if (!(mx > 0)) return 0;
            int clog = 0;
            while ((1ll << clog) < static_cast<long long>(n_idx)) ++clog;
            return std::max(-1000, std::min(1000, 61 - (std::ilogb(mx) + 1) - clog));
        };
        const int gs = shift(mg), hs = shift(mh);
        tgb::launch_hist_rows(hb->d_codes, stride, n_f, hb->d_idx, n_idx, hb->d_g, hb->d_h, gs, hs, hb->d_G, hb->d_H,
                              hb->d_C, nullptr);
        std::vector<long long> G(full), H(full);
        std::vector<int> C(full);
        tgb::check(cudaMemcpy(G.data(), hb->d_G, sizeof(long long) * full, cudaMemcpyDeviceToHost), "D2H G");
        tgb::check(cudaMemcpy(H.data(), hb->d_H, sizeof(long long) * full, cudaMemcpyDeviceToHost), "D2H H");
        tgb::check(cudaMemcpy(C.data(), hb->d_C, sizeof(int) * full, cudaMemcpyDeviceToHost), "D2H C");
        const double ig = std::ldexp(1.0, -gs), ih = std::ldexp(1.0, -hs);
        for (int f = 0; f < n_f; ++f)
            for (int b = 0; b < n_bins; ++b) {
                const size_t o = static_cast<size_t>(f) * n_bins + b;
                const size_t q = static_cast<size_t>(f) * tgb::kBins + b;
                out[3 * o] = static_cast<double>(G[q]) * ig;
                out[3 * o + 1] = static_cast<double>(H[q]) * ih;
                out[3 * o + 2] = static_cast<double>(C[q]);
            }
    });
}

}  // extern "C"

extern "C" {

int tgb_server_create(int device, double budget_bytes, int slots, tgb_server** out) {
    return guard([&] {
        need(out != nullptr, "out is NULL");
        need(budget_bytes >= 1.0 && slots >= 1, "budget and slots must be positive");
        auto* h = new tgb_server();
        h->device = device;
        h->sched = new tgb::Scheduler(static_cast<size_t>(budget_bytes), slots);
        *out = h;
    });
}

void tgb_server_free(tgb_server* s) { delete s; }

long long tgb_working_set_bytes(tgb_booster* b, int kind, int n, int n_features, int x_dtype) {
    if (!b || n < 0 || n_features < 1 || (kind != 0 && kind != 1)) return -1;
    return static_cast<long long>(working_set_bytes(b->b->cfg, kind, n, n_features, x_dtype));
}

int tgb_server_submit_fit(tgb_server* s, tgb_booster* hb, const void* X, int x_dtype, const double* y, int n,
                          int n_features, const long long* timestamps, const long long* entity, long long* id_out) {
    return guard([&] {
        need(s && hb && X && y && id_out, "NULL argument");
        const size_t bytes = working_set_bytes(hb->b->cfg, 0, n, n_features, x_dtype);
        tgb::GpuBooster* b = hb->b;
        const int device = s->device;
        *id_out = s->sched->submit(
            tgb::Scheduler::kFit, bytes,
            [=] {
                tgb::check(cudaSetDevice(device), "cudaSetDevice");
                b->fit(X, x_dtype, y, n, n_features, reinterpret_cast<const int64_t*>(timestamps),
                       reinterpret_cast<const int64_t*>(entity));
            },
            reinterpret_cast<uintptr_t>(b));
    });
}

int tgb_server_submit_predict(tgb_server* s, tgb_booster* hb, const void* X, int x_dtype, int n, int n_features,
                              double* out, long long* id_out) {
    return guard([&] {
        need(s && hb && X && out && id_out, "NULL argument");
        const size_t bytes = working_set_bytes(hb->b->cfg, 1, n, n_features, x_dtype);
        tgb::GpuBooster* b = hb->b;
        const int device = s->device;
        *id_out = s->sched->submit(
            tgb::Scheduler::kPredict, bytes,
            [=] {
                tgb::check(cudaSetDevice(device), "cudaSetDevice");
                b->predict_raw(X, x_dtype, n, n_features, out);
            },
            reinterpret_cast<uintptr_t>(b));
    });
}

int tgb_server_wait(tgb_server* s, long long id, double timeout_ms, int* state) {
    return guard([&] {
        need(s && state, "NULL argument");
        std::string err;
        *state = s->sched->wait(id, timeout_ms < 0 ? -1.0 : timeout_ms / 1000.0, &err);
        if (*state == tgb::Scheduler::kFailed) g_err = err;
    });
}

int tgb_server_stats(tgb_server* s, double* o) {
    return guard([&] {
        need(s && o, "NULL argument");
        const tgb::Scheduler::Stats st = s->sched->stats();
        o[0] = static_cast<double>(st.completed);
        o[1] = static_cast<double>(st.failed);
        o[2] = st.p50_s;
        o[3] = st.p99_s;
        o[4] = st.p50_fit_s;
        o[5] = st.p99_fit_s;
        o[6] = st.p50_predict_s;
        o[7] = st.p99_predict_s;
        o[8] = st.mean_wait_s;
        o[9] = static_cast<double>(st.peak_running);
        o[10] = static_cast<double>(st.peak_bytes);
        o[11] = st.busy_s;
    });
}

}  // extern "C"
