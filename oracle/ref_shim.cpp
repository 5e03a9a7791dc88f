// C-ABI shim over the reference TideGBM core, compiled together with the
// reference's own sources (see oracle/Makefile) into oracle/_ref/libtgbref.so.
//
// TEST INFRASTRUCTURE ONLY.  Nothing in the product links or loads this file;
// tests/, bench.py's reference arm and the oracle pinning tests use it to run
// the reference's CPU path on the same inputs as the CUDA path.
//
// It exposes:
//   * the whole Booster::fit (cpp/src/booster.cpp:231) with a flat key/value
//     config, and read-back of the fitted trees, init prefixes and evals;
//   * Binner::fit / transform (cpp/src/binning.cpp:34-128);
//   * build_hist_col (cpp/src/histogram.cpp:44-76);
//   * best_numeric_missing (cpp/src/histogram.cpp:144-193);
//   * Objective::grad_hess / loss (cpp/src/objective.cpp:102-329);
//   * apply_all (cpp/src/tree.cpp:43-55);
//   * a fitted Booster built from exported arrays, and Booster::save_binary /
//     load_binary (cpp/src/serialize.cpp:65-255), the .tgbm blob.
#include "tidegbm/booster.hpp"
#include "tidegbm/histogram.hpp"

#include <chrono>
#include <cstring>
#include <string>
#include <vector>

using namespace tidegbm;

namespace {
thread_local std::string g_err;

ObjectiveKind objective_from_code(int code) {
    switch (code) {
        case 0: return ObjectiveKind::MSE;
        case 5: return ObjectiveKind::RankPairwise;
        default: return static_cast<ObjectiveKind>(code);
    }
}
}  // namespace

extern "C" {

const char* ref_last_error(void) { return g_err.c_str(); }

void* ref_create(void) { return new Booster(); }
void ref_free(void* b) { delete static_cast<Booster*>(b); }

// Sets one Config field.  Unknown keys return -1.
int ref_set(void* hb, const char* key, double v) {
    Config& c = static_cast<Booster*>(hb)->cfg;
    const std::string k(key);
    if (k == "n_estimators") c.n_estimators = static_cast<int>(v);
    else if (k == "learning_rate") c.learning_rate = v;
    else if (k == "max_depth") c.max_depth = static_cast<int>(v);
    else if (k == "max_leaves") c.max_leaves = static_cast<int>(v);
    else if (k == "min_samples_leaf") c.min_samples_leaf = static_cast<int>(v);
    else if (k == "min_child_weight") c.min_child_weight = v;
    else if (k == "l2") c.l2 = v;
    else if (k == "min_split_gain") c.min_split_gain = v;
    else if (k == "max_bin") c.max_bin = static_cast<int>(v);
    else if (k == "n_time_buckets") c.n_time_buckets = static_cast<int>(v);
    else if (k == "horizon") c.horizon = static_cast<i64>(v);
    else if (k == "embargo") c.embargo = static_cast<i64>(v);
    else if (k == "iid_mode") c.iid_mode = v != 0;
    else if (k == "halo") c.halo = v != 0;
    else if (k == "pair_splits") c.pair_splits = v != 0;
    else if (k == "pair_trigger") c.pair_trigger = v;
    else if (k == "pair_top_k") c.pair_top_k = static_cast<int>(v);
    else if (k == "max_pair_splits_per_tree") c.max_pair_splits_per_tree = static_cast<int>(v);
    else if (k == "pair_l2") c.pair_l2 = v;
    else if (k == "cat_smooth") c.cat_smooth = v;
    else if (k == "cat_min_count") c.cat_min_count = static_cast<int>(v);
    else if (k == "objective") c.objective = objective_from_code(static_cast<int>(v));
    else if (k == "n_jobs") c.n_jobs = static_cast<int>(v);
    else if (k == "random_state") c.random_state = static_cast<int>(v);
    else if (k == "goss") c.goss = static_cast<int>(v);
    else if (k == "goss_top") c.goss_top = v;
    else if (k == "goss_other") c.goss_other = v;
    else if (k == "bin_sample") c.bin_sample = static_cast<int>(v);
    else if (k == "col_major_hist") c.col_major_hist = v != 0;
    else if (k == "torb_min_cover") c.torb_min_cover = v;
    else if (k == "finer_torb") c.finer_torb = v != 0;
    else if (k == "ooc_bytes") c.ooc_bytes = static_cast<size_t>(v);
    else {
        g_err = "unknown key " + k;
        return -1;
    }
    return 0;
}

int ref_fit(void* hb, const double* X, const double* y, int n, int n_f, const long long* ts,
            const long long* rank_groups, const long long* entity) {
    try {
        static_cast<Booster*>(hb)->fit(X, y, n, n_f, reinterpret_cast<const i64*>(ts), nullptr,
                                       nullptr, nullptr, nullptr,
                                       reinterpret_cast<const i64*>(rank_groups), nullptr, nullptr,
                                       nullptr, 0, reinterpret_cast<const i64*>(entity), nullptr);
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

// The same with categorical features: is_cat[f] != 0 marks feature f.
int ref_fit_cat(void* hb, const double* X, const double* y, int n, int n_f, const long long* ts,
                const long long* rank_groups, const long long* entity, const int* is_cat) {
    try {
        static_cast<Booster*>(hb)->fit(X, y, n, n_f, reinterpret_cast<const i64*>(ts), nullptr, is_cat,
                                       nullptr, nullptr, reinterpret_cast<const i64*>(rank_groups), nullptr,
                                       nullptr, nullptr, 0, reinterpret_cast<const i64*>(entity), nullptr);
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

// Booster::fit with the reference's own per-iteration hook (log_fn, called from
// booster.cpp:733-737 when verbose > 0): iter_seconds[m] = steady-clock seconds at the
// end of boosting iteration m, relative to the call.  The hook prints one line per
// iteration to stderr, as the reference does with verbose = 1.
int ref_fit_timed(void* hb, const double* X, const double* y, int n, int n_f, const long long* ts,
                  const long long* rank_groups, const long long* entity, double* iter_seconds) {
    auto* b = static_cast<Booster*>(hb);
    const auto t0 = std::chrono::steady_clock::now();
    b->cfg.verbose = 1;
    b->log_fn = [&](int iter, f64, f64) {
        iter_seconds[iter - 1] =
            std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    };
    const int rc = ref_fit(hb, X, y, n, n_f, ts, rank_groups, entity);
    b->log_fn = nullptr;
    b->cfg.verbose = 0;
    return rc;
}

int ref_predict_raw(void* hb, const double* X, int n, int n_f, double* out) {
    try {
        static_cast<Booster*>(hb)->predict_raw(X, n, n_f, out);
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

int ref_n_trees(void* hb) { return static_cast<int>(static_cast<Booster*>(hb)->trees.size()); }
int ref_n_bins(void* hb) { return static_cast<Booster*>(hb)->n_bins; }
int ref_n_time_buckets(void* hb) { return static_cast<Booster*>(hb)->n_time_buckets; }
double ref_init_score(void* hb) { return static_cast<Booster*>(hb)->init_score; }
int ref_n_evals(void* hb) { return static_cast<int>(static_cast<Booster*>(hb)->evals.train.size()); }

void ref_evals_train(void* hb, double* out) {
    const auto& v = static_cast<Booster*>(hb)->evals.train;
    std::memcpy(out, v.data(), v.size() * sizeof(double));
}

void ref_init_prefix(void* hb, double* out) {
    const auto& v = static_cast<Booster*>(hb)->init_prefix;
    std::memcpy(out, v.data(), v.size() * sizeof(double));
}

int ref_tree_n_nodes(void* hb, int t) {
    return static_cast<int>(static_cast<Booster*>(hb)->trees[t].nodes.size());
}

// Node fields as int32 [is_leaf, feature, threshold_bin, left, right, missing_go_left,
// n_samples, depth] and f64 [value, gain]; values/cover per node; prefix values
// n_buckets * n_nodes.
void ref_tree_export(void* hb, int t, int* inodes, double* fnodes, double* values, int* cover,
                     double* prefix) {
    const Tree& tr = static_cast<Booster*>(hb)->trees[t];
    const int nn = static_cast<int>(tr.nodes.size());
    for (int k = 0; k < nn; ++k) {
        const Node& d = tr.nodes[k];
        int* o = inodes + 8 * k;
        o[0] = d.is_leaf ? 1 : 0;
        o[1] = d.feature;
        o[2] = d.threshold_bin;
        o[3] = d.left;
        o[4] = d.right;
        o[5] = d.missing_go_left;
        o[6] = d.n_samples;
        o[7] = d.depth;
        fnodes[2 * k] = d.value;
        fnodes[2 * k + 1] = d.gain;
        values[k] = tr.values[k];
        cover[k] = tr.cover[k];
    }
    std::memcpy(prefix, tr.prefix_values.data(), tr.prefix_values.size() * sizeof(double));
}

// Per node the 256-bit left mask of a categorical split (Node::cat_left) into out[4*k].
void ref_tree_export_cat(void* hb, int t, unsigned long long* out) {
    const Tree& tr = static_cast<Booster*>(hb)->trees[t];
    for (size_t k = 0; k < tr.nodes.size(); ++k)
        for (int j = 0; j < 4; ++j) out[4 * k + j] = tr.nodes[k].cat_left[j];
}

// Per node {split_type (SplitType, types.hpp:25), feature2} into out[2*k].
void ref_tree_export_split(void* hb, int t, int* out) {
    const Tree& tr = static_cast<Booster*>(hb)->trees[t];
    for (size_t k = 0; k < tr.nodes.size(); ++k) {
        out[2 * k] = static_cast<int>(tr.nodes[k].split_type);
        out[2 * k + 1] = tr.nodes[k].feature2;
    }
}

int ref_edges(void* hb, int f, double* out) {
    const auto& e = static_cast<Booster*>(hb)->binner.edges[f];
    if (out) std::memcpy(out, e.data(), e.size() * sizeof(double));
    return static_cast<int>(e.size());
}

// ---- component entry points -------------------------------------------------

// Binner::fit on all rows (no mask) followed by transform into row-major u16 codes.
// edges_out: F x 256 f64 (first n_edges[f] used).
int ref_binner(const double* X, int n, int n_f, int max_bin, int bin_sample, unsigned seed,
               double* edges_out, int* n_edges, int* n_bins_col, int* max_bins,
               unsigned short* codes) {
    try {
        Binner b;
        std::vector<int> is_cat(n_f, 0);
        std::vector<u8> mask(n, 1);
        b.fit(X, n, n_f, is_cat.data(), mask.data(), max_bin, 5, bin_sample, seed);
        for (int f = 0; f < n_f; ++f) {
            n_edges[f] = static_cast<int>(b.edges[f].size());
            n_bins_col[f] = b.n_bins_col[f];
            std::memcpy(edges_out + static_cast<size_t>(f) * 256, b.edges[f].data(),
                        b.edges[f].size() * sizeof(double));
        }
        *max_bins = b.max_bins();
        if (codes) b.transform(X, n, n_f, codes);
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

// Binner::fit with categorical features (is_cat[f] != 0) and Binner::transform:
// edges_out[f] holds the vocabulary (cat_values) of a categorical feature, the edges of a
// numeric one; codes are the u16 bin codes.
int ref_binner_cat(const double* X, int n, int n_f, const int* is_cat, int max_bin, int cat_min_count,
                   int bin_sample, unsigned seed, double* edges_out, int* n_edges, int* max_bins,
                   unsigned short* codes) {
    try {
        Binner b;
        std::vector<u8> mask(n, 1);
        b.fit(X, n, n_f, is_cat, mask.data(), max_bin, cat_min_count, bin_sample, seed);
        for (int f = 0; f < n_f; ++f) {
            const std::vector<f64>& v = is_cat[f] ? b.cat_values[f] : b.edges[f];
            n_edges[f] = static_cast<int>(v.size());
            std::memcpy(edges_out + static_cast<size_t>(f) * 256, v.data(), v.size() * sizeof(double));
        }
        *max_bins = b.max_bins();
        if (codes) b.transform(X, n, n_f, codes);
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

// build_hist_col; out is interleaved {g, h, c(as f64)} per (feature, bin).
void ref_build_hist_col(const unsigned short* xcol, int n_rows, int n_f, const int* idx, int n_idx,
                        const double* g, const double* h, int n_bins, int n_jobs, double* out) {
    Hist hist;
    hist.resize(n_f, n_bins);
    build_hist_col(xcol, n_rows, n_f, idx, n_idx, g, h, hist, n_jobs);
    for (size_t i = 0; i < hist.B.size(); ++i) {
        out[3 * i] = hist.B[i].g;
        out[3 * i + 1] = hist.B[i].h;
        out[3 * i + 2] = static_cast<double>(hist.B[i].c);
    }
}

// best_numeric_missing on one feature of an interleaved {g, h, c} histogram.
// res: [gain], ires: [feature, threshold_bin, missing_go_left].
void ref_best_numeric(const double* ghc, int n_f, int n_bins, int f, double lam, double gamma,
                      int min_leaf, double min_hess, double* res, int* ires) {
    Hist hist;
    hist.resize(n_f, n_bins);
    for (size_t i = 0; i < hist.B.size(); ++i) {
        hist.B[i].g = ghc[3 * i];
        hist.B[i].h = ghc[3 * i + 1];
        hist.B[i].c = static_cast<i64>(ghc[3 * i + 2]);
    }
    SplitCand c = best_numeric_missing(hist, f, lam, gamma, min_leaf, min_hess, 0, 0.0);
    res[0] = c.gain;
    ires[0] = c.feature;
    ires[1] = c.threshold_bin;
    ires[2] = c.missing_go_left;
}

// Objective::grad_hess for MSE (kind 0) or RankPairwise (kind 5), unit weights.
void ref_grad_hess(int kind, const double* y, const double* pred, const long long* groups, int n,
                   double* g, double* h) {
    Objective o;
    o.kind = objective_from_code(kind);
    o.grad_hess(y, pred, nullptr, reinterpret_cast<const i64*>(groups), n, g, h);
}

double ref_loss(int kind, const double* y, const double* pred, const long long* groups, int n) {
    Objective o;
    o.kind = objective_from_code(kind);
    return o.loss(y, pred, nullptr, reinterpret_cast<const i64*>(groups), n);
}

// ---- a fitted model from exported arrays, and the .tgbm blob ------------------

// Fills a reference Booster with a model grown elsewhere (the GPU path's export):
// config fields the prediction and the .tgbm format read, the numeric binner
// (edges F x 256, first n_edges[f] used; n_bins_col = n_edges + 2 as Binner::fit sets
// it, binning.cpp:100), and the trees, concatenated: tree t has tree_nodes[t] nodes,
// int32 [is_leaf, feature, threshold_bin, left, right, missing_go_left, n_samples,
// depth] and f64 [value, gain] per node, values / cover per node and n_buckets x
// n_nodes prefix values.  This is what a TideGBM maintainer's import step does after
// Booster::fit dispatched to the GPU.
int ref_import_model(void* hb, int n_features, int n_bins, int n_buckets, double init_score,
                     const double* init_prefix, int n_prefix, const double* edges, const int* n_edges, int max_bin,
                     double learning_rate, int objective, int iid_mode, int n_trees, const int* tree_nodes,
                     const int* inodes, const double* fnodes, const double* values, const int* cover,
                     const double* prefix) {
    try {
        Booster& b = *static_cast<Booster*>(hb);
        b.cfg.n_estimators = n_trees;
        b.cfg.learning_rate = learning_rate;
        b.cfg.max_bin = max_bin;
        b.cfg.objective = objective_from_code(objective);
        b.cfg.iid_mode = iid_mode != 0;
        b.cfg.n_jobs = 1;
        b.obj.kind = b.cfg.objective;
        b.n_features = n_features;
        b.n_bins = n_bins;
        b.n_time_buckets = n_buckets;
        b.init_score = init_score;
        b.init_prefix.assign(init_prefix, init_prefix + n_prefix);
        b.is_cat.assign(n_features, 0);
        b.binner.max_bin = max_bin;
        b.binner.n_features = n_features;
        b.binner.is_cat.assign(n_features, 0);
        b.binner.edges.assign(n_features, {});
        b.binner.cat_values.assign(n_features, {});
        b.binner.n_bins_col.assign(n_features, 2);
        for (int f = 0; f < n_features; ++f) {
            const double* e = edges + static_cast<size_t>(f) * 256;
            b.binner.edges[f].assign(e, e + n_edges[f]);
            b.binner.n_bins_col[f] = n_edges[f] + 2;
        }
        b.trees.assign(n_trees, Tree());
        size_t off = 0;
        for (int t = 0; t < n_trees; ++t) {
            Tree& tr = b.trees[t];
            const int nn = tree_nodes[t];
            tr.n_buckets = n_buckets;
            tr.nodes.resize(nn);
            for (int k = 0; k < nn; ++k) {
                const int* o = inodes + 8 * (off + k);
                Node& d = tr.nodes[k];
                d.is_leaf = o[0] != 0;
                d.feature = o[1];
                d.threshold_bin = o[2];
                d.left = o[3];
                d.right = o[4];
                d.missing_go_left = o[5];
                d.n_samples = o[6];
                d.depth = o[7];
                d.value = fnodes[2 * (off + k)];
                d.gain = fnodes[2 * (off + k) + 1];
            }
            tr.values.assign(values + off, values + off + nn);
            tr.cover.assign(cover + off, cover + off + nn);
            tr.prefix_values.assign(prefix + off * n_buckets, prefix + (off + nn) * n_buckets);
            off += nn;
        }
        b.fitted = true;
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

// Booster::save_binary (serialize.cpp:65-148): returns the blob size; copies it when
// out != NULL and cap is large enough.
long long ref_save_binary(void* hb, char* out, long long cap) {
    try {
        const std::string blob = static_cast<Booster*>(hb)->save_binary();
        if (out && cap >= static_cast<long long>(blob.size())) std::memcpy(out, blob.data(), blob.size());
        return static_cast<long long>(blob.size());
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

// Booster::load_binary (serialize.cpp:150-255) into a new handle (NULL on error).
void* ref_load_binary(const char* blob, long long n) {
    try {
        return new Booster(Booster::load_binary(std::string(blob, static_cast<size_t>(n))));
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}

}  // extern "C"
