// CPU restatement of the TideGBM training hot path — TEST INFRASTRUCTURE ONLY.
//
// Used by tests/, by __graft_entry__.smoke() as the checker and by bench.py's
// cpu_baseline leg.  The product never links or calls it.  Single-threaded,
// written for clarity; every function names the reference file:line it
// restates (paths relative to the reference project root).  Compiled with
// -ffp-contract=off so the FP64 arithmetic follows the reference's statement
// order exactly.
//
// Library dependency: the reference draws its random samples with libstdc++'s
// std::mt19937 + std::shuffle and orders GOSS candidates with std::sort; this
// restatement calls the same library routines with the same arguments, so the
// same libstdc++ (GCC 13 here) gives the same samples.
#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

thread_local std::string g_err;

struct OrcNode {
    int is_leaf = 1;
    int feature = -1;
    int threshold_bin = -1;
    int left = -1;
    int right = -1;
    int missing_go_left = 1;
    double value = 0.0;
    double gain = 0.0;
    int n_samples = 0;
    int depth = 0;
    int split_type = 0;  // SplitType (cpp/include/tidegbm/types.hpp:25): 0 axis, 1 pair, 2 categorical
    int feature2 = -1;   // second feature of a pair split
    uint64_t cat_left[4] = {0, 0, 0, 0};  // categorical split: codes that go left (bit 0: missing)
};

struct OrcTree {
    std::vector<OrcNode> nodes;
    std::vector<double> values;
    std::vector<int> cover;
    std::vector<double> prefix;
};

struct OrcModel {
    orc_config cfg;
    int n_f = 0;
    int n_bins = 0;
    int n_buckets = 1;
    double init_score = 0.0;
    std::vector<double> init_prefix;
    std::vector<double> edges;  // n_f x 256
    std::vector<int> n_edges;
    std::vector<int> is_cat;                     // per feature
    std::vector<std::vector<double>> cat_values;  // vocabulary of each categorical feature
    std::vector<OrcTree> trees;
    std::vector<double> evals;
};

inline bool is_nan(double v) { return !(v == v); }

// cpp/src/binning.cpp:14-32
std::vector<double> quantile_edges(std::vector<double>& vals, int n_bins) {
    std::sort(vals.begin(), vals.end());
    vals.erase(std::unique(vals.begin(), vals.end()), vals.end());
    if (vals.empty()) return {0.0};
    if (static_cast<int>(vals.size()) <= n_bins) return vals;
    std::vector<double> e;
    for (int i = 1; i < n_bins; ++i) {
        const double q = static_cast<double>(i) / n_bins;
        const double pos = q * (vals.size() - 1);
        const size_t lo = static_cast<size_t>(pos);
        const size_t hi = std::min(lo + 1, vals.size() - 1);
        const double frac = pos - lo;
        e.push_back(vals[lo] * (1 - frac) + vals[hi] * frac);
    }
    std::sort(e.begin(), e.end());
    e.erase(std::unique(e.begin(), e.end()), e.end());
    return e;
}

// The numeric edges of feature f (cpp/src/binning.cpp:86-100): its non-NaN values, the
// std::shuffle sample when there are more than bin_sample, quantile_edges.
std::vector<double> numeric_edges(const double* X, int n, int n_f, int f, int max_bin, int bin_sample,
                                  uint32_t seed) {
    std::vector<double> vals;
    vals.reserve(n);
    for (int i = 0; i < n; ++i) {
        const double v = X[static_cast<size_t>(i) * n_f + f];
        if (!is_nan(v)) vals.push_back(v);
    }
    if (bin_sample > 0 && static_cast<int>(vals.size()) > bin_sample) {
        std::mt19937 rng(seed + static_cast<uint32_t>(f) * 2654435761u);
        std::shuffle(vals.begin(), vals.end(), rng);
        vals.resize(static_cast<size_t>(bin_sample));
    }
    return quantile_edges(vals, max_bin - 1);
}

// The vocabulary of categorical feature f (cpp/src/binning.cpp:47-84): its distinct
// non-NaN values seen at least cat_min_count times (else the most frequent one); the
// max_bin - 1 most frequent when there are more; ascending.
std::vector<double> cat_vocabulary(const double* X, int n, int n_f, int f, int max_bin, int cat_min_count) {
    std::vector<double> raw;
    raw.reserve(n);
    for (int i = 0; i < n; ++i) {
        const double v = X[static_cast<size_t>(i) * n_f + f];
        if (!is_nan(v)) raw.push_back(v);
    }
    std::sort(raw.begin(), raw.end());
    std::vector<std::pair<int, double>> freq;
    for (size_t i = 0; i < raw.size();) {
        size_t j = i + 1;
        while (j < raw.size() && raw[j] == raw[i]) ++j;
        freq.emplace_back(static_cast<int>(j - i), raw[i]);
        i = j;
    }
    const int min_c = std::max(1, cat_min_count);
    std::vector<std::pair<int, double>> kept;
    for (const auto& q : freq)
        if (q.first >= min_c) kept.push_back(q);
    if (kept.empty() && !freq.empty())
        kept.push_back(*std::max_element(freq.begin(), freq.end(),
                                         [](const auto& a, const auto& b) { return a.first < b.first; }));
    const int numeric_bins = max_bin - 1;
    if (static_cast<int>(kept.size()) > numeric_bins) {
        std::partial_sort(kept.begin(), kept.begin() + numeric_bins, kept.end(),
                          [](const auto& a, const auto& b) { return a.first > b.first; });
        kept.resize(numeric_bins);
    }
    std::vector<double> uniq;
    uniq.reserve(kept.size());
    for (const auto& q : kept) uniq.push_back(q.second);
    std::sort(uniq.begin(), uniq.end());
    return uniq;
}

// cpp/include/tidegbm/tree.hpp:53-67 with l1 = 0 and max_delta_step = 0.
inline double leaf_value(double G, double H, double l2) { return -G / (H + l2); }

// cpp/src/histogram.cpp:126-134 with l1 = 0.
inline double leaf_score(double G, double H, double lam) { return (G * G) / (H + lam); }

// pair_bin (cpp/include/tidegbm/histogram.hpp:81-85): the two codes hashed into one of
// n_bins bins, in 32-bit unsigned arithmetic.
inline int pair_bin(int b1, int b2, int n_bins) {
    return static_cast<int>((static_cast<uint32_t>(b1) * 2654435761u + static_cast<uint32_t>(b2) * 40503u) %
                            static_cast<uint32_t>(n_bins));
}

// Direction of one row at a split node: cpp/src/tree.cpp:21-28 (pair: missing if either
// code is missing, else the hashed bin against the threshold) and :36-39 (axis).
inline bool goes_left(const OrcNode& d, const uint8_t* row, int n_bins) {
    if (d.split_type == 2) {  // cat_goes_left, cpp/include/tidegbm/tree.hpp:27-30 (codes are < 256)
        const int b = row[d.feature];
        return (d.cat_left[b >> 6] >> (b & 63)) & 1ull;
    }
    if (d.split_type == 1) {
        const int b1 = row[d.feature], b2 = row[d.feature2];
        if (b1 == 0 || b2 == 0) return d.missing_go_left != 0;
        return pair_bin(b1, b2, n_bins) <= d.threshold_bin;
    }
    const int b = row[d.feature];
    return (b == 0) ? d.missing_go_left != 0 : b <= d.threshold_bin;
}

// cpp/src/tree.cpp:15-41 for axis, pair and categorical splits on uint8 codes.
int apply_one(const OrcTree& t, const uint8_t* row, int n_bins) {
    int nid = 0;
    for (;;) {
        const OrcNode& d = t.nodes[nid];
        if (d.is_leaf) return nid;
        nid = goes_left(d, row, n_bins) ? d.left : d.right;
    }
}

// cpp/src/objective.cpp:18-39
void group_runs(const int64_t* groups, int n, std::vector<int>& idx,
                std::vector<std::pair<int, int>>& runs) {
    idx.resize(n);
    std::iota(idx.begin(), idx.end(), 0);
    bool sorted = true;
    for (int i = 1; i < n; ++i)
        if (groups[i] < groups[i - 1]) {
            sorted = false;
            break;
        }
    if (!sorted)
        std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return groups[a] < groups[b]; });
    runs.clear();
    int i = 0;
    while (i < n) {
        int j = i + 1;
        while (j < n && groups[idx[j]] == groups[idx[i]]) ++j;
        runs.emplace_back(i, j - i);
        i = j;
    }
}

// cpp/src/booster.cpp:36-58
int auto_time_buckets(const int64_t* ts, int n, int64_t horizon, int uniq_cap) {
    std::vector<int64_t> u(ts, ts + n);
    std::sort(u.begin(), u.end());
    u.erase(std::unique(u.begin(), u.end()), u.end());
    int64_t step = 1;
    if (u.size() >= 2) {
        std::vector<int64_t> d;
        for (size_t i = 1; i < u.size(); ++i)
            if (u[i] - u[i - 1] > 0) d.push_back(u[i] - u[i - 1]);
        if (!d.empty()) {
            std::nth_element(d.begin(), d.begin() + d.size() / 2, d.end());
            step = std::max<int64_t>(d[d.size() / 2], 1);
        }
    }
    const int h_steps = static_cast<int>(std::max<int64_t>(horizon, 0) / step);
    const int want = h_steps >= 8 ? 64 : 32;
    return std::max(2, std::min(want, std::max(uniq_cap, 2)));
}

// Binner::fit (binning.cpp:34-102) into the model: edges of the numeric features, the
// vocabularies of the categorical ones.  Returns max_bins() (binning.cpp:130-134).
int model_binner_fit(OrcModel* M, const double* X, int n, int n_f, const orc_config& c) {
    M->edges.assign(static_cast<size_t>(n_f) * 256, 0.0);
    M->n_edges.assign(n_f, 0);
    M->cat_values.assign(n_f, {});
    int mx = 2;
    for (int f = 0; f < n_f; ++f) {
        int nbc;
        if (M->is_cat[f]) {
            M->cat_values[f] = cat_vocabulary(X, n, n_f, f, c.max_bin, c.cat_min_count);
            nbc = static_cast<int>(M->cat_values[f].size()) + 1;
        } else {
            const std::vector<double> e =
                numeric_edges(X, n, n_f, f, c.max_bin, c.bin_sample, static_cast<uint32_t>(c.random_state));
            M->n_edges[f] = static_cast<int>(e.size());
            std::copy(e.begin(), e.end(), M->edges.begin() + static_cast<size_t>(f) * 256);
            nbc = static_cast<int>(e.size()) + 2;
        }
        mx = std::max(mx, nbc);
    }
    return std::max(mx, c.max_bin);
}

// Binner::transform (binning.cpp:104-128): numeric code = 1 + upper_bound(edges, v);
// categorical code = 1 + the value's vocabulary index, 0 when it is not in the vocabulary;
// NaN -> 0.
void model_transform(const OrcModel& M, const double* X, int n, uint8_t* codes) {
    const int n_f = M.n_f;
    for (int i = 0; i < n; ++i)
        for (int f = 0; f < n_f; ++f) {
            const double v = X[static_cast<size_t>(i) * n_f + f];
            int b = 0;
            if (!is_nan(v)) {
                if (M.is_cat[f]) {
                    const auto& voc = M.cat_values[f];
                    auto it = std::lower_bound(voc.begin(), voc.end(), v);
                    if (it != voc.end() && *it == v) b = static_cast<int>(it - voc.begin()) + 1;
                } else {
                    const double* e = M.edges.data() + static_cast<size_t>(f) * 256;
                    b = static_cast<int>(std::upper_bound(e, e + M.n_edges[f], v) - e) + 1;
                }
            }
            codes[static_cast<size_t>(i) * n_f + f] = static_cast<uint8_t>(b);
        }
}

// A split candidate: orc_split plus the PAIR and categorical fields of SplitCand
// (cpp/include/tidegbm/histogram.hpp:65-74).
struct Cand {
    orc_split s{-1e300, -1, -1, 1};
    int type = 0;
    int feature2 = -1;
    uint64_t cat_left[4] = {0, 0, 0, 0};
};

// best_categorical (cpp/src/histogram.cpp:195-244) with l1 = 0: the non-empty bins (the
// missing bin 0 included) ordered by g / (h + cat_smooth) with std::sort, then the best
// prefix of that order as the left side.  missing_go_left is the missing bin's side.
Cand best_categorical(const double* ghc, int n_bins, int f, double lam, double gamma, int min_leaf,
                      double min_hess, double cat_smooth) {
    Cand best;
    const double* B = ghc + static_cast<size_t>(f) * n_bins * 3;
    std::vector<int> order;
    order.reserve(n_bins);
    double totG = 0, totH = 0;
    int64_t totC = 0;
    for (int b = 0; b < n_bins; ++b) {
        totG += B[3 * b];
        totH += B[3 * b + 1];
        totC += static_cast<int64_t>(B[3 * b + 2]);
        if (static_cast<int64_t>(B[3 * b + 2]) > 0) order.push_back(b);
    }
    if (order.size() < 2) return best;
    const double sm = std::max(cat_smooth, 0.0);
    std::sort(order.begin(), order.end(), [&](int a, int b) {
        return B[3 * a] / (B[3 * a + 1] + sm) < B[3 * b] / (B[3 * b + 1] + sm);
    });
    const double parent = leaf_score(totG, totH, lam);
    double GL = 0, HL = 0;
    int64_t CL = 0;
    uint64_t mask[4] = {0, 0, 0, 0};
    for (size_t i = 0; i + 1 < order.size(); ++i) {
        const int b = order[i];
        GL += B[3 * b];
        HL += B[3 * b + 1];
        CL += static_cast<int64_t>(B[3 * b + 2]);
        mask[b >> 6] |= (uint64_t(1) << (b & 63));
        const double GR = totG - GL, HR = totH - HL;
        const int64_t CR = totC - CL;
        if (CL < min_leaf || CR < min_leaf) continue;
        if (HL < min_hess || HR < min_hess) continue;
        const double gain = 0.5 * (leaf_score(GL, HL, lam) + leaf_score(GR, HR, lam) - parent) - gamma;
        if (gain > best.s.gain) {
            best.s = orc_split{gain, f, -1, (mask[0] & 1ull) ? 1 : 0};
            best.type = 2;
            for (int k = 0; k < 4; ++k) best.cat_left[k] = mask[k];
        }
    }
    return best;
}

// cpp/src/tree.cpp:283-472, axis and PAIR splits (no colsample, groups, HALO, regime,
// interaction constraints, monotone, forced pairs).  Rows are sorted ascending first.
OrcTree grow_tree(const uint8_t* codes, int stride, const double* g, const double* h,
                  std::vector<int32_t> sample, int n_f, int n_bins, const orc_config& c, const std::vector<int>& is_cat) {
    OrcTree tree;
    std::sort(sample.begin(), sample.end());
    const int nb_stride = n_bins;
    OrcNode root;
    root.n_samples = static_cast<int>(sample.size());
    double sg = 0, sh = 0;
    for (int32_t i : sample) {
        sg += g[i];
        sh += h[i];
    }
    root.value = leaf_value(sg, sh, c.l2);
    tree.nodes.push_back(root);
    std::vector<std::vector<int32_t>> leaf_idx(1, sample);
    std::vector<std::vector<double>> leaf_hist(1);
    leaf_hist[0].assign(static_cast<size_t>(n_f) * nb_stride * 3, 0.0);
    orc_build_hist(codes, stride, n_f, sample.data(), static_cast<int>(sample.size()), g, h, n_bins,
                   leaf_hist[0].data());
    std::vector<Cand> cached(1);
    std::vector<char> ok(1, 0);

    auto best_for_leaf = [&](int lid, int pair_budget) {
        // cpp/src/tree.cpp:106-166: the best axis or categorical split over the features in
        // ascending order
        std::vector<Cand> per_c(n_f);
        std::vector<orc_split> per_f(n_f);
        for (int f = 0; f < n_f; ++f) {
            if (is_cat[f]) {
                per_c[f] = best_categorical(leaf_hist[lid].data(), n_bins, f, c.l2, c.min_split_gain,
                                            c.min_samples_leaf, c.min_child_weight, c.cat_smooth);
            } else {
                per_c[f].s = orc_best_numeric(leaf_hist[lid].data(), n_bins, f, c.l2, c.min_split_gain,
                                              c.min_samples_leaf, c.min_child_weight);
            }
            per_f[f] = per_c[f].s;
        }
        Cand best;
        for (int f = 0; f < n_f; ++f) {
            if (per_f[f].feature < 0 || per_f[f].gain < c.min_split_gain) continue;
            if (per_f[f].gain > best.s.gain) best = per_c[f];
        }
        // cpp/src/tree.cpp:214-281: PAIR when the best axis gain is weak against the leaf's
        // gradient energy (sum of g^2 in row order, tree.cpp:355-356)
        const std::vector<int32_t>& ix = leaf_idx[lid];
        double energy = 0;
        for (int32_t i : ix) energy += g[i] * g[i];
        const bool weak = (best.s.gain < c.pair_trigger * std::max(energy * 0.01, 1e-12)) || best.s.gain <= 0;
        if (c.pair_splits && pair_budget > 0 && n_f >= 2 && weak) {
            std::vector<int> top(n_f);
            std::iota(top.begin(), top.end(), 0);
            std::sort(top.begin(), top.end(), [&](int a, int b) { return per_f[a].gain > per_f[b].gain; });
            const int k = std::min(c.pair_top_k, n_f);
            std::vector<double> hz(static_cast<size_t>(n_bins) * 3);
            for (int a = 0; a < k; ++a)
                for (int b = a + 1; b < k; ++b) {
                    const int f1 = top[a], f2 = top[b];
                    std::fill(hz.begin(), hz.end(), 0.0);
                    for (int32_t i : ix) {
                        const uint8_t* row = codes + static_cast<size_t>(i) * stride;
                        double* B = hz.data() + 3 * static_cast<size_t>(pair_bin(row[f1], row[f2], n_bins));
                        B[0] += g[i];
                        B[1] += h[i];
                        B[2] += 1;
                    }
                    Cand cand;
                    cand.s = orc_best_numeric(hz.data(), n_bins, 0, c.pair_l2, c.min_split_gain, c.min_samples_leaf,
                                              c.min_child_weight);
                    cand.s.feature = f1;
                    cand.type = 1;
                    cand.feature2 = f2;
                    if (cand.s.gain > best.s.gain) best = cand;
                }
        }
        return best;
    };
    int pair_used = 0;

    for (int iter = 0; iter < c.max_leaves - 1; ++iter) {
        int best_leaf = -1;
        Cand bestc;
        double best_score = c.min_split_gain;
        for (int lid = 0; lid < static_cast<int>(tree.nodes.size()); ++lid) {
            if (!tree.nodes[lid].is_leaf) continue;
            if (tree.nodes[lid].depth >= c.max_depth) continue;
            if (static_cast<int>(leaf_idx[lid].size()) < 2 * c.min_samples_leaf) continue;
            if (!ok[lid]) {
                cached[lid] = best_for_leaf(lid, c.max_pair_splits_per_tree - pair_used);
                ok[lid] = 1;
            }
            const Cand& rec = cached[lid];
            if (rec.s.feature >= 0 && rec.s.gain >= c.min_split_gain && rec.s.gain > best_score) {
                best_score = rec.s.gain;
                best_leaf = lid;
                bestc = rec;
            }
        }
        if (best_leaf < 0) break;
        const orc_split& best = bestc.s;
        OrcNode& p = tree.nodes[best_leaf];
        p.is_leaf = 0;
        p.feature = best.feature;
        p.feature2 = bestc.feature2;
        p.split_type = bestc.type;
        for (int k = 0; k < 4; ++k) p.cat_left[k] = bestc.cat_left[k];
        p.threshold_bin = best.threshold_bin;
        p.missing_go_left = best.missing_go_left;
        p.gain = best.gain;
        if (bestc.type == 1) {  // tree.cpp:393-396: a pair split re-scores every leaf
            pair_used += 1;
            std::fill(ok.begin(), ok.end(), 0);
        }
        ok[best_leaf] = 0;
        // cpp/src/tree.cpp:68-91 stable partition
        std::vector<int32_t> L, R;
        for (int32_t i : leaf_idx[best_leaf]) {
            const bool left = goes_left(tree.nodes[best_leaf], codes + static_cast<size_t>(i) * stride, n_bins);
            (left ? L : R).push_back(i);
        }
        OrcNode nl, nr;
        nl.depth = nr.depth = p.depth + 1;
        nl.n_samples = static_cast<int>(L.size());
        nr.n_samples = static_cast<int>(R.size());
        auto fill_val = [&](OrcNode& nd, const std::vector<int32_t>& ix) {
            double G = 0, H = 0;
            for (int32_t i : ix) {
                G += g[i];
                H += h[i];
            }
            nd.value = leaf_value(G, H, c.l2);
        };
        fill_val(nl, L);
        fill_val(nr, R);
        // cpp/src/tree.cpp:418-436: build the smaller child, subtract for the other.
        const bool left_small = L.size() <= R.size();
        const std::vector<int32_t>& small_ix = left_small ? L : R;
        std::vector<double> small(leaf_hist[best_leaf].size(), 0.0);
        orc_build_hist(codes, stride, n_f, small_ix.data(), static_cast<int>(small_ix.size()), g, h,
                       n_bins, small.data());
        std::vector<double> big = std::move(leaf_hist[best_leaf]);
        for (size_t k = 0; k < big.size(); ++k) big[k] -= small[k];
        const int left_id = static_cast<int>(tree.nodes.size());
        tree.nodes[best_leaf].left = left_id;
        tree.nodes[best_leaf].right = left_id + 1;
        tree.nodes.push_back(nl);
        tree.nodes.push_back(nr);
        leaf_idx.push_back(std::move(L));
        leaf_idx.push_back(std::move(R));
        if (left_small) {
            leaf_hist.push_back(std::move(small));
            leaf_hist.push_back(std::move(big));
        } else {
            leaf_hist.push_back(std::move(big));
            leaf_hist.push_back(std::move(small));
        }
        leaf_hist[best_leaf].clear();
        leaf_idx[best_leaf].clear();
        cached.resize(tree.nodes.size());
        ok.resize(tree.nodes.size(), 0);
    }
    const size_t nn = tree.nodes.size();
    tree.values.resize(nn);
    tree.cover.resize(nn);
    for (size_t k = 0; k < nn; ++k) {
        tree.values[k] = tree.nodes[k].value;
        tree.cover[k] = tree.nodes[k].n_samples;
    }
    return tree;
}

}  // namespace

extern "C" {

const char* orc_last_error(void) { return g_err.c_str(); }

int orc_binner_fit(const double* X, int n, int n_f, int max_bin, int bin_sample, uint32_t seed,
                   double* edges, int* n_edges, int* n_bins_col) {
    // cpp/src/binning.cpp:34-102, numeric features, mask all ones.
    int mx = 2;
    for (int f = 0; f < n_f; ++f) {
        const std::vector<double> e = numeric_edges(X, n, n_f, f, max_bin, bin_sample, seed);
        n_edges[f] = static_cast<int>(e.size());
        std::memcpy(edges + static_cast<size_t>(f) * 256, e.data(), e.size() * sizeof(double));
        n_bins_col[f] = static_cast<int>(e.size()) + 2;
        mx = std::max(mx, n_bins_col[f]);
    }
    return std::max(mx, max_bin);  // binning.cpp:130-134
}

int orc_binner_fit_cat(const double* X, int n, int n_f, const int* is_cat, int max_bin, int cat_min_count,
                       int bin_sample, uint32_t seed, double* edges, int* n_edges, uint8_t* codes) {
    // cpp/src/binning.cpp:34-134 with categorical features.
    OrcModel M;
    M.n_f = n_f;
    M.is_cat.assign(is_cat, is_cat + n_f);
    orc_config c;
    orc_config_default(&c);
    c.max_bin = max_bin;
    c.cat_min_count = cat_min_count;
    c.bin_sample = bin_sample;
    c.random_state = static_cast<int>(seed);
    const int nb = model_binner_fit(&M, X, n, n_f, c);
    for (int f = 0; f < n_f; ++f) {
        const std::vector<double> v =
            is_cat[f] ? M.cat_values[f]
                      : std::vector<double>(M.edges.begin() + static_cast<size_t>(f) * 256,
                                            M.edges.begin() + static_cast<size_t>(f) * 256 + M.n_edges[f]);
        n_edges[f] = static_cast<int>(v.size());
        std::copy(v.begin(), v.end(), edges + static_cast<size_t>(f) * 256);
    }
    if (codes) model_transform(M, X, n, codes);
    return nb;
}

void orc_bin_transform(const double* X, int n, int n_f, const double* edges, const int* n_edges,
                       uint8_t* codes, int stride) {
    // cpp/src/binning.cpp:104-128: code = 1 + upper_bound(edges, v); NaN -> 0.
    for (int i = 0; i < n; ++i)
        for (int f = 0; f < n_f; ++f) {
            const double v = X[static_cast<size_t>(i) * n_f + f];
            int b = 0;
            if (!is_nan(v)) {
                const double* e = edges + static_cast<size_t>(f) * 256;
                b = static_cast<int>(std::upper_bound(e, e + n_edges[f], v) - e) + 1;
            }
            codes[static_cast<size_t>(i) * stride + f] = static_cast<uint8_t>(b);
        }
}

void orc_build_hist(const uint8_t* codes, int stride, int n_f, const int32_t* idx, int n_idx,
                    const double* g, const double* h, int n_bins, double* out) {
    // cpp/src/histogram.cpp:44-76 (per feature, rows in idx order).
    std::memset(out, 0, sizeof(double) * 3 * static_cast<size_t>(n_f) * n_bins);
    for (int f = 0; f < n_f; ++f) {
        double* B = out + static_cast<size_t>(f) * n_bins * 3;
        for (int k = 0; k < n_idx; ++k) {
            const int32_t i = idx[k];
            const int b = codes[static_cast<size_t>(i) * stride + f];
            B[3 * b] += g[i];
            B[3 * b + 1] += h[i];
            B[3 * b + 2] += 1.0;
        }
    }
}

orc_split orc_best_numeric(const double* ghc, int n_bins, int f, double lam, double gamma,
                           int min_leaf, double min_hess) {
    // cpp/src/histogram.cpp:144-193 with l1 = 0 and monotone = 0.
    orc_split best{-1e300, -1, -1, 1};
    const double* B = ghc + static_cast<size_t>(f) * n_bins * 3;
    double totG = 0, totH = 0;
    int64_t totC = 0;
    for (int b = 0; b < n_bins; ++b) {
        totG += B[3 * b];
        totH += B[3 * b + 1];
        totC += static_cast<int64_t>(B[3 * b + 2]);
    }
    const double missG = B[0], missH = B[1];
    const int64_t missC = static_cast<int64_t>(B[2]);
    const double parent = leaf_score(totG, totH, lam);
    double GL = 0, HL = 0;
    int64_t CL = 0;
    for (int b = 1; b < n_bins - 1; ++b) {
        const int64_t cb = static_cast<int64_t>(B[3 * b + 2]);
        GL += B[3 * b];
        HL += B[3 * b + 1];
        CL += cb;
        if (cb == 0) continue;
        for (int ml = 0; ml <= 1; ++ml) {
            const double gL = GL + (ml ? missG : 0);
            const double hL = HL + (ml ? missH : 0);
            const int64_t cL = CL + (ml ? missC : 0);
            const double gR = totG - gL, hR = totH - hL;
            const int64_t cR = totC - cL;
            if (cL < min_leaf || cR < min_leaf) continue;
            if (hL < min_hess || hR < min_hess) continue;
            const double gain =
                0.5 * (leaf_score(gL, hL, lam) + leaf_score(gR, hR, lam) - parent) - gamma;
            if (gain > best.gain) best = orc_split{gain, f, b, ml};
        }
    }
    return best;
}

void orc_shuffle_prefix(int64_t m, int64_t keep, uint32_t seed, int32_t* out) {
    std::vector<int32_t> v(static_cast<size_t>(m));
    std::iota(v.begin(), v.end(), 0);
    std::mt19937 rng(seed);
    std::shuffle(v.begin(), v.end(), rng);
    std::copy(v.begin(), v.begin() + keep, out);
}

void orc_shuffle_sequence(int64_t m, int64_t keep, uint32_t seed, int n_shuffles, int32_t* out) {
    std::mt19937 rng(seed);
    std::vector<int32_t> v(static_cast<size_t>(m));
    for (int s = 0; s < n_shuffles; ++s) {
        std::iota(v.begin(), v.end(), 0);
        std::shuffle(v.begin(), v.end(), rng);  // booster.cpp:572
        std::copy(v.begin(), v.begin() + keep, out + static_cast<size_t>(s) * keep);
        (void)rng();                            // booster.cpp:588
    }
}

void orc_grad_hess(int kind, const double* y, const double* pred, const int64_t* groups, int n,
                   double* g, double* h) {
    if (kind == 0) {  // objective.cpp:105-118, w = 1, no cost terms
        for (int i = 0; i < n; ++i) {
            g[i] = 1.0 * (pred[i] - y[i]);
            h[i] = 1.0;
        }
        return;
    }
    // objective.cpp:179-219
    std::fill(g, g + n, 0.0);
    std::fill(h, h + n, 1e-6);
    if (!groups) return;
    std::vector<int> idx;
    std::vector<std::pair<int, int>> runs;
    group_runs(groups, n, idx, runs);
    for (const auto& r : runs) {
        const int* ix = idx.data() + r.first;
        const int m = r.second;
        if (m < 2) continue;
        const int step = m > 48 ? std::max(1, m / 24) : 1;
        for (int a = 0; a < m; ++a)
            for (int b = a + step; b < m; b += step) {
                const int i = ix[a], j = ix[b];
                if (y[i] == y[j]) continue;
                int hi = i, lo = j;
                if (y[j] > y[i]) {
                    hi = j;
                    lo = i;
                }
                const double s = pred[hi] - pred[lo];
                const double e = std::exp(std::clamp(1.0 * s, -30.0, 30.0));
                const double dyw = std::max(std::abs(y[hi] - y[lo]), 1e-6);
                const double lam = -1.0 / (1.0 + e) * dyw;
                const double d2 = 1.0 * 1.0 * e / ((1 + e) * (1 + e)) * dyw;
                g[hi] += 1.0 * lam;
                g[lo] -= 1.0 * lam;
                h[hi] += 1.0 * d2;
                h[lo] += 1.0 * d2;
            }
    }
}

double orc_loss(int kind, const double* y, const double* pred, const int64_t* groups, int n) {
    if (kind == 5 && groups) {  // objective.cpp:290-322
        std::vector<int> idx;
        std::vector<std::pair<int, int>> runs;
        group_runs(groups, n, idx, runs);
        double acc = 0;
        int ng = 0;
        for (const auto& r : runs) {
            const int* ix = idx.data() + r.first;
            const int m = r.second;
            if (m < 3) continue;
            double my = 0, mp = 0;
            for (int k = 0; k < m; ++k) {
                my += y[ix[k]];
                mp += pred[ix[k]];
            }
            my /= m;
            mp /= m;
            double vy = 0, vp = 0, cc = 0;
            for (int k = 0; k < m; ++k) {
                const double dy = y[ix[k]] - my, dp = pred[ix[k]] - mp;
                vy += dy * dy;
                vp += dp * dp;
                cc += dy * dp;
            }
            if (vy > 1e-18 && vp > 1e-18) {
                acc += cc / std::sqrt(vy * vp);
                ng += 1;
            }
        }
        return ng > 0 ? -acc / ng : 0.0;
    }
    double s = 0, sw = 0;  // objective.cpp:323-328
    for (int i = 0; i < n; ++i) {
        const double d = pred[i] - y[i];
        s += 1.0 * d * d;
        sw += 1.0;
    }
    return sw > 0 ? s / sw : 0;
}

void orc_config_default(orc_config* c) {
    // Defaults of cpp/include/tidegbm/config.hpp:13-76.
    c->n_estimators = 100;
    c->learning_rate = 0.1;
    c->max_depth = 6;
    c->max_leaves = 31;
    c->min_samples_leaf = 20;
    c->min_child_weight = 1e-3;
    c->l2 = 1.0;
    c->min_split_gain = 0.0;
    c->max_bin = 255;
    c->n_time_buckets = 0;
    c->horizon = -1;
    c->embargo = 0;
    c->iid_mode = 0;
    c->objective = 0;
    c->random_state = 0;
    c->goss = -1;
    c->goss_top = 0.2;
    c->goss_other = 0.1;
    c->bin_sample = 262144;
    c->torb_min_cover = 0.0;
    c->finer_torb = 1;
    c->pair_splits = 1;
    c->pair_trigger = 0.25;
    c->pair_top_k = 6;
    c->max_pair_splits_per_tree = 3;
    c->pair_l2 = 2.0;
    c->cat_smooth = 1.0;
    c->cat_min_count = 5;
}

void* orc_fit(const orc_config* cfgp, const double* X_in, const double* y_in, int n, int n_f,
              const int64_t* ts_in, const int64_t* ent_in) {
    return orc_fit_cat(cfgp, X_in, y_in, n, n_f, ts_in, ent_in, nullptr);
}

void* orc_fit_cat(const orc_config* cfgp, const double* X_in, const double* y_in, int n, int n_f,
                  const int64_t* ts_in, const int64_t* ent_in, const int* is_cat) {
    // cpp/src/booster.cpp:231-742 for the supported subset.
    try {
        orc_config c = *cfgp;
        if (n >= 1000000) c.pair_splits = 0;  // booster.cpp:237-240 (no forced pairs here)
        if (!c.iid_mode && c.horizon < 0) throw std::runtime_error("horizon is required in time mode");
        if (!c.iid_mode && !ts_in) throw std::runtime_error("timestamp is required unless iid_mode");
        auto* M = new OrcModel();
        M->cfg = c;
        M->n_f = n_f;
        if (is_cat) M->is_cat.assign(is_cat, is_cat + n_f);  // booster.cpp:246-247
        else M->is_cat.assign(n_f, 0);
        std::vector<double> X(X_in, X_in + static_cast<size_t>(n) * n_f), y(y_in, y_in + n);
        std::vector<int64_t> ts;
        if (ts_in) ts.assign(ts_in, ts_in + n);
        // booster.cpp:264-309 stable sort by (ts, entity)
        if (!c.iid_mode && n > 1) {
            std::vector<int> ord(n);
            std::iota(ord.begin(), ord.end(), 0);
            std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) {
                if (ts_in[a] != ts_in[b]) return ts_in[a] < ts_in[b];
                if (ent_in) return ent_in[a] < ent_in[b];
                return a < b;
            });
            for (int i = 0; i < n; ++i) {
                const int s = ord[i];
                std::memcpy(&X[static_cast<size_t>(i) * n_f], X_in + static_cast<size_t>(s) * n_f,
                            sizeof(double) * n_f);
                y[i] = y_in[s];
                ts[i] = ts_in[s];
            }
        }
        // booster.cpp:311-331 TORB buckets
        std::vector<int32_t> bucket(n, 0);
        int nbk = 1;
        int64_t embargo = c.embargo;
        if (!c.iid_mode) {
            std::vector<int64_t> u(ts);
            std::sort(u.begin(), u.end());
            u.erase(std::unique(u.begin(), u.end()), u.end());
            const int uniq_n = std::max(2, static_cast<int>(u.size()));
            int want = c.n_time_buckets;
            if (want <= 0) want = auto_time_buckets(ts.data(), n, std::max<int64_t>(c.horizon, 0), uniq_n);
            nbk = c.finer_torb ? std::max(2, std::min(want, uniq_n)) : std::max(2, want);
            // booster.cpp:60-72 on already-sorted rows: rank = row position.
            for (int i = 0; i < n; ++i) {
                int b = static_cast<int>(static_cast<double>(i) / std::max(n, 1) * nbk);
                if (b >= nbk) b = nbk - 1;
                bucket[i] = b;
            }
            embargo += std::max<int64_t>(c.horizon, 0);
        }
        M->n_buckets = nbk;
        // booster.cpp:337-364 prefix cuts
        std::vector<int> cut(nbk, 0);
        if (!c.iid_mode && n > 0) {
            std::vector<int> first(nbk, -1);
            for (int i = 0; i < n; ++i)
                if (first[bucket[i]] < 0) first[bucket[i]] = i;
            int run = 0;
            for (int b = 0; b < nbk; ++b) {
                int ct = 0;
                if (first[b] >= 0) {
                    const int64_t lim = ts[first[b]] - embargo;
                    ct = static_cast<int>(std::lower_bound(ts.begin(), ts.end(), lim) - ts.begin());
                }
                run = std::max(run, ct);
                cut[b] = run;
            }
        }
        // booster.cpp:378-383 binning
        M->n_bins = model_binner_fit(M, X.data(), n, n_f, c);
        std::vector<uint8_t> codes(static_cast<size_t>(n) * n_f);
        model_transform(*M, X.data(), n, codes.data());
        // booster.cpp:399-457 initial predictions (Objective::init_score,
        // objective.cpp:80-100: mean for MSE, 0 for ranking).
        auto init_of = [&](int m) -> double {
            if (c.objective == 5 || m <= 0) return 0.0;
            double sw = 0, sy = 0;
            for (int i = 0; i < m; ++i) {
                sw += 1.0;
                sy += 1.0 * y[i];
            }
            return sw > 0 ? sy / sw : 0;
        };
        std::vector<double> pred(n);
        M->init_prefix.assign(nbk, 0.0);
        if (c.iid_mode) {
            M->init_score = init_of(n);
            std::fill(pred.begin(), pred.end(), M->init_score);
        } else {
            for (int b = 0; b < nbk; ++b) M->init_prefix[b] = cut[b] > 0 ? init_of(cut[b]) : NAN;
            M->init_score = init_of(n);
            for (int b = 0; b < nbk; ++b)
                if (!std::isfinite(M->init_prefix[b])) M->init_prefix[b] = M->init_score;
            for (int i = 0; i < n; ++i) pred[i] = M->init_prefix[bucket[i]];
        }
        const int64_t* groups = (c.objective == 5) ? ts.data() : nullptr;
        std::mt19937 rng(static_cast<uint32_t>(c.random_state));
        std::vector<double> g(n), h(n);
        for (int m = 0; m < c.n_estimators; ++m) {
            orc_grad_hess(c.objective, y.data(), pred.data(), groups, n, g.data(), h.data());
            // booster.cpp:519-585 sampling: subsample = 1 keeps all rows; GOSS.
            std::vector<int32_t> sample(n);
            std::iota(sample.begin(), sample.end(), 0);
            std::vector<double> gg, hg;
            const double* gu = g.data();
            const double* hu = h.data();
            const bool use_goss = (c.goss > 0) || (c.goss < 0 && n >= 250000);
            if (use_goss && c.goss_top < 1.0 && sample.size() > 64) {
                gg = g;
                hg = h;
                std::vector<int32_t> order = sample;
                std::sort(order.begin(), order.end(),
                          [&](int32_t a, int32_t b) { return std::abs(g[a]) > std::abs(g[b]); });
                const int n_top = std::min(static_cast<int>(order.size()),
                                           std::max(1, static_cast<int>(std::ceil(c.goss_top * sample.size()))));
                std::vector<char> keep(n, 0);
                for (int i = 0; i < n_top; ++i) keep[order[i]] = 1;
                std::vector<int32_t> rest(order.begin() + n_top, order.end());
                int n_other = static_cast<int>(std::ceil(c.goss_other * sample.size()));
                n_other = std::min(n_other, static_cast<int>(rest.size()));
                std::shuffle(rest.begin(), rest.end(), rng);
                const double scale = (1.0 - c.goss_top) / std::max(c.goss_other, 1e-12);
                for (int i = 0; i < n_other; ++i) {
                    keep[rest[i]] = 1;
                    gg[rest[i]] *= scale;
                    hg[rest[i]] *= scale;
                }
                sample.clear();
                for (int32_t i : order)
                    if (keep[i]) sample.push_back(i);
                std::sort(sample.begin(), sample.end());
                gu = gg.data();
                hu = hg.data();
            }
            OrcTree tree = grow_tree(codes.data(), n_f, gu, hu, sample, n_f, M->n_bins, c, M->is_cat);
            (void)rng();  // booster.cpp:588 seeds grow_tree's own generator
            // booster.cpp:589-600 full-data leaf values from unscaled g, h
            std::vector<int> nid(n);
            for (int i = 0; i < n; ++i) nid[i] = apply_one(tree, codes.data() + static_cast<size_t>(i) * n_f, M->n_bins);
            const int nn = static_cast<int>(tree.nodes.size());
            std::vector<double> Gs(nn, 0), Hs(nn, 0);
            tree.cover.assign(nn, 0);
            for (int i = 0; i < n; ++i) {
                Gs[nid[i]] += g[i];
                Hs[nid[i]] += h[i];
                tree.cover[nid[i]] += 1;
            }
            for (int k = 0; k < nn; ++k) tree.values[k] = leaf_value(Gs[k], Hs[k], c.l2);
            // booster.cpp:604-648 TORB prefix values
            tree.prefix.assign(static_cast<size_t>(nbk) * nn, 0.0);
            if (c.iid_mode) {
                for (int b = 0; b < nbk; ++b)
                    for (int k = 0; k < nn; ++k) tree.prefix[static_cast<size_t>(b) * nn + k] = tree.values[k];
            } else {
                const double min_cover = c.torb_min_cover > 0.0
                                             ? c.torb_min_cover
                                             : static_cast<double>(2 * std::max(c.min_samples_leaf, 1));
                std::vector<double> pG(nn, 0), pH(nn, 0);
                int swept = 0;
                for (int b = 0; b < nbk; ++b) {
                    for (; swept < cut[b]; ++swept) {
                        pG[nid[swept]] += g[swept];
                        pH[nid[swept]] += h[swept];
                    }
                    const double cover = static_cast<double>(cut[b]);
                    const double alpha = cover <= 0.0 ? 0.0 : std::min(1.0, cover / std::max(min_cover, 1.0));
                    for (int k = 0; k < nn; ++k) {
                        const double full = tree.values[k];
                        const double pref = cover > 0.0 ? leaf_value(pG[k], pH[k], c.l2) : full;
                        tree.prefix[static_cast<size_t>(b) * nn + k] = alpha * pref + (1.0 - alpha) * full;
                    }
                }
            }
            // booster.cpp:655-664
            for (int i = 0; i < n; ++i) {
                if (c.iid_mode) pred[i] += c.learning_rate * tree.values[nid[i]];
                else pred[i] += c.learning_rate * tree.prefix[static_cast<size_t>(bucket[i]) * nn + nid[i]];
            }
            M->trees.push_back(std::move(tree));
            M->evals.push_back(orc_loss(c.objective, y.data(), pred.data(), groups, n));  // booster.cpp:704-706
        }
        return M;
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}

void orc_free(void* m) { delete static_cast<OrcModel*>(m); }
int orc_n_trees(void* m) { return static_cast<int>(static_cast<OrcModel*>(m)->trees.size()); }
int orc_n_bins(void* m) { return static_cast<OrcModel*>(m)->n_bins; }
int orc_n_buckets(void* m) { return static_cast<OrcModel*>(m)->n_buckets; }
double orc_init_score(void* m) { return static_cast<OrcModel*>(m)->init_score; }
void orc_init_prefix(void* m, double* out) {
    const auto& v = static_cast<OrcModel*>(m)->init_prefix;
    std::memcpy(out, v.data(), v.size() * sizeof(double));
}
void orc_evals_train(void* m, double* out) {
    const auto& v = static_cast<OrcModel*>(m)->evals;
    std::memcpy(out, v.data(), v.size() * sizeof(double));
}
int orc_tree_n_nodes(void* m, int t) {
    return static_cast<int>(static_cast<OrcModel*>(m)->trees[t].nodes.size());
}
void orc_tree_export(void* m, int t, int* inodes, double* fnodes, double* values, int* cover,
                     double* prefix) {
    const OrcTree& tr = static_cast<OrcModel*>(m)->trees[t];
    for (size_t k = 0; k < tr.nodes.size(); ++k) {
        const OrcNode& d = tr.nodes[k];
        int* o = inodes + 8 * k;
        o[0] = d.is_leaf;
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
    std::memcpy(prefix, tr.prefix.data(), tr.prefix.size() * sizeof(double));
}

void orc_tree_export_cat(void* m, int t, uint64_t* out) {
    const OrcTree& tr = static_cast<OrcModel*>(m)->trees[t];
    for (size_t k = 0; k < tr.nodes.size(); ++k)
        for (int j = 0; j < 4; ++j) out[4 * k + j] = tr.nodes[k].cat_left[j];
}

void orc_tree_export_split(void* m, int t, int* out) {
    const OrcTree& tr = static_cast<OrcModel*>(m)->trees[t];
    for (size_t k = 0; k < tr.nodes.size(); ++k) {
        out[2 * k] = tr.nodes[k].split_type;
        out[2 * k + 1] = tr.nodes[k].feature2;
    }
}

void orc_predict_raw(void* mp, const double* X, int n, double* out) {
    // booster.cpp:744-773 with tree_decay = 1 and best_iteration = n_estimators.
    const OrcModel& M = *static_cast<OrcModel*>(mp);
    std::vector<uint8_t> codes(static_cast<size_t>(n) * M.n_f);
    model_transform(M, X, n, codes.data());
    for (int i = 0; i < n; ++i) {
        double s = M.init_score;
        for (const OrcTree& t : M.trees)
            s += M.cfg.learning_rate * t.values[apply_one(t, codes.data() + static_cast<size_t>(i) * M.n_f, M.n_bins)];
        out[i] = s;
    }
}

}  // extern "C"
