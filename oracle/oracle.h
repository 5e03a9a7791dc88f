/* CPU restatement of the TideGBM training hot path (test infrastructure).
 *
 * This header and oracle.cpp are the ORACLE: a plain, single-threaded CPU
 * restatement of the reference algorithm, used only by tests/, by
 * __graft_entry__.smoke() as the checker, and by bench.py's cpu_baseline leg.
 * The product (tidegbm_b200/) never links, loads or calls it.
 *
 * Every function names the reference file:line it restates (paths relative to
 * the reference project root).  Row-major uint8 bin codes are used throughout:
 * codes fit 8 bits because max_bin <= 256 (cpp/include/tidegbm/config.hpp:81)
 * and code = 1 + count(edges <= v) <= 255 (cpp/src/binning.cpp:117-118).
 */
#ifndef TIDEGBM_ORACLE_H
#define TIDEGBM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Split candidate, the fields of SplitCand (cpp/include/tidegbm/histogram.hpp:65-74)
 * that axis splits use. */
typedef struct {
    double gain;
    int feature;
    int threshold_bin;
    int missing_go_left;
} orc_split;

/* Binner::fit for numeric features with no mask (cpp/src/binning.cpp:14-32, 34-102).
 * X is row-major f64 n x n_f.  edges: n_f x 256 (first n_edges[f] used).
 * Returns Binner::max_bins() (binning.cpp:130-134). */
int orc_binner_fit(const double* X, int n, int n_f, int max_bin, int bin_sample, uint32_t seed,
                   double* edges, int* n_edges, int* n_bins_col);

/* Binner::fit + transform with categorical features (binning.cpp:34-134): edges[f]
 * (n_f x 256) holds the vocabulary of a categorical feature (is_cat[f] != 0) or the
 * edges of a numeric one, n_edges[f] its length; codes (row-major n x n_f, may be NULL)
 * the uint8 codes.  Returns max_bins(). */
int orc_binner_fit_cat(const double* X, int n, int n_f, const int* is_cat, int max_bin, int cat_min_count,
                       int bin_sample, uint32_t seed, double* edges, int* n_edges, uint8_t* codes);

/* Binner::transform (binning.cpp:104-128) into row-major uint8 codes with row
 * stride `stride` bytes. */
void orc_bin_transform(const double* X, int n, int n_f, const double* edges, const int* n_edges,
                       uint8_t* codes, int stride);

/* build_hist_col / build_hist (cpp/src/histogram.cpp:24-76) over rows idx[0..n_idx).
 * out: interleaved {g, h, c} f64 per (feature, bin), feature-major, n_f x n_bins. */
void orc_build_hist(const uint8_t* codes, int stride, int n_f, const int32_t* idx, int n_idx,
                    const double* g, const double* h, int n_bins, double* out);

/* best_numeric_missing for one feature (histogram.cpp:126-193), l1 = 0, no monotone. */
orc_split orc_best_numeric(const double* ghc, int n_bins, int f, double lam, double gamma,
                           int min_leaf, double min_hess);

/* First `keep` elements of std::shuffle(iota(m), std::mt19937(seed)) — the draw the
 * reference makes in Binner::fit (binning.cpp:93-97) and GOSS (booster.cpp:572). */
void orc_shuffle_prefix(int64_t m, int64_t keep, uint32_t seed, int32_t* out);

/* The GOSS draw sequence of Booster::fit: one std::mt19937(seed) makes n_shuffles
 * std::shuffle's of iota(m) (booster.cpp:572), each followed by grow_tree's seed draw
 * (booster.cpp:588); out[s*keep ..] holds the first keep of shuffle s. */
void orc_shuffle_sequence(int64_t m, int64_t keep, uint32_t seed, int n_shuffles, int32_t* out);

/* Objective::grad_hess for MSE (objective.cpp:105-118) and RankPairwise
 * (objective.cpp:179-219), unit weights.  kind: 0 = MSE, 5 = RankPairwise. */
void orc_grad_hess(int kind, const double* y, const double* pred, const int64_t* groups, int n,
                   double* g, double* h);

/* Objective::loss for MSE / RankPairwise (objective.cpp:262-329). */
double orc_loss(int kind, const double* y, const double* pred, const int64_t* groups, int n);

/* Fit configuration: the subset of Config (cpp/include/tidegbm/config.hpp:12-76)
 * that the oracle restates. */
typedef struct {
    int n_estimators;
    double learning_rate;
    int max_depth;
    int max_leaves;
    int min_samples_leaf;
    double min_child_weight;
    double l2;
    double min_split_gain;
    int max_bin;
    int n_time_buckets;
    int64_t horizon;
    int64_t embargo;
    int iid_mode;
    int objective; /* 0 MSE, 5 RankPairwise */
    int random_state;
    int goss;      /* -1 auto, 0 off, 1 on */
    double goss_top;
    double goss_other;
    int bin_sample;
    double torb_min_cover;
    int finer_torb;
    /* PAIR splits (config.hpp:31-35); turned off for n >= 1M as booster.cpp:237-240 does */
    int pair_splits;
    double pair_trigger;
    int pair_top_k;
    int max_pair_splits_per_tree;
    double pair_l2;
    /* categorical features (config.hpp:70-72) */
    double cat_smooth;
    int cat_min_count;
} orc_config;

void orc_config_default(orc_config* c);

/* Booster::fit (cpp/src/booster.cpp:231-742) for the supported subset.  ts may be
 * NULL only in iid mode; rank groups are the timestamps for RankPairwise; entity
 * may be NULL.  Returns a handle or NULL (orc_last_error()). */
void* orc_fit(const orc_config* cfg, const double* X, const double* y, int n, int n_f,
              const int64_t* ts, const int64_t* entity);
/* The same with categorical features: is_cat[f] != 0 marks feature f (NULL: none). */
void* orc_fit_cat(const orc_config* cfg, const double* X, const double* y, int n, int n_f,
                  const int64_t* ts, const int64_t* entity, const int* is_cat);
void orc_free(void* model);
const char* orc_last_error(void);

int orc_n_trees(void* model);
int orc_n_bins(void* model);
int orc_n_buckets(void* model);
double orc_init_score(void* model);
void orc_init_prefix(void* model, double* out);
void orc_evals_train(void* model, double* out);
int orc_tree_n_nodes(void* model, int t);
/* Same layout as the reference shim: inodes[8*k] = {is_leaf, feature, threshold_bin,
 * left, right, missing_go_left, n_samples, depth}; fnodes[2*k] = {value, gain}. */
void orc_tree_export(void* model, int t, int* inodes, double* fnodes, double* values, int* cover,
                     double* prefix);
/* Per node the 256-bit left mask of a categorical split (Node::cat_left) into out[4*k]. */
void orc_tree_export_cat(void* model, int t, uint64_t* out);
/* Per node {split_type (0 axis, 1 pair, 2 categorical; types.hpp:25), feature2} into out[2*k]. */
void orc_tree_export_split(void* model, int t, int* out);
/* Booster::predict_raw (booster.cpp:744-811) on f64 X. */
void orc_predict_raw(void* model, const double* X, int n, double* out);

#ifdef __cplusplus
}
#endif
#endif
