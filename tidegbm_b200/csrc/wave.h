// Batched tree growth ("waves").
//
// The reference grows a tree leaf-wise, one split per iteration: the leaf of largest
// cached gain is split, its smaller child histogrammed, the larger derived by
// subtraction (cpp/src/tree.cpp:343-463).  Done literally on a GPU that is one chain of
// small launches per split.  A wave does the same work for many leaves, and for many
// trees (the folds of a walk-forward split, or any set of fit contexts), per launch:
//
//   select    replays the best-first choice exactly: while the best candidate leaf
//             (largest gain, lowest node id on ties; tree.cpp:343-383) has already been
//             expanded, it is committed: node ids, children, split records, exactly as
//             the one-split loop creates them.  It stops at the first unexpanded best
//             leaf, or when the tree is done, then plans the next expansions: every
//             unexpanded leaf among the top-B candidates, B = the splits left.  No leaf
//             outside the top B can ever be chosen (the B better ones exhaust the
//             budget first), and the best one is always expanded, so every wave commits
//             at least one split and the result is the reference's tree.
//   partition the planned leaves' rows into their children (stable, tree.cpp:68-91),
//             into the other ping-pong buffer at the leaf's own row range: a leaf whose
//             expansion is never committed keeps its rows untouched.
//   histogram the smaller child of every planned leaf, one persistent cluster launch
//             over all (context, leaf) jobs: rows x feature groups cut into one
//             contiguous range per cluster.
//   scan      both children of every planned leaf (the larger by parent - smaller,
//             histogram.cpp:108-117) for their best split and their totals.
//
// Histogram slots are handed out per expansion (slot 0: the root; expansion k of a tree
// gets slots 1 + 2k and 2 + 2k), so speculative children never overwrite committed
// ones.  A tree has at most 2 * max_leaves - 1 committed nodes and each is expanded at
// most once, so 4 * max_leaves - 1 slots always suffice.
#pragma once

#include <cuda.h>

#include "tgb_internal.h"

namespace tgb {

constexpr int kMaxWaveCtx = 64;     // fit contexts per wave launch
constexpr int kMaxLeavesCap = 256;  // max_leaves limit of the GPU path
constexpr int kMaxWaveJobs = 4096;  // (context, expansion) pairs per histogram launch

// Histogram payload (what one row contributes) and its accumulation:
//   exact: 64-bit fixed point per row, exact integer sums (results match the reference)
//   q16 / q8: gradients (and hessians) stochastically rounded to 16 / 8 bits per tree,
//   summed exactly in 32-bit shared words (the precision pattern)
// const: unit hessians (mse), H is rebuilt from row counts; var: per-row hessians.
enum HistMode : int {
    kHistExactConst = 0,
    kHistExactVar = 1,
    kHistQ16Const = 2,
    kHistQ16Var = 3,
    kHistQ8Const = 4,
    kHistQ8Var = 5,
};
inline int hist_mode(int hist_bits, bool const_h) {
    const int base = hist_bits == 16 ? kHistQ16Const : hist_bits == 8 ? kHistQ8Const : kHistExactConst;
    return base + (const_h ? 0 : 1);
}
// Bytes of a row's histogram payload in `mode` (the g payload; the exact per-row mode adds
// an 8-byte h payload).
inline int hist_pay_bytes(int mode) { return mode <= kHistExactVar ? 8 : mode <= kHistQ16Var ? 4 : 2; }

// Per-tree control of one context, device resident.
struct WaveCtl {
    int splits_done;  // splits committed so far
    int n_exp;        // expansions planned by the last select
    int exp_counter;  // expansions so far in this tree (slot hand-out)
    int tiles_total;  // partition tiles of the planned expansions
    int active;       // 1 while the tree grows
    int slot0;        // first histogram slot of the planned expansions
    int error;        // a slot, buffer or wave-count bound was hit (never expected)
    int waves;        // selects run for this tree (bounded: a tree needs at most max_leaves)
    int pair_used;    // PAIR splits committed in this tree
    int exp_total;    // expansions planned over all trees of the fit (not reset per tree)
    int pad[2];
    int exp_leaf[kMaxLeavesCap];
    int exp_tile0[kMaxLeavesCap + 1];
    int exp_left[kMaxLeavesCap];     // rows of the planned leaf going left (partition count)
    int part_ticket[kMaxLeavesCap];  // count tiles done per planned leaf (zero between launches)
    int expanded[kMaxNodes];  // 0 not expanded; 1, 2: children planned by the axis, with-pairs split
};

// Everything a wave kernel needs to know about one context (device resident array).
struct WaveCtx {
    // TMA descriptor of codes (uint8 [n][stride], box: 32 bytes of one row) for the
    // histogram's gathers; used when codes_map_ok (encode_codes_map succeeded)
    CUtensorMap codes_map;
    const uint8_t* codes;      // row-major [n][stride]
    const uint8_t* codes_col;  // column-major [F][col_pitch]
    long long col_pitch;
    int32_t* rows0;
    int32_t* rows1;
    // Histogram payloads by position: the payload of the row at position k of rows buffer b
    // (rows0: b = 0, rows1: b = 1) is element b * pay_pitch + k of gq (pay_bytes bytes) and
    // of hq (8 bytes, exact per-row hessian mode only); the partition moves them with the
    // rows, so the histogram reads them in row-list order.
    void* gq;
    void* hq;
    long long pay_pitch;
    int pay_bytes;
    int pad_pay;
    DevNode* nodes;
    DevSplit* splits;
    DevTreeState* st;
    DevNode* spec;        // [2 * kMaxNodes]: children of node k at 2k, 2k + 1
    DevSplit* spec_split;  // their best splits
    WaveCtl* ctl;
    long long* G;  // histogram slots [n_slots][F][kBins]
    long long* H;
    int* C;
    double* cand_gain;  // scan candidates [(2 * kMaxNodes + 1)][F]
    int* cand_key;
    int* tickets;      // [2 * kMaxNodes + 1], zero between launches
    int* tile_counts;  // [max tiles of a wave]
    GrowParams gp;
    double goss_scale;
    int n_slots;
    int max_tiles;
    int max_expand;  // expansions a select may plan (0: every candidate ranked within the budget)
    int codes_map_ok;
    // categorical features (nullptr: none): flags per feature, the left masks of the scan
    // candidates [(2 * kMaxNodes + 1)][F][4], and the ranking's smoothing (cat_smooth)
    const uint8_t* is_cat;
    unsigned long long* cand_cat;
    double cat_smooth;
    // PAIR splits (tree.cpp:214-281; pair_on 0: off).  A leaf whose best axis gain is weak
    // against its gradient energy also tries the pairs of its top-k features through the
    // histogram of the hashed code pair; splits_pair / spec_split_pair hold the best split
    // with those pairs (the split a leaf takes while the tree's pair budget lasts), splits /
    // spec_split the one without.  energy: per candidate index, fixed point (2^-energy_shift
    // of the rows' sum of g^2); pair_cand: per candidate index and pair, the pair's best.
    int pair_on;
    int pair_top_k;
    int max_pair;
    int pad_pair;
    double pair_trigger;
    double pair_l2;
    const double* g;           // the rows' gradients (the tree's g before GOSS scaling)
    const uint8_t* goss_flag;  // GOSS classes (nullptr: no GOSS); class 2 rows are scaled
    DevSplit* splits_pair;
    DevSplit* spec_split_pair;
    unsigned long long* energy;  // [2 * kMaxNodes + 1]
    DevSplit* pair_cand;         // [(2 * kMaxNodes + 1)][kMaxPairs]
    int* pair_tickets;           // [2 * kMaxNodes + 1], zero between launches
};
constexpr int kMaxPairs = 15;  // pairs of the top pair_top_k <= 6 features

// Per-tree set-up of one context: root node (all sampled rows, slot 0), control reset.
// use_dev_count: the sample size is st->n_sample (GOSS), else n_sample_host.
void launch_wave_tree_init(DevNode* nodes, DevSplit* splits, DevTreeState* st, WaveCtl* ctl, int n_sample_host,
                           int use_dev_count, cudaStream_t s);
// Per-tree histogram scales of one context from the sample maxima (st) or, when the
// sample is every row, the all-row maxima (all).
void launch_wave_scales(DevTreeState* st, const AllScale* all, int mode, cudaStream_t s);
// Payload of the sampled rows for `mode` (rows0[0 .. st->n_sample)), by position in rows0.
void launch_wave_quantize(int mode, const int32_t* rows, const double* g, const double* h, const uint8_t* goss_flag,
                          double goss_scale, const DevTreeState* st, unsigned long long seed, void* gq, void* hq,
                          int max_rows, cudaStream_t s);

// Wave launches over n_ctx contexts (ctxs: device array).  src 0: the roots, src 1: the
// expansions planned by the last select.
// Launch shape of the histogram: `cluster` CTAs per cluster (1, 2 or 4: how many private
// histograms one flush merges through distributed shared memory), `clusters` clusters
// (co-resident).  Picked by the autotuner.
struct HistTune {
    int cluster = 4;
    int clusters = 37;
};
int wave_hist_clusters(int cluster);  // co-resident clusters of the histogram kernel
// codes_map for a row-major uint8 code matrix [n_rows][stride]: false (map zeroed) where
// TMA cannot address it (stride not a multiple of 16 or below 32 bytes, base not 16-byte
// aligned, no driver entry point); the histogram then loads code rows directly.
bool encode_codes_map(CUtensorMap* map, const uint8_t* codes, long long n_rows, int stride);
void launch_wave_hist(int mode, const WaveCtx* ctxs, int n_ctx, int src, HistTune tune,
                      unsigned long long* rows_counter, cudaStream_t s);
void launch_wave_scan(const WaveCtx* ctxs, int n_ctx, int src, int max_f, int ys, bool any_cat, cudaStream_t s);
// gsync: 2 device ints (flag, ticket), zero.  host_flag: mapped host word or nullptr;
// cond / use_cond: the graph's loop condition (set to "any context still growing").
void launch_wave_select(const WaveCtx* ctxs, int n_ctx, int* gsync, unsigned* host_flag,
                        unsigned long long cond, int use_cond, cudaStream_t s);
void launch_wave_partition(const WaveCtx* ctxs, int n_ctx, int grid, cudaStream_t s);
// PAIR stage after a scan (contexts with pair_on): the children's (or roots') gradient
// energy, then for the weak ones the pair histograms and their best splits, merged into
// spec_split_pair (roots: splits_pair[0]).
void launch_wave_pair(const WaveCtx* ctxs, int n_ctx, int src, cudaStream_t s);
// sc->maxg_bits / maxh_bits <- max |g[rows]| and max h[rows] (h == nullptr: 1); sc zeroed.
void launch_rows_max(const int32_t* rows, int n_rows, const double* g, const double* h, AllScale* sc,
                     cudaStream_t s);

}  // namespace tgb
