// Internal declarations shared by the CUDA kernels (.cu) and the host runtime.
//
// Device data layout of one fit context (all resident in HBM):
//   codes       uint8 row-major [n][stride], stride = round_up(F, 16): one 16-byte
//               aligned row per sample, gathered whole by the histogram kernel
//   y, pred, g, h         f64 [n]
//   rows[2]     int32 [n] ping-pong row lists; every tree node owns a contiguous
//               segment [start, start+count) of one of them
//   hist slot per node: G int64 [F][256], H int64 [F][256], C int32 [F][256]
//               fixed-point sums (value * 2^shift), exact and order independent
//   nodes       DevNode[kMaxNodes], splits DevSplit[kMaxNodes], DevTreeState
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace tgb {

constexpr int kBins = 256;       // histogram width (codes are uint8)
constexpr int kMaxNodes = 511;   // max_leaves <= 256
constexpr int kPartTile = 2048;  // rows per partition tile

struct DevNode {
    int32_t start, count, buf, depth;
    int32_t is_leaf, feature, threshold, missing_left;
    int32_t left, right, parent, slot;  // slot: histogram slot (wave engine)
    double gain;        // split gain (internal nodes)
    double value;       // leaf value from the node's sample sums (Node::value)
    long long G, H, C;  // fixed-point sample sums
    int32_t type;       // split type (SplitType, cpp/include/tidegbm/types.hpp:25): 0 axis, 1 pair, 2 categorical
    int32_t feature2;   // pair split: the second feature
    unsigned long long cat[4];  // categorical split: the codes that go left (bit b: code b)
};

struct DevSplit {
    double gain;
    int feature, threshold, missing_left, valid;
    int type, feature2;
    unsigned long long cat[4];
};

#if defined(__CUDACC__)
#define TGB_HD __host__ __device__
#else
#define TGB_HD
#endif

// pair_bin (cpp/include/tidegbm/histogram.hpp:81-85): two codes hashed into one of n_bins
// bins in 32-bit unsigned arithmetic.
TGB_HD inline unsigned pair_bin(unsigned b1, unsigned b2, int n_bins) {
    return (b1 * 2654435761u + b2 * 40503u) % static_cast<unsigned>(n_bins);
}

// Routing of a row at a split node (cpp/include/tidegbm/tree.hpp:27-30, tree.cpp:15-41):
// categorical nodes test the code's bit of the left mask; pair nodes send a row missing
// either code by the learned direction, else compare the hashed pair bin; axis nodes send
// missing (code 0) by the learned direction and codes up to the threshold left.  code2:
// the row's code of the second feature (pair nodes only).
TGB_HD inline bool goes_left(int type, const unsigned long long* cat, int threshold, int missing_left, unsigned code,
                             unsigned code2 = 0u, int n_bins = 1) {
    if (type == 2) return (cat[code >> 6] >> (code & 63)) & 1ull;
    if (type == 1) {
        if (code == 0u || code2 == 0u) return missing_left != 0;
        return static_cast<int>(pair_bin(code, code2, n_bins)) <= threshold;
    }
    return code == 0u ? missing_left != 0 : static_cast<int>(code) <= threshold;
}

struct DevTreeState {
    int n_nodes;
    int done;
    int parent;  // node split in the current iteration
    int small_node, large_node;
    int n_left;
    int gshift, hshift;
    double gscale, hscale, inv_gscale, inv_hscale;
    unsigned long long max_abs_g_bits, max_h_bits;  // reductions for the scales
    int n_sample;
    int pad;
};

// Fixed-point scale for sums over all rows (post-tree leaf values).
struct AllScale {
    unsigned long long maxg_bits, maxh_bits;
    int gshift, hshift;
    double gscale, hscale, inv_gscale, inv_hscale;
};

struct PartJob {
    const int32_t* in;    // row list (nullptr: rows 0..count-1)
    int32_t* out;
    const uint8_t* flag;  // compaction mode: keep rows with flag != 0
    int* n_left_out;      // optional copy of n_left
    const uint8_t* col;   // column-major codes [F][col_n] (nullptr: read the row-major codes)
    long long col_n;
    int count;
    int feature, threshold, missing_left;
    int left_only;
    int pad;
};

struct GrowParams {
    int n_features;
    int stride;
    int n_bins;  // Binner::max_bins()
    int max_depth;
    int max_leaves;
    int min_samples_leaf;
    double min_child_weight;
    double l2;
    double min_split_gain;
};

struct PostParams {
    int n;
    int n_buckets;
    int iid_mode;
    int n_segments;
    double learning_rate;
    double l2;
    double min_cover;
};

struct HistSlotPtrs {
    long long* G;
    long long* H;
    int* C;
    size_t slot_elems;  // F * kBins
};

struct GossWork {
    void* keys_in;   // per row: 32-bit keys (fast path) or 64-bit |g| bit patterns (exact path)
    void* keys_out;
    int32_t* vals_in;
    int32_t* vals_out;
    void* cub_tmp;
    size_t cub_tmp_bytes;
    int* overflow;   // device flag: a run of equal 32-bit keys was too long to fix up
    bool exact;
};

void check(cudaError_t e, const char* what);

#if defined(__CUDACC__)
// Programmatic dependent launch.  A kernel launched with launch_pdl may start while the
// previous kernel of its stream is still running: before pdl_wait() it may only touch
// its own registers and shared memory; pdl_wait() returns once the previous kernel has
// completed and its writes are visible.  pdl_trigger() lets the next such kernel launch
// (its own pdl_wait() still waits for this kernel to complete).  Outside a programmatic
// launch both are no-ops.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

template <typename... KArgs, typename... Args>
inline void launch_pdl(void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s, const char* what,
                       Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    check(cudaLaunchKernelEx(&cfg, kern, static_cast<KArgs>(args)...), what);
}
#endif

// Device memory from the current device's stream-ordered pool, which keeps freed blocks
// for later allocations of the process (repeated fits do not map fresh pages each time).
// Both calls are ordered on `s` and do not wait: the block may be used by work queued on
// `s` after the allocation (other streams only after synchronising with `s`), and it
// returns to the pool once the work queued on `s` before the free has completed.  No
// other stream or host thread waits for either call, so boosters on their own streams
// (the serving loop) never stall one another through allocation.
void* device_alloc(size_t bytes, cudaStream_t s);
cudaError_t device_free(void* p, cudaStream_t s);

// Owning device buffer, allocated and freed in the order of one stream (freed on scope
// exit: the block returns to the pool once the stream's earlier work is done).
template <class T>
struct DBuf {
    T* p = nullptr;
    size_t n = 0;
    cudaStream_t s = nullptr;
    DBuf() = default;
    DBuf(const DBuf&) = delete;
    DBuf& operator=(const DBuf&) = delete;
    void alloc(size_t k, cudaStream_t stream) {
        release();
        s = stream;
        if (k) p = static_cast<T*>(device_alloc(k * sizeof(T), stream));
        n = k;
    }
    void release() {
        T* q = p;
        p = nullptr;
        n = 0;
        if (q) check(device_free(q, s), "cudaFreeAsync");
    }
    ~DBuf() {
        if (p) (void)device_free(p, s);  // no throw from a destructor; release() reports errors
    }
};

// binning (kernels_bin.cu)
// is_cat: device flags per feature (nullptr: every feature numeric); a categorical feature's
// "edges" are its sorted vocabulary.
void launch_bin_transform_f32(const float* X, int n, int n_f, const float* edges, const int* n_edges,
                              uint8_t* codes, int stride, cudaStream_t s, const uint8_t* is_cat = nullptr);
void launch_bin_transform_f64(const double* X, int n, int n_f, const double* edges, const int* n_edges,
                              uint8_t* codes, int stride, cudaStream_t s, const uint8_t* is_cat = nullptr);

// device half of Binner::fit (kernels_binfit.cu); X walks use chunks of kFitChunk rows
constexpr int kFitChunk = 4096;
void launch_nonnan_counts(const void* X, int x_dtype, int n, int n_f, int* counts, cudaStream_t s);
void launch_keep_bits(const int32_t* keep, int bin_sample, int n_f, const uint8_t* take_all, uint32_t* bits,
                      long long words, cudaStream_t s);

// prefixes of std::shuffle(iota(ms[r]), std::mt19937(seeds[r])) (kernels_shuffle.cu):
// out[r][0..keep) for every range with ms[r] >= max(keep, 2^16) or ms[r] == keep;
// ranges with ms[r] == 0 are skipped (their rows of out are left to the caller).
// out and cnt must hold -1 and 0 (launch_shuffle_prefix sets them); head and items are
// scratch of n_ranges * keep ints, cnt of n_ranges * (keep + 1).  *err is set when a
// range runs past its refill limit.
void launch_shuffle_prefix(const uint32_t* seeds, const long long* ms, int n_ranges, int keep, int32_t* out,
                           int32_t* head, int32_t* cnt, int32_t* items, int* err, cudaStream_t s);
// kc, kbase: scratch of (chunks x n_f) ints; total[f]: the values gathered for feature f.
void launch_sample_gather(const void* X, int x_dtype, int n, int n_f, const long long* base, const long long* m,
                          const uint32_t* bits, long long words, const uint8_t* take_all, void* sample, long long cap,
                          int* kc, int* kbase, int* total, cudaStream_t s);
size_t sample_sort_bytes(int x_dtype, long long total, int n_f);
void launch_sample_sort(int x_dtype, const void* in, void* out, long long total, int n_f, const int* seg_begin,
                        const int* seg_end, void* tmp, size_t tmp_bytes, cudaStream_t s);
// flags[f] = 1: the feature's edges depend on std::sort's order of equal values (both zero
// signs in the sample, or infinities with interpolated edges); the host recomputes them.
void launch_quantile_edges(int x_dtype, const void* sorted, void* uniq, long long cap, const int* cnt, int n_f,
                           int n_bins, double* edges, int* n_edges, int* flags, cudaStream_t s);

// histograms + tree state (kernels_hist.cu)
// const_h (mse): reads gq from launch_quantize (int64 per row) or, with q8, from
// launch_quantize8 (int16 per row); otherwise g, h and goss_flag.
void launch_hist_node(const uint8_t* codes, int stride, int n_f, int32_t* const* rows, const DevNode* nodes,
                      const DevTreeState* st, int node, const double* g, const double* h, const void* gq, bool q8,
                      const uint8_t* goss_flag, double goss_scale, HistSlotPtrs hs, int grid_rows,
                      unsigned long long* rows_counter, bool const_h, cudaStream_t s);
// int8 precision mode: gq8[r] = (q << 1) | GOSS-scaled, q the stochastically rounded
// g * factor * st->gscale in [-127, 127]; seed varies per tree.
void launch_quantize8(const int32_t* rows, const double* g, const uint8_t* goss_flag, double goss_scale,
                      const DevTreeState* st, unsigned long long seed, short* gq8, int max_rows, cudaStream_t s);
// gq[r] = (rint(g[r] * goss_factor * st->gscale) << 1) | GOSS-scaled, for the st->n_sample
// rows of rows[] (the tree's sample); run after launch_scales.
void launch_quantize(const int32_t* rows, const double* g, const uint8_t* goss_flag, double goss_scale,
                     const DevTreeState* st, long long* gq, int max_rows, cudaStream_t s);
void launch_hist_rows(const uint8_t* codes, int stride, int n_f, const int32_t* rows, int n_rows,
                      const double* g, const double* h, int gshift, int hshift, long long* G, long long* H,
                      int* C, cudaStream_t s);
void launch_tree_init(DevNode* nodes, DevSplit* splits, DevTreeState* st, int n_sample_host, int use_dev_count,
                      cudaStream_t s);
void launch_iota_rows(int32_t* rows, int n, cudaStream_t s);
// Per-tree histogram scales from the sample maxima in st (reduced by the GOSS mark), or,
// when the sample is every row, from the all-row maxima in `all`.  q8: the int8 precision
// mode's gradient scale (127 / max |g * factor|) instead of a power-of-two shift.
void launch_scales(DevTreeState* st, const AllScale* all, bool q8, cudaStream_t s);
// Row chunks per feature group of a histogram launch (const_h: a multiple of the cluster size).
int hist_grid_rows(int n_f, int max_rows, bool const_h);

// split scan + selection (kernels_split.cu); mode 0 = node `node`, 1 = children of st->parent
// (the large child's histogram is derived as parent - small child on the way).  With
// do_select the launch ends with the next leaf choice (nodes, splits, st updated).
// ScanScratch: per-CTA candidates (2 x scan_ctas_per_node) and 3 ticket counters that
// must start at zero (the kernel leaves them at zero).
struct ScanScratch {
    double* gain;
    int* key;
    int* ticket;
};
int scan_ctas_per_node(int n_f);
void launch_split_scan(const GrowParams& p, HistSlotPtrs hs, DevNode* nodes, DevSplit* splits, DevTreeState* st,
                       int mode, int node, ScanScratch sc, bool do_select, cudaStream_t s);
void launch_scan_hist(const long long* G, const long long* H, const int* C, int n_f, int n_bins,
                      double inv_gscale, double inv_hscale, double lam, double gamma, int min_leaf,
                      double min_hess, double* gain, int* thr, int* ml, cudaStream_t s);

// partition (kernels_part.cu); tile_counts: device scratch of ceil(rows / kPartTile) ints.
// Tree mode: the job is the split of st->parent read from the node table.
void launch_partition(const uint8_t* codes, int stride, const uint8_t* codes_col, long long n_rows_total,
                      int32_t* const* rows, DevNode* nodes, DevTreeState* st, int* tile_counts, int max_tiles,
                      cudaStream_t s);
// Column-major copy of the row-major codes: col[f * codes_col_pitch(n) + r] = codes[r][f].
inline long long codes_col_pitch(int n) { return (static_cast<long long>(n) + 15) / 16 * 16; }
void launch_codes_transpose(const uint8_t* codes, int stride, int n, int n_f, uint8_t* col, cudaStream_t s);
void launch_partition_rows(const uint8_t* codes, int stride, const int32_t* rows, int n_rows, int feature,
                           int threshold, int missing_left, int32_t* out, int* n_left_dev, int* tile_counts,
                           cudaStream_t s);
void launch_compact_flagged(const uint8_t* flag, int n, int32_t* out, int* n_out_dev, int* tile_counts,
                            cudaStream_t s);
// Same partition with its scratch in a fixed device array of kernels_part.cu (no allocation).
int partition_noalloc_max_rows();
void launch_partition_rows_noalloc(const uint8_t* codes, int stride, const int32_t* rows, int n_rows, int feature,
                                   int threshold, int missing_left, int32_t* out, int* n_left_dev, cudaStream_t s);

// objectives (kernels_obj.cu)
void launch_grad_mse(const double* y, const double* pred, int n, double* g, double* h, cudaStream_t s);
// g = pred - y, sc <- max |g| and max h = 1 (reset first).
void launch_grad_mse_fused(const double* y, const double* pred, int n, double* g, AllScale* sc, cudaStream_t s);
void launch_grad_pairwise(const double* y, const double* pred, const int* run_start, const int* run_len,
                          const int* order, int n_runs, int n, double* g, double* h, cudaStream_t s);
void launch_loss_mse(const double* y, const double* pred, int n, double* partials, int n_part, cudaStream_t s);
void launch_loss_pairwise(const double* y, const double* pred, const int* run_start, const int* run_len,
                          const int* order, int n_runs, double* corr, int* valid, cudaStream_t s);
void launch_loss_finalize(int kind, const double* partials, const int* valid, int n_part, int n,
                          double* out, cudaStream_t s);

// GOSS (kernels_goss.cu)
size_t goss_cub_bytes(int n, bool exact);
void launch_goss_iota(int32_t* vals, int n, cudaStream_t s);  // w.vals_in, once per fit
// all: the all-row maxima of the tree's gradients (the 32-bit sort keys are relative to max |g|);
// min_rest: the smallest of rest_pos[0..n_other).
void launch_goss_select(const double* g, const double* h, int n, int n_top, int n_other, const int32_t* rest_pos,
                        int min_rest, GossWork& w, const AllScale* all, double goss_scale, uint8_t* goss_flag,
                        int32_t* rows0, int* tile_counts, DevTreeState* st, cudaStream_t s);

// post-tree sweep (kernels_post.cu)
void launch_all_scale(const double* g, const double* h, int n, AllScale* sc, cudaStream_t s);
void launch_all_scale_finalize(AllScale* sc, int n, cudaStream_t s);
// pred += lr * prefix[bucket][leaf] and per-block sums of (pred - y)^2 into partials[n_part].
// g, sc (mse only, may be null): the next tree's gradient and its maxima from the same pass.
void launch_pred_update_loss(const PostParams& pp, const int16_t* nid, const double* prefix, const DevTreeState* st,
                             double* pred, const double* y, double* partials, int n_part, double* g, AllScale* sc,
                             cudaStream_t s);
// col: column-major codes (col[f * pitch + r], launch_codes_transpose)
void launch_apply_accum(const uint8_t* col, long long pitch, int n_f, const DevNode* nodes, const DevTreeState* st,
                        const double* g, const double* h, const int4* chunks, int n_chunks, const AllScale* sc,
                        int16_t* nid, unsigned long long* seg_sums, int n_segments, int n_bins, int kinds,
                        cudaStream_t s);
void launch_finalize_tree(const PostParams& pp, const DevTreeState* st, const unsigned long long* seg_sums,
                          const int* bucket_seg_end, const int* cuts, const AllScale* sc, double* values,
                          int* cover, double* prefix, cudaStream_t s);
void launch_pred_update(const PostParams& pp, const int16_t* nid, const double* prefix, const DevTreeState* st,
                        double* pred, cudaStream_t s);
void launch_fill_pred(const double* init_prefix, int n, int n_buckets, int iid_mode, double* pred,
                      cudaStream_t s);
void launch_predict_trees(const uint8_t* codes, int stride, int n, const int16_t* tree_feat,
                          const int16_t* tree_left, const int16_t* tree_right, const uint8_t* tree_thr,
                          const uint8_t* tree_ml, const double* tree_val, const int* tree_off, int n_trees,
                          double base, double lr, const uint8_t* tree_type, const unsigned long long* tree_cat,
                          const int16_t* tree_feat2, int n_bins, double* out, cudaStream_t s);

}  // namespace tgb
