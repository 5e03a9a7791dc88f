// device="gpu" Booster::fit (cpp/src/booster.cpp:231-742) for the hot-path subset.
//
// Host work (once per fit): (ts, entity) order check / stable sort (booster.cpp:264-309),
// TORB buckets and prefix cuts (booster.cpp:311-364), quantile edges (binner.cpp),
// initial predictions (booster.cpp:399-457), and per tree only the data-independent
// GOSS draw positions (sampling.h).  Everything that touches rows runs on the device
// and stays resident in HBM for the whole fit: bin transform, gradients, GOSS
// selection, histograms, split scans, partitions, the post-tree sweep, the prediction
// update and the loss.  The per-tree kernel sequence never waits on the host: every
// launch reads its node / row range from device memory, so the host only enqueues
// and the trees come back in one copy at the end.
#include "booster.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <mutex>
#include <numeric>
#include <thread>

#include <memory>

#include "goss_sampler.h"
#include "sampling.h"
#include "tgb_internal.h"
#include "wave.h"

namespace tgb {

std::atomic<long long> g_kernel_launches{0};

void check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw TideError(std::string("CUDA ") + what + ": " + cudaGetErrorString(e));
    const size_t L = std::strlen(what);
    if (L > 7 && std::strcmp(what + L - 7, " launch") == 0) g_kernel_launches.fetch_add(1);
}

void* device_alloc(size_t bytes, cudaStream_t s) {
    static std::mutex mu;
    static bool configured[64] = {};
    int dev = 0;
    check(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev >= 0 && dev < 64) {
        std::lock_guard<std::mutex> lock(mu);
        if (!configured[dev]) {
            cudaMemPool_t pool;
            check(cudaDeviceGetDefaultMemPool(&pool, dev), "default mem pool");
            uint64_t keep = ~0ull;  // never hand freed blocks back to the driver
            check(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep), "mem pool threshold");
            // A block freed on one stream is handed to another stream only once the free has
            // completed; the pool never makes one booster's stream wait for another's.
            int no = 0;
            check(cudaMemPoolSetAttribute(pool, cudaMemPoolReuseAllowInternalDependencies, &no), "mem pool reuse");
            configured[dev] = true;
        }
    }
    void* p = nullptr;
    check(cudaMallocAsync(&p, bytes, s), "cudaMallocAsync");
    return p;
}

cudaError_t device_free(void* p, cudaStream_t s) {
    if (!p) return cudaSuccess;
    return cudaFreeAsync(p, s);
}

void Config::validate() const {
    // The reference's own checks (cpp/include/tidegbm/config.hpp:78-97).
    if (n_estimators < 1) throw TideError("n_estimators must be >= 1");
    if (learning_rate <= 0 || learning_rate > 1.5) throw TideError("learning_rate out of range");
    if (max_bin < 8 || max_bin > 256) throw TideError("max_bin must be in [8, 256]");
    if (!iid_mode && (n_time_buckets == 1 || n_time_buckets < 0))
        throw TideError("n_time_buckets must be 0 (auto) or >= 2");
    if (!iid_mode && horizon < 0)
        throw TideError(
            "horizon is required in time mode (label length in timestamp units). "
            "Overlapping returns without horizon leak into TORB.");
    if (device != "cpu" && device != "gpu") throw TideError("device must be cpu or gpu");
    // What the GPU path implements; everything else is an error, never a CPU fallback.
    if (device != "gpu") throw TideError("this library implements device=\"gpu\" only");
    if (max_bin > 255) throw TideError("GPU path: max_bin must be <= 255 (bin codes are uint8)");
    if (max_leaves < 2 || max_leaves > 256) throw TideError("GPU path: max_leaves must be in [2, 256]");
    if (max_depth < 1) throw TideError("GPU path: max_depth must be >= 1");
    if (objective != 0 && objective != 5) throw TideError("GPU path: objective must be mse or pairwise");
    if (subsample < 1.0) throw TideError("GPU path: subsample < 1 is not supported");
    if (colsample < 1.0 || colsample_bynode < 1.0) throw TideError("GPU path: colsample < 1 is not supported");
    if (l1 != 0.0 || max_delta_step != 0.0) throw TideError("GPU path: l1 / max_delta_step are not supported");
    if (time_decay < 1.0) throw TideError("GPU path: time_decay < 1 is not supported");
    if (causal_bins || causal_structure || structure_frac < 1.0 || entity_subsample < 1.0)
        throw TideError("GPU path: causal_bins / causal_structure / structure_frac / entity_subsample unsupported");
    if (goss_top <= 0.0) throw TideError("GPU path: goss_top must be > 0");
    if (hist_bits != 0 && hist_bits != 8 && hist_bits != 16)
        throw TideError("hist_bits must be 0 (exact), 16 or 8 (quantised gradients)");
    if (wave_expand < 0) throw TideError("wave_expand must be >= 0 (0: every candidate within the budget)");
    if (hist_stage != 0 && hist_stage != 1) throw TideError("hist_stage must be 0 (direct loads) or 1 (TMA gathers)");
}

namespace {

double now() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// fn(begin, end, part) over `parts` contiguous ranges of [0, n), one thread each.
template <typename F>
void parallel_ranges(int n, int parts, F&& fn) {
    parts = std::max(1, std::min(parts, n / 65536 + 1));
    if (parts == 1) {
        fn(0, n, 0);
        return;
    }
    std::vector<std::thread> th;
    for (int k = 0; k < parts; ++k) {
        const int b = static_cast<int>(static_cast<long long>(n) * k / parts);
        const int e = static_cast<int>(static_cast<long long>(n) * (k + 1) / parts);
        th.emplace_back([&fn, b, e, k] { fn(b, e, k); });
    }
    for (auto& t : th) t.join();
}

float ceil_f32(double e) {
    float f = static_cast<float>(e);
    if (static_cast<double>(f) < e) f = std::nextafter(f, INFINITY);
    return f;
}

// cpp/src/booster.cpp:36-58
int auto_time_buckets(const std::vector<int64_t>& uniq, int64_t horizon, int uniq_cap) {
    int64_t step = 1;
    if (uniq.size() >= 2) {
        std::vector<int64_t> d;
        d.reserve(uniq.size() - 1);
        for (size_t i = 1; i < uniq.size(); ++i)
            if (uniq[i] - uniq[i - 1] > 0) d.push_back(uniq[i] - uniq[i - 1]);
        if (!d.empty()) {
            std::nth_element(d.begin(), d.begin() + d.size() / 2, d.end());
            step = std::max<int64_t>(d[d.size() / 2], 1);
        }
    }
    const int h_steps = static_cast<int>(std::max<int64_t>(horizon, 0) / step);
    const int want = h_steps >= 8 ? 64 : 32;
    return std::max(2, std::min(want, std::max(uniq_cap, 2)));
}

}  // namespace

// The booster's stream outlives its buffers: it is declared first, so it is destroyed
// last, after every buffer's stream-ordered free has been queued on it.
struct OwnedStream {
    cudaStream_t s = nullptr;
    ~OwnedStream() {
        if (s) {
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
        }
    }
};

struct DeviceState {
    OwnedStream owned;
    cudaStream_t stream = nullptr;
    DBuf<uint8_t> codes, codes_col;
    DBuf<double> y, pred, g, h;
    DBuf<long long> gq;  // per-tree packed fixed-point g (constant-hessian histograms)
    DBuf<short> gq8;     // per-tree packed int8 g (int8 precision mode)
    DBuf<int32_t> rows0, rows1;
    DBuf<long long> histG, histH;
    DBuf<int> histC;
    DBuf<DevNode> nodes, nodes_all;
    DBuf<DevSplit> splits;
    DBuf<DevTreeState> st, st_all;
    DBuf<int> tile_counts;
    DBuf<double> scan_gain;
    DBuf<int> scan_key, scan_ticket;
    DBuf<unsigned long long> keys_in, keys_out;  // 64-bit slots; the fast GOSS path uses them as 32-bit
    DBuf<int> goss_overflow;
    DBuf<int32_t> vals_in, vals_out, rest_pos;
    DBuf<unsigned char> cub_tmp;
    DBuf<uint8_t> goss_flag;
    DBuf<int16_t> nid;
    DBuf<unsigned long long> seg_sums;
    DBuf<int4> chunks;
    DBuf<int> bucket_seg_end, cuts;
    DBuf<AllScale> all_scale;
    DBuf<double> init_prefix, values_all, prefix_all, losses, loss_part;
    DBuf<int> cover_all, loss_valid;
    DBuf<int> run_start, run_len, order;
    // batched growth (wave.h)
    DBuf<unsigned char> gqw, hqw;  // per-row histogram payloads (mode dependent, <= 8 B a row)
    DBuf<DevNode> spec;
    DBuf<DevSplit> spec_split;
    DBuf<WaveCtl> ctl;
    DBuf<double> cand_gain;
    DBuf<int> cand_key, tickets;
    DBuf<WaveCtx> wctx;
    DBuf<uint8_t> is_cat;                 // categorical flags per feature (fit and predict)
    DBuf<unsigned long long> cand_cat;    // scan candidates' left masks
    DBuf<DevSplit> splits_pair, spec_split_pair, pair_cand;  // PAIR search (wave.h)
    DBuf<unsigned long long> energy;
    DBuf<int> pair_tickets;
    // predict
    DBuf<uint8_t> pcodes;
    DBuf<int16_t> t_feat, t_left, t_right, t_feat2;
    DBuf<uint8_t> t_type;
    DBuf<unsigned long long> t_cat;
    DBuf<uint8_t> t_thr, t_ml;
    DBuf<double> t_val, pout;
    DBuf<int> t_off;
    size_t trees_flat = 0;

    // Everything a fit allocates; predict's buffers (pcodes, t_*, pout) stay.
    void release_fit_buffers() {
        codes.release(); codes_col.release(); y.release(); pred.release(); g.release(); h.release();
        gq.release(); gq8.release(); rows0.release(); rows1.release(); histG.release(); histH.release();
        histC.release(); nodes.release(); nodes_all.release(); splits.release(); st.release(); st_all.release();
        tile_counts.release(); scan_gain.release(); scan_key.release(); scan_ticket.release();
        keys_in.release(); keys_out.release(); goss_overflow.release(); vals_in.release(); vals_out.release();
        rest_pos.release(); cub_tmp.release(); goss_flag.release(); nid.release(); seg_sums.release();
        chunks.release(); bucket_seg_end.release(); cuts.release(); all_scale.release(); init_prefix.release();
        values_all.release(); prefix_all.release(); losses.release(); loss_part.release(); cover_all.release();
        loss_valid.release(); run_start.release(); run_len.release(); order.release();
        gqw.release(); hqw.release(); spec.release(); spec_split.release(); ctl.release(); cand_gain.release();
        cand_key.release(); tickets.release(); wctx.release(); cand_cat.release(); splits_pair.release();
        spec_split_pair.release(); pair_cand.release(); energy.release(); pair_tickets.release();
    }

};

GpuBooster::GpuBooster(int dev) : device(dev) {
    check(cudaSetDevice(device), "cudaSetDevice");
    ds_ = new DeviceState();
    check(cudaStreamCreateWithFlags(&ds_->owned.s, cudaStreamNonBlocking), "cudaStreamCreate");
    ds_->stream = ds_->owned.s;
}

GpuBooster::~GpuBooster() {
    cudaSetDevice(device);
    delete ds_;
}

// ---------------------------------------------------------------------------------------
// One fit context: everything Booster::fit sets up before its tree loop (booster.cpp:
// 231-500), then the per-tree work around the tree growth (gradients, GOSS sample,
// post-tree sweep, booster.cpp:519-706).  The growth itself is either the one-split
// loop (grow_leafwise) or the batched waves over one or many contexts (grow_waves).
struct FitRun {
    GpuBooster& B;
    Config c;
    DeviceState& D;
    cudaStream_t s;
    bool exact_goss;
    int n = 0, n_f = 0, stride = 0, T = 0, max_nodes = 0, nbk = 1;
    int n_threads = 1;
    bool use_goss = false, const_h = true, any_cat = false;
    bool g_ready = false;  // the previous tree's sweep wrote this tree's mse gradient
    int n_top = 0, n_other = 0;
    double goss_scale = 1.0;
    std::unique_ptr<GossSampler> sampler;
    std::vector<int4> chunks;
    int n_segments = 0, n_runs = 0, max_tiles = 0, grid_rows = 0, mode = 0, n_slots = 0;
    const int* order_d = nullptr;
    GrowParams gp{};
    PostParams pp{};
    HistSlotPtrs hs{};
    ScanScratch scs{};
    GossWork gw{};
    int32_t* rows[2] = {nullptr, nullptr};
    double t0 = 0;
    long long launches0 = 0;
    FitStats st;
    // measurement hooks of the leaf-wise loop
    std::vector<cudaEvent_t> hist_ev;
    size_t hist_ev_used = 0;
    DBuf<unsigned long long> rows_counter;

    FitRun(GpuBooster& b, const Config& cfg, DeviceState& d, cudaStream_t stream, bool exact)
        : B(b), c(cfg), D(d), s(stream), exact_goss(exact) {}
    ~FitRun() {
        if (sampler) sampler->stop();
        for (auto& e : hist_ev) cudaEventDestroy(e);
    }

    void prepare(const void* X_in, int x_dtype, const double* y_in, int n_in, int n_f_in, const int64_t* ts_in,
                 const int64_t* ent_in);
    void tree_begin(int t);
    void hist_leafwise(int node, bool in_timed);
    void grow_leafwise(bool in_timed);
    void tree_end(int t);
    bool finish();  // reads the trees back; true when the 32-bit GOSS sort overflowed
    WaveCtx wave_ctx() const;
};

void FitRun::prepare(const void* X_in, int x_dtype, const double* y_in, int n_in, int n_f_in, const int64_t* ts_in,
                     const int64_t* ent_in) {
    t0 = now();
    launches0 = g_kernel_launches.load();
    n = n_in;
    n_f = n_f_in;
    check(cudaSetDevice(B.device), "cudaSetDevice");
    if (n >= 1000000) {  // booster.cpp:237-240
        c.halo = false;
        c.pair_splits = false;
    }
    c.validate();
    if (c.pair_splits && (c.grow == 0 || c.hist_bits != 0))
        throw TideError("GPU path: pair_splits needs grow = 1 and hist_bits = 0 (or pass pair_splits=False)");
    if (c.pair_splits && (c.pair_top_k > 6 || n_f_in > 1024))
        throw TideError("GPU path: pair_splits needs pair_top_k <= 6 and at most 1024 features");
    if (c.halo) throw TideError("GPU path: halo is not supported");
    if (n <= 0 || n_f <= 0) throw TideError("empty input");
    if (x_dtype != 0 && x_dtype != 1) throw TideError("x_dtype must be 0 (float32) or 1 (float64)");
    if (!c.iid_mode && !ts_in) throw TideError("timestamp is required unless iid_mode");
    if (c.objective == 5 && !ts_in) throw TideError("rank objective requires timestamps");
    if (c.grow == 0 && c.hist_bits == 16) throw TideError("hist_bits = 16 needs grow = 1 (batched waves)");
    if (c.grow == 0 && c.hist_bits == 8 && c.objective != 0)
        throw TideError("hist_bits = 8 with the one-split loop needs a constant hessian (objective mse)");
    const size_t xsz = x_dtype == 0 ? 4 : 8;
    n_threads = c.n_jobs > 0 ? c.n_jobs : std::max(1u, std::thread::hardware_concurrency());
    const_h = c.objective == 0;
    if (!B.is_cat.empty() && static_cast<int>(B.is_cat.size()) != n_f)
        throw TideError("categorical flags: one per feature");
    if (B.is_cat.empty()) B.is_cat.assign(n_f, 0);
    any_cat = std::any_of(B.is_cat.begin(), B.is_cat.end(), [](int v) { return v != 0; });
    if (any_cat && c.grow == 0) throw TideError("categorical features need grow = 1 (batched waves)");
    mode = hist_mode(c.hist_bits, const_h);

    // ---- (ts, entity) order: booster.cpp:264-309 ----
    const void* X = X_in;
    const double* y = y_in;
    const int64_t* ts = ts_in;
    std::vector<unsigned char> X_own;
    std::vector<double> y_own;
    std::vector<int64_t> ts_own;
    if (!c.iid_mode && n > 1) {
        std::atomic<bool> unsorted{false};
        parallel_ranges(n, n_threads, [&](int b, int e, int) {
            for (int i = std::max(1, b); i < e && !unsorted.load(std::memory_order_relaxed); ++i) {
                if (ts_in[i] < ts_in[i - 1] || (ts_in[i] == ts_in[i - 1] && ent_in && ent_in[i] < ent_in[i - 1])) {
                    unsorted = true;
                    break;
                }
            }
        });
        if (unsorted.load()) {
            std::vector<int> ord(n);
            std::iota(ord.begin(), ord.end(), 0);
            std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) {
                if (ts_in[a] != ts_in[b]) return ts_in[a] < ts_in[b];
                if (ent_in) return ent_in[a] < ent_in[b];
                return a < b;
            });
            X_own.resize(static_cast<size_t>(n) * n_f * xsz);
            y_own.resize(n);
            ts_own.resize(n);
            for (int i = 0; i < n; ++i) {
                std::memcpy(X_own.data() + static_cast<size_t>(i) * n_f * xsz,
                            static_cast<const unsigned char*>(X_in) + static_cast<size_t>(ord[i]) * n_f * xsz,
                            n_f * xsz);
                y_own[i] = y_in[ord[i]];
                ts_own[i] = ts_in[ord[i]];
            }
            X = X_own.data();
            y = y_own.data();
            ts = ts_own.data();
        }
    }
    st.t_sort = now() - t0;
    const double t_pre0 = now();

    // GOSS: booster.cpp:554-585 (sample = all rows since subsample = 1).  The draw
    // positions depend only on n and the config, so the sampler's producer starts now and
    // walks the generator while the data are uploaded and binned.
    T = c.n_estimators;
    use_goss = ((c.goss > 0) || (c.goss < 0 && n >= 250000)) && c.goss_top < 1.0 && n > 64;
    goss_scale = (1.0 - c.goss_top) / std::max(c.goss_other, 1e-12);
    if (use_goss) {
        n_top = std::min(n, std::max(1, static_cast<int>(std::ceil(c.goss_top * static_cast<double>(n)))));
        const int64_t m_rest = n - n_top;
        n_other = std::min(static_cast<int>(std::ceil(c.goss_other * static_cast<double>(n))), static_cast<int>(m_rest));
        // The booster's generator (booster.cpp:483) is only used by GOSS and grow_tree's
        // seed draw, so the sampler owns the whole stream.
        sampler = std::make_unique<GossSampler>(static_cast<uint32_t>(c.random_state), m_rest, n_other, T, 8,
                                                std::max(1, std::min(8, n_threads - 2)));
    }

    // ---- TORB buckets + prefix cuts: booster.cpp:311-364 ----
    int64_t embargo = c.embargo;
    std::vector<int> cut(1, 0);
    if (!c.iid_mode) {
        // distinct timestamps in row order (rows are time-sorted), per range then joined
        std::vector<std::vector<int64_t>> parts(std::max(1, n_threads));
        parallel_ranges(n, n_threads, [&](int b, int e, int k) {
            for (int i = b; i < e; ++i)
                if (i == 0 || ts[i] != ts[i - 1]) parts[k].push_back(ts[i]);
        });
        std::vector<int64_t> uniq;
        uniq.reserve(1024);
        for (auto& v : parts) uniq.insert(uniq.end(), v.begin(), v.end());
        const int uniq_n = std::max(2, static_cast<int>(uniq.size()));
        int want = c.n_time_buckets;
        if (want <= 0) want = auto_time_buckets(uniq, std::max<int64_t>(c.horizon, 0), uniq_n);
        nbk = c.finer_torb ? std::max(2, std::min(want, uniq_n)) : std::max(2, want);
        embargo += std::max<int64_t>(c.horizon, 0);
        cut.assign(nbk, 0);
        // first row of each time bucket (time_buckets, booster.cpp:60-72): the bucket of row
        // i is non-decreasing in i, so each first row is a binary search on the same expression
        auto bucket_of = [&](int i) {
            const int b = static_cast<int>(static_cast<double>(i) / std::max(n, 1) * nbk);
            return b >= nbk ? nbk - 1 : b;
        };
        std::vector<int> first(nbk, -1);
        for (int b = 0; b < nbk; ++b) {
            int lo = 0, hi = n;  // smallest i with bucket_of(i) >= b
            while (lo < hi) {
                const int mid = lo + (hi - lo) / 2;
                if (bucket_of(mid) >= b) hi = mid;
                else lo = mid + 1;
            }
            if (lo < n && bucket_of(lo) == b) first[b] = lo;
        }
        int run = 0;
        for (int b = 0; b < nbk; ++b) {
            int ct = 0;
            if (first[b] >= 0) ct = static_cast<int>(std::lower_bound(ts, ts + n, ts[first[b]] - embargo) - ts);
            run = std::max(run, ct);
            cut[b] = run;
        }
    }
    B.n_buckets = nbk;

    // ---- initial predictions: booster.cpp:399-457 ----
    // A sequential FP64 pass over y in row order (the reference's summation order); it
    // runs on the host while the X upload is in flight (below).
    std::vector<double> fill_prefix;
    auto initial_predictions = [&] {
        B.init_prefix.assign(nbk, 0.0);
        if (c.objective == 5) {
            B.init_score = 0.0;
        } else {
            // One running FP64 sum in row order: the same partial sums the reference
            // forms separately for every prefix [0, cut_b) and for [0, n).
            double sw = 0, sy = 0;
            int i = 0;
            std::vector<double> at_cut(nbk, 0.0);
            for (int b = 0; b < nbk && !c.iid_mode; ++b) {
                for (; i < cut[b]; ++i) {
                    sw += 1.0;
                    sy += 1.0 * y[i];
                }
                at_cut[b] = cut[b] > 0 ? (sw > 0 ? sy / sw : 0) : NAN;
            }
            for (; i < n; ++i) {
                sw += 1.0;
                sy += 1.0 * y[i];
            }
            B.init_score = sw > 0 ? sy / sw : 0;
            if (!c.iid_mode) B.init_prefix = at_cut;
        }
        // Device fill values: the prior of each bucket, or init_score for every row in iid
        // mode (where the reference leaves init_prefix = {0.0}, booster.cpp:400).
        if (c.iid_mode) {
            B.init_prefix.assign(1, 0.0);
            fill_prefix.assign(1, B.init_score);
        } else {
            for (int b = 0; b < nbk; ++b)
                if (!std::isfinite(B.init_prefix[b])) B.init_prefix[b] = B.init_score;
            fill_prefix = B.init_prefix;
        }
    };

    st.t_pre_upload = now() - t_pre0;  // GOSS sampler start, TORB buckets and cuts
    // ---- device buffers ----
    double tb = now();
    stride = (n_f + 15) / 16 * 16;
    max_nodes = 2 * c.max_leaves - 1;
    const size_t slot = static_cast<size_t>(n_f) * kBins;
    const bool wave = c.grow != 0;
    n_slots = wave ? 1 + 2 * max_nodes : max_nodes;
    D.codes.alloc(static_cast<size_t>(n) * stride, s);
    D.codes_col.alloc(static_cast<size_t>(n_f) * codes_col_pitch(n), s);
    D.y.alloc(n, s);
    D.pred.alloc(n, s);
    D.g.alloc(n, s);
    if (!const_h) D.h.alloc(n, s);  // MSE hessians are implicit (unit)
    if (wave) {
        // payloads by position in either rows buffer (2 x n elements)
        D.gqw.alloc(static_cast<size_t>(2) * n * hist_pay_bytes(mode), s);
        if (mode == kHistExactVar) D.hqw.alloc(static_cast<size_t>(2) * n * 8, s);
    } else {
        if (const_h && c.hist_bits == 0) D.gq.alloc(n, s);
        if (c.hist_bits == 8) D.gq8.alloc(n, s);
    }
    D.rows0.alloc(n, s);
    D.rows1.alloc(n, s);
    D.histG.alloc(slot * n_slots, s);
    D.histH.alloc(slot * n_slots, s);
    D.histC.alloc(slot * n_slots, s);
    D.nodes.alloc(kMaxNodes, s);
    D.splits.alloc(kMaxNodes, s);
    D.st.alloc(1, s);
    max_tiles = (n + kPartTile - 1) / kPartTile + kMaxLeavesCap + 1;
    D.tile_counts.alloc(max_tiles + 1, s);
    if (wave) {
        D.spec.alloc(2 * kMaxNodes, s);
        D.spec_split.alloc(2 * kMaxNodes, s);
        D.ctl.alloc(1, s);
        D.cand_gain.alloc(static_cast<size_t>(2 * kMaxNodes + 1) * n_f, s);
        D.cand_key.alloc(static_cast<size_t>(2 * kMaxNodes + 1) * n_f, s);
        D.tickets.alloc(2 * kMaxNodes + 1, s);
        if (any_cat) D.cand_cat.alloc(static_cast<size_t>(2 * kMaxNodes + 1) * n_f * 4, s);
        if (c.pair_splits) {
            D.splits_pair.alloc(kMaxNodes, s);
            D.spec_split_pair.alloc(2 * kMaxNodes, s);
            D.energy.alloc(2 * kMaxNodes + 1, s);
            D.pair_cand.alloc(static_cast<size_t>(2 * kMaxNodes + 1) * kMaxPairs, s);
            D.pair_tickets.alloc(2 * kMaxNodes + 1, s);
            check(cudaMemsetAsync(D.pair_tickets.p, 0, sizeof(int) * (2 * kMaxNodes + 1), s), "pair ticket reset");
        }
        check(cudaMemsetAsync(D.tickets.p, 0, sizeof(int) * (2 * kMaxNodes + 1), s), "ticket reset");
        check(cudaMemsetAsync(D.ctl.p, 0, sizeof(WaveCtl), s), "wave control reset");
    } else {
        D.scan_gain.alloc(2 * scan_ctas_per_node(n_f), s);
        D.scan_key.alloc(2 * scan_ctas_per_node(n_f), s);
        D.scan_ticket.alloc(3, s);
        check(cudaMemsetAsync(D.scan_ticket.p, 0, 3 * sizeof(int), s), "ticket reset");
    }
    D.nid.alloc(n, s);
    D.all_scale.alloc(1, s);
    D.init_prefix.alloc(nbk, s);
    D.nodes_all.alloc(static_cast<size_t>(T) * max_nodes, s);
    D.st_all.alloc(T, s);
    D.values_all.alloc(static_cast<size_t>(T) * max_nodes, s);
    D.cover_all.alloc(static_cast<size_t>(T) * max_nodes, s);
    D.prefix_all.alloc(static_cast<size_t>(T) * nbk * max_nodes, s);
    D.losses.alloc(T, s);

    // X upload + transform, then X is released.
    {
        st.t_alloc = now() - tb;
        DBuf<unsigned char> Xd;
        Xd.alloc(static_cast<size_t>(n) * n_f * xsz, s);
        check(cudaMemcpyAsync(Xd.p, X, static_cast<size_t>(n) * n_f * xsz, cudaMemcpyHostToDevice, s), "X upload");
        check(cudaMemcpyAsync(D.y.p, y, sizeof(double) * n, cudaMemcpyHostToDevice, s), "y upload");
        initial_predictions();  // host work while the copies run (they only read X and y)
        check(cudaStreamSynchronize(s), "X upload");
        st.t_h2d = now() - tb - st.t_alloc;
        // ---- quantile edges: Binner::fit (binning.cpp:34-102) on the uploaded X ----
        const double tbf = now();
        BinFitTimes bt;
        if (any_cat) {
            // vocabularies of the categorical features (binning.cpp:47-84) on the host, the
            // numeric features' edges with them (the host binner, bit-identical)
            B.n_bins = binner_fit_cat(X, x_dtype, n, n_f, B.is_cat.data(), c.max_bin, c.cat_min_count, c.bin_sample,
                                      static_cast<uint32_t>(c.random_state), B.edges, B.n_edges, n_threads);
        } else if (binner_fits_device(n, n_f, c.bin_sample))
            B.n_bins = binner_fit_device(Xd.p, x_dtype, n, n_f, c.max_bin, c.bin_sample,
                                         static_cast<uint32_t>(c.random_state), B.edges, B.n_edges, n_threads, s,
                                         D.codes_col.p, D.codes_col.n, &bt, X);  // scratch: codes_col, filled later
        else
            B.n_bins = binner_fit(X, x_dtype, n, n_f, c.max_bin, c.bin_sample, static_cast<uint32_t>(c.random_state),
                                  B.edges, B.n_edges, n_threads);
        B.n_features = n_f;
        st.t_binfit = now() - tbf;
        st.t_bin_counts = bt.counts;
        st.t_bin_draws = bt.draws;
        st.t_bin_edges = bt.edges;
        DBuf<int> ne;
        ne.alloc(n_f, s);
        check(cudaMemcpyAsync(ne.p, B.n_edges.data(), sizeof(int) * n_f, cudaMemcpyHostToDevice, s), "edges upload");
        if (any_cat) {
            // on the booster's own stream: the flags stay with the model for its predicts
            std::vector<uint8_t> ic(n_f);
            for (int f = 0; f < n_f; ++f) ic[f] = B.is_cat[f] ? 1 : 0;
            D.is_cat.alloc(n_f, D.stream);
            check(cudaMemcpyAsync(D.is_cat.p, ic.data(), n_f, cudaMemcpyHostToDevice, D.stream), "categorical flags");
            check(cudaStreamSynchronize(D.stream), "categorical flags");
        } else {
            D.is_cat.release();
        }
        if (x_dtype == 0) {
            std::vector<float> ef(static_cast<size_t>(n_f) * 256, INFINITY);
            for (int f = 0; f < n_f; ++f)
                for (int k = 0; k < B.n_edges[f]; ++k)
                    ef[static_cast<size_t>(f) * 256 + k] = ceil_f32(B.edges[static_cast<size_t>(f) * 256 + k]);
            DBuf<float> ed;
            ed.alloc(ef.size(), s);
            check(cudaMemcpyAsync(ed.p, ef.data(), sizeof(float) * ef.size(), cudaMemcpyHostToDevice, s), "edges upload");
            launch_bin_transform_f32(reinterpret_cast<const float*>(Xd.p), n, n_f, ed.p, ne.p, D.codes.p, stride, s,
                                     D.is_cat.p);
            check(cudaStreamSynchronize(s), "transform");
        } else {
            std::vector<double> ed_h(static_cast<size_t>(n_f) * 256, INFINITY);
            for (int f = 0; f < n_f; ++f)
                for (int k = 0; k < B.n_edges[f]; ++k)
                    ed_h[static_cast<size_t>(f) * 256 + k] = B.edges[static_cast<size_t>(f) * 256 + k];
            DBuf<double> ed;
            ed.alloc(ed_h.size(), s);
            check(cudaMemcpyAsync(ed.p, ed_h.data(), sizeof(double) * ed_h.size(), cudaMemcpyHostToDevice, s),
                  "edges upload");
            launch_bin_transform_f64(reinterpret_cast<const double*>(Xd.p), n, n_f, ed.p, ne.p, D.codes.p, stride, s,
                                     D.is_cat.p);
            check(cudaStreamSynchronize(s), "transform");
        }
    }
    // Column-major copy for the partition's reads of one feature over a row list.
    const double ttr = now();
    launch_codes_transpose(D.codes.p, stride, n, n_f, D.codes_col.p, s);
    check(cudaStreamSynchronize(s), "transpose");
    st.t_transpose = now() - ttr;
    st.t_upload = now() - tb - st.t_binfit;
    const double t_prep0 = now();

    // TORB segments: distinct cuts split the time-sorted rows into segments; CTAs of the
    // post-tree sweep own segment-aligned chunks.
    std::vector<int> bounds;
    for (int b = 0; b < nbk && !c.iid_mode; ++b)
        if (cut[b] > 0 && (bounds.empty() || bounds.back() != cut[b])) bounds.push_back(cut[b]);
    if (bounds.empty() || bounds.back() != n) bounds.push_back(n);
    std::vector<int> seg_end(nbk, 0);
    for (int b = 0; b < nbk && !c.iid_mode; ++b)
        seg_end[b] = cut[b] > 0 ? static_cast<int>(std::lower_bound(bounds.begin(), bounds.end(), cut[b]) - bounds.begin()) + 1 : 0;
    const int kChunk = 8192;
    chunks.clear();
    for (int k = 0, lo = 0; k < static_cast<int>(bounds.size()); lo = bounds[k], ++k)
        for (int a = lo; a < bounds[k]; a += kChunk) chunks.push_back(make_int4(k, a, std::min(bounds[k], a + kChunk), 0));
    n_segments = static_cast<int>(bounds.size());
    D.seg_sums.alloc(static_cast<size_t>(n_segments) * kMaxNodes * 3, s);
    D.chunks.alloc(chunks.size(), s);
    D.bucket_seg_end.alloc(nbk, s);
    D.cuts.alloc(nbk, s);
    check(cudaMemcpyAsync(D.chunks.p, chunks.data(), sizeof(int4) * chunks.size(), cudaMemcpyHostToDevice, s), "chunks");
    check(cudaMemcpyAsync(D.bucket_seg_end.p, seg_end.data(), sizeof(int) * nbk, cudaMemcpyHostToDevice, s), "segs");
    std::vector<int> cuts_h = c.iid_mode ? std::vector<int>(1, 0) : cut;
    check(cudaMemcpyAsync(D.cuts.p, cuts_h.data(), sizeof(int) * nbk, cudaMemcpyHostToDevice, s), "cuts");
    check(cudaMemcpyAsync(D.init_prefix.p, fill_prefix.data(), sizeof(double) * nbk, cudaMemcpyHostToDevice, s),
          "init prefix");
    launch_fill_pred(D.init_prefix.p, n, nbk, c.iid_mode ? 1 : 0, D.pred.p, s);

    // Rank groups (objective.cpp:18-39): runs of equal timestamps; rows are time-sorted
    // in time mode, otherwise a stable order by timestamp is uploaded.
    if (c.objective == 5) {
        std::vector<int> ord;
        const int64_t* grp = ts;
        bool sorted = true;
        for (int i = 1; i < n; ++i)
            if (grp[i] < grp[i - 1]) {
                sorted = false;
                break;
            }
        if (!sorted) {
            ord.resize(n);
            std::iota(ord.begin(), ord.end(), 0);
            std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return grp[a] < grp[b]; });
        }
        auto gat = [&](int p) { return sorted ? grp[p] : grp[ord[p]]; };
        std::vector<int> rs, rl;
        for (int i = 0; i < n;) {
            int j = i + 1;
            while (j < n && gat(j) == gat(i)) ++j;
            rs.push_back(i);
            rl.push_back(j - i);
            i = j;
        }
        n_runs = static_cast<int>(rs.size());
        D.run_start.alloc(n_runs, s);
        D.run_len.alloc(n_runs, s);
        D.loss_part.alloc(n_runs, s);
        D.loss_valid.alloc(n_runs, s);
        check(cudaMemcpyAsync(D.run_start.p, rs.data(), sizeof(int) * n_runs, cudaMemcpyHostToDevice, s), "runs");
        check(cudaMemcpyAsync(D.run_len.p, rl.data(), sizeof(int) * n_runs, cudaMemcpyHostToDevice, s), "runs");
        if (!sorted) {
            D.order.alloc(n, s);
            check(cudaMemcpyAsync(D.order.p, ord.data(), sizeof(int) * n, cudaMemcpyHostToDevice, s), "order");
            order_d = D.order.p;
        }
        check(cudaStreamSynchronize(s), "runs upload");
    } else {
        D.loss_part.alloc(2368, s);
    }

    // GOSS device buffers (the sample itself is set up with the sampler, above).
    if (use_goss) {
        D.keys_in.alloc(n, s);
        D.keys_out.alloc(n, s);
        D.vals_in.alloc(n, s);
        D.vals_out.alloc(n, s);
        D.goss_flag.alloc(n, s);
        D.rest_pos.alloc(std::max(1, n_other), s);
        const size_t cb = goss_cub_bytes(n, exact_goss);
        D.cub_tmp.alloc(cb, s);
        D.goss_overflow.alloc(1, s);
        check(cudaMemsetAsync(D.goss_overflow.p, 0, sizeof(int), s), "overflow reset");
        launch_goss_iota(D.vals_in.p, n, s);
        sampler->start_workers();
    }
    gw = GossWork{D.keys_in.p, D.keys_out.p, D.vals_in.p, D.vals_out.p, D.cub_tmp.p, D.cub_tmp.n,
                  D.goss_overflow.p, exact_goss};
    gp = GrowParams{n_f, stride, B.n_bins, c.max_depth, c.max_leaves, c.min_samples_leaf, c.min_child_weight, c.l2,
                    c.min_split_gain};
    pp = PostParams{n, nbk, c.iid_mode ? 1 : 0, n_segments, c.learning_rate, c.l2,
                    c.torb_min_cover > 0.0 ? c.torb_min_cover : static_cast<double>(2 * std::max(c.min_samples_leaf, 1))};
    hs = HistSlotPtrs{D.histG.p, D.histH.p, D.histC.p, slot};
    scs = ScanScratch{D.scan_gain.p, D.scan_key.p, D.scan_ticket.p};
    rows[0] = D.rows0.p;
    rows[1] = D.rows1.p;
    if (!wave) grid_rows = hist_grid_rows(n_f, n, const_h);
    if (wave) {
        const WaveCtx wc = wave_ctx();
        D.wctx.alloc(1, s);
        check(cudaMemcpyAsync(D.wctx.p, &wc, sizeof(WaveCtx), cudaMemcpyHostToDevice, s), "wave context upload");
        check(cudaStreamSynchronize(s), "wave context upload");
    }
    st.t_prep = now() - t_prep0;  // TORB segments, rank groups, GOSS buffers, initial predictions
}

WaveCtx FitRun::wave_ctx() const {
    WaveCtx w{};
    w.codes = D.codes.p;
    w.codes_col = D.codes_col.p;
    w.col_pitch = codes_col_pitch(n);
    w.rows0 = D.rows0.p;
    w.rows1 = D.rows1.p;
    w.gq = D.gqw.p;
    w.hq = D.hqw.p;
    w.pay_pitch = n;
    w.pay_bytes = hist_pay_bytes(mode);
    w.nodes = D.nodes.p;
    w.splits = D.splits.p;
    w.st = D.st.p;
    w.spec = D.spec.p;
    w.spec_split = D.spec_split.p;
    w.ctl = D.ctl.p;
    w.G = D.histG.p;
    w.H = D.histH.p;
    w.C = D.histC.p;
    w.cand_gain = D.cand_gain.p;
    w.cand_key = D.cand_key.p;
    w.tickets = D.tickets.p;
    w.tile_counts = D.tile_counts.p;
    w.gp = gp;
    w.goss_scale = use_goss ? goss_scale : 1.0;
    w.n_slots = n_slots;
    w.max_tiles = max_tiles;
    w.max_expand = c.wave_expand;
    w.codes_map_ok = c.hist_stage != 0 && encode_codes_map(&w.codes_map, D.codes.p, n, stride) ? 1 : 0;
    w.is_cat = D.is_cat.p;
    w.cand_cat = D.cand_cat.p;
    w.cat_smooth = c.cat_smooth;
    w.pair_on = c.pair_splits ? 1 : 0;
    w.pair_top_k = c.pair_top_k;
    w.max_pair = c.max_pair_splits_per_tree;
    w.pair_trigger = c.pair_trigger;
    w.pair_l2 = c.pair_l2;
    w.g = D.g.p;
    w.goss_flag = use_goss ? D.goss_flag.p : nullptr;
    w.splits_pair = D.splits_pair.p;
    w.spec_split_pair = D.spec_split_pair.p;
    w.energy = D.energy.p;
    w.pair_cand = D.pair_cand.p;
    w.pair_tickets = D.pair_tickets.p;
    return w;
}

// Gradients (booster.cpp:701), the GOSS sample (booster.cpp:554-585), the tree's root and
// histogram scales, and the per-row histogram payload.
void FitRun::tree_begin(int t) {
    const bool wave = c.grow != 0;
    if (const_h) {
        if (!g_ready) launch_grad_mse_fused(D.y.p, D.pred.p, n, D.g.p, D.all_scale.p, s);
        g_ready = false;
        launch_all_scale_finalize(D.all_scale.p, n, s);
    } else {
        launch_grad_pairwise(D.y.p, D.pred.p, D.run_start.p, D.run_len.p, order_d, n_runs, n, D.g.p, D.h.p, s);
        launch_all_scale(D.g.p, D.h.p, n, D.all_scale.p, s);
    }
    const double* h_rows = const_h ? nullptr : D.h.p;
    if (use_goss) {
        const double tr = now();
        const int32_t* pos = sampler->wait(t);  // host time spent waiting for the draw
        st.t_rng += now() - tr;
        check(cudaMemcpyAsync(D.rest_pos.p, pos, sizeof(int32_t) * std::max(1, n_other), cudaMemcpyHostToDevice, s),
              "positions upload");
        sampler->release(t, s);
        launch_goss_select(D.g.p, h_rows, n, n_top, n_other, D.rest_pos.p, sampler->min_pos(t), gw, D.all_scale.p,
                           goss_scale, D.goss_flag.p, D.rows0.p, D.tile_counts.p, D.st.p, s);
        if (wave) {
            launch_wave_tree_init(D.nodes.p, D.splits.p, D.st.p, D.ctl.p, 0, 1, s);
            launch_wave_scales(D.st.p, nullptr, mode, s);
        } else {
            launch_tree_init(D.nodes.p, D.splits.p, D.st.p, 0, 1, s);
            launch_scales(D.st.p, nullptr, c.hist_bits == 8, s);
        }
    } else {
        launch_iota_rows(D.rows0.p, n, s);
        if (wave) {
            launch_wave_tree_init(D.nodes.p, D.splits.p, D.st.p, D.ctl.p, n, 0, s);
            launch_wave_scales(D.st.p, D.all_scale.p, mode, s);
        } else {
            launch_tree_init(D.nodes.p, D.splits.p, D.st.p, n, 0, s);
            launch_scales(D.st.p, D.all_scale.p, c.hist_bits == 8, s);
        }
    }
    const uint8_t* flag = use_goss ? D.goss_flag.p : nullptr;
    // per-tree stream of the stochastic rounding (SplitMix64 of seed and tree)
    uint64_t z = (static_cast<uint64_t>(static_cast<uint32_t>(c.random_state)) << 32) + static_cast<uint64_t>(t);
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    const uint64_t seed = z ^ (z >> 31);
    const size_t slot = static_cast<size_t>(n_f) * kBins;
    if (wave) {
        launch_wave_quantize(mode, D.rows0.p, D.g.p, h_rows, flag, goss_scale, D.st.p, seed, D.gqw.p, D.hqw.p, n, s);
        if (c.pair_splits)
            check(cudaMemsetAsync(D.energy.p + 2 * kMaxNodes, 0, sizeof(unsigned long long), s), "energy reset");
        // the root's slot; the children's slots are cleared by the partition of their wave
        check(cudaMemsetAsync(D.histG.p, 0, sizeof(long long) * slot, s), "hist reset");
        check(cudaMemsetAsync(D.histH.p, 0, sizeof(long long) * slot, s), "hist reset");
        check(cudaMemsetAsync(D.histC.p, 0, sizeof(int) * slot, s), "hist reset");
    } else {
        if (c.hist_bits == 8)
            launch_quantize8(D.rows0.p, D.g.p, flag, goss_scale, D.st.p, seed, D.gq8.p, n, s);
        else if (const_h)
            launch_quantize(D.rows0.p, D.g.p, flag, goss_scale, D.st.p, D.gq.p, n, s);
        check(cudaMemsetAsync(D.histG.p, 0, sizeof(long long) * slot * max_nodes, s), "hist reset");
        check(cudaMemsetAsync(D.histH.p, 0, sizeof(long long) * slot * max_nodes, s), "hist reset");
        check(cudaMemsetAsync(D.histC.p, 0, sizeof(int) * slot * max_nodes, s), "hist reset");
    }
}

void FitRun::hist_leafwise(int node, bool in_timed) {
    const bool prof = in_timed && c.profile_hist && hist_ev_used + 2 <= hist_ev.size();
    if (prof) check(cudaEventRecord(hist_ev[hist_ev_used], s), "event record");
    const void* gq = c.hist_bits == 8 ? static_cast<const void*>(D.gq8.p) : static_cast<const void*>(D.gq.p);
    launch_hist_node(D.codes.p, stride, n_f, rows, D.nodes.p, D.st.p, node, D.g.p, D.h.p, gq, c.hist_bits == 8,
                     use_goss ? D.goss_flag.p : nullptr, goss_scale, hs, grid_rows,
                     in_timed ? rows_counter.p : nullptr, const_h, s);
    if (prof) {
        check(cudaEventRecord(hist_ev[hist_ev_used + 1], s), "event record");
        hist_ev_used += 2;
    }
}

// grow_tree (cpp/src/tree.cpp:283-472), one split per iteration: every scan launch ends
// with the choice of the next leaf to split, except the last.
void FitRun::grow_leafwise(bool in_timed) {
    hist_leafwise(0, in_timed);
    launch_split_scan(gp, hs, D.nodes.p, D.splits.p, D.st.p, 0, 0, scs, c.max_leaves > 1, s);
    for (int it = 0; it < c.max_leaves - 1; ++it) {
        launch_partition(D.codes.p, stride, D.codes_col.p, codes_col_pitch(n), rows, D.nodes.p, D.st.p,
                         D.tile_counts.p, max_tiles, s);
        hist_leafwise(-1, in_timed);
        launch_split_scan(gp, hs, D.nodes.p, D.splits.p, D.st.p, 1, 0, scs, it < c.max_leaves - 2, s);
    }
}

// Post-tree sweep (booster.cpp:589-664), outputs straight into tree slot t, then the
// prediction update and the training loss (booster.cpp:704-706).
void FitRun::tree_end(int t) {
    const double* h_rows = const_h ? nullptr : D.h.p;
    double* values_t = D.values_all.p + static_cast<size_t>(t) * max_nodes;
    double* prefix_t = D.prefix_all.p + static_cast<size_t>(t) * nbk * max_nodes;
    int* cover_t = D.cover_all.p + static_cast<size_t>(t) * max_nodes;
    launch_apply_accum(D.codes_col.p, codes_col_pitch(n), n_f, D.nodes.p, D.st.p, D.g.p, h_rows, D.chunks.p,
                       static_cast<int>(chunks.size()), D.all_scale.p, D.nid.p, D.seg_sums.p, n_segments, B.n_bins,
                       (any_cat ? 1 : 0) | (c.pair_splits ? 2 : 0), s);
    launch_finalize_tree(pp, D.st.p, D.seg_sums.p, D.bucket_seg_end.p, D.cuts.p, D.all_scale.p, values_t, cover_t,
                         prefix_t, s);
    if (const_h) {
        // the next tree's gradient from the same pass (not after the last tree)
        g_ready = t + 1 < T;
        launch_pred_update_loss(pp, D.nid.p, prefix_t, D.st.p, D.pred.p, D.y.p, D.loss_part.p, 2368,
                                g_ready ? D.g.p : nullptr, g_ready ? D.all_scale.p : nullptr, s);
        launch_loss_finalize(0, D.loss_part.p, nullptr, 2368, n, D.losses.p + t, s);
    } else {
        launch_pred_update(pp, D.nid.p, prefix_t, D.st.p, D.pred.p, s);
        launch_loss_pairwise(D.y.p, D.pred.p, D.run_start.p, D.run_len.p, order_d, n_runs, D.loss_part.p,
                             D.loss_valid.p, s);
        launch_loss_finalize(5, D.loss_part.p, D.loss_valid.p, n_runs, n, D.losses.p + t, s);
    }
    check(cudaMemcpyAsync(D.nodes_all.p + static_cast<size_t>(t) * max_nodes, D.nodes.p, sizeof(DevNode) * max_nodes,
                          cudaMemcpyDeviceToDevice, s),
          "nodes snapshot");
    check(cudaMemcpyAsync(D.st_all.p + t, D.st.p, sizeof(DevTreeState), cudaMemcpyDeviceToDevice, s),
          "state snapshot");
}

bool FitRun::finish() {
    const double tf = now();
    check(cudaStreamSynchronize(s), "tree loop");
    if (sampler) {
        sampler->stop();
        st.t_producer = sampler->producer_seconds();
        sampler.reset();
    }
    st.t_finish_sync = now() - tf;
    const double td = now();
    std::vector<DevNode> nodes_h(static_cast<size_t>(T) * max_nodes);
    std::vector<DevTreeState> st_h(T);
    std::vector<double> vals_h(static_cast<size_t>(T) * max_nodes), pre_h(static_cast<size_t>(T) * nbk * max_nodes);
    std::vector<int> cov_h(static_cast<size_t>(T) * max_nodes);
    B.evals_train.assign(T, 0.0);
    check(cudaMemcpyAsync(nodes_h.data(), D.nodes_all.p, sizeof(DevNode) * nodes_h.size(), cudaMemcpyDeviceToHost, s), "D2H");
    check(cudaMemcpyAsync(st_h.data(), D.st_all.p, sizeof(DevTreeState) * T, cudaMemcpyDeviceToHost, s), "D2H");
    check(cudaMemcpyAsync(vals_h.data(), D.values_all.p, sizeof(double) * vals_h.size(), cudaMemcpyDeviceToHost, s), "D2H");
    check(cudaMemcpyAsync(pre_h.data(), D.prefix_all.p, sizeof(double) * pre_h.size(), cudaMemcpyDeviceToHost, s), "D2H");
    check(cudaMemcpyAsync(cov_h.data(), D.cover_all.p, sizeof(int) * cov_h.size(), cudaMemcpyDeviceToHost, s), "D2H");
    check(cudaMemcpyAsync(B.evals_train.data(), D.losses.p, sizeof(double) * T, cudaMemcpyDeviceToHost, s), "D2H");
    int overflow = 0, wave_error = 0;
    if (use_goss && !exact_goss)
        check(cudaMemcpyAsync(&overflow, D.goss_overflow.p, sizeof(int), cudaMemcpyDeviceToHost, s), "overflow flag");
    if (c.grow != 0)
        check(cudaMemcpyAsync(&wave_error, &D.ctl.p->error, sizeof(int), cudaMemcpyDeviceToHost, s), "wave error flag");
    int exp_total = 0;
    if (c.grow != 0)
        check(cudaMemcpyAsync(&exp_total, &D.ctl.p->exp_total, sizeof(int), cudaMemcpyDeviceToHost, s), "expansions");
    check(cudaStreamSynchronize(s), "D2H");
    st.expansions = exp_total;
    if (wave_error == 3) throw TideError("GPU path: a histogram's TMA staging wait gave up");
    if (wave_error) throw TideError("GPU path: a wave outgrew its histogram slots or partition tiles");
    B.trees.assign(T, HostTree());
    for (int t = 0; t < T; ++t) {
        const int nn = st_h[t].n_nodes;
        HostTree& tr = B.trees[t];
        tr.nodes.resize(nn);
        for (int k = 0; k < nn; ++k) {
            const DevNode& d = nodes_h[static_cast<size_t>(t) * max_nodes + k];
            tr.nodes[k] = HostNode{d.is_leaf, d.feature, d.threshold, d.left, d.right, d.missing_left,
                                   d.count, d.depth, d.value, d.is_leaf ? 0.0 : d.gain, 0, {0, 0, 0, 0}};
            tr.nodes[k].feature2 = -1;
            if (!d.is_leaf && d.type == 2) {
                tr.nodes[k].type = 2;
                for (int q = 0; q < 4; ++q) tr.nodes[k].cat[q] = d.cat[q];
            }
            if (!d.is_leaf && d.type == 1) {
                tr.nodes[k].type = 1;
                tr.nodes[k].feature2 = d.feature2;
            }
        }
        tr.values.assign(vals_h.begin() + static_cast<size_t>(t) * max_nodes,
                         vals_h.begin() + static_cast<size_t>(t) * max_nodes + nn);
        tr.cover.assign(cov_h.begin() + static_cast<size_t>(t) * max_nodes,
                        cov_h.begin() + static_cast<size_t>(t) * max_nodes + nn);
        tr.prefix.assign(pre_h.begin() + static_cast<size_t>(t) * nbk * max_nodes,
                         pre_h.begin() + static_cast<size_t>(t) * nbk * max_nodes + static_cast<size_t>(nbk) * nn);
    }
    st.t_download = now() - td;
    B.cfg = c;
    B.fitted = true;
    D.trees_flat = 0;
    // The fit's working buffers go back to the pool (ordered on the stream); a fitted model
    // keeps only its host-side trees and edges, and predict allocates what it needs.
    const double trl = now();
    rows_counter.release();
    D.release_fit_buffers();
    st.t_release = now() - trl;
    st.gpu_launches = static_cast<int>(g_kernel_launches.load() - launches0);
    st.t_total = now() - t0;
    return overflow != 0;
}

// ---- batched growth over one or many contexts -------------------------------------------
//
// The wave sequence of one tree of every context: roots (histogram, scan, select), then
// waves (partition, histogram of the smaller children, scan, select) until no context
// grows.  With `graph`, the whole sequence is one CUDA graph per fit: a conditional WHILE
// node repeats the wave body while select leaves the loop condition at 1, so a tree costs
// one graph launch and no host round trip.  Without it the host enqueues waves ahead of
// the device and stops two waves after a mapped flag says every tree is done.
// Mapped host flags of the host-driven wave loop, kept for the process: allocating and
// freeing mapped pinned memory can take tens to hundreds of milliseconds, which every fit
// would otherwise pay.  Portable, so any device may use a flag.
struct WaveFlagPool {
    std::mutex mu;
    std::vector<unsigned*> free;
};
WaveFlagPool& wave_flag_pool() {
    static WaveFlagPool* p = new WaveFlagPool();  // outlives every booster (never destroyed)
    return *p;
}
unsigned* take_wave_flag() {
    WaveFlagPool& p = wave_flag_pool();
    {
        std::lock_guard<std::mutex> lk(p.mu);
        if (!p.free.empty()) {
            unsigned* f = p.free.back();
            p.free.pop_back();
            return f;
        }
    }
    unsigned* f = nullptr;
    check(cudaHostAlloc(reinterpret_cast<void**>(&f), sizeof(unsigned), cudaHostAllocMapped | cudaHostAllocPortable),
          "cudaHostAlloc (wave flag)");
    return f;
}
void give_wave_flag(unsigned* f) {
    WaveFlagPool& p = wave_flag_pool();
    std::lock_guard<std::mutex> lk(p.mu);
    p.free.push_back(f);
}

class WaveDriver {
public:
    WaveDriver(std::vector<FitRun*> runs, cudaStream_t s, bool use_graph, bool tune, unsigned long long* rows_counter)
        : runs_(std::move(runs)), s_(s), rows_counter_(rows_counter), use_graph_(use_graph), autotune_(tune) {
        n_ctx_ = static_cast<int>(runs_.size());
        if (n_ctx_ < 1 || n_ctx_ > kMaxWaveCtx) throw TideError("wave: 1 to 64 contexts per launch");
        int leaves = 0;
        for (auto* r : runs_) {
            max_f_ = std::max(max_f_, r->n_f);
            max_leaves_ = std::max(max_leaves_, r->c.max_leaves);
            leaves += r->c.max_leaves;
            rows_ += r->n;
            pair_ = pair_ || r->c.pair_splits;
            cat_ = cat_ || r->any_cat;
            if (r->mode != runs_[0]->mode) throw TideError("wave: all contexts of a launch share one histogram mode");
        }
        if (leaves > kMaxWaveJobs) throw TideError("wave: too many leaves over the contexts of one launch");
        mode_ = runs_[0]->mode;
        tune_.cluster = 4;
        tune_.clusters = wave_hist_clusters(4);
        ctx_.alloc(n_ctx_, s_);
        std::vector<WaveCtx> h(n_ctx_);
        for (int k = 0; k < n_ctx_; ++k) h[k] = runs_[k]->wave_ctx();
        check(cudaMemcpyAsync(ctx_.p, h.data(), sizeof(WaveCtx) * n_ctx_, cudaMemcpyHostToDevice, s_), "contexts");
        gsync_.alloc(3, s_);
        check(cudaMemsetAsync(gsync_.p, 0, 3 * sizeof(int), s_), "gsync reset");
        part_grid_ = 148 * 8;
        scan_ys_ = std::min(64, std::max(2, 2 * max_leaves_ * n_ctx_ / 4));
    }
    bool graph_used() const { return exec_ != nullptr; }
    const HistTune& tune() const { return tune_; }

    // Launch shape of the histogram, tuned once per (device, payload mode, contexts, feature
    // count, rows bucket) in the process: every candidate (1, 2 or 4 CTAs per cluster)
    // builds the first tree's root histograms, timed with CUDA events (a warm-up run, then
    // the better of two), and the fastest is kept.  The root
    // slots are cleared before each run and after the last, so the tree starts afresh.
    void autotune() {
        int dev = 0;
        check(cudaGetDevice(&dev), "cudaGetDevice");
        int rb = 0;
        while ((1ll << rb) < rows_) ++rb;
        const long long key = ((((static_cast<long long>(dev) * 8 + mode_) * 128 + n_ctx_) * 4096 + max_f_) * 64) + rb;
        static std::mutex mu;
        static std::vector<std::pair<long long, HistTune>> cache;
        {
            std::lock_guard<std::mutex> lk(mu);
            for (auto& kv : cache)
                if (kv.first == key) {
                    tune_ = kv.second;
                    return;
                }
        }
        cudaEvent_t a, b;
        check(cudaEventCreate(&a), "event");
        check(cudaEventCreate(&b), "event");
        HistTune best = tune_;
        float best_ms = 1e30f;
        for (int cl : {1, 2, 4}) {
            HistTune t;
            t.cluster = cl;
            t.clusters = wave_hist_clusters(cl);
            float ms_min = 1e30f;
            for (int rep = 0; rep < 3; ++rep) {
                zero_roots();
                check(cudaEventRecord(a, s_), "event record");
                launch_wave_hist(mode_, ctx_.p, n_ctx_, 0, t, nullptr, s_);
                check(cudaEventRecord(b, s_), "event record");
                check(cudaEventSynchronize(b), "tune event");
                float ms = 0.f;
                check(cudaEventElapsedTime(&ms, a, b), "tune time");
                if (rep > 0) ms_min = std::min(ms_min, ms);
            }
            if (ms_min < best_ms) {
                best_ms = ms_min;
                best = t;
            }
        }
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        zero_roots();
        tune_ = best;
        std::lock_guard<std::mutex> lk(mu);
        cache.emplace_back(key, best);
    }

    // The first tree's set-up has run (the roots' rows and payloads are on the device):
    // tune, then capture the graph with the tuned launch shape.
    void first_tree() {
        if (ready_) return;
        ready_ = true;
        if (autotune_) autotune();
        if (use_graph_) {
            try {
                build_graph();
            } catch (const TideError&) {
                // a driver without device-side graph loops: the host enqueues the waves
                cudaStreamCaptureStatus cs;
                if (cudaStreamIsCapturing(s_, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) {
                    cudaGraph_t g = nullptr;
                    cudaStreamEndCapture(s_, &g);
                    if (g) cudaGraphDestroy(g);
                }
                (void)cudaGetLastError();
                if (exec_) cudaGraphExecDestroy(exec_);
                if (graph_) cudaGraphDestroy(graph_);
                exec_ = nullptr;
                graph_ = nullptr;
            }
        }
    }
    // selects run (device counter), for the count of kernels the waves launched
    long long selects() {
        int v = 0;
        check(cudaMemcpyAsync(&v, gsync_.p + 2, sizeof(int), cudaMemcpyDeviceToHost, s_), "select count");
        check(cudaStreamSynchronize(s_), "select count");
        return v;
    }
    ~WaveDriver() {
        if (exec_) cudaGraphExecDestroy(exec_);
        if (graph_) cudaGraphDestroy(graph_);
        if (hflag_) give_wave_flag(hflag_);
        for (auto& e : ev_) cudaEventDestroy(e);
    }

    // One tree of every context.  hist_ev: optional event pairs around each histogram launch
    // (host-driven mode only); rows_counter: optional device counter of histogrammed rows.
    void grow(std::vector<cudaEvent_t>* hist_ev, size_t* hist_used) {
        first_tree();
        unsigned long long* rows_counter = rows_counter_;
        if (exec_ && hist_ev == nullptr) {
            check(cudaGraphLaunch(exec_, s_), "wave graph launch");
            return;
        }
        auto hist = [&](int src) {
            const bool prof = hist_ev && *hist_used + 2 <= hist_ev->size();
            if (prof) check(cudaEventRecord((*hist_ev)[*hist_used], s_), "event record");
            launch_wave_hist(mode_, ctx_.p, n_ctx_, src, tune_, rows_counter, s_);
            if (prof) {
                check(cudaEventRecord((*hist_ev)[*hist_used + 1], s_), "event record");
                *hist_used += 2;
            }
        };
        if (hflag_ == nullptr) {  // the loop flag of the host-driven waves (mapped host memory)
            hflag_ = take_wave_flag();
            check(cudaHostGetDevicePointer(reinterpret_cast<void**>(&dflag_), hflag_, 0), "wave flag pointer");
            *reinterpret_cast<volatile unsigned*>(hflag_) = 1u;
        }
        hist(0);
        launch_wave_scan(ctx_.p, n_ctx_, 0, max_f_, scan_ys_, cat_, s_);
        if (pair_) launch_wave_pair(ctx_.p, n_ctx_, 0, s_);
        launch_wave_select(ctx_.p, n_ctx_, gsync_.p, dflag_, 0ull, 0, s_);
        // waves, enqueued ahead; the flag written by wave w's select is read once wave w
        // has completed (its event), two waves behind the host
        const int max_waves = max_leaves_;
        if (static_cast<int>(ev_.size()) < max_waves + 1) {
            const size_t old = ev_.size();
            ev_.resize(max_waves + 1);
            for (size_t k = old; k < ev_.size(); ++k)
                check(cudaEventCreateWithFlags(&ev_[k], cudaEventDisableTiming), "event");
        }
        check(cudaEventRecord(ev_[0], s_), "event record");
        for (int w = 1; w <= max_waves; ++w) {
            if (w >= 3) {
                check(cudaEventSynchronize(ev_[w - 2]), "wave event");
                if (*reinterpret_cast<volatile unsigned*>(hflag_) == 0u) break;
            }
            launch_wave_partition(ctx_.p, n_ctx_, part_grid_, s_);
            hist(1);
            launch_wave_scan(ctx_.p, n_ctx_, 1, max_f_, scan_ys_, cat_, s_);
            if (pair_) launch_wave_pair(ctx_.p, n_ctx_, 1, s_);
            launch_wave_select(ctx_.p, n_ctx_, gsync_.p, dflag_, 0ull, 0, s_);
            check(cudaEventRecord(ev_[w], s_), "event record");
        }
    }

private:
    void zero_roots() {
        for (auto* r : runs_) {
            const size_t slot = static_cast<size_t>(r->n_f) * kBins;
            check(cudaMemsetAsync(r->D.histG.p, 0, sizeof(long long) * slot, s_), "hist reset");
            check(cudaMemsetAsync(r->D.histH.p, 0, sizeof(long long) * slot, s_), "hist reset");
            check(cudaMemsetAsync(r->D.histC.p, 0, sizeof(int) * slot, s_), "hist reset");
        }
    }

    void build_graph() {
        // root stage captured into the top graph, then a WHILE node whose body is one wave
        check(cudaGraphCreate(&graph_, 0), "graph create");
        cudaGraphConditionalHandle handle;
        check(cudaGraphConditionalHandleCreate(&handle, graph_, 1, cudaGraphCondAssignDefault),
              "graph conditional handle");
        check(cudaStreamBeginCaptureToGraph(s_, graph_, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal),
              "graph capture");
        launch_wave_hist(mode_, ctx_.p, n_ctx_, 0, tune_, rows_counter_, s_);
        launch_wave_scan(ctx_.p, n_ctx_, 0, max_f_, scan_ys_, cat_, s_);
        if (pair_) launch_wave_pair(ctx_.p, n_ctx_, 0, s_);
        launch_wave_select(ctx_.p, n_ctx_, gsync_.p, nullptr, handle, 1, s_);
        cudaStreamCaptureStatus cs;
        const cudaGraphNode_t* deps = nullptr;
        size_t n_deps = 0;
        check(cudaStreamGetCaptureInfo(s_, &cs, nullptr, nullptr, &deps, &n_deps), "capture info");
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = handle;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t cond_node;
        check(cudaGraphAddNode(&cond_node, graph_, deps, n_deps, &cp), "graph conditional node");
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        check(cudaStreamUpdateCaptureDependencies(s_, &cond_node, 1, cudaStreamSetCaptureDependencies),
              "capture dependencies");
        cudaGraph_t top = nullptr;
        check(cudaStreamEndCapture(s_, &top), "graph capture end");
        // the body: one wave
        check(cudaStreamBeginCaptureToGraph(s_, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal),
              "body capture");
        launch_wave_partition(ctx_.p, n_ctx_, part_grid_, s_);
        launch_wave_hist(mode_, ctx_.p, n_ctx_, 1, tune_, rows_counter_, s_);
        launch_wave_scan(ctx_.p, n_ctx_, 1, max_f_, scan_ys_, cat_, s_);
        if (pair_) launch_wave_pair(ctx_.p, n_ctx_, 1, s_);
        launch_wave_select(ctx_.p, n_ctx_, gsync_.p, nullptr, handle, 1, s_);
        cudaGraph_t body_out = nullptr;
        check(cudaStreamEndCapture(s_, &body_out), "body capture end");
        check(cudaGraphInstantiate(&exec_, graph_, 0), "graph instantiate");
        // launches counted per grow (the graph's kernels are this library's)
        g_kernel_launches.fetch_sub(pair_ ? 12 : 8);
    }

    std::vector<FitRun*> runs_;
    cudaStream_t s_;
    unsigned long long* rows_counter_;
    bool use_graph_, autotune_, ready_ = false, pair_ = false, cat_ = false;
    HistTune tune_;
    int n_ctx_ = 0, max_f_ = 0, max_leaves_ = 0, mode_ = 0, part_grid_ = 0, scan_ys_ = 0;
    long long rows_ = 0;
    DBuf<WaveCtx> ctx_;
    DBuf<int> gsync_;
    unsigned* hflag_ = nullptr;
    unsigned* dflag_ = nullptr;
    std::vector<cudaEvent_t> ev_;
    cudaGraph_t graph_ = nullptr;
    cudaGraphExec_t exec_ = nullptr;
};

// Trees of every run in lockstep: per tree, every run's set-up, one growth (waves over all
// runs, or each run's one-split loop), every run's post-tree sweep.  Timing hooks come
// from runs[0]'s config and cover all runs' trees.
void fit_runs(std::vector<FitRun*>& runs, cudaStream_t s) {
    FitRun& r0 = *runs[0];
    const Config& c = r0.c;
    const int T = r0.T;
    for (auto* r : runs)
        if (r->T != T) throw TideError("batched fits need equal n_estimators");
    const bool wave = c.grow != 0;
    const bool timing = c.timing_from >= 0 && c.timing_from < T;
    const int timing_end = (c.timing_to < 0 || c.timing_to > T) ? T : std::max(c.timing_to, c.timing_from + 1);
    cudaEvent_t ev_begin = nullptr, ev_end = nullptr;
    long long launches_begin = 0, launches_end = 0, selects_begin = 0, selects_end = 0;
    // rows histogrammed: [0] running count, [1] at the start of the timed range, [2] at its end
    r0.rows_counter.alloc(3, s);
    check(cudaMemsetAsync(r0.rows_counter.p, 0, 3 * sizeof(unsigned long long), s), "counter reset");
    if (timing) {
        check(cudaEventCreate(&ev_begin), "event");
        check(cudaEventCreate(&ev_end), "event");
        if (c.profile_hist) {
            r0.hist_ev.resize(static_cast<size_t>(2) * (timing_end - c.timing_from) * (c.max_leaves + 1));
            for (auto& e : r0.hist_ev) check(cudaEventCreate(&e), "event");
        }
    }
    std::unique_ptr<WaveDriver> drv;
    if (wave) {
        const double td = now();
        std::vector<FitRun*> rr(runs.begin(), runs.end());
        drv = std::make_unique<WaveDriver>(rr, s, c.graph != 0, c.hist_tune != 0, r0.rows_counter.p);
        for (auto* r : runs) r->st.t_driver = now() - td;
    }
    const double ttree = now();
    for (int t = 0; t < T; ++t) {
        const bool in_timed = timing && t >= c.timing_from && t < timing_end;
        if (timing && t == c.timing_from) {
            if (drv) selects_begin = drv->selects();  // before the timed range: it waits for the device
            check(cudaEventRecord(ev_begin, s), "event record");
            check(cudaMemcpyAsync(r0.rows_counter.p + 1, r0.rows_counter.p, 8, cudaMemcpyDeviceToDevice, s), "counter");
            launches_begin = g_kernel_launches.load();
        }
        if (timing && t == timing_end) {
            check(cudaEventRecord(ev_end, s), "event record");
            check(cudaMemcpyAsync(r0.rows_counter.p + 2, r0.rows_counter.p, 8, cudaMemcpyDeviceToDevice, s), "counter");
            launches_end = g_kernel_launches.load();
            if (drv) selects_end = drv->selects();
        }
        for (auto* r : runs) r->tree_begin(t);
        if (wave) {
            const bool prof = in_timed && c.profile_hist;
            drv->grow(prof ? &r0.hist_ev : nullptr, prof ? &r0.hist_ev_used : nullptr);
        } else {
            for (auto* r : runs) r->grow_leafwise(in_timed);
        }
        for (auto* r : runs) r->tree_end(t);
    }
    if (timing && timing_end == T) {
        check(cudaEventRecord(ev_end, s), "event record");
        check(cudaMemcpyAsync(r0.rows_counter.p + 2, r0.rows_counter.p, 8, cudaMemcpyDeviceToDevice, s), "counter");
        launches_end = g_kernel_launches.load();
        if (drv) selects_end = drv->selects();
    }
    if (drv) {
        r0.st.graph_used = drv->graph_used() ? 1 : 0;
        r0.st.hist_cluster = drv->tune().cluster;
        r0.st.hist_clusters = drv->tune().clusters;
    }
    check(cudaStreamSynchronize(s), "tree loop");
    for (auto* r : runs) r->st.t_trees = now() - ttree;
    if (timing) {
        float ms = 0.f;
        check(cudaEventElapsedTime(&ms, ev_begin, ev_end), "event time");
        r0.st.timed_ms = ms;
        r0.st.timed_trees = (timing_end - c.timing_from) * static_cast<int>(runs.size());
        r0.st.timed_launches = launches_end - launches_begin;
        r0.st.timed_selects = selects_end - selects_begin;
        unsigned long long rc[3] = {0, 0, 0};
        check(cudaMemcpy(rc, r0.rows_counter.p, sizeof(rc), cudaMemcpyDeviceToHost), "counter");
        r0.st.hist_rows = static_cast<long long>(rc[2] - rc[1]);
        for (size_t k = 0; k + 1 < r0.hist_ev_used; k += 2) {
            float hm = 0.f;
            check(cudaEventElapsedTime(&hm, r0.hist_ev[k], r0.hist_ev[k + 1]), "event time");
            r0.st.hist_ms += hm;
            r0.st.hist_launches += 1;
        }
        cudaEventDestroy(ev_begin);
        cudaEventDestroy(ev_end);
    }
    const double tdf = now();
    drv.reset();  // the tree graph, the mapped loop flag and the contexts
    for (auto* r : runs) r->st.t_driver_free = now() - tdf;
}

void GpuBooster::fit(const void* X_in, int x_dtype, const double* y_in, int n, int n_f, const int64_t* ts_in,
                     const int64_t* ent_in) {
    // The GOSS order comes from a 32-bit-key sort plus an exact fix-up of tied runs; a
    // run too long for the fix-up (many distinct |g| within 2^-21 relative of each other)
    // is reported by the device, and the fit is then repeated with the full 64-bit sort.
    const bool overflow = fit_once(X_in, x_dtype, y_in, n, n_f, ts_in, ent_in, false);
    if (overflow) {
        const FitStats first = stats;
        fit_once(X_in, x_dtype, y_in, n, n_f, ts_in, ent_in, true);
        stats.goss_refits = 1;
        stats.t_total += first.t_total;
    }
}

bool GpuBooster::fit_once(const void* X_in, int x_dtype, const double* y_in, int n, int n_f, const int64_t* ts_in,
                          const int64_t* ent_in, bool exact_goss) {
    stats = FitStats();
    FitRun run(*this, cfg, *ds_, ds_->stream, exact_goss);
    run.prepare(X_in, x_dtype, y_in, n, n_f, ts_in, ent_in);
    std::vector<FitRun*> runs{&run};
    fit_runs(runs, ds_->stream);
    const bool overflow = run.finish();
    stats = run.st;
    return overflow;
}

void GpuBooster::fit_batch(const std::vector<GpuBooster*>& bs, const std::vector<FitInput>& in) {
    if (bs.empty() || bs.size() != in.size()) throw TideError("fit_batch: one input per booster");
    GpuBooster& b0 = *bs[0];
    check(cudaSetDevice(b0.device), "cudaSetDevice");
    for (auto* b : bs)
        if (b->device != b0.device) throw TideError("fit_batch: boosters must share one device");
    cudaStream_t s = b0.ds_->stream;
    std::vector<std::unique_ptr<FitRun>> own;
    std::vector<FitRun*> runs;
    for (size_t k = 0; k < bs.size(); ++k) {
        bs[k]->stats = FitStats();
        Config ck = bs[k]->cfg;
        if (k > 0) {  // one timing range for the whole batch
            ck.timing_from = -1;
            ck.profile_hist = false;
        }
        own.push_back(std::make_unique<FitRun>(*bs[k], ck, *bs[k]->ds_, s, false));
        own.back()->prepare(in[k].X, in[k].x_dtype, in[k].y, in[k].n, in[k].n_f, in[k].ts, in[k].entity);
        runs.push_back(own.back().get());
    }
    fit_runs(runs, s);
    std::vector<size_t> refit;
    for (size_t k = 0; k < bs.size(); ++k) {
        if (runs[k]->finish()) refit.push_back(k);
        bs[k]->stats = runs[k]->st;
    }
    own.clear();
    // a run whose GOSS order needs the 64-bit sort is repeated alone (rare)
    for (size_t k : refit) {
        bs[k]->fit_once(in[k].X, in[k].x_dtype, in[k].y, in[k].n, in[k].n_f, in[k].ts, in[k].entity, true);
        bs[k]->stats.goss_refits = 1;
    }
}

void GpuBooster::predict_raw(const void* X, int x_dtype, int n, int n_f, double* out) {
    if (!fitted) throw TideError("not fitted");
    if (n_f != n_features) throw TideError("n_features mismatch");
    if (n <= 0) return;
    check(cudaSetDevice(device), "cudaSetDevice");
    DeviceState& D = *ds_;
    cudaStream_t s = D.stream;
    const int stride = (n_f + 15) / 16 * 16;
    const size_t xsz = x_dtype == 0 ? 4 : 8;
    // Flattened trees (booster.cpp:744-773 uses tree.values, not the TORB prefixes).
    if (D.trees_flat != trees.size()) {
        std::vector<int16_t> f, l, r, f2;
        std::vector<uint8_t> th, ml, ty;
        std::vector<unsigned long long> cm;
        std::vector<double> v;
        std::vector<int> off;
        for (const auto& t : trees) {
            off.push_back(static_cast<int>(f.size()));
            for (size_t k = 0; k < t.nodes.size(); ++k) {
                const HostNode& d = t.nodes[k];
                f.push_back(static_cast<int16_t>(d.is_leaf ? -1 : d.feature));
                l.push_back(static_cast<int16_t>(d.left));
                r.push_back(static_cast<int16_t>(d.right));
                th.push_back(static_cast<uint8_t>(d.threshold < 0 ? 0 : d.threshold));
                ml.push_back(static_cast<uint8_t>(d.missing_left));
                ty.push_back(static_cast<uint8_t>(d.is_leaf ? 0 : d.type));
                f2.push_back(static_cast<int16_t>(!d.is_leaf && d.type == 1 ? d.feature2 : 0));
                for (int q = 0; q < 4; ++q) cm.push_back(d.cat[q]);
                v.push_back(t.values[k]);
            }
        }
        D.t_feat2.alloc(std::max<size_t>(1, f2.size()), s);
        if (!f2.empty()) check(cudaMemcpyAsync(D.t_feat2.p, f2.data(), 2 * f2.size(), cudaMemcpyHostToDevice, s), "trees");
        D.t_type.alloc(std::max<size_t>(1, ty.size()), s);
        D.t_cat.alloc(std::max<size_t>(4, cm.size()), s);
        if (!ty.empty()) {
            check(cudaMemcpyAsync(D.t_type.p, ty.data(), ty.size(), cudaMemcpyHostToDevice, s), "trees");
            check(cudaMemcpyAsync(D.t_cat.p, cm.data(), 8 * cm.size(), cudaMemcpyHostToDevice, s), "trees");
        }
        D.t_feat.alloc(f.size(), s);
        D.t_left.alloc(l.size(), s);
        D.t_right.alloc(r.size(), s);
        D.t_thr.alloc(th.size(), s);
        D.t_ml.alloc(ml.size(), s);
        D.t_val.alloc(v.size(), s);
        D.t_off.alloc(std::max<size_t>(1, off.size()), s);
        check(cudaMemcpyAsync(D.t_feat.p, f.data(), 2 * f.size(), cudaMemcpyHostToDevice, s), "trees");
        check(cudaMemcpyAsync(D.t_left.p, l.data(), 2 * l.size(), cudaMemcpyHostToDevice, s), "trees");
        check(cudaMemcpyAsync(D.t_right.p, r.data(), 2 * r.size(), cudaMemcpyHostToDevice, s), "trees");
        check(cudaMemcpyAsync(D.t_thr.p, th.data(), th.size(), cudaMemcpyHostToDevice, s), "trees");
        check(cudaMemcpyAsync(D.t_ml.p, ml.data(), ml.size(), cudaMemcpyHostToDevice, s), "trees");
        check(cudaMemcpyAsync(D.t_val.p, v.data(), 8 * v.size(), cudaMemcpyHostToDevice, s), "trees");
        if (!off.empty())
            check(cudaMemcpyAsync(D.t_off.p, off.data(), 4 * off.size(), cudaMemcpyHostToDevice, s), "trees");
        check(cudaStreamSynchronize(s), "trees");
        D.trees_flat = trees.size();
    }
    DBuf<unsigned char> Xd;
    Xd.alloc(static_cast<size_t>(n) * n_f * xsz, s);
    D.pcodes.alloc(static_cast<size_t>(n) * stride, s);
    D.pout.alloc(n, s);
    check(cudaMemcpyAsync(Xd.p, X, static_cast<size_t>(n) * n_f * xsz, cudaMemcpyHostToDevice, s), "X upload");
    DBuf<int> ne;
    ne.alloc(n_f, s);
    check(cudaMemcpyAsync(ne.p, n_edges.data(), sizeof(int) * n_f, cudaMemcpyHostToDevice, s), "edges");
    if (x_dtype == 0) {
        std::vector<float> ef(static_cast<size_t>(n_f) * 256, INFINITY);
        for (int ff = 0; ff < n_f; ++ff)
            for (int k = 0; k < n_edges[ff]; ++k) ef[static_cast<size_t>(ff) * 256 + k] = ceil_f32(edges[static_cast<size_t>(ff) * 256 + k]);
        DBuf<float> ed;
        ed.alloc(ef.size(), s);
        check(cudaMemcpyAsync(ed.p, ef.data(), 4 * ef.size(), cudaMemcpyHostToDevice, s), "edges");
        launch_bin_transform_f32(reinterpret_cast<const float*>(Xd.p), n, n_f, ed.p, ne.p, D.pcodes.p, stride, s,
                                 D.is_cat.p);
        check(cudaStreamSynchronize(s), "transform");
    } else {
        std::vector<double> eh(static_cast<size_t>(n_f) * 256, INFINITY);
        for (int ff = 0; ff < n_f; ++ff)
            for (int k = 0; k < n_edges[ff]; ++k) eh[static_cast<size_t>(ff) * 256 + k] = edges[static_cast<size_t>(ff) * 256 + k];
        DBuf<double> ed;
        ed.alloc(eh.size(), s);
        check(cudaMemcpyAsync(ed.p, eh.data(), 8 * eh.size(), cudaMemcpyHostToDevice, s), "edges");
        launch_bin_transform_f64(reinterpret_cast<const double*>(Xd.p), n, n_f, ed.p, ne.p, D.pcodes.p, stride, s,
                                 D.is_cat.p);
        check(cudaStreamSynchronize(s), "transform");
    }
    launch_predict_trees(D.pcodes.p, stride, n, D.t_feat.p, D.t_left.p, D.t_right.p, D.t_thr.p, D.t_ml.p, D.t_val.p,
                         D.t_off.p, static_cast<int>(trees.size()), init_score, cfg.learning_rate, D.t_type.p, D.t_cat.p, D.t_feat2.p,
                         n_bins, D.pout.p, s);
    check(cudaMemcpyAsync(out, D.pout.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s), "predict D2H");
    check(cudaStreamSynchronize(s), "predict");
}

}  // namespace tgb
