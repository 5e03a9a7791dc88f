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
    if (hist_bits != 0 && hist_bits != 8) throw TideError("hist_bits must be 0 (exact) or 8 (int8 gradients)");
    if (hist_bits == 8 && objective != 0) throw TideError("hist_bits = 8 needs a constant hessian (objective mse)");
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
    // predict
    DBuf<uint8_t> pcodes;
    DBuf<int16_t> t_feat, t_left, t_right;
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
    const double t0 = now();
    stats = FitStats();
    const long long launches0 = g_kernel_launches.load();
    check(cudaSetDevice(device), "cudaSetDevice");
    Config c = cfg;
    if (n >= 1000000) {  // booster.cpp:237-240
        c.halo = false;
        c.pair_splits = false;
    }
    c.validate();
    if (c.pair_splits) throw TideError("GPU path: pair_splits is not supported; pass pair_splits=False");
    if (c.halo) throw TideError("GPU path: halo is not supported");
    if (n <= 0 || n_f <= 0) throw TideError("empty input");
    if (x_dtype != 0 && x_dtype != 1) throw TideError("x_dtype must be 0 (float32) or 1 (float64)");
    if (!c.iid_mode && !ts_in) throw TideError("timestamp is required unless iid_mode");
    if (c.objective == 5 && !ts_in) throw TideError("rank objective requires timestamps");
    const size_t xsz = x_dtype == 0 ? 4 : 8;
    cudaStream_t s = ds_->stream;
    DeviceState& D = *ds_;
    const int n_threads = c.n_jobs > 0 ? c.n_jobs : std::max(1u, std::thread::hardware_concurrency());

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
        const bool sorted = !unsorted.load();
        if (!sorted) {
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
    stats.t_sort = now() - t0;
    const double t_pre0 = now();

    // GOSS: booster.cpp:554-585 (sample = all rows since subsample = 1).  The draw
    // positions depend only on n and the config, so the sampler's producer starts now and
    // walks the generator while the data are uploaded and binned.
    const int T = c.n_estimators;
    const bool use_goss = ((c.goss > 0) || (c.goss < 0 && n >= 250000)) && c.goss_top < 1.0 && n > 64;
    int n_top = 0, n_other = 0;
    int64_t m_rest = 0;
    const double goss_scale = (1.0 - c.goss_top) / std::max(c.goss_other, 1e-12);
    std::unique_ptr<GossSampler> sampler;
    if (use_goss) {
        n_top = std::min(n, std::max(1, static_cast<int>(std::ceil(c.goss_top * static_cast<double>(n)))));
        m_rest = n - n_top;
        n_other = std::min(static_cast<int>(std::ceil(c.goss_other * static_cast<double>(n))), static_cast<int>(m_rest));
        // The booster's generator (booster.cpp:483) is only used by GOSS and grow_tree's
        // seed draw, so the sampler owns the whole stream.
        sampler = std::make_unique<GossSampler>(static_cast<uint32_t>(c.random_state), m_rest, n_other, T, 8,
                                                std::max(1, std::min(8, n_threads - 2)));
    }

    // ---- TORB buckets + prefix cuts: booster.cpp:311-364 ----
    int nbk = 1;
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
    n_buckets = nbk;

    // ---- initial predictions: booster.cpp:399-457 ----
    // A sequential FP64 pass over y in row order (the reference's summation order); it
    // runs on the host while the X upload is in flight (below).
    std::vector<double> fill_prefix;
    auto initial_predictions = [&] {
        init_prefix.assign(nbk, 0.0);
        if (c.objective == 5) {
            init_score = 0.0;
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
            init_score = sw > 0 ? sy / sw : 0;
            if (!c.iid_mode) init_prefix = at_cut;
        }
        // Device fill values: the prior of each bucket, or init_score for every row in iid
        // mode (where the reference leaves init_prefix = {0.0}, booster.cpp:400).
        if (c.iid_mode) {
            init_prefix.assign(1, 0.0);
            fill_prefix.assign(1, init_score);
        } else {
            for (int b = 0; b < nbk; ++b)
                if (!std::isfinite(init_prefix[b])) init_prefix[b] = init_score;
            fill_prefix = init_prefix;
        }
    };

    stats.t_pre_upload = now() - t_pre0;  // GOSS sampler start, TORB buckets and cuts
    // ---- device buffers ----
    double tb = now();
    const int stride = (n_f + 15) / 16 * 16;
    const int max_nodes = 2 * c.max_leaves - 1;
    const size_t slot = static_cast<size_t>(n_f) * kBins;
    D.codes.alloc(static_cast<size_t>(n) * stride, s);
    D.codes_col.alloc(static_cast<size_t>(n_f) * codes_col_pitch(n), s);
    D.y.alloc(n, s);
    D.pred.alloc(n, s);
    D.g.alloc(n, s);
    if (c.objective != 0) D.h.alloc(n, s);  // MSE hessians are implicit (unit)
    if (c.objective == 0 && c.hist_bits == 0) D.gq.alloc(n, s);
    if (c.hist_bits == 8) D.gq8.alloc(n, s);
    D.rows0.alloc(n, s);
    D.rows1.alloc(n, s);
    D.histG.alloc(slot * max_nodes, s);
    D.histH.alloc(slot * max_nodes, s);
    D.histC.alloc(slot * max_nodes, s);
    D.nodes.alloc(kMaxNodes, s);
    D.splits.alloc(kMaxNodes, s);
    D.st.alloc(1, s);
    const int max_tiles = (n + kPartTile - 1) / kPartTile;
    D.tile_counts.alloc(max_tiles + 1, s);
    D.scan_gain.alloc(2 * scan_ctas_per_node(n_f), s);
    D.scan_key.alloc(2 * scan_ctas_per_node(n_f), s);
    D.scan_ticket.alloc(3, s);
    check(cudaMemsetAsync(D.scan_ticket.p, 0, 3 * sizeof(int), s), "ticket reset");
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
        stats.t_alloc = now() - tb;
        DBuf<unsigned char> Xd;
        Xd.alloc(static_cast<size_t>(n) * n_f * xsz, s);
        check(cudaMemcpyAsync(Xd.p, X, static_cast<size_t>(n) * n_f * xsz, cudaMemcpyHostToDevice, s), "X upload");
        check(cudaMemcpyAsync(D.y.p, y, sizeof(double) * n, cudaMemcpyHostToDevice, s), "y upload");
        initial_predictions();  // host work while the copies run (they only read X and y)
        check(cudaStreamSynchronize(s), "X upload");
        stats.t_h2d = now() - tb - stats.t_alloc;
        // ---- quantile edges: Binner::fit (binning.cpp:34-102) on the uploaded X ----
        const double tbf = now();
        BinFitTimes bt;
        if (binner_fits_device(n, n_f, c.bin_sample))
            n_bins = binner_fit_device(Xd.p, x_dtype, n, n_f, c.max_bin, c.bin_sample,
                                       static_cast<uint32_t>(c.random_state), edges, n_edges, n_threads, s,
                                       D.codes_col.p, D.codes_col.n, &bt);  // scratch: codes_col, filled later
        else
            n_bins = binner_fit(X, x_dtype, n, n_f, c.max_bin, c.bin_sample, static_cast<uint32_t>(c.random_state),
                                edges, n_edges, n_threads);
        n_features = n_f;
        stats.t_binfit = now() - tbf;
        stats.t_bin_counts = bt.counts;
        stats.t_bin_draws = bt.draws;
        stats.t_bin_edges = bt.edges;
        DBuf<int> ne;
        ne.alloc(n_f, s);
        check(cudaMemcpyAsync(ne.p, n_edges.data(), sizeof(int) * n_f, cudaMemcpyHostToDevice, s), "edges upload");
        if (x_dtype == 0) {
            std::vector<float> ef(static_cast<size_t>(n_f) * 256, INFINITY);
            for (int f = 0; f < n_f; ++f)
                for (int k = 0; k < n_edges[f]; ++k) ef[static_cast<size_t>(f) * 256 + k] = ceil_f32(edges[static_cast<size_t>(f) * 256 + k]);
            DBuf<float> ed;
            ed.alloc(ef.size(), s);
            check(cudaMemcpyAsync(ed.p, ef.data(), sizeof(float) * ef.size(), cudaMemcpyHostToDevice, s), "edges upload");
            launch_bin_transform_f32(reinterpret_cast<const float*>(Xd.p), n, n_f, ed.p, ne.p, D.codes.p, stride, s);
            check(cudaStreamSynchronize(s), "transform");
        } else {
            std::vector<double> ed_h(static_cast<size_t>(n_f) * 256, INFINITY);
            for (int f = 0; f < n_f; ++f)
                for (int k = 0; k < n_edges[f]; ++k) ed_h[static_cast<size_t>(f) * 256 + k] = edges[static_cast<size_t>(f) * 256 + k];
            DBuf<double> ed;
            ed.alloc(ed_h.size(), s);
            check(cudaMemcpyAsync(ed.p, ed_h.data(), sizeof(double) * ed_h.size(), cudaMemcpyHostToDevice, s),
                  "edges upload");
            launch_bin_transform_f64(reinterpret_cast<const double*>(Xd.p), n, n_f, ed.p, ne.p, D.codes.p, stride, s);
            check(cudaStreamSynchronize(s), "transform");
        }
    }
    // Column-major copy for the partition's reads of one feature over a row list.
    const double ttr = now();
    launch_codes_transpose(D.codes.p, stride, n, n_f, D.codes_col.p, s);
    check(cudaStreamSynchronize(s), "transpose");
    stats.t_transpose = now() - ttr;
    stats.t_upload = now() - tb - stats.t_binfit;
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
    std::vector<int4> chunks;
    const int kChunk = 8192;
    for (int k = 0, lo = 0; k < static_cast<int>(bounds.size()); lo = bounds[k], ++k)
        for (int a = lo; a < bounds[k]; a += kChunk) chunks.push_back(make_int4(k, a, std::min(bounds[k], a + kChunk), 0));
    const int n_segments = static_cast<int>(bounds.size());
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
    int n_runs = 0;
    const int* order_d = nullptr;
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
    GossWork gw{D.keys_in.p, D.keys_out.p, D.vals_in.p, D.vals_out.p, D.cub_tmp.p, D.cub_tmp.n,
                D.goss_overflow.p, exact_goss};

    GrowParams gp{n_f, stride, n_bins, c.max_depth, c.max_leaves, c.min_samples_leaf, c.min_child_weight, c.l2,
                  c.min_split_gain};
    PostParams pp{n, nbk, c.iid_mode ? 1 : 0, n_segments, c.learning_rate, c.l2,
                  c.torb_min_cover > 0.0 ? c.torb_min_cover : static_cast<double>(2 * std::max(c.min_samples_leaf, 1))};
    HistSlotPtrs hs{D.histG.p, D.histH.p, D.histC.p, slot};
    ScanScratch scs{D.scan_gain.p, D.scan_key.p, D.scan_ticket.p};
    int32_t* rows[2] = {D.rows0.p, D.rows1.p};
    const int grid_rows = hist_grid_rows(n_f, n, c.objective == 0);
    const double ttree = now();
    stats.t_prep = ttree - t_prep0;  // TORB segments, rank groups, GOSS buffers, initial predictions

    // Measurement hooks: events bracket the timed trees; optional event pairs bracket
    // every histogram launch in that range; a device counter adds up the rows.
    const bool timing = c.timing_from >= 0 && c.timing_from < T;
    const int timing_end = (c.timing_to < 0 || c.timing_to > T) ? T : std::max(c.timing_to, c.timing_from + 1);
    cudaEvent_t ev_begin = nullptr, ev_end = nullptr;
    std::vector<cudaEvent_t> hist_ev;
    DBuf<unsigned long long> rows_counter;
    long long launches_begin = 0;
    if (timing) {
        check(cudaEventCreate(&ev_begin), "event");
        check(cudaEventCreate(&ev_end), "event");
        rows_counter.alloc(1, s);
        check(cudaMemsetAsync(rows_counter.p, 0, sizeof(unsigned long long), s), "counter reset");
        if (c.profile_hist) {
            hist_ev.resize(static_cast<size_t>(2) * (timing_end - c.timing_from) * c.max_leaves);
            for (auto& e : hist_ev) check(cudaEventCreate(&e), "event");
        }
    }
    size_t hist_ev_used = 0;
    auto hist_launch = [&](int node, const uint8_t* flag, bool in_timed) {
        const bool prof = in_timed && c.profile_hist && hist_ev_used + 2 <= hist_ev.size();
        if (prof) check(cudaEventRecord(hist_ev[hist_ev_used], s), "event record");
        const void* gq = c.hist_bits == 8 ? static_cast<const void*>(D.gq8.p) : static_cast<const void*>(D.gq.p);
        launch_hist_node(D.codes.p, stride, n_f, rows, D.nodes.p, D.st.p, node, D.g.p, D.h.p, gq, c.hist_bits == 8,
                         flag, goss_scale, hs,
                         grid_rows, in_timed ? rows_counter.p : nullptr, c.objective == 0, s);
        if (prof) {
            check(cudaEventRecord(hist_ev[hist_ev_used + 1], s), "event record");
            hist_ev_used += 2;
        }
    };

    long long launches_end = 0;
    for (int t = 0; t < T; ++t) {
        const bool in_timed = timing && t >= c.timing_from && t < timing_end;
        if (timing && t == c.timing_from) {
            check(cudaEventRecord(ev_begin, s), "event record");
            launches_begin = g_kernel_launches.load();
        }
        if (timing && t == timing_end) {
            check(cudaEventRecord(ev_end, s), "event record");
            launches_end = g_kernel_launches.load();
        }
        // gradients (booster.cpp:701).  MSE: one pass also reduces the all-row maxima;
        // its unit hessians are never materialised (h = nullptr below).
        const bool const_h = c.objective == 0;
        if (const_h) {
            launch_grad_mse_fused(D.y.p, D.pred.p, n, D.g.p, D.all_scale.p, s);
            launch_all_scale_finalize(D.all_scale.p, n, s);
        } else {
            launch_grad_pairwise(D.y.p, D.pred.p, D.run_start.p, D.run_len.p, order_d, n_runs, n, D.g.p, D.h.p, s);
            launch_all_scale(D.g.p, D.h.p, n, D.all_scale.p, s);
        }
        const double* h_rows = const_h ? nullptr : D.h.p;
        // sample
        if (use_goss) {
            const double tr = now();
            const int32_t* pos = sampler->wait(t);  // host time spent waiting for the draw
            stats.t_rng += now() - tr;
            check(cudaMemcpyAsync(D.rest_pos.p, pos, sizeof(int32_t) * std::max(1, n_other), cudaMemcpyHostToDevice, s),
                  "positions upload");
            sampler->release(t, s);
            launch_goss_select(D.g.p, h_rows, n, n_top, n_other, D.rest_pos.p, sampler->min_pos(t), gw,
                               D.all_scale.p, goss_scale,
                               D.goss_flag.p,
                               D.rows0.p, D.tile_counts.p, D.st.p, s);
            launch_tree_init(D.nodes.p, D.splits.p, D.st.p, 0, 1, s);
            launch_scales(D.st.p, nullptr, c.hist_bits == 8, s);
        } else {
            launch_iota_rows(D.rows0.p, n, s);
            launch_tree_init(D.nodes.p, D.splits.p, D.st.p, n, 0, s);
            launch_scales(D.st.p, D.all_scale.p, c.hist_bits == 8, s);
        }
        const uint8_t* flag = use_goss ? D.goss_flag.p : nullptr;
        if (c.hist_bits == 8) {
            // per-tree stream of the stochastic rounding (SplitMix64 of seed and tree)
            uint64_t z = (static_cast<uint64_t>(static_cast<uint32_t>(c.random_state)) << 32) + static_cast<uint64_t>(t);
            z += 0x9e3779b97f4a7c15ull;
            z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
            z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
            launch_quantize8(D.rows0.p, D.g.p, flag, goss_scale, D.st.p, z ^ (z >> 31), D.gq8.p, n, s);
        } else if (const_h) {
            launch_quantize(D.rows0.p, D.g.p, flag, goss_scale, D.st.p, D.gq.p, n, s);
        }
        check(cudaMemsetAsync(D.histG.p, 0, sizeof(long long) * slot * max_nodes, s), "hist reset");
        check(cudaMemsetAsync(D.histH.p, 0, sizeof(long long) * slot * max_nodes, s), "hist reset");
        check(cudaMemsetAsync(D.histC.p, 0, sizeof(int) * slot * max_nodes, s), "hist reset");
        // grow_tree (cpp/src/tree.cpp:283-472)
        // Every scan launch ends with the choice of the next leaf to split, except the last.
        hist_launch(0, flag, in_timed);
        launch_split_scan(gp, hs, D.nodes.p, D.splits.p, D.st.p, 0, 0, scs, c.max_leaves > 1, s);
        for (int it = 0; it < c.max_leaves - 1; ++it) {
            launch_partition(D.codes.p, stride, D.codes_col.p, codes_col_pitch(n), rows, D.nodes.p, D.st.p,
                             D.tile_counts.p, max_tiles, s);
            hist_launch(-1, flag, in_timed);
            launch_split_scan(gp, hs, D.nodes.p, D.splits.p, D.st.p, 1, 0, scs, it < c.max_leaves - 2, s);
        }
        // post-tree sweep (booster.cpp:589-664), outputs straight into tree slot t
        double* values_t = D.values_all.p + static_cast<size_t>(t) * max_nodes;
        double* prefix_t = D.prefix_all.p + static_cast<size_t>(t) * nbk * max_nodes;
        int* cover_t = D.cover_all.p + static_cast<size_t>(t) * max_nodes;
        launch_apply_accum(D.codes_col.p, codes_col_pitch(n), D.nodes.p, D.st.p, D.g.p, h_rows, D.chunks.p,
                           static_cast<int>(chunks.size()), D.all_scale.p, D.nid.p, D.seg_sums.p, n_segments, s);
        launch_finalize_tree(pp, D.st.p, D.seg_sums.p, D.bucket_seg_end.p, D.cuts.p, D.all_scale.p, values_t,
                             cover_t, prefix_t, s);
        // prediction update, then the training loss (booster.cpp:704-706)
        if (const_h) {
            launch_pred_update_loss(pp, D.nid.p, prefix_t, D.st.p, D.pred.p, D.y.p, D.loss_part.p, 2368, s);
            launch_loss_finalize(0, D.loss_part.p, nullptr, 2368, n, D.losses.p + t, s);
        } else {
            launch_pred_update(pp, D.nid.p, prefix_t, D.st.p, D.pred.p, s);
            launch_loss_pairwise(D.y.p, D.pred.p, D.run_start.p, D.run_len.p, order_d, n_runs, D.loss_part.p,
                                 D.loss_valid.p, s);
            launch_loss_finalize(5, D.loss_part.p, D.loss_valid.p, n_runs, n, D.losses.p + t, s);
        }
        check(cudaMemcpyAsync(D.nodes_all.p + static_cast<size_t>(t) * max_nodes, D.nodes.p,
                              sizeof(DevNode) * max_nodes, cudaMemcpyDeviceToDevice, s),
              "nodes snapshot");
        check(cudaMemcpyAsync(D.st_all.p + t, D.st.p, sizeof(DevTreeState), cudaMemcpyDeviceToDevice, s),
              "state snapshot");
    }
    if (timing && timing_end == T) {
        check(cudaEventRecord(ev_end, s), "event record");
        launches_end = g_kernel_launches.load();
    }
    check(cudaStreamSynchronize(s), "tree loop");
    stats.t_trees = now() - ttree;
    if (timing) {
        float ms = 0.f;
        check(cudaEventElapsedTime(&ms, ev_begin, ev_end), "event time");
        stats.timed_ms = ms;
        stats.timed_trees = timing_end - c.timing_from;
        stats.timed_launches = launches_end - launches_begin;
        for (size_t k = 0; k + 1 < hist_ev_used; k += 2) {
            float hm = 0.f;
            check(cudaEventElapsedTime(&hm, hist_ev[k], hist_ev[k + 1]), "event time");
            stats.hist_ms += hm;
            stats.hist_launches += 1;
        }
        unsigned long long rc = 0;
        check(cudaMemcpyAsync(&rc, rows_counter.p, sizeof(rc), cudaMemcpyDeviceToHost, s), "counter");
        check(cudaStreamSynchronize(s), "counter");
        stats.hist_rows = static_cast<long long>(rc);
        cudaEventDestroy(ev_begin);
        cudaEventDestroy(ev_end);
        for (auto& e : hist_ev) cudaEventDestroy(e);
    }
    if (sampler) {
        sampler->stop();
        stats.t_producer = sampler->producer_seconds();
        sampler.reset();
    }

    // ---- read back the trees ----
    const double td = now();
    std::vector<DevNode> nodes_h(static_cast<size_t>(T) * max_nodes);
    std::vector<DevTreeState> st_h(T);
    std::vector<double> vals_h(static_cast<size_t>(T) * max_nodes), pre_h(static_cast<size_t>(T) * nbk * max_nodes);
    std::vector<int> cov_h(static_cast<size_t>(T) * max_nodes);
    evals_train.assign(T, 0.0);
    check(cudaMemcpyAsync(nodes_h.data(), D.nodes_all.p, sizeof(DevNode) * nodes_h.size(), cudaMemcpyDeviceToHost, s), "D2H");
    check(cudaMemcpyAsync(st_h.data(), D.st_all.p, sizeof(DevTreeState) * T, cudaMemcpyDeviceToHost, s), "D2H");
    check(cudaMemcpyAsync(vals_h.data(), D.values_all.p, sizeof(double) * vals_h.size(), cudaMemcpyDeviceToHost, s), "D2H");
    check(cudaMemcpyAsync(pre_h.data(), D.prefix_all.p, sizeof(double) * pre_h.size(), cudaMemcpyDeviceToHost, s), "D2H");
    check(cudaMemcpyAsync(cov_h.data(), D.cover_all.p, sizeof(int) * cov_h.size(), cudaMemcpyDeviceToHost, s), "D2H");
    check(cudaMemcpyAsync(evals_train.data(), D.losses.p, sizeof(double) * T, cudaMemcpyDeviceToHost, s), "D2H");
    int overflow = 0;
    if (use_goss && !exact_goss)
        check(cudaMemcpyAsync(&overflow, D.goss_overflow.p, sizeof(int), cudaMemcpyDeviceToHost, s), "overflow flag");
    check(cudaStreamSynchronize(s), "D2H");
    trees.assign(T, HostTree());
    for (int t = 0; t < T; ++t) {
        const int nn = st_h[t].n_nodes;
        HostTree& tr = trees[t];
        tr.nodes.resize(nn);
        for (int k = 0; k < nn; ++k) {
            const DevNode& d = nodes_h[static_cast<size_t>(t) * max_nodes + k];
            tr.nodes[k] = HostNode{d.is_leaf, d.feature, d.threshold, d.left, d.right, d.missing_left,
                                   d.count, d.depth, d.value, d.is_leaf ? 0.0 : d.gain};
        }
        tr.values.assign(vals_h.begin() + static_cast<size_t>(t) * max_nodes,
                         vals_h.begin() + static_cast<size_t>(t) * max_nodes + nn);
        tr.cover.assign(cov_h.begin() + static_cast<size_t>(t) * max_nodes,
                        cov_h.begin() + static_cast<size_t>(t) * max_nodes + nn);
        tr.prefix.assign(pre_h.begin() + static_cast<size_t>(t) * nbk * max_nodes,
                         pre_h.begin() + static_cast<size_t>(t) * nbk * max_nodes + static_cast<size_t>(nbk) * nn);
    }
    stats.t_download = now() - td;
    cfg = c;
    fitted = true;
    D.trees_flat = 0;
    stats.gpu_launches = static_cast<int>(g_kernel_launches.load() - launches0);
    // The fit's working buffers go back to the pool (ordered on the stream); a fitted model
    // keeps only its host-side trees and edges, and predict allocates what it needs.
    D.release_fit_buffers();
    stats.t_total = now() - t0;
    return overflow != 0;
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
        std::vector<int16_t> f, l, r;
        std::vector<uint8_t> th, ml;
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
                v.push_back(t.values[k]);
            }
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
        launch_bin_transform_f32(reinterpret_cast<const float*>(Xd.p), n, n_f, ed.p, ne.p, D.pcodes.p, stride, s);
        check(cudaStreamSynchronize(s), "transform");
    } else {
        std::vector<double> eh(static_cast<size_t>(n_f) * 256, INFINITY);
        for (int ff = 0; ff < n_f; ++ff)
            for (int k = 0; k < n_edges[ff]; ++k) eh[static_cast<size_t>(ff) * 256 + k] = edges[static_cast<size_t>(ff) * 256 + k];
        DBuf<double> ed;
        ed.alloc(eh.size(), s);
        check(cudaMemcpyAsync(ed.p, eh.data(), 8 * eh.size(), cudaMemcpyHostToDevice, s), "edges");
        launch_bin_transform_f64(reinterpret_cast<const double*>(Xd.p), n, n_f, ed.p, ne.p, D.pcodes.p, stride, s);
        check(cudaStreamSynchronize(s), "transform");
    }
    launch_predict_trees(D.pcodes.p, stride, n, D.t_feat.p, D.t_left.p, D.t_right.p, D.t_thr.p, D.t_ml.p, D.t_val.p,
                         D.t_off.p, static_cast<int>(trees.size()), init_score, cfg.learning_rate, D.pout.p, s);
    check(cudaMemcpyAsync(out, D.pout.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s), "predict D2H");
    check(cudaStreamSynchronize(s), "predict");
}

}  // namespace tgb
