// Host part of quantile binning: Binner::fit (cpp/src/binning.cpp:14-102) for
// numeric features with no row mask.
//
// The reference collects every non-NaN value of a feature, shuffles them with
// mt19937(seed + f * 2654435761) when there are more than bin_sample, keeps the
// first bin_sample and computes quantile edges of that sample.  Only the SET of
// kept values matters (quantile_edges sorts first), and which positions are kept
// depends only on the generator and the count, so:
//   pass 1  (row chunks in parallel)  non-NaN count per (chunk, feature)
//   draws   (features in parallel)    kept positions via shuffled_prefix, sorted
//   pass 2  (row chunks in parallel)  stream X once, copy the values whose rank
//                                     among the feature's non-NaN values is kept
//   edges   (features in parallel)    quantile_edges, same FP64 statement order
// The result is bit-identical to the reference's edges.  The device transform
// (kernels_bin.cu) then maps X to codes.
//
// binner_fit_device runs the same steps on X already in device memory: the two
// passes, the sample sort and the edge arithmetic run as kernels (kernels_binfit.cu), and
// so do the shuffle draws (kernels_shuffle.cu).  The host only turns the non-NaN counts
// into rank bases, and draws the features with fewer than 2^16 values itself.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <thread>
#include <vector>

#include "booster.h"
#include "sampling.h"
#include "tgb_internal.h"

namespace tgb {

namespace {

template <typename F>
void parallel_for(int n, int n_threads, F&& fn) {
    n_threads = std::max(1, std::min(n_threads, n));
    if (n_threads == 1) {
        for (int i = 0; i < n; ++i) fn(i);
        return;
    }
    std::vector<std::thread> th;
    std::atomic<int> next{0};
    for (int t = 0; t < n_threads; ++t)
        th.emplace_back([&] {
            for (int i = next.fetch_add(1); i < n; i = next.fetch_add(1)) fn(i);
        });
    for (auto& t : th) t.join();
}

inline bool is_nan(double v) { return !(v == v); }

// Device scratch taken from a caller's arena while it has room, else allocated (and
// freed with the Scratch).  Pieces are 256-byte aligned.
class Scratch {
public:
    Scratch(void* base, size_t bytes, cudaStream_t s)
        : base_(static_cast<unsigned char*>(base)), size_(base ? bytes : 0), s_(s) {}
    template <class T>
    T* get(size_t count) {
        const size_t bytes = (std::max<size_t>(1, count * sizeof(T)) + 255) / 256 * 256;
        if (used_ + bytes <= size_) {
            T* p = reinterpret_cast<T*>(base_ + used_);
            used_ += bytes;
            return p;
        }
        owned_.push_back(std::make_unique<DBuf<unsigned char>>());
        owned_.back()->alloc(bytes, s_);
        return reinterpret_cast<T*>(owned_.back()->p);
    }

private:
    unsigned char* base_;
    size_t size_;
    size_t used_ = 0;
    cudaStream_t s_;
    std::vector<std::unique_ptr<DBuf<unsigned char>>> owned_;
};

double wall_now() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

template <typename T>
inline double at(const void* X, size_t k) {
    return static_cast<double>(static_cast<const T*>(X)[k]);
}

// cpp/src/binning.cpp:14-32
std::vector<double> quantile_edges(std::vector<double>& vals, int n_bins) {
    std::sort(vals.begin(), vals.end());
    vals.erase(std::unique(vals.begin(), vals.end()), vals.end());
    if (vals.empty()) return {0.0};
    if (static_cast<int>(vals.size()) <= n_bins) return vals;
    std::vector<double> e;
    e.reserve(n_bins - 1);
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

// fids: the reference feature index of each column of X (its generator seed), nullptr for
// columns 0 .. n_f - 1.
template <typename T>
int binner_fit_t(const void* X, int n, int n_f, int max_bin, int bin_sample, uint32_t seed,
                 std::vector<double>& edges, std::vector<int>& n_edges, int n_threads, const int* fids = nullptr) {
    const int n_chunks = std::max(1, std::min(n_threads * 4, (n + 65535) / 65536));
    std::vector<int64_t> bounds(n_chunks + 1);
    for (int c = 0; c <= n_chunks; ++c) bounds[c] = static_cast<int64_t>(n) * c / n_chunks;
    // pass 1: counts[c][f]
    std::vector<int64_t> counts(static_cast<size_t>(n_chunks) * n_f, 0);
    parallel_for(n_chunks, n_threads, [&](int c) {
        int64_t* cnt = counts.data() + static_cast<size_t>(c) * n_f;
        for (int64_t i = bounds[c]; i < bounds[c + 1]; ++i) {
            const size_t row = static_cast<size_t>(i) * n_f;
            for (int f = 0; f < n_f; ++f) cnt[f] += is_nan(at<T>(X, row + f)) ? 0 : 1;
        }
    });
    // kept positions per feature (sorted), or "all" when no sampling happens; slot[f][i] is
    // the shuffled position of the i-th smallest kept position
    std::vector<std::vector<int32_t>> keep(n_f), slot(n_f);
    std::vector<char> take_all(n_f, 0);
    std::vector<int64_t> m(n_f, 0);
    for (int c = 0; c < n_chunks; ++c)
        for (int f = 0; f < n_f; ++f) m[f] += counts[static_cast<size_t>(c) * n_f + f];
    parallel_for(n_f, n_threads, [&](int f) {
        if (bin_sample > 0 && m[f] > bin_sample) {
            Mt32 rng(seed + static_cast<uint32_t>(fids ? fids[f] : f) * 2654435761u);  // std::mt19937's stream
            std::vector<int32_t> prefix(static_cast<size_t>(bin_sample));
            shuffled_prefix(m[f], bin_sample, rng, prefix.data());
            std::vector<uint64_t> key(prefix.size());  // (position, shuffled slot), positions distinct
            for (size_t j = 0; j < prefix.size(); ++j)
                key[j] = (static_cast<uint64_t>(static_cast<uint32_t>(prefix[j])) << 32) | j;
            std::sort(key.begin(), key.end());
            keep[f].resize(key.size());
            slot[f].resize(key.size());
            for (size_t i = 0; i < key.size(); ++i) {
                keep[f][i] = static_cast<int32_t>(key[i] >> 32);
                slot[f][i] = static_cast<int32_t>(static_cast<uint32_t>(key[i]));
            }
        } else {
            take_all[f] = 1;
        }
    });
    std::vector<std::vector<double>> sample(n_f);
    for (int f = 0; f < n_f; ++f) sample[f].resize(take_all[f] ? m[f] : keep[f].size());
    // pass 2: per chunk, the rank range of each feature is known from the counts
    parallel_for(n_chunks, n_threads, [&](int c) {
        std::vector<int64_t> rank(n_f, 0), ptr(n_f, 0), end(n_f, 0);
        for (int f = 0; f < n_f; ++f) {
            int64_t r0 = 0;
            for (int cc = 0; cc < c; ++cc) r0 += counts[static_cast<size_t>(cc) * n_f + f];
            rank[f] = r0;
            const int64_t r1 = r0 + counts[static_cast<size_t>(c) * n_f + f];
            if (take_all[f]) {
                ptr[f] = r0;
                end[f] = r1;
            } else {
                const auto& k = keep[f];
                ptr[f] = std::lower_bound(k.begin(), k.end(), static_cast<int32_t>(std::min<int64_t>(r0, INT32_MAX))) -
                         k.begin();
                end[f] = std::lower_bound(k.begin(), k.end(), static_cast<int32_t>(std::min<int64_t>(r1, INT32_MAX))) -
                         k.begin();
            }
        }
        for (int64_t i = bounds[c]; i < bounds[c + 1]; ++i) {
            const size_t row = static_cast<size_t>(i) * n_f;
            for (int f = 0; f < n_f; ++f) {
                const double v = at<T>(X, row + f);
                if (is_nan(v)) continue;
                if (take_all[f]) {
                    sample[f][rank[f]] = v;
                } else if (ptr[f] < end[f] && keep[f][ptr[f]] == rank[f]) {
                    sample[f][ptr[f]] = v;
                    ++ptr[f];
                }
                ++rank[f];
            }
        }
    });
    // The reference sorts the kept values in their shuffled order (binning.cpp:93-98).  Equal
    // values stay where std::sort leaves them, which depends on that order; of equal doubles
    // only -0.0 and +0.0 differ in their bits, and the sign of a zero edge follows from it.
    parallel_for(n_f, n_threads, [&](int f) {
        if (take_all[f]) return;
        std::vector<double> shuffled(sample[f].size());
        for (size_t i = 0; i < shuffled.size(); ++i) shuffled[static_cast<size_t>(slot[f][i])] = sample[f][i];
        sample[f].swap(shuffled);
    });
    edges.assign(static_cast<size_t>(n_f) * 256, 0.0);
    n_edges.assign(n_f, 0);
    std::vector<int> nbc(n_f, 2);
    parallel_for(n_f, n_threads, [&](int f) {
        std::vector<double> e = quantile_edges(sample[f], max_bin - 1);
        n_edges[f] = static_cast<int>(e.size());
        std::memcpy(edges.data() + static_cast<size_t>(f) * 256, e.data(), e.size() * sizeof(double));
        nbc[f] = static_cast<int>(e.size()) + 2;
    });
    int mx = 2;
    for (int v : nbc) mx = std::max(mx, v);
    return std::max(mx, max_bin);  // Binner::max_bins, binning.cpp:130-134
}

}  // namespace

bool binner_fits_device(int n, int n_f, int bin_sample) {
    const long long cap = bin_sample > 0 ? std::min<long long>(bin_sample, n) : n;
    return static_cast<long long>(n_f) * std::max(1LL, cap) < (1LL << 31) - 1;
}

void binner_plan(const std::vector<int>& ch, int n, int n_f, int bin_sample, uint32_t seed, int n_threads,
                 BinPlan& plan) {
    const int n_chunks = (n + kFitChunk - 1) / kFitChunk;
    const size_t nc = static_cast<size_t>(n_chunks) * n_f;
    plan.n_chunks = n_chunks;
    // per-feature totals and the first non-NaN rank of every (chunk, feature)
    plan.m.assign(n_f, 0);
    plan.base.assign(nc, 0);
    for (int c = 0; c < n_chunks; ++c)
        for (int f = 0; f < n_f; ++f) {
            plan.base[static_cast<size_t>(c) * n_f + f] = plan.m[f];
            plan.m[f] += ch[static_cast<size_t>(c) * n_f + f];
        }
    plan.take_all.assign(n_f, 1);
    plan.kept.assign(n_f, 0);
    plan.max_sampled = 0;
    plan.cap = 1;
    for (int f = 0; f < n_f; ++f) {
        plan.take_all[f] = (bin_sample > 0 && plan.m[f] > bin_sample) ? 0 : 1;
        plan.kept[f] = plan.take_all[f] ? static_cast<int>(plan.m[f]) : bin_sample;
        if (!plan.take_all[f]) plan.max_sampled = std::max(plan.max_sampled, plan.m[f]);
        plan.cap = std::max<long long>(plan.cap, plan.kept[f]);
    }
    // kept ranks: the exact prefix of std::shuffle(mt19937(seed + f * 2654435761)), binning.cpp:93-97.
    // Features with at least 2^16 values are drawn on the device (kernels_shuffle.cu);
    // libstdc++'s two-draws path for shorter ranges runs here.
    plan.seed = seed;
    plan.host_f.clear();
    plan.keep.clear();
    for (int f = 0; f < n_f; ++f)
        if (!plan.take_all[f] && shuffle_pairs(plan.m[f])) plan.host_f.push_back(f);
    plan.keep.resize(plan.host_f.size() * static_cast<size_t>(bin_sample));
    parallel_for(static_cast<int>(plan.host_f.size()), n_threads, [&](int k) {
        const int f = plan.host_f[k];
        Mt32 rng(seed + static_cast<uint32_t>(f) * 2654435761u);
        shuffled_prefix(plan.m[f], bin_sample, rng, plan.keep.data() + static_cast<size_t>(k) * bin_sample);
    });
}

int binner_fit_from_plan(const BinPlan& plan, const void* Xd, int x_dtype, int n, int n_f, int max_bin,
                         int bin_sample, std::vector<double>& edges, std::vector<int>& n_edges, void* stream,
                         void* arena, size_t arena_bytes, std::vector<int>* flagged) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    Scratch scratch(arena, arena_bytes, s);
    const size_t nc = static_cast<size_t>(plan.n_chunks) * n_f;
    const std::vector<long long>& base = plan.base;
    const std::vector<uint8_t>& take_all = plan.take_all;
    const std::vector<int>& kept = plan.kept;
    const int64_t max_sampled = plan.max_sampled;
    const long long cap = plan.cap;
    long long* base_d = scratch.get<long long>(nc);
    check(cudaMemcpyAsync(base_d, base.data(), sizeof(long long) * nc, cudaMemcpyHostToDevice, s), "bases upload");
    uint8_t* take_d = scratch.get<uint8_t>(n_f);
    check(cudaMemcpyAsync(take_d, take_all.data(), n_f, cudaMemcpyHostToDevice, s), "flags upload");
    const long long words = max_sampled > 0 ? (max_sampled + 31) / 32 : 1;
    uint32_t* bits = scratch.get<uint32_t>(static_cast<size_t>(n_f) * words);
    int* err_d = scratch.get<int>(1);
    check(cudaMemsetAsync(err_d, 0, sizeof(int), s), "error flag reset");
    const size_t esz = x_dtype == 0 ? sizeof(float) : sizeof(double);
    const long long total = static_cast<long long>(n_f) * cap;
    unsigned char* smp_a = scratch.get<unsigned char>(static_cast<size_t>(total) * esz);
    unsigned char* smp_b = scratch.get<unsigned char>(static_cast<size_t>(total) * esz);
    if (max_sampled > 0) {
        check(cudaMemsetAsync(bits, 0, sizeof(uint32_t) * static_cast<size_t>(n_f) * words, s), "bits reset");
        // kept ranks: device draws, with the sample buffers (n_f * cap >= n_f * bin_sample
        // elements of >= 4 bytes, free until the gather) as the draws' scratch
        const size_t nk = static_cast<size_t>(n_f) * bin_sample;
        int32_t* keep_d = scratch.get<int32_t>(nk);
        int32_t* cnt_d = scratch.get<int32_t>(nk + n_f);
        std::vector<long long> ms(n_f, 0);
        std::vector<uint32_t> seeds(n_f);
        for (int f = 0; f < n_f; ++f) {
            seeds[f] = plan.seed + static_cast<uint32_t>(f) * 2654435761u;
            if (!take_all[f] && !shuffle_pairs(plan.m[f])) ms[f] = plan.m[f];
        }
        long long* ms_d = scratch.get<long long>(n_f);
        uint32_t* seeds_d = scratch.get<uint32_t>(n_f);
        check(cudaMemcpyAsync(ms_d, ms.data(), sizeof(long long) * n_f, cudaMemcpyHostToDevice, s), "sizes upload");
        check(cudaMemcpyAsync(seeds_d, seeds.data(), sizeof(uint32_t) * n_f, cudaMemcpyHostToDevice, s),
              "seeds upload");
        launch_shuffle_prefix(seeds_d, ms_d, n_f, bin_sample, keep_d, reinterpret_cast<int32_t*>(smp_a), cnt_d,
                              reinterpret_cast<int32_t*>(smp_b), err_d, s);
        for (size_t k = 0; k < plan.host_f.size(); ++k)
            check(cudaMemcpyAsync(keep_d + static_cast<size_t>(plan.host_f[k]) * bin_sample,
                                  plan.keep.data() + k * bin_sample, sizeof(int32_t) * bin_sample,
                                  cudaMemcpyHostToDevice, s),
                  "kept ranks upload");
        launch_keep_bits(keep_d, bin_sample, n_f, take_d, bits, words, s);
    }
    int* fill = scratch.get<int>(n_f);
    long long* m_d = scratch.get<long long>(n_f);
    check(cudaMemcpyAsync(m_d, plan.m.data(), sizeof(long long) * n_f, cudaMemcpyHostToDevice, s), "totals upload");
    int* kc_d = scratch.get<int>(nc);
    int* kbase_d = scratch.get<int>(nc);
    launch_sample_gather(Xd, x_dtype, n, n_f, base_d, m_d, bits, words, take_d, smp_a, cap, kc_d, kbase_d, fill, s);
    std::vector<int> seg(2 * static_cast<size_t>(n_f));
    for (int f = 0; f < n_f; ++f) {
        seg[f] = static_cast<int>(f * cap);
        seg[n_f + f] = static_cast<int>(f * cap + kept[f]);
    }
    int* seg_d = scratch.get<int>(seg.size());
    int* kept_d = scratch.get<int>(n_f);
    check(cudaMemcpyAsync(seg_d, seg.data(), sizeof(int) * seg.size(), cudaMemcpyHostToDevice, s), "segs upload");
    check(cudaMemcpyAsync(kept_d, kept.data(), sizeof(int) * n_f, cudaMemcpyHostToDevice, s), "kept upload");
    const size_t tmp_bytes = sample_sort_bytes(x_dtype, total, n_f);
    unsigned char* tmp = scratch.get<unsigned char>(std::max<size_t>(tmp_bytes, 16));
    launch_sample_sort(x_dtype, smp_a, smp_b, total, n_f, seg_d, seg_d + n_f, tmp, tmp_bytes, s);
    double* ed = scratch.get<double>(static_cast<size_t>(n_f) * 256);
    int* ne = scratch.get<int>(n_f);
    check(cudaMemsetAsync(ed, 0, sizeof(double) * static_cast<size_t>(n_f) * 256, s), "edges reset");
    int* flags_d = scratch.get<int>(n_f);
    launch_quantile_edges(x_dtype, smp_b, smp_a, cap, kept_d, n_f, max_bin - 1, ed, ne, flags_d, s);
    edges.assign(static_cast<size_t>(n_f) * 256, 0.0);
    n_edges.assign(n_f, 0);
    std::vector<int> fill_h(n_f), flags_h(n_f, 0);
    check(cudaMemcpyAsync(flags_h.data(), flags_d, sizeof(int) * n_f, cudaMemcpyDeviceToHost, s), "flags download");
    int err_h = 0;
    check(cudaMemcpyAsync(edges.data(), ed, sizeof(double) * edges.size(), cudaMemcpyDeviceToHost, s),
          "edges download");
    check(cudaMemcpyAsync(n_edges.data(), ne, sizeof(int) * n_f, cudaMemcpyDeviceToHost, s), "edges download");
    check(cudaMemcpyAsync(fill_h.data(), fill, sizeof(int) * n_f, cudaMemcpyDeviceToHost, s), "fill download");
    check(cudaMemcpyAsync(&err_h, err_d, sizeof(int), cudaMemcpyDeviceToHost, s), "error flag download");
    check(cudaStreamSynchronize(s), "quantile edges");
    if (err_h) throw TideError("device binner: shuffle draws ran past their refill limit");
    for (int f = 0; f < n_f; ++f)
        if (fill_h[f] != kept[f]) throw TideError("device binner: sample size mismatch");
    if (flagged) {
        flagged->clear();
        for (int f = 0; f < n_f; ++f)
            if (flags_h[f]) flagged->push_back(f);
    }
    int mx = 2;
    for (int f = 0; f < n_f; ++f) mx = std::max(mx, n_edges[f] + 2);
    return std::max(mx, max_bin);  // Binner::max_bins, binning.cpp:130-134
}

// Edges of the listed features recomputed on the host from their columns, in the
// reference's order (the kept sample in its shuffled order, std::sort, std::unique):
// the features whose edges depend on how std::sort places equal values.  X_host: the
// row-major X on the host, or nullptr to copy the columns from Xd.
void binner_refit_features(const std::vector<int>& fids, const void* X_host, const void* Xd, int x_dtype, int n,
                           int n_f, int max_bin, int bin_sample, uint32_t seed, std::vector<double>& edges,
                           std::vector<int>& n_edges, int n_threads, cudaStream_t s) {
    if (fids.empty()) return;
    const int k = static_cast<int>(fids.size());
    const size_t xsz = x_dtype == 0 ? 4 : 8;
    std::vector<unsigned char> cols(static_cast<size_t>(n) * k * xsz);
    if (X_host) {
        parallel_for(k, n_threads, [&](int j) {
            const unsigned char* src = static_cast<const unsigned char*>(X_host) + static_cast<size_t>(fids[j]) * xsz;
            for (int i = 0; i < n; ++i)
                std::memcpy(cols.data() + (static_cast<size_t>(i) * k + j) * xsz, src + static_cast<size_t>(i) * n_f * xsz,
                            xsz);
        });
    } else {
        for (int j = 0; j < k; ++j)
            check(cudaMemcpy2DAsync(cols.data() + j * xsz, k * xsz,
                                    static_cast<const unsigned char*>(Xd) + static_cast<size_t>(fids[j]) * xsz,
                                    static_cast<size_t>(n_f) * xsz, xsz, n, cudaMemcpyDeviceToHost, s),
                  "column download");
        check(cudaStreamSynchronize(s), "column download");
    }
    std::vector<double> e;
    std::vector<int> ne;
    if (x_dtype == 0) binner_fit_t<float>(cols.data(), n, k, max_bin, bin_sample, seed, e, ne, n_threads, fids.data());
    else binner_fit_t<double>(cols.data(), n, k, max_bin, bin_sample, seed, e, ne, n_threads, fids.data());
    for (int j = 0; j < k; ++j) {
        const int f = fids[j];
        std::fill(edges.begin() + static_cast<size_t>(f) * 256, edges.begin() + static_cast<size_t>(f + 1) * 256, 0.0);
        std::copy(e.begin() + static_cast<size_t>(j) * 256, e.begin() + static_cast<size_t>(j) * 256 + ne[j],
                  edges.begin() + static_cast<size_t>(f) * 256);
        n_edges[f] = ne[j];
    }
}

int binner_fit_device(const void* Xd, int x_dtype, int n, int n_f, int max_bin, int bin_sample, uint32_t seed,
                      std::vector<double>& edges, std::vector<int>& n_edges, int n_threads, void* stream,
                      void* arena, size_t arena_bytes, BinFitTimes* tm, const void* X_host) {
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const double t0 = wall_now();
    const int n_chunks = (n + kFitChunk - 1) / kFitChunk;
    const size_t nc = static_cast<size_t>(n_chunks) * n_f;
    std::vector<int> ch(nc);
    {
        DBuf<int> counts;
        counts.alloc(nc, s);
        launch_nonnan_counts(Xd, x_dtype, n, n_f, counts.p, s);
        check(cudaMemcpyAsync(ch.data(), counts.p, sizeof(int) * nc, cudaMemcpyDeviceToHost, s), "counts download");
        check(cudaStreamSynchronize(s), "non-NaN counts");
    }
    const double t1 = wall_now();
    BinPlan plan;
    binner_plan(ch, n, n_f, bin_sample, seed, n_threads, plan);
    const double t2 = wall_now();
    std::vector<int> flagged;
    int nb = binner_fit_from_plan(plan, Xd, x_dtype, n, n_f, max_bin, bin_sample, edges, n_edges, stream, arena,
                                  arena_bytes, &flagged);
    if (!flagged.empty()) {
        binner_refit_features(flagged, X_host, Xd, x_dtype, n, n_f, max_bin, bin_sample, seed, edges, n_edges,
                              n_threads, s);
        int mx = 2;
        for (int f = 0; f < n_f; ++f) mx = std::max(mx, n_edges[f] + 2);
        nb = std::max(mx, max_bin);  // Binner::max_bins, binning.cpp:130-134
    }
    if (tm) {
        tm->refit_features = static_cast<int>(flagged.size());
        tm->counts = t1 - t0;
        tm->draws = t2 - t1;
        tm->edges = wall_now() - t2;
    }
    return nb;
}

namespace {

// The vocabulary of one categorical feature (cpp/src/binning.cpp:47-84): the distinct
// non-NaN values with at least cat_min_count occurrences (none: the most frequent one,
// the smallest value on ties), cut to the max_bin - 1 most frequent ones when there are
// more (std::partial_sort, so ties fall as in the reference), ascending.
template <typename T>
std::vector<double> cat_vocabulary(const T* X, int n, int n_f, int f, int max_bin, int cat_min_count) {
    std::vector<double> v;
    v.reserve(static_cast<size_t>(n));
    for (int i = 0; i < n; ++i) {
        const double x = static_cast<double>(X[static_cast<size_t>(i) * n_f + f]);
        if (!is_nan(x)) v.push_back(x);
    }
    std::sort(v.begin(), v.end());
    std::vector<std::pair<int, double>> runs;  // (occurrences, value), ascending values
    for (size_t a = 0; a < v.size();) {
        size_t b = a + 1;
        while (b < v.size() && v[b] == v[a]) ++b;
        runs.emplace_back(static_cast<int>(b - a), v[a]);
        a = b;
    }
    const int min_count = std::max(1, cat_min_count);
    std::vector<std::pair<int, double>> kept;
    for (const auto& r : runs)
        if (r.first >= min_count) kept.push_back(r);
    if (kept.empty() && !runs.empty())
        kept.push_back(*std::max_element(runs.begin(), runs.end(),
                                         [](const auto& a, const auto& b) { return a.first < b.first; }));
    const int cap = max_bin - 1;
    if (static_cast<int>(kept.size()) > cap) {
        std::partial_sort(kept.begin(), kept.begin() + cap, kept.end(),
                          [](const auto& a, const auto& b) { return a.first > b.first; });
        kept.resize(static_cast<size_t>(cap));
    }
    std::vector<double> vocab;
    vocab.reserve(kept.size());
    for (const auto& r : kept) vocab.push_back(r.second);
    std::sort(vocab.begin(), vocab.end());
    return vocab;
}

}  // namespace

int binner_fit_cat(const void* X, int x_dtype, int n, int n_f, const int* is_cat, int max_bin, int cat_min_count,
                   int bin_sample, uint32_t seed, std::vector<double>& edges, std::vector<int>& n_edges,
                   int n_threads) {
    binner_fit(X, x_dtype, n, n_f, max_bin, bin_sample, seed, edges, n_edges, n_threads);
    parallel_for(n_f, n_threads, [&](int f) {
        if (!is_cat[f]) return;
        const std::vector<double> vocab =
            x_dtype == 0 ? cat_vocabulary(static_cast<const float*>(X), n, n_f, f, max_bin, cat_min_count)
                         : cat_vocabulary(static_cast<const double*>(X), n, n_f, f, max_bin, cat_min_count);
        double* e = edges.data() + static_cast<size_t>(f) * 256;
        std::fill(e, e + 256, 0.0);
        std::copy(vocab.begin(), vocab.end(), e);
        n_edges[f] = static_cast<int>(vocab.size());
    });
    int mx = 2;  // Binner::max_bins (binning.cpp:130-134): vocabulary + missing, or edges + 2
    for (int f = 0; f < n_f; ++f) mx = std::max(mx, n_edges[f] + (is_cat[f] ? 1 : 2));
    return std::max(mx, max_bin);
}

int binner_fit(const void* X, int x_dtype, int n, int n_f, int max_bin, int bin_sample, uint32_t seed,
               std::vector<double>& edges, std::vector<int>& n_edges, int n_threads) {
    if (x_dtype == 0) return binner_fit_t<float>(X, n, n_f, max_bin, bin_sample, seed, edges, n_edges, n_threads);
    return binner_fit_t<double>(X, n, n_f, max_bin, bin_sample, seed, edges, n_edges, n_threads);
}

}  // namespace tgb
