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
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

#include "booster.h"
#include "sampling.h"

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

template <typename T>
int binner_fit_t(const void* X, int n, int n_f, int max_bin, int bin_sample, uint32_t seed,
                 std::vector<double>& edges, std::vector<int>& n_edges, int n_threads) {
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
    // kept positions per feature (sorted), or "all" when no sampling happens
    std::vector<std::vector<int32_t>> keep(n_f);
    std::vector<char> take_all(n_f, 0);
    std::vector<int64_t> m(n_f, 0);
    for (int c = 0; c < n_chunks; ++c)
        for (int f = 0; f < n_f; ++f) m[f] += counts[static_cast<size_t>(c) * n_f + f];
    parallel_for(n_f, n_threads, [&](int f) {
        if (bin_sample > 0 && m[f] > bin_sample) {
            Mt32 rng(seed + static_cast<uint32_t>(f) * 2654435761u);  // std::mt19937's stream
            keep[f].resize(static_cast<size_t>(bin_sample));
            shuffled_prefix(m[f], bin_sample, rng, keep[f].data());
            std::sort(keep[f].begin(), keep[f].end());
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

int binner_fit(const void* X, int x_dtype, int n, int n_f, int max_bin, int bin_sample, uint32_t seed,
               std::vector<double>& edges, std::vector<int>& n_edges, int n_threads) {
    if (x_dtype == 0) return binner_fit_t<float>(X, n, n_f, max_bin, bin_sample, seed, edges, n_edges, n_threads);
    return binner_fit_t<double>(X, n, n_f, max_bin, bin_sample, seed, edges, n_edges, n_threads);
}

}  // namespace tgb
