// Exact prefixes of libstdc++'s std::shuffle without shuffling.
//
// TideGBM draws two random samples with std::mt19937 + std::shuffle and keeps only a
// prefix of the shuffled range: the per-feature quantile sample (cpp/src/binning.cpp:
// 93-97, bin_sample = 262,144 of ~n values) and the GOSS remainder (cpp/src/booster.cpp:
// 569-578, ceil(0.1 n) of ~0.8 n rows).  The positions that land in the prefix depend
// only on the generator state and the range length, not on the values.
//
// For ranges of at least 2^16 elements libstdc++'s shuffle draws one
// uniform_int_distribution<unsigned long> value in [0, i] per i = 1 .. m-1 and swaps
// a[i] with a[j].  Position i is untouched before step i, so a[i] still holds element
// i when it is swapped; positions >= keep never move an element back below keep.
// Tracking only the first `keep` slots therefore gives the same prefix with the same
// draws: O(keep) memory instead of O(m), and no value traffic.  Shorter ranges take
// libstdc++'s two-draws-per-call path, so they call std::shuffle itself on an index
// range.  The generator is left in exactly the state std::shuffle leaves it.
#pragma once

#include <algorithm>
#include <cstdint>
#include <numeric>
#include <random>
#include <vector>

namespace tgb {

// out[p] = index (in [0, m)) of the element that std::shuffle puts at position p, p < keep.
inline void shuffled_prefix(int64_t m, int64_t keep, std::mt19937& rng, int32_t* out) {
    if (m <= 0) return;  // std::shuffle of an empty range draws nothing
    keep = std::max<int64_t>(0, std::min(keep, m));
    const unsigned long urngrange = static_cast<unsigned long>(rng.max() - rng.min());
    const unsigned long urange = static_cast<unsigned long>(m);
    if (urngrange / urange >= urange) {
        // libstdc++ pairs two swap positions per generator call here: run it for real.
        std::vector<int32_t> v(static_cast<size_t>(m));
        std::iota(v.begin(), v.end(), 0);
        std::shuffle(v.begin(), v.end(), rng);
        std::copy(v.begin(), v.begin() + keep, out);
        return;
    }
    std::iota(out, out + keep, 0);
    std::uniform_int_distribution<unsigned long> d;
    using P = std::uniform_int_distribution<unsigned long>::param_type;
    for (int64_t i = 1; i < m; ++i) {
        const unsigned long j = d(rng, P(0, static_cast<unsigned long>(i)));
        if (i < keep) {
            std::swap(out[i], out[j]);
        } else if (static_cast<int64_t>(j) < keep) {
            out[j] = static_cast<int32_t>(i);
        }
    }
}

}  // namespace tgb
