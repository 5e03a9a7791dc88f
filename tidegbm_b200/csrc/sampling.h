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
//
// Mt32 is MT19937 (Matsumoto & Nishimura, ACM TOMACS 8(1), 1998) on 32-bit words,
// generating a block of 624 outputs per refill: the same output stream as
// std::mt19937, at a fraction of libstdc++'s per-call cost.  bounded() is Lemire's
// nearly divisionless method (ACM TOMACS 29(1), 2019, arXiv:1805.10941), the
// algorithm libstdc++'s uniform_int_distribution uses for 32-bit generators; both are
// checked against the standard library by the tests.
#pragma once

#include <algorithm>
#include <cstdint>
#if defined(__x86_64__) && defined(__GNUC__) && !defined(__clang__) && !defined(__CUDACC__)
#include <immintrin.h>
#endif
#include <numeric>
#include <random>
#include <vector>

namespace tgb {

// One MT19937 block: twist the 624-word state in place, write the 624 tempered
// outputs.  Compiled for several x86 vector ISAs and picked at load time (the three
// loops carry no dependence shorter than 227 words, so they vectorise).
inline uint32_t mt_temper(uint32_t v) {
    v ^= v >> 11;
    v ^= (v << 7) & 0x9d2c5680u;
    v ^= (v << 15) & 0xefc60000u;
    v ^= v >> 18;
    return v;
}

#if defined(__x86_64__) && defined(__GNUC__) && !defined(__clang__) && !defined(__CUDACC__)
__attribute__((target_clones("avx512f", "avx2", "default")))
#endif
inline void mt_refill(uint32_t* __restrict__ st, uint32_t* __restrict__ out) {
    constexpr uint32_t UM = 0x80000000u, LM = 0x7fffffffu, A = 0x9908b0dfu;
    for (int k = 0; k < 227; ++k) {
        const uint32_t y = (st[k] & UM) | (st[k + 1] & LM);
        const uint32_t v = st[k + 397] ^ (y >> 1) ^ ((0u - (y & 1u)) & A);
        st[k] = v;
        out[k] = mt_temper(v);
    }
    for (int k = 227; k < 623; ++k) {
        const uint32_t y = (st[k] & UM) | (st[k + 1] & LM);
        const uint32_t v = st[k - 227] ^ (y >> 1) ^ ((0u - (y & 1u)) & A);
        st[k] = v;
        out[k] = mt_temper(v);
    }
    {
        const uint32_t y = (st[623] & UM) | (st[0] & LM);
        st[623] = st[396] ^ (y >> 1) ^ ((0u - (y & 1u)) & A);
        out[623] = mt_temper(st[623]);
    }
}

struct Mt32 {
    using result_type = uint32_t;
    static constexpr result_type min() { return 0u; }
    static constexpr result_type max() { return 0xffffffffu; }

    uint32_t st[624];
    uint32_t out[624];
    int pos = 624;

    explicit Mt32(uint32_t seed = 5489u) {
        st[0] = seed;
        for (uint32_t i = 1; i < 624; ++i) st[i] = 1812433253u * (st[i - 1] ^ (st[i - 1] >> 30)) + i;
        pos = 624;
    }

    void refill() {
        mt_refill(st, out);
        pos = 0;
    }

    result_type operator()() {
        if (pos >= 624) refill();
        return out[pos++];
    }
};

// Uniform draw in [0, range), range in [1, 2^32): Lemire's method.
template <class G>
inline uint32_t bounded(G& g, uint32_t range) {
    uint64_t m = static_cast<uint64_t>(g()) * range;
    uint32_t low = static_cast<uint32_t>(m);
    if (low < range) {
        const uint32_t t = (0u - range) % range;
        while (low < t) {
            m = static_cast<uint64_t>(g()) * range;
            low = static_cast<uint32_t>(m);
        }
    }
    return static_cast<uint32_t>(m >> 32);
}

// True when libstdc++'s std::shuffle takes its two-positions-per-draw path for a
// range of m elements with a 32-bit generator.
inline bool shuffle_pairs(int64_t m) {
    const unsigned long urngrange = 0xffffffffUL;
    return m > 0 && urngrange / static_cast<unsigned long>(m) >= static_cast<unsigned long>(m);
}

#if defined(__x86_64__) && defined(__GNUC__) && !defined(__clang__) && !defined(__CUDACC__)
#define TGB_HAVE_AVX512_TAIL 1
// Groups of 16 consecutive draws of the tail with AVX-512: the 32x32->64 Lemire products
// of the 16 words, a stop at the first group holding a word whose low half is below its
// range (it goes to the exact path), and a masked scatter of out[j] = i for the draws
// that land in the prefix.  Scatter writes to one address keep the highest lane, i.e.
// the latest draw, as the sequential loop does.  Returns the number of words consumed.
__attribute__((target("avx512f"))) inline int tail_groups_avx512(const uint32_t* w, int64_t i, int k, uint32_t K,
                                                                  int32_t* out) {
    const __m512i lane = _mm512_setr_epi32(0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15);
    const __m512i vK = _mm512_set1_epi32(static_cast<int>(K));
    int l = 0;
    while (l + 16 <= k) {
        const __m512i W = _mm512_loadu_si512(w + l);
        const __m512i R = _mm512_add_epi32(_mm512_set1_epi32(static_cast<int>(i + l + 1)), lane);
        const __m512i pe = _mm512_mul_epu32(W, R);
        const __m512i po = _mm512_mul_epu32(_mm512_srli_epi64(W, 32), _mm512_srli_epi64(R, 32));
        const __m512i lo = _mm512_mask_blend_epi32(0xAAAA, pe, _mm512_slli_epi64(po, 32));
        if (_mm512_cmplt_epu32_mask(lo, R)) break;
        const __m512i hi = _mm512_mask_blend_epi32(0xAAAA, _mm512_srli_epi64(pe, 32), po);
        const __mmask16 hit = _mm512_cmplt_epu32_mask(hi, vK);
        const __m512i I = _mm512_add_epi32(_mm512_set1_epi32(static_cast<int>(i + l)), lane);
        _mm512_mask_i32scatter_epi32(out, hit, hi, I, 4);
        l += 16;
    }
    return l;
}

inline bool have_avx512() {
    static const bool ok = __builtin_cpu_supports("avx512f");
    return ok;
}
#endif

// The draws i in [i, m) of a shuffle whose first `keep` positions are tracked in out
// (which has room for keep + 1 entries: out[keep] absorbs the draws that land outside
// the prefix, so the store is branch-free).  A word whose Lemire product has low half
// >= its range is accepted as is; the first word of a 16-word group that fails that
// test sends the group to the exact bounded() path.
inline void shuffle_tail(int64_t i, int64_t m, int64_t keep, Mt32& rng, int32_t* out) {
    const uint32_t K = static_cast<uint32_t>(keep);
    while (i < m) {
        if (rng.pos >= 624) rng.refill();
        const uint32_t* w = rng.out + rng.pos;
        const int k = static_cast<int>(std::min<int64_t>(624 - rng.pos, m - i));
        int l = 0;
#ifdef TGB_HAVE_AVX512_TAIL
        if (have_avx512()) l = tail_groups_avx512(w, i, k, K, out);
#endif
        while (l + 16 <= k) {
            const uint32_t r0 = static_cast<uint32_t>(i + l + 1);
            uint32_t bad = 0;
            for (int q = 0; q < 16; ++q) bad |= static_cast<uint32_t>(w[l + q] * (r0 + q) < r0 + q);
            if (bad) break;
            for (int q = 0; q < 16; ++q) {
                const uint32_t j = static_cast<uint32_t>((static_cast<uint64_t>(w[l + q]) * (r0 + q)) >> 32);
                out[j < K ? j : K] = static_cast<int32_t>(i + l + q);
            }
            l += 16;
        }
        for (; l < k; ++l) {
            const uint32_t r = static_cast<uint32_t>(i + l + 1);
            const uint64_t p = static_cast<uint64_t>(w[l]) * r;
            if (static_cast<uint32_t>(p) < r) break;
            const uint32_t j = static_cast<uint32_t>(p >> 32);
            out[j < K ? j : K] = static_cast<int32_t>(i + l);
        }
        rng.pos += l;
        i += l;
        if (l < k) {  // a word that may be rejected: the exact draw (it can consume more words)
            const uint32_t j = bounded(rng, static_cast<uint32_t>(i + 1));
            if (j < K) out[j] = static_cast<int32_t>(i);
            ++i;
        }
    }
}

template <class G>
inline void shuffle_tail(int64_t i, int64_t m, int64_t keep, G& rng, int32_t* out) {
    for (; i < m; ++i) {
        const uint32_t j = bounded(rng, static_cast<uint32_t>(i + 1));
        if (static_cast<int64_t>(j) < keep) out[j] = static_cast<int32_t>(i);
    }
}

// The draws of std::shuffle(iota(m), rng) that land inside the prefix: the first
// `keep` (0 <= keep <= m) of them, i = 1 .. keep-1, swap within the prefix and are
// made here; out[0..keep) then holds the prefix as it stands before draw i, where i
// is the return value.  The remaining draws i .. m-1 (the tail) only overwrite prefix
// slots: out[j] = i for each draw j < keep.  Returns m when no tail is left (the
// two-draws-per-call path of short ranges runs whole here).
template <class G>
inline int64_t shuffle_head(int64_t m, int64_t keep, G& rng, int32_t* out) {
    if (m <= 0) return 0;  // std::shuffle of an empty range draws nothing
    if (shuffle_pairs(m)) {
        std::vector<int32_t> v(static_cast<size_t>(m));
        std::iota(v.begin(), v.end(), 0);
        std::shuffle(v.begin(), v.end(), rng);
        std::copy(v.begin(), v.begin() + keep, out);
        return m;
    }
    std::iota(out, out + keep, 0);
    int64_t i = 1;
    for (; i < keep; ++i) {
        const uint32_t j = bounded(rng, static_cast<uint32_t>(i + 1));
        std::swap(out[i], out[j]);
    }
    return std::max<int64_t>(i, 1);
}

// out[p] = index (in [0, m)) of the element std::shuffle(iota(m), rng) puts at p < keep.
template <class G>
inline void shuffled_prefix(int64_t m, int64_t keep, G& rng, int32_t* out) {
    if (m <= 0) return;
    keep = std::max<int64_t>(0, std::min(keep, m));
    std::vector<int32_t> buf(static_cast<size_t>(keep) + 1);
    const int64_t i = shuffle_head(m, keep, rng, buf.data());
    if (i < m) shuffle_tail(i, m, keep, rng, buf.data());
    std::copy(buf.begin(), buf.end() - 1, out);
}

// Index of the first word of w[0..k) whose draw may take more than one word: word l,
// paired with range r0 + l, whose product w * r has low half (mod 2^32) below r.  k when
// there is none.  Every other word is accepted by Lemire's method as it stands.
inline int first_candidate_scalar(const uint32_t* w, uint32_t r0, int k) {
    for (int l = 0; l < k; ++l) {
        const uint32_t r = r0 + static_cast<uint32_t>(l);
        if (w[l] * r < r) return l;
    }
    return k;
}

#ifdef TGB_HAVE_AVX512_TAIL
// The same, 16 words per step: one 32-bit multiply-low and one unsigned compare into a mask.
__attribute__((target("avx512f"))) inline int first_candidate_avx512(const uint32_t* w, uint32_t r0, int k) {
    const __m512i lane = _mm512_setr_epi32(0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15);
    int l = 0;
    for (; l + 16 <= k; l += 16) {
        const __m512i R = _mm512_add_epi32(_mm512_set1_epi32(static_cast<int>(r0 + static_cast<uint32_t>(l))), lane);
        const __m512i lo = _mm512_mullo_epi32(_mm512_loadu_si512(w + l), R);
        const __mmask16 c = _mm512_cmplt_epu32_mask(lo, R);
        if (c) return l + __builtin_ctz(c);
    }
    if (l < k) {
        const __mmask16 valid = static_cast<__mmask16>((1u << (k - l)) - 1u);
        const __m512i R = _mm512_add_epi32(_mm512_set1_epi32(static_cast<int>(r0 + static_cast<uint32_t>(l))), lane);
        const __m512i lo = _mm512_mullo_epi32(_mm512_maskz_loadu_epi32(valid, w + l), R);
        const __mmask16 c = _mm512_mask_cmplt_epu32_mask(valid, lo, R);
        if (c) return l + __builtin_ctz(c);
    }
    return k;
}
#endif

inline int first_candidate(const uint32_t* w, uint32_t r0, int k) {
#ifdef TGB_HAVE_AVX512_TAIL
    if (have_avx512()) return first_candidate_avx512(w, r0, k);
#endif
    return first_candidate_scalar(w, r0, k);
}

// Advances rng exactly as std::shuffle of m elements does, without producing positions.
// A draw consumes extra words only when its first product's low half is below the
// range (probability range / 2^32): the words before the first such candidate are
// skipped in one step, and the candidate itself takes the exact draw.
inline void skip_shuffle(int64_t m, Mt32& rng) {
    if (m <= 0) return;
    if (shuffle_pairs(m)) {
        std::vector<int32_t> v(static_cast<size_t>(m));
        std::shuffle(v.begin(), v.end(), rng);
        return;
    }
    int64_t i = 1;  // next draw uses range i + 1
    while (i < m) {
        if (rng.pos >= 624) rng.refill();
        const int k = static_cast<int>(std::min<int64_t>(624 - rng.pos, m - i));
        const int done = first_candidate(rng.out + rng.pos, static_cast<uint32_t>(i + 1), k);
        rng.pos += done;
        i += done;
        if (done == k) continue;  // block exhausted or m reached
        (void)bounded(rng, static_cast<uint32_t>(i + 1));
        ++i;
    }
}

template <class G>
inline void skip_shuffle(int64_t m, G& rng) {
    if (m <= 0) return;
    if (shuffle_pairs(m)) {
        std::vector<int32_t> v(static_cast<size_t>(m));
        std::shuffle(v.begin(), v.end(), rng);
        return;
    }
    for (int64_t i = 1; i < m; ++i) (void)bounded(rng, static_cast<uint32_t>(i + 1));
}

}  // namespace tgb
