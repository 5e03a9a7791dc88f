// GOSS row selection (cpp/src/booster.cpp:554-585): keep the ceil(top * n) rows of
// largest |g|, plus n_other rows drawn from the rest, whose g and h are scaled by
// (1 - top) / other; the sample is then re-sorted by row index.
//
// The reference orders rows by |g| descending (std::sort), shuffles the remainder with
// the booster's mt19937 (std::shuffle) and keeps the first n_other.  The shuffle's
// swap positions depend only on the generator state and the remainder's length, not
// on the data, so the host derives, per tree, the list rest_pos[p] = "position in the
// |g|-descending remainder of the p-th kept row" (see booster.cpp's sample_positions
// in this library) and the device does the data-dependent part:
//   keys = bit pattern of |g| (non-negative doubles order like their bits), radix
//   sort descending (stable; rows with equal |g| keep index order; the row indices are
//   written once per fit).  The sort runs on a 32-bit order-keeping compression of the
//   pattern (4 radix passes instead of 8) and a fix-up pass re-orders the short runs of
//   tied 32-bit keys by the full pattern, which gives exactly the order of the full
//   64-bit stable sort,
//   flag[order[p]] = 1 for p < n_top, flag[order[n_top + rest_pos[p]]] = 2, with the
//   maxima of the sample's |g| and |h| (as the tree sees them) reduced on the way,
//   compaction of flagged rows in index order -> the tree's root row list.
// The hist kernel multiplies g and h of flag-2 rows by the GOSS scale on the fly.
#include "tgb_internal.h"

#include <cub/device/device_radix_sort.cuh>

namespace tgb {

namespace {

// Sort keys from g: the full |g| bit pattern (exact path), or a 32-bit key that keeps the
// order of the patterns (ties allowed): patterns at or above lo = (e_max - 63) << 52,
// e_max the exponent of max |g| (sc), map to (pattern - lo) >> 26, i.e. 6 exponent and 26
// mantissa bits over the 64 binades below the maximum; smaller values (zeros included)
// map to 0.
template <bool kExact>
__global__ void goss_keys_kernel(const double* __restrict__ g, int n, const AllScale* __restrict__ sc,
                                 void* __restrict__ keys) {
    const unsigned long long e_max = sc->maxg_bits >> 52;
    const unsigned long long lo = e_max >= 63 ? (e_max - 63) << 52 : 0ull;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const unsigned long long b = static_cast<unsigned long long>(__double_as_longlong(fabs(g[i])));
        if (kExact) static_cast<unsigned long long*>(keys)[i] = b;
        else static_cast<unsigned int*>(keys)[i] = b >= lo ? static_cast<unsigned int>((b - lo) >> 26) : 0u;
    }
}

// After the stable sort by 32-bit keys, rows whose keys tie form runs in index order.
// Every element of a run computes its rank inside the run by the full |g| pattern
// (descending, index ascending on exact ties) and writes itself there in `fixed`, which
// gives the order of the full 64-bit stable sort at the run's positions; positions
// outside runs keep order[] (the mark kernel reads fixed[] only at run positions).  A
// run longer than kMaxRun is already in order when all its patterns are equal (checked
// pairwise); otherwise it sets *overflow (the fit then repeats with the 64-bit sort).
constexpr int kMaxRun = 64;

__device__ __forceinline__ unsigned long long abs_bits(const double* g, int32_t r) {
    return static_cast<unsigned long long>(__double_as_longlong(fabs(g[r])));
}

__device__ __forceinline__ bool in_run(const unsigned int* __restrict__ k32, int p, int n) {
    const unsigned int k = k32[p];
    return (p > 0 && k32[p - 1] == k) || (p + 1 < n && k32[p + 1] == k);
}

__global__ void goss_fixup_kernel(const unsigned int* __restrict__ k32, const int32_t* __restrict__ order,
                                  int32_t* __restrict__ fixed, const double* __restrict__ g, int n,
                                  int* __restrict__ overflow) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        if (!in_run(k32, p, n)) continue;
        const unsigned int k = k32[p];
        const int32_t me = order[p];
        int a = p;
        while (a > 0 && p - a < kMaxRun && k32[a - 1] == k) --a;
        int e = p + 1;
        while (e < n && e - a < kMaxRun && k32[e] == k) ++e;
        const unsigned long long km = abs_bits(g, me);
        if ((a > 0 && k32[a - 1] == k) || (e < n && k32[e] == k)) {
            // long run: in order as it is only if every pattern in it is equal
            if (p > 0 && k32[p - 1] == k && abs_bits(g, order[p - 1]) != km) atomicExch(overflow, 1);
            fixed[p] = me;
            continue;
        }
        int rank = 0;
        for (int q = a; q < e; ++q) {
            if (q == p) continue;
            const unsigned long long kq = abs_bits(g, order[q]);
            if (kq > km || (kq == km && q < p)) ++rank;  // inside a run, position order is index order
        }
        fixed[a + rank] = me;
    }
}

__global__ void goss_iota_kernel(int32_t* __restrict__ vals, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) vals[i] = i;
}

// Marks the sample and reduces the maxima the histogram scales need over it: |g| and
// |h| of the top rows, |g * scale| and |h * scale| of the sampled others (the values the
// tree sees).  With unit hessians (h == nullptr) the maxima are known from two rows: the
// first of the |g| order (the largest |g|) and the sampled other of smallest remainder
// rank (min_rest, the largest |g| among them); only those two threads read g.
__global__ void goss_mark_kernel(const int32_t* __restrict__ order, const unsigned int* __restrict__ k32,
                                 const int32_t* __restrict__ fixed, int n, int n_top, int n_other,
                                 const int32_t* __restrict__ rest_pos, int min_rest, const double* __restrict__ g,
                                 const double* __restrict__ h, double goss_scale, uint8_t* __restrict__ flag,
                                 DevTreeState* __restrict__ st) {
    const int total = n_top + n_other;
    double mg = 0.0, mh = 0.0;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < total; p += gridDim.x * blockDim.x) {
        const bool top = p < n_top;
        const int rp = top ? 0 : rest_pos[p - n_top];
        const int pos = top ? p : n_top + rp;
        const int r = (k32 != nullptr && in_run(k32, pos, n)) ? fixed[pos] : order[pos];
        flag[r] = top ? 1 : 2;
        if (h != nullptr) {
            mg = fmax(mg, top ? fabs(g[r]) : fabs(g[r] * goss_scale));
            mh = fmax(mh, top ? fabs(h[r]) : fabs(h[r] * goss_scale));
        } else if (top ? p == 0 : rp == min_rest) {
            mg = fmax(mg, top ? fabs(g[r]) : fabs(g[r] * goss_scale));
            mh = fmax(mh, top ? 1.0 : fabs(1.0 * goss_scale));
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mg = fmax(mg, __shfl_xor_sync(0xffffffffu, mg, o));
        mh = fmax(mh, __shfl_xor_sync(0xffffffffu, mh, o));
    }
    if ((threadIdx.x & 31) == 0 && (mg > 0.0 || mh > 0.0)) {
        atomicMax(&st->max_abs_g_bits, static_cast<unsigned long long>(__double_as_longlong(mg)));
        atomicMax(&st->max_h_bits, static_cast<unsigned long long>(__double_as_longlong(mh)));
    }
}

}  // namespace

size_t goss_cub_bytes(int n, bool exact) {
    size_t bytes = 0;
    if (exact)
        check(cub::DeviceRadixSort::SortPairsDescending(nullptr, bytes, static_cast<unsigned long long*>(nullptr),
                                                        static_cast<unsigned long long*>(nullptr),
                                                        static_cast<int32_t*>(nullptr), static_cast<int32_t*>(nullptr),
                                                        n),
              "cub sizing");
    else
        check(cub::DeviceRadixSort::SortPairsDescending(nullptr, bytes, static_cast<unsigned int*>(nullptr),
                                                        static_cast<unsigned int*>(nullptr),
                                                        static_cast<int32_t*>(nullptr), static_cast<int32_t*>(nullptr),
                                                        n),
              "cub sizing");
    return bytes;
}

void launch_goss_iota(int32_t* vals, int n, cudaStream_t s) {
    goss_iota_kernel<<<std::max(1, std::min(2368, (n + 255) / 256)), 256, 0, s>>>(vals, n);
    check(cudaGetLastError(), "goss_iota launch");
}

void launch_goss_select(const double* g, const double* h, int n, int n_top, int n_other, const int32_t* rest_pos,
                        int min_rest, GossWork& w, const AllScale* all, double goss_scale, uint8_t* goss_flag,
                        int32_t* rows0, int* tile_counts, DevTreeState* st, cudaStream_t s) {
    const int blocks = std::max(1, std::min(2368, (n + 255) / 256));
    if (w.exact) goss_keys_kernel<true><<<blocks, 256, 0, s>>>(g, n, all, w.keys_in);
    else goss_keys_kernel<false><<<blocks, 256, 0, s>>>(g, n, all, w.keys_in);
    check(cudaGetLastError(), "goss_keys launch");
    size_t tmp = w.cub_tmp_bytes;
    if (w.exact) {
        check(cub::DeviceRadixSort::SortPairsDescending(w.cub_tmp, tmp, static_cast<unsigned long long*>(w.keys_in),
                                                        static_cast<unsigned long long*>(w.keys_out), w.vals_in,
                                                        w.vals_out, n, 0, 64, s),
              "goss sort");
    } else {
        check(cub::DeviceRadixSort::SortPairsDescending(w.cub_tmp, tmp, static_cast<unsigned int*>(w.keys_in),
                                                        static_cast<unsigned int*>(w.keys_out), w.vals_in,
                                                        w.vals_out, n, 0, 32, s),
              "goss sort");
        // run positions re-ordered into keys_in's memory (free once sorted)
        goss_fixup_kernel<<<blocks, 256, 0, s>>>(static_cast<const unsigned int*>(w.keys_out), w.vals_out,
                                                  static_cast<int32_t*>(w.keys_in), g, n, w.overflow);
        check(cudaGetLastError(), "goss_fixup launch");
    }
    const unsigned int* k32 = w.exact ? nullptr : static_cast<const unsigned int*>(w.keys_out);
    const int32_t* fixed = static_cast<const int32_t*>(w.keys_in);
    check(cudaMemsetAsync(goss_flag, 0, static_cast<size_t>(n), s), "goss flag reset");
    check(cudaMemsetAsync(&st->max_abs_g_bits, 0, 2 * sizeof(unsigned long long), s), "sample max reset");
    goss_mark_kernel<<<std::max(1, std::min(2368, (n_top + n_other + 255) / 256)), 256, 0, s>>>(
        w.vals_out, k32, fixed, n, n_top, n_other, rest_pos, min_rest, g, h, goss_scale, goss_flag, st);
    check(cudaGetLastError(), "goss_mark launch");
    launch_compact_flagged(goss_flag, n, rows0, &st->n_sample, tile_counts, s);
}

}  // namespace tgb
