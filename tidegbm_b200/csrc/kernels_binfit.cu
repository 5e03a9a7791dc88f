// Device half of quantile binning: Binner::fit (cpp/src/binning.cpp:14-102) for
// numeric features with the sample gathered, sorted and reduced to edges in HBM,
// next to the X the transform reads anyway.
//
// The reference collects a feature's non-NaN values, keeps the first bin_sample after
// std::shuffle(mt19937(seed + f * 2654435761)) when there are more (binning.cpp:
// 93-97), and computes quantile_edges of that sample (binning.cpp:14-32).  Which
// values are kept is fixed by their non-NaN ranks, and the kept ranks depend only on
// the generator and the non-NaN count.  The order of the kept values is irrelevant
// (quantile_edges sorts).  So:
//   nonnan_count_kernel     non-NaN count per (chunk of kFitChunk rows, feature)
//   (host)                  counts -> per-feature totals and per-chunk rank bases;
//                           the head of the exact shuffle prefix (sampling.h)
//   shuffle_tail_kernel     the shuffle's remaining draws (kernels_shuffle.cu)
//   keep_bits_kernel        kept ranks -> one bit per non-NaN rank and feature
//   kept_counts_kernel      kept values per (chunk, feature): a popcount of the chunk's
//                           rank range of the feature's kept bits
//   kept_scan_kernel        their exclusive prefix over the chunks of each feature
//   sample_gather_kernel    X once more; each kept value goes to its feature's sample at
//                           its chunk's prefix plus its rank among the chunk's kept values
//   CUB segmented sort      every feature's sample ascending
//   quantile_edges_kernel   unique values, then the interpolated edges in the
//                           reference's FP64 statement order (this file is compiled
//                           with -fmad=false), sorted and deduplicated
// Launch shape of the two X walks: thread = feature (32 consecutive features per
// warp read 128 or 256 contiguous bytes of a row), CTA = a chunk of rows, so a
// thread meets its feature's values in row order and can count ranks locally.
#include "tgb_internal.h"

#include <cub/block/block_scan.cuh>
#include <cub/device/device_segmented_sort.cuh>

namespace tgb {

namespace {

constexpr int kWalkThreads = 128;
constexpr int kEdgeThreads = 1024;

template <typename T>
__device__ __forceinline__ bool not_nan(T v) {
    return v == v;
}

template <typename T>
__global__ void __launch_bounds__(kWalkThreads)
    nonnan_count_kernel(const T* __restrict__ X, int n, int n_f, int* __restrict__ counts) {
    const int f = blockIdx.y * kWalkThreads + threadIdx.x;
    if (f >= n_f) return;
    const int r0 = blockIdx.x * kFitChunk;
    const int r1 = min(n, r0 + kFitChunk);
    const T* p = X + static_cast<size_t>(r0) * n_f + f;
    int cnt = 0;
    int r = r0;
    for (; r + 8 <= r1; r += 8) {
        T v[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) v[k] = __ldcs(p + static_cast<size_t>(r - r0 + k) * n_f);
#pragma unroll
        for (int k = 0; k < 8; ++k) cnt += not_nan(v[k]) ? 1 : 0;
    }
    for (; r < r1; ++r) cnt += not_nan(__ldcs(p + static_cast<size_t>(r - r0) * n_f)) ? 1 : 0;
    counts[static_cast<size_t>(blockIdx.x) * n_f + f] = cnt;
}

// bits[f][rank / 32] |= 1 << (rank % 32) for each kept rank of a sampled feature.
__global__ void keep_bits_kernel(const int32_t* __restrict__ keep, int bin_sample, int n_f,
                                 const uint8_t* __restrict__ take_all, uint32_t* __restrict__ bits,
                                 long long words) {
    const long long total = static_cast<long long>(n_f) * bin_sample;
    for (long long k = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; k < total;
         k += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int f = static_cast<int>(k / bin_sample);
        if (take_all[f]) continue;
        const uint32_t r = static_cast<uint32_t>(keep[k]);
        atomicOr(bits + f * words + (r >> 5), 1u << (r & 31));
    }
}

// One warp per (chunk, feature): the kept values among the feature's non-NaN ranks
// [base[c][f], base[c + 1][f]) (the last chunk ends at the feature's total m[f]).
__global__ void kept_counts_kernel(const long long* __restrict__ base, const long long* __restrict__ m, int n_chunks,
                                   int n_f, const uint32_t* __restrict__ bits, long long words,
                                   const uint8_t* __restrict__ take_all, int* __restrict__ kc) {
    const int lane = threadIdx.x & 31;
    const long long n_pairs = static_cast<long long>(n_chunks) * n_f;
    for (long long pr = (blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x) >> 5; pr < n_pairs;
         pr += (static_cast<long long>(gridDim.x) * blockDim.x) >> 5) {
        const int c = static_cast<int>(pr / n_f), f = static_cast<int>(pr - static_cast<long long>(c) * n_f);
        const long long lo = base[pr];
        const long long hi = c + 1 < n_chunks ? base[pr + n_f] : m[f];
        int cnt = 0;
        if (take_all[f]) {
            cnt = static_cast<int>(hi - lo);
        } else if (hi > lo) {
            const uint32_t* fb = bits + f * words;
            for (long long w = (lo >> 5) + lane; w <= ((hi - 1) >> 5); w += 32) {
                uint32_t v = fb[w];
                const long long b0 = w << 5;
                if (b0 < lo) v &= ~0u << (lo - b0);                       // drop ranks below lo
                if (b0 + 32 > hi) v &= (hi - b0 >= 32) ? ~0u : ((1u << (hi - b0)) - 1u);  // and from hi on
                cnt += __popc(v);
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
        }
        if (lane == 0) kc[pr] = cnt;
    }
}

// One CTA per feature: kbase[c][f] = sum of kc[c'][f] over c' < c; total[f] = the sum.
__global__ void __launch_bounds__(256) kept_scan_kernel(const int* __restrict__ kc, int n_chunks, int n_f,
                                                       int* __restrict__ kbase, int* __restrict__ total) {
    const int f = blockIdx.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __shared__ int s_w[8];
    int run = 0;
    for (int c0 = 0; c0 < n_chunks; c0 += 256) {
        const int c = c0 + static_cast<int>(threadIdx.x);
        const int v = c < n_chunks ? kc[static_cast<size_t>(c) * n_f + f] : 0;
        int incl = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        if (lane == 31) s_w[warp] = incl;
        __syncthreads();
        int wb = 0, all = 0;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            if (k < warp) wb += s_w[k];
            all += s_w[k];
        }
        if (c < n_chunks) kbase[static_cast<size_t>(c) * n_f + f] = run + wb + incl - v;
        run += all;
        __syncthreads();  // s_w reuse
    }
    if (threadIdx.x == 0) total[f] = run;
}

template <typename T>
__global__ void __launch_bounds__(kWalkThreads)
    sample_gather_kernel(const T* __restrict__ X, int n, int n_f, const long long* __restrict__ base,
                         const uint32_t* __restrict__ bits, long long words, const uint8_t* __restrict__ take_all,
                         T* __restrict__ sample, long long cap, const int* __restrict__ kbase) {
    const int f = blockIdx.y * kWalkThreads + threadIdx.x;
    if (f >= n_f) return;
    const int r0 = blockIdx.x * kFitChunk;
    const int r1 = min(n, r0 + kFitChunk);
    const T* p = X + static_cast<size_t>(r0) * n_f + f;
    long long rank = base[static_cast<size_t>(blockIdx.x) * n_f + f];
    const bool all = take_all[f] != 0;
    const uint32_t* fb = bits + f * words;
    T* out = sample + f * cap + kbase[static_cast<size_t>(blockIdx.x) * n_f + f];
    int k_out = 0;
    auto visit = [&](T v) {
        if (!not_nan(v)) return;
        const bool kept = all || ((fb[rank >> 5] >> (rank & 31)) & 1u);
        if (kept) out[k_out++] = v;
        ++rank;
    };
    int r = r0;
    for (; r + 8 <= r1; r += 8) {
        T v[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) v[k] = __ldcs(p + static_cast<size_t>(r - r0 + k) * n_f);
#pragma unroll
        for (int k = 0; k < 8; ++k) visit(v[k]);
    }
    for (; r < r1; ++r) visit(__ldcs(p + static_cast<size_t>(r - r0) * n_f));
}

// One CTA per feature.  sorted: the feature's sample ascending (cnt[f] values at
// f * cap); uniq: scratch of the same shape.  Writes edges[f][0..n_edges[f]).
template <typename T>
__global__ void __launch_bounds__(kEdgeThreads)
    quantile_edges_kernel(const T* __restrict__ sorted, T* __restrict__ uniq, long long cap,
                          const int* __restrict__ cnt, int n_bins, double* __restrict__ edges,
                          int* __restrict__ n_edges, int* __restrict__ flags) {
    using BlockScan = cub::BlockScan<int, kEdgeThreads>;
    __shared__ typename BlockScan::TempStorage scan_tmp;
    __shared__ double e[256];
    __shared__ int both_zeros;
    const int f = blockIdx.x;
    const T* v = sorted + f * cap;
    T* u = uniq + f * cap;
    const int m = cnt[f];
    // Features whose edges depend on the order std::sort leaves equal values in (the
    // reference sorts the sample in its shuffled order): a sample holding both -0.0 and
    // +0.0 (which one std::unique keeps decides the sign of a zero edge), and a sample
    // holding an infinity when edges are interpolated (inf * 0 makes NaN edges, whose
    // place after std::sort depends on the algorithm).  flags[f] = 1 sends the feature
    // back to the host, which recomputes it in the reference's order.
    if (threadIdx.x == 0) both_zeros = 0;
    __syncthreads();
    for (int i = 1 + threadIdx.x; i < m; i += kEdgeThreads)
        if (v[i] == T(0) && v[i - 1] == T(0) && signbit(v[i]) != signbit(v[i - 1])) both_zeros = 1;
    __syncthreads();
    // std::sort + std::unique (binning.cpp:15-16): keep the first of every run of equal values
    int n_u = 0;
    for (int i0 = 0; i0 < m; i0 += kEdgeThreads) {
        const int i = i0 + threadIdx.x;
        int first = 0;
        T x = T(0);
        if (i < m) {
            x = v[i];
            first = (i == 0 || v[i - 1] != x) ? 1 : 0;
        }
        int pre = 0, agg = 0;
        BlockScan(scan_tmp).ExclusiveSum(first, pre, agg);
        if (first) u[n_u + pre] = x;
        n_u += agg;
        __syncthreads();
    }
    double* ef = edges + static_cast<size_t>(f) * 256;
    if (threadIdx.x == 0) {
        const bool inf = n_u > n_bins && (isinf(static_cast<double>(u[0])) || isinf(static_cast<double>(u[n_u - 1])));
        flags[f] = (both_zeros || inf) ? 1 : 0;
    }
    if (n_u == 0) {  // no values: edges {0.0} (binning.cpp:17)
        if (threadIdx.x == 0) {
            ef[0] = 0.0;
            n_edges[f] = 1;
        }
        return;
    }
    if (n_u <= n_bins) {  // few distinct values: they are the edges (binning.cpp:18)
        for (int k = threadIdx.x; k < n_u; k += kEdgeThreads) ef[k] = static_cast<double>(u[k]);
        if (threadIdx.x == 0) n_edges[f] = n_u;
        return;
    }
    // binning.cpp:19-29, one edge per thread, same FP64 statements
    const double last = static_cast<double>(static_cast<long long>(n_u) - 1);
    for (int i = 1 + threadIdx.x; i < n_bins; i += kEdgeThreads) {
        const double q = static_cast<double>(i) / n_bins;
        const double pos = q * last;
        const long long lo = static_cast<long long>(pos);
        const long long hi = min(lo + 1, static_cast<long long>(n_u) - 1);
        const double frac = pos - static_cast<double>(lo);
        e[i - 1] = static_cast<double>(u[lo]) * (1 - frac) + static_cast<double>(u[hi]) * frac;
    }
    __syncthreads();
    if (threadIdx.x == 0) {  // sort + unique (binning.cpp:30-31); at most 255 values, nearly sorted
        const int k = n_bins - 1;
        for (int a = 1; a < k; ++a) {
            const double x = e[a];
            int b = a - 1;
            while (b >= 0 && x < e[b]) {
                e[b + 1] = e[b];
                --b;
            }
            e[b + 1] = x;
        }
        int w = 0;
        for (int a = 0; a < k; ++a)
            if (w == 0 || !(e[a] == e[w - 1])) e[w++] = e[a];
        for (int a = 0; a < w; ++a) ef[a] = e[a];
        n_edges[f] = w;
    }
}

template <typename T>
void launch_walk_count(const T* X, int n, int n_f, int* counts, cudaStream_t s) {
    dim3 grid((n + kFitChunk - 1) / kFitChunk, (n_f + kWalkThreads - 1) / kWalkThreads);
    nonnan_count_kernel<T><<<grid, kWalkThreads, 0, s>>>(X, n, n_f, counts);
    check(cudaGetLastError(), "nonnan_count launch");
}

template <typename T>
void launch_walk_gather(const T* X, int n, int n_f, const long long* base, const uint32_t* bits, long long words,
                        const uint8_t* take_all, T* sample, long long cap, const int* kbase, cudaStream_t s) {
    dim3 grid((n + kFitChunk - 1) / kFitChunk, (n_f + kWalkThreads - 1) / kWalkThreads);
    sample_gather_kernel<T><<<grid, kWalkThreads, 0, s>>>(X, n, n_f, base, bits, words, take_all, sample, cap, kbase);
    check(cudaGetLastError(), "sample_gather launch");
}

template <typename T>
size_t sort_bytes_t(long long total, int n_f) {
    size_t bytes = 0;
    check(cub::DeviceSegmentedSort::SortKeys(nullptr, bytes, static_cast<const T*>(nullptr), static_cast<T*>(nullptr),
                                             static_cast<int>(total), n_f, static_cast<const int*>(nullptr),
                                             static_cast<const int*>(nullptr)),
          "cub sizing");
    return bytes;
}

}  // namespace

void launch_nonnan_counts(const void* X, int x_dtype, int n, int n_f, int* counts, cudaStream_t s) {
    if (n <= 0 || n_f <= 0) return;
    if (x_dtype == 0) launch_walk_count(static_cast<const float*>(X), n, n_f, counts, s);
    else launch_walk_count(static_cast<const double*>(X), n, n_f, counts, s);
}

void launch_keep_bits(const int32_t* keep, int bin_sample, int n_f, const uint8_t* take_all, uint32_t* bits,
                      long long words, cudaStream_t s) {
    const long long total = static_cast<long long>(n_f) * bin_sample;
    if (total <= 0) return;
    const int blocks = static_cast<int>(std::min<long long>(148 * 16, (total + 255) / 256));
    keep_bits_kernel<<<blocks, 256, 0, s>>>(keep, bin_sample, n_f, take_all, bits, words);
    check(cudaGetLastError(), "keep_bits launch");
}

void launch_sample_gather(const void* X, int x_dtype, int n, int n_f, const long long* base, const long long* m,
                          const uint32_t* bits, long long words, const uint8_t* take_all, void* sample, long long cap,
                          int* kc, int* kbase, int* total, cudaStream_t s) {
    if (n <= 0 || n_f <= 0) return;
    const int n_chunks = (n + kFitChunk - 1) / kFitChunk;
    const long long pairs = static_cast<long long>(n_chunks) * n_f;
    const int blocks = static_cast<int>(std::min<long long>(148 * 16, (pairs * 32 + 255) / 256));
    kept_counts_kernel<<<blocks, 256, 0, s>>>(base, m, n_chunks, n_f, bits, words, take_all, kc);
    check(cudaGetLastError(), "kept_counts launch");
    kept_scan_kernel<<<n_f, 256, 0, s>>>(kc, n_chunks, n_f, kbase, total);
    check(cudaGetLastError(), "kept_scan launch");
    if (x_dtype == 0)
        launch_walk_gather(static_cast<const float*>(X), n, n_f, base, bits, words, take_all,
                           static_cast<float*>(sample), cap, kbase, s);
    else
        launch_walk_gather(static_cast<const double*>(X), n, n_f, base, bits, words, take_all,
                           static_cast<double*>(sample), cap, kbase, s);
}

size_t sample_sort_bytes(int x_dtype, long long total, int n_f) {
    return x_dtype == 0 ? sort_bytes_t<float>(total, n_f) : sort_bytes_t<double>(total, n_f);
}

void launch_sample_sort(int x_dtype, const void* in, void* out, long long total, int n_f, const int* seg_begin,
                        const int* seg_end, void* tmp, size_t tmp_bytes, cudaStream_t s) {
    size_t bytes = tmp_bytes;
    if (x_dtype == 0)
        check(cub::DeviceSegmentedSort::SortKeys(tmp, bytes, static_cast<const float*>(in), static_cast<float*>(out),
                                                 static_cast<int>(total), n_f, seg_begin, seg_end, s),
              "sample sort");
    else
        check(cub::DeviceSegmentedSort::SortKeys(tmp, bytes, static_cast<const double*>(in),
                                                 static_cast<double*>(out), static_cast<int>(total), n_f, seg_begin,
                                                 seg_end, s),
              "sample sort");
}

void launch_quantile_edges(int x_dtype, const void* sorted, void* uniq, long long cap, const int* cnt, int n_f,
                           int n_bins, double* edges, int* n_edges, int* flags, cudaStream_t s) {
    if (n_f <= 0) return;
    if (x_dtype == 0)
        quantile_edges_kernel<float><<<n_f, kEdgeThreads, 0, s>>>(static_cast<const float*>(sorted),
                                                                  static_cast<float*>(uniq), cap, cnt, n_bins,
                                                                  edges, n_edges, flags);
    else
        quantile_edges_kernel<double><<<n_f, kEdgeThreads, 0, s>>>(static_cast<const double*>(sorted),
                                                                   static_cast<double*>(uniq), cap, cnt, n_bins,
                                                                   edges, n_edges, flags);
    check(cudaGetLastError(), "quantile_edges launch");
}

}  // namespace tgb
