// Quantile-bin transform: X (row-major f32 or f64) -> uint8 codes, row-major
// [n][stride].  Restates Binner::transform (cpp/src/binning.cpp:104-128):
// code = 1 + upper_bound(edges, v), NaN -> 0 (kMissingBin, cpp/include/tidegbm/types.hpp:20);
// a categorical feature's code is 1 + the value's vocabulary index (0 when absent).
//
// For f32 input the edges arrive as ceil_f32(edge) (the smallest float >= the f64
// edge): for a float v, v < e  <=>  v < ceil_f32(e) (a NaN edge stays NaN), so the float
// compare gives the reference's f64 upper_bound exactly.  f64 input compares against f64
// edges.
//
// Launch shape: one CTA = 8 warps x a group of 32 features; lane = feature, so a
// warp reads one row's 32 consecutive values (coalesced) and writes 32 code bytes.
// Edges of the group sit in shared memory with a 257-element feature stride so the
// first probes of the 32 lanes fall in 32 different banks.
#include "tgb_internal.h"

#include <cmath>

namespace tgb {

namespace {

constexpr int kBinWarps = 8;
constexpr int kEdgeStride = 257;

template <typename T>
__global__ void __launch_bounds__(kBinWarps * 32)
    bin_transform_kernel(const T* __restrict__ X, int n, int n_f, const T* __restrict__ edges,
                         const int* __restrict__ n_edges, uint8_t* __restrict__ codes, int stride,
                         int rows_per_cta, const uint8_t* __restrict__ is_cat) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* se = reinterpret_cast<T*>(smem_raw);
    __shared__ int sne[32];
    const int f0 = blockIdx.y * 32;
    const int nf_here = min(32, n_f - f0);
    for (int k = threadIdx.x; k < 32 * 256; k += blockDim.x) {
        const int ff = k >> 8, b = k & 255;
        T v = T(INFINITY);
        if (ff < nf_here) v = edges[static_cast<size_t>(f0 + ff) * 256 + b];
        se[ff * kEdgeStride + b] = v;
    }
    if (threadIdx.x < 32) sne[threadIdx.x] = threadIdx.x < nf_here ? n_edges[f0 + threadIdx.x] : 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane >= nf_here) return;
    const T* e = se + lane * kEdgeStride;
    const int ne = sne[lane];
    const bool cat = is_cat != nullptr && is_cat[f0 + lane] != 0;
    const int r0 = blockIdx.x * rows_per_cta;
    const int r1 = min(n, r0 + rows_per_cta);
    for (int r = r0 + warp; r < r1; r += kBinWarps) {
        const T v = X[static_cast<size_t>(r) * n_f + f0 + lane];
        int code = 0;
        if (cat && !(v != v)) {
            // categorical (binning.cpp:112-117): 1 + the value's index in the sorted
            // vocabulary (std::lower_bound's bisection), 0 when it is not in it
            int first = 0, len = ne;
            while (len > 0) {
                const int half = len >> 1;
                const int mid = first + half;
                if (e[mid] < v) {
                    first = mid + 1;
                    len = len - half - 1;
                } else {
                    len = half;
                }
            }
            code = (first < ne && e[first] == v) ? first + 1 : 0;
        } else if (!(v != v)) {
            // std::upper_bound's own bisection (libstdc++ __upper_bound): the same probes
            // and the same answer as the reference, also when NaN edges break the order
            int first = 0, len = ne;
            while (len > 0) {
                const int half = len >> 1;
                const int mid = first + half;
                if (v < e[mid]) {
                    len = half;
                } else {
                    first = mid + 1;
                    len = len - half - 1;
                }
            }
            code = first + 1;
        }
        codes[static_cast<size_t>(r) * stride + f0 + lane] = static_cast<uint8_t>(code);
    }
}

// Zero the padding bytes [n_f, stride) of every row so gathers of whole rows see 0.
__global__ void zero_pad_kernel(uint8_t* codes, int n, int n_f, int stride) {
    const int pad = stride - n_f;
    const size_t total = static_cast<size_t>(n) * pad;
    for (size_t k = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; k < total;
         k += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const size_t r = k / pad;
        codes[r * stride + n_f + (k % pad)] = 0;
    }
}

// Column-major copy for the partition's single-feature reads: a CTA moves a tile of
// 128 rows x 32 features through shared memory (16-byte loads of row chunks, 16-byte
// stores of column runs).
// col has a row pitch of round_up(n, 16) bytes, so every 16-row run is 16-byte aligned.
__global__ void __launch_bounds__(256)
    codes_transpose_kernel(const uint8_t* __restrict__ codes, int stride, int n, int n_f, uint8_t* __restrict__ col,
                           long long pitch) {
    __shared__ uint8_t tile[128][33];
    const int r0 = blockIdx.x * 128, f0 = blockIdx.y * 32;
    {
        const int r = threadIdx.x >> 1, half = threadIdx.x & 1;  // 2 x 16 bytes per row
        const int fb = f0 + half * 16;
        if (r0 + r < n && fb < stride) {
            const uint4 v = *reinterpret_cast<const uint4*>(codes + static_cast<size_t>(r0 + r) * stride + fb);
            const uint8_t* b = reinterpret_cast<const uint8_t*>(&v);
#pragma unroll
            for (int i = 0; i < 16; ++i) tile[r][half * 16 + i] = b[i];
        }
    }
    __syncthreads();
    const int fl = threadIdx.x >> 3, q = threadIdx.x & 7;  // feature, run of 16 rows
    const int f = f0 + fl;
    if (f >= n_f) return;
    const int rb = r0 + q * 16;
    if (rb + 16 <= n) {
        uint4 v;
        uint8_t* b = reinterpret_cast<uint8_t*>(&v);
#pragma unroll
        for (int i = 0; i < 16; ++i) b[i] = tile[q * 16 + i][fl];
        *reinterpret_cast<uint4*>(col + static_cast<size_t>(f) * pitch + rb) = v;
    } else {
        for (int i = 0; i < 16 && rb + i < n; ++i) col[static_cast<size_t>(f) * pitch + rb + i] = tile[q * 16 + i][fl];
    }
}

template <typename T>
void launch_bin(const T* X, int n, int n_f, const T* edges, const int* n_edges, uint8_t* codes,
                int stride, cudaStream_t s, const uint8_t* is_cat) {
    if (n <= 0 || n_f <= 0) return;
    const int rows_per_cta = 512;
    dim3 grid((n + rows_per_cta - 1) / rows_per_cta, (n_f + 31) / 32);
    const size_t smem = sizeof(T) * 32 * kEdgeStride;
    auto kern = bin_transform_kernel<T>;
    check(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)),
          "bin smem attr");
    kern<<<grid, kBinWarps * 32, smem, s>>>(X, n, n_f, edges, n_edges, codes, stride, rows_per_cta, is_cat);
    check(cudaGetLastError(), "bin_transform launch");
    if (stride > n_f) {
        zero_pad_kernel<<<1184, 256, 0, s>>>(codes, n, n_f, stride);
        check(cudaGetLastError(), "zero_pad launch");
    }
}

}  // namespace

void launch_codes_transpose(const uint8_t* codes, int stride, int n, int n_f, uint8_t* col, cudaStream_t s) {
    if (n <= 0 || n_f <= 0) return;
    dim3 grid((n + 127) / 128, (n_f + 31) / 32);
    codes_transpose_kernel<<<grid, 256, 0, s>>>(codes, stride, n, n_f, col, codes_col_pitch(n));
    check(cudaGetLastError(), "codes_transpose launch");
}

void launch_bin_transform_f32(const float* X, int n, int n_f, const float* edges, const int* n_edges,
                              uint8_t* codes, int stride, cudaStream_t s, const uint8_t* is_cat) {
    launch_bin<float>(X, n, n_f, edges, n_edges, codes, stride, s, is_cat);
}

void launch_bin_transform_f64(const double* X, int n, int n_f, const double* edges, const int* n_edges,
                              uint8_t* codes, int stride, cudaStream_t s, const uint8_t* is_cat) {
    launch_bin<double>(X, n, n_f, edges, n_edges, codes, stride, s, is_cat);
}

}  // namespace tgb
