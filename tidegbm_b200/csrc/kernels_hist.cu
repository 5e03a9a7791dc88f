// Per-node gradient/hessian histograms.  Restates build_hist_col / build_hist
// (cpp/src/histogram.cpp:24-76) and subtract_hist_inplace (histogram.cpp:108-117),
// and replaces hist_atomic_kernel + build_hist_gpu (cpp/src/histogram_cuda.cu:28-167).
//
// Numerics: every row's g and h are converted once to 64-bit fixed point,
// q = rint(v * 2^shift), with one shift per tree chosen so that no sum over the
// sample can reach 2^62.  Sums are then exact integers: deterministic, independent
// of summation order and of the launch shape, and the parent-minus-sibling
// subtraction is exact.  The error against an FP64 sum is at most
// rows * 2^-(shift+1) (about 1e-12 relative at 10M rows).
//
// Launch shape: CTA = (feature group of FG features) x (contiguous chunk of the
// node's row list).  Each thread takes one row at a time, loads the FG code bytes of
// that row with 128-bit loads (rows are 16-byte aligned), and adds (g, h, 1) to a
// CTA-private shared-memory histogram (FG x 256 x {i64, i64, u32}).  The private
// histogram is flushed to the node's global slot with one 64-bit atomic per
// non-empty bin.
#include "tgb_internal.h"

#include <cmath>

namespace tgb {

namespace {

constexpr int kHistThreads = 512;
constexpr int kMinRowsPerCta = 2048;

template <int FG>
__device__ __forceinline__ void hist_body(const uint8_t* __restrict__ codes, int stride, int n_f,
                                          const int32_t* __restrict__ rows, int count,
                                          const double* __restrict__ g, const double* __restrict__ h,
                                          const uint8_t* __restrict__ goss_flag, double goss_scale,
                                          double gscale, double hscale, long long* G, long long* H,
                                          int* C) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    unsigned long long* sG = reinterpret_cast<unsigned long long*>(smem_raw);
    unsigned long long* sH = sG + FG * kBins;
    unsigned int* sC = reinterpret_cast<unsigned int*>(sH + FG * kBins);

    // Row chunk of this CTA.
    const int need = (count + kMinRowsPerCta - 1) / kMinRowsPerCta;
    const int n_chunks = max(1, min(static_cast<int>(gridDim.y), need));
    if (static_cast<int>(blockIdx.y) >= n_chunks) return;
    const int chunk = (count + n_chunks - 1) / n_chunks;
    const int r0 = blockIdx.y * chunk;
    const int r1 = min(count, r0 + chunk);
    if (r0 >= r1) return;
    const int fg0 = blockIdx.x * FG;

    for (int k = threadIdx.x; k < FG * kBins; k += blockDim.x) {
        sG[k] = 0ull;
        sH[k] = 0ull;
        sC[k] = 0u;
    }
    __syncthreads();

    for (int k = r0 + threadIdx.x; k < r1; k += blockDim.x) {
        const int32_t r = rows[k];
        const uint8_t* src = codes + static_cast<size_t>(r) * stride + fg0;
        uint4 v[FG / 16];
#pragma unroll
        for (int q = 0; q < FG / 16; ++q) v[q] = __ldg(reinterpret_cast<const uint4*>(src) + q);
        double gv = g[r], hv = h[r];
        if (goss_flag != nullptr && goss_flag[r] == 2) {
            gv *= goss_scale;
            hv *= goss_scale;
        }
        const unsigned long long gq = static_cast<unsigned long long>(__double2ll_rn(gv * gscale));
        const unsigned long long hq = static_cast<unsigned long long>(__double2ll_rn(hv * hscale));
        const uint8_t* bytes = reinterpret_cast<const uint8_t*>(v);
#pragma unroll
        for (int j = 0; j < FG; ++j) {
            const int slot = j * kBins + bytes[j];
            atomicAdd(&sG[slot], gq);
            atomicAdd(&sH[slot], hq);
            atomicAdd(&sC[slot], 1u);
        }
    }
    __syncthreads();

    for (int k = threadIdx.x; k < FG * kBins; k += blockDim.x) {
        const int f = fg0 + k / kBins;
        if (f >= n_f) break;
        const size_t o = static_cast<size_t>(f) * kBins + (k % kBins);
        const unsigned int c = sC[k];
        if (c == 0u) continue;
        atomicAdd(reinterpret_cast<unsigned long long*>(G) + o, sG[k]);
        atomicAdd(reinterpret_cast<unsigned long long*>(H) + o, sH[k]);
        atomicAdd(C + o, static_cast<int>(c));
    }
}

template <int FG>
__global__ void __launch_bounds__(kHistThreads)
    hist_node_kernel(const uint8_t* __restrict__ codes, int stride, int n_f, int32_t* rows0,
                     int32_t* rows1, const DevNode* __restrict__ nodes,
                     const DevTreeState* __restrict__ st, int node, const double* __restrict__ g,
                     const double* __restrict__ h, const uint8_t* __restrict__ goss_flag,
                     double goss_scale, HistSlotPtrs hs, unsigned long long* rows_counter) {
    if (st->done) return;
    const int nd = node >= 0 ? node : st->small_node;
    const DevNode& N = nodes[nd];
    const int32_t* rows = (N.buf ? rows1 : rows0) + N.start;
    // Rows histogrammed, for the algorithmic-bytes figure of the benchmark.
    if (rows_counter != nullptr && blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0)
        atomicAdd(rows_counter, static_cast<unsigned long long>(N.count));
    hist_body<FG>(codes, stride, n_f, rows, N.count, g, h, goss_flag, goss_scale, st->gscale,
                  st->hscale, hs.G + nd * hs.slot_elems, hs.H + nd * hs.slot_elems,
                  hs.C + nd * hs.slot_elems);
}

template <int FG>
__global__ void __launch_bounds__(kHistThreads)
    hist_rows_kernel(const uint8_t* __restrict__ codes, int stride, int n_f,
                     const int32_t* __restrict__ rows, int count, const double* __restrict__ g,
                     const double* __restrict__ h, double gscale, double hscale, long long* G,
                     long long* H, int* C) {
    hist_body<FG>(codes, stride, n_f, rows, count, g, h, nullptr, 1.0, gscale, hscale, G, H, C);
}

__global__ void hist_subtract_kernel(const DevTreeState* __restrict__ st, HistSlotPtrs hs) {
    if (st->done) return;
    const size_t e = hs.slot_elems;
    const size_t p = static_cast<size_t>(st->parent) * e;
    const size_t sm = static_cast<size_t>(st->small_node) * e;
    const size_t lg = static_cast<size_t>(st->large_node) * e;
    for (size_t k = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; k < e;
         k += static_cast<size_t>(gridDim.x) * blockDim.x) {
        hs.G[lg + k] = hs.G[p + k] - hs.G[sm + k];
        hs.H[lg + k] = hs.H[p + k] - hs.H[sm + k];
        hs.C[lg + k] = hs.C[p + k] - hs.C[sm + k];
    }
}

__global__ void tree_init_kernel(DevNode* nodes, DevSplit* splits, DevTreeState* st, int n_sample,
                                 int use_dev_count) {
    const int count = use_dev_count ? st->n_sample : n_sample;
    DevNode r{};
    r.start = 0;
    r.count = count;
    r.buf = 0;
    r.depth = 0;
    r.is_leaf = 1;
    r.feature = -1;
    r.threshold = -1;
    r.missing_left = 1;
    r.left = r.right = r.parent = -1;
    nodes[0] = r;
    splits[0].valid = 0;
    st->n_nodes = 1;
    st->done = 0;
    st->parent = -1;
    st->small_node = st->large_node = -1;
    st->n_sample = count;
    st->max_abs_g_bits = 0ull;
    st->max_h_bits = 0ull;
}

__global__ void iota_kernel(int32_t* rows, int n) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) rows[k] = k;
}

__global__ void scales_reduce_kernel(const int32_t* __restrict__ rows, const double* __restrict__ g,
                                     const double* __restrict__ h, const uint8_t* __restrict__ goss_flag,
                                     double goss_scale, DevTreeState* st) {
    const int count = st->n_sample;
    double mg = 0.0, mh = 0.0;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x) {
        const int r = rows[k];
        double gv = fabs(g[r]), hv = fabs(h[r]);
        if (goss_flag != nullptr && goss_flag[r] == 2) {
            gv = fabs(g[r] * goss_scale);
            hv = fabs(h[r] * goss_scale);
        }
        mg = fmax(mg, gv);
        mh = fmax(mh, hv);
    }
    for (int o = 16; o > 0; o >>= 1) {
        mg = fmax(mg, __shfl_xor_sync(0xffffffffu, mg, o));
        mh = fmax(mh, __shfl_xor_sync(0xffffffffu, mh, o));
    }
    if ((threadIdx.x & 31) == 0) {
        // Non-negative doubles order like their bit patterns.
        atomicMax(&st->max_abs_g_bits, static_cast<unsigned long long>(__double_as_longlong(mg)));
        atomicMax(&st->max_h_bits, static_cast<unsigned long long>(__double_as_longlong(mh)));
    }
}

__device__ int shift_for(double max_abs, int count) {
    if (!(max_abs > 0.0) || count <= 0) return 0;
    int clog = 0;
    while ((1ll << clog) < static_cast<long long>(count)) ++clog;
    const int e = ilogb(max_abs);
    int s = 61 - (e + 1) - clog;
    return max(-1000, min(1000, s));
}

__global__ void scales_finalize_kernel(DevTreeState* st) {
    const double mg = __longlong_as_double(static_cast<long long>(st->max_abs_g_bits));
    const double mh = __longlong_as_double(static_cast<long long>(st->max_h_bits));
    st->gshift = shift_for(mg, st->n_sample);
    st->hshift = shift_for(mh, st->n_sample);
    st->gscale = ldexp(1.0, st->gshift);
    st->hscale = ldexp(1.0, st->hshift);
    st->inv_gscale = ldexp(1.0, -st->gshift);
    st->inv_hscale = ldexp(1.0, -st->hshift);
}

template <int FG>
size_t hist_smem() {
    return static_cast<size_t>(FG) * kBins * (8 + 8 + 4);
}

template <int FG, typename K>
void set_smem(K kern) {
    check(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               static_cast<int>(hist_smem<FG>())),
          "hist smem attr");
}

}  // namespace

constexpr int kFG = 16;

void launch_hist_node(const uint8_t* codes, int stride, int n_f, int32_t* const* rows,
                      const DevNode* nodes, const DevTreeState* st, int node, const double* g,
                      const double* h, const uint8_t* goss_flag, double goss_scale, HistSlotPtrs hs,
                      int grid_rows, unsigned long long* rows_counter, cudaStream_t s) {
    set_smem<kFG>(hist_node_kernel<kFG>);
    dim3 grid((n_f + kFG - 1) / kFG, max(1, grid_rows));
    hist_node_kernel<kFG><<<grid, kHistThreads, hist_smem<kFG>(), s>>>(
        codes, stride, n_f, rows[0], rows[1], nodes, st, node, g, h, goss_flag, goss_scale, hs, rows_counter);
    check(cudaGetLastError(), "hist_node launch");
}

void launch_hist_rows(const uint8_t* codes, int stride, int n_f, const int32_t* rows, int n_rows,
                      const double* g, const double* h, int gshift, int hshift, long long* G,
                      long long* H, int* C, cudaStream_t s) {
    static bool init = false;
    if (!init) {
        set_smem<kFG>(hist_rows_kernel<kFG>);
        init = true;
    }
    if (n_rows <= 0) return;
    const int need = (n_rows + kMinRowsPerCta - 1) / kMinRowsPerCta;
    const int groups = (n_f + kFG - 1) / kFG;
    const int grid_rows = max(1, min(need, (148 * 4 + groups - 1) / groups));
    dim3 grid(groups, grid_rows);
    hist_rows_kernel<kFG><<<grid, kHistThreads, hist_smem<kFG>(), s>>>(
        codes, stride, n_f, rows, n_rows, g, h, std::ldexp(1.0, gshift), std::ldexp(1.0, hshift), G, H, C);
    check(cudaGetLastError(), "hist_rows launch");
}

int hist_grid_rows(int n_f, int max_rows) {
    const int groups = (n_f + kFG - 1) / kFG;
    const int need = (max_rows + kMinRowsPerCta - 1) / kMinRowsPerCta;
    return std::max(1, std::min(need, (148 * 4 + groups - 1) / groups));
}

void launch_hist_subtract(const DevTreeState* st, HistSlotPtrs hs, cudaStream_t s) {
    const int blocks = static_cast<int>(std::min<size_t>(296, (hs.slot_elems + 255) / 256));
    hist_subtract_kernel<<<blocks, 256, 0, s>>>(st, hs);
    check(cudaGetLastError(), "hist_subtract launch");
}

void launch_tree_init(DevNode* nodes, DevSplit* splits, DevTreeState* st, int n_sample_host,
                      int use_dev_count, cudaStream_t s) {
    tree_init_kernel<<<1, 1, 0, s>>>(nodes, splits, st, n_sample_host, use_dev_count);
    check(cudaGetLastError(), "tree_init launch");
}

void launch_iota_rows(int32_t* rows, int n, cudaStream_t s) {
    iota_kernel<<<592, 256, 0, s>>>(rows, n);
    check(cudaGetLastError(), "iota launch");
}

void launch_scales(const int32_t* rows, const double* g, const double* h, const uint8_t* goss_flag,
                   double goss_scale, DevTreeState* st, int max_rows, cudaStream_t s) {
    const int blocks = std::max(1, std::min(1184, (max_rows + 255) / 256));
    scales_reduce_kernel<<<blocks, 256, 0, s>>>(rows, g, h, goss_flag, goss_scale, st);
    check(cudaGetLastError(), "scales launch");
    scales_finalize_kernel<<<1, 1, 0, s>>>(st);
    check(cudaGetLastError(), "scales_finalize launch");
}

}  // namespace tgb
