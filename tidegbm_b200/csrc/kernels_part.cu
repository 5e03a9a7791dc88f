// Stable row partition of a node's row list.  Restates split_indices
// (cpp/src/tree.cpp:68-91) for axis splits: a row goes left when its code is
// 0 (missing) and missing_go_left, or when 0 < code <= threshold; both children
// keep the parent's (ascending) row order.
//
// Two launches over fixed 2048-row tiles:
//   count    per-tile number of left rows
//   scatter  per tile: the tile's left offset and the node's left total from the tile
//            counts (a block reduction; no separate scan pass), in-tile stable ranks
//            from ballots, rows written to the other ping-pong buffer.  Block 0 also
//            records n_left and, in tree mode, fills the children's segments and picks
//            the smaller child (left on ties, cpp/src/tree.cpp:423).
// A thread owns 8 rows of a tile (rows base + i*256 + tid), so each of the kernels
// issues all its row-id loads, then all its code loads, before it waits: two memory
// round trips per tile rather than one per 256 rows.
// In tree mode the job (row segment, feature, threshold, missing direction) is read
// from the node table at st->parent, so the sequence runs without host
// synchronisation; grids are sized for the largest node and exit early.  The same
// kernels compact flagged rows (GOSS sample) in index order.
#include "tgb_internal.h"

#include <stdexcept>
#include <string>

namespace tgb {

namespace {

constexpr int kPartThreads = 256;
constexpr int kPartWarps = kPartThreads / 32;
constexpr int kPartPer = kPartTile / kPartThreads;  // rows per thread per tile (8)
static_assert(kPartTile == kPartPer * kPartThreads, "tile shape");

// Resolves the job: tree mode (st != nullptr) from the node table, else the given one.
__device__ __forceinline__ bool resolve_job(const PartJob& given, const DevNode* __restrict__ nodes,
                                            const DevTreeState* __restrict__ st, int32_t* rows0, int32_t* rows1,
                                            PartJob& j) {
    j = given;
    if (st == nullptr) return true;
    if (st->done || st->parent < 0) return false;
    const DevNode& P = nodes[st->parent];
    j.in = (P.buf ? rows1 : rows0) + P.start;
    j.out = (P.buf ? rows0 : rows1) + P.start;
    j.count = P.count;
    j.feature = P.feature;
    j.threshold = P.threshold;
    j.missing_left = P.missing_left;
    return true;
}

// Loads the tile's rows (8 per thread) and their left/right decisions.
__device__ __forceinline__ void load_tile(const uint8_t* __restrict__ codes, int stride, const PartJob& j, int base,
                                          int end, int32_t (&row)[kPartPer], bool (&left)[kPartPer]) {
#pragma unroll
    for (int i = 0; i < kPartPer; ++i) {
        const int k = base + i * kPartThreads + threadIdx.x;
        row[i] = k < end ? (j.in ? j.in[k] : k) : -1;
    }
    int b[kPartPer];
#pragma unroll
    for (int i = 0; i < kPartPer; ++i) {
        b[i] = 0;
        if (row[i] < 0) continue;
        if (j.flag) b[i] = j.flag[row[i]];
        else if (j.col) b[i] = j.col[static_cast<size_t>(j.feature) * j.col_n + row[i]];
        else b[i] = codes[static_cast<size_t>(row[i]) * stride + j.feature];
    }
#pragma unroll
    for (int i = 0; i < kPartPer; ++i) {
        if (row[i] < 0) left[i] = false;
        else if (j.flag) left[i] = b[i] != 0;
        else left[i] = b[i] == 0 ? j.missing_left != 0 : b[i] <= j.threshold;
    }
}

__device__ __forceinline__ int block_sum(int v, int* red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    int t = 0;
#pragma unroll
    for (int w = 0; w < kPartWarps; ++w) t += red[w];
    return t;
}

__global__ void __launch_bounds__(kPartThreads)
    part_count_kernel(const uint8_t* __restrict__ codes, int stride, PartJob given, const DevNode* __restrict__ nodes,
                      const DevTreeState* __restrict__ st, int32_t* rows0, int32_t* rows1,
                      int* __restrict__ tile_counts) {
    pdl_wait();
    pdl_trigger();
    PartJob j;
    if (!resolve_job(given, nodes, st, rows0, rows1, j)) return;
    __shared__ int red[kPartWarps];
    const int n_tiles = (j.count + kPartTile - 1) / kPartTile;
    for (int t = blockIdx.x; t < n_tiles; t += gridDim.x) {
        const int base = t * kPartTile;
        const int end = min(base + kPartTile, j.count);
        int32_t row[kPartPer];
        bool left[kPartPer];
        load_tile(codes, stride, j, base, end, row, left);
        int cnt = 0;
#pragma unroll
        for (int i = 0; i < kPartPer; ++i) cnt += left[i] ? 1 : 0;
        cnt = block_sum(cnt, red);
        if (threadIdx.x == 0) tile_counts[t] = cnt;
    }
}

__global__ void __launch_bounds__(kPartThreads)
    part_scatter_kernel(const uint8_t* __restrict__ codes, int stride, PartJob given, DevNode* __restrict__ nodes,
                        DevTreeState* __restrict__ st, int32_t* rows0, int32_t* rows1,
                        const int* __restrict__ tile_counts) {
    pdl_wait();
    pdl_trigger();
    PartJob j;
    if (!resolve_job(given, nodes, st, rows0, rows1, j)) return;
    __shared__ int red[kPartWarps];
    __shared__ int wc[kPartPer * kPartWarps];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned lt_mask = (1u << lane) - 1u;
    const int n_tiles = (j.count + kPartTile - 1) / kPartTile;
    if (static_cast<int>(blockIdx.x) >= n_tiles && blockIdx.x != 0) return;
    // node total of left rows
    int tot = 0;
    for (int k = threadIdx.x; k < n_tiles; k += kPartThreads) tot += tile_counts[k];
    const int n_left = block_sum(tot, red);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        if (j.n_left_out) *j.n_left_out = n_left;
        if (st != nullptr) {
            DevNode& P = nodes[st->parent];
            DevNode& L = nodes[P.left];
            DevNode& R = nodes[P.right];
            L.start = P.start;
            L.count = n_left;
            R.start = P.start + n_left;
            R.count = P.count - n_left;
            st->n_left = n_left;
            const bool left_small = L.count <= R.count;  // cpp/src/tree.cpp:423
            st->small_node = left_small ? P.left : P.right;
            st->large_node = left_small ? P.right : P.left;
        }
    }
    int prev_tiles = 0, left0 = 0;  // running prefix over this block's tiles
    for (int t = blockIdx.x; t < n_tiles; t += gridDim.x) {
        int part = 0;
        for (int k = prev_tiles + threadIdx.x; k < t; k += kPartThreads) part += tile_counts[k];
        left0 += block_sum(part, red);
        prev_tiles = t;
        const int base = t * kPartTile;
        const int end = min(base + kPartTile, j.count);
        int32_t row[kPartPer];
        bool left[kPartPer];
        load_tile(codes, stride, j, base, end, row, left);
        unsigned bal[kPartPer];
#pragma unroll
        for (int i = 0; i < kPartPer; ++i) {
            bal[i] = __ballot_sync(0xffffffffu, left[i]);
            if (lane == 0) wc[i * kPartWarps + warp] = __popc(bal[i]);
        }
        __syncthreads();
        // exclusive prefix of left rows over (i, warp) in tile order
        int before = 0;
        int excl[kPartPer];
#pragma unroll
        for (int i = 0; i < kPartPer; ++i) {
            int e = before;
            for (int w = 0; w < kPartWarps; ++w) {
                const int c = wc[i * kPartWarps + w];
                if (w < warp) e += c;
                before += c;
            }
            excl[i] = e;
        }
#pragma unroll
        for (int i = 0; i < kPartPer; ++i) {
            if (row[i] < 0) continue;
            const int k = base + i * kPartThreads + threadIdx.x;
            const int lrank = excl[i] + __popc(bal[i] & lt_mask);  // lefts before k in the tile
            if (left[i]) {
                j.out[left0 + lrank] = row[i];
            } else if (!j.left_only) {
                const int rrank = (k - base) - lrank;
                j.out[n_left + (base - left0) + rrank] = row[i];
            }
        }
        __syncthreads();  // wc reuse
    }
}

void run_partition(const uint8_t* codes, int stride, const PartJob& j, DevNode* nodes, DevTreeState* st,
                   int32_t* rows0, int32_t* rows1, int* tile_counts, int max_tiles, cudaStream_t s) {
    const int grid = max(1, min(max_tiles, 148 * 8));
    launch_pdl(part_count_kernel, dim3(grid), dim3(kPartThreads), 0, s, "part_count launch", codes, stride, j, nodes,
               st, rows0, rows1, tile_counts);
    launch_pdl(part_scatter_kernel, dim3(grid), dim3(kPartThreads), 0, s, "part_scatter launch", codes, stride, j,
               nodes, st, rows0, rows1, static_cast<const int*>(tile_counts));
}

}  // namespace

void launch_partition(const uint8_t* codes, int stride, const uint8_t* codes_col, long long n_rows_total,
                      int32_t* const* rows, DevNode* nodes, DevTreeState* st, int* tile_counts, int max_tiles,
                      cudaStream_t s) {
    PartJob j{};
    j.col = codes_col;
    j.col_n = n_rows_total;
    run_partition(codes, stride, j, nodes, st, rows[0], rows[1], tile_counts, max_tiles, s);
}

void launch_partition_rows(const uint8_t* codes, int stride, const int32_t* rows, int n_rows, int feature,
                           int threshold, int missing_left, int32_t* out, int* n_left_dev, int* tile_counts,
                           cudaStream_t s) {
    PartJob j{};
    j.in = rows;
    j.out = out;
    j.count = n_rows;
    j.feature = feature;
    j.threshold = threshold;
    j.missing_left = missing_left;
    j.n_left_out = n_left_dev;
    if (n_rows <= 0) {
        if (n_left_dev) check(cudaMemsetAsync(n_left_dev, 0, sizeof(int), s), "n_left reset");
        return;
    }
    run_partition(codes, stride, j, nullptr, nullptr, nullptr, nullptr, tile_counts,
                  (n_rows + kPartTile - 1) / kPartTile, s);
}

void launch_compact_flagged(const uint8_t* flag, int n, int32_t* out, int* n_out_dev, int* tile_counts,
                            cudaStream_t s) {
    PartJob j{};
    j.in = nullptr;  // rows are 0..n-1
    j.out = out;
    j.count = n;
    j.flag = flag;
    j.left_only = 1;
    j.n_left_out = n_out_dev;
    run_partition(nullptr, 0, j, nullptr, nullptr, nullptr, nullptr, tile_counts, (n + kPartTile - 1) / kPartTile, s);
}

// ---- partition without caller-provided scratch -------------------------------------
//
// Some callers cannot hand this library a device workspace: for example a serving
// process that reserves all device memory when it starts and treats any later
// cudaMalloc as a fault (cudaMalloc can block on the whole device and can fail under
// memory pressure), or a binding that only passes the input and output buffers of a
// call.  For them the partition's only scratch, the per-tile counts of left rows, lives
// in this fixed device array instead (the job itself travels as a kernel argument).
// Every GPU that loads the library keeps the array (32 KB) until the process exits.
// All calls on a device share it and it keeps whatever the last call left: the count
// kernel writes every tile count the scatter kernel reads, so nothing has to start at
// zero, but two calls whose kernels overlap on the GPU (different streams, or
// different host threads) race on it.
constexpr int kNoAllocMaxRows = 1 << 24;
constexpr int kNoAllocTiles = kNoAllocMaxRows / kPartTile;
constexpr size_t kNoAllocBytes = sizeof(int) * kNoAllocTiles;

static __device__ __align__(256) unsigned char g_partition_scratch[kNoAllocBytes];

namespace {
// Device address of g_partition_scratch on the current device.  Host code only sees a
// host-side stand-in under that name, so the address is looked up with the device
// current.  The lookup is repeated on every call (it is cheap once the module is loaded),
// so it stays right after a cudaDeviceReset; the first call on a device may load the
// module, which is why that first call must not happen inside a stream capture.
unsigned char* partition_scratch_address() {
    void* p = nullptr;
    check(cudaGetSymbolAddress(&p, g_partition_scratch), "cudaGetSymbolAddress(partition scratch)");
    return static_cast<unsigned char*>(p);
}
}  // namespace

int partition_noalloc_max_rows() { return kNoAllocMaxRows; }

void launch_partition_rows_noalloc(const uint8_t* codes, int stride, const int32_t* rows, int n_rows, int feature,
                                   int threshold, int missing_left, int32_t* out, int* n_left_dev, cudaStream_t s) {
    if (n_rows < 0 || n_rows > kNoAllocMaxRows)
        throw std::runtime_error("partition without workspace: n_rows must be in [0, " +
                                 std::to_string(kNoAllocMaxRows) + "], got " + std::to_string(n_rows));
    unsigned char* base = partition_scratch_address();
    launch_partition_rows(codes, stride, rows, n_rows, feature, threshold, missing_left, out, n_left_dev,
                          reinterpret_cast<int*>(base), s);
}

}  // namespace tgb
