// Stable row partition of a node's row list.  Restates split_indices
// (cpp/src/tree.cpp:68-91) for axis splits: a row goes left when its code is
// 0 (missing) and missing_go_left, or when 0 < code <= threshold; both children
// keep the parent's (ascending) row order.
//
// Three launches over fixed 2048-row tiles:
//   count   per-tile number of left rows (warp ballot + popc)
//   scan    one CTA: exclusive scan of the tile counts -> tile offsets, n_left;
//           in tree mode it also fills the children's segments and picks the
//           smaller child (left on ties, cpp/src/tree.cpp:423)
//   scatter per tile: in-tile stable rank from ballots + a shared-memory scan over
//           the 8 warps, rows written to the other ping-pong buffer
// Grids are fixed (sized for the largest node) and read the job from device memory,
// so the sequence can run without host synchronisation.  The same kernels compact
// flagged rows (GOSS sample) in index order.
#include "tgb_internal.h"

#include <mutex>
#include <stdexcept>
#include <string>

namespace tgb {

namespace {

constexpr int kPartThreads = 256;
constexpr int kPartWarps = kPartThreads / 32;

__device__ __forceinline__ int32_t job_row(const PartJob& j, int k) { return j.in ? j.in[k] : k; }

__device__ __forceinline__ bool goes_left(const uint8_t* __restrict__ codes, int stride, int32_t r,
                                          const PartJob& j) {
    if (j.flag) return j.flag[r] != 0;
    const int b = j.col ? j.col[static_cast<size_t>(j.feature) * j.col_n + r]
                        : codes[static_cast<size_t>(r) * stride + j.feature];
    return b == 0 ? j.missing_left != 0 : b <= j.threshold;
}

__global__ void part_setup_tree_kernel(const DevNode* __restrict__ nodes, const DevTreeState* __restrict__ st,
                                       int32_t* rows0, int32_t* rows1, const uint8_t* col, long long col_n,
                                       PartJob* job) {
    PartJob j{};
    j.col = col;
    j.col_n = col_n;
    if (!st->done) {
        const DevNode& P = nodes[st->parent];
        j.in = (P.buf ? rows1 : rows0) + P.start;
        j.out = (P.buf ? rows0 : rows1) + P.start;
        j.count = P.count;
        j.feature = P.feature;
        j.threshold = P.threshold;
        j.missing_left = P.missing_left;
    }
    j.n_tiles = (j.count + kPartTile - 1) / kPartTile;
    *job = j;
}

__global__ void __launch_bounds__(kPartThreads)
    part_count_kernel(const uint8_t* __restrict__ codes, int stride, const PartJob* __restrict__ jp,
                      int* __restrict__ tile_counts) {
    const PartJob j = *jp;
    __shared__ int wsum[kPartWarps];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int t = blockIdx.x; t < j.n_tiles; t += gridDim.x) {
        const int base = t * kPartTile;
        const int end = min(base + kPartTile, j.count);
        int cnt = 0;
        for (int k = base + threadIdx.x; k < end; k += kPartThreads)
            cnt += goes_left(codes, stride, job_row(j, k), j) ? 1 : 0;
        for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
        if (lane == 0) wsum[warp] = cnt;
        __syncthreads();
        if (threadIdx.x == 0) {
            int s = 0;
            for (int w = 0; w < kPartWarps; ++w) s += wsum[w];
            tile_counts[t] = s;
        }
        __syncthreads();
    }
}

// One CTA of 1024 threads: exclusive scan of tile_counts in place.
__global__ void __launch_bounds__(1024)
    part_scan_kernel(PartJob* jp, int* __restrict__ tile_counts, DevNode* nodes, DevTreeState* st,
                     int tree_mode) {
    __shared__ int warp_tot[32];
    __shared__ int carry;
    const int nt = jp->n_tiles;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < nt; base += 1024) {
        const int k = base + threadIdx.x;
        const int v = k < nt ? tile_counts[k] : 0;
        int incl = v;
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
        }
        if (lane == 31) warp_tot[warp] = incl;
        __syncthreads();
        if (warp == 0) {
            int w = warp_tot[lane];
            for (int o = 1; o < 32; o <<= 1) {
                const int t = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= o) w += t;
            }
            warp_tot[lane] = w;  // inclusive over warps
        }
        __syncthreads();
        const int warp_excl = warp == 0 ? 0 : warp_tot[warp - 1];
        if (k < nt) tile_counts[k] = carry + warp_excl + incl - v;
        __syncthreads();
        if (threadIdx.x == 0) carry += warp_tot[31];
        __syncthreads();
    }
    if (threadIdx.x != 0) return;
    const int n_left = carry;
    jp->n_left = n_left;
    if (jp->n_left_out) *jp->n_left_out = n_left;
    if (!tree_mode || st->done) return;
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

__global__ void __launch_bounds__(kPartThreads)
    part_scatter_kernel(const uint8_t* __restrict__ codes, int stride, const PartJob* __restrict__ jp,
                        const int* __restrict__ tile_offsets) {
    const PartJob j = *jp;
    __shared__ int wcnt[kPartWarps];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned lt_mask = (1u << lane) - 1u;
    for (int t = blockIdx.x; t < j.n_tiles; t += gridDim.x) {
        const int base = t * kPartTile;
        const int end = min(base + kPartTile, j.count);
        const int left0 = tile_offsets[t];  // lefts before this tile
        int run_left = 0;                   // lefts earlier in this tile
        for (int r0 = base; r0 < end; r0 += kPartThreads) {
            const int k = r0 + threadIdx.x;
            const bool valid = k < end;
            int32_t row = 0;
            bool left = false;
            if (valid) {
                row = job_row(j, k);
                left = goes_left(codes, stride, row, j);
            }
            const unsigned bal = __ballot_sync(0xffffffffu, left);
            if (lane == 0) wcnt[warp] = __popc(bal);
            __syncthreads();
            int wexcl = 0, rtot = 0;
            for (int w = 0; w < kPartWarps; ++w) {
                const int c = wcnt[w];
                if (w < warp) wexcl += c;
                rtot += c;
            }
            if (valid) {
                const int lrank = run_left + wexcl + __popc(bal & lt_mask);  // lefts before k in tile
                if (left) {
                    j.out[left0 + lrank] = row;
                } else if (!j.left_only) {
                    const int rrank = (k - base) - lrank;
                    j.out[j.n_left + (base - left0) + rrank] = row;
                }
            }
            run_left += rtot;
            __syncthreads();
        }
    }
}

__global__ void part_setup_const_kernel(PartJob j, PartJob* job) { *job = j; }

void run_partition(const uint8_t* codes, int stride, PartJob* job, int* tile_counts, int max_tiles,
                   DevNode* nodes, DevTreeState* st, int tree_mode, cudaStream_t s) {
    const int grid = max(1, min(max_tiles, 148 * 8));
    part_count_kernel<<<grid, kPartThreads, 0, s>>>(codes, stride, job, tile_counts);
    check(cudaGetLastError(), "part_count launch");
    part_scan_kernel<<<1, 1024, 0, s>>>(job, tile_counts, nodes, st, tree_mode);
    check(cudaGetLastError(), "part_scan launch");
    part_scatter_kernel<<<grid, kPartThreads, 0, s>>>(codes, stride, job, tile_counts);
    check(cudaGetLastError(), "part_scatter launch");
}

}  // namespace

void launch_partition(const uint8_t* codes, int stride, const uint8_t* codes_col, long long n_rows_total,
                      int32_t* const* rows, DevNode* nodes, DevTreeState* st, int* tile_counts, int max_tiles,
                      void* job_mem, cudaStream_t s) {
    PartJob* job = static_cast<PartJob*>(job_mem);
    part_setup_tree_kernel<<<1, 1, 0, s>>>(nodes, st, rows[0], rows[1], codes_col, n_rows_total, job);
    check(cudaGetLastError(), "part_setup launch");
    run_partition(codes, stride, job, tile_counts, max_tiles, nodes, st, 1, s);
}

void launch_partition_rows(const uint8_t* codes, int stride, const int32_t* rows, int n_rows, int feature,
                           int threshold, int missing_left, int32_t* out, int* n_left_dev, int* tile_counts,
                           void* job_mem, cudaStream_t s) {
    PartJob j{};
    j.in = rows;
    j.out = out;
    j.count = n_rows;
    j.feature = feature;
    j.threshold = threshold;
    j.missing_left = missing_left;
    j.n_tiles = (n_rows + kPartTile - 1) / kPartTile;
    j.n_left_out = n_left_dev;
    PartJob* job = static_cast<PartJob*>(job_mem);
    part_setup_const_kernel<<<1, 1, 0, s>>>(j, job);
    check(cudaGetLastError(), "part_setup launch");
    run_partition(codes, stride, job, tile_counts, j.n_tiles, nullptr, nullptr, 0, s);
}

void launch_compact_flagged(const uint8_t* flag, int n, int32_t* out, int* n_out_dev, int* tile_counts,
                            void* job_mem, cudaStream_t s) {
    PartJob j{};
    j.in = nullptr;  // rows are 0..n-1
    j.out = out;
    j.count = n;
    j.flag = flag;
    j.left_only = 1;
    j.n_tiles = (n + kPartTile - 1) / kPartTile;
    j.n_left_out = n_out_dev;
    PartJob* job = static_cast<PartJob*>(job_mem);
    part_setup_const_kernel<<<1, 1, 0, s>>>(j, job);
    check(cudaGetLastError(), "compact_setup launch");
    run_partition(nullptr, 0, job, tile_counts, j.n_tiles, nullptr, nullptr, 0, s);
}

// ---- partition without caller-provided scratch -------------------------------------
//
// Some callers cannot hand this library a device workspace: for example a serving
// process that reserves all device memory when it starts and treats any later
// cudaMalloc as a fault (cudaMalloc can block on the whole device and can fail under
// memory pressure), or a binding that only passes the input and output buffers of a
// call.  For them the partition's scratch (one PartJob and the per-tile left counts)
// lives in this fixed device array instead.  Every GPU that loads the library keeps
// the array (about 33 KB) until the process exits.  All calls on a device share it and
// it keeps whatever the last call left: each call writes the job and every tile count
// it reads before reading them, so nothing has to start at zero, but two calls whose
// kernels overlap on the GPU (different streams, or different host threads) race on it.
constexpr int kNoAllocMaxRows = 1 << 24;
constexpr int kNoAllocTiles = kNoAllocMaxRows / kPartTile;
constexpr size_t kNoAllocJobBytes = 256;
constexpr size_t kNoAllocBytes = kNoAllocJobBytes + sizeof(int) * (kNoAllocTiles + 1);
static_assert(sizeof(PartJob) <= kNoAllocJobBytes, "job does not fit its slot");

static __device__ __align__(256) unsigned char g_partition_scratch[kNoAllocBytes];

namespace {
constexpr int kNoAllocMaxDevices = 64;
void* g_scratch_addr[kNoAllocMaxDevices] = {};
std::mutex g_scratch_mu;

// Device address of g_partition_scratch on the current device.  Host code only sees a
// host-side stand-in under that name, so the address is looked up once per device,
// with the device current, on the first call there.
unsigned char* partition_scratch_address() {
    int dev = 0;
    check(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev < 0 || dev >= kNoAllocMaxDevices) throw std::runtime_error("device index out of range");
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (g_scratch_addr[dev] == nullptr) {
        void* p = nullptr;
        check(cudaGetSymbolAddress(&p, g_partition_scratch), "cudaGetSymbolAddress(partition scratch)");
        g_scratch_addr[dev] = p;
    }
    return static_cast<unsigned char*>(g_scratch_addr[dev]);
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
                          reinterpret_cast<int*>(base + kNoAllocJobBytes), base, s);
}

}  // namespace tgb
