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
//   keys = bit pattern of |g| (non-negative doubles order like their bits),
//   radix sort descending (stable; rows with equal |g| keep index order),
//   flag[order[p]] = 1 for p < n_top, flag[order[n_top + rest_pos[p]]] = 2,
//   compaction of flagged rows in index order -> the tree's root row list.
// The hist kernel multiplies g and h of flag-2 rows by the GOSS scale on the fly.
#include "tgb_internal.h"

#include <cub/device/device_radix_sort.cuh>

namespace tgb {

namespace {

__global__ void goss_keys_kernel(const double* __restrict__ g, int n, unsigned long long* __restrict__ keys,
                                 int32_t* __restrict__ vals) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        keys[i] = static_cast<unsigned long long>(__double_as_longlong(fabs(g[i])));
        vals[i] = i;
    }
}

__global__ void goss_mark_kernel(const int32_t* __restrict__ order, int n_top, int n_other,
                                 const int32_t* __restrict__ rest_pos, uint8_t* __restrict__ flag) {
    const int total = n_top + n_other;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < total; p += gridDim.x * blockDim.x) {
        if (p < n_top) flag[order[p]] = 1;
        else flag[order[n_top + rest_pos[p - n_top]]] = 2;
    }
}

}  // namespace

size_t goss_cub_bytes(int n) {
    size_t bytes = 0;
    check(cub::DeviceRadixSort::SortPairsDescending(nullptr, bytes, static_cast<unsigned long long*>(nullptr),
                                                    static_cast<unsigned long long*>(nullptr),
                                                    static_cast<int32_t*>(nullptr), static_cast<int32_t*>(nullptr),
                                                    n),
          "cub sizing");
    return bytes;
}

void launch_goss_select(const double* g, int n, int n_top, int n_other, const int32_t* rest_pos, GossWork& w,
                        uint8_t* goss_flag, int32_t* rows0, int* tile_counts, DevTreeState* st, cudaStream_t s) {
    const int blocks = std::max(1, std::min(2368, (n + 255) / 256));
    goss_keys_kernel<<<blocks, 256, 0, s>>>(g, n, w.keys_in, w.vals_in);
    check(cudaGetLastError(), "goss_keys launch");
    size_t tmp = w.cub_tmp_bytes;
    check(cub::DeviceRadixSort::SortPairsDescending(w.cub_tmp, tmp, w.keys_in, w.keys_out, w.vals_in,
                                                    w.vals_out, n, 0, 64, s),
          "goss sort");
    check(cudaMemsetAsync(goss_flag, 0, static_cast<size_t>(n), s), "goss flag reset");
    goss_mark_kernel<<<std::max(1, std::min(2368, (n_top + n_other + 255) / 256)), 256, 0, s>>>(
        w.vals_out, n_top, n_other, rest_pos, goss_flag);
    check(cudaGetLastError(), "goss_mark launch");
    launch_compact_flagged(goss_flag, n, rows0, &st->n_sample, tile_counts, s);
}

}  // namespace tgb
