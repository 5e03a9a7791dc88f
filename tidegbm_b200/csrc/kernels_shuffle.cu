// Prefixes of libstdc++'s std::shuffle on the device.
//
// std::shuffle over m >= 2^16 elements with std::mt19937 makes one draw j_t in [0, t]
// per t = 1 .. m-1 and swaps a[t] with a[j_t].  Position t is untouched before step t,
// so the step is a[t] = a[j_t]; a[j_t] = t.  For a kept slot p < keep this gives:
//   - if some step t writes p (j_t = p), the slot ends with the last such t;
//   - otherwise (p > 0) it keeps what step p moved in: the value of slot j_p after
//     step p-1.  "The value of slot q after step s" is again the last t <= s with
//     j_t = q, or, if there is none, the value of slot j_q after step q-1 (slot 0
//     starts as 0).  q falls at every step, and only draws t < keep take part.
// So the prefix needs no sequential swaps:
//   shuffle_draw_kernel     one CTA per range runs the generator: last[j] = max t over
//                           draws j < keep; the head draws (t < keep) also record
//                           head[t] = j and count cnt[j]
//   shuffle_scan_kernel     cnt -> bucket ends (one CTA per range)
//   shuffle_bucket_kernel   bucket q lists the head steps t with j_t = q
//   shuffle_resolve_kernel  every slot: last[p], else the walk above, answered from the
//                           buckets; written over last[p]
// The generator is MT19937 (Matsumoto & Nishimura, ACM TOMACS 8(1), 1998), seeded as
// std::mt19937(seed) is, with the 624-word state in shared memory, one thread per word.
// A refill is the recurrence x[k+624] = x[k+397] ^ mix(x[k], x[k+1]); with
// a[k] = mix(old[k], old[k+1]) (^ old[k+397] for k < 227) the new words are
// a[k] ^ a[k-227] ^ a[k-454] (terms with negative index omitted), and word 623 mixes
// with the new word 0: one shared-memory pass and one barrier per 624 words.
// Word q of a block serves draw t + q.  Lemire's method (the one libstdc++'s
// uniform_int_distribution uses for a 32-bit generator) rejects a word when the low
// half of w * (t + 1) is below 2^32 mod (t + 1); that draw then takes the next word,
// shifting the later ones by one.  The block tests all its words at once; at the first
// rejected word the draws before it are committed and the rest are re-tested with the
// shift.  Rejections happen with probability below (t + 1) / 2^32.
#include "tgb_internal.h"

#include <cub/block/block_scan.cuh>

namespace tgb {

namespace {

constexpr int kMtN = 624;
constexpr int kDrawThreads = 640;
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;

__device__ __forceinline__ uint32_t mt_mix(uint32_t hi, uint32_t lo) {
    const uint32_t y = (hi & 0x80000000u) | (lo & 0x7fffffffu);
    return (y >> 1) ^ ((0u - (y & 1u)) & 0x9908b0dfu);
}

__device__ __forceinline__ uint32_t mt_temper(uint32_t v) {
    v ^= v >> 11;
    v ^= (v << 7) & 0x9d2c5680u;
    v ^= (v << 15) & 0xefc60000u;
    v ^= v >> 18;
    return v;
}

// Range r: std::mt19937(seeds[r]) and draws t = 1 .. ms[r]-1 (ms[r] = 0: the range is
// not handled here).  last/head hold keep entries per range, cnt keep + 1.  A range
// whose refills exceed twice the expected count sets *err and stops.
__global__ void __launch_bounds__(kDrawThreads)
    shuffle_draw_kernel(const uint32_t* __restrict__ seeds, const long long* __restrict__ ms, int keep,
                        int32_t* __restrict__ last, int32_t* __restrict__ head, int32_t* __restrict__ cnt,
                        int* __restrict__ err) {
    __shared__ uint32_t st[kMtN];
    __shared__ uint32_t a[kMtN];
    __shared__ int first;
    const int r = blockIdx.x;
    const long long m = ms[r];
    if (m < 2 || keep <= 0) return;
    const int t = threadIdx.x;
    if (t == 0) {  // std::mt19937's seeding recurrence
        uint32_t x = seeds[r];
        st[0] = x;
        for (int k = 1; k < kMtN; ++k) {
            x = 1812433253u * (x ^ (x >> 30)) + static_cast<uint32_t>(k);
            st[k] = x;
        }
    }
    __syncthreads();
    int32_t* lst = last + static_cast<size_t>(r) * keep;
    int32_t* hd = head + static_cast<size_t>(r) * keep;
    int32_t* ct = cnt + static_cast<size_t>(r) * (keep + 1);
    const uint32_t K = static_cast<uint32_t>(keep);
    long long i = 1;  // the next draw
    int pos = kMtN;   // the next unused word of the block
    uint32_t w = 0;
    long long refills_left = 2 * (m / kMtN) + 16;
    while (i < m) {
        if (pos >= kMtN) {
            if (--refills_left < 0) {
                if (t == 0) atomicExch(err, 1);
                return;
            }
            uint32_t ak = 0;
            if (t < kMtN - 1) {
                ak = mt_mix(st[t], st[t + 1]);
                if (t < 227) ak ^= st[t + 397];
            } else if (t == kMtN - 1) {
                ak = mt_mix(st[kMtN - 1], st[397] ^ mt_mix(st[0], st[1]));
            }
            if (t < kMtN) a[t] = ak;
            __syncthreads();
            if (t < kMtN) {
                uint32_t nk = ak;
                if (t >= 227) nk ^= a[t - 227];
                if (t >= 454) nk ^= a[t - 454];
                st[t] = nk;  // read again only after the barrier of the draw loop
                w = mt_temper(nk);
            }
            pos = 0;
        }
        while (true) {
            const long long d = i + (t - pos);
            const bool live = t >= pos && t < kMtN && d < m;
            const uint32_t range = static_cast<uint32_t>(d + 1);
            const uint64_t p = static_cast<uint64_t>(w) * range;
            const uint32_t low = static_cast<uint32_t>(p);
            const bool rej = live && low < range && low < (0u - range) % range;
            const bool any = __syncthreads_or(rej);
            int fr = kMtN;
            if (any) {
                if (t == 0) first = kMtN;
                __syncthreads();
                if (rej) atomicMin(&first, t);
                __syncthreads();
                fr = first;
            }
            const uint32_t j = static_cast<uint32_t>(p >> 32);
            if (live && t < fr && j < K) {
                atomicMax(lst + j, static_cast<int>(d));
                if (d < keep) {
                    hd[d] = static_cast<int32_t>(j);
                    atomicAdd(ct + j, 1);
                }
            }
            if (!any) {
                const long long used = min(static_cast<long long>(kMtN - pos), m - i);
                i += used;
                pos += static_cast<int>(used);
                break;
            }
            i += fr - pos;  // the rejected word is consumed; draw i + (fr - pos) takes the next word
            pos = fr + 1;
            if (pos >= kMtN) break;
        }
    }
}

// cnt[r][0..keep) -> inclusive prefix sums (bucket ends); cnt[r][keep] = keep - 1 draws.
__global__ void __launch_bounds__(kScanThreads)
    shuffle_scan_kernel(const long long* __restrict__ ms, int keep, int32_t* __restrict__ cnt) {
    using Scan = cub::BlockScan<int, kScanThreads>;
    __shared__ typename Scan::TempStorage tmp;
    const int r = blockIdx.x;
    if (ms[r] < 2) return;
    int32_t* ct = cnt + static_cast<size_t>(r) * (keep + 1);
    int carry = 0;
    for (int base = 0; base < keep; base += kScanThreads * kScanItems) {
        int v[kScanItems];
        const int i0 = base + threadIdx.x * kScanItems;
#pragma unroll
        for (int k = 0; k < kScanItems; ++k) v[k] = i0 + k < keep ? ct[i0 + k] : 0;
        int total;
        Scan(tmp).InclusiveSum(v, v, total);
#pragma unroll
        for (int k = 0; k < kScanItems; ++k)
            if (i0 + k < keep) ct[i0 + k] = v[k] + carry;
        carry += total;
        __syncthreads();  // tmp is reused by the next tile
    }
    if (threadIdx.x == 0) ct[keep] = keep - 1;
}

// Head step t (1 <= t < keep) goes into bucket head[t]; afterwards cnt[q] is the start of
// bucket q and cnt[q + 1] its end.
__global__ void shuffle_bucket_kernel(const long long* __restrict__ ms, int keep, const int32_t* __restrict__ head,
                                      int32_t* __restrict__ cnt, int32_t* __restrict__ items) {
    const int r = blockIdx.y;
    if (ms[r] < 2) return;
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < 1 || t >= keep) return;
    const size_t o = static_cast<size_t>(r) * keep;
    const int q = head[o + t];
    if (q < 0 || q >= keep) return;  // only after a draw run that stopped early (reported by *err)
    const int at = atomicSub(cnt + static_cast<size_t>(r) * (keep + 1) + q, 1) - 1;
    if (at >= 0 && at < keep - 1) items[o + at] = t;
}

// Slot p: last[p] when a step wrote it, else the walk over earlier slots.
__global__ void shuffle_resolve_kernel(const long long* __restrict__ ms, int keep, int32_t* __restrict__ last,
                                       const int32_t* __restrict__ head, const int32_t* __restrict__ cnt,
                                       const int32_t* __restrict__ items) {
    const int r = blockIdx.y;
    if (ms[r] < 1) return;
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= keep) return;
    const size_t o = static_cast<size_t>(r) * keep;
    int32_t* lst = last + o;
    if (lst[p] >= 0) return;
    if (p == 0) {  // slot 0 starts as 0 (a range with ms[r] == 1 has only this slot)
        lst[0] = 0;
        return;
    }
    const int32_t* hd = head + o;
    const int32_t* ct = cnt + static_cast<size_t>(r) * (keep + 1);
    const int32_t* it = items + o;
    int q = hd[p];
    int s = p - 1;
    int out = 0;
    // q falls at every step; the index checks only matter after a draw run that stopped
    // early (reported by *err), when head and cnt are incomplete
    for (int guard = 0; guard <= keep && q >= 0 && q < keep; ++guard) {
        int best = -1;
        const int k1 = min(ct[q + 1], keep - 1);
        for (int k = max(ct[q], 0); k < k1; ++k) {
            const int v = it[k];
            if (v <= s && v > best) best = v;
        }
        if (best >= 0) {
            out = best;
            break;
        }
        if (q == 0) break;  // slot 0 starts as 0
        s = q - 1;
        q = hd[q];
    }
    lst[p] = out;
}

}  // namespace

void launch_shuffle_prefix(const uint32_t* seeds, const long long* ms, int n_ranges, int keep, int32_t* out,
                           int32_t* head, int32_t* cnt, int32_t* items, int* err, cudaStream_t s) {
    if (n_ranges <= 0 || keep <= 0) return;
    check(cudaMemsetAsync(out, 0xff, sizeof(int32_t) * static_cast<size_t>(n_ranges) * keep, s), "slots reset");
    check(cudaMemsetAsync(cnt, 0, sizeof(int32_t) * static_cast<size_t>(n_ranges) * (keep + 1), s), "counts reset");
    shuffle_draw_kernel<<<n_ranges, kDrawThreads, 0, s>>>(seeds, ms, keep, out, head, cnt, err);
    check(cudaGetLastError(), "shuffle_draw launch");
    shuffle_scan_kernel<<<n_ranges, kScanThreads, 0, s>>>(ms, keep, cnt);
    check(cudaGetLastError(), "shuffle_scan launch");
    const dim3 grid((keep + 255) / 256, n_ranges);
    shuffle_bucket_kernel<<<grid, 256, 0, s>>>(ms, keep, head, cnt, items);
    check(cudaGetLastError(), "shuffle_bucket launch");
    shuffle_resolve_kernel<<<grid, 256, 0, s>>>(ms, keep, out, head, cnt, items);
    check(cudaGetLastError(), "shuffle_resolve launch");
}

}  // namespace tgb
