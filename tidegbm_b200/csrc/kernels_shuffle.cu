// The tail of a std::shuffle prefix on the device (sampling.h has the host half).
//
// libstdc++'s std::shuffle over m >= 2^16 elements with std::mt19937 makes one
// draw j in [0, i] per i = 1 .. m-1 and swaps a[i] with a[j].  Once i >= keep, a
// draw only matters for the prefix when j < keep, and then it writes element i into
// slot j (the element there leaves the prefix for good).  The head (i < keep) runs on
// the host; this kernel makes the tail draws of one range per CTA, continuing the
// host generator's MT19937 stream exactly:
//   - the 624-word state lives in shared memory, one thread per word.  A refill is
//     the recurrence x[k+624] = x[k+397] ^ mix(x[k], x[k+1]) of Matsumoto & Nishimura
//     (ACM TOMACS 8(1), 1998); with a[k] = mix(old[k], old[k+1]) (^ old[k+397] for
//     k < 227) the new words are a[k] ^ a[k-227] ^ a[k-454] (terms with negative
//     index omitted), and word 623 mixes with the new word 0.  So a refill is one
//     shared-memory pass and one barrier.
//   - word q of the block serves draw i + q.  Lemire's method (the one libstdc++'s
//     uniform_int_distribution uses for a 32-bit generator) rejects a word when the
//     low half of w * (i + 1) is below 2^32 mod (i + 1); the draw then takes the next
//     word, which shifts every later word by one.  The block tests all its words at
//     once; at the first rejected word the draws before it are committed and the rest
//     are re-tested with the shift.  Rejections happen with probability below
//     (i + 1) / 2^32, well under one per block for ranges below 10^8.
//   - a committed draw j < keep writes slot j with atomicMax: later draws have larger
//     i, and every head entry is below keep <= i, so the maximum is the last write,
//     as in the sequential shuffle.
#include "tgb_internal.h"

namespace tgb {

namespace {

constexpr int kMtN = 624;
constexpr int kTailThreads = 640;

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

// One CTA per range r: state mt[r*625 .. +624) and position mt[r*625 + 624] of the
// host generator after the head, draws i = from[r] .. to[r]-1 into slots[r*keep ..).
// A range whose refills exceed twice the expected count sets *err and stops.
__global__ void __launch_bounds__(kTailThreads)
    shuffle_tail_kernel(const uint32_t* __restrict__ mt, const long long* __restrict__ from,
                        const long long* __restrict__ to, int keep, int32_t* __restrict__ slots,
                        int* __restrict__ err) {
    __shared__ uint32_t st[kMtN];
    __shared__ uint32_t a[kMtN];
    __shared__ int first;
    const int r = blockIdx.x;
    long long i = from[r];
    const long long m = to[r];
    if (i >= m || keep <= 0) return;
    const int t = threadIdx.x;
    const uint32_t* src = mt + static_cast<size_t>(r) * (kMtN + 1);
    if (t < kMtN) st[t] = src[t];
    int pos = static_cast<int>(src[kMtN]);
    __syncthreads();
    uint32_t w = t < kMtN ? mt_temper(st[t]) : 0u;
    int32_t* out = slots + static_cast<size_t>(r) * keep;
    const uint32_t K = static_cast<uint32_t>(keep);
    long long refills_left = 2 * ((m - i) / kMtN) + 16;
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
            if (!__syncthreads_or(rej)) {
                if (live && static_cast<uint32_t>(p >> 32) < K) atomicMax(out + (p >> 32), static_cast<int>(d));
                const long long used = min(static_cast<long long>(kMtN - pos), m - i);
                i += used;
                pos += static_cast<int>(used);
                break;
            }
            if (t == 0) first = kMtN;
            __syncthreads();
            if (rej) atomicMin(&first, t);
            __syncthreads();
            const int fr = first;
            if (live && t < fr && static_cast<uint32_t>(p >> 32) < K) atomicMax(out + (p >> 32), static_cast<int>(d));
            i += fr - pos;  // the rejected word is consumed; draw i + (fr - pos) takes the next word
            pos = fr + 1;
            if (pos >= kMtN) break;
        }
    }
}

}  // namespace

void launch_shuffle_tail(const uint32_t* mt, const long long* from, const long long* to, int n_ranges, int keep,
                         int32_t* slots, int* err, cudaStream_t s) {
    if (n_ranges <= 0 || keep <= 0) return;
    shuffle_tail_kernel<<<n_ranges, kTailThreads, 0, s>>>(mt, from, to, keep, slots, err);
    check(cudaGetLastError(), "shuffle_tail launch");
}

}  // namespace tgb
