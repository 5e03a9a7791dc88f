// Wave kernels: batched histograms and partitions over many leaves of many trees, and
// the per-tree set-up of a context (wave.h describes the scheme).
//
// Histogram (build_hist_col, cpp/src/histogram.cpp:44-76, for the smaller child of every
// planned leaf; subtract_hist_inplace's larger child is derived in the scan).  One
// persistent launch of clusters of 1, 2 or 4 CTAs (the autotuned privatisation depth:
// how many CTA-private histograms a flush merges).  The work (rows x groups of 32
// features, summed over the jobs) is cut into one contiguous range per cluster, walked as
// pieces (job, feature group, rows) whose rows the cluster's CTAs split.  Inside a CTA the
// accumulation is the lane-per-row scheme:
// a warp takes 32 rows, lane l holds its row's 32 code bytes of the group (staged in shared
// memory by TMA gathers in the constant-hessian modes, else loaded from global memory) and
// rotates them by l bytes in registers, so step j of the 32-step loop
// touches feature (j + l) & 31: 32 lanes, 32 features, 32 banks of the [bin][feature]
// layout, conflict-free whatever the codes.  Every code costs fire-and-forget 32-bit
// shared reductions only (their count depends on the payload mode, below), exact over a
// sub-chunk of rows, folded into 64-bit totals after every sub-chunk.  At the end of a
// piece the cluster adds its CTAs' totals through distributed shared memory and each CTA
// writes its share of the cells out (coalesced: consecutive bins of a feature).
//
// Payload modes (HistMode, per row):
//   exact const  int64 (v << 1 | goss):  v split into a 19-bit low and a signed high
//                part, plus a packed (unscaled, GOSS-scaled) row count: 3 reductions
//   exact var    int64 g and int64 h (both 19-bit split) and a count: 5 reductions
//   q16 const    int32 (q << 1 | goss): q and the packed count: 2 reductions
//   q16 var      int32 (qg << 16 | qh): qg, qh and a count: 3 reductions
//   q8 const     int16 (q << 1 | goss): (1 << 20 | q + 128) into the row class's
//                plane: 1 reduction
//   q8 var       uint16 (qg + 128 | qh << 8): (1 << 20 | qg + 128) and qh: 2 reductions
// Sums of quantised values are exact integers; the scan rescales them.
//
// Partition (split_indices, cpp/src/tree.cpp:68-91): stable, two launches over
// 2048-row tiles of all planned leaves (count, then scatter with in-tile ballot ranks).
#include <atomic>
#include <cstdint>
#include <cstring>
#include <cooperative_groups.h>

#include "wave.h"

namespace tgb {

namespace cg = cooperative_groups;

namespace {

constexpr int kThreads = 1024;
constexpr int kWarps = kThreads / 32;
constexpr int kFG = 32;
constexpr int kPlane = kFG * kBins;  // 32-bit words per plane (8192)
constexpr int kCells = kPlane / kThreads;  // cells a thread folds (8)
constexpr size_t kPlaneBytes = static_cast<size_t>(kPlane) * 4;
constexpr int kLoBits = 19;

template <int kMode>
struct ModeTraits;
template <>
struct ModeTraits<kHistExactConst> {
    static constexpr int planes = 3, sub = 8192;
    static constexpr bool var = false;
};
template <>
struct ModeTraits<kHistExactVar> {
    static constexpr int planes = 5, sub = 8192;
    static constexpr bool var = true;
};
template <>
struct ModeTraits<kHistQ16Const> {
    static constexpr int planes = 2, sub = 32768;
    static constexpr bool var = false;
};
template <>
struct ModeTraits<kHistQ16Var> {
    static constexpr int planes = 3, sub = 32768;
    static constexpr bool var = true;
};
template <>
struct ModeTraits<kHistQ8Const> {
    static constexpr int planes = 2, sub = 3072;
    static constexpr bool var = false;
};
template <>
struct ModeTraits<kHistQ8Var> {
    static constexpr int planes = 2, sub = 3072;
    static constexpr bool var = true;
};

// out[t] = in[(t + k) & 7] for a lane-dependent k in [0, 8): three conditional rotations.
__device__ __forceinline__ void rotate_words(unsigned int (&w)[8], int k) {
    unsigned int t[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) t[i] = (k & 1) ? w[(i + 1) & 7] : w[i];
#pragma unroll
    for (int i = 0; i < 8; ++i) w[i] = (k & 2) ? t[(i + 2) & 7] : t[i];
#pragma unroll
    for (int i = 0; i < 8; ++i) t[i] = (k & 4) ? w[(i + 4) & 7] : w[i];
#pragma unroll
    for (int i = 0; i < 8; ++i) w[i] = t[i];
}

// Rows of one histogram job: the root's sample or a planned leaf's smaller child.
struct JobRows {
    const int32_t* rows;
    const void* gq;  // payloads of rows[0 ..) (same positions)
    const void* hq;
    int count;
    int slot;
};

__device__ __forceinline__ JobRows job_rows(const WaveCtx& X, int src, int e) {
    JobRows r;
    if (src == 0) {
        r.rows = X.rows0;
        r.gq = X.gq;
        r.hq = X.hq;
        r.count = X.st->n_sample;
        r.slot = 0;
        return r;
    }
    const int L = X.ctl->exp_leaf[e];
    const DevNode& a = X.spec[2 * L];
    const DevNode& b = X.spec[2 * L + 1];
    const bool left_small = a.count <= b.count;  // cpp/src/tree.cpp:423
    const DevNode& c = left_small ? a : b;
    r.rows = (c.buf ? X.rows1 : X.rows0) + c.start;
    const long long pos = static_cast<long long>(c.buf) * X.pay_pitch + c.start;
    r.gq = static_cast<const unsigned char*>(X.gq) + pos * X.pay_bytes;
    r.hq = X.hq != nullptr ? static_cast<const long long*>(X.hq) + pos : nullptr;
    r.count = c.count;
    r.slot = c.slot;
    return r;
}

// A row's 32 code bytes of a feature group: one 32-byte load where the row stride keeps it
// 32-byte aligned (two_chunks: the group has 32 bytes before the row's end), else two
// 16-byte loads (the second only when the group has 32 bytes).
__device__ __forceinline__ void load_codes(const uint8_t* p, bool v8, bool two_chunks, uint4& a, uint4& b) {
    if (v8) {
        asm volatile("ld.global.nc.v8.u32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                     : "=r"(a.x), "=r"(a.y), "=r"(a.z), "=r"(a.w), "=r"(b.x), "=r"(b.y), "=r"(b.z), "=r"(b.w)
                     : "l"(p));
    } else {
        const uint4* p4 = reinterpret_cast<const uint4*>(p);
        a = __ldg(p4);
        b = two_chunks ? __ldg(p4 + 1) : make_uint4(0, 0, 0, 0);
    }
}

// A CTA's totals in a padded [feature][bin] layout, index f * kTotPitch + b: the fold
// writes one bin of a warp's 32 features and the flush reads 32 consecutive bins of one
// feature, and with a pitch of 257 words both touch 32 distinct banks; the flush's global
// writes are then consecutive bins of a feature (whole sectors).
constexpr int kTotPitch = kBins + 1;
constexpr int kTot = kFG * kTotPitch;  // 8224 cells
// Rows of one CTA's share of a piece: the constant-hessian modes pack their two row counts
// (unscaled, GOSS-scaled) into 16-bit halves.
constexpr int kMaxShareRows = 65535;

// Dynamic shared memory of one instantiation.  Constant-hessian modes: the working planes,
// then the totals (G as 64-bit words, packed counts), folded every sub-chunk.  Per-row
// hessian modes: 64-bit register accumulators, their totals (G, H as 64-bit words, counts)
// written over the working planes at the end of a piece.  Then the work prefix of the jobs.
template <int kMode>
struct SmemLayout {
    using T = ModeTraits<kMode>;
    static constexpr size_t work = static_cast<size_t>(T::planes) * kPlaneBytes;
    static constexpr size_t tot_bytes = static_cast<size_t>(kTot) * (T::var ? 20 : 12);
    static constexpr size_t tot_off = T::var ? 0 : work;
    static constexpr size_t region = T::var ? (work > tot_bytes ? work : tot_bytes) : work + tot_bytes;
    static constexpr size_t plan_off = (region + 15) / 16 * 16;
    static constexpr size_t bytes = plan_off + sizeof(unsigned long long) * (kMaxWaveJobs + 1);
    static_assert(bytes + 2048 <= 232448, "wave histogram shared memory above the 227 KB opt-in");
    static_assert(region % 16 == 0 && tot_off % 16 == 0, "16-byte zeroing");
};

template <int kMode>
struct ConstPayload;
template <>
struct ConstPayload<kHistExactConst> {
    using type = long long;
};
template <>
struct ConstPayload<kHistQ16Const> {
    using type = int;
};
template <>
struct ConstPayload<kHistQ8Const> {
    using type = short;
};

// One row of a constant-hessian mode: its 32 codes (two 16-byte words, rotated by the
// lane so that step j touches feature (j + lane) & 31) into the working planes.
template <int kMode>
__device__ __forceinline__ void add_row_const(unsigned int* __restrict__ P, typename ConstPayload<kMode>::type p,
                                              const uint4 ca, const uint4 cb, int lane, int q, int sh) {
    unsigned int a0, a1 = 0u, a2 = 0u;
    unsigned int* plane = P;
    if constexpr (kMode == kHistExactConst) {
        const long long v = p >> 1;
        a0 = static_cast<unsigned int>(v) & ((1u << kLoBits) - 1u);
        a1 = static_cast<unsigned int>(static_cast<int>(v >> kLoBits));
        a2 = (p & 1) ? 0x10000u : 1u;
    } else if constexpr (kMode == kHistQ16Const) {
        a0 = static_cast<unsigned int>(p >> 1);
        a1 = (p & 1) ? 0x10000u : 1u;
    } else {
        const int pv = p;
        a0 = (1u << 20) | static_cast<unsigned int>((pv >> 1) + 128);
        plane = (pv & 1) ? P + kPlane : P;
    }
    unsigned int wd[8] = {ca.x, ca.y, ca.z, ca.w, cb.x, cb.y, cb.z, cb.w};
    rotate_words(wd, q);
    unsigned int Rw[8];
#pragma unroll
    for (int t = 0; t < 8; ++t) Rw[t] = __funnelshift_r(wd[t], wd[(t + 1) & 7], sh);
#pragma unroll
    for (int jj = 0; jj < 32; ++jj) {
        const int f = (jj + lane) & 31;
        const unsigned int code = (Rw[jj >> 2] >> ((jj & 3) * 8)) & 0xffu;
        const int cell = static_cast<int>(code) * 32 + f;
        if constexpr (kMode == kHistExactConst) {
            atomicAdd(&P[cell], a0);
            atomicAdd(&P[kPlane + cell], a1);
            atomicAdd(&P[2 * kPlane + cell], a2);
        } else if constexpr (kMode == kHistQ16Const) {
            atomicAdd(&P[cell], a0);
            atomicAdd(&P[kPlane + cell], a1);
        } else {
            atomicAdd(&plane[cell], a0);
        }
    }
}

// The rows [r0, r1) of a CTA's share of one piece (one group of 32 features), constant-
// hessian modes, lane = row: every code costs the mode's fire-and-forget 32-bit shared
// reductions, exact over a sub-chunk of rows and folded into the shared 64-bit totals after
// it.  Software-pipelined: a warp's next row index is loaded two steps ahead and its codes
// and payload one step ahead, so their latency overlaps the current step's reductions.  A
// separate (not inlined) function: the loop keeps only its own state in registers.
template <int kMode>
__device__ __noinline__ void accumulate_const(unsigned int* __restrict__ P, unsigned long long* __restrict__ Gt,
                                              unsigned int* __restrict__ Ct, const int32_t* __restrict__ rows, int r0,
                                              int r1, const uint8_t* __restrict__ codes, int stride, int fg0,
                                              const void* __restrict__ gqp) {
    using T = ModeTraits<kMode>;
    using PT = typename ConstPayload<kMode>::type;
    const PT* __restrict__ pay = static_cast<const PT*>(gqp);  // by position, like rows
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int q = lane >> 2, sh = (lane & 3) * 8;
    const bool two_chunks = stride - fg0 >= 32;
    const bool v8 = two_chunks && (stride & 31) == 0;
    constexpr int kStep = kWarps * 32;
    for (int s0 = r0; s0 < r1; s0 += T::sub) {
        const int s1 = min(r1, s0 + T::sub);
        const int k0 = s0 + warp * 32 + lane;
        int r_cur = k0 < s1 ? rows[k0] : -1;
        PT p = k0 < s1 ? pay[k0] : PT(0);
        int r_nxt = k0 + kStep < s1 ? rows[k0 + kStep] : -1;
        PT p_nxt = k0 + kStep < s1 ? pay[k0 + kStep] : PT(0);
        uint4 ca = make_uint4(0, 0, 0, 0), cb = make_uint4(0, 0, 0, 0);
        if (r_cur >= 0) load_codes(codes + static_cast<size_t>(r_cur) * stride + fg0, v8, two_chunks, ca, cb);
        for (int base = s0 + warp * 32; base < s1; base += kStep) {
            const int r = r_cur;
            const uint4 xa = ca, xb = cb;
            const PT xp = p;
            r_cur = r_nxt;
            p = p_nxt;
            const int kn = base + 2 * kStep + lane;
            r_nxt = kn < s1 ? rows[kn] : -1;
            p_nxt = kn < s1 ? pay[kn] : PT(0);
            if (r_cur >= 0) load_codes(codes + static_cast<size_t>(r_cur) * stride + fg0, v8, two_chunks, ca, cb);
            if (r >= 0) add_row_const<kMode>(P, xp, xa, xb, lane, q, sh);
        }
        __syncthreads();
        // fold the sub-chunk into the totals and clear the working planes
#pragma unroll
        for (int cc = 0; cc < kCells; ++cc) {
            const int cell = threadIdx.x + cc * kThreads;
            const int ti = (cell & 31) * kTotPitch + (cell >> 5);
            long long dg;
            unsigned int dc;
            if constexpr (kMode == kHistExactConst) {
                dg = static_cast<long long>(static_cast<int>(P[kPlane + cell])) * (1ll << kLoBits) + P[cell];
                dc = P[2 * kPlane + cell];
            } else if constexpr (kMode == kHistQ16Const) {
                dg = static_cast<int>(P[cell]);
                dc = P[kPlane + cell];
            } else {
                const unsigned int w1 = P[cell], w2 = P[kPlane + cell];
                const unsigned int n1 = w1 >> 20, n2 = w2 >> 20;
                dg = static_cast<long long>(w1 & 0xfffffu) + static_cast<long long>(w2 & 0xfffffu) -
                     128ll * static_cast<long long>(n1 + n2);
                dc = n1 | (n2 << 16);
            }
            Gt[ti] += static_cast<unsigned long long>(dg);
            Ct[ti] += dc;
#pragma unroll
            for (int pl = 0; pl < T::planes; ++pl) P[pl * kPlane + cell] = 0u;
        }
        __syncthreads();
    }
}

// ---- code rows staged by TMA (constant-hessian modes) ---------------------------------
// A warp owns two 1 KB staging slots (its batch of 32 rows x the group's 32 code bytes)
// and an mbarrier per slot.  Lanes 0-7 each gather four rows of a batch with one
// cp.async.bulk.tensor tile::gather4 (box: 32 bytes of one row), two batches ahead of the
// one the warp accumulates; a lane then reads its row from the slot with two conflict-free
// 16-byte shared loads.  The direct loads cost 32 scattered sectors per warp and row batch
// on the L1 data path that the shared reductions also use; the gathers leave it to them.
constexpr int kSlotBytes = 32 * kFG;                 // one warp's batch
constexpr int kSlotStride = kWarps * kSlotBytes;     // slot 1 of every warp after slot 0 of all
constexpr int kStageBytes = 2 * kSlotStride;         // 64 KB, over the 64-bit totals
constexpr int kSpinLimit = 1 << 18;                  // polls of one mbarrier wait
constexpr int kErrStaging = 3;                       // ctl->error: a staging wait gave up
static_assert(kStageBytes + 128 <= kTot * 8, "the staging slots lie inside the G totals");

__device__ __forceinline__ unsigned int smem_u32(const void* p) {
    return static_cast<unsigned int>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(unsigned int bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned int bar, unsigned int bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
// Polls phase `parity` of the barrier at most kSpinLimit times; false when it gave up.
__device__ __forceinline__ bool mbar_wait(unsigned int bar, unsigned int parity) {
    for (int it = 0; it < kSpinLimit; ++it) {
        unsigned int done;
        asm volatile(
            "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}
// 16 bytes of shared memory at a 32-bit shared address (after the slot's barrier wait).
__device__ __forceinline__ uint4 lds16(unsigned int addr) {
    uint4 v;
    asm volatile("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "r"(addr)
                 : "memory");
    return v;
}
// Rows y0..y3, bytes [x, x + 32) of each, to dst (4 x 32 bytes), completing on bar.
__device__ __forceinline__ void tma_gather4(unsigned int dst, const CUtensorMap* map, int x, int y0, int y1, int y2,
                                            int y3, unsigned int bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile::gather4.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(dst),
        "l"(map), "r"(x), "r"(y0), "r"(y1), "r"(y2), "r"(y3), "r"(bar)
        : "memory");
}

// accumulate_const with the code rows staged by TMA.  The 64-bit G totals are kept in
// registers (a thread owns the same cells as in the fold) and written to Gt at the end: the
// staging slots lie over Gt meanwhile; the counts fold into Ct as before.  `phase` holds the
// parity of each of the warp's two barriers across calls; returned updated.  A wait that
// gives up sets ctl->error and ends the staging for the rest of the call (no new gathers,
// no further waits but one bounded wait per gather still in flight).
template <int kMode>
__device__ __noinline__ unsigned int accumulate_const_tma(unsigned int* __restrict__ P,
                                                          unsigned long long* __restrict__ Gt,
                                                          unsigned int* __restrict__ Ct, unsigned char* stage,
                                                          unsigned long long* bars, unsigned int phase,
                                                          const int32_t* __restrict__ rows, int r0, int r1,
                                                          const CUtensorMap* map, int fg0,
                                                          const void* __restrict__ gqp, int* err) {
    using T = ModeTraits<kMode>;
    using PT = typename ConstPayload<kMode>::type;
    constexpr int kStep = kWarps * 32;
    constexpr int kFoldRounds = T::sub / kStep;
    static_assert(T::sub % kStep == 0, "a sub-chunk is whole rounds of the CTA");
    const PT* __restrict__ pay = static_cast<const PT*>(gqp);  // by position, like rows
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int q = lane >> 2, sh = (lane & 3) * 8;
    const unsigned int slot0 = smem_u32(stage) + warp * kSlotBytes;
    const unsigned int bar0 = smem_u32(bars + 2 * warp);
    long long accG[kCells];
#pragma unroll
    for (int cc = 0; cc < kCells; ++cc) accG[cc] = 0;
    // the staging area's generic writes (zeroing, the previous piece's totals) before the
    // gathers' asynchronous ones; the descriptor was written by a host copy
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (lane < 8) asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(map) : "memory");
    __syncthreads();
    bool ok = true;
    unsigned int pending = 0u;  // slots with gathers in flight
    // The lane's row of batch k of this warp (the batch's first row pads a short batch),
    // loaded a round before its gather is issued.
    auto row_of = [&](int k) -> int {
        const int base = r0 + k * kStep + warp * 32;
        if (base >= r1) return 0;
        const int kk = base + lane;
        return rows[kk < r1 ? kk : base];
    };
    // Gathers batch k of this warp (lane rows `row`) into slot s; returns the lane's payload.
    auto issue = [&](int k, int s, int row) -> PT {
        const int base = r0 + k * kStep + warp * 32;
        if (!ok || base >= r1) return PT(0);
        const int kk = base + lane;
        const PT p = kk < r1 ? pay[kk] : PT(0);
        const int y0 = __shfl_sync(0xffffffffu, row, (4 * lane) & 31);
        const int y1 = __shfl_sync(0xffffffffu, row, (4 * lane + 1) & 31);
        const int y2 = __shfl_sync(0xffffffffu, row, (4 * lane + 2) & 31);
        const int y3 = __shfl_sync(0xffffffffu, row, (4 * lane + 3) & 31);
        const unsigned int bar = bar0 + 8u * s;
        if (lane == 0) mbar_expect_tx(bar, kSlotBytes);
        __syncwarp();
        if (lane < 8) tma_gather4(slot0 + s * kSlotStride + lane * 128, map, fg0, y0, y1, y2, y3, bar);
        pending |= 1u << s;
        return p;
    };
    const int n_rounds = r1 > r0 ? (r1 - r0 + kStep - 1) / kStep : 0;
    PT p0 = issue(0, 0, row_of(0));
    PT p1 = issue(1, 1, row_of(1));
    int rq = row_of(2);
    const int h = (lane >> 2) & 1;  // lanes 4-7 of each 8 read their second half first
    for (int i = 0; i < n_rounds; ++i) {
        const int s = i & 1;
        const int base = r0 + i * kStep + warp * 32;
        if (base < r1) {
            if (ok) {
                ok = __all_sync(0xffffffffu, mbar_wait(bar0 + 8u * s, (phase >> s) & 1u));
                if (ok) {
                    phase ^= 1u << s;
                    pending &= ~(1u << s);
                } else if (lane == 0) {
                    atomicExch(err, kErrStaging);
                }
            }
            const unsigned int rp = slot0 + s * kSlotStride + lane * 32;
            const uint4 c0 = lds16(rp + 16 * h);
            const uint4 c1 = lds16(rp + 16 * (h ^ 1));
            const uint4 ca = h ? c1 : c0, cb = h ? c0 : c1;
            const PT p = s ? p1 : p0;
            __syncwarp();  // every lane has read the slot before it is refilled
            const PT pn = issue(i + 2, s, rq);
            rq = row_of(i + 3);
            if (s) p1 = pn;
            else p0 = pn;
            if (base + lane < r1) add_row_const<kMode>(P, p, ca, cb, lane, q, sh);
        }
        if ((i + 1) % kFoldRounds == 0 || i + 1 == n_rounds) {
            __syncthreads();
            // fold the sub-chunk: G into registers, counts into Ct; clear the planes
#pragma unroll
            for (int cc = 0; cc < kCells; ++cc) {
                const int cell = threadIdx.x + cc * kThreads;
                const int ti = (cell & 31) * kTotPitch + (cell >> 5);
                long long dg;
                unsigned int dc;
                if constexpr (kMode == kHistExactConst) {
                    dg = static_cast<long long>(static_cast<int>(P[kPlane + cell])) * (1ll << kLoBits) + P[cell];
                    dc = P[2 * kPlane + cell];
                } else if constexpr (kMode == kHistQ16Const) {
                    dg = static_cast<int>(P[cell]);
                    dc = P[kPlane + cell];
                } else {
                    const unsigned int w1 = P[cell], w2 = P[kPlane + cell];
                    const unsigned int n1 = w1 >> 20, n2 = w2 >> 20;
                    dg = static_cast<long long>(w1 & 0xfffffu) + static_cast<long long>(w2 & 0xfffffu) -
                         128ll * static_cast<long long>(n1 + n2);
                    dc = n1 | (n2 << 16);
                }
                accG[cc] += dg;
                Ct[ti] += dc;
#pragma unroll
                for (int pl = 0; pl < T::planes; ++pl) P[pl * kPlane + cell] = 0u;
            }
            __syncthreads();
        }
    }
    if (!ok)  // warp-uniform
        for (int s = 0; s < 2; ++s)
            if (((pending >> s) & 1u) && __all_sync(0xffffffffu, mbar_wait(bar0 + 8u * s, (phase >> s) & 1u)))
                phase ^= 1u << s;
    // every warp is past its last slot read (the last round's fold): the totals over them
#pragma unroll
    for (int cc = 0; cc < kCells; ++cc) {
        const int cell = threadIdx.x + cc * kThreads;
        Gt[(cell & 31) * kTotPitch + (cell >> 5)] = static_cast<unsigned long long>(accG[cc]);
    }
    return phase;
}

// The rows [r0, r1) of a CTA's share of one piece, per-row hessian modes: the same lane-
// per-row reductions, folded into per-thread 64-bit registers every sub-chunk; the totals
// are written over the (then clear) working planes at the end.
template <int kMode>
__device__ __noinline__ void accumulate_var(unsigned int* __restrict__ P, unsigned long long* __restrict__ Gt,
                                            unsigned long long* __restrict__ Ht, unsigned int* __restrict__ Ct,
                                            const int32_t* __restrict__ rows, int r0, int r1,
                                            const uint8_t* __restrict__ codes, int stride, int fg0,
                                            const void* __restrict__ gqp, const void* __restrict__ hqp) {
    using T = ModeTraits<kMode>;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int q = lane >> 2, sh = (lane & 3) * 8;
    const bool two_chunks = stride - fg0 >= 32;
    const bool v8 = two_chunks && (stride & 31) == 0;
    long long accG[kCells], accH[kCells];
    unsigned int accC[kCells];
#pragma unroll
    for (int cc = 0; cc < kCells; ++cc) {
        accG[cc] = 0;
        accH[cc] = 0;
        accC[cc] = 0u;
    }
    for (int s0 = r0; s0 < r1; s0 += T::sub) {
        const int s1 = min(r1, s0 + T::sub);
        int r_next = s0 + warp * 32 + lane < s1 ? rows[s0 + warp * 32 + lane] : -1;
        for (int base = s0 + warp * 32; base < s1; base += kWarps * 32) {
            const int r = r_next;
            const int k = base + lane;  // the row's position: its payload's index
            const int kn = base + kWarps * 32 + lane;
            r_next = kn < s1 ? rows[kn] : -1;
            if (r < 0) continue;
            unsigned int a0 = 0, a1 = 0, a2 = 0, a3 = 0;
            if constexpr (kMode == kHistExactVar) {
                const long long gv = static_cast<const long long*>(gqp)[k];
                const long long hv = static_cast<const long long*>(hqp)[k];
                a0 = static_cast<unsigned int>(gv) & ((1u << kLoBits) - 1u);
                a1 = static_cast<unsigned int>(static_cast<int>(gv >> kLoBits));
                a2 = static_cast<unsigned int>(hv) & ((1u << kLoBits) - 1u);
                a3 = static_cast<unsigned int>(static_cast<int>(hv >> kLoBits));
            } else if constexpr (kMode == kHistQ16Var) {
                const unsigned int p = static_cast<const unsigned int*>(gqp)[k];
                a0 = static_cast<unsigned int>(static_cast<int>(p) >> 16);
                a1 = p & 0xffffu;
            } else {  // kHistQ8Var
                const unsigned int p = static_cast<const unsigned short*>(gqp)[k];
                a0 = (1u << 20) | (p & 0xffu);
                a1 = p >> 8;
            }
            uint4 ca, cb;
            load_codes(codes + static_cast<size_t>(r) * stride + fg0, v8, two_chunks, ca, cb);
            unsigned int wd[8] = {ca.x, ca.y, ca.z, ca.w, cb.x, cb.y, cb.z, cb.w};
            rotate_words(wd, q);
            unsigned int Rw[8];
#pragma unroll
            for (int t = 0; t < 8; ++t) Rw[t] = __funnelshift_r(wd[t], wd[(t + 1) & 7], sh);
#pragma unroll
            for (int jj = 0; jj < 32; ++jj) {
                const int f = (jj + lane) & 31;
                const unsigned int code = (Rw[jj >> 2] >> ((jj & 3) * 8)) & 0xffu;
                const int cell = static_cast<int>(code) * 32 + f;
                if constexpr (kMode == kHistExactVar) {
                    atomicAdd(&P[cell], a0);
                    atomicAdd(&P[kPlane + cell], a1);
                    atomicAdd(&P[2 * kPlane + cell], a2);
                    atomicAdd(&P[3 * kPlane + cell], a3);
                    atomicAdd(&P[4 * kPlane + cell], 1u);
                } else if constexpr (kMode == kHistQ16Var) {
                    atomicAdd(&P[cell], a0);
                    atomicAdd(&P[kPlane + cell], a1);
                    atomicAdd(&P[2 * kPlane + cell], 1u);
                } else {
                    atomicAdd(&P[cell], a0);
                    atomicAdd(&P[kPlane + cell], a1);
                }
            }
        }
        __syncthreads();
        // fold the sub-chunk into 64-bit registers and clear the planes
#pragma unroll
        for (int cc = 0; cc < kCells; ++cc) {
            const int cell = threadIdx.x + cc * kThreads;
            if constexpr (kMode == kHistExactVar) {
                accG[cc] += static_cast<long long>(static_cast<int>(P[kPlane + cell])) * (1ll << kLoBits) + P[cell];
                accH[cc] +=
                    static_cast<long long>(static_cast<int>(P[3 * kPlane + cell])) * (1ll << kLoBits) + P[2 * kPlane + cell];
                accC[cc] += P[4 * kPlane + cell];
            } else if constexpr (kMode == kHistQ16Var) {
                accG[cc] += static_cast<int>(P[cell]);
                accH[cc] += P[kPlane + cell];
                accC[cc] += P[2 * kPlane + cell];
            } else {
                const unsigned int w1 = P[cell];
                const unsigned int n1 = w1 >> 20;
                accG[cc] += static_cast<long long>(w1 & 0xfffffu) - 128ll * static_cast<long long>(n1);
                accH[cc] += P[kPlane + cell];
                accC[cc] += n1;
            }
#pragma unroll
            for (int pl = 0; pl < T::planes; ++pl) P[pl * kPlane + cell] = 0u;
        }
        __syncthreads();
    }
    // totals over the (clear) planes: every cell of the padded layout has one owner
#pragma unroll
    for (int cc = 0; cc < kCells; ++cc) {
        const int cell = threadIdx.x + cc * kThreads;
        const int ti = (cell & 31) * kTotPitch + (cell >> 5);
        Gt[ti] = static_cast<unsigned long long>(accG[cc]);
        Ht[ti] = static_cast<unsigned long long>(accH[cc]);
        Ct[ti] = accC[cc];
    }
}

// One launch histograms every job (context, planned leaf's smaller child; or each
// context's root) of the wave.  The work, rows x feature groups summed over the jobs, is
// cut into equal contiguous ranges, one per cluster; a cluster walks its range as pieces
// (job, feature group, row range), its CTAs split each piece's rows, and after a piece the
// cluster adds its CTAs' totals through distributed shared memory and writes them out:
// plain stores when the piece is the whole (job, feature group), 64-bit atomics when
// other clusters share it.  A job's slot is clear before the launch.
template <int kMode>
__global__ void __launch_bounds__(kThreads, 1)
    wave_hist_kernel(const WaveCtx* __restrict__ ctxs, int n_ctx, int src, unsigned long long* rows_counter) {
    using T = ModeTraits<kMode>;
    using Lay = SmemLayout<kMode>;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    unsigned int* P = reinterpret_cast<unsigned int*>(smem_raw);  // working planes
    unsigned long long* Gt = reinterpret_cast<unsigned long long*>(smem_raw + Lay::tot_off);
    unsigned long long* Ht = Gt + kTot;  // per-row hessian modes only
    unsigned int* Ct = reinterpret_cast<unsigned int*>(Gt + (T::var ? 2 : 1) * kTot);
    unsigned long long* s_wstart = reinterpret_cast<unsigned long long*>(smem_raw + Lay::plan_off);
    // TMA staging (constant-hessian modes): slots over Gt from its first 128-byte boundary,
    // two mbarriers per warp, their parities
    __shared__ __align__(8) unsigned long long s_bars[2 * kWarps];
    unsigned char* stage = smem_raw + Lay::tot_off;
    stage += (128u - (smem_u32(stage) & 127u)) & 127u;
    unsigned int phase = 0u;
    {  // private state first: it overlaps the previous kernel's tail
        uint4* z = reinterpret_cast<uint4*>(smem_raw);
        for (int k = threadIdx.x; k < static_cast<int>(Lay::region / 16); k += blockDim.x) z[k] = make_uint4(0, 0, 0, 0);
    }
    if (!T::var && (threadIdx.x & 31) == 0) {
        mbar_init(smem_u32(&s_bars[2 * (threadIdx.x >> 5)]));
        mbar_init(smem_u32(&s_bars[2 * (threadIdx.x >> 5) + 1]));
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    pdl_wait();
    pdl_trigger();

    // ---- work plan (the same in every CTA) ----
    __shared__ int s_cpref[kMaxWaveCtx + 1];
    __shared__ unsigned long long s_red[kWarps], s_rsum[kWarps];
    if (static_cast<int>(threadIdx.x) < n_ctx)
        s_cpref[threadIdx.x] = src == 0 ? (ctxs[threadIdx.x].ctl->active ? 1 : 0) : ctxs[threadIdx.x].ctl->n_exp;
    __syncthreads();
    if (threadIdx.x == 0) {
        int acc = 0;
        for (int c = 0; c < n_ctx; ++c) {
            const int v = s_cpref[c];
            s_cpref[c] = acc;
            acc += v;
        }
        s_cpref[n_ctx] = min(acc, kMaxWaveJobs);
    }
    __syncthreads();
    const int n_jobs = s_cpref[n_ctx];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    {
        // work of each job (rows x feature groups), exclusive prefix over a contiguous run
        // of jobs per thread
        const int per = (n_jobs + kThreads - 1) / kThreads;
        const int j0 = min(n_jobs, static_cast<int>(threadIdx.x) * per), j1 = min(n_jobs, j0 + per);
        unsigned long long local = 0, lrows = 0;
        for (int j = j0; j < j1; ++j) {
            int c = 0;
            while (c + 1 < n_ctx && s_cpref[c + 1] <= j) ++c;
            const WaveCtx& X = ctxs[c];
            const JobRows jr = job_rows(X, src, src == 0 ? 0 : j - s_cpref[c]);
            const unsigned long long w =
                static_cast<unsigned long long>(jr.count) * ((X.gp.n_features + kFG - 1) / kFG);
            s_wstart[j] = w;
            local += w;
            lrows += static_cast<unsigned long long>(jr.count);
        }
        unsigned long long incl = local, rs = lrows;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += t;
            rs += __shfl_xor_sync(0xffffffffu, rs, o);
        }
        if (lane == 31) s_red[warp] = incl;
        if (lane == 0) s_rsum[warp] = rs;
        __syncthreads();
        unsigned long long wbase = 0, all = 0, rows_all = 0;
        for (int k = 0; k < kWarps; ++k) {
            if (k < warp) wbase += s_red[k];
            all += s_red[k];
            rows_all += s_rsum[k];
        }
        unsigned long long run = wbase + incl - local;
        for (int j = j0; j < j1; ++j) {
            const unsigned long long w = s_wstart[j];
            s_wstart[j] = run;
            run += w;
        }
        if (threadIdx.x == 0) {
            s_wstart[n_jobs] = all;
            if (rows_counter != nullptr && blockIdx.y == 0) atomicAdd(rows_counter, rows_all);
        }
    }
    __syncthreads();
    cg::cluster_group cluster = cg::this_cluster();
    const int csize = static_cast<int>(cluster.dim_blocks().y);  // CTAs per cluster: 1, 2 or 4
    const int cl = static_cast<int>(blockIdx.y) / csize;
    const int n_cl = static_cast<int>(gridDim.y) / csize;
    const unsigned int rank = cluster.block_rank();
    const unsigned long long w_all = s_wstart[n_jobs];
    const unsigned long long w_end = w_all * static_cast<unsigned long long>(cl + 1) / static_cast<unsigned long long>(n_cl);
    const unsigned long long max_piece = static_cast<unsigned long long>(kMaxShareRows) * csize;
    for (unsigned long long w = w_all * static_cast<unsigned long long>(cl) / static_cast<unsigned long long>(n_cl);
         w < w_end;) {
        // the job holding w: the last j with s_wstart[j] <= w (a non-empty job)
        int lo = 0, hi = n_jobs - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (s_wstart[mid] <= w) lo = mid;
            else hi = mid - 1;
        }
        const int j = lo;
        int c = 0;
        while (c + 1 < n_ctx && s_cpref[c + 1] <= j) ++c;
        const WaveCtx& X = ctxs[c];
        const int n_f = X.gp.n_features;
        const JobRows jr = job_rows(X, src, src == 0 ? 0 : j - s_cpref[c]);
        const unsigned long long R = static_cast<unsigned long long>(jr.count);
        const unsigned long long off = w - s_wstart[j];
        const int fg = static_cast<int>(off / R);
        const unsigned long long ra = off - static_cast<unsigned long long>(fg) * R;
        const unsigned long long len = min(min(R - ra, w_end - w), max_piece);
        const int piece0 = static_cast<int>(ra), piece1 = static_cast<int>(ra + len);
        const int qrows = (piece1 - piece0 + csize - 1) / csize;
        const int r0 = min(piece1, piece0 + static_cast<int>(rank) * qrows), r1 = min(piece1, r0 + qrows);
        const int fg0 = fg * kFG;
        if constexpr (T::var)
            accumulate_var<kMode>(P, Gt, Ht, Ct, jr.rows, r0, r1, X.codes, X.gp.stride, fg0, jr.gq, jr.hq);
        else if (X.codes_map_ok && (reinterpret_cast<uintptr_t>(&X.codes_map) & 63u) == 0)  // TMA wants 64 B
            phase = accumulate_const_tma<kMode>(P, Gt, Ct, stage, s_bars, phase, jr.rows, r0, r1, &X.codes_map, fg0,
                                                jr.gq, &X.ctl->error);
        else
            accumulate_const<kMode>(P, Gt, Ct, jr.rows, r0, r1, X.codes, X.gp.stride, fg0, jr.gq);
        __syncthreads();
        cluster.sync();
        // rank k adds its share of the cells over the cluster and writes them out
        const bool whole = piece0 == 0 && static_cast<unsigned long long>(piece1) == R;
        const int nf_here = min(kFG, n_f - fg0);
        const size_t slot_off = static_cast<size_t>(jr.slot) * static_cast<size_t>(n_f) * kBins;
        const double hscale = X.st->hscale;
        const unsigned long long hq1 = static_cast<unsigned long long>(__double2ll_rn(1.0 * hscale));
        const unsigned long long hq2 = static_cast<unsigned long long>(__double2ll_rn(1.0 * X.goss_scale * hscale));
        const int share = (kTot + csize - 1) / csize;
        const int i1 = min(kTot, static_cast<int>(rank + 1) * share);
        for (int ti = static_cast<int>(rank) * share + threadIdx.x; ti < i1; ti += kThreads) {
            const int f = ti / kTotPitch, b = ti - f * kTotPitch;
            if (b >= kBins || f >= nf_here) continue;
            unsigned long long g = 0, hs = 0;
            unsigned int cn = 0, c1 = 0, c2 = 0;
            for (int kk = 0; kk < csize; ++kk) {
                g += cluster.map_shared_rank(Gt, kk)[ti];
                const unsigned int pc = cluster.map_shared_rank(Ct, kk)[ti];
                if constexpr (T::var) {
                    hs += cluster.map_shared_rank(Ht, kk)[ti];
                    cn += pc;
                } else {
                    c1 += pc & 0xffffu;
                    c2 += pc >> 16;
                }
            }
            if constexpr (!T::var) {
                hs = static_cast<unsigned long long>(c1) * hq1 + static_cast<unsigned long long>(c2) * hq2;
                cn = c1 + c2;
            }
            if (cn == 0u) continue;
            const size_t o = slot_off + static_cast<size_t>(fg0 + f) * kBins + b;
            if (whole) {
                reinterpret_cast<unsigned long long*>(X.G)[o] = g;
                reinterpret_cast<unsigned long long*>(X.H)[o] = hs;
                X.C[o] = static_cast<int>(cn);
            } else {
                atomicAdd(reinterpret_cast<unsigned long long*>(X.G) + o, g);
                atomicAdd(reinterpret_cast<unsigned long long*>(X.H) + o, hs);
                atomicAdd(X.C + o, static_cast<int>(cn));
            }
        }
        cluster.sync();  // no CTA clears its totals while others read them
        {
            uint4* z = reinterpret_cast<uint4*>(smem_raw + Lay::tot_off);
            for (int k = threadIdx.x; k < static_cast<int>(Lay::tot_bytes / 16); k += kThreads)
                z[k] = make_uint4(0, 0, 0, 0);
        }
        __syncthreads();
        w += len;
    }
}

// ---- partition ----------------------------------------------------------------------
constexpr int kPartThreads = 256;
constexpr int kPartWarps = kPartThreads / 32;
constexpr int kPartPer = kPartTile / kPartThreads;

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

// A row's g payload (element i of the payload array), widened to 64 bits, and back.
__device__ __forceinline__ long long load_payload(const WaveCtx& X, long long i) {
    if (X.pay_bytes == 8) return static_cast<const long long*>(X.gq)[i];
    if (X.pay_bytes == 4) return static_cast<const int*>(X.gq)[i];
    return static_cast<const short*>(X.gq)[i];
}
__device__ __forceinline__ void store_payload(const WaveCtx& X, long long i, long long v) {
    if (X.pay_bytes == 8) static_cast<long long*>(X.gq)[i] = v;
    else if (X.pay_bytes == 4) static_cast<int*>(X.gq)[i] = static_cast<int>(v);
    else static_cast<short*>(X.gq)[i] = static_cast<short>(v);
}

// Global tile t -> (context, expansion, tile within the expansion).
struct TileRef {
    int c, e, k, lt;
};

__device__ __forceinline__ TileRef find_tile(const WaveCtx* ctxs, const int* s_pref, int n_ctx, int t) {
    TileRef r;
    int c = 0;
    while (c + 1 < n_ctx && s_pref[c + 1] <= t) ++c;
    const int lt = t - s_pref[c];
    const WaveCtl* ctl = ctxs[c].ctl;
    int lo = 0, hi = ctl->n_exp - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (ctl->exp_tile0[mid] <= lt) lo = mid;
        else hi = mid - 1;
    }
    r.c = c;
    r.e = lo;
    r.k = lt - ctl->exp_tile0[lo];
    r.lt = lt;
    return r;
}

__device__ __forceinline__ void load_tile(const WaveCtx& X, const int32_t* in, const DevSplit& S, int base, int end,
                                          int32_t (&row)[kPartPer], bool (&left)[kPartPer]) {
    const int feature = S.feature, threshold = S.threshold, ml = S.missing_left, type = S.type;
    unsigned long long cat[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) cat[k] = S.cat[k];
#pragma unroll
    for (int i = 0; i < kPartPer; ++i) {
        const int k = base + i * kPartThreads + threadIdx.x;
        row[i] = k < end ? in[k] : -1;
    }
    unsigned int b[kPartPer], b2[kPartPer];
    const uint8_t* col = X.codes_col + static_cast<size_t>(feature) * X.col_pitch;
    const uint8_t* col2 = type == 1 ? X.codes_col + static_cast<size_t>(S.feature2) * X.col_pitch : col;
#pragma unroll
    for (int i = 0; i < kPartPer; ++i) {
        b[i] = row[i] >= 0 ? col[row[i]] : 0u;
        b2[i] = row[i] >= 0 && type == 1 ? col2[row[i]] : 0u;
    }
#pragma unroll
    for (int i = 0; i < kPartPer; ++i)
        left[i] = row[i] >= 0 && goes_left(type, cat, threshold, ml, b[i], b2[i], X.gp.n_bins);
}

__device__ __forceinline__ void load_tile_prefix(const WaveCtx* ctxs, int n_ctx, int* s_pref) {
    if (static_cast<int>(threadIdx.x) < n_ctx) s_pref[threadIdx.x] = ctxs[threadIdx.x].ctl->tiles_total;
    __syncthreads();
    if (threadIdx.x == 0) {
        int acc = 0;
        for (int c = 0; c < n_ctx; ++c) {
            const int v = s_pref[c];
            s_pref[c] = acc;
            acc += v;
        }
        s_pref[n_ctx] = acc;
    }
    __syncthreads();
}

__global__ void __launch_bounds__(kPartThreads)
    wave_part_count_kernel(const WaveCtx* __restrict__ ctxs, int n_ctx) {
    pdl_wait();
    pdl_trigger();
    __shared__ int s_pref[kMaxWaveCtx + 1];
    __shared__ int red[kPartWarps];
    __shared__ int s_last;
    load_tile_prefix(ctxs, n_ctx, s_pref);
    const int total = s_pref[n_ctx];
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
        const TileRef tr = find_tile(ctxs, s_pref, n_ctx, t);
        const WaveCtx& X = ctxs[tr.c];
        WaveCtl* ctl = X.ctl;
        const int L = ctl->exp_leaf[tr.e];
        const DevNode& N = X.nodes[L];
        const DevSplit& S = ctl->expanded[L] == 2 ? X.splits_pair[L] : X.splits[L];
        const int32_t* in = (N.buf ? X.rows1 : X.rows0) + N.start;
        const int base = tr.k * kPartTile, end = min(base + kPartTile, N.count);
        int32_t row[kPartPer];
        bool left[kPartPer];
        load_tile(X, in, S, base, end, row, left);
        int cnt = 0;
#pragma unroll
        for (int i = 0; i < kPartPer; ++i) cnt += left[i] ? 1 : 0;
        cnt = block_sum(cnt, red);
        const int t0 = ctl->exp_tile0[tr.e], t1 = ctl->exp_tile0[tr.e + 1];
        if (threadIdx.x == 0) {
            X.tile_counts[tr.lt] = cnt;
            __threadfence();
            s_last = atomicAdd(&ctl->part_ticket[tr.e], 1) == t1 - t0 - 1;
        }
        __syncthreads();
        if (s_last) {
            // the leaf's last tile: its tiles' counts -> exclusive prefixes (in place), and the
            // leaf's left total, for the scatter
            __threadfence();
            volatile int* tc = X.tile_counts;
            const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
            int run = 0;
            for (int k0 = t0; k0 < t1; k0 += kPartThreads) {
                const int k = k0 + static_cast<int>(threadIdx.x);
                const int v = k < t1 ? tc[k] : 0;
                int incl = v;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int u = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= o) incl += u;
                }
                if (lane == 31) red[warp] = incl;
                __syncthreads();
                int wb = 0, all = 0;
#pragma unroll
                for (int w = 0; w < kPartWarps; ++w) {
                    if (w < warp) wb += red[w];
                    all += red[w];
                }
                if (k < t1) tc[k] = run + wb + incl - v;
                run += all;
                __syncthreads();  // red reuse
            }
            if (threadIdx.x == 0) {
                ctl->exp_left[tr.e] = run;
                ctl->part_ticket[tr.e] = 0;  // ready for the next wave
            }
        }
        __syncthreads();  // s_last reuse
    }
    // Clear the histogram slots of this wave's children (2 per expansion, consecutive):
    // the smaller child's is accumulated into by the histogram launch.
    for (int c = 0; c < n_ctx; ++c) {
        const WaveCtx& X = ctxs[c];
        const int ns = 2 * X.ctl->n_exp;
        if (ns == 0) continue;
        const size_t elems = static_cast<size_t>(X.gp.n_features) * kBins;
        const size_t first = static_cast<size_t>(X.ctl->slot0) * elems;
        const size_t n8 = static_cast<size_t>(ns) * elems;  // int64 elements of G and H
        uint4* g4 = reinterpret_cast<uint4*>(X.G + first);
        uint4* h4 = reinterpret_cast<uint4*>(X.H + first);
        uint4* c4 = reinterpret_cast<uint4*>(X.C + first);
        const size_t n16_8 = n8 / 2, n16_4 = n8 / 4;  // elems is a multiple of 256
        for (size_t k = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; k < n16_8;
             k += static_cast<size_t>(gridDim.x) * blockDim.x) {
            g4[k] = make_uint4(0, 0, 0, 0);
            h4[k] = make_uint4(0, 0, 0, 0);
            if (k < n16_4) c4[k] = make_uint4(0, 0, 0, 0);
        }
    }
}

__global__ void __launch_bounds__(kPartThreads)
    wave_part_scatter_kernel(const WaveCtx* __restrict__ ctxs, int n_ctx) {
    pdl_wait();
    pdl_trigger();
    __shared__ int s_pref[kMaxWaveCtx + 1];
    __shared__ int wc[kPartPer * kPartWarps];
    load_tile_prefix(ctxs, n_ctx, s_pref);
    const int total = s_pref[n_ctx];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned lt_mask = (1u << lane) - 1u;
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
        const TileRef tr = find_tile(ctxs, s_pref, n_ctx, t);
        const WaveCtx& X = ctxs[tr.c];
        const WaveCtl* ctl = X.ctl;
        const int L = ctl->exp_leaf[tr.e];
        const DevNode& N = X.nodes[L];
        const DevSplit& S = X.ctl->expanded[L] == 2 ? X.splits_pair[L] : X.splits[L];
        const int n_left = ctl->exp_left[tr.e];   // the leaf's left rows (count launch)
        const int left0 = X.tile_counts[tr.lt];  // left rows of the leaf's earlier tiles
        if (tr.k == 0 && threadIdx.x == 0) {
            DevNode& A = X.spec[2 * L];
            DevNode& B = X.spec[2 * L + 1];
            A.start = N.start;
            A.count = n_left;
            B.start = N.start + n_left;
            B.count = N.count - n_left;
        }
        const int32_t* in = (N.buf ? X.rows1 : X.rows0) + N.start;
        int32_t* out = (N.buf ? X.rows0 : X.rows1) + N.start;
        const int base = tr.k * kPartTile, end = min(base + kPartTile, N.count);
        int32_t row[kPartPer];
        bool left[kPartPer];
        load_tile(X, in, S, base, end, row, left);
        // the rows' payloads move with them (same positions in the other buffer); loaded
        // here so that their latency overlaps the ranks below
        const long long from0 = static_cast<long long>(N.buf) * X.pay_pitch + N.start;
        const long long to0 = static_cast<long long>(1 - N.buf) * X.pay_pitch + N.start;
        long long pg[kPartPer], ph[kPartPer];
#pragma unroll
        for (int i = 0; i < kPartPer; ++i) {
            const int kk = base + i * kPartThreads + threadIdx.x;
            pg[i] = row[i] >= 0 ? load_payload(X, from0 + kk) : 0;
            ph[i] = row[i] >= 0 && X.hq != nullptr ? static_cast<const long long*>(X.hq)[from0 + kk] : 0;
        }
        unsigned bal[kPartPer];
#pragma unroll
        for (int i = 0; i < kPartPer; ++i) {
            bal[i] = __ballot_sync(0xffffffffu, left[i]);
            if (lane == 0) wc[i * kPartWarps + warp] = __popc(bal[i]);
        }
        __syncthreads();
        int run = 0;
        int excl[kPartPer];
#pragma unroll
        for (int i = 0; i < kPartPer; ++i) {
            int e = run;
            for (int w = 0; w < kPartWarps; ++w) {
                const int cw = wc[i * kPartWarps + w];
                if (w < warp) e += cw;
                run += cw;
            }
            excl[i] = e;
        }
#pragma unroll
        for (int i = 0; i < kPartPer; ++i) {
            if (row[i] < 0) continue;
            const int kk = base + i * kPartThreads + threadIdx.x;
            const int lrank = excl[i] + __popc(bal[i] & lt_mask);
            const int dst = left[i] ? left0 + lrank : n_left + (base - left0) + (kk - base - lrank);
            out[dst] = row[i];
            store_payload(X, to0 + dst, pg[i]);
            if (X.hq != nullptr) static_cast<long long*>(X.hq)[to0 + dst] = ph[i];
        }
        __syncthreads();  // wc reuse
    }
}

// ---- per-tree set-up ------------------------------------------------------------------
__global__ void wave_tree_init_kernel(DevNode* nodes, DevSplit* splits, DevTreeState* st, WaveCtl* ctl,
                                      int n_sample, int use_dev_count) {
    const int count = use_dev_count ? st->n_sample : n_sample;
    if (threadIdx.x == 0) {
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
        r.slot = 0;
        nodes[0] = r;
        splits[0].valid = 0;
        st->n_nodes = 1;
        st->done = 0;
        st->parent = -1;
        st->small_node = st->large_node = -1;
        st->n_sample = count;
        ctl->splits_done = 0;
        ctl->n_exp = 0;
        ctl->exp_counter = 0;
        ctl->tiles_total = 0;
        ctl->active = 1;
        ctl->slot0 = 1;
        ctl->error = 0;
        ctl->waves = 0;
        ctl->pair_used = 0;
    }
    ctl->expanded[0] = 0;
}

__device__ int shift_for(double max_abs, int count) {
    if (!(max_abs > 0.0) || count <= 0) return 0;
    int clog = 0;
    while ((1ll << clog) < static_cast<long long>(count)) ++clog;
    const int e = ilogb(max_abs);
    int s = min(61 - (e + 1) - clog, 36 - e);
    return max(-1000, min(1000, s));
}

// Exact modes: power-of-two shifts (no sum over the sample can reach 2^62, no row's value
// 2^37).  Quantised modes: the largest |g| (and h) of the sample maps to the largest
// code; constant-hessian modes keep the exact hessian shift (H is rebuilt from counts).
__global__ void wave_scales_kernel(DevTreeState* st, const AllScale* __restrict__ all, int mode) {
    if (all) {
        st->max_abs_g_bits = all->maxg_bits;
        st->max_h_bits = all->maxh_bits;
    }
    const double mg = __longlong_as_double(static_cast<long long>(st->max_abs_g_bits));
    const double mh = __longlong_as_double(static_cast<long long>(st->max_h_bits));
    const bool var = mode & 1;
    const int qbits = mode >= kHistQ8Const ? 8 : mode >= kHistQ16Const ? 16 : 0;
    if (qbits == 0) {
        st->gshift = shift_for(mg, st->n_sample);
        st->gscale = ldexp(1.0, st->gshift);
        st->inv_gscale = ldexp(1.0, -st->gshift);
    } else {
        const double gmax = qbits == 8 ? 127.0 : 32767.0;
        st->gshift = 0;
        st->gscale = mg > 0.0 ? gmax / mg : 1.0;
        st->inv_gscale = 1.0 / st->gscale;
    }
    if (qbits == 0 || !var) {
        st->hshift = shift_for(mh, st->n_sample);
        st->hscale = ldexp(1.0, st->hshift);
        st->inv_hscale = ldexp(1.0, -st->hshift);
    } else {
        const double hmax = qbits == 8 ? 255.0 : 65535.0;
        st->hshift = 0;
        st->hscale = mh > 0.0 ? hmax / mh : 1.0;
        st->inv_hscale = 1.0 / st->hscale;
    }
}

// SplitMix64 output function (Steele, Lea and Flood, OOPSLA 2014): the stream of uniform
// numbers of the stochastic rounding, a function of (row, tree, seed) only.
__device__ __forceinline__ unsigned long long splitmix64(unsigned long long z) {
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

__device__ __forceinline__ double uniform01(unsigned long long seed, int r, unsigned salt) {
    const unsigned long long z = splitmix64(seed ^ (static_cast<unsigned long long>(r) << 20) ^
                                            (static_cast<unsigned long long>(salt) << 52));
    return static_cast<double>(z >> 11) * (1.0 / 9007199254740992.0);  // 53 bits -> [0, 1)
}

// floor(x + u), u uniform in [0, 1): unbiased stochastic rounding, clamped to [lo, hi].
__device__ __forceinline__ int sround(double x, double u, int lo, int hi) {
    return max(lo, min(hi, static_cast<int>(floor(x + u))));
}

template <int kMode>
__global__ void wave_quantize_kernel(const int32_t* __restrict__ rows, const double* __restrict__ g,
                                     const double* __restrict__ h, const uint8_t* __restrict__ goss_flag,
                                     double goss_scale, const DevTreeState* __restrict__ st,
                                     unsigned long long seed, void* __restrict__ gq, void* __restrict__ hq) {
    const int count = st->n_sample;
    const double gscale = st->gscale, hscale = st->hscale;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x) {
        const int r = rows[k];
        double gv = g[r];
        double hv = h ? h[r] : 1.0;
        const bool sc = goss_flag != nullptr && goss_flag[r] == 2;
        if (sc) {
            gv *= goss_scale;
            hv *= goss_scale;
        }
        if constexpr (kMode == kHistExactConst) {
            const long long v = __double2ll_rn(gv * gscale);
            static_cast<long long*>(gq)[k] = static_cast<long long>((static_cast<unsigned long long>(v) << 1) | (sc ? 1ull : 0ull));
        } else if constexpr (kMode == kHistExactVar) {
            static_cast<long long*>(gq)[k] = __double2ll_rn(gv * gscale);
            static_cast<long long*>(hq)[k] = __double2ll_rn(hv * hscale);
        } else if constexpr (kMode == kHistQ16Const) {
            const int qv = sround(gv * gscale, uniform01(seed, r, 0), -32767, 32767);
            static_cast<int*>(gq)[k] = static_cast<int>((static_cast<unsigned int>(qv) << 1) | (sc ? 1u : 0u));
        } else if constexpr (kMode == kHistQ16Var) {
            const int qg = sround(gv * gscale, uniform01(seed, r, 0), -32767, 32767);
            const int qh = sround(hv * hscale, uniform01(seed, r, 1), 0, 65535);
            static_cast<unsigned int*>(gq)[k] = (static_cast<unsigned int>(qg) << 16) | static_cast<unsigned int>(qh);
        } else if constexpr (kMode == kHistQ8Const) {
            const int qv = sround(gv * gscale, uniform01(seed, r, 0), -127, 127);
            static_cast<short*>(gq)[k] = static_cast<short>((qv * 2) | (sc ? 1 : 0));
        } else {
            const int qg = sround(gv * gscale, uniform01(seed, r, 0), -127, 127);
            const int qh = sround(hv * hscale, uniform01(seed, r, 1), 0, 255);
            static_cast<unsigned short*>(gq)[k] = static_cast<unsigned short>((qg + 128) | (qh << 8));
        }
    }
}

__global__ void rows_max_kernel(const int32_t* __restrict__ rows, int n_rows, const double* __restrict__ g,
                                const double* __restrict__ h, AllScale* __restrict__ sc) {
    double mg = 0.0, mh = 0.0;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n_rows; k += gridDim.x * blockDim.x) {
        const int r = rows[k];
        mg = fmax(mg, fabs(g[r]));
        mh = fmax(mh, h ? fabs(h[r]) : 1.0);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mg = fmax(mg, __shfl_xor_sync(0xffffffffu, mg, o));
        mh = fmax(mh, __shfl_xor_sync(0xffffffffu, mh, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(&sc->maxg_bits, static_cast<unsigned long long>(__double_as_longlong(mg)));
        atomicMax(&sc->maxh_bits, static_cast<unsigned long long>(__double_as_longlong(mh)));
    }
}

template <typename K>
void set_smem(K kern, size_t bytes) {
    check(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes)),
          "wave hist smem attr");
}

// The shared-memory opt-in of each histogram instantiation, set once per device (never
// inside a stream capture: the first launches of a fit run before its graph is captured).
template <int kMode>
void ensure_smem() {
    static std::atomic<bool> done[64] = {};
    int dev = 0;
    check(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev >= 0 && dev < 64 && done[dev]) return;
    set_smem(wave_hist_kernel<kMode>, SmemLayout<kMode>::bytes);
    if (dev >= 0 && dev < 64) done[dev] = true;
}

template <int kMode>
void hist_launch(const WaveCtx* ctxs, int n_ctx, int src, HistTune tune, unsigned long long* rows_counter,
                 cudaStream_t s) {
    auto kern = wave_hist_kernel<kMode>;
    ensure_smem<kMode>();
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(1, tune.clusters * tune.cluster);
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = SmemLayout<kMode>::bytes;
    cfg.stream = s;
    cudaLaunchAttribute attr[2];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    attr[1].id = cudaLaunchAttributeClusterDimension;
    attr[1].val.clusterDim.x = 1;
    attr[1].val.clusterDim.y = tune.cluster;
    attr[1].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 2;
    check(cudaLaunchKernelEx(&cfg, kern, ctxs, n_ctx, src, rows_counter), "wave_hist launch");
}

template <int kMode>
void quantize_launch(const int32_t* rows, const double* g, const double* h, const uint8_t* flag, double gs,
                     const DevTreeState* st, unsigned long long seed, void* gq, void* hq, int blocks, cudaStream_t s) {
    wave_quantize_kernel<kMode><<<blocks, 256, 0, s>>>(rows, g, h, flag, gs, st, seed, gq, hq);
}

}  // namespace

int wave_hist_clusters(int cluster) {
    static std::atomic<int> cached[64][5] = {};
    int dev = 0;
    check(cudaGetDevice(&dev), "cudaGetDevice");
    ensure_smem<kHistExactConst>();
    ensure_smem<kHistExactVar>();
    ensure_smem<kHistQ16Const>();
    ensure_smem<kHistQ16Var>();
    ensure_smem<kHistQ8Const>();
    ensure_smem<kHistQ8Var>();
    cluster = cluster >= 4 ? 4 : cluster >= 2 ? 2 : 1;
    if (dev >= 0 && dev < 64 && cached[dev][cluster] > 0) return cached[dev][cluster];
    auto kern = wave_hist_kernel<kHistExactConst>;  // the largest shared-memory footprint
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(1, cluster * 64, 1);
    cfg.blockDim = dim3(kThreads, 1, 1);
    cfg.dynamicSmemBytes = SmemLayout<kHistExactConst>::bytes;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 1;
    attr[0].val.clusterDim.y = cluster;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int clusters = 0;
    if (cudaOccupancyMaxActiveClusters(&clusters, kern, &cfg) != cudaSuccess || clusters <= 0) {
        (void)cudaGetLastError();
        clusters = 148 / cluster;
    }
    if (dev >= 0 && dev < 64) cached[dev][cluster] = clusters;
    return clusters;
}

bool encode_codes_map(CUtensorMap* map, const uint8_t* codes, long long n_rows, int stride) {
    std::memset(map, 0, sizeof(*map));
    if (codes == nullptr || n_rows <= 0 || n_rows > 0x7fffffffll || stride < kFG || stride % 16 != 0 ||
        (reinterpret_cast<uintptr_t>(codes) & 15u) != 0)
        return false;
    using Encode = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
    static const Encode encode = [] {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            (void)cudaGetLastError();
            return static_cast<Encode>(nullptr);
        }
        return reinterpret_cast<Encode>(fn);
    }();
    if (encode == nullptr) return false;
    const cuuint64_t dims[2] = {static_cast<cuuint64_t>(stride), static_cast<cuuint64_t>(n_rows)};
    const cuuint64_t strides[1] = {static_cast<cuuint64_t>(stride)};
    const cuuint32_t box[2] = {static_cast<cuuint32_t>(kFG), 1u};  // gather4: one row high
    const cuuint32_t elem[2] = {1u, 1u};
    const CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<uint8_t*>(codes), dims, strides, box,
                              elem, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                              CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        std::memset(map, 0, sizeof(*map));
        return false;
    }
    return true;
}

void launch_wave_hist(int mode, const WaveCtx* ctxs, int n_ctx, int src, HistTune tune,
                      unsigned long long* rows_counter, cudaStream_t s) {
    switch (mode) {
        case kHistExactConst: hist_launch<kHistExactConst>(ctxs, n_ctx, src, tune, rows_counter, s); break;
        case kHistExactVar: hist_launch<kHistExactVar>(ctxs, n_ctx, src, tune, rows_counter, s); break;
        case kHistQ16Const: hist_launch<kHistQ16Const>(ctxs, n_ctx, src, tune, rows_counter, s); break;
        case kHistQ16Var: hist_launch<kHistQ16Var>(ctxs, n_ctx, src, tune, rows_counter, s); break;
        case kHistQ8Const: hist_launch<kHistQ8Const>(ctxs, n_ctx, src, tune, rows_counter, s); break;
        default: hist_launch<kHistQ8Var>(ctxs, n_ctx, src, tune, rows_counter, s); break;
    }
}

void launch_rows_max(const int32_t* rows, int n_rows, const double* g, const double* h, AllScale* sc,
                     cudaStream_t s) {
    if (n_rows <= 0) return;
    rows_max_kernel<<<std::max(1, std::min(1184, (n_rows + 255) / 256)), 256, 0, s>>>(rows, n_rows, g, h, sc);
    check(cudaGetLastError(), "rows_max launch");
}

void launch_wave_partition(const WaveCtx* ctxs, int n_ctx, int grid, cudaStream_t s) {
    launch_pdl(wave_part_count_kernel, dim3(grid), dim3(kPartThreads), 0, s, "wave_part_count launch", ctxs, n_ctx);
    launch_pdl(wave_part_scatter_kernel, dim3(grid), dim3(kPartThreads), 0, s, "wave_part_scatter launch", ctxs,
               n_ctx);
}

void launch_wave_tree_init(DevNode* nodes, DevSplit* splits, DevTreeState* st, WaveCtl* ctl, int n_sample_host,
                           int use_dev_count, cudaStream_t s) {
    wave_tree_init_kernel<<<1, 32, 0, s>>>(nodes, splits, st, ctl, n_sample_host, use_dev_count);
    check(cudaGetLastError(), "wave_tree_init launch");
}

void launch_wave_scales(DevTreeState* st, const AllScale* all, int mode, cudaStream_t s) {
    wave_scales_kernel<<<1, 1, 0, s>>>(st, all, mode);
    check(cudaGetLastError(), "wave_scales launch");
}

void launch_wave_quantize(int mode, const int32_t* rows, const double* g, const double* h, const uint8_t* goss_flag,
                          double goss_scale, const DevTreeState* st, unsigned long long seed, void* gq, void* hq,
                          int max_rows, cudaStream_t s) {
    const int blocks = std::max(1, std::min(1184, (max_rows + 255) / 256));
    switch (mode) {
        case kHistExactConst: quantize_launch<kHistExactConst>(rows, g, h, goss_flag, goss_scale, st, seed, gq, hq, blocks, s); break;
        case kHistExactVar: quantize_launch<kHistExactVar>(rows, g, h, goss_flag, goss_scale, st, seed, gq, hq, blocks, s); break;
        case kHistQ16Const: quantize_launch<kHistQ16Const>(rows, g, h, goss_flag, goss_scale, st, seed, gq, hq, blocks, s); break;
        case kHistQ16Var: quantize_launch<kHistQ16Var>(rows, g, h, goss_flag, goss_scale, st, seed, gq, hq, blocks, s); break;
        case kHistQ8Const: quantize_launch<kHistQ8Const>(rows, g, h, goss_flag, goss_scale, st, seed, gq, hq, blocks, s); break;
        default: quantize_launch<kHistQ8Var>(rows, g, h, goss_flag, goss_scale, st, seed, gq, hq, blocks, s); break;
    }
    check(cudaGetLastError(), "wave_quantize launch");
}

}  // namespace tgb
