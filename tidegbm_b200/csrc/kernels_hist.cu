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
// Launch shape: CTA = (group of 32 features) x (contiguous chunk of the node's row
// list), one CTA per SM.  A warp takes one row at a time and lane l owns feature l of
// the group: the warp reads the row's 32 code bytes with one coalesced 32-byte access,
// g and h are warp-uniform broadcasts, and each lane adds into bin (code_l, l) of the
// CTA-private shared histogram, stored at b*32 + l: every lane of a warp access owns its
// own bank whatever the codes are, and the features being distinct there are no
// same-address collisions either.
//
// Shared atomics are 32-bit only (the 64-bit shared add is not a single instruction):
// a 64-bit fixed-point value is added as two words, the low word with atomicAdd, whose
// returned old value tells whether this addition wrapped, then (high + carry) to the
// high word.  The words end up holding the exact 64-bit sum modulo 2^64.  For objectives
// with a constant hessian (mse with unit weights: h = 1, or 1 * goss_scale for sampled
// GOSS rows) the hessian and count sums are two 32-bit row counters, c1 (unscaled rows)
// and c2 (scaled rows): H = c1 * rint(2^hs) + c2 * rint(goss_scale * 2^hs), C = c1 + c2,
// the same integers the per-row sums give.  The private histogram is flushed to the
// node's global slot with one 64-bit global atomic per non-empty bin and value.
#include "tgb_internal.h"

#include <cmath>
#include <cooperative_groups.h>

namespace tgb {

namespace cg = cooperative_groups;

namespace {

constexpr int kHistThreads = 1024;
constexpr int kHistWarps = kHistThreads / 32;
constexpr int kMinRowsPerCta = 2048;
constexpr int kFG = 32;      // features per CTA (one per lane)
constexpr int kUnroll = 8;   // code loads in flight per warp
constexpr int kPlane = kFG * kBins;  // 32-bit words per plane

// Exact 64-bit add into a (low, high) pair of 32-bit shared words.
__device__ __forceinline__ void add64(unsigned int* lo, unsigned int* hi, int slot, unsigned long long v) {
    const unsigned int vlo = static_cast<unsigned int>(v);
    const unsigned int vhi = static_cast<unsigned int>(v >> 32);
    const unsigned int old = atomicAdd(&lo[slot], vlo);
    const unsigned int up = vhi + (old + vlo < old ? 1u : 0u);
    if (up != 0u) atomicAdd(&hi[slot], up);
}

template <bool kConstH>
__device__ __forceinline__ void hist_body(const uint8_t* __restrict__ codes, int stride, int n_f,
                                          const int32_t* __restrict__ rows, int count,
                                          const double* __restrict__ g, const double* __restrict__ h,
                                          const uint8_t* __restrict__ goss_flag, double goss_scale,
                                          double gscale, double hscale, long long* G, long long* H,
                                          int* C) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    unsigned int* gLo = reinterpret_cast<unsigned int*>(smem_raw);
    unsigned int* gHi = gLo + kPlane;
    // kConstH: c1, c2 row counters; otherwise hLo, hHi, count.
    unsigned int* p2 = gHi + kPlane;
    unsigned int* p3 = p2 + kPlane;
    unsigned int* p4 = p3 + kPlane;
    constexpr int n_planes = kConstH ? 4 : 5;

    // Row chunk of this CTA.
    const int need = (count + kMinRowsPerCta - 1) / kMinRowsPerCta;
    const int n_chunks = max(1, min(static_cast<int>(gridDim.y), need));
    if (static_cast<int>(blockIdx.y) >= n_chunks) return;
    const int chunk = (count + n_chunks - 1) / n_chunks;
    const int r0 = blockIdx.y * chunk;
    const int r1 = min(count, r0 + chunk);
    if (r0 >= r1) return;

    {
        uint4* z = reinterpret_cast<uint4*>(smem_raw);
        for (int k = threadIdx.x; k < n_planes * kPlane / 4; k += blockDim.x) z[k] = make_uint4(0, 0, 0, 0);
    }
    __syncthreads();

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int f = blockIdx.x * kFG + lane;
    const bool active = f < n_f;
    const int fo = active ? f : 0;  // in-bounds byte for idle lanes
    // A warp takes 32 rows at a time: lane j loads row j's index, g and h (one gather each),
    // then the warp walks the 32 rows, kBatch code loads in flight, with the row's index
    // and fixed-point values broadcast by shuffles.
    for (int base = r0 + warp * 32; base < r1; base += kHistWarps * 32) {
        const int nrow = min(32, r1 - base);
        const bool own = lane < nrow;
        const int rid = own ? rows[base + lane] : 0;
        unsigned long long gq = 0ull, hq = 0ull;
        int sc = 0;
        if (own) {
            double gv = g[rid];
            sc = goss_flag != nullptr && goss_flag[rid] == 2;
            if (sc) gv *= goss_scale;
            gq = static_cast<unsigned long long>(__double2ll_rn(gv * gscale));
            if (!kConstH) {
                double hv = h[rid];
                if (sc) hv *= goss_scale;
                hq = static_cast<unsigned long long>(__double2ll_rn(hv * hscale));
            }
        }
        for (int j0 = 0; j0 < nrow; j0 += kUnroll) {
            unsigned int cc[kUnroll];
#pragma unroll
            for (int u = 0; u < kUnroll; ++u) {
                const int j = j0 + u;
                const int rj = __shfl_sync(0xffffffffu, rid, j & 31);
                cc[u] = j < nrow ? codes[static_cast<size_t>(rj) * stride + fo] : 0u;
            }
#pragma unroll
            for (int u = 0; u < kUnroll; ++u) {
                const int j = j0 + u;
                const unsigned long long gj = __shfl_sync(0xffffffffu, gq, j & 31);
                const int sj = __shfl_sync(0xffffffffu, sc, j & 31);
                const unsigned long long hj = kConstH ? 0ull : __shfl_sync(0xffffffffu, hq, j & 31);
                if (j >= nrow || !active) continue;
                const int slot = static_cast<int>(cc[u]) * 32 + lane;
                add64(gLo, gHi, slot, gj);
                if (kConstH) {
                    atomicAdd(sj ? &p3[slot] : &p2[slot], 1u);
                } else {
                    add64(p2, p3, slot, hj);
                    atomicAdd(&p4[slot], 1u);
                }
            }
        }
    }
    __syncthreads();

    // Flush: warp w takes bins w, w + 32, ...; lane l = feature l (conflict-free reads).
    const int ff = blockIdx.x * kFG + lane;
    if (ff >= n_f) return;
    const unsigned long long hq1 = kConstH ? static_cast<unsigned long long>(__double2ll_rn(1.0 * hscale)) : 0ull;
    const unsigned long long hq2 =
        kConstH ? static_cast<unsigned long long>(__double2ll_rn(1.0 * goss_scale * hscale)) : 0ull;
    for (int b = warp; b < kBins; b += kHistWarps) {
        const int slot = b * 32 + lane;
        unsigned long long hsum;
        unsigned int c;
        if (kConstH) {
            const unsigned int c1 = p2[slot], c2 = p3[slot];
            c = c1 + c2;
            hsum = static_cast<unsigned long long>(c1) * hq1 + static_cast<unsigned long long>(c2) * hq2;
        } else {
            c = p4[slot];
            hsum = (static_cast<unsigned long long>(p3[slot]) << 32) | p2[slot];
        }
        if (c == 0u) continue;
        const unsigned long long gsum = (static_cast<unsigned long long>(gHi[slot]) << 32) | gLo[slot];
        const size_t o = static_cast<size_t>(ff) * kBins + b;
        atomicAdd(reinterpret_cast<unsigned long long*>(G) + o, gsum);
        atomicAdd(reinterpret_cast<unsigned long long*>(H) + o, hsum);
        atomicAdd(C + o, static_cast<int>(c));
    }
}

// ---- constant-hessian histogram (mse with unit weights, the GOSS workloads) ----------
//
// Lane = row.  A warp takes 32 rows, one per lane.  Each lane loads its row's 32 code
// bytes of the feature group with two 16-byte loads and rotates them in registers by
// `lane` bytes (a 3-stage word rotation by lane / 4, then a byte funnel-shift by
// lane % 4), so that step j of the 32-step loop reads the code of feature
// (j + lane) & 31.  All 32 lanes therefore touch 32 different features, i.e. 32
// different banks of the [bin][feature] layout, at every step.  Features past the end
// of the row read code 0 and add into cells that are never flushed, so the step loop
// has no bounds test.
//
// Per row the kernel gathers one int64 prepared by quantize_kernel for the tree:
// (v << 1) | s with v = rint(g * goss_factor * 2^gshift) and s = 1 for GOSS-scaled
// rows.  v (|v| < 2^37, enforced by the per-tree shift) is split into a 19-bit unsigned
// low part and a signed high part (v >> 19).  Over at most kSub = 8192 rows a bin's low
// sum stays below 2^32 and its high sum inside int32, so three fire-and-forget 32-bit
// shared reductions per code (low, high, packed counts c1 + c2<<16) are exact.  After
// every kSub rows the CTA folds the three planes into per-thread 64-bit register
// accumulators (each thread owns 8 fixed cells) and clears them.
constexpr int kSub = 8192;
constexpr int kLoBits = 19;
constexpr int kCells = kFG * kBins / kHistThreads;  // cells owned per thread (8)

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

// The CTAs of a cluster (kCluster consecutive row chunks of one feature group) add
// their partial histograms through distributed shared memory before the flush: each
// CTA writes its totals (G as two words, c1, c2) into its own shared memory, and after a
// cluster barrier CTA rank k sums cells [k, k+1) * kPlane / kCluster over the cluster and
// issues the global atomics for them, so a launch makes kCluster times fewer global
// atomics.  Every CTA of a cluster passes both cluster barriers: the only early exits
// (tree done, whole cluster past the node's chunk count) are uniform over a cluster.
constexpr int kCluster = 4;
constexpr size_t kConstSmem = static_cast<size_t>(kPlane) * 4 * 4;  // 3 accumulation planes, then 4 total planes

// kQ8 (the int8 precision mode): gq holds int16 (q << 1) | s per row, q in [-127, 127]
// the stochastically rounded g * goss_factor * gscale.  Each code then costs ONE 32-bit
// reduction, (1 << 20) | (q + 128), into the plane of its row class (unscaled / GOSS-
// scaled; the two planes share banks, so a warp mixing classes stays conflict-free):
// over kSub8 = 3072 rows the low 20 bits hold sum(q + 128) <= 255 * 3072 and the high 12
// the row count, exactly.
constexpr int kSub8 = 3072;

template <bool kQ8>
__global__ void __cluster_dims__(1, kCluster, 1) __launch_bounds__(kHistThreads)
    hist_node_const_kernel(const uint8_t* __restrict__ codes, int stride, int n_f, int32_t* rows0, int32_t* rows1,
                           const DevNode* __restrict__ nodes, const DevTreeState* __restrict__ st, int node,
                           const void* __restrict__ gq_any, double goss_scale, HistSlotPtrs hs,
                           unsigned long long* rows_counter) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    unsigned int* pLo = reinterpret_cast<unsigned int*>(smem_raw);  // kQ8: class-1 plane
    unsigned int* pHi = pLo + kPlane;                               // kQ8: class-2 plane
    unsigned int* pCn = pHi + kPlane;
    constexpr int kPlanes = kQ8 ? 2 : 3;
    constexpr int kSubRows = kQ8 ? kSub8 : kSub;
    const long long* __restrict__ gq = static_cast<const long long*>(gq_any);
    const short* __restrict__ gq8 = static_cast<const short*>(gq_any);
    {  // private state first: it overlaps the previous kernel's tail
        uint4* z = reinterpret_cast<uint4*>(smem_raw);
        for (int k = threadIdx.x; k < kPlanes * kPlane / 4; k += blockDim.x) z[k] = make_uint4(0, 0, 0, 0);
    }
    pdl_wait();
    pdl_trigger();
    if (st->done || (node < 0 && st->small_node < 0)) return;  // uniform over the grid
    const int nd = node >= 0 ? node : st->small_node;
    const DevNode& N = nodes[nd];
    const int32_t* rows = (N.buf ? rows1 : rows0) + N.start;
    const int count = N.count;
    if (rows_counter != nullptr && blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0)
        atomicAdd(rows_counter, static_cast<unsigned long long>(count));
    long long* G = hs.G + nd * hs.slot_elems;
    long long* H = hs.H + nd * hs.slot_elems;
    int* C = hs.C + nd * hs.slot_elems;
    const double hscale = st->hscale;

    // Row chunks: a multiple of kCluster, so whole clusters are active or idle.
    const int need = (count + kMinRowsPerCta - 1) / kMinRowsPerCta;
    const int n_chunks = min(static_cast<int>(gridDim.y), (max(1, need) + kCluster - 1) / kCluster * kCluster);
    if (static_cast<int>(blockIdx.y) >= n_chunks) return;  // uniform over the cluster
    const int chunk = (count + n_chunks - 1) / n_chunks;
    const int r0 = min(count, static_cast<int>(blockIdx.y) * chunk);
    const int r1 = min(count, r0 + chunk);

    long long accG[kCells];
    unsigned int accC1[kCells], accC2[kCells];
#pragma unroll
    for (int c = 0; c < kCells; ++c) {
        accG[c] = 0;
        accC1[c] = accC2[c] = 0u;
    }
    __syncthreads();

    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int fg0 = blockIdx.x * kFG;
    const int nf_here = min(kFG, n_f - fg0);
    // stride and fg0 are multiples of 16 and 32: the group has 16 or >= 32 bytes in a row
    const bool two_chunks = stride - fg0 >= 32;
    const int q = lane >> 2, sh = (lane & 3) * 8;
    for (int s0 = r0; s0 < r1; s0 += kSubRows) {
        const int s1 = min(r1, s0 + kSubRows);
        // the next row id is loaded one iteration ahead, so each iteration waits for one
        // memory round trip (its row's g and codes) instead of two
        int r_next = s0 + warp * 32 + lane < s1 ? rows[s0 + warp * 32 + lane] : -1;
        for (int base = s0 + warp * 32; base < s1; base += kHistWarps * 32) {
            const int r = r_next;
            const int kn = base + kHistWarps * 32 + lane;
            r_next = kn < s1 ? rows[kn] : -1;
            if (r >= 0) {
                unsigned int lo = 0, hi = 0, inc = 0, word = 0;
                unsigned int* plane = pLo;
                if (kQ8) {
                    const int p8 = gq8[r];
                    word = (1u << 20) | static_cast<unsigned int>((p8 >> 1) + 128);
                    plane = (p8 & 1) ? pHi : pLo;
                } else {
                    const long long p = gq[r];
                    const long long v = p >> 1;
                    lo = static_cast<unsigned int>(v) & ((1u << kLoBits) - 1u);
                    hi = static_cast<unsigned int>(static_cast<int>(v >> kLoBits));
                    inc = (p & 1) ? 0x10000u : 1u;
                }
                const uint4* src = reinterpret_cast<const uint4*>(codes + static_cast<size_t>(r) * stride + fg0);
                const uint4 a = __ldg(src);
                const uint4 b = two_chunks ? __ldg(src + 1) : make_uint4(0, 0, 0, 0);
                unsigned int w[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
                rotate_words(w, q);
                unsigned int R[8];
#pragma unroll
                for (int t = 0; t < 8; ++t) R[t] = __funnelshift_r(w[t], w[(t + 1) & 7], sh);
#pragma unroll
                for (int j = 0; j < 32; ++j) {
                    const int f = (j + lane) & 31;
                    const unsigned int code = (R[j >> 2] >> ((j & 3) * 8)) & 0xffu;
                    const int cell = static_cast<int>(code) * 32 + f;
                    if (kQ8) {
                        atomicAdd(&plane[cell], word);
                    } else {
                        atomicAdd(&pLo[cell], lo);
                        atomicAdd(&pHi[cell], hi);
                        atomicAdd(&pCn[cell], inc);
                    }
                }
            }
        }
        __syncthreads();
#pragma unroll
        for (int c = 0; c < kCells; ++c) {
            const int cell = threadIdx.x + c * kHistThreads;
            if (kQ8) {
                const unsigned int w1 = pLo[cell], w2 = pHi[cell];
                const unsigned int n1 = w1 >> 20, n2 = w2 >> 20;
                accG[c] += static_cast<long long>(w1 & 0xfffffu) + static_cast<long long>(w2 & 0xfffffu) -
                           128ll * static_cast<long long>(n1 + n2);
                accC1[c] += n1;
                accC2[c] += n2;
                pLo[cell] = pHi[cell] = 0u;
            } else {
                accG[c] += static_cast<long long>(static_cast<int>(pHi[cell])) * (1ll << kLoBits) + pLo[cell];
                const unsigned int cn = pCn[cell];
                accC1[c] += cn & 0xffffu;
                accC2[c] += cn >> 16;
                pLo[cell] = pHi[cell] = pCn[cell] = 0u;
            }
        }
        __syncthreads();
    }

    // This CTA's totals -> 4 planes of its shared memory.
    unsigned int* tot = reinterpret_cast<unsigned int*>(smem_raw);
#pragma unroll
    for (int c = 0; c < kCells; ++c) {
        const int cell = threadIdx.x + c * kHistThreads;
        tot[cell] = static_cast<unsigned int>(accG[c]);
        tot[kPlane + cell] = static_cast<unsigned int>(static_cast<unsigned long long>(accG[c]) >> 32);
        tot[2 * kPlane + cell] = accC1[c];
        tot[3 * kPlane + cell] = accC2[c];
    }
    cg::cluster_group cluster = cg::this_cluster();
    cluster.sync();
    // Rank k flushes its share of the cells, summed over the cluster.
    const unsigned int rank = cluster.block_rank();
    const unsigned long long hq1 = static_cast<unsigned long long>(__double2ll_rn(1.0 * hscale));
    const unsigned long long hq2 = static_cast<unsigned long long>(__double2ll_rn(1.0 * goss_scale * hscale));
    constexpr int kShare = kPlane / kCluster;
    for (int cell = rank * kShare + threadIdx.x; cell < static_cast<int>(rank + 1) * kShare; cell += kHistThreads) {
        unsigned long long g = 0;
        unsigned int c1 = 0, c2 = 0;
#pragma unroll
        for (int k = 0; k < kCluster; ++k) {
            const unsigned int* rt = cluster.map_shared_rank(tot, k);
            g += (static_cast<unsigned long long>(rt[kPlane + cell]) << 32) | rt[cell];
            c1 += rt[2 * kPlane + cell];
            c2 += rt[3 * kPlane + cell];
        }
        const int b = cell >> 5, f = cell & 31;
        const unsigned int cn = c1 + c2;
        if (f >= nf_here || cn == 0u) continue;
        const size_t o = static_cast<size_t>(fg0 + f) * kBins + b;
        atomicAdd(reinterpret_cast<unsigned long long*>(G) + o, g);
        atomicAdd(reinterpret_cast<unsigned long long*>(H) + o,
                  static_cast<unsigned long long>(c1) * hq1 + static_cast<unsigned long long>(c2) * hq2);
        atomicAdd(C + o, static_cast<int>(cn));
    }
    cluster.sync();  // no CTA leaves while others read its shared memory
}

// int8 precision mode: gq8[r] = (q << 1) | (GOSS-scaled ? 1 : 0) for the sampled rows,
// q = floor(x + u) with x = g[r] * goss_factor * gscale in [-127, 127] (gscale =
// 127 / max |g * factor| over the sample) and u in [0, 1) from a counter-based hash of
// (row, tree, seed): stochastic rounding, unbiased (E[q] = x) and reproducible.  The hash
// is the SplitMix64 output function (Steele, Lea and Flood, OOPSLA 2014).
__device__ __forceinline__ unsigned long long splitmix64(unsigned long long z) {
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

__global__ void quantize8_kernel(const int32_t* __restrict__ rows, const double* __restrict__ g,
                                 const uint8_t* __restrict__ goss_flag, double goss_scale,
                                 const DevTreeState* __restrict__ st, unsigned long long seed,
                                 short* __restrict__ gq8) {
    const int count = st->n_sample;
    const double gscale = st->gscale;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x) {
        const int r = rows[k];
        double gv = g[r];
        const bool sc = goss_flag != nullptr && goss_flag[r] == 2;
        if (sc) gv *= goss_scale;
        const double x = gv * gscale;
        const double u = static_cast<double>(splitmix64(seed ^ (static_cast<unsigned long long>(r) << 20)) >> 11) *
                         (1.0 / 9007199254740992.0);  // 53 bits -> [0, 1)
        const int q = max(-127, min(127, static_cast<int>(floor(x + u))));
        gq8[r] = static_cast<short>((q * 2) | (sc ? 1 : 0));
    }
}

// gq[r] = (rint(g[r] * goss_factor * 2^gshift) << 1) | (GOSS-scaled ? 1 : 0) for the rows
// of the tree's sample: the same fixed-point value the general kernel computes per code.
__global__ void quantize_kernel(const int32_t* __restrict__ rows, const double* __restrict__ g,
                                const uint8_t* __restrict__ goss_flag, double goss_scale,
                                const DevTreeState* __restrict__ st, long long* __restrict__ gq) {
    const int count = st->n_sample;
    const double gscale = st->gscale;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < count; k += gridDim.x * blockDim.x) {
        const int r = rows[k];
        double gv = g[r];
        const bool sc = goss_flag != nullptr && goss_flag[r] == 2;
        if (sc) gv *= goss_scale;
        const long long v = __double2ll_rn(gv * gscale);
        gq[r] = static_cast<long long>((static_cast<unsigned long long>(v) << 1) | (sc ? 1ull : 0ull));
    }
}

template <bool kConstH>
__global__ void __launch_bounds__(kHistThreads)
    hist_node_kernel(const uint8_t* __restrict__ codes, int stride, int n_f, int32_t* rows0,
                     int32_t* rows1, const DevNode* __restrict__ nodes,
                     const DevTreeState* __restrict__ st, int node, const double* __restrict__ g,
                     const double* __restrict__ h, const uint8_t* __restrict__ goss_flag,
                     double goss_scale, HistSlotPtrs hs, unsigned long long* rows_counter) {
    if (st->done || (node < 0 && st->small_node < 0)) return;
    const int nd = node >= 0 ? node : st->small_node;
    const DevNode& N = nodes[nd];
    const int32_t* rows = (N.buf ? rows1 : rows0) + N.start;
    // Rows histogrammed, for the algorithmic-bytes figure of the benchmark.
    if (rows_counter != nullptr && blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0)
        atomicAdd(rows_counter, static_cast<unsigned long long>(N.count));
    hist_body<kConstH>(codes, stride, n_f, rows, N.count, g, h, goss_flag, goss_scale, st->gscale, st->hscale,
                       hs.G + nd * hs.slot_elems, hs.H + nd * hs.slot_elems, hs.C + nd * hs.slot_elems);
}

__global__ void __launch_bounds__(kHistThreads)
    hist_rows_kernel(const uint8_t* __restrict__ codes, int stride, int n_f, const int32_t* __restrict__ rows,
                     int count, const double* __restrict__ g, const double* __restrict__ h, double gscale,
                     double hscale, long long* G, long long* H, int* C) {
    hist_body<false>(codes, stride, n_f, rows, count, g, h, nullptr, 1.0, gscale, hscale, G, H, C);
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
}

__global__ void iota_kernel(int32_t* rows, int n) {
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) rows[k] = k;
}

// Largest shift with count * max_abs * 2^s < 2^62 (no sum can overflow) and
// max_abs * 2^s < 2^37 (one row's value fits the split low/high words of
// hist_const_body); the per-row resolution is then 2^-37 of the largest |value| or finer.
__device__ int shift_for(double max_abs, int count) {
    if (!(max_abs > 0.0) || count <= 0) return 0;
    int clog = 0;
    while ((1ll << clog) < static_cast<long long>(count)) ++clog;
    const int e = ilogb(max_abs);
    int s = min(61 - (e + 1) - clog, 36 - e);
    return max(-1000, min(1000, s));
}

// all != nullptr: the sample is every row, whose maxima the gradient pass reduced.
// q8: the gradient scale maps max |g * factor| to 127 (int8 precision mode).
__global__ void scales_finalize_kernel(DevTreeState* st, const AllScale* __restrict__ all, int q8) {
    if (all) {
        st->max_abs_g_bits = all->maxg_bits;
        st->max_h_bits = all->maxh_bits;
    }
    const double mg = __longlong_as_double(static_cast<long long>(st->max_abs_g_bits));
    const double mh = __longlong_as_double(static_cast<long long>(st->max_h_bits));
    st->hshift = shift_for(mh, st->n_sample);
    st->hscale = ldexp(1.0, st->hshift);
    st->inv_hscale = ldexp(1.0, -st->hshift);
    if (q8) {
        st->gshift = 0;
        st->gscale = mg > 0.0 ? 127.0 / mg : 1.0;
        st->inv_gscale = 1.0 / st->gscale;
    } else {
        st->gshift = shift_for(mg, st->n_sample);
        st->gscale = ldexp(1.0, st->gshift);
        st->inv_gscale = ldexp(1.0, -st->gshift);
    }
}

constexpr size_t hist_smem(bool const_h) { return static_cast<size_t>(kPlane) * 4 * (const_h ? 4 : 5); }

template <typename K>
void set_smem(K kern, size_t bytes) {
    check(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(bytes)),
          "hist smem attr");
}

}  // namespace

int hist_grid_rows(int n_f, int max_rows, bool const_h) {
    const int groups = (n_f + kFG - 1) / kFG;
    const int need = (max_rows + kMinRowsPerCta - 1) / kMinRowsPerCta;
    if (!const_h) return std::max(1, std::min(need, (148 + groups - 1) / groups));
    // Clusters that fit on the device at once, shared among the feature groups.
    set_smem(hist_node_const_kernel<false>, kConstSmem);
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(groups, kCluster, 1);
    cfg.blockDim = dim3(kHistThreads, 1, 1);
    cfg.dynamicSmemBytes = kConstSmem;
    int clusters = 0;
    if (cudaOccupancyMaxActiveClusters(&clusters, hist_node_const_kernel<false>, &cfg) != cudaSuccess ||
        clusters <= 0) {
        (void)cudaGetLastError();
        clusters = 148 / kCluster;
    }
    const int per_group = std::max(1, clusters / groups);
    const int need_c = std::max(1, (need + kCluster - 1) / kCluster);
    return std::min(per_group, need_c) * kCluster;
}

void launch_hist_node(const uint8_t* codes, int stride, int n_f, int32_t* const* rows,
                      const DevNode* nodes, const DevTreeState* st, int node, const double* g,
                      const double* h, const void* gq, bool q8, const uint8_t* goss_flag, double goss_scale,
                      HistSlotPtrs hs, int grid_rows, unsigned long long* rows_counter, bool const_h,
                      cudaStream_t s) {
    dim3 grid((n_f + kFG - 1) / kFG, max(1, grid_rows));
    if (const_h) {
        auto kern = q8 ? hist_node_const_kernel<true> : hist_node_const_kernel<false>;
        set_smem(kern, kConstSmem);
        launch_pdl(kern, grid, dim3(kHistThreads), kConstSmem, s, "hist_node launch", codes, stride, n_f, rows[0],
                   rows[1], nodes, st, node, gq, goss_scale, hs, rows_counter);
        return;
    } else {
        set_smem(hist_node_kernel<false>, hist_smem(false));
        hist_node_kernel<false><<<grid, kHistThreads, hist_smem(false), s>>>(
            codes, stride, n_f, rows[0], rows[1], nodes, st, node, g, h, goss_flag, goss_scale, hs, rows_counter);
    }
    check(cudaGetLastError(), "hist_node launch");
}

void launch_quantize8(const int32_t* rows, const double* g, const uint8_t* goss_flag, double goss_scale,
                      const DevTreeState* st, unsigned long long seed, short* gq8, int max_rows, cudaStream_t s) {
    const int blocks = std::max(1, std::min(1184, (max_rows + 255) / 256));
    quantize8_kernel<<<blocks, 256, 0, s>>>(rows, g, goss_flag, goss_scale, st, seed, gq8);
    check(cudaGetLastError(), "quantize8 launch");
}

void launch_quantize(const int32_t* rows, const double* g, const uint8_t* goss_flag, double goss_scale,
                     const DevTreeState* st, long long* gq, int max_rows, cudaStream_t s) {
    const int blocks = std::max(1, std::min(1184, (max_rows + 255) / 256));
    quantize_kernel<<<blocks, 256, 0, s>>>(rows, g, goss_flag, goss_scale, st, gq);
    check(cudaGetLastError(), "quantize launch");
}

void launch_hist_rows(const uint8_t* codes, int stride, int n_f, const int32_t* rows, int n_rows,
                      const double* g, const double* h, int gshift, int hshift, long long* G,
                      long long* H, int* C, cudaStream_t s) {
    if (n_rows <= 0) return;
    set_smem(hist_rows_kernel, hist_smem(false));
    dim3 grid((n_f + kFG - 1) / kFG, hist_grid_rows(n_f, n_rows, false));
    hist_rows_kernel<<<grid, kHistThreads, hist_smem(false), s>>>(codes, stride, n_f, rows, n_rows, g, h,
                                                           std::ldexp(1.0, gshift), std::ldexp(1.0, hshift), G, H,
                                                           C);
    check(cudaGetLastError(), "hist_rows launch");
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

void launch_scales(DevTreeState* st, const AllScale* all, bool q8, cudaStream_t s) {
    scales_finalize_kernel<<<1, 1, 0, s>>>(st, all, q8 ? 1 : 0);
    check(cudaGetLastError(), "scales_finalize launch");
}

}  // namespace tgb
