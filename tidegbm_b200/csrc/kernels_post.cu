// Per-tree sweep over all rows after a tree is grown.  Restates
// Booster::fit's grow_head tail (cpp/src/booster.cpp:589-664):
//   apply_all (cpp/src/tree.cpp:43-55)           leaf id of every row
//   full-data leaf values                        leaf_value(sum g, sum h) over ALL rows,
//                                                unscaled g and h (booster.cpp:594-600)
//   TORB prefix values                           per time bucket b, leaf values from the
//                                                rows [0, cut_b) of its causal past,
//                                                blended toward the full value when the
//                                                past is short (booster.cpp:604-648)
//   prediction update                            pred += lr * prefix[bucket][leaf]
//                                                (booster.cpp:655-664)
//
// Rows are sorted by time, so every cut is a row position and the rows between two
// consecutive distinct cuts form a segment.  apply_accum sums (g, h, 1) per
// (segment, leaf) in exact 64-bit fixed point (one shift per tree from max |g|,
// max h over all rows); finalize turns segment sums into prefix sums per bucket.
// CTAs own segment-aligned row chunks, so each CTA accumulates into one segment in
// shared memory (32-bit atomics) and adds its totals to the segment with one global
// 64-bit atomic per leaf and value.
#include <atomic>
#include "tgb_internal.h"

namespace tgb {

namespace {

constexpr int kApplyThreads = 256;

__device__ int shift_for_all(double max_abs, long long count) {
    if (!(max_abs > 0.0) || count <= 0) return 0;
    int clog = 0;
    while ((1ll << clog) < count) ++clog;
    const int e = ilogb(max_abs);
    return max(-1000, min(1000, 61 - (e + 1) - clog));
}

__global__ void max_abs_kernel(const double* __restrict__ g, const double* __restrict__ h, int n,
                               AllScale* __restrict__ sc) {
    double mg = 0.0, mh = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        mg = fmax(mg, fabs(g[i]));
        mh = fmax(mh, fabs(h[i]));
    }
    for (int o = 16; o > 0; o >>= 1) {
        mg = fmax(mg, __shfl_xor_sync(0xffffffffu, mg, o));
        mh = fmax(mh, __shfl_xor_sync(0xffffffffu, mh, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(&sc->maxg_bits, static_cast<unsigned long long>(__double_as_longlong(mg)));
        atomicMax(&sc->maxh_bits, static_cast<unsigned long long>(__double_as_longlong(mh)));
    }
}

__global__ void all_scale_finalize_kernel(AllScale* sc, int n) {
    const double mg = __longlong_as_double(static_cast<long long>(sc->maxg_bits));
    const double mh = __longlong_as_double(static_cast<long long>(sc->maxh_bits));
    sc->gshift = shift_for_all(mg, n);
    sc->hshift = shift_for_all(mh, n);
    sc->gscale = ldexp(1.0, sc->gshift);
    sc->hscale = ldexp(1.0, sc->hshift);
    sc->inv_gscale = ldexp(1.0, -sc->gshift);
    sc->inv_hscale = ldexp(1.0, -sc->hshift);
}

// Exact 64-bit add into (low, high) 32-bit shared words: the low word's returned old
// value says whether this addition wrapped; the carry goes to the high word.
__device__ __forceinline__ void add64s(unsigned int* lo, unsigned int* hi, int k, unsigned long long v) {
    const unsigned int vlo = static_cast<unsigned int>(v);
    const unsigned int old = atomicAdd(&lo[k], vlo);
    const unsigned int up = static_cast<unsigned int>(v >> 32) + (old + vlo < old ? 1u : 0u);
    if (up != 0u) atomicAdd(&hi[k], up);
}

constexpr int kApplyRows = 8;  // rows a thread walks together

// Staged walk: a block stages, per tile of kStageRows rows, only the columns the tree
// splits on (each distinct split feature once, 16-byte loads of whole tile runs) in shared
// memory and walks its rows there: a row costs one byte per distinct split feature
// instead of one 32-byte sector share per level.  Trees over more than kMaxStaged distinct
// columns (or more than kMaxColWords * 32 features) take the gather walk: at each level
// the kApplyRows rows of a thread issue their column-major code loads together, and lanes
// at nodes with the same split feature share a sector.
constexpr int kStageRows = 512;
constexpr int kStagePitch = kStageRows + 16;  // a tile run starts up to 15 bytes early (16-byte loads)
constexpr int kMaxStaged = 64;
constexpr int kMaxColWords = 256;
constexpr size_t kApplySmem = static_cast<size_t>(kMaxStaged) * kStagePitch;

// kKinds: bit 0 the tree may hold categorical splits, bit 1 pair splits; a tree of axis
// splits only keeps neither the masks nor the second features in shared memory.
template <int kKinds>
__global__ void __launch_bounds__(kApplyThreads, 3)
    apply_accum_kernel(const uint8_t* __restrict__ col, long long pitch, int n_f, const DevNode* __restrict__ nodes,
                       const DevTreeState* __restrict__ st, const double* __restrict__ g,
                       const double* __restrict__ h, const int4* __restrict__ chunks,
                       int n_chunks, const AllScale* __restrict__ sc, int16_t* __restrict__ nid,
                       unsigned long long* __restrict__ seg_sums, int n_bins) {
    constexpr bool kCat = (kKinds & 1) != 0, kPair = (kKinds & 2) != 0;
    extern __shared__ __align__(16) uint8_t s_tile[];  // [kMaxStaged][kStagePitch]
    __shared__ int16_t s_feat[kMaxNodes], s_left[kMaxNodes], s_right[kMaxNodes];
    __shared__ uint8_t s_thr[kMaxNodes], s_ml[kMaxNodes], s_leaf[kMaxNodes], s_type[kMaxNodes];
    __shared__ int16_t s_feat2[kPair ? kMaxNodes : 1];
    __shared__ unsigned long long s_cat[kCat ? kMaxNodes : 1][4];  // left masks of categorical nodes
    __shared__ unsigned int s_bits[kMaxColWords];
    __shared__ int s_wbase[kMaxColWords], s_uf[kMaxStaged], s_nu;
    // staged walk: a node in one word (left 0-15, right 16-31, threshold 32-39, staged column
    // 40-47, missing_left 48, is_leaf 49, split type 50-51, second staged column 52-59)
    __shared__ unsigned long long s_word[kMaxNodes];
    // 64-bit sums as (low, high) 32-bit words: shared atomics stay single 32-bit operations.
    __shared__ unsigned int aGl[kMaxNodes], aGh[kMaxNodes], aHl[kMaxNodes], aHh[kMaxNodes], aC[kMaxNodes];
    const int nn = st->n_nodes;
    const int n_words = (n_f + 31) / 32;
    const bool can_stage = n_words <= kMaxColWords;
    if (can_stage)
        for (int w = threadIdx.x; w < n_words; w += blockDim.x) s_bits[w] = 0u;
    __syncthreads();
    for (int k = threadIdx.x; k < nn; k += blockDim.x) {
        const DevNode& N = nodes[k];
        s_feat[k] = static_cast<int16_t>(N.feature);
        s_left[k] = static_cast<int16_t>(N.left);
        s_right[k] = static_cast<int16_t>(N.right);
        s_thr[k] = static_cast<uint8_t>(N.threshold < 0 ? 0 : N.threshold);
        s_ml[k] = static_cast<uint8_t>(N.missing_left);
        s_type[k] = static_cast<uint8_t>(N.is_leaf ? 0 : N.type);
        if constexpr (kPair) s_feat2[k] = static_cast<int16_t>(!N.is_leaf && N.type == 1 ? N.feature2 : 0);
        if constexpr (kCat)
            for (int q = 0; q < 4; ++q) s_cat[k][q] = N.type == 2 ? N.cat[q] : 0ull;
        s_leaf[k] = static_cast<uint8_t>(N.is_leaf);
        aGl[k] = aGh[k] = aHl[k] = aHh[k] = aC[k] = 0u;
        if (can_stage && !N.is_leaf) {
            atomicOr(&s_bits[N.feature >> 5], 1u << (N.feature & 31));
            if (kPair && N.type == 1) atomicOr(&s_bits[N.feature2 >> 5], 1u << (N.feature2 & 31));
        }
    }
    __syncthreads();
    if (can_stage) {
        // distinct split columns: ranks by an exclusive prefix of the bitmap's popcounts
        if (threadIdx.x < 32) {
            const int lane = threadIdx.x;
            int run = 0;
            for (int w0 = 0; w0 < n_words; w0 += 32) {
                const int w = w0 + lane;
                const int c = w < n_words ? __popc(s_bits[w]) : 0;
                int incl = c;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int t = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= o) incl += t;
                }
                if (w < n_words) s_wbase[w] = run + incl - c;
                run += __shfl_sync(0xffffffffu, incl, 31);
            }
            if (lane == 0) s_nu = run;
        }
        __syncthreads();
        if (s_nu <= kMaxStaged) {
            for (int w = threadIdx.x; w < n_words; w += blockDim.x) {
                unsigned int bits = s_bits[w];
                int u = s_wbase[w];
                while (bits != 0u) {
                    s_uf[u++] = w * 32 + __ffs(bits) - 1;
                    bits &= bits - 1u;
                }
            }
            auto rank = [&](int f) {
                return s_wbase[f >> 5] + __popc(s_bits[f >> 5] & ((1u << (f & 31)) - 1u));
            };
            for (int k = threadIdx.x; k < nn; k += blockDim.x) {
                unsigned long long w = static_cast<unsigned long long>(static_cast<uint16_t>(s_left[k])) |
                                       static_cast<unsigned long long>(static_cast<uint16_t>(s_right[k])) << 16 |
                                       static_cast<unsigned long long>(s_thr[k]) << 32 |
                                       static_cast<unsigned long long>(s_ml[k] & 1) << 48 |
                                       static_cast<unsigned long long>(s_leaf[k] & 1) << 49 |
                                       static_cast<unsigned long long>(s_type[k] & 3) << 50;
                if (!s_leaf[k]) {
                    w |= static_cast<unsigned long long>(rank(s_feat[k])) << 40;
                    if constexpr (kPair)
                        if (s_type[k] == 1) w |= static_cast<unsigned long long>(rank(s_feat2[k])) << 52;
                }
                s_word[k] = w;
            }
        }
        __syncthreads();
    }
    const bool staged = can_stage && s_nu <= kMaxStaged;
    const double gs = sc->gscale, hs = sc->hscale;
    // unit hessians (h == nullptr): every row adds the same fixed-point 1, so H = count x that
    const unsigned long long h1 = static_cast<unsigned long long>(__double2ll_rn(1.0 * hs));
    // a CTA takes chunks in turn (the node tables above are staged once per CTA)
    for (int ci = blockIdx.x; ci < n_chunks; ci += gridDim.x) {
        const int4 ch = chunks[ci];  // {segment, row start, row end, unused}
        if (staged) {
            const int nu = s_nu;
            for (int t0 = ch.y; t0 < ch.z; t0 += kStageRows) {
                const int t1 = min(ch.z, t0 + kStageRows);
                const int a0 = t0 & ~15;
                const int n16 = (t1 - a0 + 15) >> 4;
                __syncthreads();  // the previous tile's walks are done
                {  // a warp per staged column, a lane per 16 bytes of its run
                    const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
                    for (int u = threadIdx.x >> 5; u < nu; u += nw) {
                        const uint4* src = reinterpret_cast<const uint4*>(col + static_cast<long long>(s_uf[u]) * pitch + a0);
                        uint4* dst = reinterpret_cast<uint4*>(s_tile + u * kStagePitch);
                        for (int v = lane; v < n16; v += 32) dst[v] = __ldg(src + v);
                    }
                }
                __syncthreads();
                for (int r = t0 + threadIdx.x; r < t1; r += blockDim.x) {
                    const double gv = g[r];
                    const double hv = h ? h[r] : 1.0;  // h == nullptr: unit hessians
                    const uint8_t* trow = s_tile + (r - a0);
                    int k = 0;
                    unsigned long long w = s_word[0];
                    while (!((w >> 49) & 1ull)) {
                        const unsigned int b = trow[((w >> 40) & 0xffu) * kStagePitch];
                        const unsigned int thr = static_cast<unsigned int>(w >> 32) & 0xffu;
                        const bool ml = (w >> 48) & 1ull;
                        bool left;
                        if constexpr (kCat || kPair) {
                            const int type = static_cast<int>(w >> 50) & 3;
                            unsigned int b2 = 0u;
                            if constexpr (kPair)
                                if (type == 1) b2 = trow[((w >> 52) & 0xffu) * kStagePitch];
                            left = goes_left(type, s_cat[kCat ? k : 0], static_cast<int>(thr), ml, b, b2, n_bins);
                        } else {
                            left = b == 0u ? ml : b <= thr;
                        }
                        k = left ? static_cast<int>(w & 0xffffu) : static_cast<int>((w >> 16) & 0xffffu);
                        w = s_word[k];
                    }
                    nid[r] = static_cast<int16_t>(k);
                    add64s(aGl, aGh, k, static_cast<unsigned long long>(__double2ll_rn(gv * gs)));
                    if (h != nullptr) add64s(aHl, aHh, k, static_cast<unsigned long long>(__double2ll_rn(hv * hs)));
                    atomicAdd(&aC[k], 1u);
                }
            }
        } else {
            for (int base = ch.y; base < ch.z; base += kApplyThreads * kApplyRows) {
                int r[kApplyRows], k[kApplyRows];
                double gv[kApplyRows], hv[kApplyRows];
    #pragma unroll
                for (int i = 0; i < kApplyRows; ++i) {
                    r[i] = base + threadIdx.x + i * kApplyThreads;
                    k[i] = 0;
                    const bool ok = r[i] < ch.z;
                    gv[i] = ok ? g[r[i]] : 0.0;  // loaded before the walk so their latency overlaps it
                    hv[i] = ok && h ? h[r[i]] : 1.0;
                    if (!ok) r[i] = -1;
                }
                for (int level = 0; level < kMaxNodes; ++level) {  // a path has fewer than kMaxNodes nodes
                    unsigned int b[kApplyRows], b2[kApplyRows];
                    bool any = false;
    #pragma unroll
                    for (int i = 0; i < kApplyRows; ++i) {
                        const bool walk = r[i] >= 0 && !s_leaf[k[i]];
                        b[i] = walk ? __ldg(col + static_cast<long long>(s_feat[k[i]]) * pitch + r[i]) : 0u;
                        if constexpr (kPair)
                            b2[i] = walk && s_type[k[i]] == 1
                                        ? __ldg(col + static_cast<long long>(s_feat2[k[i]]) * pitch + r[i])
                                        : 0u;
                        else
                            b2[i] = 0u;
                        any |= walk;
                    }
                    if (!any) break;
    #pragma unroll
                    for (int i = 0; i < kApplyRows; ++i) {
                        if (r[i] < 0 || s_leaf[k[i]]) continue;
                        bool left;
                        if constexpr (kCat || kPair)
                            left = goes_left(s_type[k[i]], s_cat[kCat ? k[i] : 0], s_thr[k[i]], s_ml[k[i]], b[i], b2[i],
                                             n_bins);
                        else
                            left = b[i] == 0u ? s_ml[k[i]] != 0 : static_cast<int>(b[i]) <= s_thr[k[i]];
                        k[i] = left ? s_left[k[i]] : s_right[k[i]];
                    }
                }
    #pragma unroll
                for (int i = 0; i < kApplyRows; ++i) {
                    if (r[i] < 0) continue;
                    nid[r[i]] = static_cast<int16_t>(k[i]);
                    add64s(aGl, aGh, k[i], static_cast<unsigned long long>(__double2ll_rn(gv[i] * gs)));
                    if (h != nullptr)
                        add64s(aHl, aHh, k[i], static_cast<unsigned long long>(__double2ll_rn(hv[i] * hs)));
                    atomicAdd(&aC[k[i]], 1u);
                }
            }
        }
        __syncthreads();
        unsigned long long* out = seg_sums + static_cast<size_t>(ch.x) * kMaxNodes * 3;
        for (int k = threadIdx.x; k < nn; k += blockDim.x) {
            if (aC[k] == 0u) continue;
            atomicAdd(out + 3 * k, (static_cast<unsigned long long>(aGh[k]) << 32) | aGl[k]);
            atomicAdd(out + 3 * k + 1, h != nullptr ? (static_cast<unsigned long long>(aHh[k]) << 32) | aHl[k]
                                                    : static_cast<unsigned long long>(aC[k]) * h1);
            atomicAdd(out + 3 * k + 2, static_cast<unsigned long long>(aC[k]));
            aGl[k] = aGh[k] = aHl[k] = aHh[k] = aC[k] = 0u;  // clear for the CTA's next chunk
        }
        __syncthreads();
    }
}

__device__ __forceinline__ double leaf_value(double G, double H, double l2) { return -G / (H + l2); }

__global__ void finalize_tree_kernel(PostParams pp, const DevTreeState* __restrict__ st,
                                     const unsigned long long* __restrict__ seg_sums,
                                     const int* __restrict__ bucket_seg_end, const int* __restrict__ cuts,
                                     const AllScale* __restrict__ sc, double* __restrict__ values,
                                     int* __restrict__ cover, double* __restrict__ prefix) {
    const int nn = st->n_nodes;
    const double ig = sc->inv_gscale, ih = sc->inv_hscale;
    for (int k = threadIdx.x; k < nn; k += blockDim.x) {
        long long G = 0, H = 0, Cn = 0;
        for (int s = 0; s < pp.n_segments; ++s) {
            const unsigned long long* e = seg_sums + (static_cast<size_t>(s) * kMaxNodes + k) * 3;
            G += static_cast<long long>(e[0]);
            H += static_cast<long long>(e[1]);
            Cn += static_cast<long long>(e[2]);
        }
        values[k] = leaf_value(static_cast<double>(G) * ig, static_cast<double>(H) * ih, pp.l2);
        cover[k] = static_cast<int>(Cn);
    }
    __syncthreads();
    const int nb = pp.n_buckets;
    for (int q = threadIdx.x; q < nb * nn; q += blockDim.x) {
        const int b = q / nn, k = q % nn;
        const double full = values[k];
        double v;
        if (pp.iid_mode) {
            v = full;
        } else {
            long long pG = 0, pH = 0;
            for (int s = 0; s < bucket_seg_end[b]; ++s) {
                const unsigned long long* e = seg_sums + (static_cast<size_t>(s) * kMaxNodes + k) * 3;
                pG += static_cast<long long>(e[0]);
                pH += static_cast<long long>(e[1]);
            }
            const double cov = static_cast<double>(cuts[b]);
            const double alpha = cov <= 0.0 ? 0.0 : fmin(1.0, cov / fmax(pp.min_cover, 1.0));
            const double pref = cov > 0.0 ? leaf_value(static_cast<double>(pG) * ig, static_cast<double>(pH) * ih, pp.l2)
                                          : full;
            v = alpha * pref + (1.0 - alpha) * full;
        }
        prefix[static_cast<size_t>(b) * nn + k] = v;
    }
}

__global__ void pred_update_kernel(PostParams pp, const int16_t* __restrict__ nid,
                                   const double* __restrict__ prefix, const DevTreeState* __restrict__ st,
                                   double* __restrict__ pred) {
    const int nn = st->n_nodes;
    const int n = pp.n;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int b = 0;
        if (!pp.iid_mode) {
            // time_buckets on time-sorted rows (cpp/src/booster.cpp:60-72): rank = row.
            b = static_cast<int>(static_cast<double>(i) / max(n, 1) * pp.n_buckets);
            if (b >= pp.n_buckets) b = pp.n_buckets - 1;
        }
        pred[i] += pp.learning_rate * prefix[static_cast<size_t>(b) * nn + nid[i]];
    }
}

// pred update fused with the MSE training loss on the updated predictions
// (booster.cpp:655-664 then 704-706): per-block partial sums of (pred - y)^2.
// g != nullptr: also the next tree's mse gradient g = 1 * (pred - y) (objective.cpp:105-118,
// the same double the gradient kernel computes) and its largest |g| into sc (reset by the
// caller), so that the next tree needs no separate pass over pred and y.
__global__ void pred_update_loss_kernel(PostParams pp, const int16_t* __restrict__ nid,
                                        const double* __restrict__ prefix, const DevTreeState* __restrict__ st,
                                        double* __restrict__ pred, const double* __restrict__ y,
                                        double* __restrict__ partials, double* __restrict__ g,
                                        AllScale* __restrict__ sc) {
    const int nn = st->n_nodes;
    const int n = pp.n;
    double acc = 0.0, mg = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int b = 0;
        if (!pp.iid_mode) {
            b = static_cast<int>(static_cast<double>(i) / max(n, 1) * pp.n_buckets);
            if (b >= pp.n_buckets) b = pp.n_buckets - 1;
        }
        const double p = pred[i] + pp.learning_rate * prefix[static_cast<size_t>(b) * nn + nid[i]];
        pred[i] = p;
        const double d = p - y[i];
        acc += 1.0 * d * d;
        if (g != nullptr) {
            const double gv = 1.0 * d;
            g[i] = gv;
            mg = fmax(mg, fabs(gv));
        }
    }
    if (g != nullptr) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) mg = fmax(mg, __shfl_xor_sync(0xffffffffu, mg, o));
        if ((threadIdx.x & 31) == 0)
            atomicMax(&sc->maxg_bits, static_cast<unsigned long long>(__double_as_longlong(mg)));
        if (blockIdx.x == 0 && threadIdx.x == 0)
            atomicMax(&sc->maxh_bits, static_cast<unsigned long long>(__double_as_longlong(1.0)));
    }
    __shared__ double ws[32];
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) t += ws[w];
        partials[blockIdx.x] = t;
    }
}

__global__ void fill_pred_kernel(const double* __restrict__ init_prefix, int n, int n_buckets, int iid_mode,
                                 double* __restrict__ pred) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        int b = 0;
        if (!iid_mode) {
            b = static_cast<int>(static_cast<double>(i) / max(n, 1) * n_buckets);
            if (b >= n_buckets) b = n_buckets - 1;
        }
        pred[i] = init_prefix[b];
    }
}

// Booster::predict_raw_binned (cpp/src/booster.cpp:744-773): base + sum over trees
// of lr * values[leaf], accumulated per row in tree order.
__global__ void predict_trees_kernel(const uint8_t* __restrict__ codes, int stride, int n,
                                     const int16_t* __restrict__ feat, const int16_t* __restrict__ left,
                                     const int16_t* __restrict__ right, const uint8_t* __restrict__ thr,
                                     const uint8_t* __restrict__ ml, const double* __restrict__ val,
                                     const int* __restrict__ off, int n_trees, double base, double lr,
                                     const uint8_t* __restrict__ type, const unsigned long long* __restrict__ cat,
                                     const int16_t* __restrict__ feat2, int n_bins, double* __restrict__ out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint8_t* row = codes + static_cast<size_t>(i) * stride;
        double s = base;
        for (int t = 0; t < n_trees; ++t) {
            const int o = off[t];
            int k = 0;
            while (feat[o + k] >= 0) {
                const int b = row[feat[o + k]];
                const int b2 = type[o + k] == 1 ? row[feat2[o + k]] : 0;
                const bool go_left = goes_left(type[o + k], cat + 4 * static_cast<size_t>(o + k), thr[o + k],
                                               ml[o + k], static_cast<unsigned>(b), static_cast<unsigned>(b2), n_bins);
                k = go_left ? left[o + k] : right[o + k];
            }
            s += lr * val[o + k];
        }
        out[i] = s;
    }
}

}  // namespace

void launch_fill_pred(const double* init_prefix, int n, int n_buckets, int iid_mode, double* pred,
                      cudaStream_t s) {
    fill_pred_kernel<<<std::max(1, std::min(2368, (n + 255) / 256)), 256, 0, s>>>(init_prefix, n, n_buckets,
                                                                                  iid_mode, pred);
    check(cudaGetLastError(), "fill_pred launch");
}

void launch_predict_trees(const uint8_t* codes, int stride, int n, const int16_t* tree_feat,
                          const int16_t* tree_left, const int16_t* tree_right, const uint8_t* tree_thr,
                          const uint8_t* tree_ml, const double* tree_val, const int* tree_off, int n_trees,
                          double base, double lr, const uint8_t* tree_type, const unsigned long long* tree_cat,
                          const int16_t* tree_feat2, int n_bins, double* out, cudaStream_t s) {
    if (n <= 0) return;
    predict_trees_kernel<<<std::max(1, std::min(4736, (n + 127) / 128)), 128, 0, s>>>(
        codes, stride, n, tree_feat, tree_left, tree_right, tree_thr, tree_ml, tree_val, tree_off, n_trees, base,
        lr, tree_type, tree_cat, tree_feat2, n_bins, out);
    check(cudaGetLastError(), "predict_trees launch");
}

void launch_pred_update_loss(const PostParams& pp, const int16_t* nid, const double* prefix, const DevTreeState* st,
                             double* pred, const double* y, double* partials, int n_part, double* g, AllScale* sc,
                             cudaStream_t s) {
    if (g != nullptr) check(cudaMemsetAsync(sc, 0, 2 * sizeof(unsigned long long), s), "all scale reset");
    pred_update_loss_kernel<<<n_part, 256, 0, s>>>(pp, nid, prefix, st, pred, y, partials, g, sc);
    check(cudaGetLastError(), "pred_update_loss launch");
}

void launch_all_scale_finalize(AllScale* sc, int n, cudaStream_t s) {
    all_scale_finalize_kernel<<<1, 1, 0, s>>>(sc, n);
    check(cudaGetLastError(), "all_scale_finalize launch");
}

void launch_all_scale(const double* g, const double* h, int n, AllScale* sc, cudaStream_t s) {
    check(cudaMemsetAsync(sc, 0, 2 * sizeof(unsigned long long), s), "all scale reset");
    max_abs_kernel<<<std::max(1, std::min(1184, (n + 255) / 256)), 256, 0, s>>>(g, h, n, sc);
    check(cudaGetLastError(), "max_abs launch");
    all_scale_finalize_kernel<<<1, 1, 0, s>>>(sc, n);
    check(cudaGetLastError(), "all_scale_finalize launch");
}

void launch_apply_accum(const uint8_t* col, long long pitch, int n_f, const DevNode* nodes, const DevTreeState* st,
                        const double* g, const double* h, const int4* chunks, int n_chunks,
                        const AllScale* sc, int16_t* nid, unsigned long long* seg_sums, int n_segments,
                        int n_bins, int kinds, cudaStream_t s) {
    check(cudaMemsetAsync(seg_sums, 0, sizeof(unsigned long long) * 3 * kMaxNodes * n_segments, s),
          "seg sums reset");
    auto kern = kinds == 0 ? apply_accum_kernel<0> : kinds == 1 ? apply_accum_kernel<1>
                                                   : kinds == 2 ? apply_accum_kernel<2> : apply_accum_kernel<3>;
    {  // static + dynamic shared memory above 48 KB needs the opt-in, once per device
        static std::atomic<bool> done[64][4] = {};
        int dev = 0;
        check(cudaGetDevice(&dev), "cudaGetDevice");
        if (dev < 0 || dev >= 64 || !done[dev][kinds & 3]) {
            check(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kApplySmem)),
                  "apply_accum smem attr");
            if (dev >= 0 && dev < 64) done[dev][kinds & 3] = true;
        }
    }
    // a persistent grid: 3 CTAs per SM (its register and shared-memory budget), chunks in turn
    int sms = 148;
    {
        int dev = 0;
        if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    }
    const int grid = std::max(1, std::min(n_chunks, 3 * sms));
    kern<<<grid, kApplyThreads, kApplySmem, s>>>(col, pitch, n_f, nodes, st, g, h, chunks, n_chunks, sc, nid,
                                                 seg_sums, n_bins);
    check(cudaGetLastError(), "apply_accum launch");
}

void launch_finalize_tree(const PostParams& pp, const DevTreeState* st, const unsigned long long* seg_sums,
                          const int* bucket_seg_end, const int* cuts, const AllScale* sc, double* values,
                          int* cover, double* prefix, cudaStream_t s) {
    finalize_tree_kernel<<<1, 1024, 0, s>>>(pp, st, seg_sums, bucket_seg_end, cuts, sc, values, cover, prefix);
    check(cudaGetLastError(), "finalize_tree launch");
}

void launch_pred_update(const PostParams& pp, const int16_t* nid, const double* prefix, const DevTreeState* st,
                        double* pred, cudaStream_t s) {
    pred_update_kernel<<<std::max(1, std::min(2368, (pp.n + 255) / 256)), 256, 0, s>>>(pp, nid, prefix, st, pred);
    check(cudaGetLastError(), "pred_update launch");
}

}  // namespace tgb
