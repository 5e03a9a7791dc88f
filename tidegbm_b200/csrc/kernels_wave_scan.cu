// Wave scan and select (wave.h describes the scheme).  Compiled with -fmad=false: the
// gain arithmetic follows the reference's statement order (scan_common.cuh).
//
// scan: one CTA of 256 threads (thread = bin) per (child, feature), grid-stride over the
// children of all planned leaves of all contexts (or over the roots).  The larger child's
// histogram is derived as parent - smaller child on the way (subtract_hist_inplace,
// cpp/src/histogram.cpp:108-117, exact in fixed point).  The last CTA of a child to
// finish (ticket counter, nothing waits) reduces the per-feature candidates, lowest
// feature on ties (best_for_leaf, cpp/src/tree.cpp:120-166).
//
// select: one warp per context.  It commits expanded best leaves in the reference's
// best-first order (grow_tree, cpp/src/tree.cpp:343-383) and plans the next wave's
// expansions; the last context to finish sets the launch-loop condition.
#include "scan_common.cuh"
#include "wave.h"

namespace tgb {

namespace {

using namespace scan;

constexpr int kRootCand = 2 * kMaxNodes;  // candidate / ticket index of the root
constexpr int kMaxPairFeatures = 1024;    // features the PAIR ranking sorts (host-checked)

__device__ __forceinline__ void children_prefix(const WaveCtx* ctxs, int n_ctx, int src, int* s_pref) {
    if (static_cast<int>(threadIdx.x) < n_ctx) {
        const WaveCtl* ctl = ctxs[threadIdx.x].ctl;
        s_pref[threadIdx.x] = src == 0 ? (ctl->active ? 1 : 0) : 2 * ctl->n_exp;
    }
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

// The histogram job of one child: its node and split outputs, its candidate index, its
// slot, and (the larger child) the parent and small-sibling slots it is derived from.
struct ScanTarget {
    DevNode* N;
    DevSplit* out;
    int ci, slot, pslot, sslot;
    bool derive;
};

__device__ __forceinline__ ScanTarget scan_target(const WaveCtx& X, int src, int k) {
    ScanTarget t;
    t.pslot = t.sslot = 0;
    t.derive = false;
    if (src == 0) {
        t.N = X.nodes;
        t.out = X.splits;
        t.ci = kRootCand;
        t.slot = 0;
        return t;
    }
    const int L = X.ctl->exp_leaf[k >> 1];
    const int side = k & 1;
    t.ci = 2 * L + side;
    t.N = X.spec + t.ci;
    t.out = X.spec_split + t.ci;
    t.slot = t.N->slot;
    const DevNode& A = X.spec[2 * L];
    const DevNode& B = X.spec[2 * L + 1];
    const int small = A.count <= B.count ? 0 : 1;  // cpp/src/tree.cpp:423
    t.derive = side != small;
    t.pslot = X.nodes[L].slot;
    t.sslot = X.spec[2 * L + small].slot;
    return t;
}

// The last feature job of a child (one warp): the best candidate over its features
// (best_for_leaf's ascending-feature strict '>', tree.cpp:160-166), written as its split.
__device__ __forceinline__ void finish_child(const WaveCtx& X, int ci, DevSplit* out, int lane) {
    const GrowParams& p = X.gp;
    __threadfence();
    Cand b{-1e300, 0x7fffffff};
    for (int k = lane; k < p.n_features; k += 32) {
        const size_t cs = static_cast<size_t>(ci) * p.n_features + k;
        const Cand cd{static_cast<volatile double*>(X.cand_gain)[cs], static_cast<volatile int*>(X.cand_key)[cs]};
        if (better(cd, b)) b = cd;
    }
    b = warp_best(b);
    if (lane == 0) {
        DevSplit sp{};
        sp.gain = b.gain;
        sp.valid = (b.key != 0x7fffffff) && b.gain >= p.min_split_gain;
        sp.feature = sp.valid ? b.key / 512 : -1;
        sp.threshold = sp.valid ? (b.key % 512) / 2 : -1;
        sp.missing_left = sp.valid ? (b.key & 1) : 1;
        sp.type = 0;
        if (sp.valid && X.is_cat != nullptr && X.is_cat[sp.feature]) {
            // categorical: the winning feature's left mask; missing follows bin 0's side
            const unsigned long long* m = X.cand_cat + (static_cast<size_t>(ci) * p.n_features + sp.feature) * 4;
            sp.type = 2;
            sp.threshold = -1;
            for (int k = 0; k < 4; ++k) sp.cat[k] = reinterpret_cast<const volatile unsigned long long*>(m)[k];
            sp.missing_left = static_cast<int>(sp.cat[0] & 1ull);
        }
        *out = sp;
        X.tickets[ci] = 0;  // ready for the next launch
    }
}

// Node totals from feature 0 (every feature's bins sum to the same integers) and the
// node's value (leaf_value, cpp/include/tidegbm/tree.hpp:53-67).
__device__ __forceinline__ void set_totals(DevNode* N, long long Gt, long long Ht, long long Ct, double inv_gs,
                                           double inv_hs, double l2) {
    N->G = Gt;
    N->H = Ht;
    N->C = Ct;
    const double dg = static_cast<double>(Gt) * inv_gs, dh = static_cast<double>(Ht) * inv_hs;
    N->value = -dg / (dh + l2);
}

// Numeric features, one warp per (child, feature): every child's histogram scanned by
// scan_feature_warp (the larger child first derived as parent - smaller), the per-feature
// bests kept as candidates, and the child's last job picks its split.  Categorical
// features are left to wave_scan_cat_kernel; the children's tickets count both.
constexpr int kScanWarpThreads = 256;

__global__ void __launch_bounds__(kScanWarpThreads, 2)
    wave_scan_warp_kernel(const WaveCtx* __restrict__ ctxs, int n_ctx, int src) {
    pdl_wait();
    pdl_trigger();
    __shared__ int s_pref[kMaxWaveCtx + 1];
    __shared__ int s_jpref[kMaxWaveCtx + 1];
    children_prefix(ctxs, n_ctx, src, s_pref);
    if (threadIdx.x == 0) {
        int acc = 0;
        for (int c = 0; c < n_ctx; ++c) {
            s_jpref[c] = acc;
            acc += (s_pref[c + 1] - s_pref[c]) * ctxs[c].gp.n_features;
        }
        s_jpref[n_ctx] = acc;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int wpb = kScanWarpThreads / 32;
    const int total = s_jpref[n_ctx];
    for (int jw = blockIdx.x * wpb + (threadIdx.x >> 5); jw < total; jw += gridDim.x * wpb) {
        int c = 0;
        while (c + 1 < n_ctx && s_jpref[c + 1] <= jw) ++c;
        const WaveCtx& X = ctxs[c];
        const GrowParams& p = X.gp;
        const int rem = jw - s_jpref[c];
        const int k = rem / p.n_features, f = rem - k * p.n_features;
        if (X.is_cat != nullptr && X.is_cat[f]) continue;
        const ScanTarget t = scan_target(X, src, k);
        const size_t e = static_cast<size_t>(p.n_features) * kBins;
        const bool eligible = t.N->depth < p.max_depth && t.N->count >= 2 * p.min_samples_leaf;
        const double inv_gs = X.st->inv_gscale, inv_hs = X.st->inv_hscale;
        Cand best{-1e300, 0x7fffffff};
        if (eligible || f == 0) {
            const size_t fo = static_cast<size_t>(f) * kBins;
            const size_t so = static_cast<size_t>(t.slot) * e + fo, po = static_cast<size_t>(t.pslot) * e + fo,
                         qo = static_cast<size_t>(t.sslot) * e + fo;
            long long Gt, Ht, Ct;
            best = scan_feature_warp(X.G + so, X.H + so, X.C + so, X.G + po, X.H + po, X.C + po, X.G + qo, X.H + qo,
                                     X.C + qo, t.derive, eligible, f, p.n_bins, inv_gs, inv_hs, p.l2, p.min_split_gain,
                                     p.min_samples_leaf, p.min_child_weight, Gt, Ht, Ct);
            if (f == 0 && lane == 0) set_totals(t.N, Gt, Ht, Ct, inv_gs, inv_hs, p.l2);
        }
        int last = 0;
        if (lane == 0) {
            const size_t cs = static_cast<size_t>(t.ci) * p.n_features + f;
            X.cand_gain[cs] = best.gain;
            X.cand_key[cs] = best.key;
            __threadfence();
            last = atomicAdd(&X.tickets[t.ci], 1) == p.n_features - 1;
        }
        last = __shfl_sync(0xffffffffu, last, 0);
        if (last) finish_child(X, t.ci, t.out, lane);
    }
}

// Categorical features, one CTA per (child, feature): the histogram (derived as above)
// ranked and scanned by scan_categorical (best_categorical, histogram.cpp:195-244).
__global__ void __launch_bounds__(kScanThreads)
    wave_scan_cat_kernel(const WaveCtx* __restrict__ ctxs, int n_ctx, int src) {
    pdl_wait();
    pdl_trigger();
    __shared__ int s_pref[kMaxWaveCtx + 1];
    __shared__ ScanShared sm;
    __shared__ CatShared csm;
    __shared__ int last;
    children_prefix(ctxs, n_ctx, src, s_pref);
    const int total = s_pref[n_ctx];
    const int f = blockIdx.x;
    for (int j = blockIdx.y; j < total; j += gridDim.y) {
        int c = 0;
        while (c + 1 < n_ctx && s_pref[c + 1] <= j) ++c;
        const WaveCtx& X = ctxs[c];
        const GrowParams& p = X.gp;
        if (f >= p.n_features || X.is_cat == nullptr || !X.is_cat[f]) continue;  // uniform over the CTA
        const ScanTarget t = scan_target(X, src, j - s_pref[c]);
        const size_t e = static_cast<size_t>(p.n_features) * kBins;
        const bool eligible = t.N->depth < p.max_depth && t.N->count >= 2 * p.min_samples_leaf;
        const double inv_gs = X.st->inv_gscale, inv_hs = X.st->inv_hscale;
        Cand best{-1e300, 0x7fffffff};
        if (eligible || f == 0) {
            const size_t fo = static_cast<size_t>(f) * kBins;
            const size_t so = static_cast<size_t>(t.slot) * e + fo, po = static_cast<size_t>(t.pslot) * e + fo,
                         qo = static_cast<size_t>(t.sslot) * e + fo;
            long long Gt, Ht, Ct;
            best = scan_feature(X.G + so, X.H + so, X.C + so, X.G + po, X.H + po, X.C + po, X.G + qo, X.H + qo,
                                X.C + qo, t.derive, false, f, p.n_bins, inv_gs, inv_hs, p.l2, p.min_split_gain,
                                p.min_samples_leaf, p.min_child_weight, sm, Gt, Ht, Ct);
            if (eligible) {
                // best_categorical over the stored (possibly just derived) histogram
                __syncthreads();
                best = scan_categorical(X.G + so, X.H + so, X.C + so, f, inv_gs, inv_hs, p.l2, p.min_split_gain,
                                        p.min_samples_leaf, p.min_child_weight, X.cat_smooth, Gt, Ht, Ct, csm,
                                        X.cand_cat + (static_cast<size_t>(t.ci) * p.n_features + f) * 4);
            }
            if (f == 0 && threadIdx.x == 0) set_totals(t.N, Gt, Ht, Ct, inv_gs, inv_hs, p.l2);
        }
        if (threadIdx.x == 0) {
            const size_t cs = static_cast<size_t>(t.ci) * p.n_features + f;
            X.cand_gain[cs] = best.gain;
            X.cand_key[cs] = best.key;
            __threadfence();
            last = atomicAdd(&X.tickets[t.ci], 1) == p.n_features - 1;
        }
        __syncthreads();
        if (last && threadIdx.x < 32) finish_child(X, t.ci, t.out, static_cast<int>(threadIdx.x));
        __syncthreads();  // shared state reuse
    }
}

// A leaf the reference's selection may pick: depth and size limits, a valid split of gain
// above min_split_gain (tree.cpp:343-383; the strict '>' against min_split_gain).
__device__ __forceinline__ bool candidate(const GrowParams& p, const DevNode& N, const DevSplit& S) {
    return N.is_leaf && N.depth < p.max_depth && N.count >= 2 * p.min_samples_leaf && S.valid &&
           S.gain > p.min_split_gain;
}

// better leaf: larger gain, lower id on ties
__device__ __forceinline__ bool better_leaf(double ga, int ia, double gb, int ib) {
    return ga > gb || (ga == gb && ia < ib);
}

constexpr int kSelectThreads = 256;  // all stage the selection state; warp 0 then selects

__global__ void __launch_bounds__(kSelectThreads)
    wave_select_kernel(const WaveCtx* __restrict__ ctxs, int n_ctx, int* gsync, unsigned* host_flag,
                       cudaGraphConditionalHandle cond, int use_cond) {
    pdl_wait();
    pdl_trigger();
    const WaveCtx& X = ctxs[blockIdx.x];
    const GrowParams& p = X.gp;
    WaveCtl* ctl = X.ctl;
    DevTreeState* st = X.st;
    DevNode* nodes = X.nodes;
    DevSplit* splits = X.splits;
    const int lane = threadIdx.x & 31;
    __shared__ double s_gain[kMaxLeavesCap + 1];
    __shared__ int s_id[kMaxLeavesCap + 1];
    // Selection state staged once, so that the commit loop reads no global memory: per
    // node its current split's gain, candidacy, type and with-pairs type, and whether it
    // is expanded; per expanded node the same for its two planned children.  Restaged
    // from the node table when the pair budget runs out (the splits change).
    __shared__ double s_ng[kMaxNodes];
    __shared__ unsigned char s_nc[kMaxNodes], s_ex[kMaxNodes], s_ty[kMaxNodes], s_pty[kMaxNodes];
    __shared__ double s_cg[2 * kMaxNodes];
    __shared__ unsigned char s_cc[2 * kMaxNodes], s_cty[2 * kMaxNodes], s_cpty[2 * kMaxNodes];
    __shared__ int s_commit[kMaxLeavesCap];
    int active = 0;
    if (ctl->active) {
        const int budget = p.max_leaves - 1;
        // every select commits at least one split or ends the tree, so a tree takes at most
        // max_leaves of them; past that bound the tree is ended with the error flag set
        const bool runaway = ctl->waves > p.max_leaves + 1;
        int nn = st->n_nodes;
        int done_splits = ctl->splits_done;
        int pair_used = ctl->pair_used;
        // the split a leaf takes: with the PAIR candidates while the tree's pair budget lasts
        // (tree.cpp:214-218, re-scored after every pair split, tree.cpp:393-396)
        auto pairs_on = [&]() { return X.pair_on && pair_used < X.max_pair; };
        auto stage_all = [&](int t, int step) {
            const bool pr = pairs_on();
            for (int k = t; k < nn; k += step) {
                const DevSplit S = pr ? X.splits_pair[k] : splits[k];
                s_nc[k] = candidate(p, nodes[k], S) ? 1 : 0;
                s_ng[k] = S.gain;
                s_ty[k] = static_cast<unsigned char>(S.type);
                s_pty[k] = X.pair_on ? static_cast<unsigned char>(X.splits_pair[k].type) : 0;
                const int ex = ctl->expanded[k];
                s_ex[k] = static_cast<unsigned char>(ex);
                if (ex) {
                    for (int sd = 0; sd < 2; ++sd) {
                        const int ci = 2 * k + sd;
                        const DevSplit C = pr ? X.spec_split_pair[ci] : X.spec_split[ci];
                        s_cc[ci] = candidate(p, X.spec[ci], C) ? 1 : 0;
                        s_cg[ci] = C.gain;
                        s_cty[ci] = static_cast<unsigned char>(C.type);
                        s_cpty[ci] = X.pair_on ? static_cast<unsigned char>(X.spec_split_pair[ci].type) : 0;
                    }
                }
            }
        };
        // the node-table writes of the pending commits (children ids nn_first + 2i, + 1 for
        // the i-th), issued in parallel; `pr`: the pair state they were committed under
        int n_commit = 0, nn_first = nn;
        auto flush = [&](bool pr) {
            for (int i = lane; i < n_commit; i += 32) {
                const int bi = s_commit[i], nc = nn_first + 2 * i;
                const DevSplit S = pr ? X.splits_pair[bi] : splits[bi];
                DevNode& P = nodes[bi];
                P.is_leaf = 0;
                P.feature = S.feature;
                P.threshold = S.threshold;
                P.missing_left = S.missing_left;
                P.gain = S.gain;
                P.type = S.type;
                P.feature2 = S.type == 1 ? S.feature2 : -1;
                for (int k = 0; k < 4; ++k) P.cat[k] = S.cat[k];
                P.left = nc;
                P.right = nc + 1;
                nodes[nc] = X.spec[2 * bi];
                nodes[nc + 1] = X.spec[2 * bi + 1];
                splits[nc] = X.spec_split[2 * bi];
                splits[nc + 1] = X.spec_split[2 * bi + 1];
                if (X.pair_on) {
                    X.splits_pair[nc] = X.spec_split_pair[2 * bi];
                    X.splits_pair[nc + 1] = X.spec_split_pair[2 * bi + 1];
                }
                ctl->expanded[nc] = 0;
                ctl->expanded[nc + 1] = 0;
            }
            __syncwarp();
            __threadfence_block();
            n_commit = 0;
            nn_first = nn;
        };
        stage_all(static_cast<int>(threadIdx.x), static_cast<int>(blockDim.x));
        __syncthreads();
        if (threadIdx.x >= 32) return;  // warp 0 selects
        if (lane == 0) ctl->waves += 1;
        bool finished = false;
        while (true) {
            if (done_splits >= budget || runaway) {
                finished = true;
                break;
            }
            double bg = 0.0;
            int bi = 0x7fffffff;
            for (int k = lane; k < nn; k += 32) {
                if (!s_nc[k]) continue;
                if (bi == 0x7fffffff || better_leaf(s_ng[k], k, bg, bi)) {
                    bg = s_ng[k];
                    bi = k;
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const double og = __shfl_xor_sync(0xffffffffu, bg, o);
                const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
                if (oi != 0x7fffffff && (bi == 0x7fffffff || better_leaf(og, oi, bg, bi))) {
                    bg = og;
                    bi = oi;
                }
            }
            if (bi == 0x7fffffff) {
                finished = true;
                break;
            }
            const int ex = s_ex[bi];
            if (!ex) break;
            // an expansion planned with bi's PAIR split while the budget lasted is void once the
            // budget is spent (bi now takes its axis split): plan bi again
            if (ex == 2 && !pairs_on() && s_pty[bi] == 1) {
                if (lane == 0) {
                    ctl->expanded[bi] = 0;
                    s_ex[bi] = 0;
                }
                __syncwarp();
                __threadfence_block();
                break;
            }
            // commit: the split of bi, children ids nn, nn + 1 (grow_tree's numbering)
            const bool pr_before = pairs_on();
            const int ty = s_ty[bi];
            if (lane == 0) {
                s_commit[n_commit] = bi;
                s_nc[bi] = 0;
            }
            if (lane < 2) {
                const int k = nn + lane, ci = 2 * bi + lane;
                s_nc[k] = s_cc[ci];
                s_ng[k] = s_cg[ci];
                s_ex[k] = 0;
                s_ty[k] = s_cty[ci];
                s_pty[k] = s_cpty[ci];
            }
            __syncwarp();
            n_commit += 1;
            nn += 2;
            done_splits += 1;
            if (ty == 1) pair_used += 1;
            if (pr_before != pairs_on()) {
                // the budget ran out: write the commits so far, then axis splits from here
                flush(pr_before);
                stage_all(lane, 32);
                __syncwarp();
            }
        }
        flush(pairs_on());
        int n_exp = 0;
        if (!finished) {
            // candidates of the new state, best first
            int nc = 0;
            for (int k0 = 0; k0 < nn; k0 += 32) {
                const int k = k0 + lane;
                bool is_c = false;
                double gk = 0.0;
                if (k < nn) {
                    is_c = s_nc[k] != 0;
                    gk = s_ng[k];
                }
                const unsigned m = __ballot_sync(0xffffffffu, is_c);
                if (is_c) {
                    const int pos = nc + __popc(m & ((1u << lane) - 1u));
                    if (pos < kMaxLeavesCap) {
                        s_gain[pos] = gk;
                        s_id[pos] = k;
                    }
                }
                nc += __popc(m);
            }
            nc = min(nc, kMaxLeavesCap);
            __syncwarp();
            const int B = budget - done_splits;
            // expansions: unexpanded candidates ranked below B; in candidate (node id) order
            int base_tiles = 0;
            const int slot_first = 1 + 2 * ctl->exp_counter;
            for (int i0 = 0; i0 < nc; i0 += 32) {
                const int i = i0 + lane;
                bool take = false;
                if (i < nc) {
                    int rank = 0;
                    for (int q = 0; q < nc; ++q)
                        if (q != i && better_leaf(s_gain[q], s_id[q], s_gain[i], s_id[i])) ++rank;
                    take = rank < B && (X.max_expand <= 0 || rank < X.max_expand) && !ctl->expanded[s_id[i]];
                }
                const unsigned m = __ballot_sync(0xffffffffu, take);
                int tiles = 0;
                int e = n_exp + __popc(m & ((1u << lane) - 1u));
                if (take) {
                    const int L = s_id[i];
                    const DevNode& N = nodes[L];
                    tiles = (N.count + kPartTile - 1) / kPartTile;
                    ctl->exp_leaf[e] = L;
                    // 2: the children are partitioned by L's with-pairs split, 1: by its axis split
                    ctl->expanded[L] = (X.pair_on && pair_used < X.max_pair) ? 2 : 1;
                    for (int sd = 0; sd < 2; ++sd) {
                        DevNode ch{};
                        ch.start = N.start;
                        ch.count = 0;
                        ch.buf = 1 - N.buf;
                        ch.depth = N.depth + 1;
                        ch.is_leaf = 1;
                        ch.feature = -1;
                        ch.threshold = -1;
                        ch.missing_left = 1;
                        ch.left = ch.right = -1;
                        ch.parent = L;
                        ch.slot = slot_first + 2 * e + sd;
                        ch.feature2 = -1;
                        X.spec[2 * L + sd] = ch;
                        if (X.pair_on) X.energy[2 * L + sd] = 0ull;
                    }
                }
                // tile prefix in expansion order
                int incl = tiles;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int t = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= o) incl += t;
                }
                if (take) ctl->exp_tile0[e] = base_tiles + incl - tiles;
                base_tiles += __shfl_sync(0xffffffffu, incl, 31);
                n_exp += __popc(m);
            }
            if (lane == 0) {
                ctl->exp_tile0[n_exp] = base_tiles;
                ctl->tiles_total = base_tiles;
                ctl->slot0 = slot_first;
                ctl->exp_counter += n_exp;
                ctl->exp_total += n_exp;
                if (slot_first + 2 * n_exp > X.n_slots || base_tiles > X.max_tiles) ctl->error = 1;
            }
            active = n_exp > 0 && slot_first + 2 * n_exp <= X.n_slots && base_tiles <= X.max_tiles;
        }
        if (lane == 0) {
            if (runaway) ctl->error = 1;
            st->n_nodes = nn;
            ctl->splits_done = done_splits;
            ctl->pair_used = pair_used;
            ctl->n_exp = active ? n_exp : 0;
            if (!active) {
                ctl->tiles_total = 0;
                ctl->active = 0;
                st->done = 1;
            }
        }
    }
    // launch-loop condition: any context still growing (the last context to finish sets it)
    if (threadIdx.x == 0) {
        if (active) atomicOr(&gsync[0], 1);
        __threadfence();
        const int t = atomicAdd(&gsync[1], 1);
        if (t == n_ctx - 1) {
            __threadfence();
            const unsigned v = static_cast<unsigned>(atomicExch(&gsync[0], 0));
            gsync[1] = 0;
            gsync[2] += 1;  // selects run (for the count of launched kernels)
            if (host_flag != nullptr) {
                *reinterpret_cast<volatile unsigned*>(host_flag) = v;
                __threadfence_system();
            }
            if (use_cond) cudaGraphSetConditional(cond, v);
        }
    }
}


// ---- PAIR stage (tree.cpp:214-281) --------------------------------------------------------
//
// energy: the rows' sum of g^2 (g as the tree sees it: GOSS-scaled for sampled others), one
// fixed-point sum per candidate index (exact integer adds: the same total in any order).
// pair: one CTA per (child, pair of its top features) when the child's best axis gain is
// weak against that energy: the histogram of pair_bin(code1, code2) over the child's rows
// (exact fixed-point sums of the same per-row values the main histogram adds), scanned as
// one numeric feature with pair_l2; the child's last pair CTA to finish merges the pairs'
// best splits with the axis split (strict '>' in pair order) into the with-pairs split.

struct ChildRef {
    int ci;
    const DevNode* N;
    const int32_t* rows;
    DevSplit* axis;
    DevSplit* with_pairs;
};

__device__ __forceinline__ ChildRef child_ref(const WaveCtx& X, int src, int k) {
    ChildRef r;
    if (src == 0) {
        r.ci = kRootCand;
        r.N = X.nodes;
        r.axis = X.splits;
        r.with_pairs = X.splits_pair;
    } else {
        const int L = X.ctl->exp_leaf[k >> 1];
        r.ci = 2 * L + (k & 1);
        r.N = X.spec + r.ci;
        r.axis = X.spec_split + r.ci;
        r.with_pairs = X.spec_split_pair + r.ci;
    }
    r.rows = (r.N->buf ? X.rows1 : X.rows0) + r.N->start;
    return r;
}

__device__ __forceinline__ int energy_shift(const DevTreeState* st) {
    const double mg = __longlong_as_double(static_cast<long long>(st->max_abs_g_bits));
    const double e2 = mg * mg;
    if (!(e2 > 0.0) || st->n_sample <= 0) return 0;
    int clog = 0;
    while ((1ll << clog) < static_cast<long long>(st->n_sample)) ++clog;
    return max(-1000, min(1000, 61 - (ilogb(e2) + 1) - clog));
}

constexpr int kEnergyRows = 8192;

__global__ void __launch_bounds__(256) wave_energy_kernel(const WaveCtx* __restrict__ ctxs, int n_ctx, int src) {
    pdl_wait();
    pdl_trigger();
    __shared__ int s_pref[kMaxWaveCtx + 1];
    __shared__ unsigned long long s_red[8];
    children_prefix(ctxs, n_ctx, src, s_pref);
    const int total = s_pref[n_ctx];
    for (int j = blockIdx.y; j < total; j += gridDim.y) {
        int c = 0;
        while (c + 1 < n_ctx && s_pref[c + 1] <= j) ++c;
        const WaveCtx& X = ctxs[c];
        if (!X.pair_on) continue;
        const ChildRef cr = child_ref(X, src, j - s_pref[c]);
        const GrowParams& p = X.gp;
        if (cr.N->depth >= p.max_depth || cr.N->count < 2 * p.min_samples_leaf) continue;
        const double scale = ldexp(1.0, energy_shift(X.st));
        const int count = cr.N->count;
        for (int r0 = blockIdx.x * kEnergyRows; r0 < count; r0 += gridDim.x * kEnergyRows) {
            unsigned long long acc = 0;
            const int r1 = min(count, r0 + kEnergyRows);
            for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
                const int r = cr.rows[i];
                double gv = X.g[r];
                if (X.goss_flag != nullptr && X.goss_flag[r] == 2) gv *= X.goss_scale;
                acc += static_cast<unsigned long long>(__double2ll_rn(gv * gv * scale));
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
            if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = acc;
            __syncthreads();
            if (threadIdx.x == 0) {
                unsigned long long t = 0;
                for (int w = 0; w < 8; ++w) t += s_red[w];
                atomicAdd(&X.energy[cr.ci], t);
            }
            __syncthreads();
        }
    }
}

__global__ void __launch_bounds__(kScanThreads) wave_pair_kernel(const WaveCtx* __restrict__ ctxs, int n_ctx, int src) {
    pdl_wait();
    pdl_trigger();
    __shared__ int s_pref[kMaxWaveCtx + 1];
    __shared__ ScanShared sm;
    __shared__ unsigned long long sG[kBins], sH[kBins];
    __shared__ int sC[kBins];
    __shared__ short s_top[kMaxPairFeatures];
    __shared__ int last;
    children_prefix(ctxs, n_ctx, src, s_pref);
    const int total = s_pref[n_ctx];
    const int pi = blockIdx.x;
    for (int j = blockIdx.y; j < total; j += gridDim.y) {
        int c = 0;
        while (c + 1 < n_ctx && s_pref[c + 1] <= j) ++c;
        const WaveCtx& X = ctxs[c];
        if (!X.pair_on) continue;
        const ChildRef cr = child_ref(X, src, j - s_pref[c]);
        const GrowParams& p = X.gp;
        const int n_f = p.n_features;
        const bool eligible = cr.N->depth < p.max_depth && cr.N->count >= 2 * p.min_samples_leaf;
        const DevSplit axis = *cr.axis;
        const double axis_gain = axis.valid ? axis.gain : -1e300;
        const double energy = static_cast<double>(X.energy[cr.ci]) * ldexp(1.0, -energy_shift(X.st));
        const bool weak = eligible && n_f >= 2 &&
                          ((axis_gain < X.pair_trigger * fmax(energy * 0.01, 1e-12)) || axis_gain <= 0);
        const int k = min(X.pair_top_k, n_f);
        const int n_pairs = weak ? k * (k - 1) / 2 : 0;
        if (n_pairs == 0) {
            if (pi == 0 && threadIdx.x == 0) *cr.with_pairs = axis;  // no pair search for this child
            continue;
        }
        if (pi >= n_pairs) continue;
        // top-k features by their best gain, std::sort's order (tree.cpp:223-225)
        if (threadIdx.x == 0) {
            for (int f = 0; f < n_f; ++f) s_top[f] = static_cast<short>(f);
            const double* gains = X.cand_gain + static_cast<size_t>(cr.ci) * n_f;
            libstdcxx_sort(s_top, n_f, [&](short a, short b) { return gains[a] > gains[b]; });
        }
        for (int q = threadIdx.x; q < kBins; q += blockDim.x) {
            sG[q] = sH[q] = 0ull;
            sC[q] = 0;
        }
        __syncthreads();
        int a = 0, rem = pi;
        while (rem >= k - 1 - a) {
            rem -= k - 1 - a;
            ++a;
        }
        const int f1 = s_top[a], f2 = s_top[a + 1 + rem];
        const uint8_t* c1 = X.codes_col + static_cast<size_t>(f1) * X.col_pitch;
        const uint8_t* c2 = X.codes_col + static_cast<size_t>(f2) * X.col_pitch;
        const bool var = X.hq != nullptr;
        // payloads by position (exact modes: 8-byte words), like the child's rows
        const long long pos0 = static_cast<long long>(cr.N->buf) * X.pay_pitch + cr.N->start;
        const long long* gpay = static_cast<const long long*>(X.gq) + pos0;
        const long long* hpay = var ? static_cast<const long long*>(X.hq) + pos0 : nullptr;
        const unsigned long long hq1 = static_cast<unsigned long long>(__double2ll_rn(1.0 * X.st->hscale));
        const unsigned long long hq2 = static_cast<unsigned long long>(__double2ll_rn(1.0 * X.goss_scale * X.st->hscale));
        const int count = cr.N->count;
        for (int i = threadIdx.x; i < count; i += blockDim.x) {
            const int r = cr.rows[i];
            const unsigned z = pair_bin(c1[r], c2[r], p.n_bins);
            unsigned long long gv, hv;
            if (var) {
                gv = static_cast<unsigned long long>(gpay[i]);
                hv = static_cast<unsigned long long>(hpay[i]);
            } else {
                const long long pk = gpay[i];
                gv = static_cast<unsigned long long>(pk >> 1);
                hv = (pk & 1) ? hq2 : hq1;
            }
            atomicAdd(&sG[z], gv);
            atomicAdd(&sH[z], hv);
            atomicAdd(&sC[z], 1);
        }
        __syncthreads();
        long long Gt, Ht, Ct;
        const Cand cd = scan_feature(reinterpret_cast<long long*>(sG), reinterpret_cast<long long*>(sH), sC, nullptr,
                                     nullptr, nullptr, nullptr, nullptr, nullptr, false, true, 0, p.n_bins,
                                     X.st->inv_gscale, X.st->inv_hscale, X.pair_l2, p.min_split_gain,
                                     p.min_samples_leaf, p.min_child_weight, sm, Gt, Ht, Ct);
        if (threadIdx.x == 0) {
            DevSplit ps{};
            ps.gain = cd.gain;
            ps.valid = cd.key != 0x7fffffff;  // found; min_split_gain is applied at the merge
            ps.feature = f1;
            ps.feature2 = f2;
            ps.type = 1;
            ps.threshold = ps.valid ? (cd.key % 512) / 2 : -1;
            ps.missing_left = ps.valid ? (cd.key & 1) : 1;
            X.pair_cand[static_cast<size_t>(cr.ci) * kMaxPairs + pi] = ps;
            __threadfence();
            last = atomicAdd(&X.pair_tickets[cr.ci], 1) == n_pairs - 1;
        }
        __syncthreads();
        if (last && threadIdx.x == 0) {
            __threadfence();
            DevSplit best = axis;
            double bg = axis_gain;
            for (int q = 0; q < n_pairs; ++q) {
                DevSplit pc;
                const volatile int* src_w =
                    reinterpret_cast<const volatile int*>(X.pair_cand + static_cast<size_t>(cr.ci) * kMaxPairs + q);
                int* dst_w = reinterpret_cast<int*>(&pc);
                for (int w = 0; w < static_cast<int>(sizeof(DevSplit) / 4); ++w) dst_w[w] = src_w[w];
                if (pc.valid && pc.gain > bg) {
                    bg = pc.gain;
                    best = pc;
                    best.valid = pc.gain >= p.min_split_gain;
                }
            }
            *cr.with_pairs = best;
            X.pair_tickets[cr.ci] = 0;
        }
        __syncthreads();
    }
}

}  // namespace

void launch_wave_pair(const WaveCtx* ctxs, int n_ctx, int src, cudaStream_t s) {
    launch_pdl(wave_energy_kernel, dim3(16, 32), dim3(256), 0, s, "wave_energy launch", ctxs, n_ctx, src);
    launch_pdl(wave_pair_kernel, dim3(kMaxPairs, 32), dim3(kScanThreads), 0, s, "wave_pair launch", ctxs, n_ctx, src);
}

void launch_wave_scan(const WaveCtx* ctxs, int n_ctx, int src, int max_f, int ys, bool any_cat, cudaStream_t s) {
    launch_pdl(wave_scan_warp_kernel, dim3(148 * 2), dim3(kScanWarpThreads), 0, s, "wave_scan launch", ctxs, n_ctx,
               src);
    if (any_cat)
        launch_pdl(wave_scan_cat_kernel, dim3(max_f, ys), dim3(kScanThreads), 0, s, "wave_scan_cat launch", ctxs, n_ctx,
                   src);
}

void launch_wave_select(const WaveCtx* ctxs, int n_ctx, int* gsync, unsigned* host_flag, unsigned long long cond,
                        int use_cond, cudaStream_t s) {
    launch_pdl(wave_select_kernel, dim3(n_ctx), dim3(kSelectThreads), 0, s, "wave_select launch", ctxs, n_ctx, gsync,
               host_flag,
               static_cast<cudaGraphConditionalHandle>(cond), use_cond);
}

}  // namespace tgb
