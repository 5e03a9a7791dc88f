// Best-split scan and best-first leaf selection.
//
// split_scan restates best_numeric_missing (cpp/src/histogram.cpp:126-193, l1 = 0,
// no monotone) for every feature of a node and best_for_leaf's axis reduction
// (cpp/src/tree.cpp:120-166): gain = 0.5 (GL^2/(HL+l2) + GR^2/(HR+l2) - G^2/(H+l2)) - gamma,
// thresholds b = 1 .. n_bins-2 with a non-empty bin b, missing (bin 0) sent left or
// right, min_samples_leaf on counts and min_child_weight on hessians, and ties broken
// exactly as the reference's strict '>' does: lowest (feature, threshold,
// missing_left) wins.  Prefix sums run in exact 64-bit integers; only the gain is FP64.
// This file is compiled with -fmad=false so the gain arithmetic follows the
// reference's statement order.
//
// Launch shape: one CTA of 256 threads per (node, feature), thread = bin, so every
// thread evaluates at most two candidates (missing left / right) and the launch is a
// few dependent steps deep: the scan is latency-bound, not throughput-bound.
//
// select restates the leaf choice of grow_tree (cpp/src/tree.cpp:343-383): among
// leaves with depth < max_depth and at least 2*min_samples_leaf rows, the largest
// cached gain above min_split_gain, lowest node id on ties.  It runs at the end of the
// scan launch, in the CTA that finishes last (a ticket counter; nothing waits).
#include "scan_common.cuh"

namespace tgb {

namespace {

using namespace scan;

__device__ void select_body(const GrowParams& p, DevNode* __restrict__ nodes, DevSplit* __restrict__ splits,
                            DevTreeState* __restrict__ st);

// grid = (F, nodes): one CTA per (node, feature).  Each CTA stores its best candidate;
// the last CTA of a node to finish (ticket counter, no waiting) reduces them, lowest
// feature on ties.  mode 1 (the two children of st->parent): the large child's
// histogram is derived from the parent's and the small child's on the way (no separate
// subtraction pass).  The last node of the launch to finish then picks the next leaf.
__global__ void __launch_bounds__(kScanThreads)
    split_scan_kernel(GrowParams p, HistSlotPtrs hs, DevNode* __restrict__ nodes,
                      DevSplit* __restrict__ splits, DevTreeState* __restrict__ st, int mode,
                      int node, ScanScratch sc, int do_select) {
    pdl_wait();
    pdl_trigger();
    if (st->done || (mode == 1 && st->parent < 0)) return;
    int nd = node;
    bool derive = false;
    if (mode == 1) {
        const DevNode& par = nodes[st->parent];
        nd = blockIdx.y == 0 ? par.left : par.right;
        derive = nd == st->large_node;
    }
    const size_t e = hs.slot_elems;
    const size_t po = derive ? static_cast<size_t>(st->parent) * e : 0;
    const size_t so = derive ? static_cast<size_t>(st->small_node) * e : 0;
    const double inv_gs = st->inv_gscale, inv_hs = st->inv_hscale;
    DevNode& N = nodes[nd];
    const bool eligible = N.depth < p.max_depth && N.count >= 2 * p.min_samples_leaf;
    const int f = blockIdx.x;
    __shared__ ScanShared sm;
    __shared__ int last;
    Cand best{-1e300, 0x7fffffff};
    // A node that cannot split only needs its totals (feature 0); its other CTAs carry no
    // candidate but still take part in the ticket protocol below.
    if (eligible || f == 0) {
        const size_t fo = static_cast<size_t>(f) * kBins;
        long long Gt, Ht, Ct;
        best = scan_feature(hs.G + nd * e + fo, hs.H + nd * e + fo, hs.C + nd * e + fo, hs.G + po + fo,
                            hs.H + po + fo, hs.C + po + fo, hs.G + so + fo, hs.H + so + fo, hs.C + so + fo, derive,
                            eligible, f, p.n_bins, inv_gs, inv_hs, p.l2, p.min_split_gain, p.min_samples_leaf,
                            p.min_child_weight, sm, Gt, Ht, Ct);
        if (f == 0 && threadIdx.x == 0) {
            // Node totals from feature 0 (every feature's bins sum to the same exact integers).
            N.G = Gt;
            N.H = Ht;
            N.C = Ct;
            const double dg = static_cast<double>(Gt) * inv_gs, dh = static_cast<double>(Ht) * inv_hs;
            N.value = -dg / (dh + p.l2);  // leaf_value, cpp/include/tidegbm/tree.hpp:53-67
        }
    }
    if (threadIdx.x == 0) {
        const int slot = blockIdx.y * gridDim.x + blockIdx.x;
        sc.gain[slot] = best.gain;
        sc.key[slot] = best.key;
        __threadfence();
        last = atomicAdd(&sc.ticket[blockIdx.y], 1) == static_cast<int>(gridDim.x) - 1;
    }
    __syncthreads();
    if (!last || threadIdx.x >= 32) return;
    const int lane = threadIdx.x;
    __threadfence();
    Cand b{-1e300, 0x7fffffff};
    for (int k = lane; k < static_cast<int>(gridDim.x); k += 32) {
        const int slot = blockIdx.y * gridDim.x + k;
        const Cand c{static_cast<volatile double*>(sc.gain)[slot], static_cast<volatile int*>(sc.key)[slot]};
        if (better(c, b)) b = c;
    }
    b = warp_best(b);
    if (lane == 0) {
        DevSplit s;
        s.gain = b.gain;
        s.valid = (b.key != 0x7fffffff) && b.gain >= p.min_split_gain;
        s.feature = s.valid ? b.key / 512 : -1;
        s.threshold = s.valid ? (b.key % 512) / 2 : -1;
        s.missing_left = s.valid ? (b.key & 1) : 1;
        splits[nd] = s;
        sc.ticket[blockIdx.y] = 0;  // ready for the next launch
    }
    // The last node of the launch to finish picks the next leaf to split.
    int sel = 0;
    if (lane == 0 && do_select) {
        __threadfence();
        sel = atomicAdd(&sc.ticket[2], 1) == static_cast<int>(gridDim.y) - 1;
        if (sel) sc.ticket[2] = 0;
        __threadfence();
    }
    sel = __shfl_sync(0xffffffffu, sel, 0);
    if (sel) select_body(p, nodes, splits, st);
}

// grow_tree's leaf choice (cpp/src/tree.cpp:343-383), one warp.  Split records are read
// past L1 (__ldcg): inside the fused scan they were written by other CTAs of the launch.
__device__ void select_body(const GrowParams& p, DevNode* __restrict__ nodes, DevSplit* __restrict__ splits,
                            DevTreeState* __restrict__ st) {
    const int lane = threadIdx.x & 31;
    const int nn = st->n_nodes;
    double best_gain = p.min_split_gain;
    int best_id = 0x7fffffff;
    for (int k = lane; k < nn; k += 32) {
        const DevNode& N = nodes[k];
        if (!N.is_leaf || N.depth >= p.max_depth || N.count < 2 * p.min_samples_leaf) continue;
        const int valid = __ldcg(&splits[k].valid);
        const double gain = __ldcg(&splits[k].gain);
        if (!valid || !(gain >= p.min_split_gain)) continue;
        if (gain > best_gain) {
            best_gain = gain;
            best_id = k;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double og = __shfl_xor_sync(0xffffffffu, best_gain, o);
        const int oid = __shfl_xor_sync(0xffffffffu, best_id, o);
        if (og > best_gain || (og == best_gain && oid < best_id)) {
            best_gain = og;
            best_id = oid;
        }
    }
    if (lane != 0) return;
    if (best_id == 0x7fffffff) {
        st->done = 1;
        return;
    }
    DevNode& P = nodes[best_id];
    P.is_leaf = 0;
    P.feature = __ldcg(&splits[best_id].feature);
    P.threshold = __ldcg(&splits[best_id].threshold);
    P.missing_left = __ldcg(&splits[best_id].missing_left);
    P.gain = __ldcg(&splits[best_id].gain);
    const int l = nn, r = nn + 1;
    P.left = l;
    P.right = r;
    for (int c = 0; c < 2; ++c) {
        DevNode ch{};
        ch.start = P.start;
        ch.count = 0;
        ch.buf = 1 - P.buf;
        ch.depth = P.depth + 1;
        ch.is_leaf = 1;
        ch.feature = -1;
        ch.threshold = -1;
        ch.missing_left = 1;
        ch.left = ch.right = -1;
        ch.parent = best_id;
        nodes[nn + c] = ch;
        splits[nn + c].valid = 0;
    }
    st->parent = best_id;
    st->n_nodes = nn + 2;
}

__global__ void __launch_bounds__(kScanThreads)
    scan_hist_kernel(const long long* G, const long long* H, const int* C, int n_f, int n_bins,
                     double inv_gs, double inv_hs, double lam, double gamma, int min_leaf,
                     double min_hess, double* gain, int* thr, int* ml) {
    const int f = blockIdx.x;
    __shared__ ScanShared sm;
    long long Gt, Ht, Ct;
    const size_t fo = static_cast<size_t>(f) * kBins;
    long long* Gm = const_cast<long long*>(G + fo);
    long long* Hm = const_cast<long long*>(H + fo);
    int* Cm = const_cast<int*>(C + fo);
    const Cand c = scan_feature(Gm, Hm, Cm, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, false, true, f,
                                n_bins, inv_gs, inv_hs, lam, gamma, min_leaf, min_hess, sm, Gt, Ht, Ct);
    if (threadIdx.x == 0) {
        const bool ok = c.key != 0x7fffffff;
        gain[f] = c.gain;
        thr[f] = ok ? (c.key % 512) / 2 : -1;
        ml[f] = ok ? (c.key & 1) : 1;
    }
}

}  // namespace

int scan_ctas_per_node(int n_f) { return n_f; }

void launch_split_scan(const GrowParams& p, HistSlotPtrs hs, DevNode* nodes, DevSplit* splits, DevTreeState* st,
                       int mode, int node, ScanScratch sc, bool do_select, cudaStream_t s) {
    dim3 grid(scan_ctas_per_node(p.n_features), mode == 1 ? 2 : 1);
    launch_pdl(split_scan_kernel, grid, dim3(kScanThreads), 0, s, "split_scan launch", p, hs, nodes, splits, st, mode,
               node, sc, do_select ? 1 : 0);
}

void launch_scan_hist(const long long* G, const long long* H, const int* C, int n_f, int n_bins,
                      double inv_gscale, double inv_hscale, double lam, double gamma, int min_leaf,
                      double min_hess, double* gain, int* thr, int* ml, cudaStream_t s) {
    if (n_f <= 0) return;
    scan_hist_kernel<<<n_f, kScanThreads, 0, s>>>(
        G, H, C, n_f, n_bins, inv_gscale, inv_hscale, lam, gamma, min_leaf, min_hess, gain, thr, ml);
    check(cudaGetLastError(), "scan_hist launch");
}

}  // namespace tgb
