// Split-scan building blocks shared by the per-node scan (kernels_split.cu) and the
// batched wave scan (kernels_wave_scan.cu): restates best_numeric_missing
// (cpp/src/histogram.cpp:126-193, l1 = 0, no monotone) for one feature of a fixed-point
// histogram.  Every translation unit that includes this file is compiled with
// -fmad=false so the gain arithmetic follows the reference's statement order.
#pragma once

#include "tgb_internal.h"

namespace tgb {
namespace scan {

constexpr int kScanThreads = kBins;  // thread = bin
constexpr int kScanWarps = kScanThreads / 32;

struct Cand {
    double gain;
    int key;  // feature * 512 + threshold * 2 + missing_left
};

__device__ __forceinline__ bool better(const Cand& a, const Cand& b) {
    return a.gain > b.gain || (a.gain == b.gain && a.key < b.key);
}

__device__ __forceinline__ long long warp_incl_scan(long long v, int lane) {
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const long long t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

__device__ __forceinline__ Cand warp_best(Cand best) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        Cand other{__shfl_xor_sync(0xffffffffu, best.gain, o), __shfl_xor_sync(0xffffffffu, best.key, o)};
        if (better(other, best)) best = other;
    }
    return best;
}

struct ScanShared {
    long long wg[kScanWarps], wh[kScanWarps], wc[kScanWarps];
    long long g0, h0, c0;
    Cand wbest[kScanWarps];
};

// One CTA scans one feature of a histogram; thread b owns bin b.  Returns the CTA's
// best candidate in thread 0 and the feature's totals in every thread.  derive: the
// histogram is first derived as parent - small sibling (subtract_hist_inplace,
// cpp/src/histogram.cpp:108-117, exact in fixed point) and stored to Gf / Hf / Cf.
// scan = false only derives and totals (a node that cannot split).
__device__ __forceinline__ Cand scan_feature(long long* __restrict__ Gf, long long* __restrict__ Hf, int* __restrict__ Cf,
                             const long long* __restrict__ PGf, const long long* __restrict__ PHf,
                             const int* __restrict__ PCf, const long long* __restrict__ SGf,
                             const long long* __restrict__ SHf, const int* __restrict__ SCf, bool derive, bool scan,
                             int f, int n_bins, double inv_gs, double inv_hs, double lam, double gamma, int min_leaf,
                             double min_hess, ScanShared& sm, long long& Gt, long long& Ht, long long& Ct) {
    const int b = threadIdx.x, lane = b & 31, warp = b >> 5;
    long long g, hh, c;
    if (derive) {
        g = PGf[b] - SGf[b];
        hh = PHf[b] - SHf[b];
        c = PCf[b] - SCf[b];
        Gf[b] = g;
        Hf[b] = hh;
        Cf[b] = static_cast<int>(c);
    } else {
        g = Gf[b];
        hh = Hf[b];
        c = Cf[b];
    }
    long long ig = warp_incl_scan(g, lane), ih = warp_incl_scan(hh, lane), ic = warp_incl_scan(c, lane);
    if (lane == 31) {
        sm.wg[warp] = ig;
        sm.wh[warp] = ih;
        sm.wc[warp] = ic;
    }
    if (b == 0) {
        sm.g0 = g;
        sm.h0 = hh;
        sm.c0 = c;
    }
    __syncthreads();
    Gt = Ht = Ct = 0;
#pragma unroll
    for (int w = 0; w < kScanWarps; ++w) {
        if (w < warp) {
            ig += sm.wg[w];
            ih += sm.wh[w];
            ic += sm.wc[w];
        }
        Gt += sm.wg[w];
        Ht += sm.wh[w];
        Ct += sm.wc[w];
    }
    Cand best{-1e300, 0x7fffffff};
    if (scan && b >= 1 && b <= n_bins - 2 && c != 0) {
        const long long G0 = sm.g0, H0 = sm.h0, C0 = sm.c0;
        const double dGt = static_cast<double>(Gt) * inv_gs, dHt = static_cast<double>(Ht) * inv_hs;
        const double parent = (dGt * dGt) / (dHt + lam);
        const long long GL = ig - G0, HL = ih - H0, CL = ic - C0;  // bins 1..b
#pragma unroll
        for (int ml = 0; ml <= 1; ++ml) {
            const long long gL = GL + (ml ? G0 : 0), hL = HL + (ml ? H0 : 0), cL = CL + (ml ? C0 : 0);
            const long long cR = Ct - cL;
            if (cL < min_leaf || cR < min_leaf) continue;
            const double dgL = static_cast<double>(gL) * inv_gs, dhL = static_cast<double>(hL) * inv_hs;
            const double dgR = static_cast<double>(Gt - gL) * inv_gs, dhR = static_cast<double>(Ht - hL) * inv_hs;
            if (dhL < min_hess || dhR < min_hess) continue;
            const double gain = 0.5 * ((dgL * dgL) / (dhL + lam) + (dgR * dgR) / (dhR + lam) - parent) - gamma;
            const Cand cand{gain, f * 512 + b * 2 + ml};
            if (better(cand, best)) best = cand;
        }
    }
    if (!scan) return best;
    best = warp_best(best);
    if (lane == 0) sm.wbest[warp] = best;
    __syncthreads();
    if (b == 0) {
#pragma unroll
        for (int w = 1; w < kScanWarps; ++w)
            if (better(sm.wbest[w], best)) best = sm.wbest[w];
    }
    return best;
}

// One warp scans one feature: lane l owns bins [8l, 8l + 8) (the same arithmetic, in the
// same order, as scan_feature, without block barriers).  Returns the warp's best candidate
// and the feature's totals in every lane.
__device__ __forceinline__ Cand scan_feature_warp(long long* __restrict__ Gf, long long* __restrict__ Hf,
                                                  int* __restrict__ Cf, const long long* __restrict__ PGf,
                                                  const long long* __restrict__ PHf, const int* __restrict__ PCf,
                                                  const long long* __restrict__ SGf, const long long* __restrict__ SHf,
                                                  const int* __restrict__ SCf, bool derive, bool scan, int f, int n_bins,
                                                  double inv_gs, double inv_hs, double lam, double gamma, int min_leaf,
                                                  double min_hess, long long& Gt, long long& Ht, long long& Ct) {
    constexpr int kPer = kBins / 32;
    const int lane = threadIdx.x & 31, b0 = lane * kPer;
    long long g[kPer], hh[kPer], c[kPer];
    {
        const longlong2* g2 = reinterpret_cast<const longlong2*>((derive ? PGf : Gf) + b0);
        const longlong2* h2 = reinterpret_cast<const longlong2*>((derive ? PHf : Hf) + b0);
        const int4* c4 = reinterpret_cast<const int4*>((derive ? PCf : Cf) + b0);
#pragma unroll
        for (int i = 0; i < kPer / 2; ++i) {
            const longlong2 a = g2[i], b = h2[i];
            g[2 * i] = a.x;
            g[2 * i + 1] = a.y;
            hh[2 * i] = b.x;
            hh[2 * i + 1] = b.y;
        }
#pragma unroll
        for (int i = 0; i < kPer / 4; ++i) {
            const int4 a = c4[i];
            c[4 * i] = a.x;
            c[4 * i + 1] = a.y;
            c[4 * i + 2] = a.z;
            c[4 * i + 3] = a.w;
        }
    }
    if (derive) {
        const longlong2* g2 = reinterpret_cast<const longlong2*>(SGf + b0);
        const longlong2* h2 = reinterpret_cast<const longlong2*>(SHf + b0);
        const int4* c4 = reinterpret_cast<const int4*>(SCf + b0);
#pragma unroll
        for (int i = 0; i < kPer / 2; ++i) {
            const longlong2 a = g2[i], b = h2[i];
            g[2 * i] -= a.x;
            g[2 * i + 1] -= a.y;
            hh[2 * i] -= b.x;
            hh[2 * i + 1] -= b.y;
        }
#pragma unroll
        for (int i = 0; i < kPer / 4; ++i) {
            const int4 a = c4[i];
            c[4 * i] -= a.x;
            c[4 * i + 1] -= a.y;
            c[4 * i + 2] -= a.z;
            c[4 * i + 3] -= a.w;
        }
        longlong2* go = reinterpret_cast<longlong2*>(Gf + b0);
        longlong2* ho = reinterpret_cast<longlong2*>(Hf + b0);
        int4* co = reinterpret_cast<int4*>(Cf + b0);
#pragma unroll
        for (int i = 0; i < kPer / 2; ++i) {
            go[i] = make_longlong2(g[2 * i], g[2 * i + 1]);
            ho[i] = make_longlong2(hh[2 * i], hh[2 * i + 1]);
        }
#pragma unroll
        for (int i = 0; i < kPer / 4; ++i)
            co[i] = make_int4(static_cast<int>(c[4 * i]), static_cast<int>(c[4 * i + 1]), static_cast<int>(c[4 * i + 2]),
                              static_cast<int>(c[4 * i + 3]));
    }
    long long tg = 0, th = 0, tc = 0;
#pragma unroll
    for (int i = 0; i < kPer; ++i) {
        tg += g[i];
        th += hh[i];
        tc += c[i];
    }
    const long long ig = warp_incl_scan(tg, lane), ih = warp_incl_scan(th, lane), ic = warp_incl_scan(tc, lane);
    Gt = __shfl_sync(0xffffffffu, ig, 31);
    Ht = __shfl_sync(0xffffffffu, ih, 31);
    Ct = __shfl_sync(0xffffffffu, ic, 31);
    const long long G0 = __shfl_sync(0xffffffffu, g[0], 0), H0 = __shfl_sync(0xffffffffu, hh[0], 0),
                    C0 = __shfl_sync(0xffffffffu, c[0], 0);
    Cand best{-1e300, 0x7fffffff};
    if (scan) {
        const double dGt = static_cast<double>(Gt) * inv_gs, dHt = static_cast<double>(Ht) * inv_hs;
        const double parent = (dGt * dGt) / (dHt + lam);
        long long rg = ig - tg, rh = ih - th, rc = ic - tc;  // bins before this lane's
#pragma unroll
        for (int i = 0; i < kPer; ++i) {
            rg += g[i];
            rh += hh[i];
            rc += c[i];
            const int b = b0 + i;
            if (b < 1 || b > n_bins - 2 || c[i] == 0) continue;
            const long long GL = rg - G0, HL = rh - H0, CL = rc - C0;  // bins 1..b
#pragma unroll
            for (int ml = 0; ml <= 1; ++ml) {
                const long long gL = GL + (ml ? G0 : 0), hL = HL + (ml ? H0 : 0), cL = CL + (ml ? C0 : 0);
                const long long cR = Ct - cL;
                if (cL < min_leaf || cR < min_leaf) continue;
                const double dgL = static_cast<double>(gL) * inv_gs, dhL = static_cast<double>(hL) * inv_hs;
                const double dgR = static_cast<double>(Gt - gL) * inv_gs, dhR = static_cast<double>(Ht - hL) * inv_hs;
                if (dhL < min_hess || dhR < min_hess) continue;
                const double gain = 0.5 * ((dgL * dgL) / (dhL + lam) + (dgR * dgR) / (dhR + lam) - parent) - gamma;
                const Cand cand{gain, f * 512 + b * 2 + ml};
                if (better(cand, best)) best = cand;
            }
        }
        best = warp_best(best);
    }
    return best;
}

// ---- categorical features ---------------------------------------------------------------
//
// std::sort of libstdc++ (introsort: median-of-three quicksort down to runs of 16, heap
// sort past 2 * floor(log2 n) levels, then insertion sort), restated step for step so
// that elements the comparator ties end in the order the reference's std::sort leaves
// them (best_categorical sorts bins by a ratio that ties for bins of equal sums).  One
// thread, at most 256 elements in shared memory; less(a, b) compares two elements.
template <typename Less>
__device__ void libstdcxx_sort(short* v, int n, Less less) {
    struct Sorter {
        short* v;
        Less less;
        __device__ void swap(int a, int b) {
            const short t = v[a];
            v[a] = v[b];
            v[b] = t;
        }
        __device__ void push_heap(int first, int hole, int top, short value) {
            int parent = (hole - 1) / 2;
            while (hole > top && less(v[first + parent], value)) {
                v[first + hole] = v[first + parent];
                hole = parent;
                parent = (hole - 1) / 2;
            }
            v[first + hole] = value;
        }
        __device__ void adjust_heap(int first, int hole, int len, short value) {
            const int top = hole;
            int second = hole;
            while (second < (len - 1) / 2) {
                second = 2 * (second + 1);
                if (less(v[first + second], v[first + second - 1])) --second;
                v[first + hole] = v[first + second];
                hole = second;
            }
            if ((len & 1) == 0 && second == (len - 2) / 2) {
                second = 2 * (second + 1);
                v[first + hole] = v[first + second - 1];
                hole = second - 1;
            }
            push_heap(first, hole, top, value);
        }
        __device__ void make_heap(int first, int last) {
            const int len = last - first;
            if (len < 2) return;
            for (int parent = (len - 2) / 2;; --parent) {
                adjust_heap(first, parent, len, v[first + parent]);
                if (parent == 0) return;
            }
        }
        __device__ void pop_heap(int first, int last, int result) {
            const short value = v[result];
            v[result] = v[first];
            adjust_heap(first, 0, last - first, value);
        }
        __device__ void heap_sort(int first, int last) {  // __partial_sort(first, last, last)
            make_heap(first, last);
            while (last - first > 1) {
                --last;
                pop_heap(first, last, last);
            }
        }
        __device__ void move_median_to_first(int result, int a, int b, int c) {
            if (less(v[a], v[b])) {
                if (less(v[b], v[c])) swap(result, b);
                else if (less(v[a], v[c])) swap(result, c);
                else swap(result, a);
            } else if (less(v[a], v[c])) {
                swap(result, a);
            } else if (less(v[b], v[c])) {
                swap(result, c);
            } else {
                swap(result, b);
            }
        }
        __device__ int unguarded_partition(int first, int last, int pivot) {
            while (true) {
                while (less(v[first], v[pivot])) ++first;
                --last;
                while (less(v[pivot], v[last])) --last;
                if (!(first < last)) return first;
                swap(first, last);
                ++first;
            }
        }
        __device__ void introsort_loop(int first, int last, int depth) {
            // recursion on the right part, as libstdc++ does; depth <= 2 * log2(256)
            while (last - first > 16) {
                if (depth == 0) {
                    heap_sort(first, last);
                    return;
                }
                --depth;
                const int mid = first + (last - first) / 2;
                move_median_to_first(first, first + 1, mid, last - 1);
                const int cut = unguarded_partition(first + 1, last, first);
                introsort_loop(cut, last, depth);
                last = cut;
            }
        }
        __device__ void unguarded_linear_insert(int last) {
            const short val = v[last];
            int next = last - 1;
            while (less(val, v[next])) {
                v[last] = v[next];
                last = next;
                --next;
            }
            v[last] = val;
        }
        __device__ void insertion_sort(int first, int last) {
            if (first == last) return;
            for (int i = first + 1; i != last; ++i) {
                if (less(v[i], v[first])) {
                    const short val = v[i];
                    for (int k = i; k > first; --k) v[k] = v[k - 1];
                    v[first] = val;
                } else {
                    unguarded_linear_insert(i);
                }
            }
        }
    };
    if (n < 2) return;
    Sorter s{v, less};
    int lg = 31 - __clz(n);
    s.introsort_loop(0, n, 2 * lg);
    if (n > 16) {
        s.insertion_sort(0, 16);
        for (int i = 16; i < n; ++i) s.unguarded_linear_insert(i);
    } else {
        s.insertion_sort(0, n);
    }
}

struct CatShared {
    double key[kBins];   // ranking ratio of each bin
    short order[kBins];  // non-empty bins, then sorted
    int nnz;
    int wcnt[kScanWarps];
    long long pg[kScanWarps], ph[kScanWarps], pc[kScanWarps];
    Cand wbest[kScanWarps];
    unsigned long long mask[4];
};

// best_categorical (cpp/src/histogram.cpp:195-244, l1 = 0) for one feature of a stored
// fixed-point histogram (thread b owns bin b): the non-empty bins (the missing bin 0
// included) ranked by g / (h + cat_smooth) with std::sort's own order, the best prefix
// of that ranking as the left side (strict '>' over the prefixes: the first best wins).
// Gt / Ht / Ct: the node's totals.  Returns the candidate (key f * 512) and the left mask.
static __device__ __noinline__ Cand scan_categorical(const long long* __restrict__ Gf, const long long* __restrict__ Hf,
                                              const int* __restrict__ Cf, int f, double inv_gs, double inv_hs,
                                              double lam, double gamma, int min_leaf, double min_hess,
                                              double cat_smooth, long long Gt, long long Ht, long long Ct,
                                              CatShared& cs, unsigned long long* mask_out) {
    const int b = threadIdx.x, lane = b & 31, warp = b >> 5;
    const double sm = fmax(cat_smooth, 0.0);
    const long long g = Gf[b], hh = Hf[b];
    const int c = Cf[b];
    const bool ne = c > 0;
    const unsigned bal = __ballot_sync(0xffffffffu, ne);
    if (lane == 0) cs.wcnt[warp] = __popc(bal);
    if (b < 4) cs.mask[b] = 0ull;
    cs.key[b] = (static_cast<double>(g) * inv_gs) / (static_cast<double>(hh) * inv_hs + sm);
    __syncthreads();
    int before = 0, nnz = 0;
#pragma unroll
    for (int w = 0; w < kScanWarps; ++w) {
        if (w < warp) before += cs.wcnt[w];
        nnz += cs.wcnt[w];
    }
    if (ne) cs.order[before + __popc(bal & ((1u << lane) - 1u))] = static_cast<short>(b);
    __syncthreads();
    Cand best{-1e300, 0x7fffffff};
    if (nnz < 2) return best;
    if (b == 0) libstdcxx_sort(cs.order, nnz, [&](short x, short y) { return cs.key[x] < cs.key[y]; });
    __syncthreads();
    // prefix sums over the ranking, exact
    const int o = b < nnz ? cs.order[b] : 0;
    long long pg = b < nnz ? Gf[o] : 0, ph = b < nnz ? Hf[o] : 0, pc = b < nnz ? Cf[o] : 0;
    pg = warp_incl_scan(pg, lane);
    ph = warp_incl_scan(ph, lane);
    pc = warp_incl_scan(pc, lane);
    if (lane == 31) {
        cs.pg[warp] = pg;
        cs.ph[warp] = ph;
        cs.pc[warp] = pc;
    }
    __syncthreads();
#pragma unroll
    for (int w = 0; w < kScanWarps; ++w)
        if (w < warp) {
            pg += cs.pg[w];
            ph += cs.ph[w];
            pc += cs.pc[w];
        }
    if (b + 1 < nnz) {
        const long long CL = pc, CR = Ct - pc;
        const double dGt = static_cast<double>(Gt) * inv_gs, dHt = static_cast<double>(Ht) * inv_hs;
        const double parent = (dGt * dGt) / (dHt + lam);
        const double GL = static_cast<double>(pg) * inv_gs, HL = static_cast<double>(ph) * inv_hs;
        const double GR = static_cast<double>(Gt - pg) * inv_gs, HR = static_cast<double>(Ht - ph) * inv_hs;
        if (!(CL < min_leaf || CR < min_leaf) && !(HL < min_hess || HR < min_hess)) {
            const double gain = 0.5 * ((GL * GL) / (HL + lam) + (GR * GR) / (HR + lam) - parent) - gamma;
            best = Cand{gain, b};  // key: the prefix position for now (first best wins)
        }
    }
    best = warp_best(best);
    if (lane == 0) cs.wbest[warp] = best;
    __syncthreads();
    best = cs.wbest[0];
#pragma unroll
    for (int w = 1; w < kScanWarps; ++w)
        if (better(cs.wbest[w], best)) best = cs.wbest[w];
    if (best.key == 0x7fffffff) return best;
    if (b <= best.key) atomicOr(&cs.mask[o >> 6], 1ull << (o & 63));
    __syncthreads();
    if (b < 4) mask_out[b] = cs.mask[b];
    return Cand{best.gain, f * 512};
}


}  // namespace scan
}  // namespace tgb
