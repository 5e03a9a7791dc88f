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


}  // namespace scan
}  // namespace tgb
