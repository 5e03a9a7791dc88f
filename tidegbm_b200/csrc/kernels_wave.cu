// Wave kernels: batched histograms and partitions over many leaves of many trees, and
// the per-tree set-up of a context (wave.h describes the scheme).
//
// Histogram (build_hist_col, cpp/src/histogram.cpp:44-76, for the smaller child of every
// planned leaf; subtract_hist_inplace's larger child is derived in the scan).  One
// persistent launch of clusters of 1, 2 or 4 CTAs (the autotuned privatisation depth:
// how many CTA-private histograms a flush merges).  The work is cut into units (context,
// leaf, group of 32 features, chunk of rows), about `units` per cluster; a cluster takes
// units in turn and its CTAs split the unit's rows.  Inside a CTA the accumulation is the lane-per-row scheme:
// a warp takes 32 rows, lane l loads its row's 32 code bytes of the group with two
// 16-byte loads and rotates them by l bytes in registers, so step j of the 32-step loop
// touches feature (j + l) & 31: 32 lanes, 32 features, 32 banks of the [bin][feature]
// layout, conflict-free whatever the codes.  Every code costs fire-and-forget 32-bit
// shared reductions only (their count depends on the payload mode, below), exact over a
// sub-chunk of rows, folded into per-thread 64-bit registers after every sub-chunk.  At
// the end of a unit the cluster adds its partial histograms through distributed shared
// memory and each CTA flushes its share of the cells with 64-bit global atomics.
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
constexpr int kTotPlanes = 5;  // totals: G lo, G hi, H lo, H hi, count
constexpr size_t kPlaneBytes = static_cast<size_t>(kPlane) * 4;
constexpr size_t kJobBytes = static_cast<size_t>(kMaxWaveJobs) * 4 * 3 + 4 * 8;
constexpr size_t kWaveSmem = kPlaneBytes * kTotPlanes + kJobBytes;
constexpr int kLoBits = 19;
constexpr int kMinUnitRows = 4096;

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
    int count;
    int slot;
};

__device__ __forceinline__ JobRows job_rows(const WaveCtx& X, int src, int e) {
    JobRows r;
    if (src == 0) {
        r.rows = X.rows0;
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
    r.count = c.count;
    r.slot = c.slot;
    return r;
}

// The rows [r0, r1) of one unit (one group of 32 features), lane = row: a warp takes 32
// rows, lane l loads its row's 32 code bytes with two 16-byte loads and rotates them by l
// bytes, so step j touches feature (j + l) & 31 (conflict-free banks); every code costs
// the mode's fire-and-forget 32-bit reductions, folded into 64-bit registers every
// sub-chunk.  Ends with the CTA's totals in the 5 planes (G lo, G hi, H lo, H hi, count).
// A separate (not inlined) function: the hot loop keeps only its own state in registers.
// Row counts of the constant-hessian modes travel packed (unscaled | GOSS-scaled << 16);
// a CTA's share of a unit has fewer than 2^16 rows.
template <int kMode>
__device__ __noinline__ void accumulate_unit(unsigned int* __restrict__ P, const int32_t* __restrict__ rows, int r0,
                                             int r1, const uint8_t* __restrict__ codes, int stride, int fg0,
                                             const void* __restrict__ gqp, const void* __restrict__ hqp,
                                             unsigned long long hq1, unsigned long long hq2) {
    using T = ModeTraits<kMode>;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int q = lane >> 2, sh = (lane & 3) * 8;
    const bool two_chunks = stride - fg0 >= 32;
    long long accG[kCells];
    long long accH[T::var ? kCells : 1];
    unsigned int accC[kCells];
#pragma unroll
    for (int cc = 0; cc < kCells; ++cc) {
        accG[cc] = 0;
        if constexpr (T::var) accH[cc] = 0;
        accC[cc] = 0u;
    }
    for (int s0 = r0; s0 < r1; s0 += T::sub) {
        const int s1 = min(r1, s0 + T::sub);
        int r_next = s0 + warp * 32 + lane < s1 ? rows[s0 + warp * 32 + lane] : -1;
        for (int base = s0 + warp * 32; base < s1; base += kWarps * 32) {
            const int r = r_next;
            const int kn = base + kWarps * 32 + lane;
            r_next = kn < s1 ? rows[kn] : -1;
            if (r < 0) continue;
            // payload words of this row (mode dependent)
            unsigned int a0 = 0, a1 = 0, a2 = 0, a3 = 0;
            unsigned int* plane = P;
            if constexpr (kMode == kHistExactConst) {
                const long long p = static_cast<const long long*>(gqp)[r];
                const long long v = p >> 1;
                a0 = static_cast<unsigned int>(v) & ((1u << kLoBits) - 1u);
                a1 = static_cast<unsigned int>(static_cast<int>(v >> kLoBits));
                a2 = (p & 1) ? 0x10000u : 1u;
            } else if constexpr (kMode == kHistExactVar) {
                const long long gv = static_cast<const long long*>(gqp)[r];
                const long long hv = static_cast<const long long*>(hqp)[r];
                a0 = static_cast<unsigned int>(gv) & ((1u << kLoBits) - 1u);
                a1 = static_cast<unsigned int>(static_cast<int>(gv >> kLoBits));
                a2 = static_cast<unsigned int>(hv) & ((1u << kLoBits) - 1u);
                a3 = static_cast<unsigned int>(static_cast<int>(hv >> kLoBits));
            } else if constexpr (kMode == kHistQ16Const) {
                const int p = static_cast<const int*>(gqp)[r];
                a0 = static_cast<unsigned int>(p >> 1);
                a1 = (p & 1) ? 0x10000u : 1u;
            } else if constexpr (kMode == kHistQ16Var) {
                const unsigned int p = static_cast<const unsigned int*>(gqp)[r];
                a0 = static_cast<unsigned int>(static_cast<int>(p) >> 16);
                a1 = p & 0xffffu;
            } else if constexpr (kMode == kHistQ8Const) {
                const int p = static_cast<const short*>(gqp)[r];
                a0 = (1u << 20) | static_cast<unsigned int>((p >> 1) + 128);
                plane = (p & 1) ? P + kPlane : P;
            } else {  // kHistQ8Var
                const unsigned int p = static_cast<const unsigned short*>(gqp)[r];
                a0 = (1u << 20) | (p & 0xffu);
                a1 = p >> 8;
            }
            const uint4* src4 = reinterpret_cast<const uint4*>(codes + static_cast<size_t>(r) * stride + fg0);
            const uint4 ca = __ldg(src4);
            const uint4 cb = two_chunks ? __ldg(src4 + 1) : make_uint4(0, 0, 0, 0);
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
                } else if constexpr (kMode == kHistExactVar) {
                    atomicAdd(&P[cell], a0);
                    atomicAdd(&P[kPlane + cell], a1);
                    atomicAdd(&P[2 * kPlane + cell], a2);
                    atomicAdd(&P[3 * kPlane + cell], a3);
                    atomicAdd(&P[4 * kPlane + cell], 1u);
                } else if constexpr (kMode == kHistQ16Const) {
                    atomicAdd(&P[cell], a0);
                    atomicAdd(&P[kPlane + cell], a1);
                } else if constexpr (kMode == kHistQ16Var) {
                    atomicAdd(&P[cell], a0);
                    atomicAdd(&P[kPlane + cell], a1);
                    atomicAdd(&P[2 * kPlane + cell], 1u);
                } else if constexpr (kMode == kHistQ8Const) {
                    atomicAdd(&plane[cell], a0);
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
            if constexpr (kMode == kHistExactConst) {
                accG[cc] += static_cast<long long>(static_cast<int>(P[kPlane + cell])) * (1ll << kLoBits) + P[cell];
                accC[cc] += P[2 * kPlane + cell];
            } else if constexpr (kMode == kHistExactVar) {
                accG[cc] += static_cast<long long>(static_cast<int>(P[kPlane + cell])) * (1ll << kLoBits) + P[cell];
                accH[cc] +=
                    static_cast<long long>(static_cast<int>(P[3 * kPlane + cell])) * (1ll << kLoBits) + P[2 * kPlane + cell];
                accC[cc] += P[4 * kPlane + cell];
            } else if constexpr (kMode == kHistQ16Const) {
                accG[cc] += static_cast<int>(P[cell]);
                accC[cc] += P[kPlane + cell];
            } else if constexpr (kMode == kHistQ16Var) {
                accG[cc] += static_cast<int>(P[cell]);
                accH[cc] += P[kPlane + cell];
                accC[cc] += P[2 * kPlane + cell];
            } else if constexpr (kMode == kHistQ8Const) {
                const unsigned int w1 = P[cell], w2 = P[kPlane + cell];
                const unsigned int n1 = w1 >> 20, n2 = w2 >> 20;
                accG[cc] += static_cast<long long>(w1 & 0xfffffu) + static_cast<long long>(w2 & 0xfffffu) -
                            128ll * static_cast<long long>(n1 + n2);
                accC[cc] += n1 | (n2 << 16);
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
    // totals -> 5 planes
#pragma unroll
    for (int cc = 0; cc < kCells; ++cc) {
        const int cell = threadIdx.x + cc * kThreads;
        unsigned long long Hs;
        unsigned int Cn;
        if constexpr (T::var) {
            Hs = static_cast<unsigned long long>(accH[cc]);
            Cn = accC[cc];
        } else {
            const unsigned int c1 = accC[cc] & 0xffffu, c2 = accC[cc] >> 16;
            Hs = static_cast<unsigned long long>(c1) * hq1 + static_cast<unsigned long long>(c2) * hq2;
            Cn = c1 + c2;
        }
        const unsigned long long Gs = static_cast<unsigned long long>(accG[cc]);
        P[cell] = static_cast<unsigned int>(Gs);
        P[kPlane + cell] = static_cast<unsigned int>(Gs >> 32);
        P[2 * kPlane + cell] = static_cast<unsigned int>(Hs);
        P[3 * kPlane + cell] = static_cast<unsigned int>(Hs >> 32);
        P[4 * kPlane + cell] = Cn;
    }
}

template <int kMode>
__global__ void __launch_bounds__(kThreads, 1)
    wave_hist_kernel(const WaveCtx* __restrict__ ctxs, int n_ctx, int src, unsigned long long* rows_counter,
                     int unit_target) {
    using T = ModeTraits<kMode>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    unsigned int* P = reinterpret_cast<unsigned int*>(smem_raw);  // planes
    int* s_ustart = reinterpret_cast<int*>(smem_raw + kPlaneBytes * kTotPlanes);  // [kMaxWaveJobs]
    int* s_job = s_ustart + kMaxWaveJobs;                                            // ctx << 16 | exp
    int* s_rows = s_job + kMaxWaveJobs;                                              // job row counts
    int* s_misc = s_rows + kMaxWaveJobs;  // [0] jobs, [1] units, [2] unit rows, [3..7] reduction
    {  // private state first: it overlaps the previous kernel's tail
        uint4* z = reinterpret_cast<uint4*>(smem_raw);
        for (int k = threadIdx.x; k < T::planes * kPlane / 4; k += blockDim.x) z[k] = make_uint4(0, 0, 0, 0);
    }
    pdl_wait();
    pdl_trigger();

    // ---- unit plan (the same in every CTA) ----
    __shared__ int s_cpref[kMaxWaveCtx + 1];
    __shared__ unsigned long long s_red[kWarps];
    __shared__ int s_wsum[kWarps];
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
    unsigned long long w = 0;
    for (int j = threadIdx.x; j < n_jobs; j += blockDim.x) {
        int c = 0;
        while (c + 1 < n_ctx && s_cpref[c + 1] <= j) ++c;
        const int e = src == 0 ? 0 : j - s_cpref[c];
        const WaveCtx& X = ctxs[c];
        const JobRows jr = job_rows(X, src, e);
        const int nfg = (X.gp.n_features + kFG - 1) / kFG;
        s_job[j] = (c << 16) | e;
        s_rows[j] = jr.count;
        s_ustart[j] = nfg;  // feature groups for now; units below
        w += static_cast<unsigned long long>(jr.count) * nfg;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
    if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = w;
    __syncthreads();
    int unit_rows_b;
    {
        unsigned long long tot = 0;
        for (int k = 0; k < kWarps; ++k) tot += s_red[k];
        const int n_cl0 = static_cast<int>(gridDim.y / cg::this_cluster().dim_blocks().y);
        const unsigned long long target =
            static_cast<unsigned long long>(max(1, unit_target)) * static_cast<unsigned long long>(max(1, n_cl0));
        const unsigned long long u = (tot + target - 1) / target;
        // a CTA's share of a unit stays below 2^16 rows: its row counts pack into 16-bit fields
        const unsigned long long cap = 65535ull * cg::this_cluster().dim_blocks().y;
        unit_rows_b = static_cast<int>(min(max(static_cast<unsigned long long>(kMinUnitRows), u), cap));
    }
    // units of each job: exclusive prefix over the jobs, a contiguous run per thread
    {
        const int per = (n_jobs + kThreads - 1) / kThreads;
        const int j0 = threadIdx.x * per, j1 = min(n_jobs, j0 + per);
        int local = 0;
        for (int j = j0; j < j1; ++j) {
            const int r = s_rows[j];
            const int units = r > 0 ? s_ustart[j] * ((r + unit_rows_b - 1) / unit_rows_b) : 0;
            s_ustart[j] = units;
            local += units;
        }
        const int lane0 = threadIdx.x & 31, warp0 = threadIdx.x >> 5;
        int incl = local;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int t = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane0 >= o) incl += t;
        }
        if (lane0 == 31) s_wsum[warp0] = incl;
        __syncthreads();
        int wbase = 0, all = 0;
        for (int k = 0; k < kWarps; ++k) {
            if (k < warp0) wbase += s_wsum[k];
            all += s_wsum[k];
        }
        int run = wbase + incl - local;
        for (int j = j0; j < j1; ++j) {
            const int units = s_ustart[j];
            s_ustart[j] = run;
            run += units;
        }
        if (threadIdx.x == 0) {
            s_misc[0] = n_jobs;
            s_misc[1] = all;
            s_misc[2] = unit_rows_b;
        }
    }
    __syncthreads();
    const int n_units = s_misc[1], unit_rows = s_misc[2];
    cg::cluster_group cluster = cg::this_cluster();
    const int csize = static_cast<int>(cluster.dim_blocks().y);  // CTAs per cluster: 1, 2 or 4
    const int cl = static_cast<int>(blockIdx.y) / csize;
    const int n_cl = static_cast<int>(gridDim.y) / csize;
    const unsigned int rank = cluster.block_rank();
    for (int u = cl; u < n_units; u += n_cl) {
        // unit -> job (binary search over the unit starts), feature group, row chunk
        int lo = 0, hi = n_jobs - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (s_ustart[mid] <= u) lo = mid;
            else hi = mid - 1;
        }
        const int j = lo;
        const int c = s_job[j] >> 16, e = s_job[j] & 0xffff;
        const WaveCtx& X = ctxs[c];
        const int n_f = X.gp.n_features;
        const int nfg = (n_f + kFG - 1) / kFG;
        const int k = u - s_ustart[j];
        const int fg = k % nfg, chunk = k / nfg;
        const JobRows jr = job_rows(X, src, e);
        const int R = jr.count;
        const int n_chunks = (R + unit_rows - 1) / unit_rows;
        const int crows = (R + n_chunks - 1) / n_chunks;
        const int c0 = min(R, chunk * crows), c1 = min(R, c0 + crows);
        const int qrows = (c1 - c0 + csize - 1) / csize;
        const int r0 = min(c1, c0 + static_cast<int>(rank) * qrows), r1 = min(c1, r0 + qrows);
        if (rows_counter != nullptr && rank == 0 && k == 0 && threadIdx.x == 0)
            atomicAdd(rows_counter, static_cast<unsigned long long>(R));
        const double hscale = X.st->hscale;
        // this CTA's rows of the unit -> its totals in the 5 planes of its shared memory
        accumulate_unit<kMode>(P, jr.rows, r0, r1, X.codes, X.gp.stride, fg * kFG, X.gq, X.hq,
                               static_cast<unsigned long long>(__double2ll_rn(1.0 * hscale)),
                               static_cast<unsigned long long>(__double2ll_rn(1.0 * X.goss_scale * hscale)));
        cluster.sync();
        const int share = kPlane / csize;
        const int fg0 = fg * kFG;
        const int nf_here = min(kFG, n_f - fg0);
        const size_t slot_off = static_cast<size_t>(jr.slot) * static_cast<size_t>(n_f) * kBins;
        for (int cell = rank * share + threadIdx.x; cell < static_cast<int>(rank + 1) * share; cell += kThreads) {
            unsigned long long g = 0, hsum = 0;
            unsigned int cn = 0;
            for (int kk = 0; kk < csize; ++kk) {
                const unsigned int* rt = cluster.map_shared_rank(P, kk);
                g += (static_cast<unsigned long long>(rt[kPlane + cell]) << 32) | rt[cell];
                hsum += (static_cast<unsigned long long>(rt[3 * kPlane + cell]) << 32) | rt[2 * kPlane + cell];
                cn += rt[4 * kPlane + cell];
            }
            const int b = cell >> 5, f = cell & 31;
            if (f >= nf_here || cn == 0u) continue;
            const size_t o = slot_off + static_cast<size_t>(fg0 + f) * kBins + b;
            atomicAdd(reinterpret_cast<unsigned long long*>(X.G) + o, g);
            atomicAdd(reinterpret_cast<unsigned long long*>(X.H) + o, hsum);
            atomicAdd(X.C + o, static_cast<int>(cn));
        }
        cluster.sync();  // no CTA reuses its planes while others read them
        {
            uint4* z = reinterpret_cast<uint4*>(smem_raw);
            for (int kk = threadIdx.x; kk < T::planes * kPlane / 4; kk += blockDim.x) z[kk] = make_uint4(0, 0, 0, 0);
        }
        __syncthreads();
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
    load_tile_prefix(ctxs, n_ctx, s_pref);
    const int total = s_pref[n_ctx];
    for (int t = blockIdx.x; t < total; t += gridDim.x) {
        const TileRef tr = find_tile(ctxs, s_pref, n_ctx, t);
        const WaveCtx& X = ctxs[tr.c];
        const int L = X.ctl->exp_leaf[tr.e];
        const DevNode& N = X.nodes[L];
        const DevSplit& S = X.splits[L];
        const int32_t* in = (N.buf ? X.rows1 : X.rows0) + N.start;
        const int base = tr.k * kPartTile, end = min(base + kPartTile, N.count);
        int32_t row[kPartPer];
        bool left[kPartPer];
        load_tile(X, in, S, base, end, row, left);
        int cnt = 0;
#pragma unroll
        for (int i = 0; i < kPartPer; ++i) cnt += left[i] ? 1 : 0;
        cnt = block_sum(cnt, red);
        if (threadIdx.x == 0) X.tile_counts[tr.lt] = cnt;
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
    __shared__ int red[kPartWarps];
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
        const DevSplit& S = X.splits[L];
        const int t0 = ctl->exp_tile0[tr.e], t1 = ctl->exp_tile0[tr.e + 1];
        int tot = 0, before = 0;
        for (int kk = t0 + threadIdx.x; kk < t1; kk += kPartThreads) {
            const int v = X.tile_counts[kk];
            tot += v;
            if (kk < tr.lt) before += v;
        }
        const int n_left = block_sum(tot, red);
        const int left0 = block_sum(before, red);
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
            if (left[i]) out[left0 + lrank] = row[i];
            else out[n_left + (base - left0) + (kk - base - lrank)] = row[i];
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
            static_cast<long long*>(gq)[r] = static_cast<long long>((static_cast<unsigned long long>(v) << 1) | (sc ? 1ull : 0ull));
        } else if constexpr (kMode == kHistExactVar) {
            static_cast<long long*>(gq)[r] = __double2ll_rn(gv * gscale);
            static_cast<long long*>(hq)[r] = __double2ll_rn(hv * hscale);
        } else if constexpr (kMode == kHistQ16Const) {
            const int qv = sround(gv * gscale, uniform01(seed, r, 0), -32767, 32767);
            static_cast<int*>(gq)[r] = static_cast<int>((static_cast<unsigned int>(qv) << 1) | (sc ? 1u : 0u));
        } else if constexpr (kMode == kHistQ16Var) {
            const int qg = sround(gv * gscale, uniform01(seed, r, 0), -32767, 32767);
            const int qh = sround(hv * hscale, uniform01(seed, r, 1), 0, 65535);
            static_cast<unsigned int*>(gq)[r] = (static_cast<unsigned int>(qg) << 16) | static_cast<unsigned int>(qh);
        } else if constexpr (kMode == kHistQ8Const) {
            const int qv = sround(gv * gscale, uniform01(seed, r, 0), -127, 127);
            static_cast<short*>(gq)[r] = static_cast<short>((qv * 2) | (sc ? 1 : 0));
        } else {
            const int qg = sround(gv * gscale, uniform01(seed, r, 0), -127, 127);
            const int qh = sround(hv * hscale, uniform01(seed, r, 1), 0, 255);
            static_cast<unsigned short*>(gq)[r] = static_cast<unsigned short>((qg + 128) | (qh << 8));
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
    static bool done[64] = {};
    int dev = 0;
    check(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev >= 0 && dev < 64 && done[dev]) return;
    set_smem(wave_hist_kernel<kMode>, kWaveSmem);
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
    cfg.dynamicSmemBytes = kWaveSmem;
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
    check(cudaLaunchKernelEx(&cfg, kern, ctxs, n_ctx, src, rows_counter, tune.units), "wave_hist launch");
}

template <int kMode>
void quantize_launch(const int32_t* rows, const double* g, const double* h, const uint8_t* flag, double gs,
                     const DevTreeState* st, unsigned long long seed, void* gq, void* hq, int blocks, cudaStream_t s) {
    wave_quantize_kernel<kMode><<<blocks, 256, 0, s>>>(rows, g, h, flag, gs, st, seed, gq, hq);
}

}  // namespace

int wave_hist_clusters(int cluster) {
    static int cached[64][5] = {};
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
    auto kern = wave_hist_kernel<kHistExactVar>;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(1, cluster * 64, 1);
    cfg.blockDim = dim3(kThreads, 1, 1);
    cfg.dynamicSmemBytes = kWaveSmem;
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
