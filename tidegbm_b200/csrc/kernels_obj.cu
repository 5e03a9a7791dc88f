// Gradients/hessians and training losses.
//
// MSE restates Objective::grad_hess (cpp/src/objective.cpp:105-118) with unit
// weights: g = pred - y, h = 1.
//
// RankPairwise restates objective.cpp:179-219.  Per date group of m rows (group_runs,
// objective.cpp:18-39): step = m > 48 ? max(1, m/24) : 1 and pairs (a, a + k*step).
// A row's partners are exactly the positions a -/+ k*step, so each thread owns one
// row and sums its own pair terms (gather, no atomics).  Visiting the partners in
// ascending position order reproduces the reference's accumulation order for that
// row (contributions as the later element of a pair arrive first, for smaller a),
// so g and h follow the same FP64 addition sequence; this file is compiled with
// -fmad=false to keep the statement-order rounding.
//
// Losses restate Objective::loss (objective.cpp:262-329): mean squared error, and
// for ranking the negative mean within-group Pearson correlation.
#include "tgb_internal.h"

namespace tgb {

namespace {

__global__ void grad_mse_kernel(const double* __restrict__ y, const double* __restrict__ pred, int n,
                                double* __restrict__ g, double* __restrict__ h) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        g[i] = 1.0 * (pred[i] - y[i]);
        h[i] = 1.0;
    }
}

// The MSE gradient fused with the all-row maxima the fit needs from it: g = pred - y
// (the unit hessian is implicit), max |g| and max h = 1 for the all-row fixed-point scale.
__global__ void grad_mse_fused_kernel(const double* __restrict__ y, const double* __restrict__ pred, int n,
                                      double* __restrict__ g, AllScale* __restrict__ sc) {
    double mg = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double gv = 1.0 * (pred[i] - y[i]);
        g[i] = gv;
        mg = fmax(mg, fabs(gv));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mg = fmax(mg, __shfl_xor_sync(0xffffffffu, mg, o));
    // Non-negative doubles order like their bit patterns.
    if ((threadIdx.x & 31) == 0) atomicMax(&sc->maxg_bits, static_cast<unsigned long long>(__double_as_longlong(mg)));
    if (blockIdx.x == 0 && threadIdx.x == 0)
        atomicMax(&sc->maxh_bits, static_cast<unsigned long long>(__double_as_longlong(1.0)));
}

__device__ __forceinline__ int row_at(const int* order, int p) { return order ? order[p] : p; }

__global__ void grad_pairwise_kernel(const double* __restrict__ y, const double* __restrict__ pred,
                                     const int* __restrict__ run_start, const int* __restrict__ run_len,
                                     const int* __restrict__ order, double* __restrict__ g,
                                     double* __restrict__ h) {
    const int r = blockIdx.x;
    const int s0 = run_start[r], m = run_len[r];
    for (int a = threadIdx.x; a < m; a += blockDim.x) {
        const int i = row_at(order, s0 + a);
        double ga = 0.0, ha = 1e-6;
        if (m >= 2) {
            const int step = m > 48 ? max(1, m / 24) : 1;
            const double yi = y[i], pi = pred[i];
            // Partners in ascending position: a%step, a%step+step, ..., a-step, then a+step, ...
            for (int p = a % step; p < m; p += step) {
                if (p == a) continue;
                const int j = row_at(order, s0 + p);
                const double yj = y[j];
                if (yi == yj) continue;
                const bool i_hi = yi > yj;
                const double phi = i_hi ? pi : pred[j];
                const double plo = i_hi ? pred[j] : pi;
                const double s = phi - plo;
                const double e = exp(fmin(fmax(1.0 * s, -30.0), 30.0));
                const double dyw = fmax(fabs(i_hi ? yi - yj : yj - yi), 1e-6);
                const double lam = -1.0 / (1.0 + e) * dyw;
                const double d2 = 1.0 * 1.0 * e / ((1 + e) * (1 + e)) * dyw;
                if (i_hi) ga += 1.0 * lam;
                else ga -= 1.0 * lam;
                ha += 1.0 * d2;
            }
        }
        g[i] = ga;
        h[i] = ha;
    }
}

__global__ void loss_mse_kernel(const double* __restrict__ y, const double* __restrict__ pred, int n,
                                double* __restrict__ partials) {
    double s = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const double d = pred[i] - y[i];
        s += 1.0 * d * d;
    }
    __shared__ double ws[32];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) t += ws[w];
        partials[blockIdx.x] = t;
    }
}

__global__ void loss_pairwise_kernel(const double* __restrict__ y, const double* __restrict__ pred,
                                     const int* __restrict__ run_start, const int* __restrict__ run_len,
                                     const int* __restrict__ order, double* __restrict__ corr,
                                     int* __restrict__ valid) {
    const int r = blockIdx.x;
    const int s0 = run_start[r], m = run_len[r];
    __shared__ double red[3][32];
    __shared__ double mean[2];
    double sy = 0, sp = 0;
    for (int k = threadIdx.x; k < m; k += blockDim.x) {
        const int i = row_at(order, s0 + k);
        sy += y[i];
        sp += pred[i];
    }
    for (int o = 16; o > 0; o >>= 1) {
        sy += __shfl_xor_sync(0xffffffffu, sy, o);
        sp += __shfl_xor_sync(0xffffffffu, sp, o);
    }
    const int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        red[0][w] = sy;
        red[1][w] = sp;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0, b = 0;
        for (int k = 0; k < nw; ++k) {
            a += red[0][k];
            b += red[1][k];
        }
        mean[0] = a / m;
        mean[1] = b / m;
    }
    __syncthreads();
    double vy = 0, vp = 0, c = 0;
    for (int k = threadIdx.x; k < m; k += blockDim.x) {
        const int i = row_at(order, s0 + k);
        const double dy = y[i] - mean[0], dp = pred[i] - mean[1];
        vy += dy * dy;
        vp += dp * dp;
        c += dy * dp;
    }
    for (int o = 16; o > 0; o >>= 1) {
        vy += __shfl_xor_sync(0xffffffffu, vy, o);
        vp += __shfl_xor_sync(0xffffffffu, vp, o);
        c += __shfl_xor_sync(0xffffffffu, c, o);
    }
    __syncthreads();
    if ((threadIdx.x & 31) == 0) {
        red[0][w] = vy;
        red[1][w] = vp;
        red[2][w] = c;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0, b = 0, cc = 0;
        for (int k = 0; k < nw; ++k) {
            a += red[0][k];
            b += red[1][k];
            cc += red[2][k];
        }
        const bool ok = m >= 3 && a > 1e-18 && b > 1e-18;
        corr[r] = ok ? cc / sqrt(a * b) : 0.0;
        valid[r] = ok ? 1 : 0;
    }
}

// kind 0: MSE = sum(partials) / n; kind 5: -mean(corr over valid runs).
__global__ void loss_finalize_kernel(int kind, const double* __restrict__ partials, const int* __restrict__ valid,
                                     int n_part, int n, double* __restrict__ out) {
    __shared__ double ws[32];
    __shared__ int wc[32];
    double s = 0.0;
    int c = 0;
    for (int k = threadIdx.x; k < n_part; k += blockDim.x) {
        if (kind == 5) {
            if (valid[k]) {
                s += partials[k];
                c += 1;
            }
        } else {
            s += partials[k];
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_xor_sync(0xffffffffu, s, o);
        c += __shfl_xor_sync(0xffffffffu, c, o);
    }
    if ((threadIdx.x & 31) == 0) {
        ws[threadIdx.x >> 5] = s;
        wc[threadIdx.x >> 5] = c;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        int tc = 0;
        for (int w = 0; w < static_cast<int>(blockDim.x >> 5); ++w) {
            t += ws[w];
            tc += wc[w];
        }
        if (kind == 5) *out = tc > 0 ? -t / tc : 0.0;
        else *out = n > 0 ? t / static_cast<double>(n) : 0.0;
    }
}

}  // namespace

void launch_loss_finalize(int kind, const double* partials, const int* valid, int n_part, int n, double* out,
                          cudaStream_t s) {
    loss_finalize_kernel<<<1, 1024, 0, s>>>(kind, partials, valid, n_part, n, out);
    check(cudaGetLastError(), "loss_finalize launch");
}

void launch_grad_mse(const double* y, const double* pred, int n, double* g, double* h, cudaStream_t s) {
    if (n <= 0) return;
    grad_mse_kernel<<<std::min(2368, (n + 255) / 256), 256, 0, s>>>(y, pred, n, g, h);
    check(cudaGetLastError(), "grad_mse launch");
}

void launch_grad_mse_fused(const double* y, const double* pred, int n, double* g, AllScale* sc, cudaStream_t s) {
    check(cudaMemsetAsync(sc, 0, 2 * sizeof(unsigned long long), s), "all scale reset");
    if (n <= 0) return;
    grad_mse_fused_kernel<<<std::min(2368, (n + 255) / 256), 256, 0, s>>>(y, pred, n, g, sc);
    check(cudaGetLastError(), "grad_mse_fused launch");
}

void launch_grad_pairwise(const double* y, const double* pred, const int* run_start, const int* run_len,
                          const int* order, int n_runs, int n, double* g, double* h, cudaStream_t s) {
    (void)n;
    if (n_runs <= 0) return;
    grad_pairwise_kernel<<<n_runs, 128, 0, s>>>(y, pred, run_start, run_len, order, g, h);
    check(cudaGetLastError(), "grad_pairwise launch");
}

void launch_loss_mse(const double* y, const double* pred, int n, double* partials, int n_part,
                     cudaStream_t s) {
    loss_mse_kernel<<<n_part, 256, 0, s>>>(y, pred, n, partials);
    check(cudaGetLastError(), "loss_mse launch");
}

void launch_loss_pairwise(const double* y, const double* pred, const int* run_start, const int* run_len,
                          const int* order, int n_runs, double* corr, int* valid, cudaStream_t s) {
    if (n_runs <= 0) return;
    loss_pairwise_kernel<<<n_runs, 128, 0, s>>>(y, pred, run_start, run_len, order, corr, valid);
    check(cudaGetLastError(), "loss_pairwise launch");
}

}  // namespace tgb
