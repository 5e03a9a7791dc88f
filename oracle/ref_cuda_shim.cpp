// C-ABI shim over the reference's only GPU code, build_hist_gpu
// (cpp/src/histogram_cuda.cu:81-167), compiled for sm_100a from the
// reference's own source by oracle/Makefile into oracle/_ref/libtgbref_cuda.so.
//
// TEST AND MEASUREMENT INFRASTRUCTURE ONLY: bench.py times it as the "plain GPU"
// histogram path the north-star metric compares against.  Nothing in the
// product loads it.
#include "tidegbm/histogram.hpp"

#include <string>

using namespace tidegbm;

namespace {
thread_local std::string g_err;
}

extern "C" {

const char* refgpu_last_error(void) { return g_err.c_str(); }

// Same arguments as build_hist_gpu; out is interleaved {g, h, c(as f64)}.
int refgpu_build_hist(const unsigned short* xb, int n_f, const int* idx, int n_idx,
                      const double* g, const double* h, int n_bins, int n_rows, double* out) {
    try {
        Hist hist;
        hist.resize(n_f, n_bins);
        build_hist_gpu(xb, n_f, idx, n_idx, g, h, hist, n_rows);
        for (size_t i = 0; i < hist.B.size(); ++i) {
            out[3 * i] = hist.B[i].g;
            out[3 * i + 1] = hist.B[i].h;
            out[3 * i + 2] = static_cast<double>(hist.B[i].c);
        }
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

}  // extern "C"
