// ref_tvd_shim.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Compiles the reference's own CPU restatement of the qGGMRF prior,
// cpuTotalVar in test/tvd.cpp:40-75 of lbl-camera/tomocam, straight from the
// read-only reference tree (see oracle/Makefile), and exposes it through a C
// entry point so the tests can pin the oracle's prior (oracle.qggmrf_grad)
// and the CUDA stencil against the reference's code.
//
// tomocam.h is skipped (its include guard is predefined) because it pulls in
// the NUFFT header, which needs cuFINUFFT, a library absent from this image.
// test/tvd.cpp's main() calls the reference's GPU drivers; that main is
// renamed and never called, and the two drivers get empty bodies below only
// so the shared object links.  Nothing here runs on a GPU.
#define TOMOCAM__H
#include "dist_array.h"

namespace tomocam {
    template <typename T>
    void add_total_var(DArray<T> &, DArray<T> &, float, float);
    template <typename T>
    void add_total_var2(DArray<T> &, DArray<T> &, T, T);
} // namespace tomocam

#define main reference_tvd_main
#include "tvd.cpp"
#undef main

namespace tomocam {
    template <typename T>
    void add_total_var(DArray<T> &, DArray<T> &, float, float) {}
    template <typename T>
    void add_total_var2(DArray<T> &, DArray<T> &, T, T) {}
    template void add_total_var<float>(DArray<float> &, DArray<float> &, float, float);
    template void add_total_var2<float>(DArray<float> &, DArray<float> &, float, float);
} // namespace tomocam

extern "C" {

// out = cpuTotalVar(in): the qGGMRF gradient alone, float32, [S][R][C].
int ref_cpu_total_var(const float *in, float *out, int S, int R, int C,
                      float sigma, float p) {
    if (S <= 0 || R <= 0 || C <= 0) return -1;
    tomocam::dim3_t dims(S, R, C);
    tomocam::DArray<float> a(dims);
    tomocam::DArray<float> b(dims);
    const size_t n = (size_t)S * R * C;
    for (size_t i = 0; i < n; ++i) a[i] = in[i];
    b.init(0.f);
    tomocam::cpuTotalVar(a, b, sigma, p);
    for (size_t i = 0; i < n; ++i) out[i] = b[i];
    return 0;
}

// The reference test's random stream (test/timer.h NPRandom, mt19937 seed 5489).
void ref_nprandom_fill(float *out, long n) {
    NPRandom rng;
    for (long i = 0; i < n; ++i) out[i] = rng.rand<float>();
}

} // extern "C"
