// ref_run2_shim.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Compiles the reference's own solver, Optimizer::run2 in src/optimize.h:96-154
// of lbl-camera/tomocam, straight from the read-only reference tree (see
// oracle/Makefile), over the reference's host array DArray<double>
// (src/dist_array.h), and exposes it through a C entry point.  The gradient
// and objective are callbacks, so the tests drive the reference's control
// flow (momentum, backtracking, step reset, acceptance test) with the FP64
// oracle's gradient2 + qGGMRF and sqrt(function_value2), exactly as
// src/mbir2.cpp:114-137 wires them, and pin the oracle's restatement
// (oracle.run2) to the reference's iterates and attempt counts.
//
// tomocam.h is skipped (its include guard is predefined): its NUFFT header
// needs cuFINUFFT, absent from this image, and run2 uses nothing from it.
// Nothing here touches a GPU.
#define TOMOCAM__H
#include "dist_array.h"
#include "machine.h"
#include "optimize.h"

#include <cstdint>

extern "C" {

// g[0:n] = gradient(y[0:n]); returns nothing.
typedef void (*ref_grad_fn)(const double *y, double *g, int64_t n);
// returns the objective's square root at x[0:n].
typedef double (*ref_err_fn)(const double *x, int64_t n);

// sol[S][R][C] (in: initial guess, out: result) = run2(sol, iters, step, ...).
// Returns 0, or -1 on bad sizes.  run2 prints one line per iteration to
// stdout, as the reference does.
int ref_run2(double *sol, int S, int R, int C, int num_iters, double step_size,
             ref_grad_fn grad, ref_err_fn err) {
    if (S <= 0 || R <= 0 || C <= 0 || num_iters < 0 || !grad || !err) return -1;
    tomocam::dim3_t dims(S, R, C);
    const int64_t n = (int64_t)S * R * C;
    tomocam::DArray<double> x0(dims);
    for (int64_t i = 0; i < n; ++i) x0[i] = sol[i];

    auto calc_gradient = [grad, dims, n](tomocam::DArray<double> &y) {
        tomocam::DArray<double> g(dims);
        grad(&y[0], &g[0], n);
        return g;
    };
    auto calc_error = [err, n](tomocam::DArray<double> &x) -> double {
        return err(&x[0], n);
    };
    tomocam::Optimizer<double, tomocam::DArray, decltype(calc_gradient),
                       decltype(calc_error)>
        opt(calc_gradient, calc_error);
    auto rec = opt.run2(x0, num_iters, step_size, 0.0, 0.0);
    for (int64_t i = 0; i < n; ++i) sol[i] = rec[i];
    return 0;
}

} // extern "C"
