// tc_mbir.cuh -- the MBIR attempt's device pieces shared by the
// single-volume solver (tc_mbir.cu) and the batched solver (tc_batch.cu):
// the iteration state, the fused stencil + Nesterov update body and the step
// test of Optimizer::run2 (src/optimize.h:96-154).
#pragma once

#include <type_traits>

#include "tc_plan.cuh"
#include "tc_prior.cuh"

namespace tc {

struct MbirState {
    double t, tnew, beta, step, step0, sino_sq;
    float betaf, stepf;
    int ix, isol, inew;        // buffer indices of x, sol, new iterate
    int iter, num_iters;       // accepted iterations so far / requested
    int attempts, attempts_iter, max_attempts;
    int cond;                  // 1 while more attempts are needed
    int status;                // 0 ok, 1 backtracking cap reached, 3 a bounded device wait gave up
};

// beta and theta for the next attempt (src/optimize.h:117-121)
__device__ __forceinline__ void mbir_begin(MbirState *s) {
    const double t = s->t;
    s->beta = s->tnew * (1.0 / t - 1.0);
    s->tnew = 0.5 * (sqrt(t * t * t * t + 4.0 * t * t) - t * t);
    s->betaf = (float)s->beta;
    s->stepf = (float)s->step;
}

}  // namespace tc

// the fused stencil + Nesterov update (update_body) and its tile constants
#include "tc_update.cuh"

namespace tc {

// The step test and bookkeeping of one attempt from its reduced sums
// u = {y.Hy, y.A^Ty, g.g, new.A^Ty, |new - x|^2, new.H new}; returns 1 while
// more attempts are needed (src/optimize.h:122-146).
__device__ __forceinline__ int mbir_decide_core(MbirState *s, const double *u, double *hist) {
    if (s->status != 0) {  // a kernel of this attempt gave up waiting: stop
        s->cond = 0;
        return 0;
    }
    const double yhy = u[0], yaty = u[1], gg = u[2], naty = u[3], dx2 = u[4], nhn = u[5];
    // objective sqrt(v.Hv - 2 v.A^T y + |y|^2)  (src/error2.cpp:60-63, src/mbir2.cpp:130-136)
    const double fy = sqrt(yhy - 2.0 * yaty + s->sino_sq);
    const double fx = sqrt(nhn - 2.0 * naty + s->sino_sq);
    const double gy = 0.5 * s->step * gg;
    s->attempts += 1;
    s->attempts_iter += 1;
    int cond = 1;
    if (fx > fy + gy) {
        // rejected: shrink the step, keep x, retry from the new iterate
        s->step *= 0.9;
        s->isol = s->inew;
        int f = 0;
        while (f == s->ix || f == s->isol) ++f;
        s->inew = f;
        if (s->attempts_iter >= s->max_attempts) {
            s->status = 1;
            cond = 0;
        }
    } else {
        s->step = s->step0;
        s->t = s->tnew;
        if (hist) {
            hist[3 * s->iter + 0] = fx;
            hist[3 * s->iter + 1] = sqrt(dx2);
            hist[3 * s->iter + 2] = (double)s->attempts_iter;
        }
        s->ix = s->inew;
        s->isol = s->inew;
        s->inew = (s->inew + 1) % 3;
        s->iter += 1;
        s->attempts_iter = 0;
        cond = s->iter < s->num_iters ? 1 : 0;
    }
    s->cond = cond;
    return cond;
}

}  // namespace tc
