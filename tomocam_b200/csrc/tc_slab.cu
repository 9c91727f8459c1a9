// tc_slab.cu -- the MBIR solve of one slab of a volume split across ranks by
// slices: the reference's multi-GPU scheme (src/dist_array.h:349-373,
// src/multiproc.h:95-118, src/tv_update.cpp:82-96), where every slice is
// independent except for the 3-D prior.
//
// A slab owns S slices and keeps its iterates with one halo plane on each
// side ([S + 2][N][N]).  Per attempt the caller
//   1. fills the halo planes of the buffers the attempt reads (x and sol, or
//      the one buffer when they coincide): from the neighbouring slabs'
//      boundary planes, or, at an end of the volume, with a copy of the
//      slab's own edge plane, which reproduces the clamp-to-edge stencil;
//   2. runs the attempt (begin, the fused update over the owned planes with
//      the halos as neighbours, H new by the Toeplitz operator, the six FP64
//      sums of the step test over the owned planes);
//   3. sums the six values over all slabs (an all-reduce);
//   4. applies the step test of Optimizer::run2 (src/optimize.h:122-146) to
//      the global sums, identically on every slab.
// The exchange and the all-reduce are the caller's (tomocam_b200/slab.py:
// torch.distributed, or all slabs of one process in lockstep).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "tc_mbir.cuh"

namespace tc {

struct Slab {
    Plan *pl = nullptr;
    int S = 0, ST = 0, K = 0;
    size_t plane = 0, vol = 0;
    DevBuf ws;
    float *X = nullptr, *H = nullptr, *aty = nullptr;
    double *pu = nullptr, *pt = nullptr, *sums = nullptr, *hist = nullptr;
    MbirState *st = nullptr;
    int nu = 0, nt = 0;
    PriorParams pp{};
    MbirState host{};  // state after the last decide
};

__global__ void k_slab_begin(MbirState *s) { mbir_begin(s); }

__global__ void __launch_bounds__(UT, UPD_MIN_BLOCKS)
k_slab_update(float *__restrict__ X, const float *__restrict__ H, const float *__restrict__ aty,
              int ST, int N, size_t vol, PriorParams pp, const MbirState *__restrict__ st,
              double *__restrict__ partials) {
    double *part = partials + ((size_t)blockIdx.y * gridDim.x + blockIdx.x) * NU;
    const int c0 = blockIdx.x * UX, r0 = blockIdx.y * UY;
    if (st->ix == st->isol)
        update_body<true>(X, H, aty, ST, N, N, vol, pp, st, part, c0, r0, 1, ST - 1);
    else
        update_body<false>(X, H, aty, ST, N, N, vol, pp, st, part, c0, r0, 1, ST - 1);
}

// the six sums of the step test over this slab's owned planes
__global__ void k_slab_reduce(const double *__restrict__ pu, int nu, const double *__restrict__ pt,
                              int nt, double *__restrict__ sums) {
    double u[NU + 1] = {0, 0, 0, 0, 0, 0};
    for (int i = threadIdx.x; i < nu; i += blockDim.x)
#pragma unroll
        for (int k = 0; k < NU; ++k) u[k] += pu[(size_t)i * NU + k];
    for (int i = threadIdx.x; i < nt; i += blockDim.x) u[NU] += pt[(size_t)i * 2];
    block_sum<NU + 1>(u);
    if (threadIdx.x == 0)
        for (int k = 0; k <= NU; ++k) sums[k] = u[k];
}

__global__ void k_slab_decide(MbirState *s, const double *__restrict__ sums, double *hist) {
    double u[NU + 1];
    for (int k = 0; k <= NU; ++k) u[k] = sums[k];
    mbir_decide_core(s, u, hist);
}

static int slab_toeplitz(Slab &b, float *x, float *h, double *partials, const int *sel,
                         cudaStream_t st) {
    Plan &pl = *b.pl;
    const int chunk = 2 * pl.toe_pairs;
    int off = 0;
    for (int c0 = 0; c0 < b.S; c0 += chunk) {
        const int nb = std::min(chunk, b.S - c0);
        const size_t o = (size_t)(1 + c0) * b.plane;  // skip the lower halo plane
        TC_TRY(toeplitz_chunk(pl, x + o, nullptr, h + o, nb, partials ? partials + (size_t)off * 2 : nullptr,
                              st, sel, sel ? b.vol : 0));
        off += toeplitz_partials_count(pl, nb);
    }
    return TC_OK;
}

static int slab_create(Plan &pl, const float *aty, double sino_sq, const float *x0, int S,
                       const tc_mbir_opts &o, Slab &b, cudaStream_t st) {
    const int N = pl.N;
    b.pl = &pl;
    b.S = S;
    b.ST = S + 2;
    b.K = std::max(0, (int)o.num_iters);
    b.plane = (size_t)N * N;
    b.vol = (size_t)b.ST * b.plane;
    b.nu = ceil_div(N, UX) * ceil_div(N, UY);
    b.nt = 0;
    for (int c0 = 0; c0 < S; c0 += 2 * pl.toe_pairs)
        b.nt += toeplitz_partials_count(pl, std::min(2 * pl.toe_pairs, S - c0));
    b.pp = make_prior(o.sigma, o.p, o.prior_weight);
    TC_CUDA(cudaFuncSetAttribute(k_slab_update, cudaFuncAttributeMaxDynamicSharedMemorySize, UPD_SMEM));
    TC_CUDA(cudaFuncSetAttribute(k_slab_update, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 cudaSharedmemCarveoutMaxShared));
    // 3 iterates, 3 H-images, A^T y (all with halo planes), partials, sums,
    // history, state
    const size_t fl = (size_t)7 * b.vol * sizeof(float);
    const size_t db = ((size_t)b.nu * NU + (size_t)b.nt * 2 + 8 + 3 * (size_t)std::max(b.K, 1)) *
                      sizeof(double);
    TC_TRY(b.ws.reserve(fl + db + sizeof(MbirState) + 256));
    char *base = b.ws.as<char>();
    b.X = reinterpret_cast<float *>(base);
    b.H = b.X + 3 * b.vol;
    b.aty = b.H + 3 * b.vol;
    b.pu = reinterpret_cast<double *>(base + fl);
    b.pt = b.pu + (size_t)b.nu * NU;
    b.sums = b.pt + (size_t)b.nt * 2;
    b.hist = b.sums + 8;
    b.st = reinterpret_cast<MbirState *>(base + ((fl + db + 255) / 256) * 256);
    // A^T y and x0 into the owned planes; the halo planes of A^T y are never
    // summed, zero them so that nothing reads undefined values
    TC_CUDA(cudaMemsetAsync(b.aty, 0, b.vol * sizeof(float), st));
    TC_CUDA(cudaMemcpyAsync(b.aty + b.plane, aty, (size_t)S * b.plane * sizeof(float),
                            cudaMemcpyDeviceToDevice, st));
    TC_CUDA(cudaMemsetAsync(b.X, 0, b.vol * sizeof(float), st));
    TC_CUDA(cudaMemcpyAsync(b.X + b.plane, x0, (size_t)S * b.plane * sizeof(float),
                            cudaMemcpyDeviceToDevice, st));
    MbirState h{};
    h.t = 1.0;
    h.tnew = 1.0;
    double step = o.step > 0 ? (double)o.step : 1.0 / pl.lipschitz;
    if (!(o.step > 0) && step > 1.0) step = 1.0;
    h.step = h.step0 = step;
    h.sino_sq = sino_sq;
    h.ix = h.isol = 0;
    h.inew = 1;
    h.num_iters = b.K;
    h.max_attempts = o.max_attempts > 0 ? o.max_attempts : 1000;
    h.cond = b.K > 0 ? 1 : 0;
    b.host = h;
    TC_CUDA(cudaMemcpyAsync(b.st, &h, sizeof(h), cudaMemcpyHostToDevice, st));
    // H x0 over the owned planes
    TC_TRY(slab_toeplitz(b, b.X, b.H, nullptr, nullptr, st));
    TC_CUDA(cudaStreamSynchronize(st));
    return TC_OK;
}

static int slab_attempt(Slab &b, cudaStream_t st) {
    const int N = b.pl->N;
    k_slab_begin<<<1, 1, 0, st>>>(b.st);
    TC_LAUNCH_CHECK();
    dim3 grid(ceil_div(N, UX), ceil_div(N, UY));
    k_slab_update<<<grid, UT, UPD_SMEM, st>>>(b.X, b.H, b.aty, b.ST, N, b.vol, b.pp, b.st, b.pu);
    TC_LAUNCH_CHECK();
    TC_TRY(slab_toeplitz(b, b.X, b.H, b.pt, &b.st->inew, st));
    k_slab_reduce<<<1, 1024, 0, st>>>(b.pu, b.nu, b.pt, b.nt, b.sums);
    TC_LAUNCH_CHECK();
    return TC_OK;
}

static int slab_decide(Slab &b, int *cond, cudaStream_t st) {
    k_slab_decide<<<1, 1, 0, st>>>(b.st, b.sums, b.hist);
    TC_LAUNCH_CHECK();
    TC_CUDA(cudaMemcpyAsync(&b.host, b.st, sizeof(MbirState), cudaMemcpyDeviceToHost, st));
    TC_CUDA(cudaStreamSynchronize(st));
    *cond = b.host.cond;
    return TC_OK;
}

}  // namespace tc

struct tc_slab {
    tc::Slab impl;
};

using tc::Slab;

namespace {
template <typename F>
int slab_guarded(F &&f) {
    try {
        return f();
    } catch (const std::bad_alloc &) {
        tc::set_error("host allocation failed");
        return TC_ERR_ALLOC;
    } catch (const std::exception &e) {
        tc::set_error(std::string("internal error: ") + e.what());
        return TC_ERR_STATE;
    }
}
cudaStream_t stream_of(tc_stream_t s) { return reinterpret_cast<cudaStream_t>(s); }
}  // namespace

extern "C" {

int tc_slab_create(tc_plan *plan, const float *aty, double sino_sq, const float *x0, int nslices,
                   const tc_mbir_opts *opts, tc_slab **out, tc_stream_t stream) {
    return slab_guarded([&]() -> int {
        if (!plan || !aty || !x0 || !opts || !out) TC_FAIL(TC_ERR_ARG, "NULL argument to tc_slab_create");
        *out = nullptr;
        if (nslices < 1 || nslices > 65533) TC_FAIL(TC_ERR_SHAPE, "nslices must be in [1, 65533]");
        if (!std::isfinite(sino_sq)) TC_FAIL(TC_ERR_NAN, "sino_sq is not finite");
        // the same checks as tc_mbir_solve
        if (opts->num_iters < 0) TC_FAIL(TC_ERR_ARG, "num_iters < 0");
        if (!(opts->sigma > 0) || !std::isfinite(opts->sigma)) TC_FAIL(TC_ERR_ARG, "sigma must be > 0");
        if (!(opts->p > 0 && opts->p <= 2)) TC_FAIL(TC_ERR_ARG, "p must be in (0, 2]");
        if (!std::isfinite(opts->prior_weight)) TC_FAIL(TC_ERR_ARG, "prior_weight must be finite");
        if (!plan->impl.d_phat.ptr)
            TC_FAIL(TC_ERR_STATE, "plan has no point-spread function (created with TC_PLAN_NO_PSF)");
        tc_slab *s = new tc_slab;
        const int rc = tc::slab_create(plan->impl, aty, sino_sq, x0, nslices, *opts, s->impl,
                                       stream_of(stream));
        if (rc != TC_OK) {
            delete s;
            return rc;
        }
        *out = s;
        return TC_OK;
    });
}

int tc_slab_halo(tc_slab *s, int which, float **send_lo, float **send_hi, float **recv_lo,
                 float **recv_hi, int *same) {
    return slab_guarded([&]() -> int {
        if (!s || !send_lo || !send_hi || !recv_lo || !recv_hi || !same)
            TC_FAIL(TC_ERR_ARG, "NULL argument to tc_slab_halo");
        if (which != 0 && which != 1) TC_FAIL(TC_ERR_ARG, "which must be 0 (x) or 1 (sol)");
        Slab &b = s->impl;
        const int buf = which == 0 ? b.host.ix : b.host.isol;
        float *X = b.X + (size_t)buf * b.vol;
        *recv_lo = X;
        *send_lo = X + b.plane;
        *send_hi = X + (size_t)b.S * b.plane;
        *recv_hi = X + (size_t)(b.S + 1) * b.plane;
        *same = b.host.ix == b.host.isol;
        return TC_OK;
    });
}

int tc_slab_attempt(tc_slab *s, double **sums, tc_stream_t stream) {
    return slab_guarded([&]() -> int {
        if (!s || !sums) TC_FAIL(TC_ERR_ARG, "NULL argument to tc_slab_attempt");
        if (!s->impl.host.cond) TC_FAIL(TC_ERR_STATE, "the slab solve has finished");
        TC_TRY(tc::slab_attempt(s->impl, stream_of(stream)));
        *sums = s->impl.sums;
        return TC_OK;
    });
}

int tc_slab_decide(tc_slab *s, int *cond, tc_stream_t stream) {
    return slab_guarded([&]() -> int {
        if (!s || !cond) TC_FAIL(TC_ERR_ARG, "NULL argument to tc_slab_decide");
        return tc::slab_decide(s->impl, cond, stream_of(stream));
    });
}

int tc_slab_result(tc_slab *s, float *x, double *history, int *iters, tc_stream_t stream) {
    return slab_guarded([&]() -> int {
        if (!s || !x) TC_FAIL(TC_ERR_ARG, "NULL argument to tc_slab_result");
        Slab &b = s->impl;
        cudaStream_t st = stream_of(stream);
        TC_CUDA(cudaMemcpyAsync(x, b.X + (size_t)b.host.ix * b.vol + b.plane,
                                (size_t)b.S * b.plane * sizeof(float), cudaMemcpyDeviceToDevice, st));
        if (history && b.K > 0)
            TC_CUDA(cudaMemcpyAsync(history, b.hist, 3 * (size_t)b.K * sizeof(double),
                                    cudaMemcpyDeviceToHost, st));
        TC_CUDA(cudaStreamSynchronize(st));
        if (iters) *iters = b.host.iter;
        if (b.host.status == 1)
            TC_FAIL(TC_ERR_TIMEOUT, "backtracking found no acceptable step within max_attempts "
                                    "attempts at iteration " + std::to_string(b.host.iter));
        return TC_OK;
    });
}

int tc_slab_destroy(tc_slab *s) {
    delete s;
    return TC_OK;
}

}  // extern "C"
