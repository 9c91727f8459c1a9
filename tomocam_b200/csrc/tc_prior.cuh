// tc_prior.cuh -- qGGMRF prior: potential derivative and the 26-neighbour
// stencil weights (src/gpu/potential_function.cuh:31-108).
#pragma once

#include <cmath>

#include "tc_common.cuh"

namespace tc {

// q = 2, c = 0.001 as in the reference (MRF_Q, MRF_C)
constexpr float MRF_C = 0.001f;

// 3x3x3 weights [dz][dy][dx], centre 0 (src/gpu/potential_function.cuh:38-51)
static __constant__ float c_qggmrf_w[27] = {
    0.0302f, 0.0370f, 0.0302f, 0.0370f, 0.0523f, 0.0370f, 0.0302f, 0.0370f, 0.0302f,
    0.0370f, 0.0523f, 0.0370f, 0.0523f, 0.0000f, 0.0523f, 0.0370f, 0.0523f, 0.0370f,
    0.0302f, 0.0370f, 0.0302f, 0.0370f, 0.0523f, 0.0370f, 0.0302f, 0.0370f, 0.0302f};

// parameters of rho'(delta) precomputed on the host
struct PriorParams {
    float inv_sigma;  // 1 / sigma
    float qmp;        // q - p
    float inv_sq;     // 1 / sigma^q
    float scale;      // weight of the prior gradient
    float l2s;        // (q - p) log2(1 / sigma)
    float p;          // q - (q - p)
    float qmpc;       // (q - p) c
};

inline PriorParams make_prior(float sigma, float p, float scale) {
    PriorParams pp;
    pp.inv_sigma = 1.0f / sigma;
    // q - p > 0 keeps q-p times log2(0) = -inf at delta = 0 (t = 0); p = 2
    // uses a tiny positive exponent, which gives t = 1 for every delta != 0
    pp.qmp = 2.0f - p > 1e-30f ? 2.0f - p : 1e-30f;
    pp.inv_sq = 1.0f / (sigma * sigma);
    pp.scale = scale;
    pp.l2s = (float)((double)pp.qmp * std::log2(1.0 / (double)sigma));
    pp.p = 2.0f - pp.qmp;
    pp.qmpc = pp.qmp * MRF_C;
    return pp;
}

// PTX approximate transcendental instructions (the SFU): log2, 2^x, 1/x
__device__ __forceinline__ float lg2_approx(float x) {
    float y;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float ex2_approx(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float rcp_approx(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// 1/x on the FMA pipe instead of the SFU, for finite x >= 2^-125 (larger x
// are clamped to 2^126, giving about 1e-38 where the exact value is
// smaller).  First estimate from the bits: 0x7ef311c2 minus the bit pattern
// of x, the constant that minimises the worst relative error over a binade
// (5.1 %, found by a search over the constant); then Newton-Raphson
// refinement of f(y) = 1/y - x with e = 1 - x y: one third-order step
// y (1 + e + e^2) (error e^3 <= 1.3e-4) and one second-order step y (1 + e)
// (error below 2e-8 before rounding).  One integer and five FMA-pipe
// instructions plus the clamp; within 0.78 ulp of 1/x for x up to 1e37
// (a search over 4 million x on [1e-3, 1e37] against FP64).
__device__ __forceinline__ float rcp_fma(float x) {
    x = fminf(x, 0x1p126f);
    float y = __int_as_float(0x7ef311c2 - __float_as_int(x));
    float e = fmaf(-x, y, 1.0f);
    y = fmaf(y, fmaf(e, e, e), y);
    e = fmaf(-x, y, 1.0f);
    return fmaf(y, e, y);
}

// 2^x on the FMA pipe instead of the SFU, for x in [-125, 127] (clamped):
// x = k + f with k = rint(x) formed by adding and subtracting 1.5 * 2^23
// (the integer lands in the low mantissa bits), f in [-0.5, 0.5]; 2^f from
// a degree-6 polynomial fitted here (weighted least squares on Chebyshev
// nodes, reweighted towards equal relative error: 1.9e-9 in exact
// arithmetic, 8e-8 evaluated in FP32), and 2^k added to the exponent field.
__device__ __forceinline__ float ex2_fma(float x) {
    x = fminf(fmaxf(x, -125.f), 127.f);
    const float r = x + 12582912.f;  // 1.5 * 2^23, bits 0x4B400000
    const float f = x - (r - 12582912.f);
    float p = 1.5350866e-4f;
    p = fmaf(p, f, 1.3399974e-3f);
    p = fmaf(p, f, 9.6184704e-3f);
    p = fmaf(p, f, 5.5503286e-2f);
    p = fmaf(p, f, 2.4022648e-1f);
    p = fmaf(p, f, 6.9314718e-1f);
    p = fmaf(p, f, 1.0f);
    const int k = __float_as_int(r) - 0x4B400000;
    return __int_as_float(__float_as_int(p) + (k << 23));
}

// rho'(delta) = sgn(delta) |delta| (q - (q-p) t / (c + t)) / (sigma^q (c + t)),
// t = (|delta| / sigma)^(q-p), q = 2; rho'(0) = 0.  Rearranged without the
// sign branch: rho'(delta) = delta (q c + p t) / (sigma^q (c + t)^2), and with
// r = 1 / (c + t) and t r = 1 - c r:  delta r (p + (q-p) c r) / sigma^q.
// t = 2^((q-p) log2|delta| + (q-p) log2(1/sigma)) on the SFU (a few 1e-7
// relative); at delta = 0 the log is -inf and, with q - p > 0 (make_prior),
// t = 0 and the result 0.  The 1/sigma^q factor is left to the caller
// (d_pot_unscaled), which folds it into the stencil weights.  FMA_RCP forms
// r on the FMA pipe (rcp_fma), for kernels whose SFU is the busier unit.
template <bool FMA_RCP = false, bool FMA_EX2 = false>
__device__ __forceinline__ float d_pot_unscaled(float delta, const PriorParams &pp) {
    const float l = lg2_approx(fabsf(delta));
    const float t = FMA_EX2 ? ex2_fma(fmaf(pp.qmp, l, pp.l2s)) : ex2_approx(fmaf(pp.qmp, l, pp.l2s));
    const float r = FMA_RCP ? rcp_fma(MRF_C + t) : rcp_approx(MRF_C + t);
    return delta * (r * fmaf(pp.qmpc, r, pp.p));
}

__device__ __forceinline__ float d_pot(float delta, const PriorParams &pp) {
    return pp.inv_sq * d_pot_unscaled(delta, pp);
}

}  // namespace tc
