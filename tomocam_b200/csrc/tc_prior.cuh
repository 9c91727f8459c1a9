// tc_prior.cuh -- qGGMRF prior: potential derivative and the 26-neighbour
// stencil weights (src/gpu/potential_function.cuh:31-108).
#pragma once

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
};

inline PriorParams make_prior(float sigma, float p, float scale) {
    PriorParams pp;
    pp.inv_sigma = 1.0f / sigma;
    pp.qmp = 2.0f - p;
    pp.inv_sq = 1.0f / (sigma * sigma);
    pp.scale = scale;
    return pp;
}

// rho'(delta) = sgn(delta) |delta| (q - (q-p) t / (c + t)) / (sigma^q (c + t)),
// t = (|delta| / sigma)^(q-p), q = 2; rho'(0) = 0.
__device__ __forceinline__ float d_pot(float delta, const PriorParams &pp) {
    const float ad = fabsf(delta);
    if (ad == 0.0f) return 0.0f;
    const float t = powf(ad * pp.inv_sigma, pp.qmp);
    const float den = MRF_C + t;
    const float v = ad * pp.inv_sq / den * (2.0f - pp.qmp * t / den);
    return delta > 0.0f ? v : -v;
}

}  // namespace tc
