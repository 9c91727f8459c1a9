// tc_prior_diff.cu -- derivatives of the qGGMRF prior beyond its gradient,
// for differentiating the MBIR objective and unrolled reconstructions.
//
// The prior potential whose gradient is the reference's clamped 26-neighbour
// stencil (src/gpu/cuTV2.cu:33-76 with the clamp of
// src/gpu/dev_memory.cuh:88-94) is
//   U(x) = 1/2 sum_v sum_{26 d} w_d rho(x_v - x_c(v+d)),
//   rho(delta) = u^2 / (c + u^(2-p)),  u = |delta| / sigma   (q = 2),
// with rho'(delta) = delta A(t) / sigma^2, t = u^(2-p),
//   A(t) = (2c + p t) / (c + t)^2,  A'(t) = ((p - 4) c - p t) / (c + t)^3,
//   rho''(delta) = (A + (2 - p) t A') / sigma^2   (finite at delta = 0),
// and the sigma derivatives
//   d rho / d sigma  = -delta rho'(delta) / sigma,
//   d rho' / d sigma = -(delta rho''(delta) + rho'(delta)) / sigma.
// Nothing here has a counterpart in the reference, which only evaluates the
// gradient.
#include "tc_plan.cuh"
#include "tc_prior.cuh"

namespace tc {

constexpr int DX = 32, DY = 8;
constexpr int DN = 3 * (DY + 2) * (DX + 2);

struct PriorTerms {
    float rho, d1, d2;  // rho, rho', rho'' (with the 1/sigma^2 factors)
};

__device__ __forceinline__ PriorTerms prior_terms(float delta, float inv_sigma, float inv_sq,
                                                  float qmp, float p) {
    const float l = fmaxf(lg2_approx(fabsf(delta) * inv_sigma), -200.0f);
    const float t = ex2_approx(qmp * l);
    const float r = rcp_approx(MRF_C + t);
    const float A = (2.0f * MRF_C + p * t) * (r * r);
    const float Ap = ((p - 4.0f) * MRF_C - p * t) * (r * r * r);
    PriorTerms o;
    o.rho = delta * delta * inv_sq * r;
    o.d1 = delta * A * inv_sq;
    o.d2 = (A + qmp * t * Ap) * inv_sq;
    return o;
}

// the clamped 3 x 10 x 34 neighbourhood of the CTA's 32 x 8 patch of slice s
__device__ __forceinline__ void load_nbhd(float *tile, const float *__restrict__ a, int s, int S,
                                          int R, int C, int r0, int c0) {
    const size_t plane = (size_t)R * C;
    for (int i = threadIdx.y * DX + threadIdx.x; i < DN; i += DX * DY) {
        const int dz = i / ((DY + 2) * (DX + 2));
        const int rem = i - dz * (DY + 2) * (DX + 2);
        const int dy = rem / (DX + 2), dx = rem - dy * (DX + 2);
        const int ss = min(max(s + dz - 1, 0), S - 1);
        const int rr = min(max(r0 + dy - 1, 0), R - 1);
        const int cc = min(max(c0 + dx - 1, 0), C - 1);
        tile[i] = a[ss * plane + (size_t)rr * C + cc];
    }
}

__device__ __forceinline__ int nb_index(int dz, int dy, int dx) {
    return (dz * (DY + 2) + threadIdx.y + dy) * (DX + 2) + threadIdx.x + dx;
}

// partials[cta] = {1/2 sum w rho, 1/2 sum w d rho / d sigma}
__global__ void k_qggmrf_value(const float *__restrict__ x, int S, int R, int C, float inv_sigma,
                               float inv_sq, float qmp, float p, double *__restrict__ partials) {
    __shared__ float tile[DN];
    const int c0 = blockIdx.x * DX, r0 = blockIdx.y * DY, s = blockIdx.z;
    load_nbhd(tile, x, s, S, R, C, r0, c0);
    __syncthreads();
    const int c = c0 + threadIdx.x, r = r0 + threadIdx.y;
    double acc[2] = {0.0, 0.0};
    if (c < C && r < R) {
        const float u = tile[nb_index(1, 1, 1)];
        float a0 = 0.0f, a1 = 0.0f;
#pragma unroll
        for (int dz = 0; dz < 3; ++dz)
#pragma unroll
            for (int dy = 0; dy < 3; ++dy)
#pragma unroll
                for (int dx = 0; dx < 3; ++dx) {
                    if (dz == 1 && dy == 1 && dx == 1) continue;
                    const float w = c_qggmrf_w[(dz * 3 + dy) * 3 + dx];
                    const float d = u - tile[nb_index(dz, dy, dx)];
                    const PriorTerms pt = prior_terms(d, inv_sigma, inv_sq, qmp, p);
                    a0 = fmaf(w, pt.rho, a0);
                    a1 = fmaf(w, d * pt.d1, a1);
                }
        acc[0] = 0.5 * (double)a0;
        acc[1] = -0.5 * (double)a1 * (double)inv_sigma;
    }
    block_sum<2>(acc, threadIdx.y * DX + threadIdx.x, DX * DY);
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        double *dst = partials + (((size_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x) * 2;
        dst[0] = acc[0];
        dst[1] = acc[1];
    }
}

// hv[u] = scale * sum_d w rho''(x_u - x_n) (v_u - v_n)   (if hv)
// partials[cta] = {sum_u v_u sum_d w rho'(delta),
//                  sum_u v_u sum_d w d rho'(delta) / d sigma}
__global__ void k_qggmrf_hvp(const float *__restrict__ x, const float *__restrict__ v,
                             float *__restrict__ hv, int S, int R, int C, float inv_sigma,
                             float inv_sq, float qmp, float p, float scale,
                             double *__restrict__ partials) {
    __shared__ float tx[DN], tv[DN];
    const int c0 = blockIdx.x * DX, r0 = blockIdx.y * DY, s = blockIdx.z;
    load_nbhd(tx, x, s, S, R, C, r0, c0);
    load_nbhd(tv, v, s, S, R, C, r0, c0);
    __syncthreads();
    const int c = c0 + threadIdx.x, r = r0 + threadIdx.y;
    double acc[2] = {0.0, 0.0};
    if (c < C && r < R) {
        const int o = nb_index(1, 1, 1);
        const float u = tx[o], vu = tv[o];
        float h = 0.0f, g1 = 0.0f, gs = 0.0f;
#pragma unroll
        for (int dz = 0; dz < 3; ++dz)
#pragma unroll
            for (int dy = 0; dy < 3; ++dy)
#pragma unroll
                for (int dx = 0; dx < 3; ++dx) {
                    if (dz == 1 && dy == 1 && dx == 1) continue;
                    const float w = c_qggmrf_w[(dz * 3 + dy) * 3 + dx];
                    const int n = nb_index(dz, dy, dx);
                    const float d = u - tx[n];
                    const PriorTerms pt = prior_terms(d, inv_sigma, inv_sq, qmp, p);
                    h = fmaf(w * pt.d2, vu - tv[n], h);
                    g1 = fmaf(w, pt.d1, g1);
                    gs = fmaf(w, fmaf(d, pt.d2, pt.d1), gs);
                }
        if (hv) hv[s * (size_t)R * C + (size_t)r * C + c] = scale * h;
        acc[0] = (double)vu * (double)g1;
        acc[1] = -(double)vu * (double)gs * (double)inv_sigma;
    }
    if (partials) {
        block_sum<2>(acc, threadIdx.y * DX + threadIdx.x, DX * DY);
        if (threadIdx.x == 0 && threadIdx.y == 0) {
            double *dst = partials + (((size_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x) * 2;
            dst[0] = acc[0];
            dst[1] = acc[1];
        }
    }
}

static int prior_args(int S, int R, int C, float sigma, float p) {
    if (S < 0 || R < 0 || C < 0) TC_FAIL(TC_ERR_SHAPE, "negative size");
    if (S > 65535) TC_FAIL(TC_ERR_SHAPE, "too many slices for one prior launch");
    if (!(sigma > 0) || !std::isfinite(sigma)) TC_FAIL(TC_ERR_ARG, "sigma must be > 0");
    if (!(p > 0 && p <= 2)) TC_FAIL(TC_ERR_ARG, "p must be in (0, 2]");
    return TC_OK;
}

// sum the per-CTA pairs on the device and copy the two totals to the host
static int finish_dots(double *parts, int nparts, double *a, double *b, cudaStream_t st) {
    double h[2] = {0.0, 0.0};
    TC_TRY(reduce_partials(parts, nparts, 2, parts + (size_t)nparts * 2, st));
    TC_CUDA(cudaMemcpyAsync(h, parts + (size_t)nparts * 2, 2 * sizeof(double),
                            cudaMemcpyDeviceToHost, st));
    TC_CUDA(cudaStreamSynchronize(st));
    if (a) *a = h[0];
    if (b) *b = h[1];
    return TC_OK;
}

int qggmrf_value_launch(const float *x, int S, int R, int C, float sigma, float p, double *value,
                        double *dsigma, cudaStream_t st) {
    TC_TRY(prior_args(S, R, C, sigma, p));
    if ((size_t)S * R * C == 0) {
        if (value) *value = 0.0;
        if (dsigma) *dsigma = 0.0;
        return TC_OK;
    }
    const dim3 grid(ceil_div(C, DX), ceil_div(R, DY), S);
    const int nparts = (int)(grid.x * grid.y * grid.z);
    double *parts = nullptr;
    TC_CUDA(cudaMallocAsync(&parts, ((size_t)nparts * 2 + 2) * sizeof(double), st));
    const PriorParams pp = make_prior(sigma, p, 1.0f);
    k_qggmrf_value<<<grid, dim3(DX, DY), 0, st>>>(x, S, R, C, pp.inv_sigma, pp.inv_sq, pp.qmp, p,
                                                  parts);
    cudaError_t e = cudaGetLastError();
    int rc = e == cudaSuccess ? finish_dots(parts, nparts, value, dsigma, st) : TC_ERR_CUDA;
    if (e != cudaSuccess) set_error(std::string("CUDA error: ") + cudaGetErrorString(e));
    cudaFreeAsync(parts, st);
    return rc;
}

int qggmrf_hvp_launch(const float *x, const float *v, float *hv, int S, int R, int C, float sigma,
                      float p, float scale, double *vg, double *vgs, cudaStream_t st) {
    TC_TRY(prior_args(S, R, C, sigma, p));
    if ((size_t)S * R * C == 0) {
        if (vg) *vg = 0.0;
        if (vgs) *vgs = 0.0;
        return TC_OK;
    }
    const bool dots = vg || vgs;
    const dim3 grid(ceil_div(C, DX), ceil_div(R, DY), S);
    const int nparts = (int)(grid.x * grid.y * grid.z);
    double *parts = nullptr;
    if (dots) TC_CUDA(cudaMallocAsync(&parts, ((size_t)nparts * 2 + 2) * sizeof(double), st));
    const PriorParams pp = make_prior(sigma, p, scale);
    k_qggmrf_hvp<<<grid, dim3(DX, DY), 0, st>>>(x, v, hv, S, R, C, pp.inv_sigma, pp.inv_sq,
                                                pp.qmp, p, scale, parts);
    cudaError_t e = cudaGetLastError();
    int rc = TC_OK;
    if (e != cudaSuccess) {
        set_error(std::string("CUDA error: ") + cudaGetErrorString(e));
        rc = TC_ERR_CUDA;
    } else if (dots) {
        rc = finish_dots(parts, nparts, vg, vgs, st);
    }
    if (parts) cudaFreeAsync(parts, st);
    return rc;
}

}  // namespace tc
