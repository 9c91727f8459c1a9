// tc_prep.cu -- geometry conditioning around the solver, on the device:
// detector pad + roll (src/preproc.cpp:38-108), symmetric image pad
// (src/padding.cpp:37-91), crop (src/postproc.cpp:37-102), and the small
// reductions mbir2 needs (max, sum of squares; src/mbir2.cpp:46-54,77).
#include <algorithm>
#include <cmath>
#include <vector>

#include "tc_plan.cuh"
#include "tc_prep.cuh"

namespace tc {

// out[s][p][z] = padded[(z + off) mod D2], padded[k] = in[k - npad] (0 outside)
__global__ void k_preproc(const float *__restrict__ in, float *__restrict__ out, size_t rows,
                          int D, int D2, int npad, int off) {
    const size_t total = rows * D2;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total;
         i += (size_t)gridDim.x * blockDim.x) {
        const size_t row = i / D2;
        const int z = (int)(i - row * D2);
        int k = (z + off) % D2;
        if (k < 0) k += D2;
        const int src = k - npad;
        out[i] = (src >= 0 && src < D) ? in[row * D + src] : 0.0f;
    }
}

// out[s][r][c] = in[s][r - sh][c - sh] inside, 0 outside; out is R2 x C2
__global__ void k_pad2d(const float *__restrict__ in, float *__restrict__ out, int S, int R, int C,
                        int R2, int C2, int sh) {
    const size_t total = (size_t)S * R2 * C2;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total;
         i += (size_t)gridDim.x * blockDim.x) {
        const size_t s = i / ((size_t)R2 * C2);
        const size_t rem = i - s * R2 * C2;
        const int r = (int)(rem / C2) - sh, c = (int)(rem % C2) - sh;
        out[i] = (r >= 0 && r < R && c >= 0 && c < C) ? in[(s * R + r) * C + c] : 0.0f;
    }
}

// out[s][r][c] = in[s][r + sh][c + sh]; out is R2 x C2, in is R x C
__global__ void k_crop2d(const float *__restrict__ in, float *__restrict__ out, int S, int R, int C,
                         int R2, int C2, int sh) {
    const size_t total = (size_t)S * R2 * C2;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total;
         i += (size_t)gridDim.x * blockDim.x) {
        const size_t s = i / ((size_t)R2 * C2);
        const size_t rem = i - s * R2 * C2;
        const int r = (int)(rem / C2), c = (int)(rem % C2);
        out[i] = in[(s * R + r + sh) * C + c + sh];
    }
}

__global__ void k_scale(float *__restrict__ x, size_t n, float f) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        x[i] = x[i] / f;
}

__global__ void k_axpby(float a, const float *__restrict__ x, float b, float *__restrict__ y,
                        size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        y[i] = a * x[i] + b * y[i];
}

__global__ void k_fill(float *__restrict__ x, size_t n, float v) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        x[i] = v;
}

// per-block max and FP64 sum of squares
__global__ void k_max_sumsq(const float *__restrict__ x, size_t n, float *__restrict__ pmax,
                            double *__restrict__ psq) {
    float m = -INFINITY;
    double sq[1] = {0.0};
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const float v = x[i];
        m = fmaxf(m, v);
        sq[0] += (double)v * v;
    }
    __shared__ float smax[32];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_down_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) smax[threadIdx.x >> 5] = m;
    block_sum<1>(sq);
    __syncthreads();
    if (threadIdx.x == 0) {
        float mm = -INFINITY;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) mm = fmaxf(mm, smax[w]);
        pmax[blockIdx.x] = mm;
        psq[blockIdx.x] = sq[0];
    }
}

static int grid_for(size_t n) {
    return (int)std::min<size_t>(std::max<size_t>(ceil_div64((int64_t)n, 256), 1), 148 * 16);
}

void preproc_params(int ncols, float center, int &npad, int &off) {
    // std::round: halves away from zero
    const int cen = (int)std::round((double)center);
    off = (ncols + 1) / 2 - cen;
    npad = (int)(0.42 * ncols) / 2;
    if (std::abs(off) > npad) npad = std::abs(off);
}

int preproc_dev(const float *sino, float *out, int S, int P, int D, int npad, int off,
                cudaStream_t st) {
    const int D2 = D + 2 * npad;
    const size_t rows = (size_t)S * P;
    k_preproc<<<grid_for(rows * D2), 256, 0, st>>>(sino, out, rows, D, D2, npad, off);
    TC_LAUNCH_CHECK();
    return TC_OK;
}

int pad2d_dev(const float *in, float *out, int S, int R, int C, int npad, cudaStream_t st) {
    k_pad2d<<<grid_for((size_t)S * (R + npad) * (C + npad)), 256, 0, st>>>(
        in, out, S, R, C, R + npad, C + npad, npad / 2);
    TC_LAUNCH_CHECK();
    return TC_OK;
}

int crop2d_dev(const float *in, float *out, int S, int R, int C, int npixels, cudaStream_t st) {
    const int np = (C - npixels) / 2;
    k_crop2d<<<grid_for((size_t)S * (R - 2 * np) * (C - 2 * np)), 256, 0, st>>>(
        in, out, S, R, C, R - 2 * np, C - 2 * np, np);
    TC_LAUNCH_CHECK();
    return TC_OK;
}

int scale_dev(float *x, size_t n, float divisor, cudaStream_t st) {
    k_scale<<<grid_for(n), 256, 0, st>>>(x, n, divisor);
    TC_LAUNCH_CHECK();
    return TC_OK;
}

int axpby_dev(float a, const float *x, float b, float *y, size_t n, cudaStream_t st) {
    k_axpby<<<grid_for(n), 256, 0, st>>>(a, x, b, y, n);
    TC_LAUNCH_CHECK();
    return TC_OK;
}

int fill_dev(float *x, size_t n, float v, cudaStream_t st) {
    k_fill<<<grid_for(n), 256, 0, st>>>(x, n, v);
    TC_LAUNCH_CHECK();
    return TC_OK;
}

int max_sumsq_dev(const float *x, size_t n, float *maxv, double *sumsq, cudaStream_t st) {
    const int nb = grid_for(n);
    DevBuf pm, ps;
    TC_TRY(pm.reserve(nb * sizeof(float)));
    TC_TRY(ps.reserve(nb * sizeof(double)));
    k_max_sumsq<<<nb, 256, 0, st>>>(x, n, pm.as<float>(), ps.as<double>());
    TC_LAUNCH_CHECK();
    std::vector<float> hm(nb);
    std::vector<double> hs(nb);
    TC_CUDA(cudaMemcpyAsync(hm.data(), pm.ptr, nb * sizeof(float), cudaMemcpyDeviceToHost, st));
    TC_CUDA(cudaMemcpyAsync(hs.data(), ps.ptr, nb * sizeof(double), cudaMemcpyDeviceToHost, st));
    TC_CUDA(cudaStreamSynchronize(st));
    float m = -INFINITY;
    double s = 0.0;
    for (int i = 0; i < nb; ++i) {
        m = std::max(m, hm[i]);
        s += hs[i];
    }
    if (maxv) *maxv = m;
    if (sumsq) *sumsq = s;
    return TC_OK;
}

}  // namespace tc
