// tc_prior.cu -- standalone qGGMRF gradient, g += scale * sum_26 w rho'(x_v - x_n)
// with clamp-to-edge boundaries (src/gpu/cuTV2.cu:33-93,
// src/gpu/dev_memory.cuh:88-94).
#include "tc_plan.cuh"
#include "tc_prior.cuh"

namespace tc {

// One thread per voxel along x; a CTA covers a 32 x 8 patch of one slice and
// reads the 3 x 10 x 34 neighbourhood from shared memory.
constexpr int QX = 32, QY = 8;

__global__ void k_qggmrf(const float *__restrict__ x, float *__restrict__ g, int S, int R, int C,
                         PriorParams pp) {
    __shared__ float tile[3][QY + 2][QX + 2];
    const int c0 = blockIdx.x * QX, r0 = blockIdx.y * QY, s = blockIdx.z;
    const size_t plane = (size_t)R * C;
    for (int i = threadIdx.y * QX + threadIdx.x; i < 3 * (QY + 2) * (QX + 2); i += QX * QY) {
        const int dz = i / ((QY + 2) * (QX + 2));
        const int rem = i - dz * (QY + 2) * (QX + 2);
        const int dy = rem / (QX + 2), dx = rem - dy * (QX + 2);
        const int ss = min(max(s + dz - 1, 0), S - 1);
        const int rr = min(max(r0 + dy - 1, 0), R - 1);
        const int cc = min(max(c0 + dx - 1, 0), C - 1);
        tile[dz][dy][dx] = x[ss * plane + (size_t)rr * C + cc];
    }
    __syncthreads();
    const int c = c0 + threadIdx.x, r = r0 + threadIdx.y;
    if (c >= C || r >= R) return;
    const float u = tile[1][threadIdx.y + 1][threadIdx.x + 1];
    float acc = 0.0f;
#pragma unroll
    for (int dz = 0; dz < 3; ++dz)
#pragma unroll
        for (int dy = 0; dy < 3; ++dy)
#pragma unroll
            for (int dx = 0; dx < 3; ++dx) {
                if (dz == 1 && dy == 1 && dx == 1) continue;
                const float nb = tile[dz][threadIdx.y + dy][threadIdx.x + dx];
                acc = fmaf(c_qggmrf_w[(dz * 3 + dy) * 3 + dx], d_pot_unscaled(u - nb, pp), acc);
            }
    const size_t v = s * plane + (size_t)r * C + c;
    g[v] += (pp.scale * pp.inv_sq) * acc;
}

int qggmrf_launch(const float *x, float *g, int S, int R, int C, float sigma, float p,
                  float scale, cudaStream_t st) {
    if (S > 65535) TC_FAIL(TC_ERR_SHAPE, "too many slices for one prior launch");
    dim3 grid(ceil_div(C, QX), ceil_div(R, QY), S);
    k_qggmrf<<<grid, dim3(QX, QY), 0, st>>>(x, g, S, R, C, make_prior(sigma, p, scale));
    TC_LAUNCH_CHECK();
    return TC_OK;
}

}  // namespace tc
