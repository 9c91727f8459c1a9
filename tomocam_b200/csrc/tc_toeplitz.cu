// tc_toeplitz.cu -- Toeplitz data-fidelity operator H x = A^T A x.
//
// H is the linear convolution of the image with the point-spread function
// (src/toeplitz.h:107-159):
//   (H x)[k] = sum_m x[m] psf[k - m] / N^3,   psf[d] = Re sum_j exp(i d.w_j)
// evaluated by zero-padded FFTs of size M >= 2N-1 (any such M gives the same
// linear convolution; the reference uses M = 2N-1).  psf is even, so its
// spectrum PHAT is real and two real slices ride in one complex transform:
// z = x_a + i x_b, Hz = H x_a + i H x_b.
//
// Three passes over a slice pair, the [N][M] complex workspace sized to stay
// in L2:
//   1. rows:    FFT(-) of the N image rows padded to M
//   2. columns: FFT(-) of N-row columns padded to M, * PHAT, FFT(+), keep N rows
//   3. rows:    FFT(+), keep N columns, scale, subtract A^T y, FP64 dots
#include <algorithm>
#include <cmath>

#include "tc_plan.cuh"

namespace tc {

// ---------------------------------------------------------------------------
// pass 1
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(FFT_MAX_THREADS, 1)
k_tp_rows(const float *__restrict__ x, c32 *__restrict__ W, int N, int nb,
                          const int *__restrict__ sel, size_t sel_stride, FftDev<float> dM) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    c32 *line = reinterpret_cast<c32 *>(smem_raw);
    const int r = blockIdx.x, q = blockIdx.y, M = dM.L;
    if (sel) x += (size_t)sel[0] * sel_stride;
    const float *xa = x + ((size_t)(2 * q) * N + r) * N;
    const float *xb = (2 * q + 1 < nb) ? x + ((size_t)(2 * q + 1) * N + r) * N : nullptr;
    for (int c = threadIdx.x; c < M; c += blockDim.x) {
        c32 v = mk<float>(0.f, 0.f);
        if (c < N) v = mk<float>(xa[c], xb ? xb[c] : 0.f);
        line[c] = v;
    }
    __syncthreads();
    fft_line<float, -1>(line, M, 1, dM, threadIdx.x, blockDim.x);
    c32 *dst = W + ((size_t)q * N + r) * M;
    for (int c = threadIdx.x; c < M; c += blockDim.x) dst[c] = line[c];
}

// ---------------------------------------------------------------------------
// pass 2
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(FFT_MAX_THREADS, 1)
k_tp_cols(c32 *__restrict__ W, const float *__restrict__ phat, int N, int cw,
                          FftDev<float> dM) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    c32 *buf = reinterpret_cast<c32 *>(smem_raw);
    const int q = blockIdx.y, k0 = blockIdx.x * cw, M = dM.L;
    c32 *Wq = W + (size_t)q * N * M;
    for (int i = threadIdx.x; i < M * cw; i += blockDim.x) {
        const int r = i / cw, c = i - r * cw;
        buf[(size_t)c * M + r] = (r < N) ? Wq[(size_t)r * M + k0 + c] : mk<float>(0.f, 0.f);
    }
    __syncthreads();
    fft_line<float, -1>(buf, M, cw, dM, threadIdx.x, blockDim.x);
    for (int i = threadIdx.x; i < M * cw; i += blockDim.x) {
        const int c = i / M, ky = i - c * M;
        buf[i] = buf[i] * phat[(size_t)(k0 + c) * M + ky];
    }
    __syncthreads();
    fft_line<float, +1>(buf, M, cw, dM, threadIdx.x, blockDim.x);
    for (int i = threadIdx.x; i < N * cw; i += blockDim.x) {
        const int r = i / cw, c = i - r * cw;
        Wq[(size_t)r * M + k0 + c] = buf[(size_t)c * M + r];
    }
}

// ---------------------------------------------------------------------------
// pass 3
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(FFT_MAX_THREADS, 1)
k_tp_out(const c32 *__restrict__ W, const float *x, const float *__restrict__ aty,
                         float *g, double *__restrict__ partials, int N, int nb, float scale,
                         const int *__restrict__ sel, size_t sel_stride, FftDev<float> dM) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    c32 *line = reinterpret_cast<c32 *>(smem_raw);
    const int r = blockIdx.x, q = blockIdx.y, M = dM.L;
    if (sel) {
        x += (size_t)sel[0] * sel_stride;
        g += (size_t)sel[0] * sel_stride;
    }
    const c32 *src = W + ((size_t)q * N + r) * M;
    for (int c = threadIdx.x; c < M; c += blockDim.x) line[c] = src[c];
    __syncthreads();
    fft_line<float, +1>(line, M, 1, dM, threadIdx.x, blockDim.x);
    const bool has_b = (2 * q + 1 < nb);
    const size_t oa = ((size_t)(2 * q) * N + r) * N;
    const size_t ob = ((size_t)(2 * q + 1) * N + r) * N;
    double d[2] = {0.0, 0.0};
    for (int c = threadIdx.x; c < N; c += blockDim.x) {
        const c32 v = line[c];
        const float ha = v.x * scale, hb = v.y * scale;
        const float aa = aty ? aty[oa + c] : 0.f;
        const float ab = (aty && has_b) ? aty[ob + c] : 0.f;
        if (partials) {
            const float xa = x[oa + c];
            d[0] += (double)xa * ha;
            d[1] += (double)xa * aa;
            if (has_b) {
                const float xb = x[ob + c];
                d[0] += (double)xb * hb;
                d[1] += (double)xb * ab;
            }
        }
        g[oa + c] = ha - aa;
        if (has_b) g[ob + c] = hb - ab;
    }
    if (partials) {
        block_sum<2>(d);
        if (threadIdx.x == 0) {
            partials[((size_t)q * N + r) * 2 + 0] = d[0];
            partials[((size_t)q * N + r) * 2 + 1] = d[1];
        }
    }
}

// deterministic sum of nparts rows of nvals doubles
__global__ void k_reduce_partials(const double *__restrict__ in, int nparts, int nvals,
                                  double *__restrict__ out) {
    for (int v = 0; v < nvals; ++v) {
        double s[1] = {0.0};
        for (int i = threadIdx.x; i < nparts; i += blockDim.x) s[0] += in[(size_t)i * nvals + v];
        block_sum<1>(s);
        if (threadIdx.x == 0) out[v] = s[0];
        __syncthreads();
    }
}

int reduce_partials(const double *partials, int nparts, int nvals, double *out, cudaStream_t st) {
    k_reduce_partials<<<1, 1024, 0, st>>>(partials, nparts, nvals, out);
    TC_LAUNCH_CHECK();
    return TC_OK;
}

static int tp_col_width(int M) {
    int cw = 4;
    while (cw > 1 && ((size_t)cw * M * sizeof(c32) > 128 * 1024 ||
                      fft_threads<float>(M, cw) > FFT_MAX_THREADS ||
                      M % cw))
        cw /= 2;
    return cw;
}

int toeplitz_partials_count(const Plan &pl, int nb) {
    return ((nb + 1) / 2) * ceil_div(pl.N, pl.toe_lpc);
}

// nb slices starting at x; partials (optional) receives
// toeplitz_partials_count(pl, nb) rows of {x.Hx, x.aty}
int toeplitz_chunk(Plan &pl, const float *x, const float *aty, float *g, int nb,
                   double *partials, cudaStream_t st, const int *sel, size_t sel_stride) {
    if (pl.toe_fast) return toeplitz_fast_chunk(pl, x, aty, g, nb, partials, st, sel, sel_stride);
    const int N = pl.N, M = pl.M;
    const int npairs = (nb + 1) / 2;
    TC_TRY(pl.ws_toe.reserve((size_t)npairs * N * M * sizeof(c32)));
    c32 *W = pl.ws_toe.as<c32>();
    const int nthr1 = fft_threads<float>(M, 1);
    const size_t smem1 = (size_t)M * sizeof(c32);
    TC_CUDA(cudaFuncSetAttribute(k_tp_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem1));
    TC_CUDA(cudaFuncSetAttribute(k_tp_out, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem1));
    k_tp_rows<<<dim3(N, npairs), nthr1, smem1, st>>>(x, W, N, nb, sel, sel_stride, pl.fft_M.dev);
    TC_LAUNCH_CHECK();
    const int cw = tp_col_width(M);
    const int nthr2 = fft_threads<float>(M, cw);
    const size_t smem2 = (size_t)cw * M * sizeof(c32);
    TC_CUDA(cudaFuncSetAttribute(k_tp_cols, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem2));
    k_tp_cols<<<dim3(M / cw, npairs), nthr2, smem2, st>>>(W, pl.d_phat.as<float>(), N, cw,
                                                          pl.fft_M.dev);
    TC_LAUNCH_CHECK();
    const float scale = (float)(1.0 / ((double)M * M * std::pow((double)N, 3)));
    k_tp_out<<<dim3(N, npairs), nthr1, smem1, st>>>(W, x, aty, g, partials, N, nb, scale, sel,
                                                    sel_stride, pl.fft_M.dev);
    TC_LAUNCH_CHECK();
    return TC_OK;
}

// ---------------------------------------------------------------------------
// PSF spectrum: phat[kx][ky] = Re FFT2(psf embedded circularly in M x M)
// ---------------------------------------------------------------------------
__global__ void k_embed_psf(const double *__restrict__ psf, c64 *__restrict__ out, int N, int M) {
    const int nm = 2 * N - 1;
    const size_t total = (size_t)M * M;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total;
         i += (size_t)gridDim.x * blockDim.x) {
        const int r = (int)(i / M), c = (int)(i % M);
        const int d2 = (r <= N - 1) ? r : r - M;
        const int d1 = (c <= N - 1) ? c : c - M;
        double v = 0.0;
        if (d2 >= -(N - 1) && d1 >= -(N - 1))
            v = psf[(size_t)(d2 + N - 1) * nm + (d1 + N - 1)];
        out[i] = mk<double>(v, 0.0);
    }
}

__global__ void k_transpose_c64(const c64 *__restrict__ in, c64 *__restrict__ out, int M) {
    __shared__ c64 tile[32][33];
    const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const int r = by + j, c = bx + threadIdx.x;
        if (r < M && c < M) tile[j][threadIdx.x] = in[(size_t)r * M + c];
    }
    __syncthreads();
    for (int j = threadIdx.y; j < 32; j += blockDim.y) {
        const int r = bx + j, c = by + threadIdx.x;
        if (r < M && c < M) out[(size_t)r * M + c] = tile[threadIdx.x][j];
    }
}

__global__ void k_real_to_f32(const c64 *__restrict__ in, float *__restrict__ out, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        out[i] = (float)in[i].x;
}

int phat_from_psf(Plan &pl, const double *psf, cudaStream_t st) {
    const int N = pl.N, M = pl.M;
    FftTables<double> T;
    TC_TRY(T.init(M));
    DevBuf a, b;
    TC_TRY(a.reserve((size_t)M * M * sizeof(c64)));
    TC_TRY(b.reserve((size_t)M * M * sizeof(c64)));
    k_embed_psf<<<1024, 256, 0, st>>>(psf, a.as<c64>(), N, M);
    TC_LAUNCH_CHECK();
    TC_TRY(fft_lines_launch<double>(T, a.as<c64>(), a.as<c64>(), M, -1, st));
    k_transpose_c64<<<dim3(ceil_div(M, 32), ceil_div(M, 32)), dim3(32, 8), 0, st>>>(a.as<c64>(),
                                                                                   b.as<c64>(), M);
    TC_LAUNCH_CHECK();
    TC_TRY(fft_lines_launch<double>(T, b.as<c64>(), b.as<c64>(), M, -1, st));
    TC_TRY(pl.d_phat.reserve((size_t)M * M * sizeof(float)));
    k_real_to_f32<<<1024, 256, 0, st>>>(b.as<c64>(), pl.d_phat.as<float>(), (size_t)M * M);
    TC_LAUNCH_CHECK();
    TC_CUDA(cudaStreamSynchronize(st));
    return TC_OK;
}

}  // namespace tc
