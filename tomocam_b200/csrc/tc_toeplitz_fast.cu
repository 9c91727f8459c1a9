// tc_toeplitz_fast.cu -- Toeplitz operator for power-of-two FFT sizes
// M = 64 .. 4096 (images up to 2048 x 2048) on the register-resident FFT of
// tc_fft_fast.cuh.
//
// Same three passes over a slice pair as tc_toeplitz.cu, without reordering:
//   1. rows     forward FFT of each padded row; a thread stores its 16 values
//               contiguously, so the workspace row is in kidx order
//   2. columns  forward FFT down each workspace column, multiply by the PSF
//               spectrum pre-permuted into the same (row, column) kidx
//               order, inverse FFT, keep the N image rows
//   3. rows     inverse FFT of each workspace row (its input is already in
//               kidx order), scale, subtract A^T y, FP64 dots per CTA
#include <cmath>

#include "tc_fft_fast.cuh"
#include "tc_plan.cuh"

namespace tc {

template <class F>
__device__ __forceinline__ void load16(c32 *v, const c32 *__restrict__ src) {
    const float4 *s = reinterpret_cast<const float4 *>(src);
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const float4 a = s[i];
        v[2 * i] = mk<float>(a.x, a.y);
        v[2 * i + 1] = mk<float>(a.z, a.w);
    }
}

template <class F>
__device__ __forceinline__ void store16(c32 *dst, const c32 *v) {
    float4 *d = reinterpret_cast<float4 *>(dst);
#pragma unroll
    for (int i = 0; i < 8; ++i) d[i] = make_float4(v[2 * i].x, v[2 * i].y, v[2 * i + 1].x, v[2 * i + 1].y);
}

// pass 1: LPC rows per CTA
template <class F, int LPC>
__global__ void __launch_bounds__(F::T * LPC)
k_tpf_rows(const float *__restrict__ x, c32 *__restrict__ W, int N, int nb,
           const int *__restrict__ sel, size_t sel_stride, const c32 *__restrict__ tw) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    c32 *sm = reinterpret_cast<c32 *>(smem_raw);
    const int l = threadIdx.x / F::T, t = threadIdx.x % F::T;
    const int r = blockIdx.x * LPC + l, q = blockIdx.y;
    const bool valid = r < N;
    if (sel) x += (size_t)sel[0] * sel_stride;
    const float *xa = x + ((size_t)(2 * q) * N + (valid ? r : 0)) * N;
    const float *xb = (2 * q + 1 < nb) ? x + ((size_t)(2 * q + 1) * N + (valid ? r : 0)) * N : nullptr;
    c32 v[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        const int n = F::nidx(t, i);
        v[i] = mk<float>(0.f, 0.f);
        if (valid && n < N) v[i] = mk<float>(xa[n], xb ? xb[n] : 0.f);
    }
    F::forward(v, sm + l * F::LS, t, tw);
    if (valid) store16<F>(W + ((size_t)q * N + r) * F::M + t * 16, v);
}

// pass 2: CW columns per CTA.  Pairs of adjacent columns are interleaved
// over the lanes (a warp's load of one row covers 16 contiguous bytes); no
// more than two, so the 16 consecutive t of a stage-2/3 group stay in one
// warp, which is what FastFFT's warp-level barrier relies on.
template <class F, int CW>
__global__ void __launch_bounds__(F::T * CW)
k_tpf_cols(c32 *__restrict__ W, const float *__restrict__ phatp, int N,
           const c32 *__restrict__ tw) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    c32 *sm = reinterpret_cast<c32 *>(smem_raw);
    constexpr int CI = (CW >= 2) ? 2 : 1;
    const int c = (threadIdx.x / (F::T * CI)) * CI + threadIdx.x % CI;
    const int t = (threadIdx.x / CI) % F::T;
    const int pos = blockIdx.x * CW + c, q = blockIdx.y;
    c32 *Wq = W + (size_t)q * N * F::M;
    c32 v[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        const int n = F::nidx(t, i);
        v[i] = (n < N) ? Wq[(size_t)n * F::M + pos] : mk<float>(0.f, 0.f);
    }
    F::forward(v, sm + c * F::LS, t, tw);
    const float4 *ph = reinterpret_cast<const float4 *>(phatp + (size_t)pos * F::M + t * 16);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const float4 p = __ldg(ph + i);
        v[4 * i + 0] = v[4 * i + 0] * p.x;
        v[4 * i + 1] = v[4 * i + 1] * p.y;
        v[4 * i + 2] = v[4 * i + 2] * p.z;
        v[4 * i + 3] = v[4 * i + 3] * p.w;
    }
    F::sync_before_inverse();
    F::inverse(v, sm + c * F::LS, t, tw);
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        const int n = F::nidx(t, i);
        if (n < N) Wq[(size_t)n * F::M + pos] = v[i];
    }
}

// pass 3: LPC rows per CTA; partials (optional) get one {x.Hx, x.aty} per CTA
template <class F, int LPC>
__global__ void __launch_bounds__(F::T * LPC)
k_tpf_out(const c32 *__restrict__ W, const float *x, const float *__restrict__ aty, float *g,
          double *__restrict__ partials, int N, int nb, float scale, const int *__restrict__ sel,
          size_t sel_stride, const c32 *__restrict__ tw) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    c32 *sm = reinterpret_cast<c32 *>(smem_raw);
    const int l = threadIdx.x / F::T, t = threadIdx.x % F::T;
    const int r = blockIdx.x * LPC + l, q = blockIdx.y;
    const bool valid = r < N;
    if (sel) {
        x += (size_t)sel[0] * sel_stride;
        g += (size_t)sel[0] * sel_stride;
    }
    c32 v[16];
    if (valid) {
        load16<F>(v, W + ((size_t)q * N + r) * F::M + t * 16);
    } else {
#pragma unroll
        for (int i = 0; i < 16; ++i) v[i] = mk<float>(0.f, 0.f);
    }
    F::inverse(v, sm + l * F::LS, t, tw);
    const bool has_b = (2 * q + 1 < nb);
    const size_t oa = ((size_t)(2 * q) * N + (valid ? r : 0)) * N;
    const size_t ob = ((size_t)(2 * q + 1) * N + (valid ? r : 0)) * N;
    double d[2] = {0.0, 0.0};
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        const int n = F::nidx(t, i);
        if (valid && n < N) {
            const float ha = v[i].x * scale, hb = v[i].y * scale;
            const float aa = aty ? aty[oa + n] : 0.f;
            const float ab = (aty && has_b) ? aty[ob + n] : 0.f;
            if (partials) {
                const float xa = x[oa + n];
                d[0] += (double)xa * ha;
                d[1] += (double)xa * aa;
                if (has_b) {
                    const float xb = x[ob + n];
                    d[0] += (double)xb * hb;
                    d[1] += (double)xb * ab;
                }
            }
            g[oa + n] = ha - aa;
            if (has_b) g[ob + n] = hb - ab;
        }
    }
    if (partials) {
        block_sum<2>(d);
        if (threadIdx.x == 0) {
            double *dst = partials + ((size_t)q * gridDim.x + blockIdx.x) * 2;
            dst[0] = d[0];
            dst[1] = d[1];
        }
    }
}

// PSF spectrum in pass-2 order: out[pos][t*16+v] = phat[kx(pos)][ky(t, v)]
template <class F>
__global__ void k_phat_perm(const float *__restrict__ phat, float *__restrict__ out) {
    const size_t total = (size_t)F::M * F::M;
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total;
         idx += (size_t)gridDim.x * blockDim.x) {
        const int pos = (int)(idx / F::M), i = (int)(idx % F::M);
        const int kx = F::kidx(pos / 16, pos % 16), ky = F::kidx(i / 16, i % 16);
        out[idx] = phat[(size_t)kx * F::M + ky];
    }
}

// ---------------------------------------------------------------------------
template <class F>
struct FastShape {
    static constexpr int LPC = (F::T >= 256) ? 1 : 256 / F::T;  // rows per CTA (passes 1, 3)
    static constexpr int CW = (F::T >= 256) ? 2 : 256 / F::T;    // columns per CTA (pass 2)
};

template <class F>
static int run_fast(Plan &pl, const float *x, const float *aty, float *g, int nb,
                    double *partials, cudaStream_t st, const int *sel, size_t sel_stride) {
    using S = FastShape<F>;
    const int N = pl.N;
    const int npairs = (nb + 1) / 2;
    TC_TRY(pl.ws_toe.reserve((size_t)npairs * N * F::M * sizeof(c32)));
    c32 *W = pl.ws_toe.as<c32>();
    const c32 *tw = pl.fft_M.dev.tw;
    const size_t sm_rows = (size_t)S::LPC * F::LS * sizeof(c32);
    const size_t sm_cols = (size_t)S::CW * F::LS * sizeof(c32);
    auto k1 = k_tpf_rows<F, S::LPC>;
    auto k2 = k_tpf_cols<F, S::CW>;
    auto k3 = k_tpf_out<F, S::LPC>;
    TC_CUDA(cudaFuncSetAttribute(k1, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_rows));
    TC_CUDA(cudaFuncSetAttribute(k2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_cols));
    TC_CUDA(cudaFuncSetAttribute(k3, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_rows));
    const dim3 grow(ceil_div(N, S::LPC), npairs);
    k1<<<grow, F::T * S::LPC, sm_rows, st>>>(x, W, N, nb, sel, sel_stride, tw);
    TC_LAUNCH_CHECK();
    k2<<<dim3(F::M / S::CW, npairs), F::T * S::CW, sm_cols, st>>>(W, pl.d_phatp.as<float>(), N, tw);
    TC_LAUNCH_CHECK();
    const float scale = (float)(1.0 / ((double)F::M * F::M * std::pow((double)N, 3)));
    k3<<<grow, F::T * S::LPC, sm_rows, st>>>(W, x, aty, g, partials, N, nb, scale, sel,
                                             sel_stride, tw);
    TC_LAUNCH_CHECK();
    return TC_OK;
}

template <class F>
static int perm_fast(Plan &pl, cudaStream_t st) {
    TC_TRY(pl.d_phatp.reserve((size_t)F::M * F::M * sizeof(float)));
    k_phat_perm<F><<<1024, 256, 0, st>>>(pl.d_phat.as<float>(), pl.d_phatp.as<float>());
    TC_LAUNCH_CHECK();
    return TC_OK;
}

using F64 = FastFFT<4, 4, 4>;
using F128 = FastFFT<8, 4, 4>;
using F256 = FastFFT<8, 8, 4>;
using F512 = FastFFT<2, 16, 16>;
using F1024 = FastFFT<4, 16, 16>;
using F2048 = FastFFT<8, 16, 16>;
using F4096 = FastFFT<16, 16, 16>;

bool toeplitz_fast_supported(int M) {
    return M == 64 || M == 128 || M == 256 || M == 512 || M == 1024 || M == 2048 || M == 4096;
}

int toeplitz_fast_lpc(int M) {
    switch (M) {
        case 64: return FastShape<F64>::LPC;
        case 128: return FastShape<F128>::LPC;
        case 256: return FastShape<F256>::LPC;
        case 512: return FastShape<F512>::LPC;
        case 1024: return FastShape<F1024>::LPC;
        case 2048: return FastShape<F2048>::LPC;
        case 4096: return FastShape<F4096>::LPC;
        default: return 1;
    }
}

int toeplitz_fast_chunk(Plan &pl, const float *x, const float *aty, float *g, int nb,
                        double *partials, cudaStream_t st, const int *sel, size_t sel_stride) {
    switch (pl.M) {
        case 64: return run_fast<F64>(pl, x, aty, g, nb, partials, st, sel, sel_stride);
        case 128: return run_fast<F128>(pl, x, aty, g, nb, partials, st, sel, sel_stride);
        case 256: return run_fast<F256>(pl, x, aty, g, nb, partials, st, sel, sel_stride);
        case 512: return run_fast<F512>(pl, x, aty, g, nb, partials, st, sel, sel_stride);
        case 1024: return run_fast<F1024>(pl, x, aty, g, nb, partials, st, sel, sel_stride);
        case 2048: return run_fast<F2048>(pl, x, aty, g, nb, partials, st, sel, sel_stride);
        case 4096: return run_fast<F4096>(pl, x, aty, g, nb, partials, st, sel, sel_stride);
        default: TC_FAIL(TC_ERR_STATE, "no register FFT for this Toeplitz size");
    }
}

int toeplitz_fast_permute(Plan &pl, cudaStream_t st) {
    switch (pl.M) {
        case 64: return perm_fast<F64>(pl, st);
        case 128: return perm_fast<F128>(pl, st);
        case 256: return perm_fast<F256>(pl, st);
        case 512: return perm_fast<F512>(pl, st);
        case 1024: return perm_fast<F1024>(pl, st);
        case 2048: return perm_fast<F2048>(pl, st);
        case 4096: return perm_fast<F4096>(pl, st);
        default: TC_FAIL(TC_ERR_STATE, "no register FFT for this Toeplitz size");
    }
}

}  // namespace tc
