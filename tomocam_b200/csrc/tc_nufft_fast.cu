// tc_nufft_fast.cu -- the fine-grid FFT of the type-1 NUFFT (back-projection,
// A^T y, the NUFFT gradient) on the register-resident FFT of tc_fft_fast.cuh,
// for the fine grids nf = 64 .. 4096 (powers of two), 1536, 3072 and 6144.
//
// The spreading pass stores the fine grid column-major, G[b][x][y] (column x
// is one contiguous line along y).  Then
//   A  columns  persistent CTAs walk (slice, pos) items, LC lines per CTA,
//               the next lines copied into shared memory by cp.async while the
//               current ones are transformed: FFT(+) along y of column
//               x = kidx(pos) (values gathered from shared memory in the
//               order the transform takes them), the N mode rows kept and
//               stored contiguously as row pos of R[b][pos][NS]
//   B  rows     persistent, RB mode rows of one slice per block, side by side
//               (one thread group and FFT scratch per row): the block's tile
//               R[b][:][r0 .. r0+RB) (16-byte pieces, two rows each) comes in
//               by cp.async, row r's values are taken in pos order -- the
//               order of the transform's input, because pass A stored column
//               kidx(pos) at pos -- the next block's tile is requested, then
//               FFT(+) along x, deconvolution, real part, subtraction and a
//               contiguous store of out[b][r][:].
// Mode r of an axis is frequency m = r - N/2 (index m mod nf of the fine
// grid), as in the general kernels k_t1_cols / k_t1_rows.
//
// The detector-axis DFT that precedes the spreading (centred, with the
// optional ramp, as k_t1_det) runs on the same transforms: directly when the
// detector length D is a register-FFT length, otherwise as Bluestein's chirp
// convolution on the smallest register length M >= 2D - 1 (D = 2908 on
// M = 6144): with w_n = exp(-i pi n^2 / D),
//   X_k = w_k sum_n (x_n w_n) conj(w_{k-n}),
// the convolution taken as forward FFT, product with the precomputed
// spectrum of conj(w) (in the transform's output order, 1/M folded in) and
// inverse FFT.
#include <algorithm>

#include "tc_cpasync.cuh"
#include "tc_fft_fast.cuh"
#include "tc_plan.cuh"

namespace tc {

namespace {

// slot of complex element n of a padded line: two padding slots per 16
// elements keep a warp's gathers in transform order at two-way bank
// conflicts at most and keep every pair (2k, 2k+1) in one 16-byte piece
__device__ __forceinline__ int lslot(int n) { return n + 2 * (n >> 4); }

template <class F>
struct T1Shape {
    static constexpr int LC = (F::T >= 256) ? 1 : 256 / F::T;  // pass A lines per CTA
    static constexpr int LSP = F::M + 2 * (F::M / 16);        // padded line (complex)
    static constexpr int SCR = (F::LS + 1) & ~1;               // FFT scratch (complex, even)
    static constexpr size_t SMEM_A = (size_t)LC * (SCR + LSP) * sizeof(c32);
    static constexpr int RB = (F::T >= 128) ? 2 : 256 / F::T;  // pass B rows per block
    static constexpr int TILE = RB * F::M + 2 * (F::M / 16);
    static constexpr size_t SMEM_B = (size_t)(RB * SCR + TILE) * sizeof(c32);
    static_assert(RB % 2 == 0, "pass B copies two rows per 16-byte piece");
};

// tile slot of (pos, row l) in pass B
template <int RB>
__device__ __forceinline__ int bslot(int pos, int l) { return pos * RB + l + 2 * (pos >> 4); }

// frequency m of natural index n of a length-M transform, as mode index
// m + N/2 of an N-mode axis; -1 when the frequency is not one of the modes
template <int M>
__device__ __forceinline__ int mode_of(int n, int N) {
    const int m = n < M / 2 ? n : n - M;
    const int r = m + N / 2;
    return (r >= 0 && r < N) ? r : -1;
}

template <class F, int LC>
__global__ void __launch_bounds__(F::T * LC, (F::T * LC <= 384) ? 2 : 1)
k_t1f_cols(const c32 *__restrict__ G, c32 *__restrict__ Rw, int N, int NS, int nb,
           const c32 *__restrict__ tw) {
    using S = T1Shape<F>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    c32 *scr = reinterpret_cast<c32 *>(smem_raw);
    c32 *pf = scr + LC * S::SCR;  // [LC][LSP]
    const int l = threadIdx.x / F::T, t = threadIdx.x % F::T;
    const int nitems = F::M * nb;
    const int per = nitems / gridDim.x, rem = nitems % gridDim.x;
    const int ib = blockIdx.x * per + min((int)blockIdx.x, rem);
    const int ie = ib + per + ((int)blockIdx.x < rem ? 1 : 0);
    constexpr int chunks = F::M / 2;  // 16-byte pieces per column
    auto prefetch = [&](int base) {
        for (int e = threadIdx.x; e < LC * chunks; e += F::T * LC) {
            const int ll = e / chunks, c = e - ll * chunks;
            const int it = base + ll;
            if (it < ie) {
                const int b = it / F::M, pos = it - b * F::M;
                const int x = F::kidx(pos >> 4, pos & 15);
                cp_async16(pf + ll * S::LSP + lslot(2 * c),
                           G + ((size_t)b * F::M + x) * F::M + 2 * c);
            }
        }
        cp_async_commit();
    };
    prefetch(ib);
    for (int base = ib; base < ie; base += LC) {
        cp_async_wait_all();
        __syncthreads();  // lines in; the last step's transforms are done with the scratch
        c32 v[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) v[i] = pf[l * S::LSP + lslot(F::kidx(t, i))];
        __syncthreads();  // prefetch buffer free
        if (base + LC < ie) prefetch(base + LC);
        const int it = base + l;
        F::inverse(v, scr + l * S::SCR, t, tw);
        if (it < ie) {
            const int b = it / F::M, pos = it - b * F::M;
            c32 *dst = Rw + ((size_t)b * F::M + pos) * NS;
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                const int r = mode_of<F::M>(F::nidx(t, i), N);
                if (r >= 0) dst[r] = v[i];
            }
        }
    }
    cp_async_wait_all();
}

template <class F, int RB>
__global__ void __launch_bounds__(F::T * RB, 1)
k_t1f_rows(const c32 *__restrict__ Rw, float *__restrict__ out, const float *__restrict__ sub,
           const float *__restrict__ corr, float scale, int N, int NS, int nb,
           const c32 *__restrict__ tw, int nslices, int pair) {
    using S = T1Shape<F>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    c32 *scr = reinterpret_cast<c32 *>(smem_raw);
    c32 *tile = scr + RB * S::SCR;
    const int l = threadIdx.x / F::T, t = threadIdx.x % F::T;
    const int nbr = (N + RB - 1) / RB, nblocks = nbr * nb;
    // a piece holds rows r0 + ll and r0 + ll + 1 (ll even); it is copied when
    // its first row is a mode row, and then its second row is below NS too
    // (r0 + ll is even, so r0 + ll + 1 <= N - 1 for even N and = N < NS for
    // odd N).  Slots of rows >= N are never read.
    auto issue = [&](int bb) {
        const int b = bb / nbr, r0 = (bb - b * nbr) * RB;
        const c32 *src = Rw + (size_t)b * F::M * NS + r0;
        for (int e = threadIdx.x; e < F::M * (RB / 2); e += F::T * RB) {
            const int pos = e / (RB / 2), ll = 2 * (e % (RB / 2));
            if (r0 + ll < N) cp_async16(tile + bslot<RB>(pos, ll), src + (size_t)pos * NS + ll);
        }
        cp_async_commit();
    };
    int bb = blockIdx.x;
    if (bb < nblocks) issue(bb);
    for (; bb < nblocks; bb += gridDim.x) {
        const int b = bb / nbr, r = (bb - b * nbr) * RB + l;
        const bool valid = r < N;
        cp_async_wait_all();
        __syncthreads();  // tile in; the last block's transforms are done with the scratch
        c32 v[16];
#pragma unroll
        for (int i = 0; i < 16; ++i)
            v[i] = valid ? tile[bslot<RB>(t * 16 + i, l)] : mk<float>(0.f, 0.f);
        __syncthreads();  // the tile is free: request the next block's
        if (bb + gridDim.x < nblocks) issue(bb + gridDim.x);
        F::inverse(v, scr + l * S::SCR, t, tw);
        if (valid) {
            // line b is slice b, or (pair) slices 2b (real part) and 2b + 1
            // (imaginary part)
            const float cr = corr[r] * scale;
            const int sa = pair ? 2 * b : b;
            const bool hb = pair && 2 * b + 1 < nslices;
            float *dst = out + ((size_t)sa * N + r) * N;
            const float *sb = sub ? sub + ((size_t)sa * N + r) * N : nullptr;
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                const int c = mode_of<F::M>(F::nidx(t, i), N);
                if (c >= 0) {
                    float val = v[i].x * corr[c] * cr;
                    if (sb) val -= sb[c];
                    dst[c] = val;
                    if (hb) {
                        float vb = v[i].y * corr[c] * cr;
                        if (sb) vb -= sb[(size_t)N * N + c];
                        dst[(size_t)N * N + c] = vb;
                    }
                }
            }
        }
    }
    cp_async_wait_all();
}

// detector-axis DFT of LC sinogram rows per CTA (line = slice b, angle p).
// Forward (back-projection, INV = false):
//   c[b][p][j] = sum_t y[b][p][t] exp(-2 pi i (t - h)(j - h) / D) [* |j - h| / D]
// (h = D / 2): input index n = (t - h) mod D, output c_j = X_{(j - h) mod D}.
// Inverse (radon, INV = true):
//   y[b][p][t] = scale * Re sum_j c_j exp(+2 pi i (j - h)(t - h) / D)
//              = scale * Re DFT(-)(conj c')_{(t - h) mod D},  c'_n = c_{(n + h) mod D},
// so the same forward transform runs on the conjugated point values.
// BLUE: Bluestein on M >= 2D - 1; else M == D and the transform's output is
// put in natural order through shared memory before the store.
template <class F, bool BLUE>
struct DetShape {
    static constexpr int LC = (F::T >= 256) ? 1 : 256 / F::T;
    static constexpr int LSP = F::M + 2 * (F::M / 16);
    static constexpr int SCR_ = (F::LS > LSP) ? F::LS : LSP;
    static constexpr int SCR = (SCR_ + 1) & ~1;
    static constexpr size_t SMEM = (size_t)LC * SCR * sizeof(c32);
};

// Paired lines (pair != 0): line q P + p takes slices 2q and 2q + 1 of angle
// p as one complex sequence; the point values of line q are the cstride
// values at cpts + q cstride, the mirror point of angle p (nvirt > 0, even
// D) at offset P D + p.  Forward: the j = 0 value is halved and also stored
// at the mirror point.  Inverse: the j = 0 value is replaced by the mean of
// itself and the mirror value, and slice 2q + 1 is the imaginary part.
// Blocks of up to 384 threads are held to two per SM (the 6144-point
// Bluestein lines: 102 registers left one block of 12 warps per SM; capped,
// radon at 2908² with 1969 angles went 0.321 -> 0.297 ms per slice).
template <class F, bool BLUE, bool INV>
__global__ void __launch_bounds__(F::T * DetShape<F, BLUE>::LC,
                                  (F::T * DetShape<F, BLUE>::LC <= 384) ? 2 : 1)
k_det_fast(const void *__restrict__ in, void *__restrict__ out, int D, int nlines, int ramp,
           float scale, const c32 *__restrict__ chirp, const c32 *__restrict__ bhat,
           const c32 *__restrict__ tw, int P, int nslices, int pair, size_t cstride, int nvirt) {
    using S = DetShape<F, BLUE>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int l = threadIdx.x / F::T, t = threadIdx.x % F::T;
    c32 *scr = reinterpret_cast<c32 *>(smem_raw) + l * S::SCR;
    const int line = blockIdx.x * S::LC + l;
    const bool valid = line < nlines;
    const int h = D / 2;
    const int lq = valid ? line : 0;
    const int q = pair ? lq / P : 0, p = pair ? lq - q * P : 0;
    // offsets of the input and output sequences (a: real part, b: imaginary)
    size_t in_a = (size_t)lq * D, in_b = 0, out_a = (size_t)lq * D, out_b = 0;
    bool hb = false;
    if (pair) {
        const size_t rows = ((size_t)(2 * q) * P + p) * D, pts = (size_t)q * cstride + (size_t)p * D;
        hb = 2 * q + 1 < nslices;
        if constexpr (INV) {
            in_a = pts;
            out_a = rows;
            out_b = rows + (size_t)P * D;
        } else {
            in_a = rows;
            in_b = rows + (size_t)P * D;
            out_a = pts;
        }
    }
    const bool mirror = pair && nvirt > 0;
    const size_t vslot = (size_t)q * cstride + (size_t)P * D + p;
    const float rs = 1.0f / (float)D;
    // final value of output index j (= (k + h) mod D)
    auto put = [&](int j, c32 x) {
        if constexpr (INV) {
            static_cast<float *>(out)[out_a + j] = x.x * scale;
            if (hb) static_cast<float *>(out)[out_b + j] = -x.y * scale;
        } else {
            if (ramp) x = x * ((float)abs(j - h) * rs);
            if (mirror && j == 0) {
                x = x * 0.5f;
                static_cast<c32 *>(out)[vslot] = x;
            }
            static_cast<c32 *>(out)[out_a + j] = x;
        }
    };
    c32 v[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        const int n = F::nidx(t, i);
        v[i] = mk<float>(0.f, 0.f);
        if (valid && n < D) {
            int tt = n + h;
            if (tt >= D) tt -= D;
            c32 y;
            if constexpr (INV) {
                float2 c = __ldg(reinterpret_cast<const float2 *>(in) + in_a + tt);
                if (mirror && tt == 0) {
                    const float2 m = __ldg(reinterpret_cast<const float2 *>(in) + vslot);
                    c = make_float2(0.5f * (c.x + m.x), 0.5f * (c.y + m.y));
                }
                y = mk<float>(c.x, -c.y);
            } else {
                const float *yr = static_cast<const float *>(in);
                y = mk<float>(__ldg(yr + in_a + tt), hb ? __ldg(yr + in_b + tt) : 0.f);
            }
            v[i] = BLUE ? cmul(chirp[n], y) : y;
        }
    }
    if constexpr (BLUE) {
        F::template forward<true>(v, scr, t, tw);
#pragma unroll
        for (int i = 0; i < 16; ++i) v[i] = cmul(v[i], bhat[t * 16 + i]);
        F::sync_before_inverse();
        // the chirp convolution's outputs k < D lie in the low half (M >= 2D - 1)
        F::template inverse<true, true>(v, scr, t, tw);
        if (valid) {
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                if (!F::low_half(i)) continue;
                const int k = F::nidx(t, i);
                if (k < D) {
                    int j = k + h;
                    if (j >= D) j -= D;
                    put(j, cmul(v[i], chirp[k]));
                }
            }
        }
    } else {
        F::forward(v, scr, t, tw);
        __syncthreads();  // the scratch becomes the reorder line
#pragma unroll
        for (int i = 0; i < 16; ++i) scr[lslot(F::kidx(t, i))] = v[i];
        __syncthreads();
        if (valid) {
            for (int k = t; k < D; k += F::T) {
                int j = k + h;
                if (j >= D) j -= D;
                put(j, scr[lslot(k)]);
            }
        }
    }
}

template <class F, bool BLUE, bool INV>
int run_det(const void *in, void *out, int P, int D, int nb, int ramp, float scale,
            const c32 *chirp, const c32 *bhat, const c32 *tw, cudaStream_t st, int pair,
            size_t cstride, int nvirt) {
    using S = DetShape<F, BLUE>;
    auto k = k_det_fast<F, BLUE, INV>;
    TC_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::SMEM));
    const int nlines = (pair ? (nb + 1) / 2 : nb) * P;
    k<<<ceil_div(nlines, S::LC), F::T * S::LC, S::SMEM, st>>>(in, out, D, nlines, ramp, scale,
                                                              chirp, bhat, tw, P, nb, pair,
                                                              cstride, nvirt);
    TC_LAUNCH_CHECK();
    return TC_OK;
}

// ---------------------------------------------------------------------------
// type-2 fine grid (radon, the NUFFT gradient): modes x[b][r][c] (real) ->
// column-major fine grid G[b][x][y] = FFT2(-) of the deconvolved modes placed
// at (c - N/2, r - N/2) mod nf.
//   A2 rows     LPC image rows per block (one thread group each): deconvolve,
//               FFT(-) along x, transposed through shared memory into
//               Q[b][pos][NS] (pos = the transform's output slot 16 t + v,
//               frequency kidx(t, v))
//   B2 columns  persistent, LC lines per CTA, next line copied by cp.async:
//               line Q[b][pos][:], FFT(-) along y, put in natural order
//               through shared memory and stored contiguously as column
//               x = kidx(pos) of G
// ---------------------------------------------------------------------------
template <class F>
struct T2Shape {
    static constexpr int LPC = (F::T >= 128) ? (F::T * 4 <= 1024 ? 4 : 2) : 512 / F::T;
    static constexpr int SM_A_ = (LPC * F::LS > LPC * F::M + F::M / 16) ? LPC * F::LS
                                                                         : LPC * F::M + F::M / 16;
    static constexpr int SM_A = (SM_A_ + 1) & ~1;  // FFT scratch / staging tile (complex)
    // + the image-row buffer [LPC][2][NX] and the deconvolution factors [NX]
    // (floats, NX = N rounded up to 4)
    static size_t smem_a(int N) {
        return (size_t)SM_A * sizeof(c32) + (size_t)(LPC * 2 + 1) * ((N + 3) & ~3) * sizeof(float);
    }
    static constexpr int LC = (F::T >= 256) ? 1 : 256 / F::T;
    static constexpr int LSP = F::M + 2 * (F::M / 16);
    static constexpr int SCR = (((F::LS > LSP) ? F::LS : LSP) + 1) & ~1;
};

// staging slot of (pos, line l): one padding slot per 16 positions
template <int LPC>
__device__ __forceinline__ int t2stg(int pos, int l) { return pos * LPC + l + (pos >> 4); }

// Persistent: a block is LPC image rows of one line, blocks b = blockIdx.x,
// blockIdx.x + gridDim.x, ...; the next block's rows (both slices of a
// paired line) are copied into xpf[LPC][2][NX] by cp.async while the current
// block is transformed (the image rows come from HBM; loaded in place they
// left the pass waiting on them).
template <class F, int LPC>
__global__ void __launch_bounds__(F::T * LPC, (F::T * LPC <= 512) ? 2 : 1)
k_t2f_rows(const float *__restrict__ x, c32 *__restrict__ Q, const float *__restrict__ corr,
           int N, int NS, const c32 *__restrict__ tw, int nslices, int pair, int nlines) {
    using S = T2Shape<F>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    c32 *sm = reinterpret_cast<c32 *>(smem_raw);
    const int NX = (N + 3) & ~3;
    float *xpf = reinterpret_cast<float *>(sm + S::SM_A);
    float *scorr = xpf + (size_t)LPC * 2 * NX;
    const int l = threadIdx.x / F::T, t = threadIdx.x % F::T;
    for (int c = threadIdx.x; c < N; c += F::T * LPC) scorr[c] = corr[c];  // read after the first barrier
    const int nbr = (N + LPC - 1) / LPC, nblocks = nbr * nlines;
    const bool vec = ((N & 3) == 0) && ((reinterpret_cast<uintptr_t>(x) & 15) == 0);
    // line q is slice q, or (pair) slices 2q (real part) and 2q + 1
    // (imaginary part, zero when nslices is odd)
    auto prefetch = [&](int bb) {
        const int q = bb / nbr, r0 = (bb - q * nbr) * LPC;
        const int s0 = pair ? 2 * q : q;
        const int ns = pair ? min(2, nslices - s0) : 1;
        const int per_row = vec ? N / 4 : N;
        for (int e = threadIdx.x; e < LPC * 2 * per_row; e += F::T * LPC) {
            const int row = e / per_row, c = e - row * per_row;
            const int r = r0 + (row >> 1), sl = row & 1;
            if (r >= N || sl >= ns) continue;
            const float *src = x + ((size_t)(s0 + sl) * N + r) * N;
            float *dst = xpf + (size_t)row * NX;
            if (vec) cp_async16(dst + 4 * c, src + 4 * c);
            else cp_async4(dst + c, src + c);
        }
        cp_async_commit();
    };
    int bb = blockIdx.x;
    if (bb < nblocks) prefetch(bb);
    for (; bb < nblocks; bb += gridDim.x) {
        const int b = bb / nbr, r0 = (bb - b * nbr) * LPC, r = r0 + l;
        const bool valid = r < N;
        const bool hb = pair && 2 * b + 1 < nslices;
        cp_async_wait_all();
        __syncthreads();  // rows in; the last block's staging tile is read out
        const float cr = valid ? scorr[r] : 0.f;
        const float *xa = xpf + (size_t)(2 * l) * NX, *xb = xa + NX;
        // the thread index passed through an opaque move: the 16 mode
        // indices and factors are formed anew each block rather than held in
        // registers across the loop (which spilled)
        int tl;
        asm volatile("mov.b32 %0, %1;" : "=r"(tl) : "r"(t));
        c32 v[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            const int c = mode_of<F::M>(F::nidx(tl, i), N);
            v[i] = mk<float>(0.f, 0.f);
            if (valid && c >= 0) {
                const float cc = scorr[c] * cr;
                v[i] = mk<float>(xa[c] * cc, hb ? xb[c] * cc : 0.f);
            }
        }
        __syncthreads();  // the row buffer is free: request the next block's
        const int bn = bb + gridDim.x;
        if (bn < nblocks) prefetch(bn);
        F::forward(v, sm + l * F::LS, t, tw);
        __syncthreads();  // the scratch becomes the staging tile
#pragma unroll
        for (int i = 0; i < 16; ++i) sm[t2stg<LPC>(t * 16 + i, l)] = v[i];
        __syncthreads();
        c32 *Qb = Q + (size_t)b * F::M * NS + r0;
        for (int e = threadIdx.x; e < F::M * LPC; e += F::T * LPC) {
            const int pos = e / LPC, ll = e - pos * LPC;
            if (r0 + ll < N) Qb[(size_t)pos * NS + ll] = sm[t2stg<LPC>(pos, ll)];
        }
    }
    cp_async_wait_all();
}

template <class F, int LC>
__global__ void __launch_bounds__(F::T * LC, (F::T * LC <= 384) ? 2 : 1)
k_t2f_cols(const c32 *__restrict__ Q, c32 *__restrict__ G, int N, int NS, int nb,
           const c32 *__restrict__ tw) {
    using S = T2Shape<F>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    c32 *scr = reinterpret_cast<c32 *>(smem_raw);
    c32 *pf = scr + LC * S::SCR;  // [LC][NS]
    const int l = threadIdx.x / F::T, t = threadIdx.x % F::T;
    const int nitems = F::M * nb;
    const int per = nitems / gridDim.x, rem = nitems % gridDim.x;
    const int ib = blockIdx.x * per + min((int)blockIdx.x, rem);
    const int ie = ib + per + ((int)blockIdx.x < rem ? 1 : 0);
    const int chunks = NS / 2;  // 16-byte pieces per line
    auto prefetch = [&](int base) {
        for (int e = threadIdx.x; e < LC * chunks; e += F::T * LC) {
            const int ll = e / chunks, c = e - ll * chunks;
            const int it = base + ll;
            if (it < ie) cp_async16(pf + (size_t)ll * NS + 2 * c, Q + (size_t)it * NS + 2 * c);
        }
        cp_async_commit();
    };
    prefetch(ib);
    for (int base = ib; base < ie; base += LC) {
        cp_async_wait_all();
        __syncthreads();  // lines in; the last step's stores are done with the scratch
        c32 v[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            const int r = mode_of<F::M>(F::nidx(t, i), N);
            v[i] = r >= 0 ? pf[(size_t)l * NS + r] : mk<float>(0.f, 0.f);
        }
        __syncthreads();  // prefetch buffer free
        if (base + LC < ie) prefetch(base + LC);
        const int it = base + l;
        c32 *ro = scr + l * S::SCR;
        F::forward(v, ro, t, tw);
        __syncthreads();  // the scratch becomes the reorder line
#pragma unroll
        for (int i = 0; i < 16; ++i) ro[lslot(F::kidx(t, i))] = v[i];
        __syncthreads();
        if (it < ie) {
            const int b = it / F::M, pos = it - b * F::M;
            const int xcol = F::kidx(pos >> 4, pos & 15);
            c32 *dst = G + ((size_t)b * F::M + xcol) * F::M;
            for (int y = t; y < F::M; y += F::T) dst[y] = ro[lslot(y)];
        }
    }
    cp_async_wait_all();
}

template <class F>
int run_t2f(const float *x, c32 *Q, c32 *G, const float *corr, int N, int nslices, const c32 *tw,
            cudaStream_t st, int pair) {
    const int nb = pair ? (nslices + 1) / 2 : nslices;  // lines
    using S = T2Shape<F>;
    if (2 * N > F::M) TC_FAIL(TC_ERR_STATE, "fine grid smaller than twice the modes");
    const int NS = t1_fast_stride(N);
    auto ka = k_t2f_rows<F, S::LPC>;
    auto kb = k_t2f_cols<F, S::LC>;
    const size_t smem_a = S::smem_a(N);
    const size_t smem_b = ((size_t)S::LC * S::SCR + (size_t)S::LC * NS) * sizeof(c32);
    if (smem_a > 227 * 1024 || smem_b > 227 * 1024)
        TC_FAIL(TC_ERR_STATE, "a fine-grid FFT pass does not fit shared memory");
    TC_CUDA(cudaFuncSetAttribute(ka, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_a));
    TC_CUDA(cudaFuncSetAttribute(kb, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_b));
    TC_CUDA(cudaFuncSetAttribute(ka, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 cudaSharedmemCarveoutMaxShared));
    TC_CUDA(cudaFuncSetAttribute(kb, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 cudaSharedmemCarveoutMaxShared));
    int dev = 0, nsm = 0, occa = 0, occb = 0;
    TC_CUDA(cudaGetDevice(&dev));
    TC_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    TC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occa, ka, F::T * S::LPC, smem_a));
    TC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occb, kb, F::T * S::LC, smem_b));
    if (occa < 1 || occb < 1) TC_FAIL(TC_ERR_STATE, "a fine-grid FFT pass does not fit on an SM");
    const int nblocks_a = ceil_div(N, S::LPC) * nb;
    ka<<<std::min(nblocks_a, nsm * occa), F::T * S::LPC, smem_a, st>>>(x, Q, corr, N, NS, tw,
                                                                      nslices, pair, nb);
    TC_LAUNCH_CHECK();
    const int nitems = F::M * nb;
    kb<<<std::min(ceil_div(nitems, S::LC), nsm * occb), F::T * S::LC, smem_b, st>>>(Q, G, N, NS,
                                                                                  nb, tw);
    TC_LAUNCH_CHECK();
    return TC_OK;
}

template <class F>
int run_t1f(const c32 *G, c32 *Rw, float *out, const float *sub, const float *corr, float scale,
            int N, int nslices, const c32 *tw, cudaStream_t st, int pair) {
    const int nb = pair ? (nslices + 1) / 2 : nslices;  // lines
    using S = T1Shape<F>;
    if (2 * N > F::M) TC_FAIL(TC_ERR_STATE, "fine grid smaller than twice the modes");
    const int NS = t1_fast_stride(N);
    auto ka = k_t1f_cols<F, S::LC>;
    auto kb = k_t1f_rows<F, S::RB>;
    TC_CUDA(cudaFuncSetAttribute(ka, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::SMEM_A));
    TC_CUDA(cudaFuncSetAttribute(kb, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::SMEM_B));
    TC_CUDA(cudaFuncSetAttribute(ka, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 cudaSharedmemCarveoutMaxShared));
    TC_CUDA(cudaFuncSetAttribute(kb, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 cudaSharedmemCarveoutMaxShared));
    int dev = 0, nsm = 0, occa = 0, occb = 0;
    TC_CUDA(cudaGetDevice(&dev));
    TC_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    TC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occa, ka, F::T * S::LC, S::SMEM_A));
    TC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occb, kb, F::T * S::RB, S::SMEM_B));
    if (occa < 1 || occb < 1) TC_FAIL(TC_ERR_STATE, "a fine-grid FFT pass does not fit on an SM");
    const int nitems = F::M * nb;
    ka<<<std::min(ceil_div(nitems, S::LC), nsm * occa), F::T * S::LC, S::SMEM_A, st>>>(
        G, Rw, N, NS, nb, tw);
    TC_LAUNCH_CHECK();
    const int nblocks = ceil_div(N, S::RB) * nb;
    kb<<<std::min(nblocks, nsm * occb), F::T * S::RB, S::SMEM_B, st>>>(Rw, out, sub, corr, scale,
                                                                     N, NS, nb, tw, nslices,
                                                                     pair);
    TC_LAUNCH_CHECK();
    return TC_OK;
}

}  // namespace

int t2_fast_grid(const float *x, c32 *Q, c32 *G, const float *corr, int N, int nf, int nb,
                 const c32 *tw, cudaStream_t st, int pair) {
    switch (nf) {
        case 64: return run_t2f<F64>(x, Q, G, corr, N, nb, tw, st, pair);
        case 128: return run_t2f<F128>(x, Q, G, corr, N, nb, tw, st, pair);
        case 256: return run_t2f<F256>(x, Q, G, corr, N, nb, tw, st, pair);
        case 512: return run_t2f<F512>(x, Q, G, corr, N, nb, tw, st, pair);
        case 1024: return run_t2f<F1024>(x, Q, G, corr, N, nb, tw, st, pair);
        case 1536: return run_t2f<F1536>(x, Q, G, corr, N, nb, tw, st, pair);
        case 2048: return run_t2f<F2048>(x, Q, G, corr, N, nb, tw, st, pair);
        case 3072: return run_t2f<F3072>(x, Q, G, corr, N, nb, tw, st, pair);
        case 4096: return run_t2f<F4096>(x, Q, G, corr, N, nb, tw, st, pair);
        case 6144: return run_t2f<F6144>(x, Q, G, corr, N, nb, tw, st, pair);
        default: TC_FAIL(TC_ERR_STATE, "no register FFT for this fine grid");
    }
}

bool t1_fast_supported(int nf) {
    switch (nf) {
        case 64: case 128: case 256: case 512: case 1024: case 1536: case 2048: case 3072:
        case 4096: case 6144: return true;
        default: return false;
    }
}

int t1_fast_grid(int N) {
    static const int sizes[] = {64, 128, 256, 512, 1024, 1536, 2048, 3072, 4096, 6144};
    for (int s : sizes)
        if (s >= 2 * N) return s;
    return 0;
}

int t1_fast_stride(int N) { return (N + 3) & ~3; }

// kidx of a register-FFT length (host), for the spectrum's storage order
static int kidx_of(int M, int t, int v) {
    switch (M) {
        case 64: return F64::kidx(t, v);
        case 128: return F128::kidx(t, v);
        case 256: return F256::kidx(t, v);
        case 512: return F512::kidx(t, v);
        case 1024: return F1024::kidx(t, v);
        case 1536: return F1536::kidx(t, v);
        case 2048: return F2048::kidx(t, v);
        case 3072: return F3072::kidx(t, v);
        case 4096: return F4096::kidx(t, v);
        case 6144: return F6144::kidx(t, v);
        default: return -1;
    }
}

int det_fast_setup(Plan &pl) {
    const int D = pl.N;
    pl.det_M = 0;
    pl.det_blue = false;
    if (t1_fast_supported(D)) {
        pl.det_M = D;
        return pl.fft_det_tw.init(D);
    }
    // smallest register length >= 2D - 1 (all are even, so >= 2D)
    const int M = t1_fast_grid(D);
    if (M == 0) return TC_OK;  // general engine
    // chirp w_n = exp(-i pi n^2 / D) (n^2 reduced mod 2D), spectrum of
    // b_m = conj(w_|m|) on m in (-D, D) (index m mod M), scaled by 1/M and
    // stored in the transform's output order
    std::vector<std::complex<double>> w(D), b(M, 0.0);
    for (int n = 0; n < D; ++n) {
        const long long e = (long long)n * n % (2LL * D);
        const double a = -M_PI * (double)e / (double)D;
        w[n] = std::complex<double>(std::cos(a), std::sin(a));
    }
    for (int m = 0; m < D; ++m) {
        b[m] = std::conj(w[m]);
        if (m > 0) b[M - m] = std::conj(w[m]);
    }
    host_fft(b, -1);
    std::vector<c32> hb(M), hw(D);
    for (int q = 0; q < M; ++q) {
        const std::complex<double> z = b[kidx_of(M, q / 16, q % 16)] / (double)M;
        hb[q] = mk<float>((float)z.real(), (float)z.imag());
    }
    for (int n = 0; n < D; ++n) hw[n] = mk<float>((float)w[n].real(), (float)w[n].imag());
    TC_TRY(pl.d_det_chirp.reserve((size_t)D * sizeof(c32)));
    TC_TRY(pl.d_det_bhat.reserve((size_t)M * sizeof(c32)));
    TC_CUDA(cudaMemcpy(pl.d_det_chirp.ptr, hw.data(), (size_t)D * sizeof(c32), cudaMemcpyHostToDevice));
    TC_CUDA(cudaMemcpy(pl.d_det_bhat.ptr, hb.data(), (size_t)M * sizeof(c32), cudaMemcpyHostToDevice));
    pl.det_M = M;
    pl.det_blue = true;
    return pl.fft_det_tw.init(M);
}

static int det_dispatch(const Plan &pl, const void *in, void *out, int nb, int ramp, float scale,
                        bool inv, cudaStream_t st, int pair) {
    const c32 *tw = pl.fft_det_tw.dev.tw;
    const c32 *ch = pl.d_det_chirp.as<c32>(), *bh = pl.d_det_bhat.as<c32>();
    const int P = pl.P, D = pl.N;
    const size_t cs = pl.npts_ext();
    const int nv = pl.nvirt;
#define TC_DET(MM, FF)                                                                            \
    case MM:                                                                                      \
        if (inv)                                                                                  \
            return pl.det_blue ? run_det<FF, true, true>(in, out, P, D, nb, ramp, scale, ch, bh,   \
                                                          tw, st, pair, cs, nv)                   \
                               : run_det<FF, false, true>(in, out, P, D, nb, ramp, scale, ch, bh, \
                                                          tw, st, pair, cs, nv);                  \
        return pl.det_blue ? run_det<FF, true, false>(in, out, P, D, nb, ramp, scale, ch, bh, tw, \
                                                      st, pair, cs, nv)                           \
                           : run_det<FF, false, false>(in, out, P, D, nb, ramp, scale, ch, bh,    \
                                                       tw, st, pair, cs, nv);
    switch (pl.det_M) {
        TC_DET(64, F64)
        TC_DET(128, F128)
        TC_DET(256, F256)
        TC_DET(512, F512)
        TC_DET(1024, F1024)
        TC_DET(1536, F1536)
        TC_DET(2048, F2048)
        TC_DET(3072, F3072)
        TC_DET(4096, F4096)
        TC_DET(6144, F6144)
        default: TC_FAIL(TC_ERR_STATE, "no register FFT for this detector length");
    }
#undef TC_DET
}

int det_fast(const Plan &pl, const float *sino, c32 *cpts, int nb, int ramp, cudaStream_t st,
             int pair) {
    return det_dispatch(pl, sino, cpts, nb, ramp, 1.f, false, st, pair);
}

int det_fast_inv(const Plan &pl, const c32 *cpts, float *sino, int nb, float scale,
                 cudaStream_t st, int pair) {
    return det_dispatch(pl, cpts, sino, nb, 0, scale, true, st, pair);
}

int t1_fast_fft(const c32 *G, c32 *Rw, float *out, const float *sub, const float *corr,
                float scale, int N, int nf, int nb, const c32 *tw, cudaStream_t st, int pair) {
    switch (nf) {
        case 64: return run_t1f<F64>(G, Rw, out, sub, corr, scale, N, nb, tw, st, pair);
        case 128: return run_t1f<F128>(G, Rw, out, sub, corr, scale, N, nb, tw, st, pair);
        case 256: return run_t1f<F256>(G, Rw, out, sub, corr, scale, N, nb, tw, st, pair);
        case 512: return run_t1f<F512>(G, Rw, out, sub, corr, scale, N, nb, tw, st, pair);
        case 1024: return run_t1f<F1024>(G, Rw, out, sub, corr, scale, N, nb, tw, st, pair);
        case 1536: return run_t1f<F1536>(G, Rw, out, sub, corr, scale, N, nb, tw, st, pair);
        case 2048: return run_t1f<F2048>(G, Rw, out, sub, corr, scale, N, nb, tw, st, pair);
        case 3072: return run_t1f<F3072>(G, Rw, out, sub, corr, scale, N, nb, tw, st, pair);
        case 4096: return run_t1f<F4096>(G, Rw, out, sub, corr, scale, N, nb, tw, st, pair);
        case 6144: return run_t1f<F6144>(G, Rw, out, sub, corr, scale, N, nb, tw, st, pair);
        default: TC_FAIL(TC_ERR_STATE, "no register FFT for this fine grid");
    }
}

}  // namespace tc
