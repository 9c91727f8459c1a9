// tc_toeplitz_fast.cu -- Toeplitz operator for the FFT sizes M = 64 .. 4096
// (powers of two), 1536, 3072, 6144 and 8192 (images up to 4096 x 4096) on
// the register-resident FFT of tc_fft_fast.cuh (M = 3 x 2^k: one radix-3
// stage in front of three 2^k transforms; M = 8192: one radix-2 stage in
// front of two 4096 transforms).
//
// Same three passes over a slice pair as tc_toeplitz.cu, without reordering.
// The workspace of a pair is column-major, Wt[pos][row] with a row stride NS
// (N rounded up to 4): pos is the storage position of a row-transform
// frequency (kidx order), so every column of the 2-D transform is one
// contiguous line.
//   1. rows     forward FFT of each padded row (the zero upper half of the
//               input is known at compile time); the CTA's rows are
//               transposed through shared memory into Wt
//   2. columns  persistent CTAs walk (pos, pair) items, prefetching the next
//               line with cp.async while the current one is transformed:
//               forward FFT, multiply by the PSF spectrum (pre-permuted into
//               the same order, kept in registers while pos is unchanged),
//               inverse FFT, keep the N image rows
//   3. rows     gather the CTA's rows out of Wt through shared memory, inverse
//               FFT, scale, subtract A^T y, FP64 dots per CTA
#include <cmath>

#include "tc_cpasync.cuh"
#include "tc_fft_fast.cuh"
#include "tc_plan.cuh"

namespace tc {

// row stride of the column-major workspace (16-byte aligned lines, 32-byte
// aligned column starts)
inline int toe_stride(int N) { return (N + 3) & ~3; }

template <class F>
struct FastShape {
    // image rows per block of passes 1 and 3: at least 4, so a transposed
    // workspace access covers whole 32-byte sectors
    static constexpr int LPC = (F::T >= 128) ? (F::T * 4 <= 1024 ? 4 : 2) : 512 / F::T;
    static constexpr int NT_ROWS = F::T * LPC;  // threads per CTA, passes 1 and 3
    // lines per CTA in pass 2
    static constexpr int LC = (F::T >= 256) ? 1 : 256 / F::T;
    // staging / FFT scratch of passes 1 and 3, in complex elements (even, so
    // the image-row buffer after it is 16-byte aligned)
    static constexpr int SM_ROWS_ =
        (LPC * F::LS > LPC * F::M + F::M / 16) ? LPC * F::LS : LPC * F::M + F::M / 16;
    static constexpr int SM_ROWS = (SM_ROWS_ + 1) & ~1;
    static constexpr int SCR_COLS = (LC * F::LS + 15) & ~15;
    // pass 3: rows per block, threads, FFT scratch and tile sizes (complex)
    static constexpr int LPC_OUT = (F::T >= 128) ? 2 : 256 / F::T;
    static constexpr int NT_OUT = F::T * LPC_OUT;
    static constexpr int SCR_OUT = (LPC_OUT * F::LS + 1) & ~1;
    static constexpr int TILE_OUT = F::M * LPC_OUT + 2 * (F::M / 16);
    // M = 8192: the double-buffered pass 3 would not fit shared memory; a
    // one-block-per-CTA form (tile = FFT scratch) is used instead
    static constexpr bool SIMPLE_OUT = (SCR_OUT + TILE_OUT) * 8 > 200 * 1024;
};

// staging slot of (pos, line l) when LPC lines are transposed through shared
// memory: one padding slot per 16 positions spreads a warp's register-side
// accesses (t*16+i, fixed i) over all banks; the tile side is contiguous
template <int LPC>
__device__ __forceinline__ int stg(int pos, int l) { return pos * LPC + l + (pos >> 4); }

// copy the image rows r0 .. r0+LPC-1 of both slices of pair q into
// xpf[LPC][2][NX] (16-byte pieces when rows are 16-byte aligned, else 4)
template <int LPC>
__device__ __forceinline__ void prefetch_rows(float *xpf, const float *x, int N, int NX, int nb,
                                              int q, int r0, bool vec) {
    const int per_row = vec ? N / 4 : N;
    for (int e = threadIdx.x; e < LPC * 2 * per_row; e += blockDim.x) {
        const int row = e / per_row, c = e - row * per_row;
        const int r = r0 + (row >> 1), sl = 2 * q + (row & 1);
        if (r >= N || sl >= nb) continue;
        const float *src = x + ((size_t)sl * N + r) * N;
        float *dst = xpf + (size_t)row * NX;
        if (vec) cp_async16(dst + 4 * c, src + 4 * c);
        else cp_async4(dst + c, src + c);
    }
}

// pass 1: persistent; a block is LPC image rows of one slice pair, blocks
// b = blockIdx.x, blockIdx.x + gridDim.x, ...; the next block's image rows
// are prefetched while the current block is transformed
template <class F, int LPC>
__global__ void __launch_bounds__(F::T * LPC, (F::T * LPC <= 512) ? 2 : 1)
k_tpf_rows(const float *__restrict__ x, c32 *__restrict__ W, int N, int NS, int nb,
           const int *__restrict__ sel, size_t sel_stride, const c32 *__restrict__ tw) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    c32 *sm = reinterpret_cast<c32 *>(smem_raw);
    float *xpf = reinterpret_cast<float *>(sm + FastShape<F>::SM_ROWS);
    const int l = threadIdx.x / F::T, t = threadIdx.x % F::T;
    if (sel) x += (size_t)sel[0] * sel_stride;
    const int NX = (N + 3) & ~3;
    const bool vec = ((N & 3) == 0) && ((reinterpret_cast<uintptr_t>(x) & 15) == 0);
    const int nbr = (N + LPC - 1) / LPC, nblocks = nbr * ((nb + 1) / 2);
    int b = blockIdx.x;
    if (b < nblocks) prefetch_rows<LPC>(xpf, x, N, NX, nb, b / nbr, (b % nbr) * LPC, vec);
    cp_async_commit();
    for (; b < nblocks; b += gridDim.x) {
        const int q = b / nbr, r0 = (b - q * nbr) * LPC;
        const bool valid = r0 + l < N, has_b = 2 * q + 1 < nb;
        cp_async_wait_all();
        __syncthreads();
        c32 v[16];
        const float *xa = xpf + (size_t)(2 * l) * NX, *xb = xa + NX;
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            v[i] = mk<float>(0.f, 0.f);
            if (!F::low_half(i)) continue;
            const int n = F::nidx(t, i);
            if (valid && n < N) v[i] = mk<float>(xa[n], has_b ? xb[n] : 0.f);
        }
        __syncthreads();  // the image-row buffer is free
        const int bn = b + gridDim.x;
        if (bn < nblocks) prefetch_rows<LPC>(xpf, x, N, NX, nb, bn / nbr, (bn % nbr) * LPC, vec);
        cp_async_commit();
        F::template forward<true>(v, sm + l * F::LS, t, tw);
        __syncthreads();  // the scratch becomes the staging tile
#pragma unroll
        for (int i = 0; i < 16; ++i) sm[stg<LPC>(t * 16 + i, l)] = v[i];
        __syncthreads();
        c32 *Wq = W + (size_t)q * F::M * NS + r0;
        for (int e = threadIdx.x; e < F::M * LPC; e += F::T * LPC) {
            const int pos = e / LPC, ll = e % LPC;
            if (r0 + ll < N) Wq[(size_t)pos * NS + ll] = sm[stg<LPC>(pos, ll)];
        }
    }
    cp_async_wait_all();
}

// pass 2: persistent; LC lines per CTA.  The CTA owns the contiguous range
// [ib, ie) of items it = pos * npairs + q; step s gives line l the item
// ib + s * LC + l.  The next step's lines are copied into the prefetch buffer
// (cp.async, 16 bytes per request) while the current step is transformed.
template <class F, int LC>
__global__ void __launch_bounds__(F::T * LC, (F::T * LC <= 384) ? 2 : 1)
k_tpf_cols(c32 *__restrict__ W, const float *__restrict__ phatp, int N, int NS, int npairs,
           const c32 *__restrict__ tw) {
    // TIGHT: 384-thread lines (M = 6144) under the 80-register cap of two
    // CTAs per SM.  There the PSF column is read again (from L1) for every
    // item instead of held in registers across the slice pairs of a
    // position, and the inverse forms the low half directly: fewer spills,
    // operator at 2908² 0.2518 -> 0.2462 ms per slice.  With more registers
    // (M = 4096: 128, no spill) holding the column is faster (0.0802
    // against 0.0824 ms per slice).
    constexpr bool TIGHT = F::T * LC == 384;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    c32 *scr = reinterpret_cast<c32 *>(smem_raw);
    c32 *pf = scr + FastShape<F>::SCR_COLS;  // [LC][NS]
    const int l = threadIdx.x / F::T, t = threadIdx.x % F::T;
    const int nitems = F::M * npairs;
    const int per = nitems / gridDim.x, rem = nitems % gridDim.x;
    const int ib = blockIdx.x * per + min((int)blockIdx.x, rem);
    const int ie = ib + per + ((int)blockIdx.x < rem ? 1 : 0);
    const int chunks = NS / 2;  // 16-byte pieces per line
    auto prefetch = [&](int base) {
        for (int e = threadIdx.x; e < LC * chunks; e += F::T * LC) {
            const int ll = e / chunks, cpos = e - ll * chunks;
            const int it = base + ll;
            if (it < ie) {
                const int pos = it / npairs, q = it - pos * npairs;
                cp_async16(pf + (size_t)ll * NS + 2 * cpos,
                           W + ((size_t)q * F::M + pos) * NS + 2 * cpos);
            }
        }
        cp_async_commit();
    };
    prefetch(ib);
    float ph[16];
    int ph_pos = -1;
    for (int base = ib; base < ie; base += LC) {
        cp_async_wait_all();
        __syncthreads();
        c32 v[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            v[i] = mk<float>(0.f, 0.f);
            if (!F::low_half(i)) continue;
            const int n = F::nidx(t, i);
            if (n < N) v[i] = pf[(size_t)l * NS + n];
        }
        __syncthreads();  // prefetch buffer free
        if (base + LC < ie) prefetch(base + LC);
        const int it = base + l;
        const bool valid = it < ie;
        const int pos = valid ? it / npairs : 0, q = valid ? it - pos * npairs : 0;
        if (!TIGHT && pos != ph_pos) {
            const float4 *src = reinterpret_cast<const float4 *>(phatp + (size_t)pos * F::M + t * 16);
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const float4 p = __ldg(src + i);
                ph[4 * i + 0] = p.x;
                ph[4 * i + 1] = p.y;
                ph[4 * i + 2] = p.z;
                ph[4 * i + 3] = p.w;
            }
            ph_pos = pos;
        }
        F::template forward<true>(v, scr + l * F::LS, t, tw);
        if constexpr (TIGHT) {
            const float4 *src = reinterpret_cast<const float4 *>(phatp + (size_t)pos * F::M + t * 16);
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const float4 p = __ldg(src + i);
                v[4 * i + 0] = v[4 * i + 0] * p.x;
                v[4 * i + 1] = v[4 * i + 1] * p.y;
                v[4 * i + 2] = v[4 * i + 2] * p.z;
                v[4 * i + 3] = v[4 * i + 3] * p.w;
            }
        } else {
#pragma unroll
            for (int i = 0; i < 16; ++i) v[i] = v[i] * ph[i];
        }
        F::sync_before_inverse();
        if constexpr (TIGHT) F::template inverse<true, true>(v, scr + l * F::LS, t, tw);
        else F::template inverse<true>(v, scr + l * F::LS, t, tw);
        if (valid) {
            c32 *dst = W + ((size_t)q * F::M + pos) * NS;
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                if (!F::low_half(i)) continue;
                const int n = F::nidx(t, i);
                if (n < N) dst[n] = v[i];
            }
        }
    }
    cp_async_wait_all();
}

// pass 3: persistent; a block is LPC image rows of one slice pair.  Shared
// memory holds the FFT scratch, one workspace tile [pos][LPC] (16-byte pieces,
// slot(pos, l) = pos * LPC + l + 2 (pos >> 4)) and two image-row buffers.
// Right after a block's tile has been read into registers, the next block's
// tile and image rows are requested, so those copies overlap this block's
// transforms and epilogue.  Lines are interleaved by half warps (the 16
// threads of an FFT group stay together), which makes the register-side tile
// reads conflict-free.  partials (optional) get one {x.Hx, x.aty} row per
// block: row q * ceil(N / LPC) + r0 / LPC.
template <class F, int LPC>
__device__ __forceinline__ int tslot(int pos, int l) { return pos * LPC + l + 2 * (pos >> 4); }

template <class F, int LPC>
__global__ void __launch_bounds__(F::T * LPC, 1)
k_tpf_out(const c32 *__restrict__ W, const float *x, const float *__restrict__ aty, float *g,
          double *__restrict__ partials, int N, int NS, int nb, float scale,
          const int *__restrict__ sel, size_t sel_stride, const c32 *__restrict__ tw) {
    using S = FastShape<F>;
    static_assert(LPC % 2 == 0, "pass 3 copies two rows per 16-byte piece");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    c32 *scr = reinterpret_cast<c32 *>(smem_raw);
    c32 *tile = scr + S::SCR_OUT;
    float *xbuf = reinterpret_cast<float *>(tile + S::TILE_OUT);
    constexpr bool HW = F::T >= 16;
    const int l = HW ? (int)((threadIdx.x >> 4) % LPC) : (int)(threadIdx.x / F::T);
    const int t = HW ? (int)(((threadIdx.x >> 4) / LPC) * 16 + (threadIdx.x & 15))
                     : (int)(threadIdx.x % F::T);
    if (sel) {
        x += (size_t)sel[0] * sel_stride;
        g += (size_t)sel[0] * sel_stride;
    }
    // the row buffers hold the epilogue's image rows: x for the dots, else
    // A^T y (with dots and A^T y both, A^T y is read from global memory)
    const bool need_x = partials != nullptr;
    const bool aty_buf = !need_x && aty != nullptr;
    const float *rsrc = need_x ? x : aty;
    const bool need_rows = rsrc != nullptr;
    const int NX = (N + 3) & ~3;
    const bool vec = ((N & 3) == 0) && ((reinterpret_cast<uintptr_t>(rsrc) & 15) == 0);
    const int nbr = (N + LPC - 1) / LPC, nblocks = nbr * ((nb + 1) / 2);
    // a piece holds rows r0+ll and r0+ll+1 (ll even); it is copied when its
    // first row is an image row, and then its second row is below NS too
    // (r0 + ll is even, so r0 + ll + 1 <= N - 1 for even N and = N < NS for
    // odd N).  Slots of rows >= N are never read (those lines are masked).
    auto issue = [&](int bb, float *xdst) {
        const int q = bb / nbr, r0 = (bb - q * nbr) * LPC;
        const c32 *Wq = W + (size_t)q * F::M * NS + r0;
        for (int e = threadIdx.x; e < F::M * LPC / 2; e += F::T * LPC) {
            const int pos = e / (LPC / 2), ll = 2 * (e % (LPC / 2));
            if (r0 + ll < N) cp_async16(tile + tslot<F, LPC>(pos, ll), Wq + (size_t)pos * NS + ll);
        }
        if (need_rows) prefetch_rows<LPC>(xdst, rsrc, N, NX, nb, q, r0, vec);
        cp_async_commit();
    };
    int b = blockIdx.x, cur = 0;
    if (b < nblocks) issue(b, xbuf);
    for (; b < nblocks; b += gridDim.x, cur ^= 1) {
        const int q = b / nbr, rb = b - q * nbr, r0 = rb * LPC, r = r0 + l;
        const bool valid = r < N, has_b = 2 * q + 1 < nb;
        cp_async_wait_all();
        __syncthreads();
        c32 v[16];
#pragma unroll
        for (int i = 0; i < 16; ++i)
            v[i] = valid ? tile[tslot<F, LPC>(t * 16 + i, l)] : mk<float>(0.f, 0.f);
        __syncthreads();  // the tile buffer is free: request the next block
        const int bn = b + gridDim.x;
        if (bn < nblocks) issue(bn, xbuf + (size_t)(cur ^ 1) * LPC * 2 * NX);
        F::template inverse<true>(v, scr + l * F::LS, t, tw);
        const size_t oa = ((size_t)(2 * q) * N + (valid ? r : 0)) * N;
        const size_t ob = ((size_t)(2 * q + 1) * N + (valid ? r : 0)) * N;
        const float *xa = xbuf + (size_t)cur * LPC * 2 * NX + (size_t)(2 * l) * NX, *xb = xa + NX;
        double d[2] = {0.0, 0.0};
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            if (!F::low_half(i)) continue;
            const int n = F::nidx(t, i);
            if (valid && n < N) {
                const float ha = v[i].x * scale, hb = v[i].y * scale;
                const float aa = aty_buf ? xa[n] : (aty ? aty[oa + n] : 0.f);
                const float ab = !has_b ? 0.f : (aty_buf ? xb[n] : (aty ? aty[ob + n] : 0.f));
                if (need_x) {
                    const float xva = xa[n];
                    d[0] += (double)xva * ha;
                    d[1] += (double)xva * aa;
                    if (has_b) {
                        const float xvb = xb[n];
                        d[0] += (double)xvb * hb;
                        d[1] += (double)xvb * ab;
                    }
                }
                g[oa + n] = ha - aa;
                if (has_b) g[ob + n] = hb - ab;
            }
        }
        if (need_x) {
            block_sum<2>(d);
            if (threadIdx.x == 0) {
                double *dst = partials + ((size_t)q * nbr + rb) * 2;
                dst[0] = d[0];
                dst[1] = d[1];
            }
        }
    }
    cp_async_wait_all();
}

// pass 3 where the double-buffered form does not fit (M = 8192): persistent,
// a block is image rows r0, r0 + 1 of one slice pair, F::T threads.  The
// block's workspace tile (one 16-byte piece per position holding both rows,
// slot tslot<F, 2>) is copied by cp.async; each thread takes row r0's 16
// inputs, transforms and finishes that row, takes row r0 + 1's inputs, then
// requests the next block's tile, so that copy overlaps the second row's
// transform and epilogue.  The FFT scratch is separate from the tile.
// partials (optional) get one {x.Hx, x.aty} row per block: row
// q * ceil(N / 2) + r0 / 2.
template <class F>
__global__ void __launch_bounds__(F::T, 1)
k_tpf_out_s(const c32 *__restrict__ W, const float *x, const float *__restrict__ aty, float *g,
            double *__restrict__ partials, int N, int NS, int nb, float scale,
            const int *__restrict__ sel, size_t sel_stride, const c32 *__restrict__ tw) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    c32 *scr = reinterpret_cast<c32 *>(smem_raw);
    c32 *tile = scr + ((F::LS + 1) & ~1);
    const int t = threadIdx.x;
    if (sel) {
        x += (size_t)sel[0] * sel_stride;
        g += (size_t)sel[0] * sel_stride;
    }
    const int nbr = (N + 1) / 2, nblocks = nbr * ((nb + 1) / 2);
    // rows r0 (even) and r0 + 1 share a piece; r0 + 1 <= N < NS when it is
    // not an image row, and such a row is never read
    auto issue = [&](int bb) {
        const int q = bb / nbr, r0 = (bb - q * nbr) * 2;
        const c32 *Wq = W + (size_t)q * F::M * NS + r0;
        for (int pos = threadIdx.x; pos < F::M; pos += blockDim.x)
            cp_async16(tile + tslot<F, 2>(pos, 0), Wq + (size_t)pos * NS);
        cp_async_commit();
    };
    int b = blockIdx.x;
    if (b < nblocks) issue(b);
    for (; b < nblocks; b += gridDim.x) {
        const int q = b / nbr, rb = b - q * nbr, r0 = rb * 2;
        const bool has_b = 2 * q + 1 < nb;
        cp_async_wait_all();
        __syncthreads();  // tile in; the last block's transforms are done with the scratch
        double d[2] = {0.0, 0.0};
        auto finish_row = [&](c32 (&v)[16], int r) {
            F::template inverse<true>(v, scr, t, tw);
            const size_t oa = ((size_t)(2 * q) * N + r) * N;
            const size_t ob = ((size_t)(2 * q + 1) * N + r) * N;
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                if (!F::low_half(i)) continue;
                const int n = F::nidx(t, i);
                if (n < N) {
                    const float ha = v[i].x * scale, hb = v[i].y * scale;
                    const float aa = aty ? aty[oa + n] : 0.f;
                    const float ab = (aty && has_b) ? aty[ob + n] : 0.f;
                    if (partials) {
                        const float xva = x[oa + n];
                        d[0] += (double)xva * ha;
                        d[1] += (double)xva * aa;
                        if (has_b) {
                            const float xvb = x[ob + n];
                            d[0] += (double)xvb * hb;
                            d[1] += (double)xvb * ab;
                        }
                    }
                    g[oa + n] = ha - aa;
                    if (has_b) g[ob + n] = hb - ab;
                }
            }
        };
        {
            c32 v[16];
#pragma unroll
            for (int i = 0; i < 16; ++i) v[i] = tile[tslot<F, 2>(t * 16 + i, 0)];
            finish_row(v, r0);
        }
        if (r0 + 1 < N) {
            c32 v[16];
#pragma unroll
            for (int i = 0; i < 16; ++i) v[i] = tile[tslot<F, 2>(t * 16 + i, 1)];
            __syncthreads();  // tile read by all; the first row's transform is done with the scratch
            const int bn = b + gridDim.x;
            if (bn < nblocks) issue(bn);
            finish_row(v, r0 + 1);
        } else {
            __syncthreads();
            const int bn = b + gridDim.x;
            if (bn < nblocks) issue(bn);
        }
        if (partials) {
            block_sum<2>(d);
            if (threadIdx.x == 0) {
                double *dst = partials + ((size_t)q * nbr + rb) * 2;
                dst[0] = d[0];
                dst[1] = d[1];
            }
        }
    }
    cp_async_wait_all();
}

// pass 3 as k_tpf_out_s with the block's two rows transformed side by side:
// 2 F::T threads, group l (threads l F::T ..) takes row r0 + l with its own
// FFT scratch.  Every thread reads its inputs from the tile first, then the
// next block's tile is requested and both rows are transformed, so the copy
// overlaps both transforms and epilogues.  Same partial rows as k_tpf_out_s.
template <class F>
struct OutPar {
    static constexpr int SCR = (F::LS + 1) & ~1;
    static constexpr int TILE = 2 * F::M + 2 * (F::M / 16);
    static constexpr size_t SMEM = (size_t)(2 * SCR + TILE) * sizeof(c32);
    static constexpr bool FITS = SMEM <= 220 * 1024;
};

template <class F>
__global__ void __launch_bounds__(2 * F::T, 1)
k_tpf_out_p(const c32 *__restrict__ W, const float *x, const float *__restrict__ aty, float *g,
            double *__restrict__ partials, int N, int NS, int nb, float scale,
            const int *__restrict__ sel, size_t sel_stride, const c32 *__restrict__ tw) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    c32 *scr = reinterpret_cast<c32 *>(smem_raw);
    c32 *tile = scr + 2 * OutPar<F>::SCR;
    const int l = threadIdx.x / F::T, t = threadIdx.x % F::T;
    if (sel) {
        x += (size_t)sel[0] * sel_stride;
        g += (size_t)sel[0] * sel_stride;
    }
    const int nbr = (N + 1) / 2, nblocks = nbr * ((nb + 1) / 2);
    // rows r0 (even) and r0 + 1 share a piece; r0 + 1 <= N < NS when it is
    // not an image row, and such a row is never stored
    auto issue = [&](int bb) {
        const int q = bb / nbr, r0 = (bb - q * nbr) * 2;
        const c32 *Wq = W + (size_t)q * F::M * NS + r0;
        for (int pos = threadIdx.x; pos < F::M; pos += blockDim.x)
            cp_async16(tile + tslot<F, 2>(pos, 0), Wq + (size_t)pos * NS);
        cp_async_commit();
    };
    int b = blockIdx.x;
    if (b < nblocks) issue(b);
    for (; b < nblocks; b += gridDim.x) {
        const int q = b / nbr, rb = b - q * nbr, r = rb * 2 + l;
        const bool valid = r < N, has_b = 2 * q + 1 < nb;
        cp_async_wait_all();
        __syncthreads();  // tile in; the last block's transforms are done with the scratch
        c32 v[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) v[i] = tile[tslot<F, 2>(t * 16 + i, l)];
        __syncthreads();  // the tile is free: request the next block's
        const int bn = b + gridDim.x;
        if (bn < nblocks) issue(bn);
        if (t == 0 && valid) {
            // the epilogue's rows of x and aty into L2 during the transform
            const size_t rowb = (size_t)N * sizeof(float);
            const size_t oa = ((size_t)(2 * q) * N + r) * N, ob = oa + (size_t)N * N;
            if (partials) {
                prefetch_l2_range(x + oa, rowb);
                if (has_b) prefetch_l2_range(x + ob, rowb);
            }
            if (aty) {
                prefetch_l2_range(aty + oa, rowb);
                if (has_b) prefetch_l2_range(aty + ob, rowb);
            }
        }
        F::template inverse<true, true>(v, scr + l * OutPar<F>::SCR, t, tw);
        double d[2] = {0.0, 0.0};
        if (valid) {
            const size_t oa = ((size_t)(2 * q) * N + r) * N;
            const size_t ob = ((size_t)(2 * q + 1) * N + r) * N;
            // the epilogue's global reads first, all in flight together
            // (one memory latency per block rather than one per value)
            float xa[16], xb[16], aa[16], ab[16];
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                xa[i] = xb[i] = aa[i] = ab[i] = 0.f;
                if (!F::low_half(i)) continue;
                const int n = F::nidx(t, i);
                if (n >= N) continue;
                if (aty) {
                    aa[i] = aty[oa + n];
                    if (has_b) ab[i] = aty[ob + n];
                }
                if (partials) {
                    xa[i] = x[oa + n];
                    if (has_b) xb[i] = x[ob + n];
                }
            }
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                if (!F::low_half(i)) continue;
                const int n = F::nidx(t, i);
                if (n < N) {
                    const float ha = v[i].x * scale, hb = v[i].y * scale;
                    if (partials) {
                        d[0] += (double)xa[i] * ha;
                        d[1] += (double)xa[i] * aa[i];
                        if (has_b) {
                            d[0] += (double)xb[i] * hb;
                            d[1] += (double)xb[i] * ab[i];
                        }
                    }
                    g[oa + n] = ha - aa[i];
                    if (has_b) g[ob + n] = hb - ab[i];
                }
            }
        }
        if (partials) {
            block_sum<2>(d);
            if (threadIdx.x == 0) {
                double *dst = partials + ((size_t)q * nbr + rb) * 2;
                dst[0] = d[0];
                dst[1] = d[1];
            }
        }
    }
    cp_async_wait_all();
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
static int run_fast(Plan &pl, const float *x, const float *aty, float *g, int nb,
                    double *partials, cudaStream_t st, const int *sel, size_t sel_stride) {
    using S = FastShape<F>;
    const int N = pl.N, NS = toe_stride(N);
    const int npairs = (nb + 1) / 2;
    TC_TRY(pl.ws_toe.reserve((size_t)npairs * F::M * NS * sizeof(c32)));
    c32 *W = pl.ws_toe.as<c32>();
    const c32 *tw = pl.fft_M.dev.tw;
    // passes 1 and 3: staging tile + image rows of one block (N <= M / 2)
    const size_t sm_rows = (size_t)S::SM_ROWS * sizeof(c32) + (size_t)S::LPC * 2 * ((N + 3) & ~3) * sizeof(float);
    const size_t sm_cols = ((size_t)S::SCR_COLS + (size_t)S::LC * NS) * sizeof(c32);
    auto k1 = k_tpf_rows<F, S::LPC>;
    auto k2 = k_tpf_cols<F, S::LC>;
    // pass 3: double-buffered tiles where they fit; else two rows per block,
    // side by side (k_tpf_out_p) or one after the other (k_tpf_out_s)
    constexpr bool PAR = S::SIMPLE_OUT && OutPar<F>::FITS;
    auto k3 = []() {
        if constexpr (PAR) return k_tpf_out_p<F>;
        else if constexpr (S::SIMPLE_OUT) return k_tpf_out_s<F>;
        else return k_tpf_out<F, S::LPC_OUT>;
    }();
    const size_t sm_out =
        PAR ? OutPar<F>::SMEM
        : S::SIMPLE_OUT
            ? ((size_t)((F::LS + 1) & ~1) + 2 * F::M + 2 * (F::M / 16)) * sizeof(c32)
            : ((size_t)S::SCR_OUT + S::TILE_OUT) * sizeof(c32) +
                  (size_t)2 * S::LPC_OUT * 2 * ((N + 3) & ~3) * sizeof(float);
    const int nt3 = PAR ? 2 * F::T : S::SIMPLE_OUT ? F::T : S::NT_OUT;
    TC_CUDA(cudaFuncSetAttribute(k1, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_rows));
    TC_CUDA(cudaFuncSetAttribute(k2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_cols));
    TC_CUDA(cudaFuncSetAttribute(k3, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_out));
    // the shared-memory carveout the occupancy below assumes, stated so that
    // launches from a graph get the same split
    TC_CUDA(cudaFuncSetAttribute(k1, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 cudaSharedmemCarveoutMaxShared));
    TC_CUDA(cudaFuncSetAttribute(k2, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 cudaSharedmemCarveoutMaxShared));
    TC_CUDA(cudaFuncSetAttribute(k3, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 cudaSharedmemCarveoutMaxShared));
    int dev = 0, nsm = 0, occ1 = 0, occ2 = 0, occ3 = 0;
    TC_CUDA(cudaGetDevice(&dev));
    TC_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    TC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ1, k1, S::NT_ROWS, sm_rows));
    TC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ2, k2, F::T * S::LC, sm_cols));
    TC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ3, k3, nt3, sm_out));
    if (occ1 < 1 || occ2 < 1 || occ3 < 1)
        TC_FAIL(TC_ERR_STATE, "a Toeplitz pass does not fit on an SM");
    const int nitems = F::M * npairs;
    const int nblocks = ceil_div(N, S::LPC) * npairs;
    k1<<<std::min(nblocks, nsm * occ1), S::NT_ROWS, sm_rows, st>>>(x, W, N, NS, nb, sel,
                                                                   sel_stride, tw);
    TC_LAUNCH_CHECK();
    k2<<<std::min(nitems, nsm * occ2), F::T * S::LC, sm_cols, st>>>(W, pl.d_phatp.as<float>(), N,
                                                                    NS, npairs, tw);
    TC_LAUNCH_CHECK();
    const float scale = (float)(1.0 / ((double)F::M * F::M * std::pow((double)N, 3)));
    const int nblocks3 = ceil_div(N, S::LPC_OUT) * npairs;
    const dim3 grid3 = dim3(std::min(nblocks3, nsm * occ3));
    k3<<<grid3, nt3, sm_out, st>>>(W, x, aty, g, partials, N, NS, nb, scale, sel, sel_stride,
                                         tw);
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

bool toeplitz_fast_supported(int M) {
    return M == 64 || M == 128 || M == 256 || M == 512 || M == 1024 || M == 1536 || M == 2048 ||
           M == 3072 || M == 4096 || M == 6144 || M == 8192;
}

int toeplitz_fast_lpc(int M) {
    switch (M) {
        case 64: return FastShape<F64>::LPC_OUT;
        case 128: return FastShape<F128>::LPC_OUT;
        case 256: return FastShape<F256>::LPC_OUT;
        case 512: return FastShape<F512>::LPC_OUT;
        case 1024: return FastShape<F1024>::LPC_OUT;
        case 1536: return FastShape<F1536>::LPC_OUT;
        case 2048: return FastShape<F2048>::LPC_OUT;
        case 3072: return FastShape<F3072>::LPC_OUT;
        case 4096: return FastShape<F4096>::LPC_OUT;
        case 6144: return FastShape<F6144>::LPC_OUT;
        case 8192: return FastShape<F8192>::LPC_OUT;
        default: return 1;
    }
}

int toeplitz_fast_row_block(int M) {
    switch (M) {
        case 64: return FastShape<F64>::LPC;
        case 128: return FastShape<F128>::LPC;
        case 256: return FastShape<F256>::LPC;
        case 512: return FastShape<F512>::LPC;
        case 1024: return FastShape<F1024>::LPC;
        case 1536: return FastShape<F1536>::LPC;
        case 2048: return FastShape<F2048>::LPC;
        case 3072: return FastShape<F3072>::LPC;
        case 4096: return FastShape<F4096>::LPC;
        case 6144: return FastShape<F6144>::LPC;
        case 8192: return FastShape<F8192>::LPC;
        default: return 1;
    }
}

size_t toeplitz_fast_pair_bytes(int N, int M) { return (size_t)M * toe_stride(N) * sizeof(c32); }

int toeplitz_fast_chunk(Plan &pl, const float *x, const float *aty, float *g, int nb,
                        double *partials, cudaStream_t st, const int *sel, size_t sel_stride) {
    switch (pl.M) {
        case 64: return run_fast<F64>(pl, x, aty, g, nb, partials, st, sel, sel_stride);
        case 128: return run_fast<F128>(pl, x, aty, g, nb, partials, st, sel, sel_stride);
        case 256: return run_fast<F256>(pl, x, aty, g, nb, partials, st, sel, sel_stride);
        case 512: return run_fast<F512>(pl, x, aty, g, nb, partials, st, sel, sel_stride);
        case 1024: return run_fast<F1024>(pl, x, aty, g, nb, partials, st, sel, sel_stride);
        case 1536: return run_fast<F1536>(pl, x, aty, g, nb, partials, st, sel, sel_stride);
        case 2048: return run_fast<F2048>(pl, x, aty, g, nb, partials, st, sel, sel_stride);
        case 3072: return run_fast<F3072>(pl, x, aty, g, nb, partials, st, sel, sel_stride);
        case 4096: return run_fast<F4096>(pl, x, aty, g, nb, partials, st, sel, sel_stride);
        case 6144: return run_fast<F6144>(pl, x, aty, g, nb, partials, st, sel, sel_stride);
        case 8192: return run_fast<F8192>(pl, x, aty, g, nb, partials, st, sel, sel_stride);
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
        case 1536: return perm_fast<F1536>(pl, st);
        case 2048: return perm_fast<F2048>(pl, st);
        case 3072: return perm_fast<F3072>(pl, st);
        case 4096: return perm_fast<F4096>(pl, st);
        case 6144: return perm_fast<F6144>(pl, st);
        case 8192: return perm_fast<F8192>(pl, st);
        default: TC_FAIL(TC_ERR_STATE, "no register FFT for this Toeplitz size");
    }
}

}  // namespace tc
