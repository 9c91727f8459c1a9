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
           const c32 *__restrict__ tw) {
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
            const float cr = corr[r] * scale;
            float *dst = out + ((size_t)b * N + r) * N;
            const float *sb = sub ? sub + ((size_t)b * N + r) * N : nullptr;
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                const int c = mode_of<F::M>(F::nidx(t, i), N);
                if (c >= 0) {
                    float val = v[i].x * corr[c] * cr;
                    if (sb) val -= sb[c];
                    dst[c] = val;
                }
            }
        }
    }
    cp_async_wait_all();
}

template <class F>
int run_t1f(const c32 *G, c32 *Rw, float *out, const float *sub, const float *corr, float scale,
            int N, int nb, const c32 *tw, cudaStream_t st) {
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
                                                                     N, NS, nb, tw);
    TC_LAUNCH_CHECK();
    return TC_OK;
}

}  // namespace

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

int t1_fast_fft(const c32 *G, c32 *Rw, float *out, const float *sub, const float *corr,
                float scale, int N, int nf, int nb, const c32 *tw, cudaStream_t st) {
    switch (nf) {
        case 64: return run_t1f<F64>(G, Rw, out, sub, corr, scale, N, nb, tw, st);
        case 128: return run_t1f<F128>(G, Rw, out, sub, corr, scale, N, nb, tw, st);
        case 256: return run_t1f<F256>(G, Rw, out, sub, corr, scale, N, nb, tw, st);
        case 512: return run_t1f<F512>(G, Rw, out, sub, corr, scale, N, nb, tw, st);
        case 1024: return run_t1f<F1024>(G, Rw, out, sub, corr, scale, N, nb, tw, st);
        case 1536: return run_t1f<F1536>(G, Rw, out, sub, corr, scale, N, nb, tw, st);
        case 2048: return run_t1f<F2048>(G, Rw, out, sub, corr, scale, N, nb, tw, st);
        case 3072: return run_t1f<F3072>(G, Rw, out, sub, corr, scale, N, nb, tw, st);
        case 4096: return run_t1f<F4096>(G, Rw, out, sub, corr, scale, N, nb, tw, st);
        case 6144: return run_t1f<F6144>(G, Rw, out, sub, corr, scale, N, nb, tw, st);
        default: TC_FAIL(TC_ERR_STATE, "no register FFT for this fine grid");
    }
}

}  // namespace tc
