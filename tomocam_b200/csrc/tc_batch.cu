// tc_batch.cu -- batched MBIR over independent scans of uneven size.
//
// Every scan keeps the single-volume solver's state machine (MbirState,
// Optimizer::run2 of src/optimize.h:96-154: its own beta/theta, step,
// backtracking and iteration count) and its own buffers; what is shared is
// the launch.  One attempt of all running scans is
//   begin    one thread per scan
//   update   one CTA per (scan, 32 x 16 tile): the fused stencil + Nesterov
//            update body of the single-volume solver
//   rows     one CTA per (scan, slice pair, block of rows)   \  Toeplitz H new,
//   cols     one CTA per (scan, slice pair, block of columns) | register FFT of
//   out      one CTA per (scan, slice pair, block of rows)   /  the scan's size
//   decide   one CTA per scan: reduce, step test, bookkeeping
//   cond     one thread: continue while any scan runs
// so the launch count per attempt does not grow with the number of scans,
// and the loop runs as one CUDA graph (WHILE node) or from the host.  A scan
// that has finished (or hit its attempt cap) makes its CTAs return at once.
// The Toeplitz CTAs pick the register FFT of their scan's size at run time
// (512 threads: 512 / (M / 16) lines per CTA for every size M = 64 .. 4096).
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "tc_fft_fast.cuh"
#include "tc_mbir.cuh"

namespace tc {

// device descriptor of one scan
struct BScan {
    int N, M, NS, S;       // image width, Toeplitz size, workspace stride, slices
    int npairs, nbr;       // slice pairs; row blocks of the rows/out passes
    int ntx, nty;          // update tiles across / down
    int pu_base, nu;       // this scan's rows of the update partials
    int pt_base, nt;       // this scan's entries of the Toeplitz partials
    size_t vol;            // S N N
    float *X, *H;          // 3 iterates, 3 H-images (each vol floats)
    const float *aty;
    c32 *W;                // Toeplitz workspace [npairs][M][NS]
    const float *phatp;    // PSF spectrum in register-FFT order [M][M]
    const c32 *tw;         // twiddles of length M
    float scale;           // 1 / (M^2 N^3)
    PriorParams pp;
    MbirState *st;
    double *hist;          // [num_iters][3]
};

constexpr int BT = 512;  // threads per CTA of the batched Toeplitz passes

template <class F>
struct BShape {
    static constexpr int L = BT / F::T;  // lines per CTA
    static constexpr int STAGE = L * F::M + F::M / 16;
    static constexpr int SMEM = (L * F::LS > STAGE) ? L * F::LS : STAGE;  // complex
};

using B64 = FastFFT<4, 4, 4>;
using B128 = FastFFT<8, 4, 4>;
using B256 = FastFFT<8, 8, 4>;
using B512 = FastFFT<2, 16, 16>;
using B1024 = FastFFT<4, 16, 16>;
using B2048 = FastFFT<8, 16, 16>;
using B4096 = FastFFT<16, 16, 16>;

constexpr int cmax(int a, int b) { return a > b ? a : b; }
constexpr int BT_SMEM_C =
    cmax(cmax(cmax(BShape<B64>::SMEM, BShape<B128>::SMEM), cmax(BShape<B256>::SMEM, BShape<B512>::SMEM)),
         cmax(cmax(BShape<B1024>::SMEM, BShape<B2048>::SMEM), BShape<B4096>::SMEM));
constexpr int BT_SMEM = BT_SMEM_C * (int)sizeof(c32);

template <int L>
__device__ __forceinline__ int bstg(int pos, int l) { return pos * L + l + (pos >> 4); }

// ---- Toeplitz pass bodies (one CTA, L lines) -------------------------------
template <class F>
__device__ __forceinline__ void brows(const BScan &d, int q, int rb, c32 *sm) {
    constexpr int L = BShape<F>::L;
    const int l = threadIdx.x / F::T, t = threadIdx.x % F::T;
    const int N = d.N, r0 = rb * L, r = r0 + l;
    const bool valid = r < N;
    const float *x = d.X + (size_t)d.st->inew * d.vol;
    const float *xa = x + ((size_t)(2 * q) * N + (valid ? r : 0)) * N;
    const float *xb = (2 * q + 1 < d.S) ? x + ((size_t)(2 * q + 1) * N + (valid ? r : 0)) * N : nullptr;
    c32 v[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        v[i] = mk<float>(0.f, 0.f);
        if (!F::low_half(i)) continue;
        const int n = F::nidx(t, i);
        if (valid && n < N) v[i] = mk<float>(xa[n], xb ? xb[n] : 0.f);
    }
    F::template forward<true>(v, sm + l * F::LS, t, d.tw);
    __syncthreads();
#pragma unroll
    for (int i = 0; i < 16; ++i) sm[bstg<L>(t * 16 + i, l)] = v[i];
    __syncthreads();
    c32 *Wq = d.W + (size_t)q * F::M * d.NS + r0;
    for (int e = threadIdx.x; e < F::M * L; e += BT) {
        const int pos = e / L, ll = e % L;
        if (r0 + ll < N) Wq[(size_t)pos * d.NS + ll] = sm[bstg<L>(pos, ll)];
    }
}

template <class F>
__device__ __forceinline__ void bcols(const BScan &d, int q, int pg, c32 *sm) {
    constexpr int L = BShape<F>::L;
    const int l = threadIdx.x / F::T, t = threadIdx.x % F::T;
    // with more lines per CTA than columns (M = 64) the surplus lines only
    // take part in the barriers
    const int N = d.N, pos = pg * L + l;
    const bool valid = pos < F::M;
    c32 *col = d.W + ((size_t)q * F::M + (valid ? pos : 0)) * d.NS;
    c32 v[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        v[i] = mk<float>(0.f, 0.f);
        if (!F::low_half(i)) continue;
        const int n = F::nidx(t, i);
        if (valid && n < N) v[i] = col[n];
    }
    F::template forward<true>(v, sm + l * F::LS, t, d.tw);
    const float4 *ph = reinterpret_cast<const float4 *>(d.phatp + (size_t)(valid ? pos : 0) * F::M + t * 16);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const float4 p = __ldg(ph + i);
        v[4 * i + 0] = v[4 * i + 0] * p.x;
        v[4 * i + 1] = v[4 * i + 1] * p.y;
        v[4 * i + 2] = v[4 * i + 2] * p.z;
        v[4 * i + 3] = v[4 * i + 3] * p.w;
    }
    F::sync_before_inverse();
    F::inverse(v, sm + l * F::LS, t, d.tw);
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        if (!F::low_half(i)) continue;
        const int n = F::nidx(t, i);
        if (valid && n < N) col[n] = v[i];
    }
}

// H new = scale * inverse rows; partial new.H new per CTA
template <class F>
__device__ __forceinline__ void bout(const BScan &d, int q, int rb, c32 *sm, double *pt) {
    constexpr int L = BShape<F>::L;
    const int l = threadIdx.x / F::T, t = threadIdx.x % F::T;
    const int N = d.N, r0 = rb * L, r = r0 + l;
    const bool valid = r < N, has_b = 2 * q + 1 < d.S;
    const c32 *Wq = d.W + (size_t)q * F::M * d.NS + r0;
    for (int e = threadIdx.x; e < F::M * L; e += BT) {
        const int pos = e / L, ll = e % L;
        sm[bstg<L>(pos, ll)] = (r0 + ll < N) ? Wq[(size_t)pos * d.NS + ll] : mk<float>(0.f, 0.f);
    }
    __syncthreads();
    c32 v[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = sm[bstg<L>(t * 16 + i, l)];
    __syncthreads();
    F::inverse(v, sm + l * F::LS, t, d.tw);
    const size_t off = (size_t)d.st->inew * d.vol;
    const float *x = d.X + off;
    float *g = d.H + off;
    const size_t oa = ((size_t)(2 * q) * N + (valid ? r : 0)) * N;
    const size_t ob = ((size_t)(2 * q + 1) * N + (valid ? r : 0)) * N;
    double acc[1] = {0.0};
#pragma unroll
    for (int i = 0; i < 16; ++i) {
        if (!F::low_half(i)) continue;
        const int n = F::nidx(t, i);
        if (valid && n < N) {
            const float ha = v[i].x * d.scale, hb = v[i].y * d.scale;
            g[oa + n] = ha;
            acc[0] += (double)x[oa + n] * ha;
            if (has_b) {
                g[ob + n] = hb;
                acc[0] += (double)x[ob + n] * hb;
            }
        }
    }
    block_sum<1>(acc, threadIdx.x, BT);
    if (threadIdx.x == 0) *pt = acc[0];
}

#define BDISPATCH(M, CALL)                                                   \
    switch (M) {                                                             \
        case 64: CALL(B64); break;                                           \
        case 128: CALL(B128); break;                                         \
        case 256: CALL(B256); break;                                         \
        case 512: CALL(B512); break;                                         \
        case 1024: CALL(B1024); break;                                       \
        case 2048: CALL(B2048); break;                                       \
        default: CALL(B4096); break; /* M = 4096; other sizes are refused */ \
    }

// items: {scan, slice pair, block}
__global__ void __launch_bounds__(BT, 2) k_batch_rows(const BScan *__restrict__ scans,
                                                     const int4 *__restrict__ items) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    c32 *sm = reinterpret_cast<c32 *>(smem_raw);
    const int4 it = items[blockIdx.x];
    const BScan &d = scans[it.x];
    if (!d.st->cond) return;
#define CALL_ROWS(F) brows<F>(d, it.y, it.z, sm)
    BDISPATCH(d.M, CALL_ROWS)
#undef CALL_ROWS
}

__global__ void __launch_bounds__(BT, 1) k_batch_cols(const BScan *__restrict__ scans,
                                                     const int4 *__restrict__ items) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    c32 *sm = reinterpret_cast<c32 *>(smem_raw);
    const int4 it = items[blockIdx.x];
    const BScan &d = scans[it.x];
    if (!d.st->cond) return;
#define CALL_COLS(F) bcols<F>(d, it.y, it.z, sm)
    BDISPATCH(d.M, CALL_COLS)
#undef CALL_COLS
}

__global__ void __launch_bounds__(BT, 2) k_batch_out(const BScan *__restrict__ scans,
                                                    const int4 *__restrict__ items,
                                                    double *__restrict__ pt) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    c32 *sm = reinterpret_cast<c32 *>(smem_raw);
    const int4 it = items[blockIdx.x];
    const BScan &d = scans[it.x];
    if (!d.st->cond) return;
    double *dst = pt + d.pt_base + (size_t)it.y * d.nbr + it.z;
#define CALL_OUT(F) bout<F>(d, it.y, it.z, sm, dst)
    BDISPATCH(d.M, CALL_OUT)
#undef CALL_OUT
}
#undef BDISPATCH

// items: {scan, tile x, tile y}
__global__ void __launch_bounds__(UT, UPD_MIN_BLOCKS) k_batch_update(const BScan *__restrict__ scans,
                                                       const int4 *__restrict__ items,
                                                       double *__restrict__ pu) {
    const int4 it = items[blockIdx.x];
    const BScan &d = scans[it.x];
    const MbirState *st = d.st;
    if (!st->cond) return;
    double *part = pu + ((size_t)d.pu_base + (size_t)it.z * d.ntx + it.y) * NU;
    const int c0 = it.y * UX, r0 = it.z * UY;
    if (st->ix == st->isol)
        update_body<true>(d.X, d.H, d.aty, d.S, d.N, d.N, d.vol, d.pp, st, part, c0, r0);
    else
        update_body<false>(d.X, d.H, d.aty, d.S, d.N, d.N, d.vol, d.pp, st, part, c0, r0);
}

__global__ void k_batch_begin(const BScan *__restrict__ scans, int nscans) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < nscans && scans[s].st->cond) mbir_begin(scans[s].st);
}

__global__ void k_batch_decide(const BScan *__restrict__ scans, const double *__restrict__ pu,
                               const double *__restrict__ pt) {
    const BScan &d = scans[blockIdx.x];
    if (!d.st->cond) return;
    double u[NU + 1] = {0, 0, 0, 0, 0, 0};
    const double *a = pu + (size_t)d.pu_base * NU;
    for (int i = threadIdx.x; i < d.nu; i += blockDim.x)
#pragma unroll
        for (int k = 0; k < NU; ++k) u[k] += a[(size_t)i * NU + k];
    for (int i = threadIdx.x; i < d.nt; i += blockDim.x) u[NU] += pt[d.pt_base + i];
    block_sum<NU + 1>(u);
    if (threadIdx.x == 0) mbir_decide_core(d.st, u, d.hist);
}

__global__ void k_batch_cond(const BScan *__restrict__ scans, int nscans, int *any,
                             cudaGraphConditionalHandle handle, int use_graph) {
    int c = 0;
    for (int s = threadIdx.x; s < nscans; s += blockDim.x) c |= scans[s].st->cond;
    c = __syncthreads_or(c);
    if (threadIdx.x == 0) {
        *any = c;
        if (use_graph) cudaGraphSetConditional(handle, c ? 1u : 0u);
    }
}

// ---------------------------------------------------------------------------
// host driver
// ---------------------------------------------------------------------------
struct BatchRun {
    const BScan *scans;
    const int4 *upd, *rows, *cols, *out;
    int nscans, nupd, nrows, ncols, nout;
    double *pu, *pt;
    int *any;
};

static int enqueue_batch(const BatchRun &b, cudaStream_t s, cudaGraphConditionalHandle h,
                         int use_graph) {
    k_batch_begin<<<ceil_div(b.nscans, 128), 128, 0, s>>>(b.scans, b.nscans);
    TC_LAUNCH_CHECK();
    k_batch_update<<<b.nupd, UT, UPD_SMEM, s>>>(b.scans, b.upd, b.pu);
    TC_LAUNCH_CHECK();
    k_batch_rows<<<b.nrows, BT, BT_SMEM, s>>>(b.scans, b.rows);
    TC_LAUNCH_CHECK();
    k_batch_cols<<<b.ncols, BT, BT_SMEM, s>>>(b.scans, b.cols);
    TC_LAUNCH_CHECK();
    k_batch_out<<<b.nout, BT, BT_SMEM, s>>>(b.scans, b.out, b.pt);
    TC_LAUNCH_CHECK();
    k_batch_decide<<<b.nscans, 256, 0, s>>>(b.scans, b.pu, b.pt);
    TC_LAUNCH_CHECK();
    k_batch_cond<<<1, 256, 0, s>>>(b.scans, b.nscans, b.any, h, use_graph);
    TC_LAUNCH_CHECK();
    return TC_OK;
}

static int lines_per_cta(int M) { return BT / (M / 16); }

int mbir_batched(const std::vector<BatchScanIn> &in, int num_iters, int use_graph,
                 int max_attempts, double *history, cudaStream_t st) {
    const int ns = (int)in.size();
    const int K = std::max(0, num_iters);
    if (ns == 0) return TC_OK;
    for (int i = 0; i < ns; ++i) {
        const BatchScanIn &s = in[i];
        if (!s.pl->toe_fast || s.pl->M > 4096 || (s.pl->M & (s.pl->M - 1)) != 0)
            TC_FAIL(TC_ERR_SHAPE, "scan " + std::to_string(i) +
                                      ": the batched solver needs a power-of-two Toeplitz size "
                                      "<= 4096 (n <= 2048; create the plan with "
                                      "TC_PLAN_POW2_TOEPLITZ for n of 513 .. 768 or 1025 .. 1536)");
        if (!s.pl->d_phat.ptr)
            TC_FAIL(TC_ERR_STATE, "scan " + std::to_string(i) + ": plan has no point-spread function");
        if (s.S < 1) TC_FAIL(TC_ERR_SHAPE, "scan " + std::to_string(i) + ": nslices < 1");
        if (!(s.sigma > 0) || !(s.p > 0 && s.p <= 2))
            TC_FAIL(TC_ERR_ARG, "scan " + std::to_string(i) + ": sigma must be > 0, p in (0, 2]");
    }
    // layout of one allocation: per scan X[3], H[3], W; then partials, states,
    // histories, descriptors, items
    std::vector<BScan> d(ns);
    std::vector<int4> upd, rows, cols, outs;
    size_t floats = 0, complexes = 0;
    int pu_n = 0, pt_n = 0;
    for (int i = 0; i < ns; ++i) {
        const Plan &pl = *in[i].pl;
        BScan &b = d[i];
        b.N = pl.N;
        b.M = pl.M;
        b.NS = (pl.N + 3) & ~3;
        b.S = in[i].S;
        b.npairs = (b.S + 1) / 2;
        const int L = lines_per_cta(b.M);
        b.nbr = ceil_div(b.N, L);
        b.ntx = ceil_div(b.N, UX);
        b.nty = ceil_div(b.N, UY);
        b.vol = (size_t)b.S * b.N * b.N;
        b.nu = b.ntx * b.nty;
        b.pu_base = pu_n;
        pu_n += b.nu;
        b.nt = b.npairs * b.nbr;
        b.pt_base = pt_n;
        pt_n += b.nt;
        floats += 6 * b.vol;
        complexes += (size_t)b.npairs * b.M * b.NS;
        b.scale = (float)(1.0 / ((double)b.M * b.M * std::pow((double)b.N, 3)));
        b.pp = make_prior(in[i].sigma, in[i].p, in[i].weight);
        b.phatp = pl.d_phatp.as<float>();
        b.tw = pl.fft_M.dev.tw;
        b.aty = in[i].aty;
        for (int ty = 0; ty < b.nty; ++ty)
            for (int tx = 0; tx < b.ntx; ++tx) upd.push_back(make_int4(i, tx, ty, 0));
        for (int q = 0; q < b.npairs; ++q) {
            for (int rb = 0; rb < b.nbr; ++rb) {
                rows.push_back(make_int4(i, q, rb, 0));
                outs.push_back(make_int4(i, q, rb, 0));
            }
            for (int pg = 0; pg < ceil_div(b.M, L); ++pg) cols.push_back(make_int4(i, q, pg, 0));
        }
    }
    auto al = [](size_t b) { return (b + 255) & ~size_t(255); };
    const size_t b_c = al(complexes * sizeof(c32)), b_f = al(floats * sizeof(float));
    const size_t b_pu = al((size_t)pu_n * NU * sizeof(double)), b_pt = al((size_t)pt_n * sizeof(double));
    const size_t b_st = al(ns * sizeof(MbirState)), b_h = al((size_t)ns * 3 * std::max(K, 1) * sizeof(double));
    const size_t b_d = al(ns * sizeof(BScan));
    const size_t b_i = al((upd.size() + rows.size() + cols.size() + outs.size()) * sizeof(int4));
    DevBuf buf;
    TC_TRY(buf.reserve(b_c + b_f + b_pu + b_pt + b_st + b_h + b_d + b_i + 256));
    char *base = buf.as<char>();
    c32 *Wall = reinterpret_cast<c32 *>(base);
    float *Fall = reinterpret_cast<float *>(base + b_c);
    double *pu = reinterpret_cast<double *>(base + b_c + b_f);
    double *pt = reinterpret_cast<double *>(base + b_c + b_f + b_pu);
    MbirState *sts = reinterpret_cast<MbirState *>(base + b_c + b_f + b_pu + b_pt);
    double *hist = reinterpret_cast<double *>(base + b_c + b_f + b_pu + b_pt + b_st);
    BScan *dd = reinterpret_cast<BScan *>(base + b_c + b_f + b_pu + b_pt + b_st + b_h);
    int4 *items = reinterpret_cast<int4 *>(base + b_c + b_f + b_pu + b_pt + b_st + b_h + b_d);
    int *any = reinterpret_cast<int *>(base + b_c + b_f + b_pu + b_pt + b_st + b_h + b_d + b_i);

    std::vector<MbirState> hs(ns);
    size_t fo = 0, co = 0;
    for (int i = 0; i < ns; ++i) {
        BScan &b = d[i];
        Plan &pl = *in[i].pl;
        b.X = Fall + fo;
        b.H = b.X + 3 * b.vol;
        fo += 6 * b.vol;
        b.W = Wall + co;
        co += (size_t)b.npairs * b.M * b.NS;
        b.st = sts + i;
        b.hist = hist + (size_t)i * 3 * std::max(K, 1);
        MbirState &h = hs[i];
        h = MbirState{};
        h.t = h.tnew = 1.0;
        double step = in[i].step > 0 ? (double)in[i].step : 1.0 / pl.lipschitz;
        if (!(in[i].step > 0) && step > 1.0) step = 1.0;
        h.step = h.step0 = step;
        h.sino_sq = in[i].sino_sq;
        h.ix = h.isol = 0;
        h.inew = 1;
        h.num_iters = K;
        h.max_attempts = max_attempts > 0 ? max_attempts : 1000;
        h.cond = K > 0 ? 1 : 0;
        TC_CUDA(cudaMemcpyAsync(b.X, in[i].x, b.vol * sizeof(float), cudaMemcpyDeviceToDevice, st));
        // H x0 on the scan's own plan (set-up; per scan)
        const int chunk = 2 * pl.toe_pairs;
        for (int c0 = 0; c0 < b.S; c0 += chunk) {
            const int nb = std::min(chunk, b.S - c0);
            const size_t off = (size_t)c0 * b.N * b.N;
            TC_TRY(toeplitz_chunk(pl, b.X + off, nullptr, b.H + off, nb, nullptr, st));
        }
    }
    TC_CUDA(cudaMemcpyAsync(sts, hs.data(), ns * sizeof(MbirState), cudaMemcpyHostToDevice, st));
    TC_CUDA(cudaMemcpyAsync(dd, d.data(), ns * sizeof(BScan), cudaMemcpyHostToDevice, st));
    std::vector<int4> all;
    all.insert(all.end(), upd.begin(), upd.end());
    all.insert(all.end(), rows.begin(), rows.end());
    all.insert(all.end(), cols.begin(), cols.end());
    all.insert(all.end(), outs.begin(), outs.end());
    TC_CUDA(cudaMemcpyAsync(items, all.data(), all.size() * sizeof(int4), cudaMemcpyHostToDevice, st));
    // the host vectors above are read by the copies: finish them before return
    BatchRun r;
    r.scans = dd;
    r.nscans = ns;
    r.upd = items;
    r.nupd = (int)upd.size();
    r.rows = r.upd + upd.size();
    r.nrows = (int)rows.size();
    r.cols = r.rows + rows.size();
    r.ncols = (int)cols.size();
    r.out = r.cols + cols.size();
    r.nout = (int)outs.size();
    r.pu = pu;
    r.pt = pt;
    r.any = any;
    if (r.nupd > INT32_MAX / 2 || r.ncols > INT32_MAX / 2) TC_FAIL(TC_ERR_SHAPE, "batch too large");

    for (const void *k : {(const void *)k_batch_rows, (const void *)k_batch_cols,
                          (const void *)k_batch_out}) {
        TC_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, BT_SMEM));
        TC_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout,
                                     cudaSharedmemCarveoutMaxShared));
    }
    TC_CUDA(cudaFuncSetAttribute(k_batch_update, cudaFuncAttributeMaxDynamicSharedMemorySize, UPD_SMEM));
    TC_CUDA(cudaFuncSetAttribute(k_batch_update, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 cudaSharedmemCarveoutMaxShared));
    TC_CUDA(cudaStreamSynchronize(st));

    if (K > 0) {
        if (use_graph) {
            Plan &pl0 = *in[0].pl;
            cudaEvent_t ev = nullptr;
            TC_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
            struct EvGuard {
                cudaEvent_t e;
                ~EvGuard() { if (e) cudaEventDestroy(e); }
            } eg{ev};
            TC_CUDA(cudaEventRecord(ev, st));
            TC_CUDA(cudaStreamWaitEvent(pl0.aux, ev, 0));
            cudaGraph_t g = nullptr;
            cudaGraphExec_t ge = nullptr;
            struct GGuard {
                cudaGraph_t &g;
                cudaGraphExec_t &e;
                ~GGuard() {
                    if (e) cudaGraphExecDestroy(e);
                    if (g) cudaGraphDestroy(g);
                }
            } gg{g, ge};
            TC_CUDA(cudaGraphCreate(&g, 0));
            cudaGraphConditionalHandle hd;
            TC_CUDA(cudaGraphConditionalHandleCreate(&hd, g, 1, cudaGraphCondAssignDefault));
            cudaGraphNodeParams cp = {};
            cp.type = cudaGraphNodeTypeConditional;
            cp.conditional.handle = hd;
            cp.conditional.type = cudaGraphCondTypeWhile;
            cp.conditional.size = 1;
            cudaGraphNode_t node;
            TC_CUDA(cudaGraphAddNode(&node, g, nullptr, 0, &cp));
            cudaGraph_t body = cp.conditional.phGraph_out[0];
            TC_CUDA(cudaStreamBeginCaptureToGraph(pl0.aux, body, nullptr, nullptr, 0,
                                                  cudaStreamCaptureModeRelaxed));
            int rc = enqueue_batch(r, pl0.aux, hd, 1);
            cudaGraph_t captured = nullptr;
            cudaError_t ec = cudaStreamEndCapture(pl0.aux, &captured);
            if (rc != TC_OK) return rc;
            TC_CUDA(ec);
            TC_CUDA(cudaGraphInstantiate(&ge, g, 0));
            TC_CUDA(cudaGraphLaunch(ge, pl0.aux));
            TC_CUDA(cudaEventRecord(ev, pl0.aux));
            TC_CUDA(cudaStreamWaitEvent(st, ev, 0));
            TC_CUDA(cudaStreamSynchronize(st));
        } else {
            int *any_host = nullptr;
            TC_CUDA(cudaMallocHost(&any_host, sizeof(int)));
            struct HGuard {
                int *p;
                ~HGuard() { cudaFreeHost(p); }
            } hg{any_host};
            for (;;) {
                TC_TRY(enqueue_batch(r, st, 0, 0));
                TC_CUDA(cudaMemcpyAsync(any_host, any, sizeof(int), cudaMemcpyDeviceToHost, st));
                TC_CUDA(cudaStreamSynchronize(st));
                if (!*any_host) break;
            }
        }
    }
    TC_CUDA(cudaMemcpyAsync(hs.data(), sts, ns * sizeof(MbirState), cudaMemcpyDeviceToHost, st));
    TC_CUDA(cudaStreamSynchronize(st));
    for (int i = 0; i < ns; ++i)
        TC_CUDA(cudaMemcpyAsync(in[i].x, d[i].X + (size_t)hs[i].ix * d[i].vol, d[i].vol * sizeof(float),
                                cudaMemcpyDeviceToDevice, st));
    if (history && K > 0)
        for (int i = 0; i < ns; ++i)
            TC_CUDA(cudaMemcpyAsync(history + (size_t)i * 3 * K, d[i].hist, 3 * (size_t)K * sizeof(double),
                                    cudaMemcpyDeviceToHost, st));
    TC_CUDA(cudaStreamSynchronize(st));
    for (int i = 0; i < ns; ++i)
        if (hs[i].status == 1)
            TC_FAIL(TC_ERR_TIMEOUT, "scan " + std::to_string(i) +
                                        ": backtracking found no acceptable step within "
                                        "max_attempts attempts at iteration " +
                                        std::to_string(hs[i].iter));
    return TC_OK;
}

}  // namespace tc
