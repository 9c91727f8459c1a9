// tc_mbir.cu -- device-resident MBIR iteration (Optimizer::run2,
// src/optimize.h:96-154, with the gradient and objective of
// src/mbir2.cpp:122-136).
//
// One backtracking attempt is four launches:
//   begin   beta = tnew (1/t - 1), tnew = theta(t)              (1 thread)
//   update  y = sol + beta (sol - x), Hy = (1+beta) H sol - beta H x,
//           g = Hy - A^T y + w * qGGMRF'(y), new = y - step g, partial sums
//           of y.Hy, y.A^Ty, g.g, new.A^Ty, |new - x|^2 (FP32 over 8 slices
//           per voxel column, FP64 from there on)             (fused stencil;
//           specialised for x == sol, the attempt after an accepted step)
//   H new   Toeplitz passes, FP64 partials of new.H new
//   decide  sqrt f(new) > sqrt f(y) + step/2 |g|^2 ? shrink step, retry from
//           new : accept (x = sol = new), record, count      (1 CTA)
// H is linear, so H y never needs its own transform: every attempt costs one
// Toeplitz application.  The iterate, H-image and scalar state live on the
// device; three rotating buffers hold x, sol and the new iterate, and the
// kernels read which is which from the state, so the whole solve can run as
// one CUDA graph whose WHILE node repeats the attempt until the requested
// number of iterations has been accepted.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "tc_mbir.cuh"

namespace tc {

__global__ void k_mbir_begin(MbirState *s) { mbir_begin(s); }

// Both forms are launched every attempt and the one that does not apply
// returns at once (x == sol after an accepted step, x != sol after a
// rejected one), so each gets its own register allocation.
// tmap (use_tma != 0): the three iterate buffers as one [3 S][R][C] float
// tensor with a 72 x 34 x 1 box, for the x == sol form's plane tiles.
template <bool SAME>
__global__ void __launch_bounds__(UT, UPD_MIN_BLOCKS)
k_mbir_update(float *__restrict__ X, const float *__restrict__ H, const float *__restrict__ aty,
              int S, int R, int C, size_t vol, PriorParams pp, const MbirState *__restrict__ st,
              double *__restrict__ partials, const __grid_constant__ CUtensorMap tmap, int use_tma) {
    if ((st->ix == st->isol) != SAME) return;
    double *part = partials + ((size_t)blockIdx.y * gridDim.x + blockIdx.x) * NU;
    const int c0 = blockIdx.x * UX, r0 = blockIdx.y * UY;
    update_body<SAME>(X, H, aty, S, R, C, vol, pp, st, part, c0, r0, 0, 1 << 30,
                      use_tma ? &tmap : nullptr);
}

// The tensor map of the iterate buffers for the update's plane tiles, or
// false where a tensor copy cannot serve (rows not a multiple of 16 bytes,
// no driver entry point): the update then uses cp.async pieces.
static bool iterate_tensor_map(CUtensorMap *map, float *X, int S, int R, int C) {
    using Encode = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
    static Encode encode = [] {
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) !=
                cudaSuccess || q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            return (Encode) nullptr;
        }
        return reinterpret_cast<Encode>(fn);
    }();
    if (!encode || C % 4 != 0 || (reinterpret_cast<uintptr_t>(X) & 15) != 0) return false;
    const cuuint64_t dims[3] = {(cuuint64_t)C, (cuuint64_t)R, (cuuint64_t)3 * S};
    const cuuint64_t strides[2] = {(cuuint64_t)C * sizeof(float), (cuuint64_t)R * C * sizeof(float)};
    const cuuint32_t box[3] = {(cuuint32_t)PW, (cuuint32_t)PH, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    static_assert((PW * sizeof(float)) % 16 == 0 && PW <= 256 && PH <= 256, "tensor-copy box");
    return encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, X, dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                  CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

__global__ void k_mbir_decide(MbirState *s, const double *__restrict__ pu, int nu,
                              const double *__restrict__ pt, int nt, double *__restrict__ hist,
                              cudaGraphConditionalHandle handle, int use_graph) {
    double u[NU + 1] = {0, 0, 0, 0, 0, 0};
    for (int i = threadIdx.x; i < nu; i += blockDim.x)
#pragma unroll
        for (int k = 0; k < NU; ++k) u[k] += pu[(size_t)i * NU + k];
    for (int i = threadIdx.x; i < nt; i += blockDim.x) u[NU] += pt[(size_t)i * 2];
    block_sum<NU + 1>(u);
    if (threadIdx.x != 0) return;
    const int cond = mbir_decide_core(s, u, hist);
    if (use_graph) cudaGraphSetConditional(handle, cond);
}

// ---------------------------------------------------------------------------
// host driver
// ---------------------------------------------------------------------------
struct MbirRun {
    Plan *pl;
    int S;
    size_t vol;
    float *X, *H;
    const float *aty;
    MbirState *st;
    double *pu, *pt, *hist;
    int nu, nt;
    PriorParams pp;
    CUtensorMap tmap;  // iterate buffers, for the update's plane tiles
    int use_tma;
};

// ev (host loop only, may be NULL): events recorded before the update, after
// it, after the Toeplitz passes and after the decision
static int enqueue_attempt(MbirRun &m, cudaStream_t s, cudaGraphConditionalHandle h, int use_graph,
                           cudaEvent_t *ev = nullptr) {
    Plan &pl = *m.pl;
    const int N = pl.N;
    k_mbir_begin<<<1, 1, 0, s>>>(m.st);
    TC_LAUNCH_CHECK();
    if (ev) TC_CUDA(cudaEventRecord(ev[0], s));
    dim3 grid(ceil_div(N, UX), ceil_div(N, UY));
    k_mbir_update<true><<<grid, UT, UPD_SMEM, s>>>(m.X, m.H, m.aty, m.S, N, N, m.vol, m.pp, m.st,
                                                   m.pu, m.tmap, m.use_tma);
    TC_LAUNCH_CHECK();
    k_mbir_update<false><<<grid, UT, UPD_SMEM, s>>>(m.X, m.H, m.aty, m.S, N, N, m.vol, m.pp, m.st,
                                                    m.pu, m.tmap, 0);
    TC_LAUNCH_CHECK();
    if (ev) TC_CUDA(cudaEventRecord(ev[1], s));
    const int chunk = 2 * pl.toe_pairs;
    int off = 0;
    for (int c0 = 0; c0 < m.S; c0 += chunk) {
        const int nb = std::min(chunk, m.S - c0);
        const size_t o = (size_t)c0 * N * N;
        TC_TRY(toeplitz_chunk(pl, m.X + o, nullptr, m.H + o, nb, m.pt + (size_t)off * 2, s,
                              &m.st->inew, m.vol));
        off += toeplitz_partials_count(pl, nb);
    }
    if (ev) TC_CUDA(cudaEventRecord(ev[2], s));
    k_mbir_decide<<<1, 1024, 0, s>>>(m.st, m.pu, m.nu, m.pt, m.nt, m.hist, h, use_graph);
    TC_LAUNCH_CHECK();
    if (ev) TC_CUDA(cudaEventRecord(ev[3], s));
    return TC_OK;
}

// CUDA events for the host loop's phase times, destroyed on every path
struct PhaseEvents {
    cudaEvent_t e[4] = {nullptr, nullptr, nullptr, nullptr};
    int create() {
        for (auto &x : e) TC_CUDA(cudaEventCreate(&x));
        return TC_OK;
    }
    ~PhaseEvents() {
        for (auto &x : e)
            if (x) cudaEventDestroy(x);
    }
};

struct GraphGuard {
    cudaGraph_t g = nullptr;
    cudaGraphExec_t e = nullptr;
    ~GraphGuard() {
        if (e) cudaGraphExecDestroy(e);
        if (g) cudaGraphDestroy(g);
    }
};

int mbir_solve(Plan &pl, const float *aty, double sino_sq, float *x, int S,
               const tc_mbir_opts &o, double *history, cudaStream_t st) {
    const int N = pl.N;
    const size_t vol = (size_t)S * N * N;
    MbirRun m;
    m.pl = &pl;
    m.S = S;
    m.vol = vol;
    m.aty = aty;
    m.nu = ceil_div(N, UX) * ceil_div(N, UY);
    // two CTAs per SM need 2 x UPD_SMEM of the unified L1 / shared array;
    // state the carveout so launches from a graph get the same split
    TC_CUDA(cudaFuncSetAttribute(k_mbir_update<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, UPD_SMEM));
    TC_CUDA(cudaFuncSetAttribute(k_mbir_update<true>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 cudaSharedmemCarveoutMaxShared));
    TC_CUDA(cudaFuncSetAttribute(k_mbir_update<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, UPD_SMEM));
    TC_CUDA(cudaFuncSetAttribute(k_mbir_update<false>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 cudaSharedmemCarveoutMaxShared));
    int nt = 0;
    for (int c0 = 0; c0 < S; c0 += 2 * pl.toe_pairs)
        nt += toeplitz_partials_count(pl, std::min(2 * pl.toe_pairs, S - c0));
    m.nt = nt;
    m.pp = make_prior(o.sigma, o.p, o.prior_weight);
    const int K = std::max(0, (int)o.num_iters);

    // workspace: 3 iterates, 3 H-images, partials, state, history
    const size_t bytes_vol = 6 * vol * sizeof(float);
    const size_t bytes_red = ((size_t)m.nu * NU + (size_t)nt * 2 + 3 * (size_t)std::max(K, 1)) * sizeof(double);
    TC_TRY(pl.ws_red.reserve(bytes_vol + bytes_red + sizeof(MbirState) + 256));
    char *base = pl.ws_red.as<char>();
    m.X = reinterpret_cast<float *>(base);
    m.H = m.X + 3 * vol;
    m.pu = reinterpret_cast<double *>(base + bytes_vol);
    m.pt = m.pu + (size_t)m.nu * NU;
    m.hist = m.pt + (size_t)nt * 2;
    m.st = reinterpret_cast<MbirState *>(base + ((bytes_vol + bytes_red + 255) / 256) * 256);
    std::memset(&m.tmap, 0, sizeof m.tmap);
    m.use_tma = iterate_tensor_map(&m.tmap, m.X, S, N, N) ? 1 : 0;

    MbirState h{};
    h.t = 1.0;
    h.tnew = 1.0;
    double step = o.step > 0 ? (double)o.step : 1.0 / pl.lipschitz;
    if (!(o.step > 0) && step > 1.0) step = 1.0;
    h.step = h.step0 = step;
    h.sino_sq = sino_sq;
    h.ix = h.isol = 0;
    h.inew = 1;
    h.num_iters = K;
    h.max_attempts = o.max_attempts > 0 ? o.max_attempts : 1000;
    h.cond = K > 0 ? 1 : 0;
    TC_CUDA(cudaMemcpyAsync(m.st, &h, sizeof(h), cudaMemcpyHostToDevice, st));
    TC_CUDA(cudaMemcpyAsync(m.X, x, vol * sizeof(float), cudaMemcpyDeviceToDevice, st));
    // H x0
    const int chunk = 2 * pl.toe_pairs;
    for (int c0 = 0; c0 < S; c0 += chunk) {
        const int nb = std::min(chunk, S - c0);
        const size_t off = (size_t)c0 * N * N;
        TC_TRY(toeplitz_chunk(pl, m.X + off, nullptr, m.H + off, nb, nullptr, st));
    }
    if (K > 0) {
        if (o.use_graph) {
            // the arguments the captured kernels hold: device addresses, sizes
            // and the prior parameters (by value)
            struct Key {
                const void *X, *H, *aty, *st, *pu, *pt, *hist, *toe;
                size_t vol;
                int S, nu, nt, toe_pairs;
                PriorParams pp;
            } key;
            std::memset(&key, 0, sizeof key);
            key.X = m.X;
            key.H = m.H;
            key.aty = m.aty;
            key.st = m.st;
            key.pu = m.pu;
            key.pt = m.pt;
            key.hist = m.hist;
            key.toe = pl.ws_toe.ptr;
            key.vol = m.vol;
            key.S = S;
            key.nu = m.nu;
            key.nt = m.nt;
            key.toe_pairs = pl.toe_pairs;
            key.pp = m.pp;
            const unsigned char *kb = reinterpret_cast<const unsigned char *>(&key);
            const bool hit = pl.solver_e && pl.solver_key.size() == sizeof key &&
                             std::memcmp(pl.solver_key.data(), kb, sizeof key) == 0;
            if (!hit) {
                if (pl.solver_e) cudaGraphExecDestroy(pl.solver_e);
                if (pl.solver_g) cudaGraphDestroy(pl.solver_g);
                pl.solver_e = nullptr;
                pl.solver_g = nullptr;
                pl.solver_key.clear();
                GraphGuard gg;
                TC_CUDA(cudaGraphCreate(&gg.g, 0));
                cudaGraphConditionalHandle hd;
                TC_CUDA(cudaGraphConditionalHandleCreate(&hd, gg.g, 1, cudaGraphCondAssignDefault));
                cudaGraphNodeParams cp = {};
                cp.type = cudaGraphNodeTypeConditional;
                cp.conditional.handle = hd;
                cp.conditional.type = cudaGraphCondTypeWhile;
                cp.conditional.size = 1;
                cudaGraphNode_t node;
                TC_CUDA(cudaGraphAddNode(&node, gg.g, nullptr, 0, &cp));
                cudaGraph_t body = cp.conditional.phGraph_out[0];
                TC_CUDA(cudaStreamBeginCaptureToGraph(pl.aux, body, nullptr, nullptr, 0,
                                                      cudaStreamCaptureModeRelaxed));
                int rc = enqueue_attempt(m, pl.aux, hd, 1);
                cudaGraph_t captured = nullptr;
                cudaError_t ec = cudaStreamEndCapture(pl.aux, &captured);
                if (rc != TC_OK) return rc;
                TC_CUDA(ec);
                TC_CUDA(cudaGraphInstantiate(&gg.e, gg.g, 0));
                pl.solver_g = gg.g;
                pl.solver_e = gg.e;
                gg.g = nullptr;
                gg.e = nullptr;
                pl.solver_key.assign(kb, kb + sizeof key);
            }
            cudaEvent_t ev = nullptr;
            TC_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
            cudaError_t e = cudaEventRecord(ev, st);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(pl.aux, ev, 0);
            if (e == cudaSuccess) e = cudaGraphLaunch(pl.solver_e, pl.aux);
            if (e == cudaSuccess) e = cudaEventRecord(ev, pl.aux);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(st, ev, 0);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            cudaEventDestroy(ev);
            TC_CUDA(e);
        } else {
            PhaseEvents pe;
            double phase[4] = {0.0, 0.0, 0.0, 0.0};
            if (o.phase_ms) TC_TRY(pe.create());
            int *cond_host = nullptr;
            TC_CUDA(cudaMallocHost(&cond_host, sizeof(int)));
            int rc = TC_OK;
            for (;;) {
                rc = enqueue_attempt(m, st, 0, 0, o.phase_ms ? pe.e : nullptr);
                if (rc != TC_OK) break;
                cudaError_t e = cudaMemcpyAsync(cond_host, &m.st->cond, sizeof(int),
                                                cudaMemcpyDeviceToHost, st);
                if (e == cudaSuccess) e = cudaStreamSynchronize(st);
                if (e == cudaSuccess && o.phase_ms) {
                    float t[3] = {0.f, 0.f, 0.f};
                    for (int q = 0; q < 3 && e == cudaSuccess; ++q)
                        e = cudaEventElapsedTime(&t[q], pe.e[q], pe.e[q + 1]);
                    for (int q = 0; q < 3; ++q) phase[q] += t[q];
                    phase[3] += 1.0;
                }
                if (e != cudaSuccess) {
                    set_error(std::string("CUDA error: ") + cudaGetErrorString(e));
                    rc = TC_ERR_CUDA;
                    break;
                }
                if (!*cond_host) break;
            }
            cudaFreeHost(cond_host);
            if (rc != TC_OK) return rc;
            if (o.phase_ms) std::copy(phase, phase + 4, o.phase_ms);
        }
    }
    TC_CUDA(cudaMemcpyAsync(&h, m.st, sizeof(h), cudaMemcpyDeviceToHost, st));
    TC_CUDA(cudaStreamSynchronize(st));
    TC_CUDA(cudaMemcpyAsync(x, m.X + (size_t)h.ix * vol, vol * sizeof(float),
                            cudaMemcpyDeviceToDevice, st));
    std::vector<double> hist(3 * (size_t)std::max(K, 1), 0.0);
    if (K > 0)
        TC_CUDA(cudaMemcpyAsync(hist.data(), m.hist, 3 * (size_t)K * sizeof(double),
                                cudaMemcpyDeviceToHost, st));
    TC_CUDA(cudaStreamSynchronize(st));
    if (history && K > 0) std::copy(hist.begin(), hist.begin() + 3 * K, history);
    if (o.verbose)
        for (int it = 0; it < h.iter; ++it)
            std::fprintf(stdout, "iter: %4d, error: %5.4e, x-err: %5.4e\n", it, hist[3 * it],
                         hist[3 * it + 1]);
    if (h.status == UPD_STATUS_TMA_TIMEOUT)
        TC_FAIL(TC_ERR_TIMEOUT, "a bounded device wait for a plane tile gave up at iteration " +
                                    std::to_string(h.iter));
    if (h.status == 1)
        TC_FAIL(TC_ERR_TIMEOUT, "backtracking found no acceptable step within max_attempts "
                                "attempts at iteration " + std::to_string(h.iter));
    return TC_OK;
}

}  // namespace tc
