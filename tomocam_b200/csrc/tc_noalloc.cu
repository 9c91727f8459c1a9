// tc_noalloc.cu -- the Toeplitz gradient for callers that cannot allocate
// device memory.
//
// Who needs it: applications whose own memory pool owns the GPU's memory --
// a framework's caching allocator, or a real-time pipeline that reserves all
// of HBM at start-up -- and that forbid a library to call cudaMalloc behind
// their back: such a call may fail because the pool already holds the
// memory, and cudaMalloc/cudaFree may synchronise the device in the middle of
// the caller's pipeline.  tc_toeplitz_grad grows a workspace inside its plan
// on demand; this entry point instead uses a fixed scratch array that is
// part of the loaded library image, and calls no cudaMalloc, cudaFree or
// allocating library routine.
//
// Limits and sharing:
//   * the scratch array is NOALLOC_SCRATCH_BYTES (32 MiB) per device.  One
//     slice pair needs N * M * 8 bytes of workspace plus 16 N bytes of
//     partial sums (M = the plan's FFT size, M >= 2N - 1), so every image up
//     to 1024 x 1024 fits (M <= 2048); larger plans fit only while that sum
//     stays within the scratch, and are rejected with TC_ERR_SHAPE otherwise
//     (the message gives the bytes needed and available).
//   * it runs the general FFT engine's three passes, not the register-FFT
//     kernels tc_toeplitz_grad uses for M <= 8192, so it is slower; results
//     agree within FP32 rounding.
//   * every GPU that loads the library holds the array until the process
//     exits.
//   * all calls share the one array and it keeps the last call's contents:
//     two calls whose work overlaps on the GPU (different streams, or
//     different host threads) race on it.  Serialise them on one stream.
//   * the first call on a device looks up the array's device address
//     (cudaGetSymbolAddress) once; make that first call before any stream
//     capture begins.
//   * with xhx or xaty non-NULL the call copies the two sums to the host and
//     synchronises the stream before it returns.
#include <atomic>
#include <cmath>

#include "tc_plan.cuh"

namespace tc {

constexpr size_t NOALLOC_SCRATCH_BYTES = 32u << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

// Toeplitz passes, defined in tc_toeplitz.cu
__global__ void __launch_bounds__(FFT_MAX_THREADS, 1)
k_tp_rows(const float *__restrict__ x, c32 *__restrict__ W, int N, int nb,
          const int *__restrict__ sel, size_t sel_stride, FftDev<float> dM);
__global__ void __launch_bounds__(FFT_MAX_THREADS, 1)
k_tp_cols(c32 *__restrict__ W, const float *__restrict__ phat, int N, int cw, FftDev<float> dM);
__global__ void __launch_bounds__(FFT_MAX_THREADS, 1)
k_tp_out(const c32 *__restrict__ W, const float *x, const float *__restrict__ aty, float *g,
         double *__restrict__ partials, int N, int nb, float scale, const int *__restrict__ sel,
         size_t sel_stride, FftDev<float> dM);

// acc[v] += sum of nparts rows of nvals doubles (one CTA, fixed order)
__global__ void k_accum_partials(const double *__restrict__ in, int nparts, int nvals,
                                 double *__restrict__ acc) {
    for (int v = 0; v < nvals; ++v) {
        double s[1] = {0.0};
        for (int i = threadIdx.x; i < nparts; i += blockDim.x) s[0] += in[(size_t)i * nvals + v];
        block_sum<1>(s);
        if (threadIdx.x == 0) acc[v] += s[0];
        __syncthreads();
    }
}

constexpr int NOALLOC_MAX_DEVICES = 64;
static std::atomic<void *> g_scratch_ptr[NOALLOC_MAX_DEVICES];

// device address of the scratch array on the current device (looked up once)
static int scratch_address(void **out) {
    int dev = 0;
    TC_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) TC_FAIL(TC_ERR_STATE, "device ordinal out of range");
    void *p = g_scratch_ptr[dev].load();
    if (!p) {
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            TC_FAIL(TC_ERR_CUDA, std::string("cudaGetSymbolAddress of the scratch array failed: ") +
                                     cudaGetErrorString(e));
        }
        g_scratch_ptr[dev].store(p);
    }
    *out = p;
    return TC_OK;
}

static int toeplitz_noalloc(Plan &pl, const float *x, const float *aty, float *g, int nslices,
                            double *xhx, double *xaty, cudaStream_t st) {
    const int N = pl.N, M = pl.M;
    // scratch layout: [0, 256) two FP64 accumulators, then per-chunk partials
    // (2 doubles per image row of each pair), then the [pairs][N][M] workspace
    const size_t pair_ws = (size_t)N * M * sizeof(c32);
    const size_t pair_parts = (size_t)N * 2 * sizeof(double);
    const size_t avail = NOALLOC_SCRATCH_BYTES - 256;
    size_t pairs = avail / (pair_ws + pair_parts + 256);
    if (pairs < 1)
        TC_FAIL(TC_ERR_SHAPE, "image too large for the no-allocation scratch: one slice pair at N = " +
                                  std::to_string(N) + " (FFT size M = " + std::to_string(M) +
                                  ") needs " + std::to_string(pair_ws + pair_parts + 256) +
                                  " bytes, " + std::to_string(avail) + " are available (every N <= " +
                                  "1024 fits)");
    if (!pl.d_phat.ptr)
        TC_FAIL(TC_ERR_STATE, "plan has no point-spread function (created with TC_PLAN_NO_PSF)");
    pairs = std::min<size_t>(pairs, (size_t)((nslices + 1) / 2 > 0 ? (nslices + 1) / 2 : 1));
    void *base = nullptr;
    TC_TRY(scratch_address(&base));
    char *b = static_cast<char *>(base);
    double *acc = reinterpret_cast<double *>(b);
    double *parts = reinterpret_cast<double *>(b + 256);
    const size_t parts_bytes = ((pairs * pair_parts + 255) / 256) * 256;
    c32 *W = reinterpret_cast<c32 *>(b + 256 + parts_bytes);
    if (256 + parts_bytes + pairs * pair_ws > NOALLOC_SCRATCH_BYTES)
        TC_FAIL(TC_ERR_STATE, "scratch layout overflow");

    const bool dots = (xhx || xaty);
    if (dots) TC_CUDA(cudaMemsetAsync(acc, 0, 2 * sizeof(double), st));
    const int nthr1 = fft_threads<float>(M, 1);
    const size_t smem1 = (size_t)M * sizeof(c32);
    int cw = 4;
    while (cw > 1 && ((size_t)cw * M * sizeof(c32) > 128 * 1024 ||
                      fft_threads<float>(M, cw) > FFT_MAX_THREADS || M % cw))
        cw /= 2;
    const int nthr2 = fft_threads<float>(M, cw);
    const size_t smem2 = (size_t)cw * M * sizeof(c32);
    TC_CUDA(cudaFuncSetAttribute(k_tp_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem1));
    TC_CUDA(cudaFuncSetAttribute(k_tp_out, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem1));
    TC_CUDA(cudaFuncSetAttribute(k_tp_cols, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem2));
    const float scale = (float)(1.0 / ((double)M * M * std::pow((double)N, 3)));
    const size_t vs = (size_t)N * N;
    const int chunk = 2 * (int)pairs;
    for (int b0 = 0; b0 < nslices; b0 += chunk) {
        const int nb = std::min(chunk, nslices - b0);
        const int np = (nb + 1) / 2;
        const float *xc = x + b0 * vs;
        k_tp_rows<<<dim3(N, np), nthr1, smem1, st>>>(xc, W, N, nb, nullptr, 0, pl.fft_M.dev);
        TC_LAUNCH_CHECK();
        k_tp_cols<<<dim3(M / cw, np), nthr2, smem2, st>>>(W, pl.d_phat.as<float>(), N, cw,
                                                          pl.fft_M.dev);
        TC_LAUNCH_CHECK();
        k_tp_out<<<dim3(N, np), nthr1, smem1, st>>>(W, xc, aty ? aty + b0 * vs : nullptr,
                                                    g + b0 * vs, dots ? parts : nullptr, N, nb,
                                                    scale, nullptr, 0, pl.fft_M.dev);
        TC_LAUNCH_CHECK();
        if (dots) {
            k_accum_partials<<<1, 1024, 0, st>>>(parts, np * N, 2, acc);
            TC_LAUNCH_CHECK();
        }
    }
    if (dots) {
        double h[2] = {0.0, 0.0};
        TC_CUDA(cudaMemcpyAsync(h, acc, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
        TC_CUDA(cudaStreamSynchronize(st));
        if (xhx) *xhx = h[0];
        if (xaty) *xaty = h[1];
    }
    return TC_OK;
}

}  // namespace tc

extern "C" int tc_toeplitz_grad_noalloc(tc_plan *plan, const float *x, const float *aty,
                                        float *g, int nslices, double *xhx, double *xaty,
                                        tc_stream_t stream) {
    return tc::guarded([&]() -> int {
        if (!plan || (nslices > 0 && (!x || !g)))
            TC_FAIL(TC_ERR_ARG, "NULL argument to tc_toeplitz_grad_noalloc");
        if (nslices < 0) TC_FAIL(TC_ERR_SHAPE, "nslices < 0");
        if (nslices == 0) {
            if (xhx) *xhx = 0.0;
            if (xaty) *xaty = 0.0;
            return TC_OK;
        }
        return tc::toeplitz_noalloc(plan->impl, x, aty, g, nslices, xhx, xaty,
                                    reinterpret_cast<cudaStream_t>(stream));
    });
}
