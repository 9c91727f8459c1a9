// tc_capi.cu -- the extern "C" boundary (include/tomocam_b200.h).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "tc_plan.cuh"
#include "tc_prep.cuh"

namespace tc {

// Phase timing of tc_mbir_host and plan_build: with TC_TRACE set in the
// environment, each phase ends with a device synchronisation and its wall time is written to
// stderr as "tc_trace <phase> <ms>"; unset, nothing is synchronised.
namespace {
struct PhaseTrace {
    bool on = std::getenv("TC_TRACE") != nullptr;
    std::chrono::steady_clock::time_point t = std::chrono::steady_clock::now();
    void mark(const char *phase) {
        if (!on) return;
        cudaDeviceSynchronize();
        const auto n = std::chrono::steady_clock::now();
        std::fprintf(stderr, "tc_trace %s %.3f\n", phase,
                     std::chrono::duration<double, std::milli>(n - t).count());
        t = n;
    }
};
}  // namespace


static thread_local std::string g_last_error;
void set_error(const std::string &msg) { g_last_error = msg; }
const char *last_error() { return g_last_error.c_str(); }

static int g_num_gpus = 1;

size_t Plan::table_bytes() const {
    return d_cs.bytes + d_sn.bytes + d_corr.bytes + fft_D.bytes() + fft_nf.bytes() +
           fft_M.bytes() + spread.points.bytes + spread.subs.bytes + spread.shared_tiles.bytes +
           d_psf.bytes + d_phat.bytes + d_phatp.bytes + fft_det_tw.bytes() + d_det_chirp.bytes +
           d_det_bhat.bytes + bands.entries.bytes + bands.chunks.bytes + bands.shared_bands.bytes +
           itiles.entries.bytes + itiles.subs.bytes;
}
size_t Plan::workspace_bytes() const {
    return ws_grid.bytes + ws_rows.bytes + ws_pts.bytes + ws_toe.bytes + ws_red.bytes +
           ws_scalars.bytes;
}
Plan::~Plan() {
    if (solver_e) cudaGraphExecDestroy(solver_e);
    if (solver_g) cudaGraphDestroy(solver_g);
    if (aux) cudaStreamDestroy(aux);
}

// Toeplitz workspace per chunk of slice pairs.  The passes are bound by FP32
// issue, not HBM: streaming the [N][M] complex intermediate of all pairs
// through HBM needs ~1.3 TB/s at 2048^2, well under the peak, so each pass
// covers as many pairs as this budget allows in one launch (few launches,
// few graph nodes) rather than one L2-resident pair at a time.
constexpr size_t TOE_CHUNK_BYTES = size_t(8) << 30;

int plan_build(Plan &pl, const tc_geom &g) {
    if (g.n < 4) TC_FAIL(TC_ERR_SHAPE, "n must be >= 4");
    if (g.nproj < 1) TC_FAIL(TC_ERR_SHAPE, "nproj must be >= 1");
    if (!g.angles) TC_FAIL(TC_ERR_ARG, "angles is NULL");
    if (g.flags & ~(TC_PLAN_NO_PSF | TC_PLAN_AUTOTUNE | TC_PLAN_POW2_TOEPLITZ | TC_PLAN_UNPAIRED))
        TC_FAIL(TC_ERR_ARG, "unknown flags");
    if (g.n > 8192) TC_FAIL(TC_ERR_SHAPE, "n > 8192 is not supported");
    for (int p = 0; p < g.nproj; ++p)
        if (!std::isfinite(g.angles[p])) TC_FAIL(TC_ERR_NAN, "angles contain a non-finite value");
    const double tol = g.nufft_tol > 0 ? g.nufft_tol : 1e-6;
    if (tol < 1e-14 || tol >= 1.0) TC_FAIL(TC_ERR_ARG, "nufft_tol must be in [1e-14, 1)");
    pl.N = g.n;
    pl.P = g.nproj;
    pl.es.set(tol);
    pl.es64.set(1e-12);
    // fine grid: the smallest register-FFT length >= 2N (upsampling factor
    // 2 .. 2.7; the ES kernel's accuracy only improves above 2), else the
    // smallest even 2,3,5,7-smooth size on the general engine
    pl.nf = t1_fast_grid(pl.N);
    if (pl.nf == 0) pl.nf = next_smooth_even(2 * pl.N);
    // Toeplitz FFT size: the smallest register-FFT length >= 2N-1 (powers of
    // two and 1536, 3072, 6144 -- or powers of two only with
    // TC_PLAN_POW2_TOEPLITZ; any M >= 2N-1 gives the same linear
    // convolution); larger images use the smallest 2,3,5,7-smooth size on
    // the general engine
    int m2 = 64;
    while (m2 < 2 * pl.N - 1) m2 *= 2;
    if (!(g.flags & TC_PLAN_POW2_TOEPLITZ))
        for (int m3 : {1536, 3072, 6144})
            if (2 * pl.N - 1 <= m3 && m3 < m2) m2 = m3;
    pl.M = toeplitz_fast_supported(m2) ? m2 : next_smooth(2 * pl.N - 1);
    pl.toe_fast = toeplitz_fast_supported(pl.M);
    pl.toe_lpc = pl.toe_fast ? toeplitz_fast_lpc(pl.M) : 1;
    pl.angles.assign(g.angles, g.angles + g.nproj);
    TC_CUDA(cudaStreamCreateWithFlags(&pl.aux, cudaStreamNonBlocking));
    cudaStream_t st = pl.aux;

    std::vector<double> cs(pl.P), sn(pl.P);
    for (int p = 0; p < pl.P; ++p) {
        cs[p] = std::cos((double)pl.angles[p]);
        sn[p] = std::sin((double)pl.angles[p]);
    }
    TC_TRY(pl.d_cs.reserve(pl.P * sizeof(double)));
    TC_TRY(pl.d_sn.reserve(pl.P * sizeof(double)));
    TC_CUDA(cudaMemcpy(pl.d_cs.ptr, cs.data(), pl.P * sizeof(double), cudaMemcpyHostToDevice));
    TC_CUDA(cudaMemcpy(pl.d_sn.ptr, sn.data(), pl.P * sizeof(double), cudaMemcpyHostToDevice));
    pl.geo.P = pl.P;
    pl.geo.D = pl.N;
    pl.geo.half = pl.N / 2;
    pl.geo.s = 2.0 * M_PI / (double)(pl.N - 1);
    pl.geo.cs = pl.d_cs.as<double>();
    pl.geo.sn = pl.d_sn.as<double>();

    std::vector<double> corr = es_correction(pl.N, pl.nf, pl.es);
    std::vector<float> corrf(corr.begin(), corr.end());
    TC_TRY(pl.d_corr.reserve(pl.N * sizeof(float)));
    TC_CUDA(cudaMemcpy(pl.d_corr.ptr, corrf.data(), pl.N * sizeof(float), cudaMemcpyHostToDevice));

    PhaseTrace tr;
    TC_TRY(pl.fft_D.init(pl.N));
    TC_TRY(pl.fft_nf.init(pl.nf));
    TC_TRY(pl.fft_M.init(pl.M));
    TC_TRY(det_fast_setup(pl));
    tr.mark("plan.fft_tables");
    // chunking
    const size_t pair_bytes = pl.toe_fast ? toeplitz_fast_pair_bytes(pl.N, pl.M)
                                          : (size_t)pl.N * pl.M * sizeof(c32);
    pl.toe_pairs = (int)std::max<size_t>(1, TOE_CHUNK_BYTES / pair_bytes);
    // Where a block of the first Toeplitz pass holds fewer than 4 image rows
    // (M = 6144, 8192), each block writes half of every 32-byte workspace
    // sector it touches and the neighbouring block the other half.  Measured
    // at N = 2908 (M = 6144), 256 slices: with chunks of 60 pairs that pass
    // took 0.22-0.24 ms per pair and varied from call to call (operator
    // 0.253-0.296 ms per slice), with chunks of 4-16 pairs 0.129 ms per pair
    // every time (operator 0.252-0.255); at M = 4096 (4-row blocks, whole
    // sectors) whole-volume chunks are the fastest.
    if (pl.toe_fast && toeplitz_fast_row_block(pl.M) < 4) pl.toe_pairs = std::min(pl.toe_pairs, 16);
    // paired NUFFT on the register-FFT path (two slices per complex line;
    // mirror points for even detector counts)
    pl.pair_nufft = !(g.flags & TC_PLAN_UNPAIRED) && pair_nufft_apply(pl);
    pl.nvirt = (pl.pair_nufft && pl.N % 2 == 0) ? pl.P : 0;
    const size_t slice_bytes = ((size_t)pl.nf * pl.nf + (size_t)pl.N * pl.nf +
                                pl.npts_ext()) * sizeof(c32);
    // NUFFT chunk: up to 8 lines within a 4 GiB workspace (the band
    // spreading loads each list entry and its kernel weights once per
    // chunk); a line is one slice, or two on the paired path
    const int per_line = pl.pair_nufft ? 2 : 1;
    int mb = (int)std::max<size_t>(1, (size_t(4) << 30) / slice_bytes);
    mb = std::min(mb, 8) * per_line;
    if (g.max_batch > 0) mb = std::min(g.max_batch, 8 * per_line);
    pl.max_batch = mb;
    // an explicit chunk size caps the Toeplitz chunk too (slice pairs)
    if (g.max_batch > 0) pl.toe_pairs = std::min(pl.toe_pairs, std::max(1, g.max_batch / 2));

    // type-1 spreading lists: measured choice of tile and sub-problem size,
    // or the default 32 x 32 tiles of at most 2048 points
    if (g.flags & TC_PLAN_AUTOTUNE) TC_TRY(spread_autotune(pl, cs, sn));
    else TC_TRY(pl.spread.build(pl.geo, cs, sn, pl.nf, pl.es.w, 2048, SPREAD_TILE));
    // bands of the register-FFT path (kernel widths <= 8)
    if (t1_fast_supported(pl.nf) && pl.es.w <= 8) {
        TC_TRY(pl.bands.build(pl.geo, pl.nf, pl.es.w, BAND_CHUNK, pl.nvirt));
        if (g.flags & TC_PLAN_AUTOTUNE) TC_TRY(band_autotune(pl));
    }
    // interpolation tiles of the register-FFT type-2 path
    if (interp_tiles_apply(pl)) {
        if (g.flags & TC_PLAN_AUTOTUNE) TC_TRY(interp_autotune(pl));
        else TC_TRY(pl.itiles.build(pl.geo, pl.nf, pl.es.w, INTERP_TILE, INTERP_POINTS, pl.nvirt));
    }
    tr.mark("plan.spread_lists");

    if (!(g.flags & TC_PLAN_NO_PSF)) {
        // point-spread function (FP64), its spectrum and max(H 1)
        const size_t nm = 2 * (size_t)pl.N - 1;
        TC_TRY(pl.d_psf.reserve(nm * nm * sizeof(double)));
        TC_TRY(psf_fp64(pl, cs, sn, pl.d_psf.as<double>(), st));
        tr.mark("plan.psf_fp64");
        TC_TRY(psf_finish(pl));
        tr.mark("plan.psf_spectrum_lipschitz");
    }
    TC_CUDA(cudaStreamSynchronize(st));
    return TC_OK;
}

// spectrum of d_psf and the Lipschitz constant max(H 1) (src/mbir2.cpp:100-112)
int psf_finish(Plan &pl) {
    cudaStream_t st = pl.aux;
    TC_TRY(phat_from_psf(pl, pl.d_psf.as<double>(), st));
    if (pl.toe_fast) TC_TRY(toeplitz_fast_permute(pl, st));
    const size_t n2 = (size_t)pl.N * pl.N;
    // max(H 1), formed and reduced on the device
    DevBuf ones, h1;
    TC_TRY(ones.reserve(n2 * sizeof(float)));
    TC_TRY(h1.reserve(n2 * sizeof(float)));
    TC_TRY(fill_dev(ones.as<float>(), n2, 1.0f, st));
    TC_TRY(toeplitz_chunk(pl, ones.as<float>(), nullptr, h1.as<float>(), 1, nullptr, st));
    float m = 0.f;
    TC_TRY(max_sumsq_dev(h1.as<float>(), n2, &m, nullptr, st));
    pl.lipschitz = m;
    return TC_OK;
}

static int need_psf(const Plan &pl) {
    if (!pl.d_phat.ptr)
        TC_FAIL(TC_ERR_STATE, "plan has no point-spread function (created with TC_PLAN_NO_PSF)");
    return TC_OK;
}

static cudaStream_t S_(tc_stream_t s) { return reinterpret_cast<cudaStream_t>(s); }

// RAII device allocation for the host entry points
struct DevArr {
    DevBuf b;
    template <typename T>
    int alloc(size_t n) {
        return b.reserve(std::max<size_t>(n, 1) * sizeof(T));
    }
    template <typename T>
    T *p() const {
        return b.as<T>();
    }
};

}  // namespace tc

using namespace tc;

extern "C" {

const char *tc_last_error_string(void) { return last_error(); }
const char *tc_version(void) { return "tomocam-b200 0.1.0"; }

int tc_release_cached_memory(void) {
    return guarded([&]() -> int {
        DevCache::get().flush();
        return TC_OK;
    });
}

int tc_plan_create(const tc_geom *geom, tc_plan **out) {
    return guarded([&]() -> int {
        if (!geom || !out) TC_FAIL(TC_ERR_ARG, "NULL argument to tc_plan_create");
        *out = nullptr;
        std::unique_ptr<tc_plan> p(new tc_plan());
        TC_TRY(plan_build(p->impl, *geom));
        *out = p.release();
        return TC_OK;
    });
}

int tc_plan_destroy(tc_plan *plan) {
    if (!plan) return TC_OK;
    delete plan;
    return TC_OK;
}

int tc_plan_get_info(const tc_plan *plan, tc_plan_info *info) {
    if (!plan || !info) TC_FAIL(TC_ERR_ARG, "NULL argument to tc_plan_get_info");
    const Plan &pl = plan->impl;
    info->n = pl.N;
    info->nproj = pl.P;
    info->nf = pl.nf;
    info->kernel_width = pl.es.w;
    info->toeplitz_m = pl.M;
    info->max_batch = pl.max_batch;
    info->workspace_bytes = (int64_t)pl.workspace_bytes();
    info->table_bytes = (int64_t)pl.table_bytes();
    info->lipschitz = pl.lipschitz;
    info->toeplitz_pairs = pl.toe_pairs;
    info->toeplitz_fast = pl.toe_fast ? 1 : 0;
    info->spread_tile = pl.spread.ts;
    info->spread_max_points = pl.spread.max_points;
    info->band_chunk = pl.bands.nf ? pl.bands.chunk : 0;
    info->interp_tile = pl.itiles.nsub ? pl.itiles.ts : 0;
    info->interp_max_points = pl.itiles.nsub ? pl.itiles.max_points : 0;
    info->paired_nufft = pl.pair_nufft ? 1 : 0;
    return TC_OK;
}

int tc_plan_set_psf(tc_plan *plan, const double *psf_host) {
    return guarded([&]() -> int {
        if (!plan || !psf_host) TC_FAIL(TC_ERR_ARG, "NULL argument to tc_plan_set_psf");
        Plan &pl = plan->impl;
        const size_t nm = 2 * (size_t)pl.N - 1;
        for (size_t i = 0; i < nm * nm; ++i)
            if (!std::isfinite(psf_host[i])) TC_FAIL(TC_ERR_NAN, "psf contains a non-finite value");
        TC_TRY(pl.d_psf.reserve(nm * nm * sizeof(double)));
        TC_CUDA(cudaMemcpy(pl.d_psf.ptr, psf_host, nm * nm * sizeof(double), cudaMemcpyHostToDevice));
        return psf_finish(pl);
    });
}

int tc_plan_get_psf(const tc_plan *plan, double *psf_host) {
    if (!plan || !psf_host) TC_FAIL(TC_ERR_ARG, "NULL argument to tc_plan_get_psf");
    TC_TRY(need_psf(plan->impl));
    const size_t nm = 2 * (size_t)plan->impl.N - 1;
    TC_CUDA(cudaMemcpy(psf_host, plan->impl.d_psf.ptr, nm * nm * sizeof(double),
                       cudaMemcpyDeviceToHost));
    return TC_OK;
}

int tc_radon(tc_plan *plan, const float *x, float *sino, int nslices, tc_stream_t stream) {
    return guarded([&]() -> int {
        if (!plan || (!x && nslices) || (!sino && nslices)) TC_FAIL(TC_ERR_ARG, "NULL argument to tc_radon");
        if (nslices < 0) TC_FAIL(TC_ERR_SHAPE, "nslices < 0");
        Plan &pl = plan->impl;
        const size_t in_s = (size_t)pl.N * pl.N, out_s = (size_t)pl.P * pl.N;
        for (int b0 = 0; b0 < nslices; b0 += pl.max_batch) {
            const int nb = std::min(pl.max_batch, nslices - b0);
            TC_TRY(radon_chunk(pl, x + b0 * in_s, sino + b0 * out_s, nb, S_(stream)));
        }
        return TC_OK;
    });
}

int tc_iradon(tc_plan *plan, const float *sino, float *x, int nslices, int ramp,
              tc_stream_t stream) {
    return guarded([&]() -> int {
        if (!plan || (!x && nslices) || (!sino && nslices)) TC_FAIL(TC_ERR_ARG, "NULL argument to tc_iradon");
        if (nslices < 0) TC_FAIL(TC_ERR_SHAPE, "nslices < 0");
        Plan &pl = plan->impl;
        const size_t out_s = (size_t)pl.N * pl.N, in_s = (size_t)pl.P * pl.N;
        for (int b0 = 0; b0 < nslices; b0 += pl.max_batch) {
            const int nb = std::min(pl.max_batch, nslices - b0);
            TC_TRY(iradon_chunk(pl, sino + b0 * in_s, x + b0 * out_s, nb, ramp, S_(stream)));
        }
        return TC_OK;
    });
}

int tc_nufft_grad(tc_plan *plan, const float *x, const float *aty, float *g, int nslices,
                  tc_stream_t stream) {
    return guarded([&]() -> int {
        if (!plan || (!x && nslices) || (!g && nslices)) TC_FAIL(TC_ERR_ARG, "NULL argument to tc_nufft_grad");
        if (nslices < 0) TC_FAIL(TC_ERR_SHAPE, "nslices < 0");
        Plan &pl = plan->impl;
        const size_t vs = (size_t)pl.N * pl.N;
        for (int b0 = 0; b0 < nslices; b0 += pl.max_batch) {
            const int nb = std::min(pl.max_batch, nslices - b0);
            TC_TRY(nufft_grad_chunk(pl, x + b0 * vs, aty ? aty + b0 * vs : nullptr, g + b0 * vs, nb,
                                    S_(stream)));
        }
        return TC_OK;
    });
}

int tc_toeplitz_grad(tc_plan *plan, const float *x, const float *aty, float *g, int nslices,
                     double *xhx, double *xaty, tc_stream_t stream) {
    return guarded([&]() -> int {
        if (!plan || (!x && nslices) || (!g && nslices)) TC_FAIL(TC_ERR_ARG, "NULL argument to tc_toeplitz_grad");
        if (nslices < 0) TC_FAIL(TC_ERR_SHAPE, "nslices < 0");
        Plan &pl = plan->impl;
        TC_TRY(need_psf(pl));
        cudaStream_t st = S_(stream);
        const size_t vs = (size_t)pl.N * pl.N;
        const int chunk = 2 * pl.toe_pairs;
        const bool dots = (xhx || xaty);
        int nparts = 0;
        for (int b0 = 0; b0 < nslices; b0 += chunk)
            nparts += toeplitz_partials_count(pl, std::min(chunk, nslices - b0));
        if (dots) TC_TRY(pl.ws_scalars.reserve(((size_t)nparts * 2 + 2) * sizeof(double)));
        double *parts = dots ? pl.ws_scalars.as<double>() : nullptr;
        int off = 0;
        for (int b0 = 0; b0 < nslices; b0 += chunk) {
            const int nb = std::min(chunk, nslices - b0);
            TC_TRY(toeplitz_chunk(pl, x + b0 * vs, aty ? aty + b0 * vs : nullptr, g + b0 * vs, nb,
                                  parts ? parts + (size_t)off * 2 : nullptr, st));
            off += toeplitz_partials_count(pl, nb);
        }
        if (dots) {
            double *res = parts + (size_t)nparts * 2;
            double h[2] = {0.0, 0.0};
            if (nparts > 0) {
                TC_TRY(reduce_partials(parts, nparts, 2, res, st));
                TC_CUDA(cudaMemcpyAsync(h, res, 2 * sizeof(double), cudaMemcpyDeviceToHost, st));
                TC_CUDA(cudaStreamSynchronize(st));
            }
            if (xhx) *xhx = h[0];
            if (xaty) *xaty = h[1];
        }
        return TC_OK;
    });
}

int tc_qggmrf_grad(const float *x, float *g, int nslices, int nrows, int ncols, float sigma,
                   float p, float scale, tc_stream_t stream) {
    return guarded([&]() -> int {
        if (nslices < 0 || nrows < 0 || ncols < 0) TC_FAIL(TC_ERR_SHAPE, "negative size");
        if ((size_t)nslices * nrows * ncols == 0) return TC_OK;
        if (!x || !g) TC_FAIL(TC_ERR_ARG, "NULL argument to tc_qggmrf_grad");
        if (!(sigma > 0) || !std::isfinite(sigma)) TC_FAIL(TC_ERR_ARG, "sigma must be > 0");
        if (!(p > 0 && p <= 2)) TC_FAIL(TC_ERR_ARG, "p must be in (0, 2]");
        return qggmrf_launch(x, g, nslices, nrows, ncols, sigma, p, scale, S_(stream));
    });
}

int tc_mbir_batched(const tc_scan *scans, int nscans, int num_iters, int use_graph,
                    int max_attempts, double *history, tc_stream_t stream) {
    return guarded([&]() -> int {
        if (nscans < 0) TC_FAIL(TC_ERR_SHAPE, "nscans < 0");
        if (nscans > 0 && !scans) TC_FAIL(TC_ERR_ARG, "NULL scans");
        std::vector<BatchScanIn> in((size_t)nscans);
        for (int i = 0; i < nscans; ++i) {
            const tc_scan &s = scans[i];
            if (!s.plan || !s.aty || !s.x)
                TC_FAIL(TC_ERR_ARG, "scan " + std::to_string(i) + ": NULL plan, aty or x");
            in[i] = BatchScanIn{&s.plan->impl, s.aty, s.sino_sq, s.x, s.nslices,
                                s.sigma, s.p, s.prior_weight, s.step};
        }
        return mbir_batched(in, num_iters, use_graph, max_attempts, history, S_(stream));
    });
}

int tc_qggmrf_value(const float *x, int nslices, int nrows, int ncols, float sigma, float p,
                    double *value, double *dvalue_dsigma, tc_stream_t stream) {
    return guarded([&]() -> int {
        if (!x && (size_t)nslices * nrows * ncols > 0) TC_FAIL(TC_ERR_ARG, "NULL argument to tc_qggmrf_value");
        return qggmrf_value_launch(x, nslices, nrows, ncols, sigma, p, value, dvalue_dsigma,
                                   S_(stream));
    });
}

int tc_qggmrf_hvp(const float *x, const float *v, float *hv, int nslices, int nrows, int ncols,
                  float sigma, float p, float scale, double *v_dot_grad, double *v_dot_dgrad_dsig,
                  tc_stream_t stream) {
    return guarded([&]() -> int {
        if ((!x || !v) && (size_t)nslices * nrows * ncols > 0)
            TC_FAIL(TC_ERR_ARG, "NULL argument to tc_qggmrf_hvp");
        return qggmrf_hvp_launch(x, v, hv, nslices, nrows, ncols, sigma, p, scale, v_dot_grad,
                                 v_dot_dgrad_dsig, S_(stream));
    });
}

int tc_fft_c2c(const float *in, float *out, int nbatch, int n, int dir, tc_stream_t stream) {
    return guarded([&]() -> int {
        if (nbatch < 0 || n < 1) TC_FAIL(TC_ERR_SHAPE, "invalid FFT size");
        if (dir != -1 && dir != 1) TC_FAIL(TC_ERR_ARG, "dir must be -1 or +1");
        if (nbatch == 0) return TC_OK;
        if (!in || !out) TC_FAIL(TC_ERR_ARG, "NULL argument to tc_fft_c2c");
        FftTables<float> T;
        TC_TRY(T.init(n));
        TC_TRY(fft_lines_launch<float>(T, reinterpret_cast<const c32 *>(in),
                                       reinterpret_cast<c32 *>(out), nbatch, dir, S_(stream)));
        // the tables are freed on return; finish the launch first
        TC_CUDA(cudaStreamSynchronize(S_(stream)));
        return TC_OK;
    });
}

int tc_axpby(float a, const float *x, float b, float *y, size_t n, tc_stream_t stream) {
    if (n == 0) return TC_OK;
    if (!x || !y) TC_FAIL(TC_ERR_ARG, "NULL argument to tc_axpby");
    return axpby_dev(a, x, b, y, n, S_(stream));
}

void tc_mbir_opts_default(tc_mbir_opts *o) {
    if (!o) return;
    o->num_iters = 100;
    o->sigma = 100.0f;  // 1 / smoothness with the Python default smoothness 0.01
    o->p = 1.2f;
    o->prior_weight = 1.0f;
    o->step = 0.0f;
    o->use_graph = 1;
    o->max_attempts = 1000;
    o->verbose = 0;
    o->phase_ms = nullptr;
}

static int check_opts(const tc_mbir_opts &o) {
    if (o.num_iters < 0) TC_FAIL(TC_ERR_ARG, "num_iters < 0");
    if (!(o.sigma > 0) || !std::isfinite(o.sigma)) TC_FAIL(TC_ERR_ARG, "sigma must be > 0");
    if (!(o.p > 0 && o.p <= 2)) TC_FAIL(TC_ERR_ARG, "p must be in (0, 2]");
    if (!std::isfinite(o.prior_weight)) TC_FAIL(TC_ERR_ARG, "prior_weight must be finite");
    return TC_OK;
}

int tc_mbir_solve(tc_plan *plan, const float *aty, double sino_sq, float *x, int nslices,
                  const tc_mbir_opts *opts, double *history, tc_stream_t stream) {
    return guarded([&]() -> int {
        if (!plan || !aty || !x || !opts) TC_FAIL(TC_ERR_ARG, "NULL argument to tc_mbir_solve");
        if (nslices < 1) TC_FAIL(TC_ERR_SHAPE, "nslices must be >= 1");
        if (nslices > 65535) TC_FAIL(TC_ERR_SHAPE, "nslices > 65535");
        TC_TRY(check_opts(*opts));
        if (!std::isfinite(sino_sq)) TC_FAIL(TC_ERR_NAN, "sino_sq is not finite");
        TC_TRY(need_psf(plan->impl));
        return mbir_solve(plan->impl, aty, sino_sq, x, nslices, *opts, history, S_(stream));
    });
}

// ---- host entry points ------------------------------------------------------

int tc_radon_host(const float *img, int nslices, int n, const float *angles, int nproj,
                  float *out) {
    return guarded([&]() -> int {
        if (!img || !angles || !out) TC_FAIL(TC_ERR_ARG, "NULL argument to tc_radon_host");
        if (nslices < 1) TC_FAIL(TC_ERR_SHAPE, "nslices must be >= 1");
        tc_geom g{n, nproj, angles, 0.0, 0, TC_PLAN_NO_PSF};
        tc_plan *pl = nullptr;
        TC_TRY(tc_plan_create(&g, &pl));
        std::unique_ptr<tc_plan, int (*)(tc_plan *)> guard(pl, tc_plan_destroy);
        const size_t ni = (size_t)nslices * n * n, no = (size_t)nslices * nproj * n;
        DevArr di, dout;
        TC_TRY(di.alloc<float>(ni));
        TC_TRY(dout.alloc<float>(no));
        TC_TRY(copy_h2d(di.p<float>(), img, ni * sizeof(float)));
        TC_TRY(tc_radon(pl, di.p<float>(), dout.p<float>(), nslices, nullptr));
        TC_TRY(copy_d2h(out, dout.p<float>(), no * sizeof(float)));
        return TC_OK;
    });
}

int tc_backproject_host(const float *sino, int nslices, int nproj, int ndet, const float *angles,
                        float center, float *out) {
    return guarded([&]() -> int {
        if (!sino || !angles || !out) TC_FAIL(TC_ERR_ARG, "NULL argument to tc_backproject_host");
        if (nslices < 1 || nproj < 1 || ndet < 4) TC_FAIL(TC_ERR_SHAPE, "invalid sinogram shape");
        if (!std::isfinite(center)) TC_FAIL(TC_ERR_ARG, "center is not finite");
        int npad, off;
        preproc_params(ndet, center, npad, off);
        const int D2 = ndet + 2 * npad;
        tc_geom g{D2, nproj, angles, 0.0, 0, TC_PLAN_NO_PSF};
        tc_plan *pl = nullptr;
        TC_TRY(tc_plan_create(&g, &pl));
        std::unique_ptr<tc_plan, int (*)(tc_plan *)> guard(pl, tc_plan_destroy);
        const size_t ns = (size_t)nslices * nproj * ndet, ns2 = (size_t)nslices * nproj * D2;
        const size_t nx2 = (size_t)nslices * D2 * D2, nx = (size_t)nslices * ndet * ndet;
        DevArr ds, ds2, dx2, dx;
        TC_TRY(ds.alloc<float>(ns));
        TC_TRY(ds2.alloc<float>(ns2));
        TC_TRY(dx2.alloc<float>(nx2));
        TC_TRY(dx.alloc<float>(nx));
        TC_TRY(copy_h2d(ds.p<float>(), sino, ns * sizeof(float)));
        TC_TRY(preproc_dev(ds.p<float>(), ds2.p<float>(), nslices, nproj, ndet, npad, off, nullptr));
        TC_TRY(tc_iradon(pl, ds2.p<float>(), dx2.p<float>(), nslices, 0, nullptr));
        TC_TRY(crop2d_dev(dx2.p<float>(), dx.p<float>(), nslices, D2, D2, ndet, nullptr));
        TC_TRY(copy_d2h(out, dx.p<float>(), nx * sizeof(float)));
        return TC_OK;
    });
}

int tc_mbir_host(const float *sino, int nslices, int nproj, int ndet, const float *angles,
                 float center, int num_iters, float sigma, float tol, float xtol, float *out,
                 const tc_mbir_opts *opts_in) {
    (void)tol;
    (void)xtol;  // accepted and unused, as in Optimizer::run2
    return guarded([&]() -> int {
        if (!sino || !angles || !out) TC_FAIL(TC_ERR_ARG, "NULL argument to tc_mbir_host");
        if (nslices < 1 || nproj < 1 || ndet < 4) TC_FAIL(TC_ERR_SHAPE, "invalid sinogram shape");
        if (!std::isfinite(center)) TC_FAIL(TC_ERR_ARG, "center is not finite");
        tc_mbir_opts o;
        tc_mbir_opts_default(&o);
        if (opts_in) o = *opts_in;
        o.num_iters = num_iters;
        o.sigma = sigma;
        TC_TRY(check_opts(o));
        PhaseTrace tr;
        const size_t ns = (size_t)nslices * nproj * ndet;
        // fault in the output's pages while the device works
        HostPrefault prefault(out, (size_t)nslices * ndet * ndet * sizeof(float));
        DevArr ds;
        TC_TRY(ds.alloc<float>(ns));
        TC_TRY(copy_h2d(ds.p<float>(), sino, ns * sizeof(float)));
        tr.mark("h2d");
        // normalise by the maximum (src/mbir2.cpp:46-54)
        // the maximum alone would not see a NaN (fmaxf drops it); the sum of
        // squares does
        float maxv = 0.f;
        double sq0 = 0.0;
        TC_TRY(max_sumsq_dev(ds.p<float>(), ns, &maxv, &sq0, nullptr));
        if (!std::isfinite(maxv) || !std::isfinite(sq0))
            TC_FAIL(TC_ERR_NAN, "sinogram contains a non-finite value");
        if (maxv == 0.f) TC_FAIL(TC_ERR_ARG, "sinogram has ZERO max value");
        TC_TRY(scale_dev(ds.p<float>(), ns, maxv, nullptr));
        tr.mark("normalise");
        // FBP initial guess on the unpadded sinogram (src/mbir2.cpp:56-60)
        const size_t nx = (size_t)nslices * ndet * ndet;
        DevArr dx0;
        TC_TRY(dx0.alloc<float>(nx));
        {
            tc_geom g0{ndet, nproj, angles, 0.0, 0, TC_PLAN_NO_PSF};
            tc_plan *p0 = nullptr;
            TC_TRY(tc_plan_create(&g0, &p0));
            std::unique_ptr<tc_plan, int (*)(tc_plan *)> guard0(p0, tc_plan_destroy);
            tr.mark("fbp.plan");
            TC_TRY(tc_iradon(p0, ds.p<float>(), dx0.p<float>(), nslices, 1, nullptr));
            TC_CUDA(cudaDeviceSynchronize());
        }
        tr.mark("fbp");
        // centre and pad (src/mbir2.cpp:62-66)
        int npad, off;
        preproc_params(ndet, center, npad, off);
        const int D2 = ndet + 2 * npad;
        const size_t ns2 = (size_t)nslices * nproj * D2, nx2 = (size_t)nslices * D2 * D2;
        DevArr ds2, dx2, daty;
        TC_TRY(ds2.alloc<float>(ns2));
        TC_TRY(dx2.alloc<float>(nx2));
        TC_TRY(daty.alloc<float>(nx2));
        TC_TRY(preproc_dev(ds.p<float>(), ds2.p<float>(), nslices, nproj, ndet, npad, off, nullptr));
        TC_TRY(pad2d_dev(dx0.p<float>(), dx2.p<float>(), nslices, ndet, ndet, D2 - ndet, nullptr));
        ds.b.release();
        dx0.b.release();
        tr.mark("pad");
        tc_geom g{D2, nproj, angles, 0.0, 0, 0};
        tc_plan *pl = nullptr;
        TC_TRY(tc_plan_create(&g, &pl));
        std::unique_ptr<tc_plan, int (*)(tc_plan *)> guard(pl, tc_plan_destroy);
        tr.mark("plan");
        // A^T y and |y|^2 (src/mbir2.cpp:73-77)
        TC_TRY(tc_iradon(pl, ds2.p<float>(), daty.p<float>(), nslices, 0, nullptr));
        double sino_sq = 0.0;
        TC_TRY(max_sumsq_dev(ds2.p<float>(), ns2, nullptr, &sino_sq, nullptr));
        ds2.b.release();
        tr.mark("aty");
        // with TC_TRACE the solve's attempt count is printed beside its time
        std::vector<double> hist(tr.on ? (size_t)std::max(o.num_iters, 0) * 3 : 0);
        TC_TRY(tc_mbir_solve(pl, daty.p<float>(), sino_sq, dx2.p<float>(), nslices, &o,
                             tr.on ? hist.data() : nullptr, nullptr));
        tr.mark("solve");
        if (tr.on) {
            double att = 0.0;
            for (size_t i = 2; i < hist.size(); i += 3) att += hist[i];
            std::fprintf(stderr, "tc_trace solve_attempts %.0f iterations %d\n", att, o.num_iters);
        }
        // crop (src/mbir2.cpp:144)
        DevArr dx;
        TC_TRY(dx.alloc<float>(nx));
        TC_TRY(crop2d_dev(dx2.p<float>(), dx.p<float>(), nslices, D2, D2, ndet, nullptr));
        prefault.wait();
        TC_TRY(copy_d2h(out, dx.p<float>(), nx * sizeof(float)));
        tr.mark("crop_d2h");
        return TC_OK;
    });
}

int tc_sino_ingest_psd(const float *host, int nproj, int nslices, int ndet, int s0, int ns,
                       float *dev) {
    return guarded([&]() -> int {
        if (!host || (!dev && ns > 0)) TC_FAIL(TC_ERR_ARG, "NULL argument to tc_sino_ingest_psd");
        if (nproj < 1 || nslices < 1 || ndet < 1) TC_FAIL(TC_ERR_SHAPE, "invalid sinogram shape");
        if (s0 < 0 || ns < 0 || s0 > nslices || ns > nslices - s0)
            TC_FAIL(TC_ERR_SHAPE, "slice range outside the sinogram");
        return ingest_psd(host, nproj, nslices, ndet, s0, ns, dev);
    });
}

int tc_set_num_of_gpus(int n) {
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess) {
        cudaGetLastError();
        TC_FAIL(TC_ERR_CUDA, std::string("cudaGetDeviceCount failed: ") + cudaGetErrorString(e));
    }
    if (n < 1 || n > count)
        TC_FAIL(TC_ERR_ARG, "Invalid number of GPUs: " + std::to_string(n) + " (" +
                                std::to_string(count) + " available)");
    g_num_gpus = n;
    return TC_OK;
}

}  // extern "C"
