/*
 * tomocam_b200.h -- C ABI of the B200 implementation of tomoCAM's MBIR path.
 *
 * Every entry point returns an int status (TC_OK = 0, negative on error) and
 * never exits the process; tc_last_error_string() describes the last failure
 * on the calling thread.  Arrays are float32, C order: images [S][N][N],
 * sinograms [S][P][D] with D == N (the reference ties the detector count to
 * the image width, src/radon.cpp:42-44 and src/iradon.cpp:82).
 *
 * Two layers:
 *   - plan-based device entry points: caller-owned DEVICE buffers and an
 *     explicit CUDA stream (tc_stream_t is a cudaStream_t, 0 = legacy default
 *     stream).  A plan caches geometry, the point-spread function, FFT tables
 *     and workspace; one plan must not be used by two threads at once,
 *     separate plans are independent.
 *   - host entry points (tc_*_host) that mirror the reference's pybind module
 *     cTomocam (src/pyTomocam.cpp:81-152): host buffers in and out, all
 *     host<->device traffic inside the call.
 *
 * File:line citations name the reference interface each entry replaces
 * (paths relative to the lbl-camera/tomocam project root).
 */
#ifndef TOMOCAM_B200_H
#define TOMOCAM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TC_OK 0
#define TC_ERR_ARG (-1)     /* null pointer or invalid scalar argument */
#define TC_ERR_SHAPE (-2)   /* array sizes inconsistent or unsupported */
#define TC_ERR_ALLOC (-3)   /* device or host allocation failed */
#define TC_ERR_CUDA (-4)    /* a CUDA runtime call failed */
#define TC_ERR_TIMEOUT (-5) /* a bounded device-side wait gave up */
#define TC_ERR_NAN (-6)     /* non-finite value where a finite one is required */
#define TC_ERR_STATE (-7)   /* call not valid in the object's current state */
/* Where the reference exits the process (src/gpu/utils.cuh:31-40,
 * src/mbir2.cpp:50-53) these calls return a status instead.  For testing the
 * allocation-failure path: with the environment variable
 * TOMOCAM_B200_FAIL_ALLOC_ABOVE=<bytes> set when the library loads, every
 * device allocation larger than that fails with TC_ERR_ALLOC. */

typedef void *tc_stream_t; /* cudaStream_t */
typedef struct tc_plan tc_plan;

/* Geometry of one scan.  Replaces NUFFT::Grid (src/nufft.h:55-192) and the
 * PointSpreadFunction constructor (src/toeplitz.h:51-73). */
typedef struct {
    int32_t n;           /* image width N == detector pixels D (>= 4) */
    int32_t nproj;       /* number of projection angles P (>= 1) */
    const float *angles; /* host array of P angles in radians */
    double nufft_tol;    /* ES-kernel NUFFT tolerance; <= 0 selects 1e-6 */
    int32_t max_batch;   /* slices per internal chunk (NUFFT chunks, at most 16 slices
                            when paired and 8 otherwise; Toeplitz chunks of
                            max(1, max_batch / 2) slice pairs); <= 0 selects automatically */
    int32_t flags;       /* 0 or an OR of the TC_PLAN_* flags below */
} tc_geom;

/* tc_geom.flags: skip the point-spread function (radon / back-projection
 * only; Toeplitz entry points then fail with TC_ERR_STATE until
 * tc_plan_set_psf supplies one). */
#define TC_PLAN_NO_PSF 1
/* tc_geom.flags: time the NUFFT's spreading and interpolation on this
 * geometry and keep the fastest choices (cached per geometry for the
 * process): tile edges (16, 32, 64) and sub-problem sizes of the type-1 tile
 * path, and on the register-FFT path the band lists' chunk (128 .. 1024
 * points), the slices per NUFFT chunk and the type-2 interpolation tiles
 * (edge 16 or 32, 256 .. 4096 points per sub-problem); without it 32 x 32
 * spreading tiles of at most 2048 points, 256-point band chunks, up to 8
 * complex lines per chunk (16 slices when paired, see TC_PLAN_UNPAIRED) and
 * 16 x 16 interpolation tiles of at most 256 points are used.
 * No counterpart in the reference. */
#define TC_PLAN_AUTOTUNE 2
/* tc_geom.flags: use a power-of-two Toeplitz FFT size (M >= 2N-1) even where
 * 1536, 3072 or 6144 would be smaller; tc_mbir_batched needs it for images of
 * 513 .. 768 and 1025 .. 1536 pixels.  No counterpart in the reference. */
#define TC_PLAN_POW2_TOEPLITZ 4
/* tc_geom.flags: one slice per complex line in the NUFFT operators.  By
 * default the register-FFT path (fine grids 2^k or 3 x 2^k up to 6144,
 * kernel widths 2 .. 8) carries two real slices as the real and imaginary
 * parts of one complex line through radon, back-projection and the NUFFT
 * gradient, which halves their FFT and interpolation work; the results
 * differ from the unpaired ones only by rounding.  No counterpart in the
 * reference. */
#define TC_PLAN_UNPAIRED 8

/* Sizes chosen by a plan (for diagnostics and byte models). */
typedef struct {
    int32_t n, nproj;
    int32_t nf;          /* NUFFT fine-grid size (upsampling 2) */
    int32_t kernel_width;/* ES kernel width w */
    int32_t toeplitz_m;  /* Toeplitz FFT size M >= 2N-1 */
    int32_t max_batch;   /* slices per internal chunk */
    int64_t workspace_bytes;
    int64_t table_bytes;
    double lipschitz;    /* max(H 1) as in src/mbir2.cpp:100-112 */
    int32_t toeplitz_pairs; /* slice pairs per Toeplitz launch */
    int32_t toeplitz_fast;  /* 1: register-resident FFT kernels */
    int32_t spread_tile;    /* type-1 spreading tile edge */
    int32_t spread_max_points; /* points per spreading sub-problem */
    int32_t band_chunk;     /* points per warp chunk of the band spreading (0: no bands) */
    int32_t interp_tile;    /* type-2 interpolation tile edge (0: one thread per point) */
    int32_t interp_max_points; /* points per interpolation sub-problem */
    int32_t paired_nufft;   /* 1: two slices per complex NUFFT line */
} tc_plan_info;

/* Create a plan on the current CUDA device; computes the polar grid, the
 * FP64 point-spread function and its spectrum.  Replaces Grid + PSF
 * construction in src/mbir2.cpp:83-98. */
int tc_plan_create(const tc_geom *geom, tc_plan **plan);
int tc_plan_destroy(tc_plan *plan);
int tc_plan_get_info(const tc_plan *plan, tc_plan_info *info);

/* Forward projection, sino = A x.  Replaces project() on one device,
 * src/forward.cpp:34-52 (driver src/radon.cpp:35-96). */
int tc_radon(tc_plan *plan, const float *x, float *sino, int nslices,
             tc_stream_t stream);

/* Back-projection x = A^T y (ramp != 0: Ram-Lak filtered, fbp=true).
 * Replaces backproject() on one device, src/backward.cpp:43-67
 * (driver src/iradon.cpp:36-102, filter src/gpu/ramlak.cu:15-51). */
int tc_iradon(tc_plan *plan, const float *sino, float *x, int nslices, int ramp,
              tc_stream_t stream);

/* Toeplitz data gradient g = H x - aty (aty may be NULL: g = H x), with H x
 * the PSF convolution.  Optional host outputs (NULL to skip):
 * xhx = sum x.Hx and xaty = sum x.aty, accumulated in FP64.
 * Replaces gradient2 (src/gradient2.cpp:37-68) and the dots of
 * function_value2 (src/error2.cpp:41-67), convolve (src/toeplitz.h:95-159). */
int tc_toeplitz_grad(tc_plan *plan, const float *x, const float *aty, float *g,
                     int nslices, double *xhx, double *xaty, tc_stream_t stream);

/* tc_toeplitz_grad for callers that cannot allocate device memory:
 * applications whose own pool allocator owns the GPU's memory and forbid a
 * library to call cudaMalloc (which may fail against the full pool, and may
 * synchronise the device mid-pipeline).  Same arguments and results as
 * tc_toeplitz_grad, but the slice-pair workspace is a fixed 32 MiB array
 * inside the library image (held by every GPU that loads the library until
 * exit) instead of plan memory, and nothing is allocated.  One pair needs
 * N * M * 8 + 16 N bytes (M >= 2N-1 the plan's FFT size): every N <= 1024
 * fits; larger plans fit only while that stays within the scratch and fail
 * with TC_ERR_SHAPE otherwise.  It runs the general FFT engine, not the
 * register-FFT kernels, so it is slower.  All calls share the array, which
 * keeps the last call's contents, so calls that overlap on the GPU race;
 * the first call on a device looks up the array's address and should come
 * before any stream capture.  With xhx or xaty non-NULL the call copies the
 * sums to the host and synchronises the stream.  It has no counterpart in
 * the reference. */
int tc_toeplitz_grad_noalloc(tc_plan *plan, const float *x, const float *aty, float *g,
                             int nslices, double *xhx, double *xaty, tc_stream_t stream);

/* NUFFT-pair gradient g = Re(NUFFT1(NUFFT2(x)))/N^3 - aty (aty may be NULL).
 * Replaces gradient (src/gradient.cpp:35-71). */
int tc_nufft_grad(tc_plan *plan, const float *x, const float *aty, float *g,
                  int nslices, tc_stream_t stream);

/* qGGMRF prior: g += scale * sum_{26 n} w_n rho'(x_v - x_n; sigma, p) with
 * clamp-to-edge boundaries on an [S][R][C] volume.  Replaces add_total_var2
 * (src/tv_update.cpp:76-106, kernel src/gpu/cuTV2.cu:33-93). */
int tc_qggmrf_grad(const float *x, float *g, int nslices, int nrows, int ncols,
                   float sigma, float p, float scale, tc_stream_t stream);

/* Value of the prior potential whose gradient tc_qggmrf_grad adds,
 * U(x) = 1/2 sum_v sum_{26 n} w_n rho(x_v - x_n), rho(d) = u^2 / (c + u^(2-p)),
 * u = |d| / sigma (clamp-to-edge neighbours), and dU/dsigma; either output may
 * be NULL.  Synchronises the stream.  For differentiating the MBIR objective;
 * no counterpart in the reference, which evaluates only the gradient. */
int tc_qggmrf_value(const float *x, int nslices, int nrows, int ncols, float sigma,
                    float p, double *value, double *dvalue_dsigma, tc_stream_t stream);

/* Second-order terms of the prior at x for a direction v:
 *   hv = scale * sum_{26 n} w_n rho''(x_v - x_n) (v_v - v_n)   (the Hessian of
 *        U times v, scaled; skipped when hv is NULL),
 *   *v_dot_grad       = v . grad U(x)             (unscaled),
 *   *v_dot_dgrad_dsig = v . d grad U(x) / dsigma  (unscaled).
 * The dots may be NULL (then the stream is not synchronised).  For
 * differentiating unrolled reconstructions; no counterpart in the reference. */
int tc_qggmrf_hvp(const float *x, const float *v, float *hv, int nslices, int nrows,
                  int ncols, float sigma, float p, float scale, double *v_dot_grad,
                  double *v_dot_dgrad_dsig, tc_stream_t stream);

/* Copy the plan's point-spread function, [2N-1][2N-1] doubles, offset
 * d = index - (N-1), to a host buffer (src/toeplitz.h:51-73). */
int tc_plan_get_psf(const tc_plan *plan, double *psf_host);

/* Replace the plan's point-spread function with a caller-supplied one
 * ([2N-1][2N-1] doubles, same offset convention) and recompute its spectrum
 * and the Lipschitz constant.  Serves the reference's Python
 * gradients(model, sinoT, psf) signature (tomocam/gradients.py:5-28). */
int tc_plan_set_psf(tc_plan *plan, const double *psf_host);

/* Batched complex-to-complex FFT along contiguous lines of length n (any
 * n >= 1; smooth sizes by mixed radix, others by Bluestein), unnormalised,
 * dir = -1 forward / +1 inverse, device buffers of nbatch*n interleaved
 * complex floats, in and out may alias.  The FFT engine behind all
 * operators; replaces the cuFFT plans of src/fft.h:41-209. */
int tc_fft_c2c(const float *in, float *out, int nbatch, int n, int dir,
               tc_stream_t stream);

/* y = a x + b y on n device floats (the DeviceArray arithmetic of
 * src/dev_array.h:190-256 that the operators above do not already fuse). */
int tc_axpby(float a, const float *x, float b, float *y, size_t n, tc_stream_t stream);

/* Solver options for tc_mbir_solve / tc_mbir_host. */
typedef struct {
    int32_t num_iters;   /* accepted iterations (Optimizer::run2 max_iters) */
    float sigma;         /* qGGMRF scale sigma */
    float p;             /* qGGMRF shape p; the reference hard-codes 1.2 */
    float prior_weight;  /* multiplies the prior gradient; 1 = reference */
    float step;          /* initial step; <= 0 selects min(1/max(H 1), 1) */
    int32_t use_graph;   /* 1: whole solve as one CUDA graph launch */
    int32_t max_attempts;/* per-iteration cap on backtracking attempts (<=0: 1000) */
    int32_t verbose;     /* 1: print "iter: ..., error: ..., x-err: ..." */
    double *phase_ms;    /* host, may be NULL; with use_graph = 0 it receives
                          * the summed device time (ms, CUDA events) of the
                          * update kernel, the Toeplitz passes and the step
                          * test over all attempts, then the attempt count:
                          * 4 doubles.  Ignored with the graph. */
} tc_mbir_opts;

/* Fill opts with the reference defaults (sigma 1, p 1.2, weight 1, graph on). */
void tc_mbir_opts_default(tc_mbir_opts *opts);

/* Device-resident MBIR iteration: Optimizer::run2 (src/optimize.h:96-154)
 * with gradient H x - aty + prior'(x) and objective
 * sqrt(sum x.Hx - 2 x.aty + sino_sq) (src/mbir2.cpp:122-136).  x is the
 * initial guess on entry and the solution on exit ([S][N][N], device).
 * history (host, may be NULL) receives 3 doubles per iteration: the
 * objective after the iteration, ||x_k+1 - x_k|| (the two values run2
 * prints) and the number of backtracking attempts the iteration took. */
int tc_mbir_solve(tc_plan *plan, const float *aty, double sino_sq, float *x,
                  int nslices, const tc_mbir_opts *opts, double *history,
                  tc_stream_t stream);

/* One scan of a batched solve.  Each scan has its own plan (geometry, PSF;
 * the plan's Toeplitz size must be a power of two <= 4096, i.e. n <= 2048),
 * A^T y and ||y||^2, its image (in: initial guess, out: result) and prior. */
typedef struct {
    tc_plan *plan;
    const float *aty;    /* device [nslices][n][n] */
    double sino_sq;      /* ||y||^2 of the normalised sinogram */
    float *x;            /* device [nslices][n][n], overwritten */
    int32_t nslices;
    float sigma;         /* qGGMRF sigma */
    float p;             /* qGGMRF p */
    float prior_weight;  /* beta: multiplies the prior gradient */
    float step;          /* initial step; <= 0 selects min(1/max(H 1), 1) */
} tc_scan;

/* Batched MBIR over independent scans of uneven sizes: every scan runs
 * Optimizer::run2 (src/optimize.h:96-154) exactly as tc_mbir_solve would
 * (its own step, backtracking and iteration count), and each attempt of all
 * running scans is one launch per kernel -- the fused update, the three
 * Toeplitz passes and the step test -- instead of one per scan.  use_graph
 * runs the loop as one CUDA graph with a WHILE node.  history (host, may be
 * NULL): [nscans][num_iters][3] as tc_mbir_solve.  Returns TC_ERR_TIMEOUT if
 * a scan hit max_attempts (the results of all scans are still written).
 * No counterpart in the reference, which solves one volume per call. */
int tc_mbir_batched(const tc_scan *scans, int nscans, int num_iters, int use_graph,
                    int max_attempts, double *history, tc_stream_t stream);

/* ---- one slab of a volume split across ranks by slices ----------------
 * The reference's multi-GPU scheme (src/dist_array.h:349-373,
 * src/multiproc.h:95-118, src/tv_update.cpp:82-96): each rank owns a slab
 * of slices; per attempt of Optimizer::run2 the ranks exchange one halo
 * plane with each neighbour and sum six FP64 values.  The library does the
 * per-slab work; the caller does the exchange and the sum (see
 * tomocam_b200/slab.py).  Per attempt:
 *   tc_slab_halo(which = 0 and, unless *same, 1): send the two boundary
 *     planes to the neighbours and fill the two halo planes from them (at an
 *     end of the volume, copy the slab's own edge plane into the halo);
 *   tc_slab_attempt: begin, update, H new, the six local sums (device);
 *   sum the six doubles over all slabs in place;
 *   tc_slab_decide: the step test on the global sums; *cond = 0 when done.
 * The host-driven loop only (no graph).  Results equal tc_mbir_solve of the
 * whole volume up to FP32 summation order. */
typedef struct tc_slab tc_slab;

/* aty, x0: the slab's owned slices [nslices][n][n] (device, copied);
 * sino_sq: ||y||^2 of the whole volume. */
int tc_slab_create(tc_plan *plan, const float *aty, double sino_sq, const float *x0,
                   int nslices, const tc_mbir_opts *opts, tc_slab **out,
                   tc_stream_t stream);
/* Device addresses of the planes to exchange before the next attempt:
 * which = 0 for x, 1 for sol; *same = 1 when they are one buffer.  Each
 * plane is n * n floats. */
int tc_slab_halo(tc_slab *slab, int which, float **send_lo, float **send_hi,
                 float **recv_lo, float **recv_hi, int *same);
/* Runs one attempt; *sums receives the device address of the 6 local sums. */
int tc_slab_attempt(tc_slab *slab, double **sums, tc_stream_t stream);
int tc_slab_decide(tc_slab *slab, int *cond, tc_stream_t stream);
/* The slab's owned slices of the solution (device), the history as
 * tc_mbir_solve (host, may be NULL) and the accepted iterations. */
int tc_slab_result(tc_slab *slab, float *x, double *history, int *iters,
                   tc_stream_t stream);
int tc_slab_destroy(tc_slab *slab);

/* ---- host entry points mirroring cTomocam (src/pyTomocam.cpp) ---------- */

/* cTomocam.radon(imgstack, angs): img [S][N][N] -> out [S][P][N].
 * src/pyTomocam.cpp:81-92. */
int tc_radon_host(const float *img, int nslices, int n, const float *angles,
                  int nproj, float *out);

/* cTomocam.backproject(sino, angs, cen): preproc, A^T, postproc;
 * sino [S][P][D] -> out [S][D][D].  src/pyTomocam.cpp:94-114. */
int tc_backproject_host(const float *sino, int nslices, int nproj, int ndet,
                        const float *angles, float center, float *out);

/* cTomocam.mbir(sino, angles, center, num_iters, sigma, tol, xtol):
 * tomocam::mbir2 (src/mbir2.cpp:41-145) -- normalisation, FBP guess,
 * centring/padding, A^T y, PSF, Lipschitz step, run2, crop.
 * out [S][D][D].  opts may be NULL (reference behaviour); opts->num_iters
 * and opts->sigma are overridden by the explicit arguments.  tol and xtol
 * are accepted and unused, as in the reference.  src/pyTomocam.cpp:116-134. */
int tc_mbir_host(const float *sino, int nslices, int nproj, int ndet,
                 const float *angles, float center, int num_iters, float sigma,
                 float tol, float xtol, float *out, const tc_mbir_opts *opts);

/* Sinogram ingest from the HDF5 file layout.  The reference's reader
 * (src/hdf5/reader.h:67-122) reads a dataset stored projection-major,
 * [P][S][D], and transposes it to slice-major [S][P][D] on the host.  This
 * copies slices s0 .. s0+ns-1 of a host array host [nproj][nslices][ndet]
 * into device memory dev [ns][nproj][ndet] with one strided copy per
 * projection (pinned host memory is copied directly, pageable memory through
 * the pinned staging buffers), so a slab of slices goes straight into HBM
 * in the operators' layout.  Returns when the copy is complete. */
int tc_sino_ingest_psd(const float *host, int nproj, int nslices, int ndet, int s0, int ns,
                       float *dev);

/* cTomocam.set_num_of_gpus(n) (src/pyTomocam.cpp:141-142, machine.h:44-50):
 * this implementation runs on the current device; n is validated against the
 * device count and recorded. */
int tc_set_num_of_gpus(int n);

/* Message of the last failed call on this thread ("" if none). */
const char *tc_last_error_string(void);

/* Library version string. */
const char *tc_version(void);

/* Free the device memory the library keeps for reuse on the current device.
 * Buffers the library releases (a destroyed plan's, the temporaries of the
 * host entry points) are kept, up to half the device's memory, and handed
 * to later allocations of about the same size, so that repeated calls do not
 * pay cudaMalloc / cudaFree each time; a failing allocation empties the cache
 * by itself.  Setting TOMOCAM_B200_NO_CACHE=1 in the environment turns the
 * cache off.  No counterpart in the reference (it allocates per operation). */
int tc_release_cached_memory(void);

#ifdef __cplusplus
}
#endif

#endif /* TOMOCAM_B200_H */
