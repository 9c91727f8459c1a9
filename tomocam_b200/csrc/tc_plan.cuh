// tc_plan.cuh -- the plan object shared by all operators (internal).
#pragma once

#include <thread>
#include <vector>

#include "tc_common.cuh"
#include "tc_fft.cuh"

namespace tc {

// ES kernel parameters (Barnett, Magland & af Klinteberg 2019): upsampling 2,
// width w = ceil(log10(1/tol)) + 1, beta = 2.30 w.
struct EsKernel {
    int w = 7;
    double beta = 16.1;
    void set(double tol);
};

// Geometry of the polar grid, passed by value to kernels.  Point (p, j):
//   r_j = s (j - D/2),  x = r_j cos(theta_p),  y = r_j sin(theta_p),
// s = 2 pi / (D - 1) (src/gpu/nufft_utils.cu:32-44); coordinates are formed
// in FP64 from per-angle cos/sin so the fine-grid index and offset keep
// ~1e-7 grid-cell accuracy at any N.
struct PolarDev {
    int P, D, half;           // half = D / 2
    double s;                 // radial spacing
    const double *cs, *sn;    // per-angle cos, sin (device)
};

// fine-grid spreading tiles (type-1 NUFFT)
constexpr int SPREAD_TILE = 32;
struct SpreadSub {
    int tile;      // tile index ty * ntiles + tx
    int start;     // offset into the point list
    int count;     // points in this sub-problem
    int shared;    // 1: the tile is split over several sub-problems
};

struct SpreadLists {
    int nf = 0, ntiles = 0;          // tiles per dimension
    int ts = SPREAD_TILE;            // tile edge (16, 32 or 64 cells)
    int max_points = 2048;           // points per sub-problem
    int nsub = 0, nshared_tiles = 0;
    DevBuf points;                   // int, point indices p*D + j
    DevBuf subs;                     // SpreadSub
    DevBuf shared_tiles;             // int, tiles split over several sub-problems
    int build(const PolarDev &g, const std::vector<double> &cs, const std::vector<double> &sn,
              int nf, int w, int max_points, int ts = SPREAD_TILE);
};

// fine-grid spreading bands of the register-FFT type-1 path: a band is
// BAND_H rows x BAND_W columns of the fine grid, spread by one warp into its
// own shared-memory accumulator with one point's footprint laid across the
// lanes (BAND_H rows x 8 columns, kernel widths w <= 8).  Each entry holds
// the point index, its first tap relative to the band (dx0, dy0 in
// [-(w-1), band size), packed as two int16) and the tap offsets fx, fy.
constexpr int BAND_W = 32, BAND_H = 4, BAND_CHUNK = 256;
struct BandEntry {
    int pt;
    int dxy;      // (dy0 << 16) | (dx0 & 0xffff)
    float fx, fy;
};
struct BandChunk {
    int band;     // by * (nf / BAND_W) + bx
    int start;    // offset into the entries
    int count;    // entries in this chunk (<= BAND_CHUNK)
    int shared;   // 1: the band is split over several chunks
};
struct SpreadBands {
    int nf = 0, w = 0, nvirt = 0;
    int chunk = BAND_CHUNK;       // points per warp chunk of a band's list
    int nchunk = 0, nshared = 0;
    DevBuf entries;               // BandEntry
    DevBuf chunks;                // BandChunk
    DevBuf shared_bands;          // int, bands split over several chunks
    // nvirt: the mirror points of the paired path (one per angle, j = D,
    // listed after the P * D detector points)
    int build(const PolarDev &g, int nf, int w, int chunk = BAND_CHUNK, int nvirt = 0);
};

// type-2 interpolation tiles of the register-FFT path: every point is
// listed once, under the ts x ts tile of the fine grid that holds its first
// tap; a sub-problem (one tile, at most max_points of its points) copies the
// tile's footprint region, (ts + w - 1)^2 cells from the tile origin, of the
// chunk's grids into shared memory and interpolates its points from there
constexpr int INTERP_TILE = 16, INTERP_POINTS = 256;
// one point of an interpolation tile, with its set-up done at plan time
struct InterpEntry {
    int pt;        // point index p * D + j (mirror points: P * D + p)
    int off;       // first tap in the tile's region: dx * pitch + dy
    float fx, fy;  // first-tap offsets xi - lx0, yi - ly0 (point_taps)
};
static_assert(sizeof(InterpEntry) == 16, "one 16-byte load per entry");
struct InterpTiles {
    int nf = 0, w = 0, ts = INTERP_TILE, ntiles = 0, max_points = INTERP_POINTS, nsub = 0, nvirt = 0;
    DevBuf entries;  // InterpEntry, grouped by tile
    DevBuf subs;     // SpreadSub (tile, start, count; shared unused)
    int build(const PolarDev &g, int nf, int w, int ts = INTERP_TILE,
              int max_points = INTERP_POINTS, int nvirt = 0);
};

struct Plan {
    int N = 0, P = 0;           // image width == detector pixels
    EsKernel es;                // FP32 operators
    EsKernel es64;              // FP64 point-spread function
    int nf = 0;                 // fine grid for N modes
    int M = 0;                  // Toeplitz FFT size >= 2N - 1
    int max_batch = 1;          // slices per NUFFT chunk
    // Paired NUFFT (register-FFT path with bands and interpolation tiles):
    // two real slices travel as the real and imaginary parts of one complex
    // line through every pass, so a chunk of max_batch slices is
    // ceil(max_batch / 2) lines.  For even D the polar samples j - D/2 run
    // from -D/2 to D/2 - 1; the unpaired sample j = 0 gets a mirror point
    // j = D (radius +s D/2) per angle, nvirt = P of them, stored after the
    // P * D point values of a line, so that every line's point set is
    // Hermitian-symmetric and the two slices separate exactly.
    bool pair_nufft = false;
    int nvirt = 0;
    size_t npts_ext() const { return (size_t)P * N + (size_t)nvirt; }
    int toe_pairs = 1;          // slice pairs per Toeplitz chunk
    double lipschitz = 0.0;

    std::vector<float> angles;
    DevBuf d_cs, d_sn;          // double per-angle cos / sin
    PolarDev geo{};
    DevBuf d_corr;              // float deconvolution factor per mode index, N entries
    FftTables<float> fft_D, fft_nf, fft_M;
    SpreadLists spread;
    SpreadBands bands;          // register-FFT type-1 path (built when it applies)
    InterpTiles itiles;         // register-FFT type-2 path (built when it applies)
    DevBuf d_psf;               // double [2N-1][2N-1] point-spread function
    DevBuf d_phat;              // float [M][M], transposed: phat[kx * M + ky]
    bool toe_fast = false;      // power-of-two M: register FFT kernels
    int toe_lpc = 1;            // image rows per CTA in Toeplitz pass 3
    DevBuf d_phatp;             // float [M][M] spectrum in the register-FFT order
    // detector-axis DFT on the register FFT (tc_nufft_fast.cu): transform
    // length det_M (0: general engine), Bluestein chirp and spectrum when
    // det_M != N
    int det_M = 0;
    bool det_blue = false;
    FftTables<float> fft_det_tw;
    DevBuf d_det_chirp, d_det_bhat;

    // workspace
    DevBuf ws_grid, ws_rows, ws_pts, ws_toe, ws_red;
    DevBuf ws_scalars;          // double scratch for reductions
    cudaStream_t aux = nullptr; // internal stream used for graph capture
    // the instantiated graph of the last graph-captured MBIR solve and the
    // bytes of the arguments it captured; a later solve with the same
    // arguments launches it again instead of capturing a new one
    cudaGraph_t solver_g = nullptr;
    cudaGraphExec_t solver_e = nullptr;
    std::vector<unsigned char> solver_key;

    size_t table_bytes() const;
    size_t workspace_bytes() const;
    ~Plan();
};

// ---- operator launchers (all on `st`, device pointers) -------------------
int plan_build(Plan &pl, const tc_geom &g);
int psf_finish(Plan &pl);  // spectrum + Lipschitz constant from d_psf
int radon_chunk(Plan &pl, const float *x, float *sino, int nb, cudaStream_t st);
int iradon_chunk(Plan &pl, const float *sino, float *x, int nb, int ramp, cudaStream_t st);
// Toeplitz: g = scale_h * H x - aty for nb slices (aty may be null); when
// dots != null the kernel accumulates FP64 partials of x.Hx and x.aty there
// (see toeplitz_dots_count)
// With sel != null the kernels read the buffer index sel[0] from device
// memory and offset x and g by sel[0] * sel_stride floats (solver buffers).
int toeplitz_chunk(Plan &pl, const float *x, const float *aty, float *g, int nb,
                   double *partials, cudaStream_t st, const int *sel = nullptr,
                   size_t sel_stride = 0);
int toeplitz_partials_count(const Plan &pl, int nb);
bool toeplitz_fast_supported(int M);
int toeplitz_fast_lpc(int M);
int toeplitz_fast_row_block(int M);  // image rows per block of pass 1
size_t toeplitz_fast_pair_bytes(int N, int M);  // workspace bytes per slice pair
int toeplitz_fast_chunk(Plan &pl, const float *x, const float *aty, float *g, int nb,
                        double *partials, cudaStream_t st, const int *sel, size_t sel_stride);
int toeplitz_fast_permute(Plan &pl, cudaStream_t st);
int reduce_partials(const double *partials, int nparts, int nvals, double *out,
                    cudaStream_t st);
int qggmrf_launch(const float *x, float *g, int S, int R, int C, float sigma, float p,
                  float scale, cudaStream_t st);
int qggmrf_value_launch(const float *x, int S, int R, int C, float sigma, float p, double *value,
                        double *dsigma, cudaStream_t st);
int qggmrf_hvp_launch(const float *x, const float *v, float *hv, int S, int R, int C, float sigma,
                      float p, float scale, double *vg, double *vgs, cudaStream_t st);
template <typename R>
int fft_lines_launch(const FftTables<R> &T, const cpx<R> *in, cpx<R> *out, int nbatch,
                     int dir, cudaStream_t st);

// type-1 fine-grid FFT on the register FFT (tc_nufft_fast.cu): G is the
// column-major fine grid [nb][nf][nf] (G[b][x][y]), Rw a workspace of
// nb * nf * t1_fast_stride(N) complex;
//   out[b][r][c] = Re FFT2(+)(G)[r - N/2][c - N/2] * corr[r] * corr[c] * scale - sub[b][r][c]
bool t1_fast_supported(int nf);
// With pair != 0 the passes below take the nb slices two at a time as one
// complex line (slice 2q the real part, 2q + 1 the imaginary part, zero when
// nb is odd): ceil(nb / 2) lines of grids, workspaces and point values.
// type-2 fine grid on the register FFT: x [nb][N][N] real -> column-major G
// [lines][nf][nf] = FFT2(-) of x * corr[r] * corr[c] placed at (c - N/2,
// r - N/2) mod nf; Q a workspace of lines * nf * t1_fast_stride(N) complex
int t2_fast_grid(const float *x, c32 *Q, c32 *G, const float *corr, int N, int nf, int nb,
                 const c32 *tw, cudaStream_t st, int pair = 0);
int t1_fast_grid(int N);  // smallest supported fine grid >= 2N, 0 if none
int t1_fast_stride(int N);
// type-1 fine-grid FFT: out[b][r][c] = Re (Im for the odd slice of a pair)
// FFT2(+)(G)[r - N/2][c - N/2] * corr[r] * corr[c] * scale - sub[b][r][c]
int t1_fast_fft(const c32 *G, c32 *Rw, float *out, const float *sub, const float *corr,
                float scale, int N, int nf, int nb, const c32 *tw, cudaStream_t st,
                int pair = 0);
int det_fast_setup(Plan &pl);
// centred detector DFT (+ ramp) of nb slices' sinogram rows into cpts
// [lines][P][N] (pair: lines of pl.npts_ext() values; for even N the j = 0
// value is halved and copied to its mirror point, which makes each slice's
// point set Hermitian-symmetric)
int det_fast(const Plan &pl, const float *sino, c32 *cpts, int nb, int ramp, cudaStream_t st,
             int pair = 0);
// radon's detector step: sino[b][p][t] = scale * Re (centred inverse DFT of
// cpts[b][p][:]); pair: slice 2q from the real part and 2q + 1 from the
// imaginary part of line q, its j = 0 value replaced by the mean of the
// values at j = 0 and at the mirror point
int det_fast_inv(const Plan &pl, const c32 *cpts, float *sino, int nb, float scale,
                 cudaStream_t st, int pair = 0);
std::vector<double> es_correction(int nm, int nf, const EsKernel &es);
int psf_fp64(Plan &pl, const std::vector<double> &cs, const std::vector<double> &sn,
             double *psf, cudaStream_t st);
// time the type-1 spreading for each (tile, points per sub-problem)
// candidate on the plan's geometry and keep the fastest lists in pl.spread
int spread_autotune(Plan &pl, const std::vector<double> &cs, const std::vector<double> &sn);
// register-FFT path: time the band spreading (type-1 transform) for several
// list chunk sizes and NUFFT chunk sizes (slices), keep the fastest
int band_autotune(Plan &pl);
// register-FFT type-2 path: the interpolation tiles (built when they apply)
// and their measured choice of tile edge and points per sub-problem
bool interp_tiles_apply(const Plan &pl);
bool pair_nufft_apply(const Plan &pl);
int interp_autotune(Plan &pl);
int phat_from_psf(Plan &pl, const double *psf, cudaStream_t st);
int nufft_grad_chunk(Plan &pl, const float *x, const float *aty, float *g, int nb,
                     cudaStream_t st);
int mbir_solve(Plan &pl, const float *aty, double sino_sq, float *x, int S,
               const tc_mbir_opts &o, double *history, cudaStream_t st);

// host <-> device copies of the host entry points (tc_hostio.cu): direct for
// pinned host memory, through a pinned staging ring with multi-threaded host
// copies for pageable memory; both return when the copy is complete
int copy_h2d(void *dst, const void *src, size_t bytes);
int copy_d2h(void *dst, const void *src, size_t bytes);
// host [P][S][D] slices s0 .. s0+ns-1 -> device [ns][P][D] (tc_sino_ingest_psd)
int ingest_psd(const float *host, int P, int S, int D, int s0, int ns, float *dev);
// touches every page of a pageable host buffer on background threads, so the
// first-touch page faults of a freshly allocated output overlap the device
// work instead of the final copy; pinned buffers are left alone.  wait() (or
// the destructor) joins the threads.
class HostPrefault {
  public:
    HostPrefault(void *p, size_t bytes);
    ~HostPrefault() { wait(); }
    HostPrefault(const HostPrefault &) = delete;
    HostPrefault &operator=(const HostPrefault &) = delete;
    void wait();

  private:
    std::vector<std::thread> th_;
};

// one scan of a batched solve (tc_batch.cu)
struct BatchScanIn {
    Plan *pl;
    const float *aty;
    double sino_sq;
    float *x;
    int S;
    float sigma, p, weight, step;
};
int mbir_batched(const std::vector<BatchScanIn> &in, int num_iters, int use_graph,
                 int max_attempts, double *history, cudaStream_t st);

}  // namespace tc

// the opaque handle of the C ABI (include/tomocam_b200.h)
struct tc_plan {
    tc::Plan impl;
};
