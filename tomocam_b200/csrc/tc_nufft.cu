// tc_nufft.cu -- radon (type-2 NUFFT + detector DFT) and back-projection
// (detector DFT + type-1 NUFFT) on the polar grid, and the FP64
// point-spread function.
//
// Both transforms use the exponential-of-semicircle kernel on a periodic
// fine grid upsampled by 2 or more (Barnett, Magland & af Klinteberg 2019):
//   type 2: b = FFT(-)(modes * corr) on the fine grid, then
//           c(w) = sum_l psi(w - l h) b_l          (interpolation)
//   type 1: a_l = sum_j c_j psi(l h - w_j)         (spreading)
//           f_m = corr(m) * FFT(+)(a)_m
// with corr(m) = (2 pi / nf) / psi_hat(m).  The fine-grid FFTs skip the
// all-zero rows of the padded mode array and only keep the rows holding
// modes.  Detector-axis DFTs with the reference's fftshift/ifftshift rolls
// (src/forward.cpp:44-47, src/backward.cpp:50-56) are index maps applied
// while lines move between global and shared memory.
//
// The kernels here are the general engine (any 2,3,5,7-smooth fine grid and
// the FP64 point-spread function) plus the band spreading and the
// column-major interpolation of the register-FFT path; that path's FFT and
// detector kernels are in tc_nufft_fast.cu.
#include <algorithm>
#include <cmath>
#include <numeric>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <type_traits>

#include "tc_cpasync.cuh"
#include "tc_plan.cuh"

namespace tc {

__host__ __device__ __forceinline__ int wrapi(int l, int n) {
    int r = l % n;
    return r < 0 ? r + n : r;
}

// fine-grid position of polar point (p, j): first tap index and offset
// xi - l0 in [w/2 - 1, w/2)
__device__ __forceinline__ void point_taps(const PolarDev &g, int p, int j, int nf, int w,
                                           int &lx0, double &fx, int &ly0, double &fy) {
    const double r = g.s * (double)(j - g.half);
    const double inv_h = (double)nf * 0.15915494309189533577;  // nf / (2 pi)
    const double xi = r * g.cs[p] * inv_h;
    const double yi = r * g.sn[p] * inv_h;
    lx0 = (int)ceil(xi - 0.5 * w);
    ly0 = (int)ceil(yi - 0.5 * w);
    fx = xi - (double)lx0;
    fy = yi - (double)ly0;
}

// point index -> (angle p, detector sample j): the P * D detector points,
// then (paired path, even D) the mirror points j = D of each angle
__device__ __forceinline__ void point_of(const PolarDev &g, int idx, int &p, int &j) {
    const int nd = g.P * g.D;
    if (idx < nd) {
        p = idx / g.D;
        j = idx - p * g.D;
    } else {
        p = idx - nd;
        j = g.D;
    }
}

template <typename R>
__device__ __forceinline__ R es_weight(R z, R beta) {
    R q = R(1) - z * z;
    return q > R(0) ? exp(beta * (sqrt(q) - R(1))) : R(0);
}

template <typename R, int WMAX>
__device__ __forceinline__ void es_weights(double off, int w, R beta, R *wt) {
    const R inv_half = R(2) / R(w);
#pragma unroll
    for (int t = 0; t < WMAX; ++t)
        if (t < w) wt[t] = es_weight<R>((R)((double)t - off) * inv_half, beta);
}

constexpr int WMAX32 = 16;  // FP32 operators (tol >= 1e-14)
constexpr int WMAX64 = 16;

// ---------------------------------------------------------------------------
// type 2, pass 1: deconvolve the modes of row r and FFT(-) along x
//   in : x [nb][N][N] real
//   out: rows [nb][N][nf] complex
// ---------------------------------------------------------------------------
template <typename R, typename Tin>
__global__ void __launch_bounds__(FFT_MAX_THREADS, 1)
k_t2_rows(const Tin *__restrict__ x, cpx<R> *__restrict__ rows, int N,
                          const R *__restrict__ corr, FftDev<R> dnf) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cpx<R> *line = reinterpret_cast<cpx<R> *>(smem_raw);
    const int r = blockIdx.x, b = blockIdx.y, nf = dnf.L;
    for (int l = threadIdx.x; l < nf; l += blockDim.x) line[l] = mk<R>(R(0), R(0));
    __syncthreads();
    const Tin *src = x + ((size_t)b * N + r) * N;
    const R cr = corr[r];
    for (int c = threadIdx.x; c < N; c += blockDim.x) {
        int l = wrapi(c - N / 2, nf);
        line[l] = mk<R>((R)src[c] * corr[c] * cr, R(0));
    }
    __syncthreads();
    fft_line<R, -1>(line, nf, 1, dnf, threadIdx.x, blockDim.x);
    cpx<R> *dst = rows + ((size_t)b * N + r) * nf;
    for (int l = threadIdx.x; l < nf; l += blockDim.x) dst[l] = line[l];
}

// ---------------------------------------------------------------------------
// type 2, pass 2: FFT(-) along y of cw adjacent fine-grid columns
//   in : rows [nb][N][nf]   (mode rows only)
//   out: grid [nb][nf][nf]
// ---------------------------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(FFT_MAX_THREADS, 1)
k_t2_cols(const cpx<R> *__restrict__ rows, cpx<R> *__restrict__ grid, int N,
                          int cw, FftDev<R> dnf) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cpx<R> *buf = reinterpret_cast<cpx<R> *>(smem_raw);
    const int nf = dnf.L, b = blockIdx.y, k0 = blockIdx.x * cw;
    for (int q = threadIdx.x; q < cw * nf; q += blockDim.x) buf[q] = mk<R>(R(0), R(0));
    __syncthreads();
    const cpx<R> *src = rows + (size_t)b * N * nf;
    for (int q = threadIdx.x; q < N * cw; q += blockDim.x) {
        int r = q / cw, c = q - r * cw;
        int l2 = wrapi(r - N / 2, nf);
        buf[(size_t)c * nf + l2] = src[(size_t)r * nf + k0 + c];
    }
    __syncthreads();
    fft_line<R, -1>(buf, nf, cw, dnf, threadIdx.x, blockDim.x);
    cpx<R> *dst = grid + (size_t)b * nf * nf;
    for (int q = threadIdx.x; q < nf * cw; q += blockDim.x) {
        int l2 = q / cw, c = q - l2 * cw;
        dst[(size_t)l2 * nf + k0 + c] = buf[(size_t)c * nf + l2];
    }
}

// interpolate point (p, j) from nb fine grids (CM: column-major grids,
// grid[b][x][y])
template <typename R, bool CM = false>
__device__ __forceinline__ void interp_point(const PolarDev &g, int p, int j, int nf, int w,
                                             R beta, const cpx<R> *__restrict__ grid, int nb,
                                             cpx<R> *out /* nb */) {
    int lx0, ly0;
    double fx, fy;
    point_taps(g, p, j, nf, w, lx0, fx, ly0, fy);
    R wx[WMAX32], wy[WMAX32];
    es_weights<R, WMAX32>(fx, w, beta, wx);
    es_weights<R, WMAX32>(fy, w, beta, wy);
    for (int b = 0; b < nb; ++b) out[b] = mk<R>(R(0), R(0));
    if constexpr (CM) {
        for (int tx = 0; tx < w; ++tx) {
            const int gx = wrapi(lx0 + tx, nf);
            for (int b = 0; b < nb; ++b) {
                const cpx<R> *col = grid + ((size_t)b * nf + gx) * nf;
                R ax = R(0), ay = R(0);
                for (int ty = 0; ty < w; ++ty) {
                    const cpx<R> v = col[wrapi(ly0 + ty, nf)];
                    ax += v.x * wy[ty];
                    ay += v.y * wy[ty];
                }
                out[b].x += ax * wx[tx];
                out[b].y += ay * wx[tx];
            }
        }
    } else {
        for (int ty = 0; ty < w; ++ty) {
            const int gy = wrapi(ly0 + ty, nf);
            for (int b = 0; b < nb; ++b) {
                const cpx<R> *row = grid + ((size_t)b * nf + gy) * nf;
                R ax = R(0), ay = R(0);
                for (int tx = 0; tx < w; ++tx) {
                    const cpx<R> v = row[wrapi(lx0 + tx, nf)];
                    ax += v.x * wx[tx];
                    ay += v.y * wx[tx];
                }
                out[b].x += ax * wy[ty];
                out[b].y += ay * wy[ty];
            }
        }
    }
}

constexpr int NB_MAX = 8;

// ---------------------------------------------------------------------------
// type 2, pass 3: interpolate the points of angle p and, in `radon` mode,
// apply the centred inverse DFT along the detector:
//   sino[t] = Re sum_j c_j exp(+2 pi i (j - h)(t - h) / D) / N^2
// (ifftshift, unnormalised IFFT, fftshift; src/forward.cpp:41-51).
// In raw mode the complex point values are stored to cpts [nb][P][D].
// ---------------------------------------------------------------------------
// grid.y splits the nb slices into groups of lpc (lines per CTA)
template <typename R, bool CM = false>
__global__ void __launch_bounds__(FFT_MAX_THREADS, 1)
k_t2_interp(const cpx<R> *__restrict__ grid, float *__restrict__ sino,
            cpx<R> *__restrict__ cpts, PolarDev g, int nf, int w, R beta, int nball, int lpc,
            R scale, FftDev<R> dD) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cpx<R> *buf = reinterpret_cast<cpx<R> *>(smem_raw);
    const int p = blockIdx.x, D = g.D, h = g.half, ld = dD.L;
    const int b0 = blockIdx.y * lpc;
    const int nb = min(lpc, nball - b0);
    grid += (size_t)b0 * nf * nf;
    if (sino) sino += (size_t)b0 * g.P * D;
    if (cpts) cpts += (size_t)b0 * g.P * D;
    for (int j = threadIdx.x; j < D; j += blockDim.x) {
        cpx<R> v[NB_MAX];
        interp_point<R, CM>(g, p, j, nf, w, beta, grid, nb, v);
        if (cpts) {
            for (int b = 0; b < nb; ++b) cpts[((size_t)b * g.P + p) * D + j] = v[b];
        } else {
            const int u = wrapi(j - h, D);
            for (int b = 0; b < nb; ++b) buf[(size_t)b * ld + u] = v[b];
        }
    }
    if (cpts) return;
    __syncthreads();
    fft_line<R, +1>(buf, ld, nb, dD, threadIdx.x, blockDim.x);
    for (int q = threadIdx.x; q < nb * D; q += blockDim.x) {
        const int b = q / D, t = q - b * D;
        sino[((size_t)b * g.P + p) * D + t] = (float)(buf[(size_t)b * ld + wrapi(t - h, D)].x * scale);
    }
}

// ---------------------------------------------------------------------------
// type 2, pass 3 on interpolation tiles (register-FFT path, column-major
// grids grid[b][x][y]): one CTA per sub-problem of the plan's InterpTiles.
// The tile's footprint region -- RW = TS + W - 1 cells from the tile origin
// along x, RP = RW rounded up to even along y, wrapping at nf -- of the nb
// grids is copied into shared memory ([b][dx][dy], pitch RP) as 16-byte
// pieces by cp.async, all in flight at once (a piece is two cells (gy, gy+1)
// with gy even, so it never straddles the wrap: TS and nf are even); then
// each thread interpolates points of the sub-problem from there: per slice,
// x taps outer and y taps inner as interp_point, with the kernel weights of
// the band spreading (es_weight_fast), written to cpts [nb][P][D].  A
// point's entry (InterpEntry, built with the lists) carries its index, its
// first tap's offset in the region and the fractional tap offsets, so no
// per-point geometry is evaluated here.  TS and W (tile edge, kernel width)
// are template parameters: the region's shape is compile-time, so the 49
// (say) taps of a slice are loads at immediate offsets from one address and
// the weights stay in registers.
// ---------------------------------------------------------------------------
// ES kernel weight exp(beta (sqrt(1 - z^2) - 1)) for |z| < 1, else 0, on the
// fast hardware square root and exponential (relative error ~1e-6)
__device__ __forceinline__ float es_weight_fast(float z, float beta) {
    const float q = 1.f - z * z;
    return q > 0.f ? __expf(beta * (q * rsqrtf(q) - 1.f)) : 0.f;
}

__host__ __device__ constexpr int interp_pitch(int ts, int w) { return (ts + w) & ~1; }

__device__ __forceinline__ InterpEntry load_entry(const InterpEntry *__restrict__ e, int i) {
    const int4 v = __ldg(reinterpret_cast<const int4 *>(e) + i);
    return InterpEntry{v.x, v.y, __int_as_float(v.z), __int_as_float(v.w)};
}
constexpr int INTERP_THREADS = 256;  // 512 measured the same

template <int TS, int W>
__global__ void __launch_bounds__(INTERP_THREADS)
k_t2_interp_tile(const c32 *__restrict__ grid, c32 *__restrict__ cpts,
                 const InterpEntry *__restrict__ entries, const SpreadSub *__restrict__ subs,
                 int nf, int ntiles, float beta, int nb, size_t npts) {
    constexpr int RW = TS + W - 1, RP = interp_pitch(TS, W), HP = RP / 2;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    c32 *reg = reinterpret_cast<c32 *>(smem_raw);
    const SpreadSub sb = subs[blockIdx.x];
    const int ty0 = (sb.tile / ntiles) * TS, tx0 = (sb.tile % ntiles) * TS;
    const int npiece = nb * RW * HP;
    for (int q = threadIdx.x; q < npiece; q += INTERP_THREADS) {
        const int col = q / HP, h = q - col * HP;  // col = b * RW + dx
        const int b = col / RW, dx = col - b * RW;
        int gx = tx0 + dx, gy = ty0 + 2 * h;
        if (gx >= nf) gx -= nf;
        if (gy >= nf) gy -= nf;
        cp_async16(reg + col * RP + 2 * h, grid + ((size_t)b * nf + gx) * nf + gy);
    }
    cp_async_commit();
    cp_async_wait_all();
    __syncthreads();
    constexpr float inv_half = 2.f / (float)W;
    for (int i = threadIdx.x; i < sb.count; i += INTERP_THREADS) {
        const InterpEntry e = load_entry(entries, sb.start + i);
        const int pt = e.pt;
        float wx[W], wy[W];
#pragma unroll
        for (int t = 0; t < W; ++t) {
            wx[t] = es_weight_fast(((float)t - e.fx) * inv_half, beta);
            wy[t] = es_weight_fast(((float)t - e.fy) * inv_half, beta);
        }
        // the point's first tap inside the region (its tile holds it)
        const c32 *base = reg + e.off;
        for (int b = 0; b < nb; ++b, base += RW * RP) {
            float ox = 0.f, oy = 0.f;
#pragma unroll
            for (int tx = 0; tx < W; ++tx) {
                float ax = 0.f, ay = 0.f;
#pragma unroll
                for (int ty = 0; ty < W; ++ty) {
                    const c32 v = base[tx * RP + ty];
                    ax = fmaf(v.x, wy[ty], ax);
                    ay = fmaf(v.y, wy[ty], ay);
                }
                ox = fmaf(ax, wx[tx], ox);
                oy = fmaf(ay, wx[tx], oy);
            }
            cpts[(size_t)b * npts + pt] = mk<float>(ox, oy);
        }
    }
}

// Lane form of the same interpolation for chunks of 5 .. 8 lines.  The
// thread-per-point form reads the region at 32 unrelated addresses per warp
// request, and most of its shared-memory wavefronts were bank conflicts.
// Here a point is taken by a group of 16 lanes, lane (b, h) = line b, the y
// taps of parity h; the region's planes are PL cells apart with PL = 2 mod
// 16, so the group's 8-byte reads of one tap step land on the bank pairs
// b PL + h = 2b + h (mod 16), all distinct: one wavefront per half-warp.
// The point's 2W kernel weights are evaluated once (lane k: x tap k, lane
// W + k: y tap k) and passed by shuffles; the two parities' sums are added
// by one more.  Per line the taps are summed x outer, y inner, each parity
// separately, so results match the thread-per-point form to rounding.
__host__ __device__ constexpr int interp_plane(int ts, int w) {
    return (ts + w - 1) * interp_pitch(ts, w) +
           ((2 - (ts + w - 1) * interp_pitch(ts, w)) % 16 + 16) % 16;
}
constexpr int INTERP_LANES_MIN_NB = 5;  // chunks of at least this many lines take the lane form

template <int TS, int W>
__global__ void __launch_bounds__(INTERP_THREADS)
k_t2_interp_lanes(const c32 *__restrict__ grid, c32 *__restrict__ cpts,
                  const InterpEntry *__restrict__ entries, const SpreadSub *__restrict__ subs,
                  int nf, int ntiles, float beta, int nb, size_t npts) {
    constexpr int RW = TS + W - 1, RP = interp_pitch(TS, W), HP = RP / 2, PL = interp_plane(TS, W);
    constexpr int KY = (W + 1) / 2;  // y taps of one parity, at most
    constexpr int NG = INTERP_THREADS / 16;
    static_assert(2 * W <= 16, "one kernel weight per lane of a group");
    static_assert(PL % 16 == 2 && RP % 2 == 0, "plane stride 2 mod 16 cells, 16-byte pieces");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    c32 *reg = reinterpret_cast<c32 *>(smem_raw);
    const SpreadSub sb = subs[blockIdx.x];
    const int ty0 = (sb.tile / ntiles) * TS, tx0 = (sb.tile % ntiles) * TS;
    const int npiece = nb * RW * HP;
    for (int q = threadIdx.x; q < npiece; q += INTERP_THREADS) {
        const int col = q / HP, hh = q - col * HP;  // col = b * RW + dx
        const int bb = col / RW, dx = col - bb * RW;
        int gx = tx0 + dx, gy = ty0 + 2 * hh;
        if (gx >= nf) gx -= nf;
        if (gy >= nf) gy -= nf;
        cp_async16(reg + bb * PL + dx * RP + 2 * hh, grid + ((size_t)bb * nf + gx) * nf + gy);
    }
    cp_async_commit();
    cp_async_wait_all();
    __syncthreads();
    const int lane = threadIdx.x & 31, gbase = lane & 16;
    const int gl = lane & 15, b = gl >> 1, h = gl & 1;
    constexpr float inv_half = 2.f / (float)W;
    // i0 is uniform over the warp (its two groups take points i0, i0 + 1), so
    // every lane reaches every shuffle
    for (int i0 = (threadIdx.x >> 5) * 2; i0 < sb.count; i0 += NG) {
        const int i = i0 + (gbase >> 4);
        const bool act = i < sb.count;
        const InterpEntry e = load_entry(entries, sb.start + (act ? i : i0));
        const float f = gl < W ? e.fx : e.fy;
        const int tk = gl < W ? gl : gl - W;
        const float wl = gl < 2 * W ? es_weight_fast(((float)tk - f) * inv_half, beta) : 0.f;
        float wx[W], wy[KY];
#pragma unroll
        for (int t = 0; t < W; ++t) wx[t] = __shfl_sync(0xffffffffu, wl, gbase + t);
#pragma unroll
        for (int k = 0; k < KY; ++k) {
            const int src = W + 2 * k + h;  // y tap 2k + h (lane 15 holds 0 past the last)
            wy[k] = __shfl_sync(0xffffffffu, wl, gbase + (src < 16 ? src : 15));
        }
        float ox = 0.f, oy = 0.f;
        if (b < nb) {
            // the point's first tap inside the region (its tile holds it)
            const c32 *base = reg + b * PL + e.off + h;
#pragma unroll
            for (int tx = 0; tx < W; ++tx) {
                float ax = 0.f, ay = 0.f;
#pragma unroll
                for (int k = 0; k < KY; ++k) {
                    if (2 * k + h < W) {
                        const c32 v = base[tx * RP + 2 * k];
                        ax = fmaf(v.x, wy[k], ax);
                        ay = fmaf(v.y, wy[k], ay);
                    }
                }
                ox = fmaf(ax, wx[tx], ox);
                oy = fmaf(ay, wx[tx], oy);
            }
        }
        ox += __shfl_xor_sync(0xffffffffu, ox, 1);
        oy += __shfl_xor_sync(0xffffffffu, oy, 1);
        if (act && b < nb && h == 0) cpts[(size_t)b * npts + e.pt] = mk<float>(ox, oy);
    }
}

// ---------------------------------------------------------------------------
// type 1, pass 0: centred forward DFT of sinogram rows (+ Ram-Lak ramp)
//   c_j = sum_t y_t exp(-2 pi i (t - h)(j - h) / D) [* |j - h| / D]
// (src/backward.cpp:47-58, src/gpu/ramlak.cu:15-31)
// ---------------------------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(FFT_MAX_THREADS, 1)
k_t1_det(const float *__restrict__ sino, cpx<R> *__restrict__ cpts, int P, int D, int nball,
         int lpc, int ramp, FftDev<R> dD) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cpx<R> *buf = reinterpret_cast<cpx<R> *>(smem_raw);
    const int p = blockIdx.x, h = D / 2, ld = dD.L;
    const int b0 = blockIdx.y * lpc;
    const int nb = min(lpc, nball - b0);
    sino += (size_t)b0 * P * D;
    cpts += (size_t)b0 * P * D;
    for (int q = threadIdx.x; q < nb * D; q += blockDim.x) {
        const int b = q / D, t = q - b * D;
        buf[(size_t)b * ld + wrapi(t - h, D)] = mk<R>((R)sino[((size_t)b * P + p) * D + t], R(0));
    }
    __syncthreads();
    fft_line<R, -1>(buf, ld, nb, dD, threadIdx.x, blockDim.x);
    for (int q = threadIdx.x; q < nb * D; q += blockDim.x) {
        const int b = q / D, j = q - b * D;
        cpx<R> v = buf[(size_t)b * ld + wrapi(j - h, D)];
        if (ramp) {
            const R f = (R)abs(j - h) / (R)D;
            v = v * f;
        }
        cpts[((size_t)b * P + p) * D + j] = v;
    }
}

// ---------------------------------------------------------------------------
// type 1, pass 1: spread the points of one tile sub-problem into shared
// memory and write the tile (plain store, or atomic add when the tile is
// shared between sub-problems).  cpts == null spreads unit strengths.
// ---------------------------------------------------------------------------
template <typename R, int TS, bool CM>
__global__ void k_spread(const cpx<R> *__restrict__ cpts, cpx<R> *__restrict__ grid,
                         const int *__restrict__ points, const SpreadSub *__restrict__ subs,
                         PolarDev g, int nf, int ntiles, int w, R beta, int nb) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    // [nb][2][TS][TS + 1]: real and imaginary planes, rows padded by one so
    // that a cell's bank depends on its row and column (the taps of a warp's
    // points, along any direction, spread over the banks)
    R *acc = reinterpret_cast<R *>(smem_raw);
    constexpr int RS = TS + 1, PL = TS * RS;
    const SpreadSub sb = subs[blockIdx.x];
    const int ty0 = (sb.tile / ntiles) * TS, tx0 = (sb.tile % ntiles) * TS;
    for (int q = threadIdx.x; q < nb * 2 * PL; q += blockDim.x) acc[q] = R(0);
    __syncthreads();
    const size_t npts = (size_t)g.P * g.D;
    for (int i = threadIdx.x; i < sb.count; i += blockDim.x) {
        const int pt = points[sb.start + i];
        const int p = pt / g.D, j = pt - p * g.D;
        int lx0, ly0;
        double fx, fy;
        point_taps(g, p, j, nf, w, lx0, fx, ly0, fy);
        R wx[WMAX64], wy[WMAX64];
        es_weights<R, WMAX64>(fx, w, beta, wx);
        es_weights<R, WMAX64>(fy, w, beta, wy);
        cpx<R> c[NB_MAX];
        for (int b = 0; b < nb; ++b) c[b] = cpts ? cpts[b * npts + pt] : mk<R>(R(1), R(0));
        for (int ty = 0; ty < w; ++ty) {
            const int dy = wrapi(ly0 + ty, nf) - ty0;
            if (dy < 0 || dy >= TS) continue;
            for (int tx = 0; tx < w; ++tx) {
                const int dx = wrapi(lx0 + tx, nf) - tx0;
                if (dx < 0 || dx >= TS) continue;
                const R wgt = wy[ty] * wx[tx];
                for (int b = 0; b < nb; ++b) {
                    R *a = acc + (size_t)b * 2 * PL + dy * RS + dx;
                    atomicAdd(a, c[b].x * wgt);
                    atomicAdd(a + PL, c[b].y * wgt);
                }
            }
        }
    }
    __syncthreads();
    for (int q = threadIdx.x; q < nb * TS * TS; q += blockDim.x) {
        const int b = q / (TS * TS), cell = q - b * TS * TS;
        // consecutive threads take consecutive cells of the stored layout's
        // contiguous axis (x for row-major, y for column-major)
        const int dy = CM ? cell % TS : cell / TS, dx = CM ? cell / TS : cell % TS;
        const int gy = ty0 + dy, gx = tx0 + dx;
        if (gy >= nf || gx >= nf) continue;
        cpx<R> *dst = grid + (CM ? ((size_t)b * nf + gx) * nf + gy : ((size_t)b * nf + gy) * nf + gx);
        const R *a = acc + (size_t)b * 2 * PL + dy * RS + dx;
        if (sb.shared) {
            atomicAdd(&dst->x, a[0]);
            atomicAdd(&dst->y, a[PL]);
        } else {
            *dst = mk<R>(a[0], a[PL]);
        }
    }
}

// zero the tiles that several sub-problems add into
template <typename R, int TS, bool CM>
__global__ void k_zero_tiles(cpx<R> *__restrict__ grid, const int *__restrict__ tiles,
                             int nf, int ntiles, int nb) {
    const int tile = tiles[blockIdx.x];
    const int ty0 = (tile / ntiles) * TS, tx0 = (tile % ntiles) * TS;
    for (int q = threadIdx.x; q < nb * TS * TS; q += blockDim.x) {
        const int b = q / (TS * TS), cell = q - b * TS * TS;
        const int gy = ty0 + (CM ? cell % TS : cell / TS), gx = tx0 + (CM ? cell / TS : cell % TS);
        if (gy < nf && gx < nf)
            grid[CM ? ((size_t)b * nf + gx) * nf + gy : ((size_t)b * nf + gy) * nf + gx] =
                mk<R>(R(0), R(0));
    }
}

// ---------------------------------------------------------------------------
// type 1, pass 1 on bands (register-FFT path, column-major grid
// grid[b][x][y]): one warp per chunk of a band's point list.  Lane
// (rho, c) = (lane / 8, lane % 8) takes tap (rho - dy0, c) of the current
// point, i.e. cell (rho, dx0 + c) of the band.  The accumulator holds
// [line][row][BAND_RS] complex values with BAND_RS = 40 (= 8 mod 16), so a
// point's 32 lane cells fill the 16 bank pairs twice each, the minimum for
// 8-byte accesses; it belongs to the warp alone, so plain shared-memory adds
// suffice, __syncwarp ordering consecutive points.  Each of the first 16
// lanes evaluates one kernel weight (lanes 0-7 the columns, 8-15 the rows),
// shuffled to the lanes that use it.  Entries and their point values are
// loaded two and one points ahead.
// ---------------------------------------------------------------------------
constexpr int BAND_RS = BAND_W + 8;
constexpr int BAND_WARPS = 8;
static_assert(BAND_H * 8 == 32, "a band row group is one warp of 8-lane rows");

template <int NB>
__global__ void __launch_bounds__(BAND_WARPS * 32, NB <= 3 ? 6 : NB == 4 ? 5 : 4)
k_spread_band(const c32 *__restrict__ cpts, c32 *__restrict__ grid,
              const BandEntry *__restrict__ ent, const BandChunk *__restrict__ chunks,
              int nchunk, int nf, int npts, int w, float beta) {
    constexpr int nb = NB;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int ci = blockIdx.x * BAND_WARPS + wid;
    if (ci >= nchunk) return;  // no block-wide barrier below
    constexpr int PLANE = BAND_H * BAND_RS;  // one line's complex cells
    c32 *acc = reinterpret_cast<c32 *>(smem_raw) + (size_t)wid * nb * PLANE;
    for (int q = lane; q < nb * PLANE; q += 32) acc[q] = mk<float>(0.f, 0.f);
    const BandChunk ch = chunks[ci];
    const int rho = lane >> 3, c = lane & 7;
    const float inv_half = 2.f / (float)w;
    const bool wlane = lane < 16 && (lane & 7) < w;  // evaluates weight (lane & 7)
    auto load_vals = [&](const BandEntry &e, c32 *v) {
#pragma unroll
        for (int b = 0; b < NB; ++b)
            v[b] = cpts ? cpts[(size_t)b * npts + e.pt] : mk<float>(1.f, 0.f);
    };
    __syncwarp();
    BandEntry en{}, nx{};
    c32 v[NB], vn[NB];
    if (ch.count > 0) {
        en = ent[ch.start];
        load_vals(en, v);
    }
    if (ch.count > 1) nx = ent[ch.start + 1];
    for (int e = 0; e < ch.count; ++e) {
        BandEntry nn{};
        if (e + 2 < ch.count) nn = ent[ch.start + e + 2];
        if (e + 1 < ch.count) load_vals(nx, vn);
        const int dx0 = (int)(short)(en.dxy & 0xffff), dy0 = en.dxy >> 16;
        // lane l < 8: column weight of tap l; 8 <= l < 16: row weight of tap l - 8
        const float zf = ((float)(lane & 7) - (lane < 8 ? en.fx : en.fy)) * inv_half;
        const float f = wlane ? es_weight_fast(zf, beta) : 0.f;
        const int ty = rho - dy0, col = dx0 + c;
        const float wxc = __shfl_sync(0xffffffffu, f, c);
        const float wyr = __shfl_sync(0xffffffffu, f, 8 + (ty & 7));
        if (c < w && ty >= 0 && ty < w && col >= 0 && col < BAND_W) {
            const float wgt = wxc * wyr;
            c32 *a = acc + rho * BAND_RS + col;
#pragma unroll
            for (int b = 0; b < NB; ++b) {
                c32 t = a[b * PLANE];
                t.x = fmaf(v[b].x, wgt, t.x);
                t.y = fmaf(v[b].y, wgt, t.y);
                a[b * PLANE] = t;
            }
        }
        __syncwarp();
        en = nx;
        nx = nn;
#pragma unroll
        for (int b = 0; b < NB; ++b) v[b] = vn[b];
    }
    // store the band: lane (column lane / 4 + 8 k, row lane % 4); the four
    // rows of a column are 32 contiguous bytes of the column-major grid
    const int nbx = nf / BAND_W;
    const int bx = ch.band % nbx, by = ch.band / nbx;
    const int r = lane & 3;
    for (int b = 0; b < nb; ++b)
        for (int k = 0; k < BAND_W / 8; ++k) {
            const int cc = (lane >> 2) + 8 * k;
            const c32 val = acc[b * PLANE + r * BAND_RS + cc];
            c32 *dst = grid + ((size_t)b * nf + bx * BAND_W + cc) * nf + by * BAND_H + r;
            if (ch.shared) {
                atomicAdd(&dst->x, val.x);
                atomicAdd(&dst->y, val.y);
            } else {
                *dst = val;
            }
        }
}

// ---------------------------------------------------------------------------
// type 1, pass 1 on bands with the accumulator in registers (chunks of 8
// slices): lane (b, r) = (lane / 4, lane % 4) owns row r of the band for
// slice b, 32 complex cells in registers, so a point adds its taps with no
// shared-memory traffic.  Every lane takes the point's value of its own
// slice, its row weight and the W column weights (evaluated by 2W lanes and
// shuffled, as in k_spread_band) and adds to the cells dx0 .. dx0+W-1 of its
// row: a switch on dx0 (the same for the whole warp, one point at a time)
// whose cases name the cells at compile time.  Same lists, chunks, weights,
// products and per-cell summation order as k_spread_band, so the grids are
// bit-identical; a warp issues about a quarter of the instructions per point.
// ---------------------------------------------------------------------------
template <int W, int D>
__device__ __forceinline__ void band_row_add(float2 (&acc)[BAND_W], const float (&wx)[8], float wyr,
                                             c32 v) {
#pragma unroll
    for (int c = 0; c < W; ++c) {
        const int k = D + c;
        if (k >= 0 && k < BAND_W) {
            const float wgt = wx[c] * wyr;
            acc[k].x = fmaf(v.x, wgt, acc[k].x);
            acc[k].y = fmaf(v.y, wgt, acc[k].y);
        }
    }
}

constexpr int BAND8_NB = 8;
static_assert(BAND8_NB * BAND_H == 32, "a warp's lanes are the chunk's slices x the band's rows");

template <int W>
__global__ void __launch_bounds__(BAND_WARPS * 32, 2)
k_spread_band8(const c32 *__restrict__ cpts, c32 *__restrict__ grid,
               const BandEntry *__restrict__ ent, const BandChunk *__restrict__ chunks, int nchunk,
               int nf, int npts, float beta) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int ci = blockIdx.x * BAND_WARPS + wid;
    if (ci >= nchunk) return;  // no block-wide barrier below
    const int b = lane >> 2, r = lane & 3;
    float2 acc[BAND_W];
#pragma unroll
    for (int k = 0; k < BAND_W; ++k) acc[k] = make_float2(0.f, 0.f);
    const BandChunk ch = chunks[ci];
    const float inv_half = 2.f / (float)W;
    const bool wlane = lane < 16 && (lane & 7) < W;  // evaluates weight (lane & 7)
    auto load_val = [&](const BandEntry &e) {
        return cpts ? cpts[(size_t)b * npts + e.pt] : mk<float>(1.f, 0.f);
    };
    BandEntry en{}, nx{};
    c32 v = mk<float>(0.f, 0.f), vn = v;
    if (ch.count > 0) {
        en = ent[ch.start];
        v = load_val(en);
    }
    if (ch.count > 1) nx = ent[ch.start + 1];
    for (int e = 0; e < ch.count; ++e) {
        BandEntry nn{};
        if (e + 2 < ch.count) nn = ent[ch.start + e + 2];
        if (e + 1 < ch.count) vn = load_val(nx);
        const int dx0 = (int)(short)(en.dxy & 0xffff), dy0 = en.dxy >> 16;
        // lane l < 8: column weight of tap l; 8 <= l < 16: row weight of tap l - 8
        const float zf = ((float)(lane & 7) - (lane < 8 ? en.fx : en.fy)) * inv_half;
        const float f = wlane ? es_weight_fast(zf, beta) : 0.f;
        float wx[8];
#pragma unroll
        for (int c = 0; c < 8; ++c) wx[c] = __shfl_sync(0xffffffffu, f, c);
        const int ty = r - dy0;
        const float wyr = __shfl_sync(0xffffffffu, f, 8 + (ty & 7));
        if (ty >= 0 && ty < W) {
            switch (dx0) {
#define TC_BAND_CASE(D) \
    case D: band_row_add<W, D>(acc, wx, wyr, v); break;
                TC_BAND_CASE(-7) TC_BAND_CASE(-6) TC_BAND_CASE(-5) TC_BAND_CASE(-4)
                TC_BAND_CASE(-3) TC_BAND_CASE(-2) TC_BAND_CASE(-1) TC_BAND_CASE(0)
                TC_BAND_CASE(1) TC_BAND_CASE(2) TC_BAND_CASE(3) TC_BAND_CASE(4)
                TC_BAND_CASE(5) TC_BAND_CASE(6) TC_BAND_CASE(7) TC_BAND_CASE(8)
                TC_BAND_CASE(9) TC_BAND_CASE(10) TC_BAND_CASE(11) TC_BAND_CASE(12)
                TC_BAND_CASE(13) TC_BAND_CASE(14) TC_BAND_CASE(15) TC_BAND_CASE(16)
                TC_BAND_CASE(17) TC_BAND_CASE(18) TC_BAND_CASE(19) TC_BAND_CASE(20)
                TC_BAND_CASE(21) TC_BAND_CASE(22) TC_BAND_CASE(23) TC_BAND_CASE(24)
                TC_BAND_CASE(25) TC_BAND_CASE(26) TC_BAND_CASE(27) TC_BAND_CASE(28)
                TC_BAND_CASE(29) TC_BAND_CASE(30) TC_BAND_CASE(31)
#undef TC_BAND_CASE
                default: break;
            }
        }
        en = nx;
        nx = nn;
        v = vn;
    }
    // store the band: row r of slice b, column by column (the four rows of a
    // column are 32 contiguous bytes of the column-major grid)
    const int nbx = nf / BAND_W;
    const int bx = ch.band % nbx, by = ch.band / nbx;
    c32 *dst = grid + ((size_t)b * nf + bx * BAND_W) * nf + by * BAND_H + r;
#pragma unroll
    for (int k = 0; k < BAND_W; ++k) {
        if (ch.shared) {
            atomicAdd(&dst[(size_t)k * nf].x, acc[k].x);
            atomicAdd(&dst[(size_t)k * nf].y, acc[k].y);
        } else {
            dst[(size_t)k * nf] = mk<float>(acc[k].x, acc[k].y);
        }
    }
}

// zero the bands that several chunks add into (column-major grid)
__global__ void k_zero_bands(c32 *__restrict__ grid, const int *__restrict__ bands, int nf,
                             int nb) {
    const int band = bands[blockIdx.x], nbx = nf / BAND_W;
    const int bx = band % nbx, by = band / nbx;
    for (int q = threadIdx.x; q < nb * BAND_W * BAND_H; q += blockDim.x) {
        const int b = q / (BAND_W * BAND_H), cell = q - b * BAND_W * BAND_H;
        const int cc = cell / BAND_H, r = cell - cc * BAND_H;
        grid[((size_t)b * nf + bx * BAND_W + cc) * nf + by * BAND_H + r] = mk<float>(0.f, 0.f);
    }
}

// ---------------------------------------------------------------------------
// type 1, pass 2: FFT(+) along y of cw adjacent columns, keep the mode rows
//   in : grid [nb][nf][nf];  out: rows [nb][nm][nf]
// ---------------------------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(FFT_MAX_THREADS, 1)
k_t1_cols(const cpx<R> *__restrict__ grid, cpx<R> *__restrict__ rows, int nm,
                          int cw, FftDev<R> dnf) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cpx<R> *buf = reinterpret_cast<cpx<R> *>(smem_raw);
    const int nf = dnf.L, b = blockIdx.y, k0 = blockIdx.x * cw;
    const cpx<R> *src = grid + (size_t)b * nf * nf;
    for (int q = threadIdx.x; q < nf * cw; q += blockDim.x) {
        int l2 = q / cw, c = q - l2 * cw;
        buf[(size_t)c * nf + l2] = src[(size_t)l2 * nf + k0 + c];
    }
    __syncthreads();
    fft_line<R, +1>(buf, nf, cw, dnf, threadIdx.x, blockDim.x);
    cpx<R> *dst = rows + (size_t)b * nm * nf;
    for (int q = threadIdx.x; q < nm * cw; q += blockDim.x) {
        int r = q / cw, c = q - r * cw;
        dst[(size_t)r * nf + k0 + c] = buf[(size_t)c * nf + wrapi(r - nm / 2, nf)];
    }
}

// ---------------------------------------------------------------------------
// type 1, pass 3: FFT(+) along x of mode row r, deconvolve, real part
//   out[b][r][c] = Re(.) * corr[c] * corr[r] * scale - sub[b][r][c]
// ---------------------------------------------------------------------------
template <typename R, typename Tout>
__global__ void __launch_bounds__(FFT_MAX_THREADS, 1)
k_t1_rows(const cpx<R> *__restrict__ rows, Tout *__restrict__ out,
                          const float *__restrict__ sub, int nm, const R *__restrict__ corr,
                          R scale, FftDev<R> dnf) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cpx<R> *line = reinterpret_cast<cpx<R> *>(smem_raw);
    const int r = blockIdx.x, b = blockIdx.y, nf = dnf.L;
    const cpx<R> *src = rows + ((size_t)b * nm + r) * nf;
    for (int l = threadIdx.x; l < nf; l += blockDim.x) line[l] = src[l];
    __syncthreads();
    fft_line<R, +1>(line, nf, 1, dnf, threadIdx.x, blockDim.x);
    const R cr = corr[r] * scale;
    Tout *dst = out + ((size_t)b * nm + r) * nm;
    const float *sb = sub ? sub + ((size_t)b * nm + r) * nm : nullptr;
    for (int c = threadIdx.x; c < nm; c += blockDim.x) {
        R v = line[wrapi(c - nm / 2, nf)].x * corr[c] * cr;
        if (sb) v -= (R)sb[c];
        dst[c] = (Tout)v;
    }
}

// ===========================================================================
// host side
// ===========================================================================
void EsKernel::set(double tol) {
    w = (int)std::ceil(std::log10(1.0 / tol)) + 1;
    if (w < 2) w = 2;
    if (w > 16) w = 16;
    beta = 2.30 * w;
}

// Gauss-Legendre nodes and weights on [-1, 1] (Newton iteration on P_n)
static void gauss_legendre(int n, std::vector<double> &x, std::vector<double> &wq) {
    x.resize(n);
    wq.resize(n);
    for (int i = 0; i < n; ++i) {
        double z = std::cos(M_PI * (i + 0.75) / (n + 0.5));
        double dp = 0;
        for (int it = 0; it < 100; ++it) {
            double p0 = 1.0, p1 = z;
            for (int k = 2; k <= n; ++k) {
                double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
                p0 = p1;
                p1 = p2;
            }
            dp = n * (z * p1 - p0) / (z * z - 1.0);
            double dz = p1 / dp;
            z -= dz;
            if (std::fabs(dz) < 1e-16) break;
        }
        x[i] = z;
        wq[i] = 2.0 / ((1.0 - z * z) * dp * dp);
    }
}

// corr[i] = (2 pi / nf) / psi_hat(i - nm/2), psi(t) = phi(2t / (w h)), h = 2 pi / nf
std::vector<double> es_correction(int nm, int nf, const EsKernel &es) {
    std::vector<double> xq, wq;
    gauss_legendre(4 * es.w + 40, xq, wq);
    const double half = 0.5 * es.w * (2.0 * M_PI / nf);
    std::vector<double> phi(xq.size());
    for (size_t q = 0; q < xq.size(); ++q)
        phi[q] = std::exp(es.beta * (std::sqrt(1.0 - xq[q] * xq[q]) - 1.0));
    std::vector<double> corr(nm);
    for (int i = 0; i < nm; ++i) {
        const double k = (double)(i - nm / 2);
        double s = 0;
        for (size_t q = 0; q < xq.size(); ++q) s += wq[q] * phi[q] * std::cos(k * xq[q] * half);
        corr[i] = (2.0 * M_PI / nf) / (half * s);
    }
    return corr;
}

// lines per CTA for column passes: cw * nf * sizeof <= 128 KB, threads <= 1024
template <typename R>
static int col_width(int nf) {
    int cw = 8;
    while (cw > 1 && ((size_t)cw * nf * sizeof(cpx<R>) > 128 * 1024 ||
                      fft_threads<R>(nf, cw) > FFT_MAX_THREADS || nf % cw))
        cw /= 2;
    return cw;
}

template <typename K>
static int set_smem(K kernel, size_t smem) {
    if (smem > 227 * 1024) TC_FAIL(TC_ERR_SHAPE, "transform too large for shared memory");
    TC_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    return TC_OK;
}

// tiles touched along one axis by the taps l0 - 1 .. l0 + w of a point (one
// cell of margin each side, so a rounding difference in the tap origin can
// never leave a tap outside its point's lists); at most 3 with wrap-around
__device__ __forceinline__ int axis_tiles(int l0, int w, int nf, int ts, int *t) {
    int n = 0;
    for (int l = l0 - 1; l <= l0 + w; ++l) {
        const int tt = wrapi(l, nf) / ts;
        bool seen = false;
        for (int k = 0; k < n; ++k) seen |= (t[k] == tt);
        if (!seen && n < 4) t[n++] = tt;
    }
    return n;
}

// count (cursor == null) or place (cursor != null) every point in the lists
// of the tiles its taps touch; the tap origins are the spreading kernel's own
// (point_taps)
__global__ void k_tile_lists(PolarDev g, int nf, int w, int ts, int ntiles, int *__restrict__ counts,
                             int *__restrict__ cursor, int *__restrict__ flat, unsigned stride) {
    const int npts = g.P * g.D;
    for (int it = blockIdx.x * blockDim.x + threadIdx.x; it < npts; it += gridDim.x * blockDim.x) {
        // points are visited in the order it * stride (mod npts), a
        // permutation (stride coprime to npts), so the placement atomics fill
        // each tile's list with points of many rays in turn rather than runs
        // of one ray's neighbouring points
        const int idx = (int)(((unsigned long long)it * stride) % (unsigned)npts);
        const int p = idx / g.D, j = idx - p * g.D;
        int lx0, ly0;
        double fx, fy;
        point_taps(g, p, j, nf, w, lx0, fx, ly0, fy);
        int tx[4], ty[4];
        const int nx = axis_tiles(lx0, w, nf, ts, tx), ny = axis_tiles(ly0, w, nf, ts, ty);
        for (int a = 0; a < ny; ++a)
            for (int b = 0; b < nx; ++b) {
                const int tile = ty[a] * ntiles + tx[b];
                if (cursor) flat[atomicAdd(cursor + tile, 1)] = idx;
                else atomicAdd(counts + tile, 1);
            }
    }
}

// count (cursor == null) or place (cursor != null) every point in the list
// of the interpolation tile that holds its first tap (point_taps'), in point
// order within the warps' atomics
__global__ void k_interp_lists(PolarDev g, int nf, int w, int ts, int ntiles,
                               int *__restrict__ counts, int *__restrict__ cursor,
                               InterpEntry *__restrict__ flat, int nvirt) {
    const int npts = g.P * g.D + nvirt;
    const int pitch = interp_pitch(ts, w);
    for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < npts; idx += gridDim.x * blockDim.x) {
        int p, j;
        point_of(g, idx, p, j);
        int lx0, ly0;
        double fx, fy;
        point_taps(g, p, j, nf, w, lx0, fx, ly0, fy);
        const int lx = wrapi(lx0, nf), ly = wrapi(ly0, nf);
        const int tile = (ly / ts) * ntiles + lx / ts;
        if (cursor)
            flat[atomicAdd(cursor + tile, 1)] =
                InterpEntry{idx, (lx % ts) * pitch + ly % ts, (float)fx, (float)fy};
        else atomicAdd(counts + tile, 1);
    }
}

// count (cursor == null) or place (cursor != null) every point in the lists
// of the bands its taps touch (at most 2 band columns and 3 band rows for
// w <= 8), with its first tap relative to each band; the tap origin is
// point_taps', the one the entry then carries to the spreading
__global__ void k_band_lists(PolarDev g, int nf, int w, int *__restrict__ counts,
                             int *__restrict__ cursor, BandEntry *__restrict__ out,
                             unsigned stride, int nvirt) {
    const int npts = g.P * g.D + nvirt, nbx = nf / BAND_W;
    for (int it = blockIdx.x * blockDim.x + threadIdx.x; it < npts; it += gridDim.x * blockDim.x) {
        const int idx = (int)(((unsigned long long)it * stride) % (unsigned)npts);
        int p, j;
        point_of(g, idx, p, j);
        int lx0, ly0;
        double fx, fy;
        point_taps(g, p, j, nf, w, lx0, fx, ly0, fy);
        int bxs[4], bys[4], nx = 0, ny = 0;
        for (int t = 0; t < w; ++t) {
            const int bx = wrapi(lx0 + t, nf) / BAND_W, by = wrapi(ly0 + t, nf) / BAND_H;
            if (nx == 0 || (bxs[nx - 1] != bx && bxs[0] != bx)) {
                if (nx < 4) bxs[nx++] = bx;
            }
            if (ny == 0 || (bys[ny - 1] != by && bys[0] != by)) {
                if (ny < 4) bys[ny++] = by;
            }
        }
        for (int a = 0; a < ny; ++a)
            for (int b = 0; b < nx; ++b) {
                const int band = bys[a] * nbx + bxs[b];
                if (!cursor) {
                    atomicAdd(counts + band, 1);
                    continue;
                }
                int dx0 = wrapi(lx0 - bxs[b] * BAND_W, nf), dy0 = wrapi(ly0 - bys[a] * BAND_H, nf);
                if (dx0 >= BAND_W) dx0 -= nf;
                if (dy0 >= BAND_H) dy0 -= nf;
                BandEntry e;
                e.pt = idx;
                e.dxy = (int)(((unsigned)dy0 << 16) | ((unsigned)dx0 & 0xffffu));
                e.fx = (float)fx;
                e.fy = (float)fy;
                out[atomicAdd(cursor + band, 1)] = e;
            }
    }
}

int SpreadBands::build(const PolarDev &g, int nf_, int w_, int chunk_, int nvirt_) {
    if (nf_ % BAND_W || nf_ % BAND_H) TC_FAIL(TC_ERR_ARG, "fine grid not a multiple of the band size");
    if (w_ > 8) TC_FAIL(TC_ERR_ARG, "spreading bands need a kernel width <= 8");
    if (chunk_ < 1) TC_FAIL(TC_ERR_ARG, "band chunk must be positive");
    nf = nf_;
    w = w_;
    chunk = chunk_;
    nvirt = nvirt_;
    const int nbx = nf / BAND_W, nbands = nbx * (nf / BAND_H);
    const int npts = g.P * g.D + nvirt;
    DevBuf d_counts, d_cursor;
    TC_TRY(d_counts.reserve((size_t)nbands * sizeof(int)));
    TC_CUDA(cudaMemset(d_counts.ptr, 0, (size_t)nbands * sizeof(int)));
    const int nblk = std::max(1, std::min(ceil_div(npts, 256), 148 * 16));
    k_band_lists<<<nblk, 256>>>(g, nf, w, d_counts.as<int>(), nullptr, nullptr, 1u, nvirt);
    TC_LAUNCH_CHECK();
    std::vector<int> counts(nbands);
    TC_CUDA(cudaMemcpy(counts.data(), d_counts.ptr, (size_t)nbands * sizeof(int), cudaMemcpyDeviceToHost));
    std::vector<int> start(nbands + 1, 0);
    for (int b = 0; b < nbands; ++b) start[b + 1] = start[b] + counts[b];
    const size_t total = (size_t)start[nbands];
    TC_TRY(entries.reserve(std::max<size_t>(total, 1) * sizeof(BandEntry)));
    if (total > 0) {
        TC_TRY(d_cursor.reserve((size_t)nbands * sizeof(int)));
        TC_CUDA(cudaMemcpy(d_cursor.ptr, start.data(), (size_t)nbands * sizeof(int), cudaMemcpyHostToDevice));
        // placed in point order, so a band's list runs along each ray that
        // crosses it and consecutive entries read neighbouring point values
        k_band_lists<<<nblk, 256>>>(g, nf, w, nullptr, d_cursor.as<int>(), entries.as<BandEntry>(),
                                    1u, nvirt);
        TC_LAUNCH_CHECK();
    }
    std::vector<BandChunk> cv;
    std::vector<int> sv;
    for (int b = 0; b < nbands; ++b) {
        const int c = counts[b];
        const int n = std::max(1, ceil_div(c, chunk));
        if (n > 1) sv.push_back(b);
        for (int k = 0; k < n; ++k)
            cv.push_back(BandChunk{b, start[b] + k * chunk,
                                   std::max(0, std::min(chunk, c - k * chunk)), n > 1 ? 1 : 0});
    }
    nchunk = (int)cv.size();
    nshared = (int)sv.size();
    TC_TRY(chunks.reserve(cv.size() * sizeof(BandChunk)));
    TC_CUDA(cudaMemcpy(chunks.ptr, cv.data(), cv.size() * sizeof(BandChunk), cudaMemcpyHostToDevice));
    TC_TRY(shared_bands.reserve(std::max<size_t>(sv.size(), 1) * sizeof(int)));
    if (!sv.empty())
        TC_CUDA(cudaMemcpy(shared_bands.ptr, sv.data(), sv.size() * sizeof(int), cudaMemcpyHostToDevice));
    TC_CUDA(cudaDeviceSynchronize());
    return TC_OK;
}

// Built like the spreading lists: count per tile on the device, prefix sum
// and sub-problem split on the host, then place.  Every point is in exactly
// one list, so the sub-problems write disjoint point values.
int InterpTiles::build(const PolarDev &g, int nf_, int w_, int ts_, int max_points_, int nvirt_) {
    if (ts_ != 16 && ts_ != 32) TC_FAIL(TC_ERR_ARG, "interpolation tile must be 16 or 32");
    if (w_ < 2 || w_ > 8) TC_FAIL(TC_ERR_ARG, "interpolation tiles need a kernel width 2 .. 8");
    if (max_points_ < 1) TC_FAIL(TC_ERR_ARG, "interpolation sub-problem size must be >= 1");
    if (nf_ < ts_ + w_ || nf_ % 2) TC_FAIL(TC_ERR_ARG, "fine grid odd or smaller than an interpolation region");
    nf = nf_;
    w = w_;
    ts = ts_;
    max_points = max_points_;
    nvirt = nvirt_;
    ntiles = ceil_div(nf, ts);
    const int nt2 = ntiles * ntiles;
    const int npts = g.P * g.D + nvirt;
    DevBuf d_counts, d_cursor;
    TC_TRY(d_counts.reserve((size_t)nt2 * sizeof(int)));
    TC_CUDA(cudaMemset(d_counts.ptr, 0, (size_t)nt2 * sizeof(int)));
    const int nblk = std::max(1, std::min(ceil_div(npts, 256), 148 * 16));
    k_interp_lists<<<nblk, 256>>>(g, nf, w, ts, ntiles, d_counts.as<int>(), nullptr, nullptr, nvirt);
    TC_LAUNCH_CHECK();
    std::vector<int> counts(nt2);
    TC_CUDA(cudaMemcpy(counts.data(), d_counts.ptr, (size_t)nt2 * sizeof(int), cudaMemcpyDeviceToHost));
    std::vector<int> start(nt2 + 1, 0);
    for (int t = 0; t < nt2; ++t) start[t + 1] = start[t] + counts[t];
    if (start[nt2] != npts) TC_FAIL(TC_ERR_STATE, "interpolation lists lost points");
    TC_TRY(entries.reserve(std::max<size_t>((size_t)npts, 1) * sizeof(InterpEntry)));
    if (npts > 0) {
        TC_TRY(d_cursor.reserve((size_t)nt2 * sizeof(int)));
        TC_CUDA(cudaMemcpy(d_cursor.ptr, start.data(), (size_t)nt2 * sizeof(int), cudaMemcpyHostToDevice));
        k_interp_lists<<<nblk, 256>>>(g, nf, w, ts, ntiles, nullptr, d_cursor.as<int>(),
                                      entries.as<InterpEntry>(), nvirt);
        TC_LAUNCH_CHECK();
    }
    std::vector<SpreadSub> sv;
    for (int t = 0; t < nt2; ++t)
        for (int k = 0; k * max_points < counts[t]; ++k)
            sv.push_back(SpreadSub{t, start[t] + k * max_points,
                                   std::min(max_points, counts[t] - k * max_points), 0});
    nsub = (int)sv.size();
    TC_TRY(subs.reserve(std::max<size_t>(sv.size(), 1) * sizeof(SpreadSub)));
    if (!sv.empty())
        TC_CUDA(cudaMemcpy(subs.ptr, sv.data(), sv.size() * sizeof(SpreadSub), cudaMemcpyHostToDevice));
    TC_CUDA(cudaDeviceSynchronize());
    return TC_OK;
}

// The lists are built on the device: count per tile, prefix sum and
// sub-problem split on the host (O(tiles)), then place.  The order of the
// points inside a tile follows the atomics of a scrambled visiting order; the
// spreading sums them with atomics anyway, so results differ only by
// summation order.
int SpreadLists::build(const PolarDev &g, const std::vector<double> &cs,
                       const std::vector<double> &sn, int nf_, int w, int max_points_, int ts_) {
    (void)cs;
    (void)sn;
    if (ts_ != 16 && ts_ != 32 && ts_ != 64) TC_FAIL(TC_ERR_ARG, "spread tile must be 16, 32 or 64");
    if (max_points_ < 1) TC_FAIL(TC_ERR_ARG, "spread sub-problem size must be >= 1");
    if (w + 2 > ts_) TC_FAIL(TC_ERR_ARG, "spread tile smaller than the kernel footprint");
    ts = ts_;
    max_points = max_points_;
    nf = nf_;
    ntiles = ceil_div(nf, ts);
    const int nt2 = ntiles * ntiles;
    const int npts = g.P * g.D;
    DevBuf d_counts, d_cursor;
    TC_TRY(d_counts.reserve((size_t)nt2 * sizeof(int)));
    TC_CUDA(cudaMemset(d_counts.ptr, 0, (size_t)nt2 * sizeof(int)));
    const int nblk = std::max(1, std::min(ceil_div(npts, 256), 148 * 16));
    // a visiting stride coprime to npts, near npts times the golden ratio
    unsigned stride = (unsigned)std::max<long long>(1, (long long)(0.6180339887 * npts)) | 1u;
    while (std::gcd((long long)stride, (long long)npts) != 1) stride += 2;
    k_tile_lists<<<nblk, 256>>>(g, nf, w, ts, ntiles, d_counts.as<int>(), nullptr, nullptr, 1u);
    TC_LAUNCH_CHECK();
    std::vector<int> counts(nt2);
    TC_CUDA(cudaMemcpy(counts.data(), d_counts.ptr, (size_t)nt2 * sizeof(int), cudaMemcpyDeviceToHost));
    std::vector<int> start(nt2 + 1, 0);
    for (int t = 0; t < nt2; ++t) start[t + 1] = start[t] + counts[t];
    const size_t total = (size_t)start[nt2];
    TC_TRY(points.reserve(std::max<size_t>(total, 1) * sizeof(int)));
    if (total > 0) {
        TC_TRY(d_cursor.reserve((size_t)nt2 * sizeof(int)));
        TC_CUDA(cudaMemcpy(d_cursor.ptr, start.data(), (size_t)nt2 * sizeof(int), cudaMemcpyHostToDevice));
        k_tile_lists<<<nblk, 256>>>(g, nf, w, ts, ntiles, nullptr, d_cursor.as<int>(), points.as<int>(),
                                    stride);
        TC_LAUNCH_CHECK();
    }
    std::vector<SpreadSub> sv;
    std::vector<int> shared_v;
    for (int t = 0; t < nt2; ++t) {
        const int c = counts[t];
        const int nchunk = std::max(1, ceil_div(c, max_points));
        if (nchunk > 1) shared_v.push_back(t);
        for (int k = 0; k < nchunk; ++k) {
            SpreadSub sb;
            sb.tile = t;
            sb.start = start[t] + k * max_points;
            sb.count = std::max(0, std::min(max_points, c - k * max_points));
            sb.shared = nchunk > 1 ? 1 : 0;
            sv.push_back(sb);
        }
    }
    nsub = (int)sv.size();
    nshared_tiles = (int)shared_v.size();
    TC_TRY(subs.reserve(sv.size() * sizeof(SpreadSub)));
    TC_CUDA(cudaMemcpy(subs.ptr, sv.data(), sv.size() * sizeof(SpreadSub), cudaMemcpyHostToDevice));
    TC_TRY(shared_tiles.reserve(std::max<size_t>(shared_v.size(), 1) * sizeof(int)));
    if (!shared_v.empty())
        TC_CUDA(cudaMemcpy(shared_tiles.ptr, shared_v.data(), shared_v.size() * sizeof(int),
                           cudaMemcpyHostToDevice));
    TC_CUDA(cudaDeviceSynchronize());
    return TC_OK;
}

// ---- generic pipelines ----------------------------------------------------

// type-2 passes 1-2: x (real, [nb][N][N]) -> fine grid [nb][nf][nf]
template <typename R, typename Tin>
static int t2_to_grid(const Tin *x, int N, int nb, const R *corr, const FftTables<R> &T,
                      cpx<R> *rows, cpx<R> *grid, cudaStream_t st) {
    const int nf = T.dev.L;
    {
        const int nthr = fft_threads<R>(nf, 1);
        const size_t smem = (size_t)nf * sizeof(cpx<R>);
        auto k = k_t2_rows<R, Tin>;
        TC_TRY(set_smem(k, smem));
        k<<<dim3(N, nb), nthr, smem, st>>>(x, rows, N, corr, T.dev);
        TC_LAUNCH_CHECK();
    }
    {
        const int cw = col_width<R>(nf);
        const int nthr = fft_threads<R>(nf, cw);
        const size_t smem = (size_t)cw * nf * sizeof(cpx<R>);
        auto k = k_t2_cols<R>;
        TC_TRY(set_smem(k, smem));
        k<<<dim3(nf / cw, nb), nthr, smem, st>>>(rows, grid, N, cw, T.dev);
        TC_LAUNCH_CHECK();
    }
    return TC_OK;
}

// type-1 pass 1 with TS x TS tiles: zero the shared tiles, spread (CM: the
// grid is stored column-major, grid[b][x][y])
template <typename R, int TS, bool CM = false>
static int spread_pass(const cpx<R> *cpts, const PolarDev &geo, const SpreadLists &sl,
                       const EsKernel &es, int nb, cpx<R> *grid, cudaStream_t st) {
    if (nb < 1 || nb > NB_MAX) TC_FAIL(TC_ERR_ARG, "chunk too large");
    const int nf = sl.nf;
    if (sl.nshared_tiles > 0) {
        k_zero_tiles<R, TS, CM><<<sl.nshared_tiles, 256, 0, st>>>(grid, sl.shared_tiles.as<int>(), nf,
                                                              sl.ntiles, nb);
        TC_LAUNCH_CHECK();
    }
    const size_t smem = (size_t)nb * 2 * TS * (TS + 1) * sizeof(R);
    auto k = k_spread<R, TS, CM>;
    TC_TRY(set_smem(k, smem));
    k<<<sl.nsub, 256, smem, st>>>(cpts, grid, sl.points.as<int>(), sl.subs.as<SpreadSub>(), geo,
                                  nf, sl.ntiles, es.w, (R)es.beta, nb);
    TC_LAUNCH_CHECK();
    return TC_OK;
}

// type-1 pass 1 on bands (column-major grid): zero the shared bands, spread
static int spread_band_pass(const c32 *cpts, const SpreadBands &sb, const PolarDev &geo,
                            float beta, int nb, c32 *grid, cudaStream_t st) {
    if (sb.nshared > 0) {
        k_zero_bands<<<sb.nshared, 256, 0, st>>>(grid, sb.shared_bands.as<int>(), sb.nf, nb);
        TC_LAUNCH_CHECK();
    }
    auto launch = [&](auto kern) -> int {
        const size_t smem = (size_t)BAND_WARPS * nb * BAND_H * BAND_RS * sizeof(c32);
        TC_TRY(set_smem(kern, smem));
        kern<<<ceil_div(sb.nchunk, BAND_WARPS), BAND_WARPS * 32, smem, st>>>(
            cpts, grid, sb.entries.as<BandEntry>(), sb.chunks.as<BandChunk>(), sb.nchunk, sb.nf,
            geo.P * geo.D + sb.nvirt, sb.w, beta);
        TC_LAUNCH_CHECK();
        return TC_OK;
    };
    if (nb == BAND8_NB && sb.w >= 2 && sb.w <= 8) {
        auto launch8 = [&](auto kern) -> int {
            kern<<<ceil_div(sb.nchunk, BAND_WARPS), BAND_WARPS * 32, 0, st>>>(
                cpts, grid, sb.entries.as<BandEntry>(), sb.chunks.as<BandChunk>(), sb.nchunk,
                sb.nf, geo.P * geo.D + sb.nvirt, beta);
            TC_LAUNCH_CHECK();
            return TC_OK;
        };
        switch (sb.w) {
            case 2: return launch8(k_spread_band8<2>);
            case 3: return launch8(k_spread_band8<3>);
            case 4: return launch8(k_spread_band8<4>);
            case 5: return launch8(k_spread_band8<5>);
            case 6: return launch8(k_spread_band8<6>);
            case 7: return launch8(k_spread_band8<7>);
            default: return launch8(k_spread_band8<8>);
        }
    }
    switch (nb) {
        case 1: return launch(k_spread_band<1>);
        case 2: return launch(k_spread_band<2>);
        case 3: return launch(k_spread_band<3>);
        case 4: return launch(k_spread_band<4>);
        case 5: return launch(k_spread_band<5>);
        case 6: return launch(k_spread_band<6>);
        case 7: return launch(k_spread_band<7>);
        case 8: return launch(k_spread_band<8>);
        default: TC_FAIL(TC_ERR_ARG, "chunk too large");
    }
}

// type-1 passes 1-3: points [nb][P*D] (or unit) -> out [nb][nm][nm] real
template <typename R, typename Tout>
static int t1_from_points(const cpx<R> *cpts, const PolarDev &geo, const SpreadLists &sl,
                          const EsKernel &es, int nm, int nb, const R *corr,
                          const FftTables<R> &T, cpx<R> *grid, cpx<R> *rows, Tout *out,
                          const float *sub, R scale, cudaStream_t st,
                          const SpreadBands *bands = nullptr) {
    const int nf = T.dev.L;
    if (sl.nf != nf) TC_FAIL(TC_ERR_STATE, "spread lists built for another grid");
    if constexpr (std::is_same<R, float>::value && std::is_same<Tout, float>::value) {
        if (t1_fast_supported(nf) && !T.dev.bluestein) {
            // column-major grid, then the register-FFT passes
            if (bands && bands->nf == nf && bands->w == es.w) {
                TC_TRY(spread_band_pass(cpts, *bands, geo, (float)es.beta, nb, grid, st));
                return t1_fast_fft(grid, rows, out, sub, corr, scale, nm, nf, nb, T.dev.tw, st);
            }
            switch (sl.ts) {
                case 16: TC_TRY((spread_pass<R, 16, true>(cpts, geo, sl, es, nb, grid, st))); break;
                case 32: TC_TRY((spread_pass<R, 32, true>(cpts, geo, sl, es, nb, grid, st))); break;
                case 64: TC_TRY((spread_pass<R, 64, true>(cpts, geo, sl, es, nb, grid, st))); break;
                default: TC_FAIL(TC_ERR_STATE, "spread lists with an unsupported tile size");
            }
            return t1_fast_fft(grid, rows, out, sub, corr, scale, nm, nf, nb, T.dev.tw, st);
        }
    }
    switch (sl.ts) {
        case 16: TC_TRY((spread_pass<R, 16>(cpts, geo, sl, es, nb, grid, st))); break;
        case 32: TC_TRY((spread_pass<R, 32>(cpts, geo, sl, es, nb, grid, st))); break;
        case 64: TC_TRY((spread_pass<R, 64>(cpts, geo, sl, es, nb, grid, st))); break;
        default: TC_FAIL(TC_ERR_STATE, "spread lists with an unsupported tile size");
    }
    {
        const int cw = col_width<R>(nf);
        const int nthr = fft_threads<R>(nf, cw);
        const size_t smem = (size_t)cw * nf * sizeof(cpx<R>);
        auto k = k_t1_cols<R>;
        TC_TRY(set_smem(k, smem));
        k<<<dim3(nf / cw, nb), nthr, smem, st>>>(grid, rows, nm, cw, T.dev);
        TC_LAUNCH_CHECK();
    }
    {
        const int nthr = fft_threads<R>(nf, 1);
        const size_t smem = (size_t)nf * sizeof(cpx<R>);
        auto k = k_t1_rows<R, Tout>;
        TC_TRY(set_smem(k, smem));
        k<<<dim3(nm, nb), nthr, smem, st>>>(rows, out, sub, nm, corr, scale, T.dev);
        TC_LAUNCH_CHECK();
    }
    return TC_OK;
}

static size_t grid_elems(const Plan &pl, int nb) { return (size_t)nb * pl.nf * pl.nf; }
static size_t rows_elems(const Plan &pl, int nb) {
    return (size_t)nb * std::max(pl.N, t1_fast_stride(pl.N)) * pl.nf;
}
static size_t pts_elems(const Plan &pl, int nb) { return (size_t)nb * pl.P * pl.N; }

static int reserve_nufft_ws(Plan &pl, int nb) {
    TC_TRY(pl.ws_grid.reserve(grid_elems(pl, nb) * sizeof(c32)));
    TC_TRY(pl.ws_rows.reserve(rows_elems(pl, nb) * sizeof(c32)));
    TC_TRY(pl.ws_pts.reserve(pts_elems(pl, nb) * sizeof(c32)));
    return TC_OK;
}

// launch shape of the detector-axis kernels: lpc slices (lines) per CTA
struct DetShape {
    int lpc, ngroups, nthr;
    size_t smem;
};

static DetShape det_shape(const Plan &pl, int nb) {
    const int L = pl.fft_D.dev.L;
    DetShape s;
    s.lpc = nb;
    while (s.lpc > 1 && fft_threads<float>(L, s.lpc) > FFT_MAX_THREADS) --s.lpc;
    s.ngroups = ceil_div(nb, s.lpc);
    s.nthr = std::min(FFT_MAX_THREADS, std::max(fft_threads<float>(L, s.lpc), 256));
    s.smem = (size_t)s.lpc * L * sizeof(c32);
    return s;
}

// register-FFT type-2 path (column-major grid) for the plan's fine grid
static bool t2_fast_ok(const Plan &pl) {
    return t1_fast_supported(pl.nf) && !pl.fft_nf.dev.bluestein && pl.det_M != 0;
}

bool interp_tiles_apply(const Plan &pl) { return t2_fast_ok(pl) && pl.es.w >= 2 && pl.es.w <= 8; }

static size_t interp_smem(const InterpTiles &it, int nb) {
    if (nb >= INTERP_LANES_MIN_NB) return (size_t)nb * interp_plane(it.ts, it.w) * sizeof(c32);
    const size_t rw = (size_t)it.ts + it.w - 1;
    return (size_t)nb * rw * interp_pitch(it.ts, it.w) * sizeof(c32);
}

template <int TS>
static int launch_interp_tile(Plan &pl, const InterpTiles &it, const c32 *grid, c32 *pts, int nb,
                              size_t sm, cudaStream_t st) {
    auto launch = [&](auto k) -> int {
        TC_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        k<<<it.nsub, INTERP_THREADS, sm, st>>>(grid, pts, it.entries.as<InterpEntry>(),
                                               it.subs.as<SpreadSub>(), pl.nf, it.ntiles,
                                               (float)pl.es.beta, nb,
                                               (size_t)pl.P * pl.N + (size_t)it.nvirt);
        TC_LAUNCH_CHECK();
        return TC_OK;
    };
    if (nb >= INTERP_LANES_MIN_NB) {
        switch (it.w) {
            case 2: return launch(k_t2_interp_lanes<TS, 2>);
            case 3: return launch(k_t2_interp_lanes<TS, 3>);
            case 4: return launch(k_t2_interp_lanes<TS, 4>);
            case 5: return launch(k_t2_interp_lanes<TS, 5>);
            case 6: return launch(k_t2_interp_lanes<TS, 6>);
            case 7: return launch(k_t2_interp_lanes<TS, 7>);
            default: return launch(k_t2_interp_lanes<TS, 8>);
        }
    }
    switch (it.w) {
        case 2: return launch(k_t2_interp_tile<TS, 2>);
        case 3: return launch(k_t2_interp_tile<TS, 3>);
        case 4: return launch(k_t2_interp_tile<TS, 4>);
        case 5: return launch(k_t2_interp_tile<TS, 5>);
        case 6: return launch(k_t2_interp_tile<TS, 6>);
        case 7: return launch(k_t2_interp_tile<TS, 7>);
        default: return launch(k_t2_interp_tile<TS, 8>);
    }
}

// the type-2 interpolation of the register-FFT path: from the tiles when
// the plan has them (and the region fits shared memory), else one thread
// per point straight from the grids (k_t2_interp, raw mode)
static int t2_interp_fast(Plan &pl, const InterpTiles &it, const c32 *grid, c32 *pts, int nb,
                          cudaStream_t st) {
    const size_t sm = it.nsub > 0 ? interp_smem(it, nb) : 0;
    if (it.nsub > 0 && it.nf == pl.nf && it.w == pl.es.w && sm <= 200 * 1024)
        return it.ts == 16 ? launch_interp_tile<16>(pl, it, grid, pts, nb, sm, st)
                           : launch_interp_tile<32>(pl, it, grid, pts, nb, sm, st);
    // the one-thread-per-point form knows neither mirror points nor the
    // paired lines' point stride
    if (it.nvirt > 0) TC_FAIL(TC_ERR_STATE, "paired NUFFT lines need the interpolation tiles");
    auto k = k_t2_interp<float, true>;
    TC_TRY(set_smem(k, 16));
    k<<<dim3(pl.P, 1), 256, 16, st>>>(grid, nullptr, pts, pl.geo, pl.nf, pl.es.w,
                                     (float)pl.es.beta, nb, nb, 1.0f, pl.fft_D.dev);
    TC_LAUNCH_CHECK();
    return TC_OK;
}

// ---------------------------------------------------------------------------
// the paired path (pl.pair_nufft): slices 2q and 2q + 1 are the real and
// imaginary parts of line q through every pass.  Each slice's transform is
// real (radon: the detector samples of a real image's spectrum come in
// conjugate pairs j, D - j, plus j = 0 and its mirror point; back-projection
// and the NUFFT gradient: the spread point values are Hermitian-symmetric),
// so the two slices come back as the real and imaginary parts.
// ---------------------------------------------------------------------------
bool pair_nufft_apply(const Plan &pl) { return interp_tiles_apply(pl); }

static int reserve_pair_ws(Plan &pl, int nlines) {
    TC_TRY(pl.ws_grid.reserve(grid_elems(pl, nlines) * sizeof(c32)));
    TC_TRY(pl.ws_rows.reserve(rows_elems(pl, nlines) * sizeof(c32)));
    TC_TRY(pl.ws_pts.reserve((size_t)nlines * pl.npts_ext() * sizeof(c32)));
    return TC_OK;
}

// the j = 0 value and its mirror's of every line and angle, halved: the type-2
// values at +-omega_0 of each slice become the symmetric pair whose type-1
// transform is the real part of the unpaired one's
__global__ void k_halve_mirror(c32 *__restrict__ pts, int P, int D, size_t cstride, int nlines) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nlines * P) return;
    const int q = i / P, p = i - q * P;
    c32 *a = pts + (size_t)q * cstride + (size_t)p * D;
    c32 *m = pts + (size_t)q * cstride + (size_t)P * D + p;
    *a = *a * 0.5f;
    *m = *m * 0.5f;
}

static int radon_pairs(Plan &pl, const float *x, float *sino, int nb, cudaStream_t st) {
    const int nl = (nb + 1) / 2;
    if (nl > NB_MAX) TC_FAIL(TC_ERR_ARG, "chunk too large");
    TC_TRY(reserve_pair_ws(pl, nl));
    c32 *grid = pl.ws_grid.as<c32>(), *rows = pl.ws_rows.as<c32>(), *pts = pl.ws_pts.as<c32>();
    TC_TRY(t2_fast_grid(x, rows, grid, pl.d_corr.as<float>(), pl.N, pl.nf, nb, pl.fft_nf.dev.tw,
                        st, 1));
    TC_TRY(t2_interp_fast(pl, pl.itiles, grid, pts, nl, st));
    return det_fast_inv(pl, pts, sino, nb, (float)(1.0 / ((double)pl.N * pl.N)), st, 1);
}

static int iradon_pairs(Plan &pl, const float *sino, float *x, int nb, int ramp, cudaStream_t st) {
    const int nl = (nb + 1) / 2;
    if (nl > NB_MAX) TC_FAIL(TC_ERR_ARG, "chunk too large");
    TC_TRY(reserve_pair_ws(pl, nl));
    c32 *grid = pl.ws_grid.as<c32>(), *rows = pl.ws_rows.as<c32>(), *pts = pl.ws_pts.as<c32>();
    TC_TRY(det_fast(pl, sino, pts, nb, ramp, st, 1));
    TC_TRY(spread_band_pass(pts, pl.bands, pl.geo, (float)pl.es.beta, nl, grid, st));
    return t1_fast_fft(grid, rows, x, nullptr, pl.d_corr.as<float>(),
                       (float)(1.0 / ((double)pl.N * pl.N)), pl.N, pl.nf, nb, pl.fft_nf.dev.tw,
                       st, 1);
}

static int nufft_grad_pairs(Plan &pl, const float *x, const float *aty, float *g, int nb,
                            cudaStream_t st) {
    const int nl = (nb + 1) / 2;
    if (nl > NB_MAX) TC_FAIL(TC_ERR_ARG, "chunk too large");
    TC_TRY(reserve_pair_ws(pl, nl));
    c32 *grid = pl.ws_grid.as<c32>(), *rows = pl.ws_rows.as<c32>(), *pts = pl.ws_pts.as<c32>();
    TC_TRY(t2_fast_grid(x, rows, grid, pl.d_corr.as<float>(), pl.N, pl.nf, nb, pl.fft_nf.dev.tw,
                        st, 1));
    TC_TRY(t2_interp_fast(pl, pl.itiles, grid, pts, nl, st));
    if (pl.nvirt) {
        k_halve_mirror<<<ceil_div(nl * pl.P, 256), 256, 0, st>>>(pts, pl.P, pl.N, pl.npts_ext(), nl);
        TC_LAUNCH_CHECK();
    }
    TC_TRY(spread_band_pass(pts, pl.bands, pl.geo, (float)pl.es.beta, nl, grid, st));
    return t1_fast_fft(grid, rows, g, aty, pl.d_corr.as<float>(),
                       (float)(1.0 / std::pow((double)pl.N, 3)), pl.N, pl.nf, nb,
                       pl.fft_nf.dev.tw, st, 1);
}

int radon_chunk(Plan &pl, const float *x, float *sino, int nb, cudaStream_t st) {
    if (pl.pair_nufft) return radon_pairs(pl, x, sino, nb, st);
    if (nb > NB_MAX) TC_FAIL(TC_ERR_ARG, "chunk too large");
    TC_TRY(reserve_nufft_ws(pl, nb));
    c32 *grid = pl.ws_grid.as<c32>(), *rows = pl.ws_rows.as<c32>();
    if (t2_fast_ok(pl)) {
        // fine grid, point values (raw interpolation), inverse detector DFT
        c32 *pts = pl.ws_pts.as<c32>();
        TC_TRY(t2_fast_grid(x, rows, grid, pl.d_corr.as<float>(), pl.N, pl.nf, nb,
                            pl.fft_nf.dev.tw, st));
        TC_TRY(t2_interp_fast(pl, pl.itiles, grid, pts, nb, st));
        return det_fast_inv(pl, pts, sino, nb, (float)(1.0 / ((double)pl.N * pl.N)), st);
    }
    TC_TRY((t2_to_grid<float, float>(x, pl.N, nb, pl.d_corr.as<float>(), pl.fft_nf, rows, grid, st)));
    const DetShape ds = det_shape(pl, nb);
    if (fft_threads<float>(pl.fft_D.dev.L, 1) > FFT_MAX_THREADS)
        TC_FAIL(TC_ERR_SHAPE, "detector length too large");
    auto k = k_t2_interp<float>;
    TC_TRY(set_smem(k, ds.smem));
    const float scale = (float)(1.0 / ((double)pl.N * pl.N));
    k<<<dim3(pl.P, ds.ngroups), ds.nthr, ds.smem, st>>>(grid, sino, nullptr, pl.geo, pl.nf,
                                                         pl.es.w, (float)pl.es.beta, nb, ds.lpc,
                                                         scale, pl.fft_D.dev);
    TC_LAUNCH_CHECK();
    return TC_OK;
}

int iradon_chunk(Plan &pl, const float *sino, float *x, int nb, int ramp, cudaStream_t st) {
    if (pl.pair_nufft) return iradon_pairs(pl, sino, x, nb, ramp, st);
    if (nb > NB_MAX) TC_FAIL(TC_ERR_ARG, "chunk too large");
    TC_TRY(reserve_nufft_ws(pl, nb));
    c32 *grid = pl.ws_grid.as<c32>(), *rows = pl.ws_rows.as<c32>(), *pts = pl.ws_pts.as<c32>();
    if (pl.det_M) {
        TC_TRY(det_fast(pl, sino, pts, nb, ramp, st));
    } else {
        const DetShape ds = det_shape(pl, nb);
        if (fft_threads<float>(pl.fft_D.dev.L, 1) > FFT_MAX_THREADS)
            TC_FAIL(TC_ERR_SHAPE, "detector length too large");
        auto k = k_t1_det<float>;
        TC_TRY(set_smem(k, ds.smem));
        k<<<dim3(pl.P, ds.ngroups), ds.nthr, ds.smem, st>>>(sino, pts, pl.P, pl.N, nb, ds.lpc,
                                                             ramp, pl.fft_D.dev);
        TC_LAUNCH_CHECK();
    }
    const float scale = (float)(1.0 / ((double)pl.N * pl.N));
    return t1_from_points<float, float>(pts, pl.geo, pl.spread, pl.es, pl.N, nb,
                                        pl.d_corr.as<float>(), pl.fft_nf, grid, rows, x, nullptr,
                                        scale, st, &pl.bands);
}

// g = Re(NUFFT1(NUFFT2(x))) / N^3 - aty   (src/gradient.cpp:61-65)
int nufft_grad_chunk(Plan &pl, const float *x, const float *aty, float *g, int nb,
                     cudaStream_t st) {
    if (pl.pair_nufft) return nufft_grad_pairs(pl, x, aty, g, nb, st);
    if (nb > NB_MAX) TC_FAIL(TC_ERR_ARG, "chunk too large");
    TC_TRY(reserve_nufft_ws(pl, nb));
    c32 *grid = pl.ws_grid.as<c32>(), *rows = pl.ws_rows.as<c32>(), *pts = pl.ws_pts.as<c32>();
    if (t2_fast_ok(pl)) {
        TC_TRY(t2_fast_grid(x, rows, grid, pl.d_corr.as<float>(), pl.N, pl.nf, nb,
                            pl.fft_nf.dev.tw, st));
        TC_TRY(t2_interp_fast(pl, pl.itiles, grid, pts, nb, st));
    } else {
        TC_TRY((t2_to_grid<float, float>(x, pl.N, nb, pl.d_corr.as<float>(), pl.fft_nf, rows, grid, st)));
        auto k = k_t2_interp<float>;
        TC_TRY(set_smem(k, 16));
        k<<<dim3(pl.P, 1), 256, 16, st>>>(grid, nullptr, pts, pl.geo, pl.nf, pl.es.w,
                                         (float)pl.es.beta, nb, nb, 1.0f, pl.fft_D.dev);
        TC_LAUNCH_CHECK();
    }
    const float scale = (float)(1.0 / std::pow((double)pl.N, 3));
    return t1_from_points<float, float>(pts, pl.geo, pl.spread, pl.es, pl.N, nb,
                                        pl.d_corr.as<float>(), pl.fft_nf, grid, rows, g, aty,
                                        scale, st, &pl.bands);
}

// FP64 point-spread function psf[a2][a1] = Re NUFFT1(ones) at offsets
// d = a - (N - 1), a in [0, 2N-1)  (src/toeplitz.h:51-73)
int psf_fp64(Plan &pl, const std::vector<double> &cs, const std::vector<double> &sn,
             double *psf, cudaStream_t st) {
    const int nm = 2 * pl.N - 1;
    const int nf64 = next_smooth_even(2 * nm);
    FftTables<double> T;
    TC_TRY(T.init(nf64));
    SpreadLists sl;
    TC_TRY(sl.build(pl.geo, cs, sn, nf64, pl.es64.w, 4096));
    std::vector<double> corr = es_correction(nm, nf64, pl.es64);
    DevBuf d_corr, grid, rows;
    TC_TRY(d_corr.reserve(nm * sizeof(double)));
    TC_CUDA(cudaMemcpy(d_corr.ptr, corr.data(), nm * sizeof(double), cudaMemcpyHostToDevice));
    TC_TRY(grid.reserve((size_t)nf64 * nf64 * sizeof(c64)));
    TC_TRY(rows.reserve((size_t)nm * nf64 * sizeof(c64)));
    TC_TRY((t1_from_points<double, double>(nullptr, pl.geo, sl, pl.es64, nm, 1,
                                           d_corr.as<double>(), T, grid.as<c64>(),
                                           rows.as<c64>(), psf, nullptr, 1.0, st)));
    TC_CUDA(cudaStreamSynchronize(st));
    return TC_OK;
}

// ---------------------------------------------------------------------------
// spread autotuner.  The type-1 spreading (back-projection, NUFFT gradient)
// splits the fine grid into TS x TS tiles, each accumulated in shared memory
// by one CTA per sub-problem of at most max_points points.  Small tiles cut
// the shared-memory footprint and the write-out; large tiles cut the number
// of points that straddle tiles (spread twice) and of shared tiles (global
// atomics); the sub-problem size trades parallelism against per-CTA
// overhead.  The best pair depends on the angles and sizes, so it is
// measured: every candidate's lists are built and one unit-strength
// spreading + transform pass is timed on the plan's own geometry.  Results
// are cached per geometry for the process.
// ---------------------------------------------------------------------------
static std::mutex g_tune_mu;
static std::map<std::string, std::pair<int, int>> g_tune_cache;
static std::map<std::string, std::pair<int, int>> g_band_cache;  // (list chunk, slices per chunk)
static std::map<std::string, std::pair<int, int>> g_interp_cache;  // (tile edge, points per sub-problem)

static std::string tune_key(const Plan &pl) {
    uint64_t h = 1469598103934665603ull;  // FNV-1a over the angle bytes
    const unsigned char *b = reinterpret_cast<const unsigned char *>(pl.angles.data());
    for (size_t i = 0; i < pl.angles.size() * sizeof(float); ++i) h = (h ^ b[i]) * 1099511628211ull;
    return std::to_string(pl.N) + "/" + std::to_string(pl.P) + "/" + std::to_string(pl.nf) + "/" +
           std::to_string(pl.es.w) + "/" + std::to_string(pl.max_batch) + "/" +
           std::to_string(pl.pair_nufft ? 1 : 0) + "/" + std::to_string(h);
}

int spread_autotune(Plan &pl, const std::vector<double> &cs, const std::vector<double> &sn) {
    const std::string key = tune_key(pl);
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) {
            return pl.spread.build(pl.geo, cs, sn, pl.nf, pl.es.w, it->second.second, it->second.first);
        }
    }
    const int cand[][2] = {{16, 1024}, {16, 4096}, {32, 1024}, {32, 2048}, {32, 4096},
                           {64, 2048}, {64, 8192}};
    cudaStream_t st = pl.aux;
    // timed at the chunk size the operators use (max_batch slices at once,
    // at most NB_MAX lines): the shared-memory tile grows with it and sets
    // the occupancy
    const int nb = std::min(pl.max_batch, NB_MAX);
    TC_TRY(reserve_nufft_ws(pl, nb));
    DevBuf out;
    TC_TRY(out.reserve((size_t)nb * pl.N * pl.N * sizeof(float)));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    TC_CUDA(cudaEventCreate(&e0));
    TC_CUDA(cudaEventCreate(&e1));
    struct EvGuard {
        cudaEvent_t a, b;
        ~EvGuard() {
            cudaEventDestroy(a);
            cudaEventDestroy(b);
        }
    } eg{e0, e1};
    float best = 1e30f;
    int best_ts = SPREAD_TILE, best_mp = 2048;
    for (const auto &c : cand) {
        const int ts = c[0], mp = c[1];
        if ((size_t)nb * 2 * ts * (ts + 1) * sizeof(float) > 200 * 1024) continue;
        if (pl.es.w + 2 > ts) continue;  // the kernel footprint must fit a tile
        SpreadLists sl;
        TC_TRY(sl.build(pl.geo, cs, sn, pl.nf, pl.es.w, mp, ts));
        auto run = [&]() {
            return t1_from_points<float, float>(nullptr, pl.geo, sl, pl.es, pl.N, nb,
                                                pl.d_corr.as<float>(), pl.fft_nf,
                                                pl.ws_grid.as<c32>(), pl.ws_rows.as<c32>(),
                                                out.as<float>(), nullptr, 1.0f, st);
        };
        TC_TRY(run());
        TC_CUDA(cudaEventRecord(e0, st));
        for (int r = 0; r < 3; ++r) TC_TRY(run());
        TC_CUDA(cudaEventRecord(e1, st));
        TC_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        TC_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        if (ms < best) {
            best = ms;
            best_ts = ts;
            best_mp = mp;
        }
    }
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tune_cache[key] = {best_ts, best_mp};
    }
    return pl.spread.build(pl.geo, cs, sn, pl.nf, pl.es.w, best_mp, best_ts);
}

}  // namespace tc

namespace tc {

// The band path's two free choices, measured on the plan's own geometry:
// the points per warp chunk of a band's list (short chunks balance the
// warps, long ones split fewer bands and so need fewer atomic adds) and the
// slices per NUFFT chunk (more slices reuse each list entry and kernel
// weight, fewer raise the occupancy).  Timed as whole type-1 transforms
// (spreading + register-FFT passes) per slice; cached per geometry.
int band_autotune(Plan &pl) {
    const std::string key = tune_key(pl);
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_band_cache.find(key);
        if (it != g_band_cache.end()) {
            pl.max_batch = it->second.second;
            return pl.bands.build(pl.geo, pl.nf, pl.es.w, it->second.first, pl.nvirt);
        }
    }
    const int chunks[] = {128, 256, 512, 1024};
    std::vector<int> nbs = {pl.max_batch};
    if (pl.max_batch >= 4) nbs.push_back(pl.max_batch / 2);
    cudaStream_t st = pl.aux;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    TC_CUDA(cudaEventCreate(&e0));
    TC_CUDA(cudaEventCreate(&e1));
    struct EvGuard {
        cudaEvent_t a, b;
        ~EvGuard() {
            cudaEventDestroy(a);
            cudaEventDestroy(b);
        }
    } eg{e0, e1};
    // slices per chunk -> lines (two slices per line on the paired path)
    auto lines_of = [&](int nb) { return pl.pair_nufft ? (nb + 1) / 2 : nb; };
    TC_TRY(reserve_nufft_ws(pl, lines_of(nbs[0])));
    DevBuf out;
    TC_TRY(out.reserve((size_t)lines_of(nbs[0]) * pl.N * pl.N * sizeof(float)));
    float best = 1e30f;
    int best_chunk = BAND_CHUNK, best_nb = pl.max_batch;
    for (int ch : chunks) {
        TC_TRY(pl.bands.build(pl.geo, pl.nf, pl.es.w, ch, pl.nvirt));
        for (int nb : nbs) {
            auto run = [&]() {
                return t1_from_points<float, float>(nullptr, pl.geo, pl.spread, pl.es, pl.N,
                                                    lines_of(nb), pl.d_corr.as<float>(), pl.fft_nf,
                                                    pl.ws_grid.as<c32>(), pl.ws_rows.as<c32>(),
                                                    out.as<float>(), nullptr, 1.0f, st, &pl.bands);
            };
            TC_TRY(run());
            TC_CUDA(cudaEventRecord(e0, st));
            for (int r = 0; r < 3; ++r) TC_TRY(run());
            TC_CUDA(cudaEventRecord(e1, st));
            TC_CUDA(cudaEventSynchronize(e1));
            float ms = 0.f;
            TC_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            const float per_slice = ms / (float)nb;
            if (per_slice < best) {
                best = per_slice;
                best_chunk = ch;
                best_nb = nb;
            }
        }
    }
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_band_cache[key] = {best_chunk, best_nb};
    }
    pl.max_batch = best_nb;
    return pl.bands.build(pl.geo, pl.nf, pl.es.w, best_chunk, pl.nvirt);
}

// The interpolation tiles' two free choices, measured on the plan's own
// geometry at the plan's NUFFT chunk size: the tile edge (small tiles keep
// more CTAs per SM, large ones copy less halo per point) and the points per
// sub-problem (small sub-problems balance the dense centre of the polar
// grid against its rim, large ones copy each tile's region fewer times).
// Timed as the interpolation pass alone; cached per geometry.
int interp_autotune(Plan &pl) {
    const std::string key = tune_key(pl);
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_interp_cache.find(key);
        if (it != g_interp_cache.end())
            return pl.itiles.build(pl.geo, pl.nf, pl.es.w, it->second.first, it->second.second,
                                   pl.nvirt);
    }
    const int cand[][2] = {{16, 256}, {16, 1024}, {32, 256}, {32, 1024}, {32, 4096}};
    cudaStream_t st = pl.aux;
    // lines of the plan's chunk (two slices per line on the paired path)
    const int nb = pl.pair_nufft ? (pl.max_batch + 1) / 2 : pl.max_batch;
    TC_TRY(reserve_nufft_ws(pl, nb));
    TC_TRY(pl.ws_pts.reserve((size_t)nb * pl.npts_ext() * sizeof(c32)));
    TC_CUDA(cudaMemsetAsync(pl.ws_grid.ptr, 0, pl.ws_grid.bytes, st));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    TC_CUDA(cudaEventCreate(&e0));
    TC_CUDA(cudaEventCreate(&e1));
    struct EvGuard {
        cudaEvent_t a, b;
        ~EvGuard() {
            cudaEventDestroy(a);
            cudaEventDestroy(b);
        }
    } eg{e0, e1};
    float best = 1e30f;
    int best_ts = INTERP_TILE, best_mp = INTERP_POINTS;
    for (const auto &c : cand) {
        InterpTiles it;
        TC_TRY(it.build(pl.geo, pl.nf, pl.es.w, c[0], c[1], pl.nvirt));
        if (interp_smem(it, nb) > 200 * 1024) continue;
        auto run = [&]() {
            return t2_interp_fast(pl, it, pl.ws_grid.as<c32>(), pl.ws_pts.as<c32>(), nb, st);
        };
        TC_TRY(run());
        TC_CUDA(cudaEventRecord(e0, st));
        for (int r = 0; r < 3; ++r) TC_TRY(run());
        TC_CUDA(cudaEventRecord(e1, st));
        TC_CUDA(cudaEventSynchronize(e1));
        float ms = 0.f;
        TC_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        if (ms < best) {
            best = ms;
            best_ts = c[0];
            best_mp = c[1];
        }
    }
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_interp_cache[key] = {best_ts, best_mp};
    }
    return pl.itiles.build(pl.geo, pl.nf, pl.es.w, best_ts, best_mp, pl.nvirt);
}

}  // namespace tc
