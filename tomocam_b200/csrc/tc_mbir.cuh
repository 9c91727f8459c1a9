// tc_mbir.cuh -- the MBIR attempt's device pieces shared by the
// single-volume solver (tc_mbir.cu) and the batched solver (tc_batch.cu):
// the iteration state, the fused stencil + Nesterov update body and the step
// test of Optimizer::run2 (src/optimize.h:96-154).
#pragma once

#include <type_traits>

#include "tc_plan.cuh"
#include "tc_prior.cuh"

namespace tc {

struct MbirState {
    double t, tnew, beta, step, step0, sino_sq;
    float betaf, stepf;
    int ix, isol, inew;        // buffer indices of x, sol, new iterate
    int iter, num_iters;       // accepted iterations so far / requested
    int attempts, attempts_iter, max_attempts;
    int cond;                  // 1 while more attempts are needed
    int status;                // 0 ok, 1 backtracking cap reached
};

// beta and theta for the next attempt (src/optimize.h:117-121)
__device__ __forceinline__ void mbir_begin(MbirState *s) {
    const double t = s->t;
    s->beta = s->tnew * (1.0 / t - 1.0);
    s->tnew = 0.5 * (sqrt(t * t * t * t + 4.0 * t * t) - t * t);
    s->betaf = (float)s->beta;
    s->stepf = (float)s->step;
}

constexpr int NU = 5;  // FP64 partial sums per CTA
constexpr int UX = 32, UY = 16, UT = UX * UY;           // one voxel per thread
constexpr int UPD_MIN_BLOCKS = UT >= 1024 ? 1 : 2;       // CTAs per SM the registers allow
constexpr int PW = UX + 2, PH = UY + 2, PN = PW * PH;  // tile with a one-voxel halo

// Fused stencil + Nesterov update.  A CTA owns a 32 x 16 column of voxels and
// marches through all slices with planes s and s+1 of y (one-voxel clamped
// halo) in shared memory, so every value of y is formed and loaded once.
//
// The prior uses each edge once.  With F the 13 "forward" offsets
// (dz = 1: all nine; dz = 0, dy = 1: three; (0, 0, 1)) and
//   E_d(v) = rho'(y[c(v)] - y[c(v + d)])      (c = clamp to the volume)
// the 26-neighbour sum of voxel u is  sum_{d in F} w_d (E_d(u) - E_d(u - d)),
// because rho' is odd and c(u - d + d) = u; at the volume edges c(u - d)
// reproduces the reference's clamped neighbour exactly.  Each slice step
// evaluates the 13 E_d over the haloed tile once; the nine dz = 1 values of
// plane s are kept for the backward terms of plane s + 1.
//
// Work per step: every thread evaluates the 13 edges of its own voxel (kept
// in registers for its forward terms and stored for its neighbours'
// backward terms); the edges that start in the halo and end inside the tile
// (listed once at compile time in kHalo, fewer than the threads) take one
// more evaluation on some threads.  The march is software-pipelined: the
// global loads of plane s + 3 and of the voxel data of plane s + 1 are issued
// during step s and consumed a step later, so no step waits on memory.
constexpr int NDIR = 13;
__host__ __device__ constexpr int dir_dz(int k) { return k < 9 ? 1 : 0; }
__host__ __device__ constexpr int dir_dy(int k) { return k < 9 ? k / 3 - 1 : (k < 12 ? 1 : 0); }
__host__ __device__ constexpr int dir_dx(int k) { return k < 9 ? k % 3 - 1 : (k < 12 ? k - 10 : 1); }

// a halo item packs its direction (< 16) and tile position (< 2^11) in 16 bits
constexpr int HALO_POS_BITS = 11;
static_assert(PN <= (1 << HALO_POS_BITS) && NDIR <= (1 << (16 - HALO_POS_BITS)),
              "halo item encoding: tile positions or directions out of range");
struct HaloItems {
    int n;
    unsigned short item[640];  // (direction << HALO_POS_BITS) | tile position
};
constexpr HaloItems make_halo_items() {
    HaloItems h{};
    for (int k = 0; k < NDIR; ++k)
        for (int r = 0; r < PH; ++r)
            for (int c = 0; c < PW; ++c) {
                const bool in = r >= 1 && r <= UY && c >= 1 && c <= UX;
                const int tr = r + dir_dy(k), tc = c + dir_dx(k);
                const bool tin = tr >= 1 && tr <= UY && tc >= 1 && tc <= UX;
                if (!in && tin) h.item[h.n++] = (unsigned short)((k << HALO_POS_BITS) | (r * PW + c));
            }
    return h;
}
constexpr HaloItems kHaloHost = make_halo_items();
// the (1, 0, 0) edge of a voxel ends at the same tile position one plane up,
// so no halo item has that direction (its backward term stays in a register)
constexpr bool halo_has_dir(const HaloItems &h, int k) {
    for (int i = 0; i < h.n; ++i)
        if ((h.item[i] >> HALO_POS_BITS) == k) return true;
    return false;
}
constexpr int KDOWN = 4;  // dz = 1, dy = 0, dx = 0
static_assert(dir_dz(KDOWN) == 1 && dir_dy(KDOWN) == 0 && dir_dx(KDOWN) == 0, "KDOWN");
static_assert(!halo_has_dir(kHaloHost, KDOWN), "no halo item for the (1, 0, 0) direction");
static_assert(kHaloHost.n <= UT, "one halo edge per thread at most");
static_assert(PN <= 2 * UT, "two plane items per thread at most");
constexpr int NHALO = kHaloHost.n;
static __device__ const HaloItems kHalo = make_halo_items();
// y of planes s and s+1, E of the dz = 1 edges of planes s-1 and s, E of the
// four dz = 0 edges of plane s
constexpr int UPD_SMEM = (2 + 2 * 9 + 4) * PN * (int)sizeof(float);
constexpr int ACC_CHUNK = 8;  // slices summed in FP32 before each FP64 add

// SAME: x == sol (every attempt after an accepted step), so y = sol, H y =
// H sol and neither x nor H x is read.
template <bool SAME>
__device__ __forceinline__ void update_body(float *__restrict__ X, const float *__restrict__ H,
                                            const float *__restrict__ aty, int S, int R, int C,
                                            size_t vol, const PriorParams &pp,
                                            const MbirState *__restrict__ st,
                                            double *__restrict__ part, int c0, int r0,
                                            int s_lo = 0, int s_hi = 1 << 30) {
    // planes s_lo .. s_hi-1 are written and summed; the others (the halo
    // planes of a slab) only serve as neighbours
    extern __shared__ float smf[];
    float *yp = smf;           // [2][PN]
    float *e1 = smf + 2 * PN;  // [2][9][PN]
    float *e0 = e1 + 18 * PN;  // [4][PN]
    const int ix = st->ix, isol = st->isol, inew = st->inew;
    const float beta = st->betaf, step = st->stepf;
    constexpr bool same = SAME;
    const float *xs = X + (size_t)isol * vol;
    const float *xx = X + (size_t)ix * vol;
    const float *hs = H + (size_t)isol * vol;
    const float *hx = H + (size_t)ix * vol;
    float *out = X + (size_t)inew * vol;
    const int tid = threadIdx.x, tx = tid % UX, ty = tid / UX;
    const size_t plane = (size_t)R * C;
    // the thread's plane items: tile positions tid and tid + UT, with their
    // clamped in-plane offsets (the same on every plane)
    int goff[2];
    bool has[2];
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        const int i = tid + j * UT;
        has[j] = i < PN;
        const int dy = i / PW, dx = i - dy * PW;
        const int rr = min(max(r0 + dy - 1, 0), R - 1), cc = min(max(c0 + dx - 1, 0), C - 1);
        goff[j] = rr * C + cc;
    }
    float pxs[2] = {0.f, 0.f}, pxx[2] = {0.f, 0.f};
    auto fetch_plane = [&](int s) {
        const size_t base = (size_t)min(max(s, 0), S - 1) * plane;
#pragma unroll
        for (int j = 0; j < 2; ++j)
            if (has[j]) {
                pxs[j] = xs[base + goff[j]];
                pxx[j] = same ? 0.f : xx[base + goff[j]];
            }
    };
    auto store_plane = [&](float *dst) {
#pragma unroll
        for (int j = 0; j < 2; ++j)
            if (has[j]) dst[tid + j * UT] = same ? pxs[j] : pxs[j] + (pxs[j] - pxx[j]) * beta;
    };
    // the thread's halo edge, if any
    const bool hh = tid < NHALO;
    int h_src = 0, h_nb = 0, h_dst = 0, h_k = 0;
    if (hh) {
        const int it = kHalo.item[tid];
        h_k = it >> HALO_POS_BITS;
        h_src = it & ((1 << HALO_POS_BITS) - 1);
        h_nb = h_src + dir_dy(h_k) * PW + dir_dx(h_k);
        h_dst = (h_k < 9 ? h_k : h_k - 9) * PN + h_src;
    }
    const int o = (ty + 1) * PW + tx + 1;
    const int c = c0 + tx, r = r0 + ty;
    const bool inside = (c < C && r < R);
    const size_t vo = inside ? (size_t)r * C + c : 0;
    float nhs = 0.f, nhx = 0.f, naty = 0.f, nxx = 0.f;
    auto fetch_vox = [&](int s) {
        if (inside && s < S) {
            const size_t v = s * plane + vo;
            nhs = hs[v];
            nhx = same ? 0.f : hx[v];
            naty = aty[v];
            nxx = same ? 0.f : xx[v];
        }
    };
    // edges of plane a (dz = 1 edges end in plane b): the thread's own voxel
    // (returned in f[], stored for the neighbours) and its halo edge
    auto edges = [&](const float *a, const float *b, float *e1dst, bool with_e0, float *f,
                     float &ya) {
        ya = a[o];
#pragma unroll
        for (int k = 0; k < NDIR; ++k) {
            if (k >= 9 && !with_e0) break;
            const int off = dir_dy(k) * PW + dir_dx(k);
            const float e = d_pot_unscaled(ya - (k < 9 ? b : a)[o + off], pp);
            f[k] = e;
            if (k < 9) {
                if (k != KDOWN) e1dst[k * PN + o] = e;  // KDOWN: read back from f by this thread
            } else {
                e0[(k - 9) * PN + o] = e;
            }
        }
        if (hh && (h_k < 9 || with_e0)) {
            const float e = d_pot_unscaled(a[h_src] - (h_k < 9 ? b : a)[h_nb], pp);
            (h_k < 9 ? e1dst : e0)[h_dst] = e;
        }
    };
    double acc[NU] = {0, 0, 0, 0, 0};
    float cacc[NU] = {0.f, 0.f, 0.f, 0.f, 0.f};
    float f[NDIR];
    float u = 0.f;
    // planes 0 and 1 resident, plane 2 and the voxel data of plane 0 in flight
    fetch_plane(0);
    store_plane(yp);
    fetch_plane(1);
    store_plane(yp + PN);
    fetch_plane(2);
    fetch_vox(0);
    __syncthreads();
    // plane -1 (clamped to 0) -> plane 0 edges seed the backward dz = 1 terms
    edges(yp, yp, e1, false, f, u);
    float edown = f[KDOWN];  // E of the (1, 0, 0) edge ending at this voxel
    // one slice step; CUR (compile time): yp[CUR] holds plane s, e1[CUR]
    // holds plane s-1's edges (the march is unrolled by two)
    auto slice_step = [&](int s, auto cur_c) {
        constexpr int cur = decltype(cur_c)::value, eo = cur;
        __syncthreads();  // plane s+1 resident; the last step's reads of e1[eo ^ 1], e0 done
        float *ycur = yp + cur * PN, *ynxt = yp + (cur ^ 1) * PN;
        edges(ycur, ynxt, e1 + (eo ^ 1) * 9 * PN, true, f, u);
        __syncthreads();    // all edges of plane s stored; plane s no longer read
        store_plane(ycur);  // plane s + 2
        fetch_plane(s + 3);
        const float hsv = nhs, hxv = nhx, a = naty, xxv = nxx;
        fetch_vox(s + 1);
        if (inside && s >= s_lo && s < s_hi) {
            const size_t v = s * plane + vo;
            float prior = 0.0f;
#pragma unroll
            for (int k = 0; k < NDIR; ++k) {
                const int dz = dir_dz(k), dy = dir_dy(k), dx = dir_dx(k);
                const float w = c_qggmrf_w[((dz + 1) * 3 + dy + 1) * 3 + dx + 1];
                const int back = o - dy * PW - dx;
                const float eb = k == KDOWN ? edown
                                 : k < 9    ? e1[(eo * 9 + k) * PN + back]
                                            : e0[(k - 9) * PN + back];
                prior = fmaf(w, f[k] - eb, prior);
            }
            const float hy = same ? hsv : (1.0f + beta) * hsv - beta * hxv;
            const float g = (hy - a) + (pp.scale * pp.inv_sq) * prior;
            const float sn = u - g * step;
            out[v] = sn;
            const float xv = same ? u : xxv;
            const float dxf = sn - xv;
            cacc[0] = fmaf(u, hy, cacc[0]);
            cacc[1] = fmaf(u, a, cacc[1]);
            cacc[2] = fmaf(g, g, cacc[2]);
            cacc[3] = fmaf(sn, a, cacc[3]);
            cacc[4] = fmaf(dxf, dxf, cacc[4]);
        }
        edown = f[KDOWN];
        if ((s % ACC_CHUNK) == ACC_CHUNK - 1 || s == S - 1) {
#pragma unroll
            for (int k = 0; k < NU; ++k) {
                acc[k] += (double)cacc[k];
                cacc[k] = 0.f;
            }
        }
    };
    for (int s = 0; s < S; s += 2) {
        slice_step(s, std::integral_constant<int, 0>{});
        if (s + 1 < S) slice_step(s + 1, std::integral_constant<int, 1>{});
    }
    block_sum<NU>(acc, tid, UT);
    if (tid == 0) {
#pragma unroll
        for (int k = 0; k < NU; ++k) part[k] = acc[k];
    }
}


// The step test and bookkeeping of one attempt from its reduced sums
// u = {y.Hy, y.A^Ty, g.g, new.A^Ty, |new - x|^2, new.H new}; returns 1 while
// more attempts are needed (src/optimize.h:122-146).
__device__ __forceinline__ int mbir_decide_core(MbirState *s, const double *u, double *hist) {
    const double yhy = u[0], yaty = u[1], gg = u[2], naty = u[3], dx2 = u[4], nhn = u[5];
    // objective sqrt(v.Hv - 2 v.A^T y + |y|^2)  (src/error2.cpp:60-63, src/mbir2.cpp:130-136)
    const double fy = sqrt(yhy - 2.0 * yaty + s->sino_sq);
    const double fx = sqrt(nhn - 2.0 * naty + s->sino_sq);
    const double gy = 0.5 * s->step * gg;
    s->attempts += 1;
    s->attempts_iter += 1;
    int cond = 1;
    if (fx > fy + gy) {
        // rejected: shrink the step, keep x, retry from the new iterate
        s->step *= 0.9;
        s->isol = s->inew;
        int f = 0;
        while (f == s->ix || f == s->isol) ++f;
        s->inew = f;
        if (s->attempts_iter >= s->max_attempts) {
            s->status = 1;
            cond = 0;
        }
    } else {
        s->step = s->step0;
        s->t = s->tnew;
        if (hist) {
            hist[3 * s->iter + 0] = fx;
            hist[3 * s->iter + 1] = sqrt(dx2);
            hist[3 * s->iter + 2] = (double)s->attempts_iter;
        }
        s->ix = s->inew;
        s->isol = s->inew;
        s->inew = (s->inew + 1) % 3;
        s->iter += 1;
        s->attempts_iter = 0;
        cond = s->iter < s->num_iters ? 1 : 0;
    }
    s->cond = cond;
    return cond;
}

}  // namespace tc
