// tc_update.cuh -- the fused qGGMRF stencil + Nesterov update of one MBIR
// attempt, register-blocked.
//
// Geometry.  A CTA of UT = 16 x 16 threads owns a UX x UY = 64 x 32 column of
// voxels and marches through the slices; each thread owns a BXV x BYV = 4 x 2
// micro-block of every plane.  Planes s and s+1 of y (with a one-voxel
// clamped ring) live in shared memory; each thread keeps the 6 x 4 window of
// plane s+1 around its block in registers (and the 6 x 3 window of plane s
// from the previous step), so a neighbour value costs no shared-memory
// access.
//
// The prior.  rho' is odd, so with F the 13 "forward" offsets (dz = 1: all
// nine; dz = 0: (dy, dx) = (1, -1), (1, 0), (1, 1), (0, 1)) and
//   E_d(v) = rho'(y[c(v)] - y[c(v + d)])      (c = clamp to the volume)
// the 26-neighbour sum of voxel u is  sum_{d in F} w_d (E_d(u) - E_d(u - d)),
// each edge evaluated once (src/gpu/cuTV2.cu:33-76 evaluates all 26 per
// voxel).  A thread evaluates the 13 x 8 edges of its block and adds
// w E to its producer's sum; the backward term -w E goes to the consumer
// u + d: straight into a register when the consumer is in the same block
// (this plane, or the next plane for dz = 1), otherwise through a slot of
// the block's export area in shared memory.  A block exports 48 of its 104
// edges, grouped by the neighbouring block that consumes them, so exports
// and imports are 16-byte vector accesses.  The CTA's ring of virtual blocks
// (one block around the tile) exports only the edges that end inside the
// tile; those ~870 edges per plane are listed at compile time and spread
// over the threads.  The dz = 1 edges of plane s are imported during step s
// into the sums of plane s+1, so one export area serves every step.
//
// Per step: barrier; plane s+2 requested into the third plane buffer;
// window of plane s+1; 104 own edges and the halo edges (exports written);
// barrier; imports; the update and the partial sums of the voxels of plane
// s; wait for plane s+2.  After an accepted step (x = sol) the plane comes as
// one tensor copy of the 72 x 34 box starting at (c0 - 4, r0 - 1) -- the x
// origin rounded down to 16 bytes, zeros outside the volume, clamped values
// written over those for tiles at the volume's border -- or, without a
// tensor map, as cp.async pieces with clamped addresses.  After a rejected
// step (x != sol) plane s+2 of y = sol + beta (sol - x) is formed in
// registers and stored before the next step.  The FP64 partial sums live in
// shared memory.
#pragma once

#include <cstdint>
#include <type_traits>

#include "tc_cpasync.cuh"
#include "tc_plan.cuh"
#include "tc_tma.cuh"
#include "tc_prior.cuh"

namespace tc {

constexpr int NU = 5;                               // FP64 partial sums per CTA
constexpr int BXV = 4, BYV = 2, BV = BXV * BYV;     // voxels per thread
constexpr int TXT = 16, TYT = 16, UT = TXT * TYT;   // threads per CTA
constexpr int UX = BXV * TXT, UY = BYV * TYT;       // voxel tile
constexpr int UPD_MIN_BLOCKS = 2;
// Of every 13 own edges, UPD_FMA_RCP form 1/(c + t) on the FMA pipe
// (rcp_fma) rather than the SFU: the SFU does three operations per edge and
// is the kernel's busiest unit, the FMA pipe a quarter busy.  The edges that
// move are spread evenly over the block's 104.
#ifndef UPD_FMA_RCP
#define UPD_FMA_RCP 7
#endif
constexpr int UPD_FMA_RCP_PER13 = UPD_FMA_RCP;
static_assert(UPD_FMA_RCP_PER13 >= 0 && UPD_FMA_RCP_PER13 <= 13, "0 .. 13 edges of 13");
constexpr bool edge_fma_rcp(int i) {
    return (i + 1) * UPD_FMA_RCP_PER13 / 13 != i * UPD_FMA_RCP_PER13 / 13;
}
// Of every 13 own edges, UPD_FMA_EX2 form 2^x on the FMA pipe (ex2_fma):
// measured with 7 reciprocals on the FMA pipe, 0 -> 6.38 ms per 128-slice
// launch, 3 -> 6.52, 6 -> 7.00 (and 4 + 4 -> 6.53, 10 + 3 -> 6.82), so none.
#ifndef UPD_FMA_EX2
#define UPD_FMA_EX2 0
#endif
constexpr bool edge_fma_ex2(int i) {
    // spread with an offset so the edges differ from the reciprocal's
    return (i + 7) * UPD_FMA_EX2 / 13 != (i + 6) * UPD_FMA_EX2 / 13;
}
// shared plane: rows y = -1 .. UY, columns x = -1 .. UX at index x + PX0
constexpr int PX0 = 4;
constexpr int PW = UX + 8;  // row stride, a multiple of 4 (16-byte rows)
constexpr int PH = UY + 2;
constexpr int PN = PW * PH;
constexpr int PNA = (PN + 31) & ~31;  // plane buffer stride: 128-byte aligned tensor-copy targets
// export area: virtual blocks (ring included) x SLOTS floats
constexpr int VBW = TXT + 2, VBH = TYT + 2, NVB = VBW * VBH;
constexpr int SLOTS = 52;  // 48 used; 52 = 13 x 4 keeps 8 consecutive blocks conflict-free
// three plane buffers, the export area, each thread's FP64 partial sums and
// the three plane buffers' mbarriers (tensor-copy form)
constexpr int UPD_SMEM = (3 * PNA + NVB * SLOTS) * (int)sizeof(float) + 5 * UT * (int)sizeof(double) +
                         3 * (int)sizeof(uint64_t);
constexpr unsigned TMA_WAIT_POLLS = 1u << 20;  // bounded wait for one plane tile
constexpr int UPD_STATUS_TMA_TIMEOUT = 3;      // MbirState::status after a wait gave up
constexpr int ACC_CHUNK = 8;  // slices summed in FP32 before each FP64 add
static_assert(PW % 4 == 0 && (PX0 % 4) == 0 && SLOTS % 4 == 0, "16-byte alignment");
static_assert(2 * (UPD_SMEM + 1024) <= 228 * 1024, "two CTAs per SM");

// the 13 forward directions: k < 9: dz = 1, (dy, dx) = (k / 3 - 1, k % 3 - 1);
// k = 9, 10, 11: dz = 0, dy = 1, dx = k - 10; k = 12: dz = 0, dy = 0, dx = 1
constexpr int NDIR = 13;
__host__ __device__ constexpr int dir_dz(int k) { return k < 9 ? 1 : 0; }
__host__ __device__ constexpr int dir_dy(int k) { return k < 9 ? k / 3 - 1 : (k < 12 ? 1 : 0); }
__host__ __device__ constexpr int dir_dx(int k) { return k < 9 ? k % 3 - 1 : (k < 12 ? k - 10 : 1); }
// weight of the direction (src/gpu/potential_function.cuh:38-51): face,
// edge or corner neighbour by the number of non-zero offsets
__host__ __device__ constexpr float dir_w(int k) {
    const int n = (dir_dz(k) != 0) + (dir_dy(k) != 0) + (dir_dx(k) != 0);
    return n == 1 ? 0.0523f : (n == 2 ? 0.0370f : 0.0302f);
}

// neighbour blocks that consume exports, in the order of the export area;
// (gx, gy) is the consumer block's offset from the producer block
constexpr int NGRP = 8;
__host__ __device__ constexpr int grp_dx(int g) {
    constexpr int v[NGRP] = {0, 0, 1, -1, -1, 1, -1, 1};
    return v[g];
}
__host__ __device__ constexpr int grp_dy(int g) {
    constexpr int v[NGRP] = {1, -1, 0, 0, 1, 1, -1, -1};
    return v[g];
}
// first slot of each group: down 20, up 10, right 7, left 5, down-left 2,
// down-right 2, up-left 1, up-right 1 edges; vector groups start at 16 bytes
__host__ __device__ constexpr int grp_base(int g) {
    constexpr int v[NGRP] = {0, 20, 32, 40, 46, 48, 50, 51};
    return v[g];
}
__host__ __device__ constexpr int grp_count(int g) {
    constexpr int v[NGRP] = {20, 10, 7, 5, 2, 2, 1, 1};
    return v[g];
}

// the group a slot belongs to, -1 for the unused slots
__host__ __device__ constexpr int slot_group(int j) {
    int q = -1;
    for (int i = 0; i < NGRP; ++i)
        if (j >= grp_base(i) && j < grp_base(i) + grp_count(i)) q = i;
    return q;
}

// exports and imports move runs of slots: from a group's first slot, 4 at a
// time while the offset is a multiple of 4 and the group has 4 left, then 2,
// then 1.  run_start / run_len: the run that holds slot j.
__host__ __device__ constexpr int run_start(int j) {
    const int g = slot_group(j);
    const int end = grp_base(g) + grp_count(g);
    int J = grp_base(g);
    while (J <= j) {
        const int len = (J % 4 == 0 && J + 4 <= end) ? 4 : ((J % 2 == 0 && J + 2 <= end) ? 2 : 1);
        if (j < J + len) return J;
        J += len;
    }
    return -1;
}
__host__ __device__ constexpr int run_len(int j) {
    const int J = run_start(j);
    const int end = grp_base(slot_group(j)) + grp_count(slot_group(j));
    return (J % 4 == 0 && J + 4 <= end) ? 4 : ((J % 2 == 0 && J + 2 <= end) ? 2 : 1);
}

__host__ __device__ constexpr int floordiv(int a, int b) { return a >= 0 ? a / b : -((-a + b - 1) / b); }

// one edge of a block: producer voxel (px, py), direction k; slot >= 0 when
// exported (then the consumer is in another block), else the consumer voxel
// (cx, cy) of the same block (this plane for dz = 0, the next for dz = 1)
struct EdgeInfo {
    int px, py, k, slot, cx, cy;
};
struct EdgeTable {
    EdgeInfo e[NDIR * BV];
    int nexp;
};
// exported edges first, in slot order (group by group, direction by
// direction, voxel by voxel), then the internal ones
constexpr EdgeTable make_edges() {
    EdgeTable t{};
    int n = 0;
    for (int g = 0; g < NGRP; ++g) {
        int slot = grp_base(g);
        for (int k = 0; k < NDIR; ++k)
            for (int py = 0; py < BYV; ++py)
                for (int px = 0; px < BXV; ++px) {
                    const int cx = px + dir_dx(k), cy = py + dir_dy(k);
                    if (floordiv(cx, BXV) == grp_dx(g) && floordiv(cy, BYV) == grp_dy(g))
                        t.e[n++] = EdgeInfo{px, py, k, slot++, cx - grp_dx(g) * BXV,
                                            cy - grp_dy(g) * BYV};
                }
    }
    t.nexp = n;
    for (int k = 0; k < NDIR; ++k)
        for (int py = 0; py < BYV; ++py)
            for (int px = 0; px < BXV; ++px) {
                const int cx = px + dir_dx(k), cy = py + dir_dy(k);
                if (floordiv(cx, BXV) == 0 && floordiv(cy, BYV) == 0)
                    t.e[n++] = EdgeInfo{px, py, k, -1, cx, cy};
            }
    return t;
}
constexpr EdgeTable kEdges = make_edges();

constexpr bool check_edges() {
    int cnt[NGRP] = {};
    for (int i = 0; i < kEdges.nexp; ++i) {
        int g = -1;
        for (int q = 0; q < NGRP; ++q)
            if (kEdges.e[i].slot >= grp_base(q) && kEdges.e[i].slot < grp_base(q) + grp_count(q)) g = q;
        if (g < 0) return false;
        ++cnt[g];
        if (kEdges.e[i].cx < 0 || kEdges.e[i].cx >= BXV || kEdges.e[i].cy < 0 || kEdges.e[i].cy >= BYV)
            return false;
    }
    for (int q = 0; q < NGRP; ++q)
        if (cnt[q] != grp_count(q)) return false;
    // every (voxel, direction) backward term is received exactly once
    int got[BV][NDIR] = {};
    for (int i = 0; i < NDIR * BV; ++i) got[kEdges.e[i].cy * BXV + kEdges.e[i].cx][kEdges.e[i].k]++;
    for (int v = 0; v < BV; ++v)
        for (int k = 0; k < NDIR; ++k)
            if (got[v][k] != 1) return false;
    return kEdges.nexp == 48 && grp_base(NGRP - 1) + 1 <= SLOTS;
}
static_assert(check_edges(), "edge table of the 4 x 2 block");

// Halo items: the edges that ring blocks export into the tile.  Packed as
// .x = producer plane offset | neighbour plane offset << 16,
// .y = destination float index in the export area | dz << 16.
constexpr int NHALO_MAX = 4 * UT;
struct HaloTable {
    int n;
    unsigned int x[NHALO_MAX], y[NHALO_MAX];
};
constexpr HaloTable make_halo() {
    HaloTable h{};
    for (int vby = -1; vby <= TYT; ++vby)
        for (int vbx = -1; vbx <= TXT; ++vbx) {
            if (vbx >= 0 && vbx < TXT && vby >= 0 && vby < TYT) continue;  // real block
            for (int i = 0; i < kEdges.nexp; ++i) {
                const EdgeInfo &e = kEdges.e[i];
                int g = 0;
                for (int q = 0; q < NGRP; ++q)
                    if (e.slot >= grp_base(q) && e.slot < grp_base(q) + grp_count(q)) g = q;
                const int cbx = vbx + grp_dx(g), cby = vby + grp_dy(g);
                if (cbx < 0 || cbx >= TXT || cby < 0 || cby >= TYT) continue;
                const int x = vbx * BXV + e.px, y = vby * BYV + e.py;  // producer voxel
                const int pos = (y + 1) * PW + PX0 + x;
                const int nb = (y + dir_dy(e.k) + 1) * PW + PX0 + x + dir_dx(e.k);
                const int dst = ((vby + 1) * VBW + vbx + 1) * SLOTS + e.slot;
                h.x[h.n] = (unsigned)pos | ((unsigned)nb << 16);
                h.y[h.n] = (unsigned)dst | ((unsigned)dir_dz(e.k) << 16);
                ++h.n;
            }
        }
    return h;
}
constexpr HaloTable kHaloHost = make_halo();
constexpr int NHALO = kHaloHost.n;
constexpr int HALO_PER_THREAD = (NHALO + UT - 1) / UT;
constexpr bool check_halo() {
    for (int i = 0; i < kHaloHost.n; ++i) {
        const int pos = kHaloHost.x[i] & 0xffff, nb = kHaloHost.x[i] >> 16;
        // producers lie in the one-voxel ring of the tile, neighbours inside it
        const int py = pos / PW - 1, px = pos % PW - PX0, ny = nb / PW - 1, nx = nb % PW - PX0;
        if (py < -1 || py > UY || px < -1 || px > UX) return false;
        if (ny < 0 || ny >= UY || nx < 0 || nx >= UX) return false;
        if ((int)(kHaloHost.y[i] & 0xffff) >= NVB * SLOTS) return false;
    }
    return kHaloHost.n <= NHALO_MAX && PN < 65536 && NVB * SLOTS < 65536;
}
static_assert(check_halo(), "halo items out of range");
static_assert(HALO_PER_THREAD <= 4, "at most four halo edges per thread");
struct HaloDev {
    unsigned int x[NHALO_MAX], y[NHALO_MAX];
};
constexpr HaloDev make_halo_dev() {
    HaloDev d{};
    for (int i = 0; i < kHaloHost.n; ++i) {
        d.x[i] = kHaloHost.x[i];
        d.y[i] = kHaloHost.y[i];
    }
    return d;
}
static __device__ const HaloDev kHaloDev = make_halo_dev();

// ---------------------------------------------------------------------------
// per-thread register state of the march
// ---------------------------------------------------------------------------
struct UpdRegs {
    float w0[3][6];      // plane s:   rows y0 .. y0+2, columns x0-1 .. x0+4
    float w1[4][6];      // plane s+1: rows y0-1 .. y0+2, columns x0-1 .. x0+4
    float prior[BV];     // sum w (E_d(u) - E_d(u-d)) of the voxels of plane s
    float pnext[BV];     // the part of plane s+1's sums already known
    float ex[SLOTS];     // this block's exports of the step (registers)
};

// own edge I of the block (compile-time entry of kEdges); exported edges come
// first in slot order, and each run of slots is stored to the block's export
// area dst as soon as its last edge is known.  DZ1ONLY skips the dz = 0
// edges (the seeding step before plane 0; their slots are stored as zeros).
template <int I, bool DZ1ONLY>
__device__ __forceinline__ void own_edges(UpdRegs &r, const PriorParams &pp, float *dst) {
    if constexpr (I < NDIR * BV) {
        constexpr EdgeInfo e = kEdges.e[I];
        constexpr int dz = dir_dz(e.k), dy = dir_dy(e.k), dx = dir_dx(e.k);
        constexpr float w = dir_w(e.k);
        float E = 0.f;
        if constexpr (!(DZ1ONLY && dz == 0)) {
            const float ya = r.w0[e.py][e.px + 1];
            const float yb = dz ? r.w1[e.py + dy + 1][e.px + 1 + dx] : r.w0[e.py + dy][e.px + 1 + dx];
            E = d_pot_unscaled<edge_fma_rcp(I), edge_fma_ex2(I)>(ya - yb, pp);
            if constexpr (!DZ1ONLY) r.prior[e.py * BXV + e.px] = fmaf(w, E, r.prior[e.py * BXV + e.px]);
        }
        if constexpr (e.slot >= 0) {
            r.ex[e.slot] = E;
            constexpr int j0 = run_start(e.slot), len = run_len(e.slot);
            if constexpr (e.slot == j0 + len - 1) {
                if constexpr (len == 4)
                    *reinterpret_cast<float4 *>(dst + j0) =
                        make_float4(r.ex[j0], r.ex[j0 + 1], r.ex[j0 + 2], r.ex[j0 + 3]);
                else if constexpr (len == 2)
                    *reinterpret_cast<float2 *>(dst + j0) = make_float2(r.ex[j0], r.ex[j0 + 1]);
                else
                    dst[j0] = r.ex[j0];
            }
        } else if constexpr (!(DZ1ONLY && dz == 0)) {
            if constexpr (dz == 0)
                r.prior[e.cy * BXV + e.cx] = fmaf(-w, E, r.prior[e.cy * BXV + e.cx]);
            else
                r.pnext[e.cy * BXV + e.cx] = fmaf(-w, E, r.pnext[e.cy * BXV + e.cx]);
        }
        own_edges<I + 1, DZ1ONLY>(r, pp, dst);
    }
}

// subtract w E of the imported values v[0 .. RUN) (exported edges I .. I+RUN)
// from their consumers' sums
template <int I, int J, int RUN, bool DZ1ONLY>
__device__ __forceinline__ void import_run(UpdRegs &r, const float (&v)[4]) {
    if constexpr (J < RUN) {
        constexpr EdgeInfo e = kEdges.e[I + J];
        constexpr float w = dir_w(e.k);
        if constexpr (dir_dz(e.k) == 0) {
            if constexpr (!DZ1ONLY) r.prior[e.cy * BXV + e.cx] = fmaf(-w, v[J], r.prior[e.cy * BXV + e.cx]);
        } else {
            r.pnext[e.cy * BXV + e.cx] = fmaf(-w, v[J], r.pnext[e.cy * BXV + e.cx]);
        }
        import_run<I, J + 1, RUN, DZ1ONLY>(r, v);
    }
}

// imports of exported edge I (kEdges order = slot order) from the block that
// produced it; DZ1ONLY: only the dz = 1 edges (the seeding step)
template <int I, bool DZ1ONLY>
__device__ __forceinline__ void import_edges(UpdRegs &r, const float *es, int vb) {
    if constexpr (I < kEdges.nexp) {
        constexpr EdgeInfo e = kEdges.e[I];
        constexpr int g = slot_group(e.slot);
        constexpr int nbo = -(grp_dy(g) * VBW + grp_dx(g));  // producer block relative to this one
        constexpr int end = grp_base(g) + grp_count(g);
        constexpr int run = (e.slot % 4 == 0 && e.slot + 4 <= end) ? 4
                            : (e.slot % 2 == 0 && e.slot + 2 <= end) ? 2 : 1;
        const float *src = es + (vb + nbo) * SLOTS + e.slot;
        float v[4];
        if constexpr (run == 4) {
            const float4 q = *reinterpret_cast<const float4 *>(src);
            v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
        } else if constexpr (run == 2) {
            const float2 q = *reinterpret_cast<const float2 *>(src);
            v[0] = q.x; v[1] = q.y;
        } else {
            v[0] = src[0];
        }
        import_run<I, 0, run, DZ1ONLY>(r, v);
        import_edges<I + run, DZ1ONLY>(r, es, vb);
    }
}

// ---------------------------------------------------------------------------
// the march
// ---------------------------------------------------------------------------
// SAME: x == sol (every attempt after an accepted step), so y = sol, H y =
// H sol and neither x nor H x is read.  Planes s_lo .. s_hi-1 are written and
// summed; the others (the halo planes of a slab) only serve as neighbours.
template <bool SAME>
__device__ __forceinline__ void update_body(float *__restrict__ X, const float *__restrict__ H,
                                            const float *__restrict__ aty, int S, int R, int C,
                                            size_t vol, const PriorParams &pp,
                                            const MbirState *__restrict__ st,
                                            double *__restrict__ part, int c0, int r0,
                                            int s_lo = 0, int s_hi = 1 << 30,
                                            const CUtensorMap *tmap = nullptr) {
    extern __shared__ __align__(128) float smf[];
    float *yp = smf;                                               // [3][PNA] planes
    float *es = smf + 3 * PNA;                                     // [NVB][SLOTS] exports
    double *accs = reinterpret_cast<double *>(smf + 3 * PNA + NVB * SLOTS);  // [NU][UT]
    uint64_t *bars = reinterpret_cast<uint64_t *>(accs + NU * UT);          // [3]
    const int ix = st->ix, isol = st->isol, inew = st->inew;
    const float beta = st->betaf, step = st->stepf;
    const float *xs = X + (size_t)isol * vol;
    const float *xx = X + (size_t)ix * vol;
    const float *hs = H + (size_t)isol * vol;
    const float *hx = H + (size_t)ix * vol;
    float *out = X + (size_t)inew * vol;
    const int tid = threadIdx.x, tx = tid % TXT, ty = tid / TXT;
    const int x0 = tx * BXV, y0 = ty * BYV;           // block origin in the tile
    const int vb = (ty + 1) * VBW + tx + 1;           // virtual block index
    const size_t plane = (size_t)R * C;
    // 16-byte global rows: every row and every array starts on 16 bytes
    const bool vec = (C % 4) == 0 && (vol % 4) == 0 &&
                     ((reinterpret_cast<uintptr_t>(X) | reinterpret_cast<uintptr_t>(H) |
                       reinterpret_cast<uintptr_t>(aty)) & 15u) == 0;

    // plane items: 18 pieces per tile row (left ring column, 16 runs of 4,
    // right ring column), PH rows; a thread owns items tid + j * UT
    constexpr int PIECES = UX / 4 + 2, NITEM = PIECES * PH;
    constexpr int NIT = (NITEM + UT - 1) / UT;
    // per item: the clamped in-plane offset of its first voxel (-1: none) and
    // its shared-plane offset | 1 << 16 for a run of four | 1 << 17 when the
    // run is one aligned 16-byte copy
    int goff[NIT];
    unsigned int meta[NIT];
#pragma unroll
    for (int j = 0; j < NIT; ++j) {
        const int i = tid + j * UT;
        goff[j] = -1;
        meta[j] = 0u;
        if (i < NITEM) {
            const int row = i / PIECES, pc = i - row * PIECES;
            const int rr = min(max(r0 + row - 1, 0), R - 1);
            const int x = pc == 0 ? -1 : (pc == PIECES - 1 ? UX : 4 * (pc - 1));
            const bool run4 = !(pc == 0 || pc == PIECES - 1);
            const int cc = min(max(c0 + x, 0), C - 1);
            goff[j] = rr * C + cc;
            meta[j] = (unsigned)(row * PW + PX0 + x) | (run4 ? 1u << 16 : 0u) |
                      (run4 && vec && c0 + x + 3 < C ? 1u << 17 : 0u);
        }
    }
    // x == sol: plane p of sol straight into shared memory (cp.async)
    auto copy_plane = [&](int p, float *dst) {
        const size_t base = (size_t)min(max(p, 0), S - 1) * plane;
#pragma unroll
        for (int j = 0; j < NIT; ++j) {
            if (goff[j] < 0) continue;
            const size_t g = base + goff[j];
            float *d = dst + (meta[j] & 0xffffu);
            if (meta[j] & (1u << 17)) {
                cp_async16(d, xs + g);
            } else if (!(meta[j] & (1u << 16))) {
                cp_async4(d, xs + g);
            } else {
                // a run at the right edge of the volume or in a row that is
                // not 16-byte aligned: four clamped copies
                const int cb = goff[j] % C;
                const size_t rowb = g - (size_t)cb;
#pragma unroll
                for (int q = 0; q < 4; ++q) cp_async4(d + q, xs + rowb + min(cb + q, C - 1));
            }
        }
        cp_async_commit();
    };
    // x == sol with a tensor map: one tensor copy per plane, issued by thread 0
    // (the map spans the three iterate buffers as [3 S][R][C])
    const bool tma = SAME && tmap != nullptr && (smem_addr(yp) & 127u) == 0;
    const bool edge = c0 == 0 || r0 == 0 || c0 + UX + 1 > C || r0 + UY + 1 > R;
    unsigned phase = 0;    // bit b: parity of the next completion of plane buffer b
    unsigned pending = 0;  // bit b: a copy into buffer b was issued and not yet waited for
    bool tma_ok = true;
    auto tma_plane = [&](int p, int b) {
        pending |= 1u << b;
        if (tid == 0) {
            fence_proxy_async_smem();
            mbar_arrive_expect_tx(&bars[b], (unsigned)(PW * PH * sizeof(float)));
            tma_load_3d(yp + b * PNA, tmap, c0 - PX0, r0 - 1, isol * S + min(max(p, 0), S - 1),
                        &bars[b]);
        }
    };
    // wait for plane buffer b and, at the volume's border, replace the box's
    // zero fill by clamped values (columns first, then whole rows)
    auto tma_wait = [&](int b) {
        tma_ok = tma_ok && mbar_wait(&bars[b], (phase >> b) & 1u, TMA_WAIT_POLLS);
        phase ^= 1u << b;
        pending &= ~(1u << b);
        if (!edge) return;
        float *pl_ = yp + b * PNA;
        for (int i = tid; i < PH * 2; i += UT) {
            const int row = i >> 1, side = i & 1, y = row - 1;
            if (r0 + y < 0 || r0 + y >= R) continue;
            if (side == 0) {
                if (c0 == 0) pl_[row * PW + PX0 - 1] = pl_[row * PW + PX0];
            } else {
                const int xl = C - 1 - c0;  // last column inside the volume
                for (int x = max(xl + 1, -1); x <= UX; ++x) pl_[row * PW + PX0 + x] = pl_[row * PW + PX0 + xl];
            }
        }
        __syncthreads();
        for (int i = tid; i < PH * (UX + 2); i += UT) {
            const int row = i / (UX + 2), x = i - row * (UX + 2) - 1, y = row - 1;
            const int yc = min(max(r0 + y, 0), R - 1) - r0;
            if (yc != y) pl_[row * PW + PX0 + x] = pl_[(yc + 1) * PW + PX0 + x];
        }
    };

    // x != sol: plane p of y = sol + beta (sol - x) formed in registers
    float4 pys[NIT];
    auto fetch_y = [&](int p) {
        const size_t base = (size_t)min(max(p, 0), S - 1) * plane;
#pragma unroll
        for (int j = 0; j < NIT; ++j) {
            if (goff[j] < 0) continue;
            const size_t g = base + goff[j];
            float a[4], b[4];
            if (meta[j] & (1u << 17)) {
                const float4 u = *reinterpret_cast<const float4 *>(xs + g);
                const float4 w = *reinterpret_cast<const float4 *>(xx + g);
                a[0] = u.x; a[1] = u.y; a[2] = u.z; a[3] = u.w;
                b[0] = w.x; b[1] = w.y; b[2] = w.z; b[3] = w.w;
            } else {
                const int cb = goff[j] % C;
                const size_t rowb = g - (size_t)cb;
                const int n = (meta[j] & (1u << 16)) ? 4 : 1;
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const size_t gi = rowb + min(cb + (q < n ? q : 0), C - 1);
                    a[q] = xs[gi];
                    b[q] = xx[gi];
                }
            }
            pys[j] = make_float4(a[0] + (a[0] - b[0]) * beta, a[1] + (a[1] - b[1]) * beta,
                                 a[2] + (a[2] - b[2]) * beta, a[3] + (a[3] - b[3]) * beta);
        }
    };
    auto store_y = [&](float *dst) {
#pragma unroll
        for (int j = 0; j < NIT; ++j) {
            if (goff[j] < 0) continue;
            float *d = dst + (meta[j] & 0xffffu);
            if (meta[j] & (1u << 16)) *reinterpret_cast<float4 *>(d) = pys[j];
            else d[0] = pys[j].x;
        }
    };

    // the block's voxel data (A^T y, H sol, and for !SAME H x and x) for a plane
    const int gr0 = r0 + y0, gc0 = c0 + x0;
    const bool row_in[2] = {gr0 < R, gr0 + 1 < R};
    const bool full4 = vec && gc0 + 3 < C;
    float4 vhs[2], vaty[2], vhx[2], vxx[2];
    auto ld_run = [&](const float *p, size_t rowbase, float4 &v) {
        if (full4) {
            v = *reinterpret_cast<const float4 *>(p + rowbase + gc0);
        } else {
            float a[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) a[q] = gc0 + q < C ? p[rowbase + gc0 + q] : 0.f;
            v = make_float4(a[0], a[1], a[2], a[3]);
        }
    };
    auto fetch_vox = [&](int s) {
        if (s >= S) return;
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            if (!row_in[q] || gc0 >= C) continue;
            const size_t rb = (size_t)s * plane + (size_t)(gr0 + q) * C;
            ld_run(hs, rb, vhs[q]);
            ld_run(aty, rb, vaty[q]);
            if (!SAME) {
                ld_run(hx, rb, vhx[q]);
                ld_run(xx, rb, vxx[q]);
            }
        }
    };

    // this thread's halo edges (compile-time list in global memory, read each step)
    auto halo_edges = [&](const float *pa, const float *pb, bool dz1only) {
#pragma unroll
        for (int j = 0; j < HALO_PER_THREAD; ++j) {
            const int i = tid + j * UT;
            if (i >= NHALO) continue;
            const unsigned hx_ = __ldg(&kHaloDev.x[i]), hy_ = __ldg(&kHaloDev.y[i]);
            const bool dz = (hy_ >> 16) & 1u;
            if (dz1only && !dz) continue;
            const float ya = pa[hx_ & 0xffffu];
            const float yb = (dz ? pb : pa)[hx_ >> 16];
            es[hy_ & 0xffffu] = d_pot_unscaled(ya - yb, pp);
        }
    };
    // window of plane p (shared buffer) into r.w1
    UpdRegs r;
    auto load_window = [&](const float *p) {
#pragma unroll
        for (int row = 0; row < 4; ++row) {
            const float *q = p + (y0 + row) * PW + PX0 + x0;  // shared row y0 - 1 + row
            const float4 m = *reinterpret_cast<const float4 *>(q);
            r.w1[row][0] = q[-1];
            r.w1[row][1] = m.x;
            r.w1[row][2] = m.y;
            r.w1[row][3] = m.z;
            r.w1[row][4] = m.w;
            r.w1[row][5] = q[4];
        }
    };
    auto shift_window = [&]() {
#pragma unroll
        for (int row = 0; row < 3; ++row)
#pragma unroll
            for (int c = 0; c < 6; ++c) r.w0[row][c] = r.w1[row + 1][c];
    };

#pragma unroll
    for (int k = 0; k < NU; ++k) accs[k * UT + tid] = 0.0;
    float cacc[NU] = {0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int v = 0; v < BV; ++v) r.pnext[v] = 0.f;

    // planes 0 and 1 resident, the voxel data of plane 0 in flight
    if (tma) {
        if (tid == 0) {
#pragma unroll
            for (int b = 0; b < 3; ++b) mbar_init(&bars[b], 1);
            mbar_fence_init();
        }
        __syncthreads();
        tma_plane(0, 0);
        tma_plane(1, 1);
        tma_wait(0);
        __syncthreads();
        tma_wait(1);
    } else if (SAME) {
        copy_plane(0, yp);
        copy_plane(1, yp + PNA);
        cp_async_wait_all();
    } else {
        fetch_y(0);
        store_y(yp);
        fetch_y(1);
        store_y(yp + PNA);
    }
    fetch_vox(0);
    __syncthreads();
    // seed: the dz = 1 edges from plane -1 (clamped to plane 0) into plane 0
    load_window(yp);
    shift_window();
    own_edges<0, true>(r, pp, es + vb * SLOTS);
    halo_edges(yp, yp, true);
    __syncthreads();
    import_edges<0, true>(r, es, vb);

    int bc = 0;  // buffer of plane s (plane s+1 in bc+1, s+2 in bc+2, mod 3)
    for (int s = 0; s < S; ++s) {
        const int b1 = bc == 2 ? 0 : bc + 1, b2 = b1 == 2 ? 0 : b1 + 1;
        float *ycur = yp + bc * PNA, *ynxt = yp + b1 * PNA, *yfill = yp + b2 * PNA;
        // plane s+1 resident; the last step's imports done; plane s-1 free;
        // a tensor-copy wait that gave up anywhere ends the CTA's march
        if (tma) {
            if (__syncthreads_or(!tma_ok)) {
                if (tid == 0) const_cast<MbirState *>(st)->status = UPD_STATUS_TMA_TIMEOUT;
                // copies still in flight land in this CTA's own shared memory;
                // wait for them (bounded) before the CTA exits
                if (tid == 0)
                    for (int b = 0; b < 3; ++b)
                        if (pending & (1u << b)) mbar_wait(&bars[b], (phase >> b) & 1u, TMA_WAIT_POLLS);
                return;
            }
        } else {
            __syncthreads();
        }
        if (tma) tma_plane(s + 2, b2);
        else if (SAME) copy_plane(s + 2, yfill);
        else fetch_y(s + 2);
        load_window(ynxt);
#pragma unroll
        for (int v = 0; v < BV; ++v) {
            r.prior[v] = r.pnext[v];
            r.pnext[v] = 0.f;
        }
        own_edges<0, false>(r, pp, es + vb * SLOTS);
        halo_edges(ycur, ynxt, false);
        __syncthreads();  // exports visible
        float4 chs[2], caty[2], chx[2], cxx[2];
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            chs[q] = vhs[q];
            caty[q] = vaty[q];
            chx[q] = vhx[q];
            cxx[q] = vxx[q];
        }
        fetch_vox(s + 1);
        import_edges<0, false>(r, es, vb);
        if (s >= s_lo && s < s_hi) {
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                if (!row_in[q] || gc0 >= C) continue;
                const float hsa[4] = {chs[q].x, chs[q].y, chs[q].z, chs[q].w};
                const float ata[4] = {caty[q].x, caty[q].y, caty[q].z, caty[q].w};
                const float hxa[4] = {chx[q].x, chx[q].y, chx[q].z, chx[q].w};
                const float xxa[4] = {cxx[q].x, cxx[q].y, cxx[q].z, cxx[q].w};
                float sn[4];
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    const float u = r.w0[q][c + 1];
                    const float hy = SAME ? hsa[c] : (1.0f + beta) * hsa[c] - beta * hxa[c];
                    const float a = ata[c];
                    const float g = (hy - a) + (pp.scale * pp.inv_sq) * r.prior[q * BXV + c];
                    sn[c] = u - g * step;
                    if (gc0 + c < C) {
                        const float xv = SAME ? u : xxa[c];
                        const float dxf = sn[c] - xv;
                        cacc[0] = fmaf(u, hy, cacc[0]);
                        cacc[1] = fmaf(u, a, cacc[1]);
                        cacc[2] = fmaf(g, g, cacc[2]);
                        cacc[3] = fmaf(sn[c], a, cacc[3]);
                        cacc[4] = fmaf(dxf, dxf, cacc[4]);
                    }
                }
                const size_t rb = (size_t)s * plane + (size_t)(gr0 + q) * C;
                if (full4) {
                    *reinterpret_cast<float4 *>(out + rb + gc0) = make_float4(sn[0], sn[1], sn[2], sn[3]);
                } else {
#pragma unroll
                    for (int c = 0; c < 4; ++c)
                        if (gc0 + c < C) out[rb + gc0 + c] = sn[c];
                }
            }
        }
        shift_window();
        if ((s % ACC_CHUNK) == ACC_CHUNK - 1 || s == S - 1) {
#pragma unroll
            for (int k = 0; k < NU; ++k) {
                accs[k * UT + tid] += (double)cacc[k];
                cacc[k] = 0.f;
            }
        }
        if (tma) tma_wait(b2);
        else if (SAME) cp_async_wait_all();
        else store_y(yfill);
        bc = b1;
    }
    double acc[NU];
#pragma unroll
    for (int k = 0; k < NU; ++k) acc[k] = accs[k * UT + tid];
    block_sum<NU>(acc, tid, UT);
    if (tid == 0) {
#pragma unroll
        for (int k = 0; k < NU; ++k) part[k] = acc[k];
    }
}

}  // namespace tc
