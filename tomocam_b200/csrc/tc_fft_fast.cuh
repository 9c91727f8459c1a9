// tc_fft_fast.cuh -- register-resident FFT of length M = R1 R2 R3 for the
// Toeplitz passes (R1, R2, R3 in {2, 4, 8, 16}).
//
// Each line is transformed by T = M / 16 threads holding 16 values each.
// Forward (sign -, decimation in frequency), with n = B n1 + m,
// B = R2 R3, m = R3 n2 + m3 and k = R1 R2 k3 + R1 k2 + k1:
//   stage 1  DFT_R1 over n1 for each m, twiddle W_M^(m k1)
//   stage 2  DFT_R2 over n2 for each (k1, m3), twiddle W_M^(R1 m3 k2)
//   stage 3  DFT_R3 over m3 for each (k1, k2)
// Stages exchange values through a padded shared-memory line.  The output is
// left in the order stage 3 produces it: value v of thread t holds frequency
// kidx(t, v).  The inverse (sign +) is the exact adjoint and takes its input
// in that same order, so a forward transform, a pointwise product and an
// inverse transform never reorder data.
//
// When R2 = R3 = 16 every stage-2 group (fixed k1) and its stage-3 group are
// the same 16 threads (a half warp).  The line is then laid out so that the
// stage-1/2 exchange row k1 (A1) and the stage-2/3 exchange block of group k1
// (A2) occupy the same addresses: that exchange needs only a warp barrier and
// its contiguous side moves 16 bytes per access.  One CTA barrier per
// transform remains (the stage-1/2 exchange, which spans the whole line).
#pragma once

#include "tc_fft.cuh"

namespace tc {

__device__ __forceinline__ c32 ldtw(const c32 *__restrict__ tw, int i) {
    const float2 f = __ldg(reinterpret_cast<const float2 *>(tw) + i);
    return mk<float>(f.x, f.y);
}

// wp[k] = w^k for k < R, by squarings and one multiply per odd power
// (chains of at most 4 products, a few ulp of phase error)
template <int R>
__device__ __forceinline__ void powers(c32 w, c32 *wp) {
    wp[0] = mk<float>(1.f, 0.f);
    if constexpr (R > 1) wp[1] = w;
#pragma unroll
    for (int k = 2; k < R; ++k) wp[k] = (k & 1) ? cmul(wp[k - 1], w) : cmul(wp[k / 2], wp[k / 2]);
}

template <int R, int DIR>
__device__ __forceinline__ void dft_r(c32 *v) {
    if constexpr (R == 2) dft2<float, DIR>(v[0], v[1]);
    else if constexpr (R == 4) dft4<float, DIR>(v[0], v[1], v[2], v[3]);
    else if constexpr (R == 8) dft8<float, DIR>(v);
    else dft16<float, DIR>(v);
}

// TWS: stride of the twiddle indices (1 for a stand-alone transform; R0 for
// the inner transforms of FastFFT4, whose table is that of the outer length)
template <int R1_, int R2_, int R3_, int TWS = 1>
struct FastFFT {
    static constexpr int R1 = R1_, R2 = R2_, R3 = R3_;
    static constexpr int M = R1 * R2 * R3;
    static constexpr int T = M / 16;  // threads per line
    static constexpr int B = R2 * R3;
    static constexpr int G1 = 16 / R1, G2 = 16 / R2, G3 = 16 / R3;
    static constexpr bool WG = (R2 == 16 && R3 == 16);  // half-warp stage-2/3 groups
    static constexpr int LD2 = WG ? R3 + 2 : R3 + 1;
    static constexpr int LD1 = WG ? R2 * LD2 : B + 1;
    static constexpr int SMEM = WG ? R1 * LD1
                                   : ((R1 * LD1 > R1 * R2 * LD2) ? R1 * LD1 : R1 * R2 * LD2);
    // stride between the lines of one CTA: +8 complex moves the next line 16
    // banks over, so lines interleaved within a warp do not collide
    static constexpr int LS = SMEM + 8;
    static_assert(M % 16 == 0 && T >= 1, "M must be a multiple of 16");

    __device__ __forceinline__ static int a1(int m, int k1) { return k1 * LD1 + m; }
    __device__ __forceinline__ static int a2(int k1, int k2, int m3) {
        return WG ? k1 * LD1 + k2 * LD2 + m3 : (k1 * R2 + k2) * LD2 + m3;
    }
    __device__ __forceinline__ static void sync23() {
        if constexpr (WG) __syncwarp();
        else __syncthreads();
    }

    // frequency held by value v of thread t after forward()
    __host__ __device__ static int kidx(int t, int v) {
        const int j = v / R3, k3 = v % R3;
        const int q = t + T * j;
        const int k2 = q % R2, k1 = q / R2;
        return R1 * R2 * k3 + R1 * k2 + k1;
    }
    // input index of value v of thread t for forward() / output of inverse()
    __host__ __device__ static int nidx(int t, int v) {
        const int j = v / R1, n1 = v % R1;
        return B * n1 + t + T * j;
    }
    // values whose index is below M/2: the only ones a zero-padded line of
    // length <= M/2 can hold (n1 < R1/2); the others are known zeros on input
    // and unneeded on output
    __host__ __device__ static constexpr bool low_half(int v) { return (v % R1) < R1 / 2; }

    // v[16] holds x[nidx(t, .)] on entry and X[kidx(t, .)] on exit.
    // sm: this line's shared memory, not in use by other threads on entry.
    // tw[k] = exp(-2 pi i k / M).  HALF: the input is zero from M/2 on (the
    // high-half values are treated as compile-time zeros).
    template <bool HALF = false>
    __device__ __forceinline__ static void forward(c32 *v, c32 *sm, int t,
                                                   const c32 *__restrict__ tw) {
        if constexpr (HALF) {
#pragma unroll
            for (int i = 0; i < 16; ++i)
                if (!low_half(i)) v[i] = mk<float>(0.f, 0.f);
        }
#pragma unroll
        for (int j = 0; j < G1; ++j) {
            const int m = t + T * j;
            c32 wp[R1];
            powers<R1>(ldtw(tw, m * TWS), wp);
            dft_r<R1, -1>(v + j * R1);
#pragma unroll
            for (int k1 = 0; k1 < R1; ++k1) {
                c32 a = v[j * R1 + k1];
                if (k1 > 0) a = cmul(a, wp[k1]);
                sm[a1(m, k1)] = a;
            }
        }
        __syncthreads();
#pragma unroll
        for (int j = 0; j < G2; ++j) {
            const int q = t + T * j, m3 = q % R3, k1 = q / R3;
#pragma unroll
            for (int n2 = 0; n2 < R2; ++n2) v[j * R2 + n2] = sm[a1(R3 * n2 + m3, k1)];
        }
        sync23();
#pragma unroll
        for (int j = 0; j < G2; ++j) {
            const int q = t + T * j, m3 = q % R3, k1 = q / R3;
            c32 wp[R2];
            powers<R2>(ldtw(tw, R1 * m3 * TWS), wp);
            dft_r<R2, -1>(v + j * R2);
#pragma unroll
            for (int k2 = 0; k2 < R2; ++k2) {
                c32 a = v[j * R2 + k2];
                if (k2 > 0) a = cmul(a, wp[k2]);
                sm[a2(k1, k2, m3)] = a;
            }
        }
        sync23();
#pragma unroll
        for (int j = 0; j < G3; ++j) {
            const int q = t + T * j, k2 = q % R2, k1 = q / R2;
            if constexpr (WG) {
                const float4 *p = reinterpret_cast<const float4 *>(sm + a2(k1, k2, 0));
#pragma unroll
                for (int i = 0; i < R3 / 2; ++i) {
                    const float4 f = p[i];
                    v[j * R3 + 2 * i] = mk<float>(f.x, f.y);
                    v[j * R3 + 2 * i + 1] = mk<float>(f.z, f.w);
                }
            } else {
#pragma unroll
                for (int m3 = 0; m3 < R3; ++m3) v[j * R3 + m3] = sm[a2(k1, k2, m3)];
            }
            dft_r<R3, -1>(v + j * R3);
        }
    }

    // exact adjoint of forward(): v[16] holds X[kidx(t, .)] on entry and
    // M * x[nidx(t, .)] (unnormalised inverse DFT) on exit.  On entry the
    // line must be free (after forward() on the same line, the caller calls
    // sync_before_inverse()).  HALF_OUT (only the values v with low_half(v)
    // are used) changes nothing here: the unused outputs are dead code.
    template <bool HALF_OUT = false, bool LOW_FORM = false>
    __device__ __forceinline__ static void inverse(c32 *v, c32 *sm, int t,
                                                   const c32 *__restrict__ tw) {
#pragma unroll
        for (int j = 0; j < G3; ++j) {
            const int q = t + T * j, k2 = q % R2, k1 = q / R2;
            dft_r<R3, +1>(v + j * R3);
            if constexpr (WG) {
                float4 *p = reinterpret_cast<float4 *>(sm + a2(k1, k2, 0));
#pragma unroll
                for (int i = 0; i < R3 / 2; ++i)
                    p[i] = make_float4(v[j * R3 + 2 * i].x, v[j * R3 + 2 * i].y,
                                       v[j * R3 + 2 * i + 1].x, v[j * R3 + 2 * i + 1].y);
            } else {
#pragma unroll
                for (int m3 = 0; m3 < R3; ++m3) sm[a2(k1, k2, m3)] = v[j * R3 + m3];
            }
        }
        sync23();
#pragma unroll
        for (int j = 0; j < G2; ++j) {
            const int q = t + T * j, m3 = q % R3, k1 = q / R3;
#pragma unroll
            for (int k2 = 0; k2 < R2; ++k2) v[j * R2 + k2] = sm[a2(k1, k2, m3)];
        }
        sync23();
#pragma unroll
        for (int j = 0; j < G2; ++j) {
            const int q = t + T * j, m3 = q % R3, k1 = q / R3;
            c32 wp[R2];
            powers<R2>(ldtw(tw, R1 * m3 * TWS), wp);
#pragma unroll
            for (int k2 = 1; k2 < R2; ++k2) v[j * R2 + k2] = cmulc(v[j * R2 + k2], wp[k2]);
            dft_r<R2, +1>(v + j * R2);
#pragma unroll
            for (int n2 = 0; n2 < R2; ++n2) sm[a1(R3 * n2 + m3, k1)] = v[j * R2 + n2];
        }
        __syncthreads();
#pragma unroll
        for (int j = 0; j < G1; ++j) {
            const int m = t + T * j;
            c32 wp[R1];
            powers<R1>(ldtw(tw, m * TWS), wp);
#pragma unroll
            for (int k1 = 0; k1 < R1; ++k1) {
                c32 a = sm[a1(m, k1)];
                if (k1 > 0) a = cmulc(a, wp[k1]);
                v[j * R1 + k1] = a;
            }
            dft_r<R1, +1>(v + j * R1);
        }
    }

    // between forward() and inverse() on the same line
    __device__ __forceinline__ static void sync_before_inverse() { sync23(); }
};

// Length M = R0 * Inner::M with one more radix-R0 stage in front (M = 8192 as
// 2 x 4096).  Decimation in frequency: with n = Mi n0 + m (Mi = Inner::M),
//   X[R0 k' + k0] = DFT_Mi( sum_n0 x[Mi n0 + m] W_R0^(n0 k0) W_M^(m k0) )[k'],
// so after the outer stage and one exchange through shared memory, the R0
// groups of Ti = Inner::T consecutive threads each run the inner transform on
// their k0 (Inner must use twiddle stride R0).  T = R0 Ti threads per line,
// 16 values each, as for FastFFT.
template <int R0_, class Inner>
struct FastFFT4 {
    static constexpr int R0 = R0_;
    static constexpr int Mi = Inner::M, M = R0 * Mi;
    static constexpr int Ti = Inner::T, T = R0 * Ti;
    static constexpr int G0 = 16 / R0;
    static constexpr int LDB = Mi + 8;  // exchange row of one k0
    static constexpr int SMEM = (R0 * LDB > R0 * Inner::LS) ? R0 * LDB : R0 * Inner::LS;
    static constexpr int LS = SMEM + 8;
    static_assert(16 % R0 == 0, "R0 must divide 16");

    __host__ __device__ static int kidx(int t, int v) {
        return R0 * Inner::kidx(t % Ti, v) + t / Ti;
    }
    __host__ __device__ static int nidx(int t, int v) {
        const int j = v / R0, n0 = v % R0;
        return Mi * n0 + t + T * j;
    }
    __host__ __device__ static constexpr bool low_half(int v) { return (v % R0) < R0 / 2; }

    template <bool HALF = false>
    __device__ __forceinline__ static void forward(c32 *v, c32 *sm, int t,
                                                   const c32 *__restrict__ tw) {
        if constexpr (HALF) {
#pragma unroll
            for (int i = 0; i < 16; ++i)
                if (!low_half(i)) v[i] = mk<float>(0.f, 0.f);
        }
#pragma unroll
        for (int j = 0; j < G0; ++j) {
            const int m = t + T * j;
            c32 wp[R0];
            powers<R0>(ldtw(tw, m), wp);
            dft_r<R0, -1>(v + j * R0);
#pragma unroll
            for (int k0 = 0; k0 < R0; ++k0) {
                c32 a = v[j * R0 + k0];
                if (k0 > 0) a = cmul(a, wp[k0]);
                sm[k0 * LDB + m] = a;
            }
        }
        __syncthreads();
        const int k0 = t / Ti, ti = t % Ti;
#pragma unroll
        for (int i = 0; i < 16; ++i) v[i] = sm[k0 * LDB + Inner::nidx(ti, i)];
        __syncthreads();  // the exchange rows become the inner transforms' scratch
        Inner::forward(v, sm + k0 * Inner::LS, ti, tw);
    }

    // exact adjoint of forward(); on entry the line must be free (after
    // forward() on the same line, call sync_before_inverse()).  HALF_OUT as
    // for FastFFT.
    template <bool HALF_OUT = false, bool LOW_FORM = false>
    __device__ __forceinline__ static void inverse(c32 *v, c32 *sm, int t,
                                                   const c32 *__restrict__ tw) {
        const int k0 = t / Ti, ti = t % Ti;
        Inner::inverse(v, sm + k0 * Inner::LS, ti, tw);
        __syncthreads();
#pragma unroll
        for (int i = 0; i < 16; ++i) sm[k0 * LDB + Inner::nidx(ti, i)] = v[i];
        __syncthreads();
#pragma unroll
        for (int j = 0; j < G0; ++j) {
            const int m = t + T * j;
            c32 wp[R0];
            powers<R0>(ldtw(tw, m), wp);
#pragma unroll
            for (int kk = 0; kk < R0; ++kk) {
                c32 a = sm[kk * LDB + m];
                if (kk > 0) a = cmulc(a, wp[kk]);
                v[j * R0 + kk] = a;
            }
            dft_r<R0, +1>(v + j * R0);
        }
    }

    __device__ __forceinline__ static void sync_before_inverse() { Inner::sync_before_inverse(); }
};

// cos and sin of 2 pi j / 48, j = 0 .. 31: W_48^j = (kC48[j], -kS48[j])
constexpr double kC48[32] = {
    1.0, 0.9914448613738104, 0.9659258262890683, 0.9238795325112867, 0.8660254037844387,
    0.7933533402912352, 0.7071067811865476, 0.6087614290087207, 0.5, 0.38268343236508984,
    0.25881904510252074, 0.1305261922200517, 0.0, -0.1305261922200516, -0.25881904510252063,
    -0.3826834323650895, -0.5, -0.6087614290087207, -0.7071067811865475, -0.793353340291235,
    -0.8660254037844387, -0.9238795325112867, -0.9659258262890682, -0.9914448613738104, -1.0,
    -0.9914448613738104, -0.9659258262890683, -0.9238795325112868, -0.8660254037844388,
    -0.7933533402912352, -0.7071067811865479, -0.6087614290087209};
constexpr double kS48[32] = {
    0.0, 0.13052619222005157, 0.25881904510252074, 0.3826834323650898, 0.5,
    0.6087614290087207, 0.7071067811865475, 0.7933533402912352, 0.8660254037844386,
    0.9238795325112867, 0.9659258262890683, 0.9914448613738104, 1.0, 0.9914448613738104,
    0.9659258262890683, 0.9238795325112868, 0.8660254037844387, 0.7933533402912352,
    0.7071067811865476, 0.6087614290087209, 0.5, 0.3826834323650899, 0.258819045102521,
    0.130526192220052, 0.0, -0.13052619222005177, -0.2588190451025208, -0.38268343236508967,
    -0.5, -0.6087614290087207, -0.7071067811865471, -0.7933533402912349};

// Length M = 3 * Inner::M (6144 = 3 x 2048) with one radix-3 stage in front
// (Inner must use twiddle stride 3).  T = 3 Ti threads (Ti = Inner::T), 16
// values each; on the input side value v of thread t is x[t + T v], so the
// values v >= 8 are the upper half (n >= M / 2).  Decimation in frequency:
// with n = Mi n0 + m (Mi = Inner::M),
//   X[3 k' + k0] = DFT_Mi( sum_n0 x[Mi n0 + m] W_3^(n0 k0) W_M^(m k0) )[k'].
// The radix-3 stage runs in shared memory over the whole line: column m
// (x[m], x[Mi + m], x[2 Mi + m]) is replaced in place by its three twiddled
// outputs, then the Ti threads of group k0 load row k0 and run the inner
// transform on it; the line's shared memory then serves as the three inner
// transforms' scratch.
template <class Inner>
struct FastFFT3 {
    static constexpr int R0 = 3;
    static constexpr int Mi = Inner::M, M = 3 * Mi;
    static constexpr int Ti = Inner::T, T = 3 * Ti;
    static constexpr int SMEM = (M > 3 * Inner::LS) ? M : 3 * Inner::LS;
    static constexpr int LS = SMEM + 8;
    static constexpr int RJ = (Mi + T - 1) / T;  // radix-3 columns per thread
    // inverse<true> forms the low half directly (scatter_half) up to
    // M = 3072; at M = 6144 the column pass runs under an 80-register cap
    // (two CTAs of 384 threads) where that form spills more than the radix-3
    // pass over the line, so it is the default only up to 3072 and the
    // output pass asks for it explicitly (inverse<true, true>)
    static constexpr bool INV_HALF = M <= 3072;
    static_assert(T * 16 == M, "16 values per thread");

    __host__ __device__ static int kidx(int t, int v) {
        return 3 * Inner::kidx(t % Ti, v) + t / Ti;
    }
    __host__ __device__ static int nidx(int t, int v) { return t + T * v; }
    __host__ __device__ static constexpr bool low_half(int v) { return v < 8; }

    // value of inner thread ti holding column m = ti + Ti u (u < 16) of its
    // group: Inner::nidx(ti, vslot(u)) = ti + Ti u
    __host__ __device__ static constexpr int vslot(int u) {
        return (u % Inner::G1) * Inner::R1 + u / Inner::G1;
    }

    template <bool HALF = false>
    __device__ __forceinline__ static void forward(c32 *v, c32 *sm, int t,
                                                   const c32 *__restrict__ tw) {
        if constexpr (HALF) {
            forward_half(v, sm, t, tw);
        } else {
#pragma unroll
            for (int i = 0; i < 16; ++i) sm[t + T * i] = v[i];
            __syncthreads();
            {
                // columns m = t + T j; W^m advanced by W^T (one table read
                // each, no dependent table reads inside the loop), W^2m = (W^m)^2
                c32 w = ldtw(tw, t);
                const c32 wT = ldtw(tw, T);
#pragma unroll 1
                for (int j = 0; j < RJ; ++j) {
                    const int m = t + T * j;
                    if (m < Mi) {
                        c32 y[3] = {sm[m], sm[Mi + m], sm[2 * Mi + m]};
                        dft3<float, -1>(y);
                        sm[m] = y[0];
                        sm[Mi + m] = cmul(y[1], w);
                        sm[2 * Mi + m] = cmul(y[2], cmul(w, w));
                    }
                    w = cmul(w, wT);
                }
            }
            __syncthreads();
            const int k0 = t / Ti, ti = t % Ti;
#pragma unroll
            for (int i = 0; i < 16; ++i) v[i] = sm[k0 * Mi + Inner::nidx(ti, i)];
            __syncthreads();  // the line becomes the inner transforms' scratch
            Inner::forward(v, sm + k0 * Inner::LS, ti, tw);
        }
    }

    // forward() of a line whose upper half (n >= M / 2, values v >= 8) is
    // zero.  Column m holds (x[m], x[Mi + m], 0), and x[Mi + m] = 0 too for
    // m >= Mi / 2, so the radix-3 stage reduces to y_k0[m] = (x[m] +
    // W_3^k0 x[Mi + m]) W_M^(m k0): the line's low half goes to shared
    // memory once and each thread of group k0 forms its own 16 inputs of
    // the inner transform (columns m = ti + Ti u) from it, with no radix-3
    // pass over the line.  W_M^(m k0) = W_M^(ti k0) W_48^(u k0) (Ti u / M =
    // u / 48): the first from the table, the second a compile-time constant
    // of the group's code (groups are whole warps, so the branch on k0 does
    // not diverge).
    template <int K0, int U = 0>
    __device__ __forceinline__ static void gather_half(c32 *v, const c32 *sm, int ti, c32 wt) {
        if constexpr (U < 16) {
            constexpr float c3 = K0 ? float(kc::C3) : 1.f;
            constexpr float s3 = K0 == 1 ? -float(kc::S3) : (K0 == 2 ? float(kc::S3) : 0.f);
            const int m = ti + Ti * U;
            c32 a = sm[m];
            if constexpr (U < 8) {  // m < Mi / 2: x[Mi + m] is in the low half
                const c32 b = sm[Mi + m];
                if constexpr (K0 == 0)
                    a = a + b;
                else
                    a = mk<float>(fmaf(c3, b.x, fmaf(-s3, b.y, a.x)),
                                  fmaf(c3, b.y, fmaf(s3, b.x, a.y)));
            }
            if constexpr (K0 != 0) {
                constexpr float wc = float(kC48[U * K0]), ws = -float(kS48[U * K0]);
                if constexpr (U != 0) a = cmul(a, mk<float>(wc, ws));
                a = cmul(a, wt);
            }
            v[vslot(U)] = a;
            gather_half<K0, U + 1>(v, sm, ti, wt);
        }
    }

    __device__ __forceinline__ static void forward_half(c32 *v, c32 *sm, int t,
                                                        const c32 *__restrict__ tw) {
#pragma unroll
        for (int i = 0; i < 8; ++i) sm[t + T * i] = v[i];
        __syncthreads();
        const int k0 = t / Ti, ti = t % Ti;
        const c32 wt = ldtw(tw, ti * k0);
        if (k0 == 0) gather_half<0>(v, sm, ti, wt);
        else if (k0 == 1) gather_half<1>(v, sm, ti, wt);
        else gather_half<2>(v, sm, ti, wt);
        __syncthreads();  // the line becomes the inner transforms' scratch
        Inner::forward(v, sm + k0 * Inner::LS, ti, tw);
    }

    // the inner inverse's outputs z_k0[m] W_M^(-m k0) to shared memory
    // (group k0's row; W_M^(-m k0) = conj(W_M^(ti k0) W_48^(u k0)))
    template <int K0, int U = 0>
    __device__ __forceinline__ static void scatter_half(const c32 *v, c32 *sm, int ti, c32 wt) {
        if constexpr (U < 16) {
            c32 z = v[vslot(U)];
            if constexpr (K0 != 0) {
                constexpr float wc = float(kC48[U * K0]), ws = -float(kS48[U * K0]);
                if constexpr (U != 0) z = cmulc(z, mk<float>(wc, ws));
                z = cmulc(z, wt);
            }
            sm[K0 * Mi + ti + Ti * U] = z;
            scatter_half<K0, U + 1>(v, sm, ti, wt);
        }
    }

    // exact adjoint of forward(); on entry the line must be free (after
    // forward() on the same line, call sync_before_inverse()).  HALF_OUT:
    // only the low half of the output (values v < 8, n < M / 2) is used; with
    // INV_HALF only that half is formed and the upper values are undefined.
    // LOW_FORM (default INV_HALF) picks the low-half form for a caller whose
    // register budget takes it at M = 6144.
    template <bool HALF_OUT = false, bool LOW_FORM = INV_HALF>
    __device__ __forceinline__ static void inverse(c32 *v, c32 *sm, int t,
                                                   const c32 *__restrict__ tw) {
        const int k0 = t / Ti, ti = t % Ti;
        Inner::inverse(v, sm + k0 * Inner::LS, ti, tw);
        __syncthreads();
        if constexpr (HALF_OUT && LOW_FORM) {
            // the inner outputs z'_k0[m] = z_k0[m] W_M^(-m k0) to shared
            // memory, then x[m + Mi n0] = sum_k0 W_3^(-n0 k0) z'_k0[m] for the
            // outputs n = t + T i < M / 2 (n0 = 0 or 1)
            const c32 wt = ldtw(tw, ti * k0);
            if (k0 == 0) scatter_half<0>(v, sm, ti, wt);
            else if (k0 == 1) scatter_half<1>(v, sm, ti, wt);
            else scatter_half<2>(v, sm, ti, wt);
            __syncthreads();
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const int n = t + T * i;
                const bool hi = n >= Mi;
                const int m = hi ? n - Mi : n;
                const c32 z0 = sm[m], z1 = sm[Mi + m], z2 = sm[2 * Mi + m];
                const c32 sp = z1 + z2, dm = z1 - z2;
                // n0 = 0: z0 + z1 + z2; n0 = 1: z0 - (z1 + z2) / 2 + i S3 (z1 - z2)
                const float c = hi ? float(kc::C3) : 1.f, s = hi ? float(kc::S3) : 0.f;
                v[i] = mk<float>(fmaf(c, sp.x, fmaf(-s, dm.y, z0.x)), fmaf(c, sp.y, fmaf(s, dm.x, z0.y)));
                // one output's shared-memory reads at a time: read ahead,
                // the eight outputs' 24 values would not fit the register
                // budget of the M = 6144 passes
                asm volatile("" ::: "memory");
            }
        } else {
#pragma unroll
            for (int i = 0; i < 16; ++i) sm[k0 * Mi + Inner::nidx(ti, i)] = v[i];
            __syncthreads();
            {
                c32 w = ldtw(tw, t);
                const c32 wT = ldtw(tw, T);
#pragma unroll 1
                for (int j = 0; j < RJ; ++j) {
                    const int m = t + T * j;
                    if (m < Mi) {
                        c32 y[3] = {sm[m], cmulc(sm[Mi + m], w), cmulc(sm[2 * Mi + m], cmul(w, w))};
                        dft3<float, +1>(y);
                        sm[m] = y[0];
                        sm[Mi + m] = y[1];
                        sm[2 * Mi + m] = y[2];
                    }
                    w = cmul(w, wT);
                }
            }
            __syncthreads();
#pragma unroll
            for (int i = 0; i < 16; ++i) v[i] = sm[t + T * i];
        }
    }

    __device__ __forceinline__ static void sync_before_inverse() { Inner::sync_before_inverse(); }
};

// the register-FFT lengths
using F64 = FastFFT<4, 4, 4>;
using F128 = FastFFT<8, 4, 4>;
using F256 = FastFFT<8, 8, 4>;
using F512 = FastFFT<2, 16, 16>;
using F1024 = FastFFT<4, 16, 16>;
using F1536 = FastFFT3<FastFFT<2, 16, 16, 3>>;
using F2048 = FastFFT<8, 16, 16>;
using F3072 = FastFFT3<FastFFT<4, 16, 16, 3>>;
using F4096 = FastFFT<16, 16, 16>;
using F6144 = FastFFT3<FastFFT<8, 16, 16, 3>>;
using F8192 = FastFFT4<2, FastFFT<16, 16, 16, 2>>;

}  // namespace tc
