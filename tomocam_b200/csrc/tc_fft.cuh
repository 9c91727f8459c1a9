// tc_fft.cuh -- the FFT engine behind every operator.
//
// A CTA transforms one or more lines that sit in shared memory.  Lengths
// whose prime factors are 2, 3, 5, 7 run as a self-sorting (Stockham)
// mixed-radix FFT with radix-16/8/4/2/3/5/7 butterflies; any other length
// runs through Bluestein's chirp-z identity on a smooth inner length.
// Every stage loads all of a thread's butterfly inputs into registers,
// synchronises, and writes the outputs back in place, so a line needs only
// its own length of shared memory.
//
// Twiddles come from a per-length table tw[k] = exp(-2 pi i k / L) built on
// the host in double precision.  Transforms are unnormalised; DIR = -1 is
// the forward sign exp(-i ...), DIR = +1 the inverse sign.
#pragma once

#include <complex>
#include <vector>

#include "tc_common.cuh"

namespace tc {

constexpr int FFT_MAX_STAGES = 24;
// CTAs that run the engine have at most this many threads
constexpr int FFT_MAX_THREADS = 512;
// values each thread holds per stage: a CTA of nthr threads may transform
// nlines lines of length L in one call when nlines * L <= fft_vpt<R>() * nthr
template <typename R>
__host__ __device__ constexpr int fft_vpt() {
    return sizeof(R) == 4 ? 16 : 32;
}
// threads for a CTA that transforms `lines` lines of inner length L
template <typename R>
inline int fft_threads(int L, int lines) {
    int t = (L * lines + fft_vpt<R>() - 1) / fft_vpt<R>();
    t = (t + 31) / 32 * 32;
    return t < 64 ? 64 : t;
}

template <typename R>
struct FftDev {
    int n;         // logical transform length
    int L;         // length of the Stockham transform (== n unless Bluestein)
    int nst;       // number of stages
    int bluestein; // 1: n is not 2,3,5,7-smooth
    int radix[FFT_MAX_STAGES];
    const cpx<R> *tw;      // L entries
    const cpx<R> *chirp;   // n entries exp(i pi m^2 / n) (Bluestein)
    const cpx<R> *bhat_f;  // L entries, FFT of the chirp (forward DFT)
    const cpx<R> *bhat_i;  // L entries, FFT of the conjugate chirp
};

// --------------------------------------------------------------------------
// small DFTs in registers
// --------------------------------------------------------------------------
namespace kc {
// cos / sin of 2 pi j / R
constexpr double C3 = -0.5, S3 = 0.8660254037844386467637;
constexpr double C51 = 0.3090169943749474241023, S51 = 0.9510565162951535721164;
constexpr double C52 = -0.8090169943749474241023, S52 = 0.5877852522924731291687;
constexpr double C71 = 0.623489801858733530525, S71 = 0.7818314824680298087084;
constexpr double C72 = -0.2225209339563144042889, S72 = 0.9749279121818236070181;
constexpr double C73 = -0.9009688679024191262361, S73 = 0.4338837391175581204758;
constexpr double R2 = 0.7071067811865475244008;   // cos(pi/4)
constexpr double C16 = 0.9238795325112867561282;  // cos(pi/8)
constexpr double S16 = 0.3826834323650897717285;  // sin(pi/8)
}  // namespace kc

template <typename R, int DIR>
__device__ __forceinline__ void dft2(cpx<R> &a, cpx<R> &b) {
    cpx<R> t = a;
    a = t + b;
    b = t - b;
}

// radix 4 on (v0, v1, v2, v3) in natural order
template <typename R, int DIR>
__device__ __forceinline__ void dft4(cpx<R> &v0, cpx<R> &v1, cpx<R> &v2, cpx<R> &v3) {
    cpx<R> t0 = v0 + v2, t1 = v0 - v2, t2 = v1 + v3;
    cpx<R> t3 = mul_i(v1 - v3, R(DIR));  // (v1 - v3) * (DIR i)
    v0 = t0 + t2;
    v2 = t0 - t2;
    v1 = t1 + t3;
    v3 = t1 - t3;
}

template <typename R, int DIR>
__device__ __forceinline__ cpx<R> rot8(cpx<R> a, int k) {
    // a * exp(DIR 2 pi i k / 8), k = 1..3
    const R h = R(kc::R2);
    if (k == 1) return mk<R>((a.x - R(DIR) * a.y) * h, (a.y + R(DIR) * a.x) * h);
    if (k == 2) return mul_i(a, R(DIR));
    return mk<R>((-a.x - R(DIR) * a.y) * h, (-a.y + R(DIR) * a.x) * h);
}

template <typename R, int DIR>
__device__ __forceinline__ void dft8(cpx<R> *v) {
    // decimation in time: even / odd radix-4 halves
    cpx<R> e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
    cpx<R> o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
    dft4<R, DIR>(e0, e1, e2, e3);
    dft4<R, DIR>(o0, o1, o2, o3);
    o1 = rot8<R, DIR>(o1, 1);
    o2 = rot8<R, DIR>(o2, 2);
    o3 = rot8<R, DIR>(o3, 3);
    v[0] = e0 + o0; v[4] = e0 - o0;
    v[1] = e1 + o1; v[5] = e1 - o1;
    v[2] = e2 + o2; v[6] = e2 - o2;
    v[3] = e3 + o3; v[7] = e3 - o3;
}

template <typename R, int DIR>
__device__ __forceinline__ void dft16(cpx<R> *v) {
    cpx<R> e[8], o[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        e[i] = v[2 * i];
        o[i] = v[2 * i + 1];
    }
    dft8<R, DIR>(e);
    dft8<R, DIR>(o);
    // twiddles exp(DIR 2 pi i k / 16), k = 0..7
    const R c1 = R(kc::C16), s1 = R(kc::S16), h = R(kc::R2);
    const R cs[8] = {R(1), c1, h, s1, R(0), -s1, -h, -c1};
    const R sn[8] = {R(0), s1, h, c1, R(1), c1, h, s1};
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        cpx<R> w = mk<R>(cs[k], R(DIR) * sn[k]);
        cpx<R> t = (k == 0) ? o[k] : (k == 4) ? mul_i(o[k], R(DIR)) : cmul(o[k], w);
        v[k] = e[k] + t;
        v[k + 8] = e[k] - t;
    }
}

template <typename R, int DIR>
__device__ __forceinline__ void dft3(cpx<R> *v) {
    cpx<R> a = v[0], b = v[1], c = v[2];
    cpx<R> s = b + c, d = b - c;
    cpx<R> m = a + s * R(kc::C3);
    cpx<R> t = mul_i(d, R(DIR) * R(kc::S3));
    v[0] = a + s;
    v[1] = m + t;
    v[2] = m - t;
}

template <typename R, int DIR>
__device__ __forceinline__ void dft5(cpx<R> *v) {
    cpx<R> a = v[0];
    cpx<R> s1 = v[1] + v[4], d1 = v[1] - v[4];
    cpx<R> s2 = v[2] + v[3], d2 = v[2] - v[3];
    cpx<R> A1 = a + s1 * R(kc::C51) + s2 * R(kc::C52);
    cpx<R> A2 = a + s1 * R(kc::C52) + s2 * R(kc::C51);
    cpx<R> B1 = d1 * R(kc::S51) + d2 * R(kc::S52);
    cpx<R> B2 = d1 * R(kc::S52) - d2 * R(kc::S51);
    cpx<R> t1 = mul_i(B1, R(DIR)), t2 = mul_i(B2, R(DIR));
    v[0] = a + s1 + s2;
    v[1] = A1 + t1;
    v[4] = A1 - t1;
    v[2] = A2 + t2;
    v[3] = A2 - t2;
}

template <typename R, int DIR>
__device__ __forceinline__ void dft7(cpx<R> *v) {
    cpx<R> a = v[0];
    cpx<R> s1 = v[1] + v[6], d1 = v[1] - v[6];
    cpx<R> s2 = v[2] + v[5], d2 = v[2] - v[5];
    cpx<R> s3 = v[3] + v[4], d3 = v[3] - v[4];
    const R c1 = R(kc::C71), c2 = R(kc::C72), c3 = R(kc::C73);
    const R n1 = R(kc::S71), n2 = R(kc::S72), n3 = R(kc::S73);
    // X_k = a + sum_n cos(2 pi nk/7) s_n + DIR i sum_n sin(2 pi nk/7) d_n
    cpx<R> A1 = a + s1 * c1 + s2 * c2 + s3 * c3;
    cpx<R> A2 = a + s1 * c2 + s2 * c3 + s3 * c1;
    cpx<R> A3 = a + s1 * c3 + s2 * c1 + s3 * c2;
    cpx<R> B1 = d1 * n1 + d2 * n2 + d3 * n3;
    cpx<R> B2 = d1 * n2 - d2 * n3 - d3 * n1;
    cpx<R> B3 = d1 * n3 - d2 * n1 + d3 * n2;
    cpx<R> t1 = mul_i(B1, R(DIR)), t2 = mul_i(B2, R(DIR)), t3 = mul_i(B3, R(DIR));
    v[0] = a + s1 + s2 + s3;
    v[1] = A1 + t1; v[6] = A1 - t1;
    v[2] = A2 + t2; v[5] = A2 - t2;
    v[3] = A3 + t3; v[4] = A3 - t3;
}

template <typename R, int RAD, int DIR>
__device__ __forceinline__ void dft(cpx<R> *v) {
    if constexpr (RAD == 2) dft2<R, DIR>(v[0], v[1]);
    else if constexpr (RAD == 3) dft3<R, DIR>(v);
    else if constexpr (RAD == 4) dft4<R, DIR>(v[0], v[1], v[2], v[3]);
    else if constexpr (RAD == 5) dft5<R, DIR>(v);
    else if constexpr (RAD == 7) dft7<R, DIR>(v);
    else if constexpr (RAD == 8) dft8<R, DIR>(v);
    else if constexpr (RAD == 16) dft16<R, DIR>(v);
}

// --------------------------------------------------------------------------
// one Stockham stage over nlines lines (line stride ld) of length L
// --------------------------------------------------------------------------
// (not inlined: each radix gets its own register allocation)
template <typename R, int RAD, int DIR>
__device__ __noinline__ void fft_stage(cpx<R> *buf, int ld, int nlines, int L, int Ns,
                                       const cpx<R> *__restrict__ tw, int tid, int nthr) {
    constexpr int B = (fft_vpt<R>() + RAD - 1) / RAD;
    const int nb = L / RAD;
    const int total = nb * nlines;
    const int twstep = L / (Ns * RAD);
    cpx<R> v[B][RAD];
#pragma unroll
    for (int b = 0; b < B; ++b) {
        int q = tid + b * nthr;
        if (q < total) {
            int line = q / nb;
            int j = q - line * nb;
            const cpx<R> *src = buf + (size_t)line * ld + j;
#pragma unroll
            for (int r = 0; r < RAD; ++r) v[b][r] = src[r * nb];
        }
    }
    __syncthreads();
#pragma unroll
    for (int b = 0; b < B; ++b) {
        int q = tid + b * nthr;
        if (q < total) {
            int line = q / nb;
            int j = q - line * nb;
            int k = j % Ns;
            if (Ns > 1) {
#pragma unroll
                for (int r = 1; r < RAD; ++r) {
                    cpx<R> w = tw[r * k * twstep];
                    if (DIR > 0) w.y = -w.y;
                    v[b][r] = cmul(v[b][r], w);
                }
            }
            dft<R, RAD, DIR>(v[b]);
            cpx<R> *dst = buf + (size_t)line * ld + (j - k) * RAD + k;
#pragma unroll
            for (int r = 0; r < RAD; ++r) dst[r * Ns] = v[b][r];
        }
    }
    __syncthreads();
}

// Stockham transform of length d.L on lines already in shared memory.
// Requires nlines * d.L <= fft_vpt<R>() * nthr.
template <typename R, int DIR>
__device__ void fft_stockham(cpx<R> *buf, int ld, int nlines, const FftDev<R> &d,
                             int tid, int nthr) {
    int Ns = 1;
    for (int s = 0; s < d.nst; ++s) {
        const int rad = d.radix[s];
        switch (rad) {
            case 16: fft_stage<R, 16, DIR>(buf, ld, nlines, d.L, Ns, d.tw, tid, nthr); break;
            case 8: fft_stage<R, 8, DIR>(buf, ld, nlines, d.L, Ns, d.tw, tid, nthr); break;
            case 4: fft_stage<R, 4, DIR>(buf, ld, nlines, d.L, Ns, d.tw, tid, nthr); break;
            case 2: fft_stage<R, 2, DIR>(buf, ld, nlines, d.L, Ns, d.tw, tid, nthr); break;
            case 3: fft_stage<R, 3, DIR>(buf, ld, nlines, d.L, Ns, d.tw, tid, nthr); break;
            case 5: fft_stage<R, 5, DIR>(buf, ld, nlines, d.L, Ns, d.tw, tid, nthr); break;
            case 7: fft_stage<R, 7, DIR>(buf, ld, nlines, d.L, Ns, d.tw, tid, nthr); break;
            default: break;
        }
        Ns *= rad;
    }
}

// Full transform of length d.n on lines in shared memory (line stride
// ld >= d.L).  Input in [0, n), output in [0, n); with Bluestein the slots
// [n, L) are used as scratch.
template <typename R, int DIR>
__device__ void fft_line(cpx<R> *buf, int ld, int nlines, const FftDev<R> &d, int tid,
                         int nthr) {
    if (!d.bluestein) {
        fft_stockham<R, DIR>(buf, ld, nlines, d, tid, nthr);
        return;
    }
    const int n = d.n, L = d.L;
    // a[m] = x[m] * conj(b[m]) (forward) or x[m] * b[m] (inverse), zero padded
    for (int q = tid; q < nlines * L; q += nthr) {
        int line = q / L, m = q - line * L;
        cpx<R> *p = buf + (size_t)line * ld + m;
        if (m < n) {
            cpx<R> c = d.chirp[m];
            *p = (DIR < 0) ? cmulc(*p, c) : cmul(*p, c);
        } else {
            *p = mk<R>(R(0), R(0));
        }
    }
    __syncthreads();
    fft_stockham<R, -1>(buf, ld, nlines, d, tid, nthr);
    const cpx<R> *bh = (DIR < 0) ? d.bhat_f : d.bhat_i;
    for (int q = tid; q < nlines * L; q += nthr) {
        int line = q / L, m = q - line * L;
        cpx<R> *p = buf + (size_t)line * ld + m;
        *p = cmul(*p, bh[m]);
    }
    __syncthreads();
    fft_stockham<R, +1>(buf, ld, nlines, d, tid, nthr);
    const R inv = R(1) / R(L);
    for (int q = tid; q < nlines * n; q += nthr) {
        int line = q / n, m = q - line * n;
        cpx<R> *p = buf + (size_t)line * ld + m;
        cpx<R> c = d.chirp[m];
        cpx<R> v = (DIR < 0) ? cmulc(*p, c) : cmul(*p, c);
        *p = v * inv;
    }
    __syncthreads();
}

// --------------------------------------------------------------------------
// host side: tables for one transform length and precision
// --------------------------------------------------------------------------
bool is_smooth(int n);           // only factors 2, 3, 5, 7
int next_smooth(int n);          // smallest smooth m >= n
int next_smooth_even(int n);     // smallest even smooth m >= n
// FP64 mixed-radix DFT on the host (setup tables), sign -1 or +1, unnormalised
void host_fft(std::vector<std::complex<double>> &a, int sign);
std::vector<int> fft_radices(int L);

template <typename R>
struct FftTables {
    int n = 0;
    FftDev<R> dev{};
    DevBuf tw, chirp, bhat_f, bhat_i;
    int init(int n_);            // builds and uploads the tables
    size_t bytes() const { return tw.bytes + chirp.bytes + bhat_f.bytes + bhat_i.bytes; }
};

}  // namespace tc
