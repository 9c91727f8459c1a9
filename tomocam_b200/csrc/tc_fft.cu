// tc_fft.cu -- host tables for the FFT engine and the batched line-FFT entry.
#include <cmath>
#include <complex>
#include <vector>

#include "tc_fft.cuh"

namespace tc {

bool is_smooth(int n) {
    if (n < 1) return false;
    for (int p : {2, 3, 5, 7})
        while (n % p == 0) n /= p;
    return n == 1;
}

int next_smooth(int n) {
    int m = n < 1 ? 1 : n;
    while (!is_smooth(m)) ++m;
    return m;
}

int next_smooth_even(int n) {
    int m = next_smooth(n);
    while (m & 1) m = next_smooth(m + 1);
    return m;
}

std::vector<int> fft_radices(int L) {
    std::vector<int> r;
    int e2 = 0;
    while (L % 2 == 0) {
        L /= 2;
        ++e2;
    }
    int k16 = e2 / 4, rem = e2 % 4;
    if (rem == 1 && k16 > 0) {
        for (int i = 0; i < k16 - 1; ++i) r.push_back(16);
        r.push_back(8);
        r.push_back(4);
    } else {
        for (int i = 0; i < k16; ++i) r.push_back(16);
        if (rem == 1) r.push_back(2);
        if (rem == 2) r.push_back(4);
        if (rem == 3) r.push_back(8);
    }
    for (int p : {3, 5, 7})
        while (L % p == 0) {
            r.push_back(p);
            L /= p;
        }
    return r;
}

// FP64 mixed-radix FFT on the host (setup only: Bluestein chirp spectra).
void host_fft(std::vector<std::complex<double>> &a, int sign) {
    const int n = (int)a.size();
    if (n <= 1) return;
    int p = 2;
    while (n % p) ++p;
    const int m = n / p;
    std::vector<std::vector<std::complex<double>>> sub(p, std::vector<std::complex<double>>(m));
    for (int k = 0; k < m; ++k)
        for (int r = 0; r < p; ++r) sub[r][k] = a[k * p + r];
    for (int r = 0; r < p; ++r) host_fft(sub[r], sign);
    for (int k = 0; k < n; ++k) {
        std::complex<double> s = 0;
        for (int r = 0; r < p; ++r) {
            long long e = (long long)r * k % n;
            double ang = sign * 2.0 * M_PI * (double)e / n;
            s += sub[r][k % m] * std::complex<double>(std::cos(ang), std::sin(ang));
        }
        a[k] = s;
    }
}

template <typename R>
static int upload(DevBuf &buf, const std::vector<std::complex<double>> &v) {
    std::vector<cpx<R>> h(v.size());
    for (size_t i = 0; i < v.size(); ++i) h[i] = mk<R>((R)v[i].real(), (R)v[i].imag());
    TC_TRY(buf.reserve(h.size() * sizeof(cpx<R>)));
    TC_CUDA(cudaMemcpy(buf.ptr, h.data(), h.size() * sizeof(cpx<R>), cudaMemcpyHostToDevice));
    return TC_OK;
}

template <typename R>
int FftTables<R>::init(int n_) {
    if (n_ < 1) TC_FAIL(TC_ERR_SHAPE, "FFT length must be >= 1");
    n = n_;
    FftDev<R> d{};
    d.n = n;
    d.bluestein = is_smooth(n) ? 0 : 1;
    d.L = d.bluestein ? next_smooth(2 * n - 1) : n;
    auto rad = fft_radices(d.L);
    if ((int)rad.size() > FFT_MAX_STAGES) TC_FAIL(TC_ERR_SHAPE, "FFT length has too many factors");
    d.nst = (int)rad.size();
    for (int i = 0; i < d.nst; ++i) d.radix[i] = rad[i];
    const int L = d.L;
    std::vector<std::complex<double>> tab(L);
    for (int k = 0; k < L; ++k) {
        double ang = -2.0 * M_PI * (double)k / (double)L;
        tab[k] = std::complex<double>(std::cos(ang), std::sin(ang));
    }
    TC_TRY(upload<R>(tw, tab));
    d.tw = tw.as<cpx<R>>();
    if (d.bluestein) {
        std::vector<std::complex<double>> b(n), bc(L, 0.0), bci(L, 0.0);
        for (int m = 0; m < n; ++m) {
            long long e = (long long)m * m % (2LL * n);
            double ang = M_PI * (double)e / (double)n;
            b[m] = std::complex<double>(std::cos(ang), std::sin(ang));
        }
        for (int m = 0; m < n; ++m) {
            bc[m] = b[m];
            bci[m] = std::conj(b[m]);
            if (m > 0) {
                bc[L - m] = b[m];
                bci[L - m] = std::conj(b[m]);
            }
        }
        host_fft(bc, -1);
        host_fft(bci, -1);
        TC_TRY(upload<R>(chirp, b));
        TC_TRY(upload<R>(bhat_f, bc));
        TC_TRY(upload<R>(bhat_i, bci));
        d.chirp = chirp.as<cpx<R>>();
        d.bhat_f = bhat_f.as<cpx<R>>();
        d.bhat_i = bhat_i.as<cpx<R>>();
    }
    dev = d;
    return TC_OK;
}

template struct FftTables<float>;
template struct FftTables<double>;

// ---------------------------------------------------------------------------
// batched contiguous-line FFT
// ---------------------------------------------------------------------------
template <typename R, int DIR>
__global__ void __launch_bounds__(FFT_MAX_THREADS, 1)
k_fft_lines(const cpx<R> *in, cpx<R> *out, int nbatch, int lines_per_cta, FftDev<R> d) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cpx<R> *buf = reinterpret_cast<cpx<R> *>(smem_raw);
    const int n = d.n, ld = d.L;
    const int first = blockIdx.x * lines_per_cta;
    const int nl = min(lines_per_cta, nbatch - first);
    if (nl <= 0) return;
    for (int q = threadIdx.x; q < nl * n; q += blockDim.x) {
        int l = q / n, m = q - l * n;
        buf[(size_t)l * ld + m] = in[(size_t)(first + l) * n + m];
    }
    __syncthreads();
    fft_line<R, DIR>(buf, ld, nl, d, threadIdx.x, blockDim.x);
    for (int q = threadIdx.x; q < nl * n; q += blockDim.x) {
        int l = q / n, m = q - l * n;
        out[(size_t)(first + l) * n + m] = buf[(size_t)l * ld + m];
    }
}

template <typename R>
int fft_lines_launch(const FftTables<R> &T, const cpx<R> *in, cpx<R> *out, int nbatch,
                     int dir, cudaStream_t st) {
    const int L = T.dev.L;
    int lines = 1;
    while (lines * 2 * L <= 4096 && lines * 2 <= nbatch) lines *= 2;
    const int nthr = fft_threads<R>(L, lines);
    if (nthr > FFT_MAX_THREADS) TC_FAIL(TC_ERR_SHAPE, "FFT length too large for one CTA");
    const size_t smem = (size_t)lines * L * sizeof(cpx<R>);
    if (smem > 227 * 1024) TC_FAIL(TC_ERR_SHAPE, "FFT length too large for shared memory");
    const int grid = ceil_div(nbatch, lines);
    if (dir < 0) {
        auto k = k_fft_lines<R, -1>;
        TC_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k<<<grid, nthr, smem, st>>>(in, out, nbatch, lines, T.dev);
    } else {
        auto k = k_fft_lines<R, +1>;
        TC_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k<<<grid, nthr, smem, st>>>(in, out, nbatch, lines, T.dev);
    }
    TC_LAUNCH_CHECK();
    return TC_OK;
}

template int fft_lines_launch<float>(const FftTables<float> &, const c32 *, c32 *, int, int, cudaStream_t);
template int fft_lines_launch<double>(const FftTables<double> &, const c64 *, c64 *, int, int, cudaStream_t);

}  // namespace tc
