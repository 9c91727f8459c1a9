/*
 * oracle_core.c -- TEST INFRASTRUCTURE ONLY.
 *
 * FP64 CPU kernels used by the oracle (oracle/oracle.py) to check the CUDA
 * implementation in tomocam_b200/.  Nothing in the product links or calls
 * this file; only tests/, the smoke check and bench.py's CPU-baseline leg do.
 *
 *  - orc_es_spread / orc_es_interp: exponential-of-semicircle (ES) kernel
 *    spreading and interpolation on a periodic fine grid, the published
 *    FINUFFT method (Barnett, Magland & af Klinteberg, SIAM J. Sci. Comput.
 *    41(5), 2019).  The reference reaches the same transforms through
 *    cuFINUFFT (src/nufft.h:230-384); this is a restatement of the method,
 *    not of cuFINUFFT's code.
 *  - orc_qggmrf: the 26-neighbour qGGMRF prior gradient with clamp-to-edge
 *    boundaries, following src/gpu/cuTV2.cu:33-76,
 *    src/gpu/potential_function.cuh:31-108 and test/tvd.cpp:23-75.
 *
 * Complex arrays are interleaved (re, im) doubles.  Fine grids are row-major
 * [nf][nf] with the x coordinate on the fast (column) axis.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static inline double es_kernel(double z, double beta) {
    /* phi(z) = exp(beta (sqrt(1 - z^2) - 1)), |z| < 1 */
    double q = 1.0 - z * z;
    if (q <= 0.0) return 0.0;
    return exp(beta * (sqrt(q) - 1.0));
}

/* tap weights for one coordinate: taps l0 .. l0+w-1 at grid spacing h */
static inline int es_taps(double x, double h, int w, double beta, double *wt) {
    double xi = x / h;
    int l0 = (int)ceil(xi - 0.5 * w);
    double half = 0.5 * w;
    for (int t = 0; t < w; ++t) {
        double z = ((double)(l0 + t) - xi) / half;
        wt[t] = es_kernel(z, beta);
    }
    return l0;
}

static inline int wrap(int l, int n) {
    int r = l % n;
    return r < 0 ? r + n : r;
}

/*
 * a[l] += sum_j c_j psi(l h - w_j) over a periodic nf x nf grid (type-1
 * spreading).  Threads own bands of grid rows, so the sum is race-free and
 * deterministic.  nbatch transforms share the points: c is [nbatch][npts],
 * grid is [nbatch][nf][nf].
 */
void orc_es_spread(int64_t npts, const double *x, const double *y,
                   const double *c, int nbatch, int nf, int w, double beta,
                   double *grid) {
    const double h = 2.0 * M_PI / nf;
    memset(grid, 0, sizeof(double) * 2 * (size_t)nbatch * nf * nf);
#pragma omp parallel
    {
        int nth = 1, tid = 0;
#ifdef _OPENMP
        nth = omp_get_num_threads();
        tid = omp_get_thread_num();
#endif
        int r0 = (int)((int64_t)nf * tid / nth);
        int r1 = (int)((int64_t)nf * (tid + 1) / nth);
        double wx[64], wy[64];
        for (int64_t j = 0; j < npts; ++j) {
            int ly0 = es_taps(y[j], h, w, beta, wy);
            /* does any wrapped row of this point fall in [r0, r1)? */
            int any = 0;
            for (int t = 0; t < w && !any; ++t) {
                int r = wrap(ly0 + t, nf);
                any = (r >= r0 && r < r1);
            }
            if (!any) continue;
            int lx0 = es_taps(x[j], h, w, beta, wx);
            for (int t = 0; t < w; ++t) {
                int r = wrap(ly0 + t, nf);
                if (r < r0 || r >= r1) continue;
                for (int b = 0; b < nbatch; ++b) {
                    double cre = c[2 * ((size_t)b * npts + j)] * wy[t];
                    double cim = c[2 * ((size_t)b * npts + j) + 1] * wy[t];
                    double *row = grid + 2 * ((size_t)b * nf * nf + (size_t)r * nf);
                    for (int u = 0; u < w; ++u) {
                        int cidx = wrap(lx0 + u, nf);
                        row[2 * cidx] += cre * wx[u];
                        row[2 * cidx + 1] += cim * wx[u];
                    }
                }
            }
        }
    }
}

/* c_j = sum_l psi(w_j - l h) b[l] (type-2 interpolation), c is [nbatch][npts] */
void orc_es_interp(int64_t npts, const double *x, const double *y,
                   const double *grid, int nbatch, int nf, int w, double beta,
                   double *c) {
    const double h = 2.0 * M_PI / nf;
#pragma omp parallel for schedule(static)
    for (int64_t j = 0; j < npts; ++j) {
        double wx[64], wy[64];
        int ly0 = es_taps(y[j], h, w, beta, wy);
        int lx0 = es_taps(x[j], h, w, beta, wx);
        for (int b = 0; b < nbatch; ++b) {
            double sre = 0.0, sim = 0.0;
            for (int t = 0; t < w; ++t) {
                int r = wrap(ly0 + t, nf);
                const double *row = grid + 2 * ((size_t)b * nf * nf + (size_t)r * nf);
                double are = 0.0, aim = 0.0;
                for (int u = 0; u < w; ++u) {
                    int cidx = wrap(lx0 + u, nf);
                    are += row[2 * cidx] * wx[u];
                    aim += row[2 * cidx + 1] * wx[u];
                }
                sre += are * wy[t];
                sim += aim * wy[t];
            }
            c[2 * ((size_t)b * npts + j)] = sre;
            c[2 * ((size_t)b * npts + j) + 1] = sim;
        }
    }
}

/*
 * Derivative of the qGGMRF potential, src/gpu/potential_function.cuh:90-108
 * (q = 2, c = MRF_C), evaluated in double precision.
 */
static inline double d_pot(double delta, double p, double sigma, double mrf_c) {
    const double q = 2.0;
    if (delta == 0.0) return 0.0;
    double ad = fabs(delta);
    double sq = pow(sigma, q);
    double sqp = pow(sigma, q - p);
    double t1 = pow(ad, q - p) / sqp;
    double t2 = pow(ad, q - 1.0);
    double t3 = mrf_c + t1;
    double v = (t2 / (t3 * sq)) * (q - ((q - p) * t1) / t3);
    return delta < 0.0 ? -v : v;
}

static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

/*
 * g[v] += scale * sum_{26 n} w_n rho'(x_v - x_clamp(n)), clamp-to-edge in all
 * three axes (src/gpu/cuTV2.cu:33-76 with src/gpu/dev_memory.cuh:88-94).
 * weights: 27 values, [dz][dy][dx], centre weight 0.
 */
void orc_qggmrf(int S, int R, int C, const double *x, double *g, double sigma,
                double p, double mrf_c, const double *weights, double scale) {
#pragma omp parallel for collapse(2) schedule(static)
    for (int s = 0; s < S; ++s) {
        for (int r = 0; r < R; ++r) {
            for (int c = 0; c < C; ++c) {
                size_t v = ((size_t)s * R + r) * C + c;
                double u = x[v];
                double acc = 0.0;
                for (int dz = 0; dz < 3; ++dz) {
                    int s1 = clampi(s + dz - 1, 0, S - 1);
                    for (int dy = 0; dy < 3; ++dy) {
                        int r1 = clampi(r + dy - 1, 0, R - 1);
                        for (int dx = 0; dx < 3; ++dx) {
                            int c1 = clampi(c + dx - 1, 0, C - 1);
                            double d = u - x[((size_t)s1 * R + r1) * C + c1];
                            acc += weights[(dz * 3 + dy) * 3 + dx] * d_pot(d, p, sigma, mrf_c);
                        }
                    }
                }
                g[v] += scale * acc;
            }
        }
    }
}
