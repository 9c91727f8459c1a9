// cufinufft.h -- TEST INFRASTRUCTURE ONLY: a stand-in for the cuFINUFFT
// header, so that the reference's own GPU sources (src/nufft.h and everything
// that includes it) compile against oracle/refgpu/nudft_standin.cu instead of
// the cuFINUFFT library, which is absent from this image.
//
// Only the entry points the reference calls are declared (src/nufft.h:196-384:
// default options, make plan, set points, execute, destroy; single and double
// precision), with the argument meaning of the cuFINUFFT 2.x C API that those
// call sites use (modes as int64, points as device arrays, iflag sign,
// ntransf stacked transforms).  The reference pins no cuFINUFFT version
// (cmake/Findfinufft.cmake accepts any installed one).
//
// The stand-in evaluates the transforms' definition exactly (direct
// non-uniform DFT, FP64 accumulation) rather than cuFINUFFT's ES-kernel
// approximation at tolerance `eps`, so it is slow and meant for small images,
// plus a staging hook for large-size timing runs (nudft_standin.cu).
#ifndef TC_REF_CUFINUFFT_STANDIN_H
#define TC_REF_CUFINUFFT_STANDIN_H

#include <cstdint>
#include <cuComplex.h>

typedef struct cufinufft_opts {
    int gpu_device_id;
    int modeord;       // 0: modes -n/2 .. (n-1)/2 in increasing order (the only order served)
    int gpu_method;    // accepted, ignored
    int gpu_sort;      // accepted, ignored
} cufinufft_opts;

// distinct plan types for the two precisions, as the reference overloads on them
struct tc_standin_planf;
struct tc_standin_pland;
typedef tc_standin_planf *cufinufftf_plan;
typedef tc_standin_pland *cufinufft_plan;

extern "C" {
void cufinufft_default_opts(cufinufft_opts *opts);

int cufinufftf_makeplan(int type, int dim, const int64_t *n_modes, int iflag, int ntransf,
                        float eps, cufinufftf_plan *plan, cufinufft_opts *opts);
int cufinufftf_setpts(cufinufftf_plan plan, int64_t M, float *x, float *y, float *z, int N,
                      float *s, float *t, float *u);
int cufinufftf_execute(cufinufftf_plan plan, cuFloatComplex *c, cuFloatComplex *fk);
int cufinufftf_destroy(cufinufftf_plan plan);

int cufinufft_makeplan(int type, int dim, const int64_t *n_modes, int iflag, int ntransf,
                       double eps, cufinufft_plan *plan, cufinufft_opts *opts);
int cufinufft_setpts(cufinufft_plan plan, int64_t M, double *x, double *y, double *z, int N,
                     double *s, double *t, double *u);
int cufinufft_execute(cufinufft_plan plan, cuDoubleComplex *c, cuDoubleComplex *fk);
int cufinufft_destroy(cufinufft_plan plan);
}

#endif
