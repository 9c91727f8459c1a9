// tc_prep.cuh -- pre/post-processing and reductions (internal).
#pragma once

#include "tc_common.cuh"

namespace tc {

// npad and roll offset of src/preproc.cpp:79-85
void preproc_params(int ncols, float center, int &npad, int &off);
int preproc_dev(const float *sino, float *out, int S, int P, int D, int npad, int off,
                cudaStream_t st);
int pad2d_dev(const float *in, float *out, int S, int R, int C, int npad, cudaStream_t st);
int crop2d_dev(const float *in, float *out, int S, int R, int C, int npixels, cudaStream_t st);
int scale_dev(float *x, size_t n, float divisor, cudaStream_t st);
int axpby_dev(float a, const float *x, float b, float *y, size_t n, cudaStream_t st);
int fill_dev(float *x, size_t n, float v, cudaStream_t st);
int max_sumsq_dev(const float *x, size_t n, float *maxv, double *sumsq, cudaStream_t st);

}  // namespace tc
