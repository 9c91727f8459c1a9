// ref_gpu_shim.cu -- TEST INFRASTRUCTURE ONLY.
//
// C entry points onto the reference's own GPU build (lbl-camera/tomocam
// src/*.cpp, src/gpu/*.cu, compiled from the read-only tree by
// oracle/Makefile into oracle/_ref/libref_gpu.so, with cuFINUFFT replaced by
// the exact-NUDFT stand-in of oracle/refgpu/nudft_standin.cu).  They expose
// pieces of the reference path that its Python module (src/pyTomocam.cpp,
// built beside it as oracle/_ref/cTomocam*.so) does not:
//
// * host-array pre/post-processing: preproc (src/preproc.cpp:74-102),
//   postproc (src/postproc.cpp:70-97), pad2d (src/padding.cpp), and the
//   device kernels under them (gpu::roll, src/gpu/fftshift.cu:30-50;
//   gpu::pad1d, src/gpu/padding.cu:34-62);
// * the point-spread function and its Toeplitz convolution
//   (PointSpreadFunction, src/toeplitz.h:51-159), on device arrays, the
//   per-chunk work of gradient2_ (src/gradient2.cpp:62);
// * the qGGMRF kernel on device arrays (gpu::add_total_var2,
//   src/gpu/cuTV2.cu:78-93);
// * the reference's host-array iteration: gradient2 + add_total_var2 for the
//   gradient and sqrt(function_value2) for the objective, driven by
//   Optimizer::run2, as src/mbir2.cpp:114-141 wires them.
//
// Everything runs the reference's code unchanged; this file only moves data
// in and out.  The checker uses it to pin the product and to time the
// reference's GPU path on the same device.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "dev_array.h"
#include "dist_array.h"
#include "machine.h"
#include "optimize.h"
#include "toeplitz.h"
#include "tomocam.h"
#include "gpu/fftshift.cuh"
#include "gpu/padding.cuh"
#include "gpu/totalvar.cuh"

using tomocam::DArray;
using tomocam::DeviceArray;
using tomocam::dim3_t;

namespace {

// A DeviceArray over memory the caller owns (never freed here).
template <typename T>
struct DevView : DeviceArray<T> {
    DevView(dim3_t d, T *p) {
        this->dims_ = d;
        this->size_ = (size_t)d.x * d.y * d.z;
        this->halo_ = {0, 0};
        this->dev_ptr_ = p;
    }
    ~DevView() { this->dev_ptr_ = nullptr; }
};

DArray<float> to_darray(const float *h, int S, int R, int C) {
    DArray<float> a(dim3_t(S, R, C));
    std::memcpy(&a[0], h, sizeof(float) * (size_t)S * R * C);
    return a;
}

int from_darray(const DArray<float> &a, float *out, long cap, int *rows, int *cols) {
    dim3_t d = a.dims();
    const long n = (long)d.x * d.y * d.z;
    if (rows) *rows = d.y;
    if (cols) *cols = d.z;
    if (n > cap) return -2;
    std::memcpy(out, &const_cast<DArray<float> &>(a)[0], sizeof(float) * n);
    return 0;
}

struct PsfHandle {
    int n = 0, nproj = 0, batch = 0;
    std::vector<tomocam::NUFFT::Grid<float>> grids;
    std::vector<tomocam::PointSpreadFunction<float>> psfs;
};

} // namespace

extern "C" {

int ref_num_gpus(void) { return tomocam::Machine::config.num_of_gpus(); }

// preproc: detector padding and centring (src/preproc.cpp:74-102).
int ref_preproc(const float *sino, int S, int P, int D, float center, float *out, long cap,
                int *out_cols) {
    auto a = to_darray(sino, S, P, D);
    auto b = tomocam::preproc(a, center);
    return from_darray(b, out, cap, nullptr, out_cols);
}

// postproc: crop of an [S][n][n] image to npixels (src/postproc.cpp:70-97).
int ref_postproc(const float *x, int S, int n, int npixels, float *out, long cap, int *out_n) {
    auto a = to_darray(x, S, n, n);
    auto b = tomocam::postproc(a, npixels);
    return from_darray(b, out, cap, nullptr, out_n);
}

// pad2d on a host array (src/padding.cpp), type 0 = SYMMETRIC, 1 = LEFT, 2 = RIGHT.
int ref_pad2d(const float *x, int S, int n, int npad, int type, float *out, long cap, int *out_n) {
    tomocam::PadType t = type == 1 ? tomocam::PadType::LEFT
                         : type == 2 ? tomocam::PadType::RIGHT : tomocam::PadType::SYMMETRIC;
    auto a = to_darray(x, S, n, n);
    auto b = tomocam::pad2d(a, npad, t);
    return from_darray(b, out, cap, nullptr, out_n);
}

// gpu::roll along the last axis, host arrays in and out.
int ref_roll(const float *in, float *out, int S, int R, int C, int delta) {
    const size_t bytes = sizeof(float) * (size_t)S * R * C;
    DeviceArray<float> d(dim3_t(S, R, C));
    SAFE_CALL(cudaMemcpy(d.dev_ptr(), in, bytes, cudaMemcpyHostToDevice));
    auto r = tomocam::gpu::roll(d, delta);
    SAFE_CALL(cudaMemcpy(out, r.dev_ptr(), bytes, cudaMemcpyDeviceToHost));
    return 0;
}

// gpu::pad1d along the last axis (type as ref_pad2d); out is [S][R][C+|padding|].
int ref_pad1d(const float *in, float *out, int S, int R, int C, int padding, int type) {
    tomocam::PadType t = type == 1 ? tomocam::PadType::LEFT
                         : type == 2 ? tomocam::PadType::RIGHT : tomocam::PadType::SYMMETRIC;
    DeviceArray<float> d(dim3_t(S, R, C));
    SAFE_CALL(cudaMemcpy(d.dev_ptr(), in, sizeof(float) * (size_t)S * R * C,
                         cudaMemcpyHostToDevice));
    auto r = tomocam::gpu::pad1d(d, padding, t);
    SAFE_CALL(cudaMemcpy(out, r.dev_ptr(), r.bytes(), cudaMemcpyDeviceToHost));
    return 0;
}

// g[S][R][C] += qGGMRF gradient of x (device pointers; the reference kernel,
// clamped borders, no beta).  Synchronises before returning.
int ref_qggmrf_dev(const float *x, float *g, int S, int R, int C, float sigma, float p) {
    DevView<float> dx(dim3_t(S, R, C), const_cast<float *>(x));
    DevView<float> dg(dim3_t(S, R, C), g);
    tomocam::gpu::add_total_var2<float>(dx, dg, sigma, p);
    SAFE_CALL(cudaStreamSynchronize(cudaStreamPerThread));
    return 0;
}

// The reference's PointSpreadFunction for an n-pixel image and nproj angles,
// built by its own constructor (src/toeplitz.h:51-73): the type-1 NUFFT of
// ones is evaluated by the stand-in (exact) unless an output of that size was
// staged first.  Plans for `batch`-slice chunks are created as mbir2 does.
int ref_psf_create(const float *angles, int nproj, int n, int batch, void **handle) {
    if (!angles || nproj < 1 || n < 2 || batch < 1 || !handle) return -1;
    auto *h = new PsfHandle;
    h->n = n;
    h->nproj = nproj;
    h->batch = batch;
    int dev = 0;
    SAFE_CALL(cudaGetDevice(&dev));
    h->grids.resize(1);
    h->grids[0] = tomocam::NUFFT::Grid<float>(nproj, n, angles, dev);
    h->psfs.resize(1);
    h->psfs[0] = tomocam::PointSpreadFunction<float>(h->grids[0]);
    h->psfs[0].create_plans(batch);
    *handle = h;
    return 0;
}

void ref_psf_destroy(void *handle) { delete static_cast<PsfHandle *>(handle); }

// g = H x - aty for S slices of device arrays, chunk by chunk as gradient2_
// does on the device (src/gradient2.cpp:62), each chunk `batch` slices
// (the last one may be shorter, which the reference serves by convolve1).
int ref_psf_grad_dev(void *handle, const float *x, const float *aty, float *g, int S) {
    auto *h = static_cast<PsfHandle *>(handle);
    const int n = h->n;
    const size_t plane = (size_t)n * n;
    for (int s0 = 0; s0 < S; s0 += h->batch) {
        const int b = S - s0 < h->batch ? S - s0 : h->batch;
        DevView<float> dx(dim3_t(b, n, n), const_cast<float *>(x) + s0 * plane);
        DevView<float> da(dim3_t(b, n, n), const_cast<float *>(aty) + s0 * plane);
        auto dg = h->psfs[0].convolve(dx) - da;
        SAFE_CALL(cudaMemcpyAsync(g + s0 * plane, dg.dev_ptr(), sizeof(float) * b * plane,
                                  cudaMemcpyDeviceToDevice, cudaStreamPerThread));
    }
    SAFE_CALL(cudaStreamSynchronize(cudaStreamPerThread));
    return 0;
}

// Host-array forms, as mbir2 calls them (src/gradient2.cpp:72-100,
// src/error2.cpp:70-94, src/tv_update.cpp:75-107).
int ref_gradient2_host(void *handle, const float *x, const float *aty, float *g, int S) {
    auto *h = static_cast<PsfHandle *>(handle);
    auto dx = to_darray(x, S, h->n, h->n);
    auto da = to_darray(aty, S, h->n, h->n);
    auto dg = tomocam::gradient2(dx, da, h->psfs);
    return from_darray(dg, g, (long)S * h->n * h->n, nullptr, nullptr);
}

double ref_function_value2_host(void *handle, const float *x, const float *aty, int S,
                                float sino_sq) {
    auto *h = static_cast<PsfHandle *>(handle);
    auto dx = to_darray(x, S, h->n, h->n);
    auto da = to_darray(aty, S, h->n, h->n);
    return (double)tomocam::function_value2(dx, da, h->psfs, sino_sq);
}

int ref_add_total_var2_host(const float *x, float *g, int S, int n, float sigma, float p) {
    auto dx = to_darray(x, S, n, n);
    auto dg = to_darray(g, S, n, n);
    tomocam::add_total_var2(dx, dg, sigma, p);
    return from_darray(dg, g, (long)S * n * n, nullptr, nullptr);
}

// The reference's iteration on host arrays: Optimizer::run2 over
// gradient2 + add_total_var2 and sqrt(function_value2) (src/mbir2.cpp:114-141),
// from the guess x (in: [S][n][n], out: result).
int ref_run2_host(void *handle, float *x, const float *aty, int S, float sino_sq, float sigma,
                  float p, int num_iters, float step_size) {
    auto *h = static_cast<PsfHandle *>(handle);
    auto sinoT = to_darray(aty, S, h->n, h->n);
    auto x0 = to_darray(x, S, h->n, h->n);
    auto &psfs = h->psfs;
    auto calc_gradient = [&sinoT, &psfs, sigma, p](DArray<float> &v) -> DArray<float> {
        auto g = tomocam::gradient2(v, sinoT, psfs);
        tomocam::add_total_var2(v, g, sigma, p);
        return g;
    };
    auto calc_error = [&sinoT, &psfs, sino_sq](DArray<float> &v) -> float {
        auto e = tomocam::function_value2(v, sinoT, psfs, sino_sq);
        return std::sqrt(e);
    };
    tomocam::Optimizer<float, DArray, decltype(calc_gradient), decltype(calc_error)> opt(
        calc_gradient, calc_error);
    auto rec = opt.run2(x0, num_iters, step_size, 0.f, 0.f);
    return from_darray(rec, x, (long)S * h->n * h->n, nullptr, nullptr);
}

} // extern "C"
