// tc_common.cuh -- shared types, complex arithmetic, status handling.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <cstdlib>
#include <new>
#include <stdexcept>
#include <string>

#include "tomocam_b200.h"

namespace tc {

// ---------------------------------------------------------------------------
// complex numbers (interleaved re, im); R = float or double
// ---------------------------------------------------------------------------
template <typename R>
struct __align__(2 * sizeof(R)) cpx {
    R x, y;
};

using c32 = cpx<float>;
using c64 = cpx<double>;

template <typename R>
__host__ __device__ __forceinline__ cpx<R> mk(R a, R b) {
    cpx<R> c;
    c.x = a;
    c.y = b;
    return c;
}
template <typename R>
__host__ __device__ __forceinline__ cpx<R> operator+(cpx<R> a, cpx<R> b) {
    return mk<R>(a.x + b.x, a.y + b.y);
}
template <typename R>
__host__ __device__ __forceinline__ cpx<R> operator-(cpx<R> a, cpx<R> b) {
    return mk<R>(a.x - b.x, a.y - b.y);
}
template <typename R>
__host__ __device__ __forceinline__ cpx<R> operator*(cpx<R> a, R s) {
    return mk<R>(a.x * s, a.y * s);
}
template <typename R>
__host__ __device__ __forceinline__ cpx<R> cmul(cpx<R> a, cpx<R> b) {
    return mk<R>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
template <typename R>
__host__ __device__ __forceinline__ cpx<R> cmulc(cpx<R> a, cpx<R> b) {
    return mk<R>(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
template <typename R>
__host__ __device__ __forceinline__ cpx<R> conj(cpx<R> a) {
    return mk<R>(a.x, -a.y);
}
// multiply by s*i
template <typename R>
__host__ __device__ __forceinline__ cpx<R> mul_i(cpx<R> a, R s) {
    return mk<R>(-a.y * s, a.x * s);
}

// ---------------------------------------------------------------------------
// reductions
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// block-wide sum of NV doubles (blockDim.x a multiple of 32, 1-D blocks or
// linearised 2-D blocks via tid); result valid in thread 0
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], int tid, int nthr) {
    __shared__ double red[32][NV];
    const int lane = tid & 31, wid = tid >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = warp_sum(v[k]);
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) red[wid][k] = v[k];
    __syncthreads();
    if (wid == 0) {
        const int nw = (nthr + 31) >> 5;
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            double s = lane < nw ? red[lane][k] : 0.0;
            v[k] = warp_sum(s);
        }
    }
}

template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV]) {
    block_sum<NV>(v, threadIdx.x, blockDim.x);
}

// ---------------------------------------------------------------------------
// status / last error
// ---------------------------------------------------------------------------
void set_error(const std::string &msg);
const char *last_error();

struct Status {
    int code = TC_OK;
};

#define TC_FAIL(code, msg)                                                  \
    do {                                                                    \
        ::tc::set_error(msg);                                               \
        return (code);                                                      \
    } while (0)

#define TC_CUDA(expr)                                                       \
    do {                                                                    \
        cudaError_t _e = (expr);                                            \
        if (_e != cudaSuccess) {                                            \
            ::tc::set_error(std::string("CUDA error: ") +                   \
                            cudaGetErrorString(_e) + " at " + __FILE__ +    \
                            ":" + std::to_string(__LINE__) + " (" #expr ")"); \
            return TC_ERR_CUDA;                                             \
        }                                                                   \
    } while (0)

#define TC_TRY(expr)                                                        \
    do {                                                                    \
        int _s = (expr);                                                    \
        if (_s != TC_OK) return _s;                                         \
    } while (0)

#define TC_LAUNCH_CHECK() TC_CUDA(cudaGetLastError())

// Runs an entry point's body and turns any C++ exception into a status, so
// that nothing unwinds across the C ABI.
template <typename F>
inline int guarded(F &&f) {
    try {
        return f();
    } catch (const std::bad_alloc &) {
        set_error("host allocation failed");
        return TC_ERR_ALLOC;
    } catch (const std::exception &e) {
        set_error(std::string("internal error: ") + e.what());
        return TC_ERR_STATE;
    }
}

inline int ceil_div(int a, int b) { return (a + b - 1) / b; }
inline int64_t ceil_div64(int64_t a, int64_t b) { return (a + b - 1) / b; }

// ---------------------------------------------------------------------------
// device buffer owned by the library (RAII, never exits the process)
// ---------------------------------------------------------------------------
// Host-side fault injection for the allocation-failure path: when the
// environment variable TOMOCAM_B200_FAIL_ALLOC_ABOVE holds a byte count at
// process start, every library allocation larger than it fails as a
// cudaMalloc out of memory would (TC_ERR_ALLOC), without touching the GPU.
inline size_t alloc_fault_limit() {
    static const size_t lim = [] {
        const char *v = std::getenv("TOMOCAM_B200_FAIL_ALLOC_ABOVE");
        if (!v || !*v) return (size_t)-1;
        char *end = nullptr;
        unsigned long long b = std::strtoull(v, &end, 10);
        return (end && *end == '\0') ? (size_t)b : (size_t)-1;
    }();
    return lim;
}

struct DevBuf {
    void *ptr = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
    }
    // grows to at least n bytes; keeps the old allocation when it is big enough
    int reserve(size_t n) {
        if (n <= bytes) return TC_OK;
        release();
        cudaError_t e = n > alloc_fault_limit() ? cudaErrorMemoryAllocation : cudaMalloc(&ptr, n);
        if (e != cudaSuccess) {
            ptr = nullptr;
            cudaGetLastError();
            set_error("device allocation of " + std::to_string(n) +
                      " bytes failed: " + cudaGetErrorString(e));
            return TC_ERR_ALLOC;
        }
        bytes = n;
        return TC_OK;
    }
    template <typename T>
    T *as() const {
        return static_cast<T *>(ptr);
    }
};

}  // namespace tc
