// tc_common.cuh -- shared types, complex arithmetic, status handling.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <cstdlib>
#include <chrono>
#include <cstring>
#include <map>
#include <mutex>
#include <new>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

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

// With TC_TRACE set in the environment, device allocations and frees that
// take longer than 20 ms are reported on stderr ("tc_trace cudaMalloc
// <bytes> <ms>"), to tell driver stalls apart from the phases' own work.
inline bool alloc_trace_on() {
    static const bool on = std::getenv("TC_TRACE") != nullptr;
    return on;
}
struct AllocTimer {
    const char *what;
    size_t n;
    std::chrono::steady_clock::time_point t0;
    AllocTimer(const char *w, size_t b) : what(w), n(b), t0(std::chrono::steady_clock::now()) {}
    ~AllocTimer() {
        const double ms =
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        if (ms > 20.0) std::fprintf(stderr, "tc_trace %s %zu %.3f\n", what, n, ms);
    }
};

// Device memory cache.  Blocks released by a DevBuf are kept per device and
// handed to later requests of about the same size (at most a quarter
// larger), so a process that builds and drops plans -- every
// cTomocam.mbir call builds two and drops them -- pays cudaMalloc and
// cudaFree once per size rather than once per call: on B200 these stalled
// the calling thread for 20-400 ms each for GB-sized blocks.  A block is
// cached only after its device has finished all work (the guarantee
// cudaFree gives); the cache holds at most half the device's memory,
// largest blocks evicted first; a failing cudaMalloc empties it and
// retries; tc_release_cached_memory() empties it on request; the
// environment variable TOMOCAM_B200_NO_CACHE=1 turns it off.
class DevCache {
  public:
    static DevCache &get() {
        static DevCache c;
        return c;
    }
    bool enabled() const { return enabled_; }
    // a cached block of n .. n + n / 4 bytes on the current device, or null
    void *take(size_t n, size_t *got) {
        if (!enabled_) return nullptr;
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        std::lock_guard<std::mutex> lk(mu_);
        auto it = free_.lower_bound(Key{dev, n});
        if (it == free_.end() || it->first.dev != dev || it->first.bytes > n + n / 4) return nullptr;
        void *p = it->second;
        *got = it->first.bytes;
        held_[dev] -= it->first.bytes;
        free_.erase(it);
        return p;
    }
    // keep (or free) a block of device dev once that device is idle
    void give(void *p, size_t bytes, int dev) {
        int cur = 0;
        if (!enabled_ || dev < 0 || cudaGetDevice(&cur) != cudaSuccess) {
            cudaGetLastError();
            free_now(p, bytes);
            return;
        }
        bool idle = (cur == dev || cudaSetDevice(dev) == cudaSuccess) &&
                    cudaDeviceSynchronize() == cudaSuccess;
        size_t cap = 0;
        if (idle) {
            std::lock_guard<std::mutex> lk(mu_);
            cap = limit(dev);  // device dev is current here
        }
        if (cur != dev) cudaSetDevice(cur);
        if (!idle) {
            cudaGetLastError();
            free_now(p, bytes);
            return;
        }
        std::vector<std::pair<void *, size_t>> out;
        {
            std::lock_guard<std::mutex> lk(mu_);
            if (bytes > cap) {
                out.push_back({p, bytes});
            } else {
                free_.insert({Key{dev, bytes}, p});
                held_[dev] += bytes;
                while (held_[dev] > cap) {  // evict the device's largest blocks
                    auto it = free_.lower_bound(Key{dev + 1, 0});
                    if (it == free_.begin()) break;
                    --it;
                    if (it->first.dev != dev) break;
                    out.push_back({it->second, it->first.bytes});
                    held_[dev] -= it->first.bytes;
                    free_.erase(it);
                }
            }
        }
        for (auto &b : out) free_now(b.first, b.second);
    }
    // free every cached block of the current device
    void flush() {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess) {
            cudaGetLastError();
            return;
        }
        std::vector<std::pair<void *, size_t>> out;
        {
            std::lock_guard<std::mutex> lk(mu_);
            for (auto it = free_.lower_bound(Key{dev, 0}); it != free_.end() && it->first.dev == dev;) {
                out.push_back({it->second, it->first.bytes});
                it = free_.erase(it);
            }
            held_[dev] = 0;
        }
        for (auto &b : out) free_now(b.first, b.second);
    }
    static void free_now(void *p, size_t bytes) {
        if (alloc_trace_on()) {
            AllocTimer at("cudaFree", bytes);
            cudaFree(p);
        } else {
            cudaFree(p);
        }
    }

  private:
    struct Key {
        int dev;
        size_t bytes;
        bool operator<(const Key &o) const { return dev != o.dev ? dev < o.dev : bytes < o.bytes; }
    };
    DevCache() {
        const char *v = std::getenv("TOMOCAM_B200_NO_CACHE");
        enabled_ = !(v && *v && std::strcmp(v, "0") != 0);
    }
    size_t limit(int dev) {
        auto it = cap_.find(dev);
        if (it != cap_.end()) return it->second;
        size_t fr = 0, tot = 0;
        if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) {
            cudaGetLastError();
            tot = 0;
        }
        return cap_[dev] = tot / 2;
    }
    bool enabled_ = true;
    std::mutex mu_;
    std::multimap<Key, void *> free_;
    std::map<int, size_t> held_, cap_;
};

struct DevBuf {
    void *ptr = nullptr;
    size_t bytes = 0;
    int dev = -1;  // the device the block belongs to
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (ptr) DevCache::get().give(ptr, bytes, dev);
        ptr = nullptr;
        bytes = 0;
        dev = -1;
    }
    // grows to at least n bytes; keeps the old allocation when it is big enough
    int reserve(size_t n) {
        if (n <= bytes) return TC_OK;
        release();
        if (n > alloc_fault_limit()) {
            set_error("device allocation of " + std::to_string(n) +
                      " bytes failed: " + cudaGetErrorString(cudaErrorMemoryAllocation));
            return TC_ERR_ALLOC;
        }
        if (cudaGetDevice(&dev) != cudaSuccess) {
            cudaGetLastError();
            dev = -1;
        }
        size_t got = 0;
        if (void *p = DevCache::get().take(n, &got)) {
            ptr = p;
            bytes = got;
            return TC_OK;
        }
        cudaError_t e;
        for (int attempt = 0; attempt < 2; ++attempt) {
            if (alloc_trace_on()) {
                AllocTimer at("cudaMalloc", n);
                e = cudaMalloc(&ptr, n);
            } else {
                e = cudaMalloc(&ptr, n);
            }
            if (e == cudaSuccess || attempt == 1 || !DevCache::get().enabled()) break;
            cudaGetLastError();
            DevCache::get().flush();  // out of memory: return the cached blocks and retry
        }
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
