// tc_hostio.cu -- host <-> device copies of the host entry points.
//
// Pinned (page-locked or registered) host buffers are copied directly.
// Pageable buffers (e.g. numpy arrays) go through two pinned staging buffers:
// the DMA of one chunk overlaps the host-side copy of the other, and each
// host-side copy is split over threads (a single thread copying into freshly
// allocated pageable memory is bound by page faults and memcpy bandwidth,
// far below PCIe/C2C rates).
#include <algorithm>
#include <cstring>
#include <mutex>
#include <thread>
#include <vector>

#include <unistd.h>

#include "tc_plan.cuh"

namespace tc {

namespace {

constexpr size_t STAGE_BYTES = size_t(64) << 20;

struct Staging {
    std::mutex mu;
    void *buf[2] = {nullptr, nullptr};
    cudaStream_t st = nullptr;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    int device = -1;
};

// one ring for the process (128 MiB pinned, allocated on first use)
Staging &staging() {
    static Staging s;
    return s;
}

int staging_init(Staging &s) {
    int dev = 0;
    TC_CUDA(cudaGetDevice(&dev));
    if (s.buf[0] && s.device == dev) return TC_OK;
    if (s.buf[0]) {  // a different device: events and stream belong to the old one
        cudaStreamDestroy(s.st);
        for (int i = 0; i < 2; ++i) {
            cudaEventDestroy(s.ev[i]);
            cudaFreeHost(s.buf[i]);
            s.buf[i] = nullptr;
        }
    }
    for (int i = 0; i < 2; ++i) {
        if (cudaMallocHost(&s.buf[i], STAGE_BYTES) != cudaSuccess) {
            cudaGetLastError();
            s.buf[i] = nullptr;
            TC_FAIL(TC_ERR_ALLOC, "pinned staging allocation failed");
        }
        TC_CUDA(cudaEventCreateWithFlags(&s.ev[i], cudaEventDisableTiming));
    }
    TC_CUDA(cudaStreamCreateWithFlags(&s.st, cudaStreamNonBlocking));
    s.device = dev;
    return TC_OK;
}

bool is_pinned(const void *p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

// memcpy split over up to 16 threads
void par_copy(void *dst, const void *src, size_t n) {
    const unsigned hc = std::max(1u, std::thread::hardware_concurrency());
    const size_t T = std::min<size_t>(16, hc);
    if (n < (size_t(4) << 20) || T == 1) {
        std::memcpy(dst, src, n);
        return;
    }
    const size_t per = ((n + T - 1) / T + 63) & ~size_t(63);
    std::vector<std::thread> th;
    for (size_t k = 1; k < T && k * per < n; ++k) {
        const size_t o = k * per, len = std::min(per, n - o);
        th.emplace_back([=]() {
            std::memcpy(static_cast<char *>(dst) + o, static_cast<const char *>(src) + o, len);
        });
    }
    std::memcpy(dst, src, std::min(per, n));
    for (auto &t : th) t.join();
}

}  // namespace

HostPrefault::HostPrefault(void *p, size_t bytes) {
    if (!p || bytes < (size_t(64) << 20) || is_pinned(p)) return;
    const long pg = sysconf(_SC_PAGESIZE);
    const size_t page = pg > 0 ? (size_t)pg : 4096;
    const size_t T = 4, per = ((bytes + T - 1) / T + page - 1) / page * page;
    for (size_t k = 0; k < T && k * per < bytes; ++k) {
        const size_t o = k * per, len = std::min(per, bytes - o);
        th_.emplace_back([=]() {
            volatile char *c = static_cast<char *>(p) + o;
            for (size_t q = 0; q < len; q += page) c[q] = 0;
        });
    }
}

void HostPrefault::wait() {
    for (auto &t : th_)
        if (t.joinable()) t.join();
    th_.clear();
}

int copy_h2d(void *dst, const void *src, size_t n) {
    if (n == 0) return TC_OK;
    if (n <= STAGE_BYTES || is_pinned(src)) {
        TC_CUDA(cudaMemcpy(dst, src, n, cudaMemcpyHostToDevice));
        return TC_OK;
    }
    Staging &s = staging();
    std::lock_guard<std::mutex> lk(s.mu);
    TC_TRY(staging_init(s));
    const size_t nch = (n + STAGE_BYTES - 1) / STAGE_BYTES;
    for (size_t i = 0; i < nch; ++i) {
        const int b = (int)(i & 1);
        const size_t o = i * STAGE_BYTES, len = std::min(STAGE_BYTES, n - o);
        if (i >= 2) TC_CUDA(cudaEventSynchronize(s.ev[b]));  // the DMA of chunk i-2 is done
        par_copy(s.buf[b], static_cast<const char *>(src) + o, len);
        TC_CUDA(cudaMemcpyAsync(static_cast<char *>(dst) + o, s.buf[b], len, cudaMemcpyHostToDevice, s.st));
        TC_CUDA(cudaEventRecord(s.ev[b], s.st));
    }
    TC_CUDA(cudaStreamSynchronize(s.st));
    return TC_OK;
}

int ingest_psd(const float *host, int P, int S, int D, int s0, int ns, float *dev) {
    if (ns == 0) return TC_OK;
    const size_t rowb = (size_t)D * sizeof(float), dpitch = (size_t)P * rowb;
    // rows s of projection p land at dev[s - s0][p][:]
    auto dst_of = [&](int p, int s) { return dev + ((size_t)(s - s0) * P + p) * D; };
    if (is_pinned(host)) {
        Staging &sg = staging();
        std::lock_guard<std::mutex> lk(sg.mu);
        TC_TRY(staging_init(sg));
        for (int p = 0; p < P; ++p)
            TC_CUDA(cudaMemcpy2DAsync(dst_of(p, s0), dpitch, host + ((size_t)p * S + s0) * D, rowb,
                                      rowb, ns, cudaMemcpyHostToDevice, sg.st));
        TC_CUDA(cudaStreamSynchronize(sg.st));
        return TC_OK;
    }
    if (rowb > STAGE_BYTES) TC_FAIL(TC_ERR_SHAPE, "detector row larger than the staging buffer");
    Staging &sg = staging();
    std::lock_guard<std::mutex> lk(sg.mu);
    TC_TRY(staging_init(sg));
    // pieces (projection p, rows sa .. sa+n-1) packed into one staging
    // buffer; a full buffer is sent with one 2-D copy per piece while the
    // other buffer is filled
    struct Piece {
        int p, sa, n;
        size_t row0;  // first row in the staging buffer
    };
    const size_t cap = STAGE_BYTES / rowb;
    std::vector<Piece> pend;
    int b = 0, flushes = 0;
    size_t used = 0;
    auto flush = [&]() -> int {
        for (const Piece &q : pend)
            TC_CUDA(cudaMemcpy2DAsync(dst_of(q.p, q.sa), dpitch,
                                      static_cast<char *>(sg.buf[b]) + q.row0 * rowb, rowb, rowb,
                                      q.n, cudaMemcpyHostToDevice, sg.st));
        TC_CUDA(cudaEventRecord(sg.ev[b], sg.st));
        pend.clear();
        used = 0;
        b ^= 1;
        ++flushes;
        return TC_OK;
    };
    for (int p = 0; p < P; ++p)
        for (int sa = s0; sa < s0 + ns;) {
            if (used == cap) TC_TRY(flush());
            // buffer b was last sent two flushes ago: wait for that copy
            if (used == 0 && flushes >= 2) TC_CUDA(cudaEventSynchronize(sg.ev[b]));
            const int n = (int)std::min<size_t>((size_t)(s0 + ns - sa), cap - used);
            par_copy(static_cast<char *>(sg.buf[b]) + used * rowb, host + ((size_t)p * S + sa) * D,
                     (size_t)n * rowb);
            pend.push_back(Piece{p, sa, n, used});
            used += (size_t)n;
            sa += n;
        }
    if (used) TC_TRY(flush());
    TC_CUDA(cudaStreamSynchronize(sg.st));
    return TC_OK;
}

int copy_d2h(void *dst, const void *src, size_t n) {
    if (n == 0) return TC_OK;
    if (n <= STAGE_BYTES || is_pinned(dst)) {
        TC_CUDA(cudaMemcpy(dst, src, n, cudaMemcpyDeviceToHost));
        return TC_OK;
    }
    Staging &s = staging();
    std::lock_guard<std::mutex> lk(s.mu);
    TC_TRY(staging_init(s));
    TC_CUDA(cudaDeviceSynchronize());  // the producers ran on other streams
    const size_t nch = (n + STAGE_BYTES - 1) / STAGE_BYTES;
    auto issue = [&](size_t i) -> int {
        const int b = (int)(i & 1);
        const size_t o = i * STAGE_BYTES, len = std::min(STAGE_BYTES, n - o);
        TC_CUDA(cudaMemcpyAsync(s.buf[b], static_cast<const char *>(src) + o, len, cudaMemcpyDeviceToHost, s.st));
        TC_CUDA(cudaEventRecord(s.ev[b], s.st));
        return TC_OK;
    };
    TC_TRY(issue(0));
    for (size_t i = 0; i < nch; ++i) {
        const int b = (int)(i & 1);
        const size_t o = i * STAGE_BYTES, len = std::min(STAGE_BYTES, n - o);
        if (i + 1 < nch) TC_TRY(issue(i + 1));  // its buffer's previous chunk was copied out
        TC_CUDA(cudaEventSynchronize(s.ev[b]));
        par_copy(static_cast<char *>(dst) + o, s.buf[b], len);
    }
    return TC_OK;
}

}  // namespace tc
