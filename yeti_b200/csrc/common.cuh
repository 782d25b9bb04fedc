// Shared definitions of the yeti_b200 library (host + device).
#pragma once
#include <cuda_runtime.h>
#include <atomic>
#include <cstdint>
#include <cstdio>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/yeti_b200.h"

#define YETI_API extern "C" __attribute__((visibility("default")))

namespace yeti {

// Thread-local error text returned by yeti_last_error().
void set_error(const char *fmt, ...);

// Raise from a cudaError_t: records the text and returns YETI_ECUDA.
int cuda_fail(cudaError_t e, const char *what, const char *file, int line);

#define YETI_CUDA(expr)                                                     \
    do {                                                                    \
        cudaError_t _e = (expr);                                            \
        if (_e != cudaSuccess)                                              \
            return ::yeti::cuda_fail(_e, #expr, __FILE__, __LINE__);        \
    } while (0)

#define YETI_CHECK(cond, code, ...)                                         \
    do {                                                                    \
        if (!(cond)) {                                                      \
            ::yeti::set_error(__VA_ARGS__);                                 \
            return (code);                                                  \
        }                                                                   \
    } while (0)

// Propagate a non-zero status.
#define YETI_TRY(expr)                                                      \
    do {                                                                    \
        int _rc = (expr);                                                   \
        if (_rc != YETI_OK) return _rc;                                     \
    } while (0)

}  // namespace yeti

// Context: device, stream and device-memory accounting.
struct yeti_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;      // stream all work goes to
    cudaStream_t own_stream = nullptr;  // stream created by the context
    size_t hbm_budget = 0;              // 0: unbounded
    std::atomic<size_t> bytes_in_use{0};
    // allocate with cudaMallocAsync / cudaFreeAsync on `stream` (no implicit
    // device synchronisation; for contexts driven by the serving loop)
    bool stream_ordered = false;
    // device-time accounting of the element kernels (yeti_ctx_set_timing)
    bool timing = false;
    std::mutex timing_mu;
    std::map<std::string, double> kernel_ms;
};

namespace yeti {

// Device allocation charged against the context budget.
int dev_alloc(yeti_ctx *ctx, void **ptr, size_t bytes);
void dev_free(yeti_ctx *ctx, void *ptr, size_t bytes);

// RAII device buffer owned by a context.
struct DevBuf {
    yeti_ctx *ctx = nullptr;
    void *ptr = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    DevBuf(DevBuf &&o) noexcept : ctx(o.ctx), ptr(o.ptr), bytes(o.bytes) {
        o.ptr = nullptr;
        o.bytes = 0;
    }
    DevBuf &operator=(DevBuf &&o) noexcept {
        if (this != &o) {
            release();
            ctx = o.ctx;
            ptr = o.ptr;
            bytes = o.bytes;
            o.ptr = nullptr;
            o.bytes = 0;
        }
        return *this;
    }
    ~DevBuf() { release(); }
    int alloc(yeti_ctx *c, size_t n) {
        release();
        ctx = c;
        int rc = dev_alloc(c, &ptr, n);
        if (rc == YETI_OK) bytes = n;
        return rc;
    }
    void release() {
        if (ptr) dev_free(ctx, ptr, bytes);
        ptr = nullptr;
        bytes = 0;
    }
    template <class T> T *as() const { return static_cast<T *>(ptr); }
};

// Upload a host array into a fresh DevBuf.
template <class T>
int upload(yeti_ctx *ctx, DevBuf &buf, const T *host, size_t n) {
    YETI_TRY(buf.alloc(ctx, n * sizeof(T) + 16));
    if (n)
        YETI_CUDA(cudaMemcpyAsync(buf.ptr, host, n * sizeof(T),
                                  cudaMemcpyHostToDevice, ctx->stream));
    return YETI_OK;
}

// Guard that makes ctx->device current for the scope.
struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

// Is `p` device-accessible memory (device or managed)?
bool is_device_pointer(const void *p);

// Let `func` (a kernel) use the device's whole opt-in shared memory: the
// same value on every call, so host threads that launch the kernel
// concurrently cannot lower the limit under each other's launch.  Fails with
// YETI_EUNSUPPORTED when `need` dynamic bytes exceed it.
int set_smem_optin(const void *func, int device, size_t need, const char *what);

// With the context's timing on, the device time of the work enqueued on
// ctx->stream during the object's lifetime (CUDA events on that stream,
// waited for on destruction) is added to ctx->kernel_ms[name]; with timing
// off it does nothing.
struct KernelTimer {
    yeti_ctx *ctx;
    const char *name;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    KernelTimer(yeti_ctx *c, const char *n);
    ~KernelTimer();
};

// Process-wide count of kernel launches issued by the library (reported by
// yeti_kernel_launches(); lets callers verify the device path ran).
void count_launches(uint64_t n);

}  // namespace yeti
