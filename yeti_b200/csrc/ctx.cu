// Context management, error reporting and device-memory accounting.
#include <algorithm>
#include <atomic>
#include <cstdarg>
#include <cstring>

#include "common.cuh"

namespace yeti {

static thread_local char g_err[1024] = "";

void set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

int cuda_fail(cudaError_t e, const char *what, const char *file, int line) {
    set_error("CUDA error %s (%s) in %s at %s:%d", cudaGetErrorName(e),
              cudaGetErrorString(e), what, file, line);
    return YETI_ECUDA;
}

int dev_alloc(yeti_ctx *ctx, void **ptr, size_t bytes) {
    *ptr = nullptr;
    if (bytes == 0) bytes = 16;
    if (ctx->hbm_budget && ctx->bytes_in_use + bytes > ctx->hbm_budget) {
        set_error("HBM budget exceeded: %zu in use + %zu requested > %zu",
                  ctx->bytes_in_use.load(), bytes, ctx->hbm_budget);
        return YETI_ENOMEM;
    }
    cudaError_t e = ctx->stream_ordered ? cudaMallocAsync(ptr, bytes, ctx->stream)
                                        : cudaMalloc(ptr, bytes);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        set_error("cudaMalloc of %zu bytes failed: %s", bytes,
                  cudaGetErrorString(e));
        *ptr = nullptr;
        return YETI_ENOMEM;
    }
    ctx->bytes_in_use += bytes;
    return YETI_OK;
}

void dev_free(yeti_ctx *ctx, void *ptr, size_t bytes) {
    if (!ptr) return;
    if (ctx && ctx->stream_ordered) cudaFreeAsync(ptr, ctx->stream);
    else cudaFree(ptr);
    if (ctx) ctx->bytes_in_use -= (bytes ? bytes : 16);
}

static std::atomic<uint64_t> g_launches{0};

void count_launches(uint64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

int set_smem_optin(const void *func, int device, size_t need, const char *what) {
    int optin = 0;
    YETI_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
    cudaFuncAttributes fa;
    YETI_CUDA(cudaFuncGetAttributes(&fa, func));
    const int dyn = optin - (int)fa.sharedSizeBytes;
    YETI_CHECK(need <= (size_t)std::max(dyn, 0), YETI_EUNSUPPORTED,
               "%s needs %zu bytes of dynamic shared memory (limit %d)", what, need, dyn);
    YETI_CUDA(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn));
    return YETI_OK;
}

bool is_device_pointer(const void *p) {
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        (void)cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

}  // namespace yeti

using namespace yeti;

YETI_API const char *yeti_last_error(void) { return g_err; }

YETI_API const char *yeti_version(void) { return "yeti_b200 0.1 (sm_100a)"; }

YETI_API uint64_t yeti_kernel_launches(void) {
    return g_launches.load(std::memory_order_relaxed);
}

YETI_API int yeti_ctx_create(int device, size_t hbm_budget_bytes,
                             yeti_ctx **out) {
    YETI_CHECK(out, YETI_EINVAL, "yeti_ctx_create: out is NULL");
    *out = nullptr;
    int n = 0;
    YETI_CUDA(cudaGetDeviceCount(&n));
    YETI_CHECK(device >= 0 && device < n, YETI_EINVAL,
               "yeti_ctx_create: device %d out of range (%d devices)", device,
               n);
    DeviceGuard g(device);
    yeti_ctx *c = new yeti_ctx();
    c->device = device;
    c->hbm_budget = hbm_budget_bytes;
    cudaError_t e = cudaStreamCreateWithFlags(&c->own_stream,
                                              cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete c;
        return cuda_fail(e, "cudaStreamCreate", __FILE__, __LINE__);
    }
    c->stream = c->own_stream;
    *out = c;
    return YETI_OK;
}

YETI_API int yeti_ctx_destroy(yeti_ctx *ctx) {
    if (!ctx) return YETI_OK;
    DeviceGuard g(ctx->device);
    if (ctx->own_stream) {
        cudaStreamSynchronize(ctx->own_stream);
        cudaStreamDestroy(ctx->own_stream);
    }
    delete ctx;
    return YETI_OK;
}

YETI_API int yeti_ctx_set_stream(yeti_ctx *ctx, void *stream) {
    YETI_CHECK(ctx, YETI_EINVAL, "yeti_ctx_set_stream: ctx is NULL");
    ctx->stream = stream ? static_cast<cudaStream_t>(stream) : ctx->own_stream;
    return YETI_OK;
}

YETI_API int yeti_ctx_synchronize(yeti_ctx *ctx) {
    YETI_CHECK(ctx, YETI_EINVAL, "yeti_ctx_synchronize: ctx is NULL");
    DeviceGuard g(ctx->device);
    YETI_CUDA(cudaStreamSynchronize(ctx->stream));
    return YETI_OK;
}

YETI_API size_t yeti_ctx_bytes_in_use(const yeti_ctx *ctx) {
    return ctx ? ctx->bytes_in_use.load() : 0;
}

namespace yeti {

KernelTimer::KernelTimer(yeti_ctx *c, const char *n) : ctx(c), name(n) {
    if (!ctx || !ctx->timing) return;
    if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess ||
        cudaEventRecord(e0, ctx->stream) != cudaSuccess) {
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        e0 = e1 = nullptr;
    }
}

KernelTimer::~KernelTimer() {
    if (!e0) return;
    float ms = 0.f;
    if (cudaEventRecord(e1, ctx->stream) == cudaSuccess && cudaEventSynchronize(e1) == cudaSuccess &&
        cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess) {
        std::lock_guard<std::mutex> lk(ctx->timing_mu);
        ctx->kernel_ms[name] += ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
}

}  // namespace yeti

YETI_API int yeti_ctx_set_timing(yeti_ctx *ctx, int on) {
    YETI_CHECK(ctx, YETI_EINVAL, "yeti_ctx_set_timing: ctx is NULL");
    std::lock_guard<std::mutex> lk(ctx->timing_mu);
    ctx->timing = on != 0;
    ctx->kernel_ms.clear();
    return YETI_OK;
}

YETI_API double yeti_ctx_kernel_ms(yeti_ctx *ctx, const char *kernel) {
    if (!ctx || !kernel) return -1.0;
    std::lock_guard<std::mutex> lk(ctx->timing_mu);
    auto it = ctx->kernel_ms.find(kernel);
    return it == ctx->kernel_ms.end() ? -1.0 : it->second;
}
