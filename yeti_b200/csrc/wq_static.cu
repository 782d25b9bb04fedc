// K u with host buffers and no device allocation.
//
// yeti_wq_apply with host buffers allocates two device staging vectors per
// call.  Some callers cannot allocate device memory at that point: a process
// whose device memory is entirely reserved up front by another allocator
// (cudaMalloc would fail), or a latency-critical loop in which the device
// synchronisation implied by cudaMalloc/cudaFree is not acceptable.  This
// entry point stages the vectors in one file-scope device array instead.
//
// Limits and sharing: the array holds two vectors of at most
// kStaticMaxDof doubles (2 x 16 MiB = 32 MiB).  The library's device code is
// loaded lazily by default (CUDA_MODULE_LOADING=LAZY): the array is then
// committed on a device by the first call there (its address lookup loads
// this file's module), and held until the process exits.  Make that first
// call before another allocator reserves all of the device's memory, and
// before any stream capture.  All calls on a device share the
// same array and it keeps the last call's contents (the output half is
// cleared on every call); calls that overlap on the GPU -- from several
// threads, or on several streams -- race on it.
#include <mutex>

#include "wq.cuh"

namespace yeti {

constexpr int64_t kStaticMaxDof = int64_t(1) << 21;   // 2,097,152 dofs
constexpr int kStaticMaxDevices = 64;

// Staging for u (first half) and K u (second half); FP32 calls use the same
// bytes as floats.
static __device__ __align__(256) double g_wq_static_stage[2 * kStaticMaxDof];

// Device address of g_wq_static_stage per device, looked up once per device
// (the symbol's host-side name is not a device address).
static void *g_stage_addr[kStaticMaxDevices] = {nullptr};
static std::mutex g_stage_mutex;

static int stage_address(int device, void **out) {
    YETI_CHECK(device >= 0 && device < kStaticMaxDevices, YETI_EINVAL,
               "yeti_wq_apply_static: device %d beyond the supported %d", device,
               kStaticMaxDevices);
    std::lock_guard<std::mutex> lock(g_stage_mutex);
    if (!g_stage_addr[device]) {
        void *p = nullptr;
        // the caller made `device` current (DeviceGuard)
        YETI_CUDA(cudaGetSymbolAddress(&p, g_wq_static_stage));
        g_stage_addr[device] = p;
    }
    *out = g_stage_addr[device];
    return YETI_OK;
}

}  // namespace yeti

using namespace yeti;

YETI_API int yeti_wq_apply_static(yeti_wq_op *op, const void *u, void *Ku,
                                  int prec) {
    YETI_CHECK(op && u && Ku, YETI_EINVAL, "yeti_wq_apply_static: NULL argument");
    YETI_CHECK(prec == YETI_PREC_F64 || prec == YETI_PREC_F32, YETI_EINVAL,
               "yeti_wq_apply_static: bad precision %d", prec);
    YETI_CHECK(op->ndof <= kStaticMaxDof, YETI_EINVAL,
               "yeti_wq_apply_static: %lld dofs exceed the static staging limit of "
               "%lld dofs; use yeti_wq_apply", (long long)op->ndof,
               (long long)kStaticMaxDof);
    YETI_CHECK(prec == YETI_PREC_F64 ? op->coef64.ptr != nullptr : op->coef32.ptr != nullptr,
               YETI_EINVAL, "yeti_wq_apply_static: operator was set up without that precision");
    DeviceGuard guard(op->ctx->device);
    void *stage = nullptr;
    YETI_TRY(stage_address(op->ctx->device, &stage));
    cudaStream_t s = op->ctx->stream;
    const size_t es = prec == YETI_PREC_F64 ? sizeof(double) : sizeof(float);
    const size_t nb = (size_t)op->ndof * es;
    char *du = static_cast<char *>(stage);
    char *dk = du + (size_t)kStaticMaxDof * sizeof(double);
    YETI_CUDA(cudaMemcpyAsync(du, u, nb, cudaMemcpyHostToDevice, s));
    // the array keeps the previous call's contents: the output must start at 0
    YETI_CUDA(cudaMemsetAsync(dk, 0, nb, s));
    YETI_TRY(wq_apply_dev(op, du, dk, prec, nullptr, s));
    YETI_CUDA(cudaMemcpyAsync(Ku, dk, nb, cudaMemcpyDeviceToHost, s));
    YETI_CUDA(cudaStreamSynchronize(s));
    // a bounded wait of the streaming apply that gave up: report it (and
    // clear the operator's flag, which belongs to this call)
    YETI_TRY(wq_stream_check(op));
    return YETI_OK;
}
