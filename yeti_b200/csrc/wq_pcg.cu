// Jacobi-preconditioned CG on the WQ operator (the 'WP' conjugate gradient
// of wq_mf_cg_3d, src/yeti_iga/iga_wq_mf/fsrc/mf_wq_solver.f90:764-802, with
// a Jacobi preconditioner), in two forms:
//   mode 0: FP64 operator and vectors;
//   mode 1: FP32 operator and inner PCG, FP64 true residual and solution
//           update (iterative refinement).
// All scalars stay on the device; every kernel of an iteration returns at
// once when the device-side `done` flag is set, so the host enqueues
// iterations in chunks and reads the flag once per chunk.  Reductions use a
// fixed grid and a fixed summation tree, so results are run-to-run
// deterministic.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "wq.cuh"

namespace yeti {

constexpr int kRedBlocks = 592;     // 4 x 148 SMs
constexpr int kRedThreads = 256;
constexpr int kChunk = 16;          // iterations enqueued per host check

struct CGScal {
    double rz, pAp, alpha, beta, rr, bb, tol2, scale;
    int done, iter, breakdown, maxit;
};

__device__ __forceinline__ double block_sum(double v, double *sh) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    v = 0.0;
    if (wid == 0) {
        v = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    }
    __syncthreads();
    return v;
}

__device__ __forceinline__ double block_max(double v, double *sh) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    v = 0.0;
    if (wid == 0) {
        v = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    }
    __syncthreads();
    return v;
}

// Sum of nparts partials (single block, fixed order).
__device__ inline double sum_parts(const double *parts, int nparts, int stride,
                                   int off, double *sh) {
    double v = 0.0;
    for (int i = threadIdx.x; i < nparts; i += blockDim.x) v += parts[i * stride + off];
    return block_sum(v, sh);
}

template <class A, class B>
__global__ void __launch_bounds__(kRedThreads)
k_dot(const A *a, const B *b, int64_t n, double *parts, const int *done) {
    __shared__ double sh[32];
    if (done && *done) return;
    double v = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        v += (double)a[i] * (double)b[i];
    v = block_sum(v, sh);
    if (threadIdx.x == 0) parts[blockIdx.x] = v;
}

template <class A>
__global__ void __launch_bounds__(kRedThreads)
k_absmax(const A *a, int64_t n, double *parts) {
    __shared__ double sh[32];
    double v = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        v = fmax(v, fabs((double)a[i]));
    v = block_max(v, sh);
    if (threadIdx.x == 0) parts[blockIdx.x] = v;
}

__global__ void k_alpha(const double *parts, int nparts, CGScal *s) {
    __shared__ double sh[32];
    if (s->done) return;
    const double pAp = sum_parts(parts, nparts, 1, 0, sh);
    if (threadIdx.x == 0) {
        s->pAp = pAp;
        if (!(pAp > 0.0) || !isfinite(pAp)) {
            s->breakdown = 1;
            s->done = 1;
        } else {
            s->alpha = s->rz / pAp;
        }
    }
}

// x += a p; r -= a Ap; z = dinv r; partials of r.z and r.r
template <class T>
__global__ void __launch_bounds__(kRedThreads)
k_update(T *x, T *r, const T *p, const T *Ap, const T *dinv, T *z, int64_t n,
         double *parts, const CGScal *s) {
    __shared__ double sh[32];
    if (s->done) return;
    const T a = (T)s->alpha;
    double rz = 0.0, rr = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        x[i] += a * p[i];
        const T ri = r[i] - a * Ap[i];
        r[i] = ri;
        const T zi = dinv[i] * ri;
        z[i] = zi;
        rz += (double)ri * (double)zi;
        rr += (double)ri * (double)ri;
    }
    rz = block_sum(rz, sh);
    rr = block_sum(rr, sh);
    if (threadIdx.x == 0) {
        parts[2 * blockIdx.x] = rz;
        parts[2 * blockIdx.x + 1] = rr;
    }
}

__global__ void k_beta(const double *parts, int nparts, CGScal *s) {
    __shared__ double sh[32];
    if (s->done) return;
    const double rz = sum_parts(parts, nparts, 2, 0, sh);
    const double rr = sum_parts(parts, nparts, 2, 1, sh);
    if (threadIdx.x == 0) {
        s->iter += 1;
        s->rr = rr;
        s->beta = rz / s->rz;
        s->rz = rz;
        if (!isfinite(rr)) {
            s->breakdown = 1;
            s->done = 1;
        } else if (rr <= s->tol2 || s->iter >= s->maxit) {
            s->done = 1;
        }
    }
}

// p = z + beta p; Ap = 0
template <class T>
__global__ void __launch_bounds__(kRedThreads)
k_pupdate(T *p, const T *z, T *Ap, int64_t n, const CGScal *s) {
    if (s->done) return;
    const T b = (T)s->beta;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        p[i] = z[i] + b * p[i];
        Ap[i] = T(0);
    }
}

// r = mask (b - Ax) in FP64; optional FP32 copy scaled by `scale` set later
__global__ void k_residual(const double *b, const double *Ax,
                           const double *dinv, double *r, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        r[i] = dinv[i] != 0.0 ? b[i] - Ax[i] : 0.0;
}

// CG start: z = dinv r, p = z, Ap = 0, partials of r.z and r.r
template <class T>
__global__ void __launch_bounds__(kRedThreads)
k_start(const T *r, const T *dinv, T *z, T *p, T *Ap, int64_t n,
        double *parts) {
    __shared__ double sh[32];
    double rz = 0.0, rr = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const T zi = dinv[i] * r[i];
        z[i] = zi;
        p[i] = zi;
        Ap[i] = T(0);
        rz += (double)r[i] * (double)zi;
        rr += (double)r[i] * (double)r[i];
    }
    rz = block_sum(rz, sh);
    rr = block_sum(rr, sh);
    if (threadIdx.x == 0) {
        parts[2 * blockIdx.x] = rz;
        parts[2 * blockIdx.x + 1] = rr;
    }
}

__global__ void k_start_scal(const double *parts, int nparts, CGScal *s,
                             double rel2, int maxit) {
    __shared__ double sh[32];
    const double rz = sum_parts(parts, nparts, 2, 0, sh);
    const double rr = sum_parts(parts, nparts, 2, 1, sh);
    if (threadIdx.x == 0) {
        s->rz = rz;
        s->rr = rr;
        s->iter = 0;
        s->breakdown = 0;
        s->maxit = maxit;
        s->tol2 = rel2 * s->bb;
        s->done = (rr <= s->tol2) || maxit <= 0 || !(rr == rr);
    }
}

__global__ void k_set_bb(const double *parts, int nparts, CGScal *s) {
    __shared__ double sh[32];
    const double bb = sum_parts(parts, nparts, 1, 0, sh);
    if (threadIdx.x == 0) s->bb = bb;
}

// FP32 scaled residual: r32 = r64 * scale, d32 = 0
__global__ void k_to_f32(const double *r64, float *r32, float *d32, int64_t n,
                         double scale) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        r32[i] = (float)(r64[i] * scale);
        d32[i] = 0.0f;
    }
}

// x64 += d32 / scale
__global__ void k_refine(double *x, const float *d32, int64_t n, double inv) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        x[i] += (double)d32[i] * inv;
}

// dinv = 1/diag on free dofs, 0 on clamped ones; b masked likewise
template <class T>
__global__ void k_dinv(const double *diag, T *dinv, int64_t ncp, int3 n,
                       int cm0, int cm1, int cm2) {
    const int64_t ndof = 3 * ncp;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < ndof;
         i += (int64_t)gridDim.x * blockDim.x) {
        const int c = (int)(i / ncp);
        const int64_t cp = i % ncp;
        const int u = (int)(cp % n.x), v = (int)((cp / n.x) % n.y), w = (int)(cp / ((int64_t)n.x * n.y));
        const int cm = c == 0 ? cm0 : (c == 1 ? cm1 : cm2);
        const bool cl = ((cm & 1) && u == 0) || ((cm & 2) && u == n.x - 1) ||
                        ((cm & 4) && v == 0) || ((cm & 8) && v == n.y - 1) ||
                        ((cm & 16) && w == 0) || ((cm & 32) && w == n.z - 1);
        dinv[i] = cl ? T(0) : (T)(1.0 / diag[i]);
    }
}

__global__ void k_mask(double *b, const double *dinv, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        if (dinv[i] == 0.0) b[i] = 0.0;
}

static int ensure_workspace(yeti_wq_op *op, bool f32) {
    const int64_t n = op->ndof;
    if (!op->ws64.ptr) YETI_TRY(op->ws64.alloc(op->ctx, 7 * n * sizeof(double)));
    if (f32 && !op->ws32.ptr) YETI_TRY(op->ws32.alloc(op->ctx, 5 * n * sizeof(float)));
    if (!op->scal.ptr) YETI_TRY(op->scal.alloc(op->ctx, 2 * sizeof(CGScal)));
    if (!op->parts.ptr) YETI_TRY(op->parts.alloc(op->ctx, 2 * kRedBlocks * sizeof(double)));
    cudaStream_t s = op->ctx->stream;
    if (!op->dinv64.ptr) {
        YETI_TRY(op->dinv64.alloc(op->ctx, n * sizeof(double)));
        k_dinv<double><<<kRedBlocks, kRedThreads, 0, s>>>(
            op->diag.as<double>(), op->dinv64.as<double>(), op->ncp,
            make_int3(op->n[0], op->n[1], op->n[2]), op->cmask[0], op->cmask[1], op->cmask[2]);
        count_launches(1);
        YETI_CUDA(cudaGetLastError());
    }
    if (f32 && !op->dinv32.ptr) {
        YETI_TRY(op->dinv32.alloc(op->ctx, n * sizeof(float)));
        k_dinv<float><<<kRedBlocks, kRedThreads, 0, s>>>(
            op->diag.as<double>(), op->dinv32.as<float>(), op->ncp,
            make_int3(op->n[0], op->n[1], op->n[2]), op->cmask[0], op->cmask[1], op->cmask[2]);
        count_launches(1);
        YETI_CUDA(cudaGetLastError());
    }
    return YETI_OK;
}

// Run preconditioned CG on A d = r (vectors of type T) until the device flag
// is set; the start kernels must have been enqueued.  Returns the iteration
// count and breakdown flag through the host copy of the scalars.
template <class T>
static int cg_loop(yeti_wq_op *op, int prec, T *x, T *r, T *z, T *p, T *Ap,
                   const T *dinv, CGScal *ds, CGScal *hs) {
    cudaStream_t s = op->ctx->stream;
    const int64_t n = op->ndof;
    double *parts = op->parts.as<double>();
    for (;;) {
        for (int k = 0; k < kChunk; k++) {
            YETI_TRY(wq_apply_dev(op, p, Ap, prec, &ds->done, s));
            k_dot<T, T><<<kRedBlocks, kRedThreads, 0, s>>>(p, Ap, n, parts, &ds->done);
            count_launches(1);
            k_alpha<<<1, kRedThreads, 0, s>>>(parts, kRedBlocks, ds);
            count_launches(1);
            k_update<T><<<kRedBlocks, kRedThreads, 0, s>>>(x, r, p, Ap, dinv, z, n, parts, ds);
            count_launches(1);
            k_beta<<<1, kRedThreads, 0, s>>>(parts, kRedBlocks, ds);
            count_launches(1);
            k_pupdate<T><<<kRedBlocks, kRedThreads, 0, s>>>(p, z, Ap, n, ds);
            count_launches(1);
        }
        YETI_CUDA(cudaGetLastError());
        YETI_CUDA(cudaMemcpyAsync(hs, ds, sizeof(CGScal), cudaMemcpyDeviceToHost, s));
        YETI_CUDA(cudaStreamSynchronize(s));
        if (hs->done) break;
    }
    return YETI_OK;
}

}  // namespace yeti

using namespace yeti;

YETI_API int yeti_wq_pcg(yeti_wq_op *op, const double *b, double *x,
                         double rtol, int maxit, int mode,
                         yeti_cg_stats *stats, int mem) {
    YETI_CHECK(op && b && x, YETI_EINVAL, "yeti_wq_pcg: NULL argument");
    YETI_CHECK(mode == 0 || mode == 1, YETI_EINVAL, "yeti_wq_pcg: mode %d", mode);
    YETI_CHECK(rtol > 0 && maxit > 0, YETI_EINVAL, "yeti_wq_pcg: rtol %g maxit %d", rtol, maxit);
    YETI_CHECK(op->coef64.ptr, YETI_EINVAL,
               "yeti_wq_pcg: the FP64 operator is required (true residual)");
    YETI_CHECK(mode == 0 || op->coef32.ptr, YETI_EINVAL,
               "yeti_wq_pcg: mode 1 needs the FP32 operator (YETI_WQ_F32)");
    DeviceGuard guard(op->ctx->device);
    YETI_TRY(ensure_workspace(op, mode == 1));
    cudaStream_t s = op->ctx->stream;
    const int64_t n = op->ndof;
    double *W = op->ws64.as<double>();
    double *dx = W, *dr = W + n, *dz = W + 2 * n, *dp = W + 3 * n, *dAp = W + 4 * n,
           *db = W + 5 * n, *dt = W + 6 * n;
    double *parts = op->parts.as<double>();
    CGScal *ds = op->scal.as<CGScal>();
    CGScal hs;
    memset(&hs, 0, sizeof(hs));
    cudaEvent_t e0, e1;
    YETI_CUDA(cudaEventCreate(&e0));
    YETI_CUDA(cudaEventCreate(&e1));
    const cudaMemcpyKind h2d = mem == YETI_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    YETI_CUDA(cudaEventRecord(e0, s));
    YETI_CUDA(cudaMemcpyAsync(db, b, n * sizeof(double), h2d, s));
    YETI_CUDA(cudaMemcpyAsync(dx, x, n * sizeof(double), h2d, s));
    const double *dinv = op->dinv64.as<double>();
    k_mask<<<kRedBlocks, kRedThreads, 0, s>>>(db, dinv, n);
    count_launches(1);
    k_mask<<<kRedBlocks, kRedThreads, 0, s>>>(dx, dinv, n);
    count_launches(1);
    k_dot<double, double><<<kRedBlocks, kRedThreads, 0, s>>>(db, db, n, parts, nullptr);
    count_launches(1);
    k_set_bb<<<1, kRedThreads, 0, s>>>(parts, kRedBlocks, ds);
    count_launches(1);
    // r = b - A x
    YETI_CUDA(cudaMemsetAsync(dt, 0, n * sizeof(double), s));
    YETI_TRY(wq_apply_dev(op, dx, dt, YETI_PREC_F64, nullptr, s));
    k_residual<<<kRedBlocks, kRedThreads, 0, s>>>(db, dt, dinv, dr, n);
    count_launches(1);
    YETI_CUDA(cudaGetLastError());
    int iters = 0, outer = 0, f64 = 1, f32 = 0, status = YETI_OK;
    if (mode == 0) {
        k_start<double><<<kRedBlocks, kRedThreads, 0, s>>>(dr, dinv, dz, dp, dAp, n, parts);
        count_launches(1);
        k_start_scal<<<1, kRedThreads, 0, s>>>(parts, kRedBlocks, ds, rtol * rtol, maxit);
        count_launches(1);
        YETI_CUDA(cudaGetLastError());
        YETI_TRY(cg_loop<double>(op, YETI_PREC_F64, dx, dr, dz, dp, dAp, dinv, ds, &hs));
        iters = hs.iter;
        f64 += hs.iter;
        if (hs.breakdown) status = YETI_EBREAKDOWN;
        outer = 1;
    } else {
        float *V = op->ws32.as<float>();
        float *r32 = V, *z32 = V + n, *p32 = V + 2 * n, *Ap32 = V + 3 * n, *d32 = V + 4 * n;
        const float *dinv32 = op->dinv32.as<float>();
        const double eta = 1e-4;   // inner relative tolerance
        CGScal hb;
        YETI_CUDA(cudaMemcpyAsync(&hb, ds, sizeof(CGScal), cudaMemcpyDeviceToHost, s));
        YETI_CUDA(cudaStreamSynchronize(s));
        const double bb = hb.bb;
        for (outer = 0; outer < 50; outer++) {
            // rr of the FP64 true residual (scratch scalars ds[1])
            k_dot<double, double><<<kRedBlocks, kRedThreads, 0, s>>>(dr, dr, n, parts, nullptr);
            count_launches(1);
            k_set_bb<<<1, kRedThreads, 0, s>>>(parts, kRedBlocks, ds + 1);
            count_launches(1);
            YETI_CUDA(cudaMemcpyAsync(&hs, ds + 1, sizeof(CGScal), cudaMemcpyDeviceToHost, s));
            YETI_CUDA(cudaStreamSynchronize(s));
            const double rr = hs.bb;
            if (!(rr == rr)) { status = YETI_EBREAKDOWN; break; }
            if (rr <= rtol * rtol * bb || iters >= maxit) break;
            const double scale = 1.0 / std::sqrt(rr);
            k_to_f32<<<kRedBlocks, kRedThreads, 0, s>>>(dr, r32, d32, n, scale);
            count_launches(1);
            k_start<float><<<kRedBlocks, kRedThreads, 0, s>>>(r32, dinv32, z32, p32, Ap32, n, parts);
            count_launches(1);
            // inner tolerance relative to ||r32|| = 1
            CGScal init;
            memset(&init, 0, sizeof(init));
            init.bb = 1.0;
            YETI_CUDA(cudaMemcpyAsync(ds, &init, sizeof(CGScal), cudaMemcpyHostToDevice, s));
            k_start_scal<<<1, kRedThreads, 0, s>>>(parts, kRedBlocks, ds, eta * eta, maxit - iters);
            count_launches(1);
            YETI_CUDA(cudaGetLastError());
            YETI_TRY(cg_loop<float>(op, YETI_PREC_F32, d32, r32, z32, p32, Ap32, dinv32, ds, &hs));
            iters += hs.iter;
            f32 += hs.iter;
            k_refine<<<kRedBlocks, kRedThreads, 0, s>>>(dx, d32, n, 1.0 / scale);
            count_launches(1);
            YETI_CUDA(cudaMemsetAsync(dt, 0, n * sizeof(double), s));
            YETI_TRY(wq_apply_dev(op, dx, dt, YETI_PREC_F64, nullptr, s));
            k_residual<<<kRedBlocks, kRedThreads, 0, s>>>(db, dt, dinv, dr, n);
            count_launches(1);
            YETI_CUDA(cudaGetLastError());
            f64++;
            if (hs.breakdown && hs.iter == 0) { status = YETI_EBREAKDOWN; break; }
        }
    }
    YETI_CUDA(cudaEventRecord(e1, s));
    // true FP64 residual (mode 0: recompute; mode 1: dr already holds it)
    if (mode == 0) {
        YETI_CUDA(cudaMemsetAsync(dt, 0, n * sizeof(double), s));
        YETI_TRY(wq_apply_dev(op, dx, dt, YETI_PREC_F64, nullptr, s));
        k_residual<<<kRedBlocks, kRedThreads, 0, s>>>(db, dt, dinv, dr, n);
        count_launches(1);
    }
    double h[4];
    k_dot<double, double><<<kRedBlocks, kRedThreads, 0, s>>>(dr, dr, n, parts, nullptr);
    count_launches(1);
    k_dot<double, double><<<kRedBlocks, kRedThreads, 0, s>>>(db, db, n, parts + kRedBlocks, nullptr);
    count_launches(1);
    std::vector<double> hp(2 * kRedBlocks);
    YETI_CUDA(cudaMemcpyAsync(hp.data(), parts, 2 * kRedBlocks * sizeof(double), cudaMemcpyDeviceToHost, s));
    YETI_CUDA(cudaStreamSynchronize(s));
    h[0] = h[1] = 0.0;
    for (int i = 0; i < kRedBlocks; i++) {
        h[0] += hp[i];
        h[1] += hp[kRedBlocks + i];
    }
    k_absmax<double><<<kRedBlocks, kRedThreads, 0, s>>>(dr, n, parts);
    count_launches(1);
    k_absmax<double><<<kRedBlocks, kRedThreads, 0, s>>>(db, n, parts + kRedBlocks);
    count_launches(1);
    YETI_CUDA(cudaMemcpyAsync(hp.data(), parts, 2 * kRedBlocks * sizeof(double), cudaMemcpyDeviceToHost, s));
    YETI_CUDA(cudaStreamSynchronize(s));
    h[2] = h[3] = 0.0;
    for (int i = 0; i < kRedBlocks; i++) {
        h[2] = std::max(h[2], hp[i]);
        h[3] = std::max(h[3], hp[kRedBlocks + i]);
    }
    float ms = 0.f;
    YETI_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    const cudaMemcpyKind d2h = mem == YETI_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    YETI_CUDA(cudaMemcpyAsync(x, dx, n * sizeof(double), d2h, s));
    YETI_CUDA(cudaStreamSynchronize(s));
    const double rel = h[1] > 0 ? std::sqrt(h[0] / h[1]) : 0.0;
    if (status == YETI_OK && !(rel <= rtol)) status = YETI_ENOTCONV;
    if (stats) {
        stats->iterations = iters;
        stats->outer_iterations = outer;
        stats->fp64_applies = f64;
        stats->fp32_applies = f32;
        stats->rel_residual = rel;
        stats->rel_residual_inf = h[3] > 0 ? h[2] / h[3] : 0.0;
        stats->solve_ms = ms;
        stats->status = status;
    }
    if (status == YETI_EBREAKDOWN) {
        set_error("yeti_wq_pcg: Krylov breakdown after %d iterations", iters);
        return status;
    }
    return YETI_OK;
}
