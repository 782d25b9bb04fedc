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

#include <cooperative_groups.h>

#include "reduce.cuh"
#include "wq.cuh"

namespace yeti {

constexpr int kRedBlocks = 592;     // 4 x 148 SMs
constexpr int kRedThreads = 256;
constexpr int kFusedThreads = 1024; // k_cg_fused: one CTA per SM
constexpr int kChunk = 16;          // iterations enqueued per host check

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

// a * b rounded to T (never contracted into a following add)
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }

// block_sum's total (which only thread 0 holds) given to every thread
__device__ __forceinline__ double block_sum_all(double v, double *sh) {
    __shared__ double total;
    v = block_sum(v, sh);
    if (threadIdx.x == 0) total = v;
    __syncthreads();
    v = total;
    __syncthreads();   // before a later call overwrites total
    return v;
}

// One Jacobi-PCG iteration after the apply, in one cooperative launch: the
// work of k_dot_alpha, k_update_beta and k_pupdate with two grid-wide
// barriers instead of three launches and their last-block reductions.  No
// vector is kept across a barrier (p, r and the inverse diagonal are read
// again from L2; z = dinv r is recomputed from the stored r, the same value);
// every block sums the partials in the same fixed order, so all blocks take
// the same alpha, beta and stop decision.  One CTA of kFusedThreads per SM
// (fewer blocks to meet at each grid barrier than 4 x 256-thread CTAs: 2 us
// less per iteration at 64^3); its partial sums are taken over its own
// blocks, so the results can differ from the three-kernel path's in the last
// bits.  parts: 3 * gridDim.x doubles.
template <class T>
__global__ void __launch_bounds__(kFusedThreads, 1)
k_cg_fused(T *x, T *r, T *p, T *Ap, const T *dinv, int64_t n, double *parts, CGScal *s) {
    __shared__ double sh[32];
    if (s->done) return;   // read by every block before anyone can set it
    cooperative_groups::grid_group grid = cooperative_groups::this_grid();
    const int64_t gt = (int64_t)gridDim.x * blockDim.x;
    const int64_t i0 = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int nb = (int)gridDim.x;
    const double rz_old = s->rz, tol2 = s->tol2;
    const int iter = s->iter, maxit = s->maxit;
    // each thread's elements i0, i0 + gt, ... in order, U at a time with
    // their loads issued together (the sums keep the one-by-one order)
    constexpr int U = sizeof(T) == 4 ? 4 : 2;
    double v = 0.0;
    for (int64_t i = i0; i < n; i += U * gt) {
        T pv[U], av[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int64_t j = i + u * gt;
            pv[u] = j < n ? p[j] : T(0);
            av[u] = j < n ? Ap[j] : T(0);
        }
#pragma unroll
        for (int u = 0; u < U; u++)
            if (i + u * gt < n) v += (double)pv[u] * (double)av[u];
    }
    v = block_sum(v, sh);
    if (threadIdx.x == 0) __stcg(&parts[blockIdx.x], v);
    grid.sync();
    double pAp = 0.0;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) pAp += __ldcg(&parts[i]);
    pAp = block_sum_all(pAp, sh);
    if (!(pAp > 0.0) || !isfinite(pAp)) {   // the same decision in every block
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            s->pAp = pAp;
            s->breakdown = 1;
            s->done = 1;
        }
        return;
    }
    const double alpha = rz_old / pAp;
    const T a = (T)alpha;
    double rz = 0.0, rr = 0.0;
    for (int64_t i = i0; i < n; i += U * gt) {
        T xv[U], pv[U], rv[U], av[U], dv[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int64_t j = i + u * gt;
            const bool in = j < n;
            xv[u] = in ? x[j] : T(0);
            pv[u] = in ? p[j] : T(0);
            rv[u] = in ? r[j] : T(0);
            av[u] = in ? Ap[j] : T(0);
            dv[u] = in ? dinv[j] : T(0);
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int64_t j = i + u * gt;
            if (j >= n) continue;
            x[j] = xv[u] + a * pv[u];
            const T ri = rv[u] - a * av[u];
            r[j] = ri;
            const T zi = dv[u] * ri;
            rz += (double)ri * (double)zi;
            rr += (double)ri * (double)ri;
        }
    }
    rz = block_sum(rz, sh);
    rr = block_sum(rr, sh);
    if (threadIdx.x == 0) {
        __stcg(&parts[nb + 2 * blockIdx.x], rz);
        __stcg(&parts[nb + 2 * blockIdx.x + 1], rr);
    }
    grid.sync();
    double srz = 0.0, srr = 0.0;
    for (int i = threadIdx.x; i < nb; i += blockDim.x) {
        srz += __ldcg(&parts[nb + 2 * i]);
        srr += __ldcg(&parts[nb + 2 * i + 1]);
    }
    srz = block_sum_all(srz, sh);
    srr = block_sum_all(srr, sh);
    const int it = iter + 1;
    const double beta = srz / rz_old;
    const bool bad = !isfinite(srr);
    const bool stop = bad || srr <= tol2 || it >= maxit;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        s->pAp = pAp;
        s->alpha = alpha;
        s->iter = it;
        s->rr = srr;
        s->beta = beta;
        s->rz = srz;
        if (bad) s->breakdown = 1;
        if (stop) s->done = 1;
    }
    if (stop) return;
    const T bt = (T)beta;
    for (int64_t i = i0; i < n; i += U * gt) {
        T dv[U], rv[U], pv[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int64_t j = i + u * gt;
            const bool in = j < n;
            dv[u] = in ? dinv[j] : T(0);
            rv[u] = in ? r[j] : T(0);
            pv[u] = in ? p[j] : T(0);
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int64_t j = i + u * gt;
            if (j >= n) continue;
            const T zi = mul_rn(dv[u], rv[u]);   // z as the three-kernel path stores it
            p[j] = zi + bt * pv[u];
            Ap[j] = T(0);
        }
    }
}

// End of an iteration: stop the chunk once the residual has dropped to
// pause2 (a reliable update follows on the host, the direction is kept).
__global__ void k_pause(CGScal *s) {
    if (!s->done && s->rr <= s->pause2) {
        s->done = 1;
        s->paused = 1;
    }
}

// The reference's per-iteration measures (wq_mf_cg_3d, mf_wq_solver.f90:
// 785-792): after iteration g, max|r| and (ds given) max|ds - x| into
// hist[2g], hist[2g+1]; recorded only if iteration g ran (s->iter == g).  The
// last block also applies the reference's stop test max|r| <= stop_abs
// (mf_wq_solver.f90:931-936), stop_abs = eps max|b|.
template <class S>
__global__ void __launch_bounds__(kRedThreads)
k_hist(const double *r, const double *x, const double *ds, int64_t n, double *parts,
       unsigned int *ticket, double *hist, int g, double stop_abs, S *s) {
    __shared__ double sh[32];
    if (s->iter != g) return;
    double mr = 0.0, me = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        mr = fmax(mr, fabs(r[i]));
        if (ds) me = fmax(me, fabs(ds[i] - x[i]));
    }
    mr = block_max(mr, sh);
    me = block_max(me, sh);
    if (threadIdx.x == 0) {
        __stcg(&parts[2 * blockIdx.x], mr);
        __stcg(&parts[2 * blockIdx.x + 1], me);
    }
    if (!last_block(ticket)) return;
    double tr = 0.0, te = 0.0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) {
        tr = fmax(tr, __ldcg(&parts[2 * i]));
        te = fmax(te, __ldcg(&parts[2 * i + 1]));
    }
    tr = block_max(tr, sh);
    te = block_max(te, sh);
    if (threadIdx.x == 0) {
        *ticket = 0;
        hist[2 * g] = tr;
        hist[2 * g + 1] = te;
        if (tr <= stop_abs) s->done = 1;
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

// p.Ap partials, then (last block) alpha = rz / p.Ap
template <class T>
__global__ void __launch_bounds__(kRedThreads)
k_dot_alpha(const T *p, const T *Ap, int64_t n, double *parts, CGScal *s) {
    __shared__ double sh[32];
    if (s->done) return;
    double v = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        v += (double)p[i] * (double)Ap[i];
    v = block_sum(v, sh);
    if (threadIdx.x == 0) __stcg(&parts[blockIdx.x], v);
    if (!last_block(&s->ticket)) return;
    double pAp = 0.0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) pAp += __ldcg(&parts[i]);
    pAp = block_sum(pAp, sh);
    if (threadIdx.x == 0) {
        s->ticket = 0;
        s->pAp = pAp;
        if (!(pAp > 0.0) || !isfinite(pAp)) {
            s->breakdown = 1;
            s->done = 1;
        } else {
            s->alpha = s->rz / pAp;
        }
    }
}

// x += a p; r -= a Ap; z = dinv r; then (last block) beta, rz, rr, stop test.
// dinv == nullptr (another preconditioner): no z, r.z or beta here.
template <class T>
__global__ void __launch_bounds__(kRedThreads)
k_update_beta(T *x, T *r, const T *p, const T *Ap, const T *dinv, T *z, int64_t n,
              double *parts, CGScal *s) {
    __shared__ double sh[32];
    if (s->done) return;
    const T a = (T)s->alpha;
    double rz = 0.0, rr = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        x[i] += a * p[i];
        const T ri = r[i] - a * Ap[i];
        r[i] = ri;
        if (dinv) {
            const T zi = dinv[i] * ri;
            z[i] = zi;
            rz += (double)ri * (double)zi;
        }
        rr += (double)ri * (double)ri;
    }
    rz = block_sum(rz, sh);
    rr = block_sum(rr, sh);
    if (threadIdx.x == 0) {
        __stcg(&parts[2 * blockIdx.x], rz);
        __stcg(&parts[2 * blockIdx.x + 1], rr);
    }
    if (!last_block(&s->ticket)) return;
    double srz = 0.0, srr = 0.0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) {
        srz += __ldcg(&parts[2 * i]);
        srr += __ldcg(&parts[2 * i + 1]);
    }
    srz = block_sum(srz, sh);
    srr = block_sum(srr, sh);
    if (threadIdx.x == 0) {
        s->ticket = 0;
        s->iter += 1;
        s->rr = srr;
        if (dinv) {
            s->beta = srz / s->rz;
            s->rz = srz;
        }
        if (!isfinite(srr)) {
            s->breakdown = 1;
            s->done = 1;
        } else if (srr <= s->tol2 || s->iter >= s->maxit) {
            s->done = 1;
        }
    }
}

// r = mask (b - Ax) in FP64; optional FP32 copy scaled by `scale` set later
__global__ void k_residual(const double *b, const double *Ax,
                           const double *dinv, double *r, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        r[i] = dinv[i] != 0.0 ? b[i] - Ax[i] : 0.0;
}

// CG start: z = dinv r, p = z, Ap = 0, partials of r.z and r.r (dinv ==
// nullptr: Ap = 0 and r.r only; the preconditioner sets z, p and r.z)
template <class T>
__global__ void __launch_bounds__(kRedThreads)
k_start(const T *r, const T *dinv, T *z, T *p, T *Ap, int64_t n,
        double *parts) {
    __shared__ double sh[32];
    double rz = 0.0, rr = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        if (dinv) {
            const T zi = dinv[i] * r[i];
            z[i] = zi;
            p[i] = zi;
            rz += (double)r[i] * (double)zi;
        }
        Ap[i] = T(0);
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

// Reliable update, part 1: x64 += scale * d32, d32 = 0
__global__ void k_ru_accum(double *x, float *d32, int64_t n, double scale) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        x[i] += scale * (double)d32[i];
        d32[i] = 0.0f;
    }
}

// Reliable update, part 2: r32 = r64 / s_new, z32 = dinv r32, p32 *= factor
// (or p32 = z32 to restart), partials of r.z and r.r
__global__ void __launch_bounds__(kRedThreads)
k_ru_replace(const double *r64, float *r32, float *z32, float *p32,
             const float *dinv, int64_t n, double inv_s, float factor,
             int restart, double *parts) {
    __shared__ double sh[32];
    double rz = 0.0, rr = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const float ri = (float)(r64[i] * inv_s);
        r32[i] = ri;
        if (dinv) {
            const float zi = dinv[i] * ri;
            z32[i] = zi;
            p32[i] = restart ? zi : p32[i] * factor;
            rz += (double)ri * (double)zi;
        } else if (!restart) {
            p32[i] *= factor;
        }
        rr += (double)ri * (double)ri;
    }
    rz = block_sum(rz, sh);
    rr = block_sum(rr, sh);
    if (threadIdx.x == 0) {
        parts[2 * blockIdx.x] = rz;
        parts[2 * blockIdx.x + 1] = rr;
    }
}

__global__ void k_ru_scal(const double *parts, int nparts, CGScal *s,
                          double tol2, int maxit) {
    __shared__ double sh[32];
    const double rz = sum_parts(parts, nparts, 2, 0, sh);
    const double rr = sum_parts(parts, nparts, 2, 1, sh);
    if (threadIdx.x == 0) {
        s->rz = rz;
        s->rr = rr;
        s->tol2 = tol2;
        s->maxit = maxit;
        s->done = 0;
        s->paused = 0;
    }
}

// ---------------------------------------------------------------- BiCGSTAB
// Right-preconditioned BiCGSTAB (the reference's wq_mf_bicgstab_3d,
// mf_wq_solver.f90:958-1308, with a Jacobi preconditioner).
struct BiScal {
    double rho, alpha, omega, beta, rr, tol2, ts, tt;
    int done, iter, breakdown, maxit;
};

template <class T>
__global__ void __launch_bounds__(kRedThreads)
k_bi_alpha_s(const double *parts, int nparts, BiScal *s) {
    __shared__ double sh[32];
    if (s->done) return;
    const double rv = sum_parts(parts, nparts, 1, 0, sh);
    if (threadIdx.x == 0) {
        if (!(rv != 0.0) || !isfinite(rv)) {
            s->breakdown = 1;
            s->done = 1;
        } else {
            s->alpha = s->rho / rv;
        }
    }
}

// s = r - alpha v; sh = dinv s (unless dinv == nullptr); t = 0
template <class T>
__global__ void __launch_bounds__(kRedThreads)
k_bi_s(const T *r, const T *v, const T *dinv, T *sv, T *shat, T *t, int64_t n,
       const BiScal *s) {
    if (s->done) return;
    const T a = (T)s->alpha;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const T si = r[i] - a * v[i];
        sv[i] = si;
        if (dinv) shat[i] = dinv[i] * si;
        t[i] = T(0);
    }
}

// partials of t.s and t.t
template <class T>
__global__ void __launch_bounds__(kRedThreads)
k_bi_ts(const T *t, const T *sv, int64_t n, double *parts, const BiScal *s) {
    __shared__ double sh[32];
    if (s->done) return;
    double ts = 0.0, tt = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        ts += (double)t[i] * (double)sv[i];
        tt += (double)t[i] * (double)t[i];
    }
    ts = block_sum(ts, sh);
    tt = block_sum(tt, sh);
    if (threadIdx.x == 0) {
        parts[2 * blockIdx.x] = ts;
        parts[2 * blockIdx.x + 1] = tt;
    }
}

__global__ void k_bi_omega(const double *parts, int nparts, BiScal *s) {
    __shared__ double sh[32];
    if (s->done) return;
    const double ts = sum_parts(parts, nparts, 2, 0, sh);
    const double tt = sum_parts(parts, nparts, 2, 1, sh);
    if (threadIdx.x == 0) {
        if (!(tt > 0.0) || !isfinite(ts)) {
            s->breakdown = 1;
            s->done = 1;
        } else {
            s->omega = ts / tt;
        }
    }
}

// x += alpha ph + omega sh; r = s - omega t; partials of rhat.r and r.r
template <class T>
__global__ void __launch_bounds__(kRedThreads)
k_bi_update(T *x, T *r, const T *rhat, const T *ph, const T *shat, const T *sv,
            const T *t, int64_t n, double *parts, const BiScal *s) {
    __shared__ double sh[32];
    if (s->done) return;
    const T a = (T)s->alpha, w = (T)s->omega;
    double rho = 0.0, rr = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        x[i] += a * ph[i] + w * shat[i];
        const T ri = sv[i] - w * t[i];
        r[i] = ri;
        rho += (double)rhat[i] * (double)ri;
        rr += (double)ri * (double)ri;
    }
    rho = block_sum(rho, sh);
    rr = block_sum(rr, sh);
    if (threadIdx.x == 0) {
        parts[2 * blockIdx.x] = rho;
        parts[2 * blockIdx.x + 1] = rr;
    }
}

__global__ void k_bi_beta(const double *parts, int nparts, BiScal *s) {
    __shared__ double sh[32];
    if (s->done) return;
    const double rho = sum_parts(parts, nparts, 2, 0, sh);
    const double rr = sum_parts(parts, nparts, 2, 1, sh);
    if (threadIdx.x == 0) {
        s->iter += 1;
        s->rr = rr;
        s->beta = (rho / s->rho) * (s->alpha / s->omega);
        s->rho = rho;
        if (!isfinite(rr) || rho == 0.0) {
            s->breakdown = !isfinite(rr);
            s->done = 1;
        } else if (rr <= s->tol2 || s->iter >= s->maxit) {
            s->done = 1;
        }
    }
}

// p = r + beta (p - omega v); ph = dinv p (unless dinv == nullptr); v = 0
template <class T>
__global__ void __launch_bounds__(kRedThreads)
k_bi_p(T *p, T *ph, const T *r, T *v, const T *dinv, int64_t n,
       const BiScal *s) {
    if (s->done) return;
    const T b = (T)s->beta, w = (T)s->omega;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const T pi = r[i] + b * (p[i] - w * v[i]);
        p[i] = pi;
        if (dinv) ph[i] = dinv[i] * pi;
        v[i] = T(0);
    }
}

// start: rhat = r, p = r, ph = dinv r (unless dinv == nullptr), v = 0,
// partials of r.r
template <class T>
__global__ void __launch_bounds__(kRedThreads)
k_bi_start(const T *r, T *rhat, T *p, T *ph, T *v, const T *dinv, int64_t n,
           double *parts) {
    __shared__ double sh[32];
    double rr = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        rhat[i] = r[i];
        p[i] = r[i];
        if (dinv) ph[i] = dinv[i] * r[i];
        v[i] = T(0);
        rr += (double)r[i] * (double)r[i];
    }
    rr = block_sum(rr, sh);
    if (threadIdx.x == 0) parts[blockIdx.x] = rr;
}

__global__ void k_bi_start_scal(const double *parts, int nparts, BiScal *s,
                                double tol2, int maxit) {
    __shared__ double sh[32];
    const double rr = sum_parts(parts, nparts, 1, 0, sh);
    if (threadIdx.x == 0) {
        s->rho = rr;
        s->rr = rr;
        s->iter = 0;
        s->breakdown = 0;
        s->maxit = maxit;
        s->tol2 = tol2;
        s->done = (rr <= tol2) || maxit <= 0 || !(rr == rr);
    }
}

// as k_bi_start_scal with the tolerance relative to the start residual
// (x0 = 0: r = b)
__global__ void k_bi_start_scal_rel(const double *parts, int nparts, BiScal *s,
                                    double rel2, int maxit) {
    __shared__ double sh[32];
    const double rr = sum_parts(parts, nparts, 1, 0, sh);
    if (threadIdx.x == 0) {
        s->rho = rr;
        s->rr = rr;
        s->iter = 0;
        s->breakdown = 0;
        s->maxit = maxit;
        s->tol2 = rel2 * rr;
        s->done = (rr <= s->tol2) || maxit <= 0 || !(rr == rr);
    }
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
    if (!op->ws64.ptr) YETI_TRY(op->ws64.alloc(op->ctx, 12 * n * sizeof(double)));
    if (f32 && !op->ws32.ptr) YETI_TRY(op->ws32.alloc(op->ctx, 10 * n * sizeof(float)));
    if (!op->scal.ptr) YETI_TRY(op->scal.alloc(op->ctx, 4 * sizeof(CGScal)));
    if (!op->parts.ptr) YETI_TRY(op->parts.alloc(op->ctx, 4 * kRedBlocks * sizeof(double)));
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

// Enqueue up to kChunk CG iterations (every kernel exits at once when the
// device flag is set).
// dinv == nullptr: the fast-diagonalisation preconditioner gives z, r.z and
// beta after the update.
// Grid of the cooperative k_cg_fused launch (one CTA per SM, all
// co-resident), or 0 when the iteration cannot run as one.
template <class T>
static int cg_fused_grid(const yeti_wq_op *op) {
    int dev = op->ctx->device, coop = 0, sms = 0, per_sm = 0;
    if (cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_cg_fused<T>, kFusedThreads, 0) !=
            cudaSuccess) {
        (void)cudaGetLastError();
        return 0;
    }
    if (!coop || per_sm < 1) return 0;
    return std::min(sms, kRedBlocks);   // parts holds 3 x kRedBlocks partials
}

template <class T>
static int cg_chunk(yeti_wq_op *op, int prec, T *x, T *r, T *z, T *p, T *Ap,
                    const T *dinv, CGScal *ds, bool pause = false) {
    cudaStream_t s = op->ctx->stream;
    const int64_t n = op->ndof;
    double *parts = op->parts.as<double>();
    const int fgrid = dinv && !pause ? cg_fused_grid<T>(op) : 0;
    if (fgrid > 0) {
        for (int k = 0; k < kChunk; k++) {
            YETI_TRY(wq_apply_dev(op, p, Ap, prec, &ds->done, s));
            int64_t nn = n;
            void *args[] = {&x, &r, &p, &Ap, (void *)&dinv, &nn, &parts, &ds};
            YETI_CUDA(cudaLaunchCooperativeKernel((const void *)k_cg_fused<T>, dim3(fgrid),
                                                  dim3(kFusedThreads), args, 0, s));
            count_launches(1);
        }
        YETI_CUDA(cudaGetLastError());
        return YETI_OK;
    }
    for (int k = 0; k < kChunk; k++) {
        YETI_TRY(wq_apply_dev(op, p, Ap, prec, &ds->done, s));
        k_dot_alpha<T><<<kRedBlocks, kRedThreads, 0, s>>>(p, Ap, n, parts, ds);
        k_update_beta<T><<<kRedBlocks, kRedThreads, 0, s>>>(x, r, p, Ap, dinv, z, n, parts, ds);
        if (!dinv) YETI_TRY(wq_fd_apply<T>(op, r, z, &ds->done, FD_ITER, nullptr, ds, s));
        k_pupdate<T><<<kRedBlocks, kRedThreads, 0, s>>>(p, z, Ap, n, ds);
        count_launches(3);
        if (pause) {
            k_pause<<<1, 1, 0, s>>>(ds);
            count_launches(1);
        }
    }
    YETI_CUDA(cudaGetLastError());
    return YETI_OK;
}

template <class T>
static int cg_loop(yeti_wq_op *op, int prec, T *x, T *r, T *z, T *p, T *Ap,
                   const T *dinv, CGScal *ds, CGScal *hs) {
    cudaStream_t s = op->ctx->stream;
    for (;;) {
        YETI_TRY(cg_chunk<T>(op, prec, x, r, z, p, Ap, dinv, ds));
        YETI_CUDA(cudaMemcpyAsync(hs, ds, sizeof(CGScal), cudaMemcpyDeviceToHost, s));
        YETI_CUDA(cudaStreamSynchronize(s));
        if (hs->done) break;
    }
    return YETI_OK;
}

template <class T>
static int bi_loop(yeti_wq_op *op, int prec, T *x, T *r, T *rhat, T *p, T *ph,
                   T *v, T *sv, T *shat, T *t, const T *dinv, BiScal *ds,
                   BiScal *hs) {
    cudaStream_t s = op->ctx->stream;
    const int64_t n = op->ndof;
    double *parts = op->parts.as<double>();
    for (;;) {
        for (int k = 0; k < kChunk; k++) {
            YETI_TRY(wq_apply_dev(op, ph, v, prec, &ds->done, s));
            k_dot<T, T><<<kRedBlocks, kRedThreads, 0, s>>>(rhat, v, n, parts, &ds->done);
            k_bi_alpha_s<T><<<1, kRedThreads, 0, s>>>(parts, kRedBlocks, ds);
            k_bi_s<T><<<kRedBlocks, kRedThreads, 0, s>>>(r, v, dinv, sv, shat, t, n, ds);
            if (!dinv) YETI_TRY(wq_fd_apply<T>(op, sv, shat, &ds->done, FD_NONE, nullptr, nullptr, s));
            YETI_TRY(wq_apply_dev(op, shat, t, prec, &ds->done, s));
            k_bi_ts<T><<<kRedBlocks, kRedThreads, 0, s>>>(t, sv, n, parts, ds);
            k_bi_omega<<<1, kRedThreads, 0, s>>>(parts, kRedBlocks, ds);
            k_bi_update<T><<<kRedBlocks, kRedThreads, 0, s>>>(x, r, rhat, ph, shat, sv, t, n, parts, ds);
            k_bi_beta<<<1, kRedThreads, 0, s>>>(parts, kRedBlocks, ds);
            k_bi_p<T><<<kRedBlocks, kRedThreads, 0, s>>>(p, ph, r, v, dinv, n, ds);
            if (!dinv) YETI_TRY(wq_fd_apply<T>(op, p, ph, &ds->done, FD_NONE, nullptr, nullptr, s));
            count_launches(8);
        }
        YETI_CUDA(cudaGetLastError());
        YETI_CUDA(cudaMemcpyAsync(hs, ds, sizeof(BiScal), cudaMemcpyDeviceToHost, s));
        YETI_CUDA(cudaStreamSynchronize(s));
        if (hs->done) break;
    }
    return YETI_OK;
}

// ------------------------------------------- resumable solves (serving loop)
static int ensure_dinv64(yeti_wq_op *op) {
    if (op->dinv64.ptr) return YETI_OK;
    YETI_TRY(op->dinv64.alloc(op->ctx, op->ndof * sizeof(double)));
    k_dinv<double><<<kRedBlocks, kRedThreads, 0, op->ctx->stream>>>(
        op->diag.as<double>(), op->dinv64.as<double>(), op->ncp,
        make_int3(op->n[0], op->n[1], op->n[2]), op->cmask[0], op->cmask[1], op->cmask[2]);
    count_launches(1);
    YETI_CUDA(cudaGetLastError());
    YETI_CUDA(cudaStreamSynchronize(op->ctx->stream));
    return YETI_OK;
}

size_t cgsolve_scal_bytes() { return std::max(sizeof(CGScal), sizeof(BiScal)); }

void CgSolve::release() {
    if (chunk) cudaGraphExecDestroy(chunk);
    if (ev) cudaEventDestroy(ev);
    if (dmem) cudaFreeAsync(dmem, stream);
    chunk = nullptr;
    ev = nullptr;
    dmem = nullptr;
    in_flight = false;
}

// Workspace of a resumable solve: vectors, partials, the scalars (CGScal or
// BiScal), the FD workspace.  CG: b x r z p Ap; BiCGSTAB: b x r (z unused)
// p v (in Ap) and rhat ph s shat t.
struct SolveView {
    double *b, *x, *r, *z, *p, *Ap, *parts;
    double *rhat, *ph, *sv, *shat, *t;   // BiCGSTAB
    CGScal *s;
    BiScal *bs;
    double *fdt, *fdparts;   // FD: two intermediate vectors, partials
};

static int solve_vectors(bool bicg) { return bicg ? 11 : 6; }

static SolveView solve_view(const CgSolve &cs) {
    const int64_t n = cs.op->ndof;
    double *W = static_cast<double *>(cs.dmem);
    const int nv = solve_vectors(cs.bicg);
    SolveView v;
    v.b = W;
    v.x = W + n;
    v.r = W + 2 * n;
    v.z = W + 3 * n;
    v.p = W + 4 * n;
    v.Ap = W + 5 * n;
    v.rhat = cs.bicg ? W + 6 * n : nullptr;
    v.ph = cs.bicg ? W + 7 * n : nullptr;
    v.sv = cs.bicg ? W + 8 * n : nullptr;
    v.shat = cs.bicg ? W + 9 * n : nullptr;
    v.t = cs.bicg ? W + 10 * n : nullptr;
    v.parts = W + nv * n;
    v.s = reinterpret_cast<CGScal *>(W + nv * n + 2 * cs.nblk);
    v.bs = reinterpret_cast<BiScal *>(v.s);
    // the scalar slots are multiples of 8 bytes: the FD workspace stays aligned
    v.fdt = reinterpret_cast<double *>(reinterpret_cast<char *>(v.s) + 2 * cgsolve_scal_bytes());
    v.fdparts = v.fdt + 2 * n;
    return v;
}

int cgsolve_begin(CgSolve &cs, yeti_wq_op *op, cudaStream_t st, void *host_scal,
                  const double *b_host, double rtol, int maxit, cudaStream_t capture,
                  int mode, int chunk) {
    YETI_CHECK(op && host_scal && b_host && op->coef64.ptr, YETI_EINVAL,
               "cgsolve_begin: missing operator data");
    YETI_CHECK(chunk >= 0 && chunk <= 256, YETI_EINVAL, "cgsolve_begin: chunk %d", chunk);
    const int fd_bits = YETI_PCG_FD | YETI_PCG_FD_SCALED | YETI_PCG_FD_UNIT | YETI_PCG_FD_TD;
    YETI_CHECK((mode & ~(fd_bits | YETI_PCG_BICGSTAB)) == 0 &&
                   ((mode & fd_bits) == 0 || (mode & YETI_PCG_FD)),
               YETI_EINVAL, "cgsolve_begin: mode %d", mode);
    YETI_TRY(ensure_dinv64(op));
    const bool fd = (mode & YETI_PCG_FD) != 0, bicg = (mode & YETI_PCG_BICGSTAB) != 0;
    if (fd) YETI_TRY(wq_fd_prepare(op, mode, false));
    cs.release();
    cs.op = op;
    cs.fd = fd;
    cs.bicg = bicg;
    cs.stream = st;
    cs.host_scal = host_scal;
    cs.chunk_iters = chunk ? chunk : kChunk;
    const int64_t n = op->ndof;
    cs.nblk = (int)std::max<int64_t>(1, std::min<int64_t>(kRedBlocks, (n + kRedThreads - 1) / kRedThreads));
    const size_t fd_doubles = fd ? 2 * (size_t)n + (size_t)wq_fd_parts(op) : 0;
    const size_t bytes = ((size_t)solve_vectors(bicg) * n + 2 * (size_t)cs.nblk + fd_doubles) *
                             sizeof(double) + 2 * cgsolve_scal_bytes();
    YETI_CUDA(cudaMallocAsync(&cs.dmem, bytes, st));
    const SolveView v = solve_view(cs);
    const double *dinv = op->dinv64.as<double>();
    const double *pre = fd ? nullptr : dinv;
    const int nb = cs.nblk;
    YETI_CUDA(cudaMemcpyAsync(v.b, b_host, n * sizeof(double), cudaMemcpyHostToDevice, st));
    YETI_CUDA(cudaMemsetAsync(v.x, 0, n * sizeof(double), st));
    YETI_CUDA(cudaMemsetAsync(v.s, 0, cgsolve_scal_bytes(), st));
    if (fd) {
        // the FD passes write the free boxes only: clamped entries stay 0
        for (double *w : {v.z, v.p, v.ph, v.shat})
            if (w) YETI_CUDA(cudaMemsetAsync(w, 0, n * sizeof(double), st));
    }
    k_mask<<<nb, kRedThreads, 0, st>>>(v.b, dinv, n);
    YETI_CUDA(cudaMemcpyAsync(v.r, v.b, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    if (!bicg) {
        k_dot<double, double><<<nb, kRedThreads, 0, st>>>(v.b, v.b, n, v.parts, nullptr);
        k_set_bb<<<1, kRedThreads, 0, st>>>(v.parts, nb, v.s);
        k_start<double><<<nb, kRedThreads, 0, st>>>(v.r, pre, v.z, v.p, v.Ap, n, v.parts);
        k_start_scal<<<1, kRedThreads, 0, st>>>(v.parts, nb, v.s, rtol * rtol, maxit);
        count_launches(5);
        if (fd)
            YETI_TRY(wq_fd_apply<double>(op, v.r, v.z, &v.s->done, FD_START, v.p, v.s, st, v.fdt,
                                         v.fdparts));
    } else {
        // rhat = r, p = r, ph = P r, v = 0 (v lives in Ap)
        k_bi_start<double><<<nb, kRedThreads, 0, st>>>(v.r, v.rhat, v.p, v.ph, v.Ap, pre, n,
                                                       v.parts);
        k_bi_start_scal_rel<<<1, kRedThreads, 0, st>>>(v.parts, nb, v.bs, rtol * rtol, maxit);
        count_launches(3);
        if (fd)
            YETI_TRY(wq_fd_apply<double>(op, v.r, v.ph, &v.bs->done, FD_NONE, nullptr, nullptr, st,
                                         v.fdt, v.fdparts));
    }
    YETI_CUDA(cudaGetLastError());
    // one chunk of iterations, captured once
    cudaGraph_t g = nullptr;
    cudaStream_t cap = capture ? capture : st;
    YETI_CUDA(cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal));
    int rc = YETI_OK;
    for (int k = 0; k < cs.chunk_iters && rc == YETI_OK; k++) {
        if (!bicg) {
            rc = wq_apply_dev(op, v.p, v.Ap, YETI_PREC_F64, &v.s->done, cap);
            k_dot_alpha<double><<<nb, kRedThreads, 0, cap>>>(v.p, v.Ap, n, v.parts, v.s);
            k_update_beta<double><<<nb, kRedThreads, 0, cap>>>(v.x, v.r, v.p, v.Ap, pre, v.z, n,
                                                              v.parts, v.s);
            if (fd && rc == YETI_OK)
                rc = wq_fd_apply<double>(op, v.r, v.z, &v.s->done, FD_ITER, nullptr, v.s, cap,
                                         v.fdt, v.fdparts);
            k_pupdate<double><<<nb, kRedThreads, 0, cap>>>(v.p, v.z, v.Ap, n, v.s);
        } else {
            // the BiCGSTAB iteration of bi_loop (v in Ap)
            BiScal *bs = v.bs;
            rc = wq_apply_dev(op, v.ph, v.Ap, YETI_PREC_F64, &bs->done, cap);
            k_dot<double, double><<<nb, kRedThreads, 0, cap>>>(v.rhat, v.Ap, n, v.parts, &bs->done);
            k_bi_alpha_s<double><<<1, kRedThreads, 0, cap>>>(v.parts, nb, bs);
            k_bi_s<double><<<nb, kRedThreads, 0, cap>>>(v.r, v.Ap, pre, v.sv, v.shat, v.t, n, bs);
            if (fd && rc == YETI_OK)
                rc = wq_fd_apply<double>(op, v.sv, v.shat, &bs->done, FD_NONE, nullptr, nullptr,
                                         cap, v.fdt, v.fdparts);
            if (rc == YETI_OK) rc = wq_apply_dev(op, v.shat, v.t, YETI_PREC_F64, &bs->done, cap);
            k_bi_ts<double><<<nb, kRedThreads, 0, cap>>>(v.t, v.sv, n, v.parts, bs);
            k_bi_omega<<<1, kRedThreads, 0, cap>>>(v.parts, nb, bs);
            k_bi_update<double><<<nb, kRedThreads, 0, cap>>>(v.x, v.r, v.rhat, v.ph, v.shat, v.sv,
                                                            v.t, n, v.parts, bs);
            k_bi_beta<<<1, kRedThreads, 0, cap>>>(v.parts, nb, bs);
            k_bi_p<double><<<nb, kRedThreads, 0, cap>>>(v.p, v.ph, v.r, v.Ap, pre, n, bs);
            if (fd && rc == YETI_OK)
                rc = wq_fd_apply<double>(op, v.p, v.ph, &bs->done, FD_NONE, nullptr, nullptr, cap,
                                         v.fdt, v.fdparts);
        }
    }
    cudaMemcpyAsync(cs.host_scal, v.s, cgsolve_scal_bytes(), cudaMemcpyDeviceToHost, cap);
    const cudaError_t ce = cudaStreamEndCapture(cap, &g);
    YETI_TRY(rc);
    YETI_CUDA(ce);
    const cudaError_t ie = cudaGraphInstantiate(&cs.chunk, g, 0);
    cudaGraphDestroy(g);
    YETI_CUDA(ie);
    YETI_CUDA(cudaEventCreateWithFlags(&cs.ev, cudaEventDisableTiming));
    return YETI_OK;
}

int cgsolve_launch(CgSolve &cs) {
    YETI_CUDA(cudaGraphLaunch(cs.chunk, cs.stream));
    YETI_CUDA(cudaEventRecord(cs.ev, cs.stream));
    count_launches((cs.bicg ? (cs.fd ? 20 : 10) : (cs.fd ? 9 : 4)) * cs.chunk_iters);
    cs.in_flight = true;
    return YETI_OK;
}

int cgsolve_poll(CgSolve &cs, int *state) {
    if (cs.in_flight) {
        const cudaError_t q = cudaEventQuery(cs.ev);
        if (q == cudaErrorNotReady) {
            *state = 0;
            return YETI_OK;
        }
        YETI_CUDA(q);
        cs.in_flight = false;
    }
    int iter, done, breakdown;
    if (cs.bicg) {
        const BiScal *h = static_cast<const BiScal *>(cs.host_scal);
        iter = h->iter;
        done = h->done;
        breakdown = h->breakdown;
    } else {
        const CGScal *h = static_cast<const CGScal *>(cs.host_scal);
        iter = h->iter;
        done = h->done;
        breakdown = h->breakdown;
    }
    cs.iterations = iter;
    *state = breakdown ? 3 : (done ? 2 : 1);
    return YETI_OK;
}

int cgsolve_finish(CgSolve &cs, double *x_host, cudaStream_t on) {
    const SolveView v = solve_view(cs);
    yeti_wq_op *op = cs.op;
    const int64_t n = op->ndof;
    const int nb = cs.nblk;
    cudaStream_t st = on ? on : cs.stream;
    if (on) YETI_CUDA(cudaStreamWaitEvent(on, cs.ev, 0));
    // true residual with the FP64 operator (Ap is free now)
    YETI_CUDA(cudaMemsetAsync(v.Ap, 0, n * sizeof(double), st));
    YETI_TRY(wq_apply_dev(op, v.x, v.Ap, YETI_PREC_F64, nullptr, st));
    k_residual<<<nb, kRedThreads, 0, st>>>(v.b, v.Ap, op->dinv64.as<double>(), v.r, n);
    k_dot<double, double><<<nb, kRedThreads, 0, st>>>(v.r, v.r, n, v.parts, nullptr);
    k_dot<double, double><<<nb, kRedThreads, 0, st>>>(v.b, v.b, n, v.parts + nb, nullptr);
    count_launches(3);
    std::vector<double> hp(2 * (size_t)nb);
    YETI_CUDA(cudaMemcpyAsync(hp.data(), v.parts, hp.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    YETI_CUDA(cudaMemcpyAsync(x_host, v.x, n * sizeof(double), cudaMemcpyDeviceToHost, st));
    YETI_CUDA(cudaStreamSynchronize(st));
    double rr = 0.0, bb = 0.0;
    for (int i = 0; i < nb; i++) {
        rr += hp[i];
        bb += hp[nb + i];
    }
    cs.rel_residual = bb > 0 ? std::sqrt(rr / bb) : 0.0;
    cs.release();
    return YETI_OK;
}

// Host sum of device partials (fixed order).
static int host_sum(yeti_wq_op *op, const double *parts, int n, int stride,
                    int off, double *out, bool take_max = false) {
    std::vector<double> hp((size_t)n * stride);
    YETI_CUDA(cudaMemcpyAsync(hp.data(), parts, hp.size() * sizeof(double),
                              cudaMemcpyDeviceToHost, op->ctx->stream));
    YETI_CUDA(cudaStreamSynchronize(op->ctx->stream));
    double acc = 0.0;
    for (int i = 0; i < n; i++)
        acc = take_max ? std::max(acc, hp[(size_t)i * stride + off]) : acc + hp[(size_t)i * stride + off];
    *out = acc;
    return YETI_OK;
}

}  // namespace yeti

using namespace yeti;

// History mode (relres != nullptr): FP64 only; every iteration records the
// reference's RelRes / RelError measures and the solve stops on its
// inf-norm test max|r| <= rtol max|b| instead of the 2-norm one.
static int pcg_run(yeti_wq_op *op, const double *b, double *x, double rtol, int maxit,
                   int mode, yeti_cg_stats *stats, int mem, const double *dsol,
                   double *relres, double *relerr) {
    YETI_CHECK(op && b && x, YETI_EINVAL, "yeti_wq_pcg: NULL argument");
    YETI_CHECK(mode >= 0 && mode < 64 &&
                   ((mode & (YETI_PCG_FD_SCALED | YETI_PCG_FD_UNIT | YETI_PCG_FD_TD)) == 0 ||
                    (mode & YETI_PCG_FD)) &&
                   !((mode & YETI_PCG_FD_UNIT) && (mode & YETI_PCG_FD_TD)),
               YETI_EINVAL, "yeti_wq_pcg: mode %d", mode);
    YETI_CHECK(rtol > 0 && maxit > 0, YETI_EINVAL, "yeti_wq_pcg: rtol %g maxit %d", rtol, maxit);
    YETI_CHECK(op->coef64.ptr, YETI_EINVAL,
               "yeti_wq_pcg: the FP64 operator is required (true residual)");
    const bool mixed = (mode & YETI_PCG_MIXED) != 0, bicg = (mode & YETI_PCG_BICGSTAB) != 0;
    const bool fd = (mode & YETI_PCG_FD) != 0;
    YETI_CHECK(!mixed || op->coef32.ptr, YETI_EINVAL,
               "yeti_wq_pcg: mixed precision needs the FP32 operator (YETI_WQ_F32)");
    const bool hist = relres != nullptr;
    YETI_CHECK(!hist || !mixed, YETI_EINVAL,
               "yeti_wq_pcg_history: the iteration history is recorded in FP64 only");
    DeviceGuard guard(op->ctx->device);
    YETI_TRY(ensure_workspace(op, mixed));
    if (fd) YETI_TRY(wq_fd_prepare(op, mode, mixed));
    cudaStream_t s = op->ctx->stream;
    const int64_t n = op->ndof;
    // history: 2 (maxit + 1) maxima, the reduction ticket, the direct solution
    DevBuf hbuf, dsbuf;
    double *dhist = nullptr, *dds = nullptr;
    unsigned int *hticket = nullptr;
    if (hist) {
        const size_t hbytes = (size_t)2 * (maxit + 1) * sizeof(double);
        YETI_TRY(hbuf.alloc(op->ctx, hbytes + 256));
        YETI_CUDA(cudaMemsetAsync(hbuf.ptr, 0, hbytes + 256, s));
        dhist = hbuf.as<double>();
        hticket = reinterpret_cast<unsigned int *>(hbuf.as<char>() + hbytes);
        if (dsol) {
            YETI_TRY(dsbuf.alloc(op->ctx, n * sizeof(double)));
            YETI_CUDA(cudaMemcpyAsync(dsbuf.ptr, dsol, n * sizeof(double),
                                      mem == YETI_MEM_HOST ? cudaMemcpyHostToDevice
                                                           : cudaMemcpyDeviceToDevice, s));
            dds = dsbuf.as<double>();
        }
    }
    double *W = op->ws64.as<double>();
    double *dx = W, *dr = W + n, *dz = W + 2 * n, *dp = W + 3 * n, *dAp = W + 4 * n,
           *db = W + 5 * n, *dt = W + 6 * n, *drh = W + 7 * n, *dph = W + 8 * n,
           *dsv = W + 9 * n, *dsh = W + 10 * n, *dtt = W + 11 * n;
    double *parts = op->parts.as<double>();
    CGScal *ds = op->scal.as<CGScal>();
    BiScal *bs = reinterpret_cast<BiScal *>(ds + 2);
    CGScal hs;
    BiScal hb;
    memset(&hs, 0, sizeof(hs));
    memset(&hb, 0, sizeof(hb));
    cudaEvent_t e0, e1;
    YETI_CUDA(cudaEventCreate(&e0));
    YETI_CUDA(cudaEventCreate(&e1));
    const cudaMemcpyKind h2d = mem == YETI_MEM_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    YETI_CUDA(cudaEventRecord(e0, s));
    YETI_CUDA(cudaMemcpyAsync(db, b, n * sizeof(double), h2d, s));
    YETI_CUDA(cudaMemcpyAsync(dx, x, n * sizeof(double), h2d, s));
    const double *dinv = op->dinv64.as<double>();
    // Jacobi: the kernels apply dinv; FD: nullptr, the FD passes give z
    const double *pre = fd ? nullptr : dinv;
    if (fd) {
        // the FD passes write the free boxes only: clamped entries stay 0
        for (double *v : {dz, dp, dph, dsh}) YETI_CUDA(cudaMemsetAsync(v, 0, n * sizeof(double), s));
        if (mixed)
            YETI_CUDA(cudaMemsetAsync(op->ws32.ptr, 0, 10 * n * sizeof(float), s));
    }
    k_mask<<<kRedBlocks, kRedThreads, 0, s>>>(db, dinv, n);
    k_mask<<<kRedBlocks, kRedThreads, 0, s>>>(dx, dinv, n);
    k_dot<double, double><<<kRedBlocks, kRedThreads, 0, s>>>(db, db, n, parts, nullptr);
    count_launches(3);
    double bb = 0.0;
    YETI_TRY(host_sum(op, parts, kRedBlocks, 1, 0, &bb));
    // r = b - A x
    YETI_CUDA(cudaMemsetAsync(dt, 0, n * sizeof(double), s));
    YETI_TRY(wq_apply_dev(op, dx, dt, YETI_PREC_F64, nullptr, s));
    k_residual<<<kRedBlocks, kRedThreads, 0, s>>>(db, dt, dinv, dr, n);
    count_launches(1);
    YETI_CUDA(cudaGetLastError());
    int iters = 0, outer = 0, f64 = 1, f32 = 0, status = YETI_OK;
    const double tol2 = rtol * rtol * bb;
    double bmax_h = 0.0, dsmax_h = 0.0, stop_abs = 0.0;
    if (hist) {
        k_absmax<double><<<kRedBlocks, kRedThreads, 0, s>>>(db, n, parts);
        count_launches(1);
        YETI_TRY(host_sum(op, parts, kRedBlocks, 1, 0, &bmax_h, true));
        if (dds) {
            k_absmax<double><<<kRedBlocks, kRedThreads, 0, s>>>(dds, n, parts);
            count_launches(1);
            YETI_TRY(host_sum(op, parts, kRedBlocks, 1, 0, &dsmax_h, true));
        }
        stop_abs = rtol * bmax_h;
    }
    if (!mixed && !bicg && hist) {
        // the reference's CG loop with its per-iteration measures: one
        // launch sequence per iteration (apply, alpha, updates, history with
        // the inf-norm stop test, preconditioner, direction)
        CGScal init;
        memset(&init, 0, sizeof(init));
        init.bb = bb;
        YETI_CUDA(cudaMemcpyAsync(ds, &init, sizeof(CGScal), cudaMemcpyHostToDevice, s));
        k_start<double><<<kRedBlocks, kRedThreads, 0, s>>>(dr, pre, dz, dp, dAp, n, parts);
        k_start_scal<<<1, kRedThreads, 0, s>>>(parts, kRedBlocks, ds, 0.0, maxit);
        k_hist<CGScal><<<kRedBlocks, kRedThreads, 0, s>>>(dr, dx, dds, n, parts, hticket, dhist, 0,
                                                         stop_abs, ds);
        count_launches(3);
        if (fd) YETI_TRY(wq_fd_apply<double>(op, dr, dz, &ds->done, FD_START, dp, ds, s));
        YETI_CUDA(cudaGetLastError());
        for (int g0 = 0;; g0 += kChunk) {
            for (int k = 0; k < kChunk; k++) {
                YETI_TRY(wq_apply_dev(op, dp, dAp, YETI_PREC_F64, &ds->done, s));
                k_dot_alpha<double><<<kRedBlocks, kRedThreads, 0, s>>>(dp, dAp, n, parts, ds);
                k_update_beta<double><<<kRedBlocks, kRedThreads, 0, s>>>(dx, dr, dp, dAp, pre, dz, n,
                                                                         parts, ds);
                k_hist<CGScal><<<kRedBlocks, kRedThreads, 0, s>>>(dr, dx, dds, n, parts, hticket,
                                                                 dhist, g0 + k + 1, stop_abs, ds);
                if (fd) YETI_TRY(wq_fd_apply<double>(op, dr, dz, &ds->done, FD_ITER, nullptr, ds, s));
                k_pupdate<double><<<kRedBlocks, kRedThreads, 0, s>>>(dp, dz, dAp, n, ds);
                count_launches(4);
            }
            YETI_CUDA(cudaGetLastError());
            YETI_CUDA(cudaMemcpyAsync(&hs, ds, sizeof(CGScal), cudaMemcpyDeviceToHost, s));
            YETI_CUDA(cudaStreamSynchronize(s));
            if (hs.done) break;
        }
        iters = hs.iter;
        f64 += hs.iter;
        if (hs.breakdown) status = YETI_EBREAKDOWN;
        outer = 1;
    } else if (!mixed && bicg && hist) {
        k_bi_start<double><<<kRedBlocks, kRedThreads, 0, s>>>(dr, drh, dp, dph, dAp, pre, n, parts);
        k_bi_start_scal<<<1, kRedThreads, 0, s>>>(parts, kRedBlocks, bs, 0.0, maxit);
        k_hist<BiScal><<<kRedBlocks, kRedThreads, 0, s>>>(dr, dx, dds, n, parts, hticket, dhist, 0,
                                                         stop_abs, bs);
        count_launches(3);
        if (fd) YETI_TRY(wq_fd_apply<double>(op, dr, dph, &bs->done, FD_NONE, nullptr, nullptr, s));
        YETI_CUDA(cudaGetLastError());
        for (int g0 = 0;; g0 += kChunk) {
            for (int k = 0; k < kChunk; k++) {
                YETI_TRY(wq_apply_dev(op, dph, dAp, YETI_PREC_F64, &bs->done, s));
                k_dot<double, double><<<kRedBlocks, kRedThreads, 0, s>>>(drh, dAp, n, parts, &bs->done);
                k_bi_alpha_s<double><<<1, kRedThreads, 0, s>>>(parts, kRedBlocks, bs);
                k_bi_s<double><<<kRedBlocks, kRedThreads, 0, s>>>(dr, dAp, pre, dsv, dsh, dtt, n, bs);
                if (fd) YETI_TRY(wq_fd_apply<double>(op, dsv, dsh, &bs->done, FD_NONE, nullptr, nullptr, s));
                YETI_TRY(wq_apply_dev(op, dsh, dtt, YETI_PREC_F64, &bs->done, s));
                k_bi_ts<double><<<kRedBlocks, kRedThreads, 0, s>>>(dtt, dsv, n, parts, bs);
                k_bi_omega<<<1, kRedThreads, 0, s>>>(parts, kRedBlocks, bs);
                k_bi_update<double><<<kRedBlocks, kRedThreads, 0, s>>>(dx, dr, drh, dph, dsh, dsv, dtt, n,
                                                                       parts, bs);
                k_bi_beta<<<1, kRedThreads, 0, s>>>(parts, kRedBlocks, bs);
                k_hist<BiScal><<<kRedBlocks, kRedThreads, 0, s>>>(dr, dx, dds, n, parts, hticket,
                                                                 dhist, g0 + k + 1, stop_abs, bs);
                k_bi_p<double><<<kRedBlocks, kRedThreads, 0, s>>>(dp, dph, dr, dAp, pre, n, bs);
                if (fd) YETI_TRY(wq_fd_apply<double>(op, dp, dph, &bs->done, FD_NONE, nullptr, nullptr, s));
                count_launches(9);
            }
            YETI_CUDA(cudaGetLastError());
            YETI_CUDA(cudaMemcpyAsync(&hb, bs, sizeof(BiScal), cudaMemcpyDeviceToHost, s));
            YETI_CUDA(cudaStreamSynchronize(s));
            if (hb.done) break;
        }
        iters = hb.iter;
        f64 += 2 * hb.iter;
        if (hb.breakdown) status = YETI_EBREAKDOWN;
        outer = 1;
    } else if (!mixed && !bicg) {
        CGScal init;
        memset(&init, 0, sizeof(init));
        init.bb = bb;
        YETI_CUDA(cudaMemcpyAsync(ds, &init, sizeof(CGScal), cudaMemcpyHostToDevice, s));
        k_start<double><<<kRedBlocks, kRedThreads, 0, s>>>(dr, pre, dz, dp, dAp, n, parts);
        k_start_scal<<<1, kRedThreads, 0, s>>>(parts, kRedBlocks, ds, rtol * rtol, maxit);
        count_launches(2);
        if (fd) YETI_TRY(wq_fd_apply<double>(op, dr, dz, &ds->done, FD_START, dp, ds, s));
        YETI_CUDA(cudaGetLastError());
        YETI_TRY(cg_loop<double>(op, YETI_PREC_F64, dx, dr, dz, dp, dAp, pre, ds, &hs));
        iters = hs.iter;
        f64 += hs.iter;
        if (hs.breakdown) status = YETI_EBREAKDOWN;
        outer = 1;
    } else if (!mixed && bicg) {
        k_bi_start<double><<<kRedBlocks, kRedThreads, 0, s>>>(dr, drh, dp, dph, dAp, pre, n, parts);
        k_bi_start_scal<<<1, kRedThreads, 0, s>>>(parts, kRedBlocks, bs, tol2, maxit);
        count_launches(2);
        if (fd) YETI_TRY(wq_fd_apply<double>(op, dr, dph, &bs->done, FD_NONE, nullptr, nullptr, s));
        YETI_CUDA(cudaGetLastError());
        YETI_TRY(bi_loop<double>(op, YETI_PREC_F64, dx, dr, drh, dp, dph, dAp, dsv, dsh, dtt, pre, bs, &hb));
        iters = hb.iter;
        f64 += 2 * hb.iter;
        if (hb.breakdown) status = YETI_EBREAKDOWN;
        outer = 1;
    } else if (mixed && !bicg) {
        // FP32 CG with reliable updates: the Krylov iteration runs in FP32
        // and is never restarted; whenever its recursive residual has
        // dropped 100x (or reached the tolerance), the solution correction is
        // folded into the FP64 solution, the true residual is recomputed with
        // the FP64 operator and replaces the FP32 one (search direction kept,
        // rescaled).
        float *V = op->ws32.as<float>();
        float *r32 = V, *z32 = V + n, *p32 = V + 2 * n, *Ap32 = V + 3 * n, *d32 = V + 4 * n;
        const float *dinv32 = fd ? nullptr : op->dinv32.as<float>();
        const double delta2 = 1e-4;   // replace when ||r|| fell by 100x
        // with FD: on the device, when ||r|| fell by 100x (FP32 tracks that)
        const double kFdPause2 = 1e-4;
        double rr64 = 0.0;
        k_dot<double, double><<<kRedBlocks, kRedThreads, 0, s>>>(dr, dr, n, parts, nullptr);
        count_launches(1);
        YETI_TRY(host_sum(op, parts, kRedBlocks, 1, 0, &rr64));
        double sc = std::sqrt(rr64);
        if (rr64 > tol2 && rr64 == rr64) {
            k_to_f32<<<kRedBlocks, kRedThreads, 0, s>>>(dr, r32, d32, n, 1.0 / sc);
            k_start<float><<<kRedBlocks, kRedThreads, 0, s>>>(r32, dinv32, z32, p32, Ap32, n, parts);
            CGScal init;
            memset(&init, 0, sizeof(init));
            init.bb = 1.0;
            // FD converges by decades per chunk, past what the FP32
            // recursion tracks: stop the chunk on the device for a
            // replacement at every 100x drop
            init.pause2 = fd ? kFdPause2 : 0.0;
            YETI_CUDA(cudaMemcpyAsync(ds, &init, sizeof(CGScal), cudaMemcpyHostToDevice, s));
            k_start_scal<<<1, kRedThreads, 0, s>>>(parts, kRedBlocks, ds, tol2 / rr64, maxit);
            count_launches(3);
            if (fd) YETI_TRY(wq_fd_apply<float>(op, r32, z32, &ds->done, FD_START, p32, ds, s));
            YETI_CUDA(cudaGetLastError());
            double rr_ref = 1.0;
            for (;;) {
                YETI_TRY(cg_chunk<float>(op, YETI_PREC_F32, d32, r32, z32, p32, Ap32, dinv32, ds, fd));
                YETI_CUDA(cudaMemcpyAsync(&hs, ds, sizeof(CGScal), cudaMemcpyDeviceToHost, s));
                YETI_CUDA(cudaStreamSynchronize(s));
                const int it = hs.iter;
                if (hs.breakdown) { iters = it; status = YETI_EBREAKDOWN; break; }
                if (!(hs.done || hs.rr <= delta2 * rr_ref)) continue;
                // reliable update
                k_ru_accum<<<kRedBlocks, kRedThreads, 0, s>>>(dx, d32, n, sc);
                YETI_CUDA(cudaMemsetAsync(dt, 0, n * sizeof(double), s));
                YETI_TRY(wq_apply_dev(op, dx, dt, YETI_PREC_F64, nullptr, s));
                k_residual<<<kRedBlocks, kRedThreads, 0, s>>>(db, dt, dinv, dr, n);
                k_dot<double, double><<<kRedBlocks, kRedThreads, 0, s>>>(dr, dr, n, parts, nullptr);
                count_launches(3);
                f64++;
                outer++;
                YETI_TRY(host_sum(op, parts, kRedBlocks, 1, 0, &rr64));
                iters = it;
                if (!(rr64 == rr64)) { status = YETI_EBREAKDOWN; break; }
                if (rr64 <= tol2 || it >= maxit) break;
                const double sc_new = std::sqrt(rr64);
                // a replacement after the FP32 recursion met the tolerance
                // restarts the direction (its last update was skipped); after
                // a pause the iteration was complete and the direction stays
                const int restart = (hs.done && !hs.paused) ? 1 : 0;
                k_ru_replace<<<kRedBlocks, kRedThreads, 0, s>>>(dr, r32, z32, p32, dinv32, n,
                                                                1.0 / sc_new, (float)(sc / sc_new),
                                                                restart, parts);
                k_ru_scal<<<1, kRedThreads, 0, s>>>(parts, kRedBlocks, ds, tol2 / rr64, maxit);
                count_launches(2);
                if (fd)
                    YETI_TRY(wq_fd_apply<float>(op, r32, z32, &ds->done,
                                                restart ? FD_START : FD_REPLACE, p32, ds, s));
                YETI_CUDA(cudaGetLastError());
                sc = sc_new;
                rr_ref = 1.0;
            }
            f32 = iters;
        }
    } else {
        // mixed BiCGSTAB: FP32 inner solves, FP64 residual and refinement
        float *V = op->ws32.as<float>();
        float *r32 = V, *rh = V + n, *p32 = V + 2 * n, *ph = V + 3 * n, *v32 = V + 4 * n,
              *sv = V + 5 * n, *shh = V + 6 * n, *t32 = V + 7 * n, *d32 = V + 8 * n;
        const float *dinv32 = fd ? nullptr : op->dinv32.as<float>();
        const double eta2 = 1e-8;   // inner relative tolerance 1e-4
        for (outer = 0; outer < 50; outer++) {
            double rr64 = 0.0;
            k_dot<double, double><<<kRedBlocks, kRedThreads, 0, s>>>(dr, dr, n, parts, nullptr);
            count_launches(1);
            YETI_TRY(host_sum(op, parts, kRedBlocks, 1, 0, &rr64));
            if (!(rr64 == rr64)) { status = YETI_EBREAKDOWN; break; }
            if (rr64 <= tol2 || iters >= maxit) break;
            const double sc = 1.0 / std::sqrt(rr64);
            k_to_f32<<<kRedBlocks, kRedThreads, 0, s>>>(dr, r32, d32, n, sc);
            k_bi_start<float><<<kRedBlocks, kRedThreads, 0, s>>>(r32, rh, p32, ph, v32, dinv32, n, parts);
            k_bi_start_scal<<<1, kRedThreads, 0, s>>>(parts, kRedBlocks, bs, eta2, maxit - iters);
            count_launches(3);
            if (fd) YETI_TRY(wq_fd_apply<float>(op, r32, ph, &bs->done, FD_NONE, nullptr, nullptr, s));
            YETI_TRY(bi_loop<float>(op, YETI_PREC_F32, d32, r32, rh, p32, ph, v32, sv, shh, t32, dinv32, bs, &hb));
            iters += hb.iter;
            f32 += 2 * hb.iter;
            k_refine<<<kRedBlocks, kRedThreads, 0, s>>>(dx, d32, n, 1.0 / sc);
            YETI_CUDA(cudaMemsetAsync(dt, 0, n * sizeof(double), s));
            YETI_TRY(wq_apply_dev(op, dx, dt, YETI_PREC_F64, nullptr, s));
            k_residual<<<kRedBlocks, kRedThreads, 0, s>>>(db, dt, dinv, dr, n);
            count_launches(2);
            YETI_CUDA(cudaGetLastError());
            f64++;
            if (hb.breakdown && hb.iter == 0) { status = YETI_EBREAKDOWN; break; }
        }
    }
    YETI_CUDA(cudaEventRecord(e1, s));
    // true FP64 residual of the returned solution
    YETI_CUDA(cudaMemsetAsync(dt, 0, n * sizeof(double), s));
    YETI_TRY(wq_apply_dev(op, dx, dt, YETI_PREC_F64, nullptr, s));
    k_residual<<<kRedBlocks, kRedThreads, 0, s>>>(db, dt, dinv, dr, n);
    k_dot<double, double><<<kRedBlocks, kRedThreads, 0, s>>>(dr, dr, n, parts, nullptr);
    count_launches(2);
    double rr = 0.0, rmax = 0.0, bmax = 0.0;
    YETI_TRY(host_sum(op, parts, kRedBlocks, 1, 0, &rr));
    k_absmax<double><<<kRedBlocks, kRedThreads, 0, s>>>(dr, n, parts);
    count_launches(1);
    YETI_TRY(host_sum(op, parts, kRedBlocks, 1, 0, &rmax, true));
    k_absmax<double><<<kRedBlocks, kRedThreads, 0, s>>>(db, n, parts);
    count_launches(1);
    YETI_TRY(host_sum(op, parts, kRedBlocks, 1, 0, &bmax, true));
    float ms = 0.f;
    YETI_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    const cudaMemcpyKind d2h = mem == YETI_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    YETI_CUDA(cudaMemcpyAsync(x, dx, n * sizeof(double), d2h, s));
    YETI_CUDA(cudaStreamSynchronize(s));
    YETI_TRY(wq_stream_check(op));
    const double rel = bb > 0 ? std::sqrt(rr / bb) : 0.0;
    if (hist) {
        std::vector<double> h((size_t)2 * (iters + 1));
        YETI_CUDA(cudaMemcpy(h.data(), dhist, h.size() * sizeof(double), cudaMemcpyDeviceToHost));
        for (int k = 0; k <= iters; k++) {
            relres[k] = bmax_h > 0 ? h[2 * k] / bmax_h : 0.0;
            if (relerr) relerr[k] = dsmax_h > 0 ? h[2 * k + 1] / dsmax_h : 0.0;
        }
        const double rinf = bmax > 0 ? rmax / bmax : 0.0;
        if (status == YETI_OK && !(rinf <= rtol)) status = YETI_ENOTCONV;
    } else if (status == YETI_OK && !(rel <= rtol)) {
        status = YETI_ENOTCONV;
    }
    if (stats) {
        stats->iterations = iters;
        stats->outer_iterations = outer;
        stats->fp64_applies = f64;
        stats->fp32_applies = f32;
        stats->rel_residual = rel;
        stats->rel_residual_inf = bmax > 0 ? rmax / bmax : 0.0;
        stats->solve_ms = ms;
        stats->status = status;
    }
    if (status == YETI_EBREAKDOWN) {
        set_error("yeti_wq_pcg: Krylov breakdown after %d iterations", iters);
        return status;
    }
    return YETI_OK;
}

YETI_API int yeti_wq_pcg(yeti_wq_op *op, const double *b, double *x, double rtol, int maxit,
                         int mode, yeti_cg_stats *stats, int mem) {
    return pcg_run(op, b, x, rtol, maxit, mode, stats, mem, nullptr, nullptr, nullptr);
}

YETI_API int yeti_wq_pcg_history(yeti_wq_op *op, const double *b, double *x, double rtol,
                                 int maxit, int mode, const double *directsol, double *relres,
                                 double *relerr, yeti_cg_stats *stats, int mem) {
    YETI_CHECK(relres, YETI_EINVAL, "yeti_wq_pcg_history: NULL relres");
    return pcg_run(op, b, x, rtol, maxit, mode, stats, mem, directsol, relres, relerr);
}
