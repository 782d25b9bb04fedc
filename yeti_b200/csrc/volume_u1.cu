// Volume of U1 solid patches and its analytic gradient with respect to the
// control-point coordinates.
//
// Replaces optim.volume.computevolume / computegradvolume: computeVolume
// (src/yeti_iga/optim/volume.f90:20-210) and computeGradVolume
// (src/yeti_iga/optim/gradvolume.f90:16-355), the 3-D classical-patch
// branches, called by OPTmodelling.compute_volume / compute_gradVolume_AN
// (preprocessing/igaparametrization/OPT_modelling.py:508-531).  At each Gauss
// point of an element, with the covariant vectors A_k = sum_i dR_i/dxi_k P_i,
//     V      += det[A_1 A_2 A_3] w_q J_param
//     dV/dP_i += (A_1 x A_2 dR_i/dxi_3 + A_2 x A_3 dR_i/dxi_1
//                 + A_3 x A_1 dR_i/dxi_2) w_q J_param
// (the determinant signed, as MatrixDet, operateurs.f:513-559).
//
// Kernel design: one thread per (element, Gauss point) writes the point's
// volume term and its gradient terms per node; the rational basis is
// evaluated three times in the thread (sums, covariant vectors, gradient
// terms) instead of being stored, so any element size fits in registers.
// Two gather kernels then sum the terms in the reference's order (elements,
// then points), so the result does not depend on thread timing.  Compiled
// without FMA contraction, in the reference's operation order.
#include <algorithm>
#include <cmath>
#include <memory>
#include <vector>

#include "nurbs.cuh"
#include "u1_model.cuh"

namespace yeti {

struct VolArgs {
    int p0, p1, p2, nn, nq;
    const double *U0, *U1, *U2;
    const double *gauss;    // 4 * nq: weight, parent coordinates
    const double *coords;   // (3, nb_cp)
    const int32_t *ien;     // nelem * nn, 0-based
    const double *w;        // nelem * nn element weights
    const int32_t *span;    // nelem * 3, 1-based
    int64_t nelem;
    double *vterm;          // nelem * nq
    double *gterm;          // nelem * nq * nn * 3 (nullptr: volume only)
};

// Unnormalised tensor-product value and derivatives of local node n.
struct BasisRow {
    double FN[kMaxDeg1], dFN[kMaxDeg1], FM[kMaxDeg1], dFM[kMaxDeg1], FL[kMaxDeg1],
        dFL[kMaxDeg1];
};

__global__ void __launch_bounds__(128) k_u1_volume(VolArgs a) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= a.nelem * a.nq) return;
    const int64_t e = t / a.nq;
    const int q = (int)(t % a.nq);
    const int32_t *sp = a.span + 3 * e;
    const int ni[3] = {sp[0], sp[1], sp[2]};
    const double *U[3] = {a.U0, a.U1, a.U2};
    const double *g = a.gauss + 4 * q;
    double xi[3], detJ = g[0];
    for (int d = 0; d < 3; d++) {
        const double u1 = U[d][ni[d] - 1], u2 = U[d][ni[d]];
        xi[d] = ((u2 - u1) * g[1 + d] + (u2 + u1)) * 0.5;
        detJ = detJ * 0.5 * (u2 - u1);
    }
    BasisRow B;
    bspline_ders(ni[0], a.p0, xi[0], a.U0, B.FN, B.dFN);
    bspline_ders(ni[1], a.p1, xi[1], a.U1, B.FM, B.dFM);
    bspline_ders(ni[2], a.p2, xi[2], a.U2, B.FL, B.dFL);
    const double *we = a.w + e * a.nn;
    const int32_t *ie = a.ien + e * a.nn;
    // pass 1: the sums of the rational normalisation (evalnurbs order)
    double S = 0.0, sx[3] = {0.0, 0.0, 0.0};
    {
        int n = 0;
        for (int k = 0; k <= a.p2; k++)
            for (int j = 0; j <= a.p1; j++)
                for (int i = 0; i <= a.p0; i++, n++) {
                    S = S + B.FN[a.p0 - i] * B.FM[a.p1 - j] * B.FL[a.p2 - k] * we[n];
                    sx[0] = sx[0] + B.dFN[a.p0 - i] * B.FM[a.p1 - j] * B.FL[a.p2 - k] * we[n];
                    sx[1] = sx[1] + B.FN[a.p0 - i] * B.dFM[a.p1 - j] * B.FL[a.p2 - k] * we[n];
                    sx[2] = sx[2] + B.FN[a.p0 - i] * B.FM[a.p1 - j] * B.dFL[a.p2 - k] * we[n];
                }
    }
    const double inv = 1.0 / S;
    // dR/dxi of node n, recomputed with the same operations as pass 1
    auto dR = [&](int n, int i, int j, int k, double out[3]) {
        const double R = B.FN[a.p0 - i] * B.FM[a.p1 - j] * B.FL[a.p2 - k] * we[n] * inv;
        const double d0 = B.dFN[a.p0 - i] * B.FM[a.p1 - j] * B.FL[a.p2 - k] * we[n];
        const double d1 = B.FN[a.p0 - i] * B.dFM[a.p1 - j] * B.FL[a.p2 - k] * we[n];
        const double d2 = B.FN[a.p0 - i] * B.FM[a.p1 - j] * B.dFL[a.p2 - k] * we[n];
        out[0] = (d0 - R * sx[0]) * inv;
        out[1] = (d1 - R * sx[1]) * inv;
        out[2] = (d2 - R * sx[2]) * inv;
    };
    // pass 2: covariant vectors AI(:, k) = sum_n dR(n, k) X_n
    double AI[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};   // AI[c][k]
    {
        int n = 0;
        for (int k = 0; k <= a.p2; k++)
            for (int j = 0; j <= a.p1; j++)
                for (int i = 0; i <= a.p0; i++, n++) {
                    double d[3];
                    dR(n, i, j, k, d);
                    const double *X = a.coords + 3 * (int64_t)ie[n];
                    for (int kk = 0; kk < 3; kk++)
                        for (int c = 0; c < 3; c++) AI[c][kk] = AI[c][kk] + d[kk] * X[c];
                }
    }
    // signed determinant in MatrixDet's order (AA(i, j) = AI[i-1][j-1])
    const double det = AI[0][1] * AI[1][2] * AI[2][0] - AI[0][2] * AI[1][1] * AI[2][0] +
                       AI[0][2] * AI[1][0] * AI[2][1] - AI[0][0] * AI[1][2] * AI[2][1] +
                       AI[0][0] * AI[1][1] * AI[2][2] - AI[0][1] * AI[1][0] * AI[2][2];
    a.vterm[t] = det * detJ;
    if (!a.gterm) return;
    // cofactor columns: c3 = A1 x A2, c1 = A2 x A3, c2 = A3 x A1
    double c1[3], c2[3], c3[3];
    auto cross = [](const double *u, const double *v, double *w) {
        w[0] = u[1] * v[2] - u[2] * v[1];
        w[1] = u[2] * v[0] - u[0] * v[2];
        w[2] = u[0] * v[1] - u[1] * v[0];
    };
    const double A1[3] = {AI[0][0], AI[1][0], AI[2][0]};
    const double A2[3] = {AI[0][1], AI[1][1], AI[2][1]};
    const double A3[3] = {AI[0][2], AI[1][2], AI[2][2]};
    cross(A1, A2, c3);
    cross(A2, A3, c1);
    cross(A3, A1, c2);
    double *gt = a.gterm + t * (int64_t)a.nn * 3;
    int n = 0;
    for (int k = 0; k <= a.p2; k++)
        for (int j = 0; j <= a.p1; j++)
            for (int i = 0; i <= a.p0; i++, n++) {
                double d[3];
                dR(n, i, j, k, d);
                for (int c = 0; c < 3; c++)
                    gt[3 * n + c] = (c3[c] * d[2] + c1[c] * d[0] + c2[c] * d[1]) * detJ;
            }
}

// vol = sum of the terms in order (the reference's running sum).  The
// block brings the terms into shared memory in coalesced chunks; one thread
// adds them in order, from shared memory, while nothing else is waited for.
constexpr int kVolChunk = 4096;
__global__ void __launch_bounds__(1024) k_volume_sum(const double *vterm, int64_t n, double *vol) {
    __shared__ double buf[kVolChunk];
    double v = 0.0;
    for (int64_t c0 = 0; c0 < n; c0 += kVolChunk) {
        const int m = (int)(n - c0 < kVolChunk ? n - c0 : kVolChunk);
        __syncthreads();
        for (int i = threadIdx.x; i < m; i += blockDim.x) buf[i] = vterm[c0 + i];
        __syncthreads();
        if (threadIdx.x == 0) {
            int i = 0;
            for (; i + 8 <= m; i += 8) {
                const double t0 = buf[i], t1 = buf[i + 1], t2 = buf[i + 2], t3 = buf[i + 3];
                const double t4 = buf[i + 4], t5 = buf[i + 5], t6 = buf[i + 6], t7 = buf[i + 7];
                v = v + t0;
                v = v + t1;
                v = v + t2;
                v = v + t3;
                v = v + t4;
                v = v + t5;
                v = v + t6;
                v = v + t7;
            }
            for (; i < m; i++) v = v + buf[i];
        }
    }
    if (threadIdx.x == 0) *vol = v;
}

// grad[j] = sum over the terms idx[ptr[j] .. ptr[j+1]) in order
// grad[c + 3 cp] = sum, over the active elements holding cp (in element
// order) and their points q (in order), of the point term of (q, a, c), a the
// control point's local index: ent[k] is the term of (q = 0, a, c = 0) of the
// k-th element of cp, qs[k] = (points, term stride between points).
__global__ void k_volume_gather(int64_t n, const int64_t *ptr, const int64_t *ent,
                                const int2 *qs, const double *gterm, double *grad) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int64_t cp = t / 3;
    const int c = (int)(t - 3 * cp);
    double acc = 0.0;
    for (int64_t k = ptr[cp]; k < ptr[cp + 1]; k++) {
        const double *g = gterm + ent[k] + c;
        const int nq = qs[k].x;
        const int64_t st = qs[k].y;
        for (int q = 0; q < nq; q++) acc = acc + g[q * st];
    }
    grad[t] = acc;
}

}  // namespace yeti

using namespace yeti;

YETI_API int yeti_volume_u1(yeti_ctx *ctx, const yeti_u1_model *m, double *vol,
                            double *grad, int mem) {
    YETI_CHECK(ctx && m && vol, YETI_EINVAL, "yeti_volume_u1: NULL argument");
    DeviceGuard guard(ctx->device);
    U1Model M;
    YETI_TRY(u1_prepare(ctx, m, M));
    cudaStream_t s = ctx->stream;
    const int64_t ncp = m->nb_cp;
    const bool want_grad = grad != nullptr;
    // terms of every active element's points, patches in order
    struct Seg {
        size_t patch;
        int64_t off;   // first (element, point) term
    };
    std::vector<Seg> segs;
    int64_t nterm = 0, ngterm = 0;
    for (size_t ip = 0; ip < M.patches.size(); ip++) {
        const U1Patch &P = M.patches[ip];
        if (!P.nactive) continue;
        segs.push_back({ip, nterm});
        nterm += P.nactive * P.nq;
        ngterm += P.nactive * P.nq * P.nn * 3;
    }
    DevBuf dv, dvt, dgt, dgrad, dptr, didx, dqs;
    YETI_TRY(dv.alloc(ctx, sizeof(double)));
    if (nterm == 0) {
        *vol = 0.0;
        if (want_grad) {
            if (mem == YETI_MEM_HOST) std::fill(grad, grad + 3 * ncp, 0.0);
            else YETI_CUDA(cudaMemsetAsync(grad, 0, 3 * ncp * sizeof(double), s));
            YETI_CUDA(cudaStreamSynchronize(s));
        }
        return YETI_OK;
    }
    YETI_TRY(dvt.alloc(ctx, nterm * sizeof(double)));
    if (want_grad) YETI_TRY(dgt.alloc(ctx, ngterm * sizeof(double)));
    int64_t goff = 0;
    for (const Seg &sg : segs) {
        const U1Patch &P = M.patches[sg.patch];
        VolArgs a;
        a.p0 = P.p[0];
        a.p1 = P.p[1];
        a.p2 = P.p[2];
        a.nn = P.nn;
        a.nq = P.nq;
        a.U0 = P.knots.as<double>();
        a.U1 = a.U0 + P.nkv[0];
        a.U2 = a.U1 + P.nkv[1];
        a.gauss = P.gauss.as<double>();
        a.coords = M.coords.as<double>();
        a.ien = P.ien.as<int32_t>();
        a.w = P.w.as<double>();
        a.span = P.span.as<int32_t>();
        a.nelem = P.nactive;
        a.vterm = dvt.as<double>() + sg.off;
        a.gterm = want_grad ? dgt.as<double>() + goff : nullptr;
        const int64_t nt = P.nactive * P.nq;
        k_u1_volume<<<(unsigned)((nt + 127) / 128), 128, 0, s>>>(a);
        count_launches(1);
        YETI_CUDA(cudaGetLastError());
        goff += nt * P.nn * 3;
    }
    k_volume_sum<<<1, 1024, 0, s>>>(dvt.as<double>(), nterm, dv.as<double>());
    count_launches(1);
    YETI_CUDA(cudaGetLastError());
    if (want_grad) {
        // per control point: the active elements holding it, in element
        // order (the three components and the points of each element are
        // walked by the gather kernel in the same order)
        const int64_t nout = 3 * ncp;
        std::vector<int64_t> patch_ien(M.patches.size(), 0);
        int64_t ien_off = 0;
        for (size_t ip = 0; ip < M.patches.size(); ip++) {
            patch_ien[ip] = ien_off;
            ien_off += M.patches[ip].nelem * M.patches[ip].nn;
        }
        auto cp_of = [&](const U1Patch &P, size_t ip, int64_t le, int a) {
            const int64_t jel = P.act[le];
            return m->ien[patch_ien[ip] + (jel - P.elem_begin) * P.nn + a] - 1;
        };
        std::vector<int64_t> cnt(ncp + 1, 0);
        for (const Seg &sg : segs) {
            const U1Patch &P = M.patches[sg.patch];
            for (int64_t le = 0; le < P.nactive; le++)
                for (int a = 0; a < P.nn; a++) cnt[cp_of(P, sg.patch, le, a) + 1]++;
        }
        for (int64_t i = 0; i < ncp; i++) cnt[i + 1] += cnt[i];
        const size_t nent = (size_t)std::max<int64_t>(cnt[ncp], 1);
        std::vector<int64_t> ent(nent, 0), fill(cnt.begin(), cnt.end() - 1);
        std::vector<int2> qs(nent, make_int2(0, 0));
        int64_t base = 0;
        for (const Seg &sg : segs) {
            const U1Patch &P = M.patches[sg.patch];
            for (int64_t le = 0; le < P.nactive; le++)
                for (int a = 0; a < P.nn; a++) {
                    const int64_t k = fill[cp_of(P, sg.patch, le, a)]++;
                    ent[k] = base + (le * P.nq * (int64_t)P.nn + a) * 3;
                    qs[k] = make_int2(P.nq, P.nn * 3);
                }
            base += P.nactive * P.nq * P.nn * 3;
        }
        YETI_TRY(upload(ctx, dptr, cnt.data(), cnt.size()));
        YETI_TRY(upload(ctx, didx, ent.data(), ent.size()));
        YETI_TRY(upload(ctx, dqs, qs.data(), qs.size()));
        double *g_d = grad;
        if (mem == YETI_MEM_HOST) {
            YETI_TRY(dgrad.alloc(ctx, nout * sizeof(double)));
            g_d = dgrad.as<double>();
        }
        k_volume_gather<<<(unsigned)((nout + 255) / 256), 256, 0, s>>>(
            nout, dptr.as<int64_t>(), didx.as<int64_t>(), dqs.as<int2>(), dgt.as<double>(), g_d);
        count_launches(1);
        YETI_CUDA(cudaGetLastError());
        if (mem == YETI_MEM_HOST)
            YETI_CUDA(cudaMemcpyAsync(grad, g_d, nout * sizeof(double), cudaMemcpyDeviceToHost, s));
    }
    YETI_CUDA(cudaMemcpyAsync(vol, dv.ptr, sizeof(double), cudaMemcpyDeviceToHost, s));
    YETI_CUDA(cudaStreamSynchronize(s));
    return YETI_OK;
}
