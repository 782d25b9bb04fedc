// NURBS helpers shared by the Gauss-quadrature kernels (assembly, gradient).
#pragma once
#include <cmath>

#include "common.cuh"

namespace yeti {

constexpr int kMaxDeg = 8;            // maximum degree per direction
constexpr int kMaxDeg1 = kMaxDeg + 1;

// B-spline values N[0..p] and first derivatives dN[0..p] of the p+1
// functions nonzero on knot span `ni` (1-based, the reference's Nijk
// convention) at u: the Cox-de Boor triangle of The NURBS Book A2.3 with one
// derivative (the algorithm of dersbasisfuns.f90:30-131).
__host__ __device__ inline void bspline_ders(int ni, int p, double u,
                                             const double *U, double *N,
                                             double *dN) {
    double ndu[kMaxDeg1][kMaxDeg1];
    double left[kMaxDeg1 + 1], right[kMaxDeg1 + 1];
    ndu[0][0] = 1.0;
    for (int j = 1; j <= p; j++) {
        left[j] = u - U[ni - j];
        right[j] = U[ni + j - 1] - u;
        double saved = 0.0;
        for (int r = 0; r < j; r++) {
            ndu[j][r] = right[r + 1] + left[j - r];
            double temp = ndu[r][j - 1] / ndu[j][r];
            ndu[r][j] = saved + right[r + 1] * temp;
            saved = left[j - r] * temp;
        }
        ndu[j][j] = saved;
    }
    for (int j = 0; j <= p; j++) N[j] = ndu[j][p];
    // first derivatives in the reciprocal form of the reference's k-loop
    // (dersbasisfuns.f90:79-124 with nders = 1)
    for (int r = 0; r <= p; r++) {
        double d = 0.0;
        if (p >= 1) {
            if (r >= 1) {
                double a = 1.0 / ndu[p][r - 1];
                d = a * ndu[r - 1][p - 1];
            }
            if (r <= p - 1) {
                double a = -1.0 / ndu[p][r];
                d = d + a * ndu[r][p - 1];
            }
        }
        dN[r] = d * (double)p;
    }
}

// Rational basis R[nn] and its parametric derivatives dR[3 a + i] of one
// element at xi: the tensor product with reversed 1-D indices (the
// descending local node order of the reference's IEN), times the element's
// weights, then divided by their sum (evalnurbs,
// src/yeti_iga/main/evaluatenurbsfcts.f:94-209, in its operation order).
__device__ inline void nurbs_eval_elem(int p0, int p1, int p2, const double *U0,
                                       const double *U1, const double *U2, int nn,
                                       const int *ni, const double *xi, const double *we,
                                       double *R, double *dR) {
    double FN[kMaxDeg1], dFN[kMaxDeg1], FM[kMaxDeg1], dFM[kMaxDeg1], FL[kMaxDeg1],
        dFL[kMaxDeg1];
    bspline_ders(ni[0], p0, xi[0], U0, FN, dFN);
    bspline_ders(ni[1], p1, xi[1], U1, FM, dFM);
    bspline_ders(ni[2], p2, xi[2], U2, FL, dFL);
    int n = 0;
    double S = 0.0, sx0 = 0.0, sx1 = 0.0, sx2 = 0.0;
    for (int k = 0; k <= p2; k++)
        for (int j = 0; j <= p1; j++)
            for (int i = 0; i <= p0; i++, n++) {
                R[n] = FN[p0 - i] * FM[p1 - j] * FL[p2 - k] * we[n];
                S = S + R[n];
                dR[3 * n] = dFN[p0 - i] * FM[p1 - j] * FL[p2 - k] * we[n];
                sx0 = sx0 + dR[3 * n];
                dR[3 * n + 1] = FN[p0 - i] * dFM[p1 - j] * FL[p2 - k] * we[n];
                sx1 = sx1 + dR[3 * n + 1];
                dR[3 * n + 2] = FN[p0 - i] * FM[p1 - j] * dFL[p2 - k] * we[n];
                sx2 = sx2 + dR[3 * n + 2];
            }
    const double inv = 1.0 / S;
    const double sx[3] = {sx0, sx1, sx2};
    for (int q = 0; q < nn; q++) {
        R[q] = R[q] * inv;
        for (int i = 0; i < 3; i++) dR[3 * q + i] = (dR[3 * q + i] - R[q] * sx[i]) * inv;
    }
}

constexpr int kStiffQS = 16;              // scalars per point of basis_chunk
constexpr int kBasisB1 = 6 * kMaxDeg1;    // 1-D rows per point of basis_chunk

// Stage A of the Gauss kernels for a chunk of points q0..q0+nqc-1
// (shap.f90:75-178, evalnurbs, evaluatenurbsfcts.f:94-209): the 1-D B-spline
// rows (B1, kBasisB1 per point), the rational numerators R0[ql rs + n] and
// dR/dxi at dR[ql ds + 3 n + c] of every (point, node), the per-point sums
// of the derivative numerators (qs[0..2]), 1/S (qs[3]) and dx/dxi
// (qs[4 + 3 r + c]), kStiffQS scalars per point.  The products of every (point, node) are formed in
// parallel; each sum over the nodes stays one thread's loop in node order,
// so the values are those of the point-serial evaluation bit for bit.
__device__ inline void basis_chunk(const int pd[3], const double *const Ud[3], const int *sni,
                                   const double *su1, const double *su2, const double *gauss,
                                   int q0, int nqc, int nn, const double *xe, const double *we,
                                   double *B1, double *R0, int rs, double *dR, int ds,
                                   double *qs) {
    const int tid = threadIdx.x, nth = blockDim.x;
    const int p0 = pd[0], p1 = pd[1], p2 = pd[2];
    // A1: 1-D B-spline values and derivatives, one thread per (point, dir)
    for (int t = tid; t < 3 * nqc; t += nth) {
        const int ql = t / 3, d = t - 3 * ql;
        const double tq = gauss[4 * (q0 + ql) + 1 + d];
        const double xi = ((su2[d] - su1[d]) * tq + (su2[d] + su1[d])) * 0.5;
        double *f = B1 + ((size_t)ql * 6 + 2 * d) * kMaxDeg1;
        bspline_ders(sni[d], pd[d], xi, Ud[d], f, f + kMaxDeg1);
    }
    __syncthreads();
    // A2: the four numerator products of every (point, node)
    for (int t = tid; t < nqc * nn; t += nth) {
        const int ql = t / nn, n = t - ql * nn;
        const int i = n % (p0 + 1), j = (n / (p0 + 1)) % (p1 + 1), k = n / ((p0 + 1) * (p1 + 1));
        const double *f = B1 + (size_t)ql * 6 * kMaxDeg1;
        const double FN = f[p0 - i], dFN = f[kMaxDeg1 + p0 - i];
        const double FM = f[2 * kMaxDeg1 + p1 - j], dFM = f[3 * kMaxDeg1 + p1 - j];
        const double FL = f[4 * kMaxDeg1 + p2 - k], dFL = f[5 * kMaxDeg1 + p2 - k];
        const double wa = we[n];
        R0[(size_t)ql * rs + n] = FN * FM * FL * wa;
        double *d = dR + (size_t)ql * ds + 3 * n;
        d[0] = dFN * FM * FL * wa;
        d[1] = FN * dFM * FL * wa;
        d[2] = FN * FM * dFL * wa;
    }
    __syncthreads();
    // A3: the sums over the nodes (one thread per (point, sum), node order)
    for (int t = tid; t < 4 * nqc; t += nth) {
        const int ql = t >> 2, c = t & 3;
        double acc = 0.0;
        if (c == 0) {
            const double *r = R0 + (size_t)ql * rs;
            for (int n = 0; n < nn; n++) acc += r[n];
            qs[(size_t)ql * kStiffQS + 3] = 1.0 / acc;
        } else {
            const double *d = dR + (size_t)ql * ds + (c - 1);
            for (int n = 0; n < nn; n++) acc += d[3 * n];
            qs[(size_t)ql * kStiffQS + c - 1] = acc;
        }
    }
    __syncthreads();
    // A4: rational derivatives dR/dxi, one thread per (point, node)
    for (int t = tid; t < nqc * nn; t += nth) {
        const int ql = t / nn, n = t - ql * nn;
        const double *sq = qs + (size_t)ql * kStiffQS;
        const double inv = sq[3];
        const double R = R0[(size_t)ql * rs + n] * inv;
        double *d = dR + (size_t)ql * ds + 3 * n;
        d[0] = (d[0] - R * sq[0]) * inv;
        d[1] = (d[1] - R * sq[1]) * inv;
        d[2] = (d[2] - R * sq[2]) * inv;
    }
    __syncthreads();
    // A5: dx/dxi, one thread per (point, entry), node order
    for (int t = tid; t < 9 * nqc; t += nth) {
        const int ql = t / 9, rc = t - 9 * ql, r = rc / 3, c = rc - 3 * r;
        const double *d = dR + (size_t)ql * ds + c;
        double acc = 0.0;
        for (int n = 0; n < nn; n++) acc += xe[3 * n + r] * d[3 * n];
        qs[(size_t)ql * kStiffQS + 4 + rc] = acc;
    }
    __syncthreads();
}

// Gauss-Legendre nodes/weights of order n on [-1, 1] (ascending): roots of
// the Legendre polynomial P_n by Newton iteration on its recurrence.
void gauss_legendre_host(int n, double *x, double *w);

// Volume rule with the reference's ordering (GaussLegendre.f90:175-187):
// g[4q] = weight, g[4q+1..3] = parent coordinates, xi1 slowest.
void gauss_volume_host(int n, std::vector<double> &g);
// Face rule of face 1..6 (GaussLegendre.f90:217-270).
void gauss_face_host(int n, int face, std::vector<double> &g);

}  // namespace yeti
