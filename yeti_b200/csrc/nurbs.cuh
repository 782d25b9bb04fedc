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

// Gauss-Legendre nodes/weights of order n on [-1, 1] (ascending): roots of
// the Legendre polynomial P_n by Newton iteration on its recurrence.
void gauss_legendre_host(int n, double *x, double *w);

// Volume rule with the reference's ordering (GaussLegendre.f90:175-187):
// g[4q] = weight, g[4q+1..3] = parent coordinates, xi1 slowest.
void gauss_volume_host(int n, std::vector<double> &g);
// Face rule of face 1..6 (GaussLegendre.f90:217-270).
void gauss_face_host(int n, int face, std::vector<double> &g);

}  // namespace yeti
