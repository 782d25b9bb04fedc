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

// Gauss-Legendre nodes/weights of order n on [-1, 1] (ascending): roots of
// the Legendre polynomial P_n by Newton iteration on its recurrence.
void gauss_legendre_host(int n, double *x, double *w);

// Volume rule with the reference's ordering (GaussLegendre.f90:175-187):
// g[4q] = weight, g[4q+1..3] = parent coordinates, xi1 slowest.
void gauss_volume_host(int n, std::vector<double> &g);
// Face rule of face 1..6 (GaussLegendre.f90:217-270).
void gauss_face_host(int n, int face, std::vector<double> &g);

}  // namespace yeti
