// One-dimensional weighted-quadrature rule (host side).
#pragma once
#include <vector>

namespace yeti {

// Dense row-major (nfun x nqp) matrices of one direction.  B0/B1: basis
// values/derivatives at the WQ points; Wxy: weights for test derivative
// order x and trial derivative order y.  lo/hi: 0-based inclusive point
// range stored for each function (the reference's B1 support shape).
struct WQRule1D {
    int p = 0, nel = 0, nfun = 0, nqp = 0;
    std::vector<double> x;
    std::vector<double> B0, B1, W00, W01, W10, W11;
    std::vector<int> lo, hi;
};

int wq_npts(int p, int nel);
int wq_rule_1d(int p, int nel, WQRule1D &out);
void gauss_legendre_host(int n, double *x, double *w);

}  // namespace yeti
