// One-dimensional weighted-quadrature (WQ) rule, host side.
//
// Follows the reference's Fortran rule (src/yeti_iga/iga_wq_mf/fsrc/
// iga_wq_methods.f90): uniform open knot vector with nel elements, r = 2,
// maxrule = 1, quadrature points = the knots plus p interior points in the two
// boundary elements and one midpoint in each interior element
// (wq_get_qp_positions, :38-89).  For every test function i the weights W
// solve sum_q W[i,q] B[a,q] = integral(B_a * test_i) exactly for all trial
// functions a whose support meets i's, on the points of i's support
// (wq_get_quadrature_rule_row, :330-376), for the four (test, trial)
// derivative pairings W00, W01, W10, W11 (wq_get_basis_weights_generalized,
// :420-599).  Meshes with more than p+3 elements copy the rules of a
// (p+3)-element model and rescale them (wq_get_basis_weights_model,
// :601-650; wq_get_basis_weights, :852-1011).  The small dense systems are
// solved by Householder QR: least squares when overdetermined, minimum-norm
// when underdetermined (the dgels/dgesv split of algebra.f90:87-167).
#include <algorithm>
#include <cmath>
#include <deque>
#include <map>
#include <mutex>
#include <utility>
#include <vector>

#include "wq_rule.h"

namespace yeti {

int wq_npts(int p, int nel) { return 2 * (p + 2) + nel * 2 - 2 - 3; }

namespace {

constexpr double kSpanTol = 1e-8;   // constants_iga_wq_mf (algebra.f90:11-13)
constexpr double kTol = 1e-15;

// 1-based knot span of x in a (p, nfun) open knot vector, the search of
// find_knotvector_span (bspline.f90:34-57).
int find_knot_span(int p, int nfun, const std::vector<double> &kv, double x) {
    int span = p + 2;
    while (span < nfun + 1 && (kv[span - 1] - x) <= kSpanTol) span++;
    return span - 1;
}

// 1-based element of x (find_parametric_span, bspline.f90:59-83).
int find_elem(int nel, const std::vector<double> &nodes, double x) {
    int span = 2;
    while (span < nel + 1 && (nodes[span - 1] - x) <= kSpanTol) span++;
    return span - 1;
}

// B-spline values and derivatives (The NURBS Book A2.3, one derivative).
void ders(int ni, int p, double u, const std::vector<double> &U, double *N,
          double *dN) {
    std::vector<std::vector<double>> ndu(p + 1, std::vector<double>(p + 1));
    std::vector<double> left(p + 2), right(p + 2);
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
    for (int r = 0; r <= p; r++) {
        double d = 0.0;
        if (p >= 1) {
            if (r >= 1) d = ndu[r - 1][p - 1] / ndu[p][r - 1];
            if (r <= p - 1) d -= ndu[r][p - 1] / ndu[p][r];
        }
        dN[r] = d * p;
    }
}

std::vector<double> uniform_nodes(int nel) {
    std::vector<double> n(nel + 1);
    n[0] = 0.0;
    n[nel] = 1.0;
    for (int i = 1; i < nel; i++) n[i] = double(i) / double(nel);
    return n;
}

std::vector<double> open_knots(int p, const std::vector<double> &nodes) {
    int nel = (int)nodes.size() - 1;
    std::vector<double> kv;
    for (int i = 0; i <= p; i++) kv.push_back(0.0);
    for (int i = 1; i < nel; i++) kv.push_back(nodes[i]);
    for (int i = 0; i <= p; i++) kv.push_back(1.0);
    return kv;
}

// Dense (nfun x npts) basis values / derivatives at points x (get_basis,
// bspline.f90:200-258).
void eval_basis(int p, int nel, const std::vector<double> &nodes,
                const std::vector<double> &x, std::vector<double> &B0,
                std::vector<double> &B1) {
    const int nfun = p + nel;
    const int npts = (int)x.size();
    std::vector<double> kv = open_knots(p, nodes);
    B0.assign((size_t)nfun * npts, 0.0);
    B1.assign((size_t)nfun * npts, 0.0);
    std::vector<double> N(p + 1), dN(p + 1);
    for (int q = 0; q < npts; q++) {
        int el = find_elem(nel, nodes, x[q]);          // 1-based
        int ks = find_knot_span(p, nfun, kv, x[q]);    // 1-based
        ders(ks, p, x[q], kv, N.data(), dN.data());
        for (int j = 0; j <= p; j++) {
            int f = (el - 1) + j;                      // table_functions_span
            B0[(size_t)f * npts + q] = N[j];
            B1[(size_t)f * npts + q] = dN[j];
        }
    }
}

// Householder QR solve of the m x n system A x = b (row-major A):
// least squares for m >= n, minimum norm for m < n.
void lsq_solve(int m, int n, std::vector<double> A, std::vector<double> b,
               double *x) {
    auto qr = [](int rows, int cols, std::vector<double> &M,
                 std::vector<double> &beta) {
        // in-place Householder on columns of M (rows x cols, row-major)
        beta.assign(cols, 0.0);
        for (int k = 0; k < cols; k++) {
            double nrm = 0.0;
            for (int i = k; i < rows; i++) nrm += M[i * cols + k] * M[i * cols + k];
            nrm = std::sqrt(nrm);
            if (nrm == 0.0) continue;
            double a = M[k * cols + k];
            double alpha = a > 0 ? -nrm : nrm;
            double v0 = a - alpha;
            // v = [v0, M[k+1..,k]], normalised so v[0] = 1
            for (int i = k + 1; i < rows; i++) M[i * cols + k] /= v0;
            beta[k] = -v0 / alpha;   // 2 / (v^T v) with v[0] = 1
            M[k * cols + k] = alpha;
            for (int j = k + 1; j < cols; j++) {
                double s = M[k * cols + j];
                for (int i = k + 1; i < rows; i++) s += M[i * cols + k] * M[i * cols + j];
                s *= beta[k];
                M[k * cols + j] -= s;
                for (int i = k + 1; i < rows; i++) M[i * cols + j] -= s * M[i * cols + k];
            }
        }
    };
    std::vector<double> beta;
    if (m >= n) {
        qr(m, n, A, beta);
        // b <- Q^T b
        for (int k = 0; k < n; k++) {
            double s = b[k];
            for (int i = k + 1; i < m; i++) s += A[i * n + k] * b[i];
            s *= beta[k];
            b[k] -= s;
            for (int i = k + 1; i < m; i++) b[i] -= s * A[i * n + k];
        }
        for (int k = n - 1; k >= 0; k--) {
            double s = b[k];
            for (int j = k + 1; j < n; j++) s -= A[k * n + j] * x[j];
            x[k] = s / A[k * n + k];
        }
    } else {
        // A^T = Q R  (n x m);  x = Q [R^{-T} b; 0]
        std::vector<double> At((size_t)n * m);
        for (int i = 0; i < m; i++)
            for (int j = 0; j < n; j++) At[j * m + i] = A[i * n + j];
        qr(n, m, At, beta);
        std::vector<double> y(n, 0.0);
        for (int k = 0; k < m; k++) {
            double s = b[k];
            for (int j = 0; j < k; j++) s -= At[j * m + k] * y[j];
            y[k] = s / At[k * m + k];
        }
        for (int k = m - 1; k >= 0; k--) {
            double s = y[k];
            for (int i = k + 1; i < n; i++) s += At[i * m + k] * y[i];
            s *= beta[k];
            y[k] -= s;
            for (int i = k + 1; i < n; i++) y[i] -= s * At[i * m + k];
        }
        for (int j = 0; j < n; j++) x[j] = y[j];
    }
}

// B0 / B1 supports of each function, 0-based inclusive point ranges
// (wq_get_B0_B1_shape, iga_wq_methods.f90:200-292).
void supports(int p, int nel, int nqp, std::vector<int> &b0lo,
              std::vector<int> &b0hi, std::vector<int> &b1lo,
              std::vector<int> &b1hi) {
    const int nfun = p + nel;
    // points of each element (1-based inclusive in the Fortran)
    std::vector<int> s0(nel), s1(nel);
    s0[0] = 1;
    s1[0] = p + 2;
    if (nel > 1) {
        s0[nel - 1] = nqp + 1 - (p + 2);
        s1[nel - 1] = nqp;
    }
    for (int i = 1; i < nel - 1; i++) {
        s0[i] = s1[i - 1];
        s1[i] = s0[i] + 2;
    }
    b0lo.resize(nfun); b0hi.resize(nfun); b1lo.resize(nfun); b1hi.resize(nfun);
    for (int i = 0; i < nfun; i++) {
        int smin = std::max(0, i - p), smax = std::min(nel - 1, i);
        int lo = s0[smin], hi = s1[smax];
        int l0 = lo, h0 = hi, l1 = lo, h1 = hi;
        if (i == 0) h0 -= 1;
        else if (i == nfun - 1) l0 += 1;
        else { h0 -= 1; l0 += 1; }
        if (i == 0 || i == 1) h1 -= 1;
        else if (i == nfun - 1 || i == nfun - 2) l1 += 1;
        else { h1 -= 1; l1 += 1; }
        b0lo[i] = l0 - 1; b0hi[i] = h0 - 1;
        b1lo[i] = l1 - 1; b1hi[i] = h1 - 1;
    }
}

// Rules for all nfun functions from basis MB (nrows x nqp) at the WQ points
// and exact integrals MI (nrows x nfun), restricted to support B0 of each
// function (wq_get_quadrature_rules, iga_wq_methods.f90:378-418).
void rules(int nrows, int nfun, int nqp, const std::vector<double> &MB,
           const std::vector<double> &MI, const std::vector<int> &Mint,
           const std::vector<int> &lo, const std::vector<int> &hi,
           std::vector<double> &out) {
    out.assign((size_t)nfun * nqp, 0.0);
    for (int i = 0; i < nfun; i++) {
        int fmin = 0, fmax = nrows - 1;
        for (int j = 0; j < nrows; j++)
            if (Mint[(size_t)j * nfun + i] > 0) { fmin = j; break; }
        for (int j = nrows - 1; j >= 0; j--)
            if (Mint[(size_t)j * nfun + i] > 0) { fmax = j; break; }
        const int m = fmax - fmin + 1, n = hi[i] - lo[i] + 1;
        std::vector<double> A((size_t)m * n), b(m);
        for (int r = 0; r < m; r++) {
            for (int c = 0; c < n; c++)
                A[(size_t)r * n + c] = MB[(size_t)(fmin + r) * nqp + lo[i] + c];
            b[r] = MI[(size_t)(fmin + r) * nfun + i];
        }
        lsq_solve(m, n, A, b, &out[(size_t)i * nqp + lo[i]]);
    }
}

}  // namespace


// WQ point positions (wq_get_qp_positions, iga_wq_methods.f90:38-89): the
// p+2 equidistant points of each boundary element and the 3 equidistant
// points (knots + midpoint) of each interior element, shared knots once.
std::vector<double> wq_points(int p, int nel, const std::vector<double> &nodes) {
    const int nqp = wq_npts(p, nel);
    std::vector<double> x(nqp, 0.0);
    auto linspace = [](double a, double b, int n, double *o) {
        double h = (b - a) / double(n - 1);
        o[0] = a;
        o[n - 1] = b;
        for (int i = 1; i < n - 1; i++) o[i] = a + double(i) * h;
    };
    std::vector<double> t(p + 2);
    linspace(nodes[0], nodes[1], p + 2, t.data());
    for (int j = 0; j < p + 2; j++) x[j] = t[j];
    linspace(nodes[nel - 1], nodes[nel], p + 2, t.data());
    for (int j = 0; j < p + 2; j++) x[nqp - (p + 2) + j] = t[j];
    double u[3];
    for (int i = 1; i < nel - 1; i++) {
        linspace(nodes[i], nodes[i + 1], 3, u);
        for (int j = 0; j < 3; j++) x[(p + 2) + 2 * (i - 1) + j - 1] = u[j];
    }
    return x;
}

// Direct computation for any nel (wq_get_basis_weights_generalized).
static void wq_rule_generalized(int p, int nel, WQRule1D &R) {
    const int nfun = p + nel, nqp = wq_npts(p, nel);
    std::vector<double> nodes = uniform_nodes(nel);
    R.p = p; R.nel = nel; R.nfun = nfun; R.nqp = nqp;
    R.x = wq_points(p, nel, nodes);
    // Gauss points: p+1 per element (iga_get_qp_positions_weights, :92-126)
    double xg[32], wg[32];
    gauss_legendre_host(p + 1, xg, wg);
    const int ncgg = (p + 1) * nel;
    std::vector<double> xc(ncgg), wc(ncgg);
    for (int i = 0; i < nel; i++)
        for (int j = 0; j <= p; j++) {
            xc[i * (p + 1) + j] = 0.5 * (xg[j] / double(nel) + nodes[i + 1] + nodes[i]);
            wc[i * (p + 1) + j] = 0.5 / double(nel) * wg[j];
        }
    std::vector<double> B0c, B1c, B0c1, B1c1, B0w1, B1w1;
    eval_basis(p, nel, nodes, xc, B0c, B1c);
    eval_basis(p, nel, nodes, R.x, R.B0, R.B1);
    const int nfun1 = p - 1 + nel;
    eval_basis(p - 1, nel, nodes, xc, B0c1, B1c1);
    eval_basis(p - 1, nel, nodes, R.x, B0w1, B1w1);
    std::vector<int> b0lo, b0hi, b1lo, b1hi;
    supports(p, nel, nqp, b0lo, b0hi, b1lo, b1hi);
    R.lo = b1lo;
    R.hi = b1hi;
    auto product_awb = [&](const std::vector<double> &A, int ra,
                           const std::vector<double> &B, int rb) {
        std::vector<double> M((size_t)ra * rb, 0.0);
        for (int i = 0; i < ra; i++)
            for (int j = 0; j < rb; j++) {
                double s = 0.0;
                for (int k = 0; k < ncgg; k++)
                    s += A[(size_t)i * ncgg + k] * wc[k] * B[(size_t)j * ncgg + k];
                M[(size_t)i * rb + j] = s;
            }
        return M;
    };
    auto pattern = [&](const std::vector<double> &A, int ra,
                       const std::vector<double> &B, int rb) {
        std::vector<int> M((size_t)ra * rb, 0);
        for (int i = 0; i < ra; i++)
            for (int j = 0; j < rb; j++) {
                int s = 0;
                for (int k = 0; k < ncgg; k++)
                    s += (std::fabs(A[(size_t)i * ncgg + k]) > kTol) &&
                         (std::fabs(B[(size_t)j * ncgg + k]) > kTol);
                M[(size_t)i * rb + j] = s;
            }
        return M;
    };
    std::vector<int> I0 = pattern(B0c, nfun, B0c, nfun);
    rules(nfun, nfun, nqp, R.B0, product_awb(B0c, nfun, B0c, nfun), I0, b0lo, b0hi, R.W00);
    rules(nfun, nfun, nqp, R.B0, product_awb(B0c, nfun, B1c, nfun), I0, b0lo, b0hi, R.W10);
    std::vector<int> I1 = pattern(B0c1, nfun1, B0c, nfun);
    rules(nfun1, nfun, nqp, B0w1, product_awb(B0c1, nfun1, B0c, nfun), I1, b0lo, b0hi, R.W01);
    rules(nfun1, nfun, nqp, B0w1, product_awb(B0c1, nfun1, B1c, nfun), I1, b0lo, b0hi, R.W11);
}

static int wq_rule_1d_compute(int p, int nel, WQRule1D &R) {
    if (p < 1 || nel < 2) return -1;
    if (nel <= p + 3) {
        wq_rule_generalized(p, nel, R);
        return 0;
    }
    // (p+3)-element model, rescaled to nel (wq_get_basis_weights_model)
    WQRule1D M;
    const int nm = p + 3;
    wq_rule_generalized(p, nm, M);
    const double up = double(nel) / double(nm), dn = double(nm) / double(nel);
    const int nfun = p + nel, nqp = wq_npts(p, nel);
    std::vector<int> b0lo, b0hi, b1lo, b1hi;
    supports(p, nel, nqp, b0lo, b0hi, b1lo, b1hi);
    R.p = p; R.nel = nel; R.nfun = nfun; R.nqp = nqp;
    R.lo = b1lo;
    R.hi = b1hi;
    R.x = wq_points(p, nel, uniform_nodes(nel));
    const size_t sz = (size_t)nfun * nqp;
    R.B0.assign(sz, 0.0); R.B1.assign(sz, 0.0);
    R.W00.assign(sz, 0.0); R.W01.assign(sz, 0.0);
    R.W10.assign(sz, 0.0); R.W11.assign(sz, 0.0);
    const int mq = M.nqp;
    auto put = [&](int i, int j, int mi, int mj, double sgn) {
        size_t o = (size_t)i * nqp + j, mo = (size_t)mi * mq + mj;
        R.B0[o] = M.B0[mo];
        R.B1[o] = sgn * M.B1[mo] * up;
        R.W00[o] = M.W00[mo] * dn;
        R.W01[o] = M.W01[mo] * dn;
        R.W10[o] = sgn * M.W10[mo];
        R.W11[o] = sgn * M.W11[mo];
    };
    for (int i = 0; i <= p; i++)                       // first p+1 functions
        for (int j = b1lo[i]; j <= b1hi[i]; j++) put(i, j, i, j, 1.0);
    const int mid = p + 1;                             // model row p+2 (1-based)
    const int width = M.hi[mid] - M.lo[mid] + 1;
    for (int i = p + 1; i <= nfun - p - 2; i++)        // repeated functions
        for (int j = 0; j < width; j++) put(i, b1lo[i] + j, mid, M.lo[mid] + j, 1.0);
    for (int i = 0; i <= p; i++)                       // last p+1, mirrored
        for (int j = b1lo[i]; j <= b1hi[i]; j++)
            put(nfun - 1 - i, nqp - 1 - j, i, j, -1.0);
    return 0;
}

// The rule depends on (p, nel) only.  Operators built back to back (the
// serving loop sets up one per request, over a few dozen distinct sizes)
// reuse the rules of earlier ones: a bounded cache of the rules of up to 512
// elements per direction, evicted oldest first.
int wq_rule_1d(int p, int nel, WQRule1D &R) {
    constexpr int kMaxCachedNel = 512;
    constexpr size_t kMaxEntries = 256;
    static std::mutex mtx;
    static std::map<std::pair<int, int>, WQRule1D> cache;
    static std::deque<std::pair<int, int>> order;
    const auto key = std::make_pair(p, nel);
    if (nel <= kMaxCachedNel) {
        std::lock_guard<std::mutex> lock(mtx);
        auto it = cache.find(key);
        if (it != cache.end()) {
            R = it->second;
            return 0;
        }
    }
    const int rc = wq_rule_1d_compute(p, nel, R);
    if (rc == 0 && nel <= kMaxCachedNel) {
        std::lock_guard<std::mutex> lock(mtx);
        if (cache.emplace(key, R).second) {
            order.push_back(key);
            if (order.size() > kMaxEntries) {
                cache.erase(order.front());
                order.pop_front();
            }
        }
    }
    return rc;
}

}  // namespace yeti

// ------------------------------------------------------------------ C ABI
#include "common.cuh"

YETI_API int yeti_wq_rule_1d_size(int p, int nel, int32_t *nfun,
                                  int32_t *nqp) {
    YETI_CHECK(p >= 1 && p <= 10 && nel >= 2 && nel <= (1 << 20),
               YETI_EINVAL, "yeti_wq_rule_1d_size: p=%d nel=%d", p, nel);
    if (nfun) *nfun = p + nel;
    if (nqp) *nqp = yeti::wq_npts(p, nel);
    return YETI_OK;
}

YETI_API int yeti_wq_rule_1d(int p, int nel, double *x, double *B0,
                             double *B1, double *W00, double *W01,
                             double *W10, double *W11) {
    YETI_TRY(yeti_wq_rule_1d_size(p, nel, nullptr, nullptr));
    YETI_CHECK(nel <= 4096, YETI_EINVAL,
               "yeti_wq_rule_1d: dense output limited to nel <= 4096");
    yeti::WQRule1D R;
    YETI_CHECK(yeti::wq_rule_1d(p, nel, R) == 0, YETI_EINVAL,
               "yeti_wq_rule_1d: rule construction failed");
    const size_t n = (size_t)R.nfun * R.nqp;
    if (x) std::copy(R.x.begin(), R.x.end(), x);
    if (B0) std::copy(R.B0.begin(), R.B0.begin() + n, B0);
    if (B1) std::copy(R.B1.begin(), R.B1.begin() + n, B1);
    if (W00) std::copy(R.W00.begin(), R.W00.begin() + n, W00);
    if (W01) std::copy(R.W01.begin(), R.W01.begin() + n, W01);
    if (W10) std::copy(R.W10.begin(), R.W10.begin() + n, W10);
    if (W11) std::copy(R.W11.begin(), R.W11.begin() + n, W11);
    return YETI_OK;
}
