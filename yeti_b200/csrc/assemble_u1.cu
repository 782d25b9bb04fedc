// U1 solid element stiffness and COO assembly on the GPU.
//
// Replaces stiffmtrx_elemstorage.sys_linmat_lindef_static
// (src/yeti_iga/main/build_system_elemStorage.f90:24-315) and the element
// routine UELMAT_byCP (src/yeti_iga/main/UELMAT.f90:22-225) with its helpers
// shap (shap.f90:21-180), stiffmatrix_byCP (stiffmatrix.F90:130-225),
// material_lib (material_lib.f90:75-87) and shapPress (shapPress.f:18-262).
//
// Kernel design: one CTA per element.  Stage A: one thread per Gauss point
// evaluates the rational basis derivatives dR/dx (3 x nnode) and the volume
// weight into shared memory.  Stage B: one thread per control-point pair
// (i <= j) accumulates the 3x3 block over the Gauss points and writes its 9
// (or 6, diagonal) COO entries at the reference's slot positions, so the
// writes of consecutive threads are contiguous.  Elements whose Gauss data do
// not fit shared memory are processed in Gauss-point chunks (read-modify-write
// of the element's own slots).  The load vector is a second kernel over the
// elements that carry distributed loads.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>

#include "nurbs.cuh"
#include "u1_model.cuh"

namespace yeti {

// ---------------------------------------------------------------- Gauss rules
/* Gauss-Legendre rules of orders 1..9 on [-1, 1]: the nodes of the upper
 * half (ascending, x >= 0) and their weights, as tabulated by the reference
 * (GaussLegendre.f90:41-153, 30 significant digits; these are the standard
 * published values of the rules, rounded to double by the compiler).  The
 * lower half mirrors them exactly; the order-3 weights are the divisions
 * 5/9 and 8/9, as the reference writes them. */
static const double kGLX[10][5] = {
    {0, 0, 0, 0, 0},
    {0.0},
    {0.577350269189625764509148780502},
    {0.0, 0.774596669241483377035853079956},
    {0.339981043584856264802665759103, 0.861136311594052575223946488893},
    {0.0, 0.538469310105683091036314420700, 0.906179845938663992797626878299},
    {0.238619186083196908630501721681, 0.661209386466264513661399595020,
     0.932469514203152027812301554494},
    {0.0, 0.405845151377397166906606412077, 0.741531185599394439863864773281,
     0.949107912342758524526189684048},
    {0.183434642495649804939476142360, 0.525532409916328985817739049189,
     0.796666477413626739591553936476, 0.960289856497536231683560868569},
    {0.0, 0.324253423403808929038538014643, 0.613371432700590397308702039341,
     0.836031107326635794299429788070, 0.968160239507626089835576202904},
};
static const double kGLW[10][5] = {
    {0, 0, 0, 0, 0},
    {2.0},
    {1.0},
    {0.0, 0.0},   /* 8/9, 5/9: computed */
    {0.652145154862546142626936050778, 0.347854845137453857373063949222},
    {0.568888888888888888888888888889, 0.478628670499366468041291514836,
     0.236926885056189087514264040720},
    {0.467913934572691047389870343990, 0.360761573048138607569833513838,
     0.171324492379170345040296142173},
    {0.417959183673469387755102040816, 0.381830050505118944950369775489,
     0.279705391489276667901467771424, 0.129484966168869693270611432679},
    {0.362683783378361982965150449277, 0.313706645877887287337962201987,
     0.222381034453374470544355994426, 0.101228536290376259152531354310},
    {0.330239355001259763164525069287, 0.312347077040002840068630406584,
     0.260610696402935462318742869419, 0.180648160694857404058472031243,
     0.812743883615744119718921581105e-01},
};

/* Rule of order n from the table (1 <= n <= 9): ascending nodes x[0..n-1]. */
static void gauss_table(int n, double *x, double *w)
{
    for (int j = 0; j < (n + 1) / 2; j++) {
        const double xv = kGLX[n][j];
        const double wv = n == 3 ? (j == 0 ? 8.0 / 9.0 : 5.0 / 9.0) : kGLW[n][j];
        const int hi = n / 2 + j;                              /* x >= 0 */
        const int lo = n % 2 ? n / 2 - j : n / 2 - 1 - j;      /* mirror */
        x[lo] = -xv;
        w[lo] = wv;
        x[hi] = xv;   /* odd n, j = 0: the centre, +0.0 as tabulated */
        w[hi] = wv;
    }
}

// Gauss-Legendre rule of order n on [-1, 1] (Gauss, GaussLegendre.f90:27-153):
// the table for orders 1..9; beyond, where the reference has no rule, the
// roots of P_n by Newton iteration on the three-term recurrence with the
// weights 2/((1-x^2) P_n'(x)^2).
void gauss_legendre_host(int n, double *x, double *w) {
    if (n >= 1 && n <= 9) {
        gauss_table(n, x, w);
        return;
    }
    for (int i = 0; i < n; i++) {
        double z = -std::cos(M_PI * (i + 0.75) / (n + 0.5));
        double pp = 1.0;
        for (int it = 0; it < 100; it++) {
            double p1 = 1.0, p2 = 0.0;
            for (int k = 1; k <= n; k++) {
                double p3 = p2;
                p2 = p1;
                p1 = ((2.0 * k - 1.0) * z * p2 - (k - 1.0) * p3) / k;
            }
            pp = n * (z * p1 - p2) / (z * z - 1.0);
            double dz = p1 / pp;
            z -= dz;
            if (std::fabs(dz) < 1e-17) break;
        }
        double p1 = 1.0, p2 = 0.0;
        for (int k = 1; k <= n; k++) {
            double p3 = p2;
            p2 = p1;
            p1 = ((2.0 * k - 1.0) * z * p2 - (k - 1.0) * p3) / k;
        }
        pp = n * (z * p1 - p2) / (z * z - 1.0);
        x[i] = z;
        w[i] = 2.0 / ((1.0 - z * z) * pp * pp);
    }
    for (int i = 0; i < n / 2; i++) {
        double a = 0.5 * (x[n - 1 - i] - x[i]);
        double b = 0.5 * (w[n - 1 - i] + w[i]);
        x[i] = -a;
        x[n - 1 - i] = a;
        w[i] = b;
        w[n - 1 - i] = b;
    }
    if (n % 2) x[n / 2] = 0.0;
}

void gauss_volume_host(int n, std::vector<double> &g) {
    double x[32], w[32];
    gauss_legendre_host(n, x, w);
    g.assign(4 * n * n * n, 0.0);
    int q = 0;
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++)
            for (int k = 0; k < n; k++, q++) {
                g[4 * q] = w[i] * w[j] * w[k];
                g[4 * q + 1] = x[i];
                g[4 * q + 2] = x[j];
                g[4 * q + 3] = x[k];
            }
}

void gauss_face_host(int n, int face, std::vector<double> &g) {
    double x[32], w[32];
    gauss_legendre_host(n, x, w);
    g.assign(4 * n * n, 0.0);
    for (int j = 0; j < n; j++)
        for (int i = 0; i < n; i++) {
            double *p = &g[4 * (i + n * j)];
            p[0] = w[i] * w[j];
            switch (face) {
                case 1: p[1] = -1.0; p[2] = x[i]; p[3] = x[j]; break;
                case 2: p[1] = 1.0; p[2] = x[i]; p[3] = x[j]; break;
                case 3: p[1] = x[i]; p[2] = -1.0; p[3] = x[j]; break;
                case 4: p[1] = x[i]; p[2] = 1.0; p[3] = x[j]; break;
                case 5: p[1] = x[j]; p[2] = x[i]; p[3] = -1.0; break;
                default: p[1] = x[j]; p[2] = x[i]; p[3] = 1.0; break;
            }
        }
}

// ------------------------------------------------------------ model preparing
int u1_prepare(yeti_ctx *ctx, const yeti_u1_model *m, U1Model &out) {
    YETI_CHECK(m && m->coords && m->ien && m->nb_elem_patch && m->nkv &&
                   m->ukv && m->nijk && m->weight && m->jpqr && m->nnode &&
                   m->nbint && m->matprops && m->active,
               YETI_EINVAL, "U1 model: a required array is NULL");
    YETI_CHECK(m->nb_patch > 0 && m->nb_elem >= 0 && m->nb_cp > 0,
               YETI_EINVAL, "U1 model: bad sizes");
    out.patches.clear();
    out.patches.resize(m->nb_patch);
    out.nb_cp = m->nb_cp;
    int64_t jelem = 0, ukv_off = 0, ien_off = 0, count = 0;
    for (int64_t ip = 0; ip < m->nb_patch; ip++) {
        U1Patch &P = out.patches[ip];
        for (int d = 0; d < 3; d++) {
            P.p[d] = (int)m->jpqr[3 * ip + d];
            P.nkv[d] = (int)m->nkv[3 * ip + d];
        }
        P.nelem = m->nb_elem_patch[ip];
        P.elem_begin = jelem;
        P.nn = (int)m->nnode[ip];
        bool any_active = false;
        for (int64_t e = 0; e < P.nelem; e++)
            if (m->active[jelem + e] == 1) any_active = true;
        if (any_active) {
            YETI_CHECK(!m->is_u1 || m->is_u1[ip], YETI_EUNSUPPORTED,
                       "patch %lld: only U1/THREED solid elements are on this "
                       "path", (long long)ip + 1);
            YETI_CHECK(P.nkv[1] > 0 && P.nkv[2] > 0, YETI_EUNSUPPORTED,
                       "patch %lld: only 3D patches are supported",
                       (long long)ip + 1);
            for (int d = 0; d < 3; d++)
                YETI_CHECK(P.p[d] >= 1 && P.p[d] <= kMaxDeg &&
                               P.nkv[d] >= 2 * P.p[d] + 2,
                           YETI_EINVAL, "patch %lld: degree %d / knots %d",
                           (long long)ip + 1, P.p[d], P.nkv[d]);
            YETI_CHECK(P.nn == (P.p[0] + 1) * (P.p[1] + 1) * (P.p[2] + 1),
                       YETI_EINVAL, "patch %lld: nnode %d does not match the "
                       "degrees", (long long)ip + 1, P.nn);
        }
        P.nq = (int)m->nbint[ip];
        int ng = (int)std::pow((double)P.nq, 1.0 / 3.0);
        if (ng < 1) ng = 1;
        while (ng * ng * ng < P.nq) ng++;
        P.ng = ng;
        YETI_CHECK(P.nq >= 1 && ng <= 32, YETI_EINVAL,
                   "patch %lld: NBINT %d", (long long)ip + 1, P.nq);
        P.E = m->matprops[2 * ip];
        P.nu = m->matprops[2 * ip + 1];
        P.rho = m->rho ? m->rho[ip] : 0.0;
        P.nb_data_elem = 9LL * P.nn * (P.nn - 1) / 2 + 6LL * P.nn;
        const int nn = P.nn;
        std::vector<int32_t> ien, span, gid;
        std::vector<double> w;
        for (int64_t e = 0; e < P.nelem; e++, jelem++) {
            if (m->active[jelem] != 1) continue;
            P.act.push_back(jelem);
            P.slot.push_back(count);
            count += P.nb_data_elem;
            gid.push_back((int32_t)jelem);
            for (int a = 0; a < nn; a++) {
                int64_t cp = m->ien[ien_off + e * nn + a];
                YETI_CHECK(cp >= 1 && cp <= m->nb_cp, YETI_EINVAL,
                           "IEN entry %lld of element %lld out of range",
                           (long long)cp, (long long)jelem + 1);
                ien.push_back((int32_t)(cp - 1));
                w.push_back(m->weight[ien_off + e * nn + a]);
            }
            for (int d = 0; d < 3; d++) {
                int64_t ni = m->nijk[3 * jelem + d];
                YETI_CHECK(ni >= P.p[d] + 1 && ni <= P.nkv[d] - P.p[d] - 1,
                           YETI_EINVAL, "Nijk of element %lld out of range",
                           (long long)jelem + 1);
                span.push_back((int32_t)ni);
            }
        }
        P.nactive = (int64_t)P.act.size();
        int nk = P.nkv[0] + P.nkv[1] + P.nkv[2];
        if (P.nactive) {
            YETI_TRY(upload(ctx, P.knots, m->ukv + ukv_off, nk));
            std::vector<double> g;
            gauss_volume_host(P.ng, g);
            YETI_TRY(upload(ctx, P.gauss, g.data(), g.size()));
            YETI_TRY(upload(ctx, P.ien, ien.data(), ien.size()));
            YETI_TRY(upload(ctx, P.w, w.data(), w.size()));
            YETI_TRY(upload(ctx, P.span, span.data(), span.size()));
            YETI_TRY(upload(ctx, P.slotd, P.slot.data(), P.slot.size()));
            YETI_TRY(upload(ctx, P.gid, gid.data(), gid.size()));
        }
        ukv_off += nk;
        ien_off += P.nelem * nn;
    }
    YETI_CHECK(jelem == m->nb_elem, YETI_EINVAL,
               "sum of nb_elem_patch (%lld) != nb_elem (%lld)",
               (long long)jelem, (long long)m->nb_elem);
    out.nb_data = count;
    YETI_TRY(upload(ctx, out.coords, m->coords, (size_t)3 * m->nb_cp));
    return YETI_OK;
}

// ---------------------------------------------------------------- kernels
struct StiffArgs {
    int p0, p1, p2, nn, nq, qchunk;
    const double *U0, *U1, *U2;
    const double *gauss;
    const double *coords;
    const int32_t *ien;
    const double *w;
    const int32_t *span;
    const int64_t *slot;
    double lam, mu;
    double *kdata;
    int32_t *krow, *kcol;
};

// Rational basis at parent point t of an element: dR/dxi into dRdxi_out
// (3*nn, stride 3 per node), and the 3x3 d x / d xi into J.  Two passes over
// the nodes (normalisation sums, then values) so no per-thread node arrays
// are needed.  Follows shap.f90:90-140.
__device__ inline void rational_derivs(
    int p0, int p1, int p2, int nn, const double *U0, const double *U1,
    const double *U2, const int *ni, const double *u1, const double *u2,
    const double *t, const double *w, const double *xe, double *dRdxi_out,
    double J[3][3], double *Rsum_inv, double *Fv /* 6*kMaxDeg1 */) {
    double xi[3];
    for (int d = 0; d < 3; d++)
        xi[d] = ((u2[d] - u1[d]) * t[d] + (u2[d] + u1[d])) * 0.5;
    double *FN = Fv, *dFN = Fv + kMaxDeg1, *FM = Fv + 2 * kMaxDeg1,
           *dFM = Fv + 3 * kMaxDeg1, *FL = Fv + 4 * kMaxDeg1,
           *dFL = Fv + 5 * kMaxDeg1;
    bspline_ders(ni[0], p0, xi[0], U0, FN, dFN);
    bspline_ders(ni[1], p1, xi[1], U1, FM, dFM);
    bspline_ders(ni[2], p2, xi[2], U2, FL, dFL);
    double S = 0.0, sx0 = 0.0, sx1 = 0.0, sx2 = 0.0;
    int a = 0;
    for (int k = 0; k <= p2; k++)
        for (int j = 0; j <= p1; j++)
            for (int i = 0; i <= p0; i++, a++) {
                double wa = w[a];
                S += FN[p0 - i] * FM[p1 - j] * FL[p2 - k] * wa;
                sx0 += dFN[p0 - i] * FM[p1 - j] * FL[p2 - k] * wa;
                sx1 += FN[p0 - i] * dFM[p1 - j] * FL[p2 - k] * wa;
                sx2 += FN[p0 - i] * FM[p1 - j] * dFL[p2 - k] * wa;
            }
    double inv = 1.0 / S;
    *Rsum_inv = inv;
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) J[r][c] = 0.0;
    a = 0;
    for (int k = 0; k <= p2; k++)
        for (int j = 0; j <= p1; j++)
            for (int i = 0; i <= p0; i++, a++) {
                double wa = w[a];
                double R = FN[p0 - i] * FM[p1 - j] * FL[p2 - k] * wa * inv;
                double d0 = (dFN[p0 - i] * FM[p1 - j] * FL[p2 - k] * wa - R * sx0) * inv;
                double d1 = (FN[p0 - i] * dFM[p1 - j] * FL[p2 - k] * wa - R * sx1) * inv;
                double d2 = (FN[p0 - i] * FM[p1 - j] * dFL[p2 - k] * wa - R * sx2) * inv;
                if (dRdxi_out) {
                    dRdxi_out[3 * a] = d0;
                    dRdxi_out[3 * a + 1] = d1;
                    dRdxi_out[3 * a + 2] = d2;
                }
                for (int r = 0; r < 3; r++) {
                    double x = xe[3 * a + r];
                    J[r][0] += x * d0;
                    J[r][1] += x * d1;
                    J[r][2] += x * d2;
                }
            }
}

// MatrixInv for 3x3 (operateurs.f:385-423); returns the determinant.
__device__ inline double inv3(const double B[3][3], double A[3][3]) {
    double det = B[0][1] * B[1][2] * B[2][0] - B[0][2] * B[1][1] * B[2][0] +
                 B[0][2] * B[1][0] * B[2][1] - B[0][0] * B[1][2] * B[2][1] +
                 B[0][0] * B[1][1] * B[2][2] - B[0][1] * B[1][0] * B[2][2];
    A[0][0] = (B[1][1] * B[2][2] - B[1][2] * B[2][1]) / det;
    A[0][1] = (B[0][2] * B[2][1] - B[0][1] * B[2][2]) / det;
    A[0][2] = (B[0][1] * B[1][2] - B[0][2] * B[1][1]) / det;
    A[1][0] = (B[1][2] * B[2][0] - B[1][0] * B[2][2]) / det;
    A[1][1] = (B[0][0] * B[2][2] - B[0][2] * B[2][0]) / det;
    A[1][2] = (B[0][2] * B[1][0] - B[0][0] * B[1][2]) / det;
    A[2][0] = (B[1][0] * B[2][1] - B[1][1] * B[2][0]) / det;
    A[2][1] = (B[0][1] * B[2][0] - B[0][0] * B[2][1]) / det;
    A[2][2] = (B[0][0] * B[1][1] - B[0][1] * B[1][0]) / det;
    return det;
}

// Parent-element Jacobian determinant (shap.f90:155-178).
__device__ inline double parent_det(const double J[3][3], const double *u1,
                                    const double *u2) {
    double A[3][3];
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) A[r][c] = J[r][c] * (0.5 * (u2[c] - u1[c]));
    return A[0][0] * A[1][1] * A[2][2] + A[0][1] * A[1][2] * A[2][0] +
           A[1][0] * A[2][1] * A[0][2] - A[0][2] * A[1][1] * A[2][0] -
           A[0][1] * A[1][0] * A[2][2] - A[1][2] * A[2][1] * A[0][0];
}

// Shared-memory layout of one Gauss-point chunk of the stiffness and mass
// kernels: per point the six 1-D rows (FN dFN FM dFM FL dFL, kMaxDeg1 each),
// the nn rational numerators, 3 nn derivative values and kStiffQS scalars
// (sx[3], 1/S, J then J^-1 [9], dv).
__host__ __device__ inline size_t stiff_perq(int nn) {
    return (size_t)6 * kMaxDeg1 + 4 * (size_t)nn + kStiffQS;
}

__global__ void __launch_bounds__(256)
k_u1_stiffness(StiffArgs a) {
    extern __shared__ double smem[];
    const int nn = a.nn;
    double *xe = smem;                      // 3*nn element CP coordinates
    double *we = xe + 3 * nn;               // nn element weights
    double *B1 = we + nn;                   // qchunk * 6 * kMaxDeg1
    double *R0 = B1 + (size_t)a.qchunk * 6 * kMaxDeg1;   // qchunk * nn
    double *dR = R0 + (size_t)a.qchunk * nn;             // qchunk * nn * 3
    double *qs = dR + (size_t)a.qchunk * nn * 3;         // qchunk * kStiffQS
    __shared__ double su1[3], su2[3];
    __shared__ int sni[3];
    const int e = blockIdx.x;
    const int tid = threadIdx.x, nth = blockDim.x;
    const int32_t *ien = a.ien + (size_t)e * nn;
    for (int i = tid; i < nn; i += nth) {
        int cp = ien[i];
        xe[3 * i] = a.coords[3 * cp];
        xe[3 * i + 1] = a.coords[3 * cp + 1];
        xe[3 * i + 2] = a.coords[3 * cp + 2];
        we[i] = a.w[(size_t)e * nn + i];
    }
    if (tid < 3) {
        const double *U = tid == 0 ? a.U0 : (tid == 1 ? a.U1 : a.U2);
        int ni = a.span[3 * e + tid];
        sni[tid] = ni;
        su1[tid] = U[ni - 1];
        su2[tid] = U[ni];
    }
    const int npairs = nn * (nn + 1) / 2;
    const int64_t base = a.slot[e];
    const double lam = a.lam, mu = a.mu, l2m = lam + 2.0 * mu;
    const int pd[3] = {a.p0, a.p1, a.p2};
    const double *Ud[3] = {a.U0, a.U1, a.U2};
    for (int q0 = 0; q0 < a.nq; q0 += a.qchunk) {
        const int nqc = min(a.qchunk, a.nq - q0);
        __syncthreads();
        // ---- stage A: basis derivatives at the chunk's Gauss points
        basis_chunk(pd, Ud, sni, su1, su2, a.gauss, q0, nqc, nn, xe, we, B1, R0, nn, dR, 3 * nn, qs);
        // A6: inverse Jacobian and the point's weight
        for (int ql = tid; ql < nqc; ql += nth) {
            double *sq = qs + (size_t)ql * kStiffQS;
            double J[3][3], Ji[3][3];
            for (int r = 0; r < 3; r++)
                for (int c = 0; c < 3; c++) J[r][c] = sq[4 + 3 * r + c];
            inv3(J, Ji);
            sq[13] = a.gauss[4 * (q0 + ql)] * fabs(parent_det(J, su1, su2));
            for (int r = 0; r < 3; r++)
                for (int c = 0; c < 3; c++) sq[4 + 3 * r + c] = Ji[r][c];
        }
        __syncthreads();
        // A7: physical gradients dR/dx, one thread per (point, node)
        for (int t = tid; t < nqc * nn; t += nth) {
            const int ql = t / nn, n = t - ql * nn;
            const double *Ji = qs + (size_t)ql * kStiffQS + 4;
            double *d = dR + ((size_t)ql * nn + n) * 3;
            const double d0 = d[0], d1 = d[1], d2 = d[2];
            for (int c = 0; c < 3; c++) d[c] = d0 * Ji[c] + d1 * Ji[3 + c] + d2 * Ji[6 + c];
        }
        __syncthreads();
        // ---- stage B: one thread per control-point pair (i <= j)
        for (int t = tid; t < npairs; t += blockDim.x) {
            int j = (int)((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
            while (j * (j + 1) / 2 > t) j--;
            while ((j + 1) * (j + 2) / 2 <= t) j++;
            const int i = t - j * (j + 1) / 2;
            const int64_t jb = base + 9LL * j * (j - 1) / 2 + 6LL * j;
            double K[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
            if (q0 > 0) {
                // resume the running sums of the earlier chunks (the stored
                // diagonal of a diagonal block is halved; x2 is exact), so the
                // points are added in one sequence as in the reference
                if (i < j) {
                    for (int ll = 0; ll < 3; ll++)
                        for (int kk = 0; kk < 3; kk++) K[kk][ll] = a.kdata[jb + 9LL * i + 3 * ll + kk];
                } else {
                    for (int ll = 0; ll < 3; ll++)
                        for (int kk = 0; kk <= ll; kk++) {
                            const double v = a.kdata[jb + 9LL * j + ll * (ll + 1) / 2 + kk];
                            K[kk][ll] = kk == ll ? v * 2.0 : v;
                        }
                }
            }
            for (int q = 0; q < nqc; q++) {
                const double *A = dR + ((size_t)q * nn + i) * 3;
                const double *B = dR + ((size_t)q * nn + j) * 3;
                const double a0 = A[0], a1 = A[1], a2 = A[2];
                const double b0 = B[0], b1 = B[1], b2 = B[2];
                const double d = qs[(size_t)q * kStiffQS + 13];
                // B_i^T D B_j for isotropic D (stiffmatrix.F90:167-216)
                K[0][0] += (a0 * (l2m * b0) + a1 * (mu * b1) + a2 * (mu * b2)) * d;
                K[1][1] += (a1 * (l2m * b1) + a0 * (mu * b0) + a2 * (mu * b2)) * d;
                K[2][2] += (a2 * (l2m * b2) + a0 * (mu * b0) + a1 * (mu * b1)) * d;
                K[0][1] += (a0 * (lam * b1) + a1 * (mu * b0)) * d;
                K[1][0] += (a1 * (lam * b0) + a0 * (mu * b1)) * d;
                K[0][2] += (a0 * (lam * b2) + a2 * (mu * b0)) * d;
                K[2][0] += (a2 * (lam * b0) + a0 * (mu * b2)) * d;
                K[1][2] += (a1 * (lam * b2) + a2 * (mu * b1)) * d;
                K[2][1] += (a2 * (lam * b1) + a1 * (mu * b2)) * d;
            }
            const int dofi = 3 * ien[i], dofj = 3 * ien[j];
            if (i < j) {
                const int64_t s = jb + 9LL * i;
                for (int ll = 0; ll < 3; ll++)
                    for (int kk = 0; kk < 3; kk++) {
                        const int64_t o = s + 3 * ll + kk;
                        a.kdata[o] = K[kk][ll];
                        if (q0 == 0) {
                            a.krow[o] = dofi + kk;
                            a.kcol[o] = dofj + ll;
                        }
                    }
            } else {
                const int64_t s = jb + 9LL * j;
                for (int ll = 0; ll < 3; ll++)
                    for (int kk = 0; kk <= ll; kk++) {
                        const int64_t o = s + ll * (ll + 1) / 2 + kk;
                        a.kdata[o] = (kk == ll) ? K[kk][ll] * 0.5 : K[kk][ll];
                        if (q0 == 0) {
                            a.krow[o] = dofj + kk;
                            a.kcol[o] = dofj + ll;
                        }
                    }
            }
        }
    }
}

// Consistent mass matrix (build_CMASSMatrix, compute_CMASSMatrix.f:30-199,
// with UMASSMAT_byCP's U1 branch, UMASSMAT.f): the stiffness kernel's layout
// with, per Gauss point, R and dvol = rho (w_q DetJac) (DetJac signed, as
// shap returns it) in shared memory; one thread per node pair (i <= j)
// accumulates (dvol R_j) R_i over the points in order onto the diagonal of
// the 3x3 block and writes the block into the pair's COO slots (diagonal of
// the diagonal blocks halved, off-diagonal entries 0).
struct MassArgs {
    int p0, p1, p2, nn, nq, qchunk;
    const double *U0, *U1, *U2;
    const double *gauss;
    const double *coords;
    const int32_t *ien;
    const double *w;
    const int32_t *span;
    const int64_t *slot;
    double rho;
    double *mdata;
    int32_t *mrow, *mcol;
};

__global__ void __launch_bounds__(256) k_u1_mass(MassArgs a) {
    extern __shared__ double smem[];
    const int nn = a.nn;
    double *xe = smem;                          // 3*nn element CP coordinates
    double *we = xe + 3 * nn;                   // nn element weights
    double *B1 = we + nn;                       // qchunk * 6 * kMaxDeg1
    double *Rq = B1 + (size_t)a.qchunk * 6 * kMaxDeg1;   // qchunk * nn basis values
    double *dR = Rq + (size_t)a.qchunk * nn;             // qchunk * nn * 3 (dR/dxi)
    double *qs = dR + (size_t)a.qchunk * nn * 3;         // qchunk * kStiffQS
    __shared__ double su1[3], su2[3];
    __shared__ int sni[3];
    const int e = blockIdx.x;
    const int tid = threadIdx.x;
    const int32_t *ien = a.ien + (size_t)e * nn;
    for (int i = tid; i < nn; i += blockDim.x) {
        int cp = ien[i];
        xe[3 * i] = a.coords[3 * cp];
        xe[3 * i + 1] = a.coords[3 * cp + 1];
        xe[3 * i + 2] = a.coords[3 * cp + 2];
        we[i] = a.w[(size_t)e * nn + i];
    }
    if (tid < 3) {
        const double *U = tid == 0 ? a.U0 : (tid == 1 ? a.U1 : a.U2);
        int ni = a.span[3 * e + tid];
        sni[tid] = ni;
        su1[tid] = U[ni - 1];
        su2[tid] = U[ni];
    }
    const int npairs = nn * (nn + 1) / 2;
    const int64_t base = a.slot[e];
    const int pd[3] = {a.p0, a.p1, a.p2};
    const double *Ud[3] = {a.U0, a.U1, a.U2};
    for (int q0 = 0; q0 < a.nq; q0 += a.qchunk) {
        const int nqc = min(a.qchunk, a.nq - q0);
        __syncthreads();
        // ---- stage A: basis values and dvol at the chunk's Gauss points
        basis_chunk(pd, Ud, sni, su1, su2, a.gauss, q0, nqc, nn, xe, we, B1, Rq, nn, dR, 3 * nn, qs);
        for (int t = tid; t < nqc * nn; t += blockDim.x) {
            const int ql = t / nn;
            Rq[t] = Rq[t] * qs[(size_t)ql * kStiffQS + 3];
        }
        for (int ql = tid; ql < nqc; ql += blockDim.x) {
            double *sq = qs + (size_t)ql * kStiffQS;
            double J[3][3];
            for (int r = 0; r < 3; r++)
                for (int c = 0; c < 3; c++) J[r][c] = sq[4 + 3 * r + c];
            const double dvol = a.gauss[4 * (q0 + ql)] * parent_det(J, su1, su2);
            sq[13] = a.rho * dvol;
        }
        __syncthreads();
        // ---- stage B: one thread per control-point pair (i <= j)
        for (int t = tid; t < npairs; t += blockDim.x) {
            int j = (int)((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
            while (j * (j + 1) / 2 > t) j--;
            while ((j + 1) * (j + 2) / 2 <= t) j++;
            const int i = t - j * (j + 1) / 2;
            const int64_t jb = base + 9LL * j * (j - 1) / 2 + 6LL * j;
            // resume the running sum of the earlier chunks (a diagonal
            // block's stored value is halved; x2 is exact)
            double m = 0.0;
            if (q0 > 0) m = i < j ? a.mdata[jb + 9LL * i] : a.mdata[jb + 9LL * j] * 2.0;
            for (int q = 0; q < nqc; q++) {
                const double t1 = qs[(size_t)q * kStiffQS + 13] * Rq[(size_t)q * nn + j];
                m += t1 * Rq[(size_t)q * nn + i];
            }
            const int dofi = 3 * ien[i], dofj = 3 * ien[j];
            if (i < j) {
                const int64_t s = jb + 9LL * i;
                for (int ll = 0; ll < 3; ll++)
                    for (int kk = 0; kk < 3; kk++) {
                        const int64_t o = s + 3 * ll + kk;
                        a.mdata[o] = kk == ll ? m : 0.0;
                        if (q0 == 0) {
                            a.mrow[o] = dofi + kk;
                            a.mcol[o] = dofj + ll;
                        }
                    }
            } else {
                const int64_t s = jb + 9LL * j;
                for (int ll = 0; ll < 3; ll++)
                    for (int kk = 0; kk <= ll; kk++) {
                        const int64_t o = s + ll * (ll + 1) / 2 + kk;
                        a.mdata[o] = kk == ll ? m * 0.5 : 0.0;
                        if (q0 == 0) {
                            a.mrow[o] = dofj + kk;
                            a.mcol[o] = dofj + ll;
                        }
                    }
            }
        }
    }
}

// Distributed loads (UELMAT.f90:121-223), deterministic and in the reference's
// operation order.  Phase 1 (k_u1_elem_rhs) evaluates the RHS of each loaded
// element into a buffer: per-point data first (one thread per quadrature
// point), then one thread per element dof accumulates over the points in
// order.  Phase 2 (k_u1_rhs_gather) adds, for every dof, the element
// contributions in element order (build_system_elemStorage.f90:295-303).
struct LoadTerm {
    int kind;        // 0: body 101, 1: body 102, 2: surface
    int face, type;  // surface: face 1..6, type 0..4
    int ifield;      // nodal distribution row (type 4), 0-based
    double mag;      // ADLMAG
    double info[6];  // additional infos (axis points / direction)
};

struct RhsArgs {
    int p0, p1, p2, nn, nq, ng;
    const double *U0, *U1, *U2;
    const double *gauss;      // volume rule
    const double *gface;      // 6 faces x ng^2 x 4
    const double *coords;
    const int32_t *ien;       // per active element
    const double *w;
    const int32_t *span;
    const int32_t *elems;     // active-element local indices with loads
    const int32_t *term_ptr;  // CSR into terms
    const LoadTerm *terms;
    double rho;
    int nb_n_dist;
    const double *nodal_dist;
    double *erhs;             // (n loaded elements, 3*nn)
};

__global__ void __launch_bounds__(1024) k_u1_elem_rhs(RhsArgs a) {
    extern __shared__ double smem[];
    const int nn = a.nn;
    const int e = a.elems[blockIdx.x];
    const int n0 = a.p0 + 1, n1 = a.p1 + 1, n2 = a.p2 + 1;
    const int nb = n0 + n1 + n2;
    double *xe = smem;                 // 3*nn
    double *we = xe + 3 * nn;          // nn
    double *qd = we + nn;              // per-point data
    __shared__ double su1[3], su2[3];
    __shared__ int sni[3];
    const int tid = threadIdx.x;
    const int32_t *ien = a.ien + (size_t)e * nn;
    for (int i = tid; i < nn; i += blockDim.x) {
        int cp = ien[i];
        for (int d = 0; d < 3; d++) xe[3 * i + d] = a.coords[3 * cp + d];
        we[i] = a.w[(size_t)e * nn + i];
    }
    if (tid < 3) {
        const double *U = tid == 0 ? a.U0 : (tid == 1 ? a.U1 : a.U2);
        int ni = a.span[3 * e + tid];
        sni[tid] = ni;
        su1[tid] = U[ni - 1];
        su2[tid] = U[ni];
    }
    const int t0 = a.term_ptr[blockIdx.x], t1 = a.term_ptr[blockIdx.x + 1];
    int nbody = 0;
    for (int t = t0; t < t1; t++) nbody += (a.terms[t].kind != 2);
    __syncthreads();
    // R of node n at a point whose basis values are stored at bv
    auto Rval = [&](const double *bv, double inv, int n) {
        int i = n % n0, j = (n / n0) % n1, k = n / (n0 * n1);
        return bv[a.p0 - i] * bv[n0 + a.p1 - j] * bv[n0 + n1 + a.p2 - k] * we[n] * inv;
    };
    double acc = 0.0;   // RHS entry (node tid/3, component tid%3)
    const int node = tid / 3, comp = tid % 3;
    const bool mine_ok = tid < 3 * nn;
    // ---- body loads, volume rule (UELMAT.f90:109-171)
    if (nbody > 0) {
        const int stride = nb + 2 + 3 * nbody;
        for (int q = tid; q < a.nq; q += blockDim.x) {
            const double *g = a.gauss + 4 * q;
            double Fv[6 * kMaxDeg1], J[3][3], inv;
            rational_derivs(a.p0, a.p1, a.p2, nn, a.U0, a.U1, a.U2, sni, su1,
                            su2, g + 1, we, xe, nullptr, J, &inv, Fv);
            double *o = qd + (size_t)q * stride;
            for (int i = 0; i < n0; i++) o[i] = Fv[i];
            for (int i = 0; i < n1; i++) o[n0 + i] = Fv[2 * kMaxDeg1 + i];
            for (int i = 0; i < n2; i++) o[n0 + n1 + i] = Fv[4 * kMaxDeg1 + i];
            o[nb] = inv;
            double dvol = g[0] * fabs(parent_det(J, su1, su2));
            o[nb + 1] = dvol;
            double pg[3] = {0.0, 0.0, 0.0};
            for (int n = 0; n < nn; n++) {
                double R = Rval(o, inv, n);
                for (int d = 0; d < 3; d++) pg[d] = pg[d] + R * xe[3 * n + d];
            }
            int bt = 0;
            for (int t = t0; t < t1; t++) {
                const LoadTerm &T = a.terms[t];
                if (T.kind == 2) continue;
                double *pre = o + nb + 2 + 3 * bt;
                if (T.kind == 0) {      // centrifugal (UELMAT.f90:125-151)
                    double vd[3], ag[3];
                    for (int d = 0; d < 3; d++) vd[d] = T.info[3 + d] - T.info[d];
                    double nr = sqrt(vd[0] * vd[0] + vd[1] * vd[1] + vd[2] * vd[2]);
                    for (int d = 0; d < 3; d++) vd[d] = vd[d] / nr;
                    for (int d = 0; d < 3; d++) ag[d] = pg[d] - T.info[d];
                    double sc = ag[0] * vd[0] + ag[1] * vd[1] + ag[2] * vd[2];
                    for (int d = 0; d < 3; d++)
                        pre[d] = a.rho * (T.mag * T.mag) * (ag[d] - sc * vd[d]);
                } else {                // volume force (UELMAT.f90:153-166)
                    for (int d = 0; d < 3; d++) pre[d] = T.mag * T.info[d];
                }
                bt++;
            }
        }
        __syncthreads();
        if (mine_ok) {
            for (int q = 0; q < a.nq; q++) {
                const double *o = qd + (size_t)q * stride;
                const double R = Rval(o, o[nb], node), dvol = o[nb + 1];
                for (int bt = 0; bt < nbody; bt++)
                    acc = acc + o[nb + 2 + 3 * bt + comp] * R * dvol;
            }
        }
        __syncthreads();
    }
    // ---- surface loads, face rule (UELMAT.f90:173-223, shapPress.f)
    const int nf = a.ng * a.ng;
    const int fstride = nb + 6;
    for (int t = t0; t < t1; t++) {
        const LoadTerm T = a.terms[t];
        if (T.kind != 2) continue;
        const double *rule = a.gface + (size_t)(T.face - 1) * nf * 4;
        for (int q = tid; q < nf; q += blockDim.x) {
            const double *g = rule + 4 * q;
            double Fv[6 * kMaxDeg1], J[3][3], inv;
            rational_derivs(a.p0, a.p1, a.p2, nn, a.U0, a.U1, a.U2, sni, su1,
                            su2, g + 1, we, xe, nullptr, J, &inv, Fv);
            double *o = qd + (size_t)q * fstride;
            for (int i = 0; i < n0; i++) o[i] = Fv[i];
            for (int i = 0; i < n1; i++) o[n0 + i] = Fv[2 * kMaxDeg1 + i];
            for (int i = 0; i < n2; i++) o[n0 + n1 + i] = Fv[4 * kMaxDeg1 + i];
            o[nb] = inv;
            double A[3][3];
            for (int r = 0; r < 3; r++)
                for (int c = 0; c < 3; c++) A[r][c] = J[r][c] * (0.5 * (su2[c] - su1[c]));
            double c1[3] = {A[0][0], A[1][0], A[2][0]};
            double c2[3] = {A[0][1], A[1][1], A[2][1]};
            double c3[3] = {A[0][2], A[1][2], A[2][2]};
            const double *P = c2, *Q = c3;   // surface measure pair
            switch (T.face) {
                case 1: case 2: P = c2; Q = c3; break;
                case 3: case 4: P = c3; Q = c1; break;
                default: P = c1; Q = c2; break;
            }
            double nx = P[1] * Q[2] - P[2] * Q[1];
            double ny = P[2] * Q[0] - P[0] * Q[2];
            double nz = P[0] * Q[1] - P[1] * Q[0];
            double detj = sqrt(nx * nx + ny * ny + nz * nz);
            double vec[3] = {0.0, 0.0, 0.0};
            if (T.type >= 1 && T.type <= 3) {
                vec[T.type - 1] = 1.0;
            } else {   // normal pressure, orientation of shapPress.f:229-258
                const double *U = c1, *V = c2;
                switch (T.face) {
                    case 1: U = c2; V = c3; break;
                    case 2: U = c3; V = c2; break;
                    case 3: U = c3; V = c1; break;
                    case 4: U = c1; V = c3; break;
                    case 5: U = c1; V = c2; break;
                    default: U = c2; V = c1; break;
                }
                vec[0] = (U[1] * V[2] - U[2] * V[1]) / detj;
                vec[1] = (U[2] * V[0] - U[0] * V[2]) / detj;
                vec[2] = (U[0] * V[1] - U[1] * V[0]) / detj;
            }
            double fmag = T.mag;
            if (T.type == 4) {
                fmag = 0.0;
                for (int n = 0; n < nn; n++)
                    fmag = fmag + a.nodal_dist[T.ifield + (size_t)a.nb_n_dist * ien[n]] * Rval(o, inv, n);
            }
            o[nb + 1] = vec[0];
            o[nb + 2] = vec[1];
            o[nb + 3] = vec[2];
            o[nb + 4] = g[0] * detj;
            o[nb + 5] = fmag;
        }
        __syncthreads();
        if (mine_ok) {
            double fbl = 0.0;
            for (int q = 0; q < nf; q++) {
                const double *o = qd + (size_t)q * fstride;
                const double R = Rval(o, o[nb], node);
                fbl = fbl + R * o[nb + 1 + comp] * o[nb + 4] * o[nb + 5];
            }
            acc = acc + fbl;
        }
        __syncthreads();
    }
    if (mine_ok) a.erhs[(size_t)blockIdx.x * 3 * nn + tid] = acc;
}

// F[dof] += element contributions in element order.
__global__ void k_u1_rhs_gather(int64_t ndof, const int64_t *ptr,
                                const int64_t *idx, const double *erhs,
                                double *F) {
    int64_t dof = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (dof >= ndof) return;
    double acc = F[dof];
    for (int64_t k = ptr[dof]; k < ptr[dof + 1]; k++) acc = acc + erhs[idx[k]];
    F[dof] = acc;
}

static bool in_list(const int64_t *l, int64_t n, int64_t v) {
    for (int64_t i = 0; i < n; i++)
        if (l[i] == v) return true;
    return false;
}

}  // namespace yeti

using namespace yeti;

YETI_API int yeti_assemble_u1_coo_ex(yeti_ctx *ctx, const yeti_u1_model *m,
                                     int64_t nb_data, double *kdata,
                                     int32_t *krow, int32_t *kcol, double *F,
                                     int mem, int kernel) {
    YETI_CHECK(ctx && m && kdata && krow && kcol && F, YETI_EINVAL,
               "yeti_assemble_u1_coo: NULL argument");
    YETI_CHECK(mem == YETI_MEM_HOST || mem == YETI_MEM_DEVICE, YETI_EINVAL,
               "yeti_assemble_u1_coo: bad mem flag %d", mem);
    YETI_CHECK(kernel == YETI_STIFF_PAIRS || kernel == YETI_STIFF_SUMFACT, YETI_EINVAL,
               "yeti_assemble_u1_coo: bad element kernel %d", kernel);
    DeviceGuard guard(ctx->device);
    U1Model M;
    YETI_TRY(u1_prepare(ctx, m, M));
    YETI_CHECK(M.nb_data <= nb_data, YETI_EINVAL,
               "nb_data %lld smaller than the %lld slots of the active "
               "elements", (long long)nb_data, (long long)M.nb_data);
    const int64_t ndof = 3 * m->nb_cp;
    // ---- load vector: concentrated loads are assigned (not added) first,
    // build_system_elemStorage.f90:137-152
    std::vector<double> F0(ndof, 0.0);
    int64_t kk = 0;
    for (int64_t il = 0; il < m->nb_load; il++) {
        int64_t ty = m->jdltype[il];
        if (ty / 10 < 1) {
            YETI_CHECK(ty >= 1 && ty <= 3, YETI_EUNSUPPORTED,
                       "concentrated load direction %lld", (long long)ty);
            for (int64_t c = 0; c < m->load_target_nbelem[il]; c++) {
                int64_t cp = m->inddload[kk + c];
                YETI_CHECK(cp >= 1 && cp <= m->nb_cp, YETI_EINVAL,
                           "concentrated load CP %lld", (long long)cp);
                F0[(cp - 1) * 3 + ty - 1] = m->adlmag[il];
            }
        } else if (ty != 101 && ty != 102) {
            YETI_CHECK(ty > 9 && ty < 100 && (ty % 10) <= 4 &&
                           ty / 10 >= 1 && ty / 10 <= 6,
                       YETI_EUNSUPPORTED, "distributed load type U%lld is not "
                       "on the U1 path", (long long)ty);
        }
        kk += m->load_target_nbelem[il];
    }
    DevBuf dK, dR, dC, dF;
    double *k_ = kdata, *f_ = F;
    int32_t *r_ = krow, *c_ = kcol;
    if (mem == YETI_MEM_HOST) {
        YETI_TRY(dK.alloc(ctx, nb_data * sizeof(double)));
        YETI_TRY(dR.alloc(ctx, nb_data * sizeof(int32_t)));
        YETI_TRY(dC.alloc(ctx, nb_data * sizeof(int32_t)));
        YETI_TRY(dF.alloc(ctx, ndof * sizeof(double)));
        k_ = dK.as<double>();
        r_ = dR.as<int32_t>();
        c_ = dC.as<int32_t>();
        f_ = dF.as<double>();
    }
    if (M.nb_data < nb_data) {   // slots beyond the active elements stay 0
        YETI_CUDA(cudaMemsetAsync(k_ + M.nb_data, 0, (nb_data - M.nb_data) * sizeof(double), ctx->stream));
        YETI_CUDA(cudaMemsetAsync(r_ + M.nb_data, 0, (nb_data - M.nb_data) * sizeof(int32_t), ctx->stream));
        YETI_CUDA(cudaMemsetAsync(c_ + M.nb_data, 0, (nb_data - M.nb_data) * sizeof(int32_t), ctx->stream));
    }
    YETI_CUDA(cudaMemcpyAsync(f_, F0.data(), ndof * sizeof(double),
                              cudaMemcpyHostToDevice, ctx->stream));
    int smem_optin = 0;
    YETI_CUDA(cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device));
    const size_t smem_cap = std::min<size_t>(smem_optin, 200 * 1024);
    YETI_CUDA(cudaFuncSetAttribute(k_u1_stiffness, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_cap));
    std::vector<std::unique_ptr<DevBuf>> keep;
    auto newbuf = [&keep]() -> DevBuf & {
        keep.emplace_back(new DevBuf());
        return *keep.back();
    };
    struct Loaded { int patch; int64_t local; int64_t off; };
    struct PatchRhs { DevBuf *buf; size_t first; };
    std::vector<Loaded> loaded;
    std::vector<PatchRhs> patch_erhs;
    int64_t erhs_total = 0;
    std::vector<int64_t> ien_offset(M.patches.size(), 0);
    for (size_t ip = 1; ip < M.patches.size(); ip++)
        ien_offset[ip] = ien_offset[ip - 1] + M.patches[ip - 1].nelem * M.patches[ip - 1].nn;
    for (size_t ip = 0; ip < M.patches.size(); ip++) {
        U1Patch &P = M.patches[ip];
        if (!P.nactive) continue;
        const size_t fixed = sizeof(double) * 4 * P.nn;
        const size_t perq = sizeof(double) * stiff_perq(P.nn);
        YETI_CHECK(fixed + perq <= smem_cap, YETI_EUNSUPPORTED,
                   "element with %d nodes does not fit shared memory", P.nn);
        int qchunk = (int)std::min<size_t>(P.nq, (smem_cap - fixed) / perq);
        StiffArgs a;
        a.p0 = P.p[0]; a.p1 = P.p[1]; a.p2 = P.p[2];
        a.nn = P.nn; a.nq = P.nq; a.qchunk = qchunk;
        a.U0 = P.knots.as<double>();
        a.U1 = a.U0 + P.nkv[0];
        a.U2 = a.U1 + P.nkv[1];
        a.gauss = P.gauss.as<double>();
        a.coords = M.coords.as<double>();
        a.ien = P.ien.as<int32_t>();
        a.w = P.w.as<double>();
        a.span = P.span.as<int32_t>();
        a.slot = P.slotd.as<int64_t>();
        a.lam = (P.E * P.nu) / ((1.0 + P.nu) * (1.0 - 2.0 * P.nu));
        a.mu = P.E / (2.0 * (1.0 + P.nu));
        a.kdata = k_; a.krow = r_; a.kcol = c_;
        const size_t smem = fixed + perq * qchunk;
        if (kernel == YETI_STIFF_SUMFACT) {
            KernelTimer timer(ctx, "k_u1_stiffness_sf");
            YETI_TRY(launch_u1_stiffness_sf(ctx, P, a.coords, a.lam, a.mu, k_, r_, c_, smem_cap));
        } else {
            KernelTimer timer(ctx, "k_u1_stiffness");
            int64_t left = P.nactive, off = 0;
            while (left > 0) {   // grid.x limit
                int64_t n = std::min<int64_t>(left, 1 << 30);
                StiffArgs b = a;
                b.ien += off * P.nn; b.w += off * P.nn; b.span += off * 3; b.slot += off;
                k_u1_stiffness<<<(unsigned)n, 256, smem, ctx->stream>>>(b);
                count_launches(1);
                YETI_CUDA(cudaGetLastError());
                left -= n; off += n;
            }
        }
        // ---- distributed loads of this patch's elements
        std::vector<int32_t> elems, tptr(1, 0);
        std::vector<LoadTerm> terms;
        int max_body = 0;
        for (int64_t le = 0; le < P.nactive; le++) {
            const int64_t jel = P.act[le] + 1;   // 1-based element number
            int64_t k2 = 0, cinfo = 0;
            size_t before = terms.size();
            int nbody = 0;
            for (int64_t il = 0; il < m->nb_load; il++) {
                int64_t nt = m->load_target_nbelem[il], ty = m->jdltype[il];
                if ((ty == 101 || ty == 102 || (ty > 9 && ty < 100)) &&
                    in_list(m->inddload + k2, nt, jel)) {
                    LoadTerm T;
                    memset(&T, 0, sizeof(T));
                    T.mag = m->adlmag[il];
                    if (ty == 101 || ty == 102) {
                        T.kind = ty == 101 ? 0 : 1;
                        int nneed = ty == 101 ? 6 : 3;
                        YETI_CHECK(cinfo + nneed <= m->len_load_addinfos, YETI_EINVAL,
                                   "load %lld: missing additional infos", (long long)il + 1);
                        for (int d = 0; d < nneed; d++) T.info[d] = m->load_addinfos[cinfo + d];
                        nbody++;
                    } else {
                        T.kind = 2;
                        T.face = (int)(ty / 10);
                        T.type = (int)(ty % 10);
                        if (T.type == 4) {
                            YETI_CHECK(cinfo < m->len_load_addinfos && m->nodal_dist, YETI_EINVAL,
                                       "load %lld: nodal distribution missing", (long long)il + 1);
                            T.ifield = (int)m->load_addinfos[cinfo] - 1;
                            YETI_CHECK(T.ifield >= 0 && T.ifield < m->nb_n_dist, YETI_EINVAL,
                                       "load %lld: nodal field index", (long long)il + 1);
                        }
                    }
                    terms.push_back(T);
                }
                k2 += nt;
                cinfo += m->nb_load_addinfos ? m->nb_load_addinfos[il] : 0;
            }
            if (terms.size() > before) {
                elems.push_back((int32_t)le);
                tptr.push_back((int32_t)terms.size());
                max_body = std::max(max_body, nbody);
                loaded.push_back({(int)ip, le, erhs_total});
                erhs_total += 3LL * P.nn;
            }
        }
        if (!elems.empty()) {
            YETI_CHECK(P.nn * 3 <= 1024, YETI_EUNSUPPORTED,
                       "distributed loads on elements with more than 341 nodes "
                       "are not supported");
            std::vector<double> gf(6 * 4 * P.ng * P.ng), tmp;
            for (int f = 1; f <= 6; f++) {
                gauss_face_host(P.ng, f, tmp);
                std::copy(tmp.begin(), tmp.end(), gf.begin() + (f - 1) * 4 * P.ng * P.ng);
            }
            DevBuf &dgf = newbuf();
            YETI_TRY(upload(ctx, dgf, gf.data(), gf.size()));
            DevBuf &del = newbuf();
            YETI_TRY(upload(ctx, del, elems.data(), elems.size()));
            DevBuf &dtp = newbuf();
            YETI_TRY(upload(ctx, dtp, tptr.data(), tptr.size()));
            DevBuf &dtm = newbuf();
            YETI_TRY(upload(ctx, dtm, terms.data(), terms.size()));
            DevBuf *dnd = nullptr;
            if (m->nodal_dist && m->nb_n_dist > 0) {
                dnd = &newbuf();
                YETI_TRY(upload(ctx, *dnd, m->nodal_dist, (size_t)m->nb_n_dist * m->nb_cp));
            }
            DevBuf &der = newbuf();
            YETI_TRY(der.alloc(ctx, sizeof(double) * 3 * P.nn * elems.size()));
            patch_erhs.push_back({&der, loaded.size() - elems.size()});
            RhsArgs r;
            r.p0 = P.p[0]; r.p1 = P.p[1]; r.p2 = P.p[2];
            r.nn = P.nn; r.nq = P.nq; r.ng = P.ng;
            r.U0 = P.knots.as<double>(); r.U1 = r.U0 + P.nkv[0]; r.U2 = r.U1 + P.nkv[1];
            r.gauss = P.gauss.as<double>();
            r.gface = dgf.as<double>();
            r.coords = M.coords.as<double>();
            r.ien = P.ien.as<int32_t>();
            r.w = P.w.as<double>();
            r.span = P.span.as<int32_t>();
            r.elems = del.as<int32_t>();
            r.term_ptr = dtp.as<int32_t>();
            r.terms = dtm.as<LoadTerm>();
            r.rho = P.rho;
            r.nb_n_dist = (int)m->nb_n_dist;
            r.nodal_dist = dnd ? dnd->as<double>() : nullptr;
            r.erhs = der.as<double>();
            const int nb = P.p[0] + P.p[1] + P.p[2] + 3;
            const size_t per = std::max<size_t>((size_t)P.nq * (nb + 2 + 3 * max_body),
                                                (size_t)P.ng * P.ng * (nb + 6));
            size_t smem = sizeof(double) * (4 * P.nn + per);
            YETI_CHECK(smem <= smem_cap, YETI_EUNSUPPORTED, "element too large for the load kernel");
            YETI_CUDA(cudaFuncSetAttribute(k_u1_elem_rhs, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_cap));
            const int nthr = std::max(128, (3 * P.nn + 31) / 32 * 32);
            k_u1_elem_rhs<<<(unsigned)elems.size(), nthr, smem, ctx->stream>>>(r);
            count_launches(1);
            YETI_CUDA(cudaGetLastError());
        }
    }
    // ---- phase 2: per-dof sums of the element contributions, element order
    if (!loaded.empty()) {
        // one contiguous buffer: copy each patch's element RHS slice in order
        DevBuf &dall = newbuf();
        YETI_TRY(dall.alloc(ctx, sizeof(double) * erhs_total));
        int64_t off = 0;
        for (auto &pe : patch_erhs) {
            YETI_CUDA(cudaMemcpyAsync(dall.as<double>() + off, pe.buf->ptr, pe.buf->bytes,
                                      cudaMemcpyDeviceToDevice, ctx->stream));
            off += (int64_t)(pe.buf->bytes / sizeof(double));
        }
        std::vector<int64_t> cnt(ndof + 1, 0), idx;
        std::vector<std::vector<int64_t>> lists(ndof);
        for (auto &L : loaded) {
            const U1Patch &P = M.patches[L.patch];
            const int64_t jel = P.act[L.local];
            const int64_t ien_base = ien_offset[L.patch] + (jel - P.elem_begin) * P.nn;
            for (int n = 0; n < P.nn; n++) {
                int64_t cp = m->ien[ien_base + n] - 1;
                for (int d = 0; d < 3; d++) lists[3 * cp + d].push_back(L.off + 3 * n + d);
            }
        }
        for (int64_t i = 0; i < ndof; i++) {
            cnt[i + 1] = cnt[i] + (int64_t)lists[i].size();
            idx.insert(idx.end(), lists[i].begin(), lists[i].end());
        }
        DevBuf &dptr = newbuf();
        YETI_TRY(upload(ctx, dptr, cnt.data(), cnt.size()));
        DevBuf &didx = newbuf();
        YETI_TRY(upload(ctx, didx, idx.data(), idx.size()));
        k_u1_rhs_gather<<<(unsigned)((ndof + 255) / 256), 256, 0, ctx->stream>>>(
            ndof, dptr.as<int64_t>(), didx.as<int64_t>(), dall.as<double>(), f_);
        count_launches(1);
        YETI_CUDA(cudaGetLastError());
    }
    if (mem == YETI_MEM_HOST) {
        YETI_CUDA(cudaMemcpyAsync(kdata, k_, nb_data * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        YETI_CUDA(cudaMemcpyAsync(krow, r_, nb_data * sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
        YETI_CUDA(cudaMemcpyAsync(kcol, c_, nb_data * sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
        YETI_CUDA(cudaMemcpyAsync(F, f_, ndof * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    }
    // the model's device arrays are released on return: wait for the work
    YETI_CUDA(cudaStreamSynchronize(ctx->stream));
    return YETI_OK;
}

YETI_API int yeti_assemble_u1_coo(yeti_ctx *ctx, const yeti_u1_model *m,
                                  int64_t nb_data, double *kdata,
                                  int32_t *krow, int32_t *kcol, double *F,
                                  int mem) {
    return yeti_assemble_u1_coo_ex(ctx, m, nb_data, kdata, krow, kcol, F, mem, YETI_STIFF_PAIRS);
}

YETI_API int yeti_assemble_u1_mass_coo(yeti_ctx *ctx, const yeti_u1_model *m,
                                       int64_t nb_data, double *mdata, int32_t *mrow,
                                       int32_t *mcol, int mem) {
    YETI_CHECK(ctx && m && mdata && mrow && mcol, YETI_EINVAL,
               "yeti_assemble_u1_mass_coo: NULL argument");
    YETI_CHECK(mem == YETI_MEM_HOST || mem == YETI_MEM_DEVICE, YETI_EINVAL,
               "yeti_assemble_u1_mass_coo: bad mem flag %d", mem);
    DeviceGuard guard(ctx->device);
    U1Model M;
    YETI_TRY(u1_prepare(ctx, m, M));
    YETI_CHECK(M.nb_data <= nb_data, YETI_EINVAL,
               "nb_data %lld smaller than the %lld slots of the active elements",
               (long long)nb_data, (long long)M.nb_data);
    YETI_CHECK(m->rho, YETI_EINVAL, "yeti_assemble_u1_mass_coo: no densities");
    DevBuf dM, dR, dC;
    double *m_ = mdata;
    int32_t *r_ = mrow, *c_ = mcol;
    if (mem == YETI_MEM_HOST) {
        YETI_TRY(dM.alloc(ctx, nb_data * sizeof(double)));
        YETI_TRY(dR.alloc(ctx, nb_data * sizeof(int32_t)));
        YETI_TRY(dC.alloc(ctx, nb_data * sizeof(int32_t)));
        m_ = dM.as<double>();
        r_ = dR.as<int32_t>();
        c_ = dC.as<int32_t>();
    }
    if (M.nb_data < nb_data) {   // slots beyond the active elements stay 0
        YETI_CUDA(cudaMemsetAsync(m_ + M.nb_data, 0, (nb_data - M.nb_data) * sizeof(double), ctx->stream));
        YETI_CUDA(cudaMemsetAsync(r_ + M.nb_data, 0, (nb_data - M.nb_data) * sizeof(int32_t), ctx->stream));
        YETI_CUDA(cudaMemsetAsync(c_ + M.nb_data, 0, (nb_data - M.nb_data) * sizeof(int32_t), ctx->stream));
    }
    int smem_optin = 0;
    YETI_CUDA(cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device));
    const size_t smem_cap = std::min<size_t>(smem_optin, 200 * 1024);
    YETI_CUDA(cudaFuncSetAttribute(k_u1_mass, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_cap));
    for (size_t ip = 0; ip < M.patches.size(); ip++) {
        U1Patch &P = M.patches[ip];
        if (!P.nactive) continue;
        const size_t fixed = sizeof(double) * 4 * P.nn;
        const size_t perq = sizeof(double) * stiff_perq(P.nn);
        YETI_CHECK(fixed + perq <= smem_cap, YETI_EUNSUPPORTED,
                   "element with %d nodes does not fit shared memory", P.nn);
        const int qchunk = (int)std::min<size_t>(P.nq, (smem_cap - fixed) / perq);
        MassArgs a;
        a.p0 = P.p[0]; a.p1 = P.p[1]; a.p2 = P.p[2];
        a.nn = P.nn; a.nq = P.nq; a.qchunk = qchunk;
        a.U0 = P.knots.as<double>();
        a.U1 = a.U0 + P.nkv[0];
        a.U2 = a.U1 + P.nkv[1];
        a.gauss = P.gauss.as<double>();
        a.coords = M.coords.as<double>();
        a.ien = P.ien.as<int32_t>();
        a.w = P.w.as<double>();
        a.span = P.span.as<int32_t>();
        a.slot = P.slotd.as<int64_t>();
        a.rho = P.rho;
        a.mdata = m_; a.mrow = r_; a.mcol = c_;
        const size_t smem = fixed + perq * qchunk;
        KernelTimer timer(ctx, "k_u1_mass");
        int64_t left = P.nactive, off = 0;
        while (left > 0) {   // grid.x limit
            const int64_t n = std::min<int64_t>(left, 1 << 30);
            MassArgs b = a;
            b.ien += off * P.nn; b.w += off * P.nn; b.span += off * 3; b.slot += off;
            k_u1_mass<<<(unsigned)n, 256, smem, ctx->stream>>>(b);
            count_launches(1);
            YETI_CUDA(cudaGetLastError());
            left -= n; off += n;
        }
    }
    if (mem == YETI_MEM_HOST) {
        YETI_CUDA(cudaMemcpyAsync(mdata, m_, nb_data * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
        YETI_CUDA(cudaMemcpyAsync(mrow, r_, nb_data * sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
        YETI_CUDA(cudaMemcpyAsync(mcol, c_, nb_data * sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
    }
    // the model's device arrays are released on return: wait for the work
    YETI_CUDA(cudaStreamSynchronize(ctx->stream));
    return YETI_OK;
}
