/*
 * CPU oracle for the U1 solid NURBS path of YETI (arnaudduval/yeti).
 *
 * TEST INFRASTRUCTURE ONLY.  This file restates, in plain C, the reference's
 * Fortran algorithm so that the CUDA product path can be checked against it.
 * Nothing in the product (the yeti_b200 package and libyeti_b200.so) links,
 * loads or calls this code; only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py do.
 *
 * Each routine follows the loop and rounding order of the Fortran routine it
 * cites (paths relative to the reference's source tree), so that the COO
 * values agree with the reference to round-off.  Compile with
 * -ffp-contract=off (no FMA contraction; gfortran -O2 on x86-64 does not fuse
 * either).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define MAXP 10            /* maximum degree per direction */
#define MAXNN 1331         /* maximum nodes per element (p=10 cubed) */

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

/* ------------------------------------------------------------------ */
/* Gauss-Legendre rule of order n on [-1,1] (Gauss, GaussLegendre.f90: */
/* 27-153): the table for orders 1..9; beyond, where the reference has */
/* no rule, the roots of P_n by Newton iteration on the three-term     */
/* recurrence with the weights 2/((1-x^2) P_n'(x)^2).                  */
/* ------------------------------------------------------------------ */
void oracle_gauss_legendre(int n, double *x, double *w)
{
    if (n >= 1 && n <= 9) {
        gauss_table(n, x, w);
        return;
    }
    for (int i = 0; i < n; i++) {
        /* initial guess: Chebyshev-like approximation of the i-th root,
         * ascending order */
        double z = -cos(M_PI * (i + 0.75) / (n + 0.5));
        double pp = 0.0;
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
            if (fabs(dz) < 1e-17) break;
        }
        {
            double p1 = 1.0, p2 = 0.0;
            for (int k = 1; k <= n; k++) {
                double p3 = p2;
                p2 = p1;
                p1 = ((2.0 * k - 1.0) * z * p2 - (k - 1.0) * p3) / k;
            }
            pp = n * (z * p1 - p2) / (z * z - 1.0);
        }
        x[i] = z;
        w[i] = 2.0 / ((1.0 - z * z) * pp * pp);
    }
    /* exact symmetry and exact zero for odd orders */
    for (int i = 0; i < n / 2; i++) {
        double a = 0.5 * (x[n - 1 - i] - x[i]);
        double b = 0.5 * (w[n - 1 - i] + w[i]);
        x[i] = -a; x[n - 1 - i] = a;
        w[i] = b;  w[n - 1 - i] = b;
    }
    if (n % 2) x[n / 2] = 0.0;
}

/* Volume rule, ordering of GaussLegendre.f90:175-187: xi1 outermost,
 * xi3 innermost; weight = (w_i*w_j)*w_k.  out[4*q] = weight,
 * out[4*q+1..3] = parent coordinates. */
static void gauss_volume(int n, double *out)
{
    double x[16], w[16];
    oracle_gauss_legendre(n, x, w);
    int q = 0;
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++)
            for (int k = 0; k < n; k++, q++) {
                out[4 * q] = w[i] * w[j] * w[k];
                out[4 * q + 1] = x[i];
                out[4 * q + 2] = x[j];
                out[4 * q + 3] = x[k];
            }
}

/* Face rules, GaussLegendre.f90:217-270 (3D faces 1..6). */
static void gauss_face(int n, int face, double *out)
{
    double x[16], w[16];
    oracle_gauss_legendre(n, x, w);
    for (int j = 0; j < n; j++)
        for (int i = 0; i < n; i++) {
            double *g = out + 4 * (i + n * j);
            g[0] = w[i] * w[j];
            switch (face) {
            case 1: g[1] = -1.0; g[2] = x[i]; g[3] = x[j]; break;
            case 2: g[1] = 1.0;  g[2] = x[i]; g[3] = x[j]; break;
            case 3: g[1] = x[i]; g[2] = -1.0; g[3] = x[j]; break;
            case 4: g[1] = x[i]; g[2] = 1.0;  g[3] = x[j]; break;
            case 5: g[1] = x[j]; g[2] = x[i]; g[3] = -1.0; break;
            default: g[1] = x[j]; g[2] = x[i]; g[3] = 1.0; break;
            }
        }
}

/* ------------------------------------------------------------------ */
/* B-spline values and first derivatives (dersbasisfuns.f90:30-131,    */
/* The NURBS Book A2.3 with n=1).  ni: 1-based span index of the knot   */
/* vector U (0-based C array).                                          */
/* ------------------------------------------------------------------ */
static void ders_basis(int ni, int p, double u, const double *U,
                       double *N, double *dN)
{
    double ndu[MAXP + 1][MAXP + 1], left[MAXP + 2], right[MAXP + 2];
    ndu[0][0] = 1.0;
    for (int j = 1; j <= p; j++) {
        left[j] = u - U[ni - j];         /* u_knotl(ni+1-j) */
        right[j] = U[ni + j - 1] - u;    /* u_knotl(ni+j)   */
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

/* ------------------------------------------------------------------ */
/* patch / element description                                          */
/* ------------------------------------------------------------------ */
typedef struct {
    int p[3];
    int nkv[3];
    const double *U[3];       /* knot vectors of the patch */
    int nnode;
} patch_t;

typedef struct {
    double u1[3], u2[3];      /* knot span of the element, per direction */
    int ni[3];                /* 1-based span index */
    const double *w;          /* nnode element weights */
    double coords[3 * MAXNN]; /* (3, nnode) */
} elem_t;

/* Rational basis, parametric derivatives and the parent->physical
 * Jacobian at one point (shap.f90:21-180, shapPress.f:18-160).
 * Outputs R[nnode], dRdxi[3*nnode] (dRdxi[3*a+d]), dxdxi[3][3]
 * (dxdxi[a][b] = d x_a / d xi_b), AJ[3][3] (parent Jacobian). */
static void nurbs_point(const patch_t *pt, const elem_t *el, const double *t,
                        double *R, double *dRdxi, double dxdxi[3][3],
                        double AJ[3][3])
{
    double FN[MAXP + 1], dFN[MAXP + 1], FM[MAXP + 1], dFM[MAXP + 1],
        FL[MAXP + 1], dFL[MAXP + 1];
    double xi[3];
    for (int d = 0; d < 3; d++)
        xi[d] = ((el->u2[d] - el->u1[d]) * t[d] + (el->u2[d] + el->u1[d])) * 0.5;
    ders_basis(el->ni[0], pt->p[0], xi[0], pt->U[0], FN, dFN);
    ders_basis(el->ni[1], pt->p[1], xi[1], pt->U[1], FM, dFM);
    ders_basis(el->ni[2], pt->p[2], xi[2], pt->U[2], FL, dFL);
    const int p1 = pt->p[0], p2 = pt->p[1], p3 = pt->p[2];
    int n = 0;
    double sum = 0.0, sx[3] = {0.0, 0.0, 0.0};
    for (int k = 0; k <= p3; k++)
        for (int j = 0; j <= p2; j++)
            for (int i = 0; i <= p1; i++, n++) {
                double w = el->w[n];
                R[n] = FN[p1 - i] * FM[p2 - j] * FL[p3 - k] * w;
                sum = sum + R[n];
                dRdxi[3 * n + 0] = dFN[p1 - i] * FM[p2 - j] * FL[p3 - k] * w;
                sx[0] = sx[0] + dRdxi[3 * n + 0];
                dRdxi[3 * n + 1] = FN[p1 - i] * dFM[p2 - j] * FL[p3 - k] * w;
                sx[1] = sx[1] + dRdxi[3 * n + 1];
                dRdxi[3 * n + 2] = FN[p1 - i] * FM[p2 - j] * dFL[p3 - k] * w;
                sx[2] = sx[2] + dRdxi[3 * n + 2];
            }
    double inv = 1.0 / sum;
    for (int a = 0; a < pt->nnode; a++) {
        R[a] = R[a] * inv;
        for (int d = 0; d < 3; d++)
            dRdxi[3 * a + d] = (dRdxi[3 * a + d] - R[a] * sx[d]) * inv;
    }
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) dxdxi[a][b] = 0.0;
    for (int nl = 0; nl < pt->nnode; nl++)
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++)
                dxdxi[a][b] = dxdxi[a][b] + el->coords[3 * nl + a] * dRdxi[3 * nl + b];
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++)
            AJ[a][b] = dxdxi[a][b] * (0.5 * (el->u2[b] - el->u1[b]));
}

/* MatrixInv, MCRD=3 (operateurs.f:385-423). */
static double mat_inv3(double A[3][3], double B[3][3])
{
    double det = B[0][1] * B[1][2] * B[2][0] - B[0][2] * B[1][1] * B[2][0]
               + B[0][2] * B[1][0] * B[2][1] - B[0][0] * B[1][2] * B[2][1]
               + B[0][0] * B[1][1] * B[2][2] - B[0][1] * B[1][0] * B[2][2];
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

/* shap.f90:21-180: physical derivatives dRdx[3*a+d] and DetJac. */
static double shap(const patch_t *pt, const elem_t *el, const double *t,
                   double *R, double *dRdx)
{
    double dRdxi[3 * MAXNN], dxdxi[3][3], AJ[3][3], dxidx[3][3];
    nurbs_point(pt, el, t, R, dRdxi, dxdxi, AJ);
    mat_inv3(dxidx, dxdxi);
    for (int a = 0; a < pt->nnode; a++)
        for (int na = 0; na < 3; na++) {
            double s = 0.0;
            for (int nb = 0; nb < 3; nb++) s = s + dRdxi[3 * a + nb] * dxidx[nb][na];
            dRdx[3 * a + na] = s;
        }
    return AJ[0][0] * AJ[1][1] * AJ[2][2] + AJ[0][1] * AJ[1][2] * AJ[2][0]
         + AJ[1][0] * AJ[2][1] * AJ[0][2] - AJ[0][2] * AJ[1][1] * AJ[2][0]
         - AJ[0][1] * AJ[1][0] * AJ[2][2] - AJ[1][2] * AJ[2][1] * AJ[0][0];
}

static void cross3(const double *b, const double *c, double *a)
{
    a[0] = b[1] * c[2] - b[2] * c[1];
    a[1] = b[2] * c[0] - b[0] * c[2];
    a[2] = b[0] * c[1] - b[1] * c[0];
}

/* shapPress.f:18-262 (3D): face basis, surface measure and load direction.
 * Returns 0, or -1 for an unsupported load type. */
static int shap_press(const patch_t *pt, const elem_t *el, const double *t,
                      int face, int type, double *R, double *vect, double *detj)
{
    double dRdxi[3 * MAXNN], dxdxi[3][3], AJ[3][3];
    nurbs_point(pt, el, t, R, dRdxi, dxdxi, AJ);
    double c1[3] = {AJ[0][0], AJ[1][0], AJ[2][0]};
    double c2[3] = {AJ[0][1], AJ[1][1], AJ[2][1]};
    double c3[3] = {AJ[0][2], AJ[1][2], AJ[2][2]};
    const double *A = c1, *B = c2;
    switch (face) {
    case 1: case 2: A = c2; B = c3; break;
    case 3: case 4: A = c3; B = c1; break;
    case 5: case 6: A = c1; B = c2; break;
    default: return -1;
    }
    double n[3];
    cross3(A, B, n);
    *detj = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
    if (type >= 1 && type <= 3) {
        vect[0] = vect[1] = vect[2] = 0.0;
        vect[type - 1] = 1.0;
        return 0;
    }
    if (type == 0 || type == 4) {
        const double *P = c1, *Q = c2;
        switch (face) {
        case 1: P = c2; Q = c3; break;
        case 2: P = c3; Q = c2; break;
        case 3: P = c3; Q = c1; break;
        case 4: P = c1; Q = c3; break;
        case 5: P = c1; Q = c2; break;
        default: P = c2; Q = c1; break;
        }
        vect[0] = (P[1] * Q[2] - P[2] * Q[1]) / *detj;
        vect[1] = (P[2] * Q[0] - P[0] * Q[2]) / *detj;
        vect[2] = (P[0] * Q[1] - P[1] * Q[0]) / *detj;
        return 0;
    }
    return -1;
}

/* material_lib.f90:75-87 (THREED). */
static void material_threed(double E, double nu, double D[6][6])
{
    memset(D, 0, sizeof(double) * 36);
    double lambda = (E * nu) / ((1.0 + nu) * (1.0 - 2.0 * nu));
    double mu = E / (2.0 * (1.0 + nu));
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) D[i][j] = lambda;
    for (int i = 0; i < 3; i++) D[i][i] = lambda + 2.0 * mu;
    D[3][3] = D[4][4] = D[5][5] = mu;
}

/* stiffmatrix_byCP (stiffmatrix.F90:130-225) accumulated into AMATRX with
 * weight dvol (UELMAT.f90:113-119).  amatrx: (3,3,npairs) column-major
 * per pair, amatrx[9*pair + kk + 3*ll]. */
static void stiff_accumulate(int nnode, double D[6][6], const double *dRdx,
                             double dvol, double *amatrx)
{
    int count = 0;
    for (int nodj = 0; nodj < nnode; nodj++) {
        const double *dj = dRdx + 3 * nodj;
        double BoJ[6][3];
        memset(BoJ, 0, sizeof(BoJ));
        for (int i = 0; i < 3; i++) BoJ[i][i] = dj[i];
        BoJ[3][0] = dj[1]; BoJ[3][1] = dj[0];
        BoJ[4][0] = dj[2]; BoJ[4][2] = dj[0];
        BoJ[5][1] = dj[2]; BoJ[5][2] = dj[1];
        double SBoJ[6][3];
        memset(SBoJ, 0, sizeof(SBoJ));
        for (int j = 0; j < 3; j++)
            for (int i = 0; i < 3; i++) SBoJ[i][j] = D[i][j] * BoJ[j][j];
        SBoJ[3][0] = D[3][3] * BoJ[3][0];
        SBoJ[3][1] = D[3][3] * BoJ[3][1];
        SBoJ[4][0] = D[4][4] * BoJ[4][0];
        SBoJ[4][2] = D[4][4] * BoJ[4][2];
        SBoJ[5][1] = D[3][3] * BoJ[5][1];
        SBoJ[5][2] = D[3][3] * BoJ[5][2];
        for (int nodi = 0; nodi <= nodj; nodi++, count++) {
            const double *di = dRdx + 3 * nodi;
            double BoIt[3][6];
            memset(BoIt, 0, sizeof(BoIt));
            for (int i = 0; i < 3; i++) BoIt[i][i] = di[i];
            BoIt[0][3] = di[1]; BoIt[1][3] = di[0];
            BoIt[0][4] = di[2]; BoIt[2][4] = di[0];
            BoIt[1][5] = di[2]; BoIt[2][5] = di[1];
            double *am = amatrx + 9 * count;
            for (int ii = 0; ii < 3; ii++)
                for (int jj = 0; jj < 3; jj++) {
                    double s = 0.0;
                    for (int kk = 0; kk < 6; kk++) s = s + BoIt[ii][kk] * SBoJ[kk][jj];
                    am[ii + 3 * jj] = am[ii + 3 * jj] + s * dvol;
                }
        }
    }
}

static int elem_in_list(const int64_t *list, int64_t n, int64_t jelem)
{
    for (int64_t i = 0; i < n; i++)
        if (list[i] == jelem) return 1;
    return 0;
}

/* load set shared by the element routines */
typedef struct {
    int nb_load;
    const int64_t *inddload, *jdltype, *load_target_nbelem, *nb_addinfos;
    const double *adlmag, *addinfos;
    int nb_n_dist;
    const double *nodal_dist;   /* (nb_n_dist, nb_cp) column-major */
} loads_t;

/* UELMAT_byCP (UELMAT.f90:22-225) for one U1 element: AMATRX and RHS.
 * ien_e: 1-based CP indices of the element (for nodal distributions). */
static int uelmat_u1(const patch_t *pt, const elem_t *el, int nbint,
                     double E, double nu, double density, int64_t jelem,
                     const loads_t *ld, const int64_t *ien_e,
                     double *rhs, double *amatrx)
{
    const int nn = pt->nnode;
    int ng = (int)pow((double)nbint, 1.0 / 3.0);
    if (ng < 1) ng = 1;
    while (ng * ng * ng < nbint) ng++;
    double *gp = (double *)malloc(sizeof(double) * 4 * ng * ng * ng);
    double *R = (double *)malloc(sizeof(double) * nn);
    double *dRdx = (double *)malloc(sizeof(double) * 3 * nn);
    gauss_volume(ng, gp);
    double D[6][6];
    material_threed(E, nu, D);
    memset(rhs, 0, sizeof(double) * 3 * nn);
    memset(amatrx, 0, sizeof(double) * 9 * (size_t)nn * (nn + 1) / 2);
    for (int q = 0; q < nbint; q++) {
        double detj = shap(pt, el, gp + 4 * q + 1, R, dRdx);
        double dvol = gp[4 * q] * fabs(detj);
        stiff_accumulate(nn, D, dRdx, dvol, amatrx);
        int64_t kload = 0, cinfo = 0;
        for (int il = 0; il < ld->nb_load; il++) {
            int64_t nt = ld->load_target_nbelem[il];
            int64_t ty = ld->jdltype[il];
            if ((ty == 101 || ty == 102) && elem_in_list(ld->inddload + kload, nt, jelem)) {
                double vr[3];
                if (ty == 101) {
                    const double *A = ld->addinfos + cinfo, *B = ld->addinfos + cinfo + 3;
                    double pg[3] = {0.0, 0.0, 0.0};
                    for (int a = 0; a < nn; a++)
                        for (int d = 0; d < 3; d++) pg[d] = pg[d] + R[a] * el->coords[3 * a + d];
                    double vd[3], ag[3];
                    for (int d = 0; d < 3; d++) vd[d] = B[d] - A[d];
                    double nrm = sqrt(vd[0] * vd[0] + vd[1] * vd[1] + vd[2] * vd[2]);
                    for (int d = 0; d < 3; d++) vd[d] = vd[d] / nrm;
                    for (int d = 0; d < 3; d++) ag[d] = pg[d] - A[d];
                    double sc = ag[0] * vd[0] + ag[1] * vd[1] + ag[2] * vd[2];
                    for (int d = 0; d < 3; d++) vr[d] = ag[d] - sc * vd[d];
                    int kk = 0;
                    for (int a = 0; a < nn; a++)
                        for (int d = 0; d < 3; d++, kk++)
                            rhs[kk] = rhs[kk] + density * (ld->adlmag[il] * ld->adlmag[il]) * vr[d] * R[a] * dvol;
                } else {
                    for (int d = 0; d < 3; d++) vr[d] = ld->addinfos[cinfo + d];
                    int kk = 0;
                    for (int a = 0; a < nn; a++)
                        for (int d = 0; d < 3; d++, kk++)
                            rhs[kk] = rhs[kk] + ld->adlmag[il] * vr[d] * R[a] * dvol;
                }
            }
            kload += nt;
            cinfo += ld->nb_addinfos[il];
        }
    }
    int err = 0;
    int64_t kk = 0, cinfo = 0;
    double *fbl = (double *)malloc(sizeof(double) * 3 * nn);
    double *gf = (double *)malloc(sizeof(double) * 4 * ng * ng);
    for (int il = 0; il < ld->nb_load; il++) {
        int64_t nt = ld->load_target_nbelem[il];
        int64_t ty = ld->jdltype[il];
        if (ty > 9 && ty < 100 && elem_in_list(ld->inddload + kk, nt, jelem)) {
            int face = (int)(ty / 10), type = (int)(ty % 10);
            int ifield = 0;
            if (type == 4) ifield = (int)ld->addinfos[cinfo];
            gauss_face(ng, face, gf);
            memset(fbl, 0, sizeof(double) * 3 * nn);
            for (int q = 0; q < ng * ng; q++) {
                double vect[3], detj;
                if (shap_press(pt, el, gf + 4 * q + 1, face, type, R, vect, &detj)) {
                    err = -1;
                    break;
                }
                double dvol = gf[4 * q] * detj;
                double fmag;
                if (type == 4) {
                    fmag = 0.0;
                    for (int a = 0; a < nn; a++)
                        fmag = fmag + ld->nodal_dist[(ifield - 1) + (int64_t)ld->nb_n_dist * (ien_e[a] - 1)] * R[a];
                } else {
                    fmag = ld->adlmag[il];
                }
                int ni = 0;
                for (int a = 0; a < nn; a++)
                    for (int d = 0; d < 3; d++, ni++)
                        fbl[ni] = fbl[ni] + R[a] * vect[d] * dvol * fmag;
            }
            for (int k = 0; k < 3 * nn; k++) rhs[k] = rhs[k] + fbl[k];
        }
        kk += nt;
        cinfo += ld->nb_addinfos[il];
    }
    free(fbl); free(gf); free(gp); free(R); free(dRdx);
    return err;
}

/*
 * sys_linmat_lindef_static (build_system_elemStorage.f90:24-315), U1 solids
 * in 3D.  Integer inputs are int64 (the Python wrapper converts).  COO slots
 * are compacted over active elements like the sequential Fortran
 * (`count` only advances for active elements).  Returns 0, or a negative
 * code for unsupported input (non-U1 element, load type outside 0..4).
 */
int oracle_sys_linmat_lindef_static(
    int64_t nb_patch, int64_t nb_elem, int64_t nb_cp,
    const double *coords, const int64_t *ien, const int64_t *nb_elem_patch,
    const int64_t *nkv, const double *ukv, const int64_t *nijk,
    const double *weight, const int64_t *jpqr, const int64_t *nnode,
    const int64_t *nbint, const double *matprops, const double *rho,
    const int64_t *active,
    int64_t nb_load, const int64_t *inddload, const int64_t *jdltype,
    const double *adlmag, const int64_t *load_target_nbelem,
    const double *addinfos, const int64_t *nb_addinfos,
    int64_t nb_n_dist, const double *nodal_dist,
    int64_t nb_data, int64_t nb_dof_tot,
    double *kdata, int32_t *krow, int32_t *kcol, double *F)
{
    (void)nb_cp;
    memset(kdata, 0, sizeof(double) * nb_data);
    memset(krow, 0, sizeof(int32_t) * nb_data);
    memset(kcol, 0, sizeof(int32_t) * nb_data);
    memset(F, 0, sizeof(double) * nb_dof_tot);
    loads_t ld = {(int)nb_load, inddload, jdltype, load_target_nbelem,
                  nb_addinfos, adlmag, addinfos, (int)nb_n_dist, nodal_dist};
    int64_t kk = 0;
    for (int64_t il = 0; il < nb_load; il++) {
        int64_t ty = jdltype[il];
        if (ty / 10 < 1)
            for (int64_t c = 0; c < load_target_nbelem[il]; c++)
                F[(inddload[kk + c] - 1) * 3 + ty - 1] = adlmag[il];
        kk += load_target_nbelem[il];
    }
    int64_t count = 0, jelem = 0, ukv_off = 0, ien_off = 0, w_off = 0;
    int err = 0;
    for (int64_t ip = 0; ip < nb_patch && !err; ip++) {
        patch_t pt;
        for (int d = 0; d < 3; d++) {
            pt.p[d] = (int)jpqr[3 * ip + d];
            pt.nkv[d] = (int)nkv[3 * ip + d];
        }
        if (pt.nkv[2] <= 0 || pt.nkv[1] <= 0) return -2;   /* 3D only */
        pt.U[0] = ukv + ukv_off;
        pt.U[1] = pt.U[0] + pt.nkv[0];
        pt.U[2] = pt.U[1] + pt.nkv[1];
        pt.nnode = (pt.p[0] + 1) * (pt.p[1] + 1) * (pt.p[2] + 1);
        if (pt.nnode != nnode[ip] || pt.nnode > MAXNN) return -3;
        const int nn = pt.nnode;
        /* OpenMP over the elements, as sys_linmat_lindef_static_omp
         * (build_system_elemStorage_OMP.f90:190-278): every active element
         * owns a fixed run of COO slots; its load vector is kept and added
         * to F after the loop, in element order, so that F has the same bits
         * as the sequential sum */
        const int64_t nep = nb_elem_patch[ip], j0 = jelem;
        const int64_t ndat = 9 * (int64_t)nn * (nn - 1) / 2 + 6 * (int64_t)nn;
        int64_t *slot = (int64_t *)malloc(sizeof(int64_t) * (nep + 1));
        double *rhs_all = (double *)calloc((size_t)nep * 3 * nn, sizeof(double));
        for (int64_t ie = 0; ie < nep; ie++) {
            slot[ie] = count;
            if (active[j0 + ie] == 1) count += ndat;
        }
        if (count > nb_data) { free(slot); free(rhs_all); return -5; }
#pragma omp parallel
        {
            double *amatrx = (double *)malloc(sizeof(double) * 9 * (size_t)nn * (nn + 1) / 2);
            elem_t el;
#pragma omp for schedule(dynamic, 4)
            for (int64_t ie = 0; ie < nep; ie++) {
                const int64_t je = j0 + ie;
                const int64_t *ien_e = ien + ien_off + ie * nn;
                if (active[je] != 1) continue;
                double *rhs = rhs_all + (size_t)ie * 3 * nn;
                for (int a = 0; a < nn; a++)
                    for (int d = 0; d < 3; d++)
                        el.coords[3 * a + d] = coords[3 * (ien_e[a] - 1) + d];
                el.w = weight + w_off + ie * nn;
                for (int d = 0; d < 3; d++) {
                    el.ni[d] = (int)nijk[3 * je + d];
                    el.u1[d] = pt.U[d][el.ni[d] - 1];
                    el.u2[d] = pt.U[d][el.ni[d]];
                }
                if (uelmat_u1(&pt, &el, (int)nbint[ip], matprops[2 * ip],
                              matprops[2 * ip + 1], rho[ip], je + 1, &ld, ien_e,
                              rhs, amatrx)) {
#pragma omp atomic write
                    err = -4;
                    continue;
                }
                int64_t at = slot[ie];
                int i = 0;
                for (int cpj = 0; cpj < nn; cpj++) {
                    int64_t dofj = (ien_e[cpj] - 1) * 3;
                    for (int cpi = 0; cpi < cpj; cpi++, i++) {
                        int64_t dofi = (ien_e[cpi] - 1) * 3;
                        for (int ll = 0; ll < 3; ll++)
                            for (int k2 = 0; k2 < 3; k2++, at++) {
                                kdata[at] = amatrx[9 * i + k2 + 3 * ll];
                                krow[at] = (int32_t)(dofi + k2);
                                kcol[at] = (int32_t)(dofj + ll);
                            }
                    }
                    for (int ll = 0; ll < 3; ll++) {
                        amatrx[9 * i + ll + 3 * ll] = amatrx[9 * i + ll + 3 * ll] * 0.5;
                        for (int k2 = 0; k2 <= ll; k2++, at++) {
                            kdata[at] = amatrx[9 * i + k2 + 3 * ll];
                            krow[at] = (int32_t)(dofj + k2);
                            kcol[at] = (int32_t)(dofj + ll);
                        }
                    }
                    i++;
                }
            }
            free(amatrx);
        }
        for (int64_t ie = 0; ie < nep; ie++) {
            if (active[j0 + ie] != 1) continue;
            const int64_t *ien_e = ien + ien_off + ie * nn;
            const double *rhs = rhs_all + (size_t)ie * 3 * nn;
            for (int a = 0; a < nn; a++)
                for (int d = 0; d < 3; d++)
                    F[(ien_e[a] - 1) * 3 + d] = F[(ien_e[a] - 1) * 3 + d] + rhs[3 * a + d];
        }
        jelem += nep;
        free(slot);
        free(rhs_all);
        for (int d = 0; d < 3; d++) ukv_off += pt.nkv[d];
        ien_off += nb_elem_patch[ip] * nn;
        w_off += nb_elem_patch[ip] * nn;
    }
    if (count > nb_data) return -5;
    return err;
}

/* build_CMASSMatrix (src/yeti_iga/main/compute_CMASSMatrix.f:30-199) with
 * UMASSMAT_byCP's U1 branch (main/UMASSMAT.f): per Gauss point
 * dvol = rho (w_q DetJac) (DetJac signed, as shap returns it), and for every
 * node pair i <= j the diagonal of the 3x3 block gets (dvol R_j) R_i.  The
 * blocks are scattered in the stiffness assembly's COO slot order, the
 * diagonal of the diagonal blocks halved. */
int oracle_build_cmassmatrix(
    int64_t nb_patch, int64_t nb_elem, int64_t nb_cp,
    const double *coords, const int64_t *ien, const int64_t *nb_elem_patch,
    const int64_t *nkv, const double *ukv, const int64_t *nijk,
    const double *weight, const int64_t *jpqr, const int64_t *nnode,
    const int64_t *nbint, const double *rho, const int64_t *active,
    int64_t nb_data, double *mdata, int32_t *mrow, int32_t *mcol)
{
    (void)nb_cp;
    (void)nb_elem;
    memset(mdata, 0, sizeof(double) * nb_data);
    memset(mrow, 0, sizeof(int32_t) * nb_data);
    memset(mcol, 0, sizeof(int32_t) * nb_data);
    int64_t count = 0, jelem = 0, ukv_off = 0, ien_off = 0, w_off = 0;
    for (int64_t ip = 0; ip < nb_patch; ip++) {
        patch_t pt;
        for (int d = 0; d < 3; d++) {
            pt.p[d] = (int)jpqr[3 * ip + d];
            pt.nkv[d] = (int)nkv[3 * ip + d];
        }
        if (pt.nkv[2] <= 0 || pt.nkv[1] <= 0) return -2;
        pt.U[0] = ukv + ukv_off;
        pt.U[1] = pt.U[0] + pt.nkv[0];
        pt.U[2] = pt.U[1] + pt.nkv[1];
        pt.nnode = (pt.p[0] + 1) * (pt.p[1] + 1) * (pt.p[2] + 1);
        if (pt.nnode != nnode[ip] || pt.nnode > MAXNN) return -3;
        const int nn = pt.nnode, nbi = (int)nbint[ip];
        int ng = (int)pow((double)nbi, 1.0 / 3.0);
        if (ng < 1) ng = 1;
        while (ng * ng * ng < nbi) ng++;
        double *gp = (double *)malloc(sizeof(double) * 4 * ng * ng * ng);
        gauss_volume(ng, gp);
        /* OpenMP over the elements (the element loop of
         * build_system_elemStorage_OMP.f90:190-278); each active element
         * owns a fixed run of COO slots, so the result does not depend on
         * the thread count */
        const int64_t nep = nb_elem_patch[ip], j0 = jelem;
        const int64_t ndat = 9 * (int64_t)nn * (nn - 1) / 2 + 6 * (int64_t)nn;
        int64_t *slot = (int64_t *)malloc(sizeof(int64_t) * (nep + 1));
        for (int64_t ie = 0; ie < nep; ie++) {
            slot[ie] = count;
            if (active[j0 + ie] == 1) count += ndat;
        }
        if (count > nb_data) { free(slot); free(gp); return -5; }
#pragma omp parallel
        {
            double *cm = (double *)malloc(sizeof(double) * (size_t)nn * (nn + 1) / 2);
            double *R = (double *)malloc(sizeof(double) * nn);
            double *dRdx = (double *)malloc(sizeof(double) * 3 * nn);
            elem_t el;
#pragma omp for schedule(dynamic, 4)
            for (int64_t ie = 0; ie < nep; ie++) {
                const int64_t je = j0 + ie;
                const int64_t *ien_e = ien + ien_off + ie * nn;
                if (active[je] != 1) continue;
                for (int a = 0; a < nn; a++)
                    for (int d = 0; d < 3; d++)
                        el.coords[3 * a + d] = coords[3 * (ien_e[a] - 1) + d];
                el.w = weight + w_off + ie * nn;
                for (int d = 0; d < 3; d++) {
                    el.ni[d] = (int)nijk[3 * je + d];
                    el.u1[d] = pt.U[d][el.ni[d] - 1];
                    el.u2[d] = pt.U[d][el.ni[d]];
                }
                memset(cm, 0, sizeof(double) * (size_t)nn * (nn + 1) / 2);
                for (int q = 0; q < nbi; q++) {
                    double detj = shap(&pt, &el, gp + 4 * q + 1, R, dRdx);
                    double dvol = gp[4 * q] * detj;
                    dvol = rho[ip] * dvol;
                    int c = 0;
                    for (int j = 0; j < nn; j++) {
                        double t1 = dvol * R[j];
                        for (int i = 0; i <= j; i++, c++) cm[c] = cm[c] + t1 * R[i];
                    }
                }
                int64_t at = slot[ie];
                int i = 0;
                for (int cpj = 0; cpj < nn; cpj++) {
                    int64_t dofj = (ien_e[cpj] - 1) * 3;
                    for (int cpi = 0; cpi < cpj; cpi++, i++) {
                        int64_t dofi = (ien_e[cpi] - 1) * 3;
                        for (int ll = 0; ll < 3; ll++)
                            for (int k2 = 0; k2 < 3; k2++, at++) {
                                mdata[at] = k2 == ll ? cm[i] : 0.0;
                                mrow[at] = (int32_t)(dofi + k2);
                                mcol[at] = (int32_t)(dofj + ll);
                            }
                    }
                    for (int ll = 0; ll < 3; ll++)
                        for (int k2 = 0; k2 <= ll; k2++, at++) {
                            mdata[at] = k2 == ll ? cm[i] * 0.5 : 0.0;
                            mrow[at] = (int32_t)(dofj + k2);
                            mcol[at] = (int32_t)(dofj + ll);
                        }
                    i++;
                }
            }
            free(cm); free(R); free(dRdx);
        }
        jelem += nep;
        free(slot);
        free(gp);
        for (int d = 0; d < 3; d++) ukv_off += pt.nkv[d];
        ien_off += nb_elem_patch[ip] * nn;
        w_off += nb_elem_patch[ip] * nn;
    }
    if (count > nb_data) return -5;
    return 0;
}
