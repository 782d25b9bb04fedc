/*
 * CPU oracle of the analytic shape gradient of the linear-elastic work for U1
 * solids.  TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).
 *
 * Restates gradLinElastWork_AN (src/yeti_iga/optim/gradtotalwork_fullAN.f90:
 * 17-300) and gradUELMAT1adj (src/yeti_iga/optim/gradUELMAT_solid.f90:18-479)
 * with evalnurbs (src/yeti_iga/main/evaluatenurbsfcts.f:94-209) in their loop
 * and rounding order (compile without FMA contraction).  The reference leaves
 * the surface-load sensitivity as "to do" (gradUELMAT_solid.f90:463-477);
 * with include_surface != 0 this oracle adds it: for a distributed load on a
 * face, W_ext = fmag * sum_q w_q UA(xi_q) . v(xi_q), with v = P x Q (normal
 * pressure, shapPress.f face ordering) or e_t |A x B| (fixed direction), and
 * its derivative with respect to the control points through the face
 * tangents.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define GMAXP 10
#define GMAXNN 1331

/* Gauss-Legendre rule of order n (GaussLegendre.f90:27-153), shared with
 * the assembly oracle (yeti_oracle.c). */
void oracle_gauss_legendre(int n, double *x, double *w);
#define g_gauss_legendre oracle_gauss_legendre

static void g_ders(int ni, int p, double u, const double *U, double *N, double *dN)
{
    double ndu[GMAXP + 1][GMAXP + 1], left[GMAXP + 2], right[GMAXP + 2];
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
            if (r >= 1) { double a = 1.0 / ndu[p][r - 1]; d = a * ndu[r - 1][p - 1]; }
            if (r <= p - 1) { double a = -1.0 / ndu[p][r]; d = d + a * ndu[r][p - 1]; }
        }
        dN[r] = d * (double)p;
    }
}

/* evalnurbs: R[nn], dRdxi[3*a+i] at parametric point xi */
static void g_evalnurbs(const int *p, const double *const *U, const int *ni,
                        const double *w, const double *xi, double *R, double *dRdxi)
{
    double FN[GMAXP + 1], dFN[GMAXP + 1], FM[GMAXP + 1], dFM[GMAXP + 1], FL[GMAXP + 1], dFL[GMAXP + 1];
    g_ders(ni[0], p[0], xi[0], U[0], FN, dFN);
    g_ders(ni[1], p[1], xi[1], U[1], FM, dFM);
    g_ders(ni[2], p[2], xi[2], U[2], FL, dFL);
    int n = 0, nn = (p[0] + 1) * (p[1] + 1) * (p[2] + 1);
    double S = 0.0, sx[3] = {0.0, 0.0, 0.0};
    for (int k = 0; k <= p[2]; k++)
        for (int j = 0; j <= p[1]; j++)
            for (int i = 0; i <= p[0]; i++, n++) {
                R[n] = FN[p[0] - i] * FM[p[1] - j] * FL[p[2] - k] * w[n];
                S = S + R[n];
                dRdxi[3 * n] = dFN[p[0] - i] * FM[p[1] - j] * FL[p[2] - k] * w[n];
                sx[0] = sx[0] + dRdxi[3 * n];
                dRdxi[3 * n + 1] = FN[p[0] - i] * dFM[p[1] - j] * FL[p[2] - k] * w[n];
                sx[1] = sx[1] + dRdxi[3 * n + 1];
                dRdxi[3 * n + 2] = FN[p[0] - i] * FM[p[1] - j] * dFL[p[2] - k] * w[n];
                sx[2] = sx[2] + dRdxi[3 * n + 2];
            }
    double inv = 1.0 / S;
    for (int a = 0; a < nn; a++) {
        R[a] = R[a] * inv;
        for (int i = 0; i < 3; i++) dRdxi[3 * a + i] = (dRdxi[3 * a + i] - R[a] * sx[i]) * inv;
    }
}

static void g_cross(const double *u, const double *v, double *w)
{
    w[0] = u[1] * v[2] - u[2] * v[1];
    w[1] = u[2] * v[0] - u[0] * v[2];
    w[2] = u[0] * v[1] - u[1] * v[0];
}

static double g_dot(const double *u, const double *v) { return u[0] * v[0] + u[1] * v[1] + u[2] * v[2]; }

static void g_inv3(double A[3][3], double B[3][3])
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
}

static const int VI[6] = {0, 1, 2, 0, 0, 1}, VJ[6] = {0, 1, 2, 1, 2, 2};

static int g_in_list(const int64_t *l, int64_t n, int64_t v)
{
    for (int64_t i = 0; i < n; i++)
        if (l[i] == v) return 1;
    return 0;
}

/* gradUELMAT1adj for one element (3D).  Ue (3,nn), UAe (3,nn,nadj) column
 * major as in the Fortran; gint/gext (nadj,3,nn). */
static void g_element(int nadj, int nn, int nbint, const double *coords, const double *Ue,
                      const double *UAe, const int *p, const double *const *U, const int *ni,
                      const double *u1, const double *u2, const double *w, double E, double nu,
                      double density, int64_t jelem, int nb_load, const int64_t *inddload,
                      const int64_t *load_target_nbelem, const int64_t *jdltype,
                      const double *adlmag, const double *addinfos, int compute_int,
                      int compute_ext, int include_surface, const double *nodal_dist,
                      int nb_n_dist, const int64_t *ien_e, double *gint, double *gext)
{
    int ng = (int)pow((double)nbint, 1.0 / 3.0);
    if (ng < 1) ng = 1;
    while (ng * ng * ng < nbint) ng++;
    double gx[32], gw[32];
    g_gauss_legendre(ng, gx, gw);
    double lambda = E * nu / (1.0 + nu) / (1.0 - 2.0 * nu);
    double mu = E / 2.0 / (1.0 + nu);
    memset(gint, 0, sizeof(double) * nadj * 3 * nn);
    memset(gext, 0, sizeof(double) * nadj * 3 * nn);
    double *R = (double *)malloc(sizeof(double) * nn);
    double *dR = (double *)malloc(sizeof(double) * 3 * nn);
    double *dUA = (double *)malloc(sizeof(double) * 9 * nadj);
    double *strainA = (double *)malloc(sizeof(double) * 6 * nadj);
    double *stressA = (double *)malloc(sizeof(double) * 6 * nadj);
    double *work = (double *)malloc(sizeof(double) * nadj);
    double *vA = (double *)malloc(sizeof(double) * 3 * nadj);
    int q = 0;
    for (int i0 = 0; i0 < ng; i0++)
        for (int j0 = 0; j0 < ng; j0++)
            for (int k0 = 0; k0 < ng; k0++, q++) {
                if (q >= nbint) break;
                double t[3] = {gx[i0], gx[j0], gx[k0]};
                double detJac = gw[i0] * gw[j0] * gw[k0], xi[3];
                for (int i = 0; i < 3; i++) {
                    xi[i] = ((u2[i] - u1[i]) * t[i] + (u2[i] + u1[i])) * 0.5;
                    detJac = detJac * 0.5 * (u2[i] - u1[i]);
                }
                g_evalnurbs(p, U, ni, w, xi, R, dR);
                double AI[3][3] = {{0}};   /* AI[i] = column i */
                for (int i = 0; i < 3; i++)
                    for (int cp = 0; cp < nn; cp++)
                        for (int c = 0; c < 3; c++) AI[i][c] = AI[i][c] + dR[3 * cp + i] * coords[3 * cp + c];
                double AxA[3][3];
                g_cross(AI[0], AI[1], AxA[2]);
                double Area = g_dot(AxA[2], AI[2]);
                g_cross(AI[1], AI[2], AxA[0]);
                g_cross(AI[2], AI[0], AxA[1]);
                double AAE[3][3] = {{0}}, stress[6] = {0}, strain[6] = {0}, dU[3][3] = {{0}};
                if (compute_int) {
                    double AAI[3][3];
                    for (int i = 0; i < 3; i++)
                        for (int j = 0; j < 3; j++) AAI[i][j] = g_dot(AI[i], AI[j]);
                    g_inv3(AAE, AAI);
                    double H[6][6];
                    for (int kl = 0; kl < 6; kl++) {
                        int k = VI[kl], l = VJ[kl];
                        for (int ij = 0; ij <= kl; ij++) {
                            int i = VI[ij], j = VJ[ij];
                            H[ij][kl] = lambda * AAE[i][j] * AAE[k][l] +
                                        mu * (AAE[i][k] * AAE[j][l] + AAE[i][l] * AAE[j][k]);
                        }
                    }
                    for (int kl = 1; kl < 6; kl++)
                        for (int r = kl; r < 6; r++) H[r][kl - 1] = H[kl - 1][r];
                    for (int i = 0; i < 3; i++)
                        for (int cp = 0; cp < nn; cp++)
                            for (int c = 0; c < 3; c++) dU[i][c] = dU[i][c] + dR[3 * cp + i] * Ue[3 * cp + c];
                    memset(dUA, 0, sizeof(double) * 9 * nadj);
                    for (int a = 0; a < nadj; a++)
                        for (int i = 0; i < 3; i++)
                            for (int cp = 0; cp < nn; cp++)
                                for (int c = 0; c < 3; c++)
                                    dUA[9 * a + 3 * i + c] = dUA[9 * a + 3 * i + c] +
                                        dR[3 * cp + i] * UAe[3 * cp + c + 3 * nn * a];
                    for (int ij = 0; ij < 6; ij++) {
                        int i = VI[ij], j = VJ[ij];
                        if (i == j) strain[ij] = g_dot(AI[i], dU[i]);
                        else strain[ij] = g_dot(AI[i], dU[j]) + g_dot(AI[j], dU[i]);
                    }
                    for (int ii = 0; ii < 6; ii++) {
                        double s = 0.0;
                        for (int jj = 0; jj < 6; jj++) s = s + H[ii][jj] * strain[jj];
                        stress[ii] = s;
                    }
                    for (int a = 0; a < nadj; a++) {
                        const double *d = dUA + 9 * a;
                        for (int ij = 0; ij < 6; ij++) {
                            int i = VI[ij], j = VJ[ij];
                            if (i == j) strainA[6 * a + ij] = g_dot(AI[i], d + 3 * i);
                            else strainA[6 * a + ij] = g_dot(AI[i], d + 3 * j) + g_dot(AI[j], d + 3 * i);
                        }
                        for (int ii = 0; ii < 6; ii++) {
                            double s = 0.0;
                            for (int jj = 0; jj < 6; jj++) s = s + H[ii][jj] * strainA[6 * a + jj];
                            stressA[6 * a + ii] = s;
                        }
                    }
                    for (int a = 0; a < nadj; a++) work[a] = 0.0;
                    for (int ij = 0; ij < 6; ij++)
                        for (int a = 0; a < nadj; a++) work[a] = work[a] + strainA[6 * a + ij] * stress[ij];
                    for (int cp = 0; cp < nn; cp++) {
                        const double *dr = dR + 3 * cp;
                        double dJ[3] = {0, 0, 0};
                        for (int i = 0; i < 3; i++)
                            for (int c = 0; c < 3; c++) dJ[c] = dJ[c] + AxA[i][c] * dr[i];
                        for (int a = 0; a < nadj; a++)
                            for (int c = 0; c < 3; c++)
                                gint[a + nadj * (c + 3 * cp)] = gint[a + nadj * (c + 3 * cp)] - work[a] * dJ[c] * detJac;
                        for (int a = 0; a < nadj; a++) {
                            const double *d = dUA + 9 * a;
                            double e[3] = {0, 0, 0};
                            for (int ij = 0; ij < 6; ij++) {
                                int i = VI[ij], j = VJ[ij];
                                for (int c = 0; c < 3; c++) {
                                    if (i == j) e[c] = e[c] + stress[ij] * d[3 * i + c] * dr[i];
                                    else e[c] = e[c] + stress[ij] * d[3 * i + c] * dr[j] + stress[ij] * d[3 * j + c] * dr[i];
                                }
                            }
                            for (int c = 0; c < 3; c++)
                                gint[a + nadj * (c + 3 * cp)] = gint[a + nadj * (c + 3 * cp)] - e[c] * Area * detJac;
                        }
                        double dAAI[3][3][3], dAAE[3][3][3];
                        for (int j = 0; j < 3; j++)
                            for (int i = 0; i < 3; i++)
                                for (int c = 0; c < 3; c++) dAAI[i][j][c] = dr[i] * AI[j][c] + AI[i][c] * dr[j];
                        memset(dAAE, 0, sizeof(dAAE));
                        for (int j = 0; j < 3; j++)
                            for (int i = 0; i < 3; i++)
                                for (int l = 0; l < 3; l++)
                                    for (int k = 0; k < 3; k++)
                                        for (int c = 0; c < 3; c++)
                                            dAAE[i][j][c] = dAAE[i][j][c] - AAE[i][k] * AAE[l][j] * dAAI[k][l][c];
                        for (int a = 0; a < nadj; a++) {
                            const double *sA = stressA + 6 * a;
                            double e[3] = {0, 0, 0};
                            for (int ij = 0; ij < 6; ij++) {
                                int i = VI[ij], j = VJ[ij];
                                for (int c = 0; c < 3; c++) {
                                    if (i == j) e[c] = e[c] + sA[ij] * dU[i][c] * dr[i];
                                    else e[c] = e[c] + sA[ij] * dU[i][c] * dr[j] + sA[ij] * dU[j][c] * dr[i];
                                }
                            }
                            for (int c = 0; c < 3; c++) vA[3 * a + c] = e[c];
                        }
                        for (int kl = 0; kl < 6; kl++) {
                            int k = VI[kl], l = VJ[kl];
                            for (int ij = 0; ij < 6; ij++) {
                                int i = VI[ij], j = VJ[ij];
                                double dC[3];
                                for (int c = 0; c < 3; c++)
                                    dC[c] = lambda * dAAE[i][j][c] * AAE[k][l] + lambda * AAE[i][j] * dAAE[k][l][c] +
                                            mu * dAAE[i][k][c] * AAE[j][l] + mu * AAE[i][k] * dAAE[j][l][c] +
                                            mu * dAAE[i][l][c] * AAE[j][k] + mu * AAE[i][l] * dAAE[j][k][c];
                                for (int a = 0; a < nadj; a++)
                                    for (int c = 0; c < 3; c++)
                                        vA[3 * a + c] = vA[3 * a + c] + dC[c] * strain[ij] * strainA[6 * a + kl];
                            }
                        }
                        for (int a = 0; a < nadj; a++)
                            for (int c = 0; c < 3; c++)
                                gint[a + nadj * (c + 3 * cp)] = gint[a + nadj * (c + 3 * cp)] - vA[3 * a + c] * Area * detJac;
                    }
                }
                if (compute_ext) {
                    /* body loads (centrifugal), gradUELMAT_solid.f90:370-457 */
                    for (int a = 0; a < nadj; a++)
                        for (int c = 0; c < 3; c++) {
                            double s = 0.0;
                            for (int cp = 0; cp < nn; cp++) s = s + R[cp] * UAe[3 * cp + c + 3 * nn * a];
                            vA[3 * a + c] = s;
                        }
                    int loadcount = 0;
                    int64_t kload = 0;
                    for (int nl = 0; nl < nb_load; nl++) {
                        if (jdltype[nl] == 101 && g_in_list(inddload + kload, load_target_nbelem[nl], jelem)) {
                            double pg[3] = {0, 0, 0}, A[3], B[3], vd[3], ag[3], vr[3], lf[3];
                            for (int cp = 0; cp < nn; cp++)
                                for (int c = 0; c < 3; c++) pg[c] = pg[c] + R[cp] * coords[3 * cp + c];
                            for (int c = 0; c < 3; c++) A[c] = addinfos[loadcount + c];
                            loadcount += 3;
                            for (int c = 0; c < 3; c++) B[c] = addinfos[loadcount + c];
                            loadcount += 3;
                            for (int c = 0; c < 3; c++) vd[c] = B[c] - A[c];
                            double nr = sqrt(vd[0] * vd[0] + vd[1] * vd[1] + vd[2] * vd[2]);
                            for (int c = 0; c < 3; c++) vd[c] = vd[c] / nr;
                            for (int c = 0; c < 3; c++) ag[c] = pg[c] - A[c];
                            double sc = g_dot(ag, vd);
                            for (int c = 0; c < 3; c++) vr[c] = ag[c] - sc * vd[c];
                            for (int c = 0; c < 3; c++) lf[c] = density * (adlmag[nl] * adlmag[nl]) * vr[c];
                            for (int cp = 0; cp < nn; cp++) {
                                const double *dr = dR + 3 * cp;
                                double dJ[3] = {0, 0, 0};
                                for (int i = 0; i < 3; i++)
                                    for (int c = 0; c < 3; c++) dJ[c] = dJ[c] + AxA[i][c] * dr[i];
                                for (int a = 0; a < nadj; a++) {
                                    double sf = g_dot(lf, vA + 3 * a);
                                    for (int c = 0; c < 3; c++)
                                        gext[a + nadj * (c + 3 * cp)] = gext[a + nadj * (c + 3 * cp)] + sf * dJ[c] * detJac;
                                }
                                for (int a = 0; a < nadj; a++) {
                                    double df[3] = {0, 0, 0};
                                    for (int id = 0; id < 3; id++)
                                        for (int jd = 0; jd < 3; jd++) {
                                            if (id == jd) df[jd] = df[jd] + vA[3 * a + id] * (1.0 - vd[id] * vd[jd]);
                                            else df[jd] = df[jd] - vA[3 * a + id] * (vd[id] * vd[jd]);
                                        }
                                    for (int c = 0; c < 3; c++) {
                                        df[c] = df[c] * (density * (adlmag[nl] * adlmag[nl]) * R[cp]);
                                        gext[a + nadj * (c + 3 * cp)] = gext[a + nadj * (c + 3 * cp)] + df[c] * Area * detJac;
                                    }
                                }
                            }
                        }
                        kload += load_target_nbelem[nl];
                    }
                }
            }
    if (compute_ext && include_surface) {
        int64_t kk = 0;
        int64_t cinfo = 0;
        (void)cinfo;
        for (int nl = 0; nl < nb_load; nl++) {
            int64_t ty = jdltype[nl];
            if (ty > 9 && ty < 100 && g_in_list(inddload + kk, load_target_nbelem[nl], jelem)) {
                int face = (int)(ty / 10), type = (int)(ty % 10);
                int ifield = type == 4 ? (int)addinfos[0] - 1 : 0;
                for (int jf = 0; jf < ng; jf++)
                    for (int if0 = 0; if0 < ng; if0++) {
                        double t[3], wq = gw[if0] * gw[jf];
                        switch (face) {
                        case 1: t[0] = -1.0; t[1] = gx[if0]; t[2] = gx[jf]; break;
                        case 2: t[0] = 1.0; t[1] = gx[if0]; t[2] = gx[jf]; break;
                        case 3: t[0] = gx[if0]; t[1] = -1.0; t[2] = gx[jf]; break;
                        case 4: t[0] = gx[if0]; t[1] = 1.0; t[2] = gx[jf]; break;
                        case 5: t[0] = gx[jf]; t[1] = gx[if0]; t[2] = -1.0; break;
                        default: t[0] = gx[jf]; t[1] = gx[if0]; t[2] = 1.0; break;
                        }
                        double xi[3], h[3];
                        for (int i = 0; i < 3; i++) {
                            xi[i] = ((u2[i] - u1[i]) * t[i] + (u2[i] + u1[i])) * 0.5;
                            h[i] = 0.5 * (u2[i] - u1[i]);
                        }
                        g_evalnurbs(p, U, ni, w, xi, R, dR);
                        double AJ[3][3] = {{0}};   /* AJ[b] = column b of the parent Jacobian */
                        for (int cp = 0; cp < nn; cp++)
                            for (int b = 0; b < 3; b++)
                                for (int c = 0; c < 3; c++) AJ[b][c] = AJ[b][c] + coords[3 * cp + c] * dR[3 * cp + b];
                        for (int b = 0; b < 3; b++)
                            for (int c = 0; c < 3; c++) AJ[b][c] = AJ[b][c] * h[b];
                        int ia, ib;   /* surface-measure pair (shapPress.f:164-175) */
                        switch (face) { case 1: case 2: ia = 1; ib = 2; break; case 3: case 4: ia = 2; ib = 0; break; default: ia = 0; ib = 1; }
                        int ip, iq;   /* normal orientation pair (shapPress.f:229-243) */
                        switch (face) {
                        case 1: ip = 1; iq = 2; break; case 2: ip = 2; iq = 1; break;
                        case 3: ip = 2; iq = 0; break; case 4: ip = 0; iq = 2; break;
                        case 5: ip = 0; iq = 1; break; default: ip = 1; iq = 0; break;
                        }
                        double fmag = adlmag[nl];
                        if (type == 4) {
                            fmag = 0.0;
                            for (int cp = 0; cp < nn; cp++)
                                fmag = fmag + nodal_dist[ifield + (int64_t)nb_n_dist * (ien_e[cp] - 1)] * R[cp];
                        }
                        for (int a = 0; a < nadj; a++)
                            for (int c = 0; c < 3; c++) {
                                double s = 0.0;
                                for (int cp = 0; cp < nn; cp++) s = s + R[cp] * UAe[3 * cp + c + 3 * nn * a];
                                vA[3 * a + c] = s;
                            }
                        for (int cp = 0; cp < nn; cp++) {
                            for (int a = 0; a < nadj; a++) {
                                double g[3];
                                const double *ua = vA + 3 * a;
                                if (type == 0 || type == 4) {
                                    /* d/dP (UA . (P x Q)) */
                                    double cP = dR[3 * cp + ip] * h[ip], cQ = dR[3 * cp + iq] * h[iq];
                                    double QxU[3], UxP[3];
                                    g_cross(AJ[iq], ua, QxU);
                                    g_cross(ua, AJ[ip], UxP);
                                    for (int c = 0; c < 3; c++) g[c] = cP * QxU[c] + cQ * UxP[c];
                                } else {
                                    /* d/dP (UA_t |A x B|) */
                                    double n[3];
                                    g_cross(AJ[ia], AJ[ib], n);
                                    double nr = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
                                    for (int c = 0; c < 3; c++) n[c] = n[c] / nr;
                                    double cA = dR[3 * cp + ia] * h[ia], cB = dR[3 * cp + ib] * h[ib];
                                    double Bxn[3], nxA[3];
                                    g_cross(AJ[ib], n, Bxn);
                                    g_cross(n, AJ[ia], nxA);
                                    for (int c = 0; c < 3; c++) g[c] = ua[type - 1] * (cA * Bxn[c] + cB * nxA[c]);
                                }
                                for (int c = 0; c < 3; c++)
                                    gext[a + nadj * (c + 3 * cp)] = gext[a + nadj * (c + 3 * cp)] + g[c] * wq * fmag;
                            }
                        }
                    }
            }
            kk += load_target_nbelem[nl];
        }
    }
    free(R); free(dR); free(dUA); free(strainA); free(stressA); free(work); free(vA);
}

/* gradLinElastWork_AN (gradtotalwork_fullAN.f90:107-300), U1 / 3D patches. */
int oracle_grad_lin_elast_work(
    int64_t nb_patch, int64_t nb_elem, int64_t nb_cp, const double *coords,
    const int64_t *ien, const int64_t *nb_elem_patch, const int64_t *nkv,
    const double *ukv, const int64_t *nijk, const double *weight,
    const int64_t *jpqr, const int64_t *nnode, const int64_t *nbint,
    const double *matprops, const double *rho, const int64_t *active,
    int64_t nb_load, const int64_t *inddload, const int64_t *jdltype,
    const double *adlmag, const int64_t *load_target_nbelem,
    const double *addinfos, int64_t nb_n_dist, const double *nodal_dist,
    const double *sol, const double *adj, int64_t nadj, int compute_int,
    int compute_ext, int include_surface, double *gwint, double *gwext)
{
    (void)nb_elem;
    memset(gwint, 0, sizeof(double) * nadj * 3 * nb_cp);
    memset(gwext, 0, sizeof(double) * nadj * 3 * nb_cp);
    int64_t jelem = 0, ukv_off = 0, ien_off = 0, w_off = 0;
    for (int64_t ip = 0; ip < nb_patch; ip++) {
        int p[3];
        const double *U[3];
        for (int d = 0; d < 3; d++) p[d] = (int)jpqr[3 * ip + d];
        U[0] = ukv + ukv_off;
        U[1] = U[0] + nkv[3 * ip];
        U[2] = U[1] + nkv[3 * ip + 1];
        int nn = (int)nnode[ip];
        if (nn > GMAXNN) return -3;
        /* elements in parallel (OpenMP), each into its own slot of gi_all /
         * ge_all; the scatter into gwint / gwext follows in element order,
         * so the sums have the bits of the sequential loop */
        const int64_t nep = nb_elem_patch[ip], j0 = jelem;
        const size_t ne = (size_t)nadj * 3 * nn;
        double *gi_all = (double *)calloc((size_t)nep * ne, sizeof(double));
        double *ge_all = (double *)calloc((size_t)nep * ne, sizeof(double));
#pragma omp parallel
        {
            double *ce = (double *)malloc(sizeof(double) * 3 * nn);
            double *ue = (double *)malloc(sizeof(double) * 3 * nn);
            double *uae = (double *)malloc(sizeof(double) * 3 * nn * nadj);
#pragma omp for schedule(dynamic, 4)
            for (int64_t ie = 0; ie < nep; ie++) {
                const int64_t je = j0 + ie;
                const int64_t *ien_e = ien + ien_off + ie * nn;
                if (active[je] != 1) continue;
                int ni[3];
                double u1[3], u2[3];
                for (int d = 0; d < 3; d++) {
                    ni[d] = (int)nijk[3 * je + d];
                    u1[d] = U[d][ni[d] - 1];
                    u2[d] = U[d][ni[d]];
                }
                for (int a = 0; a < nn; a++) {
                    int64_t cp = ien_e[a] - 1;
                    for (int c = 0; c < 3; c++) {
                        ce[3 * a + c] = coords[3 * cp + c];
                        ue[3 * a + c] = sol[3 * cp + c];
                        for (int k = 0; k < nadj; k++)
                            uae[3 * a + c + 3 * nn * k] = adj[k + nadj * (c + 3 * cp)];
                    }
                }
                g_element((int)nadj, nn, (int)nbint[ip], ce, ue, uae, p, U, ni, u1, u2,
                          weight + w_off + ie * nn, matprops[2 * ip], matprops[2 * ip + 1], rho[ip],
                          je + 1, (int)nb_load, inddload, load_target_nbelem, jdltype, adlmag,
                          addinfos, compute_int, compute_ext, include_surface, nodal_dist,
                          (int)nb_n_dist, ien_e, gi_all + ie * ne, ge_all + ie * ne);
            }
            free(ce); free(ue); free(uae);
        }
        for (int64_t ie = 0; ie < nep; ie++) {
            if (active[j0 + ie] != 1) continue;
            const int64_t *ien_e = ien + ien_off + ie * nn;
            const double *gi = gi_all + ie * ne, *ge = ge_all + ie * ne;
            for (int a = 0; a < nn; a++) {
                int64_t cp = ien_e[a] - 1;
                for (int c = 0; c < 3; c++)
                    for (int k = 0; k < nadj; k++) {
                        if (compute_int)
                            gwint[k + nadj * (c + 3 * cp)] = gwint[k + nadj * (c + 3 * cp)] + gi[k + nadj * (c + 3 * a)];
                        if (compute_ext)
                            gwext[k + nadj * (c + 3 * cp)] = gwext[k + nadj * (c + 3 * cp)] + ge[k + nadj * (c + 3 * a)];
                    }
            }
        }
        jelem += nep;
        free(gi_all); free(ge_all);
        for (int d = 0; d < 3; d++) ukv_off += nkv[3 * ip + d];
        ien_off += nb_elem_patch[ip] * nn;
        w_off += nb_elem_patch[ip] * nn;
    }
    return 0;
}

/* computeVolume (src/yeti_iga/optim/volume.f90:20-210) and computeGradVolume
 * (optim/gradvolume.f90:16-355), 3-D classical patches, restated loop for
 * loop: every element of a patch with listpatch = 1, every Gauss point,
 * VOL += det(AI) detJ and gradV(:, k) += (AIxAJ(:,3) dR(i,3) + AIxAJ(:,1)
 * dR(i,1) + AIxAJ(:,2) dR(i,2)) detJ as running sums.  grad may be NULL. */
int oracle_volume(int64_t nb_patch, int64_t nb_cp, const double *coords,
                  const int64_t *ien, const int64_t *nb_elem_patch, const int64_t *nkv,
                  const double *ukv, const int64_t *nijk, const double *weight,
                  const int64_t *jpqr, const int64_t *nnode, const int64_t *nbint,
                  const int64_t *listpatch, double *vol, double *grad)
{
    double V = 0.0;
    if (grad) memset(grad, 0, sizeof(double) * 3 * nb_cp);
    int64_t jelem = 0, ukv_off = 0, ien_off = 0;
    for (int64_t ip = 0; ip < nb_patch; ip++) {
        int p[3];
        const double *U[3];
        for (int d = 0; d < 3; d++) p[d] = (int)jpqr[3 * ip + d];
        U[0] = ukv + ukv_off;
        U[1] = U[0] + nkv[3 * ip];
        U[2] = U[1] + nkv[3 * ip + 1];
        int nn = (int)nnode[ip];
        if (nn > GMAXNN) return -3;
        if (listpatch[ip] == 1) {
            int nq = (int)nbint[ip];
            int ng = (int)pow((double)nq, 1.0 / 3.0);
            if (ng < 1) ng = 1;
            while (ng * ng * ng < nq) ng++;
            double gx[32], gw[32];
            g_gauss_legendre(ng, gx, gw);
            /* the terms of every Gauss point are evaluated in parallel
             * (OpenMP over elements) into term buffers; the running sums
             * are then replayed in the loop order above, so V and grad have
             * the bits of the sequential loop */
            const int64_t nep = nb_elem_patch[ip];
            const int nqe = ng * ng * ng < nq ? ng * ng * ng : nq;
            const size_t per_q = 1 + (grad ? 3 * (size_t)nn : 0);
            double *terms = (double *)malloc(sizeof(double) * (size_t)nep * nqe * per_q);
#pragma omp parallel
            {
                double *R = (double *)malloc(sizeof(double) * nn);
                double *dR = (double *)malloc(sizeof(double) * 3 * nn);
                double *ce = (double *)malloc(sizeof(double) * 3 * nn);
#pragma omp for schedule(dynamic, 4)
                for (int64_t ie = 0; ie < nep; ie++) {
                    const int64_t *ien_e = ien + ien_off + ie * nn;
                    const int64_t je = jelem + ie;
                    double *tq = terms + (size_t)ie * nqe * per_q;
                    int ni[3];
                    double u1[3], u2[3];
                    for (int d = 0; d < 3; d++) {
                        ni[d] = (int)nijk[3 * je + d];
                        u1[d] = U[d][ni[d] - 1];
                        u2[d] = U[d][ni[d]];
                    }
                    for (int a = 0; a < nn; a++)
                        for (int c = 0; c < 3; c++) ce[3 * a + c] = coords[3 * (ien_e[a] - 1) + c];
                    int q = 0;
                    for (int i0 = 0; i0 < ng; i0++)
                        for (int j0 = 0; j0 < ng; j0++)
                            for (int k0 = 0; k0 < ng; k0++, q++) {
                                if (q >= nq) break;
                                double t[3] = {gx[i0], gx[j0], gx[k0]};
                                double detJ = gw[i0] * gw[j0] * gw[k0], xi[3];
                                for (int i = 0; i < 3; i++) {
                                    xi[i] = ((u2[i] - u1[i]) * t[i] + (u2[i] + u1[i])) * 0.5;
                                    detJ = detJ * 0.5 * (u2[i] - u1[i]);
                                }
                                g_evalnurbs(p, U, ni, weight + ien_off + ie * nn, xi, R, dR);
                                double AI[3][3] = {{0}};   /* AI[k] = column k */
                                for (int k = 0; k < 3; k++)
                                    for (int a = 0; a < nn; a++)
                                        for (int c = 0; c < 3; c++)
                                            AI[k][c] = AI[k][c] + dR[3 * a + k] * ce[3 * a + c];
                                /* MatrixDet with AA(i, j) = AI[j-1][i-1] */
                                double det = AI[1][0] * AI[2][1] * AI[0][2] - AI[2][0] * AI[1][1] * AI[0][2] +
                                             AI[2][0] * AI[0][1] * AI[1][2] - AI[0][0] * AI[2][1] * AI[1][2] +
                                             AI[0][0] * AI[1][1] * AI[2][2] - AI[1][0] * AI[0][1] * AI[2][2];
                                double *tp = tq + (size_t)q * per_q;
                                tp[0] = det * detJ;
                                if (!grad) continue;
                                double AxA[3][3];
                                g_cross(AI[0], AI[1], AxA[2]);
                                g_cross(AI[1], AI[2], AxA[0]);
                                g_cross(AI[2], AI[0], AxA[1]);
                                for (int a = 0; a < nn; a++)
                                    for (int c = 0; c < 3; c++)
                                        tp[1 + 3 * a + c] =
                                            (AxA[2][c] * dR[3 * a + 2] + AxA[0][c] * dR[3 * a] +
                                             AxA[1][c] * dR[3 * a + 1]) * detJ;
                            }
                }
                free(R); free(dR); free(ce);
            }
            for (int64_t ie = 0; ie < nep; ie++) {
                const int64_t *ien_e = ien + ien_off + ie * nn;
                const double *tq = terms + (size_t)ie * nqe * per_q;
                for (int q = 0; q < nqe; q++) {
                    const double *tp = tq + (size_t)q * per_q;
                    V = V + tp[0];
                    if (!grad) continue;
                    for (int a = 0; a < nn; a++) {
                        int64_t k = ien_e[a] - 1;
                        for (int c = 0; c < 3; c++)
                            grad[c + 3 * k] = grad[c + 3 * k] + tp[1 + 3 * a + c];
                    }
                }
            }
            free(terms);
        }
        jelem += nb_elem_patch[ip];
        for (int d = 0; d < 3; d++) ukv_off += nkv[3 * ip + d];
        ien_off += nb_elem_patch[ip] * nn;
    }
    *vol = V;
    return 0;
}
