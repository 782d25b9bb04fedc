/*
 * CPU oracle / baseline of the weighted-quadrature elastic operator with the
 * reference's own algorithm.  TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).
 *
 * The reference applies its WQ operator with tensor3d_sparsedot_vector
 * (src/yeti_iga/iga_wq_mf/fsrc/tensor_algebra.f90:369-486): every output entry
 * is one rank-one dot product of the three CSR rows with the gathered input
 * block -- O(nnz_u nnz_v nnz_w) per output, not sum-factorised -- under an
 * OpenMP loop over outputs.  mf_wq_get_ku_3d (mf_wq_solver.f90:284-544) calls
 * it once per trial derivative (forward, with B^T) and once per
 * (test, trial) pair (backward, with W), scaling by the pointwise
 * coefficients in between.  This file restates that structure for the
 * elastic operator defined in oracle/wq_ops.py (B-spline test and trial
 * functions on the exact NURBS geometry: 9 forward and 27 backward products
 * per apply), and restates jacobien_physicalposition_3d /
 * eval_mech_coefficient (wq_assembly.f90:233-473, 52-138) for the
 * coefficients, with the NURBS weights in the geometry map and the geometric
 * orientation of the inverse Jacobian.
 */
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    int nrows, ncols;
    int *ptr, *idx;
    double *val;
} csr_t;

typedef struct {
    int n[3], q[3];
    int64_t ncp, nqp;
    csr_t BT[3][2];   /* B0^T, B1^T: (nqp_d x nfun_d) */
    csr_t W[3][4];    /* W00 W01 W10 W11: (nfun_d x nqp_d) */
    csr_t WB[3][4];   /* W_t (.) B_(t & 1), elementwise (nfun_d x nqp_d): diagonal */
    double *coef;     /* nqp * 45: upper triangle of S */
    unsigned char *mask;   /* 3*ncp: 1 free, 0 clamped */
} wq_t;

static int sym9(int I, int J)
{
    if (I > J) { int t = I; I = J; J = t; }
    return I * 9 - I * (I - 1) / 2 + (J - I);
}

static void csr_from_dense(csr_t *m, const double *A, int nr, int nc, int transpose)
{
    /* A: nr x nc row-major; transpose builds A^T */
    int R = transpose ? nc : nr, C = transpose ? nr : nc;
    m->nrows = R;
    m->ncols = C;
    m->ptr = (int *)calloc(R + 1, sizeof(int));
    int nnz = 0;
    for (int r = 0; r < R; r++)
        for (int c = 0; c < C; c++) {
            double v = transpose ? A[(size_t)c * nc + r] : A[(size_t)r * nc + c];
            if (v != 0.0) nnz++;
        }
    m->idx = (int *)malloc(sizeof(int) * (nnz + 1));
    m->val = (double *)malloc(sizeof(double) * (nnz + 1));
    nnz = 0;
    for (int r = 0; r < R; r++) {
        for (int c = 0; c < C; c++) {
            double v = transpose ? A[(size_t)c * nc + r] : A[(size_t)r * nc + c];
            if (v != 0.0) {
                m->idx[nnz] = c;
                m->val[nnz] = v;
                nnz++;
            }
        }
        m->ptr[r + 1] = nnz;
    }
}

static void csr_free(csr_t *m)
{
    free(m->ptr);
    free(m->idx);
    free(m->val);
}

/* out[iu,iv,iw] += sum (Mu[iu,:] x Mv[iv,:] x Mw[iw,:]) . in
 * (tensor3d_sparsedot_vector, u fastest in both index spaces) */
static void sparsedot3(const csr_t *Mu, const csr_t *Mv, const csr_t *Mw,
                       const double *in, double *out)
{
    const int ru = Mu->nrows, rv = Mv->nrows, rw = Mw->nrows;
    const int cu = Mu->ncols, cv = Mv->ncols;
    #pragma omp parallel for collapse(2) schedule(static)
    for (int iw = 0; iw < rw; iw++)
        for (int iv = 0; iv < rv; iv++)
            for (int iu = 0; iu < ru; iu++) {
                double sum = 0.0;
                for (int kw = Mw->ptr[iw]; kw < Mw->ptr[iw + 1]; kw++) {
                    const double aw = Mw->val[kw];
                    const int jw = Mw->idx[kw];
                    for (int kv = Mv->ptr[iv]; kv < Mv->ptr[iv + 1]; kv++) {
                        const double avw = aw * Mv->val[kv];
                        const int jv = Mv->idx[kv];
                        const double *row = in + ((size_t)jw * cv + jv) * cu;
                        for (int ku = Mu->ptr[iu]; ku < Mu->ptr[iu + 1]; ku++)
                            sum += avw * Mu->val[ku] * row[Mu->idx[ku]];
                    }
                }
                out[((size_t)iw * rv + iv) * ru + iu] += sum;
            }
}

int oracle_wq_threads(void) { return omp_get_max_threads(); }

/* rules: for each direction d, dense (nfun_d x nqp_d) row-major arrays in the
 * order B0, B1, W00, W01, W10, W11 (6 pointers per direction). */
void *oracle_wq_create(const int *n, const int *q, const double *const *rules,
                       const double *cps, const double *w, double E, double nu,
                       const unsigned char *mask)
{
    wq_t *op = (wq_t *)calloc(1, sizeof(wq_t));
    for (int d = 0; d < 3; d++) {
        op->n[d] = n[d];
        op->q[d] = q[d];
        const double *const *R = rules + 6 * d;
        csr_from_dense(&op->BT[d][0], R[0], n[d], q[d], 1);
        csr_from_dense(&op->BT[d][1], R[1], n[d], q[d], 1);
        for (int t = 0; t < 4; t++) csr_from_dense(&op->W[d][t], R[2 + t], n[d], q[d], 0);
        /* find_physical_diag_3d (tensor_algebra.f90:1484-1596) contracts the
         * coefficient with the products (W (.) B) of each direction */
        double *wb = (double *)malloc(sizeof(double) * (size_t)n[d] * q[d]);
        for (int t = 0; t < 4; t++) {
            const double *B = R[t & 1];
            for (size_t k = 0; k < (size_t)n[d] * q[d]; k++) wb[k] = R[2 + t][k] * B[k];
            csr_from_dense(&op->WB[d][t], wb, n[d], q[d], 0);
        }
        free(wb);
    }
    op->ncp = (int64_t)n[0] * n[1] * n[2];
    op->nqp = (int64_t)q[0] * q[1] * q[2];
    op->mask = (unsigned char *)malloc(3 * op->ncp);
    memcpy(op->mask, mask, 3 * op->ncp);
    op->coef = (double *)malloc(sizeof(double) * 45 * op->nqp);
    /* geometry: forward products of (w x, w y, w z, w) with B0/B1 */
    const int64_t NQ = op->nqp;
    double *F = (double *)calloc((size_t)16 * NQ, sizeof(double));
    double *in = (double *)malloc(sizeof(double) * op->ncp);
    for (int c = 0; c < 4; c++) {
        for (int64_t a = 0; a < op->ncp; a++) in[a] = c < 3 ? w[a] * cps[3 * a + c] : w[a];
        for (int l = 0; l < 4; l++)
            sparsedot3(&op->BT[0][l == 1], &op->BT[1][l == 2], &op->BT[2][l == 3], in,
                       F + (size_t)(4 * l + c) * NQ);
    }
    free(in);
    /* MDM = MM^T DD MM (wq_assembly.f90:92-109) */
    double lam = (E * nu) / ((1.0 + nu) * (1.0 - 2.0 * nu)), mu = E / (2.0 * (1.0 + nu));
    double DD[6][6] = {{0}};
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) DD[i][j] = lam;
    for (int i = 0; i < 3; i++) DD[i][i] = lam + 2.0 * mu;
    DD[3][3] = DD[4][4] = DD[5][5] = mu;
    double MM[6][9] = {{0}};
    const int nz[9][2] = {{0, 0}, {1, 4}, {2, 8}, {3, 1}, {3, 3}, {4, 5}, {4, 7}, {5, 2}, {5, 6}};
    for (int e = 0; e < 9; e++) MM[nz[e][0]][nz[e][1]] = 1.0;
    double MDM[9][9];
    for (int a = 0; a < 9; a++)
        for (int b = 0; b < 9; b++) {
            double s = 0.0;
            for (int r = 0; r < 6; r++)
                for (int t = 0; t < 6; t++) s += MM[r][a] * DD[r][t] * MM[t][b];
            MDM[a][b] = s;
        }
    #pragma omp parallel for schedule(static)
    for (int64_t qq = 0; qq < NQ; qq++) {
        double f[4][4];
        for (int l = 0; l < 4; l++)
            for (int c = 0; c < 4; c++) f[l][c] = F[(size_t)(4 * l + c) * NQ + qq];
        double W = f[0][3], x[3], J[3][3];
        for (int c = 0; c < 3; c++) x[c] = f[0][c] / W;
        for (int c = 0; c < 3; c++)
            for (int l = 0; l < 3; l++) J[c][l] = (f[l + 1][c] - x[c] * f[l + 1][3]) / W;
        double det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
                     J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
                     J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
        double id = 1.0 / det, iJ[3][3];
        iJ[0][0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) * id;
        iJ[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) * id;
        iJ[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) * id;
        iJ[1][0] = (J[1][2] * J[2][0] - J[1][0] * J[2][2]) * id;
        iJ[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * id;
        iJ[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * id;
        iJ[2][0] = (J[1][0] * J[2][1] - J[1][1] * J[2][0]) * id;
        iJ[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * id;
        iJ[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * id;
        double scale = fabs(det);
        double *co = op->coef + 45 * qq;
        for (int I = 0; I < 9; I++)
            for (int Jn = I; Jn < 9; Jn++) {
                int i = I / 3, k = I % 3, j = Jn / 3, l = Jn % 3;
                double s = 0.0;
                for (int d = 0; d < 3; d++)
                    for (int ff = 0; ff < 3; ff++)
                        s += iJ[k][d] * MDM[3 * i + d][3 * j + ff] * iJ[l][ff];
                co[sym9(I, Jn)] = s * scale;
            }
    }
    free(F);
    return op;
}

void oracle_wq_free(void *h)
{
    wq_t *op = (wq_t *)h;
    if (!op) return;
    for (int d = 0; d < 3; d++) {
        csr_free(&op->BT[d][0]);
        csr_free(&op->BT[d][1]);
        for (int t = 0; t < 4; t++) {
            csr_free(&op->W[d][t]);
            csr_free(&op->WB[d][t]);
        }
    }
    free(op->coef);
    free(op->mask);
    free(op);
}

/* Ku = K u (component-major vectors of 3*ncp) */
int oracle_wq_apply(void *h, const double *u, double *Ku)
{
    wq_t *op = (wq_t *)h;
    const int64_t NC = op->ncp, NQ = op->nqp;
    double *v = (double *)malloc(sizeof(double) * NC);
    double *F = (double *)calloc((size_t)9 * NQ, sizeof(double));
    /* F[(3*l + j)] = d u_j / d xi_(l+1) at the points */
    for (int j = 0; j < 3; j++) {
        for (int64_t a = 0; a < NC; a++) v[a] = op->mask[j * NC + a] ? u[j * NC + a] : 0.0;
        for (int l = 0; l < 3; l++)
            sparsedot3(&op->BT[0][l == 0], &op->BT[1][l == 1], &op->BT[2][l == 2], v,
                       F + (size_t)(3 * l + j) * NQ);
    }
    double *H = (double *)malloc(sizeof(double) * 9 * NQ);
    double *out = (double *)malloc(sizeof(double) * NC);
    for (int i = 0; i < 3; i++) {
        #pragma omp parallel for schedule(static)
        for (int64_t qq = 0; qq < NQ; qq++) {
            const double *co = op->coef + 45 * qq;
            double f[3][3];
            for (int l = 0; l < 3; l++)
                for (int j = 0; j < 3; j++) f[l][j] = F[(size_t)(3 * l + j) * NQ + qq];
            for (int k = 0; k < 3; k++)
                for (int l = 0; l < 3; l++) {
                    double a = 0.0;
                    for (int j = 0; j < 3; j++) a += co[sym9(3 * i + k, 3 * j + l)] * f[l][j];
                    H[(size_t)(3 * k + l) * NQ + qq] = a;
                }
        }
        memset(out, 0, sizeof(double) * NC);
        for (int ch = 0; ch < 9; ch++) {
            int kap = ch / 3, lam = ch % 3;
            sparsedot3(&op->W[0][2 * (kap == 0) + (lam == 0)],
                       &op->W[1][2 * (kap == 1) + (lam == 1)],
                       &op->W[2][2 * (kap == 2) + (lam == 2)], H + (size_t)ch * NQ, out);
        }
        for (int64_t a = 0; a < NC; a++) Ku[i * NC + a] = op->mask[i * NC + a] ? out[a] : 0.0;
    }
    free(v);
    free(F);
    free(H);
    free(out);
    return 0;
}

/* Seconds of the vector work of one CG iteration (two dots, three axpy-like
 * updates and the Jacobi scaling over n entries), timed once. */
double oracle_cg_vector_seconds(int64_t n, int reps)
{
    double *x = (double *)calloc(n, sizeof(double)), *r = (double *)malloc(sizeof(double) * n),
           *p = (double *)malloc(sizeof(double) * n), *Ap = (double *)malloc(sizeof(double) * n),
           *z = (double *)malloc(sizeof(double) * n), *di = (double *)malloc(sizeof(double) * n);
    for (int64_t i = 0; i < n; i++) { r[i] = 1.0; p[i] = 0.5; Ap[i] = 0.25; di[i] = 0.9; }
    double t0 = omp_get_wtime(), acc = 0.0;
    for (int k = 0; k < reps; k++) {
        double pAp = 0.0, rz = 0.0;
        #pragma omp parallel for reduction(+ : pAp)
        for (int64_t i = 0; i < n; i++) pAp += p[i] * Ap[i];
        double a = 1e-3 / (pAp + 1.0);
        #pragma omp parallel for reduction(+ : rz)
        for (int64_t i = 0; i < n; i++) {
            x[i] += a * p[i];
            r[i] -= a * Ap[i];
            z[i] = di[i] * r[i];
            rz += r[i] * z[i];
        }
        double b = rz / (rz + 1.0);
        #pragma omp parallel for
        for (int64_t i = 0; i < n; i++) p[i] = z[i] + b * p[i];
        acc += rz;
    }
    double t = (omp_get_wtime() - t0) / reps;
    free(x); free(r); free(p); free(Ap); free(z); free(di);
    return acc > -1.0 ? t : -t;
}

/* Diagonal of K (3*ncp; clamped dofs 1): for component c, the sum over the
 * 9 (test, trial) derivative pairs (k, l) of the rank-one products of
 * W_(k,l) (.) B_l in the three directions with the coefficient
 * S[(c,k),(c,l)] -- find_physical_diag_3d (tensor_algebra.f90:1484-1596)
 * per diagonal block, as wq_find_conductivity_diagonal_3d
 * (mf_wq_solver.f90:6-164) calls it. */
int oracle_wq_diag(void *h, double *d)
{
    wq_t *op = (wq_t *)h;
    const int64_t NC = op->ncp, NQ = op->nqp;
    double *cf = (double *)malloc(sizeof(double) * NQ);
    double *out = (double *)malloc(sizeof(double) * NC);
    for (int c = 0; c < 3; c++) {
        memset(out, 0, sizeof(double) * NC);
        for (int k = 0; k < 3; k++)
            for (int l = 0; l < 3; l++) {
                const int e = sym9(3 * c + k, 3 * c + l);
                #pragma omp parallel for schedule(static)
                for (int64_t qq = 0; qq < NQ; qq++) cf[qq] = op->coef[45 * qq + e];
                sparsedot3(&op->WB[0][2 * (k == 0) + (l == 0)], &op->WB[1][2 * (k == 1) + (l == 1)],
                           &op->WB[2][2 * (k == 2) + (l == 2)], cf, out);
            }
        for (int64_t a = 0; a < NC; a++) d[c * NC + a] = op->mask[c * NC + a] ? out[a] : 1.0;
    }
    free(cf);
    free(out);
    return 0;
}

/* `iters` consecutive iterations of the Jacobi-preconditioned CG of
 * wq_mf_cg_3d (mf_wq_solver.f90:764-802: apply, alpha = r.z / p.Ap, x and r
 * updates, z = r / diag, beta, p update) from x = 0, on the host cores, the
 * whole loop timed as one.  Returns seconds per iteration; x (3*ncp) holds
 * the iterate and *relres ||r||_2 / ||b||_2 on return. */
double oracle_wq_pcg_seconds(void *h, const double *b, const double *diag, int iters, double *x,
                             double *relres)
{
    wq_t *op = (wq_t *)h;
    const int64_t n = 3 * op->ncp;
    double *r = (double *)malloc(sizeof(double) * n), *z = (double *)malloc(sizeof(double) * n),
           *p = (double *)malloc(sizeof(double) * n), *Ap = (double *)malloc(sizeof(double) * n);
    double rz = 0.0, bb = 0.0;
    #pragma omp parallel for reduction(+ : rz, bb)
    for (int64_t i = 0; i < n; i++) {
        x[i] = 0.0;
        r[i] = op->mask[i] ? b[i] : 0.0;
        z[i] = r[i] / diag[i];
        p[i] = z[i];
        rz += r[i] * z[i];
        bb += r[i] * r[i];
    }
    double rr = bb;
    const double t0 = omp_get_wtime();
    for (int k = 0; k < iters; k++) {
        oracle_wq_apply(h, p, Ap);
        double pAp = 0.0;
        #pragma omp parallel for reduction(+ : pAp)
        for (int64_t i = 0; i < n; i++) pAp += p[i] * Ap[i];
        const double alpha = rz / pAp;
        double rzn = 0.0;
        rr = 0.0;
        #pragma omp parallel for reduction(+ : rzn, rr)
        for (int64_t i = 0; i < n; i++) {
            x[i] += alpha * p[i];
            r[i] -= alpha * Ap[i];
            z[i] = r[i] / diag[i];
            rzn += r[i] * z[i];
            rr += r[i] * r[i];
        }
        const double beta = rzn / rz;
        rz = rzn;
        #pragma omp parallel for
        for (int64_t i = 0; i < n; i++) p[i] = z[i] + beta * p[i];
    }
    const double t = (omp_get_wtime() - t0) / (iters > 0 ? iters : 1);
    *relres = sqrt(rr / bb);
    free(r); free(z); free(p); free(Ap);
    return t;
}
