// Adjoint shape gradient of the linear-elastic work for U1 solids.
//
// Replaces gradadjointwork.gradlinelastwork_an: gradLinElastWork_AN
// (src/yeti_iga/optim/gradtotalwork_fullAN.f90:17-300) and gradUELMAT1adj
// (src/yeti_iga/optim/gradUELMAT_solid.f90:18-479), with evalnurbs
// (src/yeti_iga/main/evaluatenurbsfcts.f:94-209).  The quadrature-point
// geometry is recomputed from the control points (nothing is stored between
// the solve and the gradient).  Optionally adds the surface-load sensitivity
// the reference leaves out (gradUELMAT_solid.f90:463-477): for a load of
// magnitude f on a face, W_ext = f sum_q w_q UA(xi_q).v(xi_q) with
// v = P x Q (normal pressure, shapPress.f face ordering) or e_t |A x B|
// (fixed direction), differentiated through the face tangents.
//
// Kernel design: one CTA per active element.  Stage A: one thread per
// quadrature point computes the basis, covariant frame, metrics, strains and
// stresses of the state and adjoint fields into shared memory (all the
// points when their records fit, else chunk by chunk, every sum continued
// across the chunks in point order).  Stage B: one
// thread per control point accumulates its (nadj x 3) derivative over the
// points in order.  A second kernel sums element contributions per control
// point in element order (deterministic).  Compiled without FMA contraction
// and following the reference's operation order.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>

#include "nurbs.cuh"
#include "u1_model.cuh"

namespace yeti {

constexpr int kGradMaxAdj = 4;

__device__ __constant__ int c_vi[6] = {0, 1, 2, 0, 0, 1};
__device__ __constant__ int c_vj[6] = {0, 1, 2, 1, 2, 2};

struct GradArgs {
    int p0, p1, p2, nn, nq, ng, nadj, qchunk, pchunk;
    int compute_int, compute_ext, include_surface;
    const double *U0, *U1, *U2;
    const double *gauss;      // volume rule (4 * nq)
    const double *gface;      // 6 faces x ng^2 x 4
    const double *coords;
    const int32_t *ien;       // per active element
    const double *w;
    const int32_t *span;
    const int32_t *elems;     // elements of this launch (active-local index)
    const int32_t *term_ptr;  // loads of each element (CSR)
    const int32_t *terms;     // load indices
    const int32_t *jdltype;
    const double *adlmag;
    const double *addinfos;
    const double *nodal_dist;
    int nb_n_dist;
    const double *sol;        // (3, nb_cp)
    const double *adj;        // (nadj, 3, nb_cp)
    double E, nu, rho;
    double *egi, *ege;        // (n elements, nadj*3*nn)
};

// evalnurbs at parametric xi: R[nn], dR[3*a+i]
__device__ void eval_nurbs(const GradArgs &a, const int *ni, const double *xi,
                           const double *we, double *R, double *dR) {
    nurbs_eval_elem(a.p0, a.p1, a.p2, a.U0, a.U1, a.U2, a.nn, ni, xi, we, R, dR);
}

__device__ __forceinline__ void gcross(const double *u, const double *v, double *w) {
    w[0] = u[1] * v[2] - u[2] * v[1];
    w[1] = u[2] * v[0] - u[0] * v[2];
    w[2] = u[0] * v[1] - u[1] * v[0];
}

__device__ __forceinline__ double gdot(const double *u, const double *v) {
    return u[0] * v[0] + u[1] * v[1] + u[2] * v[2];
}

__device__ void ginv3(const double B[3][3], double A[3][3]) {
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
}

// Per-point record layout in shared memory (doubles).
struct PtLayout {
    int R, dR, AI, AxA, area, dj, AAE, strain, stress, dU, dUA, sA, tA, work,
        vA, body, size;
};

__host__ __device__ inline PtLayout pt_layout(int nn, int nadj, int nbody) {
    PtLayout L;
    int o = 0;
    L.R = o; o += nn;
    L.dR = o; o += 3 * nn;
    L.AI = o; o += 9;
    L.AxA = o; o += 9;
    L.area = o; o += 1;
    L.dj = o; o += 1;
    L.AAE = o; o += 9;
    L.strain = o; o += 6;
    L.stress = o; o += 6;
    L.dU = o; o += 9;
    L.dUA = o; o += 9 * nadj;
    L.sA = o; o += 6 * nadj;    // adjoint strain
    L.tA = o; o += 6 * nadj;    // adjoint stress
    L.work = o; o += nadj;
    L.vA = o; o += 3 * nadj;    // adjoint displacement at the point
    L.body = o; o += 6 * nbody; // (loadF, vectD) of each centrifugal load
    L.size = o;
    return L;
}

// Shared memory of one element: xe, ue, uae, we, then the point records
// (PtLayout) of one chunk of pchunk points, then the basis scratch
// (kBasisB1 + kStiffQS per point of the chunk), the external- and
// internal-work accumulators of the (control point, component) tasks and
// the term buffer of stage B (qchunk points).
__host__ __device__ inline size_t grad_smem_doubles(int nn, int pchunk, int nadj, const PtLayout &L,
                                                    size_t face, int qchunk) {
    const size_t vol = (size_t)pchunk * L.size;
    return (size_t)(6 + 3 * nadj) * nn + nn + (vol > face ? vol : face) +
           (size_t)pchunk * (kBasisB1 + kStiffQS) + (size_t)2 * 3 * nn * nadj +
           (size_t)3 * nn * qchunk * 3 * nadj;
}

// gradUELMAT1adj (gradUELMAT_solid.f90:18-479) of one element per CTA.
// Stage A evaluates the basis and the point quantities: the products of
// every (point, node) in parallel (basis_chunk), every sum over the nodes as
// one thread's loop in node order, then the per-point tensors (one thread
// per point).  Stage B runs one task per (control point, component c): every
// quantity the reference indexes by c -- dJ, the strain variations, dAAI,
// dAAE, dC and the accumulated gradient -- depends on that component alone,
// so each task performs exactly the operations the reference performs for
// its component, in the same order, and the results keep their bits.
__global__ void __launch_bounds__(256) k_u1_grad(GradArgs a) {
    extern __shared__ double sm[];
    const int nn = a.nn, nadj = a.nadj;
    const int e = a.elems[blockIdx.x];
    double *xe = sm;                    // 3*nn coords
    double *ue = xe + 3 * nn;           // 3*nn state
    double *uae = ue + 3 * nn;          // 3*nn*nadj adjoint
    double *we = uae + 3 * nn * nadj;   // nn weights
    double *pts = we + nn;
    __shared__ double su1[3], su2[3];
    __shared__ int sni[3];
    __shared__ int s_body[8], s_nbody;
    const int tid = threadIdx.x, nth = blockDim.x;
    const int32_t *ien = a.ien + (size_t)e * nn;
    for (int i = tid; i < nn; i += nth) {
        const int cp = ien[i];
        for (int c = 0; c < 3; c++) {
            xe[3 * i + c] = a.coords[3 * cp + c];
            ue[3 * i + c] = a.sol[3 * cp + c];
            for (int k = 0; k < nadj; k++)
                uae[3 * i + c + 3 * nn * k] = a.adj[k + nadj * (c + 3 * cp)];
        }
        we[i] = a.w[(size_t)e * nn + i];
    }
    if (tid < 3) {
        const double *U = tid == 0 ? a.U0 : (tid == 1 ? a.U1 : a.U2);
        const int ni = a.span[3 * e + tid];
        sni[tid] = ni;
        su1[tid] = U[ni - 1];
        su2[tid] = U[ni];
    }
    if (tid == 0) {
        int nb = 0;
        if (a.compute_ext)
            for (int t = a.term_ptr[blockIdx.x]; t < a.term_ptr[blockIdx.x + 1]; t++)
                if (a.jdltype[a.terms[t]] == 101 && nb < 8) s_body[nb++] = a.terms[t];
        s_nbody = nb;
    }
    __syncthreads();
    const int nbody = s_nbody;
    const PtLayout L = pt_layout(nn, nadj, nbody);
    const size_t face = (size_t)a.ng * a.ng * (4 * nn + 11 + 3 * nadj);
    const int pc = a.pchunk;
    const size_t vol = (size_t)pc * L.size;
    double *B1 = pts + (vol > face ? vol : face);
    double *qs = B1 + (size_t)pc * kBasisB1;
    double *ge_s = qs + (size_t)pc * kStiffQS;
    double *gi_s = ge_s + (size_t)3 * nn * nadj;   // 3 nn nadj accumulators
    double *terms = gi_s + (size_t)3 * nn * nadj;  // 3 nn qchunk 3 nadj terms
    const double lambda = a.E * a.nu / (1.0 + a.nu) / (1.0 - 2.0 * a.nu);
    const double mu = a.E / 2.0 / (1.0 + a.nu);
    for (int t = tid; t < 3 * nn * nadj; t += nth) gi_s[t] = ge_s[t] = 0.0;
    // The points are taken in chunks of pc (their records in shared memory);
    // every accumulator continues over the chunks in point order, so the
    // sums are the same sequences as over all points at once.
    for (int p0 = 0; p0 < a.nq; p0 += pc) {
        const int np = min(pc, a.nq - p0);
        __syncthreads();
        // ---------------- stage A: per volume point of the chunk
        {
            const int pd[3] = {a.p0, a.p1, a.p2};
            const double *Ud[3] = {a.U0, a.U1, a.U2};
            // R numerators and dR/dxi into the point records, dx/dxi into qs
            basis_chunk(pd, Ud, sni, su1, su2, a.gauss, p0, np, nn, xe, we, B1, pts + L.R, L.size,
                        pts + L.dR, L.size, qs);
        }
        for (int t = tid; t < np * nn; t += nth) {
            const int q = t / nn, n = t - q * nn;
            double *R = pts + (size_t)q * L.size + L.R;
            R[n] = R[n] * qs[(size_t)q * kStiffQS + 3];
        }
        if (a.compute_int) {
            // the gradients of the state and of the adjoints: ordered sums over
            // the nodes, one thread per (point, entry)
            const int ns = 9 * (1 + nadj);
            for (int t = tid; t < np * ns; t += nth) {
                const int q = t / ns, s = t - q * ns;
                double *P = pts + (size_t)q * L.size;
                const double *dR = P + L.dR;
                const int k = s / 9 - 1, ic = s % 9, i = ic / 3, c = ic % 3;
                const double *v = k < 0 ? ue : uae + 3 * nn * k;
                double acc = 0.0;
                for (int cp = 0; cp < nn; cp++) acc = acc + dR[3 * cp + i] * v[3 * cp + c];
                if (k < 0) P[L.dU + ic] = acc;
                else P[L.dUA + 9 * k + ic] = acc;
            }
        }
        __syncthreads();
        for (int ql = tid; ql < np; ql += nth) {
            const int q = ql;   // the point's record and basis scratch (chunk-local)
            double *P = pts + (size_t)q * L.size;
            const double *g = a.gauss + 4 * (p0 + ql);
            double detJac = g[0];
            for (int i = 0; i < 3; i++) detJac = detJac * 0.5 * (su2[i] - su1[i]);
            const double *R = P + L.R;
            double AI[3][3];
            for (int i = 0; i < 3; i++)
                for (int c = 0; c < 3; c++) AI[i][c] = qs[(size_t)q * kStiffQS + 4 + 3 * c + i];
            double AxA[3][3];
            gcross(AI[0], AI[1], AxA[2]);
            const double Area = gdot(AxA[2], AI[2]);
            gcross(AI[1], AI[2], AxA[0]);
            gcross(AI[2], AI[0], AxA[1]);
            for (int i = 0; i < 3; i++)
                for (int c = 0; c < 3; c++) {
                    P[L.AI + 3 * i + c] = AI[i][c];
                    P[L.AxA + 3 * i + c] = AxA[i][c];
                }
            P[L.area] = Area;
            P[L.dj] = detJac;
            if (a.compute_int) {
                double AAI[3][3], AAE[3][3];
                for (int i = 0; i < 3; i++)
                    for (int j = 0; j < 3; j++) AAI[i][j] = gdot(AI[i], AI[j]);
                ginv3(AAI, AAE);
                double H[6][6];
                for (int kl = 0; kl < 6; kl++) {
                    const int k = c_vi[kl], l = c_vj[kl];
                    for (int ij = 0; ij <= kl; ij++) {
                        const int i = c_vi[ij], j = c_vj[ij];
                        H[ij][kl] = lambda * AAE[i][j] * AAE[k][l] +
                                    mu * (AAE[i][k] * AAE[j][l] + AAE[i][l] * AAE[j][k]);
                    }
                }
                for (int kl = 1; kl < 6; kl++)
                    for (int r = kl; r < 6; r++) H[r][kl - 1] = H[kl - 1][r];
                double dU[3][3];
                for (int i = 0; i < 3; i++)
                    for (int c = 0; c < 3; c++) dU[i][c] = P[L.dU + 3 * i + c];
                double strain[6], stress[6];
                for (int ij = 0; ij < 6; ij++) {
                    const int i = c_vi[ij], j = c_vj[ij];
                    if (i == j) strain[ij] = gdot(AI[i], dU[i]);
                    else strain[ij] = gdot(AI[i], dU[j]) + gdot(AI[j], dU[i]);
                }
                for (int ii = 0; ii < 6; ii++) {
                    double s = 0.0;
                    for (int jj = 0; jj < 6; jj++) s = s + H[ii][jj] * strain[jj];
                    stress[ii] = s;
                }
                for (int i = 0; i < 3; i++)
                    for (int c = 0; c < 3; c++) P[L.AAE + 3 * i + c] = AAE[i][c];
                for (int ij = 0; ij < 6; ij++) {
                    P[L.strain + ij] = strain[ij];
                    P[L.stress + ij] = stress[ij];
                }
                for (int k = 0; k < nadj; k++) {
                    double dA[3][3];
                    for (int i = 0; i < 3; i++)
                        for (int c = 0; c < 3; c++) dA[i][c] = P[L.dUA + 9 * k + 3 * i + c];
                    double sA[6], tA[6];
                    for (int ij = 0; ij < 6; ij++) {
                        const int i = c_vi[ij], j = c_vj[ij];
                        if (i == j) sA[ij] = gdot(AI[i], dA[i]);
                        else sA[ij] = gdot(AI[i], dA[j]) + gdot(AI[j], dA[i]);
                    }
                    for (int ii = 0; ii < 6; ii++) {
                        double s = 0.0;
                        for (int jj = 0; jj < 6; jj++) s = s + H[ii][jj] * sA[jj];
                        tA[ii] = s;
                    }
                    for (int ij = 0; ij < 6; ij++) {
                        P[L.sA + 6 * k + ij] = sA[ij];
                        P[L.tA + 6 * k + ij] = tA[ij];
                    }
                }
                for (int k = 0; k < nadj; k++) P[L.work + k] = 0.0;
                for (int ij = 0; ij < 6; ij++)
                    for (int k = 0; k < nadj; k++)
                        P[L.work + k] = P[L.work + k] + P[L.sA + 6 * k + ij] * stress[ij];
            }
            if (a.compute_ext && nbody > 0) {
                for (int k = 0; k < nadj; k++)
                    for (int c = 0; c < 3; c++) {
                        double s = 0.0;
                        for (int cp = 0; cp < nn; cp++) s = s + R[cp] * uae[3 * cp + c + 3 * nn * k];
                        P[L.vA + 3 * k + c] = s;
                    }
                // centrifugal loads: the reference advances its info cursor by
                // 2*MCRD for every centrifugal load acting on the element
                int loadcount = 0;
                for (int b = 0; b < nbody; b++) {
                    const int nl = s_body[b];
                    double pg[3] = {0, 0, 0}, A[3], B[3], vd[3], ag[3];
                    for (int cp = 0; cp < nn; cp++)
                        for (int c = 0; c < 3; c++) pg[c] = pg[c] + R[cp] * xe[3 * cp + c];
                    for (int c = 0; c < 3; c++) A[c] = a.addinfos[loadcount + c];
                    loadcount += 3;
                    for (int c = 0; c < 3; c++) B[c] = a.addinfos[loadcount + c];
                    loadcount += 3;
                    for (int c = 0; c < 3; c++) vd[c] = B[c] - A[c];
                    const double nr = sqrt(vd[0] * vd[0] + vd[1] * vd[1] + vd[2] * vd[2]);
                    for (int c = 0; c < 3; c++) vd[c] = vd[c] / nr;
                    for (int c = 0; c < 3; c++) ag[c] = pg[c] - A[c];
                    const double sc = gdot(ag, vd);
                    for (int c = 0; c < 3; c++) {
                        P[L.body + 6 * b + c] = a.rho * (a.adlmag[nl] * a.adlmag[nl]) * (ag[c] - sc * vd[c]);
                        P[L.body + 6 * b + 3 + c] = vd[c];
                    }
                }
            }
        }
        __syncthreads();
        // ---------------- stage B: interior work, per (control point, component,
        // point) in parallel.  Each thread forms the three terms the reference
        // subtracts from the gradient at its point (work dJ detJ, the
        // stress-times-strain-variation term, the material-variation term); one
        // thread per (control point, component) then subtracts them in point
        // order, the reference's order, so the sums keep their bits.  Points are
        // taken in chunks of a.qchunk (the term buffer).
        if (a.compute_int) {
            for (int q0 = 0; q0 < np; q0 += a.qchunk) {
                const int nqc = min(a.qchunk, np - q0);
                __syncthreads();
                for (int t = tid; t < 3 * nn * nqc; t += nth) {
                    const int task = t / nqc, ql = t - task * nqc, q = q0 + ql;
                    const int cp = task / 3, c = task - 3 * cp;
                    const double *P = pts + (size_t)q * L.size;
                    const double *dr = P + L.dR + 3 * cp;
                    const double Area = P[L.area], detJac = P[L.dj];
                    const double *AxA = P + L.AxA;
                    const double *AI = P + L.AI, *AAE = P + L.AAE;
                    const double *stress = P + L.stress, *strain = P + L.strain, *dU = P + L.dU;
                    double *tt = terms + ((size_t)task * a.qchunk + ql) * 3 * nadj;
                    double dJ = 0.0;
                    for (int i = 0; i < 3; i++) dJ = dJ + AxA[3 * i + c] * dr[i];
                    for (int k = 0; k < nadj; k++) tt[3 * k] = P[L.work + k] * dJ * detJac;
                    for (int k = 0; k < nadj; k++) {
                        const double *d = P + L.dUA + 9 * k;
                        double ev = 0.0;
                        for (int ij = 0; ij < 6; ij++) {
                            const int i = c_vi[ij], j = c_vj[ij];
                            if (i == j) ev = ev + stress[ij] * d[3 * i + c] * dr[i];
                            else ev = ev + stress[ij] * d[3 * i + c] * dr[j] + stress[ij] * d[3 * j + c] * dr[i];
                        }
                        tt[3 * k + 1] = ev * Area * detJac;
                    }
                    double dAAI[3][3], dAAE[3][3];
                    for (int j = 0; j < 3; j++)
                        for (int i = 0; i < 3; i++) dAAI[i][j] = dr[i] * AI[3 * j + c] + AI[3 * i + c] * dr[j];
                    for (int i = 0; i < 3; i++)
                        for (int j = 0; j < 3; j++) dAAE[i][j] = 0.0;
                    for (int j = 0; j < 3; j++)
                        for (int i = 0; i < 3; i++)
                            for (int l = 0; l < 3; l++)
                                for (int k = 0; k < 3; k++)
                                    dAAE[i][j] = dAAE[i][j] - AAE[3 * i + k] * AAE[3 * l + j] * dAAI[k][l];
                    double vA[kGradMaxAdj];
                    for (int k = 0; k < nadj; k++) {
                        const double *tA = P + L.tA + 6 * k;
                        double ev = 0.0;
                        for (int ij = 0; ij < 6; ij++) {
                            const int i = c_vi[ij], j = c_vj[ij];
                            if (i == j) ev = ev + tA[ij] * dU[3 * i + c] * dr[i];
                            else ev = ev + tA[ij] * dU[3 * i + c] * dr[j] + tA[ij] * dU[3 * j + c] * dr[i];
                        }
                        vA[k] = ev;
                    }
                    for (int kl = 0; kl < 6; kl++) {
                        const int k = c_vi[kl], l = c_vj[kl];
                        for (int ij = 0; ij < 6; ij++) {
                            const int i = c_vi[ij], j = c_vj[ij];
                            const double dC =
                                lambda * dAAE[i][j] * AAE[3 * k + l] + lambda * AAE[3 * i + j] * dAAE[k][l] +
                                mu * dAAE[i][k] * AAE[3 * j + l] + mu * AAE[3 * i + k] * dAAE[j][l] +
                                mu * dAAE[i][l] * AAE[3 * j + k] + mu * AAE[3 * i + l] * dAAE[j][k];
                            for (int kk = 0; kk < nadj; kk++)
                                vA[kk] = vA[kk] + dC * strain[ij] * P[L.sA + 6 * kk + kl];
                        }
                    }
                    for (int k = 0; k < nadj; k++) tt[3 * k + 2] = vA[k] * Area * detJac;
                }
                __syncthreads();
                for (int task = tid; task < 3 * nn; task += nth)
                    for (int k = 0; k < nadj; k++) {
                        double g = gi_s[task * nadj + k];
                        for (int ql = 0; ql < nqc; ql++) {
                            const double *tt = terms + ((size_t)task * a.qchunk + ql) * 3 * nadj + 3 * k;
                            g = g - tt[0];
                            g = g - tt[1];
                            g = g - tt[2];
                        }
                        gi_s[task * nadj + k] = g;
                    }
            }
        }
        // ---------------- stage B': body-load work, one task per (control
        // point, component), points in order
        for (int task = tid; task < 3 * nn; task += nth) {
            const int cp = task / 3, c = task - 3 * cp;
            double ge[kGradMaxAdj];
            for (int k = 0; k < kGradMaxAdj; k++) ge[k] = k < nadj ? ge_s[task * nadj + k] : 0.0;
            if (a.compute_ext && nbody > 0) {
                for (int q = 0; q < np; q++) {
                    const double *P = pts + (size_t)q * L.size;
                    const double *dr = P + L.dR + 3 * cp;
                    const double Area = P[L.area], detJac = P[L.dj];
                    const double *AxA = P + L.AxA;
                    for (int b = 0; b < nbody; b++) {
                        const double *lf = P + L.body + 6 * b, *vd = lf + 3;
                        const int nl = s_body[b];
                        double dJ = 0.0;
                        for (int i = 0; i < 3; i++) dJ = dJ + AxA[3 * i + c] * dr[i];
                        for (int k = 0; k < nadj; k++) {
                            const double sf = gdot(lf, P + L.vA + 3 * k);
                            ge[k] = ge[k] + sf * dJ * detJac;
                        }
                        for (int k = 0; k < nadj; k++) {
                            const double *ua = P + L.vA + 3 * k;
                            double df = 0.0;
                            for (int id = 0; id < 3; id++) {
                                if (id == c) df = df + ua[id] * (1.0 - vd[id] * vd[c]);
                                else df = df - ua[id] * (vd[id] * vd[c]);
                            }
                            df = df * (a.rho * (a.adlmag[nl] * a.adlmag[nl]) * P[L.R + cp]);
                            ge[k] = ge[k] + df * Area * detJac;
                        }
                    }
                }
            }
            for (int k = 0; k < nadj; k++) ge_s[task * nadj + k] = ge[k];
        }
    }   // point chunks
    __syncthreads();
    {
        double *oi = a.egi + (size_t)blockIdx.x * nadj * 3 * nn;
        for (int task = tid; task < 3 * nn; task += nth) {
            const int cp = task / 3, c = task - 3 * cp;
            for (int k = 0; k < nadj; k++) oi[k + nadj * (c + 3 * cp)] = gi_s[task * nadj + k];
        }
    }
    // ---------------- surface loads (not in the reference)
    if (a.compute_ext && a.include_surface) {
        const int nf = a.ng * a.ng;
        for (int t = a.term_ptr[blockIdx.x]; t < a.term_ptr[blockIdx.x + 1]; t++) {
            const int nl = a.terms[t];
            const int ty = a.jdltype[nl];
            if (!(ty > 9 && ty < 100)) continue;
            const int face = ty / 10, type = ty % 10;
            // per face point: R (nn), dR (3nn), AJ (9), fmag, w, vA (3nadj)
            const int fs = 4 * nn + 11 + 3 * nadj;
            __syncthreads();
            for (int q = tid; q < nf; q += nth) {
                double *P = pts + (size_t)q * fs;
                const double *g = a.gface + ((size_t)(face - 1) * nf + q) * 4;
                double xi[3], h[3];
                for (int i = 0; i < 3; i++) {
                    xi[i] = ((su2[i] - su1[i]) * g[1 + i] + (su2[i] + su1[i])) * 0.5;
                    h[i] = 0.5 * (su2[i] - su1[i]);
                }
                double *R = P, *dR = P + nn;
                eval_nurbs(a, sni, xi, we, R, dR);
                double AJ[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
                for (int cq = 0; cq < nn; cq++)
                    for (int b = 0; b < 3; b++)
                        for (int c = 0; c < 3; c++) AJ[b][c] = AJ[b][c] + xe[3 * cq + c] * dR[3 * cq + b];
                for (int b = 0; b < 3; b++)
                    for (int c = 0; c < 3; c++) P[4 * nn + 3 * b + c] = AJ[b][c] * h[b];
                double fmag = a.adlmag[nl];
                if (type == 4) {
                    const int ifield = (int)a.addinfos[0] - 1;
                    fmag = 0.0;
                    for (int cq = 0; cq < nn; cq++)
                        fmag = fmag + a.nodal_dist[ifield + (size_t)a.nb_n_dist * ien[cq]] * R[cq];
                }
                P[4 * nn + 9] = fmag;
                P[4 * nn + 10] = g[0];
                for (int k = 0; k < nadj; k++)
                    for (int c = 0; c < 3; c++) {
                        double s = 0.0;
                        for (int cq = 0; cq < nn; cq++) s = s + R[cq] * uae[3 * cq + c + 3 * nn * k];
                        P[4 * nn + 11 + 3 * k + c] = s;
                    }
            }
            __syncthreads();
            int ia, ib, ip, iq;
            switch (face) { case 1: case 2: ia = 1; ib = 2; break; case 3: case 4: ia = 2; ib = 0; break; default: ia = 0; ib = 1; }
            switch (face) {
                case 1: ip = 1; iq = 2; break; case 2: ip = 2; iq = 1; break;
                case 3: ip = 2; iq = 0; break; case 4: ip = 0; iq = 2; break;
                case 5: ip = 0; iq = 1; break; default: ip = 1; iq = 0; break;
            }
            double h[3];
            for (int i = 0; i < 3; i++) h[i] = 0.5 * (su2[i] - su1[i]);
            for (int task = tid; task < 3 * nn; task += nth) {
                const int cp = task / 3, c = task - 3 * cp;
                double ge[kGradMaxAdj];
                for (int k = 0; k < nadj; k++) ge[k] = ge_s[task * nadj + k];
                for (int q = 0; q < nf; q++) {
                    const double *P = pts + (size_t)q * fs;
                    const double *dR = P + nn;
                    const double *AJ = P + 4 * nn;
                    const double fmag = P[4 * nn + 9], wq = P[4 * nn + 10];
                    for (int k = 0; k < nadj; k++) {
                        const double *ua = P + 4 * nn + 11 + 3 * k;
                        double gg;
                        if (type == 0 || type == 4) {
                            const double cP = dR[3 * cp + ip] * h[ip], cQ = dR[3 * cp + iq] * h[iq];
                            double QxU[3], UxP[3];
                            gcross(AJ + 3 * iq, ua, QxU);
                            gcross(ua, AJ + 3 * ip, UxP);
                            gg = cP * QxU[c] + cQ * UxP[c];
                        } else {
                            double n[3];
                            gcross(AJ + 3 * ia, AJ + 3 * ib, n);
                            const double nr = sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
                            for (int cc = 0; cc < 3; cc++) n[cc] = n[cc] / nr;
                            const double cA = dR[3 * cp + ia] * h[ia], cB = dR[3 * cp + ib] * h[ib];
                            double Bxn[3], nxA[3];
                            gcross(AJ + 3 * ib, n, Bxn);
                            gcross(n, AJ + 3 * ia, nxA);
                            gg = ua[type - 1] * (cA * Bxn[c] + cB * nxA[c]);
                        }
                        ge[k] = ge[k] + gg * wq * fmag;
                    }
                }
                for (int k = 0; k < nadj; k++) ge_s[task * nadj + k] = ge[k];
            }
        }
    }
    __syncthreads();
    double *oe = a.ege + (size_t)blockIdx.x * nadj * 3 * nn;
    for (int task = tid; task < 3 * nn; task += nth) {
        const int cp = task / 3, c = task - 3 * cp;
        for (int k = 0; k < nadj; k++) oe[k + nadj * (c + 3 * cp)] = ge_s[task * nadj + k];
    }
}

// g[k + nadj*(c + 3*cp)] = sum over elements (in order) of their entries
__global__ void k_grad_gather(int64_t n, const int64_t *ptr, const int64_t *idx,
                              const double *egi, const double *ege, double *gi,
                              double *ge) {
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (t >= n) return;
    double ai = 0.0, ae = 0.0;
    for (int64_t k = ptr[t]; k < ptr[t + 1]; k++) {
        ai = ai + egi[idx[k]];
        ae = ae + ege[idx[k]];
    }
    gi[t] = ai;
    ge[t] = ae;
}

static bool in_list_g(const int64_t *l, int64_t n, int64_t v) {
    for (int64_t i = 0; i < n; i++)
        if (l[i] == v) return true;
    return false;
}

}  // namespace yeti

using namespace yeti;

YETI_API int yeti_grad_lin_elast_work(yeti_ctx *ctx, const yeti_u1_model *m,
                                      const double *sol, const double *adj,
                                      int64_t nadj, int compute_wint,
                                      int compute_wext, int include_surface,
                                      double *gwint, double *gwext, int mem) {
    YETI_CHECK(ctx && m && sol && adj && gwint && gwext, YETI_EINVAL,
               "yeti_grad_lin_elast_work: NULL argument");
    YETI_CHECK(nadj >= 1 && nadj <= kGradMaxAdj, YETI_EINVAL,
               "yeti_grad_lin_elast_work: nadj %lld outside 1..%d", (long long)nadj, kGradMaxAdj);
    DeviceGuard guard(ctx->device);
    U1Model M;
    YETI_TRY(u1_prepare(ctx, m, M));
    cudaStream_t s = ctx->stream;
    const int64_t ncp = m->nb_cp;
    const int64_t nout = nadj * 3 * ncp;
    DevBuf dsol, dadj, dgi, dge;
    const double *sol_d = sol, *adj_d = adj;
    double *gi_d = gwint, *ge_d = gwext;
    if (mem == YETI_MEM_HOST) {
        YETI_TRY(upload(ctx, dsol, sol, (size_t)3 * ncp));
        YETI_TRY(upload(ctx, dadj, adj, (size_t)nout));
        YETI_TRY(dgi.alloc(ctx, nout * sizeof(double)));
        YETI_TRY(dge.alloc(ctx, nout * sizeof(double)));
        sol_d = dsol.as<double>();
        adj_d = dadj.as<double>();
        gi_d = dgi.as<double>();
        ge_d = dge.as<double>();
    }
    int smem_optin = 0;
    YETI_CUDA(cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device));
    cudaFuncAttributes fattr;
    YETI_CUDA(cudaFuncGetAttributes(&fattr, k_u1_grad));
    smem_optin -= (int)fattr.sharedSizeBytes;   // the kernel's static shared memory
    std::vector<std::unique_ptr<DevBuf>> keep;
    auto newbuf = [&keep]() -> DevBuf & {
        keep.emplace_back(new DevBuf());
        return *keep.back();
    };
    DevBuf dj, da, dinfo, dnd;
    std::vector<int32_t> jdl(m->nb_load > 0 ? m->nb_load : 1, 0);
    for (int64_t i = 0; i < m->nb_load; i++) jdl[i] = (int32_t)m->jdltype[i];
    YETI_TRY(upload(ctx, dj, jdl.data(), jdl.size()));
    std::vector<double> adl(m->nb_load > 0 ? m->nb_load : 1, 0.0);
    for (int64_t i = 0; i < m->nb_load; i++) adl[i] = m->adlmag[i];
    YETI_TRY(upload(ctx, da, adl.data(), adl.size()));
    std::vector<double> inf(m->len_load_addinfos > 0 ? m->len_load_addinfos : 1, 0.0);
    for (int64_t i = 0; i < m->len_load_addinfos; i++) inf[i] = m->load_addinfos[i];
    YETI_TRY(upload(ctx, dinfo, inf.data(), inf.size()));
    if (m->nodal_dist && m->nb_n_dist > 0)
        YETI_TRY(upload(ctx, dnd, m->nodal_dist, (size_t)m->nb_n_dist * m->nb_cp));
    // element contributions, in global element order
    struct Done { int patch; int64_t local; int64_t off; };
    std::vector<Done> done;
    std::vector<DevBuf *> ebufs_i, ebufs_e;
    std::vector<int64_t> ien_offset(M.patches.size(), 0);
    for (size_t ip = 1; ip < M.patches.size(); ip++)
        ien_offset[ip] = ien_offset[ip - 1] + M.patches[ip - 1].nelem * M.patches[ip - 1].nn;
    int64_t etotal = 0;
    for (size_t ip = 0; ip < M.patches.size(); ip++) {
        U1Patch &P = M.patches[ip];
        if (!P.nactive) continue;
        YETI_CHECK(P.nn <= 256, YETI_EUNSUPPORTED,
                   "shape gradient: elements with more than 256 nodes are not supported");
        std::vector<int32_t> elems, tptr(1, 0), terms;
        int max_body = 0;
        for (int64_t le = 0; le < P.nactive; le++) {
            const int64_t jel = P.act[le] + 1;
            int64_t k2 = 0;
            int nb = 0;
            for (int64_t il = 0; il < m->nb_load; il++) {
                const int64_t nt = m->load_target_nbelem[il], ty = m->jdltype[il];
                if ((ty == 101 || (ty > 9 && ty < 100)) && in_list_g(m->inddload + k2, nt, jel)) {
                    terms.push_back((int32_t)il);
                    nb += ty == 101;
                    if (ty == 4 % 10 && 0) {}
                }
                k2 += nt;
            }
            YETI_CHECK(nb <= 8, YETI_EUNSUPPORTED, "more than 8 centrifugal loads on one element");
            max_body = std::max(max_body, nb);
            elems.push_back((int32_t)le);
            tptr.push_back((int32_t)terms.size());
            done.push_back({(int)ip, le, etotal});
            etotal += nadj * 3 * P.nn;
        }
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
        if (terms.empty()) terms.push_back(0);
        YETI_TRY(upload(ctx, dtm, terms.data(), terms.size()));
        DevBuf &bi = newbuf();
        DevBuf &be = newbuf();
        YETI_TRY(bi.alloc(ctx, sizeof(double) * nadj * 3 * P.nn * elems.size()));
        YETI_TRY(be.alloc(ctx, sizeof(double) * nadj * 3 * P.nn * elems.size()));
        ebufs_i.push_back(&bi);
        ebufs_e.push_back(&be);
        GradArgs g;
        g.p0 = P.p[0]; g.p1 = P.p[1]; g.p2 = P.p[2];
        g.nn = P.nn; g.nq = P.nq; g.ng = P.ng; g.nadj = (int)nadj;
        g.compute_int = compute_wint; g.compute_ext = compute_wext;
        g.include_surface = include_surface;
        g.U0 = P.knots.as<double>(); g.U1 = g.U0 + P.nkv[0]; g.U2 = g.U1 + P.nkv[1];
        g.gauss = P.gauss.as<double>();
        g.gface = dgf.as<double>();
        g.coords = M.coords.as<double>();
        g.ien = P.ien.as<int32_t>();
        g.w = P.w.as<double>();
        g.span = P.span.as<int32_t>();
        g.elems = del.as<int32_t>();
        g.term_ptr = dtp.as<int32_t>();
        g.terms = dtm.as<int32_t>();
        g.jdltype = dj.as<int32_t>();
        g.adlmag = da.as<double>();
        g.addinfos = dinfo.as<double>();
        g.nodal_dist = dnd.ptr ? dnd.as<double>() : nullptr;
        g.nb_n_dist = (int)m->nb_n_dist;
        g.sol = sol_d;
        g.adj = adj_d;
        g.E = P.E; g.nu = P.nu; g.rho = P.rho;
        g.egi = bi.as<double>();
        g.ege = be.as<double>();
        const PtLayout L = pt_layout(P.nn, (int)nadj, max_body);
        const size_t face = (size_t)P.ng * P.ng * (4 * P.nn + 11 + 3 * nadj);
        // term buffer of stage B: up to 6144 doubles (48 KB), whole chunks of points
        const int qchunk = (int)std::max<int64_t>(
            1, std::min<int64_t>(P.nq, 6144 / (9 * (int64_t)P.nn * nadj)));
        // point records: all the points when they fit, else the largest
        // chunk that does (at least the term buffer's)
        int pchunk = P.nq;
        while (pchunk > qchunk &&
               sizeof(double) * grad_smem_doubles(P.nn, pchunk, (int)nadj, L, face, qchunk) > (size_t)smem_optin)
            pchunk--;
        g.qchunk = std::min(qchunk, pchunk);
        g.pchunk = pchunk;
        const size_t smem = sizeof(double) * grad_smem_doubles(P.nn, pchunk, (int)nadj, L, face, g.qchunk);
        YETI_CHECK(smem <= (size_t)smem_optin, YETI_EUNSUPPORTED,
                   "shape gradient: element needs %zu bytes of shared memory", smem);
        YETI_TRY(set_smem_optin((const void *)k_u1_grad, ctx->device, smem, "shape gradient element"));
        KernelTimer timer(ctx, "k_u1_grad");
        k_u1_grad<<<(unsigned)elems.size(), 256, smem, s>>>(g);
        count_launches(1);
        YETI_CUDA(cudaGetLastError());
    }
    // gather per (adjoint, component, control point) in element order
    DevBuf &ai = newbuf();
    DevBuf &ae = newbuf();
    YETI_TRY(ai.alloc(ctx, sizeof(double) * std::max<int64_t>(etotal, 1)));
    YETI_TRY(ae.alloc(ctx, sizeof(double) * std::max<int64_t>(etotal, 1)));
    {
        int64_t off = 0;
        for (size_t i = 0; i < ebufs_i.size(); i++) {
            YETI_CUDA(cudaMemcpyAsync(ai.as<double>() + off, ebufs_i[i]->ptr, ebufs_i[i]->bytes, cudaMemcpyDeviceToDevice, s));
            YETI_CUDA(cudaMemcpyAsync(ae.as<double>() + off, ebufs_e[i]->ptr, ebufs_e[i]->bytes, cudaMemcpyDeviceToDevice, s));
            off += (int64_t)(ebufs_i[i]->bytes / sizeof(double));
        }
    }
    // CSR of the element entries of each output, elements in order: count,
    // then fill in the same loop order
    std::vector<int64_t> ptr(nout + 1, 0);
    auto walk = [&](auto &&visit) {
        for (auto &D : done) {
            const U1Patch &P = M.patches[D.patch];
            const int64_t jel = P.act[D.local];
            const int64_t base = ien_offset[D.patch] + (jel - P.elem_begin) * P.nn;
            for (int a = 0; a < P.nn; a++) {
                const int64_t cp = m->ien[base + a] - 1;
                for (int c = 0; c < 3; c++)
                    for (int k = 0; k < nadj; k++)
                        visit(k + nadj * (c + 3 * cp), D.off + k + nadj * (c + 3 * a));
            }
        }
    };
    walk([&](int64_t o, int64_t) { ptr[o + 1]++; });
    for (int64_t i = 0; i < nout; i++) ptr[i + 1] += ptr[i];
    std::vector<int64_t> idx(std::max<int64_t>(ptr[nout], 1), 0), fill(ptr.begin(), ptr.end() - 1);
    walk([&](int64_t o, int64_t e) { idx[fill[o]++] = e; });
    DevBuf &dptr = newbuf();
    DevBuf &didx = newbuf();
    YETI_TRY(upload(ctx, dptr, ptr.data(), ptr.size()));
    YETI_TRY(upload(ctx, didx, idx.data(), idx.size()));
    k_grad_gather<<<(unsigned)((nout + 255) / 256), 256, 0, s>>>(
        nout, dptr.as<int64_t>(), didx.as<int64_t>(), ai.as<double>(), ae.as<double>(), gi_d, ge_d);
    count_launches(1);
    YETI_CUDA(cudaGetLastError());
    if (!compute_wint) YETI_CUDA(cudaMemsetAsync(gi_d, 0, nout * sizeof(double), s));
    if (!compute_wext) YETI_CUDA(cudaMemsetAsync(ge_d, 0, nout * sizeof(double), s));
    if (mem == YETI_MEM_HOST) {
        YETI_CUDA(cudaMemcpyAsync(gwint, gi_d, nout * sizeof(double), cudaMemcpyDeviceToHost, s));
        YETI_CUDA(cudaMemcpyAsync(gwext, ge_d, nout * sizeof(double), cudaMemcpyDeviceToHost, s));
    }
    YETI_CUDA(cudaStreamSynchronize(s));
    return YETI_OK;
}
