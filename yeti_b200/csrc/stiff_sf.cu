// Sum-factorised U1 element stiffness: the same COO slots and values as the
// point-by-pair kernel of assemble_u1.cu (stiffmatrix.F90:130-225,
// UELMAT.f90:109-171), with the B^T D B contraction done direction by
// direction over the 1-D basis tables instead of pair by pair.  The sums run
// in another order, so the values agree with the reference to rounding
// (relative 1e-14 on the test meshes), not bit for bit.
//
// Factorisation
// -------------
// With N_a = N1_{i1}(q1) N2_{i2}(q2) N3_{i3}(q3) the B-spline product of
// local node a, W = sum_a w_a N_a and W_d = sum_a w_a dN_a/dxi_d, the
// physical gradient of the rational function R_a = w_a N_a / W is
//
//     dR_a/dx_r = w_a sum_kappa Phi^kappa_a(q) c^kappa_r(q),
//
// over the four kinds kappa = value, d/du, d/dv, d/dw of the tensor product
// (Phi^value = N_a, Phi^u = N1' N2 N3, ...) with the point coefficients
// c^{d}_r = Jinv[d][r] / W and c^{value}_r = -sum_d W_d Jinv[d][r] / W^2.
// For the isotropic D of stiffmatrix.F90:167-216 the 3x3 block of a node
// pair is
//
//     K_kl(a, b) = lam G_kl + mu G_lk + [k = l] mu (G_00 + G_11 + G_22),
//     G_rs(a, b) = sum_q dv(q) dR_a/dx_r dR_b/dx_s,
//
// so the nine integrals G_rs carry the element matrix; they are contracted
// along w, then v, then u.  After the w contraction the value and d/dw kinds
// share their factors in u and v (class 0), d/du is class 1 and d/dv class
// 2; after v only the kind along u (value or derivative) remains.  Each
// contraction runs one side (the row node a) and then the other (b).  For
// one pair (i3, j3) of w indices the steps cost about 81 g^3,
// 30 n2 g^3 + 27 n2^2 g^2 and 36 n1 n2^2 g + 18 n1^2 n2^2 g multiply-adds
// (n = p+1 functions, g Gauss points per direction); only the pairs
// i3 <= j3 are needed, the slots hold the upper triangle.
//
// One CTA per element.  Shared memory holds the point coefficients (13 per
// point), T1 = G_rs per class pair and (q1, q2), and T2 per u-kind pair, i2,
// j2 and q1.  The u contraction runs in lane groups of three (one r each,
// the three s in registers); lane r gathers the column G_{k,r} and the
// diagonal from the other two with warp shuffles and writes column l = r of
// the node pair's slot (three values; diagonal pair: r + 1), consecutive
// groups taking consecutive row nodes, whose slots are contiguous.
#include "nurbs.cuh"
#include "u1_model.cuh"

namespace yeti {

constexpr int kSfThreads = 256;
constexpr int kSfMaxG = 8;   // Gauss points per direction (template instances)

struct SfArgs {
    int n[3];        // functions per direction (p+1)
    int p[3];
    int nn;          // nodes
    const double *U[3];
    const double *gauss;   // 4 * g^3: weight, t1, t2, t3 (t3 fastest)
    const double *coords;
    const int32_t *ien;
    const double *w;
    const int32_t *span;
    const int64_t *slot;
    double lam, mu;
    double *kdata;
    int32_t *krow, *kcol;
};

// Shared-memory doubles of one CTA.
// The control-point coordinates (3 nn) are needed only by the per-point
// pass and share their space with T1/T2.
size_t sf_smem_doubles(const int n[3], int g) {
    const size_t nn = (size_t)n[0] * n[1] * n[2], nq = (size_t)g * g * g;
    const size_t work = 81 * (size_t)g * g + 36 * (size_t)n[1] * n[1] * g;
    return nn + (nn + 1) / 2 + 2 * (size_t)g * (n[0] + n[1] + n[2]) + 13 * nq +
           (work > 3 * nn ? work : 3 * nn);
}

__device__ __forceinline__ double det3(const double J[3][3]) {
    return J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
           J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
           J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
}

// Three CTAs per SM for g <= 4 (registers capped at 85), two above.
template <int G>
__global__ void __launch_bounds__(kSfThreads, G <= 4 ? 3 : 2) k_u1_stiffness_sf(SfArgs a) {
    extern __shared__ double smem[];
    constexpr int g = G, gg = G * G, nq = G * G * G;
    const int n1 = a.n[0], n2 = a.n[1], n3 = a.n[2], nn = a.nn;
    const int n12 = n1 * n2;
    double *we = smem;                        // nn
    int *sien = reinterpret_cast<int *>(we + nn);   // nn ints
    double *A1 = we + nn + (nn + 1) / 2;      // A_d[kind][i][q], d = u, v, w
    double *A2 = A1 + 2 * n1 * g, *A3 = A2 + 2 * n2 * g;
    double *cq = A3 + 2 * n3 * g;             // 13 nq: c[kind][r], dv
    double *T1 = cq + 13 * nq;                // [rs][ck ce][q1 q2]
    double *T2 = T1 + 81 * gg;                // [rs][al be][i2][j2][q1]
    double *xe = T1;                          // 3 nn, per-point pass only
    __shared__ double su1[3], su2[3];
    __shared__ int sni[3];
    const int e = blockIdx.x, tid = threadIdx.x;
    const int32_t *ien = a.ien + (size_t)e * nn;
    for (int i = tid; i < nn; i += kSfThreads) {
        const int cp = ien[i];
        sien[i] = cp;
        xe[3 * i] = a.coords[3 * cp];
        xe[3 * i + 1] = a.coords[3 * cp + 1];
        xe[3 * i + 2] = a.coords[3 * cp + 2];
        we[i] = a.w[(size_t)e * nn + i];
    }
    if (tid < 3) {
        const int ni = a.span[3 * e + tid];
        sni[tid] = ni;
        su1[tid] = a.U[tid][ni - 1];
        su2[tid] = a.U[tid][ni];
    }
    __syncthreads();
    // ---- 1-D tables: local index i uses the span's function p - i
    // (descending local node order of the reference's IEN)
    if (tid < 3 * g) {
        const int d = tid / g, q = tid - d * g;
        const int qq = d == 0 ? q * gg : (d == 1 ? q * g : q);
        const double t = a.gauss[4 * qq + 1 + d];
        const double xi = ((su2[d] - su1[d]) * t + (su2[d] + su1[d])) * 0.5;
        double N[kMaxDeg1], dN[kMaxDeg1];
        bspline_ders(sni[d], a.p[d], xi, a.U[d], N, dN);
        const int nd = a.n[d];
        double *A = d == 0 ? A1 : (d == 1 ? A2 : A3);
        for (int i = 0; i < nd; i++) {
            A[i * g + q] = N[a.p[d] - i];
            A[(nd + i) * g + q] = dN[a.p[d] - i];
        }
    }
    __syncthreads();
    // ---- per point: W, dW, x sums -> Jacobian, its inverse, dv, c
    for (int q = tid; q < nq; q += kSfThreads) {
        const int q1 = q / gg, q2 = (q / g) % g, q3 = q % g;
        double W = 0, Wd[3] = {0, 0, 0}, P[4][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        int n = 0;
        for (int i3 = 0; i3 < n3; i3++) {
            const double c0 = A3[i3 * g + q3], c1 = A3[(n3 + i3) * g + q3];
            for (int i2 = 0; i2 < n2; i2++) {
                const double b0 = A2[i2 * g + q2], b1 = A2[(n2 + i2) * g + q2];
                const double v23 = b0 * c0, d2 = b1 * c0, d3 = b0 * c1;
                for (int i1 = 0; i1 < n1; i1++, n++) {
                    const double a0 = A1[i1 * g + q1], a1 = A1[(n1 + i1) * g + q1];
                    const double wn = we[n];
                    const double ph[4] = {a0 * v23 * wn, a1 * v23 * wn, a0 * d2 * wn, a0 * d3 * wn};
                    W += ph[0];
                    Wd[0] += ph[1];
                    Wd[1] += ph[2];
                    Wd[2] += ph[3];
#pragma unroll
                    for (int k = 0; k < 4; k++)
#pragma unroll
                        for (int r = 0; r < 3; r++) P[k][r] += xe[3 * n + r] * ph[k];
                }
            }
        }
        const double iW = 1.0 / W;
        double J[3][3], Ji[3][3];
        for (int r = 0; r < 3; r++)
            for (int d = 0; d < 3; d++) J[r][d] = (P[d + 1][r] - P[0][r] * Wd[d] * iW) * iW;
        const double det = det3(J), idet = 1.0 / det;
        Ji[0][0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) * idet;
        Ji[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) * idet;
        Ji[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) * idet;
        Ji[1][0] = (J[1][2] * J[2][0] - J[1][0] * J[2][2]) * idet;
        Ji[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * idet;
        Ji[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * idet;
        Ji[2][0] = (J[1][0] * J[2][1] - J[1][1] * J[2][0]) * idet;
        Ji[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * idet;
        Ji[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * idet;
        // dv = w_q |det(J diag(h/2))| (shap.f90:155-178)
        const double hs = 0.125 * (su2[0] - su1[0]) * (su2[1] - su1[1]) * (su2[2] - su1[2]);
        double *c = cq + 13 * q;
        for (int r = 0; r < 3; r++) {
            c[r] = -(Wd[0] * Ji[0][r] + Wd[1] * Ji[1][r] + Wd[2] * Ji[2][r]) * iW * iW;
            for (int d = 0; d < 3; d++) c[3 * (d + 1) + r] = Ji[d][r] * iW;
        }
        c[12] = a.gauss[4 * q] * fabs(det * hs);
    }
    const int64_t base_slot = a.slot[e];
    const double lam = a.lam, mu = a.mu;
    for (int i3 = 0; i3 < n3; i3++)
        for (int j3 = i3; j3 < n3; j3++) {
            __syncthreads();
            // ---- step 1 (w): T1[rs][ck ce][q1 q2] = sum_q3 dv Pa_r Pb_s, with
            // P^{class}_r(i3, q) = sum_{kinds of the class} A3[kind along w][i3][q3] c_r
            for (int t = tid; t < 9 * gg; t += kSfThreads) {
                const int cc = t / gg, q12 = t - cc * gg, ck = cc / 3, ce = cc - 3 * ck;
                double acc[9];
#pragma unroll
                for (int k = 0; k < 9; k++) acc[k] = 0.0;
#pragma unroll
                for (int q3 = 0; q3 < G; q3++) {
                    const double *c = cq + 13 * (q12 * g + q3);
                    const double ai0 = A3[i3 * g + q3], bj0 = A3[j3 * g + q3];
                    double pa[3], pb[3];
                    if (ck == 0) {
                        const double ai1 = A3[(n3 + i3) * g + q3];
#pragma unroll
                        for (int r = 0; r < 3; r++) pa[r] = ai0 * c[r] + ai1 * c[9 + r];
                    } else {
#pragma unroll
                        for (int r = 0; r < 3; r++) pa[r] = ai0 * c[3 * ck + r];
                    }
                    if (ce == 0) {
                        const double bj1 = A3[(n3 + j3) * g + q3];
#pragma unroll
                        for (int s = 0; s < 3; s++) pb[s] = bj0 * c[s] + bj1 * c[9 + s];
                    } else {
#pragma unroll
                        for (int s = 0; s < 3; s++) pb[s] = bj0 * c[3 * ce + s];
                    }
                    const double dv = c[12];
#pragma unroll
                    for (int r = 0; r < 3; r++) {
                        const double pd = pa[r] * dv;
#pragma unroll
                        for (int s = 0; s < 3; s++) acc[3 * r + s] += pd * pb[s];
                    }
                }
#pragma unroll
                for (int rs = 0; rs < 9; rs++) T1[(rs * 9 + cc) * gg + q12] = acc[rs];
            }
            __syncthreads();
            // ---- step 2 (v): T2[rs][al be][i2][j2][q1]; along u the classes
            // 0 and 2 carry the value kind, class 1 the derivative.  One task
            // per (rs, i2, q1) for both u-kinds al, so each A2 value read
            // serves six multiply-adds.
            for (int t = tid; t < 9 * n2 * g; t += kSfThreads) {
                int r = t;
                const int q1 = r % g; r /= g;
                const int i2 = r % n2;
                const int rs = r / n2;
                const double *t1 = T1 + rs * 9 * gg + q1 * g;
                double V[2][3][G];   // V[al][ce][q2] = sum_{ck of u-kind al} A2 T1
#pragma unroll
                for (int q2 = 0; q2 < G; q2++) {
                    const double b0 = A2[i2 * g + q2], b1 = A2[(n2 + i2) * g + q2];
#pragma unroll
                    for (int ce = 0; ce < 3; ce++) {
                        V[0][ce][q2] = b0 * t1[(0 * 3 + ce) * gg + q2] + b1 * t1[(2 * 3 + ce) * gg + q2];
                        V[1][ce][q2] = b0 * t1[(1 * 3 + ce) * gg + q2];
                    }
                }
                double *t2 = T2 + ((size_t)rs * 4 * n2 + i2) * n2 * g + q1;
                const size_t sk = (size_t)n2 * n2 * g;   // stride of the (al, be) index
                for (int j2 = 0; j2 < n2; j2++) {
                    double s00 = 0.0, s01 = 0.0, s10 = 0.0, s11 = 0.0;
#pragma unroll
                    for (int q2 = 0; q2 < G; q2++) {
                        const double c0 = A2[j2 * g + q2], c1 = A2[(n2 + j2) * g + q2];
                        s00 += c0 * V[0][0][q2] + c1 * V[0][2][q2];
                        s01 += c0 * V[0][1][q2];
                        s10 += c0 * V[1][0][q2] + c1 * V[1][2][q2];
                        s11 += c0 * V[1][1][q2];
                    }
                    t2[j2 * g] = s00;
                    t2[sk + j2 * g] = s01;
                    t2[2 * sk + j2 * g] = s10;
                    t2[3 * sk + j2 * g] = s11;
                }
            }
            __syncthreads();
            // ---- steps 3 (u) and 4 (the COO slot): lanes in groups of three
            // (r = 0, 1, 2) per (a12, j2), ten groups per warp; each lane
            // contracts the three G_rs of its r along u and, with the
            // column G_{k,r} gathered through warp shuffles, writes column
            // l = r of the pair's slot (consecutive groups take consecutive
            // row nodes, whose slots are contiguous)
            {
                const int warp = tid >> 5, lane = tid & 31, gl = lane / 3, rr = lane - 3 * gl;
                const int ngroups = n12 * n2;
                const size_t sk = (size_t)n2 * n2 * g;
                for (int g0 = 10 * warp; g0 < ngroups; g0 += 10 * (kSfThreads / 32)) {
                    const int grp = g0 + gl;
                    const bool act = gl < 10 && grp < ngroups;
                    const int a12 = act ? grp % n12 : 0, j2 = act ? grp / n12 : 0;
                    const int i1 = a12 % n1, i2 = a12 / n1;
                    double Uu[3][2][G];   // Uu[s][be][q1] = sum_al A1[al][i1][q1] T2[3rr+s][al be]
#pragma unroll
                    for (int q1 = 0; q1 < G; q1++) {
                        const double a0 = A1[i1 * g + q1], a1 = A1[(n1 + i1) * g + q1];
#pragma unroll
                        for (int ss = 0; ss < 3; ss++) {
                            const double *t2 = T2 + (((size_t)(3 * rr + ss) * 4 * n2 + i2) * n2 + j2) * g + q1;
                            Uu[ss][0][q1] = a0 * t2[0] + a1 * t2[2 * sk];
                            Uu[ss][1][q1] = a0 * t2[sk] + a1 * t2[3 * sk];
                        }
                    }
                    const int ia = a12 + n12 * i3;
                    const int base = 3 * gl;
                    for (int j1 = 0; j1 < n1; j1++) {
                        double o[3] = {0.0, 0.0, 0.0};
#pragma unroll
                        for (int q1 = 0; q1 < G; q1++) {
                            const double c0 = A1[j1 * g + q1], c1 = A1[(n1 + j1) * g + q1];
#pragma unroll
                            for (int ss = 0; ss < 3; ss++) o[ss] += c0 * Uu[ss][0][q1] + c1 * Uu[ss][1][q1];
                        }
                        // K_kl = lam G_kl + mu G_lk + [k=l] mu tr G.  Lane rr writes
                        // column l = rr of the slot: it holds the row G_{rr,s} (o[s]);
                        // the column G_{k,rr} comes from lanes k by two rotating
                        // shuffles (at step t a lane sends o[(rr - t) mod 3], which
                        // is what lane (rr - t) mod 3 of the group reads), the trace
                        // from the three diagonals.
                        const double dg = rr == 0 ? o[0] : rr == 1 ? o[1] : o[2];
                        const double s1 = rr == 0 ? o[2] : rr == 1 ? o[0] : o[1];
                        const double s2 = rr == 0 ? o[1] : rr == 1 ? o[2] : o[0];
                        const int l1 = (base + (rr == 2 ? 0 : rr + 1)) & 31;   // lane (rr+1)%3
                        const int l2 = (base + (rr == 0 ? 2 : rr - 1)) & 31;   // lane (rr+2)%3
                        const double c1 = __shfl_sync(0xffffffffu, s1, l1);   // G_{(rr+1)%3, rr}
                        const double c2 = __shfl_sync(0xffffffffu, s2, l2);   // G_{(rr+2)%3, rr}
                        const double d1 = __shfl_sync(0xffffffffu, dg, l1);
                        const double d2 = __shfl_sync(0xffffffffu, dg, l2);
                        const int ib = j1 + n1 * j2 + n12 * j3;
                        if (!act || ia > ib) continue;
                        const double wab = we[ia] * we[ib];
                        // the trace summed as G_00 + G_11 + G_22 on every lane
                        const double t0 = rr == 0 ? dg : rr == 1 ? d2 : d1;
                        const double t1 = rr == 0 ? d1 : rr == 1 ? dg : d2;
                        const double t2 = rr == 0 ? d2 : rr == 1 ? d1 : dg;
                        const double tr = mu * (wab * t0 + wab * t1 + wab * t2);
                        double col[3], row[3];
#pragma unroll
                        for (int kk = 0; kk < 3; kk++) {
                            const int dk = kk - rr;   // 0, 1 or 2 steps down the column
                            col[kk] = wab * (dk == 0 ? dg : (dk == 1 || dk == -2) ? c1 : c2);
                            row[kk] = wab * o[kk];
                        }
                        const int dofa = 3 * sien[ia], dofb = 3 * sien[ib];
                        const int ll = rr;
                        if (ia < ib) {
                            const int64_t s0 = base_slot + 9LL * ib * (ib - 1) / 2 + 6LL * ib + 9LL * ia + 3 * ll;
#pragma unroll
                            for (int kk = 0; kk < 3; kk++) {
                                double v = lam * col[kk] + mu * row[kk];
                                if (kk == ll) v += tr;
                                a.kdata[s0 + kk] = v;
                                a.krow[s0 + kk] = dofa + kk;
                                a.kcol[s0 + kk] = dofb + ll;
                            }
                        } else {
                            const int64_t s0 = base_slot + 9LL * ia * (ia - 1) / 2 + 15LL * ia + ll * (ll + 1) / 2;
#pragma unroll
                            for (int kk = 0; kk < 3; kk++) {
                                if (kk > ll) continue;
                                double v = lam * col[kk] + mu * row[kk];
                                if (kk == ll) v = (v + tr) * 0.5;
                                a.kdata[s0 + kk] = v;
                                a.krow[s0 + kk] = dofa + kk;
                                a.kcol[s0 + kk] = dofa + ll;
                            }
                        }
                    }
                }
            }
        }
}

int launch_u1_stiffness_sf(yeti_ctx *ctx, const U1Patch &P, const double *coords,
                           double lam, double mu, double *kdata, int32_t *krow,
                           int32_t *kcol, size_t smem_cap) {
    YETI_CHECK(P.nq == P.ng * P.ng * P.ng && P.ng >= 2 && P.ng <= kSfMaxG, YETI_EUNSUPPORTED,
               "sum-factorised stiffness: needs a full tensor Gauss rule of at "
               "least 2 and at most %d points per direction (NBINT %d)", kSfMaxG, P.nq);
    SfArgs a;
    for (int d = 0; d < 3; d++) {
        a.p[d] = P.p[d];
        a.n[d] = P.p[d] + 1;
    }
    a.nn = P.nn;
    const size_t smem = sf_smem_doubles(a.n, P.ng) * sizeof(double);
    YETI_CHECK(smem <= smem_cap, YETI_EUNSUPPORTED,
               "sum-factorised stiffness: an element of degrees (%d,%d,%d) "
               "with %d Gauss points per direction does not fit shared memory",
               P.p[0], P.p[1], P.p[2], P.ng);
    a.U[0] = P.knots.as<double>();
    a.U[1] = a.U[0] + P.nkv[0];
    a.U[2] = a.U[1] + P.nkv[1];
    a.gauss = P.gauss.as<double>();
    a.coords = coords;
    a.ien = P.ien.as<int32_t>();
    a.w = P.w.as<double>();
    a.span = P.span.as<int32_t>();
    a.slot = P.slotd.as<int64_t>();
    a.lam = lam;
    a.mu = mu;
    a.kdata = kdata;
    a.krow = krow;
    a.kcol = kcol;
    void (*kern)(SfArgs) = nullptr;
    switch (P.ng) {
        case 2: kern = k_u1_stiffness_sf<2>; break;
        case 3: kern = k_u1_stiffness_sf<3>; break;
        case 4: kern = k_u1_stiffness_sf<4>; break;
        case 5: kern = k_u1_stiffness_sf<5>; break;
        case 6: kern = k_u1_stiffness_sf<6>; break;
        case 7: kern = k_u1_stiffness_sf<7>; break;
        case 8: kern = k_u1_stiffness_sf<8>; break;
        default: break;
    }
    YETI_CHECK(kern, YETI_EUNSUPPORTED, "sum-factorised stiffness: %d Gauss points per direction", P.ng);
    YETI_TRY(set_smem_optin((const void *)kern, ctx->device, smem, "sum-factorised stiffness element"));
    int64_t left = P.nactive, off = 0;
    while (left > 0) {   // grid.x limit
        const int64_t n = std::min<int64_t>(left, 1 << 30);
        SfArgs b = a;
        b.ien += off * P.nn;
        b.w += off * P.nn;
        b.span += off * 3;
        b.slot += off;
        kern<<<(unsigned)n, kSfThreads, smem, ctx->stream>>>(b);
        count_launches(1);
        YETI_CUDA(cudaGetLastError());
        left -= n;
        off += n;
    }
    return YETI_OK;
}

}  // namespace yeti
