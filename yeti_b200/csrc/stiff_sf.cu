// Sum-factorised U1 element stiffness: the same COO slots and values as the
// point-by-pair kernel of assemble_u1.cu (stiffmatrix.F90:130-225,
// UELMAT.f90:109-171), with the B^T D B contraction done direction by
// direction over the 1-D basis tables instead of pair by pair.  The sums run
// in another order, so the values agree with the reference to rounding
// (relative 1e-13 on the test meshes), not bit for bit.
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
// The 3x3 block (k, l) of the element matrix is then
//
//     K_kl(a, b) = w_a w_b sum_q sum_{kappa,eta} Phi^kappa_a Phi^eta_b M^{kappa eta}_kl(q),
//     M^{kappa eta}_kl = dv (lam c^kappa_k c^eta_l + mu c^kappa_l c^eta_k
//                            + [k = l] mu sum_r c^kappa_r c^eta_r),
//
// (isotropic D of stiffmatrix.F90:167-216), and each sum over q is
// contracted along w, then v, then u.  Kinds that share their 1-D factors in
// the remaining directions are added before a contraction: after w the
// value and d/dw kinds fall together (class 0), d/du is class 1, d/dv class
// 2; after v only the (value or derivative) kind along u remains.  Per block
// the three steps cost 16 n^2 g^3, 9 n^4 g^2 and 4 n^6 g multiply-adds (n =
// p+1 functions, g Gauss points per direction), against about 22 n^6 g^3
// for the pair loop.
//
// One CTA per element; the six blocks (k <= l) run in turn, each through
// shared memory: M (16 per point), T1 (class pairs x i3 j3 x q1 q2) and T2
// (kind pairs along u x i2 j2 x i3 j3 x q1, for a chunk of i3 at a time).
// Every COO value is written once: block (k, l) gives entry (k, l) of pair
// (a, b) for a < b, entry (l, k) of pair (b, a) for a > b (k < l only: the
// diagonal blocks are symmetric) and the upper triangle of the diagonal
// pair, halved on its diagonal.
#include "nurbs.cuh"
#include "u1_model.cuh"

namespace yeti {

constexpr int kSfThreads = 256;
constexpr int kSfMaxG = 8;   // Gauss points per direction (template instances)

struct SfArgs {
    int n[3];        // functions per direction (p+1)
    int p[3];
    int nn, ng, nq, i3c;
    const double *U[3];
    const double *gauss;   // 4 * ng^3: weight, t1, t2, t3 (t3 fastest)
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
size_t sf_smem_doubles(const int n[3], int ng, int i3c) {
    const size_t nn = (size_t)n[0] * n[1] * n[2], nq = (size_t)ng * ng * ng;
    const size_t t2 = 4 * (size_t)n[1] * n[1] * i3c * n[2] * ng;
    return 4 * nn + 2 * (size_t)ng * (n[0] + n[1] + n[2]) + 13 * nq +
           9 * (size_t)n[2] * n[2] * ng * ng + (t2 > 16 * nq ? t2 : 16 * nq);
}

__device__ __forceinline__ double det3(const double J[3][3]) {
    return J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
           J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
           J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
}

template <int G>
__global__ void __launch_bounds__(kSfThreads) k_u1_stiffness_sf(SfArgs a) {
    extern __shared__ double smem[];
    constexpr int ng = G, nq = G * G * G;
    const int nu = a.n[0], nv = a.n[1], nw = a.n[2], nn = a.nn;
    double *xe = smem;                       // 3 nn
    double *we = xe + 3 * nn;                // nn
    double *tab = we + nn;                   // A_d[kind][i][q], d = u, v, w
    double *A1 = tab, *A2 = A1 + 2 * nu * ng, *A3 = A2 + 2 * nv * ng;
    double *cq = A3 + 2 * nw * ng;           // 13 nq: c[kind][r], dv
    double *T1 = cq + 13 * nq;               // 9 nw^2 ng^2
    double *MT = T1 + 9 * nw * nw * ng * ng; // M (16 nq), then T2
    __shared__ double su1[3], su2[3];
    __shared__ int sni[3];
    const int e = blockIdx.x, tid = threadIdx.x;
    const int32_t *ien = a.ien + (size_t)e * nn;
    for (int i = tid; i < nn; i += kSfThreads) {
        const int cp = ien[i];
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
    if (tid < 3 * ng) {
        const int d = tid / ng, q = tid - d * ng;
        const int qq = d == 0 ? q * ng * ng : (d == 1 ? q * ng : q);
        const double t = a.gauss[4 * qq + 1 + d];
        const double xi = ((su2[d] - su1[d]) * t + (su2[d] + su1[d])) * 0.5;
        double N[kMaxDeg1], dN[kMaxDeg1];
        bspline_ders(sni[d], a.p[d], xi, a.U[d], N, dN);
        const int nd = a.n[d];
        double *A = d == 0 ? A1 : (d == 1 ? A2 : A3);
        for (int i = 0; i < nd; i++) {
            A[i * ng + q] = N[a.p[d] - i];
            A[(nd + i) * ng + q] = dN[a.p[d] - i];
        }
    }
    __syncthreads();
    // ---- per point: W, dW, x sums -> Jacobian, its inverse, dv, c
    for (int q = tid; q < nq; q += kSfThreads) {
        const int q1 = q / (ng * ng), q2 = (q / ng) % ng, q3 = q % ng;
        double W = 0, Wd[3] = {0, 0, 0}, P[4][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        int n = 0;
        for (int i3 = 0; i3 < nw; i3++) {
            const double c0 = A3[i3 * ng + q3], c1 = A3[(nw + i3) * ng + q3];
            for (int i2 = 0; i2 < nv; i2++) {
                const double b0 = A2[i2 * ng + q2], b1 = A2[(nv + i2) * ng + q2];
                const double v23 = b0 * c0, d2 = b1 * c0, d3 = b0 * c1;
                for (int i1 = 0; i1 < nu; i1++, n++) {
                    const double a0 = A1[i1 * ng + q1], a1 = A1[(nu + i1) * ng + q1];
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
    const int64_t base = a.slot[e];
    const double lam = a.lam, mu = a.mu;
    const int ngg = ng * ng;
    for (int kl = 0; kl < 6; kl++) {
        const int k = kl < 3 ? kl : (kl == 5 ? 1 : 0);
        const int l = kl < 3 ? kl : (kl == 3 ? 1 : 2);
        __syncthreads();
        // ---- M^{kappa eta}(q), kinds 0 value, 1 u, 2 v, 3 w
        for (int t = tid; t < 16 * nq; t += kSfThreads) {
            const int ke = t / nq, q = t - ke * nq, ka = ke >> 2, et = ke & 3;
            const double *c = cq + 13 * q;
            const double *ck = c + 3 * ka, *ce = c + 3 * et;
            double m = lam * ck[k] * ce[l] + mu * ck[l] * ce[k];
            if (k == l) m += mu * (ck[0] * ce[0] + ck[1] * ce[1] + ck[2] * ce[2]);
            MT[t] = m * c[12];
        }
        __syncthreads();
        // ---- step 1 (w): T1[ck,ce][i3][j3][q1 q2], classes 0 {value, w}, 1 {u}, 2 {v}
        for (int t = tid; t < 3 * nw * ngg; t += kSfThreads) {
            const int ck = t / (nw * ngg), r = t - ck * nw * ngg, i3 = r / ngg, q12 = r - i3 * ngg;
            double X[4][G];   // X[eta][q3] = sum_{kappa in ck} A3[kappa is w][i3][q3] M
#pragma unroll
            for (int q3 = 0; q3 < G; q3++) {
                {
                    const int q = q12 * ng + q3;
#pragma unroll
                    for (int et = 0; et < 4; et++) {
                        double x;
                        if (ck == 0)
                            x = A3[i3 * ng + q3] * MT[(0 * 4 + et) * nq + q] +
                                A3[(nw + i3) * ng + q3] * MT[(3 * 4 + et) * nq + q];
                        else
                            x = A3[i3 * ng + q3] * MT[(ck * 4 + et) * nq + q];
                        X[et][q3] = x;
                    }
                }
            }
#pragma unroll
            for (int ce = 0; ce < 3; ce++)
                for (int j3 = 0; j3 < nw; j3++) {
                    double s = 0;
#pragma unroll
                    for (int q3 = 0; q3 < G; q3++) {
                        {
                            const double b0 = A3[j3 * ng + q3];
                            if (ce == 0)
                                s += b0 * X[0][q3] + A3[(nw + j3) * ng + q3] * X[3][q3];
                            else
                                s += b0 * X[ce][q3];
                        }
                    }
                    T1[((ck * 3 + ce) * nw * nw + i3 * nw + j3) * ngg + q12] = s;
                }
        }
        for (int i3s = 0; i3s < nw; i3s += a.i3c) {
            const int i3n = min(a.i3c, nw - i3s);
            __syncthreads();
            // ---- step 2 (v): T2[al,be][i2][j2][i3l][j3][q1]; along u the
            // classes 0 and 2 carry the value kind, class 1 the derivative
            for (int t = tid; t < 2 * nv * i3n * nw * ng; t += kSfThreads) {
                int r = t;
                const int q1 = r % ng; r /= ng;
                const int j3 = r % nw; r /= nw;
                const int i3l = r % i3n; r /= i3n;
                const int i2 = r % nv; r /= nv;
                const int al = r;
                const int i3 = i3s + i3l;
                double V[3][G];   // V[ce][q2] = sum_{ck: u-kind al} A2 T1
#pragma unroll
                for (int q2 = 0; q2 < G; q2++) {
                    {
                        const int o = (i3 * nw + j3) * ngg + q1 * ng + q2;
                        const double b0 = A2[i2 * ng + q2];
#pragma unroll
                        for (int ce = 0; ce < 3; ce++) {
                            const int so = ce * nw * nw * ngg + o;
                            V[ce][q2] = al == 0
                                ? b0 * T1[0 * 3 * nw * nw * ngg + so] +
                                      A2[(nv + i2) * ng + q2] * T1[2 * 3 * nw * nw * ngg + so]
                                : b0 * T1[1 * 3 * nw * nw * ngg + so];
                        }
                    }
                }
#pragma unroll
                for (int be = 0; be < 2; be++)
                    for (int j2 = 0; j2 < nv; j2++) {
                        double s = 0;
#pragma unroll
                        for (int q2 = 0; q2 < G; q2++) {
                            {
                                const double c0 = A2[j2 * ng + q2];
                                s += be == 0 ? c0 * V[0][q2] + A2[(nv + j2) * ng + q2] * V[2][q2]
                                             : c0 * V[1][q2];
                            }
                        }
                        MT[((((al * 2 + be) * nv + i2) * nv + j2) * i3n + i3l) * nw * ng + j3 * ng + q1] = s;
                    }
            }
            __syncthreads();
            // ---- step 3 (u) and the COO writes
            for (int t = tid; t < nu * nv * i3n * nv * nw; t += kSfThreads) {
                int r = t;
                const int j3 = r % nw; r /= nw;
                const int j2 = r % nv; r /= nv;
                const int i3l = r % i3n; r /= i3n;
                const int i2 = r % nv; r /= nv;
                const int i1 = r;
                const int ia = i1 + nu * (i2 + nv * (i3s + i3l));
                double Uu[2][G];   // U[be][q1] = sum_al A1[al][i1][q1] T2[al,be]
#pragma unroll
                for (int q1 = 0; q1 < G; q1++) {
                    {
                        const double a0 = A1[i1 * ng + q1], a1 = A1[(nu + i1) * ng + q1];
#pragma unroll
                        for (int be = 0; be < 2; be++) {
                            const size_t o0 = ((((0 * 2 + be) * nv + i2) * nv + j2) * i3n + i3l) * nw * ng + j3 * ng + q1;
                            const size_t o1 = ((((1 * 2 + be) * nv + i2) * nv + j2) * i3n + i3l) * nw * ng + j3 * ng + q1;
                            Uu[be][q1] = a0 * MT[o0] + a1 * MT[o1];
                        }
                    }
                }
                const double wa = we[ia];
                const int dofa = 3 * ien[ia];
                for (int j1 = 0; j1 < nu; j1++) {
                    const int ib = j1 + nu * (j2 + nv * j3);
                    if (k == l && ia > ib) continue;
                    double s = 0;
#pragma unroll
                    for (int q1 = 0; q1 < G; q1++)
                        s += A1[j1 * ng + q1] * Uu[0][q1] + A1[(nu + j1) * ng + q1] * Uu[1][q1];
                    s *= wa * we[ib];
                    const int dofb = 3 * ien[ib];
                    int64_t o;
                    int row, col;
                    if (ia != ib) {
                        const int i = ia < ib ? ia : ib, j = ia < ib ? ib : ia;
                        const int kk = ia < ib ? k : l, ll = ia < ib ? l : k;
                        o = base + 9LL * j * (j - 1) / 2 + 6LL * j + 9LL * i + 3 * ll + kk;
                        row = (ia < ib ? dofa : dofb) + kk;
                        col = (ia < ib ? dofb : dofa) + ll;
                    } else {
                        o = base + 9LL * ia * (ia - 1) / 2 + 15LL * ia + l * (l + 1) / 2 + k;
                        if (k == l) s *= 0.5;
                        row = dofa + k;
                        col = dofa + l;
                    }
                    a.kdata[o] = s;
                    a.krow[o] = row;
                    a.kcol[o] = col;
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
    a.ng = P.ng;
    a.nq = P.nq;
    // the largest chunk of i3 whose buffers leave room for two CTAs per SM
    // (one when even a single i3 does not)
    const size_t two = smem_cap / 2 > 1024 ? smem_cap / 2 - 1024 : 0;
    int i3c = a.n[2];
    while (i3c > 1 && sf_smem_doubles(a.n, a.ng, i3c) * sizeof(double) > two) i3c--;
    const size_t smem = sf_smem_doubles(a.n, a.ng, i3c) * sizeof(double);
    YETI_CHECK(smem <= smem_cap, YETI_EUNSUPPORTED,
               "sum-factorised stiffness: an element of degrees (%d,%d,%d) "
               "with %d Gauss points per direction does not fit shared memory",
               P.p[0], P.p[1], P.p[2], P.ng);
    a.i3c = i3c;
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
