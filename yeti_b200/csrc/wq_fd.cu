// Fast-diagonalisation (FD) preconditioner of the WQ elasticity operator:
// the reference's fast_diagonalization_3d (src/yeti_iga/iga_wq_mf/fsrc/
// tensor_algebra.f90:1107-1161) with its eigen_decomposition (:992-1105),
// find_parametric_diag_3d (:1452-1482) and scaling_FastDiag (:1598-1625), as
// used by wq_mf_cg_3d (mf_wq_solver.f90:803-953), generalised from the
// scalar problem to the three displacement components.
//
// For component c the preconditioner inverts the separable operator
//     P_c = a[c][u] K_u (x) M_v (x) M_w + a[c][v] M_u (x) K_v (x) M_w
//         + a[c][w] M_u (x) M_v (x) K_w
// on the component's free box (the dofs off its clamped faces).  K_d / M_d
// are the 1-D WQ stiffness and mass matrices W11 B1^T and W00 B0^T
// (eigen_decomposition's KK and MM).  With K_d U_d = M_d U_d Lambda_d and
// U_d^T M_d U_d = I,
//     P_c^{-1} = (U_w (x) U_v (x) U_u) diag(1 / Lambda_c) (U_w (x) U_v (x) U_u)^T,
//     Lambda_c(i,j,k) = a[c][u] lu_i + a[c][v] lv_j + a[c][w] lw_k.
// a[c][d] is 1 (the reference's method 'C') or the mean over the WQ points
// of the coefficient S[(c,d),(c,d)] (the elastic counterpart of the
// Jacobian-mean lengths of jacobien_mean_3d, tensor_algebra.f90:1384-1448:
// method 'JM').  The scaled form ('JMS') applies z = s (P^{-1} (s r)) with
// s = sqrt(diag(P) / diag(K)).
//
// Device work per application: six passes of dense 1-D products along u, v,
// w (forward with U^T, the eigenvalue division fused into the w pass, then
// backward with U).  Each pass is a small-K GEMM over the lines of the box,
// tiled in shared memory (16-deep K chunks, 4x4 register tiles); the
// vectors (a few MB) stay in L2 between passes.
#include <algorithm>
#include <cmath>
#include <deque>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "reduce.cuh"
#include "wq.cuh"

namespace yeti {

constexpr int kFdThreads = 256;
constexpr int kFdTA = 128;     // max output rows per CTA
constexpr int kFdTL = 128;     // max lines per CTA
constexpr int kFdMaxM = 512;   // largest 1-D free size accepted
constexpr size_t kFdSmem = 200 * 1024;   // staged G and line tiles per CTA

// ------------------------------------------------------------------ host
// Symmetric eigenpairs of A (n x n, row-major, destroyed) by cyclic Jacobi
// rotations (Golub & Van Loan, Matrix Computations, sec. 8.5): A = V diag(w)
// V^T, V's columns the eigenvectors.  Returns false if it did not converge.
static bool sym_eig_jacobi(int n, std::vector<double> &A, std::vector<double> &w,
                           std::vector<double> &V) {
    V.assign((size_t)n * n, 0.0);
    for (int i = 0; i < n; i++) V[(size_t)i * n + i] = 1.0;
    auto at = [&](int i, int j) -> double & { return A[(size_t)i * n + j]; };
    double fro = 0.0;
    for (double v : A) fro += v * v;
    fro = std::sqrt(fro);
    bool ok = false;
    for (int sweep = 0; sweep < 60; sweep++) {
        double off = 0.0;
        for (int i = 0; i < n; i++)
            for (int j = i + 1; j < n; j++) off += at(i, j) * at(i, j);
        if (std::sqrt(2.0 * off) <= 1e-15 * fro) {
            ok = true;
            break;
        }
        for (int p = 0; p < n - 1; p++)
            for (int q = p + 1; q < n; q++) {
                const double apq = at(p, q);
                if (std::fabs(apq) <= 1e-300) continue;
                const double theta = (at(q, q) - at(p, p)) / (2.0 * apq);
                const double t = (theta >= 0 ? 1.0 : -1.0) /
                                 (std::fabs(theta) + std::sqrt(1.0 + theta * theta));
                const double cs = 1.0 / std::sqrt(1.0 + t * t), sn = t * cs;
                // A <- J^T A J with J the rotation in the (p, q) plane
                for (int k = 0; k < n; k++) {
                    const double akp = at(k, p), akq = at(k, q);
                    at(k, p) = cs * akp - sn * akq;
                    at(k, q) = sn * akp + cs * akq;
                }
                for (int k = 0; k < n; k++) {
                    const double apk = at(p, k), aqk = at(q, k);
                    at(p, k) = cs * apk - sn * aqk;
                    at(q, k) = sn * apk + cs * aqk;
                }
                at(p, q) = at(q, p) = 0.0;
                for (int k = 0; k < n; k++) {
                    double *vr = &V[(size_t)k * n];
                    const double vkp = vr[p], vkq = vr[q];
                    vr[p] = cs * vkp - sn * vkq;
                    vr[q] = sn * vkp + cs * vkq;
                }
            }
    }
    w.resize(n);
    for (int i = 0; i < n; i++) w[i] = at(i, i);
    return ok;
}

// Generalised symmetric-definite pencil K U = M U diag(lam), U^T M U = I,
// through M = L L^T and the standard form L^{-1} K L^{-T}.
static bool gen_eig(int n, const std::vector<double> &K, const std::vector<double> &M,
                    std::vector<double> &lam, std::vector<double> &U) {
    std::vector<double> L((size_t)n * n, 0.0);
    for (int j = 0; j < n; j++) {
        double d = M[(size_t)j * n + j];
        for (int k = 0; k < j; k++) d -= L[(size_t)j * n + k] * L[(size_t)j * n + k];
        if (!(d > 0.0)) return false;
        const double ljj = std::sqrt(d);
        L[(size_t)j * n + j] = ljj;
        for (int i = j + 1; i < n; i++) {
            double v = M[(size_t)i * n + j];
            for (int k = 0; k < j; k++) v -= L[(size_t)i * n + k] * L[(size_t)j * n + k];
            L[(size_t)i * n + j] = v / ljj;
        }
    }
    // Y = L^{-1} K (forward substitution per column), C = L^{-1} Y^T
    std::vector<double> Y((size_t)n * n), C((size_t)n * n);
    for (int col = 0; col < n; col++)
        for (int i = 0; i < n; i++) {
            double v = K[(size_t)i * n + col];
            for (int k = 0; k < i; k++) v -= L[(size_t)i * n + k] * Y[(size_t)k * n + col];
            Y[(size_t)i * n + col] = v / L[(size_t)i * n + i];
        }
    for (int col = 0; col < n; col++)
        for (int i = 0; i < n; i++) {
            double v = Y[(size_t)col * n + i];   // (Y^T)[i][col]
            for (int k = 0; k < i; k++) v -= L[(size_t)i * n + k] * C[(size_t)k * n + col];
            C[(size_t)i * n + col] = v / L[(size_t)i * n + i];
        }
    for (int i = 0; i < n; i++)
        for (int j = i + 1; j < n; j++) {
            const double s = 0.5 * (C[(size_t)i * n + j] + C[(size_t)j * n + i]);
            C[(size_t)i * n + j] = C[(size_t)j * n + i] = s;
        }
    std::vector<double> Q;
    if (!sym_eig_jacobi(n, C, lam, Q)) return false;
    // U = L^{-T} Q (back substitution per column)
    U.assign((size_t)n * n, 0.0);
    for (int col = 0; col < n; col++)
        for (int i = n - 1; i >= 0; i--) {
            double v = Q[(size_t)i * n + col];
            for (int k = i + 1; k < n; k++) v -= L[(size_t)k * n + i] * U[(size_t)k * n + col];
            U[(size_t)i * n + col] = v / L[(size_t)i * n + i];
        }
    return true;
}

// 1-D WQ matrices of one direction restricted to functions [lo, hi),
// symmetrised: M = W00 B0^T, K = W11 B1^T (eigen_decomposition's MM, KK).
static void wq_1d_matrices(const WQRule1D &R, int lo, int hi, std::vector<double> &K,
                           std::vector<double> &M) {
    const int m = hi - lo, nq = R.nqp;
    K.assign((size_t)m * m, 0.0);
    M.assign((size_t)m * m, 0.0);
    for (int i = 0; i < m; i++)
        for (int j = 0; j < m; j++) {
            const double *w0 = &R.W00[(size_t)(lo + i) * nq], *b0 = &R.B0[(size_t)(lo + j) * nq];
            const double *w1 = &R.W11[(size_t)(lo + i) * nq], *b1 = &R.B1[(size_t)(lo + j) * nq];
            double sm = 0.0, sk = 0.0;
            for (int q = 0; q < nq; q++) {
                sm += w0[q] * b0[q];
                sk += w1[q] * b1[q];
            }
            M[(size_t)i * m + j] = sm;
            K[(size_t)i * m + j] = sk;
        }
    for (int i = 0; i < m; i++)
        for (int j = i + 1; j < m; j++) {
            const double a = 0.5 * (M[(size_t)i * m + j] + M[(size_t)j * m + i]);
            const double b = 0.5 * (K[(size_t)i * m + j] + K[(size_t)j * m + i]);
            M[(size_t)i * m + j] = M[(size_t)j * m + i] = a;
            K[(size_t)i * m + j] = K[(size_t)j * m + i] = b;
        }
}

// ---------------------------------------------------------------- device
template <class T>
struct FdArgs {
    const T *in;
    T *out;
    const T *g;        // G for this pass: out_row = sum_k G[k][row] in_k
    const T *dsc;      // a[c][d] * lambda_d
    const T *s;        // scaling (nullptr: none)
    const T *r;        // residual (reduction modes)
    T *p;              // FD_START: p = z
    const int *done;
    CGScal *cg;
    double *parts;
    int red;
    int n[3];
    int64_t ncp;
    int lo[3][3], m[3][3];
    int64_t goff[3];   // per component, for this pass
    int64_t goff2[3];  // fused w pass: the backward matrix
    int64_t doff[3][3];
    int nag[3], nlg[3], ntA[3], cta_end[3];
};

// Tiles of one pass for one component: ntA tiles of TA = 4 nag output rows
// times tiles of TL = 4 nlg lines, the whole contraction (m rows of G and of
// the lines) staged in shared memory.  The fused w pass (two G matrices)
// needs one row tile.  Lines per CTA are cut until the pass has at least two
// CTAs per SM (148 SMs) so that no SM idles behind a neighbour with twice
// its work.
struct FdTile {
    int ntA, nag, nlg, ctas, threads;
    size_t smem;
};
static FdTile fd_tile(int m, int64_t nlines, size_t esize, bool fused) {
    FdTile t;
    const int ng = fused ? 2 : 1;
    t.ntA = fused ? 1 : (m + kFdTA - 1) / kFdTA;
    auto bytes = [&](int nag, int nlg) {
        return (size_t)m * (ng * 4 * nag + 4 * nlg + 4) * esize;
    };
    auto ctas = [&](int ntA, int nlg) {
        return ntA * (int)((nlines + 4 * nlg - 1) / (4 * nlg));
    };
    for (;;) {
        t.nag = ((m + t.ntA - 1) / t.ntA + 3) / 4;
        // the most lines per CTA that still give the pass (three components)
        // two CTAs per SM
        int nlg = std::min(kFdTL / 4, kFdThreads / t.nag);
        while (nlg > 4 && ctas(t.ntA, nlg) < (2 * 148 + 2) / 3) nlg--;
        while (nlg > 4 && bytes(t.nag, nlg) > kFdSmem) nlg--;
        t.nlg = nlg;
        if (bytes(t.nag, nlg) <= kFdSmem || fused) break;
        t.ntA++;
    }
    t.smem = bytes(t.nag, t.nlg);
    t.ctas = ctas(t.ntA, t.nlg);
    t.threads = (t.nag * t.nlg + 31) / 32 * 32;
    if (fused && t.smem > kFdSmem) t.ctas = -1;   // not possible: separate passes
    return t;
}

template <class T> struct Vec4;
template <> struct Vec4<float> {
    static __device__ __forceinline__ void ld(const float *p, float v[4]) {
        const float4 q = *reinterpret_cast<const float4 *>(p);
        v[0] = q.x; v[1] = q.y; v[2] = q.z; v[3] = q.w;
    }
};
template <> struct Vec4<double> {
    static __device__ __forceinline__ void ld(const double *p, double v[4]) {
        const double2 q0 = *reinterpret_cast<const double2 *>(p);
        const double2 q1 = *reinterpret_cast<const double2 *>(p + 2);
        v[0] = q0.x; v[1] = q0.y; v[2] = q1.x; v[3] = q1.y;
    }
};

template <class T>
__device__ __forceinline__ void fma44(T acc[4][4], const T g[4], const T x[4]) {
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] += g[i] * x[j];
}

// FP32: the 4x4 tile as pairs of columns on packed FP32x2 FMAs (each lane
// of a pair is the scalar FMA acc += g x, so the sums keep their bits).
__device__ __forceinline__ void fma44_2(float2 acc[4][2], const float g[4], const float2 x[2]) {
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const float2 gg = make_float2(g[i], g[i]);
        acc[i][0] = __ffma2_rn(gg, x[0], acc[i][0]);
        acc[i][1] = __ffma2_rn(gg, x[1], acc[i][1]);
    }
}

// acc[i][j] = sum_{k < m} gp[k ldg + i] xp[k ldx + j], the next row's
// operands loaded while the current row's products issue.
__device__ __forceinline__ void fd_contract(const float *gp, int ldg, const float *xp, int ldx,
                                            int m, float acc[4][4]) {
    float2 a2[4][2];
#pragma unroll
    for (int i = 0; i < 4; i++) a2[i][0] = a2[i][1] = make_float2(0.f, 0.f);
    float g0[4], g1[4];
    float2 x0[2], x1[2];
    auto ldx2 = [](const float *p, float2 v[2]) {
        const float4 q = *reinterpret_cast<const float4 *>(p);
        v[0] = make_float2(q.x, q.y);
        v[1] = make_float2(q.z, q.w);
    };
    Vec4<float>::ld(gp, g0);
    ldx2(xp, x0);
    int k = 0;
    for (; k + 1 < m; k += 2) {
        Vec4<float>::ld(gp + (k + 1) * ldg, g1);
        ldx2(xp + (k + 1) * ldx, x1);
        fma44_2(a2, g0, x0);
        if (k + 2 < m) {
            Vec4<float>::ld(gp + (k + 2) * ldg, g0);
            ldx2(xp + (k + 2) * ldx, x0);
        }
        fma44_2(a2, g1, x1);
    }
    if (k < m) fma44_2(a2, g0, x0);
#pragma unroll
    for (int i = 0; i < 4; i++) {
        acc[i][0] = a2[i][0].x;
        acc[i][1] = a2[i][0].y;
        acc[i][2] = a2[i][1].x;
        acc[i][3] = a2[i][1].y;
    }
}

template <class T>
__device__ __forceinline__ void fd_contract(const T *gp, int ldg, const T *xp, int ldx, int m,
                                            T acc[4][4]) {
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = T(0);
    T g0[4], x0[4], g1[4], x1[4];
    Vec4<T>::ld(gp, g0);
    Vec4<T>::ld(xp, x0);
    int k = 0;
    for (; k + 1 < m; k += 2) {
        Vec4<T>::ld(gp + (k + 1) * ldg, g1);
        Vec4<T>::ld(xp + (k + 1) * ldx, x1);
        fma44(acc, g0, x0);
        if (k + 2 < m) {
            Vec4<T>::ld(gp + (k + 2) * ldg, g0);
            Vec4<T>::ld(xp + (k + 2) * ldx, x0);
        }
        fma44(acc, g1, x1);
    }
    if (k < m) fma44(acc, g0, x0);
}

// Asynchronous global -> shared copy of one element (cp.async, sm_80+);
// valid == false writes zero and reads nothing.
template <class T>
__device__ __forceinline__ void cp_elem(T *sdst, const T *gsrc, bool valid) {
    const unsigned saddr = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(saddr), "l"(gsrc),
                 "n"((int)sizeof(T)), "r"(valid ? (int)sizeof(T) : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// End of the last pass of a CG application: the r.z partials of the block,
// then (last block) the CG scalars of the reduction mode.
template <class T>
__device__ __forceinline__ void fd_finish_rz(const FdArgs<T> &a, double rz, double *sh) {
    rz = block_sum(rz, sh);
    if (threadIdx.x == 0) __stcg(&a.parts[blockIdx.x], rz);
    if (!last_block(&a.cg->ticket)) return;
    double srz = 0.0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) srz += __ldcg(&a.parts[i]);
    srz = block_sum(srz, sh);
    if (threadIdx.x == 0) {
        CGScal *s = a.cg;
        s->ticket = 0;
        if (a.red == FD_ITER) {
            const double old = s->rz;
            s->beta = srz / old;
            if (!isfinite(srz) || !(old != 0.0)) {
                s->breakdown = 1;
                s->done = 1;
            }
        }
        s->rz = srz;
    }
}

// One pass along axis AX: out_row(line) = sum_k G[k][row] in_k(line).
// EPI 1: divide by Lambda; EPI 2: multiply by s, r.z partials and the
// reduction mode; EPI 3 (AX == 2, one row tile): forward product, division
// by Lambda and backward product in one CTA, the intermediate kept in shared
// memory.  The G columns and the lines are staged by cp.async (all copies in
// flight at once), then contracted from shared memory.
template <class T, int AX, int EPI>
__global__ void __launch_bounds__(kFdThreads) k_fd_pass(FdArgs<T> a) {
    extern __shared__ __align__(16) unsigned char fd_smem[];
    __shared__ int64_t lb[kFdTL];
    __shared__ int2 lc[kFdTL];   // (i1, i2) of a line
    __shared__ double sh[32];
    if (a.done && *a.done) return;
    int b = blockIdx.x, c = 0;
    while (c < 2 && b >= a.cta_end[c]) c++;
    if (c > 0) b -= a.cta_end[c - 1];
    constexpr int D1 = AX == 0 ? 1 : 0, D2 = AX == 2 ? 1 : 2;
    const int nag = a.nag[c], nlg = a.nlg[c], ntA = a.ntA[c];
    const int m = a.m[c][AX], m1 = a.m[c][D1], m2 = a.m[c][D2];
    const int64_t nlines = (int64_t)m1 * m2;
    const int TA = 4 * nag, TL = 4 * nlg, TLp = TL + 4;
    T *Gs = reinterpret_cast<T *>(fd_smem);    // [m][TA]
    T *G2 = Gs + (size_t)m * TA;               // EPI 3: [m][TA]
    T *Xs = EPI == 3 ? G2 + (size_t)m * TA : G2;   // [m][TLp]
    const int a0 = (b % ntA) * TA;
    const int64_t l0 = (int64_t)(b / ntA) * TL;
    const int64_t st[3] = {1, (int64_t)a.n[0], (int64_t)a.n[0] * a.n[1]};
    const int64_t sk = st[AX];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nthr = blockDim.x, nwarp = nthr >> 5;
    for (int ll = tid; ll < TL; ll += nthr) {
        const int64_t l = l0 + ll;
        int64_t base = -1;
        int i1 = 0, i2 = 0;
        if (l < nlines) {
            i1 = (int)(l % m1);
            i2 = (int)(l / m1);
            base = c * a.ncp + (int64_t)a.lo[c][AX] * sk + (int64_t)(a.lo[c][D1] + i1) * st[D1] +
                   (int64_t)(a.lo[c][D2] + i2) * st[D2];
        }
        lb[ll] = base;
        lc[ll] = make_int2(i1, i2);
    }
    // G columns a0 .. a0 + TA of every row k (a warp per row)
    const T *G = a.g + a.goff[c];
    for (int k = warp; k < m; k += nwarp) {
        const T *src = G + (int64_t)k * m;
        for (int aa = lane; aa < TA; aa += 32) {
            const int col = a0 + aa;
            cp_elem(Gs + k * TA + aa, col < m ? src + col : G, col < m);
        }
    }
    if (EPI == 3) {
        const T *Gb = a.g + a.goff2[c];
        for (int k = warp; k < m; k += nwarp) {
            const T *src = Gb + (int64_t)k * m;
            for (int aa = lane; aa < TA; aa += 32)
                cp_elem(G2 + k * TA + aa, aa < m ? src + aa : Gb, aa < m);
        }
    }
    __syncthreads();   // lb
    if (AX == 0) {
        // lines are contiguous: a warp per line, lanes along k
        for (int ll = warp; ll < TL; ll += nwarp) {
            const int64_t base = lb[ll];
            for (int k = lane; k < m; k += 32)
                cp_elem(Xs + k * TLp + ll, base >= 0 ? a.in + base + k : a.in, base >= 0);
        }
    } else {
        // row k of the tile is contiguous along the lines: a warp per row
        for (int k = warp; k < m; k += nwarp) {
            for (int ll = lane; ll < TL; ll += 32) {
                const int64_t base = lb[ll];
                cp_elem(Xs + k * TLp + ll, base >= 0 ? a.in + base + (int64_t)k * sk : a.in,
                        base >= 0);
            }
        }
    }
    cp_wait_all();
    __syncthreads();
    int ag, lg;
    if (AX == 0) {
        ag = tid % nag;
        lg = tid / nag;
    } else {
        lg = tid % nlg;
        ag = tid / nlg;
    }
    const bool act = tid < nag * nlg;
    T acc[4][4];
    if (act) fd_contract(Gs + 4 * ag, TA, Xs + 4 * lg, TLp, m, acc);
    if (EPI == 3) {
        // divide by Lambda, park the eigen-space values in Xs, contract back
        __syncthreads();
        if (act) {
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const int e = 4 * ag + i;
                if (e >= m) continue;
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    const int ll = 4 * lg + j;
                    const int2 q = lc[ll];
                    const T lam = a.dsc[a.doff[c][0] + q.x] + a.dsc[a.doff[c][1] + q.y] +
                                  a.dsc[a.doff[c][2] + e];
                    Xs[e * TLp + ll] = lb[ll] >= 0 ? acc[i][j] / lam : T(0);
                }
            }
        }
        __syncthreads();
        if (act) fd_contract(G2 + 4 * ag, TA, Xs + 4 * lg, TLp, m, acc);
    }
    double rz = 0.0;
    if (act) {
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const int row = a0 + 4 * ag + i;
            if (row >= m) continue;
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int ll = 4 * lg + j;
                const int64_t base = lb[ll];
                if (base < 0) continue;
                const int64_t idx = base + (int64_t)row * sk;
                T v = acc[i][j];
                if (EPI == 1) {
                    int e3[3];
                    e3[AX] = row;
                    e3[D1] = lc[ll].x;
                    e3[D2] = lc[ll].y;
                    const T lam = a.dsc[a.doff[c][0] + e3[0]] + a.dsc[a.doff[c][1] + e3[1]] +
                                  a.dsc[a.doff[c][2] + e3[2]];
                    v = v / lam;
                }
                if (EPI == 2) {
                    if (a.s) v *= a.s[idx];
                    if (a.red != FD_NONE) rz += (double)a.r[idx] * (double)v;
                    if (a.red == FD_START) a.p[idx] = v;
                }
                a.out[idx] = v;
            }
        }
    }
    if (EPI != 2 || a.red == FD_NONE) return;
    fd_finish_rz(a, rz, sh);
}

// The u and v products of one w plane in one CTA: with X the plane's values
// (rows v, columns u of the component's free box),
//     T[v][a] = sum_i X[v][i] Gu[i][a],   Y[b][a] = sum_j Gv[j][b] T[j][a],
// forward (Gu = U_u, Gv = U_v; in positions, out eigen indices) or backward
// (Gu = U_u^T, Gv = U_v^T).  The plane, Gu's columns of the CTA's column
// split, Gv and T stay in shared memory.  goff: Gu, goff2: Gv; ntA: column
// splits, nag: 4-column groups per split, nlg: 4-row groups (ceil(m_v / 4)).
// EPI 2 as k_fd_pass.
template <class T, int EPI>
__global__ void __launch_bounds__(kFdThreads) k_fd_plane(FdArgs<T> a) {
    extern __shared__ __align__(16) unsigned char fd_smem[];
    __shared__ double sh[32];
    if (a.done && *a.done) return;
    int b = blockIdx.x, c = 0;
    while (c < 2 && b >= a.cta_end[c]) c++;
    if (c > 0) b -= a.cta_end[c - 1];
    const int mu = a.m[c][0], mv = a.m[c][1];
    const int nsplit = a.ntA[c], nag = a.nag[c], nvg = a.nlg[c];
    const int TA = 4 * nag, ldv = 4 * nvg + 4, ldb = 4 * nvg;
    const int sp = b % nsplit, kw = b / nsplit;
    const int a0 = sp * TA;
    T *Xt = reinterpret_cast<T *>(fd_smem);   // [mu][ldv]: X transposed
    T *Gu = Xt + (size_t)mu * ldv;            // [mu][TA]
    T *Gv = Gu + (size_t)mu * TA;             // [mv][ldb]
    T *Tm = Gv + (size_t)mv * ldb;            // [mv][TA]
    const int64_t nu = a.n[0], nv = a.n[1];
    const int64_t plane = c * a.ncp + (int64_t)(a.lo[c][2] + kw) * nu * nv +
                          (int64_t)a.lo[c][1] * nu + a.lo[c][0];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nwarp = blockDim.x >> 5;
    // the plane, a warp per row v (contiguous along u); rows mv .. 4 nvg zero
    for (int v = warp; v < 4 * nvg; v += nwarp) {
        const T *src = a.in + plane + (int64_t)v * nu;
        for (int i = lane; i < mu; i += 32)
            cp_elem(Xt + i * ldv + v, v < mv ? src + i : a.in, v < mv);
    }
    const T *G = a.g + a.goff[c];
    for (int i = warp; i < mu; i += nwarp)
        for (int aa = lane; aa < TA; aa += 32) {
            const int col = a0 + aa;
            cp_elem(Gu + i * TA + aa, col < mu ? G + (int64_t)i * mu + col : G, col < mu);
        }
    const T *H = a.g + a.goff2[c];
    for (int j = warp; j < mv; j += nwarp)
        for (int bb = lane; bb < ldb; bb += 32)
            cp_elem(Gv + j * ldb + bb, bb < mv ? H + (int64_t)j * mv + bb : H, bb < mv);
    cp_wait_all();
    __syncthreads();
    const int ag = tid % nag, vg = tid / nag;
    const bool act = vg < nvg;
    T acc[4][4];
    if (act) {
        fd_contract(Xt + 4 * vg, ldv, Gu + 4 * ag, TA, mu, acc);
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const int v = 4 * vg + i;
            if (v < mv)
#pragma unroll
                for (int j = 0; j < 4; j++) Tm[v * TA + 4 * ag + j] = acc[i][j];
        }
    }
    __syncthreads();
    double rz = 0.0;
    if (act) {
        fd_contract(Gv + 4 * vg, ldb, Tm + 4 * ag, TA, mv, acc);
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const int row = 4 * vg + i;
            if (row >= mv) continue;
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int col = a0 + 4 * ag + j;
                if (4 * ag + j >= TA || col >= mu) continue;
                const int64_t idx = plane + (int64_t)row * nu + col;
                T v = acc[i][j];
                if (EPI == 2) {
                    if (a.s) v *= a.s[idx];
                    if (a.red != FD_NONE) rz += (double)a.r[idx] * (double)v;
                    if (a.red == FD_START) a.p[idx] = v;
                }
                a.out[idx] = v;
            }
        }
    }
    if (EPI != 2 || a.red == FD_NONE) return;
    fd_finish_rz(a, rz, sh);
}

// out = s in (elementwise; s is zero off the free boxes)
template <class T>
__global__ void k_fd_scale_in(const T *in, const T *sv, T *out, int64_t n, const int *done) {
    if (done && *done) return;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x)
        out[i] = in[i] * sv[i];
}

// s = sqrt(diag(P) / diag(K)) on every component's free box, 0 elsewhere;
// diag(P) from the 1-D diagonals (find_parametric_diag_3d).
__global__ void k_fd_scaling(const double *diagK, const double *kdmd, double *s64, float *s32, int3 n, int64_t ncp, int lo0, int lo1,
                             int lo2, int m0, int m1, int m2, int c, int64_t off_u,
                             int64_t off_v, int64_t off_w, double au, double av, double aw) {
    const int64_t tot = (int64_t)m0 * m1 * m2;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < tot;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int i = (int)(t % m0), j = (int)((t / m0) % m1), k = (int)(t / ((int64_t)m0 * m1));
        const double ku = kdmd[off_u + i], mu = kdmd[off_u + m0 + i];
        const double kv = kdmd[off_v + j], mv = kdmd[off_v + m1 + j];
        const double kw = kdmd[off_w + k], mw = kdmd[off_w + m2 + k];
        const double dp = au * ku * mv * mw + av * mu * kv * mw + aw * mu * mv * kw;
        const int64_t idx = c * ncp + (int64_t)(lo0 + i) + (int64_t)n.x * ((lo1 + j) + (int64_t)n.y * (lo2 + k));
        const double v = sqrt(dp / diagK[idx]);
        if (s64) s64[idx] = v;
        if (s32) s32[idx] = (float)v;
    }
}

// ------------------------------------------------------------------ plan
// Tiling of the fused plane pass for one component: column splits of the
// u products (each CTA recomputes nothing, it reads the whole plane), at
// most 256 threads, the staged plane, Gu columns, Gv and T within kFdSmem,
// and splits added while the pass (three components) has fewer than two
// CTAs per SM.  ctas = -1: does not fit (the line passes run instead).
struct FdPlane {
    int nsplit, nag, nvg, ctas, threads;
    size_t smem;
};
static FdPlane fd_plane_tile(int mu, int mv, int mw, size_t esize) {
    FdPlane t;
    t.nvg = (mv + 3) / 4;
    t.ctas = -1;
    const int ldv = 4 * t.nvg + 4, ldb = 4 * t.nvg;
    bool ok = false;
    for (t.nsplit = 1; t.nsplit <= mu; t.nsplit++) {
        t.nag = ((mu + t.nsplit - 1) / t.nsplit + 3) / 4;
        const int TA = 4 * t.nag;
        t.smem = ((size_t)mu * ldv + (size_t)mu * TA + (size_t)mv * ldb + (size_t)mv * TA) * esize;
        if (t.nag * t.nvg > kFdThreads || t.smem > kFdSmem) continue;
        ok = true;
        if (3 * mw * t.nsplit >= 2 * 148 || t.nag <= 2) break;
    }
    if (!ok) return t;
    t.ctas = mw * t.nsplit;
    t.threads = (t.nag * t.nvg + 31) / 32 * 32;
    return t;
}

template <class T>
static int fd_set_attrs() {
    const int b = (int)kFdSmem;
    const cudaFuncAttribute a = cudaFuncAttributeMaxDynamicSharedMemorySize;
    YETI_CUDA(cudaFuncSetAttribute(k_fd_pass<T, 0, 0>, a, b));
    YETI_CUDA(cudaFuncSetAttribute(k_fd_pass<T, 1, 0>, a, b));
    YETI_CUDA(cudaFuncSetAttribute(k_fd_pass<T, 2, 0>, a, b));
    YETI_CUDA(cudaFuncSetAttribute(k_fd_pass<T, 2, 1>, a, b));
    YETI_CUDA(cudaFuncSetAttribute(k_fd_pass<T, 2, 3>, a, b));
    YETI_CUDA(cudaFuncSetAttribute(k_fd_pass<T, 0, 2>, a, b));
    YETI_CUDA(cudaFuncSetAttribute(k_fd_plane<T, 0>, a, b));
    YETI_CUDA(cudaFuncSetAttribute(k_fd_plane<T, 2>, a, b));
    return YETI_OK;
}

// 1-D matrices with per-point weights (eigen_decomposition's 'TD' branch,
// tensor_algebra.f90:1045-1071): M = W00 (B0 diag(mw))^T and K = W11 (B1
// diag(kw))^T on the rows lo..hi-1, made symmetric by averaging with the
// transpose, as the unweighted matrices are.  (The reference hands the
// non-symmetric products to dsygvd, which reads their upper triangle; with
// the point-to-point variation of a rough coefficient field that triangle
// is indefinite, its eigenvalue sums negative, while the symmetric part
// stays definite.)
static void wq_1d_matrices_weighted(const WQRule1D &R, int lo, int hi, const double *mw,
                                    const double *kw, std::vector<double> &K,
                                    std::vector<double> &M) {
    const int m = hi - lo, nq = R.nqp;
    K.assign((size_t)m * m, 0.0);
    M.assign((size_t)m * m, 0.0);
    for (int i = 0; i < m; i++)
        for (int j = 0; j < m; j++) {
            const double *w0 = &R.W00[(size_t)(lo + i) * nq], *b0 = &R.B0[(size_t)(lo + j) * nq];
            const double *w1 = &R.W11[(size_t)(lo + i) * nq], *b1 = &R.B1[(size_t)(lo + j) * nq];
            double sm = 0.0, sk = 0.0;
            for (int q = 0; q < nq; q++) {
                sm += w0[q] * (b0[q] * mw[q]);
                sk += w1[q] * (b1[q] * kw[q]);
            }
            M[(size_t)i * m + j] = sm;
            K[(size_t)i * m + j] = sk;
        }
    for (int i = 0; i < m; i++)
        for (int j = i + 1; j < m; j++) {
            const double a = 0.5 * (M[(size_t)i * m + j] + M[(size_t)j * m + i]);
            const double b = 0.5 * (K[(size_t)i * m + j] + K[(size_t)j * m + i]);
            M[(size_t)i * m + j] = M[(size_t)j * m + i] = a;
            K[(size_t)i * m + j] = K[(size_t)j * m + i] = b;
        }
}

// One sweep of tensor_decomposition_3d (tensor_algebra.f90:1256-1382) for
// one displacement component: cc[k] the diagonal coefficient S[(c,k),(c,k)]
// at every WQ point (u fastest), M[d] / K[d] the per-point 1-D weights of
// direction d, updated in place.  Stiffness weights first: K_k(i) =
// sqrt(min V max V) over the slice i of direction k, V = cc_k M_k /
// (M_u M_v M_w); then mass weights: M_k(i) = sqrt(min N max W) over the
// slice, from cc_k M_k M_l / (M_u M_v M_w K_k), l != k.  (The reference
// bounds its direction-3 slice loops by the v count; the w count is used
// here, which agrees whenever the two are equal.)
static void td_sweep(const int nq[3], const double *const cc[3], std::vector<double> M[3],
                     std::vector<double> K[3]) {
    const int64_t n = (int64_t)nq[0] * nq[1] * nq[2];
    for (int k = 0; k < 3; k++) {
        std::vector<double> vmin(nq[k], INFINITY), vmax(nq[k], -INFINITY);
        int64_t g = 0;
        for (int i2 = 0; i2 < nq[2]; i2++)
            for (int i1 = 0; i1 < nq[1]; i1++)
                for (int i0 = 0; i0 < nq[0]; i0++, g++) {
                    const int i[3] = {i0, i1, i2};
                    const double uu[3] = {M[0][i0], M[1][i1], M[2][i2]};
                    const double v = cc[k][g] * uu[k] / (uu[0] * uu[1] * uu[2]);
                    vmin[i[k]] = std::min(vmin[i[k]], v);
                    vmax[i[k]] = std::max(vmax[i[k]], v);
                }
        for (int a = 0; a < nq[k]; a++) K[k][a] = std::sqrt(vmin[a] * vmax[a]);
    }
    for (int k = 0; k < 3; k++) {
        std::vector<double> nmin(nq[k], INFINITY), mmax(nq[k], -INFINITY);
        int64_t g = 0;
        for (int i2 = 0; i2 < nq[2]; i2++)
            for (int i1 = 0; i1 < nq[1]; i1++)
                for (int i0 = 0; i0 < nq[0]; i0++, g++) {
                    const int i[3] = {i0, i1, i2};
                    const double uu[3] = {M[0][i0], M[1][i1], M[2][i2]};
                    const double ww[3] = {K[0][i0], K[1][i1], K[2][i2]};
                    double lo = INFINITY, hi = -INFINITY;
                    for (int l = 0; l < 3; l++) {
                        if (l == k) continue;
                        const double w = cc[k][g] * uu[k] * uu[l] / (uu[0] * uu[1] * uu[2] * ww[k]);
                        lo = std::min(lo, w);
                        hi = std::max(hi, w);
                    }
                    nmin[i[k]] = std::min(nmin[i[k]], lo);
                    mmax[i[k]] = std::max(mmax[i[k]], hi);
                }
        for (int a = 0; a < nq[k]; a++) M[k][a] = std::sqrt(nmin[a] * mmax[a]);
    }
    (void)n;
}

// The diagonal coefficients S[(c,k),(c,k)] of every WQ point, in point
// order (u fastest), gathered from the streaming FP64 layout: out[(3c+k) n + g].
__global__ void k_fd_diag_coef(const double *coef, const int64_t *tile_off, const int *pstride,
                               const int *tq0u, const int *tnqu, const int *tq0v,
                               const int *tnqv, int ntu, int nqu, int nqv, int nqw,
                               double *out) {
    const int64_t n = (int64_t)nqu * nqv * nqw;
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < n;
         g += (int64_t)gridDim.x * blockDim.x) {
        const int qu = (int)(g % nqu), qv = (int)((g / nqu) % nqv);
        const int qw = (int)(g / ((int64_t)nqu * nqv));
        int tu = 0, tv = 0;
        while (tq0u[tu] + tnqu[tu] <= qu) tu++;
        while (tq0v[tv] + tnqv[tv] <= qv) tv++;
        const int t = tu + ntu * tv;
        const int npts = tnqu[tu] * tnqv[tv];
        const int pt = (qv - tq0v[tv]) * tnqu[tu] + (qu - tq0u[tu]);
        const double *blk = coef + tile_off[t] + (int64_t)qw * pstride[t] + pt;
        for (int c = 0; c < 3; c++)
            for (int k = 0; k < 3; k++)
                out[(int64_t)(3 * c + k) * n + g] = blk[(int64_t)sym9(3 * c + k, 3 * c + k) * npts];
    }
}

// The same gather from the element-block layout of the setup kernels
// (operators of mixed degrees or degree > 5): point (qu, qv, qw) of block b
// at coef[qoff[b] 45 + e nq_b + (lw nv_b + lv) nu_b + lu].
__global__ void k_fd_diag_coef_blk(const double *coef, const int64_t *qoff,
                                   const int *const *blk1, const int *const *loc1,
                                   const int *const *nq1, int nbu, int nbv, int nqu, int nqv,
                                   int nqw, double *out) {
    const int64_t n = (int64_t)nqu * nqv * nqw;
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < n;
         g += (int64_t)gridDim.x * blockDim.x) {
        const int qu = (int)(g % nqu), qv = (int)((g / nqu) % nqv);
        const int qw = (int)(g / ((int64_t)nqu * nqv));
        const int bu = blk1[0][qu], bv = blk1[1][qv], bw = blk1[2][qw];
        const int64_t b = bu + (int64_t)nbu * (bv + (int64_t)nbv * bw);
        const int nu1 = nq1[0][bu], nv1 = nq1[1][bv], nw1 = nq1[2][bw];
        const int64_t nqb = (int64_t)nu1 * nv1 * nw1;
        const double *base = coef + qoff[b] * kWQCoef +
                             (loc1[2][qw] * (int64_t)nv1 + loc1[1][qv]) * nu1 + loc1[0][qu];
        for (int c = 0; c < 3; c++)
            for (int k = 0; k < 3; k++)
                out[(int64_t)(3 * c + k) * n + g] = base[(int64_t)sym9(3 * c + k, 3 * c + k) * nqb];
    }
}

int wq_fd_prepare(yeti_wq_op *op, int variant, bool f32) {
    WQFdPlan &F = op->fd;
    variant &= (YETI_PCG_FD | YETI_PCG_FD_SCALED | YETI_PCG_FD_UNIT | YETI_PCG_FD_TD);
    if (F.variant == variant && (!f32 || F.g32.ptr)) return YETI_OK;
    const bool td = (variant & YETI_PCG_FD_TD) != 0;
    YETI_CHECK(!td || op->coef64.ptr, YETI_EUNSUPPORTED,
               "fast diagonalisation 'TD': needs the operator's FP64 data");
    // the passes stage up to kFdSmem bytes: opt in once per device (the
    // attribute is always this maximum, so concurrent callers agree)
    YETI_TRY(fd_set_attrs<double>());
    YETI_TRY(fd_set_attrs<float>());
    yeti_ctx *ctx = op->ctx;
    cudaStream_t s = ctx->stream;
    const bool unit = (variant & YETI_PCG_FD_UNIT) != 0;
    const bool scaled = (variant & YETI_PCG_FD_SCALED) != 0;
    // free boxes
    for (int c = 0; c < 3; c++) {
        YETI_CHECK(op->cmask[c] != 0, YETI_EINVAL,
                   "fast diagonalisation: component %d has no clamped face (singular)", c);
        for (int d = 0; d < 3; d++) {
            const int lo = (op->cmask[c] >> (2 * d)) & 1;
            const int hi = op->n[d] - ((op->cmask[c] >> (2 * d + 1)) & 1);
            F.lo[c][d] = lo;
            F.m[c][d] = hi - lo;
            YETI_CHECK(F.m[c][d] >= 1 && F.m[c][d] <= kFdMaxM, YETI_EINVAL,
                       "fast diagonalisation: %d free functions along direction %d "
                       "(1..%d supported)", F.m[c][d], d, kFdMaxM);
        }
    }
    // coefficients a[c][d] ('TD': 1, the weights carry the coefficients)
    double acoef[3][3];
    if (unit || td) {
        for (int c = 0; c < 3; c++)
            for (int d = 0; d < 3; d++) acoef[c][d] = 1.0;
    } else {
        std::vector<double> sd((size_t)op->nblocks * 9);
        YETI_CUDA(cudaMemcpyAsync(sd.data(), op->sdiag.ptr, sd.size() * sizeof(double),
                                  cudaMemcpyDeviceToHost, s));
        YETI_CUDA(cudaStreamSynchronize(s));
        double sum[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int64_t b = 0; b < op->nblocks; b++)
            for (int k = 0; k < 9; k++) sum[k] += sd[(size_t)b * 9 + k];
        for (int c = 0; c < 3; c++)
            for (int d = 0; d < 3; d++) {
                acoef[c][d] = sum[3 * c + d] / (double)op->nqp_total;
                YETI_CHECK(acoef[c][d] > 0.0 && std::isfinite(acoef[c][d]), YETI_ENUMERIC,
                           "fast diagonalisation: mean coefficient %g", acoef[c][d]);
            }
    }
    // eigenpairs per distinct (p, nel, lo, hi)
    WQRule1D R[3];
    for (int d = 0; d < 3; d++)
        YETI_CHECK(wq_rule_1d(op->p[d], op->nel[d], R[d]) == 0, YETI_EINVAL,
                   "fast diagonalisation: WQ rule failed");
    // 'TD': per component, two sweeps of the tensor decomposition of the
    // diagonal coefficients give per-point 1-D weights (wq_mf_cg_3d,
    // mf_wq_solver.f90:809-826, per displacement component)
    std::vector<double> tdM[3][3], tdK[3][3];
    if (td) {
        const int nq[3] = {op->nqp[0], op->nqp[1], op->nqp[2]};
        const int64_t n = (int64_t)nq[0] * nq[1] * nq[2];
        DevBuf dcc;
        YETI_TRY(dcc.alloc(ctx, (size_t)9 * n * sizeof(double)));
        WQStreamPlan &st = op->st;
        DevBuf blk[3], loc[3], nqb[3], ptrs;   // block-layout maps (freed on return)
        if (st.active) {
            k_fd_diag_coef<<<592, 256, 0, s>>>(op->coef64.as<double>(), st.tile_off.as<int64_t>(),
                                               st.tile_pstride.as<int>(), st.tq0[0].as<int>(),
                                               st.tnq[0].as<int>(), st.tq0[1].as<int>(),
                                               st.tnq[1].as<int>(), st.ntile[0], nq[0], nq[1],
                                               nq[2], dcc.as<double>());
        } else {
            const int *hp[9];
            for (int d = 0; d < 3; d++) {
                std::vector<int> b(nq[d]), l(nq[d]), m(op->blk[d].size());
                for (size_t k = 0; k < op->blk[d].size(); k++) {
                    const BlkInfo &B = op->blk[d][k];
                    m[k] = B.nq;
                    for (int q = 0; q < B.nq; q++) {
                        b[B.q0 + q] = (int)k;
                        l[B.q0 + q] = q;
                    }
                }
                YETI_TRY(upload(ctx, blk[d], b.data(), b.size()));
                YETI_TRY(upload(ctx, loc[d], l.data(), l.size()));
                YETI_TRY(upload(ctx, nqb[d], m.data(), m.size()));
                hp[d] = blk[d].as<int>();
                hp[3 + d] = loc[d].as<int>();
                hp[6 + d] = nqb[d].as<int>();
            }
            YETI_TRY(upload(ctx, ptrs, hp, 9));
            const int *const *dp = ptrs.as<const int *>();
            k_fd_diag_coef_blk<<<592, 256, 0, s>>>(op->coef64.as<double>(), op->qoff.as<int64_t>(),
                                                   dp, dp + 3, dp + 6, (int)op->blk[0].size(),
                                                   (int)op->blk[1].size(), nq[0], nq[1], nq[2],
                                                   dcc.as<double>());
        }
        count_launches(1);
        YETI_CUDA(cudaGetLastError());
        std::vector<double> cc((size_t)9 * n);
        YETI_CUDA(cudaMemcpyAsync(cc.data(), dcc.ptr, cc.size() * sizeof(double),
                                  cudaMemcpyDeviceToHost, s));
        YETI_CUDA(cudaStreamSynchronize(s));
        for (int c = 0; c < 3; c++) {
            std::vector<double> Mw[3], Kw[3];
            for (int d = 0; d < 3; d++) {
                Mw[d].assign(nq[d], 1.0);
                Kw[d].assign(nq[d], 1.0);
            }
            const double *ccp[3] = {&cc[(size_t)(3 * c) * n], &cc[(size_t)(3 * c + 1) * n],
                                    &cc[(size_t)(3 * c + 2) * n]};
            for (int sweep = 0; sweep < 2; sweep++) td_sweep(nq, ccp, Mw, Kw);
            for (int d = 0; d < 3; d++) {
                for (int q = 0; q < nq[d]; q++)
                    YETI_CHECK(Mw[d][q] > 0.0 && Kw[d][q] > 0.0 && std::isfinite(Mw[d][q]) &&
                                   std::isfinite(Kw[d][q]),
                               YETI_ENUMERIC, "fast diagonalisation 'TD': weight %g / %g",
                               Mw[d][q], Kw[d][q]);
                tdM[c][d] = Mw[d];
                tdK[c][d] = Kw[d];
            }
        }
    }
    struct Eig {
        std::vector<double> lam, U, kd, md;
    };
    // unweighted eigenpairs depend on (p, nel, lo, hi) only: operators set
    // up back to back (the serving loop's) share them through a bounded
    // process-wide cache; 'TD' ones are the operator's own
    static std::mutex g_eig_mtx;
    static std::map<std::tuple<int, int, int, int>, Eig> g_eig;
    static std::deque<std::tuple<int, int, int, int>> g_eig_order;
    constexpr size_t kEigCacheEntries = 512;
    std::map<std::tuple<int, int, int, int, int>, Eig> cache;
    Eig *E[3][3];
    for (int c = 0; c < 3; c++)
        for (int d = 0; d < 3; d++) {
            const int lo = F.lo[c][d], hi = lo + F.m[c][d];
            // 'TD' weights differ per component: no sharing between components
            auto key = std::make_tuple(op->p[d], op->nel[d], lo, hi, td ? 3 * c + d : -1);
            auto it = cache.find(key);
            if (it == cache.end() && !td) {
                std::lock_guard<std::mutex> lock(g_eig_mtx);
                auto g = g_eig.find(std::make_tuple(op->p[d], op->nel[d], lo, hi));
                if (g != g_eig.end()) it = cache.emplace(key, g->second).first;
            }
            if (it == cache.end()) {
                Eig e;
                std::vector<double> K, M;
                if (td)
                    wq_1d_matrices_weighted(R[d], lo, hi, tdM[c][d].data(), tdK[c][d].data(), K, M);
                else
                    wq_1d_matrices(R[d], lo, hi, K, M);
                const int m = hi - lo;
                e.kd.resize(m);
                e.md.resize(m);
                for (int i = 0; i < m; i++) {
                    e.kd[i] = K[(size_t)i * m + i];
                    e.md[i] = M[(size_t)i * m + i];
                }
                YETI_CHECK(gen_eig(m, K, M, e.lam, e.U), YETI_ENUMERIC,
                           "fast diagonalisation: eigen decomposition failed (direction %d)", d);
                if (!td) {
                    std::lock_guard<std::mutex> lock(g_eig_mtx);
                    const auto gk = std::make_tuple(op->p[d], op->nel[d], lo, hi);
                    if (g_eig.emplace(gk, e).second) {
                        g_eig_order.push_back(gk);
                        if (g_eig_order.size() > kEigCacheEntries) {
                            g_eig.erase(g_eig_order.front());
                            g_eig_order.pop_front();
                        }
                    }
                }
                it = cache.emplace(key, std::move(e)).first;
            }
            E[c][d] = &it->second;
        }
    // Lambda_c > 0 needs at least one direction without a zero eigenvalue
    for (int c = 0; c < 3; c++) {
        double lmin = 0.0;
        for (int d = 0; d < 3; d++)
            lmin += acoef[c][d] * *std::min_element(E[c][d]->lam.begin(), E[c][d]->lam.end());
        YETI_CHECK(lmin > 0.0, YETI_ENUMERIC,
                   "fast diagonalisation: separable operator of component %d is singular", c);
    }
    // device tables: G (U then U^T) per (c, d); a * lambda; 1-D diagonals
    std::vector<double> g, dsc, kdmd;
    for (int c = 0; c < 3; c++)
        for (int d = 0; d < 3; d++) {
            const int m = F.m[c][d];
            const Eig &e = *E[c][d];
            F.goff[c][d] = (int64_t)g.size();
            g.insert(g.end(), e.U.begin(), e.U.end());
            for (int i = 0; i < m; i++)
                for (int j = 0; j < m; j++) g.push_back(e.U[(size_t)j * m + i]);
            F.doff[c][d] = (int64_t)dsc.size();
            for (int i = 0; i < m; i++) dsc.push_back(acoef[c][d] * e.lam[i]);
            for (int i = 0; i < m; i++) kdmd.push_back(e.kd[i]);
            for (int i = 0; i < m; i++) kdmd.push_back(e.md[i]);
        }
    YETI_TRY(upload(ctx, F.g64, g.data(), g.size()));
    YETI_TRY(upload(ctx, F.d64, dsc.data(), dsc.size()));
    F.g32.release();
    F.d32.release();
    if (f32) {
        std::vector<float> gf(g.begin(), g.end()), df(dsc.begin(), dsc.end());
        YETI_TRY(upload(ctx, F.g32, gf.data(), gf.size()));
        YETI_TRY(upload(ctx, F.d32, df.data(), df.size()));
    }
    // scaling vector
    F.scaled = scaled;
    F.s64.release();
    F.s32.release();
    if (scaled) {
        DevBuf dk;
        YETI_TRY(upload(ctx, dk, kdmd.data(), kdmd.size()));
        YETI_TRY(F.s64.alloc(ctx, op->ndof * sizeof(double)));
        YETI_CUDA(cudaMemsetAsync(F.s64.ptr, 0, op->ndof * sizeof(double), s));
        if (f32) {
            YETI_TRY(F.s32.alloc(ctx, op->ndof * sizeof(float)));
            YETI_CUDA(cudaMemsetAsync(F.s32.ptr, 0, op->ndof * sizeof(float), s));
        }
        for (int c = 0; c < 3; c++) {
            // kdmd offsets: twice the dsc offsets (kd then md per block)
            k_fd_scaling<<<592, 256, 0, s>>>(
                op->diag.as<double>(), dk.as<double>(), F.s64.as<double>(),
                f32 ? F.s32.as<float>() : nullptr, make_int3(op->n[0], op->n[1], op->n[2]),
                op->ncp, F.lo[c][0], F.lo[c][1], F.lo[c][2], F.m[c][0], F.m[c][1], F.m[c][2], c,
                2 * F.doff[c][0], 2 * F.doff[c][1], 2 * F.doff[c][2], acoef[c][0], acoef[c][1],
                acoef[c][2]);
            count_launches(1);
        }
        YETI_CUDA(cudaGetLastError());
        YETI_CUDA(cudaStreamSynchronize(s));   // dk is freed on return
    }
    // intermediates and reduction partials
    YETI_TRY(F.t64.alloc(ctx, 2 * op->ndof * sizeof(double)));
    F.t32.release();
    if (f32) YETI_TRY(F.t32.alloc(ctx, 2 * op->ndof * sizeof(float)));
    int maxg = 0;
    for (int ax = 0; ax < 3; ax++)
        for (int fused = 0; fused < 2; fused++) {
            int tot = 0;
            for (int c = 0; c < 3; c++) {
                const int64_t nl = (int64_t)F.m[c][(ax == 0) ? 1 : 0] * F.m[c][(ax == 2) ? 1 : 2];
                for (size_t es : {sizeof(double), sizeof(float)})
                    tot += std::max(0, fd_tile(F.m[c][ax], nl, es, fused).ctas);
            }
            maxg = std::max(maxg, tot);
        }
    for (size_t es : {sizeof(double), sizeof(float)}) {
        int tot = 0;
        for (int c = 0; c < 3; c++)
            tot += std::max(0, fd_plane_tile(F.m[c][0], F.m[c][1], F.m[c][2], es).ctas);
        maxg = std::max(maxg, tot);
    }
    F.max_grid = maxg;
    YETI_TRY(F.parts.alloc(ctx, (size_t)maxg * sizeof(double)));
    // the tables were uploaded (and, on a stream-ordered context,
    // allocated) on the context's stream; solves may run on other streams
    YETI_CUDA(cudaStreamSynchronize(s));
    F.variant = variant;
    return YETI_OK;
}

template <class T> struct FdBufs;
template <> struct FdBufs<double> {
    static const double *g(const WQFdPlan &F) { return F.g64.as<double>(); }
    static const double *d(const WQFdPlan &F) { return F.d64.as<double>(); }
    static const double *s(const WQFdPlan &F) { return F.s64.as<double>(); }
    static double *t(const WQFdPlan &F) { return F.t64.as<double>(); }
};
template <> struct FdBufs<float> {
    static const float *g(const WQFdPlan &F) { return F.g32.as<float>(); }
    static const float *d(const WQFdPlan &F) { return F.d32.as<float>(); }
    static const float *s(const WQFdPlan &F) { return F.s32.as<float>(); }
    static float *t(const WQFdPlan &F) { return F.t32.as<float>(); }
};

template <class T, int AX, int EPI>
static int fd_pass(yeti_wq_op *op, FdArgs<T> a, bool bwd, cudaStream_t s) {
    const WQFdPlan &F = op->fd;
    int tot = 0, threads = 32;
    size_t smem = 0;
    for (int c = 0; c < 3; c++) {
        const int m = F.m[c][AX];
        const int64_t nl = (int64_t)F.m[c][AX == 0 ? 1 : 0] * F.m[c][AX == 2 ? 1 : 2];
        const FdTile t = fd_tile(m, nl, sizeof(T), EPI == 3);
        YETI_CHECK(t.ctas > 0, YETI_EINVAL, "fast diagonalisation: no tiling for m=%d", m);
        a.nag[c] = t.nag;
        a.nlg[c] = t.nlg;
        a.ntA[c] = t.ntA;
        tot += t.ctas;
        a.cta_end[c] = tot;
        a.goff[c] = F.goff[c][AX] + (bwd ? (int64_t)m * m : 0);
        a.goff2[c] = F.goff[c][AX] + (int64_t)m * m;
        smem = std::max(smem, t.smem);
        threads = std::max(threads, t.threads);
    }
    // every component's tile fits `threads` (nag nlg <= threads).  The
    // shared-memory opt-in (the 48 KB default covers static plus dynamic
    // memory) is set by wq_fd_prepare on this device, outside any capture
    k_fd_pass<T, AX, EPI><<<tot, threads, smem, s>>>(a);
    count_launches(1);
    return YETI_OK;
}

// The fused u and v products of every w plane (forward or backward).
template <class T, int EPI>
static int fd_plane(yeti_wq_op *op, FdArgs<T> a, bool bwd, cudaStream_t s) {
    const WQFdPlan &F = op->fd;
    int tot = 0, threads = 32;
    size_t smem = 0;
    for (int c = 0; c < 3; c++) {
        const int mu = F.m[c][0], mv = F.m[c][1];
        const FdPlane t = fd_plane_tile(mu, mv, F.m[c][2], sizeof(T));
        YETI_CHECK(t.ctas > 0, YETI_EINVAL, "fast diagonalisation: plane %dx%d does not fit", mu, mv);
        a.ntA[c] = t.nsplit;
        a.nag[c] = t.nag;
        a.nlg[c] = t.nvg;
        tot += t.ctas;
        a.cta_end[c] = tot;
        a.goff[c] = F.goff[c][0] + (bwd ? (int64_t)mu * mu : 0);
        a.goff2[c] = F.goff[c][1] + (bwd ? (int64_t)mv * mv : 0);
        smem = std::max(smem, t.smem);
        threads = std::max(threads, t.threads);
    }
    k_fd_plane<T, EPI><<<tot, threads, smem, s>>>(a);
    count_launches(1);
    return YETI_OK;
}

// The fused plane pass pays off when its tile leaves room for two CTAs per
// SM (measured at 64^3: FP32, 57 KB, 24 us against 2 x 16.5 us for the two
// line passes; FP64, 114 KB, one CTA per SM, 63 us against 2 x 29 us).
constexpr size_t kFdPlaneSmem = 100 * 1024;
static bool fd_planes_fit(const WQFdPlan &F, size_t esize) {
    for (int c = 0; c < 3; c++) {
        const FdPlane t = fd_plane_tile(F.m[c][0], F.m[c][1], F.m[c][2], esize);
        if (t.ctas <= 0 || t.smem > kFdPlaneSmem) return false;
    }
    return true;
}

// The w pass can run fused (forward, division, backward in one CTA) when
// every component's w tile is a single row tile that fits.
static bool fd_w_fused(const WQFdPlan &F, size_t esize) {
    for (int c = 0; c < 3; c++) {
        if (F.m[c][2] > kFdTA) return false;
        if (fd_tile(F.m[c][2], (int64_t)F.m[c][0] * F.m[c][1], esize, true).ctas <= 0) return false;
    }
    return true;
}

template <class T>
int wq_fd_apply(yeti_wq_op *op, const T *in, T *out, const int *done, int red, T *p,
                CGScal *cg, cudaStream_t s, T *tmp, double *parts) {
    const WQFdPlan &F = op->fd;
    FdArgs<T> a;
    a.g = FdBufs<T>::g(F);
    a.dsc = FdBufs<T>::d(F);
    a.s = F.scaled ? FdBufs<T>::s(F) : nullptr;
    a.r = in;
    a.p = p;
    a.done = done;
    a.cg = cg;
    a.parts = parts ? parts : F.parts.as<double>();
    a.red = red;
    for (int d = 0; d < 3; d++) a.n[d] = op->n[d];
    a.ncp = op->ncp;
    for (int c = 0; c < 3; c++)
        for (int d = 0; d < 3; d++) {
            a.lo[c][d] = F.lo[c][d];
            a.m[c][d] = F.m[c][d];
            a.doff[c][d] = F.doff[c][d];
        }
    T *t0 = tmp ? tmp : FdBufs<T>::t(F), *t1 = t0 + op->ndof;
    a.in = in;
    if (F.scaled) {
        // t1 = s r on the free boxes (the first pass reads the boxes only)
        k_fd_scale_in<T><<<592, 256, 0, s>>>(in, a.s, t1, op->ndof, done);
        count_launches(1);
        a.in = t1;
    }
    if (fd_planes_fit(F, sizeof(T)) && fd_w_fused(F, sizeof(T))) {
        // three launches: u and v forward per plane, w, u and v backward
        a.out = t0;
        YETI_TRY((fd_plane<T, 0>(op, a, false, s)));
        a.in = t0;
        a.out = t1;
        YETI_TRY((fd_pass<T, 2, 3>(op, a, false, s)));
        a.in = t1;
        a.out = out;
        YETI_TRY((fd_plane<T, 2>(op, a, true, s)));
        YETI_CUDA(cudaGetLastError());
        return YETI_OK;
    }
    a.out = t0;
    YETI_TRY((fd_pass<T, 0, 0>(op, a, false, s)));
    a.in = t0;
    a.out = t1;
    YETI_TRY((fd_pass<T, 1, 0>(op, a, false, s)));
    a.in = t1;
    a.out = t0;
    if (fd_w_fused(F, sizeof(T))) {
        YETI_TRY((fd_pass<T, 2, 3>(op, a, false, s)));
    } else {
        YETI_TRY((fd_pass<T, 2, 1>(op, a, false, s)));
        a.in = t0;
        a.out = t1;
        YETI_TRY((fd_pass<T, 2, 0>(op, a, true, s)));
        std::swap(t0, t1);
    }
    a.in = t0;
    a.out = t1;
    YETI_TRY((fd_pass<T, 1, 0>(op, a, true, s)));
    a.in = t1;
    a.out = out;
    YETI_TRY((fd_pass<T, 0, 2>(op, a, true, s)));
    YETI_CUDA(cudaGetLastError());
    return YETI_OK;
}

template int wq_fd_apply<double>(yeti_wq_op *, const double *, double *, const int *, int,
                                 double *, CGScal *, cudaStream_t, double *, double *);
template int wq_fd_apply<float>(yeti_wq_op *, const float *, float *, const int *, int, float *,
                                CGScal *, cudaStream_t, float *, double *);

int wq_fd_parts(const yeti_wq_op *op) { return op->fd.max_grid; }

}  // namespace yeti

using namespace yeti;

YETI_API int yeti_wq_fd_apply(yeti_wq_op *op, const void *r, void *z, int prec, int variant,
                              int mem) {
    YETI_CHECK(op && r && z, YETI_EINVAL, "yeti_wq_fd_apply: NULL argument");
    YETI_CHECK(prec == YETI_PREC_F64 || prec == YETI_PREC_F32, YETI_EINVAL,
               "yeti_wq_fd_apply: prec %d", prec);
    YETI_CHECK((variant & YETI_PCG_FD) && !(variant & ~(YETI_PCG_FD | YETI_PCG_FD_SCALED |
                                                       YETI_PCG_FD_UNIT | YETI_PCG_FD_TD)) &&
                   !((variant & YETI_PCG_FD_UNIT) && (variant & YETI_PCG_FD_TD)),
               YETI_EINVAL, "yeti_wq_fd_apply: variant %d", variant);
    DeviceGuard guard(op->ctx->device);
    const bool f32 = prec == YETI_PREC_F32;
    YETI_TRY(wq_fd_prepare(op, variant, f32));
    cudaStream_t s = op->ctx->stream;
    const size_t es = f32 ? sizeof(float) : sizeof(double);
    const size_t bytes = (size_t)op->ndof * es;
    DevBuf dr, dz;
    const void *rin = r;
    void *zout = z;
    if (mem == YETI_MEM_HOST) {
        YETI_TRY(dr.alloc(op->ctx, bytes));
        YETI_TRY(dz.alloc(op->ctx, bytes));
        YETI_CUDA(cudaMemcpyAsync(dr.ptr, r, bytes, cudaMemcpyHostToDevice, s));
        rin = dr.ptr;
        zout = dz.ptr;
    }
    YETI_CUDA(cudaMemsetAsync(zout, 0, bytes, s));
    if (f32)
        YETI_TRY(wq_fd_apply<float>(op, (const float *)rin, (float *)zout, nullptr, FD_NONE,
                                    nullptr, nullptr, s));
    else
        YETI_TRY(wq_fd_apply<double>(op, (const double *)rin, (double *)zout, nullptr, FD_NONE,
                                     nullptr, nullptr, s));
    if (mem == YETI_MEM_HOST)
        YETI_CUDA(cudaMemcpyAsync(z, zout, bytes, cudaMemcpyDeviceToHost, s));
    YETI_CUDA(cudaStreamSynchronize(s));
    return YETI_OK;
}
