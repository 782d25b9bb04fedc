// Weighted-quadrature (WQ) matrix-free elasticity on one NURBS patch.
//
// Replaces the reference's WQ path (src/yeti_iga/iga_wq_mf/fsrc):
//   jacobien_physicalposition_3d (wq_assembly.f90:233-473) and
//   eval_mech_coefficient (wq_assembly.f90:52-138)       -> k_wq_setup
//   mf_wq_get_ku_3d (mf_wq_solver.f90:284-544)            -> k_wq_apply
//   wq_find_conductivity_diagonal_3d / find_physical_diag_3d
//     (mf_wq_solver.f90:6-164, tensor_algebra.f90:1484-1596) -> k_wq_diag
//   wq_get_force_3d (wq_assembly.f90:1193-1251)           -> k_wq_force
//   wq_mf_cg_3d 'WP' (mf_wq_solver.f90:764-802)           -> yeti_wq_pcg
// generalised from the scalar operator to 3x3 elastic blocks, with B-spline
// test and trial functions on the exact NURBS geometry (the Jacobian uses
// the control-point weights); the math is stated in oracle/wq_ops.py.
//
// Kernel design (one CTA per element block, all stages in shared memory):
//   load    the block's dense 1-D tiles (functions x owned points) for the
//           three directions and the block's control-point values;
//   forward sum factorisation w -> v -> u: 4 trial kinds (value, d/du,
//           d/dv, d/dw) per component at the block's points;
//   point   per component i, the channels H^{kappa,lambda}_i from the
//           streamed 45 coefficients (the HBM stream of the operator);
//           the value channels (kappa or lambda = 0) are zero;
//   backward sum factorisation u -> v -> w with the 1-D weights
//           W^{[d==kappa][d==lambda]}, channels merged as soon as their
//           remaining weights coincide (16 -> 9 -> 4 -> 1);
//   store   atomic adds of the block's function values into K u (functions
//           are shared with neighbouring blocks; the output vector is a few
//           MB and stays in L2).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>

#include "wq.cuh"

namespace yeti {

// ----------------------------------------------------------- channel tables
// channel ch = 4*kappa + lambda; group g = distinct (t_v, t_w); tv, tw, tu
// encode (test order, trial order) of a direction as 2*test + trial.
__constant__ int c_grp_nch[9] = {4, 2, 2, 2, 1, 1, 2, 1, 1};
__constant__ int c_grp_ch[9][4] = {{0, 1, 4, 5}, {2, 6, 0, 0}, {3, 7, 0, 0},
                                   {8, 9, 0, 0}, {10, 0, 0, 0}, {11, 0, 0, 0},
                                   {12, 13, 0, 0}, {14, 0, 0, 0}, {15, 0, 0, 0}};
__constant__ int c_grp_tv[9] = {0, 1, 0, 2, 3, 2, 0, 1, 0};
__constant__ int c_h_ng[4] = {4, 2, 2, 1};
__constant__ int c_h_g[4][4] = {{0, 1, 3, 4}, {2, 5, 0, 0}, {6, 7, 0, 0},
                                {8, 0, 0, 0}};

__device__ __forceinline__ int ch_tu(int ch) {
    const int k = ch >> 2, l = ch & 3;
    return 2 * (k == 1) + (l == 1);
}

struct BlkCtx {
    BlkInfo b[3];
    int nf[3], nq[3];
    int nqb;
    int64_t qoff;
};

__device__ inline void block_ctx(const WQAxis *ax, const int64_t *qoff,
                                 int64_t bid, BlkCtx &c) {
    const int bu = (int)(bid % ax[0].nb);
    const int64_t r = bid / ax[0].nb;
    const int bv = (int)(r % ax[1].nb);
    const int bw = (int)(r / ax[1].nb);
    c.b[0] = ax[0].blk[bu];
    c.b[1] = ax[1].blk[bv];
    c.b[2] = ax[2].blk[bw];
    for (int d = 0; d < 3; d++) {
        c.nf[d] = c.b[d].ne + ax[d].p;
        c.nq[d] = c.b[d].nq;
    }
    c.nqb = c.nq[0] * c.nq[1] * c.nq[2];
    c.qoff = qoff[bid];
}

__device__ __forceinline__ bool clamped(int cm, const WQAxis *ax, int gu,
                                        int gv, int gw) {
    return ((cm & 1) && gu == 0) || ((cm & 2) && gu == ax[0].nfun - 1) ||
           ((cm & 4) && gv == 0) || ((cm & 8) && gv == ax[1].nfun - 1) ||
           ((cm & 16) && gw == 0) || ((cm & 32) && gw == ax[2].nfun - 1);
}

// Shared-memory carve-up (in elements of T), identical on host and device.
struct SmemPlan {
    int tile[3];     // offsets of the three direction tiles
    int X, F, R1;    // control-point values, point values, scratch union
    int total;
};

__host__ __device__ inline SmemPlan smem_plan(const int NF[3], const int NQ[3],
                                              int NC, int ntile) {
    SmemPlan s;
    int o = 0;
    for (int d = 0; d < 3; d++) {
        s.tile[d] = o;
        o += ntile * NF[d] * NQ[d];
    }
    s.X = o;
    o += NC * NF[0] * NF[1] * NF[2];
    s.F = o;
    const int nq = NQ[0] * NQ[1] * NQ[2];
    o += 4 * NC * nq;
    s.R1 = o;
    const int y = 2 * NC * NQ[2] * NF[1] * NF[0];
    const int z = 3 * NC * NQ[2] * NQ[1] * NF[0];
    const int h = 16 * nq;
    const int g = 9 * NQ[2] * NQ[1] * NF[0];
    const int k = 4 * NQ[2] * NF[1] * NF[0];
    o += (y + z > h + g + k) ? (y + z) : (h + g + k);
    s.total = o;
    return s;
}

// Forward sum factorisation: X[NC][nfw][nfv][nfu] -> F[4][NC][nqw][nqv][nqu].
template <class T, int NC>
__device__ void forward(const T *tu, const T *tv, const T *tw, const int NF[3],
                        const int NQ[3], const BlkCtx &c, const T *X, T *Y,
                        T *Z, T *F) {
    const int nfu = c.nf[0], nfv = c.nf[1], nfw = c.nf[2];
    const int nqu = c.nq[0], nqv = c.nq[1], nqw = c.nq[2];
    // Y[t][c][qw][fv][fu] = sum_fw Bw_t[fw][qw] X[c][fw][fv][fu]
    const int n1 = 2 * NC * nqw * nfv * nfu;
    for (int o = threadIdx.x; o < n1; o += blockDim.x) {
        const int fu = o % nfu;
        int r = o / nfu;
        const int fv = r % nfv;
        r /= nfv;
        const int qw = r % nqw;
        r /= nqw;
        const int cc = r % NC, t = r / NC;
        const T *B = tw + t * NF[2] * NQ[2] + qw;
        const T *x = X + (cc * nfw * nfv + fv) * nfu + fu;
        T acc = 0;
        for (int fw = 0; fw < nfw; fw++) acc += B[fw * NQ[2]] * x[fw * nfv * nfu];
        Y[o] = acc;
    }
    __syncthreads();
    // Z[s][c][qw][qv][fu]: s=0 Bv0.Y0, s=1 Bv1.Y0, s=2 Bv0.Y1
    const int n2 = 3 * NC * nqw * nqv * nfu;
    for (int o = threadIdx.x; o < n2; o += blockDim.x) {
        const int fu = o % nfu;
        int r = o / nfu;
        const int qv = r % nqv;
        r /= nqv;
        const int qw = r % nqw;
        r /= nqw;
        const int cc = r % NC, s = r / NC;
        const int ms = (s == 1), ys = (s == 2);
        const T *B = tv + ms * NF[1] * NQ[1] + qv;
        const T *y = Y + (((ys * NC + cc) * nqw + qw) * nfv) * nfu + fu;
        T acc = 0;
        for (int fv = 0; fv < nfv; fv++) acc += B[fv * NQ[1]] * y[fv * nfu];
        Z[o] = acc;
    }
    __syncthreads();
    // F[l][c][qw][qv][qu]: l=0 Bu0.Z0, 1 Bu1.Z0, 2 Bu0.Z1, 3 Bu0.Z2
    const int n3 = 4 * NC * nqw * nqv * nqu;
    for (int o = threadIdx.x; o < n3; o += blockDim.x) {
        const int qu = o % nqu;
        int r = o / nqu;
        const int qv = r % nqv;
        r /= nqv;
        const int qw = r % nqw;
        r /= nqw;
        const int cc = r % NC, l = r / NC;
        const int ml = (l == 1), zl = (l >= 2) ? l - 1 : 0;
        const T *B = tu + ml * NF[0] * NQ[0] + qu;
        const T *z = Z + (((zl * NC + cc) * nqw + qw) * nqv + qv) * nfu;
        T acc = 0;
        for (int fu = 0; fu < nfu; fu++) acc += B[fu * NQ[0]] * z[fu];
        F[o] = acc;
    }
    __syncthreads();
}

// Backward sum factorisation of one component:
// H[16][nqw][nqv][nqu] -> out[nfw][nfv][nfu], weights at tile slots
// wbase + (2*test + trial).
template <class T>
__device__ void backward(const T *tu, const T *tv, const T *tw, int wbase,
                         const int NF[3], const int NQ[3], const BlkCtx &c,
                         const T *H, T *G, T *K, T *out) {
    const int nfu = c.nf[0], nfv = c.nf[1], nfw = c.nf[2];
    const int nqu = c.nq[0], nqv = c.nq[1], nqw = c.nq[2];
    const int nqb = c.nqb;
    // G[g][qw][qv][fu] = sum_{ch in g} sum_qu Wu_tu(ch)[fu][qu] H[ch][qw][qv][qu]
    const int n1 = 9 * nqw * nqv * nfu;
    for (int o = threadIdx.x; o < n1; o += blockDim.x) {
        const int fu = o % nfu;
        int r = o / nfu;
        const int qv = r % nqv;
        r /= nqv;
        const int qw = r % nqw;
        const int g = r / nqw;
        T acc = 0;
        const int nch = c_grp_nch[g];
        for (int k = 0; k < nch; k++) {
            const int ch = c_grp_ch[g][k];
            const T *W = tu + (wbase + ch_tu(ch)) * NF[0] * NQ[0] + fu * NQ[0];
            const T *h = H + ch * nqb + (qw * nqv + qv) * nqu;
            for (int qu = 0; qu < nqu; qu++) acc += W[qu] * h[qu];
        }
        G[o] = acc;
    }
    __syncthreads();
    // K[h][qw][fv][fu] = sum_{g in h} sum_qv Wv_tv(g)[fv][qv] G[g][qw][qv][fu]
    const int n2 = 4 * nqw * nfv * nfu;
    for (int o = threadIdx.x; o < n2; o += blockDim.x) {
        const int fu = o % nfu;
        int r = o / nfu;
        const int fv = r % nfv;
        r /= nfv;
        const int qw = r % nqw;
        const int h = r / nqw;
        T acc = 0;
        const int ng = c_h_ng[h];
        for (int k = 0; k < ng; k++) {
            const int g = c_h_g[h][k];
            const T *W = tv + (wbase + c_grp_tv[g]) * NF[1] * NQ[1] + fv * NQ[1];
            const T *gg = G + ((g * nqw + qw) * nqv) * nfu + fu;
            for (int qv = 0; qv < nqv; qv++) acc += W[qv] * gg[qv * nfu];
        }
        K[o] = acc;
    }
    __syncthreads();
    // out[fw][fv][fu] = sum_h sum_qw Ww_h[fw][qw] K[h][qw][fv][fu]
    const int n3 = nfw * nfv * nfu;
    for (int o = threadIdx.x; o < n3; o += blockDim.x) {
        const int fu = o % nfu;
        int r = o / nfu;
        const int fv = r % nfv;
        const int fw = r / nfv;
        T acc = 0;
        for (int h = 0; h < 4; h++) {
            const T *W = tw + (wbase + h) * NF[2] * NQ[2] + fw * NQ[2];
            const T *kk = K + ((h * nqw) * nfv + fv) * nfu + fu;
            for (int qw = 0; qw < nqw; qw++) acc += W[qw] * kk[qw * nfv * nfu];
        }
        out[o] = acc;
    }
    __syncthreads();
}

// Block position of the block index along each direction.
__device__ __forceinline__ void block_pos(const WQAxis *ax, int64_t bid,
                                          int pos[3]) {
    pos[0] = (int)(bid % ax[0].nb);
    const int64_t r = bid / ax[0].nb;
    pos[1] = (int)(r % ax[1].nb);
    pos[2] = (int)(r / ax[1].nb);
}

template <class T>
__device__ inline void copy_tiles(const WQAxis *ax, const T *const *tiles,
                                  const int pos[3], int ntile_src,
                                  int first_src, int nt, int dst_slot, T *sm,
                                  const SmemPlan &P, int ntile_dst) {
    for (int d = 0; d < 3; d++) {
        const int per = ax[d].NF * ax[d].NQ;
        const T *src = tiles[d] + ((size_t)pos[d] * ntile_src + first_src) * per;
        T *dst = sm + P.tile[d] + (size_t)dst_slot * per;
        for (int i = threadIdx.x; i < nt * per; i += blockDim.x) dst[i] = src[i];
        (void)ntile_dst;
    }
}

// ------------------------------------------------------------------ setup
struct SetupArgs {
    WQView<double> v;          // tiles64 + axes (coef unused)
    const double *cps;         // (3, ncp)
    const double *wts;         // ncp: geometry weights
    double mdm[81];
    double *coef64;            // may be null
    float *coef32;             // may be null
    double *jw;                // |detJ|
    double *sdiag;             // [block][9]: sums of S[(c,d),(c,d)]
    int *flags;                // bit0: detJ > 0 seen, bit1: < 0, bit2: bad
};

__global__ void __launch_bounds__(kWQThreads) k_wq_setup(SetupArgs a) {
    extern __shared__ __align__(16) unsigned char smraw[];
    double *sm = reinterpret_cast<double *>(smraw);
    const WQAxis *ax = a.v.ax;
    const int NF[3] = {ax[0].NF, ax[1].NF, ax[2].NF};
    const int NQ[3] = {ax[0].NQ, ax[1].NQ, ax[2].NQ};
    const SmemPlan P = smem_plan(NF, NQ, 4, 2);
    BlkCtx c;
    block_ctx(ax, a.v.qoff, blockIdx.x, c);
    int pos[3];
    block_pos(ax, blockIdx.x, pos);
    copy_tiles<double>(ax, a.v.tiles, pos, 6, 0, 2, 0, sm, P, 2);
    // X[4][fw][fv][fu] = (w x, w y, w z, w)
    const int nfu = c.nf[0], nfv = c.nf[1], nfw = c.nf[2];
    double *X = sm + P.X;
    const int nx = nfu * nfv * nfw;
    for (int o = threadIdx.x; o < nx; o += blockDim.x) {
        const int fu = o % nfu, fv = (o / nfu) % nfv, fw = o / (nfu * nfv);
        const int64_t cp = (c.b[0].e0 + fu) +
                           (int64_t)ax[0].nfun * ((c.b[1].e0 + fv) + (int64_t)ax[1].nfun * (c.b[2].e0 + fw));
        const double w = a.wts[cp];
        for (int cc = 0; cc < 3; cc++) X[cc * nx + o] = w * a.cps[3 * cp + cc];
        X[3 * nx + o] = w;
    }
    __syncthreads();
    double *F = sm + P.F;
    double *Y = sm + P.R1;
    double *Z = Y + 2 * 4 * NQ[2] * NF[1] * NF[0];
    forward<double, 4>(sm + P.tile[0], sm + P.tile[1], sm + P.tile[2], NF, NQ,
                       c, X, Y, Z, F);
    const int nqb = c.nqb;
    int flags = 0;
    double sd[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int q = threadIdx.x; q < nqb; q += blockDim.x) {
        double f[4][4];   // [lambda][component]
        for (int l = 0; l < 4; l++)
            for (int cc = 0; cc < 4; cc++) f[l][cc] = F[(l * 4 + cc) * nqb + q];
        const double W = f[0][3];
        double J[3][3], x[3];
        for (int cc = 0; cc < 3; cc++) x[cc] = f[0][cc] / W;
        for (int cc = 0; cc < 3; cc++)
            for (int l = 0; l < 3; l++) J[cc][l] = (f[l + 1][cc] - x[cc] * f[l + 1][3]) / W;
        const double det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
                           J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
                           J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
        if (!(det == det) || det == 0.0 || !(W > 0.0)) flags |= 4;
        else flags |= det > 0 ? 1 : 2;
        const double id = 1.0 / det;
        double iJ[3][3];   // iJ[k][d] = dxi_k / dx_d
        iJ[0][0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) * id;
        iJ[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) * id;
        iJ[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) * id;
        iJ[1][0] = (J[1][2] * J[2][0] - J[1][0] * J[2][2]) * id;
        iJ[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * id;
        iJ[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * id;
        iJ[2][0] = (J[1][0] * J[2][1] - J[1][1] * J[2][0]) * id;
        iJ[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * id;
        iJ[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * id;
        const double scale = fabs(det);
        const int64_t base = c.qoff * kWQCoef;
        // S[(i,k),(j,l)] = sum_{d,f} iJ[k][d] MDM[(i,d),(j,f)] iJ[l][f] |det|
        for (int I = 0; I < 9; I++) {
            const int i = I / 3, k = I % 3;
            for (int Jn = I; Jn < 9; Jn++) {
                const int j = Jn / 3, l = Jn % 3;
                double s = 0.0;
                for (int d = 0; d < 3; d++) {
                    double t = 0.0;
                    for (int ff = 0; ff < 3; ff++) t += a.mdm[(3 * i + d) * 9 + 3 * j + ff] * iJ[l][ff];
                    s += iJ[k][d] * t;
                }
                s *= scale;
                if (Jn == I) sd[I] += s;
                const int e = sym9(I, Jn);
                if (a.coef64) a.coef64[base + (int64_t)e * nqb + q] = s;
                if (a.coef32) a.coef32[base + (int64_t)e * nqb + q] = (float)s;
            }
        }
        a.jw[c.qoff + q] = fabs(det);
    }
    if (flags) atomicOr(a.flags, flags);
    // block sums of the coefficient diagonal (fixed order: warp tree, then
    // warps in index order)
    __syncthreads();
    double *red = sm;   // the tiles are no longer needed
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int I = 0; I < 9; I++) {
        double v = sd[I];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) red[I * 8 + wid] = v;
    }
    __syncthreads();
    if (threadIdx.x < 9) {
        double v = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) v += red[threadIdx.x * 8 + w];
        a.sdiag[(int64_t)blockIdx.x * 9 + threadIdx.x] = v;
    }
}

// ------------------------------------------------------------------ apply
template <class T>
struct ApplyArgs {
    WQView<T> v;
    const T *u;
    T *Ku;
    const int *done;   // optional early-exit flag (PCG)
};

// Pointwise map of component i: the 16 channels from the 9 derivative
// trial values (value channels are zero).
template <class T>
__device__ __forceinline__ void point_channels(const T *coef, int64_t base,
                                               int nqb, int q, int i,
                                               const T *F, T *H) {
    T f[3][3];
    for (int l = 0; l < 3; l++)
        for (int j = 0; j < 3; j++) f[l][j] = F[((l + 1) * 3 + j) * nqb + q];
    T h[16];
    for (int ch = 0; ch < 4; ch++) h[ch] = 0;
    for (int k = 0; k < 3; k++) {
        T S[9];
        for (int Jn = 0; Jn < 9; Jn++) S[Jn] = coef[base + (int64_t)sym9(3 * i + k, Jn) * nqb + q];
        h[(k + 1) * 4] = 0;
        for (int l = 0; l < 3; l++) {
            T acc = 0;
            for (int j = 0; j < 3; j++) acc += S[3 * j + l] * f[l][j];
            h[(k + 1) * 4 + (l + 1)] = acc;
        }
    }
    for (int ch = 0; ch < 16; ch++) H[ch * nqb + q] = h[ch];
}

template <class T>
__global__ void __launch_bounds__(kWQThreads) k_wq_apply(ApplyArgs<T> a) {
    if (a.done && *a.done) return;
    extern __shared__ __align__(16) unsigned char smraw[];
    T *sm = reinterpret_cast<T *>(smraw);
    const WQAxis *ax = a.v.ax;
    const int NF[3] = {ax[0].NF, ax[1].NF, ax[2].NF};
    const int NQ[3] = {ax[0].NQ, ax[1].NQ, ax[2].NQ};
    const SmemPlan P = smem_plan(NF, NQ, 3, 6);
    BlkCtx c;
    block_ctx(ax, a.v.qoff, blockIdx.x, c);
    int pos[3];
    block_pos(ax, blockIdx.x, pos);
    copy_tiles<T>(ax, a.v.tiles, pos, 6, 0, 6, 0, sm, P, 6);
    const int nfu = c.nf[0], nfv = c.nf[1], nfw = c.nf[2];
    const int nx = nfu * nfv * nfw;
    T *X = sm + P.X;
    for (int o = threadIdx.x; o < nx; o += blockDim.x) {
        const int fu = o % nfu, fv = (o / nfu) % nfv, fw = o / (nfu * nfv);
        const int gu = c.b[0].e0 + fu, gv = c.b[1].e0 + fv, gw = c.b[2].e0 + fw;
        const int64_t cp = gu + (int64_t)ax[0].nfun * (gv + (int64_t)ax[1].nfun * gw);
        for (int cc = 0; cc < 3; cc++)
            X[cc * nx + o] = clamped(a.v.cmask[cc], ax, gu, gv, gw) ? T(0) : a.u[cc * a.v.ncp + cp];
    }
    __syncthreads();
    T *F = sm + P.F;
    T *Y = sm + P.R1;
    T *Z = Y + 2 * 3 * NQ[2] * NF[1] * NF[0];
    forward<T, 3>(sm + P.tile[0], sm + P.tile[1], sm + P.tile[2], NF, NQ, c, X,
                  Y, Z, F);
    const int nqb = c.nqb;
    T *H = sm + P.R1;
    T *G = H + 16 * NQ[0] * NQ[1] * NQ[2];
    T *K = G + 9 * NQ[2] * NQ[1] * NF[0];
    T *out = X;   // X is dead after the forward pass
    const int64_t base = c.qoff * kWQCoef;
    for (int i = 0; i < 3; i++) {
        for (int q = threadIdx.x; q < nqb; q += blockDim.x)
            point_channels<T>(a.v.coef, base, nqb, q, i, F, H);
        __syncthreads();
        backward<T>(sm + P.tile[0], sm + P.tile[1], sm + P.tile[2], 2, NF, NQ, c,
                    H, G, K, out);
        for (int o = threadIdx.x; o < nx; o += blockDim.x) {
            const int fu = o % nfu, fv = (o / nfu) % nfv, fw = o / (nfu * nfv);
            const int gu = c.b[0].e0 + fu, gv = c.b[1].e0 + fv, gw = c.b[2].e0 + fw;
            if (clamped(a.v.cmask[i], ax, gu, gv, gw)) continue;
            const int64_t cp = gu + (int64_t)ax[0].nfun * (gv + (int64_t)ax[1].nfun * gw);
            atomicAdd(&a.Ku[i * a.v.ncp + cp], out[o]);
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------------- diag
// diag_(a,i) = sum_{kappa,lambda >= 1} sum_q (W^{kappa,lambda} .* B^lambda)_a(q)
//              S[(i,kappa),(i,lambda)](q)
template <class T>
struct DiagArgs {
    WQView<T> v;
    const T *dtiles[3];   // [nb][4][NF][NQ]: W00.B0 W01.B1 W10.B0 W11.B1
    double *diag;
};

template <class T>
__global__ void __launch_bounds__(kWQThreads) k_wq_diag(DiagArgs<T> a) {
    extern __shared__ __align__(16) unsigned char smraw[];
    T *sm = reinterpret_cast<T *>(smraw);
    const WQAxis *ax = a.v.ax;
    const int NF[3] = {ax[0].NF, ax[1].NF, ax[2].NF};
    const int NQ[3] = {ax[0].NQ, ax[1].NQ, ax[2].NQ};
    const SmemPlan P = smem_plan(NF, NQ, 3, 6);
    BlkCtx c;
    block_ctx(ax, a.v.qoff, blockIdx.x, c);
    int pos[3];
    block_pos(ax, blockIdx.x, pos);
    copy_tiles<T>(ax, a.dtiles, pos, 4, 0, 4, 2, sm, P, 6);
    __syncthreads();
    const int nfu = c.nf[0], nfv = c.nf[1], nfw = c.nf[2];
    const int nx = nfu * nfv * nfw;
    const int nqb = c.nqb;
    T *H = sm + P.R1;
    T *G = H + 16 * NQ[0] * NQ[1] * NQ[2];
    T *K = G + 9 * NQ[2] * NQ[1] * NF[0];
    T *out = sm + P.X;
    const int64_t base = c.qoff * kWQCoef;
    const T *coef = a.v.coef;
    for (int i = 0; i < 3; i++) {
        for (int q = threadIdx.x; q < nqb; q += blockDim.x) {
            for (int kap = 0; kap < 4; kap++)
                for (int lam = 0; lam < 4; lam++)
                    H[(kap * 4 + lam) * nqb + q] =
                        (kap && lam) ? coef[base + (int64_t)sym9(3 * i + kap - 1, 3 * i + lam - 1) * nqb + q]
                                     : T(0);
        }
        __syncthreads();
        backward<T>(sm + P.tile[0], sm + P.tile[1], sm + P.tile[2], 2, NF, NQ, c,
                    H, G, K, out);
        for (int o = threadIdx.x; o < nx; o += blockDim.x) {
            const int fu = o % nfu, fv = (o / nfu) % nfv, fw = o / (nfu * nfv);
            const int gu = c.b[0].e0 + fu, gv = c.b[1].e0 + fv, gw = c.b[2].e0 + fw;
            const int64_t cp = gu + (int64_t)ax[0].nfun * (gv + (int64_t)ax[1].nfun * gw);
            atomicAdd(&a.diag[i * a.v.ncp + cp], (double)out[o]);
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------ body force
struct ForceArgs {
    WQView<double> v;
    const double *jw;
    double f[3];
    double *F;
};

__global__ void __launch_bounds__(kWQThreads) k_wq_force(ForceArgs a) {
    extern __shared__ __align__(16) unsigned char smraw[];
    double *sm = reinterpret_cast<double *>(smraw);
    const WQAxis *ax = a.v.ax;
    const int NF[3] = {ax[0].NF, ax[1].NF, ax[2].NF};
    const int NQ[3] = {ax[0].NQ, ax[1].NQ, ax[2].NQ};
    const SmemPlan P = smem_plan(NF, NQ, 3, 6);
    BlkCtx c;
    block_ctx(ax, a.v.qoff, blockIdx.x, c);
    int pos[3];
    block_pos(ax, blockIdx.x, pos);
    copy_tiles<double>(ax, a.v.tiles, pos, 6, 0, 6, 0, sm, P, 6);
    __syncthreads();
    const int nfu = c.nf[0], nfv = c.nf[1], nfw = c.nf[2];
    const int nx = nfu * nfv * nfw;
    const int nqb = c.nqb;
    double *H = sm + P.R1;
    double *G = H + 16 * NQ[0] * NQ[1] * NQ[2];
    double *K = G + 9 * NQ[2] * NQ[1] * NF[0];
    double *out = sm + P.X;
    for (int i = 0; i < 3; i++) {
        for (int q = threadIdx.x; q < nqb; q += blockDim.x) {
            for (int ch = 1; ch < 16; ch++) H[ch * nqb + q] = 0.0;
            H[q] = a.f[i] * a.jw[c.qoff + q];
        }
        __syncthreads();
        backward<double>(sm + P.tile[0], sm + P.tile[1], sm + P.tile[2], 2, NF,
                         NQ, c, H, G, K, out);
        for (int o = threadIdx.x; o < nx; o += blockDim.x) {
            const int fu = o % nfu, fv = (o / nfu) % nfv, fw = o / (nfu * nfv);
            const int gu = c.b[0].e0 + fu, gv = c.b[1].e0 + fv, gw = c.b[2].e0 + fw;
            if (clamped(a.v.cmask[i], ax, gu, gv, gw)) continue;
            const int64_t cp = gu + (int64_t)ax[0].nfun * (gv + (int64_t)ax[1].nfun * gw);
            atomicAdd(&a.F[i * a.v.ncp + cp], out[o]);
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------ host setup
static std::vector<BlkInfo> partition(int p, int nel, int QB) {
    auto own = [&](int e) { return e == 0 ? p + 1 : (e == nel - 1 ? p + 2 : 2); };
    std::vector<BlkInfo> out;
    int e = 0, q = 0;
    while (e < nel) {
        BlkInfo b;
        b.e0 = e;
        b.q0 = q;
        b.ne = 0;
        b.nq = 0;
        while (e < nel && (b.ne == 0 || b.nq + own(e) <= QB)) {
            b.nq += own(e);
            b.ne++;
            e++;
        }
        q += b.nq;
        out.push_back(b);
    }
    return out;
}

template <class T>
static void build_tiles(const WQRule1D &R, const std::vector<BlkInfo> &blk,
                        int NF, int NQ, std::vector<T> &t6, std::vector<T> *t4) {
    const int nb = (int)blk.size();
    t6.assign((size_t)nb * 6 * NF * NQ, T(0));
    if (t4) t4->assign((size_t)nb * 4 * NF * NQ, T(0));
    const std::vector<double> *M[6] = {&R.B0, &R.B1, &R.W00, &R.W01, &R.W10, &R.W11};
    for (int b = 0; b < nb; b++) {
        const BlkInfo &B = blk[b];
        const int nf = B.ne + R.p;
        for (int f = 0; f < nf; f++)
            for (int q = 0; q < B.nq; q++) {
                const size_t src = (size_t)(B.e0 + f) * R.nqp + (B.q0 + q);
                for (int m = 0; m < 6; m++)
                    t6[(((size_t)b * 6 + m) * NF + f) * NQ + q] = (T)(*M[m])[src];
                if (t4) {
                    // W00.B0, W01.B1, W10.B0, W11.B1
                    const double P4[4] = {R.W00[src] * R.B0[src], R.W01[src] * R.B1[src],
                                          R.W10[src] * R.B0[src], R.W11[src] * R.B1[src]};
                    for (int m = 0; m < 4; m++)
                        (*t4)[(((size_t)b * 4 + m) * NF + f) * NQ + q] = (T)P4[m];
                }
            }
    }
}

template <class T>
static WQView<T> make_view(const yeti_wq_op *op, const DevBuf *tiles,
                           const DevBuf &coef) {
    WQView<T> v;
    for (int d = 0; d < 3; d++) {
        v.ax[d].p = op->p[d];
        v.ax[d].nfun = op->n[d];
        v.ax[d].nqp = op->nqp[d];
        v.ax[d].nb = (int)op->blk[d].size();
        v.ax[d].NF = op->NF[d];
        v.ax[d].NQ = op->NQ[d];
        v.ax[d].blk = op->blkd[d].as<BlkInfo>();
        v.tiles[d] = tiles[d].as<T>();
        v.cmask[d] = op->cmask[d];
    }
    v.qoff = op->qoff.as<int64_t>();
    v.coef = coef.as<T>();
    v.ncp = op->ncp;
    return v;
}

static size_t smem_bytes(const yeti_wq_op *op, int NC, int ntile, size_t elem) {
    SmemPlan P = smem_plan(op->NF, op->NQ, NC, ntile);
    return (size_t)P.total * elem;
}

static int wq_smem_limit(yeti_ctx *ctx, size_t need) {
    int optin = 0;
    YETI_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx->device));
    YETI_CHECK(need <= (size_t)optin, YETI_EUNSUPPORTED,
               "WQ block needs %zu bytes of shared memory (limit %d)", need, optin);
    return YETI_OK;
}

template <class T>
static int launch_apply(yeti_wq_op *op, const T *u, T *Ku, const int *done,
                        cudaStream_t s) {
    const bool f64 = sizeof(T) == 8;
    ApplyArgs<T> a;
    a.v = make_view<T>(op, f64 ? op->tiles64 : op->tiles32, f64 ? op->coef64 : op->coef32);
    a.u = u;
    a.Ku = Ku;
    a.done = done;
    const size_t smem = smem_bytes(op, 3, 6, sizeof(T));
    YETI_TRY(set_smem_optin((const void *)k_wq_apply<T>, op->ctx->device, smem, "WQ apply block"));
    k_wq_apply<T><<<(unsigned)op->nblocks, kWQThreads, smem, s>>>(a);
    count_launches(1);
    YETI_CUDA(cudaGetLastError());
    return YETI_OK;
}

int wq_apply_dev(yeti_wq_op *op, const void *u, void *Ku, int prec,
                 const int *done, cudaStream_t s) {
    if (op->st.active) {
        if (prec == YETI_PREC_F64)
            return wq_stream_apply<double>(op, (const double *)u, (double *)Ku, done, s);
        return wq_stream_apply<float>(op, (const float *)u, (float *)Ku, done, s);
    }
    if (prec == YETI_PREC_F64)
        return launch_apply<double>(op, (const double *)u, (double *)Ku, done, s);
    return launch_apply<float>(op, (const float *)u, (float *)Ku, done, s);
}

}  // namespace yeti

using namespace yeti;

// ---------------------------------------------------------------- C ABI
YETI_API int yeti_wq_setup(yeti_ctx *ctx, const int32_t p[3],
                           const int32_t nel[3], const double *cps,
                           const double *weights, double E, double nu,
                           const uint8_t dirichlet[18], int prec_mask,
                           yeti_wq_op **out) {
    YETI_CHECK(ctx && p && nel && cps && weights && out, YETI_EINVAL,
               "yeti_wq_setup: NULL argument");
    *out = nullptr;
    YETI_CHECK((prec_mask & (YETI_WQ_F64 | YETI_WQ_F32)) != 0, YETI_EINVAL,
               "yeti_wq_setup: prec_mask selects no precision");
    YETI_CHECK(E > 0 && nu > -1.0 && nu < 0.5, YETI_EINVAL,
               "yeti_wq_setup: E=%g nu=%g", E, nu);
    DeviceGuard guard(ctx->device);
    auto t0 = std::chrono::steady_clock::now();
    std::unique_ptr<yeti_wq_op> op(new yeti_wq_op());
    op->ctx = ctx;
    op->prec_mask = prec_mask;
    op->E = E;
    op->nu = nu;
    const int QB[3] = {8, 8, 4};
    int64_t ncp = 1;
    for (int d = 0; d < 3; d++) {
        YETI_CHECK(p[d] >= 2 && p[d] <= 8 && nel[d] >= 2 && nel[d] <= 100000,
                   YETI_EINVAL, "yeti_wq_setup: p[%d]=%d nel[%d]=%d", d, p[d], d,
                   nel[d]);
        op->p[d] = p[d];
        op->nel[d] = nel[d];
        op->n[d] = p[d] + nel[d];
        op->nqp[d] = wq_npts(p[d], nel[d]);
        ncp *= op->n[d];
    }
    op->ncp = ncp;
    op->ndof = 3 * ncp;
    for (int c = 0; c < 3; c++) {
        op->cmask[c] = 0;
        if (dirichlet)
            for (int f = 0; f < 6; f++)
                if (dirichlet[6 * c + f]) op->cmask[c] |= 1 << f;
    }
    // free dofs
    {
        int64_t nfree = 0;
        for (int c = 0; c < 3; c++)
            for (int w = 0; w < op->n[2]; w++)
                for (int v = 0; v < op->n[1]; v++)
                    for (int u = 0; u < op->n[0]; u++) {
                        const int cm = op->cmask[c];
                        bool cl = ((cm & 1) && u == 0) || ((cm & 2) && u == op->n[0] - 1) ||
                                  ((cm & 4) && v == 0) || ((cm & 8) && v == op->n[1] - 1) ||
                                  ((cm & 16) && w == 0) || ((cm & 32) && w == op->n[2] - 1);
                        nfree += !cl;
                    }
        op->nfree = nfree;
    }
    for (int i = 0; i < ncp; i++)
        YETI_CHECK(weights[i] > 0 && std::isfinite(weights[i]), YETI_EINVAL,
                   "yeti_wq_setup: weight %d is %g", i, weights[i]);
    // 1-D rules, block partition, tiles
    WQRule1D R[3];
    for (int d = 0; d < 3; d++) {
        YETI_CHECK(wq_rule_1d(p[d], nel[d], R[d]) == 0, YETI_EINVAL,
                   "yeti_wq_setup: WQ rule failed");
        op->blk[d] = partition(p[d], nel[d], std::max(QB[d], p[d] + 2));
        int NF = 0, NQ = 0;
        for (auto &b : op->blk[d]) {
            NF = std::max(NF, b.ne + p[d]);
            NQ = std::max(NQ, b.nq);
        }
        op->NF[d] = NF;
        op->NQ[d] = NQ;
        YETI_TRY(upload(ctx, op->blkd[d], op->blk[d].data(), op->blk[d].size()));
        std::vector<double> t6, t4;
        build_tiles<double>(R[d], op->blk[d], NF, NQ, t6, &t4);
        YETI_TRY(upload(ctx, op->tiles64[d], t6.data(), t6.size()));
        std::vector<float> f6;
        build_tiles<float>(R[d], op->blk[d], NF, NQ, f6, nullptr);
        YETI_TRY(upload(ctx, op->tiles32[d], f6.data(), f6.size()));
        YETI_TRY(upload(ctx, op->dtiles[d], t4.data(), t4.size()));
    }
    const int nb[3] = {(int)op->blk[0].size(), (int)op->blk[1].size(), (int)op->blk[2].size()};
    op->nblocks = (int64_t)nb[0] * nb[1] * nb[2];
    YETI_CHECK(op->nblocks < (1LL << 31), YETI_EINVAL, "yeti_wq_setup: patch too large");
    std::vector<int64_t> qoff(op->nblocks + 1, 0);
    for (int64_t b = 0; b < op->nblocks; b++) {
        const int bu = (int)(b % nb[0]), bv = (int)((b / nb[0]) % nb[1]),
                  bw = (int)(b / ((int64_t)nb[0] * nb[1]));
        qoff[b + 1] = qoff[b] + (int64_t)op->blk[0][bu].nq * op->blk[1][bv].nq * op->blk[2][bw].nq;
    }
    op->nqp_total = qoff[op->nblocks];
    YETI_TRY(upload(ctx, op->qoff, qoff.data(), qoff.size()));
    // geometry -> coefficients
    DevBuf dcps, dw, flags;
    YETI_TRY(upload(ctx, dcps, cps, (size_t)3 * ncp));
    YETI_TRY(upload(ctx, dw, weights, (size_t)ncp));
    const int64_t ncoef = op->nqp_total * kWQCoef;
    if (prec_mask & YETI_WQ_F64) YETI_TRY(op->coef64.alloc(ctx, ncoef * sizeof(double)));
    if (prec_mask & YETI_WQ_F32) YETI_TRY(op->coef32.alloc(ctx, ncoef * sizeof(float)));
    YETI_TRY(op->jw.alloc(ctx, op->nqp_total * sizeof(double)));
    YETI_TRY(flags.alloc(ctx, sizeof(int)));
    YETI_CUDA(cudaMemsetAsync(flags.ptr, 0, sizeof(int), ctx->stream));
    SetupArgs sa;
    sa.v = make_view<double>(op.get(), op->tiles64, op->coef64);
    sa.cps = dcps.as<double>();
    sa.wts = dw.as<double>();
    {
        // MDM = MM^T DD MM (wq_assembly.f90:92-109)
        const double lam = (E * nu) / ((1.0 + nu) * (1.0 - 2.0 * nu));
        const double mu = E / (2.0 * (1.0 + nu));
        double DD[6][6] = {};
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) DD[i][j] = lam;
        for (int i = 0; i < 3; i++) DD[i][i] = lam + 2.0 * mu;
        DD[3][3] = DD[4][4] = DD[5][5] = mu;
        double MM[6][9] = {};
        const int nz[9][2] = {{0, 0}, {1, 4}, {2, 8}, {3, 1}, {3, 3}, {4, 5}, {4, 7}, {5, 2}, {5, 6}};
        for (auto &e : nz) MM[e[0]][e[1]] = 1.0;
        for (int a = 0; a < 9; a++)
            for (int b = 0; b < 9; b++) {
                double s = 0.0;
                for (int r = 0; r < 6; r++)
                    for (int t = 0; t < 6; t++) s += MM[r][a] * DD[r][t] * MM[t][b];
                sa.mdm[a * 9 + b] = s;
            }
    }
    sa.coef64 = op->coef64.ptr ? op->coef64.as<double>() : nullptr;
    sa.coef32 = op->coef32.ptr ? op->coef32.as<float>() : nullptr;
    sa.jw = op->jw.as<double>();
    YETI_TRY(op->sdiag.alloc(ctx, (size_t)op->nblocks * 9 * sizeof(double)));
    sa.sdiag = op->sdiag.as<double>();
    sa.flags = flags.as<int>();
    {
        const size_t smem = smem_bytes(op.get(), 4, 2, sizeof(double));
        YETI_TRY(wq_smem_limit(ctx, smem));
        YETI_TRY(set_smem_optin((const void *)k_wq_setup, ctx->device, smem, "WQ setup block"));
        k_wq_setup<<<(unsigned)op->nblocks, kWQThreads, smem, ctx->stream>>>(sa);
        count_launches(1);
        YETI_CUDA(cudaGetLastError());
    }
    int hflags = 0;
    YETI_CUDA(cudaMemcpyAsync(&hflags, flags.ptr, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
    YETI_CUDA(cudaStreamSynchronize(ctx->stream));
    YETI_CHECK(!(hflags & 4) && !((hflags & 1) && (hflags & 2)), YETI_ENUMERIC,
               "yeti_wq_setup: singular or folded geometry (Jacobian sign flags %d)", hflags);
    // diagonal (Jacobi preconditioner)
    YETI_TRY(op->diag.alloc(ctx, op->ndof * sizeof(double)));
    YETI_CUDA(cudaMemsetAsync(op->diag.ptr, 0, op->ndof * sizeof(double), ctx->stream));
    {
        const size_t smem = (prec_mask & YETI_WQ_F64) ? smem_bytes(op.get(), 3, 6, sizeof(double))
                                                      : smem_bytes(op.get(), 3, 6, sizeof(float));
        YETI_TRY(wq_smem_limit(ctx, smem));
        if (prec_mask & YETI_WQ_F64) {
            DiagArgs<double> da;
            da.v = make_view<double>(op.get(), op->tiles64, op->coef64);
            for (int d = 0; d < 3; d++) da.dtiles[d] = op->dtiles[d].as<double>();
            da.diag = op->diag.as<double>();
            YETI_TRY(set_smem_optin((const void *)k_wq_diag<double>, ctx->device, smem, "WQ diagonal block"));
            k_wq_diag<double><<<(unsigned)op->nblocks, kWQThreads, smem, ctx->stream>>>(da);
            count_launches(1);
        } else {
            // FP32 coefficients only: diagonal from FP64 product tiles cast
            std::vector<std::vector<float>> t4f(3);
            DevBuf dt[3];
            for (int d = 0; d < 3; d++) {
                std::vector<double> t6, t4;
                build_tiles<double>(R[d], op->blk[d], op->NF[d], op->NQ[d], t6, &t4);
                t4f[d].assign(t4.begin(), t4.end());
                YETI_TRY(upload(ctx, dt[d], t4f[d].data(), t4f[d].size()));
            }
            DiagArgs<float> da;
            da.v = make_view<float>(op.get(), op->tiles32, op->coef32);
            for (int d = 0; d < 3; d++) da.dtiles[d] = dt[d].as<float>();
            da.diag = op->diag.as<double>();
            YETI_TRY(set_smem_optin((const void *)k_wq_diag<float>, ctx->device, smem, "WQ diagonal block"));
            k_wq_diag<float><<<(unsigned)op->nblocks, kWQThreads, smem, ctx->stream>>>(da);
            count_launches(1);
            YETI_CUDA(cudaStreamSynchronize(ctx->stream));
        }
        YETI_CUDA(cudaGetLastError());
    }
    YETI_CUDA(cudaStreamSynchronize(ctx->stream));
    // the streaming apply (degrees 2..5) takes the coefficients in its own layout
    if (wq_stream_supported(op.get())) {
        YETI_TRY(wq_stream_setup(op.get(), R));
        YETI_TRY(wq_stream_permute(op.get()));
    }
    op->setup_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    op->bytes_data = (op->coef64.bytes + op->coef32.bytes);
    *out = op.release();
    return YETI_OK;
}

YETI_API int yeti_wq_destroy(yeti_wq_op *op) {
    if (!op) return YETI_OK;
    DeviceGuard guard(op->ctx->device);
    cudaStreamSynchronize(op->ctx->stream);
    delete op;
    return YETI_OK;
}

YETI_API int yeti_wq_info(const yeti_wq_op *op, int64_t *ncp, int64_t *ndof,
                          int64_t *nfree, int64_t *nqp, int64_t *bytes) {
    YETI_CHECK(op, YETI_EINVAL, "yeti_wq_info: NULL op");
    if (ncp) *ncp = op->ncp;
    if (ndof) *ndof = op->ndof;
    if (nfree) *nfree = op->nfree;
    if (nqp) *nqp = op->nqp_total;
    if (bytes) *bytes = op->bytes_data;
    return YETI_OK;
}

YETI_API int yeti_wq_apply(yeti_wq_op *op, const void *u, void *Ku, int prec,
                           int mem) {
    YETI_CHECK(op && u && Ku, YETI_EINVAL, "yeti_wq_apply: NULL argument");
    YETI_CHECK(prec == YETI_PREC_F64 || prec == YETI_PREC_F32, YETI_EINVAL,
               "yeti_wq_apply: bad precision %d", prec);
    YETI_CHECK(prec == YETI_PREC_F64 ? op->coef64.ptr != nullptr : op->coef32.ptr != nullptr,
               YETI_EINVAL, "yeti_wq_apply: operator was set up without that precision");
    DeviceGuard guard(op->ctx->device);
    cudaStream_t s = op->ctx->stream;
    const size_t es = prec == YETI_PREC_F64 ? 8 : 4;
    const size_t nb = op->ndof * es;
    DevBuf du, dk;
    const void *uu = u;
    void *kk = Ku;
    if (mem == YETI_MEM_HOST) {
        YETI_TRY(du.alloc(op->ctx, nb));
        YETI_TRY(dk.alloc(op->ctx, nb));
        YETI_CUDA(cudaMemcpyAsync(du.ptr, u, nb, cudaMemcpyHostToDevice, s));
        uu = du.ptr;
        kk = dk.ptr;
    }
    YETI_CUDA(cudaMemsetAsync(kk, 0, nb, s));
    YETI_TRY(wq_apply_dev(op, uu, kk, prec, nullptr, s));
    if (mem == YETI_MEM_HOST) {
        YETI_CUDA(cudaMemcpyAsync(Ku, kk, nb, cudaMemcpyDeviceToHost, s));
        YETI_CUDA(cudaStreamSynchronize(s));
        YETI_TRY(wq_stream_check(op));
    }
    return YETI_OK;
}

YETI_API int yeti_wq_set_wait_limit(yeti_wq_op *op, int tries) {
    YETI_CHECK(op, YETI_EINVAL, "yeti_wq_set_wait_limit: NULL op");
    op->st.wait_tries = tries < 0 ? (1 << 16) : tries;
    return YETI_OK;
}

YETI_API int yeti_wq_diag(yeti_wq_op *op, double *d, int mem) {
    YETI_CHECK(op && d, YETI_EINVAL, "yeti_wq_diag: NULL argument");
    DeviceGuard guard(op->ctx->device);
    // clamped dofs report 1 (they are not part of the system)
    std::vector<double> h(op->ndof);
    YETI_CUDA(cudaMemcpyAsync(h.data(), op->diag.ptr, op->ndof * sizeof(double),
                              cudaMemcpyDeviceToHost, op->ctx->stream));
    YETI_CUDA(cudaStreamSynchronize(op->ctx->stream));
    for (int c = 0; c < 3; c++)
        for (int w = 0; w < op->n[2]; w++)
            for (int v = 0; v < op->n[1]; v++)
                for (int u = 0; u < op->n[0]; u++) {
                    const int cm = op->cmask[c];
                    bool cl = ((cm & 1) && u == 0) || ((cm & 2) && u == op->n[0] - 1) ||
                              ((cm & 4) && v == 0) || ((cm & 8) && v == op->n[1] - 1) ||
                              ((cm & 16) && w == 0) || ((cm & 32) && w == op->n[2] - 1);
                    if (cl) h[c * op->ncp + u + (int64_t)op->n[0] * (v + (int64_t)op->n[1] * w)] = 1.0;
                }
    if (mem == YETI_MEM_HOST) {
        std::copy(h.begin(), h.end(), d);
    } else {
        YETI_CUDA(cudaMemcpyAsync(d, h.data(), op->ndof * sizeof(double),
                                  cudaMemcpyHostToDevice, op->ctx->stream));
        YETI_CUDA(cudaStreamSynchronize(op->ctx->stream));
    }
    return YETI_OK;
}

YETI_API int yeti_wq_body_force(yeti_wq_op *op, const double f[3], double *F,
                                int mem) {
    YETI_CHECK(op && f && F, YETI_EINVAL, "yeti_wq_body_force: NULL argument");
    YETI_CHECK(op->coef64.ptr || op->tiles64[0].ptr, YETI_EINVAL, "yeti_wq_body_force: no FP64 data");
    DeviceGuard guard(op->ctx->device);
    cudaStream_t s = op->ctx->stream;
    DevBuf dF;
    double *FF = F;
    if (mem == YETI_MEM_HOST) {
        YETI_TRY(dF.alloc(op->ctx, op->ndof * sizeof(double)));
        FF = dF.as<double>();
    }
    YETI_CUDA(cudaMemsetAsync(FF, 0, op->ndof * sizeof(double), s));
    ForceArgs a;
    a.v = make_view<double>(op, op->tiles64, op->coef64);
    a.jw = op->jw.as<double>();
    for (int d = 0; d < 3; d++) a.f[d] = f[d];
    a.F = FF;
    const size_t smem = smem_bytes(op, 3, 6, sizeof(double));
    YETI_TRY(wq_smem_limit(op->ctx, smem));
    YETI_TRY(set_smem_optin((const void *)k_wq_force, op->ctx->device, smem, "WQ force block"));
    k_wq_force<<<(unsigned)op->nblocks, kWQThreads, smem, s>>>(a);
    count_launches(1);
    YETI_CUDA(cudaGetLastError());
    if (mem == YETI_MEM_HOST) {
        YETI_CUDA(cudaMemcpyAsync(F, FF, op->ndof * sizeof(double), cudaMemcpyDeviceToHost, s));
    }
    YETI_CUDA(cudaStreamSynchronize(s));
    return YETI_OK;
}
