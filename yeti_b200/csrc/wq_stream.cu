// Streaming WQ apply: Ku += K u for degrees 2..5, the kernel every Krylov
// iteration of the WQ solve runs (mf_wq_get_ku_3d, mf_wq_solver.f90:284-544,
// generalised to 3x3 elastic blocks).
//
// Work decomposition
// ------------------
// The (u, v) point grid is cut into tiles of at most 16 x 16 points made of
// whole elements; a CTA takes a tile and a range of elements along w and
// marches through the w point planes of that range.  Every WQ point belongs
// to one element and, in each direction, its B0/B1/W** rows are non-zero for
// the p+1 functions elem(q)..elem(q)+p only (checked on the host), so every
// 1-D contraction is a band of width p+1:
//
//   A  forward w : Y_t[c][fv][fu] = sum_m Bt_w(qw,m) X[c][fv][fu][e+m]
//                  (one thread per (c, fv, fu) column; X for functions
//                  e..e+p lives in a register ring that advances with e)
//   B  forward v : Z_s[c][qv][fu]  (s: B0v.Y0, B1v.Y0, B0v.Y1)
//   C1 forward u : F[l][j][qv][qu] = d u_j / d xi_l   (one thread per row,
//                  register ring of p+1 Z values along u)
//   C2 point     : h[i][k][l] = sum_j S[(i,k),(j,l)] F[l][j] with the 45
//                  streamed coefficients of the point (the HBM stream)
//   C3 backward u: G[i][k][l][qv][fu] with weights W^{[k==u][l==u]}
//                  (one thread per (row, i, k), rings along u)
//   D  backward v: K[i][k][lw][fv][fu], channels merged on (l == w)
//   E  backward w: accumulation into a register ring of output planes
//                  e..e+p; plane e is complete after element e and is added
//                  to Ku (atomics: tiles overlap on the p halo functions,
//                  element ranges overlap on p planes)
//
// Shared memory holds one plane's intermediates in two regions whose
// lifetimes alternate (R1: Y, F, G; R2: Z, h, K), so every stage reads one
// region and writes the other.  While a plane is processed, the next plane's
// coefficient block (contiguous, 256-byte aligned) is prefetched into L2.
#include <algorithm>
#include <numeric>

#include "wq.cuh"

namespace yeti {

namespace {

constexpr int kTQ = 16;          // max points of a tile per direction
constexpr int kThreads = 256;    // one thread per point of a plane tile
constexpr int kQP = 17;          // padded pitch of point-indexed rows

constexpr int cmax(int a, int b) { return a > b ? a : b; }

template <int P>
struct Dims {
    static constexpr int PB = P + 1;
    static constexpr int NFM = kTQ / 2 + P;   // max functions of a tile
    static constexpr int Y = 2 * 3 * NFM * NFM;
    static constexpr int F = 9 * kTQ * kQP;
    static constexpr int G = 27 * kTQ * NFM;
    static constexpr int Z = 9 * kTQ * NFM;
    static constexpr int H = 27 * kTQ * kQP;
    static constexpr int K = 18 * NFM * NFM;
    static constexpr int R1 = cmax(Y, cmax(F, G));
    static constexpr int R2 = cmax(Z, cmax(H, K));
    static constexpr int TAB = kTQ * 6 * PB;
    static constexpr int NCOL = 3 * NFM * NFM;
    static constexpr int CPT = (NCOL + kThreads - 1) / kThreads;
    template <class T>
    static constexpr size_t smem_bytes() {
        return (size_t)(R1 + R2 + 2 * TAB) * sizeof(T) + 2 * kTQ * sizeof(int);
    }
};

__device__ __forceinline__ void prefetch_l2(const void *p) {
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

__device__ __forceinline__ float ld_stream(const float *p) { return __ldcs(p); }
__device__ __forceinline__ double ld_stream(const double *p) { return __ldcs(p); }

}  // namespace

template <class T>
struct StreamArgs {
    const T *u;
    T *Ku;
    const int *done;
    const T *coef;
    const int64_t *tile_off;   // first coefficient of a tile
    const int *tile_pstride;   // coefficients per w plane of a tile (padded)
    const int *tq0[2];         // first point of a u / v tile
    const int *tnq[2];         // points of a u / v tile
    int ntile[2];
    const int *elem[3];        // element owning each point
    const T *band[3];          // [nqp][6][p+1]: B0 B1 W00 W01 W10 W11
    const int *wq0;            // first w point of each element (nel_w + 1)
    int nqw;                   // w points
    const int4 *seg;           // (tile, e_begin, e_end, -)
    const int *cta_seg;        // segments of a CTA
    int nfun[3];
    int64_t ncp;
    int cmask[3];
};

template <class T, int P>
__global__ void __launch_bounds__(kThreads, 2) k_wq_apply_stream(StreamArgs<T> a) {
    using D = Dims<P>;
    constexpr int PB = D::PB, NFM = D::NFM, CPT = D::CPT;
    if (a.done && *a.done) return;
    extern __shared__ __align__(16) unsigned char smraw[];
    T *R1 = reinterpret_cast<T *>(smraw);
    T *R2 = R1 + D::R1;
    T *tabu = R2 + D::R2;
    T *tabv = tabu + D::TAB;
    int *relu = reinterpret_cast<int *>(tabv + D::TAB);
    int *relv = relu + kTQ;
    const int tid = threadIdx.x;
    const int64_t plane = (int64_t)a.nfun[0] * a.nfun[1];

    for (int si = a.cta_seg[blockIdx.x]; si < a.cta_seg[blockIdx.x + 1]; si++) {
        const int4 sg = a.seg[si];
        const int tu = sg.x % a.ntile[0], tv = sg.x / a.ntile[0];
        const int qu0 = a.tq0[0][tu], nqu = a.tnq[0][tu];
        const int qv0 = a.tq0[1][tv], nqv = a.tnq[1][tv];
        const int fu0 = a.elem[0][qu0], fv0 = a.elem[1][qv0];
        const int nfu = a.elem[0][qu0 + nqu - 1] + PB - fu0;
        const int nfv = a.elem[1][qv0 + nqv - 1] + PB - fv0;
        const int npts = nqu * nqv;
        const T *coef_t = a.coef + a.tile_off[sg.x];
        const int pstride = a.tile_pstride[sg.x];
        const int pbytes = npts * kWQCoef * (int)sizeof(T);

        __syncthreads();   // the previous segment is done with the tables
        for (int i = tid; i < kTQ * 6 * PB; i += kThreads) {
            const int q = i / (6 * PB), r = i - q * (6 * PB);
            tabu[i] = q < nqu ? a.band[0][(size_t)(qu0 + q) * 6 * PB + r] : T(0);
            tabv[i] = q < nqv ? a.band[1][(size_t)(qv0 + q) * 6 * PB + r] : T(0);
        }
        if (tid < kTQ) {
            relu[tid] = tid < nqu ? a.elem[0][qu0 + tid] - fu0 : 0;
            relv[tid] = tid < nqv ? a.elem[1][qv0 + tid] - fv0 : 0;
        }

        // columns (c, fv, fu) of this thread: stages A and E
        const int ncol = 3 * nfv * nfu;
        int64_t cbase[CPT];
        int cinfo[CPT];   // bit 0..1: component; bit 2: active; bits 3..: fv*NFM+fu
        bool cclamp_uv[CPT];
        T x[CPT][PB], acc[CPT][PB];
#pragma unroll
        for (int cc = 0; cc < CPT; cc++) {
            const int col = tid + cc * kThreads;
            const bool act = col < ncol;
            int c = 0, fv = 0, fu = 0;
            if (act) {
                c = col / (nfv * nfu);
                const int r = col - c * nfv * nfu;
                fv = r / nfu;
                fu = r - fv * nfu;
            }
            const int gu = fu0 + fu, gv = fv0 + fv;
            const int cm = a.cmask[c];
            cbase[cc] = c * a.ncp + gu + (int64_t)a.nfun[0] * gv;
            cinfo[cc] = c | (act ? 4 : 0) | ((fv * NFM + fu) << 3);
            cclamp_uv[cc] = ((cm & 1) && gu == 0) || ((cm & 2) && gu == a.nfun[0] - 1) ||
                            ((cm & 4) && gv == 0) || ((cm & 8) && gv == a.nfun[1] - 1);
#pragma unroll
            for (int m = 0; m < PB; m++) {
                x[cc][m] = T(0);
                acc[cc][m] = T(0);
            }
        }
        auto clamped_w = [&](int cc, int fw) {
            const int cm = a.cmask[cinfo[cc] & 3];
            return cclamp_uv[cc] || ((cm & 16) && fw == 0) || ((cm & 32) && fw == a.nfun[2] - 1);
        };
        auto load_x = [&](int cc, int fw) -> T {
            if (!(cinfo[cc] & 4) || clamped_w(cc, fw)) return T(0);
            return a.u[cbase[cc] + plane * fw];
        };
        auto retire = [&](int cc, int fw, T v) {
            if ((cinfo[cc] & 4) && !clamped_w(cc, fw)) atomicAdd(&a.Ku[cbase[cc] + plane * fw], v);
        };
#pragma unroll
        for (int cc = 0; cc < CPT; cc++)
#pragma unroll
            for (int m = 0; m < P; m++) x[cc][m] = load_x(cc, sg.y + m);
        {
            const char *p0 = reinterpret_cast<const char *>(coef_t + (int64_t)a.wq0[sg.y] * pstride);
            for (int off = tid * 128; off < pbytes; off += kThreads * 128) prefetch_l2(p0 + off);
        }

        for (int e = sg.y; e < sg.z; e++) {
#pragma unroll
            for (int cc = 0; cc < CPT; cc++) {
                x[cc][P] = load_x(cc, e + P);
                acc[cc][P] = T(0);
            }
            const int qw_end = a.wq0[e + 1];
            for (int qw = a.wq0[e]; qw < qw_end; qw++) {
                const T *bw = a.band[2] + (size_t)qw * 6 * PB;
                if (qw + 1 < a.nqw) {
                    const char *pn = reinterpret_cast<const char *>(coef_t + (int64_t)(qw + 1) * pstride);
                    for (int off = tid * 128; off < pbytes; off += kThreads * 128) prefetch_l2(pn + off);
                }
                // ---- A: forward w
                {
                    T b0[PB], b1[PB];
#pragma unroll
                    for (int m = 0; m < PB; m++) {
                        b0[m] = bw[m];
                        b1[m] = bw[PB + m];
                    }
#pragma unroll
                    for (int cc = 0; cc < CPT; cc++) {
                        if (!(cinfo[cc] & 4)) continue;
                        T y0 = 0, y1 = 0;
#pragma unroll
                        for (int m = 0; m < PB; m++) {
                            y0 += b0[m] * x[cc][m];
                            y1 += b1[m] * x[cc][m];
                        }
                        const int c = cinfo[cc] & 3, k = cinfo[cc] >> 3;
                        R1[c * NFM * NFM + k] = y0;
                        R1[(3 + c) * NFM * NFM + k] = y1;
                    }
                }
                __syncthreads();
                // ---- B: forward v, thread (qv, fu)
                {
                    const int qv = tid >> 4, fu = tid & 15;
                    if (qv < nqv && fu < nfu) {
                        const int rv = relv[qv];
                        const T *w0 = tabv + (qv * 6 + 0) * PB;
                        const T *w1 = tabv + (qv * 6 + 1) * PB;
                        T b0[PB], b1[PB];
#pragma unroll
                        for (int m = 0; m < PB; m++) {
                            b0[m] = w0[m];
                            b1[m] = w1[m];
                        }
#pragma unroll
                        for (int c = 0; c < 3; c++) {
                            const T *y0 = R1 + (c * NFM + rv) * NFM + fu;
                            const T *y1 = R1 + ((3 + c) * NFM + rv) * NFM + fu;
                            T z0 = 0, z1 = 0, z2 = 0;
#pragma unroll
                            for (int m = 0; m < PB; m++) {
                                const T a0 = y0[m * NFM], a1 = y1[m * NFM];
                                z0 += b0[m] * a0;
                                z1 += b1[m] * a0;
                                z2 += b0[m] * a1;
                            }
                            R2[((0 * 3 + c) * kTQ + qv) * NFM + fu] = z0;
                            R2[((1 * 3 + c) * kTQ + qv) * NFM + fu] = z1;
                            R2[((2 * 3 + c) * kTQ + qv) * NFM + fu] = z2;
                        }
                    }
                }
                __syncthreads();
                // ---- C1: forward u, thread (row qv, s, j), ring along u
                if (tid < 9 * kTQ) {
                    const int qv = tid & 15, sj = tid >> 4;
                    if (qv < nqv) {
                        const int kind = sj < 3 ? 1 : 0;   // s = 0 takes d/du
                        const T *zr = R2 + (sj * kTQ + qv) * NFM;
                        T *fr = R1 + (sj * kTQ + qv) * kQP;
                        T z[PB];
#pragma unroll
                        for (int m = 0; m < PB; m++) z[m] = zr[m];
                        int cur = 0;
                        for (int qu = 0; qu < nqu; qu++) {
                            const int r = relu[qu];
                            if (r != cur) {
#pragma unroll
                                for (int m = 0; m < P; m++) z[m] = z[m + 1];
                                z[P] = zr[r + P];
                                cur = r;
                            }
                            const T *w = tabu + (qu * 6 + kind) * PB;
                            T v = 0;
#pragma unroll
                            for (int m = 0; m < PB; m++) v += w[m] * z[m];
                            fr[qu] = v;
                        }
                    }
                }
                __syncthreads();
                // ---- C2: pointwise coefficients, thread (qv, qu)
                {
                    const int qv = tid >> 4, qu = tid & 15;
                    if (qv < nqv && qu < nqu) {
                        T f[3][3];
#pragma unroll
                        for (int l = 0; l < 3; l++)
#pragma unroll
                            for (int j = 0; j < 3; j++) f[l][j] = R1[((l * 3 + j) * kTQ + qv) * kQP + qu];
                        const T *cp = coef_t + (int64_t)qw * pstride + qv * nqu + qu;
                        T h[27];
#pragma unroll
                        for (int ch = 0; ch < 27; ch++) h[ch] = T(0);
#pragma unroll
                        for (int I = 0; I < 9; I++) {
#pragma unroll
                            for (int J = I; J < 9; J++) {
                                const T s = ld_stream(cp + sym9(I, J) * npts);
                                const int i = I / 3, k = I % 3, j = J / 3, l = J % 3;
                                h[(i * 3 + k) * 3 + l] += s * f[l][j];
                                if (I != J) h[(j * 3 + l) * 3 + k] += s * f[k][i];
                            }
                        }
#pragma unroll
                        for (int ch = 0; ch < 27; ch++) R2[(ch * kTQ + qv) * kQP + qu] = h[ch];
                    }
                }
                __syncthreads();
                // ---- C3: backward u, thread (row qv, i, k), rings along u
                if (tid < 9 * kTQ) {
                    const int qv = tid & 15, ik = tid >> 4;
                    if (qv < nqv) {
                        const int ka = 2 + 2 * (ik % 3 == 0);   // W_{[k==u], 0}
                        const T *h0 = R2 + ((ik * 3 + 0) * kTQ + qv) * kQP;
                        const T *h1 = R2 + ((ik * 3 + 1) * kTQ + qv) * kQP;
                        const T *h2 = R2 + ((ik * 3 + 2) * kTQ + qv) * kQP;
                        T *g0 = R1 + ((ik * 3 + 0) * kTQ + qv) * NFM;
                        T *g1 = R1 + ((ik * 3 + 1) * kTQ + qv) * NFM;
                        T *g2 = R1 + ((ik * 3 + 2) * kTQ + qv) * NFM;
                        T a0[PB], a1[PB], a2[PB];
#pragma unroll
                        for (int m = 0; m < PB; m++) a0[m] = a1[m] = a2[m] = T(0);
                        int cur = 0;
                        for (int qu = 0; qu < nqu; qu++) {
                            const int r = relu[qu];
                            if (r != cur) {
                                g0[cur] = a0[0];
                                g1[cur] = a1[0];
                                g2[cur] = a2[0];
#pragma unroll
                                for (int m = 0; m < P; m++) {
                                    a0[m] = a0[m + 1];
                                    a1[m] = a1[m + 1];
                                    a2[m] = a2[m + 1];
                                }
                                a0[P] = a1[P] = a2[P] = T(0);
                                cur = r;
                            }
                            const T *wa = tabu + (qu * 6 + ka + 1) * PB;   // trial d/du
                            const T *wb = tabu + (qu * 6 + ka) * PB;       // trial d/dv, d/dw
                            const T x0 = h0[qu], x1 = h1[qu], x2 = h2[qu];
#pragma unroll
                            for (int m = 0; m < PB; m++) {
                                a0[m] += wa[m] * x0;
                                a1[m] += wb[m] * x1;
                                a2[m] += wb[m] * x2;
                            }
                        }
#pragma unroll
                        for (int m = 0; m < PB; m++) {
                            g0[cur + m] = a0[m];
                            g1[cur + m] = a1[m];
                            g2[cur + m] = a2[m];
                        }
                    }
                }
                __syncthreads();
                // ---- D: backward v, thread (fu, i, k), rings along v
                if (tid < 9 * kTQ) {
                    const int fu = tid & 15, ik = tid >> 4;
                    if (fu < nfu) {
                        const int ka = 2 + 2 * (ik % 3 == 1);   // W_{[k==v], 0}
                        const T *g0 = R1 + ((ik * 3 + 0) * kTQ) * NFM + fu;
                        const T *g1 = R1 + ((ik * 3 + 1) * kTQ) * NFM + fu;
                        const T *g2 = R1 + ((ik * 3 + 2) * kTQ) * NFM + fu;
                        T *k0 = R2 + ((ik * 2 + 0) * NFM) * NFM + fu;
                        T *k1 = R2 + ((ik * 2 + 1) * NFM) * NFM + fu;
                        T A0[PB], A1[PB];
#pragma unroll
                        for (int m = 0; m < PB; m++) A0[m] = A1[m] = T(0);
                        int cur = 0;
                        for (int qv = 0; qv < nqv; qv++) {
                            const int r = relv[qv];
                            if (r != cur) {
                                k0[cur * NFM] = A0[0];
                                k1[cur * NFM] = A1[0];
#pragma unroll
                                for (int m = 0; m < P; m++) {
                                    A0[m] = A0[m + 1];
                                    A1[m] = A1[m + 1];
                                }
                                A0[P] = A1[P] = T(0);
                                cur = r;
                            }
                            const T *wa = tabv + (qv * 6 + ka) * PB;       // trial d/du, d/dw
                            const T *wb = tabv + (qv * 6 + ka + 1) * PB;   // trial d/dv
                            const T x0 = g0[qv * NFM], x1 = g1[qv * NFM], x2 = g2[qv * NFM];
#pragma unroll
                            for (int m = 0; m < PB; m++) {
                                A0[m] += wa[m] * x0 + wb[m] * x1;
                                A1[m] += wa[m] * x2;
                            }
                        }
#pragma unroll
                        for (int m = 0; m < PB; m++) {
                            k0[(cur + m) * NFM] = A0[m];
                            k1[(cur + m) * NFM] = A1[m];
                        }
                    }
                }
                __syncthreads();
                // ---- E: backward w into the register ring of output planes
                {
                    T w00[PB], w01[PB], w10[PB], w11[PB];
#pragma unroll
                    for (int m = 0; m < PB; m++) {
                        w00[m] = bw[2 * PB + m];
                        w01[m] = bw[3 * PB + m];
                        w10[m] = bw[4 * PB + m];
                        w11[m] = bw[5 * PB + m];
                    }
#pragma unroll
                    for (int cc = 0; cc < CPT; cc++) {
                        if (!(cinfo[cc] & 4)) continue;
                        const int i = cinfo[cc] & 3, kidx = cinfo[cc] >> 3;
                        const T *kb = R2 + (i * 6) * NFM * NFM + kidx;
                        const T s00 = kb[0 * NFM * NFM] + kb[2 * NFM * NFM];
                        const T s01 = kb[1 * NFM * NFM] + kb[3 * NFM * NFM];
                        const T s10 = kb[4 * NFM * NFM];
                        const T s11 = kb[5 * NFM * NFM];
#pragma unroll
                        for (int m = 0; m < PB; m++)
                            acc[cc][m] += w00[m] * s00 + w01[m] * s01 + w10[m] * s10 + w11[m] * s11;
                    }
                }
                // no barrier: the next plane's stage A writes R1, last read
                // by stage D before the barrier above
            }
            // output plane e is complete for this element range
#pragma unroll
            for (int cc = 0; cc < CPT; cc++) {
                retire(cc, e, acc[cc][0]);
#pragma unroll
                for (int m = 0; m < P; m++) {
                    x[cc][m] = x[cc][m + 1];
                    acc[cc][m] = acc[cc][m + 1];
                }
            }
        }
        // partial sums of the planes after the range
#pragma unroll
        for (int cc = 0; cc < CPT; cc++)
#pragma unroll
            for (int m = 0; m < P; m++) retire(cc, sg.z + m, acc[cc][m]);
    }
}

// ------------------------------------------------------------------ host
// Tiles of whole elements with at most kTQ points, balanced in size.
static void make_tiles(const std::vector<int> &elem_q0, int nel, std::vector<int> &q0,
                       std::vector<int> &nq) {
    const int nqp = elem_q0[nel];
    const int nt0 = (nqp + kTQ - 1) / kTQ;
    q0.clear();
    nq.clear();
    int e = 0, t = 0;
    while (e < nel) {
        const int start = elem_q0[e];
        // aim for an even split of the remaining points over the remaining tiles
        const int left_tiles = std::max(1, nt0 - t);
        const int target = (nqp - start + left_tiles - 1) / left_tiles;
        int end = e;
        while (end < nel && elem_q0[end + 1] - start <= kTQ &&
               (end == e || elem_q0[end] - start < target))
            end++;
        q0.push_back(start);
        nq.push_back(elem_q0[end] - start);
        e = end;
        t++;
    }
}

template <class T>
static int upload_vec(yeti_ctx *ctx, DevBuf &b, const std::vector<T> &v) {
    return upload(ctx, b, v.data(), v.size());
}

// Copy the coefficients from the element-block layout of the setup kernels
// into the tile/plane layout of the streaming kernel.
template <class T>
__global__ void k_wq_stream_permute(const T *src, T *dst, const int64_t *qoff1,
                                    const int *blk1[3], const int *loc1[3],
                                    const int *nq1[3], int nb1u, int nb1v,
                                    const int *tq0u, const int *tnqu, const int *tq0v,
                                    const int *tnqv, int ntu, const int64_t *tile_off,
                                    const int *tile_pstride, int nqu_all, int nqv_all,
                                    int nqw_all) {
    const int64_t n = (int64_t)nqu_all * nqv_all * nqw_all;
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < n;
         g += (int64_t)gridDim.x * blockDim.x) {
        const int qu = (int)(g % nqu_all);
        const int qv = (int)((g / nqu_all) % nqv_all);
        const int qw = (int)(g / ((int64_t)nqu_all * nqv_all));
        // source: element block of the setup layout
        const int bu = blk1[0][qu], bv = blk1[1][qv], bw = blk1[2][qw];
        const int64_t b = bu + (int64_t)nb1u * (bv + (int64_t)nb1v * bw);
        const int nu1 = nq1[0][bu], nv1 = nq1[1][bv], nw1 = nq1[2][bw];
        const int64_t nqb = (int64_t)nu1 * nv1 * nw1;
        const int64_t sbase = qoff1[b] * kWQCoef +
                              (loc1[2][qw] * (int64_t)nv1 + loc1[1][qv]) * nu1 + loc1[0][qu];
        // destination: tile (tu, tv), plane qw
        int tu = 0, tv = 0;
        while (tq0u[tu] + tnqu[tu] <= qu) tu++;
        while (tq0v[tv] + tnqv[tv] <= qv) tv++;
        const int t = tu + ntu * tv;
        const int nqt = tnqu[tu] * tnqv[tv];
        const int64_t dbase = tile_off[t] + (int64_t)qw * tile_pstride[t] +
                              (qv - tq0v[tv]) * tnqu[tu] + (qu - tq0u[tu]);
        for (int e = 0; e < kWQCoef; e++) dst[dbase + (int64_t)e * nqt] = src[sbase + e * nqb];
    }
}

template <class T, int P>
static int stream_attr(yeti_wq_op *op, int which) {
    const size_t smem = Dims<P>::template smem_bytes<T>();
    YETI_CUDA(cudaFuncSetAttribute(k_wq_apply_stream<T, P>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    YETI_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_wq_apply_stream<T, P>,
                                                            kThreads, smem));
    YETI_CHECK(per_sm >= 1, YETI_EUNSUPPORTED, "WQ streaming kernel does not fit on an SM");
    op->st.smem[which] = smem;
    op->st.per_sm[which] = per_sm;
    return YETI_OK;
}

static int stream_prepare_kernels(yeti_wq_op *op) {
    const int P = op->p[0];
    int rc = YETI_OK;
    switch (P) {
#define YETI_CASE(PP)                                                  \
    case PP:                                                           \
        rc = stream_attr<double, PP>(op, 0);                           \
        if (rc == YETI_OK) rc = stream_attr<float, PP>(op, 1);         \
        break;
        YETI_CASE(2)
        YETI_CASE(3)
        YETI_CASE(4)
        YETI_CASE(5)
#undef YETI_CASE
        default:
            rc = YETI_EUNSUPPORTED;
    }
    return rc;
}

bool wq_stream_supported(const yeti_wq_op *op) {
    return op->p[0] == op->p[1] && op->p[1] == op->p[2] && op->p[0] >= 2 && op->p[0] <= 5;
}

int wq_stream_setup(yeti_wq_op *op, const WQRule1D R[3]) {
    yeti_ctx *ctx = op->ctx;
    WQStreamPlan &st = op->st;
    const int P = op->p[0], PB = P + 1;
    std::vector<int> elem_q0[3];
    for (int d = 0; d < 3; d++) {
        const int nel = op->nel[d], nq = op->nqp[d];
        // element ownership of the points (first element p+1 points, last
        // p+2, the others 2: the WQ rule's point layout)
        elem_q0[d].assign(nel + 1, 0);
        for (int e = 0; e < nel; e++) {
            const int own = e == 0 ? P + 1 : (e == nel - 1 ? P + 2 : 2);
            elem_q0[d][e + 1] = elem_q0[d][e] + own;
        }
        YETI_CHECK(elem_q0[d][nel] == nq, YETI_EINVAL, "WQ streaming: point count mismatch");
        std::vector<int> elem(nq);
        for (int e = 0; e < nel; e++)
            for (int q = elem_q0[d][e]; q < elem_q0[d][e + 1]; q++) elem[q] = e;
        // banded 1-D tables; every non-zero must lie in the band
        const std::vector<double> *M[6] = {&R[d].B0, &R[d].B1, &R[d].W00,
                                           &R[d].W01, &R[d].W10, &R[d].W11};
        std::vector<double> band((size_t)nq * 6 * PB, 0.0);
        for (int q = 0; q < nq; q++)
            for (int k = 0; k < 6; k++)
                for (int f = 0; f < R[d].nfun; f++) {
                    const double v = (*M[k])[(size_t)f * nq + q];
                    const int m = f - elem[q];
                    if (m >= 0 && m <= P) band[((size_t)q * 6 + k) * PB + m] = v;
                    else YETI_CHECK(v == 0.0, YETI_EUNSUPPORTED,
                                    "WQ streaming: rule entry outside the band (dir %d, f %d, q %d)",
                                    d, f, q);
                }
        std::vector<float> bandf(band.begin(), band.end());
        YETI_TRY(upload_vec(ctx, st.elem[d], elem));
        YETI_TRY(upload_vec(ctx, st.band64[d], band));
        YETI_TRY(upload_vec(ctx, st.band32[d], bandf));
    }
    YETI_TRY(upload_vec(ctx, st.wq0, elem_q0[2]));
    std::vector<int> tq0[2], tnq[2];
    for (int d = 0; d < 2; d++) {
        make_tiles(elem_q0[d], op->nel[d], tq0[d], tnq[d]);
        st.ntile[d] = (int)tq0[d].size();
        YETI_TRY(upload_vec(ctx, st.tq0[d], tq0[d]));
        YETI_TRY(upload_vec(ctx, st.tnq[d], tnq[d]));
    }
    // coefficient layout: tile-major, then w plane, then entry, then point
    const int ntiles = st.ntile[0] * st.ntile[1];
    const int nqw = op->nqp[2];
    std::vector<int64_t> toff(ntiles + 1, 0);
    std::vector<int> pstride(ntiles);
    for (int t = 0; t < ntiles; t++) {
        const int tu = t % st.ntile[0], tv = t / st.ntile[0];
        const int npts = tnq[0][tu] * tnq[1][tv];
        pstride[t] = (kWQCoef * npts + 63) / 64 * 64;
        toff[t + 1] = toff[t] + (int64_t)nqw * pstride[t];
    }
    st.ncoef = toff[ntiles];
    YETI_TRY(upload_vec(ctx, st.tile_off, toff));
    YETI_TRY(upload_vec(ctx, st.tile_pstride, pstride));

    // kernels and grid
    YETI_TRY(stream_prepare_kernels(op));
    int nsm = 0;
    YETI_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, ctx->device));
    // segments: (tile, element range) cut from the tile-major sequence so
    // that every CTA gets about the same number of point-planes
    for (int which = 0; which < 2; which++) {
        // item (t, e) goes to CTA floor(work before it * ncta / total work);
        // consecutive items of one CTA and one tile form a segment
        int64_t total = 0;
        for (int t = 0; t < ntiles; t++) {
            const int tu = t % st.ntile[0], tv = t / st.ntile[0];
            total += (int64_t)tnq[0][tu] * tnq[1][tv] * nqw;
        }
        const int64_t nitems = (int64_t)ntiles * op->nel[2];
        const int ncta = (int)std::max<int64_t>(
            1, std::min<int64_t>((int64_t)nsm * st.per_sm[which], nitems));
        std::vector<int4> seg;
        std::vector<int> cta_seg(ncta + 1, 0);
        int64_t before = 0;
        int last_cta = -1;
        for (int t = 0; t < ntiles; t++) {
            const int tu = t % st.ntile[0], tv = t / st.ntile[0];
            const int64_t npts = (int64_t)tnq[0][tu] * tnq[1][tv];
            for (int e = 0; e < op->nel[2]; e++) {
                const int c = (int)std::min<int64_t>(ncta - 1, before * ncta / total);
                before += npts * (elem_q0[2][e + 1] - elem_q0[2][e]);
                if (c != last_cta || seg.empty() || seg.back().x != t) {
                    for (int k = last_cta + 1; k <= c; k++) cta_seg[k] = (int)seg.size();
                    seg.push_back(make_int4(t, e, e + 1, 0));
                    last_cta = c;
                } else {
                    seg.back().z = e + 1;
                }
            }
        }
        for (int k = last_cta + 1; k <= ncta; k++) cta_seg[k] = (int)seg.size();
        st.grid[which] = ncta;
        YETI_TRY(upload_vec(ctx, st.seg[which], seg));
        YETI_TRY(upload_vec(ctx, st.cta_seg[which], cta_seg));
    }
    return YETI_OK;
}

template <class T>
static int permute_one(yeti_wq_op *op, const DevBuf &src, DevBuf &dst) {
    yeti_ctx *ctx = op->ctx;
    WQStreamPlan &st = op->st;
    YETI_TRY(dst.alloc(ctx, st.ncoef * sizeof(T)));
    YETI_CUDA(cudaMemsetAsync(dst.ptr, 0, st.ncoef * sizeof(T), ctx->stream));
    // per-direction maps of the setup layout: point -> (block, local index)
    DevBuf blk[3], loc[3], nq1[3], ptrs;
    const int *hp[9];
    for (int d = 0; d < 3; d++) {
        std::vector<int> b(op->nqp[d]), l(op->nqp[d]), n(op->blk[d].size());
        for (size_t k = 0; k < op->blk[d].size(); k++) {
            const BlkInfo &B = op->blk[d][k];
            n[k] = B.nq;
            for (int q = 0; q < B.nq; q++) {
                b[B.q0 + q] = (int)k;
                l[B.q0 + q] = q;
            }
        }
        YETI_TRY(upload_vec(ctx, blk[d], b));
        YETI_TRY(upload_vec(ctx, loc[d], l));
        YETI_TRY(upload_vec(ctx, nq1[d], n));
        hp[d] = blk[d].as<int>();
        hp[3 + d] = loc[d].as<int>();
        hp[6 + d] = nq1[d].as<int>();
    }
    YETI_TRY(upload(ctx, ptrs, hp, 9));
    const int **dp = ptrs.as<const int *>();
    const int64_t n = (int64_t)op->nqp[0] * op->nqp[1] * op->nqp[2];
    const int grid = (int)std::min<int64_t>((n + 255) / 256, 148 * 16);
    k_wq_stream_permute<T><<<grid, 256, 0, ctx->stream>>>(
        src.as<T>(), dst.as<T>(), op->qoff.as<int64_t>(), dp, dp + 3, dp + 6,
        (int)op->blk[0].size(), (int)op->blk[1].size(), st.tq0[0].as<int>(),
        st.tnq[0].as<int>(), st.tq0[1].as<int>(), st.tnq[1].as<int>(), st.ntile[0],
        st.tile_off.as<int64_t>(), st.tile_pstride.as<int>(), op->nqp[0], op->nqp[1],
        op->nqp[2]);
    count_launches(1);
    YETI_CUDA(cudaGetLastError());
    YETI_CUDA(cudaStreamSynchronize(ctx->stream));
    return YETI_OK;
}

int wq_stream_permute(yeti_wq_op *op) {
    if (op->coef64.ptr) {
        DevBuf d;
        YETI_TRY(permute_one<double>(op, op->coef64, d));
        op->coef64 = std::move(d);
    }
    if (op->coef32.ptr) {
        DevBuf d;
        YETI_TRY(permute_one<float>(op, op->coef32, d));
        op->coef32 = std::move(d);
    }
    op->st.active = true;
    return YETI_OK;
}

template <class T, int P>
static int launch_stream(yeti_wq_op *op, const T *u, T *Ku, const int *done, cudaStream_t s) {
    const bool f64 = sizeof(T) == 8;
    const int which = f64 ? 0 : 1;
    WQStreamPlan &st = op->st;
    StreamArgs<T> a;
    a.u = u;
    a.Ku = Ku;
    a.done = done;
    a.coef = (f64 ? op->coef64 : op->coef32).template as<T>();
    a.tile_off = st.tile_off.as<int64_t>();
    a.tile_pstride = st.tile_pstride.as<int>();
    for (int d = 0; d < 2; d++) {
        a.tq0[d] = st.tq0[d].as<int>();
        a.tnq[d] = st.tnq[d].as<int>();
        a.ntile[d] = st.ntile[d];
    }
    for (int d = 0; d < 3; d++) {
        a.elem[d] = st.elem[d].as<int>();
        a.band[d] = (f64 ? st.band64[d] : st.band32[d]).template as<T>();
        a.nfun[d] = op->n[d];
        a.cmask[d] = op->cmask[d];
    }
    a.wq0 = st.wq0.as<int>();
    a.nqw = op->nqp[2];
    a.seg = st.seg[which].as<int4>();
    a.cta_seg = st.cta_seg[which].as<int>();
    a.ncp = op->ncp;
    k_wq_apply_stream<T, P><<<st.grid[which], kThreads, st.smem[which], s>>>(a);
    count_launches(1);
    YETI_CUDA(cudaGetLastError());
    return YETI_OK;
}

template <class T>
int wq_stream_apply(yeti_wq_op *op, const T *u, T *Ku, const int *done, cudaStream_t s) {
    switch (op->p[0]) {
        case 2: return launch_stream<T, 2>(op, u, Ku, done, s);
        case 3: return launch_stream<T, 3>(op, u, Ku, done, s);
        case 4: return launch_stream<T, 4>(op, u, Ku, done, s);
        case 5: return launch_stream<T, 5>(op, u, Ku, done, s);
        default:
            set_error("WQ streaming: degree %d", op->p[0]);
            return YETI_EUNSUPPORTED;
    }
}

template int wq_stream_apply<float>(yeti_wq_op *, const float *, float *, const int *, cudaStream_t);
template int wq_stream_apply<double>(yeti_wq_op *, const double *, double *, const int *,
                                     cudaStream_t);

}  // namespace yeti
