// FP32 streaming WQ apply, two point planes per step: Ku += K u for degrees
// 2..5 (mf_wq_get_ku_3d, mf_wq_solver.f90:284-544, generalised to 3x3
// elastic blocks), the kernel every iteration of the mixed-precision solvers
// runs.
//
// The work decomposition is the streaming kernel's (wq_stream.cu): the (u, v)
// point grid is cut into tiles of at most 16 x 16 points made of whole
// elements, a CTA takes a tile and a range of elements along w, and every
// 1-D contraction is a band of width p+1.  What differs is the step: one step
// is one w element's worth of points, taken two planes at a time (an interior
// element owns exactly two WQ points along w; the first and last elements own
// p+1 and p+2, taken as ceil(n/2) steps, a missing second plane carrying zero
// weights).  Every value that flows through a step is a pair (plane 0, plane
// 1) held in a float2, and every contraction is a packed FP32x2 FMA:
//
//   A  forward w : Y = sum_m (Bw(q0,m), Bw(q1,m)) * (x_m, x_m)  per column
//   -- barrier --
//   per warp (two point rows of the tile), warp synchronisation only:
//   B  forward v : Z[c][row][fu]          weights duplicated (v is shared)
//   C  forward u : F[l][j] per point, then the pointwise product with the 45
//                  coefficients of both planes (read as pairs straight from
//                  global memory, prefetched into L2 one step ahead by a bulk
//                  prefetch) into h[i][k][l]
//   G  backward u: one lane per (row, channel (i,k,l)) walks the row
//   -- barrier --
//   D  backward v: one thread per (i, k, fu) walks the tile's rows
//   -- barrier --
//   E  backward w: acc_m += (Ww(q0,m), Ww(q1,m)) * K  per column; the two
//                  planes' halves are added when an output plane retires.
//
// Against one plane per step this halves the instructions and barriers per
// point, and frees the shared memory the staged coefficient block took.
#include "wq.cuh"

namespace yeti {

namespace {

constexpr int kTQ = 16;          // max points of a tile per direction
constexpr int kNE = kTQ / 2;     // max elements of a regular tile
constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kHQ = 2 * 27 + 1;  // h: pairs per point column (27 channels x 2 rows, +1)

constexpr int cmax(int a, int b) { return a > b ? a : b; }

template <int P>
struct PairDims {
    static constexpr int PB = P + 1;
    static constexpr int PBW = (PB + 1) / 2 * 2;   // band row in pairs (16-byte rows)
    static constexpr int NFM = kNE + P;           // max functions of a tile
    static constexpr int GC = NFM;                // G: channel stride (pairs)
    // shared memory, in pairs
    static constexpr int Y = 2 * 3 * NFM * NFM;              // Y0, Y1 [c][fv][fu]
    static constexpr int ZH = cmax(9 * 2 * NFM, kTQ * kHQ);  // per warp: Z, then h
    static constexpr int G = kTQ * 27 * GC;                  // [qv][ch][fu]
    static constexpr int K = 9 * NFM * NFM * 2;              // aliases the Z/h parts
    static constexpr int OFF_ZH = Y;
    static constexpr int OFF_G = OFF_ZH + kWarps * ZH;
    static constexpr int TOTAL = OFF_G + G;
    static constexpr int NCOL = 3 * NFM * NFM;
    static constexpr int CPT = (NCOL + kThreads - 1) / kThreads;
    static_assert(K <= kWarps * ZH, "K must fit in the Z/h parts");
    static constexpr size_t smem_bytes() {
        return (size_t)TOTAL * sizeof(float2) + 2 * kTQ * sizeof(int);
    }
};

__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 ffma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 fadd2(float2 a, float2 b) { return __fadd2_rn(a, b); }

// The p+1 pairs of one band row (rows of PBW pairs, 16-byte aligned).
template <int P>
__device__ __forceinline__ void load_band2(const float2 *p, float2 (&w)[P + 1]) {
    constexpr int NV = PairDims<P>::PBW / 2;
    float2 t[2 * NV];
#pragma unroll
    for (int i = 0; i < NV; i++) {
        const float4 v = __ldg(reinterpret_cast<const float4 *>(p) + i);
        t[2 * i] = f2(v.x, v.y);
        t[2 * i + 1] = f2(v.z, v.w);
    }
#pragma unroll
    for (int m = 0; m <= P; m++) w[m] = t[m];
}

// Streamed coefficient pair: read once, not kept in L1.  Not volatile: the
// values are used, and the compiler may then issue the loads of a point
// ahead of the products that consume them.
__device__ __forceinline__ float2 ld_stream(const float2 *p) {
    float2 v;
    asm("ld.global.nc.L1::no_allocate.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "l"(p));
    return v;
}

// Bulk prefetch of a contiguous range into L2 (16-byte aligned, multiple of
// 16 bytes), in pieces of at most 32 KiB issued by consecutive threads.
__device__ __forceinline__ void prefetch_block(const void *p, uint32_t bytes, int tid) {
    constexpr uint32_t kPiece = 32768;
    const uint32_t off = (uint32_t)tid * kPiece;
    if (off < bytes) {
        const uint32_t n = min(kPiece, bytes - off);
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(
                         reinterpret_cast<const char *>(p) + off),
                     "r"(n)
                     : "memory");
    }
}

// Tile patterns of one direction (host flag), as in wq_stream.cu: 1 every
// element owns two points; 2 the first element owns p+1 points, the others
// two (the first tile); 3 the last element owns p+2 points, the others two
// (the last tile); 0 anything else (run-time walk).
__host__ __device__ constexpr int pat_nemax(int P, int pat) {
    return pat == 1 ? kNE : pat == 2 ? 1 + (kTQ - (P + 1)) / 2 : 1 + (kTQ - (P + 2)) / 2;
}
__host__ __device__ constexpr int pat_q0(int P, int pat, int e) {
    return pat == 2 ? (e == 0 ? 0 : P + 1 + 2 * (e - 1)) : 2 * e;
}

// Backward u of one channel of one row (pairs): g[f] = sum_q W(q, f - rel(q))
// h[q], h at stride kHQ, weights from the duplicated band table.
template <int P, int PAT>
__device__ __forceinline__ void walk_u2(const float2 *h, float2 *g, const float2 *tab, int kind,
                                        int ne) {
    constexpr int PBW = PairDims<P>::PBW, NEM = pat_nemax(P, PAT), NF = NEM + P;
    float2 a[NF];
#pragma unroll
    for (int f = 0; f < NF; f++) a[f] = f2(0.f, 0.f);
#pragma unroll
    for (int e = 0; e < NEM; e++) {
        if (e < ne) {
            const int q0 = pat_q0(P, PAT, e);
            const int np = PAT == 2 ? (e == 0 ? P + 1 : 2) : (PAT == 3 && e == ne - 1 ? P + 2 : 2);
#pragma unroll
            for (int pt = 0; pt < P + 2; pt++) {
                if (pt < np) {
                    const int q = q0 + pt;
                    float2 w[P + 1];
                    load_band2<P>(tab + (q * 6 + kind) * PBW, w);
                    const float2 x = h[q * kHQ];
#pragma unroll
                    for (int m = 0; m <= P; m++) a[e + m] = ffma2(w[m], x, a[e + m]);
                }
            }
            g[e] = a[e];
        }
    }
#pragma unroll
    for (int f = 1; f < NF; f++)
        if (f >= ne && f < ne + P) g[f] = a[f];
}

template <int P>
__device__ __forceinline__ void walk_u2_generic(const float2 *h, float2 *g, const float2 *tab,
                                                int kind, const int *rel, int nq) {
    constexpr int PBW = PairDims<P>::PBW;
    float2 a[P + 1];
#pragma unroll
    for (int m = 0; m <= P; m++) a[m] = f2(0.f, 0.f);
    int cur = 0;
    for (int q = 0; q < nq; q++) {
        const int r = rel[q];
        if (r != cur) {
            g[cur] = a[0];
#pragma unroll
            for (int m = 0; m < P; m++) a[m] = a[m + 1];
            a[P] = f2(0.f, 0.f);
            cur = r;
        }
        float2 w[P + 1];
        load_band2<P>(tab + (q * 6 + kind) * PBW, w);
        const float2 x = h[q * kHQ];
#pragma unroll
        for (int m = 0; m <= P; m++) a[m] = ffma2(w[m], x, a[m]);
    }
#pragma unroll
    for (int m = 0; m <= P; m++) g[cur + m] = a[m];
}

// Backward v of the three channels (i,k,l=0..2) of one fu column, merged on
// the w key: K0[fv] = sum wa g0 + wb g1, K1[fv] = sum wa g2 (wa: table row
// ka, trial l != v; wb: row ka+1, trial l == v).  g of row q at gb + q*27*GC.
template <int P, int PAT>
__device__ __forceinline__ void walk_v2(const float2 *gb, float4 *kp, const float2 *tab, int ka,
                                        int ne) {
    using D = PairDims<P>;
    constexpr int PBW = D::PBW, NEM = pat_nemax(P, PAT), NF = NEM + P, NFM = D::NFM;
    constexpr int GC = D::GC, GQ = 27 * D::GC;
    float2 A0[NF], A1[NF];
#pragma unroll
    for (int f = 0; f < NF; f++) A0[f] = A1[f] = f2(0.f, 0.f);
#pragma unroll
    for (int e = 0; e < NEM; e++) {
        if (e < ne) {
            const int q0 = pat_q0(P, PAT, e);
            const int np = PAT == 2 ? (e == 0 ? P + 1 : 2) : (PAT == 3 && e == ne - 1 ? P + 2 : 2);
#pragma unroll
            for (int pt = 0; pt < P + 2; pt++) {
                if (pt < np) {
                    const int q = q0 + pt;
                    float2 wa[P + 1], wb[P + 1];
                    load_band2<P>(tab + (q * 6 + ka) * PBW, wa);
                    load_band2<P>(tab + (q * 6 + ka + 1) * PBW, wb);
                    const float2 *g = gb + q * GQ;
                    const float2 x0 = g[0], x1 = g[GC], x2 = g[2 * GC];
#pragma unroll
                    for (int m = 0; m <= P; m++) {
                        A0[e + m] = ffma2(wb[m], x1, ffma2(wa[m], x0, A0[e + m]));
                        A1[e + m] = ffma2(wa[m], x2, A1[e + m]);
                    }
                }
            }
            kp[e * NFM] = make_float4(A0[e].x, A0[e].y, A1[e].x, A1[e].y);
        }
    }
#pragma unroll
    for (int f = 1; f < NF; f++)
        if (f >= ne && f < ne + P) kp[f * NFM] = make_float4(A0[f].x, A0[f].y, A1[f].x, A1[f].y);
}

template <int P>
__device__ __forceinline__ void walk_v2_generic(const float2 *gb, float4 *kp, const float2 *tab,
                                                int ka, const int *rel, int nq) {
    using D = PairDims<P>;
    constexpr int PBW = D::PBW, NFM = D::NFM, GC = D::GC, GQ = 27 * D::GC;
    float2 A0[P + 1], A1[P + 1];
#pragma unroll
    for (int m = 0; m <= P; m++) A0[m] = A1[m] = f2(0.f, 0.f);
    int cur = 0;
    for (int q = 0; q < nq; q++) {
        const int r = rel[q];
        if (r != cur) {
            kp[cur * NFM] = make_float4(A0[0].x, A0[0].y, A1[0].x, A1[0].y);
#pragma unroll
            for (int m = 0; m < P; m++) {
                A0[m] = A0[m + 1];
                A1[m] = A1[m + 1];
            }
            A0[P] = A1[P] = f2(0.f, 0.f);
            cur = r;
        }
        float2 wa[P + 1], wb[P + 1];
        load_band2<P>(tab + (q * 6 + ka) * PBW, wa);
        load_band2<P>(tab + (q * 6 + ka + 1) * PBW, wb);
        const float2 *g = gb + q * GQ;
        const float2 x0 = g[0], x1 = g[GC], x2 = g[2 * GC];
#pragma unroll
        for (int m = 0; m <= P; m++) {
            A0[m] = ffma2(wb[m], x1, ffma2(wa[m], x0, A0[m]));
            A1[m] = ffma2(wa[m], x2, A1[m]);
        }
    }
#pragma unroll
    for (int m = 0; m <= P; m++)
        kp[(cur + m) * NFM] = make_float4(A0[m].x, A0[m].y, A1[m].x, A1[m].y);
}

}  // namespace

struct PairArgs {
    const float *u;
    float *Ku;
    const int *done;
    const float2 *coef;        // pair-step layout
    const int64_t *tile_off;   // first pair of a tile
    const int *tile_sstride;   // pairs per step of a tile (padded)
    const int *tq0[2];         // first point of a u / v tile
    const int *tnq[2];         // points of a u / v tile
    const int *treg[2];        // tile pattern: 1 regular, 2 first, 3 last, 0 other
    int ntile[2];
    const int *elem[2];        // element owning each u / v point
    const float2 *bandd[2];    // u, v bands duplicated: [nqp][6][PBW] pairs
    const float2 *bandw;       // w bands per step: [nstep][6][PBW] (plane 0, plane 1)
    const int *sstart;         // first step of each w element (nel_w + 1)
    const int4 *seg;           // (tile, e_begin, e_end, -)
    const int *cta_seg;        // segments of a CTA
    int nfun[3];
    int64_t ncp;
    int cmask[3];
};

template <int P>
__global__ void __launch_bounds__(kThreads, 2) k_wq_apply_pair(PairArgs a) {
    using D = PairDims<P>;
    constexpr int PB = D::PB, PBW = D::PBW, NFM = D::NFM, CPT = D::CPT;
    constexpr int GC = D::GC, ZH = D::ZH;
    if (a.done && *a.done) return;
    extern __shared__ __align__(16) unsigned char smraw[];
    float2 *const sm = reinterpret_cast<float2 *>(smraw);
    float2 *const RY = sm;
    float2 *const RZH = sm + D::OFF_ZH;   // per warp: Z, then h; K (all warps) after G
    float2 *const RG = sm + D::OFF_G;
    int *const relu = reinterpret_cast<int *>(sm + D::TOTAL);
    int *const relv = relu + kTQ;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int64_t plane = (int64_t)a.nfun[0] * a.nfun[1];
    const float2 *const tabu = a.bandd[0];
    const float2 *const tabv = a.bandd[1];

    for (int si = a.cta_seg[blockIdx.x]; si < a.cta_seg[blockIdx.x + 1]; si++) {
        const int4 sg = a.seg[si];
        const int tu = sg.x % a.ntile[0], tv = sg.x / a.ntile[0];
        const int qu0 = a.tq0[0][tu], nqu = a.tnq[0][tu];
        const int qv0 = a.tq0[1][tv], nqv = a.tnq[1][tv];
        const int patu = a.treg[0][tu], patv = a.treg[1][tv];
        const bool regu = patu == 1, regv = patv == 1;
        const int fu0 = a.elem[0][qu0], fv0 = a.elem[1][qv0];
        const int nfu = a.elem[0][qu0 + nqu - 1] + PB - fu0;
        const int nfv = a.elem[1][qv0 + nqv - 1] + PB - fv0;
        const int neu = a.elem[0][qu0 + nqu - 1] - fu0 + 1;   // elements of the tile
        const int nev = a.elem[1][qv0 + nqv - 1] - fv0 + 1;
        const int npts = nqu * nqv;
        const float2 *const coef_t = a.coef + a.tile_off[sg.x];
        const int sstride = a.tile_sstride[sg.x];
        const uint32_t sbytes = (uint32_t)((npts * kWQCoef * 8 + 15) & ~15);
        const int nrow = min(2, nqv - 2 * warp);   // rows of this warp (may be <= 0)
        const float2 *const tu_tab = tabu + (size_t)qu0 * 6 * PBW;
        const float2 *const tv_tab = tabv + (size_t)qv0 * 6 * PBW;
        const int s_first = a.sstart[sg.y], s_end = a.sstart[sg.z];

        __syncthreads();   // the previous segment is done with relu / relv
        if (tid < kTQ) {
            relu[tid] = tid < nqu ? a.elem[0][qu0 + tid] - fu0 : 0;
            relv[tid] = tid < nqv ? a.elem[1][qv0 + tid] - fv0 : 0;
        }
        prefetch_block(coef_t + (int64_t)s_first * sstride, sbytes, tid);
        // stage D thread: (ik, fu)
        const bool d_act = tid < 9 * nfu;
        const int d_ik = d_act ? tid / nfu : 0, d_fu = d_act ? tid - d_ik * nfu : 0;

        // columns (c, fv, fu) of this thread: stages A and E
        const int ncol = 3 * nfv * nfu;
        int64_t cbase[CPT];
        int cinfo[CPT];   // bit 0..1: component; bit 2: active; bits 3..: fv*NFM+fu
        bool cclamp_uv[CPT];
        float2 x[CPT][PB], acc[CPT][PB];
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
                x[cc][m] = f2(0.f, 0.f);
                acc[cc][m] = f2(0.f, 0.f);
            }
        }
        auto clamped_w = [&](int cc, int fw) {
            const int cm = a.cmask[cinfo[cc] & 3];
            return cclamp_uv[cc] || ((cm & 16) && fw == 0) || ((cm & 32) && fw == a.nfun[2] - 1);
        };
        auto load_x = [&](int cc, int fw) -> float2 {
            if (!(cinfo[cc] & 4) || clamped_w(cc, fw)) return f2(0.f, 0.f);
            const float v = a.u[cbase[cc] + plane * fw];
            return f2(v, v);
        };
        auto retire = [&](int cc, int fw, float2 v) {
            if ((cinfo[cc] & 4) && !clamped_w(cc, fw))
                atomicAdd(&a.Ku[cbase[cc] + plane * fw], v.x + v.y);
        };
#pragma unroll
        for (int cc = 0; cc < CPT; cc++)
#pragma unroll
            for (int m = 0; m < P; m++) x[cc][m] = load_x(cc, sg.y + m);

        for (int e = sg.y; e < sg.z; e++) {
#pragma unroll
            for (int cc = 0; cc < CPT; cc++) {
                x[cc][P] = load_x(cc, e + P);
                acc[cc][P] = f2(0.f, 0.f);
            }
            const int s_e1 = a.sstart[e + 1];
            for (int s = a.sstart[e]; s < s_e1; s++) {
                const float2 *const bw = a.bandw + (size_t)s * 6 * PBW;
                const float2 *const cstep = coef_t + (int64_t)s * sstride;
                if (s + 1 < s_end) prefetch_block(cstep + sstride, sbytes, tid);
                // ---- A: forward w (pairs of planes)
                {
                    float2 b0[PB], b1[PB];
                    load_band2<P>(bw, b0);
                    load_band2<P>(bw + PBW, b1);
#pragma unroll
                    for (int cc = 0; cc < CPT; cc++) {
                        if (!(cinfo[cc] & 4)) continue;
                        float2 y0 = f2(0.f, 0.f), y1 = f2(0.f, 0.f);
#pragma unroll
                        for (int m = 0; m < PB; m++) {
                            y0 = ffma2(b0[m], x[cc][m], y0);
                            y1 = ffma2(b1[m], x[cc][m], y1);
                        }
                        const int c = cinfo[cc] & 3, k = cinfo[cc] >> 3;
                        RY[c * NFM * NFM + k] = y0;
                        RY[(3 + c) * NFM * NFM + k] = y1;
                    }
                }
                __syncthreads();
                if (nrow > 0) {
                    float2 *const zh = RZH + warp * ZH;
                    // ---- B: forward v of this warp's rows, lane (row, fu)
                    {
                        const int row = lane >> 4, fu = lane & 15;
                        if (row < nrow && fu < nfu) {
                            const int qv = 2 * warp + row;
                            const int rv = regv ? (qv >> 1) : relv[qv];
                            float2 b0[PB], b1[PB];
                            load_band2<P>(tv_tab + (qv * 6 + 0) * PBW, b0);
                            load_band2<P>(tv_tab + (qv * 6 + 1) * PBW, b1);
#pragma unroll
                            for (int c = 0; c < 3; c++) {
                                const float2 *y0 = RY + (c * NFM + rv) * NFM + fu;
                                const float2 *y1 = RY + ((3 + c) * NFM + rv) * NFM + fu;
                                float2 z0 = f2(0.f, 0.f), z1 = f2(0.f, 0.f), z2 = f2(0.f, 0.f);
#pragma unroll
                                for (int m = 0; m < PB; m++) {
                                    const float2 a0 = y0[m * NFM], a1 = y1[m * NFM];
                                    z0 = ffma2(b0[m], a0, z0);
                                    z1 = ffma2(b1[m], a0, z1);
                                    z2 = ffma2(b0[m], a1, z2);
                                }
                                zh[(0 * 3 + c) * (2 * NFM) + row * NFM + fu] = z0;
                                zh[(1 * 3 + c) * (2 * NFM) + row * NFM + fu] = z1;
                                zh[(2 * 3 + c) * (2 * NFM) + row * NFM + fu] = z2;
                            }
                        }
                    }
                    __syncwarp();
                    // ---- C: forward u and the pointwise coefficients, lane (row, qu)
                    {
                        const int row = lane >> 4, qu = lane & 15;
                        const bool act = row < nrow && qu < nqu;
                        float2 f[3][3];
                        if (act) {
                            const int ru = regu ? (qu >> 1) : relu[qu];
                            float2 b0[PB], b1[PB];
                            load_band2<P>(tu_tab + (qu * 6 + 0) * PBW, b0);
                            load_band2<P>(tu_tab + (qu * 6 + 1) * PBW, b1);
#pragma unroll
                            for (int l = 0; l < 3; l++)
#pragma unroll
                                for (int j = 0; j < 3; j++) {
                                    const float2 *zr = zh + (l * 3 + j) * (2 * NFM) + row * NFM + ru;
                                    float2 v = f2(0.f, 0.f);
#pragma unroll
                                    for (int m = 0; m < PB; m++) v = ffma2(l == 0 ? b1[m] : b0[m], zr[m], v);
                                    f[l][j] = v;
                                }
                        }
                        __syncwarp();   // the warp's Z is read; h takes its place
                        if (act) {
                            const int pt = (2 * warp + row) * nqu + qu;
                            // entry-major pairs: entry e of point pt at e*npts + pt
                            const float2 *cp = cstep + pt;
                            float2 h[27];
#pragma unroll
                            for (int ch = 0; ch < 27; ch++) h[ch] = f2(0.f, 0.f);
#pragma unroll
                            for (int I = 0; I < 9; I++) {
#pragma unroll
                                for (int J = I; J < 9; J++) {
                                    const float2 sv = ld_stream(cp + sym9(I, J) * npts);
                                    const int i = I / 3, k = I % 3, j = J / 3, l = J % 3;
                                    h[(i * 3 + k) * 3 + l] = ffma2(sv, f[l][j], h[(i * 3 + k) * 3 + l]);
                                    if (I != J) h[(j * 3 + l) * 3 + k] = ffma2(sv, f[k][i], h[(j * 3 + l) * 3 + k]);
                                }
                            }
                            float2 *hp = zh + qu * kHQ + row;
#pragma unroll
                            for (int ch = 0; ch < 27; ch++) hp[2 * ch] = h[ch];
                        }
                    }
                    __syncwarp();
                    // ---- G: backward u, lane (row, channel), 54 walks per warp
                    for (int wk = lane; wk < 54; wk += 32) {
                        const int row = wk & 1, ch = wk >> 1;
                        if (row < nrow) {
                            const int k = (ch / 3) % 3, l = ch % 3;
                            const int kind = 2 + 2 * (k == 0) + (l == 0);   // W_{[k==u][l==u]}
                            const float2 *hr = zh + 2 * ch + row;
                            float2 *gr = RG + ((2 * warp + row) * 27 + ch) * GC;
                            switch (patu) {
                                case 1: walk_u2<P, 1>(hr, gr, tu_tab, kind, neu); break;
                                case 2: walk_u2<P, 2>(hr, gr, tu_tab, kind, neu); break;
                                case 3: walk_u2<P, 3>(hr, gr, tu_tab, kind, neu); break;
                                default: walk_u2_generic<P>(hr, gr, tu_tab, kind, relu, nqu);
                            }
                        }
                    }
                }
                __syncthreads();
                // ---- D: backward v, thread (i, k, fu); K aliases the Z/h parts
                if (d_act) {
                    const int ik = d_ik, fu = d_fu;
                    const int ka = 2 + 2 * (ik % 3 == 1);   // W_{[k==v], 0}
                    const float2 *gb = RG + (ik * 3) * GC + fu;
                    float4 *kp = reinterpret_cast<float4 *>(RZH) + ik * NFM * NFM + fu;
                    switch (patv) {
                        case 1: walk_v2<P, 1>(gb, kp, tv_tab, ka, nev); break;
                        case 2: walk_v2<P, 2>(gb, kp, tv_tab, ka, nev); break;
                        case 3: walk_v2<P, 3>(gb, kp, tv_tab, ka, nev); break;
                        default: walk_v2_generic<P>(gb, kp, tv_tab, ka, relv, nqv);
                    }
                }
                __syncthreads();
                // ---- E: backward w into the register ring of output planes
                {
                    float2 w00[PB], w01[PB], w10[PB], w11[PB];
                    load_band2<P>(bw + 2 * PBW, w00);
                    load_band2<P>(bw + 3 * PBW, w01);
                    load_band2<P>(bw + 4 * PBW, w10);
                    load_band2<P>(bw + 5 * PBW, w11);
                    const float4 *K4 = reinterpret_cast<const float4 *>(RZH);
#pragma unroll
                    for (int cc = 0; cc < CPT; cc++) {
                        if (!(cinfo[cc] & 4)) continue;
                        const int i = cinfo[cc] & 3, kidx = cinfo[cc] >> 3;
                        const float4 *kb = K4 + (i * 3) * NFM * NFM + kidx;
                        const float4 ka = kb[0], kb1 = kb[NFM * NFM], kc = kb[2 * NFM * NFM];
                        const float2 s00 = fadd2(f2(ka.x, ka.y), f2(kb1.x, kb1.y));
                        const float2 s01 = fadd2(f2(ka.z, ka.w), f2(kb1.z, kb1.w));
                        const float2 k20 = f2(kc.x, kc.y), k21 = f2(kc.z, kc.w);
#pragma unroll
                        for (int m = 0; m < PB; m++) {
                            float2 t = ffma2(w00[m], s00, acc[cc][m]);
                            t = ffma2(w01[m], s01, t);
                            t = ffma2(w10[m], k20, t);
                            acc[cc][m] = ffma2(w11[m], k21, t);
                        }
                    }
                }
                // no barrier: the next step's stage A writes only RY, and
                // the next B writes the Z/h parts after the barrier that
                // follows A
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

// Copy FP32 coefficients from the element-block layout of the setup kernels
// into the pair-step layout: per tile, per w step, entry-major pairs
// (entry e of point pt: pair e*npts + pt; .x plane 2k, .y plane 2k+1 of the
// element).  The second plane of a step that has only one stays zero.
__global__ void k_wq_pair_permute(const float *src, float2 *dst, const int64_t *qoff1,
                                  const int *const *blk1, const int *const *loc1,
                                  const int *const *nq1, int nb1u, int nb1v, const int *tq0u,
                                  const int *tnqu, const int *tq0v, const int *tnqv, int ntu,
                                  const int64_t *tile_off, const int *tile_sstride,
                                  const int *qw_step, int nqu_all, int nqv_all, int nqw_all) {
    const int64_t n = (int64_t)nqu_all * nqv_all * nqw_all;
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < n;
         g += (int64_t)gridDim.x * blockDim.x) {
        const int qu = (int)(g % nqu_all);
        const int qv = (int)((g / nqu_all) % nqv_all);
        const int qw = (int)(g / ((int64_t)nqu_all * nqv_all));
        const int bu = blk1[0][qu], bv = blk1[1][qv], bw = blk1[2][qw];
        const int64_t b = bu + (int64_t)nb1u * (bv + (int64_t)nb1v * bw);
        const int nu1 = nq1[0][bu], nv1 = nq1[1][bv], nw1 = nq1[2][bw];
        const int64_t nqb = (int64_t)nu1 * nv1 * nw1;
        const int64_t sbase = qoff1[b] * kWQCoef +
                              (loc1[2][qw] * (int64_t)nv1 + loc1[1][qv]) * nu1 + loc1[0][qu];
        int tu = 0, tv = 0;
        while (tq0u[tu] + tnqu[tu] <= qu) tu++;
        while (tq0v[tv] + tnqv[tv] <= qv) tv++;
        const int t = tu + ntu * tv;
        const int npts = tnqu[tu] * tnqv[tv];
        const int pt = (qv - tq0v[tv]) * tnqu[tu] + (qu - tq0u[tu]);
        const int st = qw_step[qw];
        float *d = reinterpret_cast<float *>(dst + tile_off[t] + (int64_t)(st >> 1) * tile_sstride[t] + pt);
        const int slot = st & 1;
        for (int e = 0; e < kWQCoef; e++) d[(int64_t)e * npts * 2 + slot] = src[sbase + e * nqb];
    }
}

template <int P>
static int pair_attr(yeti_wq_op *op) {
    const size_t smem = PairDims<P>::smem_bytes();
    YETI_CUDA(cudaFuncSetAttribute(k_wq_apply_pair<P>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)smem));
    int per_sm = 0;
    YETI_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_wq_apply_pair<P>, kThreads,
                                                            smem));
    YETI_CHECK(per_sm >= 1, YETI_EUNSUPPORTED, "WQ pair kernel does not fit on an SM");
    op->st.pair_smem = smem;
    op->st.pair_per_sm = per_sm;
    return YETI_OK;
}

int wq_pair_prepare(yeti_wq_op *op) {
    switch (op->p[0]) {
        case 2: return pair_attr<2>(op);
        case 3: return pair_attr<3>(op);
        case 4: return pair_attr<4>(op);
        case 5: return pair_attr<5>(op);
        default:
            set_error("WQ pair kernel: degree %d", op->p[0]);
            return YETI_EUNSUPPORTED;
    }
}

int wq_pair_band_width(int p) { return (p + 2) / 2 * 2; }

int wq_pair_permute(yeti_wq_op *op, const float *src, float2 *dst, const int64_t *qoff1,
                    const int *const *blk1, const int *const *loc1, const int *const *nq1,
                    const int *qw_step) {
    WQStreamPlan &st = op->st;
    const int64_t n = (int64_t)op->nqp[0] * op->nqp[1] * op->nqp[2];
    const int grid = (int)std::min<int64_t>((n + 255) / 256, 148 * 16);
    k_wq_pair_permute<<<grid, 256, 0, op->ctx->stream>>>(
        src, dst, qoff1, blk1, loc1, nq1, (int)op->blk[0].size(), (int)op->blk[1].size(),
        st.tq0[0].as<int>(), st.tnq[0].as<int>(), st.tq0[1].as<int>(), st.tnq[1].as<int>(),
        st.ntile[0], st.pair_tile_off.as<int64_t>(), st.pair_sstride.as<int>(), qw_step,
        op->nqp[0], op->nqp[1], op->nqp[2]);
    count_launches(1);
    YETI_CUDA(cudaGetLastError());
    return YETI_OK;
}

template <int P>
static int launch_pair(yeti_wq_op *op, const float *u, float *Ku, const int *done, cudaStream_t s) {
    WQStreamPlan &st = op->st;
    PairArgs a;
    a.u = u;
    a.Ku = Ku;
    a.done = done;
    a.coef = op->coef32.as<float2>();
    a.tile_off = st.pair_tile_off.as<int64_t>();
    a.tile_sstride = st.pair_sstride.as<int>();
    for (int d = 0; d < 2; d++) {
        a.tq0[d] = st.tq0[d].as<int>();
        a.tnq[d] = st.tnq[d].as<int>();
        a.treg[d] = st.treg[d].as<int>();
        a.ntile[d] = st.ntile[d];
        a.elem[d] = st.elem[d].as<int>();
        a.bandd[d] = st.pair_band[d].as<float2>();
    }
    a.bandw = st.pair_bandw.as<float2>();
    a.sstart = st.pair_sstart.as<int>();
    a.seg = st.seg[1].as<int4>();
    a.cta_seg = st.cta_seg[1].as<int>();
    for (int d = 0; d < 3; d++) {
        a.nfun[d] = op->n[d];
        a.cmask[d] = op->cmask[d];
    }
    a.ncp = op->ncp;
    k_wq_apply_pair<P><<<st.grid[1], kThreads, st.pair_smem, s>>>(a);
    count_launches(1);
    YETI_CUDA(cudaGetLastError());
    return YETI_OK;
}

int wq_pair_apply(yeti_wq_op *op, const float *u, float *Ku, const int *done, cudaStream_t s) {
    switch (op->p[0]) {
        case 2: return launch_pair<2>(op, u, Ku, done, s);
        case 3: return launch_pair<3>(op, u, Ku, done, s);
        case 4: return launch_pair<4>(op, u, Ku, done, s);
        case 5: return launch_pair<5>(op, u, Ku, done, s);
        default:
            set_error("WQ pair kernel: degree %d", op->p[0]);
            return YETI_EUNSUPPORTED;
    }
}

}  // namespace yeti
