// Streaming WQ apply: Ku += K u for degrees 2..5, the kernel every Krylov
// iteration of the WQ solve runs (mf_wq_get_ku_3d, mf_wq_solver.f90:284-544,
// generalised to 3x3 elastic blocks).
//
// Work decomposition
// ------------------
// The (u, v) point grid is cut into tiles of at most 16 x YETI_WQ_TV (8)
// points made of whole elements; a CTA takes a tile and a range of elements
// along w and marches through the w point planes of that range.  Every WQ point belongs
// to one element and, in each direction, its B0/B1/W** rows are non-zero for
// the p+1 functions elem(q)..elem(q)+p only (checked on the host), so every
// 1-D contraction is a band of width p+1.  Per plane:
//
//   A  forward w : Y_t[c][fv][fu] = sum_m Bt_w(qw,m) X[c][fv][fu][e+m]
//                  (one thread per (c, fv, fu) column; X for functions
//                  e..e+p lives in a register ring that advances with e)
//                  (computed for the next plane beside stage D of this one)
//   -- barrier --
//   each warp owns two point rows qv of the tile and runs, with warp
//   synchronisation only:
//   B  forward v : Z_s[c][row][fu]  (s: B0v.Y0, B1v.Y0, B0v.Y1)
//   C  forward u + pointwise, one lane per point: F[l][j] = d u_j / d xi_l,
//                  then h[i][k][l] = sum_j S[(i,k),(j,l)] F[l][j] with the
//                  45 streamed coefficients of the point (the HBM stream)
//   G  backward u: one lane per channel (i,k,l) walks the warp's two rows,
//                  weights W^{[k==u][l==u]}
//   -- barrier --
//   D  backward v: one thread per (i, k) and two fu (FP32; one fu in FP64)
//                  walks the columns over the tile's rows (one pair of band
//                  rows serves both); channels merged on (l == w):
//                  K[fv][fu][i][k][lw]
//   -- barrier --
//   E  backward w: accumulation into a register ring of output planes
//                  e..e+p; plane e is complete after element e and is added
//                  to Ku (atomics: tiles overlap on the p halo functions,
//                  element ranges overlap on p planes)
//
// The walks keep the p+1 functions of the current element in registers.  In
// a regular tile (every element owns two points: all but the first and last
// element of a direction) the walk is unrolled at compile time and the ring
// is register renaming; the first and last tiles take a run-time walk.
// While a plane is processed, the next plane's coefficient block
// (contiguous, 256-byte aligned) is prefetched into L2.
#include <algorithm>
#include <cstring>
#include <numeric>

#include "wq.cuh"

namespace yeti {

namespace {

// Tile height along v.  16 x 8 point tiles (128 threads, four CTAs per SM:
// four independent barrier domains) measured faster than 16 x 16 tiles (256
// threads, two per SM) on B200: FP32 apply 179 against 192 us at 64^3 p=3.
#ifndef YETI_WQ_TV
#define YETI_WQ_TV 8
#endif
constexpr int kTQ = 16;          // max points of a tile along u
constexpr int kTV = YETI_WQ_TV;  // max points of a tile along v (16 or 8)
constexpr int kNE = kTQ / 2;     // max elements of a regular tile along u
constexpr int kNEV = kTV / 2;    // ... along v
constexpr int kThreads = kTQ * kTV;   // one thread per point of a plane tile
constexpr int kWarps = kThreads / 32;
constexpr int kCtasPerSm = 512 / kThreads;   // 2 (16 x 16 tiles) or 4 (16 x 8)
constexpr int kHS = 2 * kTQ + 1; // channel stride of a warp's h block

constexpr int cmax(int a, int b) { return a > b ? a : b; }
constexpr int round4(int a) { return (a + 3) / 4 * 4; }

template <int P>
struct Dims {
    static constexpr int PB = P + 1;
    static constexpr int PBP = round4(PB);     // padded band row
    static constexpr int TS = 6 * PBP + 4;     // table row of one point: six bands, padded so
                                               // that the 16-byte loads of consecutive points
                                               // fall on different banks
    static constexpr int NFM = kNE + P;        // max functions of a tile along u
    static constexpr int NFV = kNEV + P;       // ... along v
    static constexpr int Y = round4(2 * 3 * NFV * NFM);
    static constexpr int ZHP = round4(cmax(9 * 2 * NFM, 27 * kHS));   // Z, then h
    // a warp's G block: [row][function][channel], the 27 channels
    // consecutive (stage G's lanes are channels; stage D's threads, with
    // the 9 (i,k) fastest, read 3 (i,k) + l at a function stride of 27:
    // banks 3 * tid, all distinct)
    static constexpr int RS = 27 * NFM;                               // row of G
    static constexpr int GP = round4(2 * RS);                         // G
    static constexpr int K = 9 * NFV * NFM * 2;                       // aliases the Z/h parts
    static constexpr int TAB = kTQ * TS;                              // u (v: kTV rows)
    static constexpr int OFF_ZH = Y;
    static constexpr int OFF_G = OFF_ZH + kWarps * ZHP;
    static constexpr int OFF_TAB = OFF_G + kWarps * GP;
    static constexpr int TOTAL = OFF_TAB + TAB + kTV * TS;
    static constexpr int NCOL = 3 * NFV * NFM;
    static constexpr int CPT = (NCOL + kThreads - 1) / kThreads;
    static constexpr int CB = kTQ * kTV * 45;   // one plane's coefficients (staged kernels)
    static_assert(K <= kWarps * ZHP, "K must fit in the Z/h parts");
    // values, then the staged coefficient block (FP32), the two rel tables
    // and the mbarrier
    template <class T>
    static constexpr size_t smem_bytes() {
        return (size_t)(TOTAL + (sizeof(T) == 4 ? CB : 0)) * sizeof(T) + (kTQ + kTV) * sizeof(int) +
               sizeof(uint64_t);
    }
};

__device__ __forceinline__ void prefetch_l2(const void *p) {
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

// The p+1 band values of one row of a band table (rows padded to a multiple
// of 4 values, 16-byte aligned), with vector loads.
template <int P>
__device__ __forceinline__ void load_band(const float *p, float (&w)[P + 1]) {
    constexpr int NV = round4(P + 1) / 4;
    float t[4 * NV];
#pragma unroll
    for (int i = 0; i < NV; i++) {
        const float4 v = reinterpret_cast<const float4 *>(p)[i];
        t[4 * i] = v.x;
        t[4 * i + 1] = v.y;
        t[4 * i + 2] = v.z;
        t[4 * i + 3] = v.w;
    }
#pragma unroll
    for (int m = 0; m <= P; m++) w[m] = t[m];
}

template <int P>
__device__ __forceinline__ void load_band(const double *p, double (&w)[P + 1]) {
    constexpr int NV = round4(P + 1) / 2;
    double t[2 * NV];
#pragma unroll
    for (int i = 0; i < NV; i++) {
        const double2 v = reinterpret_cast<const double2 *>(p)[i];
        t[2 * i] = v.x;
        t[2 * i + 1] = v.y;
    }
#pragma unroll
    for (int m = 0; m <= P; m++) w[m] = t[m];
}

__device__ __forceinline__ void store_pair(float *p, float a, float b) {
    *reinterpret_cast<float2 *>(p) = make_float2(a, b);
}
__device__ __forceinline__ void store_pair(double *p, double a, double b) {
    *reinterpret_cast<double2 *>(p) = make_double2(a, b);
}
__device__ __forceinline__ void load_pair(const float *p, float &a, float &b) {
    const float2 v = *reinterpret_cast<const float2 *>(p);
    a = v.x;
    b = v.y;
}
__device__ __forceinline__ void load_pair(const double *p, double &a, double &b) {
    const double2 v = *reinterpret_cast<const double2 *>(p);
    a = v.x;
    b = v.y;
}

// ------------------------------------------------ bulk copies (TMA engine)
constexpr int kWaitTries = 1 << 16;   // bound of every mbarrier wait

__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t *bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// One bulk copy global -> shared that completes the barrier's current phase.
// dst and src 16-byte aligned, bytes a multiple of 16.
// The coefficient stream is read once per apply and is several times the L2:
// its lines are marked evict-first, so that the solver's vectors (u, Ku and
// the Krylov vectors, a few MB each) stay in L2 across the apply.
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    uint64_t policy;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(policy));
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], "
        "%2, [%3], %4;" ::"r"(smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar)), "l"(policy)
        : "memory");
}
// Wait for the phase with the given parity, at most `tries` polls.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, int tries) {
    for (int i = 0; i < tries; i++) {
        uint32_t ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
            " selp.u32 %0, 1, 0, p;\n}"
            : "=r"(ok)
            : "r"(smem_addr(bar)), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

// ---------------------------------------------------------------- walks
// Tile patterns of one direction (host flag): 1 every element owns two
// points and the tile is full (tq / 2 elements: the walks' element count is
// a compile-time constant); 4 every element owns two points, fewer
// elements; 2 the first element owns p+1 points, the others two (the first
// tile); 3 the last element owns p+2 points, the others two (the last tile);
// 0 anything else (run-time walk).
__host__ __device__ constexpr int pat_nemax(int P, int pat, int tq = kTQ) {
    return pat == 1 || pat == 4 ? tq / 2 : pat == 2 ? 1 + (tq - (P + 1)) / 2 : 1 + (tq - (P + 2)) / 2;
}
// first point of element e in a tile of pattern pat
__host__ __device__ constexpr int pat_q0(int P, int pat, int e) {
    return pat == 2 ? (e == 0 ? 0 : P + 1 + 2 * (e - 1)) : 2 * e;
}

// Backward u of one channel of a warp's two rows: g[f] = sum_q W_kind(q,
// f - rel(q)) h[q], walked element by element with the accumulators of the
// element's p+1 functions named at compile time; one band row serves both
// rows.  h: row 0 at h[q], row 1 at h[kTQ + q]; g: function f of row r at
// g[r * RS + 27 f] (the G block's channel stride is 1).
template <class T, int P, int PAT, bool PER>
__device__ __forceinline__ void walk_u(const T *h, T *g, const T *tab, int kind, int ne_rt) {
    using D = Dims<P>;
    constexpr int TS = D::TS, PBP = D::PBP, RS = D::RS;
    constexpr int NEM = pat_nemax(P, PAT), NF = NEM + P;
    const int ne = PAT == 1 ? NEM : ne_rt;
    // periodic tile: every element's two points have the band rows of the
    // tile's first two points, read once
    T wr[2][P + 1];
    if constexpr (PER) {
        load_band<P>(tab + kind * PBP, wr[0]);
        load_band<P>(tab + TS + kind * PBP, wr[1]);
    }
    T a0[NF], a1[NF];
#pragma unroll
    for (int f = 0; f < NF; f++) a0[f] = a1[f] = T(0);
#pragma unroll
    for (int e = 0; e < NEM; e++) {
        if (e < ne) {
            const int q0 = pat_q0(P, PAT, e);
            const int np = PAT == 2 ? (e == 0 ? P + 1 : 2) : (PAT == 3 && e == ne - 1 ? P + 2 : 2);
#pragma unroll
            for (int pt = 0; pt < P + 2; pt++) {
                if (pt < np) {
                    const int q = q0 + pt;
                    T w[P + 1];
                    if constexpr (PER) {
#pragma unroll
                        for (int m = 0; m <= P; m++) w[m] = wr[pt & 1][m];
                    } else {
                        load_band<P>(tab + q * TS + kind * PBP, w);
                    }
                    const T x0 = h[q], x1 = h[kTQ + q];
#pragma unroll
                    for (int m = 0; m <= P; m++) {
                        a0[e + m] += w[m] * x0;
                        a1[e + m] += w[m] * x1;
                    }
                }
            }
            g[27 * e] = a0[e];
            g[RS + 27 * e] = a1[e];
        }
    }
#pragma unroll
    for (int f = 1; f < NF; f++)
        if (f >= ne && f < ne + P) {
            g[27 * f] = a0[f];
            g[RS + 27 * f] = a1[f];
        }
}

template <class T, int P>
__device__ __forceinline__ void walk_u_generic(const T *h, T *g, const T *tab, int kind,
                                               const int *rel, int nq) {
    using D = Dims<P>;
    constexpr int TS = D::TS, PBP = D::PBP, RS = D::RS;
    T a0[P + 1], a1[P + 1];
#pragma unroll
    for (int m = 0; m <= P; m++) a0[m] = a1[m] = T(0);
    int cur = 0;
    for (int q = 0; q < nq; q++) {
        const int r = rel[q];
        if (r != cur) {
            g[27 * cur] = a0[0];
            g[RS + 27 * cur] = a1[0];
#pragma unroll
            for (int m = 0; m < P; m++) {
                a0[m] = a0[m + 1];
                a1[m] = a1[m + 1];
            }
            a0[P] = a1[P] = T(0);
            cur = r;
        }
        T w[P + 1];
        load_band<P>(tab + q * TS + kind * PBP, w);
        const T x0 = h[q], x1 = h[kTQ + q];
#pragma unroll
        for (int m = 0; m <= P; m++) {
            a0[m] += w[m] * x0;
            a1[m] += w[m] * x1;
        }
    }
#pragma unroll
    for (int m = 0; m <= P; m++) {
        g[27 * (cur + m)] = a0[m];
        g[RS + 27 * (cur + m)] = a1[m];
    }
}

// Backward v of the three channels (i,k,l=0..2) of two fu columns (fu and
// fu + dfu: one pair of band rows serves both), merged on the w key:
// kp[fv] = (sum wa g0 + wb g1, sum wa g2), wa at table row ka (trial
// l != v), wb at ka+1 (trial l == v).  G of row qv of the tile lives in the
// block of warp qv/2: gb + (qv/2)*GP + (qv%2)*RS + l (second column: + 27
// dfu); the pairs of K are NFM * 18 apart from one fv to the next (second
// column: + 18 dfu).  two = false: the second column is not stored.  NC = 1:
// one column only (FP64, whose registers do not hold two).
template <class T, int P, int PAT, int NC, bool PER>
__device__ __forceinline__ void walk_v(const T *gb, T *kp, int dfu, bool two, const T *tab, int ka,
                                       int ne_rt) {
    using D = Dims<P>;
    constexpr int PBP = D::PBP, TS = D::TS, NEM = pat_nemax(P, PAT, kTV), NF = NEM + P;
    constexpr int KS = D::NFM * 18, RS = D::RS, GP = D::GP;
    const int ne = PAT == 1 ? NEM : ne_rt;
    // periodic tile: the band rows of the tile's first two points, read once
    T war[2][P + 1], wbr[2][P + 1];
    if constexpr (PER) {
        load_band<P>(tab + ka * PBP, war[0]);
        load_band<P>(tab + (ka + 1) * PBP, wbr[0]);
        load_band<P>(tab + TS + ka * PBP, war[1]);
        load_band<P>(tab + TS + (ka + 1) * PBP, wbr[1]);
    }
    const int dg = 27 * dfu;
    T *const kp1 = kp + 18 * dfu;
    T A0[NF], A1[NF], B0[NF], B1[NF];
#pragma unroll
    for (int f = 0; f < NF; f++) A0[f] = A1[f] = B0[f] = B1[f] = T(0);
#pragma unroll
    for (int e = 0; e < NEM; e++) {
        if (e < ne) {
            const int q0 = pat_q0(P, PAT, e);
            const int np = PAT == 2 ? (e == 0 ? P + 1 : 2) : (PAT == 3 && e == ne - 1 ? P + 2 : 2);
#pragma unroll
            for (int pt = 0; pt < P + 2; pt++) {
                if (pt < np) {
                    const int q = q0 + pt;
                    T wa[P + 1], wb[P + 1];
                    if constexpr (PER) {
#pragma unroll
                        for (int m = 0; m <= P; m++) {
                            wa[m] = war[pt & 1][m];
                            wb[m] = wbr[pt & 1][m];
                        }
                    } else {
                        load_band<P>(tab + q * TS + ka * PBP, wa);
                        load_band<P>(tab + q * TS + (ka + 1) * PBP, wb);
                    }
                    const T *g = gb + (q >> 1) * GP + (q & 1) * RS;
                    const T x0 = g[0], x1 = g[1], x2 = g[2];
#pragma unroll
                    for (int m = 0; m <= P; m++) {
                        A0[e + m] += wa[m] * x0 + wb[m] * x1;
                        A1[e + m] += wa[m] * x2;
                    }
                    if constexpr (NC == 2) {
                        const T y0 = g[dg], y1 = g[dg + 1], y2 = g[dg + 2];
#pragma unroll
                        for (int m = 0; m <= P; m++) {
                            B0[e + m] += wa[m] * y0 + wb[m] * y1;
                            B1[e + m] += wa[m] * y2;
                        }
                    }
                }
            }
            store_pair(kp + e * KS, A0[e], A1[e]);
            if (NC == 2 && two) store_pair(kp1 + e * KS, B0[e], B1[e]);
        }
    }
#pragma unroll
    for (int f = 1; f < NF; f++)
        if (f >= ne && f < ne + P) {
            store_pair(kp + f * KS, A0[f], A1[f]);
            if (NC == 2 && two) store_pair(kp1 + f * KS, B0[f], B1[f]);
        }
}

template <class T, int P, int NC>
__device__ __forceinline__ void walk_v_generic(const T *gb, T *kp, int dfu, bool two, const T *tab,
                                               int ka, const int *rel, int nq) {
    using D = Dims<P>;
    constexpr int PBP = D::PBP, TS = D::TS, KS = D::NFM * 18, RS = D::RS, GP = D::GP;
    const int dg = 27 * dfu;
    T *const kp1 = kp + 18 * dfu;
    T A0[P + 1], A1[P + 1], B0[P + 1], B1[P + 1];
#pragma unroll
    for (int m = 0; m <= P; m++) A0[m] = A1[m] = B0[m] = B1[m] = T(0);
    int cur = 0;
    for (int q = 0; q < nq; q++) {
        const int r = rel[q];
        if (r != cur) {
            store_pair(kp + cur * KS, A0[0], A1[0]);
            if (NC == 2 && two) store_pair(kp1 + cur * KS, B0[0], B1[0]);
#pragma unroll
            for (int m = 0; m < P; m++) {
                A0[m] = A0[m + 1];
                A1[m] = A1[m + 1];
                B0[m] = B0[m + 1];
                B1[m] = B1[m + 1];
            }
            A0[P] = A1[P] = B0[P] = B1[P] = T(0);
            cur = r;
        }
        T wa[P + 1], wb[P + 1];
        load_band<P>(tab + q * TS + ka * PBP, wa);
        load_band<P>(tab + q * TS + (ka + 1) * PBP, wb);
        const T *g = gb + (q >> 1) * GP + (q & 1) * RS;
        const T x0 = g[0], x1 = g[1], x2 = g[2];
#pragma unroll
        for (int m = 0; m <= P; m++) {
            A0[m] += wa[m] * x0 + wb[m] * x1;
            A1[m] += wa[m] * x2;
        }
        if constexpr (NC == 2) {
            const T y0 = g[dg], y1 = g[dg + 1], y2 = g[dg + 2];
#pragma unroll
            for (int m = 0; m <= P; m++) {
                B0[m] += wa[m] * y0 + wb[m] * y1;
                B1[m] += wa[m] * y2;
            }
        }
    }
#pragma unroll
    for (int m = 0; m <= P; m++) {
        store_pair(kp + (cur + m) * KS, A0[m], A1[m]);
        if (NC == 2 && two) store_pair(kp1 + (cur + m) * KS, B0[m], B1[m]);
    }
}

__device__ __forceinline__ int relu_last_plus1(const int *elem, int q0, int nq, int f0) {
    return elem[q0 + nq - 1] - f0 + 1;
}

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
    const int *treg[2];        // tile pattern (walk_u): 1 regular full, 4 regular, 2 first, 3 last, 0 other
    int ntile[2];
    const int *elem[3];        // element owning each point
    const T *band[3];          // [nqp][6][round4(p+1)]: B0 B1 W00 W01 W10 W11
    const int *wq0;            // first w point of each element (nel_w + 1)
    int nqw;                   // w points
    const int4 *seg;           // (tile, e_begin, e_end, -)
    const int *cta_seg;        // segments of a CTA
    int nfun[3];
    int64_t ncp;
    int cmask[3];
    int *err;                  // set to 1 when a bounded wait gave up
    int wait_tries;            // polls of a wait for a coefficient copy
};

template <class T, int P>
__global__ void __launch_bounds__(kThreads, kCtasPerSm) k_wq_apply_stream(StreamArgs<T> a) {
    using D = Dims<P>;
    constexpr int PB = D::PB, PBP = D::PBP, NFM = D::NFM, CPT = D::CPT;
    constexpr int TS = D::TS, GP = D::GP, ZHP = D::ZHP;
    // FP32: each plane's coefficient block is brought into shared memory by a
    // bulk copy issued one plane ahead; FP64 reads it from HBM directly
    constexpr bool kStaged = sizeof(T) == 4;
    if (a.done && *a.done) return;
    extern __shared__ __align__(16) unsigned char smraw[];
    T *const sm = reinterpret_cast<T *>(smraw);
    T *const RY = sm;
    T *const RZH = sm + D::OFF_ZH;   // per warp: Z, then h; K (all warps) after G
    T *const RG = sm + D::OFF_G;     // per warp: G
    T *const tabu = sm + D::OFF_TAB;
    T *const tabv = tabu + D::TAB;
    T *const cbuf = sm + D::TOTAL;
    int *const relu = reinterpret_cast<int *>(sm + D::TOTAL + (kStaged ? D::CB : 0));
    int *const relv = relu + kTQ;
    uint64_t *const bar = reinterpret_cast<uint64_t *>(relv + kTV);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    uint32_t phase = 0;
    if constexpr (kStaged) {
        if (tid == 0) mbar_init(bar);
        __syncthreads();
    }
    const int64_t plane = (int64_t)a.nfun[0] * a.nfun[1];

    for (int si = a.cta_seg[blockIdx.x]; si < a.cta_seg[blockIdx.x + 1]; si++) {
        const int4 sg = a.seg[si];
        const int tu = sg.x % a.ntile[0], tv = sg.x / a.ntile[0];
        const int qu0 = a.tq0[0][tu], nqu = a.tnq[0][tu];
        const int qv0 = a.tq0[1][tv], nqv = a.tnq[1][tv];
        // pattern in bits 0..2, bit 3: periodic band rows (pattern 1 or 4)
        const int patu = a.treg[0][tu] & 7, patv = a.treg[1][tv] & 7;
        const bool peru = (a.treg[0][tu] & 8) != 0, perv = (a.treg[1][tv] & 8) != 0;
        const bool regu = patu == 1 || patu == 4, regv = patv == 1 || patv == 4;
        const int fu0 = a.elem[0][qu0], fv0 = a.elem[1][qv0];
        const int nfu = a.elem[0][qu0 + nqu - 1] + PB - fu0;
        const int nfv = a.elem[1][qv0 + nqv - 1] + PB - fv0;
        const int neu = relu_last_plus1(a.elem[0], qu0, nqu, fu0);   // elements of the tile
        const int nev = relu_last_plus1(a.elem[1], qv0, nqv, fv0);
        const int npts = nqu * nqv;
        const T *coef_t = a.coef + a.tile_off[sg.x];
        const int pstride = a.tile_pstride[sg.x];
        const int pbytes = npts * kWQCoef * (int)sizeof(T);
        const int nrow = min(2, nqv - 2 * warp);   // rows of this warp (may be <= 0)

        __syncthreads();   // the previous segment is done with the tables
        for (int i = tid; i < kTQ * 6 * PBP; i += kThreads) {
            const int q = i / (6 * PBP), r = i - q * (6 * PBP);
            tabu[q * TS + r] = q < nqu ? a.band[0][(size_t)(qu0 + q) * 6 * PBP + r] : T(0);
            if (q < kTV) tabv[q * TS + r] = q < nqv ? a.band[1][(size_t)(qv0 + q) * 6 * PBP + r] : T(0);
        }
        if (tid < kTQ) relu[tid] = tid < nqu ? a.elem[0][qu0 + tid] - fu0 : 0;
        if (tid < kTV) relv[tid] = tid < nqv ? a.elem[1][qv0 + tid] - fv0 : 0;
        const uint32_t cbytes = (uint32_t)((npts * kWQCoef * (int)sizeof(T) + 15) & ~15);
        if constexpr (kStaged) {
            if (tid == 0) bulk_load(cbuf, coef_t + (int64_t)a.wq0[sg.y] * pstride, cbytes, bar);
        }
        // stage D thread: (ik, fu) and (ik, fu + nfp), the nine ik fastest
        // (FP64: one fu, nfp = nfu)
        constexpr int kDC = sizeof(T) == 4 ? 2 : 1;
        const int nfp = kDC == 2 ? (nfu + 1) >> 1 : nfu;
        const bool d_act = tid < 9 * nfp;
        const int d_fu = d_act ? tid / 9 : 0, d_ik = d_act ? tid - 9 * d_fu : 0;
        const bool d_two = d_fu + nfp < nfu;

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
        // ---- A: forward w of plane qa into RY
        auto stage_a = [&](int qa) {
            const T *bwa = a.band[2] + (size_t)qa * 6 * PBP;
            T b0[PB], b1[PB];
            load_band<P>(bwa, b0);
            load_band<P>(bwa + PBP, b1);
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
                RY[c * D::NFV * NFM + k] = y0;
                RY[(3 + c) * D::NFV * NFM + k] = y1;
            }
        };
#pragma unroll
        for (int cc = 0; cc < CPT; cc++)
#pragma unroll
            for (int m = 0; m <= P; m++) x[cc][m] = load_x(cc, sg.y + m);
        stage_a(a.wq0[sg.y]);
        if (!kStaged) {
            const char *p0 = reinterpret_cast<const char *>(coef_t + (int64_t)a.wq0[sg.y] * pstride);
            for (int off = tid * 128; off < pbytes; off += kThreads * 128) prefetch_l2(p0 + off);
        }

        for (int e = sg.y; e < sg.z; e++) {
#pragma unroll
            for (int cc = 0; cc < CPT; cc++) acc[cc][P] = T(0);
            const int qw_end = a.wq0[e + 1];
            for (int qw = a.wq0[e]; qw < qw_end; qw++) {
                const T *bw = a.band[2] + (size_t)qw * 6 * PBP;
                if (!kStaged && qw + 1 < a.nqw) {
                    // FP64 reads the coefficients straight from HBM: prefetch
                    // the next plane into L2 (FP32 stages it with a bulk copy)
                    const char *pn = reinterpret_cast<const char *>(coef_t + (int64_t)(qw + 1) * pstride);
                    for (int off = tid * 128; off < pbytes; off += kThreads * 128) prefetch_l2(pn + off);
                }
                if constexpr (kStaged) {
                    // this plane's coefficient block has landed in shared memory
                    const bool ok = mbar_wait(bar, phase, a.wait_tries);
                    if (__syncthreads_or(!ok)) {
                        if (tid == 0) atomicOr(a.err, 1);
                        // let the copy still in flight land (default bound)
                        mbar_wait(bar, phase, kWaitTries);
                        return;
                    }
                    phase ^= 1;
                } else {
                    __syncthreads();
                }
                if (nrow > 0) {
                    T *const zh = RZH + warp * ZHP;
                    T *const gp = RG + warp * GP;
                    // ---- B: forward v of this warp's rows, lane (row, fu)
                    {
                        const int row = lane >> 4, fu = lane & 15;
                        if (row < nrow && fu < nfu) {
                            const int qv = 2 * warp + row;
                            const int rv = regv ? (qv >> 1) : relv[qv];
                            T b0[PB], b1[PB];
                            load_band<P>(tabv + qv * TS, b0);
                            load_band<P>(tabv + qv * TS + PBP, b1);
#pragma unroll
                            for (int c = 0; c < 3; c++) {
                                const T *y0 = RY + (c * D::NFV + rv) * NFM + fu;
                                const T *y1 = RY + ((3 + c) * D::NFV + rv) * NFM + fu;
                                T z0 = 0, z1 = 0, z2 = 0;
#pragma unroll
                                for (int m = 0; m < PB; m++) {
                                    const T a0 = y0[m * NFM], a1 = y1[m * NFM];
                                    z0 += b0[m] * a0;
                                    z1 += b1[m] * a0;
                                    z2 += b0[m] * a1;
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
                        T f[3][3];
                        if (act) {
                            const int ru = regu ? (qu >> 1) : relu[qu];
                            T b0[PB], b1[PB];
                            load_band<P>(tabu + qu * TS, b0);
                            load_band<P>(tabu + qu * TS + PBP, b1);
#pragma unroll
                            for (int l = 0; l < 3; l++)
#pragma unroll
                                for (int j = 0; j < 3; j++) {
                                    const T *zr = zh + (l * 3 + j) * (2 * NFM) + row * NFM + ru;
                                    T v = 0;
#pragma unroll
                                    for (int m = 0; m < PB; m++) v += (l == 0 ? b1[m] : b0[m]) * zr[m];
                                    f[l][j] = v;
                                }
                        }
                        __syncwarp();   // the warp's Z is read; h takes its place
                        if (act) {
                            const int pt = (2 * warp + row) * nqu + qu;
                            if constexpr (kStaged) {
                                // point-major block in shared memory: 45 values per point
                                const T *cp = cbuf + pt * kWQCoef;
                                T h[27];
#pragma unroll
                                for (int ch = 0; ch < 27; ch++) h[ch] = T(0);
#pragma unroll
                                for (int I = 0; I < 9; I++) {
#pragma unroll
                                    for (int J = I; J < 9; J++) {
                                        const T sv = cp[sym9(I, J)];
                                        const int i = I / 3, k = I % 3, j = J / 3, l = J % 3;
                                        h[(i * 3 + k) * 3 + l] += sv * f[l][j];
                                        if (I != J) h[(j * 3 + l) * 3 + k] += sv * f[k][i];
                                    }
                                }
#pragma unroll
                                for (int ch = 0; ch < 27; ch++) zh[ch * kHS + row * kTQ + qu] = h[ch];
                            } else {
                                // entry-major block in HBM, one output component at a
                                // time (the symmetric partner entries hit L1)
                                const T *cp = coef_t + (int64_t)qw * pstride + pt;
#pragma unroll
                                for (int i = 0; i < 3; i++) {
#pragma unroll
                                    for (int k = 0; k < 3; k++) {
                                        T h0 = 0, h1 = 0, h2 = 0;
#pragma unroll
                                        for (int J = 0; J < 9; J++) {
                                            const T sv = __ldg(cp + sym9(3 * i + k, J) * npts);
                                            const int j = J / 3, l = J % 3;
                                            if (l == 0) h0 += sv * f[0][j];
                                            else if (l == 1) h1 += sv * f[1][j];
                                            else h2 += sv * f[2][j];
                                        }
                                        const int ch = (i * 3 + k) * 3;
                                        zh[(ch + 0) * kHS + row * kTQ + qu] = h0;
                                        zh[(ch + 1) * kHS + row * kTQ + qu] = h1;
                                        zh[(ch + 2) * kHS + row * kTQ + qu] = h2;
                                    }
                                }
                            }
                        }
                    }
                    __syncwarp();
                    // ---- G: backward u, lane = channel (i,k,l), both rows of the warp
                    // (with one row the second walks stale values that nothing reads)
                    if (lane < 27) {
                        const int ch = lane;
                        const int k = (ch / 3) % 3, l = ch % 3;
                        const int kind = 2 + 2 * (k == 0) + (l == 0);   // W_{[k==u][l==u]}
                        const T *hr = zh + ch * kHS;
                        T *gr = gp + ch;
                        switch (patu) {
                            case 1:
                                if (peru) walk_u<T, P, 1, true>(hr, gr, tabu, kind, neu);
                                else walk_u<T, P, 1, false>(hr, gr, tabu, kind, neu);
                                break;
                            case 4:
                                if (peru) walk_u<T, P, 4, true>(hr, gr, tabu, kind, neu);
                                else walk_u<T, P, 4, false>(hr, gr, tabu, kind, neu);
                                break;
                            case 2: walk_u<T, P, 2, false>(hr, gr, tabu, kind, neu); break;
                            case 3: walk_u<T, P, 3, false>(hr, gr, tabu, kind, neu); break;
                            default: walk_u_generic<T, P>(hr, gr, tabu, kind, relu, nqu);
                        }
                    }
                }
                __syncthreads();
                if constexpr (kStaged) {
                    // every warp is done with the block: bring in the next plane's
                    if (tid == 0 && qw + 1 < a.wq0[sg.z])
                        bulk_load(cbuf, coef_t + (int64_t)(qw + 1) * pstride, cbytes, bar);
                }
                // ---- D: backward v, thread (i, k) x two fu; K aliases the Z/h parts
                if (d_act) {
                    const int ik = d_ik, fu = d_fu;
                    const int ka = 2 + 2 * (ik % 3 == 1);   // W_{[k==v], 0}
                    const T *gb = RG + fu * 27 + ik * 3;
                    T *kp = RZH + (fu * 9 + ik) * 2;
                    switch (patv) {
                        case 1:
                            if (perv) walk_v<T, P, 1, kDC, true>(gb, kp, d_two ? nfp : 0, d_two, tabv, ka, nev);
                            else walk_v<T, P, 1, kDC, false>(gb, kp, d_two ? nfp : 0, d_two, tabv, ka, nev);
                            break;
                        case 4:
                            if (perv) walk_v<T, P, 4, kDC, true>(gb, kp, d_two ? nfp : 0, d_two, tabv, ka, nev);
                            else walk_v<T, P, 4, kDC, false>(gb, kp, d_two ? nfp : 0, d_two, tabv, ka, nev);
                            break;
                        case 2: walk_v<T, P, 2, kDC, false>(gb, kp, d_two ? nfp : 0, d_two, tabv, ka, nev); break;
                        case 3: walk_v<T, P, 3, kDC, false>(gb, kp, d_two ? nfp : 0, d_two, tabv, ka, nev); break;
                        default: walk_v_generic<T, P, kDC>(gb, kp, d_two ? nfp : 0, d_two, tabv, ka, relv, nqv);
                    }
                }
                // ---- A of the next plane, beside D (RY is free once B is done);
                // at an element's last plane the u ring advances first
                if (qw + 1 < a.wq0[sg.z]) {
                    if (qw + 1 == qw_end) {
#pragma unroll
                        for (int cc = 0; cc < CPT; cc++) {
#pragma unroll
                            for (int m = 0; m < P; m++) x[cc][m] = x[cc][m + 1];
                            x[cc][P] = load_x(cc, e + 1 + P);
                        }
                    }
                    stage_a(qw + 1);
                }
                __syncthreads();
                // ---- E: backward w into the register ring of output planes
                {
                    T w00[PB], w01[PB], w10[PB], w11[PB];
                    load_band<P>(bw + 2 * PBP, w00);
                    load_band<P>(bw + 3 * PBP, w01);
                    load_band<P>(bw + 4 * PBP, w10);
                    load_band<P>(bw + 5 * PBP, w11);
#pragma unroll
                    for (int cc = 0; cc < CPT; cc++) {
                        if (!(cinfo[cc] & 4)) continue;
                        const int i = cinfo[cc] & 3, kidx = cinfo[cc] >> 3;
                        const T *kb = RZH + (kidx * 9 + i * 3) * 2;   // K[fv][fu][ik][2]
                        T k00, k01, k10, k11, k20, k21;
                        load_pair(kb, k00, k01);
                        load_pair(kb + 2, k10, k11);
                        load_pair(kb + 4, k20, k21);
                        const T s00 = k00 + k10, s01 = k01 + k11;
#pragma unroll
                        for (int m = 0; m < PB; m++)
                            acc[cc][m] += w00[m] * s00 + w01[m] * s01 + w10[m] * k20 + w11[m] * k21;
                    }
                }
                // no barrier: the next B writes the Z/h parts after the
                // barrier that opens the next plane
            }
            // output plane e is complete for this element range
#pragma unroll
            for (int cc = 0; cc < CPT; cc++) {
                retire(cc, e, acc[cc][0]);
#pragma unroll
                for (int m = 0; m < P; m++) acc[cc][m] = acc[cc][m + 1];
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
// Tiles of whole elements with at most maxq points (kTQ along u, kTV along
// v): the first and last tiles take the boundary elements (which own more
// than two points) and as many neighbours as fit; the elements between (two
// points each) are split into balanced regular tiles of at most maxq / 2
// elements.
static void make_tiles(const std::vector<int> &elem_q0, int nel, std::vector<int> &q0,
                       std::vector<int> &nq, std::vector<int> &reg, int maxq) {
    const int maxe = maxq / 2;
    q0.clear();
    nq.clear();
    reg.clear();
    auto pts = [&](int a, int b) { return elem_q0[b] - elem_q0[a]; };   // elements [a, b)
    int first_end = 1;
    while (first_end < nel && pts(0, first_end + 1) <= maxq) first_end++;
    int last_begin = nel;
    if (first_end < nel) {
        last_begin = nel - 1;
        while (last_begin - 1 >= first_end && pts(last_begin - 1, nel) <= maxq) last_begin--;
    }
    // walk pattern of a tile (see walk_u): 1 all elements own two points and
    // the tile is full, 4 all own two, 2 only the first element of the patch
    // differs, 3 only the last
    auto add = [&](int a, int b) {
        bool inner2 = true;   // elements other than the patch's first / last own 2
        for (int e = a; e < b; e++)
            if (e != 0 && e != nel - 1) inner2 = inner2 && (pts(e, e + 1) == 2);
        const bool has_first = a == 0, has_last = b == nel;
        int pat = 0;
        if (inner2 && !has_first && !has_last) pat = b - a == maxe ? 1 : 4;
        else if (inner2 && has_first && !has_last) pat = 2;
        else if (inner2 && has_last && !has_first) pat = 3;
        q0.push_back(elem_q0[a]);
        nq.push_back(pts(a, b));
        reg.push_back(pat);
    };
    add(0, first_end);
    const int nmid = last_begin - first_end;
    if (nmid > 0) {
        const int t = (nmid + maxe - 1) / maxe;
        for (int k = 0; k < t; k++)
            add(first_end + (int)((int64_t)nmid * k / t), first_end + (int)((int64_t)nmid * (k + 1) / t));
    }
    if (last_begin < nel) add(last_begin, nel);
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
        const int pt = (qv - tq0v[tv]) * tnqu[tu] + (qu - tq0u[tu]);
        const int64_t pbase = tile_off[t] + (int64_t)qw * tile_pstride[t];
        // FP32 blocks point-major (staged whole into shared memory), FP64
        // blocks entry-major (read straight from HBM, coalesced per entry)
        if (sizeof(T) == 4)
            for (int e = 0; e < kWQCoef; e++) dst[pbase + (int64_t)pt * kWQCoef + e] = src[sbase + e * nqb];
        else
            for (int e = 0; e < kWQCoef; e++) dst[pbase + (int64_t)e * nqt + pt] = src[sbase + e * nqb];
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
    const int P = op->p[0], PBP = (P + 1 + 3) / 4 * 4;
    std::vector<int> elem_q0[3];
    std::vector<double> band_uv[2];
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
        std::vector<double> band((size_t)nq * 6 * PBP, 0.0);
        for (int q = 0; q < nq; q++)
            for (int k = 0; k < 6; k++)
                for (int f = 0; f < R[d].nfun; f++) {
                    const double v = (*M[k])[(size_t)f * nq + q];
                    const int m = f - elem[q];
                    if (m >= 0 && m <= P) band[((size_t)q * 6 + k) * PBP + m] = v;
                    else YETI_CHECK(v == 0.0, YETI_EUNSUPPORTED,
                                    "WQ streaming: rule entry outside the band (dir %d, f %d, q %d)",
                                    d, f, q);
                }
        std::vector<float> bandf(band.begin(), band.end());
        if (d < 2) band_uv[d] = band;
        YETI_TRY(upload_vec(ctx, st.elem[d], elem));
        YETI_TRY(upload_vec(ctx, st.band64[d], band));
        YETI_TRY(upload_vec(ctx, st.band32[d], bandf));
    }
    YETI_TRY(upload_vec(ctx, st.wq0, elem_q0[2]));
    std::vector<int> tq0[2], tnq[2], treg[2];
    for (int d = 0; d < 2; d++) {
        make_tiles(elem_q0[d], op->nel[d], tq0[d], tnq[d], treg[d], d == 0 ? kTQ : kTV);
        // a regular tile whose points' band rows repeat, bit for bit, those
        // of its first two points (interior elements of a uniform knot
        // vector) is flagged (bit 3): its walks read two rows once
        const size_t row = (size_t)6 * PBP;
        for (size_t t = 0; t < treg[d].size(); t++) {
            if (treg[d][t] != 1 && treg[d][t] != 4) continue;
            const double *b0 = band_uv[d].data() + (size_t)tq0[d][t] * row;
            bool per = tnq[d][t] >= 2;
            for (int q = 2; per && q < tnq[d][t]; q++)
                per = std::memcmp(b0 + (size_t)q * row, b0 + (size_t)(q & 1) * row,
                                  row * sizeof(double)) == 0;
            if (per) treg[d][t] |= 8;
        }
        YETI_TRY(upload_vec(ctx, st.treg[d], treg[d]));
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
    YETI_TRY(st.err.alloc(ctx, sizeof(int)));
    YETI_CUDA(cudaMemsetAsync(st.err.ptr, 0, sizeof(int), ctx->stream));

    // kernels and grid
    YETI_TRY(stream_prepare_kernels(op));
    int nsm = 0;
    YETI_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, ctx->device));
    // segments: (tile, element range) cut from the tile-major sequence so
    // that every CTA gets about the same number of tile planes (a plane of a
    // narrow tile costs a CTA about as much as a full one: the same stages,
    // barriers and walks, with lanes idle)
    for (int which = 0; which < 2; which++) {
        // item (t, e) goes to CTA floor(work before it * ncta / total work);
        // consecutive items of one CTA and one tile form a segment
        const int64_t total = (int64_t)ntiles * nqw;
        const int64_t nitems = (int64_t)ntiles * op->nel[2];
        const int ncta = (int)std::max<int64_t>(
            1, std::min<int64_t>((int64_t)nsm * st.per_sm[which], nitems));
        std::vector<int4> seg;
        std::vector<int> cta_seg(ncta + 1, 0);
        int64_t before = 0;
        int last_cta = -1;
        for (int t = 0; t < ntiles; t++) {
            for (int e = 0; e < op->nel[2]; e++) {
                const int c = (int)std::min<int64_t>(ncta - 1, before * ncta / total);
                before += elem_q0[2][e + 1] - elem_q0[2][e];
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
        a.treg[d] = st.treg[d].as<int>();
        a.ntile[d] = st.ntile[d];
    }
    for (int d = 0; d < 3; d++) {
        a.elem[d] = st.elem[d].as<int>();
        a.band[d] = (f64 ? st.band64[d] : st.band32[d]).template as<T>();
        a.nfun[d] = op->n[d];
        a.cmask[d] = op->cmask[d];
    }
    a.wq0 = st.wq0.as<int>();
    a.err = st.err.as<int>();
    a.wait_tries = st.wait_tries;
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

int wq_stream_check(yeti_wq_op *op) {
    if (!op->st.active) return YETI_OK;
    int h = 0;
    YETI_CUDA(cudaMemcpyAsync(&h, op->st.err.ptr, sizeof(int), cudaMemcpyDeviceToHost, op->ctx->stream));
    YETI_CUDA(cudaStreamSynchronize(op->ctx->stream));
    if (h) {
        YETI_CUDA(cudaMemsetAsync(op->st.err.ptr, 0, sizeof(int), op->ctx->stream));
        set_error("WQ apply: a bounded wait for a coefficient copy gave up; results are invalid");
        return YETI_ETIMEDOUT;
    }
    return YETI_OK;
}

template int wq_stream_apply<float>(yeti_wq_op *, const float *, float *, const int *, cudaStream_t);
template int wq_stream_apply<double>(yeti_wq_op *, const double *, double *, const int *,
                                     cudaStream_t);

}  // namespace yeti
