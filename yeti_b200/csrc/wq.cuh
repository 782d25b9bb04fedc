// Weighted-quadrature (WQ) elasticity on one NURBS patch: shared definitions
// of the host setup and the device kernels.
//
// Data layout in HBM
// ------------------
// The patch's tensor grid of WQ points is cut into element blocks
// (blk_u x blk_v x blk_w).  Every point belongs to exactly one element (the
// element whose half-open knot span holds it; the last element also owns
// the end point), hence to exactly one block.  Per-point operator data are
// stored block by block, entry-major inside a block:
//     coef[(qoff[b] * 48) + e * nq_b + local_point]
// so one CTA streams one contiguous chunk and consecutive threads read
// consecutive addresses.  The 45 entries are the upper triangle of the
// symmetric 9x9 coefficient S (row-major, index sym9).
// Vectors are component-major [c][iw][iv][iu].
#pragma once
#include <vector>

#include "common.cuh"
#include "wq_rule.h"

namespace yeti {

constexpr int kWQCoef = 45;
constexpr int kWQThreads = 256;

__host__ __device__ constexpr int sym9(int I, int J) {
    return I <= J ? I * 9 - I * (I - 1) / 2 + (J - I)
                  : J * 9 - J * (J - 1) / 2 + (I - J);
}

// Per block position along one direction: first element, element count,
// first owned point, owned point count.
struct BlkInfo {
    int e0, ne, q0, nq;
};

// One direction as seen by the kernels.
struct WQAxis {
    int p, nfun, nqp, nb;   // degree, functions, points, blocks
    int NF, NQ;             // max functions / points of a block (tile dims)
    const BlkInfo *blk;     // nb entries
};

// Everything a kernel needs about the patch (passed by value).
template <class T>
struct WQView {
    WQAxis ax[3];
    const T *tiles[3];      // [nb][6][NF][NQ]: B0 B1 W00 W01 W10 W11
    const int64_t *qoff;    // first point (block-tiled numbering) of a block
    const T *coef;          // [nqp_total * 45] block-tiled, entry-major
    int cmask[3];           // clamped faces per component (bit f)
    int64_t ncp;
};

}  // namespace yeti

struct yeti_wq_op;
namespace yeti {

// Tables of the streaming apply kernel (degrees 2..5, wq_stream.cu); index
// [0] / [1] of grid, smem, seg: FP64 / FP32 kernel.
struct WQStreamPlan {
    bool active = false;     // coefficients are in the streaming layout
    int ntile[2] = {0, 0};   // (u, v) tiles
    int grid[2] = {0, 0};
    int per_sm[2] = {0, 0};
    size_t smem[2] = {0, 0};
    int64_t ncoef = 0;
    DevBuf elem[3], band64[3], band32[3], wq0, tq0[2], tnq[2], treg[2];
    DevBuf tile_off, tile_pstride, seg[2], cta_seg[2];
    DevBuf err;              // int: a kernel's bounded wait gave up
    int wait_tries = 1 << 16;   // polls of a wait for a coefficient copy
};

// Device-side scalars of one CG solve (wq_pcg.cu); the fast-diagonalisation
// kernels finish the r.z reduction of an iteration into them.
struct CGScal {
    double rz, pAp, alpha, beta, rr, bb, tol2, scale;
    double pause2;         // stop a chunk once rr <= pause2 (0: never)
    int done, iter, breakdown, maxit;
    int paused;            // done was set by pause2, not by the tolerance
    unsigned int ticket;   // blocks of a fused reduction that have finished
};

// Fast-diagonalisation preconditioner (wq_fd.cu): per displacement component
// c, the separable operator sum_d a[c][d] K_d (x) M (x) M on the component's
// free box, inverted through the generalised eigenpairs K_d U = M_d U Lambda
// of the 1-D WQ matrices; optionally scaled by sqrt(diag(P) / diag(K)).
struct WQFdPlan {
    int variant = -1;          // YETI_PCG_FD bits it was built for (-1: none)
    int lo[3][3], m[3][3];     // free box per [component][direction]
    int64_t goff[3][3];        // U (fwd) at goff, U^T (bwd) at goff + m*m
    int64_t doff[3][3];        // a[c][d] * lambda_d
    bool scaled = false;
    DevBuf g64, g32, d64, d32, s64, s32;   // matrices, eigenvalues, scaling
    DevBuf t64, t32;           // two intermediate vectors
    DevBuf parts;              // partials of the r.z reduction
    int max_grid = 0;
};
// FD reduction modes of the last (u, backward) pass.
enum FdRed { FD_NONE = 0, FD_ITER = 1, FD_START = 2, FD_REPLACE = 3 };
// Build the plan for the YETI_PCG_FD* bits of `variant` (no-op when built).
int wq_fd_prepare(yeti_wq_op *op, int variant, bool f32);
// out = P in.  red FD_ITER: beta = r.z / rz, rz = r.z into *cg; FD_START:
// rz = r.z and p = z; FD_REPLACE: rz = r.z.  (in is r for those modes.)
// tmp (2 ndof) and parts (wq_fd_parts(op) doubles): the caller's
// workspace, for solves that share the operator concurrently; nullptr:
// the plan's own.  Launch-only (graph-capturable) once the plan exists.
template <class T>
int wq_fd_apply(yeti_wq_op *op, const T *in, T *out, const int *done, int red,
                T *p, CGScal *cg, cudaStream_t s, T *tmp = nullptr, double *parts = nullptr);
// Doubles of reduction partials one FD application needs.
int wq_fd_parts(const yeti_wq_op *op);

bool wq_stream_supported(const yeti_wq_op *op);
// Build the tile tables and work segments (after the 1-D rules).
int wq_stream_setup(yeti_wq_op *op, const WQRule1D R[3]);
// Move coef64 / coef32 from the element-block layout into the streaming
// layout (after every kernel that reads the element-block layout).
int wq_stream_permute(yeti_wq_op *op);
template <class T>
int wq_stream_apply(yeti_wq_op *op, const T *u, T *Ku, const int *done, cudaStream_t s);
// One FP64 preconditioned Krylov solve (CG or BiCGSTAB; Jacobi or fast
// diagonalisation) of a WQ operator (x0 = 0) that advances in
// chunks of iterations captured once in a CUDA graph, on its own stream and
// without host synchronisation: the serving loop launches a chunk, polls its
// event, and launches the next until the device-side scalars say done.  The
// workspace is allocated stream-ordered on that stream.
struct CgSolve {
    yeti_wq_op *op = nullptr;
    bool fd = false;             // fast-diagonalisation preconditioner
    bool bicg = false;           // BiCGSTAB instead of CG
    cudaStream_t stream = nullptr;
    void *dmem = nullptr;        // b x r z p Ap (6n doubles), partials, scalars
    void *host_scal = nullptr;   // pinned copy of the scalars (owned by the caller)
    cudaGraphExec_t chunk = nullptr;
    cudaEvent_t ev = nullptr;
    int nblk = 0;
    int chunk_iters = 0;         // iterations per chunk graph
    bool in_flight = false;
    int iterations = 0;
    double rel_residual = 0.0;   // true FP64 residual of the returned x
    void release();
    ~CgSolve() { release(); }
};
// Bytes of host memory the caller provides as host_scal (pinned).
size_t cgsolve_scal_bytes();
// The chunk graph is captured on `capture` when given (a stream no other
// thread enqueues into while it is captured), else on s.
// mode: YETI_PCG_BICGSTAB and the YETI_PCG_FD* bits (clear: Jacobi CG).
// chunk: iterations per chunk graph (0: the default, 16); the capture and
// instantiation cost and the iterations launched past convergence both grow
// with it, the host round trips shrink.
int cgsolve_begin(CgSolve &cs, yeti_wq_op *op, cudaStream_t s, void *host_scal,
                  const double *b_host, double rtol, int maxit,
                  cudaStream_t capture = nullptr, int mode = 0, int chunk = 0);
// Enqueue the next chunk (graph launch + event).
int cgsolve_launch(CgSolve &cs);
// *state: 0 a chunk is in flight, 1 chunk done and more iterations needed,
// 2 converged or iteration limit, 3 breakdown.
int cgsolve_poll(CgSolve &cs, int *state);
// Copy x to the host, compute the true residual, free the workspace.
// The work runs on `on` (after the solve's last chunk) when given, else on
// the solve's stream.
int cgsolve_finish(CgSolve &cs, double *x_host, cudaStream_t on = nullptr);

// YETI_ETIMEDOUT (and clears the flag) if a streaming kernel reported a
// bounded wait that gave up since the last check; synchronises the stream.
int wq_stream_check(yeti_wq_op *op);

// Enqueue Ku += K u (Ku must be zeroed by the caller) on stream s; prec
// YETI_PREC_F64 / F32 selects the operator data and the vector type.  done:
// optional device flag, the kernel returns at once when it is set.
int wq_apply_dev(yeti_wq_op *op, const void *u, void *Ku, int prec,
                 const int *done, cudaStream_t s);
}  // namespace yeti

// The operator object behind the opaque yeti_wq_op handle.
struct yeti_wq_op {
    yeti_ctx *ctx = nullptr;
    int p[3] = {0, 0, 0}, nel[3] = {0, 0, 0}, n[3] = {0, 0, 0};
    int nqp[3] = {0, 0, 0};
    int64_t ncp = 0, ndof = 0, nfree = 0, nqp_total = 0, nblocks = 0;
    int prec_mask = 0;
    int cmask[3] = {0, 0, 0};
    double E = 0, nu = 0;
    std::vector<yeti::BlkInfo> blk[3];
    int NF[3] = {0, 0, 0}, NQ[3] = {0, 0, 0};
    yeti::DevBuf blkd[3];
    yeti::DevBuf tiles64[3], tiles32[3], dtiles[3];
    yeti::DevBuf qoff;
    yeti::DevBuf coef64, coef32;
    yeti::DevBuf jw;        // |detJ| per point (FP64, block-tiled)
    yeti::DevBuf diag;      // diagonal (FP64, clamped dofs = 1)
    yeti::DevBuf dinv64, dinv32;
    yeti::DevBuf ws64, ws32, scal, parts;   // PCG workspaces
    yeti::WQStreamPlan st;
    yeti::DevBuf sdiag;     // per element block: sums of S[(c,d),(c,d)] (9)
    yeti::WQFdPlan fd;
    double setup_ms = 0.0;
    int64_t bytes_data = 0;
};
