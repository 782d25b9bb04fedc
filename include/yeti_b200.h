/*
 * yeti_b200 -- B200-native (sm_100a) implementation of YETI's U1 solid NURBS
 * path behind a C ABI.
 *
 * All entry points return an int status (YETI_OK == 0).  On failure,
 * yeti_last_error() returns a thread-local message.  Buffers are owned by the
 * caller.  A pointer argument documented as "mem" is host or device memory
 * according to the accompanying `mem` flag (YETI_MEM_HOST / YETI_MEM_DEVICE);
 * model descriptions are always host memory.  Contexts are independent: the
 * library keeps no global mutable state besides the thread-local error text.
 *
 * Reference interfaces replaced (paths relative to the reference's tree):
 *   yeti_assemble_u1_coo   <- stiffmtrx_elemstorage.sys_linmat_lindef_static
 *                             (src/yeti_iga/main/build_system_elemStorage.f90:24,
 *                              called at src/yeti_iga/overlay/iga_model.py:387-389)
 *   yeti_wq_*              <- iga_wq_mf assembly/solver f2py modules used by
 *                             ThermoMechaIGA/pysrc/lib/fortran_mf_wq.py:29-560
 *                             (mf_wq_get_ku_3d  src/yeti_iga/iga_wq_mf/fsrc/mf_wq_solver.f90:284,
 *                              wq_mf_cg_3d      mf_wq_solver.f90:642,
 *                              eval_mech_coefficient, jacobien_physicalposition_3d,
 *                              wq_get_force_3d  src/yeti_iga/iga_wq_mf/fsrc/wq_assembly.f90:52,233,1193)
 *   yeti_grad_lin_elast_work <- optim.gradadjointwork.gradlinelastwork_an
 *                             (src/yeti_iga/optim/gradtotalwork_fullAN.f90:17,
 *                              called at preprocessing/igaparametrization/OPT_modelling.py:474-477)
 */
#ifndef YETI_B200_H
#define YETI_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define YETI_OK 0
#define YETI_EINVAL (-1)        /* invalid argument / malformed model */
#define YETI_ECUDA (-2)         /* CUDA runtime error */
#define YETI_ENOMEM (-3)        /* device allocation failed or over budget */
#define YETI_EUNSUPPORTED (-4)  /* element type / load type not on this path */
#define YETI_ETIMEDOUT (-5)     /* bounded device wait gave up */
#define YETI_EBREAKDOWN (-6)    /* Krylov breakdown (p.Ap <= 0 or NaN) */
#define YETI_ENUMERIC (-7)      /* non-positive Jacobian / NaN in setup */
#define YETI_ENOTCONV (-8)      /* iteration limit reached before tolerance */

#define YETI_MEM_HOST 0
#define YETI_MEM_DEVICE 1

#define YETI_PREC_F64 0
#define YETI_PREC_F32 1

typedef struct yeti_ctx yeti_ctx;

/* Thread-local description of the last failure of a yeti_* call. */
const char *yeti_last_error(void);
/* Library version string. */
const char *yeti_version(void);
/* Number of CUDA kernels the library has launched in this process (no
 * counterpart in the reference: evidence that the device path ran). */
uint64_t yeti_kernel_launches(void);

/* Create a context on CUDA device `device`.  The context owns a stream
 * (non-blocking) unless yeti_ctx_set_stream() supplies one.  hbm_budget_bytes
 * bounds the device memory the context's operators may hold (0 = no bound). */
int yeti_ctx_create(int device, size_t hbm_budget_bytes, yeti_ctx **out);
int yeti_ctx_destroy(yeti_ctx *ctx);
/* Use an existing cudaStream_t (passed as void*) for all work of the
 * context; NULL restores the context's own stream (pass cudaStreamLegacy,
 * (void*)0x1, for the legacy default stream). */
int yeti_ctx_set_stream(yeti_ctx *ctx, void *stream);
int yeti_ctx_synchronize(yeti_ctx *ctx);
/* Bytes of device memory currently held by the context's objects. */
size_t yeti_ctx_bytes_in_use(const yeti_ctx *ctx);
/* Device-time accounting (no counterpart in the reference).  With timing
 * on, the element kernels of the Gauss-quadrature calls ("k_u1_stiffness",
 * "k_u1_stiffness_sf", "k_u1_mass", "k_u1_grad") are bracketed by CUDA
 * events on the context's stream and their durations summed per name;
 * yeti_ctx_set_timing() clears the sums.  Each timed launch waits for its
 * end event, so leave timing off outside measurements. */
int yeti_ctx_set_timing(yeti_ctx *ctx, int on);
/* Summed device milliseconds of `kernel` since timing was set; -1 if none. */
double yeti_ctx_kernel_ms(yeti_ctx *ctx, const char *kernel);

/* ------------------------------------------------------------------------
 * U1 element stiffness + COO assembly (drop-in for sys_linmat_lindef_static)
 * ------------------------------------------------------------------------
 * The model arrays are exactly those IGAparametrization.get_inputs4system_
 * elemStorage() passes (IGA_parametrization.py:1705-1716), flattened in
 * Fortran (column-major) order, integers as int64.  Only U1 patches with
 * TENSOR=THREED and MCRD=3 are on this path; a patch of another element type
 * that is marked active returns YETI_EUNSUPPORTED.
 */
typedef struct {
    int64_t nb_patch, nb_elem, nb_cp;
    const double *coords;            /* (3, nb_cp)                         */
    const int64_t *ien;              /* sum_p nnode_p*nb_elem_p, 1-based    */
    const int64_t *nb_elem_patch;    /* (nb_patch)                          */
    const int64_t *nkv;              /* (3, nb_patch) knot vector lengths   */
    const double *ukv;               /* concatenated knot vectors           */
    const int64_t *nijk;             /* (3, nb_elem) 1-based knot spans     */
    const double *weight;            /* sum_p nnode_p*nb_elem_p             */
    const int64_t *jpqr;             /* (3, nb_patch) degrees               */
    const int64_t *nnode;            /* (nb_patch)                          */
    const int64_t *nbint;            /* (nb_patch) Gauss points / element   */
    const int32_t *is_u1;            /* (nb_patch) 1 if U1/THREED           */
    const double *matprops;          /* (2, nb_patch): E, nu                */
    const double *rho;               /* (nb_patch) density                  */
    const int64_t *active;           /* (nb_elem) 1 = assemble              */
    int64_t nb_load;
    const int64_t *inddload;         /* element (or CP) lists of the loads  */
    const int64_t *jdltype;          /* (nb_load) load codes                */
    const double *adlmag;            /* (nb_load) magnitudes                */
    const int64_t *load_target_nbelem; /* (nb_load) list lengths           */
    const double *load_addinfos;     /* additional load data                */
    int64_t len_load_addinfos;
    const int64_t *nb_load_addinfos; /* (nb_load)                           */
    int64_t nb_n_dist;               /* rows of nodal_dist                  */
    const double *nodal_dist;        /* (nb_n_dist, nb_cp)                  */
} yeti_u1_model;

/* Replaces sys_linmat_lindef_static (build_system_elemStorage.f90:24-315).
 * Writes the upper-triangle element blocks in the reference's COO slot order
 * (slots compacted over active elements, diagonal blocks halved) and the
 * load vector F (concentrated loads assigned, then element loads added).
 * kdata/krow/kcol: nb_data entries, F: 3*nb_cp entries; all `mem`. */
int yeti_assemble_u1_coo(yeti_ctx *ctx, const yeti_u1_model *model,
                         int64_t nb_data, double *kdata, int32_t *krow,
                         int32_t *kcol, double *F, int mem);
/* The same, with a choice of element kernel (no counterpart in the
 * reference, whose element routine is the pair loop):
 *   YETI_STIFF_PAIRS    one thread per control-point pair summing over the
 *                       Gauss points in the reference's operation order
 *                       (bit-identical to it; what yeti_assemble_u1_coo runs);
 *   YETI_STIFF_SUMFACT  B^T D B contracted direction by direction over the
 *                       1-D basis tables (sum factorisation): the same slots,
 *                       values equal to rounding (not bit for bit), fewer
 *                       operations from degree 3 on.  Needs NBINT = g^3 with
 *                       g <= 8 and the element's buffers in shared memory
 *                       (degree <= 5 at g = p+1), else YETI_EUNSUPPORTED. */
#define YETI_STIFF_PAIRS 0
#define YETI_STIFF_SUMFACT 1
int yeti_assemble_u1_coo_ex(yeti_ctx *ctx, const yeti_u1_model *model,
                            int64_t nb_data, double *kdata, int32_t *krow,
                            int32_t *kcol, double *F, int mem, int kernel);
/* Consistent mass matrix of the active U1 elements in the same COO slot
 * order (replaces massmtrx.build_cmassmatrix: build_CMASSMatrix,
 * src/yeti_iga/main/compute_CMASSMatrix.f:30-199, with UMASSMAT_byCP's U1
 * branch, main/UMASSMAT.f; called at
 * preprocessing/igaparametrization/OPT_modelling.py:369-371).  Density:
 * model->rho per patch; loads and material moduli are ignored.  The caller
 * adds the transpose as for the stiffness (M = Mside + Mside^T). */
int yeti_assemble_u1_mass_coo(yeti_ctx *ctx, const yeti_u1_model *model,
                              int64_t nb_data, double *mdata, int32_t *mrow,
                              int32_t *mcol, int mem);

/* ------------------------------------------------------------------------
 * Weighted-quadrature (WQ) matrix-free elasticity on one NURBS patch
 * ------------------------------------------------------------------------
 * Patch: degree p[d], nel[d] uniform elements per direction on an open
 * uniform knot vector (the reference's WQ hypothesis,
 * iga_wq_mf/fsrc/iga_wq_methods.f90:1-10), control points cps (3, ncp) and
 * weights (ncp), CP index = iu + n_u*(iv + n_v*iw).  Vectors are
 * component-major [c][iw][iv][iu] (the layout of wq_get_force_3d,
 * wq_assembly.f90:1239-1249).  dirichlet[6*c + f] != 0 clamps component c on
 * face f (0:u=0 1:u=1 2:v=0 3:v=1 4:w=0 5:w=1); clamped dofs are kept in the
 * vectors and held at zero (the reference erases their rows,
 * fortran_mf_wq.py:240-267).
 */
typedef struct yeti_wq_op yeti_wq_op;

/* One-direction WQ rule of degree p on nel uniform elements (host memory,
 * dense row-major nfun x nqp, nfun = p + nel, nqp = 2(p + nel) - 1):
 * point positions x, basis values B0 and derivatives B1, and weights Wxy for
 * test derivative order x and trial derivative order y.  Replaces
 * basis_weights.wq_get_size_data / wq_get_data
 * (src/yeti_iga/iga_wq_mf/fsrc/iga_wq_basis_weights.f90:198-260); any output
 * pointer may be NULL. */
int yeti_wq_rule_1d_size(int p, int nel, int32_t *nfun, int32_t *nqp);
int yeti_wq_rule_1d(int p, int nel, double *x, double *B0, double *B1,
                    double *W00, double *W01, double *W10, double *W11);

typedef struct {
    int32_t iterations;        /* total inner (Krylov) iterations        */
    int32_t outer_iterations;  /* FP64 refinement steps (mixed mode)      */
    int32_t fp64_applies;      /* operator applications in FP64           */
    int32_t fp32_applies;      /* operator applications in FP32           */
    double rel_residual;       /* ||b - A x||_2 / ||b||_2 (FP64, true)    */
    double rel_residual_inf;   /* max|b - A x| / max|b| (reference's
                                  criterion, mf_wq_solver.f90:931)        */
    double solve_ms;           /* device time of the solve                */
    int32_t status;            /* YETI_OK / YETI_ENOTCONV / ...           */
} yeti_cg_stats;

#define YETI_WQ_F64 1     /* keep FP64 operator data                    */
#define YETI_WQ_F32 2     /* keep FP32 operator data                    */

/* p[d] in 2..8 and nel[d] >= 2 per direction (the WQ rule's construction
 * needs two elements); otherwise YETI_EINVAL. */
int yeti_wq_setup(yeti_ctx *ctx, const int32_t p[3], const int32_t nel[3],
                  const double *cps, const double *weights, double E,
                  double nu, const uint8_t dirichlet[18], int prec_mask,
                  yeti_wq_op **out);
int yeti_wq_destroy(yeti_wq_op *op);
/* Sizes: number of control points, total dofs (3*ncp), free dofs,
 * quadrature points, bytes of operator data held on the device. */
int yeti_wq_info(const yeti_wq_op *op, int64_t *ncp, int64_t *ndof,
                 int64_t *nfree, int64_t *nqp, int64_t *bytes);
/* Ku = K u.  prec YETI_PREC_F64: u, Ku are double; YETI_PREC_F32: float. */
int yeti_wq_apply(yeti_wq_op *op, const void *u, void *Ku, int prec, int mem);
/* K u with HOST buffers u and Ku (as yeti_wq_apply with YETI_MEM_HOST) that
 * allocates no device memory.  No counterpart in the reference.  For callers
 * that cannot allocate device memory at this point -- a process whose device
 * memory is all reserved by another allocator, or a latency-critical loop that
 * must not pay cudaMalloc/cudaFree's implicit synchronisation -- the two
 * vectors are staged in one file-scope device array of at most 2,097,152 dofs
 * per vector (32 MiB, held until the process exits); larger operators return
 * YETI_EINVAL.  The first call on a device looks the array's device address
 * up (cudaGetSymbolAddress); under CUDA's default lazy module loading that
 * lookup is also when the 32 MiB are committed on the device.  Make that
 * first call before device memory is all reserved and before any stream
 * capture.  All calls share the array: calls that overlap on the GPU race.
 * Returns YETI_ETIMEDOUT, as yeti_wq_apply does, when a bounded device wait
 * gave up. */
int yeti_wq_apply_static(yeti_wq_op *op, const void *u, void *Ku, int prec);
/* Polls of each bounded wait for a coefficient copy in the streaming apply
 * (default 65536; tries < 0 restores it).  A wait that runs out makes the
 * apply (and the solvers) return YETI_ETIMEDOUT with invalid results and the
 * device context intact.  Applies to launches issued after the call
 * (graphs captured before keep the old bound).  Diagnostic knob; no
 * counterpart in the reference. */
int yeti_wq_set_wait_limit(yeti_wq_op *op, int tries);
/* Diagonal of K (3*ncp doubles; clamped dofs hold 1). */
int yeti_wq_diag(yeti_wq_op *op, double *d, int mem);
/* Body-force load vector for a constant force density f[3]
 * (wq_get_force_3d, wq_assembly.f90:1193-1251). */
int yeti_wq_body_force(yeti_wq_op *op, const double f[3], double *F, int mem);
/* Mode bits of yeti_wq_pcg. */
#define YETI_PCG_MIXED 1       /* FP32 operator and Krylov vectors          */
#define YETI_PCG_BICGSTAB 2    /* BiCGSTAB instead of CG                    */
#define YETI_PCG_FD 4          /* fast-diagonalisation preconditioner
                                  (mf_wq_solver.f90:803-953) instead of
                                  Jacobi; a[c][d] = mean of S[(c,d),(c,d)]
                                  (the reference's 'JM')                    */
#define YETI_PCG_FD_SCALED 8   /* with YETI_PCG_FD: diagonal scaling
                                  sqrt(diag(P)/diag(K)) ('JMS', 'TDS')      */
#define YETI_PCG_FD_UNIT 16    /* with YETI_PCG_FD: a[c][d] = 1 ('C')       */
#define YETI_PCG_FD_TD 32      /* with YETI_PCG_FD: 1-D matrices weighted by
                                  the tensor decomposition of the diagonal
                                  coefficients ('TD', 'TDS' with
                                  YETI_PCG_FD_SCALED;
                                  tensor_decomposition_3d,
                                  tensor_algebra.f90:1256-1382)            */

/* Preconditioned Krylov solve of K x = b (x holds the initial guess;
 * replaces wq_mf_cg_3d / wq_mf_bicgstab_3d, mf_wq_solver.f90:642,958).
 * mode bit 0: mixed precision (FP32 operator and Krylov vectors, FP64 true
 * residual and solution: reliable updates for CG, iterative refinement for
 * BiCGSTAB); bit 1: BiCGSTAB instead of CG; bits 2-4: the fast-diagonalisation
 * preconditioner (YETI_PCG_FD*), Jacobi when clear.  Stops when the FP64
 * true residual satisfies ||r||_2 <= rtol ||b||_2. */
int yeti_wq_pcg(yeti_wq_op *op, const double *b, double *x, double rtol,
                int maxit, int mode, yeti_cg_stats *stats, int mem);
/* As yeti_wq_pcg, FP64 modes only, with the reference's iteration history
 * (the RelRes / RelError outputs of wq_mf_cg_3d and wq_mf_bicgstab_3d,
 * mf_wq_solver.f90:656,697,785-792): relres[k] = max|r_k| / max|b| and, when
 * directsol is given, relerr[k] = max|directsol - x_k| / max|directsol|, for
 * k = 0..iterations (host arrays of maxit + 1 doubles; relerr may be NULL).
 * Stops on the reference's test relres[k] <= rtol (mf_wq_solver.f90:931-936)
 * instead of the 2-norm one. */
int yeti_wq_pcg_history(yeti_wq_op *op, const double *b, double *x, double rtol,
                        int maxit, int mode, const double *directsol,
                        double *relres, double *relerr, yeti_cg_stats *stats,
                        int mem);
/* z = P^{-1} r for the fast-diagonalisation preconditioner selected by the
 * YETI_PCG_FD* bits of `variant` (fast_diagonalization_3d,
 * tensor_algebra.f90:1107-1161, per displacement component, with
 * scaling_FastDiag :1598-1625 when YETI_PCG_FD_SCALED).  prec YETI_PREC_F64 /
 * F32: r and z are double / float; z is zero on clamped dofs. */
int yeti_wq_fd_apply(yeti_wq_op *op, const void *r, void *z, int prec,
                     int variant, int mem);

/* ------------------------------------------------------------------------
 * Adjoint shape gradient of the linear-elastic work (U1, 3D)
 * ------------------------------------------------------------------------
 * Replaces gradLinElastWork_AN (gradtotalwork_fullAN.f90:17-300): for each
 * adjoint field a, gWint[a] = d(-ADJ_a^T K U)/dP and gWext[a] = d(ADJ_a^T F)/dP
 * with respect to the control-point coordinates P (3, nb_cp).
 * sol: (3, nb_cp); adj: (nadj, 3, nb_cp) Fortran order; outputs
 * (nadj, 3, nb_cp) Fortran order.  include_surface_loads: 0 reproduces the
 * reference (surface-load sensitivity left out, gradUELMAT_solid.f90:463-477);
 * 1 adds the traction term.  sol/adj/outputs are `mem`. */
int yeti_grad_lin_elast_work(yeti_ctx *ctx, const yeti_u1_model *model,
                             const double *sol, const double *adj,
                             int64_t nadj, int compute_wint, int compute_wext,
                             int include_surface_loads, double *gwint,
                             double *gwext, int mem);

/* Volume of the model's active U1 elements and, when grad != NULL, its
 * gradient with respect to the control-point coordinates (3, nb_cp), Fortran
 * order, `mem`).  Replaces optim.volume.computevolume / computegradvolume
 * (computeVolume, src/yeti_iga/optim/volume.f90:20-210; computeGradVolume,
 * optim/gradvolume.f90:16-355; called at
 * preprocessing/igaparametrization/OPT_modelling.py:508-531), whose
 * listpatch selects whole patches: set `active` to 1 on their elements.
 * The determinant is signed, as the reference's.  vol is host memory. */
int yeti_volume_u1(yeti_ctx *ctx, const yeti_u1_model *model, double *vol,
                   double *grad, int mem);

/* ------------------------------------------------------------------------
 * Serving: persistent request loop (no counterpart in the reference)
 * ------------------------------------------------------------------------
 * A server owns an engine thread and a private context on `device`.
 * Submitted requests wait in arrival order and are admitted while fewer than
 * max_active are active and their estimated device bytes fit in
 * hbm_budget_bytes (0: no bound) beside the active ones.  An admitted request
 * gets its WQ operator (FP64 data) and one FP64 preconditioned Krylov solve
 * per right-hand side (the request's mode: CG or BiCGSTAB, Jacobi or fast
 * diagonalisation);
 * the solves of all active requests run concurrently on the device (CUDA
 * graphs of 16 iterations on a pool of streams) with operators and Krylov
 * state resident in HBM.  Submit, poll and wait may be called from any host
 * thread.
 */
typedef struct yeti_server yeti_server;

typedef struct {
    int32_t p[3], nel[3];         /* degrees 2..8, elements per direction  */
    const double *cps;            /* (3, ncp) host, as yeti_wq_setup       */
    const double *weights;        /* (ncp) host                            */
    double E, nu;
    uint8_t dirichlet[18];        /* as yeti_wq_setup                      */
    int32_t nrhs;                 /* 1..8                                  */
    const double *rhs;            /* nrhs x 3*ncp host, component-major    */
    double rtol;                  /* ||r||_2 <= rtol ||b||_2               */
    int32_t maxit;
    int32_t mode;                 /* FP64 Krylov method and preconditioner:
                                     0 Jacobi CG; YETI_PCG_BICGSTAB and the
                                     YETI_PCG_FD* bits as yeti_wq_pcg      */
} yeti_serve_request;

typedef struct {
    int32_t status;               /* YETI_OK or the error code             */
    int32_t nrhs;
    int64_t ndof;
    int32_t iterations[8];
    double rel_residual[8];       /* true FP64 residual of each solution   */
    double queue_ms;              /* submit -> admission                   */
    double solve_ms;              /* admission -> last solution            */
    double total_ms;              /* submit -> last solution               */
} yeti_serve_result;

int yeti_serve_open(int device, size_t hbm_budget_bytes, int max_active,
                    yeti_server **out);
/* Copies the request's arrays; returns at once with a ticket.  A request
 * whose estimated device bytes exceed the budget is refused (YETI_ENOMEM). */
int yeti_serve_submit(yeti_server *srv, const yeti_serve_request *req,
                      int64_t *ticket);
/* 1: done (x gets nrhs x ndof doubles, res filled, ticket released),
 * 0: pending, < 0: the request failed (error code; ticket released). */
int yeti_serve_poll(yeti_server *srv, int64_t ticket, double *x,
                    yeti_serve_result *res);
/* As poll, blocking up to timeout_ms (< 0: no limit; YETI_ETIMEDOUT). */
int yeti_serve_wait(yeti_server *srv, int64_t ticket, double timeout_ms,
                    double *x, yeti_serve_result *res);
int yeti_serve_stats(yeti_server *srv, int64_t *done, int64_t *queued,
                     int32_t *active, int32_t *peak_active,
                     size_t *committed_bytes);
/* Cumulative thread time (ms): worker threads in operator setups and solve
 * starts, worker threads in retirements (solution copies, frees), the engine
 * thread in polling and relaunching chunks. */
int yeti_serve_times(yeti_server *srv, double *setup_ms, double *retire_ms,
                     double *poll_ms);
/* Finishes the active requests, fails the queued ones, joins the threads. */
int yeti_serve_close(yeti_server *srv);

#ifdef __cplusplus
}
#endif
#endif /* YETI_B200_H */
