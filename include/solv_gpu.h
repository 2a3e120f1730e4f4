/*
 * solv_gpu.h -- C-ABI of the B200 face-addressed Krylov solvers
 * (libsolv_gpu.so).
 *
 * Drop-in for the linear-solver hot path of spray-simulation:
 *
 *   subroutine solv_cg  (imat,reduc,n_iter,phi,res0,res0_n,not_r0)
 *                                     spray-simulation/solv_cg.f90:7-13
 *   subroutine solv_bicg(imat,reduc,n_iter,phi,res0,res0_n,not_r0)
 *                                     spray-simulation/solv_bicg.f90:7-13
 *   subroutine solv_res (phi,res0,res0_n,not_r0)       solv_res.f90:5-9
 *   subroutine solv_precond(imat,c,c_r)                solv_precond.f90:5-7
 *   subroutine solv_direct(imat,c,c_r,x,b)             solv_direct.f90:5-8
 *
 * The reference takes its matrix from module globals pl, ng(:)%{ip,in,p,n}
 * and v_lst (solv_data.f90:10-22, wired by grd_solv.f90:7-24); here the
 * matrix is handed over once per structure with solv_gpu_matrix_set (the
 * grd_solv step) and its coefficients refreshed with solv_gpu_matrix_values
 * (what cfd_setup.f90 does before every solve).  v_lst is derived from the
 * face list in ascending face order, the order grd_conn.f90:129-152 gives.
 *
 * Conventions (as the Fortran):
 *   - indices are 1-based; in[f] == 0 marks a boundary face (skipped);
 *   - phi is cell-major,   phi[(ip-1)*n_vc + ivc]    (phi(ip)%vc(ivc));
 *   - res0 is column-major, res0[ivc*n_cell + ip-1]  (res0(ip,ivc));
 *     on entry the right-hand side b, on exit the initial residual;
 *   - res0_n[ivc] returns the initial L1 norms (not the final ones);
 *   - the stopping rule is |r|_1 / (|r0|_1 + 1e-20) < reduc, per component.
 *   - imat: 0 Jacobi, 1 DIC, 2 DILU (solv_precond.f90:13-24).  The solvers
 *     reject other values; solv_gpu_precond / solv_gpu_direct take them as
 *     the reference does (<= 0 Jacobi, >= 3 the unmodified diagonal with
 *     both triangular sweeps).
 * Every pointer argument is a HOST pointer unless the name ends in _dev.
 * The reference has no error return; these return a status code.
 *
 * Thread-safety: one context per host thread / stream; a context is not
 * re-entrant (the reference keeps its matrix in module globals, too).
 */
#ifndef SOLV_GPU_H
#define SOLV_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define SOLV_GPU_OK 0           /* every component reached reduc           */
#define SOLV_GPU_MAXITER 1      /* a component stopped at n_iter (the
                                   reference's normal exit with a cap)     */
#define SOLV_GPU_NAN 3          /* NaN / Inf seen in a reduction           */
#define SOLV_GPU_BAD_INPUT 4    /* index out of range, sizes, null, ...    */
#define SOLV_GPU_DEVICE_ERROR 5 /* CUDA error (message: solv_gpu_last_error) */
#define SOLV_GPU_TIMEOUT 6      /* a bounded device wait ran out (a DIC/DILU
                                   recurrence's neighbour never arrived);
                                   the context stays usable                 */
#define SOLV_GPU_NO_MATRIX 7    /* no solv_gpu_matrix_set yet              */
#define SOLV_GPU_ZERO_RHS 8     /* maxval(res0_n) < small: the solve ends
                                   at once as solv_cg.f90:21 does; reported
                                   in stats.status, the call returns OK    */
#define SOLV_GPU_TOO_LARGE 9    /* beyond the fixed scratch of
                                   solv_gpu_res_noalloc (n_vc > 4)         */

#define SOLV_GPU_MAX_VC 4

/* option keys for solv_gpu_set_option */
#define SOLV_OPT_PRECISION 1    /* 0 = FP64 (default), the reference's
                                   arithmetic; 1 = FP32 inner Krylov with
                                   FP64 reliable updates (CG) or iterative
                                   refinement (BiCGSTAB); its FP32 steps
                                   divide without the absolute 1e-20 guard,
                                   so weakly driven systems converge       */
#define SOLV_OPT_INNER_REDUC 2  /* inner relative drop per refinement
                                   sweep (FP32 mode), default 1e-6         */
#define SOLV_OPT_GRAPH_ITERS 3  /* Krylov iterations per CUDA-graph launch
                                   (0 = no graphs, plain launches); with
                                   SOLV_OPT_GRAPH_LOOP 1 the host checks
                                   (reliable updates, stall windows) come
                                   every this many iterations             */
#define SOLV_OPT_GRAPH_LOOP 21  /* 1: the iterations run in a conditional
                                   WHILE graph that stops on the device
                                   once every lane has stopped (no
                                   iterations past it, no host round trip
                                   in between; each pass of the loop costs
                                   about 3 us, which small systems feel);
                                   0: a graph of exactly
                                   SOLV_OPT_GRAPH_ITERS iterations per
                                   launch; 2 (default): WHILE graphs for
                                   the learned flexible CG, whose lanes
                                   stop inside a graph for each reliable
                                   update, fixed ones for CG and BiCGSTAB.
                                   Where the CUDA driver has no conditional
                                   graph nodes, 0 is used                  */
#define SOLV_OPT_BLOCK 4        /* threads per block for the cell kernels
                                   (64..256, multiple of 32)               */
#define SOLV_OPT_GRID_PER_SM 5  /* resident blocks per SM for reductions
                                   (at most 2048 threads per SM are used)  */
#define SOLV_OPT_MAX_REFINE 6   /* cap on refinement sweeps (FP32 mode)    */
#define SOLV_OPT_INNER_MAX_ITER 7 /* cap on FP32 iterations per refinement
                                   sweep (default 2000)                    */
#define SOLV_OPT_RELIABLE_DELTA 8 /* FP32 CG: replace the recursive residual
                                   by the FP64 one each time it has dropped
                                   by this factor (default 0.1)            */
#define SOLV_OPT_GNN_LOSS 9     /* training loss of the learned
                                   preconditioner: 0 = energy of z,
                                   1 = energy after the best step along z
                                   (scale-free, default), both for the
                                   network's operator alone; 2 = the
                                   V-cycle with the network as finest-level
                                   smoother, -log((z.b)^2/(z.Az)) per
                                   sample                                  */
#define SOLV_OPT_MG_LEVELS 10   /* learned preconditioner: coarse levels of
                                   the aggregation hierarchy at most (default
                                   12; 0 = the network's one-level operator
                                   alone)                                  */
#define SOLV_OPT_MG_SMOOTHER 11 /* finest-level smoother of the hierarchy:
                                   1 = the network's operator (default),
                                   2 = its diagonal alone: Jacobi with the
                                   network's per-cell weights (as cheap as
                                   Jacobi), 0 = damped Jacobi (no network) */
#define SOLV_OPT_MG_OMEGA 12    /* smoother damping (default 0.8)          */
#define SOLV_OPT_MG_ALPHA 13    /* coarse-correction scale (default 2)     */
#define SOLV_OPT_FCG_STALL_ITERS 14 /* learned preconditioner: iterations
                                   without the residual falling below
                                   SOLV_OPT_FCG_STALL_DROP times its value
                                   at the start of the window after which
                                   Jacobi-PCG takes over (default 1000)    */
#define SOLV_OPT_FCG_STALL_DROP 15 /* the drop a window must reach
                                   (default 0.9: a stall is no progress,
                                   not slow progress)                      */
#define SOLV_OPT_MG_SCALE_MIN 16 /* floor on the network's per-cell scales
                                   (default 0.5; 0 leaves them as the
                                   network makes them)                     */
#define SOLV_OPT_PERSISTENT 19  /* FP64 Jacobi PCG (imat 0, n_vc 1, one
                                   system or a batch): 1 runs the whole
                                   Krylov loop as one launch, a cluster of
                                   8 thread blocks per system with the step
                                   kernels fused (no host polls, no graph);
                                   0 (default) the graph of step kernels   */
#define SOLV_OPT_VECTOR_WIDTH 18 /* FP32 matrix products (mixed-precision
                                   Krylov, flexible CG, V-cycle): matrix
                                   slots each thread loads before it sums
                                   them, 2, 4 (default) or 8              */
#define SOLV_OPT_FCG_SLOW_ITERS 23 /* the learned solve: when the network-
                                   smoothed V-cycle needs more than this
                                   many flexible-CG iterations for one
                                   reliable-update drop, damped Jacobi
                                   smooths the same hierarchy for the rest
                                   of the solve (default 15; 0 never)     */
#define SOLV_OPT_FCG_FALLBACK 22 /* the PCG a stalled learned solve hands
                                   over to: 0 (default) Jacobi, 1 DIC, 2
                                   DILU (the reference's pressure solver is
                                   DIC-PCG, cfd_setup.f90:662); the
                                   factorisation is made at the hand-over  */
#define SOLV_OPT_FCG_RELIABLE_DELTA 20 /* the learned flexible CG (FP32
                                   inner iterations): the drop of the FP32
                                   residual at which a lane stops for a
                                   reliable update (default 0.1; CG lanes
                                   use SOLV_OPT_RELIABLE_DELTA)            */
#define SOLV_OPT_MG_BUILD 17    /* where the aggregation hierarchy is built:
                                   0 on the GPU (default: handshake
                                   matching, Galerkin structure by one warp
                                   per coarse row), 1 on the host
                                   (sequential greedy matching)            */

typedef struct solv_gpu_ctx solv_gpu_ctx;

typedef struct {
  int n_vc;                      /* components solved                      */
  int iters[SOLV_GPU_MAX_VC];    /* Krylov iterations (inner, summed over
                                    refinement sweeps in FP32 mode)        */
  double ratio[SOLV_GPU_MAX_VC]; /* last |r|_1 / |r0|_1 per component      */
  int status;                    /* as the return value                    */
  int n_levels;                  /* wavefront levels of the factorisation  */
  int refinements;               /* FP64 refinement sweeps (FP32 mode)     */
  int graph_launches;            /* CUDA-graph launches in the solve       */
  int kernel_launches;           /* kernels launched in the solve          */
  double solve_ms;               /* device time of the solve (events)      */
  int fallbacks;                 /* learned preconditioner handed over to
                                    plain PCG (solv_gpu_fcg)               */
  int mg_levels;                 /* coarse levels of the aggregation
                                    hierarchy used (solv_gpu_fcg)          */
  int smoother_switches;         /* the learned solve's network smoother
                                    gave way to damped Jacobi in the same
                                    V-cycle (SOLV_OPT_FCG_SLOW_ITERS)      */
} solv_gpu_stats;

/* -- context ------------------------------------------------------------ */
int solv_gpu_create(solv_gpu_ctx **ctx, int device);
int solv_gpu_destroy(solv_gpu_ctx *ctx);
/* Run on a caller stream (a cudaStream_t); NULL restores the own stream. */
int solv_gpu_set_stream(solv_gpu_ctx *ctx, void *stream);
int solv_gpu_set_option(solv_gpu_ctx *ctx, int key, double value);
const char *solv_gpu_status_string(int status);
const char *solv_gpu_last_error(const solv_gpu_ctx *ctx);

/* -- matrix (grd_solv.f90:7-24 + the coefficient fill of cfd_setup) ----- */
/* Structure + coefficients.  ip/in/p/n have n_face entries (interior and
 * boundary faces, as size(ng)), pl has n_cell.  Replaces the module
 * globals ng, pl, v_lst of solv_data.f90:10-22. */
int solv_gpu_matrix_set(solv_gpu_ctx *ctx, int n_cell, int n_face,
                        const int *ip, const int *in, const double *p,
                        const double *n, const double *pl);
/* New coefficients for the same structure (host pointers). */
int solv_gpu_matrix_values(solv_gpu_ctx *ctx, const double *p,
                           const double *n, const double *pl);
/* Same, device pointers (coefficients assembled on the GPU). */
int solv_gpu_matrix_values_dev(solv_gpu_ctx *ctx, const double *p_dev,
                               const double *n_dev, const double *pl_dev);
/* Wavefront levels of the lower-triangular DAG (the sweep depth). */
int solv_gpu_matrix_levels(const solv_gpu_ctx *ctx);

/* -- the hot path ------------------------------------------------------- */
/* solv_res.f90:5-30 */
int solv_gpu_res(solv_gpu_ctx *ctx, int n_vc, const double *phi,
                 double *res0, double *res0_n, int not_r0);
/* solv_precond.f90:5-30: c = 1/(d+small), c_r = d (n_cell each) */
int solv_gpu_precond(solv_gpu_ctx *ctx, int imat, double *c, double *c_r);
/* solv_direct.f90:5-43: x = M^-1 b with the given c, c_r */
int solv_gpu_direct(solv_gpu_ctx *ctx, int imat, const double *c,
                    const double *c_r, double *x, const double *b);
/* y = A x with the face-loop arithmetic of solv_cg.f90:56-64 */
int solv_gpu_spmv(solv_gpu_ctx *ctx, const double *x, double *y);
/* solv_cg.f90:7-87 */
int solv_gpu_cg(solv_gpu_ctx *ctx, int imat, double reduc, int n_iter,
                int n_vc, double *phi, double *res0, double *res0_n,
                int not_r0, solv_gpu_stats *stats);
/* solv_bicg.f90:7-121 */
int solv_gpu_bicg(solv_gpu_ctx *ctx, int imat, double reduc, int n_iter,
                  int n_vc, double *phi, double *res0, double *res0_n,
                  int not_r0, solv_gpu_stats *stats);

/* Device-resident forms: phi_dev / res0_dev in the caller layouts above,
 * already in HBM; res0_n stays a host array.  Same semantics. */
int solv_gpu_cg_dev(solv_gpu_ctx *ctx, int imat, double reduc, int n_iter,
                    int n_vc, double *phi_dev, double *res0_dev,
                    double *res0_n, int not_r0, solv_gpu_stats *stats);
int solv_gpu_bicg_dev(solv_gpu_ctx *ctx, int imat, double reduc, int n_iter,
                      int n_vc, double *phi_dev, double *res0_dev,
                      double *res0_n, int not_r0, solv_gpu_stats *stats);
int solv_gpu_spmv_dev(solv_gpu_ctx *ctx, const double *x_dev, double *y_dev,
                      int repeat, float *ms_per_call);
/* Device time per launch (CUDA events on the context's stream, `repeat`
 * back-to-back launches on workspace vectors) of a kernel of the solve
 * path: which 0 = FP64 matrix product, 1 = FP32 matrix product, 2 = the
 * learned preconditioner's one-level application (FP32), 3 = one V-cycle
 * of the multigrid preconditioner (FP32, all its kernels, with the current
 * SOLV_OPT_MG_* settings), 4 = the V-cycle's level-0 residual t = b - A x
 * (FP32), 5 = the network operator's smoothing step (FP32), 6 = the
 * flexible-CG product q = A p with p.q and p.r (FP32), 7 = the FP64 CG
 * product q = A p with p.q, 8 = one DILU application M^-1 r (forward and
 * backward recurrence, FP64).  No counterpart in the reference; used for
 * roofline reporting. */
int solv_gpu_kernel_time(solv_gpu_ctx *ctx, int which, int repeat,
                         float *ms_per_launch);

/* Diagnostic (no counterpart in the reference): one DIC/DILU-style bounded
 * wait on a value that nothing writes, through the sweeps' own wait driver.
 * Returns SOLV_GPU_TIMEOUT after about a second when the bound works; the
 * context stays usable. */
int solv_gpu_selftest_sweep_wait(solv_gpu_ctx *ctx);

/* -- learned preconditioner ---------------------------------------------- */
/* No counterpart in the reference.  Flexible CG, FCG(1), in FP32 with
 * FP64 reliable updates.  A 3-layer, width-32 message-passing network over
 * the face graph (BF16 weights, per-cell MLPs on the tensor cores, FP32
 * accumulate) reads the cell diagonal, the face coefficients and the
 * initial residual once per solve and emits the per-cell scales S and the
 * symmetric face weights E of K = D^-1/2 S (I + E) S D^-1/2 (|E| < 1 by
 * construction, so K is symmetric positive definite).  K is the finest-
 * level smoother of a symmetric V-cycle over an aggregation hierarchy
 * (about 8 cells per aggregate, Galerkin coarse matrices, damped Jacobi on
 * the coarse levels, dense inverse on the coarsest), and the V-cycle is the
 * preconditioner (SOLV_OPT_MG_*; the hierarchy is built, on the GPU, at the
 * first such solve after solv_gpu_matrix_set, from the coefficients then;
 * SOLV_OPT_MG_LEVELS 0 uses K alone).  Each solve bounds the smoother:
 * per-cell scales are held at 0.5 or more and K is scaled so that eight
 * power iterations find lambda_max(omega K A) <= 1.9.  If
 * the iteration loses positive curvature or produces NaN, or its residual
 * stalls (SOLV_OPT_FCG_STALL_*, or the FP64 residual fails to improve by
 * 10% over three reliable updates), plain Jacobi-PCG takes over from the
 * current iterate (stats.fallbacks); the FP64 residual
 * test |b - A x|_1 / |r0|_1 < reduc decides convergence either way.  Same
 * argument meaning as solv_gpu_cg with imat ignored, n_vc = 1, one system;
 * the matrix must be symmetric (the pressure system). */
int solv_gpu_fcg(solv_gpu_ctx *ctx, double reduc, int n_iter, double *phi,
                 double *res0, double *res0_n, int not_r0,
                 solv_gpu_stats *stats);
int solv_gpu_fcg_dev(solv_gpu_ctx *ctx, double reduc, int n_iter,
                     double *phi_dev, double *res0_dev, double *res0_n,
                     int not_r0, solv_gpu_stats *stats);
/* The hierarchy's aggregation rule on a caller graph (host only, no GPU):
 * `passes` passes of pairwise matching along the strongest coupling, then
 * cells left alone join their strongest neighbour's aggregate.  Graph in
 * CSR (ptr n+1, adj, positive strengths w); agg[i] = aggregate of cell i,
 * *n_agg = their number.  No counterpart in the reference. */
int solv_gpu_mg_aggregate(int n, const long long *ptr, const int *adj, const float *w,
                          int passes, int *agg, int *n_agg);
/* Aggregation of the hierarchy: for each cell of level - 1 (caller order
 * for level 1, i.e. the caller's cells), the index of its aggregate on
 * `level` (1..levels); n = that finer level's size, *n_coarse = the size of
 * `level`.  Builds the hierarchy if needed. */
int solv_gpu_mg_aggregates(solv_gpu_ctx *ctx, int level, int *agg, int n,
                           int *n_coarse);
/* Network parameters (FP32 master copy, solv_gpu_gnn_n_params() floats). */
int solv_gpu_gnn_n_params(void);
int solv_gpu_gnn_set_params(solv_gpu_ctx *ctx, const float *params, int n);
int solv_gpu_gnn_get_params(solv_gpu_ctx *ctx, float *params, int n);
/* z = M^-1 r with the preconditioner the network builds from r0 (the
 * solve's initial residual); r0_dev, r_dev, z_dev caller order, device.
 * path 0: inference kernels (BF16, tensor cores); 1: training kernels. */
int solv_gpu_gnn_forward_dev(solv_gpu_ctx *ctx, const double *r0_dev,
                             const double *r_dev, double *z_dev, int path);
/* Training: forward + backward of the loss SOLV_OPT_GNN_LOSS selects, for
 * the preconditioner built from r0, over n_samples residuals u (each
 * n_cell long, consecutive, caller order, device): 0 the energy
 * J = 1/2 z'Âz - z'u of z = K u in the Jacobi-scaled space (minimised by
 * K u = Â^-1 u); 1 the scale-free J = -(z'u)^2 / (z'Âz), twice the energy
 * after the best step along z; 2 J = -log((z'u)^2 / (z'Az)) with z the
 * V-cycle applied to u (needs the hierarchy).  Gradients add up in an FP32
 * accumulator (zeroed first unless accumulate); loss = sum J / (n_cell
 * n_samples). */
int solv_gpu_gnn_grad_dev(solv_gpu_ctx *ctx, const double *r0_dev,
                          const double *samples_dev, int n_samples,
                          double *loss, int accumulate);
int solv_gpu_gnn_get_grad(solv_gpu_ctx *ctx, float *grad, int n);
int solv_gpu_gnn_zero_grad(solv_gpu_ctx *ctx);
/* Adam step on the accumulated gradient (scaled by grad_scale), zeroes it. */
int solv_gpu_gnn_adam(solv_gpu_ctx *ctx, float lr, float grad_scale);

/* -- autotuner ------------------------------------------------------------ */
/* No counterpart in the reference (it has no tunables).  Times candidate
 * launch shapes (threads per block 128/256, resident blocks per SM 4/8/16
 * for the reduction kernels, at most 2048 threads per SM, Krylov
 * iterations per CUDA graph 8/32 and, where the iteration runs in FP32 --
 * precision 1, or the learned solve -- the products' vector width 2/4/8)
 * on the current matrix (one system or a batch) with the given solver
 * (0 CG, 1 BiCGSTAB, 2 the learned flexible CG of solv_gpu_fcg: one
 * system, n_vc = 1, parameters set), preconditioner, component count and
 * the context's precision, and leaves the fastest set on the context.
 * ms_per_iter_before is the per-iteration time of the settings in effect
 * before the call, measured the same way; those settings stay eligible, so
 * ms_per_iter <= ms_per_iter_before. */
typedef struct {
  int block, grid_per_sm, graph_iters, candidates;
  double ms_per_iter;
  int vector_width;
  double ms_per_iter_before;
} solv_gpu_tune;
int solv_gpu_autotune(solv_gpu_ctx *ctx, int solver, int imat, int n_vc,
                      solv_gpu_tune *out);

/* -- batches of independent systems ----------------------------------- */
/* No counterpart call in the reference, which solves one system per call
 * (solv_cg.f90:26 loops over the n_vc components of one matrix); a batch
 * is n_sys such calls done together.  The systems are concatenated:
 * system k owns cells cell_ptr[k]+1 .. cell_ptr[k+1] (1-based in ip/in),
 * cell_ptr[0] = 0, and no face may couple two systems.  Each system and
 * component iterates and stops on its own (own Krylov scalars, own
 * res0_n, own stopping test), exactly as n_sys separate solv_cg calls. */
int solv_gpu_matrix_set_batch(solv_gpu_ctx *ctx, int n_sys, const int *cell_ptr,
                              int n_face, const int *ip, const int *in,
                              const double *p, const double *n,
                              const double *pl);
int solv_gpu_n_systems(const solv_gpu_ctx *ctx);
/* phi: cell-major over all cells; res0: column-major over all cells
 * (res0[ivc*n_cell_total + i]); res0_n, iters, ratio: [k*n_vc + ivc]
 * (iters / ratio may be NULL). */
int solv_gpu_cg_batch(solv_gpu_ctx *ctx, int imat, double reduc, int n_iter,
                      int n_vc, double *phi, double *res0, double *res0_n,
                      int not_r0, int *iters, double *ratio,
                      solv_gpu_stats *stats);
int solv_gpu_bicg_batch(solv_gpu_ctx *ctx, int imat, double reduc, int n_iter,
                        int n_vc, double *phi, double *res0, double *res0_n,
                        int not_r0, int *iters, double *ratio,
                        solv_gpu_stats *stats);
int solv_gpu_cg_batch_dev(solv_gpu_ctx *ctx, int imat, double reduc,
                          int n_iter, int n_vc, double *phi_dev,
                          double *res0_dev, double *res0_n, int not_r0,
                          int *iters, double *ratio, solv_gpu_stats *stats);
int solv_gpu_bicg_batch_dev(solv_gpu_ctx *ctx, int imat, double reduc,
                            int n_iter, int n_vc, double *phi_dev,
                            double *res0_dev, double *res0_n, int not_r0,
                            int *iters, double *ratio, solv_gpu_stats *stats);

/* -- residual without any allocation -------------------------------------- */
/* No counterpart in the reference: an entry point for callers that cannot
 * allocate device memory (their memory pool belongs to another runtime, or
 * a long-running service forbids allocation once started).
 * Computes solv_res (r = b - A phi, res0_n = sum |r| per component,
 * solv_res.f90:5-30) straight from caller-owned DEVICE arrays: the face
 * list ip/in/p/n (n_face, 1-based, in = 0 on boundary faces) and pl
 * (n_cell), phi (cell-major), res0 (column-major; in: b, out: r) and
 * res0_n (device, n_vc doubles).  Needs no context; runs on `stream` (a
 * cudaStream_t, NULL for the default stream) on the current device and
 * returns when the result is there.  It calls no cudaMalloc / cudaFree:
 * its scratch is one fixed file-scope device array (about 19 KB per GPU
 * that loads the library, held until exit); the first call on a device
 * looks its address up (cudaGetSymbolAddress) -- make that first call
 * before any stream capture.  Calls overlapping on the GPU share that
 * scratch and race.  The scratch's counters are cleared by every call;
 * nothing the caller passes must start at zero (res0_n is overwritten).
 * Limits: n_vc <= 4 (SOLV_GPU_TOO_LARGE beyond; n_vc < 1 is
 * SOLV_GPU_BAD_INPUT).  Face contributions are added with atomics, so r
 * agrees with solv_res to rounding, not bit for bit.  Face indices are
 * checked on the GPU before res0 is written: if one is out of range the
 * call returns SOLV_GPU_BAD_INPUT and res0, res0_n are left unchanged.  A
 * launch error still pending from the caller's earlier work is cleared at
 * entry and not reported as this call's. */
int solv_gpu_res_noalloc(int n_cell, int n_face, const int *ip_dev,
                         const int *in_dev, const double *p_dev,
                         const double *n_dev, const double *pl_dev, int n_vc,
                         const double *phi_dev, double *res0_dev,
                         double *res0_n_dev, int not_r0, void *stream);

/* -- Fortran bindings (gfortran mangling, everything by reference) ------ */
/* ctx is passed as an integer(c_intptr_t) holding the context address.
 * status receives the return code.  Mirrors parms_solv_ in
 * pcns/src/parms_intf.h:9-11, the reference's own C-from-Fortran shim. */
void solv_gpu_create_(int64_t *ctx, int *device, int *status);
void solv_gpu_destroy_(int64_t *ctx, int *status);
void solv_gpu_matrix_set_(int64_t *ctx, int *n_cell, int *n_face,
                          const int *ip, const int *in, const double *p,
                          const double *n, const double *pl, int *status);
void solv_gpu_matrix_values_(int64_t *ctx, const double *p, const double *n,
                             const double *pl, int *status);
void solv_gpu_res_(int64_t *ctx, int *n_vc, const double *phi, double *res0,
                   double *res0_n, int *not_r0, int *status);
void solv_gpu_precond_(int64_t *ctx, int *imat, double *c, double *c_r,
                       int *status);
void solv_gpu_direct_(int64_t *ctx, int *imat, const double *c,
                      const double *c_r, double *x, const double *b,
                      int *status);
void solv_gpu_cg_(int64_t *ctx, int *imat, double *reduc, int *n_iter,
                  int *n_vc, double *phi, double *res0, double *res0_n,
                  int *not_r0, int *status);
void solv_gpu_bicg_(int64_t *ctx, int *imat, double *reduc, int *n_iter,
                    int *n_vc, double *phi, double *res0, double *res0_n,
                    int *not_r0, int *status);

#ifdef __cplusplus
}
#endif
#endif
