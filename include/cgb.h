/*
 * cgb.h -- C ABI of libcgb.so, a B200 (sm_100a) implementation of the NPB CG
 * benchmark's hot path: the makea matrix generator and the inverse power
 * iteration around conj_grad, from GMAP/NPB-GPU CUDA/CG/cg.cu.
 *
 * Conventions
 *   - Every entry point returns an int status (CGB_OK == 0).  Nothing here
 *     calls exit(); the reference does (cg.cu:1670-1674, :1748-1751, :1424-1426).
 *     cgb_last_error() gives a one-line description of the last failure on
 *     the calling thread.
 *   - Matrices use the reference's CSR layout: 0-based int32 rowstr[n+1] and
 *     colidx[nnz], FP64 a[nnz], columns sorted and unique within each row
 *     (cg.cu:1763-1784).
 *   - Vectors passed to the conj_grad-compatible call hold at least n+1
 *     doubles, as the reference's do (cg.cu:105-122, NA+2 entries).
 *   - A session is bound to one CUDA device and one stream; it is not
 *     re-entrant: one thread at a time per session.
 *   - There is no CPU fallback.  Without a usable sm_100 device the solver
 *     entry points fail with CGB_ERR_NO_DEVICE.  cgb_makea and the option
 *     helpers are host code and work without a GPU.
 */
#ifndef CGB_H
#define CGB_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
#define CGB_OK 0
#define CGB_ERR_INVALID 1     /* bad argument (sizes, seed, null pointer, mode) */
#define CGB_ERR_NOMEM 2       /* host or device allocation failed */
#define CGB_ERR_CAPACITY 3    /* caller's output arrays too small (*nnz_out has the need) */
#define CGB_ERR_CUDA 4        /* a CUDA runtime call failed */
#define CGB_ERR_TIMEOUT 5     /* a device-side wait hit its limit; the session stays usable */
#define CGB_ERR_NO_DEVICE 6   /* no CUDA device, or not compute capability 10.x */
#define CGB_ERR_STATE 7       /* call not valid in the session's current state */
#define CGB_ERR_NUMERIC 8     /* non-finite value met (NaN/Inf in A or a breakdown) */
#define CGB_ERR_BAD_MATRIX 9  /* CSR fails validation (rowstr not monotone, col out of range) */

const char *cgb_status_string(int status);
const char *cgb_last_error(void);
/* Library version as 10000*major + 100*minor + patch. */
int cgb_version(void);

/* ------------------------------------------------------------- generator */
/* Capacity the reference allocates for the CSR arrays: NZ = n*(nonzer+1)^2
 * (cg.cu:81).  Always >= the nnz cgb_makea produces. */
long long cgb_nz_bound(int n, int nonzer);

/* Replaces makea() (cg.cu:1303-1368) with sparse() (cg.cu:1611-1785) and the
 * LCG seeding of main() (cg.cu:404-408): the generator's state starts at
 * `seed` (314159265.0 for every NPB class), one draw is discarded, then n
 * sparse vectors are drawn and their scaled outer products summed into A,
 * with (rcond - shift) added to the diagonal.  Output is bit-identical to the
 * reference for any odd seed in (1, 2^46).
 *   rowstr: n+1 ints; colidx, a: nz_capacity entries each.
 *   *nnz_out receives the stored-entry count (also on CGB_ERR_CAPACITY).
 * The reference's firstrow/lastrow/firstcol/lastcol arguments are always the
 * full range (cg.cu:367-370) and its arow/acol/aelt/iv workspaces are
 * internal here.  Host code; needs no GPU. */
int cgb_makea(int n, int nonzer, double rcond, double shift, double seed, int *rowstr,
              int *colidx, double *a, long long nz_capacity, long long *nnz_out);

/* cgb_makea on CUDA device `device`: the vectors (sprnvc/vecset, one LCG
 * stream with rejection sampling, cg.cu:1798-1857) drawn in parallel -- every
 * possible start parsed at once, the chain from the first draw followed by
 * jump pointers -- and the assembly (the n*(nonzer+1)^2 outer-product
 * contributions, their per-row sort and in-order duplicate sums, sparse(),
 * cg.cu:1611-1785) on the device; only the running product of the
 * geometric weights stays on the host.  Same arguments, outputs and
 * bit-identical result as cgb_makea; nonzer <= 31.  CGB_ERR_CAPACITY also
 * when one row has more than 2048 contributions. */
int cgb_makea_device(int device, int n, int nonzer, double rcond, double shift, double seed,
                     int *rowstr, int *colidx, double *a, long long nz_capacity,
                     long long *nnz_out);

/* --------------------------------------------------------------- session */
typedef struct cgb_session cgb_session;

typedef struct cgb_options {
    int device;               /* CUDA device ordinal (reference: GPU_DEVICE, gpu.config:1) */
    int lanes_per_row;        /* SpMV lanes per row: 0 = autotuned, else 2, 4, 8, 16 or 32 */
    int block_threads;        /* threads per CTA of the persistent kernels: 0 = 512 */
    long long wait_limit_ns;  /* limit of every device-side wait (grid barrier): 0 = 2 s */
    int use_graph;            /* 1 (default): outer loop replayed as one CUDA graph */
    int keep_fp32_copy;       /* 1 (default): also hold FP32 values for the mixed mode */
    int spmv_kernel;          /* 0 = autotuned, 1 = row kernel on the CSR (gathered vector read
                                 through L1/L2), 2 = sliced kernel (a sliced copy of the matrix
                                 with 16-bit local columns, gathered vector staged in shared
                                 memory by TMA bulk copies), 3 = sliced with an L2 prefetch
                                 of each warp's slices of the next column block (0 times
                                 2 against 3 and keeps the faster) */
    int panel_rows;           /* sliced kernel: most rows a CTA sums at a time, rounded down to
                                 a multiple of 32 (0 = as many as its shared accumulators
                                 hold, about 2100).  A CTA with more rows walks them in row
                                 panels, every column block once per panel (class D: 5
                                 panels); every row is summed in the same order, the fused dot
                                 products add rows in another order.  No counterpart
                                 in the reference. */
} cgb_options;

void cgb_default_options(cgb_options *opts);

/* Uploads the CSR (host pointers) and sets the session up (the part of the
 * reference's setup_gpu that matters, cg.cu:1390-1603).  The matrix is
 * validated first.  `opts` may be NULL for the defaults. */
int cgb_create(int n, const int *rowstr, const int *colidx, const double *a,
               const cgb_options *opts, cgb_session **out);

/* A session on the generator's matrix (cgb_makea_device's arguments; the
 * device is opts->device) without the CSR ever leaving the device: the
 * generated arrays become the session's copy.  Same matrix, bit for bit, as
 * cgb_create on cgb_makea's output.  No counterpart in the reference. */
int cgb_create_generated(int n, int nonzer, double rcond, double shift, double seed,
                         const cgb_options *opts, cgb_session **out);

/* Replaces the session's matrix values/structure with another CSR of the
 * same order n from host memory (an H2D copy; same validation). */
int cgb_upload(cgb_session *s, const int *rowstr, const int *colidx, const double *a);

int cgb_destroy(cgb_session *s);

/* Same call surface as the reference conj_grad (cg.cu:225-233, :653-801), on
 * host pointers: 25 CG iterations on A z = x from z = 0, then
 * rnorm = ||x - A z||.  On return z, p, q, r hold what the reference leaves
 * there (r = A z).  If colidx/rowstr/a differ from the arrays the session was
 * created or last uploaded with, they are uploaded first (n is the
 * session's).  Vectors: n+1 doubles (entry n copied as the reference sets it). */
int cgb_conj_grad(cgb_session *s, const int *colidx, const int *rowstr, const double *x,
                  double *z, const double *a, double *p, double *q, double *r, double *rnorm);

/* Tells the session that the caller changed, in place, the host arrays it was
 * created or last uploaded with: the next cgb_conj_grad uploads them again
 * even though the pointers are the same.  (The reference's CPU conj_grad
 * reads a[] on every call, cg.cu:653-801; its GPU path copies the matrix once
 * in setup_gpu, cg.cu:1390-1603.  cgb_conj_grad compares pointers only, so
 * without this call an edit in place is not seen.)  No other effect. */
int cgb_matrix_changed(cgb_session *s);

/* ------------------------------------------------------- power iteration */
#define CGB_MODE_FP64 0         /* reference algorithm: fixed cgitmax FP64 CG steps */
#define CGB_MODE_FP64_TOL 1     /* FP64 CG stopped at relative residual tol */
#define CGB_MODE_MIXED 2        /* FP32 SpMV inside FP64 iterative refinement */
#define CGB_MODE_MIXED_LEARNED 3 /* MIXED, preconditioned by M = F^T F (cgb_set_preconditioner),
                                   falling back to plain CG when it stalls */

typedef struct cgb_solve_params {
    int niter;          /* outer steps (reference NITER, setparams.cpp:751-785) */
    double shift;       /* zeta = shift + 1/(x.z) (cg.cu:513) */
    int mode;           /* CGB_MODE_* */
    int cgitmax;        /* inner iterations: exact count in FP64 mode (25 = reference),
                           the cap in the tolerance modes */
    double tol;         /* tolerance modes: stop when ||r|| <= tol * ||x|| */
    int refresh_every;  /* MIXED*: replace r by x - A z in FP64 (and restart) at least every
                           k steps (10); also when the recursive residual fell 1e-6 since the
                           last replacement, and before accepting convergence */
    int recycle;        /* tolerance modes: start each solve from the Galerkin solution on the
                           last `recycle` power-iteration iterates (0..4, default 4; 0 = from
                           z = 0).  The iterates span a Krylov space of A, and A times each
                           comes from the previous step's residual product, so the start
                           costs dot products only.  Ignored in CGB_MODE_FP64. */
} cgb_solve_params;

void cgb_default_solve_params(cgb_solve_params *p);

typedef struct cgb_solve_result {
    double zeta;          /* final zeta */
    double rnorm;         /* final ||x - A z|| (FP64) */
    double device_ms;     /* device time of the whole outer loop (CUDA events) */
    int total_inner;      /* inner iterations summed over the outer steps */
    int fallbacks;        /* outer steps that fell back to plain FP64 CG */
    int refreshes;        /* true-residual replacements (MIXED*) summed over the outer steps */
} cgb_solve_result;

/* The reference's timed region (cg.cu:491-522): x = 1, then niter times
 * { z = conj_grad(x); zeta = shift + 1/(x.z); x = z/||z|| }.  Each trace
 * (nullable) gets niter entries: zeta, rnorm, inner iterations.  x_out
 * (nullable) receives the final x (n doubles).  res may be NULL. */
int cgb_power_iterate(cgb_session *s, const cgb_solve_params *params, double *zeta_trace,
                      double *rnorm_trace, int *iters_trace, double *x_out,
                      cgb_solve_result *res);

/* Installs the preconditioner of CGB_MODE_MIXED_LEARNED: the factor F of
 * M = F^T F, which approximates (-A)^-1 (A is negative definite; the solver
 * runs CG on -A).  F is lower triangular in CSR (n+1 row pointers, columns
 * <= row, every row holding a positive diagonal).  On the device the
 * values are FP32 (row plan) or BF16 in sliced copies that gather a BF16
 * vector (sliced plan).  The learned factor is G diag(-A)^-1/2 with G from
 * cgb_gnn_infer; F = diag(-A)^-1/2 is Jacobi.  No counterpart in the
 * reference. */
int cgb_set_preconditioner(cgb_session *s, const int *fptr, const int *fcol, const double *fval);

/* --------------------------------------------- learned preconditioner */
/* A message-passing network over the sparsity graph of A (3 layers, width 32,
 * FP32 weights) that emits G on A's lower pattern, g_ii > 0, so M = G^T G is
 * SPD; it is trained to make M / delta approximate (-A)^-1 on residual
 * vectors (delta = mean of diag(-A)).  Forward, backward (training) and inference
 * run on the GPU.  No counterpart in the reference. */
typedef struct cgb_gnn cgb_gnn;
typedef struct cgb_gnn_graph cgb_gnn_graph;

int cgb_gnn_param_count(void);
/* New model with deterministic initial weights from `seed`. */
int cgb_gnn_create(int device, unsigned seed, cgb_gnn **out);
int cgb_gnn_destroy(cgb_gnn *m);
int cgb_gnn_get_params(cgb_gnn *m, float *out, int count);
/* Loads weights (and resets the optimiser state). */
int cgb_gnn_set_params(cgb_gnn *m, const float *in, int count);
/* A matrix (the generator's CSR, negative diagonal) prepared for the model. */
int cgb_gnn_graph_create(cgb_gnn *m, int n, const int *rowstr, const int *colidx, const double *a,
                         cgb_gnn_graph **out);
int cgb_gnn_graph_destroy(cgb_gnn_graph *g);
/* n, strict-lower entry count, the per-row factor scale 1/sqrt(delta) (n
 * doubles); outputs nullable. */
int cgb_gnn_graph_info(cgb_gnn_graph *g, int *n, long long *nnz_low, double *dscale_out);
/* Loss and gradient (cgb_gnn_param_count floats) on 32 probe vectors: the
 * caller's (`probes`, n x 32 row-major) or, when NULL, generated from `seed`:
 * normal vectors, or with cg_steps > 0 the residuals after cg_steps batched
 * CG steps on them (residual histories).  Outputs nullable. */
int cgb_gnn_loss_grad(cgb_gnn *m, cgb_gnn_graph *g, const float *probes, unsigned seed,
                      int cg_steps, float *loss, float *grad);
/* One Adam step on generated probes; *loss (nullable) is the step's loss. */
int cgb_gnn_train_step(cgb_gnn *m, cgb_gnn_graph *g, unsigned seed, int cg_steps, float lr,
                       float *loss);
/* G for the graph: strict lower values (graph order: rows ascending, then
 * the CSR order of the row) and the diagonal; outputs nullable. */
int cgb_gnn_infer(cgb_gnn *m, cgb_gnn_graph *g, float *goff, float *gdiag);
/* Infers G and installs F = G / sqrt(delta) as the session's preconditioner. */
int cgb_gnn_attach(cgb_gnn *m, cgb_gnn_graph *g, cgb_session *s);
/* The same for system `sys` of a batch (g built on that system's matrix). */
typedef struct cgb_batch cgb_batch;
int cgb_gnn_attach_batch(cgb_gnn *m, cgb_gnn_graph *g, cgb_batch *b, int sys);

/* ------------------------------------------------------------- batches */
/* Many independent systems of uneven order (n <= 27000 each) solved in one
 * persistent cooperative launch: every CTA takes work from a device queue
 * (the largest systems first) and runs a system's whole inverse power
 * iteration, alone or -- the largest systems -- as one of a team of CTAs
 * that split its rows, the search vector in each CTA's shared memory.  Lanes per row per system and the
 * block shape come from cgb_batch_tune (defaults otherwise).  In
 * CGB_MODE_MIXED a system whose iteration meets p.Ap >= 0 (not negative
 * definite), a non-finite residual, or does not converge within cgitmax is
 * solved again at once, by the same CTA in the same launch, with the FP64
 * reference algorithm (25 steps, the reference's cgitmax); its status is
 * then 1 and its outputs are that solve's.  No counterpart in the
 * reference (it solves one system). */
typedef struct cgb_batch cgb_batch;

typedef struct cgb_batch_params {
    int niter;          /* outer steps per system */
    int mode;           /* CGB_MODE_FP64 (fixed cgitmax steps), CGB_MODE_MIXED or
                           CGB_MODE_MIXED_LEARNED (MIXED preconditioned by each system's
                           M = F^T F, cgb_batch_set_preconditioner) */
    int cgitmax;        /* inner steps: exact (FP64) or cap (MIXED*) */
    double tol;         /* MIXED*: stop when ||x - A z|| <= tol ||x|| */
    int refresh_every;  /* MIXED*: true-residual replacement at least every k steps */
    int recycle;        /* MIXED*: Galerkin start on the last `recycle` iterates (0..4, default 4) */
} cgb_batch_params;

void cgb_default_batch_params(cgb_batch_params *p);
/* nsys systems: n[s], and rowstr[s] / colidx[s] / a[s] host CSR arrays, shift[s]. */
int cgb_batch_create(int device, int nsys, const int *n, const int *const *rowstr,
                     const int *const *colidx, const double *const *a, const double *shift,
                     cgb_batch **out);
int cgb_batch_destroy(cgb_batch *b);
/* Per-system outputs (nsys entries each, nullable): final zeta, rnorm, inner
 * iterations summed over the outer steps, status (0; 1 = re-solved in FP64
 * with the reference algorithm; 2 = CGB_MODE_MIXED_LEARNED, where some outer
 * step's preconditioned iteration stalled and that step finished as plain
 * CG, cgb_batch_fallbacks counts them); *device_ms the launch's device time. */
int cgb_batch_solve(cgb_batch *b, const cgb_batch_params *params, double *zeta, double *rnorm,
                    int *iters, int *status, double *device_ms);
/* Autotuner: times the batch for each candidate block shape and lane policy
 * (row-length thresholds t0 < t1 < t2 for 8 / 16 / 32 lanes per row, 4 below
 * t0), then for the best of those each team policy, keeps the fastest for
 * later solves and reports it (cgb_batch_policy gives the rest). */
int cgb_batch_tune(cgb_batch *b, const cgb_batch_params *params, int *block, double *t0,
                   double *t1, double *t2, double *best_ms);
/* The batch's current policy: entries a lane loads ahead (4 or 8), the team
 * fraction, and how many systems the last launch gave a team of 2, 4 or 8
 * CTAs (a system gets one while its SpMV work per CTA is above team_frac x
 * the batch's work per resident CTA; the members split its rows and
 * exchange the search vector through global memory at each update, with
 * bounded waits: CGB_ERR_TIMEOUT past 2 s).  Any output may be NULL. */
int cgb_batch_policy(cgb_batch *b, int *unroll, double *team_frac, int *teams);
/* Sets the team fraction (0 = every system on one CTA; default 0.5). */
int cgb_batch_set_team_frac(cgb_batch *b, double team_frac);
/* The preconditioner of system `sys` in CGB_MODE_MIXED_LEARNED: M = F^T F with
 * F lower triangular in CSR (n+1 row pointers, columns <= row, a positive
 * diagonal in every row), as cgb_set_preconditioner takes it; stored with
 * the diagonal in FP32 and the other entries as BF16 values with 16-bit
 * columns.  Every system needs one before a learned
 * solve (the learned factor is G diag(-A)^-1/2 with G from cgb_gnn_infer;
 * cgb_gnn_attach_batch installs it).  In the solve, both factor products
 * gather from a shared-memory copy of the vector.  No counterpart in the
 * reference. */
int cgb_batch_set_preconditioner(cgb_batch *b, int sys, const int *fptr, const int *fcol,
                                 const double *fval);
/* Outer steps per system (nsys ints) of the last learned solve that fell back
 * to plain CG (0 for the other modes). */
int cgb_batch_fallbacks(cgb_batch *b, int *fallbacks);

/* ---------------------------------------------------------- diagnostics */
/* Time `reps` launches of the standalone SpMV (q = A p with the p.q
 * reduction fused, the operation of kernel three + four, cg.cu:937-1004) of
 * the session's plan, FP64 or (fp32 != 0) the FP32 copy, and return the mean
 * device milliseconds per launch. */
int cgb_time_spmv(cgb_session *s, int reps, int fp32, double *ms_per_launch);

/* Per-launch device time of the FP64 outer step kernel (`niter` steps of the
 * reference algorithm with events between the kernels, mean in ms) and what
 * one kernel boundary costs the solve's CUDA graph (graph_gap_ms): graphs of
 * niter and of 1 launches of an empty kernel with the outer step's shape
 * (grid, block, shared memory, cooperative), timed with events, their
 * difference over niter - 1 (best of five; ms per outer step). */
int cgb_time_outer_steps(cgb_session *s, int niter, double shift, double *kernel_ms,
                         double *graph_gap_ms);

/* The kernel configuration the session's autotuner chose: kind 1 = row,
 * 2 = sliced, 3 = sliced with the L2 prefetch of each warp's next column
 * block (the FP64 and FP32 SpMVs of the matrix; not the factor products);
 * lanes per row (row kind), grid, block, dynamic shared memory
 * bytes, and the stored entries of the layout the SpMV streams (nnz for the
 * CSR, nnz plus slice padding for the sliced copy).  Any output may be NULL. */
int cgb_plan_info(cgb_session *s, int *kind, int *lanes_per_row, int *grid, int *block,
                  long long *smem_bytes, long long *layout_entries);

/* Bytes of the sliced matrix stream that the solves keep resident in L2
 * from one product to the next (a fraction budget / stream of its lines is
 * loaded at L2 priority evict_last, the rest evict_first); chosen by the
 * autotuner among 0, 48 MB and 64 MB; 0 for the row plan.  Products whose
 * stream fits the budget read the matrix from L2 after the first. */
int cgb_plan_l2_keep(cgb_session *s, double *bytes);
/* Overrides the autotuner's choice (>= 0; 0 = pure stream).  Results do not
 * depend on it: it changes cache priorities only. */
int cgb_set_l2_keep(cgb_session *s, double bytes);
/* Row panels of the sliced plan: each CTA walks its rows of A in `*panels`
 * pieces and the preconditioner's copies in `*prec_panels` (1 = one walk;
 * more above about 2100 rows a CTA, or below opts->panel_rows); 0 and 0 for
 * the row plan.  No counterpart in the reference. */
int cgb_plan_panels(cgb_session *s, int *panels, int *prec_panels);

/* The checked build (lib/libcgb_checked.so, compiled with -DCGB_CHECKED)
 * tests every index of the single-system SpMVs against its buffer and skips
 * an access that would leave it.  *word receives the first failure since the
 * last call (0 none; 1 matrix stream, 2 gathered vector, 3 output row) and
 * is reset; -1 from the normal build. */
int cgb_check_status(int *word);

/* Device microseconds per grid barrier: `iters` barriers back to back in
 * one cooperative launch of the plan's grid and the FP64 outer step's
 * block size (after a short warm-up launch). */
int cgb_time_barrier(cgb_session *s, int iters, double *us_per_barrier);

/* Grid barrier time-out self-test: runs a 2-CTA kernel whose second CTA never
 * arrives, with a wait limit of `limit_ns`, and reports the status the host
 * reads back (CGB_ERR_TIMEOUT expected).  The session stays usable. */
int cgb_selftest_wait_timeout(cgb_session *s, long long limit_ns, int *device_status);

/* conj_grad for callers that cannot allocate GPU memory.  No counterpart in
 * the reference: it exists for hosts that forbid device allocation on this
 * path (their device memory is handed out by their own pool, or the loop must
 * never allocate).  Same computation as cgb_conj_grad (25 CG iterations from
 * z = 0, then rnorm = ||x - A z||), but every pointer is caller-owned device
 * memory and the work space (p, q, r, partial sums, barrier words) sits in
 * one fixed array inside the library; this call allocates nothing.
 *   d_rowstr n+1, d_colidx / d_a nnz entries (sorted or not; d_a 16-byte,
 *   d_colidx 8-byte aligned, as cudaMalloc returns them), d_x and d_z
 *   n+1 doubles (entry n as the reference sets it), d_rnorm one double,
 *   d_status (nullable) one int: 0, or the device status on a failed wait.
 *   stream: a cudaStream_t (NULL = legacy default stream).  Asynchronous:
 *   synchronise the stream before reading the outputs.  A solve that gave
 *   up on a device wait leaves *d_rnorm NaN (and *d_status nonzero), so a
 *   caller that passes no status word still sees the failure.
 * Limit: n <= 262144 (CGB_ERR_CAPACITY above).  The array (about 6.3 MB) is
 * held on every GPU that loads the library until exit.  Calls share it:
 * calls that overlap on the GPU race, so serialise them.  Runs on the
 * calling thread's current device; the first call on a device (per CUDA
 * context: again after a cudaDeviceReset) looks the array up there and
 * caches its address, so make that first call before any stream capture. */
int cgb_conj_grad_noalloc(int n, long long nnz, const int *d_rowstr, const int *d_colidx,
                          const double *d_a, const double *d_x, double *d_z, double *d_rnorm,
                          int *d_status, void *stream);

/* ---- One system split by rows over several GPUs -----------------------
 * The reference algorithm (conj_grad of cg.cu:653-801, cgitmax FP64 steps,
 * inside the outer loop of cg.cu:485-520) on a matrix whose rows are
 * divided among `world` ranks, one process (or one call) per GPU.  Rank r
 * owns the rows [r m, min((r+1) m, n)), m = ceil(n / world)
 * (cgb_part_rows), stored as CSR with GLOBAL column indices.  Per CG step
 * the ranks exchange the search vector once (an all-gather of their rows)
 * and two scalars (all-reduces of p.q and r.r); scalars stay on the device.
 * The result is the reference's to rounding: the sums are ordered
 * differently than on one GPU, but identically from run to run. */
typedef struct cgb_part cgb_part;

#define CGB_NCCL_ID_BYTES 128

/* Rows [*row0, *row1) of `rank` among `world` for an n-row matrix.  No GPU
 * needed. */
int cgb_part_rows(int n, int world, int rank, int *row0, int *row1);

/* A new NCCL unique id (CGB_NCCL_ID_BYTES bytes) for rank 0 to hand to the
 * others.  NCCL is loaded on first use (libnccl.so.2); CGB_ERR_STATE when it
 * cannot be found. */
int cgb_nccl_unique_id(void *id_out);

/* One rank's share.  rowstr (row1 - row0 + 1 entries, rowstr[0] == 0),
 * colidx and a are this rank's rows of the global CSR: its rows
 * row0..row1-1 with their global columns.  With nccl_id (from
 * cgb_nccl_unique_id on one rank, the same bytes on all) the call joins the
 * world's communicator, a collective call: every rank makes it.  Without it
 * the part can only be driven by cgb_part_group_power_iterate (world 1 also
 * by cgb_part_power_iterate). */
int cgb_part_create(int device, int n, int world, int rank, const int *rowstr, const int *colidx,
                    const double *a, const void *nccl_id, cgb_part **out);
int cgb_part_destroy(cgb_part *p);

/* Joins the world's NCCL communicator (a collective call: every rank makes
 * it with the same id) -- for parts created without an id, e.g. after every
 * rank has checked that all ranks built their blocks. */
int cgb_part_join(cgb_part *p, const void *nccl_id);

/* Longest a rank waits for a solve's collectives (default 600 s).  A rank
 * whose peers fail (NCCL's asynchronous error) or stay silent past the limit
 * aborts its communicator and returns CGB_ERR_TIMEOUT / CGB_ERR_CUDA instead
 * of waiting for ever; the part then makes no more collectives. */
int cgb_part_set_wait_limit(cgb_part *p, double seconds);

/* The part's rows [*row0, *row1) and its stored entries.  Any output may be
 * NULL. */
int cgb_part_info(const cgb_part *p, int *row0, int *row1, long long *nnz);

/* One rank's share of the NPB matrix makea(n, nonzer, rcond, shift, seed)
 * generated on the device: only this rank's rows are assembled (the same
 * entries, bit for bit, as those rows of cgb_makea), so no rank -- and no
 * host -- ever holds the whole matrix.  Each rank's block needs fewer than
 * 2^31 entries; the whole matrix may have more (class E: about 6.4e9). */
int cgb_part_create_generated(int device, int n, int nonzer, double rcond, double shift, double seed,
                              int world, int rank, const void *nccl_id, cgb_part **out);

/* niter outer steps of the power iteration from x = 1, every rank calling
 * it with the same arguments (collective).  zeta_trace / rnorm_trace (niter
 * doubles each, nullable) get every step's zeta and ||x - A z||, the same on
 * every rank; device_ms the device time of this rank's steps. */
int cgb_part_power_iterate(cgb_part *p, int niter, double shift, int cgitmax, double *zeta_trace,
                           double *rnorm_trace, double *device_ms);

/* The same solve for all `k` == world ranks of one world from one process,
 * all parts on one device and created without an NCCL id: the ranks'
 * kernels run one after another on one stream and the exchanges are device
 * copies and a summing kernel, so the partitioned data flow runs -- and is
 * tested -- on a single GPU.  parts[i] must be rank i. */
int cgb_part_group_power_iterate(cgb_part **parts, int k, int niter, double shift, int cgitmax,
                                 double *zeta_trace, double *rnorm_trace, double *device_ms);

/* ---- NPB MG: the V-cycle multigrid benchmark ----------------------------
 * The reference's MG (CUDA/MG/mg.cu): a multigrid V-cycle for the 3-D
 * Poisson problem on a periodic 2^lt cube.  The right-hand side v is zero
 * except +1 at the ten largest and -1 at the ten smallest values of the LCG
 * laid over the grid (zran3, mg.cu:2175-2303); u starts at zero.  Classes
 * (mg.cu:388-410): S lt 5 nit 4, W 7/4, A 8/4, B 8/20, C 9/20, D 10/50;
 * smoother 0 (the S(a) coefficients) for S, W, A and 1 (S(b)) otherwise
 * (mg.cu:422-442).  Grids are (2^lt + 2)^3 doubles with one ghost layer. */
typedef struct cgb_mg cgb_mg;

/* Grids for every level on `device`, v generated on the device. */
int cgb_mg_create(int device, int lt, int smoother, cgb_mg **out);
int cgb_mg_destroy(cgb_mg *g);

/* The reference's timed region (mg.cu:498-508) from u = 0: resid, norm,
 * nit x (V-cycle mg3P, resid), norm.  rnm2 = sqrt(sum r^2 / n^3), rnmu =
 * max |r| of the final residual (norm2u3, mg.cu:1201-1230); device_ms the
 * device time of the region (any output may be NULL).  Verify rnm2 against
 * the class's value at relative 1e-8 (mg.cu:528-543). */
int cgb_mg_run(cgb_mg *g, int nit, double *rnm2, double *rnmu, double *device_ms);

/* The finest level's u (which 0), v (1) or r (2): (2^lt + 2)^3 doubles,
 * index (i3 * m + i2) * m + i1. */
int cgb_mg_read(cgb_mg *g, int which, double *out, long long count);

/* zran3's points (i1, i2, i3), ten each: plus in ascending value (largest
 * last), minus in descending value (smallest last), the reference's lists. */
int cgb_mg_points(cgb_mg *g, int *plus, int *minus);

/* One operator on host grids (tests): op 0 resid (in1 u, in2 v -> out r),
 * 1 psinv (in1 r; out u, updated), 2 rprj3 (in1 r of side m -> out of side
 * m/2 + 1), 3 interp (in1 z of side m; out u of side 2m - 2, added to),
 * 4 interp assigning.  m even, at least 4. */
int cgb_mg_apply(int device, int op, int m, int smoother, const double *in1, const double *in2,
                 double *out);

/* ---- NPB EP: Gaussian pairs from one random stream -----------------------
 * The reference's EP (CUDA/EP/ep.cu): 2^m pairs of uniform deviates from the
 * LCG seeded 271828183 (multiplier 5^13), the pairs inside the unit disc
 * turned into Gaussian deviates; their sums sx, sy and the counts q[0..9]
 * of pairs with floor(max(|X|, |Y|)) = l.  Classes (setparams.cpp:826-845):
 * m = 24 S, 25 W, 28 A, 30 B, 32 C, 36 D, 40 E; verify sx, sy at relative
 * 1e-8 against ep.cu:189-212.  device_ms: the kernel's device time.  Any
 * output may be NULL; q holds 10 doubles. */
int cgb_ep_run(int device, int m, double *sx, double *sy, double *q, double *device_ms);

/* ---- NPB IS: ranking integer keys ---------------------------------------
 * The reference's IS (CUDA/IS/is.cu): 2^total_log2 keys below 2^max_log2,
 * key i = (int)(2^max_log2 / 4 * (r1 + r2 + r3 + r4)) from the LCG's draws
 * 4i+1 .. 4i+4 (seed 314159265, multiplier 5^13), generated on the device.
 * Classes (is.cu:86-140): S 16/11, W 20/16, A 23/19, B 25/21, C 27/23,
 * D 31/27; cls 'U' takes any sizes and skips the class's partial checks. */
typedef struct cgb_is cgb_is;

int cgb_is_create(int device, char cls, int total_log2, int max_log2, cgb_is **out);
int cgb_is_destroy(cgb_is *s);

/* main's sequence (is.cu:398-505): one untimed ranking pass, the timed ten
 * passes (each rewrites two keys, counts the keys by value, takes the
 * running sums and checks the class's five test ranks, is.cu:157-190), then
 * the full check (every key placed by the last running sums, the result in
 * order).  *passed: the checks passed -- 5 x 10 + 1 = 51 verifies (1 for
 * cls 'U'); *device_ms: the ten passes' device time.  Repeatable: the keys
 * a run rewrites are restored first. */
int cgb_is_run(cgb_is *s, long long *passed, double *device_ms);

/* After a run: which 0 the keys (int32, 2^total_log2), 1 per value the
 * number of keys below it (uint32, 2^max_log2), 2 the sorted keys (int32). */
int cgb_is_read(cgb_is *s, int which, void *out, long long count);

/* ---- NPB FT: a 3-D FFT evolution ---------------------------------------
 * The reference's FT (CUDA/FT/ft.cu): an nx x ny x nz complex field (x
 * fastest, interleaved real and imaginary doubles) from the LCG's stream
 * (element e: draws 2e+1, 2e+2 after the seed 314159265), transformed
 * forward once, then each iteration multiplied by exp(-4 alpha pi^2 |k|^2)
 * (alpha 1e-6), transformed back and checksummed.  Dimensions: powers of
 * two in [32, 2048].  Classes (setparams.cpp:797-803): S 64^3 (6
 * iterations), W 128x128x32 (6), A 256x256x128 (6), B 512x256x256 (20),
 * C 512^3 (20), D 2048x1024x1024 (25). */
typedef struct cgb_ft cgb_ft;

/* Replaces main's setup_gpu (ft.cu:1469-1636): the device arrays. */
int cgb_ft_create(int device, int nx, int ny, int nz, cgb_ft **out);
int cgb_ft_destroy(cgb_ft *f);

/* main's timed region (ft.cu:391-408): the index map, the initial
 * conditions, the roots, the forward transform (x, y, z lines, exponent
 * sign +1), then niter x (evolve, the inverse transform: z, y, x lines,
 * sign -1, and the checksum of ft.cu:1124-1153).  sums: 2 niter doubles
 * (real, imaginary of each iteration's checksum), verified by a class at
 * relative 1e-12 (ft.cu:1638-1830); device_ms: the region's device time.
 * niter in [1, 64]; either output may be NULL. */
int cgb_ft_run(cgb_ft *f, int niter, double *sums, double *device_ms);

/* After a run: which 0 u0 (the evolved field in Fourier space), 1 u1 (the
 * last inverse transform), 2 the twiddle factors (nx ny nz doubles);
 * count: doubles available at out (2 nx ny nz for u0 and u1). */
int cgb_ft_read(cgb_ft *f, int which, double *out, long long count);

/* Host memory that the device copies at full speed (cudaHostAlloc). */
int cgb_host_alloc(void **ptr, long long bytes);
int cgb_host_free(void *ptr);

/* Device count and properties, for drivers and tests. */
int cgb_device_info(int device, int *sm_count, int *cc_major, int *cc_minor,
                    long long *global_mem_bytes);

#ifdef __cplusplus
}
#endif
#endif /* CGB_H */
