/*
 * fluxion_cuda.h -- C ABI of the B200 (sm_100a) backend for fluxion's
 * matrix-free solve path.
 *
 * One `extern "C"` entry point per operation of the reference's backend
 * trait `fluxion_core::Backend` (crates/core/src/backend.rs:43-406), plus
 * the non-trait fast paths the reference runtime already calls on its GPU
 * backend (crates/backend-hip/src/backend.rs:463-668) and the solver
 * structs of crates/runtime.  Every function returns an `int` status
 * (FX_OK == 0) and writes results through out-pointers; on error,
 * fx_last_error() returns a message for the calling thread.
 *
 * Conventions
 *  - Buffers are opaque handles owned by the library (the reference's
 *    `BackendBuffer`, crates/core/src/backend.rs:13-36): fx_alloc returns a
 *    zero-filled buffer, fx_free releases it (HipBuffer's Drop,
 *    crates/backend-hip/src/buffer.rs:81-87).
 *  - A grid is rows x cols INCLUDING the boundary ring, row-major
 *    (crates/core/src/grid.rs:4-9, :59-61).
 *  - Every operation is enqueued on the context's stream in call order.
 *    Calls that return a host scalar (reductions, solves) synchronise.
 *  - F64 buffers compute in double precision, F32 buffers in single
 *    precision; all reductions accumulate in compensated double precision
 *    and are bitwise deterministic for a given length.
 *  - Status codes map onto the reference's `CoreError` variants
 *    (crates/core/src/error.rs:4-20).
 */
#ifndef FLUXION_CUDA_H
#define FLUXION_CUDA_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ */
/* Status, dtypes, descriptors                                        */
/* ------------------------------------------------------------------ */

enum {
    FX_OK = 0,
    FX_ERR_DIMENSION_MISMATCH = 1, /* CoreError::DimensionMismatch */
    FX_ERR_INVALID_GRID = 2,       /* CoreError::InvalidGrid */
    FX_ERR_INVALID_STENCIL = 3,    /* CoreError::InvalidStencil */
    FX_ERR_BACKEND = 4,            /* CoreError::BackendError (CUDA failure) */
    FX_ERR_INVALID_ARGUMENT = 5,   /* null handle, dtype mismatch, bad parameter */
    FX_ERR_UNSUPPORTED = 6,        /* e.g. periodic boundaries (ops.rs:9-23) */
    FX_ERR_NO_DEVICE = 7           /* no CUDA device / driver */
};

enum { FX_F32 = 0, FX_F64 = 1 }; /* crates/core/src/dtype.rs:2-5 */

/* crates/core/src/boundary.rs:2-15 */
enum { FX_BC_DIRICHLET = 0, FX_BC_NEUMANN = 1, FX_BC_ROBIN = 2, FX_BC_PERIODIC = 3 };

typedef struct {
    int kind;
    double a; /* Dirichlet value | Neumann flux | Robin alpha */
    double b; /* Robin beta */
    double g; /* Robin g */
} fx_bc;

/* Boundaries {top, bottom, left, right} (crates/core/src/boundary.rs:17-24). */
typedef struct {
    fx_bc side[4];
} fx_boundaries;

/* crates/core/src/grid.rs:3-9 */
typedef struct {
    size_t rows, cols;
    double dx, dy;
} fx_grid;

/* crates/core/src/stencil.rs:1-14: n entries of (dr, dc, weight). */
typedef struct {
    int n;
    const int *dr;
    const int *dc;
    const double *w;
} fx_stencil;

/* SolveStats (crates/runtime/src/cg.rs:9-29). */
enum { FX_CONVERGED = 0, FX_MAX_ITERATIONS = 1, FX_BREAKDOWN = 2 };
typedef struct {
    size_t iterations;
    double residual;
    int reason;
} fx_stats;

typedef struct fx_ctx fx_ctx;
typedef struct fx_buf fx_buf;
typedef struct fx_precond fx_precond;
typedef struct fx_mg fx_mg;
typedef struct fx_cg fx_cg;
typedef struct fx_pipelined_cg fx_pipelined_cg;
typedef struct fx_bicgstab fx_bicgstab;
typedef struct fx_gmres fx_gmres;
typedef struct fx_graph fx_graph;
typedef struct fx_fcg fx_fcg;
typedef struct fx_fgmres fx_fgmres;
typedef struct fx_op fx_op;
typedef struct fx_cdmg fx_cdmg;
typedef struct fx_ir fx_ir;
typedef struct fx_lsm fx_lsm;
typedef struct fx_lsm_data fx_lsm_data;
typedef struct fx_batch fx_batch;

/* ------------------------------------------------------------------ */
/* Context (HipBackend::new / singleton, backend-hip/src/backend.rs:103-264) */
/* ------------------------------------------------------------------ */

const char *fx_last_error(void);
int fx_version(void);
int fx_device_count(int *count);
/* Backend::name (backend.rs:47) -> "cuda" */
const char *fx_backend_name(void);
int fx_ctx_create(int device, fx_ctx **out);
int fx_ctx_destroy(fx_ctx *ctx);
int fx_ctx_synchronize(fx_ctx *ctx);
/* Use an external cudaStream_t (e.g. the caller's); NULL restores the context's own.  Waits for
 * the old stream first.  FX_ERR_INVALID_ARGUMENT while the current stream is being captured
 * (between fx_graph_begin and fx_graph_end, or in a caller's capture) and `stream` differs. */
int fx_ctx_set_stream(fx_ctx *ctx, void *stream);
void *fx_ctx_get_stream(fx_ctx *ctx);
/* Programmatic dependent launch for this context's kernels: 1 (the default) lets each kernel's
 * blocks be scheduled while the previous kernel drains and wait on the SM for its results; 0
 * launches them plainly.  A context that shares the GPU with other busy contexts may do better
 * with 0, since the waiting blocks hold SM slots that the others' kernels could use.  Results
 * are the same either way. */
int fx_ctx_set_pdl(fx_ctx *ctx, int enabled);
/* Number of kernels this context has launched (for launch accounting). */
unsigned long long fx_ctx_launch_count(fx_ctx *ctx);
/* Per-kernel timing: from fx_ctx_timing_begin until fx_ctx_timing_end, every launch of the
 * kernel named `kernel` is bracketed by CUDA events on the launching stream.  End returns the
 * summed device time, the launch count and the summed grid points those launches covered. */
int fx_ctx_timing_begin(fx_ctx *ctx, const char *kernel);
int fx_ctx_timing_end(fx_ctx *ctx, double *total_ms, unsigned long long *launches,
                      double *total_points);
/* Like fx_ctx_timing_end, but also returns up to `max` individual launches in launch order:
 * device ms, grid points, and the launch's algorithmic DRAM bytes (0 where the launcher does not
 * state them; `bytes` may be NULL) through ms[] / points[] / bytes[]; *count = number written. */
int fx_ctx_timing_end_records(fx_ctx *ctx, double *ms, double *points, double *bytes, size_t max,
                              size_t *count);

/* Graph capture and replay (HipGraph, backend-hip/src/graph.rs:14-108).  Between begin and end,
 * the operations enqueued on the context's stream are recorded (relaxed capture mode, as the
 * reference's) instead of run; launch replays them on the context's stream.  Operations that
 * return a host value (reductions, copies to the host, solves) cannot be recorded: they fail
 * during capture and end then reports the capture as failed. */
int fx_graph_begin(fx_ctx *ctx);                          /* HipGraph::begin_capture :35-46 */
int fx_graph_end(fx_ctx *ctx, fx_graph **out);            /* HipGraph::end_capture :48-70 */
int fx_graph_launch(fx_ctx *ctx, const fx_graph *graph);  /* HipGraph::launch :72-85 */
int fx_graph_destroy(fx_graph *graph);                    /* Drop for HipGraph :88-99 */

/* ------------------------------------------------------------------ */
/* Memory (Backend::allocate / upload_f64 / upload_f32, backend.rs:49-77;
 * BackendBuffer::copy_to_host_*, :25-35)                             */
/* ------------------------------------------------------------------ */

int fx_alloc(fx_ctx *ctx, size_t len, int dtype, fx_buf **out);
/* Test hook (no counterpart in the reference): the next `count` buffer allocations (fx_alloc and
 * everything built on it: uploads, solver and multigrid creation) fail with FX_ERR_BACKEND, as an
 * out-of-memory would; 0 clears it.  Process-wide. */
int fx_test_fail_allocations(int count);
int fx_upload_f64(fx_ctx *ctx, const double *data, size_t len, fx_buf **out);
int fx_upload_f32(fx_ctx *ctx, const float *data, size_t len, fx_buf **out);
/* Non-owning view of existing device memory (interop); fx_free releases only the handle. */
int fx_wrap(fx_ctx *ctx, void *device_ptr, size_t len, int dtype, fx_buf **out);
int fx_free(fx_buf *buf);
size_t fx_buf_len(const fx_buf *buf);
int fx_buf_dtype(const fx_buf *buf);
void *fx_buf_device_ptr(const fx_buf *buf);
/* Length mismatch is an error here (the reference panics, buffer.rs:100-110). */
int fx_copy_to_host_f64(fx_ctx *ctx, const fx_buf *buf, double *dst, size_t len);
int fx_copy_to_host_f32(fx_ctx *ctx, const fx_buf *buf, float *dst, size_t len);
/* Host -> existing buffer (no reallocation), converting to the buffer's dtype. */
int fx_write_f64(fx_ctx *ctx, fx_buf *buf, const double *src, size_t len);
int fx_write_f32(fx_ctx *ctx, fx_buf *buf, const float *src, size_t len);
/* Asynchronous copies between an F64 buffer and page-locked host memory (new): enqueued on `stream`
 * (a cudaStream_t; NULL = the context's stream), no wait.  The caller orders them against the
 * library's work with events, so that uploads and read-backs of a stream of solves overlap the
 * solves.  From pageable memory the driver copies synchronously. */
int fx_write_f64_async(fx_ctx *ctx, fx_buf *buf, const double *src, size_t len, void *stream);
int fx_copy_to_host_f64_async(fx_ctx *ctx, const fx_buf *buf, double *dst, size_t len, void *stream);

/* ------------------------------------------------------------------ */
/* Backend trait ops (crates/core/src/backend.rs)                      */
/* ------------------------------------------------------------------ */

/* apply_stencil :88-95 -- out = S(in); ring = boundary values. */
int fx_apply_stencil(fx_ctx *ctx, const fx_buf *in, fx_buf *out, const fx_grid *g,
                     const fx_stencil *s, const fx_boundaries *bc);
/* apply_stencil_var :148-156 -- out = coeff .* S(in) (whole array). */
int fx_apply_stencil_var(fx_ctx *ctx, const fx_buf *in, fx_buf *out, const fx_buf *coeff,
                         const fx_grid *g, const fx_stencil *s, const fx_boundaries *bc);
/* stencil_axpy :166-174 -- y[interior] += alpha * S(x); ring untouched. */
int fx_stencil_axpy(fx_ctx *ctx, double alpha, const fx_buf *x, fx_buf *y, const fx_grid *g,
                    const fx_stencil *s, const fx_boundaries *bc);
int fx_copy(fx_ctx *ctx, const fx_buf *src, fx_buf *dst);                      /* :101-105 */
int fx_fill(fx_ctx *ctx, fx_buf *buf, double value);                            /* :111-115 */
int fx_axpy(fx_ctx *ctx, double alpha, const fx_buf *x, fx_buf *y);             /* :121-126 */
int fx_scale(fx_ctx *ctx, fx_buf *buf, double alpha);                           /* :132-136 */
int fx_norm_l2(fx_ctx *ctx, const fx_buf *buf, double *out);                    /* :180 */
int fx_reduce_sum(fx_ctx *ctx, const fx_buf *buf, double *out);                 /* :188 */
int fx_reduce_max(fx_ctx *ctx, const fx_buf *buf, double *out);                 /* :194 */
int fx_reduce_min(fx_ctx *ctx, const fx_buf *buf, double *out);                 /* :200 */
int fx_dot(fx_ctx *ctx, const fx_buf *x, const fx_buf *y, double *out);         /* :206-210 */
/* dot2 :219-230 -- (a.b, c.d) in one pass. */
int fx_dot2(fx_ctx *ctx, const fx_buf *a, const fx_buf *b, const fx_buf *c, const fx_buf *d,
            double *ab, double *cd);
/* No counterpart in the reference.  Dot product of two FP64 device arrays (plain device
 * pointers) that allocates nothing, for callers that cannot let the library allocate device
 * memory (an application owning all device memory through its own pool, a loop that must not
 * reach the allocator).  Its reduction scratch is a fixed static device array (64 KiB per
 * GPU, held until exit), so n is limited to 8,388,608 elements (FX_ERR_INVALID_ARGUMENT
 * above that).  Runs on `stream` (a cudaStream_t; NULL = default stream) and synchronises it.
 * Calls share the scratch: calls that overlap on the GPU race.  The first call on a device
 * resolves the array's device address; make it before any stream capture.  The address is kept
 * for the process's life, so calls after a reset of the device (cudaDeviceReset) are not
 * supported. */
int fx_dot_f64_noalloc(const double *x, const double *y, size_t n, double *out, void *stream);
/* restrict :240-246 (reference semantics: clamped 2x2 average). */
int fx_restrict(fx_ctx *ctx, const fx_buf *fine, fx_buf *coarse, const fx_grid *fine_grid,
                const fx_grid *coarse_grid);
/* prolong :254-260 (reference semantics: fine[i,j] += coarse[i/2,j/2]). */
int fx_prolong(fx_ctx *ctx, const fx_buf *coarse, fx_buf *fine, const fx_grid *coarse_grid,
               const fx_grid *fine_grid);
/* weighted_jacobi :269-277 -- reference CPU semantics: one in-place lexicographic sweep
 * (ops.rs:425-473), bitwise equal to it. */
int fx_weighted_jacobi(fx_ctx *ctx, fx_buf *x, const fx_buf *b, double omega, const fx_grid *g,
                       const fx_stencil *s, const fx_boundaries *bc);
int fx_pointwise_mult(fx_ctx *ctx, const fx_buf *x, const fx_buf *y, fx_buf *z); /* :285-290 */
int fx_pointwise_div(fx_ctx *ctx, const fx_buf *x, const fx_buf *y, fx_buf *z);  /* :296-301 */
int fx_waxpy(fx_ctx *ctx, double alpha, const fx_buf *x, double beta, const fx_buf *y,
             fx_buf *w);                                                          /* :309-316 */
int fx_aypx(fx_ctx *ctx, double alpha, const fx_buf *x, fx_buf *y);              /* :322-327 */
int fx_reciprocal(fx_ctx *ctx, fx_buf *buf);                                     /* :333-336 */
int fx_abs_val(fx_ctx *ctx, fx_buf *buf);                                        /* :342-345 */
int fx_pointwise_max(fx_ctx *ctx, const fx_buf *x, const fx_buf *y, fx_buf *z);  /* :348-353 */
int fx_pointwise_min(fx_ctx *ctx, const fx_buf *x, const fx_buf *y, fx_buf *z);  /* :356-361 */
/* apply_conv_diff :375-384 -- out = kappa .* Lap(u) + v . grad(u) (upwind); ring = 0. */
int fx_apply_conv_diff(fx_ctx *ctx, const fx_buf *u, fx_buf *out, const fx_buf *kappa,
                       const fx_buf *vx, const fx_buf *vy, const fx_grid *g,
                       const fx_boundaries *bc);
/* conv_diff_axpy :395-405 -- out[interior] += alpha * (...); ring untouched. */
int fx_conv_diff_axpy(fx_ctx *ctx, double alpha, const fx_buf *u, fx_buf *out,
                      const fx_buf *kappa, const fx_buf *vx, const fx_buf *vy, const fx_grid *g,
                      const fx_boundaries *bc);

/* ------------------------------------------------------------------ */
/* Non-trait fast paths (HipBackend extras, backend-hip/src/backend.rs:463-668) */
/* ------------------------------------------------------------------ */

/* zero_boundaries (backend.rs:510-531; field.rs:386-431) */
int fx_zero_boundaries(fx_ctx *ctx, fx_buf *buf, size_t rows, size_t cols);
/* pipelined_cg_fused (backend.rs:469-504): z=q+b*z; t=w+b*t; p=r+b*p; x+=a*p; r-=a*t; w-=a*z */
int fx_pcg_fused_update(fx_ctx *ctx, double alpha, double beta, fx_buf *z, fx_buf *t, fx_buf *p,
                        fx_buf *x, fx_buf *r, fx_buf *w, const fx_buf *q);
/* Same update plus (r.r, r.w) of the updated r, w in the same pass. */
int fx_pcg_fused_update_dot2(fx_ctx *ctx, double alpha, double beta, fx_buf *z, fx_buf *t,
                             fx_buf *p, fx_buf *x, fx_buf *r, fx_buf *w, const fx_buf *q,
                             double *rr, double *rw);

/* ------------------------------------------------------------------ */
/* Vertex-centred multigrid primitives (full weighting, bilinear prolongation, true weighted
 * Jacobi).  Grids are (2^k+1) x (2^k+1)-style: fine = 2*(coarse-1)+1 in each direction.
 * a5 = {centre, north, south, west, east} weights of the level operator.
 * ------------------------------------------------------------------ */
int fx_jacobi_sweep(fx_ctx *ctx, const fx_buf *x_in, fx_buf *x_out, const fx_buf *b,
                    double omega, size_t rows, size_t cols, const double a5[5]);
int fx_residual5(fx_ctx *ctx, const fx_buf *x, const fx_buf *b, fx_buf *r, size_t rows,
                 size_t cols, const double a5[5]);
int fx_restrict_fw(fx_ctx *ctx, const fx_buf *fine, fx_buf *coarse, size_t frows, size_t fcols,
                   size_t crows, size_t ccols);
int fx_prolong_bilinear(fx_ctx *ctx, const fx_buf *coarse, fx_buf *fine, size_t crows,
                        size_t ccols, size_t frows, size_t fcols);

/* ------------------------------------------------------------------ */
/* Preconditioners (crates/runtime/src/preconditioner.rs:10-37; multigrid.rs) */
/* ------------------------------------------------------------------ */

/* Identity: z = r (preconditioner.rs:31-37). */
int fx_precond_identity(fx_ctx *ctx, fx_precond **out);
int fx_precond_destroy(fx_precond *pc);
/* Preconditioner::apply(z, r) (preconditioner.rs:19-29).  The solvers zero-fill z first. */
int fx_precond_apply(fx_precond *pc, fx_buf *z, const fx_buf *r);
/* Inner-CG preconditioner (new): z = steps[k mod nsteps] CG steps on (I + coeff S) z = r from
 * z = 0 at the k-th application (preconditioned by `inner` when non-null, which must outlive
 * it), with tolerance 0.  A schedule of different counts makes it vary between applications,
 * the case fx_fcg_* and fx_fgmres_* are for.  F64 vectors; st and bc are copied. */
int fx_precond_inner_cg(fx_ctx *ctx, const fx_grid *g, double coeff, const fx_stencil *st,
                        const fx_boundaries *bc, const size_t *steps, size_t nsteps, fx_precond *inner,
                        fx_precond **out);
/* Inner FP32 PCG preconditioner (new): z = (double) d, d the FP32 CG solution of (I + coeff S) d =
 * (float) r from d = 0, preconditioned by inner_f32 (an FP32 vertex multigrid, borrowed; it must
 * outlive this), stopped at ||r - A d|| < rel_tol ||r|| or max_iter iterations.  It varies between
 * applications: a preconditioner for fx_fcg_* and fx_fgmres_* (FP64 outer Krylov, FP32 inner
 * solves).  F64 vectors of grid g.  stats: applications and inner iterations so far. */
int fx_precond_inner_pcg_f32(fx_ctx *ctx, const fx_grid *g, double coeff, const fx_stencil *st,
                             const fx_boundaries *bc, fx_precond *inner_f32, double rel_tol, size_t max_iter,
                             fx_precond **out);
int fx_precond_inner_pcg_f32_stats(const fx_precond *pc, size_t *applications, size_t *inner_iterations);

/* Multigrid::new / ::build (multigrid.rs:61-146): reference hierarchy (rows/2 per level,
 * Laplacian on each level, clamped 2x2 restriction, piecewise-constant prolongation,
 * lexicographic weighted-Jacobi smoother, coarsest level n_pre+n_post+10 sweeps).
 * smoother: 0 = Jacobi, 1 = Chebyshev (multigrid.rs:308-473: first-kind recurrence for D^-1 A,
 * emax = 2, emin = 0.2, built from the backend ops, two extra vectors per level). */
int fx_mg_create(fx_ctx *ctx, const fx_grid *g, const fx_boundaries *bc, size_t n_pre,
                 size_t n_post, double omega, int smoother, fx_mg **out);

/* Vertex-centred V-cycle for the operator actually solved, A = I + coeff*S with S a 5-point
 * stencil: coarsening (rows-1)/2 per level down to an interior of at most coarse_max, full
 * weighting, bilinear prolongation, n_pre/n_post true weighted-Jacobi sweeps (omega), and
 * coarse_sweeps sweeps on the coarsest level.  dtype FX_F32 runs the cycle in single
 * precision (inputs/outputs stay in their own dtype).  Homogeneous Dirichlet ring. */
typedef struct {
    size_t n_pre, n_post;
    double omega;
    size_t coarse_max;
    size_t coarse_sweeps;
    int dtype;
    double op_coeff;
    fx_stencil op_stencil;
} fx_mg_vertex_opts;
int fx_mg_create_vertex(fx_ctx *ctx, const fx_grid *g, const fx_boundaries *bc,
                        const fx_mg_vertex_opts *opts, fx_mg **out);
int fx_mg_destroy(fx_mg *mg);
/* Layout of the fused vertex cycle (new; no reference counterpart): the strip kernels' row
 * chunks per launch in percent of one wave of resident warps (default 100), and the largest
 * level, in points, that the one-block tail takes (0 = as large as it can hold: 9216 points).
 * Neither changes any value the cycle computes. */
typedef struct {
    int chunk_pct;
    size_t tail_top_points;
} fx_mg_tuning;
int fx_mg_set_tuning(fx_mg *mg, const fx_mg_tuning *t);
int fx_mg_get_tuning(const fx_mg *mg, fx_mg_tuning *t);
/* Autotuner (new): times `reps` cycles z = M^-1 r (after two untimed ones) for each candidate
 * layout -- chunk_pct in {50, 100, 200} x tail_top_points in {9216, 2048}, in that order --
 * on the caller's vectors (F64, the fused vertex V(2,2)-cycle of either precision), keeps the
 * fastest in the multigrid and returns it, its time per cycle, and up to cand_cap candidate
 * times (ncand of them).  FX_ERR_UNSUPPORTED for other cycles.  z is overwritten. */
int fx_mg_autotune(fx_mg *mg, fx_buf *z, const fx_buf *r, int reps, fx_mg_tuning *best, double *best_ms,
                   double *cand_ms, size_t cand_cap, size_t *ncand);
/* Multigrid::depth (multigrid.rs:174-178) */
int fx_mg_depth(const fx_mg *mg, size_t *depth);
int fx_mg_level_dims(const fx_mg *mg, size_t level, size_t *rows, size_t *cols);
/* Multigrid::v_cycle (multigrid.rs:188-230): x (initial guess, in/out), b (rhs). */
int fx_mg_v_cycle(fx_mg *mg, fx_buf *x, const fx_buf *b);
/* Preconditioner application from a zero initial guess: z = M^-1 r, i.e. the reference's
 * z.fill(0); pc.apply(z, r) (cg.rs:196-197).  Uses the fused V(2,2) kernels when they apply. */
int fx_mg_precondition(fx_mg *mg, fx_buf *z, const fx_buf *r);
/* Borrowed view of the multigrid as a preconditioner (impl Preconditioner, :600-608).
 * Valid until fx_mg_destroy; do not pass it to fx_precond_destroy. */
fx_precond *fx_mg_as_precond(fx_mg *mg);

/* ------------------------------------------------------------------ */
/* Krylov solvers.  Operator A v = v + coeff * S v (linear_solver.rs:7-22).  `tol` is the
 * absolute tolerance on ||r||_2 (cg.rs:61-64).  Solver parameters are fixed at creation, as
 * the reference's `tol` / `max_iter` fields are; fx_*_set_params changes them.
 * ------------------------------------------------------------------ */

/* CgSolver (cg.rs:52-256) */
int fx_cg_create(fx_ctx *ctx, const fx_grid *g, double tol, size_t max_iter, fx_cg **out);
int fx_cg_destroy(fx_cg *s);
int fx_cg_set_params(fx_cg *s, double tol, size_t max_iter);
int fx_cg_solve(fx_cg *s, fx_buf *x, const fx_buf *b, double coeff, const fx_stencil *st,
                const fx_boundaries *bc, fx_stats *out);
int fx_cg_solve_preconditioned(fx_cg *s, fx_buf *x, const fx_buf *b, double coeff,
                               const fx_stencil *st, const fx_boundaries *bc, fx_precond *pc,
                               fx_stats *out);

/* PipelinedCgSolver (pipelined_cg.rs:25-237) */
int fx_pipelined_cg_create(fx_ctx *ctx, const fx_grid *g, double tol, size_t max_iter,
                           fx_pipelined_cg **out);
int fx_pipelined_cg_destroy(fx_pipelined_cg *s);
int fx_pipelined_cg_set_params(fx_pipelined_cg *s, double tol, size_t max_iter);
int fx_pipelined_cg_solve(fx_pipelined_cg *s, fx_buf *x, const fx_buf *b, double coeff,
                          const fx_stencil *st, const fx_boundaries *bc, fx_stats *out);
/* Preconditioned pipelined CG (Ghysels & Vanroose 2014, Algorithm 4), new: the reference's
 * PipelinedCgSolver is its unpreconditioned case (same scalar recurrence, same update forms).
 * Per iteration one preconditioner application m = M w and one fused pass (n = A m on the fly,
 * the 8-way vector update, (r.u, w.u, r.r) reduced); stops on ||r||_2 < tol as CgSolver does. */
int fx_pipelined_cg_solve_preconditioned(fx_pipelined_cg *s, fx_buf *x, const fx_buf *b, double coeff,
                                         const fx_stencil *st, const fx_boundaries *bc, fx_precond *pc,
                                         fx_stats *out);

/* Mixed-precision iterative refinement (new: the reference has no refinement loop).  FP64
 * refinement x += d around FP32 preconditioned CG: each outer step computes r = b - A x and its
 * norm in FP64 (one pass that also writes r in FP32), stops when ||r||_2 < tol (absolute, as the
 * solvers' tol) or after max_outer corrections, and otherwise solves A d = r on FP32 vectors
 * with `pc` (which must accept FP32 vectors, e.g. an FX_F32 vertex multigrid) until
 * ||r_inner||_2 < inner_tol * ||r||_2 or inner_max_iter iterations.  The inner products and CG
 * scalars stay compensated FP64.  x and b are F64.  out->iterations counts the corrections;
 * *inner_iterations (may be NULL) the inner CG iterations over all of them. */
int fx_ir_create(fx_ctx *ctx, const fx_grid *g, double tol, size_t max_outer, double inner_tol,
                 size_t inner_max_iter, fx_ir **out);
int fx_ir_destroy(fx_ir *s);
int fx_ir_solve_preconditioned(fx_ir *s, fx_buf *x, const fx_buf *b, double coeff, const fx_stencil *st,
                               const fx_boundaries *bc, fx_precond *pc, fx_stats *out,
                               size_t *inner_iterations);

/* BiCgStabSolver (bicgstab.rs:19-346) */
int fx_bicgstab_create(fx_ctx *ctx, const fx_grid *g, double tol, size_t max_iter,
                       fx_bicgstab **out);
int fx_bicgstab_destroy(fx_bicgstab *s);
int fx_bicgstab_set_params(fx_bicgstab *s, double tol, size_t max_iter);
int fx_bicgstab_solve(fx_bicgstab *s, fx_buf *x, const fx_buf *b, double coeff,
                      const fx_stencil *st, const fx_boundaries *bc, fx_stats *out);
int fx_bicgstab_solve_preconditioned(fx_bicgstab *s, fx_buf *x, const fx_buf *b, double coeff,
                                     const fx_stencil *st, const fx_boundaries *bc,
                                     fx_precond *pc, fx_stats *out);

/* GmresSolver (gmres.rs:24-491) */
int fx_gmres_create(fx_ctx *ctx, const fx_grid *g, size_t restart, double tol, size_t max_iter,
                    fx_gmres **out);
int fx_gmres_destroy(fx_gmres *s);
int fx_gmres_set_params(fx_gmres *s, double tol, size_t max_iter);
int fx_gmres_solve(fx_gmres *s, fx_buf *x, const fx_buf *b, double coeff, const fx_stencil *st,
                   const fx_boundaries *bc, fx_stats *out);
int fx_gmres_solve_preconditioned(fx_gmres *s, fx_buf *x, const fx_buf *b, double coeff,
                                  const fx_stencil *st, const fx_boundaries *bc, fx_precond *pc,
                                  fx_stats *out);

/* Flexible CG (new; the reference has no flexible solver): PCG with the Polak-Ribiere beta
 * z_{k+1}.(r_{k+1} - r_k) / (z_k.r_k) (Golub & Ye 1999; Notay's FCG(1), 2000), for
 * preconditioners that change between applications.  Same stop and breakdown tests as
 * fx_cg_solve_preconditioned; fx_fcg_solve uses the identity (and is then CG). */
int fx_fcg_create(fx_ctx *ctx, const fx_grid *g, double tol, size_t max_iter, fx_fcg **out);
int fx_fcg_destroy(fx_fcg *s);
int fx_fcg_set_params(fx_fcg *s, double tol, size_t max_iter);
int fx_fcg_solve(fx_fcg *s, fx_buf *x, const fx_buf *b, double coeff, const fx_stencil *st,
                 const fx_boundaries *bc, fx_stats *out);
int fx_fcg_solve_preconditioned(fx_fcg *s, fx_buf *x, const fx_buf *b, double coeff, const fx_stencil *st,
                                const fx_boundaries *bc, fx_precond *pc, fx_stats *out);

/* Flexible GMRES(m) (new; Saad 1993): right preconditioning with the m preconditioned
 * directions kept, so the preconditioner may change between applications; the residual it
 * stops on is the true ||b - A x||.  Gram-Schmidt, Givens rotations and restarts as
 * fx_gmres_*; without a preconditioner it is GMRES step for step. */
int fx_fgmres_create(fx_ctx *ctx, const fx_grid *g, size_t restart, double tol, size_t max_iter,
                     fx_fgmres **out);
int fx_fgmres_destroy(fx_fgmres *s);
/* Orthogonalisation of the Arnoldi step: 0 = modified Gram-Schmidt (default; the reference's,
 * gmres.rs:185-189), 1 = classical Gram-Schmidt twice (CGS2: three passes over the basis per step
 * instead of one per basis vector; restart <= 32).  New. */
int fx_fgmres_set_orthogonalization(fx_fgmres *s, int method);
int fx_fgmres_set_params(fx_fgmres *s, double tol, size_t max_iter);
int fx_fgmres_solve(fx_fgmres *s, fx_buf *x, const fx_buf *b, double coeff, const fx_stencil *st,
                    const fx_boundaries *bc, fx_stats *out);
int fx_fgmres_solve_preconditioned(fx_fgmres *s, fx_buf *x, const fx_buf *b, double coeff,
                                   const fx_stencil *st, const fx_boundaries *bc, fx_precond *pc,
                                   fx_stats *out);

/* Convection-diffusion operator for the non-symmetric solvers (new; the reference applies
 * apply_conv_diff / conv_diff_axpy (backend.rs:375-405) but solves only v + coeff S v):
 * A v = sigma v + coeff (kappa Lap v + vx dv/dx + vy dv/dy) on the interior, first-order
 * upwind on the sign of v as apply_conv_diff, A v = v on the ring.  sigma = 1 is the
 * implicit-step operator (conv_diff_axpy(coeff, v, v)); sigma = 0 the steady operator.
 * kappa: an F64 field, or NULL for the scalar kappa_s; vx, vy: F64 fields.  The fields are
 * borrowed and must outlive the operator. */
int fx_op_conv_diff(fx_ctx *ctx, const fx_grid *g, double sigma, double coeff, const fx_buf *kappa,
                    double kappa_s, const fx_buf *vx, const fx_buf *vy, fx_op **out);
int fx_op_destroy(fx_op *op);
/* out = A v (v and out distinct F64 fields of the operator's grid) */
int fx_op_apply(const fx_op *op, const fx_buf *v, fx_buf *out);
/* Jacobi preconditioner of the operator: z = r / diag(A); valid while op lives */
int fx_precond_jacobi_op(const fx_op *op, fx_precond **out);
/* Multigrid V-cycle preconditioner for the operator (new): vertex hierarchy as
 * fx_mg_create_vertex (rows - 1 halves while both interiors exceed coarse_max), each coarse
 * level the operator rediscretised with h doubled and kappa / vx / vy injected from the
 * coincident fine points; weighted Jacobi (omega) with the operator's diagonal
 * (x += omega (b - A x) (1 / diag)), full weighting
 * and bilinear transfers, `coarse_sweeps` sweeps on the coarsest level; one cycle from z = 0
 * per application.  The operator (and its fields) must outlive it; fx_cdmg_as_precond gives
 * a borrowed handle valid until fx_cdmg_destroy. */
int fx_cdmg_create(const fx_op *op, size_t n_pre, size_t n_post, double omega, size_t coarse_max,
                   size_t coarse_sweeps, fx_cdmg **out);
/* The same cycle computed and stored in `dtype` (FX_F64: fx_cdmg_create; FX_F32: every level,
 * including F32 copies of the operator's fields on level 0, in single precision).  The vectors
 * z and r of an application stay F64: r is rounded to F32 on entry, z is the F64 image of the
 * F32 cycle.  An FP32 preconditioner inside an FP64 Krylov solver. */
int fx_cdmg_create_typed(const fx_op *op, size_t n_pre, size_t n_post, double omega, size_t coarse_max,
                         size_t coarse_sweeps, int dtype, fx_cdmg **out);
/* Replay (new; off by default): the first application to a given (z, r) pair on a stream is
 * recorded into a CUDA graph, later ones launch that graph.  The results are the same.  It
 * pays for a hierarchy applied many times; recording costs more host time than a short-lived
 * hierarchy saves.  Applications inside a caller's own capture are never recorded. */
int fx_cdmg_set_replay(fx_cdmg *mg, int enabled);
int fx_cdmg_destroy(fx_cdmg *mg);
int fx_cdmg_depth(const fx_cdmg *mg, size_t *depth);
fx_precond *fx_cdmg_as_precond(fx_cdmg *mg);
/* ------------------------------------------------------------------ */
/* Learned smoother (new; the reference smooths with weighted Jacobi only, multigrid.rs:245-306).
 * A 3 -> 16 -> 16 -> 1 network of 3 x 3 convolutions (ReLU after the first two; BF16 weights and
 * activations, FP32 accumulation and biases; 2913 parameters) corrects the weighted-Jacobi step
 * of the conv-diff multigrid: with q = (b - A x) / diag(A) (0 on the ring) and s the RMS of q
 * over the interior, one learned step is x <- x + omega q + s N(q / s, vx / (dx diag), vy / (dy diag))
 * on the interior, evaluated on the tensor cores.  With the last layer zero (as created) the
 * step is the Jacobi sweep.  The network is trained on the GPU by the library's own forward,
 * backward and Adam kernels on samples cut from plain V-cycle iterates: the loss of a sample is
 * ||H e'||^2 / ||H e||^2, e' the error after the step and H = I - P R the part of an error that
 * the coarse grid cannot represent (full weighting R, bilinear P), plus lambda ||e'||^2 / ||e||^2
 * (both parts normalised by the Jacobi-free denominator ||H e||^2 + lambda ||e||^2).
 * ------------------------------------------------------------------ */
int fx_lsm_param_count(size_t *n);  /* 2913 */
/* Parameters W1[16][3][9], b1[16], W2[16][16][9], b2[16], W3[16][9], b3: He-normal W1, W2 from
 * `seed`, zero biases, zero last layer. */
int fx_lsm_create(fx_ctx *ctx, unsigned long long seed, fx_lsm **out);
int fx_lsm_destroy(fx_lsm *m);
/* FP32 master parameters in the order above (set also resets the optimiser state). */
int fx_lsm_get_params(fx_lsm *m, float *dst, size_t n);
int fx_lsm_set_params(fx_lsm *m, const float *src, size_t n);
/* `steps` learned smoothing steps on op's grid: x (in/out) and b are F64 fields of the grid;
 * the operator's fields must be F64.  Synchronises. */
int fx_lsm_smooth(fx_lsm *m, const fx_op *op, fx_buf *x, const fx_buf *b, double omega, size_t steps);
/* Training samples on the device, up to `capacity` of them.  A sample is a 16 x 16 loss patch
 * whose first point (row, col) is even: the network inputs over the 25 x 25 region from
 * (row - 4, col - 4) (BF16, channel-major); over the patch the targets tH = (H e - omega H q) / s
 * and tE = (e - omega q) / s; and nH = ||H e||^2 / s^2, nE = ||e||^2 / s^2 (FP32). */
int fx_lsm_data_create(fx_ctx *ctx, size_t capacity, fx_lsm_data **out);
int fx_lsm_data_destroy(fx_lsm_data *d);
int fx_lsm_data_size(const fx_lsm_data *d, size_t *n);
/* Samples from an iterate x with error e for A u = b: one per (row, col) pair in origins[2 count]
 * (even, with 4 <= row <= rows - 21 and 4 <= col <= cols - 21); s is the RMS of q over the grid. */
int fx_lsm_data_add_patches(fx_lsm_data *d, const fx_op *op, const fx_buf *x, const fx_buf *e, const fx_buf *b,
                            double omega, const int *origins, size_t count);
/* Samples from the plain V-cycle on A u = b: u is solved to 1e-12 (FGMRES(30) with the conv-diff
 * V(2,2)-cycle), then from x = 0 `iterates` iterates x <- x + M (b - A x) each give
 * patches_per_iterate samples at seeded random origins.  *added = samples stored. */
int fx_lsm_data_add_problem(fx_lsm_data *d, const fx_op *op, const fx_buf *b, size_t iterates,
                            size_t patches_per_iterate, double omega, unsigned long long seed, size_t *added);
/* Sample `index` back on the host: inputs[3 * 25 * 25] (the BF16 values, exactly), target[512]
 * (tH then tE), norm[2] (nH, nE). */
int fx_lsm_data_get(const fx_lsm_data *d, size_t index, float *inputs, float *target, float *norm);
/* Mean loss (weight lambda >= 0 on the whole error) of the samples indices[0..count) and, when
 * grad is not NULL, its gradient grad[2913] with respect to the parameters (bitwise reproducible). */
int fx_lsm_loss_grad(fx_lsm *m, const fx_lsm_data *d, const size_t *indices, size_t count, double lambda,
                     double *loss, float *grad);
/* Adam (lr; beta 0.9 / 0.999, eps 1e-8) on the loss with weight lambda, over `epochs` seeded
 * shuffles of the samples in batches of `batch`; epoch_loss[e] (may be NULL) = mean sample loss of
 * epoch e, each batch's loss taken before its step. */
int fx_lsm_train(fx_lsm *m, const fx_lsm_data *d, size_t epochs, size_t batch, double lr, double lambda,
                 unsigned long long seed, double *epoch_loss);
/* Learned smoothing in a conv-diff multigrid: every level of min_points to max_points points (0: no
 * upper bound) except the coarsest smooths with learned steps in place of the Jacobi sweeps (n_pre and
 * n_post of them).
 * Each application is checked on the device: when ||r - A z|| > fallback_ratio ||r|| the plain
 * cycle recomputes z (the flexible solvers accept either).  lsm NULL switches it off; lsm must
 * outlive the multigrid's use of it.  stats: checked applications and fallbacks so far. */
int fx_cdmg_set_learned(fx_cdmg *mg, const fx_lsm *lsm, size_t min_points, size_t max_points, double fallback_ratio);
int fx_cdmg_learned_stats(fx_cdmg *mg, unsigned long long *applications, unsigned long long *fallbacks);
/* Patience of the learned cycle (new): after `patience` fallbacks in a row the learned cycle is
 * switched off, on the device, and the plain cycle alone runs from then on (no check); 0 (the
 * default) never switches it off.  This call and fx_cdmg_set_learned switch it back on.
 * fx_cdmg_learned_disabled reports whether it is off. */
int fx_cdmg_set_learned_patience(fx_cdmg *mg, size_t patience);
int fx_cdmg_learned_disabled(fx_cdmg *mg, int *disabled);

/* ------------------------------------------------------------------ */
/* Batched solve (new; the reference solves one grid at a time, bicgstab.rs:218-346).  `count`
 * independent steady problems sigma u + coeff (kappa Lap u + v.grad u) = f, kappa = -nu, each on
 * its own square grid of side grid_side[p] = 2^k + 1 (ring included) over the unit square, with
 * Dirichlet 0.  Vectors of the batch are F64 buffers holding every problem's grid one after the
 * other (fx_batch_layout gives the offsets); vx and vy are such buffers, borrowed for the
 * batch's life.  Each problem is solved by right-preconditioned BiCGSTAB with the conv-diff
 * V-cycle of fx_cdmg_create_typed (cycle_dtype FX_F64 or FX_F32), every problem in the same
 * launches: each phase of the algorithm is one launch over the whole batch, its blocks taking
 * (problem, chunk) or (problem, tile) items from tables built here, so a launch fills the GPU
 * with every problem's share.  The cycle equals fx_cdmg's bit for bit. */
int fx_batch_create(fx_ctx *ctx, size_t count, const size_t *grid_side, double nu, double sigma, double coeff,
                    const fx_buf *vx, const fx_buf *vy, int cycle_dtype, size_t n_pre, size_t n_post, double omega,
                    size_t coarse_max, size_t coarse_sweeps, fx_batch **out);
int fx_batch_destroy(fx_batch *b);
/* offsets[count + 1]: where each problem's grid starts in a batch vector (and the total);
 * levels[count] (may be NULL): each problem's multigrid depth */
int fx_batch_layout(const fx_batch *b, size_t *offsets, size_t *levels);
/* Elements per flat work item of the batch's launches (a multiple of 256 in [256, 65536];
 * 2048 at creation).  Changes no computed value; the autotuner picks it. */
int fx_batch_set_chunk(fx_batch *b, size_t elements);
/* out = A v for every problem (synchronises) */
int fx_batch_apply(fx_batch *b, const fx_buf *v, fx_buf *out);
/* norms[count] = ||b_p - A x_p|| of every problem, computed on the device (synchronises) */
int fx_batch_residual_norms(fx_batch *b, const fx_buf *x, const fx_buf *rhs, double *norms);
/* z = M r (one V-cycle from zero) for every problem (synchronises) */
int fx_batch_precondition(fx_batch *b, fx_buf *z, const fx_buf *r);
/* BiCGSTAB (bicgstab.rs:218-346, right-preconditioned by the batch's cycle) of every problem from
 * its initial x, each to ||r_p|| < rel_tol ||b_p|| or max_iter iterations; stats[count] get each
 * problem's iterations, residual and reason.  use_graph: each iteration of the whole batch is
 * recorded once (per (x, b) pair) into a CUDA graph and replayed.  *iterations_run (may be
 * NULL): batch iterations launched. */
int fx_batch_bicgstab(fx_batch *b, fx_buf *x, const fx_buf *rhs, double rel_tol, size_t max_iter, int use_graph,
                      fx_stats *stats, size_t *iterations_run);

/* BiCGSTAB, GMRES(m) and flexible GMRES(m) on the operator (pc may be NULL): the same loops,
 * recurrences and stop tests as fx_bicgstab_solve*, fx_gmres_solve* and fx_fgmres_solve* */
int fx_bicgstab_solve_op(fx_bicgstab *s, fx_buf *x, const fx_buf *b, const fx_op *op, fx_precond *pc,
                         fx_stats *out);
int fx_gmres_solve_op(fx_gmres *s, fx_buf *x, const fx_buf *b, const fx_op *op, fx_precond *pc,
                      fx_stats *out);
int fx_fgmres_solve_op(fx_fgmres *s, fx_buf *x, const fx_buf *b, const fx_op *op, fx_precond *pc,
                       fx_stats *out);

/* ------------------------------------------------------------------ */
/* Checked build (new; the reference has no sanitizer mode).  libfluxion_cuda_checked.so is the
 * same library compiled with FX_CHECKED: its kernels test every index they compute against the
 * extent of the array addressed, skip an access outside it (a load gives zero, a store is
 * dropped) and record the first such event of each source unit in a device status word.  It
 * never traps.  fx_checked_build returns 1 in that library and 0 in the default one, whose checks
 * are compiled away. */
int fx_checked_build(void);
/* Synchronises the context's device, then reads and clears the status words: *count = the number
 * of units that recorded an out-of-range index since the last call, and for the first of them the
 * source file of the check (file, NUL-terminated, at most file_cap bytes; may be NULL), its line,
 * the index and the extent.  The default build reports count 0. */
int fx_checked_status(fx_ctx *ctx, size_t *count, char *file, size_t file_cap, int *line, long long *index,
                      long long *extent);
/* Test hook: a kernel that tests `index` against `extent` with the checked build's check and
 * makes no memory access, so an out-of-range pair is recorded (checked build) or nothing happens
 * (default build). */
int fx_test_check_index(fx_ctx *ctx, long long index, long long extent);

#ifdef __cplusplus
}
#endif
#endif /* FLUXION_CUDA_H */
