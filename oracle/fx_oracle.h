/*
 * fx_oracle.h -- CPU oracle for the fluxion matrix-free solve path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the
 * reference CPU backend (crates/backend-cpu/src/ops.rs) and of the
 * runtime solver loops (crates/runtime/src/{cg,pipelined_cg,bicgstab,
 * gmres,multigrid}.rs) of DenisChpt/fluxion.  It exists so that the
 * CUDA library can be checked against it; only tests/, the smoke check
 * and bench.py's CPU-baseline leg may load it.  The product path never
 * calls into this code.
 *
 * Parity pin: the restatement is checked against every known-answer test
 * the reference ships for this path (ops.rs:1191-1338 and
 * crates/runtime/tests/solvers.rs, analytical.rs, properties.rs); see
 * tests/test_oracle_golden.py.  The reference itself is Rust and cannot
 * be compiled in this environment (no cargo/rustc).
 *
 * All arrays are row-major, rows x cols, boundary ring included
 * (crates/core/src/grid.rs:4-9, :59-61).
 */
#ifndef FX_ORACLE_H
#define FX_ORACLE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Boundary kinds (crates/core/src/boundary.rs:2-15). */
enum { FXO_BC_DIRICHLET = 0, FXO_BC_NEUMANN = 1, FXO_BC_ROBIN = 2, FXO_BC_PERIODIC = 3 };

typedef struct {
    int kind;
    double a; /* Dirichlet value / Neumann flux / Robin alpha */
    double b; /* Robin beta */
    double g; /* Robin g */
} fxo_bc;

/* Status codes, same meaning as the CUDA library's. */
enum {
    FXO_OK = 0,
    FXO_ERR_DIMENSION_MISMATCH = 1,
    FXO_ERR_INVALID_GRID = 2,
    FXO_ERR_INVALID_STENCIL = 3,
    FXO_ERR_BACKEND = 4,
    FXO_ERR_INVALID_ARGUMENT = 5,
    FXO_ERR_UNSUPPORTED = 6
};

void fxo_set_threads(int n);
int fxo_get_threads(void);

/* ---- BLAS-1 (ops.rs:156-223, :474-655) ---- */
void fxo_fill(double *x, size_t n, double v);
void fxo_copy(const double *src, double *dst, size_t n);
void fxo_axpy(double alpha, const double *x, double *y, size_t n);
void fxo_scale(double *x, size_t n, double alpha);
void fxo_waxpy(double alpha, const double *x, double beta, const double *y, double *w, size_t n);
void fxo_aypx(double alpha, const double *x, double *y, size_t n);
void fxo_pointwise_mult(const double *x, const double *y, double *z, size_t n);
void fxo_pointwise_div(const double *x, const double *y, double *z, size_t n);
void fxo_pointwise_max(const double *x, const double *y, double *z, size_t n);
void fxo_pointwise_min(const double *x, const double *y, double *z, size_t n);
void fxo_reciprocal(double *x, size_t n);
void fxo_abs_val(double *x, size_t n);

/* ---- reductions (ops.rs:271-367, :657-671, kahan_merge :1129-1137) ---- */
double fxo_norm_l2(const double *x, size_t n);
double fxo_reduce_sum(const double *x, size_t n);
double fxo_reduce_max(const double *x, size_t n);
double fxo_reduce_min(const double *x, size_t n);
double fxo_dot(const double *x, const double *y, size_t n);
void fxo_dot2(const double *a, const double *b, const double *c, const double *d, size_t n,
              double *ab, double *cd);

/* ---- stencil (ops.rs:76-127, :225-269, :794-1125) ---- */
int fxo_apply_stencil(const double *in, double *out, size_t rows, size_t cols, double dx, double dy,
                      int ne, const int *dr, const int *dc, const double *w, const fxo_bc *bcs);
int fxo_apply_stencil_var(const double *in, double *out, const double *coeff, size_t rows,
                          size_t cols, double dx, double dy, int ne, const int *dr, const int *dc,
                          const double *w, const fxo_bc *bcs);
int fxo_stencil_axpy(double alpha, const double *x, double *y, size_t rows, size_t cols, int ne,
                     const int *dr, const int *dc, const double *w, const fxo_bc *bcs);
void fxo_zero_boundaries(double *x, size_t rows, size_t cols);

/* ---- convection-diffusion (ops.rs:673-791) ---- */
void fxo_apply_conv_diff(const double *u, double *out, const double *kappa, const double *vx,
                         const double *vy, size_t rows, size_t cols, double dx, double dy);
void fxo_conv_diff_axpy(double alpha, const double *u, double *out, const double *kappa,
                        const double *vx, const double *vy, size_t rows, size_t cols, double dx,
                        double dy);

/* ---- multigrid transfer / smoother, reference semantics (ops.rs:369-473) ---- */
int fxo_restrict(const double *fine, double *coarse, size_t frows, size_t fcols, size_t crows,
                 size_t ccols);
int fxo_prolong(const double *coarse, double *fine, size_t crows, size_t ccols, size_t frows,
                size_t fcols);
int fxo_weighted_jacobi(double *x, const double *b, double omega, size_t rows, size_t cols, int ne,
                        const int *dr, const int *dc, const double *w);

/* ---- pipelined-CG 6-way update (backend-hip elementwise pipelined_cg_fused; CPU fallback
 *      pipelined_cg.rs:440-456) ---- */
void fxo_pcg_fused_update(double alpha, double beta, double *z, double *t, double *p, double *x,
                          double *r, double *w, const double *q, size_t n);

/* ---- vertex-centred geometric multigrid primitives (full weighting, bilinear, true
 *      weighted Jacobi).  The reference's own transfer operators are the 2x2 average and
 *      piecewise-constant ones above; these are the ones the solve configurations ask for. ---- */
void fxo_jacobi_sweep(const double *x_in, double *x_out, const double *b, double omega,
                      size_t rows, size_t cols, const double *a5 /* c,n,s,w,e */);
void fxo_residual(const double *x, const double *b, double *r, size_t rows, size_t cols,
                  const double *a5);
int fxo_restrict_fw(const double *fine, double *coarse, size_t frows, size_t fcols, size_t crows,
                    size_t ccols);
int fxo_prolong_bilinear(const double *coarse, double *fine, size_t crows, size_t ccols,
                         size_t frows, size_t fcols);

/* ---- solvers ---- */
typedef struct {
    size_t iterations;
    double residual;
    int reason; /* 0 converged, 1 max iterations, 2 breakdown (cg.rs:9-18) */
} fxo_stats;

/* Preconditioner callback: z <- M^-1 r, z zero-filled on entry. */
typedef void (*fxo_pc_fn)(void *ctx, double *z, const double *r);

typedef struct {
    size_t rows, cols;
    double coeff;
    int ne;
    const int *dr, *dc;
    const double *w;
    const fxo_bc *bcs;
    /* cd != 0: the convection-diffusion operator instead of the stencil (new; no reference
     * solver takes it): A v = sigma v + coeff (kappa Lap v + vx dv/dx + vy dv/dy) on the
     * interior, first-order upwind as apply_conv_diff (ops.rs:673-791), A v = v on the ring;
     * kappa from the field when non-null, else kappa_s */
    int cd;
    double sigma, kappa_s, dx, dy;
    const double *kappa, *vx, *vy;
} fxo_op;
/* out = A v for either operator kind (out != v) */
int fxo_op_apply(const fxo_op *op, double *out, const double *v);
/* pointwise Jacobi for the conv-diff operator, usable as fxo_pc_fn with ctx = the fxo_op:
 * z = r / diag(A), diag = sigma + coeff (-kappa 2 (1/dx^2 + 1/dy^2) + |vx|/dx + |vy|/dy) inside,
 * 1 on the ring */
void fxo_cd_jacobi_apply(void *op, double *z, const double *r);
/* Multigrid for the conv-diff operator: vertex hierarchy, rediscretised coarse operators with
 * injected fields, weighted Jacobi with the operator's diagonal, full weighting / bilinear,
 * `coarse_sweeps` sweeps on the coarsest level; fxo_cdmg_pc_apply runs one cycle from z = 0. */
typedef struct fxo_cdmg fxo_cdmg;
fxo_cdmg *fxo_cdmg_create(const fxo_op *op, int n_pre, int n_post, double omega, int coarse_max,
                          int coarse_sweeps);
void fxo_cdmg_destroy(fxo_cdmg *mg);
int fxo_cdmg_depth(const fxo_cdmg *mg);
void fxo_cdmg_pc_apply(void *mg, double *z, const double *r);

int fxo_cg_solve(const fxo_op *op, double *x, const double *b, double tol, size_t max_iter,
                 fxo_pc_fn pc, void *pc_ctx, fxo_stats *st);
int fxo_pipelined_cg_solve(const fxo_op *op, double *x, const double *b, double tol,
                           size_t max_iter, fxo_stats *st);
int fxo_pipelined_pcg_solve(const fxo_op *op, double *x, const double *b, double tol, size_t max_iter,
                            fxo_pc_fn pc, void *pc_ctx, fxo_stats *st);
int fxo_bicgstab_solve(const fxo_op *op, double *x, const double *b, double tol, size_t max_iter,
                       fxo_pc_fn pc, void *pc_ctx, fxo_stats *st);
int fxo_gmres_solve(const fxo_op *op, double *x, const double *b, size_t restart, double tol,
                    size_t max_iter, fxo_pc_fn pc, void *pc_ctx, fxo_stats *st);
/* flexible solvers (new): flexible CG (Polak-Ribiere beta) and flexible GMRES(m) (Saad 1993) */
int fxo_fcg_solve(const fxo_op *op, double *x, const double *b, double tol, size_t max_iter,
                  fxo_pc_fn pc, void *pc_ctx, fxo_stats *st);
int fxo_fgmres_solve(const fxo_op *op, double *x, const double *b, size_t restart, double tol,
                     size_t max_iter, fxo_pc_fn pc, void *pc_ctx, fxo_stats *st);
/* nonlinear preconditioner: steps[calls mod nsteps] CG steps (preconditioned by pc when set)
 * from z = 0; calls counts the applications */
typedef struct {
    const fxo_op *op;
    const size_t *steps;
    size_t nsteps, calls;
    fxo_pc_fn pc;
    void *pc_ctx;
} fxo_inner_cg;
void fxo_inner_cg_pc_apply(void *ctx, double *z, const double *r);

/* Multigrid (multigrid.rs).  mode 0 = reference hierarchy and operators
 * (rows/2 coarsening, 2x2 average, piecewise-constant prolongation, lexicographic
 * weighted "Jacobi", Laplacian on every level, coarsest n_pre+n_post+10 sweeps).
 * mode 1 = vertex-centred hierarchy (rows-1 halves), full weighting, bilinear,
 * true weighted Jacobi on the operator being solved, coarsest `coarse_sweeps`. */
typedef struct fxo_mg fxo_mg;
fxo_mg *fxo_mg_create(size_t rows, size_t cols, double dx, double dy, const fxo_bc *bcs,
                      int n_pre, int n_post, double omega, int mode, double op_coeff, int ne,
                      const int *dr, const int *dc, const double *w, int coarse_max,
                      int coarse_sweeps);
void fxo_mg_destroy(fxo_mg *mg);
/* reference mode only: 0 weighted Jacobi (default), 1 Chebyshev (multigrid.rs:308-473) */
int fxo_mg_set_smoother(fxo_mg *mg, int smoother);
int fxo_mg_depth(const fxo_mg *mg);
void fxo_mg_level_dims(const fxo_mg *mg, int lvl, size_t *rows, size_t *cols);
void fxo_mg_v_cycle(fxo_mg *mg, double *x, const double *b);
/* usable as fxo_pc_fn with ctx = the fxo_mg */
void fxo_mg_pc_apply(void *mg, double *z, const double *r);
/* FP32 vertex cycle (the CUDA library's dtype-F32 multigrid on FP64 vectors): z = (double) of
 * the float cycle of (float) r from zero.  FXO_ERR_INVALID_ARGUMENT for a reference-mode mg. */
int fxo_mg_v_cycle_f32(fxo_mg *mg, double *z, const double *r);
void fxo_mg_pc_apply_f32(void *mg, double *z, const double *r);
/* coarse-level operator weights of the vertex hierarchy */
void fxo_mg_coarse_op(const double *fine, double sigma, double *coarse);

#ifdef __cplusplus
}
#endif
#endif
