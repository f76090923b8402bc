/*
 * fx_oracle.c -- CPU oracle for the fluxion matrix-free solve path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker, never the product).  A plain-C
 * restatement of DenisChpt/fluxion's CPU backend and runtime solver loops;
 * every function cites the reference file:line it follows.  Build with
 * -ffp-contract=off so that the only fused multiply-adds are the explicit
 * fma() calls, exactly where the reference writes f64::mul_add.
 *
 * Threading: rayon's par_chunks loops become OpenMP row/chunk loops.  Every
 * parallel loop writes disjoint outputs, and every reduction first computes
 * its per-4096-chunk Kahan partials in parallel and then merges them in
 * chunk order with kahan_merge, so results do not depend on the thread
 * count.  (rayon merges the chunk partials in a work-stealing tree whose
 * shape is not fixed; the left fold used here is one of its valid orders.)
 */
#include "fx_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define KCHUNK 4096

void fxo_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

int fxo_get_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ------------------------------------------------------------------ */
/* BLAS-1: ops.rs:156-223 (copy/fill/axpy/scale), :474-655            */
/* ------------------------------------------------------------------ */

void fxo_fill(double *x, size_t n, double v) { /* ops.rs:173-181 */
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < n; i++) x[i] = v;
}

void fxo_copy(const double *src, double *dst, size_t n) { /* ops.rs:156-171 */
    memmove(dst, src, n * sizeof(double));
}

void fxo_axpy(double alpha, const double *x, double *y, size_t n) { /* ops.rs:183-207 */
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < n; i++) y[i] = fma(alpha, x[i], y[i]);
}

void fxo_scale(double *x, size_t n, double alpha) { /* ops.rs:209-223 */
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < n; i++) x[i] *= alpha;
}

void fxo_waxpy(double alpha, const double *x, double beta, const double *y, double *w,
               size_t n) { /* ops.rs:529-559: alpha.mul_add(x, beta * y) */
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < n; i++) w[i] = fma(alpha, x[i], beta * y[i]);
}

void fxo_aypx(double alpha, const double *x, double *y, size_t n) { /* ops.rs:561-585 */
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < n; i++) y[i] = fma(alpha, y[i], x[i]);
}

void fxo_pointwise_mult(const double *x, const double *y, double *z, size_t n) { /* :475-500 */
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < n; i++) z[i] = x[i] * y[i];
}

void fxo_pointwise_div(const double *x, const double *y, double *z, size_t n) { /* :502-527 */
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < n; i++) z[i] = x[i] / y[i];
}

void fxo_pointwise_max(const double *x, const double *y, double *z, size_t n) { /* :617-635 */
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < n; i++) z[i] = fmax(x[i], y[i]);
}

void fxo_pointwise_min(const double *x, const double *y, double *z, size_t n) { /* :637-655 */
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < n; i++) z[i] = fmin(x[i], y[i]);
}

void fxo_reciprocal(double *x, size_t n) { /* ops.rs:587-600 */
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < n; i++) x[i] = 1.0 / x[i];
}

void fxo_abs_val(double *x, size_t n) { /* ops.rs:602-615 */
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < n; i++) x[i] = fabs(x[i]);
}

/* ------------------------------------------------------------------ */
/* Reductions: Kahan per 4096-element chunk, kahan_merge across chunks */
/* ------------------------------------------------------------------ */

/* ops.rs:1127-1137 */
static void kahan_merge(double *a, double *ca, double b, double cb) {
    double y = b - (*ca + cb);
    double t = *a + y;
    double c = (t - *a) - y;
    *a = t;
    *ca = c;
}

enum { RK_SUMSQ = 0, RK_SUM = 1, RK_DOT = 2 };

static void chunk_kahan(int kind, const double *x, const double *y, size_t lo, size_t hi,
                        double *acc_out, double *comp_out) {
    double acc = 0.0, comp = 0.0;
    for (size_t i = lo; i < hi; i++) {
        double t_y;
        if (kind == RK_SUMSQ) {
            t_y = fma(x[i], x[i], -comp); /* ops.rs:280 v.mul_add(v, -comp) */
        } else if (kind == RK_SUM) {
            t_y = x[i] - comp; /* ops.rs:303 */
        } else {
            double prod = x[i] * y[i]; /* ops.rs:354-355 */
            t_y = prod - comp;
        }
        double t = acc + t_y;
        comp = (t - acc) - t_y;
        acc = t;
    }
    *acc_out = acc;
    *comp_out = comp;
}

static double kahan_reduce(int kind, const double *x, const double *y, size_t n) {
    if (n == 0) return 0.0;
    size_t nch = (n + KCHUNK - 1) / KCHUNK;
    double *parts = (double *)malloc(2 * nch * sizeof(double));
#pragma omp parallel for schedule(static)
    for (size_t c = 0; c < nch; c++) {
        size_t lo = c * KCHUNK, hi = lo + KCHUNK < n ? lo + KCHUNK : n;
        chunk_kahan(kind, x, y, lo, hi, &parts[2 * c], &parts[2 * c + 1]);
    }
    double s = 0.0, cs = 0.0;
    for (size_t c = 0; c < nch; c++) kahan_merge(&s, &cs, parts[2 * c], parts[2 * c + 1]);
    free(parts);
    return s;
}

double fxo_norm_l2(const double *x, size_t n) { return sqrt(kahan_reduce(RK_SUMSQ, x, 0, n)); }
double fxo_reduce_sum(const double *x, size_t n) { return kahan_reduce(RK_SUM, x, 0, n); }
double fxo_dot(const double *x, const double *y, size_t n) { return kahan_reduce(RK_DOT, x, y, n); }

/* ops.rs:317-331 / :657-671: per-chunk f64::max, then max across chunks.
 * f64::max / f64::min ignore a NaN operand, as C fmax / fmin do. */
double fxo_reduce_max(const double *x, size_t n) {
    double m = -INFINITY;
    for (size_t i = 0; i < n; i++) m = fmax(m, x[i]);
    return m;
}

double fxo_reduce_min(const double *x, size_t n) {
    double m = INFINITY;
    for (size_t i = 0; i < n; i++) m = fmin(m, x[i]);
    return m;
}

/* Trait default dot2 = two dots (crates/core/src/backend.rs:219-230). */
void fxo_dot2(const double *a, const double *b, const double *c, const double *d, size_t n,
              double *ab, double *cd) {
    *ab = fxo_dot(a, b, n);
    *cd = fxo_dot(c, d, n);
}

/* ------------------------------------------------------------------ */
/* Stencil                                                             */
/* ------------------------------------------------------------------ */

static int has_periodic(const fxo_bc *bcs) { /* ops.rs:9-23 */
    for (int i = 0; i < 4; i++)
        if (bcs[i].kind == FXO_BC_PERIODIC) return 1;
    return 0;
}

/* ops.rs:1139-1180 */
static double bc_value(const fxo_bc *bc, double self_val, double neighbor_val, double spacing) {
    switch (bc->kind) {
    case FXO_BC_DIRICHLET:
        return bc->a;
    case FXO_BC_NEUMANN:
        return fma(spacing, bc->a, neighbor_val);
    case FXO_BC_ROBIN: {
        double alpha = bc->a, beta = bc->b, g = bc->g;
        if (fabs(beta) < 1e-30) {
            if (fabs(alpha) < 1e-30) return 0.0;
            return g / alpha;
        }
        double du_dn = (g - alpha * self_val) / beta;
        return fma(spacing, du_dn, neighbor_val);
    }
    default:
        return 0.0;
    }
}

/* ops.rs:796-843; bcs = {top, bottom, left, right} */
static void apply_boundaries(const double *src, double *dst, size_t rows, size_t cols, double dx,
                             double dy, const fxo_bc *bcs) {
    size_t last_row = rows - 1, last_col = cols - 1;
    for (size_t col = 0; col < cols; col++) {
        dst[col] = bc_value(&bcs[0], src[col], src[cols + col], dy);
        dst[last_row * cols + col] = bc_value(&bcs[1], src[last_row * cols + col],
                                              src[(last_row - 1) * cols + col], dy);
    }
    for (size_t row = 1; row < last_row; row++) {
        size_t idx = row * cols;
        dst[idx] = bc_value(&bcs[2], src[idx], src[idx + 1], dx);
        dst[idx + last_col] = bc_value(&bcs[3], src[idx + last_col], src[idx + last_col - 1], dx);
    }
}

typedef struct {
    int mode; /* 5 = five-point by offset, 9 = nine-point by offset, 0 = generic list */
    double c, n, s, w, e, nw, ne, sw, se;
    int ne_;
    const int *dr, *dc;
    const double *wt;
} stencil_w;

/* Weight extraction by offset, ops.rs:898-916 (5-pt) and :953-975 (9-pt). */
static int stencil_setup(stencil_w *sw, int ne, const int *dr, const int *dc, const double *w) {
    memset(sw, 0, sizeof(*sw));
    if (ne < 1) return FXO_ERR_INVALID_STENCIL; /* stencil.rs:116-126 */
    sw->ne_ = ne;
    sw->dr = dr;
    sw->dc = dc;
    sw->wt = w;
    if (ne == 5 || ne == 9) {
        sw->mode = ne;
        for (int k = 0; k < ne; k++) {
            int r = dr[k], c = dc[k];
            if (r == 0 && c == 0) sw->c = w[k];
            else if (r == -1 && c == 0) sw->n = w[k];
            else if (r == 1 && c == 0) sw->s = w[k];
            else if (r == 0 && c == -1) sw->w = w[k];
            else if (r == 0 && c == 1) sw->e = w[k];
            else if (ne == 9 && r == -1 && c == -1) sw->nw = w[k];
            else if (ne == 9 && r == -1 && c == 1) sw->ne = w[k];
            else if (ne == 9 && r == 1 && c == -1) sw->sw = w[k];
            else if (ne == 9 && r == 1 && c == 1) sw->se = w[k];
        }
        return FXO_OK;
    }
    /* Generic path (ops.rs:869-883) indexes (row+dr, col+dc) unchecked; only radius-1
     * offsets stay inside the grid for every interior point. */
    for (int k = 0; k < ne; k++)
        if (dr[k] < -1 || dr[k] > 1 || dc[k] < -1 || dc[k] > 1) return FXO_ERR_INVALID_STENCIL;
    sw->mode = 0;
    return FXO_OK;
}

/* Stencil value at an interior point, with the reference's FMA nesting
 * (ops.rs:922-935 five-point, :981-1006 nine-point, :875-881 generic). */
static inline double stencil_at(const stencil_w *sw, const double *src, size_t row, size_t col,
                                size_t cols) {
    size_t base = row * cols, north = (row - 1) * cols, south = (row + 1) * cols;
    if (sw->mode == 5) {
        return fma(sw->c, src[base + col],
                   fma(sw->n, src[north + col],
                       fma(sw->s, src[south + col],
                           fma(sw->w, src[base + col - 1], sw->e * src[base + col + 1]))));
    }
    if (sw->mode == 9) {
        return fma(sw->c, src[base + col],
               fma(sw->n, src[north + col],
               fma(sw->s, src[south + col],
               fma(sw->w, src[base + col - 1],
               fma(sw->e, src[base + col + 1],
               fma(sw->nw, src[north + col - 1],
               fma(sw->ne, src[north + col + 1],
               fma(sw->sw, src[south + col - 1], sw->se * src[south + col + 1]))))))));
    }
    double acc = 0.0;
    for (int k = 0; k < sw->ne_; k++) {
        size_t r = (size_t)((long)row + sw->dr[k]);
        size_t c = (size_t)((long)col + sw->dc[k]);
        acc = fma(sw->wt[k], src[r * cols + c], acc);
    }
    return acc;
}

/* ops.rs:76-127 */
int fxo_apply_stencil(const double *in, double *out, size_t rows, size_t cols, double dx, double dy,
                      int ne, const int *dr, const int *dc, const double *w, const fxo_bc *bcs) {
    if (has_periodic(bcs)) return FXO_ERR_UNSUPPORTED;
    stencil_w sw;
    int st = stencil_setup(&sw, ne, dr, dc, w);
    if (st) return st;
    apply_boundaries(in, out, rows, cols, dx, dy, bcs);
#pragma omp parallel for schedule(static)
    for (size_t row = 1; row < rows - 1; row++)
        for (size_t col = 1; col < cols - 1; col++)
            out[row * cols + col] = stencil_at(&sw, in, row, col, cols);
    return FXO_OK;
}

/* ops.rs:129-154: apply_stencil, then output *= coeff over the whole array. */
int fxo_apply_stencil_var(const double *in, double *out, const double *coeff, size_t rows,
                          size_t cols, double dx, double dy, int ne, const int *dr, const int *dc,
                          const double *w, const fxo_bc *bcs) {
    int st = fxo_apply_stencil(in, out, rows, cols, dx, dy, ne, dr, dc, w, bcs);
    if (st) return st;
    size_t n = rows * cols;
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < n; i++) out[i] *= coeff[i];
    return FXO_OK;
}

/* ops.rs:225-269 + fused_5pt_axpy_row :1011-1125; boundary points of y untouched. */
int fxo_stencil_axpy(double alpha, const double *x, double *y, size_t rows, size_t cols, int ne,
                     const int *dr, const int *dc, const double *w, const fxo_bc *bcs) {
    if (has_periodic(bcs)) return FXO_ERR_UNSUPPORTED;
    stencil_w sw;
    int st = stencil_setup(&sw, ne, dr, dc, w);
    if (st) return st;
#pragma omp parallel for schedule(static)
    for (size_t row = 1; row < rows - 1; row++)
        for (size_t col = 1; col < cols - 1; col++) {
            size_t i = row * cols + col;
            y[i] = fma(alpha, stencil_at(&sw, x, row, col, cols), y[i]);
        }
    return FXO_OK;
}

/* crates/runtime/src/field.rs:386-431 */
void fxo_zero_boundaries(double *x, size_t rows, size_t cols) {
    for (size_t c = 0; c < cols; c++) {
        x[c] = 0.0;
        x[(rows - 1) * cols + c] = 0.0;
    }
    for (size_t r = 1; r < rows - 1; r++) {
        x[r * cols] = 0.0;
        x[r * cols + cols - 1] = 0.0;
    }
}

/* ------------------------------------------------------------------ */
/* Convection-diffusion, ops.rs:673-791                                */
/* ------------------------------------------------------------------ */

static inline double conv_diff_at_k(const double *src, double kap, const double *vxs,
                                    const double *vys, size_t idx, size_t cols, double inv_dx,
                                    double inv_dy, double inv_dx2, double inv_dy2) {
    double c = src[idx];
    double lap = fma(src[idx - 1] + src[idx + 1], inv_dx2,
                     (src[idx - cols] + src[idx + cols]) * inv_dy2) -
                 2.0 * (inv_dx2 + inv_dy2) * c; /* ops.rs:711-713 */
    double diff = kap * lap;
    double vx_i = vxs[idx], vy_i = vys[idx];
    double dudx = vx_i >= 0.0 ? (c - src[idx - 1]) * inv_dx : (src[idx + 1] - c) * inv_dx;
    double dudy = vy_i >= 0.0 ? (c - src[idx - cols]) * inv_dy : (src[idx + cols] - c) * inv_dy;
    double conv = fma(vx_i, dudx, vy_i * dudy); /* ops.rs:729-730 */
    return diff + conv;
}

static inline double conv_diff_at(const double *src, const double *k, const double *vxs,
                                  const double *vys, size_t idx, size_t cols, double inv_dx,
                                  double inv_dy, double inv_dx2, double inv_dy2) {
    return conv_diff_at_k(src, k[idx], vxs, vys, idx, cols, inv_dx, inv_dy, inv_dx2, inv_dy2);
}

void fxo_apply_conv_diff(const double *u, double *out, const double *kappa, const double *vx,
                         const double *vy, size_t rows, size_t cols, double dx, double dy) {
    double inv_dx = 1.0 / dx, inv_dy = 1.0 / dy;
    double inv_dx2 = inv_dx * inv_dx, inv_dy2 = inv_dy * inv_dy;
    for (size_t col = 0; col < cols; col++) { /* ops.rs:696-704 */
        out[col] = 0.0;
        out[(rows - 1) * cols + col] = 0.0;
    }
    for (size_t row = 1; row < rows - 1; row++) {
        out[row * cols] = 0.0;
        out[row * cols + cols - 1] = 0.0;
    }
#pragma omp parallel for schedule(static)
    for (size_t row = 1; row < rows - 1; row++)
        for (size_t col = 1; col < cols - 1; col++) {
            size_t idx = row * cols + col;
            out[idx] = conv_diff_at(u, kappa, vx, vy, idx, cols, inv_dx, inv_dy, inv_dx2, inv_dy2);
        }
}

void fxo_conv_diff_axpy(double alpha, const double *u, double *out, const double *kappa,
                        const double *vx, const double *vy, size_t rows, size_t cols, double dx,
                        double dy) {
    double inv_dx = 1.0 / dx, inv_dy = 1.0 / dy;
    double inv_dx2 = inv_dx * inv_dx, inv_dy2 = inv_dy * inv_dy;
#pragma omp parallel for schedule(static)
    for (size_t row = 1; row < rows - 1; row++)
        for (size_t col = 1; col < cols - 1; col++) {
            size_t idx = row * cols + col;
            double v = conv_diff_at(u, kappa, vx, vy, idx, cols, inv_dx, inv_dy, inv_dx2, inv_dy2);
            out[idx] = fma(alpha, v, out[idx]); /* ops.rs:786-787 */
        }
}

/* ------------------------------------------------------------------ */
/* Multigrid ops, reference semantics: ops.rs:369-473                  */
/* ------------------------------------------------------------------ */

/* ops.rs:369-399: 2x2 average with clamped indices.  The reference indexes
 * fine[2*row] unchecked; a coarse grid whose row 2*(crows-1) lies outside the
 * fine grid makes it panic, here it is a dimension error. */
int fxo_restrict(const double *fs, double *cs, size_t frows, size_t fcols, size_t crows,
                 size_t ccols) {
    if (crows == 0 || ccols == 0 || 2 * (crows - 1) > frows - 1 || 2 * (ccols - 1) > fcols - 1)
        return FXO_ERR_DIMENSION_MISMATCH;
    size_t fr_max = frows - 1, fc_max = fcols - 1, fc = fcols;
#pragma omp parallel for schedule(static)
    for (size_t row = 0; row < crows; row++)
        for (size_t col = 0; col < ccols; col++) {
            size_t fr = row * 2, fcc = col * 2;
            size_t fr1 = fr + 1 < fr_max ? fr + 1 : fr_max;
            size_t fc1 = fcc + 1 < fc_max ? fcc + 1 : fc_max;
            cs[row * ccols + col] = 0.25 * (fs[fr * fc + fcc] + fs[fr1 * fc + fcc] +
                                            fs[fr * fc + fc1] + fs[fr1 * fc + fc1]);
        }
    return FXO_OK;
}

/* ops.rs:401-423: fine[i,j] += coarse[i/2, j/2].  Out-of-range coarse index
 * (a panic in the reference) is a dimension error. */
int fxo_prolong(const double *cs, double *fs, size_t crows, size_t ccols, size_t frows,
                size_t fcols) {
    if ((frows - 1) / 2 > crows - 1 || (fcols - 1) / 2 > ccols - 1)
        return FXO_ERR_DIMENSION_MISMATCH;
#pragma omp parallel for schedule(static)
    for (size_t row = 0; row < frows; row++) {
        size_t cr = row / 2;
        for (size_t col = 0; col < fcols; col++) fs[row * fcols + col] += cs[cr * ccols + col / 2];
    }
    return FXO_OK;
}

/* ops.rs:425-473: in-place lexicographic sweep, x += omega * D^-1 (b - A x),
 * with A x summed over the stencil entries in entry order. */
int fxo_weighted_jacobi(double *x, const double *b, double omega, size_t rows, size_t cols, int ne,
                        const int *dr, const int *dc, const double *w) {
    if (ne < 1) return FXO_ERR_INVALID_STENCIL;
    for (int k = 0; k < ne; k++)
        if (dr[k] < -1 || dr[k] > 1 || dc[k] < -1 || dc[k] > 1) return FXO_ERR_INVALID_STENCIL;
    double diag = -4.0;
    for (int k = 0; k < ne; k++)
        if (dr[k] == 0 && dc[k] == 0) {
            diag = w[k];
            break;
        }
    double inv_diag = 1.0 / diag;
    for (size_t row = 1; row < rows - 1; row++)
        for (size_t col = 1; col < cols - 1; col++) {
            size_t idx = row * cols + col;
            double ax = 0.0;
            for (int k = 0; k < ne; k++) {
                size_t r = (size_t)((long)row + dr[k]), c = (size_t)((long)col + dc[k]);
                ax = fma(w[k], x[r * cols + c], ax);
            }
            double residual = b[idx] - ax;
            x[idx] = fma(omega, inv_diag * residual, x[idx]);
        }
    return FXO_OK;
}

/* pipelined_cg.rs:440-456 (separate-op fallback of the 6-way update). */
void fxo_pcg_fused_update(double alpha, double beta, double *z, double *t, double *p, double *x,
                          double *r, double *w, const double *q, size_t n) {
#pragma omp parallel for schedule(static)
    for (size_t i = 0; i < n; i++) {
        z[i] = fma(1.0, q[i], z[i] * beta);
        t[i] = fma(1.0, w[i], t[i] * beta);
        p[i] = fma(1.0, r[i], p[i] * beta);
        x[i] = fma(alpha, p[i], x[i]);
        r[i] = fma(-alpha, t[i], r[i]);
        w[i] = fma(-alpha, z[i], w[i]);
    }
}

/* ------------------------------------------------------------------ */
/* Vertex-centred multigrid primitives                                 */
/* a5 = {a_c, a_n, a_s, a_w, a_e}: the 5-point operator on this level.  */
/* ------------------------------------------------------------------ */

static inline double op5(const double *a5, const double *x, size_t i, size_t cols) {
    return fma(a5[0], x[i],
               fma(a5[1], x[i - cols], fma(a5[2], x[i + cols], fma(a5[3], x[i - 1], a5[4] * x[i + 1]))));
}

/* x_out = x_in + (omega / a_c) (b - A x_in) on interior points. */
void fxo_jacobi_sweep(const double *x_in, double *x_out, const double *b, double omega,
                      size_t rows, size_t cols, const double *a5) {
    double wd = omega / a5[0];
#pragma omp parallel for schedule(static)
    for (size_t row = 1; row < rows - 1; row++)
        for (size_t col = 1; col < cols - 1; col++) {
            size_t i = row * cols + col;
            double r = b[i] - op5(a5, x_in, i, cols);
            x_out[i] = fma(wd, r, x_in[i]);
        }
}

void fxo_residual(const double *x, const double *b, double *r, size_t rows, size_t cols,
                  const double *a5) {
#pragma omp parallel for schedule(static)
    for (size_t row = 1; row < rows - 1; row++)
        for (size_t col = 1; col < cols - 1; col++) {
            size_t i = row * cols + col;
            r[i] = b[i] - op5(a5, x, i, cols);
        }
}

static inline double fw_at(const double *f, size_t i, size_t fc) {
    double e = (f[i - fc] + f[i + fc]) + (f[i - 1] + f[i + 1]);
    double d = (f[i - fc - 1] + f[i - fc + 1]) + (f[i + fc - 1] + f[i + fc + 1]);
    return (4.0 * f[i] + (2.0 * e + d)) * 0.0625;
}

/* Full weighting onto coarse interior points; coarse ring set to 0. */
int fxo_restrict_fw(const double *fine, double *coarse, size_t frows, size_t fcols, size_t crows,
                    size_t ccols) {
    if (frows != 2 * (crows - 1) + 1 || fcols != 2 * (ccols - 1) + 1)
        return FXO_ERR_DIMENSION_MISMATCH;
    fxo_zero_boundaries(coarse, crows, ccols);
#pragma omp parallel for schedule(static)
    for (size_t I = 1; I < crows - 1; I++)
        for (size_t J = 1; J < ccols - 1; J++)
            coarse[I * ccols + J] = fw_at(fine, (2 * I) * fcols + 2 * J, fcols);
    return FXO_OK;
}

/* fine[interior] += bilinear interpolation of coarse. */
int fxo_prolong_bilinear(const double *c, double *fine, size_t crows, size_t ccols, size_t frows,
                         size_t fcols) {
    if (frows != 2 * (crows - 1) + 1 || fcols != 2 * (ccols - 1) + 1)
        return FXO_ERR_DIMENSION_MISMATCH;
#pragma omp parallel for schedule(static)
    for (size_t i = 1; i < frows - 1; i++)
        for (size_t j = 1; j < fcols - 1; j++) {
            size_t I = i / 2, J = j / 2, k = I * ccols + J;
            double e;
            if (!(i & 1) && !(j & 1)) e = c[k];
            else if ((i & 1) && !(j & 1)) e = 0.5 * (c[k] + c[k + ccols]);
            else if (!(i & 1) && (j & 1)) e = 0.5 * (c[k] + c[k + 1]);
            else e = 0.25 * ((c[k] + c[k + ccols]) + (c[k + 1] + c[k + ccols + 1]));
            fine[i * fcols + j] += e;
        }
    return FXO_OK;
}

/* ------------------------------------------------------------------ */
/* Operator A v = v + coeff * S v (linear_solver.rs:7-22)              */
/* ------------------------------------------------------------------ */

static size_t op_len(const fxo_op *op) { return op->rows * op->cols; }

/* conv-diff operator: ring out = inp; interior fma(coeff, CD(inp), sigma * inp) */
static void apply_cd(const fxo_op *op, double *out, const double *inp) {
    size_t rows = op->rows, cols = op->cols;
    double inv_dx = 1.0 / op->dx, inv_dy = 1.0 / op->dy;
    double inv_dx2 = inv_dx * inv_dx, inv_dy2 = inv_dy * inv_dy;
    for (size_t col = 0; col < cols; col++) {
        out[col] = inp[col];
        out[(rows - 1) * cols + col] = inp[(rows - 1) * cols + col];
    }
    for (size_t row = 1; row < rows - 1; row++) {
        out[row * cols] = inp[row * cols];
        out[row * cols + cols - 1] = inp[row * cols + cols - 1];
    }
#pragma omp parallel for schedule(static)
    for (size_t row = 1; row < rows - 1; row++)
        for (size_t col = 1; col < cols - 1; col++) {
            size_t idx = row * cols + col;
            double kap = op->kappa ? op->kappa[idx] : op->kappa_s;
            double v = conv_diff_at_k(inp, kap, op->vx, op->vy, idx, cols, inv_dx, inv_dy, inv_dx2, inv_dy2);
            out[idx] = fma(op->coeff, v, op->sigma * inp[idx]);
        }
}

void fxo_cd_jacobi_apply(void *ctx, double *z, const double *r) {
    const fxo_op *op = (const fxo_op *)ctx;
    size_t rows = op->rows, cols = op->cols;
    double inv_dx = 1.0 / op->dx, inv_dy = 1.0 / op->dy;
    double k2 = 2.0 * (inv_dx * inv_dx + inv_dy * inv_dy);
#pragma omp parallel for schedule(static)
    for (size_t row = 0; row < rows; row++)
        for (size_t col = 0; col < cols; col++) {
            size_t idx = row * cols + col;
            if (row == 0 || col == 0 || row == rows - 1 || col == cols - 1) {
                z[idx] = r[idx];
                continue;
            }
            double kap = op->kappa ? op->kappa[idx] : op->kappa_s;
            double dcd = fma(-kap, k2, fma(fabs(op->vx[idx]), inv_dx, fabs(op->vy[idx]) * inv_dy));
            z[idx] = r[idx] / fma(op->coeff, dcd, op->sigma);
        }
}

/* out = inp; out += coeff * S(inp)  (cg.rs:106-109, pipelined_cg.rs:332-343) */
static int apply_op(const fxo_op *op, double *out, const double *inp) {
    if (op->cd) {
        apply_cd(op, out, inp);
        return 0;
    }
    if (out != inp) fxo_copy(inp, out, op_len(op));
    /* stencil_axpy reads inp while writing out; out != inp here so a copy suffices */
    return fxo_stencil_axpy(op->coeff, inp, out, op->rows, op->cols, op->ne, op->dr, op->dc,
                            op->w, op->bcs);
}

int fxo_op_apply(const fxo_op *op, double *out, const double *v) { return apply_op(op, out, v); }

static void set_stats(fxo_stats *st, size_t it, double res, int reason) {
    st->iterations = it;
    st->residual = res;
    st->reason = reason;
}

/* cg.rs:96-164 (pc == NULL) and cg.rs:178-256 (preconditioned). */
int fxo_cg_solve(const fxo_op *op, double *x, const double *b, double tol, size_t max_iter,
                 fxo_pc_fn pc, void *pc_ctx, fxo_stats *st) {
    size_t n = op_len(op);
    double *r = calloc(n, sizeof(double)), *z = calloc(n, sizeof(double));
    double *p = calloc(n, sizeof(double)), *ap = calloc(n, sizeof(double));
    int rc = apply_op(op, ap, x);
    if (rc) goto out;
    fxo_copy(b, r, n);
    fxo_axpy(-1.0, ap, r, n);
    if (!pc) {
        fxo_copy(r, p, n);
        double rs_old = fxo_dot(r, r, n);
        for (size_t i = 0; i < max_iter; i++) {
            if (sqrt(rs_old) < tol) {
                set_stats(st, i, sqrt(rs_old), 0);
                goto out;
            }
            apply_op(op, ap, p);
            double p_ap = fxo_dot(p, ap, n);
            if (fabs(p_ap) < 1e-30) {
                set_stats(st, i, sqrt(rs_old), 2);
                goto out;
            }
            double alpha = rs_old / p_ap;
            fxo_axpy(alpha, p, x, n);
            fxo_axpy(-alpha, ap, r, n);
            double rs_new = fxo_dot(r, r, n);
            double beta = rs_new / rs_old;
            fxo_scale(p, n, beta);
            fxo_axpy(1.0, r, p, n);
            rs_old = rs_new;
        }
        set_stats(st, max_iter, sqrt(rs_old), 1);
        goto out;
    }
    fxo_fill(z, n, 0.0);
    pc(pc_ctx, z, r);
    fxo_copy(z, p, n);
    double rz_old = fxo_dot(r, z, n);
    for (size_t i = 0; i < max_iter; i++) {
        double r_norm = sqrt(fxo_dot(r, r, n));
        if (r_norm < tol) {
            set_stats(st, i, r_norm, 0);
            goto out;
        }
        apply_op(op, ap, p);
        double p_ap = fxo_dot(p, ap, n);
        if (fabs(p_ap) < 1e-30) {
            set_stats(st, i, r_norm, 2);
            goto out;
        }
        double alpha = rz_old / p_ap;
        fxo_axpy(alpha, p, x, n);
        fxo_axpy(-alpha, ap, r, n);
        fxo_fill(z, n, 0.0);
        pc(pc_ctx, z, r);
        double rz_new = fxo_dot(r, z, n);
        double beta = rz_new / rz_old;
        fxo_scale(p, n, beta);
        fxo_axpy(1.0, z, p, n);
        rz_old = rz_new;
    }
    set_stats(st, max_iter, sqrt(fxo_dot(r, r, n)), 1);
out:
    free(r);
    free(z);
    free(p);
    free(ap);
    return rc;
}

/* pipelined_cg.rs:353-424 */
int fxo_pipelined_cg_solve(const fxo_op *op, double *x, const double *b, double tol,
                           size_t max_iter, fxo_stats *st) {
    size_t n = op_len(op);
    double *r = calloc(n, 8), *p = calloc(n, 8), *w = calloc(n, 8), *t = calloc(n, 8);
    double *z = calloc(n, 8), *q = calloc(n, 8);
    int rc = apply_op(op, q, x);
    if (rc) goto out;
    fxo_copy(b, r, n);
    fxo_axpy(-1.0, q, r, n);
    apply_op(op, w, r);
    fxo_fill(p, n, 0.0);
    fxo_fill(t, n, 0.0);
    fxo_fill(z, n, 0.0);
    double gamma_prev = INFINITY, alpha_prev = INFINITY;
    for (size_t k = 0; k < max_iter; k++) {
        double gamma, delta;
        fxo_dot2(r, r, r, w, n, &gamma, &delta);
        if (sqrt(gamma) < tol) {
            set_stats(st, k, sqrt(gamma), 0);
            goto out;
        }
        apply_op(op, q, w);
        double beta = gamma / gamma_prev;
        double alpha = gamma / (delta - beta * gamma / alpha_prev);
        fxo_pcg_fused_update(alpha, beta, z, t, p, x, r, w, q, n);
        gamma_prev = gamma;
        alpha_prev = alpha;
    }
    set_stats(st, max_iter, sqrt(fxo_dot(r, r, n)), 1);
out:
    free(r); free(p); free(w); free(t); free(z); free(q);
    return rc;
}

/* Preconditioned pipelined CG (Ghysels & Vanroose 2014, Algorithm 4).  The reference's
 * PipelinedCgSolver (pipelined_cg.rs:353-424) is its unpreconditioned case; the scalar
 * recurrence and the fma forms of the update are kept from it (fxo_pcg_fused_update).  Stop test
 * on ||r||_2 at the loop top, as cg.rs does. */
int fxo_pipelined_pcg_solve(const fxo_op *op, double *x, const double *b, double tol, size_t max_iter,
                            fxo_pc_fn pc, void *pc_ctx, fxo_stats *st) {
    size_t n = op_len(op);
    double *r = calloc(n, 8), *u = calloc(n, 8), *w = calloc(n, 8), *m = calloc(n, 8);
    double *nn = calloc(n, 8), *z = calloc(n, 8), *q = calloc(n, 8), *s = calloc(n, 8);
    double *p = calloc(n, 8);
    int rc = apply_op(op, nn, x);
    if (rc) goto out;
    fxo_copy(b, r, n);
    fxo_axpy(-1.0, nn, r, n);
    fxo_fill(u, n, 0.0);
    pc(pc_ctx, u, r);
    apply_op(op, w, u);
    double gamma_prev = INFINITY, alpha_prev = INFINITY;
    for (size_t k = 0; k < max_iter; k++) {
        double gamma = fxo_dot(r, u, n), delta = fxo_dot(w, u, n), rr = fxo_dot(r, r, n);
        if (sqrt(rr) < tol) {
            set_stats(st, k, sqrt(rr), 0);
            goto out;
        }
        fxo_fill(m, n, 0.0);
        pc(pc_ctx, m, w);
        apply_op(op, nn, m);
        double beta = gamma / gamma_prev;
        double alpha = gamma / (delta - beta * gamma / alpha_prev);
#pragma omp parallel for schedule(static)
        for (size_t i = 0; i < n; i++) {
            z[i] = fma(1.0, nn[i], z[i] * beta);
            q[i] = fma(1.0, m[i], q[i] * beta);
            s[i] = fma(1.0, w[i], s[i] * beta);
            p[i] = fma(1.0, u[i], p[i] * beta);
            x[i] = fma(alpha, p[i], x[i]);
            r[i] = fma(-alpha, s[i], r[i]);
            u[i] = fma(-alpha, q[i], u[i]);
            w[i] = fma(-alpha, z[i], w[i]);
        }
        gamma_prev = gamma;
        alpha_prev = alpha;
    }
    set_stats(st, max_iter, sqrt(fxo_dot(r, r, n)), 1);
out:
    free(r); free(u); free(w); free(m); free(nn); free(z); free(q); free(s); free(p);
    return rc;
}

/* bicgstab.rs:90-210 (pc == NULL) and :218-346 (right-preconditioned). */
int fxo_bicgstab_solve(const fxo_op *op, double *x, const double *b, double tol, size_t max_iter,
                       fxo_pc_fn pc, void *pc_ctx, fxo_stats *st) {
    size_t n = op_len(op);
    double *r = calloc(n, 8), *r_hat = calloc(n, 8), *p = calloc(n, 8), *v = calloc(n, 8);
    double *s = calloc(n, 8), *t = calloc(n, 8), *ph = calloc(n, 8), *sh = calloc(n, 8);
    int rc = apply_op(op, v, x);
    if (rc) goto out;
    fxo_copy(b, r, n);
    fxo_axpy(-1.0, v, r, n);
    fxo_copy(r, r_hat, n);
    double rho = 1.0, alpha = 1.0, omega = 1.0;
    fxo_fill(v, n, 0.0);
    fxo_fill(p, n, 0.0);
    for (size_t i = 0; i < max_iter; i++) {
        double r_norm = sqrt(fxo_dot(r, r, n));
        if (r_norm < tol) {
            set_stats(st, i, r_norm, 0);
            goto out;
        }
        double rho_new = fxo_dot(r_hat, r, n);
        if (fabs(rho_new) < 1e-30) {
            set_stats(st, i, r_norm, 2);
            goto out;
        }
        double beta = (rho_new / rho) * (alpha / omega);
        fxo_axpy(-omega, v, p, n);
        fxo_scale(p, n, beta);
        fxo_axpy(1.0, r, p, n);
        const double *pp = p;
        if (pc) {
            fxo_fill(ph, n, 0.0);
            pc(pc_ctx, ph, p);
            pp = ph;
        }
        apply_op(op, v, pp);
        double rv = fxo_dot(r_hat, v, n);
        if (fabs(rv) < 1e-30) {
            set_stats(st, i, r_norm, 2);
            goto out;
        }
        alpha = rho_new / rv;
        fxo_copy(r, s, n);
        fxo_axpy(-alpha, v, s, n);
        double s_norm = sqrt(fxo_dot(s, s, n));
        if (s_norm < tol) {
            fxo_axpy(alpha, pp, x, n);
            set_stats(st, i, s_norm, 0);
            goto out;
        }
        const double *ss = s;
        if (pc) {
            fxo_fill(sh, n, 0.0);
            pc(pc_ctx, sh, s);
            ss = sh;
        }
        apply_op(op, t, ss);
        double ts = fxo_dot(t, s, n);
        double tt = fxo_dot(t, t, n);
        if (fabs(tt) < 1e-30) {
            fxo_axpy(alpha, pp, x, n);
            set_stats(st, i, s_norm, 2);
            goto out;
        }
        omega = ts / tt;
        fxo_axpy(alpha, pp, x, n);
        fxo_axpy(omega, ss, x, n);
        fxo_copy(s, r, n);
        fxo_axpy(-omega, t, r, n);
        rho = rho_new;
    }
    set_stats(st, max_iter, sqrt(fxo_dot(r, r, n)), 1);
out:
    free(r); free(r_hat); free(p); free(v); free(s); free(t); free(ph); free(sh);
    return rc;
}

/* gmres.rs:803-837 */
static void gmres_build_solution(double *x, double **vv, const double *hh, const double *grs,
                                 size_t restart, size_t k, size_t n) {
    if (k == 0) return;
    size_t mp1 = restart + 1;
    double *y = calloc(k, sizeof(double));
    for (size_t ii = k; ii-- > 0;) {
        double s = grs[ii];
        for (size_t j = ii + 1; j < k; j++) s -= hh[j * mp1 + ii] * y[j];
        double diag = hh[ii * mp1 + ii];
        if (fabs(diag) < 1e-30) break;
        y[ii] = s / diag;
    }
    for (size_t ii = 0; ii < k; ii++) fxo_axpy(y[ii], vv[ii], x, n);
    free(y);
}

/* gmres.rs:463-633 (pc == NULL) and :641-801 (left-preconditioned). */
int fxo_gmres_solve(const fxo_op *op, double *x, const double *b, size_t m, double tol,
                    size_t max_iter, fxo_pc_fn pc, void *pc_ctx, fxo_stats *st) {
    size_t n = op_len(op), mp1 = m + 1;
    double **vv = malloc(mp1 * sizeof(double *));
    for (size_t i = 0; i < mp1; i++) vv[i] = calloc(n, 8);
    double *w = calloc(n, 8), *hh = calloc(mp1 * m, 8), *cc = calloc(m, 8), *ss = calloc(m, 8);
    double *grs = calloc(mp1, 8);
    size_t total_its = 0;
    int rc = 0;
#define H(i, j) hh[(j) * mp1 + (i)]
    for (;;) {
        double *v0 = vv[0];
        if (!pc) {
            rc = apply_op(op, v0, x);
            if (rc) goto out;
            fxo_scale(v0, n, -1.0);
            fxo_axpy(1.0, b, v0, n);
        } else {
            rc = apply_op(op, w, x);
            if (rc) goto out;
            fxo_scale(w, n, -1.0);
            fxo_axpy(1.0, b, w, n);
            fxo_fill(v0, n, 0.0);
            pc(pc_ctx, v0, w);
        }
        double beta = sqrt(fxo_dot(v0, v0, n));
        if (beta < tol) {
            set_stats(st, total_its, beta, 0);
            goto out;
        }
        fxo_scale(v0, n, 1.0 / beta);
        memset(grs, 0, mp1 * 8);
        grs[0] = beta;
        memset(hh, 0, mp1 * m * 8);
        double cur_resid = beta;
        size_t k = 0;
        while (k < m) {
            if (total_its >= max_iter) {
                gmres_build_solution(x, vv, hh, grs, m, k, n);
                set_stats(st, total_its, cur_resid, 1);
                goto out;
            }
            apply_op(op, w, vv[k]);
            if (pc) {
                fxo_fill(vv[k + 1], n, 0.0);
                pc(pc_ctx, vv[k + 1], w);
                fxo_copy(vv[k + 1], w, n);
            }
            for (size_t j = 0; j <= k; j++) {
                double h = fxo_dot(w, vv[j], n);
                H(j, k) = h;
                fxo_axpy(-h, vv[j], w, n);
            }
            double h_kp1_k = sqrt(fxo_dot(w, w, n));
            H(k + 1, k) = h_kp1_k;
            if (h_kp1_k > 1e-30) {
                fxo_copy(w, vv[k + 1], n);
                fxo_scale(vv[k + 1], n, 1.0 / h_kp1_k);
            }
            for (size_t j = 0; j < k; j++) {
                double h_j = H(j, k), h_jp1 = H(j + 1, k);
                double cj = cc[j], sj = ss[j];
                H(j, k) = fma(cj, h_j, sj * h_jp1);
                H(j + 1, k) = fma(cj, h_jp1, -sj * h_j);
            }
            double a = H(k, k), bv = H(k + 1, k);
            double rr = hypot(a, bv);
            if (fabs(rr) < 1e-30) {
                gmres_build_solution(x, vv, hh, grs, m, k, n);
                set_stats(st, total_its, cur_resid, 2);
                goto out;
            }
            cc[k] = a / rr;
            ss[k] = bv / rr;
            H(k, k) = rr;
            H(k + 1, k) = 0.0;
            double g_k = grs[k];
            grs[k] = cc[k] * g_k;
            grs[k + 1] = -ss[k] * g_k;
            cur_resid = fabs(grs[k + 1]);
            total_its++;
            k++;
            if (cur_resid < tol) break;
            if (h_kp1_k <= 1e-30) break;
        }
        gmres_build_solution(x, vv, hh, grs, m, k, n);
        if (cur_resid < tol) {
            set_stats(st, total_its, cur_resid, 0);
            goto out;
        }
        if (total_its >= max_iter) {
            set_stats(st, total_its, cur_resid, 1);
            goto out;
        }
    }
#undef H
out:
    for (size_t i = 0; i < mp1; i++) free(vv[i]);
    free(vv); free(w); free(hh); free(cc); free(ss); free(grs);
    return rc;
}

/* Flexible CG.  New (the reference has no flexible solver): PCG whose beta is the
 * Polak-Ribiere form z_{k+1}.(r_{k+1} - r_k) / (z_k.r_k) of Golub & Ye (1999, inexact
 * preconditioned CG) -- equal, in exact arithmetic, to Notay's FCG(1) (2000) -- evaluated as
 * (r_{k+1}.z_{k+1} - r_k.z_{k+1}) / rz_old.  With a fixed SPD preconditioner r_k.z_{k+1} = 0
 * in exact arithmetic and the method is PCG; with one that changes between applications
 * (an inner iterative solve) the directions stay locally A-orthogonal.  Loop, stop test
 * (||r|| < tol at the loop top) and breakdown test as fxo_cg_solve's preconditioned branch. */
int fxo_fcg_solve(const fxo_op *op, double *x, const double *b, double tol, size_t max_iter,
                  fxo_pc_fn pc, void *pc_ctx, fxo_stats *st) {
    size_t n = op_len(op);
    double *r = calloc(n, 8), *rp = calloc(n, 8), *z = calloc(n, 8), *p = calloc(n, 8), *ap = calloc(n, 8);
    int rc = apply_op(op, ap, x);
    if (rc) goto out;
    fxo_copy(b, r, n);
    fxo_axpy(-1.0, ap, r, n);
    fxo_fill(z, n, 0.0);
    pc(pc_ctx, z, r);
    fxo_copy(z, p, n);
    double rz_old = fxo_dot(r, z, n);
    for (size_t i = 0; i < max_iter; i++) {
        double r_norm = sqrt(fxo_dot(r, r, n));
        if (r_norm < tol) {
            set_stats(st, i, r_norm, 0);
            goto out;
        }
        apply_op(op, ap, p);
        double p_ap = fxo_dot(p, ap, n);
        if (fabs(p_ap) < 1e-30) {
            set_stats(st, i, r_norm, 2);
            goto out;
        }
        double alpha = rz_old / p_ap;
        fxo_axpy(alpha, p, x, n);
        fxo_copy(r, rp, n);
        fxo_axpy(-alpha, ap, r, n);
        fxo_fill(z, n, 0.0);
        pc(pc_ctx, z, r);
        double rz_new, zr_prev;
        fxo_dot2(r, z, rp, z, n, &rz_new, &zr_prev);
        double beta = (rz_new - zr_prev) / rz_old;
        fxo_scale(p, n, beta);
        fxo_axpy(1.0, z, p, n);
        rz_old = rz_new;
    }
    set_stats(st, max_iter, sqrt(fxo_dot(r, r, n)), 1);
out:
    free(r); free(rp); free(z); free(p); free(ap);
    return rc;
}

/* Flexible GMRES(m) (Saad 1993): right preconditioning with the preconditioned directions
 * z_k = M_k^-1 v_k kept, so M may change from one application to the next; the Arnoldi
 * relation is A Z_k = V_{k+1} H, the Givens residual estimate is the true ||b - A x||, and
 * x += Z y at the end of a cycle.  Gram-Schmidt, Givens rotations, breakdown thresholds and
 * restarts as fxo_gmres_solve. */
int fxo_fgmres_solve(const fxo_op *op, double *x, const double *b, size_t m, double tol,
                     size_t max_iter, fxo_pc_fn pc, void *pc_ctx, fxo_stats *st) {
    size_t n = op_len(op), mp1 = m + 1;
    double **vv = malloc(mp1 * sizeof(double *)), **zz = malloc(m * sizeof(double *));
    for (size_t i = 0; i < mp1; i++) vv[i] = calloc(n, 8);
    for (size_t i = 0; i < m; i++) zz[i] = calloc(n, 8);
    double *w = calloc(n, 8), *hh = calloc(mp1 * m, 8), *cc = calloc(m, 8), *ss = calloc(m, 8);
    double *grs = calloc(mp1, 8);
    size_t total_its = 0;
    int rc = 0;
#define H(i, j) hh[(j) * mp1 + (i)]
    for (;;) {
        double *v0 = vv[0];
        rc = apply_op(op, v0, x);
        if (rc) goto out;
        fxo_scale(v0, n, -1.0);
        fxo_axpy(1.0, b, v0, n);
        double beta = sqrt(fxo_dot(v0, v0, n));
        if (beta < tol) {
            set_stats(st, total_its, beta, 0);
            goto out;
        }
        fxo_scale(v0, n, 1.0 / beta);
        memset(grs, 0, mp1 * 8);
        grs[0] = beta;
        memset(hh, 0, mp1 * m * 8);
        double cur_resid = beta;
        size_t k = 0;
        while (k < m) {
            if (total_its >= max_iter) {
                gmres_build_solution(x, zz, hh, grs, m, k, n);
                set_stats(st, total_its, cur_resid, 1);
                goto out;
            }
            fxo_fill(zz[k], n, 0.0);
            if (pc) pc(pc_ctx, zz[k], vv[k]);
            else fxo_copy(vv[k], zz[k], n);
            apply_op(op, w, zz[k]);
            for (size_t j = 0; j <= k; j++) {
                double h = fxo_dot(w, vv[j], n);
                H(j, k) = h;
                fxo_axpy(-h, vv[j], w, n);
            }
            double h_kp1_k = sqrt(fxo_dot(w, w, n));
            H(k + 1, k) = h_kp1_k;
            if (h_kp1_k > 1e-30) {
                fxo_copy(w, vv[k + 1], n);
                fxo_scale(vv[k + 1], n, 1.0 / h_kp1_k);
            }
            for (size_t j = 0; j < k; j++) {
                double h_j = H(j, k), h_jp1 = H(j + 1, k);
                double cj = cc[j], sj = ss[j];
                H(j, k) = fma(cj, h_j, sj * h_jp1);
                H(j + 1, k) = fma(cj, h_jp1, -sj * h_j);
            }
            double a = H(k, k), bv = H(k + 1, k);
            double rr = hypot(a, bv);
            if (fabs(rr) < 1e-30) {
                gmres_build_solution(x, zz, hh, grs, m, k, n);
                set_stats(st, total_its, cur_resid, 2);
                goto out;
            }
            cc[k] = a / rr;
            ss[k] = bv / rr;
            H(k, k) = rr;
            H(k + 1, k) = 0.0;
            double g_k = grs[k];
            grs[k] = cc[k] * g_k;
            grs[k + 1] = -ss[k] * g_k;
            cur_resid = fabs(grs[k + 1]);
            total_its++;
            k++;
            if (cur_resid < tol) break;
            if (h_kp1_k <= 1e-30) break;
        }
        gmres_build_solution(x, zz, hh, grs, m, k, n);
        if (cur_resid < tol) {
            set_stats(st, total_its, cur_resid, 0);
            goto out;
        }
        if (total_its >= max_iter) {
            set_stats(st, total_its, cur_resid, 1);
            goto out;
        }
    }
#undef H
out:
    for (size_t i = 0; i < mp1; i++) free(vv[i]);
    for (size_t i = 0; i < m; i++) free(zz[i]);
    free(vv); free(zz); free(w); free(hh); free(cc); free(ss); free(grs);
    return rc;
}

/* A preconditioner that is itself a number of (optionally preconditioned) CG steps on A z = r
 * from z = 0 (tolerance 0: the count alone ends it, or a breakdown), the count of the k-th
 * application being steps[k mod nsteps].  Its action depends on r nonlinearly, and with
 * different counts it changes between applications: the test case for the flexible solvers. */
void fxo_inner_cg_pc_apply(void *ctx, double *z, const double *r) {
    fxo_inner_cg *ic = (fxo_inner_cg *)ctx;
    fxo_stats st;
    const size_t k = ic->steps[ic->calls++ % ic->nsteps];
    fxo_cg_solve(ic->op, z, r, 0.0, k, ic->pc, ic->pc_ctx, &st);
}

/* ------------------------------------------------------------------ */
/* Multigrid for the conv-diff operator (new)                          */
/* ------------------------------------------------------------------ */
/* Vertex hierarchy as fxo_mg mode 1 (rows-1 halves while both interiors exceed coarse_max).
 * Each coarse level rediscretises the operator with h doubled and kappa / vx / vy injected
 * from the coincident fine points.  Smoother: x <- x + omega (b - A x) (1 / diag(A)) inside, the
 * ring left at 0; full weighting down, bilinear up; `coarse_sweeps` sweeps on the coarsest
 * level; every cycle from x = 0. */

struct fxo_cdmg {
    int nlev, n_pre, n_post, coarse_sweeps;
    double omega;
    fxo_op op[40];
    double *vx[40], *vy[40], *kappa[40], *u[40], *rhs[40], *tmp[40];
};

static double cd_diag(const fxo_op *op, size_t idx, double inv_dx, double inv_dy, double k2) {
    double kap = op->kappa ? op->kappa[idx] : op->kappa_s;
    return fma(op->coeff, fma(-kap, k2, fma(fabs(op->vx[idx]), inv_dx, fabs(op->vy[idx]) * inv_dy)), op->sigma);
}

/* out = x + omega (b - A x) (1 / diag) inside (out's ring untouched): one division per point,
 * as the GPU sweeps do */
static void cd_sweep(const fxo_op *op, const double *x, double *out, const double *b, double omega) {
    size_t rows = op->rows, cols = op->cols;
    double inv_dx = 1.0 / op->dx, inv_dy = 1.0 / op->dy;
    double inv_dx2 = inv_dx * inv_dx, inv_dy2 = inv_dy * inv_dy, k2 = 2.0 * (inv_dx2 + inv_dy2);
#pragma omp parallel for schedule(static)
    for (size_t row = 1; row < rows - 1; row++)
        for (size_t col = 1; col < cols - 1; col++) {
            size_t idx = row * cols + col;
            double kap = op->kappa ? op->kappa[idx] : op->kappa_s;
            double v = conv_diff_at_k(x, kap, op->vx, op->vy, idx, cols, inv_dx, inv_dy, inv_dx2, inv_dy2);
            double ax = fma(op->coeff, v, op->sigma * x[idx]);
            double inv_d = 1.0 / cd_diag(op, idx, inv_dx, inv_dy, k2);
            out[idx] = fma(omega, (b[idx] - ax) * inv_d, x[idx]);
        }
}

static void cd_resid(const fxo_op *op, const double *x, const double *b, double *r) {
    size_t rows = op->rows, cols = op->cols;
    double inv_dx = 1.0 / op->dx, inv_dy = 1.0 / op->dy;
    double inv_dx2 = inv_dx * inv_dx, inv_dy2 = inv_dy * inv_dy;
#pragma omp parallel for schedule(static)
    for (size_t row = 1; row < rows - 1; row++)
        for (size_t col = 1; col < cols - 1; col++) {
            size_t idx = row * cols + col;
            double kap = op->kappa ? op->kappa[idx] : op->kappa_s;
            double v = conv_diff_at_k(x, kap, op->vx, op->vy, idx, cols, inv_dx, inv_dy, inv_dx2, inv_dy2);
            r[idx] = b[idx] - fma(op->coeff, v, op->sigma * x[idx]);
        }
}

static double *inject(const double *f, size_t fcols, size_t crows, size_t ccols) {
    double *c = malloc(crows * ccols * 8);
    for (size_t I = 0; I < crows; I++)
        for (size_t J = 0; J < ccols; J++) c[I * ccols + J] = f[(2 * I) * fcols + 2 * J];
    return c;
}

fxo_cdmg *fxo_cdmg_create(const fxo_op *op, int n_pre, int n_post, double omega, int coarse_max,
                          int coarse_sweeps) {
    if (!op->cd) return NULL;
    fxo_cdmg *mg = calloc(1, sizeof(fxo_cdmg));
    mg->n_pre = n_pre;
    mg->n_post = n_post;
    mg->omega = omega;
    mg->coarse_sweeps = coarse_sweeps;
    size_t r = op->rows, c = op->cols;
    for (int l = 0; l < 40; l++) {
        fxo_op *L = &mg->op[l];
        if (l == 0) {
            *L = *op;
        } else {
            const fxo_op *F = &mg->op[l - 1];
            *L = *F;
            L->rows = r;
            L->cols = c;
            L->dx = F->dx * 2.0;
            L->dy = F->dy * 2.0;
            mg->vx[l] = inject(F->vx, F->cols, r, c);
            mg->vy[l] = inject(F->vy, F->cols, r, c);
            L->vx = mg->vx[l];
            L->vy = mg->vy[l];
            if (F->kappa) {
                mg->kappa[l] = inject(F->kappa, F->cols, r, c);
                L->kappa = mg->kappa[l];
            }
        }
        mg->u[l] = calloc(r * c, 8);
        mg->rhs[l] = calloc(r * c, 8);
        mg->tmp[l] = calloc(r * c, 8);
        mg->nlev = l + 1;
        if (!(r - 2 > (size_t)coarse_max && c - 2 > (size_t)coarse_max && (r - 1) % 2 == 0 && (c - 1) % 2 == 0))
            break;
        r = (r - 1) / 2 + 1;
        c = (c - 1) / 2 + 1;
    }
    return mg;
}

void fxo_cdmg_destroy(fxo_cdmg *mg) {
    if (!mg) return;
    for (int l = 0; l < mg->nlev; l++) {
        free(mg->vx[l]); free(mg->vy[l]); free(mg->kappa[l]);
        free(mg->u[l]); free(mg->rhs[l]); free(mg->tmp[l]);
    }
    free(mg);
}

int fxo_cdmg_depth(const fxo_cdmg *mg) { return mg->nlev; }

/* z = V-cycle(r) from z = 0 (usable as fxo_pc_fn with ctx = the fxo_cdmg) */
void fxo_cdmg_pc_apply(void *ctx, double *z, const double *r) {
    fxo_cdmg *mg = (fxo_cdmg *)ctx;
    int nl = mg->nlev;
    size_t n0 = mg->op[0].rows * mg->op[0].cols;
    double *cur[40], *oth[40];
    const double *rhs[40];
    cur[0] = mg->u[0];
    oth[0] = mg->tmp[0];
    rhs[0] = r;
    memset(cur[0], 0, n0 * 8);
    memset(oth[0], 0, n0 * 8);
    for (int l = 1; l < nl; l++) {
        cur[l] = mg->u[l];
        oth[l] = mg->tmp[l];
        rhs[l] = mg->rhs[l];
    }
    for (int l = 0; l < nl - 1; l++) {
        const fxo_op *L = &mg->op[l], *Cc = &mg->op[l + 1];
        for (int k = 0; k < mg->n_pre; k++) {
            cd_sweep(L, cur[l], oth[l], rhs[l], mg->omega);
            double *t = cur[l]; cur[l] = oth[l]; oth[l] = t;
        }
        cd_resid(L, cur[l], rhs[l], oth[l]);
        fxo_restrict_fw(oth[l], mg->rhs[l + 1], L->rows, L->cols, Cc->rows, Cc->cols);
        memset(cur[l + 1], 0, Cc->rows * Cc->cols * 8);
        memset(oth[l + 1], 0, Cc->rows * Cc->cols * 8);
    }
    {
        const fxo_op *L = &mg->op[nl - 1];
        for (int k = 0; k < mg->coarse_sweeps; k++) {
            cd_sweep(L, cur[nl - 1], oth[nl - 1], rhs[nl - 1], mg->omega);
            double *t = cur[nl - 1]; cur[nl - 1] = oth[nl - 1]; oth[nl - 1] = t;
        }
    }
    for (int l = nl - 2; l >= 0; l--) {
        const fxo_op *L = &mg->op[l], *Cc = &mg->op[l + 1];
        fxo_prolong_bilinear(cur[l + 1], cur[l], Cc->rows, Cc->cols, L->rows, L->cols);
        for (int k = 0; k < mg->n_post; k++) {
            cd_sweep(L, cur[l], oth[l], rhs[l], mg->omega);
            double *t = cur[l]; cur[l] = oth[l]; oth[l] = t;
        }
    }
    memcpy(z, cur[0], n0 * 8);
}

/* ------------------------------------------------------------------ */
/* Multigrid (multigrid.rs)                                            */
/* ------------------------------------------------------------------ */

typedef struct {
    size_t rows, cols;
    double dx, dy;
    double a5[5];       /* vertex mode: operator on this level */
    double lap5[5];     /* reference mode: Laplacian (stencil.rs:152-168) c,n,s,w,e */
    double *u, *rhs, *tmp;
    double *w0, *w1; /* reference mode, Chebyshev smoother: recurrence work vectors */
} mg_level;

struct fxo_mg {
    int mode, n_pre, n_post, coarse_sweeps, nlev;
    int smoother; /* reference mode: 0 weighted Jacobi, 1 Chebyshev (multigrid.rs:11-20) */
    double omega;
    fxo_bc bcs[4];
    mg_level lv[40];
};

int fxo_mg_depth(const fxo_mg *mg) { return mg->nlev; }
void fxo_mg_level_dims(const fxo_mg *mg, int l, size_t *rows, size_t *cols) {
    *rows = mg->lv[l].rows;
    *cols = mg->lv[l].cols;
}

static void lap5_of(double dx, double dy, double *a) { /* stencil.rs:152-168 */
    double inv_dx2 = 1.0 / (dx * dx), inv_dy2 = 1.0 / (dy * dy);
    a[0] = -2.0 * (inv_dx2 + inv_dy2);
    a[1] = inv_dy2;
    a[2] = inv_dy2;
    a[3] = inv_dx2;
    a[4] = inv_dx2;
}

/* Coarse-level operator for the vertex hierarchy: off-diagonal (diffusion)
 * weights scale by 1/4 when h doubles; the reaction part sigma = sum of all
 * weights is kept.  Same arithmetic as the CUDA library's host code. */
void fxo_mg_coarse_op(const double *fine, double sigma, double *coarse) {
    coarse[1] = fine[1] * 0.25;
    coarse[2] = fine[2] * 0.25;
    coarse[3] = fine[3] * 0.25;
    coarse[4] = fine[4] * 0.25;
    coarse[0] = sigma - ((coarse[1] + coarse[2]) + (coarse[3] + coarse[4]));
}

fxo_mg *fxo_mg_create(size_t rows, size_t cols, double dx, double dy, const fxo_bc *bcs,
                      int n_pre, int n_post, double omega, int mode, double op_coeff, int ne,
                      const int *dr, const int *dc, const double *w, int coarse_max,
                      int coarse_sweeps) {
    fxo_mg *mg = calloc(1, sizeof(fxo_mg));
    mg->mode = mode;
    mg->n_pre = n_pre;
    mg->n_post = n_post;
    mg->omega = omega;
    mg->coarse_sweeps = coarse_sweeps;
    memcpy(mg->bcs, bcs, 4 * sizeof(fxo_bc));
    size_t r = rows, c = cols;
    double hx = dx, hy = dy;
    double a5[5] = {0, 0, 0, 0, 0}, sigma = 0.0;
    if (mode == 1) {
        stencil_w sw;
        if (ne != 5 || stencil_setup(&sw, ne, dr, dc, w) != FXO_OK) {
            free(mg);
            return NULL;
        }
        a5[0] = 1.0 + op_coeff * sw.c;
        a5[1] = op_coeff * sw.n;
        a5[2] = op_coeff * sw.s;
        a5[3] = op_coeff * sw.w;
        a5[4] = op_coeff * sw.e;
        sigma = a5[0] + ((a5[1] + a5[2]) + (a5[3] + a5[4]));
    }
    for (int l = 0; l < 40; l++) {
        mg_level *L = &mg->lv[l];
        L->rows = r;
        L->cols = c;
        L->dx = hx;
        L->dy = hy;
        lap5_of(hx, hy, L->lap5);
        if (mode == 1) {
            if (l == 0) memcpy(L->a5, a5, sizeof(a5));
            else fxo_mg_coarse_op(mg->lv[l - 1].a5, sigma, L->a5);
        }
        L->u = calloc(r * c, 8);
        L->rhs = calloc(r * c, 8);
        L->tmp = calloc(r * c, 8);
        mg->nlev = l + 1;
        if (mode == 0) { /* multigrid.rs:121-135 */
            if (r <= 4 || c <= 4) break;
            size_t cr = r / 2, cc2 = c / 2;
            if (cr < 3 || cc2 < 3) break;
            r = cr;
            c = cc2;
        } else {
            if (!(r - 2 > (size_t)coarse_max && c - 2 > (size_t)coarse_max && (r - 1) % 2 == 0 &&
                  (c - 1) % 2 == 0))
                break;
            r = (r - 1) / 2 + 1;
            c = (c - 1) / 2 + 1;
        }
        hx *= 2.0;
        hy *= 2.0;
    }
    return mg;
}

void fxo_mg_destroy(fxo_mg *mg) {
    if (!mg) return;
    for (int l = 0; l < mg->nlev; l++) {
        free(mg->lv[l].u);
        free(mg->lv[l].rhs);
        free(mg->lv[l].tmp);
        free(mg->lv[l].w0);
        free(mg->lv[l].w1);
    }
    free(mg);
}

int fxo_mg_set_smoother(fxo_mg *mg, int smoother) {
    if (mg->mode != 0 || smoother < 0 || smoother > 1) return FXO_ERR_INVALID_ARGUMENT;
    mg->smoother = smoother;
    if (smoother == 1)
        for (int l = 0; l < mg->nlev; l++) {
            size_t n = mg->lv[l].rows * mg->lv[l].cols;
            if (!mg->lv[l].w0) mg->lv[l].w0 = calloc(n, 8);
            if (!mg->lv[l].w1) mg->lv[l].w1 = calloc(n, 8);
        }
    return FXO_OK;
}

static const int LAP_DR[5] = {0, -1, 1, 0, 0}, LAP_DC[5] = {0, 0, 0, -1, 1};

/* Reference-mode Chebyshev smoother (multigrid.rs:308-473): first-kind Chebyshev recurrence for
 * D^-1 A with the bounds emax = 2, emin = 0.2, D the Laplacian's diagonal, on three rotating
 * vectors (u, w0, w1), each step built from the backend ops in the reference's order. */
static void ref_smooth_cheby(fxo_mg *mg, int l, int n) {
    if (n == 0) return;
    mg_level *L = &mg->lv[l];
    size_t len = L->rows * L->cols;
    double emax = 2.0, emin = 0.1 * emax;
    double scale = 2.0 / (emax + emin);
    double alpha = 1.0 - scale * emin;
    double mu = 1.0 / alpha, omegaprod = 2.0 / alpha;
    double inv_dx2 = 1.0 / (L->dx * L->dx), inv_dy2 = 1.0 / (L->dy * L->dy);
    double inv_diag = -1.0 / (2.0 * inv_dx2 + 2.0 * inv_dy2);
    double c_km1 = 1.0, c_k = mu;
    fxo_apply_stencil(L->u, L->tmp, L->rows, L->cols, L->dx, L->dy, 5, LAP_DR, LAP_DC, L->lap5, mg->bcs);
    fxo_copy(L->rhs, L->w0, len);
    fxo_axpy(-1.0, L->tmp, L->w0, len);
    fxo_scale(L->w0, len, scale * inv_diag);
    fxo_axpy(1.0, L->u, L->w0, len);
    fxo_zero_boundaries(L->w0, L->rows, L->cols);
    if (n == 1) {
        fxo_copy(L->w0, L->u, len);
        return;
    }
    double *buf[3] = {L->u, L->w0, L->w1};
    int km1 = 0, k = 1, kp1 = 2;
    for (int i = 1; i < n; i++) {
        fxo_apply_stencil(buf[k], L->tmp, L->rows, L->cols, L->dx, L->dy, 5, LAP_DR, LAP_DC, L->lap5, mg->bcs);
        fxo_copy(L->rhs, buf[kp1], len);
        fxo_axpy(-1.0, L->tmp, buf[kp1], len);
        fxo_scale(buf[kp1], len, inv_diag);
        double c_kp1 = 2.0 * mu * c_k - c_km1;
        double omega = omegaprod * c_k / c_kp1;
        fxo_scale(buf[kp1], len, omega * scale);
        fxo_axpy(omega, buf[k], buf[kp1], len);
        fxo_axpy(1.0 - omega, buf[km1], buf[kp1], len);
        fxo_zero_boundaries(buf[kp1], L->rows, L->cols);
        c_km1 = c_k;
        c_k = c_kp1;
        int t = km1;
        km1 = k;
        k = kp1;
        kp1 = t;
    }
    if (k == 1) fxo_copy(L->w0, L->u, len);
    else if (k == 2) fxo_copy(L->w1, L->u, len);
}

/* Reference-mode smoother: n lexicographic sweeps (multigrid.rs:245-306). */
static void ref_smooth(fxo_mg *mg, int l, int n) {
    mg_level *L = &mg->lv[l];
    if (mg->smoother == 1) {
        ref_smooth_cheby(mg, l, n);
        return;
    }
    for (int k = 0; k < n; k++)
        fxo_weighted_jacobi(L->u, L->rhs, mg->omega, L->rows, L->cols, 5, LAP_DR, LAP_DC, L->lap5);
}

/* Vertex-mode smoother: n true Jacobi sweeps, ping-ponging u <-> tmp. */
static void vtx_smooth(fxo_mg *mg, int l, int n) {
    mg_level *L = &mg->lv[l];
    size_t len = L->rows * L->cols;
    for (int k = 0; k < n; k++) {
        fxo_jacobi_sweep(L->u, L->tmp, L->rhs, mg->omega, L->rows, L->cols, L->a5);
        double *t = L->u;
        L->u = L->tmp;
        L->tmp = t;
    }
    (void)len;
}

void fxo_mg_v_cycle(fxo_mg *mg, double *x, const double *b) {
    int nl = mg->nlev;
    mg_level *L0 = &mg->lv[0];
    size_t n0 = L0->rows * L0->cols;
    if (mg->mode == 0) { /* multigrid.rs:188-230 */
        fxo_copy(b, L0->rhs, n0);
        fxo_copy(x, L0->u, n0);
        for (int l = 0; l < nl - 1; l++) {
            mg_level *L = &mg->lv[l], *C = &mg->lv[l + 1];
            ref_smooth(mg, l, mg->n_pre);
            /* compute_residual, multigrid.rs:476-491 */
            fxo_apply_stencil(L->u, L->tmp, L->rows, L->cols, L->dx, L->dy, 5, LAP_DR, LAP_DC,
                              L->lap5, mg->bcs);
            fxo_scale(L->tmp, L->rows * L->cols, -1.0);
            fxo_axpy(1.0, L->rhs, L->tmp, L->rows * L->cols);
            fxo_restrict(L->tmp, C->rhs, L->rows, L->cols, C->rows, C->cols);
            fxo_fill(C->u, C->rows * C->cols, 0.0);
        }
        ref_smooth(mg, nl - 1, mg->n_pre + mg->n_post + 10);
        for (int l = nl - 2; l >= 0; l--) {
            mg_level *L = &mg->lv[l], *C = &mg->lv[l + 1];
            fxo_prolong(C->u, L->u, C->rows, C->cols, L->rows, L->cols);
            ref_smooth(mg, l, mg->n_post);
        }
        fxo_copy(L0->u, x, n0);
        return;
    }
    /* vertex mode: level-0 rhs = b, u = x (ring treated as homogeneous Dirichlet) */
    fxo_copy(b, L0->rhs, n0);
    fxo_copy(x, L0->u, n0);
    fxo_zero_boundaries(L0->u, L0->rows, L0->cols);
    fxo_zero_boundaries(L0->tmp, L0->rows, L0->cols);
    for (int l = 0; l < nl - 1; l++) {
        mg_level *L = &mg->lv[l], *C = &mg->lv[l + 1];
        vtx_smooth(mg, l, mg->n_pre);
        fxo_residual(L->u, L->rhs, L->tmp, L->rows, L->cols, L->a5);
        fxo_restrict_fw(L->tmp, C->rhs, L->rows, L->cols, C->rows, C->cols);
        fxo_fill(C->u, C->rows * C->cols, 0.0);
        fxo_fill(C->tmp, C->rows * C->cols, 0.0);
    }
    vtx_smooth(mg, nl - 1, nl == 1 ? mg->coarse_sweeps : mg->coarse_sweeps);
    for (int l = nl - 2; l >= 0; l--) {
        mg_level *L = &mg->lv[l], *C = &mg->lv[l + 1];
        fxo_prolong_bilinear(C->u, L->u, C->rows, C->cols, L->rows, L->cols);
        vtx_smooth(mg, l, mg->n_post);
    }
    fxo_copy(L0->u, x, n0);
}

void fxo_mg_pc_apply(void *ctx, double *z, const double *r) {
    fxo_mg_v_cycle((fxo_mg *)ctx, z, r);
}

/* ------------------------------------------------------------------ */
/* FP32 vertex cycle: the cycle above evaluated in single precision, as the CUDA library runs a
 * vertex multigrid created with dtype F32 on FP64 vectors.  Per level the operator weights are
 * the FP64 weights rounded to float and the Jacobi factor is (float)(omega / a_c); every sweep,
 * residual, restriction and prolongation is the FP64 expression above in float arithmetic
 * (explicit fmaf where the FP64 code has fma, no other contraction).  The FP64 rhs is rounded to
 * float on entry, the cycle starts from zero, and z is the float result widened to FP64.      */
/* ------------------------------------------------------------------ */

static inline float op5f(const float *a5, const float *x, size_t i, size_t cols) {
    return fmaf(a5[0], x[i],
                fmaf(a5[1], x[i - cols], fmaf(a5[2], x[i + cols], fmaf(a5[3], x[i - 1], a5[4] * x[i + 1]))));
}

static void jacobi_f(const float *x_in, float *x_out, const float *b, float wd, size_t rows, size_t cols,
                     const float *a5) {
#pragma omp parallel for schedule(static)
    for (size_t row = 1; row < rows - 1; row++)
        for (size_t col = 1; col < cols - 1; col++) {
            size_t i = row * cols + col;
            float r = b[i] - op5f(a5, x_in, i, cols);
            x_out[i] = fmaf(wd, r, x_in[i]);
        }
}

static void residual_f(const float *x, const float *b, float *r, size_t rows, size_t cols, const float *a5) {
#pragma omp parallel for schedule(static)
    for (size_t row = 1; row < rows - 1; row++)
        for (size_t col = 1; col < cols - 1; col++) {
            size_t i = row * cols + col;
            r[i] = b[i] - op5f(a5, x, i, cols);
        }
}

static void restrict_fw_f(const float *f, float *c, size_t frows, size_t fcols, size_t crows, size_t ccols) {
    (void)frows;
    memset(c, 0, crows * ccols * sizeof(float));
#pragma omp parallel for schedule(static)
    for (size_t I = 1; I < crows - 1; I++)
        for (size_t J = 1; J < ccols - 1; J++) {
            size_t i = (2 * I) * fcols + 2 * J, fc = fcols;
            float e = (f[i - fc] + f[i + fc]) + (f[i - 1] + f[i + 1]);
            float d = (f[i - fc - 1] + f[i - fc + 1]) + (f[i + fc - 1] + f[i + fc + 1]);
            c[I * ccols + J] = (4.0f * f[i] + (2.0f * e + d)) * 0.0625f;
        }
}

static void prolong_bilinear_f(const float *c, float *fine, size_t ccols, size_t frows, size_t fcols) {
#pragma omp parallel for schedule(static)
    for (size_t i = 1; i < frows - 1; i++)
        for (size_t j = 1; j < fcols - 1; j++) {
            size_t I = i / 2, J = j / 2, k = I * ccols + J;
            float e;
            if (!(i & 1) && !(j & 1)) e = c[k];
            else if ((i & 1) && !(j & 1)) e = 0.5f * (c[k] + c[k + ccols]);
            else if (!(i & 1) && (j & 1)) e = 0.5f * (c[k] + c[k + 1]);
            else e = 0.25f * ((c[k] + c[k + ccols]) + (c[k + 1] + c[k + ccols + 1]));
            fine[i * fcols + j] += e;
        }
}

int fxo_mg_v_cycle_f32(fxo_mg *mg, double *z, const double *r) {
    if (mg->mode != 1) return FXO_ERR_INVALID_ARGUMENT;
    int nl = mg->nlev;
    float *u[40], *t[40], *b[40], a5[40][5], wd[40];
    for (int l = 0; l < nl; l++) {
        size_t n = mg->lv[l].rows * mg->lv[l].cols;
        u[l] = calloc(n, sizeof(float));
        t[l] = calloc(n, sizeof(float));
        b[l] = calloc(n, sizeof(float));
        for (int k = 0; k < 5; k++) a5[l][k] = (float)mg->lv[l].a5[k];
        wd[l] = (float)(mg->omega / mg->lv[l].a5[0]);
    }
    size_t n0 = mg->lv[0].rows * mg->lv[0].cols;
    for (size_t i = 0; i < n0; i++) b[0][i] = (float)r[i];
#define FXO_SMOOTH(l, cnt)                                                                            \
    for (int k_ = 0; k_ < (cnt); k_++) {                                                              \
        jacobi_f(u[l], t[l], b[l], wd[l], mg->lv[l].rows, mg->lv[l].cols, a5[l]);                    \
        float *s_ = u[l];                                                                             \
        u[l] = t[l];                                                                                  \
        t[l] = s_;                                                                                    \
    }
    for (int l = 0; l < nl - 1; l++) {
        mg_level *L = &mg->lv[l], *Cl = &mg->lv[l + 1];
        FXO_SMOOTH(l, mg->n_pre);
        residual_f(u[l], b[l], t[l], L->rows, L->cols, a5[l]);
        restrict_fw_f(t[l], b[l + 1], L->rows, L->cols, Cl->rows, Cl->cols);
    }
    FXO_SMOOTH(nl - 1, mg->coarse_sweeps);
    for (int l = nl - 2; l >= 0; l--) {
        mg_level *L = &mg->lv[l], *Cl = &mg->lv[l + 1];
        prolong_bilinear_f(u[l + 1], u[l], Cl->cols, L->rows, L->cols);
        FXO_SMOOTH(l, mg->n_post);
    }
#undef FXO_SMOOTH
    for (size_t i = 0; i < n0; i++) z[i] = (double)u[0][i];
    for (int l = 0; l < nl; l++) {
        free(u[l]);
        free(t[l]);
        free(b[l]);
    }
    return FXO_OK;
}

void fxo_mg_pc_apply_f32(void *ctx, double *z, const double *r) { fxo_mg_v_cycle_f32((fxo_mg *)ctx, z, r); }
