// fx_solvers.cu -- preconditioners, multigrid and the Krylov solver loops.
//
// The solver loops restate crates/runtime/src/{cg,pipelined_cg,bicgstab,gmres}.rs with
// the same scalar recurrences, stop tests and iteration counts, but the vector work is
// fused: each kernel applies the operator on the fly, updates several vectors and emits
// the next inner products in the same pass.  The scalars (alpha, beta, rho, omega, ...)
// live in device memory and are updated by the last block of each reduction, so an
// iteration needs no host round trip; the host enqueues iterations in batches and a
// `done` word in device memory turns the surplus launches into no-ops once the stop
// test (evaluated on the device, exactly as the reference evaluates it) has fired.
#include <cmath>
#include <random>
#include <type_traits>
#include <utility>
#include <vector>

#include "fx_learned.cuh"
#include "fx_points.cuh"
#include "fx_wcycle.cuh"

using namespace fx;

FX_CHECK_FILE(solvers);

// ---------------------------------------------------------------- device solver state

namespace fx {

struct DevState {
    double tol;
    long long max_iter;
    long long iter;
    int done;     // solve finished: every later kernel is a no-op
    int halt;     // done, or a pending early exit (BiCGSTAB): kernels that must skip read this
    int reason;
    int pending;  // BiCGSTAB: 1 = converged on s, 2 = breakdown on t.t (x += alpha*p still due)
    double resid, r0;
    // CG / PCG
    double rs_old, alpha, beta, rr;
    // pipelined CG
    double gamma, delta, gamma_prev, alpha_prev;
    // BiCGSTAB
    double rho, rho_new, omega, r_norm, s_norm;
};

__device__ __forceinline__ void st_finish(DevState *S, int reason, long long iters, double resid) {
    S->done = 1;
    S->halt = 1;
    S->reason = reason;
    S->iter = iters;
    S->resid = resid;
}

// PCG inner product r.z -> beta (cg.rs:202-212 at the start, :240-247 per iteration)
struct FinPcgRzInit {  // rz_old = r.z, beta = 0, loop-top test of iteration 0 (cg.rs:202-212)
    DevState *S;
    __device__ void operator()(const double *v) const {
        S->rs_old = v[0];
        S->beta = 0.0;
        S->iter = 0;
        S->r0 = S->resid;
        if (S->max_iter == 0) st_finish(S, FX_MAX_ITERATIONS, 0, S->resid);
        else if (S->resid < S->tol) st_finish(S, FX_CONVERGED, 0, S->resid);
    }
};

struct FinPcgRz {  // beta = rz_new / rz_old (cg.rs:240-247)
    DevState *S;
    __device__ void operator()(const double *v) const {
        S->beta = v[0] / S->rs_old;
        S->rs_old = v[0];
    }
};

}  // namespace fx

// ---------------------------------------------------------------- operators

// A conv-diff operator for the solvers' *_solve_op entry points (fx_op_conv_diff).  The field
// buffers are borrowed: they must outlive the fx_op.
struct fx_op {
    fx_ctx *ctx = nullptr;
    fx_grid g{};
    double sigma = 1.0, coeff = 1.0, kappa_s = 0.0;
    const fx_buf *kappa = nullptr, *vx = nullptr, *vy = nullptr;
};

// ---------------------------------------------------------------- preconditioners

struct fx_precond {
    fx_ctx *ctx = nullptr;
    bool borrowed = false;
    virtual ~fx_precond() {}
    // z <- M^-1 r.  z_zero: z holds zeros on entry (the solvers zero-fill z first, as the
    // reference does); skip: device word, nonzero means the solve is over.
    virtual int apply(fx_buf *z, const fx_buf *r, const int *skip, bool z_zero) = 0;
    // z <- M^-1 r from a zero z, followed by rz = r.z handed to the PCG state S (first = the
    // initial product).  Returns FX_ERR_UNSUPPORTED when the preconditioner has no fused form.
    virtual int apply_pcg(fx_buf *, const fx_buf *, const int *, DevState *, bool) { return FX_ERR_UNSUPPORTED; }
    // true when apply(z, r, skip, true) writes every interior point of z from r alone and leaves
    // z's ring as it is, so a z whose ring is zero needs no zero-fill before each application
    virtual bool fills_from_zero(const fx_buf *) const { return false; }
};

namespace {


// ---------------------------------------------------------------- operator A v = v + coeff*S v

template <typename T, int MODE>
struct OpA {
    StencilP P;
    T coeff;
    int rows, cols;
    // copy_from + stencil_axpy (cg.rs:106-109): interior fma(coeff, S v, v), ring = v
    __device__ __forceinline__ T apply(bool ring, const Nb<T> &nb, size_t) const {
        return ring ? nb.c : fx_fma(coeff, stencil_eval<T, MODE>(P, nb), nb.c);
    }
};

// The convection-diffusion operator of an fx_op (new; no reference solver takes it):
// interior fma(coeff, kappa Lap v + v.grad v, sigma v), upwind as apply_conv_diff
// (ops.rs:673-791, conv_diff_at), ring = v.  With sigma = 1 it is conv_diff_axpy(coeff, v, v),
// the implicit-step operator I + coeff CD; with sigma = 0 the steady operator CD.
constexpr int kModeCD = 100;

template <typename T>
struct OpA<T, kModeCD> {
    ConvDiffC<T> K;
    T sigma, coeff, kap_s;
    const T *kappa, *vx, *vy;  // kappa null: the scalar kap_s
    __device__ __forceinline__ T apply(bool ring, const Nb<T> &nb, size_t idx) const {
        if (ring) return nb.c;
        const T kap = kappa ? kappa[idx] : kap_s;
        return fx_fma(coeff, conv_diff_at<T>(K, nb, kap, vx[idx], vy[idx]), sigma * nb.c);
    }
};

// The operator a solver applies: the stencil form from (P, coeff), or the solver's fx_op.
template <typename T, int MODE>
struct OpMaker {
    static OpA<T, MODE> make(const StencilP &P, double coeff, size_t rows, size_t cols, const fx_op *) {
        return OpA<T, MODE>{P, (T)coeff, (int)rows, (int)cols};
    }
};
template <typename T>
struct OpMaker<T, kModeCD> {
    static OpA<T, kModeCD> make(const StencilP &, double, size_t, size_t, const fx_op *op) {
        OpA<T, kModeCD> A;
        A.K = conv_consts<T>(op->g.dx, op->g.dy);
        A.sigma = (T)op->sigma;
        A.coeff = (T)op->coeff;
        A.kap_s = (T)op->kappa_s;
        A.kappa = op->kappa ? (const T *)op->kappa->ptr : nullptr;
        A.vx = (const T *)op->vx->ptr;
        A.vy = (const T *)op->vy->ptr;
        return A;
    }
};

// A solver pass over the grid: the row march, or the one-point-per-thread form (k_point) when
// the pass applies the convection-diffusion operator, whose velocity and kappa loads the
// march does not prefetch.
template <typename P, typename = void>
struct applies_cd : std::false_type {};
template <typename P>
struct applies_cd<P, std::void_t<decltype(std::declval<P>().A)>>
    : std::bool_constant<std::is_same<std::decay_t<decltype(std::declval<P>().A)>, OpA<double, kModeCD>>::value ||
                         std::is_same<std::decay_t<decltype(std::declval<P>().A)>, OpA<float, kModeCD>>::value> {};

template <typename T, int K, typename Loader, typename Point, typename Fin>
int launch_pt(fx_ctx *ctx, size_t rows, size_t cols, Loader ld, Point pt, Fin fin, const int *skip,
              const char *what) {
    if constexpr (applies_cd<Point>::value)
        return launch_point<T, K>(ctx, rows, cols, ld, pt, fin, skip, what);
    else
        return launch_march<T, K>(ctx, rows, cols, ld, pt, fin, skip, what);
}

template <typename T>
struct Ld1 {
    static constexpr int NL = 1;
    const T *p;
    __device__ __forceinline__ void load(size_t i, T (&v)[1]) const { v[0] = p[i]; }
    __device__ __forceinline__ T combine(const T (&v)[1]) const { return v[0]; }
};

// r + beta*p, rounded as p.scale(beta); p.axpy(1.0, r) (cg.rs:153-154)
template <typename T>
struct LdAypx {
    static constexpr int NL = 2;
    const T *r, *p;
    const DevState *S;
    T beta;
    __device__ __forceinline__ void prepare() { beta = (T)S->beta; }
    __device__ __forceinline__ void load(size_t i, T (&v)[2]) const {
        v[0] = r[i];
        v[1] = p[i];
    }
    __device__ __forceinline__ T combine(const T (&v)[2]) const { return v[0] + v[1] * beta; }
};

// ------------------------------------------------ flat (pointwise) functors

template <typename T>
struct FlatCopy {
    T *dst;
    const T *src;
    __device__ __forceinline__ void operator()(size_t i, CSum *) const { dst[i] = src[i]; }
};

template <typename T>
struct FlatZero {
    T *p;
    __device__ __forceinline__ void operator()(size_t i, CSum *) const { p[i] = (T)0; }
};

template <typename S, typename D>
struct FlatConvert {
    const S *src;
    D *dst;
    __device__ __forceinline__ void operator()(size_t i, CSum *) const { dst[i] = (D)src[i]; }
};

template <typename T>
struct FlatDot {
    const T *a, *b;
    __device__ __forceinline__ void operator()(size_t i, CSum *acc) const {
        csum_add_prod(acc[0], (double)a[i], (double)b[i]);
    }
};

template <typename T>
struct FlatScaleInto {  // dst = src * f (copy_from + scale)
    T *dst;
    const T *src;
    T f;
    __device__ __forceinline__ void operator()(size_t i, CSum *) const { dst[i] = src[i] * f; }
};

template <typename T>
struct FlatRestrictFW {
    const T *f;
    T *c;
    size_t fcols, crows, ccols;
    __device__ __forceinline__ void operator()(size_t i, CSum *) const {
        const size_t I = i / ccols, J = i % ccols;
        if (I == 0 || J == 0 || I == crows - 1 || J == ccols - 1) {
            c[i] = (T)0;
            return;
        }
        const size_t k = (2 * I) * fcols + 2 * J;
        const T e = (f[k - fcols] + f[k + fcols]) + (f[k - 1] + f[k + 1]);
        const T d = (f[k - fcols - 1] + f[k - fcols + 1]) + (f[k + fcols - 1] + f[k + fcols + 1]);
        c[i] = ((T)4 * f[k] + ((T)2 * e + d)) * (T)0.0625;
    }
};

template <typename T>
struct FlatProlongBil {
    const T *c;
    T *f;
    size_t ccols, fcols, iw;
    __device__ __forceinline__ void operator()(size_t q, CSum *) const {
        const size_t i = 1 + q / iw, j = 1 + q % iw;
        const size_t k = (i / 2) * ccols + (j / 2);
        T e;
        if (!(i & 1) && !(j & 1)) e = c[k];
        else if ((i & 1) && !(j & 1)) e = (T)0.5 * (c[k] + c[k + ccols]);
        else if (!(i & 1) && (j & 1)) e = (T)0.5 * (c[k] + c[k + 1]);
        else e = (T)0.25 * ((c[k] + c[k + ccols]) + (c[k + 1] + c[k + ccols + 1]));
        f[i * fcols + j] += e;
    }
};

struct IdentityPc : fx_precond {
    int apply(fx_buf *z, const fx_buf *r, const int *skip, bool) override {
        FX_TRY(check_same(z, r));
        FX_DISPATCH(z->dtype, {
            return launch_flat<0>(ctx, z->len, FlatCopy<T>{(T *)z->ptr, (const T *)r->ptr}, NoFin{}, skip,
                                  "identity_pc");
        });
    }
};

// ------------------------------------------------ generic kernels used by several solvers

// out = A v (no reduction) or with <v, out> / <out, y> reductions.
template <typename T, int MODE>
struct PtApplyOp {
    static constexpr int NA = 0;
    OpA<T, MODE> A;
    T *out;
    __device__ __forceinline__ const T *aux(int) const { return nullptr; }
    __device__ __forceinline__ void operator()(bool ring, int r, int c, size_t idx, const Nb<T> &nb, const T *, CSum *) const {
        out[idx] = A.apply(ring, nb, idx);
    }
};

}  // namespace

// ================================================================ multigrid

namespace {

struct MgLevel {
    size_t rows = 0, cols = 0;
    double dx = 0, dy = 0;
    double a5[5] = {0, 0, 0, 0, 0};    // vertex: operator on this level
    double lap5[5] = {0, 0, 0, 0, 0};  // reference: Laplacian weights
    fx_buf *u = nullptr, *rhs = nullptr, *tmp = nullptr;
    fx_buf *w0 = nullptr, *w1 = nullptr;  // reference mode, Chebyshev smoother
};

}  // namespace

struct fx_mg {
    fx_ctx *ctx = nullptr;
    int mode = 0;  // 0 reference, 1 vertex
    int smoother = 0;  // reference mode: 0 weighted Jacobi, 1 Chebyshev (multigrid.rs:11-20)
    int dtype = FX_F64;
    size_t n_pre = 2, n_post = 2, coarse_sweeps = 200;
    double omega = 2.0 / 3.0;
    fx_boundaries bc{};
    std::vector<MgLevel> lv;
    fx_buf *tmp0 = nullptr;  // level-0 ping-pong partner (vertex mode)
    fx_buf *x32 = nullptr, *b32 = nullptr;  // level-0 single-precision copies (F32 cycle)
    // layout of the fused cycle (fx_mg_autotune): strip row chunks per launch in percent of one
    // wave, and the largest level the one-block tail takes (0: as many points as it can hold)
    int chunk_pct = 100;
    size_t tail_top_max = 0;
    struct View : fx_precond {
        fx_mg *mg = nullptr;
        int apply(fx_buf *z, const fx_buf *r, const int *skip, bool z_zero) override;
        int apply_pcg(fx_buf *z, const fx_buf *r, const int *skip, DevState *S, bool first) override;
        bool fills_from_zero(const fx_buf *z) const override;
    } view;
    ~fx_mg() {
        for (auto &L : lv) {
            fx_free(L.u);
            fx_free(L.rhs);
            fx_free(L.tmp);
            fx_free(L.w0);
            fx_free(L.w1);
        }
        fx_free(tmp0);
        fx_free(x32);
        fx_free(b32);
    }
};

namespace {

const int LAP_DR[5] = {0, -1, 1, 0, 0};
const int LAP_DC[5] = {0, 0, 0, -1, 1};

void lap5_of(double dx, double dy, double *a) {  // stencil.rs:152-168
    const double inv_dx2 = 1.0 / (dx * dx), inv_dy2 = 1.0 / (dy * dy);
    a[0] = -2.0 * (inv_dx2 + inv_dy2);
    a[1] = inv_dy2;
    a[2] = inv_dy2;
    a[3] = inv_dx2;
    a[4] = inv_dx2;
}

// Vertex hierarchy: off-diagonal (diffusion) weights scale by 1/4 when h doubles; the
// reaction part sigma (sum of all weights) is kept.
void coarse_op(const double *fine, double sigma, double *coarse) {
    coarse[1] = fine[1] * 0.25;
    coarse[2] = fine[2] * 0.25;
    coarse[3] = fine[3] * 0.25;
    coarse[4] = fine[4] * 0.25;
    coarse[0] = sigma - ((coarse[1] + coarse[2]) + (coarse[3] + coarse[4]));
}

// ---- vertex-cycle kernels (with skip support)

template <typename T>
int sweep(fx_ctx *ctx, const T *in, T *out, const T *b, const double *a5, double omega, size_t rows, size_t cols,
          const int *skip) {
    const size_t RR = rows, CC = cols;
    PtJacobi<T> pt{out, b, make_a5<T>(a5), (T)(omega / a5[0]), (int)RR, (int)CC};
    return launch_pt<T, 0>(ctx, RR, CC, LoadArr<T>{in}, pt, NoFin{}, skip, "mg_sweep");
}

template <typename T>
int residual(fx_ctx *ctx, const T *x, const T *b, T *r, const double *a5, size_t rows, size_t cols,
             const int *skip) {
    const size_t RR = rows, CC = cols;
    PtResidual<T> pt{r, b, make_a5<T>(a5), (int)RR, (int)CC};
    return launch_pt<T, 0>(ctx, RR, CC, LoadArr<T>{x}, pt, NoFin{}, skip, "mg_residual");
}

template <typename T>
int restrict_fw(fx_ctx *ctx, const T *f, T *c, size_t fcols, size_t crows, size_t ccols, const int *skip) {
    return launch_flat<0>(ctx, crows * ccols, FlatRestrictFW<T>{f, c, fcols, crows, ccols}, NoFin{}, skip,
                          "mg_restrict_fw");
}

template <typename T>
int prolong_bilinear(fx_ctx *ctx, const T *c, T *f, size_t ccols, size_t frows, size_t fcols, const int *skip) {
    return launch_flat<0>(ctx, (frows - 2) * (fcols - 2), FlatProlongBil<T>{c, f, ccols, fcols, fcols - 2}, NoFin{},
                          skip, "mg_prolong_bilinear");
}

template <typename T>
int zero_fill(fx_ctx *ctx, T *p, size_t n, const int *skip) {
    return launch_flat<0>(ctx, n, FlatZero<T>{p}, NoFin{}, skip, "mg_zero");
}

// Coarsest level: all sweeps in one block, the grid held in shared memory.  Each point
// evaluates exactly the expression of the sweep kernel, so the result is bitwise equal
// to running `nsweeps` separate sweeps.
// One-block coarsest solve: at most 4 points per thread (4096 points) and two smem copies.
inline bool coarse_fits(size_t n, size_t esize) { return n <= 4096 && 2 * n * esize <= 48 * 1024; }
inline int coarse_threads(size_t n) {
    // one point per thread while the grid fits a block (each sweep is a latency chain), up to
    // 4 points per thread above that
    size_t t = ((n + 31) / 32) * 32;
    if (t < 32) t = 32;
    if (t > 1024) t = 1024;
    return (int)t;
}

template <typename T>
__global__ void __launch_bounds__(1024) k_coarse_solve(T *u, const T *__restrict__ b, int rows, int cols,
                                                       A5<T> a, T wd, int nsweeps, bool zero_init, const int *skip) {
    if (skip && *(volatile const int *)skip) return;
    // Each thread owns up to kCoarsePts points (fixed for the whole solve): its rhs values and
    // interior flags stay in registers, the iterate ping-pongs between two smem copies.
    constexpr int kCoarsePts = 4;
    extern __shared__ unsigned char smem_raw[];
    T *s0 = reinterpret_cast<T *>(smem_raw);
    T *s1 = s0 + rows * cols;
    const int n = rows * cols;
#ifdef FX_CHECKED
    {
        unsigned dyn;
        asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dyn));
        if (!(FX_IN(n - 1, kCoarsePts * (int)blockDim.x) && FX_IN(2LL * n - 1, dyn / sizeof(T)))) return;
    }
#endif
    int idx[kCoarsePts];
    bool inner[kCoarsePts];
    T bv[kCoarsePts];
#pragma unroll
    for (int k = 0; k < kCoarsePts; k++) {
        const int i = threadIdx.x + k * blockDim.x;
        idx[k] = i;
        const int r = i / cols, c = i % cols;
        inner[k] = i < n && r > 0 && c > 0 && r < rows - 1 && c < cols - 1;
        bv[k] = i < n ? b[i] : (T)0;
        if (i < n) {
            const T v = zero_init ? (T)0 : u[i];
            s0[i] = v;
            s1[i] = v;
        }
    }
    __syncthreads();
    for (int k = 0; k < nsweeps; k++) {
        const T *src = (k & 1) ? s1 : s0;
        T *dst = (k & 1) ? s0 : s1;
#pragma unroll
        for (int q = 0; q < kCoarsePts; q++) {
            if (!inner[q]) continue;
            const int i = idx[q];
            Nb<T> nb;
            nb.c = src[i];
            nb.n = src[i - cols];
            nb.s = src[i + cols];
            nb.w = src[i - 1];
            nb.e = src[i + 1];
            dst[i] = fx_fma(wd, bv[q] - op5<T>(a, nb), nb.c);
        }
        __syncthreads();
    }
    const T *fin = (nsweeps & 1) ? s1 : s0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) u[i] = fin[i];
}

template <typename T>
int vertex_cycle(fx_mg *mg, T *x, const T *b, const int *skip, bool x_zero) {
    fx_ctx *ctx = mg->ctx;
    const int nl = (int)mg->lv.size();
    MgLevel &L0 = mg->lv[0];
    // Level 0 iterates between x and tmp0; the ring is homogeneous Dirichlet.
    if (!x_zero) {
        fx_buf xb;
        xb.ctx = ctx;
        xb.ptr = x;
        xb.len = L0.rows * L0.cols;
        xb.dtype = mg->dtype;
        xb.owned = false;
        FX_TRY(fx_zero_boundaries(ctx, &xb, L0.rows, L0.cols));
    }
    std::vector<T *> cur(nl), oth(nl);
    std::vector<const T *> rhs(nl);
    cur[0] = x;
    oth[0] = (T *)mg->tmp0->ptr;
    rhs[0] = b;
    for (int l = 1; l < nl; l++) {
        cur[l] = (T *)mg->lv[l].u->ptr;
        oth[l] = (T *)mg->lv[l].tmp->ptr;
        rhs[l] = (const T *)mg->lv[l].rhs->ptr;
    }
    auto smooth = [&](int l, size_t n) -> int {
        MgLevel &L = mg->lv[l];
        for (size_t k = 0; k < n; k++) {
            FX_TRY(sweep<T>(ctx, cur[l], oth[l], rhs[l], L.a5, mg->omega, L.rows, L.cols, skip));
            std::swap(cur[l], oth[l]);
        }
        return FX_OK;
    };
    for (int l = 0; l < nl - 1; l++) {
        MgLevel &L = mg->lv[l], &C = mg->lv[l + 1];
        FX_TRY(smooth(l, mg->n_pre));
        FX_TRY(residual<T>(ctx, cur[l], rhs[l], oth[l], L.a5, L.rows, L.cols, skip));
        FX_TRY(restrict_fw<T>(ctx, oth[l], (T *)C.rhs->ptr, L.cols, C.rows, C.cols, skip));
        FX_TRY(zero_fill<T>(ctx, cur[l + 1], C.rows * C.cols, skip));
    }
    {
        const int l = nl - 1;
        MgLevel &L = mg->lv[l];
        const size_t n = L.rows * L.cols;
        const size_t smem = 2 * n * sizeof(T);
        if (coarse_fits(n, sizeof(T)) && mg->coarse_sweeps > 0) {
            k_coarse_solve<T><<<1, coarse_threads(n), smem, ctx->stream>>>(cur[l], rhs[l], (int)L.rows, (int)L.cols,
                                                              make_a5<T>(L.a5), (T)(mg->omega / L.a5[0]),
                                                              (int)mg->coarse_sweeps, false, skip);
            FX_TRY(check_launch(ctx, "mg_coarse_solve"));
            // the kernel writes the final iterate back into cur[l]; cur/oth roles unchanged
        } else {
            FX_TRY(smooth(l, mg->coarse_sweeps));
        }
    }
    for (int l = nl - 2; l >= 0; l--) {
        MgLevel &L = mg->lv[l], &C = mg->lv[l + 1];
        FX_TRY(prolong_bilinear<T>(ctx, cur[l + 1], cur[l], C.cols, L.rows, L.cols, skip));
        FX_TRY(smooth(l, mg->n_post));
    }
    if (cur[0] != x) {
        FX_CUDA(cudaMemcpyAsync(x, cur[0], L0.rows * L0.cols * sizeof(T), cudaMemcpyDeviceToDevice, ctx->stream));
    }
    return FX_OK;
}

// F64 <-> F32 conversion with skip, for a single-precision cycle inside an F64 solve.
template <typename S, typename D>
int convert(fx_ctx *ctx, const S *src, D *dst, size_t n, const int *skip) {
    return launch_flat<0>(ctx, n, FlatConvert<S, D>{src, dst}, NoFin{}, skip, "mg_convert");
}

// Chebyshev smoother of the reference hierarchy (multigrid.rs:308-473): the first-kind
// Chebyshev recurrence for D^-1 A with the bounds emax = 2, emin = 0.2 (D the level Laplacian's
// diagonal) on three rotating vectors u, w0, w1, each step the reference's sequence of backend
// ops (stencil apply, copy, axpy, scale, zero_boundaries) -- no inner products, no host sync.
int chebyshev_smooth(fx_ctx *ctx, MgLevel &L, const fx_grid &g, const fx_stencil &s, const fx_boundaries &bc,
                     size_t n) {
    if (n == 0) return FX_OK;
    const double emax = 2.0, emin = 0.1 * emax;
    const double scale = 2.0 / (emax + emin);
    const double alpha = 1.0 - scale * emin;
    const double mu = 1.0 / alpha, omegaprod = 2.0 / alpha;
    const double inv_dx2 = 1.0 / (L.dx * L.dx), inv_dy2 = 1.0 / (L.dy * L.dy);
    const double inv_diag = -1.0 / (2.0 * inv_dx2 + 2.0 * inv_dy2);
    double c_km1 = 1.0, c_k = mu;
    FX_TRY(fx_apply_stencil(ctx, L.u, L.tmp, &g, &s, &bc));
    FX_TRY(fx_copy(ctx, L.rhs, L.w0));
    FX_TRY(fx_axpy(ctx, -1.0, L.tmp, L.w0));
    FX_TRY(fx_scale(ctx, L.w0, scale * inv_diag));
    FX_TRY(fx_axpy(ctx, 1.0, L.u, L.w0));
    FX_TRY(fx_zero_boundaries(ctx, L.w0, L.rows, L.cols));
    if (n == 1) return fx_copy(ctx, L.w0, L.u);
    fx_buf *buf[3] = {L.u, L.w0, L.w1};
    int km1 = 0, k = 1, kp1 = 2;
    for (size_t i = 1; i < n; i++) {
        FX_TRY(fx_apply_stencil(ctx, buf[k], L.tmp, &g, &s, &bc));
        FX_TRY(fx_copy(ctx, L.rhs, buf[kp1]));
        FX_TRY(fx_axpy(ctx, -1.0, L.tmp, buf[kp1]));
        FX_TRY(fx_scale(ctx, buf[kp1], inv_diag));
        const double c_kp1 = 2.0 * mu * c_k - c_km1;
        const double omega = omegaprod * c_k / c_kp1;
        FX_TRY(fx_scale(ctx, buf[kp1], omega * scale));
        FX_TRY(fx_axpy(ctx, omega, buf[k], buf[kp1]));
        FX_TRY(fx_axpy(ctx, 1.0 - omega, buf[km1], buf[kp1]));
        FX_TRY(fx_zero_boundaries(ctx, buf[kp1], L.rows, L.cols));
        c_km1 = c_k;
        c_k = c_kp1;
        const int t = km1;
        km1 = k;
        k = kp1;
        kp1 = t;
    }
    if (k == 1) return fx_copy(ctx, L.w0, L.u);
    if (k == 2) return fx_copy(ctx, L.w1, L.u);
    return FX_OK;
}

// Reference-semantics cycle (multigrid.rs:188-230), built from the trait ops.
int reference_cycle(fx_mg *mg, fx_buf *x, const fx_buf *b, bool x_zero) {
    fx_ctx *ctx = mg->ctx;
    const int nl = (int)mg->lv.size();
    MgLevel &L0 = mg->lv[0];
    FX_TRY(fx_copy(ctx, b, L0.rhs));
    if (x_zero) FX_TRY(fx_fill(ctx, L0.u, 0.0));
    else FX_TRY(fx_copy(ctx, x, L0.u));
    auto smooth = [&](int l, size_t n) -> int {
        MgLevel &L = mg->lv[l];
        fx_grid g{L.rows, L.cols, L.dx, L.dy};
        fx_stencil s{5, LAP_DR, LAP_DC, L.lap5};
        if (mg->smoother == 1) return chebyshev_smooth(ctx, L, g, s, mg->bc, n);
        for (size_t k = 0; k < n; k++) FX_TRY(fx_weighted_jacobi(ctx, L.u, L.rhs, mg->omega, &g, &s, &mg->bc));
        return FX_OK;
    };
    for (int l = 0; l < nl - 1; l++) {
        MgLevel &L = mg->lv[l], &C = mg->lv[l + 1];
        FX_TRY(smooth(l, mg->n_pre));
        fx_grid g{L.rows, L.cols, L.dx, L.dy}, cg{C.rows, C.cols, C.dx, C.dy};
        fx_stencil s{5, LAP_DR, LAP_DC, L.lap5};
        FX_TRY(fx_apply_stencil(ctx, L.u, L.tmp, &g, &s, &mg->bc));  // multigrid.rs:476-491
        FX_TRY(fx_scale(ctx, L.tmp, -1.0));
        FX_TRY(fx_axpy(ctx, 1.0, L.rhs, L.tmp));
        FX_TRY(fx_restrict(ctx, L.tmp, C.rhs, &g, &cg));
        FX_TRY(fx_fill(ctx, C.u, 0.0));
    }
    FX_TRY(smooth(nl - 1, mg->n_pre + mg->n_post + 10));
    for (int l = nl - 2; l >= 0; l--) {
        MgLevel &L = mg->lv[l], &C = mg->lv[l + 1];
        fx_grid g{L.rows, L.cols, L.dx, L.dy}, cg{C.rows, C.cols, C.dx, C.dy};
        FX_TRY(fx_prolong(ctx, C.u, L.u, &cg, &g));
        FX_TRY(smooth(l, mg->n_post));
    }
    return fx_copy(ctx, L0.u, x);
}

}  // namespace

namespace {

// Fused V(2,2)-cycle from a zero initial guess: per level one down and one up kernel, the
// coarsest level solved in one block.  b0 / z0 are the finest-level rhs and result (TB / TZ
// may be double while the cycle runs in T = float); with RZ the finest up kernel also
// reduces r.z into `fin`.

template <typename T, typename TB, typename TZ, bool RZ, typename Fin>
int fused_cycle(fx_mg *mg, const TB *b0, TZ *z0, Fin fin, const int *skip) {
    fx_ctx *ctx = mg->ctx;
    const int nl = (int)mg->lv.size();
    auto vop = [&](int l) {
        const MgLevel &L = mg->lv[l];
        return VOp<T>{make_a5<T>(L.a5), (T)(mg->omega / L.a5[0])};
    };
    // down: level 0 reads b0 (TB), the others their rhs (T); x2 of level 0 lives in tmp0
    {
        const MgLevel &L = mg->lv[0], &C = mg->lv[1];
        FX_TRY((launch_wdown<T, TB>(ctx, L.rows, L.cols, b0, (T *)mg->tmp0->ptr, (T *)C.rhs->ptr, C.cols,
                                    vop(0), skip, mg->chunk_pct)));
    }
    // levels top .. nl-1 run in the one-block tail kernel: top is the finest level >= 1 whose
    // tail working set fits in shared memory
    const size_t top_cap = mg->tail_top_max ? std::min(mg->tail_top_max, (size_t)tail_kt<T>() * kTailThreads)
                                            : (size_t)tail_kt<T>() * kTailThreads;
    int top = nl - 1;
    size_t tail_smem = 2 * mg->lv[nl - 1].rows * mg->lv[nl - 1].cols * sizeof(T);
    for (int t = nl - 2; t >= 1 && nl - t <= kTailMaxLevels; t--) {
        size_t n[kTailMaxLevels];
        for (int l = t; l < nl; l++) n[l - t] = mg->lv[l].rows * mg->lv[l].cols;
        const size_t bytes = tail_smem_bytes(n, nl - t, sizeof(T));
        if (bytes > kTailSmemMax || n[0] > top_cap) break;
        top = t;
        tail_smem = bytes;
    }
    if (nl - top > kTailMaxLevels || tail_smem > kTailSmemMax ||
        (top == nl - 1 ? mg->lv[top].rows * mg->lv[top].cols > 4096
                       : mg->lv[top].rows * mg->lv[top].cols > top_cap))
        return fail(FX_ERR_UNSUPPORTED, "coarsest level too large for the one-block solve");
    const int mid_pct = mg->chunk_pct;
    for (int l = 1; l < top; l++) {
        const MgLevel &L = mg->lv[l], &C = mg->lv[l + 1];
        FX_TRY((launch_wdown<T, T>(ctx, L.rows, L.cols, (const T *)L.rhs->ptr, (T *)L.tmp->ptr, (T *)C.rhs->ptr,
                                   C.cols, vop(l), skip, mid_pct)));
    }
    {
        TailArgs<T> A{};
        A.nlev = nl - top;
        for (int k = 0; k < A.nlev; k++) {
            A.rows[k] = (int)mg->lv[top + k].rows;
            A.cols[k] = (int)mg->lv[top + k].cols;
            A.op[k] = vop(top + k);
        }
        const MgLevel &T0 = mg->lv[top];
        A.b_top = (const T *)T0.rhs->ptr;
        A.u_top = (T *)T0.u->ptr;
        A.coarse_sweeps = (int)mg->coarse_sweeps;
        FX_TRY(launch_vtail<T>(ctx, A, tail_smem, skip));
    }
    for (int l = top - 1; l >= 1; l--) {
        const MgLevel &L = mg->lv[l], &C = mg->lv[l + 1];
        FX_TRY((launch_wup<T, T, T, false>(ctx, L.rows, L.cols, (const T *)L.tmp->ptr, (const T *)C.u->ptr, C.cols,
                                           (const T *)L.rhs->ptr, (T *)L.u->ptr, vop(l), NoFin{}, skip,
                                           mid_pct)));
    }
    const MgLevel &L = mg->lv[0], &C = mg->lv[1];
    return launch_wup<T, TB, TZ, RZ>(ctx, L.rows, L.cols, (const T *)mg->tmp0->ptr, (const T *)C.u->ptr, C.cols, b0,
                                     z0, vop(0), fin, skip, mg->chunk_pct);
}

bool fusable(const fx_mg *m) {
    if (m->mode != 1 || m->n_pre != 2 || m->n_post != 2 || m->lv.size() < 2) return false;
    const MgLevel &L = m->lv.back();
    return coarse_fits(L.rows * L.cols, m->dtype == FX_F64 ? 8 : 4);
}

}  // namespace

int fx_mg::View::apply_pcg(fx_buf *z, const fx_buf *r, const int *skip, DevState *S, bool first) {
    fx_mg *m = mg;
    if (!fusable(m) || z->len != m->lv[0].rows * m->lv[0].cols || z->dtype != r->dtype) return FX_ERR_UNSUPPORTED;
    if (z->dtype == FX_F32) {  // single-precision vectors (the inner solves of iterative refinement)
        if (m->dtype != FX_F32) return FX_ERR_UNSUPPORTED;
        const float *b0 = (const float *)r->ptr;
        float *z0 = (float *)z->ptr;
        if (first) return fused_cycle<float, float, float, true>(m, b0, z0, FinPcgRzInit{S}, skip);
        return fused_cycle<float, float, float, true>(m, b0, z0, FinPcgRz{S}, skip);
    }
    const double *b0 = (const double *)r->ptr;
    double *z0 = (double *)z->ptr;
    if (m->dtype == FX_F64) {
        if (first) return fused_cycle<double, double, double, true>(m, b0, z0, FinPcgRzInit{S}, skip);
        return fused_cycle<double, double, double, true>(m, b0, z0, FinPcgRz{S}, skip);
    }
    if (first) return fused_cycle<float, double, double, true>(m, b0, z0, FinPcgRzInit{S}, skip);
    return fused_cycle<float, double, double, true>(m, b0, z0, FinPcgRz{S}, skip);
}

bool fx_mg::View::fills_from_zero(const fx_buf *z) const {
    return fusable(mg) && z->dtype == FX_F64 && z->len == mg->lv[0].rows * mg->lv[0].cols;
}

int fx_mg::View::apply(fx_buf *z, const fx_buf *r, const int *skip, bool z_zero) {
    fx_mg *m = mg;
    const MgLevel &L0 = m->lv[0];
    if (z->len != L0.rows * L0.cols || r->len != z->len)
        return fail(FX_ERR_DIMENSION_MISMATCH, "dimension mismatch: expected " +
                                                   std::to_string(L0.rows * L0.cols) + ", got " +
                                                   std::to_string(z->len));
    if (z->dtype != r->dtype) return fail(FX_ERR_INVALID_ARGUMENT, "dtype mismatch between buffers");
    if (m->mode == 0) return reference_cycle(m, z, r, z_zero);
    if (z_zero && fusable(m) && z->dtype == FX_F64) {
        if (m->dtype == FX_F64)
            return fused_cycle<double, double, double, false>(m, (const double *)r->ptr, (double *)z->ptr, NoFin{}, skip);
        return fused_cycle<float, double, double, false>(m, (const double *)r->ptr, (double *)z->ptr, NoFin{}, skip);
    }
    if (z_zero) {  // the unfused cycle reads z as its initial guess
        FX_TRY(launch_flat<0>(m->ctx, z->len, FlatZero<double>{(double *)z->ptr}, NoFin{}, skip, "mg_zero"));
    }
    if (m->dtype == z->dtype) {
        if (z->dtype == FX_F64) return vertex_cycle<double>(m, (double *)z->ptr, (const double *)r->ptr, skip, z_zero);
        return vertex_cycle<float>(m, (float *)z->ptr, (const float *)r->ptr, skip, z_zero);
    }
    // single-precision cycle on double-precision vectors
    if (m->dtype == FX_F32 && z->dtype == FX_F64) {
        const size_t n = z->len;
        float *x32 = (float *)m->x32->ptr, *b32 = (float *)m->b32->ptr;
        FX_TRY(convert<double, float>(m->ctx, (const double *)r->ptr, b32, n, skip));
        if (z_zero) FX_TRY(zero_fill<float>(m->ctx, x32, n, skip));
        else FX_TRY(convert<double, float>(m->ctx, (const double *)z->ptr, x32, n, skip));
        FX_TRY(vertex_cycle<float>(m, x32, b32, skip, z_zero));
        return convert<float, double>(m->ctx, x32, (double *)z->ptr, n, skip);
    }
    return fail(FX_ERR_UNSUPPORTED, "multigrid dtype combination not supported");
}

// ================================================================ Krylov solvers

namespace {

// The solver state moves between host and device without the copy engines: the device writes
// it into mapped page-locked memory (k_state_out) and takes its initial value as a kernel
// parameter (k_state_in).  A cudaMemcpyAsync of a few bytes queues on a copy engine behind
// whatever large transfer that engine is doing: in a stream of solves whose 134 MB right-hand
// sides and solutions are copied on other streams while the previous solve runs, every read-back
// of the drive loop waited for a whole solution transfer.
__global__ void k_state_in(DevState *d, DevState v) { *d = v; }
__global__ void k_state_out(const DevState *d, DevState *h) { *h = *d; }
__global__ void k_state_stop(DevState *d, int reason) {
    d->done = 1;
    d->halt = 1;
    d->reason = reason;
}

struct SolverBase {
    fx_ctx *ctx = nullptr;
    fx_grid g{};
    double tol = 0;
    size_t max_iter = 0;
    DevState *d_st = nullptr;
    DevState *h_st = nullptr;     // mapped page-locked memory
    DevState *h_st_dev = nullptr; // its device address
    std::vector<fx_buf *> bufs;
    int dtype = FX_F64;  // of the solver's vectors (x, b and the work vectors)
    const fx_op *op = nullptr;  // set for the duration of a *_solve_op call

    int init_base(fx_ctx *c, const fx_grid *grid, double t, size_t mi, int nvec, int dt = FX_F64) {
        ctx = c;
        g = *grid;
        tol = t;
        max_iter = mi;
        dtype = dt;
        FX_CUDA(cudaMalloc(&d_st, sizeof(DevState)));
        FX_CUDA(cudaHostAlloc(&h_st, sizeof(DevState), cudaHostAllocMapped));
        FX_CUDA(cudaHostGetDevicePointer((void **)&h_st_dev, h_st, 0));
        for (int i = 0; i < nvec; i++) {
            fx_buf *b = nullptr;
            FX_TRY(fx_alloc(ctx, g.rows * g.cols, dt, &b));
            bufs.push_back(b);
        }
        return FX_OK;
    }
    virtual ~SolverBase() {
        if (ctx) cudaStreamSynchronize(ctx->stream);
        for (auto *b : bufs) fx_free(b);
        if (d_st) cudaFree(d_st);
        if (h_st) cudaFreeHost(h_st);
    }
    int reset_state() {
        DevState s;
        std::memset(&s, 0, sizeof(s));
        s.tol = tol;
        s.max_iter = (long long)max_iter;
        *h_st = s;
        k_state_in<<<1, 1, 0, ctx->stream>>>(d_st, s);
        return check_launch(ctx, "state_in");
    }
    int read_state() {
        k_state_out<<<1, 1, 0, ctx->stream>>>(d_st, h_st_dev);
        FX_TRY(check_launch(ctx, "state_out"));
        FX_CUDA(cudaStreamSynchronize(ctx->stream));
        return FX_OK;
    }
    // A residual that is not a finite number (a NaN or Inf in b, x or the operator) never passes
    // the reference's stop test and would run to max_iter; the solve stops with Breakdown instead.
    int stop_nonfinite() {
        h_st->done = 1;
        h_st->halt = 1;
        h_st->reason = FX_BREAKDOWN;
        k_state_stop<<<1, 1, 0, ctx->stream>>>(d_st, FX_BREAKDOWN);
        FX_TRY(check_launch(ctx, "state_stop"));
        FX_CUDA(cudaStreamSynchronize(ctx->stream));
        return FX_OK;
    }
    int check_io(const fx_buf *x, const fx_buf *b) {
        FX_TRY(check_buf(x, "x"));
        FX_TRY(check_buf(b, "b"));
        FX_TRY(check_grid_len(&g, x));
        FX_TRY(check_grid_len(&g, b));
        if (x->dtype != dtype || b->dtype != dtype)
            return fail(FX_ERR_INVALID_ARGUMENT, dtype == FX_F64 ? "solver vectors must be F64"
                                                                   : "solver vectors must be F32");
        return FX_OK;
    }
    // Run `step(i)` for i = 0, 1, ... until the device says done.  Iterations are enqueued
    // in batches sized from the observed convergence rate; surplus iterations are no-ops.
    // The first batch follows the setup kernels without a read-back in between (a solve the
    // setup already finished makes it a no-op), so the device never idles before it.
    template <typename Step>
    int drive(Step step, size_t max_launch, bool expensive) {
        size_t launched = 0;
        size_t batch = expensive ? 1 : 4;
        while (launched < max_launch) {
            const size_t nb = std::min(batch, max_launch - launched);
            for (size_t k = 0; k < nb; k++) FX_TRY(step(launched + k));
            launched += nb;
            FX_TRY(read_state());
            if (h_st->done) return FX_OK;
            if (!std::isfinite(h_st->resid)) return stop_nonfinite();
            // predict the iterations still needed from the mean reduction rate so far (r0: the
            // initial residual, recorded on the device by every solver's setup finaliser)
            const double r0 = h_st->r0 > 0 ? h_st->r0 : 1.0;
            const double rk = h_st->resid;
            size_t pred = 1;
            if (rk > 0 && rk < r0 && launched > 0 && h_st->tol > 0) {
                const double rate = std::log(rk / r0) / (double)launched;
                const double need = std::log(h_st->tol / rk) / rate;
                if (need > 1 && need < 1e6) pred = (size_t)std::ceil(need);
            } else {
                pred = batch * 2;
            }
            batch = std::max<size_t>(1, std::min<size_t>(pred, expensive ? 8 : 128));
        }
        return read_state();
    }
    void stats(fx_stats *out) {
        out->iterations = (size_t)h_st->iter;
        out->residual = h_st->resid;
        out->reason = h_st->reason;
    }
};

#define SOLVER_MODE_DISPATCH(P, ...)     \
    do {                                 \
        if ((P).mode == 5) {             \
            constexpr int MODE = 5;      \
            __VA_ARGS__;                 \
        } else if ((P).mode == 9) {      \
            constexpr int MODE = 9;      \
            __VA_ARGS__;                 \
        } else {                         \
            constexpr int MODE = 0;      \
            __VA_ARGS__;                 \
        }                                \
    } while (0)

int prep_op(const fx_grid &g, const fx_stencil *st, const fx_boundaries *bc, StencilP *P) {
    BcP B;
    FX_TRY(make_bc(bc, g.dx, g.dy, &B, true));
    return make_stencil(st, P);
}

// ------------------------------------------------ CG / PCG kernels (cg.rs:96-256)

// r = b - A x (cg.rs:104-111); reduction r.r
template <typename T, int MODE>
struct PtInitResid {
    static constexpr int NA = 1;
    OpA<T, MODE> A;
    const T *b;
    T *r;
    T *r2;  // optional second copy (BiCGSTAB r_hat)
    __device__ __forceinline__ const T *aux(int) const { return b; }
    __device__ __forceinline__ void operator()(bool ring, int rr, int c, size_t idx, const Nb<T> &nb, const T *a, CSum *acc) const {
        const T ax = A.apply(ring, nb, idx);
        const T rv = fx_fma((T)-1, ax, a[0]);
        r[idx] = rv;
        if (r2) r2[idx] = rv;
        csum_fma(acc[0], (double)rv, (double)rv);
    }
};

struct FinCgInit {  // unpreconditioned: rs_old = r.r; loop-top test of iteration 0
    DevState *S;
    __device__ void operator()(const double *v) const {
        S->rs_old = v[0];
        S->beta = 0.0;
        S->iter = 0;
        S->resid = sqrt(v[0]);
        S->r0 = S->resid;
        if (S->max_iter == 0) st_finish(S, FX_MAX_ITERATIONS, 0, sqrt(v[0]));
        else if (sqrt(v[0]) < S->tol) st_finish(S, FX_CONVERGED, 0, sqrt(v[0]));
    }
};

// p_new = (r|z) + beta p_old; ap = A p_new; reduction p.ap
template <typename T, int MODE>
struct PtCgDir {
    static constexpr int NA = 0;
    static constexpr int MINB = 4;  // FP64: 4 band blocks per SM (56 registers, no spill)
    OpA<T, MODE> A;
    T *p_new;
    __device__ __forceinline__ const T *aux(int) const { return nullptr; }
    __device__ __forceinline__ void operator()(bool ring, int r, int c, size_t idx, const Nb<T> &nb, const T *a, CSum *acc) const {
        p_new[idx] = nb.c;
        const T ap = A.apply(ring, nb, idx);
        csum_fma(acc[0], (double)nb.c, (double)ap);
    }
};

struct FinCgDir {  // alpha = rs_old / p.ap, breakdown test (cg.rs:133-142)
    DevState *S;
    __device__ void operator()(const double *v) const {
        const double p_ap = v[0];
        if (fabs(p_ap) < 1e-30) {
            st_finish(S, FX_BREAKDOWN, S->iter, S->resid);
            return;
        }
        S->alpha = S->rs_old / p_ap;
    }
};

// x += alpha p; r -= alpha A p (A p recomputed from p); reduction r.r
template <typename T, int MODE>
struct PtCgUpd {
    static constexpr int NA = 2;
    static constexpr int MINB = 4;  // FP64: 4 band blocks per SM (56 registers, no spill)
    OpA<T, MODE> A;
    T *x, *r;
    const DevState *S;
    T alpha;
    __device__ __forceinline__ void prepare() { alpha = (T)S->alpha; }
    __device__ __forceinline__ const T *aux(int k) const { return k == 0 ? x : r; }
    __device__ __forceinline__ void operator()(bool ring, int rr, int c, size_t idx, const Nb<T> &nb, const T *a, CSum *acc) const {
        const T ap = A.apply(ring, nb, idx);
        x[idx] = fx_fma(alpha, nb.c, a[0]);
        const T rv = fx_fma(-alpha, ap, a[1]);
        r[idx] = rv;
        csum_fma(acc[0], (double)rv, (double)rv);
    }
};

struct FinCgUpd {  // beta = rs_new / rs_old; loop-top test of the next iteration
    DevState *S;
    __device__ void operator()(const double *v) const {
        const double rs_new = v[0];
        S->beta = rs_new / S->rs_old;
        S->rs_old = rs_new;
        S->iter += 1;
        S->resid = sqrt(rs_new);
        if (S->iter >= S->max_iter) st_finish(S, FX_MAX_ITERATIONS, S->max_iter, sqrt(rs_new));
        else if (sqrt(rs_new) < S->tol) st_finish(S, FX_CONVERGED, S->iter, sqrt(rs_new));
    }
};

// PCG: after r update, rr stored; stop test; then z = M^-1 r; rz = r.z -> beta
struct FinPcgResid {
    DevState *S;
    __device__ void operator()(const double *v) const {
        S->rr = v[0];
        S->resid = sqrt(v[0]);
    }
};

struct FinPcgUpd {
    DevState *S;
    __device__ void operator()(const double *v) const {
        S->rr = v[0];
        S->iter += 1;
        S->resid = sqrt(v[0]);
        if (S->iter >= S->max_iter) st_finish(S, FX_MAX_ITERATIONS, S->max_iter, sqrt(v[0]));
        else if (sqrt(v[0]) < S->tol) st_finish(S, FX_CONVERGED, S->iter, sqrt(v[0]));
    }
};

}  // namespace

struct fx_cg : SolverBase {
    // bufs: 0 r, 1 z, 2 p0, 3 p1
};

namespace {

template <typename T, int MODE>
int cg_solve_impl(fx_cg *s, fx_buf *x, const fx_buf *b, double coeff, const StencilP &P, fx_precond *pc) {
    fx_ctx *ctx = s->ctx;
    constexpr int DT = sizeof(T) == 8 ? FX_F64 : FX_F32;
    const size_t RR = s->g.rows, CC = s->g.cols;
    OpA<T, MODE> A{P, (T)coeff, (int)RR, (int)CC};
    T *r = (T *)s->bufs[0]->ptr, *z = (T *)s->bufs[1]->ptr;
    T *pb[2] = {(T *)s->bufs[2]->ptr, (T *)s->bufs[3]->ptr};
    T *xp = (T *)x->ptr;
    const T *bp = (const T *)b->ptr;
    const size_t n = s->g.rows * s->g.cols;
    DevState *S = s->d_st;
    const int *halt = &S->halt;
    FX_TRY(s->reset_state());
    FX_CUDA(cudaMemsetAsync(pb[0], 0, n * sizeof(T), ctx->stream));
    FX_CUDA(cudaMemsetAsync(pb[1], 0, n * sizeof(T), ctx->stream));
    if (!pc) {
        FX_TRY((launch_pt<T, 1>(ctx, RR, CC, Ld1<T>{xp}, PtInitResid<T, MODE>{A, bp, r, nullptr}, FinCgInit{S},
                                      nullptr, "cg_init")));
        auto step = [&](size_t i) -> int {
            T *po = pb[i & 1], *pn = pb[(i + 1) & 1];
            FX_TRY((launch_pt<T, 1>(ctx, RR, CC, LdAypx<T>{r, po, S}, PtCgDir<T, MODE>{A, pn}, FinCgDir{S}, halt,
                                          "cg_dir")));
            return launch_pt<T, 1>(ctx, RR, CC, Ld1<T>{pn}, PtCgUpd<T, MODE>{A, xp, r, S}, FinCgUpd{S}, halt,
                                         "cg_update");
        };
        return s->drive(step, s->max_iter + 1, n >= (1u << 20));
    }
    // preconditioned (cg.rs:178-256)
    FX_TRY((launch_pt<T, 1>(ctx, RR, CC, Ld1<T>{xp}, PtInitResid<T, MODE>{A, bp, r, nullptr}, FinPcgResid{S},
                                  nullptr, "pcg_init")));
    fx_buf rb{ctx, r, n, DT, false}, zb{ctx, z, n, DT, false};
    // z = M^-1 r and rz = r.z, fused into the preconditioner when it has a fused form
    auto precondition = [&](bool first) -> int {
        const int st = pc->apply_pcg(&zb, &rb, halt, S, first);
        if (st != FX_ERR_UNSUPPORTED) return st;
        FX_TRY(zero_fill<T>(ctx, z, n, halt));
        FX_TRY(pc->apply(&zb, &rb, halt, true));
        if (first) return launch_flat<1>(ctx, n, FlatDot<T>{r, z}, FinPcgRzInit{S}, halt, "pcg_rz");
        return launch_flat<1>(ctx, n, FlatDot<T>{r, z}, FinPcgRz{S}, halt, "pcg_rz");
    };
    FX_TRY(precondition(true));
    auto step = [&](size_t i) -> int {
        T *po = pb[i & 1], *pn = pb[(i + 1) & 1];
        FX_TRY((launch_pt<T, 1>(ctx, RR, CC, LdAypx<T>{z, po, S}, PtCgDir<T, MODE>{A, pn}, FinCgDir{S}, halt,
                                      "pcg_dir")));
        FX_TRY((launch_pt<T, 1>(ctx, RR, CC, Ld1<T>{pn}, PtCgUpd<T, MODE>{A, xp, r, S}, FinPcgUpd{S}, halt,
                                      "pcg_update")));
        return precondition(false);
    };
    return s->drive(step, s->max_iter + 1, true);
}

// ------------------------------------------------ pipelined CG (pipelined_cg.rs:353-424)

template <typename T, int MODE>
struct PtPipeInitQ {  // q = A x; r = b - q
    static constexpr int NA = 1;
    OpA<T, MODE> A;
    const T *b;
    T *r;
    __device__ __forceinline__ const T *aux(int) const { return b; }
    __device__ __forceinline__ void operator()(bool ring, int rr, int c, size_t idx, const Nb<T> &nb, const T *a, CSum *) const {
        r[idx] = fx_fma((T)-1, A.apply(ring, nb, idx), a[0]);
    }
};

template <typename T, int MODE>
struct PtPipeInitW {  // w = A r; p = t = z = 0; reductions (r.r, r.w)
    static constexpr int NA = 0;
    OpA<T, MODE> A;
    T *w, *p, *t, *z;
    __device__ __forceinline__ const T *aux(int) const { return nullptr; }
    __device__ __forceinline__ void operator()(bool ring, int rr, int c, size_t idx, const Nb<T> &nb, const T *a, CSum *acc) const {
        const T wv = A.apply(ring, nb, idx);
        w[idx] = wv;
        p[idx] = (T)0;
        t[idx] = (T)0;
        z[idx] = (T)0;
        csum_fma(acc[0], (double)nb.c, (double)nb.c);
        csum_fma(acc[1], (double)nb.c, (double)wv);
    }
};

__device__ __forceinline__ void pipe_scalars(DevState *S) {
    const double beta = S->gamma / S->gamma_prev;
    S->beta = beta;
    S->alpha = S->gamma / (S->delta - beta * S->gamma / S->alpha_prev);
}

struct FinPipeInit {
    DevState *S;
    __device__ void operator()(const double *v) const {
        S->gamma = v[0];
        S->delta = v[1];
        S->gamma_prev = INFINITY;
        S->alpha_prev = INFINITY;
        S->iter = 0;
        S->resid = sqrt(v[0]);
        S->r0 = S->resid;
        if (S->max_iter == 0) st_finish(S, FX_MAX_ITERATIONS, 0, sqrt(v[0]));
        else if (sqrt(v[0]) < S->tol) st_finish(S, FX_CONVERGED, 0, sqrt(v[0]));
        else pipe_scalars(S);
    }
};

// One whole iteration: q = A w (on the fly), the 6-way update, and (r.r, r.w) of the
// updated vectors for the next iteration's scalars.
template <typename T, int MODE>
struct PtPipeIter {
    static constexpr int NA = 5;
    OpA<T, MODE> A;
    T *z, *t, *p, *x, *r, *w_new;
    const DevState *S;
    T alpha, beta;
    __device__ __forceinline__ void prepare() {
        alpha = (T)S->alpha;
        beta = (T)S->beta;
    }
    __device__ __forceinline__ const T *aux(int k) const {
        return k == 0 ? z : (k == 1 ? t : (k == 2 ? p : (k == 3 ? x : r)));
    }
    __device__ __forceinline__ void operator()(bool ring, int rr, int c, size_t idx, const Nb<T> &nb, const T *a, CSum *acc) const {
        const T q = A.apply(ring, nb, idx);
        const T w = nb.c;
        const T zn = q + a[0] * beta;
        const T tn = w + a[1] * beta;
        const T pn = a[4] + a[2] * beta;
        z[idx] = zn;
        t[idx] = tn;
        p[idx] = pn;
        x[idx] = fx_fma(alpha, pn, a[3]);
        const T rn = fx_fma(-alpha, tn, a[4]);
        const T wn = fx_fma(-alpha, zn, w);
        r[idx] = rn;
        w_new[idx] = wn;
        csum_fma(acc[0], (double)rn, (double)rn);
        csum_fma(acc[1], (double)rn, (double)wn);
    }
};

struct FinPipeIter {
    DevState *S;
    __device__ void operator()(const double *v) const {
        S->gamma_prev = S->gamma;
        S->alpha_prev = S->alpha;
        S->gamma = v[0];
        S->delta = v[1];
        S->iter += 1;
        S->resid = sqrt(v[0]);
        if (S->iter >= S->max_iter) st_finish(S, FX_MAX_ITERATIONS, S->max_iter, sqrt(v[0]));
        else if (sqrt(v[0]) < S->tol) st_finish(S, FX_CONVERGED, S->iter, sqrt(v[0]));
        else pipe_scalars(S);
    }
};

}  // namespace

struct fx_pipelined_cg : SolverBase {
    // bufs: 0 r, 1 p, 2 t, 3 z, 4 w0, 5 w1
};

namespace {

template <int MODE>
int pipe_solve_impl(fx_pipelined_cg *s, fx_buf *x, const fx_buf *b, double coeff, const StencilP &P) {
    using T = double;
    fx_ctx *ctx = s->ctx;
    const size_t RR = s->g.rows, CC = s->g.cols;
    OpA<T, MODE> A{P, (T)coeff, (int)RR, (int)CC};
    T *r = (T *)s->bufs[0]->ptr, *p = (T *)s->bufs[1]->ptr, *t = (T *)s->bufs[2]->ptr, *z = (T *)s->bufs[3]->ptr;
    T *w[2] = {(T *)s->bufs[4]->ptr, (T *)s->bufs[5]->ptr};
    T *xp = (T *)x->ptr;
    const T *bp = (const T *)b->ptr;
    DevState *S = s->d_st;
    const int *halt = &S->halt;
    FX_TRY(s->reset_state());
    FX_TRY((launch_pt<T, 0>(ctx, RR, CC, Ld1<T>{xp}, PtPipeInitQ<T, MODE>{A, bp, r}, NoFin{}, nullptr, "pipe_init_q")));
    FX_TRY((launch_pt<T, 2>(ctx, RR, CC, Ld1<T>{r}, PtPipeInitW<T, MODE>{A, w[0], p, t, z}, FinPipeInit{S}, nullptr,
                                  "pipe_init_w")));
    auto step = [&](size_t i) -> int {
        T *wo = w[i & 1], *wn = w[(i + 1) & 1];
        return launch_pt<T, 2>(ctx, RR, CC, Ld1<T>{wo}, PtPipeIter<T, MODE>{A, z, t, p, xp, r, wn, S},
                                     FinPipeIter{S}, halt, "pipe_iter");
    };
    return s->drive(step, s->max_iter + 1, s->g.rows * s->g.cols >= (1u << 22));
}

// ------------------------------------------------ preconditioned pipelined CG
//
// Ghysels & Vanroose (2014), Algorithm 4: the reference's PipelinedCgSolver (pipelined_cg.rs)
// is its unpreconditioned case, and the scalar recurrence (pipe_scalars) and the update forms
// (z = n + beta z, x += alpha p, ...) are those of its fused update.  With u = M r and m = M w:
//   init:  r = b - A x;  u = M r;  w = A u;  p = s = z = q = 0
//   iter:  m = M w;  n = A m;  z = n + b z;  q = m + b q;  s = w + b s;  p = u + b p;
//          x += a p;  r -= a s;  u -= a q;  w -= a z
// with gamma = (r, u), delta = (w, u) and the stop test on ||r||_2 reduced in the same pass.

template <typename T, int MODE>
struct PtPpcgInitW {  // w = A u; p = s = z = q = 0; reductions (r.u, w.u, r.r)
    static constexpr int NA = 1;
    OpA<T, MODE> A;
    const T *r;
    T *w, *p, *sv, *z, *q;
    __device__ __forceinline__ const T *aux(int) const { return r; }
    __device__ __forceinline__ void operator()(bool ring, int rr, int c, size_t idx, const Nb<T> &nb, const T *a, CSum *acc) const {
        const T u = nb.c;
        const T wv = A.apply(ring, nb, idx);
        w[idx] = wv;
        p[idx] = (T)0;
        sv[idx] = (T)0;
        z[idx] = (T)0;
        q[idx] = (T)0;
        csum_fma(acc[0], (double)a[0], (double)u);
        csum_fma(acc[1], (double)wv, (double)u);
        csum_fma(acc[2], (double)a[0], (double)a[0]);
    }
};

struct FinPpcgInit {
    DevState *S;
    __device__ void operator()(const double *v) const {
        S->gamma = v[0];
        S->delta = v[1];
        S->rr = v[2];
        S->gamma_prev = INFINITY;
        S->alpha_prev = INFINITY;
        S->iter = 0;
        S->resid = sqrt(v[2]);
        S->r0 = S->resid;
        if (S->max_iter == 0) st_finish(S, FX_MAX_ITERATIONS, 0, sqrt(v[2]));
        else if (sqrt(v[2]) < S->tol) st_finish(S, FX_CONVERGED, 0, sqrt(v[2]));
        else pipe_scalars(S);
    }
};

// One iteration after m = M w: n = A m on the fly, the 8-way update, and (r.u, w.u, r.r) of the
// updated vectors for the next iteration's scalars and stop test.
template <typename T, int MODE>
struct PtPpcgIter {
    static constexpr int NA = 8;
    OpA<T, MODE> A;
    T *z, *q, *sv, *p, *x, *r, *u, *w;
    const DevState *S;
    T alpha, beta;
    __device__ __forceinline__ void prepare() {
        alpha = (T)S->alpha;
        beta = (T)S->beta;
    }
    __device__ __forceinline__ const T *aux(int k) const {
        return k == 0 ? z : k == 1 ? q : k == 2 ? sv : k == 3 ? p : k == 4 ? x : k == 5 ? r : k == 6 ? u : w;
    }
    __device__ __forceinline__ void operator()(bool ring, int rr, int c, size_t idx, const Nb<T> &nb, const T *a, CSum *acc) const {
        const T n = A.apply(ring, nb, idx);
        const T m = nb.c;
        const T zn = n + a[0] * beta;
        const T qn = m + a[1] * beta;
        const T sn = a[7] + a[2] * beta;
        const T pn = a[6] + a[3] * beta;
        const T rn = fx_fma(-alpha, sn, a[5]);
        const T un = fx_fma(-alpha, qn, a[6]);
        const T wn = fx_fma(-alpha, zn, a[7]);
        z[idx] = zn;
        q[idx] = qn;
        sv[idx] = sn;
        p[idx] = pn;
        x[idx] = fx_fma(alpha, pn, a[4]);
        r[idx] = rn;
        u[idx] = un;
        w[idx] = wn;
        csum_fma(acc[0], (double)rn, (double)un);
        csum_fma(acc[1], (double)wn, (double)un);
        csum_fma(acc[2], (double)rn, (double)rn);
    }
};

struct FinPpcgIter {
    DevState *S;
    __device__ void operator()(const double *v) const {
        S->gamma_prev = S->gamma;
        S->alpha_prev = S->alpha;
        S->gamma = v[0];
        S->delta = v[1];
        S->rr = v[2];
        S->iter += 1;
        S->resid = sqrt(v[2]);
        if (S->iter >= S->max_iter) st_finish(S, FX_MAX_ITERATIONS, S->max_iter, sqrt(v[2]));
        else if (sqrt(v[2]) < S->tol) st_finish(S, FX_CONVERGED, S->iter, sqrt(v[2]));
        else pipe_scalars(S);
    }
};

template <int MODE>
int ppcg_solve_impl(fx_pipelined_cg *s, fx_buf *x, const fx_buf *b, double coeff, const StencilP &P,
                    fx_precond *pc) {
    using T = double;
    fx_ctx *ctx = s->ctx;
    const size_t RR = s->g.rows, CC = s->g.cols, n = RR * CC;
    while (s->bufs.size() < 8) {  // u and q join the unpreconditioned solver's vectors
        fx_buf *nb = nullptr;
        FX_TRY(fx_alloc(ctx, n, FX_F64, &nb));
        s->bufs.push_back(nb);
    }
    OpA<T, MODE> A{P, (T)coeff, (int)RR, (int)CC};
    T *r = (T *)s->bufs[0]->ptr, *p = (T *)s->bufs[1]->ptr, *sv = (T *)s->bufs[2]->ptr, *z = (T *)s->bufs[3]->ptr;
    T *w = (T *)s->bufs[4]->ptr, *m = (T *)s->bufs[5]->ptr, *u = (T *)s->bufs[6]->ptr, *q = (T *)s->bufs[7]->ptr;
    T *xp = (T *)x->ptr;
    const T *bp = (const T *)b->ptr;
    DevState *S = s->d_st;
    const int *halt = &S->halt;
    fx_buf rb{ctx, r, n, FX_F64, false}, ub{ctx, u, n, FX_F64, false};
    fx_buf wb{ctx, w, n, FX_F64, false}, mb{ctx, m, n, FX_F64, false};
    // out = M in from a zero initial guess (z.fill(0); pc.apply(z, r), cg.rs:196-197)
    const bool reuse = pc->fills_from_zero(&mb);
    auto precondition = [&](fx_buf *out, const fx_buf *in, const int *skip) -> int {
        if (!reuse) FX_TRY(zero_fill<T>(ctx, (T *)out->ptr, n, skip));
        return pc->apply(out, in, skip, true);
    };
    FX_TRY(s->reset_state());
    if (reuse) {  // rings stay zero from here on
        FX_CUDA(cudaMemsetAsync(u, 0, n * sizeof(T), ctx->stream));
        FX_CUDA(cudaMemsetAsync(m, 0, n * sizeof(T), ctx->stream));
    }
    FX_TRY((launch_pt<T, 0>(ctx, RR, CC, Ld1<T>{xp}, PtPipeInitQ<T, MODE>{A, bp, r}, NoFin{}, nullptr, "ppcg_init_r")));
    FX_TRY(precondition(&ub, &rb, nullptr));
    FX_TRY((launch_pt<T, 3>(ctx, RR, CC, Ld1<T>{u}, PtPpcgInitW<T, MODE>{A, r, w, p, sv, z, q}, FinPpcgInit{S},
                                  nullptr, "ppcg_init_w")));
    auto step = [&](size_t) -> int {
        FX_TRY(precondition(&mb, &wb, halt));
        return launch_pt<T, 3>(ctx, RR, CC, Ld1<T>{m}, PtPpcgIter<T, MODE>{A, z, q, sv, p, xp, r, u, w, S},
                                     FinPpcgIter{S}, halt, "ppcg_iter");
    };
    return s->drive(step, s->max_iter + 1, true);
}

// ------------------------------------------------ mixed-precision iterative refinement
//
// New (the reference has no refinement loop): FP64 iterative refinement around FP32
// preconditioned CG.  FP64 appears only in the outer residual r = b - A x (with its norm) and
// the update x += d; the inner solve A d = r runs on FP32 vectors with an FP32 V-cycle, its inner
// products and scalars still compensated FP64.

template <int MODE>
struct PtIrResid {  // r32 = (float)(b - A x), computed in FP64; reduction ||b - A x||^2
    static constexpr int NA = 1;
    OpA<double, MODE> A;
    const double *b;
    float *r32;
    __device__ __forceinline__ const double *aux(int) const { return b; }
    __device__ __forceinline__ void operator()(bool ring, int rr, int c, size_t idx, const Nb<double> &nb,
                                               const double *a, CSum *acc) const {
        const double rv = fx_fma(-1.0, A.apply(ring, nb, idx), a[0]);
        r32[idx] = (float)rv;
        csum_fma(acc[0], rv, rv);
    }
};

struct FlatIrUpdate {  // x += (double)d
    double *x;
    const float *d;
    __device__ __forceinline__ void operator()(size_t i, CSum *) const { x[i] = x[i] + (double)d[i]; }
};

}  // namespace

struct fx_ir : SolverBase {
    // bufs (F32): 0 r32 (outer residual, the inner right-hand side), 1 d (the correction)
    double inner_tol = 1e-4;  // inner stop: ||r_inner|| < inner_tol * ||r_outer||
    size_t inner_max_iter = 100;
    fx_cg *inner = nullptr;  // FP32 preconditioned CG
    size_t inner_total = 0;
    ~fx_ir() override { delete inner; }
};

namespace {

template <int MODE>
int ir_solve_impl(fx_ir *s, fx_buf *x, const fx_buf *b, double coeff, const fx_stencil *st, const fx_boundaries *bc,
                  const StencilP &P, fx_precond *pc) {
    fx_ctx *ctx = s->ctx;
    const size_t RR = s->g.rows, CC = s->g.cols, n = RR * CC;
    OpA<double, MODE> A{P, coeff, (int)RR, (int)CC};
    float *r32 = (float *)s->bufs[0]->ptr, *d = (float *)s->bufs[1]->ptr;
    double *xp = (double *)x->ptr;
    const double *bp = (const double *)b->ptr;
    s->inner_total = 0;
    DevState &H = *s->h_st;
    std::memset(&H, 0, sizeof(H));
    for (size_t k = 0;; k++) {
        FX_TRY((launch_pt<double, 1>(ctx, RR, CC, Ld1<double>{xp}, PtIrResid<MODE>{A, bp, r32},
                                          StoreFin<1>{ctx->d_result}, nullptr, "ir_residual")));
        double rr = 0;
        FX_TRY(read_results(ctx, 1, &rr));
        const double rnorm = std::sqrt(rr);
        H.iter = (long long)k;
        H.resid = rnorm;
        if (k == 0) H.r0 = rnorm;
        if (rnorm < s->tol) {
            H.reason = FX_CONVERGED;
            return FX_OK;
        }
        if (!std::isfinite(rnorm)) {  // NaN / Inf: stop with Breakdown rather than run to max_outer
            H.reason = FX_BREAKDOWN;
            return FX_OK;
        }
        if (k >= s->max_iter) {
            H.reason = FX_MAX_ITERATIONS;
            return FX_OK;
        }
        FX_CUDA(cudaMemsetAsync(d, 0, n * sizeof(float), ctx->stream));
        s->inner->tol = s->inner_tol * rnorm;
        s->inner->max_iter = s->inner_max_iter;
        FX_TRY((cg_solve_impl<float, MODE>(s->inner, s->bufs[1], s->bufs[0], coeff, P, pc)));
        s->inner_total += (size_t)s->inner->h_st->iter;
        if (s->inner->h_st->reason == FX_BREAKDOWN && s->inner->h_st->iter == 0) {
            H.reason = FX_BREAKDOWN;
            return FX_OK;
        }
        FX_TRY(launch_flat<0>(ctx, n, FlatIrUpdate{xp, d}, NoFin{}, nullptr, "ir_update"));
    }
    (void)st;
    (void)bc;
}

// ------------------------------------------------ BiCGSTAB (bicgstab.rs:90-346)

__device__ __forceinline__ void bicg_top(DevState *S, double rr, double rho_new) {
    // loop-top of iteration S->iter: ||r|| test, rho = r_hat.r breakdown test, beta
    const double r_norm = sqrt(rr);
    S->r_norm = r_norm;
    S->resid = r_norm;
    if (S->iter >= S->max_iter) {
        st_finish(S, FX_MAX_ITERATIONS, S->max_iter, r_norm);
        return;
    }
    if (r_norm < S->tol) {
        st_finish(S, FX_CONVERGED, S->iter, r_norm);
        return;
    }
    S->rho_new = rho_new;
    if (fabs(rho_new) < 1e-30) {
        st_finish(S, FX_BREAKDOWN, S->iter, r_norm);
        return;
    }
    S->beta = (rho_new / S->rho) * (S->alpha / S->omega);
}

struct FinBicgInit {
    DevState *S;
    __device__ void operator()(const double *v) const {
        S->rho = 1.0;
        S->alpha = 1.0;
        S->omega = 1.0;
        S->iter = 0;
        S->r0 = sqrt(v[0]);
        bicg_top(S, v[0], v[1]);
    }
};

// p_new = r + beta (p_old - omega v_old), rounded as p.axpy(-omega, v); p.scale(beta); p.axpy(1, r)
template <typename T>
struct LdBicgP {
    static constexpr int NL = 3;
    const T *r, *p, *v;
    const DevState *S;
    T beta, omega;
    __device__ __forceinline__ void prepare() {
        beta = (T)S->beta;
        omega = (T)S->omega;
    }
    __device__ __forceinline__ void load(size_t i, T (&x)[3]) const {
        x[0] = r[i];
        x[1] = p[i];
        x[2] = v[i];
    }
    __device__ __forceinline__ T combine(const T (&x)[3]) const { return x[0] + fx_fma(-omega, x[2], x[1]) * beta; }
};

// v = A (p or p_hat); store p_new when marching the fused p; reduction r_hat.v
template <typename T, int MODE>
struct PtBicgV {
    static constexpr int NA = 1;
    OpA<T, MODE> A;
    T *p_store;  // null when the marched field is already stored (p_hat)
    T *v;
    const T *r_hat;
    __device__ __forceinline__ const T *aux(int) const { return r_hat; }
    __device__ __forceinline__ void operator()(bool ring, int rr, int c, size_t idx, const Nb<T> &nb, const T *a, CSum *acc) const {
        if (p_store) p_store[idx] = nb.c;
        const T vv = A.apply(ring, nb, idx);
        v[idx] = vv;
        csum_add_prod(acc[0], (double)a[0], (double)vv);
    }
};

struct FinBicgRv {
    DevState *S;
    __device__ void operator()(const double *v) const {
        const double rv = v[0];
        if (fabs(rv) < 1e-30) {
            st_finish(S, FX_BREAKDOWN, S->iter, S->r_norm);
            return;
        }
        S->alpha = S->rho_new / rv;
    }
};

struct FinBicgS {
    DevState *S;
    __device__ void operator()(const double *v) const {
        S->s_norm = sqrt(v[0]);
        if (S->s_norm < S->tol) {
            S->pending = 1;
            S->halt = 1;
        }
    }
};

// t = A (s or s_hat); reductions (t.s, t.t)
template <typename T, int MODE>
struct PtBicgT {
    static constexpr int NA = 1;
    OpA<T, MODE> A;
    T *t;
    const T *s;
    __device__ __forceinline__ const T *aux(int) const { return s; }
    __device__ __forceinline__ void operator()(bool ring, int rr, int c, size_t idx, const Nb<T> &nb, const T *a, CSum *acc) const {
        const T tv = A.apply(ring, nb, idx);
        t[idx] = tv;
        csum_add_prod(acc[0], (double)tv, (double)a[0]);
        csum_add_prod(acc[1], (double)tv, (double)tv);
    }
};

struct FinBicgT {
    DevState *S;
    __device__ void operator()(const double *v) const {
        const double ts = v[0], tt = v[1];
        if (fabs(tt) < 1e-30) {
            S->pending = 2;
            S->halt = 1;
            return;
        }
        S->omega = ts / tt;
    }
};

struct FinBicgEnd {
    DevState *S;
    __device__ void operator()(const double *v) const {
        if (S->pending) {
            st_finish(S, S->pending == 1 ? FX_CONVERGED : FX_BREAKDOWN, S->iter, S->s_norm);
            return;
        }
        S->rho = S->rho_new;
        S->iter += 1;
        bicg_top(S, v[0], v[1]);
    }
};

// s = r - alpha v; reduction s.s (bicgstab.rs:159-164)
template <typename T>
struct FlatBicgS {
    const T *r, *v;
    T *s;
    const DevState *S;
    T alpha;
    __device__ __forceinline__ void prepare() { alpha = (T)S->alpha; }
    __device__ __forceinline__ void operator()(size_t i, CSum *acc) const {
        const T sv = fx_fma(-alpha, v[i], r[i]);
        s[i] = sv;
        csum_add_prod(acc[0], (double)sv, (double)sv);
    }
};

// x += alpha pp + omega ss; r = s - omega t; reductions (r.r, r_hat.r) (bicgstab.rs:193-201).
// With a pending early exit only x += alpha pp is due (bicgstab.rs:165-172, :183-190).
template <typename T>
struct FlatBicgFinish {
    T *x, *r;
    const T *pp, *ss, *t, *s, *rh;
    const DevState *S;
    T alpha, omega;
    int pending;
    __device__ __forceinline__ void prepare() {
        alpha = (T)S->alpha;
        omega = (T)S->omega;
        pending = S->pending;
    }
    __device__ __forceinline__ void operator()(size_t i, CSum *acc) const {
        if (pending) {
            x[i] = fx_fma(alpha, pp[i], x[i]);
            return;
        }
        x[i] = fx_fma(omega, ss[i], fx_fma(alpha, pp[i], x[i]));
        const T rv = fx_fma(-omega, t[i], s[i]);
        r[i] = rv;
        csum_add_prod(acc[0], (double)rv, (double)rv);
        csum_add_prod(acc[1], (double)rh[i], (double)rv);
    }
};

// p = r + beta (p - omega v) in place (bicgstab.rs:266-269)
template <typename T>
struct FlatBicgP {
    T *p;
    const T *r, *v;
    const DevState *S;
    T beta, omega;
    __device__ __forceinline__ void prepare() {
        beta = (T)S->beta;
        omega = (T)S->omega;
    }
    __device__ __forceinline__ void operator()(size_t i, CSum *) const {
        p[i] = r[i] + fx_fma(-omega, v[i], p[i]) * beta;
    }
};

// r = b - A x; r_hat = r; reductions (r.r, r_hat.r)
template <typename T, int MODE>
struct PtBicgInit {
    static constexpr int NA = 1;
    OpA<T, MODE> A;
    const T *b;
    T *r, *rh;
    __device__ __forceinline__ const T *aux(int) const { return b; }
    __device__ __forceinline__ void operator()(bool ring, int rr, int c, size_t idx, const Nb<T> &nb, const T *a, CSum *acc) const {
        const T rv = fx_fma((T)-1, A.apply(ring, nb, idx), a[0]);
        r[idx] = rv;
        rh[idx] = rv;
        csum_add_prod(acc[0], (double)rv, (double)rv);
        csum_add_prod(acc[1], (double)rv, (double)rv);
    }
};

}  // namespace

struct fx_bicgstab : SolverBase {
    // bufs: 0 r, 1 r_hat, 2 p0, 3 p1, 4 v0, 5 v1, 6 s, 7 t, 8 ph, 9 sh
};

namespace {

template <int MODE>
int bicg_solve_impl(fx_bicgstab *s, fx_buf *x, const fx_buf *b, double coeff, const StencilP &P, fx_precond *pc) {
    using T = double;
    fx_ctx *ctx = s->ctx;
    const size_t RR = s->g.rows, CC = s->g.cols;
    const auto A = OpMaker<T, MODE>::make(P, coeff, RR, CC, s->op);
    const size_t n = s->g.rows * s->g.cols;
    T *r = (T *)s->bufs[0]->ptr, *rh = (T *)s->bufs[1]->ptr;
    T *pb[2] = {(T *)s->bufs[2]->ptr, (T *)s->bufs[3]->ptr};
    T *vb[2] = {(T *)s->bufs[4]->ptr, (T *)s->bufs[5]->ptr};
    T *sv = (T *)s->bufs[6]->ptr, *tv = (T *)s->bufs[7]->ptr, *ph = (T *)s->bufs[8]->ptr, *sh = (T *)s->bufs[9]->ptr;
    T *xp = (T *)x->ptr;
    const T *bp = (const T *)b->ptr;
    DevState *S = s->d_st;
    const int *halt = &S->halt;
    const int *done = &S->done;
    FX_TRY(s->reset_state());
    for (int k = 0; k < 2; k++) {
        FX_CUDA(cudaMemsetAsync(pb[k], 0, n * sizeof(T), ctx->stream));
        FX_CUDA(cudaMemsetAsync(vb[k], 0, n * sizeof(T), ctx->stream));
    }
    // r = b - A x; r_hat = r; (r.r, r_hat.r)
    FX_TRY((launch_pt<T, 2>(ctx, RR, CC, Ld1<T>{xp}, PtBicgInit<T, MODE>{A, bp, r, rh}, FinBicgInit{S}, nullptr,
                                  "bicg_init")));
    auto s_update = [&](const T *v) -> int {
        return launch_flat<1>(ctx, n, FlatBicgS<T>{r, v, sv, S}, FinBicgS{S}, halt, "bicg_s");
    };
    auto finish = [&](const T *pp, const T *ss) -> int {
        return launch_flat<2>(ctx, n, FlatBicgFinish<T>{xp, r, pp, ss, tv, sv, rh, S}, FinBicgEnd{S}, done,
                              "bicg_finish");
    };
    if (!pc) {
        auto step = [&](size_t i) -> int {
            T *po = pb[i & 1], *pn = pb[(i + 1) & 1], *vo = vb[i & 1], *vn = vb[(i + 1) & 1];
            FX_TRY((launch_pt<T, 1>(ctx, RR, CC, LdBicgP<T>{r, po, vo, S}, PtBicgV<T, MODE>{A, pn, vn, rh},
                                          FinBicgRv{S}, halt, "bicg_pv")));
            FX_TRY(s_update(vn));
            FX_TRY((launch_pt<T, 2>(ctx, RR, CC, Ld1<T>{sv}, PtBicgT<T, MODE>{A, tv, sv}, FinBicgT{S}, halt,
                                          "bicg_t")));
            return finish(pn, sv);
        };
        return s->drive(step, s->max_iter + 1, n >= (1u << 21));
    }
    T *p = pb[0], *v = vb[0];
    fx_buf pbuf{ctx, p, n, FX_F64, false}, phb{ctx, ph, n, FX_F64, false};
    fx_buf sbuf{ctx, sv, n, FX_F64, false}, shb{ctx, sh, n, FX_F64, false};
    auto step = [&](size_t) -> int {
        FX_TRY(launch_flat<0>(ctx, n, FlatBicgP<T>{p, r, v, S}, NoFin{}, halt, "bicg_p"));
        FX_TRY(zero_fill<T>(ctx, ph, n, halt));
        FX_TRY(pc->apply(&phb, &pbuf, halt, true));
        FX_TRY((launch_pt<T, 1>(ctx, RR, CC, Ld1<T>{ph}, PtBicgV<T, MODE>{A, nullptr, v, rh}, FinBicgRv{S}, halt,
                                      "bicg_v")));
        FX_TRY(s_update(v));
        FX_TRY(zero_fill<T>(ctx, sh, n, halt));
        FX_TRY(pc->apply(&shb, &sbuf, halt, true));
        FX_TRY((launch_pt<T, 2>(ctx, RR, CC, Ld1<T>{sh}, PtBicgT<T, MODE>{A, tv, sv}, FinBicgT{S}, halt, "bicg_t")));
        return finish(ph, sh);
    };
    return s->drive(step, s->max_iter + 1, true);
}

}  // namespace

// ------------------------------------------------ GMRES (gmres.rs:463-837)

struct fx_gmres : SolverBase {
    size_t restart = 30;
    double *d_h = nullptr;  // device column of dots
    double *h_h = nullptr;      // mapped page-locked, 2 (restart + 2) values (CGS2 reads two columns)
    double *h_h_dev = nullptr;  // its device address
    std::vector<double> hh, cc, ss, grs;
    std::vector<fx_buf *> vv;  // m+1 basis vectors (bufs[0..m]); w = bufs[m+1]
    ~fx_gmres() {
        if (d_h) cudaFree(d_h);
        if (h_h) cudaFreeHost(h_h);
    }
};

namespace {

struct FinSlot {
    double *dst;
    __device__ void operator()(const double *v) const { *dst = v[0]; }
};

template <typename T, int MODE>
struct PtGmResid {  // out = b - A x (gmres.rs:477-485); reduction out.out
    static constexpr int NA = 1;
    OpA<T, MODE> A;
    const T *b;
    T *out;
    __device__ __forceinline__ const T *aux(int) const { return b; }
    __device__ __forceinline__ void operator()(bool ring, int rr, int c, size_t idx, const Nb<T> &nb, const T *a, CSum *acc) const {
        const T ax = A.apply(ring, nb, idx);
        const T v = fx_fma((T)1, a[0], -ax);
        out[idx] = v;
        csum_add_prod(acc[0], (double)v, (double)v);
    }
};

template <typename T, int MODE, bool HAS_V0>
struct PtGmAv {  // w = A v; reduction w.v0 (when v0 given)
    static constexpr int NA = HAS_V0 ? 1 : 0;
    OpA<T, MODE> A;
    T *w;
    const T *v0;
    __device__ __forceinline__ const T *aux(int) const { return v0; }
    __device__ __forceinline__ void operator()(bool ring, int rr, int c, size_t idx, const Nb<T> &nb, const T *a, CSum *acc) const {
        const T wv = A.apply(ring, nb, idx);
        w[idx] = wv;
        if (HAS_V0) csum_add_prod(acc[0], (double)wv, (double)a[0]);
    }
};

template <typename T>
struct FlatGmBuild {  // x += y_j v_j, j in order (gmres.rs:832-835)
    T *x;
    const T *v[8];
    T y[8];
    int cnt;
    __device__ __forceinline__ void operator()(size_t i, CSum *) const {
        T xv = x[i];
        for (int j = 0; j < cnt; j++) xv = fx_fma(y[j], v[j][i], xv);
        x[i] = xv;
    }
};

template <typename T>
struct FlatGmPcCopy {  // w = M^-1 A v_k (held in src); reduction w.v0
    T *w;
    const T *src, *v0;
    __device__ __forceinline__ void operator()(size_t i, CSum *acc) const {
        const T wv = src[i];
        w[i] = wv;
        csum_add_prod(acc[0], (double)wv, (double)v0[i]);
    }
};

template <typename T>
struct FlatGmMgs {  // w -= h_j v_j; reduction w.v_{j+1} (or w.w after the last)
    T *w;
    const T *vj, *vn;
    const double *hj;
    T h;
    __device__ __forceinline__ void prepare() { h = (T)(*hj); }
    __device__ __forceinline__ void operator()(size_t i, CSum *acc) const {
        const T wv = fx_fma(-h, vj[i], w[i]);
        w[i] = wv;
        if (vn) csum_add_prod(acc[0], (double)wv, (double)vn[i]);
        else csum_add_prod(acc[0], (double)wv, (double)wv);
    }
};

template <int MODE>
int gmres_solve_impl(fx_gmres *s, fx_buf *x, const fx_buf *b, double coeff, const StencilP &P, fx_precond *pc) {
    using T = double;
    fx_ctx *ctx = s->ctx;
    const size_t RR = s->g.rows, CC = s->g.cols;
    const auto A = OpMaker<T, MODE>::make(P, coeff, RR, CC, s->op);
    const size_t n = s->g.rows * s->g.cols, m = s->restart, mp1 = m + 1;
    std::vector<T *> V(mp1);
    for (size_t i = 0; i < mp1; i++) V[i] = (T *)s->bufs[i]->ptr;
    T *w = (T *)s->bufs[mp1]->ptr;
    T *xp = (T *)x->ptr;
    const T *bp = (const T *)b->ptr;
    double *dh = s->d_h;
    auto H = [&](size_t i, size_t j) -> double & { return s->hh[j * mp1 + i]; };
    size_t total_its = 0;
    fx_stats st{0, 0.0, FX_CONVERGED};

    auto read_h = [&](size_t k) -> int {
        return read_mapped(ctx, dh, s->h_h_dev, k + 2);
    };
    auto scale_into = [&](T *dst, const T *src, double f) -> int {  // copy_from + scale(f)
        return launch_flat<0>(ctx, n, FlatScaleInto<T>{dst, src, (T)f}, NoFin{}, nullptr, "gmres_scale");
    };
    auto build_solution = [&](size_t k) -> int {  // gmres.rs:808-837
        if (k == 0) return FX_OK;
        std::vector<double> y(k, 0.0);
        for (size_t ii = k; ii-- > 0;) {
            double sacc = s->grs[ii];
            for (size_t j = ii + 1; j < k; j++) sacc -= s->hh[j * mp1 + ii] * y[j];
            const double diag = s->hh[ii * mp1 + ii];
            if (std::fabs(diag) < 1e-30) break;
            y[ii] = sacc / diag;
        }
        // x += y_i v_i in order i = 0..k-1, one pass (same per-element sequence of fma)
        for (size_t i0 = 0; i0 < k; i0 += 8) {
            const size_t cnt = std::min<size_t>(8, k - i0);
            FlatGmBuild<T> fb;
            fb.x = xp;
            for (size_t j = 0; j < cnt; j++) {
                fb.v[j] = V[i0 + j];
                fb.y[j] = (T)y[i0 + j];
            }
            fb.cnt = (int)cnt;
            FX_TRY(launch_flat<0>(ctx, n, fb, NoFin{}, nullptr, "gmres_build"));
        }
        return FX_OK;
    };
    fx_buf wb{ctx, w, n, FX_F64, false};
    for (;;) {
        double beta;
        if (!pc) {
            FX_TRY((launch_pt<T, 1>(ctx, RR, CC, Ld1<T>{xp}, PtGmResid<T, MODE>{A, bp, V[0]}, FinSlot{dh}, nullptr,
                                          "gmres_resid")));
            FX_TRY(read_h(0));
            beta = std::sqrt(s->h_h[0]);
        } else {
            FX_TRY((launch_pt<T, 0>(ctx, RR, CC, Ld1<T>{xp}, PtGmResid<T, MODE>{A, bp, w}, NoFin{}, nullptr, "gmres_resid")));
            fx_buf v0b{ctx, V[0], n, FX_F64, false};
            FX_TRY(zero_fill<T>(ctx, V[0], n, nullptr));
            FX_TRY(pc->apply(&v0b, &wb, nullptr, true));
            T *v0 = V[0];
            FX_TRY(launch_flat<1>(ctx, n, FlatDot<T>{v0, v0}, FinSlot{dh}, nullptr, "gmres_beta"));
            FX_TRY(read_h(0));
            beta = std::sqrt(s->h_h[0]);
        }
        if (beta < s->tol) {
            st = {total_its, beta, FX_CONVERGED};
            break;
        }
        if (!std::isfinite(beta)) {  // NaN / Inf in b, x or the operator: Breakdown, not max_iter
            st = {total_its, beta, FX_BREAKDOWN};
            break;
        }
        FX_TRY(scale_into(V[0], V[0], 1.0 / beta));
        std::fill(s->grs.begin(), s->grs.end(), 0.0);
        s->grs[0] = beta;
        std::fill(s->hh.begin(), s->hh.end(), 0.0);
        double cur_resid = beta;
        size_t k = 0;
        bool finished = false;
        while (k < m) {
            if (total_its >= s->max_iter) {
                FX_TRY(build_solution(k));
                st = {total_its, cur_resid, FX_MAX_ITERATIONS};
                finished = true;
                break;
            }
            // w = A v_k (+ left preconditioning), then modified Gram-Schmidt with every dot
            // fused into the preceding AXPY
            if (!pc) {
                FX_TRY((launch_pt<T, 1>(ctx, RR, CC, Ld1<T>{V[k]}, PtGmAv<T, MODE, true>{A, w, V[0]}, FinSlot{dh + 0}, nullptr,
                                              "gmres_av")));
            } else {
                FX_TRY((launch_pt<T, 0>(ctx, RR, CC, Ld1<T>{V[k]}, PtGmAv<T, MODE, false>{A, w, nullptr}, NoFin{}, nullptr,
                                              "gmres_av")));
                fx_buf vk1{ctx, V[k + 1], n, FX_F64, false};
                FX_TRY(zero_fill<T>(ctx, V[k + 1], n, nullptr));
                FX_TRY(pc->apply(&vk1, &wb, nullptr, true));
                T *src = V[k + 1], *v0 = V[0];
                FX_TRY(launch_flat<1>(ctx, n, FlatGmPcCopy<T>{w, src, v0}, FinSlot{dh + 0}, nullptr, "gmres_pc_copy"));
            }
            for (size_t j = 0; j <= k; j++) {
                const T *vj = V[j];
                const T *vn = j < k ? V[j + 1] : nullptr;
                const double *hj = dh + j;
                FX_TRY(launch_flat<1>(ctx, n, FlatGmMgs<T>{w, vj, vn, hj}, FinSlot{dh + j + 1}, nullptr, "gmres_mgs"));
            }
            FX_TRY(read_h(k));
            for (size_t j = 0; j <= k; j++) H(j, k) = s->h_h[j];
            const double h_kp1_k = std::sqrt(s->h_h[k + 1]);
            H(k + 1, k) = h_kp1_k;
            if (h_kp1_k > 1e-30) FX_TRY(scale_into(V[k + 1], w, 1.0 / h_kp1_k));
            for (size_t j = 0; j < k; j++) {
                const double h_j = H(j, k), h_jp1 = H(j + 1, k), cj = s->cc[j], sj = s->ss[j];
                H(j, k) = std::fma(cj, h_j, sj * h_jp1);
                H(j + 1, k) = std::fma(cj, h_jp1, -sj * h_j);
            }
            const double a = H(k, k), bv = H(k + 1, k);
            const double rr = std::hypot(a, bv);
            if (std::fabs(rr) < 1e-30) {
                FX_TRY(build_solution(k));
                st = {total_its, cur_resid, FX_BREAKDOWN};
                finished = true;
                break;
            }
            s->cc[k] = a / rr;
            s->ss[k] = bv / rr;
            H(k, k) = rr;
            H(k + 1, k) = 0.0;
            const double g_k = s->grs[k];
            s->grs[k] = s->cc[k] * g_k;
            s->grs[k + 1] = -s->ss[k] * g_k;
            cur_resid = std::fabs(s->grs[k + 1]);
            total_its++;
            k++;
            if (!std::isfinite(cur_resid)) {
                st = {total_its, cur_resid, FX_BREAKDOWN};
                finished = true;
                break;
            }
            if (cur_resid < s->tol) break;
            if (h_kp1_k <= 1e-30) break;
        }
        if (finished) break;
        FX_TRY(build_solution(k));
        if (cur_resid < s->tol) {
            st = {total_its, cur_resid, FX_CONVERGED};
            break;
        }
        if (total_its >= s->max_iter) {
            st = {total_its, cur_resid, FX_MAX_ITERATIONS};
            break;
        }
    }
    s->h_st->iter = (long long)st.iterations;
    s->h_st->resid = st.residual;
    s->h_st->reason = st.reason;
    FX_CUDA(cudaStreamSynchronize(ctx->stream));
    return FX_OK;
}

template <typename Solver>
int create_solver(fx_ctx *ctx, const fx_grid *g, double tol, size_t max_iter, int nvec, Solver **out,
                  int dtype = FX_F64) {
    if (!ctx || !out) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    FX_TRY(check_grid(g));
    *out = nullptr;
    Solver *s = new Solver();
    int st = s->init_base(ctx, g, tol, max_iter, nvec, dtype);
    if (st) {
        delete s;
        return st;
    }
    *out = s;
    return FX_OK;
}

// ------------------------------------------------ flexible CG (new; no reference solver)
//
// PCG whose beta is the Polak-Ribiere form z_{k+1}.(r_{k+1} - r_k) / (z_k.r_k) (Golub & Ye 1999;
// Notay's FCG(1), 2000), evaluated as (r_{k+1}.z_{k+1} - r_k.z_{k+1}) / rz_old, so that a
// preconditioner that changes between applications (an inner iterative solve) keeps the
// directions locally A-orthogonal.  Per iteration: pcg_dir and an update pass that writes
// r_{k+1} beside r_k (the two residual buffers swap roles), z = M^-1 r_{k+1} through the
// preconditioner's plain apply, and one pass for both inner products.

template <typename T, int MODE>
struct PtFcgUpd {  // x += alpha p; r_out = r_in - alpha A p, r_in kept; reduction r_out.r_out
    static constexpr int NA = 2;
    OpA<T, MODE> A;
    T *x;
    const T *r_in;
    T *r_out;
    const DevState *S;
    T alpha;
    __device__ __forceinline__ void prepare() { alpha = (T)S->alpha; }
    __device__ __forceinline__ const T *aux(int k) const { return k == 0 ? x : r_in; }
    __device__ __forceinline__ void operator()(bool ring, int rr, int c, size_t idx, const Nb<T> &nb, const T *a, CSum *acc) const {
        const T ap = A.apply(ring, nb, idx);
        x[idx] = fx_fma(alpha, nb.c, a[0]);
        const T rv = fx_fma(-alpha, ap, a[1]);
        r_out[idx] = rv;
        csum_fma(acc[0], (double)rv, (double)rv);
    }
};

// (r_new.z, r_prev.z) with exact products: the second is near zero by construction
template <typename T>
struct FlatFcgDots {
    const T *r_new, *r_prev, *z;
    __device__ __forceinline__ void operator()(size_t i, CSum *acc) const {
        const double zv = (double)z[i];
        csum_add_prod(acc[0], (double)r_new[i], zv);
        csum_add_prod(acc[1], (double)r_prev[i], zv);
    }
};

struct FinFcgBeta {  // beta = (r_new.z - r_prev.z) / rz_old; rz_old = r_new.z
    DevState *S;
    __device__ void operator()(const double *v) const {
        S->beta = (v[0] - v[1]) / S->rs_old;
        S->rs_old = v[0];
    }
};

}  // namespace

struct fx_fcg : SolverBase {
    // bufs: 0, 1 residuals (current / previous, swapped every iteration), 2 z, 3, 4 directions
};

namespace {

template <int MODE>
int fcg_solve_impl(fx_fcg *s, fx_buf *x, const fx_buf *b, double coeff, const StencilP &P, fx_precond *pc) {
    using T = double;
    fx_ctx *ctx = s->ctx;
    const size_t RR = s->g.rows, CC = s->g.cols, n = RR * CC;
    OpA<T, MODE> A{P, (T)coeff, (int)RR, (int)CC};
    T *rb[2] = {(T *)s->bufs[0]->ptr, (T *)s->bufs[1]->ptr};
    T *z = (T *)s->bufs[2]->ptr;
    T *pb[2] = {(T *)s->bufs[3]->ptr, (T *)s->bufs[4]->ptr};
    T *xp = (T *)x->ptr;
    const T *bp = (const T *)b->ptr;
    DevState *S = s->d_st;
    const int *halt = &S->halt;
    FX_TRY(s->reset_state());
    FX_CUDA(cudaMemsetAsync(pb[0], 0, n * sizeof(T), ctx->stream));
    FX_CUDA(cudaMemsetAsync(pb[1], 0, n * sizeof(T), ctx->stream));
    FX_TRY((launch_pt<T, 1>(ctx, RR, CC, Ld1<T>{xp}, PtInitResid<T, MODE>{A, bp, rb[0], nullptr}, FinPcgResid{S},
                               nullptr, "fcg_init")));
    fx_buf zb{ctx, z, n, FX_F64, false};
    auto precondition = [&](T *r) -> int {  // z = M^-1 r from a zero z
        fx_buf rbuf{ctx, r, n, FX_F64, false};
        FX_TRY(zero_fill<T>(ctx, z, n, halt));
        return pc->apply(&zb, &rbuf, halt, true);
    };
    FX_TRY(precondition(rb[0]));
    FX_TRY(launch_flat<1>(ctx, n, FlatDot<T>{rb[0], z}, FinPcgRzInit{S}, halt, "fcg_rz"));
    auto step = [&](size_t i) -> int {
        T *po = pb[i & 1], *pn = pb[(i + 1) & 1];
        T *rc = rb[i & 1], *rn = rb[(i + 1) & 1];
        FX_TRY((launch_pt<T, 1>(ctx, RR, CC, LdAypx<T>{z, po, S}, PtCgDir<T, MODE>{A, pn}, FinCgDir{S}, halt,
                                   "fcg_dir")));
        FX_TRY((launch_pt<T, 1>(ctx, RR, CC, Ld1<T>{pn}, PtFcgUpd<T, MODE>{A, xp, rc, rn, S}, FinPcgUpd{S}, halt,
                                   "fcg_update")));
        FX_TRY(precondition(rn));
        return launch_flat<2>(ctx, n, FlatFcgDots<T>{rn, rc, z}, FinFcgBeta{S}, halt, "fcg_beta");
    };
    return s->drive(step, s->max_iter + 1, n >= (1u << 20));
}

// ------------------------------------------------ flexible GMRES(m) (new; Saad 1993)
//
// Right preconditioning with the preconditioned directions kept: z_k = M_k^-1 v_k,
// w = A z_k, then the same fused modified Gram-Schmidt, host Givens rotations and restarts as
// GMRES; the Givens estimate is the true ||b - A x||, and a cycle ends with x += Z y.  Without
// a preconditioner z_k is v_k itself, and the method is GMRES step for step.

}  // namespace

struct fx_fgmres : fx_gmres {
    // bufs: 0..m the basis V, m+1 w, m+2 .. 2m+1 the directions Z
    bool cgs2 = false;               // fx_fgmres_set_orthogonalization
    double *d_cgs = nullptr;         // [2 (restart + 2)]: the two passes' coefficients
    double *d_part = nullptr;        // [blocks][kCgsMax] block partials of the multi-dot
    unsigned *d_ticket = nullptr;
    ~fx_fgmres() {
        if (d_cgs) cudaFree(d_cgs);
        if (d_part) cudaFree(d_part);
        if (d_ticket) cudaFree(d_ticket);
    }
};

namespace {

// ------------------------------------------------ classical Gram-Schmidt, twice (CGS2), for FGMRES
//
// Option (fx_fgmres_set_orthogonalization): the Arnoldi step orthogonalises w against the whole
// basis v_0 .. v_k in three passes, each reading w and the basis once, instead of one modified
// Gram-Schmidt pass per basis vector:
//   pass 0: h1_j = v_j . w
//   pass 1: w -= sum_j h1_j v_j, then h2_j = v_j . w (the same pass, from the updated element)
//   pass 2: w -= sum_j h2_j v_j, then ||w||^2
// and h_jk = h1_j + h2_j (Giraud, Langou, Rozloznik 2005: twice is enough).  The sums of a pass are
// per-thread FP64 partials folded in a fixed order (block, then the blocks by a last-block
// ticket), so the coefficients are deterministic.
constexpr int kCgsMax = 32;  // basis vectors per pass (restart <= 32)

struct CgsArgs {
    double *w;
    const double *v[kCgsMax];
    int kb;                  // basis vectors v_0 .. v_{kb-1}
    const double *coef;      // pass 1 / 2: the coefficients subtracted
    double *out;             // pass 0 / 1: kb dots; pass 2: out[0] = ||w||^2
    double *part;
    unsigned *ticket;
};

// The grid walks tiles of 2 kBlock elements.  In a tile, thread t first owns elements t and
// t + kBlock: in passes 1 and 2 it reads w and the basis once and writes the updated w (loads in
// batches of 8 per element, all issued before the first use).  For the multi-dot (passes 0 and 1)
// warp q then owns the basis vectors j = q, q + 8, q + 16, q + 24 and lane l the tile's elements
// l, l + 32, ..., two rows of 32 per step, with w from shared memory: a thread keeps four partial
// sums, so the kernel needs few registers and many resident warps keep the loads in flight.  (One
// element and 32 partial sums per thread measured 0.42 of HBM bandwidth, latency-bound at 16
// warps per SM; one element per thread and tile, 0.63.)  The sums of a basis vector are
// added in a fixed order: over a warp's tiles, the lanes' shuffle tree, then the blocks.
template <int PASS>
__global__ void __launch_bounds__(kBlock) k_cgs(size_t n, CgsArgs a) {
    grid_dep_enter();
    constexpr int kW = kBlock / 32;     // warps per block
    constexpr int kJ = kCgsMax / kW;    // basis vectors per warp in the multi-dot
    constexpr int kB = 8;               // loads per batch in the update
    const int kb = a.kb, ns = PASS == 2 ? 1 : kb;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __shared__ double c[kCgsMax];
    __shared__ const double *vp[kCgsMax];
    constexpr int kU = 2;               // elements per thread in a tile (both phases keep 2x the loads in flight)
    constexpr int kTile = kU * kBlock;
    __shared__ double sw[kTile];
    __shared__ double red[kW];
    __shared__ bool is_last;
    if (threadIdx.x < kCgsMax) {
        c[threadIdx.x] = (PASS > 0 && threadIdx.x < kb) ? a.coef[threadIdx.x] : 0.0;
        vp[threadIdx.x] = threadIdx.x < kb ? a.v[threadIdx.x] : nullptr;
    }
    __syncthreads();
    double acc[kJ];
#pragma unroll
    for (int q = 0; q < kJ; q++) acc[q] = 0.0;
    const size_t ntiles = (n + kTile - 1) / kTile;
    for (size_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const size_t i0 = tile * kTile;
        double wv[kU];
#pragma unroll
        for (int u = 0; u < kU; u++) {
            const size_t i = i0 + u * kBlock + threadIdx.x;
            wv[u] = i < n ? a.w[i] : 0.0;
        }
        if (PASS > 0) {
#pragma unroll
            for (int j0 = 0; j0 < kCgsMax; j0 += kB) {
                if (j0 < kb) {
                    double vv[kU][kB];
#pragma unroll
                    for (int u = 0; u < kU; u++) {
                        const size_t i = i0 + u * kBlock + threadIdx.x;
#pragma unroll
                        for (int t = 0; t < kB; t++) vv[u][t] = (j0 + t < kb && i < n) ? vp[j0 + t][i] : 0.0;
                    }
#pragma unroll
                    for (int u = 0; u < kU; u++)
#pragma unroll
                        for (int t = 0; t < kB; t++)
                            if (j0 + t < kb) wv[u] = fma(-c[j0 + t], vv[u][t], wv[u]);
                }
            }
#pragma unroll
            for (int u = 0; u < kU; u++) {
                const size_t i = i0 + u * kBlock + threadIdx.x;
                if (i < n) a.w[i] = wv[u];
            }
        }
        if (PASS == 2) {
#pragma unroll
            for (int u = 0; u < kU; u++) acc[0] = fma(wv[u], wv[u], acc[0]);
            continue;
        }
#pragma unroll
        for (int u = 0; u < kU; u++) sw[u * kBlock + threadIdx.x] = wv[u];
        __syncthreads();
#pragma unroll
        for (int e = 0; e < kTile; e += 64) {  // two 32-element rows of the tile per step
            double vv[2][kJ], xs[2];
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const size_t ie = i0 + e + 32 * h + lane;
                xs[h] = sw[e + 32 * h + lane];
#pragma unroll
                for (int q = 0; q < kJ; q++) {
                    const int j = wid + kW * q;
                    vv[h][q] = (j < kb && ie < n) ? vp[j][ie] : 0.0;
                }
            }
#pragma unroll
            for (int h = 0; h < 2; h++)
#pragma unroll
                for (int q = 0; q < kJ; q++)
                    if (wid + kW * q < kb && i0 + e + 32 * h + lane < n) acc[q] = fma(vv[h][q], xs[h], acc[q]);
        }
        __syncthreads();  // sw is rewritten by the next tile
    }
    // block partials: basis vector j is one warp's (a shuffle tree); ||w||^2 is every thread's
    if (PASS == 2) {
        double v = acc[0];
        for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
        if (lane == 0) red[wid] = v;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0.0;
            for (int k = 0; k < kW; k++) t += red[k];
            a.part[(size_t)blockIdx.x * kCgsMax] = t;
        }
    } else {
#pragma unroll
        for (int q = 0; q < kJ; q++) {
            double v = acc[q];
            for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
            const int j = wid + kW * q;
            if (lane == 0 && j < kb) a.part[(size_t)blockIdx.x * kCgsMax + j] = v;
        }
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) is_last = atomicAdd(a.ticket, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    // last block: warp w folds sums j = w, w + 8, ...; lane l takes blocks l, l + 32, ... (four
    // loads in flight), then a fixed shuffle tree merges the lanes' compensated sums
    const unsigned nb = gridDim.x;
    for (int j = wid; j < ns; j += kW) {
        CSum t{0.0, 0.0};
        unsigned bb = lane;
        for (; bb + 96 < nb; bb += 128) {
            const double p0 = __ldcg(a.part + (size_t)bb * kCgsMax + j);
            const double p1 = __ldcg(a.part + (size_t)(bb + 32) * kCgsMax + j);
            const double p2 = __ldcg(a.part + (size_t)(bb + 64) * kCgsMax + j);
            const double p3 = __ldcg(a.part + (size_t)(bb + 96) * kCgsMax + j);
            csum_add(t, p0);
            csum_add(t, p1);
            csum_add(t, p2);
            csum_add(t, p3);
        }
        for (; bb < nb; bb += 32) csum_add(t, __ldcg(a.part + (size_t)bb * kCgsMax + j));
        for (int off = 16; off > 0; off >>= 1) {
            CSum o;
            o.s = __shfl_down_sync(0xffffffffu, t.s, off);
            o.c = __shfl_down_sync(0xffffffffu, t.c, off);
            t = csum_merge(t, o);
        }
        if (lane == 0) a.out[j] = csum_value(t);
    }
    if (threadIdx.x == 0) *a.ticket = 0u;
}

// One wave of resident blocks (at most the partial buffer's num_sms * 8 rows): the fold in the
// last block then reads a few hundred partials per sum.
template <int PASS>
int launch_cgs(fx_ctx *ctx, size_t n, const CgsArgs &a) {
    static std::atomic<int> occ_cache{0};
    int occ = occ_cache.load(std::memory_order_relaxed);
    if (!occ) {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_cgs<PASS>, kBlock, 0) != cudaSuccess || occ < 1)
            occ = 1;
        if (occ > 8) occ = 8;
        occ_cache.store(occ, std::memory_order_relaxed);
    }
    size_t blocks = (n + 2 * kBlock - 1) / (2 * kBlock);  // tiles of 2 kBlock elements
    if (blocks > (size_t)ctx->num_sms * occ) blocks = (size_t)ctx->num_sms * occ;
    if (blocks < 1) blocks = 1;
    timing_pre(ctx, "fgmres_cgs2");
    launch_pdl(ctx, k_cgs<PASS>, (int)blocks, kBlock, 0, n, a);
    timing_post(ctx, (double)n, (double)n * 8.0 * (a.kb + 1 + (PASS > 0 ? 1 : 0)));
    return check_launch(ctx, "fgmres_cgs2");
}

}  // namespace

namespace {

template <int MODE>
int fgmres_solve_impl(fx_fgmres *s, fx_buf *x, const fx_buf *b, double coeff, const StencilP &P, fx_precond *pc) {
    using T = double;
    fx_ctx *ctx = s->ctx;
    const size_t RR = s->g.rows, CC = s->g.cols;
    const auto A = OpMaker<T, MODE>::make(P, coeff, RR, CC, s->op);
    const size_t n = s->g.rows * s->g.cols, m = s->restart, mp1 = m + 1;
    std::vector<T *> V(mp1), Z(m);
    for (size_t i = 0; i < mp1; i++) V[i] = (T *)s->bufs[i]->ptr;
    T *w = (T *)s->bufs[mp1]->ptr;
    for (size_t i = 0; i < m; i++) Z[i] = pc ? (T *)s->bufs[mp1 + 1 + i]->ptr : V[i];
    T *xp = (T *)x->ptr;
    const T *bp = (const T *)b->ptr;
    double *dh = s->d_h;
    auto H = [&](size_t i, size_t j) -> double & { return s->hh[j * mp1 + i]; };
    size_t total_its = 0;
    fx_stats st{0, 0.0, FX_CONVERGED};
    auto read_h = [&](size_t k) -> int {
        return read_mapped(ctx, dh, s->h_h_dev, k + 2);
    };
    auto scale_into = [&](T *dst, const T *src, double f) -> int {
        return launch_flat<0>(ctx, n, FlatScaleInto<T>{dst, src, (T)f}, NoFin{}, nullptr, "fgmres_scale");
    };
    auto build_solution = [&](size_t k) -> int {  // x += Z y (gmres.rs:808-837 with Z for V)
        if (k == 0) return FX_OK;
        std::vector<double> y(k, 0.0);
        for (size_t ii = k; ii-- > 0;) {
            double sacc = s->grs[ii];
            for (size_t j = ii + 1; j < k; j++) sacc -= s->hh[j * mp1 + ii] * y[j];
            const double diag = s->hh[ii * mp1 + ii];
            if (std::fabs(diag) < 1e-30) break;
            y[ii] = sacc / diag;
        }
        for (size_t i0 = 0; i0 < k; i0 += 8) {
            const size_t cnt = std::min<size_t>(8, k - i0);
            FlatGmBuild<T> fb;
            fb.x = xp;
            for (size_t j = 0; j < cnt; j++) {
                fb.v[j] = Z[i0 + j];
                fb.y[j] = (T)y[i0 + j];
            }
            fb.cnt = (int)cnt;
            FX_TRY(launch_flat<0>(ctx, n, fb, NoFin{}, nullptr, "fgmres_build"));
        }
        return FX_OK;
    };
    for (;;) {
        FX_TRY((launch_pt<T, 1>(ctx, RR, CC, Ld1<T>{xp}, PtGmResid<T, MODE>{A, bp, V[0]}, FinSlot{dh}, nullptr,
                                   "fgmres_resid")));
        FX_TRY(read_h(0));
        const double beta = std::sqrt(s->h_h[0]);
        if (beta < s->tol) {
            st = {total_its, beta, FX_CONVERGED};
            break;
        }
        if (!std::isfinite(beta)) {  // NaN / Inf in b, x or the operator: Breakdown, not max_iter
            st = {total_its, beta, FX_BREAKDOWN};
            break;
        }
        FX_TRY(scale_into(V[0], V[0], 1.0 / beta));
        std::fill(s->grs.begin(), s->grs.end(), 0.0);
        s->grs[0] = beta;
        std::fill(s->hh.begin(), s->hh.end(), 0.0);
        double cur_resid = beta;
        size_t k = 0;
        bool finished = false;
        while (k < m) {
            if (total_its >= s->max_iter) {
                FX_TRY(build_solution(k));
                st = {total_its, cur_resid, FX_MAX_ITERATIONS};
                finished = true;
                break;
            }
            if (pc) {  // z_k = M^-1 v_k from a zero z_k
                fx_buf zk{ctx, Z[k], n, FX_F64, false}, vk{ctx, V[k], n, FX_F64, false};
                FX_TRY(zero_fill<T>(ctx, Z[k], n, nullptr));
                FX_TRY(pc->apply(&zk, &vk, nullptr, true));
            }
            double h_kp1_k = 0.0;
            if (s->cgs2) {  // w = A z_k, then CGS2 (three passes over the basis)
                FX_TRY((launch_pt<T, 0>(ctx, RR, CC, Ld1<T>{Z[k]}, PtGmAv<T, MODE, false>{A, w, nullptr}, NoFin{},
                                           nullptr, "fgmres_av")));
                CgsArgs ca{};
                ca.w = w;
                ca.kb = (int)k + 1;
                for (size_t j = 0; j <= k; j++) ca.v[j] = V[j];
                ca.part = s->d_part;
                ca.ticket = s->d_ticket;
                double *h1 = s->d_cgs, *h2 = s->d_cgs + (m + 2);
                ca.out = h1;
                FX_TRY(launch_cgs<0>(ctx, n, ca));
                ca.coef = h1;
                ca.out = h2;
                FX_TRY(launch_cgs<1>(ctx, n, ca));
                ca.coef = h2;
                ca.out = h2 + k + 1;
                FX_TRY(launch_cgs<2>(ctx, n, ca));
                FX_TRY(read_mapped(ctx, s->d_cgs, s->h_h_dev, 2 * (m + 2)));
                const double *hv = s->h_h;
                for (size_t j = 0; j <= k; j++) H(j, k) = hv[j] + hv[m + 2 + j];
                h_kp1_k = std::sqrt(hv[m + 2 + k + 1]);
            } else {
                // w = A z_k with w.v_0, then modified Gram-Schmidt with each dot fused into the AXPY
                FX_TRY((launch_pt<T, 1>(ctx, RR, CC, Ld1<T>{Z[k]}, PtGmAv<T, MODE, true>{A, w, V[0]}, FinSlot{dh + 0},
                                           nullptr, "fgmres_av")));
                for (size_t j = 0; j <= k; j++) {
                    const T *vj = V[j];
                    const T *vn = j < k ? V[j + 1] : nullptr;
                    const double *hj = dh + j;
                    FX_TRY(launch_flat<1>(ctx, n, FlatGmMgs<T>{w, vj, vn, hj}, FinSlot{dh + j + 1}, nullptr,
                                          "fgmres_mgs"));
                }
                FX_TRY(read_h(k));
                for (size_t j = 0; j <= k; j++) H(j, k) = s->h_h[j];
                h_kp1_k = std::sqrt(s->h_h[k + 1]);
            }
            H(k + 1, k) = h_kp1_k;
            if (h_kp1_k > 1e-30) FX_TRY(scale_into(V[k + 1], w, 1.0 / h_kp1_k));
            for (size_t j = 0; j < k; j++) {
                const double h_j = H(j, k), h_jp1 = H(j + 1, k), cj = s->cc[j], sj = s->ss[j];
                H(j, k) = std::fma(cj, h_j, sj * h_jp1);
                H(j + 1, k) = std::fma(cj, h_jp1, -sj * h_j);
            }
            const double a = H(k, k), bv = H(k + 1, k);
            const double rr = std::hypot(a, bv);
            if (std::fabs(rr) < 1e-30) {
                FX_TRY(build_solution(k));
                st = {total_its, cur_resid, FX_BREAKDOWN};
                finished = true;
                break;
            }
            s->cc[k] = a / rr;
            s->ss[k] = bv / rr;
            H(k, k) = rr;
            H(k + 1, k) = 0.0;
            const double g_k = s->grs[k];
            s->grs[k] = s->cc[k] * g_k;
            s->grs[k + 1] = -s->ss[k] * g_k;
            cur_resid = std::fabs(s->grs[k + 1]);
            total_its++;
            k++;
            if (!std::isfinite(cur_resid)) {
                st = {total_its, cur_resid, FX_BREAKDOWN};
                finished = true;
                break;
            }
            if (cur_resid < s->tol) break;
            if (h_kp1_k <= 1e-30) break;
        }
        if (finished) break;
        FX_TRY(build_solution(k));
        if (cur_resid < s->tol) {
            st = {total_its, cur_resid, FX_CONVERGED};
            break;
        }
        if (total_its >= s->max_iter) {
            st = {total_its, cur_resid, FX_MAX_ITERATIONS};
            break;
        }
    }
    s->h_st->iter = (long long)st.iterations;
    s->h_st->resid = st.residual;
    s->h_st->reason = st.reason;
    FX_CUDA(cudaStreamSynchronize(ctx->stream));
    return FX_OK;
}

// ------------------------------------------------ Jacobi for the conv-diff operator (new)
//
// z = r / diag(A): diag = sigma + coeff (-kappa 2 (1/dx^2 + 1/dy^2) + |vx|/dx + |vy|/dy) inside
// (the upwind differences put |v|/h on the diagonal), 1 on the ring.
struct FlatCdJacobi {
    double *z;
    const double *r, *kappa, *vx, *vy;
    double kap_s, sigma, coeff, inv_dx, inv_dy, k2;
    size_t rows, cols;
    __device__ __forceinline__ void operator()(size_t i, CSum *) const {
        const size_t row = i / cols, col = i - row * cols;
        if (row == 0 || col == 0 || row == rows - 1 || col == cols - 1) {
            z[i] = r[i];
            return;
        }
        const double kap = kappa ? kappa[i] : kap_s;
        const double dcd = fma(-kap, k2, fma(fabs(vx[i]), inv_dx, fabs(vy[i]) * inv_dy));
        z[i] = r[i] / fma(coeff, dcd, sigma);
    }
};

struct CdJacobiPc : fx_precond {
    const fx_op *op = nullptr;
    int apply(fx_buf *z, const fx_buf *r, const int *skip, bool) override {
        FX_TRY(check_same(z, r));
        if (z->dtype != FX_F64 || z->len != op->g.rows * op->g.cols)
            return fail(FX_ERR_DIMENSION_MISMATCH, "Jacobi preconditioner: vectors must be F64 fields of the operator's grid");
        const ConvDiffC<double> K = conv_consts<double>(op->g.dx, op->g.dy);
        FlatCdJacobi f{(double *)z->ptr, (const double *)r->ptr,
                       op->kappa ? (const double *)op->kappa->ptr : nullptr, (const double *)op->vx->ptr,
                       (const double *)op->vy->ptr, op->kappa_s, op->sigma, op->coeff, K.inv_dx, K.inv_dy, K.k2,
                       op->g.rows, op->g.cols};
        return launch_flat<0>(ctx, z->len, f, NoFin{}, skip, "cd_jacobi");
    }
};

int check_op(const fx_grid &g, const fx_op *op) {
    if (!op) return fail(FX_ERR_INVALID_ARGUMENT, "null operator");
    if (op->g.rows != g.rows || op->g.cols != g.cols)
        return fail(FX_ERR_DIMENSION_MISMATCH, "operator grid does not match the solver grid");
    return FX_OK;
}

// ------------------------------------------------ multigrid for the conv-diff operator (new)
//
// Vertex hierarchy (rows - 1 halves while both interiors exceed coarse_max, as the vertex
// multigrid).  Each coarse level rediscretises the operator with h doubled and kappa / vx / vy
// injected from the coincident fine points.  Smoother: x <- x + omega (b - A x) / diag(A)
// inside; full weighting down, bilinear up; `coarse_sweeps` sweeps on the coarsest level in
// one block; every cycle from x = 0.  Unfused (a sweep, residual and transfer pass each): the
// variable coefficients do not fit the constant-stencil level kernels.

template <typename T>
__device__ __forceinline__ T cd_diag(const OpA<T, kModeCD> &A, size_t idx) {
    const T kap = A.kappa ? A.kappa[idx] : A.kap_s;
    return fx_fma(A.coeff, fx_fma(-kap, A.K.k2, fx_fma(fabs(A.vx[idx]), A.K.inv_dx, fabs(A.vy[idx]) * A.K.inv_dy)),
                  A.sigma);
}

// Smoothing sweep (out = x + omega (b - A x) (1 / diag(A)), one division per point) and
// residual (out = b - A x), inside
// only: the ring of `out` is not written.  One point per thread, neighbours read straight from
// memory (west / east from the same cache lines, north / south from L2): with four input arrays
// a row march holds too few loads in flight per SM (it measured 2.8 TB/s on the finest 4097^2
// sweep), these run at full occupancy.
template <typename T>
struct FlatCdSweep {
    OpA<T, kModeCD> A;
    const T *x;
    T *out;
    const T *b;
    T omega;
    size_t rows, cols;
    __device__ __forceinline__ void operator()(size_t i, CSum *) const {
        const size_t row = i / cols, col = i - row * cols;
        if (row == 0 || col == 0 || row == rows - 1 || col == cols - 1) return;
        Nb<T> nb;
        nb.c = x[i];
        nb.n = x[i - cols];
        nb.s = x[i + cols];
        nb.w = x[i - 1];
        nb.e = x[i + 1];
        const T inv_d = (T)1 / cd_diag(A, i);
        out[i] = fx_fma(omega, (b[i] - A.apply(false, nb, i)) * inv_d, nb.c);
    }
};

template <typename T>
struct FlatCdResid {
    OpA<T, kModeCD> A;
    const T *x;
    T *out;
    const T *b;
    size_t rows, cols;
    __device__ __forceinline__ void operator()(size_t i, CSum *) const {
        const size_t row = i / cols, col = i - row * cols;
        if (row == 0 || col == 0 || row == rows - 1 || col == cols - 1) return;
        Nb<T> nb;
        nb.c = x[i];
        nb.n = x[i - cols];
        nb.s = x[i + cols];
        nb.w = x[i - 1];
        nb.e = x[i + 1];
        out[i] = b[i] - A.apply(false, nb, i);
    }
};

// ---- learned smoother (fx_learned.cuh): the level operator as the network kernels see it, the
// residual pass that feeds the network, the training-sample extractor and the per-cycle check

template <typename T>
struct LsmOp {
    OpA<T, kModeCD> A;
    __device__ __forceinline__ T diag(size_t i) const { return cd_diag(A, i); }
    __device__ __forceinline__ T vxv(size_t i) const { return A.vx[i]; }
    __device__ __forceinline__ T vyv(size_t i) const { return A.vy[i]; }
};

// q = (b - A x) (1 / diag(A)) on the interior (the increment of FlatCdSweep divided by omega),
// 0 on the ring; sum of q^2 over the interior reduced for the scale
template <typename T>
struct FlatLsmResid {
    OpA<T, kModeCD> A;
    const T *x;
    T *q;
    const T *b;
    size_t rows, cols;
    __device__ __forceinline__ void operator()(size_t i, CSum *acc) const {
        const size_t row = i / cols, col = i - row * cols;
        if (row == 0 || col == 0 || row == rows - 1 || col == cols - 1) {
            q[i] = (T)0;
            return;
        }
        Nb<T> nb;
        nb.c = x[i];
        nb.n = x[i - cols];
        nb.s = x[i + cols];
        nb.w = x[i - 1];
        nb.e = x[i + 1];
        const T inv_d = (T)1 / cd_diag(A, i);
        const T v = (b[i] - A.apply(false, nb, i)) * inv_d;
        q[i] = v;
        csum_fma(acc[0], (double)v, (double)v);
    }
};

// scale[0] = s = sqrt(sum q^2 / interior points), scale[1] = 1 / s (0 when s = 0)
struct FinLsmScale {
    double *scale;
    double inv_n;
    __device__ void operator()(const double *v) const {
        const double s = sqrt(v[0] * inv_n);
        scale[0] = s;
        scale[1] = s > 0.0 ? 1.0 / s : 0.0;
    }
};

// One training sample per block from the fields of one iterate (see fx_learned.cuh): the network
// inputs over the 25 x 25 input region and, over the 16 x 16 loss patch, t = (H e - omega H q) / s
// and n = ||H e||^2 / s^2.  origins: (row, col) of each patch's first loss point.
template <typename Op>
__global__ void __launch_bounds__(256) k_lsm_extract(Op A, const double *__restrict__ q, const double *__restrict__ e,
                                                     const double *__restrict__ scale, double omega,
                                                     const int *__restrict__ origins, __nv_bfloat16 *d_in,
                                                     float *d_tgt, float *d_norm, int rows, int cols, double inv_dx,
                                                     double inv_dy) {
    using namespace lsm;
    __shared__ double se[kP3 * kP3], sq[kP3 * kP3], re[kNCo * kNCo], rq[kNCo * kNCo], red[16];
    const int tid = threadIdx.x;
    const int y0 = origins[2 * blockIdx.x], x0 = origins[2 * blockIdx.x + 1];
    const double inv_s = scale[1];
    __nv_bfloat16 *in = d_in + (size_t)blockIdx.x * kInLen;
    for (int k = tid; k < kPin * kPin; k += 256) {
        const int iy = k / kPin, ix = k - iy * kPin;
        const size_t i = (size_t)(y0 - 4 + iy) * cols + (x0 - 4 + ix);
        if (!FX_IN((long long)(y0 - 4 + iy) * cols + (x0 - 4 + ix), (long long)rows * cols)) continue;
        float c0, c1, c2;
        input_channels<double>(q[i], A.vxv(i), A.vyv(i), A.diag(i), inv_s, inv_dx, inv_dy, c0, c1, c2);
        in[k] = __float2bfloat16_rn(c0);
        in[kPin * kPin + k] = __float2bfloat16_rn(c1);
        in[2 * kPin * kPin + k] = __float2bfloat16_rn(c2);
    }
    for (int k = tid; k < kP3 * kP3; k += 256) {
        const int y = k / kP3, x = k - y * kP3;
        const size_t i = (size_t)(y0 - 1 + y) * cols + (x0 - 1 + x);
        if (!FX_IN((long long)(y0 - 1 + y) * cols + (x0 - 1 + x), (long long)rows * cols)) continue;
        se[k] = e[i];
        sq[k] = q[i];
    }
    __syncthreads();
    for (int k = tid; k < kNCo * kNCo; k += 256) {  // full weighting at the coarse points
        const int I = k / kNCo, J = k - I * kNCo;
        const int c = (2 * I + 1) * kP3 + 2 * J + 1;
        const double *f[2] = {se, sq};
        double *o[2] = {re, rq};
        for (int t = 0; t < 2; t++) {
            const double *v = f[t];
            const double ee = (v[c - kP3] + v[c + kP3]) + (v[c - 1] + v[c + 1]);
            const double dd = (v[c - kP3 - 1] + v[c - kP3 + 1]) + (v[c + kP3 - 1] + v[c + kP3 + 1]);
            o[t][k] = (4.0 * v[c] + (2.0 * ee + dd)) * 0.0625;
        }
    }
    __syncthreads();
    double nsum = 0.0, esum = 0.0;
    for (int k = tid; k < kT * kT; k += 256) {
        const int py = k / kT, px = k - py * kT;
        const int I = py >> 1, J = px >> 1;
        const bool oy = py & 1, ox = px & 1;
        double pe, pq;
        const int b = I * kNCo + J;
        if (!oy && !ox) {
            pe = re[b];
            pq = rq[b];
        } else if (oy && !ox) {
            pe = 0.5 * (re[b] + re[b + kNCo]);
            pq = 0.5 * (rq[b] + rq[b + kNCo]);
        } else if (!oy && ox) {
            pe = 0.5 * (re[b] + re[b + 1]);
            pq = 0.5 * (rq[b] + rq[b + 1]);
        } else {
            pe = 0.25 * ((re[b] + re[b + kNCo]) + (re[b + 1] + re[b + kNCo + 1]));
            pq = 0.25 * ((rq[b] + rq[b + kNCo]) + (rq[b + 1] + rq[b + kNCo + 1]));
        }
        const int c = (py + 1) * kP3 + px + 1;
        const double he = se[c] - pe, hq = sq[c] - pq;
        d_tgt[(size_t)blockIdx.x * kTgtLen + k] = (float)((he - omega * hq) * inv_s);
        d_tgt[(size_t)blockIdx.x * kTgtLen + kT * kT + k] = (float)((se[c] - omega * sq[c]) * inv_s);
        nsum += he * he;
        esum += se[c] * se[c];
    }
    for (int off = 16; off > 0; off >>= 1) {
        nsum += __shfl_down_sync(0xffffffffu, nsum, off);
        esum += __shfl_down_sync(0xffffffffu, esum, off);
    }
    if ((tid & 31) == 0) {
        red[tid >> 5] = nsum;
        red[8 + (tid >> 5)] = esum;
    }
    __syncthreads();
    if (tid == 0) {
        double t = 0.0, te = 0.0;
        for (int w = 0; w < 8; w++) {
            t += red[w];
            te += red[8 + w];
        }
        d_norm[2 * blockIdx.x] = (float)(t * inv_s * inv_s);
        d_norm[2 * blockIdx.x + 1] = (float)(te * inv_s * inv_s);
    }
}

// Per-cycle check of the learned cycle (on the F64 vectors of the application): ||r||^2 and
// ||r - A z||^2 over the interior.
struct FlatLsmCheck {
    OpA<double, kModeCD> A;
    const double *z, *r;
    size_t rows, cols;
    __device__ __forceinline__ void operator()(size_t i, CSum *acc) const {
        const size_t row = i / cols, col = i - row * cols;
        if (row == 0 || col == 0 || row == rows - 1 || col == cols - 1) return;
        Nb<double> nb;
        nb.c = z[i];
        nb.n = z[i - cols];
        nb.s = z[i + cols];
        nb.w = z[i - 1];
        nb.e = z[i + 1];
        const double rv = r[i], d = rv - A.apply(false, nb, i);
        csum_fma(acc[0], rv, rv);
        csum_fma(acc[1], d, d);
    }
};

// plain_skip = (the learned cycle reduced ||r|| by at least `ratio`, or the solve is over);
// counts applications and fallbacks while the solve runs.  With a patience (state non-null),
// `patience` fallbacks in a row switch the learned cycle off (state[1]).
struct FinLsmCheck {
    double ratio2;
    const int *skip;
    int *plain_skip;
    unsigned long long *counts;  // [0] applications, [1] fallbacks
    int *state;                  // LsmGate's [learned skip, off, fallbacks in a row], or null
    int patience;
    __device__ void operator()(const double *v) const {
        const bool done = skip && *(volatile const int *)skip;
        const bool ok = v[1] <= ratio2 * v[0];
        *plain_skip = (ok || done) ? 1 : 0;
        if (!done) {
            counts[0] += 1;
            if (!ok) counts[1] += 1;
            if (state) {
                state[2] = ok ? 0 : state[2] + 1;
                if (state[2] >= patience) state[1] = 1;
            }
        }
    }
};

// Gate of a learned application under a patience (one thread): the learned cycle and its check
// run unless the solve is over or the learned cycle is off; when it is off, the plain cycle runs
// alone (plain_skip 0) until the solve is over.
struct FlatLsmGate {
    const int *skip;
    int *state;  // [0] learned skip (written here), [1] off, [2] fallbacks in a row
    int *plain_skip;
    __device__ __forceinline__ void operator()(size_t, CSum *) const {
        const bool done = skip && *(volatile const int *)skip;
        const bool off = state[1] != 0;
        state[0] = (done || off) ? 1 : 0;
        if (done)
            *plain_skip = 1;
        else if (off)
            *plain_skip = 0;
    }
};

// One learned smoothing step on a level (fx_learned.cuh): q and the scale s in one pass, then the
// network and the update x <- x + omega q + s c in place.  q may be any scratch vector of the level.
template <typename T>
int lsm_step(fx_ctx *ctx, const fx_lsm *m, const OpA<T, kModeCD> &A, T *x, T *q, const T *b, T omega, size_t rows,
             size_t cols, double dx, double dy, double *scale, const int *skip) {
    using namespace lsm;
    if (rows < 3 || cols < 3) return fail(FX_ERR_INVALID_GRID, "learned smoother: grid too small");
    const double n_int = (double)(rows - 2) * (double)(cols - 2);
    FX_TRY((launch_flat<1>(ctx, rows * cols, FlatLsmResid<T>{A, x, q, b, rows, cols}, FinLsmScale{scale, 1.0 / n_int},
                           skip, "lsm_resid")));
    static std::atomic<unsigned long long> attr_done{0};  // one bit per device
    const unsigned long long bit = 1ull << (ctx->device & 63);
    if (!(attr_done.load() & bit)) {
        FX_CUDA(cudaFuncSetAttribute(k_lsm_apply<T, LsmOp<T>>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     kSmemApply));
        attr_done.fetch_or(bit);
    }
    const dim3 grid((unsigned)((cols + kTile - 1) / kTile), (unsigned)((rows + kTile - 1) / kTile));
    timing_pre(ctx, "lsm_apply");
    launch_pdl(ctx, k_lsm_apply<T, LsmOp<T>>, grid, dim3(256), (size_t)kSmemApply, LsmOp<T>{A},
               (const uint32_t *)m->d_frag, (const float *)m->d_wq, (const T *)q, x, (const double *)scale, omega,
               (int)rows, (int)cols, 1.0 / dx, 1.0 / dy, skip);
    timing_post(ctx, (double)rows * (double)cols);
    return check_launch(ctx, "lsm_apply");
}

// Two sweeps in one pass (temporal blocking): a 32 x 32 tile of the second sweep's points,
// with x over the tile plus a two-point halo and the first sweep's values over the tile plus
// a one-point halo in shared memory.  x is read once and only the second sweep's values are
// written (40 B/point against 80 for two passes).  Every value is FlatCdSweep's expression of
// the same operands: the first sweep's ring values are those of `out` (the buffer the first of
// two separate sweeps would have written, whose ring it leaves alone), so the pair equals two
// FlatCdSweep passes bit for bit, with the result in `out` instead of back in x.
constexpr int kSw2T = 32;           // tile side
constexpr int kSw2X = kSw2T + 4;    // x tile side (halo 2)
constexpr int kSw2Y = kSw2T + 2;    // first-sweep tile side (halo 1)

template <typename T>
__global__ void __launch_bounds__(256) k_cd_sweep2(OpA<T, kModeCD> A, const T *__restrict__ x, T *out,
                                                   const T *__restrict__ b, T omega, int rows, int cols,
                                                   const int *skip) {
    grid_dep_enter();
    if (skip && *(volatile const int *)skip) return;
    __shared__ T xs[kSw2X * kSw2X];
    __shared__ T ys[kSw2Y * kSw2Y];
    __shared__ T ds[kSw2Y * kSw2Y];  // 1 / diag(A) over the first sweep's tile
    const int tid = threadIdx.x;
    const int r0 = blockIdx.y * kSw2T, c0 = blockIdx.x * kSw2T;
    // fixed trip counts (256 threads), unrolled so that each thread's loads issue together
#pragma unroll
    for (int j = 0; j < (kSw2X * kSw2X + 255) / 256; j++) {
        const int k = tid + j * 256;
        if (k >= kSw2X * kSw2X) break;
        const int gr = r0 - 2 + k / kSw2X, gc = c0 - 2 + k % kSw2X;
        xs[k] = (gr >= 0 && gr < rows && gc >= 0 && gc < cols && FX_IN((long long)gr * cols + gc, (long long)rows * cols))
                    ? x[(size_t)gr * cols + gc]
                    : (T)0;
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < (kSw2Y * kSw2Y + 255) / 256; j++) {
        const int k = tid + j * 256;
        if (k >= kSw2Y * kSw2Y) break;
        const int lr = k / kSw2Y, lc = k % kSw2Y;
        const int gr = r0 - 1 + lr, gc = c0 - 1 + lc;
        T y = (T)0, inv_d = (T)0;
        if (gr >= 0 && gr < rows && gc >= 0 && gc < cols) {
            const size_t g = (size_t)gr * cols + gc;
            if (gr == 0 || gc == 0 || gr == rows - 1 || gc == cols - 1) {
                y = out[g];
            } else {
                inv_d = (T)1 / cd_diag(A, g);
                const int q = (lr + 1) * kSw2X + (lc + 1);
                Nb<T> nb;
                nb.c = xs[q];
                nb.n = xs[q - kSw2X];
                nb.s = xs[q + kSw2X];
                nb.w = xs[q - 1];
                nb.e = xs[q + 1];
                y = fx_fma(omega, (b[g] - A.apply(false, nb, g)) * inv_d, nb.c);
            }
        }
        ys[k] = y;
        ds[k] = inv_d;
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kSw2T * kSw2T / 256; j++) {
        const int k = tid + j * 256;
        const int lr = k / kSw2T, lc = k % kSw2T;
        const int gr = r0 + lr, gc = c0 + lc;
        if (gr <= 0 || gc <= 0 || gr >= rows - 1 || gc >= cols - 1) continue;
        const size_t g = (size_t)gr * cols + gc;
        const int q = (lr + 1) * kSw2Y + (lc + 1);
        if (!(FX_IN(g, (long long)rows * cols) && FX_IN(q + kSw2Y, kSw2Y * kSw2Y))) continue;
        Nb<T> nb;
        nb.c = ys[q];
        nb.n = ys[q - kSw2Y];
        nb.s = ys[q + kSw2Y];
        nb.w = ys[q - 1];
        nb.e = ys[q + 1];
        out[g] = fx_fma(omega, (b[g] - A.apply(false, nb, g)) * ds[q], nb.c);
    }
}

template <typename S, typename D>
struct FlatInject {  // coarse field = fine field at the coincident points (S -> D)
    const S *f;
    D *c;
    size_t fcols, ccols;
    __device__ __forceinline__ void operator()(size_t i, CSum *) const {
        const size_t I = i / ccols, J = i - I * ccols;
        c[i] = (D)f[(2 * I) * fcols + 2 * J];
    }
};

template <typename S, typename D>
struct FlatCast {  // d = (D) s
    const S *s;
    D *d;
    __device__ __forceinline__ void operator()(size_t i, CSum *) const { d[i] = (D)s[i]; }
};

// Coarsest level in one block: the iterate ping-pongs in shared memory, each thread keeps its
// points' rhs and reciprocal diagonal in registers; every point value is FlatCdSweep's
// expression.
template <typename T>
__global__ void __launch_bounds__(1024) k_cd_coarse(T *u, const T *__restrict__ b, int rows, int cols,
                                                    OpA<T, kModeCD> A, T omega, int nsweeps, const int *skip) {
    if (skip && *(volatile const int *)skip) return;
    constexpr int kPts = 4;
    extern __shared__ unsigned char smem_raw[];
    T *s0 = reinterpret_cast<T *>(smem_raw);
    T *s1 = s0 + rows * cols;
    const int n = rows * cols;
#ifdef FX_CHECKED
    {
        unsigned dyn;
        asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dyn));
        if (!(FX_IN(n - 1, kPts * (int)blockDim.x) && FX_IN(2LL * n - 1, dyn / sizeof(T)))) return;
    }
#endif
    int idx[kPts];
    bool inner[kPts];
    T bv[kPts], dv[kPts];
#pragma unroll
    for (int k = 0; k < kPts; k++) {
        const int i = threadIdx.x + k * blockDim.x;
        idx[k] = i;
        const int r = i / cols, c = i % cols;
        inner[k] = i < n && r > 0 && c > 0 && r < rows - 1 && c < cols - 1;
        bv[k] = inner[k] ? b[i] : (T)0;
        dv[k] = inner[k] ? (T)1 / cd_diag(A, (size_t)i) : (T)1;  // 1 / diag
        if (i < n) {
            s0[i] = (T)0;
            s1[i] = (T)0;
        }
    }
    __syncthreads();
    for (int k = 0; k < nsweeps; k++) {
        const T *src = (k & 1) ? s1 : s0;
        T *dst = (k & 1) ? s0 : s1;
#pragma unroll
        for (int q = 0; q < kPts; q++) {
            if (!inner[q]) continue;
            const int i = idx[q];
            Nb<T> nb;
            nb.c = src[i];
            nb.n = src[i - cols];
            nb.s = src[i + cols];
            nb.w = src[i - 1];
            nb.e = src[i + 1];
            dst[i] = fx_fma(omega, (bv[q] - A.apply(false, nb, (size_t)i)) * dv[q], nb.c);
        }
        __syncthreads();
    }
    const T *fin = (nsweeps & 1) ? s1 : s0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) u[i] = fin[i];
}

struct CdLevel {
    size_t rows = 0, cols = 0;
    double dx = 0, dy = 0;
    // levels >= 1, and level 0 of an F32 cycle: iterate, right-hand side, ping-pong partner
    fx_buf *u = nullptr, *rhs = nullptr, *tmp = nullptr;
    // levels >= 1 (injected), and level 0 of an F32 cycle (the operator's fields in F32)
    fx_buf *vx = nullptr, *vy = nullptr, *kappa = nullptr;
};

}  // namespace

struct fx_cdmg {
    fx_ctx *ctx = nullptr;
    const fx_op *op = nullptr;
    size_t n_pre = 2, n_post = 2, coarse_sweeps = 200;
    double omega = 0.8;
    int dtype = FX_F64;  // arithmetic and storage of the cycle; the vectors z, r stay F64
    std::vector<CdLevel> lv;
    fx_buf *tmp0 = nullptr;  // level-0 ping-pong partner of an F64 cycle
    struct View : fx_precond {
        fx_cdmg *mg = nullptr;
        int apply(fx_buf *z, const fx_buf *r, const int *skip, bool z_zero) override;
        int record(fx_buf *z, const fx_buf *r, const int *skip, bool z_zero);
    } view;
    // One application is a fixed sequence of launches for given (z, r, halt flag, stream).  With
    // replay on (fx_cdmg_set_replay), it is recorded into a CUDA graph the first time and
    // replayed after that: one launch instead of 20-50.  Off by default: recording and
    // instantiating costs more than a short-lived hierarchy's replays save (the batched
    // workload, one new hierarchy per problem, same box: -5 % on one lane, -4 to -9 % on 8).
    struct Replay {
        const void *z, *r;
        const int *skip;
        bool z_zero;
        cudaStream_t stream;
        cudaGraphExec_t exec;
        std::vector<void *> frees;  // pool memory freed during the recording, still addressed by exec
    };
    std::vector<Replay> replays;
    bool replay = false;      // fx_cdmg_set_replay
    bool replay_off = false;  // a recording failed: launch directly from then on
    // learned smoothing (fx_cdmg_set_learned): levels of at least lsm_min_points points smooth
    // with the network; each application is checked and, when the learned cycle reduced
    // ||r|| by less than lsm_ratio, recomputed with the plain cycle
    const fx_lsm *lsm = nullptr;
    size_t lsm_min_points = 0, lsm_max_points = 0;  // 0: no upper bound
    double lsm_ratio = 0.9;
    double *d_lsm_scale = nullptr;          // [2]: s, 1 / s of the current learned step
    int *d_plain_skip = nullptr;            // 1: the plain recomputation is not needed
    int lsm_patience = 0;                   // fallbacks in a row that switch the learned cycle off (0: never)
    int *d_lsm_state = nullptr;             // FlatLsmGate's state
    unsigned long long *d_lsm_counts = nullptr;  // [2]: checked applications, fallbacks
    void drop_replays() {
        for (auto &g : replays) {
            cudaGraphExecDestroy(g.exec);
            for (void *p : g.frees) cudaFree(p);  // waits for the device: a replay may still run
        }
        replays.clear();
    }
    ~fx_cdmg() {
        drop_replays();
        if (d_lsm_scale) cudaFree(d_lsm_scale);
        if (d_plain_skip) cudaFree(d_plain_skip);
        if (d_lsm_state) cudaFree(d_lsm_state);
        if (d_lsm_counts) cudaFree(d_lsm_counts);
        for (auto &L : lv)
            for (fx_buf *f : {L.u, L.rhs, L.tmp, L.vx, L.vy, L.kappa}) fx_free(f);
        fx_free(tmp0);
    }
    // The operator on level l: h doubled per level, the injected fields; level 0 of an F64
    // cycle reads the operator's own fields.
    template <typename T>
    OpA<T, kModeCD> level_op(size_t l) const {
        const CdLevel &L = lv[l];
        OpA<T, kModeCD> A;
        A.K = conv_consts<T>(L.dx, L.dy);
        A.sigma = (T)op->sigma;
        A.coeff = (T)op->coeff;
        A.kap_s = (T)op->kappa_s;
        const bool own = l == 0 && dtype == FX_F64;
        A.vx = (const T *)(own ? op->vx->ptr : L.vx->ptr);
        A.vy = (const T *)(own ? op->vy->ptr : L.vy->ptr);
        const fx_buf *k = own ? op->kappa : L.kappa;
        A.kappa = k ? (const T *)k->ptr : nullptr;
        return A;
    }
};

namespace {

template <typename T>
int cd_cycle(fx_cdmg *mg, T *x, const T *b, T *x_other, const int *skip, bool learned) {  // x holds zeros on entry
    fx_ctx *ctx = mg->ctx;
    const int nl = (int)mg->lv.size();
    std::vector<T *> cur(nl), oth(nl);
    std::vector<const T *> rhs(nl);
    cur[0] = x;
    oth[0] = x_other;
    rhs[0] = b;
    for (int l = 1; l < nl; l++) {
        cur[l] = (T *)mg->lv[l].u->ptr;
        oth[l] = (T *)mg->lv[l].tmp->ptr;
        rhs[l] = (const T *)mg->lv[l].rhs->ptr;
    }
    const T omega = (T)mg->omega;
    auto smooth = [&](int l, size_t n) -> int {
        const CdLevel &L = mg->lv[l];
        const auto A = mg->level_op<T>(l);
        if (learned && l < nl - 1 && L.rows * L.cols >= mg->lsm_min_points &&
            (!mg->lsm_max_points || L.rows * L.cols <= mg->lsm_max_points)) {  // in place; oth[l] holds q
            for (size_t k = 0; k < n; k++)
                FX_TRY(lsm_step<T>(ctx, mg->lsm, A, cur[l], oth[l], rhs[l], omega, L.rows, L.cols, L.dx, L.dy,
                                   mg->d_lsm_scale, skip));
            return FX_OK;
        }
        size_t k = 0;
        for (; k + 2 <= n; k += 2) {  // pairs in one pass; the result lands in the partner buffer
            const dim3 grid((unsigned)((L.cols + kSw2T - 1) / kSw2T), (unsigned)((L.rows + kSw2T - 1) / kSw2T));
            timing_pre(ctx, "cdmg_sweep2");
            launch_pdl(ctx, k_cd_sweep2<T>, grid, dim3(256), 0, A, (const T *)cur[l], oth[l], rhs[l], omega,
                       (int)L.rows, (int)L.cols, skip);
            timing_post(ctx, (double)L.rows * (double)L.cols);
            FX_TRY(check_launch(ctx, "cdmg_sweep2"));
            std::swap(cur[l], oth[l]);
        }
        for (; k < n; k++) {
            FX_TRY((launch_flat<0>(ctx, L.rows * L.cols,
                                   FlatCdSweep<T>{A, cur[l], oth[l], rhs[l], omega, L.rows, L.cols}, NoFin{}, skip,
                                   "cdmg_sweep")));
            std::swap(cur[l], oth[l]);
        }
        return FX_OK;
    };
    for (int l = 0; l < nl - 1; l++) {
        const CdLevel &L = mg->lv[l], &Cl = mg->lv[l + 1];
        FX_TRY(smooth(l, mg->n_pre));
        FX_TRY((launch_flat<0>(ctx, L.rows * L.cols,
                               FlatCdResid<T>{mg->level_op<T>(l), cur[l], oth[l], rhs[l], L.rows, L.cols}, NoFin{},
                               skip, "cdmg_residual")));
        FX_TRY(restrict_fw<T>(ctx, oth[l], (T *)Cl.rhs->ptr, L.cols, Cl.rows, Cl.cols, skip));
        FX_TRY(zero_fill<T>(ctx, cur[l + 1], Cl.rows * Cl.cols, skip));
    }
    {
        const int l = nl - 1;
        const CdLevel &L = mg->lv[l];
        const size_t n = L.rows * L.cols;
        if (coarse_fits(n, sizeof(T)) && mg->coarse_sweeps > 0) {
            k_cd_coarse<T><<<1, coarse_threads(n), 2 * n * sizeof(T), ctx->stream>>>(
                cur[l], rhs[l], (int)L.rows, (int)L.cols, mg->level_op<T>(l), omega, (int)mg->coarse_sweeps, skip);
            FX_TRY(check_launch(ctx, "cdmg_coarse_solve"));
        } else {
            FX_TRY(smooth(l, mg->coarse_sweeps));
        }
    }
    for (int l = nl - 2; l >= 0; l--) {
        const CdLevel &L = mg->lv[l], &Cl = mg->lv[l + 1];
        FX_TRY(prolong_bilinear<T>(ctx, cur[l + 1], cur[l], Cl.cols, L.rows, L.cols, skip));
        FX_TRY(smooth(l, mg->n_post));
    }
    if (cur[0] != x) {
        const CdLevel &L0 = mg->lv[0];
        FX_CUDA(cudaMemcpyAsync(x, cur[0], L0.rows * L0.cols * sizeof(T), cudaMemcpyDeviceToDevice, ctx->stream));
    }
    return FX_OK;
}

}  // namespace

int fx_cdmg::View::apply(fx_buf *z, const fx_buf *r, const int *skip, bool z_zero) {
    FX_TRY(check_same(z, r));
    // the checks of record(), before a replay: a recycled address must carry the same extent
    const CdLevel &L0 = mg->lv[0];
    if (z->dtype != FX_F64 || z->len != L0.rows * L0.cols)
        return fail(FX_ERR_DIMENSION_MISMATCH, "conv-diff multigrid: vectors must be F64 fields of the operator's grid");
    if (z->ptr == r->ptr) return fail(FX_ERR_INVALID_ARGUMENT, "z and r must be distinct");
    // Per-launch timing records events on the stream, which a recording would capture: while
    // timing is on, the application runs directly.
    if (!mg->replay || mg->replay_off || ctx->timing || capturing(ctx->stream)) return record(z, r, skip, z_zero);
    for (auto &g : mg->replays)
        if (g.z == z->ptr && g.r == r->ptr && g.skip == skip && g.z_zero == z_zero && g.stream == ctx->stream) {
            FX_CUDA(cudaGraphLaunch(g.exec, ctx->stream));
            ctx->launches++;
            return FX_OK;
        }
    if (mg->replays.size() >= 16) return record(z, r, skip, z_zero);  // many distinct pairs: no cache
    const size_t nf0 = ctx->deferred_free.size();
    FX_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeRelaxed));
    const int st = record(z, r, skip, z_zero);
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(ctx->stream, &graph);
    // buffers freed while recording: they belong to this graph (or, if it failed, to no graph)
    std::vector<void *> frees(ctx->deferred_free.begin() + (std::ptrdiff_t)std::min(nf0, ctx->deferred_free.size()),
                              ctx->deferred_free.end());
    ctx->deferred_free.resize(std::min(nf0, ctx->deferred_free.size()));
    cudaGraphExec_t exec = nullptr;
    if (st == FX_OK && e == cudaSuccess && graph && cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess) {
        cudaGraphDestroy(graph);
        mg->replays.push_back({z->ptr, r->ptr, skip, z_zero, ctx->stream, exec, std::move(frees)});
        FX_CUDA(cudaGraphLaunch(exec, ctx->stream));
        ctx->launches++;
        return FX_OK;
    }
    if (graph) cudaGraphDestroy(graph);
    (void)cudaGetLastError();
    for (void *p : frees) cudaFreeAsync(p, ctx->stream);
    // Not recordable here (a capture-illegal call inside, or the capture was invalidated): run
    // the application directly, now and from now on.  A genuine error shows again in that run.
    mg->replay_off = true;
    return record(z, r, skip, z_zero);
}

// The launches of one application (recorded by apply, or run directly).
int fx_cdmg::View::record(fx_buf *z, const fx_buf *r, const int *skip, bool z_zero) {
    CdLevel &L0 = mg->lv[0];
    const size_t n = L0.rows * L0.cols;
    if (z->dtype != FX_F64 || z->len != n)
        return fail(FX_ERR_DIMENSION_MISMATCH, "conv-diff multigrid: vectors must be F64 fields of the operator's grid");
    if (z->ptr == r->ptr) return fail(FX_ERR_INVALID_ARGUMENT, "z and r must be distinct");
    auto run = [&](bool learned, const int *sk, bool zz) -> int {
        if (mg->dtype == FX_F32) {  // r -> F32, the cycle in F32, z = its F64 image
            float *x = (float *)L0.u->ptr, *b = (float *)L0.rhs->ptr;
            FX_TRY((launch_flat<0>(ctx, n, FlatCast<double, float>{(const double *)r->ptr, b}, NoFin{}, sk,
                                   "cdmg_convert")));
            FX_TRY(zero_fill<float>(ctx, x, n, sk));
            FX_TRY(cd_cycle<float>(mg, x, b, (float *)L0.tmp->ptr, sk, learned));
            return launch_flat<0>(ctx, n, FlatCast<float, double>{x, (double *)z->ptr}, NoFin{}, sk, "cdmg_convert");
        }
        if (!zz) FX_TRY(zero_fill<double>(ctx, (double *)z->ptr, z->len, sk));
        return cd_cycle<double>(mg, (double *)z->ptr, (const double *)r->ptr, (double *)mg->tmp0->ptr, sk, learned);
    };
    if (!mg->lsm) return run(false, skip, z_zero);
    // the learned cycle, its check, and the plain cycle where the check failed (all on the device)
    const bool gated = mg->lsm_patience > 0;
    const int *lskip = skip;
    if (gated) {
        FX_TRY(launch_flat<0>(ctx, 1, FlatLsmGate{skip, mg->d_lsm_state, mg->d_plain_skip}, NoFin{}, nullptr,
                              "cdmg_learned_gate"));
        lskip = mg->d_lsm_state;
    }
    FX_TRY(run(true, lskip, z_zero));
    const double ratio2 = mg->lsm_ratio * mg->lsm_ratio;
    FX_TRY((launch_flat<2>(ctx, n,
                           FlatLsmCheck{mg->level_op<double>(0), (const double *)z->ptr, (const double *)r->ptr,
                                        L0.rows, L0.cols},
                           FinLsmCheck{ratio2, skip, mg->d_plain_skip, mg->d_lsm_counts,
                                       gated ? mg->d_lsm_state : nullptr, mg->lsm_patience},
                           gated ? lskip : nullptr, "cdmg_learned_check")));
    return run(false, mg->d_plain_skip, false);
}

namespace {

// ------------------------------------------------ inner-CG preconditioner (new)
//
// z = a fixed number of CG steps (preconditioned by `inner` when set) on A z = r from z = 0,
// with tolerance 0 so the step count alone ends it (or a breakdown).  The count of the k-th
// application is steps[k mod nsteps], so a schedule of different counts gives a
// preconditioner that changes from one application to the next -- the case the flexible
// solvers exist for; PCG and left-preconditioned GMRES lose their guarantees with it.
// ------------------------------------------------ inner FP32 PCG preconditioner (new)
//
// z = the FP32 solution d of A d = r, by FP32 CG preconditioned by an FP32 V-cycle from d = 0 to
// ||r - A d|| < rel_tol ||r|| (or max_iter): one pass casts r to FP32 and reduces ||r||^2, the
// inner solve runs on FP32 vectors, one pass widens d into z.  It varies from one application
// to the next (the inner stop depends on r), so it is for the flexible solvers (FCG, FGMRES),
// which keep the outer Krylov information in FP64.

struct FlatCastNorm {  // r32 = (float) r; ||r||^2
    const double *r;
    float *r32;
    __device__ __forceinline__ void operator()(size_t i, CSum *acc) const {
        const double v = r[i];
        r32[i] = (float)v;
        csum_fma(acc[0], v, v);
    }
};

struct FlatWiden {  // z = (double) d
    const float *d;
    double *z;
    __device__ __forceinline__ void operator()(size_t i, CSum *) const { z[i] = (double)d[i]; }
};

struct InnerPcgF32Pc : fx_precond {
    fx_cg *cg = nullptr;  // FP32 CG: its vectors and state
    fx_buf *r32 = nullptr, *d32 = nullptr;
    fx_precond *inner = nullptr;  // FP32 V-cycle, borrowed
    fx_grid g{};
    double coeff = 0.0;
    StencilP P{};
    double rel_tol = 1e-4;
    size_t max_iter = 100;
    size_t total = 0, calls = 0;
    ~InnerPcgF32Pc() override {
        if (cg) fx_cg_destroy(cg);
        if (r32) fx_free(r32);
        if (d32) fx_free(d32);
    }
    int apply(fx_buf *z, const fx_buf *r, const int *, bool) override {
        FX_TRY(check_same(z, r));
        if (z->dtype != FX_F64 || z->len != g.rows * g.cols)
            return fail(FX_ERR_INVALID_ARGUMENT, "inner FP32 PCG: vectors must be F64 fields of its grid");
        const size_t n = z->len;
        FX_TRY(launch_flat<1>(ctx, n, FlatCastNorm{(const double *)r->ptr, (float *)r32->ptr},
                              StoreFin<1>{ctx->d_result}, nullptr, "inner_pcg_cast"));
        double rr = 0.0;
        FX_TRY(read_results(ctx, 1, &rr));
        FX_TRY(zero_fill<float>(ctx, (float *)d32->ptr, n, nullptr));
        calls++;
        if (rr > 0.0 && std::isfinite(rr)) {
            cg->tol = rel_tol * std::sqrt(rr);
            cg->max_iter = max_iter;
            SOLVER_MODE_DISPATCH(P, FX_TRY((cg_solve_impl<float, MODE>(cg, d32, r32, coeff, P, inner))));
            total += (size_t)cg->h_st->iter;
        }
        return launch_flat<0>(ctx, n, FlatWiden{(const float *)d32->ptr, (double *)z->ptr}, NoFin{}, nullptr,
                              "inner_pcg_widen");
    }
};

struct InnerCgPc : fx_precond {
    fx_cg *cg = nullptr;
    fx_precond *inner = nullptr;
    double coeff = 0.0;
    std::vector<int> dr, dc;
    std::vector<double> wt;
    fx_boundaries bc{};
    std::vector<size_t> steps;
    size_t calls = 0;
    ~InnerCgPc() override {
        if (cg) fx_cg_destroy(cg);
    }
    int apply(fx_buf *z, const fx_buf *r, const int *, bool z_zero) override {
        FX_TRY(check_same(z, r));
        if (z->dtype != FX_F64) return fail(FX_ERR_INVALID_ARGUMENT, "inner-CG preconditioner vectors must be F64");
        if (!z_zero) FX_TRY(zero_fill<double>(ctx, (double *)z->ptr, z->len, nullptr));
        FX_TRY(fx_cg_set_params(cg, 0.0, steps[calls++ % steps.size()]));
        const fx_stencil st{(int)wt.size(), dr.data(), dc.data(), wt.data()};
        fx_stats out;
        if (inner) return fx_cg_solve_preconditioned(cg, z, r, coeff, &st, &bc, inner, &out);
        return fx_cg_solve(cg, z, r, coeff, &st, &bc, &out);
    }
};

}  // namespace

// ================================================================ C ABI

extern "C" {

int fx_precond_identity(fx_ctx *ctx, fx_precond **out) {
    if (!ctx || !out) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    IdentityPc *p = new IdentityPc();
    p->ctx = ctx;
    *out = p;
    return FX_OK;
}

int fx_precond_destroy(fx_precond *pc) {
    if (!pc) return FX_OK;
    if (pc->borrowed) return fail(FX_ERR_INVALID_ARGUMENT, "borrowed preconditioner: destroy its owner");
    delete pc;
    return FX_OK;
}

int fx_precond_apply(fx_precond *pc, fx_buf *z, const fx_buf *r) {
    FX_RANGE("fx_precond_apply");
    if (!pc) return fail(FX_ERR_INVALID_ARGUMENT, "null preconditioner");
    FX_TRY(check_buf(z, "z"));
    FX_TRY(check_buf(r, "r"));
    return pc->apply(z, r, nullptr, false);
}

int fx_mg_create(fx_ctx *ctx, const fx_grid *g, const fx_boundaries *bc, size_t n_pre, size_t n_post, double omega,
                 int smoother, fx_mg **out) {
    if (!ctx || !out) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    FX_TRY(check_grid(g));
    if (smoother != 0 && smoother != 1) return fail(FX_ERR_INVALID_ARGUMENT, "smoother must be 0 (Jacobi) or 1 (Chebyshev)");
    *out = nullptr;
    fx_mg *mg = new fx_mg();
    mg->ctx = ctx;
    mg->mode = 0;
    mg->smoother = smoother;
    mg->n_pre = n_pre;
    mg->n_post = n_post;
    mg->omega = omega;
    if (bc) mg->bc = *bc;
    mg->view.mg = mg;
    mg->view.ctx = ctx;
    mg->view.borrowed = true;
    size_t r = g->rows, c = g->cols;
    double hx = g->dx, hy = g->dy;
    for (;;) {  // multigrid.rs:101-136
        MgLevel L;
        L.rows = r;
        L.cols = c;
        L.dx = hx;
        L.dy = hy;
        lap5_of(hx, hy, L.lap5);
        int st = fx_alloc(ctx, r * c, FX_F64, &L.u);
        if (!st) st = fx_alloc(ctx, r * c, FX_F64, &L.rhs);
        if (!st) st = fx_alloc(ctx, r * c, FX_F64, &L.tmp);
        if (!st && smoother == 1) st = fx_alloc(ctx, r * c, FX_F64, &L.w0);  // multigrid.rs:113-119
        if (!st && smoother == 1) st = fx_alloc(ctx, r * c, FX_F64, &L.w1);
        mg->lv.push_back(L);
        if (st) {
            delete mg;
            return st;
        }
        if (r <= 4 || c <= 4) break;
        const size_t cr = r / 2, cc = c / 2;
        if (cr < 3 || cc < 3) break;
        r = cr;
        c = cc;
        hx *= 2.0;
        hy *= 2.0;
    }
    *out = mg;
    return FX_OK;
}

int fx_mg_create_vertex(fx_ctx *ctx, const fx_grid *g, const fx_boundaries *bc, const fx_mg_vertex_opts *o,
                        fx_mg **out) {
    if (!ctx || !out || !o) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    FX_TRY(check_grid(g));
    if (bc) {
        for (int i = 0; i < 4; i++)
            if (bc->side[i].kind != FX_BC_DIRICHLET || bc->side[i].a != 0.0)
                return fail(FX_ERR_UNSUPPORTED, "vertex multigrid needs homogeneous Dirichlet boundaries");
    }
    if (o->dtype != FX_F32 && o->dtype != FX_F64) return fail(FX_ERR_INVALID_ARGUMENT, "unknown dtype");
    StencilP P;
    FX_TRY(make_stencil(&o->op_stencil, &P));
    if (P.mode != 5) return fail(FX_ERR_UNSUPPORTED, "vertex multigrid needs a 5-point operator");
    *out = nullptr;
    fx_mg *mg = new fx_mg();
    mg->ctx = ctx;
    mg->mode = 1;
    mg->dtype = o->dtype;
    mg->n_pre = o->n_pre;
    mg->n_post = o->n_post;
    mg->omega = o->omega;
    mg->coarse_sweeps = o->coarse_sweeps;
    if (bc) mg->bc = *bc;
    mg->view.mg = mg;
    mg->view.ctx = ctx;
    mg->view.borrowed = true;
    double a5[5];
    const double cf = o->op_coeff;
    a5[0] = 1.0 + cf * P.c;
    a5[1] = cf * P.n;
    a5[2] = cf * P.s;
    a5[3] = cf * P.w;
    a5[4] = cf * P.e;
    const double sigma = a5[0] + ((a5[1] + a5[2]) + (a5[3] + a5[4]));
    size_t r = g->rows, c = g->cols;
    double hx = g->dx, hy = g->dy;
    int st = FX_OK;
    for (int l = 0;; l++) {
        MgLevel L;
        L.rows = r;
        L.cols = c;
        L.dx = hx;
        L.dy = hy;
        if (l == 0) std::memcpy(L.a5, a5, sizeof(a5));
        else coarse_op(mg->lv[l - 1].a5, sigma, L.a5);
        if (l > 0) {
            st = fx_alloc(ctx, r * c, o->dtype, &L.u);
            if (!st) st = fx_alloc(ctx, r * c, o->dtype, &L.rhs);
            if (!st) st = fx_alloc(ctx, r * c, o->dtype, &L.tmp);
        }
        mg->lv.push_back(L);
        if (st) break;
        if (!(r - 2 > o->coarse_max && c - 2 > o->coarse_max && (r - 1) % 2 == 0 && (c - 1) % 2 == 0)) break;
        r = (r - 1) / 2 + 1;
        c = (c - 1) / 2 + 1;
        hx *= 2.0;
        hy *= 2.0;
    }
    const size_t n0 = g->rows * g->cols;
    if (!st) st = fx_alloc(ctx, n0, o->dtype, &mg->tmp0);
    if (!st && o->dtype == FX_F32) {
        st = fx_alloc(ctx, n0, FX_F32, &mg->x32);
        if (!st) st = fx_alloc(ctx, n0, FX_F32, &mg->b32);
    }
    if (st) {
        delete mg;
        return st;
    }
    *out = mg;
    return FX_OK;
}

int fx_mg_destroy(fx_mg *mg) {
    if (!mg) return FX_OK;
    cudaStreamSynchronize(mg->ctx->stream);
    delete mg;
    return FX_OK;
}

int fx_mg_depth(const fx_mg *mg, size_t *depth) {
    if (!mg || !depth) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    *depth = mg->lv.size();
    return FX_OK;
}

int fx_mg_level_dims(const fx_mg *mg, size_t level, size_t *rows, size_t *cols) {
    if (!mg || !rows || !cols) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    if (level >= mg->lv.size()) return fail(FX_ERR_INVALID_ARGUMENT, "level out of range");
    *rows = mg->lv[level].rows;
    *cols = mg->lv[level].cols;
    return FX_OK;
}

int fx_mg_v_cycle(fx_mg *mg, fx_buf *x, const fx_buf *b) {
    FX_RANGE("fx_mg_v_cycle");
    if (!mg) return fail(FX_ERR_INVALID_ARGUMENT, "null multigrid");
    FX_TRY(check_buf(x, "x"));
    FX_TRY(check_buf(b, "b"));
    return mg->view.apply(x, b, nullptr, false);
}

int fx_mg_precondition(fx_mg *mg, fx_buf *z, const fx_buf *r) {
    if (!mg) return fail(FX_ERR_INVALID_ARGUMENT, "null multigrid");
    FX_TRY(check_buf(z, "z"));
    FX_TRY(check_buf(r, "r"));
    return mg->view.apply(z, r, nullptr, true);
}

fx_precond *fx_mg_as_precond(fx_mg *mg) { return mg ? &mg->view : nullptr; }

int fx_mg_set_tuning(fx_mg *mg, const fx_mg_tuning *t) {
    if (!mg || !t) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    if (t->chunk_pct < 10 || t->chunk_pct > 1000) return fail(FX_ERR_INVALID_ARGUMENT, "chunk_pct must lie in 10..1000");
    mg->chunk_pct = t->chunk_pct;
    mg->tail_top_max = t->tail_top_points;
    return FX_OK;
}

int fx_mg_get_tuning(const fx_mg *mg, fx_mg_tuning *t) {
    if (!mg || !t) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    t->chunk_pct = mg->chunk_pct;
    t->tail_top_points = mg->tail_top_max;
    return FX_OK;
}

int fx_mg_autotune(fx_mg *mg, fx_buf *z, const fx_buf *r, int reps, fx_mg_tuning *best, double *best_ms,
                   double *cand_ms, size_t cand_cap, size_t *ncand) {
    if (!mg || !z || !r || !best) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    if (reps < 1) return fail(FX_ERR_INVALID_ARGUMENT, "reps must be at least 1");
    if (mg->mode != 1 || !fusable(mg) || z->dtype != FX_F64)
        return fail(FX_ERR_UNSUPPORTED, "autotuning covers the fused vertex V(2,2)-cycle on F64 vectors");
    static const int kPct[] = {50, 100, 200};
    static const size_t kTop[] = {9 * 1024, 2 * 1024};  // 65^2 and 33^2 tails on 2^k + 1 grids
    fx_ctx *ctx = mg->ctx;
    const int saved_pct = mg->chunk_pct;
    const size_t saved_top = mg->tail_top_max;
    cudaEvent_t e0, e1;
    FX_CUDA(cudaEventCreate(&e0));
    FX_CUDA(cudaEventCreate(&e1));
    double best_t = 1e300;
    size_t k = 0;
    int rc = FX_OK;
    for (int ip = 0; ip < 3 && rc == FX_OK; ip++)
        for (int it = 0; it < 2 && rc == FX_OK; it++, k++) {
            mg->chunk_pct = kPct[ip];
            mg->tail_top_max = kTop[it];
            for (int w = 0; w < 2 && rc == FX_OK; w++) rc = mg->view.apply(z, r, nullptr, true);
            if (rc != FX_OK) break;
            cudaEventRecord(e0, ctx->stream);
            for (int q = 0; q < reps && rc == FX_OK; q++) rc = mg->view.apply(z, r, nullptr, true);
            cudaEventRecord(e1, ctx->stream);
            if (cudaEventSynchronize(e1) != cudaSuccess) rc = fail(FX_ERR_BACKEND, "autotune timing failed");
            if (rc != FX_OK) break;
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            const double per = (double)ms / reps;
            if (cand_ms && k < cand_cap) cand_ms[k] = per;
            if (per < best_t) {
                best_t = per;
                best->chunk_pct = kPct[ip];
                best->tail_top_points = kTop[it];
            }
        }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc != FX_OK) {
        mg->chunk_pct = saved_pct;
        mg->tail_top_max = saved_top;
        return rc;
    }
    mg->chunk_pct = best->chunk_pct;
    mg->tail_top_max = best->tail_top_points;
    if (best_ms) *best_ms = best_t;
    if (ncand) *ncand = k;
    return FX_OK;
}

// ---- CG

int fx_cg_create(fx_ctx *ctx, const fx_grid *g, double tol, size_t max_iter, fx_cg **out) {
    return create_solver(ctx, g, tol, max_iter, 4, out);
}
int fx_cg_destroy(fx_cg *s) {
    delete s;
    return FX_OK;
}
int fx_cg_set_params(fx_cg *s, double tol, size_t max_iter) {
    if (!s) return fail(FX_ERR_INVALID_ARGUMENT, "null solver");
    s->tol = tol;
    s->max_iter = max_iter;
    return FX_OK;
}

static int cg_entry(fx_cg *s, fx_buf *x, const fx_buf *b, double coeff, const fx_stencil *st, const fx_boundaries *bc,
                    fx_precond *pc, fx_stats *out) {
    if (!s || !out) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    FX_TRY(s->check_io(x, b));
    StencilP P;
    FX_TRY(prep_op(s->g, st, bc, &P));
    if (s->dtype == FX_F32) SOLVER_MODE_DISPATCH(P, FX_TRY((cg_solve_impl<float, MODE>(s, x, b, coeff, P, pc))));
    else SOLVER_MODE_DISPATCH(P, FX_TRY((cg_solve_impl<double, MODE>(s, x, b, coeff, P, pc))));
    s->stats(out);
    return FX_OK;
}

int fx_cg_solve(fx_cg *s, fx_buf *x, const fx_buf *b, double coeff, const fx_stencil *st, const fx_boundaries *bc,
                fx_stats *out) {
    FX_RANGE("fx_cg_solve");
    return cg_entry(s, x, b, coeff, st, bc, nullptr, out);
}

int fx_cg_solve_preconditioned(fx_cg *s, fx_buf *x, const fx_buf *b, double coeff, const fx_stencil *st,
                               const fx_boundaries *bc, fx_precond *pc, fx_stats *out) {
    FX_RANGE("fx_cg_solve_preconditioned");
    if (!pc) return fail(FX_ERR_INVALID_ARGUMENT, "null preconditioner");
    return cg_entry(s, x, b, coeff, st, bc, pc, out);
}

// ---- pipelined CG

int fx_pipelined_cg_create(fx_ctx *ctx, const fx_grid *g, double tol, size_t max_iter, fx_pipelined_cg **out) {
    return create_solver(ctx, g, tol, max_iter, 6, out);
}
int fx_pipelined_cg_destroy(fx_pipelined_cg *s) {
    delete s;
    return FX_OK;
}
int fx_pipelined_cg_set_params(fx_pipelined_cg *s, double tol, size_t max_iter) {
    if (!s) return fail(FX_ERR_INVALID_ARGUMENT, "null solver");
    s->tol = tol;
    s->max_iter = max_iter;
    return FX_OK;
}
int fx_pipelined_cg_solve(fx_pipelined_cg *s, fx_buf *x, const fx_buf *b, double coeff, const fx_stencil *st,
                          const fx_boundaries *bc, fx_stats *out) {
    FX_RANGE("fx_pipelined_cg_solve");
    if (!s || !out) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    FX_TRY(s->check_io(x, b));
    StencilP P;
    FX_TRY(prep_op(s->g, st, bc, &P));
    SOLVER_MODE_DISPATCH(P, FX_TRY(pipe_solve_impl<MODE>(s, x, b, coeff, P)));
    s->stats(out);
    return FX_OK;
}

int fx_pipelined_cg_solve_preconditioned(fx_pipelined_cg *s, fx_buf *x, const fx_buf *b, double coeff,
                                         const fx_stencil *st, const fx_boundaries *bc, fx_precond *pc,
                                         fx_stats *out) {
    FX_RANGE("fx_pipelined_cg_solve_preconditioned");
    if (!s || !out) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    if (!pc) return fail(FX_ERR_INVALID_ARGUMENT, "null preconditioner");
    FX_TRY(s->check_io(x, b));
    StencilP P;
    FX_TRY(prep_op(s->g, st, bc, &P));
    SOLVER_MODE_DISPATCH(P, FX_TRY(ppcg_solve_impl<MODE>(s, x, b, coeff, P, pc)));
    s->stats(out);
    return FX_OK;
}

// ---- mixed-precision iterative refinement

int fx_ir_create(fx_ctx *ctx, const fx_grid *g, double tol, size_t max_outer, double inner_tol,
                 size_t inner_max_iter, fx_ir **out) {
    if (!(inner_tol > 0 && inner_tol < 1)) return fail(FX_ERR_INVALID_ARGUMENT, "inner_tol must lie in (0, 1)");
    FX_TRY(create_solver(ctx, g, tol, max_outer, 2, out, FX_F32));
    (*out)->inner_tol = inner_tol;
    (*out)->inner_max_iter = inner_max_iter;
    const int st = create_solver(ctx, g, 0.0, inner_max_iter, 4, &(*out)->inner, FX_F32);
    if (st) {
        delete *out;
        *out = nullptr;
    }
    return st;
}
int fx_ir_destroy(fx_ir *s) {
    delete s;
    return FX_OK;
}
int fx_ir_solve_preconditioned(fx_ir *s, fx_buf *x, const fx_buf *b, double coeff, const fx_stencil *st,
                               const fx_boundaries *bc, fx_precond *pc, fx_stats *out, size_t *inner_iterations) {
    FX_RANGE("fx_ir_solve_preconditioned");
    if (!s || !out) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    if (!pc) return fail(FX_ERR_INVALID_ARGUMENT, "null preconditioner");
    FX_TRY(check_buf(x, "x"));
    FX_TRY(check_buf(b, "b"));
    FX_TRY(check_grid_len(&s->g, x));
    FX_TRY(check_grid_len(&s->g, b));
    if (x->dtype != FX_F64 || b->dtype != FX_F64) return fail(FX_ERR_INVALID_ARGUMENT, "x and b must be F64");
    StencilP P;
    FX_TRY(prep_op(s->g, st, bc, &P));
    SOLVER_MODE_DISPATCH(P, FX_TRY(ir_solve_impl<MODE>(s, x, b, coeff, st, bc, P, pc)));
    s->stats(out);
    if (inner_iterations) *inner_iterations = s->inner_total;
    return FX_OK;
}

// ---- BiCGSTAB

int fx_bicgstab_create(fx_ctx *ctx, const fx_grid *g, double tol, size_t max_iter, fx_bicgstab **out) {
    return create_solver(ctx, g, tol, max_iter, 10, out);
}
int fx_bicgstab_destroy(fx_bicgstab *s) {
    delete s;
    return FX_OK;
}
int fx_bicgstab_set_params(fx_bicgstab *s, double tol, size_t max_iter) {
    if (!s) return fail(FX_ERR_INVALID_ARGUMENT, "null solver");
    s->tol = tol;
    s->max_iter = max_iter;
    return FX_OK;
}
static int bicg_entry(fx_bicgstab *s, fx_buf *x, const fx_buf *b, double coeff, const fx_stencil *st,
                      const fx_boundaries *bc, fx_precond *pc, fx_stats *out) {
    if (!s || !out) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    FX_TRY(s->check_io(x, b));
    StencilP P;
    FX_TRY(prep_op(s->g, st, bc, &P));
    SOLVER_MODE_DISPATCH(P, FX_TRY(bicg_solve_impl<MODE>(s, x, b, coeff, P, pc)));
    s->stats(out);
    return FX_OK;
}
int fx_bicgstab_solve(fx_bicgstab *s, fx_buf *x, const fx_buf *b, double coeff, const fx_stencil *st,
                      const fx_boundaries *bc, fx_stats *out) {
    FX_RANGE("fx_bicgstab_solve");
    return bicg_entry(s, x, b, coeff, st, bc, nullptr, out);
}
int fx_bicgstab_solve_preconditioned(fx_bicgstab *s, fx_buf *x, const fx_buf *b, double coeff, const fx_stencil *st,
                                     const fx_boundaries *bc, fx_precond *pc, fx_stats *out) {
    FX_RANGE("fx_bicgstab_solve_preconditioned");
    if (!pc) return fail(FX_ERR_INVALID_ARGUMENT, "null preconditioner");
    return bicg_entry(s, x, b, coeff, st, bc, pc, out);
}

// ---- GMRES

int fx_gmres_create(fx_ctx *ctx, const fx_grid *g, size_t restart, double tol, size_t max_iter, fx_gmres **out) {
    if (restart < 1) return fail(FX_ERR_INVALID_ARGUMENT, "restart must be at least 1");
    FX_TRY(create_solver(ctx, g, tol, max_iter, (int)restart + 2, out));
    fx_gmres *s = *out;
    s->restart = restart;
    s->hh.assign((restart + 1) * restart, 0.0);
    s->cc.assign(restart, 0.0);
    s->ss.assign(restart, 0.0);
    s->grs.assign(restart + 1, 0.0);
    if (cudaMalloc(&s->d_h, (restart + 2) * sizeof(double)) != cudaSuccess ||
        cudaHostAlloc(&s->h_h, 2 * (restart + 2) * sizeof(double), cudaHostAllocMapped) != cudaSuccess ||
        cudaHostGetDevicePointer((void **)&s->h_h_dev, s->h_h, 0) != cudaSuccess) {
        delete s;
        *out = nullptr;
        return fail(FX_ERR_BACKEND, "gmres scratch allocation failed");
    }
    return FX_OK;
}
int fx_gmres_destroy(fx_gmres *s) {
    delete s;
    return FX_OK;
}
int fx_gmres_set_params(fx_gmres *s, double tol, size_t max_iter) {
    if (!s) return fail(FX_ERR_INVALID_ARGUMENT, "null solver");
    s->tol = tol;
    s->max_iter = max_iter;
    return FX_OK;
}
static int gmres_entry(fx_gmres *s, fx_buf *x, const fx_buf *b, double coeff, const fx_stencil *st,
                       const fx_boundaries *bc, fx_precond *pc, fx_stats *out) {
    if (!s || !out) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    FX_TRY(s->check_io(x, b));
    StencilP P;
    FX_TRY(prep_op(s->g, st, bc, &P));
    SOLVER_MODE_DISPATCH(P, FX_TRY(gmres_solve_impl<MODE>(s, x, b, coeff, P, pc)));
    s->stats(out);
    return FX_OK;
}
int fx_gmres_solve(fx_gmres *s, fx_buf *x, const fx_buf *b, double coeff, const fx_stencil *st,
                   const fx_boundaries *bc, fx_stats *out) {
    FX_RANGE("fx_gmres_solve");
    return gmres_entry(s, x, b, coeff, st, bc, nullptr, out);
}
int fx_gmres_solve_preconditioned(fx_gmres *s, fx_buf *x, const fx_buf *b, double coeff, const fx_stencil *st,
                                  const fx_boundaries *bc, fx_precond *pc, fx_stats *out) {
    FX_RANGE("fx_gmres_solve_preconditioned");
    if (!pc) return fail(FX_ERR_INVALID_ARGUMENT, "null preconditioner");
    return gmres_entry(s, x, b, coeff, st, bc, pc, out);
}

// ---- flexible CG / flexible GMRES / inner-CG preconditioner (new)

int fx_fcg_create(fx_ctx *ctx, const fx_grid *g, double tol, size_t max_iter, fx_fcg **out) {
    return create_solver(ctx, g, tol, max_iter, 5, out);
}
int fx_fcg_destroy(fx_fcg *s) {
    delete s;
    return FX_OK;
}
int fx_fcg_set_params(fx_fcg *s, double tol, size_t max_iter) {
    if (!s) return fail(FX_ERR_INVALID_ARGUMENT, "null solver");
    s->tol = tol;
    s->max_iter = max_iter;
    return FX_OK;
}
static int fcg_entry(fx_fcg *s, fx_buf *x, const fx_buf *b, double coeff, const fx_stencil *st,
                     const fx_boundaries *bc, fx_precond *pc, fx_stats *out) {
    if (!s || !out) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    FX_TRY(s->check_io(x, b));
    StencilP P;
    FX_TRY(prep_op(s->g, st, bc, &P));
    IdentityPc idp;
    idp.ctx = s->ctx;
    SOLVER_MODE_DISPATCH(P, FX_TRY(fcg_solve_impl<MODE>(s, x, b, coeff, P, pc ? pc : &idp)));
    s->stats(out);
    return FX_OK;
}
int fx_fcg_solve(fx_fcg *s, fx_buf *x, const fx_buf *b, double coeff, const fx_stencil *st, const fx_boundaries *bc,
                 fx_stats *out) {
    FX_RANGE("fx_fcg_solve");
    return fcg_entry(s, x, b, coeff, st, bc, nullptr, out);
}
int fx_fcg_solve_preconditioned(fx_fcg *s, fx_buf *x, const fx_buf *b, double coeff, const fx_stencil *st,
                                const fx_boundaries *bc, fx_precond *pc, fx_stats *out) {
    FX_RANGE("fx_fcg_solve_preconditioned");
    if (!pc) return fail(FX_ERR_INVALID_ARGUMENT, "null preconditioner");
    return fcg_entry(s, x, b, coeff, st, bc, pc, out);
}

int fx_fgmres_create(fx_ctx *ctx, const fx_grid *g, size_t restart, double tol, size_t max_iter, fx_fgmres **out) {
    if (restart < 1) return fail(FX_ERR_INVALID_ARGUMENT, "restart must be at least 1");
    FX_TRY(create_solver(ctx, g, tol, max_iter, 2 * (int)restart + 2, out));
    fx_fgmres *s = *out;
    s->restart = restart;
    s->hh.assign((restart + 1) * restart, 0.0);
    s->cc.assign(restart, 0.0);
    s->ss.assign(restart, 0.0);
    s->grs.assign(restart + 1, 0.0);
    if (cudaMalloc(&s->d_h, (restart + 2) * sizeof(double)) != cudaSuccess ||
        cudaHostAlloc(&s->h_h, 2 * (restart + 2) * sizeof(double), cudaHostAllocMapped) != cudaSuccess ||
        cudaHostGetDevicePointer((void **)&s->h_h_dev, s->h_h, 0) != cudaSuccess) {
        delete s;
        *out = nullptr;
        return fail(FX_ERR_BACKEND, "fgmres scratch allocation failed");
    }
    return FX_OK;
}
int fx_fgmres_destroy(fx_fgmres *s) {
    delete s;
    return FX_OK;
}
int fx_fgmres_set_orthogonalization(fx_fgmres *s, int method) {
    if (!s) return fail(FX_ERR_INVALID_ARGUMENT, "null solver");
    if (method != 0 && method != 1) return fail(FX_ERR_INVALID_ARGUMENT, "method: 0 = MGS, 1 = CGS2");
    if (method == 1 && s->restart > (size_t)kCgsMax)
        return fail(FX_ERR_UNSUPPORTED, "CGS2 orthogonalisation needs restart <= 32");
    if (method == 1 && !s->d_cgs) {
        const size_t blocks = (size_t)s->ctx->num_sms * 8;  // flat_geom's cap
        if (cudaMalloc(&s->d_cgs, 2 * (s->restart + 2) * sizeof(double)) != cudaSuccess ||
            cudaMalloc(&s->d_part, blocks * kCgsMax * sizeof(double)) != cudaSuccess ||
            cudaMalloc(&s->d_ticket, sizeof(unsigned)) != cudaSuccess ||
            cudaMemset(s->d_ticket, 0, sizeof(unsigned)) != cudaSuccess) {
            (void)cudaGetLastError();
            return fail(FX_ERR_BACKEND, "fgmres CGS2 scratch allocation failed");
        }
    }
    s->cgs2 = method == 1;
    return FX_OK;
}
int fx_fgmres_set_params(fx_fgmres *s, double tol, size_t max_iter) {
    if (!s) return fail(FX_ERR_INVALID_ARGUMENT, "null solver");
    s->tol = tol;
    s->max_iter = max_iter;
    return FX_OK;
}
static int fgmres_entry(fx_fgmres *s, fx_buf *x, const fx_buf *b, double coeff, const fx_stencil *st,
                        const fx_boundaries *bc, fx_precond *pc, fx_stats *out) {
    if (!s || !out) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    FX_TRY(s->check_io(x, b));
    StencilP P;
    FX_TRY(prep_op(s->g, st, bc, &P));
    SOLVER_MODE_DISPATCH(P, FX_TRY(fgmres_solve_impl<MODE>(s, x, b, coeff, P, pc)));
    s->stats(out);
    return FX_OK;
}
int fx_fgmres_solve(fx_fgmres *s, fx_buf *x, const fx_buf *b, double coeff, const fx_stencil *st,
                    const fx_boundaries *bc, fx_stats *out) {
    FX_RANGE("fx_fgmres_solve");
    return fgmres_entry(s, x, b, coeff, st, bc, nullptr, out);
}
int fx_fgmres_solve_preconditioned(fx_fgmres *s, fx_buf *x, const fx_buf *b, double coeff, const fx_stencil *st,
                                   const fx_boundaries *bc, fx_precond *pc, fx_stats *out) {
    FX_RANGE("fx_fgmres_solve_preconditioned");
    if (!pc) return fail(FX_ERR_INVALID_ARGUMENT, "null preconditioner");
    return fgmres_entry(s, x, b, coeff, st, bc, pc, out);
}

// ---- conv-diff operator in the solvers (new)

int fx_op_conv_diff(fx_ctx *ctx, const fx_grid *g, double sigma, double coeff, const fx_buf *kappa, double kappa_s,
                    const fx_buf *vx, const fx_buf *vy, fx_op **out) {
    if (!ctx || !g || !out) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    FX_TRY(check_grid(g));
    const size_t n = g->rows * g->cols;
    if (g->rows < 3 || g->cols < 3) return fail(FX_ERR_INVALID_ARGUMENT, "conv-diff operator needs at least 3 x 3 points");
    for (const fx_buf *f : {vx, vy, kappa}) {
        if (f == kappa && !kappa) continue;
        FX_TRY(check_buf(f, "conv-diff field"));
        if (f->dtype != FX_F64) return fail(FX_ERR_INVALID_ARGUMENT, "conv-diff fields must be F64");
        if (f->len != n) return fail(FX_ERR_DIMENSION_MISMATCH, "conv-diff field length does not match the grid");
    }
    fx_op *op = new fx_op();
    op->ctx = ctx;
    op->g = *g;
    op->sigma = sigma;
    op->coeff = coeff;
    op->kappa = kappa;
    op->kappa_s = kappa_s;
    op->vx = vx;
    op->vy = vy;
    *out = op;
    return FX_OK;
}
int fx_op_destroy(fx_op *op) {
    delete op;
    return FX_OK;
}
int fx_op_apply(const fx_op *op, const fx_buf *v, fx_buf *out) {
    if (!op) return fail(FX_ERR_INVALID_ARGUMENT, "null operator");
    FX_TRY(check_buf(v, "v"));
    FX_TRY(check_buf(out, "out"));
    FX_TRY(check_grid_len(&op->g, v));
    FX_TRY(check_grid_len(&op->g, out));
    if (v->dtype != FX_F64 || out->dtype != FX_F64) return fail(FX_ERR_INVALID_ARGUMENT, "operator vectors must be F64");
    if (v->ptr == out->ptr) return fail(FX_ERR_INVALID_ARGUMENT, "v and out must be distinct");
    const auto A = OpMaker<double, kModeCD>::make(StencilP{}, 0.0, op->g.rows, op->g.cols, op);
    return launch_pt<double, 0>(op->ctx, op->g.rows, op->g.cols, Ld1<double>{(const double *)v->ptr},
                                   PtApplyOp<double, kModeCD>{A, (double *)out->ptr}, NoFin{}, nullptr, "op_apply");
}

int fx_precond_jacobi_op(const fx_op *op, fx_precond **out) {
    if (!op || !out) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    CdJacobiPc *p = new CdJacobiPc();
    p->ctx = op->ctx;
    p->op = op;
    *out = p;
    return FX_OK;
}

extern "C++" {
template <typename S, typename Run>
static int op_entry(S *s, fx_buf *x, const fx_buf *b, const fx_op *op, fx_stats *out, Run run) {
    if (!s || !out) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    FX_TRY(s->check_io(x, b));
    FX_TRY(check_op(s->g, op));
    if (s->dtype != FX_F64) return fail(FX_ERR_INVALID_ARGUMENT, "the conv-diff operator runs in F64");
    s->op = op;
    const int rc = run();
    s->op = nullptr;
    FX_TRY(rc);
    s->stats(out);
    return FX_OK;
}
}  // extern "C++"

int fx_bicgstab_solve_op(fx_bicgstab *s, fx_buf *x, const fx_buf *b, const fx_op *op, fx_precond *pc, fx_stats *out) {
    FX_RANGE("fx_bicgstab_solve_op");
    return op_entry(s, x, b, op, out, [&] { return bicg_solve_impl<kModeCD>(s, x, b, op->coeff, StencilP{}, pc); });
}
int fx_gmres_solve_op(fx_gmres *s, fx_buf *x, const fx_buf *b, const fx_op *op, fx_precond *pc, fx_stats *out) {
    FX_RANGE("fx_gmres_solve_op");
    return op_entry(s, x, b, op, out, [&] { return gmres_solve_impl<kModeCD>(s, x, b, op->coeff, StencilP{}, pc); });
}
int fx_fgmres_solve_op(fx_fgmres *s, fx_buf *x, const fx_buf *b, const fx_op *op, fx_precond *pc, fx_stats *out) {
    FX_RANGE("fx_fgmres_solve_op");
    return op_entry(s, x, b, op, out, [&] { return fgmres_solve_impl<kModeCD>(s, x, b, op->coeff, StencilP{}, pc); });
}

int fx_cdmg_create(const fx_op *op, size_t n_pre, size_t n_post, double omega, size_t coarse_max,
                   size_t coarse_sweeps, fx_cdmg **out) {
    return fx_cdmg_create_typed(op, n_pre, n_post, omega, coarse_max, coarse_sweeps, FX_F64, out);
}

int fx_cdmg_create_typed(const fx_op *op, size_t n_pre, size_t n_post, double omega, size_t coarse_max,
                         size_t coarse_sweeps, int dtype, fx_cdmg **out) {
    if (!op || !out) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    if (dtype != FX_F32 && dtype != FX_F64) return fail(FX_ERR_INVALID_ARGUMENT, "unknown dtype");
    *out = nullptr;
    fx_cdmg *mg = new fx_cdmg();
    mg->ctx = op->ctx;
    mg->op = op;
    mg->n_pre = n_pre;
    mg->n_post = n_post;
    mg->omega = omega;
    mg->coarse_sweeps = coarse_sweeps;
    mg->dtype = dtype;
    mg->view.ctx = op->ctx;
    mg->view.mg = mg;
    mg->view.borrowed = true;
    const bool f32 = dtype == FX_F32;
    size_t r = op->g.rows, c = op->g.cols;
    double hx = op->g.dx, hy = op->g.dy;
    int rc = FX_OK;
    // the level fields in the cycle's type: level 0 casts the operator's own (F32 cycle only),
    // coarser levels inject from the level above
    auto fields = [&](CdLevel &L, size_t l) -> int {
        const fx_buf *src[3] = {op->vx, op->vy, op->kappa};
        fx_buf **dst[3] = {&L.vx, &L.vy, &L.kappa};
        for (int k = 0; k < 3 && rc == FX_OK; k++) {
            if (!src[k]) continue;
            FX_TRY(fx_alloc(op->ctx, r * c, dtype, dst[k]));
            const double *own = (const double *)src[k]->ptr;
            if (l == 0) {
                FX_TRY((launch_flat<0>(op->ctx, r * c, FlatCast<double, float>{own, (float *)(*dst[k])->ptr}, NoFin{},
                                       nullptr, "cdmg_inject")));
                continue;
            }
            const CdLevel &F = mg->lv[l - 1];
            const fx_buf *fine = l == 1 && !f32 ? src[k] : (k == 0 ? F.vx : (k == 1 ? F.vy : F.kappa));
            if (f32)
                FX_TRY((launch_flat<0>(op->ctx, r * c,
                                       FlatInject<float, float>{(const float *)fine->ptr, (float *)(*dst[k])->ptr,
                                                                F.cols, c},
                                       NoFin{}, nullptr, "cdmg_inject")));
            else
                FX_TRY((launch_flat<0>(op->ctx, r * c,
                                       FlatInject<double, double>{(const double *)fine->ptr,
                                                                  (double *)(*dst[k])->ptr, F.cols, c},
                                       NoFin{}, nullptr, "cdmg_inject")));
        }
        return FX_OK;
    };
    for (size_t l = 0; l < 40 && rc == FX_OK; l++) {
        CdLevel L;
        L.rows = r;
        L.cols = c;
        L.dx = hx;
        L.dy = hy;
        if (l > 0 || f32) {
            for (fx_buf **bp : {&L.u, &L.rhs, &L.tmp})
                if (rc == FX_OK) rc = fx_alloc(op->ctx, r * c, dtype, bp);
            if (rc == FX_OK) rc = fields(L, l);
        }
        mg->lv.push_back(L);
        if (rc != FX_OK) break;
        if (!(r - 2 > coarse_max && c - 2 > coarse_max && (r - 1) % 2 == 0 && (c - 1) % 2 == 0)) break;
        r = (r - 1) / 2 + 1;
        c = (c - 1) / 2 + 1;
        hx *= 2.0;
        hy *= 2.0;
    }
    if (rc == FX_OK && !f32) rc = fx_alloc(op->ctx, op->g.rows * op->g.cols, FX_F64, &mg->tmp0);
    if (rc != FX_OK) {
        delete mg;
        return rc;
    }
    *out = mg;
    return FX_OK;
}
int fx_cdmg_destroy(fx_cdmg *mg) {
    delete mg;
    return FX_OK;
}
int fx_cdmg_depth(const fx_cdmg *mg, size_t *depth) {
    if (!mg || !depth) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    *depth = mg->lv.size();
    return FX_OK;
}
fx_precond *fx_cdmg_as_precond(fx_cdmg *mg) { return mg ? &mg->view : nullptr; }
int fx_cdmg_set_replay(fx_cdmg *mg, int enabled) {
    if (!mg) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    mg->replay = enabled != 0;
    return FX_OK;
}

int fx_cdmg_set_learned(fx_cdmg *mg, const fx_lsm *lsm, size_t min_points, size_t max_points, double fallback_ratio) {
    if (!mg) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    if (lsm && lsm->ctx->device != mg->ctx->device)
        return fail(FX_ERR_INVALID_ARGUMENT, "learned smoother lives on another device");
    if (lsm && !(fallback_ratio > 0.0)) return fail(FX_ERR_INVALID_ARGUMENT, "fallback ratio must be positive");
    if (lsm) {
        bool any = false;
        for (size_t l = 0; l + 1 < mg->lv.size(); l++) {
            const size_t pts = mg->lv[l].rows * mg->lv[l].cols;
            any = any || (pts >= min_points && (!max_points || pts <= max_points));
        }
        if (!any)
            return fail(FX_ERR_INVALID_ARGUMENT,
                        "no level in [min_points, max_points]: the cycle would not use the network");
    }
    FX_CUDA(cudaStreamSynchronize(mg->ctx->stream));
    mg->drop_replays();  // the recorded launch sequence changes
    if (lsm && !mg->d_lsm_scale) {
        FX_CUDA(cudaMalloc(&mg->d_lsm_scale, 2 * sizeof(double)));
        FX_CUDA(cudaMalloc(&mg->d_plain_skip, sizeof(int)));
        FX_CUDA(cudaMalloc(&mg->d_lsm_counts, 2 * sizeof(unsigned long long)));
        FX_CUDA(cudaMemset(mg->d_lsm_counts, 0, 2 * sizeof(unsigned long long)));
    }
    mg->lsm = lsm;
    mg->lsm_min_points = min_points;
    mg->lsm_max_points = max_points;
    mg->lsm_ratio = fallback_ratio;
    if (mg->d_lsm_state) FX_CUDA(cudaMemset(mg->d_lsm_state, 0, 3 * sizeof(int)));
    return FX_OK;
}

int fx_cdmg_set_learned_patience(fx_cdmg *mg, size_t patience) {
    if (!mg) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    if (patience > (size_t)1 << 30) return fail(FX_ERR_INVALID_ARGUMENT, "patience out of range");
    FX_CUDA(cudaStreamSynchronize(mg->ctx->stream));
    if (!mg->d_lsm_state) FX_CUDA(cudaMalloc(&mg->d_lsm_state, 3 * sizeof(int)));
    FX_CUDA(cudaMemset(mg->d_lsm_state, 0, 3 * sizeof(int)));
    if ((int)patience != mg->lsm_patience) mg->drop_replays();  // the gate joins or leaves the sequence
    mg->lsm_patience = (int)patience;
    return FX_OK;
}

int fx_cdmg_learned_disabled(fx_cdmg *mg, int *disabled) {
    if (!mg || !disabled) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    int st[3] = {0, 0, 0};
    if (mg->d_lsm_state) {
        FX_CUDA(cudaStreamSynchronize(mg->ctx->stream));
        FX_CUDA(cudaMemcpy(st, mg->d_lsm_state, sizeof(st), cudaMemcpyDeviceToHost));
    }
    *disabled = st[1];
    return FX_OK;
}

int fx_cdmg_learned_stats(fx_cdmg *mg, unsigned long long *applications, unsigned long long *fallbacks) {
    if (!mg || !applications || !fallbacks) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    unsigned long long c[2] = {0, 0};
    if (mg->d_lsm_counts) {
        FX_CUDA(cudaStreamSynchronize(mg->ctx->stream));
        FX_CUDA(cudaMemcpy(c, mg->d_lsm_counts, sizeof(c), cudaMemcpyDeviceToHost));
    }
    *applications = c[0];
    *fallbacks = c[1];
    return FX_OK;
}

// ------------------------------------------------ learned smoother: operator-side entry points

namespace {

int lsm_check_op(const fx_op *op) {
    if (!op) return fail(FX_ERR_INVALID_ARGUMENT, "null operator");
    if (op->vx->dtype != FX_F64 || op->vy->dtype != FX_F64 || (op->kappa && op->kappa->dtype != FX_F64))
        return fail(FX_ERR_INVALID_ARGUMENT, "learned smoother: operator fields must be F64");
    return FX_OK;
}

int lsm_check_field(const fx_op *op, const fx_buf *v, const char *name) {
    FX_TRY(check_buf(v, name));
    if (v->dtype != FX_F64 || v->len != op->g.rows * op->g.cols)
        return fail(FX_ERR_DIMENSION_MISMATCH, std::string("learned smoother: ") + name +
                                                   " must be an F64 field of the operator's grid");
    return FX_OK;
}

}  // namespace

int fx_lsm_smooth(fx_lsm *m, const fx_op *op, fx_buf *x, const fx_buf *b, double omega, size_t steps) {
    if (!m) return fail(FX_ERR_INVALID_ARGUMENT, "null learned smoother");
    FX_TRY(lsm_check_op(op));
    FX_TRY(lsm_check_field(op, x, "x"));
    FX_TRY(lsm_check_field(op, b, "b"));
    if (x->ptr == b->ptr) return fail(FX_ERR_INVALID_ARGUMENT, "x and b must be distinct");
    fx_ctx *ctx = op->ctx;
    if (m->ctx->device != ctx->device) return fail(FX_ERR_INVALID_ARGUMENT, "learned smoother lives on another device");
    if (!steps) return FX_OK;
    fx_buf *q = nullptr;
    FX_TRY(fx_alloc(ctx, x->len, FX_F64, &q));
    double *scale = nullptr;
    int st = cudaMallocAsync(&scale, 2 * sizeof(double), ctx->stream) == cudaSuccess
                 ? FX_OK
                 : fail(FX_ERR_BACKEND, "learned smoother: scratch allocation failed");
    const OpA<double, kModeCD> A = OpMaker<double, kModeCD>::make(StencilP{}, 0.0, 0, 0, op);
    for (size_t k = 0; k < steps && st == FX_OK; k++)
        st = lsm_step<double>(ctx, m, A, (double *)x->ptr, (double *)q->ptr, (const double *)b->ptr, omega,
                              op->g.rows, op->g.cols, op->g.dx, op->g.dy, scale, nullptr);
    if (scale) cudaFreeAsync(scale, ctx->stream);
    fx_free(q);
    if (st == FX_OK) FX_CUDA(cudaStreamSynchronize(ctx->stream));
    return st;
}

int fx_lsm_data_add_patches(fx_lsm_data *d, const fx_op *op, const fx_buf *x, const fx_buf *e, const fx_buf *b,
                            double omega, const int *origins, size_t count) {
    using namespace lsm;
    if (!d || !origins) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    FX_TRY(lsm_check_op(op));
    FX_TRY(lsm_check_field(op, x, "x"));
    FX_TRY(lsm_check_field(op, e, "e"));
    FX_TRY(lsm_check_field(op, b, "b"));
    if (d->ctx->device != op->ctx->device) return fail(FX_ERR_INVALID_ARGUMENT, "samples live on another device");
    if (count == 0) return FX_OK;
    if (count > d->cap - d->count) return fail(FX_ERR_INVALID_ARGUMENT, "sample capacity exceeded");
    const long rows = (long)op->g.rows, cols = (long)op->g.cols;
    for (size_t k = 0; k < count; k++) {  // input region inside the grid, output region inside the interior
        const long y0 = origins[2 * k], x0 = origins[2 * k + 1];
        if ((y0 & 1) || (x0 & 1) || y0 < 4 || x0 < 4 || y0 + kT + 4 >= rows || x0 + kT + 4 >= cols)
            return fail(FX_ERR_INVALID_ARGUMENT,
                        "patch origin " + std::to_string(y0) + "," + std::to_string(x0) +
                            " must be even and leave the 25 x 25 input region inside the grid");
    }
    fx_ctx *ctx = op->ctx;
    fx_buf *q = nullptr;
    FX_TRY(fx_alloc(ctx, x->len, FX_F64, &q));
    void *scratch = nullptr;  // scale [2 doubles] + origins
    const size_t obytes = count * 2 * sizeof(int);
    int st = cudaMallocAsync(&scratch, 16 + obytes, ctx->stream) == cudaSuccess
                 ? FX_OK
                 : fail(FX_ERR_BACKEND, "learned smoother: scratch allocation failed");
    double *scale = (double *)scratch;
    int *d_orig = (int *)((char *)scratch + 16);
    const OpA<double, kModeCD> A = OpMaker<double, kModeCD>::make(StencilP{}, 0.0, 0, 0, op);
    const size_t n = x->len;
    if (st == FX_OK && cudaMemcpyAsync(d_orig, origins, obytes, cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess)
        st = fail(FX_ERR_BACKEND, "learned smoother: origin upload failed");
    if (st == FX_OK)
        st = launch_flat<1>(ctx, n,
                            FlatLsmResid<double>{A, (const double *)x->ptr, (double *)q->ptr, (const double *)b->ptr,
                                                 op->g.rows, op->g.cols},
                            FinLsmScale{scale, 1.0 / ((double)(rows - 2) * (double)(cols - 2))}, nullptr, "lsm_resid");
    if (st == FX_OK) {
        k_lsm_extract<LsmOp<double>><<<(unsigned)count, 256, 0, ctx->stream>>>(
            LsmOp<double>{A}, (const double *)q->ptr, (const double *)e->ptr, scale, omega, d_orig,
            d->d_in + d->count * kInLen, d->d_tgt + d->count * kTgtLen, d->d_norm + 2 * d->count, (int)rows, (int)cols,
            1.0 / op->g.dx, 1.0 / op->g.dy);
        st = check_launch(ctx, "lsm_extract");
    }
    if (scratch) cudaFreeAsync(scratch, ctx->stream);
    fx_free(q);
    if (st == FX_OK) {
        FX_CUDA(cudaStreamSynchronize(ctx->stream));
        d->count += count;
    }
    return st;
}

int fx_lsm_data_add_problem(fx_lsm_data *d, const fx_op *op, const fx_buf *b, size_t iterates,
                            size_t patches_per_iterate, double omega, unsigned long long seed, size_t *added) {
    using namespace lsm;
    if (!d || !added) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    *added = 0;
    FX_TRY(lsm_check_op(op));
    FX_TRY(lsm_check_field(op, b, "b"));
    const long rows = (long)op->g.rows, cols = (long)op->g.cols;
    if (rows < 2 * kT + 10 || cols < 2 * kT + 10)
        return fail(FX_ERR_INVALID_GRID, "learned smoother samples need a grid of at least 42 x 42 points");
    fx_ctx *ctx = op->ctx;
    const size_t n = b->len;
    double bnorm = 0.0;
    FX_TRY(fx_norm_l2(ctx, b, &bnorm));
    // the exact solution u of A u = b: FGMRES(30) with the plain cycle, to 1e-12 relative
    fx_cdmg *mg = nullptr;
    FX_TRY(fx_cdmg_create(op, 2, 2, omega, 15, 200, &mg));
    fx_fgmres *solver = nullptr;
    std::vector<fx_buf *> bufs(5, nullptr);  // u, x, e, r, z
    int st = fx_fgmres_create(ctx, &op->g, 30, 1e-12 * bnorm, 600, &solver);
    for (auto &p : bufs)
        if (st == FX_OK) st = fx_alloc(ctx, n, FX_F64, &p);
    fx_stats stats{};
    if (st == FX_OK) st = fx_fgmres_solve_op(solver, bufs[0], b, op, fx_cdmg_as_precond(mg), &stats);
    if (st == FX_OK && stats.residual > 1e-9 * bnorm)
        st = fail(FX_ERR_BACKEND, "learned smoother samples: reference solve did not converge");
    std::mt19937_64 rng(seed);
    std::uniform_int_distribution<long> ry(2, (rows - kT - 5) / 2), rx(2, (cols - kT - 5) / 2);
    std::vector<int> org;
    fx_buf *u = bufs[0], *x = bufs[1], *e = bufs[2], *r = bufs[3], *z = bufs[4];
    for (size_t it = 0; it < iterates && st == FX_OK; it++) {
        // e = u - x; samples from (x, e); then one plain cycle: x += M (b - A x)
        st = fx_waxpy(ctx, 1.0, u, -1.0, x, e);
        const size_t room = d->cap - d->count;
        const size_t k = std::min(room, patches_per_iterate);
        if (st == FX_OK && k) {
            org.resize(2 * k);
            for (size_t j = 0; j < k; j++) {
                org[2 * j] = (int)(2 * ry(rng));
                org[2 * j + 1] = (int)(2 * rx(rng));
            }
            st = fx_lsm_data_add_patches(d, op, x, e, b, omega, org.data(), k);
            if (st == FX_OK) *added += k;
        }
        if (st == FX_OK) st = fx_op_apply(op, x, r);
        if (st == FX_OK) st = fx_waxpy(ctx, 1.0, b, -1.0, r, r);
        if (st == FX_OK) st = fx_fill(ctx, z, 0.0);
        if (st == FX_OK) st = fx_precond_apply(fx_cdmg_as_precond(mg), z, r);
        if (st == FX_OK) st = fx_axpy(ctx, 1.0, z, x);
    }
    for (auto *p : bufs) fx_free(p);
    if (solver) fx_fgmres_destroy(solver);
    fx_cdmg_destroy(mg);
    return st;
}

int fx_precond_inner_pcg_f32(fx_ctx *ctx, const fx_grid *g, double coeff, const fx_stencil *st,
                             const fx_boundaries *bc, fx_precond *inner_f32, double rel_tol, size_t max_iter,
                             fx_precond **out) {
    if (!ctx || !g || !st || !bc || !inner_f32 || !out) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    if (!(rel_tol > 0.0 && rel_tol < 1.0)) return fail(FX_ERR_INVALID_ARGUMENT, "rel_tol must lie in (0, 1)");
    if (max_iter < 1) return fail(FX_ERR_INVALID_ARGUMENT, "max_iter must be at least 1");
    *out = nullptr;
    InnerPcgF32Pc *p = new InnerPcgF32Pc();
    p->ctx = ctx;
    p->g = *g;
    p->coeff = coeff;
    p->inner = inner_f32;
    p->rel_tol = rel_tol;
    p->max_iter = max_iter;
    int rc = prep_op(*g, st, bc, &p->P);
    if (rc == FX_OK) rc = create_solver(ctx, g, 0.0, max_iter, 4, &p->cg, FX_F32);
    if (rc == FX_OK) rc = fx_alloc(ctx, g->rows * g->cols, FX_F32, &p->r32);
    if (rc == FX_OK) rc = fx_alloc(ctx, g->rows * g->cols, FX_F32, &p->d32);
    if (rc != FX_OK) {
        delete p;
        return rc;
    }
    *out = p;
    return FX_OK;
}

int fx_precond_inner_pcg_f32_stats(const fx_precond *pc, size_t *applications, size_t *inner_iterations) {
    const InnerPcgF32Pc *p = dynamic_cast<const InnerPcgF32Pc *>(pc);
    if (!p || !applications || !inner_iterations)
        return fail(FX_ERR_INVALID_ARGUMENT, "not an inner FP32 PCG preconditioner");
    *applications = p->calls;
    *inner_iterations = p->total;
    return FX_OK;
}

int fx_precond_inner_cg(fx_ctx *ctx, const fx_grid *g, double coeff, const fx_stencil *st, const fx_boundaries *bc,
                        const size_t *steps, size_t nsteps, fx_precond *inner, fx_precond **out) {
    if (!ctx || !g || !st || !bc || !steps || !out) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    if (nsteps == 0) return fail(FX_ERR_INVALID_ARGUMENT, "empty step schedule");
    if (st->n < 1 || !st->dr || !st->dc || !st->w) return fail(FX_ERR_INVALID_ARGUMENT, "empty stencil");
    *out = nullptr;
    InnerCgPc *p = new InnerCgPc();
    p->ctx = ctx;
    p->inner = inner;
    p->coeff = coeff;
    p->dr.assign(st->dr, st->dr + st->n);
    p->dc.assign(st->dc, st->dc + st->n);
    p->wt.assign(st->w, st->w + st->n);
    p->bc = *bc;
    p->steps.assign(steps, steps + nsteps);
    const int rc = fx_cg_create(ctx, g, 0.0, steps[0], &p->cg);
    if (rc) {
        delete p;
        return rc;
    }
    *out = p;
    return FX_OK;
}

}  // extern "C"
