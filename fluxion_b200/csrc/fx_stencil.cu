// fx_stencil.cu -- stencil apply / fused stencil+AXPY / variable-coefficient stencil,
// upwind convection-diffusion, boundary ring, and the multigrid grid-transfer and
// smoothing primitives.  All grid kernels use the row-marching framework
// (fx_internal.cuh): one HBM read per element of the marched field.
#include "fx_points.cuh"
#include "fx_wcycle.cuh"

using namespace fx;

FX_CHECK_FILE(stencil);

namespace {

// ------------------------------------------------ five-point stencil as a strip march
//
// apply_stencil and stencil_axpy with the five-point stencil (constant coefficient) take a leaner
// path than the band march: a warp owns a strip of 64 columns (two per lane: lanes 1..30 own
// theirs, lanes 0 and 31 hold the halo columns) and marches it down a chunk of rows.  Each lane
// keeps its columns' rows q-2, q-1, q in registers; west / east neighbours come by one shuffle
// each; the rows ahead (of x, and of y for the axpy) are loaded sstrip_d rows early into a
// register FIFO.  The march is unrolled by that many rows, so every FIFO slot is a compile-time register, and a
// step whose rows all lie inside the grid and the chunk takes a path without row tests.  No block
// barrier and no shared-memory ring.  Every value is stencil_eval's expression (ops.rs:923-935
// nesting), so the result equals the band march's bit for bit.
constexpr int kSOwn = 60;  // own columns per strip
constexpr int kSWarps = 8;
// rows in flight (= the unroll): 6 for FP32, 4 for FP64 (6 spills under the register caps)
#ifndef FX_SSTRIP_F32_D
#define FX_SSTRIP_F32_D 6
#endif
template <typename T>
__host__ __device__ constexpr int sstrip_d() {
    return sizeof(T) == 4 ? FX_SSTRIP_F32_D : 4;
}
// FP64 five-point ops keep the band march (FX_SSTRIP_F64 = 1 switches them to the strip march):
// on a 16384^2 grid the strip march gave 0.80 / 0.95 of HBM bandwidth for the FP64 stencil /
// stencil-AXPY against the band march's 0.88 / 1.00, and 0.81 / 0.85 for FP32 against 0.64 / 0.62.
#ifndef FX_SSTRIP_F64
#define FX_SSTRIP_F64 0
#endif

// resident blocks per SM the launch bound asks for (the register cap: 64 / 85 / 85 / 128)
template <typename T, bool AXPY>
constexpr int sstrip_minb() {
    return sizeof(T) == 4 ? (AXPY ? 3 : 4) : (AXPY ? 2 : 3);
}

template <typename T, bool AXPY>
__global__ void __launch_bounds__(kSWarps * 32, sstrip_minb<T, AXPY>()) k_sstrip(StripGeom G, const T *__restrict__ x, T *__restrict__ out,
                                                         StencilP P, T alpha) {
    grid_dep_enter();
    constexpr int kSD = sstrip_d<T>();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int item = blockIdx.x * kSWarps + w;
    if (item >= G.nitems) return;  // whole warps
    const int strip = item % G.nstrips, chunk = item / G.nstrips;
    const int rows = G.rows, cols = G.cols;
    const int ca = strip * kSOwn - 1 + 2 * lane, cb = ca + 1;
    const bool lda = ca >= 0 && ca < cols, ldb = cb >= 0 && cb < cols;
    const bool own = lane >= 1 && lane <= 30;
    const bool sta = own && ca >= 1 && ca <= cols - 2, stb = own && cb >= 1 && cb <= cols - 2;
    const int r0 = chunk * G.chunk_rows, r1 = min(r0 + G.chunk_rows, rows);
    const int rlo = max(r0, 1), rhi = min(r1, rows - 1);  // output rows [rlo, rhi)
    const long long n = (long long)rows * cols;
    (void)n;
    const T pc = (T)P.c, pn = (T)P.n, ps = (T)P.s, pw = (T)P.w, pe = (T)P.e;
    // step q: row q + kSD is fetched, row q leaves the FIFO, row q - 1 is computed; rows r0 - 1 .. r1
    // are read
    const int qa = r0 - 1, qb = r1;
    // steps with every row test true: q - 1 in [rlo, rhi) and q + kSD <= min(qb, rows - 1)
    const int q_lo = rlo + 1, q_hi = min(rhi, min(qb, rows - 1) - kSD);
    T fa[kSD], fb[kSD], ga[kSD], gb[kSD];  // FIFO rows of x (f) and y (g)
    auto fetch = [&](int k, int q, long long o, bool fast) {
        const bool rv = fast || (q >= 0 && q < rows && q <= qb);
        if (!fast) {
            fa[k] = fb[k] = (T)0;
            if (AXPY) ga[k] = gb[k] = (T)0;
        }
        if (rv && lda && FX_IN(o, n)) {
            fa[k] = x[o];
            if (AXPY) ga[k] = out[o];
        }
        if (rv && ldb && FX_IN(o + 1, n)) {
            fb[k] = x[o + 1];
            if (AXPY) gb[k] = out[o + 1];
        }
    };
#pragma unroll
    for (int k = 0; k < kSD; k++) fetch(k, qa + k, (long long)(qa + k) * cols + ca, false);
    long long of = (long long)(qa + kSD) * cols + ca;  // element offset of (q + kSD, ca)
    long long oo = (long long)(qa - 1) * cols + ca;    // element offset of (q - 1, ca)
    T xna = (T)0, xnb = (T)0, xca = (T)0, xcb = (T)0, yca = (T)0, ycb = (T)0;
    auto step = [&](int k, int q, auto fast) {
        constexpr bool F = decltype(fast)::value;
        const T xsa = fa[k], xsb = fb[k];
        T ysa = (T)0, ysb = (T)0;
        if (AXPY) {
            ysa = ga[k];
            ysb = gb[k];
        }
        fetch(k, q + kSD, of, F);
        of += cols;
        if (F || (q - 1 >= rlo && q - 1 < rhi)) {  // uniform over the warp
            const T wa = shfl_w(xcb), eb = shfl_e(xca);
            const T va = fx_fma(pc, xca, fx_fma(pn, xna, fx_fma(ps, xsa, fx_fma(pw, wa, pe * xcb))));
            const T vb = fx_fma(pc, xcb, fx_fma(pn, xnb, fx_fma(ps, xsb, fx_fma(pw, xca, pe * eb))));
            if (sta && FX_IN(oo, n)) out[oo] = AXPY ? fx_fma(alpha, va, yca) : va;
            if (stb && FX_IN(oo + 1, n)) out[oo + 1] = AXPY ? fx_fma(alpha, vb, ycb) : vb;
        }
        oo += cols;
        xna = xca;
        xnb = xcb;
        xca = xsa;
        xcb = xsb;
        yca = ysa;
        ycb = ysb;
    };
    for (int q0 = qa; q0 <= qb; q0 += kSD) {
        if (q0 >= q_lo && q0 + kSD - 1 <= q_hi) {
#pragma unroll
            for (int k = 0; k < kSD; k++) step(k, q0 + k, fast_t<true>{});
        } else {
#pragma unroll
            for (int k = 0; k < kSD; k++) {
                if (q0 + k > qb) break;  // uniform over the warp
                step(k, q0 + k, fast_t<false>{});
            }
        }
    }
}

template <typename T, bool AXPY>
int launch_sstrip(fx_ctx *ctx, size_t rows, size_t cols, const T *x, T *out, const StencilP &P, T alpha,
                  const char *what) {
    static std::atomic<int> occ{0};
    const long cap = (long)band_capacity(ctx, k_sstrip<T, AXPY>, occ, kSWarps * 32) * kSWarps;
    const StripGeom G = strip_geom(rows, cols, kSOwn, cap);
    const int blocks = (G.nitems + kSWarps - 1) / kSWarps;
    timing_pre(ctx, what);
    launch_pdl(ctx, k_sstrip<T, AXPY>, blocks, kSWarps * 32, 0, G, x, out, P, alpha);
    timing_post(ctx, (double)rows * (double)cols);
    return check_launch(ctx, what);
}

// Boundary ring of apply_stencil / apply_stencil_var (ops.rs:796-843): top and bottom rows
// (corners included) first, then the left and right columns of rows 1..rows-2; each value
// from the point itself and its inward neighbour.  The interior is written by the band
// kernel, so the two writes never overlap.
template <typename T, bool VAR>
__global__ void k_ring_values(const T *__restrict__ in, T *__restrict__ out, const T *__restrict__ coeff,
                              int rows, int cols, BcP B) {
    const int nring = 2 * cols + 2 * (rows - 2);
    const long long n = (long long)rows * cols;
    (void)n;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nring; i += gridDim.x * blockDim.x) {
        size_t idx, nb;  // the point and its inward neighbour
        int side;
        double h;
        if (i < cols) {
            idx = i;
            nb = idx + cols;
            side = 0;
            h = B.dy;
        } else if (i < 2 * cols) {
            idx = (size_t)(rows - 1) * cols + (i - cols);
            nb = idx - cols;
            side = 1;
            h = B.dy;
        } else {
            const int j = i - 2 * cols;
            const size_t r = 1 + j / 2;
            if (j & 1) {
                idx = r * cols + cols - 1;
                nb = idx - 1;
                side = 3;
            } else {
                idx = r * cols;
                nb = idx + 1;
                side = 2;
            }
            h = B.dx;
        }
        if (!(FX_IN(idx, n) && FX_IN(nb, n))) continue;
        const double v = bc_value(B, side, (double)in[idx], (double)in[nb], h);
        T o = (T)v;
        if (VAR) o = o * coeff[idx];
        out[idx] = o;
    }
}

template <typename T, bool VAR>
int ring_values(fx_ctx *ctx, const T *in, T *out, const T *coeff, int rows, int cols, const BcP &B) {
    const int nring = 2 * cols + 2 * (rows - 2);
    const int blocks = (nring + 255) / 256;
    timing_pre(ctx, "ring_values");
    k_ring_values<T, VAR><<<blocks, 256, 0, ctx->stream>>>(in, out, coeff, rows, cols, B);
    timing_post(ctx, (double)nring);
    return check_launch(ctx, "ring_values");
}

// Reference weighted_jacobi (ops.rs:425-473): an in-place lexicographic sweep.  Executed
// as a wavefront over hyperplanes 2r + c = t: for radius-1 stencils every neighbour that
// the lexicographic order updates first lies on an earlier hyperplane and every later one
// on a later hyperplane, so each point sees exactly the values the sequential sweep sees.
template <typename T>
__global__ void __launch_bounds__(1024) k_lex_jacobi(T *x, const T *__restrict__ b, int rows, int cols,
                                                     StencilP P, double omega, double inv_diag) {
    const int tmin = 3, tmax = 2 * (rows - 2) + (cols - 2);
    const T om = (T)omega, id = (T)inv_diag;
    for (int t = tmin; t <= tmax; t++) {
        int rlo = (t - (cols - 2) + 1) / 2;
        if (rlo < 1) rlo = 1;
        int rhi = (t - 1) / 2;
        if (rhi > rows - 2) rhi = rows - 2;
        for (int r = rlo + (int)threadIdx.x; r <= rhi; r += blockDim.x) {
            const int c = t - 2 * r;
            const size_t idx = (size_t)r * cols + c;
            if (!FX_IN(idx, (long long)rows * cols)) continue;
            T ax = (T)0;
            for (int k = 0; k < P.ne_; k++) {
                const int dr = P.gi[k] / 3 - 1, dc = P.gi[k] % 3 - 1;
                const long long j = (long long)idx + (long long)dr * cols + dc;
                if (FX_IN(j, (long long)rows * cols)) ax = fx_fma((T)P.gw[k], x[j], ax);
            }
            const T residual = b[idx] - ax;
            x[idx] = fx_fma(om, id * residual, x[idx]);
        }
        __syncthreads();
    }
}

int pre_grid2(fx_ctx *ctx, const fx_buf *a, const fx_buf *b, const fx_grid *g) {
    if (!ctx) return fail(FX_ERR_INVALID_ARGUMENT, "null context");
    FX_TRY(check_grid(g));
    FX_TRY(check_buf(a, "input"));
    FX_TRY(check_buf(b, "output"));
    FX_TRY(check_grid_len(g, a));
    FX_TRY(check_grid_len(g, b));
    if (a->dtype != b->dtype) return fail(FX_ERR_INVALID_ARGUMENT, "dtype mismatch between buffers");
    if (a->ptr == b->ptr) return fail(FX_ERR_INVALID_ARGUMENT, "input and output must be distinct buffers");
    return FX_OK;
}

int pre_vec(const fx_buf *ref, const fx_buf *b, const char *name) {
    FX_TRY(check_buf(b, name));
    return check_same(ref, b);
}

}  // namespace

extern "C" {

int fx_apply_stencil(fx_ctx *ctx, const fx_buf *in, fx_buf *out, const fx_grid *g, const fx_stencil *s,
                     const fx_boundaries *bc) {
    FX_TRY(pre_grid2(ctx, in, out, g));
    BcP B;
    FX_TRY(make_bc(bc, g->dx, g->dy, &B, true));
    StencilP P;
    FX_TRY(make_stencil(s, &P));
    FX_DISPATCH(in->dtype, {
        const size_t RR = g->rows, CC = g->cols;
        if (P.mode == 5 && (sizeof(T) == 4 || FX_SSTRIP_F64)) {
            FX_TRY((launch_sstrip<T, false>(ctx, RR, CC, (const T *)in->ptr, (T *)out->ptr, P, (T)0,
                                            "apply_stencil")));
        } else {
            FX_MODE_DISPATCH(P.mode, {
                PtApply<T, MODE, false> pt{(T *)out->ptr, nullptr, P, B, (int)RR, (int)CC};
                FX_TRY(launch_march<T, 0>(ctx, RR, CC, LoadArr<T>{(const T *)in->ptr}, pt, NoFin{}, nullptr,
                                          "apply_stencil"));
            });
        }
        return ring_values<T, false>(ctx, (const T *)in->ptr, (T *)out->ptr, nullptr, (int)RR, (int)CC, B);
    });
}

int fx_apply_stencil_var(fx_ctx *ctx, const fx_buf *in, fx_buf *out, const fx_buf *coeff, const fx_grid *g,
                         const fx_stencil *s, const fx_boundaries *bc) {
    FX_TRY(pre_grid2(ctx, in, out, g));
    FX_TRY(pre_vec(in, coeff, "coeff"));
    BcP B;
    FX_TRY(make_bc(bc, g->dx, g->dy, &B, true));
    StencilP P;
    FX_TRY(make_stencil(s, &P));
    FX_DISPATCH(in->dtype, {
        const size_t RR = g->rows, CC = g->cols;
        FX_MODE_DISPATCH(P.mode, {
            PtApply<T, MODE, true> pt{(T *)out->ptr, (const T *)coeff->ptr, P, B, (int)RR, (int)CC};
            FX_TRY(launch_march<T, 0>(ctx, RR, CC, LoadArr<T>{(const T *)in->ptr}, pt, NoFin{}, nullptr,
                                      "apply_stencil_var"));
        });
        return ring_values<T, true>(ctx, (const T *)in->ptr, (T *)out->ptr, (const T *)coeff->ptr, (int)RR,
                                    (int)CC, B);
    });
}

int fx_stencil_axpy(fx_ctx *ctx, double alpha, const fx_buf *x, fx_buf *y, const fx_grid *g,
                    const fx_stencil *s, const fx_boundaries *bc) {
    FX_TRY(pre_grid2(ctx, x, y, g));
    BcP B;
    FX_TRY(make_bc(bc, g->dx, g->dy, &B, true));
    StencilP P;
    FX_TRY(make_stencil(s, &P));
    FX_DISPATCH(x->dtype, {
        const size_t RR = g->rows, CC = g->cols;
        if (P.mode == 5 && (sizeof(T) == 4 || FX_SSTRIP_F64))
            return launch_sstrip<T, true>(ctx, RR, CC, (const T *)x->ptr, (T *)y->ptr, P, (T)alpha, "stencil_axpy");
        FX_MODE_DISPATCH(P.mode, {
            PtAxpy<T, MODE> pt{(T *)y->ptr, P, (T)alpha, (int)RR, (int)CC};
            return launch_march<T, 0>(ctx, RR, CC, LoadArr<T>{(const T *)x->ptr}, pt, NoFin{}, nullptr,
                                         "stencil_axpy");
        });
    });
}

int fx_zero_boundaries(fx_ctx *ctx, fx_buf *buf, size_t rows, size_t cols) {
    if (!ctx) return fail(FX_ERR_INVALID_ARGUMENT, "null context");
    FX_TRY(check_buf(buf, "buf"));
    if (rows < 1 || cols < 1 || rows * cols != buf->len)
        return fail(FX_ERR_DIMENSION_MISMATCH, "dimension mismatch: expected " + std::to_string(rows * cols) +
                                                   ", got " + std::to_string(buf->len));
    const size_t nring = 2 * cols + 2 * (rows > 2 ? rows - 2 : 0);
    FX_DISPATCH(buf->dtype, {
        T *p = (T *)buf->ptr;
        return launch_flat<0>(ctx, nring,
                              [=] __device__(size_t i, CSum *) {
                                  size_t idx;
                                  if (i < cols) idx = i;
                                  else if (i < 2 * cols) idx = (rows - 1) * cols + (i - cols);
                                  else {
                                      const size_t j = i - 2 * cols;
                                      const size_t r = 1 + j / 2;
                                      idx = r * cols + ((j & 1) ? cols - 1 : 0);
                                  }
                                  p[idx] = (T)0;
                              },
                              NoFin{}, nullptr, "zero_boundaries");
    });
}

int fx_apply_conv_diff(fx_ctx *ctx, const fx_buf *u, fx_buf *out, const fx_buf *kappa, const fx_buf *vx,
                       const fx_buf *vy, const fx_grid *g, const fx_boundaries *) {
    FX_TRY(pre_grid2(ctx, u, out, g));
    FX_TRY(pre_vec(u, kappa, "kappa"));
    FX_TRY(pre_vec(u, vx, "vx"));
    FX_TRY(pre_vec(u, vy, "vy"));
    FX_DISPATCH(u->dtype, {
        const size_t RR = g->rows, CC = g->cols;
        PtConvDiff<T, false> pt{(T *)out->ptr, (const T *)kappa->ptr, (const T *)vx->ptr, (const T *)vy->ptr,
                                conv_consts<T>(g->dx, g->dy), (T)0, (int)RR, (int)CC};
        return launch_march<T, 0>(ctx, RR, CC, LoadArr<T>{(const T *)u->ptr}, pt, NoFin{}, nullptr,
                                     "apply_conv_diff");
    });
}

int fx_conv_diff_axpy(fx_ctx *ctx, double alpha, const fx_buf *u, fx_buf *out, const fx_buf *kappa,
                      const fx_buf *vx, const fx_buf *vy, const fx_grid *g, const fx_boundaries *) {
    FX_TRY(pre_grid2(ctx, u, out, g));
    FX_TRY(pre_vec(u, kappa, "kappa"));
    FX_TRY(pre_vec(u, vx, "vx"));
    FX_TRY(pre_vec(u, vy, "vy"));
    FX_DISPATCH(u->dtype, {
        const size_t RR = g->rows, CC = g->cols;
        PtConvDiff<T, true> pt{(T *)out->ptr, (const T *)kappa->ptr, (const T *)vx->ptr, (const T *)vy->ptr,
                               conv_consts<T>(g->dx, g->dy), (T)alpha, (int)RR, (int)CC};
        return launch_march<T, 0>(ctx, RR, CC, LoadArr<T>{(const T *)u->ptr}, pt, NoFin{}, nullptr,
                                     "conv_diff_axpy");
    });
}

// ---------------------------------------------------------------- multigrid, reference semantics

int fx_restrict(fx_ctx *ctx, const fx_buf *fine, fx_buf *coarse, const fx_grid *fg, const fx_grid *cg) {
    if (!ctx || !fg || !cg) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    FX_TRY(check_buf(fine, "fine"));
    FX_TRY(check_buf(coarse, "coarse"));
    FX_TRY(check_grid_len(fg, fine));
    FX_TRY(check_grid_len(cg, coarse));
    if (fine->dtype != coarse->dtype) return fail(FX_ERR_INVALID_ARGUMENT, "dtype mismatch between buffers");
    const size_t frows = fg->rows, fcols = fg->cols, crows = cg->rows, ccols = cg->cols;
    // ops.rs:380-395 indexes fine[2*row] unchecked (a panic past the fine grid).
    if (crows == 0 || ccols == 0 || 2 * (crows - 1) > frows - 1 || 2 * (ccols - 1) > fcols - 1)
        return fail(FX_ERR_DIMENSION_MISMATCH, "restrict: coarse grid does not fit the fine grid");
    FX_DISPATCH(fine->dtype, {
        const T *f = (const T *)fine->ptr;
        T *c = (T *)coarse->ptr;
        return launch_flat<0>(ctx, crows * ccols,
                              [=] __device__(size_t i, CSum *) {
                                  const size_t row = i / ccols, col = i % ccols;
                                  const size_t fr = row * 2, fcc = col * 2;
                                  const size_t fr1 = fr + 1 < frows - 1 ? fr + 1 : frows - 1;
                                  const size_t fc1 = fcc + 1 < fcols - 1 ? fcc + 1 : fcols - 1;
                                  c[i] = (T)0.25 * (((f[fr * fcols + fcc] + f[fr1 * fcols + fcc]) +
                                                     f[fr * fcols + fc1]) + f[fr1 * fcols + fc1]);
                              },
                              NoFin{}, nullptr, "restrict");
    });
}

int fx_prolong(fx_ctx *ctx, const fx_buf *coarse, fx_buf *fine, const fx_grid *cg, const fx_grid *fg) {
    if (!ctx || !fg || !cg) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    FX_TRY(check_buf(fine, "fine"));
    FX_TRY(check_buf(coarse, "coarse"));
    FX_TRY(check_grid_len(fg, fine));
    FX_TRY(check_grid_len(cg, coarse));
    if (fine->dtype != coarse->dtype) return fail(FX_ERR_INVALID_ARGUMENT, "dtype mismatch between buffers");
    const size_t frows = fg->rows, fcols = fg->cols, crows = cg->rows, ccols = cg->cols;
    // ops.rs:413-420 indexes coarse[row/2] unchecked (a panic past the coarse grid).
    if ((frows - 1) / 2 > crows - 1 || (fcols - 1) / 2 > ccols - 1)
        return fail(FX_ERR_DIMENSION_MISMATCH, "prolong: fine grid maps outside the coarse grid");
    FX_DISPATCH(fine->dtype, {
        const T *c = (const T *)coarse->ptr;
        T *f = (T *)fine->ptr;
        return launch_flat<0>(ctx, frows * fcols,
                              [=] __device__(size_t i, CSum *) {
                                  const size_t row = i / fcols, col = i % fcols;
                                  f[i] += c[(row / 2) * ccols + col / 2];
                              },
                              NoFin{}, nullptr, "prolong");
    });
}

int fx_weighted_jacobi(fx_ctx *ctx, fx_buf *x, const fx_buf *b, double omega, const fx_grid *g,
                       const fx_stencil *s, const fx_boundaries *) {
    if (!ctx) return fail(FX_ERR_INVALID_ARGUMENT, "null context");
    FX_TRY(check_grid(g));
    FX_TRY(check_buf(x, "x"));
    FX_TRY(check_buf(b, "b"));
    FX_TRY(check_grid_len(g, x));
    FX_TRY(check_grid_len(g, b));
    if (x->dtype != b->dtype) return fail(FX_ERR_INVALID_ARGUMENT, "dtype mismatch between buffers");
    if (!s || s->n < 1) return fail(FX_ERR_INVALID_STENCIL, "invalid stencil: stencil must have at least one entry");
    // ops.rs:440-457 uses the entry list in order (no 5/9-point fast path) -> generic form.
    StencilP P;
    std::memset(&P, 0, sizeof(P));
    if (s->n > kMaxGeneric) return fail(FX_ERR_INVALID_STENCIL, "invalid stencil: more than 27 entries");
    double diag = -4.0;
    bool found = false;
    for (int k = 0; k < s->n; k++) {
        if (s->dr[k] < -1 || s->dr[k] > 1 || s->dc[k] < -1 || s->dc[k] > 1)
            return fail(FX_ERR_INVALID_STENCIL, "invalid stencil: offsets beyond radius 1");
        P.gi[k] = (signed char)((s->dr[k] + 1) * 3 + (s->dc[k] + 1));
        P.gw[k] = s->w[k];
        if (!found && s->dr[k] == 0 && s->dc[k] == 0) {
            diag = s->w[k];
            found = true;
        }
    }
    P.ne_ = s->n;
    const double inv_diag = 1.0 / diag;
    FX_DISPATCH(x->dtype, {
        k_lex_jacobi<T><<<1, 1024, 0, ctx->stream>>>((T *)x->ptr, (const T *)b->ptr, (int)g->rows,
                                                      (int)g->cols, P, omega, inv_diag);
        return check_launch(ctx, "weighted_jacobi");
    });
}

// ---------------------------------------------------------------- vertex-centred primitives

int fx_jacobi_sweep(fx_ctx *ctx, const fx_buf *x_in, fx_buf *x_out, const fx_buf *b, double omega, size_t rows,
                    size_t cols, const double a5[5]) {
    if (!ctx || !a5) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    fx_grid g{rows, cols, 1.0, 1.0};
    FX_TRY(pre_grid2(ctx, x_in, x_out, &g));
    FX_TRY(pre_vec(x_in, b, "b"));
    const double wd = omega / a5[0];
    FX_DISPATCH(x_in->dtype, {
        const size_t RR = rows, CC = cols;
        PtJacobi<T> pt{(T *)x_out->ptr, (const T *)b->ptr, make_a5<T>(a5), (T)wd, (int)RR, (int)CC};
        return launch_march<T, 0>(ctx, RR, CC, LoadArr<T>{(const T *)x_in->ptr}, pt, NoFin{}, nullptr,
                                     "jacobi_sweep");
    });
}

int fx_residual5(fx_ctx *ctx, const fx_buf *x, const fx_buf *b, fx_buf *r, size_t rows, size_t cols,
                 const double a5[5]) {
    if (!ctx || !a5) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    fx_grid g{rows, cols, 1.0, 1.0};
    FX_TRY(pre_grid2(ctx, x, r, &g));
    FX_TRY(pre_vec(x, b, "b"));
    FX_DISPATCH(x->dtype, {
        const size_t RR = rows, CC = cols;
        PtResidual<T> pt{(T *)r->ptr, (const T *)b->ptr, make_a5<T>(a5), (int)RR, (int)CC};
        return launch_march<T, 0>(ctx, RR, CC, LoadArr<T>{(const T *)x->ptr}, pt, NoFin{}, nullptr, "residual5");
    });
}

int fx_restrict_fw(fx_ctx *ctx, const fx_buf *fine, fx_buf *coarse, size_t frows, size_t fcols, size_t crows,
                   size_t ccols) {
    if (!ctx) return fail(FX_ERR_INVALID_ARGUMENT, "null context");
    FX_TRY(check_buf(fine, "fine"));
    FX_TRY(check_buf(coarse, "coarse"));
    if (crows < 3 || ccols < 3 || frows != 2 * (crows - 1) + 1 || fcols != 2 * (ccols - 1) + 1 ||
        fine->len != frows * fcols || coarse->len != crows * ccols)
        return fail(FX_ERR_DIMENSION_MISMATCH, "restrict_fw: grids are not a vertex-centred pair");
    if (fine->dtype != coarse->dtype) return fail(FX_ERR_INVALID_ARGUMENT, "dtype mismatch between buffers");
    FX_DISPATCH(fine->dtype, {
        const T *f = (const T *)fine->ptr;
        T *c = (T *)coarse->ptr;
        return launch_flat<0>(ctx, crows * ccols,
                              [=] __device__(size_t i, CSum *) {
                                  const size_t I = i / ccols, J = i % ccols;
                                  if (I == 0 || J == 0 || I == crows - 1 || J == ccols - 1) {
                                      c[i] = (T)0;
                                      return;
                                  }
                                  const size_t k = (2 * I) * fcols + 2 * J;
                                  const T e = (f[k - fcols] + f[k + fcols]) + (f[k - 1] + f[k + 1]);
                                  const T d = (f[k - fcols - 1] + f[k - fcols + 1]) + (f[k + fcols - 1] + f[k + fcols + 1]);
                                  c[i] = ((T)4 * f[k] + ((T)2 * e + d)) * (T)0.0625;
                              },
                              NoFin{}, nullptr, "restrict_fw");
    });
}

int fx_prolong_bilinear(fx_ctx *ctx, const fx_buf *coarse, fx_buf *fine, size_t crows, size_t ccols, size_t frows,
                        size_t fcols) {
    if (!ctx) return fail(FX_ERR_INVALID_ARGUMENT, "null context");
    FX_TRY(check_buf(fine, "fine"));
    FX_TRY(check_buf(coarse, "coarse"));
    if (crows < 3 || ccols < 3 || frows != 2 * (crows - 1) + 1 || fcols != 2 * (ccols - 1) + 1 ||
        fine->len != frows * fcols || coarse->len != crows * ccols)
        return fail(FX_ERR_DIMENSION_MISMATCH, "prolong_bilinear: grids are not a vertex-centred pair");
    if (fine->dtype != coarse->dtype) return fail(FX_ERR_INVALID_ARGUMENT, "dtype mismatch between buffers");
    FX_DISPATCH(fine->dtype, {
        const T *c = (const T *)coarse->ptr;
        T *f = (T *)fine->ptr;
        const size_t iw = fcols - 2;
        return launch_flat<0>(ctx, (frows - 2) * (fcols - 2),
                              [=] __device__(size_t q, CSum *) {
                                  const size_t i = 1 + q / iw, j = 1 + q % iw;
                                  const size_t k = (i / 2) * ccols + (j / 2);
                                  T e;
                                  if (!(i & 1) && !(j & 1)) e = c[k];
                                  else if ((i & 1) && !(j & 1)) e = (T)0.5 * (c[k] + c[k + ccols]);
                                  else if (!(i & 1) && (j & 1)) e = (T)0.5 * (c[k] + c[k + 1]);
                                  else e = (T)0.25 * ((c[k] + c[k + ccols]) + (c[k + 1] + c[k + ccols + 1]));
                                  f[i * fcols + j] += e;
                              },
                              NoFin{}, nullptr, "prolong_bilinear");
    });
}

}  // extern "C"
