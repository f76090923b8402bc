// fx_blas1.cu -- BLAS-1 vector ops and deterministic compensated reductions.
//
// Elementwise semantics follow crates/backend-cpu/src/ops.rs (the same fma nesting, so
// F64 results are bitwise equal to the CPU backend).  Reductions replace the CPU's
// Kahan-per-4096-chunk + rayon merge (ops.rs:271-367) with TwoSum/TwoProduct compensated
// per-thread sums, a fixed warp-shuffle tree and a last-block fold of the per-block
// partials in block order: faithful to about one ulp and bitwise deterministic.
#include "fx_internal.cuh"

using namespace fx;

#define FX_DISPATCH(dtype, ...)             \
    do {                                    \
        if ((dtype) == FX_F64) {            \
            using T = double;               \
            __VA_ARGS__;                    \
        } else {                            \
            using T = float;                \
            __VA_ARGS__;                    \
        }                                   \
    } while (0)

namespace {

// F32 fast path of the BLAS-1 ops that stream whole vectors: with 4-byte elements one access per
// thread and iteration keeps too few bytes in flight (axpy measured 0.75, dot2 0.61 of HBM), so when
// every pointer is 16-byte aligned each thread moves four elements per access (float4).  fv takes
// the vector index j (elements 4j .. 4j+3), fs the scalar index of the n % 4 tail elements, which
// the first threads of the grid take.  Elementwise results equal the scalar path's; the sums are
// deterministic for a given n.
template <int K, typename V, typename S, typename Fin>
__global__ void __launch_bounds__(kBlock) k_vec4(size_t n, V fv, S fs, Fin fin, RedArgs<K> ra) {
    grid_dep_enter();
    CSum acc[K > 0 ? K : 1];
#pragma unroll
    for (int k = 0; k < (K > 0 ? K : 1); k++) acc[k] = CSum{0.0, 0.0};
    const size_t n4 = n / 4, stride = (size_t)gridDim.x * blockDim.x;
    const size_t gid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    for (size_t j = gid; j < n4; j += stride) fv(j, acc);
    if (4 * n4 + gid < n) fs(4 * n4 + gid, acc);
    if constexpr (K > 0) grid_reduce<K>(acc, ra, fin);
}

bool aligned16(const void *p) { return ((uintptr_t)p & 15u) == 0; }

template <int K, typename V, typename S, typename Fin>
int launch_vec4(fx_ctx *ctx, size_t n, V fv, S fs, Fin fin, const char *what) {
    FlatGeom g = flat_geom(ctx, (n + 3) / 4);
    if (g.blocks == 0) return FX_OK;
    timing_pre(ctx, what);
    launch_pdl(ctx, k_vec4<K, V, S, Fin>, g.blocks, kBlock, 0, n, fv, fs, fin, red_args<K>(ctx));
    timing_post(ctx, (double)n);
    return check_launch(ctx, what);
}

template <typename T>
__device__ __forceinline__ T tmax(T a, T b) { return fmax(a, b); }
template <>
__device__ __forceinline__ float tmax<float>(float a, float b) { return fmaxf(a, b); }
template <typename T>
__device__ __forceinline__ T tmin(T a, T b) { return fmin(a, b); }
template <>
__device__ __forceinline__ float tmin<float>(float a, float b) { return fminf(a, b); }

// max / min reduction (ops.rs:317-331, :657-671): f64::max/min ignore NaN, as fmax/fmin do.
template <typename T, bool IS_MAX>
__global__ void __launch_bounds__(kBlock) k_minmax(const T *__restrict__ x, size_t n, double *partials,
                                                   unsigned *counter, double *out) {
    __shared__ double sh[kBlock / 32];
    __shared__ bool is_last;
    double m = IS_MAX ? -INFINITY : INFINITY;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
        m = IS_MAX ? fmax(m, (double)x[i]) : fmin(m, (double)x[i]);
    auto wred = [&](double v) {
        for (int off = 16; off > 0; off >>= 1) {
            double o = __shfl_down_sync(0xffffffffu, v, off);
            v = IS_MAX ? fmax(v, o) : fmin(v, o);
        }
        return v;
    };
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    m = wred(m);
    if (lane == 0) sh[wid] = m;
    __syncthreads();
    if (wid == 0) {
        m = lane < (int)(blockDim.x >> 5) ? sh[lane] : (IS_MAX ? -INFINITY : INFINITY);
        m = wred(m);
        if (lane == 0) {
            partials[blockIdx.x] = m;
            __threadfence();
            is_last = atomicAdd(counter, 1u) == gridDim.x - 1;
        }
    }
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    double a = IS_MAX ? -INFINITY : INFINITY;
    for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
        double v = ((volatile double *)partials)[b];
        a = IS_MAX ? fmax(a, v) : fmin(a, v);
    }
    a = wred(a);
    __syncthreads();
    if (lane == 0) sh[wid] = a;
    __syncthreads();
    if (threadIdx.x == 0) {
        double r = sh[0];
        for (int w = 1; w < (int)(blockDim.x >> 5); w++) r = IS_MAX ? fmax(r, sh[w]) : fmin(r, sh[w]);
        *out = r;
        *counter = 0u;
    }
}

template <bool IS_MAX>
int minmax(fx_ctx *ctx, const fx_buf *b, double *out) {
    FX_TRY(check_buf(b, "buf"));
    if (!out) return fail(FX_ERR_INVALID_ARGUMENT, "null out");
    if (b->len == 0) {
        *out = IS_MAX ? -INFINITY : INFINITY;
        return FX_OK;
    }
    FlatGeom g = flat_geom(ctx, b->len);
    FX_DISPATCH(b->dtype, (k_minmax<T, IS_MAX><<<g.blocks, kBlock, 0, ctx->stream>>>(
                              (const T *)b->ptr, b->len, ctx->d_partials, ctx->d_counter,
                              ctx->d_result)));
    FX_TRY(check_launch(ctx, "reduce_minmax"));
    return read_results(ctx, 1, out);
}

int pre2(fx_ctx *ctx, const fx_buf *x, const fx_buf *y) {
    if (!ctx) return fail(FX_ERR_INVALID_ARGUMENT, "null context");
    FX_TRY(check_buf(x, "x"));
    FX_TRY(check_buf(y, "y"));
    return check_same(x, y);
}

}  // namespace

extern "C" {

int fx_copy(fx_ctx *ctx, const fx_buf *src, fx_buf *dst) {
    FX_TRY(pre2(ctx, src, dst));
    if (src == dst || src->ptr == dst->ptr || !src->len) return FX_OK;
    FX_CUDA(cudaMemcpyAsync(dst->ptr, src->ptr, src->len * elem_size(src->dtype), cudaMemcpyDeviceToDevice,
                            ctx->stream));
    return FX_OK;
}

int fx_fill(fx_ctx *ctx, fx_buf *buf, double value) {
    if (!ctx) return fail(FX_ERR_INVALID_ARGUMENT, "null context");
    FX_TRY(check_buf(buf, "buf"));
    FX_DISPATCH(buf->dtype, {
        T *p = (T *)buf->ptr;
        const T v = (T)value;
        return launch_flat<0>(ctx, buf->len, [=] __device__(size_t i, CSum *) { p[i] = v; }, NoFin{},
                              nullptr, "fill");
    });
}

int fx_axpy(fx_ctx *ctx, double alpha, const fx_buf *x, fx_buf *y) {
    FX_TRY(pre2(ctx, x, y));
    FX_DISPATCH(x->dtype, {
        const T *xp = (const T *)x->ptr;
        T *yp = (T *)y->ptr;
        const T a = (T)alpha;
        if constexpr (sizeof(T) == 4) {
            if (aligned16(xp) && aligned16(yp) && x->len >= 4096)
                return launch_vec4<0>(
                    ctx, x->len,
                    [=] __device__(size_t j, CSum *) {
                        const float4 xv = reinterpret_cast<const float4 *>(xp)[j];
                        float4 yv = reinterpret_cast<float4 *>(yp)[j];
                        yv.x = fx_fma(a, xv.x, yv.x);
                        yv.y = fx_fma(a, xv.y, yv.y);
                        yv.z = fx_fma(a, xv.z, yv.z);
                        yv.w = fx_fma(a, xv.w, yv.w);
                        reinterpret_cast<float4 *>(yp)[j] = yv;
                    },
                    [=] __device__(size_t i, CSum *) { yp[i] = fx_fma(a, xp[i], yp[i]); }, NoFin{}, "axpy");
        }
        return launch_flat<0>(ctx, x->len, [=] __device__(size_t i, CSum *) { yp[i] = fx_fma(a, xp[i], yp[i]); },
                              NoFin{}, nullptr, "axpy");
    });
}

int fx_scale(fx_ctx *ctx, fx_buf *buf, double alpha) {
    if (!ctx) return fail(FX_ERR_INVALID_ARGUMENT, "null context");
    FX_TRY(check_buf(buf, "buf"));
    FX_DISPATCH(buf->dtype, {
        T *p = (T *)buf->ptr;
        const T a = (T)alpha;
        return launch_flat<0>(ctx, buf->len, [=] __device__(size_t i, CSum *) { p[i] = p[i] * a; }, NoFin{},
                              nullptr, "scale");
    });
}

int fx_waxpy(fx_ctx *ctx, double alpha, const fx_buf *x, double beta, const fx_buf *y, fx_buf *w) {
    FX_TRY(pre2(ctx, x, y));
    FX_TRY(check_buf(w, "w"));
    FX_TRY(check_same(x, w));
    FX_DISPATCH(x->dtype, {
        const T *xp = (const T *)x->ptr;
        const T *yp = (const T *)y->ptr;
        T *wp = (T *)w->ptr;
        const T a = (T)alpha, b = (T)beta;
        return launch_flat<0>(ctx, x->len,
                              [=] __device__(size_t i, CSum *) { wp[i] = fx_fma(a, xp[i], b * yp[i]); },
                              NoFin{}, nullptr, "waxpy");
    });
}

int fx_aypx(fx_ctx *ctx, double alpha, const fx_buf *x, fx_buf *y) {
    FX_TRY(pre2(ctx, x, y));
    FX_DISPATCH(x->dtype, {
        const T *xp = (const T *)x->ptr;
        T *yp = (T *)y->ptr;
        const T a = (T)alpha;
        return launch_flat<0>(ctx, x->len, [=] __device__(size_t i, CSum *) { yp[i] = fx_fma(a, yp[i], xp[i]); },
                              NoFin{}, nullptr, "aypx");
    });
}

#define FX_POINTWISE(NAME, EXPR)                                                                      \
    int NAME(fx_ctx *ctx, const fx_buf *x, const fx_buf *y, fx_buf *z) {                              \
        FX_TRY(pre2(ctx, x, y));                                                                      \
        FX_TRY(check_buf(z, "z"));                                                                    \
        FX_TRY(check_same(x, z));                                                                     \
        FX_DISPATCH(x->dtype, {                                                                       \
            const T *xp = (const T *)x->ptr;                                                          \
            const T *yp = (const T *)y->ptr;                                                          \
            T *zp = (T *)z->ptr;                                                                      \
            return launch_flat<0>(ctx, x->len,                                                        \
                                  [=] __device__(size_t i, CSum *) {                                  \
                                      const T a = xp[i], b = yp[i];                                   \
                                      zp[i] = (EXPR);                                                 \
                                  },                                                                  \
                                  NoFin{}, nullptr, #NAME);                                           \
        });                                                                                           \
    }

FX_POINTWISE(fx_pointwise_mult, a *b)
FX_POINTWISE(fx_pointwise_div, a / b)
FX_POINTWISE(fx_pointwise_max, tmax<T>(a, b))
FX_POINTWISE(fx_pointwise_min, tmin<T>(a, b))

int fx_reciprocal(fx_ctx *ctx, fx_buf *buf) {
    if (!ctx) return fail(FX_ERR_INVALID_ARGUMENT, "null context");
    FX_TRY(check_buf(buf, "buf"));
    FX_DISPATCH(buf->dtype, {
        T *p = (T *)buf->ptr;
        return launch_flat<0>(ctx, buf->len, [=] __device__(size_t i, CSum *) { p[i] = (T)1 / p[i]; },
                              NoFin{}, nullptr, "reciprocal");
    });
}

int fx_abs_val(fx_ctx *ctx, fx_buf *buf) {
    if (!ctx) return fail(FX_ERR_INVALID_ARGUMENT, "null context");
    FX_TRY(check_buf(buf, "buf"));
    FX_DISPATCH(buf->dtype, {
        T *p = (T *)buf->ptr;
        return launch_flat<0>(ctx, buf->len, [=] __device__(size_t i, CSum *) { p[i] = fabs(p[i]); }, NoFin{},
                              nullptr, "abs_val");
    });
}

// ---------------------------------------------------------------- reductions

int fx_norm_l2(fx_ctx *ctx, const fx_buf *buf, double *out) {
    if (!ctx || !out) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    FX_TRY(check_buf(buf, "buf"));
    if (!buf->len) {
        *out = 0.0;
        return FX_OK;
    }
    FX_DISPATCH(buf->dtype, {
        const T *p = (const T *)buf->ptr;
        FX_TRY(launch_flat<1>(ctx, buf->len,
                              [=] __device__(size_t i, CSum *acc) {
                                  csum_add_prod_t<T>(acc[0], p[i], p[i]);
                              },
                              StoreFin<1>{ctx->d_result}, nullptr, "norm_l2"));
    });
    FX_TRY(read_results(ctx, 1, out));
    *out = sqrt(*out);
    return FX_OK;
}

int fx_reduce_sum(fx_ctx *ctx, const fx_buf *buf, double *out) {
    if (!ctx || !out) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    FX_TRY(check_buf(buf, "buf"));
    if (!buf->len) {
        *out = 0.0;
        return FX_OK;
    }
    FX_DISPATCH(buf->dtype, {
        const T *p = (const T *)buf->ptr;
        FX_TRY(launch_flat<1>(ctx, buf->len, [=] __device__(size_t i, CSum *acc) { csum_add(acc[0], (double)p[i]); },
                              StoreFin<1>{ctx->d_result}, nullptr, "reduce_sum"));
    });
    return read_results(ctx, 1, out);
}

int fx_reduce_max(fx_ctx *ctx, const fx_buf *buf, double *out) { return minmax<true>(ctx, buf, out); }
int fx_reduce_min(fx_ctx *ctx, const fx_buf *buf, double *out) { return minmax<false>(ctx, buf, out); }

int fx_dot(fx_ctx *ctx, const fx_buf *x, const fx_buf *y, double *out) {
    FX_TRY(pre2(ctx, x, y));
    if (!out) return fail(FX_ERR_INVALID_ARGUMENT, "null out");
    if (!x->len) {
        *out = 0.0;
        return FX_OK;
    }
    FX_DISPATCH(x->dtype, {
        const T *xp = (const T *)x->ptr;
        const T *yp = (const T *)y->ptr;
        bool vec = false;
        if constexpr (sizeof(T) == 4) {
            if (aligned16(xp) && aligned16(yp) && x->len >= 4096) {
                vec = true;
                FX_TRY(launch_vec4<1>(
                    ctx, x->len,
                    [=] __device__(size_t j, CSum *acc) {
                        const float4 a = reinterpret_cast<const float4 *>(xp)[j];
                        const float4 b = reinterpret_cast<const float4 *>(yp)[j];
                        csum_add_prod_t<float>(acc[0], a.x, b.x);
                        csum_add_prod_t<float>(acc[0], a.y, b.y);
                        csum_add_prod_t<float>(acc[0], a.z, b.z);
                        csum_add_prod_t<float>(acc[0], a.w, b.w);
                    },
                    [=] __device__(size_t i, CSum *acc) { csum_add_prod_t<float>(acc[0], xp[i], yp[i]); },
                    StoreFin<1>{ctx->d_result}, "dot"));
            }
        }
        if (!vec)
            FX_TRY(launch_flat<1>(ctx, x->len,
                                  [=] __device__(size_t i, CSum *acc) { csum_add_prod_t<T>(acc[0], xp[i], yp[i]); },
                                  StoreFin<1>{ctx->d_result}, nullptr, "dot"));
    });
    return read_results(ctx, 1, out);
}

int fx_dot2(fx_ctx *ctx, const fx_buf *a, const fx_buf *b, const fx_buf *c, const fx_buf *d, double *ab,
            double *cd) {
    FX_TRY(pre2(ctx, a, b));
    FX_TRY(pre2(ctx, c, d));
    FX_TRY(check_same(a, c));
    if (!ab || !cd) return fail(FX_ERR_INVALID_ARGUMENT, "null out");
    if (!a->len) {
        *ab = *cd = 0.0;
        return FX_OK;
    }
    FX_DISPATCH(a->dtype, {
        const T *ap = (const T *)a->ptr;
        const T *bp = (const T *)b->ptr;
        const T *cp = (const T *)c->ptr;
        const T *dp = (const T *)d->ptr;
        bool vec = false;
        if constexpr (sizeof(T) == 4) {
            if (aligned16(ap) && aligned16(bp) && aligned16(cp) && aligned16(dp) && a->len >= 4096) {
                vec = true;
                FX_TRY(launch_vec4<2>(
                    ctx, a->len,
                    [=] __device__(size_t j, CSum *acc) {
                        const float4 va = reinterpret_cast<const float4 *>(ap)[j];
                        const float4 vb = reinterpret_cast<const float4 *>(bp)[j];
                        const float4 vc = reinterpret_cast<const float4 *>(cp)[j];
                        const float4 vd = reinterpret_cast<const float4 *>(dp)[j];
                        csum_add_prod_t<float>(acc[0], va.x, vb.x);
                        csum_add_prod_t<float>(acc[0], va.y, vb.y);
                        csum_add_prod_t<float>(acc[0], va.z, vb.z);
                        csum_add_prod_t<float>(acc[0], va.w, vb.w);
                        csum_add_prod_t<float>(acc[1], vc.x, vd.x);
                        csum_add_prod_t<float>(acc[1], vc.y, vd.y);
                        csum_add_prod_t<float>(acc[1], vc.z, vd.z);
                        csum_add_prod_t<float>(acc[1], vc.w, vd.w);
                    },
                    [=] __device__(size_t i, CSum *acc) {
                        csum_add_prod_t<float>(acc[0], ap[i], bp[i]);
                        csum_add_prod_t<float>(acc[1], cp[i], dp[i]);
                    },
                    StoreFin<2>{ctx->d_result}, "dot2"));
            }
        }
        if (!vec)
            FX_TRY(launch_flat<2>(ctx, a->len,
                                  [=] __device__(size_t i, CSum *acc) {
                                      csum_add_prod_t<T>(acc[0], ap[i], bp[i]);
                                      csum_add_prod_t<T>(acc[1], cp[i], dp[i]);
                                  },
                                  StoreFin<2>{ctx->d_result}, nullptr, "dot2"));
    });
    double v[2];
    FX_TRY(read_results(ctx, 2, v));
    *ab = v[0];
    *cd = v[1];
    return FX_OK;
}

// ---------------------------------------------------------------- pipelined-CG update

int fx_pcg_fused_update(fx_ctx *ctx, double alpha, double beta, fx_buf *z, fx_buf *t, fx_buf *p, fx_buf *x,
                        fx_buf *r, fx_buf *w, const fx_buf *q) {
    if (!ctx) return fail(FX_ERR_INVALID_ARGUMENT, "null context");
    const fx_buf *all[7] = {z, t, p, x, r, w, q};
    for (auto *b : all) {
        FX_TRY(check_buf(b, "pcg vector"));
        FX_TRY(check_same(z, b));
    }
    FX_DISPATCH(z->dtype, {
        T *zp = (T *)z->ptr, *tp = (T *)t->ptr, *pp = (T *)p->ptr, *xp = (T *)x->ptr, *rp = (T *)r->ptr,
          *wp = (T *)w->ptr;
        const T *qp = (const T *)q->ptr;
        const T a = (T)alpha, be = (T)beta;
        return launch_flat<0>(ctx, z->len,
                              [=] __device__(size_t i, CSum *) {
                                  // pipelined_cg.rs:440-456: scale then axpy(1, .) per vector
                                  const T zn = qp[i] + zp[i] * be;
                                  const T tn = wp[i] + tp[i] * be;
                                  const T pn = rp[i] + pp[i] * be;
                                  zp[i] = zn;
                                  tp[i] = tn;
                                  pp[i] = pn;
                                  xp[i] = fx_fma(a, pn, xp[i]);
                                  rp[i] = fx_fma(-a, tn, rp[i]);
                                  wp[i] = fx_fma(-a, zn, wp[i]);
                              },
                              NoFin{}, nullptr, "pcg_fused_update");
    });
}

int fx_pcg_fused_update_dot2(fx_ctx *ctx, double alpha, double beta, fx_buf *z, fx_buf *t, fx_buf *p, fx_buf *x,
                             fx_buf *r, fx_buf *w, const fx_buf *q, double *rr, double *rw) {
    if (!ctx || !rr || !rw) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    const fx_buf *all[7] = {z, t, p, x, r, w, q};
    for (auto *b : all) {
        FX_TRY(check_buf(b, "pcg vector"));
        FX_TRY(check_same(z, b));
    }
    FX_DISPATCH(z->dtype, {
        T *zp = (T *)z->ptr, *tp = (T *)t->ptr, *pp = (T *)p->ptr, *xp = (T *)x->ptr, *rp = (T *)r->ptr,
          *wp = (T *)w->ptr;
        const T *qp = (const T *)q->ptr;
        const T a = (T)alpha, be = (T)beta;
        FX_TRY(launch_flat<2>(ctx, z->len,
                              [=] __device__(size_t i, CSum *acc) {
                                  const T zn = qp[i] + zp[i] * be;
                                  const T tn = wp[i] + tp[i] * be;
                                  const T pn = rp[i] + pp[i] * be;
                                  zp[i] = zn;
                                  tp[i] = tn;
                                  pp[i] = pn;
                                  xp[i] = fx_fma(a, pn, xp[i]);
                                  const T rn = fx_fma(-a, tn, rp[i]);
                                  const T wn = fx_fma(-a, zn, wp[i]);
                                  rp[i] = rn;
                                  wp[i] = wn;
                                  csum_add_prod(acc[0], (double)rn, (double)rn);
                                  csum_add_prod(acc[1], (double)rn, (double)wn);
                              },
                              StoreFin<2>{ctx->d_result}, nullptr, "pcg_fused_update_dot2"));
    });
    double v[2];
    FX_TRY(read_results(ctx, 2, v));
    *rr = v[0];
    *rw = v[1];
    return FX_OK;
}

}  // extern "C"
