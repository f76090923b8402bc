// fx_points.cuh -- per-point functors of the grid kernels (stencil apply / axpy,
// convection-diffusion, Jacobi sweep, residual) and the dtype / stencil-mode dispatch
// macros, shared by the stencil ops, the multigrid cycle and the fused solver kernels.
#pragma once

#include "fx_internal.cuh"

#define FX_DISPATCH(dtype, ...)  \
    do {                         \
        if ((dtype) == FX_F64) { \
            using T = double;    \
            __VA_ARGS__;         \
        } else {                 \
            using T = float;     \
            __VA_ARGS__;         \
        }                        \
    } while (0)

#define FX_MODE_DISPATCH(mode, ...)       \
    do {                                  \
        if ((mode) == 5) {                \
            constexpr int MODE = 5;       \
            __VA_ARGS__;                  \
        } else if ((mode) == 9) {         \
            constexpr int MODE = 9;       \
            __VA_ARGS__;                  \
        } else {                          \
            constexpr int MODE = 0;       \
            __VA_ARGS__;                  \
        }                                 \
    } while (0)

namespace fx {

template <typename T>
struct LoadArr {
    static constexpr int NL = 1;
    const T *p;
    __device__ __forceinline__ void load(size_t i, T (&v)[1]) const { v[0] = p[i]; }
    __device__ __forceinline__ T combine(const T (&v)[1]) const { return v[0]; }
};

template <typename T>
constexpr int unroll_for() {
    return sizeof(T) == 8 ? 4 : 8;
}

// apply_stencil (ops.rs:76-127 + apply_boundaries :796-843) and apply_stencil_var (:129-154)
template <typename T, int MODE, bool VAR>
struct PtApply {
    static constexpr int NA = VAR ? 1 : 0;
    T *out;
    const T *coeff;
    StencilP P;
    BcP B;
    int rows, cols;
    __device__ __forceinline__ const T *aux(int) const { return coeff; }
    __device__ __forceinline__ void operator()(bool ring, int r, int c, size_t idx, const Nb<T> &nb, const T *a,
                                               CSum *) const {
        if (ring) return;  // boundary values come from k_ring_values
        T v = stencil_eval<T, MODE>(P, nb);
        if (VAR) v = v * a[0];
        out[idx] = v;
    }
};

// stencil_axpy (ops.rs:225-269, fused_5pt_axpy_row :1011-1125): ring untouched
template <typename T, int MODE>
struct PtAxpy {
    static constexpr int NA = 1;
    T *y;
    StencilP P;
    T alpha;
    int rows, cols;
    __device__ __forceinline__ const T *aux(int) const { return y; }
    __device__ __forceinline__ void operator()(bool ring, int, int, size_t idx, const Nb<T> &nb, const T *a,
                                               CSum *) const {
        if (ring) return;
        y[idx] = fx_fma(alpha, stencil_eval<T, MODE>(P, nb), a[0]);
    }
};

// convection-diffusion (ops.rs:673-791)
template <typename T>
struct ConvDiffC {
    T inv_dx, inv_dy, inv_dx2, inv_dy2, k2;  // k2 = 2*(inv_dx2 + inv_dy2)
};

template <typename T>
__device__ __forceinline__ T conv_diff_at(const ConvDiffC<T> &K, const Nb<T> &nb, T kap, T vx, T vy) {
    const T c = nb.c;
    const T lap = fx_fma(nb.w + nb.e, K.inv_dx2, (nb.n + nb.s) * K.inv_dy2) - K.k2 * c;
    const T diff = kap * lap;
    const T dudx = vx >= (T)0 ? (c - nb.w) * K.inv_dx : (nb.e - c) * K.inv_dx;
    const T dudy = vy >= (T)0 ? (c - nb.n) * K.inv_dy : (nb.s - c) * K.inv_dy;
    const T conv = fx_fma(vx, dudx, vy * dudy);
    return diff + conv;
}

template <typename T, bool AXPY>
struct PtConvDiff {
    static constexpr int NA = AXPY ? 4 : 3;
    T *out;
    const T *kappa, *vx, *vy;
    ConvDiffC<T> K;
    T alpha;
    int rows, cols;
    __device__ __forceinline__ const T *aux(int k) const {
        return k == 0 ? kappa : (k == 1 ? vx : (k == 2 ? vy : (const T *)out));
    }
    __device__ __forceinline__ void operator()(bool ring, int, int, size_t idx, const Nb<T> &nb, const T *a,
                                               CSum *) const {
        if (ring) {
            if (!AXPY) out[idx] = (T)0;
            return;
        }
        const T v = conv_diff_at<T>(K, nb, a[0], a[1], a[2]);
        out[idx] = AXPY ? fx_fma(alpha, v, a[AXPY ? 3 : 0]) : v;
    }
};

template <typename T>
ConvDiffC<T> conv_consts(double dx, double dy) {
    const double inv_dx = 1.0 / dx, inv_dy = 1.0 / dy;
    const double inv_dx2 = inv_dx * inv_dx, inv_dy2 = inv_dy * inv_dy;
    ConvDiffC<T> K;
    K.inv_dx = (T)inv_dx;
    K.inv_dy = (T)inv_dy;
    K.inv_dx2 = (T)inv_dx2;
    K.inv_dy2 = (T)inv_dy2;
    K.k2 = (T)(2.0 * (inv_dx2 + inv_dy2));
    return K;
}

// true weighted Jacobi sweep: x_out = x_in + wd * (b - A x_in), wd = omega / a_c
template <typename T>
struct A5 {
    T c, n, s, w, e;
};

template <typename T>
__device__ __forceinline__ T op5(const A5<T> &a, const Nb<T> &v) {
    return fx_fma(a.c, v.c, fx_fma(a.n, v.n, fx_fma(a.s, v.s, fx_fma(a.w, v.w, a.e * v.e))));
}

template <typename T>
struct PtJacobi {
    static constexpr int NA = 1;
    T *out;
    const T *b;
    A5<T> a;
    T wd;
    int rows, cols;
    __device__ __forceinline__ const T *aux(int) const { return b; }
    __device__ __forceinline__ void operator()(bool ring, int, int, size_t idx, const Nb<T> &nb, const T *av,
                                               CSum *) const {
        if (ring) return;
        out[idx] = fx_fma(wd, av[0] - op5<T>(a, nb), nb.c);
    }
};

template <typename T>
struct PtResidual {
    static constexpr int NA = 1;
    T *out;
    const T *b;
    A5<T> a;
    int rows, cols;
    __device__ __forceinline__ const T *aux(int) const { return b; }
    __device__ __forceinline__ void operator()(bool ring, int, int, size_t idx, const Nb<T> &nb, const T *av,
                                               CSum *) const {
        if (ring) return;
        out[idx] = av[0] - op5<T>(a, nb);
    }
};

template <typename T>
A5<T> make_a5(const double *a5) {
    return A5<T>{(T)a5[0], (T)a5[1], (T)a5[2], (T)a5[3], (T)a5[4]};
}

}  // namespace fx
