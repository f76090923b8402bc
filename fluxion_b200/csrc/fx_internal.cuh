// fx_internal.cuh -- shared internals of the sm_100a backend: context and buffer
// objects, error plumbing, compensated deterministic reductions and the
// row-marching stencil framework every grid kernel is built on.
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/fluxion_cuda.h"

// ------------------------------------------------------------------ errors

namespace fx {

void set_error(const std::string &msg);
int fail(int code, const std::string &msg);

#define FX_CUDA(call)                                                                   \
    do {                                                                                \
        cudaError_t e_ = (call);                                                        \
        if (e_ != cudaSuccess)                                                          \
            return ::fx::fail(FX_ERR_BACKEND, std::string(#call) + ": " +               \
                                                  cudaGetErrorString(e_));              \
    } while (0)

#define FX_TRY(...)                                                                     \
    do {                                                                                \
        int s_ = (__VA_ARGS__);                                                         \
        if (s_ != FX_OK) return s_;                                                     \
    } while (0)

// Maximum number of blocks any reduction kernel may launch, and of sums per kernel.
constexpr int kMaxRedBlocks = 1 << 16;
constexpr int kMaxSums = 4;
constexpr int kBlock = 256;  // threads per block for grid kernels (8 warps)

}  // namespace fx

struct fx_timing_rec {
    cudaEvent_t a, b;
    double points;
};

struct fx_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;
    int num_sms = 148;
    double *d_partials = nullptr;  // [kMaxRedBlocks][2*kMaxSums]
    unsigned *d_counter = nullptr; // last-block ticket
    double *d_result = nullptr;    // results of standalone reductions [kMaxSums]
    double *h_result = nullptr;    // pinned mirror
    unsigned long long launches = 0;
    // per-kernel timing (fx_ctx_timing_begin / _end)
    bool timing = false;
    std::string timing_name;
    std::vector<fx_timing_rec> timing_recs;
    std::vector<cudaEvent_t> event_pool;
    size_t pool_next = 0;
    bool timing_open = false;
};

struct fx_buf {
    fx_ctx *ctx = nullptr;
    void *ptr = nullptr;
    size_t len = 0;
    int dtype = FX_F64;
    bool owned = true;
};

namespace fx {

int check_launch(fx_ctx *ctx, const char *what);
// Timing hooks around a launch (no-ops unless fx_ctx_timing_begin named this kernel).
void timing_pre(fx_ctx *ctx, const char *what);
void timing_post(fx_ctx *ctx, double points);

inline size_t elem_size(int dtype) { return dtype == FX_F32 ? 4 : 8; }

// ------------------------------------------------------------------ compensated sums
// Error-free transformations (Knuth TwoSum; TwoProduct via fma, Ogita-Rump-Oishi 2005).
// Every kernel here is compiled with -fmad=false, so no expression below is contracted.

struct CSum {
    double s, c;
};

__device__ __forceinline__ void two_sum(double a, double b, double &s, double &e) {
    s = a + b;
    double bb = s - a;
    e = (a - (s - bb)) + (b - bb);
}

__device__ __forceinline__ void csum_add(CSum &acc, double x) {
    double s, e;
    two_sum(acc.s, x, s, e);
    acc.s = s;
    acc.c += e;
}

__device__ __forceinline__ void csum_add_prod(CSum &acc, double a, double b) {
    double p = a * b;
    double pe = fma(a, b, -p);
    double s, e;
    two_sum(acc.s, p, s, e);
    acc.s = s;
    acc.c += e + pe;
}

__device__ __forceinline__ CSum csum_merge(CSum a, CSum b) {
    double s, e;
    two_sum(a.s, b.s, s, e);
    return CSum{s, (a.c + b.c) + e};
}

__device__ __forceinline__ double csum_value(CSum a) { return a.s + a.c; }

// ------------------------------------------------------------------ block / grid reduction
// Each block reduces its K compensated sums in a fixed shuffle tree, writes one partial
// per sum, and the last block to finish (ticket counter) folds the partials in block
// order and calls the finaliser with the K results.  Deterministic for a fixed grid.

template <int K>
struct RedArgs {
    double *partials;
    unsigned *counter;
};

template <int K>
__device__ __forceinline__ void warp_reduce(CSum (&acc)[K]) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
#pragma unroll
        for (int k = 0; k < K; k++) {
            CSum o;
            o.s = __shfl_down_sync(0xffffffffu, acc[k].s, off);
            o.c = __shfl_down_sync(0xffffffffu, acc[k].c, off);
            acc[k] = csum_merge(acc[k], o);
        }
    }
}

// Reduce acc over the block; result valid in thread 0.
template <int K>
__device__ __forceinline__ void block_reduce(CSum (&acc)[K]) {
    __shared__ CSum sh[kBlock / 32][K > 0 ? K : 1];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    warp_reduce<K>(acc);
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < K; k++) sh[wid][k] = acc[k];
    }
    __syncthreads();
    if (wid == 0) {
        const int nw = blockDim.x >> 5;
#pragma unroll
        for (int k = 0; k < K; k++) acc[k] = lane < nw ? sh[lane][k] : CSum{0.0, 0.0};
        warp_reduce<K>(acc);
    }
    __syncthreads();
}

// Grid-level completion: call fin(double vals[K]) once, in the last block, thread 0.
template <int K, typename Fin>
__device__ __forceinline__ void grid_reduce(CSum (&acc)[K], RedArgs<K> ra, Fin fin) {
    __shared__ bool is_last;
    block_reduce<K>(acc);
    if (threadIdx.x == 0) {
        double *p = ra.partials + (size_t)blockIdx.x * (2 * K);
#pragma unroll
        for (int k = 0; k < K; k++) {
            p[2 * k] = acc[k].s;
            p[2 * k + 1] = acc[k].c;
        }
        __threadfence();
        unsigned t = atomicAdd(ra.counter, 1u);
        is_last = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    CSum a2[K];
#pragma unroll
    for (int k = 0; k < K; k++) a2[k] = CSum{0.0, 0.0};
    for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
        const volatile double *p = ra.partials + (size_t)b * (2 * K);
#pragma unroll
        for (int k = 0; k < K; k++) a2[k] = csum_merge(a2[k], CSum{p[2 * k], p[2 * k + 1]});
    }
    block_reduce<K>(a2);
    if (threadIdx.x == 0) {
        double v[K > 0 ? K : 1];
#pragma unroll
        for (int k = 0; k < K; k++) v[k] = csum_value(a2[k]);
        fin(v);
        *ra.counter = 0u;
    }
}

template <int K>
inline RedArgs<K> red_args(fx_ctx *ctx) {
    return RedArgs<K>{ctx->d_partials, ctx->d_counter};
}

// ------------------------------------------------------------------ stencil descriptors

// Stencil weights in evaluation form.  mode 5: five-point by offset (ops.rs:898-937);
// mode 9: nine-point by offset (ops.rs:953-1008); mode 0: generic entry list in entry
// order (ops.rs:869-883), radius 1, at most kMaxGeneric entries.
constexpr int kMaxGeneric = 27;
struct StencilP {
    int mode;
    double c, n, s, w, e, nw, ne, sw, se;
    int ne_;
    signed char gi[kMaxGeneric];  // index in the 3x3 window: (dr+1)*3 + (dc+1)
    double gw[kMaxGeneric];
};

int make_stencil(const fx_stencil *s, StencilP *out);

// Boundary values (ops.rs:1139-1180), sides {top, bottom, left, right}.
struct BcP {
    int kind[4];
    double a[4], b[4], g[4];
    double dx, dy;
};

int make_bc(const fx_boundaries *bc, double dx, double dy, BcP *out, bool reject_periodic);

__device__ __forceinline__ double bc_value(const BcP &P, int side, double self_val,
                                           double neighbor_val, double spacing) {
    switch (P.kind[side]) {
        case FX_BC_DIRICHLET:
            return P.a[side];
        case FX_BC_NEUMANN:
            return fma(spacing, P.a[side], neighbor_val);
        case FX_BC_ROBIN: {
            double alpha = P.a[side], beta = P.b[side], g = P.g[side];
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

// 3x3 neighbourhood of one point.
template <typename T>
struct Nb {
    T c, n, s, w, e, nw, ne, sw, se;
};

__device__ __forceinline__ float fx_fma(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double fx_fma(double a, double b, double c) { return fma(a, b, c); }

// Stencil value with the reference's FMA nesting.
template <typename T, int MODE>
__device__ __forceinline__ T stencil_eval(const StencilP &P, const Nb<T> &v) {
    if (MODE == 5) {
        return fx_fma((T)P.c, v.c,
                      fx_fma((T)P.n, v.n,
                             fx_fma((T)P.s, v.s, fx_fma((T)P.w, v.w, (T)P.e * v.e))));
    } else if (MODE == 9) {
        return fx_fma((T)P.c, v.c, fx_fma((T)P.n, v.n, fx_fma((T)P.s, v.s,
               fx_fma((T)P.w, v.w, fx_fma((T)P.e, v.e, fx_fma((T)P.nw, v.nw,
               fx_fma((T)P.ne, v.ne, fx_fma((T)P.sw, v.sw, (T)P.se * v.se))))))));
    } else {
        const T win[9] = {v.nw, v.n, v.ne, v.w, v.c, v.e, v.sw, v.s, v.se};
        T acc = (T)0;
        for (int k = 0; k < P.ne_; k++) acc = fx_fma((T)P.gw[k], win[P.gi[k]], acc);
        return acc;
    }
}

// ------------------------------------------------------------------ row-marching framework
//
// A warp owns a strip of 32 consecutive columns and marches down a chunk of rows,
// keeping the rows above, at and below the current one in registers.  Each row of
// the marched field is loaded exactly once per warp (one coalesced 32-wide load plus
// two halo values for the strip edges, exchanged by shuffles), so the field costs one
// HBM read per element instead of five.  U rows are loaded per step so that U
// independent loads are in flight per thread.
//
// Loader  : T operator()(size_t idx) const       -- value of the marched field at idx
//           (may combine several arrays, e.g. r + beta*p for a fused CG update).
// Point   : void operator()(int r, int c, size_t idx, const Nb<T>& nb, CSum* acc) const
//           -- called for every grid point (r, c) of the chunk, ring included.
// The kernel ends with a grid reduction of K compensated sums and a finaliser.

struct MarchGeom {
    int rows, cols;
    int nstrips;
    int chunk_rows;  // multiple of U
    int nwarps;      // strips * chunks
};

MarchGeom march_geom(fx_ctx *ctx, size_t rows, size_t cols, int U);

template <typename T, int U, int K, typename Loader, typename Point, typename Fin>
__global__ void __launch_bounds__(kBlock) k_march(MarchGeom G, Loader ld, Point pt, Fin fin,
                                                  RedArgs<K> ra, const int *skip) {
    if (skip && *(volatile const int *)skip) return;
    CSum acc[K > 0 ? K : 1];
#pragma unroll
    for (int k = 0; k < (K > 0 ? K : 1); k++) acc[k] = CSum{0.0, 0.0};

    const int lane = threadIdx.x & 31;
    const int gw = blockIdx.x * (kBlock / 32) + (threadIdx.x >> 5);
    if (gw < G.nwarps) {
        const int strip = gw % G.nstrips;
        const int chunk = gw / G.nstrips;
        const int r0 = chunk * G.chunk_rows;
        const int r1 = min(r0 + G.chunk_rows, G.rows);
        const int col0 = strip * 32;
        const int col = col0 + lane;
        const bool cin = col < G.cols;
        const bool has_w = col0 > 0;
        const bool has_e = col0 + 32 < G.cols;
        auto load = [&](int r, T &v, T &hw, T &he) {
            v = (T)0;
            hw = (T)0;
            he = (T)0;
            if (r >= 0 && r < G.rows) {
                const size_t base = (size_t)r * G.cols;
                if (cin) v = ld(base + col);
                if (lane == 0 && has_w) hw = ld(base + col0 - 1);
                if (lane == 31 && has_e) he = ld(base + col0 + 32);
            }
        };
        // window: index 0 = row r-1, 1 = row r, ..., U+1 = row r+U
        T v[U + 2], hw[U + 2], he[U + 2];
        load(r0 - 1, v[0], hw[0], he[0]);
        load(r0, v[1], hw[1], he[1]);
        for (int r = r0; r < r1; r += U) {
#pragma unroll
            for (int u = 0; u < U; u++) load(r + 1 + u, v[u + 2], hw[u + 2], he[u + 2]);
            // west / east neighbours of every window row
            T wv[U + 2], ev[U + 2];
#pragma unroll
            for (int u = 0; u < U + 2; u++) {
                T up = __shfl_up_sync(0xffffffffu, v[u], 1);
                T dn = __shfl_down_sync(0xffffffffu, v[u], 1);
                wv[u] = lane == 0 ? hw[u] : up;
                ev[u] = lane == 31 ? he[u] : dn;
            }
#pragma unroll
            for (int u = 0; u < U; u++) {
                const int rr = r + u;
                if (rr < r1 && cin) {
                    Nb<T> nb;
                    nb.c = v[u + 1];
                    nb.n = v[u];
                    nb.s = v[u + 2];
                    nb.w = wv[u + 1];
                    nb.e = ev[u + 1];
                    nb.nw = wv[u];
                    nb.ne = ev[u];
                    nb.sw = wv[u + 2];
                    nb.se = ev[u + 2];
                    pt(rr, col, (size_t)rr * G.cols + col, nb, acc);
                }
            }
            v[0] = v[U];
            hw[0] = hw[U];
            he[0] = he[U];
            v[1] = v[U + 1];
            hw[1] = hw[U + 1];
            he[1] = he[U + 1];
        }
    }
    if constexpr (K > 0) grid_reduce<K>(acc, ra, fin);
}

struct NoFin {
    __device__ void operator()(const double *) const {}
};

template <typename T, int U, int K, typename Loader, typename Point, typename Fin>
int launch_march(fx_ctx *ctx, const MarchGeom &G, Loader ld, Point pt, Fin fin,
                 const int *skip, const char *what) {
    const int blocks = (G.nwarps + (kBlock / 32) - 1) / (kBlock / 32);
    if (K > 0 && blocks > kMaxRedBlocks) return fail(FX_ERR_INVALID_ARGUMENT, "grid too large");
    timing_pre(ctx, what);
    k_march<T, U, K><<<blocks, kBlock, 0, ctx->stream>>>(G, ld, pt, fin, red_args<K>(ctx), skip);
    timing_post(ctx, (double)G.rows * (double)G.cols);
    return check_launch(ctx, what);
}

// ------------------------------------------------------------------ flat (1-D) kernels

struct FlatGeom {
    size_t n;
    int blocks;
};

FlatGeom flat_geom(fx_ctx *ctx, size_t n);

template <int K, typename F, typename Fin>
__global__ void __launch_bounds__(kBlock) k_flat(size_t n, F f, Fin fin, RedArgs<K> ra,
                                                 const int *skip) {
    if (skip && *(volatile const int *)skip) return;
    CSum acc[K > 0 ? K : 1];
#pragma unroll
    for (int k = 0; k < (K > 0 ? K : 1); k++) acc[k] = CSum{0.0, 0.0};
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) f(i, acc);
    if constexpr (K > 0) grid_reduce<K>(acc, ra, fin);
}

template <int K, typename F, typename Fin>
int launch_flat(fx_ctx *ctx, size_t n, F f, Fin fin, const int *skip, const char *what) {
    FlatGeom g = flat_geom(ctx, n);
    if (g.blocks == 0) return FX_OK;
    timing_pre(ctx, what);
    k_flat<K><<<g.blocks, kBlock, 0, ctx->stream>>>(n, f, fin, red_args<K>(ctx), skip);
    timing_post(ctx, (double)n);
    return check_launch(ctx, what);
}

// Finaliser writing the K reduction values to a device array.
template <int K>
struct StoreFin {
    double *out;
    __device__ void operator()(const double *v) const {
        for (int k = 0; k < K; k++) out[k] = v[k];
    }
};

// Read K doubles of ctx->d_result back to the host (synchronising).
int read_results(fx_ctx *ctx, int k, double *out);

// ------------------------------------------------------------------ misc helpers

int check_buf(const fx_buf *b, const char *name);
int check_same(const fx_buf *a, const fx_buf *b);  // same dtype, same length
int check_grid(const fx_grid *g);
int check_grid_len(const fx_grid *g, const fx_buf *b);

}  // namespace fx
