// fx_wcycle.cuh -- fused vertex-centred V(2,2)-cycle level kernels, one warp per strip.
//
// The same two passes per level as the band kernels of fx_vcycle.cuh (down: x1 = w b, x2 =
// x1 + w (b - A x1), res = b - A x2 and its full-weighting restriction; up: f = x2 + P e,
// x3 = f + w (b - A f), z = x3 + w (b - A x3)), organised for the instruction budget of a
// memory-bound pass:
//
//  - a warp owns a strip of 32 consecutive columns (32 - 2H of them its own, H halo columns
//    on each side recomputed by the neighbouring strip) and marches it down a chunk of rows;
//  - each lane holds its column's last three rows of every stage in registers; the row above
//    and below are register reads, the west / east neighbours one shuffle each;
//  - every global load is a raw value issued D rows ahead into a register FIFO;
//  - no shared memory and no block barrier: the warps of a block are independent.
//
// Every point value is the expression of the band kernels (and so of the separate sweep /
// residual / restriction / prolongation kernels), so the cycle stays bitwise equal.
#pragma once

#include "fx_vcycle.cuh"

namespace fx {

constexpr int kStripWarps = 8;  // warps per block
constexpr int kStripFifo = 6;   // FIFO depth in rows; the march is unrolled by 6 (= lcm(2, 3))

struct StripGeom {
    int rows, cols;
    int nstrips;
    int chunk_rows;  // even
    int nitems;      // strips x chunks, one per warp
};

// capacity: warps of the kernel resident on the whole GPU at once
inline StripGeom strip_geom(size_t rows, size_t cols, int useful, long capacity) {
    StripGeom G;
    G.rows = (int)rows;
    G.cols = (int)cols;
    G.nstrips = (int)((cols - 2 + useful - 1) / useful);
    if (G.nstrips < 1) G.nstrips = 1;
    // one wave of resident warps; chunks of at least 6 rows (an unrolled step)
    const long target = capacity;
    long chunks = target / G.nstrips;
    if (chunks < 1) chunks = 1;
    long cr = ((long)rows + chunks - 1) / chunks;
    if (cr < kStripFifo) cr = kStripFifo;
    cr = (cr + 1) & ~1L;
    G.chunk_rows = (int)cr;
    G.nitems = (int)(G.nstrips * (((long)rows + cr - 1) / cr));
    return G;
}

__device__ __forceinline__ float shfl_w(float v) { return __shfl_up_sync(0xffffffffu, v, 1); }
__device__ __forceinline__ float shfl_e(float v) { return __shfl_down_sync(0xffffffffu, v, 1); }
__device__ __forceinline__ double shfl_w(double v) { return __shfl_up_sync(0xffffffffu, v, 1); }
__device__ __forceinline__ double shfl_e(double v) { return __shfl_down_sync(0xffffffffu, v, 1); }

// a.c c + a.n n + a.s s + a.w w + a.e e in the order of ring_op5
template <typename T>
__device__ __forceinline__ T op5v(const A5<T> &a, T c, T n, T s, T w, T e) {
    return fx_fma(a.c, c, fx_fma(a.n, n, fx_fma(a.s, s, fx_fma(a.w, w, a.e * e))));
}

// ---------------------------------------------------------------- down

template <typename T, typename TB>
__global__ void __launch_bounds__(kStripWarps * 32) k_wdown(StripGeom G, const TB *__restrict__ b, T *__restrict__ x2g,
                                                             T *__restrict__ coarse, int ccols, VOp<T> op,
                                                             const int *skip) {
    if (skip && *(volatile const int *)skip) return;
    constexpr int H = 3, U = 32 - 2 * H, D = kStripFifo;
    const int lane = threadIdx.x & 31;
    const int item = blockIdx.x * kStripWarps + (threadIdx.x >> 5);
    if (item >= G.nitems) return;  // whole warps
    const int strip = item % G.nstrips, chunk = item / G.nstrips;
    const int rows = G.rows, cols = G.cols;
    const int c = 1 + strip * U - H + lane;
    const bool cin = c >= 1 && c <= cols - 2;
    const bool own = lane >= H && lane < H + U && cin;
    const bool cpt = own && !(c & 1) && c >= 2 && c <= cols - 3;  // a coarse point's column
    const int r0 = chunk * G.chunk_rows, r1 = min(r0 + G.chunk_rows, rows);  // r0 even
    // step q: b row q arrives; x1 row q; x2 row q-1; residual row q-2; restriction of fine row
    // q-3 (even q-3 only)
    const int q_first = r0 - 3, q_last = r1 + 2;

    TB fb[D];
    auto load = [&](int q, TB &v) {
        v = (TB)0;
        if (q >= 1 && q <= rows - 2 && q <= q_last && cin) v = b[(size_t)q * cols + c];
    };
#pragma unroll
    for (int k = 0; k < D; k++) load(q_first + k, fb[k]);

    T bw[3] = {}, x1[3] = {}, x2[3] = {}, rs[3] = {}, rw[3] = {}, re[3] = {};
    for (int qb = q_first; qb <= q_last; qb += D) {
#pragma unroll
        for (int k = 0; k < D; k++) {
            const int q = qb + k;
            if (q > q_last) break;  // uniform over the warp
            const int s0 = k % 3, s1 = (k + 2) % 3, s2 = (k + 1) % 3;  // slots of rows q, q-1, q-2
            // row q: rhs and x1 = w b (0 on the ring)
            const T bq = (T)fb[k];
            load(q + D, fb[k]);
            const bool in0 = q >= 1 && q <= rows - 2 && cin;
            bw[s0] = bq;
            x1[s0] = in0 ? fx_fma(op.wd, bq, (T)0) : (T)0;
            // row q-1: x2
            {
                const int r = q - 1;
                const T xc = x1[s1];
                const T xw = shfl_w(xc), xe = shfl_e(xc);
                T v = (T)0;
                if (r >= 1 && r <= rows - 2 && cin)
                    v = fx_fma(op.wd, bw[s1] - op5v(op.a, xc, x1[s2], x1[s0], xw, xe), xc);
                x2[s1] = v;
                if (own && r >= r0 && r < r1 && r >= 1 && r <= rows - 2) x2g[(size_t)r * cols + c] = v;
            }
            // row q-2: residual (and its west / east neighbours for the restriction)
            {
                const int r = q - 2;
                const T xc = x2[s2];
                const T xw = shfl_w(xc), xe = shfl_e(xc);
                T v = (T)0;
                if (r >= 1 && r <= rows - 2 && cin) v = bw[s2] - op5v(op.a, xc, x2[s0], x2[s1], xw, xe);
                rs[s2] = v;
                rw[s2] = shfl_w(v);
                re[s2] = shfl_e(v);
            }
            // fine row q-3 (slot s0 of the residual window, rows q-4 / q-2 in s1 / s2): full
            // weighting onto coarse row (q-3) / 2
            if (!(k & 1)) {  // q - 3 even (r0 even, so q_first odd)
                const int fr = q - 3;
                if (cpt && fr >= r0 && fr < r1 && fr >= 2 && fr <= rows - 3) {
                    const T e = (rs[s1] + rs[s2]) + (rw[s0] + re[s0]);
                    const T d = (rw[s1] + re[s1]) + (rw[s2] + re[s2]);
                    coarse[(size_t)(fr >> 1) * ccols + (c >> 1)] = ((T)4 * rs[s0] + ((T)2 * e + d)) * (T)0.0625;
                }
            }
        }
    }
}

// ---------------------------------------------------------------- up

template <typename T, typename TB, typename TZ, bool RZ, typename Fin>
__global__ void __launch_bounds__(kStripWarps * 32) k_wup(StripGeom G, const T *__restrict__ x2g,
                                                           const T *__restrict__ e, int ccols,
                                                           const TB *__restrict__ b, TZ *__restrict__ z, VOp<T> op,
                                                           Fin fin, RedArgs<1> ra, const int *skip) {
    if (skip && *(volatile const int *)skip) return;
    constexpr int H = 2, U = 32 - 2 * H, D = kStripFifo;
    const int lane = threadIdx.x & 31;
    const int item = blockIdx.x * kStripWarps + (threadIdx.x >> 5);
    const bool live = item < G.nitems;  // idle warps still join the block reduction
    CSum acc[1] = {CSum{0.0, 0.0}};
    if (live) {
        const int strip = item % G.nstrips, chunk = item / G.nstrips;
        const int rows = G.rows, cols = G.cols, crows = (rows - 1) / 2 + 1;
        const int c = 1 + strip * U - H + lane;
        const bool cin = c >= 1 && c <= cols - 2;
        const bool own = lane >= H && lane < H + U && cin;
        const bool co = c & 1;
        const int kc = c >> 1;  // coarse column (c >= 1 wherever it is used)
        const int r0 = chunk * G.chunk_rows, r1 = min(r0 + G.chunk_rows, rows);  // r0 even
        // step q: F0 row q = x2 + P e; x3 row q-1; z row q-2
        const int q_first = r0 - 2, q_last = r1 + 1;  // q_first even

        // FIFO per row: raw x2 and b; for even rows q = 2m also coarse row m+1 at columns kc,
        // kc+1 (with row m, kept from the previous pair, the two rows rows 2m and 2m+1 need)
        T fx[D], fe0[D / 2], fe1[D / 2];
        TB fb[D];
        auto load = [&](int q, T &xv, TB &bv) {
            xv = (T)0;
            bv = (TB)0;
            if (q >= 1 && q <= rows - 2 && q <= q_last && cin) {
                const size_t o = (size_t)q * cols + c;
                xv = x2g[o];
                bv = b[o];
            }
        };
        auto load_coarse = [&](int m, T &v0, T &v1) {
            v0 = (T)0;
            v1 = (T)0;
            if (m >= 0 && m < crows && m <= (q_last >> 1) + 1 && cin) {
                const size_t o = (size_t)m * ccols + kc;
                v0 = e[o];
                if (co) v1 = e[o + 1];
            }
        };
        T ec0, ec1;  // coarse row (q >> 1) for the current pair
        load_coarse(q_first >> 1, ec0, ec1);
#pragma unroll
        for (int k = 0; k < D; k++) {
            load(q_first + k, fx[k], fb[k]);
            if (!(k & 1)) load_coarse(((q_first + k) >> 1) + 1, fe0[k / 2], fe1[k / 2]);
        }

        T f[3] = {}, x3[3] = {};
        TB bw[3] = {};
        for (int qb = q_first; qb <= q_last; qb += D) {
#pragma unroll
            for (int k = 0; k < D; k++) {
                const int q = qb + k;
                if (q > q_last) break;
                const int s0 = k % 3, s1 = (k + 2) % 3, s2 = (k + 1) % 3;  // rows q, q-1, q-2
                // row q: f = x2 + bilinear(e)
                {
                    const bool ro = k & 1;  // q_first even
                    const T n0 = fe0[k / 2], n1 = fe1[k / 2];  // coarse row (q >> 1) + 1
                    const T e00 = ec0;
                    const T e01 = co ? ec1 : (T)0;
                    const T e10 = ro ? n0 : (T)0;
                    const T e11 = (ro && co) ? n1 : (T)0;
                    const T v_oe = (T)0.5 * (e00 + e10);
                    const T v_eo = (T)0.5 * (e00 + e01);
                    const T v_oo = (T)0.25 * ((e00 + e10) + (e01 + e11));
                    const T pe = ro ? (co ? v_oo : v_oe) : (co ? v_eo : e00);
                    const bool in0 = q >= 1 && q <= rows - 2 && cin;
                    f[s0] = in0 ? fx[k] + pe : (T)0;
                    bw[s0] = fb[k];
                    if (ro) {  // the pair is done: its lower coarse row becomes the upper one
                        ec0 = n0;
                        ec1 = n1;
                        load_coarse((q + D + 1) >> 1, fe0[k / 2], fe1[k / 2]);
                    }
                    load(q + D, fx[k], fb[k]);
                }
                // row q-1: x3
                {
                    const int r = q - 1;
                    const T fc = f[s1];
                    const T fw = shfl_w(fc), fe = shfl_e(fc);
                    T v = (T)0;
                    if (r >= 1 && r <= rows - 2 && cin)
                        v = fx_fma(op.wd, (T)bw[s1] - op5v(op.a, fc, f[s2], f[s0], fw, fe), fc);
                    x3[s1] = v;
                }
                // row q-2: z
                {
                    const int r = q - 2;
                    const T xc = x3[s2];
                    const T xw = shfl_w(xc), xe = shfl_e(xc);
                    if (own && r >= r0 && r < r1 && r >= 1 && r <= rows - 2) {
                        const TB bv = bw[s2];
                        const T v = fx_fma(op.wd, (T)bv - op5v(op.a, xc, x3[s0], x3[s1], xw, xe), xc);
                        z[(size_t)r * cols + c] = (TZ)v;
                        if (RZ) csum_add_prod(acc[0], (double)bv, (double)(TZ)v);
                    }
                }
            }
        }
    }
    if constexpr (RZ) grid_reduce<1>(acc, ra, fin);
}

template <typename T, typename TB>
int launch_wdown(fx_ctx *ctx, size_t rows, size_t cols, const TB *b, T *x2, T *coarse, size_t ccols,
                 const VOp<T> &op, const int *skip) {
    static int occ = 0;
    const long cap = (long)band_capacity(ctx, k_wdown<T, TB>, occ, kStripWarps * 32) * kStripWarps;
    const StripGeom G = strip_geom(rows, cols, 32 - 6, cap);
    const int blocks = (G.nitems + kStripWarps - 1) / kStripWarps;
    timing_pre(ctx, "mg_down");
    k_wdown<T, TB><<<blocks, kStripWarps * 32, 0, ctx->stream>>>(G, b, x2, coarse, (int)ccols, op, skip);
    // reads b, writes the smoothed x2 and the restricted coarse rhs
    const double pts = (double)rows * (double)cols, cpts = (double)((rows - 1) / 2 + 1) * (double)ccols;
    timing_post(ctx, pts, pts * (sizeof(TB) + sizeof(T)) + cpts * sizeof(T));
    return check_launch(ctx, "mg_down");
}

template <typename T, typename TB, typename TZ, bool RZ, typename Fin>
int launch_wup(fx_ctx *ctx, size_t rows, size_t cols, const T *x2, const T *e, size_t ccols, const TB *b, TZ *z,
               const VOp<T> &op, Fin fin, const int *skip) {
    static int occ = 0;
    const long cap = (long)band_capacity(ctx, k_wup<T, TB, TZ, RZ, Fin>, occ, kStripWarps * 32) * kStripWarps;
    const StripGeom G = strip_geom(rows, cols, 32 - 4, cap);
    const int blocks = (G.nitems + kStripWarps - 1) / kStripWarps;
    if (RZ && blocks > kMaxRedBlocks) return fail(FX_ERR_INVALID_ARGUMENT, "grid too large");
    timing_pre(ctx, "mg_up");
    k_wup<T, TB, TZ, RZ, Fin><<<blocks, kStripWarps * 32, 0, ctx->stream>>>(G, x2, e, (int)ccols, b, z, op, fin,
                                                                             red_args<1>(ctx), skip);
    // reads x2, the coarse correction e and b, writes z
    const double pts = (double)rows * (double)cols, cpts = (double)((rows - 1) / 2 + 1) * (double)ccols;
    timing_post(ctx, pts, pts * (sizeof(T) + sizeof(TB) + sizeof(TZ)) + cpts * sizeof(T));
    return check_launch(ctx, "mg_up");
}

}  // namespace fx
