// fx_vcycle.cuh -- fused vertex-centred V(2,2)-cycle kernels.
//
// Two band kernels per level replace the separate sweep / residual / restriction /
// prolongation passes of a V(2,2)-cycle with a zero initial guess:
//
//   k_vdown: from the right-hand side b alone, x1 = w b (first sweep from zero), x2 = x1 +
//            w (b - A x1) (second sweep), res = b - A x2 and its full-weighting restriction
//            onto the coarse grid -- one pass that reads b and writes x2 and the coarse rhs;
//   k_vup:   x = x2 + bilinear(e_coarse), two weighted-Jacobi sweeps, and the result written
//            out (at the finest level directly as the caller's vector, optionally with the
//            inner product <b, z> the preconditioned CG needs next).
//
// Each kernel is a row-lagged pipeline inside one band march that advances two rows per
// step: stage k works on rows 2 behind stage k-1 while the next two input rows arrive,
// every intermediate row lives in a shared-memory ring, and the band carries H halo
// columns on each side so that the stages can be evaluated on the columns their successors
// need (H = 3 down, 2 up).  The 8 column warps run a flag-free path over their CPT columns;
// the 9th warp computes the halo columns.  Every point value is computed with exactly the
// expression of the separate kernels (w = omega / a_c), so the fused cycle is bitwise equal
// to the unfused one.
#pragma once

#include "fx_points.cuh"

namespace fx {

template <typename T>
struct VOp {
    A5<T> a;
    T wd;  // omega / a_c
};

template <typename T>
__device__ __forceinline__ T ring_op5(const A5<T> &a, const T *rn, const T *rc, const T *rs, int j) {
    return fx_fma(a.c, rc[j], fx_fma(a.n, rn[j], fx_fma(a.s, rs[j], fx_fma(a.w, rc[j - 1], a.e * rc[j + 1]))));
}

// Per-thread column slots.  Band threads: CPT columns c0 + t + 256 s (smem j = H + t + 256 s).
// Halo lane h < 2H: one column, smem j = h (left) or BX + h (right), `hoff` columns outside.
template <int CPT, int H>
struct VSlots {
    int col[CPT], j[CPT];
    bool ingrid[CPT], inner[CPT];
    int hoff;
    __device__ __forceinline__ void init(int t, int c0, int cols) {
        constexpr int BX = kBlock * CPT;
        if (t < kBlock) {
#pragma unroll
            for (int s = 0; s < CPT; s++) {
                col[s] = c0 + t + s * kBlock;
                j[s] = H + t + s * kBlock;
                ingrid[s] = col[s] < cols;
                inner[s] = col[s] <= cols - 2;  // col >= 1 always
            }
            hoff = 0;
        } else {
            const int h = t - kBlock;
            const bool used = h < 2 * H;
#pragma unroll
            for (int s = 0; s < CPT; s++) {
                j[s] = (s == 0 && used) ? (h < H ? h : BX + h) : 0;
                col[s] = c0 - H + j[s];
                ingrid[s] = s == 0 && used && col[s] >= 0 && col[s] < cols;
                inner[s] = s == 0 && used && col[s] >= 1 && col[s] <= cols - 2;
            }
            hoff = used ? (h < H ? H - h : h - H + 1) : 1 << 20;
        }
    }
};

// ---------------------------------------------------------------- down

template <typename T, typename TB, int CPT>
__global__ void __launch_bounds__(kBandThreads, 2)
    k_vdown(MarchGeom G, const TB *__restrict__ b, T *__restrict__ x2g, T *__restrict__ coarse, int ccols,
            VOp<T> op, const int *skip) {
    if (skip && *(volatile const int *)skip) return;
    constexpr int H = 3, DP = 2, BX = kBlock * CPT, W = BX + 2 * H;  // DP: row pairs in flight
    __shared__ T sb[4][W], sx1[4][W], sx2[4][W], sres[4][W];
    const int t = threadIdx.x;
    const int band = blockIdx.x % G.nbands, chunk = blockIdx.x / G.nbands;
    const int c0 = 1 + band * BX;
    const int r0 = chunk * G.chunk_rows, r1 = min(r0 + G.chunk_rows, G.rows);  // r0 even
    const int rows = G.rows, cols = G.cols;
    const bool is_band = t < kBlock;
    const bool is_halo = !is_band && (t - kBlock) < 2 * H;
    VSlots<CPT, H> S;
    S.init(t, c0, cols);
    const int r_need = r1 + 3;  // last rhs row any stage reads

    auto ld_b = [&](int r, TB (&v)[CPT]) {
        const bool rin = r >= 0 && r < rows && r <= r_need;
        const size_t ro = (size_t)(rin ? r : 0) * cols;
#pragma unroll
        for (int s = 0; s < CPT; s++) v[s] = (rin && S.ingrid[s]) ? b[ro + S.col[s]] : (TB)0;
    };
    // b row r (as T) and x1 = w b (0 on the ring) into the rings; slot r & 3 (two's complement)
    auto put_b = [&](int r, const TB (&v)[CPT]) {
        const bool irow = r >= 1 && r <= rows - 2;
        T *rb = sb[r & 3];
        T *rx = sx1[r & 3];
        if (is_band) {
#pragma unroll
            for (int s = 0; s < CPT; s++) {
                const T bv = (T)v[s];
                rb[S.j[s]] = bv;
                rx[S.j[s]] = (irow && S.inner[s]) ? fx_fma(op.wd, bv, (T)0) : (T)0;
            }
        } else if (is_halo) {
            const T bv = (T)v[0];
            rb[S.j[0]] = bv;
            rx[S.j[0]] = (irow && S.inner[0]) ? fx_fma(op.wd, bv, (T)0) : (T)0;
        }
    };
    auto x2_row = [&](int i) {  // x2 row i on the band and 2 halo columns each side
        const bool irow = i >= 1 && i <= rows - 2;
        const T *xn = sx1[(i + 3) & 3], *xc = sx1[i & 3], *xs = sx1[(i + 1) & 3];
        const T *bc = sb[i & 3];
        T *out = sx2[i & 3];
        if (is_band) {
            const bool store = irow && i >= r0 && i < r1;
            T *grow = x2g + (size_t)(store ? i : 0) * cols;
#pragma unroll
            for (int s = 0; s < CPT; s++) {
                const int j = S.j[s];
                const T v = (irow && S.inner[s]) ? fx_fma(op.wd, bc[j] - ring_op5(op.a, xn, xc, xs, j), xc[j]) : (T)0;
                out[j] = v;
                if (store && S.inner[s]) grow[S.col[s]] = v;
            }
        } else if (is_halo && S.hoff <= 2) {
            const int j = S.j[0];
            out[j] = (irow && S.inner[0]) ? fx_fma(op.wd, bc[j] - ring_op5(op.a, xn, xc, xs, j), xc[j]) : (T)0;
        }
    };
    auto res_row = [&](int ir) {  // residual row ir on the band and 1 halo column each side
        const bool irow = ir >= 1 && ir <= rows - 2;
        const T *xn = sx2[(ir + 3) & 3], *xc = sx2[ir & 3], *xs = sx2[(ir + 1) & 3];
        const T *bc = sb[ir & 3];
        T *out = sres[ir & 3];
        if (is_band) {
#pragma unroll
            for (int s = 0; s < CPT; s++) {
                const int j = S.j[s];
                out[j] = (irow && S.inner[s]) ? bc[j] - ring_op5(op.a, xn, xc, xs, j) : (T)0;
            }
        } else if (is_halo && S.hoff <= 1) {
            const int j = S.j[0];
            out[j] = (irow && S.inner[0]) ? bc[j] - ring_op5(op.a, xn, xc, xs, j) : (T)0;
        }
    };

    // prologue: rows r0-3, r0-2 straight to the rings; the FIFO holds row pairs starting at
    // (r0-1, r0), the pair the first step (i = r0-2) consumes
    TB fifo[DP][2][CPT];
    {
        TB v[CPT];
        ld_b(r0 - 3, v);
        put_b(r0 - 3, v);
        ld_b(r0 - 2, v);
        put_b(r0 - 2, v);
    }
#pragma unroll
    for (int p = 0; p < DP; p++) {
        ld_b(r0 - 1 + 2 * p, fifo[p][0]);
        ld_b(r0 + 2 * p, fifo[p][1]);
    }

    // step i (even): rhs rows i+1, i+2 arrive; x2 rows i, i+1; residual rows i-1, i; coarse row
    // from fine row i-2
    const int i_first = r0 - 2, i_last = r1 + 1;
    for (int ib = i_first; ib <= i_last; ib += 2 * DP) {
#pragma unroll
        for (int p = 0; p < DP; p++) {
            const int i = ib + 2 * p;
            if (i > i_last) break;  // uniform across the block
            put_b(i + 1, fifo[p][0]);
            put_b(i + 2, fifo[p][1]);
            ld_b(i + 1 + 2 * DP, fifo[p][0]);
            ld_b(i + 2 + 2 * DP, fifo[p][1]);
            __syncthreads();
            x2_row(i);
            x2_row(i + 1);
            __syncthreads();
            res_row(i - 1);
            res_row(i);
            __syncthreads();
            // full weighting onto coarse row I = fr / 2 for the even fine row fr = i-2
            const int fr = i - 2;
            if (is_band && fr >= r0 && fr < r1 && fr >= 2 && fr <= rows - 3) {
                const T *rn = sres[(fr + 3) & 3], *rc = sres[fr & 3], *rs = sres[(fr + 1) & 3];
                T *crow = coarse + (size_t)(fr >> 1) * ccols;
#pragma unroll
                for (int s = 0; s < CPT; s++) {
                    const int c = S.col[s];
                    if ((c & 1) || c < 2 || c > cols - 3) continue;
                    const int j = S.j[s];
                    const T e = (rn[j] + rs[j]) + (rc[j - 1] + rc[j + 1]);
                    const T d = (rn[j - 1] + rn[j + 1]) + (rs[j - 1] + rs[j + 1]);
                    crow[c >> 1] = ((T)4 * rc[j] + ((T)2 * e + d)) * (T)0.0625;
                }
            }
        }
    }
}

// ---------------------------------------------------------------- up

// Bilinear interpolation of the coarse correction at fine point (r, c), the same expression
// per parity case as the separate prolongation kernel, selected without divergence.
template <typename T>
__device__ __forceinline__ T bil_interp(const T *__restrict__ e, int ccols, int r, int c) {
    const bool ro = r & 1, co = c & 1;
    const size_t k = (size_t)(r >> 1) * ccols + (c >> 1);
    const T e00 = e[k];
    const T e01 = co ? e[k + 1] : (T)0;
    const T e10 = ro ? e[k + ccols] : (T)0;
    const T e11 = (ro && co) ? e[k + ccols + 1] : (T)0;
    const T v_oe = (T)0.5 * (e00 + e10);
    const T v_eo = (T)0.5 * (e00 + e01);
    const T v_oo = (T)0.25 * ((e00 + e10) + (e01 + e11));
    return ro ? (co ? v_oo : v_oe) : (co ? v_eo : e00);
}

template <typename T, typename TB, typename TZ, int CPT, bool RZ, typename Fin>
__global__ void __launch_bounds__(kBandThreads, 2)
    k_vup(MarchGeom G, const T *__restrict__ x2g, const T *__restrict__ e, int ccols, const TB *__restrict__ b,
          TZ *__restrict__ z, VOp<T> op, Fin fin, RedArgs<1> ra, const int *skip) {
    if (skip && *(volatile const int *)skip) return;
    constexpr int H = 2, DP = 2, BX = kBlock * CPT, W = BX + 2 * H;
    __shared__ T sf[8][W], sb[8][W], sx3[4][W];
    const int t = threadIdx.x;
    const int band = blockIdx.x % G.nbands, chunk = blockIdx.x / G.nbands;
    const int c0 = 1 + band * BX;
    const int r0 = chunk * G.chunk_rows, r1 = min(r0 + G.chunk_rows, G.rows);
    const int rows = G.rows, cols = G.cols;
    const bool is_band = t < kBlock;
    const bool is_halo = !is_band && (t - kBlock) < 2 * H;
    VSlots<CPT, H> S;
    S.init(t, c0, cols);
    CSum acc[1] = {CSum{0.0, 0.0}};
    const int r_need = r1 + 2;  // last input row any stage reads

    // F0 = x2 + bilinear(e) at interior points, 0 on the ring; b alongside (kept in its own
    // precision in registers for the final inner product)
    auto ld = [&](int r, T (&f)[CPT], TB (&bv)[CPT]) {
        const bool irow = r >= 1 && r <= rows - 2 && r <= r_need;
        const size_t ro = (size_t)(irow ? r : 0) * cols;
#pragma unroll
        for (int s = 0; s < CPT; s++) {
            const bool in = irow && S.inner[s];
            f[s] = in ? x2g[ro + S.col[s]] + bil_interp(e, ccols, r, S.col[s]) : (T)0;
            bv[s] = in ? b[ro + S.col[s]] : (TB)0;
        }
    };
    auto put = [&](int r, const T (&f)[CPT], const TB (&bv)[CPT]) {
        T *rf = sf[r & 7];
        T *rb = sb[r & 7];
        if (is_band) {
#pragma unroll
            for (int s = 0; s < CPT; s++) {
                rf[S.j[s]] = f[s];
                rb[S.j[s]] = (T)bv[s];
            }
        } else if (is_halo) {
            rf[S.j[0]] = f[0];
            rb[S.j[0]] = (T)bv[0];
        }
    };
    auto x3_row = [&](int i) {  // x3 row i on the band and 1 halo column each side
        const bool irow = i >= 1 && i <= rows - 2;
        const T *fn = sf[(i + 7) & 7], *fc = sf[i & 7], *fs = sf[(i + 1) & 7];
        const T *bc = sb[i & 7];
        T *out = sx3[i & 3];
        if (is_band) {
#pragma unroll
            for (int s = 0; s < CPT; s++) {
                const int j = S.j[s];
                out[j] = (irow && S.inner[s]) ? fx_fma(op.wd, bc[j] - ring_op5(op.a, fn, fc, fs, j), fc[j]) : (T)0;
            }
        } else if (is_halo && S.hoff <= 1) {
            const int j = S.j[0];
            out[j] = (irow && S.inner[0]) ? fx_fma(op.wd, bc[j] - ring_op5(op.a, fn, fc, fs, j), fc[j]) : (T)0;
        }
    };
    auto z_row = [&](int iz, const TB (&bv)[CPT]) {  // x4 row iz -> z (band columns)
        if (!(is_band && iz >= r0 && iz < r1 && iz >= 1 && iz <= rows - 2)) return;
        const T *xn = sx3[(iz + 3) & 3], *xc = sx3[iz & 3], *xs = sx3[(iz + 1) & 3];
        TZ *zrow = z + (size_t)iz * cols;
#pragma unroll
        for (int s = 0; s < CPT; s++) {
            if (!S.inner[s]) continue;
            const int j = S.j[s];
            const T v = fx_fma(op.wd, (T)bv[s] - ring_op5(op.a, xn, xc, xs, j), xc[j]);
            zrow[S.col[s]] = (TZ)v;
            if (RZ) csum_add_prod(acc[0], (double)bv[s], (double)(TZ)v);
        }
    };

    // prologue: rows r0-2, r0-1 to the rings; FIFO pairs from (r0, r0+1), the pair the first
    // step (i = r0-1) consumes; `bp` keeps the rhs of the pair being finished
    T ff[DP][2][CPT];
    TB fb[DP][2][CPT];
    TB bp[2][CPT];
    {
        T f[CPT];
        ld(r0 - 2, f, bp[0]);
        put(r0 - 2, f, bp[0]);
        ld(r0 - 1, f, bp[1]);
        put(r0 - 1, f, bp[1]);
    }
#pragma unroll
    for (int p = 0; p < DP; p++) {
        ld(r0 + 2 * p, ff[p][0], fb[p][0]);
        ld(r0 + 1 + 2 * p, ff[p][1], fb[p][1]);
    }

    // step i: F0 rows i+1, i+2 arrive; x3 rows i, i+1; x4 rows i-1, i -> z
    const int i_first = r0 - 1, i_last = r1;
    for (int ib = i_first; ib <= i_last; ib += 2 * DP) {
#pragma unroll
        for (int p = 0; p < DP; p++) {
            const int i = ib + 2 * p;
            if (i > i_last) break;
            put(i + 1, ff[p][0], fb[p][0]);
            put(i + 2, ff[p][1], fb[p][1]);
            TB bnew[2][CPT];
#pragma unroll
            for (int s = 0; s < CPT; s++) {
                bnew[0][s] = fb[p][0][s];
                bnew[1][s] = fb[p][1][s];
            }
            ld(i + 1 + 2 * DP, ff[p][0], fb[p][0]);
            ld(i + 2 + 2 * DP, ff[p][1], fb[p][1]);
            __syncthreads();
            x3_row(i);
            x3_row(i + 1);
            __syncthreads();
            z_row(i - 1, bp[0]);  // rows i-1, i arrived as the previous step's pair
            z_row(i, bp[1]);
#pragma unroll
            for (int s = 0; s < CPT; s++) {
                bp[0][s] = bnew[0][s];
                bp[1][s] = bnew[1][s];
            }
        }
    }
    if constexpr (RZ) grid_reduce<1>(acc, ra, fin);
}

template <typename K>
int band_capacity(fx_ctx *ctx, K kernel, int &cache) {
    if (!cache) {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&cache, kernel, kBandThreads, 0) != cudaSuccess || cache < 1)
            cache = 1;
    }
    return cache * ctx->num_sms;
}

template <typename T, typename TB>
int launch_vdown(fx_ctx *ctx, size_t rows, size_t cols, const TB *b, T *x2, T *coarse, size_t ccols,
                 const VOp<T> &op, const int *skip) {
    constexpr int CPT = band_cpt<T>();
    static int occ = 0;
    const int cap = band_capacity(ctx, k_vdown<T, TB, CPT>, occ);
    const MarchGeom G = march_geom(rows, cols, kBlock * CPT, 4, cap);
    timing_pre(ctx, "mg_down");
    k_vdown<T, TB, CPT><<<G.nblocks, kBandThreads, 0, ctx->stream>>>(G, b, x2, coarse, (int)ccols, op, skip);
    timing_post(ctx, (double)rows * (double)cols);
    return check_launch(ctx, "mg_down");
}

template <typename T, typename TB, typename TZ, bool RZ, typename Fin>
int launch_vup(fx_ctx *ctx, size_t rows, size_t cols, const T *x2, const T *e, size_t ccols, const TB *b, TZ *z,
               const VOp<T> &op, Fin fin, const int *skip) {
    constexpr int CPT = band_cpt<T>();
    static int occ = 0;
    const int cap = band_capacity(ctx, k_vup<T, TB, TZ, CPT, RZ, Fin>, occ);
    const MarchGeom G = march_geom(rows, cols, kBlock * CPT, 4, cap);
    if (RZ && G.nblocks > kMaxRedBlocks) return fail(FX_ERR_INVALID_ARGUMENT, "grid too large");
    timing_pre(ctx, "mg_up");
    k_vup<T, TB, TZ, CPT, RZ, Fin><<<G.nblocks, kBandThreads, 0, ctx->stream>>>(G, x2, e, (int)ccols, b, z, op, fin,
                                                                                red_args<1>(ctx), skip);
    timing_post(ctx, (double)rows * (double)cols);
    return check_launch(ctx, "mg_up");
}

}  // namespace fx
