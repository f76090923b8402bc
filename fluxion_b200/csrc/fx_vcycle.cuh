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

    // zero-initialised predicated loads: nothing consumes the value until put_b
    auto ld_b = [&](int r, TB (&v)[CPT]) {
        const bool rin = r >= 0 && r < rows && r <= r_need;
#pragma unroll
        for (int s = 0; s < CPT; s++) {
            v[s] = (TB)0;
            if (rin && S.ingrid[s]) v[s] = b[(size_t)r * cols + S.col[s]];
        }
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

// The same interpolation from two coarse rows held in shared memory: e0 = coarse row r >> 1,
// e1 = the row below it, k = coarse column c >> 1 relative to the rows' first column.
template <typename T>
__device__ __forceinline__ T bil_rows(const T *e0, const T *e1, bool ro, bool co, int k) {
    const T e00 = e0[k];
    const T e01 = co ? e0[k + 1] : (T)0;
    const T e10 = ro ? e1[k] : (T)0;
    const T e11 = (ro && co) ? e1[k + 1] : (T)0;
    const T v_oe = (T)0.5 * (e00 + e10);
    const T v_eo = (T)0.5 * (e00 + e01);
    const T v_oo = (T)0.25 * ((e00 + e10) + (e01 + e11));
    return ro ? (co ? v_oo : v_oe) : (co ? v_eo : e00);
}

// Every global load of k_vup is a raw value issued two row pairs ahead (x2 and b of the fine
// rows, one coarse row of e per pair); nothing waits on them until the rows enter the rings.
// Coarse rows of e live in a 4-row shared ring: step i (rows i+1 = 2m, i+2 = 2m+1 arrive)
// interpolates from coarse rows m, m+1 and stores row m+2 for the next step.
template <typename T, typename TB, typename TZ, int CPT, bool RZ, typename Fin>
__global__ void __launch_bounds__(kBandThreads, 2)
    k_vup(MarchGeom G, const T *__restrict__ x2g, const T *__restrict__ e, int ccols, const TB *__restrict__ b,
          TZ *__restrict__ z, VOp<T> op, Fin fin, RedArgs<1> ra, const int *skip) {
    if (skip && *(volatile const int *)skip) return;
    constexpr int H = 2, DP = 2, BX = kBlock * CPT, W = BX + 2 * H;
    constexpr int WC = BX / 2 + 4;  // coarse columns a band's rows interpolate from (+1 spare)
    __shared__ T sf[8][W], sb[8][W], sx3[4][W], ec[4][WC];
    const int t = threadIdx.x;
    const int band = blockIdx.x % G.nbands, chunk = blockIdx.x / G.nbands;
    const int c0 = 1 + band * BX;
    const int r0 = chunk * G.chunk_rows, r1 = min(r0 + G.chunk_rows, G.rows);  // r0 even
    const int rows = G.rows, cols = G.cols, crows = (rows - 1) / 2 + 1;
    const bool is_band = t < kBlock;
    const bool is_halo = !is_band && (t - kBlock) < 2 * H;
    VSlots<CPT, H> S;
    S.init(t, c0, cols);
    CSum acc[1] = {CSum{0.0, 0.0}};
    const int r_need = r1 + 2;  // last input row any stage reads
    // coarse column of ring index 0: (c0 - H) >> 1 (c0 - H is odd); thread t loads index t
    const int cbase = (c0 - H - 1) / 2;
    const int ccol = cbase + t;
    const bool cload = t < WC - 1 && ccol >= 0 && ccol < ccols;

    auto ld = [&](int r, T (&xv)[CPT], TB (&bv)[CPT]) {
        const bool irow = r >= 1 && r <= rows - 2 && r <= r_need;
#pragma unroll
        for (int s = 0; s < CPT; s++) {
            xv[s] = (T)0;
            bv[s] = (TB)0;
            if (irow && S.inner[s]) {
                const size_t o = (size_t)r * cols + S.col[s];
                xv[s] = x2g[o];
                bv[s] = b[o];
            }
        }
    };
    auto ld_coarse = [&](int m) -> T {
        T v = (T)0;
        if (cload && m >= 0 && m < crows) v = e[(size_t)m * ccols + ccol];
        return v;
    };
    auto put_coarse = [&](int m, T v) {
        if (t < WC - 1) ec[m & 3][t] = v;
    };
    // F0 = x2 + bilinear(e) at interior points, 0 on the ring; b alongside (kept in its own
    // precision in registers for the final inner product)
    auto put = [&](int r, const T (&xv)[CPT], const TB (&bv)[CPT]) {
        const bool irow = r >= 1 && r <= rows - 2;
        const bool ro = r & 1;
        const T *e0 = ec[(r >> 1) & 3], *e1 = ec[((r >> 1) + 1) & 3];
        T *rf = sf[r & 7];
        T *rb = sb[r & 7];
        if (is_band) {
#pragma unroll
            for (int s = 0; s < CPT; s++) {
                const int c = S.col[s];
                const T f = xv[s] + bil_rows(e0, e1, ro, c & 1, (c >> 1) - cbase);
                rf[S.j[s]] = (irow && S.inner[s]) ? f : (T)0;
                rb[S.j[s]] = (T)bv[s];
            }
        } else if (is_halo) {
            const int c = S.col[0];
            const T f = xv[0] + bil_rows(e0, e1, ro, c & 1, (c >> 1) - cbase);
            rf[S.j[0]] = (irow && S.inner[0]) ? f : (T)0;
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

    // prologue: coarse rows m0-1 .. m0+1 (m0 = r0 / 2) to the ring; fine rows r0-2, r0-1 to the
    // rings; FIFO pairs from (r0, r0+1), the pair the first step (i = r0-1) consumes, with
    // coarse rows from m0+2; `bp` keeps the rhs of the pair being finished
    const int m0 = r0 >> 1;
    T fx[DP][2][CPT];
    TB fb[DP][2][CPT];
    T fe[DP];
    TB bp[2][CPT];
    {
        const T c_a = ld_coarse(m0 - 1), c_b = ld_coarse(m0), c_c = ld_coarse(m0 + 1);
        T xv[2][CPT];
        ld(r0 - 2, xv[0], bp[0]);
        ld(r0 - 1, xv[1], bp[1]);
#pragma unroll
        for (int p = 0; p < DP; p++) {
            ld(r0 + 2 * p, fx[p][0], fb[p][0]);
            ld(r0 + 1 + 2 * p, fx[p][1], fb[p][1]);
            fe[p] = ld_coarse(m0 + 2 + p);
        }
        put_coarse(m0 - 1, c_a);
        put_coarse(m0, c_b);
        put_coarse(m0 + 1, c_c);
        __syncthreads();
        put(r0 - 2, xv[0], bp[0]);
        put(r0 - 1, xv[1], bp[1]);
    }

    // step i: coarse row m+2 stored; F0 rows i+1, i+2 arrive; x3 rows i, i+1; x4 rows i-1, i -> z
    const int i_first = r0 - 1, i_last = r1;
    for (int ib = i_first; ib <= i_last; ib += 2 * DP) {
#pragma unroll
        for (int p = 0; p < DP; p++) {
            const int i = ib + 2 * p;
            if (i > i_last) break;
            const int m = (i + 1) >> 1;
            put_coarse(m + 2, fe[p]);
            put(i + 1, fx[p][0], fb[p][0]);
            put(i + 2, fx[p][1], fb[p][1]);
            TB bnew[2][CPT];
#pragma unroll
            for (int s = 0; s < CPT; s++) {
                bnew[0][s] = fb[p][0][s];
                bnew[1][s] = fb[p][1][s];
            }
            ld(i + 1 + 2 * DP, fx[p][0], fb[p][0]);
            ld(i + 2 + 2 * DP, fx[p][1], fb[p][1]);
            fe[p] = ld_coarse(m + 2 + DP);
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

// ---------------------------------------------------------------- tail
//
// The coarse end of the cycle in one block: from the first level whose working set fits in
// shared memory down to the coarsest solve and back up.  On these grids a band launch is
// latency-bound (a few dozen rows marched in sequence, 15-20 us per launch whatever the
// size), while one 1024-thread block evaluates a whole level phase in a microsecond or two.
//
// Shared memory, for a first tail level of n0 points:
//   X [n0]  its pre-smoothed x2, kept for the up leg (and turned into x2 + P e in place);
//   Y [n0]  its rhs, overwritten in place by its residual; after the restriction Y is free
//           and holds the coarser levels' two work buffers P, Q (x1 / residual / iterate /
//           correction; the coarsest solve ping-pongs between them), and on the way up the
//           first level's x3;
//   then per coarser level its rhs and x2 (the coarsest only its rhs).
// The first level's x1 = w b is never stored: x2 evaluates it at the neighbours from the rhs.
// Its rhs comes from global memory (and again, into registers, for the last two phases);
// its result goes to global memory.  Every point value is the expression of k_vdown / k_vup
// / k_coarse_solve, so the cycle stays bitwise equal to the per-level one.

constexpr int kTailMaxLevels = 12;
constexpr int kTailThreads = 1024;
constexpr size_t kTailSmemMax = 200 * 1024;  // of the 227 KB a block may opt in to

// most points per thread of the first tail level (its rhs is held in registers once)
template <typename T>
__host__ __device__ constexpr int tail_kt() {
    return sizeof(T) == 4 ? 17 : 9;
}

template <typename T>
struct TailArgs {
    int nlev;  // levels in the tail; the last is the coarsest
    int rows[kTailMaxLevels], cols[kTailMaxLevels];
    VOp<T> op[kTailMaxLevels];
    const T *b_top;  // rhs of the first tail level
    T *u_top;        // its result (interior written; the ring is left as it is)
    int coarse_sweeps;
};

// shared-memory bytes of a tail whose first level has n[0] points (n[1..] the coarser ones)
inline size_t tail_smem_bytes(const size_t *n, int nlev, size_t esize) {
    size_t words = 2 * n[0];
    for (int l = 1; l < nlev; l++) words += (l < nlev - 1 ? 2 : 1) * n[l];
    return words * esize;
}

template <typename T>
__device__ __forceinline__ T op5_at(const A5<T> &a, const T *x, int p, int cols) {
    return fx_fma(a.c, x[p], fx_fma(a.n, x[p - cols], fx_fma(a.s, x[p + cols], fx_fma(a.w, x[p - 1], a.e * x[p + 1]))));
}

// One weighted-Jacobi sweep over NP points of a thread (p < 0: no point).  src and dst are
// distinct buffers; saying so lets the compiler issue every point's loads before any store.
template <typename T, int NP>
__device__ __forceinline__ void jacobi_pts(const T *__restrict__ src, T *__restrict__ dst, const int (&cp)[NP],
                                           const T (&cb)[NP], const VOp<T> &op, int cols) {
    T v[NP];
#pragma unroll
    for (int q = 0; q < NP; q++) {
        const int p = cp[q];
        if (p >= 0) v[q] = fx_fma(op.wd, cb[q] - op5_at(op.a, src, p, cols), src[p]);
    }
#pragma unroll
    for (int q = 0; q < NP; q++)
        if (cp[q] >= 0) dst[cp[q]] = v[q];
}

template <typename T>
__global__ void __launch_bounds__(kTailThreads, 1) k_vtail(TailArgs<T> A, const int *skip) {
    if (skip && *(volatile const int *)skip) return;
    constexpr int KT = tail_kt<T>();
    extern __shared__ __align__(16) unsigned char tail_smem[];
    const int tid = threadIdx.x;
    const int nlev = A.nlev, top_rows = A.rows[0], top_cols = A.cols[0], top_n = top_rows * top_cols;
    T *X = reinterpret_cast<T *>(tail_smem);
    T *Y = X + top_n;
    const int n1 = nlev > 1 ? A.rows[1] * A.cols[1] : 0;
    T *P = Y;       // coarser-level work buffers, inside Y
    T *Q = Y + n1;  // (n1 >= every coarser level; 2 n1 <= n0)

    // rhs / x2 of a coarser level l >= 1, packed after Y
    auto level_b = [&](int l) -> T * {
        T *q = Y + top_n;
        for (int k = 1; k < l; k++) q += 2 * A.rows[k] * A.cols[k];
        return q;
    };
    auto level_x2 = [&](int l) -> T * { return level_b(l) + A.rows[l] * A.cols[l]; };

    // visit points first, first + stride, ... of a rows x cols level with their (r, c) stepped
    // incrementally (one division per call)
    auto each = [&](int rows, int cols, int first, int stride, auto &&f) {
        const int n = rows * cols;
        const int dr = stride / cols, dc = stride - dr * cols;
        int r = first / cols, c = first - r * cols;
        for (int p = first; p < n; p += stride) {
            f(p, r, c, r >= 1 && r <= rows - 2 && c >= 1 && c <= cols - 2);
            c += dc;
            r += dr;
            if (c >= cols) {
                c -= cols;
                r++;
            }
        }
    };
    // full-weighting restriction of R (level l) onto the interior of level l+1's rhs
    auto restrict_to = [&](const T *R, int l) {
        const int cols = A.cols[l];
        T *Bc = level_b(l + 1);
        each(A.rows[l + 1], A.cols[l + 1], tid, kTailThreads, [&](int pc, int I, int J, bool in) {
            if (!in) return;  // the coarse ring of the rhs is never read
            const int p = (2 * I) * cols + 2 * J;
            const T e = (R[p - cols] + R[p + cols]) + (R[p - 1] + R[p + 1]);
            const T d = (R[p - cols - 1] + R[p - cols + 1]) + (R[p + cols - 1] + R[p + cols + 1]);
            Bc[pc] = ((T)4 * R[p] + ((T)2 * e + d)) * (T)0.0625;
        });
    };

    if (nlev == 1) {  // the tail is the coarsest solve alone: its rhs straight from global memory
        P = X;
        Q = Y;
    } else {
        // ---- down, first tail level: rhs -> Y; x2 -> X (x1 = w b evaluated where needed);
        // residual -> Y in place; restriction
        const VOp<T> op = A.op[0];
        const int cols = top_cols;
        {
            T v[KT];  // all loads in flight at once
#pragma unroll
            for (int k = 0; k < KT; k++) {
                const int p = tid + k * kTailThreads;
                v[k] = p < top_n ? A.b_top[p] : (T)0;
            }
#pragma unroll
            for (int k = 0; k < KT; k++) {
                const int p = tid + k * kTailThreads;
                if (p < top_n) Y[p] = v[k];
            }
        }
        __syncthreads();
        each(top_rows, cols, tid, kTailThreads, [&](int p, int r, int c, bool in) {
            T v = (T)0;
            if (in) {
                // x1 at the five points: w b inside, 0 on the ring
                const T xc = fx_fma(op.wd, Y[p], (T)0);
                const T xn = r > 1 ? fx_fma(op.wd, Y[p - cols], (T)0) : (T)0;
                const T xs = r < top_rows - 2 ? fx_fma(op.wd, Y[p + cols], (T)0) : (T)0;
                const T xw = c > 1 ? fx_fma(op.wd, Y[p - 1], (T)0) : (T)0;
                const T xe = c < cols - 2 ? fx_fma(op.wd, Y[p + 1], (T)0) : (T)0;
                const T ax = fx_fma(op.a.c, xc, fx_fma(op.a.n, xn, fx_fma(op.a.s, xs, fx_fma(op.a.w, xw, op.a.e * xe))));
                v = fx_fma(op.wd, Y[p] - ax, xc);
            }
            X[p] = v;
        });
        __syncthreads();
        each(top_rows, cols, tid, kTailThreads, [&](int p, int, int, bool in) {
            if (in) Y[p] = Y[p] - op5_at(op.a, X, p, cols);  // each thread reads only its own Y[p]
            else Y[p] = (T)0;
        });
        __syncthreads();
        restrict_to(Y, 0);
        __syncthreads();
    }
    // ---- down, levels 1 .. nlev-2: x1 -> P, x2 -> its slot, residual -> Q
    for (int l = 1; l < nlev - 1; l++) {
        const int rows = A.rows[l], cols = A.cols[l];
        const VOp<T> op = A.op[l];
        const T *B = level_b(l);
        T *X2 = level_x2(l);
        each(rows, cols, tid, kTailThreads, [&](int p, int, int, bool in) {
            P[p] = in ? fx_fma(op.wd, B[p], (T)0) : (T)0;
        });
        __syncthreads();
        each(rows, cols, tid, kTailThreads, [&](int p, int, int, bool in) {
            T v = (T)0;
            if (in) v = fx_fma(op.wd, B[p] - op5_at(op.a, P, p, cols), P[p]);
            X2[p] = v;
        });
        __syncthreads();
        each(rows, cols, tid, kTailThreads, [&](int p, int, int, bool in) {
            T v = (T)0;
            if (in) v = B[p] - op5_at(op.a, X2, p, cols);
            Q[p] = v;
        });
        __syncthreads();
        restrict_to(Q, l);
        __syncthreads();
    }

    // ---- coarsest: `coarse_sweeps` weighted-Jacobi sweeps from zero, P <-> Q.  Each of the
    // first warps owns up to 4 points (rhs in registers); a named barrier joins them.
    {
        const int l = nlev - 1, rows = A.rows[l], cols = A.cols[l], n = rows * cols;
        const VOp<T> op = A.op[l];
        const T *B = nlev == 1 ? A.b_top : level_b(l);
        for (int p = tid; p < n; p += kTailThreads) {
            P[p] = (T)0;
            Q[p] = (T)0;
        }
        __syncthreads();
        {
            constexpr int kPts = 4;  // n <= 4096
            const int nthr = min(kTailThreads, ((n + 31) / 32) * 32);
            if (tid < nthr) {
                int cp[kPts];
                T cb[kPts];
#pragma unroll
                for (int q = 0; q < kPts; q++) {
                    const int p = tid + q * nthr;
                    const int r = p / cols, c = p - (p / cols) * cols;
                    const bool in = p < n && r >= 1 && r <= rows - 2 && c >= 1 && c <= cols - 2;
                    cp[q] = in ? p : -1;
                    cb[q] = in ? B[p] : (T)0;
                }
                for (int k = 0; k < A.coarse_sweeps; k++) {
                    if (k & 1) jacobi_pts<T, kPts>(Q, P, cp, cb, op, cols);
                    else jacobi_pts<T, kPts>(P, Q, cp, cb, op, cols);
                    asm volatile("bar.sync 1, %0;" ::"r"(nthr) : "memory");
                }
            }
        }
        __syncthreads();
        if (nlev == 1) {
            const T *fin = (A.coarse_sweeps & 1) ? Q : P;
            for (int p = tid; p < n; p += kTailThreads) A.u_top[p] = fin[p];
            return;
        }
    }

    // ---- up, levels nlev-2 .. 1: E holds the coarser level's result, F is free
    T *E = (A.coarse_sweeps & 1) ? Q : P;
    T *F = (A.coarse_sweeps & 1) ? P : Q;
    for (int l = nlev - 2; l >= 1; l--) {
        const int rows = A.rows[l], cols = A.cols[l], ccols = A.cols[l + 1];
        const VOp<T> op = A.op[l];
        const T *B = level_b(l);
        const T *X2 = level_x2(l);
        each(rows, cols, tid, kTailThreads, [&](int p, int r, int c, bool in) {
            F[p] = in ? X2[p] + bil_interp(E, ccols, r, c) : (T)0;  // x2 + P e
        });
        __syncthreads();
        each(rows, cols, tid, kTailThreads, [&](int p, int, int, bool in) {
            T v = (T)0;
            if (in) v = fx_fma(op.wd, B[p] - op5_at(op.a, F, p, cols), F[p]);  // x3
            E[p] = v;
        });
        __syncthreads();
        each(rows, cols, tid, kTailThreads, [&](int p, int, int, bool in) {
            T v = (T)0;
            if (in) v = fx_fma(op.wd, B[p] - op5_at(op.a, E, p, cols), E[p]);
            F[p] = v;
        });
        __syncthreads();
        T *t = E;
        E = F;
        F = t;
    }
    // ---- up, first tail level: f = x2 + P e in place in X; x3 -> Y; result to global
    {
        const VOp<T> op = A.op[0];
        const int cols = top_cols, ccols = A.cols[1];
        T bt[KT];  // this thread's rhs values, loaded in one batch
#pragma unroll
        for (int k = 0; k < KT; k++) {
            const int p = tid + k * kTailThreads;
            bt[k] = p < top_n ? A.b_top[p] : (T)0;
        }
        each(top_rows, cols, tid, kTailThreads, [&](int p, int r, int c, bool in) {
            X[p] = in ? X[p] + bil_interp(E, ccols, r, c) : (T)0;
        });
        __syncthreads();
        // thread tid owns points tid + k * 1024, k < KT (top_n <= KT * 1024)
        const int dr = kTailThreads / cols, dc = kTailThreads - dr * cols;
        {
            int r = tid / cols, c = tid - r * cols;
#pragma unroll
            for (int k = 0; k < KT; k++) {
                const int p = tid + k * kTailThreads;
                if (p < top_n) {
                    T v = (T)0;
                    if (r >= 1 && r <= top_rows - 2 && c >= 1 && c <= cols - 2)
                        v = fx_fma(op.wd, bt[k] - op5_at(op.a, X, p, cols), X[p]);  // x3
                    Y[p] = v;
                }
                c += dc;
                r += dr;
                if (c >= cols) {
                    c -= cols;
                    r++;
                }
            }
        }
        __syncthreads();
        {
            int r = tid / cols, c = tid - r * cols;
#pragma unroll
            for (int k = 0; k < KT; k++) {
                const int p = tid + k * kTailThreads;
                if (p < top_n && r >= 1 && r <= top_rows - 2 && c >= 1 && c <= cols - 2)
                    A.u_top[p] = fx_fma(op.wd, bt[k] - op5_at(op.a, Y, p, cols), Y[p]);
                c += dc;
                r += dr;
                if (c >= cols) {
                    c -= cols;
                    r++;
                }
            }
        }
    }
}

template <typename T>
int launch_vtail(fx_ctx *ctx, const TailArgs<T> &A, size_t smem, const int *skip) {
    static size_t attr = 0;  // dynamic shared memory opted in for this instantiation so far
    if (smem > 48 * 1024 && smem > attr) {
        FX_CUDA(cudaFuncSetAttribute(k_vtail<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        attr = smem;
    }
    timing_pre(ctx, "mg_tail");
    k_vtail<T><<<1, kTailThreads, smem, ctx->stream>>>(A, skip);
    timing_post(ctx, (double)A.rows[0] * (double)A.cols[0]);
    return check_launch(ctx, "mg_tail");
}

// blocks of `kernel` (of `threads` threads) resident on the whole GPU at once
template <typename K>
int band_capacity(fx_ctx *ctx, K kernel, int &cache, int threads = kBandThreads) {
    if (!cache) {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&cache, kernel, threads, 0) != cudaSuccess || cache < 1)
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
    // reads b, writes the smoothed x2 and the restricted coarse rhs
    const double pts = (double)rows * (double)cols, cpts = (double)((rows - 1) / 2 + 1) * (double)ccols;
    timing_post(ctx, pts, pts * (sizeof(TB) + sizeof(T)) + cpts * sizeof(T));
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
    // reads x2, the coarse correction e and b, writes z
    const double pts = (double)rows * (double)cols, cpts = (double)((rows - 1) / 2 + 1) * (double)ccols;
    timing_post(ctx, pts, pts * (sizeof(T) + sizeof(TB) + sizeof(TZ)) + cpts * sizeof(T));
    return check_launch(ctx, "mg_up");
}

}  // namespace fx
