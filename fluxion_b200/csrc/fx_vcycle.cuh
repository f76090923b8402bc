// fx_vcycle.cuh -- vertex-centred V(2,2)-cycle pieces shared by the fused cycle: the level
// operator (VOp), the bilinear interpolation, and the one-block tail kernel that runs the
// coarse end of the cycle.  The per-level down / up passes are in fx_wcycle.cuh.
//
// Every point value is computed with exactly the expression of the separate sweep /
// residual / restriction / prolongation kernels (w = omega / a_c), so the fused cycle is
// bitwise equal to the unfused one.
#pragma once

#include <atomic>
#include <type_traits>

#include "fx_points.cuh"

FX_CHECK_FILE(vcycle);

namespace fx {

template <typename T>
struct VOp {
    A5<T> a;
    T wd;  // omega / a_c
};

// a.c c + a.n n + a.s s + a.w w + a.e e, in the order of op5 (fx_points.cuh)
template <typename T>
__device__ __forceinline__ T op5v(const A5<T> &a, T c, T n, T s, T w, T e) {
    return fx_fma(a.c, c, fx_fma(a.n, n, fx_fma(a.s, s, fx_fma(a.w, w, a.e * e))));
}

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

// ---------------------------------------------------------------- tail
//
// The coarse end of the cycle in one block: from the first level of at most 9 x 1024 points
// (65 x 65 on 2^k + 1 grids) whose working set fits in shared memory, down to the coarsest
// solve and back up.  Below that size a strip launch costs a few microseconds of latency
// whatever the level's size, while one 1024-thread block evaluates a phase of a 65 x 65 level
// in about a microsecond.  A 129 x 129 level is past the crossover: one block spends about
// 20 us on its two legs, more than its two strip launches take.
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
// its result goes to global memory.  Every point value is the expression of k_wdown / k_wup
// / k_coarse_solve, so the cycle stays bitwise equal to the per-level one.

constexpr int kTailMaxLevels = 12;
constexpr int kTailThreads = 1024;
constexpr size_t kTailSmemMax = 200 * 1024;  // of the 227 KB a block may opt in to

// most points per thread of the first tail level (its rhs is held in registers once)
template <typename T>
__host__ __device__ constexpr int tail_kt() {
    return 9;
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

// Widest coarsest grid, ring included, that coarse_rows2 takes (a column per lane).
constexpr int kRows2MaxCols = 32;

// `sweeps` weighted-Jacobi sweeps from zero on a coarsest grid of at most 32 columns and
// 2 (kTailThreads / 32) + 2 rows.  Warp w owns grid rows 1 + 2w and 2 + 2w, lane l column l,
// both values in registers.  West / east neighbours come by shuffle (columns past the grid
// hold 0, as the ring does), the pair's inner neighbours from registers, and the rows above
// and below from the neighbouring warps through shared memory: each sweep reads those two rows
// from the current full-grid buffer and writes the warp's own two rows into the other one (P
// and Q alternate, ring 0), then one named barrier joins the warps.  Per sweep a thread makes
// two shared-memory loads and two stores, where the one-point-per-thread sweep makes five
// loads.  The update is the expression of jacobi_pts, so the result equals it bit for bit, and
// it lands in P for an even sweep count and in Q for an odd one.  Both buffers must hold zeros.
// Measured on the 17 x 17 coarsest grid: 162 cycles a sweep at F32, against 182 for one warp
// holding the whole grid in registers; at F64 it takes the same 250 cycles as the
// one-point-per-thread sweeps, which stay in use there.
template <typename T>
__device__ __forceinline__ void coarse_rows2(const T *B, T *P, T *Q, int rows, int cols, const VOp<T> &op,
                                             int sweeps) {
    constexpr unsigned kAll = 0xffffffffu;
    const int nw = (rows - 1) / 2;  // warps holding rows: ceil((rows - 2) / 2)
    const int warp = threadIdx.x >> 5, c = threadIdx.x & 31;
    if (warp >= nw) return;
    const int r0 = 1 + 2 * warp, n = rows * cols;
    bool in[2];
    T b[2], x[2];
#pragma unroll
    for (int i = 0; i < 2; i++) {
        const int r = r0 + i;
        in[i] = r <= rows - 2 && c >= 1 && c <= cols - 2 && FX_IN(r * cols + c, n);
        b[i] = in[i] ? B[r * cols + c] : (T)0;
        x[i] = (T)0;
    }
    const int on = (r0 - 1) * cols + c, os = (r0 + 2) * cols + c;  // rows above and below the pair
    const bool hn = c < cols && FX_IN(on, n), hs = r0 + 2 <= rows - 1 && c < cols && FX_IN(os, n);
    const int o0 = r0 * cols + c, o1 = o0 + cols;
    const int nthr = nw * 32;
    for (int k = 0; k < sweeps; k++) {
        const T *cur = (k & 1) ? Q : P;
        T *nxt = (k & 1) ? P : Q;
        const T xn = hn ? cur[on] : (T)0;
        const T xs = hs ? cur[os] : (T)0;
        const T w0 = __shfl_up_sync(kAll, x[0], 1), e0 = __shfl_down_sync(kAll, x[0], 1);
        const T w1 = __shfl_up_sync(kAll, x[1], 1), e1 = __shfl_down_sync(kAll, x[1], 1);
        const T v0 = in[0] ? fx_fma(op.wd, b[0] - op5v(op.a, x[0], xn, x[1], w0, e0), x[0]) : (T)0;
        const T v1 = in[1] ? fx_fma(op.wd, b[1] - op5v(op.a, x[1], x[0], xs, w1, e1), x[1]) : (T)0;
        x[0] = v0;
        x[1] = v1;
        if (in[0]) nxt[o0] = v0;
        if (in[1]) nxt[o1] = v1;
        asm volatile("bar.sync 1, %0;" ::"r"(nthr) : "memory");
    }
}

template <typename T>
__global__ void __launch_bounds__(kTailThreads, 1) k_vtail(TailArgs<T> A, const int *skip) {
    grid_dep_enter();
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
#ifdef FX_CHECKED
    {  // the layout the launcher sized: shared memory, register batches, the coarsest's points per thread
        unsigned dyn;
        asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dyn));
        long long words = 2LL * top_n;
        for (int l = 1; l < nlev; l++) words += (l < nlev - 1 ? 2LL : 1LL) * A.rows[l] * A.cols[l];
        const long long nco = (long long)A.rows[nlev - 1] * A.cols[nlev - 1];
        bool ok = FX_IN(top_n - 1, (long long)KT * kTailThreads) && FX_IN(words - 1, dyn / sizeof(T)) &&
                  FX_IN(nco - 1, 4LL * kTailThreads);
        if (nlev > 1) ok = ok && FX_IN(2LL * n1 - 1, top_n);
        if (!ok) return;  // uniform over the block: every thread tests the same values
    }
#endif

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

    // ---- coarsest: `coarse_sweeps` weighted-Jacobi sweeps from zero.  F32 grids of up to 32
    // columns: a row pair per warp in registers (coarse_rows2); F64 and wider grids: P <-> Q in
    // shared memory, each of the first warps owning up to 4 points (rhs in registers) and a
    // named barrier joining them.  Either way the result lands in P for an even sweep count and
    // in Q for an odd one.
    {
        const int l = nlev - 1, rows = A.rows[l], cols = A.cols[l], n = rows * cols;
        const VOp<T> op = A.op[l];
        const T *B = nlev == 1 ? A.b_top : level_b(l);
        for (int p = tid; p < n; p += kTailThreads) {
            P[p] = (T)0;
            Q[p] = (T)0;
        }
        __syncthreads();
        if (sizeof(T) == 4 && cols <= kRows2MaxCols && rows <= 2 * (kTailThreads / 32) + 2) {
            coarse_rows2<T>(B, P, Q, rows, cols, op, A.coarse_sweeps);
        } else {
            // kPts points per thread: 1 while n fits the block (a predicated-off point still
            // costs its instructions every sweep), else 4 (n <= 4096)
            auto smem_sweeps = [&](auto kp) {
                constexpr int kPts = decltype(kp)::value;
                const int nthr = min(kTailThreads, ((n + 31) / 32) * 32);
                if (tid >= nthr) return;
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
            };
            if (n <= kTailThreads) smem_sweeps(std::integral_constant<int, 1>{});
            else smem_sweeps(std::integral_constant<int, 4>{});
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
    static std::atomic<size_t> attr{0};  // dynamic shared memory opted in for this instantiation so far
    if (smem > 48 * 1024 && smem > attr.load()) {
        FX_CUDA(cudaFuncSetAttribute(k_vtail<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        size_t cur = attr.load();
        while (smem > cur && !attr.compare_exchange_weak(cur, smem)) {
        }
    }
    timing_pre(ctx, "mg_tail");
    launch_pdl(ctx, k_vtail<T>, 1, kTailThreads, smem, A, skip);
    timing_post(ctx, (double)A.rows[0] * (double)A.cols[0]);
    return check_launch(ctx, "mg_tail");
}

// blocks of `kernel` (of `threads` threads) resident on the whole GPU at once
template <typename K>
int band_capacity(fx_ctx *ctx, K kernel, std::atomic<int> &cache, int threads = kBandThreads, size_t smem = 0) {
    int occ = cache.load(std::memory_order_relaxed);
    if (!occ) {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, threads, smem) != cudaSuccess || occ < 1)
            occ = 1;
        cache.store(occ, std::memory_order_relaxed);
    }
    return occ * ctx->num_sms;
}

}  // namespace fx
