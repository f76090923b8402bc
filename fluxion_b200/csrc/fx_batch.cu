// fx_batch.cu -- many independent convection-diffusion problems solved together (new; the
// reference solves one grid at a time, crates/runtime/src/bicgstab.rs:218-346 with the V-cycle of
// crates/runtime/src/multigrid.rs:188-230).
//
// Every problem is -nu Lap u + v.grad u = f (first-order upwind, the operator of fx_op_conv_diff
// with sigma / coeff / scalar kappa shared by the batch) on its own square (2^k + 1)^2 grid,
// solved by right-preconditioned BiCGSTAB with the conv-diff V-cycle of fx_cdmg (vertex
// hierarchy, rediscretised levels, injected velocities, weighted Jacobi with the reciprocal
// diagonal, full weighting / bilinear, a one-block coarsest solve), cycle in FP64 or FP32.
//
// The batch runs in lockstep: each phase of the algorithm (a BiCGSTAB vector pass, a sweep pair on
// level l, a residual, a transfer, the coarsest solves) is one launch over every problem that takes
// part in it.  A launch's blocks read their work from a table of (problem, chunk) or (problem,
// 32 x 32 tile) items built once per batch, so problems of every size share each launch and the
// GPU is filled by the batch, not by one problem.  A problem whose solve is over skips its items
// (the per-problem halt / done words of the BiCGSTAB state).  Problems of different depth
// share the down leg level by level (a problem's coarsest solve runs at its own last level) and
// the up leg likewise, so every problem sees exactly the launch sequence of its single-problem
// cycle.  Every point value is the single-problem kernel's expression, so the batched cycle equals
// fx_cdmg's bit for bit; the BiCGSTAB inner products are per-problem compensated sums in a fixed
// order (deterministic, within roundoff of the single-problem solver's).  One iteration of the
// whole batch is a fixed launch sequence and is replayed from a CUDA graph.
#include <algorithm>
#include <cmath>
#include <vector>

#include "fx_points.cuh"

using namespace fx;

FX_CHECK_FILE(batch);

namespace {

constexpr int kBT = 256;             // threads per block
constexpr int kChunkDefault = 8 * kBT;  // elements per flat work item (fx_batch_set_chunk changes it)
constexpr int kTileB = 32;           // sweep-pair tile side (as k_cd_sweep2)
constexpr int kTileX = kTileB + 4;   // x with a two-point halo
constexpr int kTileY = kTileB + 2;   // first sweep with a one-point halo

struct Chunk {
    int prob, start, len, first, count;  // first / count: the problem's items in this table
};
struct Tile {
    int prob, ty, tx;
};

// per (level, problem): offset into the level's arrays, side n (rows = cols = n), constants
template <typename T>
struct Lvl {
    long long off;
    int n;
    ConvDiffC<T> K;
};

// operator constants shared by the batch
template <typename T>
struct BOpC {
    T sigma, coeff, kap;
};

// the conv-diff operator at a point (OpA<T, kModeCD>::apply: interior fma(coeff, CD v, sigma v))
template <typename T>
__device__ __forceinline__ T bop_apply(const BOpC<T> &O, const ConvDiffC<T> &K, const Nb<T> &nb, T vx, T vy) {
    return fx_fma(O.coeff, conv_diff_at<T>(K, nb, O.kap, vx, vy), O.sigma * nb.c);
}

// diag(A) at a point (the conv-diff multigrid's cd_diag)
template <typename T>
__device__ __forceinline__ T bop_diag(const BOpC<T> &O, const ConvDiffC<T> &K, T vx, T vy) {
    return fx_fma(O.coeff, fx_fma(-O.kap, K.k2, fx_fma(fabs(vx), K.inv_dx, fabs(vy) * K.inv_dy)), O.sigma);
}

template <typename T>
__device__ __forceinline__ Nb<T> nb_at(const T *x, size_t i, int n) {
    Nb<T> nb;
    nb.c = x[i];
    nb.n = x[i - n];
    nb.s = x[i + n];
    nb.w = x[i - 1];
    nb.e = x[i + 1];
    return nb;
}

__device__ __forceinline__ bool ring_at(int i, int n) {
    const int r = i / n, c = i - r * n;
    return r == 0 || c == 0 || r == n - 1 || c == n - 1;
}

// BiCGSTAB state per problem (the single-problem DevState's BiCGSTAB fields)
struct BState {
    double tol, r0, resid, r_norm, s_norm, rho, rho_new, alpha, beta, omega;
    long long iter, max_iter;
    int done, halt, pending, reason;
};

__device__ __forceinline__ void bs_finish(BState *S, int reason, long long iters, double resid) {
    S->done = 1;
    S->halt = 1;
    S->reason = reason;
    S->iter = iters;
    S->resid = resid;
}

// points of problem p's level in a flat pass (the checked build's extent of its items): the level
// of the functor's K0 (k) or LvlArgs (a) entries; functors with neither are not checked
template <typename F>
__device__ __forceinline__ auto bf_points_impl(const F &f, int p, int) -> decltype((long long)f.k.L[p].n) {
    return (long long)f.k.L[p].n * f.k.L[p].n;
}
template <typename F>
__device__ __forceinline__ auto bf_points_impl(const F &f, int p, long) -> decltype((long long)f.a.L[p].n) {
    return (long long)f.a.L[p].n * f.a.L[p].n;
}
template <typename F>
__device__ __forceinline__ long long bf_points_impl(const F &, int, ...) {
    return 1LL << 62;
}

// ---------------------------------------------------------------- generic batched flat pass
// One block per item of a chunk table; K compensated sums per problem, folded in item order by the
// problem's last block (a per-problem ticket), which calls fin(problem, values).
template <int K, typename F, typename Fin>
__global__ void __launch_bounds__(kBT) k_bflat(const Chunk *__restrict__ items, F f, Fin fin, double *partials,
                                               unsigned *tickets) {
    const Chunk c = items[blockIdx.x];
    if (f.skip(c.prob)) return;  // the same answer for every item of the problem
    CSum acc[K > 0 ? K : 1];
#pragma unroll
    for (int k = 0; k < (K > 0 ? K : 1); k++) acc[k] = CSum{0.0, 0.0};
    // an item past its problem's level is not run (it still joins the problem's ticket)
    const int hi = FX_IN((long long)c.start + c.len - 1, bf_points_impl(f, c.prob, 0)) ? c.start + c.len : c.start;
    f.run(c.prob, c.start + (int)threadIdx.x, hi, kBT, acc);
    if constexpr (K > 0) {
        __shared__ bool is_last;
        block_reduce<K>(acc);
        if (threadIdx.x == 0) {
            double *p = partials + (size_t)blockIdx.x * (2 * K);
#pragma unroll
            for (int k = 0; k < K; k++) {
                p[2 * k] = acc[k].s;
                p[2 * k + 1] = acc[k].c;
            }
            __threadfence();
            const unsigned t = atomicAdd(tickets + c.prob, 1u);
            is_last = t == (unsigned)c.count - 1;
        }
        __syncthreads();
        if (!is_last) return;
        __threadfence();
        CSum a2[K];
#pragma unroll
        for (int k = 0; k < K; k++) a2[k] = CSum{0.0, 0.0};
        for (int b = threadIdx.x; b < c.count; b += kBT) {
            const volatile double *p = partials + (size_t)(c.first + b) * (2 * K);
#pragma unroll
            for (int k = 0; k < K; k++) a2[k] = csum_merge(a2[k], CSum{p[2 * k], p[2 * k + 1]});
        }
        block_reduce<K>(a2);
        if (threadIdx.x == 0) {
            double v[K];
#pragma unroll
            for (int k = 0; k < K; k++) v[k] = csum_value(a2[k]);
            fin(c.prob, v);
            tickets[c.prob] = 0u;
        }
    }
}

struct NoFinB {
    __device__ void operator()(int, const double *) const {}
};

// ---------------------------------------------------------------- BiCGSTAB passes (level 0, FP64)
// The bicgstab.rs recurrences as the single-problem solver evaluates them (fx_solvers.cu).

struct K0 {  // what every level-0 pass needs
    const Lvl<double> *L;  // level-0 entries, one per problem
    const double *vx, *vy;
    BOpC<double> O;
    BState *S;
};

struct BfNorm {  // ||b||^2 (the relative tolerance's scale)
    K0 k;
    const double *b;
    __device__ bool skip(int) const { return false; }
    __device__ void run(int p, int lo, int hi, int st, CSum *acc) const {
        const double *bb = b + k.L[p].off;
        for (int i = lo; i < hi; i += st) csum_add_prod(acc[0], bb[i], bb[i]);
    }
};
struct FinTol {
    BState *S;
    double rel, max_iter;
    __device__ void operator()(int p, const double *v) const {
        BState *s = S + p;
        s->tol = rel * sqrt(v[0]);
        s->max_iter = (long long)max_iter;
        s->done = s->halt = s->pending = 0;
        s->reason = 0;
        s->iter = 0;
    }
};

struct BfInit {  // r = b - A x; r_hat = r; (r.r, r_hat.r)
    K0 k;
    const double *x, *b;
    double *r, *rh;
    __device__ bool skip(int) const { return false; }
    __device__ void run(int p, int lo, int hi, int st, CSum *acc) const {
        const Lvl<double> &Lp = k.L[p];
        const long long o = Lp.off;
        for (int i = lo; i < hi; i += st) {
            const size_t g = (size_t)(o + i);
            const Nb<double> nb = ring_at(i, Lp.n) ? Nb<double>{x[g], 0, 0, 0, 0} : nb_at(x, g, Lp.n);
            const double ax = ring_at(i, Lp.n) ? nb.c : bop_apply(k.O, Lp.K, nb, k.vx[g], k.vy[g]);
            const double rv = fx_fma(-1.0, ax, b[g]);
            r[g] = rv;
            rh[g] = rv;
            csum_add_prod(acc[0], rv, rv);
            csum_add_prod(acc[1], rv, rv);
        }
    }
};

__device__ __forceinline__ void bs_top(BState *S, double rr, double rho_new) {
    const double r_norm = sqrt(rr);
    S->r_norm = r_norm;
    S->resid = r_norm;
    if (S->iter >= S->max_iter) {
        bs_finish(S, FX_MAX_ITERATIONS, S->max_iter, r_norm);
        return;
    }
    if (r_norm < S->tol) {
        bs_finish(S, FX_CONVERGED, S->iter, r_norm);
        return;
    }
    if (!isfinite(r_norm)) {  // NaN / Inf in the problem: Breakdown rather than max_iter
        bs_finish(S, FX_BREAKDOWN, S->iter, r_norm);
        return;
    }
    S->rho_new = rho_new;
    if (fabs(rho_new) < 1e-30) {
        bs_finish(S, FX_BREAKDOWN, S->iter, r_norm);
        return;
    }
    S->beta = (rho_new / S->rho) * (S->alpha / S->omega);
}

struct FinNorm2 {  // resid = ||r|| (the batch's residual check)
    BState *S;
    __device__ void operator()(int p, const double *v) const { S[p].resid = sqrt(v[0]); }
};

struct FinInit {
    BState *S;
    __device__ void operator()(int p, const double *v) const {
        BState *s = S + p;
        s->rho = 1.0;
        s->alpha = 1.0;
        s->omega = 1.0;
        s->iter = 0;
        s->r0 = sqrt(v[0]);
        bs_top(s, v[0], v[1]);
    }
};

struct BfP {  // p = r + beta (p - omega v)
    K0 k;
    double *pv;
    const double *r, *v;
    __device__ bool skip(int p) const { return k.S[p].halt; }
    __device__ void run(int p, int lo, int hi, int st, CSum *) const {
        const double beta = k.S[p].beta, omega = k.S[p].omega;
        const long long o = k.L[p].off;
        for (int i = lo; i < hi; i += st) {
            const size_t g = (size_t)(o + i);
            pv[g] = r[g] + fx_fma(-omega, v[g], pv[g]) * beta;
        }
    }
};

struct BfAr {  // out = A in; (rr . out) when WITH_DOT, else (out.s, out.out) for t = A s_hat
    K0 k;
    const double *in;
    double *out;
    const double *dot_with;  // r_hat (v pass) or s (t pass)
    int tpass;
    __device__ bool skip(int p) const { return k.S[p].halt; }
    __device__ void run(int p, int lo, int hi, int st, CSum *acc) const {
        const Lvl<double> &Lp = k.L[p];
        const long long o = Lp.off;
        for (int i = lo; i < hi; i += st) {
            const size_t g = (size_t)(o + i);
            const bool ring = ring_at(i, Lp.n);
            const Nb<double> nb = ring ? Nb<double>{in[g], 0, 0, 0, 0} : nb_at(in, g, Lp.n);
            const double av = ring ? nb.c : bop_apply(k.O, Lp.K, nb, k.vx[g], k.vy[g]);
            out[g] = av;
            if (tpass) {
                csum_add_prod(acc[0], av, dot_with[g]);
                csum_add_prod(acc[1], av, av);
            } else {
                csum_add_prod(acc[0], dot_with[g], av);
            }
        }
    }
};

struct FinRv {
    BState *S;
    __device__ void operator()(int p, const double *v) const {
        BState *s = S + p;
        if (fabs(v[0]) < 1e-30) {
            bs_finish(s, FX_BREAKDOWN, s->iter, s->r_norm);
            return;
        }
        s->alpha = s->rho_new / v[0];
    }
};

struct BfS {  // s = r - alpha v; s.s
    K0 k;
    const double *r, *v;
    double *s;
    __device__ bool skip(int p) const { return k.S[p].halt; }
    __device__ void run(int p, int lo, int hi, int st, CSum *acc) const {
        const double alpha = k.S[p].alpha;
        const long long o = k.L[p].off;
        for (int i = lo; i < hi; i += st) {
            const size_t g = (size_t)(o + i);
            const double sv = fx_fma(-alpha, v[g], r[g]);
            s[g] = sv;
            csum_add_prod(acc[0], sv, sv);
        }
    }
};

struct FinS {
    BState *S;
    __device__ void operator()(int p, const double *v) const {
        BState *s = S + p;
        s->s_norm = sqrt(v[0]);
        if (s->s_norm < s->tol) {
            s->pending = 1;
            s->halt = 1;
        }
    }
};

struct FinT {
    BState *S;
    __device__ void operator()(int p, const double *v) const {
        BState *s = S + p;
        if (fabs(v[1]) < 1e-30) {
            s->pending = 2;
            s->halt = 1;
            return;
        }
        s->omega = v[0] / v[1];
    }
};

struct BfFinish {  // x += alpha pp + omega ss; r = s - omega t; (r.r, r_hat.r)
    K0 k;
    double *x, *r;
    const double *pp, *ss, *t, *s, *rh;
    __device__ bool skip(int p) const { return k.S[p].done; }
    __device__ void run(int p, int lo, int hi, int st, CSum *acc) const {
        const BState &S = k.S[p];
        const double alpha = S.alpha, omega = S.omega;
        const int pending = S.pending;
        const long long o = k.L[p].off;
        for (int i = lo; i < hi; i += st) {
            const size_t g = (size_t)(o + i);
            if (pending) {
                x[g] = fx_fma(alpha, pp[g], x[g]);
                continue;
            }
            x[g] = fx_fma(omega, ss[g], fx_fma(alpha, pp[g], x[g]));
            const double rv = fx_fma(-omega, t[g], s[g]);
            r[g] = rv;
            csum_add_prod(acc[0], rv, rv);
            csum_add_prod(acc[1], rh[g], rv);
        }
    }
};

struct FinEnd {
    BState *S;
    __device__ void operator()(int p, const double *v) const {
        BState *s = S + p;
        if (s->pending) {
            bs_finish(s, s->pending == 1 ? FX_CONVERGED : FX_BREAKDOWN, s->iter, s->s_norm);
            return;
        }
        s->rho = s->rho_new;
        s->iter += 1;
        bs_top(s, v[0], v[1]);
    }
};

// ---------------------------------------------------------------- V-cycle passes (level arrays)

// The cycle's operands on one level: arrays of the level (offsets from the level table), the
// velocity fields of the level, and the skip words (the problem's halt).
template <typename T>
struct LvlArgs {
    const Lvl<T> *L;  // entries of this level, indexed by problem
    const T *vx, *vy;
    BOpC<T> O;
    const BState *S;  // skip when S[p].halt
};

template <typename T>
struct BfZero {
    LvlArgs<T> a;
    T *x;
    __device__ bool skip(int p) const { return a.S[p].halt; }
    __device__ void run(int p, int lo, int hi, int st, CSum *) const {
        T *xx = x + a.L[p].off;
        for (int i = lo; i < hi; i += st) xx[i] = (T)0;
    }
};

template <typename S_, typename D_>
struct BfCast {  // d = (D) s; with zero_other also other = 0 (the F32 cycle's entry)
    const Lvl<S_> *Ls;
    const Lvl<D_> *Ld;
    const S_ *s;
    D_ *d;
    D_ *zero_other;
    const BState *S;  // null: never skip
    __device__ bool skip(int p) const { return S && S[p].halt; }
    __device__ void run(int p, int lo, int hi, int st, CSum *) const {
        const S_ *ss = s + Ls[p].off;
        D_ *dd = d + Ld[p].off;
        D_ *zz = zero_other ? zero_other + Ld[p].off : nullptr;
        for (int i = lo; i < hi; i += st) {
            dd[i] = (D_)ss[i];
            if (zz) zz[i] = (D_)0;
        }
    }
};

template <typename T>
struct BfSweep {  // out = x + omega (b - A x) (1 / diag), interior (FlatCdSweep)
    LvlArgs<T> a;
    const T *x, *b;
    T *out;
    T omega;
    __device__ bool skip(int p) const { return a.S[p].halt; }
    __device__ void run(int p, int lo, int hi, int st, CSum *) const {
        const Lvl<T> &Lp = a.L[p];
        const long long o = Lp.off;
        for (int i = lo; i < hi; i += st) {
            if (ring_at(i, Lp.n)) continue;
            const size_t g = (size_t)(o + i);
            const Nb<T> nb = nb_at(x, g, Lp.n);
            const T inv_d = (T)1 / bop_diag(a.O, Lp.K, a.vx[g], a.vy[g]);
            out[g] = fx_fma(omega, (b[g] - bop_apply(a.O, Lp.K, nb, a.vx[g], a.vy[g])) * inv_d, nb.c);
        }
    }
};

template <typename T>
struct BfResid {  // out = b - A x, interior (FlatCdResid)
    LvlArgs<T> a;
    const T *x, *b;
    T *out;
    __device__ bool skip(int p) const { return a.S[p].halt; }
    __device__ void run(int p, int lo, int hi, int st, CSum *) const {
        const Lvl<T> &Lp = a.L[p];
        const long long o = Lp.off;
        for (int i = lo; i < hi; i += st) {
            if (ring_at(i, Lp.n)) continue;
            const size_t g = (size_t)(o + i);
            out[g] = b[g] - bop_apply(a.O, Lp.K, nb_at(x, g, Lp.n), a.vx[g], a.vy[g]);
        }
    }
};

template <typename T>
struct BfRestrict {  // coarse rhs = full weighting of the fine residual (ring 0), coarse u = 0
    const Lvl<T> *Lf, *Lc;
    const T *f;
    T *c, *u;
    const BState *S;
    __device__ bool skip(int p) const { return S[p].halt; }
    __device__ void run(int p, int lo, int hi, int st, CSum *) const {
        const int nc = Lc[p].n, nf = Lf[p].n;
        const T *ff = f + Lf[p].off;
        T *cc = c + Lc[p].off, *uu = u + Lc[p].off;
        for (int i = lo; i < hi; i += st) {
            uu[i] = (T)0;
            const int I = i / nc, J = i - I * nc;
            if (I == 0 || J == 0 || I == nc - 1 || J == nc - 1) {
                cc[i] = (T)0;
                continue;
            }
            const size_t k = (size_t)(2 * I) * nf + 2 * J;
            const T e = (ff[k - nf] + ff[k + nf]) + (ff[k - 1] + ff[k + 1]);
            const T d = (ff[k - nf - 1] + ff[k - nf + 1]) + (ff[k + nf - 1] + ff[k + nf + 1]);
            cc[i] = ((T)4 * ff[k] + ((T)2 * e + d)) * (T)0.0625;
        }
    }
};

template <typename T>
struct BfProlong {  // fine interior += bilinear interpolation of the coarse correction
    const Lvl<T> *Lf, *Lc;
    const T *c;
    T *f;
    const BState *S;
    __device__ bool skip(int p) const { return S[p].halt; }
    __device__ void run(int p, int lo, int hi, int st, CSum *) const {
        const int nf = Lf[p].n, nc = Lc[p].n;
        const T *cc = c + Lc[p].off;
        T *fv = f + Lf[p].off;
        for (int q = lo; q < hi; q += st) {
            const int i = q / nf, j = q - i * nf;
            if (i == 0 || j == 0 || i == nf - 1 || j == nf - 1) continue;
            const size_t k = (size_t)(i / 2) * nc + (j / 2);
            T e;
            if (!(i & 1) && !(j & 1)) e = cc[k];
            else if ((i & 1) && !(j & 1)) e = (T)0.5 * (cc[k] + cc[k + nc]);
            else if (!(i & 1) && (j & 1)) e = (T)0.5 * (cc[k] + cc[k + 1]);
            else e = (T)0.25 * ((cc[k] + cc[k + nc]) + (cc[k + 1] + cc[k + nc + 1]));
            fv[q] += e;
        }
    }
};

template <typename T>
struct BfCopy {
    const Lvl<T> *L;
    const T *src;
    T *dst;
    const BState *S;
    __device__ bool skip(int p) const { return S[p].halt; }
    __device__ void run(int p, int lo, int hi, int st, CSum *) const {
        const long long o = L[p].off;
        for (int i = lo; i < hi; i += st) dst[o + i] = src[o + i];
    }
};

// Two sweeps in one pass over a 32 x 32 tile of one problem's level (k_cd_sweep2's expressions:
// the pair equals two BfSweep passes bit for bit, the result in `out`).
template <typename T>
__global__ void __launch_bounds__(256) k_bsweep2(const Tile *__restrict__ tiles, LvlArgs<T> a, const T *xb, T *outb,
                                                 const T *bb, T omega) {
    const Tile tl = tiles[blockIdx.x];
    if (a.S[tl.prob].halt) return;
    __shared__ T xs[kTileX * kTileX];
    __shared__ T ys[kTileY * kTileY];
    __shared__ T ds[kTileY * kTileY];
    const Lvl<T> &Lp = a.L[tl.prob];
    const int rows = Lp.n, cols = Lp.n;
    const T *x = xb + Lp.off, *b = bb + Lp.off, *vx = a.vx + Lp.off, *vy = a.vy + Lp.off;
    T *out = outb + Lp.off;
    const int tid = threadIdx.x;
    const int r0 = tl.ty * kTileB, c0 = tl.tx * kTileB;
    if (!(FX_IN(r0, rows) && FX_IN(c0, cols))) return;  // a tile of the table outside its problem's level
#pragma unroll
    for (int j = 0; j < (kTileX * kTileX + 255) / 256; j++) {
        const int k = tid + j * 256;
        if (k >= kTileX * kTileX) break;
        const int gr = r0 - 2 + k / kTileX, gc = c0 - 2 + k % kTileX;
        xs[k] = (gr >= 0 && gr < rows && gc >= 0 && gc < cols) ? x[(size_t)gr * cols + gc] : (T)0;
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < (kTileY * kTileY + 255) / 256; j++) {
        const int k = tid + j * 256;
        if (k >= kTileY * kTileY) break;
        const int lr = k / kTileY, lc = k % kTileY;
        const int gr = r0 - 1 + lr, gc = c0 - 1 + lc;
        T y = (T)0, inv_d = (T)0;
        if (gr >= 0 && gr < rows && gc >= 0 && gc < cols) {
            const size_t g = (size_t)gr * cols + gc;
            if (gr == 0 || gc == 0 || gr == rows - 1 || gc == cols - 1) {
                y = out[g];
            } else {
                inv_d = (T)1 / bop_diag(a.O, Lp.K, vx[g], vy[g]);
                const int q = (lr + 1) * kTileX + (lc + 1);
                Nb<T> nb;
                nb.c = xs[q];
                nb.n = xs[q - kTileX];
                nb.s = xs[q + kTileX];
                nb.w = xs[q - 1];
                nb.e = xs[q + 1];
                y = fx_fma(omega, (b[g] - bop_apply(a.O, Lp.K, nb, vx[g], vy[g])) * inv_d, nb.c);
            }
        }
        ys[k] = y;
        ds[k] = inv_d;
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kTileB * kTileB / 256; j++) {
        const int k = tid + j * 256;
        const int lr = k / kTileB, lc = k % kTileB;
        const int gr = r0 + lr, gc = c0 + lc;
        if (gr <= 0 || gc <= 0 || gr >= rows - 1 || gc >= cols - 1) continue;
        const size_t g = (size_t)gr * cols + gc;
        const int q = (lr + 1) * kTileY + (lc + 1);
        Nb<T> nb;
        nb.c = ys[q];
        nb.n = ys[q - kTileY];
        nb.s = ys[q + kTileY];
        nb.w = ys[q - 1];
        nb.e = ys[q + 1];
        out[g] = fx_fma(omega, (b[g] - bop_apply(a.O, Lp.K, nb, vx[g], vy[g])) * ds[q], nb.c);
    }
}

// The coarsest solve of one problem per block (k_cd_coarse's expressions): nsweeps sweeps from
// zero in shared memory, the result written to u.
template <typename T>
__global__ void __launch_bounds__(1024) k_bcoarse(const int *__restrict__ probs, LvlArgs<T> a, T *ub, const T *bb,
                                                  T omega, int nsweeps) {
    const int prob = probs[blockIdx.x];
    if (a.S[prob].halt) return;
    constexpr int kPts = 4;
    extern __shared__ unsigned char bsm[];
    const Lvl<T> &Lp = a.L[prob];
    const int rows = Lp.n, cols = Lp.n, n = rows * cols;
#ifdef FX_CHECKED
    {
        unsigned dyn;
        asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dyn));
        if (!(FX_IN(n - 1, kPts * (int)blockDim.x) && FX_IN(2LL * n - 1, dyn / sizeof(T)))) return;
    }
#endif
    T *s0 = reinterpret_cast<T *>(bsm);
    T *s1 = s0 + n;
    T *u = ub + Lp.off;
    const T *b = bb + Lp.off, *vx = a.vx + Lp.off, *vy = a.vy + Lp.off;
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
        dv[k] = inner[k] ? (T)1 / bop_diag(a.O, Lp.K, vx[i], vy[i]) : (T)1;
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
            dst[i] = fx_fma(omega, (bv[q] - bop_apply(a.O, Lp.K, nb, vx[i], vy[i])) * dv[q], nb.c);
        }
        __syncthreads();
    }
    const T *fin = (nsweeps & 1) ? s1 : s0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) u[i] = fin[i];
}

template <typename S_, typename D_>
struct BfInject {  // coarse field = fine field at the coincident points
    const Lvl<S_> *Lf;
    const Lvl<D_> *Lc;
    const S_ *f;
    D_ *c;
    __device__ bool skip(int) const { return false; }
    __device__ void run(int p, int lo, int hi, int st, CSum *) const {
        const int nf = Lf[p].n, nc = Lc[p].n;
        const S_ *ff = f + Lf[p].off;
        D_ *cc = c + Lc[p].off;
        for (int i = lo; i < hi; i += st) {
            const int I = i / nc, J = i - I * nc;
            cc[i] = (D_)ff[(size_t)(2 * I) * nf + 2 * J];
        }
    }
};

__global__ void k_bcount(const BState *__restrict__ S, int n, int *out) {
    __shared__ int c;
    if (threadIdx.x == 0) c = 0;
    __syncthreads();
    int mine = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) mine += S[i].done ? 0 : 1;
    atomicAdd(&c, mine);
    __syncthreads();
    if (threadIdx.x == 0) *out = c;
}

}  // namespace

// ================================================================ the batch object

struct fx_batch {
    fx_ctx *ctx = nullptr;
    int dtype = FX_F64;  // of the cycle
    size_t np = 0;       // problems
    std::vector<int> n0;  // grid side per problem
    std::vector<int> depth;
    double nu = 0, sigma = 0, coeff = 1, omega = 0.8;
    size_t n_pre = 2, n_post = 2, coarse_sweeps = 200;
    int nlev = 0;  // the deepest problem's level count
    int chunk = kChunkDefault;  // elements per flat work item
    std::vector<std::vector<int>> lv_side, lv_have, lv_smooth;  // per level: sides, problem lists
    std::vector<long long> off0;  // level-0 offsets (+ total at the end)
    long long total0 = 0;
    const fx_buf *vx = nullptr, *vy = nullptr;  // level-0 F64 fields (borrowed)
    // device tables
    std::vector<std::pair<void *, bool>> dev_allocs;  // (pointer, from the pool)
    Chunk *d_chunk0 = nullptr;  // level 0, every problem
    int nchunk0 = 0;
    struct LevelDev {
        void *lvl = nullptr;  // Lvl<T>[np] (entries of problems without the level unused)
        Chunk *chunks = nullptr;  // all problems having the level
        int nchunks = 0;
        Chunk *smooth_chunks = nullptr;  // problems that smooth on the level (it is not their coarsest)
        int nsmooth = 0;
        Tile *tiles = nullptr;  // 32 x 32 tiles of the smoothing problems
        int ntiles = 0;
        int *coarse = nullptr;  // problems whose coarsest level this is
        int ncoarse = 0;
        int coarse_n = 0;       // their side (the largest)
        void *u = nullptr, *rhs = nullptr, *tmp = nullptr, *fvx = nullptr, *fvy = nullptr;  // level arrays (T)
    };
    std::vector<LevelDev> lv;
    Lvl<double> *d_lvl0_f64 = nullptr;  // level-0 entries in F64 (the Krylov passes)
    double *d_partials = nullptr;
    unsigned *d_tickets = nullptr;
    BState *d_state = nullptr;
    // per-problem states and the active count reach mapped page-locked memory written by the
    // device: no copy engine, so no wait behind a large transfer another stream has queued on it
    BState *h_state = nullptr, *h_state_dev = nullptr;
    int *h_count = nullptr, *h_count_dev = nullptr;
    // Krylov vectors (level-0 layout, F64): r, r_hat, p, v, s, t, p_hat, s_hat, tmp0 (the F64 cycle's partner)
    double *kv[9] = {};
    // graph of one iteration
    cudaGraphExec_t step_exec = nullptr;
    const void *graph_key[2] = {nullptr, nullptr};  // (x, b) the graph was recorded for
    ~fx_batch() {
        if (ctx) cudaStreamSynchronize(ctx->stream);
        if (step_exec) cudaGraphExecDestroy(step_exec);
        for (auto &a : dev_allocs) pool_free(ctx, a.first, a.second);
        if (h_state) cudaFreeHost(h_state);
        if (h_count) cudaFreeHost(h_count);
    }
    template <typename P>
    int dalloc(P **p, size_t bytes) {  // from the device's pool: a rebuilt batch reuses the memory
        void *q = nullptr;
        bool pooled = false;
        FX_TRY(pool_alloc(ctx, bytes, &q, &pooled));
        dev_allocs.emplace_back(q, pooled);
        *p = (P *)q;
        return FX_OK;
    }
    template <typename P>
    int upload(P **dst, const std::vector<P> &v) {  // ordered on the context's stream
        FX_TRY(dalloc(dst, v.size() * sizeof(P)));
        if (!v.empty())
            FX_CUDA(cudaMemcpyAsync(*dst, v.data(), v.size() * sizeof(P), cudaMemcpyHostToDevice, ctx->stream));
        return FX_OK;
    }
    K0 k0() const {
        return K0{d_lvl0_f64, (const double *)vx->ptr, (const double *)vy->ptr,
                  BOpC<double>{sigma, coeff, -nu}, d_state};
    }
};

namespace {

// chunk table of the given problems' arrays of side ns[p], `chunk` elements per item
std::vector<Chunk> make_chunks(const std::vector<int> &probs, const std::vector<int> &side, int chunk) {
    std::vector<Chunk> out;
    for (int p : probs) {
        const int n = side[p] * side[p];
        const int first = (int)out.size(), count = (n + chunk - 1) / chunk;
        for (int k = 0; k < count; k++) out.push_back(Chunk{p, k * chunk, std::min(chunk, n - k * chunk), first, count});
    }
    return out;
}

template <int K, typename F, typename Fin>
int bflat(fx_batch *B, const Chunk *items, int n, F f, Fin fin, const char *what) {
    if (n == 0) return FX_OK;
    timing_pre(B->ctx, what);
    k_bflat<K, F, Fin><<<n, kBT, 0, B->ctx->stream>>>(items, f, fin, B->d_partials, B->d_tickets);
    timing_post(B->ctx, 0.0);
    return check_launch(B->ctx, what);
}

// (re)build the chunk tables of level l for the batch's chunk size
int upload_chunks(fx_batch *B, int l) {
    auto &D = B->lv[l];
    const auto ch = make_chunks(B->lv_have[l], B->lv_side[l], B->chunk);
    const auto sch = make_chunks(B->lv_smooth[l], B->lv_side[l], B->chunk);
    FX_TRY(B->upload(&D.chunks, ch));
    FX_TRY(B->upload(&D.smooth_chunks, sch));
    D.nchunks = (int)ch.size();
    D.nsmooth = (int)sch.size();
    return FX_OK;
}

template <typename T>
int build_levels(fx_batch *B) {
    const int np = (int)B->np;
    std::vector<std::vector<Lvl<T>>> L(B->nlev, std::vector<Lvl<T>>(np, Lvl<T>{-1, 0, {}}));
    std::vector<std::vector<int>> side(B->nlev, std::vector<int>(np, 0));
    std::vector<long long> tot(B->nlev, 0);
    for (int p = 0; p < np; p++) {
        int n = B->n0[p];
        double h = 1.0 / (double)(n - 1);  // unit square: dx = dy = 1 / (n - 1)
        for (int l = 0; l < B->depth[p]; l++) {
            L[l][p] = Lvl<T>{tot[l], n, conv_consts<T>(h, h)};
            side[l][p] = n;
            tot[l] += (long long)n * n;
            n = (n - 1) / 2 + 1;
            h *= 2.0;
        }
    }
    B->lv.resize(B->nlev);
    const bool f32 = B->dtype == FX_F32;
    for (int l = 0; l < B->nlev; l++) {
        auto &D = B->lv[l];
        std::vector<int> have, smooth, coarse;
        for (int p = 0; p < np; p++) {
            if (B->depth[p] > l) have.push_back(p);
            if (B->depth[p] - 1 > l) smooth.push_back(p);
            if (B->depth[p] - 1 == l) coarse.push_back(p);
        }
        Lvl<T> *dl = nullptr;
        FX_TRY(B->upload(&dl, L[l]));
        D.lvl = dl;
        B->lv_side.push_back(side[l]);
        B->lv_have.push_back(have);
        B->lv_smooth.push_back(smooth);
        FX_TRY(upload_chunks(B, l));
        std::vector<Tile> tiles;
        for (int p : smooth) {
            const int nt = (side[l][p] + kTileB - 1) / kTileB;
            for (int ty = 0; ty < nt; ty++)
                for (int tx = 0; tx < nt; tx++) tiles.push_back(Tile{p, ty, tx});
        }
        FX_TRY(B->upload(&D.tiles, tiles));
        D.ntiles = (int)tiles.size();
        FX_TRY(B->upload(&D.coarse, coarse));
        D.ncoarse = (int)coarse.size();
        for (int p : coarse) D.coarse_n = std::max(D.coarse_n, side[l][p]);
        if (l > 0 || f32) {
            T *u, *rhs, *tmp, *fx_, *fy;
            FX_TRY(B->dalloc(&u, tot[l] * sizeof(T)));
            FX_TRY(B->dalloc(&rhs, tot[l] * sizeof(T)));
            FX_TRY(B->dalloc(&tmp, tot[l] * sizeof(T)));
            FX_TRY(B->dalloc(&fx_, tot[l] * sizeof(T)));
            FX_TRY(B->dalloc(&fy, tot[l] * sizeof(T)));
            D.u = u;
            D.rhs = rhs;
            D.tmp = tmp;
            D.fvx = fx_;
            D.fvy = fy;
        }
    }
    // level fields: level 0 of an F32 cycle casts the F64 fields, coarser levels inject
    fx_ctx *ctx = B->ctx;
    for (int l = (f32 ? 0 : 1); l < B->nlev; l++) {
        auto &D = B->lv[l];
        for (int k = 0; k < 2; k++) {
            T *dst = (T *)(k ? D.fvy : D.fvx);
            if (l == 0) {
                FX_TRY((bflat<0>(B, D.chunks, D.nchunks,
                                 BfCast<double, T>{B->d_lvl0_f64, (const Lvl<T> *)D.lvl,
                                                   (const double *)(k ? B->vy : B->vx)->ptr, dst, nullptr, nullptr},
                                 NoFinB{}, "batch_fields")));
            } else if (l == 1 && !f32) {
                FX_TRY((bflat<0>(B, D.chunks, D.nchunks,
                                 BfInject<double, T>{B->d_lvl0_f64, (const Lvl<T> *)D.lvl,
                                                     (const double *)(k ? B->vy : B->vx)->ptr, dst},
                                 NoFinB{}, "batch_fields")));
            } else {
                const auto &F = B->lv[l - 1];
                FX_TRY((bflat<0>(B, D.chunks, D.nchunks,
                                 BfInject<T, T>{(const Lvl<T> *)F.lvl, (const Lvl<T> *)D.lvl,
                                                (const T *)(k ? F.fvy : F.fvx), dst},
                                 NoFinB{}, "batch_fields")));
            }
        }
    }
    FX_CUDA(cudaStreamSynchronize(ctx->stream));
    return FX_OK;
}

// z = M r for every problem that has not halted, z and r level-0 F64 vectors (z zeroed here).
template <typename T>
int batch_cycle(fx_batch *B, double *z, const double *r) {
    fx_ctx *ctx = B->ctx;
    const int nl = B->nlev;
    const BOpC<T> O{(T)B->sigma, (T)B->coeff, (T)-B->nu};
    const T omega = (T)B->omega;
    auto args = [&](int l) -> LvlArgs<T> {
        const auto &D = B->lv[l];
        const T *fvx = (const T *)D.fvx, *fvy = (const T *)D.fvy;
        if (l == 0 && B->dtype == FX_F64) {
            fvx = (const T *)B->vx->ptr;
            fvy = (const T *)B->vy->ptr;
        }
        return LvlArgs<T>{(const Lvl<T> *)D.lvl, fvx, fvy, O, B->d_state};
    };
    std::vector<T *> cur(nl), oth(nl);
    std::vector<const T *> rhs(nl);
    const auto &D0 = B->lv[0];
    if (B->dtype == FX_F64) {
        cur[0] = (T *)z;
        oth[0] = (T *)B->kv[8];
        rhs[0] = (const T *)r;
        FX_TRY((bflat<0>(B, B->d_chunk0, B->nchunk0, BfZero<T>{args(0), cur[0]}, NoFinB{}, "batch_zero")));
    } else {
        cur[0] = (T *)D0.u;
        oth[0] = (T *)D0.tmp;
        rhs[0] = (const T *)D0.rhs;
        FX_TRY((bflat<0>(B, B->d_chunk0, B->nchunk0,
                         BfCast<double, T>{B->d_lvl0_f64, (const Lvl<T> *)D0.lvl, r, (T *)D0.rhs, (T *)D0.u,
                                           B->d_state},
                         NoFinB{}, "batch_convert")));
    }
    for (int l = 1; l < nl; l++) {
        cur[l] = (T *)B->lv[l].u;
        oth[l] = (T *)B->lv[l].tmp;
        rhs[l] = (const T *)B->lv[l].rhs;
    }
    auto smooth = [&](int l, size_t n) -> int {
        const auto &D = B->lv[l];
        size_t k = 0;
        for (; k + 2 <= n; k += 2) {
            if (D.ntiles) {
                timing_pre(ctx, "batch_sweep2");
                k_bsweep2<T><<<D.ntiles, 256, 0, ctx->stream>>>(D.tiles, args(l), cur[l], oth[l], rhs[l], omega);
                timing_post(ctx, 0.0);
                FX_TRY(check_launch(ctx, "batch_sweep2"));
            }
            std::swap(cur[l], oth[l]);
        }
        for (; k < n; k++) {
            FX_TRY((bflat<0>(B, D.smooth_chunks, D.nsmooth, BfSweep<T>{args(l), cur[l], rhs[l], oth[l], omega},
                             NoFinB{}, "batch_sweep")));
            std::swap(cur[l], oth[l]);
        }
        return FX_OK;
    };
    auto coarse = [&](int l) -> int {
        const auto &D = B->lv[l];
        if (!D.ncoarse) return FX_OK;
        const size_t n = (size_t)D.coarse_n * D.coarse_n;
        size_t t = ((n + 31) / 32) * 32;
        t = std::min<size_t>(std::max<size_t>(t, 32), 1024);
        k_bcoarse<T><<<D.ncoarse, (unsigned)t, 2 * n * sizeof(T), ctx->stream>>>(D.coarse, args(l), cur[l], rhs[l],
                                                                                  omega, (int)B->coarse_sweeps);
        return check_launch(ctx, "batch_coarse_solve");
    };
    for (int l = 0; l < nl; l++) {
        const auto &D = B->lv[l];
        FX_TRY(coarse(l));  // problems whose coarsest level this is
        if (l == nl - 1) break;
        FX_TRY(smooth(l, B->n_pre));
        FX_TRY((bflat<0>(B, D.smooth_chunks, D.nsmooth, BfResid<T>{args(l), cur[l], rhs[l], oth[l]}, NoFinB{},
                         "batch_residual")));
        const auto &C = B->lv[l + 1];
        FX_TRY((bflat<0>(B, C.chunks, C.nchunks,
                         BfRestrict<T>{(const Lvl<T> *)D.lvl, (const Lvl<T> *)C.lvl, oth[l], (T *)C.rhs, cur[l + 1],
                                       B->d_state},
                         NoFinB{}, "batch_restrict")));
    }
    for (int l = nl - 2; l >= 0; l--) {
        const auto &D = B->lv[l], &C = B->lv[l + 1];
        FX_TRY((bflat<0>(B, D.smooth_chunks, D.nsmooth,
                         BfProlong<T>{(const Lvl<T> *)D.lvl, (const Lvl<T> *)C.lvl, cur[l + 1], cur[l], B->d_state},
                         NoFinB{}, "batch_prolong")));
        FX_TRY(smooth(l, B->n_post));
    }
    if (B->dtype == FX_F64) {
        if (cur[0] != (T *)z)
            FX_TRY((bflat<0>(B, B->d_chunk0, B->nchunk0, BfCopy<T>{(const Lvl<T> *)D0.lvl, cur[0], (T *)z, B->d_state},
                             NoFinB{}, "batch_copy")));
        return FX_OK;
    }
    return bflat<0>(B, B->d_chunk0, B->nchunk0,
                    BfCast<T, double>{(const Lvl<T> *)D0.lvl, B->d_lvl0_f64, cur[0], z, nullptr, B->d_state}, NoFinB{},
                    "batch_convert");
}

int cycle(fx_batch *B, double *z, const double *r) {
    return B->dtype == FX_F64 ? batch_cycle<double>(B, z, r) : batch_cycle<float>(B, z, r);
}

// One BiCGSTAB iteration of every problem still running (bicgstab.rs:244-338, right-preconditioned).
int bicg_step(fx_batch *B, double *x) {
    double *r = B->kv[0], *rh = B->kv[1], *p = B->kv[2], *v = B->kv[3], *s = B->kv[4], *t = B->kv[5], *ph = B->kv[6],
           *sh = B->kv[7];
    const K0 k = B->k0();
    FX_TRY((bflat<0>(B, B->d_chunk0, B->nchunk0, BfP{k, p, r, v}, NoFinB{}, "batch_bicg_p")));
    FX_TRY(cycle(B, ph, p));
    FX_TRY((bflat<1>(B, B->d_chunk0, B->nchunk0, BfAr{k, ph, v, rh, 0}, FinRv{B->d_state}, "batch_bicg_v")));
    FX_TRY((bflat<1>(B, B->d_chunk0, B->nchunk0, BfS{k, r, v, s}, FinS{B->d_state}, "batch_bicg_s")));
    FX_TRY(cycle(B, sh, s));
    FX_TRY((bflat<2>(B, B->d_chunk0, B->nchunk0, BfAr{k, sh, t, s, 1}, FinT{B->d_state}, "batch_bicg_t")));
    return bflat<2>(B, B->d_chunk0, B->nchunk0, BfFinish{k, x, r, ph, sh, t, s, rh}, FinEnd{B->d_state},
                    "batch_bicg_finish");
}

__global__ void k_bstates_out(const BState *__restrict__ d, BState *h, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) h[i] = d[i];
}

// every problem's state into the mapped host array (synchronises)
int states_out(fx_batch *B) {
    const int n = (int)B->np;
    k_bstates_out<<<(n + 255) / 256, 256, 0, B->ctx->stream>>>(B->d_state, B->h_state_dev, n);
    FX_TRY(check_launch(B->ctx, "batch_states_out"));
    FX_CUDA(cudaStreamSynchronize(B->ctx->stream));
    return FX_OK;
}

int read_active(fx_batch *B, int *active) {
    k_bcount<<<1, 256, 0, B->ctx->stream>>>(B->d_state, (int)B->np, B->h_count_dev);
    FX_TRY(check_launch(B->ctx, "batch_count"));
    FX_CUDA(cudaStreamSynchronize(B->ctx->stream));
    *active = *(volatile int *)B->h_count;
    return FX_OK;
}

int check_vec(const fx_batch *B, const fx_buf *v, const char *name) {
    FX_TRY(check_buf(v, name));
    if (v->dtype != FX_F64 || (long long)v->len != B->total0)
        return fail(FX_ERR_DIMENSION_MISMATCH, std::string("batch: ") + name + " must be an F64 buffer of " +
                                                   std::to_string(B->total0) + " values (every problem's grid)");
    return FX_OK;
}

}  // namespace

extern "C" {

int fx_batch_destroy(fx_batch *B) {
    delete B;
    return FX_OK;
}

int fx_batch_create(fx_ctx *ctx, size_t count, const size_t *grid_side, double nu, double sigma, double coeff,
                    const fx_buf *vx, const fx_buf *vy, int cycle_dtype, size_t n_pre, size_t n_post, double omega,
                    size_t coarse_max, size_t coarse_sweeps, fx_batch **out) {
    if (!ctx || !grid_side || !vx || !vy || !out) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    if (count == 0 || count > (1u << 20)) return fail(FX_ERR_INVALID_ARGUMENT, "batch: 1 to 2^20 problems");
    if (cycle_dtype != FX_F32 && cycle_dtype != FX_F64) return fail(FX_ERR_INVALID_ARGUMENT, "unknown dtype");
    if (vx->dtype != FX_F64 || vy->dtype != FX_F64) return fail(FX_ERR_INVALID_ARGUMENT, "batch: velocity fields must be F64");
    fx_batch *B = new fx_batch();
    B->ctx = ctx;
    B->dtype = cycle_dtype;
    B->np = count;
    B->nu = nu;
    B->sigma = sigma;
    B->coeff = coeff;
    B->omega = omega;
    B->n_pre = n_pre;
    B->n_post = n_post;
    B->coarse_sweeps = coarse_sweeps;
    B->vx = vx;
    B->vy = vy;
    auto bad = [&](const std::string &m) {
        delete B;
        return fail(FX_ERR_INVALID_GRID, "batch: " + m);
    };
    long long tot = 0;
    for (size_t p = 0; p < count; p++) {
        const size_t n = grid_side[p];
        if (n < 5 || n > 65537 || ((n - 1) & (n - 2)) != 0) return bad("every grid side must be 2^k + 1 (5 <= side <= 65537)");
        B->off0.push_back(tot);
        tot += (long long)n * (long long)n;
        if (tot > (1ll << 31) - 1) return bad("too many points for one batch");
        int d = 1;
        for (size_t r = n; r - 2 > coarse_max && (r - 1) % 2 == 0; r = (r - 1) / 2 + 1) d++;
        const size_t cn = (n - 1) / (1u << (d - 1)) + 1;
        if (cn * cn > 4096 || 2 * cn * cn * (cycle_dtype == FX_F64 ? 8 : 4) > 48 * 1024)
            return bad("coarsest level too large for the one-block solve (lower coarse_max)");
        B->n0.push_back((int)n);
        B->depth.push_back(d);
        B->nlev = std::max(B->nlev, d);
    }
    B->off0.push_back(tot);
    B->total0 = tot;
    if ((long long)vx->len != tot || (long long)vy->len != tot) return bad("velocity fields must hold every problem's grid");
    std::vector<int> all(count), side0(B->n0);
    for (size_t p = 0; p < count; p++) all[p] = (int)p;
    const auto ch0 = make_chunks(all, side0, B->chunk);
    int st = B->upload(&B->d_chunk0, ch0);
    B->nchunk0 = (int)ch0.size();
    std::vector<Lvl<double>> l0(count);
    for (size_t p = 0; p < count; p++) {
        const double h = 1.0 / (double)(B->n0[p] - 1);
        l0[p] = Lvl<double>{B->off0[p], B->n0[p], conv_consts<double>(h, h)};
    }
    if (st == FX_OK) st = B->upload(&B->d_lvl0_f64, l0);
    // partials for the smallest chunk a batch may be given (fx_batch_set_chunk)
    size_t maxchunks = 0;
    for (size_t p = 0; p < count; p++) maxchunks += ((size_t)B->n0[p] * B->n0[p] + 255) / 256;
    if (st == FX_OK) st = B->dalloc(&B->d_partials, maxchunks * 4 * sizeof(double));
    if (st == FX_OK) st = B->dalloc(&B->d_tickets, count * sizeof(unsigned));
    if (st == FX_OK) st = B->dalloc(&B->d_state, count * sizeof(BState));
    for (int k = 0; k < 9 && st == FX_OK; k++) st = B->dalloc(&B->kv[k], (size_t)tot * sizeof(double));
    if (st == FX_OK && (cudaHostAlloc(&B->h_state, count * sizeof(BState), cudaHostAllocMapped) != cudaSuccess ||
                        cudaHostGetDevicePointer((void **)&B->h_state_dev, B->h_state, 0) != cudaSuccess ||
                        cudaHostAlloc(&B->h_count, sizeof(int), cudaHostAllocMapped) != cudaSuccess ||
                        cudaHostGetDevicePointer((void **)&B->h_count_dev, B->h_count, 0) != cudaSuccess))
        st = fail(FX_ERR_BACKEND, "batch: host allocation failed");
    if (st == FX_OK) st = B->dtype == FX_F64 ? build_levels<double>(B) : build_levels<float>(B);
    if (st != FX_OK) {
        delete B;
        return st;
    }
    *out = B;
    return FX_OK;
}

int fx_batch_set_chunk(fx_batch *B, size_t elements) {
    if (!B) return fail(FX_ERR_INVALID_ARGUMENT, "null batch");
    if (elements < 256 || elements > 65536 || (elements % 256) != 0)
        return fail(FX_ERR_INVALID_ARGUMENT, "batch: chunk must be a multiple of 256 elements in [256, 65536]");
    FX_CUDA(cudaStreamSynchronize(B->ctx->stream));
    B->chunk = (int)elements;
    std::vector<int> all(B->np);
    for (size_t p = 0; p < B->np; p++) all[p] = (int)p;
    const auto ch0 = make_chunks(all, B->n0, B->chunk);
    FX_TRY(B->upload(&B->d_chunk0, ch0));  // the old tables stay allocated until the batch goes
    B->nchunk0 = (int)ch0.size();
    for (int l = 0; l < B->nlev; l++) FX_TRY(upload_chunks(B, l));
    if (B->step_exec) cudaGraphExecDestroy(B->step_exec);  // recorded with the old tables
    B->step_exec = nullptr;
    B->graph_key[0] = B->graph_key[1] = nullptr;
    return FX_OK;
}

int fx_batch_layout(const fx_batch *B, size_t *offsets, size_t *levels) {
    if (!B || !offsets) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    for (size_t p = 0; p <= B->np; p++) offsets[p] = (size_t)B->off0[p];
    if (levels)
        for (size_t p = 0; p < B->np; p++) levels[p] = (size_t)B->depth[p];
    return FX_OK;
}

int fx_batch_apply(fx_batch *B, const fx_buf *v, fx_buf *out) {
    if (!B) return fail(FX_ERR_INVALID_ARGUMENT, "null batch");
    FX_TRY(check_vec(B, v, "v"));
    FX_TRY(check_vec(B, out, "out"));
    if (v->ptr == out->ptr) return fail(FX_ERR_INVALID_ARGUMENT, "v and out must be distinct");
    FX_CUDA(cudaMemsetAsync(B->d_state, 0, B->np * sizeof(BState), B->ctx->stream));
    K0 k = B->k0();
    FX_TRY((bflat<1>(B, B->d_chunk0, B->nchunk0,
                     BfAr{k, (const double *)v->ptr, (double *)out->ptr, (const double *)v->ptr, 0}, NoFinB{},
                     "batch_apply")));
    FX_CUDA(cudaStreamSynchronize(B->ctx->stream));
    return FX_OK;
}

int fx_batch_residual_norms(fx_batch *B, const fx_buf *x, const fx_buf *b, double *norms) {
    if (!B || !norms) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    FX_TRY(check_vec(B, x, "x"));
    FX_TRY(check_vec(B, b, "b"));
    fx_ctx *ctx = B->ctx;
    FX_CUDA(cudaMemsetAsync(B->d_state, 0, B->np * sizeof(BState), ctx->stream));
    // r = b - A x into the batch's r vector; ||r||^2 per problem into the state's resid slot
    FX_TRY((bflat<2>(B, B->d_chunk0, B->nchunk0,
                     BfInit{B->k0(), (const double *)x->ptr, (const double *)b->ptr, B->kv[0], B->kv[1]},
                     FinNorm2{B->d_state}, "batch_residual_norm")));
    FX_TRY(states_out(B));
    for (size_t p = 0; p < B->np; p++) norms[p] = B->h_state[p].resid;
    return FX_OK;
}

int fx_batch_precondition(fx_batch *B, fx_buf *z, const fx_buf *r) {
    if (!B) return fail(FX_ERR_INVALID_ARGUMENT, "null batch");
    FX_TRY(check_vec(B, z, "z"));
    FX_TRY(check_vec(B, r, "r"));
    if (z->ptr == r->ptr) return fail(FX_ERR_INVALID_ARGUMENT, "z and r must be distinct");
    FX_CUDA(cudaMemsetAsync(B->d_state, 0, B->np * sizeof(BState), B->ctx->stream));  // nobody halted
    FX_TRY(cycle(B, (double *)z->ptr, (const double *)r->ptr));
    FX_CUDA(cudaStreamSynchronize(B->ctx->stream));
    return FX_OK;
}

int fx_batch_bicgstab(fx_batch *B, fx_buf *x, const fx_buf *b, double rel_tol, size_t max_iter, int use_graph,
                      fx_stats *stats, size_t *iterations_run) {
    FX_RANGE("fx_batch_bicgstab");
    if (!B || !stats) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    FX_TRY(check_vec(B, x, "x"));
    FX_TRY(check_vec(B, b, "b"));
    if (x->ptr == b->ptr) return fail(FX_ERR_INVALID_ARGUMENT, "x and b must be distinct");
    if (!(rel_tol >= 0.0)) return fail(FX_ERR_INVALID_ARGUMENT, "tolerance must be non-negative");
    fx_ctx *ctx = B->ctx;
    double *xp = (double *)x->ptr;
    const K0 k = B->k0();
    // setup: tolerances, p = v = 0, r = b - A x, r_hat = r, the loop-top test of iteration 0
    FX_CUDA(cudaMemsetAsync(B->d_state, 0, B->np * sizeof(BState), ctx->stream));
    FX_TRY((bflat<1>(B, B->d_chunk0, B->nchunk0, BfNorm{k, (const double *)b->ptr}, FinTol{B->d_state, rel_tol,
                                                                                          (double)max_iter},
                     "batch_bicg_norm")));
    FX_CUDA(cudaMemsetAsync(B->kv[2], 0, (size_t)B->total0 * sizeof(double), ctx->stream));
    FX_CUDA(cudaMemsetAsync(B->kv[3], 0, (size_t)B->total0 * sizeof(double), ctx->stream));
    FX_TRY((bflat<2>(B, B->d_chunk0, B->nchunk0, BfInit{k, xp, (const double *)b->ptr, B->kv[0], B->kv[1]},
                     FinInit{B->d_state}, "batch_bicg_init")));
    // one iteration, recorded once into a graph for this (x, b) and replayed
    if (use_graph && (B->graph_key[0] != x->ptr || B->graph_key[1] != b->ptr || !B->step_exec)) {
        if (B->step_exec) cudaGraphExecDestroy(B->step_exec);
        B->step_exec = nullptr;
        FX_CUDA(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeRelaxed));
        const int st = bicg_step(B, xp);
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(ctx->stream, &g);
        if (st != FX_OK || e != cudaSuccess || !g || cudaGraphInstantiate(&B->step_exec, g, 0) != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            (void)cudaGetLastError();
            B->step_exec = nullptr;
            return st != FX_OK ? st : fail(FX_ERR_BACKEND, "batch: iteration graph could not be recorded");
        }
        cudaGraphDestroy(g);
        B->graph_key[0] = x->ptr;
        B->graph_key[1] = b->ptr;
    }
    auto step = [&]() -> int {
        if (use_graph) {
            FX_CUDA(cudaGraphLaunch(B->step_exec, ctx->stream));
            ctx->launches++;
            return FX_OK;
        }
        return bicg_step(B, xp);
    };
    // the solve needs at most max_iter + 1 iterations (the last one only runs the loop-top test);
    // the first check comes after a few, then after each one
    size_t run = 0;
    int active = 1;
    const size_t limit = max_iter + 1;
    while (run < limit && active > 0) {
        const size_t nb = run == 0 ? std::min<size_t>(4, limit) : 1;
        for (size_t j = 0; j < nb; j++) FX_TRY(step());
        run += nb;
        FX_TRY(read_active(B, &active));
    }
    if (iterations_run) *iterations_run = run;
    FX_TRY(states_out(B));
    for (size_t p = 0; p < B->np; p++) {
        const BState &S = B->h_state[p];
        stats[p].iterations = (size_t)S.iter;
        stats[p].residual = S.resid;
        stats[p].reason = S.done ? S.reason : FX_MAX_ITERATIONS;
    }
    return FX_OK;
}

}  // extern "C"
