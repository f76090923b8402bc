// fx_wcycle.cuh -- fused vertex-centred V(2,2)-cycle level kernels, one warp per strip.
//
// Two passes per level replace the separate sweep / residual / restriction / prolongation
// passes of a V(2,2)-cycle with a zero initial guess:
//
//   k_wdown: from the right-hand side b alone, x1 = w b (first sweep from zero), x2 = x1 +
//            w (b - A x1) (second sweep), res = b - A x2 and its full-weighting restriction
//            onto the coarse grid -- one pass that reads b and writes x2 and the coarse rhs;
//   k_wup:   f = x2 + bilinear(e_coarse), x3 = f + w (b - A f), z = x3 + w (b - A x3), written
//            out (at the finest level directly as the caller's vector, optionally with the
//            inner product <b, z> the preconditioned CG needs next).
//
// Both are organised for the instruction budget of a memory-bound pass:
//
//  - a warp owns a strip of 64 consecutive columns (its own ones plus halo columns on each
//    side that the neighbouring strips own) and marches it down a chunk of rows;
//  - each lane holds two adjacent columns' last three rows of every stage in registers; the
//    row above and below are register reads, the outer west / east neighbours one shuffle;
//  - every global load is a raw value issued D rows ahead into a register FIFO;
//  - no shared memory and no block barrier: the warps of a block are independent.
//
// Every point value is the expression of the separate kernels, so the fused cycle is
// bitwise equal to the unfused one.
#pragma once

#include <mutex>
#include <type_traits>
#include <utility>
#include <vector>

#include "fx_vcycle.cuh"

FX_CHECK_FILE(wcycle);

namespace fx {

constexpr int kStripWarps = 8;  // warps per block
constexpr int kStripUnroll = 6;  // the march is unrolled by 6 rows (= lcm(2, 3): row parity x 3-row windows)
// Shortest row chunk of a warp (even).  A chunk shorter than the unroll never takes the
// unrolled path without row tests, which costs instructions; but on the small levels, with
// fewer warps than the GPU has SMs, each warp's march is pure latency (a step waits on
// shuffles and dependent FP64 operations, with no other warp to hide them), and a chunk of
// c rows takes c + 5 (down) or c + 4 (up) steps, so short chunks finish sooner.
#ifndef FX_STRIP_MIN_CHUNK
#define FX_STRIP_MIN_CHUNK 2
#endif
constexpr int kStripMinChunk = FX_STRIP_MIN_CHUNK;
static_assert(kStripMinChunk >= 2 && kStripMinChunk % 2 == 0, "chunks start on even rows");
constexpr int kDownFifo = 6;    // rows of raw loads in flight (a divisor of kStripUnroll)
constexpr int kUpFifo = 6;
static_assert(kStripUnroll % kDownFifo == 0 && kStripUnroll % kUpFifo == 0, "FIFO depth must divide the unroll");

// The FP64 kernels hold twice the register bytes per value.  Their block shape, FIFO depth and
// minimum resident blocks per SM (the register cap of the launch bound) are set separately.  With
// 8-warp blocks the FP64 up pass needed 171 registers, one block (8 warps) per SM, and ran at 45 %
// of DRAM cycles; 4-warp blocks capped at 168 registers hold 12 warps per SM, and the down pass
// with a 3-row FIFO fits 128 registers at 16 warps.  On the 4095^2 FP64 MG-PCG solve (same box):
// 5.77 ms before, 4.93 ms with these settings (3-row FIFOs in both passes at 8 warps: 5.07 ms).
#ifndef FX_STRIP_F64_WARPS
#define FX_STRIP_F64_WARPS 4
#endif
#ifndef FX_STRIP_F64_UP_FIFO
#define FX_STRIP_F64_UP_FIFO 6
#endif
#ifndef FX_STRIP_F64_DOWN_FIFO
#define FX_STRIP_F64_DOWN_FIFO 3
#endif
#ifndef FX_STRIP_F64_UP_MINB
#if !defined(FX_STRIP_ASYNC) || FX_STRIP_ASYNC
#define FX_STRIP_F64_UP_MINB 4  // the row FIFO in shared memory leaves the up pass under 128 registers
#else
#define FX_STRIP_F64_UP_MINB 3
#endif
#endif
#ifndef FX_STRIP_F64_DOWN_MINB
#define FX_STRIP_F64_DOWN_MINB 4
#endif
template <typename T>
__host__ __device__ constexpr int strip_warps() { return sizeof(T) == 8 ? FX_STRIP_F64_WARPS : kStripWarps; }
template <typename T>
__host__ __device__ constexpr int up_fifo() { return sizeof(T) == 8 ? FX_STRIP_F64_UP_FIFO : kUpFifo; }
template <typename T>
__host__ __device__ constexpr int down_fifo() { return sizeof(T) == 8 ? FX_STRIP_F64_DOWN_FIFO : kDownFifo; }
template <typename T>
__host__ __device__ constexpr int up_minb() { return sizeof(T) == 8 ? FX_STRIP_F64_UP_MINB : 1; }
template <typename T>
__host__ __device__ constexpr int down_minb() { return sizeof(T) == 8 ? FX_STRIP_F64_DOWN_MINB : 1; }
static_assert(kStripUnroll % FX_STRIP_F64_UP_FIFO == 0 && kStripUnroll % FX_STRIP_F64_DOWN_FIFO == 0,
              "FIFO depth must divide the unroll");

// Row FIFOs in shared memory (FX_STRIP_ASYNC, the default): the raw loads of the rows ahead go to
// shared memory by cp.async instead of to registers, so a deep prefetch costs no registers.  PF
// rows are in flight per strip.  On the 4095^2 FP64 MG-PCG solve (CUDA events): 4.91 ms with the
// register FIFOs, 4.81 ms with PF = 6, 4.86 ms with PF = 8, 5.46 ms with PF = 12 (one box); 4.64
// against 4.82 ms for PF = 4 against 6 (another box, two alternating runs each).  The level-0 down
// pass went from 87.5 to 69.1 us (PF = 8), and the FP64 up pass, out of its register FIFO, fits
// 128 registers (16 warps per SM instead of 12).
#ifndef FX_STRIP_ASYNC
#define FX_STRIP_ASYNC 1
#endif
#ifndef FX_STRIP_F64_DOWN_PF
#define FX_STRIP_F64_DOWN_PF 4
#endif
#ifndef FX_STRIP_F64_UP_PF
#define FX_STRIP_F64_UP_PF 4
#endif
#ifndef FX_STRIP_F32_DOWN_PF
#define FX_STRIP_F32_DOWN_PF 4
#endif
#ifndef FX_STRIP_F32_UP_PF
#define FX_STRIP_F32_UP_PF 4
#endif
template <typename T>
__host__ __device__ constexpr int down_pf() { return sizeof(T) == 8 ? FX_STRIP_F64_DOWN_PF : FX_STRIP_F32_DOWN_PF; }
template <typename T>
__host__ __device__ constexpr int up_pf() { return sizeof(T) == 8 ? FX_STRIP_F64_UP_PF : FX_STRIP_F32_UP_PF; }

// One element (4 or 8 bytes) from global to shared memory, asynchronously; zero-filled when !valid
// (nothing is read then: src-size 0, and the address given is `any`, a valid one).
template <typename E>
__device__ __forceinline__ void cp_async_elem(E *dst, const E *src, bool valid, const E *any) {
    static_assert(sizeof(E) == 4 || sizeof(E) == 8, "4- or 8-byte elements");
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(d), "l"(valid ? src : any),
                 "n"((int)sizeof(E)), "r"(valid ? (int)sizeof(E) : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// A lane's two columns of PF + 1 rows of one array in shared memory.  The caller commits one
// cp.async group per step (every FIFO of the kernel in it) and waits for the group of the row it
// reads; a step refills the slot the previous step read (its value is in registers by then), so
// no copy lands in a slot that is still to be read.
template <typename E, int PF>
struct SmemFifo {
    E *base;  // this lane's column pair in slot 0; slot s at base + 64 s
    int rd, wr;
    __device__ __forceinline__ void init(E *warp_base, int lane) {
        base = warp_base + 2 * lane;
        rd = 0;
        wr = PF;
    }
    __device__ __forceinline__ void put_at(int slot, const E *src, bool va, bool vb, const E *any) {
        cp_async_elem(base + slot * 64, src, va, any);
        cp_async_elem(base + slot * 64 + 1, src + 1, vb, any);
    }
    __device__ __forceinline__ void put(const E *src, bool va, bool vb, const E *any) { put_at(wr, src, va, vb, any); }
    __device__ __forceinline__ E a() const { return base[rd * 64]; }
    __device__ __forceinline__ E b() const { return base[rd * 64 + 1]; }
    __device__ __forceinline__ void advance() {
        rd = rd == PF ? 0 : rd + 1;
        wr = wr == PF ? 0 : wr + 1;
    }
};

// dynamic shared memory of a strip launch: per warp, PF + 1 rows of 64 elements of each FIFO array
template <typename T, typename TB>
constexpr size_t wdown_smem() {
    return FX_STRIP_ASYNC ? (size_t)strip_warps<T>() * (down_pf<T>() + 1) * 64 * sizeof(TB) : 0;
}
template <typename T, typename TB>
constexpr size_t wup_smem() {
    return FX_STRIP_ASYNC ? (size_t)strip_warps<T>() * (up_pf<T>() + 1) * 64 * (sizeof(T) + sizeof(TB)) : 0;
}

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
    G.nstrips = (int)((cols - 1 + useful - 1) / useful);  // own ranges tile [0, cols - 1)
    if (G.nstrips < 1) G.nstrips = 1;
    // one wave of resident warps; chunks of at least kStripMinChunk rows
    const long target = capacity;
    long chunks = target / G.nstrips;
    if (chunks < 1) chunks = 1;
    long cr = ((long)rows + chunks - 1) / chunks;
    if (cr < kStripMinChunk) cr = kStripMinChunk;
    cr = (cr + 1) & ~1L;
    G.chunk_rows = (int)cr;
    G.nitems = (int)(G.nstrips * (((long)rows + cr - 1) / cr));
    return G;
}

__device__ __forceinline__ float shfl_w(float v) { return __shfl_up_sync(0xffffffffu, v, 1); }
__device__ __forceinline__ float shfl_e(float v) { return __shfl_down_sync(0xffffffffu, v, 1); }
__device__ __forceinline__ double shfl_w(double v) { return __shfl_up_sync(0xffffffffu, v, 1); }
__device__ __forceinline__ double shfl_e(double v) { return __shfl_down_sync(0xffffffffu, v, 1); }

// Two adjacent columns per lane: lane l of a strip holds columns ca = sb + 2l (even) and
// cb = ca + 1, so one shuffle per stage gives both points their outer neighbour, the column
// parity of every register is fixed, and a strip spans 64 columns.  A step whose rows all lie
// inside the chunk's interior takes a path without row tests (FAST); the first and last few
// steps of a chunk test every row.

template <bool B>
using fast_t = std::integral_constant<bool, B>;

// ---------------------------------------------------------------- down

constexpr int kDownOwn = 56;  // own columns per strip: lanes 2..29 (x1 -> x2 -> res -> FW: halo 4)

template <typename T, typename TB>
__global__ void __launch_bounds__(strip_warps<T>() * 32, down_minb<T>()) k_wdown(StripGeom G, const TB *__restrict__ b, T *__restrict__ x2g,
                                                             T *__restrict__ coarse, int ccols, VOp<T> op,
                                                             const int *skip) {
    grid_dep_enter();
    if (skip && *(volatile const int *)skip) return;
    [[maybe_unused]] constexpr int D = down_fifo<T>();
    constexpr int R = kStripUnroll;
    const int lane = threadIdx.x & 31;
    const int item = blockIdx.x * strip_warps<T>() + (threadIdx.x >> 5);
    if (item >= G.nitems) return;  // whole warps
    const int strip = item % G.nstrips, chunk = item / G.nstrips;
    const int rows = G.rows, cols = G.cols;
    const int ca = strip * kDownOwn - 4 + 2 * lane, cb = ca + 1;
    const bool ina = ca >= 1 && ca <= cols - 2, inb = cb >= 1 && cb <= cols - 2;
    const bool own = lane >= 2 && lane < 30;
    const bool sta = own && ina, stb = own && inb;
    const bool cpt = own && ca >= 2 && ca <= cols - 3;  // coarse point (fr, ca) for even fr
    const int r0 = chunk * G.chunk_rows, r1 = min(r0 + G.chunk_rows, rows);  // r0 even
    const long long nf = (long long)rows * cols, nc = (long long)((rows - 1) / 2 + 1) * ccols;  // extents
    (void)nf;
    (void)nc;
    // step q: b row q arrives; x1 row q; x2 row q-1; residual row q-2; full weighting of fine
    // row q-3 (even q-3 only)
    const int q_first = r0 - 3, q_last = r1 + 2;
    auto row_in = [&](int r) { return r >= 1 && r <= rows - 2; };
#if FX_STRIP_ASYNC
    constexpr int PF = down_pf<T>();
    // steps with every row test true: q-3 >= max(r0, 2), q + PF <= min(rows - 2, q_last)
    const int q_lo = max(r0, 2) + 3, q_hi = min(rows - 2, q_last) - PF;
    extern __shared__ __align__(16) unsigned char strip_smem[];
    SmemFifo<TB, PF> fifo;
    fifo.init(reinterpret_cast<TB *>(strip_smem) + (threadIdx.x >> 5) * ((PF + 1) * 64), lane);
#pragma unroll
    for (int k = 0; k < PF; k++) {
        const int q = q_first + k;
        const long long o = (long long)q * cols + ca;
        const bool rv = row_in(q) && q <= q_last;
        fifo.put_at(k, b + o, rv && ina && FX_IN(o, nf), rv && inb && FX_IN(o + 1, nf), b);
        cp_async_commit();
    }
#else
    // steps with every row test true: q-3 >= max(r0, 2), q + D <= min(rows - 2, q_last)
    const int q_lo = max(r0, 2) + 3, q_hi = min(rows - 2, q_last) - D;
    TB fa[D], fb[D];
#pragma unroll
    for (int k = 0; k < D; k++) {
        const int q = q_first + k;
        fa[k] = (TB)0;
        fb[k] = (TB)0;
        if (row_in(q) && q <= q_last) {
            if (ina && FX_IN((long long)q * cols + ca, nf)) fa[k] = b[(size_t)q * cols + ca];
            if (inb && FX_IN((long long)q * cols + cb, nf)) fb[k] = b[(size_t)q * cols + cb];
        }
    }
#endif

    T bwa[3] = {}, bwb[3] = {}, x1a[3] = {}, x1b[3] = {}, x2a[3] = {}, x2b[3] = {};
    T rsa[3] = {}, rsb[3] = {}, rwa[3] = {};
    // element offsets of this lane's column ca, advanced one row per step: the rhs row being
    // fetched (q + D), the x2 row being stored (q - 1), and the coarse row of fine row q - 3
#if FX_STRIP_ASYNC
    long long ob = (long long)(q_first + PF) * cols + ca;
#else
    long long ob = (long long)(q_first + D) * cols + ca;
#endif
    long long ox = (long long)(q_first - 1) * cols + ca;
    long long oc = (long long)((q_first - 3) >> 1) * ccols + (ca >> 1);  // q_first - 3 even
    auto step = [&](int k, int q, auto fast) {
        constexpr bool F = decltype(fast)::value;
        const int s0 = k % 3, s1 = (k + 2) % 3, s2 = (k + 1) % 3;  // slots of rows q, q-1, q-2
        // row q: rhs and x1 = w b (0 on the ring); refill with row q + D
        {
#if FX_STRIP_ASYNC
            cp_async_wait<PF - 1>();  // row q's group is complete
            const T ba = (T)fifo.a(), bb = (T)fifo.b();
#else
            const T ba = (T)fa[k % D], bb = (T)fb[k % D];
#endif
            const bool rin = F || row_in(q);
            bwa[s0] = ba;
            bwb[s0] = bb;
            x1a[s0] = (rin && ina) ? fx_fma(op.wd, ba, (T)0) : (T)0;
            x1b[s0] = (rin && inb) ? fx_fma(op.wd, bb, (T)0) : (T)0;
#if FX_STRIP_ASYNC
            const int qn = q + PF;
            const bool rv = F || (row_in(qn) && qn <= q_last);
            fifo.put(b + ob, rv && ina && FX_IN(ob, nf), rv && inb && FX_IN(ob + 1, nf), b);
            cp_async_commit();
            fifo.advance();
#else
            const int qn = q + D;
            if (F || (row_in(qn) && qn <= q_last)) {
                if (ina && FX_IN(ob, nf)) fa[k % D] = b[ob];
                if (inb && FX_IN(ob + 1, nf)) fb[k % D] = b[ob + 1];
            }
#endif
            ob += cols;
        }
        // row q-1: x2
        {
            const T xa = x1a[s1], xb = x1b[s1];
            const T wa = shfl_w(xb), eb = shfl_e(xa);
            const bool rin = F || row_in(q - 1);
            T va = (T)0, vb = (T)0;
            if (rin && ina) va = fx_fma(op.wd, bwa[s1] - op5v(op.a, xa, x1a[s2], x1a[s0], wa, xb), xa);
            if (rin && inb) vb = fx_fma(op.wd, bwb[s1] - op5v(op.a, xb, x1b[s2], x1b[s0], xa, eb), xb);
            x2a[s1] = va;
            x2b[s1] = vb;
            if (F || (rin && q - 1 >= r0 && q - 1 < r1)) {
                if (sta && FX_IN(ox, nf)) x2g[ox] = va;
                if (stb && FX_IN(ox + 1, nf)) x2g[ox + 1] = vb;
            }
            ox += cols;
        }
        // row q-2: residual, and the residual west of ca for the restriction
        {
            const T xa = x2a[s2], xb = x2b[s2];
            const T wa = shfl_w(xb), eb = shfl_e(xa);
            const bool rin = F || row_in(q - 2);
            T va = (T)0, vb = (T)0;
            if (rin && ina) va = bwa[s2] - op5v(op.a, xa, x2a[s0], x2a[s1], wa, xb);
            if (rin && inb) vb = bwb[s2] - op5v(op.a, xb, x2b[s0], x2b[s1], xa, eb);
            rsa[s2] = va;
            rsb[s2] = vb;
            rwa[s2] = shfl_w(vb);
        }
        // fine row q-3 (residual rows q-4 / q-3 / q-2 in slots s1 / s0 / s2): full weighting
        // onto coarse row (q-3) / 2 at coarse column ca / 2
        if (!(k & 1)) {  // q - 3 even (r0 even, so q_first odd)
            const int fr = q - 3;
            if (cpt && (F || (fr >= r0 && fr < r1 && fr >= 2 && fr <= rows - 3)) && FX_IN(oc, nc)) {
                const T e = (rsa[s1] + rsa[s2]) + (rwa[s0] + rsb[s0]);
                const T d = (rwa[s1] + rsb[s1]) + (rwa[s2] + rsb[s2]);
                coarse[oc] = ((T)4 * rsa[s0] + ((T)2 * e + d)) * (T)0.0625;
            }
            oc += ccols;
        }
    };
    for (int qb = q_first; qb <= q_last; qb += R) {
        if (qb >= q_lo && qb + R - 1 <= q_hi) {
#pragma unroll
            for (int k = 0; k < R; k++) step(k, qb + k, fast_t<true>{});
        } else {
#pragma unroll
            for (int k = 0; k < R; k++) {
                if (qb + k > q_last) break;  // uniform over the warp
                step(k, qb + k, fast_t<false>{});
            }
        }
    }
#if FX_STRIP_ASYNC
    cp_async_wait<0>();  // no copy outlives the warp
#endif
}

// ---------------------------------------------------------------- up

constexpr int kUpOwn = 60;  // own columns per strip: lanes 1..30 (f -> x3 -> z: halo 2)

template <typename T, typename TB, typename TZ, bool RZ, typename Fin>
__global__ void __launch_bounds__(strip_warps<T>() * 32, up_minb<T>()) k_wup(StripGeom G, const T *__restrict__ x2g,
                                                           const T *__restrict__ e, int ccols,
                                                           const TB *__restrict__ b, TZ *__restrict__ z, VOp<T> op,
                                                           Fin fin, RedArgs<1> ra, const int *skip) {
    grid_dep_enter();
    if (skip && *(volatile const int *)skip) return;
    [[maybe_unused]] constexpr int D = up_fifo<T>();
    constexpr int R = kStripUnroll;
#if FX_STRIP_ASYNC
    constexpr int PF = up_pf<T>();
    extern __shared__ __align__(16) unsigned char strip_smem[];
#endif
    const int lane = threadIdx.x & 31;
    const int item = blockIdx.x * strip_warps<T>() + (threadIdx.x >> 5);
    CSum acc[1] = {CSum{0.0, 0.0}};
    if (item < G.nitems) {  // idle warps still join the block reduction
        const int strip = item % G.nstrips, chunk = item / G.nstrips;
        const int rows = G.rows, cols = G.cols, crows = (rows - 1) / 2 + 1;
        const int ca = strip * kUpOwn - 2 + 2 * lane, cb = ca + 1;
        const bool ina = ca >= 1 && ca <= cols - 2, inb = cb >= 1 && cb <= cols - 2;
        const bool own = lane >= 1 && lane < 31;
        const bool sta = own && ina, stb = own && inb;
        const int kc = ca >> 1;  // coarse column of ca; cb interpolates between kc and kc + 1
        const bool ce0 = kc >= 0 && kc < ccols && (ina || inb), ce1 = kc + 1 < ccols && inb;
        const int r0 = chunk * G.chunk_rows, r1 = min(r0 + G.chunk_rows, rows);  // r0 even
        // step q: F0 row q = x2 + P e; x3 row q-1; z row q-2
        const int q_first = r0 - 2, q_last = r1 + 1;  // q_first even
#if FX_STRIP_ASYNC
        // steps with every row test true: q-2 >= max(r0, 1), q + PF <= min(rows - 2, q_last)
        const int q_lo = max(r0, 1) + 2, q_hi = min(rows - 2, q_last) - PF;
#else
        // steps with every row test true: q-2 >= max(r0, 1), q + D <= min(rows - 2, q_last)
        const int q_lo = max(r0, 1) + 2, q_hi = min(rows - 2, q_last) - D;
#endif
        const int m_last = (q_last >> 1) + 1;  // last coarse row any step reads
        const long long nf = (long long)rows * cols, nc = (long long)crows * ccols;  // extents
        (void)nf;
        (void)nc;
        auto row_in = [&](int r) { return r >= 1 && r <= rows - 2; };

        // FIFO of D fine rows: raw x2 and b of both columns; per fine row pair (2m, 2m+1) of the
        // unrolled step the coarse row m+1 at columns kc, kc+1, R rows ahead (row m is kept
        // from the previous pair)
        T ea_[R / 2], eb_[R / 2];
#if FX_STRIP_ASYNC
        // x2 FIFOs of the block's warps, then their b FIFOs
        SmemFifo<T, PF> fx;
        SmemFifo<TB, PF> fbq;
        fx.init(reinterpret_cast<T *>(strip_smem) + (threadIdx.x >> 5) * ((PF + 1) * 64), lane);
        fbq.init(reinterpret_cast<TB *>(strip_smem + (size_t)strip_warps<T>() * (PF + 1) * 64 * sizeof(T)) +
                     (threadIdx.x >> 5) * ((PF + 1) * 64),
                 lane);
        auto put_row = [&](int slot, int q, long long o, bool fast) {  // slot < 0: the FIFOs' next slot
            const bool rv = fast || (row_in(q) && q <= q_last);
            const bool va = rv && ina && FX_IN(o, nf), vb = rv && inb && FX_IN(o + 1, nf);
            if (slot < 0) {
                fx.put(x2g + o, va, vb, x2g);
                fbq.put(b + o, va, vb, b);
            } else {
                fx.put_at(slot, x2g + o, va, vb, x2g);
                fbq.put_at(slot, b + o, va, vb, b);
            }
            cp_async_commit();
        };
#else
        T xa_[D], xb_[D];
        TB ba_[D], bb_[D];
#endif
        // o: element offset of (q, ca) / (m, kc)
        [[maybe_unused]] auto load_row = [&](int q, int k, long long o) {
#if !FX_STRIP_ASYNC
            xa_[k] = (T)0;
            xb_[k] = (T)0;
            ba_[k] = (TB)0;
            bb_[k] = (TB)0;
            if (row_in(q) && q <= q_last) {
                if (ina && FX_IN(o, nf)) {
                    xa_[k] = x2g[o];
                    ba_[k] = b[o];
                }
                if (inb && FX_IN(o + 1, nf)) {
                    xb_[k] = x2g[o + 1];
                    bb_[k] = b[o + 1];
                }
            }
#else
            (void)q;
            (void)k;
            (void)o;
#endif
        };
        auto load_coarse = [&](int m, T &v0, T &v1, long long o) {
            v0 = (T)0;
            v1 = (T)0;
            if (m >= 0 && m < crows && m <= m_last) {
                if (ce0 && FX_IN(o, nc)) v0 = e[o];
                if (ce1 && FX_IN(o + 1, nc)) v1 = e[o + 1];
            }
        };
        T c0a, c0b;  // coarse row q >> 1 of the current pair, columns kc, kc+1
        load_coarse(q_first >> 1, c0a, c0b, (long long)(q_first >> 1) * ccols + kc);
#if FX_STRIP_ASYNC
#pragma unroll
        for (int k = 0; k < PF; k++) put_row(k, q_first + k, (long long)(q_first + k) * cols + ca, false);
#else
#pragma unroll
        for (int k = 0; k < D; k++) load_row(q_first + k, k, (long long)(q_first + k) * cols + ca);
#endif
#pragma unroll
        for (int k = 0; k < R; k += 2) {
            const int m = ((q_first + k) >> 1) + 1;
            load_coarse(m, ea_[k / 2], eb_[k / 2], (long long)m * ccols + kc);
        }
        // running element offsets, advanced as the march goes: the fine row being fetched
        // (q + D), the coarse row fetched at odd steps ((q + R + 1) / 2), the z row (q - 2)
#if FX_STRIP_ASYNC
        long long orow = (long long)(q_first + PF) * cols + ca;
#else
        long long orow = (long long)(q_first + D) * cols + ca;
#endif
        long long oe = (long long)((q_first + R + 2) >> 1) * ccols + kc;
        long long oz = (long long)(q_first - 2) * cols + ca;

        T fa[3] = {}, fb[3] = {}, x3a[3] = {}, x3b[3] = {};
        TB bwa[3] = {}, bwb[3] = {};
        auto step = [&](int k, int q, auto fast) {
            constexpr bool F = decltype(fast)::value;
            const int s0 = k % 3, s1 = (k + 2) % 3, s2 = (k + 1) % 3;  // rows q, q-1, q-2
            // row q: f = x2 + bilinear(e); the parities are fixed: ca even, cb odd, q odd <=> k odd
            {
                const bool ro = k & 1;
                const T e00 = c0a, e01 = c0b;              // coarse row q >> 1
                const T e10 = ea_[k / 2], e11 = eb_[k / 2];  // coarse row (q >> 1) + 1
                T pa, pb;
                if (ro) {
                    pa = (T)0.5 * (e00 + e10);                    // v_oe
                    pb = (T)0.25 * ((e00 + e10) + (e01 + e11));   // v_oo
                } else {
                    pa = e00;
                    pb = (T)0.5 * (e00 + e01);                    // v_eo
                }
                const bool rin = F || row_in(q);
#if FX_STRIP_ASYNC
                cp_async_wait<PF - 1>();  // row q's group is complete
                fa[s0] = (rin && ina) ? fx.a() + pa : (T)0;
                fb[s0] = (rin && inb) ? fx.b() + pb : (T)0;
                bwa[s0] = fbq.a();
                bwb[s0] = fbq.b();
#else
                fa[s0] = (rin && ina) ? xa_[k % D] + pa : (T)0;
                fb[s0] = (rin && inb) ? xb_[k % D] + pb : (T)0;
                bwa[s0] = ba_[k % D];
                bwb[s0] = bb_[k % D];
#endif
                if (ro) {  // the pair is done: its lower coarse row becomes the upper one
                    c0a = e10;
                    c0b = e11;
                    load_coarse((q + R + 1) >> 1, ea_[k / 2], eb_[k / 2], oe);
                    oe += ccols;
                }
#if FX_STRIP_ASYNC
                put_row(-1, q + PF, orow, F);
                fx.advance();
                fbq.advance();
#else
                const int qn = q + D;
                if (F) {
                    if (ina && FX_IN(orow, nf)) {
                        xa_[k % D] = x2g[orow];
                        ba_[k % D] = b[orow];
                    }
                    if (inb && FX_IN(orow + 1, nf)) {
                        xb_[k % D] = x2g[orow + 1];
                        bb_[k % D] = b[orow + 1];
                    }
                } else {
                    load_row(qn, k % D, orow);
                }
#endif
                orow += cols;
            }
            // row q-1: x3
            {
                const T fca = fa[s1], fcb = fb[s1];
                const T wa = shfl_w(fcb), eb = shfl_e(fca);
                const bool rin = F || row_in(q - 1);
                T va = (T)0, vb = (T)0;
                if (rin && ina) va = fx_fma(op.wd, (T)bwa[s1] - op5v(op.a, fca, fa[s2], fa[s0], wa, fcb), fca);
                if (rin && inb) vb = fx_fma(op.wd, (T)bwb[s1] - op5v(op.a, fcb, fb[s2], fb[s0], fca, eb), fcb);
                x3a[s1] = va;
                x3b[s1] = vb;
            }
            // row q-2: z
            {
                const T xa = x3a[s2], xb = x3b[s2];
                const T wa = shfl_w(xb), eb = shfl_e(xa);
                const int r = q - 2;
                if (F || (row_in(r) && r >= r0 && r < r1)) {
                    TZ *row = z + oz;
                    if (sta && FX_IN(oz, nf)) {
                        const TB bv = bwa[s2];
                        const T v = fx_fma(op.wd, (T)bv - op5v(op.a, xa, x3a[s0], x3a[s1], wa, xb), xa);
                        row[0] = (TZ)v;
                        if (RZ) csum_fma(acc[0], (double)bv, (double)(TZ)v);
                    }
                    if (stb && FX_IN(oz + 1, nf)) {
                        const TB bv = bwb[s2];
                        const T v = fx_fma(op.wd, (T)bv - op5v(op.a, xb, x3b[s0], x3b[s1], xa, eb), xb);
                        row[1] = (TZ)v;
                        if (RZ) csum_fma(acc[0], (double)bv, (double)(TZ)v);
                    }
                }
                oz += cols;
            }
        };
        for (int qb = q_first; qb <= q_last; qb += R) {
            if (qb >= q_lo && qb + R - 1 <= q_hi) {
#pragma unroll
                for (int k = 0; k < R; k++) step(k, qb + k, fast_t<true>{});
            } else {
#pragma unroll
                for (int k = 0; k < R; k++) {
                    if (qb + k > q_last) break;
                    step(k, qb + k, fast_t<false>{});
                }
            }
        }
#if FX_STRIP_ASYNC
        cp_async_wait<0>();  // no copy outlives the warp
#endif
    }
    if constexpr (RZ) grid_reduce<1>(acc, ra, fin);
}

// chunk_pct: the row chunks of a launch as a percentage of one wave of resident warps (100: one
// warp per resident slot; fewer, longer chunks below, more, shorter ones above)
inline long strip_capacity(long resident_warps, int chunk_pct) {
    const long cap = resident_warps * chunk_pct / 100;
    return cap < 1 ? 1 : cap;
}

// opt a strip kernel in to more than 48 KB of dynamic shared memory (the attribute is set per
// device and kernel; setting it again is harmless, so the record only saves calls)
template <typename K>
int strip_smem_optin(K kernel, size_t smem) {
    static std::mutex mu;
    static std::vector<std::pair<const void *, int>> done;
    int dev = 0;
    FX_CUDA(cudaGetDevice(&dev));
    const std::pair<const void *, int> key{reinterpret_cast<const void *>(kernel), dev};
    std::lock_guard<std::mutex> lk(mu);
    for (const auto &d : done)
        if (d == key) return FX_OK;
    FX_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    done.push_back(key);
    return FX_OK;
}

template <typename T, typename TB>
int launch_wdown(fx_ctx *ctx, size_t rows, size_t cols, const TB *b, T *x2, T *coarse, size_t ccols,
                 const VOp<T> &op, const int *skip, int chunk_pct = 100) {
    static std::atomic<int> occ{0};
    constexpr int W = strip_warps<T>();
    constexpr size_t smem = wdown_smem<T, TB>();
    if (smem > 48 * 1024) FX_TRY(strip_smem_optin(k_wdown<T, TB>, smem));
    const long cap = strip_capacity((long)band_capacity(ctx, k_wdown<T, TB>, occ, W * 32, smem) * W, chunk_pct);
    const StripGeom G = strip_geom(rows, cols, kDownOwn, cap);
    const int blocks = (G.nitems + W - 1) / W;
    timing_pre(ctx, "mg_down");
    launch_pdl(ctx, k_wdown<T, TB>, blocks, W * 32, smem, G, b, x2, coarse, (int)ccols, op, skip);
    // reads b, writes the smoothed x2 and the restricted coarse rhs
    const double pts = (double)rows * (double)cols, cpts = (double)((rows - 1) / 2 + 1) * (double)ccols;
    timing_post(ctx, pts, pts * (sizeof(TB) + sizeof(T)) + cpts * sizeof(T));
    return check_launch(ctx, "mg_down");
}

template <typename T, typename TB, typename TZ, bool RZ, typename Fin>
int launch_wup(fx_ctx *ctx, size_t rows, size_t cols, const T *x2, const T *e, size_t ccols, const TB *b, TZ *z,
               const VOp<T> &op, Fin fin, const int *skip, int chunk_pct = 100) {
    static std::atomic<int> occ{0};
    constexpr int W = strip_warps<T>();
    constexpr size_t smem = wup_smem<T, TB>();
    if (smem > 48 * 1024) FX_TRY(strip_smem_optin(k_wup<T, TB, TZ, RZ, Fin>, smem));
    const long cap =
        strip_capacity((long)band_capacity(ctx, k_wup<T, TB, TZ, RZ, Fin>, occ, W * 32, smem) * W, chunk_pct);
    const StripGeom G = strip_geom(rows, cols, kUpOwn, cap);
    const int blocks = (G.nitems + W - 1) / W;
    if (RZ && blocks > kMaxRedBlocks) return fail(FX_ERR_INVALID_ARGUMENT, "grid too large");
    timing_pre(ctx, "mg_up");
    launch_pdl(ctx, k_wup<T, TB, TZ, RZ, Fin>, blocks, W * 32, smem, G, x2, e, (int)ccols, b, z, op, fin,
               red_args<1>(ctx), skip);
    // reads x2, the coarse correction e and b, writes z
    const double pts = (double)rows * (double)cols, cpts = (double)((rows - 1) / 2 + 1) * (double)ccols;
    timing_post(ctx, pts, pts * (sizeof(T) + sizeof(TB) + sizeof(TZ)) + cpts * sizeof(T));
    return check_launch(ctx, "mg_up");
}

}  // namespace fx
