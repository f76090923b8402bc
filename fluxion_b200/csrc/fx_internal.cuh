// fx_internal.cuh -- shared internals of the sm_100a backend: context and buffer
// objects, error plumbing, compensated deterministic reductions and the
// row-marching stencil framework every grid kernel is built on.
#pragma once

#include <atomic>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

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
constexpr int kBandThreads = kBlock + 32;  // band kernels: 8 column warps + 1 halo warp

// ------------------------------------------------------------------ checked build
//
// Compiled with FX_CHECKED (the separate libfluxion_cuda_checked.so), the kernels test the
// indices they compute -- global offsets and shared-memory slots -- against the extent of the
// array addressed before each access.  An access outside is not made (a load gives zero, a
// store is dropped) and the first such event of each translation unit is written to that unit's
// device status word: the source file (as a hash of its name), the line, the index and the
// extent.  fx_checked_status reads and clears the words.  Nothing traps and nothing waits.  In
// the default build FX_IN is the constant true and every check compiles away.
struct CheckWord {
    unsigned code;  // 0: clear; 1: an index was out of range
    unsigned file;  // check_hash of the source file of the check
    int line;
    int pad;
    long long index, extent;
};

__host__ __device__ constexpr unsigned check_hash(const char *s, unsigned h = 2166136261u) {
    return *s ? check_hash(s + 1, (h ^ (unsigned char)*s) * 16777619u) : h;
}

// host: the readers of the units' words and the names of the files holding checks
using CheckReader = int (*)(CheckWord *out);
void check_register_unit(CheckReader reader);
void check_register_file(unsigned hash, const char *name);

#ifdef FX_CHECKED
static __device__ CheckWord g_check_word;

static __device__ __noinline__ void check_record(long long i, long long n, unsigned file, int line) {
    if (atomicCAS(&g_check_word.code, 0u, 1u) == 0u) {
        g_check_word.file = file;
        g_check_word.line = line;
        g_check_word.index = i;
        g_check_word.extent = n;
        __threadfence();
    }
}

__device__ __forceinline__ bool check_in(long long i, long long n, unsigned file, int line) {
    if ((unsigned long long)i < (unsigned long long)n) return true;
    check_record(i, n, file, line);
    return false;
}

#define FX_IN(i, n) (::fx::check_in((long long)(i), (long long)(n), ::fx::check_hash(__FILE__), __LINE__))

// one reader per translation unit (it reads that unit's copy of the word, then clears it)
static int check_read_unit(CheckWord *out) {
    if (cudaMemcpyFromSymbol(out, g_check_word, sizeof(CheckWord)) != cudaSuccess) return 1;
    const CheckWord zero{};
    return cudaMemcpyToSymbol(g_check_word, &zero, sizeof(CheckWord)) != cudaSuccess;
}
struct CheckUnitReg {
    CheckUnitReg() { check_register_unit(&check_read_unit); }
};
static CheckUnitReg g_check_unit_reg;
struct CheckFileReg {
    explicit CheckFileReg(const char *name) { check_register_file(check_hash(name), name); }
};
#define FX_CHECK_FILE(tag) static ::fx::CheckFileReg g_check_file_##tag(__FILE__)
#else
#define FX_IN(i, n) (true)
#define FX_CHECK_FILE(tag) static_assert(true, "")
#endif

}  // namespace fx

FX_CHECK_FILE(internal);

struct fx_timing_rec {
    cudaEvent_t a, b;
    double points;
    double bytes;  // algorithmic DRAM bytes of the launch where the launcher knows them, else 0
};

struct fx_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaStream_t own_stream = nullptr;
    int num_sms = 148;
    bool pdl = true;  // programmatic dependent launch (fx_ctx_set_pdl)
    double *d_partials = nullptr;  // [kMaxRedBlocks][2*kMaxSums]
    unsigned *d_counter = nullptr; // last-block ticket
    double *d_result = nullptr;    // results of standalone reductions [kMaxSums]
    double *h_result = nullptr;    // mapped page-locked mirror
    double *h_result_dev = nullptr; // its device address
    unsigned long long launches = 0;
    // per-kernel timing (fx_ctx_timing_begin / _end)
    bool timing = false;
    std::string timing_name;
    std::vector<fx_timing_rec> timing_recs;
    std::vector<cudaEvent_t> event_pool;
    size_t pool_next = 0;
    bool timing_open = false;
    // pool memory whose buffer was freed while the stream was being captured.  The graph made
    // from that capture may still address it, so the capture's owner takes the list when the
    // capture ends and frees the memory only once the graph is destroyed (fx_graph_end /
    // fx_graph_destroy, the conv-diff cycle's replay); a failed capture frees it at once, and
    // the context frees what is left when it is destroyed.
    std::vector<void *> deferred_free;
};

struct fx_buf {
    fx_ctx *ctx = nullptr;
    void *ptr = nullptr;
    size_t len = 0;
    int dtype = FX_F64;
    bool owned = true;
    bool pooled = false;  // from the device's stream-ordered pool (else plain cudaMalloc)
};

namespace fx {

int check_launch(fx_ctx *ctx, const char *what);

// NVTX range over a solve-level entry point: nsys / ncu timelines show each solve, cycle and
// training run by name.  A no-op unless a tool attaches.
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange &) = delete;
    NvtxRange &operator=(const NvtxRange &) = delete;
};
#define FX_RANGE(name) ::fx::NvtxRange fx_nvtx_range_(name)
bool capturing(cudaStream_t s);  // the stream is being captured into a graph

// Programmatic dependent launch.  Kernels of the solve path are launched with programmatic
// stream serialisation, so the next kernel's launch and block scheduling overlap the end of
// the current one.  Each such kernel first waits for the grid it depends on to complete and
// flush (griddepcontrol.wait; a no-op when the launch had no programmatic dependency), so no
// memory access moves ahead of the previous kernel, and then allows its own dependent to be
// scheduled.  The dependent can start only once every block of this grid has passed that
// point, i.e. once all of them are resident, so its waiting blocks never hold back ours.
__device__ __forceinline__ void grid_dep_enter() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

template <typename... KArgs, typename... Args>
inline void launch_pdl(fx_ctx *ctx, void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, Args... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = ctx->stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = ctx->pdl ? 1 : 0;
    (void)cudaLaunchKernelEx(&cfg, kernel, args...);  // errors surface in check_launch
}
// Timing hooks around a launch (no-ops unless fx_ctx_timing_begin named this kernel).
void timing_pre(fx_ctx *ctx, const char *what);
void timing_post(fx_ctx *ctx, double points, double bytes = 0.0);

inline size_t elem_size(int dtype) { return dtype == FX_F32 ? 4 : 8; }

// ------------------------------------------------------------------ compensated sums
// Error-free transformations (Knuth TwoSum; TwoProduct via fma, Ogita-Rump-Oishi 2005).
// Every kernel here is compiled with -fmad=false, so no expression below is contracted.

// s + c: the compensated sum.  p: a plain partial of the products added by csum_fma since the
// last csum_flush (value-initialised to 0 by CSum{s, c}).
struct CSum {
    double s, c, p;
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

// Partial form for the solvers' quadratic forms (p.Ap, r.r, r.z, ...), whose terms are mostly of
// one sign: each product goes into the thread's plain partial with one fma, and the partial is
// folded into the compensated sum once, when the reduction starts (warp_reduce); the sums
// across threads, blocks and the grid stay compensated.  A thread's partial holds its share
// of the grid (rows x cols / resident threads: about 150 terms per thread on a 4097 x 4097 F64
// grid), so the result is within n u sum|terms| for n terms per thread, against u sum|terms|
// for a Kahan sum of rounded products.  It costs one FP64 operation per term instead of
// csum_add_prod's ten, which is what keeps the level-0 passes memory-bound rather than
// FP64-bound.  Flushing every few rows inside the marching loops measured 20 us slower per
// 4097 x 4097 pass.  Dots whose terms may cancel (the BLAS-1 dot, BiCGSTAB, GMRES) keep
// csum_add_prod.
__device__ __forceinline__ void csum_fma(CSum &acc, double a, double b) { acc.p = fma(a, b, acc.p); }

// A product of two FP32 values is exact in FP64 (24 + 24 significant bits), so it needs no
// TwoProduct: it goes straight into the thread's FP64 partial (one FP64 operation per term,
// against ten for csum_add_prod), which keeps the FP32 dots memory-bound.  The partial is folded
// into the compensated sum when the reduction starts, as csum_fma's.  FP64 values keep the exact
// TwoProduct form.
template <typename T>
__device__ __forceinline__ void csum_add_prod_t(CSum &acc, T a, T b) {
    if constexpr (sizeof(T) == 4)
        acc.p = fma((double)a, (double)b, acc.p);
    else
        csum_add_prod(acc, (double)a, (double)b);
}

__device__ __forceinline__ void csum_flush(CSum &acc) {
    double s, e;
    two_sum(acc.s, acc.p, s, e);
    acc.s = s;
    acc.c += e;
    acc.p = 0.0;
}

// all accumulators of a thread that hold a partial
template <int K>
__device__ __forceinline__ void csum_flush_all(CSum (&acc)[K]) {
#pragma unroll
    for (int k = 0; k < K; k++)
        if (acc[k].p != 0.0) csum_flush(acc[k]);
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
    csum_flush_all<K>(acc);
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
    __shared__ CSum sh[32][K > 0 ? K : 1];
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

// ------------------------------------------------------------------ band-marching framework
//
// A CTA owns a band of BX = 256*CPT consecutive columns (the first band starts at column 1)
// and marches down a chunk of rows: 8 warps hold the band columns, a 9th warp loads the two
// halo columns (its lane 0 also computes column 0 in band 0).  The rows above, at and below the current one live in a
// 4-row shared-memory ring (plus one halo column on each side).  Every value a point needs
// from HBM -- the marched field row r+1 and the NA per-point "aux" arrays of row r -- is
// prefetched D rows ahead through a register FIFO, so D rows of loads are always in flight
// and no load sits on the critical path of the compute.  One __syncthreads per row.
//
// Loader : T operator()(size_t idx) const -- value of the marched field at idx (may
//          combine several arrays, e.g. r + beta*p for a fused CG update).
// Point  : static constexpr int NA;  const T *aux(int k) const;
//          void operator()(bool ring, int r, int c, size_t idx, const Nb<T>& nb, const T *a,
//                          CSum *acc)
//          -- called once for every grid point with ring = (point on the boundary ring) and
//          a[k] = aux(k)[idx].
// The kernel ends with a grid reduction of K compensated sums and a finaliser.

struct MarchGeom {
    int rows, cols;
    int nbands;
    int chunk_rows;  // multiple of D
    int nblocks;     // bands * chunks
};

// capacity: CTAs of the kernel resident on the whole GPU at once
MarchGeom march_geom(size_t rows, size_t cols, int bx, int d, int capacity);

// Functors may define `void prepare()`, called once per thread at kernel start, to read the
// solver scalars they need from device memory into registers.
template <typename X>
__device__ __forceinline__ auto fx_prepare_impl(X &x, int) -> decltype(x.prepare(), void()) {
    x.prepare();
}
template <typename X>
__device__ __forceinline__ void fx_prepare_impl(X &, long) {}
template <typename X>
__device__ __forceinline__ void fx_prepare(X &x) {
    fx_prepare_impl(x, 0);
}

template <typename T>
constexpr int band_cpt() {
    return sizeof(T) == 8 ? 1 : 2;
}

// FIFO depth in rows for S streamed arrays besides the marched field (the point's per-point
// arrays plus the loader's extra ones): deep enough to cover DRAM latency, shallow enough to
// keep two or three blocks per SM.  Even: rows are consumed in pairs.
template <int S>
constexpr int band_depth() {
    return S == 0 ? 8 : (S == 1 ? 6 : (S == 2 ? 4 : 2));
}

// Resident blocks per SM the band march's launch bound asks for (its register cap): 2, or the
// point functor's MINB for FP64.  The CG direction and update passes ask for 4 (56 registers):
// on the 4095^2 FP64 PCG solve pcg_dir went from 0.77 to 0.71 ms and the solve from 4.64 to 4.56
// ms, while the plain stencil ops lose at 4 (0.89 -> 0.85 of HBM bandwidth), so they keep 2.
template <typename P>
__host__ __device__ constexpr auto point_minb(int) -> decltype(P::MINB, int()) {
    return P::MINB;
}
template <typename P>
__host__ __device__ constexpr int point_minb(long) {
    return 2;
}
template <typename T, typename P>
__host__ __device__ constexpr int march_minb() {
    return sizeof(T) == 8 ? point_minb<P>(0) : 2;
}

template <typename T, int CPT, int D, int K, typename Loader, typename Point, typename Fin>
__global__ void __launch_bounds__(kBandThreads, march_minb<T, Point>()) k_march(MarchGeom G, Loader ld_in, Point pt_in, Fin fin,
                                                           RedArgs<K> ra, const int *skip) {
    grid_dep_enter();
    if (skip && *(volatile const int *)skip) return;
    Loader ld = ld_in;  // device-resident scalars (alpha, beta, ...) read once per kernel
    fx_prepare(ld);
    Point pt = pt_in;
    fx_prepare(pt);
    constexpr int BX = kBlock * CPT;
    constexpr int W = BX + 2;
    constexpr int NA = Point::NA;
    __shared__ T ring[8][W];
    CSum acc[K > 0 ? K : 1];
#pragma unroll
    for (int k = 0; k < (K > 0 ? K : 1); k++) acc[k] = CSum{0.0, 0.0};

    const int t = threadIdx.x;
    const int band = blockIdx.x % G.nbands;
    const int chunk = blockIdx.x / G.nbands;
    const int c0 = 1 + band * BX;
    const int r0 = chunk * G.chunk_rows;
    const int r1 = min(r0 + G.chunk_rows, G.rows);
    const int rows = G.rows, cols = G.cols;

    // column warps: slot s -> column c0 + t + s*256 (smem index 1 + t + s*256)
    // halo warp (t >= 256): lane 0 -> column c0-1 (smem 0; in band 0 that is column 0, which
    // this lane also computes), lane 1 -> column c0+BX (smem BX+1, halo only)
    const bool halo_warp = t >= kBlock;
    const int hl = t - kBlock;
    int col[CPT], sidx[CPT];
    bool valid[CPT], point[CPT], ringcol[CPT];
#pragma unroll
    for (int s = 0; s < CPT; s++) {
        if (!halo_warp) {
            col[s] = c0 + t + s * kBlock;
            sidx[s] = 1 + t + s * kBlock;
            valid[s] = col[s] < cols;
            point[s] = valid[s];
            ringcol[s] = col[s] == cols - 1;
        } else {
            col[s] = (hl == 0) ? c0 - 1 : c0 + BX;
            sidx[s] = (hl == 0) ? 0 : BX + 1;
            valid[s] = s == 0 && ((hl == 0) || (hl == 1 && c0 + BX < cols));
            point[s] = s == 0 && hl == 0 && band == 0;
            ringcol[s] = true;  // the only computed halo-warp point is column 0
        }
    }
    const bool writes_smem = !halo_warp || hl < 2;

    constexpr int NL = Loader::NL;
    T fv[D][CPT][NL];                  // raw loads of the marched field, row r+1 (D rows ahead)
    T fa[D][CPT][NA > 0 ? NA : 1];     // aux arrays, row r (D rows ahead)

    // raw values only: the loader combines them (e.g. r + beta p) when the row enters the
    // ring, so no prefetched load is waited on before its row is due.  Positions outside the
    // grid hold raw zeros, and every loader's combine maps all-zero inputs to zero; selecting
    // zero at store time instead measured 2x slower with an 8-deep FIFO.
    auto load_field = [&](int r, T (&v)[CPT][NL]) {
#pragma unroll
        for (int s = 0; s < CPT; s++) {
#pragma unroll
            for (int q = 0; q < NL; q++) v[s][q] = (T)0;
            if (r >= 0 && r < rows && valid[s] && FX_IN((size_t)r * cols + col[s], (size_t)rows * cols))
                ld.load((size_t)r * cols + col[s], v[s]);
        }
    };
    auto load_aux = [&](int r, T (&a)[CPT][NA > 0 ? NA : 1]) {
        if constexpr (NA > 0) {
#pragma unroll
            for (int s = 0; s < CPT; s++) {
#pragma unroll
                for (int k = 0; k < NA; k++) {
                    a[s][k] = (T)0;
                    if (point[s] && r < r1 && FX_IN((size_t)r * cols + col[s], (size_t)rows * cols))
                        a[s][k] = pt.aux(k)[(size_t)r * cols + col[s]];
                }
            }
        }
    };
    auto store_row = [&](int r, const T (&v)[CPT][NL]) {
        if (!writes_smem) return;
        T *row = ring[r & 7];
#pragma unroll
        for (int s = 0; s < CPT; s++)
            if ((!halo_warp || s == 0) && FX_IN(sidx[s], W)) row[sidx[s]] = ld.combine(v[s]);
    };
    auto compute_row = [&](int r, const T (&a)[CPT][NA > 0 ? NA : 1]) {
        const T *rn = ring[(r + 7) & 7];
        const T *rc = ring[r & 7];
        const T *rs = ring[(r + 1) & 7];
        const bool ringrow = (r == 0) || (r == rows - 1);
        const size_t rowoff = (size_t)r * cols;
#pragma unroll
        for (int s = 0; s < CPT; s++) {
            if (point[s] && FX_IN(sidx[s] + 1, W) && FX_IN(rowoff + col[s], (size_t)rows * cols)) {
                const int i = sidx[s];
                const bool edge = i == 0;  // column 0: no west neighbours
                Nb<T> nb;
                nb.c = rc[i];
                nb.n = rn[i];
                nb.s = rs[i];
                nb.w = edge ? (T)0 : rc[i - 1];
                nb.e = rc[i + 1];
                nb.nw = edge ? (T)0 : rn[i - 1];
                nb.ne = rn[i + 1];
                nb.sw = edge ? (T)0 : rs[i - 1];
                nb.se = rs[i + 1];
                pt(ringrow || ringcol[s], r, col[s], rowoff + col[s], nb, a[s], acc);
            }
        }
    };

    {
        T v[CPT][NL];
        load_field(r0 - 1, v);
        store_row(r0 - 1, v);  // slot (r0 - 1) & 7 (two's complement for r0 = 0)
        load_field(r0, v);
        store_row(r0, v);
    }
#pragma unroll
    for (int u = 0; u < D; u++) {
        load_field(r0 + 1 + u, fv[u]);
        load_aux(r0 + u, fa[u]);
    }

    // Two rows per step: rows r+1, r+2 of the field arrive, rows r, r+1 are computed.  The
    // 8-row ring keeps every row a later step may still read (rows r-1 .. r+2 are needed;
    // the slots being overwritten were last read three steps, and two barriers, earlier).
    for (int rb = r0; rb < r1; rb += D) {
#pragma unroll
        for (int u = 0; u < D; u += 2) {
            const int r = rb + u;
            store_row(r + 1, fv[u]);
            store_row(r + 2, fv[u + 1]);
            __syncthreads();
            if (r < r1) compute_row(r, fa[u]);
            if (r + 1 < r1) compute_row(r + 1, fa[u + 1]);
            // refill these FIFO stages: field rows r+1+D, r+2+D and aux rows r+D, r+1+D
            if (r + 1 + D <= r1) load_field(r + 1 + D, fv[u]);
            if (r + 2 + D <= r1) load_field(r + 2 + D, fv[u + 1]);
            load_aux(r + D, fa[u]);
            load_aux(r + 1 + D, fa[u + 1]);
        }
    }
    if constexpr (K > 0) grid_reduce<K>(acc, ra, fin);
}

struct NoFin {
    __device__ void operator()(const double *) const {}
};

template <typename T, int K, typename Loader, typename Point, typename Fin>
int launch_march(fx_ctx *ctx, size_t rows, size_t cols, Loader ld, Point pt, Fin fin, const int *skip,
                 const char *what) {
    constexpr int CPT = band_cpt<T>();
    constexpr int D = band_depth<Point::NA + Loader::NL - 1>();
    // resident CTAs per SM for this instantiation, cached (contexts may launch from several
    // host threads: every thread computes the same value)
    static std::atomic<int> occ_cache{0};
    int occ = occ_cache.load(std::memory_order_relaxed);
    if (!occ) {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_march<T, CPT, D, K, Loader, Point, Fin>,
                                                          kBandThreads, 0) != cudaSuccess || occ < 1)
            occ = 1;
        occ_cache.store(occ, std::memory_order_relaxed);
    }
    const MarchGeom G = march_geom(rows, cols, kBlock * CPT, D, occ * ctx->num_sms);
    if (K > 0 && G.nblocks > kMaxRedBlocks) return fail(FX_ERR_INVALID_ARGUMENT, "grid too large");
    timing_pre(ctx, what);
    launch_pdl(ctx, k_march<T, CPT, D, K, Loader, Point, Fin>, G.nblocks, kBandThreads, 0, G, ld, pt, fin,
               red_args<K>(ctx), skip);
    timing_post(ctx, (double)rows * (double)cols);
    return check_launch(ctx, what);
}

// The point functor of a march, one point per thread: the field's neighbours are loaded
// straight from memory (zeros outside the grid, as the march's ring holds), the aux arrays at
// the point, and the point is called with the same arguments the march passes.  For point
// functors that read further arrays of their own at every point (the convection-diffusion
// operator's velocity and kappa fields), whose loads the march's FIFO does not run ahead of,
// full occupancy hides the latency instead.  Diagonal neighbours are not loaded: the functors
// launched this way use the 5-point neighbourhood only.
template <typename T, int K, typename Loader, typename Point, typename Fin>
__global__ void __launch_bounds__(kBlock) k_point(size_t rows, size_t cols, Loader ld_in, Point pt_in, Fin fin,
                                                  RedArgs<K> ra, const int *skip) {
    grid_dep_enter();
    if (skip && *(volatile const int *)skip) return;
    Loader ld = ld_in;
    fx_prepare(ld);
    Point pt = pt_in;
    fx_prepare(pt);
    constexpr int NA = Point::NA;
    constexpr int NL = Loader::NL;
    CSum acc[K > 0 ? K : 1];
#pragma unroll
    for (int k = 0; k < (K > 0 ? K : 1); k++) acc[k] = CSum{0.0, 0.0};
    const size_t n = rows * cols, stride = (size_t)gridDim.x * blockDim.x;
    auto val = [&](size_t j) -> T {
        T v[NL];
#pragma unroll
        for (int q = 0; q < NL; q++) v[q] = (T)0;
        if (FX_IN(j, n)) ld.load(j, v);
        return ld.combine(v);
    };
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const size_t r = i / cols, c = i - r * cols;
        Nb<T> nb;
        nb.c = val(i);
        nb.n = r > 0 ? val(i - cols) : (T)0;
        nb.s = r + 1 < rows ? val(i + cols) : (T)0;
        nb.w = c > 0 ? val(i - 1) : (T)0;
        nb.e = c + 1 < cols ? val(i + 1) : (T)0;
        nb.nw = nb.ne = nb.sw = nb.se = (T)0;
        T a[NA > 0 ? NA : 1];
#pragma unroll
        for (int k = 0; k < NA; k++) a[k] = pt.aux(k)[i];
        const bool ring = r == 0 || c == 0 || r + 1 == rows || c + 1 == cols;
        pt(ring, (int)r, (int)c, i, nb, a, acc);
    }
    if constexpr (K > 0) grid_reduce<K>(acc, ra, fin);
}

// ------------------------------------------------------------------ flat (1-D) kernels

struct FlatGeom {
    size_t n;
    int blocks;
};

FlatGeom flat_geom(fx_ctx *ctx, size_t n);

template <int K, typename F, typename Fin>
__global__ void __launch_bounds__(kBlock) k_flat(size_t n, F f_in, Fin fin, RedArgs<K> ra,
                                                 const int *skip) {
    grid_dep_enter();
    if (skip && *(volatile const int *)skip) return;
    F f = f_in;
    fx_prepare(f);
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
    launch_pdl(ctx, k_flat<K, F, Fin>, g.blocks, kBlock, 0, n, f, fin, red_args<K>(ctx), skip);
    timing_post(ctx, (double)n);
    return check_launch(ctx, what);
}

template <typename T, int K, typename Loader, typename Point, typename Fin>
int launch_point(fx_ctx *ctx, size_t rows, size_t cols, Loader ld, Point pt, Fin fin, const int *skip,
                 const char *what) {
    FlatGeom g = flat_geom(ctx, rows * cols);
    if (g.blocks == 0) return FX_OK;
    timing_pre(ctx, what);
    launch_pdl(ctx, k_point<T, K, Loader, Point, Fin>, g.blocks, kBlock, 0, rows, cols, ld, pt, fin, red_args<K>(ctx),
               skip);
    timing_post(ctx, (double)rows * (double)cols);
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
// Scratch arrays of a library object from the device's stream-ordered pool, ordered on the
// context's stream and zero-filled (plain cudaMalloc while the stream is being captured);
// pool_free releases them in stream order (or after the graph, during a capture).
int pool_alloc(fx_ctx *ctx, size_t bytes, void **out, bool *pooled);
void pool_free(fx_ctx *ctx, void *p, bool pooled);
// n device values into mapped page-locked memory (h_dev: its device address), written by a kernel
// (no copy engine), then wait for them
int read_mapped(fx_ctx *ctx, const double *d, double *h_dev, size_t n);
int read_results(fx_ctx *ctx, int k, double *out);

// ------------------------------------------------------------------ misc helpers

int check_buf(const fx_buf *b, const char *name);
int check_same(const fx_buf *a, const fx_buf *b);  // same dtype, same length
int check_grid(const fx_grid *g);
int check_grid_len(const fx_grid *g, const fx_buf *b);

}  // namespace fx
