// fx_context.cu -- context, buffers, host<->device transfers and the shared host helpers.
//
// The context plays the role of the reference's process-wide HIP backend singleton
// (crates/backend-hip/src/backend.rs:61-79, :103-264): one device, one stream, the
// reduction scratch.  Buffers play HipBuffer (crates/backend-hip/src/buffer.rs:16-123).
#include <cstring>
#include <mutex>

#include "fx_internal.cuh"

FX_CHECK_FILE(context);

namespace fx {

static thread_local std::string g_err;

void set_error(const std::string &msg) { g_err = msg; }

int fail(int code, const std::string &msg) {
    g_err = msg;
    return code;
}

int check_launch(fx_ctx *ctx, const char *what) {
    ctx->launches++;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(FX_ERR_BACKEND, std::string(what) + ": " + cudaGetErrorString(e));
    return FX_OK;
}

// Buffers come from one stream-ordered memory pool per device, owned by the library and never
// trimmed (its release threshold is the maximum), so that creating and dropping fields and
// hierarchies neither synchronises the device nor maps memory again: cudaFree would wait for
// every stream of the device, which serialises contexts that run independent problems side by
// side.  An allocation is ordered on the context's stream; fx_ctx_set_stream waits for the old
// stream before switching, so buffers made earlier are ready on the new one (and refuses to switch
// while the old stream is being captured, when that wait cannot be made).
static cudaMemPool_t device_pool(int device) {
    static std::mutex mu;
    static cudaMemPool_t pools[64] = {};
    if (device < 0 || device >= 64) return nullptr;
    std::lock_guard<std::mutex> lock(mu);
    if (!pools[device]) {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        cudaMemPool_t p = nullptr;
        if (cudaMemPoolCreate(&p, &props) != cudaSuccess) {
            (void)cudaGetLastError();
            return nullptr;
        }
        unsigned long long keep = ~0ull;
        cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
        pools[device] = p;
    }
    return pools[device];
}

int pool_alloc(fx_ctx *ctx, size_t bytes, void **out, bool *pooled) {
    *out = nullptr;
    *pooled = false;
    if (bytes == 0) bytes = 16;
    cudaMemPool_t pool = capturing(ctx->stream) ? nullptr : device_pool(ctx->device);
    const cudaError_t e = pool ? cudaMallocFromPoolAsync(out, bytes, pool, ctx->stream) : cudaMalloc(out, bytes);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        *out = nullptr;
        return fail(FX_ERR_BACKEND, std::string("device allocation failed: ") + cudaGetErrorString(e));
    }
    *pooled = pool != nullptr;
    if (cudaMemsetAsync(*out, 0, bytes, ctx->stream) != cudaSuccess) {
        (void)cudaGetLastError();
        pool_free(ctx, *out, *pooled);
        *out = nullptr;
        return fail(FX_ERR_BACKEND, "memset failed");
    }
    return FX_OK;
}

void pool_free(fx_ctx *ctx, void *p, bool pooled) {
    if (!p) return;
    if (!pooled) {
        cudaStreamSynchronize(ctx->stream);
        cudaFree(p);
    } else if (capturing(ctx->stream)) {
        ctx->deferred_free.push_back(p);
    } else {
        cudaFreeAsync(p, ctx->stream);
    }
}

bool capturing(cudaStream_t s) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) != cudaSuccess) {
        (void)cudaGetLastError();
        return false;
    }
    return cs != cudaStreamCaptureStatusNone;
}

void timing_pre(fx_ctx *ctx, const char *what) {
    if (!ctx->timing || ctx->timing_name != what) return;
    if (ctx->pool_next + 2 > ctx->event_pool.size()) {
        for (int i = 0; i < 64; i++) {
            cudaEvent_t e;
            if (cudaEventCreate(&e) != cudaSuccess) return;
            ctx->event_pool.push_back(e);
        }
    }
    fx_timing_rec r;
    r.a = ctx->event_pool[ctx->pool_next++];
    r.b = ctx->event_pool[ctx->pool_next++];
    r.points = 0;
    cudaEventRecord(r.a, ctx->stream);
    ctx->timing_recs.push_back(r);
    ctx->timing_open = true;
}

void timing_post(fx_ctx *ctx, double points, double bytes) {
    if (!ctx->timing_open) return;
    fx_timing_rec &r = ctx->timing_recs.back();
    cudaEventRecord(r.b, ctx->stream);
    r.points = points;
    r.bytes = bytes;
    ctx->timing_open = false;
}

int check_buf(const fx_buf *b, const char *name) {
    if (!b) return fail(FX_ERR_INVALID_ARGUMENT, std::string("null buffer: ") + name);
    return FX_OK;
}

int check_same(const fx_buf *a, const fx_buf *b) {
    if (a->len != b->len) {
        return fail(FX_ERR_DIMENSION_MISMATCH, "dimension mismatch: expected " +
                                                   std::to_string(a->len) + ", got " +
                                                   std::to_string(b->len));
    }
    if (a->dtype != b->dtype) return fail(FX_ERR_INVALID_ARGUMENT, "dtype mismatch between buffers");
    return FX_OK;
}

int check_grid(const fx_grid *g) {
    if (!g) return fail(FX_ERR_INVALID_ARGUMENT, "null grid");
    if (g->rows < 3 || g->cols < 3)
        return fail(FX_ERR_INVALID_GRID, "invalid grid: minimum 3x3, got " + std::to_string(g->rows) +
                                             "x" + std::to_string(g->cols));
    if (!(g->dx > 0.0) || !(g->dy > 0.0) || !std::isfinite(g->dx) || !std::isfinite(g->dy))
        return fail(FX_ERR_INVALID_GRID, "invalid grid: spacing must be finite and positive");
    if (g->rows > (size_t)0x7fffffff || g->cols > (size_t)0x7fffffff ||
        g->rows * g->cols > ((size_t)1 << 40))
        return fail(FX_ERR_INVALID_GRID, "invalid grid: too large");
    return FX_OK;
}

int check_grid_len(const fx_grid *g, const fx_buf *b) {
    const size_t n = g->rows * g->cols;
    if (b->len != n)
        return fail(FX_ERR_DIMENSION_MISMATCH, "dimension mismatch: expected " + std::to_string(n) +
                                                   ", got " + std::to_string(b->len));
    return FX_OK;
}

int make_stencil(const fx_stencil *s, StencilP *P) {
    std::memset(P, 0, sizeof(*P));
    if (!s || s->n < 1 || !s->dr || !s->dc || !s->w)
        return fail(FX_ERR_INVALID_STENCIL, "invalid stencil: stencil must have at least one entry");
    const int n = s->n;
    if (n == 5 || n == 9) {  // ops.rs:898-916, :953-975: weights by offset, others ignored
        P->mode = n;
        for (int k = 0; k < n; k++) {
            const int r = s->dr[k], c = s->dc[k];
            const double w = s->w[k];
            if (r == 0 && c == 0) P->c = w;
            else if (r == -1 && c == 0) P->n = w;
            else if (r == 1 && c == 0) P->s = w;
            else if (r == 0 && c == -1) P->w = w;
            else if (r == 0 && c == 1) P->e = w;
            else if (n == 9 && r == -1 && c == -1) P->nw = w;
            else if (n == 9 && r == -1 && c == 1) P->ne = w;
            else if (n == 9 && r == 1 && c == -1) P->sw = w;
            else if (n == 9 && r == 1 && c == 1) P->se = w;
        }
        return FX_OK;
    }
    if (n > kMaxGeneric)
        return fail(FX_ERR_INVALID_STENCIL, "invalid stencil: more than 27 entries");
    for (int k = 0; k < n; k++) {
        if (s->dr[k] < -1 || s->dr[k] > 1 || s->dc[k] < -1 || s->dc[k] > 1)
            return fail(FX_ERR_INVALID_STENCIL, "invalid stencil: offsets beyond radius 1");
        P->gi[k] = (signed char)((s->dr[k] + 1) * 3 + (s->dc[k] + 1));
        P->gw[k] = s->w[k];
    }
    P->mode = 0;
    P->ne_ = n;
    return FX_OK;
}

int make_bc(const fx_boundaries *bc, double dx, double dy, BcP *P, bool reject_periodic) {
    std::memset(P, 0, sizeof(*P));
    P->dx = dx;
    P->dy = dy;
    if (!bc) {
        for (int i = 0; i < 4; i++) P->kind[i] = FX_BC_DIRICHLET;
        return FX_OK;
    }
    for (int i = 0; i < 4; i++) {
        const int k = bc->side[i].kind;
        if (k < 0 || k > 3) return fail(FX_ERR_INVALID_ARGUMENT, "unknown boundary kind");
        if (k == FX_BC_PERIODIC && reject_periodic)  // ops.rs:9-23
            return fail(FX_ERR_UNSUPPORTED, "backend error: periodic boundaries are not yet implemented");
        P->kind[i] = k;
        P->a[i] = bc->side[i].a;
        P->b[i] = bc->side[i].b;
        P->g[i] = bc->side[i].g;
    }
    return FX_OK;
}

MarchGeom march_geom(size_t rows, size_t cols, int bx, int d, int capacity) {
    MarchGeom G;
    G.rows = (int)rows;
    G.cols = (int)cols;
    G.nbands = (int)((cols - 1 + bx - 1) / bx);
    if (G.nbands < 1) G.nbands = 1;
    // Split the rows into chunks so that bands x chunks fills whole waves of resident CTAs
    // (one work item per CTA, equal work per item).  A chunk is at least one FIFO depth d
    // long: on small grids, where a launch is bound by the rows each CTA marches in
    // sequence, short chunks cut that latency at the cost of a few recomputed halo rows.
    const long R = (long)rows, B = G.nbands;
    long best_chunks = 1;
    double best_eff = -1.0;
    for (int w = 1; w <= 8; w++) {
        long chunks = (long)w * capacity / B;
        if (chunks < 1) chunks = 1;
        long cr = (R + chunks - 1) / chunks;
        if (cr < d) cr = d;
        cr = ((cr + d - 1) / d) * d;
        chunks = (R + cr - 1) / cr;
        const long nb = chunks * B;
        const long waves = (nb + capacity - 1) / capacity;
        const double eff = (double)nb / (double)(waves * capacity);
        if (eff > best_eff + 0.02) {
            best_eff = eff;
            best_chunks = chunks;
        }
    }
    long cr = (R + best_chunks - 1) / best_chunks;
    if (cr < d) cr = d;
    cr = ((cr + d - 1) / d) * d;
    G.chunk_rows = (int)cr;
    G.nblocks = (int)(((R + cr - 1) / cr) * B);
    return G;
}

FlatGeom flat_geom(fx_ctx *ctx, size_t n) {
    FlatGeom g;
    g.n = n;
    size_t b = (n + kBlock - 1) / kBlock;
    const size_t cap = (size_t)ctx->num_sms * 8;
    if (b > cap) b = cap;
    g.blocks = (int)b;
    return g;
}

// Registry of the checked build: the readers of the units' status words and the names of the
// files holding checks (by hash).  Filled by static initialisers when the library loads; empty in
// the default build.
// test hook: one index check, no memory access (fx_test_check_index)
__global__ void k_check_index(long long index, long long extent) {
    if (threadIdx.x == 0) (void)FX_IN(index, extent);
}

struct CheckRegistry {
    std::mutex mu;
    std::vector<CheckReader> readers;
    std::vector<std::pair<unsigned, std::string>> files;
};
static CheckRegistry &check_registry() {
    static CheckRegistry r;
    return r;
}

void check_register_unit(CheckReader reader) {
    CheckRegistry &r = check_registry();
    std::lock_guard<std::mutex> lk(r.mu);
    r.readers.push_back(reader);
}

void check_register_file(unsigned hash, const char *name) {
    CheckRegistry &r = check_registry();
    std::lock_guard<std::mutex> lk(r.mu);
    for (auto &f : r.files)
        if (f.first == hash) return;
    const char *base = std::strrchr(name, '/');
    r.files.emplace_back(hash, base ? base + 1 : name);
}

// standalone reductions' results to mapped page-locked memory, written by the device (no copy
// engine: a small cudaMemcpyAsync would queue behind any large transfer on the same engine)
__global__ void k_results_out(const double *d, double *h, int k) {
    if ((int)threadIdx.x < k) h[threadIdx.x] = d[threadIdx.x];
}

__global__ void k_copy_out_f64(const double *d, double *h, int n) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) h[i] = d[i];
}

int read_mapped(fx_ctx *ctx, const double *d, double *h_dev, size_t n) {
    if (n > (1u << 20)) return fail(FX_ERR_INVALID_ARGUMENT, "read_mapped: at most 2^20 values");
    k_copy_out_f64<<<1, 256, 0, ctx->stream>>>(d, h_dev, (int)n);
    FX_TRY(check_launch(ctx, "copy_out"));
    FX_CUDA(cudaStreamSynchronize(ctx->stream));
    return FX_OK;
}

int read_results(fx_ctx *ctx, int k, double *out) {
    k_results_out<<<1, 32, 0, ctx->stream>>>(ctx->d_result, ctx->h_result_dev, k);
    FX_TRY(check_launch(ctx, "results_out"));
    FX_CUDA(cudaStreamSynchronize(ctx->stream));
    for (int i = 0; i < k; i++) out[i] = ctx->h_result[i];
    return FX_OK;
}

}  // namespace fx

using namespace fx;

extern "C" {

const char *fx_last_error(void) { return g_err.c_str(); }

int fx_version(void) { return 10000; }

const char *fx_backend_name(void) { return "cuda"; }

int fx_device_count(int *count) {
    if (!count) return fail(FX_ERR_INVALID_ARGUMENT, "null out");
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *count = 0;
        return fail(FX_ERR_NO_DEVICE, std::string("no CUDA device: ") + cudaGetErrorString(e));
    }
    *count = n;
    return FX_OK;
}

int fx_ctx_create(int device, fx_ctx **out) {
    if (!out) return fail(FX_ERR_INVALID_ARGUMENT, "null out");
    *out = nullptr;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        cudaGetLastError();
        return fail(FX_ERR_NO_DEVICE, "no CUDA device available");
    }
    if (device < 0 || device >= n) return fail(FX_ERR_INVALID_ARGUMENT, "device ordinal out of range");
    FX_CUDA(cudaSetDevice(device));
    fx_ctx *c = new fx_ctx();
    c->device = device;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) == cudaSuccess) c->num_sms = prop.multiProcessorCount;
    if (cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&c->d_partials, sizeof(double) * 2 * kMaxSums * (size_t)kMaxRedBlocks) != cudaSuccess ||
        cudaMalloc(&c->d_counter, sizeof(unsigned) * 4) != cudaSuccess ||
        cudaMalloc(&c->d_result, sizeof(double) * 8) != cudaSuccess ||
        cudaHostAlloc(&c->h_result, sizeof(double) * 8, cudaHostAllocMapped) != cudaSuccess ||
        cudaHostGetDevicePointer((void **)&c->h_result_dev, c->h_result, 0) != cudaSuccess ||
        cudaMemset(c->d_counter, 0, sizeof(unsigned) * 4) != cudaSuccess) {
        std::string m = cudaGetErrorString(cudaGetLastError());
        fx_ctx_destroy(c);
        return fail(FX_ERR_BACKEND, "context allocation failed: " + m);
    }
    c->stream = c->own_stream;
    *out = c;
    return FX_OK;
}

int fx_ctx_destroy(fx_ctx *c) {
    if (!c) return FX_OK;
    cudaSetDevice(c->device);
    for (void *p : c->deferred_free) cudaFree(p);  // waits for the device, as it should here
    if (c->own_stream) cudaStreamSynchronize(c->own_stream);
    if (c->d_partials) cudaFree(c->d_partials);
    if (c->d_counter) cudaFree(c->d_counter);
    if (c->d_result) cudaFree(c->d_result);
    if (c->h_result) cudaFreeHost(c->h_result);
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    for (auto e : c->event_pool) cudaEventDestroy(e);
    delete c;
    return FX_OK;
}

int fx_ctx_synchronize(fx_ctx *c) {
    if (!c) return fail(FX_ERR_INVALID_ARGUMENT, "null context");
    FX_CUDA(cudaStreamSynchronize(c->stream));
    return FX_OK;
}

// ---- graph capture (HipGraph, backend-hip/src/graph.rs:14-108)

struct fx_graph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int device = 0;
    // pool memory of buffers freed while this graph was being recorded: the graph's kernels
    // still address it, so it returns to the pool only when the graph is destroyed
    std::vector<void *> frees;
};

int fx_graph_begin(fx_ctx *c) {
    if (!c) return fail(FX_ERR_INVALID_ARGUMENT, "null context");
    if (!c->stream) return fail(FX_ERR_INVALID_ARGUMENT, "graph capture needs a non-default stream");
    FX_CUDA(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeRelaxed));
    return FX_OK;
}

int fx_graph_end(fx_ctx *c, fx_graph **out) {
    if (!c || !out) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(c->stream, &g);
    std::vector<void *> frees;
    frees.swap(c->deferred_free);
    auto release_now = [&] {  // no graph refers to the memory: back to the pool in stream order
        for (void *p : frees) cudaFreeAsync(p, c->stream);
    };
    if (e != cudaSuccess || !g) {
        if (g) cudaGraphDestroy(g);
        (void)cudaGetLastError();
        release_now();
        return fail(FX_ERR_BACKEND, std::string("graph capture failed: ") +
                                        (e != cudaSuccess ? cudaGetErrorString(e) : "empty capture"));
    }
    cudaGraphExec_t x = nullptr;
    e = cudaGraphInstantiate(&x, g, 0);
    if (e != cudaSuccess) {
        cudaGraphDestroy(g);
        (void)cudaGetLastError();
        release_now();
        return fail(FX_ERR_BACKEND, std::string("graph instantiation failed: ") + cudaGetErrorString(e));
    }
    fx_graph *G = new fx_graph();
    G->graph = g;
    G->exec = x;
    G->device = c->device;
    G->frees.swap(frees);
    *out = G;
    return FX_OK;
}

int fx_graph_launch(fx_ctx *c, const fx_graph *g) {
    if (!c || !g) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    FX_CUDA(cudaGraphLaunch(g->exec, c->stream));
    return FX_OK;
}

int fx_graph_destroy(fx_graph *g) {
    if (!g) return FX_OK;
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    if (!g->frees.empty()) {
        // a launch of the graph may still be running on some stream: cudaFree waits for the device
        cudaSetDevice(g->device);
        for (void *p : g->frees) cudaFree(p);
    }
    delete g;
    return FX_OK;
}

int fx_ctx_set_stream(fx_ctx *c, void *stream) {
    if (!c) return fail(FX_ERR_INVALID_ARGUMENT, "null context");
    cudaStream_t next = stream ? (cudaStream_t)stream : c->own_stream;
    if (next != c->stream) {
        // Work on the old stream (pool allocations and their zero fill included) must be complete
        // before the new stream may touch it.  A stream being captured cannot be waited for, and
        // moving away from it would also end the capture on the wrong stream: refused.
        if (capturing(c->stream))
            return fail(FX_ERR_INVALID_ARGUMENT,
                        "cannot switch the context's stream while it is being captured into a graph");
        FX_CUDA(cudaStreamSynchronize(c->stream));
    }
    c->stream = next;
    return FX_OK;
}

int fx_ctx_set_pdl(fx_ctx *c, int enabled) {
    if (!c) return fail(FX_ERR_INVALID_ARGUMENT, "null context");
    c->pdl = enabled != 0;
    return FX_OK;
}

void *fx_ctx_get_stream(fx_ctx *c) { return c ? (void *)c->stream : nullptr; }

unsigned long long fx_ctx_launch_count(fx_ctx *c) { return c ? c->launches : 0ull; }

int fx_ctx_timing_begin(fx_ctx *c, const char *kernel) {
    if (!c || !kernel) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    c->timing = true;
    c->timing_name = kernel;
    c->timing_recs.clear();
    c->pool_next = 0;
    c->timing_open = false;
    return FX_OK;
}

int fx_ctx_timing_end_records(fx_ctx *c, double *ms, double *points, double *bytes, size_t max, size_t *count) {
    if (!c || !ms || !points || !count) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    FX_CUDA(cudaStreamSynchronize(c->stream));
    size_t k = 0;
    for (auto &r : c->timing_recs) {
        if (k >= max) break;
        float t = 0.f;
        FX_CUDA(cudaEventElapsedTime(&t, r.a, r.b));
        ms[k] = t;
        points[k] = r.points;
        if (bytes) bytes[k] = r.bytes;
        k++;
    }
    *count = k;
    c->timing = false;
    c->timing_recs.clear();
    c->pool_next = 0;
    return FX_OK;
}

int fx_ctx_timing_end(fx_ctx *c, double *total_ms, unsigned long long *launches, double *total_points) {
    if (!c || !total_ms || !launches || !total_points) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    FX_CUDA(cudaStreamSynchronize(c->stream));
    double ms = 0.0, pts = 0.0;
    for (auto &r : c->timing_recs) {
        float t = 0.f;
        FX_CUDA(cudaEventElapsedTime(&t, r.a, r.b));
        ms += t;
        pts += r.points;
    }
    *total_ms = ms;
    *launches = c->timing_recs.size();
    *total_points = pts;
    c->timing = false;
    c->timing_recs.clear();
    c->pool_next = 0;
    return FX_OK;
}

// test hook: the next g_fail_allocs buffer allocations fail (fx_test_fail_allocations)
static std::atomic<int> g_fail_allocs{0};

int fx_test_fail_allocations(int count) {
    g_fail_allocs.store(count < 0 ? 0 : count);
    return FX_OK;
}

int fx_alloc(fx_ctx *ctx, size_t len, int dtype, fx_buf **out) {
    if (!ctx || !out) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    if (dtype != FX_F32 && dtype != FX_F64) return fail(FX_ERR_INVALID_ARGUMENT, "unknown dtype");
    *out = nullptr;
    for (int k = g_fail_allocs.load(); k > 0; k = g_fail_allocs.load())
        if (g_fail_allocs.compare_exchange_weak(k, k - 1))
            return fail(FX_ERR_BACKEND, "backend error: allocation failed (test hook)");
    fx_buf *b = new fx_buf();
    b->ctx = ctx;
    b->len = len;
    b->dtype = dtype;
    const size_t bytes = len * elem_size(dtype);
    if (bytes) {
        // While the stream is being captured a pool allocation would become a node of the
        // graph; a plain allocation is made outside it instead.
        cudaMemPool_t pool = capturing(ctx->stream) ? nullptr : device_pool(ctx->device);
        cudaError_t e = pool ? cudaMallocFromPoolAsync(&b->ptr, bytes, pool, ctx->stream) : cudaMalloc(&b->ptr, bytes);
        if (e != cudaSuccess) {
            (void)cudaGetLastError();
            delete b;
            return fail(FX_ERR_BACKEND, std::string("backend error: allocation failed: ") + cudaGetErrorString(e));
        }
        b->pooled = pool != nullptr;
        if (cudaMemsetAsync(b->ptr, 0, bytes, ctx->stream) != cudaSuccess) {
            if (b->pooled)
                cudaFreeAsync(b->ptr, ctx->stream);
            else
                cudaFree(b->ptr);
            delete b;
            return fail(FX_ERR_BACKEND, "backend error: memset failed");
        }
    }
    *out = b;
    return FX_OK;
}

int fx_wrap(fx_ctx *ctx, void *ptr, size_t len, int dtype, fx_buf **out) {
    if (!ctx || !out || (!ptr && len)) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    if (dtype != FX_F32 && dtype != FX_F64) return fail(FX_ERR_INVALID_ARGUMENT, "unknown dtype");
    fx_buf *b = new fx_buf();
    b->ctx = ctx;
    b->ptr = ptr;
    b->len = len;
    b->dtype = dtype;
    b->owned = false;
    *out = b;
    return FX_OK;
}

int fx_free(fx_buf *b) {
    if (!b) return FX_OK;
    if (b->owned && b->ptr) {
        if (!b->pooled) {
            cudaStreamSynchronize(b->ctx->stream);
            cudaFree(b->ptr);
        } else if (capturing(b->ctx->stream)) {
            b->ctx->deferred_free.push_back(b->ptr);
        } else {
            cudaFreeAsync(b->ptr, b->ctx->stream);  // after the work queued on it so far
        }
    }
    delete b;
    return FX_OK;
}

size_t fx_buf_len(const fx_buf *b) { return b ? b->len : 0; }
int fx_buf_dtype(const fx_buf *b) { return b ? b->dtype : -1; }
void *fx_buf_device_ptr(const fx_buf *b) { return b ? b->ptr : nullptr; }

}  // extern "C"

// Conversion kernels for uploads / downloads across dtypes.
namespace {
__global__ void k_f64_to_f32(const double *__restrict__ s, float *__restrict__ d, size_t n) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        d[i] = (float)s[i];
}
__global__ void k_f32_to_f64(const float *__restrict__ s, double *__restrict__ d, size_t n) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        d[i] = (double)s[i];
}

int write_host(fx_ctx *ctx, fx_buf *b, const void *src, int src_dtype, size_t len) {
    if (!ctx || !b || (!src && len)) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    if (len != b->len)
        return fail(FX_ERR_DIMENSION_MISMATCH, "dimension mismatch: expected " + std::to_string(b->len) +
                                                   ", got " + std::to_string(len));
    if (!len) return FX_OK;
    if (src_dtype == b->dtype) {
        FX_CUDA(cudaMemcpyAsync(b->ptr, src, len * elem_size(b->dtype), cudaMemcpyHostToDevice, ctx->stream));
        FX_CUDA(cudaStreamSynchronize(ctx->stream));
        return FX_OK;
    }
    void *tmp = nullptr;
    cudaMemPool_t pool = device_pool(ctx->device);
    FX_CUDA(pool ? cudaMallocFromPoolAsync(&tmp, len * elem_size(src_dtype), pool, ctx->stream)
                 : cudaMallocAsync(&tmp, len * elem_size(src_dtype), ctx->stream));
    FX_CUDA(cudaMemcpyAsync(tmp, src, len * elem_size(src_dtype), cudaMemcpyHostToDevice, ctx->stream));
    FlatGeom g = flat_geom(ctx, len);
    if (src_dtype == FX_F64)
        k_f64_to_f32<<<g.blocks, kBlock, 0, ctx->stream>>>((const double *)tmp, (float *)b->ptr, len);
    else
        k_f32_to_f64<<<g.blocks, kBlock, 0, ctx->stream>>>((const float *)tmp, (double *)b->ptr, len);
    int st = check_launch(ctx, "convert");
    cudaFreeAsync(tmp, ctx->stream);
    FX_CUDA(cudaStreamSynchronize(ctx->stream));
    return st;
}

int read_host(fx_ctx *ctx, const fx_buf *b, void *dst, int dst_dtype, size_t len) {
    if (!ctx || !b || (!dst && len)) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    if (len != b->len)
        return fail(FX_ERR_DIMENSION_MISMATCH, "destination length mismatch: expected " +
                                                   std::to_string(b->len) + ", got " + std::to_string(len));
    if (!len) return FX_OK;
    if (dst_dtype == b->dtype) {
        FX_CUDA(cudaMemcpyAsync(dst, b->ptr, len * elem_size(b->dtype), cudaMemcpyDeviceToHost, ctx->stream));
        FX_CUDA(cudaStreamSynchronize(ctx->stream));
        return FX_OK;
    }
    void *tmp = nullptr;
    cudaMemPool_t pool = device_pool(ctx->device);
    FX_CUDA(pool ? cudaMallocFromPoolAsync(&tmp, len * elem_size(dst_dtype), pool, ctx->stream)
                 : cudaMallocAsync(&tmp, len * elem_size(dst_dtype), ctx->stream));
    FlatGeom g = flat_geom(ctx, len);
    if (dst_dtype == FX_F32)
        k_f64_to_f32<<<g.blocks, kBlock, 0, ctx->stream>>>((const double *)b->ptr, (float *)tmp, len);
    else
        k_f32_to_f64<<<g.blocks, kBlock, 0, ctx->stream>>>((const float *)b->ptr, (double *)tmp, len);
    int st = check_launch(ctx, "convert");
    FX_CUDA(cudaMemcpyAsync(dst, tmp, len * elem_size(dst_dtype), cudaMemcpyDeviceToHost, ctx->stream));
    cudaFreeAsync(tmp, ctx->stream);
    FX_CUDA(cudaStreamSynchronize(ctx->stream));
    return st;
}
}  // namespace

extern "C" {

int fx_upload_f64(fx_ctx *ctx, const double *data, size_t len, fx_buf **out) {
    FX_TRY(fx_alloc(ctx, len, FX_F64, out));
    int st = write_host(ctx, *out, data, FX_F64, len);
    if (st) {
        fx_free(*out);
        *out = nullptr;
    }
    return st;
}

int fx_upload_f32(fx_ctx *ctx, const float *data, size_t len, fx_buf **out) {
    FX_TRY(fx_alloc(ctx, len, FX_F32, out));
    int st = write_host(ctx, *out, data, FX_F32, len);
    if (st) {
        fx_free(*out);
        *out = nullptr;
    }
    return st;
}

int fx_write_f64(fx_ctx *ctx, fx_buf *b, const double *src, size_t len) {
    return write_host(ctx, b, src, FX_F64, len);
}

int fx_write_f32(fx_ctx *ctx, fx_buf *b, const float *src, size_t len) {
    return write_host(ctx, b, src, FX_F32, len);
}

int fx_copy_to_host_f64(fx_ctx *ctx, const fx_buf *b, double *dst, size_t len) {
    return read_host(ctx, b, dst, FX_F64, len);
}

int fx_copy_to_host_f32(fx_ctx *ctx, const fx_buf *b, float *dst, size_t len) {
    return read_host(ctx, b, dst, FX_F32, len);
}

// Asynchronous copies between an F64 buffer and page-locked host memory, enqueued on `stream`
// (NULL: the context's stream) without waiting; the caller orders them with events.
int fx_write_f64_async(fx_ctx *ctx, fx_buf *b, const double *src, size_t len, void *stream) {
    if (!ctx || !b || (!src && len)) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    if (b->dtype != FX_F64) return fail(FX_ERR_INVALID_ARGUMENT, "asynchronous copies take F64 buffers");
    if (len != b->len)
        return fail(FX_ERR_DIMENSION_MISMATCH, "dimension mismatch: expected " + std::to_string(b->len) +
                                                   ", got " + std::to_string(len));
    if (!len) return FX_OK;
    FX_CUDA(cudaMemcpyAsync(b->ptr, src, len * sizeof(double), cudaMemcpyHostToDevice,
                            stream ? (cudaStream_t)stream : ctx->stream));
    return FX_OK;
}

int fx_copy_to_host_f64_async(fx_ctx *ctx, const fx_buf *b, double *dst, size_t len, void *stream) {
    if (!ctx || !b || (!dst && len)) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    if (b->dtype != FX_F64) return fail(FX_ERR_INVALID_ARGUMENT, "asynchronous copies take F64 buffers");
    if (len != b->len)
        return fail(FX_ERR_DIMENSION_MISMATCH, "destination length mismatch: expected " + std::to_string(b->len) +
                                                   ", got " + std::to_string(len));
    if (!len) return FX_OK;
    FX_CUDA(cudaMemcpyAsync(dst, b->ptr, len * sizeof(double), cudaMemcpyDeviceToHost,
                            stream ? (cudaStream_t)stream : ctx->stream));
    return FX_OK;
}

int fx_test_check_index(fx_ctx *ctx, long long index, long long extent) {
    if (!ctx) return fail(FX_ERR_INVALID_ARGUMENT, "null context");
    k_check_index<<<1, 32, 0, ctx->stream>>>(index, extent);
    return check_launch(ctx, "test_check_index");
}

int fx_checked_build(void) {
#ifdef FX_CHECKED
    return 1;
#else
    return 0;
#endif
}

int fx_checked_status(fx_ctx *ctx, size_t *count, char *file, size_t file_cap, int *line, long long *index,
                      long long *extent) {
    if (!ctx || !count || !line || !index || !extent) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    *count = 0;
    *line = 0;
    *index = 0;
    *extent = 0;
    if (file && file_cap) file[0] = '\0';
    int prev = 0;
    FX_CUDA(cudaGetDevice(&prev));
    struct Restore {  // the caller's current device is left as it was
        int d;
        ~Restore() { cudaSetDevice(d); }
    } restore{prev};
    FX_CUDA(cudaSetDevice(ctx->device));
    FX_CUDA(cudaDeviceSynchronize());
    CheckRegistry &r = check_registry();
    std::lock_guard<std::mutex> lk(r.mu);
    for (CheckReader rd : r.readers) {
        CheckWord w{};
        if (rd(&w)) return fail(FX_ERR_BACKEND, "reading a checked-build status word failed");
        if (!w.code) continue;
        if ((*count)++ == 0) {
            *line = w.line;
            *index = w.index;
            *extent = w.extent;
            if (file && file_cap) {
                std::string name = "?";
                for (auto &f : r.files)
                    if (f.first == w.file) name = f.second;
                std::strncpy(file, name.c_str(), file_cap - 1);
                file[file_cap - 1] = '\0';
            }
        }
    }
    return FX_OK;
}

}  // extern "C"
