// fx_learned.cu -- training of the learned smoother's network (new; no reference counterpart):
// parameters, the per-sample forward and backward pass, the deterministic batch gradient, Adam,
// and the packing of the trained weights into the inference kernel's MMA operand fragments.
// The network, the loss and the sample layout are described in fx_learned.cuh.
//
// Training runs on the CUDA cores in FP32 with the network's own rounding: weights and hidden
// activations rounded to BF16 exactly as the tensor-core inference kernel rounds them, so a
// trained network computes in training what it computes when applied.  Each block takes whole
// samples; a thread owns a fixed set of parameters and accumulates their gradient over the
// block's samples in registers, and one reduction kernel adds the blocks' partials in block
// order, so a gradient is bitwise reproducible.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>

#include "fx_learned.cuh"

using namespace fx;
using namespace fx::lsm;

namespace {

constexpr int kTrThreads = 256;
constexpr int kOwn = (kNParams + kTrThreads - 1) / kTrThreads;  // parameters per thread (12)
constexpr int kMaxPartBlocks = 1024;

// shared-memory layout of the training kernel (floats)
constexpr int kSmIn = kIn * kPin * kPin;   // 1875
constexpr int kSmA1 = kC * kP1 * kP1;      // 8464: a1, later the gradient at a1's pre-activation
constexpr int kSmA2 = kC * kP2 * kP2;      // 7056: a2, later the gradient at a2's pre-activation
constexpr int kSmC = kP3 * kP3;            // 361: network output c, later dL/dc
constexpr int kSmG = kT * kT;              // 256: dL/d(Hc), then 256: the whole-error part of dL/dc
constexpr int kSmR = kNCo * kNCo;          // 81: R c, later P^T dL/d(Hc)
constexpr int kSmW = kNParams;             // parameters (weights BF16-rounded)
constexpr int kSmTrain = (kSmIn + kSmA1 + kSmA2 + 2 * kSmC + 2 * kSmG + kSmR + kSmW + 32) * 4;

// R at coarse point (I, J) of a field over the output region [-1, 17]^2 (index offset 1)
__device__ __forceinline__ float fw19(const float *f, int I, int J) {
    const int y = 2 * I + 1, x = 2 * J + 1;
    const float *c = f + y * kP3 + x;
    const float e = (c[-kP3] + c[kP3]) + (c[-1] + c[1]);
    const float d = (c[-kP3 - 1] + c[-kP3 + 1]) + (c[kP3 - 1] + c[kP3 + 1]);
    return (4.f * c[0] + (2.f * e + d)) * 0.0625f;
}

// bilinear interpolation of the coarse values Rc at loss point (py, px)
__device__ __forceinline__ float bil9(const float *Rc, int py, int px) {
    const int I = py >> 1, J = px >> 1;
    const float *r = Rc + I * kNCo + J;
    const bool oy = py & 1, ox = px & 1;
    if (!oy && !ox) return r[0];
    if (oy && !ox) return 0.5f * (r[0] + r[kNCo]);
    if (!oy && ox) return 0.5f * (r[0] + r[1]);
    return 0.25f * ((r[0] + r[kNCo]) + (r[1] + r[kNCo + 1]));
}

// One block per group of samples: forward, loss and backward of each, gradients accumulated per
// owned parameter; writes part[block][p] and part[block][kNParams] = the block's summed loss.
__global__ void __launch_bounds__(kTrThreads) k_lsm_train(const float *__restrict__ wq,
                                                          const __nv_bfloat16 *__restrict__ in_all,
                                                          const float *__restrict__ tgt_all,
                                                          const float *__restrict__ norm_all,
                                                          const int *__restrict__ idx, int count, float lambda,
                                                          float *__restrict__ part) {
    extern __shared__ __align__(16) float tsm[];
    float *S_in = tsm;
    float *S_a1 = S_in + kSmIn;
    float *S_a2 = S_a1 + kSmA1;
    float *S_c = S_a2 + kSmA2;
    float *S_gc = S_c + kSmC;
    float *S_gh = S_gc + kSmC;
    float *S_ge = S_gh + kSmG;
    float *S_r = S_ge + kSmG;
    float *S_w = S_r + kSmR;
    float *S_red = S_w + kSmW;
    const int tid = threadIdx.x;
    for (int p = tid; p < kNParams; p += kTrThreads) S_w[p] = wq[p];
    float gacc[kOwn];
#pragma unroll
    for (int j = 0; j < kOwn; j++) gacc[j] = 0.f;
    float loss_acc = 0.f;
    __syncthreads();

    for (int sidx = blockIdx.x; sidx < count; sidx += gridDim.x) {
        const int s = idx[sidx];
        const __nv_bfloat16 *in = in_all + (size_t)s * kInLen;
        const float *tgt = tgt_all + (size_t)s * kTgtLen;  // tH [256], tE [256]
        const float nrm = norm_all[2 * s] + lambda * norm_all[2 * s + 1];
        const float inv_n = nrm > 0.f ? 1.f / nrm : 0.f;
        for (int k = tid; k < kSmIn; k += kTrThreads) S_in[k] = __bfloat162float(in[k]);
        __syncthreads();
        // ---- forward
        for (int o = tid; o < kC * kP1 * kP1; o += kTrThreads) {  // a1 = bf16(relu(conv1 + b1))
            const int co = o / (kP1 * kP1), pix = o - co * (kP1 * kP1);
            const int y = pix / kP1, x = pix - y * kP1;
            float z = S_w[kOffB1 + co];
            for (int ci = 0; ci < kIn; ci++)
#pragma unroll
                for (int tap = 0; tap < 9; tap++)
                    z = fmaf(S_w[w1(co, ci, tap)], S_in[ci * kPin * kPin + (y + tap / 3) * kPin + x + tap % 3], z);
            S_a1[o] = bf16r(fmaxf(z, 0.f));
        }
        __syncthreads();
        for (int o = tid; o < kC * kP2 * kP2; o += kTrThreads) {  // a2 = bf16(relu(conv2 + b2))
            const int co = o / (kP2 * kP2), pix = o - co * (kP2 * kP2);
            const int y = pix / kP2, x = pix - y * kP2;
            float z = S_w[kOffB2 + co];
            for (int ci = 0; ci < kC; ci++) {
                const float *a = S_a1 + ci * kP1 * kP1 + y * kP1 + x;
                const float *w = S_w + w2(co, ci, 0);
#pragma unroll
                for (int tap = 0; tap < 9; tap++) z = fmaf(w[tap], a[(tap / 3) * kP1 + tap % 3], z);
            }
            S_a2[o] = bf16r(fmaxf(z, 0.f));
        }
        __syncthreads();
        for (int o = tid; o < kP3 * kP3; o += kTrThreads) {  // c = conv3 + b3
            const int y = o / kP3, x = o - y * kP3;
            float z = S_w[kOffB3];
            for (int ci = 0; ci < kC; ci++) {
                const float *a = S_a2 + ci * kP2 * kP2 + y * kP2 + x;
#pragma unroll
                for (int tap = 0; tap < 9; tap++) z = fmaf(S_w[w3(ci, tap)], a[(tap / 3) * kP2 + tap % 3], z);
            }
            S_c[o] = z;
        }
        __syncthreads();
        for (int o = tid; o < kSmR; o += kTrThreads) S_r[o] = fw19(S_c, o / kNCo, o % kNCo);
        __syncthreads();
        // ---- loss; dL/d(Hc) = -2 (tH - Hc) / n and the whole-error part -2 lambda (tE - c) / n
        float lsum = 0.f;
        for (int o = tid; o < kT * kT; o += kTrThreads) {
            const int py = o / kT, px = o - py * kT;
            const float cv = S_c[(py + 1) * kP3 + px + 1];
            const float u = tgt[o] - (cv - bil9(S_r, py, px));
            const float w = tgt[kT * kT + o] - cv;
            lsum = fmaf(u, u, lsum);
            lsum = fmaf(lambda * w, w, lsum);
            S_gh[o] = -2.f * u * inv_n;
            S_ge[o] = -2.f * lambda * w * inv_n;
        }
        // block sum of lsum: warp shuffles, then the 8 warp partials (the barrier also publishes
        // S_gh and ends the previous sample's reads of S_red)
        for (int off = 16; off > 0; off >>= 1) lsum += __shfl_down_sync(0xffffffffu, lsum, off);
        __syncthreads();
        if ((tid & 31) == 0) S_red[tid >> 5] = lsum;
        __syncthreads();
        if (tid == 0) {
            float t = 0.f;
            for (int w = 0; w < kTrThreads / 32; w++) t += S_red[w];
            loss_acc += t * inv_n;
        }
        // ---- backward through H = I - P R: dL/dc = g - R^T P^T g (g on the loss region)
        for (int o = tid; o < kSmR; o += kTrThreads) {  // (P^T g) at coarse (I, J)
            const int I = o / kNCo, J = o - I * kNCo;
            float acc = 0.f;
            for (int dy = -1; dy <= 1; dy++)
                for (int dx = -1; dx <= 1; dx++) {
                    const int py = 2 * I + dy, px = 2 * J + dx;
                    if (py < 0 || px < 0 || py >= kT || px >= kT) continue;
                    const float wgt = (dy == 0 ? 1.f : 0.5f) * (dx == 0 ? 1.f : 0.5f);
                    acc = fmaf(wgt, S_gh[py * kT + px], acc);
                }
            S_r[o] = acc;
        }
        __syncthreads();
        for (int o = tid; o < kP3 * kP3; o += kTrThreads) {  // dL/dc over [-1, 17]^2
            const int y = o / kP3, x = o - y * kP3;
            const int ly = y - 1, lx = x - 1;  // loss coordinates
            float g = (ly >= 0 && lx >= 0 && ly < kT && lx < kT) ? S_gh[ly * kT + lx] + S_ge[ly * kT + lx] : 0.f;
            for (int I = (ly - 1 + 1) >> 1; I <= (ly + 1) >> 1; I++) {
                if (I < 0 || I >= kNCo || 2 * I < ly - 1 || 2 * I > ly + 1) continue;
                for (int J = (lx - 1 + 1) >> 1; J <= (lx + 1) >> 1; J++) {
                    if (J < 0 || J >= kNCo || 2 * J < lx - 1 || 2 * J > lx + 1) continue;
                    const float wr = (2 * I == ly ? 2.f : 1.f) * (2 * J == lx ? 2.f : 1.f) * 0.0625f;
                    g = fmaf(-wr, S_r[I * kNCo + J], g);
                }
            }
            S_gc[o] = g;
        }
        __syncthreads();
        // ---- conv3: dW3, db3 (owned parameters), then dL/dz2 in place of a2
#pragma unroll
        for (int j = 0; j < kOwn; j++) {
            const int p = tid + j * kTrThreads;
            if (p < kOffW3 || p >= kNParams) continue;
            float acc = 0.f;
            if (p == kOffB3) {
                for (int o = 0; o < kP3 * kP3; o++) acc += S_gc[o];
            } else {
                const int ci = (p - kOffW3) / 9, tap = (p - kOffW3) % 9;
                const float *a = S_a2 + ci * kP2 * kP2 + (tap / 3) * kP2 + tap % 3;
                for (int y = 0; y < kP3; y++)
                    for (int x = 0; x < kP3; x++) acc = fmaf(S_gc[y * kP3 + x], a[y * kP2 + x], acc);
            }
            gacc[j] += acc;
        }
        __syncthreads();
        for (int o = tid; o < kC * kP2 * kP2; o += kTrThreads) {
            const int ci = o / (kP2 * kP2), pix = o - ci * (kP2 * kP2);
            const int y = pix / kP2, x = pix - y * kP2;
            float g = 0.f;
            if (S_a2[o] > 0.f) {
#pragma unroll
                for (int tap = 0; tap < 9; tap++) {
                    const int cy = y - tap / 3, cx = x - tap % 3;
                    if (cy < 0 || cx < 0 || cy >= kP3 || cx >= kP3) continue;
                    g = fmaf(S_w[w3(ci, tap)], S_gc[cy * kP3 + cx], g);
                }
            }
            S_a2[o] = g;  // dL/dz2 (ReLU mask from a2 itself)
        }
        __syncthreads();
        // ---- conv2: dW2, db2, then dL/dz1 in place of a1
#pragma unroll
        for (int j = 0; j < kOwn; j++) {
            const int p = tid + j * kTrThreads;
            if (p < kOffW2 || p >= kOffW3) continue;
            float acc = 0.f;
            if (p >= kOffB2) {
                const float *g = S_a2 + (p - kOffB2) * kP2 * kP2;
                for (int o = 0; o < kP2 * kP2; o++) acc += g[o];
            } else {
                const int co = (p - kOffW2) / (kC * 9), ci = ((p - kOffW2) / 9) % kC, tap = (p - kOffW2) % 9;
                const float *g = S_a2 + co * kP2 * kP2;
                const float *a = S_a1 + ci * kP1 * kP1 + (tap / 3) * kP1 + tap % 3;
                for (int y = 0; y < kP2; y++)
                    for (int x = 0; x < kP2; x++) acc = fmaf(g[y * kP2 + x], a[y * kP1 + x], acc);
            }
            gacc[j] += acc;
        }
        __syncthreads();
        for (int o = tid; o < kC * kP1 * kP1; o += kTrThreads) {
            const int ci = o / (kP1 * kP1), pix = o - ci * (kP1 * kP1);
            const int y = pix / kP1, x = pix - y * kP1;
            float g = 0.f;
            if (S_a1[o] > 0.f) {
                for (int co = 0; co < kC; co++) {
                    const float *gz = S_a2 + co * kP2 * kP2;
                    const float *w = S_w + w2(co, ci, 0);
#pragma unroll
                    for (int tap = 0; tap < 9; tap++) {
                        const int zy = y - tap / 3, zx = x - tap % 3;
                        if (zy < 0 || zx < 0 || zy >= kP2 || zx >= kP2) continue;
                        g = fmaf(w[tap], gz[zy * kP2 + zx], g);
                    }
                }
            }
            S_a1[o] = g;  // dL/dz1
        }
        __syncthreads();
        // ---- conv1: dW1, db1
#pragma unroll
        for (int j = 0; j < kOwn; j++) {
            const int p = tid + j * kTrThreads;
            if (p >= kOffW2) continue;
            float acc = 0.f;
            if (p >= kOffB1) {
                const float *g = S_a1 + (p - kOffB1) * kP1 * kP1;
                for (int o = 0; o < kP1 * kP1; o++) acc += g[o];
            } else {
                const int co = p / (kIn * 9), ci = (p / 9) % kIn, tap = p % 9;
                const float *g = S_a1 + co * kP1 * kP1;
                const float *a = S_in + ci * kPin * kPin + (tap / 3) * kPin + tap % 3;
                for (int y = 0; y < kP1; y++)
                    for (int x = 0; x < kP1; x++) acc = fmaf(g[y * kP1 + x], a[y * kPin + x], acc);
            }
            gacc[j] += acc;
        }
        __syncthreads();
    }
    float *out = part + (size_t)blockIdx.x * (kNParams + 1);
#pragma unroll
    for (int j = 0; j < kOwn; j++) {
        const int p = tid + j * kTrThreads;
        if (p < kNParams) out[p] = gacc[j];
    }
    if (tid == 0) out[kNParams] = loss_acc;
}

// grad[p] = sum over blocks of part[b][p], in block order (p = kNParams: the loss)
__global__ void k_lsm_reduce(const float *__restrict__ part, int nblocks, float *__restrict__ grad) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p > kNParams) return;
    float s = 0.f;
    for (int b = 0; b < nblocks; b++) s += part[(size_t)b * (kNParams + 1) + p];
    grad[p] = s;
}

// Adam (Kingma & Ba 2015) on the mean gradient grad / batch, with bias correction.
__global__ void k_lsm_adam(float *__restrict__ w, float *__restrict__ m, float *__restrict__ v,
                           const float *__restrict__ grad, float inv_batch, float lr, float b1, float b2, float eps,
                           float c1, float c2) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kNParams) return;
    const float g = grad[p] * inv_batch;
    const float mm = b1 * m[p] + (1.f - b1) * g;
    const float vv = b2 * v[p] + (1.f - b2) * g * g;
    m[p] = mm;
    v[p] = vv;
    w[p] -= lr * (mm / c1) / (sqrtf(vv / c2) + eps);
}

__device__ __forceinline__ bool is_bias(int p) {
    return (p >= kOffB1 && p < kOffW2) || (p >= kOffB2 && p < kOffW3) || p == kOffB3;
}

// wq = the parameters as the network uses them; frag = the MMA B-operand fragments (see
// fx_learned.cuh).  Fragment element (k, n) of lane l: k = 2 (l % 4) + {0, 1} (+ 8 for the second
// register), n = l / 4.
__global__ void k_lsm_pack(const float *__restrict__ w, float *__restrict__ wq, uint32_t *__restrict__ frag) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < kNParams) wq[t] = is_bias(t) ? w[t] : __bfloat162float(__float2bfloat16_rn(w[t]));
    if (t >= kFragWords) return;
    auto r = [&](int p) { return w[p]; };
    float lo = 0.f, hi = 0.f;
    if (t < kFrag1) {  // conv1: [ks][nh][lane][reg], k = tap * 4 + ch (ch 3 and k >= 36 are zero)
        const int reg = t & 1, lane = (t >> 1) & 31, nh = (t >> 6) & 1, ks = t >> 7;
        const int k = ks * 16 + reg * 8 + (lane & 3) * 2, co = nh * 8 + (lane >> 2);
        auto b1 = [&](int kk) {
            const int tap = kk >> 2, ch = kk & 3;
            return (tap < 9 && ch < kIn) ? r(w1(co, ch, tap)) : 0.f;
        };
        lo = b1(k);
        hi = b1(k + 1);
    } else if (t < kFrag1 + kFrag2) {  // conv2: [tap][nh][lane][reg], k = ci
        const int u = t - kFrag1;
        const int reg = u & 1, lane = (u >> 1) & 31, nh = (u >> 6) & 1, tap = u >> 7;
        const int ci = reg * 8 + (lane & 3) * 2, co = nh * 8 + (lane >> 2);
        lo = r(w2(co, ci, tap));
        hi = r(w2(co, ci + 1, tap));
    } else {  // conv3: [tap][lane][reg], k = ci, only n = 0 nonzero
        const int u = t - kFrag1 - kFrag2;
        const int reg = u & 1, lane = (u >> 1) & 31, tap = u >> 6;
        const int ci = reg * 8 + (lane & 3) * 2;
        if ((lane >> 2) == 0) {
            lo = r(w3(ci, tap));
            hi = r(w3(ci + 1, tap));
        }
    }
    frag[t] = pack_bf16x2(lo, hi);
}

}  // namespace

int fx_lsm::pack() {
    const int n = kFragWords > kNParams ? kFragWords : kNParams;
    k_lsm_pack<<<(n + 255) / 256, 256, 0, ctx->stream>>>(d_w, d_wq, d_frag);
    return check_launch(ctx, "lsm_pack");
}

namespace fx {

// The summed gradient and loss of the samples h_idx[0..count) -> m->d_grad (asynchronous).
int lsm_batch_grad(fx_lsm *m, const fx_lsm_data *d, const int *h_idx, size_t count, float lambda) {
    fx_ctx *ctx = m->ctx;
    if (count == 0) return fail(FX_ERR_INVALID_ARGUMENT, "empty batch");
    for (size_t i = 0; i < count; i++)
        if (h_idx[i] < 0 || (size_t)h_idx[i] >= d->count)
            return fail(FX_ERR_INVALID_ARGUMENT, "sample index out of range");
    if (count > m->idx_cap) {
        if (m->d_idx) cudaFreeAsync(m->d_idx, ctx->stream);
        m->d_idx = nullptr;
        FX_CUDA(cudaMallocAsync(&m->d_idx, count * sizeof(int), ctx->stream));
        m->idx_cap = count;
    }
    FX_CUDA(cudaMemcpyAsync(m->d_idx, h_idx, count * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
    const int blocks = (int)std::min<size_t>(count, (size_t)m->part_blocks);
    timing_pre(ctx, "lsm_train");
    k_lsm_train<<<blocks, kTrThreads, kSmTrain, ctx->stream>>>(m->d_wq, d->d_in, d->d_tgt, d->d_norm, m->d_idx,
                                                               (int)count, lambda, m->d_part);
    timing_post(ctx, (double)count);
    FX_TRY(check_launch(ctx, "lsm_train"));
    k_lsm_reduce<<<(kNParams + 1 + 255) / 256, 256, 0, ctx->stream>>>(m->d_part, blocks, m->d_grad);
    return check_launch(ctx, "lsm_reduce");
}

}  // namespace fx

extern "C" {

int fx_lsm_param_count(size_t *n) {
    if (!n) return fail(FX_ERR_INVALID_ARGUMENT, "null out");
    *n = kNParams;
    return FX_OK;
}

int fx_lsm_destroy(fx_lsm *m) {
    if (!m) return FX_OK;
    cudaSetDevice(m->ctx->device);
    cudaStreamSynchronize(m->ctx->stream);
    for (void *p : {(void *)m->d_w, (void *)m->d_wq, (void *)m->d_frag, (void *)m->d_m, (void *)m->d_v,
                    (void *)m->d_part, (void *)m->d_grad, (void *)m->d_idx})
        if (p) cudaFree(p);
    delete m;
    return FX_OK;
}

int fx_lsm_create(fx_ctx *ctx, unsigned long long seed, fx_lsm **out) {
    if (!ctx || !out) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    static bool attr_set[64] = {};
    if (ctx->device >= 0 && ctx->device < 64 && !attr_set[ctx->device]) {
        FX_CUDA(cudaFuncSetAttribute(k_lsm_train, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmTrain));
        attr_set[ctx->device] = true;
    }
    fx_lsm *m = new fx_lsm();
    m->ctx = ctx;
    int occ = 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_lsm_train, kTrThreads, kSmTrain) != cudaSuccess || occ < 1)
        occ = 1;
    m->part_blocks = std::min(kMaxPartBlocks, occ * ctx->num_sms);
    const size_t P = kNParams;
    if (cudaMalloc(&m->d_w, P * 4) != cudaSuccess || cudaMalloc(&m->d_wq, P * 4) != cudaSuccess ||
        cudaMalloc(&m->d_frag, kFragWords * 4) != cudaSuccess || cudaMalloc(&m->d_m, P * 4) != cudaSuccess ||
        cudaMalloc(&m->d_v, P * 4) != cudaSuccess || cudaMalloc(&m->d_grad, (P + 1) * 4) != cudaSuccess ||
        cudaMalloc(&m->d_part, (size_t)m->part_blocks * (P + 1) * 4) != cudaSuccess) {
        (void)cudaGetLastError();
        fx_lsm_destroy(m);
        return fail(FX_ERR_BACKEND, "learned smoother: allocation failed");
    }
    // He-normal initialisation of W1 and W2 (std sqrt(2 / fan_in)), zero biases, and a zero last
    // layer, so that the untrained smoother is the weighted-Jacobi step
    std::vector<float> h(P, 0.f);
    std::mt19937_64 rng(seed);
    std::normal_distribution<float> nd(0.f, 1.f);
    const float s1 = std::sqrt(2.f / (kIn * 9)), s2 = std::sqrt(2.f / (kC * 9));
    for (int p = kOffW1; p < kOffB1; p++) h[p] = s1 * nd(rng);
    for (int p = kOffW2; p < kOffB2; p++) h[p] = s2 * nd(rng);
    int st = FX_OK;
    if (cudaMemcpyAsync(m->d_w, h.data(), P * 4, cudaMemcpyHostToDevice, ctx->stream) != cudaSuccess ||
        cudaMemsetAsync(m->d_m, 0, P * 4, ctx->stream) != cudaSuccess ||
        cudaMemsetAsync(m->d_v, 0, P * 4, ctx->stream) != cudaSuccess ||
        cudaStreamSynchronize(ctx->stream) != cudaSuccess)
        st = fail(FX_ERR_BACKEND, "learned smoother: initialisation failed");
    if (st == FX_OK) st = m->pack();
    if (st != FX_OK) {
        fx_lsm_destroy(m);
        return st;
    }
    *out = m;
    return FX_OK;
}

int fx_lsm_get_params(fx_lsm *m, float *dst, size_t n) {
    if (!m || !dst) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    if (n != (size_t)kNParams) return fail(FX_ERR_DIMENSION_MISMATCH, "parameter count is " + std::to_string(kNParams));
    FX_CUDA(cudaMemcpyAsync(dst, m->d_w, n * 4, cudaMemcpyDeviceToHost, m->ctx->stream));
    FX_CUDA(cudaStreamSynchronize(m->ctx->stream));
    return FX_OK;
}

int fx_lsm_set_params(fx_lsm *m, const float *src, size_t n) {
    if (!m || !src) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    if (n != (size_t)kNParams) return fail(FX_ERR_DIMENSION_MISMATCH, "parameter count is " + std::to_string(kNParams));
    FX_CUDA(cudaMemcpyAsync(m->d_w, src, n * 4, cudaMemcpyHostToDevice, m->ctx->stream));
    FX_CUDA(cudaMemsetAsync(m->d_m, 0, n * 4, m->ctx->stream));
    FX_CUDA(cudaMemsetAsync(m->d_v, 0, n * 4, m->ctx->stream));
    m->adam_t = 0;
    FX_TRY(m->pack());
    FX_CUDA(cudaStreamSynchronize(m->ctx->stream));
    return FX_OK;
}

int fx_lsm_data_create(fx_ctx *ctx, size_t capacity, fx_lsm_data **out) {
    if (!ctx || !out) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    if (capacity == 0 || capacity > ((size_t)1 << 24)) return fail(FX_ERR_INVALID_ARGUMENT, "capacity out of range");
    fx_lsm_data *d = new fx_lsm_data();
    d->ctx = ctx;
    d->cap = capacity;
    if (cudaMalloc(&d->d_in, capacity * kInLen * sizeof(__nv_bfloat16)) != cudaSuccess ||
        cudaMalloc(&d->d_tgt, capacity * kTgtLen * 4) != cudaSuccess ||
        cudaMalloc(&d->d_norm, capacity * 2 * 4) != cudaSuccess) {
        (void)cudaGetLastError();
        if (d->d_in) cudaFree(d->d_in);
        if (d->d_tgt) cudaFree(d->d_tgt);
        if (d->d_norm) cudaFree(d->d_norm);
        delete d;
        return fail(FX_ERR_BACKEND, "learned smoother samples: allocation failed");
    }
    *out = d;
    return FX_OK;
}

int fx_lsm_data_destroy(fx_lsm_data *d) {
    if (!d) return FX_OK;
    cudaSetDevice(d->ctx->device);
    cudaStreamSynchronize(d->ctx->stream);
    cudaFree(d->d_in);
    cudaFree(d->d_tgt);
    cudaFree(d->d_norm);
    delete d;
    return FX_OK;
}

int fx_lsm_data_size(const fx_lsm_data *d, size_t *n) {
    if (!d || !n) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    *n = d->count;
    return FX_OK;
}

int fx_lsm_data_get(const fx_lsm_data *d, size_t index, float *inputs, float *target, float *norm) {
    if (!d || !inputs || !target || !norm) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    if (index >= d->count) return fail(FX_ERR_INVALID_ARGUMENT, "sample index out of range");
    std::vector<__nv_bfloat16> b(kInLen);
    cudaStream_t s = d->ctx->stream;
    FX_CUDA(cudaMemcpyAsync(b.data(), d->d_in + index * kInLen, kInLen * 2, cudaMemcpyDeviceToHost, s));
    FX_CUDA(cudaMemcpyAsync(target, d->d_tgt + index * kTgtLen, kTgtLen * 4, cudaMemcpyDeviceToHost, s));
    FX_CUDA(cudaMemcpyAsync(norm, d->d_norm + 2 * index, 8, cudaMemcpyDeviceToHost, s));
    FX_CUDA(cudaStreamSynchronize(s));
    for (int k = 0; k < kInLen; k++) {  // BF16 -> FP32 is exact: the high half of the word
        uint16_t u;
        std::memcpy(&u, &b[k], 2);
        const uint32_t w = (uint32_t)u << 16;
        std::memcpy(&inputs[k], &w, 4);
    }
    return FX_OK;
}

int fx_lsm_loss_grad(fx_lsm *m, const fx_lsm_data *d, const size_t *indices, size_t count, double lambda,
                     double *loss, float *grad) {
    if (!m || !d || !indices || !loss) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    if (d->ctx->device != m->ctx->device) return fail(FX_ERR_INVALID_ARGUMENT, "samples on another device");
    std::vector<int> idx(count);
    for (size_t i = 0; i < count; i++) {
        if (indices[i] >= d->count) return fail(FX_ERR_INVALID_ARGUMENT, "sample index out of range");
        idx[i] = (int)indices[i];
    }
    if (!(lambda >= 0.0)) return fail(FX_ERR_INVALID_ARGUMENT, "lambda must be non-negative");
    FX_TRY(lsm_batch_grad(m, d, idx.data(), count, (float)lambda));
    std::vector<float> g(kNParams + 1);
    FX_CUDA(cudaMemcpyAsync(g.data(), m->d_grad, (kNParams + 1) * 4, cudaMemcpyDeviceToHost, m->ctx->stream));
    FX_CUDA(cudaStreamSynchronize(m->ctx->stream));
    *loss = (double)g[kNParams] / (double)count;
    if (grad)
        for (int p = 0; p < kNParams; p++) grad[p] = g[p] / (float)count;
    return FX_OK;
}

int fx_lsm_train(fx_lsm *m, const fx_lsm_data *d, size_t epochs, size_t batch, double lr, double lambda,
                 unsigned long long seed, double *epoch_loss) {
    FX_RANGE("fx_lsm_train");
    if (!m || !d) return fail(FX_ERR_INVALID_ARGUMENT, "null argument");
    if (!(lambda >= 0.0)) return fail(FX_ERR_INVALID_ARGUMENT, "lambda must be non-negative");
    if (d->count == 0 || batch == 0) return fail(FX_ERR_INVALID_ARGUMENT, "no samples or zero batch");
    if (!(lr > 0.0)) return fail(FX_ERR_INVALID_ARGUMENT, "learning rate must be positive");
    fx_ctx *ctx = m->ctx;
    batch = std::min(batch, d->count);
    const size_t steps = d->count / batch;
    std::vector<int> order(d->count);
    for (size_t i = 0; i < d->count; i++) order[i] = (int)i;
    std::mt19937_64 rng(seed);
    // the per-step losses stay on the device until the end of each epoch
    float *d_losses = nullptr;
    FX_CUDA(cudaMallocAsync(&d_losses, steps * sizeof(float), ctx->stream));
    std::vector<float> h_losses(steps);
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    int st = FX_OK;
    for (size_t e = 0; e < epochs && st == FX_OK; e++) {
        std::shuffle(order.begin(), order.end(), rng);
        for (size_t k = 0; k < steps && st == FX_OK; k++) {
            st = lsm_batch_grad(m, d, order.data() + k * batch, batch, (float)lambda);
            if (st != FX_OK) break;
            m->adam_t++;
            const float c1 = 1.f - (float)std::pow((double)b1, (double)m->adam_t);
            const float c2 = 1.f - (float)std::pow((double)b2, (double)m->adam_t);
            k_lsm_adam<<<(kNParams + 255) / 256, 256, 0, ctx->stream>>>(m->d_w, m->d_m, m->d_v, m->d_grad,
                                                                        1.f / (float)batch, (float)lr, b1, b2, eps, c1, c2);
            st = check_launch(ctx, "lsm_adam");
            if (st == FX_OK) st = m->pack();
            if (st == FX_OK && cudaMemcpyAsync(d_losses + k, m->d_grad + kNParams, 4, cudaMemcpyDeviceToDevice,
                                               ctx->stream) != cudaSuccess)
                st = fail(FX_ERR_BACKEND, "learned smoother: loss copy failed");
        }
        if (st == FX_OK && epoch_loss) {
            if (cudaMemcpyAsync(h_losses.data(), d_losses, steps * 4, cudaMemcpyDeviceToHost, ctx->stream) !=
                    cudaSuccess ||
                cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
                st = fail(FX_ERR_BACKEND, "learned smoother: loss read failed");
                break;
            }
            double s = 0.0;
            for (float v : h_losses) s += v;
            epoch_loss[e] = s / (double)(steps * batch);  // mean per-sample loss over the epoch (before each step)
        }
    }
    cudaFreeAsync(d_losses, ctx->stream);
    if (st == FX_OK) FX_CUDA(cudaStreamSynchronize(ctx->stream));
    return st;
}

}  // extern "C"
