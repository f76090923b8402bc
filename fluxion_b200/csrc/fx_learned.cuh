// fx_learned.cuh -- the learned smoother: a 3 -> 16 -> 16 -> 1 convolutional network of 3 x 3
// filters (ReLU after the first two) that corrects a weighted-Jacobi step of the
// convection-diffusion multigrid (new; the reference smooths with weighted Jacobi only,
// crates/runtime/src/multigrid.rs:245-306).
//
// One learned smoothing step on a level with operator A, diagonal d, iterate x and rhs b:
//   q = (b - A x) / d                      (q = 0 on the ring)
//   s = sqrt(mean of q^2 over the interior)
//   c = N(q / s, vx / (dx d), vy / (dy d)) (the network, per point, zero padding outside the grid)
//   x <- x + omega q + s c                 (interior points)
// With the last layer's weights and bias zero, c = 0 and the step is the Jacobi sweep.
//
// Arithmetic: weights and activations are BF16 (inputs rounded to BF16, each hidden activation
// rounded to BF16 after bias and ReLU), every accumulation is FP32, the biases are FP32.  The
// update runs in the level's precision.
//
// Training target (one sample = a 16 x 16 patch of a plain V-cycle iterate's residual and
// error, with the network's input halo): the error after the step, e' = e - omega q - s c,
// measured by its part that the coarse grid cannot represent, H e' with H = I - P R (R full
// weighting onto the even points, P bilinear interpolation back), plus lambda times the whole
// error (a smoother must not add error that is smooth, which H alone would not see).  Per sample
//   loss = (|| H e' ||^2 + lambda || e' ||^2) / (|| H e ||^2 + lambda || e ||^2)
//        = (|| tH - H c ||^2 + lambda || tE - c ||^2) / (nH + lambda nE),
//   tH = (H e - omega H q) / s, tE = (e - omega q) / s on the patch, nH = ||H e||^2 / s^2,
//   nE = ||e||^2 / s^2,
// so the untrained network (c = 0) scores the Jacobi step's loss.
#pragma once

#include <cuda_bf16.h>

#include "fx_internal.cuh"

FX_CHECK_FILE(learned_h);

namespace fx {
namespace lsm {

constexpr int kC = 16;  // hidden channels
constexpr int kIn = 3;  // input channels: q / s, vx / (dx d), vy / (dy d)
// flat parameter vector: W1 [16][3][9], b1 [16], W2 [16][16][9], b2 [16], W3 [1][16][9], b3 [1];
// W[co][ci][tap] with tap = 3 ky + kx weighting input (y + ky - 1, x + kx - 1) (cross-correlation)
constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + kC * kIn * 9;
constexpr int kOffW2 = kOffB1 + kC;
constexpr int kOffB2 = kOffW2 + kC * kC * 9;
constexpr int kOffW3 = kOffB2 + kC;
constexpr int kOffB3 = kOffW3 + kC * 9;
constexpr int kNParams = kOffB3 + 1;  // 2913

// training patch geometry (regions relative to the loss patch's first point)
constexpr int kT = 16;         // loss region [0, 16)^2; its first point has even grid coordinates
constexpr int kPin = kT + 9;   // 25: network input on [-4, 20]^2
constexpr int kP1 = kT + 7;    // 23: first hidden layer on [-3, 19]^2
constexpr int kP2 = kT + 5;    // 21: second hidden layer on [-2, 18]^2
constexpr int kP3 = kT + 3;    // 19: network output on [-1, 17]^2 (what H needs)
constexpr int kNCo = kT / 2 + 1;  // 9 coarse points per side, at loss coordinates 0, 2, .., 16
constexpr int kInLen = kIn * kPin * kPin;  // 1875 BF16 values per sample
constexpr int kTgtLen = 2 * kT * kT;       // tH then tE, 256 each

// packed BF16 operand fragments of the three convolutions for mma.m16n8k16 (32-bit words):
// conv1 [kstep 3][n-half 2][lane 32][2], conv2 [tap 9][n-half 2][lane 32][2], conv3 [tap 9][lane 32][2]
constexpr int kFrag1 = 3 * 2 * 32 * 2;
constexpr int kFrag2 = 9 * 2 * 32 * 2;
constexpr int kFrag3 = 9 * 32 * 2;
constexpr int kFragWords = kFrag1 + kFrag2 + kFrag3;

// inference tile: 28 x 28 updated points per block; the layers are evaluated in 16-point row
// segments (the MMA's M), so the first hidden layer covers 32 x 32 points, the second 30 x 32, the
// output 28 x 32 (the extra columns are computed and dropped)
constexpr int kTile = 28;
constexpr int kBufW = 34;  // row pitch (points) of the shared-memory buffers
constexpr int kInRows = kTile + 6, kA1Rows = kTile + 4, kA2Rows = kTile + 2;
constexpr int kSmemA1 = kA1Rows * kBufW * 32;           // 16 BF16 channels per point
constexpr int kSmemA2 = kA2Rows * kBufW * 32;           // aliased with the input (8 B per point)
constexpr int kSmemIn = kInRows * kBufW * 8;
constexpr int kSmemApply = kSmemA1 + (kSmemA2 > kSmemIn ? kSmemA2 : kSmemIn);

__host__ __device__ constexpr int w1(int co, int ci, int tap) { return kOffW1 + (co * kIn + ci) * 9 + tap; }
__host__ __device__ constexpr int w2(int co, int ci, int tap) { return kOffW2 + (co * kC + ci) * 9 + tap; }
__host__ __device__ constexpr int w3(int ci, int tap) { return kOffW3 + ci * 9 + tap; }

__device__ __forceinline__ float bf16r(float v) { return __bfloat162float(__float2bfloat16_rn(v)); }

// round-to-nearest-even BF16 pair, lower k in the low half (the MMA operand order)
__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
    const uint32_t l = (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(lo));
    const uint32_t h = (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(hi));
    return l | (h << 16);
}

// Network input channels of one grid point from its q, vx, vy and diagonal d (d = 0: velocity
// channels 0).
template <typename T>
__device__ __forceinline__ void input_channels(T q, T vx, T vy, T d, double inv_s, double inv_dx, double inv_dy,
                                               float &c0, float &c1, float &c2) {
    c0 = (float)((double)q * inv_s);
    if (d != (T)0) {
        const double id = 1.0 / (double)d;
        c1 = (float)((double)vx * inv_dx * id);
        c2 = (float)((double)vy * inv_dy * id);
    } else {
        c1 = c2 = 0.f;
    }
}

// ---------------------------------------------------------------- inference (tensor cores)

__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ void ldsm_x4(uint32_t (&a)[4], uint32_t saddr) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];"
                 : "=r"(a[0]), "=r"(a[1]), "=r"(a[2]), "=r"(a[3])
                 : "r"(saddr));
}

// byte offset of (point p, 8-channel half h) in a 16-channel buffer: the two 16-byte halves of a
// point are swapped when bit 2 of its index is set, so that the eight rows of every ldmatrix
// phase (eight consecutive points) fall in distinct bank groups
__device__ __forceinline__ uint32_t hoff(int p, int h) { return (uint32_t)(p * 32 + 16 * (h ^ ((p >> 2) & 1))); }

// One learned step's network evaluation and update on a 28 x 28 tile (see the file comment).
// Op provides diag(i), vxv(i), vyv(i) of the level's operator.  frag: the packed fragments;
// bias: the FP32 parameter vector (biases read at their offsets).  scale[0] = s, scale[1] = 1/s
// (0 when s = 0).  x is updated in place: each point reads and writes only its own x.
template <typename T, typename Op>
__global__ void __launch_bounds__(256) k_lsm_apply(Op A, const uint32_t *__restrict__ frag,
                                                   const float *__restrict__ bias, const T *__restrict__ q, T *x,
                                                   const double *__restrict__ scale, T omega, int rows, int cols,
                                                   double inv_dx, double inv_dy, const int *skip) {
    grid_dep_enter();
    if (skip && *(volatile const int *)skip) return;
    extern __shared__ __align__(128) unsigned char lsm_smem[];
    unsigned char *A1 = lsm_smem;             // first hidden layer, 32 x 34 points x 16 ch
    unsigned char *XB = lsm_smem + kSmemA1;   // input (34 x 34 x 4 ch), then second hidden layer
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 2, tig = lane & 3;
    const int r0 = blockIdx.y * kTile, c0 = blockIdx.x * kTile;
    const double s = scale[0], inv_s = scale[1];

    // ---- input: 34 x 34 points from (r0 - 3, c0 - 3), zero outside the grid.  A thread's points
    // are loaded first (all of them in flight at once), then turned into channels.
    {
        constexpr int kIt = (kInRows * kBufW + 255) / 256;
        T qv[kIt], xv[kIt], yv[kIt], dv[kIt];
#pragma unroll
        for (int j = 0; j < kIt; j++) {
            const int k = tid + j * 256;
            const int iy = k / kBufW, ix = k - iy * kBufW;
            const int gr = r0 - 3 + iy, gc = c0 - 3 + ix;
            qv[j] = xv[j] = yv[j] = dv[j] = (T)0;
            if (k < kInRows * kBufW && gr >= 0 && gr < rows && gc >= 0 && gc < cols &&
                FX_IN((long long)gr * cols + gc, (long long)rows * cols)) {
                const size_t i = (size_t)gr * cols + gc;
                qv[j] = q[i];
                xv[j] = A.vxv(i);
                yv[j] = A.vyv(i);
                dv[j] = A.diag(i);
            }
        }
#pragma unroll
        for (int j = 0; j < kIt; j++) {
            const int k = tid + j * 256;
            if (k >= kInRows * kBufW) break;
            float ch0, ch1, ch2;  // zero for points outside the grid (all inputs zero there)
            input_channels<T>(qv[j], xv[j], yv[j], dv[j], inv_s, inv_dx, inv_dy, ch0, ch1, ch2);
            uint2 v;
            v.x = pack_bf16x2(ch0, ch1);
            v.y = pack_bf16x2(ch2, 0.f);
            *reinterpret_cast<uint2 *>(XB + (size_t)k * 8) = v;
        }
    }
    __syncthreads();

    const uint32_t sA1 = (uint32_t)__cvta_generic_to_shared(A1);
    const uint32_t sXB = (uint32_t)__cvta_generic_to_shared(XB);
    const uint32_t *Xw = reinterpret_cast<const uint32_t *>(XB);

    // ---- conv1 (K = 9 taps x 4 channels, padded to 48) -> A1 over 32 x 32 points from (r0 - 2, c0 - 2)
    {
        uint32_t bw[3][2][2];
#pragma unroll
        for (int ks = 0; ks < 3; ks++)
#pragma unroll
            for (int nh = 0; nh < 2; nh++) {
                const uint2 v = *reinterpret_cast<const uint2 *>(frag + ((ks * 2 + nh) * 32 + lane) * 2);
                bw[ks][nh][0] = v.x;
                bw[ks][nh][1] = v.y;
            }
        float bl[2][2];
#pragma unroll
        for (int nh = 0; nh < 2; nh++)
#pragma unroll
            for (int j = 0; j < 2; j++) bl[nh][j] = bias[kOffB1 + nh * 8 + tig * 2 + j];
        for (int t = warp; t < kA1Rows * 2; t += 8) {
            const int ay = t >> 1, ax0 = (t & 1) * 16;
            float acc[2][4] = {};
#pragma unroll
            for (int ks = 0; ks < 3; ks++) {
                uint32_t a[4];
#pragma unroll
                for (int hk = 0; hk < 2; hk++) {  // k = ks*16 + hk*8 + tig*2
                    const int k = ks * 16 + hk * 8 + tig * 2;
                    const int tap = (k >> 2) < 9 ? (k >> 2) : 8;  // k >= 36: zero weights, any finite input
                    const int ky = tap / 3, kx = tap - ky * 3;
                    const int p0 = (ay + ky) * kBufW + ax0 + kx;
                    a[hk * 2 + 0] = Xw[(p0 + g) * 2 + ((k & 3) >> 1)];
                    a[hk * 2 + 1] = Xw[(p0 + g + 8) * 2 + ((k & 3) >> 1)];
                }
#pragma unroll
                for (int nh = 0; nh < 2; nh++) mma_bf16(acc[nh], a, bw[ks][nh][0], bw[ks][nh][1]);
            }
            // epilogue: bias, ReLU, BF16, zero outside the grid
#pragma unroll
            for (int hm = 0; hm < 2; hm++) {
                const int m = g + hm * 8;
                const int gr = r0 - 2 + ay, gc = c0 - 2 + ax0 + m;
                const bool in = gr >= 0 && gr < rows && gc >= 0 && gc < cols;
                const int p = ay * kBufW + ax0 + m;
#pragma unroll
                for (int nh = 0; nh < 2; nh++) {
                    const float v0 = in ? fmaxf(acc[nh][hm * 2 + 0] + bl[nh][0], 0.f) : 0.f;
                    const float v1 = in ? fmaxf(acc[nh][hm * 2 + 1] + bl[nh][1], 0.f) : 0.f;
                    *reinterpret_cast<uint32_t *>(A1 + hoff(p, nh) + 4 * tig) = pack_bf16x2(v0, v1);
                }
            }
        }
    }
    __syncthreads();

    // ---- conv2 (16 -> 16, per tap K = 16) -> A2 (over the input) on 30 x 32 points from (r0 - 1, c0 - 1)
    {
        uint32_t bw[9][2][2];
        const uint32_t *f2 = frag + kFrag1;
#pragma unroll
        for (int tap = 0; tap < 9; tap++)
#pragma unroll
            for (int nh = 0; nh < 2; nh++) {
                const uint2 v = *reinterpret_cast<const uint2 *>(f2 + ((tap * 2 + nh) * 32 + lane) * 2);
                bw[tap][nh][0] = v.x;
                bw[tap][nh][1] = v.y;
            }
        float bl[2][2];
#pragma unroll
        for (int nh = 0; nh < 2; nh++)
#pragma unroll
            for (int j = 0; j < 2; j++) bl[nh][j] = bias[kOffB2 + nh * 8 + tig * 2 + j];
        const int lm = lane & 15, lh = lane >> 4;
        for (int t = warp; t < kA2Rows * 2; t += 8) {
            const int y2 = t >> 1, x0 = (t & 1) * 16;
            float acc[2][4] = {};
#pragma unroll
            for (int tap = 0; tap < 9; tap++) {
                const int ky = tap / 3, kx = tap - ky * 3;
                const int p = (y2 + ky) * kBufW + x0 + lm + kx;
                uint32_t a[4];
                ldsm_x4(a, sA1 + hoff(p, lh));
#pragma unroll
                for (int nh = 0; nh < 2; nh++) mma_bf16(acc[nh], a, bw[tap][nh][0], bw[tap][nh][1]);
            }
            // epilogue (the input under XB is dead: conv1 finished before the barrier above)
#pragma unroll
            for (int hm = 0; hm < 2; hm++) {
                const int m = g + hm * 8;
                const int gr = r0 - 1 + y2, gc = c0 - 1 + x0 + m;
                const bool in = gr >= 0 && gr < rows && gc >= 0 && gc < cols;
                const int p = y2 * kBufW + x0 + m;
#pragma unroll
                for (int nh = 0; nh < 2; nh++) {
                    const float v0 = in ? fmaxf(acc[nh][hm * 2 + 0] + bl[nh][0], 0.f) : 0.f;
                    const float v1 = in ? fmaxf(acc[nh][hm * 2 + 1] + bl[nh][1], 0.f) : 0.f;
                    *reinterpret_cast<uint32_t *>(XB + hoff(p, nh) + 4 * tig) = pack_bf16x2(v0, v1);
                }
            }
        }
    }
    __syncthreads();

    // ---- conv3 (16 -> 1, N padded to 8) and the update on 28 x 28 points from (r0, c0)
    {
        uint32_t bw[9][2];
        const uint32_t *f3 = frag + kFrag1 + kFrag2;
#pragma unroll
        for (int tap = 0; tap < 9; tap++) {
            const uint2 v = *reinterpret_cast<const uint2 *>(f3 + (tap * 32 + lane) * 2);
            bw[tap][0] = v.x;
            bw[tap][1] = v.y;
        }
        const float b3 = bias[kOffB3];
        const int lm = lane & 15, lh = lane >> 4;
        for (int t = warp; t < kTile * 2; t += 8) {
            const int oy = t >> 1, ox0 = (t & 1) * 16;
            float acc[4] = {};
#pragma unroll
            for (int tap = 0; tap < 9; tap++) {
                const int ky = tap / 3, kx = tap - ky * 3;
                const int p = (oy + ky) * kBufW + ox0 + lm + kx;
                uint32_t a[4];
                ldsm_x4(a, sXB + hoff(p, lh));
                mma_bf16(acc, a, bw[tap][0], bw[tap][1]);
            }
            if (tig == 0) {  // output channel 0 of points g and g + 8
#pragma unroll
                for (int hm = 0; hm < 2; hm++) {
                    const int ox = ox0 + g + hm * 8;
                    const int gr = r0 + oy, gc = c0 + ox;
                    if (ox >= kTile || gr <= 0 || gc <= 0 || gr >= rows - 1 || gc >= cols - 1) continue;
                    const size_t i = (size_t)gr * cols + gc;
                    if (!FX_IN(i, (long long)rows * cols)) continue;
                    const double c = (double)(acc[hm * 2] + b3);
                    x[i] = (T)((double)fx_fma(omega, q[i], x[i]) + s * c);
                }
            }
        }
    }
}

}  // namespace lsm
}  // namespace fx

// The network and its optimiser state (fx_lsm_*), and a set of training samples.
struct fx_lsm {
    fx_ctx *ctx = nullptr;
    float *d_w = nullptr;      // FP32 master parameters [kNParams]
    float *d_wq = nullptr;     // parameters as the network uses them: weights rounded to BF16, biases FP32
    uint32_t *d_frag = nullptr;  // packed BF16 MMA operand fragments [kFragWords]
    float *d_m = nullptr, *d_v = nullptr;  // Adam moments
    float *d_part = nullptr;   // per-block partial gradients [part_blocks][kNParams + 1] (last: loss)
    float *d_grad = nullptr;   // summed gradient [kNParams + 1]
    int *d_idx = nullptr;      // sample indices of a batch
    size_t idx_cap = 0;
    int part_blocks = 0;
    long long adam_t = 0;
    int pack();                // d_w -> d_wq, d_frag
};

struct fx_lsm_data {
    fx_ctx *ctx = nullptr;
    size_t cap = 0, count = 0;
    __nv_bfloat16 *d_in = nullptr;  // [cap][3][25][25]
    float *d_tgt = nullptr;         // [cap][2][16][16]: tH, tE
    float *d_norm = nullptr;        // [cap][2]: nH, nE
};

namespace fx {
// training-side entry points of fx_learned.cu used by the operator code in fx_solvers.cu
int lsm_batch_grad(fx_lsm *m, const fx_lsm_data *d, const int *h_idx, size_t count, float lambda);  // -> m->d_grad
}  // namespace fx
