// mlp.cu — the learned orientation proposal network (include/mbs_mlp.h).
//
// 4 -> 128 -> 128 -> 128 -> 1 with erf GELU.  Every layer product runs on
// the 5th-generation tensor cores as BF16 x BF16 -> FP32: tcgen05.mma
// (M = 128, N <= 128, K = 16 per instruction) issued by one thread per CTA,
// both operands in shared memory in the K-major no-swizzle layout (8 x 16-byte
// core matrices), the accumulator in tensor memory, read back with
// tcgen05.ld for the epilogue.  Operands are staged from global memory with
// arbitrary strides, so the transposed operands of the backward pass need no
// copies.  The 128 -> 1 head is a per-sample dot product in FP32.  Master parameters,
// gradients and Adam moments are FP32; the BF16 weight copies are refreshed
// after every update.  All reductions (bias gradients, loss) run in a fixed
// order, so training is bitwise repeatable for a given seed.
#include "mbs_mlp.h"

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>
#include <string>
#include <vector>

namespace mlp {

constexpr int kH = MBS_MLP_HIDDEN;   // 128
constexpr int kIn = MBS_MLP_IN;      // 4
constexpr int kInPad = 16;           // K of the first layer, padded for the MMA
constexpr int kTile = 128;           // M of one tcgen05.mma tile (batch rows padded to it)
constexpr int kTileN = 32;           // N of one CTA's tile: four CTAs share a 128-wide layer
constexpr int kTileK = 128;          // K staged per round
constexpr int kGemmSmem = 2 * kTile * kTileK * 2 + 1024;   // A, B tiles (BF16) + barrier

// Flat parameter offsets (include/mbs_mlp.h)
constexpr int oW1 = 0, ob1 = oW1 + kH * kIn, oW2 = ob1 + kH, ob2 = oW2 + kH * kH;
constexpr int oW3 = ob2 + kH, ob3 = oW3 + kH * kH, ow4 = ob3 + kH, ob4 = ow4 + kH;
constexpr int kNParams = ob4 + 1;
static_assert(kNParams == MBS_MLP_N_PARAMS, "parameter layout");

using bf16 = __nv_bfloat16;

__device__ __forceinline__ float gelu(float z)
{
    return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f));
}

__device__ __forceinline__ float gelu_grad(float z)
{
    return 0.5f * (1.0f + erff(z * 0.70710678118654752f))
         + z * 0.39894228040143268f * expf(-0.5f * z * z);
}

// Logical matrix view: X[r][c] = p[r * sr + c * sc].
struct Mat {
    const bf16 *p;
    long sr, sc;
};

enum { kModeFwd = 0, kModeBwd = 1, kModeF32 = 2 };

struct GemmOut {
    const float *bias;   // kModeFwd: [N]
    const float *zin;    // kModeBwd: pre-activation of the layer below [M][ldo]
    float *z;            // kModeFwd: pre-activation out
    bf16 *h;             // kModeFwd: activation out; kModeBwd: gradient out
    float *f;            // kModeF32: plain product out
    int ldo;
};

// ---- tcgen05 helpers --------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor, K-major without swizzle: start address,
// leading byte offset (between the two 8-element core matrices along K),
// stride byte offset (between 8-row groups), version 1, swizzle none.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16)
         | ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both
// K-major, N and M of the tile.
__host__ __device__ constexpr uint32_t umma_idesc(int M, int N)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// Byte offset of element (row, k) in a K-major no-swizzle tile whose rows hold
// kt elements: core matrix (row / 8, k / 8), 16 bytes per row inside it.
__device__ __forceinline__ uint32_t kmajor_off(int row, int k, int kt)
{
    return (uint32_t)((row >> 3) * (kt * 16) + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

// Bounded wait on an mbarrier phase (at most `limit` polls); false when it
// did not complete.
constexpr int kDefaultPollLimit = 1 << 22;

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t phase, int limit)
{
    for (int it = 0; it < limit; ++it) {
        uint32_t done;
        asm volatile("{\n\t.reg .pred P1;\n\t"
                     "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
                     "selp.b32 %0, 1, 0, P1;\n\t}"
                     : "=r"(done) : "r"(bar), "r"(phase) : "memory");
        if (done)
            return true;
    }
    return false;
}

// C[M][N] = A[M][K] B[K][N] with the epilogue of MODE.  M a multiple of 128,
// N a multiple of 16 (at most 128 per CTA), K a multiple of 16.  Grid: x over
// N tiles, y over M tiles; 128 threads, thread i owns accumulator row i
// (tensor-memory lane i).  On a barrier timeout *err is set and the CTA
// frees its tensor memory and returns without storing.
// Stages the rows x kt operand tile whose element (r, k) is
// p[(row0 + r) * rs + (k0 + k) * ks] into shared memory in the K-major core-
// matrix layout (kmajor_off); rows at or beyond row_limit read as zero.
// Operands contiguous along K move in 16-byte vectors (one core-matrix row
// each); operands contiguous along the rows move in 16-byte vectors of 8 rows
// at one k; anything else element by element.  Every path is unrolled so a
// thread keeps several global loads in flight.
__device__ __forceinline__ void stage_operand(unsigned char *dst, const bf16 *p, long rs, long ks,
                                              int row0, int rows, int row_limit, int k0, int kt)
{
    const bool aligned = (reinterpret_cast<uintptr_t>(p) & 15) == 0;
    if (ks == 1 && (rs & 7) == 0 && aligned) {
        const int kc = kt >> 3;
        const int n = rows * kc;
#pragma unroll 4
        for (int v = threadIdx.x; v < n; v += blockDim.x) {
            const int r = v / kc, c = v - r * kc;
            uint4 val = make_uint4(0u, 0u, 0u, 0u);
            if (row0 + r < row_limit)
                val = *reinterpret_cast<const uint4 *>(p + (long)(row0 + r) * rs + k0 + c * 8);
            *reinterpret_cast<uint4 *>(dst + kmajor_off(r, c * 8, kt)) = val;
        }
    } else if (rs == 1 && (ks & 7) == 0 && aligned && (rows & 7) == 0 && (row0 & 7) == 0
               && (row_limit & 7) == 0) {
        const int rc = rows >> 3;
        const int n = kt * rc;
#pragma unroll 4
        for (int v = threadIdx.x; v < n; v += blockDim.x) {
            const int k = v / rc, r = (v - k * rc) * 8;
            uint4 val = make_uint4(0u, 0u, 0u, 0u);
            if (row0 + r < row_limit)
                val = *reinterpret_cast<const uint4 *>(p + (long)(row0 + r) + (long)(k0 + k) * ks);
            const bf16 *e = reinterpret_cast<const bf16 *>(&val);
#pragma unroll
            for (int j = 0; j < 8; ++j)
                *reinterpret_cast<bf16 *>(dst + kmajor_off(r + j, k, kt)) = e[j];
        }
    } else {
        const bf16 zero = __float2bfloat16(0.f);
#pragma unroll 4
        for (int i = threadIdx.x; i < rows * kt; i += blockDim.x) {
            const int r = i / kt, k = i - r * kt;
            *reinterpret_cast<bf16 *>(dst + kmajor_off(r, k, kt)) =
                row0 + r < row_limit ? p[(long)(row0 + r) * rs + (long)(k0 + k) * ks] : zero;
        }
    }
}

constexpr int kGemmThreads = 256;   // 8 warps: all stage, two warpgroups read TMEM

// Watchdog of the tensor-core barrier waits: the device error flag, the
// poll limit, and (test hook) whether to leave out the MMAs and their
// commit, so that the wait runs out with no asynchronous operation pending.
struct Watch {
    int *err;
    int poll_limit;
    int skip_mma;
};

template <int MODE>
__global__ void __launch_bounds__(kGemmThreads) k_gemm(int M, int N, int K, Mat A, Mat B, GemmOut o, Watch w)
{
    extern __shared__ __align__(1024) unsigned char gsm[];
    bf16 *sA = reinterpret_cast<bf16 *>(gsm);
    bf16 *sB = reinterpret_cast<bf16 *>(gsm + kTile * kTileK * 2);
    uint64_t *bar = reinterpret_cast<uint64_t *>(gsm + 2 * kTile * kTileK * 2);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(bar + 1);
    const int m0 = blockIdx.y * kTile, n0 = blockIdx.x * kTileN;
    const int nt = min(kTileN, N - n0);                  // multiple of 16
    const int ncols = nt <= 32 ? 32 : (nt <= 64 ? 64 : 128);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(smem_u32(tslot)), "r"(ncols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (threadIdx.x == 0)
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(bar)), "r"(1));
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const uint32_t tmem = *tslot;
    const uint32_t idesc = umma_idesc(kTile, nt);
    uint32_t phase = 0;
    bool ok = true;
    for (int k0 = 0; k0 < K && ok; k0 += kTileK) {
        const int kt = min(kTileK, K - k0);              // multiple of 16
        // stage A (kTile x kt: element (m, k) = A.p[m sr + k sc]) and B
        // (nt x kt: element (n, k) = B.p[k sr + n sc]) in the K-major layout
        stage_operand(reinterpret_cast<unsigned char *>(sA), A.p, A.sr, A.sc, m0, kTile, M, k0, kt);
        stage_operand(reinterpret_cast<unsigned char *>(sB), B.p, B.sc, B.sr, n0, nt, n0 + nt, k0, kt);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (threadIdx.x == 0 && !w.skip_mma) {
            asm volatile("tcgen05.fence::after_thread_sync;");
            const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB), sbo = (uint32_t)kt * 16;
            for (int s = 0; s < kt / 16; ++s) {
                const uint64_t da = umma_desc(a0 + 256 * s, 128, sbo);
                const uint64_t db = umma_desc(b0 + 256 * s, 128, sbo);
                const uint32_t acc = (k0 > 0 || s > 0) ? 1u : 0u;
                asm volatile("{\n\t.reg .pred p;\n\t"
                             "setp.ne.b32 p, %4, 0;\n\t"
                             "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                             :: "r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(acc));
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                         :: "r"(smem_u32(bar)) : "memory");
        }
        // the tiles may be overwritten once the MMAs that read them are done
        ok = mbar_wait(smem_u32(bar), phase, w.poll_limit);
        phase ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;");
        __syncthreads();
    }
    if (!ok) {
        if (threadIdx.x == 0)
            atomicExch(w.err, 1);
        mbar_wait(smem_u32(bar), phase ^ 1u, w.poll_limit);   // let any MMA in flight finish, bounded
    } else {
        // warp w reads TMEM lanes 32 (w % 4) .. + 31 (its lane quarter); the
        // two warpgroups take alternate 16-column chunks
        const int wq = warp & 3, wg = warp >> 2;
        const int r = m0 + wq * 32 + lane;
        for (int c0 = wg * 16; c0 < nt; c0 += 32) {
            uint32_t v[16];
            const uint32_t ta = tmem + ((uint32_t)(wq * 32) << 16) + (uint32_t)c0;
            asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 "
                         "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
                         : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]),
                           "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]),
                           "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
                         : "r"(ta));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (r < M) {
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    const int c = n0 + c0 + i;
                    const long idx = (long)r * o.ldo + c;
                    const float val = __uint_as_float(v[i]);
                    if (MODE == kModeFwd) {
                        const float z = val + o.bias[c];
                        o.z[idx] = z;
                        o.h[idx] = __float2bfloat16(gelu(z));
                    } else if (MODE == kModeBwd) {
                        o.h[idx] = __float2bfloat16(val * gelu_grad(o.zin[idx]));
                    } else {
                        o.f[idx] = val;
                    }
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(ncols));
}

// X0[b][0..15] (BF16): the quaternion in columns 0..3, zeros elsewhere and
// on padding rows.
__global__ void k_input(const float *q, int n, int bpad, bf16 *x0)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= bpad * kInPad)
        return;
    const int b = i / kInPad, c = i - b * kInPad;
    x0[i] = __float2bfloat16((b < n && c < kIn) ? q[b * kIn + c] : 0.f);
}

// y[b] = sum_j H3[b][j] w4[j] + b4: one warp per sample, fixed lane order.
__global__ void k_head_fwd(const bf16 *h3, const float *params, int n, float *y)
{
    const int b = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (b >= n)
        return;
    float s = 0.f;
    for (int j = lane; j < kH; j += 32)
        s = fmaf(__bfloat162float(h3[(long)b * kH + j]), params[ow4 + j], s);
#pragma unroll
    for (int w = 16; w > 0; w >>= 1)
        s += __shfl_xor_sync(0xffffffffu, s, w);
    if (lane == 0)
        y[b] = s + params[ob4];
}

// dy[b] = 2 (y_b - t_b) / n (0 on padding rows);
// dZ3[b][j] = dy_b w4[j] gelu'(Z3[b][j]).
__global__ void k_head_bwd(const float *y, const float *t, int n, int bpad, const float *params,
                           const float *z3, float *dy, bf16 *dz3)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= bpad * kH)
        return;
    const int b = i / kH, j = i - b * kH;
    const float d = b < n ? 2.f * (y[b] - t[b]) / (float)n : 0.f;
    if (j == 0)
        dy[b] = d;
    dz3[i] = __float2bfloat16(d * params[ow4 + j] * gelu_grad(z3[i]));
}

// Column sums of a [rows][cols] BF16 matrix, fixed row order: out[c].
// Column sums in fixed order: block b sums columns 32 b .. 32 b + 31, its 8
// row groups g (threadIdx.x / 32) take rows g, g + 8, ... in turn, and the
// group sums are added in group order.  Launch with 256 threads and
// ceil(cols / 32) blocks.
__global__ void __launch_bounds__(256) k_colsum_bf16(const bf16 *x, int rows, int cols, float *out)
{
    __shared__ float part[8][32];
    const int cl = threadIdx.x & 31, g = threadIdx.x >> 5;
    const int c = blockIdx.x * 32 + cl;
    float s = 0.f;
    if (c < cols)
        for (int r = g; r < rows; r += 8)
            s += __bfloat162float(x[(long)r * cols + c]);
    part[g][cl] = s;
    __syncthreads();
    if (g == 0 && c < cols) {
        float t = part[0][cl];
        for (int k = 1; k < 8; ++k)
            t += part[k][cl];
        out[c] = t;
    }
}

// Head gradients: gw4[j] = sum_b dy_b H3[b][j] (j < 128), gb4 = sum_b dy_b.
// (fixed order as k_colsum_bf16: block b covers outputs j = 32 b .. 32 b + 31,
// output kH is gb4; launch with 256 threads and kH / 32 + 1 blocks)
__global__ void __launch_bounds__(256) k_head_grad(const float *dy, const bf16 *h3, int bpad, float *grad)
{
    __shared__ float part[8][32];
    const int jl = threadIdx.x & 31, g = threadIdx.x >> 5;
    const int j = blockIdx.x * 32 + jl;
    float s = 0.f;
    if (j <= kH)
        for (int b = g; b < bpad; b += 8)
            s += j < kH ? dy[b] * __bfloat162float(h3[(long)b * kH + j]) : dy[b];
    part[g][jl] = s;
    __syncthreads();
    if (g == 0 && j <= kH) {
        float t = part[0][jl];
        for (int k = 1; k < 8; ++k)
            t += part[k][jl];
        grad[j < kH ? ow4 + j : ob4] = t;
    }
}

// W1 gradient: the first kIn columns of the padded [128][16] product.
__global__ void k_pack_w1_grad(const float *gw1p, float *grad)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kH * kIn)
        return;
    const int r = i / kIn, c = i - r * kIn;
    grad[oW1 + i] = gw1p[r * kInPad + c];
}

// BF16 copies of the weights (W1 padded to [128][16]).
__global__ void k_refresh(const float *params, bf16 *w1p, bf16 *w2, bf16 *w3)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < kH * kInPad) {
        const int r = i / kInPad, c = i - r * kInPad;
        w1p[i] = __float2bfloat16(c < kIn ? params[oW1 + r * kIn + c] : 0.f);
    }
    if (i < kH * kH) {
        w2[i] = __float2bfloat16(params[oW2 + i]);
        w3[i] = __float2bfloat16(params[oW3 + i]);
    }
}

// Mean-squared loss of n samples, one CTA, fixed-order tree sum.
__global__ void __launch_bounds__(256) k_loss(const float *y, const float *t, int n, float *out)
{
    __shared__ float red[256];
    float s = 0.f;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const float d = y[i] - t[i];
        s = fmaf(d, d, s);
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
            red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        *out = red[0] / (float)max(n, 1);
}

// The training step's minibatch at offset b0 of the epoch the device counter
// holds (so one captured epoch replays over every epoch's shuffled order):
// t_b[i] = t[s], X0[i] = the BF16 quaternion of s padded to kInPad columns,
// s = idx[epoch n + b0 + i]; rows n_b .. bpad-1 of X0 are zeros (k_input's
// layout, without the FP32 copy of the quaternions).
__global__ void k_gather_input(const float *q, const float *t, const int *idx, const int *epoch,
                               int n, int b0, int nb, int bpad, bf16 *x0, float *tb)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= bpad)
        return;
    if (i < nb) {
        const int s = idx[(size_t)(*epoch) * n + b0 + i];
#pragma unroll
        for (int c = 0; c < kInPad; ++c)
            x0[i * kInPad + c] = __float2bfloat16(c < kIn ? q[s * kIn + c] : 0.f);
        tb[i] = t[s];
    } else {
#pragma unroll
        for (int c = 0; c < kInPad; ++c)
            x0[i * kInPad + c] = __float2bfloat16(0.f);
    }
}

// Adam with the bias corrections of step epoch * steps_per_epoch + k (bc[2 j],
// bc[2 j + 1] for the call's j-th step), and the BF16 copies of the updated
// weights (k_refresh's layout; W1's padding columns stay the zeros that
// k_refresh wrote).
__global__ void k_adam_refresh(float *p, const float *g, float *m, float *v, int n, float lr,
                               const float *bc, const int *epoch, int steps_per_epoch, int k,
                               bf16 *w1p, bf16 *w2, bf16 *w3)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const int j = (*epoch) * steps_per_epoch + k;
    const float bc1 = bc[2 * j], bc2 = bc[2 * j + 1];
    const float gi = g[i];
    const float mi = 0.9f * m[i] + 0.1f * gi;
    const float vi = 0.999f * v[i] + 0.001f * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float pi = p[i] - lr * (mi / bc1) / (sqrtf(vi / bc2) + 1e-8f);
    p[i] = pi;
    if (i < ob1) {
        const int r = (i - oW1) / kIn, c = (i - oW1) - r * kIn;
        w1p[r * kInPad + c] = __float2bfloat16(pi);
    } else if (i >= oW2 && i < ob2) {
        w2[i - oW2] = __float2bfloat16(pi);
    } else if (i >= oW3 && i < ob3) {
        w3[i - oW3] = __float2bfloat16(pi);
    }
}

// End of a captured epoch: the epoch counter moves on.
__global__ void k_next_epoch(int *epoch)
{
    *epoch += 1;
}

inline int pad_rows(int n) { return (n + kTile - 1) / kTile * kTile; }

}  // namespace mlp

using namespace mlp;

struct mbs_mlp {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    float *params = nullptr, *grad = nullptr, *m = nullptr, *v = nullptr;
    bf16 *w1p = nullptr, *w2 = nullptr, *w3 = nullptr;
    int step = 0;
    // activations for up to `cap` padded rows
    int cap = 0;
    bf16 *x0 = nullptr, *h1 = nullptr, *h2 = nullptr, *h3 = nullptr;
    bf16 *dz1 = nullptr, *dz2 = nullptr, *dz3 = nullptr;
    float *z1 = nullptr, *z2 = nullptr, *z3 = nullptr;
    float *y = nullptr, *t = nullptr, *dy = nullptr, *q = nullptr;
    float *gw1p = nullptr, *scalar = nullptr;
    int poll_limit = kDefaultPollLimit;   // mbs_mlp_set_watchdog
    int skip_mma = 0;
};

namespace {

int mfail(mbs_mlp *net, int code, const std::string &msg)
{
    if (net)
        net->err = msg;
    return code;
}

#define MK(expr, where)                                                          \
    do {                                                                         \
        cudaError_t e_ = (expr);                                                 \
        if (e_ != cudaSuccess)                                                   \
            return mfail(net, -3, std::string(where) + ": " + cudaGetErrorString(e_)); \
    } while (0)

void free_acts(mbs_mlp *net)
{
    void *ps[] = {net->x0, net->h1, net->h2, net->h3, net->dz1, net->dz2, net->dz3, net->z1,
                  net->z2, net->z3, net->y, net->t, net->dy, net->q};
    for (void *p : ps)
        cudaFree(p);
    net->x0 = net->h1 = net->h2 = net->h3 = net->dz1 = net->dz2 = net->dz3 = nullptr;
    net->z1 = net->z2 = net->z3 = net->y = net->t = net->dy = net->q = nullptr;
    net->cap = 0;
}

int ensure_acts(mbs_mlp *net, int rows)
{
    const int need = pad_rows(std::max(rows, 1));
    if (need <= net->cap)
        return 0;
    free_acts(net);
    const size_t hb = (size_t)need * kH;
    MK(cudaMalloc((void **)&net->x0, (size_t)need * kInPad * sizeof(bf16)), "cudaMalloc mlp");
    MK(cudaMalloc((void **)&net->h1, hb * sizeof(bf16)), "cudaMalloc mlp");
    MK(cudaMalloc((void **)&net->h2, hb * sizeof(bf16)), "cudaMalloc mlp");
    MK(cudaMalloc((void **)&net->h3, hb * sizeof(bf16)), "cudaMalloc mlp");
    MK(cudaMalloc((void **)&net->dz1, hb * sizeof(bf16)), "cudaMalloc mlp");
    MK(cudaMalloc((void **)&net->dz2, hb * sizeof(bf16)), "cudaMalloc mlp");
    MK(cudaMalloc((void **)&net->dz3, hb * sizeof(bf16)), "cudaMalloc mlp");
    MK(cudaMalloc((void **)&net->z1, hb * sizeof(float)), "cudaMalloc mlp");
    MK(cudaMalloc((void **)&net->z2, hb * sizeof(float)), "cudaMalloc mlp");
    MK(cudaMalloc((void **)&net->z3, hb * sizeof(float)), "cudaMalloc mlp");
    MK(cudaMalloc((void **)&net->y, need * sizeof(float)), "cudaMalloc mlp");
    MK(cudaMalloc((void **)&net->t, need * sizeof(float)), "cudaMalloc mlp");
    MK(cudaMalloc((void **)&net->dy, need * sizeof(float)), "cudaMalloc mlp");
    MK(cudaMalloc((void **)&net->q, (size_t)need * kIn * sizeof(float)), "cudaMalloc mlp");
    net->cap = need;
    return 0;
}

dim3 tiles(int M, int N) { return dim3((N + kTileN - 1) / kTileN, (M + kTile - 1) / kTile); }

// Device flag set by a GEMM whose tensor-core barrier wait ran out (the
// third int of the network's scalar scratch).
int *mlp_err(mbs_mlp *net) { return reinterpret_cast<int *>(net->scalar) + 2; }

Watch watch(mbs_mlp *net) { return Watch{mlp_err(net), net->poll_limit, net->skip_mma}; }

// Reset before a call's kernels, checked after its final synchronisation.
int check_err(mbs_mlp *net)
{
    int e = 0;
    MK(cudaMemcpy(&e, mlp_err(net), sizeof(int), cudaMemcpyDeviceToHost), "D2H error flag");
    if (e) {
        cudaMemset(mlp_err(net), 0, sizeof(int));
        return mfail(net, -6, "tensor-core barrier wait timed out");
    }
    return 0;
}

// The GEMM kernels' dynamic shared-memory limit, set once per process
// (before any graph capture: the training epoch is captured).
void gemm_attrs()
{
    static bool done = false;
    if (!done) {
        cudaFuncSetAttribute(k_gemm<kModeFwd>, cudaFuncAttributeMaxDynamicSharedMemorySize, kGemmSmem);
        cudaFuncSetAttribute(k_gemm<kModeBwd>, cudaFuncAttributeMaxDynamicSharedMemorySize, kGemmSmem);
        cudaFuncSetAttribute(k_gemm<kModeF32>, cudaFuncAttributeMaxDynamicSharedMemorySize, kGemmSmem);
        done = true;
    }
}

template <int MODE>
void gemm(cudaStream_t s, int M, int N, int K, Mat A, Mat B, GemmOut o, Watch w)
{
    gemm_attrs();
    k_gemm<MODE><<<tiles(M, N), kGemmThreads, kGemmSmem, s>>>(M, N, K, A, B, o, w);
}

// Forward pass of n samples already in net->q (device); train keeps the
// pre-activations for the backward pass.
int forward_dev(mbs_mlp *net, int n, bool x0_ready = false)
{
    const int bp = pad_rows(n);
    cudaStream_t s = net->stream;
    if (!x0_ready)
        k_input<<<(bp * kInPad + 255) / 256, 256, 0, s>>>(net->q, n, bp, net->x0);
    GemmOut o{};
    o.ldo = kH;
    o.bias = net->params + ob1; o.z = net->z1; o.h = net->h1;
    gemm<kModeFwd>(s, bp, kH, kInPad, Mat{net->x0, kInPad, 1},
                   Mat{net->w1p, 1, kInPad}, o, watch(net));
    o.bias = net->params + ob2; o.z = net->z2; o.h = net->h2;
    gemm<kModeFwd>(s, bp, kH, kH, Mat{net->h1, kH, 1},
                   Mat{net->w2, 1, kH}, o, watch(net));
    o.bias = net->params + ob3; o.z = net->z3; o.h = net->h3;
    gemm<kModeFwd>(s, bp, kH, kH, Mat{net->h2, kH, 1},
                   Mat{net->w3, 1, kH}, o, watch(net));
    k_head_fwd<<<(n + 7) / 8, 256, 0, s>>>(net->h3, net->params, n, net->y);
    MK(cudaGetLastError(), "mlp forward launch");
    return 0;
}

// Backward pass after forward_dev (targets in net->t): net->grad (flat).
int backward_dev(mbs_mlp *net, int n)
{
    const int bp = pad_rows(n);
    cudaStream_t s = net->stream;
    k_head_bwd<<<(bp * kH + 255) / 256, 256, 0, s>>>(net->y, net->t, n, bp, net->params, net->z3,
                                                     net->dy, net->dz3);
    k_head_grad<<<kH / 32 + 1, 256, 0, s>>>(net->dy, net->h3, bp, net->grad);
    GemmOut o{};
    // layer 3: dW3 = dZ3^T H2, db3 = colsum dZ3, dZ2 = (dZ3 W3) * gelu'(Z2)
    o.ldo = kH; o.f = net->grad + oW3;
    gemm<kModeF32>(s, kH, kH, bp, Mat{net->dz3, 1, kH},
                   Mat{net->h2, kH, 1}, o, watch(net));
    k_colsum_bf16<<<(kH + 31) / 32, 256, 0, s>>>(net->dz3, bp, kH, net->grad + ob3);
    o = GemmOut{}; o.ldo = kH; o.zin = net->z2; o.h = net->dz2;
    gemm<kModeBwd>(s, bp, kH, kH, Mat{net->dz3, kH, 1},
                   Mat{net->w3, kH, 1}, o, watch(net));
    // layer 2
    o = GemmOut{}; o.ldo = kH; o.f = net->grad + oW2;
    gemm<kModeF32>(s, kH, kH, bp, Mat{net->dz2, 1, kH},
                   Mat{net->h1, kH, 1}, o, watch(net));
    k_colsum_bf16<<<(kH + 31) / 32, 256, 0, s>>>(net->dz2, bp, kH, net->grad + ob2);
    o = GemmOut{}; o.ldo = kH; o.zin = net->z1; o.h = net->dz1;
    gemm<kModeBwd>(s, bp, kH, kH, Mat{net->dz2, kH, 1},
                   Mat{net->w2, kH, 1}, o, watch(net));
    // layer 1
    o = GemmOut{}; o.ldo = kInPad; o.f = net->gw1p;
    gemm<kModeF32>(s, kH, kInPad, bp, Mat{net->dz1, 1, kH},
                   Mat{net->x0, kInPad, 1}, o, watch(net));
    k_pack_w1_grad<<<(kH * kIn + 127) / 128, 128, 0, s>>>(net->gw1p, net->grad);
    k_colsum_bf16<<<(kH + 31) / 32, 256, 0, s>>>(net->dz1, bp, kH, net->grad + ob1);
    MK(cudaGetLastError(), "mlp backward launch");
    return 0;
}

int refresh(mbs_mlp *net)
{
    k_refresh<<<(kH * kH + 255) / 256, 256, 0, net->stream>>>(net->params, net->w1p, net->w2, net->w3);
    MK(cudaGetLastError(), "mlp refresh launch");
    return 0;
}

}  // namespace

extern "C" int mbs_mlp_create(mbs_mlp **out, int device, uint64_t seed)
{
    if (!out)
        return -1;
    *out = nullptr;
    mbs_mlp *net = new mbs_mlp();
    net->device = device;
    auto bail = [&](int rc) { mbs_mlp_destroy(net); return rc; };
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&net->stream, cudaStreamNonBlocking) != cudaSuccess)
        return bail(-3);
    const size_t np = kNParams;
    if (cudaMalloc((void **)&net->params, np * 4) || cudaMalloc((void **)&net->grad, np * 4)
        || cudaMalloc((void **)&net->m, np * 4) || cudaMalloc((void **)&net->v, np * 4)
        || cudaMalloc((void **)&net->w1p, kH * kInPad * sizeof(bf16))
        || cudaMalloc((void **)&net->w2, kH * kH * sizeof(bf16))
        || cudaMalloc((void **)&net->w3, kH * kH * sizeof(bf16))
        || cudaMalloc((void **)&net->gw1p, kH * kInPad * 4) || cudaMalloc((void **)&net->scalar, 16)
        || cudaMemset(net->scalar, 0, 16))
        return bail(-4);
    // uniform +-sqrt(6 / fan_in) weights, zero biases
    std::vector<float> p(np, 0.f);
    std::mt19937_64 rng(seed);
    auto fill = [&](int off, int count, int fan_in) {
        std::uniform_real_distribution<float> u(-std::sqrt(6.f / fan_in), std::sqrt(6.f / fan_in));
        for (int i = 0; i < count; ++i)
            p[off + i] = u(rng);
    };
    fill(oW1, kH * kIn, kIn);
    fill(oW2, kH * kH, kH);
    fill(oW3, kH * kH, kH);
    fill(ow4, kH, kH);
    const int rc = mbs_mlp_set_params(net, p.data());
    if (rc)
        return bail(rc);
    *out = net;
    return 0;
}

extern "C" int mbs_mlp_destroy(mbs_mlp *net)
{
    if (!net)
        return -1;
    cudaSetDevice(net->device);
    free_acts(net);
    void *ps[] = {net->params, net->grad, net->m, net->v, net->w1p, net->w2, net->w3, net->gw1p,
                  net->scalar};
    for (void *p : ps)
        cudaFree(p);
    if (net->stream)
        cudaStreamDestroy(net->stream);
    delete net;
    return 0;
}

extern "C" int mbs_mlp_set_watchdog(mbs_mlp *net, int poll_limit, int skip_mma)
{
    if (!net)
        return -1;
    net->poll_limit = poll_limit > 0 ? poll_limit : kDefaultPollLimit;
    net->skip_mma = skip_mma ? 1 : 0;
    return 0;
}

extern "C" const char *mbs_mlp_last_error(const mbs_mlp *net)
{
    return net ? net->err.c_str() : "null network";
}

extern "C" int mbs_mlp_get_params(mbs_mlp *net, float *params)
{
    if (!net || !params)
        return mfail(net, -1, "null argument");
    MK(cudaSetDevice(net->device), "cudaSetDevice");
    MK(cudaMemcpyAsync(params, net->params, kNParams * 4, cudaMemcpyDeviceToHost, net->stream), "D2H params");
    MK(cudaStreamSynchronize(net->stream), "sync");
    return 0;
}

extern "C" int mbs_mlp_set_params(mbs_mlp *net, const float *params)
{
    if (!net || !params)
        return mfail(net, -1, "null argument");
    MK(cudaSetDevice(net->device), "cudaSetDevice");
    MK(cudaMemcpyAsync(net->params, params, kNParams * 4, cudaMemcpyHostToDevice, net->stream), "H2D params");
    MK(cudaMemsetAsync(net->m, 0, kNParams * 4, net->stream), "memset");
    MK(cudaMemsetAsync(net->v, 0, kNParams * 4, net->stream), "memset");
    net->step = 0;
    int rc = refresh(net);
    if (rc)
        return rc;
    MK(cudaStreamSynchronize(net->stream), "sync");
    return 0;
}

extern "C" int mbs_mlp_forward(mbs_mlp *net, const float *q, int n, float *y)
{
    if (!net || n < 0 || (n > 0 && (!q || !y)))
        return mfail(net, -1, "bad arguments");
    if (n == 0)
        return 0;
    MK(cudaSetDevice(net->device), "cudaSetDevice");
    int rc = ensure_acts(net, n);
    if (rc)
        return rc;
    MK(cudaMemcpyAsync(net->q, q, (size_t)n * kIn * 4, cudaMemcpyHostToDevice, net->stream), "H2D q");
    if ((rc = forward_dev(net, n)))
        return rc;
    MK(cudaMemcpyAsync(y, net->y, (size_t)n * 4, cudaMemcpyDeviceToHost, net->stream), "D2H y");
    MK(cudaStreamSynchronize(net->stream), "sync");
    return check_err(net);
}

extern "C" int mbs_mlp_loss_grad(mbs_mlp *net, const float *q, const float *t, int n, float *loss,
                                 float *grad)
{
    if (!net || n <= 0 || !q || !t)
        return mfail(net, -1, "bad arguments");
    MK(cudaSetDevice(net->device), "cudaSetDevice");
    int rc = ensure_acts(net, n);
    if (rc)
        return rc;
    MK(cudaMemcpyAsync(net->q, q, (size_t)n * kIn * 4, cudaMemcpyHostToDevice, net->stream), "H2D q");
    MK(cudaMemcpyAsync(net->t, t, (size_t)n * 4, cudaMemcpyHostToDevice, net->stream), "H2D t");
    if ((rc = forward_dev(net, n)) || (rc = backward_dev(net, n)))
        return rc;
    k_loss<<<1, 256, 0, net->stream>>>(net->y, net->t, n, net->scalar);
    MK(cudaGetLastError(), "loss launch");
    float l = 0.f;
    MK(cudaMemcpyAsync(&l, net->scalar, 4, cudaMemcpyDeviceToHost, net->stream), "D2H loss");
    if (grad)
        MK(cudaMemcpyAsync(grad, net->grad, kNParams * 4, cudaMemcpyDeviceToHost, net->stream), "D2H grad");
    MK(cudaStreamSynchronize(net->stream), "sync");
    if (loss)
        *loss = l;
    return check_err(net);
}

extern "C" int mbs_mlp_train(mbs_mlp *net, const float *q, const float *t, int n, int epochs,
                             int batch, float lr, uint64_t seed, float *final_loss)
{
    if (!net || n <= 0 || !q || !t || epochs < 0 || batch <= 0 || !(lr > 0.f))
        return mfail(net, -1, "bad arguments");
    MK(cudaSetDevice(net->device), "cudaSetDevice");
    batch = std::min(batch, n);
    int rc = ensure_acts(net, std::max(batch, n));
    if (rc)
        return rc;
    cudaStream_t s = net->stream;
    // one epoch's steps: minibatches of `batch`, the last one shorter
    std::vector<int> sizes;
    for (int b0 = 0; b0 < n; b0 += batch)
        sizes.push_back(std::min(batch, n - b0));
    const size_t steps = (size_t)epochs * sizes.size();
    float *dq = nullptr, *dt = nullptr, *dbc = nullptr;
    int *didx = nullptr, *dstate = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    auto cleanup = [&]() {
        if (exec)
            cudaGraphExecDestroy(exec);
        if (graph)
            cudaGraphDestroy(graph);
        cudaFree(dq); cudaFree(dt); cudaFree(didx); cudaFree(dbc); cudaFree(dstate);
    };
    if (cudaMalloc((void **)&dq, (size_t)n * kIn * 4) || cudaMalloc((void **)&dt, (size_t)n * 4)
        || cudaMalloc((void **)&didx, (size_t)epochs * n * 4 + 4)
        || cudaMalloc((void **)&dbc, steps * 2 * 4 + 8) || cudaMalloc((void **)&dstate, 8)) {
        cleanup();
        return mfail(net, -4, "cudaMalloc training set");
    }
    // the shuffled order of every epoch and every step's Adam bias
    // corrections, uploaded once
    std::vector<int> order((size_t)epochs * n);
    std::mt19937_64 rng(seed);
    std::vector<int> perm(n);
    for (int e = 0; e < epochs; ++e) {
        for (int i = 0; i < n; ++i)
            perm[i] = i;
        std::shuffle(perm.begin(), perm.end(), rng);
        std::copy(perm.begin(), perm.end(), order.begin() + (size_t)e * n);
    }
    std::vector<float> bc(steps * 2 + 2);
    for (size_t k = 0; k < steps; ++k) {
        const float step = (float)(net->step + 1 + (long long)k);
        bc[2 * k] = 1.f - std::pow(0.9f, step);
        bc[2 * k + 1] = 1.f - std::pow(0.999f, step);
    }
    const int zero2[2] = {0, 0};
    cudaError_t e = cudaMemcpyAsync(dq, q, (size_t)n * kIn * 4, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(dt, t, (size_t)n * 4, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && epochs > 0)
        e = cudaMemcpyAsync(didx, order.data(), order.size() * 4, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess && epochs > 0)
        e = cudaMemcpyAsync(dbc, bc.data(), steps * 2 * 4, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(dstate, zero2, 8, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(s);   // the host arrays are read before they go
    if (e != cudaSuccess) {
        cleanup();
        return mfail(net, -3, std::string("training upload: ") + cudaGetErrorString(e));
    }
    // One epoch (every minibatch: gather, forward, backward, Adam, BF16
    // weight copies, cursor advance) captured once as a graph and replayed
    // per epoch: about twenty small launches per step would otherwise bound
    // the training by launch latency.
    if (epochs > 0) {
        gemm_attrs();
        e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            const int spe = (int)sizes.size();
            for (int k = 0, b0 = 0; k < spe; b0 += sizes[k], ++k) {
                const int nb = sizes[k], bp = pad_rows(nb);
                k_gather_input<<<(bp + 127) / 128, 128, 0, s>>>(dq, dt, didx, dstate, n, b0, nb, bp,
                                                                net->x0, net->t);
                if ((rc = forward_dev(net, nb, true)) || (rc = backward_dev(net, nb)))
                    break;
                k_adam_refresh<<<(kNParams + 255) / 256, 256, 0, s>>>(
                    net->params, net->grad, net->m, net->v, kNParams, lr, dbc, dstate, spe, k,
                    net->w1p, net->w2, net->w3);
            }
            if (rc == 0)
                k_next_epoch<<<1, 1, 0, s>>>(dstate);
            const cudaError_t ec = cudaStreamEndCapture(s, &graph);
            if (e == cudaSuccess)
                e = ec;
        }
        if (e == cudaSuccess && rc == 0)
            e = cudaGraphInstantiate(&exec, graph, 0);
        for (int ep = 0; ep < epochs && e == cudaSuccess && rc == 0; ++ep)
            e = cudaGraphLaunch(exec, s);
        if (e != cudaSuccess || rc) {
            cudaGetLastError();
            cleanup();
            if (rc)
                return rc;
            return mfail(net, -3, std::string("training graph: ") + cudaGetErrorString(e));
        }
        net->step += (int)steps;
    }
    if (rc == 0 && final_loss) {
        // loss over the whole set with the trained parameters
        e = cudaMemcpyAsync(net->q, dq, (size_t)n * kIn * 4, cudaMemcpyDeviceToDevice, s);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(net->t, dt, (size_t)n * 4, cudaMemcpyDeviceToDevice, s);
        if (e == cudaSuccess && (rc = forward_dev(net, n)) == 0) {
            k_loss<<<1, 256, 0, s>>>(net->y, net->t, n, net->scalar);
            e = cudaMemcpyAsync(final_loss, net->scalar, 4, cudaMemcpyDeviceToHost, s);
        }
    }
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(s);
    cleanup();
    if (rc)
        return rc;
    if (e != cudaSuccess)
        return mfail(net, -3, std::string("training: ") + cudaGetErrorString(e));
    return check_err(net);
}
