// pb_mlp.cuh - the learned scheduler's network: 781 -> 256 -> 256 -> 4.
//
// Input: 781 binary features of a position - 12 x 64 piece-square (colour x
// piece type x square), side to move (white), 4 castle rights, 8 en-passant
// files.  Output: log2(1 + perft(k)) for k = 1..4.  Weights are BF16 (with an
// FP32 master copy for Adam), every accumulation is FP32.
//
// A position has at most 38 active inputs, so layer 1 is an embedding bag
// (sum of the active rows of W1), not a GEMM over a 95 %-zero matrix; its
// weight gradient is a scatter-add into the active rows.  Layer 2 (256x256)
// runs on the tensor cores with mma.sync m16n8k16 BF16 -> FP32; layer 3
// (256x4) is a per-sample dot product.
#pragma once
#include <cuda_bf16.h>

#include "pb_core.cuh"

namespace pb {

constexpr int MLP_IN = 781;
constexpr int MLP_H = 256;
constexpr int MLP_OUT = 4;
constexpr int MLP_MAX_ACTIVE = 40;

// ---------------------------------------------------------------- features
// Active feature indices of each position (padded with -1).
__global__ void k_features(const Board *__restrict__ boards, const uint8_t *__restrict__ states,
                           const uint8_t *__restrict__ colors, int n, int16_t *__restrict__ idx)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Board b = boards[i];
    u32 st = states[i];
    int16_t *o = idx + (size_t)i * MLP_MAX_ACTIVE;
    int k = 0;
    u64 occ = b.bb[1] | b.bb[2] | b.bb[3];
    while (occ && k < 32) {
        int sq = lsb(occ);
        int piece = (int)(((b.bb[1] >> sq) & 1) | (((b.bb[2] >> sq) & 1) << 1) | (((b.bb[3] >> sq) & 1) << 2));
        int col = (int)((b.bb[0] >> sq) & 1);
        o[k++] = (int16_t)((col * 6 + piece - 1) * 64 + sq);
        occ &= occ - 1;
    }
    if (colors[i] == WHITE) o[k++] = 768;
    for (int c = 0; c < 4; c++)
        if (st & (1u << c)) o[k++] = (int16_t)(769 + c);
    if (st >> 4) o[k++] = (int16_t)(773 + (st >> 4) - 1);
    while (k < MLP_MAX_ACTIVE) o[k++] = -1;
}

// ---------------------------------------------------------------- layer 1
// h1 = relu(b1 + sum of active rows of W1); stored FP32 (for backward) and
// BF16 (GEMM operand).  One block of 256 threads per sample.
__global__ void k_mlp_layer1(const int16_t *__restrict__ idx, const __nv_bfloat16 *__restrict__ w1,
                             const float *__restrict__ b1, int n, float *__restrict__ h1f,
                             __nv_bfloat16 *__restrict__ h1b)
{
    int s = blockIdx.x, j = threadIdx.x;
    if (s >= n) return;
    float acc = b1[j];
    const int16_t *a = idx + (size_t)s * MLP_MAX_ACTIVE;
#pragma unroll 4
    for (int k = 0; k < MLP_MAX_ACTIVE; k++) {
        int f = a[k];
        if (f < 0) break;
        acc += __bfloat162float(w1[(size_t)f * MLP_H + j]);
    }
    acc = fmaxf(acc, 0.f);
    h1f[(size_t)s * MLP_H + j] = acc;
    h1b[(size_t)s * MLP_H + j] = __float2bfloat16(acc);
}

// ---------------------------------------------------------------- tensor-core GEMM
// C[M x N] (FP32) = A[M x K] * B[K x N] with BF16 operands, FP32 accumulation.
// A is row-major (lda) or, with TA, stored as A^T row-major (element (m,k) at
// A[k*lda + m]); B likewise with TB.  64x64 block tile, 4 warps (each 32x32 =
// 2x4 mma tiles of 16x8), K step 16.  M, N multiples of 64, K of 16.
template <bool TA, bool TB>
__global__ void __launch_bounds__(128) k_gemm_bf16(const __nv_bfloat16 *__restrict__ A, int lda,
                                                   const __nv_bfloat16 *__restrict__ B, int ldb,
                                                   float *__restrict__ C, int ldc, int M, int N, int K,
                                                   float beta)
{
    __shared__ __nv_bfloat16 sA[64][16 + 8];   // [m][k]
    __shared__ __nv_bfloat16 sB[16][64 + 8];   // [k][n]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int m0 = blockIdx.y * 64, n0 = blockIdx.x * 64;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
    const int g = lane >> 2, t4 = lane & 3;
    float acc[2][4][4];
#pragma unroll
    for (int a = 0; a < 2; a++)
#pragma unroll
        for (int b = 0; b < 4; b++)
#pragma unroll
            for (int c = 0; c < 4; c++) acc[a][b][c] = 0.f;

    for (int k0 = 0; k0 < K; k0 += 16) {
        // stage A tile 64x16 and B tile 16x64 (8 elements per thread each)
        for (int e = tid; e < 64 * 16; e += 128) {
            int m = e / 16, k = e % 16;
            sA[m][k] = TA ? A[(size_t)(k0 + k) * lda + (m0 + m)] : A[(size_t)(m0 + m) * lda + (k0 + k)];
        }
        for (int e = tid; e < 16 * 64; e += 128) {
            int k = e / 64, nn = e % 64;
            sB[k][nn] = TB ? B[(size_t)(n0 + nn) * ldb + (k0 + k)] : B[(size_t)(k0 + k) * ldb + (n0 + nn)];
        }
        __syncthreads();
#pragma unroll
        for (int mi = 0; mi < 2; mi++) {
            const int r = wm + mi * 16;
            // A fragment (row-major 16x16): regs hold (row g | g+8, cols 2*t4 + {0,1} | +8)
            u32 a0 = *reinterpret_cast<const u32 *>(&sA[r + g][2 * t4]);
            u32 a1 = *reinterpret_cast<const u32 *>(&sA[r + g + 8][2 * t4]);
            u32 a2 = *reinterpret_cast<const u32 *>(&sA[r + g][2 * t4 + 8]);
            u32 a3 = *reinterpret_cast<const u32 *>(&sA[r + g + 8][2 * t4 + 8]);
#pragma unroll
            for (int ni = 0; ni < 4; ni++) {
                const int c = wn + ni * 8;
                // B fragment (16x8, k-major pairs): (k 2*t4 + {0,1} | +8, col g)
                __nv_bfloat162 b01, b23;
                b01.x = sB[2 * t4][c + g];
                b01.y = sB[2 * t4 + 1][c + g];
                b23.x = sB[2 * t4 + 8][c + g];
                b23.y = sB[2 * t4 + 9][c + g];
                u32 b0 = *reinterpret_cast<u32 *>(&b01), b1 = *reinterpret_cast<u32 *>(&b23);
                asm volatile(
                    "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
                    "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
                    : "+f"(acc[mi][ni][0]), "+f"(acc[mi][ni][1]), "+f"(acc[mi][ni][2]), "+f"(acc[mi][ni][3])
                    : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int mi = 0; mi < 2; mi++)
#pragma unroll
        for (int ni = 0; ni < 4; ni++) {
            int r = m0 + wm + mi * 16 + g, c = n0 + wn + ni * 8 + 2 * t4;
            float *p0 = C + (size_t)r * ldc + c, *p1 = C + (size_t)(r + 8) * ldc + c;
            if (beta != 0.f) {
                p0[0] = beta * p0[0] + acc[mi][ni][0];
                p0[1] = beta * p0[1] + acc[mi][ni][1];
                p1[0] = beta * p1[0] + acc[mi][ni][2];
                p1[1] = beta * p1[1] + acc[mi][ni][3];
            } else {
                p0[0] = acc[mi][ni][0];
                p0[1] = acc[mi][ni][1];
                p1[0] = acc[mi][ni][2];
                p1[1] = acc[mi][ni][3];
            }
        }
}

// h2 = relu(z2 + b2): FP32 and BF16 copies.
__global__ void k_bias_relu(const float *__restrict__ z, const float *__restrict__ bias, int n, float *__restrict__ hf,
                            __nv_bfloat16 *__restrict__ hb)
{
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)n * MLP_H) return;
    float v = fmaxf(z[i] + bias[i % MLP_H], 0.f);
    hf[i] = v;
    hb[i] = __float2bfloat16(v);
}

// y = b3 + h2 . W3 (one warp per sample), and with targets the loss gradient
// dy = 2 (y - t) / (n * 4) and the squared error sum.
__global__ void k_mlp_out(const float *__restrict__ h2, const __nv_bfloat16 *__restrict__ w3,
                          const float *__restrict__ b3, int n, float *__restrict__ y, const float *__restrict__ t,
                          float *__restrict__ dy, float *__restrict__ loss)
{
    int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (s >= n) return;
    float acc[MLP_OUT] = {0.f, 0.f, 0.f, 0.f};
    for (int j = lane; j < MLP_H; j += 32) {
        float h = h2[(size_t)s * MLP_H + j];
#pragma unroll
        for (int o = 0; o < MLP_OUT; o++) acc[o] += h * __bfloat162float(w3[j * MLP_OUT + o]);
    }
#pragma unroll
    for (int o = 0; o < MLP_OUT; o++)
#pragma unroll
        for (int off = 16; off; off >>= 1) acc[o] += __shfl_xor_sync(0xffffffffu, acc[o], off);
    if (lane == 0) {
        float se = 0.f;
#pragma unroll
        for (int o = 0; o < MLP_OUT; o++) {
            float v = acc[o] + b3[o];
            y[s * MLP_OUT + o] = v;
            if (t) {
                float d = v - t[s * MLP_OUT + o];
                dy[s * MLP_OUT + o] = 2.f * d / (float)(n * MLP_OUT);
                se += d * d;
            }
        }
        if (t) atomicAdd(loss, se);
    }
}

// dW3[j][o] = sum_s h2[s][j] dy[s][o]; db3[o] = sum_s dy[s][o].
__global__ void k_grad_w3(const float *__restrict__ h2, const float *__restrict__ dy, int n, float *__restrict__ gw3,
                          float *__restrict__ gb3)
{
    int j = blockIdx.x;  // 0..MLP_H (MLP_H = bias row)
    int o = threadIdx.x & 3, part = threadIdx.x >> 2;  // 64 partial sums per output
    float acc = 0.f;
    for (int s = part; s < n; s += 64) acc += (j < MLP_H ? h2[(size_t)s * MLP_H + j] : 1.f) * dy[s * MLP_OUT + o];
    __shared__ float red[256];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int w = 128; w >= 4; w >>= 1) {
        if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x < 4) {
        if (j < MLP_H)
            gw3[j * MLP_OUT + threadIdx.x] = red[threadIdx.x];
        else
            gb3[threadIdx.x] = red[threadIdx.x];
    }
}

// dh2 = (dy . W3^T) * relu'(h2) in FP32 and BF16.
__global__ void k_back_h2(const float *__restrict__ dy, const __nv_bfloat16 *__restrict__ w3,
                          const float *__restrict__ h2, int n, float *__restrict__ dh2f,
                          __nv_bfloat16 *__restrict__ dh2b)
{
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (size_t)n * MLP_H) return;
    size_t s = i / MLP_H;
    int j = (int)(i % MLP_H);
    float g = 0.f;
#pragma unroll
    for (int o = 0; o < MLP_OUT; o++) g += dy[s * MLP_OUT + o] * __bfloat162float(w3[j * MLP_OUT + o]);
    g = h2[i] > 0.f ? g : 0.f;
    dh2f[i] = g;
    dh2b[i] = __float2bfloat16(g);
}

// Column sums of a [n x MLP_H] FP32 matrix (bias gradients).
__global__ void k_colsum(const float *__restrict__ m, int n, float *__restrict__ out)
{
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= MLP_H) return;
    float acc = 0.f;
    for (int s = 0; s < n; s++) acc += m[(size_t)s * MLP_H + j];
    out[j] = acc;
}

// dh1 (FP32, from the GEMM) masked by relu'(h1), then scattered into the
// active rows of dW1 (FP32 atomics) and summed into db1.
__global__ void k_back_l1(const int16_t *__restrict__ idx, const float *__restrict__ dh1raw,
                          const float *__restrict__ h1, int n, float *__restrict__ gw1, float *__restrict__ gb1)
{
    int s = blockIdx.x, j = threadIdx.x;
    if (s >= n) return;
    float g = dh1raw[(size_t)s * MLP_H + j];
    g = h1[(size_t)s * MLP_H + j] > 0.f ? g : 0.f;
    if (g == 0.f) return;
    atomicAdd(gb1 + j, g);
    const int16_t *a = idx + (size_t)s * MLP_MAX_ACTIVE;
    for (int k = 0; k < MLP_MAX_ACTIVE; k++) {
        int f = a[k];
        if (f < 0) break;
        atomicAdd(gw1 + (size_t)f * MLP_H + j, g);
    }
}

// Adam (Kingma and Ba 2015) on FP32 master weights; writes the BF16 copy.
__global__ void k_adam(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                       float *__restrict__ v, __nv_bfloat16 *__restrict__ pb, size_t n, float lr, float b1,
                       float b2, float eps, float c1, float c2)
{
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float gi = g[i];
    float mi = b1 * m[i] + (1.f - b1) * gi;
    float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    float upd = lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    float np = p[i] - upd;
    p[i] = np;
    if (pb) pb[i] = __float2bfloat16(np);
}

__global__ void k_to_bf16(const float *__restrict__ x, size_t n, __nv_bfloat16 *__restrict__ y)
{
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] = __float2bfloat16(x[i]);
}

}  // namespace pb
