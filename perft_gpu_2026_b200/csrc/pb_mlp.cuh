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
// and its two backward products run on the tcgen05 tensor cores (BF16
// operands, FP32 accumulation in tensor memory); layer 3 (256x4) is a
// per-sample dot product.
#pragma once
#include <cuda.h>  // CUtensorMap; the encoder is taken from the driver at run time
#include <cuda_bf16.h>

#include <algorithm>

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

// Training batch from the device-resident training set: row k of the batch
// is example order[b0 + k] (feature indices, 80 B, and targets, 16 B, as
// 16-byte vectors).
__global__ void k_gather_batch(const int16_t *__restrict__ all_idx, const float *__restrict__ all_t,
                               const int *__restrict__ order, int b0, int B, int16_t *__restrict__ idx,
                               float *__restrict__ t)
{
    static_assert(MLP_MAX_ACTIVE * sizeof(int16_t) % 16 == 0 && MLP_OUT * sizeof(float) == 16, "16-byte rows");
    constexpr int V = MLP_MAX_ACTIVE * (int)sizeof(int16_t) / 16;  // vectors per feature row
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= B * (V + 1)) return;
    const int k = i / (V + 1), v = i % (V + 1);
    const size_t src = (size_t)order[b0 + k];
    if (v < V)
        reinterpret_cast<uint4 *>(idx + (size_t)k * MLP_MAX_ACTIVE)[v] =
            reinterpret_cast<const uint4 *>(all_idx + src * MLP_MAX_ACTIVE)[v];
    else
        reinterpret_cast<float4 *>(t)[k] = reinterpret_cast<const float4 *>(all_t)[src];
}

// acc += loss * scale, in FP64 and in step order (one thread).
__global__ void k_accum_loss(const float *__restrict__ loss, double *__restrict__ acc, double scale)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) *acc += (double)*loss * scale;
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
// C[M x N] (FP32) = A[M x K] * B[K x N], BF16 operands, FP32 accumulation in
// tensor memory, on the 5th-generation tensor cores (tcgen05), operands
// brought into shared memory by the tensor memory accelerator (TMA).
//
// Element (m, k) of A is A[m*lda + k], or with TA A[k*lda + m]; element
// (k, n) of B is B[k*ldb + n], or with TB B[n*ldb + k].  M a multiple of 8
// (rows past M read as zero and are not stored), N of 128, K of 64; base
// addresses 16-byte aligned, lda and ldb multiples of 8.
//
// One CTA of 128 threads per 128 x 128 tile of C (and per K split, below).
// K advances 64 at a time through a ring of three shared-memory stages (two
// CTAs per SM).  Thread 0 keeps up to three chunks of both operands in
// flight with cp.async.bulk.tensor loads (each stage's mbarrier counts the
// bytes in),
// issues the four 128x128x16 tcgen05.mma of a chunk once its bytes have
// landed, and commits them to the stage's second mbarrier; after queueing a
// chunk's MMAs it waits on the previous chunk's commit and loads that stage
// again, so one chunk of MMAs is always queued while loads are issued.
// Each operand keeps the layout it has in global memory, as one of the two
// canonical 128-byte-swizzled layouts that TMA writes and the MMA reads: K-major for an operand contiguous along K
// (one 64 x 128 box: rows of 64 k, 8-row groups 1024 B apart; an MMA's
// 16-k step moves the start address 32 B) or MN-major for one contiguous
// along M or N (two 64 x 64 boxes of 64 k rows x 64 elements: 8-k groups
// 1024 B apart, the two 64-wide halves 8192 B apart; a 16-k step moves
// 2048 B); the instruction descriptor names which.  A last commit to a
// third mbarrier tells all four warps the accumulator (128 lanes x 128 FP32
// columns of tensor memory) is final; warp w reads rows 32w..32w+31 back.
//
// Few output tiles with a long K (the weight gradient: 256 x 256 over the
// batch) split K across gridDim.z CTAs per tile; each writes its partial
// tile to a workspace and k_sum_splits adds the splits in a fixed order, so
// results do not depend on scheduling.  Every mbarrier wait gives up after
// about a second, sets *err and skips the epilogue; the loads and MMAs
// still in flight are then waited for (bounded again) and tensor memory is
// freed on every path.
namespace tc {
#ifndef PB_GEMM_STAGES
// shared-memory stages of k_gemm_tc: 3 x 32 KB lets two CTAs share an SM, so
// one CTA's setup and epilogue overlap the other's MMAs (16384 x 1024 x 1024:
// 545 against 400 TFLOP/s with 4 stages and one CTA per SM)
#define PB_GEMM_STAGES 3
#endif
#define PB_GEMM_CTAS_PER_SM (PB_GEMM_STAGES <= 2 ? 3 : PB_GEMM_STAGES == 3 ? 2 : 1)
constexpr int BM = 128, BN = 128, BK = 64, STAGES = PB_GEMM_STAGES;
constexpr u32 OPERAND_BYTES = BM * BK * 2;         // one operand chunk, 16 KB
constexpr u32 STAGE_BYTES = 2 * OPERAND_BYTES;     // A chunk + B chunk
constexpr u32 SMEM_BYTES = STAGES * STAGE_BYTES + 1024;  // + slack to align the ring to 1024 B
constexpr u32 TMEM_COLS = 128;
constexpr int MAX_SPLITS = 16;

__device__ __forceinline__ u32 smem_addr(const void *p) { return (u32)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor, 128-byte swizzle (layout type 2 at bit
// 61), version 1 at bit 46.
__device__ __forceinline__ u64 smem_desc_sw128(u32 addr, u32 lbo, u32 sbo)
{
    return (u64)((addr & 0x3FFFFu) >> 4) | ((u64)(lbo >> 4) << 16) | ((u64)(sbo >> 4) << 32) | (1ull << 46) |
           (2ull << 61);
}

// Instruction descriptor, kind::f16: FP32 accumulator (bit 4), BF16 A and B
// (bits 7, 10), A / B MN-major (bits 15 / 16), N >> 3 at bit 17, M >> 4 at
// bit 24.
__host__ __device__ constexpr u32 instr_desc(int m, int n, bool a_mn, bool b_mn)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((u32)a_mn << 15) | ((u32)b_mn << 16) | ((u32)(n >> 3) << 17) |
           ((u32)(m >> 4) << 24);
}

__device__ __forceinline__ bool mbar_wait(u32 bar, u32 parity)
{
    const long long t0 = clock64();
    for (;;) {
        u32 done;
        asm volatile(
            "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
        if (clock64() - t0 > 2000000000ll) return false;
    }
}

// A 2-D TMA tile load of this CTA's own box into shared memory at `dst`, counted
// into mbarrier `bar`; x (the contiguous coordinate) a multiple of 64.
__device__ __forceinline__ void tma_load_2d(u32 dst, const CUtensorMap *map, int x, int y, u32 bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
        :: "r"(dst), "l"(reinterpret_cast<u64>(map)), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

// One operand chunk (64 k x 128 rows from row0, k from k0) into stage memory
// at `dst`.
template <bool KMAJOR>
__device__ __forceinline__ void load_operand(u32 dst, const CUtensorMap *map, int row0, int k0, u32 bar)
{
    if (KMAJOR) {
        tma_load_2d(dst, map, k0, row0, bar);
    } else {
        tma_load_2d(dst, map, row0, k0, bar);
        tma_load_2d(dst + OPERAND_BYTES / 2, map, row0 + 64, k0, bar);
    }
}

// Descriptor of the 16-k slice kk (0..3) of an operand chunk at `base`.
template <bool KMAJOR>
__device__ __forceinline__ u64 operand_desc(u32 base, int kk)
{
    return KMAJOR ? smem_desc_sw128(base + kk * 32, 16, 1024) : smem_desc_sw128(base + kk * 2048, 8192, 1024);
}
}  // namespace tc

// C (or, with gridDim.z > 1, split z's partial tile at C + z * split_stride)
// for the tile (blockIdx.y, blockIdx.x) over this split's share of K.
template <bool TA, bool TB>
__global__ void __launch_bounds__(128, PB_GEMM_CTAS_PER_SM) k_gemm_tc(const __grid_constant__ CUtensorMap map_a,
                                                     const __grid_constant__ CUtensorMap map_b,
                                                     float *__restrict__ C, int ldc, size_t split_stride, int M,
                                                     int N, int K, u32 *__restrict__ err)
{
    using namespace tc;
    constexpr bool A_KMAJOR = !TA, B_KMAJOR = TB;
    extern __shared__ __align__(1024) uint8_t smem[];
    __shared__ __align__(8) uint64_t full[STAGES], empty[STAGES], done;
    __shared__ u32 s_tmem;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    const int rows_a = min(BM, M - m0);
    const int nk = K / BK, splits = gridDim.z, z = blockIdx.z;
    const int kc0 = (int)((long long)z * nk / splits), kc1 = (int)((long long)(z + 1) * nk / splits);
    const int cnt = kc1 - kc0;
    C += (size_t)z * split_stride;
    // the stage ring, aligned to the 1024-byte swizzle atom
    const u32 ring = (smem_addr(smem) + 1023u) & ~1023u;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(smem_addr(&s_tmem)), "r"(TMEM_COLS) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int st = 0; st < STAGES; st++) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_addr(&full[st])) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_addr(&empty[st])) : "memory");
        }
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_addr(&done)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("prefetch.tensormap [%0];" :: "l"(reinterpret_cast<u64>(&map_a)) : "memory");
        asm volatile("prefetch.tensormap [%0];" :: "l"(reinterpret_cast<u64>(&map_b)) : "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const u32 tmem = s_tmem;

    bool ok = true;
    if (tid == 0 && cnt > 0) {
        const u32 idesc = instr_desc(BM, BN, !A_KMAJOR, !B_KMAJOR);
        auto issue = [&](int j) {
            const int st = j % STAGES;
            const u32 a = ring + st * STAGE_BYTES, b = a + OPERAND_BYTES, bar = smem_addr(&full[st]);
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(bar), "r"(STAGE_BYTES)
                         : "memory");
            load_operand<A_KMAJOR>(a, &map_a, m0, (kc0 + j) * BK, bar);
            load_operand<B_KMAJOR>(b, &map_b, n0, (kc0 + j) * BK, bar);
        };
        int issued = 0, landed = 0;  // chunks whose loads were issued / have landed
        for (; issued < cnt && issued < STAGES; issued++) issue(issued);
        for (int j = 0; j < cnt; j++) {
            const int st = j % STAGES;
            const u32 ph = (u32)(j / STAGES) & 1u;
            if (!mbar_wait(smem_addr(&full[st]), ph)) {
                ok = false;
                break;
            }
            landed = j + 1;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const u32 a = ring + st * STAGE_BYTES, b = a + OPERAND_BYTES;
#pragma unroll
            for (int kk = 0; kk < BK / 16; kk++) {
                const u64 da = operand_desc<A_KMAJOR>(a, kk), db = operand_desc<B_KMAJOR>(b, kk);
                const u32 acc = (j > 0 || kk > 0) ? 1u : 0u;
                asm volatile(
                    "{ .reg .pred p; setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p; }"
                    :: "r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0u) : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                         :: "r"(smem_addr(&empty[st])) : "memory");
            if (j >= 1 && j - 1 + STAGES < cnt) {
                // refill the previous chunk's stage once its MMAs have read
                // it; this chunk's MMAs stay queued behind them meanwhile, so
                // the tensor pipe does not drain while the loads are issued
                const int jp = j - 1;
                if (!mbar_wait(smem_addr(&empty[jp % STAGES]), (u32)(jp / STAGES) & 1u)) {
                    ok = false;
                    break;
                }
                issue(issued++);
            }
        }
        // covers every MMA issued before it
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                     :: "r"(smem_addr(&done)) : "memory");
        if (!ok) {
            // a wait gave up: before the CTA frees its memory, let the loads
            // still in flight land and the issued MMAs finish (each wait
            // bounded again)
            for (int j = landed; j < issued; j++) mbar_wait(smem_addr(&full[j % STAGES]), (u32)(j / STAGES) & 1u);
            mbar_wait(smem_addr(&done), 0);
        }
    }
    if (cnt > 0 && __syncthreads_and(ok)) ok = mbar_wait(smem_addr(&done), 0);
    ok = __syncthreads_and(ok) != 0;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (ok && cnt > 0) {
        const int row = warp * 32 + lane;
        float *out = C + (size_t)(m0 + row) * ldc + n0;
#pragma unroll 1
        for (int c = 0; c < BN; c += 32) {
            u32 v[32];
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
                "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
                "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
                : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
                  "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]),
                  "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]),
                  "=r"(v[22]), "=r"(v[23]), "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]),
                  "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
                : "r"(tmem + ((u32)(warp * 32) << 16) + (u32)c));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (row < rows_a) {
#pragma unroll
                for (int q = 0; q < 32; q += 4)
                    *reinterpret_cast<float4 *>(out + c + q) =
                        make_float4(__uint_as_float(v[q]), __uint_as_float(v[q + 1]), __uint_as_float(v[q + 2]),
                                    __uint_as_float(v[q + 3]));
            }
        }
    } else if (!ok && tid == 0) {
        atomicOr(err, 1u);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(TMEM_COLS) : "memory");
    }
}

// C[m][n] (row stride ldc) = the sum over z = 0..splits-1, in that order, of
// the partial tiles w[z][m][n] (M x N each).
__global__ void k_sum_splits(const float *__restrict__ w, int splits, int M, int N, float *__restrict__ C, int ldc)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x, mn = (size_t)M * N;
    if (i >= mn) return;
    float acc = 0.f;
    for (int z = 0; z < splits; z++) acc += w[z * mn + i];
    C[(i / N) * ldc + i % N] = acc;
}

// K splits for a product: only when the output has under 32 tiles, about
// four 64-wide K chunks per split, at most MAX_SPLITS, and only as many as
// `work_elems` floats of workspace hold.
inline int gemm_splits(int M, int N, int K, size_t work_elems)
{
    const int tiles = (N / tc::BN) * ((M + tc::BM - 1) / tc::BM), nk = K / tc::BK;
    if (tiles >= 32) return 1;
    int s = std::min(tc::MAX_SPLITS, std::max(1, nk / 4));
    while (s > 1 && (size_t)s * M * N > work_elems) s--;
    return s;
}

// The driver's tensor-map encoder, looked up once through the runtime (the
// library does not link the driver library itself).
typedef CUresult (*TensorMapEncodeTiled)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                         const cuuint64_t *, const cuuint32_t *, const cuuint32_t *,
                                         CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
                                         CUtensorMapFloatOOBfill);
inline TensorMapEncodeTiled tensor_map_encoder()
{
    static TensorMapEncodeTiled fn = [] {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            f = nullptr;
        return reinterpret_cast<TensorMapEncodeTiled>(f);
    }();
    return fn;
}

// Tensor map of a row-major BF16 matrix (`outer` rows of `inner` elements,
// `ld` elements apart) read in boxes of box_inner x box_outer with the
// 128-byte swizzle; boxes reaching past the matrix read zeros.
inline cudaError_t make_tensor_map(CUtensorMap *map, const __nv_bfloat16 *base, u64 inner, u64 outer, u64 ld,
                                   u32 box_inner, u32 box_outer)
{
    TensorMapEncodeTiled encode = tensor_map_encoder();
    if (!encode) return cudaErrorNotSupported;
    if ((reinterpret_cast<uintptr_t>(base) & 15) || (ld * 2) % 16) return cudaErrorInvalidValue;
    const cuuint64_t dims[2] = {inner, outer};
    const cuuint64_t strides[1] = {ld * 2};
    const cuuint32_t box[2] = {box_inner, box_outer};
    const cuuint32_t estr[2] = {1, 1};
    CUresult r = encode(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<__nv_bfloat16 *>(base), dims, strides,
                        box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

// Tensor map of one GEMM operand: `rows` (M or N) x K, K-major when the
// operand is contiguous along K (element (r, k) at p[r*ld + k]: boxes of 64 k
// x 128 rows), MN-major otherwise (element (r, k) at p[k*ld + r]: boxes of
// 64 rows x 64 k).
inline cudaError_t operand_map(CUtensorMap *map, const __nv_bfloat16 *p, bool kmajor, int rows, int K, int ld)
{
    return kmajor ? make_tensor_map(map, p, (u64)K, (u64)rows, (u64)ld, tc::BK, tc::BM)
                  : make_tensor_map(map, p, (u64)rows, (u64)K, (u64)ld, 64, tc::BK);
}

// Launches k_gemm_tc (see above for the operand layouts and size rules),
// split over K into `work` (work_elems floats) when gemm_splits says so.
template <bool TA, bool TB>
inline cudaError_t gemm_tc(const __nv_bfloat16 *A, int lda, const __nv_bfloat16 *B, int ldb, float *C, int ldc, int M,
                           int N, int K, u32 *err, float *work, size_t work_elems, cudaStream_t s)
{
    if (M <= 0 || M % 8 || N <= 0 || N % tc::BN || K <= 0 || K % tc::BK || lda % 8 || ldb % 8)
        return cudaErrorInvalidValue;
    CUtensorMap map_a, map_b;
    cudaError_t e = operand_map(&map_a, A, !TA, M, K, lda);
    if (e == cudaSuccess) e = operand_map(&map_b, B, TB, N, K, ldb);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_gemm_tc<TA, TB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tc::SMEM_BYTES);
    if (e != cudaSuccess) return e;
    const int splits = work ? gemm_splits(M, N, K, work_elems) : 1;
    dim3 grid(N / tc::BN, (M + tc::BM - 1) / tc::BM, splits);
    if (splits == 1) {
        k_gemm_tc<TA, TB><<<grid, 128, tc::SMEM_BYTES, s>>>(map_a, map_b, C, ldc, 0, M, N, K, err);
        return cudaGetLastError();
    }
    const size_t mn = (size_t)M * N;
    k_gemm_tc<TA, TB><<<grid, 128, tc::SMEM_BYTES, s>>>(map_a, map_b, work, N, mn, M, N, K, err);
    k_sum_splits<<<(unsigned)((mn + 255) / 256), 256, 0, s>>>(work, splits, M, N, C, ldc);
    return cudaGetLastError();
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
