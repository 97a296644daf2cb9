// pb_engine.cu - host driver and C ABI of the B200 perft engine.
//
// Single translation unit: the tables, the kernels and the host code are
// compiled together so the __device__ tables have one definition.
//
// Call structure (reference equivalents in brackets):
//   pb_create            device init, table upload, arena   [initGPU, initMoveGen]
//   pb_perft             per-depth loop over pb_perft_launch [perft.cu main loop]
//   pb_perft_launch      host recursion above the launch depth, host TT
//                        [perftLauncher / perft_cpu_recurse]
//   pb_perft_position    one GPU breadth-first perft          [perft_gpu_host_bfs]
//   pb_perft_cpu         host-only perft                     [perft_cpu_dispatch]
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include <nvtx3/nvToolsExt.h>
#include "../../include/perft_b200.h"
#include "pb_tables.cuh"
#include "pb_util.cuh"
#include "pb_kernels.cuh"
#include "pb_tt.cuh"
#include "pb_devtt.cuh"
#include "pb_mlp_host.cuh"

using namespace pb;

#define PB_VERSION "perft-b200 0.1"

namespace pb {
struct GraphPlan {
    u64 n = 0;
    int depth = 0;
    bool strict = false;
    int mode = 0;        // leaf mode (leaf_mode)
    bool queue = false;  // persistent work-queue leaf instead of the grid leaf
    std::vector<u64> caps;
    cudaGraphExec_t exec = nullptr;
    // device buffers inside the arena (fixed for the captured graph)
    Board *b0 = nullptr;
    uint8_t *s0 = nullptr;
    u32 *r0 = nullptr;
    unsigned long long *rc = nullptr;
    u64 *sizes = nullptr;
    bool same(u64 n_, int d_, bool s_, int mode_, bool queue_, const std::vector<u64> &c_) const
    {
        return exec && n == n_ && depth == d_ && strict == s_ && mode == mode_ && queue == queue_ && caps == c_;
    }
};

}  // namespace pb

struct pb_ctx {
    int device = -1;
    bool gpu = false;
    pb_opts opts{};
    cudaStream_t stream = nullptr;
    char *arena = nullptr;
    size_t arena_bytes = 0;
    // small device scratch: counter, error word, scan ticket, level total
    unsigned long long *d_counter = nullptr;
    u32 *d_err = nullptr;
    u32 *d_ticket = nullptr;
    u64 *d_total = nullptr;
    u64 *h_pinned = nullptr;  // pinned host words for readbacks
    int launch_depth = 0;
    bool timing = false;
    pb_tuning tuning{6, 0, 1024, 128, 2, 1, 1, 1, 2};
    int num_sms = 0;
    uint16_t *spill = nullptr;  // cooperative-leaf spill area (device)
    size_t spill_blocks = 0;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};  // call start, leaf start, leaf end, call end
    pb_stats stats{};
    HostTT htt;
    DeviceTT dtt;
    Mlp mlp;
    GraphPlan graph;
    int dtt_max_depth = 0;
    size_t dtt_free_bytes = 0;
    u32 dedup_gen = 0;
    int htt_last = 0;
    u64 tt_batch = 1;  // roots per batched table-mode call that fit last time
    std::string err;
};

namespace {

int fail(pb_ctx *ctx, int code, const std::string &msg)
{
    if (ctx) ctx->err = msg;
    return code;
}

int cuda_fail(pb_ctx *ctx, cudaError_t e, const char *what)
{
    return fail(ctx, PB_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

#define PB_CUDA(call)                                        \
    do {                                                     \
        cudaError_t e_ = (call);                             \
        if (e_ != cudaSuccess) return cuda_fail(ctx, e_, #call); \
    } while (0)

inline Board to_board(const pb_pos &p)
{
    Board b;
    for (int i = 0; i < 4; i++) b.bb[i] = p.bb[i];
    return b;
}
inline void to_pos(const Board &b, u32 st, int color, pb_pos &p)
{
    memset(&p, 0, sizeof(p));
    for (int i = 0; i < 4; i++) p.bb[i] = b.bb[i];
    p.state = (uint8_t)st;
    p.color = (uint8_t)color;
}

// ---------------------------------------------------------------- host core wrappers
u32 host_count(const Board &b, u32 st, int c, bool strict)
{
    if (c == WHITE) return strict ? count_moves<WHITE, true>(b, st) : count_moves<WHITE, false>(b, st);
    return strict ? count_moves<BLACK, true>(b, st) : count_moves<BLACK, false>(b, st);
}
int host_gen(const Board &b, u32 st, int c, uint16_t *out)
{
    ArraySink s{out, 0};
    if (c == WHITE)
        gen_moves<WHITE>(b, st, s);
    else
        gen_moves<BLACK>(b, st, s);
    return s.n;
}
void host_make(Board &b, u32 &st, int c, uint16_t m)
{
    if (c == WHITE)
        make_move<WHITE>(b, st, m);
    else
        make_move<BLACK>(b, st, m);
}

u64 host_perft(const Board &b, u32 st, int c, int depth, bool strict)
{
    if (depth <= 0) return 1;
    if (depth == 1) return host_count(b, st, c, strict);
    uint16_t mv[MAX_MOVES];
    int n = host_gen(b, st, c, mv);
    u64 total = 0;
    for (int i = 0; i < n; i++) {
        Board cb = b;
        u32 cs = st;
        host_make(cb, cs, c, mv[i]);
        total += host_perft(cb, cs, 1 - c, depth - 1, strict);
    }
    return total;
}

// ---------------------------------------------------------------- arena
struct Arena {
    char *base;
    size_t cap, off = 0;
    template <class T> T *take(u64 n)
    {
        size_t bytes = ((size_t)n * sizeof(T) + 255) & ~(size_t)255;
        if (off + bytes > cap) return nullptr;
        T *p = reinterpret_cast<T *>(base + off);
        off += bytes;
        return p;
    }
};

inline unsigned grid_for(u64 n, int threads) { return (unsigned)((n + threads - 1) / threads); }

// Leaf mode of the batched, planned and table leaves (grandchild_counts):
// 3 for leaf kernel 6 (ranked, listed pieces, balanced warps), 2 for 5
// (ranked, listed pieces), 1 for 4 (ranked), else 0.
inline int leaf_mode(const pb_ctx *ctx)
{
    return ctx->tuning.leaf_kernel == 6 ? 3 : ctx->tuning.leaf_kernel == 5 ? 2 : ctx->tuning.leaf_kernel == 4 ? 1 : 0;
}

// CTA size of a balanced leaf over n edges (PB_BALANCED_K per thread): the
// tuned size, halved down to 256 while the grid would have fewer than 8 CTAs
// per SM (a small launch of big CTAs leaves its last wave half empty).
inline int balanced_threads(const pb_ctx *ctx, u64 n, int tuned)
{
    int t = tuned;
    while (t > 256 && n < (u64)PB_BALANCED_K * (u64)t * 8u * (u64)ctx->num_sms) t /= 2;
    return t;
}
// Below this many edges even 256-thread balanced CTAs would not give every SM
// 8 of them: such small leaves run one edge per thread (the listed leaf) so
// the launch still covers the GPU (one perft-5 root has about 3e4 edges).
inline bool balanced_fits(const pb_ctx *ctx, u64 n)
{
    return n >= (u64)PB_BALANCED_K * 256u * 8u * (u64)ctx->num_sms;
}

// NVTX range for profilers (header-only NVTX v3: free unless a tool attaches):
// marks each BFS pass, level and leaf launch on the host timeline, so a
// capture can select kernels by phase (ncu --nvtx --nvtx-include).
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange &) = delete;
    NvtxRange &operator=(const NvtxRange &) = delete;
};

enum { BFS_OK = 0, BFS_TOO_BIG = 1 };

template <int C, bool S>
int launch_leaf_t(pb_ctx *ctx, const Board *b, const uint8_t *st, const u32 *pi, const uint16_t *mv, u64 n, u64 npar)
{
    cudaStream_t s = ctx->stream;
    if (ctx->tuning.leaf_fuse == 1) {
        k_leaf1<C, S><<<grid_for(n, 256), 256, 0, s>>>(b, st, pi, mv, n, npar, ctx->d_counter);
        PB_CUDA(cudaGetLastError());
        return PB_OK;
    }
    if (ctx->tuning.leaf_kernel == 3) {
        switch (ctx->tuning.leaf_threads) {
        case 128: k_leaf2_defer<C, S, 128><<<grid_for(n, 128), 128, 0, s>>>(b, st, pi, mv, n, npar, ctx->d_counter); break;
        default: k_leaf2_defer<C, S, 256><<<grid_for(n, 256), 256, 0, s>>>(b, st, pi, mv, n, npar, ctx->d_counter); break;
        }
        PB_CUDA(cudaGetLastError());
        return PB_OK;
    }
    if (ctx->tuning.leaf_kernel == 6 && balanced_fits(ctx, n)) {
        // PB_BALANCED_K edges per thread
        const int lt = balanced_threads(ctx, n, ctx->tuning.leaf_threads);
        const u64 per = (u64)PB_BALANCED_K * (u64)lt;
        const unsigned g = (unsigned)((n + per - 1) / per);
        switch (lt) {
        case 128: k_leaf2_balanced<C, S, 128><<<g, 128, 0, s>>>(b, st, pi, mv, n, npar, ctx->d_counter); break;
        case 512: k_leaf2_balanced<C, S, 512><<<g, 512, 0, s>>>(b, st, pi, mv, n, npar, ctx->d_counter); break;
        case 1024: k_leaf2_balanced<C, S, 1024><<<g, 1024, 0, s>>>(b, st, pi, mv, n, npar, ctx->d_counter); break;
        default: k_leaf2_balanced<C, S, 256><<<g, 256, 0, s>>>(b, st, pi, mv, n, npar, ctx->d_counter); break;
        }
        PB_CUDA(cudaGetLastError());
        return PB_OK;
    }
    if (ctx->tuning.leaf_kernel == 5 || ctx->tuning.leaf_kernel == 6) {
        switch (ctx->tuning.leaf_kernel == 6 ? 256 : ctx->tuning.leaf_threads) {
        case 128: k_leaf2_listed<C, S, 128><<<grid_for(n, 128), 128, 0, s>>>(b, st, pi, mv, n, npar, ctx->d_counter); break;
        case 512: k_leaf2_listed<C, S, 512><<<grid_for(n, 512), 512, 0, s>>>(b, st, pi, mv, n, npar, ctx->d_counter); break;
        default: k_leaf2_listed<C, S, 256><<<grid_for(n, 256), 256, 0, s>>>(b, st, pi, mv, n, npar, ctx->d_counter); break;
        }
        PB_CUDA(cudaGetLastError());
        return PB_OK;
    }
    if (ctx->tuning.leaf_kernel == 4) {
        switch (ctx->tuning.leaf_threads) {
        case 128: k_leaf2_sorted<C, S, 128><<<grid_for(n, 128), 128, 0, s>>>(b, st, pi, mv, n, npar, ctx->d_counter); break;
        case 512: k_leaf2_sorted<C, S, 512><<<grid_for(n, 512), 512, 0, s>>>(b, st, pi, mv, n, npar, ctx->d_counter); break;
        default: k_leaf2_sorted<C, S, 256><<<grid_for(n, 256), 256, 0, s>>>(b, st, pi, mv, n, npar, ctx->d_counter); break;
        }
        PB_CUDA(cudaGetLastError());
        return PB_OK;
    }
    if (ctx->tuning.leaf_kernel == 1) {
        switch (ctx->tuning.leaf_threads) {
        case 128: k_leaf2<C, S, 128><<<grid_for(n, 128), 128, 0, s>>>(b, st, pi, mv, n, npar, ctx->d_counter); break;
        case 512: k_leaf2<C, S, 512><<<grid_for(n, 512), 512, 0, s>>>(b, st, pi, mv, n, npar, ctx->d_counter); break;
        default: k_leaf2<C, S, 256><<<grid_for(n, 256), 256, 0, s>>>(b, st, pi, mv, n, npar, ctx->d_counter); break;
        }
        PB_CUDA(cudaGetLastError());
        return PB_OK;
    }
    u64 nchunks = (n + LEAF_T - 1) / LEAF_T;
    int per_sm = ctx->tuning.leaf_blocks_per_sm;
    if (per_sm <= 0) {
        PB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_leaf2_coop<C, S>, LEAF_T, 0));
        if (per_sm <= 0) per_sm = 1;
    }
    u64 grid = std::min<u64>(nchunks, (u64)ctx->num_sms * per_sm);
    if (grid > ctx->spill_blocks) return fail(ctx, PB_ERR_NOMEM, "leaf spill area too small");
    k_leaf2_coop<C, S><<<(unsigned)grid, LEAF_T, 0, s>>>(b, st, pi, mv, n, npar, ctx->spill, ctx->d_counter);
    PB_CUDA(cudaGetLastError());
    return PB_OK;
}

int launch_leaf(pb_ctx *ctx, int c, bool strict, const Board *b, const uint8_t *st, const u32 *pi,
                const uint16_t *mv, u64 n, u64 npar)
{
    if (c == WHITE) return strict ? launch_leaf_t<WHITE, true>(ctx, b, st, pi, mv, n, npar)
                                  : launch_leaf_t<WHITE, false>(ctx, b, st, pi, mv, n, npar);
    return strict ? launch_leaf_t<BLACK, true>(ctx, b, st, pi, mv, n, npar)
                  : launch_leaf_t<BLACK, false>(ctx, b, st, pi, mv, n, npar);
}

// Staged generation with the tuned CTA size.
void launch_generate(pb_ctx *ctx, int c, const Board *b, const uint8_t *st, const u64 *offs, u64 n, uint16_t *mv,
                     u32 *pi)
{
    cudaStream_t s = ctx->stream;
    if (ctx->tuning.gen_threads == 64) {
        if (c == WHITE) k_generate<WHITE, 64><<<grid_for(n, 64), 64, 0, s>>>(b, st, offs, ctx->d_total, n, mv, pi, ctx->d_err);
        else k_generate<BLACK, 64><<<grid_for(n, 64), 64, 0, s>>>(b, st, offs, ctx->d_total, n, mv, pi, ctx->d_err);
    } else {
        if (c == WHITE) k_generate<WHITE, 128><<<grid_for(n, 128), 128, 0, s>>>(b, st, offs, ctx->d_total, n, mv, pi, ctx->d_err);
        else k_generate<BLACK, 128><<<grid_for(n, 128), 128, 0, s>>>(b, st, offs, ctx->d_total, n, mv, pi, ctx->d_err);
    }
}

// One GPU breadth-first perft; status BFS_TOO_BIG when a level would not fit.
int bfs_perft(pb_ctx *ctx, const Board &root, u32 root_st, int color, int depth, u64 *out, int *bfs_status)
{
    NvtxRange nvtx_pass("bfs_perft");
    *bfs_status = BFS_OK;
    const bool strict = ctx->opts.strict != 0;
    if (depth <= 2) {
        *out = host_perft(root, root_st, color, depth, strict);
        return PB_OK;
    }
    uint16_t root_moves[MAX_MOVES];
    int n0 = host_gen(root, root_st, color, root_moves);
    if (n0 == 0) {
        *out = 0;
        return PB_OK;
    }
    cudaStream_t s = ctx->stream;
    pb_stats &stats = ctx->stats;
    Arena ar{ctx->arena, ctx->arena_bytes};
    Board *pb_ = ar.take<Board>(1);
    uint8_t *ps = ar.take<uint8_t>(1);
    uint16_t *emv = ar.take<uint16_t>(n0);
    u32 *epi = ar.take<u32>(n0);
    if (!pb_ || !ps || !emv || !epi) {
        *bfs_status = BFS_TOO_BIG;
        return PB_OK;
    }
    uint8_t st8 = (uint8_t)root_st;
    PB_CUDA(cudaMemcpyAsync(pb_, &root, sizeof(Board), cudaMemcpyHostToDevice, s));
    PB_CUDA(cudaMemcpyAsync(ps, &st8, 1, cudaMemcpyHostToDevice, s));
    PB_CUDA(cudaMemcpyAsync(emv, root_moves, sizeof(uint16_t) * n0, cudaMemcpyHostToDevice, s));
    PB_CUDA(cudaMemsetAsync(epi, 0, sizeof(u32) * n0, s));
    PB_CUDA(cudaMemsetAsync(ctx->d_err, 0, sizeof(u32), s));
    stats.h2d_bytes += sizeof(Board) + 1 + sizeof(uint16_t) * n0;
    if (stats.levels < 16) stats.level_sizes[stats.levels] = (u64)n0;
    if (ctx->timing) PB_CUDA(cudaEventRecord(ctx->ev[0], s));

    Board *cur_b = pb_;
    uint8_t *cur_s = ps;
    u64 n = (u64)n0;
    u64 n_par = 1;  // positions the current edges point into
    int c = color;
    const int fuse = ctx->tuning.leaf_fuse == 1 ? 1 : 2;
    for (int rem = depth - 1; rem > fuse; rem--) {
        Board *cb = ar.take<Board>(n);
        uint8_t *cs = ar.take<uint8_t>(n);
        u32 *cnt = ar.take<u32>(n);
        u64 *offs = ar.take<u64>(n);
        u64 tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
        u64 *status = ar.take<u64>(tiles);
        if (!cb || !cs || !cnt || !offs || !status) {
            *bfs_status = BFS_TOO_BIG;
            return PB_OK;
        }
        if (c == WHITE)
            k_expand_count<WHITE><<<grid_for(n, 256), 256, 0, s>>>(cur_b, cur_s, epi, emv, n, n_par, cb, cs, cnt, ctx->d_err);
        else
            k_expand_count<BLACK><<<grid_for(n, 256), 256, 0, s>>>(cur_b, cur_s, epi, emv, n, n_par, cb, cs, cnt, ctx->d_err);
        PB_CUDA(cudaGetLastError());
        PB_CUDA(cudaMemsetAsync(status, 0, sizeof(u64) * tiles, s));
        PB_CUDA(cudaMemsetAsync(ctx->d_ticket, 0, sizeof(u32), s));
        k_scan<<<(unsigned)tiles, SCAN_THREADS, 0, s>>>(cnt, n, offs, status, ctx->d_ticket, ctx->d_total, ctx->d_err);
        PB_CUDA(cudaGetLastError());
        PB_CUDA(cudaMemcpyAsync(ctx->h_pinned, ctx->d_total, sizeof(u64), cudaMemcpyDeviceToHost, s));
        PB_CUDA(cudaMemcpyAsync(ctx->h_pinned + 1, ctx->d_err, sizeof(u32), cudaMemcpyDeviceToHost, s));
        PB_CUDA(cudaStreamSynchronize(s));
        stats.kernels += 2;
        stats.d2h_bytes += 12;
        if ((u32)ctx->h_pinned[1]) return fail(ctx, PB_ERR_DEVICE, "scan reported a device error");
        u64 next = ctx->h_pinned[0];
        stats.levels++;
        if (stats.levels < 16) stats.level_sizes[stats.levels] = next;
        if (next == 0) {
            *out = 0;
            return PB_OK;
        }
        if (next > 0xFFFFFFFFULL) {  // parent indices are u32
            *bfs_status = BFS_TOO_BIG;
            return PB_OK;
        }
        uint16_t *nmv = ar.take<uint16_t>(next);
        u32 *npi = ar.take<u32>(next);
        if (!nmv || !npi) {
            *bfs_status = BFS_TOO_BIG;
            return PB_OK;
        }
        launch_generate(ctx, 1 - c, cb, cs, offs, n, nmv, npi);
        PB_CUDA(cudaGetLastError());
        stats.kernels += 1;
        cur_b = cb;
        cur_s = cs;
        emv = nmv;
        epi = npi;
        n_par = n;
        n = next;
        c = 1 - c;
    }
    PB_CUDA(cudaMemsetAsync(ctx->d_counter, 0, 2 * sizeof(unsigned long long), s));
    if (ctx->timing) PB_CUDA(cudaEventRecord(ctx->ev[1], s));
    int rc;
    {
        NvtxRange nvtx_leaf("leaf");
        rc = launch_leaf(ctx, c, strict, cur_b, cur_s, epi, emv, n, n_par);
    }
    if (rc != PB_OK) return rc;
    PB_CUDA(cudaGetLastError());
    if (ctx->timing) {
        PB_CUDA(cudaEventRecord(ctx->ev[2], s));
        PB_CUDA(cudaEventRecord(ctx->ev[3], s));
    }
    PB_CUDA(cudaMemcpyAsync(ctx->h_pinned, ctx->d_counter, 2 * sizeof(u64), cudaMemcpyDeviceToHost, s));
    PB_CUDA(cudaMemcpyAsync(ctx->h_pinned + 2, ctx->d_err, sizeof(u32), cudaMemcpyDeviceToHost, s));
    PB_CUDA(cudaStreamSynchronize(s));
    if ((u32)ctx->h_pinned[2]) return fail(ctx, PB_ERR_DEVICE, "kernel reported a device error");
    *out = ctx->h_pinned[0];
    stats.kernels += 1;
    stats.leaf_edges += n;
    stats.leaf_positions += ctx->h_pinned[1];
    stats.d2h_bytes += 20;
    if (ctx->timing) {
        float a = 0, b2 = 0;
        PB_CUDA(cudaEventElapsedTime(&a, ctx->ev[0], ctx->ev[3]));
        PB_CUDA(cudaEventElapsedTime(&b2, ctx->ev[1], ctx->ev[2]));
        stats.device_ms += a;
        stats.leaf_ms += b2;
    }
    return PB_OK;
}

// Device tables for remaining depths 2..max_r (allocated on first use, kept
// for the context's lifetime like the reference's initTT).
int ensure_dtt(pb_ctx *ctx, int max_r)
{
    if (max_r < 3) max_r = 3;
    if (ctx->dtt.ready() && ctx->dtt_max_depth >= max_r) return PB_OK;
    // (re)size for depths 2..max_r; a deeper call than prepared drops the
    // current contents, which only costs hits
    ctx->dtt.buckets = ctx->tuning.tt_replace == 2 ? 1 : 0;
    ctx->dtt.init(ctx->opts.device_tt_mb, ctx->dtt_free_bytes, max_r, ctx->opts.verbose, &ctx->err);
    ctx->dtt_max_depth = max_r;
    return PB_OK;
}

struct TTLevel {
    Hash128 *hash;
    u32 *counts;
    u64 *vals;
    uint8_t *flags;
    u32 *redirect;
    u64 *offs;
    u64 n;
    int rem;
};

// The persistent table leaf: one CTA per resident slot, at most one per T edges.
template <int C, bool S, int MODE>
int launch_tt_fill_t(pb_ctx *ctx, const Board *b, const uint8_t *st, const Hash128 *h, const u32 *pi,
                     const uint16_t *mv, u64 n, u64 npar, TTView tv, u32 *out, unsigned long long *cursor)
{
    int per_sm = 0;
    PB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_leaf2_tt_fill<C, S, MODE>, PB_LEAF_THREADS, 0));
    if (per_sm <= 0) per_sm = 1;
    const u64 grid = std::min<u64>((u64)ctx->num_sms * per_sm, (n + PB_LEAF_THREADS - 1) / PB_LEAF_THREADS);
    k_leaf2_tt_fill<C, S, MODE><<<(unsigned)grid, PB_LEAF_THREADS, 0, ctx->stream>>>(b, st, h, pi, mv, n, npar, tv, out,
                                                                                     cursor, ctx->d_counter);
    PB_CUDA(cudaGetLastError());
    return PB_OK;
}
int launch_tt_fill(pb_ctx *ctx, int c, bool strict, int mode, const Board *b, const uint8_t *st, const Hash128 *h,
                   const u32 *pi, const uint16_t *mv, u64 n, u64 npar, TTView tv, u32 *out,
                   unsigned long long *cursor)
{
#define PB_FILL(CC, SS, MM) return launch_tt_fill_t<CC, SS, MM>(ctx, b, st, h, pi, mv, n, npar, tv, out, cursor)
    if (c == WHITE) {
        if (strict) {
            if (mode == 2) PB_FILL(WHITE, true, 2);
            PB_FILL(WHITE, true, 1);
        }
        if (mode == 2) PB_FILL(WHITE, false, 2);
        PB_FILL(WHITE, false, 1);
    }
    if (strict) {
        if (mode == 2) PB_FILL(BLACK, true, 2);
        PB_FILL(BLACK, true, 1);
    }
    if (mode == 2) PB_FILL(BLACK, false, 2);
    PB_FILL(BLACK, false, 1);
#undef PB_FILL
}

// GPU breadth-first perft with the device TTs (perft_gpu_host_bfs with
// g_useTT, perft_kernels.cu:620-990) of n roots of one colour at once: probe
// at every level, dedup (across all the roots' subtrees of a level), leaf TT,
// then the upsweep stores every level's counts and a last upsweep over the
// roots' own moves gives each root's count.  out[k] = perft(depth) of root k.
int bfs_tt_roots(pb_ctx *ctx, const Board *rb, const uint8_t *rs, const Hash128 *rh, u64 nroots, int color,
                 int depth, u64 *out, int *bfs_status)
{
    NvtxRange nvtx_pass("bfs_perft_tt");
    *bfs_status = BFS_OK;
    const bool strict = ctx->opts.strict != 0;
    if (nroots == 0) return PB_OK;
    if (depth <= 2) {
        for (u64 k = 0; k < nroots; k++) out[k] = host_perft(rb[k], rs[k], color, depth, strict);
        return PB_OK;
    }
    int rc = ensure_dtt(ctx, depth - 1);
    if (rc != PB_OK) return rc;
    cudaStream_t s = ctx->stream;
    pb_stats &stats = ctx->stats;
    Arena ar{ctx->arena, ctx->arena_bytes};
    Board *pb_ = ar.take<Board>(nroots);
    uint8_t *ps = ar.take<uint8_t>(nroots);
    Hash128 *ph = ar.take<Hash128>(nroots);
    u32 *rcnt = ar.take<u32>(nroots);       // root move counts
    u64 *roff = ar.take<u64>(nroots);       // root edge offsets
    uint8_t *rflags = ar.take<uint8_t>(nroots);
    u64 *rvals = ar.take<u64>(nroots);
    if (!pb_ || !ps || !ph || !rcnt || !roff || !rflags || !rvals) {
        *bfs_status = BFS_TOO_BIG;
        return PB_OK;
    }
    std::vector<uint8_t> st8(rs, rs + nroots);
    PB_CUDA(cudaMemcpyAsync(pb_, rb, sizeof(Board) * nroots, cudaMemcpyHostToDevice, s));
    PB_CUDA(cudaMemcpyAsync(ps, st8.data(), nroots, cudaMemcpyHostToDevice, s));
    PB_CUDA(cudaMemcpyAsync(ph, rh, sizeof(Hash128) * nroots, cudaMemcpyHostToDevice, s));
    PB_CUDA(cudaMemsetAsync(rflags, 0, nroots, s));
    PB_CUDA(cudaMemsetAsync(ctx->d_err, 0, sizeof(u32), s));
    stats.h2d_bytes += (sizeof(Board) + 1 + sizeof(Hash128)) * nroots;
    if (ctx->timing) PB_CUDA(cudaEventRecord(ctx->ev[0], s));

    // the roots' moves: from the host for one root, else counted, scanned and
    // generated on the device like every other level
    uint16_t *emv = nullptr;
    u32 *epi = nullptr;
    u64 n = 0;
    if (nroots == 1) {
        uint16_t root_moves[MAX_MOVES];
        int n0 = host_gen(rb[0], rs[0], color, root_moves);
        n = (u64)n0;
        emv = ar.take<uint16_t>(n ? n : 1);
        epi = ar.take<u32>(n ? n : 1);
        if (!emv || !epi) {
            *bfs_status = BFS_TOO_BIG;
            return PB_OK;
        }
        u32 c0 = (u32)n0;
        u64 z = 0;
        PB_CUDA(cudaMemcpyAsync(rcnt, &c0, sizeof(u32), cudaMemcpyHostToDevice, s));
        PB_CUDA(cudaMemcpyAsync(roff, &z, sizeof(u64), cudaMemcpyHostToDevice, s));
        if (n) {
            PB_CUDA(cudaMemcpyAsync(emv, root_moves, sizeof(uint16_t) * n, cudaMemcpyHostToDevice, s));
            PB_CUDA(cudaMemsetAsync(epi, 0, sizeof(u32) * n, s));
        }
        stats.h2d_bytes += sizeof(uint16_t) * n + 12;
    } else {
        u64 tiles0 = (nroots + SCAN_TILE - 1) / SCAN_TILE;
        u64 *status0 = ar.take<u64>(tiles0);
        if (!status0) {
            *bfs_status = BFS_TOO_BIG;
            return PB_OK;
        }
        if (color == WHITE)
            k_count_positions<WHITE, true><<<grid_for(nroots, 256), 256, 0, s>>>(pb_, ps, nroots, rcnt);
        else
            k_count_positions<BLACK, true><<<grid_for(nroots, 256), 256, 0, s>>>(pb_, ps, nroots, rcnt);
        PB_CUDA(cudaMemsetAsync(status0, 0, sizeof(u64) * tiles0, s));
        PB_CUDA(cudaMemsetAsync(ctx->d_ticket, 0, sizeof(u32), s));
        k_scan<<<(unsigned)tiles0, SCAN_THREADS, 0, s>>>(rcnt, nroots, roff, status0, ctx->d_ticket, ctx->d_total,
                                                          ctx->d_err);
        PB_CUDA(cudaGetLastError());
        PB_CUDA(cudaMemcpyAsync(ctx->h_pinned, ctx->d_total, sizeof(u64), cudaMemcpyDeviceToHost, s));
        PB_CUDA(cudaStreamSynchronize(s));
        stats.kernels += 2;
        stats.d2h_bytes += 8;
        n = ctx->h_pinned[0];
        if (n > 0xFFFFFFFFULL) {
            *bfs_status = BFS_TOO_BIG;
            return PB_OK;
        }
        emv = ar.take<uint16_t>(n ? n : 1);
        epi = ar.take<u32>(n ? n : 1);
        if (!emv || !epi) {
            *bfs_status = BFS_TOO_BIG;
            return PB_OK;
        }
        if (n) {
            launch_generate(ctx, color, pb_, ps, roff, nroots, emv, epi);
            PB_CUDA(cudaGetLastError());
            stats.kernels += 1;
        }
    }

    std::vector<TTLevel> levels;
    Board *cur_b = pb_;
    uint8_t *cur_s = ps;
    Hash128 *cur_h = ph;
    u64 n_par = nroots;
    int c = color;
    for (int rem = depth - 1; rem > 2 && n; rem--) {
        TTLevel L{};
        Board *cb = ar.take<Board>(n);
        uint8_t *cs = ar.take<uint8_t>(n);
        L.hash = ar.take<Hash128>(n);
        L.counts = ar.take<u32>(n);
        L.vals = ar.take<u64>(n);
        L.flags = ar.take<uint8_t>(n);
        L.redirect = ar.take<u32>(n);
        L.offs = ar.take<u64>(n);
        u64 dsz = 1;
        while (dsz < 2 * n) dsz *= 2;
        unsigned long long *slots = ar.take<unsigned long long>(dsz);
        u64 tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
        u64 *status = ar.take<u64>(tiles);
        if (!cb || !cs || !L.hash || !L.counts || !L.vals || !L.flags || !L.redirect || !L.offs || !slots || !status) {
            *bfs_status = BFS_TOO_BIG;
            return PB_OK;
        }
        L.n = n;
        L.rem = rem;
        TTView tv = ctx->dtt.at(rem);
        unsigned g = grid_for(n, 256);
        if (c == WHITE)
            k_expand_count_tt<WHITE><<<g, 256, 0, s>>>(cur_b, cur_s, cur_h, epi, emv, n, n_par, tv, cb, cs, L.hash,
                                                       L.counts, L.vals, L.flags, ctx->d_err);
        else
            k_expand_count_tt<BLACK><<<g, 256, 0, s>>>(cur_b, cur_s, cur_h, epi, emv, n, n_par, tv, cb, cs, L.hash,
                                                       L.counts, L.vals, L.flags, ctx->d_err);
        PB_CUDA(cudaGetLastError());
        PB_CUDA(cudaMemsetAsync(slots, 0, sizeof(unsigned long long) * dsz, s));
        u32 gen = ++ctx->dedup_gen;
        k_dedup_claim<<<g, 256, 0, s>>>(L.hash, L.flags, n, slots, dsz - 1, gen);
        k_dedup_resolve<<<g, 256, 0, s>>>(L.hash, L.flags, n, slots, dsz - 1, gen, L.counts, L.redirect);
        PB_CUDA(cudaGetLastError());
        PB_CUDA(cudaMemsetAsync(status, 0, sizeof(u64) * tiles, s));
        PB_CUDA(cudaMemsetAsync(ctx->d_ticket, 0, sizeof(u32), s));
        k_scan<<<(unsigned)tiles, SCAN_THREADS, 0, s>>>(L.counts, n, L.offs, status, ctx->d_ticket, ctx->d_total,
                                                         ctx->d_err);
        PB_CUDA(cudaGetLastError());
        PB_CUDA(cudaMemcpyAsync(ctx->h_pinned, ctx->d_total, sizeof(u64), cudaMemcpyDeviceToHost, s));
        PB_CUDA(cudaMemcpyAsync(ctx->h_pinned + 1, ctx->d_err, sizeof(u32), cudaMemcpyDeviceToHost, s));
        PB_CUDA(cudaStreamSynchronize(s));
        stats.kernels += 4;
        stats.d2h_bytes += 12;
        if ((u32)ctx->h_pinned[1]) return fail(ctx, PB_ERR_DEVICE, "TT level reported a device error");
        u64 next = ctx->h_pinned[0];
        stats.levels++;
        if (stats.levels < 16) stats.level_sizes[stats.levels] = next;
        levels.push_back(L);
        cur_b = cb;
        cur_s = cs;
        cur_h = L.hash;
        n_par = n;
        c = 1 - c;
        if (next == 0) {
            n = 0;
            break;
        }
        if (next > 0xFFFFFFFFULL) {
            *bfs_status = BFS_TOO_BIG;
            return PB_OK;
        }
        uint16_t *nmv = ar.take<uint16_t>(next);
        u32 *npi = ar.take<u32>(next);
        if (!nmv || !npi) {
            *bfs_status = BFS_TOO_BIG;
            return PB_OK;
        }
        if (c == WHITE)
            k_generate<WHITE><<<grid_for(n_par, GEN_THREADS), GEN_THREADS, 0, s>>>(cb, cs, L.offs, ctx->d_total, n_par,
                                                                                   nmv, npi, ctx->d_err);
        else
            k_generate<BLACK><<<grid_for(n_par, GEN_THREADS), GEN_THREADS, 0, s>>>(cb, cs, L.offs, ctx->d_total, n_par,
                                                                                   nmv, npi, ctx->d_err);
        PB_CUDA(cudaGetLastError());
        stats.kernels += 1;
        emv = nmv;
        epi = npi;
        n = next;
    }
    // leaf: per-edge perft(2) with the depth-2 table
    u32 *leafcnt = ar.take<u32>(n > 0 ? n : 1);
    unsigned long long *cursor = ar.take<unsigned long long>(1);
    if (!leafcnt || !cursor) {
        *bfs_status = BFS_TOO_BIG;
        return PB_OK;
    }
    PB_CUDA(cudaMemsetAsync(ctx->d_counter, 0, 2 * sizeof(unsigned long long), s));
    if (ctx->timing) PB_CUDA(cudaEventRecord(ctx->ev[1], s));
    if (n > 0 && leaf_mode(ctx) >= 1 && ctx->tuning.tt_leaf == 2) {
        PB_CUDA(cudaMemsetAsync(cursor, 0, sizeof(unsigned long long), s));
        int rc2 = launch_tt_fill(ctx, c, strict, std::min(leaf_mode(ctx), 2), cur_b, cur_s, cur_h, epi, emv, n,
                                 n_par, ctx->dtt.at(2), leafcnt, cursor);
        if (rc2 != PB_OK) return rc2;
        stats.kernels += 1;
    } else if (n > 0) {
        TTView tv = ctx->dtt.at(2);
        unsigned g = grid_for(n, PB_LEAF_THREADS);
        const int mode = std::min(leaf_mode(ctx), 2);
#define PB_TT_LEAF(CC, SS)                                                                                     \
    if (mode == 2)                                                                                             \
        k_leaf2_tt<CC, SS, 2><<<g, PB_LEAF_THREADS, 0, s>>>(cur_b, cur_s, cur_h, epi, emv, n, n_par, tv,        \
                                                            leafcnt, ctx->d_counter);                         \
    else if (mode == 1)                                                                                        \
        k_leaf2_tt<CC, SS, 1><<<g, PB_LEAF_THREADS, 0, s>>>(cur_b, cur_s, cur_h, epi, emv, n, n_par, tv,        \
                                                            leafcnt, ctx->d_counter);                         \
    else                                                                                                       \
        k_leaf2_tt<CC, SS, 0><<<g, PB_LEAF_THREADS, 0, s>>>(cur_b, cur_s, cur_h, epi, emv, n, n_par, tv,        \
                                                            leafcnt, ctx->d_counter);
        if (c == WHITE) {
            if (strict) {
                PB_TT_LEAF(WHITE, true)
            } else {
                PB_TT_LEAF(WHITE, false)
            }
        } else {
            if (strict) {
                PB_TT_LEAF(BLACK, true)
            } else {
                PB_TT_LEAF(BLACK, false)
            }
        }
#undef PB_TT_LEAF
        PB_CUDA(cudaGetLastError());
        stats.kernels += 1;
    }
    if (ctx->timing) PB_CUDA(cudaEventRecord(ctx->ev[2], s));
    // upsweep, deepest level first, then the roots (their counts are not
    // stored: the root depth has no device table, the host keeps them)
    const u32 *child32 = leafcnt;
    const u64 *child64 = nullptr;
    for (int li = (int)levels.size() - 1; li >= 0; li--) {
        TTLevel &L = levels[li];
        unsigned g = grid_for(L.n, 256);
        TTView tv = ctx->dtt.at(L.rem);
        if (child64)
            k_upsweep<u64><<<g, 256, 0, s>>>(child64, L.offs, L.counts, L.flags, L.hash, L.n, tv, L.vals);
        else
            k_upsweep<u32><<<g, 256, 0, s>>>(child32, L.offs, L.counts, L.flags, L.hash, L.n, tv, L.vals);
        k_resolve_dups<<<g, 256, 0, s>>>(L.flags, L.redirect, L.n, L.vals);
        PB_CUDA(cudaGetLastError());
        stats.kernels += 2;
        child64 = L.vals;
    }
    const TTView none{nullptr, 0, TT_NONE, 0};
    if (child64)
        k_upsweep<u64><<<grid_for(nroots, 256), 256, 0, s>>>(child64, roff, rcnt, rflags, ph, nroots, none, rvals);
    else
        k_upsweep<u32><<<grid_for(nroots, 256), 256, 0, s>>>(child32, roff, rcnt, rflags, ph, nroots, none, rvals);
    PB_CUDA(cudaGetLastError());
    stats.kernels += 1;
    if (ctx->timing) PB_CUDA(cudaEventRecord(ctx->ev[3], s));
    std::vector<u64> tmp(nroots);
    PB_CUDA(cudaMemcpyAsync(tmp.data(), rvals, sizeof(u64) * nroots, cudaMemcpyDeviceToHost, s));
    PB_CUDA(cudaMemcpyAsync(ctx->h_pinned, ctx->d_counter, 2 * sizeof(u64), cudaMemcpyDeviceToHost, s));
    PB_CUDA(cudaMemcpyAsync(ctx->h_pinned + 2, ctx->d_err, sizeof(u32), cudaMemcpyDeviceToHost, s));
    PB_CUDA(cudaStreamSynchronize(s));
    if ((u32)ctx->h_pinned[2]) return fail(ctx, PB_ERR_DEVICE, "TT kernel reported a device error");
    for (u64 k = 0; k < nroots; k++) out[k] = tmp[k];
    stats.leaf_edges += n;
    stats.leaf_positions += ctx->h_pinned[1];
    stats.d2h_bytes += 8 * nroots + 20;
    if (ctx->timing) {
        float a = 0, b2 = 0;
        PB_CUDA(cudaEventElapsedTime(&a, ctx->ev[0], ctx->ev[3]));
        PB_CUDA(cudaEventElapsedTime(&b2, ctx->ev[1], ctx->ev[2]));
        stats.device_ms += a;
        stats.leaf_ms += b2;
    }
    return PB_OK;
}

int bfs_perft_tt(pb_ctx *ctx, const Board &root, u32 root_st, int color, int depth, const Hash128 &root_hash,
                 u64 *out, int *bfs_status)
{
    const uint8_t st8 = (uint8_t)root_st;
    return bfs_tt_roots(ctx, &root, &st8, &root_hash, 1, color, depth, out, bfs_status);
}

// perft of one position on the GPU; a level too big for the arena splits the
// root on the host and recurses (the reference's OOM path recomputes one
// level down the same way, launcher.cu:600-610, but on the CPU).
int gpu_perft(pb_ctx *ctx, const Board &b, u32 st, int c, int depth, u64 *out)
{
    int status = BFS_OK;
    int rc = ctx->opts.use_tt ? bfs_perft_tt(ctx, b, st, c, depth, hash_position(b, st, c), out, &status)
                              : bfs_perft(ctx, b, st, c, depth, out, &status);
    if (rc != PB_OK) return rc;
    if (status == BFS_OK) return PB_OK;
    if (depth <= 3) return fail(ctx, PB_ERR_NOMEM, "BFS arena too small for a depth-3 perft");
    uint16_t mv[MAX_MOVES];
    int n = host_gen(b, st, c, mv);
    u64 total = 0;
    for (int i = 0; i < n; i++) {
        Board cb = b;
        u32 cs = st;
        host_make(cb, cs, c, mv[i]);
        u64 sub = 0;
        rc = gpu_perft(ctx, cb, cs, 1 - c, depth - 1, &sub);
        if (rc != PB_OK) return rc;
        total += sub;
    }
    *out = total;
    return PB_OK;
}

// ---------------------------------------------------------------- batched roots
// Colour normalisation: a position with black to move becomes its mirror
// image with white to move (ranks reversed, colours swapped, castle rights
// swapped); perft is unchanged.
inline void to_white_to_move(const pb_pos &p, Board &b, uint8_t &st)
{
    b = to_board(p);
    st = p.state;
    if (p.color == WHITE) return;
    u64 occ = b.bb[1] | b.bb[2] | b.bb[3];
    u64 white = occ & ~b.bb[0];
    b.bb[0] = __builtin_bswap64(white);
    for (int k = 1; k < 4; k++) b.bb[k] = __builtin_bswap64(b.bb[k]);
    st = (uint8_t)((st & 0xF0) | ((st & 3) << 2) | ((st >> 2) & 3));
}

// Batched breadth-first perft of n white-to-move roots at one depth;
// out[i] = perft(depth) of root i.  BFS_TOO_BIG when a level does not fit.
int bfs_batch(pb_ctx *ctx, const Board *rb, const uint8_t *rs, u64 n, int depth, u64 *out, int *bfs_status)
{
    NvtxRange nvtx_pass("bfs_batch");
    *bfs_status = BFS_OK;
    const bool strict = ctx->opts.strict != 0;
    if (n == 0) return PB_OK;
    if (depth == 0) {
        for (u64 i = 0; i < n; i++) out[i] = 1;
        return PB_OK;
    }
    cudaStream_t s = ctx->stream;
    pb_stats &stats = ctx->stats;
    Arena ar{ctx->arena, ctx->arena_bytes};
    Board *b0 = ar.take<Board>(n);
    uint8_t *s0 = ar.take<uint8_t>(n);
    u32 *r0 = ar.take<u32>(n);
    u32 *cnt0 = ar.take<u32>(n);
    u64 *off0 = ar.take<u64>(n);
    unsigned long long *rc = ar.take<unsigned long long>(n);
    u64 tiles0 = (n + SCAN_TILE - 1) / SCAN_TILE;
    u64 *status0 = ar.take<u64>(tiles0);
    if (!b0 || !s0 || !r0 || !cnt0 || !off0 || !rc || !status0) {
        *bfs_status = BFS_TOO_BIG;
        return PB_OK;
    }
    std::vector<u32> iota(n);
    for (u64 i = 0; i < n; i++) iota[i] = (u32)i;
    PB_CUDA(cudaMemcpyAsync(b0, rb, sizeof(Board) * n, cudaMemcpyHostToDevice, s));
    PB_CUDA(cudaMemcpyAsync(s0, rs, n, cudaMemcpyHostToDevice, s));
    PB_CUDA(cudaMemcpyAsync(r0, iota.data(), sizeof(u32) * n, cudaMemcpyHostToDevice, s));
    PB_CUDA(cudaMemsetAsync(rc, 0, sizeof(unsigned long long) * n, s));
    PB_CUDA(cudaMemsetAsync(ctx->d_err, 0, sizeof(u32), s));
    PB_CUDA(cudaMemsetAsync(ctx->d_counter, 0, 2 * sizeof(unsigned long long), s));
    stats.h2d_bytes += (sizeof(Board) + 1 + 4) * n;
    if (ctx->timing) PB_CUDA(cudaEventRecord(ctx->ev[0], s));
    if (depth == 1) {
        if (strict)
            k_count_positions<WHITE, true><<<grid_for(n, 256), 256, 0, s>>>(b0, s0, n, cnt0);
        else
            k_count_positions<WHITE, false><<<grid_for(n, 256), 256, 0, s>>>(b0, s0, n, cnt0);
        PB_CUDA(cudaGetLastError());
        std::vector<u32> tmp(n);
        PB_CUDA(cudaMemcpyAsync(tmp.data(), cnt0, sizeof(u32) * n, cudaMemcpyDeviceToHost, s));
        PB_CUDA(cudaStreamSynchronize(s));
        for (u64 i = 0; i < n; i++) out[i] = tmp[i];
        stats.kernels += 1;
        stats.d2h_bytes += 4 * n;
        return PB_OK;
    }
    // root moves as the first edges
    k_count_positions<WHITE, true><<<grid_for(n, 256), 256, 0, s>>>(b0, s0, n, cnt0);
    PB_CUDA(cudaMemsetAsync(status0, 0, sizeof(u64) * tiles0, s));
    PB_CUDA(cudaMemsetAsync(ctx->d_ticket, 0, sizeof(u32), s));
    k_scan<<<(unsigned)tiles0, SCAN_THREADS, 0, s>>>(cnt0, n, off0, status0, ctx->d_ticket, ctx->d_total, ctx->d_err);
    PB_CUDA(cudaGetLastError());
    PB_CUDA(cudaMemcpyAsync(ctx->h_pinned, ctx->d_total, sizeof(u64), cudaMemcpyDeviceToHost, s));
    PB_CUDA(cudaStreamSynchronize(s));
    stats.kernels += 2;
    u64 ne = ctx->h_pinned[0];
    if (ne > 0xFFFFFFFFULL) {
        *bfs_status = BFS_TOO_BIG;
        return PB_OK;
    }
    uint16_t *emv = ar.take<uint16_t>(ne ? ne : 1);
    u32 *epi = ar.take<u32>(ne ? ne : 1);
    if (!emv || !epi) {
        *bfs_status = BFS_TOO_BIG;
        return PB_OK;
    }
    if (ne) {
        k_generate<WHITE><<<grid_for(n, GEN_THREADS), GEN_THREADS, 0, s>>>(b0, s0, off0, ctx->d_total, n, emv, epi,
                                                                         ctx->d_err);
        PB_CUDA(cudaGetLastError());
        stats.kernels += 1;
    }
    if (stats.levels < 16) stats.level_sizes[stats.levels] = ne;
    Board *cur_b = b0;
    uint8_t *cur_s = s0;
    u32 *cur_r = r0;
    u64 n_par = n;
    int c = WHITE;
    for (int rem = depth - 1; rem > 2 && ne; rem--) {
        Board *cb = ar.take<Board>(ne);
        uint8_t *cs = ar.take<uint8_t>(ne);
        u32 *cr = ar.take<u32>(ne);
        u32 *cnt = ar.take<u32>(ne);
        u64 *offs = ar.take<u64>(ne);
        u64 tiles = (ne + SCAN_TILE - 1) / SCAN_TILE;
        u64 *status = ar.take<u64>(tiles);
        if (!cb || !cs || !cr || !cnt || !offs || !status) {
            *bfs_status = BFS_TOO_BIG;
            return PB_OK;
        }
        unsigned g = grid_for(ne, 256);
        if (c == WHITE)
            k_expand_count_rooted<WHITE><<<g, 256, 0, s>>>(cur_b, cur_s, cur_r, epi, emv, ne, n_par, cb, cs, cr, cnt, ctx->d_err);
        else
            k_expand_count_rooted<BLACK><<<g, 256, 0, s>>>(cur_b, cur_s, cur_r, epi, emv, ne, n_par, cb, cs, cr, cnt, ctx->d_err);
        PB_CUDA(cudaMemsetAsync(status, 0, sizeof(u64) * tiles, s));
        PB_CUDA(cudaMemsetAsync(ctx->d_ticket, 0, sizeof(u32), s));
        k_scan<<<(unsigned)tiles, SCAN_THREADS, 0, s>>>(cnt, ne, offs, status, ctx->d_ticket, ctx->d_total, ctx->d_err);
        PB_CUDA(cudaGetLastError());
        PB_CUDA(cudaMemcpyAsync(ctx->h_pinned, ctx->d_total, sizeof(u64), cudaMemcpyDeviceToHost, s));
        PB_CUDA(cudaMemcpyAsync(ctx->h_pinned + 1, ctx->d_err, sizeof(u32), cudaMemcpyDeviceToHost, s));
        PB_CUDA(cudaStreamSynchronize(s));
        stats.kernels += 2;
        stats.d2h_bytes += 12;
        if ((u32)ctx->h_pinned[1]) return fail(ctx, PB_ERR_DEVICE, "batched level reported a device error");
        u64 next = ctx->h_pinned[0];
        stats.levels++;
        if (stats.levels < 16) stats.level_sizes[stats.levels] = next;
        cur_b = cb;
        cur_s = cs;
        cur_r = cr;
        n_par = ne;
        c = 1 - c;
        if (next > 0xFFFFFFFFULL) {
            *bfs_status = BFS_TOO_BIG;
            return PB_OK;
        }
        uint16_t *nmv = ar.take<uint16_t>(next ? next : 1);
        u32 *npi = ar.take<u32>(next ? next : 1);
        if (!nmv || !npi) {
            *bfs_status = BFS_TOO_BIG;
            return PB_OK;
        }
        if (next) {
            if (c == WHITE)
                k_generate<WHITE><<<grid_for(n_par, GEN_THREADS), GEN_THREADS, 0, s>>>(cb, cs, offs, ctx->d_total, n_par, nmv, npi, ctx->d_err);
            else
                k_generate<BLACK><<<grid_for(n_par, GEN_THREADS), GEN_THREADS, 0, s>>>(cb, cs, offs, ctx->d_total, n_par, nmv, npi, ctx->d_err);
            PB_CUDA(cudaGetLastError());
            stats.kernels += 1;
        }
        emv = nmv;
        epi = npi;
        ne = next;
    }
    if (ctx->timing) PB_CUDA(cudaEventRecord(ctx->ev[1], s));
    if (ne) {
        if (depth == 2) {
            unsigned g = grid_for(ne, 256);
            if (c == WHITE) {
                if (strict) k_leaf1_rooted<WHITE, true><<<g, 256, 0, s>>>(cur_b, cur_s, cur_r, epi, emv, ne, n_par, rc);
                else k_leaf1_rooted<WHITE, false><<<g, 256, 0, s>>>(cur_b, cur_s, cur_r, epi, emv, ne, n_par, rc);
            } else {
                if (strict) k_leaf1_rooted<BLACK, true><<<g, 256, 0, s>>>(cur_b, cur_s, cur_r, epi, emv, ne, n_par, rc);
                else k_leaf1_rooted<BLACK, false><<<g, 256, 0, s>>>(cur_b, cur_s, cur_r, epi, emv, ne, n_par, rc);
            }
        } else {
            unsigned g = grid_for(ne, PB_LEAF_THREADS);
            const int mode = (leaf_mode(ctx) == 3 && !balanced_fits(ctx, ne)) ? 2 : leaf_mode(ctx);
            const int bt = balanced_threads(ctx, ne, 1024);
            const unsigned gb = (unsigned)((ne + (u64)PB_BALANCED_K * bt - 1) / ((u64)PB_BALANCED_K * bt));
#define PB_ROOTED_LEAF(CC, SS)                                                                                   \
    if (mode == 3 && bt == 1024)                                                                                 \
        k_leaf2_rooted_balanced<CC, SS, 1024><<<gb, 1024, 0, s>>>(cur_b, cur_s, cur_r, epi, emv, ne, n_par, rc,  \
                                                                  ctx->d_counter);                               \
    else if (mode == 3 && bt == 512)                                                                             \
        k_leaf2_rooted_balanced<CC, SS, 512><<<gb, 512, 0, s>>>(cur_b, cur_s, cur_r, epi, emv, ne, n_par, rc,    \
                                                                ctx->d_counter);                                 \
    else if (mode == 3)                                                                                          \
        k_leaf2_rooted_balanced<CC, SS, 256><<<gb, 256, 0, s>>>(cur_b, cur_s, cur_r, epi, emv, ne, n_par, rc,    \
                                                                ctx->d_counter);                                 \
    else if (mode == 2)                                                                                          \
        k_leaf2_rooted<CC, SS, 2><<<g, PB_LEAF_THREADS, 0, s>>>(cur_b, cur_s, cur_r, epi, emv, ne, n_par, rc,    \
                                                                ctx->d_counter);                                 \
    else if (mode == 1)                                                                                          \
        k_leaf2_rooted<CC, SS, 1><<<g, PB_LEAF_THREADS, 0, s>>>(cur_b, cur_s, cur_r, epi, emv, ne, n_par, rc,    \
                                                                ctx->d_counter);                                 \
    else                                                                                                         \
        k_leaf2_rooted<CC, SS, 0><<<g, PB_LEAF_THREADS, 0, s>>>(cur_b, cur_s, cur_r, epi, emv, ne, n_par, rc,    \
                                                                ctx->d_counter);
            if (c == WHITE) {
                if (strict) {
                    PB_ROOTED_LEAF(WHITE, true)
                } else {
                    PB_ROOTED_LEAF(WHITE, false)
                }
            } else {
                if (strict) {
                    PB_ROOTED_LEAF(BLACK, true)
                } else {
                    PB_ROOTED_LEAF(BLACK, false)
                }
            }
#undef PB_ROOTED_LEAF
        }
        PB_CUDA(cudaGetLastError());
        stats.kernels += 1;
    }
    if (ctx->timing) {
        PB_CUDA(cudaEventRecord(ctx->ev[2], s));
        PB_CUDA(cudaEventRecord(ctx->ev[3], s));
    }
    std::vector<unsigned long long> tmp(n);
    PB_CUDA(cudaMemcpyAsync(tmp.data(), rc, sizeof(unsigned long long) * n, cudaMemcpyDeviceToHost, s));
    PB_CUDA(cudaMemcpyAsync(ctx->h_pinned, ctx->d_counter, 2 * sizeof(u64), cudaMemcpyDeviceToHost, s));
    PB_CUDA(cudaMemcpyAsync(ctx->h_pinned + 2, ctx->d_err, sizeof(u32), cudaMemcpyDeviceToHost, s));
    PB_CUDA(cudaStreamSynchronize(s));
    if ((u32)ctx->h_pinned[2]) return fail(ctx, PB_ERR_DEVICE, "batched leaf reported a device error");
    for (u64 i = 0; i < n; i++) out[i] = tmp[i];
    stats.leaf_edges += ne;
    stats.leaf_positions += ctx->h_pinned[1];
    stats.d2h_bytes += 8 * n + 20;
    if (ctx->timing) {
        float a = 0, b2 = 0;
        PB_CUDA(cudaEventElapsedTime(&a, ctx->ev[0], ctx->ev[3]));
        PB_CUDA(cudaEventElapsedTime(&b2, ctx->ev[1], ctx->ev[2]));
        stats.device_ms += a;
        stats.leaf_ms += b2;
    }
    return PB_OK;
}

// Batched perft with automatic halving when a level does not fit.
int gpu_batch(pb_ctx *ctx, const Board *rb, const uint8_t *rs, u64 n, int depth, u64 *out)
{
    int status = BFS_OK;
    int rc = bfs_batch(ctx, rb, rs, n, depth, out, &status);
    if (rc != PB_OK || status == BFS_OK) return rc;
    if (n == 1) {
        // one root too big for a batched pass: the single-root path splits it
        pb_pos p;
        to_pos(rb[0], rs[0], WHITE, p);
        return gpu_perft(ctx, rb[0], rs[0], WHITE, depth, out);
    }
    u64 h = n / 2;
    rc = gpu_batch(ctx, rb, rs, h, depth, out);
    if (rc != PB_OK) return rc;
    return gpu_batch(ctx, rb + h, rs + h, n - h, depth, out + h);
}

// ---------------------------------------------------------------- planned batches (CUDA graph)
// A batch whose level sizes were planned ahead (from the learned size
// predictions) runs as one captured CUDA graph: every level's kernels read
// their sizes from device memory, the leaf is a persistent kernel fed by a
// device work queue, and nothing returns to the host until the root counts
// do.  caps[k] bounds the edges of level k+1 (k = 0: root moves).
struct GraphLevel {
    Board *b;
    uint8_t *s;
    u32 *r, *cnt;
    u64 *off, *status;
    uint16_t *mv;
    u32 *pi;
    u64 tiles;
};

template <int C, bool S, int MODE>
void launch_leaf_queue_t(cudaStream_t s, int sms, const Board *b, const uint8_t *st, const u32 *r, const u32 *pi,
                         const uint16_t *mv, const u64 *n_dev, u64 cap, const u64 *npar_dev, u64 npar_cap,
                         unsigned long long *cursor, unsigned long long *rc, unsigned long long *counter, u32 *err)
{
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_leaf2_rooted_queue<C, S, MODE>, PB_LEAF_THREADS, 0);
    if (per_sm <= 0) per_sm = 1;
    unsigned grid = (unsigned)std::min<u64>((u64)sms * per_sm, (cap + PB_LEAF_THREADS - 1) / PB_LEAF_THREADS + 1);
    k_leaf2_rooted_queue<C, S, MODE><<<grid, PB_LEAF_THREADS, 0, s>>>(b, st, r, pi, mv, n_dev, cap, npar_dev,
                                                                      npar_cap, cursor, rc, counter, err);
}
template <int C, bool S, int MODE>
void launch_leaf_grid_t(cudaStream_t s, const Board *b, const uint8_t *st, const u32 *r, const u32 *pi,
                        const uint16_t *mv, const u64 *n_dev, u64 cap, const u64 *npar_dev, u64 npar_cap,
                        unsigned long long *rc, unsigned long long *counter, u32 *err)
{
    unsigned grid = (unsigned)std::max<u64>((cap + PB_LEAF_THREADS - 1) / PB_LEAF_THREADS, 1);
    k_leaf2_rooted_dev<C, S, MODE><<<grid, PB_LEAF_THREADS, 0, s>>>(b, st, r, pi, mv, n_dev, cap, npar_dev, npar_cap,
                                                                    rc, counter, err);
}
// Leaf of a planned batch: the grid leaf over the planned capacity, or the
// persistent work-queue leaf (queue).
// Balanced leaf over a planned level: the grid covers the capacity.
template <int C, bool S>
void launch_leaf_balanced_dev(cudaStream_t s, int sms, const Board *b, const uint8_t *st, const u32 *r,
                              const u32 *pi, const uint16_t *mv, const u64 *n_dev, u64 cap, const u64 *npar_dev,
                              u64 npar_cap, unsigned long long *rc, unsigned long long *counter, u32 *err)
{
    const bool big = cap >= (u64)PB_BALANCED_K * 1024u * 8u * (u64)sms;
    const u64 per = (u64)PB_BALANCED_K * (big ? 1024u : 256u);
    const unsigned grid = (unsigned)std::max<u64>((cap + per - 1) / per, 1);
    if (big)
        k_leaf2_rooted_balanced_dev<C, S, 1024><<<grid, 1024, 0, s>>>(b, st, r, pi, mv, n_dev, cap, npar_dev, npar_cap,
                                                                      rc, counter, err);
    else
        k_leaf2_rooted_balanced_dev<C, S, 256><<<grid, 256, 0, s>>>(b, st, r, pi, mv, n_dev, cap, npar_dev, npar_cap,
                                                                    rc, counter, err);
}
template <int C, bool S, int MODE>
void launch_leaf_planned_t(bool queue, cudaStream_t s, int sms, const Board *b, const uint8_t *st, const u32 *r,
                           const u32 *pi, const uint16_t *mv, const u64 *n_dev, u64 cap, const u64 *npar_dev,
                           u64 npar_cap, unsigned long long *cursor, unsigned long long *rc,
                           unsigned long long *counter, u32 *err)
{
    if (queue)
        launch_leaf_queue_t<C, S, MODE>(s, sms, b, st, r, pi, mv, n_dev, cap, npar_dev, npar_cap, cursor, rc, counter,
                                        err);
    else
        launch_leaf_grid_t<C, S, MODE>(s, b, st, r, pi, mv, n_dev, cap, npar_dev, npar_cap, rc, counter, err);
}
template <int C, bool S>
void launch_leaf_queue(int mode, bool queue, cudaStream_t s, int sms, const Board *b, const uint8_t *st,
                       const u32 *r, const u32 *pi, const uint16_t *mv, const u64 *n_dev, u64 cap,
                       const u64 *npar_dev, u64 npar_cap, unsigned long long *cursor, unsigned long long *rc,
                       unsigned long long *counter, u32 *err)
{
    if (mode == 3 && !queue && cap >= (u64)PB_BALANCED_K * 256u * 8u * (u64)sms)
        launch_leaf_balanced_dev<C, S>(s, sms, b, st, r, pi, mv, n_dev, cap, npar_dev, npar_cap, rc, counter, err);
    else if (mode >= 2)
        launch_leaf_planned_t<C, S, 2>(queue, s, sms, b, st, r, pi, mv, n_dev, cap, npar_dev, npar_cap, cursor, rc,
                                       counter, err);
    else if (mode == 1)
        launch_leaf_planned_t<C, S, 1>(queue, s, sms, b, st, r, pi, mv, n_dev, cap, npar_dev, npar_cap, cursor, rc,
                                       counter, err);
    else
        launch_leaf_planned_t<C, S, 0>(queue, s, sms, b, st, r, pi, mv, n_dev, cap, npar_dev, npar_cap, cursor, rc,
                                       counter, err);
}

// Builds (captures) the graph for a planned batch shape.
int capture_batch_graph(pb_ctx *ctx, GraphPlan &g)
{
    cudaStream_t s = ctx->stream;
    const u64 n = g.n;
    const int depth = g.depth;
    Arena ar{ctx->arena, ctx->arena_bytes};
    g.b0 = ar.take<Board>(n);
    g.s0 = ar.take<uint8_t>(n);
    g.r0 = ar.take<u32>(n);
    g.rc = ar.take<unsigned long long>(n);
    u32 *cnt0 = ar.take<u32>(n);
    u64 *off0 = ar.take<u64>(n);
    u64 tiles0 = (n + SCAN_TILE - 1) / SCAN_TILE;
    u64 *status0 = ar.take<u64>(tiles0);
    const int nlev = std::max(depth - 2, 1);  // edge levels E_1 .. E_nlev
    g.sizes = ar.take<u64>(nlev + 4);
    unsigned long long *cursor = ar.take<unsigned long long>(1);
    if (!g.b0 || !g.s0 || !g.r0 || !g.rc || !cnt0 || !off0 || !status0 || !g.sizes || !cursor) return PB_ERR_NOMEM;
    std::vector<GraphLevel> L(nlev + 1);
    for (int k = 1; k <= nlev; k++) {
        u64 cap = g.caps[k - 1];
        L[k].mv = ar.take<uint16_t>(cap);
        L[k].pi = ar.take<u32>(cap);
        if (!L[k].mv || !L[k].pi) return PB_ERR_NOMEM;
        if (k < nlev || depth == 2) {
            // positions of level k (the children of E_k) are materialised
            // for every level but the last (the leaf makes those itself)
        }
        if (k < nlev) {
            L[k].b = ar.take<Board>(cap);
            L[k].s = ar.take<uint8_t>(cap);
            L[k].r = ar.take<u32>(cap);
            L[k].cnt = ar.take<u32>(cap);
            L[k].off = ar.take<u64>(cap);
            L[k].tiles = (cap + SCAN_TILE - 1) / SCAN_TILE;
            L[k].status = ar.take<u64>(L[k].tiles);
            if (!L[k].b || !L[k].s || !L[k].r || !L[k].cnt || !L[k].off || !L[k].status) return PB_ERR_NOMEM;
        }
    }
    u64 *d_n0 = g.sizes;  // [0] = roots, [k] = edges of level k
    std::vector<u64> init(nlev + 4, 0);
    init[0] = n;
    PB_CUDA(cudaMemcpy(g.sizes, init.data(), sizeof(u64) * init.size(), cudaMemcpyHostToDevice));
    {
        std::vector<u32> iota(n);
        for (u64 i = 0; i < n; i++) iota[i] = (u32)i;
        PB_CUDA(cudaMemcpy(g.r0, iota.data(), sizeof(u32) * n, cudaMemcpyHostToDevice));
    }
    cudaGraph_t graph = nullptr;
    PB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    cudaMemsetAsync(g.rc, 0, sizeof(unsigned long long) * n, s);
    cudaMemsetAsync(ctx->d_err, 0, sizeof(u32), s);
    cudaMemsetAsync(ctx->d_counter, 0, 2 * sizeof(unsigned long long), s);
    cudaMemsetAsync(cursor, 0, sizeof(unsigned long long), s);
    // level 0: root move counts -> E_1
    k_count_positions<WHITE, true><<<grid_for(n, 256), 256, 0, s>>>(g.b0, g.s0, n, cnt0);
    cudaMemsetAsync(status0, 0, sizeof(u64) * tiles0, s);
    cudaMemsetAsync(ctx->d_ticket, 0, sizeof(u32), s);
    k_scan_dev<<<(unsigned)tiles0, SCAN_THREADS, 0, s>>>(cnt0, d_n0, n, off0, status0, ctx->d_ticket, d_n0 + 1, ctx->d_err);
    k_generate_dev<WHITE><<<grid_for(n, GEN_THREADS), GEN_THREADS, 0, s>>>(g.b0, g.s0, off0, d_n0 + 1, d_n0, n,
                                                                           g.caps[0], L[1].mv, L[1].pi, ctx->d_err);
    // middle levels: E_k -> positions P_k -> E_{k+1}
    const Board *pb_ = g.b0;
    const uint8_t *ps = g.s0;
    const u32 *pr = g.r0;
    const u64 *npar = d_n0;
    u64 npar_cap = n;
    int c = WHITE;
    for (int k = 1; k < nlev; k++) {
        u64 cap = g.caps[k - 1];
        unsigned ge = (unsigned)std::min<u64>((cap + 255) / 256, (u64)ctx->num_sms * 16);
        if (c == WHITE)
            k_expand_rooted_dev<WHITE><<<ge, 256, 0, s>>>(pb_, ps, pr, L[k].pi, L[k].mv, d_n0 + k, cap, npar, npar_cap,
                                                          L[k].b, L[k].s, L[k].r, L[k].cnt, ctx->d_err);
        else
            k_expand_rooted_dev<BLACK><<<ge, 256, 0, s>>>(pb_, ps, pr, L[k].pi, L[k].mv, d_n0 + k, cap, npar, npar_cap,
                                                          L[k].b, L[k].s, L[k].r, L[k].cnt, ctx->d_err);
        c = 1 - c;
        cudaMemsetAsync(L[k].status, 0, sizeof(u64) * L[k].tiles, s);
        cudaMemsetAsync(ctx->d_ticket, 0, sizeof(u32), s);
        k_scan_dev<<<(unsigned)L[k].tiles, SCAN_THREADS, 0, s>>>(L[k].cnt, d_n0 + k, cap, L[k].off, L[k].status,
                                                                 ctx->d_ticket, d_n0 + k + 1, ctx->d_err);
        if (c == WHITE)
            k_generate_dev<WHITE><<<grid_for(cap, GEN_THREADS), GEN_THREADS, 0, s>>>(
                L[k].b, L[k].s, L[k].off, d_n0 + k + 1, d_n0 + k, cap, g.caps[k], L[k + 1].mv, L[k + 1].pi, ctx->d_err);
        else
            k_generate_dev<BLACK><<<grid_for(cap, GEN_THREADS), GEN_THREADS, 0, s>>>(
                L[k].b, L[k].s, L[k].off, d_n0 + k + 1, d_n0 + k, cap, g.caps[k], L[k + 1].mv, L[k + 1].pi, ctx->d_err);
        pb_ = L[k].b;
        ps = L[k].s;
        pr = L[k].r;
        npar = d_n0 + k;
        npar_cap = cap;
    }
    // leaf over E_nlev
    const u64 lcap = g.caps[nlev - 1];
    if (depth == 2) {
        unsigned gl = (unsigned)std::min<u64>((lcap + 255) / 256, (u64)ctx->num_sms * 16);
        if (g.strict)
            k_leaf1_rooted_dev<WHITE, true><<<gl, 256, 0, s>>>(pb_, ps, pr, L[1].pi, L[1].mv, d_n0 + 1, lcap, npar,
                                                               npar_cap, g.rc, ctx->d_err);
        else
            k_leaf1_rooted_dev<WHITE, false><<<gl, 256, 0, s>>>(pb_, ps, pr, L[1].pi, L[1].mv, d_n0 + 1, lcap, npar,
                                                                npar_cap, g.rc, ctx->d_err);
    } else if (c == WHITE) {
        if (g.strict)
            launch_leaf_queue<WHITE, true>(g.mode, g.queue, s, ctx->num_sms, pb_, ps, pr, L[nlev].pi, L[nlev].mv, d_n0 + nlev, lcap, npar,
                                           npar_cap, cursor, g.rc, ctx->d_counter, ctx->d_err);
        else
            launch_leaf_queue<WHITE, false>(g.mode, g.queue, s, ctx->num_sms, pb_, ps, pr, L[nlev].pi, L[nlev].mv, d_n0 + nlev, lcap,
                                            npar, npar_cap, cursor, g.rc, ctx->d_counter, ctx->d_err);
    } else {
        if (g.strict)
            launch_leaf_queue<BLACK, true>(g.mode, g.queue, s, ctx->num_sms, pb_, ps, pr, L[nlev].pi, L[nlev].mv, d_n0 + nlev, lcap, npar,
                                           npar_cap, cursor, g.rc, ctx->d_counter, ctx->d_err);
        else
            launch_leaf_queue<BLACK, false>(g.mode, g.queue, s, ctx->num_sms, pb_, ps, pr, L[nlev].pi, L[nlev].mv, d_n0 + nlev, lcap,
                                            npar, npar_cap, cursor, g.rc, ctx->d_counter, ctx->d_err);
    }
    cudaError_t ce = cudaStreamEndCapture(s, &graph);
    if (ce != cudaSuccess) return cuda_fail(ctx, ce, "end capture");
    if (g.exec) cudaGraphExecDestroy(g.exec);
    g.exec = nullptr;
    ce = cudaGraphInstantiate(&g.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ce != cudaSuccess) return cuda_fail(ctx, ce, "graph instantiate");
    return PB_OK;
}

// Runs one planned batch; *overflow = true when a level outgrew its planned
// capacity (results then invalid: the caller reruns with exact sizing).
int run_planned_batch(pb_ctx *ctx, GraphPlan &g, const Board *rb, const uint8_t *rs, u64 n, int depth,
                      const std::vector<u64> &caps, u64 *out, bool *overflow)
{
    NvtxRange nvtx_pass("planned_batch");
    *overflow = false;
    const bool strict = ctx->opts.strict != 0;
    const int mode = leaf_mode(ctx);
    const bool queue = ctx->tuning.planned_leaf == 2;
    if (!g.same(n, depth, strict, mode, queue, caps)) {
        g.n = n;
        g.depth = depth;
        g.strict = strict;
        g.mode = mode;
        g.queue = queue;
        g.caps = caps;
        int rc = capture_batch_graph(ctx, g);
        if (rc != PB_OK) {
            if (g.exec) cudaGraphExecDestroy(g.exec);
            g.exec = nullptr;
            return rc;
        }
    }
    cudaStream_t s = ctx->stream;
    PB_CUDA(cudaMemcpyAsync(g.b0, rb, sizeof(Board) * n, cudaMemcpyHostToDevice, s));
    PB_CUDA(cudaMemcpyAsync(g.s0, rs, n, cudaMemcpyHostToDevice, s));
    if (ctx->timing) PB_CUDA(cudaEventRecord(ctx->ev[0], s));
    PB_CUDA(cudaGraphLaunch(g.exec, s));
    if (ctx->timing) PB_CUDA(cudaEventRecord(ctx->ev[3], s));
    std::vector<unsigned long long> tmp(n);
    PB_CUDA(cudaMemcpyAsync(tmp.data(), g.rc, sizeof(unsigned long long) * n, cudaMemcpyDeviceToHost, s));
    PB_CUDA(cudaMemcpyAsync(ctx->h_pinned, ctx->d_counter, 2 * sizeof(u64), cudaMemcpyDeviceToHost, s));
    PB_CUDA(cudaMemcpyAsync(ctx->h_pinned + 2, ctx->d_err, sizeof(u32), cudaMemcpyDeviceToHost, s));
    PB_CUDA(cudaStreamSynchronize(s));
    u32 err = (u32)ctx->h_pinned[2];
    ctx->stats.kernels += 3 * (u32)std::max(depth - 3, 0) + 3 + 1;
    ctx->stats.h2d_bytes += (sizeof(Board) + 1) * n;
    ctx->stats.d2h_bytes += 8 * n + 20;
    if (ctx->timing) {
        float a = 0;
        PB_CUDA(cudaEventElapsedTime(&a, ctx->ev[0], ctx->ev[3]));
        ctx->stats.device_ms += a;
    }
    if (err & DEVERR_OVERFLOW) {
        *overflow = true;
        return PB_OK;
    }
    if (err) return fail(ctx, PB_ERR_DEVICE, "planned batch reported a device error");
    for (u64 i = 0; i < n; i++) out[i] = tmp[i];
    ctx->stats.leaf_positions += ctx->h_pinned[1];
    return PB_OK;
}

// ---------------------------------------------------------------- learned planning
// Level sizes of a depth-d batched perft of one root, from the network's
// predicted log2(1 + perft(k)), k = 1..4 (geometric beyond 4).
// Number of planned levels of a depth-d batch (depth <= 12).
constexpr int PLAN_LEVELS = 10;
inline int plan_levels(int depth) { return std::max(depth - 2, 1); }

void predicted_levels(const float *y, int depth, double *e)
{
    // only the predictions the levels use (exp2 is most of the planner's
    // per-root host time)
    const int nlev = plan_levels(depth), need = std::min(nlev, 4);
    double p[5] = {1, 0, 0, 0, 0};
    for (int k = 1; k <= need; k++) p[k] = std::max((double)exp2f(y[k - 1]) - 1.0, 0.0);
    const double bf = (nlev > 4 && p[3] > 0) ? std::max(p[4] / p[3], 1.0) : 30.0;
    for (int k = 1; k <= nlev; k++) e[k - 1] = k <= 4 ? p[k] : e[k - 2] * bf;
}

// bytes one root's batched levels take: 6 B per edge, 50 B per materialised position
double level_bytes(const double *e, int nlev)
{
    double b = 0;
    for (int k = 0; k < nlev; k++) b += e[k] * (6.0 + (k + 1 < nlev ? 50.0 : 0.0));
    return b;
}

// One root (or a split-off child of one) in the plan; plain data, so the
// planner's per-root bookkeeping allocates nothing.
struct PlanItem {
    Board b;
    uint8_t s;
    int depth;
    int owner;
    double bytes;
    double lv[PLAN_LEVELS];
};

}  // namespace
namespace {

// Learned batch planner: predictions size every level of a batch up front,
// bin-pack roots into batches that fit the arena, and split roots too big
// for one batch into their children (the per-root launch-depth choice).
// Batches then run as captured graphs; a batch whose levels outgrow the plan
// is rerun with exact count-then-allocate sizing (counted in plan stats).
int plan_and_run(pb_ctx *ctx, const pb_pos *roots, const int *depths, int n, uint64_t *counts, pb_plan_stats *ps)
{
    const double margin = 1.3;
    const double budget = (double)ctx->arena_bytes * 0.45 / margin;
    std::vector<PlanItem> items;
    items.reserve(n);
    for (int i = 0; i < n; i++) {
        PlanItem it;
        to_white_to_move(roots[i], it.b, it.s);
        it.depth = depths[i];
        it.owner = i;
        it.bytes = 0;
        items.push_back(it);
        counts[i] = 0;
    }
    std::vector<PlanItem> ready;
    ready.reserve(n);
    int guard = 0;
    while (!items.empty() && guard++ < 8) {
        // predict
        std::vector<pb_pos> pp(items.size());
        for (size_t k = 0; k < items.size(); k++) to_pos(items[k].b, items[k].s, WHITE, pp[k]);
        std::vector<float> y(items.size() * MLP_OUT);
        int rc = pb_mlp_predict(ctx, pp.data(), (int)pp.size(), y.data());
        if (rc != PB_OK) return rc;
        std::vector<PlanItem> next;
        for (size_t k = 0; k < items.size(); k++) {
            PlanItem &it = items[k];
            predicted_levels(&y[k * MLP_OUT], it.depth, it.lv);
            it.bytes = level_bytes(it.lv, plan_levels(it.depth));
            if (it.depth >= 4 && it.bytes > budget) {
                // too big for any batch: split into children one ply down
                uint16_t mv[MAX_MOVES];
                int m = host_gen(it.b, it.s, WHITE, mv);
                for (int j = 0; j < m; j++) {
                    PlanItem c;
                    c.b = it.b;
                    u32 st = it.s;
                    host_make(c.b, st, WHITE, mv[j]);
                    // child has black to move: mirror it back to white
                    pb_pos cp;
                    to_pos(c.b, st, BLACK, cp);
                    to_white_to_move(cp, c.b, c.s);
                    c.depth = it.depth - 1;
                    c.owner = it.owner;
                    c.bytes = 0;
                    next.push_back(c);
                }
                if (ps) ps->split_roots++;
            } else {
                ready.push_back(it);
            }
        }
        items.swap(next);
    }
    if (!items.empty()) return fail(ctx, PB_ERR_NOMEM, "planner could not fit a root");
    // bin-pack per depth: largest first, fill to the budget (an index sort:
    // the items themselves stay in place)
    std::vector<u32> order(ready.size());
    for (size_t k = 0; k < order.size(); k++) order[k] = (u32)k;
    bool one_batch = true;  // one depth and within the budget: no packing to do
    double all_bytes = 0;
    for (const PlanItem &it : ready) {
        one_batch = one_batch && it.depth == ready[0].depth;
        all_bytes += it.bytes;
    }
    if (!one_batch || all_bytes > budget)
        std::sort(order.begin(), order.end(), [&](u32 a, u32 b) {
            const PlanItem &x = ready[a], &y2 = ready[b];
            return x.depth != y2.depth ? x.depth < y2.depth : x.bytes > y2.bytes;
        });
    std::vector<Board> rb;
    std::vector<uint8_t> rs;
    std::vector<u64> out;
    size_t i = 0;
    while (i < order.size()) {
        int d = ready[order[i]].depth;
        size_t j = i;
        double used = 0;
        while (j < order.size() && ready[order[j]].depth == d &&
               (j == i || used + ready[order[j]].bytes <= budget) && j - i < 0xFFFFFFF) {
            used += ready[order[j]].bytes;
            j++;
        }
        u64 m = j - i;
        rb.resize(m);
        rs.resize(m);
        out.assign(m, 0);
        for (u64 k = 0; k < m; k++) {
            rb[k] = ready[order[i + k]].b;
            rs[k] = ready[order[i + k]].s;
        }
        int rc = PB_OK;
        bool overflow = false;
        if (d <= 1) {
            rc = gpu_batch(ctx, rb.data(), rs.data(), m, d, out.data());
        } else {
            std::vector<u64> caps(plan_levels(d), 0);
            for (u64 k = 0; k < m; k++)
                for (size_t l = 0; l < caps.size(); l++) caps[l] += (u64)ready[order[i + k]].lv[l];
            for (auto &c : caps) c = (u64)((double)c * margin) + 4096;
            rc = run_planned_batch(ctx, ctx->graph, rb.data(), rs.data(), m, d, caps, out.data(), &overflow);
            if (rc == PB_OK && overflow) {
                if (ps) ps->retries++;
                rc = gpu_batch(ctx, rb.data(), rs.data(), m, d, out.data());
            }
            if (ps) ps->graph_batches++;
        }
        if (rc != PB_OK) return rc;
        for (u64 k = 0; k < m; k++) counts[ready[order[i + k]].owner] += out[k];
        if (ps) ps->batches++;
        i = j;
    }
    return PB_OK;
}

// ---------------------------------------------------------------- workload generator
// Sort key equal to the order of the moves' UCI text: from file, from rank,
// to file, to rank, then the promotion letter ("" < b < n < q < r).
inline u32 uci_key(uint16_t m)
{
    static const u32 promo_rank[4] = {2, 1, 4, 3};  // flags&3: N, B, R, Q -> n=2, b=1, r=4, q=3
    int from = move_from(m), to = move_to(m), fl = move_flags(m);
    u32 k = (u32)(((from & 7) * 8 + (from >> 3)) * 64 + (to & 7) * 8 + (to >> 3));
    return k * 5 + ((fl & MF_PROMO) ? promo_rank[fl & 3] : 0);
}

// `plies` uniformly random legal moves from the initial array (fewer at a
// terminal position); returns the plies played.
int playout(u64 *st, int plies, pb_pos *out)
{
    parse_fen("rnbqkbnr/pppppppp/8/8/8/8/PPPPPPPP/RNBQKBNR w KQkq - 0 1", out);
    Board b = to_board(*out);
    u32 s = out->state;
    int c = WHITE, played = 0;
    for (int i = 0; i < plies; i++) {
        uint16_t mv[MAX_MOVES];
        int n = host_gen(b, s, c, mv);
        if (n <= 0) break;
        std::sort(mv, mv + n, [](uint16_t a, uint16_t z) { return uci_key(a) < uci_key(z); });
        u64 r = splitmix64(st);
        u32 pick = (u32)(((unsigned __int128)r * (u32)n) >> 64);
        host_make(b, s, c, mv[pick]);
        c = 1 - c;
        played++;
    }
    to_pos(b, s, c, *out);
    return played;
}

// ---------------------------------------------------------------- 128-bit helpers
inline void add128(pb_u128 &a, const pb_u128 &b)
{
    u64 old = a.lo;
    a.lo += b.lo;
    a.hi += b.hi + (a.lo < old ? 1 : 0);
}

// Decimal text of a 128-bit value: repeated division of four 32-bit limbs by
// 10^9, nine digits per step, most significant group unpadded.
int u128_decimal(pb_u128 v, char *buf, size_t len)
{
    if (!buf || len < 40) return PB_ERR_ARG;  // 2^128 - 1 has 39 digits
    uint32_t limb[4] = {(uint32_t)v.lo, (uint32_t)(v.lo >> 32), (uint32_t)v.hi, (uint32_t)(v.hi >> 32)};
    uint32_t groups[5];
    int ng = 0;
    do {
        u64 rem = 0;
        for (int i = 3; i >= 0; i--) {
            u64 cur = (rem << 32) | limb[i];
            limb[i] = (uint32_t)(cur / 1000000000ULL);
            rem = cur % 1000000000ULL;
        }
        groups[ng++] = (uint32_t)rem;
    } while (limb[0] | limb[1] | limb[2] | limb[3]);
    int k = snprintf(buf, len, "%u", groups[ng - 1]);
    for (int i = ng - 2; i >= 0; i--) k += snprintf(buf + k, len - k, "%09u", groups[i]);
    return k;
}

// Host recursion above the launch depth (perft_cpu_recurse, launcher.cu:572-715).
int launch_recurse(pb_ctx *ctx, const Board &b, u32 st, int c, int depth, const Hash128 &h, pb_u128 *out)
{
    const bool tt = ctx->opts.use_tt && ctx->htt.ready();
    if (tt && depth >= 2) {
        u64 hit;
        if (ctx->htt.probe(depth, h, &hit)) {
            out->lo = hit;
            out->hi = 0;
            return PB_OK;
        }
    }
    pb_u128 total{0, 0};
    if (depth <= ctx->launch_depth) {
        u64 v = 0;
        int rc = ctx->gpu ? gpu_perft(ctx, b, st, c, depth, &v) : PB_OK;
        if (rc != PB_OK) return rc;
        if (!ctx->gpu) v = host_perft(b, st, c, depth, ctx->opts.strict != 0);
        total.lo = v;
    } else {
        uint16_t mv[MAX_MOVES];
        int n = host_gen(b, st, c, mv);
        for (int i = 0; i < n; i++) {
            Board cb = b;
            u32 cs = st;
            host_make(cb, cs, c, mv[i]);
            Hash128 ch = tt ? hash_move(h, b, st, cs, c, mv[i]) : Hash128{0, 0};
            pb_u128 sub;
            int rc = launch_recurse(ctx, cb, cs, 1 - c, depth - 1, ch, &sub);
            if (rc != PB_OK) return rc;
            add128(total, sub);
        }
    }
    if (tt && depth >= 2 && total.hi == 0) ctx->htt.store(depth, h, total.lo);
    *out = total;
    return PB_OK;
}

// Table-mode perft of n roots of one colour in batched GPU calls that fit the
// arena: a batch whose levels do not fit is halved (a single root that does
// not fit goes to the single-root path, which splits it on the host); the
// batch size that fit last seeds the next call and doubles after a success.
int gpu_tt_roots(pb_ctx *ctx, const Board *rb, const uint8_t *rs, const Hash128 *rh, u64 n, int color, int depth,
                 u64 *out)
{
    u64 b = std::max<u64>(ctx->tt_batch, 1);
    u64 i = 0;
    while (i < n) {
        const u64 m = std::min(b, n - i);
        int status = BFS_OK;
        int rc = bfs_tt_roots(ctx, rb + i, rs + i, rh + i, m, color, depth, out + i, &status);
        if (rc != PB_OK) return rc;
        if (status == BFS_OK) {
            i += m;
            if (m == b && b < (1u << 20)) b *= 2;
            continue;
        }
        if (m == 1) {
            rc = gpu_perft(ctx, rb[i], rs[i], color, depth, out + i);
            if (rc != PB_OK) return rc;
            i++;
            continue;
        }
        b = m / 2;
    }
    ctx->tt_batch = b;
    return PB_OK;
}

// Host driver above the launch depth, breadth first (pb_tuning.host_driver =
// 2).  The reference walks the tree above the launch depth depth first and
// makes one GPU call per subtree (perft_cpu_recurse, launcher.cu:572-715).
// Here the tree is expanded on the host ply by ply down to the launch depth;
// with tables, positions reached by several move orders are merged by their
// 128-bit key (each keeps the number of paths that reach it) and positions
// found in the host table are answered from it.  The positions left at the
// launch depth then run in batched GPU calls, table mode with duplicates also
// merged across the batch's subtrees at every level, and
// perft = sum over them of paths x perft(launch depth), in 128 bits.  Without
// tables nothing is merged (no key is computed) and the batches run through
// the count-then-allocate batched path.
struct HostNode {
    Board b;
    uint8_t s;
    Hash128 h;
    u64 paths;
};
struct KeyHash {
    size_t operator()(const Hash128 &h) const { return (size_t)(h.lo ^ (h.hi * 0x9E3779B97F4A7C15ULL)); }
};
struct KeyEq {
    bool operator()(const Hash128 &a, const Hash128 &b) const { return a.lo == b.lo && a.hi == b.hi; }
};

inline void add_product(pb_u128 &acc, u64 a, u64 b)
{
    unsigned __int128 p = (unsigned __int128)a * b;
    pb_u128 v{(u64)p, (u64)(p >> 64)};
    add128(acc, v);
}

int launch_breadth_first(pb_ctx *ctx, const Board &root, u32 root_st, int c, int depth, const Hash128 &root_h,
                         pb_u128 *out)
{
    const bool tt = ctx->opts.use_tt && ctx->htt.ready();
    const int ld = ctx->launch_depth;
    pb_u128 total{0, 0};
    std::vector<HostNode> level{HostNode{root, (uint8_t)root_st, root_h, 1}};
    int col = c;
    constexpr size_t MAX_HOST_NODES = 1u << 22;
    for (int rem = depth; rem > ld && !level.empty(); rem--) {
        std::vector<HostNode> next;
        std::unordered_map<Hash128, u32, KeyHash, KeyEq> index;
        for (const HostNode &nd : level) {
            uint16_t mv[MAX_MOVES];
            int m = host_gen(nd.b, nd.s, col, mv);
            for (int k = 0; k < m; k++) {
                HostNode ch{nd.b, nd.s, Hash128{0, 0}, nd.paths};
                u32 cs = nd.s;
                host_make(ch.b, cs, col, mv[k]);
                ch.s = (uint8_t)cs;
                if (tt) {
                    ch.h = hash_move(nd.h, nd.b, nd.s, cs, col, mv[k]);
                    auto it = index.find(ch.h);
                    if (it != index.end()) {
                        next[it->second].paths += nd.paths;
                        continue;
                    }
                    index.emplace(ch.h, (u32)next.size());
                }
                next.push_back(ch);
            }
            if (next.size() > MAX_HOST_NODES) {
                // too wide to hold: walk this call depth first instead
                return launch_recurse(ctx, root, root_st, c, depth, root_h, out);
            }
        }
        col = 1 - col;
        if (tt) {
            // answered by the host table at this remaining depth
            std::vector<HostNode> keep;
            keep.reserve(next.size());
            for (const HostNode &nd : next) {
                u64 hit;
                if (rem - 1 >= 2 && ctx->htt.probe(rem - 1, nd.h, &hit))
                    add_product(total, nd.paths, hit);
                else
                    keep.push_back(nd);
            }
            next.swap(keep);
        }
        level.swap(next);
    }
    const int d = std::min(ld, depth);
    const u64 n = level.size();
    if (n) {
        std::vector<u64> vals(n, 0);
        int rc = PB_OK;
        if (!ctx->gpu) {
            for (u64 k = 0; k < n; k++) vals[k] = host_perft(level[k].b, level[k].s, col, d, ctx->opts.strict != 0);
        } else if (ctx->opts.use_tt) {
            std::vector<Board> rb(n);
            std::vector<uint8_t> rs(n);
            std::vector<Hash128> rh(n);
            for (u64 k = 0; k < n; k++) {
                rb[k] = level[k].b;
                rs[k] = level[k].s;
                rh[k] = level[k].h;
            }
            rc = gpu_tt_roots(ctx, rb.data(), rs.data(), rh.data(), n, col, d, vals.data());
        } else {
            // count-then-allocate batches of white-to-move roots
            std::vector<Board> rb(n);
            std::vector<uint8_t> rs(n);
            for (u64 k = 0; k < n; k++) {
                pb_pos p;
                to_pos(level[k].b, level[k].s, col, p);
                to_white_to_move(p, rb[k], rs[k]);
            }
            rc = gpu_batch(ctx, rb.data(), rs.data(), n, d, vals.data());
        }
        if (rc != PB_OK) return rc;
        for (u64 k = 0; k < n; k++) {
            add_product(total, level[k].paths, vals[k]);
            if (tt && d >= 2) ctx->htt.store(d, level[k].h, vals[k]);
        }
    }
    *out = total;
    return PB_OK;
}

// Listed-piece counting against the bitboard counter on every child of
// `y` (side Z to move): the lists of side 1-Z are taken from y, as the fused
// leaf takes them from its child position.  Compares both counters (reference
// and strict conventions) and, for children not in check, the not-in-check
// counter; returns the number of disagreements, *checked the children compared
// (0 when a kind has more than four pieces).
template <int Z>
u64 check_listed_t(const Board &y, u32 ys, u64 *checked)
{
    constexpr int C = 1 - Z;
    u32 lists[3];
    u64 listed;
    *checked = 0;
    if (!ListedPieces::build<C>(y, lists, &listed)) return 0;
    const ListedView own{lists, &listed};
    uint16_t mv[MAX_MOVES];
    ArraySink sink{mv, 0};
    gen_moves<Z>(y, ys, sink);
    u64 bad = 0;
    for (int k = 0; k < sink.n; k++) {
        Board g = y;
        u32 gs = ys;
        make_move<Z>(g, gs, mv[k]);
        bad += count_moves<C, false>(g, gs) != count_moves<C, false>(g, gs, own);
        bad += count_moves<C, true>(g, gs) != count_moves<C, true>(g, gs, own);
        const CountPrep p = count_prep<C>(g);
        if (!prep_in_check<C>(p)) {
            bad += count_quiet<C, false>(p.s, gs, p.pinned, p.threat, p.ksq) !=
                   count_quiet<C, false>(p.s, gs, p.pinned, p.threat, p.ksq, own);
            bad += count_quiet<C, true>(p.s, gs, p.pinned, p.threat, p.ksq) !=
                   count_quiet<C, true>(p.s, gs, p.pinned, p.threat, p.ksq, own);
        }
        ++*checked;
    }
    return bad;
}

// Launch depth: the deepest GPU call whose BFS levels fit half the arena,
// from the root's branching factor (estimateLaunchDepth, launcher.cu:533-562).
int estimate_launch_depth(pb_ctx *ctx, const Board &b, u32 st, int c)
{
    double p1 = (double)host_perft(b, st, c, 1, true);
    double p2 = (double)host_perft(b, st, c, 2, true);
    double p3 = (double)host_perft(b, st, c, 3, true);
    if (p1 < 1 || p2 < 1 || p3 < 1) return 6;
    double bf = 0.5 * (sqrt((p3 / p2) * (p2 / p1)) + 0.5 * ((p3 / p2) + (p2 / p1)));
    bf = std::max(bf, 2.0);
    // a GPU call of depth L materialises about bf^(L-2) edges of ~6 B and
    // bf^(L-3) positions of ~45 B; allow a factor 4 for uneven subtrees
    double budget = (double)ctx->arena_bytes / 4.0;
    int ld = 3;
    for (int L = 4; L <= 12; L++) {
        double need = 6.0 * pow(bf, L - 2) + 45.0 * pow(bf, L - 3);
        if (need > budget) break;
        ld = L;
    }
    return std::max(ld, 4);
}

}  // namespace

// ---------------------------------------------------------------- allocation-free scan
// Scratch of pb_scan_u32_noalloc: the scan's tile status words, its tile
// ticket and its error word live in this fixed device array instead of memory
// the caller or the engine allocates.  Every GPU that loads the library holds
// it (8.25 KB: 1,024 status words and 32 spare words) until the process exits.
constexpr u64 NOALLOC_SCAN_MAX_ITEMS = 8388608;                       // counts per call
constexpr u64 NOALLOC_SCAN_TILES = NOALLOC_SCAN_MAX_ITEMS / SCAN_TILE;  // status words
static_assert(NOALLOC_SCAN_TILES * SCAN_TILE == NOALLOC_SCAN_MAX_ITEMS,
              "the status words cover exactly the largest allowed scan");
static __device__ __align__(256) u64 g_noalloc_scratch[NOALLOC_SCAN_TILES + 32];

// ==================================================================== C ABI
extern "C" {

const char *pb_version(void) { return PB_VERSION; }

void pb_default_opts(pb_opts *o)
{
    memset(o, 0, sizeof(*o));
    o->use_tt = 1;
}

int pb_create(int device, const pb_opts *opts, pb_ctx **out)
{
    if (!out) return PB_ERR_ARG;
    *out = nullptr;
    if (!build_host_tables()) return PB_ERR_ARG;
    pb_ctx *ctx = new pb_ctx();
    if (opts)
        ctx->opts = *opts;
    else
        pb_default_opts(&ctx->opts);
    ctx->device = device;
    if (device >= 0) {
        int count = 0;
        cudaError_t e = cudaGetDeviceCount(&count);
        if (e != cudaSuccess || count == 0 || device >= count) {
            delete ctx;
            return PB_ERR_NODEVICE;
        }
        ctx->gpu = true;
        int rc = PB_OK;
        do {
            if ((e = cudaSetDevice(device)) != cudaSuccess) { rc = cuda_fail(ctx, e, "cudaSetDevice"); break; }
            if ((e = cudaMemcpyToSymbol(g_attacks, h_attacks, sizeof(h_attacks))) != cudaSuccess) { rc = cuda_fail(ctx, e, "upload attacks"); break; }
            void *dev_att = nullptr;
            if ((e = cudaGetSymbolAddress(&dev_att, g_attacks)) != cudaSuccess) { rc = cuda_fail(ctx, e, "attack table address"); break; }
            {
                Tables dt = device_tables(reinterpret_cast<const u64 *>(dev_att));
                if ((e = cudaMemcpyToSymbol(g_tab, &dt, sizeof(Tables))) != cudaSuccess) { rc = cuda_fail(ctx, e, "upload tables"); break; }
            }
            if ((e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking)) != cudaSuccess) { rc = cuda_fail(ctx, e, "stream"); break; }
            char *small = nullptr;
            if ((e = cudaMalloc(&small, 256)) != cudaSuccess) { rc = cuda_fail(ctx, e, "scratch"); break; }
            ctx->d_counter = reinterpret_cast<unsigned long long *>(small);  // two words
            ctx->d_err = reinterpret_cast<u32 *>(small + 64);
            ctx->d_ticket = reinterpret_cast<u32 *>(small + 128);
            ctx->d_total = reinterpret_cast<u64 *>(small + 192);
            if ((e = cudaMallocHost(&ctx->h_pinned, 4096)) != cudaSuccess) { rc = cuda_fail(ctx, e, "pinned"); break; }
            if ((e = cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device)) != cudaSuccess) { rc = cuda_fail(ctx, e, "sm count"); break; }
            ctx->spill_blocks = (size_t)ctx->num_sms * 8;
            if ((e = cudaMalloc(&ctx->spill, ctx->spill_blocks * LEAF_T * LEAF_OVF * sizeof(uint16_t))) != cudaSuccess) { rc = cuda_fail(ctx, e, "spill"); break; }
            size_t freeb = 0, totalb = 0;
            cudaMemGetInfo(&freeb, &totalb);
            size_t want = ctx->opts.arena_bytes;
            if (!want) {
                // no TT: half of free memory up to 32 GiB; TT mode keeps room for the tables
                size_t cap = ctx->opts.use_tt ? (16ULL << 30) : (32ULL << 30);
                want = std::min(freeb / 2, cap);
            }
            if ((e = cudaMalloc(&ctx->arena, want)) != cudaSuccess) { rc = cuda_fail(ctx, e, "arena"); break; }
            ctx->arena_bytes = want;
            build_zobrist();
            if ((e = cudaMemcpyToSymbol(g_zob, &h_zob, sizeof(Zobrist))) != cudaSuccess) { rc = cuda_fail(ctx, e, "upload keys"); break; }
            ctx->dtt_free_bytes = freeb > want + (4ULL << 30) ? freeb - want - (4ULL << 30) : 0;
        } while (0);
        if (rc != PB_OK) {
            std::string msg = ctx->err;
            pb_destroy(ctx);
            return rc;
        }
        if (ctx->opts.verbose)
            printf("Allocated BFS buffer: %llu MB\n", (unsigned long long)(ctx->arena_bytes >> 20));
    }
    *out = ctx;
    return PB_OK;
}

void pb_destroy(pb_ctx *ctx)
{
    if (!ctx) return;
    if (ctx->gpu) {
        cudaSetDevice(ctx->device);
        if (ctx->stream) cudaStreamSynchronize(ctx->stream);
        ctx->dtt.release();
        ctx->mlp.release();
        if (ctx->graph.exec) cudaGraphExecDestroy(ctx->graph.exec);
        for (int i = 0; i < 4; i++)
            if (ctx->ev[i]) cudaEventDestroy(ctx->ev[i]);
        if (ctx->arena) cudaFree(ctx->arena);
        if (ctx->d_counter) cudaFree(ctx->d_counter);
        if (ctx->spill) cudaFree(ctx->spill);
        if (ctx->h_pinned) cudaFreeHost(ctx->h_pinned);
        if (ctx->stream) cudaStreamDestroy(ctx->stream);
    }
    delete ctx;
}

const char *pb_last_error(const pb_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int pb_parse_fen(const char *fen, pb_pos *out)
{
    if (!fen || !out) return PB_ERR_ARG;
    build_host_tables();
    return parse_fen(fen, out) ? PB_OK : PB_ERR_FEN;
}

int pb_to_fen(const pb_pos *pos, char *buf, size_t len)
{
    if (!pos || !buf || len < 96) return PB_ERR_ARG;
    write_fen(*pos, buf);
    return PB_OK;
}

int pb_count_moves(const pb_pos *pos, int strict)
{
    if (!pos) return PB_ERR_ARG;
    build_host_tables();
    return (int)host_count(to_board(*pos), pos->state, pos->color, strict != 0);
}

int pb_generate_moves(const pb_pos *pos, uint16_t *moves)
{
    if (!pos || !moves) return PB_ERR_ARG;
    build_host_tables();
    return host_gen(to_board(*pos), pos->state, pos->color, moves);
}

int pb_position_hash(const pb_pos *pos, pb_u128 *out)
{
    if (!pos || !out) return PB_ERR_ARG;
    build_zobrist();
    const Hash128 h = hash_position(to_board(*pos), pos->state, pos->color);
    out->lo = h.lo;
    out->hi = h.hi;
    return PB_OK;
}

int pb_hash_after_move(const pb_u128 *key, const pb_pos *pos, uint16_t move, pb_u128 *out)
{
    if (!key || !pos || !out) return PB_ERR_ARG;
    build_zobrist();
    const Board b = to_board(*pos);
    Board after = b;
    u32 st = pos->state;
    host_make(after, st, pos->color, move);
    const Hash128 h = hash_move(Hash128{key->lo, key->hi}, b, pos->state, st, pos->color, move);
    out->lo = h.lo;
    out->hi = h.hi;
    return PB_OK;
}

int pb_make_move(pb_pos *pos, uint16_t move)
{
    if (!pos) return PB_ERR_ARG;
    Board b = to_board(*pos);
    u32 st = pos->state;
    host_make(b, st, pos->color, move);
    to_pos(b, st, 1 - pos->color, *pos);
    return PB_OK;
}

void pb_u128_add(pb_u128 *acc, const pb_u128 *v)
{
    if (acc && v) add128(*acc, *v);
}

int pb_u128_text(const pb_u128 *v, char *buf, size_t len)
{
    if (!v) return PB_ERR_ARG;
    return u128_decimal(*v, buf, len);
}

int pb_selftest_listed_counts(const pb_pos *pos, int n, uint64_t *checked, uint64_t *mismatches)
{
    if (!pos || n < 0 || !checked || !mismatches) return PB_ERR_ARG;
    build_host_tables();
    *checked = 0;
    *mismatches = 0;
    for (int i = 0; i < n; i++) {
        u64 c = 0;
        Board y = to_board(pos[i]);
        *mismatches += pos[i].color == WHITE ? check_listed_t<WHITE>(y, pos[i].state, &c)
                                             : check_listed_t<BLACK>(y, pos[i].state, &c);
        *checked += c;
    }
    return PB_OK;
}

int pb_perft_cpu(pb_ctx *ctx, const pb_pos *pos, int depth, uint64_t *count)
{
    if (!pos || !count || depth < 0) return PB_ERR_ARG;
    build_host_tables();
    bool strict = ctx ? ctx->opts.strict != 0 : false;
    *count = host_perft(to_board(*pos), pos->state, pos->color, depth, strict);
    return PB_OK;
}

int pb_perft_position(pb_ctx *ctx, const pb_pos *pos, int depth, uint64_t *count)
{
    if (!ctx || !pos || !count || depth < 0 || depth > 20) return PB_ERR_ARG;
    if (!ctx->gpu) return fail(ctx, PB_ERR_NODEVICE, "context has no GPU");
    PB_CUDA(cudaSetDevice(ctx->device));
    memset(&ctx->stats, 0, sizeof(ctx->stats));
    int rc = gpu_perft(ctx, to_board(*pos), pos->state, pos->color, depth, reinterpret_cast<u64 *>(count));
    ctx->stats.nodes = *count;
    return rc;
}

int pb_set_timing(pb_ctx *ctx, int enable)
{
    if (!ctx || !ctx->gpu) return PB_ERR_ARG;
    PB_CUDA(cudaSetDevice(ctx->device));
    if (enable && !ctx->ev[0])
        for (int i = 0; i < 4; i++) PB_CUDA(cudaEventCreate(&ctx->ev[i]));
    ctx->timing = enable != 0;
    return PB_OK;
}

int pb_set_tuning(pb_ctx *ctx, const pb_tuning *t)
{
    if (!ctx || !t) return PB_ERR_ARG;
    if (t->leaf_kernel) {
        if (t->leaf_kernel < 1 || t->leaf_kernel > 6) return PB_ERR_ARG;
        ctx->tuning.leaf_kernel = t->leaf_kernel;
    }
    if (t->leaf_blocks_per_sm) {
        if (t->leaf_blocks_per_sm < 0 || t->leaf_blocks_per_sm > 8) return PB_ERR_ARG;
        ctx->tuning.leaf_blocks_per_sm = t->leaf_blocks_per_sm;
    }
    if (t->leaf_threads) {
        const int lk = t->leaf_kernel ? t->leaf_kernel : ctx->tuning.leaf_kernel;
        if (t->leaf_threads != 128 && t->leaf_threads != 256 && t->leaf_threads != 512 &&
            !(t->leaf_threads == 1024 && lk == 6))
            return PB_ERR_ARG;
        ctx->tuning.leaf_threads = t->leaf_threads;
    }
    if (t->gen_threads) {
        if (t->gen_threads != 64 && t->gen_threads != 128) return PB_ERR_ARG;
        ctx->tuning.gen_threads = t->gen_threads;
    }
    if (t->leaf_fuse) {
        if (t->leaf_fuse != 1 && t->leaf_fuse != 2) return PB_ERR_ARG;
        ctx->tuning.leaf_fuse = t->leaf_fuse;
    }
    if (t->tt_replace) {
        if (t->tt_replace != 1 && t->tt_replace != 2) return PB_ERR_ARG;
        if (t->tt_replace != ctx->tuning.tt_replace) {
            ctx->tuning.tt_replace = t->tt_replace;
            ctx->dtt.release();  // resized (and re-laid-out) on the next TT call
            ctx->dtt_max_depth = 0;
        }
    }
    if (t->planned_leaf) {
        if (t->planned_leaf != 1 && t->planned_leaf != 2) return PB_ERR_ARG;
        ctx->tuning.planned_leaf = t->planned_leaf;
    }
    if (t->host_driver) {
        if (t->host_driver != 1 && t->host_driver != 2) return PB_ERR_ARG;
        ctx->tuning.host_driver = t->host_driver;
    }
    if (t->tt_leaf) {
        if (t->tt_leaf != 1 && t->tt_leaf != 2) return PB_ERR_ARG;
        ctx->tuning.tt_leaf = t->tt_leaf;
    }
    return PB_OK;
}

int pb_get_tuning(const pb_ctx *ctx, pb_tuning *t)
{
    if (!ctx || !t) return PB_ERR_ARG;
    *t = ctx->tuning;
    return PB_OK;
}

int pb_last_stats(const pb_ctx *ctx, pb_stats *out)
{
    if (!ctx || !out) return PB_ERR_ARG;
    *out = ctx->stats;
    return PB_OK;
}

int pb_device_count(void)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
    return n;
}

int pb_choose_launch_depth(pb_ctx *ctx, const pb_pos *pos)
{
    if (!ctx || !pos) return PB_ERR_ARG;
    build_host_tables();
    if (!ctx->launch_depth)
        ctx->launch_depth = ctx->opts.launch_depth > 0
                                ? ctx->opts.launch_depth
                                : (ctx->gpu ? estimate_launch_depth(ctx, to_board(*pos), pos->state, pos->color) : 64);
    return ctx->launch_depth;
}

int pb_prepare(pb_ctx *ctx, const pb_pos *pos, int max_depth)
{
    if (!ctx || !pos || max_depth < 0 || max_depth > 30) return PB_ERR_ARG;
    // With tables the BFS levels shrink (hits and duplicates are not
    // expanded), so deep runs call the GPU one ply higher, as the reference
    // does for perft 10 and beyond (perft.cu:126-130).
    if (ctx->gpu && ctx->opts.use_tt && ctx->opts.launch_depth <= 0 && !ctx->launch_depth && max_depth >= 10)
        ctx->launch_depth = std::max(estimate_launch_depth(ctx, to_board(*pos), pos->state, pos->color), 9);
    int ld = pb_choose_launch_depth(ctx, pos);
    if (ctx->gpu && ctx->opts.use_tt) {
        int rc = ensure_dtt(ctx, std::min(ld, max_depth) - 1);
        if (rc != PB_OK) return rc;
    }
    if (ctx->opts.use_tt && (!ctx->htt.ready() || ctx->htt_last < max_depth)) {
        ctx->htt.init(ctx->opts.host_tt_mb, ld, max_depth);
        ctx->htt_last = max_depth;
    }
    return ld;
}

int pb_perft_launch(pb_ctx *ctx, const pb_pos *pos, int depth, pb_u128 *count, double *seconds)
{
    if (!ctx || !pos || !count || depth < 0 || depth > 30) return PB_ERR_ARG;
    if (ctx->gpu) PB_CUDA(cudaSetDevice(ctx->device));
    Board b = to_board(*pos);
    pb_choose_launch_depth(ctx, pos);
    if (ctx->opts.use_tt && (!ctx->htt.ready() || ctx->htt_last < depth)) {
        ctx->htt.init(ctx->opts.host_tt_mb, ctx->launch_depth, depth);
        ctx->htt_last = depth;
    }
    auto t0 = std::chrono::steady_clock::now();
    pb_u128 r{0, 0};
    int rc;
    if (depth == 0) {
        r.lo = 1;
        rc = PB_OK;
    } else {
        Hash128 h = ctx->opts.use_tt ? hash_position(b, pos->state, pos->color) : Hash128{0, 0};
        const bool tt = ctx->opts.use_tt && ctx->htt.ready();
        u64 hit = 0;
        if (ctx->tuning.host_driver == 2 && depth > ctx->launch_depth) {
            if (tt && ctx->htt.probe(depth, h, &hit)) {
                r.lo = hit;
                rc = PB_OK;
            } else {
                rc = launch_breadth_first(ctx, b, pos->state, pos->color, depth, h, &r);
                if (rc == PB_OK && tt && r.hi == 0) ctx->htt.store(depth, h, r.lo);
            }
        } else {
            rc = launch_recurse(ctx, b, pos->state, pos->color, depth, h, &r);
        }
    }
    auto t1 = std::chrono::steady_clock::now();
    if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
    *count = r;
    return rc;
}

int pb_perft(pb_ctx *ctx, const char *fen, int max_depth, pb_u128 *per_depth, double *per_depth_secs)
{
    if (!ctx || !fen || !per_depth || max_depth < 1 || max_depth > 30) return PB_ERR_ARG;
    pb_pos pos;
    if (!parse_fen(fen, &pos)) return fail(ctx, PB_ERR_FEN, "invalid FEN");
    pb_prepare(ctx, &pos, max_depth);
    for (int d = 1; d <= max_depth; d++) {
        double secs = 0;
        int rc = pb_perft_launch(ctx, &pos, d, &per_depth[d - 1], &secs);
        if (rc != PB_OK) return rc;
        if (per_depth_secs) per_depth_secs[d - 1] = secs;
    }
    return PB_OK;
}

int pb_random_playout(uint64_t *rng_state, int plies, pb_pos *out)
{
    if (!rng_state || !out || plies < 0) return PB_ERR_ARG;
    build_host_tables();
    return playout(reinterpret_cast<u64 *>(rng_state), plies, out);
}

int pb_random_playouts(uint64_t seed, int n, int min_plies, int max_plies, pb_pos *out, int *played)
{
    if (!out || n < 0 || min_plies < 0 || max_plies < min_plies) return PB_ERR_ARG;
    build_host_tables();
    // per-position generator states: the i-th draw of the master stream
    std::vector<u64> seeds(n);
    u64 master = seed;
    for (int i = 0; i < n; i++) seeds[i] = splitmix64(&master);
    const u64 span = (u64)(max_plies - min_plies + 1);
    unsigned nt = std::max(1u, std::min(std::thread::hardware_concurrency(), 64u));
    std::vector<std::thread> pool;
    for (unsigned t = 0; t < nt; t++)
        pool.emplace_back([&, t]() {
            for (int i = (int)t; i < n; i += (int)nt) {
                u64 st = seeds[i];
                int plies = min_plies + (int)(((unsigned __int128)splitmix64(&st) * span) >> 64);
                int k = playout(&st, plies, &out[i]);
                if (played) played[i] = k;
            }
        });
    for (auto &th : pool) th.join();
    return PB_OK;
}

int pb_perft_batch(pb_ctx *ctx, const pb_pos *roots, const int *depths, int n, uint64_t *counts)
{
    if (!ctx || !roots || !depths || !counts || n < 0) return PB_ERR_ARG;
    if (!ctx->gpu) return fail(ctx, PB_ERR_NODEVICE, "context has no GPU");
    PB_CUDA(cudaSetDevice(ctx->device));
    memset(&ctx->stats, 0, sizeof(ctx->stats));
    // one batched pass per distinct depth
    std::vector<int> ds(depths, depths + n);
    std::sort(ds.begin(), ds.end());
    ds.erase(std::unique(ds.begin(), ds.end()), ds.end());
    for (int d : ds) {
        if (d < 0 || d > 20) return PB_ERR_ARG;
        std::vector<int> idx;
        for (int i = 0; i < n; i++)
            if (depths[i] == d) idx.push_back(i);
        std::vector<Board> rb(idx.size());
        std::vector<uint8_t> rs(idx.size());
        for (size_t k = 0; k < idx.size(); k++) to_white_to_move(roots[idx[k]], rb[k], rs[k]);
        std::vector<u64> out(idx.size());
        int rc = gpu_batch(ctx, rb.data(), rs.data(), idx.size(), d, out.data());
        if (rc != PB_OK) return rc;
        for (size_t k = 0; k < idx.size(); k++) {
            counts[idx[k]] = out[k];
            ctx->stats.nodes += out[k];
        }
    }
    return PB_OK;
}

int pb_dev_scan(pb_ctx *ctx, const uint32_t *d_in, uint64_t n, uint64_t *d_out, uint64_t *d_total)
{
    if (!ctx || !ctx->gpu || !d_in || !d_out || !d_total) return PB_ERR_ARG;
    if (n == 0) return PB_OK;
    PB_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    u64 tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    Arena ar{ctx->arena, ctx->arena_bytes};
    u64 *status = ar.take<u64>(tiles);
    if (!status) return fail(ctx, PB_ERR_NOMEM, "arena too small for scan status");
    PB_CUDA(cudaMemsetAsync(status, 0, sizeof(u64) * tiles, s));
    PB_CUDA(cudaMemsetAsync(ctx->d_ticket, 0, sizeof(u32), s));
    PB_CUDA(cudaMemsetAsync(ctx->d_err, 0, sizeof(u32), s));
    k_scan<<<(unsigned)tiles, SCAN_THREADS, 0, s>>>(d_in, n, reinterpret_cast<u64 *>(d_out), status, ctx->d_ticket, reinterpret_cast<u64 *>(d_total), ctx->d_err);
    PB_CUDA(cudaGetLastError());
    PB_CUDA(cudaMemcpyAsync(ctx->h_pinned + 1, ctx->d_err, sizeof(u32), cudaMemcpyDeviceToHost, s));
    PB_CUDA(cudaStreamSynchronize(s));
    if ((u32)ctx->h_pinned[1]) return fail(ctx, PB_ERR_DEVICE, "scan reported a device error");
    return PB_OK;
}

// Finishes a test launch: waits, reads the error word.
static int finish_test_launch(pb_ctx *ctx, const char *what)
{
    cudaStream_t s = ctx->stream;
    PB_CUDA(cudaGetLastError());
    PB_CUDA(cudaMemcpyAsync(ctx->h_pinned + 1, ctx->d_err, sizeof(u32), cudaMemcpyDeviceToHost, s));
    PB_CUDA(cudaStreamSynchronize(s));
    if ((u32)ctx->h_pinned[1]) return fail(ctx, PB_ERR_DEVICE, what);
    return PB_OK;
}

int pb_dev_expand(pb_ctx *ctx, const void *d_boards, const uint8_t *d_states, int color, const uint32_t *d_pidx,
                  const uint16_t *d_moves, uint64_t n, uint64_t nparents, void *d_child_boards,
                  uint8_t *d_child_states, uint32_t *d_counts)
{
    if (!ctx || !ctx->gpu || !d_boards || !d_states || !d_pidx || !d_moves || !d_child_boards || !d_child_states ||
        !d_counts || (color != WHITE && color != BLACK))
        return PB_ERR_ARG;
    if (((uintptr_t)d_boards | (uintptr_t)d_child_boards) & 31) return PB_ERR_ARG;  // 256-bit accesses
    if (n == 0) return PB_OK;
    PB_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    PB_CUDA(cudaMemsetAsync(ctx->d_err, 0, sizeof(u32), s));
    const Board *pb_ = static_cast<const Board *>(d_boards);
    Board *cb = static_cast<Board *>(d_child_boards);
    if (color == WHITE)
        k_expand_count<WHITE><<<grid_for(n, 256), 256, 0, s>>>(pb_, d_states, d_pidx, d_moves, n, nparents, cb,
                                                               d_child_states, d_counts, ctx->d_err);
    else
        k_expand_count<BLACK><<<grid_for(n, 256), 256, 0, s>>>(pb_, d_states, d_pidx, d_moves, n, nparents, cb,
                                                               d_child_states, d_counts, ctx->d_err);
    return finish_test_launch(ctx, "make+count kernel reported a device error");
}

int pb_dev_generate(pb_ctx *ctx, const void *d_boards, const uint8_t *d_states, int color, const uint64_t *d_offs,
                    const uint64_t *d_total, uint64_t n, uint16_t *d_moves, uint32_t *d_pidx)
{
    if (!ctx || !ctx->gpu || !d_boards || !d_states || !d_offs || !d_total || !d_moves || !d_pidx ||
        (color != WHITE && color != BLACK))
        return PB_ERR_ARG;
    if ((uintptr_t)d_boards & 31) return PB_ERR_ARG;
    if (n == 0) return PB_OK;
    PB_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    PB_CUDA(cudaMemsetAsync(ctx->d_err, 0, sizeof(u32), s));
    const Board *pb_ = static_cast<const Board *>(d_boards);
    const u64 *offs = reinterpret_cast<const u64 *>(d_offs);
    const u64 *total = reinterpret_cast<const u64 *>(d_total);
    if (color == WHITE)
        k_generate<WHITE, GEN_THREADS><<<grid_for(n, GEN_THREADS), GEN_THREADS, 0, s>>>(pb_, d_states, offs, total, n,
                                                                                      d_moves, d_pidx, ctx->d_err);
    else
        k_generate<BLACK, GEN_THREADS><<<grid_for(n, GEN_THREADS), GEN_THREADS, 0, s>>>(pb_, d_states, offs, total, n,
                                                                                      d_moves, d_pidx, ctx->d_err);
    return finish_test_launch(ctx, "generation kernel reported a device error");
}

int pb_selftest_tt_race(pb_ctx *ctx, int mode, uint64_t *bad, uint64_t *hits)
{
    if (!ctx || !ctx->gpu || !bad || !hits || mode < 0 || mode > 2) return PB_ERR_ARG;
    PB_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    const bool deep = mode == 1, packed = mode == 2;
    // far fewer slots than keys (constant collisions); mode 2: the smallest
    // shallow table the engine builds, with every key packed into 8 slots
    const u64 slots = packed ? (1ULL << 24) : 1024;
    Arena ar{ctx->arena, ctx->arena_bytes};
    u64 *entries = ar.take<u64>(slots * (deep ? 4 : 2));
    unsigned long long *cnt = ar.take<unsigned long long>(2);
    if (!entries || !cnt) return fail(ctx, PB_ERR_NOMEM, "arena too small for the self-test");
    PB_CUDA(cudaMemsetAsync(entries, 0, slots * (deep ? 32 : 16), s));
    PB_CUDA(cudaMemsetAsync(cnt, 0, 2 * sizeof(unsigned long long), s));
    const TTView t{entries, slots, deep ? TT_DEEP : TT_SHALLOW, 0};
    k_tt_race<<<4 * ctx->num_sms, 256, 0, s>>>(t, 8192, 64, packed ? 1u : 0u, cnt, cnt + 1);
    PB_CUDA(cudaGetLastError());
    PB_CUDA(cudaMemcpyAsync(ctx->h_pinned, cnt, 2 * sizeof(u64), cudaMemcpyDeviceToHost, s));
    PB_CUDA(cudaStreamSynchronize(s));
    *bad = ctx->h_pinned[0];
    *hits = ctx->h_pinned[1];
    return PB_OK;
}

int pb_selftest_wait_timeout(pb_ctx *ctx, uint32_t *device_error, double *seconds)
{
    if (!ctx || !ctx->gpu || !device_error) return PB_ERR_ARG;
    PB_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    // two scan tiles, one CTA: it draws ticket 1, so tile 0 (whose prefix
    // tile 1 waits for) is never published and the wait has to give up
    const u64 n = 2 * (u64)SCAN_TILE;
    Arena ar{ctx->arena, ctx->arena_bytes};
    u32 *in = ar.take<u32>(n);
    u64 *out = ar.take<u64>(n);
    u64 *status = ar.take<u64>(2);
    u64 *total = ar.take<u64>(1);
    if (!in || !out || !status || !total) return fail(ctx, PB_ERR_NOMEM, "arena too small for the self-test");
    PB_CUDA(cudaMemsetAsync(in, 0, sizeof(u32) * n, s));
    PB_CUDA(cudaMemsetAsync(status, 0, 2 * sizeof(u64), s));
    PB_CUDA(cudaMemsetAsync(ctx->d_err, 0, sizeof(u32), s));
    ctx->h_pinned[3] = 1;
    PB_CUDA(cudaMemcpyAsync(ctx->d_ticket, &ctx->h_pinned[3], sizeof(u32), cudaMemcpyHostToDevice, s));
    PB_CUDA(cudaStreamSynchronize(s));
    const auto t0 = std::chrono::steady_clock::now();
    k_scan<<<1, SCAN_THREADS, 0, s>>>(in, n, out, status, ctx->d_ticket, total, ctx->d_err);
    PB_CUDA(cudaGetLastError());
    PB_CUDA(cudaMemcpyAsync(ctx->h_pinned + 1, ctx->d_err, sizeof(u32), cudaMemcpyDeviceToHost, s));
    PB_CUDA(cudaStreamSynchronize(s));
    if (seconds) *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    *device_error = (u32)ctx->h_pinned[1];
    return PB_OK;
}

int pb_scan_u32_noalloc(const uint32_t *d_in, uint64_t n, uint64_t *d_out, uint64_t *d_total, void *stream)
{
    if (!d_in || !d_out || !d_total) return PB_ERR_ARG;
    if (n > NOALLOC_SCAN_MAX_ITEMS) return PB_ERR_ARG;  // beyond the fixed scratch
    if (n == 0) return PB_OK;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    // the call waits for its stream, which a capture cannot record
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cap) != cudaSuccess) return PB_ERR_CUDA;
    if (cap != cudaStreamCaptureStatusNone) return PB_ERR_ARG;
    build_host_tables();
    // The device address of the array, looked up on every call with the
    // caller's device current: the lookup allocates nothing, and a context
    // reset (which reloads the module and may move the array) cannot leave a
    // stale address behind.  The first call on a device loads the module.
    void *addr = nullptr;
    if (cudaGetSymbolAddress(&addr, g_noalloc_scratch) != cudaSuccess || !addr) return PB_ERR_CUDA;
    u64 *scratch = reinterpret_cast<u64 *>(addr);
    const u64 tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    u64 *status = scratch;
    u32 *ticket = reinterpret_cast<u32 *>(scratch + NOALLOC_SCAN_TILES);
    u32 *err = reinterpret_cast<u32 *>(scratch + NOALLOC_SCAN_TILES + 1);
    // status words, ticket and error word must start at zero; the array keeps
    // whatever the previous call left
    if (cudaMemsetAsync(status, 0, sizeof(u64) * tiles, s) != cudaSuccess) return PB_ERR_CUDA;
    if (cudaMemsetAsync(ticket, 0, 2 * sizeof(u64), s) != cudaSuccess) return PB_ERR_CUDA;
    k_scan<<<(unsigned)tiles, SCAN_THREADS, 0, s>>>(d_in, n, reinterpret_cast<u64 *>(d_out), status, ticket,
                                                     reinterpret_cast<u64 *>(d_total), err);
    if (cudaGetLastError() != cudaSuccess) return PB_ERR_CUDA;
    u32 herr = 0;
    if (cudaMemcpyAsync(&herr, err, sizeof(u32), cudaMemcpyDeviceToHost, s) != cudaSuccess) return PB_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return PB_ERR_CUDA;
    return herr ? PB_ERR_DEVICE : PB_OK;
}

// ---------------------------------------------------------------- learned scheduler network
size_t pb_mlp_param_count(void) { return MLP_PARAMS; }

int pb_mlp_init(pb_ctx *ctx, uint64_t seed, const float *out_bias)
{
    if (!ctx || !ctx->gpu) return PB_ERR_ARG;
    PB_CUDA(cudaSetDevice(ctx->device));
    PB_CUDA(ctx->mlp.init(seed, out_bias, ctx->stream));
    PB_CUDA(cudaStreamSynchronize(ctx->stream));
    return PB_OK;
}

int pb_mlp_get_params(pb_ctx *ctx, float *out, size_t count)
{
    if (!ctx || !ctx->mlp.ready || !out || count != MLP_PARAMS) return PB_ERR_ARG;
    PB_CUDA(cudaSetDevice(ctx->device));
    PB_CUDA(cudaMemcpyAsync(out, ctx->mlp.p, MLP_PARAMS * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
    PB_CUDA(cudaStreamSynchronize(ctx->stream));
    return PB_OK;
}

int pb_mlp_set_params(pb_ctx *ctx, const float *in, size_t count)
{
    if (!ctx || !ctx->mlp.ready || !in || count != MLP_PARAMS) return PB_ERR_ARG;
    PB_CUDA(cudaSetDevice(ctx->device));
    PB_CUDA(ctx->mlp.set_params(in, ctx->stream));
    PB_CUDA(cudaStreamSynchronize(ctx->stream));
    return PB_OK;
}

// The network's GEMM error word (set when a tensor-core wait gave up), read
// here unless the caller already copied it (*copied): PB_ERR_DEVICE if it
// was set, and the word is cleared.
static int mlp_check(pb_ctx *ctx, const u32 *copied = nullptr)
{
    u32 e = 0;
    if (copied)
        e = *copied;
    else
        PB_CUDA(cudaMemcpy(&e, ctx->mlp.err, sizeof(u32), cudaMemcpyDeviceToHost));
    if (!e) return PB_OK;
    PB_CUDA(cudaMemset(ctx->mlp.err, 0, sizeof(u32)));
    return fail(ctx, PB_ERR_DEVICE, "tensor-core GEMM: an mbarrier wait timed out");
}

int pb_selftest_gemm(pb_ctx *ctx, int ta, int tb, int M, int N, int K, const uint16_t *a, const uint16_t *b,
                     float *c, int reps, double *ms)
{
    if (!ctx || !a || !b || !c || M <= 0 || M % 8 || N <= 0 || N % tc::BN || K <= 0 || K % tc::BK || reps < 0 ||
        (reps > 0 && !ms))
        return PB_ERR_ARG;
    if (!ctx->gpu) return fail(ctx, PB_ERR_NODEVICE, "context has no GPU");
    PB_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t s = ctx->stream;
    const size_t na = (size_t)M * K, nb = (size_t)K * N, nc = (size_t)M * N;
    __nv_bfloat16 *da = nullptr, *db = nullptr;
    float *dc = nullptr, *dw = nullptr;
    u32 *derr = nullptr;
    int rc = PB_OK;
    // workspace for as many K splits as the product would use
    const size_t nw = (size_t)gemm_splits(M, N, K, (size_t)-1) * M * N;
    cudaError_t e = cudaMalloc(&da, na * 2);
    if (e == cudaSuccess) e = cudaMalloc(&dw, nw * 4);
    if (e == cudaSuccess) e = cudaMalloc(&db, nb * 2);
    if (e == cudaSuccess) e = cudaMalloc(&dc, nc * 4);
    if (e == cudaSuccess) e = cudaMalloc(&derr, sizeof(u32));
    if (e == cudaSuccess) e = cudaMemcpyAsync(da, a, na * 2, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(db, b, nb * 2, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(derr, 0, sizeof(u32), s);
    const int lda = ta ? M : K, ldb = tb ? K : N;
    auto launch = [&]() {
        if (ta && tb) return gemm_tc<true, true>(da, lda, db, ldb, dc, N, M, N, K, derr, dw, nw, s);
        if (ta) return gemm_tc<true, false>(da, lda, db, ldb, dc, N, M, N, K, derr, dw, nw, s);
        if (tb) return gemm_tc<false, true>(da, lda, db, ldb, dc, N, M, N, K, derr, dw, nw, s);
        return gemm_tc<false, false>(da, lda, db, ldb, dc, N, M, N, K, derr, dw, nw, s);
    };
    if (e == cudaSuccess) e = launch();
    if (e == cudaSuccess && reps > 0) {
        // the same product `reps` more times between two events on the stream
        for (int i = 0; i < 4 && e == cudaSuccess; i++)
            if (!ctx->ev[i]) e = cudaEventCreate(&ctx->ev[i]);
        if (e == cudaSuccess) e = cudaEventRecord(ctx->ev[0], s);
        for (int r = 0; r < reps && e == cudaSuccess; r++) e = launch();
        if (e == cudaSuccess) e = cudaEventRecord(ctx->ev[1], s);
        float t = 0;
        if (e == cudaSuccess) e = cudaEventSynchronize(ctx->ev[1]);
        if (e == cudaSuccess) e = cudaEventElapsedTime(&t, ctx->ev[0], ctx->ev[1]);
        if (e == cudaSuccess) *ms = (double)t / reps;
    }
    u32 herr = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(c, dc, nc * 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, derr, sizeof(u32), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) rc = cuda_fail(ctx, e, "gemm self-test");
    else if (herr) rc = fail(ctx, PB_ERR_DEVICE, "tensor-core GEMM: an mbarrier wait timed out");
    cudaFree(da);
    cudaFree(db);
    cudaFree(dc);
    cudaFree(dw);
    cudaFree(derr);
    return rc;
}

// Loss and parameter gradients of one batch (n a multiple of 64), no update.
int pb_mlp_gradients(pb_ctx *ctx, const pb_pos *pos, const float *targets, int n, float *grads, float *loss)
{
    if (!ctx || !ctx->mlp.ready || !pos || !targets || n <= 0 || n % 64) return PB_ERR_ARG;
    PB_CUDA(cudaSetDevice(ctx->device));
    Mlp &m = ctx->mlp;
    cudaStream_t s = ctx->stream;
    PB_CUDA(m.alloc_batch(n));
    PB_CUDA(m.load_positions(pos, n, s));
    PB_CUDA(cudaMemcpyAsync(m.t, targets, sizeof(float) * MLP_OUT * n, cudaMemcpyHostToDevice, s));
    PB_CUDA(m.forward_backward(n, true, s));
    if (grads) PB_CUDA(cudaMemcpyAsync(grads, m.g, MLP_PARAMS * sizeof(float), cudaMemcpyDeviceToHost, s));
    float l = 0;
    PB_CUDA(cudaMemcpyAsync(&l, m.loss, sizeof(float), cudaMemcpyDeviceToHost, s));
    PB_CUDA(cudaStreamSynchronize(s));
    if (loss) *loss = l / (float)(n * MLP_OUT);
    return mlp_check(ctx);
}

// Adam training on n examples: `epochs` passes over a fresh shuffle each, in
// batches of `batch` (a multiple of 64; the tail that does not fill a batch
// is left out of that epoch).  *final_loss = mean squared error of the last
// epoch.
int pb_mlp_train(pb_ctx *ctx, const pb_pos *pos, const float *targets, int n, int epochs, int batch, float lr,
                 uint64_t seed, float *final_loss)
{
    if (!ctx || !ctx->mlp.ready || !pos || !targets || n <= 0 || batch <= 0 || batch % 64 || epochs <= 0)
        return PB_ERR_ARG;
    PB_CUDA(cudaSetDevice(ctx->device));
    Mlp &m = ctx->mlp;
    cudaStream_t s = ctx->stream;
    PB_CUDA(m.alloc_batch(batch));
    // The training set goes to the device once (feature indices and
    // targets); every step gathers its batch there, so a step is kernel
    // launches only and the host reads the loss once per epoch.
    DeviceBuffer<int16_t> all_idx;
    DeviceBuffer<float> all_t;
    DeviceBuffer<int> order_d;
    DeviceBuffer<double> acc;
    PB_CUDA(all_idx.alloc((size_t)n * MLP_MAX_ACTIVE));
    PB_CUDA(all_t.alloc((size_t)n * MLP_OUT));
    PB_CUDA(order_d.alloc((size_t)n));
    PB_CUDA(acc.alloc(1));
    for (int c0 = 0; c0 < n; c0 += batch) {
        const int k = std::min(batch, n - c0);
        PB_CUDA(m.features_to(pos + c0, k, all_idx.p + (size_t)c0 * MLP_MAX_ACTIVE, s));
    }
    PB_CUDA(cudaMemcpyAsync(all_t.p, targets, sizeof(float) * MLP_OUT * (size_t)n, cudaMemcpyHostToDevice, s));
    std::vector<int> order(n);
    for (int i = 0; i < n; i++) order[i] = i;
    u64 rng = seed;
    double epoch_loss = 0;
    const int V = MLP_MAX_ACTIVE * (int)sizeof(int16_t) / 16 + 1;  // gather threads per row
    for (int ep = 0; ep < epochs; ep++) {
        for (int i = n - 1; i > 0; i--) {
            u64 r = splitmix64(&rng);
            int j = (int)(((unsigned __int128)r * (u64)(i + 1)) >> 64);
            std::swap(order[i], order[j]);
        }
        PB_CUDA(cudaMemcpyAsync(order_d.p, order.data(), sizeof(int) * (size_t)n, cudaMemcpyHostToDevice, s));
        PB_CUDA(cudaMemsetAsync(acc.p, 0, sizeof(double), s));
        int steps = 0;
        for (int b0 = 0; b0 + batch <= n; b0 += batch) {
            k_gather_batch<<<(batch * V + 255) / 256, 256, 0, s>>>(all_idx.p, all_t.p, order_d.p, b0, batch, m.idx,
                                                                  m.t);
            PB_CUDA(m.forward_backward(batch, true, s));
            PB_CUDA(m.adam_step(lr, s));
            k_accum_loss<<<1, 32, 0, s>>>(m.loss, acc.p, 1.0 / (double)(batch * MLP_OUT));
            steps++;
        }
        PB_CUDA(cudaGetLastError());
        double total = 0;
        PB_CUDA(cudaMemcpyAsync(&total, acc.p, sizeof(double), cudaMemcpyDeviceToHost, s));
        PB_CUDA(cudaStreamSynchronize(s));
        epoch_loss = steps ? total / steps : 0.0;
    }
    if (final_loss) *final_loss = (float)epoch_loss;
    return mlp_check(ctx);
}

// Predicted log2(1 + perft(k)), k = 1..4, for n positions (out: n x 4).
int pb_mlp_predict(pb_ctx *ctx, const pb_pos *pos, int n, float *out)
{
    if (!ctx || !ctx->mlp.ready || !pos || !out || n < 0) return PB_ERR_ARG;
    if (n == 0) return PB_OK;
    PB_CUDA(cudaSetDevice(ctx->device));
    Mlp &m = ctx->mlp;
    cudaStream_t s = ctx->stream;
    const int chunk = 8192;
    PB_CUDA(m.alloc_batch(chunk));
    for (int b0 = 0; b0 < n; b0 += chunk) {
        int k = std::min(chunk, n - b0);
        int padded = (k + 63) / 64 * 64;
        std::vector<pb_pos> tmp(pos + b0, pos + b0 + k);
        tmp.resize(padded, pos[b0]);
        PB_CUDA(m.load_positions(tmp.data(), padded, s));
        PB_CUDA(m.forward_backward(padded, false, s));
        PB_CUDA(cudaMemcpyAsync(out + (size_t)b0 * MLP_OUT, m.y, sizeof(float) * MLP_OUT * k, cudaMemcpyDeviceToHost, s));
        PB_CUDA(cudaMemcpyAsync(ctx->h_pinned + 3, m.err, sizeof(u32), cudaMemcpyDeviceToHost, s));
        PB_CUDA(cudaStreamSynchronize(s));
        const u32 e = (u32)ctx->h_pinned[3];
        if (e) return mlp_check(ctx, &e);
    }
    return PB_OK;
}

int pb_perft_batch_planned(pb_ctx *ctx, const pb_pos *roots, const int *depths, int n, uint64_t *counts,
                           pb_plan_stats *stats)
{
    if (!ctx || !roots || !depths || !counts || n < 0) return PB_ERR_ARG;
    if (!ctx->gpu) return fail(ctx, PB_ERR_NODEVICE, "context has no GPU");
    if (!ctx->mlp.ready) return fail(ctx, PB_ERR_ARG, "planner needs a trained network (pb_mlp_init/train)");
    for (int i = 0; i < n; i++)
        if (depths[i] < 0 || depths[i] > 12) return PB_ERR_ARG;
    PB_CUDA(cudaSetDevice(ctx->device));
    memset(&ctx->stats, 0, sizeof(ctx->stats));
    if (stats) memset(stats, 0, sizeof(*stats));
    int rc = plan_and_run(ctx, roots, depths, n, counts, stats);
    for (int i = 0; i < n && rc == PB_OK; i++) ctx->stats.nodes += counts[i];
    return rc;
}

}  // extern "C"
