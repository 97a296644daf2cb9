// pb_kernels.cuh - sm_100a kernels of the breadth-first perft engine.
//
// A BFS level is a list of edges (parent index u32, move u16) over the
// previous level's positions (Board 32 B + state 1 B, structure of arrays).
// Per level the host launches
//   k_expand_count  make each edge's move, store the child position and its
//                   exact legal-move count
//   k_scan_*        decoupled look-back exclusive scan of the counts (u64)
//   k_generate      write every child's moves as the next level's edges,
//                   staged through shared memory so global stores coalesce
// and the last two plies run in k_leaf2 (fused: make, generate, then count
// every grandchild).  These replace, in order, the reference's
// makemove_and_count_moves_kernel (perft_kernels.cu:201-257), CUB
// InclusiveSum (:786), merge_path_partitions + mp_interval_expand_kernel +
// generate_moves_kernel (:77-173, :263-311) and fused_2level_leaf_kernel
// (:405-480).  The interval expand (child slot -> parent index) is done
// inside k_generate: each parent writes its own index next to each of its
// moves in the shared-memory tile, so no separate search pass is needed.
#pragma once
#include "pb_core.cuh"

namespace pb {

// 256-bit position load/store (one ld/st.global.v4.u64 on sm_100).
__device__ __forceinline__ Board load_board(const Board *p)
{
    Board b;
    asm volatile("ld.global.nc.v4.u64 {%0,%1,%2,%3}, [%4];"
                 : "=l"(b.bb[0]), "=l"(b.bb[1]), "=l"(b.bb[2]), "=l"(b.bb[3])
                 : "l"(p));
    return b;
}
__device__ __forceinline__ void store_board(Board *p, const Board &b)
{
    asm volatile("st.global.v4.u64 [%0], {%1,%2,%3,%4};" ::"l"(p), "l"(b.bb[0]), "l"(b.bb[1]), "l"(b.bb[2]),
                 "l"(b.bb[3])
                 : "memory");
}

// Device-side error word: kernels OR a code in and return instead of trapping.
enum : u32 {
    DEVERR_SCAN_TIMEOUT = 1u,
    DEVERR_CAPACITY = 2u,
};

// ---------------------------------------------------------------- expand/count
// Child c of edge e: board/state written at index e, count[e] = exact number
// of moves of the child (side to move 1-C).
template <int C>
__global__ void __launch_bounds__(256) k_expand_count(const Board *__restrict__ pboards,
                                                      const uint8_t *__restrict__ pstates,
                                                      const u32 *__restrict__ pidx,
                                                      const uint16_t *__restrict__ moves, u64 n, u64 nparents,
                                                      Board *__restrict__ cboards, uint8_t *__restrict__ cstates,
                                                      u32 *__restrict__ counts, u32 *__restrict__ err)
{
    u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    u32 p = pidx[i];
    if (p >= nparents) {  // only after a count/generation mismatch upstream
        atomicOr(err, DEVERR_CAPACITY);
        counts[i] = 0;
        return;
    }
    Board b = load_board(pboards + p);
    u32 st = pstates[p];
    make_move<C>(b, st, moves[i]);
    store_board(cboards + i, b);
    cstates[i] = (uint8_t)st;
    counts[i] = count_moves<1 - C, true>(b, st);
}

// ---------------------------------------------------------------- scan
// Decoupled look-back exclusive scan of u32 counts into u64 offsets; the
// grand total lands in *total.  Tile status words: [63:62] flag (1 = tile
// aggregate, 2 = inclusive prefix), [61:0] value.  Tiles are taken in launch
// order from an atomic ticket so every predecessor is already resident.
// 32 counts per thread: the scan is bound by each CTA's load -> look-back ->
// store latency, so a larger tile moves more bytes per round trip (measured
// on B200: 8 -> 16 -> 32 counts per thread = 2.3 -> 2.9 -> 3.4 TB/s at 400 M
// counts; 64, or 512 threads, gain nothing more).
constexpr int SCAN_THREADS = 256;
constexpr int SCAN_ITEMS = 32;  // a multiple of 8
constexpr int SCAN_TILE = SCAN_THREADS * SCAN_ITEMS;
constexpr u64 ST_AGG = 1ULL << 62, ST_PREFIX = 2ULL << 62, ST_VALUE = (1ULL << 62) - 1;
constexpr u32 SCAN_SPIN_LIMIT = 1u << 20;  // look-back rounds (about a second) before giving up

__device__ __forceinline__ void st_release(u64 *p, u64 v)
{
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ u64 ld_acquire(const u64 *p)
{
    u64 v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

// Exclusive prefix of `tile` by decoupled look-back, run by one whole warp:
// each step reads the status words of 32 predecessors at once, adds every
// aggregate up to the nearest inclusive prefix, and retries while one of
// those is not yet published.  Publishes the tile's aggregate first and its
// inclusive prefix last.  Every lane returns the same value.  A wait longer
// than SCAN_SPIN_LIMIT rounds sets DEVERR_SCAN_TIMEOUT and gives up.
__device__ __forceinline__ u64 scan_lookback(u64 *status, u32 tile, u64 block_total, u32 *err)
{
    const int lane = threadIdx.x & 31;
    if (tile == 0) {
        if (lane == 0) st_release(status, ST_PREFIX | block_total);
        return 0;
    }
    if (lane == 0) st_release(status + tile, ST_AGG | block_total);
    u64 excl = 0;
    long long p = (long long)tile - 1;
    u32 spins = 0;
    while (true) {
        const long long q = p - lane;
        const u64 w = q >= 0 ? ld_acquire(status + q) : ST_PREFIX;
        const u32 flag = (u32)(w >> 62);
        const unsigned not_ready = __ballot_sync(0xffffffffu, flag == 0);
        const unsigned prefix = __ballot_sync(0xffffffffu, flag == 2);
        // lanes from the nearest predecessor up to the nearest inclusive prefix
        const unsigned upto = prefix ? (prefix & (0u - prefix)) * 2u - 1u : 0xffffffffu;
        if (not_ready & upto) {
            if (++spins > SCAN_SPIN_LIMIT) {
                if (lane == 0) atomicOr(err, DEVERR_SCAN_TIMEOUT);
                break;
            }
            continue;
        }
        u64 v = ((upto >> lane) & 1u) ? (w & ST_VALUE) : 0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        excl += v;
        if (prefix) break;
        p -= 32;
    }
    if (lane == 0) st_release(status + tile, ST_PREFIX | (excl + block_total));
    return excl;
}

// One tile of the scan: SCAN_ITEMS consecutive counts per thread, read and
// written with 256-bit accesses when both arrays are 32-byte aligned (the
// engine's arena always is; callers' pointers may not be).
__device__ __forceinline__ void scan_tile(const u32 *__restrict__ in, u64 n, u64 *__restrict__ out, u64 *status,
                                          u32 tile, u64 *__restrict__ total, u32 *__restrict__ err)
{
    static_assert(SCAN_ITEMS % 8 == 0, "the vector path moves counts in 32-byte groups of 8");
    __shared__ u64 s_warp[SCAN_THREADS / 32];
    __shared__ u64 s_exclusive;
    const u64 base = (u64)tile * SCAN_TILE + (u64)threadIdx.x * SCAN_ITEMS;
    const bool vec = ((reinterpret_cast<uintptr_t>(in) | reinterpret_cast<uintptr_t>(out)) & 31) == 0 &&
                     base + SCAN_ITEMS <= n;
    u32 v[SCAN_ITEMS];
    if (vec) {
#pragma unroll
        for (int g = 0; g < SCAN_ITEMS; g += 8) {
            u64 a, b, c, d;
            asm("ld.global.nc.v4.u64 {%0,%1,%2,%3}, [%4];" : "=l"(a), "=l"(b), "=l"(c), "=l"(d) : "l"(in + base + g));
            v[g + 0] = (u32)a, v[g + 1] = (u32)(a >> 32), v[g + 2] = (u32)b, v[g + 3] = (u32)(b >> 32);
            v[g + 4] = (u32)c, v[g + 5] = (u32)(c >> 32), v[g + 6] = (u32)d, v[g + 7] = (u32)(d >> 32);
        }
    } else {
#pragma unroll
        for (int k = 0; k < SCAN_ITEMS; k++) v[k] = (base + k < n) ? in[base + k] : 0u;
    }
    u64 local = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; k++) local += v[k];
    // block-wide exclusive scan of the per-thread sums
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    u64 x = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        u64 y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        u64 w = (lane < SCAN_THREADS / 32) ? s_warp[lane] : 0;
#pragma unroll
        for (int o = 1; o < SCAN_THREADS / 32; o <<= 1) {
            u64 y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < SCAN_THREADS / 32) s_warp[lane] = w;
        __syncwarp();
        const u64 block_total = s_warp[SCAN_THREADS / 32 - 1];
        const u64 excl = scan_lookback(status, tile, block_total, err);
        if (lane == 0) {
            s_exclusive = excl;
            if ((u64)(tile + 1) * SCAN_TILE >= n) *total = excl + block_total;
        }
    }
    __syncthreads();
    u64 run = s_exclusive + x - local + (warp ? s_warp[warp - 1] : 0);
    if (vec) {
#pragma unroll
        for (int g = 0; g < SCAN_ITEMS; g += 4) {
            Board o;  // four offsets, one 256-bit store
            o.bb[0] = run, run += v[g];
            o.bb[1] = run, run += v[g + 1];
            o.bb[2] = run, run += v[g + 2];
            o.bb[3] = run, run += v[g + 3];
            store_board(reinterpret_cast<Board *>(out + base + g), o);
        }
    } else {
#pragma unroll
        for (int k = 0; k < SCAN_ITEMS; k++) {
            if (base + k < n) out[base + k] = run;
            run += v[k];
        }
    }
}

__global__ void __launch_bounds__(SCAN_THREADS) k_scan(const u32 *__restrict__ in, u64 n, u64 *__restrict__ out,
                                                       u64 *__restrict__ status, u32 *__restrict__ ticket,
                                                       u64 *__restrict__ total, u32 *__restrict__ err)
{
    __shared__ u32 s_tile;
    if (threadIdx.x == 0) s_tile = atomicAdd(ticket, 1u);
    __syncthreads();
    scan_tile(in, n, out, status, s_tile, total, err);
}

// ---------------------------------------------------------------- generate
// Each thread owns one position of the level; its moves go to
// [offs[i], offs[i] + counts[i]) of the next level as (parent i, move).
constexpr int GEN_THREADS = 128;
// Staged moves per thread of a CTA.  A staged move takes 3 bytes of shared
// memory: the move and the index of the thread (position) that owns it; the
// copy-out turns that index into the global parent index.
// Against 6 bytes (move + global parent index) this raised the resident
// warps from 16 to 36 per SM and cut the generation time 1.64x on B200; 48
// instead of 64 moves per thread, or a register cap for more warps, gained
// nothing more.
constexpr int GEN_MPT = 64;
constexpr int GEN_CAP = GEN_THREADS * GEN_MPT;  // moves staged per CTA of k_generate_dev

// Both sinks stop at `cap` moves: the level was sized with the exact count,
// so more moves than that means the count and the generator disagree; the
// excess is dropped and reported through the error word instead of being
// written past the allocation.
struct SmemSink {
    uint16_t *mv;
    uint8_t *owner;  // thread index of the position each move belongs to
    uint8_t me;
    int n, cap;
    bool over;
    __device__ __forceinline__ void put(uint16_t m)
    {
        if (n < cap) {
            mv[n] = m;
            owner[n] = me;
        } else {
            over = true;
        }
        n++;
    }
};
struct GlobalSink {
    uint16_t *mv;
    u32 *pi;
    u32 parent;
    u64 n, cap;
    bool over;
    __device__ __forceinline__ void put(uint16_t m)
    {
        if (n < cap) {
            mv[n] = m;
            pi[n] = parent;
        } else {
            over = true;
        }
        n++;
    }
};

template <int C, int GT = GEN_THREADS>
__global__ void __launch_bounds__(GT) k_generate(const Board *__restrict__ boards,
                                             const uint8_t *__restrict__ states,
                                             const u64 *__restrict__ offs, const u64 *__restrict__ total,
                                             u64 n, uint16_t *__restrict__ out_mv,
                                             u32 *__restrict__ out_pi, u32 *__restrict__ err)
{
    static_assert(GT <= 256, "owner indices are one byte");
    constexpr int CAP = GT * GEN_MPT;  // staged moves per CTA (3 B each)
    __shared__ uint16_t s_mv[CAP];
    __shared__ uint8_t s_own[CAP];
    const u64 first = (u64)blockIdx.x * GT;
    const u64 last = min(first + GT, n);  // exclusive
    const u64 tile_begin = offs[first];
    const u64 tile_end = (last < n) ? offs[last] : *total;
    const u64 i = first + threadIdx.x;
    const bool staged = (tile_end - tile_begin) <= (u64)CAP;
    if (i < n) {
        Board b = load_board(boards + i);
        u32 st = states[i];
        const u64 mine_begin = offs[i];
        const u64 mine_end = (i + 1 < n) ? offs[i + 1] : *total;
        bool over = false;
        if (mine_end == mine_begin) {
            // no moves allotted: mate, stalemate, a TT hit or a duplicate
        } else if (staged) {
            SmemSink s{s_mv, s_own, (uint8_t)threadIdx.x, (int)(mine_begin - tile_begin),
                       (int)(mine_end - tile_begin), false};
            gen_moves<C>(b, st, s);
            over = s.over || s.n != s.cap;
        } else {
            GlobalSink s{out_mv, out_pi, (u32)i, mine_begin, mine_end, false};
            gen_moves<C>(b, st, s);
            over = s.over || s.n != s.cap;
        }
        if (over) atomicOr(err, DEVERR_CAPACITY);
    }
    if (!staged) return;
    __syncthreads();
    const int cnt = (int)(tile_end - tile_begin);
    for (int k = threadIdx.x; k < cnt; k += GT) {
        out_mv[tile_begin + k] = s_mv[k];
        out_pi[tile_begin + k] = (u32)first + s_own[k];
    }
}

// ---------------------------------------------------------------- leaves
// Sum over the moves mv[0..n) of child b of their grandchildren's move counts
// (each move made on a copy of b, then counted).  With LISTED the counts
// iterate the child's own-piece lists (ListedPieces, read back through
// ListedView from this thread's slot of a shared-memory array of T slots); a
// child with more than four pieces of one kind counts with bitboard scans.
// Leaf modes of the ranked leaves: 0 = unranked, 1 = the CTA's children
// ranked by move count, 2 = ranked and counted with listed pieces.
template <int C, bool STRICT, bool LISTED, int T>
__device__ __forceinline__ u32 grandchild_counts(const Board &b, u32 st, const uint16_t *mv, int n)
{
    u32 total = 0;
    if (LISTED) {
        __shared__ u32 s_lists[T][3];
        __shared__ u64 s_listed[T];
        u32 *l = s_lists[threadIdx.x];
        u64 *m = &s_listed[threadIdx.x];
        if (ListedPieces::build<C>(b, l, m)) {
            const ListedView own{l, m};
            for (int k = 0; k < n; k++) {
                Board g = b;
                u32 gs = st;
                make_move<1 - C>(g, gs, mv[k]);
                total += count_moves<C, STRICT>(g, gs, own);
            }
            return total;
        }
    }
    for (int k = 0; k < n; k++) {
        Board g = b;
        u32 gs = st;
        make_move<1 - C>(g, gs, mv[k]);
        total += count_moves<C, STRICT>(g, gs);
    }
    return total;
}

// One-ply leaf: the move count of each edge's child (perft 1 of the child).
template <int C, bool STRICT>
__global__ void __launch_bounds__(256) k_leaf1(const Board *__restrict__ pboards, const uint8_t *__restrict__ pstates,
                                               const u32 *__restrict__ pidx, const uint16_t *__restrict__ moves, u64 n,
                                               u64 nparents, unsigned long long *__restrict__ counter)
{
    u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    u32 cnt = 0;
    if (i < n && pidx[i] < nparents) {
        u32 p = pidx[i];
        Board b = load_board(pboards + p);
        u32 st = pstates[p];
        make_move<C>(b, st, moves[i]);
        cnt = count_moves<1 - C, STRICT>(b, st);
    }
    cnt = __reduce_add_sync(0xffffffffu, cnt);
    if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(counter, (unsigned long long)cnt);
}

// Fused two-ply leaf: perft 2 of each edge's child, summed.
// counter[0] += leaf nodes, counter[1] += positions counted (move-count calls).
// Block size and the minimum resident blocks per SM trade registers against
// warps in flight; the kernel is ALU-pipe bound, so enough warps must be
// resident to keep the pipe fed through the table-load latency.
#ifndef PB_LEAF_THREADS
#define PB_LEAF_THREADS 256
#endif
#ifndef PB_LEAF_MIN_BLOCKS
#define PB_LEAF_MIN_BLOCKS 4
#endif
template <int C, bool STRICT, int T = PB_LEAF_THREADS>
__global__ void __launch_bounds__(T, 1024 / T) k_leaf2(const Board *__restrict__ pboards, const uint8_t *__restrict__ pstates,
                                               const u32 *__restrict__ pidx, const uint16_t *__restrict__ moves, u64 n,
                                               u64 nparents, unsigned long long *__restrict__ counter)
{
    u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    u32 total = 0, counted = 0;
    if (i < n && pidx[i] < nparents) {
        u32 p = pidx[i];
        Board b = load_board(pboards + p);
        u32 st = pstates[p];
        make_move<C>(b, st, moves[i]);
        uint16_t mv[MAX_MOVES];
        ArraySink sink{mv, 0};
        gen_moves<1 - C>(b, st, sink);
        for (int k = 0; k < sink.n; k++) {
            Board g = b;
            u32 gs = st;
            make_move<1 - C>(g, gs, mv[k]);
            total += count_moves<C, STRICT>(g, gs);
        }
        counted = sink.n;
    }
    total = __reduce_add_sync(0xffffffffu, total);
    counted = __reduce_add_sync(0xffffffffu, counted);
    if ((threadIdx.x & 31) == 0 && counted) {
        atomicAdd(counter, (unsigned long long)total);
        atomicAdd(counter + 1, (unsigned long long)counted);
    }
}

}  // namespace pb

namespace pb {

// ---------------------------------------------------------------- balanced leaf
// Fused two-ply leaf with the CTA's children handed to threads in order of
// their move counts.  In k_leaf2 a warp runs as many grandchild iterations as
// its longest move list, so lanes with short lists idle (about 11 % of the
// lane-iterations on sibling edges).  Here each thread makes its edge's child
// and counts its moves; a shared-memory histogram of those counts (every
// count is below 256) ranks the T children, and the child of rank r moves to
// thread r, which generates the moves and counts every grandchild.  Warps then
// hold children with similar move counts.  Costs one extra count per child
// (about 1/31 of the work) and 34 B of shared memory per thread.  Measured on
// B200 against k_leaf2: +2.5 % on the bench position, +1.6 % on Kiwipete with
// 256-thread CTAs; 128 or 512 threads, or a pseudo-legal count as the key,
// balance worse.
// Ranks of this thread's K keys (each < 256) among the K * T keys of its CTA,
// ascending; equal keys get distinct ranks in arbitrary order.  `below1` =
// how many keys are 0.  A shared-memory histogram and its exclusive prefix;
// every thread of the CTA must call it.
template <int T, int K>
__device__ __forceinline__ void cta_rank_u8(const u32 (&key)[K], u32 (&rank)[K], u32 *below1 = nullptr)
{
    __shared__ u32 s_hist[256];
    __shared__ u32 s_wsum[T / 32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int k = tid; k < 256; k += T) s_hist[k] = 0;
    __syncthreads();
    u32 slot[K];
#pragma unroll
    for (int k = 0; k < K; k++) slot[k] = atomicAdd(&s_hist[key[k]], 1u);
    __syncthreads();
    constexpr int PER = T >= 256 ? 1 : 256 / T;
    u32 h[PER], local = 0;
#pragma unroll
    for (int k = 0; k < PER; k++) {
        h[k] = (tid * PER + k < 256) ? s_hist[tid * PER + k] : 0u;
        local += h[k];
    }
    u32 x = local;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        u32 y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_wsum[warp] = x;
    __syncthreads();
    u32 base = x - local;
    for (int w = 0; w < warp; w++) base += s_wsum[w];
#pragma unroll
    for (int k = 0; k < PER; k++) {
        if (tid * PER + k < 256) s_hist[tid * PER + k] = base;
        base += h[k];
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < K; k++) rank[k] = s_hist[key[k]] + slot[k];
    if (below1) *below1 = s_hist[1];
    __syncthreads();  // s_hist is free again for the next call
}
template <int T> __device__ __forceinline__ u32 cta_rank_u8(u32 key)
{
    u32 k[1] = {key}, r[1];
    cta_rank_u8<T, 1>(k, r);
    return r[0];
}

template <int C, bool STRICT, int T>
__global__ void __launch_bounds__(T, 1024 / T) k_leaf2_sorted(const Board *__restrict__ pboards,
                                                              const uint8_t *__restrict__ pstates,
                                                              const u32 *__restrict__ pidx,
                                                              const uint16_t *__restrict__ moves, u64 n, u64 nparents,
                                                              unsigned long long *__restrict__ counter)
{
    __shared__ Board s_b[T];
    __shared__ uint8_t s_st[T];
    __shared__ uint8_t s_key[T];  // 0 = no child, else 1 + its move count
    const int tid = threadIdx.x;
    const u64 i = (u64)blockIdx.x * T + tid;
    Board b{};
    u32 st = 0, key = 0;
    if (i < n && pidx[i] < nparents) {
        u32 p = pidx[i];
        b = load_board(pboards + p);
        st = pstates[p];
        make_move<C>(b, st, moves[i]);
        key = 1 + min(count_moves<1 - C, true>(b, st), 254u);
    }
    const u32 rank = cta_rank_u8<T>(key);
    s_b[rank] = b;
    s_st[rank] = (uint8_t)st;
    s_key[rank] = (uint8_t)key;
    __syncthreads();
    u32 total = 0, counted = 0;
    if (s_key[tid]) {
        b = s_b[tid];
        st = s_st[tid];
        uint16_t mv[MAX_MOVES];
        ArraySink sink{mv, 0};
        gen_moves<1 - C>(b, st, sink);
        for (int k = 0; k < sink.n; k++) {
            Board g = b;
            u32 gs = st;
            make_move<1 - C>(g, gs, mv[k]);
            total += count_moves<C, STRICT>(g, gs);
        }
        counted = sink.n;
    }
    total = __reduce_add_sync(0xffffffffu, total);
    counted = __reduce_add_sync(0xffffffffu, counted);
    if ((tid & 31) == 0 && counted) {
        atomicAdd(counter, (unsigned long long)total);
        atomicAdd(counter + 1, (unsigned long long)counted);
    }
}

// Ranked two-ply leaf whose grandchild counts iterate the child's own-piece
// lists (ListedPieces) instead of scanning piece bitboards: every grandchild
// of a child has the pieces of side C that the child has, less at most one
// captured piece, so the knight and slider squares are listed once per child.
// A child with more than four pieces of one kind counts with the bitboard
// scans.  Same counts as k_leaf2_sorted.  Measured on B200 (perft 7 of the
// bench position): 21.16 ms against 21.97 ms for k_leaf2_sorted, 21.38 ms
// with the lists held in registers (which spilled).
#ifndef PB_LISTED_WARPS_PER_SM
#define PB_LISTED_WARPS_PER_SM 32  // resident warps the listed leaf is compiled for (64 registers)
#endif
template <int C, bool STRICT, int T>
__global__ void __launch_bounds__(T, PB_LISTED_WARPS_PER_SM * 32 / T) k_leaf2_listed(const Board *__restrict__ pboards,
                                                              const uint8_t *__restrict__ pstates,
                                                              const u32 *__restrict__ pidx,
                                                              const uint16_t *__restrict__ moves, u64 n, u64 nparents,
                                                              unsigned long long *__restrict__ counter)
{
    __shared__ Board s_b[T];
    __shared__ uint8_t s_st[T];
    __shared__ uint8_t s_key[T];  // 0 = no child, else 1 + its move count
    const int tid = threadIdx.x;
    const u64 i = (u64)blockIdx.x * T + tid;
    Board b{};
    u32 st = 0, key = 0;
    if (i < n && pidx[i] < nparents) {
        u32 p = pidx[i];
        b = load_board(pboards + p);
        st = pstates[p];
        make_move<C>(b, st, moves[i]);
        key = 1 + min(count_moves<1 - C, true>(b, st), 254u);
    }
    const u32 rank = cta_rank_u8<T>(key);
    s_b[rank] = b;
    s_st[rank] = (uint8_t)st;
    s_key[rank] = (uint8_t)key;
    __syncthreads();
    u32 total = 0, counted = 0;
    if (s_key[tid]) {
        b = s_b[tid];
        st = s_st[tid];
        uint16_t mv[MAX_MOVES];
        ArraySink sink{mv, 0};
        gen_moves<1 - C>(b, st, sink);
        total = grandchild_counts<C, STRICT, true, T>(b, st, mv, sink.n);
        counted = sink.n;
    }
    total = __reduce_add_sync(0xffffffffu, total);
    counted = __reduce_add_sync(0xffffffffu, counted);
    if ((tid & 31) == 0 && counted) {
        atomicAdd(counter, (unsigned long long)total);
        atomicAdd(counter + 1, (unsigned long long)counted);
    }
}

// ---------------------------------------------------------------- cooperative leaf
// Fused two-ply leaf with the grandchild work spread over the whole CTA.
//
// Per chunk of LEAF_T edges:
//   phase A  thread t makes edge t's move (child X_t in shared memory) and
//            generates X_t's moves into its column of a shared-memory move
//            table (moves beyond LEAF_CAP spill to a per-CTA global area);
//   scan     block-wide exclusive scan of the move counts, and an owner map
//            item -> t (one byte per item) built from it;
//   phase B  the chunk's N = sum n_t (child, move) items are dealt round-robin
//            to the CTA's threads: each item makes the move on X_owner and
//            counts the grandchild's moves.
// Adjacent lanes therefore count grandchildren of the same child, so a warp
// stays converged far better than with one edge per thread, and no thread
// idles while a neighbour finishes a long move list.
constexpr int LEAF_T = 256;
constexpr int LEAF_CAP = 40;                 // moves per child kept in shared memory
constexpr int LEAF_OVF = MAX_MOVES - LEAF_CAP;  // spill slots per child (global)

struct ColumnSink {
    uint16_t *col;   // shared: column t of a [LEAF_CAP][LEAF_T] table
    uint16_t *ovf;   // global spill slots of this child
    int n;
    __device__ __forceinline__ void put(uint16_t m)
    {
        if (n < LEAF_CAP)
            col[n * LEAF_T] = m;
        else
            ovf[n - LEAF_CAP] = m;
        n++;
    }
};

template <int C, bool STRICT>
__global__ void __launch_bounds__(LEAF_T, 4) k_leaf2_coop(const Board *__restrict__ pboards,
                                                          const uint8_t *__restrict__ pstates,
                                                          const u32 *__restrict__ pidx,
                                                          const uint16_t *__restrict__ moves, u64 n, u64 nparents,
                                                          uint16_t *__restrict__ spill,
                                                          unsigned long long *__restrict__ counter)
{
    __shared__ Board s_child[LEAF_T];
    __shared__ uint8_t s_cst[LEAF_T];
    __shared__ uint16_t s_mv[LEAF_CAP * LEAF_T];
    __shared__ u32 s_off[LEAF_T + 1];
    __shared__ uint8_t s_own[LEAF_CAP * LEAF_T];
    __shared__ u32 s_wsum[LEAF_T / 32];

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    uint16_t *my_spill = spill + ((u64)blockIdx.x * LEAF_T + tid) * LEAF_OVF;
    u64 total = 0, counted = 0;
    const u64 nchunks = (n + LEAF_T - 1) / LEAF_T;
    for (u64 chunk = blockIdx.x; chunk < nchunks; chunk += gridDim.x) {
        // ---- phase A: child position and its move list
        const u64 e = chunk * LEAF_T + tid;
        int cnt = 0;
        if (e < n && pidx[e] < nparents) {
            u32 p = pidx[e];
            Board b = load_board(pboards + p);
            u32 st = pstates[p];
            make_move<C>(b, st, moves[e]);
            s_child[tid] = b;
            s_cst[tid] = (uint8_t)st;
            ColumnSink sink{s_mv + tid, my_spill, 0};
            gen_moves<1 - C>(b, st, sink);
            cnt = sink.n;
        }
        // ---- block exclusive scan of cnt
        u32 x = (u32)cnt;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            u32 y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) s_wsum[warp] = x;
        __syncthreads();
        if (warp == 0) {
            u32 w = (lane < LEAF_T / 32) ? s_wsum[lane] : 0;
#pragma unroll
            for (int o = 1; o < LEAF_T / 32; o <<= 1) {
                u32 y = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= o) w += y;
            }
            if (lane < LEAF_T / 32) s_wsum[lane] = w;
        }
        __syncthreads();
        const u32 excl = x - (u32)cnt + (warp ? s_wsum[warp - 1] : 0);
        s_off[tid] = excl;
        if (tid == LEAF_T - 1) s_off[LEAF_T] = excl + (u32)cnt;
        const u32 items = s_wsum[LEAF_T / 32 - 1];
        counted += (tid == 0) ? items : 0;
        // ---- phase B in windows of LEAF_CAP * LEAF_T items (owner map size)
        for (u32 w0 = 0; w0 < items; w0 += LEAF_CAP * LEAF_T) {
            const u32 w1 = min(items, w0 + (u32)(LEAF_CAP * LEAF_T));
            // owner map for [w0, w1): thread t marks its items inside the window
            {
                u32 a = max(excl, w0), z = min(excl + (u32)cnt, w1);
                for (u32 k = a; k < z; k++) s_own[k - w0] = (uint8_t)tid;
            }
            __syncthreads();
            for (u32 i = w0 + tid; i < w1; i += LEAF_T) {
                const int t = s_own[i - w0];
                const u32 j = i - s_off[t];
                uint16_t m = (j < (u32)LEAF_CAP)
                                 ? s_mv[j * LEAF_T + t]
                                 : spill[((u64)blockIdx.x * LEAF_T + t) * LEAF_OVF + (j - LEAF_CAP)];
                Board g = s_child[t];
                u32 gs = s_cst[t];
                make_move<1 - C>(g, gs, m);
                total += count_moves<C, STRICT>(g, gs);
            }
            __syncthreads();
        }
        __syncthreads();  // s_wsum / s_child are rewritten by the next chunk
    }
    // ---- one atomic pair per warp
    unsigned long long t64 = total;
#pragma unroll
    for (int o = 16; o; o >>= 1) t64 += __shfl_xor_sync(0xffffffffu, t64, o);
    unsigned long long c64 = counted;
#pragma unroll
    for (int o = 16; o; o >>= 1) c64 += __shfl_xor_sync(0xffffffffu, c64, o);
    if (lane == 0) {
        if (t64) atomicAdd(counter, t64);
        if (c64) atomicAdd(counter + 1, c64);
    }
}

}  // namespace pb

namespace pb {

// ---------------------------------------------------------------- batched roots
// Batched BFS over many roots at once.  Roots are normalised on the host so
// that every root has white to move (a colour-flipped, rank-mirrored position
// has the same perft), which keeps each level one colour.  Every position
// carries the index of its root; the leaves add their counts to that root's
// counter, aggregating lanes of a warp that share a root first.

// Move count of each position (strict = sizing for the next level).
template <int C, bool STRICT>
__global__ void __launch_bounds__(256) k_count_positions(const Board *__restrict__ boards,
                                                         const uint8_t *__restrict__ states, u64 n,
                                                         u32 *__restrict__ counts)
{
    u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    counts[i] = count_moves<C, STRICT>(load_board(boards + i), states[i]);
}

template <int C>
__global__ void __launch_bounds__(256) k_expand_count_rooted(const Board *__restrict__ pboards,
                                                             const uint8_t *__restrict__ pstates,
                                                             const u32 *__restrict__ proot,
                                                             const u32 *__restrict__ pidx,
                                                             const uint16_t *__restrict__ moves, u64 n,
                                                             u64 nparents, Board *__restrict__ cboards,
                                                             uint8_t *__restrict__ cstates, u32 *__restrict__ croot,
                                                             u32 *__restrict__ counts, u32 *__restrict__ err)
{
    u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    u32 p = pidx[i];
    if (p >= nparents) {
        atomicOr(err, DEVERR_CAPACITY);
        counts[i] = 0;
        croot[i] = 0;
        return;
    }
    Board b = load_board(pboards + p);
    u32 st = pstates[p];
    make_move<C>(b, st, moves[i]);
    store_board(cboards + i, b);
    cstates[i] = (uint8_t)st;
    croot[i] = proot[p];
    counts[i] = count_moves<1 - C, true>(b, st);
}

// Adds v to out[key] once per group of lanes holding the same key (edges of
// one root are contiguous, so a warp usually forms one or two groups).
__device__ __forceinline__ void add_by_key(unsigned long long *out, u32 key, u32 v, bool valid)
{
    const unsigned active = __ballot_sync(0xffffffffu, valid);
    if (!valid) return;
    const unsigned peers = __match_any_sync(active, key);
    const u32 total = __reduce_add_sync(peers, v);
    if ((int)(threadIdx.x & 31) == __ffs(peers) - 1 && total) atomicAdd(out + key, (unsigned long long)total);
}

// Ranked leaf with work balanced across the CTA's warps (leaf kernel 6).  In
// the ranked leaves warp 0 gets the CTA's lightest children and the last warp
// the heaviest; a warp that finishes early keeps its registers until its
// CTA ends, so on the bench position only 26.6 of the 32 resident warps were
// active on average.  Here each thread makes K = PB_BALANCED_K children (the
// CTA covers KT edges) and counts their moves; the 4T children are ranked by move count
// and cut into 32-child chunks in rank order; chunk j is paired with chunk
// NCH - 1 - j (a light and a heavy one) and pair j goes to warp j % W, so
// every warp gets about the same work while the lanes of a chunk still have
// similar loop lengths.  Only edge indices pass through shared memory (4 B
// per child): each lane remakes its child from the parent and the move, then
// generates its moves and counts the grandchildren with listed pieces.
#ifndef PB_BALANCED_K
#define PB_BALANCED_K 4  // children per thread of k_leaf2_balanced
#endif
// With ROOTED every edge's count goes to its root's counter (batched roots).
template <int C, bool STRICT, int T, bool ROOTED>
__device__ __forceinline__ void leaf2_balanced_cta(const Board *__restrict__ pboards,
                                                   const uint8_t *__restrict__ pstates,
                                                   const u32 *__restrict__ proot, const u32 *__restrict__ pidx,
                                                   const uint16_t *__restrict__ moves, u64 n, u64 nparents,
                                                   unsigned long long *__restrict__ root_counts,
                                                   unsigned long long *__restrict__ counter)
{
    constexpr int K = PB_BALANCED_K;
    constexpr int W = T / 32;
    constexpr int NCH = K * T / 32;
    static_assert(K % 2 == 0 && NCH == K * W, "K/2 chunk pairs per warp");
    constexpr u32 NONE = 0xFFFFFFFFu;
    __shared__ u32 s_edge[K * T];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const u64 first = (u64)blockIdx.x * (K * T);
    u32 key[K], rank[K];
#pragma unroll
    for (int k = 0; k < K; k++) {
        const u64 i = first + (u64)k * T + tid;
        key[k] = 0;
        if (i < n && pidx[i] < nparents) {
            const u32 p = pidx[i];
            Board b = load_board(pboards + p);
            u32 st = pstates[p];
            make_move<C>(b, st, moves[i]);
            key[k] = 1 + min(count_moves<1 - C, true>(b, st), 254u);
        }
    }
    cta_rank_u8<T, K>(key, rank);
#pragma unroll
    for (int k = 0; k < K; k++) s_edge[rank[k]] = key[k] ? (u32)(first + (u64)k * T + tid) : NONE;
    __syncthreads();
    u32 total = 0, counted = 0;
    for (int q = 0; q < K; q++) {
        const int pair = warp + (q >> 1) * W;
        const int chunk = (q & 1) ? NCH - 1 - pair : pair;
        const u32 e = s_edge[chunk * 32 + lane];
        u32 t = 0, root = 0;
        if (e != NONE) {
            const u32 p = pidx[e];
            if (ROOTED) root = proot[p];
            Board b = load_board(pboards + p);
            u32 st = pstates[p];
            make_move<C>(b, st, moves[e]);
            uint16_t mv[MAX_MOVES];
            ArraySink sink{mv, 0};
            gen_moves<1 - C>(b, st, sink);
            t = grandchild_counts<C, STRICT, true, T>(b, st, mv, sink.n);
            counted += sink.n;
        }
        if (ROOTED)
            add_by_key(root_counts, root, t, e != NONE);
        else
            total += t;
    }
    counted = __reduce_add_sync(0xffffffffu, counted);
    if (!ROOTED) total = __reduce_add_sync(0xffffffffu, total);
    if (lane == 0 && counted) {
        if (!ROOTED) atomicAdd(counter, (unsigned long long)total);
        atomicAdd(counter + 1, (unsigned long long)counted);
    }
}

template <int C, bool STRICT, int T>
__global__ void __launch_bounds__(T, 1024 / T) k_leaf2_balanced(const Board *__restrict__ pboards,
                                                                const uint8_t *__restrict__ pstates,
                                                                const u32 *__restrict__ pidx,
                                                                const uint16_t *__restrict__ moves, u64 n,
                                                                u64 nparents, unsigned long long *__restrict__ counter)
{
    leaf2_balanced_cta<C, STRICT, T, false>(pboards, pstates, nullptr, pidx, moves, n, nparents, nullptr, counter);
}

// The balanced leaf over batched roots (leaf mode 3 of the batched paths).
template <int C, bool STRICT, int T>
__global__ void __launch_bounds__(T, 1024 / T)
    k_leaf2_rooted_balanced(const Board *__restrict__ pboards, const uint8_t *__restrict__ pstates,
                            const u32 *__restrict__ proot, const u32 *__restrict__ pidx,
                            const uint16_t *__restrict__ moves, u64 n, u64 nparents,
                            unsigned long long *__restrict__ root_counts, unsigned long long *__restrict__ counter)
{
    leaf2_balanced_cta<C, STRICT, T, true>(pboards, pstates, proot, pidx, moves, n, nparents, root_counts, counter);
}

// Children of a CTA (one per thread) handed to threads in order of their
// move counts, as in k_leaf2_sorted, carrying their root index along.  On
// return thread t holds the child of rank t; `valid` says whether it has one.
template <int C, int T>
__device__ __forceinline__ void rank_children(Board &b, u32 &st, u32 &root, bool &valid)
{
    __shared__ Board s_b[T];
    __shared__ u32 s_root[T];
    __shared__ uint8_t s_st[T];
    __shared__ uint8_t s_key[T];
    const u32 key = valid ? 1 + min(count_moves<1 - C, true>(b, st), 254u) : 0u;
    const u32 rank = cta_rank_u8<T>(key);
    s_b[rank] = b;
    s_root[rank] = root;
    s_st[rank] = (uint8_t)st;
    s_key[rank] = (uint8_t)key;
    __syncthreads();
    const int tid = threadIdx.x;
    b = s_b[tid];
    root = s_root[tid];
    st = s_st[tid];
    valid = s_key[tid] != 0;
    __syncthreads();  // the exchange arrays are free again
}

// Two-ply leaf over edges, counts credited to each edge's root.  MODE is the
// leaf mode of grandchild_counts: with 1 or 2 the CTA's children are ranked
// by move count first (blockDim.x must be PB_LEAF_THREADS).
template <int C, bool STRICT, int MODE>
__device__ __forceinline__ void leaf2_rooted_cta(const Board *__restrict__ pboards,
                                                 const uint8_t *__restrict__ pstates, const u32 *__restrict__ proot,
                                                 const u32 *__restrict__ pidx, const uint16_t *__restrict__ moves,
                                                 u64 n, u64 nparents, unsigned long long *__restrict__ root_counts,
                                                 unsigned long long *__restrict__ counter)
{
    u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    u32 total = 0, counted = 0, root = 0;
    bool valid = i < n && pidx[i] < nparents;
    Board b{};
    u32 st = 0;
    if (valid) {
        u32 p = pidx[i];
        root = proot[p];
        b = load_board(pboards + p);
        st = pstates[p];
        make_move<C>(b, st, moves[i]);
    }
    if (MODE >= 1) rank_children<C, PB_LEAF_THREADS>(b, st, root, valid);
    if (valid) {
        uint16_t mv[MAX_MOVES];
        ArraySink sink{mv, 0};
        gen_moves<1 - C>(b, st, sink);
        total = grandchild_counts<C, STRICT, MODE >= 2, PB_LEAF_THREADS>(b, st, mv, sink.n);
        counted = sink.n;
    }
    add_by_key(root_counts, root, total, valid);
    counted = __reduce_add_sync(0xffffffffu, counted);
    if ((threadIdx.x & 31) == 0 && counted) atomicAdd(counter + 1, (unsigned long long)counted);
}

template <int C, bool STRICT, int MODE = 0>
__global__ void __launch_bounds__(PB_LEAF_THREADS, PB_LEAF_MIN_BLOCKS)
    k_leaf2_rooted(const Board *__restrict__ pboards, const uint8_t *__restrict__ pstates,
                   const u32 *__restrict__ proot, const u32 *__restrict__ pidx, const uint16_t *__restrict__ moves,
                   u64 n, u64 nparents, unsigned long long *__restrict__ root_counts,
                   unsigned long long *__restrict__ counter)
{
    leaf2_rooted_cta<C, STRICT, MODE>(pboards, pstates, proot, pidx, moves, n, nparents, root_counts, counter);
}

// One-ply leaf over edges (perft 1 of each edge's child), per root.
template <int C, bool STRICT>
__global__ void __launch_bounds__(256) k_leaf1_rooted(const Board *__restrict__ pboards,
                                                      const uint8_t *__restrict__ pstates,
                                                      const u32 *__restrict__ proot, const u32 *__restrict__ pidx,
                                                      const uint16_t *__restrict__ moves, u64 n, u64 nparents,
                                                      unsigned long long *__restrict__ root_counts)
{
    u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    u32 cnt = 0, root = 0;
    bool valid = i < n && pidx[i] < nparents;
    if (valid) {
        u32 p = pidx[i];
        root = proot[p];
        Board b = load_board(pboards + p);
        u32 st = pstates[p];
        make_move<C>(b, st, moves[i]);
        cnt = count_moves<1 - C, STRICT>(b, st);
    }
    add_by_key(root_counts, root, cnt, valid);
}

}  // namespace pb

namespace pb {

// ---------------------------------------------------------------- graph-captured batch
// Variants of the batched-level kernels whose sizes live in device memory, so
// a whole batched perft (every level and the leaf) can be captured once as a
// CUDA graph and replayed without host round trips.  Buffers have fixed
// capacities planned on the host (from the learned size predictions); a level
// that outgrows its capacity sets OVERFLOW in the error word, writes nothing
// past the capacity, and the host then reruns the batch with exact sizing.
enum : u32 { DEVERR_OVERFLOW = 4u };

__device__ __forceinline__ u64 dev_size(const u64 *n_dev, u64 cap, u32 *err)
{
    u64 n = *n_dev;
    if (n > cap) {
        atomicOr(err, DEVERR_OVERFLOW);
        n = cap;
    }
    return n;
}

// True in every thread of the CTA when a level already outgrew its plan: the
// batch will be rerun, so its leaf leaves at once instead of counting
// truncated levels.  Called by all threads before any other barrier.
__device__ __forceinline__ bool plan_overflowed(const u32 *err)
{
    return __syncthreads_or((*reinterpret_cast<const volatile u32 *>(err) & DEVERR_OVERFLOW) != 0) != 0;
}

// The same leaf with the level sizes in device memory, for captured graphs:
// the grid covers the planned capacity and the CTAs past the level's actual
// size leave at once (a whole CTA at a time, so the ranking's barriers are
// reached by all of its threads or by none).
template <int C, bool STRICT, int MODE = 0>
__global__ void __launch_bounds__(PB_LEAF_THREADS, PB_LEAF_MIN_BLOCKS)
    k_leaf2_rooted_dev(const Board *__restrict__ pboards, const uint8_t *__restrict__ pstates,
                       const u32 *__restrict__ proot, const u32 *__restrict__ pidx,
                       const uint16_t *__restrict__ moves, const u64 *__restrict__ n_dev, u64 cap,
                       const u64 *__restrict__ npar_dev, u64 npar_cap, unsigned long long *__restrict__ root_counts,
                       unsigned long long *__restrict__ counter, u32 *__restrict__ err)
{
    if (plan_overflowed(err)) return;
    const u64 n = dev_size(n_dev, cap, err);
    if ((u64)blockIdx.x * blockDim.x >= n) return;
    const u64 npar = min(*npar_dev, npar_cap);
    leaf2_rooted_cta<C, STRICT, MODE>(pboards, pstates, proot, pidx, moves, n, npar, root_counts, counter);
}

// The balanced rooted leaf with the level sizes in device memory (planned
// graphs): the grid covers the planned capacity; CTAs past the level's
// actual size leave at once.
template <int C, bool STRICT, int T>
__global__ void __launch_bounds__(T, 1024 / T)
    k_leaf2_rooted_balanced_dev(const Board *__restrict__ pboards, const uint8_t *__restrict__ pstates,
                                const u32 *__restrict__ proot, const u32 *__restrict__ pidx,
                                const uint16_t *__restrict__ moves, const u64 *__restrict__ n_dev, u64 cap,
                                const u64 *__restrict__ npar_dev, u64 npar_cap,
                                unsigned long long *__restrict__ root_counts, unsigned long long *__restrict__ counter,
                                u32 *__restrict__ err)
{
    if (plan_overflowed(err)) return;
    const u64 n = dev_size(n_dev, cap, err);
    if ((u64)blockIdx.x * (PB_BALANCED_K * T) >= n) return;
    const u64 npar = min(*npar_dev, npar_cap);
    leaf2_balanced_cta<C, STRICT, T, true>(pboards, pstates, proot, pidx, moves, n, npar, root_counts, counter);
}

// Scan with a device-resident length (grid = tiles of the capacity; surplus
// CTAs take a ticket and leave).
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_dev(const u32 *__restrict__ in, const u64 *__restrict__ n_dev,
                                                           u64 cap, u64 *__restrict__ out, u64 *__restrict__ status,
                                                           u32 *__restrict__ ticket, u64 *__restrict__ total,
                                                           u32 *__restrict__ err)
{
    __shared__ u32 s_tile;
    const u64 n = dev_size(n_dev, cap, err);
    const u64 tiles = (n + SCAN_TILE - 1) / SCAN_TILE;
    if (threadIdx.x == 0) s_tile = atomicAdd(ticket, 1u);
    __syncthreads();
    if ((u64)s_tile >= tiles) {
        if (n == 0 && s_tile == 0 && threadIdx.x == 0) *total = 0;
        return;
    }
    scan_tile(in, n, out, status, s_tile, total, err);
}

// Generation with device-resident sizes: positions [0, npos) (npos from the
// previous level), offsets and total from the scan; writes stay below `cap`.
template <int C>
__global__ void __launch_bounds__(GEN_THREADS) k_generate_dev(const Board *__restrict__ boards,
                                                              const uint8_t *__restrict__ states,
                                                              const u64 *__restrict__ offs,
                                                              const u64 *__restrict__ total_dev,
                                                              const u64 *__restrict__ npos_dev, u64 npos_cap, u64 cap,
                                                              uint16_t *__restrict__ out_mv, u32 *__restrict__ out_pi,
                                                              u32 *__restrict__ err)
{
    __shared__ uint16_t s_mv[GEN_CAP];
    __shared__ uint8_t s_own[GEN_CAP];
    const u64 n = dev_size(npos_dev, npos_cap, err);
    const u64 total = *total_dev;
    const u64 first = (u64)blockIdx.x * GEN_THREADS;
    if (first >= n) return;
    const u64 last = min(first + GEN_THREADS, n);
    const u64 tile_begin = offs[first];
    const u64 tile_end = (last < n) ? offs[last] : total;
    const u64 i = first + threadIdx.x;
    const bool staged = (tile_end - tile_begin) <= (u64)GEN_CAP;
    if (i < n) {
        Board b = load_board(boards + i);
        u32 st = states[i];
        const u64 mine_begin = offs[i];
        u64 mine_end = (i + 1 < n) ? offs[i + 1] : total;
        bool over = false;
        if (mine_end > cap) {
            atomicOr(err, DEVERR_OVERFLOW);
            mine_end = cap;
        }
        if (mine_end <= mine_begin) {
        } else if (staged) {
            SmemSink s{s_mv, s_own, (uint8_t)threadIdx.x, (int)(mine_begin - tile_begin),
                       (int)(mine_end - tile_begin), false};
            gen_moves<C>(b, st, s);
            over = s.over || s.n < s.cap;
        } else {
            GlobalSink s{out_mv, out_pi, (u32)i, mine_begin, mine_end, false};
            gen_moves<C>(b, st, s);
            over = s.over || s.n < s.cap;
        }
        if (over && total <= cap) atomicOr(err, DEVERR_CAPACITY);
    }
    if (!staged) return;
    __syncthreads();
    const u64 end = min(tile_end, cap);
    const int cnt = end > tile_begin ? (int)(end - tile_begin) : 0;
    for (int k = threadIdx.x; k < cnt; k += GEN_THREADS) {
        out_mv[tile_begin + k] = s_mv[k];
        out_pi[tile_begin + k] = (u32)first + s_own[k];
    }
}

template <int C>
__global__ void __launch_bounds__(256) k_expand_rooted_dev(const Board *__restrict__ pboards,
                                                           const uint8_t *__restrict__ pstates,
                                                           const u32 *__restrict__ proot,
                                                           const u32 *__restrict__ pidx,
                                                           const uint16_t *__restrict__ moves,
                                                           const u64 *__restrict__ n_dev, u64 cap,
                                                           const u64 *__restrict__ npar_dev, u64 npar_cap,
                                                           Board *__restrict__ cboards, uint8_t *__restrict__ cstates,
                                                           u32 *__restrict__ croot, u32 *__restrict__ counts,
                                                           u32 *__restrict__ err)
{
    const u64 n = dev_size(n_dev, cap, err);
    const u64 npar = min(*npar_dev, npar_cap);
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) {
        u32 p = pidx[i];
        if (p >= npar) {
            counts[i] = 0;
            croot[i] = 0;
            atomicOr(err, DEVERR_CAPACITY);
            continue;
        }
        Board b = load_board(pboards + p);
        u32 st = pstates[p];
        make_move<C>(b, st, moves[i]);
        store_board(cboards + i, b);
        cstates[i] = (uint8_t)st;
        croot[i] = proot[p];
        counts[i] = count_moves<1 - C, true>(b, st);
    }
}

// Persistent two-ply leaf driven by a device work queue: each CTA takes
// blockDim.x consecutive edges from an atomic cursor until the level is
// exhausted, so uneven subtrees balance across the SMs without a per-edge
// grid.  The grab is per CTA, not per warp: the CTA's warps then work on
// sibling edges whose attack-table lines they share in L1 (per-warp grabs of
// 32, 64 or 128 edges measured 2.6-6 % slower on B200).
template <int C, bool STRICT, int MODE = 0>
__global__ void __launch_bounds__(PB_LEAF_THREADS, PB_LEAF_MIN_BLOCKS)
    k_leaf2_rooted_queue(const Board *__restrict__ pboards, const uint8_t *__restrict__ pstates,
                         const u32 *__restrict__ proot, const u32 *__restrict__ pidx,
                         const uint16_t *__restrict__ moves, const u64 *__restrict__ n_dev, u64 cap,
                         const u64 *__restrict__ npar_dev, u64 npar_cap, unsigned long long *__restrict__ cursor,
                         unsigned long long *__restrict__ root_counts, unsigned long long *__restrict__ counter,
                         u32 *__restrict__ err)
{
    if (plan_overflowed(err)) return;
    const u64 n = dev_size(n_dev, cap, err);
    const u64 npar = min(*npar_dev, npar_cap);
    const int lane = threadIdx.x & 31;
    u32 counted = 0;
    __shared__ unsigned long long s_base;
    for (;;) {
        if (threadIdx.x == 0) s_base = atomicAdd(cursor, (unsigned long long)blockDim.x);
        __syncthreads();
        const unsigned long long base = s_base;
        __syncthreads();
        if (base >= n) break;
        const u64 i = base + threadIdx.x;
        u32 total = 0, root = 0;
        bool valid = i < n && pidx[i] < npar;
        Board b{};
        u32 st = 0;
        if (valid) {
            u32 p = pidx[i];
            root = proot[p];
            b = load_board(pboards + p);
            st = pstates[p];
            make_move<C>(b, st, moves[i]);
        }
        if (MODE >= 1) rank_children<C, PB_LEAF_THREADS>(b, st, root, valid);
        if (valid) {
            uint16_t mv[MAX_MOVES];
            ArraySink sink{mv, 0};
            gen_moves<1 - C>(b, st, sink);
            total = grandchild_counts<C, STRICT, MODE >= 2, PB_LEAF_THREADS>(b, st, mv, sink.n);
            counted += sink.n;
        }
        add_by_key(root_counts, root, total, valid);
    }
    counted = __reduce_add_sync(0xffffffffu, counted);
    if (lane == 0 && counted) atomicAdd(counter + 1, (unsigned long long)counted);
}

template <int C, bool STRICT>
__global__ void __launch_bounds__(256) k_leaf1_rooted_dev(const Board *__restrict__ pboards,
                                                          const uint8_t *__restrict__ pstates,
                                                          const u32 *__restrict__ proot, const u32 *__restrict__ pidx,
                                                          const uint16_t *__restrict__ moves,
                                                          const u64 *__restrict__ n_dev, u64 cap,
                                                          const u64 *__restrict__ npar_dev, u64 npar_cap,
                                                          unsigned long long *__restrict__ root_counts,
                                                          u32 *__restrict__ err)
{
    const u64 n = dev_size(n_dev, cap, err);
    const u64 npar = min(*npar_dev, npar_cap);
    for (u64 base = (u64)blockIdx.x * blockDim.x; base < n; base += (u64)gridDim.x * blockDim.x) {
        u64 i = base + threadIdx.x;
        u32 cnt = 0, root = 0;
        bool valid = i < n && pidx[i] < npar;
        if (valid) {
            u32 p = pidx[i];
            root = proot[p];
            Board b = load_board(pboards + p);
            u32 st = pstates[p];
            make_move<C>(b, st, moves[i]);
            cnt = count_moves<1 - C, STRICT>(b, st);
        }
        add_by_key(root_counts, root, cnt, valid);
    }
}

}  // namespace pb

namespace pb {

// ---------------------------------------------------------------- leaf with deferred evasions
// The fused two-ply leaf, but a grandchild in check is not counted on the
// spot: its board, state, pinned set and attack map go to a per-warp queue in
// shared memory, and once 32 are queued the whole warp counts them together.
// In-check positions are rare (about 1-2 % of the counted positions) but
// frequent per warp (one lane in 32 often enough), and counting an evasion
// costs about as much as counting a quiet position, so a warp that met one
// used to pay for both paths on every such step.
constexpr int DEFER_CAP = 64;  // <= 31 waiting + 32 new

template <int C, bool STRICT, int T>
__global__ void __launch_bounds__(T, 1024 / T) k_leaf2_defer(const Board *__restrict__ pboards,
                                                             const uint8_t *__restrict__ pstates,
                                                             const u32 *__restrict__ pidx,
                                                             const uint16_t *__restrict__ moves, u64 n, u64 nparents,
                                                             unsigned long long *__restrict__ counter)
{
    __shared__ Board q_b[T / 32][DEFER_CAP];
    __shared__ u64 q_pin[T / 32][DEFER_CAP];
    __shared__ u64 q_thr[T / 32][DEFER_CAP];
    __shared__ uint8_t q_st[T / 32][DEFER_CAP];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const u64 i = (u64)blockIdx.x * T + threadIdx.x;
    u32 total = 0;
    int nm = 0;
    Board b;
    u32 st = 0;
    uint16_t mv[MAX_MOVES];
    if (i < n && pidx[i] < nparents) {
        u32 p = pidx[i];
        b = load_board(pboards + p);
        st = pstates[p];
        make_move<C>(b, st, moves[i]);
        ArraySink sink{mv, 0};
        gen_moves<1 - C>(b, st, sink);
        nm = sink.n;
    }
    const u32 counted = (u32)nm;
    const int kmax = (int)__reduce_max_sync(0xffffffffu, (u32)nm);
    int qn = 0;
    for (int k = 0; k < kmax; k++) {
        bool check = false;
        Board g;
        u32 gs = 0;
        CountPrep pr;
        if (k < nm) {
            g = b;
            gs = st;
            make_move<1 - C>(g, gs, mv[k]);
            pr = count_prep<C>(g);
            check = prep_in_check<C>(pr);
            if (!check) total += count_quiet<C, STRICT>(pr.s, gs, pr.pinned, pr.threat, pr.ksq);
        }
        const unsigned dm = __ballot_sync(0xffffffffu, check);
        if (dm) {
            if (check) {
                const int slot = qn + __popc(dm & ((1u << lane) - 1u));
                q_b[warp][slot] = g;
                q_pin[warp][slot] = pr.pinned;
                q_thr[warp][slot] = pr.threat;
                q_st[warp][slot] = (uint8_t)gs;
            }
            qn += __popc(dm);
            __syncwarp();
            if (qn >= 32) {
                const int slot = qn - 32 + lane;
                const Board e = q_b[warp][slot];
                const Sets es = derive<C>(e);
                total += count_evasions<C, STRICT>(es, q_st[warp][slot], q_pin[warp][slot], q_thr[warp][slot],
                                                   bit_index(es.kings & es.us));
                qn -= 32;
                __syncwarp();
            }
        }
    }
    if (lane < qn) {
        const Board e = q_b[warp][lane];
        const Sets es = derive<C>(e);
        total += count_evasions<C, STRICT>(es, q_st[warp][lane], q_pin[warp][lane], q_thr[warp][lane],
                                           bit_index(es.kings & es.us));
    }
    const u32 t = __reduce_add_sync(0xffffffffu, total);
    const u32 c = __reduce_add_sync(0xffffffffu, counted);
    if (lane == 0 && c) {
        atomicAdd(counter, (unsigned long long)t);
        atomicAdd(counter + 1, (unsigned long long)c);
    }
}

}  // namespace pb
