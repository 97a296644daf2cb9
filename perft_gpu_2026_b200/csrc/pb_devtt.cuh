// pb_devtt.cuh - device transposition tables and the TT-mode BFS kernels.
//
// One table per remaining depth r, like the reference's deviceTTs[r]
// (tt.h:16-156, launcher.cu:128-351), but every hit is verified against the
// full 128-bit key:
//   r = 2, 3  ("shallow", 16 B): w1 = (lo << 24) | (count + 1), w0 = hi ^ w1.
//             The slot is floor(lo * slots / 2^64), so a slot holds keys whose
//             lo lies in an interval shorter than 2^40 when the table has at
//             least 2^24 slots: lo's low 40 bits in w1 then pin lo exactly,
//             and w0 ^ w1 gives the whole hi.
//   r >= 4    ("deep", 32 B): {lo ^ c, hi ^ c, c, lo ^ hi ^ c}, one 256-bit
//             store; a torn read cannot verify unless both halves carry the
//             same key.
// Replacement is always-overwrite (tt.h:60-70).
//
// TT-mode BFS (perft_kernels.cu:700-982): the expand kernel also derives each
// child's key incrementally, probes TT[r] and marks hits (not expanded);
// duplicates inside a level are expanded once (owner = smallest index among
// equal 128-bit keys, elected with a 64-bit atomicMax); the leaf probes and
// stores TT[2]; an upsweep then sums every position's children over its
// contiguous child range, stores TT[r] and copies owners' counts to their
// duplicates.
#pragma once
#include "pb_core.cuh"
#include "pb_kernels.cuh"
#include "pb_tt.cuh"

namespace pb {

enum { TT_NONE = 0, TT_SHALLOW = 1, TT_DEEP = 2 };
constexpr int TT_MAX_DEPTH = 32;
constexpr u64 SHALLOW_COUNT_MASK = 0xFFFFFFULL;

struct TTView {
    u64 *entries;  // SHALLOW: 2 words per slot, DEEP: 4 words per slot
    u64 slots;     // any size: the slot is the high word of lo * slots
    int kind;
    int buckets;   // 0: one slot, always overwrite; 1: two-slot buckets, size priority
};

__device__ __forceinline__ u64 tt_slot(const TTView &t, u64 lo) { return __umul64hi(lo, t.slots); }

// Entry in slot `slot` matching the key?  (*count = its count; *used = slot holds anything)
__device__ __forceinline__ bool tt_read(const TTView &t, u64 slot, const Hash128 &h, u64 *count, u64 *held)
{
    if (t.kind == TT_SHALLOW) {
        u64 w0, w1;
        asm volatile("ld.global.v2.u64 {%0,%1}, [%2];" : "=l"(w0), "=l"(w1) : "l"(t.entries + 2 * slot));
        *held = (w1 & SHALLOW_COUNT_MASK) ? (w1 & SHALLOW_COUNT_MASK) - 1 : 0;
        if ((w0 ^ w1) == h.hi && ((w1 ^ (h.lo << 24)) & ~SHALLOW_COUNT_MASK) == 0 && (w1 & SHALLOW_COUNT_MASK)) {
            *count = (w1 & SHALLOW_COUNT_MASK) - 1;
            return true;
        }
        return false;
    }
    u64 w0, w1, w2, w3;
    asm volatile("ld.global.v4.u64 {%0,%1,%2,%3}, [%4];"
                 : "=l"(w0), "=l"(w1), "=l"(w2), "=l"(w3)
                 : "l"(t.entries + 4 * slot));
    *held = (w0 | w1 | w2 | w3) ? w2 : 0;
    if ((w0 ^ w2) == h.lo && (w1 ^ w2) == h.hi && (w3 ^ w2) == (h.lo ^ h.hi) && (w0 | w1 | w2 | w3)) {
        *count = w2;
        return true;
    }
    return false;
}

__device__ __forceinline__ void tt_write(const TTView &t, u64 slot, const Hash128 &h, u64 count)
{
    if (t.kind == TT_SHALLOW) {
        if (count + 1 > SHALLOW_COUNT_MASK) return;  // never truncate a count
        u64 w1 = (h.lo << 24) | (count + 1);
        u64 w0 = h.hi ^ w1;
        asm volatile("st.global.v2.u64 [%0], {%1,%2};" ::"l"(t.entries + 2 * slot), "l"(w0), "l"(w1) : "memory");
        return;
    }
    asm volatile("st.global.v4.u64 [%0], {%1,%2,%3,%4};" ::"l"(t.entries + 4 * slot), "l"(h.lo ^ count),
                 "l"(h.hi ^ count), "l"(count), "l"(h.lo ^ h.hi ^ count)
                 : "memory");
}

__device__ __forceinline__ bool tt_probe(const TTView &t, const Hash128 &h, u64 *out)
{
    if (t.kind == TT_NONE) return false;
    u64 slot = tt_slot(t, h.lo), held;
    if (!t.buckets) return tt_read(t, slot, h, out, &held);
    slot &= ~1ULL;
    return tt_read(t, slot, h, out, &held) || tt_read(t, slot + 1, h, out, &held);
}

// Always-overwrite (the reference's rule, tt.h:60-70), or with two-slot
// buckets: a key already present is refreshed in place, otherwise the first
// slot keeps the larger subtree and the second takes whatever is displaced
// or stored.
__device__ __forceinline__ void tt_store(const TTView &t, const Hash128 &h, u64 count)
{
    if (t.kind == TT_NONE) return;
    u64 slot = tt_slot(t, h.lo);
    if (!t.buckets) {
        tt_write(t, slot, h, count);
        return;
    }
    slot &= ~1ULL;
    u64 c0, c1, held0, held1;
    if (tt_read(t, slot, h, &c0, &held0)) return;
    if (tt_read(t, slot + 1, h, &c1, &held1)) return;
    if (count >= held0)
        tt_write(t, slot, h, count);
    else
        tt_write(t, slot + 1, h, count);
}

// Race self-test: every thread stores and probes keys of a small key set in
// a table far smaller than the set, so stores and probes of different keys
// hit the same slots at the same time.  Each key's count is a function of the
// key; a probe that reports a hit with any other count (a torn or foreign
// entry accepted) increments *bad.  No waits; every slot index is in range.
__device__ __forceinline__ u64 race_mix(u64 z)
{
    // splitmix64 output function (Steele, Lea and Flood 2014)
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
__device__ __forceinline__ Hash128 race_key(u32 k)
{
    Hash128 h;
    h.lo = race_mix(0x9E3779B97F4A7C15ULL * (2ULL * k + 1));
    h.hi = race_mix(0xD1B54A32D192ED03ULL * (2ULL * k + 2));
    return h;
}
__device__ __forceinline__ u64 race_count(const Hash128 &h) { return (h.lo ^ (h.hi >> 7)) & 0xFFFFFULL; }
// With `packed`, bits 40..42 of the key's lo are the key's number mod 8 and
// the bits above are zero, so in a table of 2^24 slots (slot = lo >> 40) all
// keys fall into 8 slots: the shallow format at the size the engine allows,
// under the same contention as the small table.
__device__ __forceinline__ Hash128 race_key_in(u32 k, bool packed)
{
    Hash128 h = race_key(k);
    if (packed) h.lo = (h.lo & ((1ULL << 40) - 1)) | ((u64)(k & 7u) << 40);
    return h;
}
__global__ void k_tt_race(TTView t, u32 nkeys, u32 iters, u32 packed, unsigned long long *bad,
                          unsigned long long *hits)
{
    const u32 tid = blockIdx.x * blockDim.x + threadIdx.x;
    u64 wrong = 0, seen = 0;
    for (u32 it = 0; it < iters; it++) {
        const Hash128 a = race_key_in((tid * 2654435761u + it * 40503u) % nkeys, packed != 0);
        tt_store(t, a, race_count(a));
        const Hash128 b = race_key_in((tid * 97u + it * 7919u + 1u) % nkeys, packed != 0);
        u64 c;
        if (tt_probe(t, b, &c)) {
            seen++;
            if (c != race_count(b)) wrong++;
        }
    }
    if (wrong) atomicAdd(bad, (unsigned long long)wrong);
    if (seen) atomicAdd(hits, (unsigned long long)seen);
}

struct TTViews {
    TTView v[TT_MAX_DEPTH];
};

// Device tables, one per remaining depth in [2, max_depth].
struct DeviceTT {
    TTViews views{};
    std::vector<void *> blocks;
    u64 bytes = 0;

    bool ready() const { return !blocks.empty(); }

    // budget_mb 0 = auto (a share of `free_bytes`).  Depths 2 to 4 use the
    // 16-byte shallow format (twice the entries of the 32-byte one; a count
    // that does not fit its 24 bits is not stored; depth 4 shallow ran perft
    // 11 1.1 % faster than depth 4 deep); the split gives the leaf table (depth 2) 55 %, depth 3
    // 15 % and the rest to depths 4..max_depth.  The leaf table takes most
    // because the leaf does almost all the work: on start position perft 11
    // with 150 GB this split ran 2.3 % faster than quarters for depths 2 and 3
    // (4.6 % fewer leaf move-count calls); 70 % / 10 % was slower again.
    int buckets = 0;

    int init(int budget_mb, size_t free_bytes, int max_depth, int verbose, std::string *err)
    {
        release();
        u64 budget = budget_mb > 0 ? (u64)budget_mb << 20 : (u64)(free_bytes * 0.85);
        if (max_depth < 3) max_depth = 3;
        if (max_depth > TT_MAX_DEPTH - 1) max_depth = TT_MAX_DEPTH - 1;
        int deep = max_depth - 4 + 1;  // depths 4..max_depth
        for (int r = 2; r <= max_depth; r++) {
            double share = (r == 2) ? 0.55 : (r == 3) ? 0.15 : (deep > 0 ? 0.30 / deep : 0.0);
            if (deep <= 0 && r <= 3) share = 0.5;
            u64 want = (u64)(budget * share);
            bool shallow = r <= 4;  // counts of depth <= 4 fit the 24-bit shallow count
            u64 esz = shallow ? 16 : 32;
            u64 slots = want / esz;
            // the stored 40 low bits of lo pin the key only while a slot (or a
            // two-slot bucket) spans less than 2^40 values of lo
            if (shallow && slots < (buckets ? (1ULL << 25) : (1ULL << 24))) continue;
            if (!shallow && slots < 1024) continue;
            void *p = nullptr;
            if (cudaMalloc(&p, slots * esz) != cudaSuccess) {
                cudaGetLastError();
                continue;
            }
            cudaMemset(p, 0, slots * esz);
            blocks.push_back(p);
            views.v[r] = TTView{reinterpret_cast<u64 *>(p), slots, shallow ? TT_SHALLOW : TT_DEEP, buckets};
            bytes += slots * esz;
            if (verbose)
                printf("Device TT[%d]%s: %lluM entries (%llu MB)\n", r, shallow ? " (shallow)" : "",
                       (unsigned long long)(slots >> 20), (unsigned long long)((slots * esz) >> 20));
        }
        (void)err;
        return 0;
    }
    void clear()
    {
        for (int r = 0; r < TT_MAX_DEPTH; r++)
            if (views.v[r].kind != TT_NONE)
                cudaMemset(views.v[r].entries, 0, views.v[r].slots * (views.v[r].kind == TT_SHALLOW ? 16 : 32));
    }
    void release()
    {
        for (void *p : blocks) cudaFree(p);
        blocks.clear();
        views = TTViews{};
        bytes = 0;
    }
    TTView at(int r) const { return (r >= 0 && r < TT_MAX_DEPTH) ? views.v[r] : TTView{nullptr, 0, TT_NONE, 0}; }
};

// ---------------------------------------------------------------- TT-mode kernels
enum : uint8_t { PF_HIT = 1, PF_DUP = 2 };

// Expand with keys: child board/state/key, TT[r] probe, exact child count
// (0 on a hit, the hit value in vals[i]).
template <int C>
__global__ void __launch_bounds__(256) k_expand_count_tt(const Board *__restrict__ pboards,
                                                         const uint8_t *__restrict__ pstates,
                                                         const Hash128 *__restrict__ phash,
                                                         const u32 *__restrict__ pidx,
                                                         const uint16_t *__restrict__ moves, u64 n, u64 nparents,
                                                         TTView tt, Board *__restrict__ cboards,
                                                         uint8_t *__restrict__ cstates, Hash128 *__restrict__ chash,
                                                         u32 *__restrict__ counts, u64 *__restrict__ vals,
                                                         uint8_t *__restrict__ flags, u32 *__restrict__ err)
{
    u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    u32 p = pidx[i];
    if (p >= nparents) {
        atomicOr(err, DEVERR_CAPACITY);
        counts[i] = 0;
        flags[i] = PF_HIT;
        vals[i] = 0;
        return;
    }
    Board b = load_board(pboards + p);
    u32 st = pstates[p];
    Board before = b;
    uint16_t mv = moves[i];
    make_move<C>(b, st, mv);
    Hash128 h = hash_move(phash[p], before, pstates[p], st, C, mv);
    store_board(cboards + i, b);
    cstates[i] = (uint8_t)st;
    chash[i] = h;
    u64 hit;
    if (tt_probe(tt, h, &hit)) {
        counts[i] = 0;
        vals[i] = hit;
        flags[i] = PF_HIT;
    } else {
        counts[i] = count_moves<1 - C, true>(b, st);
        vals[i] = 0;
        flags[i] = 0;
    }
}

// Duplicate election inside a level: slot word = (generation << 32) | ~index;
// atomicMax keeps the current generation and the smallest index.
__global__ void k_dedup_claim(const Hash128 *__restrict__ h, const uint8_t *__restrict__ flags, u64 n,
                              unsigned long long *__restrict__ slots, u64 mask, u32 gen)
{
    u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || (flags[i] & PF_HIT)) return;
    unsigned long long w = ((unsigned long long)gen << 32) | (unsigned long long)(~(u32)i);
    atomicMax(slots + (h[i].lo & mask), w);
}

__global__ void k_dedup_resolve(const Hash128 *__restrict__ h, uint8_t *__restrict__ flags, u64 n,
                                const unsigned long long *__restrict__ slots, u64 mask, u32 gen,
                                u32 *__restrict__ counts, u32 *__restrict__ redirect)
{
    u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || (flags[i] & PF_HIT)) return;
    unsigned long long w = slots[h[i].lo & mask];
    if ((u32)(w >> 32) != gen) return;
    u32 owner = ~(u32)w;
    if (owner == (u32)i || owner >= n) return;
    Hash128 a = h[i], o = h[owner];
    if (a.lo == o.lo && a.hi == o.hi) {
        flags[i] |= PF_DUP;
        counts[i] = 0;
        redirect[i] = owner;
    }
}

// Leaf with the depth-2 table: perft 2 of each edge's child, per edge.  MODE
// is the leaf mode of grandchild_counts.  With MODE >= 1 (blockDim.x must be
// PB_LEAF_THREADS) table hits are answered first and
// the CTA's misses are ranked by move count and handed to threads in that
// order, so the misses fill whole warps (all-hit warps then have no work) and
// each warp's misses have similar loop lengths.
template <int C, bool STRICT, int MODE = 0>
__global__ void __launch_bounds__(PB_LEAF_THREADS, PB_LEAF_MIN_BLOCKS)
    k_leaf2_tt(const Board *__restrict__ pboards, const uint8_t *__restrict__ pstates,
               const Hash128 *__restrict__ phash, const u32 *__restrict__ pidx, const uint16_t *__restrict__ moves,
               u64 n, u64 nparents, TTView tt, u32 *__restrict__ out, unsigned long long *__restrict__ counter)
{
    u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    u32 total = 0, counted = 0;
    bool miss = false;
    Board b{};
    u32 st = 0;
    Hash128 h{};
    if (i < n && pidx[i] < nparents) {
        u32 p = pidx[i];
        b = load_board(pboards + p);
        st = pstates[p];
        Board before = b;
        uint16_t mv0 = moves[i];
        make_move<C>(b, st, mv0);
        h = hash_move(phash[p], before, pstates[p], st, C, mv0);
        u64 hit;
        if (tt_probe(tt, h, &hit))
            out[i] = (u32)hit;
        else
            miss = true;
    }
    if (MODE >= 1) {
        __shared__ Board s_b[PB_LEAF_THREADS];
        __shared__ Hash128 s_h[PB_LEAF_THREADS];
        __shared__ u32 s_i[PB_LEAF_THREADS];
        __shared__ uint8_t s_st[PB_LEAF_THREADS];
        __shared__ uint8_t s_key[PB_LEAF_THREADS];
        const u32 key = miss ? 1 + min(count_moves<1 - C, true>(b, st), 254u) : 0u;
        const u32 rank = cta_rank_u8<PB_LEAF_THREADS>(key);
        s_b[rank] = b;
        s_h[rank] = h;
        s_i[rank] = (u32)(i - (u64)blockIdx.x * blockDim.x);
        s_st[rank] = (uint8_t)st;
        s_key[rank] = (uint8_t)key;
        __syncthreads();
        b = s_b[threadIdx.x];
        h = s_h[threadIdx.x];
        i = (u64)blockIdx.x * blockDim.x + s_i[threadIdx.x];
        st = s_st[threadIdx.x];
        miss = s_key[threadIdx.x] != 0;
    }
    if (miss) {
        uint16_t mv[MAX_MOVES];
        ArraySink sink{mv, 0};
        gen_moves<1 - C>(b, st, sink);
        total = grandchild_counts<C, STRICT, MODE >= 2, PB_LEAF_THREADS>(b, st, mv, sink.n);
        counted = sink.n;
        tt_store(tt, h, total);
        out[i] = total;
    }
    counted = __reduce_add_sync(0xffffffffu, counted);
    if ((threadIdx.x & 31) == 0 && counted) atomicAdd(counter + 1, (unsigned long long)counted);
}

// Persistent table leaf that keeps every warp counting (pb_tuning.tt_leaf =
// 2).  In k_leaf2_tt a thread whose edge hits the table idles through its
// CTA's grandchild loop, and a CTA holds its registers until its last warp
// is done, so at the leaf's ~45 % hit rate nearly half the warps of the SM
// have nothing to do.  Here each CTA takes T edges at a time from an atomic
// cursor, makes their children, probes the depth-2 table (hits are written
// at once) and appends each miss (edge index, key) to a shared-memory queue;
// whenever the queue holds 2T misses, or the edges are exhausted, the CTA
// takes 2T of them (two per thread), remakes their children from the parent
// and the move, ranks them by move count and cuts the ranking into 32-miss
// chunks; warp w counts chunks w and 2W - 1 - w (a light and a heavy one),
// so the warps of a pass reach its closing barrier at about the same time
// while the lanes of a chunk still have similar loop lengths.  The queue
// holds at most 3T entries: the passes drain it below 2T, and one probe round
// adds at most T.  MODE is the leaf mode (1 or 2).  Measured on
// B200 against k_leaf2_tt (same counts): start position perft 10 with 150 GB
// of tables 1.923 -> 1.787 s, the 2-ply seed-4 position perft 10 3.487 ->
// 3.240 s (27.4 -> 30.1 G move-count calls/s), start position perft 9 with
// 16 GB 171.8 -> 163.6 ms of leaf time.
template <int C, bool STRICT, int MODE>
__global__ void __launch_bounds__(PB_LEAF_THREADS, PB_LEAF_MIN_BLOCKS)
    k_leaf2_tt_fill(const Board *__restrict__ pboards, const uint8_t *__restrict__ pstates,
                    const Hash128 *__restrict__ phash, const u32 *__restrict__ pidx,
                    const uint16_t *__restrict__ moves, u64 n, u64 nparents, TTView tt, u32 *__restrict__ out,
                    unsigned long long *__restrict__ cursor, unsigned long long *__restrict__ counter)
{
    constexpr int T = PB_LEAF_THREADS;
    constexpr int PASS = 2 * T;      // misses per count pass, two per thread
    constexpr int Q = PASS + T;      // drained below PASS; one probe round adds at most T
    constexpr int W = T / 32;
    constexpr int NCH = PASS / 32;   // 32-miss chunks of a pass, paired (j, NCH - 1 - j) per warp
    static_assert(NCH == 2 * W, "one chunk pair per warp");
    constexpr u32 NONE = 0xFFFFFFFFu;
    __shared__ u32 q_i[Q];
    __shared__ Hash128 q_h[Q];
    __shared__ u32 s_slot[PASS];
    __shared__ u32 q_n;
    __shared__ unsigned long long s_base;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    u32 counted = 0;
    if (tid == 0) q_n = 0;
    for (;;) {
        if (tid == 0) s_base = atomicAdd(cursor, (unsigned long long)T);
        __syncthreads();
        const u64 base = s_base;
        const bool done = base >= n;
        if (!done) {
            const u64 i = base + tid;
            if (i < n && pidx[i] < nparents) {
                const u32 p = pidx[i];
                Board b = load_board(pboards + p);
                u32 st = pstates[p];
                const Board before = b;
                const uint16_t mv0 = moves[i];
                make_move<C>(b, st, mv0);
                const Hash128 h = hash_move(phash[p], before, pstates[p], st, C, mv0);
                u64 hit;
                if (tt_probe(tt, h, &hit)) {
                    out[i] = (u32)hit;
                } else {
                    const u32 slot = atomicAdd(&q_n, 1u);
                    q_i[slot] = (u32)i;
                    q_h[slot] = h;
                }
            }
        }
        __syncthreads();
        // count passes over PASS misses (the rest once the edges are done)
        for (;;) {
            const u32 qn = q_n;
            if (!(qn >= (u32)PASS || (done && qn > 0))) break;
            const u32 take = min(qn, (u32)PASS), first = qn - take;
            u32 key[2], rank[2];
#pragma unroll
            for (int k = 0; k < 2; k++) {
                const u32 e = (u32)(k * T + tid);
                key[k] = 0;
                if (e < take) {
                    const u32 i = q_i[first + e], p = pidx[i];
                    Board b = load_board(pboards + p);
                    u32 st = pstates[p];
                    make_move<C>(b, st, moves[i]);
                    key[k] = 1 + min(count_moves<1 - C, true>(b, st), 254u);
                }
            }
            cta_rank_u8<T, 2>(key, rank);
#pragma unroll
            for (int k = 0; k < 2; k++) s_slot[rank[k]] = key[k] ? first + (u32)(k * T + tid) : NONE;
            __syncthreads();
#pragma unroll 1
            for (int q = 0; q < 2; q++) {
                const int chunk = q ? NCH - 1 - warp : warp;
                const u32 slot = s_slot[chunk * 32 + lane];
                if (slot != NONE) {
                    const u32 i = q_i[slot], p = pidx[i];
                    const Hash128 h = q_h[slot];
                    Board b = load_board(pboards + p);
                    u32 st = pstates[p];
                    make_move<C>(b, st, moves[i]);
                    uint16_t mv[MAX_MOVES];
                    ArraySink sink{mv, 0};
                    gen_moves<1 - C>(b, st, sink);
                    const u32 total = grandchild_counts<C, STRICT, MODE >= 2, T>(b, st, mv, sink.n);
                    counted += sink.n;
                    tt_store(tt, h, total);
                    out[i] = total;
                }
            }
            __syncthreads();  // every queued entry of the pass read
            if (tid == 0) q_n = first;
            __syncthreads();
        }
        if (done) break;
    }
    counted = __reduce_add_sync(0xffffffffu, counted);
    if ((tid & 31) == 0 && counted) atomicAdd(counter + 1, (unsigned long long)counted);
}

// Upsweep of one level: vals[i] = sum of the children's counts over
// [offs[i], offs[i] + counts[i]) unless i was a TT hit or a duplicate; the
// result is stored in TT[r].
template <class ChildT>
__global__ void k_upsweep(const ChildT *__restrict__ child, const u64 *__restrict__ offs,
                          const u32 *__restrict__ counts, const uint8_t *__restrict__ flags,
                          const Hash128 *__restrict__ h, u64 n, TTView tt, u64 *__restrict__ vals)
{
    u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || flags[i]) return;
    u64 a = offs[i], z = a + counts[i], s = 0;
    for (u64 k = a; k < z; k++) s += (u64)child[k];
    vals[i] = s;
    tt_store(tt, h[i], s);
}

__global__ void k_resolve_dups(const uint8_t *__restrict__ flags, const u32 *__restrict__ redirect, u64 n,
                               u64 *__restrict__ vals)
{
    u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !(flags[i] & PF_DUP)) return;
    vals[i] = vals[redirect[i]];
}

template <class T>
__global__ void k_sum(const T *__restrict__ v, u64 n, unsigned long long *__restrict__ out)
{
    u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long x = (i < n) ? (unsigned long long)v[i] : 0ULL;
#pragma unroll
    for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) == 0 && x) atomicAdd(out, x);
}

}  // namespace pb
