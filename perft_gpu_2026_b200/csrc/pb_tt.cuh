// pb_tt.cuh - 128-bit Zobrist keys and the transposition tables.
//
// Keys: two independent 64-bit Zobrist sets (lo, hi) over [colour][piece]
// [square], the four castle bits, the eight en-passant files and the side to
// move - the layout of the reference's ZobristRandoms (zobrist.h:20-26).  The
// random words are this project's own, drawn from splitmix64 with fixed
// seeds; only equality of keys matters for counts, never their values.
//
// Host TT (the reference's LosslessTT, tt.h:165-229): one open-addressing
// table per remaining depth, full 128-bit key check, never overwritten; a full
// table stops accepting stores instead of evicting, so a stored count is
// always exact.
//
// Device TT: see pb_devtt.cuh.
#pragma once
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include <string>
#include <vector>

#include "pb_core.cuh"
#include "pb_util.cuh"

namespace pb {

struct Hash128 {
    u64 lo, hi;
};

struct Zobrist {
    u64 piece[2][2][6][64];  // [half: 0 lo, 1 hi][colour][piece-1][square]
    u64 castle[2][4];
    u64 ep[2][8];
    u64 side[2];
};

Zobrist h_zob;
__device__ Zobrist g_zob;

inline void build_zobrist()
{
    static bool done = false;
    if (done) return;
    for (int half = 0; half < 2; half++) {
        u64 s = half ? 0xC0FFEE1234567ULL : 0xB200B200B200ULL;
        for (int c = 0; c < 2; c++)
            for (int p = 0; p < 6; p++)
                for (int q = 0; q < 64; q++) h_zob.piece[half][c][p][q] = splitmix64(&s);
        for (int k = 0; k < 4; k++) h_zob.castle[half][k] = splitmix64(&s);
        for (int k = 0; k < 8; k++) h_zob.ep[half][k] = splitmix64(&s);
        h_zob.side[half] = splitmix64(&s);
    }
    done = true;
}

#ifdef __CUDA_ARCH__
#define PB_ZOB g_zob
#else
#define PB_ZOB h_zob
#endif

PB_HD void zpiece(Hash128 &h, int c, int piece, int sq)
{
    h.lo ^= PB_ZOB.piece[0][c][piece - 1][sq];
    h.hi ^= PB_ZOB.piece[1][c][piece - 1][sq];
}
PB_HD void zstate(Hash128 &h, u32 st)
{
    for (int k = 0; k < 4; k++)
        if (st & (1u << k)) {
            h.lo ^= PB_ZOB.castle[0][k];
            h.hi ^= PB_ZOB.castle[1][k];
        }
    u32 ep = st >> 4;
    if (ep) {
        h.lo ^= PB_ZOB.ep[0][ep - 1];
        h.hi ^= PB_ZOB.ep[1][ep - 1];
    }
}

// Key of a whole position (computeHash, zobrist.h:81-134).
PB_HD Hash128 hash_position(const Board &b, u32 st, int color)
{
    Hash128 h{0, 0};
    if (color == WHITE) {
        h.lo ^= PB_ZOB.side[0];
        h.hi ^= PB_ZOB.side[1];
    }
    zstate(h, st);
    u64 occ = b.bb[1] | b.bb[2] | b.bb[3];
    while (occ) {
        int sq = lsb(occ);
        int piece = (int)(((b.bb[1] >> sq) & 1) | (((b.bb[2] >> sq) & 1) << 1) | (((b.bb[3] >> sq) & 1) << 2));
        zpiece(h, (int)((b.bb[0] >> sq) & 1), piece, sq);
        occ &= occ - 1;
    }
    return h;
}

// Key after `mv` by side c from (before, st_before) to a position whose state
// is st_after (updateHashAfterMove, zobrist.h:149-227).
PB_HD Hash128 hash_move(Hash128 h, const Board &before, u32 st_before, u32 st_after, int c, uint16_t mv)
{
    int from = move_from(mv), to = move_to(mv), fl = move_flags(mv);
    int src = (int)(((before.bb[1] >> from) & 1) | (((before.bb[2] >> from) & 1) << 1) |
                    (((before.bb[3] >> from) & 1) << 2));
    int cap = (int)(((before.bb[1] >> to) & 1) | (((before.bb[2] >> to) & 1) << 1) | (((before.bb[3] >> to) & 1) << 2));
    h.lo ^= PB_ZOB.side[0];
    h.hi ^= PB_ZOB.side[1];
    zpiece(h, c, src, from);
    zpiece(h, c, (fl & MF_PROMO) ? (fl & 3) + KNIGHT : src, to);
    if (cap) zpiece(h, 1 - c, cap, to);
    if (fl == MF_EP) zpiece(h, 1 - c, PAWN, c == WHITE ? to - 8 : to + 8);
    if (fl == MF_KING_CASTLE) {
        zpiece(h, c, ROOK, c == WHITE ? 7 : 63);
        zpiece(h, c, ROOK, c == WHITE ? 5 : 61);
    } else if (fl == MF_QUEEN_CASTLE) {
        zpiece(h, c, ROOK, c == WHITE ? 0 : 56);
        zpiece(h, c, ROOK, c == WHITE ? 3 : 59);
    }
    zstate(h, st_before);
    zstate(h, st_after);
    return h;
}

// ---------------------------------------------------------------- host TT
struct HostEntry {
    u64 lo, hi, count;
};

struct HostTT {
    std::vector<std::vector<HostEntry>> tab;  // per remaining depth
    std::vector<u64> used;
    bool ok = false;

    bool ready() const { return ok; }

    // Budget split over depths [first, last] proportional to 30^(last - d)
    // (launcher.cu:300-346 weights by branching factor the same way).
    void init(int budget_mb, int first, int last)
    {
        build_zobrist();
        if (first < 2) first = 2;
        if (last < first) last = first;
        u64 budget = budget_mb > 0 ? (u64)budget_mb << 20 : 0;
        if (!budget) {
            long pages = sysconf(_SC_PHYS_PAGES), psz = sysconf(_SC_PAGE_SIZE);
            u64 total = (pages > 0 && psz > 0) ? (u64)pages * (u64)psz : (8ULL << 30);
            budget = std::min<u64>(total / 4, 32ULL << 30);
        }
        tab.assign(last + 1, {});
        used.assign(last + 1, 0);
        double wsum = 0;
        for (int d = first; d <= last; d++) wsum += pow(30.0, last - d);
        for (int d = first; d <= last; d++) {
            double w = pow(30.0, last - d) / wsum;
            u64 slots = (u64)(budget * w) / sizeof(HostEntry);
            u64 p2 = 1024;
            while (p2 * 2 <= slots) p2 *= 2;
            tab[d].assign(p2, HostEntry{0, 0, 0});
        }
        ok = true;
    }
    bool probe(int depth, const Hash128 &h, u64 *out) const
    {
        if (depth >= (int)tab.size() || tab[depth].empty()) return false;
        const std::vector<HostEntry> &t = tab[depth];
        u64 mask = t.size() - 1;
        for (u64 i = h.lo & mask, k = 0; k < 64; k++, i = (i + 1) & mask) {
            const HostEntry &e = t[i];
            if (e.count == 0 && e.lo == 0 && e.hi == 0) return false;
            if (e.lo == h.lo && e.hi == h.hi) {
                *out = e.count - 1;
                return true;
            }
        }
        return false;
    }
    void store(int depth, const Hash128 &h, u64 count)
    {
        if (depth >= (int)tab.size() || tab[depth].empty()) return;
        std::vector<HostEntry> &t = tab[depth];
        if (used[depth] * 4 >= t.size() * 3) return;  // keep the load factor bounded
        u64 mask = t.size() - 1;
        for (u64 i = h.lo & mask, k = 0; k < 64; k++, i = (i + 1) & mask) {
            HostEntry &e = t[i];
            if (e.count == 0 && e.lo == 0 && e.hi == 0) {
                e.lo = h.lo;
                e.hi = h.hi;
                e.count = count + 1;  // +1 so an all-zero entry means empty
                used[depth]++;
                return;
            }
            if (e.lo == h.lo && e.hi == h.hi) return;
        }
    }
};


}  // namespace pb
