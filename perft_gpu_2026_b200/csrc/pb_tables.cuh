// pb_tables.cuh - builds the attack and geometry tables on the host and
// copies them into device global memory.
//
// The tables hold the same information as the reference's
// (GlobalVars.cpp:4-161, perft_kernels.cu:995-1134): empty-board knight and
// king attacks, between/line masks for every square pair, and fancy-magic
// slider attack tables.  The magic multipliers are this project's own
// (magic_numbers.inc, produced by magic_search.cpp) and the attack sets are
// filled by walking rays, so no table content is taken from the reference.
#pragma once
#include <string.h>
#include "pb_core.cuh"

namespace pb {

#include "magic_numbers.inc"

Tables h_tab;
u64 h_attacks[ATTACK_TABLE_SIZE];

namespace tables_detail {

static const int kRookDirs[4][2] = {{1, 0}, {-1, 0}, {0, 1}, {0, -1}};
static const int kBishopDirs[4][2] = {{1, 1}, {1, -1}, {-1, 1}, {-1, -1}};

// Ray walk from sq; with `inner_only` the last square of each ray (the board
// edge) is left out, which gives the relevant-occupancy mask.
static u64 slide(int sq, u64 occ, const int (*dirs)[2], bool inner_only)
{
    u64 out = 0;
    int f0 = sq & 7, r0 = sq >> 3;
    for (int d = 0; d < 4; d++) {
        int f = f0 + dirs[d][0], r = r0 + dirs[d][1];
        while (f >= 0 && f < 8 && r >= 0 && r < 8) {
            int nf = f + dirs[d][0], nr = r + dirs[d][1];
            bool at_edge = !(nf >= 0 && nf < 8 && nr >= 0 && nr < 8);
            if (inner_only && at_edge) break;
            out |= 1ULL << (r * 8 + f);
            if (occ & (1ULL << (r * 8 + f))) break;
            f = nf;
            r = nr;
        }
    }
    return out;
}

// Fills one square's slice of the attack table; returns false on a
// destructive collision (a wrong multiplier).
static bool fill_magic(Magic &m, int sq, u64 mul, const int (*dirs)[2], u32 offset)
{
    u64 mask = slide(sq, 0, dirs, true);
    int bits = popc(mask);
    m.mask = mask;
    m.magic = mul;
    m.base = offset;
    m.shift = 64 - bits;
    m.shift_hi = 32 - bits;
    u32 n = 1u << bits;
    for (u32 i = 0; i < n; i++) h_attacks[offset + i] = ~0ULL;
    u64 sub = 0;
    do {
        u64 att = slide(sq, sub, dirs, false);
        u32 idx = (u32)((sub * mul) >> m.shift);
        u64 &slot = h_attacks[offset + idx];
        if (slot != ~0ULL && slot != att) return false;
        slot = att;
        sub = (sub - mask) & mask;
    } while (sub);
    return true;
}

}  // namespace tables_detail

// Device copy of h_tab: magic slices point at their device addresses.
inline Tables device_tables(const u64 *dev_attacks)
{
    Tables t = h_tab;
    for (int sq = 0; sq < 64; sq++) {
        t.rook[sq].base = (u64)(uintptr_t)(dev_attacks + h_tab.rook[sq].base);
        t.bishop[sq].base = (u64)(uintptr_t)(dev_attacks + h_tab.bishop[sq].base);
    }
    return t;
}

// Builds h_tab / h_attacks.  Returns false if a multiplier is wrong.
inline bool build_host_tables()
{
    using namespace tables_detail;
    static bool built = false, ok = true;
    if (built) return ok;
    memset(&h_tab, 0, sizeof(h_tab));
    for (int sq = 0; sq < 64; sq++) {
        int f = sq & 7, r = sq >> 3;
        u64 kn = 0, kg = 0;
        static const int KN[8][2] = {{1, 2}, {2, 1}, {2, -1}, {1, -2}, {-1, -2}, {-2, -1}, {-2, 1}, {-1, 2}};
        for (int i = 0; i < 8; i++) {
            int nf = f + KN[i][0], nr = r + KN[i][1];
            if (nf >= 0 && nf < 8 && nr >= 0 && nr < 8) kn |= 1ULL << (nr * 8 + nf);
        }
        for (int df = -1; df <= 1; df++)
            for (int dr = -1; dr <= 1; dr++) {
                int nf = f + df, nr = r + dr;
                if ((df || dr) && nf >= 0 && nf < 8 && nr >= 0 && nr < 8) kg |= 1ULL << (nr * 8 + nf);
            }
        h_tab.knight[sq] = kn;
        h_tab.king[sq] = kg;
        h_tab.rook_empty[sq] = slide(sq, 0, kRookDirs, false);
        h_tab.bishop_empty[sq] = slide(sq, 0, kBishopDirs, false);
    }
    // between / line: walk each of the 8 directions from a
    static const int D8[8][2] = {{1, 0}, {-1, 0}, {0, 1}, {0, -1}, {1, 1}, {-1, -1}, {1, -1}, {-1, 1}};  // (2k, 2k+1) opposite
    for (int a = 0; a < 64; a++) {
        for (int d = 0; d < 8; d++) {
            u64 path = 0;
            int f = (a & 7) + D8[d][0], r = (a >> 3) + D8[d][1];
            while (f >= 0 && f < 8 && r >= 0 && r < 8) {
                int b = r * 8 + f;
                h_tab.between[a][b] = path;
                path |= 1ULL << b;
                f += D8[d][0];
                r += D8[d][1];
            }
        }
        for (int d = 0; d < 8; d += 2) {
            // full line through a in direction pair (d, d+1)
            u64 full = 1ULL << a;
            for (int k = d; k < d + 2; k++) {
                int f = (a & 7) + D8[k][0], r = (a >> 3) + D8[k][1];
                while (f >= 0 && f < 8 && r >= 0 && r < 8) {
                    full |= 1ULL << (r * 8 + f);
                    f += D8[k][0];
                    r += D8[k][1];
                }
            }
            u64 rest = full & ~(1ULL << a);
            while (rest) {
                int b = lsb(rest);
                h_tab.line[a][b] = full;
                rest &= rest - 1;
            }
        }
    }
    // zone reach: every square whose empty-board slider rays touch the zone
    for (int k = 0; k < 64; k++) {
        u64 zone = h_tab.king[k] | (1ULL << k);
        if (k == 4) zone |= 0x7CULL;                   // c1..g1
        if (k == 60) zone |= 0x7CULL << 56;            // c8..g8
        u64 rr = 0, br = 0, nr = 0;
        for (int sq = 0; sq < 64; sq++) {
            if (h_tab.rook_empty[sq] & zone) rr |= 1ULL << sq;
            if (h_tab.bishop_empty[sq] & zone) br |= 1ULL << sq;
            if (h_tab.knight[sq] & zone) nr |= 1ULL << sq;
        }
        h_tab.rook_reach[k] = rr;
        h_tab.bishop_reach[k] = br;
        h_tab.knight_reach[k] = nr;
    }
    u32 offset = 0;
    for (int sq = 0; sq < 64; sq++) {
        ok = ok && fill_magic(h_tab.rook[sq], sq, kRookMagic[sq], kRookDirs, offset);
        offset += 1u << (64 - h_tab.rook[sq].shift);
    }
    for (int sq = 0; sq < 64; sq++) {
        ok = ok && fill_magic(h_tab.bishop[sq], sq, kBishopMagic[sq], kBishopDirs, offset);
        offset += 1u << (64 - h_tab.bishop[sq].shift);
    }
    ok = ok && offset == (u32)ATTACK_TABLE_SIZE;
    built = true;
    return ok;
}

}  // namespace pb
