// pb_core.cuh - chess core shared by the host driver and the sm_100a kernels.
//
// Position = quad-bitboard (4 x u64 = 32 B; bb[0] = black pieces, bb[1..3] =
// the three bits of the piece code PAWN=1 .. KING=6), the same layout as the
// reference's QuadBitBoard (chess.h:66-76) so that 32-byte vector loads move
// a whole position.  The per-position state is one byte: castle rights in
// bits [3:0] (white K=1, Q=2, black K=4, Q=8) and the en-passant file + 1 in
// bits [7:4] (chess.h:78-92).  The side to move is not stored: every BFS level
// holds positions of one colour, passed as a template argument.
//
// Moves use the 16-bit from/to/flags layout of chess.h:94-144 so move lists
// printed by the tools read the same as the reference's.
//
// Legal-move counting follows the reference's countMoves
// (MoveGeneratorBitboard.h:1564-1943) step for step in what it counts,
// including its two counting conventions (two pawns capture-promoting onto
// one square, two pawns taking a checking pawn en passant: each counted once);
// the STRICT template flag counts those cases exactly.  Generation
// (MoveGeneratorBitboard.h:978-1554) is always exact, and the BFS sizes its
// levels with the STRICT count so a level never holds more moves than it was
// sized for.
#pragma once
#include <stdint.h>

#ifdef __CUDACC__
#define PB_HD __host__ __device__ __forceinline__
#else
#define PB_HD inline
#endif

namespace pb {

typedef unsigned long long u64;
typedef unsigned int u32;

enum { WHITE = 0, BLACK = 1 };
enum { PAWN = 1, KNIGHT = 2, BISHOP = 3, ROOK = 4, QUEEN = 5, KING = 6 };
enum {
    MF_QUIET = 0, MF_DOUBLE_PUSH = 1, MF_KING_CASTLE = 2, MF_QUEEN_CASTLE = 3,
    MF_CAPTURE = 4, MF_EP = 5, MF_PROMO = 8
};
enum { MAX_MOVES = 256 };

struct __align__(32) Board {
    u64 bb[4];
};

constexpr u64 RANK1 = 0x00000000000000FFULL;
constexpr u64 RANK3 = 0x0000000000FF0000ULL;
constexpr u64 RANK6 = 0x0000FF0000000000ULL;
constexpr u64 RANK8 = 0xFF00000000000000ULL;
constexpr u64 FILEA = 0x0101010101010101ULL;
constexpr u64 FILEH = 0x8080808080808080ULL;
constexpr u64 PROMO_RANKS = RANK1 | RANK8;

// Slider magic entry: attacks = table[offset + ((occ & mask) * magic) >> (64 - bits)].
// `base` is the slice's offset into the attack table on the host and, in the
// device copy, the slice's device address, so a lookup ends in one IMAD-based
// address computation and one load.
struct __align__(32) Magic {
    u64 mask;
    u64 magic;
    u64 base;
    u32 shift_hi;  // 32 - bits: the index is the product's high word >> shift_hi
    u32 shift;     // 64 - bits
};

// Attack and geometry tables.  One copy lives in device global memory
// (g_tab, read with the non-coherent path) and one on the host (h_tab).
struct Tables {
    Magic rook[64];
    Magic bishop[64];
    u64 knight[64];
    u64 king[64];
    u64 rook_empty[64];
    u64 bishop_empty[64];
    u64 between[64][64];
    u64 line[64][64];
    // Squares from which a rook / bishop on an empty board attacks the zone
    // of a king on that square: its 3x3 block and, for e1/e8, the castling
    // squares c..g of its back rank.
    u64 rook_reach[64];
    u64 bishop_reach[64];
    u64 knight_reach[64];  // squares from which a knight attacks that zone
};
constexpr int ATTACK_TABLE_SIZE = 107648;  // sum over squares of 2^bits (rook 102400 + bishop 5248)

extern Tables h_tab;
extern u64 h_attacks[ATTACK_TABLE_SIZE];

// Device copies; the engine is one translation unit, so they are defined here.
__device__ Tables g_tab;
__device__ u64 g_attacks[ATTACK_TABLE_SIZE];

// ---------------------------------------------------------------- bit ops
PB_HD int popc(u64 x)
{
#ifdef __CUDA_ARCH__
    return __popcll(x);
#else
    return __builtin_popcountll(x);
#endif
}
// Index of the lowest set bit (x != 0).  On the GPU this is a population
// count of the bits below it: POPC issues on the XU pipe, which leaves the
// ALU pipe (the leaf kernel's bottleneck) free.
PB_HD int lsb(u64 x)
{
#ifdef __CUDA_ARCH__
    return __popcll((x - 1) & ~x);
#else
    return __builtin_ctzll(x);
#endif
}
// Index of a single set bit.
PB_HD int bit_index(u64 single)
{
#ifdef __CUDA_ARCH__
    return __popcll(single - 1);
#else
    return __builtin_ctzll(single);
#endif
}
PB_HD bool more_than_one(u64 x) { return (x & (x - 1)) != 0; }

PB_HD u64 north(u64 x) { return x << 8; }
PB_HD u64 south(u64 x) { return x >> 8; }
PB_HD u64 east1(u64 x) { return (x << 1) & ~FILEA; }
PB_HD u64 west1(u64 x) { return (x >> 1) & ~FILEH; }

// Side-relative pawn geometry.
template <int C> PB_HD u64 push1(u64 x) { return C == WHITE ? (x << 8) : (x >> 8); }
template <int C> PB_HD u64 cap_west(u64 x) { return C == WHITE ? ((x << 7) & ~FILEH) : ((x >> 9) & ~FILEH); }
template <int C> PB_HD u64 cap_east(u64 x) { return C == WHITE ? ((x << 9) & ~FILEA) : ((x >> 7) & ~FILEA); }
template <int C> PB_HD u64 double_push_rank() { return C == WHITE ? RANK3 : RANK6; }

// ---------------------------------------------------------------- table access
#ifdef __CUDA_ARCH__
__device__ __forceinline__ u64 ldg64(const u64 *p) { return __ldg(p); }
#define PB_TAB g_tab
#define PB_ATT g_attacks
#else
PB_HD u64 ldg64(const u64 *p) { return *p; }
#define PB_TAB h_tab
#define PB_ATT h_attacks
#endif

PB_HD u64 magic_lookup(const Magic *e, u64 occ)
{
#ifdef __CUDA_ARCH__
    // bits <= 12, so the index lies in the high word of the product: one
    // 32-bit shift instead of a 64-bit variable shift
    // the whole 32-byte entry in one 256-bit load
    u64 mask, mul, base, sh;
    asm("ld.global.nc.v4.u64 {%0,%1,%2,%3}, [%4];" : "=l"(mask), "=l"(mul), "=l"(base), "=l"(sh) : "l"(e));
    u32 hi = (u32)(((occ & mask) * mul) >> 32);
    return __ldg(reinterpret_cast<const u64 *>(base) + (hi >> (u32)sh));
#else
    u64 idx = ((occ & e->mask) * e->magic) >> e->shift;
    return h_attacks[e->base + (u32)idx];
#endif
}
PB_HD u64 rook_att(int sq, u64 occ) { return magic_lookup(&PB_TAB.rook[sq], occ); }
PB_HD u64 bishop_att(int sq, u64 occ) { return magic_lookup(&PB_TAB.bishop[sq], occ); }
PB_HD u64 knight_att(int sq) { return ldg64(&PB_TAB.knight[sq]); }
PB_HD u64 king_att(int sq) { return ldg64(&PB_TAB.king[sq]); }
PB_HD u64 between(int a, int b) { return ldg64(&PB_TAB.between[a][b]); }
PB_HD u64 line_through(int a, int b) { return ldg64(&PB_TAB.line[a][b]); }
PB_HD u64 rook_empty(int sq) { return ldg64(&PB_TAB.rook_empty[sq]); }
PB_HD u64 bishop_empty(int sq) { return ldg64(&PB_TAB.bishop_empty[sq]); }
PB_HD u64 rook_reach(int ksq) { return ldg64(&PB_TAB.rook_reach[ksq]); }
PB_HD u64 bishop_reach(int ksq) { return ldg64(&PB_TAB.bishop_reach[ksq]); }
PB_HD u64 knight_reach(int ksq) { return ldg64(&PB_TAB.knight_reach[ksq]); }

// Knight attacks of a whole set by shifts (no per-piece loop).
PB_HD u64 knights_bulk(u64 n)
{
    u64 l1 = (n >> 1) & 0x7f7f7f7f7f7f7f7fULL;
    u64 l2 = (n >> 2) & 0x3f3f3f3f3f3f3f3fULL;
    u64 r1 = (n << 1) & 0xfefefefefefefefeULL;
    u64 r2 = (n << 2) & 0xfcfcfcfcfcfcfcfcULL;
    u64 h1 = l1 | r1, h2 = l2 | r2;
    return (h1 << 16) | (h1 >> 16) | (h2 << 8) | (h2 >> 8);
}

// ---------------------------------------------------------------- moves
PB_HD uint16_t make_move_code(int from, int to, int flags)
{
    return (uint16_t)((flags << 12) | (to << 6) | from);
}
PB_HD int move_from(uint16_t m) { return m & 63; }
PB_HD int move_to(uint16_t m) { return (m >> 6) & 63; }
PB_HD int move_flags(uint16_t m) { return m >> 12; }

// EP target square for the side to move C (the capturing side).
template <int C> PB_HD u64 ep_target(u32 state)
{
    u32 f = state >> 4;
    if (!f) return 0;
    return C == WHITE ? (1ULL << (39 + f)) : (1ULL << (15 + f));
}

// ---------------------------------------------------------------- piece sets
struct Sets {
    u64 occ, us, them, pawns, knights, bq, rq, kings;
};

template <int C> PB_HD Sets derive(const Board &b)
{
    Sets s;
    s.occ = b.bb[1] | b.bb[2] | b.bb[3];
    u64 black = b.bb[0];
    s.us = C == WHITE ? (s.occ & ~black) : black;
    s.them = s.occ ^ s.us;
    s.pawns = b.bb[1] & ~b.bb[2] & ~b.bb[3];
    s.knights = b.bb[2] & ~b.bb[1] & ~b.bb[3];
    s.bq = b.bb[1] & (b.bb[2] ^ b.bb[3]);
    s.rq = b.bb[3] & ~b.bb[2];
    s.kings = b.bb[2] & b.bb[3] & ~b.bb[1];
    return s;
}

// Pieces standing alone between the king and an aligned enemy slider
// (findPinnedPieces, MoveGeneratorBitboard.h:803-831).
PB_HD u64 pinned_set(int ksq, u64 eb, u64 er, u64 occ)
{
    u64 snipers = (bishop_empty(ksq) & eb) | (rook_empty(ksq) & er);
    u64 pinned = 0;
    while (snipers) {
        int s = lsb(snipers);
        u64 bt = between(s, ksq) & occ;
        if (bt && !more_than_one(bt)) pinned |= bt;
        snipers &= snipers - 1;
    }
    return pinned;
}

// Squares attacked by the side not to move, sliders looking through the
// moving side's king (findAttackedSquares, MoveGeneratorBitboard.h:835-875).
// Callers only test the zone of the king on `ksq` (its 3x3 block and the
// castling squares), so the map is exact there and may miss squares
// elsewhere: sliders that cannot reach the zone even on an empty board are
// skipped before the lookup loop, which shortens the loop for every lane.
template <int C> PB_HD u64 enemy_attacks(const Sets &s, u64 my_king, int ksq)
{
    u64 ep = s.pawns & s.them;
    u64 a = cap_west<1 - C>(ep) | cap_east<1 - C>(ep);
    a |= king_att(bit_index(s.kings & s.them));
    for (u64 kn = s.knights & s.them & knight_reach(ksq); kn; kn &= kn - 1) a |= knight_att(lsb(kn));
    u64 occ = s.occ ^ my_king;
    u64 b = s.bq & s.them & bishop_reach(ksq);
    while (b) {
        a |= bishop_att(lsb(b), occ);
        b &= b - 1;
    }
    u64 r = s.rq & s.them & rook_reach(ksq);
    while (r) {
        a |= rook_att(lsb(r), occ);
        r &= r - 1;
    }
    return a;
}

// ---------------------------------------------------------------- own pieces
// Moves of the side to move's knights, bishops, rooks and queens, counted for
// the move counters below: pieces in `movable` (own and not pinned) move to
// `targets`; pinned own sliders in `pinned_lines` (empty when in check) move
// along the line through their king to squares without an own piece.
//
// BitboardPieces walks the piece sets of the position being counted.
struct BitboardPieces {
    PB_HD u32 count(const Sets &s, u64 movable, u64 targets, u64 pinned_lines, int ksq) const
    {
        u32 n = 0;
        for (u64 kn = s.knights & movable; kn; kn &= kn - 1) n += popc(knight_att(lsb(kn)) & targets);
        for (u64 bs = s.bq & movable; bs; bs &= bs - 1) n += popc(bishop_att(lsb(bs), s.occ) & targets);
        for (u64 rs = s.rq & movable; rs; rs &= rs - 1) n += popc(rook_att(lsb(rs), s.occ) & targets);
        if (pinned_lines & (s.bq | s.rq)) {
            // a pinned slider moves only along the line through its king
            for (u64 bs = s.bq & s.us & pinned_lines; bs; bs &= bs - 1) {
                int sq = lsb(bs);
                n += popc(bishop_att(sq, s.occ) & ~s.us & line_through(sq, ksq));
            }
            for (u64 rs = s.rq & s.us & pinned_lines; rs; rs &= rs - 1) {
                int sq = lsb(rs);
                n += popc(rook_att(sq, s.occ) & ~s.us & line_through(sq, ksq));
            }
        }
        return n;
    }
};

// Listed pieces serve the positions one move of the OTHER side away from a
// position P (the grandchildren of the fused leaf): the side to move there has
// the pieces it had in P, less at most one that the other side captured.  Its
// knight, diagonal-mover (bishop, queen) and orthogonal-mover (rook, queen)
// squares are listed once from P, four per kind at most, one byte each
// (square + 1, 0 = end), so the counts iterate the lists instead of scanning
// bitboards.  Pieces whose move set differs from the plain one (captured, or
// pinned) are corrected afterwards; that path is rare.
//
// ListedPieces::build writes the three lists and the listed squares to
// caller storage (shared memory in the leaf kernels: kept in registers across
// the grandchild loop they made the kernel spill); ListedView is the counting
// policy that reads them back at every count.
struct ListedPieces {
    // Lists side C's pieces of `b` into l[0..2] and *listed; false if a kind
    // has more than four.
    template <int C> static PB_HD bool build(const Board &b, u32 *l, u64 *listed)
    {
        Sets s = derive<C>(b);
        u64 k = s.knights & s.us, d = s.bq & s.us, o = s.rq & s.us;
        *listed = k | d | o;
        return pack(k, l[0]) && pack(d, l[1]) && pack(o, l[2]);
    }
    static PB_HD bool pack(u64 set, u32 &out)
    {
        out = 0;
        for (int k = 0; set; k++, set &= set - 1) {
            if (k == 4) return false;
            out |= (u32)(lsb(set) + 1) << (8 * k);
        }
        return true;
    }
    // true if one of the list's bytes equals key (1..64): a zero-byte test of
    // the list XOR the key repeated in every byte
    static PB_HD bool has(u32 list, u32 key)
    {
        u32 x = list ^ (key * 0x01010101u);
        return ((x - 0x01010101u) & ~x & 0x80808080u) != 0;
    }
};

struct ListedView {
    const volatile u32 *l;  // knights, diagonal movers, orthogonal movers
    const volatile u64 *m;  // the listed squares
    PB_HD u32 count(const Sets &s, u64 movable, u64 targets, u64 pinned_lines, int ksq) const
    {
        const u32 kn = l[0], dg = l[1], og = l[2];
        u32 n = 0;
        for (u32 q = kn; q; q >>= 8) n += popc(knight_att((int)(q & 255) - 1) & targets);
        for (u32 q = dg; q; q >>= 8) n += popc(bishop_att((int)(q & 255) - 1, s.occ) & targets);
        for (u32 q = og; q; q >>= 8) n += popc(rook_att((int)(q & 255) - 1, s.occ) & targets);
        // listed squares that are not movable: captured (no longer own) or
        // pinned.  Take back what the lists counted for them and add the
        // pinned sliders' moves along their lines.
        for (u64 fix = *m & ~movable; fix; fix &= fix - 1) {
            const int sq = lsb(fix);
            const u32 key = (u32)sq + 1;
            const u64 line = ((pinned_lines & s.us) >> sq) & 1 ? line_through(sq, ksq) : 0;
            if (ListedPieces::has(kn, key)) n -= popc(knight_att(sq) & targets);
            if (ListedPieces::has(dg, key)) {
                u64 a = bishop_att(sq, s.occ);
                n += popc(a & ~s.us & line) - popc(a & targets);
            }
            if (ListedPieces::has(og, key)) {
                u64 a = rook_att(sq, s.occ);
                n += popc(a & ~s.us & line) - popc(a & targets);
            }
        }
        return n;
    }
};

// ---------------------------------------------------------------- counting
// Legal-move count when the side to move is in check
// (countMovesOutOfCheck, MoveGeneratorBitboard.h:1564-1694).
template <int C, bool STRICT>
PB_HD u32 count_evasions(const Sets &s, u32 state, u64 pinned, u64 threat, int ksq)
{
    u64 king = 1ULL << ksq;
    u64 checkers = (cap_west<C>(king) | cap_east<C>(king)) & s.pawns & s.them;
    checkers |= knight_att(ksq) & s.knights & s.them;
    checkers |= bishop_att(ksq, s.occ) & s.bq & s.them;
    checkers |= rook_att(ksq, s.occ) & s.rq & s.them;
    u32 n = popc(king_att(ksq) & ~(threat | s.us));
    if (more_than_one(checkers)) return n;

    u64 safe = checkers | between(ksq, bit_index(checkers));
    u64 mine = s.us & ~pinned;
    u64 empty = ~s.occ;
    u64 pawns = s.pawns & mine;
    u64 p1 = push1<C>(pawns) & empty;
    u64 d = p1 & safe;
    u64 pr = d & PROMO_RANKS;
    n += popc(d ^ pr) + 4 * popc(pr);
    n += popc(push1<C>(p1 & double_push_rank<C>()) & empty & safe);
    u64 cw = cap_west<C>(pawns) & s.them & safe;
    u64 ce = cap_east<C>(pawns) & s.them & safe;
    u64 pw = cw & PROMO_RANKS, pe = ce & PROMO_RANKS;
    n += popc(cw ^ pw) + 4 * popc(pw) + popc(ce ^ pe) + 4 * popc(pe);
    u64 ept = ep_target<C>(state);
    if (ept) {
        u64 victim = push1<1 - C>(ept);
        if (victim == checkers) {
            u64 w = cap_west<C>(pawns) & ept, e = cap_east<C>(pawns) & ept;
            n += STRICT ? popc(w) + popc(e) : popc(w | e);
        }
    }
    u64 kn = s.knights & mine;
    while (kn) {
        n += popc(knight_att(lsb(kn)) & safe);
        kn &= kn - 1;
    }
    u64 b = s.bq & mine;
    while (b) {
        n += popc(bishop_att(lsb(b), s.occ) & safe);
        b &= b - 1;
    }
    u64 r = s.rq & mine;
    while (r) {
        n += popc(rook_att(lsb(r), s.occ) & safe);
        r &= r - 1;
    }
    return n;
}

// Legal-move count when the side to move is not in check (the main part of
// countMoves, MoveGeneratorBitboard.h:1729-1943).
template <int C, bool STRICT, class Own = BitboardPieces>
PB_HD u32 count_quiet(const Sets &s, u32 state, u64 pinned, u64 threat, int ksq, const Own &own = Own())
{
    const u64 er = s.rq & s.them;
    u32 n = 0;
    u64 empty = ~s.occ;
    u64 my_pawns = s.pawns & s.us;

    u64 ept = ep_target<C>(state);
    if (ept) {
        u64 victim = push1<1 - C>(ept);
        u64 src = (east1(victim) | west1(victim)) & my_pawns;
        while (src) {
            int psq = lsb(src);
            u64 pawn = 1ULL << psq;
            if (pawn & pinned) {
                if (ept & line_through(psq, ksq)) n++;
            } else {
                u64 occ2 = s.occ ^ victim ^ pawn;
                u64 rank = RANK1 << (ksq & 56);
                if (!(rook_att(ksq, occ2) & er & rank)) n++;
            }
            src &= src - 1;
        }
    }

    u64 pp = my_pawns & pinned;
    while (pp) {
        int psq = lsb(pp);
        u64 pawn = 1ULL << psq;
        u64 ln = line_through(psq, ksq);
        u64 d = push1<C>(pawn) & ln & empty;
        if (d) {
            n++;
            if (push1<C>(d & double_push_rank<C>()) & empty) n++;
        }
        d = (cap_west<C>(pawn) | cap_east<C>(pawn)) & ln & s.them;
        if (d) n += (d & PROMO_RANKS) ? 4 : 1;
        pp &= pp - 1;
    }

    u64 fp = my_pawns & ~pinned;
    u64 p1 = push1<C>(fp) & empty;
    n += popc(push1<C>(p1 & double_push_rank<C>()) & empty);
    u64 cw = cap_west<C>(fp) & s.them, ce = cap_east<C>(fp) & s.them;
    constexpr u64 RANK7 = C == WHITE ? 0x00FF000000000000ULL : 0x000000000000FF00ULL;
    if (!(fp & RANK7)) {
        // no pawn can promote: every push and capture is one move
        n += popc(p1) + popc(cw) + popc(ce);
    } else {
        u64 promos = p1 & PROMO_RANKS;
        u64 pw = cw & PROMO_RANKS, pe = ce & PROMO_RANKS;
        n += popc(p1 ^ promos) + popc(cw ^ pw) + popc(ce ^ pe);
        if (STRICT)
            n += 4 * (popc(promos) + popc(pw) + popc(pe));
        else
            n += 4 * popc(promos | pw | pe);
    }

    u32 castle = C == WHITE ? (state & 3) : ((state >> 2) & 3);
    if (castle) {
        constexpr u64 KS = C == WHITE ? 0x60ULL : 0x6000000000000000ULL;
        constexpr u64 QS_EMPTY = C == WHITE ? 0x0EULL : 0x0E00000000000000ULL;
        constexpr u64 QS_SAFE = C == WHITE ? 0x0CULL : 0x0C00000000000000ULL;
        if ((castle & 1) && !(KS & (s.occ | threat))) n++;
        if ((castle & 2) && !(QS_EMPTY & s.occ) && !(QS_SAFE & threat)) n++;
    }

    n += popc(king_att(ksq) & ~(threat | s.us));
    n += own.count(s, s.us & ~pinned, ~s.us, pinned, ksq);
    return n;
}

// What every move count needs first: piece sets, king square, pinned pieces
// and the enemy attack map (findPinnedPieces + findAttackedSquares).
struct CountPrep {
    Sets s;
    u64 pinned, threat;
    int ksq;
};
template <int C> PB_HD CountPrep count_prep(const Board &b)
{
    CountPrep p;
    p.s = derive<C>(b);
    u64 my_king = p.s.kings & p.s.us;
    p.ksq = bit_index(my_king);
    p.pinned = pinned_set(p.ksq, p.s.bq & p.s.them, p.s.rq & p.s.them, p.s.occ);
    p.threat = enemy_attacks<C>(p.s, my_king, p.ksq);
    return p;
}
template <int C> PB_HD bool prep_in_check(const CountPrep &p) { return (p.threat >> p.ksq) & 1; }

// Number of legal moves (countMoves, MoveGeneratorBitboard.h:1700-1943, and
// countMovesOutOfCheck, :1564-1694, for a side in check).
//
// One code path for both cases, so a warp whose lanes disagree on being in
// check does not run two count routines one after the other: every non-king
// move must end on `safe` (all squares when not in check; the checker and
// the squares between it and the king in single check; none in double
// check), pinned pieces and castling are skipped in check, and the in-check
// conventions of the out-of-check counter are kept (promotions counted per
// capture direction, one en-passant capture of a checking pawn however many
// pawns can take it).  Equal to count_quiet / count_evasions.  On the GPU a
// group of lanes none of which is in check takes count_quiet, which skips
// the masking.
template <int C, bool STRICT, class Own = BitboardPieces>
PB_HD u32 count_moves(const Board &b, u32 state, const Own &own = Own())
{
    const CountPrep p = count_prep<C>(b);
    const Sets &s = p.s;
    const int ksq = p.ksq;
    const u64 king = 1ULL << ksq;
    const bool check = (p.threat & king) != 0;
#ifdef __CUDA_ARCH__
    // no lane of the converged group in check: the leaner not-in-check path
    if (!__any_sync(__activemask(), check)) return count_quiet<C, STRICT>(s, state, p.pinned, p.threat, ksq, own);
#endif
    u64 safe = ~0ULL, checkers = 0;
    if (check) {
        checkers = (cap_west<C>(king) | cap_east<C>(king)) & s.pawns & s.them;
        checkers |= knight_att(ksq) & s.knights & s.them;
        checkers |= bishop_att(ksq, s.occ) & s.bq & s.them;
        checkers |= rook_att(ksq, s.occ) & s.rq & s.them;
        safe = more_than_one(checkers) ? 0 : checkers | between(ksq, bit_index(checkers));
    }
    const u64 pinned = check ? 0 : p.pinned;  // in check a pinned piece never moves
    const u64 movable = s.us & ~p.pinned;
    const u64 er = s.rq & s.them;
    const u64 empty = ~s.occ;
    const u64 my_pawns = s.pawns & s.us;
    u32 n = popc(king_att(ksq) & ~(p.threat | s.us));

    u64 ept = ep_target<C>(state);
    if (ept) {
        u64 victim = push1<1 - C>(ept);
        if (!check || victim == checkers) {
            u64 src = (east1(victim) | west1(victim)) & (check ? my_pawns & movable : my_pawns);
            u32 e = 0;
            while (src) {
                int psq = lsb(src);
                u64 pawn = 1ULL << psq;
                if (pawn & pinned) {
                    if (ept & line_through(psq, ksq)) e++;
                } else {
                    u64 occ2 = s.occ ^ victim ^ pawn;
                    u64 rank = RANK1 << (ksq & 56);
                    if (!(rook_att(ksq, occ2) & er & rank)) e++;
                }
                src &= src - 1;
            }
            n += (check && !STRICT && e > 1u) ? 1u : e;
        }
    }

    u64 pp = my_pawns & pinned;
    while (pp) {
        int psq = lsb(pp);
        u64 pawn = 1ULL << psq;
        u64 ln = line_through(psq, ksq);
        u64 d = push1<C>(pawn) & ln & empty;
        if (d) {
            n++;
            if (push1<C>(d & double_push_rank<C>()) & empty) n++;
        }
        d = (cap_west<C>(pawn) | cap_east<C>(pawn)) & ln & s.them;
        if (d) n += (d & PROMO_RANKS) ? 4 : 1;
        pp &= pp - 1;
    }

    const u64 fp = my_pawns & movable;
    const u64 p1 = push1<C>(fp) & empty;
    const u64 s1 = p1 & safe;
    n += popc(push1<C>(p1 & double_push_rank<C>()) & empty & safe);
    const u64 cw = cap_west<C>(fp) & s.them & safe, ce = cap_east<C>(fp) & s.them & safe;
    constexpr u64 RANK7 = C == WHITE ? 0x00FF000000000000ULL : 0x000000000000FF00ULL;
    if (!(fp & RANK7)) {
        n += popc(s1) + popc(cw) + popc(ce);
    } else {
        u64 promos = s1 & PROMO_RANKS;
        u64 pw = cw & PROMO_RANKS, pe = ce & PROMO_RANKS;
        n += popc(s1 ^ promos) + popc(cw ^ pw) + popc(ce ^ pe);
        if (STRICT || check)
            n += 4 * (popc(promos) + popc(pw) + popc(pe));
        else
            n += 4 * popc(promos | pw | pe);
    }

    u32 castle = C == WHITE ? (state & 3) : ((state >> 2) & 3);
    if (castle && !check) {
        constexpr u64 KS = C == WHITE ? 0x60ULL : 0x6000000000000000ULL;
        constexpr u64 QS_EMPTY = C == WHITE ? 0x0EULL : 0x0E00000000000000ULL;
        constexpr u64 QS_SAFE = C == WHITE ? 0x0CULL : 0x0C00000000000000ULL;
        if ((castle & 1) && !(KS & (s.occ | p.threat))) n++;
        if ((castle & 2) && !(QS_EMPTY & s.occ) && !(QS_SAFE & p.threat)) n++;
    }

    n += own.count(s, movable, ~s.us & safe, pinned, ksq);
    return n;
}

// ---------------------------------------------------------------- generation
// A move sink receives moves one by one.  ArraySink writes a plain array.
struct ArraySink {
    uint16_t *p;
    int n;
    PB_HD void put(uint16_t m) { p[n++] = m; }
};

template <class Sink> PB_HD void emit_targets(Sink &sink, int from, u64 dsts)
{
    while (dsts) {
        sink.put(make_move_code(from, lsb(dsts), MF_QUIET));
        dsts &= dsts - 1;
    }
}
template <class Sink> PB_HD void emit_pawn(Sink &sink, int from, int to, int flags)
{
    if ((1ULL << to) & PROMO_RANKS) {
        sink.put(make_move_code(from, to, flags | 8));
        sink.put(make_move_code(from, to, flags | 9));
        sink.put(make_move_code(from, to, flags | 10));
        sink.put(make_move_code(from, to, flags | 11));
    } else {
        sink.put(make_move_code(from, to, flags));
    }
}

// Moves out of check (generateMovesOutOfCheck, MoveGeneratorBitboard.h:978-1154).
template <int C, class Sink>
PB_HD void gen_evasions(const Sets &s, u32 state, u64 pinned, u64 threat, int ksq, Sink &sink)
{
    u64 king = 1ULL << ksq;
    u64 checkers = (cap_west<C>(king) | cap_east<C>(king)) & s.pawns & s.them;
    checkers |= knight_att(ksq) & s.knights & s.them;
    checkers |= bishop_att(ksq, s.occ) & s.bq & s.them;
    checkers |= rook_att(ksq, s.occ) & s.rq & s.them;
    emit_targets(sink, ksq, king_att(ksq) & ~(threat | s.us));
    if (more_than_one(checkers)) return;

    u64 safe = checkers | between(ksq, bit_index(checkers));
    u64 mine = s.us & ~pinned;
    u64 empty = ~s.occ;
    u64 ept = ep_target<C>(state);
    if (ept && push1<1 - C>(ept) != checkers) ept = 0;
    u64 pawns = s.pawns & mine;
    while (pawns) {
        int psq = lsb(pawns);
        u64 pawn = 1ULL << psq;
        u64 d = push1<C>(pawn) & empty;
        if (d) {
            if (d & safe) {
                emit_pawn(sink, psq, lsb(d), MF_QUIET);
            } else {
                d = push1<C>(d & double_push_rank<C>()) & empty & safe;
                if (d) {
                    int fl = ((east1(d) | west1(d)) & s.pawns & s.them) ? MF_DOUBLE_PUSH : MF_QUIET;
                    sink.put(make_move_code(psq, lsb(d), fl));
                }
            }
        }
        u64 caps = cap_west<C>(pawn) | cap_east<C>(pawn);
        d = caps & s.them & safe;
        if (d) emit_pawn(sink, psq, lsb(d), MF_CAPTURE);
        if (caps & ept) sink.put(make_move_code(psq, lsb(ept), MF_EP));
        pawns &= pawns - 1;
    }
    u64 kn = s.knights & mine;
    while (kn) {
        int sq = lsb(kn);
        emit_targets(sink, sq, knight_att(sq) & safe);
        kn &= kn - 1;
    }
    u64 b = s.bq & mine;
    while (b) {
        int sq = lsb(b);
        emit_targets(sink, sq, bishop_att(sq, s.occ) & safe);
        b &= b - 1;
    }
    u64 r = s.rq & mine;
    while (r) {
        int sq = lsb(r);
        emit_targets(sink, sq, rook_att(sq, s.occ) & safe);
        r &= r - 1;
    }
}

// All legal moves (generateMovesToSink, MoveGeneratorBitboard.h:1160-1554).
// Capture flags are not set (make_move does not need them); a double push
// carries MF_DOUBLE_PUSH only when an enemy pawn stands beside the target
// square, so the en-passant state is set only when a capture can follow.
template <int C, class Sink> PB_HD void gen_moves(const Board &b, u32 state, Sink &sink)
{
    Sets s = derive<C>(b);
    u64 my_king = s.kings & s.us;
    int ksq = bit_index(my_king);
    u64 eb = s.bq & s.them, er = s.rq & s.them;
    u64 pinned = pinned_set(ksq, eb, er, s.occ);
    u64 threat = enemy_attacks<C>(s, my_king, ksq);
    if (threat & my_king) {
        gen_evasions<C>(s, state, pinned, threat, ksq, sink);
        return;
    }
    u64 empty = ~s.occ;
    u64 my_pawns = s.pawns & s.us;
    u64 enemy_pawns = s.pawns & s.them;

    u64 pp = my_pawns & pinned;
    while (pp) {
        int psq = lsb(pp);
        u64 pawn = 1ULL << psq;
        u64 ln = line_through(psq, ksq);
        u64 d = (cap_west<C>(pawn) | cap_east<C>(pawn)) & ln & s.them;
        if (d) emit_pawn(sink, psq, lsb(d), MF_CAPTURE);
        d = push1<C>(pawn) & ln & empty;
        if (d) {
            sink.put(make_move_code(psq, lsb(d), MF_QUIET));
            d = push1<C>(d & double_push_rank<C>()) & empty;
            if (d) {
                int fl = ((east1(d) | west1(d)) & enemy_pawns) ? MF_DOUBLE_PUSH : MF_QUIET;
                sink.put(make_move_code(psq, lsb(d), fl));
            }
        }
        pp &= pp - 1;
    }
    u64 fp = my_pawns & ~pinned;
    while (fp) {
        int psq = lsb(fp);
        u64 pawn = 1ULL << psq;
        u64 d = cap_west<C>(pawn) & s.them;
        if (d) emit_pawn(sink, psq, lsb(d), MF_CAPTURE);
        d = cap_east<C>(pawn) & s.them;
        if (d) emit_pawn(sink, psq, lsb(d), MF_CAPTURE);
        d = push1<C>(pawn) & empty;
        if (d) {
            emit_pawn(sink, psq, lsb(d), MF_QUIET);
            d = push1<C>(d & double_push_rank<C>()) & empty;
            if (d) {
                int fl = ((east1(d) | west1(d)) & enemy_pawns) ? MF_DOUBLE_PUSH : MF_QUIET;
                sink.put(make_move_code(psq, lsb(d), fl));
            }
        }
        fp &= fp - 1;
    }
    u64 ept = ep_target<C>(state);
    if (ept) {
        u64 victim = push1<1 - C>(ept);
        u64 src = (east1(victim) | west1(victim)) & my_pawns;
        while (src) {
            int psq = lsb(src);
            u64 pawn = 1ULL << psq;
            bool ok;
            if (pawn & pinned) {
                ok = (ept & line_through(psq, ksq)) != 0;
            } else {
                u64 occ2 = s.occ ^ victim ^ pawn;
                u64 rank = RANK1 << (ksq & 56);
                ok = !(rook_att(ksq, occ2) & er & rank);
            }
            if (ok) sink.put(make_move_code(psq, lsb(ept), MF_EP));
            src &= src - 1;
        }
    }
    emit_targets(sink, ksq, king_att(ksq) & ~(threat | s.us));
    u64 kn = s.knights & s.us & ~pinned;
    while (kn) {
        int sq = lsb(kn);
        emit_targets(sink, sq, knight_att(sq) & ~s.us);
        kn &= kn - 1;
    }
    u64 bs = s.bq & s.us;
    while (bs) {
        int sq = lsb(bs);
        u64 m = bishop_att(sq, s.occ) & ~s.us;
        if (pinned & (1ULL << sq)) m &= line_through(sq, ksq);
        emit_targets(sink, sq, m);
        bs &= bs - 1;
    }
    u64 rs = s.rq & s.us;
    while (rs) {
        int sq = lsb(rs);
        u64 m = rook_att(sq, s.occ) & ~s.us;
        if (pinned & (1ULL << sq)) m &= line_through(sq, ksq);
        emit_targets(sink, sq, m);
        rs &= rs - 1;
    }
    u32 castle = C == WHITE ? (state & 3) : ((state >> 2) & 3);
    if (castle) {
        constexpr u64 KS = C == WHITE ? 0x60ULL : 0x6000000000000000ULL;
        constexpr u64 QS_EMPTY = C == WHITE ? 0x0EULL : 0x0E00000000000000ULL;
        constexpr u64 QS_SAFE = C == WHITE ? 0x0CULL : 0x0C00000000000000ULL;
        constexpr int KSQ = C == WHITE ? 4 : 60;
        if ((castle & 1) && !(KS & (s.occ | threat))) sink.put(make_move_code(KSQ, KSQ + 2, MF_KING_CASTLE));
        if ((castle & 2) && !(QS_EMPTY & s.occ) && !(QS_SAFE & threat))
            sink.put(make_move_code(KSQ, KSQ - 2, MF_QUEEN_CASTLE));
    }
}

// ---------------------------------------------------------------- make move
// Applies a move for side C (makeMove, MoveGeneratorBitboard.h:1945-2040).
// Castle rights drop whenever a move starts or ends on a king or rook home
// square; the EP file is set only by a flagged double push.
template <int C> PB_HD void make_move(Board &b, u32 &state, uint16_t mv)
{
    u32 from = mv & 63, to = (mv >> 6) & 63, flags = mv >> 12;
    u64 src = 1ULL << from, dst = 1ULL << to;
    u32 piece = (u32)((b.bb[1] >> from) & 1) | (u32)(((b.bb[2] >> from) & 1) << 1) |
                (u32)(((b.bb[3] >> from) & 1) << 2);
    if (flags & MF_PROMO) piece = (flags & 3) + KNIGHT;
    u64 clr = ~(src | dst);
    b.bb[0] &= clr;
    b.bb[1] &= clr;
    b.bb[2] &= clr;
    b.bb[3] &= clr;
    if (C == BLACK) b.bb[0] |= dst;
    b.bb[1] |= (u64)(piece & 1) << to;
    b.bb[2] |= (u64)((piece >> 1) & 1) << to;
    b.bb[3] |= (u64)((piece >> 2) & 1) << to;
    if (flags == MF_EP) {
        u64 v = C == WHITE ? (dst >> 8) : (dst << 8);
        b.bb[0] &= ~v;
        b.bb[1] &= ~v;
    } else if (flags == MF_KING_CASTLE) {
        constexpr u64 R = C == WHITE ? 0xA0ULL : 0xA000000000000000ULL;  // h-file rook to f-file
        b.bb[3] ^= R;
        if (C == BLACK) b.bb[0] ^= R;
    } else if (flags == MF_QUEEN_CASTLE) {
        constexpr u64 R = C == WHITE ? 0x09ULL : 0x0900000000000000ULL;  // a-file rook to d-file
        b.bb[3] ^= R;
        if (C == BLACK) b.bb[0] ^= R;
    }
    u32 st = state & 15;
    u64 touched = src | dst;
    if (touched & 0x9100000000000091ULL) {
        u32 t = (u32)touched & 0x91, h = (u32)(touched >> 56) & 0x91;
        // bit 7 = h-file rook, bit 0 = a-file rook, bit 4 = king
        u32 wclr = ((t >> 7) | (t >> 4)) & 1;
        wclr |= (((t >> 0) | (t >> 4)) & 1) << 1;
        u32 bclr = ((h >> 7) | (h >> 4)) & 1;
        bclr |= (((h >> 0) | (h >> 4)) & 1) << 1;
        st &= ~(wclr | (bclr << 2));
    }
    if (flags == MF_DOUBLE_PUSH) st |= ((from & 7) + 1) << 4;
    state = st;
}

}  // namespace pb
