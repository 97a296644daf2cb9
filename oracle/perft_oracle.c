/*
 * perft_oracle.c - CPU restatement of the reference perft path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker; see perft_oracle.h).  Nothing in the
 * product library links or calls this file.
 *
 * Each function names the reference lines it restates.  The control flow
 * (pins first, then attacked squares, a separate in-check branch, pawns in
 * bulk for counting, pinned sliders restricted to the king line, the
 * rank-only discovered-check test for en passant) follows the reference so
 * that counts agree on every input the reference accepts, including its
 * conventions for en passant and castling rights.
 */
#include "perft_oracle.h"

#include <stdlib.h>
#include <string.h>

typedef uint64_t u64;

enum { EMPTY = 0, PAWN = 1, KNIGHT = 2, BISHOP = 3, ROOK = 4, QUEEN = 5, KING = 6 };
enum { WHITE = 0, BLACK = 1 };

/* move flags, chess.h:120-144 */
enum {
    F_QUIET = 0, F_DOUBLE = 1, F_KCASTLE = 2, F_QCASTLE = 3, F_CAPTURE = 4,
    F_EP = 5, F_PROMO = 8
};

#define BIT(s) (1ULL << (s))
#define RANK1 0x00000000000000FFULL
#define RANK3 0x0000000000FF0000ULL
#define RANK8 0xFF00000000000000ULL
#define FILEA 0x0101010101010101ULL
#define FILEH 0x8080808080808080ULL

static u64 knight_att[64], king_att[64];
static u64 rays[8][64];              /* N, E, NE, NW (increasing), S, W, SW, SE: d and d+4 are opposite */
static u64 between_tab[64][64], line_tab[64][64];
static u64 rook_empty[64], bishop_empty[64];
static int tables_ready;

static inline int lsb(u64 x) { return __builtin_ctzll(x); }
static inline int msb(u64 x) { return 63 - __builtin_clzll(x); }
static inline int popc(u64 x) { return __builtin_popcountll(x); }

/* shifts, MoveGeneratorBitboard.h:320-350 */
static inline u64 north(u64 x) { return x << 8; }
static inline u64 south(u64 x) { return x >> 8; }
static inline u64 east(u64 x) { return (x << 1) & ~FILEA; }
static inline u64 west(u64 x) { return (x >> 1) & ~FILEH; }
static inline u64 ne(u64 x) { return (x << 9) & ~FILEA; }
static inline u64 nw(u64 x) { return (x << 7) & ~FILEH; }
static inline u64 se(u64 x) { return (x >> 7) & ~FILEA; }
static inline u64 sw(u64 x) { return (x >> 9) & ~FILEH; }

static const int DFILE[8] = {0, 1, 1, -1, 0, -1, -1, 1};
static const int DRANK[8] = {1, 0, 1, 1, -1, 0, -1, -1};

/* Empty-board tables, perft_kernels.cu:995-1025. */
static void init_tables(void)
{
    if (tables_ready) return;
    for (int sq = 0; sq < 64; sq++) {
        int f = sq & 7, r = sq >> 3;
        u64 kn = 0, kg = 0;
        static const int KN[8][2] = {{1,2},{2,1},{2,-1},{1,-2},{-1,-2},{-2,-1},{-2,1},{-1,2}};
        for (int i = 0; i < 8; i++) {
            int nf = f + KN[i][0], nr = r + KN[i][1];
            if (nf >= 0 && nf < 8 && nr >= 0 && nr < 8) kn |= BIT(nr * 8 + nf);
        }
        for (int df = -1; df <= 1; df++)
            for (int dr = -1; dr <= 1; dr++) {
                if (!df && !dr) continue;
                int nf = f + df, nr = r + dr;
                if (nf >= 0 && nf < 8 && nr >= 0 && nr < 8) kg |= BIT(nr * 8 + nf);
            }
        knight_att[sq] = kn;
        king_att[sq] = kg;
        for (int d = 0; d < 8; d++) {
            u64 m = 0;
            int nf = f + DFILE[d], nr = r + DRANK[d];
            while (nf >= 0 && nf < 8 && nr >= 0 && nr < 8) {
                m |= BIT(nr * 8 + nf);
                nf += DFILE[d];
                nr += DRANK[d];
            }
            rays[d][sq] = m;
        }
    }
    for (int sq = 0; sq < 64; sq++) {
        rook_empty[sq] = rays[0][sq] | rays[1][sq] | rays[4][sq] | rays[5][sq];
        bishop_empty[sq] = rays[2][sq] | rays[3][sq] | rays[6][sq] | rays[7][sq];
    }
    for (int a = 0; a < 64; a++)
        for (int b = 0; b < 64; b++) {
            between_tab[a][b] = 0;
            line_tab[a][b] = 0;
            for (int d = 0; d < 8; d++) {
                if (rays[d][a] & BIT(b)) {
                    int opp = (d < 4) ? d + 4 : d - 4;
                    between_tab[a][b] = rays[d][a] & rays[opp][b];
                    line_tab[a][b] = rays[d][a] | rays[opp][a] | BIT(a);
                }
            }
        }
    tables_ready = 1;
}

/* Slider attack set by ray walk (the reference uses fancy magics,
 * MoveGeneratorBitboard.h:589-648; the attack set is the same). */
static inline u64 ray_att(int d, int sq, u64 occ)
{
    u64 r = rays[d][sq];
    u64 blk = r & occ;
    if (!blk) return r;
    int b = (d < 4) ? lsb(blk) : msb(blk);
    return r ^ rays[d][b];
}
static inline u64 rook_att(int sq, u64 occ)
{
    return ray_att(0, sq, occ) | ray_att(1, sq, occ) | ray_att(4, sq, occ) | ray_att(5, sq, occ);
}
static inline u64 bishop_att(int sq, u64 occ)
{
    return ray_att(2, sq, occ) | ray_att(3, sq, occ) | ray_att(6, sq, occ) | ray_att(7, sq, occ);
}

/* Derived piece sets, DERIVE_PIECE_BITBOARDS (MoveGeneratorBitboard.h:966-974). */
typedef struct {
    u64 all, mine, them, pawns, knights, bq, rq, kings;
} sets;

static inline void derive(const or_pos *p, sets *s)
{
    s->all = p->bb[1] | p->bb[2] | p->bb[3];
    u64 black = p->bb[0];
    u64 white = s->all & ~black;
    s->pawns = p->bb[1] & ~p->bb[2] & ~p->bb[3];
    s->knights = p->bb[2] & ~p->bb[1] & ~p->bb[3];
    s->bq = p->bb[1] & (p->bb[2] ^ p->bb[3]);
    s->rq = p->bb[3] & ~p->bb[2];
    s->kings = p->bb[2] & p->bb[3] & ~p->bb[1];
    s->mine = p->color == WHITE ? white : black;
    s->them = p->color == WHITE ? black : white;
}

/* findPinnedPieces, MoveGeneratorBitboard.h:803-831 */
static u64 find_pinned(int ksq, u64 eb, u64 er, u64 all)
{
    u64 att = (bishop_empty[ksq] & eb) | (rook_empty[ksq] & er);
    u64 pinned = 0;
    while (att) {
        int a = lsb(att);
        u64 inb = between_tab[a][ksq] & all;
        if (inb && !(inb & (inb - 1))) pinned |= inb;
        att &= att - 1;
    }
    return pinned;
}

/* findAttackedSquares, MoveGeneratorBitboard.h:835-875: slider attacks see
 * through the side-to-move's king. */
static u64 attacked_squares(const sets *s, int color, u64 my_king)
{
    u64 e = s->them;
    u64 ep = s->pawns & e;
    u64 a = (color == WHITE) ? (se(ep) | sw(ep)) : (ne(ep) | nw(ep));
    u64 en = s->knights & e;
    while (en) { a |= knight_att[lsb(en)]; en &= en - 1; }
    u64 occ = s->all & ~my_king;
    u64 b = s->bq & e;
    while (b) { a |= bishop_att(lsb(b), occ); b &= b - 1; }
    u64 r = s->rq & e;
    while (r) { a |= rook_att(lsb(r), occ); r &= r - 1; }
    u64 k = s->kings & e;
    if (k) a |= king_att[lsb(k)];
    return a;
}

static inline u64 fwd(int c, u64 x) { return c == WHITE ? north(x) : south(x); }
static inline u64 cap_w(int c, u64 x) { return c == WHITE ? nw(x) : sw(x); }
static inline u64 cap_e(int c, u64 x) { return c == WHITE ? ne(x) : se(x); }

/* EP target square from the state byte (getEpTarget, MoveGeneratorBitboard.h:183-193). */
static inline u64 ep_target(int c, uint8_t state)
{
    int f = state >> 4;
    if (!f) return 0;
    return c == BLACK ? (BIT(f - 1) << 16) : (BIT(f - 1) << 40);
}

/* ------------------------------------------------------------------ */
/* countMovesOutOfCheck, MoveGeneratorBitboard.h:1564-1694             */
static uint32_t count_evasions(const or_pos *p, const sets *s, u64 pinned, u64 threat, int ksq, int strict)
{
    int c = p->color;
    u64 king = BIT(ksq);
    uint32_t n = 0;
    u64 ep_ = s->pawns & s->them;
    u64 attackers = (c == WHITE ? (ne(king) | nw(king)) : (se(king) | sw(king))) & ep_;
    attackers |= knight_att[ksq] & s->knights & s->them;
    attackers |= bishop_att(ksq, s->all) & s->bq & s->them;
    attackers |= rook_att(ksq, s->all) & s->rq & s->them;

    n += popc(king_att[ksq] & ~(threat | s->mine));
    if (attackers & (attackers - 1)) return n;

    u64 safe = attackers | between_tab[ksq][lsb(attackers)];
    u64 mine = s->mine & ~pinned;
    u64 empty = ~s->all;
    u64 pawns = s->pawns & mine;
    u64 dbl_rank = RANK3 << (c * 24);

    u64 push = fwd(c, pawns) & empty;
    u64 d = push & safe;
    u64 promo = d & (RANK1 | RANK8);
    n += popc(d ^ promo) + 4 * popc(promo);
    n += popc(fwd(c, push & dbl_rank) & empty & safe);
    d = cap_w(c, pawns) & s->them & safe;
    promo = d & (RANK1 | RANK8);
    n += popc(d ^ promo) + 4 * popc(promo);
    d = cap_e(c, pawns) & s->them & safe;
    promo = d & (RANK1 | RANK8);
    n += popc(d ^ promo) + 4 * popc(promo);

    u64 ept = ep_target(c, p->state);
    if (ept) {
        u64 victim = c == WHITE ? south(ept) : north(ept);
        /* The reference ORs the two capture directions (:1639-1650), so two
         * pawns that can both take en passant count once; strict mode counts
         * both. */
        if (victim == attackers) {
            u64 w = cap_w(c, pawns) & ept, e = cap_e(c, pawns) & ept;
            n += strict ? popc(w) + popc(e) : popc(w | e);
        }
    }
    u64 kn = s->knights & mine;
    while (kn) { n += popc(knight_att[lsb(kn)] & safe); kn &= kn - 1; }
    u64 b = s->bq & mine;
    while (b) { n += popc(bishop_att(lsb(b), s->all) & safe); b &= b - 1; }
    u64 r = s->rq & mine;
    while (r) { n += popc(rook_att(lsb(r), s->all) & safe); r &= r - 1; }
    return n;
}

/* countMoves, MoveGeneratorBitboard.h:1700-1943 */
static uint32_t count_moves(const or_pos *p, int strict)
{
    init_tables();
    sets s;
    derive(p, &s);
    int c = p->color;
    u64 eb = s.bq & s.them, er = s.rq & s.them;
    u64 my_king = s.kings & s.mine;
    if (!my_king) return 0;
    int ksq = lsb(my_king);
    u64 empty = ~s.all;
    u64 pinned = find_pinned(ksq, eb, er, s.all);
    u64 threat = attacked_squares(&s, c, my_king);
    if (threat & my_king) return count_evasions(p, &s, pinned, threat, ksq, strict);

    uint32_t n = 0;
    u64 my_pawns = s.pawns & s.mine;

    /* en passant (:1732-1770) */
    u64 ept = ep_target(c, p->state);
    if (ept) {
        u64 victim = c == WHITE ? south(ept) : north(ept);
        u64 src = (east(victim) | west(victim)) & my_pawns;
        while (src) {
            int psq = lsb(src);
            u64 pawn = BIT(psq);
            if (pawn & pinned) {
                if (ept & line_tab[psq][ksq]) n++;
            } else {
                u64 occ = s.all ^ victim ^ pawn;
                u64 rank = RANK1 << ((ksq >> 3) * 8);
                if (!(rook_att(ksq, occ) & er & rank)) n++;
            }
            src &= src - 1;
        }
    }

    u64 dbl_rank = RANK3 << (c * 24);
    /* pinned pawns (:1775-1816) */
    u64 pp = my_pawns & pinned;
    while (pp) {
        int psq = lsb(pp);
        u64 pawn = BIT(psq);
        u64 line = line_tab[psq][ksq];
        u64 d = fwd(c, pawn) & line & empty;
        if (d) {
            n++;
            if (fwd(c, d & dbl_rank) & empty) n++;
        }
        d = (cap_w(c, pawn) | cap_e(c, pawn)) & line;
        if (d & s.them) n += (d & (RANK1 | RANK8)) ? 4 : 1;
        pp &= pp - 1;
    }
    /* free pawns in bulk (:1818-1846) */
    u64 fp = my_pawns & ~pinned;
    u64 d = fwd(c, fp) & empty;
    u64 promos = d & (RANK1 | RANK8);
    n += popc(d ^ promos);
    n += popc(fwd(c, d & dbl_rank) & empty);
    u64 cw = cap_w(c, fp) & s.them, ce = cap_e(c, fp) & s.them;
    u64 pw = cw & (RANK1 | RANK8), pe = ce & (RANK1 | RANK8);
    n += popc(cw ^ pw) + popc(ce ^ pe);
    /* The reference ORs the three promotion sets before counting
     * (:1823-1846).  A west and an east capture from two different pawns can
     * land on the same square, so the OR undercounts by 4 per shared square;
     * strict mode counts each set on its own. */
    if (strict) n += 4 * (popc(promos) + popc(pw) + popc(pe));
    else n += 4 * popc(promos | pw | pe);

    /* castling (:1848-1867) */
    int castle = c == WHITE ? (p->state & 3) : ((p->state >> 2) & 3);
    if (c == WHITE) {
        if ((castle & 1) && !(0x60ULL & s.all) && !(0x60ULL & threat)) n++;
        if ((castle & 2) && !(0x0EULL & s.all) && !(0x0CULL & threat)) n++;
    } else {
        if ((castle & 1) && !(0x6000000000000000ULL & s.all) && !(0x6000000000000000ULL & threat)) n++;
        if ((castle & 2) && !(0x0E00000000000000ULL & s.all) && !(0x0C00000000000000ULL & threat)) n++;
    }
    /* king (:1870-1873) */
    n += popc(king_att[ksq] & ~(threat | s.mine));
    /* knights (:1876-1884) */
    u64 kn = s.knights & s.mine & ~pinned;
    while (kn) { n += popc(knight_att[lsb(kn)] & ~s.mine); kn &= kn - 1; }
    /* bishops/queens (:1887-1912) */
    u64 b = s.bq & s.mine;
    while (b) {
        int sq = lsb(b);
        u64 m = bishop_att(sq, s.all) & ~s.mine;
        if (BIT(sq) & pinned) m &= line_tab[sq][ksq];
        n += popc(m);
        b &= b - 1;
    }
    /* rooks/queens (:1914-1940) */
    u64 r = s.rq & s.mine;
    while (r) {
        int sq = lsb(r);
        u64 m = rook_att(sq, s.all) & ~s.mine;
        if (BIT(sq) & pinned) m &= line_tab[sq][ksq];
        n += popc(m);
        r &= r - 1;
    }
    return n;
}

uint32_t or_count_moves(const or_pos *p) { return count_moves(p, 0); }
uint32_t or_count_moves_strict(const or_pos *p) { return count_moves(p, 1); }

/* ------------------------------------------------------------------ */
/* move emission helpers (chess.h:94-118, MoveGeneratorBitboard.h:887-925) */
static inline uint16_t mk(int from, int to, int flags)
{
    return (uint16_t)(((flags & 0xF) << 12) | ((to & 0x3F) << 6) | (from & 0x3F));
}
static inline int emit_pawn(uint16_t *m, int n, int from, int to, int flags)
{
    if (BIT(to) & (RANK1 | RANK8)) {
        m[n++] = mk(from, to, flags | 8);
        m[n++] = mk(from, to, flags | 9);
        m[n++] = mk(from, to, flags | 11);
        m[n++] = mk(from, to, flags | 10);
    } else {
        m[n++] = mk(from, to, flags);
    }
    return n;
}
static inline int emit_set(uint16_t *m, int n, int from, u64 dsts, u64 them)
{
    while (dsts) {
        int to = lsb(dsts);
        m[n++] = mk(from, to, (BIT(to) & them) ? F_CAPTURE : F_QUIET);
        dsts &= dsts - 1;
    }
    return n;
}

/* generateMovesOutOfCheck, MoveGeneratorBitboard.h:978-1154 */
static int gen_evasions(const or_pos *p, const sets *s, u64 pinned, u64 threat, int ksq, uint16_t *m)
{
    int c = p->color;
    int n = 0;
    u64 king = BIT(ksq);
    u64 ep_ = s->pawns & s->them;
    u64 attackers = (c == WHITE ? (ne(king) | nw(king)) : (se(king) | sw(king))) & ep_;
    attackers |= knight_att[ksq] & s->knights & s->them;
    attackers |= bishop_att(ksq, s->all) & s->bq & s->them;
    attackers |= rook_att(ksq, s->all) & s->rq & s->them;

    n = emit_set(m, n, ksq, king_att[ksq] & ~(threat | s->mine), s->them);
    if (attackers & (attackers - 1)) return n;

    u64 safe = attackers | between_tab[ksq][lsb(attackers)];
    u64 mine = s->mine & ~pinned;
    u64 empty = ~s->all;
    u64 dbl_rank = RANK3 << (c * 24);
    u64 ept = ep_target(c, p->state);
    if (ept) {
        u64 victim = c == WHITE ? south(ept) : north(ept);
        if (victim != attackers) ept = 0;
    }
    u64 pawns = s->pawns & mine;
    while (pawns) {
        int psq = lsb(pawns);
        u64 pawn = BIT(psq);
        u64 d = fwd(c, pawn) & empty;
        if (d) {
            if (d & safe) {
                n = emit_pawn(m, n, psq, lsb(d), F_QUIET);
            } else {
                d = fwd(c, d & dbl_rank) & safe & empty;
                if (d) m[n++] = mk(psq, lsb(d), F_DOUBLE);
            }
        }
        u64 caps = (cap_w(c, pawn) | cap_e(c, pawn));
        d = caps & s->them & safe;
        if (d) n = emit_pawn(m, n, psq, lsb(d), F_CAPTURE);
        d = caps & ept;
        if (d) m[n++] = mk(psq, lsb(d), F_EP);
        pawns &= pawns - 1;
    }
    u64 kn = s->knights & mine;
    while (kn) { int sq = lsb(kn); n = emit_set(m, n, sq, knight_att[sq] & safe, s->them); kn &= kn - 1; }
    u64 b = s->bq & mine;
    while (b) { int sq = lsb(b); n = emit_set(m, n, sq, bishop_att(sq, s->all) & safe, s->them); b &= b - 1; }
    u64 r = s->rq & mine;
    while (r) { int sq = lsb(r); n = emit_set(m, n, sq, rook_att(sq, s->all) & safe, s->them); r &= r - 1; }
    return n;
}

/* generateMovesToSink, MoveGeneratorBitboard.h:1160-1554 (CPU flags: captures
 * flagged, double pushes always flagged). */
uint32_t or_generate_moves(const or_pos *p, uint16_t *m)
{
    init_tables();
    sets s;
    derive(p, &s);
    int c = p->color;
    u64 eb = s.bq & s.them, er = s.rq & s.them;
    u64 my_king = s.kings & s.mine;
    if (!my_king) return 0;
    int ksq = lsb(my_king);
    u64 empty = ~s.all;
    u64 pinned = find_pinned(ksq, eb, er, s.all);
    u64 threat = attacked_squares(&s, c, my_king);
    if (threat & my_king) return (uint32_t)gen_evasions(p, &s, pinned, threat, ksq, m);

    int n = 0;
    u64 my_pawns = s.pawns & s.mine;
    u64 dbl_rank = RANK3 << (c * 24);

    u64 pp = my_pawns & pinned;
    while (pp) {
        int psq = lsb(pp);
        u64 pawn = BIT(psq);
        u64 line = line_tab[psq][ksq];
        u64 d = (cap_w(c, pawn) | cap_e(c, pawn)) & line;
        if (d & s.them) n = emit_pawn(m, n, psq, lsb(d & s.them), F_CAPTURE);
        d = fwd(c, pawn) & line & empty;
        if (d) {
            m[n++] = mk(psq, lsb(d), F_QUIET);
            d = fwd(c, d & dbl_rank) & empty;
            if (d) m[n++] = mk(psq, lsb(d), F_DOUBLE);
        }
        pp &= pp - 1;
    }
    u64 fp = my_pawns & ~pinned;
    while (fp) {
        int psq = lsb(fp);
        u64 pawn = BIT(psq);
        u64 d = cap_w(c, pawn) & s.them;
        if (d) n = emit_pawn(m, n, psq, lsb(d), F_CAPTURE);
        d = cap_e(c, pawn) & s.them;
        if (d) n = emit_pawn(m, n, psq, lsb(d), F_CAPTURE);
        d = fwd(c, pawn) & empty;
        if (d) {
            n = emit_pawn(m, n, psq, lsb(d), F_QUIET);
            d = fwd(c, d & dbl_rank) & empty;
            if (d) m[n++] = mk(psq, lsb(d), F_DOUBLE);
        }
        fp &= fp - 1;
    }
    u64 ept = ep_target(c, p->state);
    if (ept) {
        u64 victim = c == WHITE ? south(ept) : north(ept);
        u64 src = (east(victim) | west(victim)) & my_pawns;
        while (src) {
            int psq = lsb(src);
            u64 pawn = BIT(psq);
            if (pawn & pinned) {
                if (ept & line_tab[psq][ksq]) m[n++] = mk(psq, lsb(ept), F_EP);
            } else {
                u64 occ = s.all ^ victim ^ pawn;
                u64 rank = RANK1 << ((ksq >> 3) * 8);
                if (!(rook_att(ksq, occ) & er & rank)) m[n++] = mk(psq, lsb(ept), F_EP);
            }
            src &= src - 1;
        }
    }
    n = emit_set(m, n, ksq, king_att[ksq] & ~(threat | s.mine), s.them);
    u64 kn = s.knights & s.mine & ~pinned;
    while (kn) { int sq = lsb(kn); n = emit_set(m, n, sq, knight_att[sq] & ~s.mine, s.them); kn &= kn - 1; }
    u64 b = s.bq & s.mine;
    while (b) {
        int sq = lsb(b);
        u64 d = bishop_att(sq, s.all) & ~s.mine;
        if (BIT(sq) & pinned) d &= line_tab[sq][ksq];
        n = emit_set(m, n, sq, d, s.them);
        b &= b - 1;
    }
    u64 r = s.rq & s.mine;
    while (r) {
        int sq = lsb(r);
        u64 d = rook_att(sq, s.all) & ~s.mine;
        if (BIT(sq) & pinned) d &= line_tab[sq][ksq];
        n = emit_set(m, n, sq, d, s.them);
        r &= r - 1;
    }
    int castle = c == WHITE ? (p->state & 3) : ((p->state >> 2) & 3);
    if (c == WHITE) {
        if ((castle & 1) && !(0x60ULL & s.all) && !(0x60ULL & threat)) m[n++] = mk(4, 6, F_KCASTLE);
        if ((castle & 2) && !(0x0EULL & s.all) && !(0x0CULL & threat)) m[n++] = mk(4, 2, F_QCASTLE);
    } else {
        if ((castle & 1) && !(0x6000000000000000ULL & s.all) && !(0x6000000000000000ULL & threat))
            m[n++] = mk(60, 62, F_KCASTLE);
        if ((castle & 2) && !(0x0E00000000000000ULL & s.all) && !(0x0C00000000000000ULL & threat))
            m[n++] = mk(60, 58, F_QCASTLE);
    }
    return (uint32_t)n;
}

/* makeMove, MoveGeneratorBitboard.h:1945-2066 (CPU branch for the state). */
void or_make_move(or_pos *p, uint16_t mv)
{
    int from = mv & 0x3F, to = (mv >> 6) & 0x3F, flags = mv >> 12;
    int c = p->color;
    u64 src = BIT(from), dst = BIT(to);
    int piece = ((p->bb[1] & src) ? 1 : 0) | ((p->bb[2] & src) ? 2 : 0) | ((p->bb[3] & src) ? 4 : 0);
    int moved = piece;
    if (flags & F_PROMO) piece = (flags & 3) + KNIGHT;
    u64 clr = ~(src | dst);
    for (int i = 0; i < 4; i++) p->bb[i] &= clr;
    if (c == BLACK) p->bb[0] |= dst;
    if (piece & 1) p->bb[1] |= dst;
    if (piece & 2) p->bb[2] |= dst;
    if (piece & 4) p->bb[3] |= dst;
    if (flags == F_EP) {
        u64 v = c == WHITE ? south(dst) : north(dst);
        p->bb[0] &= ~v;
        p->bb[1] &= ~v;
    }
    if (flags == F_KCASTLE) {
        int rf = c == WHITE ? 7 : 63, rt = c == WHITE ? 5 : 61;
        p->bb[3] = (p->bb[3] ^ BIT(rf)) | BIT(rt);
        if (c == BLACK) p->bb[0] = (p->bb[0] ^ BIT(rf)) | BIT(rt);
    } else if (flags == F_QCASTLE) {
        int rf = c == WHITE ? 0 : 56, rt = c == WHITE ? 3 : 59;
        p->bb[3] = (p->bb[3] ^ BIT(rf)) | BIT(rt);
        if (c == BLACK) p->bb[0] = (p->bb[0] ^ BIT(rf)) | BIT(rt);
    }
    /* state update (:2041-2066) */
    int wc = p->state & 3, bc = (p->state >> 2) & 3, ep = 0;
    if (c == WHITE) {
        if (dst & BIT(63)) bc &= ~1;
        if (dst & BIT(56)) bc &= ~2;
        if (moved == KING) wc = 0;
        if (moved == ROOK) { if (src & BIT(7)) wc &= ~1; if (src & BIT(0)) wc &= ~2; }
    } else {
        if (dst & BIT(7)) wc &= ~1;
        if (dst & BIT(0)) wc &= ~2;
        if (moved == KING) bc = 0;
        if (moved == ROOK) { if (src & BIT(63)) bc &= ~1; if (src & BIT(56)) bc &= ~2; }
    }
    if (flags == F_DOUBLE) ep = (from & 7) + 1;
    p->state = (uint8_t)(wc | (bc << 2) | (ep << 4));
    p->color ^= 1;
}

/* perft_cpu<chance>, launcher.cu:762-805; depth 0 is 1 (launcher.cu:809-810).
 * The last ply is counted with countMoves, so the reference's counting
 * conventions apply there; strict mode counts the last ply exactly. */
static uint64_t perft_impl(const or_pos *p, int depth, int strict)
{
    if (depth <= 0) return 1;
    if (depth == 1) return count_moves(p, strict);
    uint16_t m[256];
    uint32_t n = or_generate_moves(p, m);
    uint64_t total = 0;
    for (uint32_t i = 0; i < n; i++) {
        or_pos c = *p;
        or_make_move(&c, m[i]);
        total += perft_impl(&c, depth - 1, strict);
    }
    return total;
}

uint64_t or_perft(const or_pos *p, int depth) { init_tables(); return perft_impl(p, depth, 0); }
uint64_t or_perft_strict(const or_pos *p, int depth) { init_tables(); return perft_impl(p, depth, 1); }

void or_perft_batch(const or_pos *ps, const int *depths, int n, uint64_t *out)
{
    for (int i = 0; i < n; i++) out[i] = or_perft(&ps[i], depths[i]);
}

int or_perft_divide(const or_pos *p, int depth, uint16_t *moves, uint64_t *counts)
{
    init_tables();
    uint32_t n = or_generate_moves(p, moves);
    for (uint32_t i = 0; i < n; i++) {
        or_pos c = *p;
        or_make_move(&c, moves[i]);
        counts[i] = or_perft(&c, depth - 1);
    }
    return (int)n;
}

/* ------------------------------------------------------------------ */
/* FEN parsing, util.cpp:7-95 */
int or_parse_fen(const char *fen, or_pos *out)
{
    init_tables();
    memset(out, 0, sizeof(*out));
    int i, row = 0, col = 0;
    for (i = 0; fen[i]; i++) {
        char ch = fen[i];
        if (ch == '/' || ch == '\\') { row++; col = 0; }
        else if (ch >= '1' && ch <= '8') col += ch - '0';
        else {
            int piece = 0, black = 0;
            switch (ch) {
            case 'p': piece = PAWN; black = 1; break;
            case 'n': piece = KNIGHT; black = 1; break;
            case 'b': piece = BISHOP; black = 1; break;
            case 'r': piece = ROOK; black = 1; break;
            case 'q': piece = QUEEN; black = 1; break;
            case 'k': piece = KING; black = 1; break;
            case 'P': piece = PAWN; break;
            case 'N': piece = KNIGHT; break;
            case 'B': piece = BISHOP; break;
            case 'R': piece = ROOK; break;
            case 'Q': piece = QUEEN; break;
            case 'K': piece = KING; break;
            default: break;
            }
            if (piece) {
                if (row > 7 || col > 7) return -1;
                u64 bit = BIT((7 - row) * 8 + col);
                if (black) out->bb[0] |= bit;
                if (piece & 1) out->bb[1] |= bit;
                if (piece & 2) out->bb[2] |= bit;
                if (piece & 4) out->bb[3] |= bit;
                col++;
            }
        }
        if (row >= 7 && col == 8) break;
    }
    if (!fen[i]) return -1;
    i++;
    while (fen[i] == ' ') i++;
    out->color = (fen[i] == 'b' || fen[i] == 'B') ? BLACK : WHITE;
    if (fen[i]) i++;
    while (fen[i] == ' ') i++;
    int wc = 0, bc = 0;
    while (fen[i] && fen[i] != ' ') {
        switch (fen[i]) {
        case 'K': wc |= 1; break;
        case 'Q': wc |= 2; break;
        case 'k': bc |= 1; break;
        case 'q': bc |= 2; break;
        }
        i++;
    }
    while (fen[i] == ' ') i++;
    int ep = 0;
    if (fen[i] >= 'a' && fen[i] <= 'h') ep = fen[i] - 'a' + 1;
    out->state = (uint8_t)(wc | (bc << 2) | (ep << 4));
    return 0;
}

static int piece_at(const or_pos *p, int sq)
{
    u64 b = BIT(sq);
    return ((p->bb[1] & b) ? 1 : 0) | ((p->bb[2] & b) ? 2 : 0) | ((p->bb[3] & b) ? 4 : 0);
}

void or_to_fen(const or_pos *p, char *buf)
{
    static const char W[] = " PNBRQK", B[] = " pnbrqk";
    int k = 0;
    for (int r = 7; r >= 0; r--) {
        int run = 0;
        for (int f = 0; f < 8; f++) {
            int sq = r * 8 + f, pc = piece_at(p, sq);
            if (!pc) { run++; continue; }
            if (run) { buf[k++] = (char)('0' + run); run = 0; }
            buf[k++] = (p->bb[0] & BIT(sq)) ? B[pc] : W[pc];
        }
        if (run) buf[k++] = (char)('0' + run);
        if (r) buf[k++] = '/';
    }
    buf[k++] = ' ';
    buf[k++] = p->color ? 'b' : 'w';
    buf[k++] = ' ';
    int any = 0;
    if (p->state & 1) { buf[k++] = 'K'; any = 1; }
    if (p->state & 2) { buf[k++] = 'Q'; any = 1; }
    if (p->state & 4) { buf[k++] = 'k'; any = 1; }
    if (p->state & 8) { buf[k++] = 'q'; any = 1; }
    if (!any) buf[k++] = '-';
    buf[k++] = ' ';
    int ep = p->state >> 4;
    if (ep) {
        buf[k++] = (char)('a' + ep - 1);
        buf[k++] = p->color == WHITE ? '6' : '3';
    } else {
        buf[k++] = '-';
    }
    memcpy(buf + k, " 0 1", 5);
}

/* ------------------------------------------------------------------ */
/* Workload generator: splitmix64 (Steele, Lea and Flood, 2014) and uniform
 * choice among the legal moves sorted by their UCI text. */
uint64_t or_splitmix64(uint64_t *state)
{
    uint64_t z = (*state += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

void or_move_uci(uint16_t mv, char *buf)
{
    int from = mv & 0x3F, to = (mv >> 6) & 0x3F, flags = mv >> 12;
    buf[0] = (char)('a' + (from & 7));
    buf[1] = (char)('1' + (from >> 3));
    buf[2] = (char)('a' + (to & 7));
    buf[3] = (char)('1' + (to >> 3));
    int k = 4;
    if (flags & F_PROMO) buf[k++] = "nbrq"[flags & 3];
    buf[k] = 0;
}

static int cmp_uci(const void *a, const void *b)
{
    char x[8], y[8];
    or_move_uci(*(const uint16_t *)a, x);
    or_move_uci(*(const uint16_t *)b, y);
    return strcmp(x, y);
}

int or_random_playout(uint64_t *rng, int plies, or_pos *out)
{
    or_parse_fen("rnbqkbnr/pppppppp/8/8/8/8/PPPPPPPP/RNBQKBNR w KQkq - 0 1", out);
    int played = 0;
    for (int i = 0; i < plies; i++) {
        uint16_t m[256];
        uint32_t n = or_generate_moves(out, m);
        if (!n) break;
        qsort(m, n, sizeof(uint16_t), cmp_uci);
        uint64_t r = or_splitmix64(rng);
        uint32_t pick = (uint32_t)(((unsigned __int128)r * n) >> 64);
        or_make_move(out, m[pick]);
        played++;
    }
    return played;
}
