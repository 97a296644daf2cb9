// pb_util.cuh - host utilities: FEN parsing/writing (util.cpp:7-95), UCI move
// text and the splitmix64 generator used by the workload generator.
#pragma once
#include <string.h>

#include <string>

#include "../../include/perft_b200.h"
#include "pb_core.cuh"

namespace pb {

// splitmix64 (Steele, Lea and Flood 2014): state += golden gamma, then two
// xor-shift-multiply rounds.
inline u64 splitmix64(u64 *state)
{
    u64 z = (*state += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

inline std::string move_uci(uint16_t m)
{
    char b[6];
    int from = move_from(m), to = move_to(m), fl = move_flags(m);
    b[0] = (char)('a' + (from & 7));
    b[1] = (char)('1' + (from >> 3));
    b[2] = (char)('a' + (to & 7));
    b[3] = (char)('1' + (to >> 3));
    int k = 4;
    if (fl & MF_PROMO) b[k++] = "nbrq"[fl & 3];
    return std::string(b, k);
}

inline int piece_on(const Board &b, int sq)
{
    return (int)(((b.bb[1] >> sq) & 1) | (((b.bb[2] >> sq) & 1) << 1) | (((b.bb[3] >> sq) & 1) << 2));
}

// Parses the placement, side, castling and en-passant fields the way the
// reference does (util.cpp:7-95: halfmove/fullmove ignored), then checks the
// position could arise in a legal game.  Inconsistent castle rights and
// en-passant squares are dropped; impossible positions are rejected.
inline bool parse_fen(const char *fen, pb_pos *out)
{
    memset(out, 0, sizeof(*out));
    Board b{};
    int i = 0, row = 0, col = 0;
    for (; fen[i]; i++) {
        char ch = fen[i];
        if (ch == ' ' && (row > 0 || col > 0)) break;
        if (ch == '/' || ch == '\\') {
            row++;
            col = 0;
            continue;
        }
        if (ch >= '1' && ch <= '8') {
            col += ch - '0';
            continue;
        }
        const char *pcs = "PNBRQKpnbrqk";
        const char *q = ch ? strchr(pcs, ch) : nullptr;
        if (!q) continue;
        int idx = (int)(q - pcs);
        int piece = idx % 6 + 1;
        bool black = idx >= 6;
        if (row > 7 || col > 7) return false;
        u64 bit = 1ULL << ((7 - row) * 8 + col);
        if (black) b.bb[0] |= bit;
        if (piece & 1) b.bb[1] |= bit;
        if (piece & 2) b.bb[2] |= bit;
        if (piece & 4) b.bb[3] |= bit;
        col++;
    }
    if (row != 7) return false;
    while (fen[i] == ' ') i++;
    int color = (fen[i] == 'b' || fen[i] == 'B') ? BLACK : WHITE;
    if (fen[i]) i++;
    while (fen[i] == ' ') i++;
    u32 castle = 0;
    while (fen[i] && fen[i] != ' ') {
        switch (fen[i]) {
        case 'K': castle |= 1; break;
        case 'Q': castle |= 2; break;
        case 'k': castle |= 4; break;
        case 'q': castle |= 8; break;
        }
        i++;
    }
    while (fen[i] == ' ') i++;
    int ep = 0;
    if (fen[i] >= 'a' && fen[i] <= 'h') ep = fen[i] - 'a' + 1;

    // legality of the placement
    u64 occ = b.bb[1] | b.bb[2] | b.bb[3];
    if (b.bb[0] & ~occ) return false;
    u64 kings = b.bb[2] & b.bb[3] & ~b.bb[1];
    u64 white = occ & ~b.bb[0], black = b.bb[0];
    u64 pawns = b.bb[1] & ~b.bb[2] & ~b.bb[3];
    if ((b.bb[1] & b.bb[2] & b.bb[3])) return false;  // piece code 7
    if (popc(kings & white) != 1 || popc(kings & black) != 1) return false;
    if (pawns & PROMO_RANKS) return false;
    int wk = lsb(kings & white), bk = lsb(kings & black);
    if (king_att(wk) & (1ULL << bk)) return false;
    // drop castle rights whose king or rook is not at home
    auto is_at = [&](int sq, int piece, bool blk) {
        return piece_on(b, sq) == piece && (((b.bb[0] >> sq) & 1) != 0) == blk;
    };
    if (!is_at(4, KING, false)) castle &= ~3u;
    if (!is_at(7, ROOK, false)) castle &= ~1u;
    if (!is_at(0, ROOK, false)) castle &= ~2u;
    if (!is_at(60, KING, true)) castle &= ~12u;
    if (!is_at(63, ROOK, true)) castle &= ~4u;
    if (!is_at(56, ROOK, true)) castle &= ~8u;
    // keep an en-passant file only if the side that just moved has a pawn
    // that could have double-pushed past an empty target square
    if (ep) {
        int f = ep - 1;
        int victim = color == WHITE ? 32 + f : 24 + f;
        int target = color == WHITE ? 40 + f : 16 + f;
        int origin = color == WHITE ? 48 + f : 8 + f;
        bool ok = is_at(victim, PAWN, color == WHITE) && !(occ & (1ULL << target)) && !(occ & (1ULL << origin));
        if (!ok) ep = 0;
    }
    u32 st = castle | ((u32)ep << 4);
    // the side not to move must not be in check
    {
        Sets s = color == WHITE ? derive<BLACK>(b) : derive<WHITE>(b);  // sets from the other side's view
        u64 their_king = s.kings & s.us;
        int tk = bit_index(their_king);
        u64 att = color == WHITE ? enemy_attacks<BLACK>(s, 0, tk) : enemy_attacks<WHITE>(s, 0, tk);
        if (att & their_king) return false;
    }
    for (int k = 0; k < 4; k++) out->bb[k] = b.bb[k];
    out->state = (uint8_t)st;
    out->color = (uint8_t)color;
    return true;
}

inline void write_fen(const pb_pos &p, char *buf)
{
    static const char W[] = " PNBRQK", B[] = " pnbrqk";
    Board b;
    for (int k = 0; k < 4; k++) b.bb[k] = p.bb[k];
    int k = 0;
    for (int r = 7; r >= 0; r--) {
        int run = 0;
        for (int f = 0; f < 8; f++) {
            int sq = r * 8 + f, pc = piece_on(b, sq);
            if (!pc) {
                run++;
                continue;
            }
            if (run) buf[k++] = (char)('0' + run);
            run = 0;
            buf[k++] = ((b.bb[0] >> sq) & 1) ? B[pc] : W[pc];
        }
        if (run) buf[k++] = (char)('0' + run);
        if (r) buf[k++] = '/';
    }
    buf[k++] = ' ';
    buf[k++] = p.color ? 'b' : 'w';
    buf[k++] = ' ';
    if (p.state & 15) {
        if (p.state & 1) buf[k++] = 'K';
        if (p.state & 2) buf[k++] = 'Q';
        if (p.state & 4) buf[k++] = 'k';
        if (p.state & 8) buf[k++] = 'q';
    } else {
        buf[k++] = '-';
    }
    buf[k++] = ' ';
    int ep = p.state >> 4;
    if (ep) {
        buf[k++] = (char)('a' + ep - 1);
        buf[k++] = p.color == WHITE ? '6' : '3';
    } else {
        buf[k++] = '-';
    }
    memcpy(buf + k, " 0 1", 5);
}

}  // namespace pb
