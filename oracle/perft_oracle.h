/*
 * perft_oracle.h - CPU restatement of the reference perft path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker: tests/, the smoke
 * check and bench.py's CPU-baseline leg may load it; the product library
 * (perft_gpu_2026_b200/) never links, imports or calls it.
 *
 * It restates, in plain C, the reference's CPU perft (the `-cpu` path of
 * perft_gpu): FEN parsing (util.cpp:7-95), the quad-bitboard make-move
 * (MoveGeneratorBitboard.h:1946-2066, CPU branch), legal move generation
 * (MoveGeneratorBitboard.h:978-1154, 1161-1554), legal move counting
 * (MoveGeneratorBitboard.h:1564-1943) and the recursion
 * (launcher.cu:762-816).  Slider attacks are computed by ray walks instead of
 * the reference's magic lookups, which gives an independent check of the
 * product's magic tables.
 *
 * Parity is pinned against the reference program itself (oracle/_ref) and the
 * known-answer totals in the reference README (README.md:49-103); see
 * tests/test_oracle_pins.py.
 */
#ifndef PERFT_ORACLE_H
#define PERFT_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Quad-bitboard position (chess.h:66-92): bb[0] = black pieces, bb[1..3] =
 * piece-code bits (PAWN=1 .. KING=6); state = castle bits [3:0] + EP file+1
 * in [7:4]; color = side to move (0 white, 1 black). */
typedef struct {
    uint64_t bb[4];
    uint8_t state;
    uint8_t color;
    uint8_t pad[6];
} or_pos;

int      or_parse_fen(const char *fen, or_pos *out);
uint32_t or_count_moves(const or_pos *p);
/* Exact legal-move count; differs from or_count_moves only where the
 * reference's counting merges two moves that share a target square (two
 * pawns promoting by capture onto one square, or two pawns taking the same
 * checking pawn en passant). */
uint32_t or_count_moves_strict(const or_pos *p);
uint32_t or_generate_moves(const or_pos *p, uint16_t *moves);
void     or_make_move(or_pos *p, uint16_t move);
uint64_t or_perft(const or_pos *p, int depth);
uint64_t or_perft_strict(const or_pos *p, int depth);
/* Per-root perft over a batch of positions (one thread). */
void     or_perft_batch(const or_pos *ps, const int *depths, int n, uint64_t *out);
/* Perft of each child of p at depth-1, in generation order; returns the
 * number of children. */
int      or_perft_divide(const or_pos *p, int depth, uint16_t *moves, uint64_t *counts);
/* Random legal playout from the standard initial array: `plies` moves, each
 * chosen with a splitmix64 draw among the legal moves sorted by UCI string.
 * Returns the number of plies actually played (fewer if a terminal position
 * is reached). */
int      or_random_playout(uint64_t *rng_state, int plies, or_pos *out);
uint64_t or_splitmix64(uint64_t *state);
/* Writes the UCI text of a move (at most 6 bytes including NUL). */
void     or_move_uci(uint16_t move, char *buf);
/* Writes the FEN of a position (halfmove/fullmove written as "0 1"). */
void     or_to_fen(const or_pos *p, char *buf);

#ifdef __cplusplus
}
#endif
#endif
