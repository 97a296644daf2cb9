/*
 * perft_b200.h - C ABI of the B200 perft engine (libperftb200.so).
 *
 * The reference (perft_gpu) has no library API: its boundary is the
 * perft_gpu command line (perft.cu:13-186) over an internal C++ function set
 * (launcher.h:13-35).  Each entry point below names the reference function it
 * stands in for.  All calls are synchronous, return a PB_* status code and
 * never exit the process; a context owns its device memory and stream and is
 * used from one host thread at a time.  Counts are bit-exact with the
 * reference's `-cpu` path (launcher.cu:762-816) on the same FEN and depth.
 */
#ifndef PERFT_B200_H
#define PERFT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    PB_OK = 0,
    PB_ERR_ARG = -1,        /* bad argument (null pointer, depth out of range) */
    PB_ERR_FEN = -2,        /* FEN rejected (see pb_parse_fen) */
    PB_ERR_CUDA = -3,       /* a CUDA call failed; pb_last_error has the text */
    PB_ERR_NOMEM = -4,      /* device or host allocation failed */
    PB_ERR_DEVICE = -5,     /* a kernel reported an error word (timeout, capacity) */
    PB_ERR_NODEVICE = -6    /* no CUDA device (GPU entry points only) */
};

/* Position: quad bitboard (chess.h:66-76) + packed state byte (castle bits
 * [3:0] = white K,Q black K,Q; en-passant file+1 in [7:4], chess.h:78-92) +
 * side to move (0 white, 1 black). 40 bytes. */
typedef struct {
    uint64_t bb[4];
    uint8_t state;
    uint8_t color;
    uint8_t pad[6];
} pb_pos;

typedef struct {
    uint64_t lo, hi;
} pb_u128;

typedef struct {
    size_t arena_bytes;   /* BFS arena; 0 = auto (launcher.cu:59-88 sizes it from VRAM) */
    int use_tt;           /* transposition tables on (-nott clears it, perft.cu:26-29) */
    int device_tt_mb;     /* -dtt: device TT budget in MB, 0 = auto */
    int host_tt_mb;       /* -htt: host TT budget in MB, 0 = auto */
    int launch_depth;     /* -ld: GPU/CPU split depth, 0 = auto (launcher.cu:533-562) */
    int strict;           /* 1 = exact counts where the reference's counting merges moves */
    int verbose;          /* print allocation lines like the reference's preamble */
} pb_opts;

typedef struct pb_ctx pb_ctx;

/* Library version string. */
const char *pb_version(void);

/* Fills opts with defaults (TT on, auto budgets, auto launch depth). */
void pb_default_opts(pb_opts *opts);

/* Replaces initGPU + initMoveGen + initTT (launcher.cu:59-88, :128-351;
 * perft_kernels.cu:995-1134). device < 0 creates a host-only context (the
 * -cpu mode, perft.cu:100-116). */
int pb_create(int device, const pb_opts *opts, pb_ctx **out);

/* Replaces freeTT + cudaFree of the arena (launcher.cu:509-531, perft.cu:180-181). */
void pb_destroy(pb_ctx *ctx);

/* Text of the last error on this context (never NULL). */
const char *pb_last_error(const pb_ctx *ctx);

/* Replaces readFENString (util.cpp:7-95).  The halfmove/fullmove fields are
 * ignored like the reference.  Unlike the reference, positions a legal game
 * cannot reach are rejected (missing or extra king, adjacent kings, side not
 * to move in check, pawns on the first/last rank), castle rights without the
 * king and rook on their home squares are dropped, and an en-passant square
 * without a pawn that just double-pushed is dropped. */
int pb_parse_fen(const char *fen, pb_pos *out);

/* Writes the FEN of pos into buf (at least 96 bytes). */
int pb_to_fen(const pb_pos *pos, char *buf, size_t len);

/* Number of CUDA devices (cudaGetDeviceCount, perft.cu:62-69); 0 if none. */
int pb_device_count(void);

/* Fixes the launch depth used by pb_perft_launch for this context and
 * returns it: opts.launch_depth when set, else estimated from the branching
 * factor of pos and the arena size (estimateLaunchDepth, launcher.cu:533-562). */
int pb_choose_launch_depth(pb_ctx *ctx, const pb_pos *pos);

/* Replaces initTT (launcher.cu:128-351) for a run up to max_depth: fixes the
 * launch depth (as pb_choose_launch_depth) and, in TT mode, sizes the host
 * tables for remaining depths launch_depth..max_depth.  Device tables are
 * sized on the first GPU call. */
int pb_prepare(pb_ctx *ctx, const pb_pos *pos, int max_depth);

/* Replaces perft_gpu_host_bfs (perft_kernels.cu:620-990): perft(depth) of one
 * position, the whole subtree on the GPU (the host only splits the root when
 * a level would not fit the arena). */
int pb_perft_position(pb_ctx *ctx, const pb_pos *pos, int depth, uint64_t *count);

/* Replaces perftLauncher (launcher.cu:718-737): perft(depth) with the tree
 * above the launch depth walked on the host (with the host TT when enabled)
 * and GPU calls below it.  128-bit result. */
int pb_perft_launch(pb_ctx *ctx, const pb_pos *pos, int depth, pb_u128 *count, double *seconds);

/* The CLI loop (perft.cu:156-177): perft for depths 1..max_depth of a FEN,
 * cumulative per-depth results and wall times. */
int pb_perft(pb_ctx *ctx, const char *fen, int max_depth, pb_u128 *per_depth, double *per_depth_secs);

/* 128-bit counts (uint128.h:13-108).  pb_u128_add is the accumulation the
 * host recursion above the launch depth applies to every subtree count
 * (perft_cpu_recurse, launcher.cu:570-571, 700-705): *acc += *v with the
 * carry into the high word.  pb_u128_text writes the decimal text of *v
 * (uint128::toDecimalString, uint128.h:46-108) into buf; returns the text
 * length, or PB_ERR_ARG when buf holds fewer than 40 bytes. */
void pb_u128_add(pb_u128 *acc, const pb_u128 *v);
int pb_u128_text(const pb_u128 *v, char *buf, size_t len);

/* Self-test of the listed-piece move count (leaf kernel 5), on the host: for
 * every child of each position, the count with the side's piece squares
 * listed from the parent position equals the count from the child's piece
 * bitboards (both counting conventions, in and out of check).  No
 * counterpart in the reference.  *checked = children compared (positions
 * with more than four knights, diagonal or orthogonal movers are skipped),
 * *mismatches = disagreements. */
int pb_selftest_listed_counts(const pb_pos *pos, int n, uint64_t *checked, uint64_t *mismatches);

/* Replaces perft_cpu_dispatch (launcher.cu:807-816): host-only perft. */
int pb_perft_cpu(pb_ctx *ctx, const pb_pos *pos, int depth, uint64_t *count);

/* No reference counterpart: perft of n independent roots in one batched GPU
 * pass; counts[i] = perft(depths[i]) of roots[i]. */
int pb_perft_batch(pb_ctx *ctx, const pb_pos *roots, const int *depths, int n, uint64_t *counts);

/* Host chess core (MoveGeneratorBitboard.h:1700-2067): legal-move count with
 * the reference's counting conventions (strict = 0) or exact (strict = 1),
 * move generation (returns the number of moves written, buffer >= 256) and
 * make-move. */
int pb_count_moves(const pb_pos *pos, int strict);
int pb_generate_moves(const pb_pos *pos, uint16_t *moves);
int pb_make_move(pb_pos *pos, uint16_t move);

/* 128-bit Zobrist key of a position (computeHash, zobrist.h:81-147), and the
 * key after `move` updated incrementally from the parent's key
 * (updateHashAfterMove, zobrist.h:149-227): the keys the transposition tables
 * use, on host and device alike. */
int pb_position_hash(const pb_pos *pos, pb_u128 *out);
int pb_hash_after_move(const pb_u128 *key, const pb_pos *pos, uint16_t move, pb_u128 *out);

/* Workload generator (no reference counterpart): a playout of `plies`
 * uniformly random legal moves from the standard initial array; each move is
 * drawn with splitmix64 (state advanced in place) among the legal moves sorted
 * by UCI text.  Returns the number of plies played (fewer at mate/stalemate). */
int pb_random_playout(uint64_t *rng_state, int plies, pb_pos *out);

/* Statistics of the last GPU perft call on a context.  The device times are
 * CUDA events on the context's stream; no reference counterpart (the
 * reference keeps host-timer histograms behind VERBOSE_LOGGING,
 * launcher.cu:35-57). */
typedef struct {
    double device_ms;          /* first kernel to last kernel, engine stream */
    double leaf_ms;            /* the fused two-ply leaf kernel alone */
    uint64_t leaf_edges;       /* edges the leaf kernel took (one perft(2) each) */
    uint64_t leaf_positions;   /* positions the leaf kernel counted (move-count calls) */
    uint64_t nodes;            /* the perft result of the call */
    uint32_t kernels;          /* kernel launches of the call */
    uint32_t levels;           /* BFS expand levels */
    uint64_t level_sizes[16];  /* edges per level, level 0 = root moves */
    uint64_t h2d_bytes;        /* host-to-device bytes copied */
    uint64_t d2h_bytes;        /* device-to-host bytes copied */
} pb_stats;

/* Launch parameters of the GPU path (no reference counterpart: the
 * reference fixes them at compile time, switches.h:8-24, perft_kernels.cu:74).
 * Zero fields keep the current value.  leaf_kernel: 1 = one edge per thread,
 * 2 = cooperative (grandchildren spread over the CTA), 3 = in-check children
 * deferred to a second pass, 4 = one edge per thread with the CTA's children
 * ranked by move count first, 5 = as 4 with each child's own-piece squares
 * listed once for all of its grandchild counts, 6 = as 5 with four children
 * per thread ranked across the CTA and dealt to the warps in light/heavy
 * chunk pairs (default, with 1024-thread CTAs); batched, planned and table
 * leaves rank their children for 4 to 6 and list pieces for 5 and 6;
 * leaf_blocks_per_sm: persistent grid of the cooperative leaf. */
typedef struct {
    int leaf_kernel;
    int leaf_blocks_per_sm;
    int leaf_threads;   /* CTA size of leaf kernels 1, 3 to 6: 128, 256, 512 (not 3) or, with leaf
                           kernel 6 only, 1024 (default; other kernels then run 256) */
    int gen_threads;    /* CTA size of the staged generator: 64 or 128 (default); stages 64 moves per thread */
    int leaf_fuse;      /* plies fused in the leaf kernel: 2 (default) or 1 (one more BFS level) */
    int tt_replace;     /* device TT replacement: 1 = always overwrite (default, tt.h:60-70),
                           2 = two-slot buckets, the larger subtree keeps the first slot;
                           takes effect when the device tables are next sized */
    int planned_leaf;   /* leaf of planned (graph-captured) batches: 1 = grid over the planned
                           capacity, CTAs past the level's size leave at once (default);
                           2 = persistent CTAs fed by an atomic work queue */
    int host_driver;    /* tree above the launch depth in pb_perft_launch: 1 = depth first, one GPU
                           call per subtree (perft_cpu_recurse, launcher.cu:572-715; default);
                           2 = breadth first, transpositions merged by key with tables, the
                           launch-depth positions in batched GPU calls */
    int tt_leaf;        /* table leaf with leaf kernels 4 and 5: 1 = one edge per thread;
                           2 = persistent CTAs that queue their table misses in shared memory and
                           count only full CTAs of misses (default) */
} pb_tuning;

int pb_set_tuning(pb_ctx *ctx, const pb_tuning *t);
int pb_get_tuning(const pb_ctx *ctx, pb_tuning *t);

/* Turns per-call event timing on or off (off by default). */
int pb_set_timing(pb_ctx *ctx, int enable);
int pb_last_stats(const pb_ctx *ctx, pb_stats *out);

/* n playouts at once (threads): position i uses the generator state drawn
 * i-th from a splitmix64 stream seeded with `seed`; from that state it draws
 * its length uniformly in [min_plies, max_plies], then plays as
 * pb_random_playout.  played[i] (optional) = plies actually played. */
int pb_random_playouts(uint64_t seed, int n, int min_plies, int max_plies, pb_pos *out, int *played);

/* Device kernels on caller-owned device buffers, for tests: exclusive scan of
 * n u32 counts into n u64 offsets and a device u64 total. */
int pb_dev_scan(pb_ctx *ctx, const uint32_t *d_in, uint64_t n, uint64_t *d_out, uint64_t *d_total);

/* The BFS level kernels on caller-owned device buffers, for unit tests
 * against the host functions.  Boards are 4 x u64 (the pb_pos bitboards),
 * 32-byte aligned; color = side to move at the parents.
 * pb_dev_expand: child i = parent d_pidx[i] after move d_moves[i]; writes its
 * board, state and exact legal-move count (makemove_and_count_moves_kernel,
 * perft_kernels.cu:201-257).
 * pb_dev_generate: the moves of parent j go to [d_offs[j], d_offs[j+1]) (the
 * last ends at *d_total) as (move, parent j), in the generator's order
 * (generate_moves_kernel + mp_interval_expand_kernel, perft_kernels.cu:77-173,
 * :263-311); the offsets must come from the exact counts. */
int pb_dev_expand(pb_ctx *ctx, const void *d_boards, const uint8_t *d_states, int color, const uint32_t *d_pidx,
                  const uint16_t *d_moves, uint64_t n, uint64_t nparents, void *d_child_boards,
                  uint8_t *d_child_states, uint32_t *d_counts);
int pb_dev_generate(pb_ctx *ctx, const void *d_boards, const uint8_t *d_states, int color, const uint64_t *d_offs,
                    const uint64_t *d_total, uint64_t n, uint16_t *d_moves, uint32_t *d_pidx);

/* Self-test of the device-side failure detection (no reference counterpart:
 * the reference's waits are inside CUB).  Runs one tile of the scan whose
 * predecessor never publishes: the look-back gives up after its bounded wait
 * (about a second) and the kernel returns.  *device_error receives the error
 * word (1 = scan wait timed out), *seconds (optional) the wait's wall time.
 * Returns PB_OK when the launch completed; the context stays usable. */
int pb_selftest_wait_timeout(pb_ctx *ctx, uint32_t *device_error, double *seconds);

/* Race self-test of the device tables (no reference counterpart; the
 * reference relies on the same kind of XOR lock, tt.h:9-14,49-57): all the
 * GPU's threads store and probe 8192 keys at once in a 1024-slot table of the
 * 16-byte (mode 0) or 32-byte (mode 1) format, or (mode 2) in a 2^24-slot
 * 16-byte table, the smallest the engine builds in that format, with the
 * keys chosen to fall into 8 of its slots.  *bad = probes that reported a
 * hit with a count that is not the key's own (must be 0), *hits = probes
 * that hit. */
int pb_selftest_tt_race(pb_ctx *ctx, int mode, uint64_t *bad, uint64_t *hits);

/* Learned scheduler network (no reference counterpart): 781 binary inputs
 * (12x64 piece-square, side to move, 4 castle rights, 8 en-passant files) ->
 * 256 -> 256 -> 4 outputs = predicted log2(1 + perft(k)), k = 1..4.  BF16
 * weights with an FP32 master copy, FP32 accumulation, Adam; trained and run
 * by the library's own kernels on the context's GPU.  Parameter layout of
 * get/set: [W1 781x256 | b1 256 | W2 256x256 | b2 256 | W3 256x4 | b3 4]. */
size_t pb_mlp_param_count(void);
int pb_mlp_init(pb_ctx *ctx, uint64_t seed, const float *out_bias);
int pb_mlp_get_params(pb_ctx *ctx, float *out, size_t count);
int pb_mlp_set_params(pb_ctx *ctx, const float *in, size_t count);
/* Mean squared error and gradients of one batch (n a multiple of 64). */
int pb_mlp_gradients(pb_ctx *ctx, const pb_pos *pos, const float *targets, int n, float *grads, float *loss);
int pb_mlp_train(pb_ctx *ctx, const pb_pos *pos, const float *targets, int n, int epochs, int batch, float lr,
                 uint64_t seed, float *final_loss);
int pb_mlp_predict(pb_ctx *ctx, const pb_pos *pos, int n, float *out);

/* Self-test of the network's tensor-core GEMM (tcgen05, BF16 operands, FP32
 * accumulation) on the context's GPU: c[M x N] (row-major) = A * B, where
 * element (m, k) of A is a[m*K + k], or with ta a[k*M + m], and element
 * (k, n) of B is b[k*N + n], or with tb b[n*K + k]; a and b hold BF16 bit
 * patterns.  M a multiple of 8, N of 128, K of 64 (else PB_ERR_ARG).  With
 * reps > 0 the product then runs reps more times between two CUDA events on
 * the context's stream and *ms = their mean duration.  No reference
 * counterpart. */
int pb_selftest_gemm(pb_ctx *ctx, int ta, int tb, int M, int N, int K, const uint16_t *a, const uint16_t *b,
                     float *c, int reps, double *ms);

/* Learned batch planner (no reference counterpart): like pb_perft_batch, but
 * the network's predictions size every BFS level up front, bin-pack the roots
 * into batches that fit the arena and split roots too large for one batch;
 * each batch runs as one captured CUDA graph (device-side sizes, a persistent
 * leaf fed by a device work queue).  A batch that outgrows its planned sizes
 * is rerun with the exact count-then-allocate path; counts are exact either
 * way.  Needs pb_mlp_init (and normally pb_mlp_train) first. */
typedef struct {
    uint32_t batches;        /* batches run */
    uint32_t graph_batches;  /* of which as planned CUDA graphs */
    uint32_t retries;        /* planned batches rerun with exact sizing */
    uint32_t split_roots;    /* roots split into children for size */
} pb_plan_stats;
int pb_perft_batch_planned(pb_ctx *ctx, const pb_pos *roots, const int *depths, int n, uint64_t *counts,
                           pb_plan_stats *stats);

/* Allocation-free variant of pb_dev_scan.  No counterpart in the reference.
 * For callers that may not allocate device memory at the point they need the
 * scan: allocator and out-of-memory handling paths, hosts whose framework
 * owns every device buffer and forbids raw cudaMalloc, and latency-critical
 * loops where cudaMalloc's implicit device synchronisation is not allowed.
 * The caller passes the input and output buffers; the scan's own
 * scratch (tile status words, ticket, error word) is a fixed device array
 * inside the library, so the call makes no cudaMalloc/cudaFree and no
 * allocating library call.
 *   - n is limited to 8,388,608 counts (the array's status words cover that
 *     many scan tiles); larger n returns PB_ERR_ARG without touching the GPU.
 *   - Runs on `stream` (NULL = default stream) of the current device and waits
 *     for it before returning; n == 0 returns PB_OK and writes nothing.
 *   - Because it waits for its stream, it cannot run inside a stream capture:
 *     a call on a capturing stream returns PB_ERR_ARG and records nothing.
 *   - Every call looks up the array's device address with the caller's device
 *     current (the lookup allocates nothing; the first call on a device also
 *     loads the library's module there).
 *   - The array is 8.25 KB per device and stays until the process exits.
 *   - All calls share the one array, so calls that overlap on the GPU (other
 *     threads or streams of the same device) race; serialise them. */
int pb_scan_u32_noalloc(const uint32_t *d_in, uint64_t n, uint64_t *d_out, uint64_t *d_total, void *stream);

#ifdef __cplusplus
}
#endif
#endif
