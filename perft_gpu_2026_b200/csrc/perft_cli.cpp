// perft_cli.cpp - the perft_gpu command line on top of the C ABI.
//
//   perft_gpu <fen> <depth> [<launchdepth>] [-nott] [-dtt <MB>] [-htt <MB>] [-ld <N>] [-cpu] [-strict] [-json]
//             [-journal <file>]
//   perft_gpu -batch <file> [<depth>] [-cpu] [-strict] [-json]
//
// Same surface and output as the reference program (perft.cu:13-186):
// flags may appear anywhere, a third positional argument is the launch depth,
// no arguments runs the initial position to depth 10, and every depth prints
//   "\nPerft(%02d): <count>, time: <s> seconds, nps: <n>\n"
// (launcher.cu:732-735).  -strict is new: it counts the two cases where the
// reference's move counting merges two moves (see include/perft_b200.h).
// -json adds one JSON object per depth after the usual line.  -batch runs a
// file of positions, one per line: a FEN followed by optional ";D<k> <count>"
// expected counts (EPD-style); every depth up to the largest listed (or the
// <depth> argument) runs as one batched GPU pass over all positions, and
// mismatches against the listed counts are reported.  -journal <file> makes
// a long run resumable: the final depth runs root move by root move, each
// finished subtree is appended to the file, and a rerun with the same file,
// FEN and depth skips the moves already recorded there.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/perft_b200.h"


// Decimal text of a 128-bit count (the library's formatter, the reference's
// uint128::toDecimalString).
static std::string u128_text(pb_u128 v)
{
    char buf[48];
    pb_u128_text(&v, buf, sizeof(buf));
    return buf;
}

static double u128_double(pb_u128 v) { return (double)v.hi * 18446744073709551616.0 + (double)v.lo; }

static void print_depth(int d, pb_u128 v, double secs)
{
    printf("\nPerft(%02d): %s, time: %g seconds", d, u128_text(v).c_str(), secs);
    if (secs > 0) printf(", nps: %llu", (unsigned long long)(u128_double(v) / secs));
    printf("\n");
    fflush(stdout);
}

static void print_json(int d, pb_u128 v, double secs)
{
    printf("{\"depth\": %d, \"nodes\": \"%s\", \"seconds\": %.9g, \"nps\": %.6g}\n", d, u128_text(v).c_str(), secs,
           secs > 0 ? u128_double(v) / secs : 0.0);
    fflush(stdout);
}

struct BatchLine {
    std::string fen;
    std::vector<std::pair<int, unsigned long long>> expect;
};

static int run_batch(const std::string &path, int depth_arg, bool cpu, bool json, pb_opts opts)
{
    std::ifstream in(path);
    if (!in) {
        fprintf(stderr, "cannot open %s\n", path.c_str());
        return 1;
    }
    std::vector<BatchLine> lines;
    std::vector<pb_pos> roots;
    std::string line;
    int maxd = 0;
    while (std::getline(in, line)) {
        if (line.empty() || line[0] == '#') continue;
        BatchLine bl;
        size_t semi = line.find(';');
        bl.fen = line.substr(0, semi);
        while (semi != std::string::npos) {
            size_t next = line.find(';', semi + 1);
            std::string item = line.substr(semi + 1, next == std::string::npos ? std::string::npos : next - semi - 1);
            std::istringstream is(item);
            std::string tag;
            unsigned long long cnt = 0;
            if (is >> tag >> cnt && tag.size() >= 2 && (tag[0] == 'D' || tag[0] == 'd'))
                bl.expect.push_back({atoi(tag.c_str() + 1), cnt});
            semi = next;
        }
        pb_pos p;
        if (pb_parse_fen(bl.fen.c_str(), &p) != PB_OK) {
            fprintf(stderr, "invalid FEN in %s: %s\n", path.c_str(), bl.fen.c_str());
            return 1;
        }
        for (auto &e : bl.expect) maxd = std::max(maxd, e.first);
        lines.push_back(bl);
        roots.push_back(p);
    }
    int depth = depth_arg > 0 ? depth_arg : (maxd > 0 ? maxd : 1);
    pb_ctx *ctx = nullptr;
    opts.use_tt = 0;
    if (pb_create(cpu ? -1 : 0, &opts, &ctx) != PB_OK) {
        fprintf(stderr, "init failed\n");
        return 1;
    }
    int n = (int)roots.size(), bad = 0;
    std::vector<uint64_t> counts(n);
    std::vector<int> depths(n);
    for (int d = 1; d <= depth; d++) {
        auto t0 = std::chrono::steady_clock::now();
        int rc;
        if (cpu) {
            rc = PB_OK;
            for (int i = 0; i < n && rc == PB_OK; i++) rc = pb_perft_cpu(ctx, &roots[i], d, &counts[i]);
        } else {
            for (int i = 0; i < n; i++) depths[i] = d;
            rc = pb_perft_batch(ctx, roots.data(), depths.data(), n, counts.data());
        }
        double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (rc != PB_OK) {
            fprintf(stderr, "error: %s\n", pb_last_error(ctx));
            pb_destroy(ctx);
            return 1;
        }
        pb_u128 total{0, 0};
        for (int i = 0; i < n; i++) {
            pb_u128 c{counts[i], 0};
            pb_u128_add(&total, &c);
            const char *mark = "";
            for (auto &e : lines[i].expect)
                if (e.first == d && e.second != counts[i]) {
                    mark = "  MISMATCH";
                    bad++;
                }
            printf("pos %d Perft(%02d): %llu%s\n", i + 1, d, (unsigned long long)counts[i], mark);
        }
        printf("\nBatch Perft(%02d): %s over %d positions, time: %g seconds, nps: %llu\n", d, u128_text(total).c_str(), n,
               secs, (unsigned long long)(secs > 0 ? u128_double(total) / secs : 0));
        if (json) print_json(d, total, secs);
        fflush(stdout);
    }
    printf("batch: %d positions, %d mismatches\n", n, bad);
    pb_destroy(ctx);
    return bad ? 2 : 0;
}

static std::string move_text(uint16_t m)
{
    const char *files = "abcdefgh";
    int f = m & 63, t = (m >> 6) & 63, fl = m >> 12;
    std::string out;
    out += files[f & 7];
    out += char('1' + (f >> 3));
    out += files[t & 7];
    out += char('1' + (t >> 3));
    if (fl & 8) out += "nbrq"[fl & 3];
    return out;
}

static pb_u128 add_u128(pb_u128 a, uint64_t b)
{
    pb_u128 c{b, 0};
    pb_u128_add(&a, &c);
    return a;
}

// The final depth, one root move at a time, with the journal file: lines
// "<depth> <move> <count> <fen>" for finished subtrees.  Recorded moves of the
// same FEN and depth are read back instead of recomputed; every subtree
// finished here is appended (and flushed) as soon as it is known.
static int journaled_depth(pb_ctx *ctx, const pb_pos &root, const std::string &fen, int depth,
                           const std::string &path, pb_u128 *total, double *secs, int *reused)
{
    std::vector<std::pair<std::string, uint64_t>> done;
    {
        std::ifstream in(path);
        std::string line;
        while (std::getline(in, line)) {
            std::istringstream ls(line);
            int d;
            std::string mv, f, rest;
            unsigned long long c;
            if (!(ls >> d >> mv >> c)) continue;
            std::getline(ls, rest);
            f = rest.substr(rest.find_first_not_of(' ') == std::string::npos ? 0 : rest.find_first_not_of(' '));
            if (d == depth && f == fen) done.emplace_back(mv, c);
        }
    }
    FILE *out = fopen(path.c_str(), "a");
    if (!out) {
        fprintf(stderr, "cannot open journal %s\n", path.c_str());
        return PB_ERR_ARG;
    }
    uint16_t moves[256];
    int n = pb_generate_moves(&root, moves);
    *total = pb_u128{0, 0};
    *reused = 0;
    auto t0 = std::chrono::steady_clock::now();
    for (int i = 0; i < n; i++) {
        const std::string mt = move_text(moves[i]);
        auto hit = std::find_if(done.begin(), done.end(), [&](const auto &e) { return e.first == mt; });
        if (hit != done.end()) {
            *total = add_u128(*total, hit->second);
            (*reused)++;
            continue;
        }
        pb_pos child = root;
        pb_make_move(&child, moves[i]);
        pb_u128 v;
        double s = 0;
        int rc = pb_perft_launch(ctx, &child, depth - 1, &v, &s);
        if (rc != PB_OK) {
            fclose(out);
            return rc;
        }
        if (v.hi) {  // a subtree above 2^64 is not journalled; count it all the same
            total->hi += v.hi;
        } else {
            fprintf(out, "%d %s %llu %s\n", depth, mt.c_str(), (unsigned long long)v.lo, fen.c_str());
            fflush(out);
        }
        *total = add_u128(*total, v.lo);
    }
    fclose(out);
    *secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return PB_OK;
}

// -hd: host driver above the launch depth (1 = depth first, 2 = breadth
// first with batched GPU calls); -lk: leaf kernel.  0 keeps the default.
static int apply_tuning(pb_ctx *ctx, int host_driver, int leaf_kernel)
{
    pb_tuning t;
    memset(&t, 0, sizeof(t));
    t.host_driver = host_driver;
    t.leaf_kernel = leaf_kernel;
    int rc = pb_set_tuning(ctx, &t);
    if (rc != PB_OK) fprintf(stderr, "invalid -hd or -lk value\n");
    return rc;
}

int main(int argc, char **argv)
{
    bool cpu = false, json = false;
    int host_driver = 0, leaf_kernel = 0;
    std::string batch_file, journal;
    pb_opts opts;
    pb_default_opts(&opts);
    std::vector<std::string> pos;
    for (int i = 1; i < argc; i++) {
        std::string a = argv[i];
        if (a == "-cpu") cpu = true;
        else if (a == "-nott") opts.use_tt = 0;
        else if (a == "-strict") opts.strict = 1;
        else if (a == "-json") json = true;
        else if (a == "-batch" && i + 1 < argc) batch_file = argv[++i];
        else if (a == "-journal" && i + 1 < argc) journal = argv[++i];
        else if (a == "-ld" && i + 1 < argc) opts.launch_depth = atoi(argv[++i]);
        else if (a == "-dtt" && i + 1 < argc) opts.device_tt_mb = atoi(argv[++i]);
        else if (a == "-htt" && i + 1 < argc) opts.host_tt_mb = atoi(argv[++i]);
        else if (a == "-hd" && i + 1 < argc) host_driver = atoi(argv[++i]);
        else if (a == "-lk" && i + 1 < argc) leaf_kernel = atoi(argv[++i]);
        else pos.push_back(a);
    }
    if (!batch_file.empty()) return run_batch(batch_file, pos.empty() ? 0 : atoi(pos[0].c_str()), cpu, json, opts);
    std::string fen = "rnbqkbnr/pppppppp/8/8/8/8/PPPPPPPP/RNBQKBNR w KQkq - 0 1";
    int max_depth = 10;
    if (pos.size() >= 2) {
        if (pos[0].size() > 5) fen = pos[0];
        max_depth = atoi(pos[1].c_str());
        if (pos.size() >= 3 && opts.launch_depth == 0) opts.launch_depth = atoi(pos[2].c_str());
    } else {
        printf("\nUsage: perft_gpu <fen> <depth> [<launchdepth>] [-nott] [-dtt <MB>] [-htt <MB>] [-ld <N>] [-cpu] [-strict]"
               " [-json] [-journal <file>] [-hd 1|2] [-lk <leaf kernel>]\n");
        printf("\nAs no parameters were provided... running default test\n");
    }
    pb_pos root;
    if (pb_parse_fen(fen.c_str(), &root) != PB_OK) {
        fprintf(stderr, "invalid FEN: %s\n", fen.c_str());
        return 1;
    }
    if (max_depth < 1 || max_depth > 30) {
        fprintf(stderr, "depth must be 1..30\n");
        return 1;
    }
    pb_ctx *ctx = nullptr;
    if (cpu) {
        printf("CPU mode\n");
        fflush(stdout);
        opts.use_tt = 0;
        if (pb_create(-1, &opts, &ctx) != PB_OK) return 1;
        if (apply_tuning(ctx, host_driver, leaf_kernel) != PB_OK) return 1;
        for (int d = 1; d <= max_depth; d++) {
            pb_u128 v;
            double secs = 0;
            int reused = 0;
            int rc = (!journal.empty() && d == max_depth && d > 1)
                         ? journaled_depth(ctx, root, fen, d, journal, &v, &secs, &reused)
                         : pb_perft_launch(ctx, &root, d, &v, &secs);
            if (reused) printf("\njournal: %d root moves read back from %s\n", reused, journal.c_str());
            if (rc != PB_OK) {
                fprintf(stderr, "error: %s\n", pb_last_error(ctx));
                return 1;
            }
            print_depth(d, v, secs);
            if (json) print_json(d, v, secs);
        }
        pb_destroy(ctx);
        return 0;
    }
    int ngpu = pb_device_count();
    printf("No of GPUs detected: %d\n", ngpu);
    if (ngpu == 0) {
        printf("No CUDA GPUs found. Exiting.\n");
        return 1;
    }
    opts.verbose = 1;
    int rc = pb_create(0, &opts, &ctx);
    if (rc != PB_OK) {
        fprintf(stderr, "init failed (%d)\n", rc);
        return 1;
    }
    if (apply_tuning(ctx, host_driver, leaf_kernel) != PB_OK) return 1;
    printf("Launch depth: %d\n", pb_prepare(ctx, &root, max_depth));
    fflush(stdout);
    for (int d = 1; d <= max_depth; d++) {
        pb_u128 v;
        double secs = 0;
        int reused = 0;
        rc = (!journal.empty() && d == max_depth && d > 1) ? journaled_depth(ctx, root, fen, d, journal, &v, &secs, &reused)
                                                           : pb_perft_launch(ctx, &root, d, &v, &secs);
        if (reused) printf("\njournal: %d root moves read back from %s\n", reused, journal.c_str());
        if (rc != PB_OK) {
            fprintf(stderr, "error: %s\n", pb_last_error(ctx));
            pb_destroy(ctx);
            return 1;
        }
        print_depth(d, v, secs);
        if (json) print_json(d, v, secs);
    }
    pb_destroy(ctx);
    return 0;
}
