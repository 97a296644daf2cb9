// magic_search.cpp - generates magic_numbers.inc, the slider-attack magic
// multipliers used by the engine's attack tables.
//
// For every square and slider kind the relevant-occupancy mask has b bits;
// a multiplier M is accepted when (occ * M) >> (64 - b) maps every one of the
// 2^b occupancy subsets to a slot holding its attack set, i.e. the map has no
// destructive collision.  Candidates are sparse random words drawn from a
// splitmix64 stream (seed fixed below), so the output is reproducible.
//
// Build and run (writes to stdout):
//   g++ -O2 -o magic_search magic_search.cpp && ./magic_search > magic_numbers.inc
#include <cstdint>
#include <cstdio>
#include <vector>

static uint64_t sm_state = 0x5EED0F3A61C5ULL;
static uint64_t splitmix64()
{
    uint64_t z = (sm_state += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

static uint64_t slide(int sq, uint64_t occ, const int (*dirs)[2], bool mask_only)
{
    uint64_t out = 0;
    int f0 = sq & 7, r0 = sq >> 3;
    for (int d = 0; d < 4; d++) {
        int f = f0 + dirs[d][0], r = r0 + dirs[d][1];
        while (f >= 0 && f < 8 && r >= 0 && r < 8) {
            int nf = f + dirs[d][0], nr = r + dirs[d][1];
            bool edge = !(nf >= 0 && nf < 8 && nr >= 0 && nr < 8);
            if (mask_only && edge) break;
            out |= 1ULL << (r * 8 + f);
            if (occ & (1ULL << (r * 8 + f))) break;
            f = nf;
            r = nr;
        }
    }
    return out;
}

static const int ROOK_DIRS[4][2] = {{1, 0}, {-1, 0}, {0, 1}, {0, -1}};
static const int BISHOP_DIRS[4][2] = {{1, 1}, {1, -1}, {-1, 1}, {-1, -1}};

static uint64_t find_magic(int sq, const int (*dirs)[2])
{
    uint64_t mask = slide(sq, 0, dirs, true);
    int bits = __builtin_popcountll(mask);
    int n = 1 << bits;
    std::vector<uint64_t> occ(n), att(n), used(n);
    // enumerate subsets of mask (Carry-Rippler)
    uint64_t sub = 0;
    for (int i = 0; i < n; i++) {
        occ[i] = sub;
        att[i] = slide(sq, sub, dirs, false);
        sub = (sub - mask) & mask;
    }
    std::vector<int> epoch(n, 0);
    for (int attempt = 1;; attempt++) {
        uint64_t m = splitmix64() & splitmix64() & splitmix64();
        if (__builtin_popcountll((mask * m) & 0xFF00000000000000ULL) < 6) continue;
        bool ok = true;
        for (int i = 0; i < n && ok; i++) {
            int idx = (int)((occ[i] * m) >> (64 - bits));
            if (epoch[idx] != attempt) {
                epoch[idx] = attempt;
                used[idx] = att[i];
            } else if (used[idx] != att[i]) {
                ok = false;
            }
        }
        if (ok) return m;
    }
}

int main()
{
    printf("// Generated by magic_search.cpp (splitmix64 seed 0x5EED0F3A61C5); do not edit.\n");
    printf("// Rook multipliers, squares a1..h8.\n");
    printf("static const uint64_t kRookMagic[64] = {\n");
    for (int sq = 0; sq < 64; sq++)
        printf("    0x%016llxULL,%s", (unsigned long long)find_magic(sq, ROOK_DIRS), (sq % 2 == 1) ? "\n" : "");
    printf("};\n");
    printf("// Bishop multipliers, squares a1..h8.\n");
    printf("static const uint64_t kBishopMagic[64] = {\n");
    for (int sq = 0; sq < 64; sq++)
        printf("    0x%016llxULL,%s", (unsigned long long)find_magic(sq, BISHOP_DIRS), (sq % 2 == 1) ? "\n" : "");
    printf("};\n");
    return 0;
}
