// Host build of the ungapped walk (rmb_ungapped.cuh, the code each lane of k_ungapped runs)
// checked against the oracle's extension (search/ungapped.rs:38-121 restated in
// oracle/rmb_oracle_align.cpp) on seeded random hits.
//
//   ungapped_host <hits> <seed> <xdrop> <matrix>
//
// Prints one line: "hits N bad B steps S".
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <vector>

#include "../oracle/rmb_oracle.hpp"
#include "../rmblast_b200/csrc/rmb_ungapped.cuh"

int main(int argc, char** argv) {
    if (argc < 5) {
        fprintf(stderr, "usage: ungapped_host hits seed xdrop matrix\n");
        return 2;
    }
    const int n = atoi(argv[1]);
    std::mt19937_64 rng((uint64_t)atoll(argv[2]));
    const int xdrop = atoi(argv[3]);
    const rmbo::Matrix mat = rmbo::load_matrix(argv[4]);
    int32_t flat[256];
    for (int a = 0; a < 16; ++a)
        for (int b = 0; b < 16; ++b) flat[a * 16 + b] = mat.s[a][b];
    int bad = 0;
    unsigned long long steps = 0;
    for (int k = 0; k < n; ++k) {
        // a subject, and a query sharing a mutated segment of it around the seed
        const int sl = 20 + (int)(rng() % 3000), ql = 20 + (int)(rng() % 3000);
        std::vector<uint8_t> s(sl), q(ql);
        for (auto& c : s) c = (uint8_t)(rng() % 4);
        for (auto& c : q) c = (uint8_t)(rng() % 4);
        const int seg = 1 + (int)(rng() % std::min(sl, ql));
        const int s0 = (int)(rng() % (sl - seg + 1)), q0 = (int)(rng() % (ql - seg + 1));
        const int div = (int)(rng() % 30);
        for (int j = 0; j < seg; ++j) q[q0 + j] = (int)(rng() % 100) < div ? (uint8_t)(rng() % 4) : s[s0 + j];
        for (int j = 0; j < ql; ++j)
            if (rng() % 500 == 0) q[j] = 14;  // N
        std::vector<uint8_t> qw(ql + 2, 15), sw(sl + 2, 15);
        memcpy(qw.data() + 1, q.data(), ql);
        memcpy(sw.data() + 1, s.data(), sl);
        const int qo = q0 + (int)(rng() % seg), so = s0 + (qo - q0);
        const rmbo::UngappedResult want =
            rmbo::extend_ungapped(qw.data(), qw.size(), sw.data(), sw.size(), (uint32_t)qo, (uint32_t)so, mat, xdrop);
        rmb::UngWalk w;
        w.start(qw.data(), sw.data(), ql, sl, qo, so, xdrop);
        int r;
        do {
            r = w.step(flat);
            ++steps;
        } while (r != 2);
        int32_t sc;
        uint32_t a, b, c, d;
        w.result(sc, a, b, c, d);
        if (sc != want.score || a != want.q_start || b != want.q_end || c != want.s_start || d != want.s_end) {
            if (bad < 5)
                fprintf(stderr, "hit %d: want %d %u-%u %u-%u got %d %u-%u %u-%u\n", k, want.score, want.q_start,
                        want.q_end, want.s_start, want.s_end, sc, a, b, c, d);
            ++bad;
        }
    }
    printf("hits %d bad %d steps %llu\n", n, bad, steps);
    return bad != 0;
}
