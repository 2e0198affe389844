// Host build of the preliminary-DP thread body (rmb_prelim_stream.cuh, the code k_prelim_stream
// runs on every GPU thread) checked against the oracle's score-only X-drop extension
// (search/gapped.rs:124-337 restated in oracle/rmb_oracle_align.cpp) on seeded random records.
//
//   stream_host <records> <seed> <max_subject_len> <max_divergence_pct> <cutoff> <max_cells>
//
// Prints one line: "records R checked C overflow W bad B cells X oracle_cells Y big Z".
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <vector>

#include "../oracle/rmb_oracle.hpp"
#include "../rmblast_b200/csrc/rmb_prelim_stream.cuh"

namespace {

// One thread's ring (64 slots), the queue and the overflow list, in host memory.
struct HostEnv {
    uint32_t ring[rmb::STREAM_RING];
    uint32_t* queue;
    std::vector<uint32_t>* overflow_list;
    uint32_t& at(uint32_t j) { return ring[j % rmb::STREAM_RING]; }
    uint32_t take() { return (*queue)++; }
    void overflow(uint32_t t) { overflow_list->push_back(t); }
    bool any(bool p) { return p; }
    void fill_rows(bool pending, const uint8_t* qal, int32_t pb, int32_t dir, uint32_t n) {
        if (pending)
            for (uint32_t k = 0; k < n; ++k) at(k) = qal[pb + dir * (int32_t)k] & 15u;
    }
};

}  // namespace

int main(int argc, char** argv) {
    if (argc < 8) {
        fprintf(stderr, "usage: stream_host records seed max_len max_div cutoff max_cells matrix\n");
        return 2;
    }
    const int n = atoi(argv[1]);
    std::mt19937_64 rng((uint64_t)atoll(argv[2]));
    const int max_len = atoi(argv[3]), max_div = atoi(argv[4]), cutoff = atoi(argv[5]);
    const uint32_t max_cells = (uint32_t)atoll(argv[6]);
    const rmbo::Matrix mat = rmbo::load_matrix(argv[7]);
    const int go = 20, ge = 5;
    const int xs[] = {25, 30, 60, 100, 100, 100, 150, 300};

    // records: a random subject and a mutated copy (substitutions, indels, a few N) as the
    // query, each sentinel-wrapped and padded for the kernel's aligned word reads; the query
    // starts at a random byte offset so the column words are misaligned
    std::vector<std::vector<uint8_t>> qbuf(n), sbuf(n);
    std::vector<rmb::PrelimGeo> geo(n);
    for (int i = 0; i < n; ++i) {
        const int sl = 1 + (int)(rng() % (uint64_t)max_len);
        std::vector<uint8_t> s(sl), q;
        for (auto& c : s) c = (uint8_t)(rng() % 4);
        const int div = max_div > 0 ? (int)(rng() % (uint64_t)max_div) : 0;
        for (int j = 0; j < sl; ++j) {
            const int r = (int)(rng() % 100);
            if (r < div / 4) continue;
            if (r < div / 2) q.push_back((uint8_t)(rng() % 4));
            q.push_back(r < div ? (uint8_t)(rng() % 4) : s[j]);
            if (rng() % 200 == 0) q.back() = 14;
        }
        if (q.empty()) q.push_back(0);
        if (rng() % 10 == 0) {  // an unrelated query: bands that collapse or run wide
            q.resize(1 + rng() % 3000);
            for (auto& c : q) c = (uint8_t)(rng() % 4);
        }
        const int qoff = 4 + (int)(rng() % 4);
        qbuf[i].assign(q.size() + 16, 15);
        sbuf[i].assign(s.size() + 16, 15);
        memcpy(qbuf[i].data() + qoff, q.data(), q.size());
        memcpy(sbuf[i].data() + 4, s.data(), s.size());
        rmb::PrelimGeo& g = geo[i];
        g.qseq = (uint64_t)(qbuf[i].data() + qoff);
        g.sseq = (uint64_t)(sbuf[i].data() + 4);
        g.qa = (uint32_t)q.size();
        g.sa = (uint32_t)s.size();
        g.qp = (uint32_t)(rng() % (q.size() + 1));
        g.sp = (uint32_t)(rng() % (s.size() + 1));
        if (rng() % 2) g.qp = g.sp < g.qa ? g.sp : g.qa;
        g.tbq = (uint32_t)i;
        g.tbs = (uint32_t)i * 3;
        g.xdrop = (uint32_t)xs[rng() % 8];
        const bool plus = rng() % 2;
        const uint8_t* sp = (const uint8_t*)g.sseq;
        const uint8_t al = g.sp > 0 ? sp[g.sp - 1] : 0, ar = g.sa > g.sp ? sp[g.sp] : 0;
        g.flags = (plus ? 1u : 0u) | ((uint32_t)al << 8) | ((uint32_t)ar << 16);
    }

    // the kernel's score table: clamped below at -(X + 1) for the largest X
    int32_t smat[256];
    for (int a = 0; a < 16; ++a)
        for (int b = 0; b < 16; ++b) smat[a * 16 + b] = mat.s[a][b] > -301 ? mat.s[a][b] : -301;
    std::vector<rmb::PrelimOut> out(n);
    std::vector<uint32_t> overflow;
    uint32_t queue = 0;
    const rmb::StreamArgs A{smat, ge, go + ge, cutoff, (uint64_t)n, geo.data(), out.data(), max_cells};
    unsigned long long cells = 0;
    for (int th = 0; th < 3; ++th) {  // three threads take records from one queue in turn
        HostEnv env;
        env.queue = &queue;
        env.overflow_list = &overflow;
        for (auto& r : env.ring) r = 0xdeadbeefu;  // slots are written before they are read
        cells += rmb::prelim_stream_thread<8>(A, env);
    }

    std::vector<char> listed(n, 0);
    for (uint32_t t : overflow) listed[t] = 1;
    int bad = 0, checked = 0, big = 0;
    unsigned long long ocells = 0;
    for (int i = 0; i < n; ++i) {
        if (listed[i]) continue;
        const rmb::PrelimGeo& g = geo[i];
        const uint8_t* sa = (const uint8_t*)g.sseq;
        const uint8_t* qa = (const uint8_t*)g.qseq;
        // engine.rs:1350-1397: left extension (reversed) from the pivot, then the right one
        const rmbo::ScoreOnly l = rmbo::align_ex_score_only(sa, qa, g.sp, g.qp, go, ge, (int)g.xdrop, mat, true);
        rmbo::ScoreOnly r{0, 0, 0, 0};
        if (g.sa > g.sp && g.qa > g.qp)
            r = rmbo::align_ex_score_only(sa + g.sp, qa + g.qp, g.sa - g.sp, g.qa - g.qp, go, ge, (int)g.xdrop, mat,
                                          false);
        ocells += l.cells + r.cells;
        ++checked;
        if (l.score > 4300 || r.score > 4300) ++big;  // past the origin move
        const int32_t total = l.score + r.score;
        rmb::PrelimOut want{INT32_MIN, 0, 0, 0, 0, 0, 0};
        if (total >= 0 && total >= cutoff) {
            uint32_t q0 = g.qp - l.b_len, s0 = g.sp - l.a_len, q1 = g.qp + r.b_len, s1 = g.sp + r.a_len;
            if (!(g.flags & 1u)) {
                const uint32_t t0 = g.qa - q1, t1 = g.qa - q0, t2 = g.sa - s1, t3 = g.sa - s0;
                q0 = t0; q1 = t1; s0 = t2; s1 = t3;
            }
            want = rmb::PrelimOut{total, q0, q1, s0, s1, g.tbq, g.tbs};
        }
        if (memcmp(&want, &out[i], sizeof want) != 0) {
            if (bad < 5)
                fprintf(stderr, "record %d: want %d %u-%u %u-%u got %d %u-%u %u-%u\n", i, want.score, want.q_start,
                        want.q_end, want.s_start, want.s_end, out[i].score, out[i].q_start, out[i].q_end,
                        out[i].s_start, out[i].s_end);
            ++bad;
        }
    }
    printf("records %d checked %d overflow %zu bad %d cells %llu oracle_cells %llu big %d\n", n, checked,
           overflow.size(), bad, cells, ocells, big);
    return bad != 0;
}
