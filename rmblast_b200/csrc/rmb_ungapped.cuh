#pragma once
// The ungapped X-drop extension of one word hit (search/ungapped.rs:38-121) as a resumable walk:
// the left walk from the seed, then the right walk, one base a step.  k_ungapped keeps one walk
// per lane and refills lanes whose walk is done; the same code built for the host is checked
// against the oracle's extension.
#include <cstdint>

namespace rmb {

struct UngWalk {
    const uint8_t* qb = nullptr;  // sentinel-wrapped query in the walk's strand frame (base q at qb[1 + q])
    const uint8_t* sb = nullptr;  // sentinel-wrapped plus-strand subject
    int32_t q = 0, s = 0, qlim = 0, slim = 0, dir = -1;
    int32_t sum = 0, score = 0, x = 0, xc = 0, best = 0, q_beg = 0;
    int32_t wq = 0, wsx = 0, qlen = 0, slen = 0;

    // From the seed (wq, wsx) with X-drop xdrop: the left walk first.
    __host__ __device__ __forceinline__ void start(const uint8_t* query, const uint8_t* subject, int32_t query_len,
                                                   int32_t subject_len, int32_t seed_q, int32_t seed_s, int32_t xdrop) {
        qb = query;
        sb = subject;
        qlen = query_len;
        slen = subject_len;
        wq = seed_q;
        wsx = seed_s;
        x = -xdrop;
        q = wq - 1; s = wsx - 1; dir = -1; qlim = -1; slim = -1;
        sum = 0; score = 0; xc = x; best = wq;
    }

    // One base: the walk's step on query base a and subject base c at (q, s), or its end when
    // at_end (q or s at its limit).  Returns 0 while walking, 1 when the left walk ended (the
    // right one starts at the seed), 2 when the right walk ended (the extension is done).
    __host__ __device__ __forceinline__ int on_base(bool at_end, uint8_t a, uint8_t c, const int32_t* mat) {
        bool stop = at_end;
        if (!stop) {
            if (a == 15 || c == 15) {
                stop = true;
            } else {
                sum += mat[((a & 15) << 4) | (c & 15)];
                if (sum > 0) {
                    best = dir < 0 ? q : q + 1;
                    score += sum;
                    if (dir > 0) xc = -score > x ? -score : x;
                    sum = 0;
                } else if (sum < xc) {
                    stop = true;
                }
            }
        }
        if (!stop) {
            q += dir;
            s += dir;
            return 0;
        }
        if (dir < 0) {
            q_beg = best;
            q = wq; s = wsx; dir = 1; qlim = qlen; slim = slen;
            sum = 0; xc = x; best = wq;
            return 1;
        }
        return 2;
    }

    // One base, as on_base.
    __host__ __device__ __forceinline__ int step(const int32_t* mat) {
        const bool end = q == qlim || s == slim;
        return on_base(end, end ? (uint8_t)15 : qb[1 + q], end ? (uint8_t)15 : sb[1 + s], mat);
    }

    // After step() returned 2: the extension in the walk's frame.
    __host__ __device__ __forceinline__ void result(int32_t& sc, uint32_t& q0, uint32_t& q1, uint32_t& s0,
                                                    uint32_t& s1) const {
        sc = score;
        q0 = (uint32_t)q_beg;
        q1 = (uint32_t)best;
        s0 = (uint32_t)(wsx - (wq - q_beg));
        s1 = (uint32_t)(wsx + (best - wq));
    }
};

}  // namespace rmb
