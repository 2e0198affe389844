// rmb_dust.cuh -- NCBI symmetric DUST query masking (filter/dust.rs:15-331, 462-489), as code that
// compiles for the device and for the host.
//
// One query is one sequential pass, as in the reference: the pass draws NCBI CRandom numbers for
// N bases in order (dust.rs:24-57, 339-360) and restarts a window scan from the last window start
// after each low-complexity run (dust.rs:400-460), so the masked positions depend on the whole
// prefix.  The device runs one query per warp (one working lane); the queries of a batch run in
// parallel.
//
// Storage differs from the reference's growable vectors, not the results:
//  - the triplet list (at most window - 2 = 62 entries) is a 64-entry ring;
//  - the "perfect interval" list is a ring over caller scratch of DUST_PERFECT_CAP entries, with
//    O(1) front insertion and back removal.  Entries leave it once the window start passes them
//    and each step adds at most one per window position, so it never holds more than 62 x 62 =
//    3,844; the pass still reports an overflow instead of dropping entries;
//  - the base conversion (N -> random base) of positions j .. j+2 is kept in an 8-entry ring:
//    like the reference, each window restart converts again from its start.
#pragma once
#include <cstdint>

#ifdef __CUDACC__
#define RMB_HD __host__ __device__ __forceinline__
#else
#define RMB_HD inline
#endif

namespace rmb {

constexpr uint32_t DUST_WINDOW = 64, DUST_LEVEL = 20, DUST_LINKER = 1;
constexpr uint32_t DUST_PERFECT_CAP = 4096;  // power of two

struct DustPerfect {
    uint32_t start, stop, score, len;
};

// NCBI CRandom with the fixed initial state DUST uses (dust.rs:24-57); same table and steps as the
// reference, since the masked positions of N-containing windows depend on this exact stream.
struct DustRng {
    uint32_t st[33];
    int rk, rj;
    RMB_HD void init() {
        const uint32_t s0[33] = {0xd53f1852u, 0xdfc78b83u, 0x4f256096u, 0x0e643df7u, 0x82c359bfu, 0xc7794dfau,
                                 0xd5e9ffaau, 0x2c8cb64au, 0x2f07b334u, 0xad5a7eb5u, 0x96dc0cdeu, 0x6fc24589u,
                                 0xa5853646u, 0xe71576e2u, 0x0dae30dfu, 0xb09ce711u, 0x5e56ef87u, 0x4b4b0082u,
                                 0x6f4f340eu, 0xc5bb17e8u, 0xd788d765u, 0x67498087u, 0x9d7aba26u, 0x261351d4u,
                                 0x411ee7eau, 0x0393a263u, 0x2c5a5835u, 0xc115fcd8u, 0x25e9132cu, 0xd0c6e906u,
                                 0xc2bc5b2du, 0x6c065c98u, 0x6e37bd55u};
        for (int i = 0; i < 33; ++i) st[i] = s0[i];
        rk = 32;
        rj = 12;
    }
    RMB_HD uint32_t get() {
        const uint32_t r = st[rk] + st[rj];
        st[rk] = r;
        --rk;
        --rj;
        if (rk < 0) rk = 32;
        else if (rj < 0) rj = 32;
        return r >> 1;
    }
};

// dust.rs:62-75: A, C, G, T -> 0..3, N -> a random base, every other code -> 0
RMB_HD uint8_t dust_cvt(uint8_t b, DustRng& rng) {
    switch (b) {
        case 1: return 1;
        case 2: return 2;
        case 3: return 3;
        case 14: return (uint8_t)(rng.get() & 3u);
        default: return 0;
    }
}

struct DustPerfectList {  // logical 0 = front (newest), size - 1 = back (oldest)
    DustPerfect* buf;
    uint32_t head, size;
    bool overflow;
    RMB_HD DustPerfect& at(uint32_t i) { return buf[(head + i) & (DUST_PERFECT_CAP - 1)]; }
    RMB_HD void insert(uint32_t pos, const DustPerfect& v) {  // before logical index pos
        if (size == DUST_PERFECT_CAP) {
            overflow = true;
            return;
        }
        head = (head - 1) & (DUST_PERFECT_CAP - 1);
        for (uint32_t i = 0; i < pos; ++i) at(i) = at(i + 1);
        at(pos) = v;
        ++size;
    }
    RMB_HD void clear() { size = 0; }
};

// dust.rs:95-274 triplet window
struct DustTriplets {
    uint8_t list[64];  // logical 0 = newest
    uint32_t lhead, lsize;
    uint8_t c_w[64], c_v[64];
    uint32_t r_w, r_v, num_diff;
    uint32_t max_size, low_k;
    uint32_t start, stop, l;

    RMB_HD void init(uint32_t js) {
        lhead = 0;
        lsize = 0;
        for (int i = 0; i < 64; ++i) c_w[i] = c_v[i] = 0;
        r_w = r_v = num_diff = 0;
        max_size = DUST_WINDOW - 2;
        low_k = DUST_LEVEL / 5;
        start = stop = l = js;
    }
    RMB_HD uint8_t item(uint32_t i) const { return list[(lhead + i) & 63u]; }
    RMB_HD uint8_t pop_back() { return list[(lhead + --lsize) & 63u]; }
    RMB_HD void push_front(uint8_t t) {
        lhead = (lhead - 1) & 63u;
        list[lhead] = t;
        ++lsize;
    }
    RMB_HD void add_w(uint8_t t) {
        if (c_w[t] == 0) ++num_diff;
        r_w += c_w[t];
        ++c_w[t];
    }
    RMB_HD void rem_w(uint8_t t) {
        --c_w[t];
        if (c_w[t] == 0) --num_diff;
        r_w -= c_w[t];
    }
    RMB_HD void add_v(uint8_t t) {
        r_v += c_v[t];
        ++c_v[t];
    }
    RMB_HD void rem_v(uint8_t t) {
        --c_v[t];
        r_v -= c_v[t];
    }
    RMB_HD bool shift_high(uint8_t t, DustPerfectList& perfect) {
        const uint8_t s = pop_back();
        rem_w(s);
        ++start;
        push_front(t);
        add_w(t);
        ++stop;
        if (num_diff <= 1) {
            perfect.insert(0, DustPerfect{start, stop + 1, 0, 0});
            return false;
        }
        return true;
    }
    RMB_HD bool shift_window(uint8_t t, DustPerfectList& perfect) {
        if (lsize >= max_size) {
            if (num_diff <= 1) return shift_high(t, perfect);
            const uint8_t s = pop_back();
            rem_w(s);
            if (l == start) {
                ++l;
                rem_v(s);
            }
            ++start;
        }
        push_front(t);
        add_w(t);
        add_v(t);
        if (c_v[t] > low_k) {
            uint32_t idx = lsize - (l - start) - 1;
            for (;;) {
                const uint8_t s = item(idx);
                rem_v(s);
                ++l;
                if (s == t) break;
                if (idx == 0) break;
                --idx;
            }
        }
        ++stop;
        if (lsize >= max_size && num_diff <= 1) {
            perfect.clear();
            perfect.insert(0, DustPerfect{start, stop + 1, 0, 0});
            return false;
        }
        return true;
    }
    static RMB_HD uint32_t threshold(uint32_t count) { return count ? count * DUST_LEVEL : 1u; }
    RMB_HD bool needs_processing() const {
        const uint32_t count = stop - l;
        return count < lsize && r_w * 10 > threshold(count);
    }
    RMB_HD void find_perfect(DustPerfectList& perfect) const {
        uint8_t counts[64];
        for (int i = 0; i < 64; ++i) counts[i] = c_v[i];
        uint32_t score = r_v;
        uint32_t count = stop - l;
        uint32_t it = 0;
        uint32_t max_score = 0, max_len = 0;
        for (uint32_t idx = stop - l; idx < lsize; ++idx) {
            const uint8_t ti = item(idx);
            const uint32_t cnt = counts[ti];
            score += cnt;
            counts[ti] = (uint8_t)(cnt + 1);
            if (cnt > 0 && score * 10 > threshold(count)) {
                const uint32_t pos = stop - idx - 1;
                while (it < perfect.size && pos <= perfect.at(it).start) {
                    const DustPerfect& pi = perfect.at(it);
                    if (max_score == 0 || max_len * pi.score > max_score * pi.len) {
                        max_score = pi.score;
                        max_len = pi.len;
                    }
                    ++it;
                }
                if (max_score == 0 || score * max_len >= max_score * count) {
                    max_score = score;
                    max_len = count;
                    perfect.insert(it, DustPerfect{pos, stop + 1, max_score, count});
                }
            }
            ++count;
        }
    }
};

// dust.rs:284-331 result list: only its last interval is ever extended, so an interval is final
// (and masked) once the next one starts
struct DustMasker {
    uint8_t* out;    // masked copy of the query bases (no sentinel), length n; or null
    uint32_t* bits;  // or null: bit p set for every position inside an interval (the plain
                     // intervals, which pairwise output prints in lower case)
    uint32_t n;
    bool compat;     // the multi-chunk path's off-by-one: also mask e + 1 (dust.rs:614-630)
    bool has;
    uint32_t cs, ce;
    RMB_HD void flush() {
        if (!has) return;
        const uint32_t end = ce < n - 1 ? ce : n - 1;
        for (uint32_t p = cs; p <= end; ++p) {
            if (out) out[p] = 14;
            if (bits) bits[p >> 5] |= 1u << (p & 31);
        }
        if (out && compat && ce + 1 < n) out[ce + 1] = 14;
    }
    RMB_HD void save(DustPerfectList& perfect, uint32_t wstart) {
        if (perfect.size == 0) return;
        const DustPerfect& b = perfect.at(perfect.size - 1);
        const uint32_t b0 = b.start, b1 = b.stop;
        if (b0 < wstart) {
            if (has && ce + DUST_LINKER >= b0) {
                if (b1 > ce) ce = b1;
            } else {
                flush();
                has = true;
                cs = b0;
                ce = b1;
            }
            while (perfect.size && perfect.at(perfect.size - 1).start < wstart) --perfect.size;
        }
    }
};

// dust.rs:339-460 + 462-489 for one query: masks the low-complexity intervals of bases[0..n) in
// out[0..n) (out holds a copy of bases); `compat` adds the multi-chunk path's extra base after
// each interval (dust.rs:614-630).  `scratch` holds DUST_PERFECT_CAP entries.  Returns false
// if the perfect list would have outgrown its ring (then `out` is incomplete).
RMB_HD bool dust_query(const uint8_t* bases, uint32_t n, uint8_t* out, DustPerfect* scratch, bool compat = false,
                       uint32_t* bits = nullptr) {
    if (n < 3) return true;
    DustRng rng;
    rng.init();
    DustPerfectList perfect{scratch, 0, 0, false};
    DustMasker mk{out, bits, n, compat, false, 0, 0};
    DustTriplets w;
    uint8_t conv[8];
    uint32_t j_start = 0;
    for (;;) {
        if ((uint64_t)n < (uint64_t)j_start + 4) break;
        perfect.clear();
        w.init(j_start);
        const uint32_t j_end = n - 2;
        uint32_t j = j_start, conv_from = j_start;
        for (;;) {
            if (j >= j_end) break;
            mk.save(perfect, w.start);
            while (conv_from <= j + 2) {
                conv[conv_from & 7u] = dust_cvt(bases[conv_from], rng);
                ++conv_from;
            }
            const uint8_t t = (uint8_t)((conv[j & 7u] << 4) | (conv[(j + 1) & 7u] << 2) | conv[(j + 2) & 7u]);
            ++j;
            if (w.shift_window(t, perfect)) {
                if (w.needs_processing()) w.find_perfect(perfect);
            } else {
                for (;;) {
                    if (j >= j_end) break;
                    mk.save(perfect, w.start);
                    while (conv_from <= j + 2) {
                        conv[conv_from & 7u] = dust_cvt(bases[conv_from], rng);
                        ++conv_from;
                    }
                    const uint8_t t2 =
                        (uint8_t)((conv[j & 7u] << 4) | (conv[(j + 1) & 7u] << 2) | conv[(j + 2) & 7u]);
                    if (w.shift_window(t2, perfect)) break;
                    ++j;
                }
                break;
            }
            if (perfect.overflow) return false;
        }
        if (perfect.overflow) return false;
        uint32_t wstart = w.start;
        while (perfect.size) {
            mk.save(perfect, wstart);
            ++wstart;
        }
        if (w.start > j_start) j_start = w.start;
        else break;
    }
    mk.flush();
    return !perfect.overflow;
}

}  // namespace rmb
