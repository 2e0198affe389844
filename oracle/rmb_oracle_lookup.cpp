// rmb_oracle_lookup.cpp -- query lookup tables and subject scanners.
// TEST INFRASTRUCTURE: the CPU oracle.  See rmb_oracle.hpp.
#include "rmb_oracle.hpp"

#include <stdexcept>

namespace rmbo {

// blast/nalookup.rs:254-291
int choose_lut_width(int ws, size_t e) {
    if (ws >= 4 && ws <= 6) return ws;
    switch (ws) {
        case 7: return e < 250 ? 6 : 7;
        case 8: return e < 8500 ? 7 : 8;
        case 9: return e < 1250 ? 7 : e < 21000 ? 8 : 9;
        case 10: return e < 1250 ? 7 : e < 8500 ? 8 : e < 18000 ? 9 : 10;
        case 11: return e < 12000 ? 8 : e < 180000 ? 10 : 11;
        case 12: return e < 8500 ? 8 : e < 18000 ? 9 : e < 60000 ? 10 : e < 900000 ? 11 : 12;
        default: break;
    }
    if (ws >= 13) return e < 8500 ? 8 : e < 300000 ? 11 : 12;
    throw std::runtime_error("word_size below the minimum of 4");
}

// blast/nalookup.rs:128-181 (index) + 187-246 (finalize) + 301-335 (new)
static void build_na(Lookup& L, const std::vector<uint8_t>& q, const std::vector<std::pair<int, int>>& locs,
                     int wl, int lw) {
    int32_t backbone = 1 << (2 * lw);
    L.mega = false;
    L.mask = backbone - 1;
    L.word_length = wl;
    L.lut_word_length = lw;
    L.scan_step = wl - lw + 1;
    std::vector<std::vector<int32_t>> thin(backbone);
    auto add = [&](int start) {
        int32_t idx = 0;
        for (int k = 0; k < lw; ++k) idx = (idx << 2) | q[start + k];
        thin[idx].push_back(start);
    };
    for (auto [from, to] : locs) {
        if (wl > to - from + 1) continue;
        int word_target = lw, i = 0;
        while (from + i <= to) {
            uint8_t b = q[from + i];
            if (i >= word_target) add(from + i - lw);
            if (b & 0xFC) word_target = i + lw + 1;
            ++i;
        }
        if (i >= word_target) add(from + i - lw);
    }
    L.num_used.assign(backbone, 0);
    L.cell_entries.assign((size_t)backbone * 3, 0);
    L.cell_cursor.assign(backbone, 0);
    L.pv.assign((backbone >> 5) + 1, 0);
    int longest = 0;
    int32_t cursor = 0;
    L.overflow.clear();
    for (int32_t i = 0; i < backbone; ++i) {
        if (thin[i].empty()) continue;
        int n = (int)thin[i].size();
        longest = std::max(longest, n);
        L.num_used[i] = n;
        L.pv[i >> 5] |= 1u << (i & 31);
        if (n <= 3) {
            for (int k = 0; k < n; ++k) L.cell_entries[(size_t)i * 3 + k] = thin[i][k];
        } else {
            L.cell_cursor[i] = cursor;
            for (int k = 0; k < n; ++k) L.overflow.push_back(thin[i][k]);
            cursor += n;
        }
    }
    L.longest_chain = longest;
}

// blast/mblookup.rs:106-235
static void build_mb(Lookup& L, const std::vector<uint8_t>& q, const std::vector<std::pair<int, int>>& locs,
                     int wl, int lw, size_t approx) {
    L.mega = true;
    L.word_length = wl;
    L.lut_word_length = lw;
    L.scan_step = wl - lw + 1;
    L.hashsize = (int64_t)1 << (2 * lw);
    int64_t pv_size = L.hashsize <= 8 * 131072 ? (L.hashsize >> 5) : 131072 / 4;
    if (approx <= 15000 || approx >= 800000) pv_size /= 2;
    uint64_t ratio = (uint64_t)(L.hashsize / pv_size);
    L.pv_bts = 63 - __builtin_clzll(ratio);
    L.hashtable.assign((size_t)L.hashsize, 0);
    L.next_pos.assign(q.size() + 1, 0);
    L.pv.assign((size_t)pv_size, 0);
    int64_t mask = L.hashsize - 1;
    size_t helper_len = std::max<size_t>((size_t)L.hashsize / 2048, 1);
    std::vector<uint32_t> helper(helper_len, 0);
    for (auto [left, right] : locs) {
        if (wl > right - left + 1) continue;
        int64_t ecode = 0;
        size_t valid_from = (size_t)left + lw - 1;
        for (size_t rp = (size_t)left; rp <= (size_t)right; ++rp) {
            uint8_t base = q[rp];
            if (base & 0xFC) {
                ecode = 0;
                valid_from = rp + lw;
                continue;
            }
            ecode = ((ecode << 2) & mask) | base;
            if (rp < valid_from) continue;
            int32_t q1 = (int32_t)(rp + 2 - lw);
            if (L.hashtable[ecode] == 0) L.pv[ecode >> L.pv_bts] |= 1u << (ecode & 31);
            else helper[ecode / 2048] += 1;
            L.next_pos[q1] = L.hashtable[ecode];
            L.hashtable[ecode] = q1;
        }
    }
    uint32_t longest = 0;
    for (uint32_t h : helper) longest = std::max(longest, h);
    L.longest_chain = std::max<int>((int)longest, 2);
}

// engine.rs:606-649 build_query_lookup / combined_lookup
QueryLookup build_query_lookup(const std::vector<uint8_t>& query, const Params& p) {
    QueryLookup ql;
    ql.masked = query;
    if (p.dust) dust_mask(ql.masked);
    size_t n = query.size() - 2;
    ql.fwd_n = (uint32_t)n;
    ql.c1_start = (uint32_t)n + 1;
    std::vector<uint8_t> comb;
    comb.reserve(2 * n + 1);
    comb.insert(comb.end(), ql.masked.begin() + 1, ql.masked.begin() + 1 + n);
    comb.push_back(14);
    auto rc = revcomp(ql.masked.data() + 1, n);
    comb.insert(comb.end(), rc.begin(), rc.end());
    std::vector<std::pair<int, int>> locs = {{0, (int)n - 1}, {(int)n + 1, 2 * (int)n}};
    size_t approx = 2 * n;
    int lw = choose_lut_width(p.word_size, approx);
    if (lw > 8) build_mb(ql.lut, comb, locs, p.word_size, lw, approx);
    else build_na(ql.lut, comb, locs, p.word_size, lw);
    ql.query_rc = revcomp(query.data(), query.size());
    return ql;
}

// ---- scanners ---------------------------------------------------------------------------
// blast/nascan.rs:41-82 get_num_hits / retrieve
static inline int na_num_hits(const Lookup& L, int32_t idx) {
    return (L.pv[idx >> 5] & (1u << (idx & 31))) ? L.num_used[idx] : 0;
}
static inline void na_retrieve(const Lookup& L, int32_t idx, OffsetPair* out, int32_t s_off) {
    int n = L.num_used[idx];
    const int32_t* src = n <= 3 ? &L.cell_entries[(size_t)idx * 3] : &L.overflow[L.cell_cursor[idx]];
    for (int i = 0; i < n; ++i) out[i] = OffsetPair{(uint32_t)src[i], (uint32_t)s_off};
}

// nascan.rs:72-261 and mblookup.rs:247-343.  `packed` points at the first packed base byte.
int Lookup::scan(const uint8_t* s, OffsetPair* out, int max_hits, int32_t range[2]) const {
    int total = 0;
    const int lw = lut_word_length, step = scan_step;
    if (!mega) {
        if (lw == 8 && step == 4) {  // nascan.rs:72-108
            size_t sb = range[0] / 4, se = range[1] / 4;
            while (sb <= se) {
                int32_t idx = ((int32_t)s[sb] << 8) | s[sb + 1];
                int nh = na_num_hits(*this, idx);
                if (nh == 0) { ++sb; continue; }
                if (nh > max_hits - total) break;
                na_retrieve(*this, idx, out + total, (int32_t)sb * 4);
                total += nh;
                ++sb;
            }
            range[0] = (int32_t)sb * 4;
            return total;
        }
        if (lw > 5) {
            if (step % 4 == 0) {  // nascan.rs:142-175
                int shift = 2 * (8 - lw);
                size_t bstep = step / 4, sb = range[0] / 4, se = range[1] / 4;
                while (sb <= se) {
                    int32_t raw = ((int32_t)s[sb] << 8) | s[sb + 1];
                    int32_t idx = raw >> shift;
                    int nh = na_num_hits(*this, idx);
                    if (nh == 0) { sb += bstep; continue; }
                    if (nh > max_hits - total) break;
                    na_retrieve(*this, idx, out + total, (int32_t)sb * 4);
                    total += nh;
                    sb += bstep;
                }
                range[0] = (int32_t)sb * 4;
            } else {  // nascan.rs:177-204
                while (range[0] <= range[1]) {
                    int32_t so = range[0];
                    int shift = 2 * (12 - (so % 4 + lw));
                    size_t sb = so / 4;
                    int32_t raw = ((int32_t)s[sb] << 16) | ((int32_t)s[sb + 1] << 8) | s[sb + 2];
                    int32_t idx = (raw >> shift) & mask;
                    int nh = na_num_hits(*this, idx);
                    if (nh == 0) { range[0] += step; continue; }
                    if (nh > max_hits - total) break;
                    na_retrieve(*this, idx, out + total, so);
                    total += nh;
                    range[0] += step;
                }
            }
        } else {  // nascan.rs:208-238
            while (range[0] <= range[1]) {
                int32_t so = range[0];
                int shift = 2 * (8 - (so % 4 + lw));
                size_t sb = so / 4;
                int32_t raw = ((int32_t)s[sb] << 8) | s[sb + 1];
                int32_t idx = (raw >> shift) & mask;
                int nh = na_num_hits(*this, idx);
                if (nh == 0) { range[0] += step; continue; }
                if (nh > max_hits - total) break;
                na_retrieve(*this, idx, out + total, so);
                total += nh;
                range[0] += step;
            }
        }
        return total;
    }
    // megablast scanner, mblookup.rs:247-343
    int mh = max_hits - longest_chain;
    int64_t msk = hashsize - 1;
    auto has = [&](int64_t idx) { return (pv[idx >> pv_bts] & (1u << (idx & 31))) != 0; };
    auto retrieve = [&](int64_t idx, OffsetPair* o, int32_t so) {
        int i = 0;
        int32_t q = hashtable[idx];
        while (q != 0) {
            o[i++] = OffsetPair{(uint32_t)(q - 1), (uint32_t)so};
            q = next_pos[q];
        }
        return i;
    };
    if (step % 4 == 0) {
        uint32_t shift = 2 * (12 - lw);
        size_t bstep = step / 4, sb = range[0] / 4, se = range[1] / 4;
        while (sb <= se) {
            uint32_t raw = ((uint32_t)s[sb] << 16) | ((uint32_t)s[sb + 1] << 8) | s[sb + 2];
            int64_t idx = raw >> shift;
            if (has(idx)) {
                if (total >= mh) break;
                total += retrieve(idx, out + total, (int32_t)sb * 4);
            }
            sb += bstep;
        }
        range[0] = (int32_t)sb * 4;
    } else if (lw > 9) {
        while (range[0] <= range[1]) {
            int32_t so = range[0];
            size_t sb = so / 4;
            uint32_t shift = 2 * (16 - (so % 4 + lw));
            uint32_t raw = ((uint32_t)s[sb] << 24) | ((uint32_t)s[sb + 1] << 16) | ((uint32_t)s[sb + 2] << 8) |
                           s[sb + 3];
            int64_t idx = (int64_t)(raw >> shift) & msk;
            if (has(idx)) {
                if (total >= mh) break;
                total += retrieve(idx, out + total, so);
            }
            range[0] += step;
        }
    } else {
        while (range[0] <= range[1]) {
            int32_t so = range[0];
            size_t sb = so / 4;
            uint32_t shift = 2 * (12 - (so % 4 + lw));
            uint32_t raw = ((uint32_t)s[sb] << 16) | ((uint32_t)s[sb + 1] << 8) | s[sb + 2];
            int64_t idx = (int64_t)(raw >> shift) & msk;
            if (has(idx)) {
                if (total >= mh) break;
                total += retrieve(idx, out + total, so);
            }
            range[0] += step;
        }
    }
    return total;
}

}  // namespace rmbo
