// rmb_oracle_engine.cpp -- the per-pair pipeline and the per-query steps.
// TEST INFRASTRUCTURE: the CPU oracle.  See rmb_oracle.hpp.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <map>
#include <mutex>
#include <stdexcept>
#include <thread>
#include <atomic>

#include "rmb_oracle.hpp"
#include "rmb_oracle_itree.hpp"

namespace rmbo {

namespace {
constexpr int64_t MIN_DIAG_SEP = 50;  // engine.rs:173

// search/diag_hash.rs:15-111
struct DiagHash {
    struct Cell { int32_t diag; uint32_t level, next; };
    uint32_t backbone[512];
    std::vector<Cell> chain;
    uint32_t occ = 1;
    DiagHash() : chain(257, Cell{0, 0, 0}) { std::fill(backbone, backbone + 512, 0u); }
    static size_t bucket(int32_t d) { return (size_t)(((uint32_t)d * 0x9E370001u) % 512u); }
    uint32_t get(int32_t d) const {
        uint32_t i = backbone[bucket(d)];
        while (i) {
            if (chain[i].diag == d) return chain[i].level;
            i = chain[i].next;
        }
        return 0;
    }
    void insert(int32_t d, uint32_t s_end, uint32_t s_off, int32_t window) {
        size_t b = bucket(d);
        uint32_t i = backbone[b];
        while (i) {
            Cell& c = chain[i];
            if (c.diag == d) { c.level = s_end; return; }
            if ((int32_t)(s_off - c.level) > window) { c.diag = d; c.level = s_end; return; }
            i = c.next;
        }
        if (occ >= chain.size()) chain.push_back(Cell{0, 0, 0});
        chain[occ] = Cell{d, s_end, backbone[b]};
        backbone[b] = occ;
        ++occ;
    }
};

struct UngappedRecord {  // engine.rs:138-154
    uint32_t q_seed, s_seed, q_start, q_end, s_start, s_end;
    int32_t score;
    Strand strand;
};

// engine.rs:1063-1277 collect_ungapped_combined
void collect_ungapped(const std::vector<uint8_t>& query, const QueryLookup& ql, const Subject& subj,
                      const Params& p, const Matrix& m, std::vector<SeedRecord>* seed_out,
                      std::vector<UngappedRecord>& out, Counters* ctr) {
    const std::vector<uint8_t>& ext_q = ql.masked;
    const uint8_t* splus = subj.plus.data();
    const uint8_t* src = subj.rc.data();
    const size_t s_real = subj.plus.size() - 2;
    const int64_t lw = ql.lut.lut_word_length;
    int64_t er = (int64_t)s_real - lw;
    if (er < 0) return;
    const int32_t end_range = (int32_t)er;
    const int64_t ext_needed = (int64_t)p.word_size - lw;
    const int64_t q_real_len = (int64_t)query.size() - 2;
    const int64_t s_real_len = (int64_t)s_real;
    const uint32_t s_len = (uint32_t)s_real, q_len = (uint32_t)q_real_len;
    const int32_t ucut = p.ungapped_cutoff >= 0 ? p.ungapped_cutoff : p.cutoff_score_max();
    const int64_t c1 = ql.c1_start, fn = ql.fwd_n;
    const size_t batch = std::max<size_t>(4096, (size_t)ql.lut.longest_chain + 4096);
    std::vector<OffsetPair> pairs(batch);
    DiagHash dh;
    const int32_t window = 1 - p.word_size;
    int32_t range[2] = {0, end_range};
    for (;;) {
        int n = ql.lut.scan(subj.packed.data() + 3, pairs.data(), (int)batch, range);
        if (ctr) ctr->word_hits += (uint64_t)n;
        for (int i = 0; i < n; ++i) {
            const int64_t q0c = pairs[i].q_off, s_fwd = pairs[i].s_off;
            if (q0c < c1) {
                uint32_t q_off = pairs[i].q_off, s_off = pairs[i].s_off;
                if (ext_needed > 0) {
                    int64_t el = 0;
                    while (el < ext_needed) {
                        int64_t qi = q0c - el - 1, si = s_fwd - el - 1;
                        if (qi < 0 || si < 0) break;
                        uint8_t qb = ext_q[1 + qi], sb = splus[1 + si];
                        if (qb >= 4 || sb >= 4 || qb != sb) break;
                        ++el;
                    }
                    int64_t er2 = 0;
                    while (el + er2 < ext_needed) {
                        int64_t qi = q0c + lw + er2, si = s_fwd + lw + er2;
                        if (qi >= q_real_len || si >= s_real_len) break;
                        uint8_t qb = ext_q[1 + qi], sb = splus[1 + si];
                        if (qb >= 4 || sb >= 4 || qb != sb) break;
                        ++er2;
                    }
                    if (el + er2 < ext_needed) continue;
                    q_off = (uint32_t)(q0c - el);
                    s_off = (uint32_t)(s_fwd - el);
                }
                int32_t diag = (int32_t)(s_off - q_off);
                uint32_t last = dh.get(diag);
                if (s_off < last) continue;
                if (seed_out) seed_out->push_back(SeedRecord{q_off, s_off, PLUS});
                if (ctr) ctr->seeds++;
                UngappedResult u = extend_ungapped(query.data(), query.size(), splus, subj.plus.size(), q_off, s_off,
                                                   m, p.xdrop_ungap);
                uint32_t store = u.score >= ucut ? u.s_end : s_off + (uint32_t)p.word_size;
                dh.insert(diag, store, s_off, window);
                if (u.score < ucut) continue;
                if (ctr) ctr->ungapped++;
                out.push_back(UngappedRecord{q_off, s_off, u.q_start, u.q_end, u.s_start, u.s_end, u.score, PLUS});
            } else {
                const int64_t rcq = q0c - c1;
                const int64_t q0 = fn - rcq - lw, s0 = s_real_len - s_fwd - lw;
                if (q0 < 0 || s0 < 0) continue;
                uint32_t q_off = (uint32_t)q0, s_off = (uint32_t)s0;
                if (ext_needed > 0) {
                    int64_t er2 = 0;
                    while (er2 < ext_needed) {
                        int64_t qi = q0 + lw + er2, si = s0 + lw + er2;
                        if (qi >= q_real_len || si >= s_real_len) break;
                        uint8_t qb = ext_q[1 + qi], sb = src[1 + si];
                        if (qb >= 4 || sb >= 4 || qb != sb) break;
                        ++er2;
                    }
                    int64_t el = 0;
                    while (el + er2 < ext_needed) {
                        int64_t qi = q0 - el - 1, si = s0 - el - 1;
                        if (qi < 0 || si < 0) break;
                        uint8_t qb = ext_q[1 + qi], sb = src[1 + si];
                        if (qb >= 4 || sb >= 4 || qb != sb) break;
                        ++el;
                    }
                    if (el + er2 < ext_needed) continue;
                    q_off = (uint32_t)(q0 + er2);
                    s_off = (uint32_t)(s0 + er2);
                }
                int32_t diag = (int32_t)((uint32_t)s_fwd - (uint32_t)q0c);
                uint32_t s_fwd_eff = s_len - s_off - (uint32_t)lw;
                uint32_t fwd_s_end = s_fwd_eff + (uint32_t)p.word_size;
                uint32_t last = dh.get(diag);
                if (s_fwd_eff < last) continue;
                uint32_t en = ext_needed > 0 ? (uint32_t)ext_needed : 0;
                uint32_t q_seed = q_off >= en ? q_off - en : 0;
                uint32_t sl = s_off + (uint32_t)lw;
                uint32_t s_seed = s_len >= sl ? s_len - sl : 0;
                if (seed_out) seed_out->push_back(SeedRecord{q_seed, s_seed, MINUS});
                if (ctr) ctr->seeds++;
                uint32_t qn = q_len - 1 - q_off, sn = s_len - 1 - s_off;
                UngappedResult u = extend_ungapped(ql.query_rc.data(), ql.query_rc.size(), splus, subj.plus.size(),
                                                   qn, sn, m, p.xdrop_ungap);
                uint32_t store = u.score >= ucut ? u.s_end : fwd_s_end;
                dh.insert(diag, store, s_fwd_eff, window);
                if (u.score < ucut) continue;
                if (ctr) ctr->ungapped++;
                out.push_back(UngappedRecord{q_off, s_off, q_len - u.q_end, q_len - u.q_start, s_len - u.s_end,
                                             s_len - u.s_start, u.score, MINUS});
            }
        }
        if (range[0] > end_range) break;
    }
}

// engine.rs:1280-1309 sort_ungapped_like_ncbi (full ties are identical records)
void sort_ungapped(std::vector<UngappedRecord>& u, uint32_t q_len, uint32_t s_len) {
    auto key_ss = [&](const UngappedRecord& r) { return r.strand == PLUS ? r.s_start : s_len - r.s_end; };
    auto key_qk = [&](const UngappedRecord& r) -> uint64_t {
        if (r.strand == PLUS) return r.q_start;
        uint64_t ql = q_len;
        return (ql + 1) + (ql >= r.q_end ? ql - r.q_end : 0);
    };
    auto key_sk = [&](const UngappedRecord& r) { return r.strand == PLUS ? r.s_seed : s_len - r.s_seed; };
    std::sort(u.begin(), u.end(), [&](const UngappedRecord& a, const UngappedRecord& b) {
        if (a.score != b.score) return a.score > b.score;
        uint32_t as = key_ss(a), bs = key_ss(b);
        if (as != bs) return as < bs;
        uint32_t la = a.s_end - a.s_start, lb = b.s_end - b.s_start;
        if (la != lb) return la > lb;
        uint64_t aq = key_qk(a), bq = key_qk(b);
        if (aq != bq) return aq < bq;
        return key_sk(a) < key_sk(b);
    });
}

// engine.rs:1850-1895 prelim_pivot -> (pivot_q, pivot_s, tb_q, tb_s)
void prelim_pivot(const UngappedRecord& u, uint32_t qa, uint32_t sa, uint32_t lw, uint32_t out[4]) {
    if (u.strand == PLUS) {
        uint32_t tq = u.q_seed, ts = u.s_seed;
        if (u.s_end >= u.s_seed + 8) { tq += 3; ts += 3; }
        uint32_t oa = 4 - (ts % 4);
        uint32_t ps = ts + oa, pq = tq + oa;
        if (ps >= sa || pq >= qa) { ps -= 4; pq -= 4; }
        out[0] = pq; out[1] = ps; out[2] = tq; out[3] = ts;
    } else {
        uint32_t saved = sa - u.s_seed - lw;
        uint32_t s_end_fwd = sa - u.s_start;
        bool ext = s_end_fwd >= saved + 8;
        uint32_t tq = u.q_seed, ts = u.s_seed;
        if (ext) { tq = u.q_seed + lw - 4; ts = u.s_seed + lw - 4; }
        uint32_t shift = ext ? 3 : 0;
        uint32_t qn = (qa - u.q_seed - lw) + shift, sn = (sa - u.s_seed - lw) + shift;
        uint32_t oa = 4 - (sn % 4);
        uint32_t ql = qn + oa, sl = sn + oa;
        if (ql > qa || sl > sa) { ql -= 4; sl -= 4; }
        out[0] = ql; out[1] = sl; out[2] = tq; out[3] = ts;
    }
}

// search/gapped.rs:360-418 gapped_extend_score_only (subject outer, query inner)
bool gapped_score_only(const std::vector<uint8_t>& q, const std::vector<uint8_t>& s, uint32_t q_seed,
                       uint32_t s_seed, int go, int ge, int xdrop, const Matrix& m, int32_t res[5], Counters* ctr) {
    const uint8_t* qa = q.data() + 1;
    const uint8_t* sa = s.data() + 1;
    size_t qn = q.size() - 2, sn = s.size() - 2;
    ScoreOnly l = align_ex_score_only(sa, qa, s_seed, q_seed, go, ge, xdrop, m, true);
    uint32_t s_start = s_seed - l.a_len, q_start = q_seed - l.b_len;
    size_t rm = sn > s_seed ? sn - s_seed : 0, rn = qn > q_seed ? qn - q_seed : 0;
    ScoreOnly r{0, 0, 0, 0};
    if (rm > 0 && rn > 0) r = align_ex_score_only(sa + s_seed, qa + q_seed, rm, rn, go, ge, xdrop, m, false);
    if (ctr) ctr->so_cells += l.cells + r.cells;
    int32_t total = l.score + r.score;
    if (total < 0) return false;
    res[0] = total;
    res[1] = (int32_t)q_start;
    res[2] = (int32_t)(q_seed + r.b_len);
    res[3] = (int32_t)s_start;
    res[4] = (int32_t)(s_seed + r.a_len);
    return true;
}

// engine.rs:1969-2083 purge_prelim_common_endpoints
void purge_prelims(std::vector<PrelimHsp>& v, uint32_t sa) {
    size_t n = v.size();
    if (n < 2) return;
    std::vector<uint8_t> keep(n, 1);
    auto fss = [&](const PrelimHsp& h) { return h.strand == PLUS ? h.s_start : sa - h.s_end; };
    auto fse = [&](const PrelimHsp& h) { return h.strand == PLUS ? h.s_end : sa - h.s_start; };
    auto qoff = [&](const PrelimHsp& h) { return h.strand == PLUS ? h.q_start : h.q_end; };
    auto qend = [&](const PrelimHsp& h) { return h.strand == PLUS ? h.q_end : h.q_start; };
    std::vector<size_t> idx(n);
    for (size_t i = 0; i < n; ++i) idx[i] = i;
    std::sort(idx.begin(), idx.end(), [&](size_t a, size_t b) {
        const PrelimHsp &ha = v[a], &hb = v[b];
        if (ha.strand != hb.strand) return ha.strand < hb.strand;
        if (qoff(ha) != qoff(hb)) return qoff(ha) < qoff(hb);
        if (fss(ha) != fss(hb)) return fss(ha) < fss(hb);
        if (ha.score != hb.score) return ha.score > hb.score;
        if (qend(ha) != qend(hb)) return ha.strand == PLUS ? qend(ha) > qend(hb) : qend(ha) < qend(hb);
        if (fse(ha) != fse(hb)) return fse(ha) > fse(hb);
        return a < b;
    });
    for (size_t i = 0; i < n;) {
        if (!keep[idx[i]]) { ++i; continue; }
        const PrelimHsp& h0 = v[idx[i]];
        size_t j = i + 1;
        while (j < n) {
            const PrelimHsp& hj = v[idx[j]];
            if (hj.strand != h0.strand || qoff(hj) != qoff(h0) || fss(hj) != fss(h0)) break;
            keep[idx[j]] = 0;
            ++j;
        }
        i = j;
    }
    for (size_t i = 0; i < n; ++i) idx[i] = i;
    std::sort(idx.begin(), idx.end(), [&](size_t a, size_t b) {
        const PrelimHsp &ha = v[a], &hb = v[b];
        if (ha.strand != hb.strand) return ha.strand < hb.strand;
        if (qend(ha) != qend(hb)) return qend(ha) < qend(hb);
        if (fse(ha) != fse(hb)) return fse(ha) < fse(hb);
        if (ha.score != hb.score) return ha.score > hb.score;
        if (qoff(ha) != qoff(hb)) return ha.strand == PLUS ? qoff(ha) > qoff(hb) : qoff(ha) < qoff(hb);
        if (fss(ha) != fss(hb)) return fss(ha) > fss(hb);
        return a < b;
    });
    for (size_t i = 0; i < n;) {
        if (!keep[idx[i]]) { ++i; continue; }
        const PrelimHsp& h0 = v[idx[i]];
        size_t j = i + 1;
        while (j < n) {
            const PrelimHsp& hj = v[idx[j]];
            if (hj.strand != h0.strand || qend(hj) != qend(h0) || fse(hj) != fse(h0)) break;
            keep[idx[j]] = 0;
            ++j;
        }
        i = j;
    }
    std::vector<PrelimHsp> out;
    for (size_t i = 0; i < n; ++i)
        if (keep[i]) out.push_back(v[i]);
    v.swap(out);
}

// engine.rs:1317-1411 run_phase2a_inner
std::vector<PrelimHsp> phase2a(const std::vector<uint8_t>& query, const std::vector<uint8_t>& query_rc,
                               const Subject& subj, const std::vector<UngappedRecord>& ung, const Params& p,
                               const Matrix& m, uint32_t lw, Counters* ctr) {
    uint32_t qa = (uint32_t)query.size() - 2, sa = subj.len();
    IntervalTree tp(0, qa + 1, 0, sa + 1), tm(0, qa + 1, 0, sa + 1);
    std::vector<PrelimHsp> out;
    for (const UngappedRecord& u : ung) {
        uint32_t css = u.strand == PLUS ? u.s_start : sa - u.s_end;
        uint32_t cse = u.strand == PLUS ? u.s_end : sa - u.s_start;
        bool plus = u.strand == PLUS;
        if ((plus ? tp : tm).contains(ITreeHsp{u.q_start, u.q_end, css, cse, u.score}, plus, MIN_DIAG_SEP)) continue;
        uint32_t piv[4];
        prelim_pivot(u, qa, sa, lw, piv);
        int xd = std::min(p.xdrop_gap, u.score);
        if (ctr) ctr->prelim_dp++;
        int32_t r[5];
        if (!gapped_score_only(plus ? query : query_rc, subj.plus, piv[0], piv[1], p.gap_open, p.gap_extend, xd, m,
                               r, ctr))
            continue;
        int32_t sc = r[0];
        uint32_t q0 = r[1], q1 = r[2], s0 = r[3], s1 = r[4];
        uint32_t qs, qe, ss, se;
        if (!plus) { qs = qa - q1; qe = qa - q0; ss = sa - s1; se = sa - s0; }
        else { qs = q0; qe = q1; ss = s0; se = s1; }
        if (sc < p.gapped_cutoff()) continue;
        uint32_t nss = plus ? ss : sa - se, nse = plus ? se : sa - ss;
        (plus ? tp : tm).add(ITreeHsp{qs, qe, nss, nse, sc}, plus);
        out.push_back(PrelimHsp{piv[2], piv[3], qs, qe, ss, se, sc, u.strand});
    }
    purge_prelims(out, sa);
    return out;
}

// engine.rs:383-572 improve_seed
void improve_seed(const uint8_t* query, size_t qlen, const uint8_t* subject, size_t slen, uint32_t q_seed32,
                  uint32_t s_seed32, uint32_t pqs, uint32_t pqe, uint32_t pss, uint32_t pse, bool minus,
                  uint32_t& oq, uint32_t& os) {
    const int32_t RUN = 10;
    size_t q_seed = q_seed32, s_seed = s_seed32;
    int32_t hmax = (int32_t)((double)RUN * 1.5);
    oq = q_seed32;
    os = s_seed32;
    auto sat = [](size_t a, size_t b) { return a > b ? a - b : 0; };
    if (!minus) {
        int32_t score = -1;
        size_t qf = q_seed, sf = s_seed;
        while (qf < pqe && qf < qlen && sf < slen && query[qf] == subject[sf]) {
            ++score;
            if (score > RUN) return;
            ++qf;
            ++sf;
        }
        size_t qb = q_seed, sb = s_seed;
        for (;;) {
            if (query[qb] != subject[sb]) break;
            ++score;
            if (score > RUN) return;
            if (qb == 0 || sb == 0) break;
            --qb;
            --sb;
        }
        size_t offset = std::min(sat(q_seed, pqs), sat(s_seed, pss));
        size_t sqs = q_seed - offset, sss = s_seed - offset;
        size_t q_len = std::min(sat(pse, sss), sat(pqe, sqs));
        int32_t max_score = 0, sc = 0;
        size_t max_off = sqs;
        bool is_match = false, prev = false;
        for (size_t i = 0; i < q_len; ++i) {
            size_t qi = sqs + i, si = sss + i;
            if (qi >= qlen || si >= slen) break;
            is_match = query[qi] == subject[si];
            if (is_match != prev) {
                prev = is_match;
                if (is_match) sc = 1;
                else if (sc > max_score) { max_score = sc; max_off = qi - (size_t)(sc / 2); }
            } else if (is_match) {
                ++sc;
                if (sc > hmax) {
                    size_t nq = qi - (size_t)(hmax / 2);
                    oq = (uint32_t)nq;
                    os = (uint32_t)(sss + (nq - sqs));
                    return;
                }
            }
        }
        if (is_match && sc > max_score) {
            max_score = sc;
            size_t qi = sqs + q_len;
            max_off = qi - (size_t)(sc / 2);
        }
        if (max_score > 0) {
            oq = (uint32_t)max_off;
            os = (uint32_t)(sss + (max_off - sqs));
        }
        return;
    }
    int32_t score = -1;
    size_t qf = q_seed, sf = s_seed;
    while (qf < qlen && sf < slen && query[qf] == subject[sf]) {
        ++score;
        if (score > RUN) return;
        ++qf;
        ++sf;
    }
    size_t qb = q_seed, sb = s_seed;
    for (;;) {
        if (query[qb] != subject[sb]) break;
        ++score;
        if (score > RUN) return;
        if (qb <= pqs || sb == 0) break;
        --qb;
        --sb;
    }
    size_t offset = std::min(sat(sat(pqe, 1), q_seed), sat(sat(pse, 1), s_seed));
    size_t top_q = q_seed + offset, top_s = s_seed + offset;
    size_t q_len = std::min(sat(top_q, pqs) + 1, sat(top_s, pss) + 1);
    int32_t max_score = 0, sc = 0;
    int64_t max_off = (int64_t)q_seed;
    bool is_match = false, prev = false;
    for (size_t i = 0; i < q_len; ++i) {
        size_t qi = top_q - i, si = top_s - i;
        if (qi >= qlen || si >= slen) continue;
        is_match = query[qi] == subject[si];
        if (is_match != prev) {
            prev = is_match;
            if (is_match) sc = 1;
            else if (sc > max_score) { max_score = sc; max_off = (int64_t)qi + sc / 2; }
        } else if (is_match) {
            ++sc;
            if (sc > hmax) {
                size_t nq = qi + (size_t)(hmax / 2);
                oq = (uint32_t)nq;
                os = (uint32_t)(top_s - (top_q - nq));
                return;
            }
        }
    }
    if (is_match && sc > max_score) {
        max_score = sc;
        int64_t qi = (int64_t)top_q - (int64_t)q_len;
        max_off = qi + sc / 2;
    }
    if (max_score > 0) {
        if (max_off < 0) return;
        int64_t delta = (int64_t)top_q - max_off;
        int64_t ns = (int64_t)top_s - delta;
        if (ns < 0) ns = 0;
        oq = (uint32_t)max_off;
        os = (uint32_t)ns;
    }
}

// engine.rs:2953-3039 gapped_extend_bidirectional
bool gapped_bidir(const std::vector<uint8_t>& q, const std::vector<uint8_t>& s, uint32_t q_seed, uint32_t s_seed,
                  int go, int ge, int xdrop, const Matrix& m, int32_t& score, uint32_t& qs, uint32_t& qe, uint32_t& ss,
                  uint32_t& se, Script& es, Counters* ctr) {
    const uint8_t* qa = q.data() + 1;
    const uint8_t* sa = s.data() + 1;
    size_t qn = q.size() - 2, sn = s.size() - 2;
    size_t lm = (size_t)q_seed + 1, ln = (size_t)s_seed + 1;
    GapAlign l = align_ex(qa, sa, lm, ln, go, ge, xdrop, m, true);
    uint32_t q_start = q_seed + 1 - l.a_len, s_start = s_seed + 1 - l.b_len;
    size_t rq = (size_t)q_seed + 1, rs = (size_t)s_seed + 1;
    size_t rm = qn > rq ? qn - rq : 0, rn = sn > rs ? sn - rs : 0;
    GapAlign r{0, 0, 0, {}, 0};
    if (rm > 0 && rn > 0) r = align_ex(qa + rq, sa + rs, rm, rn, go, ge, xdrop, m, false);
    if (ctr) ctr->tb_cells += l.cells + r.cells;
    int32_t total = l.score + r.score;
    uint32_t q_end = q_seed + 1 + r.a_len, s_end = s_seed + 1 + r.b_len;
    Script sc;
    for (size_t i = l.script.size(); i-- > 0;) script_push(sc, l.script[i].op, l.script[i].n);
    for (const Op& o : r.script) script_push(sc, o.op, o.n);
    while (!sc.empty() && sc.front().op != SUB) {
        Op o = sc.front();
        total += go + (int32_t)o.n * ge;
        if (o.op == GAP_IN_QUERY) s_start += o.n;
        else q_start += o.n;
        sc.erase(sc.begin());
    }
    while (!sc.empty() && sc.back().op != SUB) {
        Op o = sc.back();
        total += go + (int32_t)o.n * ge;
        if (o.op == GAP_IN_QUERY) s_end -= o.n;
        else q_end -= o.n;
        sc.pop_back();
    }
    if (total < 0) return false;
    score = total;
    qs = q_start; qe = q_end; ss = s_start; se = s_end;
    es = std::move(sc);
    return true;
}

// search/gapped.rs:773-820 extract_aligned
void extract_aligned(const uint8_t* a, size_t alen, const uint8_t* b, size_t blen, size_t a_start, size_t b_start,
                     const Script& s, const std::vector<uint8_t>& nmask, std::vector<uint8_t>& qa,
                     std::vector<uint8_t>& sa) {
    auto subj_base = [&](size_t si) -> uint8_t {
        uint8_t v = si < blen ? (b[si] & 15) : 14;
        if (si < nmask.size() && nmask[si] != 0) return nmask[si];
        return v;
    };
    qa.clear();
    sa.clear();
    size_t qi = a_start, si = b_start;
    for (const Op& o : s) {
        for (uint32_t k = 0; k < o.n; ++k) {
            if (o.op == SUB) {
                qa.push_back(qi < alen ? (a[qi] & 15) : 14);
                sa.push_back(subj_base(si));
                ++qi;
                ++si;
            } else if (o.op == GAP_IN_SUBJECT) {
                qa.push_back(qi < alen ? (a[qi] & 15) : 14);
                sa.push_back(15);
                ++qi;
            } else {
                qa.push_back(15);
                sa.push_back(subj_base(si));
                ++si;
            }
        }
    }
}

// search/complexity_adjust.rs:19-132
bool complexity_adjust(int32_t raw, const std::vector<uint8_t>& query, uint32_t q_start, const Script& es,
                       const Matrix& m, int32_t cutoff, bool minus, int32_t& out) {
    uint32_t counts[16] = {0};
    size_t nb = 0;
    size_t qp = q_start;
    for (const Op& o : es) {
        if (o.op == SUB) {
            for (uint32_t i = 0; i < o.n; ++i) {
                size_t idx = 1 + qp + i;
                if (idx < query.size()) {
                    uint8_t b = query[idx];
                    if (b != 15) {
                        if (minus) b = COMPLEMENT[b & 15];
                        counts[b & 15]++;
                        ++nb;
                    }
                }
            }
            qp += o.n;
        } else if (o.op == GAP_IN_SUBJECT) {
            qp += o.n;
        }
    }
    double adj;
    if (m.lambda <= 0.0 || nb == 0) {
        adj = (double)raw;
    } else {
        double tf = 0.0, ts = 0.0, tc = 0.0;
        for (int i = 0; i < 16; ++i) {
            uint32_t c = counts[i];
            double f = m.freqs[i];
            if (c > 0 && f > 0.0 && std::log(f) != 0.0) {
                double cf = (double)c;
                tf += cf * std::log(cf);
                ts += cf * std::log(f);
                tc += cf;
            }
        }
        if (tc == 0.0) return false;  // NaN in the reference
        tf -= tc * std::log(tc);
        ts -= tf;
        adj = (double)raw + ts / m.lambda + 0.999;
        if (adj < 0.0) adj = 0.0;
    }
    if (std::isnan(adj)) return false;
    int32_t r = (int32_t)adj;  // saturating truncation as in Rust `as i32` (values here are in range)
    if (r < cutoff) return false;
    out = r;
    return true;
}

// ---- purge with cuts: engine.rs:2090-2769 ------------------------------------------------
struct Cut { bool ok; uint32_t gq, gs; };

Cut cut_scan_front(const Script& ops, uint32_t need_q, uint32_t need_s, size_t& cut_i, uint32_t& partial) {
    uint32_t gq = 0, gs = 0;
    for (size_t i = 0; i < ops.size(); ++i) {
        const Op o = ops[i];
        if (o.op == SUB) {
            for (uint32_t j = 0; j < o.n; ++j) {
                ++gq; ++gs;
                if (gq >= need_q && gs >= need_s) { cut_i = i; partial = j + 1; return Cut{true, gq, gs}; }
            }
        } else if (o.op == GAP_IN_QUERY) {
            gs += o.n;
            if (gq >= need_q && gs >= need_s) { cut_i = i; partial = o.n; return Cut{true, gq, gs}; }
        } else {
            gq += o.n;
            if (gq >= need_q && gs >= need_s) { cut_i = i; partial = o.n; return Cut{true, gq, gs}; }
        }
    }
    return Cut{false, gq, gs};
}
Cut cut_scan_back(const Script& ops, uint32_t need_q, uint32_t need_s, size_t& cut_i, uint32_t& partial) {
    uint32_t gq = 0, gs = 0;
    for (size_t i = ops.size(); i-- > 0;) {
        const Op o = ops[i];
        if (o.op == SUB) {
            for (uint32_t j = 0; j < o.n; ++j) {
                ++gq; ++gs;
                if (gq >= need_q && gs >= need_s) { cut_i = i; partial = j + 1; return Cut{true, gq, gs}; }
            }
        } else if (o.op == GAP_IN_QUERY) {
            gs += o.n;
            if (gq >= need_q && gs >= need_s) { cut_i = i; partial = o.n; return Cut{true, gq, gs}; }
        } else {
            gq += o.n;
            if (gq >= need_q && gs >= need_s) { cut_i = i; partial = o.n; return Cut{true, gq, gs}; }
        }
    }
    return Cut{false, gq, gs};
}
// engine.rs:2090 cut_ops_keep_front
Cut cut_ops_keep_front(Script& ops, uint32_t nq, uint32_t ns) {
    if (nq == 0 && ns == 0) return Cut{true, 0, 0};
    size_t ci = 0; uint32_t part = 0;
    Cut c = cut_scan_front(ops, nq, ns, ci, part);
    if (!c.ok) return c;
    if (part < ops[ci].n) ops[ci].n = part;
    ops.resize(ci + 1);
    return c;
}
// engine.rs:2131 cut_ops_front
Cut cut_ops_front(Script& ops, uint32_t nq, uint32_t ns) {
    if (nq == 0 && ns == 0) return Cut{true, 0, 0};
    size_t ci = 0; uint32_t part = 0;
    Cut c = cut_scan_front(ops, nq, ns, ci, part);
    if (!c.ok) return c;
    Op o = ops[ci];
    uint32_t rem = o.n - part;
    ops.erase(ops.begin(), ops.begin() + ci + 1);
    if (rem > 0) ops.insert(ops.begin(), Op{o.op, rem});
    return c;
}
// engine.rs:2172 cut_ops_back
Cut cut_ops_back(Script& ops, uint32_t nq, uint32_t ns) {
    if (nq == 0 && ns == 0) return Cut{true, 0, 0};
    size_t ci = 0; uint32_t part = 0;
    Cut c = cut_scan_back(ops, nq, ns, ci, part);
    if (!c.ok) return c;
    Op o = ops[ci];
    uint32_t keep = o.n - part;
    ops.resize(ci);
    if (keep > 0) ops.push_back(Op{o.op, keep});
    return c;
}
// engine.rs:2217 keep_ops_back
Cut keep_ops_back(Script& ops, uint32_t nq, uint32_t ns) {
    if (nq == 0 && ns == 0) return Cut{true, 0, 0};
    size_t ci = 0; uint32_t part = 0;
    Cut c = cut_scan_back(ops, nq, ns, ci, part);
    if (!c.ok) return c;
    Op o = ops[ci];
    ops.erase(ops.begin(), ops.begin() + ci);
    if (part < o.n) ops[0] = Op{o.op, part};
    return c;
}

uint32_t satsub(uint32_t a, uint32_t b) { return a > b ? a - b : 0; }

bool cut_start_secondary(const AlignResult& pr, AlignResult& sec) {  // engine.rs:2650
    const Hsp &p = pr.hsp;
    Hsp& s = sec.hsp;
    bool extends = p.strand == PLUS ? s.q_end > p.q_end : s.q_start < p.q_start;
    if (!extends) return false;
    if (p.strand == PLUS) {
        uint32_t dq = satsub(p.q_end, s.q_start), ds = satsub(p.s_end, s.s_start);
        uint32_t oq = s.q_start, os = s.s_start;
        Cut c = cut_ops_front(s.script, dq, ds);
        if (c.ok) { s.q_start = oq + c.gq; s.s_start = os + c.gs; }
    } else {
        uint32_t dq = satsub(s.q_end, p.q_start), ds = satsub(p.s_end, s.s_start);
        uint32_t oqe = s.q_end, os = s.s_start;
        Cut c = cut_ops_back(s.script, dq, ds);
        if (c.ok) { s.q_end = oqe - c.gq; s.s_start = os + c.gs; }
    }
    return !s.script.empty();
}
bool cut_end_secondary(const AlignResult& pr, AlignResult& sec) {  // engine.rs:2683
    const Hsp& p = pr.hsp;
    Hsp& s = sec.hsp;
    bool extends = p.strand == PLUS ? s.q_start < p.q_start : s.q_end > p.q_end;
    if (!extends) return false;
    if (p.strand == PLUS) {
        uint32_t nq = satsub(p.q_start, s.q_start), ns = satsub(p.s_start, s.s_start);
        Cut c = cut_ops_keep_front(s.script, nq, ns);
        if (c.ok) { s.q_end = s.q_start + c.gq; s.s_end = s.s_start + c.gs; }
    } else {
        uint32_t nq = satsub(s.q_end, p.q_end), ns = satsub(p.s_start, s.s_start);
        Cut c = keep_ops_back(s.script, nq, ns);
        if (c.ok) { s.q_start = satsub(s.q_end, c.gq); s.s_end = s.s_start + c.gs; }
    }
    return !s.script.empty();
}
bool cmp_query_offset(const AlignResult& a, const AlignResult& b) {  // engine.rs:2592 (less-than)
    const Hsp &ha = a.hsp, &hb = b.hsp;
    if (ha.strand != hb.strand) return ha.strand < hb.strand;
    uint32_t ka = ha.strand == PLUS ? ha.q_start : ha.q_end, kb = hb.strand == PLUS ? hb.q_start : hb.q_end;
    if (ka != kb) return ka < kb;
    if (ha.s_start != hb.s_start) return ha.s_start < hb.s_start;
    if (ha.score != hb.score) return ha.score > hb.score;
    if (ha.strand == PLUS) { if (ha.q_end != hb.q_end) return ha.q_end > hb.q_end; }
    else { if (ha.q_start != hb.q_start) return ha.q_start < hb.q_start; }
    return ha.s_end > hb.s_end;
}
bool cmp_query_end(const AlignResult& a, const AlignResult& b) {  // engine.rs:2611
    const Hsp &ha = a.hsp, &hb = b.hsp;
    if (ha.strand != hb.strand) return ha.strand < hb.strand;
    uint32_t ka = ha.strand == PLUS ? ha.q_end : ha.q_start, kb = hb.strand == PLUS ? hb.q_end : hb.q_start;
    if (ka != kb) return ka < kb;
    if (ha.s_end != hb.s_end) return ha.s_end < hb.s_end;
    if (ha.score != hb.score) return ha.score > hb.score;
    if (ha.strand == PLUS) { if (ha.q_start != hb.q_start) return ha.q_start > hb.q_start; }
    else { if (ha.q_end != hb.q_end) return ha.q_end < hb.q_end; }
    return ha.s_start > hb.s_start;
}
bool same_start(const AlignResult& a, const AlignResult& b) {
    if (a.hsp.strand != b.hsp.strand) return false;
    uint32_t ka = a.hsp.strand == PLUS ? a.hsp.q_start : a.hsp.q_end;
    uint32_t kb = b.hsp.strand == PLUS ? b.hsp.q_start : b.hsp.q_end;
    return ka == kb && a.hsp.s_start == b.hsp.s_start;
}
bool same_end(const AlignResult& a, const AlignResult& b) {
    if (a.hsp.strand != b.hsp.strand) return false;
    uint32_t ka = a.hsp.strand == PLUS ? a.hsp.q_end : a.hsp.q_start;
    uint32_t kb = b.hsp.strand == PLUS ? b.hsp.q_end : b.hsp.q_start;
    return ka == kb && a.hsp.s_end == b.hsp.s_end;
}

using Slot = std::vector<AlignResult*>;  // nullptr = freed slot

// engine.rs:2743-2769 collapse_common_endpoint_groups
size_t collapse(std::vector<AlignResult*>& arr, size_t count, bool purge,
                bool (*same)(const AlignResult&, const AlignResult&),
                bool (*cut)(const AlignResult&, AlignResult&), std::vector<AlignResult*>& freed) {
    std::vector<AlignResult*> removed;
    size_t surv = 0;
    for (size_t r = 0; r < count; ++r) {
        bool joins = surv > 0 && same(*arr[surv - 1], *arr[r]);
        if (joins) {
            AlignResult* sec = arr[r];
            arr[r] = nullptr;
            bool keep = !purge && cut(*arr[surv - 1], *sec);
            if (keep) removed.push_back(sec);
            else { freed.push_back(sec); removed.push_back(nullptr); }
        } else {
            std::swap(arr[surv], arr[r]);
            ++surv;
        }
    }
    size_t k = removed.size();
    for (size_t i = surv; i < count; ++i) arr[i] = removed[--k];
    return surv;
}
// engine.rs:2717 purge_hsps_with_common_endpoints
size_t purge_common(std::vector<AlignResult*>& arr, bool purge, std::vector<AlignResult*>& freed) {
    size_t n = arr.size();
    if (n < 2) return n;
    std::stable_sort(arr.begin(), arr.begin() + n,
                     [](const AlignResult* a, const AlignResult* b) { return cmp_query_offset(*a, *b); });
    size_t c = collapse(arr, n, purge, same_start, cut_start_secondary, freed);
    std::stable_sort(arr.begin(), arr.begin() + c,
                     [](const AlignResult* a, const AlignResult* b) { return cmp_query_end(*a, *b); });
    return collapse(arr, c, purge, same_end, cut_end_secondary, freed);
}

// engine.rs:2268-2567 reevaluate_gapped.  Returns true if the HSP is to be deleted.
bool reevaluate(Hsp& hsp, const std::vector<uint8_t>& q_seq, const std::vector<uint8_t>& s_seq, const Matrix& m,
                int go, int ge, int32_t min_score, bool minus, const uint8_t* raw_q, size_t raw_q_len,
                size_t q_raw_start, const uint8_t* raw_s, size_t raw_s_len, size_t s_raw_start) {
    if (hsp.script.empty()) return true;
    int32_t sum = 0, score = 0;
    size_t seq_i = 0;
    uint32_t q_pos = 0, s_pos = 0;
    uint32_t bqs = 0, bss = 0, bqe = 0, bse = 0, cqs = 0, css = 0;
    size_t bsi = 0, bei = 0, csi = 0;
    uint32_t ben = 0, cskip = 0, bskip = 0;
    const Script snap = hsp.script;
    const size_t esp = snap.size();
    Script rops;
    std::vector<uint8_t> rq, rs;
    const Script* sops = &snap;
    const std::vector<uint8_t>* sq = &q_seq;
    const std::vector<uint8_t>* ss = &s_seq;
    if (minus) {
        rops.assign(snap.rbegin(), snap.rend());
        rq.assign(q_seq.rbegin(), q_seq.rend());
        rs.assign(s_seq.rbegin(), s_seq.rend());
        sops = &rops; sq = &rq; ss = &rs;
    }
    for (size_t ei = 0; ei < sops->size(); ++ei) {
        const Op o = (*sops)[ei];
        if (o.op == SUB) {
            for (uint32_t k = 0; k < o.n; ++k) {
                uint8_t qb0 = (seq_i < sq->size() ? (*sq)[seq_i] : 14) & 0xf;
                uint8_t sb0 = (seq_i < ss->size() ? (*ss)[seq_i] : 14) & 0xf;
                uint8_t qb = minus ? (COMPLEMENT[qb0] & 0xf) : qb0;
                uint8_t sb = minus ? (COMPLEMENT[sb0] & 0xf) : sb0;
                sum += m.s[qb][sb];
                ++seq_i; ++q_pos; ++s_pos;
                uint32_t op_idx = k + 1;
                if (sum < 0) {
                    if (op_idx < o.n) { csi = ei; cskip = op_idx; }
                    else { csi = ei + 1; cskip = 0; }
                    sum = 0;
                    cqs = q_pos; css = s_pos;
                    if (score < min_score) {
                        bqs = q_pos; bss = s_pos; score = 0;
                        bsi = csi; bskip = cskip; bei = csi; ben = 0;
                    }
                } else if (sum > score) {
                    score = sum;
                    bqs = cqs; bss = css; bqe = q_pos; bse = s_pos;
                    bsi = csi; bskip = cskip; bei = ei; ben = op_idx;
                }
            }
        } else {
            sum -= go + ge * (int32_t)o.n;
            if (o.op == GAP_IN_QUERY) { seq_i += o.n; s_pos += o.n; }
            else { seq_i += o.n; q_pos += o.n; }
            if (sum < 0) {
                csi = ei + 1; cskip = 0;
                sum = 0; cqs = q_pos; css = s_pos;
                if (score < min_score) {
                    bqs = q_pos; bss = s_pos; score = 0;
                    bsi = csi; bskip = 0; bei = csi; ben = 0;
                }
            } else if (sum > score) {
                score = sum;
                bqs = cqs; bss = css; bqe = q_pos; bse = s_pos;
                bsi = csi; bskip = cskip; bei = ei; ben = o.n;
            }
        }
    }
    if (score < min_score) return true;
    if (minus) {
        uint32_t qtot = 0, stot = 0;
        for (const Op& o : snap) {
            if (o.op == SUB) { qtot += o.n; stot += o.n; }
            else if (o.op == GAP_IN_SUBJECT) qtot += o.n;
            else stot += o.n;
        }
        size_t fsi = esp - 1 - bei, fei = esp - 1 - bsi;
        uint32_t fen = snap[fei].n - bskip;
        uint32_t fskip = snap[fsi].n - ben;
        uint32_t fqs = qtot - bqe, fqe = qtot - bqs, fss = stot - bse, fse = stot - bss;
        bsi = fsi; bei = fei; bskip = fskip; ben = fen;
        bqs = fqs; bqe = fqe; bss = fss; bse = fse;
    }
    {
        Script& ops = hsp.script;
        if (bei < (esp > 0 ? esp - 1 : 0) || ben < snap[bei].n) {
            ops.resize(bei + 1);
            if (ben > 0) ops[bei].n = ben;
            else ops.resize(bei);
        }
        if (bsi > 0) ops.erase(ops.begin(), ops.begin() + std::min(bsi, ops.size()));
        if (bskip > 0 && !ops.empty()) {
            Op o0 = ops[0];
            if (bskip < o0.n) ops[0].n = o0.n - bskip;
            else ops.erase(ops.begin());
        }
    }
    int64_t xbqs = bqs, xbss = bss, xbqe = bqe, xbse = bse;
    for (;;) {
        int64_t qi = (int64_t)q_raw_start + xbqs, si = (int64_t)s_raw_start + xbss;
        if (qi <= 0 || si <= 0) break;
        uint8_t qb = raw_q[qi - 1], sb = raw_s[si - 1];
        if (qb < 4 && qb == sb) {
            --xbqs; --xbss;
            Script& ops = hsp.script;
            if (!ops.empty() && ops.front().op == SUB) ops[0].n += 1;
            else ops.insert(ops.begin(), Op{SUB, 1});
        } else break;
    }
    for (;;) {
        int64_t qi = (int64_t)q_raw_start + xbqe, si = (int64_t)s_raw_start + xbse;
        if (qi >= (int64_t)raw_q_len || si >= (int64_t)raw_s_len) break;
        uint8_t qb = raw_q[qi], sb = raw_s[si];
        if (qb < 4 && qb == sb) {
            ++xbqe; ++xbse;
            Script& ops = hsp.script;
            if (!ops.empty() && ops.back().op == SUB) ops.back().n += 1;
            else ops.push_back(Op{SUB, 1});
        } else break;
    }
    hsp.score = score;
    auto clamp0 = [](int64_t v) { return (uint32_t)(v < 0 ? 0 : v); };
    if (minus) {
        int64_t oqs = hsp.q_start, ose = hsp.s_end;
        hsp.q_start = clamp0(oqs + xbqs);
        hsp.q_end = clamp0(oqs + xbqe);
        hsp.s_end = clamp0(ose - xbss);
        hsp.s_start = clamp0(ose - xbse);
    } else {
        int64_t oqs = hsp.q_start, oss = hsp.s_start;
        uint32_t nqs = clamp0(oqs + xbqs), nss = clamp0(oss + xbss);
        hsp.q_start = nqs;
        hsp.q_end = nqs + (uint32_t)(xbqe - xbqs);
        hsp.s_start = nss;
        hsp.s_end = nss + (uint32_t)(xbse - xbss);
    }
    return false;
}

// engine.rs:1438-1762 traceback_phase
std::vector<AlignResult> phase2b(const std::vector<uint8_t>& query, const std::vector<uint8_t>& query_rc,
                                 const std::string& qid, const Subject& subj, std::vector<PrelimHsp> pre,
                                 const Params& p, const Matrix& m, Counters* ctr) {
    const uint32_t qa = (uint32_t)query.size() - 2, sl = subj.len(), sa = sl;
    const std::vector<uint8_t>& splus = subj.align;
    const std::vector<uint8_t>& src = subj.align_rc;
    std::stable_sort(pre.begin(), pre.end(), [&](const PrelimHsp& a, const PrelimHsp& b) {
        uint32_t fsa = a.strand == PLUS ? a.s_start : sl - a.s_end, fsb = b.strand == PLUS ? b.s_start : sl - b.s_end;
        uint32_t fea = a.strand == PLUS ? a.s_end : sl - a.s_start, feb = b.strand == PLUS ? b.s_end : sl - b.s_start;
        uint32_t qoa = a.strand == PLUS ? a.q_start : qa - a.q_end, qob = b.strand == PLUS ? b.q_start : qa - b.q_end;
        uint32_t qea = a.strand == PLUS ? a.q_end : qa - a.q_start, qeb = b.strand == PLUS ? b.q_end : qa - b.q_start;
        if (a.score != b.score) return a.score > b.score;
        if (fsa != fsb) return fsa < fsb;
        if (fea != feb) return fea > feb;
        if (qoa != qob) return qoa < qob;
        return qea > qeb;
    });
    IntervalTree tp(0, qa + 1, 0, sl + 1), tm(0, qa + 1, 0, sl + 1, true);
    std::vector<AlignResult> results;
    std::vector<uint8_t> qb, sb;
    for (const PrelimHsp& ph : pre) {
        bool plus = ph.strand == PLUS;
        uint32_t pss = plus ? ph.s_start : sl - ph.s_end, pse = plus ? ph.s_end : sl - ph.s_start;
        uint32_t cqs = plus ? ph.q_start : qa - ph.q_end, cqe = plus ? ph.q_end : qa - ph.q_start;
        if ((plus ? tp : tm).contains(ITreeHsp{cqs, cqe, pss, pse, ph.score}, plus, MIN_DIAG_SEP)) continue;
        const std::vector<uint8_t>& sfs = plus ? splus : src;
        uint32_t nq, ns;
        improve_seed(query.data() + 1, qa, sfs.data() + 1, sfs.size() - 2, ph.q_seed, ph.s_seed, ph.q_start, ph.q_end,
                     ph.s_start, ph.s_end, !plus, nq, ns);
        uint32_t tq = plus ? nq : qa - 1 - nq, ts = plus ? ns : sa - 1 - ns;
        if (ctr) ctr->tb_dp++;
        int32_t sc;
        uint32_t q0, q1, s0, s1;
        Script es;
        if (!gapped_bidir(plus ? query : query_rc, splus, tq, ts, p.gap_open, p.gap_extend, p.xdrop_gap_final, m, sc,
                          q0, q1, s0, s1, es, ctr))
            continue;
        uint32_t qs, qe, ss, se;
        if (!plus) {
            extract_aligned(query_rc.data() + 1, query_rc.size() - 2, splus.data() + 1, splus.size() - 2, q0, s0, es,
                            subj.n_mask, qb, sb);
            qb = revcomp(qb.data(), qb.size());
            sb = revcomp(sb.data(), sb.size());
            qs = qa - q1; qe = qa - q0; ss = sa - s1; se = sa - s0;
            std::reverse(es.begin(), es.end());
        } else {
            extract_aligned(query.data() + 1, qa, splus.data() + 1, splus.size() - 2, q0, s0, es, subj.n_mask, qb, sb);
            qs = q0; qe = q1; ss = s0; se = s1;
        }
        if (p.complexity_adjust) {
            int32_t adj;
            if (!complexity_adjust(sc, query, qs, es, m, p.gapped_cutoff(), !plus, adj)) continue;
            sc = adj;
        }
        uint32_t rqs = qs, rqe = qe, rss = plus ? ss : sl - se, rse = plus ? se : sl - ss;
        {
            uint32_t tqs = plus ? rqs : qa - rqe, tqe = plus ? rqe : qa - rqs;
            (plus ? tp : tm).add(ITreeHsp{tqs, tqe, rss, rse, sc}, true);
        }
        AlignResult r;
        r.hsp.score = sc;
        r.hsp.q_start = rqs; r.hsp.q_end = rqe; r.hsp.q_len = qa;
        r.hsp.s_start = rss; r.hsp.s_end = rse; r.hsp.s_len = sl;
        r.hsp.strand = ph.strand;
        r.hsp.script = std::move(es);
        r.hsp.q_seq = qb;
        r.hsp.s_seq = sb;
        r.query_id = qid;
        r.subject_id = subj.id;
        r.stats = compute_align_stats(to_iupac(qb), to_iupac(sb));
        results.push_back(std::move(r));
        if (ctr) ctr->finals++;
    }
    // purge(FALSE) + reevaluate + purge(TRUE): engine.rs:1648-1726
    {
        std::vector<AlignResult> store = std::move(results);
        std::vector<AlignResult*> arr;
        for (auto& r : store) arr.push_back(&r);
        std::vector<AlignResult*> freed;
        size_t extra = purge_common(arr, false, freed);
        const uint8_t* qcore = query.data() + 1;
        const uint8_t* score_ = splus.data() + 1;
        const uint8_t* rcore = src.data() + 1;
        size_t slen = splus.size() - 2;
        for (size_t i = extra; i < arr.size(); ++i) {
            AlignResult* r = arr[i];
            if (!r) continue;
            bool minus = r->hsp.strand == MINUS;
            size_t as = r->hsp.q_start;
            size_t bs = minus ? (size_t)(sa - r->hsp.s_end) : r->hsp.s_start;
            const uint8_t* bcore = minus ? rcore : score_;
            const std::vector<uint8_t>& bmask = minus ? subj.n_mask_rc : subj.n_mask;
            std::vector<uint8_t> q1, s1;
            extract_aligned(qcore, qa, bcore, slen, as, bs, r->hsp.script, bmask, q1, s1);
            bool del = reevaluate(r->hsp, q1, s1, m, p.gap_open, p.gap_extend, p.gapped_cutoff(), minus, qcore, qa, as,
                                  bcore, slen, bs);
            if (del) { arr[i] = nullptr; continue; }
            size_t as2 = r->hsp.q_start;
            size_t bs2 = minus ? (size_t)(sa - r->hsp.s_end) : r->hsp.s_start;
            extract_aligned(qcore, qa, bcore, slen, as2, bs2, r->hsp.script, bmask, q1, s1);
            r->stats = compute_align_stats(to_iupac(q1), to_iupac(s1));
            r->hsp.q_seq = q1;
            r->hsp.s_seq = s1;
        }
        std::vector<AlignResult*> arr2;
        for (AlignResult* r : arr)
            if (r) arr2.push_back(r);
        std::vector<AlignResult*> freed2;
        size_t n2 = purge_common(arr2, true, freed2);
        (void)n2;
        for (AlignResult* r : arr2)
            if (r) results.push_back(std::move(*r));
    }
    // Phase 2c: engine.rs:1732-1759
    std::stable_sort(results.begin(), results.end(), [&](const AlignResult& A, const AlignResult& B) {
        const Hsp &a = A.hsp, &b = B.hsp;
        uint32_t qoa = a.strand == PLUS ? a.q_start : qa - a.q_end, qob = b.strand == PLUS ? b.q_start : qa - b.q_end;
        uint32_t qea = a.strand == PLUS ? a.q_end : qa - a.q_start, qeb = b.strand == PLUS ? b.q_end : qa - b.q_start;
        if (a.score != b.score) return a.score > b.score;
        if (a.s_start != b.s_start) return a.s_start < b.s_start;
        if (a.s_end != b.s_end) return a.s_end > b.s_end;
        if (qoa != qob) return qoa < qob;
        return qea > qeb;
    });
    IntervalTree fp(0, qa + 1, 0, sl + 1), fm(0, qa + 1, 0, sl + 1);
    std::vector<AlignResult> kept;
    for (auto& r : results) {
        bool plus = r.hsp.strand == PLUS;
        ITreeHsp h{r.hsp.q_start, r.hsp.q_end, r.hsp.s_start, r.hsp.s_end, r.hsp.score};
        if ((plus ? fp : fm).contains(h, plus, MIN_DIAG_SEP)) continue;
        (plus ? fp : fm).add_simple(h);
        kept.push_back(std::move(r));
    }
    return kept;
}
}  // namespace

// engine.rs:734-794 search_one_subject + engine.rs:1905-1966 run_gapped_phase
std::vector<AlignResult> search_pair(const QueryLookup& ql, const std::vector<uint8_t>& query,
                                     const std::string& qid, const Subject& subj, const Params& p, const Matrix& m,
                                     const Taps& taps) {
    uint32_t q_len = (uint32_t)query.size() - 2, s_len = subj.len();
    if (q_len < (uint32_t)p.word_size || s_len < (uint32_t)p.word_size) return {};
    std::vector<UngappedRecord> ung;
    collect_ungapped(query, ql, subj, p, m, taps.seeds, ung, taps.counters);
    sort_ungapped(ung, q_len, s_len);
    if (taps.ungapped)
        for (auto& u : ung) {
            uint32_t ss = u.strand == PLUS ? u.s_start : s_len - u.s_end;
            uint32_t se = u.strand == PLUS ? u.s_end : s_len - u.s_start;
            taps.ungapped->push_back(UngappedHit{u.q_start, u.q_end, ss, se, u.score, u.strand});
        }
    if (ung.empty()) return {};
    std::vector<PrelimHsp> pre = phase2a(query, ql.query_rc, subj, ung, p, m, ql.lut.lut_word_length, taps.counters);
    if (taps.counters) taps.counters->prelims += pre.size();
    if (taps.prelims) taps.prelims->insert(taps.prelims->end(), pre.begin(), pre.end());
    return phase2b(query, ql.query_rc, qid, subj, std::move(pre), p, m, taps.counters);
}

// Traceback of every post-purge prelim of one pair, in the order traceback_phase visits them
// (engine.rs:1471-1485 stable sort), containment not applied: per prelim (strand, status
// 0 = alignment / 1 = none, score, q0, q1, s0, s1 in the DP frame, n_ops, FNV-1a of the ops).
std::vector<uint32_t> pair_tracebacks(const QueryLookup& ql, const std::vector<uint8_t>& query, const Subject& subj,
                                      const Params& p, const Matrix& m) {
    std::vector<uint32_t> out;
    std::vector<PrelimHsp> pre;
    Taps t;
    t.prelims = &pre;
    search_pair(ql, query, "", subj, p, m, t);
    const uint32_t qa = (uint32_t)query.size() - 2, sl = subj.len();
    std::stable_sort(pre.begin(), pre.end(), [&](const PrelimHsp& a, const PrelimHsp& b) {
        uint32_t fsa = a.strand == PLUS ? a.s_start : sl - a.s_end, fsb = b.strand == PLUS ? b.s_start : sl - b.s_end;
        uint32_t fea = a.strand == PLUS ? a.s_end : sl - a.s_start, feb = b.strand == PLUS ? b.s_end : sl - b.s_start;
        uint32_t qoa = a.strand == PLUS ? a.q_start : qa - a.q_end, qob = b.strand == PLUS ? b.q_start : qa - b.q_end;
        uint32_t qea = a.strand == PLUS ? a.q_end : qa - a.q_start, qeb = b.strand == PLUS ? b.q_end : qa - b.q_start;
        if (a.score != b.score) return a.score > b.score;
        if (fsa != fsb) return fsa < fsb;
        if (fea != feb) return fea > feb;
        if (qoa != qob) return qoa < qob;
        return qea > qeb;
    });
    for (const PrelimHsp& ph : pre) {
        const bool plus = ph.strand == PLUS;
        const std::vector<uint8_t>& sfs = plus ? subj.align : subj.align_rc;
        uint32_t nq, ns;
        improve_seed(query.data() + 1, qa, sfs.data() + 1, sfs.size() - 2, ph.q_seed, ph.s_seed, ph.q_start, ph.q_end,
                     ph.s_start, ph.s_end, !plus, nq, ns);
        const uint32_t tq = plus ? nq : qa - 1 - nq, ts = plus ? ns : sl - 1 - ns;
        int32_t sc = 0;
        uint32_t q0 = 0, q1 = 0, s0 = 0, s1 = 0;
        Script es;
        const bool ok = gapped_bidir(plus ? query : ql.query_rc, subj.align, tq, ts, p.gap_open, p.gap_extend,
                                     p.xdrop_gap_final, m, sc, q0, q1, s0, s1, es, nullptr);
        uint32_t h = 2166136261u;
        for (const Op& o : es) {
            const uint32_t v = ((uint32_t)o.op << 30) | o.n;
            for (int b = 0; b < 4; ++b) h = (h ^ ((v >> (8 * b)) & 0xffu)) * 16777619u;
        }
        if (!ok) { sc = 0; q0 = q1 = s0 = s1 = 0; es.clear(); h = 2166136261u; }
        out.insert(out.end(), {(uint32_t)ph.strand, ok ? 0u : 1u, (uint32_t)sc, q0, q1, s0, s1, (uint32_t)es.size(), h});
    }
    return out;
}

// engine.rs:863-974 apply_mask_level (cross-subject mode; oid = subject index)
void apply_mask_level(std::vector<AlignResult>& res, uint32_t level) {
    if (level >= 100) return;
    std::sort(res.begin(), res.end(), [](const AlignResult& A, const AlignResult& B) {
        const Hsp &a = A.hsp, &b = B.hsp;
        if (a.score != b.score) return a.score > b.score;
        if (A.oid != B.oid) return A.oid > B.oid;
        if (a.s_start != b.s_start) return a.s_start < b.s_start;
        if (a.s_end != b.s_end) return a.s_end > b.s_end;
        uint32_t qoa = a.strand == PLUS ? a.q_start : a.q_len - a.q_end;
        uint32_t qob = b.strand == PLUS ? b.q_start : b.q_len - b.q_end;
        if (qoa != qob) return qoa < qob;
        uint32_t qea = a.strand == PLUS ? a.q_end : a.q_len - a.q_start;
        uint32_t qeb = b.strand == PLUS ? b.q_end : b.q_len - b.q_start;
        return qea > qeb;
    });
    size_t n = res.size();
    if (!n) return;
    // Accepted ranges by start; a range that ends before the candidate starts cannot mask it,
    // so only starts in [qs - longest accepted span, hi] are examined.
    std::multimap<uint32_t, std::pair<uint32_t, int32_t>> acc;
    uint32_t max_span = 0;
    std::vector<uint8_t> keep(n, 1);
    const bool touching = level == 0;
    for (size_t i = 0; i < n; ++i) {
        const Hsp& h = res[i].hsp;
        uint32_t qs = h.q_start, qe = h.q_end;
        if (h.strand == MINUS) { qs += 1; qe += 1; }
        int32_t sc = h.score;
        int64_t span = (int64_t)qe - qs;
        if (span == 0) { keep[i] = 0; continue; }
        uint32_t hi = touching ? qe : qe - 1;
        uint32_t lo = qs > max_span ? qs - max_span : 0;
        bool masked = false;
        for (auto it = acc.lower_bound(lo); it != acc.end() && it->first <= hi; ++it) {
            uint32_t qsj = it->first, qej = it->second.first;
            int32_t scj = it->second.second;
            if (qej < qs || (qej == qs && !touching)) continue;
            if (scj < sc) continue;
            int64_t ov = (int64_t)std::min(qej, qe) - (int64_t)std::max(qsj, qs);
            int64_t perc = (int64_t)(100.0 * ((double)ov / (double)span));
            if (perc >= (int64_t)level) { masked = true; break; }
        }
        if (masked) keep[i] = 0;
        else {
            acc.emplace(qs, std::make_pair(qe, sc));
            max_span = std::max(max_span, qe - qs);
        }
    }
    std::vector<AlignResult> out;
    for (size_t i = 0; i < n; ++i)
        if (keep[i]) out.push_back(std::move(res[i]));
    res.swap(out);
}

static bool score_compare(const Hsp& a, const Hsp& b) {  // hits.rs:104-112 (less-than)
    uint32_t qoa = a.strand == PLUS ? a.q_start : a.q_len - a.q_end;
    uint32_t qea = a.strand == PLUS ? a.q_end : a.q_len - a.q_start;
    uint32_t qob = b.strand == PLUS ? b.q_start : b.q_len - b.q_end;
    uint32_t qeb = b.strand == PLUS ? b.q_end : b.q_len - b.q_start;
    if (a.score != b.score) return a.score > b.score;
    if (a.s_start != b.s_start) return a.s_start < b.s_start;
    if (a.s_end != b.s_end) return a.s_end > b.s_end;
    if (qoa != qob) return qoa < qob;
    return qea > qeb;
}

// main.rs:1230-1234 then engine.rs:998-1017 sort_hit_list_order_by_oid
void sort_hit_list_order(std::vector<AlignResult>& res) {
    std::sort(res.begin(), res.end(), [](const AlignResult& a, const AlignResult& b) {
        int c = a.subject_id.compare(b.subject_id);
        if (c != 0) return c < 0;
        if (a.hsp.strand != b.hsp.strand) return a.hsp.strand < b.hsp.strand;  // "+" < "-"
        return a.hsp.q_start < b.hsp.q_start;
    });
    std::map<uint32_t, int32_t> best;
    for (auto& r : res) {
        auto it = best.find(r.oid);
        if (it == best.end()) best[r.oid] = r.hsp.score;
        else it->second = std::max(it->second, r.hsp.score);
    }
    std::stable_sort(res.begin(), res.end(), [&](const AlignResult& a, const AlignResult& b) {
        int32_t ba = best[a.oid], bb = best[b.oid];
        if (ba != bb) return ba > bb;
        if (a.oid != b.oid) return a.oid > b.oid;
        return score_compare(a.hsp, b.hsp);
    });
}

// main.rs:1018-1085 merge_chunk_prelims: NCBI's cross-chunk merge (plus strand only), called
// once per chunk in chunk order; `split` is the chunk's start in the full query.
void merge_chunk_prelims(std::vector<PrelimHsp>& acc, std::vector<PrelimHsp> add, uint32_t split) {
    const uint32_t OVERLAP = 100;
    const int64_t DIAG_CLOSE = 10;
    auto order = [](const PrelimHsp& a, const PrelimHsp& b) {  // ScoreCompareHSPs, plus strand
        if (a.score != b.score) return a.score > b.score;
        if (a.s_start != b.s_start) return a.s_start < b.s_start;
        if (a.s_end != b.s_end) return a.s_end > b.s_end;
        if (a.q_start != b.q_start) return a.q_start < b.q_start;
        return a.q_end > b.q_end;
    };
    std::vector<uint8_t> absorbed(add.size(), 0);
    std::vector<size_t> ac, nc;
    for (size_t i = 0; i < acc.size(); ++i)
        if (acc[i].strand == PLUS && acc[i].q_end > split) ac.push_back(i);
    std::stable_sort(ac.begin(), ac.end(), [&](size_t a, size_t b) { return order(acc[a], acc[b]); });
    for (size_t j = 0; j < add.size(); ++j)
        if (add[j].strand == PLUS && add[j].q_start < split + OVERLAP) nc.push_back(j);
    std::stable_sort(nc.begin(), nc.end(), [&](size_t a, size_t b) { return order(add[a], add[b]); });
    for (size_t i : ac) {
        PrelimHsp& h1 = acc[i];
        for (size_t j : nc) {
            if (absorbed[j]) continue;
            const PrelimHsp& h2 = add[j];
            const int64_t end_diag = (int64_t)h1.q_end - (int64_t)h1.s_end;
            const int64_t start_diag = (int64_t)h2.q_start - (int64_t)h2.s_start;
            const int64_t dd = end_diag - start_diag;
            if ((dd < 0 ? -dd : dd) >= DIAG_CLOSE) continue;
            const bool start_in = h2.q_start >= h1.q_start && h2.q_start <= h1.q_end && h2.s_start >= h1.s_start &&
                                  h2.s_start <= h1.s_end;
            const bool end_in = h2.q_end >= h1.q_start && h2.q_end <= h1.q_end && h2.s_end >= h1.s_start &&
                                h2.s_end <= h1.s_end;
            if (!start_in && !end_in) continue;
            const double density = (double)(h1.score + h2.score) /
                                   (double)((h1.q_end - h1.q_start) + (h2.q_end - h2.q_start));
            h1.q_start = std::min(h1.q_start, h2.q_start);
            h1.s_start = std::min(h1.s_start, h2.s_start);
            h1.q_end = std::max(h1.q_end, h2.q_end);
            h1.s_end = std::max(h1.s_end, h2.s_end);
            if (h2.score > h1.score) {
                h1.q_seed = h2.q_seed;
                h1.s_seed = h2.s_seed;
                h1.score = h2.score;
            }
            h1.score = std::max(h1.score, (int32_t)(density * (double)(h1.q_end - h1.q_start)));
            absorbed[j] = 1;
        }
    }
    for (size_t j = 0; j < add.size(); ++j)
        if (!absorbed[j]) acc.push_back(add[j]);
}

// main.rs:1236-1251 (SplitQuery_CalculateNumChunks + x_ComputeChunkRanges): chunk starts and
// ends; a single chunk below 1,999,800 bp.
std::vector<std::pair<uint32_t, uint32_t>> query_chunks(size_t qlen, int word_size) {
    const size_t CHUNK = 1000000, OVERLAP = 100;
    const size_t n = qlen / (CHUNK - OVERLAP);
    std::vector<std::pair<uint32_t, uint32_t>> out;
    if (n <= 1) {
        out.push_back({0, (uint32_t)qlen});
        return out;
    }
    size_t cs = (qlen + (n - 1) * OVERLAP) / n;
    if (n < (cs > OVERLAP ? cs - OVERLAP : 0)) ++cs;
    const size_t step = cs > OVERLAP ? cs - OVERLAP : 0;
    for (size_t k = 0; k < n; ++k) {
        const size_t b = k * step;
        if (b >= qlen) break;
        const size_t e = std::min(b + cs, qlen);
        if (e - b < (size_t)word_size) break;
        out.push_back({(uint32_t)b, (uint32_t)e});
    }
    return out;
}

// main.rs:1281-1400 multi-chunk search of one query: DUST on the whole query (with the chunked
// off-by-one, engine.rs:697-707 / dust.rs:614-630), Phase 1 + 2a per chunk against every
// subject (engine.rs:1775-1848 search_phase2a), the cross-chunk merge per subject, then
// Phase 2b against the full query (engine.rs:1418-1431).
static std::vector<std::vector<AlignResult>> search_chunked(const std::vector<uint8_t>& query, const std::string& qid,
                                                           const std::vector<Subject>& db, const Params& p,
                                                           const Matrix& m, int threads, Counters* counters) {
    const size_t qlen = query.size() - 2;
    std::vector<uint8_t> masked = query;
    if (p.dust) {
        auto iv = dust_mask(masked);
        for (auto& [s, e] : iv)
            if (e + 1 < qlen) masked[e + 2] = 14;
    }
    Params pc = p;
    pc.dust = false;  // chunk tables come from the masked full query
    std::vector<std::vector<PrelimHsp>> acc(db.size());
    const auto chunks = query_chunks(qlen, p.word_size);
    auto run_parallel = [&](auto&& body) {
        std::atomic<size_t> next{0};
        auto worker = [&]() {
            for (;;) {
                size_t i = next.fetch_add(1);
                if (i >= db.size()) break;
                body(i);
            }
        };
        int nt = std::max(1, threads);
        std::vector<std::thread> th;
        for (int t = 1; t < nt; ++t) th.emplace_back(worker);
        worker();
        for (auto& x : th) x.join();
    };
    for (size_t k = 0; k < chunks.size(); ++k) {
        const uint32_t b = chunks[k].first, e = chunks[k].second;
        std::vector<uint8_t> chunk, mchunk;
        chunk.push_back(query.front());
        chunk.insert(chunk.end(), query.begin() + 1 + b, query.begin() + 1 + e);
        chunk.push_back(query.back());
        mchunk.push_back(masked.front());
        mchunk.insert(mchunk.end(), masked.begin() + 1 + b, masked.begin() + 1 + e);
        mchunk.push_back(masked.back());
        QueryLookup ql = build_query_lookup(mchunk, pc);
        ql.query_rc = revcomp(chunk.data(), chunk.size());
        std::vector<std::vector<PrelimHsp>> pre(db.size());
        run_parallel([&](size_t i) {
            const uint32_t q_len = (uint32_t)chunk.size() - 2, s_len = db[i].len();
            if (q_len < (uint32_t)p.word_size || s_len < (uint32_t)p.word_size) return;
            std::vector<UngappedRecord> ung;
            collect_ungapped(chunk, ql, db[i], pc, m, nullptr, ung, nullptr);
            sort_ungapped(ung, q_len, s_len);
            if (ung.empty()) return;
            pre[i] = phase2a(chunk, ql.query_rc, db[i], ung, pc, m, ql.lut.lut_word_length, nullptr);
            for (auto& h : pre[i]) {
                h.q_start += b;
                h.q_end += b;
                h.q_seed += b;
            }
        });
        for (size_t i = 0; i < db.size(); ++i) {
            if (k == 0) acc[i] = std::move(pre[i]);
            else merge_chunk_prelims(acc[i], std::move(pre[i]), b);
        }
    }
    const std::vector<uint8_t> qrc = revcomp(query.data(), query.size());
    std::vector<std::vector<AlignResult>> per(db.size());
    run_parallel([&](size_t i) {
        if (acc[i].empty()) return;
        per[i] = phase2b(query, qrc, qid, db[i], std::move(acc[i]), p, m, nullptr);
        for (auto& r : per[i]) { r.hsp.q_len = (uint32_t)qlen; r.oid = (uint32_t)i; }
    });
    return per;
}

// main.rs:1224-1234 + 758-763: E-values and bit scores for the query (ka_stats.rs:382
// for_query: the query length against the database's letters and sequences), the --evalue
// reap before masklevel, masklevel, then the hit order.
static void finish_query(std::vector<AlignResult>& res, const Params& p, const Matrix& m, size_t qlen,
                         uint64_t db_letters, size_t db_seqs) {
    const KaStats ka = resolve_stats(p.matrix_name, p.gap_open, p.gap_extend, p.cli_stats, m);
    const int64_t sp = effective_search_space(ka, (int32_t)qlen, (int64_t)db_letters, (int32_t)db_seqs);
    for (auto& r : res) {
        r.evalue = evalue_of(r.hsp.score, ka, sp);
        r.bitscore = bitscore_of(r.hsp.score, ka);
    }
    if (p.evalue > 0.0 && ka.lambda > 0.0) {
        std::vector<AlignResult> kept;
        for (auto& r : res)
            if (r.evalue <= p.evalue) kept.push_back(std::move(r));
        res.swap(kept);
    }
    apply_mask_level(res, p.mask_level);
    sort_hit_list_order(res);
}

std::vector<AlignResult> search_query(const std::vector<uint8_t>& query, const std::string& qid,
                                      const std::vector<Subject>& db, const Params& p0, const Matrix& m, int threads,
                                      Counters* counters) {
    size_t qlen = query.size() - 2;
    uint64_t total = 0;
    for (auto& s : db) total += s.len();
    uint64_t avg = db.empty() ? 0 : total / db.size();
    Params p = p0;
    p.ungapped_cutoff = ungapped_cutoff(p.matrix_name, p.gap_open, p.gap_extend, p.min_raw_gapped_score, qlen, avg);
    if (query_chunks(qlen, p.word_size).size() > 1) {
        auto per = search_chunked(query, qid, db, p, m, threads, counters);
        std::vector<AlignResult> res;
        for (auto& v : per)
            for (auto& r : v) res.push_back(std::move(r));
        finish_query(res, p, m, qlen, total, db.size());
        return res;
    }
    QueryLookup ql = build_query_lookup(query, p);
    std::vector<std::vector<AlignResult>> per(db.size());
    std::vector<Counters> ctrs(threads > 0 ? threads : 1);
    std::atomic<size_t> next{0};
    auto worker = [&](int t) {
        for (;;) {
            size_t i = next.fetch_add(1);
            if (i >= db.size()) break;
            Taps taps;
            taps.counters = counters ? &ctrs[t] : nullptr;
            per[i] = search_pair(ql, query, qid, db[i], p, m, taps);
            for (auto& r : per[i]) { r.hsp.q_len = (uint32_t)qlen; r.oid = (uint32_t)i; }
        }
    };
    int nt = std::max(1, threads);
    if (nt == 1) worker(0);
    else {
        std::vector<std::thread> th;
        for (int t = 0; t < nt; ++t) th.emplace_back(worker, t);
        for (auto& x : th) x.join();
    }
    if (counters)
        for (auto& c : ctrs) {
            counters->word_hits += c.word_hits; counters->seeds += c.seeds; counters->ungapped += c.ungapped;
            counters->prelim_dp += c.prelim_dp; counters->prelims += c.prelims; counters->tb_dp += c.tb_dp;
            counters->finals += c.finals; counters->so_cells += c.so_cells; counters->tb_cells += c.tb_cells;
        }
    std::vector<AlignResult> res;
    for (auto& v : per)
        for (auto& r : v) res.push_back(std::move(r));
    finish_query(res, p, m, qlen, total, db.size());
    return res;
}

}  // namespace rmbo
