// rmb_glue.cpp -- order-dependent host steps of the search core (see rmb_glue.hpp).
#include "rmb_glue.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <strings.h>

namespace rmb {

static const uint8_t COMP[16] = {3, 2, 1, 0, 5, 4, 7, 6, 8, 9, 13, 12, 11, 10, 14, 15};  // encoding.rs:65
static const char IUPAC[17] = "ACGTRYMKWSBDHVN-";
static constexpr int64_t MIN_DIAG_SEP = 50;  // engine.rs:173

static inline void push_op(Script& s, uint8_t op, uint32_t n) {  // hits.rs:44-53
    if (!n) return;
    if (!s.empty() && s.back().op == op) s.back().n += n;
    else s.push_back(RunOp{op, n});
}

// ---------------------------------------------------------------------------------------
// 2-D interval tree: search/itree.rs:60-555 (node arena, query axis then nested subject
// trees, endpoint-sharing dedup for add(), MB_HSP_CLOSE containment)
// ---------------------------------------------------------------------------------------
namespace {
struct Box { uint32_t qs, qe, ss, se; int32_t score; };

class ITree {
    static constexpr uint32_t LEAF_NONE = 0xFFFFFFFFu;
    struct N { uint32_t le, re, l, m, r, h; };
    std::vector<N> nd;
    std::vector<Box> hs;
    std::vector<uint8_t> dead;
    std::map<std::pair<uint32_t, uint32_t>, std::pair<int32_t, uint32_t>> lep, rep;
    uint32_t smin, smax;
    bool rcq;

    uint32_t node(uint32_t le, uint32_t re) {
        nd.push_back(N{le, re, 0, 0, 0, LEAF_NONE});
        return (uint32_t)nd.size() - 1;
    }
    uint32_t leaf(const Box& b) {
        hs.push_back(b);
        dead.push_back(0);
        nd.push_back(N{0, 0, 0, 0, 0, (uint32_t)hs.size() - 1});
        return (uint32_t)nd.size() - 1;
    }
    static std::pair<uint32_t, uint32_t> left_key(const Box& b, bool plus) {
        return plus ? std::make_pair(b.qs, b.ss) : std::make_pair(b.qe, b.ss);
    }
    static std::pair<uint32_t, uint32_t> right_key(const Box& b, bool plus) {
        return plus ? std::make_pair(b.qe, b.se) : std::make_pair(b.qs, b.se);
    }
    static bool wins(const Box& n, const Box& e) {  // itree.rs:217-228
        if (n.score != e.score) return n.score > e.score;
        if (n.qe - n.qs != e.qe - e.qs) return n.qe - n.qs < e.qe - e.qs;
        if (n.se - n.ss != e.se - e.ss) return n.se - n.ss < e.se - e.ss;
        return false;
    }
    void drop(uint32_t idx, bool plus) {  // itree.rs:198-212
        dead[idx] = 1;
        auto it = lep.find(left_key(hs[idx], plus));
        if (it != lep.end() && it->second.second == idx) lep.erase(it);
        it = rep.find(right_key(hs[idx], plus));
        if (it != rep.end() && it->second.second == idx) rep.erase(it);
    }
    void place(uint32_t ni) {  // itree.rs:251-371
        const Box b = hs[nd[ni].h];
        uint32_t lo = b.qs, hi = b.qe, root = 0;
        bool subj = false;
        for (;;) {
            const uint32_t rle = nd[root].le, rre = nd[root].re;
            const uint64_t mid = ((uint64_t)rle + rre) / 2;
            bool left;
            uint32_t old;
            if ((uint64_t)hi < mid) {
                const uint32_t c = nd[root].l;
                if (!c) { nd[root].l = ni; return; }
                if (nd[c].h == LEAF_NONE) { root = c; continue; }
                old = c;
                left = true;
            } else if ((uint64_t)lo > mid) {
                const uint32_t c = nd[root].r;
                if (!c) { nd[root].r = ni; return; }
                if (nd[c].h == LEAF_NONE) { root = c; continue; }
                old = c;
                left = false;
            } else {
                if (subj) {
                    nd[ni].m = nd[root].m;
                    nd[root].m = ni;
                    return;
                }
                subj = true;
                if (!nd[root].m) { const uint32_t t = node(smin, smax); nd[root].m = t; }
                root = nd[root].m;
                lo = b.ss;
                hi = b.se;
                continue;
            }
            const uint32_t mle = left ? rle : (uint32_t)mid + 1, mre = left ? (uint32_t)mid : rre;
            const uint32_t mi = node(mle, mre);
            if (left) nd[root].l = mi;
            else nd[root].r = mi;
            const Box o = hs[nd[old].h];
            const uint32_t olo = subj ? o.ss : o.qs, ohi = subj ? o.se : o.qe;
            root = mi;
            const uint64_t mm = ((uint64_t)mle + mre) / 2;
            if ((uint64_t)ohi < mm) nd[mi].l = old;
            else if ((uint64_t)olo > mm) nd[mi].r = old;
            else if (subj) nd[mi].m = old;
            else {
                const uint32_t m2 = node(smin, smax);
                nd[mi].m = m2;
                const uint64_t m2m = ((uint64_t)smin + smax) / 2;
                if ((uint64_t)o.se < m2m) nd[m2].l = old;
                else if ((uint64_t)o.ss > m2m) nd[m2].r = old;
                else nd[m2].m = old;
            }
        }
    }
    bool held_by(const Box& c, bool plus, uint32_t idx) const {  // itree.rs:496-554
        if (dead[idx]) return false;
        const Box& h = hs[idx];
        if (c.score > h.score) return false;
        if (!(h.qs <= c.qs && h.qe >= c.qe && h.ss <= c.ss && h.se >= c.se)) return false;
        int64_t d0, d1;
        if (plus || rcq) {
            d0 = std::llabs(((int64_t)c.qs - c.ss) - ((int64_t)h.qs - h.ss));
            d1 = std::llabs(((int64_t)c.qe - c.se) - ((int64_t)h.qe - h.se));
        } else {
            d0 = std::llabs(((int64_t)c.qe + c.ss) - ((int64_t)h.qe + h.ss));
            d1 = std::llabs(((int64_t)c.qs + c.se) - ((int64_t)h.qs + h.se));
        }
        return d0 < MIN_DIAG_SEP || d1 < MIN_DIAG_SEP;
    }
    bool mid_contains(uint32_t n, const Box& c, bool plus) const {  // itree.rs:437-494
        for (;;) {
            if (nd[n].h != LEAF_NONE) return held_by(c, plus, nd[n].h);
            for (uint32_t k = nd[n].m; k; k = nd[k].m)
                if (held_by(c, plus, nd[k].h)) return true;
            const uint64_t mid = ((uint64_t)nd[n].le + nd[n].re) / 2;
            uint32_t nx;
            if ((uint64_t)c.se < mid) nx = nd[n].l;
            else if ((uint64_t)c.ss > mid) nx = nd[n].r;
            else return false;
            if (!nx) return false;
            n = nx;
        }
    }

   public:
    ITree(uint32_t q1, uint32_t s1, bool rc_query) : smin(0), smax(s1), rcq(rc_query) {
        nd.push_back(N{0, q1, 0, 0, 0, LEAF_NONE});
    }
    bool add(const Box& b, bool plus) {  // itree.rs:151-230
        auto it = lep.find(left_key(b, plus));
        if (it != lep.end()) {
            if (!wins(b, hs[it->second.second])) return false;
            drop(it->second.second, plus);
        }
        it = rep.find(right_key(b, plus));
        if (it != rep.end()) {
            if (!wins(b, hs[it->second.second])) return false;
            drop(it->second.second, plus);
        }
        const uint32_t ni = leaf(b);
        lep[left_key(b, plus)] = {b.score, nd[ni].h};
        rep[right_key(b, plus)] = {b.score, nd[ni].h};
        place(ni);
        return true;
    }
    void add_simple(const Box& b) { place(leaf(b)); }
    bool contains(const Box& c, bool plus) const {  // itree.rs:376-435
        uint32_t n = 0;
        for (;;) {
            if (nd[n].m && mid_contains(nd[n].m, c, plus)) return true;
            const uint64_t mid = ((uint64_t)nd[n].le + nd[n].re) / 2;
            uint32_t nx;
            if ((uint64_t)c.qe < mid) nx = nd[n].l;
            else if ((uint64_t)c.qs > mid) nx = nd[n].r;
            else return false;
            if (!nx) return false;
            if (nd[nx].h != LEAF_NONE) return held_by(c, plus, nd[nx].h);
            n = nx;
        }
    }
};
}  // namespace

// ---------------------------------------------------------------------------------------
// Phase 2a filter: engine.rs:1280-1309 (sort), 1317-1411 (contain + add), 1969-2083 (purge)
// ---------------------------------------------------------------------------------------
static void purge_prelim_endpoints(std::vector<Prelim>& v, uint32_t sa) {
    const size_t n = v.size();
    if (n < 2) return;
    auto fss = [&](const Prelim& h) { return h.strand == 0 ? h.s_start : sa - h.s_end; };
    auto fse = [&](const Prelim& h) { return h.strand == 0 ? h.s_end : sa - h.s_start; };
    auto qoff = [&](const Prelim& h) { return h.strand == 0 ? h.q_start : h.q_end; };
    auto qend = [&](const Prelim& h) { return h.strand == 0 ? h.q_end : h.q_start; };
    std::vector<uint8_t> keep(n, 1);
    std::vector<uint32_t> idx(n);
    for (int pass = 0; pass < 2; ++pass) {
        for (uint32_t i = 0; i < n; ++i) idx[i] = i;
        std::sort(idx.begin(), idx.end(), [&](uint32_t a, uint32_t b) {
            const Prelim &x = v[a], &y = v[b];
            if (x.strand != y.strand) return x.strand < y.strand;
            const uint32_t k1x = pass ? qend(x) : qoff(x), k1y = pass ? qend(y) : qoff(y);
            if (k1x != k1y) return k1x < k1y;
            const uint32_t k2x = pass ? fse(x) : fss(x), k2y = pass ? fse(y) : fss(y);
            if (k2x != k2y) return k2x < k2y;
            if (x.score != y.score) return x.score > y.score;
            const uint32_t k3x = pass ? qoff(x) : qend(x), k3y = pass ? qoff(y) : qend(y);
            if (k3x != k3y) return x.strand == 0 ? k3x > k3y : k3x < k3y;
            const uint32_t k4x = pass ? fss(x) : fse(x), k4y = pass ? fss(y) : fse(y);
            if (k4x != k4y) return k4x > k4y;
            return a < b;
        });
        for (size_t i = 0; i < n;) {
            if (!keep[idx[i]]) { ++i; continue; }
            const Prelim& h0 = v[idx[i]];
            size_t j = i + 1;
            for (; j < n; ++j) {
                const Prelim& hj = v[idx[j]];
                const bool same = hj.strand == h0.strand &&
                                  (pass ? (qend(hj) == qend(h0) && fse(hj) == fse(h0))
                                        : (qoff(hj) == qoff(h0) && fss(hj) == fss(h0)));
                if (!same) break;
                keep[idx[j]] = 0;
            }
            i = j;
        }
    }
    std::vector<Prelim> out;
    out.reserve(n);
    for (size_t i = 0; i < n; ++i)
        if (keep[i]) out.push_back(v[i]);
    v.swap(out);
}

std::vector<Prelim> phase2a_filter(std::vector<UngSurvivor>& u, uint32_t qa, uint32_t sa) {
    auto ss = [&](const UngSurvivor& r) { return r.strand == 0 ? r.s_start : sa - r.s_end; };
    auto qk = [&](const UngSurvivor& r) -> uint64_t {
        if (r.strand == 0) return r.q_start;
        return ((uint64_t)qa + 1) + ((uint64_t)qa >= r.q_end ? (uint64_t)qa - r.q_end : 0);
    };
    auto sk = [&](const UngSurvivor& r) { return r.strand == 0 ? r.s_seed : sa - r.s_seed; };
    std::sort(u.begin(), u.end(), [&](const UngSurvivor& a, const UngSurvivor& b) {
        if (a.score != b.score) return a.score > b.score;
        if (ss(a) != ss(b)) return ss(a) < ss(b);
        const uint32_t la = a.s_end - a.s_start, lb = b.s_end - b.s_start;
        if (la != lb) return la > lb;
        if (qk(a) != qk(b)) return qk(a) < qk(b);
        return sk(a) < sk(b);
    });
    ITree tp(qa + 1, sa + 1, false), tm(qa + 1, sa + 1, false);
    std::vector<Prelim> out;
    for (const UngSurvivor& r : u) {
        const bool plus = r.strand == 0;
        const uint32_t cs = plus ? r.s_start : sa - r.s_end, ce = plus ? r.s_end : sa - r.s_start;
        if ((plus ? tp : tm).contains(Box{r.q_start, r.q_end, cs, ce, r.score}, plus)) continue;
        const uint32_t ns = plus ? r.p_ss : sa - r.p_se, ne = plus ? r.p_se : sa - r.p_ss;
        (plus ? tp : tm).add(Box{r.p_qs, r.p_qe, ns, ne, r.p_score}, plus);
        out.push_back(Prelim{r.tb_q, r.tb_s, r.p_qs, r.p_qe, r.p_ss, r.p_se, r.p_score, r.strand});
    }
    purge_prelim_endpoints(out, sa);
    return out;
}

void sort_prelims_for_traceback(std::vector<Prelim>& p, uint32_t qa, uint32_t sl) {  // engine.rs:1471-1485
    std::stable_sort(p.begin(), p.end(), [&](const Prelim& a, const Prelim& b) {
        const uint32_t fsa = a.strand == 0 ? a.s_start : sl - a.s_end, fsb = b.strand == 0 ? b.s_start : sl - b.s_end;
        const uint32_t fea = a.strand == 0 ? a.s_end : sl - a.s_start, feb = b.strand == 0 ? b.s_end : sl - b.s_start;
        const uint32_t qoa = a.strand == 0 ? a.q_start : qa - a.q_end, qob = b.strand == 0 ? b.q_start : qa - b.q_end;
        const uint32_t qea = a.strand == 0 ? a.q_end : qa - a.q_start, qeb = b.strand == 0 ? b.q_end : qa - b.q_start;
        if (a.score != b.score) return a.score > b.score;
        if (fsa != fsb) return fsa < fsb;
        if (fea != feb) return fea > feb;
        if (qoa != qob) return qoa < qob;
        return qea > qeb;
    });
}

// ---------------------------------------------------------------------------------------
// Phase 2b helpers
// ---------------------------------------------------------------------------------------
static std::vector<uint8_t> revcomp(const std::vector<uint8_t>& s) {
    std::vector<uint8_t> o(s.size());
    for (size_t i = 0; i < s.size(); ++i) o[i] = COMP[s[s.size() - 1 - i] & 15];
    return o;
}

// search/gapped.rs:773-820 extract_aligned
static void extract(const uint8_t* a, size_t alen, const uint8_t* b, size_t blen, size_t as, size_t bs,
                    const Script& sc, const uint8_t* mask, size_t mask_len, std::vector<uint8_t>& qa,
                    std::vector<uint8_t>& sa) {
    qa.clear();
    sa.clear();
    auto sb = [&](size_t si) -> uint8_t {
        const uint8_t v = si < blen ? (b[si] & 15) : 14;
        if (mask && si < mask_len && mask[si]) return mask[si];
        return v;
    };
    size_t qi = as, si = bs;
    for (const RunOp& o : sc)
        for (uint32_t k = 0; k < o.n; ++k) {
            if (o.op == OP_SUB) {
                qa.push_back(qi < alen ? (a[qi] & 15) : 14);
                sa.push_back(sb(si));
                ++qi;
                ++si;
            } else if (o.op == OP_GAP_S) {
                qa.push_back(qi < alen ? (a[qi] & 15) : 14);
                sa.push_back(15);
                ++qi;
            } else {
                qa.push_back(15);
                sa.push_back(sb(si));
                ++si;
            }
        }
}

// search/complexity_adjust.rs:19-132; query is sentinel-wrapped.
static bool complexity(int32_t raw, const uint8_t* query, size_t qsz, uint32_t q_start, const Script& es,
                       const GlueParams& gp, bool minus, int32_t& out) {
    uint32_t cnt[16] = {0};
    size_t nb = 0, qp = q_start;
    for (const RunOp& o : es) {
        if (o.op == OP_SUB) {
            for (uint32_t i = 0; i < o.n; ++i) {
                const size_t k = 1 + qp + i;
                if (k < qsz && query[k] != 15) {
                    uint8_t b = query[k];
                    if (minus) b = COMP[b & 15];
                    cnt[b & 15]++;
                    ++nb;
                }
            }
            qp += o.n;
        } else if (o.op == OP_GAP_S) {
            qp += o.n;
        }
    }
    double adj;
    if (gp.lambda <= 0.0 || nb == 0) {
        adj = (double)raw;
    } else {
        double tf = 0, ts = 0, tc = 0;
        for (int i = 0; i < 16; ++i) {
            const double f = gp.freqs[i];
            if (cnt[i] > 0 && f > 0.0 && std::log(f) != 0.0) {
                const double cf = (double)cnt[i];
                tf += cf * std::log(cf);
                ts += cf * std::log(f);
                tc += cf;
            }
        }
        if (tc == 0.0) return false;
        tf -= tc * std::log(tc);
        ts -= tf;
        adj = (double)raw + ts / gp.lambda + 0.999;
        if (adj < 0.0) adj = 0.0;
    }
    if (std::isnan(adj)) return false;
    const int32_t r = (int32_t)adj;
    if (r < gp.gapped_cutoff) return false;
    out = r;
    return true;
}

// stats.rs:52-245
namespace {
enum Pair { P_ID, P_TI, P_TV, P_IUBM, P_IUBS, P_GAP, P_UNK };
inline bool pure(uint8_t c) { return c == 'A' || c == 'C' || c == 'G' || c == 'T'; }
inline uint8_t bits(uint8_t c) {
    switch (c) {
        case 'A': return 1; case 'C': return 2; case 'G': return 4; case 'T': case 'U': return 8;
        case 'R': return 5; case 'Y': return 10; case 'M': return 3; case 'K': return 12; case 'W': return 9;
        case 'S': return 6; case 'B': return 14; case 'D': return 13; case 'H': return 11; case 'V': return 7;
        default: return 15;
    }
}
inline Pair kind(uint8_t a, uint8_t b) {
    if (a == '-' || b == '-') return P_GAP;
    if (a == b) return P_ID;
    if (!pure(a) || !pure(b)) return ((pure(a) ^ pure(b)) && (bits(a) & bits(b))) ? P_IUBM : P_IUBS;
    return ((a == 'A' || a == 'G') == (b == 'A' || b == 'G')) ? P_TI : P_TV;
}
inline double kimura(double p, double q) {
    const double x = (1.0 - 2.0 * p - q) * std::sqrt(1.0 - 2.0 * q);
    return x > 0.0 ? std::fabs(-0.5 * std::log(x)) * 100.0 : 100.0;
}
}  // namespace

Stats align_stats(const std::vector<uint8_t>& qb, const std::vector<uint8_t>& sb) {
    Stats st;
    uint32_t ql = 0, dl = 0, unamb = 0;
    double cti = 0.0;
    uint8_t prev_anc = ' ';
    Pair prev = P_UNK;
    for (size_t i = 0; i < qb.size(); ++i) {
        const uint8_t dq = qb[i] == 15 ? '-' : (uint8_t)IUPAC[qb[i] & 15];
        const uint8_t an = sb[i] == 15 ? '-' : (uint8_t)IUPAC[sb[i] & 15];
        if (dq != '-') ++ql;
        if (an != '-') ++dl;
        if (prev_anc == 'C' && an == 'G') {
            ++st.cpg_sites;
            const Pair cur = kind(an, dq);
            if (prev == P_TI && cur == P_TI) cti -= 1.0;
            else if (prev == P_TI || cur == P_TI) cti -= 0.9;
        }
        if (an == '-' || dq == '-') {
            if (dq == '-') ++st.query_gaps;
            else ++st.subject_gaps;
            if (an != '-') { prev_anc = an; prev = P_GAP; }
        } else {
            const Pair p = kind(an, dq);
            const bool u = pure(an) && pure(dq);
            if (p == P_ID) { ++st.matches; if (u) ++unamb; }
            else if (p == P_TI) { ++st.mismatches; if (u) { ++unamb; ++st.transitions; cti += 1.0; } }
            else if (p == P_TV) { ++st.mismatches; if (u) { ++unamb; ++st.transversions; } }
            else if (p == P_IUBS) ++st.mismatches;
            prev_anc = an;
            prev = p;
        }
    }
    if (unamb < 1) { st.kdiv = 100.0; st.cpg_kdiv = 100.0; }
    else {
        const double n = (double)unamb;
        st.kdiv = kimura((double)st.transitions / n, (double)st.transversions / n);
        st.cpg_kdiv = kimura(cti / n, (double)st.transversions / n);
    }
    st.perc_sub = ql > 0 ? ((float)st.mismatches / (float)ql) * 100.0f : 0.0f;
    st.perc_query_gap = ql > 0 ? ((float)st.query_gaps / (float)ql) * 100.0f : 0.0f;
    st.perc_db_gap = dl > 0 ? ((float)st.subject_gaps / (float)dl) * 100.0f : 0.0f;
    return st;
}

// ---- common-endpoint cuts: engine.rs:2090-2254, 2650-2716 ------------------------------
namespace {
struct CutRes { bool ok; uint32_t gq, gs; };
template <bool FROM_BACK>
CutRes cut_scan(const Script& ops, uint32_t nq, uint32_t ns, size_t& ci, uint32_t& part) {
    uint32_t gq = 0, gs = 0;
    const size_t n = ops.size();
    for (size_t k = 0; k < n; ++k) {
        const size_t i = FROM_BACK ? n - 1 - k : k;
        const RunOp o = ops[i];
        if (o.op == OP_SUB) {
            for (uint32_t j = 0; j < o.n; ++j) {
                ++gq;
                ++gs;
                if (gq >= nq && gs >= ns) { ci = i; part = j + 1; return CutRes{true, gq, gs}; }
            }
        } else {
            if (o.op == OP_GAP_Q) gs += o.n;
            else gq += o.n;
            if (gq >= nq && gs >= ns) { ci = i; part = o.n; return CutRes{true, gq, gs}; }
        }
    }
    return CutRes{false, gq, gs};
}
CutRes keep_front(Script& ops, uint32_t nq, uint32_t ns) {  // cut_ops_keep_front
    if (!nq && !ns) return CutRes{true, 0, 0};
    size_t ci = 0; uint32_t part = 0;
    const CutRes c = cut_scan<false>(ops, nq, ns, ci, part);
    if (!c.ok) return c;
    if (part < ops[ci].n) ops[ci].n = part;
    ops.resize(ci + 1);
    return c;
}
CutRes drop_front(Script& ops, uint32_t nq, uint32_t ns) {  // cut_ops_front
    if (!nq && !ns) return CutRes{true, 0, 0};
    size_t ci = 0; uint32_t part = 0;
    const CutRes c = cut_scan<false>(ops, nq, ns, ci, part);
    if (!c.ok) return c;
    const RunOp o = ops[ci];
    ops.erase(ops.begin(), ops.begin() + ci + 1);
    if (o.n - part > 0) ops.insert(ops.begin(), RunOp{o.op, o.n - part});
    return c;
}
CutRes drop_back(Script& ops, uint32_t nq, uint32_t ns) {  // cut_ops_back
    if (!nq && !ns) return CutRes{true, 0, 0};
    size_t ci = 0; uint32_t part = 0;
    const CutRes c = cut_scan<true>(ops, nq, ns, ci, part);
    if (!c.ok) return c;
    const RunOp o = ops[ci];
    ops.resize(ci);
    if (o.n - part > 0) ops.push_back(RunOp{o.op, o.n - part});
    return c;
}
CutRes keep_back(Script& ops, uint32_t nq, uint32_t ns) {  // keep_ops_back
    if (!nq && !ns) return CutRes{true, 0, 0};
    size_t ci = 0; uint32_t part = 0;
    const CutRes c = cut_scan<true>(ops, nq, ns, ci, part);
    if (!c.ok) return c;
    const RunOp o = ops[ci];
    ops.erase(ops.begin(), ops.begin() + ci);
    if (part < o.n) ops[0] = RunOp{o.op, part};
    return c;
}
inline uint32_t sub0(uint32_t a, uint32_t b) { return a > b ? a - b : 0; }
bool cut_start(const Hit& p, Hit& s) {
    if (!(p.strand == 0 ? s.q_end > p.q_end : s.q_start < p.q_start)) return false;
    if (p.strand == 0) {
        const CutRes c = drop_front(s.script, sub0(p.q_end, s.q_start), sub0(p.s_end, s.s_start));
        if (c.ok) { s.q_start += c.gq; s.s_start += c.gs; }
    } else {
        const CutRes c = drop_back(s.script, sub0(s.q_end, p.q_start), sub0(p.s_end, s.s_start));
        if (c.ok) { s.q_end -= c.gq; s.s_start += c.gs; }
    }
    return !s.script.empty();
}
bool cut_end(const Hit& p, Hit& s) {
    if (!(p.strand == 0 ? s.q_start < p.q_start : s.q_end > p.q_end)) return false;
    if (p.strand == 0) {
        const CutRes c = keep_front(s.script, sub0(p.q_start, s.q_start), sub0(p.s_start, s.s_start));
        if (c.ok) { s.q_end = s.q_start + c.gq; s.s_end = s.s_start + c.gs; }
    } else {
        const CutRes c = keep_back(s.script, sub0(s.q_end, p.q_end), sub0(p.s_start, s.s_start));
        if (c.ok) { s.q_start = sub0(s.q_end, c.gq); s.s_end = s.s_start + c.gs; }
    }
    return !s.script.empty();
}
bool less_qoff(const Hit* a, const Hit* b) {  // engine.rs:2592
    if (a->strand != b->strand) return a->strand < b->strand;
    const uint32_t ka = a->strand == 0 ? a->q_start : a->q_end, kb = b->strand == 0 ? b->q_start : b->q_end;
    if (ka != kb) return ka < kb;
    if (a->s_start != b->s_start) return a->s_start < b->s_start;
    if (a->score != b->score) return a->score > b->score;
    if (a->strand == 0) { if (a->q_end != b->q_end) return a->q_end > b->q_end; }
    else if (a->q_start != b->q_start) return a->q_start < b->q_start;
    return a->s_end > b->s_end;
}
bool less_qend(const Hit* a, const Hit* b) {  // engine.rs:2611
    if (a->strand != b->strand) return a->strand < b->strand;
    const uint32_t ka = a->strand == 0 ? a->q_end : a->q_start, kb = b->strand == 0 ? b->q_end : b->q_start;
    if (ka != kb) return ka < kb;
    if (a->s_end != b->s_end) return a->s_end < b->s_end;
    if (a->score != b->score) return a->score > b->score;
    if (a->strand == 0) { if (a->q_start != b->q_start) return a->q_start > b->q_start; }
    else if (a->q_end != b->q_end) return a->q_end < b->q_end;
    return a->s_start > b->s_start;
}
bool same_start(const Hit& a, const Hit& b) {
    return a.strand == b.strand && (a.strand == 0 ? a.q_start : a.q_end) == (b.strand == 0 ? b.q_start : b.q_end) &&
           a.s_start == b.s_start;
}
bool same_end(const Hit& a, const Hit& b) {
    return a.strand == b.strand && (a.strand == 0 ? a.q_end : a.q_start) == (b.strand == 0 ? b.q_end : b.q_start) &&
           a.s_end == b.s_end;
}
// engine.rs:2743-2769
size_t collapse(std::vector<Hit*>& arr, size_t count, bool purge, bool (*same)(const Hit&, const Hit&),
                bool (*cut)(const Hit&, Hit&)) {
    std::vector<Hit*> removed;
    size_t surv = 0;
    for (size_t r = 0; r < count; ++r) {
        if (surv > 0 && same(*arr[surv - 1], *arr[r])) {
            Hit* sec = arr[r];
            arr[r] = nullptr;
            const bool keep = !purge && cut(*arr[surv - 1], *sec);
            removed.push_back(keep ? sec : nullptr);
        } else {
            std::swap(arr[surv], arr[r]);
            ++surv;
        }
    }
    size_t k = removed.size();
    for (size_t i = surv; i < count; ++i) arr[i] = removed[--k];
    return surv;
}
// engine.rs:2717-2741
size_t purge_common(std::vector<Hit*>& arr, bool purge) {
    const size_t n = arr.size();
    if (n < 2) return n;
    std::stable_sort(arr.begin(), arr.begin() + n, less_qoff);
    const size_t c = collapse(arr, n, purge, same_start, cut_start);
    std::stable_sort(arr.begin(), arr.begin() + c, less_qend);
    return collapse(arr, c, purge, same_end, cut_end);
}

// engine.rs:2268-2567 reevaluate_gapped; true = delete
bool reevaluate(Hit& h, const std::vector<uint8_t>& q_seq, const std::vector<uint8_t>& s_seq, const GlueParams& gp,
                bool minus, const uint8_t* rq, size_t rqn, size_t q0, const uint8_t* rs, size_t rsn, size_t s0) {
    if (h.script.empty()) return true;
    const int32_t min_score = gp.gapped_cutoff;
    int32_t sum = 0, score = 0;
    size_t si = 0;
    uint32_t qp = 0, sp = 0, bqs = 0, bss = 0, bqe = 0, bse = 0, cqs = 0, css = 0;
    size_t bsi = 0, bei = 0, csi = 0;
    uint32_t ben = 0, cskip = 0, bskip = 0;
    const Script snap = h.script;
    const size_t esp = snap.size();
    Script rops = snap;
    std::vector<uint8_t> rqv = q_seq, rsv = s_seq;
    if (minus) {
        std::reverse(rops.begin(), rops.end());
        std::reverse(rqv.begin(), rqv.end());
        std::reverse(rsv.begin(), rsv.end());
    }
    for (size_t ei = 0; ei < rops.size(); ++ei) {
        const RunOp o = rops[ei];
        if (o.op == OP_SUB) {
            for (uint32_t k = 0; k < o.n; ++k) {
                uint8_t qb = (si < rqv.size() ? rqv[si] : 14) & 15, sb = (si < rsv.size() ? rsv[si] : 14) & 15;
                if (minus) { qb = COMP[qb] & 15; sb = COMP[sb] & 15; }
                sum += gp.matrix[qb][sb];
                ++si; ++qp; ++sp;
                const uint32_t oi = k + 1;
                if (sum < 0) {
                    if (oi < o.n) { csi = ei; cskip = oi; }
                    else { csi = ei + 1; cskip = 0; }
                    sum = 0; cqs = qp; css = sp;
                    if (score < min_score) {
                        bqs = qp; bss = sp; score = 0;
                        bsi = csi; bskip = cskip; bei = csi; ben = 0;
                    }
                } else if (sum > score) {
                    score = sum;
                    bqs = cqs; bss = css; bqe = qp; bse = sp;
                    bsi = csi; bskip = cskip; bei = ei; ben = oi;
                }
            }
        } else {
            sum -= gp.gap_open + gp.gap_extend * (int32_t)o.n;
            si += o.n;
            if (o.op == OP_GAP_Q) sp += o.n;
            else qp += o.n;
            if (sum < 0) {
                csi = ei + 1; cskip = 0; sum = 0; cqs = qp; css = sp;
                if (score < min_score) {
                    bqs = qp; bss = sp; score = 0;
                    bsi = csi; bskip = 0; bei = csi; ben = 0;
                }
            } else if (sum > score) {
                score = sum;
                bqs = cqs; bss = css; bqe = qp; bse = sp;
                bsi = csi; bskip = cskip; bei = ei; ben = o.n;
            }
        }
    }
    if (score < min_score) return true;
    if (minus) {
        uint32_t qt = 0, st = 0;
        for (const RunOp& o : snap) {
            if (o.op == OP_SUB) { qt += o.n; st += o.n; }
            else if (o.op == OP_GAP_S) qt += o.n;
            else st += o.n;
        }
        const size_t fs = esp - 1 - bei, fe = esp - 1 - bsi;
        const uint32_t fen = snap[fe].n - bskip, fsk = snap[fs].n - ben;
        const uint32_t a1 = qt - bqe, a2 = qt - bqs, a3 = st - bse, a4 = st - bss;
        bsi = fs; bei = fe; bskip = fsk; ben = fen; bqs = a1; bqe = a2; bss = a3; bse = a4;
    }
    Script& ops = h.script;
    if (bei < (esp ? esp - 1 : 0) || ben < snap[bei].n) {
        ops.resize(bei + 1);
        if (ben > 0) ops[bei].n = ben;
        else ops.resize(bei);
    }
    if (bsi > 0) ops.erase(ops.begin(), ops.begin() + std::min(bsi, ops.size()));
    if (bskip > 0 && !ops.empty()) {
        if (bskip < ops[0].n) ops[0].n -= bskip;
        else ops.erase(ops.begin());
    }
    int64_t xqs = bqs, xss = bss, xqe = bqe, xse = bse;
    for (;;) {
        const int64_t qi = (int64_t)q0 + xqs, sj = (int64_t)s0 + xss;
        if (qi <= 0 || sj <= 0) break;
        const uint8_t qb = rq[qi - 1], sb = rs[sj - 1];
        if (!(qb < 4 && qb == sb)) break;
        --xqs; --xss;
        if (!ops.empty() && ops.front().op == OP_SUB) ops[0].n += 1;
        else ops.insert(ops.begin(), RunOp{OP_SUB, 1});
    }
    for (;;) {
        const int64_t qi = (int64_t)q0 + xqe, sj = (int64_t)s0 + xse;
        if (qi >= (int64_t)rqn || sj >= (int64_t)rsn) break;
        const uint8_t qb = rq[qi], sb = rs[sj];
        if (!(qb < 4 && qb == sb)) break;
        ++xqe; ++xse;
        if (!ops.empty() && ops.back().op == OP_SUB) ops.back().n += 1;
        else ops.push_back(RunOp{OP_SUB, 1});
    }
    h.score = score;
    auto c0 = [](int64_t v) { return (uint32_t)(v < 0 ? 0 : v); };
    if (minus) {
        const int64_t oq = h.q_start, ose = h.s_end;
        h.q_start = c0(oq + xqs);
        h.q_end = c0(oq + xqe);
        h.s_end = c0(ose - xss);
        h.s_start = c0(ose - xse);
    } else {
        const int64_t oq = h.q_start, os = h.s_start;
        h.q_start = c0(oq + xqs);
        h.q_end = h.q_start + (uint32_t)(xqe - xqs);
        h.s_start = c0(os + xss);
        h.s_end = h.s_start + (uint32_t)(xse - xss);
    }
    return false;
}
}  // namespace

std::vector<Hit> phase2b_filter(std::vector<Prelim>& pre, std::vector<TbResult>& tbs, const uint8_t* query,
                                const uint8_t* query_rc, uint32_t qa, const SubjectView& sv, uint32_t oid,
                                const GlueParams& gp) {
    const uint32_t sl = sv.len;
    const size_t qsz = (size_t)qa + 2;
    ITree tp(qa + 1, sl + 1, false), tm(qa + 1, sl + 1, true);
    std::vector<Hit> res;
    std::vector<uint8_t> qb, sb;
    for (size_t k = 0; k < pre.size(); ++k) {
        const Prelim& ph = pre[k];
        const bool plus = ph.strand == 0;
        const uint32_t ps = plus ? ph.s_start : sl - ph.s_end, pe = plus ? ph.s_end : sl - ph.s_start;
        const uint32_t cqs = plus ? ph.q_start : qa - ph.q_end, cqe = plus ? ph.q_end : qa - ph.q_start;
        if ((plus ? tp : tm).contains(Box{cqs, cqe, ps, pe, ph.score}, plus)) continue;
        TbResult& t = tbs[k];
        if (t.status != 0) continue;  // no alignment (score < 0)
        int32_t sc = t.score;
        uint32_t qs, qe, ss, se;
        if (!plus) {
            extract(query_rc + 1, qa, sv.align + 1, sl, t.q0, t.s0, t.script, sv.n_mask, sv.n_mask ? sl : 0, qb, sb);
            qb = revcomp(qb);
            sb = revcomp(sb);
            qs = qa - t.q1; qe = qa - t.q0; ss = sl - t.s1; se = sl - t.s0;
            std::reverse(t.script.begin(), t.script.end());
        } else {
            extract(query + 1, qa, sv.align + 1, sl, t.q0, t.s0, t.script, sv.n_mask, sv.n_mask ? sl : 0, qb, sb);
            qs = t.q0; qe = t.q1; ss = t.s0; se = t.s1;
        }
        if (gp.complexity_adjust) {
            int32_t adj;
            if (!complexity(sc, query, qsz, qs, t.script, gp, !plus, adj)) continue;
            sc = adj;
        }
        const uint32_t rss = plus ? ss : sl - se, rse = plus ? se : sl - ss;
        (plus ? tp : tm).add(Box{plus ? qs : qa - qe, plus ? qe : qa - qs, rss, rse, sc}, true);
        Hit h;
        h.score = sc;
        h.q_start = qs; h.q_end = qe; h.q_len = qa;
        h.s_start = rss; h.s_end = rse; h.s_len = sl;
        h.oid = oid;
        h.strand = ph.strand;
        h.script = std::move(t.script);
        h.q_seq = qb;
        h.s_seq = sb;
        h.stats = align_stats(qb, sb);
        res.push_back(std::move(h));
    }
    // engine.rs:1648-1726: purge(FALSE) cut, re-evaluate the cut remainders, purge(TRUE)
    {
        std::vector<Hit> store = std::move(res);
        res.clear();
        std::vector<Hit*> arr;
        for (auto& h : store) arr.push_back(&h);
        const size_t extra = purge_common(arr, false);
        const uint8_t* qcore = query + 1;
        const uint8_t* pcore = sv.align + 1;
        const uint8_t* rcore = sv.align_rc + 1;
        for (size_t i = extra; i < arr.size(); ++i) {
            Hit* h = arr[i];
            if (!h) continue;
            const bool minus = h->strand == 1;
            const size_t as = h->q_start, bs = minus ? (size_t)(sl - h->s_end) : h->s_start;
            const uint8_t* bc = minus ? rcore : pcore;
            const uint8_t* bm = minus ? sv.n_mask_rc : sv.n_mask;
            std::vector<uint8_t> q1, s1;
            extract(qcore, qa, bc, sl, as, bs, h->script, bm, bm ? sl : 0, q1, s1);
            if (reevaluate(*h, q1, s1, gp, minus, qcore, qa, as, bc, sl, bs)) { arr[i] = nullptr; continue; }
            const size_t as2 = h->q_start, bs2 = minus ? (size_t)(sl - h->s_end) : h->s_start;
            extract(qcore, qa, bc, sl, as2, bs2, h->script, bm, bm ? sl : 0, q1, s1);
            h->stats = align_stats(q1, s1);
            h->q_seq = q1;
            h->s_seq = s1;
        }
        std::vector<Hit*> arr2;
        for (Hit* h : arr)
            if (h) arr2.push_back(h);
        purge_common(arr2, true);
        for (Hit* h : arr2)
            if (h) res.push_back(std::move(*h));
    }
    // Phase 2c: engine.rs:1732-1759
    std::stable_sort(res.begin(), res.end(), [&](const Hit& a, const Hit& b) {
        const uint32_t qoa = a.strand == 0 ? a.q_start : qa - a.q_end, qob = b.strand == 0 ? b.q_start : qa - b.q_end;
        const uint32_t qea = a.strand == 0 ? a.q_end : qa - a.q_start, qeb = b.strand == 0 ? b.q_end : qa - b.q_start;
        if (a.score != b.score) return a.score > b.score;
        if (a.s_start != b.s_start) return a.s_start < b.s_start;
        if (a.s_end != b.s_end) return a.s_end > b.s_end;
        if (qoa != qob) return qoa < qob;
        return qea > qeb;
    });
    ITree fp(qa + 1, sl + 1, false), fm(qa + 1, sl + 1, false);
    std::vector<Hit> kept;
    for (auto& h : res) {
        const bool plus = h.strand == 0;
        const Box b{h.q_start, h.q_end, h.s_start, h.s_end, h.score};
        if ((plus ? fp : fm).contains(b, plus)) continue;
        (plus ? fp : fm).add_simple(b);
        kept.push_back(std::move(h));
    }
    return kept;
}

// ---------------------------------------------------------------------------------------
// per query: masklevel (engine.rs:863-974) and order (main.rs:1230-1234, engine.rs:998-1017)
// ---------------------------------------------------------------------------------------
void apply_mask_level(std::vector<Hit>& r, uint32_t level) {
    if (level >= 100) return;
    std::sort(r.begin(), r.end(), [](const Hit& a, const Hit& b) {
        if (a.score != b.score) return a.score > b.score;
        if (a.oid != b.oid) return a.oid > b.oid;
        if (a.s_start != b.s_start) return a.s_start < b.s_start;
        if (a.s_end != b.s_end) return a.s_end > b.s_end;
        const uint32_t qoa = a.strand == 0 ? a.q_start : a.q_len - a.q_end, qob = b.strand == 0 ? b.q_start : b.q_len - b.q_end;
        if (qoa != qob) return qoa < qob;
        const uint32_t qea = a.strand == 0 ? a.q_end : a.q_len - a.q_start, qeb = b.strand == 0 ? b.q_end : b.q_len - b.q_start;
        return qea > qeb;
    });
    // accepted spans keyed by start; a span that ends before the candidate starts cannot
    // mask it, so only starts in [qs - longest accepted span, hi] are visited.
    std::multimap<uint32_t, std::pair<uint32_t, int32_t>> acc;
    uint32_t longest = 0;
    const bool touching = level == 0;
    std::vector<Hit> out;
    out.reserve(r.size());
    for (auto& h : r) {
        uint32_t qs = h.q_start, qe = h.q_end;
        if (h.strand == 1) { ++qs; ++qe; }
        const int64_t span = (int64_t)qe - qs;
        if (span == 0) continue;
        const uint32_t hi = touching ? qe : qe - 1;
        const uint32_t lo = qs > longest ? qs - longest : 0;
        bool masked = false;
        for (auto it = acc.lower_bound(lo); it != acc.end() && it->first <= hi; ++it) {
            const uint32_t qsj = it->first, qej = it->second.first;
            if (qej < qs || (qej == qs && !touching)) continue;
            if (it->second.second < h.score) continue;
            const int64_t ov = (int64_t)std::min(qej, qe) - (int64_t)std::max(qsj, qs);
            if ((int64_t)(100.0 * ((double)ov / (double)span)) >= (int64_t)level) { masked = true; break; }
        }
        if (masked) continue;
        acc.emplace(qs, std::make_pair(qe, h.score));
        longest = std::max(longest, qe - qs);
        out.push_back(std::move(h));
    }
    r.swap(out);
}

void sort_hit_list_order(std::vector<Hit>& r, const std::vector<std::string>& ids) {
    std::sort(r.begin(), r.end(), [&](const Hit& a, const Hit& b) {
        const int c = ids[a.oid].compare(ids[b.oid]);
        if (c != 0) return c < 0;
        if (a.strand != b.strand) return a.strand < b.strand;
        return a.q_start < b.q_start;
    });
    std::map<uint32_t, int32_t> best;
    for (auto& h : r) {
        auto it = best.find(h.oid);
        if (it == best.end()) best.emplace(h.oid, h.score);
        else it->second = std::max(it->second, h.score);
    }
    std::stable_sort(r.begin(), r.end(), [&](const Hit& a, const Hit& b) {
        const int32_t ba = best[a.oid], bb = best[b.oid];
        if (ba != bb) return ba > bb;
        if (a.oid != b.oid) return a.oid > b.oid;
        const uint32_t qoa = a.strand == 0 ? a.q_start : a.q_len - a.q_end, qob = b.strand == 0 ? b.q_start : b.q_len - b.q_end;
        const uint32_t qea = a.strand == 0 ? a.q_end : a.q_len - a.q_start, qeb = b.strand == 0 ? b.q_end : b.q_len - b.q_start;
        if (a.score != b.score) return a.score > b.score;
        if (a.s_start != b.s_start) return a.s_start < b.s_start;
        if (a.s_end != b.s_end) return a.s_end > b.s_end;
        if (qoa != qob) return qoa < qob;
        return qea > qeb;
    });
}

bool format_line(std::string& out, const Hit& h, const std::string& qid, const std::string& sid,
                 const std::vector<std::string>& fields) {
    char buf[64];
    const uint32_t s1 = h.s_start + 1, se = h.s_end;
    bool first = true;
    for (const std::string& f : fields) {
        if (!first) out.push_back('\t');
        first = false;
        if (f == "score") out += std::to_string(h.score);
        else if (f == "perc_sub") { snprintf(buf, sizeof buf, "%.2f", (double)h.stats.perc_sub); out += buf; }
        else if (f == "perc_query_gap") { snprintf(buf, sizeof buf, "%.2f", (double)h.stats.perc_query_gap); out += buf; }
        else if (f == "perc_db_gap") { snprintf(buf, sizeof buf, "%.2f", (double)h.stats.perc_db_gap); out += buf; }
        else if (f == "qseqid") out += qid;
        else if (f == "qstart") out += std::to_string(h.q_start + 1);
        else if (f == "qend") out += std::to_string(h.q_end);
        else if (f == "qlen") out += std::to_string(h.q_len);
        else if (f == "sstrand") out += h.strand == 0 ? "plus" : "minus";
        else if (f == "sseqid") out += sid;
        else if (f == "sstart") out += std::to_string(h.strand == 0 ? s1 : se);
        else if (f == "send") out += std::to_string(h.strand == 0 ? se : s1);
        else if (f == "slen") out += std::to_string(h.s_len);
        else if (f == "kdiv") { snprintf(buf, sizeof buf, "%.2f", h.stats.kdiv); out += buf; }
        else if (f == "cpg_kdiv") { snprintf(buf, sizeof buf, "%.2f", h.stats.cpg_kdiv); out += buf; }
        else if (f == "transi") out += std::to_string(h.stats.transversions);  // output.rs:160-164
        else if (f == "transv") out += std::to_string(h.stats.cpg_sites);
        else if (f == "cpg_sites") out += std::to_string(h.stats.transitions);
        else if (f == "qseq") for (uint8_t b : h.q_seq) out.push_back(b == 15 ? '-' : IUPAC[b & 15]);
        else if (f == "sseq") for (uint8_t b : h.s_seq) out.push_back(b == 15 ? '-' : IUPAC[b & 15]);
        else if (f == "evalue") append_evalue(out, h.evalue);
        else if (f == "bitscore") append_bitscore(out, h.bitscore);
        else return false;
    }
    return true;
}

// ---------------------------------------------------------------------------------------
// Karlin-Altschul statistics for E-values and bit scores (rmblast-lib/src/ka_stats.rs:153-300,
// rmblast-stats/rmstats: rmblast_tables.rs, eff_lengths.rs, length_adjust.rs, evalue.rs)
// ---------------------------------------------------------------------------------------
namespace {
// rmstats tables_data.rs: RMBlast's gapped (lambda, K, H) per matrix file name and gap costs,
// with the refitted 30p53g row and comparison.matrix; kept value for value.
struct KaStatRow { const char* name; int go, ge; double lambda, k, h; };
const KaStatRow KA_STATS[] = {
    {"14p35g.matrix", 29, 6, 0.1241860392, 0.2565118357, 0.3349210581}, {"14p37g.matrix", 29, 6, 0.1243509013, 0.2538327145, 0.3484386549},
    {"14p39g.matrix", 29, 6, 0.118108197, 0.2381799563, 0.3209988017}, {"14p41g.matrix", 29, 6, 0.1209164962, 0.251696198, 0.3474870514},
    {"14p43g.matrix", 29, 6, 0.1204338701, 0.2484920137, 0.3397421893}, {"14p45g.matrix", 29, 6, 0.1281012415, 0.2651519027, 0.3664022073},
    {"14p47g.matrix", 29, 6, 0.116957149, 0.2334091021, 0.3226817428}, {"14p49g.matrix", 29, 6, 0.1167697593, 0.2289233061, 0.3136272703},
    {"14p51g.matrix", 29, 6, 0.1238779017, 0.2467119379, 0.32413383}, {"14p53g.matrix", 29, 6, 0.1211022467, 0.2307304663, 0.2949314272},
    {"18p35g.matrix", 28, 5, 0.120477663, 0.2111410357, 0.2484902185}, {"18p37g.matrix", 28, 5, 0.1213800379, 0.2057492194, 0.2637651575},
    {"18p39g.matrix", 28, 5, 0.1228853168, 0.2111281814, 0.2802003038}, {"18p41g.matrix", 28, 5, 0.1096830298, 0.1715966796, 0.2171487218},
    {"18p43g.matrix", 28, 5, 0.1179924113, 0.1957371364, 0.2544060456}, {"18p45g.matrix", 28, 5, 0.1184247414, 0.2068045787, 0.2641082233},
    {"18p47g.matrix", 28, 5, 0.115878332, 0.1842046578, 0.2407688057}, {"18p49g.matrix", 28, 5, 0.1248964218, 0.2141853759, 0.2675489103},
    {"18p51g.matrix", 28, 5, 0.1106793836, 0.1621592148, 0.1979815532}, {"18p53g.matrix", 28, 5, 0.1082347513, 0.1408677318, 0.1771724651},
    {"20p35g.matrix", 25, 5, 0.1112832877, 0.1466667286, 0.1741696491}, {"20p37g.matrix", 25, 5, 0.1134511409, 0.1501236494, 0.193180875},
    {"20p39g.matrix", 25, 5, 0.1233401001, 0.1853070864, 0.2324952723}, {"20p41g.matrix", 25, 5, 0.1088138918, 0.1409300313, 0.1778018484},
    {"20p43g.matrix", 25, 5, 0.1097495426, 0.1408421343, 0.1813610542}, {"20p45g.matrix", 25, 5, 0.1101110565, 0.1402262486, 0.1803401526},
    {"20p47g.matrix", 25, 5, 0.1198508511, 0.175230183, 0.2232474228}, {"20p49g.matrix", 25, 5, 0.1150022018, 0.1500562415, 0.1891763921},
    {"20p51g.matrix", 25, 5, 0.1101356126, 0.1310353805, 0.1457676446}, {"20p53g.matrix", 25, 5, 0.1239625969, 0.1752022586, 0.210665934},
    {"25p35g.matrix", 22, 5, 0.0965155465, 0.0677355511, 0.0964040436}, {"25p37g.matrix", 22, 5, 0.0989264764, 0.076371967, 0.1025772304},
    {"25p39g.matrix", 22, 5, 0.1005843197, 0.0805691511, 0.1108913867}, {"25p41g.matrix", 22, 5, 0.1030661339, 0.0840485952, 0.1237017673},
    {"25p43g.matrix", 22, 5, 0.115543436, 0.1226554129, 0.1495157932}, {"25p45g.matrix", 22, 5, 0.0973402625, 0.074202019, 0.1029029688},
    {"25p47g.matrix", 22, 5, 0.0967346256, 0.0743885008, 0.0995494785}, {"25p49g.matrix", 22, 5, 0.1070577141, 0.0941947942, 0.1181023643},
    {"25p51g.matrix", 22, 5, 0.1044972455, 0.0789036639, 0.1081508568}, {"25p53g.matrix", 22, 5, 0.0977828435, 0.0607500307, 0.0834178835},
    {"30p53g.matrix", 22, 5, 0.1204393447, 0.1065198197, 0.1243912966}, {"comparison.matrix", 20, 5, 0.09836223, 0.0789918084, 0.1116129577},
};
}  // namespace

int ka_resolve(const std::string& matrix_name, int go, int ge, const double cli[4], const double* karlin,
               KaBlock& out) {
    std::string base = matrix_name;
    const size_t sl = base.find_last_of('/');
    if (sl != std::string::npos) base = base.substr(sl + 1);
    const bool cli_set = cli && cli[0] > 0.0 && cli[1] > 0.0 && cli[2] > 0.0;
    out = KaBlock{};
    for (const KaStatRow& r : KA_STATS) {  // the table, by base name and exact gap costs
        if (r.go != go || r.ge != ge || strcasecmp(r.name, base.c_str()) != 0) continue;
        out.lambda = r.lambda;
        out.k = r.k;
        out.log_k = std::log(r.k);
        out.h = r.h;
        // eff_lengths.rs: alpha/beta from the command line when given, else lambda/H and 0
        out.alpha = cli_set ? cli[2] : r.lambda / r.h;
        out.beta = cli_set ? cli[3] : 0.0;
        return KA_TABLE;
    }
    auto cli_like = [&](double lambda, double k, double alpha, double beta) {
        out.lambda = lambda;
        out.k = k;
        out.log_k = std::log(k);
        out.h = lambda / alpha;
        out.alpha = alpha;
        out.beta = beta;
    };
    if (cli_set) {
        cli_like(cli[0], cli[1], cli[2], cli[3]);
        return KA_CLI;
    }
    if (karlin) {  // a "# KARLIN" matrix comment: lambda, K, H, alpha, beta (alpha = lambda/H if absent)
        const double alpha = karlin[3] > 0.0 ? karlin[3] : karlin[2] > 0.0 ? karlin[0] / karlin[2] : 0.0;
        if (karlin[0] > 0.0 && karlin[1] > 0.0 && alpha > 0.0) {
            cli_like(karlin[0], karlin[1], alpha, karlin[4]);
            return KA_MATRIX_COMMENT;
        }
    }
    return KA_NONE;  // the sentinel: E-value 1.0, bit score 0.0, nothing reaped
}

// length_adjust.rs (BLAST_ComputeLengthAdjustment): the fixed point of
// ell = alpha/lambda * (ln K + ln((m - ell)(n - N ell))) + beta, by bisection.
static int32_t length_adjustment(double k, double log_k, double alpha_d_lambda, double beta, int32_t qlen,
                                 int64_t db_len, int32_t db_num) {
    const int kMaxIter = 20;
    const double m = qlen, n = (double)db_len, bn = db_num;
    double ell_min = 0.0, ell_max, ell_next = 0.0;
    bool converged = false;
    {
        const double a = bn, mb = m * bn + n, c = n * m - std::max(m, n) / k;
        if (c < 0.0) return 0;
        ell_max = 2.0 * c / (mb + std::sqrt(mb * mb - 4.0 * a * c));
    }
    for (int i = 1; i <= kMaxIter; ++i) {
        const double ell = ell_next;
        const double ss = (m - ell) * (n - bn * ell);
        const double ell_bar = alpha_d_lambda * (log_k + std::log(ss)) + beta;
        if (ell_bar >= ell) {
            ell_min = ell;
            if (ell_bar - ell_min <= 1.0) {
                converged = true;
                break;
            }
            if (ell_min == ell_max) break;
        } else {
            ell_max = ell;
        }
        if (ell_min <= ell_bar && ell_bar <= ell_max) ell_next = ell_bar;
        else ell_next = i == 1 ? ell_max : (ell_min + ell_max) / 2.0;
    }
    int32_t la = (int32_t)ell_min;
    if (converged) {
        const double ell = std::ceil(ell_min);
        if (ell <= ell_max) {
            const double ss = (m - ell) * (n - bn * ell);
            if (alpha_d_lambda * (log_k + std::log(ss)) + beta >= ell) la = (int32_t)ell;
        }
    }
    return la;
}

int64_t eff_searchsp(const KaBlock& kb, int32_t qlen, int64_t db_len, int32_t db_num) {  // eff_lengths.rs
    if (qlen <= 0 || !(kb.lambda > 0.0)) return 0;
    const int32_t la = length_adjustment(kb.k, kb.log_k, kb.alpha / kb.lambda, kb.beta, qlen, db_len, db_num);
    int64_t eff_db = db_len - (int64_t)db_num * (int64_t)la;
    if (eff_db <= 0) eff_db = 1;
    return eff_db * (int64_t)(qlen - la);
}

double hsp_evalue(int32_t score, const KaBlock& kb, int64_t searchsp) {  // evalue.rs hsp_evalue
    if (!(kb.lambda > 0.0)) return 1.0;
    if (kb.lambda < 0.0 || kb.k < 0.0 || kb.h < 0.0) return -1.0;
    return (double)searchsp * std::exp(-kb.lambda * (double)score + kb.log_k);
}

double hsp_bitscore(int32_t score, const KaBlock& kb) {  // evalue.rs hsp_bit_score
    if (!(kb.lambda > 0.0)) return 0.0;
    return ((double)score * kb.lambda - kb.log_k) / 0.6931471805599453;
}

// output.rs:244-289: NCBI's tabular renderings (CAlignFormatUtil::GetScoreString)
static void c_sci(std::string& out, double v, int prec) {
    char buf[64];
    snprintf(buf, sizeof buf, "%.*e", prec, v);
    out += buf;
}
void append_evalue(std::string& out, double e) {
    char buf[64];
    if (e < 1.0e-180) { out += "0.0"; return; }
    if (e < 0.0009) { c_sci(out, e, 2); return; }
    if (e < 0.1) snprintf(buf, sizeof buf, "%.3f", e);
    else if (e < 1.0) snprintf(buf, sizeof buf, "%.2f", e);
    else if (e < 10.0) snprintf(buf, sizeof buf, "%.1f", e);
    else snprintf(buf, sizeof buf, "%.0f", e);
    out += buf;
}
void append_bitscore(std::string& out, double b) {
    char buf[64];
    if (b > 99999.0) { c_sci(out, b, 3); return; }
    if (b > 99.9) snprintf(buf, sizeof buf, "%3ld", (long)b);
    else snprintf(buf, sizeof buf, "%4.1f", b);
    out += buf;
}

// ---------------------------------------------------------------------------------------
// Pairwise output, outfmt 0 (rmblast-lib/src/output.rs:25-126, 369-720)
// ---------------------------------------------------------------------------------------
static std::string commas(uint64_t n) {  // NStr::Int8ToString(n, fWithCommas)
    const std::string d = std::to_string(n);
    std::string o;
    for (size_t i = 0; i < d.size(); ++i) {
        if (i > 0 && (d.size() - i) % 3 == 0) o.push_back(',');
        o.push_back(d[i]);
    }
    return o;
}

// NStr::Wrap(fWrap_FlatFile) as output.rs:44-106: break after a space, a comma or a hyphen
// (spaces preferred), forced at `width`
static std::vector<std::string> wrap_flat(const std::string& s, size_t width) {
    const size_t len = s.size();
    std::vector<std::string> lines;
    size_t pos = 0;
    while (pos < len) {
        size_t column = 0, best_pos = SIZE_MAX;
        int best = 0;  // 0 forced, 1 hyphen, 2 comma, 3 space, 4 newline
        size_t nl = s.find('\n', pos);
        if (nl == std::string::npos) nl = len;
        const size_t pos0 = nl - pos <= width ? nl : pos;
        for (size_t p2 = pos0; p2 < len && column <= width; ++p2, ++column) {
            const char c = s[p2];
            int score = 0;
            size_t sp = p2;
            if (c == '\n') {
                best_pos = p2;
                best = 4;
                break;
            }
            if (std::isspace((unsigned char)c)) score = 3;
            else if (c == ',' && column < width && sp < len - 1) { score = 2; ++sp; }
            else if (c == '-' && sp < len - 1 && column < width) { score = 1; ++sp; }
            if (score >= best && sp > pos0) {
                best_pos = sp;
                best = score;
            }
        }
        if (best != 4 && column <= width) best_pos = len;
        best_pos = std::max(std::min(best_pos, len), pos + 1);
        lines.push_back(s.substr(pos, best_pos - pos));
        pos = best_pos;
        if (best == 3) {
            while (pos < len && s[pos] == ' ') ++pos;
            if (pos < len && s[pos] == '\n') ++pos;
        } else if (best == 4) {
            ++pos;
        }
    }
    if (lines.empty()) lines.push_back("");
    return lines;
}

// s_WrapOutputLine as output.rs:108-126: past every 60th character, a break after the next
// whitespace character
static std::string wrap_title(const std::string& s) {
    if (s.size() <= 60) return s;
    std::string o;
    bool wrap = false;
    for (size_t i = 0; i < s.size(); ++i) {
        if (i > 0 && i % 60 == 0) wrap = true;
        o.push_back(s[i]);
        if (wrap && std::isspace((unsigned char)s[i])) {
            o.push_back('\n');
            wrap = false;
        }
    }
    return o;
}

static uint32_t pct(uint32_t n, uint32_t d) {  // output.rs:369 get_percent_match
    if (d == 0) return 0;
    if (n == d) return 100;
    return std::min((uint32_t)(0.5 + 100.0 * n / d), 99u);
}

std::string pairwise_header(const std::string& db_name, uint64_t n_seqs, uint64_t letters) {
    std::string o = "RMBLASTN 2.17.1+\n\n\n"
                    "Reference: Robert M. Hubley, Arian Smit\n"
                    "RMBlast - RepeatMasker Search Engine\n"
                    "2010 <http://www.repeatmasker.org>\n\n"
                    "Reference: Stephen F. Altschul, Thomas L. Madden, Alejandro A.\n"
                    "Schaffer, Jinghui Zhang, Zheng Zhang, Webb Miller, and David J.\n"
                    "Lipman (1997), \"Gapped BLAST and PSI-BLAST: a new generation of\n"
                    "protein database search programs\", Nucleic Acids Res. 25:3389-3402.\n\n\n\n"
                    "Database: ";
    for (const auto& l : wrap_flat(db_name, 68)) o += l + "\n";
    o += "           " + commas(n_seqs) + " sequences; " + commas(letters) + " total letters\n\n\n\n";
    return o;
}

// One HSP (output.rs:509-653): the statistics block, then rows of 60 columns.  qmask: bit p set
// when query position p lies in a DUST interval (printed in lower case), or null.
static void pairwise_hsp(std::string& o, const Hit& h, const uint32_t* qmask) {
    const Stats& st = h.stats;
    const uint32_t aln = (uint32_t)h.q_seq.size();
    const uint32_t ident = st.matches, gaps = st.query_gaps + st.subject_gaps;
    char b[256];
    o += " Score = " + std::to_string(h.score) + "\n";
    snprintf(b, sizeof b, " Substitutions = %.2f%%, Query Gaps = %.2f%%, DB Gaps = %.2f%%\n", (double)st.perc_sub,
             (double)st.perc_query_gap, (double)st.perc_db_gap);
    o += b;
    snprintf(b, sizeof b, " TransI/TransV = %u/%u,  CpG_sites = %u\n", st.transitions, st.transversions,
             st.cpg_sites);
    o += b;
    snprintf(b, sizeof b, " Kimura Div = %.2f%%, Kimura Div CpG Adjusted = %.2f%%\n", st.kdiv, st.cpg_kdiv);
    o += b;
    snprintf(b, sizeof b, " Identities = %u/%u (%u%%), Gaps = %u/%u (%u%%)\n", ident, aln, pct(ident, aln), gaps, aln,
             pct(gaps, aln));
    o += b;
    o += h.strand == 0 ? " Strand=Plus/Plus\n\n" : " Strand=Plus/Minus\n\n";
    std::string qs(aln, ' '), ss(aln, ' ');
    uint32_t qp = h.q_start;
    for (uint32_t i = 0; i < aln; ++i) {
        qs[i] = h.q_seq[i] == 15 ? '-' : IUPAC[h.q_seq[i] & 15];
        ss[i] = h.s_seq[i] == 15 ? '-' : IUPAC[h.s_seq[i] & 15];
        if (qs[i] != '-') {
            if (qmask && ((qmask[qp >> 5] >> (qp & 31)) & 1u)) qs[i] = (char)std::tolower((unsigned char)qs[i]);
            ++qp;
        }
    }
    const int w = (int)std::to_string(std::max(h.q_end, h.s_end)).size();
    uint32_t q_pos = h.q_start + 1, s_pos = h.strand == 0 ? h.s_start + 1 : h.s_end;
    for (uint32_t i = 0; i < aln; i += 60) {
        const uint32_t e = std::min(i + 60, aln);
        uint32_t qn = 0, sn = 0;
        std::string mid;
        for (uint32_t k = i; k < e; ++k) {
            qn += qs[k] != '-';
            sn += ss[k] != '-';
            const bool same = qs[k] != '-' && ss[k] != '-' &&
                              std::tolower((unsigned char)qs[k]) == std::tolower((unsigned char)ss[k]);
            mid.push_back(same ? '|' : ' ');
        }
        const uint32_t q_last = qn ? q_pos + qn - 1 : q_pos;
        const uint32_t s_last = h.strand == 0 ? (sn ? s_pos + sn - 1 : s_pos) : (sn ? s_pos - (sn - 1) : s_pos);
        snprintf(b, sizeof b, "Query  %-*u  ", w, q_pos);
        o += b;
        o.append(qs, i, e - i);
        o += "  " + std::to_string(q_last) + "\n" + std::string(9 + w, ' ') + mid + "\n";
        snprintf(b, sizeof b, "Sbjct  %-*u  ", w, s_pos);
        o += b;
        o.append(ss, i, e - i);
        o += "  " + std::to_string(s_last) + "\n\n";
        q_pos += qn;
        if (h.strand == 0) s_pos += sn;
        else s_pos = s_pos >= sn ? s_pos - sn : 0;
    }
    o += "\n";
}

void pairwise_query(std::string& o, const std::vector<Hit>& hits, const std::string& defline, uint32_t qlen,
                    const std::vector<std::string>& subject_ids, const char* const* subject_deflines,
                    const uint32_t* qmask) {
    std::string d = defline;  // NCBI trims a query's defline, not a subject's
    while (!d.empty() && std::isspace((unsigned char)d.back())) d.pop_back();
    o += "Query= " + d + "\n\nLength=" + std::to_string(qlen) + "\n\n";
    if (hits.empty()) {
        o += "\n***** No hits found *****\n\n\n\n\n";
        return;
    }
    std::vector<uint32_t> order;  // subjects in order of first appearance
    std::map<uint32_t, std::vector<const Hit*>> groups;
    for (const Hit& h : hits) {
        auto& g = groups[h.oid];
        if (g.empty()) order.push_back(h.oid);
        g.push_back(&h);
    }
    for (uint32_t oid : order) {
        const std::string& id = subject_ids.at(oid);
        std::string title;
        if (subject_deflines && subject_deflines[oid]) {
            const std::string dl = subject_deflines[oid];
            if (dl.compare(0, id.size(), id) == 0 && dl.size() > id.size()) title = dl.substr(id.size() + 1);
        }
        const auto& g = groups[oid];
        o += ">" + id + " " + wrap_title(title) + "\nLength=" + std::to_string(g[0]->s_len) + "\n\n";
        for (const Hit* h : g) pairwise_hsp(o, *h, qmask);
    }
    o += "\n\n";
}

// output.rs:379-411 format_ncbi_date: "Mon D, YYYY  H:MM AM/PM" (UTC), days-to-civil by the
// published public-domain algorithm of H. Hinnant
static std::string ncbi_date(uint64_t secs) {
    static const char* MON[12] = {"Jan", "Feb", "Mar", "Apr", "May", "Jun", "Jul", "Aug", "Sep", "Oct", "Nov", "Dec"};
    const uint64_t tod = secs % 86400, minute = (tod / 60) % 60, hour = tod / 3600;
    const int64_t z = (int64_t)(secs / 86400) + 719468;
    const int64_t era = (z >= 0 ? z : z - 146096) / 146097;
    const int64_t doe = z - era * 146097;
    const int64_t yoe = (doe - doe / 1460 + doe / 36524 - doe / 146096) / 365;
    const int64_t doy = doe - (365 * yoe + yoe / 4 - yoe / 100);
    const int64_t mp = (5 * doy + 2) / 153;
    const int64_t d = doy - (153 * mp + 2) / 5 + 1;
    const int64_t m = mp < 10 ? mp + 3 : mp - 9;
    const int64_t y = yoe + era * 400 + (m <= 2 ? 1 : 0);
    const uint64_t h12 = hour == 0 ? 12 : hour <= 12 ? hour : hour - 12;
    char b[64];
    snprintf(b, sizeof b, "%s %lld, %lld  %llu:%02llu %s", MON[m - 1], (long long)d, (long long)y,
             (unsigned long long)h12, (unsigned long long)minute, hour < 12 ? "AM" : "PM");
    return b;
}

std::string pairwise_footer(const std::string& db_name, uint64_t n_seqs, uint64_t letters, int64_t mtime, int go,
                            int ge) {
    std::string o = "  Database: ";
    for (const auto& l : wrap_flat(db_name, 68)) o += l + "\n";
    if (mtime >= 0) o += "    Posted date:  " + ncbi_date((uint64_t)mtime) + "\n";
    o += "  Number of letters in database: " + commas(letters) + "\n";
    o += "  Number of sequences in database:  " + commas(n_seqs) + "\n\n\n\n";
    char b[128];
    snprintf(b, sizeof b, "Matrix: blastn matrix 0 0\nGap Penalties: Existence: %d, Extension: %.2f\n", go, (double)ge);
    return o + b;
}

int choose_lut_width(int ws, uint64_t e) {  // blast/nalookup.rs:254-291
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
    return -1;
}

// search/ka_cutoff.rs:44-155: NCBI's (lambda, K) per RepeatMasker matrix file name and gap
// costs; the entries select the ungapped cutoff so they are kept value for value.
namespace {
struct Ka { const char* name; int go, ge; double lambda, k; };
const Ka KA[] = {
    {"14p35g.matrix", 29, 6, 0.1241860392, 0.2565118357}, {"14p37g.matrix", 29, 6, 0.1243509013, 0.2538327145},
    {"14p39g.matrix", 29, 6, 0.1181081970, 0.2381799563}, {"14p41g.matrix", 29, 6, 0.1209164962, 0.2516961980},
    {"14p43g.matrix", 29, 6, 0.1204338701, 0.2484920137}, {"14p45g.matrix", 29, 6, 0.1281012415, 0.2651519027},
    {"14p47g.matrix", 29, 6, 0.1169571490, 0.2334091021}, {"14p49g.matrix", 29, 6, 0.1167697593, 0.2289233061},
    {"14p51g.matrix", 29, 6, 0.1238779017, 0.2467119379}, {"14p53g.matrix", 29, 6, 0.1211022467, 0.2307304663},
    {"18p35g.matrix", 28, 5, 0.1204776630, 0.2111410357}, {"18p37g.matrix", 28, 5, 0.1213800379, 0.2057492194},
    {"18p39g.matrix", 28, 5, 0.1228853168, 0.2111281814}, {"18p41g.matrix", 28, 5, 0.1096830298, 0.1715966796},
    {"18p43g.matrix", 28, 5, 0.1179924113, 0.1957371364}, {"18p45g.matrix", 28, 5, 0.1184247414, 0.2068045787},
    {"18p47g.matrix", 28, 5, 0.1158783320, 0.1842046578}, {"18p49g.matrix", 28, 5, 0.1248964218, 0.2141853759},
    {"18p51g.matrix", 28, 5, 0.1106793836, 0.1621592148}, {"18p53g.matrix", 28, 5, 0.1082347513, 0.1408677318},
    {"20p35g.matrix", 25, 5, 0.1112832877, 0.1466667286}, {"20p37g.matrix", 25, 5, 0.1134511409, 0.1501236494},
    {"20p39g.matrix", 25, 5, 0.1233401001, 0.1853070864}, {"20p41g.matrix", 25, 5, 0.1088138918, 0.1409300313},
    {"20p43g.matrix", 25, 5, 0.1097495426, 0.1408421343}, {"20p45g.matrix", 25, 5, 0.1101110565, 0.1402262486},
    {"20p47g.matrix", 25, 5, 0.1198508511, 0.1752301830}, {"20p49g.matrix", 25, 5, 0.1150022018, 0.1500562415},
    {"20p51g.matrix", 25, 5, 0.1101356126, 0.1310353805}, {"20p53g.matrix", 25, 5, 0.1239625969, 0.1752022586},
    {"25p35g.matrix", 22, 5, 0.0965155465, 0.0677355511}, {"25p37g.matrix", 22, 5, 0.0989264764, 0.0763719670},
    {"25p39g.matrix", 22, 5, 0.1005843197, 0.0805691511}, {"25p41g.matrix", 22, 5, 0.1030661339, 0.0840485952},
    {"25p43g.matrix", 22, 5, 0.1155434360, 0.1226554129}, {"25p45g.matrix", 22, 5, 0.0973402625, 0.0742020190},
    {"25p47g.matrix", 22, 5, 0.0967346256, 0.0743885008}, {"25p49g.matrix", 22, 5, 0.1070577141, 0.0941947942},
    {"25p51g.matrix", 22, 5, 0.1044972455, 0.0789036639}, {"25p53g.matrix", 22, 5, 0.0977828435, 0.0607500307},
    {"30p53g.matrix", 22, 5, 0.1, 0.1},
};
}  // namespace

int ungapped_cutoff_for(const std::string& matrix_name, int go, int ge, int min_raw, uint64_t qlen, uint64_t avg) {
    const int fallback = min_raw > 0 ? min_raw / 2 : 1;
    std::string base = matrix_name;
    const size_t sl = base.find_last_of('/');
    if (sl != std::string::npos) base = base.substr(sl + 1);
    for (const Ka& r : KA) {
        if (r.go != go || r.ge != ge || strcasecmp(r.name, base.c_str()) != 0) continue;
        if (avg == 0) return fallback;
        const uint64_t sp = std::min(avg, qlen * 2) * avg;
        const int es = (int)std::ceil(std::log(r.k * (double)sp / 0.05) / r.lambda);
        const int c = es > 1 ? es : 1;
        return c < fallback ? c : fallback;
    }
    return fallback;
}

}  // namespace rmb
