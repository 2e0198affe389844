// rmb_oracle_itree.hpp -- the 2-D interval tree of search/itree.rs (TEST INFRASTRUCTURE).
#pragma once
#include <cstdint>
#include <cstdlib>
#include <map>
#include <vector>

namespace rmbo {

struct ITreeHsp { uint32_t q_start, q_end, s_start, s_end; int32_t score; };

// search/itree.rs:60-555 BlastIntervalTree (eQueryAndSubject)
class IntervalTree {
    static constexpr uint32_t INTERNAL = 0xFFFFFFFFu, NIL = 0;
    struct Node { uint32_t le, re, left, mid, right, hsp; };
    std::vector<Node> nodes;
    std::vector<ITreeHsp> hsps;
    std::vector<uint8_t> deleted;
    std::map<std::pair<uint32_t, uint32_t>, std::pair<int32_t, uint32_t>> left_ep, right_ep;
    uint32_t s_min, s_max;

   public:
    bool rc_query = false;
    IntervalTree(uint32_t q0, uint32_t q1, uint32_t s0, uint32_t s1, bool rc = false)
        : s_min(s0), s_max(s1), rc_query(rc) {
        nodes.push_back(Node{q0, q1, NIL, NIL, NIL, INTERNAL});
    }

   private:
    uint32_t alloc_internal(uint32_t le, uint32_t re) {
        nodes.push_back(Node{le, re, NIL, NIL, NIL, INTERNAL});
        return (uint32_t)nodes.size() - 1;
    }
    uint32_t alloc_leaf(const ITreeHsp& h) {
        hsps.push_back(h);
        deleted.push_back(0);
        nodes.push_back(Node{0, 0, NIL, NIL, NIL, (uint32_t)hsps.size() - 1});
        return (uint32_t)nodes.size() - 1;
    }
    static bool new_wins(int32_t ns, uint32_t nq, uint32_t nsl, int32_t es, uint32_t eq, uint32_t esl) {
        if (ns != es) return ns > es;
        if (nq != eq) return nq < eq;
        if (nsl != esl) return nsl < esl;
        return false;
    }
    void remove_endpoints(uint32_t idx, bool plus) {
        deleted[idx] = 1;
        const ITreeHsp& e = hsps[idx];
        std::pair<uint32_t, uint32_t> l = plus ? std::make_pair(e.q_start, e.s_start) : std::make_pair(e.q_end, e.s_start);
        std::pair<uint32_t, uint32_t> r = plus ? std::make_pair(e.q_end, e.s_end) : std::make_pair(e.q_start, e.s_end);
        auto it = left_ep.find(l);
        if (it != left_ep.end() && it->second.second == idx) left_ep.erase(it);
        it = right_ep.find(r);
        if (it != right_ep.end() && it->second.second == idx) right_ep.erase(it);
    }
    // itree.rs:251-371 insert_structural
    void insert_structural(uint32_t new_idx) {
        const ITreeHsp h = hsps[nodes[new_idx].hsp];
        uint32_t rs = h.q_start, re = h.q_end;
        bool subj = false;
        uint32_t root = 0;
        for (;;) {
            uint32_t r_le = nodes[root].le, r_re = nodes[root].re;
            uint64_t middle = ((uint64_t)r_le + r_re) / 2;
            bool left_half;
            uint32_t old_index;
            if ((uint64_t)re < middle) {
                uint32_t l = nodes[root].left;
                if (l == NIL) { nodes[root].left = new_idx; return; }
                if (nodes[l].hsp == INTERNAL) { root = l; continue; }
                old_index = l;
                left_half = true;
            } else if ((uint64_t)rs > middle) {
                uint32_t r = nodes[root].right;
                if (r == NIL) { nodes[root].right = new_idx; return; }
                if (nodes[r].hsp == INTERNAL) { root = r; continue; }
                old_index = r;
                left_half = false;
            } else {
                if (subj) {
                    nodes[new_idx].mid = nodes[root].mid;
                    nodes[root].mid = new_idx;
                    return;
                }
                subj = true;
                if (nodes[root].mid == NIL) {
                    uint32_t mid = alloc_internal(s_min, s_max);
                    nodes[root].mid = mid;
                }
                root = nodes[root].mid;
                rs = h.s_start;
                re = h.s_end;
                continue;
            }
            uint32_t mle = left_half ? r_le : (uint32_t)middle + 1;
            uint32_t mre = left_half ? (uint32_t)middle : r_re;
            uint32_t mi = alloc_internal(mle, mre);
            if (left_half) nodes[root].left = mi;
            else nodes[root].right = mi;
            const ITreeHsp& o = hsps[nodes[old_index].hsp];
            uint32_t ors = subj ? o.s_start : o.q_start, ore = subj ? o.s_end : o.q_end;
            root = mi;
            uint64_t mm = ((uint64_t)mle + mre) / 2;
            if ((uint64_t)ore < mm) nodes[mi].left = old_index;
            else if ((uint64_t)ors > mm) nodes[mi].right = old_index;
            else if (subj) nodes[mi].mid = old_index;
            else {
                uint32_t os = o.s_start, oe = o.s_end;
                uint32_t m2 = alloc_internal(s_min, s_max);
                nodes[mi].mid = m2;
                uint64_t m2mid = ((uint64_t)s_min + s_max) / 2;
                if ((uint64_t)oe < m2mid) nodes[m2].left = old_index;
                else if ((uint64_t)os > m2mid) nodes[m2].right = old_index;
                else nodes[m2].mid = old_index;
            }
        }
    }
    // itree.rs:496-554 hsp_is_contained
    bool contained_by(const ITreeHsp& c, bool plus, int64_t sep, uint32_t idx) const {
        if (deleted[idx]) return false;
        const ITreeHsp& h = hsps[idx];
        if (c.score > h.score) return false;
        if (!(h.q_start <= c.q_start && h.q_end >= c.q_end && h.s_start <= c.s_start && h.s_end >= c.s_end))
            return false;
        int64_t d0, d1;
        if (plus || rc_query) {
            d0 = std::llabs(((int64_t)c.q_start - c.s_start) - ((int64_t)h.q_start - h.s_start));
            d1 = std::llabs(((int64_t)c.q_end - c.s_end) - ((int64_t)h.q_end - h.s_end));
        } else {
            d0 = std::llabs(((int64_t)c.q_end + c.s_start) - ((int64_t)h.q_end + h.s_start));
            d1 = std::llabs(((int64_t)c.q_start + c.s_end) - ((int64_t)h.q_start + h.s_end));
        }
        return d0 < sep || d1 < sep;
    }
    bool midpoint_contains(uint32_t node, const ITreeHsp& c, bool plus, int64_t sep) const {
        for (;;) {
            if (nodes[node].hsp != INTERNAL) return contained_by(c, plus, sep, nodes[node].hsp);
            for (uint32_t mid = nodes[node].mid; mid != NIL; mid = nodes[mid].mid)
                if (contained_by(c, plus, sep, nodes[mid].hsp)) return true;
            uint64_t middle = ((uint64_t)nodes[node].le + nodes[node].re) / 2;
            uint32_t next;
            if ((uint64_t)c.s_end < middle) next = nodes[node].left;
            else if ((uint64_t)c.s_start > middle) next = nodes[node].right;
            else return false;
            if (next == NIL) return false;
            node = next;
        }
    }

   public:
    // itree.rs:151-230 add (endpoint-sharing dedup)
    bool add(const ITreeHsp& h, bool plus) {
        std::pair<uint32_t, uint32_t> l = plus ? std::make_pair(h.q_start, h.s_start) : std::make_pair(h.q_end, h.s_start);
        std::pair<uint32_t, uint32_t> r = plus ? std::make_pair(h.q_end, h.s_end) : std::make_pair(h.q_start, h.s_end);
        uint32_t nq = h.q_end - h.q_start, ns = h.s_end - h.s_start;
        auto it = left_ep.find(l);
        if (it != left_ep.end()) {
            uint32_t ei = it->second.second;
            const ITreeHsp& e = hsps[ei];
            if (!new_wins(h.score, nq, ns, it->second.first, e.q_end - e.q_start, e.s_end - e.s_start)) return false;
            remove_endpoints(ei, plus);
        }
        it = right_ep.find(r);
        if (it != right_ep.end()) {
            uint32_t ei = it->second.second;
            const ITreeHsp& e = hsps[ei];
            if (!new_wins(h.score, nq, ns, it->second.first, e.q_end - e.q_start, e.s_end - e.s_start)) return false;
            remove_endpoints(ei, plus);
        }
        uint32_t ni = alloc_leaf(h);
        uint32_t hi = nodes[ni].hsp;
        left_ep[l] = {h.score, hi};
        right_ep[r] = {h.score, hi};
        insert_structural(ni);
        return true;
    }
    void add_simple(const ITreeHsp& h) { insert_structural(alloc_leaf(h)); }
    // itree.rs:376-435 contains
    bool contains(const ITreeHsp& c, bool plus, int64_t sep) const {
        uint32_t node = 0;
        for (;;) {
            uint32_t mid = nodes[node].mid;
            if (mid != NIL && midpoint_contains(mid, c, plus, sep)) return true;
            uint64_t middle = ((uint64_t)nodes[node].le + nodes[node].re) / 2;
            uint32_t next;
            if ((uint64_t)c.q_end < middle) next = nodes[node].left;
            else if ((uint64_t)c.q_start > middle) next = nodes[node].right;
            else return false;
            if (next == NIL) return false;
            if (nodes[next].hsp != INTERNAL) return contained_by(c, plus, sep, nodes[next].hsp);
            node = next;
        }
    }
};

}  // namespace rmbo
