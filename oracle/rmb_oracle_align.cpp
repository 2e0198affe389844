// rmb_oracle_align.cpp -- ungapped extension and the two X-drop gapped DPs.
// TEST INFRASTRUCTURE: the CPU oracle.  See rmb_oracle.hpp.
#include "rmb_oracle.hpp"

#include <stdexcept>

namespace rmbo {

void script_push(Script& s, EditOp op, uint32_t n) {  // hits.rs:44-53
    if (n == 0) return;
    if (!s.empty() && s.back().op == op) { s.back().n += n; return; }
    s.push_back(Op{op, n});
}

// search/ungapped.rs:38-121.  query/subject are sentinel-wrapped (index 0 = sentinel).
UngappedResult extend_ungapped(const uint8_t* query, size_t qsz, const uint8_t* subject, size_t ssz,
                               uint32_t q_off, uint32_t s_off, const Matrix& m, int xdrop) {
    const int32_t x = -xdrop;
    const int64_t q_real = (int64_t)qsz - 1, s_real = (int64_t)ssz - 1;
    const int64_t qo = q_off, so = s_off;
    int32_t score = 0, sum = 0;
    int64_t q_beg = qo;
    {
        int64_t q = qo - 1, s = so - 1;
        for (;;) {
            if (q < 0 || s < 0) break;
            uint8_t qb = query[1 + q], sb = subject[1 + s];
            if (qb == 15 || sb == 15) break;
            sum += m.s[qb & 15][sb & 15];
            if (sum > 0) {
                q_beg = q;
                score += sum;
                sum = 0;
            } else if (sum < x) {
                break;
            }
            --q;
            --s;
        }
    }
    uint32_t q_start = (uint32_t)q_beg;
    uint32_t s_start = (uint32_t)(so - (qo - q_beg));
    int64_t q_end = qo;
    int32_t x_cur = x;
    sum = 0;
    {
        int64_t q = qo, s = so;
        for (;;) {
            if (q >= q_real || s >= s_real) break;
            uint8_t qb = query[1 + q], sb = subject[1 + s];
            if (qb == 15 || sb == 15) break;
            sum += m.s[qb & 15][sb & 15];
            if (sum > 0) {
                q_end = q + 1;
                score += sum;
                x_cur = (-score > x) ? -score : x;
                sum = 0;
            } else if (sum < x_cur) {
                break;
            }
            ++q;
            ++s;
        }
    }
    uint32_t s_end = (uint32_t)(so + (q_end - qo));
    return UngappedResult{score, q_start, (uint32_t)q_end, s_start, s_end};
}

namespace {
constexpr int32_t MININT = INT32_MIN / 2;
struct DpCell { int32_t best, best_gap; };
thread_local std::vector<DpCell> tl_dp;

// Cells are always written in the current call before they are read (the band only
// reads [first_b, b_size), every cell of which the call wrote), so the buffer needs
// capacity, not initialisation.
inline DpCell* dp_reserve(size_t need) {
    if (tl_dp.size() < need) tl_dp.resize(need);
    return tl_dp.data();
}
}  // namespace

// search/gapped.rs:124-337 align_ex_score_only_inner.  a = outer sequence, b = inner.
ScoreOnly align_ex_score_only(const uint8_t* a, const uint8_t* b, size_t m, size_t n, int go, int ge,
                              int x_dropoff, const Matrix& mat, bool reverse) {
    if (m == 0 || n == 0) return ScoreOnly{0, 0, 0, 0};
    const int32_t goe = go + ge;
    const int32_t xdrop = x_dropoff > goe ? x_dropoff : goe;
    const size_t num_extra = ge > 0 ? (size_t)(xdrop / ge + 3) : n + 3;
    const size_t max_cap = n + 2;
    size_t cap = std::min(num_extra + 102, max_cap);
    DpCell* dp = dp_reserve(cap);
    dp[0].best = 0;
    dp[0].best_gap = -goe;
    int32_t score = -goe;
    size_t b_size = 1;
    for (size_t j = 1; j <= n; ++j) {
        if (score < -xdrop || j >= cap) break;
        dp[j].best = score;
        dp[j].best_gap = score - goe;
        score -= ge;
        b_size = j + 1;
    }
    int32_t best_score = 0;
    size_t best_a = 0, best_b = 0, first_b = 0;
    uint64_t cells = 0;
    for (size_t ai = 0; ai < m; ++ai) {
        size_t ap = reverse ? m - 1 - ai : ai;
        const int32_t* row = mat.s[a[ap] & 15];
        int32_t sc = MININT, gap_row = MININT;
        size_t last_b = first_b;
        int32_t prev_best = best_score;
        cells += b_size - first_b;
        for (size_t bi = first_b; bi < b_size; ++bi) {
            int32_t gap_col = dp[bi].best_gap;
            int32_t next_score = 0;
            if (bi < n) {
                size_t bp = reverse ? n - 1 - bi : bi;
                next_score = dp[bi].best + row[b[bp]];
            }
            int32_t cell = sc;
            if (gap_col > cell) cell = gap_col;
            if (gap_row > cell) cell = gap_row;
            if (best_score - cell > xdrop) {
                if (bi == first_b) ++first_b;
                else dp[bi].best = MININT;
            } else {
                last_b = bi;
                if (cell > best_score) { best_b = bi; best_score = cell; }
                gap_row -= ge;
                int32_t open = cell - goe;
                int32_t col_ext = gap_col - ge;
                dp[bi].best_gap = col_ext > open ? col_ext : open;
                dp[bi].best = cell;
                if (open > gap_row) gap_row = open;
            }
            sc = next_score;
        }
        if (best_score > prev_best) best_a = ai + 1;
        if (first_b >= b_size) break;
        if (last_b + num_extra + 3 >= cap && cap < max_cap) {
            cap = std::min(std::max(last_b + num_extra + 100, cap * 2), max_cap);
            dp = dp_reserve(cap);
        }
        if (last_b + 1 < b_size) {
            b_size = last_b + 1;
        } else {
            while (gap_row >= best_score - xdrop && b_size <= n && b_size < cap - 1) {
                dp[b_size].best = gap_row;
                dp[b_size].best_gap = gap_row - goe;
                gap_row -= ge;
                ++b_size;
            }
        }
        if (b_size <= n && b_size < cap) {
            dp[b_size].best = MININT;
            dp[b_size].best_gap = MININT;
            ++b_size;
        }
    }
    return ScoreOnly{best_score, (uint32_t)best_a, (uint32_t)best_b, cells};
}

// search/gapped.rs:38-43 trace op bytes
constexpr uint8_t T_GAP_A = 0, T_SUB = 3, T_GAP_B = 6, T_MASK = 7, T_EXT_A = 0x10, T_EXT_B = 0x40;

namespace {
thread_local std::vector<uint8_t> tl_flat;
thread_local std::vector<std::pair<size_t, size_t>> tl_rows;
}  // namespace

// search/gapped.rs:692-757 traceback_flat
static Script traceback_flat(const std::vector<uint8_t>& flat, size_t flat_len,
                             const std::vector<std::pair<size_t, size_t>>& rows, size_t end_a, size_t end_b) {
    Script out;
    if (end_a == 0 && end_b == 0) return out;
    std::vector<Op> rev;
    auto push_rev = [&](EditOp op) {
        if (!rev.empty() && rev.back().op == op) ++rev.back().n;
        else rev.push_back(Op{op, 1});
    };
    size_t a = end_a, b = end_b;
    uint8_t prev = T_SUB;
    for (size_t step = 0; step < end_a + end_b; ++step) {
        size_t off = rows[a].first, fb = rows[a].second;
        size_t row_end = a + 1 < rows.size() ? rows[a + 1].first : flat_len;
        uint8_t raw = T_GAP_A;
        if (b >= fb) {
            size_t bi = off + (b - fb);
            raw = bi < row_end ? flat[bi] : T_GAP_A;
        }
        uint8_t op;
        if ((prev & T_MASK) == T_GAP_A) op = (raw & T_EXT_A) ? T_GAP_A : (raw & T_MASK);
        else if ((prev & T_MASK) == T_GAP_B) op = (raw & T_EXT_B) ? T_GAP_B : (raw & T_MASK);
        else op = raw & T_MASK;
        prev = op;
        if (op == T_GAP_A) { push_rev(GAP_IN_QUERY); b = b ? b - 1 : 0; }
        else if (op == T_GAP_B) { push_rev(GAP_IN_SUBJECT); a = a ? a - 1 : 0; }
        else { push_rev(SUB); a = a ? a - 1 : 0; b = b ? b - 1 : 0; }
        if (a == 0 && b == 0) break;
    }
    if (a != 0 || b != 0) throw std::runtime_error("traceback did not reach the origin");
    for (size_t i = rev.size(); i-- > 0;) script_push(out, rev[i].op, rev[i].n);
    return out;
}

// search/gapped.rs:450-689 align_ex_inner.  a = query (outer), b = subject (inner).
GapAlign align_ex(const uint8_t* a, const uint8_t* b, size_t m, size_t n, int go, int ge, int x_dropoff,
                  const Matrix& mat, bool reverse) {
    if (m == 0 || n == 0) return GapAlign{0, 0, 0, {}, 0};
    const int32_t goe = go + ge;
    const int32_t xdrop = x_dropoff > goe ? x_dropoff : goe;
    const size_t num_extra = ge > 0 ? (size_t)(xdrop / ge + 3) : n + 3;
    const size_t max_cap = n + 2;
    size_t cap = std::min(num_extra + 101, max_cap);
    DpCell* dp = dp_reserve(cap);
    auto& flat = tl_flat;
    auto& rows = tl_rows;
    rows.clear();
    size_t flen = 0;
    auto put = [&](uint8_t v) {
        if (flen >= flat.size()) flat.resize(std::max<size_t>(flat.size() * 2, 4096));
        flat[flen++] = v;
    };
    dp[0].best = 0;
    dp[0].best_gap = -goe;
    rows.push_back({0, 0});
    put(T_GAP_B);
    int32_t score = -goe;
    size_t b_size = 1;
    for (size_t j = 1; j <= n; ++j) {
        if (score < -xdrop || j >= cap) break;
        dp[j].best = score;
        dp[j].best_gap = score - goe;
        put(T_GAP_A);
        score -= ge;
        b_size = j + 1;
    }
    int32_t best_score = 0;
    size_t best_a = 0, best_b = 0, first_b = 0;
    uint64_t cells = 0;
    for (size_t ai = 0; ai < m; ++ai) {
        size_t ap = reverse ? m - 1 - ai : ai;
        const int32_t* row = mat.s[a[ap] & 15];
        rows.push_back({flen, first_b});
        int32_t sc = MININT, gap_row = MININT;
        size_t last_b = first_b;
        cells += b_size - first_b;
        for (size_t bi = first_b; bi < b_size; ++bi) {
            uint8_t bb = 0;
            if (bi < n) bb = b[reverse ? n - 1 - bi : bi] & 15;
            int32_t gap_col = dp[bi].best_gap;
            int32_t next_score = dp[bi].best + row[bb];
            uint8_t op = T_SUB;
            int32_t cell = sc;
            if (gap_col > cell) { cell = gap_col; op = T_GAP_B; }
            if (gap_row > cell) { cell = gap_row; op = T_GAP_A; }
            if (best_score - cell > xdrop) {
                if (bi == first_b) ++first_b;
                else dp[bi].best = MININT;
            } else {
                last_b = bi;
                if (cell > best_score) { best_score = cell; best_a = ai + 1; best_b = bi; }
                gap_row -= ge;
                gap_col -= ge;
                int32_t open = cell - goe;
                if (gap_col < open) dp[bi].best_gap = open;
                else { dp[bi].best_gap = gap_col; op |= T_EXT_B; }
                dp[bi].best = cell;
                if (gap_row < open) gap_row = open;
                else op |= T_EXT_A;
            }
            sc = next_score;
            put(op);
        }
        if (first_b >= b_size) break;
        if (last_b + num_extra + 3 >= cap && cap < max_cap) {
            cap = std::min(std::max(last_b + num_extra + 100, cap * 2), max_cap);
            dp = dp_reserve(cap);
        }
        if (last_b + 1 < b_size) {
            b_size = last_b + 1;
        } else {
            while (gap_row >= best_score - xdrop && b_size <= n && b_size < cap) {
                dp[b_size].best = gap_row;
                dp[b_size].best_gap = gap_row - goe;
                gap_row -= ge;
                put(T_GAP_A);
                ++b_size;
            }
        }
        if (b_size <= n && b_size < cap) {
            dp[b_size].best = MININT;
            dp[b_size].best_gap = MININT;
            ++b_size;
        }
    }
    Script s = traceback_flat(flat, flen, rows, best_a, best_b);
    return GapAlign{best_score, (uint32_t)best_a, (uint32_t)best_b, std::move(s), cells};
}

}  // namespace rmbo
