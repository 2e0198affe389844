// rmb_oracle_output.cpp -- alignment statistics and outfmt-6 formatting.
// TEST INFRASTRUCTURE: the CPU oracle.  See rmb_oracle.hpp.
#include <cmath>
#include <cstdio>
#include <stdexcept>

#include "rmb_oracle.hpp"

namespace rmbo {

std::vector<uint8_t> to_iupac(const std::vector<uint8_t>& s) {  // stats.rs:247
    std::vector<uint8_t> o(s.size());
    for (size_t i = 0; i < s.size(); ++i) o[i] = s[i] == 15 ? '-' : BLASTNA_TO_IUPAC[s[i] & 15];
    return o;
}

namespace {
enum Pair { IDENT, TRANSI, TRANSV, IUB_MATCH, IUB_SUB, GAP, UNKNOWN };
bool unambig(uint8_t c) { return c == 'A' || c == 'C' || c == 'G' || c == 'T'; }
uint8_t bitmask(uint8_t c) {  // stats.rs:200
    switch (c) {
        case 'A': return 1; case 'C': return 2; case 'G': return 4; case 'T': case 'U': return 8;
        case 'R': return 5; case 'Y': return 10; case 'M': return 3; case 'K': return 12;
        case 'W': return 9; case 'S': return 6; case 'B': return 14; case 'D': return 13;
        case 'H': return 11; case 'V': return 7; default: return 15;
    }
}
Pair classify(uint8_t a, uint8_t b) {  // stats.rs:162-197
    if (a == '-' || b == '-') return GAP;
    if (a == b) return IDENT;
    if (!unambig(a) || !unambig(b)) {
        bool one_pure = unambig(a) ^ unambig(b);
        return (one_pure && (bitmask(a) & bitmask(b))) ? IUB_MATCH : IUB_SUB;
    }
    bool ap = a == 'A' || a == 'G', bp = b == 'A' || b == 'G';
    return ap == bp ? TRANSI : TRANSV;
}
double kimura(double p, double q) {  // stats.rs:237-245
    double operand = (1.0 - 2.0 * p - q) * std::sqrt(1.0 - 2.0 * q);
    if (operand > 0.0) return std::fabs(-0.5 * std::log(operand)) * 100.0;
    return 100.0;
}
}  // namespace

// stats.rs:52-160 (query_is_ancestral = false: ancestral = subject, derived = query)
AlignStats compute_align_stats(const std::vector<uint8_t>& qs, const std::vector<uint8_t>& ss) {
    AlignStats st;
    const std::vector<uint8_t>& anc = ss;
    const std::vector<uint8_t>& der = qs;
    uint32_t matches = 0, mism = 0, qg = 0, sg = 0, ti = 0, tv = 0, cpg = 0, unamb = 0, ql = 0, dl = 0;
    double cpg_ti = 0.0;
    uint8_t prev_anc = ' ';
    Pair prev_pair = UNKNOWN;
    for (size_t i = 0; i < anc.size(); ++i) {
        uint8_t ac = (uint8_t)toupper(anc[i]), dc = (uint8_t)toupper(der[i]);
        if (qs[i] != '-') ++ql;
        if (ss[i] != '-') ++dl;
        if (prev_anc == 'C' && ac == 'G') {
            ++cpg;
            Pair cur = classify(ac, dc);
            if (prev_pair == TRANSI && cur == TRANSI) cpg_ti -= 1.0;
            else if (prev_pair == TRANSI || cur == TRANSI) cpg_ti -= 0.9;
        }
        if (ac == '-' || dc == '-') {
            if (qs[i] == '-') ++qg;
            else ++sg;
            if (ac != '-') { prev_anc = ac; prev_pair = GAP; }
        } else {
            Pair pr = classify(ac, dc);
            switch (pr) {
                case IDENT: ++matches; if (unambig(ac) && unambig(dc)) ++unamb; break;
                case TRANSI: ++mism; if (unambig(ac) && unambig(dc)) { ++unamb; ++ti; cpg_ti += 1.0; } break;
                case TRANSV: ++mism; if (unambig(ac) && unambig(dc)) { ++unamb; ++tv; } break;
                case IUB_SUB: ++mism; break;
                default: break;
            }
            prev_anc = ac;
            prev_pair = pr;
        }
    }
    if (unamb < 1) { st.kdiv = 100.0; st.cpg_kdiv = 100.0; }
    else {
        double n = (double)unamb;
        double p = (double)ti / n, cp = cpg_ti / n, q = (double)tv / n;
        st.kdiv = kimura(p, q);
        st.cpg_kdiv = kimura(cp, q);
    }
    st.matches = matches; st.mismatches = mism; st.query_gaps = qg; st.subject_gaps = sg;
    st.transitions = ti; st.transversions = tv; st.cpg_sites = cpg;
    st.perc_sub = ql > 0 ? ((float)mism / (float)ql) * 100.0f : 0.0f;
    st.perc_query_gap = ql > 0 ? ((float)qg / (float)ql) * 100.0f : 0.0f;
    st.perc_db_gap = dl > 0 ? ((float)sg / (float)dl) * 100.0f : 0.0f;
    return st;
}

// output.rs:294-367 write_tabular (tab-separated, no trailing newline)
std::string format_tabular(const AlignResult& r, const std::vector<std::string>& fields) {
    const Hsp& h = r.hsp;
    const AlignStats& st = r.stats;
    uint32_t s1 = h.s_start + 1, se = h.s_end;
    uint32_t ss = h.strand == PLUS ? s1 : se, sn = h.strand == PLUS ? se : s1;
    std::string out;
    char buf[64];
    bool first = true;
    for (const std::string& f : fields) {
        if (!first) out.push_back('\t');
        first = false;
        if (f == "score") out += std::to_string(h.score);
        else if (f == "perc_sub") { snprintf(buf, sizeof buf, "%.2f", (double)st.perc_sub); out += buf; }
        else if (f == "perc_query_gap") { snprintf(buf, sizeof buf, "%.2f", (double)st.perc_query_gap); out += buf; }
        else if (f == "perc_db_gap") { snprintf(buf, sizeof buf, "%.2f", (double)st.perc_db_gap); out += buf; }
        else if (f == "qseqid") out += r.query_id;
        else if (f == "qstart") out += std::to_string(h.q_start + 1);
        else if (f == "qend") out += std::to_string(h.q_end);
        else if (f == "qlen") out += std::to_string(h.q_len);
        else if (f == "sstrand") out += h.strand == PLUS ? "plus" : "minus";
        else if (f == "sseqid") out += r.subject_id;
        else if (f == "sstart") out += std::to_string(ss);
        else if (f == "send") out += std::to_string(sn);
        else if (f == "slen") out += std::to_string(h.s_len);
        else if (f == "kdiv") { snprintf(buf, sizeof buf, "%.2f", st.kdiv); out += buf; }
        else if (f == "cpg_kdiv") { snprintf(buf, sizeof buf, "%.2f", st.cpg_kdiv); out += buf; }
        else if (f == "transi") out += std::to_string(st.transversions);  // output.rs:160-164 quirk
        else if (f == "transv") out += std::to_string(st.cpg_sites);
        else if (f == "cpg_sites") out += std::to_string(st.transitions);
        else if (f == "qseq") { auto v = to_iupac(h.q_seq); out.append(v.begin(), v.end()); }
        else if (f == "sseq") { auto v = to_iupac(h.s_seq); out.append(v.begin(), v.end()); }
        else if (f == "evalue") out += format_evalue(r.evalue);
        else if (f == "bitscore") out += format_bitscore(r.bitscore);
        else throw std::runtime_error("unknown -outfmt field '" + f + "'");
    }
    return out;
}

}  // namespace rmbo

// ---- pairwise output (outfmt 0): rmblast-lib/src/output.rs:25-126, 369-720 ------------------
namespace rmbo {

std::string with_commas(uint64_t n) {  // output.rs:28 NStr::Int8ToString(n, fWithCommas)
    std::string d = std::to_string(n), o;
    for (size_t i = 0; i < d.size(); ++i) {
        if (i > 0 && (d.size() - i) % 3 == 0) o.push_back(',');
        o.push_back(d[i]);
    }
    return o;
}

// output.rs:44-106 ncbi_wrap_flat (NStr::Wrap with fWrap_FlatFile)
std::vector<std::string> ncbi_wrap_flat(const std::string& s, size_t width) {
    enum Score { Forced = 0, Punct = 1, Comma = 2, Space = 3, Newline = 4 };
    const size_t len = s.size();
    std::vector<std::string> lines;
    size_t pos = 0;
    while (pos < len) {
        size_t column = 0, best_pos = SIZE_MAX;
        int best = Forced;
        size_t nl = s.find('\n', pos);
        if (nl == std::string::npos) nl = len;
        const size_t pos0 = (nl - pos <= width) ? nl : pos;
        size_t pos2 = pos0;
        while (pos2 < len && column <= width) {
            const char c = s[pos2];
            int score = Forced;
            size_t score_pos = pos2;
            if (c == '\n') {
                best_pos = pos2;
                best = Newline;
                break;
            } else if (isspace((unsigned char)c)) {
                score = Space;
            } else if (c == ',' && column < width && score_pos < len - 1) {
                score = Comma;
                ++score_pos;
            } else if (c == '-' && score_pos < len - 1 && column < width) {
                score = Punct;
                ++score_pos;
            }
            if (score >= best && score_pos > pos0) {
                best_pos = score_pos;
                best = score;
            }
            ++pos2;
            ++column;
        }
        if (best != Newline && column <= width) best_pos = len;
        best_pos = std::max(std::min(best_pos, len), pos + 1);
        lines.push_back(s.substr(pos, best_pos - pos));
        pos = best_pos;
        if (best == Space) {
            while (pos < len && s[pos] == ' ') ++pos;
            if (pos < len && s[pos] == '\n') ++pos;
        } else if (best == Newline) {
            ++pos;
        }
    }
    if (lines.empty()) lines.push_back("");
    return lines;
}

// output.rs:108-126 ncbi_wrap_title (s_WrapOutputLine): past every 60th character, break after
// the next whitespace
std::string ncbi_wrap_title(const std::string& s) {
    if (s.size() <= 60) return s;
    std::string o;
    bool wrap = false;
    for (size_t i = 0; i < s.size(); ++i) {
        if (i > 0 && i % 60 == 0) wrap = true;
        o.push_back(s[i]);
        if (wrap && isspace((unsigned char)s[i])) {
            o.push_back('\n');
            wrap = false;
        }
    }
    return o;
}

static uint32_t percent_match(uint32_t n, uint32_t d) {  // output.rs:369
    if (d == 0) return 0;
    if (n == d) return 100;
    const uint32_t r = (uint32_t)(0.5 + 100.0 * n / d);
    return std::min(r, 99u);
}

std::string pairwise_program_header(const std::string& db_name, size_t n_seqs, uint64_t total) {  // :431-455
    std::string o = "RMBLASTN 2.17.1+\n\n\n";
    o += "Reference: Robert M. Hubley, Arian Smit\nRMBlast - RepeatMasker Search Engine\n"
         "2010 <http://www.repeatmasker.org>\n\n";
    o += "Reference: Stephen F. Altschul, Thomas L. Madden, Alejandro A.\n"
         "Schaffer, Jinghui Zhang, Zheng Zhang, Webb Miller, and David J.\n"
         "Lipman (1997), \"Gapped BLAST and PSI-BLAST: a new generation of\n"
         "protein database search programs\", Nucleic Acids Res. 25:3389-3402.\n\n\n\n";
    o += "Database: ";
    for (auto& l : ncbi_wrap_flat(db_name, 68)) o += l + "\n";
    o += "           " + with_commas(n_seqs) + " sequences; " + with_commas(total) + " total letters\n\n\n\n";
    return o;
}

static std::string pairwise_hsp(const AlignResult& r, const std::vector<std::pair<size_t, size_t>>& mask) {  // :509-653
    const Hsp& h = r.hsp;
    const AlignStats& st = r.stats;
    const uint32_t aln_len = (uint32_t)h.q_seq.size();
    const uint32_t n_ident = st.matches, n_gaps = st.query_gaps + st.subject_gaps;
    char b[256];
    std::string o;
    o += " Score = " + std::to_string(h.score) + "\n";
    snprintf(b, sizeof b, " Substitutions = %.2f%%, Query Gaps = %.2f%%, DB Gaps = %.2f%%\n", (double)st.perc_sub,
             (double)st.perc_query_gap, (double)st.perc_db_gap);
    o += b;
    snprintf(b, sizeof b, " TransI/TransV = %u/%u,  CpG_sites = %u\n", st.transitions, st.transversions, st.cpg_sites);
    o += b;
    snprintf(b, sizeof b, " Kimura Div = %.2f%%, Kimura Div CpG Adjusted = %.2f%%\n", st.kdiv, st.cpg_kdiv);
    o += b;
    snprintf(b, sizeof b, " Identities = %u/%u (%u%%), Gaps = %u/%u (%u%%)\n", n_ident, aln_len,
             percent_match(n_ident, aln_len), n_gaps, aln_len, percent_match(n_gaps, aln_len));
    o += b;
    o += std::string(" Strand=") + (h.strand == PLUS ? "Plus/Plus" : "Plus/Minus") + "\n\n";
    std::vector<uint8_t> qi = to_iupac(h.q_seq), si = to_iupac(h.s_seq);
    if (!mask.empty()) {
        size_t q = h.q_start, m = 0;
        while (m < mask.size() && mask[m].second < q) ++m;
        for (auto& c : qi) {
            if (c == '-') continue;
            while (m < mask.size() && mask[m].second < q) ++m;
            if (m < mask.size() && mask[m].first <= q) c = (uint8_t)tolower(c);
            ++q;
        }
    }
    const uint32_t maxc = std::max(h.q_end, h.s_end);
    const int pos_w = (int)std::to_string(maxc).size();
    uint32_t q_pos = h.q_start + 1;
    uint32_t s_pos = h.strand == PLUS ? h.s_start + 1 : h.s_end;
    for (size_t i = 0; i < qi.size(); i += 60) {
        const size_t e = std::min(i + 60, qi.size());
        uint32_t qn = 0, sn = 0;
        std::string match;
        for (size_t k = i; k < e; ++k) {
            qn += qi[k] != '-';
            sn += si[k] != '-';
            match.push_back(qi[k] == '-' || si[k] == '-' ? ' ' : (tolower(qi[k]) == tolower(si[k]) ? '|' : ' '));
        }
        const uint32_t q_end_row = qn ? q_pos + qn - 1 : q_pos;
        const uint32_t s_end_row = h.strand == PLUS ? (sn ? s_pos + sn - 1 : s_pos) : (sn ? s_pos - (sn - 1) : s_pos);
        snprintf(b, sizeof b, "Query  %-*u  ", pos_w, q_pos);
        o += b;
        o.append((const char*)qi.data() + i, e - i);
        o += "  " + std::to_string(q_end_row) + "\n";
        o += std::string(9 + pos_w, ' ') + match + "\n";
        snprintf(b, sizeof b, "Sbjct  %-*u  ", pos_w, s_pos);
        o += b;
        o.append((const char*)si.data() + i, e - i);
        o += "  " + std::to_string(s_end_row) + "\n\n";
        q_pos += qn;
        if (h.strand == PLUS) s_pos += sn;
        else s_pos = s_pos >= sn ? s_pos - sn : 0;
    }
    o += "\n";
    return o;
}

// output.rs:684-720 write_pairwise_results (+ the query and subject headers, :469-505)
std::string pairwise_results(const std::vector<AlignResult>& res, const std::string& query_defline, uint32_t qlen,
                             const std::map<std::string, std::string>* subject_deflines,
                             const std::vector<std::pair<size_t, size_t>>& query_mask) {
    std::string d = query_defline;
    while (!d.empty() && isspace((unsigned char)d.back())) d.pop_back();
    std::string o = "Query= " + d + "\n\nLength=" + std::to_string(qlen) + "\n\n";
    if (res.empty()) return o + "\n***** No hits found *****\n\n\n\n\n";
    std::vector<std::string> order;
    std::map<std::string, std::vector<const AlignResult*>> groups;
    for (auto& r : res) {
        auto it = groups.find(r.subject_id);
        if (it == groups.end()) {
            order.push_back(r.subject_id);
            groups[r.subject_id].push_back(&r);
        } else {
            it->second.push_back(&r);
        }
    }
    for (auto& id : order) {
        const auto& g = groups[id];
        std::string title;
        if (subject_deflines) {
            auto it = subject_deflines->find(id);
            if (it != subject_deflines->end() && it->second.compare(0, id.size(), id) == 0 && it->second.size() > id.size())
                title = it->second.substr(id.size() + 1);
        }
        o += ">" + id + " " + ncbi_wrap_title(title) + "\nLength=" + std::to_string(g[0]->hsp.s_len) + "\n\n";
        for (auto* r : g) o += pairwise_hsp(*r, query_mask);
    }
    return o + "\n\n";
}

std::string pairwise_footer(const std::string& db_name, size_t n_seqs, uint64_t total, int go, int ge) {  // :666-680
    std::string o = "  Database: ";
    for (auto& l : ncbi_wrap_flat(db_name, 68)) o += l + "\n";
    o += "  Number of letters in database: " + with_commas(total) + "\n";
    o += "  Number of sequences in database:  " + with_commas(n_seqs) + "\n\n\n\n";
    char b[128];
    snprintf(b, sizeof b, "Matrix: blastn matrix 0 0\nGap Penalties: Existence: %d, Extension: %.2f\n", go, (double)ge);
    return o + b;
}

}  // namespace rmbo
