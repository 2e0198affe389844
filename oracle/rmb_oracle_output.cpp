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
