// rmb_oracle_seq.cpp -- encoding, FASTA/.2bit input, CRandom, packing, matrix, DUST.
// TEST INFRASTRUCTURE: the CPU oracle.  See rmb_oracle.hpp.
#include "rmb_oracle.hpp"

#include <cmath>
#include <cstring>
#include <deque>
#include <fstream>
#include <sstream>
#include <stdexcept>

namespace rmbo {

// encoding.rs:53 BLASTNA_TO_IUPAC, encoding.rs:65 BLASTNA_COMPLEMENT
const uint8_t BLASTNA_TO_IUPAC[17] = "ACGTRYMKWSBDHVN-";
const uint8_t COMPLEMENT[16] = {3, 2, 1, 0, 5, 4, 7, 6, 8, 9, 13, 12, 11, 10, 14, 15};

// encoding.rs:19-50: unknown characters map to N; '-' and 'X' are N in a sequence.
uint8_t iupac_to_blastna(uint8_t c) {
    switch (c | 0x20) {
        case 'a': return 0;
        case 'c': return 1;
        case 'g': return 2;
        case 't': case 'u': return 3;
        case 'r': return 4;
        case 'y': return 5;
        case 'm': return 6;
        case 'k': return 7;
        case 'w': return 8;
        case 's': return 9;
        case 'b': return 10;
        case 'd': return 11;
        case 'h': return 12;
        case 'v': return 13;
        default: return 14;
    }
}

std::vector<uint8_t> encode_iupac(const std::string& ascii) {
    std::vector<uint8_t> out;
    out.reserve(ascii.size() + 2);
    out.push_back(SENTINEL);
    for (unsigned char c : ascii) out.push_back(c < 128 ? iupac_to_blastna(c) : 14);
    out.push_back(SENTINEL);
    return out;
}

std::vector<uint8_t> revcomp(const uint8_t* s, size_t n) {
    std::vector<uint8_t> out(n);
    for (size_t i = 0; i < n; ++i) out[i] = COMPLEMENT[s[n - 1 - i] & 15];
    return out;
}

// ---- CRandom: seq/twobit.rs:73-135 -------------------------------------------------------
NcbiRandom::NcbiRandom(uint32_t seed) {
    state[0] = seed;
    for (int i = 1; i < 33; ++i) state[i] = 1103515245u * state[i - 1] + 12345u;
    rj = 12;
    rk = 32;
    for (int i = 0; i < 330; ++i) raw();
}
uint32_t NcbiRandom::raw() {
    uint32_t r = state[rk] + state[rj];
    state[rk] = r;
    rk -= 1;
    rj -= 1;
    if (rk < 0) rk = 32;
    else if (rj < 0) rj = 32;
    return r;
}
// encoding.rs:92 NCBI_AMBIG_ALLOWED: [count, base0, base1, base2]
static const uint8_t AMBIG_ALLOWED[16][4] = {
    {0, 0, 0, 0}, {0, 0, 0, 0}, {0, 0, 0, 0}, {0, 0, 0, 0}, {2, 0, 2, 0}, {2, 1, 3, 0},
    {2, 0, 1, 0}, {2, 2, 3, 0}, {2, 0, 3, 0}, {2, 1, 2, 0}, {3, 1, 2, 3}, {3, 0, 2, 3},
    {3, 0, 1, 3}, {3, 0, 1, 2}, {4, 0, 0, 0}, {0, 0, 0, 0}};
uint8_t NcbiRandom::next_base_iupac(uint8_t code) {
    uint32_t r = get_rand();
    if (code == 14) return (uint8_t)(r & 3);
    const uint8_t* e = AMBIG_ALLOWED[code];
    return e[1 + (r % e[0])];
}

// ---- FASTA: seq/fasta.rs:83-170 ----------------------------------------------------------
static bool is_sequence_char(unsigned char c) {
    switch (c & ~0x20) {
        case 'A': case 'C': case 'G': case 'T': case 'U': case 'R': case 'Y': case 'M': case 'K':
        case 'W': case 'S': case 'B': case 'D': case 'H': case 'V': case 'N': case 'X':
            return true;
        default:
            return c == '-';
    }
}

std::vector<FastaRecord> read_fasta_text(const std::string& text) {
    std::vector<FastaRecord> out;
    std::string seq;
    bool have = false;
    FastaRecord cur;
    size_t pos = 0;
    auto flush = [&]() {
        if (have) {
            cur.seq = encode_iupac(seq);
            out.push_back(std::move(cur));
            cur = FastaRecord();
        }
        seq.clear();
    };
    while (pos < text.size()) {
        size_t e = text.find('\n', pos);
        if (e == std::string::npos) e = text.size();
        std::string line = text.substr(pos, e - pos);
        pos = e + 1;
        if (!line.empty() && line[0] == '>') {
            flush();
            std::string def = line.substr(1);
            while (!def.empty() && (def.back() == '\r' || def.back() == '\n')) def.pop_back();
            std::istringstream is(def);
            std::string id;
            is >> id;
            if (id.empty()) throw std::runtime_error("'>' with no sequence id");
            cur.id = id;
            cur.defline = def;
            have = true;
            continue;
        }
        size_t a = 0, b = line.size();
        while (a < b && isspace((unsigned char)line[a])) ++a;
        while (b > a && isspace((unsigned char)line[b - 1])) --b;
        if (a == b) continue;
        if (!have) throw std::runtime_error("sequence data before the first '>' header");
        for (size_t i = a; i < b; ++i)
            if (!is_sequence_char((unsigned char)line[i]))
                throw std::runtime_error("invalid nucleotide code in record " + cur.id);
        seq.append(line, a, b - a);
    }
    flush();
    return out;
}

static std::string slurp(const std::string& path) {
    std::ifstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("cannot open " + path);
    std::ostringstream ss;
    ss << f.rdbuf();
    return ss.str();
}

std::vector<FastaRecord> read_fasta(const std::string& path) { return read_fasta_text(slurp(path)); }

// ---- packing: blast/util.rs:41-115 -------------------------------------------------------
static const uint8_t BLASTNA_TO_NCBI4NA[16] = {1, 2, 4, 8, 5, 10, 3, 12, 9, 6, 14, 13, 11, 7, 15, 0};

std::vector<uint8_t> pack_ncbi2na(const uint8_t* bases, size_t len) {
    std::vector<uint8_t> packed(3 + (len + 3) / 4 + 3, 0);
    NcbiRandom* rng = nullptr;
    NcbiRandom storage(0);
    auto conv = [&](uint8_t b) -> uint8_t {
        if (b < 4) return b;
        if (!rng) { storage = NcbiRandom((uint32_t)len); rng = &storage; }
        uint8_t n4 = BLASTNA_TO_NCBI4NA[b];
        if (n4 == 0 || n4 == 15) return (uint8_t)(rng->get_rand() & 3);
        uint32_t bits = __builtin_popcount(n4);
        uint32_t pick = rng->get_rand() % bits;
        for (uint8_t j = 0; j < 4; ++j)
            if (n4 & (1 << j)) {
                if (pick == 0) return j;
                --pick;
            }
        return 0;
    };
    for (size_t j = 0; j < len / 4; ++j) {
        uint8_t b0 = conv(bases[4 * j]), b1 = conv(bases[4 * j + 1]), b2 = conv(bases[4 * j + 2]),
                b3 = conv(bases[4 * j + 3]);
        packed[3 + j] = (uint8_t)((b0 << 6) | (b1 << 4) | (b2 << 2) | b3);
    }
    size_t rem = len % 4;
    if (rem) {
        size_t base = len / 4;
        uint8_t byte = 0;
        for (size_t k = 0; k < rem; ++k) byte = (uint8_t)((byte << 2) | conv(bases[4 * base + k]));
        packed[3 + base] = (uint8_t)(byte << (2 * (4 - rem)));
    }
    return packed;
}

// ---- subjects: seq/fasta_db.rs:86-131, seq/mod.rs:56-100 ---------------------------------
Subject make_subject_resolved(const std::string& id, std::vector<uint8_t> plus,
                              std::vector<uint8_t> n_mask) {
    Subject s;
    s.id = id;
    s.plus = std::move(plus);
    s.n_mask = std::move(n_mask);
    size_t n = s.plus.size() - 2;
    s.rc = revcomp(s.plus.data(), s.plus.size());
    s.packed = pack_ncbi2na(s.plus.data() + 1, n);
    if (s.n_mask.empty()) {
        s.align = s.plus;
        s.align_rc = s.rc;
    } else {
        s.align = s.plus;
        for (size_t i = 0; i < s.n_mask.size(); ++i)
            if (s.n_mask[i]) s.align[i + 1] = s.n_mask[i];
        s.align_rc = revcomp(s.align.data(), s.align.size());
        s.n_mask_rc.resize(s.n_mask.size());
        for (size_t i = 0; i < s.n_mask.size(); ++i) {
            uint8_t c = s.n_mask[s.n_mask.size() - 1 - i];
            s.n_mask_rc[i] = c == 0 ? 0 : COMPLEMENT[c];
        }
    }
    return s;
}

Subject make_subject(const std::string& id, const std::vector<uint8_t>& raw) {
    size_t n = raw.size() - 2;
    std::vector<uint8_t> plus = raw;
    std::vector<uint8_t> mask;
    bool any = false;
    for (size_t i = 1; i <= n; ++i)
        if (raw[i] >= 4 && raw[i] <= 14) { any = true; break; }
    if (any) {
        NcbiRandom rng((uint32_t)n);
        mask.assign(n, 0);
        for (size_t i = 1; i <= n; ++i) {
            uint8_t c = raw[i];
            if (c >= 4 && c <= 14) {
                plus[i] = rng.next_base_iupac(c);
                mask[i - 1] = c;
            }
        }
    }
    return make_subject_resolved(id, std::move(plus), std::move(mask));
}

// ---- .2bit: seq/twobit.rs:171-390 ---------------------------------------------------------
std::vector<Subject> read_twobit(const std::string& path) {
    std::string d = slurp(path);
    auto u32le = [&](size_t p) -> uint32_t {
        if (p + 4 > d.size()) throw std::runtime_error("corrupt 2bit");
        uint32_t v;
        memcpy(&v, d.data() + p, 4);
        return v;
    };
    uint32_t magic = u32le(0);
    bool swap = false;
    if (magic == 0x1A412743u) swap = false;
    else if (magic == 0x4327411Au) swap = true;
    else throw std::runtime_error("bad 2bit magic");
    auto r32 = [&](size_t p) { uint32_t v = u32le(p); return swap ? __builtin_bswap32(v) : v; };
    uint32_t count = r32(8);
    size_t pos = 16;
    std::vector<std::pair<std::string, uint32_t>> idx;
    for (uint32_t i = 0; i < count; ++i) {
        uint8_t nl = (uint8_t)d[pos++];
        std::string name = d.substr(pos, nl);
        pos += nl;
        idx.push_back({name, r32(pos)});
        pos += 4;
    }
    static const uint8_t UCSC[4] = {3, 1, 0, 2};
    std::vector<Subject> out;
    for (auto& [name, off] : idx) {
        size_t base = off;
        uint32_t dna = r32(base);
        uint32_t nbc = r32(base + 4);
        size_t nstarts = base + 8, nsizes = nstarts + 4 * (size_t)nbc;
        size_t mcount_off = nsizes + 4 * (size_t)nbc;
        uint32_t mbc = r32(mcount_off);
        size_t reserved = mcount_off + 4 + 8 * (size_t)mbc;
        size_t dna_off = reserved + 4;
        std::vector<uint8_t> plus(dna + 2, SENTINEL);
        for (uint32_t i = 0; i < dna; ++i) {
            uint8_t byte = (uint8_t)d[dna_off + i / 4];
            plus[i + 1] = UCSC[(byte >> (6 - (i % 4) * 2)) & 3];
        }
        std::vector<uint8_t> mask;
        if (nbc > 0) {
            mask.assign(dna, 0);
            NcbiRandom rng(dna);
            for (uint32_t bi = 0; bi < nbc; ++bi) {
                uint32_t st = r32(nstarts + 4 * bi), sz = r32(nsizes + 4 * bi);
                uint64_t en64 = std::min<uint64_t>((uint64_t)st + sz, dna);
                uint32_t en = (uint32_t)en64;
                st = std::min(st, en);
                for (uint32_t p = st; p < en; ++p) {
                    plus[p + 1] = (uint8_t)(rng.get_rand() & 3);
                    mask[p] = 14;
                }
            }
        }
        out.push_back(make_subject_resolved(name, std::move(plus), std::move(mask)));
    }
    return out;
}

// ---- matrix: matrix.rs:76-324 -------------------------------------------------------------
static uint8_t matrix_symbol_to_blastna(char c) {
    switch (c) {
        case 'A': return 0; case 'C': return 1; case 'G': return 2; case 'T': return 3;
        case 'R': return 4; case 'Y': return 5; case 'M': return 6; case 'K': return 7;
        case 'W': return 8; case 'S': return 9; case 'B': return 10; case 'D': return 11;
        case 'H': return 12; case 'V': return 13; case 'N': return 14;
        default: return 15;
    }
}

static std::vector<std::string> split_ws(const std::string& s) {
    std::vector<std::string> t;
    std::istringstream is(s);
    std::string x;
    while (is >> x) t.push_back(x);
    return t;
}

static bool parse_i32(const std::string& t, int32_t& v) {
    if (t.empty()) return false;
    size_t i = 0;
    bool neg = false;
    if (t[0] == '+' || t[0] == '-') { neg = t[0] == '-'; i = 1; }
    if (i == t.size()) return false;
    int64_t acc = 0;
    for (; i < t.size(); ++i) {
        if (t[i] < '0' || t[i] > '9') return false;
        acc = acc * 10 + (t[i] - '0');
        if (acc > (int64_t)2147483648LL) return false;
    }
    if (neg) acc = -acc;
    if (acc < INT32_MIN || acc > INT32_MAX) return false;
    v = (int32_t)acc;
    return true;
}

// matrix.rs:290-324 estimate_lambda (exact operation order kept: f64 sum over i, j)
static double estimate_lambda(const int32_t s[16][16], const double f[16]) {
    double total = f[0] + f[1] + f[2] + f[3];
    if (total < 1e-9) return 0.0;
    auto eval = [&](double lambda) {
        double sum = 0.0;
        for (int i = 0; i < 16; ++i)
            for (int j = 0; j < 16; ++j)
                if (f[i] > 0.0 && f[j] > 0.0) sum += f[i] * f[j] * std::exp(lambda * (double)s[i][j]);
        return sum;
    };
    double lo = 0.0, lambda = 0.5;
    for (;;) {
        double sum = eval(lambda);
        if (sum < 1.0) {
            lo = lambda;
            lambda *= 2.0;
            if (lambda > 1000.0) return 0.0;
        } else {
            break;
        }
    }
    double hi = lambda;
    while (hi - lo > 0.00001) {
        lambda = (lo + hi) / 2.0;
        double sum = eval(lambda);
        if (sum >= 1.0) hi = lambda;
        else lo = lambda;
    }
    return lambda;
}

Matrix parse_matrix(const std::string& text, const std::string& name) {
    Matrix m;
    m.name = name;
    for (double& x : m.freqs) x = 0.0;
    bool have_freqs = false;
    std::vector<char> cols;
    bool have_header = false;
    std::vector<std::vector<int32_t>> rows;
    std::istringstream is(text);
    std::string line;
    int lineno = 0;
    auto fail = [&](const std::string& msg) {
        throw std::runtime_error("matrix line " + std::to_string(lineno) + ": " + msg);
    };
    while (std::getline(is, line)) {
        ++lineno;
        size_t a = 0, b = line.size();
        while (a < b && isspace((unsigned char)line[a])) ++a;
        while (b > a && isspace((unsigned char)line[b - 1])) --b;
        std::string t = line.substr(a, b - a);
        if (t.empty()) continue;
        if (t[0] == '#') {
            if (t.rfind("# KARLIN", 0) == 0 || t.rfind("#KARLIN", 0) == 0) {  // matrix.rs:100-103, 248-264
                auto tok = split_ws(t.substr(t[1] == ' ' ? 8 : 7));
                for (int i = 0; i < 5; ++i) m.karlin[i] = 0.0;
                for (size_t i = 0; i + 1 < tok.size(); i += 2) {
                    char* end = nullptr;
                    double v = strtod(tok[i + 1].c_str(), &end);
                    if (*end != 0 || tok[i + 1].empty()) fail("bad KARLIN value");
                    std::string key = tok[i];
                    for (auto& ch : key) ch = (char)tolower((unsigned char)ch);
                    if (key == "lambda") m.karlin[0] = v;
                    else if (key == "k") m.karlin[1] = v;
                    else if (key == "h") m.karlin[2] = v;
                    else if (key == "alpha") m.karlin[3] = v;
                    else if (key == "beta") m.karlin[4] = v;
                    else fail("unknown KARLIN key");
                }
                m.has_karlin = true;
                continue;
            }
            size_t at = t.find("FREQS");
            if (at != std::string::npos) {
                if (have_freqs) fail("a second FREQS line");
                auto tok = split_ws(t.substr(at + 5));
                if (tok.size() != 8) fail("FREQS needs 4 base/frequency pairs");
                bool seen[4] = {false, false, false, false};
                for (int k = 0; k < 4; ++k) {
                    std::string bname = tok[2 * k];
                    int idx = -1;
                    if (bname.size() == 1) {
                        char c = (char)toupper((unsigned char)bname[0]);
                        idx = c == 'A' ? 0 : c == 'C' ? 1 : c == 'G' ? 2 : c == 'T' ? 3 : -1;
                    }
                    if (idx < 0) fail("FREQS base is not A, C, G or T");
                    if (seen[idx]) fail("FREQS gives a base twice");
                    seen[idx] = true;
                    char* end = nullptr;
                    double fv = strtod(tok[2 * k + 1].c_str(), &end);
                    if (*end != 0 || !std::isfinite(fv) || fv < 0.0) fail("FREQS value is not a frequency");
                    m.freqs[idx] = fv;
                }
                double sum = m.freqs[0] + m.freqs[1] + m.freqs[2] + m.freqs[3];
                if (!(sum >= 0.999 && sum <= 1.001)) fail("FREQS frequencies do not sum to 1");
                have_freqs = true;
            }
            continue;
        }
        auto tok = split_ws(t);
        if (!have_header) {
            for (auto& x : tok) {
                if (x.size() != 1 || !(isalpha((unsigned char)x[0]) || x[0] == '-'))
                    fail("expected the column header");
                char c = (char)toupper((unsigned char)x[0]);
                for (char e : cols)
                    if (e == c) fail("column symbol appears twice");
                cols.push_back(c);
            }
            have_header = true;
            continue;
        }
        size_t row = rows.size();
        if (row == cols.size()) fail("more rows than columns");
        int32_t dummy;
        size_t first = 0;
        if (!parse_i32(tok[0], dummy)) {
            if (tok[0].size() != 1 || toupper((unsigned char)tok[0][0]) != cols[row]) fail("bad row label");
            first = 1;
        }
        std::vector<int32_t> sc;
        for (size_t i = first; i < tok.size(); ++i) {
            int32_t v;
            if (!parse_i32(tok[i], v)) fail("score is not an integer");
            sc.push_back(v);
        }
        if (sc.size() != cols.size()) fail("wrong number of scores");
        rows.push_back(sc);
    }
    if (!have_header) throw std::runtime_error("no column header found");
    if (rows.size() != cols.size()) throw std::runtime_error("the matrix must be square");
    if (!have_freqs) throw std::runtime_error("no FREQS line");
    for (auto& r : m.s)
        for (auto& v : r) v = -32768;
    for (size_t ri = 0; ri < rows.size(); ++ri) {
        uint8_t r = matrix_symbol_to_blastna(cols[ri]);
        for (size_t ci = 0; ci < rows[ri].size(); ++ci) m.s[r][matrix_symbol_to_blastna(cols[ci])] = rows[ri][ci];
    }
    for (int i = 0; i < 16; ++i) {
        m.s[15][i] = INT32_MIN / 2;
        m.s[i][15] = INT32_MIN / 2;
    }
    double expected = 0.0;
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) expected += m.freqs[i] * m.freqs[j] * (double)m.s[i][j];
    if (expected >= 0.0) throw std::runtime_error("the expected score of an aligned pair must be negative");
    m.lambda = estimate_lambda(m.s, m.freqs);
    return m;
}

Matrix load_matrix(const std::string& path) { return parse_matrix(slurp(path), path); }

// ---- KA ungapped cutoff: search/ka_cutoff.rs:44-155 ---------------------------------------
// NCBI blast_stat.c rmblast_*_values (lambda, K) per RepeatMasker matrix and gap costs; the
// values must match the reference's table entry for entry because they pick the cutoff.
struct KaRow { const char* name; int go, ge; double lambda, k; };
static const KaRow KA_TABLE[] = {
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

int ungapped_cutoff(const std::string& matrix_name, int go, int ge, int min_raw, uint64_t qlen,
                    uint64_t avg) {
    int fallback = min_raw > 0 ? min_raw / 2 : 1;
    std::string base = matrix_name;
    size_t sl = base.find_last_of('/');
    if (sl != std::string::npos) base = base.substr(sl + 1);
    for (const KaRow& r : KA_TABLE) {
        if (r.go != go || r.ge != ge || strcasecmp(r.name, base.c_str()) != 0) continue;
        if (avg == 0 || r.lambda <= 0.0 || r.k <= 0.0) return fallback;
        uint64_t q2 = qlen * 2;
        uint64_t searchsp = std::min(avg, q2) * avg;
        int es = (int)std::ceil(std::log(r.k * (double)searchsp / 0.05) / r.lambda);
        int c = es > 1 ? es : 1;
        return c < fallback ? c : fallback;
    }
    return fallback;
}

// ---- DUST: filter/dust.rs:15-331, 462-489 --------------------------------------------------
namespace {
struct Lfg {  // dust.rs:24-57, NCBI CRandom with its fixed initial state
    uint32_t st[33] = {0xd53f1852, 0xdfc78b83, 0x4f256096, 0x0e643df7, 0x82c359bf, 0xc7794dfa, 0xd5e9ffaa,
                       0x2c8cb64a, 0x2f07b334, 0xad5a7eb5, 0x96dc0cde, 0x6fc24589, 0xa5853646, 0xe71576e2,
                       0x0dae30df, 0xb09ce711, 0x5e56ef87, 0x4b4b0082, 0x6f4f340e, 0xc5bb17e8, 0xd788d765,
                       0x67498087, 0x9d7aba26, 0x261351d4, 0x411ee7ea, 0x0393a263, 0x2c5a5835, 0xc115fcd8,
                       0x25e9132c, 0xd0c6e906, 0xc2bc5b2d, 0x6c065c98, 0x6e37bd55};
    long rk = 32, rj = 12;
    uint32_t get() {
        uint32_t r = st[rk] + st[rj];
        st[rk] = r;
        --rk;
        --rj;
        if (rk < 0) rk = 32;
        else if (rj < 0) rj = 32;
        return r >> 1;
    }
};
uint8_t cvt_base(uint8_t b, Lfg& rng) {
    switch (b) {
        case 1: return 1;
        case 2: return 2;
        case 3: return 3;
        case 14: return (uint8_t)(rng.get() & 3);
        default: return 0;
    }
}
struct Perfect { size_t start, stop; uint32_t score, len; };

struct Triplets {  // dust.rs:95-274
    std::deque<uint8_t> list;  // front = newest
    uint32_t c_w[64] = {0}, r_w = 0, c_v[64] = {0}, r_v = 0, num_diff = 0;
    size_t max_size;
    uint32_t low_k;
    size_t start, stop, l;
    Triplets(size_t window, uint32_t lk, size_t js) : max_size(window >= 2 ? window - 2 : 0), low_k(lk),
                                                       start(js), stop(js), l(js) {}
    void add_w(uint8_t t) { if (c_w[t] == 0) ++num_diff; r_w += c_w[t]; ++c_w[t]; }
    void rem_w(uint8_t t) { --c_w[t]; if (c_w[t] == 0) --num_diff; r_w -= c_w[t]; }
    void add_v(uint8_t t) { r_v += c_v[t]; ++c_v[t]; }
    void rem_v(uint8_t t) { --c_v[t]; r_v -= c_v[t]; }
    bool shift_high(uint8_t t, std::vector<Perfect>& perfect) {
        uint8_t s = list.back();
        list.pop_back();
        rem_w(s);
        ++start;
        list.push_front(t);
        add_w(t);
        ++stop;
        if (num_diff <= 1) {
            perfect.insert(perfect.begin(), Perfect{start, stop + 1, 0, 0});
            return false;
        }
        return true;
    }
    bool shift_window(uint8_t t, std::vector<Perfect>& perfect) {
        if (list.size() >= max_size) {
            if (num_diff <= 1) return shift_high(t, perfect);
            uint8_t s = list.back();
            list.pop_back();
            rem_w(s);
            if (l == start) { ++l; rem_v(s); }
            ++start;
        }
        list.push_front(t);
        add_w(t);
        add_v(t);
        if (c_v[t] > low_k) {
            size_t off = list.size() - (l - start) - 1;
            size_t idx = off;
            for (;;) {
                uint8_t s = list[idx];
                rem_v(s);
                ++l;
                if (s == t) break;
                if (idx == 0) break;
                --idx;
            }
        }
        ++stop;
        if (list.size() >= max_size && num_diff <= 1) {
            perfect.clear();
            perfect.insert(perfect.begin(), Perfect{start, stop + 1, 0, 0});
            return false;
        }
        return true;
    }
    bool needs_processing(const std::vector<uint32_t>& th) const {
        size_t count = stop - l;
        return count < list.size() && r_w * 10 > th[count];
    }
    void find_perfect(std::vector<Perfect>& perfect, const std::vector<uint32_t>& th) const {
        uint32_t counts[64];
        memcpy(counts, c_v, sizeof(counts));
        uint32_t score = r_v;
        uint32_t count = (uint32_t)(stop - l);
        size_t it = 0;
        uint32_t max_score = 0, max_len = 0;
        size_t start_idx = stop - l;
        for (size_t idx = start_idx; idx < list.size(); ++idx) {
            uint8_t ti = list[idx];
            uint32_t cnt = counts[ti];
            score += counts[ti];
            counts[ti] += 1;
            if (cnt > 0 && score * 10 > th[count]) {
                size_t seq_pos = stop - idx;
                size_t pos = seq_pos - 1;  // wraps like the reference's usize
                while (it < perfect.size() && pos <= perfect[it].start) {
                    const Perfect& pi = perfect[it];
                    if (max_score == 0 || max_len * pi.score > max_score * pi.len) {
                        max_score = pi.score;
                        max_len = pi.len;
                    }
                    ++it;
                }
                if (max_score == 0 || score * max_len >= max_score * count) {
                    max_score = score;
                    max_len = count;
                    perfect.insert(perfect.begin() + it, Perfect{pos, stop + 1, max_score, count});
                }
            }
            ++count;
        }
    }
};

void save_masked(std::vector<Perfect>& perfect, std::vector<std::pair<size_t, size_t>>& res, size_t wstart,
                 size_t linker) {
    if (perfect.empty()) return;
    size_t b0 = perfect.back().start, b1 = perfect.back().stop;
    if (b0 < wstart) {
        if (!res.empty() && res.back().second + linker >= b0) {
            if (b1 > res.back().second) res.back().second = b1;
        } else {
            res.push_back({b0, b1});
        }
        while (!perfect.empty() && perfect.back().start < wstart) perfect.pop_back();
    }
}

std::vector<std::pair<size_t, size_t>> dust_intervals(const uint8_t* bases, size_t n, Lfg& rng) {
    const size_t window = 64, linker = 1;
    const uint32_t level = 20;
    std::vector<std::pair<size_t, size_t>> res;
    if (n < 3) return res;
    std::vector<uint8_t> conv(n, 0);
    std::vector<uint32_t> th(window - 2, 1);
    for (size_t i = 1; i < th.size(); ++i) th[i] = (uint32_t)i * level;
    uint32_t low_k = level / 5;
    std::vector<Perfect> perfect;
    size_t j_start = 0;
    for (;;) {
        if (n < j_start + 4) break;
        perfect.clear();
        Triplets w(window, low_k, j_start);
        size_t num_local = n - 2 - j_start;
        size_t j = j_start, j_end = j_start + num_local;
        size_t conv_from = j_start;
        for (;;) {
            if (j >= j_end) break;
            save_masked(perfect, res, w.start, linker);
            while (conv_from <= j + 2) { conv[conv_from] = cvt_base(bases[conv_from], rng); ++conv_from; }
            uint8_t t = (uint8_t)((conv[j] << 4) | (conv[j + 1] << 2) | conv[j + 2]);
            ++j;
            if (w.shift_window(t, perfect)) {
                if (w.needs_processing(th)) w.find_perfect(perfect, th);
            } else {
                for (;;) {
                    if (j >= j_end) break;
                    save_masked(perfect, res, w.start, linker);
                    while (conv_from <= j + 2) { conv[conv_from] = cvt_base(bases[conv_from], rng); ++conv_from; }
                    uint8_t t2 = (uint8_t)((conv[j] << 4) | (conv[j + 1] << 2) | conv[j + 2]);
                    if (w.shift_window(t2, perfect)) break;
                    ++j;
                }
                break;
            }
        }
        size_t wstart = w.start;
        while (!perfect.empty()) {
            save_masked(perfect, res, wstart, linker);
            ++wstart;
        }
        if (w.start > j_start) j_start = w.start;
        else break;
    }
    return res;
}
}  // namespace

std::vector<std::pair<size_t, size_t>> dust_mask(std::vector<uint8_t>& seq) {
    size_t n = seq.size() >= 2 ? seq.size() - 2 : 0;
    if (n < 3) return {};
    Lfg rng;
    auto merged = dust_intervals(seq.data() + 1, n, rng);
    for (auto& [s, e] : merged) {
        size_t end = std::min(e, n - 1);
        for (size_t p = s; p <= end; ++p) seq[p + 1] = 14;
    }
    return merged;
}

}  // namespace rmbo
