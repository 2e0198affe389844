// rmb_io.cpp -- input preparation entry points of include/rmb_gpu.h: matrix parsing, IUPAC
// encoding and CRandom resolution of subject ambiguity codes.
#include <algorithm>
#include <cctype>
#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/rmb_gpu.h"
#include "rmb_glue.hpp"

namespace {

uint8_t code_of(unsigned char c) {  // encoding.rs:19-50
    switch (c | 0x20) {
        case 'a': return 0; case 'c': return 1; case 'g': return 2; case 't': case 'u': return 3;
        case 'r': return 4; case 'y': return 5; case 'm': return 6; case 'k': return 7;
        case 'w': return 8; case 's': return 9; case 'b': return 10; case 'd': return 11;
        case 'h': return 12; case 'v': return 13; default: return 14;
    }
}

uint8_t header_slot(char c) {  // matrix.rs:251-258: non-IUPAC header symbols land in the gap slot
    const char* order = "ACGTRYMKWSBDHVN";
    for (int i = 0; i < 15; ++i)
        if (order[i] == c) return (uint8_t)i;
    return 15;
}

// NCBI CRandom (seq/twobit.rs:73-135): lagged-Fibonacci state of 33 words seeded by a
// linear congruence, 330 warm-up draws, output = raw >> 1.
struct CRandom {
    uint32_t s[33];
    int j = 12, k = 32;
    explicit CRandom(uint32_t seed) {
        s[0] = seed;
        for (int i = 1; i < 33; ++i) s[i] = 1103515245u * s[i - 1] + 12345u;
        for (int i = 0; i < 330; ++i) next();
    }
    uint32_t next() {
        const uint32_t r = s[k] + s[j];
        s[k] = r;
        if (--k < 0) { k = 32; --j; }
        else if (--j < 0) j = 32;
        return r;
    }
};

// encoding.rs:92-110: allowed bases per ambiguity code in A,C,G,T order
const uint8_t ALLOWED[16][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}, {0, 0, 0, 0}, {0, 0, 0, 0}, {2, 0, 2, 0}, {2, 1, 3, 0},
                                {2, 0, 1, 0}, {2, 2, 3, 0}, {2, 0, 3, 0}, {2, 1, 2, 0}, {3, 1, 2, 3}, {3, 0, 2, 3},
                                {3, 0, 1, 3}, {3, 0, 1, 2}, {4, 0, 0, 0}, {0, 0, 0, 0}};

std::vector<std::string> tokens(const std::string& s) {
    std::vector<std::string> t;
    std::istringstream is(s);
    std::string x;
    while (is >> x) t.push_back(x);
    return t;
}

bool to_i32(const std::string& t, int32_t& v) {
    if (t.empty()) return false;
    char* end = nullptr;
    errno = 0;
    const long long x = strtoll(t.c_str(), &end, 10);
    if (*end || errno || x < INT32_MIN || x > INT32_MAX || t[0] == ' ') return false;
    v = (int32_t)x;
    return true;
}

}  // namespace

extern "C" {

void rmb_encode_iupac(const char* ascii, size_t n, uint8_t* out) {
    out[0] = 15;
    for (size_t i = 0; i < n; ++i) {
        const unsigned char c = (unsigned char)ascii[i];
        out[i + 1] = c < 128 ? code_of(c) : 14;
    }
    out[n + 1] = 15;
}

void rmb_resolve_subject(const uint8_t* raw, uint32_t n, uint8_t* plus, uint8_t* n_mask, int32_t* has_mask) {
    memcpy(plus, raw, (size_t)n + 2);
    memset(n_mask, 0, n);
    *has_mask = 0;
    CRandom* rng = nullptr;
    CRandom storage(0);
    for (uint32_t i = 1; i <= n; ++i) {
        const uint8_t c = raw[i];
        if (c < 4 || c > 14) continue;
        if (!rng) { storage = CRandom(n); rng = &storage; }
        const uint32_t r = rng->next() >> 1;
        plus[i] = c == 14 ? (uint8_t)(r & 3) : ALLOWED[c][1 + r % ALLOWED[c][0]];
        n_mask[i - 1] = c;
        *has_mask = 1;
    }
}

// seq/twobit.rs:73-135 (the .2bit path of SubjectDb): the N blocks of a .2bit record, drawn from
// CRandom seeded with the record's length, block by block in file order; n_mask gets 14 there.
void rmb_resolve_twobit_n(uint32_t n, uint32_t n_blocks, const uint32_t* starts, const uint32_t* sizes,
                          uint8_t* plus, uint8_t* n_mask) {
    if (!n_blocks) return;
    CRandom rng(n);
    for (uint32_t b = 0; b < n_blocks; ++b) {
        const uint64_t e64 = std::min<uint64_t>((uint64_t)starts[b] + sizes[b], n);
        const uint32_t e = (uint32_t)e64, st = std::min(starts[b], e);
        for (uint32_t p = st; p < e; ++p) {
            plus[p + 1] = (uint8_t)((rng.next() >> 1) & 3u);
            n_mask[p] = 14;
        }
    }
}

int rmb_matrix_parse(const char* text, int32_t scores[256], double freqs[16], double* lambda, char* err,
                     size_t errlen) {
    try {
        double f[16] = {0};
        bool have_freqs = false, have_header = false;
        std::vector<char> cols;
        std::vector<std::vector<int32_t>> rows;
        std::istringstream is(text ? text : "");
        std::string line;
        int ln = 0;
        auto fail = [&](const std::string& m) { throw std::runtime_error("line " + std::to_string(ln) + ": " + m); };
        while (std::getline(is, line)) {
            ++ln;
            const size_t a = line.find_first_not_of(" \t\r\n");
            if (a == std::string::npos) continue;
            const std::string t = line.substr(a, line.find_last_not_of(" \t\r\n") - a + 1);
            if (t[0] == '#') {
                const size_t at = t.find("FREQS");
                if (at == std::string::npos) continue;
                if (have_freqs) fail("a second FREQS line");
                const auto tk = tokens(t.substr(at + 5));
                if (tk.size() != 8) fail("FREQS needs 4 base/frequency pairs (A, C, G and T)");
                bool seen[4] = {false, false, false, false};
                for (int k = 0; k < 4; ++k) {
                    const std::string& b = tk[2 * k];
                    const int idx = b.size() != 1 ? -1 : std::string("ACGT").find((char)toupper(b[0]));
                    if (idx < 0 || idx > 3) fail("FREQS base is not A, C, G or T");
                    if (seen[idx]) fail("FREQS gives a base twice");
                    seen[idx] = true;
                    char* e = nullptr;
                    const double v = strtod(tk[2 * k + 1].c_str(), &e);
                    if (*e || !std::isfinite(v) || v < 0.0) fail("FREQS value is not a frequency");
                    f[idx] = v;
                }
                const double sum = f[0] + f[1] + f[2] + f[3];
                if (!(sum >= 0.999 && sum <= 1.001)) fail("FREQS frequencies do not sum to 1");
                have_freqs = true;
                continue;
            }
            const auto tk = tokens(t);
            if (!have_header) {
                for (const auto& x : tk) {
                    if (x.size() != 1 || !(isalpha((unsigned char)x[0]) || x[0] == '-')) fail("expected the column header");
                    const char c = (char)toupper((unsigned char)x[0]);
                    for (char e : cols)
                        if (e == c) fail("column symbol appears twice");
                    cols.push_back(c);
                }
                have_header = true;
                continue;
            }
            if (rows.size() == cols.size()) fail("more rows than columns");
            int32_t v;
            size_t first = 0;
            if (!to_i32(tk[0], v)) {
                if (tk[0].size() != 1 || toupper((unsigned char)tk[0][0]) != cols[rows.size()]) fail("bad row label");
                first = 1;
            }
            std::vector<int32_t> r;
            for (size_t i = first; i < tk.size(); ++i) {
                if (!to_i32(tk[i], v)) fail("score is not an integer");
                r.push_back(v);
            }
            if (r.size() != cols.size()) fail("wrong number of scores");
            rows.push_back(r);
        }
        if (!have_header) throw std::runtime_error("no column header found");
        if (rows.size() != cols.size()) throw std::runtime_error("the matrix must be square");
        if (!have_freqs) throw std::runtime_error("no FREQS line; NCBI requires one");
        int32_t s[16][16];
        for (auto& r : s)
            for (auto& v : r) v = -32768;
        for (size_t ri = 0; ri < rows.size(); ++ri)
            for (size_t ci = 0; ci < rows[ri].size(); ++ci) s[header_slot(cols[ri])][header_slot(cols[ci])] = rows[ri][ci];
        for (int i = 0; i < 16; ++i) { s[15][i] = INT32_MIN / 2; s[i][15] = INT32_MIN / 2; }
        double expected = 0.0;
        for (int i = 0; i < 4; ++i)
            for (int j = 0; j < 4; ++j) expected += f[i] * f[j] * (double)s[i][j];
        if (expected >= 0.0) throw std::runtime_error("the expected score of an aligned pair must be negative");
        // matrix.rs:290-324: double from 0.5 until the sum reaches 1, then bisect to 1e-5
        auto eval = [&](double l) {
            double sum = 0.0;
            for (int i = 0; i < 16; ++i)
                for (int j = 0; j < 16; ++j)
                    if (f[i] > 0.0 && f[j] > 0.0) sum += f[i] * f[j] * std::exp(l * (double)s[i][j]);
            return sum;
        };
        double lam = 0.0;
        if (f[0] + f[1] + f[2] + f[3] >= 1e-9) {
            double lo = 0.0, x = 0.5;
            bool none = false;
            for (;;) {
                if (eval(x) < 1.0) {
                    lo = x;
                    x *= 2.0;
                    if (x > 1000.0) { none = true; break; }
                } else break;
            }
            if (!none) {
                double hi = x;
                while (hi - lo > 0.00001) {
                    x = (lo + hi) / 2.0;
                    if (eval(x) >= 1.0) hi = x;
                    else lo = x;
                }
                lam = x;
            }
        }
        for (int i = 0; i < 16; ++i)
            for (int j = 0; j < 16; ++j) scores[i * 16 + j] = s[i][j];
        for (int i = 0; i < 16; ++i) freqs[i] = f[i];
        *lambda = lam;
        return RMB_OK;
    } catch (const std::exception& e) {
        if (err && errlen) {
            strncpy(err, e.what(), errlen - 1);
            err[errlen - 1] = 0;
        }
        return RMB_EINVAL;
    }
}

}  // extern "C"

// rmblast-lib/src/matrix.rs:100-103, 248-264: the key/value pairs of a "# KARLIN" comment line.
static bool karlin_comment(const char* text, double kc[5], std::string& err) {
    std::istringstream is(text ? text : "");
    std::string line;
    bool found = false;
    while (std::getline(is, line)) {
        const size_t a = line.find_first_not_of(" \t\r\n");
        if (a == std::string::npos) continue;
        std::string t = line.substr(a);
        std::string rest;
        if (t.rfind("# KARLIN", 0) == 0) rest = t.substr(8);
        else if (t.rfind("#KARLIN", 0) == 0) rest = t.substr(7);
        else continue;
        for (int i = 0; i < 5; ++i) kc[i] = 0.0;
        std::istringstream ts(rest);
        std::vector<std::string> tk;
        std::string w;
        while (ts >> w) tk.push_back(w);
        for (size_t i = 0; i + 1 < tk.size(); i += 2) {
            char* e = nullptr;
            const double v = strtod(tk[i + 1].c_str(), &e);
            if (!e || *e || tk[i + 1].empty()) {
                err = "bad KARLIN value '" + tk[i + 1] + "' for key '" + tk[i] + "'";
                return false;
            }
            std::string key = tk[i];
            for (auto& c : key) c = (char)std::tolower((unsigned char)c);
            if (key == "lambda") kc[0] = v;
            else if (key == "k") kc[1] = v;
            else if (key == "h") kc[2] = v;
            else if (key == "alpha") kc[3] = v;
            else if (key == "beta") kc[4] = v;
            else {
                err = "unknown KARLIN key '" + tk[i] + "'";
                return false;
            }
        }
        found = true;
    }
    if (!found) err.clear();
    return found;
}

int rmb_ka_resolve(const char* matrix_name, const char* matrix_text, int32_t gap_open, int32_t gap_extend,
                   const double cli[4], double ka[5], int32_t* source, char* err, size_t errlen) {
    try {
        if (!ka) throw std::runtime_error("null argument");
        double kc[5] = {0, 0, 0, 0, 0};
        std::string kerr;
        const bool have_kc = karlin_comment(matrix_text, kc, kerr);
        if (!have_kc && !kerr.empty()) throw std::runtime_error(kerr);
        rmb::KaBlock kb;
        const int src = rmb::ka_resolve(matrix_name ? matrix_name : "", gap_open, gap_extend, cli, have_kc ? kc : nullptr,
                                        kb);
        ka[0] = kb.lambda;
        ka[1] = kb.k;
        ka[2] = kb.h;
        ka[3] = kb.alpha;
        ka[4] = kb.beta;
        if (source) *source = src;
        return RMB_OK;
    } catch (const std::exception& e) {
        if (err && errlen) {
            strncpy(err, e.what(), errlen - 1);
            err[errlen - 1] = 0;
        }
        return RMB_EINVAL;
    }
}
