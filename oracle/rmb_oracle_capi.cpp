// rmb_oracle_capi.cpp -- C entry points of the CPU oracle for the Python tests and the
// CPU-baseline leg of bench.py (TEST INFRASTRUCTURE; the product never links this).
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cmath>
#include <cstring>
#include <sstream>
#include <stdexcept>

#include "rmb_oracle.hpp"

using namespace rmbo;

extern "C" {

struct rmbo_params {
    int32_t gap_open, gap_extend, word_size, xdrop_ungap, xdrop_gap, xdrop_gap_final;
    int32_t min_raw_gapped_score, complexity_adjust, dust, mask_level;  // mask_level < 0 = off
    double evalue;         // --evalue; 0 = off
    double cli_stats[4];   // -matrix_lambda, -matrix_k, -matrix_alpha, -matrix_beta; zeros = unset
};

static Params to_params(const rmbo_params* c, const std::string& mname) {
    Params p;
    p.gap_open = c->gap_open;
    p.gap_extend = c->gap_extend;
    p.word_size = c->word_size;
    p.xdrop_ungap = c->xdrop_ungap;
    p.xdrop_gap = c->xdrop_gap;
    p.xdrop_gap_final = c->xdrop_gap_final;
    p.min_raw_gapped_score = c->min_raw_gapped_score;
    p.complexity_adjust = c->complexity_adjust != 0;
    p.dust = c->dust != 0;
    p.mask_level = c->mask_level < 0 ? 101u : (uint32_t)c->mask_level;
    p.matrix_name = mname;
    p.evalue = c->evalue;
    for (int i = 0; i < 4; ++i) p.cli_stats[i] = c->cli_stats[i];
    return p;
}

static char* dup_string(const std::string& s) {
    char* o = (char*)malloc(s.size() + 1);
    memcpy(o, s.data(), s.size());
    o[s.size()] = 0;
    return o;
}

static void set_err(char* err, size_t errlen, const char* msg) {
    if (err && errlen) {
        strncpy(err, msg, errlen - 1);
        err[errlen - 1] = 0;
    }
}

// The statistics of a matrix: out = lambda, K, H, alpha, beta, source.
int rmbo_stats(const char* matrix_name, const char* matrix_text, int32_t go, int32_t ge, const double cli[4],
               double out[6], char* err, size_t errlen) {
    try {
        Matrix m = parse_matrix(matrix_text, matrix_name);
        const double zero[4] = {0, 0, 0, 0};
        KaStats s = resolve_stats(matrix_name, go, ge, cli ? cli : zero, m);
        out[0] = s.lambda; out[1] = s.k; out[2] = s.h; out[3] = s.alpha; out[4] = s.beta; out[5] = s.source;
        return 0;
    } catch (const std::exception& e) {
        set_err(err, errlen, e.what());
        return 1;
    }
}

int32_t rmbo_length_adjustment(double k, double log_k, double alpha_d_lambda, double beta, int32_t qlen,
                               int64_t db_len, int32_t db_num, int32_t* converged) {
    bool c = false;
    const int32_t la = length_adjustment(k, log_k, alpha_d_lambda, beta, qlen, db_len, db_num, &c);
    if (converged) *converged = c ? 1 : 0;
    return la;
}

// E-value and bit score of a raw score with stats ka = lambda, K, H, alpha, beta
void rmbo_evalue(const double ka[5], int32_t score, int32_t qlen, int64_t db_len, int32_t db_num, double out[3]) {
    KaStats s;
    s.lambda = ka[0]; s.k = ka[1]; s.log_k = ka[1] > 0 ? std::log(ka[1]) : -1.0; s.h = ka[2];
    s.alpha = ka[3]; s.beta = ka[4];
    const int64_t sp = effective_search_space(s, qlen, db_len, db_num);
    out[0] = evalue_of(score, s, sp);
    out[1] = bitscore_of(score, s);
    out[2] = (double)sp;
}

// Full search of every query against every subject; writes the outfmt-6 text.
// counters (may be NULL) receives 9 values: word_hits seeds ungapped prelim_dp prelims tb_dp
// finals so_cells tb_cells.  Returns 0 on success.
int rmbo_search_text(const char* query_fasta, const char* db_fasta, const char* matrix_text,
                     const char* matrix_name, const rmbo_params* cp, const char* outfmt, int threads,
                     char** out_text, uint64_t* counters, double* seconds, char* err, size_t errlen) {
    try {
        Matrix m = parse_matrix(matrix_text, matrix_name);
        Params p = to_params(cp, matrix_name);
        std::vector<Subject> db;
        for (auto& r : read_fasta_text(db_fasta)) db.push_back(make_subject(r.id, r.seq));
        auto qs = read_fasta_text(query_fasta);
        std::istringstream fs(outfmt);
        std::string t;
        std::vector<std::string> fields;
        fs >> t;
        while (fs >> t) fields.push_back(t);
        Counters ctr;
        std::string out;
        auto t0 = std::chrono::steady_clock::now();
        for (auto& q : qs) {
            auto res = search_query(q.seq, q.id, db, p, m, threads, &ctr);
            for (auto& r : res) {
                out += format_tabular(r, fields);
                out.push_back('\n');
            }
        }
        if (seconds) *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (counters) {
            uint64_t v[9] = {ctr.word_hits, ctr.seeds, ctr.ungapped, ctr.prelim_dp, ctr.prelims,
                             ctr.tb_dp,     ctr.finals, ctr.so_cells, ctr.tb_cells};
            memcpy(counters, v, sizeof v);
        }
        *out_text = dup_string(out);
        return 0;
    } catch (const std::exception& e) {
        set_err(err, errlen, e.what());
        return 1;
    }
}

// Stage taps of the reference's library regression tests (rmblast-lib/tests/*_regression.rs):
// the query FASTA's first record is split into NCBI query chunks (1 Mb, overlap 100) and each
// chunk is searched against every database record.  stage 0 = post-dedup seeds
// ("SEED strand=+ q=.. s=..", sorted as text), stage 1 = sorted ungapped hits
// ("UNGAP strand=.. qs=.. qe=.. ss=.. se=.. score=..", in pipeline order).
int rmbo_stage_file(const char* query_path, const char* db_path, const char* matrix_path, const rmbo_params* cp,
                    int stage, char** out_text, char* err, size_t errlen) {
    try {
        Matrix m = load_matrix(matrix_path);
        Params p = to_params(cp, matrix_path);
        std::string dbp = db_path;
        std::vector<Subject> db;
        if (dbp.size() > 5 && dbp.substr(dbp.size() - 5) == ".2bit") db = read_twobit(dbp);
        else
            for (auto& r : read_fasta(dbp)) db.push_back(make_subject(r.id, r.seq));
        auto qs = read_fasta(query_path);
        const FastaRecord& q = qs.at(0);
        size_t qlen = q.seq.size() - 2;
        // rmblast-lib/tests/ungapped_regression.rs:29-50 compute_chunks
        size_t nch = qlen / (1000000 - 100);
        size_t cs = qlen, eff = 1;
        if (nch > 1) {
            cs = (qlen + (nch - 1) * 100) / nch;
            if (nch < (cs > 100 ? cs - 100 : 0)) ++cs;
            eff = nch;
        }
        size_t step = cs > 100 ? cs - 100 : 0;
        std::vector<std::string> lines;
        char buf[160];
        for (size_t k = 0; k < eff; ++k) {
            size_t st = k * step;
            if (st >= qlen) break;
            size_t en = std::min(st + cs, qlen);
            if (en - st < (size_t)p.word_size) continue;
            std::vector<uint8_t> chunk;
            chunk.push_back(q.seq.front());
            chunk.insert(chunk.end(), q.seq.begin() + 1 + st, q.seq.begin() + 1 + en);
            chunk.push_back(q.seq.back());
            QueryLookup ql = build_query_lookup(chunk, p);
            for (auto& s : db) {
                std::vector<SeedRecord> seeds;
                std::vector<UngappedHit> ung;
                Taps taps;
                if (stage == 0) taps.seeds = &seeds;
                else taps.ungapped = &ung;
                search_pair(ql, chunk, q.id, s, p, m, taps);
                for (auto& x : seeds) {
                    snprintf(buf, sizeof buf, "SEED strand=%c q=%u s=%u", x.strand == PLUS ? '+' : '-', x.q_off, x.s_off);
                    lines.push_back(buf);
                }
                for (auto& h : ung) {
                    snprintf(buf, sizeof buf, "UNGAP strand=%c qs=%u qe=%u ss=%u se=%u score=%d",
                             h.strand == PLUS ? '+' : '-', h.q_start, h.q_end, h.s_start, h.s_end, h.score);
                    lines.push_back(buf);
                }
            }
        }
        if (stage == 0) std::sort(lines.begin(), lines.end());
        std::string out;
        for (auto& l : lines) { out += l; out.push_back('\n'); }
        *out_text = dup_string(out);
        return 0;
    } catch (const std::exception& e) {
        set_err(err, errlen, e.what());
        return 1;
    }
}

void rmbo_free(char* p) { free(p); }

}  // extern "C"

extern "C" {
// Stage taps per (query, subject) pair in pair order, as uint32 records: stage 0 seeds
// (strand, q, s), 1 sorted ungapped hits (strand, qs, qe, ss, se, score), 2 prelims after the
// prelim purge (strand, qs, qe, ss, se, score, q_seed, s_seed).
int rmbo_stage_text(const char* query_fasta, const char* db_fasta, const char* matrix_text, const char* matrix_name,
                    const rmbo_params* cp, int stage, uint32_t** out, uint64_t* n_out, char* err, size_t errlen) {
    try {
        Matrix m = parse_matrix(matrix_text, matrix_name);
        Params p = to_params(cp, matrix_name);
        std::vector<Subject> db;
        for (auto& r : read_fasta_text(db_fasta)) db.push_back(make_subject(r.id, r.seq));
        auto qs = read_fasta_text(query_fasta);
        uint64_t total = 0;
        for (auto& s : db) total += s.len();
        std::vector<uint32_t> rec;
        for (auto& q : qs) {
            Params pq = p;
            pq.ungapped_cutoff = ungapped_cutoff(p.matrix_name, p.gap_open, p.gap_extend, p.min_raw_gapped_score,
                                                 q.seq.size() - 2, db.empty() ? 0 : total / db.size());
            QueryLookup ql = build_query_lookup(q.seq, pq);
            for (auto& s : db) {
                if (stage == 4) {
                    auto v = pair_tracebacks(ql, q.seq, s, pq, m);
                    rec.insert(rec.end(), v.begin(), v.end());
                    continue;
                }
                std::vector<SeedRecord> seeds;
                std::vector<UngappedHit> ung;
                std::vector<PrelimHsp> pre;
                Taps t;
                if (stage == 0) t.seeds = &seeds;
                else if (stage == 1) t.ungapped = &ung;
                else t.prelims = &pre;
                search_pair(ql, q.seq, q.id, s, pq, m, t);
                for (auto& x : seeds) rec.insert(rec.end(), {(uint32_t)x.strand, x.q_off, x.s_off});
                for (auto& h : ung)
                    rec.insert(rec.end(), {(uint32_t)h.strand, h.q_start, h.q_end, h.s_start, h.s_end, (uint32_t)h.score});
                for (auto& h : pre)
                    rec.insert(rec.end(), {(uint32_t)h.strand, h.q_start, h.q_end, h.s_start, h.s_end, (uint32_t)h.score,
                                           h.q_seed, h.s_seed});
            }
        }
        uint32_t* o = (uint32_t*)malloc(std::max<size_t>(rec.size(), 1) * 4);
        if (!rec.empty()) memcpy(o, rec.data(), rec.size() * 4);
        *out = o;
        *n_out = rec.size() / (stage == 0 ? 3 : stage == 1 ? 6 : stage == 2 ? 8 : 9);
        return 0;
    } catch (const std::exception& e) {
        set_err(err, errlen, e.what());
        return 1;
    }
}
}
