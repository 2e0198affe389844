// rmb_glue.hpp -- host steps of the search core that are order-dependent per (query, subject)
// pair and cost O(HSPs), not O(cells): the interval-tree filters, the endpoint purges, the
// cut/re-evaluation of common-endpoint HSPs, complexity adjustment, alignment statistics,
// masklevel and the output order.  The DP and scan work they consume comes from the GPU.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace rmb {

enum : uint8_t { OP_SUB = 0, OP_GAP_Q = 1, OP_GAP_S = 2 };  // hits.rs:21-31 EditOp
struct RunOp { uint8_t op; uint32_t n; };
using Script = std::vector<RunOp>;

struct Stats {
    uint32_t matches = 0, mismatches = 0, query_gaps = 0, subject_gaps = 0;
    uint32_t transitions = 0, transversions = 0, cpg_sites = 0;
    double kdiv = 0, cpg_kdiv = 0;
    float perc_sub = 0, perc_query_gap = 0, perc_db_gap = 0;
};

struct Hit {  // output.rs:132 AlignResult
    int32_t score = 0;
    uint32_t q_start = 0, q_end = 0, q_len = 0, s_start = 0, s_end = 0, s_len = 0;
    uint32_t oid = 0;
    uint8_t strand = 0;  // 0 plus, 1 minus
    Script script;
    std::vector<uint8_t> q_seq, s_seq;
    Stats stats;
    double evalue = 1.0, bitscore = 0.0;  // the statistics sentinel until set
};

// The host views of one subject the glue reads (sentinel-wrapped BLASTNA).
struct SubjectView {
    const uint8_t* align;     // IUB-restored plus strand
    const uint8_t* align_rc;  // its reverse complement
    const uint8_t* n_mask;    // nullptr or len bytes
    const uint8_t* n_mask_rc; // nullptr or len bytes
    uint32_t len;
};

struct GlueParams {
    int32_t gap_open, gap_extend, gapped_cutoff;
    bool complexity_adjust;
    int32_t matrix[16][16];
    double freqs[16];
    double lambda;
};

// An ungapped record that passed the GPU prelim DP with a score >= the gapped cutoff.
struct UngSurvivor {
    uint32_t q_seed, s_seed, q_start, q_end, s_start, s_end;  // record frame
    int32_t score;
    uint8_t strand;
    // prelim DP result (record frame) and traceback seed
    int32_t p_score;
    uint32_t p_qs, p_qe, p_ss, p_se, tb_q, tb_s;
};
struct Prelim {  // engine.rs:158-169 PrelimHsp
    uint32_t q_seed, s_seed, q_start, q_end, s_start, s_end;
    int32_t score;
    uint8_t strand;
};

// engine.rs:1280-1411 + 1969-2083: sort, contain-filter and purge one pair's survivors.
std::vector<Prelim> phase2a_filter(std::vector<UngSurvivor>& surv, uint32_t qa, uint32_t sa);

// A traceback result from the GPU for one prelim (DP frame: query_rc for minus).
struct TbResult {
    int32_t status;
    int32_t score;
    uint32_t q0, q1, s0, s1;
    Script script;
};

// engine.rs:1438-1762 on one pair: prelims (post purge, pipeline order) with their GPU
// traceback results; returns the pair's final HSPs.
std::vector<Hit> phase2b_filter(std::vector<Prelim>& prelims, std::vector<TbResult>& tbs, const uint8_t* query,
                                const uint8_t* query_rc, uint32_t qa, const SubjectView& sv, uint32_t oid,
                                const GlueParams& gp);

// The stable order phase2b_filter processes prelims in (engine.rs:1471-1485); the caller
// sorts before launching tracebacks so both sides agree.
void sort_prelims_for_traceback(std::vector<Prelim>& p, uint32_t qa, uint32_t sa);

// engine.rs:863-974 (cross-subject mode) and main.rs:1230-1234 + engine.rs:998-1017.
void apply_mask_level(std::vector<Hit>& hits, uint32_t mask_level);
void sort_hit_list_order(std::vector<Hit>& hits, const std::vector<std::string>& subject_ids);

// output.rs:294-367 one tabular line (no newline); returns false on an unknown field.
bool format_line(std::string& out, const Hit& h, const std::string& qid, const std::string& sid,
                 const std::vector<std::string>& fields);

int choose_lut_width(int word_size, uint64_t approx_entries);

// Gapped Karlin-Altschul block (lambda <= 0: no statistics) with the alpha/beta of the length
// adjustment.
struct KaBlock {
    double lambda = -1.0, k = -1.0, log_k = -1.0, h = -1.0, alpha = 0.0, beta = 0.0;
};
enum { KA_NONE = 0, KA_TABLE = 1, KA_CLI = 2, KA_MATRIX_COMMENT = 3 };
// ka_stats.rs:153-300 default mode without the ALP fit: the built-in table (base name, exact
// gap costs), then cli = {lambda, K, alpha, beta} (used when lambda, K, alpha > 0), then a
// "# KARLIN" comment {lambda, K, H, alpha, beta} (or null), else none.  Returns the source.
int ka_resolve(const std::string& matrix_name, int go, int ge, const double cli[4], const double* karlin,
               KaBlock& out);
// eff_lengths.rs: the effective search space of one query against the database.
int64_t eff_searchsp(const KaBlock& kb, int32_t qlen, int64_t db_len, int32_t db_num);
double hsp_evalue(int32_t score, const KaBlock& kb, int64_t searchsp);
double hsp_bitscore(int32_t score, const KaBlock& kb);
void append_evalue(std::string& out, double e);
// pairwise output (outfmt 0): the program header, one query's block (hits in output order;
// subject_deflines indexed by oid, or null for id-only databases; qmask: one bit per query
// position inside a DUST interval, or null), and the footer (mtime < 0: no "Posted date")
std::string pairwise_header(const std::string& db_name, uint64_t n_seqs, uint64_t letters);
void pairwise_query(std::string& out, const std::vector<Hit>& hits, const std::string& defline, uint32_t qlen,
                    const std::vector<std::string>& subject_ids, const char* const* subject_deflines,
                    const uint32_t* qmask);
std::string pairwise_footer(const std::string& db_name, uint64_t n_seqs, uint64_t letters, int64_t mtime, int go,
                            int ge);
void append_bitscore(std::string& out, double b);
int ungapped_cutoff_for(const std::string& matrix_name, int go, int ge, int min_raw, uint64_t qlen, uint64_t avg);
Stats align_stats(const std::vector<uint8_t>& q, const std::vector<uint8_t>& s);

}  // namespace rmb
