// rmb_oracle.hpp -- CPU restatement of the rmblastn search core (TEST INFRASTRUCTURE).
//
// This is the parity oracle.  Only the tests, the smoke check and the CPU-baseline leg of
// bench.py may link or run it, and only as the checker.  The product (rmblast_b200/) never
// links it.  Every function cites the reference file:line it restates; paths are relative
// to the Dfam-consortium/RMBlast source tree (Rust port 3.1.0 of NCBI rmblastn 2.17.1).
//
// Parity status: pinned against the reference's NCBI-2.17.1 golden outputs
// (rmblastn/tests/data/expected_*.tsv) and its chr22 stage goldens, see tests/.
#pragma once
#include <cstdint>
#include <map>
#include <string>
#include <vector>
#include <utility>

namespace rmbo {

// ---- encoding (rmblast-lib/src/encoding.rs) ---------------------------------------------
constexpr uint8_t SENTINEL = 15;
extern const uint8_t BLASTNA_TO_IUPAC[17];
extern const uint8_t COMPLEMENT[16];
uint8_t iupac_to_blastna(uint8_t c);
std::vector<uint8_t> encode_iupac(const std::string& ascii);     // encoding.rs:125
std::vector<uint8_t> revcomp(const uint8_t* s, size_t n);        // encoding.rs:136

// ---- NCBI CRandom (rmblast-lib/src/seq/twobit.rs:50-135) --------------------------------
struct NcbiRandom {
    uint32_t state[33];
    int rj, rk;
    explicit NcbiRandom(uint32_t seed);
    uint32_t raw();
    uint32_t get_rand() { return raw() >> 1; }
    uint8_t next_base_iupac(uint8_t code);
};

// ---- records -----------------------------------------------------------------------------
struct FastaRecord { std::string id, defline; std::vector<uint8_t> seq; };  // seq sentinel-wrapped
std::vector<FastaRecord> read_fasta(const std::string& path);             // seq/fasta.rs:83
std::vector<FastaRecord> read_fasta_text(const std::string& text);

struct Subject {
    std::string id;
    std::vector<uint8_t> plus;      // sentinel-wrapped, ambiguity codes CRandom-resolved
    std::vector<uint8_t> n_mask;    // empty, or original codes (4..14) at ambiguous positions
    std::vector<uint8_t> rc;        // revcomp(plus)
    std::vector<uint8_t> packed;    // 3 pad + ceil(len/4) + 3 pad, NCBI2NA, MSB first
    std::vector<uint8_t> align;     // plus with n_mask codes restored
    std::vector<uint8_t> align_rc;  // revcomp(align)
    std::vector<uint8_t> n_mask_rc; // reversed + complemented n_mask
    uint32_t len() const { return (uint32_t)(plus.size() - 2); }
};
// seq/fasta_db.rs:86-131 + seq/mod.rs:56-100
Subject make_subject(const std::string& id, const std::vector<uint8_t>& raw_blastna);
// Subject built from an already-resolved sequence plus its n_mask (2bit decode path).
Subject make_subject_resolved(const std::string& id, std::vector<uint8_t> plus,
                              std::vector<uint8_t> n_mask);
std::vector<uint8_t> pack_ncbi2na(const uint8_t* bases, size_t len);   // blast/util.rs:85

// UCSC .2bit database (seq/twobit.rs), decoded with N blocks CRandom-resolved.
std::vector<Subject> read_twobit(const std::string& path);

// ---- matrix (rmblast-lib/src/matrix.rs) -------------------------------------------------
struct Matrix {
    int32_t s[16][16];
    double freqs[16];
    double lambda = 0.0;
    std::string name;
    bool has_karlin = false;          // a "# KARLIN" comment line (matrix.rs:38-70, 100-103)
    double karlin[5] = {0, 0, 0, 0, 0};  // lambda, K, H, alpha, beta
};
Matrix parse_matrix(const std::string& text, const std::string& name);  // matrix.rs:76
Matrix load_matrix(const std::string& path);

// ---- parameters (rmblast-lib/src/options.rs) --------------------------------------------
struct Params {
    int gap_open = 4, gap_extend = 4;
    std::string matrix_name;
    int word_size = 8;
    int xdrop_ungap = 20, xdrop_gap = 30, xdrop_gap_final = 100;
    int min_raw_gapped_score = 0;
    int ungapped_cutoff = -1;  // -1 = unset (cutoff_score_max)
    bool complexity_adjust = false;
    bool dust = true;
    uint32_t mask_level = 101;
    double evalue = 0.0;                  // --evalue reap threshold; 0 = off
    double cli_stats[4] = {0, 0, 0, 0};   // -matrix_lambda, -matrix_k, -matrix_alpha, -matrix_beta
    int gapped_cutoff() const { return min_raw_gapped_score > 1 ? min_raw_gapped_score : 1; }
    int cutoff_score_max() const { return min_raw_gapped_score > 0 ? min_raw_gapped_score / 2 : 1; }
};
// search/ka_cutoff.rs:126
int ungapped_cutoff(const std::string& matrix_name, int gap_open, int gap_extend,
                    int min_raw, uint64_t query_length, uint64_t avg_subj_length);

// ---- DUST (rmblast-lib/src/filter/dust.rs) ----------------------------------------------
std::vector<std::pair<size_t, size_t>> dust_mask(std::vector<uint8_t>& seq);  // dust.rs:462

// ---- hits --------------------------------------------------------------------------------
enum Strand : uint8_t { PLUS = 0, MINUS = 1 };
enum EditOp : uint8_t { SUB = 0, GAP_IN_QUERY = 1, GAP_IN_SUBJECT = 2 };
struct Op { EditOp op; uint32_t n; };
using Script = std::vector<Op>;
void script_push(Script& s, EditOp op, uint32_t n);

struct AlignStats {
    uint32_t matches = 0, mismatches = 0, query_gaps = 0, subject_gaps = 0;
    uint32_t transitions = 0, transversions = 0, cpg_sites = 0;
    double kdiv = 0, cpg_kdiv = 0;
    float perc_sub = 0, perc_query_gap = 0, perc_db_gap = 0;
};

struct Hsp {
    int32_t score = 0;
    uint32_t q_start = 0, q_end = 0, q_len = 0, s_start = 0, s_end = 0, s_len = 0;
    Strand strand = PLUS;
    Script script;
    std::vector<uint8_t> q_seq, s_seq;
};
struct AlignResult {
    Hsp hsp;
    std::string query_id, subject_id;
    uint32_t oid = 0;
    AlignStats stats;
    double evalue = 1.0, bitscore = 0.0;  // the no-statistics rendering until set
};

// ---- lookup table (blast/nalookup.rs, blast/mblookup.rs) --------------------------------
int choose_lut_width(int word_size, size_t approx_entries);  // nalookup.rs:254
struct OffsetPair { uint32_t q_off, s_off; };
struct Lookup {
    bool mega = false;
    int lut_word_length = 0, word_length = 0, scan_step = 0;
    int longest_chain = 0;
    // small table
    int32_t mask = 0;
    std::vector<int32_t> num_used, cell_entries, cell_cursor, overflow;  // cell_entries: 3/cell
    std::vector<uint32_t> pv;
    // megablast table
    int64_t hashsize = 0;
    std::vector<int32_t> hashtable, next_pos;
    uint32_t pv_bts = 5;
    int scan(const uint8_t* packed, OffsetPair* out, int max_hits, int32_t range[2]) const;
};
struct QueryLookup {
    Lookup lut;
    uint32_t fwd_n = 0, c1_start = 0;
    std::vector<uint8_t> masked;   // DUST-masked query (== query when dust off)
    std::vector<uint8_t> query_rc; // revcomp(query)
};
QueryLookup build_query_lookup(const std::vector<uint8_t>& query, const Params& p);

// ---- stage records and taps (search/engine.rs) ------------------------------------------
struct SeedRecord { uint32_t q_off, s_off; Strand strand; };
struct UngappedHit { uint32_t q_start, q_end, s_start, s_end; int32_t score; Strand strand; };
struct PrelimHsp {
    uint32_t q_seed, s_seed, q_start, q_end, s_start, s_end;
    int32_t score;
    Strand strand;
};
struct Counters {
    uint64_t word_hits = 0, seeds = 0, ungapped = 0, prelim_dp = 0, prelims = 0,
             tb_dp = 0, finals = 0, so_cells = 0, tb_cells = 0;
};
struct Taps {
    std::vector<SeedRecord>* seeds = nullptr;
    std::vector<UngappedHit>* ungapped = nullptr;  // sorted, FWD-normalised
    std::vector<PrelimHsp>* prelims = nullptr;     // after the prelim endpoint purge
    Counters* counters = nullptr;
};

// engine.rs:715 search_with_query_lookup (single pair)
std::vector<AlignResult> search_pair(const QueryLookup& ql, const std::vector<uint8_t>& query,
                                     const std::string& query_id, const Subject& subj,
                                     const Params& p, const Matrix& m, const Taps& taps);

// main.rs:1133-1236 single-chunk search_db_parallel + engine.rs:998 ordering.
std::vector<AlignResult> search_query(const std::vector<uint8_t>& query, const std::string& query_id,
                                      const std::vector<Subject>& db, const Params& p,
                                      const Matrix& m, int threads, Counters* counters);

// Traceback stage tap: every post-purge prelim of one pair, unfiltered (see the engine).
std::vector<uint32_t> pair_tracebacks(const QueryLookup& ql, const std::vector<uint8_t>& query, const Subject& subj,
                                      const Params& p, const Matrix& m);

// engine.rs:863 (cross-subject mode, oid = subject index)
void apply_mask_level(std::vector<AlignResult>& r, uint32_t mask_level);
// engine.rs:998
void sort_hit_list_order(std::vector<AlignResult>& r);

// ---- alignment kernels (search/ungapped.rs, search/gapped.rs) ---------------------------
struct UngappedResult { int32_t score; uint32_t q_start, q_end, s_start, s_end; };
UngappedResult extend_ungapped(const uint8_t* query, size_t qlen_with_sent, const uint8_t* subject,
                               size_t slen_with_sent, uint32_t q_off, uint32_t s_off,
                               const Matrix& m, int xdrop);
struct ScoreOnly { int32_t score; uint32_t a_len, b_len; uint64_t cells; };
ScoreOnly align_ex_score_only(const uint8_t* a, const uint8_t* b, size_t m, size_t n, int go, int ge,
                              int xdrop, const Matrix& mat, bool reverse);
struct GapAlign { int32_t score; uint32_t a_len, b_len; Script script; uint64_t cells; };
GapAlign align_ex(const uint8_t* a, const uint8_t* b, size_t m, size_t n, int go, int ge, int xdrop,
                  const Matrix& mat, bool reverse);

// ---- stats and output (stats.rs, output.rs) ---------------------------------------------
AlignStats compute_align_stats(const std::vector<uint8_t>& q_iupac, const std::vector<uint8_t>& s_iupac);
std::vector<uint8_t> to_iupac(const std::vector<uint8_t>& aligned);
std::string format_tabular(const AlignResult& r, const std::vector<std::string>& fields);
// pairwise output (outfmt 0, output.rs:369-720); query_mask: the query's DUST intervals
std::string pairwise_program_header(const std::string& db_name, size_t n_seqs, uint64_t total);
std::string pairwise_results(const std::vector<AlignResult>& res, const std::string& query_defline, uint32_t qlen,
                             const std::map<std::string, std::string>* subject_deflines,
                             const std::vector<std::pair<size_t, size_t>>& query_mask);
std::string pairwise_footer(const std::string& db_name, size_t n_seqs, uint64_t total, int go, int ge);

// ---- E-value statistics (rmb_oracle_stats.cpp) -----------------------------------------
struct KaStats {  // gapped Karlin block + the length adjustment's alpha/beta; lambda <= 0: none
    double lambda = -1.0, k = -1.0, log_k = -1.0, h = -1.0, alpha = 0.0, beta = 0.0;
    int source = 0;  // 0 none, 1 table, 2 command line, 3 matrix comment
};
KaStats resolve_stats(const std::string& matrix_name, int go, int ge, const double cli[4], const Matrix& m);
int32_t length_adjustment(double k, double log_k, double alpha_d_lambda, double beta, int32_t query_length,
                          int64_t db_length, int32_t db_num_seqs, bool* converged);
int64_t effective_search_space(const KaStats& s, int32_t query_length, int64_t db_length, int32_t db_num_seqs);
double evalue_of(int32_t score, const KaStats& s, int64_t searchsp);
double bitscore_of(int32_t score, const KaStats& s);
std::string format_evalue(double e);
std::string format_bitscore(double b);

}  // namespace rmbo
