/* rmb_gpu.h -- C ABI of the B200 rmblastn search core (librmb_b200.so).
 *
 * The library replaces the search body that the reference runs per query under
 * `--mt-mode` (rmblastn/src/main.rs:739-915 -> search_db_parallel, main.rs:1133-1236):
 * lookup table, subject scan, exact word extension, diagonal dedup, ungapped X-drop,
 * preliminary score-only gapped X-drop DP, interval-tree filters, traceback DP,
 * complexity adjustment, endpoint purges, masklevel and the final hit order.
 * Every DP, the scan and the extensions run as sm_100a kernels; there is no CPU path
 * for them.  Plain pointers and sizes only; every call returns 0 on success or a
 * nonzero status with a message in `err` (the alp_shim pattern of
 * rmblast-stats/rmstats/csrc/alp_shim.cpp:44-110).  No C++ exception crosses the ABI.
 * One context per host thread; calls on one context are not reentrant.
 */
#ifndef RMB_GPU_H
#define RMB_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RMB_OK 0
#define RMB_EINVAL 1   /* bad argument */
#define RMB_ECUDA 2    /* CUDA error (message carries cudaGetErrorString) */
#define RMB_ENOMEM 3   /* device or host allocation failed */
#define RMB_ESTATE 4   /* call out of order (e.g. search before rmb_db_load) */
#define RMB_ELIMIT 5   /* input beyond a documented limit */

/* Search options: rmblast-lib/src/options.rs:12-67 SearchParams.  mask_level < 0 or
 * >= 100 disables masklevel (main.rs:560).  ungapped_cutoff < 0 derives it as the
 * reference does per query (search/ka_cutoff.rs:126).  dust = 1 masks low-complexity
 * query intervals with NCBI symmetric DUST (window 64, level 20, linker 1; filter/dust.rs)
 * before the lookup tables and the exact word extension, as the reference does
 * (engine.rs:606-616); the masked copy is made on the device on the first search of a
 * query set. */
typedef struct rmb_params {
    int32_t gap_open, gap_extend, word_size;
    int32_t xdrop_ungap, xdrop_gap, xdrop_gap_final;
    int32_t min_raw_gapped_score;
    int32_t complexity_adjust, dust, mask_level;
    int32_t ungapped_cutoff;
    int32_t device;       /* CUDA device ordinal */
    int32_t schedule;     /* 0 = FIFO record queue; 1 = learned, front-loaded: the records the
                             network (rmb_sched_set_model) predicts costliest, about 1/32 of them,
                             go first and the rest keep their arrival order (reversed); 2 = learned,
                             every record in descending predicted cost */
    int32_t kernels;      /* 0 = automatic; 1 = run every preliminary DP on the warp-cooperative
                             kernel (the thread-per-extension kernel's fallback), for testing */
    int32_t pipeline;     /* 0 = batched: the ungapped extension and the preliminary DP run as
                             persistent kernels fed by device work queues, the traceback takes
                             the largest alignments first; 1 = plain: one launch per stage with
                             one work item per thread (per warp for the traceback) in arrival
                             order, no queues.  Same results either way; schedule = 1 needs 0. */
    /* Gapped Karlin-Altschul statistics for E-values and bit scores, as rmb_ka_resolve returns
     * them: lambda, K, H, and the alpha/beta of the length adjustment.  ka_lambda <= 0: none
     * (every E-value 1.0 and bit score 0.0, the reference's rendering without statistics). */
    double ka_lambda, ka_k, ka_h, ka_alpha, ka_beta;
    /* --evalue (main.rs:1224-1226, NCBI Blast_HSPListReapByEvalue): HSPs whose E-value is above
     * this are dropped before masklevel; 0 = off; no effect without statistics. */
    double evalue;
} rmb_params;

typedef struct rmb_ctx rmb_ctx;

/* Launch knobs of the batched pipeline (no counterpart in the reference; none changes a result,
 * only how work is laid out on the GPU).  rmb_ctx_create starts from the hand-swept defaults;
 * rmb_autotune times candidates on sample queries and keeps the fastest; rmb_tune_get/set read
 * and write them (a caller can persist and reuse a tuned set).
 *   prelim_group            cell steps a lane of the thread-per-extension DP runs between its
 *                           row-end blocks: 4, 8 or 16
 *   prelim_blocks_per_sm    resident blocks per SM of that DP's persistent grid, 1..6
 *   prelim_window           widest band, in cells, one thread keeps, 16..60: a wider extension is
 *                           handed to a warp (32 threads per alignment)
 *   prelim_budget_div       DP cells one thread spends on a record before a warp takes it:
 *                           records / div, within 8,192 .. 2^20; 16..4096
 *   ungapped_blocks_per_sm  blocks per SM of the persistent ungapped-extension grid, 1..8
 *   dedup_extend_hits_per_pair  pair ranges averaging at least this many word hits per
 *                           (query, subject) pair take the dedup kernel that extends only the
 *                           hits the diagonal hash admits; 0 = always, < 0 = never
 *   lanes                   1 or 2 pipeline lanes: with 2, a search's queries go in about four
 *                           sub-batches to two streams with their own buffers and host threads,
 *                           so one lane's host steps overlap the other's kernels (twice the
 *                           per-batch device memory)
 *   graph                   1: each pair range's device chain from the dedup to the prelim
 *                           survivors runs as one CUDA graph, its counts kept on the device;
 *                           0: stage by stage, the host reading each count; 2: the graph with
 *                           room for one warp-kernel record and one survivor, so that every range
 *                           also runs the stage-by-stage finish past those capacities (a test
 *                           setting) */
typedef struct rmb_tune {
    int32_t prelim_group, prelim_blocks_per_sm, prelim_window, prelim_budget_div;
    int32_t ungapped_blocks_per_sm, dedup_extend_hits_per_pair, lanes, graph;
} rmb_tune;

/* Learned schedule of the preliminary DP (no counterpart in the reference, whose records run in
 * a fixed order; the order changes no result).  A 12 -> 64 -> 64 -> 1 ReLU network with BF16
 * weights predicts each ungapped record's DP cells (log1p), and with params.schedule = 1 or 2 the
 * records leave the DP queue with the long extensions first (schedule 1 moves only the predicted
 * costliest ~1/32 to the front, so the others keep the neighbours they share sequences with;
 * schedule 2 orders all of them by predicted cost).
 * Parameters: RMB_SCHED_NPARAM floats, W1[12][64] (W1[k*64+n]), b1[64], W2[64][64], b2[64],
 * w3[64], b3, then the features' mean[12] and 1/std[12].  Features of a record: ungapped score /
 * 100, log1p ungapped extent, log1p of the room left and right of the pivot on query and
 * subject, X / 100, strand, GC of ~32 subject bases at the pivot, score per base, log1p of the
 * pair's word hits, log1p of the diagonal room.
 *
 * rmb_sched_set_model: the network for this context's searches with schedule 1 or 2 (such a search
 * with no model fails with RMB_ESTATE).
 * rmb_sched_log: one FIFO search of the queries, returning for every record the thread kernel
 * completed its raw features (n x 12, malloc'd) and DP cells (n, malloc'd); free both with
 * rmb_text_free.  Training pairs for rmb_sched_train.
 * rmb_sched_train: Adam on the GPU (hand-written kernels, FP32 with BF16-rounded weights; the
 * rate lr falls linearly to lr / 10 over the run) from
 * params_io (initial weights and the normalisation) over (features, targets = log1p cells);
 * params_io gets the trained BF16-rounded weights; stats_out[epochs + 1]: each epoch's training
 * mean squared error, then the held-out RMSE (log-cells) on val_fraction of the rows.
 * rmb_sched_grad: mean squared error and its gradient (RMB_SCHED_NET floats, in the parameter
 * layout) on n rows, by the training kernels.
 * rmb_sched_predict: the inference kernel (BF16 mma, FP32 accumulation) on n rows of raw features. */
#define RMB_SCHED_NET 5057
#define RMB_SCHED_NPARAM 5081
int rmb_sched_set_model(rmb_ctx* ctx, const float* params, uint32_t n_params, char* err, size_t errlen);
int rmb_sched_log(rmb_ctx* ctx, uint32_t n_queries, const uint8_t* const* query, const uint32_t* qlen,
                  float** features, uint32_t** cells, uint64_t* n_records, char* err, size_t errlen);
int rmb_sched_train(int32_t device, const float* features, const float* targets, uint64_t n, uint32_t epochs,
                    uint32_t batch, float lr, uint64_t seed, float val_fraction, float* params_io, float* stats_out,
                    char* err, size_t errlen);
int rmb_sched_grad(int32_t device, const float* params, const float* features, const float* targets, uint32_t n,
                   float* grad_out, float* loss_out, char* err, size_t errlen);
int rmb_sched_predict(int32_t device, const float* params, const float* features, uint64_t n, float* pred_out,
                      char* err, size_t errlen);

/* rmblast-lib/src/matrix.rs:62-214 ScoreMatrix: scores[q][s] in BLASTNA order
 * (A C G T R Y M K W S B D H V N GAP), 16x16 row-major; freqs in BLASTNA order; lambda as
 * the reference estimates it (matrix.rs:290).  matrix_name is the path or file name the
 * user gave (used only for the Karlin-Altschul ungapped-cutoff table lookup). */
int rmb_ctx_create(const rmb_params* params, const int32_t scores[256], const double freqs[16],
                   double lambda, const char* matrix_name, rmb_ctx** out, char* err, size_t errlen);

/* rmblast-lib/src/seq/mod.rs:155-291 SubjectDb::open + get_prepared: the library, one call.
 * plus[i]: sentinel-wrapped BLASTNA (len[i] + 2 bytes) with ambiguity codes already resolved
 * by NCBI CRandom (seq/fasta_db.rs:86-107); n_mask[i]: NULL or len[i] bytes holding the
 * original code (4..14) at ambiguous positions, 0 elsewhere (fasta_db.rs:115-131);
 * ids[i]: subject id.  The subject's oid is its index i. */
int rmb_db_load(rmb_ctx* ctx, uint32_t n_subjects, const uint8_t* const* plus, const uint32_t* len,
                const uint8_t* const* n_mask, const char* const* ids, char* err, size_t errlen);

/* One reported HSP: rmblast-lib/src/output.rs:132-138 AlignResult (hits.rs:56-79 Hsp,
 * stats.rs:25-44 AlignStats).  Coordinates 0-based half-open, subject on the plus strand. */
typedef struct rmb_hsp {
    int32_t score;
    uint32_t q_start, q_end, q_len, s_start, s_end, s_len;
    uint32_t subject_oid;
    uint32_t strand;  /* 0 plus, 1 minus */
    uint32_t matches, mismatches, query_gaps, subject_gaps, transitions, transversions, cpg_sites;
    float perc_sub, perc_query_gap, perc_db_gap;
    double kdiv, cpg_kdiv;
    uint64_t ops_off;  /* into rmb_results.ops */
    uint32_t ops_len;
    uint32_t aln_len;  /* length of the aligned strings */
    uint64_t seq_off;  /* into rmb_results.q_seq / s_seq (BLASTNA, gap = 15) */
    double evalue, bitscore;  /* Karlin-Altschul E-value and bit score (1.0 / 0.0 without statistics) */
} rmb_hsp;

/* Stage counters of one search call (the reference's diagnostics counters,
 * search/engine.rs:28-37 and search/gapped.rs:25-36). */
typedef struct rmb_counters {
    uint64_t word_hits, seeds, ungapped, prelim_dp, prelims, tb_dp, finals;
    uint64_t so_cells, tb_cells;
    double ms_lookup, ms_scan, ms_ungapped, ms_dedup, ms_prelim_dp, ms_host_2a, ms_traceback, ms_host_2b;
    /* device time of the kernels (CUDA events on the library's stream) and the number of
     * this library's own kernel launches (CUB scans/sorts/selects not counted) */
    double gpu_ms_scan, gpu_ms_ungapped, gpu_ms_dedup, gpu_ms_prelim, gpu_ms_traceback, gpu_ms_lookup;
    uint64_t launches;
    /* the preliminary DP's main kernel alone: its device time and the DP cells of the records
     * it completed (the rest of gpu_ms_prelim / so_cells is its fallbacks and setup) */
    double gpu_ms_prelim_main;
    uint64_t so_cells_main;
    /* DUST masking of the query set (once per uploaded query set, when dust = 1) */
    double gpu_ms_dust;
    /* the learned record order (schedule 1 or 2): features, network and order, a part of
     * gpu_ms_prelim */
    double gpu_ms_sched;
} rmb_counters;

/* Results of rmb_search_batch, in the reference's output order per query
 * (main.rs:1229-1234 then search/engine.rs:998-1017). */
typedef struct rmb_results {
    uint32_t n_queries;
    uint64_t* query_off;  /* n_queries + 1 offsets into hsps */
    uint64_t n_hsps;
    rmb_hsp* hsps;
    uint32_t* ops;        /* edit script: (op << 30) | count; op 0 Sub, 1 GapInQuery, 2 GapInSubject */
    uint8_t* q_seq;
    uint8_t* s_seq;
    rmb_counters counters;
} rmb_results;

/* main.rs:1133-1236 search_db_parallel for n_queries queries: the single-chunk path, and for
 * queries of 1,999,800 bp or more the multi-chunk path (main.rs:1236-1400: 1 Mb chunks with a
 * 100 bp overlap, whole-query DUST, cross-chunk merge, full-query traceback); both in one call.
 * query[i]: sentinel-wrapped BLASTNA (qlen[i] + 2 bytes), not CRandom-resolved (queries keep
 * N).  Stage taps (rmb_debug_stage) take single-chunk queries only.  The batched pipeline runs
 * some host steps on threads of its own beside its kernels and joins them before returning;
 * calls on one context must not overlap. */
int rmb_search_batch(rmb_ctx* ctx, uint32_t n_queries, const uint8_t* const* query, const uint32_t* qlen,
                     rmb_results** out, char* err, size_t errlen);

/* The same search split at the host/device boundary: rmb_queries_upload copies the queries
 * into device memory once (the reference's per-query BLASTNA buffers, main.rs:740-746), and
 * rmb_search_resident runs search_db_parallel on them; rmb_search_batch is upload + search +
 * free.  A query set belongs to the device of the context that uploaded it. */
typedef struct rmb_queries rmb_queries;
int rmb_queries_upload(rmb_ctx* ctx, uint32_t n_queries, const uint8_t* const* query, const uint32_t* qlen,
                       rmb_queries** out, char* err, size_t errlen);
int rmb_search_resident(rmb_ctx* ctx, rmb_queries* queries, rmb_results** out, char* err, size_t errlen);
void rmb_queries_free(rmb_queries* queries);

/* output.rs:223-367 parse_outfmt + write_tabular: "6 <fields>" lines for every HSP, query by
 * query; query_ids[i] names query i.  *text is NUL-terminated; free with rmb_text_free. */
int rmb_format_tabular(const rmb_ctx* ctx, const rmb_results* res, const char* const* query_ids,
                       const char* outfmt, char** text, size_t* text_len, char* err, size_t errlen);

/* Stage taps, as search/engine.rs:796-832 search_with_query_lookup_seeds/_ungapped expose
 * them: stage 0 = post-dedup seeds (strand, q, s per record: 3 uint32), stage 1 = sorted
 * ungapped hits (strand, qs, qe, ss, se, score: 6 uint32), stage 2 = preliminary HSPs after the
 * prelim endpoint purge (strand, qs, qe, ss, se, score, q_seed, s_seed: 8 uint32), for every
 * (query, subject) pair in pair order; stage 3 = the query lookup tables (query, cell, position:
 * 3 uint32 per entry in retrieval order; position 0xffffffff flags a cell whose presence bit
 * disagrees with its entries) -- blast/nalookup.rs:301 / blast/mblookup.rs:190; stage 4 = the
 * traceback of every post-purge prelim in the order engine.rs:1471-1485 visits them, before the
 * Phase 2b containment filter (strand, status 0 = alignment / 1 = none, score, q0, q1, s0, s1 in
 * the DP frame, number of edit runs, FNV-1a of the runs: 9 uint32) -- engine.rs:2953-3039.  *records is malloc'd; free with rmb_text_free. */
int rmb_debug_stage(rmb_ctx* ctx, uint32_t n_queries, const uint8_t* const* query, const uint32_t* qlen,
                    int32_t stage, uint32_t** records, uint64_t* n_records, char* err, size_t errlen);

/* Input preparation the reference does before the search (host side, no GPU needed).
 * rmb_matrix_parse: rmblast-lib/src/matrix.rs:76-324 ScoreMatrix::from_reader (FREQS line,
 * header, rows by position, -32768 for undefined codes, INT32_MIN/2 for the gap row/column,
 * lambda by the reference's bisection).  Same refusals as the reference (bad FREQS, non-square
 * matrix, non-negative expected score).
 * rmb_encode_iupac: encoding.rs:125 encode_iupac (n ASCII bytes -> n + 2 BLASTNA bytes).
 * rmb_resolve_subject: seq/fasta_db.rs:86-131 -- CRandom (seeded with the length) replaces each
 * ambiguity code 4..14 by a base, and n_mask (n bytes) keeps the original codes; *has_mask is
 * 0 when the subject has no ambiguity code (n_mask then stays all zero). */
int rmb_matrix_parse(const char* text, int32_t scores[256], double freqs[16], double* lambda, char* err,
                     size_t errlen);
void rmb_encode_iupac(const char* ascii, size_t n, uint8_t* out);
void rmb_resolve_subject(const uint8_t* raw, uint32_t n, uint8_t* plus, uint8_t* n_mask, int32_t* has_mask);
/* rmb_resolve_twobit_n: seq/twobit.rs:73-135 -- a .2bit record's N blocks (starts/sizes as in the
 * file, clipped to n) get bases drawn from CRandom seeded with n, block by block; n_mask (n bytes,
 * zeroed by the caller) gets 14 there.  plus is the sentinel-wrapped record (n + 2 bytes). */
void rmb_resolve_twobit_n(uint32_t n, uint32_t n_blocks, const uint32_t* starts, const uint32_t* sizes,
                          uint8_t* plus, uint8_t* n_mask);

/* rmb_ka_resolve: the statistics for rmb_params.ka_* (rmblast-lib/src/ka_stats.rs:153-300, the
 * default mode): RMBlast's built-in table by matrix file base name and exact gap costs; else the
 * -matrix_lambda/-matrix_k/-matrix_alpha/-matrix_beta values in cli[4] (used when lambda, K and
 * alpha are > 0; zeros otherwise; NULL for none); else a "# KARLIN lambda .. k .. h|alpha ..
 * [beta ..]" line of matrix_text (NULL for none; matrix.rs:38-70); else none (ka[0] = -1).
 * The reference's last resort, an ALP simulation fit of the matrix, is not provided: such a
 * matrix gets no statistics here.  ka[5] = lambda, K, H, alpha, beta; *source = 0 none,
 * 1 table, 2 command line, 3 matrix comment. */
int rmb_ka_resolve(const char* matrix_name, const char* matrix_text, int32_t gap_open, int32_t gap_extend,
                   const double cli[4], double ka[5], int32_t* source, char* err, size_t errlen);

/* rmb_format_pairwise: pairwise output, outfmt 0 (rmblast-lib/src/output.rs:369-720), of the
 * results of one search.  query[i] and qlen[i] are the searched queries (with dust = 1 their DUST
 * intervals print in lower case; query may be NULL with dust = 0); query_deflines[i] is the full
 * FASTA header after '>'; subject_deflines[oid] each subject's full header, or NULL for a
 * database of ids only (.2bit).  db_name: as given to -db.  parts: bit 0 the program header,
 * bit 1 the footer (for output split across calls).  db_mtime >= 0 (seconds since 1970, UTC)
 * adds the footer's "Posted date" line.  The text is freed with rmb_text_free. */
int rmb_format_pairwise(rmb_ctx* ctx, const rmb_results* res, const uint8_t* const* query, const uint32_t* qlen,
                        const char* const* query_deflines, const char* const* subject_deflines,
                        const char* db_name, int64_t db_mtime, int32_t parts, char** text, size_t* text_len,
                        char* err, size_t errlen);

void rmb_results_free(rmb_results* res);
void rmb_text_free(void* p);
void rmb_ctx_destroy(rmb_ctx* ctx);

/* Traceback of one (query, subject) pair's prelim HSPs without any allocation.  It has no
 * counterpart in the reference; it is the GPU traceback of stage 4 above for callers that may not
 * call cudaMalloc -- code embedded in a process whose device memory belongs to another allocator
 * (a caching allocator that must account for every byte, a stream-ordered pool) or running where
 * an allocation could fail or stall.  All pointers are device memory the caller owns:
 * query/query_rc and subject/subject_rc are sentinel-wrapped BLASTNA (the subject with its
 * ambiguity codes restored), prelims n x 8 uint32 in the stage-2 record layout, out n x 9 uint32
 * in the stage-4 layout, ops n x ops_cap edit runs.  Record status (out word 1): 0 aligned,
 * 1 negative score, 2 did not fit the scratch, 3 the trace walk did not reach the seed (an
 * internal error), 4 the record's box or seed lies outside the sequences (skipped, no sequence
 * byte read), 5 the edit script is longer than ops_cap.
 * The scratch is a fixed 32 MiB array in the library that every GPU loading the library holds
 * until the process exits; query + subject must satisfy 8 (subject + 2) + 8 (query + 2) + 64 KiB
 * <= 32 MiB or the call fails with RMB_ELIMIT before any launch.  The array is shared out among
 * up to 256 threads; records whose trace outgrows a share run again on a quarter of the threads,
 * down to one thread holding all of it, and only a record that fails there too leaves status 2
 * (the call then returns RMB_ELIMIT, as it does for status 5).  The first call on a device looks
 * the array up (cudaGetSymbolAddress); make that first call before any stream capture.  Calls
 * share the array: two calls whose work overlaps on the GPU race.  The call waits for its
 * stream, and the caller's current device is the same on return. */
int rmb_traceback_noalloc(int32_t device, const uint8_t* query, const uint8_t* query_rc, uint32_t qlen,
                          const uint8_t* subject, const uint8_t* subject_rc, uint32_t slen, const uint32_t* prelims,
                          uint32_t n, int32_t gap_open, int32_t gap_extend, int32_t xdrop_gap_final,
                          const int32_t scores[256], uint32_t* out, uint32_t* ops, uint32_t ops_cap, void* stream,
                          char* err, size_t errlen);

/* The context's launch knobs (rmb_tune above).  rmb_tune_set rejects values outside the
 * ranges given there.  rmb_autotune: one search of the sample queries per candidate set (the
 * defaults, then one knob at a time around the best so far), each timed on the device; the
 * fastest set stays on the context and is written to *best, its device time per search to
 * *best_ms and the defaults' to *default_ms.  The sample's output is the same under every set. */
int rmb_tune_get(const rmb_ctx* ctx, rmb_tune* out);
int rmb_tune_set(rmb_ctx* ctx, const rmb_tune* tune, char* err, size_t errlen);
int rmb_autotune(rmb_ctx* ctx, uint32_t n_queries, const uint8_t* const* query, const uint32_t* qlen,
                 rmb_tune* best, double* best_ms, double* default_ms, char* err, size_t errlen);

/* Measurement helper: sustained int32 add/max throughput of the device in Tops/s (the
 * roofline denominator for the integer DP kernels). */
int rmb_probe_int32_peak(int32_t device, double* tops, char* err, size_t errlen);

/* Library version string. */
const char* rmb_version(void);

#ifdef __cplusplus
}
#endif
#endif /* RMB_GPU_H */
