// rmb_device.cuh -- device data layout shared by the kernels and their host launchers.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace rmb {

constexpr int32_t MININT = INT32_MIN / 2;  // search/gapped.rs:47

// The library on the device.  Every subject i occupies plus_off[i] .. plus_off[i] + len[i] + 2
// in plus / rc / align / align_rc (byte 0 and the last byte are the 15 sentinels), and
// packed_off[i] .. (+ ceil(len/4)) in `packed` with 3 zero pad bytes on each side.
struct DevLib {
    const uint8_t* plus;      // CRandom-resolved BLASTNA (scan, ungapped, prelim DP)
    const uint8_t* rc;        // reverse complement of plus
    const uint8_t* align;     // plus with the original ambiguity codes restored (traceback)
    const uint8_t* align_rc;  // reverse complement of align
    const uint8_t* packed;    // NCBI2NA, 4 bases per byte, first base in bits 7:6
    const uint64_t* plus_off;
    const uint64_t* packed_off;
    const uint32_t* len;
    uint32_t n;
};

// One batch of queries with their lookup tables.  Query i occupies off[i] .. off[i] + len[i] + 2
// in q / qrc / qmask.  Its table maps every lut_word_length-mer (a 2*lw-bit code) to the query
// offsets the reference's table returns for it, in the reference's retrieval order
// (ascending for the small table, descending for the megablast table): cell c holds
// cell_q[cq_off + cell_start[cs_off + c] .. cell_start[cs_off + c + 1]).  pv is an exact
// presence bitset of 4^lw bits.
struct DevQueries {
    const uint8_t* q;
    const uint8_t* qrc;
    const uint8_t* qmask;     // DUST-masked q (q itself when masking is off): table and exact word extension
    const uint8_t* qmask_rc;  // reverse complement of qmask
    const uint64_t* off;
    const uint32_t* len;
    const uint32_t* pv;
    const uint64_t* pv_off;
    const uint32_t* cell_start;
    const uint64_t* cs_off;
    const uint32_t* cell_q;
    const uint64_t* cq_off;
    const int32_t* lw;
    uint32_t n;
};

struct DevParams {
    int32_t gap_open, gap_extend, word_size;
    int32_t xdrop_ungap, xdrop_gap, xdrop_gap_final;
    int32_t gapped_cutoff;
    int32_t matrix[256];  // scores[q][s]
};

// Per word-hit record after the exact word extension (pair-major, scan order within a pair).
// qs: q_off | strand << 31 in the reference's record frame (forward query; RC subject for
// minus), s: s_off in that frame.
struct SeedHit { uint32_t qs, s; };

// Ungapped extension of a seed (search/ungapped.rs), box in the record frame.
struct UngBox { int32_t score; uint32_t q_start, q_end, s_start, s_end; uint32_t store; };

// Preliminary gapped result of one ungapped record (engine.rs:1317-1411), coordinates in the
// strand's record frame, plus the traceback seed prelim_pivot returns.
struct PrelimOut {
    int32_t score;  // < gapped cutoff or DP failure: INT32_MIN
    uint32_t q_start, q_end, s_start, s_end, tb_q, tb_s;
};

// Input of one traceback (engine.rs:1497-1560): the prelim HSP and its pair.
struct TbIn {
    uint32_t pair;
    uint32_t strand;
    uint32_t q_seed, s_seed, q_start, q_end, s_start, s_end;
};
struct TbOut {
    int32_t status;   // 0 ok, 1 no alignment (score < 0), 2 scratch overflow
    int32_t score;    // raw traceback score
    uint32_t q0, q1, s0, s1;  // in the DP frame (query_rc / plus subject for minus)
    uint32_t n_ops;
    uint32_t need;    // scratch bytes a retry needs (status 2)
};
// One extension's traceback (left or right of the improved seed).
struct TbHalf {
    int32_t status;  // 0 ok, 2 scratch overflow, 3 walk failure
    int32_t score;
    uint32_t a_len, b_len, n_ops, need;
    uint32_t tq, ts;  // the improved seed (DP frame)
};

}  // namespace rmb
