// rmb_kernels.hpp -- host-side launchers of the search-core kernels (rmb_kernels.cu).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "rmb_device.cuh"

namespace rmb {

cudaError_t launch_scan(bool write, const DevLib& L, const DevQueries& Q, int32_t ws, uint64_t pair0, uint64_t n_pairs,
                        uint32_t* counts, const uint64_t* offs, SeedHit* hits, uint32_t* hit_pair, int sms,
                        cudaStream_t st);
// Single-pass scan: counts plus the hits staged per warp (scan_stage_entries(n_pairs, sms)
// SeedHits of stage), then k_scan_gather puts a range of pairs' hits in pair order at their offsets.  A set
// *stage_over (a warp's stretch of SCAN_STAGE_PER_WARP entries ran out) means the staged hits are
// incomplete: the caller runs launch_scan(write) instead.
constexpr uint32_t SCAN_STAGE_PER_WARP = 32768;
uint64_t scan_stage_entries(uint64_t n_pairs, int sms);
cudaError_t launch_scan_stage(const DevLib& L, const DevQueries& Q, int32_t ws, uint64_t n_pairs, uint32_t* counts,
                              uint32_t* stage_start, SeedHit* stage, unsigned int* stage_over, int sms,
                              cudaStream_t st, bool queue);
cudaError_t launch_scan_gather(uint64_t pair0, uint64_t n_pairs, const uint32_t* counts, const uint64_t* offs,
                               const uint32_t* stage_start, const SeedHit* stage, SeedHit* hits, uint32_t* hit_pair,
                               int sms, cudaStream_t st);
// queue: 8 bytes of device scratch (the hit queue counter; zeroed here)
cudaError_t launch_ungapped(const DevLib& L, const DevQueries& Q, const DevParams* P, int32_t ucut, uint64_t n,
                            const SeedHit* hits, const uint32_t* hit_pair, UngBox* out, int sms, cudaStream_t st,
                            unsigned long long* queue, int blocks_per_sm = 8);
uint64_t dedup_threads(int sms);
// Bucket-parallel diagonal dedup that extends only the hits the hash admits (one warp per pair):
// flags and boxes as launch_ungapped + launch_dedup give them.
// device bytes of the fused dedup's unit lists (units_buf below) for a pair range
size_t dedup_units_bytes(uint64_t n_pairs, uint64_t n_hits, int sms);
cudaError_t launch_dedup_extend(const DevLib& L, const DevQueries& Q, const DevParams* P, int32_t ucut,
                                uint64_t pair0, uint64_t n_pairs, uint64_t n_hits, const uint64_t* offs,
                                const SeedHit* hits, UngBox* ub, uint8_t* flags, void* cells,
                                unsigned long long* queue, void* units_buf, int sms, cudaStream_t st);
size_t diag_cell_bytes();
cudaError_t launch_dedup(const DevLib& L, const DevQueries& Q, int32_t ws, int32_t ucut, uint64_t pair0,
                         uint64_t n_pairs, const uint64_t* offs, const SeedHit* hits, const UngBox* ub, uint8_t* flags,
                         uint32_t* scratch, void* cells, int sms, cudaStream_t st);
cudaError_t launch_prelim(const DevLib& L, const DevQueries& Q, const DevParams* P, uint64_t n, const uint32_t* list,
                          const uint32_t* idx, const SeedHit* hits, const uint32_t* hit_pair, const UngBox* ub,
                          PrelimOut* out, uint32_t* wide, unsigned int* n_wide, unsigned long long* cells, int sms,
                          cudaStream_t st);
// Whether the thread-per-extension kernel's int16 band entries and int8 score rows hold the
// parameters exactly (scores <= 127; X-drop and gap_open + gap_extend <= 8000).
// launch_prelim_stream uses n_wide[0] (overflow count) and n_wide[1] (record queue), both zeroed.
bool prelim_stream_eligible(const int32_t* matrix256, int32_t gap_open, int32_t gap_extend, int32_t xdrop_gap);
// geo: n x prelim_geo_bytes() of scratch for the per-record geometry.
size_t prelim_geo_bytes();
cudaError_t launch_prelim_prep(const DevLib& L, const DevQueries& Q, const DevParams* P, uint64_t n,
                               const uint32_t* idx, const SeedHit* hits, const uint32_t* hit_pair, const UngBox* ub,
                               void* geo, int sms, cudaStream_t st, const unsigned int* n_dev = nullptr);
// Launch shape of the thread-per-extension DP (from rmb_tune): group of cell steps between
// row-end blocks (4, 8, 16), resident blocks per SM, widest band a thread keeps, cell budget divisor.
// Counts a graph-captured chain keeps on the device: the DP's record count (its cell budget then
// follows on the device) and, for the front-loaded order, the front's length and the order
// buffer's length (the records past the front are read from its end).
// The fused dedup's work units (built on the device from the pair offsets).
struct DedupUnits {
    unsigned long long* heavy = nullptr;  // groups of the split pairs: pair | group << 32 | log2 G << 40
    uint32_t* light = nullptr;            // pairs with hits kept whole
    unsigned int* counts = nullptr;       // [0] heavy entries, [1] light entries
    uint64_t heavy_cap = 0;
};

struct StreamDevCounts {
    const unsigned int* n = nullptr;
    const unsigned int* n_front = nullptr;
    uint64_t order_end = 0;
};
struct StreamLaunch {
    int group = 8, blocks_per_sm = 6, window = 60, budget_div = 128;
};
cudaError_t launch_prelim_stream(const DevParams* P, uint64_t n, const void* geo, PrelimOut* out, uint32_t* wide,
                                 unsigned int* n_wide, unsigned long long* cells, int sms, cudaStream_t st,
                                 const uint32_t* order, uint32_t* cells_out, bool plain, const StreamLaunch& cfg,
                                 StreamDevCounts dc = StreamDevCounts{});
// Learned schedule (rmb_sched.cuh).  Raw features of each record (n x SCHED_NF floats); the
// network's predicted log1p cells of every record and the records in descending predicted cost
// (order, for launch_prelim_stream; scratch: sched_order_scratch_bytes()); the network on given
// raw features.  params: SCHED_NPARAM floats on the device.
cudaError_t launch_sched_features(const DevLib& L, const DevQueries& Q, const DevParams* P, uint64_t n,
                                  const uint32_t* idx, const SeedHit* hits, const uint32_t* hit_pair, const UngBox* ub,
                                  const uint32_t* pair_hits, float* out, int sms, cudaStream_t st);
size_t sched_order_scratch_bytes();
// layout 1: the predicted-costliest ~1/32 of the records first, the rest after in reverse arrival
// order (temp: sched_front_temp_bytes(n) bytes); 2: all records in descending predicted cost
size_t sched_front_temp_bytes(uint64_t n);
// the front-loaded order's front length, on the device, in launch_sched_order's scratch
const unsigned int* sched_front_count(const void* scratch);
cudaError_t launch_sched_order(const DevLib& L, const DevQueries& Q, const DevParams* P, uint64_t n,
                               const uint32_t* idx, const SeedHit* hits, const uint32_t* hit_pair, const UngBox* ub,
                               const uint32_t* pair_hits, const float* params, float* pred, void* scratch,
                               uint32_t* order, int sms, cudaStream_t st, int layout, void* temp, size_t temp_bytes, const unsigned int* n_dev = nullptr);
cudaError_t launch_sched_predict_features(uint64_t n, const float* feats, const float* params, float* pred, int sms,
                                          cudaStream_t st);
// Records `list` (the thread kernel's overflow), one warp per extension; dres holds 2 x n_list
// int4.  Records that overflow the warp rings go to `wide` (count in n_wide[0]).
cudaError_t launch_prelim_split(const DevLib& L, const DevQueries& Q, const DevParams* P, uint32_t n_list,
                                const uint32_t* list, const uint32_t* idx, const SeedHit* hits,
                                const uint32_t* hit_pair, const UngBox* ub, int4* dres, PrelimOut* out,
                                uint32_t* wide, unsigned int* n_wide, unsigned long long* cells, int sms,
                                cudaStream_t st, const unsigned int* n_dev = nullptr);
cudaError_t launch_prelim_wide(const DevLib& L, const DevQueries& Q, const DevParams* P, uint32_t n_wide,
                               const uint32_t* wide, const uint32_t* idx, const SeedHit* hits, const uint32_t* hit_pair,
                               const UngBox* ub, PrelimOut* out, int2* band_mem, uint64_t band_cap, uint32_t threads,
                               unsigned long long* cells, unsigned int* failures, cudaStream_t st, const unsigned int* n_dev = nullptr);
cudaError_t launch_traceback(const DevLib& L, const DevQueries& Q, const DevParams* P, uint32_t n, const TbIn* in,
                             TbOut* out, TbHalf* half, uint32_t* ops, uint32_t ops_cap, uint8_t* scratch,
                             uint64_t per_thread, uint64_t band_cells, uint32_t rows_cap, uint32_t threads,
                             unsigned long long* cells, bool whole, cudaStream_t st);
// The ops of the finished items of a traceback launch, packed at the host-computed offsets off[i]
// (items with status 2 are skipped), so only the ops in use cross to the host.
cudaError_t launch_gather_ops(uint32_t n, const uint32_t* ops, uint32_t ops_cap, const TbOut* out, const uint64_t* off,
                              uint32_t* dst, int sms, cudaStream_t st);

}  // namespace rmb

namespace rmb {
// Gathers, for the prelim DP results that passed the gapped cutoff, everything the host
// Phase 2a filter needs.  sel[k] indexes the prelim output array.
struct SurvivorRec {
    uint32_t pair;
    SeedHit hit;
    UngBox ub;
    PrelimOut po;
};
cudaError_t launch_gather_survivors(uint32_t n, const uint32_t* sel, const uint32_t* idx, const SeedHit* hits,
                                    const uint32_t* hit_pair, const UngBox* ub, const PrelimOut* po,
                                    SurvivorRec* out, cudaStream_t st, const unsigned int* n_dev = nullptr);
// flags[i] == want  ->  out list of i (order kept); returns the count through *n_out (device).
cudaError_t launch_select_eq(const uint8_t* flags, uint64_t n, uint8_t want, uint32_t* out, uint32_t* n_out,
                             void* temp, size_t& temp_bytes, cudaStream_t st);
// prelim score != INT32_MIN -> list of positions.
cudaError_t launch_select_prelim(const PrelimOut* po, uint64_t n, uint32_t* out, uint32_t* n_out, void* temp,
                                 size_t& temp_bytes, cudaStream_t st, const unsigned int* n_dev = nullptr);
// exclusive sum of counts[0..n) into offs[0..n] (offs[n] = total).
cudaError_t launch_offsets(const uint32_t* counts, uint64_t n, uint64_t* offs, void* temp, size_t& temp_bytes,
                           cudaStream_t st);
}  // namespace rmb

namespace rmb {
// Builds the lookup tables of nq queries on the device (Q.q/qrc/off/len/lw/cs_off/pv_off set;
// cell_start values are global offsets into cell_q, so Q.cq_off must be all zero).
// pos_off[i] = sum over earlier queries of (2 len + 1); n_pos the total; n_cells the sum of
// (4^lw + 1); n_pv the pv words.  Returns cudaErrorNotReady with temp_bytes set when temp is
// too small.  n_valid = table entries.
cudaError_t launch_lut_build(const DevQueries& Q, int32_t ws, uint32_t nq, const uint64_t* pos_off, uint64_t n_pos,
                             uint64_t n_cells, uint64_t n_pv, uint32_t* keys, uint32_t* vals, uint32_t* keys2,
                             uint32_t* vals2, uint32_t* counts, uint32_t* cs, uint32_t* cell_q, uint32_t* pv,
                             void* temp, size_t& temp_bytes, uint64_t& n_valid, cudaStream_t st);
}  // namespace rmb

namespace rmb {
cudaError_t launch_revcomp(const uint8_t* q, const uint64_t* off, const uint32_t* len, uint32_t nq, uint8_t* rc,
                           cudaStream_t st);
// DUST masking of a query batch: qm must hold a copy of q; `scratch` holds
// dust_scratch_bytes(nthreads); overflow counts queries whose interval list overflowed; compat
// adds the multi-chunk path's extra masked base after each interval.  qm may be null; bits
// (zeroed, per query at word offset bits_off[i]) gets one bit per position inside an interval.
uint32_t dust_threads(uint32_t nq, int sms);
size_t dust_scratch_bytes(uint32_t nthreads);
cudaError_t launch_dust(const uint8_t* q, const uint64_t* off, const uint32_t* len, uint32_t nq, uint8_t* qm,
                        void* scratch, uint32_t nthreads, unsigned int* overflow, bool compat, cudaStream_t st,
                        uint32_t* bits = nullptr, const uint64_t* bits_off = nullptr);
}  // namespace rmb
