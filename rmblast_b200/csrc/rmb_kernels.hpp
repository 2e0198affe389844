// rmb_kernels.hpp -- host-side launchers of the search-core kernels (rmb_kernels.cu).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "rmb_device.cuh"

namespace rmb {

cudaError_t launch_scan(bool write, const DevLib& L, const DevQueries& Q, int32_t ws, uint64_t pair0, uint64_t n_pairs,
                        uint32_t* counts, const uint64_t* offs, SeedHit* hits, uint32_t* hit_pair, int sms,
                        cudaStream_t st);
cudaError_t launch_ungapped(const DevLib& L, const DevQueries& Q, const DevParams* P, int32_t ucut, uint64_t n,
                            const SeedHit* hits, const uint32_t* hit_pair, UngBox* out, int sms, cudaStream_t st);
uint64_t dedup_threads(int sms);
size_t diag_cell_bytes();
cudaError_t launch_dedup(const DevLib& L, const DevQueries& Q, int32_t ws, int32_t ucut, uint64_t pair0,
                         uint64_t n_pairs, const uint64_t* offs, const SeedHit* hits, const UngBox* ub, uint8_t* flags,
                         uint32_t* scratch, void* cells, int sms, cudaStream_t st);
cudaError_t launch_prelim(const DevLib& L, const DevQueries& Q, const DevParams* P, uint64_t n, const uint32_t* idx,
                          const SeedHit* hits, const uint32_t* hit_pair, const UngBox* ub, PrelimOut* out,
                          uint32_t* wide, unsigned int* n_wide, unsigned long long* cells, int sms, cudaStream_t st);
cudaError_t launch_prelim_wide(const DevLib& L, const DevQueries& Q, const DevParams* P, uint32_t n_wide,
                               const uint32_t* wide, const uint32_t* idx, const SeedHit* hits, const uint32_t* hit_pair,
                               const UngBox* ub, PrelimOut* out, int2* band_mem, uint64_t band_cap, uint32_t threads,
                               unsigned long long* cells, unsigned int* failures, cudaStream_t st);
cudaError_t launch_traceback(const DevLib& L, const DevQueries& Q, const DevParams* P, uint32_t n, const TbIn* in,
                             TbOut* out, uint32_t* ops, uint32_t ops_cap, uint8_t* scratch, uint64_t per_thread,
                             uint64_t band_cells, uint32_t rows_cap, uint32_t threads, unsigned long long* cells,
                             cudaStream_t st);

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
                                    SurvivorRec* out, cudaStream_t st);
// flags[i] == want  ->  out list of i (order kept); returns the count through *n_out (device).
cudaError_t launch_select_eq(const uint8_t* flags, uint64_t n, uint8_t want, uint32_t* out, uint32_t* n_out,
                             void* temp, size_t& temp_bytes, cudaStream_t st);
// prelim score != INT32_MIN -> list of positions.
cudaError_t launch_select_prelim(const PrelimOut* po, uint64_t n, uint32_t* out, uint32_t* n_out, void* temp,
                                 size_t& temp_bytes, cudaStream_t st);
// exclusive sum of counts[0..n) into offs[0..n] (offs[n] = total).
cudaError_t launch_offsets(const uint32_t* counts, uint64_t n, uint64_t* offs, void* temp, size_t& temp_bytes,
                           cudaStream_t st);
}  // namespace rmb
