// rmb_kernels.cu -- sm_100a kernels of the search core.
//
//   k_scan        lookup-table scan of the packed library + exact word extension
//                 (blast/nascan.rs, blast/mblookup.rs:247-343, engine.rs:1118-1218); a warp per
//                 (query, subject) pair, lanes on consecutive scan offsets, two passes (count,
//                 then write at the pair's prefix offset) so every pair's hits keep scan order.
//   k_ungapped    ungapped X-drop extension of every word hit (search/ungapped.rs:38-121),
//                 one thread per hit, computed for all hits ahead of the dedup.
//   k_dedup       the order-dependent diagonal hash (search/diag_hash.rs) replayed per pair in
//                 scan order on the precomputed extensions, one thread per pair.
//   k_prelim_warp preliminary score-only X-drop DP (search/gapped.rs:124-418) of every ungapped
//                 record, one warp per record, the DP band in a shared-memory ring;
//                 k_prelim_wide reruns the records whose band outgrew the ring with the band in
//                 global memory (one thread per record).
//   k_traceback_warp  improve_seed + traceback X-drop DP + trace walk (engine.rs:383-572,
//                 engine.rs:2953-3039, search/gapped.rs:450-757), one warp per prelim HSP.
//
// All scores are int32; the arithmetic and the order of every comparison follow the cited
// reference functions so results are bit-identical.
#include <algorithm>
#include <cstdint>
#include <cstdio>

#include "rmb_device.cuh"
#include "rmb_dust.cuh"
#include "rmb_kernels.hpp"
#include "rmb_prelim_stream.cuh"

#include <cub/device/device_partition.cuh>
#include <thrust/iterator/counting_iterator.h>
#include "rmb_sched.cuh"
#include "rmb_ungapped.cuh"

namespace rmb {

// ---------------------------------------------------------------------------------------
// scan
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t kmer_at(const uint8_t* pk, uint32_t p, int lw) {
    const uint8_t* b = pk + (p >> 2);
    uint32_t raw = ((uint32_t)b[0] << 24) | ((uint32_t)b[1] << 16) | ((uint32_t)b[2] << 8) | (uint32_t)b[3];
    uint32_t sh = 2u * (16u - (p & 3u) - (uint32_t)lw);
    return (raw >> sh) & ((1u << (2 * lw)) - 1u);
}

struct PairView {
    const uint8_t* qmask;  // sentinel-wrapped
    const uint8_t* splus;  // sentinel-wrapped
    const uint8_t* src;    // sentinel-wrapped
    int64_t qlen, slen;
    int lw, ext_needed;
};

// engine.rs:1118-1149 (plus) and 1187-1218 (minus): exact extension to word_size on the
// masked query; returns false if the word hit is dropped.
__device__ __forceinline__ bool exact_extend(const PairView& v, uint32_t q0c, uint32_t p, uint32_t& qs, uint32_t& so) {
    const int64_t c1 = v.qlen + 1;
    const int64_t lw = v.lw, need = v.ext_needed;
    if ((int64_t)q0c < c1) {
        int64_t el = 0, er = 0;
        if (need > 0) {
            while (el < need) {
                int64_t qi = (int64_t)q0c - el - 1, si = (int64_t)p - el - 1;
                if (qi < 0 || si < 0) break;
                uint8_t qb = v.qmask[1 + qi], sb = v.splus[1 + si];
                if (qb >= 4 || sb >= 4 || qb != sb) break;
                ++el;
            }
            while (el + er < need) {
                int64_t qi = (int64_t)q0c + lw + er, si = (int64_t)p + lw + er;
                if (qi >= v.qlen || si >= v.slen) break;
                uint8_t qb = v.qmask[1 + qi], sb = v.splus[1 + si];
                if (qb >= 4 || sb >= 4 || qb != sb) break;
                ++er;
            }
            if (el + er < need) return false;
        }
        qs = (uint32_t)((int64_t)q0c - el);
        so = (uint32_t)((int64_t)p - el);
        return true;
    }
    const int64_t rcq = (int64_t)q0c - c1;
    const int64_t q0 = v.qlen - rcq - lw, s0 = v.slen - (int64_t)p - lw;
    if (q0 < 0 || s0 < 0) return false;
    int64_t el = 0, er = 0;
    if (need > 0) {
        while (er < need) {
            int64_t qi = q0 + lw + er, si = s0 + lw + er;
            if (qi >= v.qlen || si >= v.slen) break;
            uint8_t qb = v.qmask[1 + qi], sb = v.src[1 + si];
            if (qb >= 4 || sb >= 4 || qb != sb) break;
            ++er;
        }
        while (el + er < need) {
            int64_t qi = q0 - el - 1, si = s0 - el - 1;
            if (qi < 0 || si < 0) break;
            uint8_t qb = v.qmask[1 + qi], sb = v.src[1 + si];
            if (qb >= 4 || sb >= 4 || qb != sb) break;
            ++el;
        }
        if (el + er < need) return false;
    }
    qs = (uint32_t)(q0 + er) | 0x80000000u;
    so = (uint32_t)(s0 + er);
    return true;
}

// One warp per (query, subject) pair: the subject's words at the scan stride against the query's
// lookup table (lookup.rs scan), each word hit extended exactly to word_size.  Hits leave in scan
// order (subject position, then lookup-cell order).
//   SCAN_COUNT: per-pair hit counts only.
//   SCAN_WRITE: hits at the pair's offset in `hits` (offs from the counts).
//   SCAN_STAGE: counts, and the hits appended to this warp's stretch of `hits` (stage_cap entries
//               from warp * stage_cap), the pair's first entry in stage_start; if a stretch runs
//               out, *stage_over is set and the batch takes the SCAN_WRITE pass instead.
enum { SCAN_COUNT = 0, SCAN_WRITE = 1, SCAN_STAGE = 2 };

template <int MODE>
__global__ void __launch_bounds__(256) k_scan(DevLib L, DevQueries Q, int32_t ws, uint64_t pair0, uint64_t n_pairs,
                                               uint32_t* counts, const uint64_t* offs, SeedHit* hits,
                                               uint32_t* hit_pair, uint32_t* stage_start, uint32_t stage_cap,
                                               unsigned int* stage_over, unsigned long long* pair_queue) {
    constexpr bool WRITE = MODE != SCAN_COUNT;
    // per warp: each lane's first candidate index, lookup-cell start and scan position
    __shared__ uint32_t s_first[8][32], s_cell[8][32], s_pos[8][32];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    const uint32_t stage0 = MODE == SCAN_STAGE ? (uint32_t)warp * stage_cap : 0u;  // this warp's stretch
    uint32_t cursor = 0;                                                            // entries of it used
    bool fits = true;
    // pairs by warp stride, or, with pair_queue, the next pair off a grid-wide counter as a warp
    // finishes one (subject lengths vary 100-fold, so fixed strides leave warps idle at the end)
    uint64_t w_next = warp;
    auto next_pair = [&]() -> uint64_t {
        if (pair_queue) {
            unsigned long long x = 0;
            if (lane == 0) x = atomicAdd(pair_queue, 1ull);
            return __shfl_sync(0xffffffffu, x, 0);
        }
        const uint64_t r = w_next;
        w_next += nwarps;
        return r;
    };
    for (uint64_t w = next_pair(); w < n_pairs; w = next_pair()) {
        const uint64_t pair = pair0 + w;
        const uint32_t qi = (uint32_t)(pair / L.n), si = (uint32_t)(pair % L.n);
        const uint32_t qlen = Q.len[qi], slen = L.len[si];
        uint64_t out = MODE == SCAN_WRITE ? offs[w] : MODE == SCAN_STAGE ? (uint64_t)(stage0 + cursor) : 0;
        uint32_t total = 0;
        if (qlen >= (uint32_t)ws && slen >= (uint32_t)ws) {
            PairView v;
            v.qmask = Q.qmask + Q.off[qi];
            v.splus = L.plus + L.plus_off[si];
            v.src = L.rc + L.plus_off[si];
            v.qlen = qlen;
            v.slen = slen;
            v.lw = Q.lw[qi];
            v.ext_needed = ws - v.lw;
            const uint32_t step = (uint32_t)(ws - v.lw + 1);
            const uint32_t npos = (slen - (uint32_t)v.lw) / step + 1;
            const uint8_t* pk = L.packed + L.packed_off[si];
            const uint32_t* pv = Q.pv + Q.pv_off[qi];
            const uint32_t* cs = Q.cell_start + Q.cs_off[qi];
            const uint32_t* cq = Q.cell_q + Q.cq_off[qi];
            for (uint32_t k0 = 0; k0 < npos; k0 += 32) {
                // lane l looks up position k0 + l; its lookup cell's entries b .. b + cnt are
                // then spread over the warp, one entry a lane, in (position, entry) order
                const uint32_t k = k0 + lane;
                uint32_t cnt = 0, b = 0, p = 0;
                if (k < npos) {
                    p = k * step;
                    const uint32_t idx = kmer_at(pk, p, v.lw);
                    if (__ldg(pv + (idx >> 5)) & (1u << (idx & 31))) {
                        b = __ldg(cs + idx);
                        cnt = __ldg(cs + idx + 1) - b;
                    }
                }
                uint32_t incl = cnt;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const uint32_t t = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= o) incl += t;
                }
                const uint32_t n_cand = __shfl_sync(0xffffffffu, incl, 31);
                s_first[wib][lane] = incl - cnt;
                s_cell[wib][lane] = b;
                s_pos[wib][lane] = p;
                __syncwarp();
                uint32_t chunk = 0;  // hits of this chunk so far
                for (uint32_t r0 = 0; r0 < n_cand; r0 += 32) {
                    const uint32_t t = r0 + lane;
                    bool ok = false;
                    uint32_t qs = 0, so = 0;
                    if (t < n_cand) {
                        int owner = 0;  // the last lane whose first entry is <= t
#pragma unroll
                        for (int st = 16; st; st >>= 1)
                            if (s_first[wib][owner + st] <= t) owner += st;
                        ok = exact_extend(v, __ldg(cq + s_cell[wib][owner] + (t - s_first[wib][owner])),
                                          s_pos[wib][owner], qs, so);
                    }
                    const unsigned m = __ballot_sync(0xffffffffu, ok);
                    const uint32_t nm = (uint32_t)__popc(m);
                    if (MODE == SCAN_STAGE && fits && cursor + total + chunk + nm > stage_cap) {
                        fits = false;
                        if (lane == 0) atomicExch(stage_over, 1u);
                    }
                    if (WRITE && fits && ok) {
                        const uint64_t o = out + total + chunk + (uint32_t)__popc(m & ((1u << lane) - 1u));
                        hits[o] = SeedHit{qs, so};
                        if (MODE == SCAN_WRITE) hit_pair[o] = (uint32_t)pair;
                    }
                    chunk += nm;
                }
                __syncwarp();
                total += chunk;
            }
        }
        if (MODE != SCAN_WRITE && lane == 0) counts[w] = total;
        if (MODE == SCAN_STAGE) {
            if (lane == 0) stage_start[w] = stage0 + cursor;
            cursor += total;
        }
    }
}

// The staged hits of each pair into pair order: hits[offs[w] ..] = stage[stage_start[w] ..], with
// the pair id; one warp per pair.
__global__ void __launch_bounds__(256) k_scan_gather(uint64_t pair0, uint64_t n_pairs, const uint32_t* counts,
                                                      const uint64_t* offs, const uint32_t* stage_start,
                                                      const SeedHit* __restrict__ stage, SeedHit* __restrict__ hits,
                                                      uint32_t* __restrict__ hit_pair) {
    const int lane = threadIdx.x & 31;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t w = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < n_pairs; w += nwarps) {
        const uint32_t c = counts[pair0 + w];
        const uint64_t o = offs[w];
        const SeedHit* src = stage + stage_start[pair0 + w];
        for (uint32_t i = lane; i < c; i += 32) {
            hits[o + i] = src[i];
            hit_pair[o + i] = (uint32_t)(pair0 + w);
        }
    }
}

// ---------------------------------------------------------------------------------------
// ungapped extension: search/ungapped.rs:38-121
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ void extend_ungapped(const uint8_t* query, int64_t q_real, const uint8_t* subject,
                                                int64_t s_real, uint32_t q_off, uint32_t s_off, const int32_t* mat,
                                                int32_t xdrop, int32_t& score_out, uint32_t& qs_out, uint32_t& qe_out,
                                                uint32_t& ss_out, uint32_t& se_out) {
    const int32_t x = -xdrop;
    const int64_t qo = q_off, so = s_off;
    int32_t score = 0, sum = 0;
    int64_t q_beg = qo;
    {
        int64_t q = qo - 1, s = so - 1;
        while (q >= 0 && s >= 0) {
            const uint8_t qb = query[1 + q], sb = subject[1 + s];
            if (qb == 15 || sb == 15) break;
            sum += mat[((qb & 15) << 4) | (sb & 15)];
            if (sum > 0) {
                q_beg = q;
                score += sum;
                sum = 0;
            } else if (sum < x) {
                break;
            }
            --q;
            --s;
        }
    }
    int64_t q_end = qo;
    int32_t xc = x;
    sum = 0;
    {
        int64_t q = qo, s = so;
        while (q < q_real && s < s_real) {
            const uint8_t qb = query[1 + q], sb = subject[1 + s];
            if (qb == 15 || sb == 15) break;
            sum += mat[((qb & 15) << 4) | (sb & 15)];
            if (sum > 0) {
                q_end = q + 1;
                score += sum;
                xc = (-score > x) ? -score : x;
                sum = 0;
            } else if (sum < xc) {
                break;
            }
            ++q;
            ++s;
        }
    }
    score_out = score;
    qs_out = (uint32_t)q_beg;
    qe_out = (uint32_t)q_end;
    ss_out = (uint32_t)(so - (qo - q_beg));
    se_out = (uint32_t)(so + (q_end - qo));
}

// engine.rs:1165-1170 (plus) and 1244-1261 (minus): the extension in NCBI's frame, its box in
// the record frame, and the value the diagonal hash stores for the seed.
// One word hit per lane at a time: the two walks of extend_ungapped (left, then right, in the
// strand's frame) as one resumable walk of UNG_GROUP steps per round; a lane whose hit is done
// takes the next hit index from the grid-wide queue (one atomic per warp and round), so lanes do
// not wait for the longest walk of the warp.  Same arithmetic as extend_ungapped + the box of
// engine.rs:1165-1170 / 1244-1261.
// 16 steps a round: the walks at the default size run hundreds of bases, so fewer refills pay
// for the idle steps after a walk ends (8 measured 49-50 ms, 16 47 ms a step).  Four bases a
// step with their loads issued together measured slower, on this kernel (27 -> 32 ms a step on
// 1,000 queries of 1-200 kb) and in the fused dedup's lane walks
constexpr int UNG_GROUP = 16;
// QUEUE: a persistent grid whose lanes take hits from a grid-wide queue as their walks end (the
// batched pipeline); otherwise one hit per thread, thread i taking hit i (the plain pipeline).
template <bool QUEUE>
__global__ void __launch_bounds__(256) k_ungapped(DevLib L, DevQueries Q, const DevParams* __restrict__ P,
                                                   int32_t ucut, uint64_t n, const SeedHit* __restrict__ hits,
                                                   const uint32_t* __restrict__ hit_pair, UngBox* __restrict__ out,
                                                   unsigned long long* __restrict__ queue) {
    __shared__ int32_t mat[256];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) mat[i] = P->matrix[i];
    __syncthreads();
    const int32_t ws = P->word_size, xdrop = P->xdrop_ungap;
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    int phase = 0;  // 0 needs a hit, 1 walking, 3 queue empty
    uint64_t i = 0;
    UngWalk walk;
    SeedHit h{0, 0};
    uint32_t lw = 0;
    bool taken = false;
    for (;;) {
        const unsigned need = __ballot_sync(FULL, phase == 0);
        if (need) {
            unsigned long long base = 0;
            if (QUEUE) {
                const int leader = __ffs(need) - 1;
                if (lane == leader) base = atomicAdd(queue, (unsigned long long)__popc(need));
                base = __shfl_sync(FULL, base, leader);
            }
            if (phase == 0) {
                if (QUEUE) {
                    i = base + (uint64_t)__popc(need & ((1u << lane) - 1u));
                } else {
                    i = taken ? n : (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
                    taken = true;
                }
                if (i >= n) {
                    phase = 3;
                } else {
                    h = hits[i];
                    const uint32_t pair = hit_pair[i];
                    const uint32_t qi = pair / L.n, si = pair % L.n;
                    const int32_t qlen = (int32_t)Q.len[qi], slen = (int32_t)L.len[si];
                    lw = (uint32_t)Q.lw[qi];
                    const int32_t qo = (int32_t)(h.qs & 0x7fffffffu), so = (int32_t)h.s;
                    if (!(h.qs >> 31))
                        walk.start(Q.q + Q.off[qi], L.plus + L.plus_off[si], qlen, slen, qo, so, xdrop);
                    else
                        walk.start(Q.qrc + Q.off[qi], L.plus + L.plus_off[si], qlen, slen, qlen - 1 - qo, slen - 1 - so,
                                   xdrop);
                    phase = 1;
                }
            }
        }
        if (!__any_sync(FULL, phase == 1)) break;
#pragma unroll
        for (int g = 0; g < UNG_GROUP; ++g) {
            if (phase == 1 && walk.step(mat) == 2) {
                // the box in the record frame, and the value the diagonal hash stores
                int32_t sc;
                uint32_t a, b, c, d;
                walk.result(sc, a, b, c, d);
                UngBox u;
                u.score = sc;
                if (!(h.qs >> 31)) {
                    u.q_start = a;
                    u.q_end = b;
                    u.s_start = c;
                    u.s_end = d;
                    u.store = sc >= ucut ? d : h.s + (uint32_t)ws;
                } else {
                    const uint32_t qlen = (uint32_t)walk.qlen, slen = (uint32_t)walk.slen;
                    u.q_start = qlen - b;
                    u.q_end = qlen - a;
                    u.s_start = slen - d;
                    u.s_end = slen - c;
                    const uint32_t key = slen - h.s - lw;
                    u.store = sc >= ucut ? d : key + (uint32_t)ws;
                }
                out[i] = u;
                phase = 0;
            }
        }
    }
}

// ---------------------------------------------------------------------------------------
// diagonal dedup: search/diag_hash.rs:24-111 replayed in scan order (engine.rs:1151-1170,
// 1220-1261).  flags[i]: 0 = dropped by the hash, 1 = seed, 3 = seed kept as an ungapped hit.
// ---------------------------------------------------------------------------------------
struct DiagCell { int32_t diag; uint32_t level, next; };

__device__ __forceinline__ uint32_t diag_bucket(int32_t d) { return ((uint32_t)d * 0x9E370001u) % 512u; }

__device__ void dedup_pair(uint32_t tag, uint64_t b, uint64_t e, int32_t ws, int32_t lw, uint32_t qlen, uint32_t slen,
                           int32_t ucut, const SeedHit* __restrict__ hits, const UngBox* __restrict__ ub,
                           uint8_t* __restrict__ flags, uint32_t* bb, uint32_t* bt, DiagCell* cells) {
    const int32_t window = 1 - ws;
    uint32_t occ = 1;  // cells are 1-based, cells[k - 1] holds cell k
    for (uint64_t i = b; i < e; ++i) {
        const SeedHit h = hits[i];
        const uint32_t qo = h.qs & 0x7fffffffu, so = h.s;
        int32_t diag;
        uint32_t key;
        if (!(h.qs >> 31)) {
            diag = (int32_t)(so - qo);
            key = so;
        } else {
            diag = (int32_t)(slen - 2u * qlen - 1u + (qo - so));
            key = slen - so - (uint32_t)lw;
        }
        const uint32_t bk = diag_bucket(diag);
        const uint32_t head = bt[bk] == tag ? bb[bk] : 0u;
        uint32_t last = 0;
        for (uint32_t c = head; c; c = cells[c - 1].next)
            if (cells[c - 1].diag == diag) { last = cells[c - 1].level; break; }
        if (key < last) { flags[i] = 0; continue; }
        const UngBox u = ub[i];
        flags[i] = u.score >= ucut ? 3 : 1;
        bool done = false;
        for (uint32_t c = head; c; c = cells[c - 1].next) {
            DiagCell& cl = cells[c - 1];
            if (cl.diag == diag) { cl.level = u.store; done = true; break; }
            if ((int32_t)(key - cl.level) > window) { cl.diag = diag; cl.level = u.store; done = true; break; }
        }
        if (!done) {
            cells[occ - 1] = DiagCell{diag, u.store, head};
            bb[bk] = occ;
            bt[bk] = tag;
            ++occ;
        }
    }
}

__global__ void __launch_bounds__(128) k_dedup(DevLib L, DevQueries Q, int32_t ws, int32_t ucut, uint64_t pair0,
                                                uint64_t n_pairs, const uint64_t* __restrict__ offs,
                                                const SeedHit* __restrict__ hits, const UngBox* __restrict__ ub,
                                                uint8_t* __restrict__ flags, uint32_t* __restrict__ scratch,
                                                DiagCell* __restrict__ cells) {
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t nth = (uint64_t)gridDim.x * blockDim.x;
    uint32_t* bb = scratch + tid * 1024;
    uint32_t* bt = bb + 512;
    for (int k = 0; k < 512; ++k) bt[k] = 0;
    for (uint64_t w = tid; w < n_pairs; w += nth) {
        const uint64_t b = offs[w], e = offs[w + 1];
        if (b == e) continue;
        const uint64_t pair = pair0 + w;
        const uint32_t qi = (uint32_t)(pair / L.n), si = (uint32_t)(pair % L.n);
        dedup_pair((uint32_t)w + 1u, b, e, ws, Q.lw[qi], Q.len[qi], L.len[si], ucut, hits, ub, flags, bb, bt, cells + b);
    }
}

// Bucket-parallel dedup with the ungapped extension of the hits the hash admits.  The reference
// checks a word hit's diagonal against the hash first and extends only the hits it admits
// (engine.rs:1151-1172, 1220-1261).  The hash's 512 buckets are independent: get and insert walk
// only the chain of bucket(diag), and a stale cell is recycled only inside that chain
// (diag_hash.rs:51-110); cells are drawn from one pool, but which index a cell gets changes
// nothing.  So one warp replays one (query, subject) pair: the pair's hits go by in scan order,
// 32 a round; the hits of a round that share a bucket are decided in scan order, the buckets at
// once, and only an admitted hit is extended.  The reference's work,
// in its order per bucket, with the buckets in parallel: for hit-dense pairs (an all-against-
// all search keeps ~1% of its hits), where extending every hit first wastes most of the work.
constexpr int DDX_WARPS = 8;
// a pass whose admitted hits are at most this many extends them one after another with the whole
// warp (ung_walk_warp); more run one a lane (UngWalk)
constexpr int DDX_COOP = 6;
// a hit-heavy pair's hits go to at most 2^DDX_GLOG_MAX bucket groups
constexpr uint32_t DDX_GLOG_MAX = 5;

// Warp-cooperative ungapped X-drop extension: UngWalk's result (left walk, then right walk), 32
// bases a round.  Every lane calls it with the same arguments and gets the same result.  A round
// scores 32 consecutive bases and forms the running sum P of the walk and its running maximum M
// with warp scans.  The sequential walk's sum is P - M_before (M_before: M up to the previous
// base), so it banks where P > M_before, and it stops at the first base that is past a sequence
// end or has code 15 on either side, or where it does not bank and P - M_before < xc: xc is
// -xdrop on the left, and on the right -xdrop until the first bank, then
// max(-(left score + M_before), -xdrop).  The last bank before the stop is the extension's end,
// and M_before at the stop its gain.
__device__ __forceinline__ void ung_walk_warp(const uint8_t* __restrict__ qb, const uint8_t* __restrict__ sb, int32_t qlen,
                              int32_t slen, int32_t wq, int32_t wsx, int32_t xdrop, const int32_t* mat, int32_t& score,
                              int32_t& q_beg, int32_t& q_end) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int32_t x = -xdrop;
    int32_t score0 = 0;
#pragma unroll 1
    for (int dir = -1; dir <= 1; dir += 2) {
        const int32_t q0 = dir < 0 ? wq - 1 : wq, s0 = dir < 0 ? wsx - 1 : wsx;
        int32_t P = 0, M = 0, best = wq, gain = 0;
#pragma unroll 1
        for (int32_t base = 0;; base += 32) {
            const int32_t qj = q0 + dir * (base + lane), sj = s0 + dir * (base + lane);
            bool hard = dir < 0 ? (qj < 0 || sj < 0) : (qj >= qlen || sj >= slen);
            int32_t d = 0;
            if (!hard) {
                const uint8_t a = qb[1 + qj], c = sb[1 + sj];
                hard = a == 15 || c == 15;
                if (!hard) d = mat[((a & 15) << 4) | (c & 15)];
            }
            int32_t p = d;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int32_t v = __shfl_up_sync(FULL, p, o);
                if (lane >= o) p += v;
            }
            p += P;
            int32_t mx = p;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int32_t v = __shfl_up_sync(FULL, mx, o);
                if (lane >= o) mx = max(mx, v);
            }
            mx = max(mx, M);
            int32_t mprev = __shfl_up_sync(FULL, mx, 1);
            if (lane == 0) mprev = M;
            const bool bank = !hard && p > mprev;
            const int32_t xc = dir < 0 || mprev <= 0 ? x : max(-(score0 + mprev), x);
            const bool stop = hard || (!bank && p - mprev < xc);
            const unsigned sm = __ballot_sync(FULL, stop);
            const int f = sm ? __ffs((int)sm) - 1 : 32;
            const unsigned bm = __ballot_sync(FULL, bank) & (f == 32 ? FULL : ((1u << f) - 1u));
            if (bm) {
                const int32_t ql = q0 + dir * (base + (31 - __clz((int)bm)));
                best = dir < 0 ? ql : ql + 1;
            }
            if (f < 32) {
                gain = __shfl_sync(FULL, mprev, f);
                break;
            }
            P = __shfl_sync(FULL, p, 31);
            M = __shfl_sync(FULL, mx, 31);
        }
        if (dir < 0) {
            q_beg = best;
            score0 = gain;
        } else {
            q_end = best;
            score = score0 + gain;
        }
    }
}

// The fused dedup's units: a pair with h > 0 hits gets G = 2^gl groups, gl the smallest at or
// above glog with h <= unit_hits << gl (at most DDX_GLOG_MAX).  Pairs with G > 1 list their
// groups in `heavy` (pair | group << 32 | gl << 40), the others themselves in `light`.
__global__ void k_dedup_units(uint64_t n_pairs, const uint64_t* __restrict__ offs, uint32_t glog, uint64_t unit_hits,
                              DedupUnits units) {
    for (uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n_pairs;
         p += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t hp = offs[p + 1] - offs[p];
        uint32_t gl = glog;
        while (gl < DDX_GLOG_MAX && hp > (unit_hits << gl)) ++gl;
        const bool light = hp != 0 && gl == 0;
        const unsigned am = __activemask();
        const unsigned lm = __ballot_sync(am, light);
        const int lead = __ffs((int)am) - 1, lane = threadIdx.x & 31;
        unsigned int lb = 0;
        if (lane == lead && lm) lb = atomicAdd(&units.counts[1], (unsigned)__popc(lm));
        lb = __shfl_sync(am, lb, lead);
        if (light) units.light[lb + __popc(lm & ((1u << lane) - 1u))] = (uint32_t)p;
        if (hp != 0 && gl > 0) {
            const unsigned int hb = atomicAdd(&units.counts[0], 1u << gl);
            for (uint32_t g = 0; g < (1u << gl); ++g)
                if (hb + g < units.heavy_cap)  // never false: heavy_cap bounds the sum of the G
                    units.heavy[hb + g] = (unsigned long long)p | ((unsigned long long)g << 32) |
                                          ((unsigned long long)gl << 40);
        }
    }
}

__global__ void __launch_bounds__(DDX_WARPS * 32, 4) k_dedup_extend(DevLib L, DevQueries Q,
                                                                 const DevParams* __restrict__ P, int32_t ucut,
                                                                 uint64_t pair0, uint64_t n_pairs,
                                                                 const uint64_t* __restrict__ offs,
                                                                 const SeedHit* __restrict__ hits,
                                                                 UngBox* __restrict__ ub, uint8_t* __restrict__ flags,
                                                                 DiagCell* __restrict__ cells,
                                                                 unsigned long long* __restrict__ queue,
                                                                 DedupUnits units) {
    __shared__ int32_t mat[256];
    __shared__ uint32_t heads[DDX_WARPS][512];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) mat[i] = P->matrix[i];
    __syncthreads();
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    uint32_t* hd = heads[threadIdx.x >> 5];
    const int32_t ws = P->word_size, xdrop = P->xdrop_ungap, window = 1 - ws;
    // A unit is one pair's hits in the buckets of one group (bucket & (G - 1)).  A pair is split
    // when it holds more than a warp's share of the launch's hits (each group reads all the
    // pair's hits and runs its passes with fewer lanes, so splitting only pays where one pair
    // would hold the end of the launch).  The units of the pairs split into groups come first (units.heavy, a pair's groups one after another), then
    // one unit for each other pair with hits (units.light), so a hit-heavy pair's groups start
    // early and run side by side instead of holding the end of the launch.
    const unsigned int n_heavy = units.counts[0], n_units = n_heavy + units.counts[1];
    for (;;) {
        unsigned long long u_id = 0;
        if (lane == 0) u_id = atomicAdd(queue, 1ull);
        u_id = __shfl_sync(FULL, u_id, 0);
        if (u_id >= n_units) break;
        uint64_t w;
        uint32_t grp = 0, gmask = 0;
        if (u_id < n_heavy) {
            const unsigned long long v = units.heavy[u_id];
            w = (uint32_t)v;
            grp = (uint32_t)(v >> 32) & 0xffu;
            gmask = (1u << ((uint32_t)(v >> 40) & 0xffu)) - 1u;
        } else {
            w = units.light[u_id - n_heavy];
        }
        {
            const uint64_t b = offs[w], e = offs[w + 1];
            const uint64_t pair = pair0 + w;
            const uint32_t qi = (uint32_t)(pair / L.n), si = (uint32_t)(pair % L.n);
            const uint32_t qlen = Q.len[qi], slen = L.len[si];
            const int32_t lw = Q.lw[qi];
            const uint8_t* qf = Q.q + Q.off[qi];
            const uint8_t* qr = Q.qrc + Q.off[qi];
            const uint8_t* sp = L.plus + L.plus_off[si];
            DiagCell* pool = cells + b;  // hit i's cell, if it inserts one, is pool[i - b]
            for (int k = lane; k < 512; k += 32) hd[k] = 0;
            __syncwarp();
            for (uint64_t r = b; r < e; r += 32) {
                const uint64_t i = r + (uint64_t)lane;
                bool have = i < e;
                SeedHit h{0, 0};
                int32_t diag = 0;
                uint32_t key = 0, bk = 512u + (uint32_t)lane;  // lanes without a hit: a bucket of their own
                if (have) {
                    h = hits[i];
                    const uint32_t qo = h.qs & 0x7fffffffu, so = h.s;
                    if (!(h.qs >> 31)) {
                        diag = (int32_t)(so - qo);
                        key = so;
                    } else {
                        diag = (int32_t)(slen - 2u * qlen - 1u + (qo - so));
                        key = slen - so - (uint32_t)lw;
                    }
                    bk = diag_bucket(diag);
                    if ((bk & gmask) != grp) {  // another unit's bucket
                        have = false;
                        bk = 512u + (uint32_t)lane;
                    }
                }
                const unsigned same = __match_any_sync(FULL, bk);
                // Passes over the round's pending hits.  Each looks its diagonal up in the chains as
                // they stand; in each bucket the pending hits before the first one the hash admits are
                // dropped at once (a dropped hit changes no chain, so the lookups of the ones after it
                // stay right), the first admitted one is extended and inserted, and the bucket's hits
                // after it wait for the next pass.  A run of dropped hits on one repeat's diagonal
                // takes one pass instead of one turn each.
                bool pending = have;
                while (__any_sync(FULL, pending)) {
                    uint32_t head = 0;
                    bool admitted = false;
                    if (pending) {
                        head = hd[bk];
                        uint32_t last = 0;
                        for (uint32_t c = head; c; c = pool[c - 1].next)
                            if (pool[c - 1].diag == diag) { last = pool[c - 1].level; break; }
                        admitted = key >= last;
                    }
                    const unsigned adm = __ballot_sync(FULL, pending && admitted) & same;
                    const int first = adm ? __ffs((int)adm) - 1 : 32;
                    bool ext = false;
                    if (pending) {
                        if (lane < first) {
                            flags[i] = 0;
                            pending = false;
                        } else if (lane == first) {
                            ext = true;
                            pending = false;
                        }
                    }
                    UngBox u{};
                    int32_t sc = 0;
                    uint32_t a0 = 0, a1 = 0, c0 = 0, c1 = 0;
                    const unsigned em = __ballot_sync(FULL, ext);
                    if (em && __popc(em) <= DDX_COOP) {
                        // few extensions: each with the whole warp, one after another
                        for (unsigned m = em; m; m &= m - 1u) {
                            const int src = __ffs((int)m) - 1;
                            const uint32_t hqs = __shfl_sync(FULL, h.qs, src), hs = __shfl_sync(FULL, h.s, src);
                            const bool minus = hqs >> 31;
                            const int32_t qo = (int32_t)(hqs & 0x7fffffffu), so = (int32_t)hs;
                            const int32_t wq = minus ? (int32_t)qlen - 1 - qo : qo;
                            const int32_t wsx = minus ? (int32_t)slen - 1 - so : so;
                            int32_t s_, qb_, qe_;
                            ung_walk_warp(minus ? qr : qf, sp, (int32_t)qlen, (int32_t)slen, wq, wsx, xdrop, mat, s_, qb_,
                                          qe_);
                            if (lane == src) {
                                sc = s_;
                                a0 = (uint32_t)qb_;
                                a1 = (uint32_t)qe_;
                                c0 = (uint32_t)(wsx - (wq - qb_));
                                c1 = (uint32_t)(wsx + (qe_ - wq));
                            }
                        }
                    } else if (ext) {
                        const int32_t qo = (int32_t)(h.qs & 0x7fffffffu), so = (int32_t)h.s;
                        UngWalk walk;
                        if (!(h.qs >> 31)) walk.start(qf, sp, (int32_t)qlen, (int32_t)slen, qo, so, xdrop);
                        else walk.start(qr, sp, (int32_t)qlen, (int32_t)slen, (int32_t)qlen - 1 - qo,
                                        (int32_t)slen - 1 - so, xdrop);
                        while (walk.step(mat) != 2) {
                        }
                        walk.result(sc, a0, a1, c0, c1);
                    }
                    if (ext) {
                        u.score = sc;
                        if (!(h.qs >> 31)) {
                            u.q_start = a0; u.q_end = a1; u.s_start = c0; u.s_end = c1;
                            u.store = sc >= ucut ? c1 : h.s + (uint32_t)ws;
                        } else {
                            u.q_start = qlen - a1; u.q_end = qlen - a0; u.s_start = slen - c1; u.s_end = slen - c0;
                            u.store = sc >= ucut ? c1 : key + (uint32_t)ws;
                        }
                        ub[i] = u;
                        flags[i] = sc >= ucut ? 3 : 1;
                    }
                    bool append = false;
                    if (ext) {
                        append = true;
                        for (uint32_t c = head; c; c = pool[c - 1].next) {
                            DiagCell& cl = pool[c - 1];
                            if (cl.diag == diag) { cl.level = u.store; append = false; break; }
                            if ((int32_t)(key - cl.level) > window) { cl.diag = diag; cl.level = u.store; append = false; break; }
                        }
                    }
                    if (append) {
                        const uint32_t idx = (uint32_t)(i - b) + 1u;
                        pool[idx - 1] = DiagCell{diag, u.store, head};
                        hd[bk] = idx;
                    }
                    __syncwarp();  // this pass's chain updates before the next pass reads them
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------------------
// score-only X-drop DP: search/gapped.rs:124-337 (outer sequence a, inner sequence b)
// ---------------------------------------------------------------------------------------
struct RingBand {  // band cells b live at ring[b & (W-1)]; valid while the band is < W wide
    int2* ring;
    uint32_t mask;
    __device__ __forceinline__ int2 get(uint32_t b) const { return ring[b & mask]; }
    __device__ __forceinline__ void set(uint32_t b, int2 v) { ring[b & mask] = v; }
    __device__ __forceinline__ void set_best(uint32_t b, int32_t v) { ring[b & mask].x = v; }
    __device__ __forceinline__ bool fits(uint32_t b, uint32_t first_b) const { return b - first_b <= mask; }
};
struct FlatBand {  // band cells at absolute index b; capacity >= n + 2
    int2* cell;
    __device__ __forceinline__ int2 get(uint32_t b) const { return cell[b]; }
    __device__ __forceinline__ void set(uint32_t b, int2 v) { cell[b] = v; }
    __device__ __forceinline__ void set_best(uint32_t b, int32_t v) { cell[b].x = v; }
    __device__ __forceinline__ bool fits(uint32_t, uint32_t) const { return true; }
};

struct DpResult { int32_t score; uint32_t a_len, b_len; };

// Returns false if the band outgrew the storage.  b bytes are BLASTNA codes (0..15).
template <bool REVERSE, class Band>
__device__ bool so_dp(const uint8_t* __restrict__ a, const uint8_t* __restrict__ b, uint32_t m, uint32_t n, int32_t go,
                      int32_t ge, int32_t x_dropoff, const int32_t* __restrict__ mat, Band band, DpResult& res,
                      uint64_t& cells) {
    res = DpResult{0, 0, 0};
    if (m == 0 || n == 0) return true;
    const int32_t goe = go + ge;
    const int32_t xdrop = x_dropoff > goe ? x_dropoff : goe;
    band.set(0, make_int2(0, -goe));
    int32_t score = -goe;
    uint32_t b_size = 1;
    for (uint32_t j = 1; j <= n; ++j) {
        if (score < -xdrop) break;
        if (!band.fits(j, 0)) return false;
        band.set(j, make_int2(score, score - goe));
        score -= ge;
        b_size = j + 1;
    }
    int32_t best = 0;
    uint32_t best_a = 0, best_b = 0, first_b = 0;
    for (uint32_t ai = 0; ai < m; ++ai) {
        const uint32_t ap = REVERSE ? m - 1 - ai : ai;
        const int32_t* row = mat + ((a[ap] & 15) << 4);
        int32_t sc = MININT, gap_row = MININT;
        uint32_t last_b = first_b;
        const int32_t prev_best = best;
        cells += b_size - first_b;
        for (uint32_t bi = first_b; bi < b_size; ++bi) {
            const int2 c = band.get(bi);
            int32_t next_score = 0;
            if (bi < n) next_score = c.x + row[b[REVERSE ? n - 1 - bi : bi]];
            int32_t cell = sc;
            if (c.y > cell) cell = c.y;
            if (gap_row > cell) cell = gap_row;
            if (best - cell > xdrop) {
                if (bi == first_b) ++first_b;
                else band.set_best(bi, MININT);
            } else {
                last_b = bi;
                if (cell > best) { best_b = bi; best = cell; }
                gap_row -= ge;
                const int32_t open = cell - goe;
                const int32_t col_ext = c.y - ge;
                band.set(bi, make_int2(cell, col_ext > open ? col_ext : open));
                if (open > gap_row) gap_row = open;
            }
            sc = next_score;
        }
        if (best > prev_best) best_a = ai + 1;
        if (first_b >= b_size) break;
        if (last_b + 1 < b_size) {
            b_size = last_b + 1;
        } else {
            while (gap_row >= best - xdrop && b_size <= n) {
                if (!band.fits(b_size, first_b)) return false;
                band.set(b_size, make_int2(gap_row, gap_row - goe));
                gap_row -= ge;
                ++b_size;
            }
        }
        if (b_size <= n) {
            if (!band.fits(b_size, first_b)) return false;
            band.set(b_size, make_int2(MININT, MININT));
            ++b_size;
        }
    }
    res = DpResult{best, best_a, best_b};
    return true;
}

// ---------------------------------------------------------------------------------------
// Warp-cooperative score-only X-drop DP: the same rows as so_dp, each row computed by the 32
// lanes of a warp over consecutive band cells, in chunks of 32.
//
// Exactness.  In the reference's row loop (gapped.rs:222-296) the horizontal-gap value F
// decays by ge at every unpruned cell and keeps its value at a pruned one, and the prune test
// uses the running row-major best.  Let F* be the plain recurrence F*(b+1) =
// max(F*(b) - ge, t(b) - goe) applied at every cell, t = max(diagonal, vertical gap).  By
// induction over the row, at every cell either F = F* or both are below T = best - X (a pruned
// cell has F <= cell < T, so its frozen F stays below T and so does F*), hence
// max(t, F) and max(t, F*) agree on every cell that survives, on every prune decision, on the
// stored cells, on the end-of-row F that drives the band extension, and on the running best
// (pruned cells are below it).  F* is a max-plus prefix scan and the running best a prefix max,
// both warp scans.
// ---------------------------------------------------------------------------------------
// Number of band-extension cells of the row loops (gapped.rs:313-327): the i = 0, 1, ... with
// gap_row - i ge >= thr, at most `room`; gap_row >= thr.  Counted by ballot, 32 at a time.
__device__ __forceinline__ uint32_t ext_count(int32_t gap_row, int32_t thr, int32_t ge, uint32_t room) {
    const uint32_t lane = threadIdx.x & 31;
    uint32_t k = 0;
    for (;;) {
        const uint32_t i = k + lane;
        const bool ok = i < room && (int64_t)gap_row - (int64_t)i * ge >= (int64_t)thr;
        const unsigned m = __ballot_sync(0xffffffffu, ok);
        const uint32_t c = __popc(m);
        k += c;
        if (c < 32) return k;
    }
}

template <bool REVERSE, class Band>
__device__ bool so_dp_warp(const uint8_t* __restrict__ a, const uint8_t* __restrict__ b, uint32_t m, uint32_t n,
                           int32_t go, int32_t ge, int32_t x_dropoff, const int32_t* __restrict__ mat, Band band,
                           DpResult& res, uint64_t& cells) {
    const uint32_t lane = threadIdx.x & 31;
    const unsigned FULL = 0xffffffffu;
    res = DpResult{0, 0, 0};
    if (m == 0 || n == 0) return true;
    const int32_t goe = go + ge;
    const int32_t xdrop = x_dropoff > goe ? x_dropoff : goe;
    // first row: cells 0..J, J = min(n, (xdrop - goe) / ge + 1)
    const uint32_t J = min(n, (uint32_t)((xdrop - goe) / ge) + 1u);
    if (!band.fits(J, 0)) return false;
    for (uint32_t j = lane; j <= J; j += 32) {
        if (j == 0) band.set(0, make_int2(0, -goe));
        else {
            const int32_t sc = -goe - (int32_t)(j - 1) * ge;
            band.set(j, make_int2(sc, sc - goe));
        }
    }
    uint32_t b_size = J + 1, first_b = 0, best_a = 0, best_b = 0;
    int32_t best = 0;
    for (uint32_t ai = 0; ai < m; ++ai) {
        __syncwarp();
        const uint32_t ap = REVERSE ? m - 1 - ai : ai;
        const int32_t* row = mat + ((a[ap] & 15) << 4);
        cells += b_size - first_b;
        int32_t carry_h = MININT;   // old H of the cell left of the chunk
        int32_t carry_g = MININT;   // F* entering the chunk
        int32_t carry_best = best;  // running best entering the chunk
        int32_t row_max = MININT;
        uint32_t row_arg = 0, last_b = first_b, new_first = first_b;
        bool leading = true;
        for (uint32_t c0 = first_b; c0 < b_size; c0 += 32) {
            const uint32_t bi = c0 + lane;
            const bool valid = bi < b_size;
            const int2 cur = valid ? band.get(bi) : make_int2(MININT, MININT);
            int32_t hl = __shfl_up_sync(FULL, cur.x, 1);
            if (lane == 0) hl = carry_h;
            int32_t d = MININT;
            if (valid && bi != first_b) d = hl + row[b[REVERSE ? n - bi : bi - 1]];
            const int32_t t = valid ? (d > cur.y ? d : cur.y) : MININT;
            // Chunk maximum of t = chunk maximum of the cells (F* never exceeds an earlier t).
            const int32_t tmax = __reduce_max_sync(FULL, t);
            const int32_t thr = carry_best - xdrop;  // threshold at the chunk start (only rises)
            int32_t g, f;
            if (carry_g >= thr || tmax - goe >= thr) {
                // G(b) = max(G(b-1) - ge, t(b) - goe); F*(b) = G(b-1)
                // shfl_up hands a lane below the offset its own value, and max(g - k ge, g) = g,
                // so every lane takes the step
                g = valid ? t - goe : MININT;
#pragma unroll
                for (uint32_t k = 1; k < 32; k <<= 1) g = __viaddmax_s32(__shfl_up_sync(FULL, g, k), -(int32_t)k * ge, g);
                g = __viaddmax_s32(carry_g, -(int32_t)(lane + 1) * ge, g);
                f = __shfl_up_sync(FULL, g, 1);
                if (lane == 0) f = carry_g;
            } else {
                // every F* of the chunk is below the threshold: it decides nothing, and any value
                // below the threshold carried on leaves the later cells' decisions unchanged
                f = MININT;
                g = carry_g > tmax - goe ? carry_g : tmax - goe;
            }
            const int32_t cell = valid ? max(t, f) : MININT;
            // running best before this cell: max(carry_best, earlier t of the chunk)
            int32_t before = carry_best, mx = t;
            if (tmax > carry_best) {
#pragma unroll
                for (uint32_t k = 1; k < 32; k <<= 1) mx = max(mx, __shfl_up_sync(FULL, mx, k));
                const int32_t ex = __shfl_up_sync(FULL, mx, 1);
                if (lane != 0) before = max(before, ex);
            }
            const bool pruned = valid && (before - cell > xdrop);
            const bool alive = valid && !pruned;
            const unsigned alive_mask = __ballot_sync(FULL, alive);
            const unsigned valid_mask = __ballot_sync(FULL, valid);
            uint32_t lead_end = 0;  // lanes below this are in the leading pruned run
            if (leading) {
                if (alive_mask) {
                    lead_end = __ffs(alive_mask) - 1;
                    new_first += lead_end;
                    leading = false;
                } else {
                    lead_end = 32;
                    new_first += __popc(valid_mask);
                }
            }
            if (alive) band.set(bi, make_int2(cell, __viaddmax_s32(cur.y, -ge, cell - goe))); else if (pruned && lane >= lead_end) {
                band.set_best(bi, MININT);
            }
            if (alive_mask) last_b = c0 + 31 - __clz(alive_mask);
            if (tmax > row_max) {
                row_max = tmax;
                row_arg = c0 + __ffs(__ballot_sync(FULL, valid && t == tmax)) - 1;
            }
            if (tmax > carry_best) carry_best = tmax;
            const uint32_t last_lane = 31 - __clz(valid_mask);
            carry_g = __shfl_sync(FULL, g, last_lane);
            carry_h = __shfl_sync(FULL, cur.x, 31);
        }
        first_b = new_first;
        if (row_max > best) {
            best = row_max;
            best_b = row_arg;
            best_a = ai + 1;
        }
        if (first_b >= b_size) break;
        int32_t gap_row = carry_g;
        if (last_b + 1 < b_size) {
            b_size = last_b + 1;
        } else if (gap_row >= best - xdrop && b_size <= n) {
            const uint32_t k = ext_count(gap_row, best - xdrop, ge, n + 1 - b_size);
            if (!band.fits(b_size + k - 1, first_b)) return false;
            __syncwarp();
            for (uint32_t i = lane; i < k; i += 32) {
                const int32_t v = gap_row - (int32_t)i * ge;
                band.set(b_size + i, make_int2(v, v - goe));
            }
            b_size += k;
        }
        if (b_size <= n) {
            if (!band.fits(b_size, first_b)) return false;
            if (lane == 0) band.set(b_size, make_int2(MININT, MININT));
            ++b_size;
        }
    }
    res = DpResult{best, best_a, best_b};
    return true;
}

// engine.rs:1850-1895 prelim_pivot: (pivot_q, pivot_s, tb_q, tb_s)
__device__ __forceinline__ void prelim_pivot(bool plus, uint32_t q_seed, uint32_t s_seed, uint32_t s_start,
                                             uint32_t s_end, uint32_t qa, uint32_t sa, uint32_t lw, uint32_t o[4]) {
    if (plus) {
        uint32_t tq = q_seed, ts = s_seed;
        if (s_end >= s_seed + 8) { tq += 3; ts += 3; }
        const uint32_t oa = 4 - (ts % 4);
        uint32_t ps = ts + oa, pq = tq + oa;
        if (ps >= sa || pq >= qa) { ps -= 4; pq -= 4; }
        o[0] = pq; o[1] = ps; o[2] = tq; o[3] = ts;
    } else {
        const uint32_t saved = sa - s_seed - lw;
        const uint32_t s_end_fwd = sa - s_start;
        const bool ext = s_end_fwd >= saved + 8;
        uint32_t tq = q_seed, ts = s_seed;
        if (ext) { tq = q_seed + lw - 4; ts = s_seed + lw - 4; }
        const uint32_t shift = ext ? 3 : 0;
        const uint32_t qn = (qa - q_seed - lw) + shift, sn = (sa - s_seed - lw) + shift;
        const uint32_t oa = 4 - (sn % 4);
        uint32_t ql = qn + oa, sl = sn + oa;
        if (ql > qa || sl > sa) { ql -= 4; sl -= 4; }
        o[0] = ql; o[1] = sl; o[2] = tq; o[3] = ts;
    }
}

// One record of engine.rs:1350-1397: pivot, X = min(xdrop_gap, ungapped score), the two
// score-only extensions (gapped.rs:360-418), frame conversion and the gapped cutoff.
template <class BandL, class BandR>
__device__ bool prelim_one(const DevLib& L, const DevQueries& Q, const DevParams* P, const int32_t* mat,
                           uint32_t pair, const SeedHit h, const UngBox u, BandL bl, BandR br, PrelimOut& out,
                           uint64_t& cells) {
    const uint32_t qi = pair / L.n, si = pair % L.n;
    const uint32_t qa = Q.len[qi], sa = L.len[si];
    const bool plus = !(h.qs >> 31);
    uint32_t piv[4];
    prelim_pivot(plus, h.qs & 0x7fffffffu, h.s, u.s_start, u.s_end, qa, sa, (uint32_t)Q.lw[qi], piv);
    const int32_t xd = P->xdrop_gap < u.score ? P->xdrop_gap : u.score;
    const uint8_t* qseq = (plus ? Q.q : Q.qrc) + Q.off[qi] + 1;
    const uint8_t* sseq = L.plus + L.plus_off[si] + 1;
    const uint32_t qp = piv[0], sp = piv[1];
    DpResult l, r{0, 0, 0};
    if (!so_dp<true>(sseq, qseq, sp, qp, P->gap_open, P->gap_extend, xd, mat, bl, l, cells)) return false;
    const uint32_t rm = sa > sp ? sa - sp : 0, rn = qa > qp ? qa - qp : 0;
    if (rm > 0 && rn > 0)
        if (!so_dp<false>(sseq + sp, qseq + qp, rm, rn, P->gap_open, P->gap_extend, xd, mat, br, r, cells)) return false;
    const int32_t total = l.score + r.score;
    out.score = INT32_MIN;
    if (total < 0) return true;
    uint32_t q0 = qp - l.b_len, s0 = sp - l.a_len, q1 = qp + r.b_len, s1 = sp + r.a_len;
    if (!plus) {
        const uint32_t t0 = qa - q1, t1 = qa - q0, t2 = sa - s1, t3 = sa - s0;
        q0 = t0; q1 = t1; s0 = t2; s1 = t3;
    }
    if (total < P->gapped_cutoff) return true;
    out = PrelimOut{total, q0, q1, s0, s1, piv[2], piv[3]};
    return true;
}

template <int W>
__global__ void __launch_bounds__(128) k_prelim(DevLib L, DevQueries Q, const DevParams* __restrict__ P, uint64_t n,
                                                 const uint32_t* __restrict__ idx, const SeedHit* __restrict__ hits,
                                                 const uint32_t* __restrict__ hit_pair, const UngBox* __restrict__ ub,
                                                 PrelimOut* __restrict__ out, uint32_t* __restrict__ wide,
                                                 unsigned int* __restrict__ n_wide,
                                                 unsigned long long* __restrict__ cells_total) {
    extern __shared__ int2 smem_ring[];
    __shared__ int32_t mat[256];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) mat[i] = P->matrix[i];
    __syncthreads();
    RingBand band{smem_ring + threadIdx.x * W, W - 1};
    uint64_t cells = 0;
    for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t i = idx[t];
        PrelimOut o{INT32_MIN, 0, 0, 0, 0, 0, 0};
        uint64_t c = 0;
        if (prelim_one(L, Q, P, mat, hit_pair[i], hits[i], ub[i], band, band, o, c)) {
            out[t] = o;
            cells += c;
        } else {
            const unsigned int k = atomicAdd(n_wide, 1u);
            wide[k] = (uint32_t)t;
        }
    }
    for (int o = 16; o; o >>= 1) cells += __shfl_down_sync(0xffffffffu, cells, o);
    if ((threadIdx.x & 31) == 0 && cells) atomicAdd(cells_total, (unsigned long long)cells);
}

// One ungapped record per warp (records list[0..n), or 0..n without a list); each warp's band
// lives in a RING_W-cell shared-memory ring.
template <int RING_W>
__global__ void __launch_bounds__(256) k_prelim_warp(DevLib L, DevQueries Q, const DevParams* __restrict__ P,
                                                      uint64_t n, const uint32_t* __restrict__ idx,
                                                      const SeedHit* __restrict__ hits,
                                                      const uint32_t* __restrict__ hit_pair,
                                                      const UngBox* __restrict__ ub, PrelimOut* __restrict__ out,
                                                      const uint32_t* __restrict__ list,
                                                      uint32_t* __restrict__ wide, unsigned int* __restrict__ n_wide,
                                                      unsigned long long* __restrict__ cells_total) {
    __shared__ int2 ring[(256 / 32) * RING_W];
    __shared__ int32_t mat[256];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) mat[i] = P->matrix[i];
    __syncthreads();
    const uint32_t lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    RingBand band{ring + wib * RING_W, RING_W - 1};
    uint64_t cells = 0;
    const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t k = warp; k < n; k += nwarps) {
        const uint64_t t = list ? list[k] : k;
        const uint32_t i = idx[t];
        const uint32_t pair = hit_pair[i];
        const SeedHit h = hits[i];
        const UngBox u = ub[i];
        const uint32_t qi = pair / L.n, si = pair % L.n;
        const uint32_t qa = Q.len[qi], sa = L.len[si];
        const bool plus = !(h.qs >> 31);
        uint32_t piv[4];
        prelim_pivot(plus, h.qs & 0x7fffffffu, h.s, u.s_start, u.s_end, qa, sa, (uint32_t)Q.lw[qi], piv);
        const int32_t xd = P->xdrop_gap < u.score ? P->xdrop_gap : u.score;
        const uint8_t* qseq = (plus ? Q.q : Q.qrc) + Q.off[qi] + 1;
        const uint8_t* sseq = L.plus + L.plus_off[si] + 1;
        const uint32_t qp = piv[0], sp = piv[1];
        DpResult l, r{0, 0, 0};
        uint64_t c = 0;
        bool ok = so_dp_warp<true>(sseq, qseq, sp, qp, P->gap_open, P->gap_extend, xd, mat, band, l, c);
        const uint32_t rm = sa > sp ? sa - sp : 0, rn = qa > qp ? qa - qp : 0;
        if (ok && rm > 0 && rn > 0)
            ok = so_dp_warp<false>(sseq + sp, qseq + qp, rm, rn, P->gap_open, P->gap_extend, xd, mat, band, r, c);
        if (!ok) {
            if (lane == 0) wide[atomicAdd(n_wide, 1u)] = (uint32_t)t;
            continue;
        }
        cells += c;
        if (lane == 0) {
            PrelimOut o{INT32_MIN, 0, 0, 0, 0, 0, 0};
            const int32_t total = l.score + r.score;
            if (total >= 0) {
                uint32_t q0 = qp - l.b_len, s0 = sp - l.a_len, q1 = qp + r.b_len, s1 = sp + r.a_len;
                if (!plus) {
                    const uint32_t t0 = qa - q1, t1 = qa - q0, t2 = sa - s1, t3 = sa - s0;
                    q0 = t0; q1 = t1; s0 = t2; s1 = t3;
                }
                if (total >= P->gapped_cutoff) o = PrelimOut{total, q0, q1, s0, s1, piv[2], piv[3]};
            }
            out[t] = o;
        }
    }
    if (lane == 0 && cells) atomicAdd(cells_total, (unsigned long long)cells);
}

// Geometry of one ungapped record's preliminary DP (engine.rs:1350-1372).
struct RecGeom {
    bool plus;
    uint32_t qa, sa, qp, sp, tbq, tbs;
    int32_t xd;
    const uint8_t *qseq, *sseq;
};
__device__ __forceinline__ RecGeom rec_geom(const DevLib& L, const DevQueries& Q, const DevParams* P, uint32_t i,
                                            const SeedHit* hits, const uint32_t* hit_pair, const UngBox* ub) {
    const uint32_t pair = hit_pair[i];
    const SeedHit h = hits[i];
    const UngBox u = ub[i];
    const uint32_t qi = pair / L.n, si = pair % L.n;
    RecGeom g;
    g.qa = Q.len[qi];
    g.sa = L.len[si];
    g.plus = !(h.qs >> 31);
    uint32_t piv[4];
    prelim_pivot(g.plus, h.qs & 0x7fffffffu, h.s, u.s_start, u.s_end, g.qa, g.sa, (uint32_t)Q.lw[qi], piv);
    g.xd = P->xdrop_gap < u.score ? P->xdrop_gap : u.score;
    g.qseq = (g.plus ? Q.q : Q.qrc) + Q.off[qi] + 1;
    g.sseq = L.plus + L.plus_off[si] + 1;
    g.qp = piv[0]; g.sp = piv[1]; g.tbq = piv[2]; g.tbs = piv[3];
    return g;
}

// The records list[0..n_list) with each of their two extensions on its own warp: task 2k is
// record list[k]'s left extension, 2k + 1 its right one.  Results (score, a_len, b_len, ok) go
// to dres[task]; k_prelim_combine joins them.  These are the records the thread kernel passed
// on, a few of them thousands of rows long, so the launch lasts as long as its longest
// extension and not its longest record.
template <int RING_W>
__global__ void __launch_bounds__(256) k_prelim_warp_dir(DevLib L, DevQueries Q, const DevParams* __restrict__ P,
                                                          uint32_t n_list, const uint32_t* __restrict__ list,
                                                          const uint32_t* __restrict__ idx,
                                                          const SeedHit* __restrict__ hits,
                                                          const uint32_t* __restrict__ hit_pair,
                                                          const UngBox* __restrict__ ub, int4* __restrict__ dres,
                                                          unsigned long long* __restrict__ cells_total,
                                                          const unsigned int* __restrict__ n_dev) {
    if (n_dev) n_list = min(*n_dev, n_list);  // the count on the device, n_list the list's capacity
    __shared__ int2 ring[(256 / 32) * RING_W];
    __shared__ int32_t mat[256];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) mat[i] = P->matrix[i];
    __syncthreads();
    const uint32_t lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    RingBand band{ring + wib * RING_W, RING_W - 1};
    uint64_t cells = 0;
    const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t k = warp; k < 2ull * n_list; k += nwarps) {
        const RecGeom g = rec_geom(L, Q, P, idx[list[k >> 1]], hits, hit_pair, ub);
        DpResult r{0, 0, 0};
        uint64_t c = 0;
        bool ok = true;
        if (!(k & 1)) {
            ok = so_dp_warp<true>(g.sseq, g.qseq, g.sp, g.qp, P->gap_open, P->gap_extend, g.xd, mat, band, r, c);
        } else {
            const uint32_t rm = g.sa > g.sp ? g.sa - g.sp : 0, rn = g.qa > g.qp ? g.qa - g.qp : 0;
            if (rm > 0 && rn > 0)
                ok = so_dp_warp<false>(g.sseq + g.sp, g.qseq + g.qp, rm, rn, P->gap_open, P->gap_extend, g.xd, mat,
                                       band, r, c);
        }
        if (ok) cells += c;
        if (lane == 0) dres[k] = make_int4(r.score, (int32_t)r.a_len, (int32_t)r.b_len, ok ? 1 : 0);
    }
    if (lane == 0 && cells) atomicAdd(cells_total, (unsigned long long)cells);
}

// Joins k_prelim_warp_dir's two extensions of each listed record (engine.rs:1380-1397); a record
// with an extension wider than the warp ring goes to `wide`.
__global__ void k_prelim_combine(DevLib L, DevQueries Q, const DevParams* __restrict__ P, uint32_t n_list,
                                 const uint32_t* __restrict__ list, const uint32_t* __restrict__ idx,
                                 const SeedHit* __restrict__ hits, const uint32_t* __restrict__ hit_pair,
                                 const UngBox* __restrict__ ub, const int4* __restrict__ dres,
                                 PrelimOut* __restrict__ out, uint32_t* __restrict__ wide,
                                 unsigned int* __restrict__ n_wide, const unsigned int* __restrict__ n_dev) {
    if (n_dev) n_list = min(*n_dev, n_list);
    const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n_list) return;
    const uint32_t t = list[k];
    const int4 l = dres[2 * k], r = dres[2 * k + 1];
    if (!l.w || !r.w) {
        wide[atomicAdd(n_wide, 1u)] = t;
        return;
    }
    const RecGeom g = rec_geom(L, Q, P, idx[t], hits, hit_pair, ub);
    PrelimOut o{INT32_MIN, 0, 0, 0, 0, 0, 0};
    const int32_t total = l.x + r.x;
    if (total >= 0) {
        uint32_t q0 = g.qp - (uint32_t)l.z, s0 = g.sp - (uint32_t)l.y, q1 = g.qp + (uint32_t)r.z,
                 s1 = g.sp + (uint32_t)r.y;
        if (!g.plus) {
            const uint32_t t0 = g.qa - q1, t1 = g.qa - q0, t2 = g.sa - s1, t3 = g.sa - s0;
            q0 = t0; q1 = t1; s0 = t2; s1 = t3;
        }
        if (total >= P->gapped_cutoff) o = PrelimOut{total, q0, q1, s0, s1, g.tbq, g.tbs};
    }
    out[t] = o;
}

// The records whose band outgrew the ring, with the band at absolute indices in global memory
// (`band_cap` cells per thread, at least the longest inner sequence + 2).
__global__ void __launch_bounds__(128) k_prelim_wide(DevLib L, DevQueries Q, const DevParams* __restrict__ P,
                                                      uint32_t n_wide, const uint32_t* __restrict__ wide,
                                                      const uint32_t* __restrict__ idx, const SeedHit* __restrict__ hits,
                                                      const uint32_t* __restrict__ hit_pair,
                                                      const UngBox* __restrict__ ub, PrelimOut* __restrict__ out,
                                                      int2* __restrict__ band_mem, uint64_t band_cap,
                                                      unsigned long long* __restrict__ cells_total,
                                                      unsigned int* __restrict__ failures,
                                                      const unsigned int* __restrict__ n_dev) {
    if (n_dev) n_wide = min(*n_dev, n_wide);
    __shared__ int32_t mat[256];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) mat[i] = P->matrix[i];
    __syncthreads();
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    FlatBand band{band_mem + tid * band_cap};
    uint64_t cells = 0;
    for (uint64_t k = tid; k < n_wide; k += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t t = wide[k];
        const uint32_t i = idx[t];
        PrelimOut o{INT32_MIN, 0, 0, 0, 0, 0, 0};
        uint64_t c = 0;
        if (!prelim_one(L, Q, P, mat, hit_pair[i], hits[i], ub[i], band, band, o, c)) atomicAdd(failures, 1u);
        out[t] = o;
        cells += c;
    }
    if (cells) atomicAdd(cells_total, (unsigned long long)cells);
}

// ---------------------------------------------------------------------------------------
// Learned schedule (rmb_sched.cuh): the features of an ungapped record, the network's cost
// prediction for every record, and the records in descending predicted cost.
// ---------------------------------------------------------------------------------------
// The 12 raw features of record i (a hit index): ungapped score / 100, log1p ungapped extent,
// log1p of the room left and right of the pivot on each sequence, X / 100, strand, GC fraction of
// ~32 subject bases at the pivot (packed bytes), ungapped score per base, log1p of the pair's word
// hits, log1p of the diagonal room (min of the two sides' rooms, left plus right).
__device__ __forceinline__ void sched_features(const DevLib& L, const DevQueries& Q, const DevParams* P, uint32_t i,
                                               const SeedHit* hits, const uint32_t* hit_pair, const UngBox* ub,
                                               const uint32_t* pair_hits, float f[SCHED_NF]) {
    const RecGeom g = rec_geom(L, Q, P, i, hits, hit_pair, ub);
    const UngBox u = ub[i];
    const uint32_t ext = u.s_end - u.s_start;
    f[0] = (float)u.score * 0.01f;
    f[1] = log1pf((float)ext);
    f[2] = log1pf((float)g.qp);
    f[3] = log1pf((float)g.sp);
    f[4] = log1pf((float)(g.qa - g.qp));
    f[5] = log1pf((float)(g.sa - g.sp));
    f[6] = (float)g.xd * 0.01f;
    f[7] = g.plus ? 1.0f : 0.0f;
    {
        const uint32_t si = hit_pair[i] % L.n;
        const uint8_t* pk = L.packed + L.packed_off[si];
        const uint32_t nbytes = (g.sa + 3) / 4;
        const uint32_t b1 = min(nbytes, g.sp / 4 + 4), b0 = b1 > 8 ? b1 - 8 : 0;
        uint32_t gc = 0;
        for (uint32_t b = b0; b < b1; ++b) {
            const uint32_t x = pk[b];
            gc += __popc((x ^ (x >> 1)) & 0x55u);  // 2-bit codes 1 (C) and 2 (G)
        }
        f[8] = b1 > b0 ? (float)gc / (float)(4 * (b1 - b0)) : 0.5f;
    }
    f[9] = (float)u.score / (float)(ext > 0 ? ext : 1);
    f[10] = log1pf((float)pair_hits[hit_pair[i]]);
    f[11] = log1pf((float)(min(g.qp, g.sp) + min(g.qa - g.qp, g.sa - g.sp)));
}

__global__ void __launch_bounds__(256) k_sched_features(DevLib L, DevQueries Q, const DevParams* __restrict__ P,
                                                         uint64_t n, const uint32_t* __restrict__ idx,
                                                         const SeedHit* __restrict__ hits,
                                                         const uint32_t* __restrict__ hit_pair,
                                                         const UngBox* __restrict__ ub,
                                                         const uint32_t* __restrict__ pair_hits, float* __restrict__ out) {
    for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (uint64_t)gridDim.x * blockDim.x) {
        float f[SCHED_NF];
        sched_features(L, Q, P, idx[t], hits, hit_pair, ub, pair_hits, f);
#pragma unroll
        for (int k = 0; k < SCHED_NF; ++k) out[t * SCHED_NF + k] = f[k];
    }
}

// Predictions for records 0..n): from the records themselves (feats null) or from given raw
// features (n x 12); the histogram of cost bins is added to hist[SCHED_BINS] when hist is set.
// Warps take 32 consecutive records at a time, so every lane reaches the warp-wide network.
constexpr int SCHED_BLOCK = 128;
__global__ void __launch_bounds__(SCHED_BLOCK) k_sched_predict(DevLib L, DevQueries Q, const DevParams* __restrict__ P,
                                                                uint64_t n, const uint32_t* __restrict__ idx,
                                                                const SeedHit* __restrict__ hits,
                                                                const uint32_t* __restrict__ hit_pair,
                                                                const UngBox* __restrict__ ub,
                                                                const uint32_t* __restrict__ pair_hits,
                                                                const float* __restrict__ feats,
                                                                const float* __restrict__ params,
                                                                float* __restrict__ pred, unsigned int* __restrict__ hist,
                                                                const unsigned int* __restrict__ n_dev) {
    if (n_dev) n = *n_dev;
    __shared__ SchedSmem S;
    __shared__ __align__(16) uint16_t xs[SCHED_BLOCK / 32][32][16];
    __shared__ float ys[SCHED_BLOCK / 32][32];
    __shared__ unsigned int h[SCHED_BINS];
    sched_load(S, params);
    for (int i = threadIdx.x; i < SCHED_BINS; i += blockDim.x) h[i] = 0;
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint64_t nwarps = (uint64_t)gridDim.x * (SCHED_BLOCK / 32);
    for (uint64_t base = ((uint64_t)blockIdx.x * (SCHED_BLOCK / 32) + warp) * 32; base < n; base += nwarps * 32) {
        const uint64_t t = base + lane;
        float f[SCHED_NF];
        if (t < n) {
            if (feats) {
#pragma unroll
                for (int k = 0; k < SCHED_NF; ++k) f[k] = feats[t * SCHED_NF + k];
            } else {
                sched_features(L, Q, P, idx[t], hits, hit_pair, ub, pair_hits, f);
            }
#pragma unroll
            for (int k = 0; k < SCHED_NF; ++k) f[k] = (f[k] - S.mean[k]) * S.istd[k];
        } else {
#pragma unroll
            for (int k = 0; k < SCHED_NF; ++k) f[k] = 0.0f;
        }
        const float y = sched_mlp_warp(S, xs[warp], ys[warp], f);
        if (t < n) {
            pred[t] = y;
            if (hist) atomicAdd(&h[sched_bin(y)], 1u);
        }
    }
    if (hist) {
        __syncthreads();
        for (int i = threadIdx.x; i < SCHED_BINS; i += blockDim.x)
            if (h[i]) atomicAdd(&hist[i], h[i]);
    }
}

// Start of each cost bin in the order, costliest bin first; fill[] zeroed for the scatter.
__global__ void k_sched_binstart(const unsigned int* __restrict__ hist, unsigned int* __restrict__ start,
                                 unsigned int* __restrict__ fill) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    unsigned int acc = 0;
    for (int b = SCHED_BINS - 1; b >= 0; --b) {
        start[b] = acc;
        acc += hist[b];
        fill[b] = 0;
    }
}

// order[start[bin] + k] = record: each block ranks a tile of records per bin in shared memory and
// takes its stretch of every bin with one global atomic (order within a bin is arbitrary).
constexpr int SCHED_TILE_PER_THREAD = 16;
__global__ void __launch_bounds__(256) k_sched_scatter(uint64_t n, const float* __restrict__ pred,
                                                        const unsigned int* __restrict__ start,
                                                        unsigned int* __restrict__ fill, uint32_t* __restrict__ order) {
    __shared__ unsigned int cnt[SCHED_BINS], base[SCHED_BINS];
    const uint64_t tile = (uint64_t)blockDim.x * SCHED_TILE_PER_THREAD;
    for (uint64_t t0 = (uint64_t)blockIdx.x * tile; t0 < n; t0 += (uint64_t)gridDim.x * tile) {
        for (int i = threadIdx.x; i < SCHED_BINS; i += blockDim.x) cnt[i] = 0;
        __syncthreads();
        uint32_t bin[SCHED_TILE_PER_THREAD], rank[SCHED_TILE_PER_THREAD];
#pragma unroll
        for (int j = 0; j < SCHED_TILE_PER_THREAD; ++j) {
            const uint64_t t = t0 + (uint64_t)j * blockDim.x + threadIdx.x;
            bin[j] = t < n ? sched_bin(pred[t]) : 0u;
            rank[j] = t < n ? atomicAdd(&cnt[bin[j]], 1u) : 0u;
        }
        __syncthreads();
        for (int i = threadIdx.x; i < SCHED_BINS; i += blockDim.x)
            base[i] = cnt[i] ? start[i] + atomicAdd(&fill[i], cnt[i]) : 0u;
        __syncthreads();
#pragma unroll
        for (int j = 0; j < SCHED_TILE_PER_THREAD; ++j) {
            const uint64_t t = t0 + (uint64_t)j * blockDim.x + threadIdx.x;
            if (t < n) order[base[bin[j]] + rank[j]] = (uint32_t)t;
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------------------
// Thread-per-extension score-only X-drop DP: the body is prelim_stream_thread
// (rmb_prelim_stream.cuh), shared with a host build of the same code.
// ---------------------------------------------------------------------------------------

__global__ void __launch_bounds__(256) k_prelim_prep(DevLib L, DevQueries Q, const DevParams* __restrict__ P,
                                                      uint64_t n, const uint32_t* __restrict__ idx,
                                                      const SeedHit* __restrict__ hits,
                                                      const uint32_t* __restrict__ hit_pair,
                                                      const UngBox* __restrict__ ub, PrelimGeo* __restrict__ geo,
                                                      const unsigned int* __restrict__ n_dev) {
    if (n_dev) n = *n_dev;  // the count on the device (a graph-captured chain), n its capacity
    const int32_t goe = P->gap_open + P->gap_extend;
    for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (uint64_t)gridDim.x * blockDim.x) {
        const RecGeom g = rec_geom(L, Q, P, idx[t], hits, hit_pair, ub);
        const uint8_t al = g.sp > 0 ? g.sseq[g.sp - 1] : 0, ar = g.sa > g.sp ? g.sseq[g.sp] : 0;
        PrelimGeo o;
        o.qseq = (uint64_t)g.qseq;
        o.sseq = (uint64_t)g.sseq;
        o.qa = g.qa; o.sa = g.sa; o.qp = g.qp; o.sp = g.sp;
        o.tbq = g.tbq; o.tbs = g.tbs;
        o.xdrop = (uint32_t)(g.xd > goe ? g.xd : goe);
        o.flags = (g.plus ? 1u : 0u) | ((uint32_t)al << 8) | ((uint32_t)ar << 16);
        geo[t] = o;
    }
}

// The ring of a block: band entry j of thread x at ring[(j % STREAM_RING) * STREAM_BLOCK + x], so
// the threads of a warp touch 32 consecutive words whatever their band indices.  QUEUE: records
// come from a grid-wide queue (the batched pipeline's persistent grid); otherwise thread i runs
// record i alone (the plain pipeline's one record per thread).
template <bool QUEUE>
struct StreamDevEnv {
    uint32_t* my;
    unsigned int *queue, *n_wide;
    uint32_t* wide;
    bool taken = false;
    __device__ __forceinline__ uint32_t& at(uint32_t j) { return my[(j % STREAM_RING) * STREAM_BLOCK]; }
    __device__ __forceinline__ uint32_t take() {
        if (QUEUE) return atomicAdd(queue, 1u);
        const uint32_t t = taken ? 0xFFFFFFFFu : blockIdx.x * STREAM_BLOCK + threadIdx.x;
        taken = true;
        return t;
    }
    __device__ __forceinline__ void overflow(uint32_t t) { wide[atomicAdd(n_wide, 1u)] = t; }
    __device__ __forceinline__ bool any(bool p) { return __any_sync(0xffffffffu, p); }
    // the initial-row residues of every lane that started an extension: lane k copies index k
    // (and k + 32) into that lane's ring, so the byte loads of one row go out together
    __device__ __forceinline__ void fill_rows(bool pending, const uint8_t* qal, int32_t pb, int32_t dir, uint32_t n) {
        unsigned need = __ballot_sync(0xffffffffu, pending);
        if (!need) return;
        const int lane = threadIdx.x & 31;
        while (need) {
            const int L = __ffs(need) - 1;
            need &= need - 1;
            const uint8_t* q = (const uint8_t*)__shfl_sync(0xffffffffu, (unsigned long long)qal, L);
            const int32_t p = __shfl_sync(0xffffffffu, pb, L), d = __shfl_sync(0xffffffffu, dir, L);
            const uint32_t c = __shfl_sync(0xffffffffu, n, L);
            uint32_t* ringL = my - lane + L;
            for (uint32_t k = lane; k < c; k += 32) ringL[(k % STREAM_RING) * STREAM_BLOCK] = q[p + d * (int32_t)k] & 15u;
        }
        __syncwarp();
    }
};

template <int U, bool QUEUE>
__global__ void __launch_bounds__(STREAM_BLOCK, STREAM_BLOCKS_PER_SM)
k_prelim_stream(const DevParams* __restrict__ P, uint64_t n, const PrelimGeo* __restrict__ geo,
                PrelimOut* __restrict__ out,
                uint32_t* __restrict__ wide, unsigned int* __restrict__ n_wide, unsigned int* __restrict__ queue,
                unsigned long long* __restrict__ cells_total, uint32_t max_cells,
                const uint32_t* __restrict__ order, uint32_t* __restrict__ cells_out, uint32_t window,
                StreamDevCounts dc, uint32_t budget_div) {
    __shared__ uint32_t ring[STREAM_RING * STREAM_BLOCK];
    __shared__ int32_t smat[256];
    {
        // scores below -(X + 1), X the largest X-drop of any record, only ever make a diagonal
        // value below the threshold (a stored cell never exceeds the running best), so they are
        // all held as -(X + 1), which keeps every sum far from overflow
        const int32_t xmax = max(P->xdrop_gap, P->gap_open + P->gap_extend);
        for (int i = threadIdx.x; i < 256; i += blockDim.x) smat[i] = max(P->matrix[i], -(xmax + 1));
    }
    __syncthreads();
    StreamDevEnv<QUEUE> env{ring + threadIdx.x, queue, n_wide, wide};
    if (dc.n) {
        // the record count on the device (a graph-captured chain): the cell budget follows from it
        n = *dc.n;
        if (!order) {
            const uint64_t b = n / budget_div;
            max_cells = (uint32_t)(b < STREAM_MIN_CELLS ? STREAM_MIN_CELLS : b > STREAM_MAX_CELLS ? STREAM_MAX_CELLS : b);
        }
    }
    StreamArgs A{smat, P->gap_extend, P->gap_open + P->gap_extend, P->gapped_cutoff, n, geo, out, max_cells,
                 order, cells_out, window};
    if (dc.n_front) {
        A.n_front = *dc.n_front;
        A.order_end = dc.order_end;
    }
    const unsigned long long cells = prelim_stream_thread<U>(A, env);
    if (cells) atomicAdd(cells_total, cells);
}

// ---------------------------------------------------------------------------------------
// traceback: engine.rs:383-572 improve_seed, search/gapped.rs:450-757 align_ex +
// traceback_flat, engine.rs:2953-3039 gapped_extend_bidirectional
// ---------------------------------------------------------------------------------------
constexpr uint8_t T_GAP_A = 0, T_SUB = 3, T_GAP_B = 6, T_MASK = 7, T_EXT_A = 0x10, T_EXT_B = 0x40;

__device__ __forceinline__ uint32_t satsub(uint32_t a, uint32_t b) { return a > b ? a - b : 0; }

__device__ void improve_seed(const uint8_t* query, uint32_t qlen, const uint8_t* subject, uint32_t slen, uint32_t q_seed,
                             uint32_t s_seed, uint32_t pqs, uint32_t pqe, uint32_t pss, uint32_t pse, bool minus,
                             uint32_t& oq, uint32_t& os) {
    const int32_t RUN = 10;
    const int32_t hmax = 15;  // (int)(10 * 1.5)
    oq = q_seed;
    os = s_seed;
    if (!minus) {
        int32_t score = -1;
        uint32_t qf = q_seed, sf = s_seed;
        while (qf < pqe && qf < qlen && sf < slen && query[qf] == subject[sf]) {
            if (++score > RUN) return;
            ++qf;
            ++sf;
        }
        uint32_t qb = q_seed, sb = s_seed;
        for (;;) {
            if (query[qb] != subject[sb]) break;
            if (++score > RUN) return;
            if (qb == 0 || sb == 0) break;
            --qb;
            --sb;
        }
        const uint32_t offset = min(satsub(q_seed, pqs), satsub(s_seed, pss));
        const uint32_t sqs = q_seed - offset, sss = s_seed - offset;
        const uint32_t qn = min(satsub(pse, sss), satsub(pqe, sqs));
        int32_t max_score = 0, sc = 0;
        uint32_t max_off = sqs;
        bool is_match = false, prev = false;
        for (uint32_t i = 0; i < qn; ++i) {
            const uint32_t qi = sqs + i, si = sss + i;
            if (qi >= qlen || si >= slen) break;
            is_match = query[qi] == subject[si];
            if (is_match != prev) {
                prev = is_match;
                if (is_match) sc = 1;
                else if (sc > max_score) { max_score = sc; max_off = qi - (uint32_t)(sc / 2); }
            } else if (is_match) {
                if (++sc > hmax) {
                    const uint32_t nq = qi - (uint32_t)(hmax / 2);
                    oq = nq;
                    os = sss + (nq - sqs);
                    return;
                }
            }
        }
        if (is_match && sc > max_score) {
            max_score = sc;
            max_off = sqs + qn - (uint32_t)(sc / 2);
        }
        if (max_score > 0) {
            oq = max_off;
            os = sss + (max_off - sqs);
        }
        return;
    }
    int32_t score = -1;
    uint32_t qf = q_seed, sf = s_seed;
    while (qf < qlen && sf < slen && query[qf] == subject[sf]) {
        if (++score > RUN) return;
        ++qf;
        ++sf;
    }
    uint32_t qb = q_seed, sb = s_seed;
    for (;;) {
        if (query[qb] != subject[sb]) break;
        if (++score > RUN) return;
        if (qb <= pqs || sb == 0) break;
        --qb;
        --sb;
    }
    const uint32_t offset = min(satsub(satsub(pqe, 1), q_seed), satsub(satsub(pse, 1), s_seed));
    const uint32_t top_q = q_seed + offset, top_s = s_seed + offset;
    const uint32_t qn = min(satsub(top_q, pqs) + 1, satsub(top_s, pss) + 1);
    int32_t max_score = 0, sc = 0;
    int64_t max_off = q_seed;
    bool is_match = false, prev = false;
    for (uint32_t i = 0; i < qn; ++i) {
        const uint32_t qi = top_q - i, si = top_s - i;
        if (qi >= qlen || si >= slen) continue;
        is_match = query[qi] == subject[si];
        if (is_match != prev) {
            prev = is_match;
            if (is_match) sc = 1;
            else if (sc > max_score) { max_score = sc; max_off = (int64_t)qi + sc / 2; }
        } else if (is_match) {
            if (++sc > hmax) {
                const uint32_t nq = qi + (uint32_t)(hmax / 2);
                oq = nq;
                os = top_s - (top_q - nq);
                return;
            }
        }
    }
    if (is_match && sc > max_score) {
        max_score = sc;
        max_off = (int64_t)top_q - (int64_t)qn + sc / 2;
    }
    if (max_score > 0) {
        if (max_off < 0) return;
        const int64_t delta = (int64_t)top_q - max_off;
        int64_t ns = (int64_t)top_s - delta;
        if (ns < 0) ns = 0;
        oq = (uint32_t)max_off;
        os = (uint32_t)ns;
    }
}

// Per-thread traceback scratch: the band (absolute indices), the row table and the trace
// bytes.  Any write past a capacity sets `overflow` and the DP stops.
struct TbScratch {
    int2* band;
    uint2* rows;     // (byte offset of the row, first_b of the row)
    uint32_t rows_cap;
    uint8_t* trace;
    uint64_t trace_cap;
};

// search/gapped.rs:450-689 align_ex (a = query outer, b = subject inner) and 692-757
// traceback_flat.  Writes the script in reverse order (last op first) into ops_rev.
// Returns 0 ok, 2 overflow (need = trace bytes wanted).
template <bool REVERSE>
__device__ int align_ex_tb(const uint8_t* __restrict__ a, const uint8_t* __restrict__ b, uint32_t m, uint32_t n,
                           int32_t go, int32_t ge, int32_t x_dropoff, const int32_t* __restrict__ mat, TbScratch& S,
                           int32_t& score_out, uint32_t& a_len, uint32_t& b_len, uint32_t* ops_rev, uint32_t ops_cap,
                           uint32_t& n_ops, uint64_t& cells, uint64_t& need) {
    score_out = 0;
    a_len = b_len = 0;
    n_ops = 0;
    if (m == 0 || n == 0) return 0;
    const int32_t goe = go + ge;
    const int32_t xdrop = x_dropoff > goe ? x_dropoff : goe;
    uint64_t flen = 0;
    uint32_t nrows = 0;
#define TB_PUT(v)                                   \
    do {                                            \
        if (flen >= S.trace_cap) { need = flen * 2 + 4096; return 2; } \
        S.trace[flen++] = (v);                      \
    } while (0)
    S.band[0] = make_int2(0, -goe);
    if (nrows >= S.rows_cap) { need = 0; return 2; }
    S.rows[nrows++] = make_uint2(0, 0);
    TB_PUT(T_GAP_B);
    int32_t score = -goe;
    uint32_t b_size = 1;
    for (uint32_t j = 1; j <= n; ++j) {
        if (score < -xdrop) break;
        S.band[j] = make_int2(score, score - goe);
        TB_PUT(T_GAP_A);
        score -= ge;
        b_size = j + 1;
    }
    int32_t best = 0;
    uint32_t best_a = 0, best_b = 0, first_b = 0;
    for (uint32_t ai = 0; ai < m; ++ai) {
        const uint32_t ap = REVERSE ? m - 1 - ai : ai;
        const int32_t* row = mat + ((a[ap] & 15) << 4);
        if (nrows >= S.rows_cap) { need = 0; return 2; }
        S.rows[nrows++] = make_uint2((uint32_t)flen, first_b);
        int32_t sc = MININT, gap_row = MININT;
        uint32_t last_b = first_b;
        cells += b_size - first_b;
        for (uint32_t bi = first_b; bi < b_size; ++bi) {
            uint32_t bb = 0;
            if (bi < n) bb = b[REVERSE ? n - 1 - bi : bi] & 15;
            int2 c = S.band[bi];
            const int32_t next_score = c.x + row[bb];
            uint8_t op = T_SUB;
            int32_t cell = sc;
            if (c.y > cell) { cell = c.y; op = T_GAP_B; }
            if (gap_row > cell) { cell = gap_row; op = T_GAP_A; }
            if (best - cell > xdrop) {
                if (bi == first_b) ++first_b;
                else S.band[bi].x = MININT;
            } else {
                last_b = bi;
                if (cell > best) { best = cell; best_a = ai + 1; best_b = bi; }
                gap_row -= ge;
                const int32_t gcol = c.y - ge;
                const int32_t open = cell - goe;
                int32_t bg;
                if (gcol < open) bg = open;
                else { bg = gcol; op |= T_EXT_B; }
                S.band[bi] = make_int2(cell, bg);
                if (gap_row < open) gap_row = open;
                else op |= T_EXT_A;
            }
            sc = next_score;
            TB_PUT(op);
        }
        if (first_b >= b_size) break;
        if (last_b + 1 < b_size) {
            b_size = last_b + 1;
        } else {
            while (gap_row >= best - xdrop && b_size <= n) {
                S.band[b_size] = make_int2(gap_row, gap_row - goe);
                gap_row -= ge;
                TB_PUT(T_GAP_A);
                ++b_size;
            }
        }
        if (b_size <= n) {
            S.band[b_size] = make_int2(MININT, MININT);
            ++b_size;
        }
    }
#undef TB_PUT
    score_out = best;
    a_len = best_a;
    b_len = best_b;
    // traceback_flat: walk from (best_a, best_b) to (0, 0)
    if (best_a == 0 && best_b == 0) return 0;
    uint32_t aa = best_a, bq = best_b;
    uint8_t prev = T_SUB;
    uint32_t cur_op = 0xffffffffu, cur_n = 0;
    const uint64_t steps = (uint64_t)best_a + best_b;
    for (uint64_t st = 0; st < steps; ++st) {
        const uint2 ri = S.rows[aa];
        const uint64_t row_end = aa + 1 < nrows ? S.rows[aa + 1].x : flen;
        uint8_t raw = T_GAP_A;
        if (bq >= ri.y) {
            const uint64_t k = (uint64_t)ri.x + (bq - ri.y);
            raw = k < row_end ? S.trace[k] : T_GAP_A;
        }
        uint8_t op;
        if ((prev & T_MASK) == T_GAP_A) op = (raw & T_EXT_A) ? T_GAP_A : (raw & T_MASK);
        else if ((prev & T_MASK) == T_GAP_B) op = (raw & T_EXT_B) ? T_GAP_B : (raw & T_MASK);
        else op = raw & T_MASK;
        prev = op;
        uint32_t eop;
        if (op == T_GAP_A) { eop = 1; bq = bq ? bq - 1 : 0; }
        else if (op == T_GAP_B) { eop = 2; aa = aa ? aa - 1 : 0; }
        else { eop = 0; aa = aa ? aa - 1 : 0; bq = bq ? bq - 1 : 0; }
        if (eop == cur_op) ++cur_n;
        else {
            if (cur_n) {
                if (n_ops >= ops_cap) { need = 0; return 2; }
                ops_rev[n_ops++] = (cur_op << 30) | cur_n;
            }
            cur_op = eop;
            cur_n = 1;
        }
        if (aa == 0 && bq == 0) break;
    }
    if (cur_n) {
        if (n_ops >= ops_cap) { need = 0; return 2; }
        ops_rev[n_ops++] = (cur_op << 30) | cur_n;
    }
    if (aa != 0 || bq != 0) return 3;  // the walk did not reach the origin
    return 0;
}

// Warp-cooperative align_ex (gapped.rs:450-689) + traceback_flat (692-757): the rows of
// so_dp_warp with the per-cell op byte (SUB / GAP_B / GAP_A with the extend flags) written by
// the lanes in row order, then the walk by lane 0.  With F* in place of the reference's F the
// op bytes can differ only on cells below the X-drop threshold, and no traceback path visits
// such a cell: a cell on the path holds a value at or above it (cells below are pruned), and a
// horizontal-gap step into a cell needs F >= threshold there, where F = F*.
// Returns 0 ok, 2 scratch overflow, 3 walk did not reach the origin.  ops_rev is written by
// lane 0 as in align_ex_tb (last op first).
template <bool REVERSE>
__device__ int align_ex_tb_warp(const uint8_t* __restrict__ a, const uint8_t* __restrict__ b, uint32_t m,
                                uint32_t n, int32_t go, int32_t ge, int32_t x_dropoff, const int32_t* __restrict__ mat,
                                TbScratch& S, int32_t& score_out, uint32_t& a_len, uint32_t& b_len, uint32_t* ops_rev,
                                uint32_t ops_cap, uint32_t& n_ops, uint64_t& cells, uint64_t& need) {
    const uint32_t lane = threadIdx.x & 31;
    const unsigned FULL = 0xffffffffu;
    score_out = 0;
    a_len = b_len = 0;
    n_ops = 0;
    if (m == 0 || n == 0) return 0;
    const int32_t goe = go + ge;
    const int32_t xdrop = x_dropoff > goe ? x_dropoff : goe;
    const uint32_t J = min(n, (uint32_t)((xdrop - goe) / ge) + 1u);
    if (J + 1 > S.trace_cap || S.rows_cap < 1) { need = S.trace_cap * 2 + 4096; return 2; }
    for (uint32_t j = lane; j <= J; j += 32) {
        if (j == 0) {
            S.band[0] = make_int2(0, -goe);
            S.trace[0] = T_GAP_B;
        } else {
            const int32_t sc = -goe - (int32_t)(j - 1) * ge;
            S.band[j] = make_int2(sc, sc - goe);
            S.trace[j] = T_GAP_A;
        }
    }
    if (lane == 0) S.rows[0] = make_uint2(0, 0);
    uint64_t flen = J + 1;
    uint32_t nrows = 1;
    uint32_t b_size = J + 1, first_b = 0, best_a = 0, best_b = 0;
    int32_t best = 0;
    for (uint32_t ai = 0; ai < m; ++ai) {
        __syncwarp();
        const uint32_t ap = REVERSE ? m - 1 - ai : ai;
        const int32_t* row = mat + ((a[ap] & 15) << 4);
        const uint32_t first0 = first_b;
        if (nrows >= S.rows_cap || flen + (b_size - first0) > S.trace_cap) { need = S.trace_cap * 2 + 4096; return 2; }
        if (lane == 0) S.rows[nrows] = make_uint2((uint32_t)flen, first0);
        ++nrows;
        cells += b_size - first_b;
        int32_t carry_h = MININT, carry_g = MININT, carry_best = best, row_max = MININT;
        uint32_t row_arg = 0, last_b = first_b, new_first = first_b;
        bool leading = true;
        for (uint32_t c0 = first_b; c0 < b_size; c0 += 32) {
            const uint32_t bi = c0 + lane;
            const bool valid = bi < b_size;
            const int2 cur = valid ? S.band[bi] : make_int2(MININT, MININT);
            int32_t hl = __shfl_up_sync(FULL, cur.x, 1);
            if (lane == 0) hl = carry_h;
            int32_t d = MININT;
            if (valid && bi != first_b) d = hl + row[b[REVERSE ? n - bi : bi - 1] & 15];
            const int32_t t = valid ? (d > cur.y ? d : cur.y) : MININT;
            const int32_t tmax = __reduce_max_sync(FULL, t);
            const int32_t thr = carry_best - xdrop;
            int32_t g, f;
            if (carry_g >= thr || tmax - goe >= thr) {
                // shfl_up hands a lane below the offset its own value, and max(g - k ge, g) = g,
                // so every lane takes the step
                g = valid ? t - goe : MININT;
#pragma unroll
                for (uint32_t k = 1; k < 32; k <<= 1) g = __viaddmax_s32(__shfl_up_sync(FULL, g, k), -(int32_t)k * ge, g);
                g = __viaddmax_s32(carry_g, -(int32_t)(lane + 1) * ge, g);
                f = __shfl_up_sync(FULL, g, 1);
                if (lane == 0) f = carry_g;
            } else {
                // F* below the threshold over the whole chunk: no surviving cell, prune decision or
                // traceback step can see it (see the function comment)
                f = MININT;
                g = carry_g > tmax - goe ? carry_g : tmax - goe;
            }
            // op choice with the reference's tie order: diagonal, then vertical, then horizontal
            uint8_t op = T_SUB;
            int32_t cell = d;
            if (cur.y > cell) { cell = cur.y; op = T_GAP_B; }
            if (f > cell) { cell = f; op = T_GAP_A; }
            if (!valid) cell = MININT;
            int32_t before = carry_best, mx = t;
            if (tmax > carry_best) {
#pragma unroll
                for (uint32_t k = 1; k < 32; k <<= 1) mx = max(mx, __shfl_up_sync(FULL, mx, k));
                const int32_t ex = __shfl_up_sync(FULL, mx, 1);
                if (lane != 0) before = max(before, ex);
            }
            const bool pruned = valid && (before - cell > xdrop);
            const bool alive = valid && !pruned;
            const unsigned alive_mask = __ballot_sync(FULL, alive);
            const unsigned valid_mask = __ballot_sync(FULL, valid);
            uint32_t lead_end = 0;
            if (leading) {
                if (alive_mask) {
                    lead_end = __ffs(alive_mask) - 1;
                    new_first += lead_end;
                    leading = false;
                } else {
                    lead_end = 32;
                    new_first += __popc(valid_mask);
                }
            }
            if (alive) {
                const int32_t gcol = cur.y - ge, open = cell - goe;
                int32_t bg;
                if (gcol < open) bg = open;
                else { bg = gcol; op |= T_EXT_B; }
                S.band[bi] = make_int2(cell, bg);
                if (!(f - ge < open)) op |= T_EXT_A;
            } else if (pruned && lane >= lead_end) {
                S.band[bi].x = MININT;
            }
            if (valid) S.trace[flen + (bi - first0)] = op;
            if (alive_mask) last_b = c0 + 31 - __clz(alive_mask);
            if (tmax > row_max) {
                row_max = tmax;
                row_arg = c0 + __ffs(__ballot_sync(FULL, valid && t == tmax)) - 1;
            }
            if (tmax > carry_best) carry_best = tmax;
            carry_g = __shfl_sync(FULL, g, 31 - __clz(valid_mask));
            carry_h = __shfl_sync(FULL, cur.x, 31);
        }
        flen += b_size - first0;
        first_b = new_first;
        if (row_max > best) {
            best = row_max;
            best_b = row_arg;
            best_a = ai + 1;
        }
        if (first_b >= b_size) break;
        const int32_t gap_row = carry_g;
        if (last_b + 1 < b_size) {
            b_size = last_b + 1;
        } else if (gap_row >= best - xdrop && b_size <= n) {
            const uint32_t k = ext_count(gap_row, best - xdrop, ge, n + 1 - b_size);
            if (flen + k > S.trace_cap) { need = S.trace_cap * 2 + 4096; return 2; }
            __syncwarp();
            for (uint32_t i = lane; i < k; i += 32) {
                const int32_t v = gap_row - (int32_t)i * ge;
                S.band[b_size + i] = make_int2(v, v - goe);
                S.trace[flen + i] = T_GAP_A;
            }
            flen += k;
            b_size += k;
        }
        if (b_size <= n) {
            if (lane == 0) S.band[b_size] = make_int2(MININT, MININT);
            ++b_size;
        }
    }
    __syncwarp();
    score_out = best;
    a_len = best_a;
    b_len = best_b;
    if (best_a == 0 && best_b == 0) return 0;
    int st = 0;
    if (lane == 0) {
        uint32_t aa = best_a, bq = best_b;
        uint8_t prev = T_SUB;
        uint32_t cur_op = 0xffffffffu, cur_n = 0, nops = 0;
        const uint64_t steps = (uint64_t)best_a + best_b;
        for (uint64_t s2 = 0; s2 < steps && st == 0; ++s2) {
            const uint2 ri = S.rows[aa];
            const uint64_t row_end = aa + 1 < nrows ? S.rows[aa + 1].x : flen;
            uint8_t raw = T_GAP_A;
            if (bq >= ri.y) {
                const uint64_t k = (uint64_t)ri.x + (bq - ri.y);
                raw = k < row_end ? S.trace[k] : T_GAP_A;
            }
            uint8_t op;
            if ((prev & T_MASK) == T_GAP_A) op = (raw & T_EXT_A) ? T_GAP_A : (raw & T_MASK);
            else if ((prev & T_MASK) == T_GAP_B) op = (raw & T_EXT_B) ? T_GAP_B : (raw & T_MASK);
            else op = raw & T_MASK;
            prev = op;
            uint32_t eop;
            if (op == T_GAP_A) { eop = 1; bq = bq ? bq - 1 : 0; }
            else if (op == T_GAP_B) { eop = 2; aa = aa ? aa - 1 : 0; }
            else { eop = 0; aa = aa ? aa - 1 : 0; bq = bq ? bq - 1 : 0; }
            if (eop == cur_op) ++cur_n;
            else {
                if (cur_n) {
                    if (nops >= ops_cap) { st = 2; break; }
                    ops_rev[nops++] = (cur_op << 30) | cur_n;
                }
                cur_op = eop;
                cur_n = 1;
            }
            if (aa == 0 && bq == 0) break;
        }
        if (st == 0 && cur_n) {
            if (nops >= ops_cap) st = 2;
            else ops_rev[nops++] = (cur_op << 30) | cur_n;
        }
        if (st == 0 && (aa != 0 || bq != 0)) st = 3;
        n_ops = nops;
    }
    st = __shfl_sync(FULL, st, 0);
    n_ops = __shfl_sync(FULL, n_ops, 0);
    if (st == 2) need = 0;
    return st;
}

// One extension of a prelim per warp: item 2t is prelim t's left extension, item 2t + 1 its right
// one (both from the improved seed, independent of each other), so a long alignment's two DPs
// run side by side on two warps; k_traceback_join then merges the two scripts.  Each item's ops
// go to its own ops_cap slot; `half` gets its status, score, extents and op count.  With `whole`
// a warp takes a prelim's two items one after the other (one prelim per warp, the plain
// pipeline's work unit).
__global__ void __launch_bounds__(256) k_traceback_warp(DevLib L, DevQueries Q, const DevParams* __restrict__ P,
                                                         uint32_t n, const TbIn* __restrict__ in,
                                                         TbHalf* __restrict__ half, uint32_t* __restrict__ ops_out,
                                                         uint32_t ops_cap, uint8_t* __restrict__ scratch,
                                                         uint64_t per_warp, uint64_t band_cells, uint32_t rows_cap,
                                                         unsigned long long* __restrict__ cells_total, bool whole) {
    __shared__ int32_t mat[256];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) mat[i] = P->matrix[i];
    __syncthreads();
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    // item sequence of this warp: k = warp, warp + nwarps, ...; or, whole, 2w, 2w + 1, 2(w + nwarps), ...
    const uint64_t k_first = whole ? 2 * warp : warp, k_stride = whole ? 2 * nwarps : nwarps;
    uint8_t* base = scratch + warp * per_warp;
    TbScratch S;
    S.band = (int2*)base;
    S.rows = (uint2*)(base + band_cells * sizeof(int2));
    S.rows_cap = rows_cap;
    S.trace = base + band_cells * sizeof(int2) + (uint64_t)rows_cap * sizeof(uint2);
    S.trace_cap = per_warp - band_cells * sizeof(int2) - (uint64_t)rows_cap * sizeof(uint2);
    uint64_t cells = 0;
    for (uint64_t k0 = k_first; k0 < 2ull * n; k0 += k_stride)
    for (uint64_t k = k0; k < (whole ? k0 + 2 : k0 + 1); ++k) {
        const uint64_t t = k >> 1;
        const bool right = k & 1;
        const TbIn h = in[t];
        const uint32_t qi = h.pair / L.n, si = h.pair % L.n;
        const uint32_t qa = Q.len[qi], sa = L.len[si];
        const bool plus = h.strand == 0;
        const uint8_t* qfwd = Q.q + Q.off[qi] + 1;
        const uint8_t* sfs = (plus ? L.align : L.align_rc) + L.plus_off[si] + 1;
        uint32_t nq = 0, ns = 0;
        if (lane == 0) improve_seed(qfwd, qa, sfs, sa, h.q_seed, h.s_seed, h.q_start, h.q_end, h.s_start, h.s_end, !plus, nq, ns);
        nq = __shfl_sync(0xffffffffu, nq, 0);
        ns = __shfl_sync(0xffffffffu, ns, 0);
        const uint32_t tq = plus ? nq : qa - 1 - nq, ts = plus ? ns : sa - 1 - ns;
        const uint8_t* qa_ = (plus ? Q.q : Q.qrc) + Q.off[qi] + 1;
        const uint8_t* sa_ = L.align + L.plus_off[si] + 1;
        uint32_t* ops = ops_out + k * (uint64_t)ops_cap;
        uint64_t need = 0;
        int32_t sc = 0;
        uint32_t a = 0, b = 0, nops = 0;
        int st = 0;
        if (!right) {
            st = align_ex_tb_warp<true>(qa_, sa_, tq + 1, ts + 1, P->gap_open, P->gap_extend, P->xdrop_gap_final, mat,
                                        S, sc, a, b, ops, ops_cap, nops, cells, need);
        } else {
            const uint32_t rq = tq + 1, rsd = ts + 1;
            const uint32_t rm = qa > rq ? qa - rq : 0, rn = sa > rsd ? sa - rsd : 0;
            if (rm > 0 && rn > 0)
                st = align_ex_tb_warp<false>(qa_ + rq, sa_ + rsd, rm, rn, P->gap_open, P->gap_extend,
                                             P->xdrop_gap_final, mat, S, sc, a, b, ops, ops_cap, nops, cells, need);
        }
        if (lane == 0)
            half[k] = TbHalf{st, sc, a, b, nops, (uint32_t)min(need, (uint64_t)0xffffffffu), tq, ts};
    }
    if (lane == 0 && cells) atomicAdd(cells_total, (unsigned long long)cells);
}

// One prelim per thread: its two extensions' scripts merged (the right one reversed after the
// left one, runs of one op joined), the end gaps pruned, and the box and score of the whole
// alignment (engine.rs:2953-3039).  The merged script goes to the left item's ops slot.
__global__ void k_traceback_join(const DevParams* __restrict__ P, uint32_t n, const TbHalf* __restrict__ half,
                                 uint32_t* __restrict__ ops_out, uint32_t ops_cap, TbOut* __restrict__ out) {
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const TbHalf lh = half[2 * t], rh = half[2 * t + 1];
    TbOut o{0, 0, 0, 0, 0, 0, 0, 0};
    if (lh.status != 0 || rh.status != 0) {
        o.status = lh.status == 3 || rh.status == 3 ? 3 : 2;
        o.need = max(lh.status ? lh.need : 0u, rh.status ? rh.need : 0u);
        out[t] = o;
        return;
    }
    uint32_t* ops = ops_out + 2 * t * (uint64_t)ops_cap;
    const uint32_t* rops = ops_out + (2 * t + 1) * (uint64_t)ops_cap;
    const uint32_t nl = lh.n_ops, nr = rh.n_ops;
    const uint32_t tq = lh.tq, ts = lh.ts;
    uint32_t nops = nl;
    for (uint32_t i = 0; i < nr; ++i) {
        const uint32_t v = rops[nr - 1 - i];
        if (nops > 0 && (ops[nops - 1] >> 30) == (v >> 30)) {
            ops[nops - 1] += v & 0x3fffffffu;
        } else {
            if (nops >= ops_cap) {  // the joined script does not fit the slot: again with larger slots
                o.status = 2;
                out[t] = o;
                return;
            }
            ops[nops++] = v;
        }
    }
    int32_t total = lh.score + rh.score;
    uint32_t q_start = tq + 1 - lh.a_len, s_start = ts + 1 - lh.b_len, q_end = tq + 1 + rh.a_len,
             s_end = ts + 1 + rh.b_len;
    uint32_t first = 0;
    while (first < nops && (ops[first] >> 30) != 0) {
        const uint32_t op = ops[first] >> 30, cnt = ops[first] & 0x3fffffffu;
        total += P->gap_open + (int32_t)cnt * P->gap_extend;
        if (op == 1) s_start += cnt;
        else q_start += cnt;
        ++first;
    }
    while (nops > first && (ops[nops - 1] >> 30) != 0) {
        const uint32_t op = ops[nops - 1] >> 30, cnt = ops[nops - 1] & 0x3fffffffu;
        total += P->gap_open + (int32_t)cnt * P->gap_extend;
        if (op == 1) s_end -= cnt;
        else q_end -= cnt;
        --nops;
    }
    if (first) {
        for (uint32_t i = first; i < nops; ++i) ops[i - first] = ops[i];
        nops -= first;
    }
    if (total < 0) {
        o.status = 1;
        out[t] = o;
        return;
    }
    o.score = total;
    o.q0 = q_start;
    o.q1 = q_end;
    o.s0 = s_start;
    o.s1 = s_end;
    o.n_ops = nops;
    out[t] = o;
}

// ---------------------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------------------
static int grid_for(uint64_t work, int block, int per_sm_blocks, int sms) {
    uint64_t g = (work + block - 1) / block;
    uint64_t cap = (uint64_t)sms * per_sm_blocks;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return (int)g;
}

// The run-length ops of the finished traceback items (status 0/1), packed back to back:
// dst[off[i] ..] = ops[i * ops_cap ..][0 .. n_ops); one warp per item.
__global__ void __launch_bounds__(256) k_gather_ops(uint32_t n, const uint32_t* __restrict__ ops, uint32_t ops_cap,
                                                     const TbOut* __restrict__ out, const uint64_t* __restrict__ off,
                                                     uint32_t* __restrict__ dst) {
    const int lane = threadIdx.x & 31;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += nwarps) {
        if (out[i].status == 2) continue;
        const uint32_t c = out[i].n_ops;
        for (uint32_t k = lane; k < c; k += 32) dst[off[i] + k] = ops[(uint64_t)i * ops_cap + k];
    }
}

cudaError_t launch_gather_ops(uint32_t n, const uint32_t* ops, uint32_t ops_cap, const TbOut* out, const uint64_t* off,
                              uint32_t* dst, int sms, cudaStream_t st) {
    if (!n) return cudaSuccess;
    k_gather_ops<<<grid_for((uint64_t)n * 32, 256, 8, sms), 256, 0, st>>>(n, ops, ops_cap, out, off, dst);
    return cudaGetLastError();
}

cudaError_t launch_scan(bool write, const DevLib& L, const DevQueries& Q, int32_t ws, uint64_t pair0, uint64_t n_pairs,
                        uint32_t* counts, const uint64_t* offs, SeedHit* hits, uint32_t* hit_pair, int sms,
                        cudaStream_t st) {
    const int block = 256;
    const int grid = grid_for(n_pairs * 32, block, 8, sms);
    if (write)
        k_scan<SCAN_WRITE><<<grid, block, 0, st>>>(L, Q, ws, pair0, n_pairs, counts, offs, hits, hit_pair, nullptr,
                                                   0, nullptr, nullptr);
    else
        k_scan<SCAN_COUNT><<<grid, block, 0, st>>>(L, Q, ws, pair0, n_pairs, counts, offs, hits, hit_pair, nullptr,
                                                   0, nullptr, nullptr);
    return cudaGetLastError();
}

uint64_t scan_stage_entries(uint64_t n_pairs, int sms) {
    return (uint64_t)grid_for(n_pairs * 32, 256, 8, sms) * (256 / 32) * SCAN_STAGE_PER_WARP;
}

cudaError_t launch_scan_stage(const DevLib& L, const DevQueries& Q, int32_t ws, uint64_t n_pairs, uint32_t* counts,
                              uint32_t* stage_start, SeedHit* stage, unsigned int* stage_over, int sms,
                              cudaStream_t st, bool queue) {
    // stage_over: [0] the overflow flag, [2..3] the pair queue (both zeroed by the caller); without
    // `queue` the warps take pairs by stride
    const int block = 256;
    const int grid = grid_for(n_pairs * 32, block, 8, sms);
    k_scan<SCAN_STAGE><<<grid, block, 0, st>>>(L, Q, ws, 0, n_pairs, counts, nullptr, stage, nullptr, stage_start,
                                               SCAN_STAGE_PER_WARP, stage_over,
                                               queue ? reinterpret_cast<unsigned long long*>(stage_over + 2) : nullptr);
    return cudaGetLastError();
}

cudaError_t launch_scan_gather(uint64_t pair0, uint64_t n_pairs, const uint32_t* counts, const uint64_t* offs,
                               const uint32_t* stage_start, const SeedHit* stage, SeedHit* hits, uint32_t* hit_pair,
                               int sms, cudaStream_t st) {
    if (!n_pairs) return cudaSuccess;
    k_scan_gather<<<grid_for(n_pairs * 32, 256, 8, sms), 256, 0, st>>>(pair0, n_pairs, counts, offs, stage_start,
                                                                       stage, hits, hit_pair);
    return cudaGetLastError();
}

cudaError_t launch_ungapped(const DevLib& L, const DevQueries& Q, const DevParams* P, int32_t ucut, uint64_t n,
                            const SeedHit* hits, const uint32_t* hit_pair, UngBox* out, int sms, cudaStream_t st,
                            unsigned long long* queue, int blocks_per_sm) {
    if (!n) return cudaSuccess;
    const int block = 256;
    if (!queue) {  // plain: one hit per thread
        k_ungapped<false><<<(unsigned)((n + block - 1) / block), block, 0, st>>>(L, Q, P, ucut, n, hits, hit_pair,
                                                                                 out, nullptr);
        return cudaGetLastError();
    }
    cudaError_t e = cudaMemsetAsync(queue, 0, sizeof(unsigned long long), st);
    if (e != cudaSuccess) return e;
    const int bps = blocks_per_sm < 1 ? 1 : blocks_per_sm > 8 ? 8 : blocks_per_sm;
    k_ungapped<true><<<grid_for(n, block, bps, sms), block, 0, st>>>(L, Q, P, ucut, n, hits, hit_pair, out, queue);
    return cudaGetLastError();
}

uint64_t dedup_threads(int sms) { return (uint64_t)sms * 8 * 128; }

cudaError_t launch_dedup(const DevLib& L, const DevQueries& Q, int32_t ws, int32_t ucut, uint64_t pair0,
                         uint64_t n_pairs, const uint64_t* offs, const SeedHit* hits, const UngBox* ub, uint8_t* flags,
                         uint32_t* scratch, void* cells, int sms, cudaStream_t st) {
    const int block = 128;
    const uint64_t want = (n_pairs + block - 1) / block;
    const uint64_t cap = dedup_threads(sms) / block;
    const int grid = (int)(want < cap ? (want ? want : 1) : cap);
    k_dedup<<<grid, block, 0, st>>>(L, Q, ws, ucut, pair0, n_pairs, offs, hits, ub, flags, scratch, (DiagCell*)cells);
    return cudaGetLastError();
}

size_t diag_cell_bytes() { return sizeof(DiagCell); }
uint32_t dedup_glog(uint64_t n_pairs, uint64_t n_hits, int sms) {
    // few pairs with many hits each (one genome against a small library): every pair's buckets
    // split into at least 2^glog groups, one warp a group, until the grid's warps have work
    uint32_t glog = 0;
    while (glog < DDX_GLOG_MAX && n_pairs && (n_pairs << glog) < (uint64_t)sms * 48 &&
           n_hits / (n_pairs << glog) >= 1024)
        ++glog;
    return glog;
}

// hits a unit may hold before its pair is split: a warp's share of the launch's hits
uint64_t dedup_unit_hits(uint64_t n_hits, int sms) {
    const uint64_t share = n_hits / ((uint64_t)sms * 32);
    return share > 2048 ? share : 2048;
}

size_t dedup_units_bytes(uint64_t n_pairs, uint64_t n_hits, int sms) {
    // a pair split past glog has G < 2 h / unit_hits, so the groups of all pairs with G > 1
    // number at most n_pairs 2^glog + 2 n_hits / unit_hits
    const uint64_t heavy =
        (n_pairs << dedup_glog(n_pairs, n_hits, sms)) + 2 * n_hits / dedup_unit_hits(n_hits, sms) + 1;
    return 16 + heavy * 8 + n_pairs * 4 + 16;
}

cudaError_t launch_dedup_extend(const DevLib& L, const DevQueries& Q, const DevParams* P, int32_t ucut,
                                uint64_t pair0, uint64_t n_pairs, uint64_t n_hits, const uint64_t* offs,
                                const SeedHit* hits, UngBox* ub, uint8_t* flags, void* cells,
                                unsigned long long* queue, void* units_buf, int sms, cudaStream_t st) {
    if (!n_pairs) return cudaSuccess;
    const uint32_t glog = dedup_glog(n_pairs, n_hits, sms);
    const uint64_t unit_hits = dedup_unit_hits(n_hits, sms);
    const uint64_t heavy_cap = (n_pairs << glog) + 2 * n_hits / unit_hits + 1;
    DedupUnits du;
    du.counts = (unsigned int*)units_buf;
    du.heavy = (unsigned long long*)((char*)units_buf + 16);
    du.light = (uint32_t*)(du.heavy + heavy_cap);
    du.heavy_cap = heavy_cap;
    cudaError_t e = cudaMemsetAsync(queue, 0, sizeof(unsigned long long), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(du.counts, 0, 16, st);
    if (e != cudaSuccess) return e;
    const uint64_t bb = (n_pairs + 255) / 256;
    k_dedup_units<<<(unsigned)(bb < 4096 ? bb : 4096), 256, 0, st>>>(n_pairs, offs, glog, unit_hits, du);
    const uint64_t units = n_pairs << glog;
    const uint64_t want = (units + DDX_WARPS - 1) / DDX_WARPS;
    const uint64_t cap = (uint64_t)sms * 8;
    k_dedup_extend<<<(unsigned)(want < cap ? want : cap), DDX_WARPS * 32, 0, st>>>(
        L, Q, P, ucut, pair0, n_pairs, offs, hits, ub, flags, (DiagCell*)cells, queue, du);
    return cudaGetLastError();
}

constexpr int PRELIM_RING = 256;

cudaError_t launch_prelim(const DevLib& L, const DevQueries& Q, const DevParams* P, uint64_t n, const uint32_t* list,
                          const uint32_t* idx, const SeedHit* hits, const uint32_t* hit_pair, const UngBox* ub,
                          PrelimOut* out, uint32_t* wide, unsigned int* n_wide, unsigned long long* cells, int sms,
                          cudaStream_t st) {
    if (!n) return cudaSuccess;
    const int block = 256;
    const uint64_t blocks_wanted = (n + 7) / 8;
    const uint64_t cap = (uint64_t)sms * 8;
    const int grid = (int)(blocks_wanted < cap ? blocks_wanted : cap);
    k_prelim_warp<PRELIM_RING><<<grid, block, 0, st>>>(L, Q, P, n, idx, hits, hit_pair, ub, out, list, wide, n_wide,
                                                       cells);
    return cudaGetLastError();
}

bool prelim_stream_eligible(const int32_t* matrix256, int32_t gap_open, int32_t gap_extend, int32_t xdrop_gap) {
    // 14-bit band values: live ones within X + max score of the row threshold, dead ones at
    // FLOOR = -8192 (below every later threshold minus the best score)
    const int32_t xmax = std::max(xdrop_gap, gap_open + gap_extend);
    if (gap_extend < 1 || gap_open < 0 || xmax > 8000) return false;
    for (int i = 0; i < 256; ++i)
        if (matrix256[i] > 127) return false;
    return true;
}

size_t prelim_geo_bytes() { return sizeof(PrelimGeo); }

cudaError_t launch_prelim_prep(const DevLib& L, const DevQueries& Q, const DevParams* P, uint64_t n,
                               const uint32_t* idx, const SeedHit* hits, const uint32_t* hit_pair, const UngBox* ub,
                               void* geo, int sms, cudaStream_t st, const unsigned int* n_dev) {
    if (!n) return cudaSuccess;
    k_prelim_prep<<<grid_for(n, 256, 8, sms), 256, 0, st>>>(L, Q, P, n, idx, hits, hit_pair, ub, (PrelimGeo*)geo,
                                                            n_dev);
    return cudaGetLastError();
}

cudaError_t launch_prelim_stream(const DevParams* P, uint64_t n, const void* geo, PrelimOut* out, uint32_t* wide,
                                 unsigned int* n_wide, unsigned long long* cells, int sms, cudaStream_t st,
                                 const uint32_t* order, uint32_t* cells_out, bool plain, const StreamLaunch& cfg,
                                 StreamDevCounts dc) {
    if (!n) return cudaSuccess;
    const uint64_t want = (n + STREAM_BLOCK - 1) / STREAM_BLOCK;
    const int bps = cfg.blocks_per_sm < 1 ? 1 : cfg.blocks_per_sm > STREAM_BLOCKS_PER_SM ? STREAM_BLOCKS_PER_SM
                                                                                          : cfg.blocks_per_sm;
    const uint64_t cap = (uint64_t)sms * bps;
    const int grid = (int)(want < cap ? want : cap);
    // the record queue counter sits after the overflow count in n_wide (zeroed by the caller)
    const uint32_t bdiv = (uint32_t)(cfg.budget_div > 0 ? cfg.budget_div : 128);
    const uint64_t budget = n / bdiv;
    // with the records in descending predicted cost the long ones start first: the full budget
    const uint32_t max_cells = order ? STREAM_MAX_CELLS
                                     : (uint32_t)(budget < STREAM_MIN_CELLS ? STREAM_MIN_CELLS
                                                  : budget > STREAM_MAX_CELLS ? STREAM_MAX_CELLS : budget);
    const uint32_t window = cfg.window < 1 ? 1 : cfg.window > STREAM_WINDOW ? STREAM_WINDOW : (uint32_t)cfg.window;
    const PrelimGeo* g = (const PrelimGeo*)geo;
#define RMB_STREAM_LAUNCH(U)                                                                                      \
    do {                                                                                                         \
        if (plain) /* one record per thread, the whole grid at once */                                           \
            k_prelim_stream<U, false><<<(unsigned)want, STREAM_BLOCK, 0, st>>>(P, n, g, out, wide, n_wide,       \
                                                                               n_wide + 1, cells, max_cells,     \
                                                                               order, cells_out, window, dc,     \
                                                                               bdiv);                            \
        else                                                                                                     \
            k_prelim_stream<U, true><<<grid, STREAM_BLOCK, 0, st>>>(P, n, g, out, wide, n_wide, n_wide + 1,      \
                                                                    cells, max_cells, order, cells_out, window,  \
                                                                    dc, bdiv);                                   \
    } while (0)
    // groups of cell steps between row-end blocks: smaller groups run more row-end blocks, larger
    // ones leave lanes idle longer (8 was the B200 hand sweep's best on the genome workloads)
    if (cfg.group == 4) RMB_STREAM_LAUNCH(4);
    else if (cfg.group == 16) RMB_STREAM_LAUNCH(16);
    else RMB_STREAM_LAUNCH(8);
#undef RMB_STREAM_LAUNCH
    return cudaGetLastError();
}

cudaError_t launch_sched_features(const DevLib& L, const DevQueries& Q, const DevParams* P, uint64_t n,
                                  const uint32_t* idx, const SeedHit* hits, const uint32_t* hit_pair, const UngBox* ub,
                                  const uint32_t* pair_hits, float* out, int sms, cudaStream_t st) {
    if (!n) return cudaSuccess;
    k_sched_features<<<grid_for(n, 256, 8, sms), 256, 0, st>>>(L, Q, P, n, idx, hits, hit_pair, ub, pair_hits, out);
    return cudaGetLastError();
}

size_t sched_order_scratch_bytes() { return 3 * SCHED_BINS * sizeof(unsigned int); }

// The front of the front-loaded order: the lowest cost bin b such that the records in bins >= b
// are at most n / SCHED_FRONT_DIV (SCHED_BINS when even the costliest bin holds more).
constexpr uint64_t SCHED_FRONT_DIV = 32;
__global__ void k_sched_cut(const unsigned int* __restrict__ hist, uint64_t n, unsigned int* __restrict__ cut,
                            const unsigned int* __restrict__ n_dev) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    if (n_dev) n = *n_dev;
    const uint64_t limit = n / SCHED_FRONT_DIV;
    uint64_t acc = 0;
    unsigned int c = SCHED_BINS;
    for (int b = SCHED_BINS - 1; b >= 0; --b) {
        if (acc + hist[b] > limit) break;
        acc += hist[b];
        c = (unsigned int)b;
    }
    *cut = c;
}

struct SchedFront {
    const float* pred;
    const unsigned int* cut;
    const unsigned int* n_dev;  // records past the device count are never at the front
    __host__ __device__ bool operator()(const uint32_t& i) const {
        return (!n_dev || i < *n_dev) && sched_bin(pred[i]) >= *cut;
    }
};

const unsigned int* sched_front_count(const void* scratch) { return (const unsigned int*)scratch + SCHED_BINS + 1; }

size_t sched_front_temp_bytes(uint64_t n) {
    size_t tb = 0;
    thrust::counting_iterator<uint32_t> it(0);
    cub::DevicePartition::If(nullptr, tb, it, (uint32_t*)nullptr, (uint32_t*)nullptr, (int64_t)n,
                             SchedFront{nullptr, nullptr, nullptr});
    return tb;
}

cudaError_t launch_sched_order(const DevLib& L, const DevQueries& Q, const DevParams* P, uint64_t n,
                               const uint32_t* idx, const SeedHit* hits, const uint32_t* hit_pair, const UngBox* ub,
                               const uint32_t* pair_hits, const float* params, float* pred, void* scratch,
                               uint32_t* order, int sms, cudaStream_t st, int layout, void* temp, size_t temp_bytes,
                               const unsigned int* n_dev) {
    if (!n) return cudaSuccess;
    unsigned int* hist = (unsigned int*)scratch;
    cudaError_t e = cudaMemsetAsync(hist, 0, SCHED_BINS * sizeof(unsigned int), st);
    if (e != cudaSuccess) return e;
    const uint64_t warps = (n + 31) / 32;
    const int grid = (int)std::min<uint64_t>((warps + SCHED_BLOCK / 32 - 1) / (SCHED_BLOCK / 32), (uint64_t)sms * 8);
    k_sched_predict<<<grid, SCHED_BLOCK, 0, st>>>(L, Q, P, n, idx, hits, hit_pair, ub, pair_hits, nullptr, params, pred,
                                                  hist, n_dev);
    if (layout == 1) {
        // front-loaded: the predicted-costliest records (about n / 32) first, in arrival order, then
        // the rest in reverse arrival order -- neighbouring records keep sharing their sequences
        unsigned int* cut = hist + SCHED_BINS;
        k_sched_cut<<<1, 1, 0, st>>>(hist, n, cut, n_dev);
        thrust::counting_iterator<uint32_t> it(0);
        unsigned int* n_front = hist + SCHED_BINS + 1;
        e = cub::DevicePartition::If(temp, temp_bytes, it, order, n_front, (int64_t)n, SchedFront{pred, cut, n_dev},
                                     st);
        if (e != cudaSuccess) return e;
        return cudaGetLastError();
    }
    // the full descending cost order
    k_sched_binstart<<<1, 1, 0, st>>>(hist, hist + SCHED_BINS, hist + 2 * SCHED_BINS);
    const uint64_t tile = 256ull * SCHED_TILE_PER_THREAD;
    const int g2 = (int)std::min<uint64_t>((n + tile - 1) / tile, (uint64_t)sms * 8);
    k_sched_scatter<<<g2, 256, 0, st>>>(n, pred, hist + SCHED_BINS, hist + 2 * SCHED_BINS, order);
    return cudaGetLastError();
}

cudaError_t launch_sched_predict_features(uint64_t n, const float* feats, const float* params, float* pred, int sms,
                                          cudaStream_t st) {
    if (!n) return cudaSuccess;
    const uint64_t warps = (n + 31) / 32;
    const int grid = (int)std::min<uint64_t>((warps + SCHED_BLOCK / 32 - 1) / (SCHED_BLOCK / 32), (uint64_t)sms * 8);
    k_sched_predict<<<grid, SCHED_BLOCK, 0, st>>>(DevLib{}, DevQueries{}, nullptr, n, nullptr, nullptr, nullptr, nullptr,
                                                  nullptr, feats, params, pred, nullptr, nullptr);
    return cudaGetLastError();
}

cudaError_t launch_prelim_split(const DevLib& L, const DevQueries& Q, const DevParams* P, uint32_t n_list,
                                const uint32_t* list, const uint32_t* idx, const SeedHit* hits,
                                const uint32_t* hit_pair, const UngBox* ub, int4* dres, PrelimOut* out,
                                uint32_t* wide, unsigned int* n_wide, unsigned long long* cells, int sms,
                                cudaStream_t st, const unsigned int* n_dev) {
    if (!n_list) return cudaSuccess;
    const int block = 256;
    const uint64_t blocks_wanted = (2ull * n_list + 7) / 8;
    const uint64_t cap = (uint64_t)sms * 8;
    const int grid = (int)(blocks_wanted < cap ? blocks_wanted : cap);
    k_prelim_warp_dir<PRELIM_RING><<<grid, block, 0, st>>>(L, Q, P, n_list, list, idx, hits, hit_pair, ub, dres, cells,
                                                           n_dev);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_prelim_combine<<<(n_list + 127) / 128, 128, 0, st>>>(L, Q, P, n_list, list, idx, hits, hit_pair, ub, dres, out,
                                                          wide, n_wide, n_dev);
    return cudaGetLastError();
}

cudaError_t launch_prelim_wide(const DevLib& L, const DevQueries& Q, const DevParams* P, uint32_t n_wide,
                               const uint32_t* wide, const uint32_t* idx, const SeedHit* hits, const uint32_t* hit_pair,
                               const UngBox* ub, PrelimOut* out, int2* band_mem, uint64_t band_cap, uint32_t threads,
                               unsigned long long* cells, unsigned int* failures, cudaStream_t st,
                               const unsigned int* n_dev) {
    if (!n_wide) return cudaSuccess;
    const int block = 128;
    const int grid = (int)((threads + block - 1) / block);
    k_prelim_wide<<<grid, block, 0, st>>>(L, Q, P, n_wide, wide, idx, hits, hit_pair, ub, out, band_mem, band_cap, cells,
                                          failures, n_dev);
    return cudaGetLastError();
}

cudaError_t launch_traceback(const DevLib& L, const DevQueries& Q, const DevParams* P, uint32_t n, const TbIn* in,
                             TbOut* out, TbHalf* half, uint32_t* ops, uint32_t ops_cap, uint8_t* scratch,
                             uint64_t per_thread, uint64_t band_cells, uint32_t rows_cap, uint32_t threads,
                             unsigned long long* cells, bool whole, cudaStream_t st) {
    // `threads` scratch slots of `per_thread` bytes: one warp per slot, two items per prelim;
    // ops: 2 n slots of ops_cap, the merged script of prelim t in slot 2 t
    if (!n) return cudaSuccess;
    const int block = 256;
    const uint32_t warps = threads;
    const int grid = (int)((warps * 32 + block - 1) / block);
    k_traceback_warp<<<grid, block, 0, st>>>(L, Q, P, n, in, half, ops, ops_cap, scratch, per_thread, band_cells,
                                             rows_cap, cells, whole);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    k_traceback_join<<<(n + 127) / 128, 128, 0, st>>>(P, n, half, ops, ops_cap, out);
    return cudaGetLastError();
}

}  // namespace rmb

// ---------------------------------------------------------------------------------------
// compaction helpers (CUB device-wide scan / select)
// ---------------------------------------------------------------------------------------
#include <cub/device/device_scan.cuh>
#include <cub/device/device_select.cuh>
#include <thrust/iterator/counting_iterator.h>

namespace rmb {

struct U64Add {
    __host__ __device__ __forceinline__ uint64_t operator()(uint64_t a, uint64_t b) const { return a + b; }
};

__global__ void k_gather_survivors(uint32_t n, const uint32_t* __restrict__ sel, const uint32_t* __restrict__ idx,
                                   const SeedHit* __restrict__ hits, const uint32_t* __restrict__ hit_pair,
                                   const UngBox* __restrict__ ub, const PrelimOut* __restrict__ po,
                                   SurvivorRec* __restrict__ out, const unsigned int* __restrict__ n_dev) {
    if (n_dev) n = min(*n_dev, n);  // the count on the device, n the output's capacity
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const uint32_t t = sel[k];
        const uint32_t i = idx[t];
        out[k] = SurvivorRec{hit_pair[i], hits[i], ub[i], po[t]};
    }
}

cudaError_t launch_gather_survivors(uint32_t n, const uint32_t* sel, const uint32_t* idx, const SeedHit* hits,
                                    const uint32_t* hit_pair, const UngBox* ub, const PrelimOut* po,
                                    SurvivorRec* out, cudaStream_t st, const unsigned int* n_dev) {
    if (!n) return cudaSuccess;
    const uint32_t blocks = (n + 255) / 256;
    k_gather_survivors<<<blocks < 4096 ? blocks : 4096, 256, 0, st>>>(n, sel, idx, hits, hit_pair, ub, po, out, n_dev);
    return cudaGetLastError();
}

struct FlagEq {
    const uint8_t* f;
    uint8_t want;
    __host__ __device__ bool operator()(const uint32_t& i) const { return f[i] == want; }
};
struct PrelimPass {
    const PrelimOut* p;
    const unsigned int* n_dev;  // records past the device count are stale
    __host__ __device__ bool operator()(const uint32_t& i) const {
        return (!n_dev || i < *n_dev) && p[i].score != INT32_MIN;
    }
};

cudaError_t launch_select_eq(const uint8_t* flags, uint64_t n, uint8_t want, uint32_t* out, uint32_t* n_out,
                             void* temp, size_t& temp_bytes, cudaStream_t st) {
    thrust::counting_iterator<uint32_t> it(0);
    return cub::DeviceSelect::If(temp, temp_bytes, it, out, n_out, (int64_t)n, FlagEq{flags, want}, st);
}

cudaError_t launch_select_prelim(const PrelimOut* po, uint64_t n, uint32_t* out, uint32_t* n_out, void* temp,
                                 size_t& temp_bytes, cudaStream_t st, const unsigned int* n_dev) {
    thrust::counting_iterator<uint32_t> it(0);
    return cub::DeviceSelect::If(temp, temp_bytes, it, out, n_out, (int64_t)n, PrelimPass{po, n_dev}, st);
}

cudaError_t launch_offsets(const uint32_t* counts, uint64_t n, uint64_t* offs, void* temp, size_t& temp_bytes,
                           cudaStream_t st) {
    // a 64-bit initial value makes the scan accumulate in 64 bits: the counts are 32-bit, their
    // sums are not (ExclusiveSum would add them up in the counts' type)
    return cub::DeviceScan::ExclusiveScan(temp, temp_bytes, counts, offs, U64Add{}, (uint64_t)0, (int64_t)n, st);
}

}  // namespace rmb

// ---------------------------------------------------------------------------------------
// lookup tables on the device: blast/nalookup.rs:128-335 and blast/mblookup.rs:106-235 as one
// CSR per query.  Every lw-mer of [fwd | N | rc] whose bases are all A/C/G/T, inside a context
// at least word_size long, goes to cell `code`; a stable radix sort by (query, code) keeps the
// positions ascending, and the megablast tables (lw > 8) are reversed per cell, which is the
// order their hash chains return (mblookup.rs:80-95).
// ---------------------------------------------------------------------------------------
#include <cub/device/device_radix_sort.cuh>

namespace rmb {

constexpr uint32_t NO_CODE = 0xffffffffu;

__global__ void k_lut_codes(DevQueries Q, int32_t ws, const uint64_t* __restrict__ pos_off,
                            uint32_t* __restrict__ keys, uint32_t* __restrict__ vals, uint32_t* __restrict__ counts) {
    const uint32_t qi = blockIdx.x;
    const uint32_t n = Q.len[qi];
    const int lw = Q.lw[qi];
    const uint8_t* q = Q.qmask + Q.off[qi];     // sentinel-wrapped forward query (DUST-masked)
    const uint8_t* r = Q.qmask_rc + Q.off[qi];  // its reverse complement
    const uint64_t base = pos_off[qi];
    const uint64_t cbase = Q.cs_off[qi];
    const uint32_t total = 2 * n + 1;
    const bool ok = (int64_t)ws <= (int64_t)n;  // each context is n bases long
    for (uint32_t s = threadIdx.x; s < total; s += blockDim.x) {
        uint32_t code = NO_CODE;
        if (ok && s != n) {
            // context 0 = [0, n-1], context 1 = [n+1, 2n]
            const uint32_t ctx_end = s < n ? n - 1 : 2 * n;
            if (s + (uint32_t)lw - 1 <= ctx_end) {
                uint32_t c = 0;
                bool valid = true;
                for (int k = 0; k < lw; ++k) {
                    const uint32_t t = s + k;
                    const uint8_t b = t < n ? q[1 + t] : r[1 + (t - n - 1)];
                    if (b & 0xFC) { valid = false; break; }
                    c = (c << 2) | b;
                }
                if (valid) code = c;
            }
        }
        keys[base + s] = code == NO_CODE ? NO_CODE : (uint32_t)(cbase + code);
        vals[base + s] = s;
        if (code != NO_CODE) atomicAdd(counts + cbase + code, 1u);
    }
}

__global__ void k_lut_place(uint64_t n_valid, const uint32_t* __restrict__ keys, const uint32_t* __restrict__ vals,
                            const uint32_t* __restrict__ cs, const uint64_t* __restrict__ cs_off, const int32_t* lw,
                            uint32_t nq, uint32_t* __restrict__ cell_q) {
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n_valid;
         k += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t key = keys[k];
        // query of this key: last cs_off <= key
        uint32_t lo = 0, hi = nq;
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) / 2;
            if (cs_off[mid] <= key) lo = mid;
            else hi = mid;
        }
        uint64_t dst = k;
        if (lw[lo] > 8) dst = (uint64_t)cs[key + 1] - 1 - (k - cs[key]);  // reverse within the cell
        cell_q[dst] = vals[k];
    }
}

__global__ void k_lut_pv(uint64_t n_words_total, const uint64_t* __restrict__ pv_off, const uint64_t* __restrict__ cs_off,
                         const int32_t* __restrict__ lw, uint32_t nq, const uint32_t* __restrict__ counts,
                         uint32_t* __restrict__ pv) {
    for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < n_words_total;
         w += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t lo = 0, hi = nq;
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) / 2;
            if (pv_off[mid] <= w) lo = mid;
            else hi = mid;
        }
        const uint64_t cells = 1ull << (2 * lw[lo]);
        const uint64_t c0 = (w - pv_off[lo]) * 32;
        uint32_t bits = 0;
        for (uint32_t b = 0; b < 32 && c0 + b < cells; ++b)
            if (counts[cs_off[lo] + c0 + b]) bits |= 1u << b;
        pv[w] = bits;
    }
}

cudaError_t launch_lut_build(const DevQueries& Q, int32_t ws, uint32_t nq, const uint64_t* pos_off, uint64_t n_pos,
                             uint64_t n_cells, uint64_t n_pv, uint32_t* keys, uint32_t* vals, uint32_t* keys2,
                             uint32_t* vals2, uint32_t* counts, uint32_t* cs, uint32_t* cell_q, uint32_t* pv,
                             void* temp, size_t& temp_bytes, uint64_t& n_valid, cudaStream_t st) {
    // temp sizing pass
    size_t t_scan = 0, t_sort = 0;
    cudaError_t e = cub::DeviceScan::ExclusiveSum(nullptr, t_scan, counts, cs, (int64_t)n_cells + 1, st);
    if (e != cudaSuccess) return e;
    e = cub::DeviceRadixSort::SortPairs(nullptr, t_sort, keys, keys2, vals, vals2, (int64_t)n_pos, 0, 32, st);
    if (e != cudaSuccess) return e;
    const size_t need = t_scan > t_sort ? t_scan : t_sort;
    if (!temp || temp_bytes < need) {
        temp_bytes = need;
        return cudaErrorNotReady;  // caller grows temp and calls again
    }
    e = cudaMemsetAsync(counts, 0, (n_cells + 1) * sizeof(uint32_t), st);
    if (e != cudaSuccess) return e;
    k_lut_codes<<<nq, 512, 0, st>>>(Q, ws, pos_off, keys, vals, counts);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    size_t tb = temp_bytes;
    e = cub::DeviceScan::ExclusiveSum(temp, tb, counts, cs, (int64_t)n_cells + 1, st);
    if (e != cudaSuccess) return e;
    tb = temp_bytes;
    e = cub::DeviceRadixSort::SortPairs(temp, tb, keys, keys2, vals, vals2, (int64_t)n_pos, 0, 32, st);
    if (e != cudaSuccess) return e;
    uint32_t nv = 0;
    e = cudaMemcpyAsync(&nv, cs + n_cells, 4, cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return e;
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return e;
    n_valid = nv;
    if (nv) {
        const int blocks = (int)((nv + 255) / 256 < 65536 ? (nv + 255) / 256 : 65536);
        k_lut_place<<<blocks, 256, 0, st>>>(nv, keys2, vals2, cs, Q.cs_off, Q.lw, nq, cell_q);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    const int pb = (int)((n_pv + 255) / 256 < 65536 ? (n_pv + 255) / 256 : 65536);
    k_lut_pv<<<pb, 256, 0, st>>>(n_pv, Q.pv_off, Q.cs_off, Q.lw, nq, counts, pv);
    return cudaGetLastError();
}

}  // namespace rmb

namespace rmb {
// reverse complement of every sentinel-wrapped query (encoding.rs:136 revcomp_blastna)
__global__ void k_revcomp(const uint8_t* __restrict__ q, const uint64_t* __restrict__ off,
                          const uint32_t* __restrict__ len, uint8_t* __restrict__ rc) {
    __shared__ uint8_t comp[16];
    if (threadIdx.x < 16) {
        const uint8_t c[16] = {3, 2, 1, 0, 5, 4, 7, 6, 8, 9, 13, 12, 11, 10, 14, 15};
        comp[threadIdx.x] = c[threadIdx.x];
    }
    __syncthreads();
    const uint64_t o = off[blockIdx.x];
    const uint32_t n = len[blockIdx.x] + 2;
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) rc[o + i] = comp[q[o + n - 1 - i] & 15];
}

cudaError_t launch_revcomp(const uint8_t* q, const uint64_t* off, const uint32_t* len, uint32_t nq, uint8_t* rc,
                           cudaStream_t st) {
    if (!nq) return cudaSuccess;
    k_revcomp<<<nq, 256, 0, st>>>(q, off, len, rc);
    return cudaGetLastError();
}

// DUST masking (filter/dust.rs:462-489).  A query's pass is one sequential chain of data-dependent
// branches, so each query gets a warp of its own with one working lane: lanes of one warp on
// different queries would diverge at nearly every step and run one after another.  Up to 32
// such warps share an SM.  Each worker's perfect-interval list is in `scratch`; qm holds a copy
// of q and gets the masked bases (code 14).
__global__ void __launch_bounds__(32) k_dust(const uint8_t* __restrict__ q, const uint64_t* __restrict__ off,
                                             const uint32_t* __restrict__ len, uint32_t nq, uint8_t* __restrict__ qm,
                                             DustPerfect* __restrict__ scratch, uint32_t nworkers,
                                             unsigned int* __restrict__ overflow, bool compat,
                                             uint32_t* __restrict__ bits, const uint64_t* __restrict__ bits_off) {
    if (threadIdx.x != 0 || blockIdx.x >= nworkers) return;
    for (uint32_t i = blockIdx.x; i < nq; i += nworkers) {
        const uint64_t o = off[i] + 1;
        if (!dust_query(q + o, len[i], qm ? qm + o : nullptr, scratch + (uint64_t)blockIdx.x * DUST_PERFECT_CAP,
                        compat, bits ? bits + bits_off[i] : nullptr))
            atomicAdd(overflow, 1u);
    }
}

uint32_t dust_threads(uint32_t nq, int sms) {
    const uint32_t cap = (uint32_t)sms * 32u;  // one working lane per warp, 32 single-warp blocks per SM
    return nq < cap ? nq : cap;
}
size_t dust_scratch_bytes(uint32_t nthreads) { return (size_t)nthreads * DUST_PERFECT_CAP * sizeof(DustPerfect); }

cudaError_t launch_dust(const uint8_t* q, const uint64_t* off, const uint32_t* len, uint32_t nq, uint8_t* qm,
                        void* scratch, uint32_t nthreads, unsigned int* overflow, bool compat, cudaStream_t st,
                        uint32_t* bits, const uint64_t* bits_off) {
    if (!nq || !nthreads) return cudaSuccess;
    k_dust<<<nthreads, 32, 0, st>>>(q, off, len, nq, qm, (DustPerfect*)scratch, nthreads, overflow, compat, bits,
                                    bits_off);
    return cudaGetLastError();
}
}  // namespace rmb

// ---------------------------------------------------------------------------------------
// Traceback without allocation (rmb_traceback_noalloc in include/rmb_gpu.h).
//
// For callers that may not call cudaMalloc: a library embedded in a process whose device memory
// is owned by another allocator (a caching allocator that must see every byte, a stream-ordered
// pool), or code running where an allocation could fail or stall.  The per-thread scratch of the
// traceback (DP band, row table, trace bytes) comes from this fixed array, which every GPU that
// loads the library holds until the process exits.
// ---------------------------------------------------------------------------------------
#include <mutex>

#include "../../include/rmb_gpu.h"

namespace rmb {

constexpr uint64_t NOALLOC_SCRATCH_BYTES = 32ull << 20;  // 32 MiB
constexpr uint32_t NOALLOC_MAX_THREADS = 256;

static __device__ __align__(256) uint8_t g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];
// [0] records that did not fit their share of the scratch (status 2), [1] records whose edit
// script did not fit ops_cap (status 5)
static __device__ unsigned int g_noalloc_overflow[2];

struct NoallocSeqs {
    const uint8_t* q;      // query, sentinel-wrapped
    const uint8_t* qrc;    // its reverse complement, sentinel-wrapped
    const uint8_t* s;      // subject with ambiguity codes restored, sentinel-wrapped
    const uint8_t* src;    // its reverse complement, sentinel-wrapped
    uint32_t qlen, slen;
};

// k_traceback for one (query, subject) pair: the same improve_seed + bidirectional traceback +
// gap pruning, the scratch taken from `scratch` (the address of g_noalloc_scratch).  With
// `retry` set, only the records whose status is 2 (scratch too small) from an earlier launch
// with more threads run again, each thread now holding a larger share of the array.
// Record status: 0 aligned, 1 negative score, 2 scratch too small, 3 the trace walk did not
// reach the seed, 4 record outside the sequences (skipped), 5 edit script longer than ops_cap.
__global__ void __launch_bounds__(128) k_traceback_noalloc(NoallocSeqs S, DevParams P, uint32_t n,
                                                            const uint32_t* __restrict__ pre,
                                                            uint32_t* __restrict__ out, uint32_t* __restrict__ ops_out,
                                                            uint32_t ops_cap, uint8_t* __restrict__ scratch,
                                                            uint64_t per_thread, uint64_t band_cells,
                                                            uint32_t rows_cap, unsigned int* overflow, bool retry) {
    __shared__ int32_t mat[256];
    for (int i = threadIdx.x; i < 256; i += blockDim.x) mat[i] = P.matrix[i];
    __syncthreads();
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    uint8_t* base = scratch + tid * per_thread;
    TbScratch T;
    T.band = (int2*)base;
    T.rows = (uint2*)(base + band_cells * sizeof(int2));
    T.rows_cap = rows_cap;
    T.trace = base + band_cells * sizeof(int2) + (uint64_t)rows_cap * sizeof(uint2);
    T.trace_cap = per_thread - band_cells * sizeof(int2) - (uint64_t)rows_cap * sizeof(uint2);
    const uint32_t qa = S.qlen, sa = S.slen;
    for (uint64_t t = tid; t < n; t += (uint64_t)gridDim.x * blockDim.x) {
        // record: strand, q_start, q_end, s_start, s_end, score, q_seed, s_seed
        const uint32_t* r = pre + t * 8;
        uint32_t* o = out + t * 9;
        if (retry && o[1] != 2u) continue;
        // the caller's records are checked before any sequence byte is read: the box inside both
        // sequences and the seed inside both (improve_seed and the DPs index from them)
        const bool in_range = r[0] <= 1u && r[1] <= r[2] && r[2] <= qa && r[3] <= r[4] && r[4] <= sa &&
                              r[6] < qa && r[7] < sa;
        uint32_t nq = 0, ns = 0;
        const bool plus = r[0] == 0;
        if (in_range)
            improve_seed(S.q + 1, qa, (plus ? S.s : S.src) + 1, sa, r[6], r[7], r[1], r[2], r[3], r[4], !plus, nq, ns);
        if (!in_range || nq >= qa || ns >= sa) {
            o[0] = r[0];
            o[1] = 4u;  // outside the sequences: skipped
            for (int k = 2; k < 9; ++k) o[k] = 0;
            continue;
        }
        const uint32_t tq = plus ? nq : qa - 1 - nq, ts = plus ? ns : sa - 1 - ns;
        const uint8_t* qa_ = (plus ? S.q : S.qrc) + 1;
        const uint8_t* sa_ = S.s + 1;
        uint32_t* ops = ops_out + t * (uint64_t)ops_cap;
        uint64_t cells = 0, need = 0;
        int32_t ls, rs = 0;
        uint32_t la, lb, ra = 0, rb = 0, nl = 0, nr = 0;
        int st = align_ex_tb<true>(qa_, sa_, tq + 1, ts + 1, P.gap_open, P.gap_extend, P.xdrop_gap_final, mat, T, ls,
                                   la, lb, ops, ops_cap, nl, cells, need);
        if (st == 0) {
            const uint32_t rq = tq + 1, rsd = ts + 1;
            const uint32_t rm = qa > rq ? qa - rq : 0, rn = sa > rsd ? sa - rsd : 0;
            if (rm > 0 && rn > 0)
                st = align_ex_tb<false>(qa_ + rq, sa_ + rsd, rm, rn, P.gap_open, P.gap_extend, P.xdrop_gap_final, mat,
                                        T, rs, ra, rb, ops + nl, ops_cap - nl, nr, cells, need);
        }
        if (st != 0) {
            // align_ex_tb: 3 = the walk did not reach the seed; 2 with need > 0 = the trace did not
            // fit the thread's scratch; 2 with need = 0 = the script did not fit ops_cap
            const uint32_t code = st == 3 ? 3u : need > 0 ? 2u : 5u;
            if (code == 2u) atomicAdd(overflow, 1u);
            if (code == 5u) atomicAdd(overflow + 1, 1u);
            o[0] = r[0];
            o[1] = code;
            for (int k = 2; k < 9; ++k) o[k] = 0;
            continue;
        }
        for (uint32_t i = 0, j = nr ? nr - 1 : 0; i < j; ++i, --j) {
            const uint32_t tmp = ops[nl + i];
            ops[nl + i] = ops[nl + j];
            ops[nl + j] = tmp;
        }
        uint32_t nops = nl;
        for (uint32_t i = 0; i < nr; ++i) {
            const uint32_t v = ops[nl + i];
            if (nops > 0 && (ops[nops - 1] >> 30) == (v >> 30)) ops[nops - 1] += v & 0x3fffffffu;
            else ops[nops++] = v;
        }
        int32_t total = ls + rs;
        uint32_t q_start = tq + 1 - la, s_start = ts + 1 - lb, q_end = tq + 1 + ra, s_end = ts + 1 + rb;
        uint32_t first = 0;
        while (first < nops && (ops[first] >> 30) != 0) {
            const uint32_t op = ops[first] >> 30, cnt = ops[first] & 0x3fffffffu;
            total += P.gap_open + (int32_t)cnt * P.gap_extend;
            if (op == 1) s_start += cnt;
            else q_start += cnt;
            ++first;
        }
        while (nops > first && (ops[nops - 1] >> 30) != 0) {
            const uint32_t op = ops[nops - 1] >> 30, cnt = ops[nops - 1] & 0x3fffffffu;
            total += P.gap_open + (int32_t)cnt * P.gap_extend;
            if (op == 1) s_end -= cnt;
            else q_end -= cnt;
            --nops;
        }
        if (first) {
            for (uint32_t i = first; i < nops; ++i) ops[i - first] = ops[i];
            nops -= first;
        }
        o[0] = r[0];
        if (total < 0) {
            o[1] = 1u;
            for (int k = 2; k < 8; ++k) o[k] = 0;
            o[8] = 2166136261u;
            continue;
        }
        uint32_t h = 2166136261u;
        for (uint32_t i = 0; i < nops; ++i)
            for (int b = 0; b < 4; ++b) h = (h ^ ((ops[i] >> (8 * b)) & 0xffu)) * 16777619u;
        o[1] = 0u;
        o[2] = (uint32_t)total;
        o[3] = q_start;
        o[4] = q_end;
        o[5] = s_start;
        o[6] = s_end;
        o[7] = nops;
        o[8] = h;
    }
}

// Device address of the scratch array and the overflow counter, looked up once per device.
static std::mutex g_noalloc_mu;
static void* g_noalloc_addr[64];
static void* g_noalloc_flag[64];

static cudaError_t noalloc_setup(int device, uint8_t** scratch, unsigned int** flag) {
    std::lock_guard<std::mutex> g(g_noalloc_mu);
    if (device < 0 || device >= 64) return cudaErrorInvalidDevice;
    if (!g_noalloc_addr[device]) {
        void* a = nullptr;
        void* f = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&a, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        e = cudaGetSymbolAddress(&f, g_noalloc_overflow);
        if (e != cudaSuccess) return e;
        g_noalloc_addr[device] = a;
        g_noalloc_flag[device] = f;
    }
    *scratch = (uint8_t*)g_noalloc_addr[device];
    *flag = (unsigned int*)g_noalloc_flag[device];
    return cudaSuccess;
}

}  // namespace rmb

extern "C" int rmb_traceback_noalloc(int32_t device, const uint8_t* query, const uint8_t* query_rc, uint32_t qlen,
                                     const uint8_t* subject, const uint8_t* subject_rc, uint32_t slen,
                                     const uint32_t* prelims, uint32_t n, int32_t gap_open, int32_t gap_extend,
                                     int32_t xdrop_gap_final, const int32_t scores[256], uint32_t* out,
                                     uint32_t* ops, uint32_t ops_cap, void* stream, char* err, size_t errlen) {
    using namespace rmb;
    auto fail = [&](int code, const char* msg) {
        if (err && errlen) {
            size_t i = 0;
            for (; msg[i] && i + 1 < errlen; ++i) err[i] = msg[i];
            err[i] = 0;
        }
        return code;
    };
    if (!query || !query_rc || !subject || !subject_rc || !scores || (n && (!prelims || !out || !ops)))
        return fail(RMB_EINVAL, "null argument");
    if (ops_cap == 0) return fail(RMB_EINVAL, "ops_cap must be positive");
    if (gap_open < 0 || gap_extend < 1 || xdrop_gap_final < 0) return fail(RMB_EINVAL, "gap costs or X-drop out of range");
    // band (slen + 2 cells) + row table (qlen + 2 rows) + at least 64 KiB of trace per thread
    const uint64_t band_cells = (uint64_t)slen + 2;
    const uint32_t rows_cap = qlen + 2;
    const uint64_t fixed = band_cells * sizeof(int2) + (uint64_t)rows_cap * sizeof(uint2);
    const uint64_t min_thread = ((fixed + (64ull << 10)) + 255) & ~255ull;
    if (min_thread > NOALLOC_SCRATCH_BYTES)
        return fail(RMB_ELIMIT, "query and subject too long for the 32 MiB scratch of rmb_traceback_noalloc "
                                "(8 bytes x (subject + 2) + 8 bytes x (query + 2) + 64 KiB must fit)");
    // the caller's current device is put back on every return
    int caller_device = -1;
    cudaError_t e = cudaGetDevice(&caller_device);
    if (e != cudaSuccess) return fail(RMB_ECUDA, cudaGetErrorString(e));
    struct RestoreDevice {
        int d;
        ~RestoreDevice() { cudaSetDevice(d); }
    } restore{caller_device};
    if ((e = cudaSetDevice(device)) != cudaSuccess) return fail(RMB_ECUDA, cudaGetErrorString(e));
    uint8_t* scratch = nullptr;
    unsigned int* flag = nullptr;
    if ((e = noalloc_setup(device, &scratch, &flag)) != cudaSuccess) return fail(RMB_ECUDA, cudaGetErrorString(e));
    if (n == 0) return RMB_OK;
    cudaStream_t st = (cudaStream_t)stream;
    DevParams P{};
    P.gap_open = gap_open;
    P.gap_extend = gap_extend;
    P.xdrop_gap_final = xdrop_gap_final;
    for (int i = 0; i < 256; ++i) P.matrix[i] = scores[i];
    NoallocSeqs S{query, query_rc, subject, subject_rc, qlen, slen};
    uint32_t threads = (uint32_t)(NOALLOC_SCRATCH_BYTES / min_thread);
    if (threads > NOALLOC_MAX_THREADS) threads = NOALLOC_MAX_THREADS;
    if (threads > n) threads = n;
    // Records whose trace did not fit a thread's share run again with a quarter of the threads,
    // so each gets four times the space, down to one thread holding the whole array.
    unsigned int over[2] = {0, 0};
    for (bool retry = false;; retry = true) {
        const uint32_t block = threads >= 128 ? 128 : threads;
        const uint32_t grid = threads / block;
        const uint64_t per_thread = (NOALLOC_SCRATCH_BYTES / ((uint64_t)grid * block)) & ~255ull;  // >= min_thread
        if ((e = cudaMemsetAsync(flag, 0, 2 * sizeof(unsigned int), st)) != cudaSuccess)
            return fail(RMB_ECUDA, cudaGetErrorString(e));
        k_traceback_noalloc<<<grid, block, 0, st>>>(S, P, n, prelims, out, ops, ops_cap, scratch, per_thread,
                                                     band_cells, rows_cap, flag, retry);
        if ((e = cudaGetLastError()) != cudaSuccess) return fail(RMB_ECUDA, cudaGetErrorString(e));
        unsigned int o[2] = {0, 0};
        if ((e = cudaMemcpyAsync(o, flag, sizeof o, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
            return fail(RMB_ECUDA, cudaGetErrorString(e));
        if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return fail(RMB_ECUDA, cudaGetErrorString(e));
        over[0] = o[0];
        over[1] += o[1];
        if (!over[0] || threads == 1) break;
        threads = threads >= 4 ? threads / 4 : 1;
    }
    if (over[0])
        return fail(RMB_ELIMIT, "some alignments did not fit the 32 MiB scratch even on one thread (status 2 in "
                                "their records)");
    if (over[1]) return fail(RMB_ELIMIT, "some edit scripts were longer than ops_cap (status 5 in their records)");
    return RMB_OK;
}
