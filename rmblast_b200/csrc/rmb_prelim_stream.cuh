#pragma once
// Thread-per-extension score-only X-drop DP over a flat cell stream (the body of k_prelim_stream).
//
// Each thread runs the two extensions of one ungapped record after another (left, reversed,
// then right), and takes the next record from a grid-wide queue when it is done.  The cell step
// is the reference's (search/gapped.rs:222-296); the row end is gapped.rs:298-334 and the
// initial row gapped.rs:165-200.
//
// Lanes of a warp work in groups of U cell steps.  A lane whose row ends inside a group sits out
// the rest of the group, and every lane whose row ended runs its row end after the group, in one
// branch: row ends (~22 cells apart, at a different cell on every lane) then cost one divergent
// block per group instead of one per cell step, at the price of ~(U - 1) / 2 idle cell steps a
// row.  Record changes happen in the same place.  A warp-wide vote at the top of every group
// brings the lanes back together.  The cell step itself has no branch: a lane that sits out runs
// it on a MININT cell with its store and its gap_row update predicated off (measured on the B200:
// 10 % fewer instructions and 60 % fewer branches than a guarded step, 14 % less time).
//
// Storage differs from the reference's in three ways, none of which changes a result:
//  - The band entries that the reference writes in a loop, the initial row (gapped.rs:187-200)
//    and the end-of-row extension cells (gapped.rs:307-319), are not written: a row computes
//    them from (vlo, nvirt, ext_val) when it reads them, a few predicated operations a cell
//    (cheaper than a loop in the row end, which runs divergently).  The MININT sentinel
//    (gapped.rs:325-330) is read the same way, as the virtual index after them.
//  - An entry is 32 bits: bits 0-3 the column residue, bits 4-17 the cell and bits 18-31 the
//    vertical gap, both as 14-bit values relative to the extension's origin and clamped below at
//    FLOOR.  The DP runs in the same frame, so entries are read and written without conversion.
//    The origin starts at score 0 and moves up to the best score at a row end where the best
//    has passed REBASE, so stored values (never above the best) stay below 4096 + 127, and the
//    threshold best - X stays at or above -X >= -8000 (X <= 8000, scores <= 127, checked by the
//    host).  A value below FLOOR stays below every later threshold even after adding the best
//    score, so the clamp only moves values that can no longer make a cell survive (MININT
//    included).  The residues of a row's band are copied in (a word of the column sequence at a
//    time) at the row end that sets the band, so the cell step reads the residue with the entry.
//  - The band window of a row (b_size - first_b cells) must fit the launch's window (at most
//    STREAM_WINDOW); a record whose window grows past it, or whose cell count passes the budget,
//    is listed for the warp kernel.
#include <cstdint>

#include "rmb_device.cuh"

namespace rmb {

constexpr int STREAM_RING = 64;
// The band window of a row may span at most this many indices: whole-word residue fills run up
// to 3 indices past its end, which must stay inside the ring.
constexpr int STREAM_WINDOW = 60;
// A record whose two extensions pass `max_cells` cells is handed to the warp kernel, so that a few
// extensions millions of cells long cannot hold their thread (and the end of the launch) for a
// large part of the launch.  A thread does ~3 M cells/s, so the budget sets the worst tail; the
// host makes it records / 128 within [STREAM_MIN_CELLS, STREAM_MAX_CELLS].  On the 132 M records
// of the plain workload the 2^20 budget adds ~13 ms of tail to an ~830 ms launch while the warp
// kernel's share drops from 11 G cells (~130 ms) to 0.06 G; a launch of 1.3 M records keeps a
// ~3 ms tail with its 10 k budget (a 65 k budget there made a 20 ms launch of a 9 ms one).
constexpr uint32_t STREAM_MIN_CELLS = 8192, STREAM_MAX_CELLS = 1u << 20;
constexpr int STREAM_BLOCK = 128;
constexpr int STREAM_BLOCKS_PER_SM = 6;
constexpr int32_t STREAM_FLOOR = -8192;
// the origin moves to the best score when the best passes this (stored values stay <= 4096 + 127)
constexpr int32_t STREAM_REBASE = 4096;

// One record's DP geometry (engine.rs:1350-1372), written by k_prelim_prep so that the DP kernel
// starts a record with one 48-byte load: query and subject sequence starts (record frame),
// their lengths, the pivot, the traceback seed, X = max(min(xdrop_gap, ungapped score),
// gap_open + gap_extend), and the strand with the first row residue of each extension.
struct __align__(16) PrelimGeo {
    uint64_t qseq, sseq;
    uint32_t qa, sa, qp, sp;
    uint32_t tbq, tbs, xdrop, flags;  // flags: plus | a[sp - 1] << 8 | a[sp] << 16
};

// Entry from (cell, vertical gap), both relative and in [FLOOR, -FLOOR), keeping w's residue.
__host__ __device__ __forceinline__ uint32_t stream_pack(int32_t ex, int32_t ey, uint32_t w) {
    return (w & 15u) | (((uint32_t)ex << 4) & 0x3fff0u) | ((uint32_t)ey << 18);
}

// Constants of one launch.
struct StreamArgs {
    const int32_t* smat;  // 16 x 16 scores, clamped below at -(X + 1) for the largest X
    int32_t ge, goe, cutoff;
    uint64_t n;
    const PrelimGeo* geo;
    PrelimOut* out;
    uint32_t max_cells;
    const uint32_t* order = nullptr;  // queue position -> record (a cost order); null: FIFO
    uint32_t* cells_out = nullptr;    // per-record DP cells (UINT32_MAX: passed on), or null
    uint32_t window = STREAM_WINDOW;  // widest band window kept by the thread (<= STREAM_WINDOW)
    // a front-loaded order: queue positions below n_front read order[p], the others read the
    // order from its end (order[order_end - 1 - (p - n_front)]), where a partition left them
    uint32_t n_front = 0xFFFFFFFFu;
    uint64_t order_end = 0;
};

// floor(num / d) for 0 <= num <= 8000 and 1 <= d <= 8000: num * ceil(2^32 / d) >> 32 (exact for
// num < 2^32 / (d - 1)); d = 1 passes num through.
struct StreamDiv {
    uint32_t m;
    __host__ __device__ explicit StreamDiv(int32_t d) : m(d > 1 ? (uint32_t)((0xFFFFFFFFull + (uint64_t)d) / (uint64_t)d) : 0u) {}
    __host__ __device__ __forceinline__ uint32_t operator()(uint32_t num) const {
#ifdef __CUDA_ARCH__
        return m ? __umulhi(num, m) : num;
#else
        return m ? (uint32_t)(((uint64_t)num * m) >> 32) : num;
#endif
    }
};

// The work of one thread until the record queue is empty; returns the DP cells of the records
// it completed.  Env supplies the thread's ring (`uint32_t& at(j)`: the entry of band index j,
// slot j % STREAM_RING), the queue (`uint32_t take()`), the overflow list (`overflow(t)`), a
// warp-wide vote (`bool any(bool)`) and `fill_rows(pending, qal, pb, dir, n)`: called by every
// lane of the warp together, it sets entry k (k < n) of each pending lane's ring to the residue
// qal[pb + dir * k] & 15.
template <int U, class Env>
__host__ __device__ __forceinline__ unsigned long long prelim_stream_thread(const StreamArgs& A, Env& env) {
    const int32_t ge = A.ge, goe = A.goe;
    const StreamDiv div_ge(ge);

    // record
    uint64_t t = 0;
    uint32_t qa = 0, sa = 0, qp = 0, sp = 0, tbq = 0, tbs = 0, rec_cells = 0;
    bool plus = true;
    int32_t xdrop = 0;
    const uint8_t *qseq = nullptr, *sseq = nullptr;
    int32_t l_score = 0;
    uint32_t l_a = 0, l_b = 0;
    int phase = 0;  // 0: need a record, 1: left extension, 2: right extension, 3: no right extension
    // extension: row residue a[ai] at abase[dir * ai]; column residue b[bi] at qal[pb + dir * bi]
    const uint8_t *abase = nullptr, *qal = nullptr;
    int32_t dir = 1, pb = 0, r0 = 0;
    uint32_t filled = 0;  // residues of band indices [.., filled) are in the ring
    uint8_t a_nx = 0, a0_left = 0, a0_right = 0;
    const int32_t* srow = A.smat;
    uint32_t m = 0, nb = 0, ai = 0, bi = 0, first_b = 0, b_size = 0, last_b = 0, best_a = 0, best_b = 0;
    uint32_t first_alive = 0xFFFFFFFFu;  // the current row's first live cell
    // scores relative to `origin` (the extension's score 0 until the first rebase)
    int32_t best = 0, prev_best = 0, thr = 0, sc = 0, gap_row = 0, origin = 0;
    // the extension cells of the last row end (gapped.rs:307-319), computed when read: band
    // indices vlo .. vlo + nvirt - 1 hold ext_val - (j - vlo) * ge and that minus gap_open_extend
    uint32_t vlo = 0, nvirt = 0;
    int32_t ext_val = 0;
    unsigned long long cells = 0;
    // records come from one queue; the next index is fetched one record ahead
    uint32_t next_t = env.take();
    bool fetch = true;  // no extension running: finish the last one and start the next
    bool dp_fail = false;
    bool out_of_records = false;
    bool init_pending = false;  // an extension started whose initial residues are not in yet

    auto new_row = [&]() {
        srow = A.smat + (uint32_t)(a_nx & 15) * 16u;
        if (ai + 1 < m) a_nx = abase[(ptrdiff_t)dir * (ptrdiff_t)(ai + 1)];  // next row's residue
        sc = MININT; gap_row = MININT;
        last_b = first_b; prev_best = best; bi = first_b; first_alive = 0xFFFFFFFFu;
        rec_cells += b_size - first_b;
    };
    // The residues of the band indices of one aligned word of the column sequence, from the
    // word holding index `filled`'s residue (the other entry bits cleared).  `filled` sits on a
    // word boundary (the initial fill stops on one), so the word's indices are filled .. +3:
    // below the window's end + 3 < first_b + RING (the window is at most STREAM_WINDOW).
    auto fill_word = [&]() {
        const int32_t addr = pb + dir * (int32_t)filled;
        uint32_t wv = *(const uint32_t*)(qal + (ptrdiff_t)(addr & ~3));
        int32_t i0;
        if (dir > 0) {
            i0 = (int32_t)filled - (addr & 3);
        } else {
            i0 = (int32_t)filled - (3 - (addr & 3));
#ifdef __CUDA_ARCH__
            wv = __byte_perm(wv, 0, 0x0123);  // band order
#else
            wv = __builtin_bswap32(wv);
#endif
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) env.at((uint32_t)(i0 + q)) = (wv >> (8 * q)) & 15u;
        filled = (uint32_t)(i0 + 4);
    };

    for (;;) {
        if (!env.any(!out_of_records)) break;
        // U cell steps (gapped.rs:234-296); a lane whose row has ended waits for the row end
#pragma unroll
        for (int u = 0; u < U; ++u) {
            {
                // every lane runs the step; one whose row has ended computes a dead cell from
                // MININT, stores nothing and keeps its gap_row for the row end
                const bool act = bi < b_size;
                uint32_t& slot = env.at(bi);
                const uint32_t w = slot;
                const uint32_t rel = bi - vlo;
                const bool virt = rel < nvirt;
                const int32_t v = ext_val - (int32_t)rel * ge;
                const int32_t cx = virt ? v : (int32_t)(w << 14) >> 18;
                const int32_t cy = virt ? v - goe : (int32_t)w >> 18;
                // the diagonal of the next cell; at bi == nb (the row's last cell) it is not used
                const int32_t nxt = cx + srow[w & 15u];
                const int32_t cell = act ? __vimax3_s32(sc, cy, gap_row) : MININT;
                const bool alive = cell >= thr;
                if (alive) first_alive = min(first_alive, bi);
                if (alive) last_b = bi;
                if (cell > best) best_b = bi;
                best = max(best, cell);
                thr = __viaddmax_s32(cell, -xdrop, thr);  // best - xdrop
                const int32_t open = cell - goe;
                // at a dead cell the reference keeps gap_row and the vertical gap; both are then
                // below the threshold (cell >= each), and so is what is kept here, so they stay dead
                if (act) gap_row = __viaddmax_s32(gap_row, -ge, open);
                const int32_t ex = alive ? cell : STREAM_FLOOR;
                const int32_t ey = __vimax3_s32(cy - ge, open, STREAM_FLOOR);
                if (act) slot = stream_pack(ex, ey, w);
                sc = nxt;
                ++bi;
            }
        }
        if (!fetch && bi >= b_size) {
            // end of row (gapped.rs:298-334).  The band keeps [first_b, last_b] and, when the
            // row's last cell survived, extends by the k cells that gap_row keeps above the
            // threshold; a MININT sentinel follows while the band has not reached nb.
            if (best > prev_best) best_a = ai + 1;
            ++ai;
            // the band's first cell: the row's first live cell (gapped.rs:265-268 advance it over
            // the leading dead ones), b_size when none lived
            first_b = min(first_alive, b_size);
            const bool empty = first_b >= b_size;
            vlo = last_b + 1;
            uint32_t k = 0;
            const int32_t num = gap_row - thr;  // <= xdrop (gap_row never exceeds best)
            if (vlo == b_size && b_size <= nb && num >= 0) {
                const uint32_t kk = div_ge((uint32_t)num) + 1u;
                k = kk < nb + 1 - b_size ? kk : nb + 1 - b_size;
            }
            const uint32_t nbs = vlo + k;
            b_size = nbs + (nbs <= nb ? 1u : 0u);
            const uint32_t width = b_size - first_b;
            if (empty || ai >= m || width > A.window || rec_cells + width > A.max_cells) {
                dp_fail = !empty && ai < m;
                fetch = true;
                b_size = 0;  // no cell steps until the next extension starts
            } else {
                if (best > STREAM_REBASE) {
                    // move the origin to the best score: the entries the next row reads from the
                    // ring shift with it (values pushed below FLOOR are dead: the threshold is
                    // then -xdrop >= FLOOR + max score)
                    const int32_t d = best;
                    for (uint32_t j = first_b; j < vlo; ++j) {
                        uint32_t& e = env.at(j);
                        const uint32_t w = e;
                        e = stream_pack(max(((int32_t)(w << 14) >> 18) - d, STREAM_FLOOR),
                                        max(((int32_t)w >> 18) - d, STREAM_FLOOR), w);
                    }
                    origin += d; best = 0; thr -= d; gap_row -= d;
                }
                while (filled < b_size) fill_word();
                // the k extension cells and the sentinel after them are read as computed values:
                // the sentinel's (index nbs, k past vlo) vertical gap ext_val - k * ge - goe is
                // below the threshold like the reference's MININT (k = 0: then gap_row is below
                // it, or the band's end cell did not live), and its diagonal feeds no cell (it
                // is the row's last)
                nvirt = k + 1u;
                ext_val = gap_row;
                new_row();
            }
        }
        if (fetch && !out_of_records) {
            // the extension that just ended (best, best_a, best_b; zero for an empty one), then the
            // next non-empty extension
            while (fetch) {
                if (phase != 0 && dp_fail) {
                    env.overflow((uint32_t)t);
                    if (A.cells_out) A.cells_out[t] = 0xFFFFFFFFu;
                    phase = 0;
                }
                if (phase == 1) {
                    l_score = best + origin; l_a = best_a; l_b = best_b;
                    const uint32_t rm = sa > sp ? sa - sp : 0, rn = qa > qp ? qa - qp : 0;
                    if (rm > 0 && rn > 0) {
                        abase = sseq + sp; pb = r0 + (int32_t)qp; m = rm; nb = rn; dir = 1;
                        phase = 2;
                    } else {
                        best = 0; best_a = 0; best_b = 0; origin = 0;
                        phase = 3;
                    }
                } else if (phase == 2 || phase == 3) {
                    // both extensions done: engine.rs:1380-1397
                    PrelimOut o{INT32_MIN, 0, 0, 0, 0, 0, 0};
                    const int32_t total = l_score + best + origin;
                    if (total >= 0) {
                        uint32_t q0 = qp - l_b, s0 = sp - l_a, q1 = qp + best_b, s1 = sp + best_a;
                        if (!plus) {
                            const uint32_t t0 = qa - q1, t1 = qa - q0, t2 = sa - s1, t3 = sa - s0;
                            q0 = t0; q1 = t1; s0 = t2; s1 = t3;
                        }
                        if (total >= A.cutoff) o = PrelimOut{total, q0, q1, s0, s1, tbq, tbs};
                    }
                    A.out[t] = o;
                    if (A.cells_out) A.cells_out[t] = rec_cells;
                    cells += rec_cells;
                    phase = 0;
                }
                if (phase == 0) {
                    // next record
                    if (next_t >= A.n) { out_of_records = true; break; }
                    t = !A.order ? next_t
                        : next_t < A.n_front ? A.order[next_t]
                                             : A.order[A.order_end - 1 - (uint64_t)(next_t - A.n_front)];
                    next_t = env.take();
                    const uint4* gp = reinterpret_cast<const uint4*>(A.geo + t);
                    const uint4 g0 = gp[0], g1 = gp[1], g2 = gp[2];
                    qseq = (const uint8_t*)(((uint64_t)g0.y << 32) | g0.x);
                    sseq = (const uint8_t*)(((uint64_t)g0.w << 32) | g0.z);
                    qa = g1.x; sa = g1.y; qp = g1.z; sp = g1.w;
                    tbq = g2.x; tbs = g2.y; xdrop = (int32_t)g2.z;
                    plus = g2.w & 1u;
                    a0_left = (uint8_t)(g2.w >> 8);
                    a0_right = (uint8_t)(g2.w >> 16);
                    qal = (const uint8_t*)((uintptr_t)qseq & ~(uintptr_t)3);
                    r0 = (int32_t)(qseq - qal);
                    rec_cells = 0;
                    abase = sseq; pb = r0; m = sp; nb = qp; dir = -1;
                    phase = 1;
                }
                if (phase == 3) continue;
                // start the extension set up above (gapped.rs:165-200)
                dp_fail = false;
                best = 0; best_a = 0; best_b = 0; origin = 0;
                if (m == 0 || nb == 0) continue;  // empty: result 0
                if (dir < 0) { abase += m - 1; pb += (int32_t)nb - 1; }
                const uint32_t jmax = div_ge((uint32_t)(xdrop - goe)) + 1u;
                const uint32_t J = jmax < nb ? jmax : nb;
                if (J + 1 > A.window) { dp_fail = true; continue; }
                // initial row: cell 0 written, the J gap cells -goe - (i - 1) * ge computed on read
                b_size = J + 1; vlo = 1; nvirt = J; ext_val = -goe;
                first_b = 0; ai = 0; thr = -xdrop;
                // residues of indices 0 .. filled - 1 come in below, with the warp's help: up to
                // the next word boundary of the column sequence, so later whole-word fills start
                // on one (at most 3 past b_size <= STREAM_WINDOW: inside the ring)
                filled = b_size + (uint32_t)(dir > 0 ? -(pb + (int32_t)b_size) & 3 : (pb - (int32_t)b_size + 1) & 3);
                init_pending = true;
                a_nx = dir < 0 ? a0_left : a0_right;
                new_row();
                fetch = false;
            }
        }
        // the initial rows of the extensions started above: all lanes copy residues into the
        // rings of the lanes that started one, one band index a lane at a time
        env.fill_rows(init_pending, qal, pb, dir, filled);
        if (init_pending) {
            env.at(0) = stream_pack(0, -goe, env.at(0));
            init_pending = false;
        }
    }
    return cells;
}

}  // namespace rmb
