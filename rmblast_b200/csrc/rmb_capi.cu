// rmb_capi.cu -- the C ABI of include/rmb_gpu.h: context, library upload, the batched search
// pipeline (GPU stages + host order-dependent filters) and result packing.
#include <algorithm>
#include <cmath>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <future>
#include <memory>
#include <mutex>
#include <new>
#include <sstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../../include/rmb_gpu.h"
#include "rmb_device.cuh"
#include "rmb_glue.hpp"
#include "rmb_kernels.hpp"

using namespace rmb;

namespace {

struct Fail : std::runtime_error {
    int code;
    Fail(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define CK(x)                                                                                          \
    do {                                                                                               \
        cudaError_t e_ = (x);                                                                          \
        if (e_ != cudaSuccess)                                                                         \
            throw Fail(e_ == cudaErrorMemoryAllocation ? RMB_ENOMEM : RMB_ECUDA,                        \
                       std::string(#x) + ": " + cudaGetErrorString(e_));                                \
    } while (0)

struct DBuf {  // growable device buffer
    void* p = nullptr;
    size_t cap = 0;
    void ensure(size_t n) {
        if (n <= cap && p) return;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        // whole 16-byte words, so an aligned word read around any valid byte stays inside
        size_t nc = std::max<size_t>((n + 15) & ~(size_t)15, 256);
        CK(cudaMalloc(&p, nc));
        cap = nc;
    }
    template <class T>
    T* as() const { return (T*)p; }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
    }
};

struct HostBuf {  // growable pinned host buffer (contents undefined after a resize)
    uint8_t* p = nullptr;
    size_t n = 0, cap = 0;
    HostBuf() = default;
    HostBuf(const HostBuf&) = delete;
    HostBuf& operator=(const HostBuf&) = delete;
    ~HostBuf() {
        if (p) cudaFreeHost(p);
    }
    void resize(size_t m) {
        if (m > cap) {
            if (p) cudaFreeHost(p);
            p = nullptr;
            cap = 0;
            CK(cudaMallocHost(&p, m));
            cap = m;
        }
        n = m;
    }
    uint8_t* data() { return p; }
    size_t size() const { return n; }
    const uint8_t* begin() const { return p; }
    const uint8_t* end() const { return p + n; }
};

template <class T>
void upload(DBuf& b, const std::vector<T>& v, cudaStream_t st) {
    b.ensure(std::max<size_t>(v.size() * sizeof(T), 16));
    if (!v.empty()) CK(cudaMemcpyAsync(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st));
}

const uint8_t COMPL[16] = {3, 2, 1, 0, 5, 4, 7, 6, 8, 9, 13, 12, 11, 10, 14, 15};

void parallel_for(size_t n, const std::function<void(size_t)>& fn) {
    const size_t nt = std::max<size_t>(1, std::min<size_t>(std::thread::hardware_concurrency(), n));
    if (nt <= 1) {
        for (size_t i = 0; i < n; ++i) fn(i);
        return;
    }
    std::atomic<size_t> next{0};
    std::vector<std::thread> th;
    std::exception_ptr err;
    std::mutex mu;
    for (size_t t = 0; t < nt; ++t)
        th.emplace_back([&]() {
            for (;;) {
                size_t i = next.fetch_add(1);
                if (i >= n) break;
                try {
                    fn(i);
                } catch (...) {
                    std::lock_guard<std::mutex> g(mu);
                    if (!err) err = std::current_exception();
                }
            }
        });
    for (auto& x : th) x.join();
    if (err) std::rethrow_exception(err);
}

struct EvTimer {  // device time between two events on one stream
    cudaEvent_t a = nullptr, b = nullptr;
    EvTimer() {
        cudaEventCreate(&a);
        cudaEventCreate(&b);
    }
    ~EvTimer() {
        cudaEventDestroy(a);
        cudaEventDestroy(b);
    }
    void start(cudaStream_t st) { cudaEventRecord(a, st); }
    void stop(cudaStream_t st) { cudaEventRecord(b, st); }
    double ms() {
        float m = 0;
        cudaEventSynchronize(b);
        cudaEventElapsedTime(&m, a, b);
        return m;
    }
};

double ms_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace

// One pipeline lane: a stream and the device buffers of the sub-batch it is working on.  Two
// lanes take alternate sub-batches, so one lane's host steps (Phase 2a/2b, the per-query end) run
// while the other's kernels do, and the kernels of both fill each other's launch tails.
struct Work {
    cudaStream_t st = nullptr;
    // the batched pipeline's traceback of a range, beside the lane's next kernels; tb_mu keeps
    // one traceback at a time on the lane's traceback buffers (a sub-batch's last one can still
    // run when the next sub-batch's first starts)
    cudaStream_t st2 = nullptr;
    std::mutex tb_mu;
    DBuf pv, pv_off, cs, cs_off, cq, cq_off, pos_off, lut_keys, lut_vals, lut_keys2, lut_vals2, lut_counts;
    DBuf counts, offs, hits, hit_pair, ub, flags, dd_scratch, dd_cells, ung_idx, n_sel, po, wide, wide2, dres, geo,
        n_wide, band, sel, surv, cells, fails, temp, tb_in, tb_out, tb_ops, tb_scratch, stage, stage_start, stage_over,
        tb_ooff, tb_ops2, ung_queue, dd_units, tb_half, tb_cells;
    DBuf sched_pred, sched_order, sched_scratch, sched_feat, sched_cells;
    // the device chain as a CUDA graph (chain_graph): its executable, its timing events and the
    // pinned block its counts come back in
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t ev[7] = {};
    HostBuf hcount;
    void release() {
        if (exec) cudaGraphExecDestroy(exec);
        exec = nullptr;
        for (cudaEvent_t& e : ev)
            if (e) {
                cudaEventDestroy(e);
                e = nullptr;
            }
        DBuf* all[] = {&pv, &pv_off, &cs, &cs_off, &cq, &cq_off, &pos_off, &lut_keys, &lut_vals, &lut_keys2,
                       &lut_vals2, &lut_counts, &counts, &offs, &hits, &hit_pair, &ub, &flags, &dd_scratch, &dd_cells,
                       &ung_idx, &n_sel, &po, &wide, &wide2, &dres, &geo, &n_wide, &band, &sel, &surv, &cells, &fails,
                       &temp, &tb_in, &tb_out, &tb_ops, &tb_scratch, &stage, &stage_start, &stage_over, &tb_ooff,
                       &tb_ops2, &ung_queue, &dd_units, &tb_half, &tb_cells, &sched_pred, &sched_order, &sched_scratch, &sched_feat, &sched_cells};
        for (DBuf* b : all) b->release();
        if (st) cudaStreamDestroy(st);
        if (st2) cudaStreamDestroy(st2);
        st2 = nullptr;
        st = nullptr;
    }
};

// The hand-swept launch shape (B200, genome-vs-library workloads): the starting point of
// rmb_autotune and the plain pipeline's fixed shape.
static rmb_tune default_tune() {
    rmb_tune t;
    t.prelim_group = 8;
    t.prelim_blocks_per_sm = 6;
    t.prelim_window = 60;
    t.prelim_budget_div = 128;
    t.ungapped_blocks_per_sm = 8;
    t.dedup_extend_hits_per_pair = 256;
    t.lanes = 1;
    t.graph = 1;
    return t;
}

struct rmb_ctx {
    rmb_params p{};
    GlueParams gp{};
    std::string matrix_name;
    int sms = 148;
    cudaStream_t st = nullptr;
    // library, host
    std::vector<std::string> ids;
    std::vector<uint32_t> slen;
    std::vector<uint64_t> plus_off, packed_off;
    std::vector<uint8_t> h_align, h_align_rc;
    std::vector<uint8_t> h_mask, h_mask_rc;  // len bytes per subject that has a mask
    std::vector<int64_t> mask_off;            // -1 = no mask
    uint64_t total_letters = 0;
    uint32_t max_slen = 0;
    bool loaded = false;
    // library, device
    DBuf d_plus, d_rc, d_align, d_align_rc, d_packed, d_plus_off, d_packed_off, d_len, d_params;
    // the query set's lookup widths (read by every lane)
    DBuf lw;
    bool prelim_stream = false;  // thread-per-extension prelim kernel (else the warp kernel)
    rmb_tune tune = default_tune();  // launch knobs of the batched pipeline (rmb_tune_set / rmb_autotune)
    KaBlock ka;                  // E-value statistics (lambda <= 0: none)
    DBuf dust_scratch, fails;    // per-thread DUST interval lists, their overflow flag
    // the pipeline lanes: each a stream and the device buffers of one sub-batch at a time
    Work work[2];
    DevLib L{};
    rmb_queries* batch = nullptr;  // the query set of rmb_search_batch, reused from call to call
    // learned schedule: the network's parameters (rmb_sched_set_model) and its per-batch buffers;
    // sched_log, while rmb_sched_log runs, collects (features, cells) of the FIFO run
    DBuf sched_params;
    bool sched_ready = false;
    struct SchedLog {
        std::vector<float> feats;
        std::vector<uint32_t> cells;
    }* sched_log = nullptr;
};

// Queries resident on the device (rmb_queries_upload); the host copy feeds the host steps.
struct rmb_queries {
    uint32_t n = 0;
    int device = 0;
    HostBuf host;                  // concatenated sentinel-wrapped queries (pinned)
    std::vector<uint64_t> off;     // offset of query i in host / d_q / d_qrc
    std::vector<uint32_t> len;
    DBuf d_q, d_qrc, d_off, d_len;
    DBuf d_qm, d_qmrc;   // DUST-masked queries and their reverse complements (made on first use)
    bool dusted = false;
    void release() {
        d_q.release();
        d_qrc.release();
        d_off.release();
        d_len.release();
        d_qm.release();
        d_qmrc.release();
    }
};

namespace {

std::vector<uint8_t> revcomp_full(const uint8_t* s, size_t n) {
    std::vector<uint8_t> o(n);
    for (size_t i = 0; i < n; ++i) o[i] = COMPL[s[n - 1 - i] & 15];
    return o;
}

struct Taps {
    std::vector<uint32_t>* seeds = nullptr;     // strand, q, s
    std::vector<uint32_t>* ungapped = nullptr;  // strand, qs, qe, ss, se, score
    std::vector<uint32_t>* prelims = nullptr;   // strand, qs, qe, ss, se, score, q_seed, s_seed
    std::vector<uint32_t>* lookup = nullptr;    // query, cell, position (retrieval order)
    std::vector<uint32_t>* tracebacks = nullptr;  // strand, status, score, q0, q1, s0, s1, n_ops, ops hash
};

// DUST masking of a query set (engine.rs:606-616 -> filter/dust.rs:462), on the device: the
// masked copy and its reverse complement feed the lookup tables and the exact word extension
// only.  `compat` is the multi-chunk path's variant (engine.rs:697-707).
void mask_queries(rmb_ctx& C, rmb_queries& QH, bool compat, rmb_counters& ctr) {
    cudaStream_t st = C.st;
    const uint32_t nq = QH.n;
    auto t0 = std::chrono::steady_clock::now();
    const size_t bytes = QH.host.size();
    QH.d_qm.ensure(bytes);
    QH.d_qmrc.ensure(bytes);
    CK(cudaMemcpyAsync(QH.d_qm.p, QH.d_q.p, bytes, cudaMemcpyDeviceToDevice, st));
    const uint32_t nt = dust_threads(nq, C.sms);
    C.dust_scratch.ensure(dust_scratch_bytes(nt));
    C.fails.ensure(16);
    CK(cudaMemsetAsync(C.fails.p, 0, 4, st));
    EvTimer ev;
    ev.start(st);
    CK(launch_dust(QH.d_q.as<uint8_t>(), QH.d_off.as<uint64_t>(), QH.d_len.as<uint32_t>(), nq, QH.d_qm.as<uint8_t>(),
                   C.dust_scratch.p, nt, C.fails.as<unsigned int>(), compat, st));
    CK(launch_revcomp(QH.d_qm.as<uint8_t>(), QH.d_off.as<uint64_t>(), QH.d_len.as<uint32_t>(), nq,
                      QH.d_qmrc.as<uint8_t>(), st));
    ev.stop(st);
    ctr.launches += 2;
    unsigned int over = 0;
    CK(cudaMemcpyAsync(&over, C.fails.p, 4, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    if (over) throw Fail(RMB_ELIMIT, "DUST interval list outgrew its fixed capacity");
    ctr.gpu_ms_dust += ev.ms();
    ctr.ms_lookup += ms_since(t0);
    QH.dusted = true;
}

// One (query, subject) pair's Phase 2a output, in the reference's order (purge order).
constexpr uint64_t MAX_RANGE_HITS = 1ull << 29;
constexpr uint64_t SCHED_NF_HOST = 12;  // features per record of the learned schedule (rmb_sched.cuh)

struct PairPrelims {
    uint32_t q, s;
    std::vector<Prelim> p;
};

bool traceback_2b(rmb_ctx& C, Work& W, const DevQueries& Q, const uint32_t* hqlen, uint32_t nb,
                  const std::function<const uint8_t*(uint32_t)>& qhost, const std::vector<uint32_t>& pair_ids,
                  std::vector<std::vector<Prelim>>& prelims, std::vector<Hit>* out, rmb_counters& ctr, Taps* taps,
                  std::future<rmb_counters>* defer = nullptr);

// The per-query end of a search: E-values and bit scores (rmstats RmStats for the query's length
// against the whole database), the --evalue reap (main.rs:1224-1226, before masklevel), then
// masklevel (engine.rs:863) and the hit order (main.rs:1230-1234, engine.rs:998).
void finish_query(const rmb_ctx& C, std::vector<Hit>& v, uint32_t qlen) {
    const rmb_params& P = C.p;
    const int64_t sp = eff_searchsp(C.ka, (int32_t)qlen, (int64_t)C.total_letters, (int32_t)C.ids.size());
    for (Hit& h : v) {
        h.evalue = hsp_evalue(h.score, C.ka, sp);
        h.bitscore = hsp_bitscore(h.score, C.ka);
    }
    if (P.evalue > 0.0 && C.ka.lambda > 0.0)
        v.erase(std::remove_if(v.begin(), v.end(), [&](const Hit& h) { return h.evalue > P.evalue; }), v.end());
    apply_mask_level(v, P.mask_level < 0 ? 101u : (uint32_t)P.mask_level);
    sort_hit_list_order(v, C.ids);
}

// The batched pipeline's device chain of one pair range as one CUDA graph: the dedup with the
// ungapped extension, the ungapped records' selection, the prelim DP geometry, the learned order,
// the prelim DP with its warp fallback for the records it passes on, and the survivors' selection
// and gather.  Every count after the word hits is read by the kernels from device memory, so the
// chain runs with no host round trip; buffers are sized for the range's word hits, an upper bound
// on every later count.  The graph is captured per pair range and updated in place
// (cudaGraphExecUpdate) while its shape repeats.  The rare cases past the graph's capacities (a
// fallback list longer than it holds, records wider than the warp ring, more survivors than it
// gathers) finish stage by stage after it.  Sets the survivors and the counters the
// stage-by-stage path sets.
void chain_graph(rmb_ctx& C, Work& W, const DevQueries& Q, int32_t ucut, uint64_t pair0, uint64_t npairs,
                 uint64_t nh, uint32_t qmax, std::vector<SurvivorRec>& sv, rmb_counters& ctr) {
    const rmb_params& P = C.p;
    cudaStream_t st = W.st;
    const int32_t dx = C.tune.dedup_extend_hits_per_pair;
    const bool fused = dx >= 0 && nh >= (uint64_t)dx * npairs;
    const bool learned = P.schedule == 1;
    const uint64_t n1 = std::max<uint64_t>(nh, 1);
    // the warp kernel's list and the survivors gathered in the graph (graph knob 2: one of each,
    // so that every range also takes the finish past them)
    const uint64_t cap_min = C.tune.graph == 2 ? 1 : 1u << 16;
    const uint64_t wcap = std::min<uint64_t>(n1, std::max<uint64_t>(cap_min, C.tune.graph == 2 ? 1 : n1 / 64));
    const uint64_t scap = std::min<uint64_t>(n1, std::max<uint64_t>(cap_min, C.tune.graph == 2 ? 1 : n1 / 256));
    W.flags.ensure(nh + 1);
    W.dd_cells.ensure(n1 * diag_cell_bytes());
    W.ung_queue.ensure(16);
    if (!fused) W.dd_scratch.ensure(dedup_threads(C.sms) * 1024 * 4);
    else W.dd_units.ensure(dedup_units_bytes(npairs, nh, C.sms));
    W.ung_idx.ensure(n1 * 4);
    W.n_sel.ensure(16);   // [0] ungapped records, [1] survivors
    W.n_wide.ensure(16);  // [0] records the thread kernel passed on, [1] its queue, [2] those the warp kernel did
    W.cells.ensure(16);   // [0] DP cells, [1] the thread kernel's alone
    W.fails.ensure(16);
    W.po.ensure(n1 * sizeof(PrelimOut));
    W.geo.ensure(n1 * prelim_geo_bytes());
    W.wide.ensure(n1 * 4);
    W.wide2.ensure(wcap * 4);
    W.dres.ensure(wcap * 2 * sizeof(int4));
    W.sel.ensure(n1 * 4);
    W.surv.ensure(scap * sizeof(SurvivorRec));
    if (learned) {
        W.sched_pred.ensure(n1 * 4);
        W.sched_order.ensure(n1 * 4);
        W.sched_scratch.ensure(sched_order_scratch_bytes());
    }
    size_t t_eq = 0, t_pre = 0, t_front = learned ? sched_front_temp_bytes(n1) : 0;
    CK(launch_select_eq(W.flags.as<uint8_t>(), nh, 3, W.ung_idx.as<uint32_t>(), W.n_sel.as<uint32_t>(), nullptr, t_eq,
                        st));
    CK(launch_select_prelim(W.po.as<PrelimOut>(), n1, W.sel.as<uint32_t>(), W.n_sel.as<uint32_t>() + 1, nullptr, t_pre,
                            st, W.n_sel.as<unsigned int>()));
    W.temp.ensure(std::max(t_eq, std::max(t_pre, t_front)));
    W.hcount.resize(64);
    for (cudaEvent_t& e : W.ev)
        if (!e) CK(cudaEventCreate(&e));
    const rmb_tune& tn = C.tune;
    StreamLaunch cfg;
    cfg.group = tn.prelim_group;
    cfg.blocks_per_sm = tn.prelim_blocks_per_sm;
    cfg.window = tn.prelim_window;
    cfg.budget_div = tn.prelim_budget_div;
    auto rec = [&](int k) { CK(cudaEventRecordWithFlags(W.ev[k], st, cudaEventRecordExternal)); };

    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    try {
        CK(cudaMemsetAsync(W.n_wide.p, 0, 16, st));
        CK(cudaMemsetAsync(W.cells.p, 0, 16, st));
        CK(cudaMemsetAsync(W.fails.p, 0, 16, st));
        rec(0);
        if (fused) {
            CK(launch_dedup_extend(C.L, Q, C.d_params.as<DevParams>(), ucut, pair0, npairs, nh, W.offs.as<uint64_t>(),
                                   W.hits.as<SeedHit>(), W.ub.as<UngBox>(), W.flags.as<uint8_t>(), W.dd_cells.p,
                                   W.ung_queue.as<unsigned long long>(), W.dd_units.p, C.sms, st));
        } else {
            CK(launch_ungapped(C.L, Q, C.d_params.as<DevParams>(), ucut, nh, W.hits.as<SeedHit>(),
                               W.hit_pair.as<uint32_t>(), W.ub.as<UngBox>(), C.sms, st,
                               W.ung_queue.as<unsigned long long>(), tn.ungapped_blocks_per_sm));
            CK(launch_dedup(C.L, Q, P.word_size, ucut, pair0, npairs, W.offs.as<uint64_t>(), W.hits.as<SeedHit>(),
                            W.ub.as<UngBox>(), W.flags.as<uint8_t>(), W.dd_scratch.as<uint32_t>(), W.dd_cells.p,
                            C.sms, st));
        }
        CK(launch_select_eq(W.flags.as<uint8_t>(), nh, 3, W.ung_idx.as<uint32_t>(), W.n_sel.as<uint32_t>(), W.temp.p,
                            t_eq, st));
        rec(1);
        const unsigned int* nu_dev = W.n_sel.as<unsigned int>();
        CK(launch_prelim_prep(C.L, Q, C.d_params.as<DevParams>(), n1, W.ung_idx.as<uint32_t>(), W.hits.as<SeedHit>(),
                              W.hit_pair.as<uint32_t>(), W.ub.as<UngBox>(), W.geo.p, C.sms, st, nu_dev));
        const uint32_t* order = nullptr;
        rec(6);
        if (learned) {
            CK(launch_sched_order(C.L, Q, C.d_params.as<DevParams>(), n1, W.ung_idx.as<uint32_t>(),
                                  W.hits.as<SeedHit>(), W.hit_pair.as<uint32_t>(), W.ub.as<UngBox>(),
                                  W.counts.as<uint32_t>(), C.sched_params.as<float>(), W.sched_pred.as<float>(),
                                  W.sched_scratch.p, W.sched_order.as<uint32_t>(), C.sms, st, 1, W.temp.p, t_front,
                                  nu_dev));
            order = W.sched_order.as<uint32_t>();
        }
        rec(2);
        CK(launch_prelim_stream(C.d_params.as<DevParams>(), n1, W.geo.p, W.po.as<PrelimOut>(), W.wide.as<uint32_t>(),
                                W.n_wide.as<unsigned int>(), W.cells.as<unsigned long long>(), C.sms, st, order,
                                nullptr, false, cfg,
                                StreamDevCounts{nu_dev, learned ? sched_front_count(W.sched_scratch.p) : nullptr, n1}));
        rec(3);
        CK(cudaMemcpyAsync(W.cells.as<unsigned long long>() + 1, W.cells.p, 8, cudaMemcpyDeviceToDevice, st));
        CK(launch_prelim_split(C.L, Q, C.d_params.as<DevParams>(), (uint32_t)wcap, W.wide.as<uint32_t>(),
                               W.ung_idx.as<uint32_t>(), W.hits.as<SeedHit>(), W.hit_pair.as<uint32_t>(),
                               W.ub.as<UngBox>(), W.dres.as<int4>(), W.po.as<PrelimOut>(), W.wide2.as<uint32_t>(),
                               W.n_wide.as<unsigned int>() + 2, W.cells.as<unsigned long long>(), C.sms, st,
                               W.n_wide.as<unsigned int>()));
        rec(4);
        CK(launch_select_prelim(W.po.as<PrelimOut>(), n1, W.sel.as<uint32_t>(), W.n_sel.as<uint32_t>() + 1, W.temp.p,
                                t_pre, st, nu_dev));
        CK(launch_gather_survivors((uint32_t)scap, W.sel.as<uint32_t>(), W.ung_idx.as<uint32_t>(), W.hits.as<SeedHit>(),
                                   W.hit_pair.as<uint32_t>(), W.ub.as<UngBox>(), W.po.as<PrelimOut>(),
                                   W.surv.as<SurvivorRec>(), st, W.n_sel.as<unsigned int>() + 1));
        rec(5);
        uint8_t* hc = W.hcount.data();
        CK(cudaMemcpyAsync(hc, W.n_sel.p, 8, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(hc + 8, W.n_wide.p, 12, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(hc + 24, W.cells.p, 16, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(hc + 40, W.fails.p, 4, cudaMemcpyDeviceToHost, st));
    } catch (...) {
        cudaStreamEndCapture(st, &g);
        if (g) cudaGraphDestroy(g);
        throw;
    }
    CK(cudaStreamEndCapture(st, &g));
    if (W.exec) {
        cudaGraphExecUpdateResultInfo info;
        if (cudaGraphExecUpdate(W.exec, g, &info) != cudaSuccess) {
            cudaGetLastError();
            cudaGraphExecDestroy(W.exec);
            W.exec = nullptr;
        }
    }
    if (!W.exec) {
        const cudaError_t e = cudaGraphInstantiate(&W.exec, g, 0);
        if (e != cudaSuccess) {
            cudaGraphDestroy(g);
            CK(e);
        }
    }
    cudaGraphDestroy(g);
    CK(cudaGraphLaunch(W.exec, st));
    CK(cudaStreamSynchronize(st));
    const uint8_t* hc = W.hcount.data();
    uint32_t nu, nsv, nw, nw2;
    unsigned long long cells, main_cells;
    unsigned int fails;
    memcpy(&nu, hc, 4);
    memcpy(&nsv, hc + 4, 4);
    memcpy(&nw, hc + 8, 4);
    memcpy(&nw2, hc + 16, 4);
    memcpy(&cells, hc + 24, 8);
    memcpy(&main_cells, hc + 32, 8);
    memcpy(&fails, hc + 40, 4);
    auto ms = [&](int a, int b) {
        float m = 0;
        if (cudaEventElapsedTime(&m, W.ev[a], W.ev[b]) != cudaSuccess) {
            cudaGetLastError();  // a timing gap is not a search failure
            m = 0;
        }
        return (double)m;
    };
    ctr.gpu_ms_dedup += ms(0, 1);
    ctr.gpu_ms_prelim += ms(1, 5);
    ctr.gpu_ms_prelim_main += ms(2, 3);
    if (learned) ctr.gpu_ms_sched += ms(6, 2);
    ctr.so_cells_main += main_cells;
    ctr.launches += 2 + 1 + 1 + (learned ? 3 : 0) + 1 + 2 + 1 + 1;
    ctr.ungapped += nu;
    ctr.prelim_dp += nu;
    if (nw > wcap || nw2 || nsv > scap) {
        // past the graph's capacities: the fallbacks, the selection and the gather stage by stage
        EvTimer ex;
        ex.start(st);
        if (nw > wcap) {
            W.wide2.ensure((uint64_t)nw * 4);
            W.dres.ensure((uint64_t)nw * 2 * sizeof(int4));
            CK(cudaMemsetAsync(W.n_wide.as<unsigned int>() + 2, 0, 4, st));
            // the listed records again, all of them (the same results for the first wcap)
            CK(cudaMemsetAsync(W.cells.p, 0, 8, st));
            CK(launch_prelim_split(C.L, Q, C.d_params.as<DevParams>(), nw, W.wide.as<uint32_t>(),
                                   W.ung_idx.as<uint32_t>(), W.hits.as<SeedHit>(), W.hit_pair.as<uint32_t>(),
                                   W.ub.as<UngBox>(), W.dres.as<int4>(), W.po.as<PrelimOut>(), W.wide2.as<uint32_t>(),
                                   W.n_wide.as<unsigned int>() + 2, W.cells.as<unsigned long long>(), C.sms, st));
            unsigned long long warp_cells = 0;
            CK(cudaMemcpyAsync(&nw2, W.n_wide.as<unsigned int>() + 2, 4, cudaMemcpyDeviceToHost, st));
            CK(cudaMemcpyAsync(&warp_cells, W.cells.p, 8, cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            cells = main_cells + warp_cells;
            ctr.launches += 2;
        }
        if (nw2) {
            const uint64_t cap = (uint64_t)std::max(qmax, C.max_slen) + 2;
            const uint32_t threads = std::min<uint32_t>(nw2, (uint32_t)std::max<uint64_t>(128, (1ull << 31) / (cap * 8)));
            W.band.ensure((uint64_t)((threads + 127) / 128 * 128) * cap * 8);
            CK(cudaMemsetAsync(W.cells.p, 0, 8, st));
            CK(launch_prelim_wide(C.L, Q, C.d_params.as<DevParams>(), nw2, W.wide2.as<uint32_t>(),
                                  W.ung_idx.as<uint32_t>(), W.hits.as<SeedHit>(), W.hit_pair.as<uint32_t>(),
                                  W.ub.as<UngBox>(), W.po.as<PrelimOut>(), W.band.as<int2>(), cap, threads,
                                  W.cells.as<unsigned long long>(), W.fails.as<unsigned int>(), st));
            unsigned long long wide_cells = 0;
            CK(cudaMemcpyAsync(&wide_cells, W.cells.p, 8, cudaMemcpyDeviceToHost, st));
            CK(cudaMemcpyAsync(&fails, W.fails.p, 4, cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            cells += wide_cells;
            ctr.launches += 1;
        }
        size_t tb = 0;
        CK(launch_select_prelim(W.po.as<PrelimOut>(), nu, W.sel.as<uint32_t>(), W.n_sel.as<uint32_t>() + 1, nullptr, tb,
                                st));
        W.temp.ensure(tb);
        CK(launch_select_prelim(W.po.as<PrelimOut>(), nu, W.sel.as<uint32_t>(), W.n_sel.as<uint32_t>() + 1, W.temp.p,
                                tb, st));
        CK(cudaMemcpyAsync(&nsv, W.n_sel.as<uint32_t>() + 1, 4, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        W.surv.ensure(std::max<uint64_t>(nsv, 1) * sizeof(SurvivorRec));
        CK(launch_gather_survivors(nsv, W.sel.as<uint32_t>(), W.ung_idx.as<uint32_t>(), W.hits.as<SeedHit>(),
                                   W.hit_pair.as<uint32_t>(), W.ub.as<UngBox>(), W.po.as<PrelimOut>(),
                                   W.surv.as<SurvivorRec>(), st));
        ex.stop(st);
        ctr.gpu_ms_prelim += ex.ms();
        ctr.launches += 2;
    }
    if (fails) throw Fail(RMB_ECUDA, "prelim DP band exceeded its storage");
    ctr.so_cells += cells;
    sv.resize(nsv);
    if (nsv) CK(cudaMemcpyAsync(sv.data(), W.surv.p, nsv * sizeof(SurvivorRec), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
}

// Counters of one lane added into another's (the device times of the two lanes add up: they
// overlap in wall time).
void add_counters(rmb_counters& a, const rmb_counters& b) {
    a.word_hits += b.word_hits; a.seeds += b.seeds; a.ungapped += b.ungapped; a.prelim_dp += b.prelim_dp;
    a.prelims += b.prelims; a.tb_dp += b.tb_dp; a.finals += b.finals; a.so_cells += b.so_cells;
    a.tb_cells += b.tb_cells;
    a.ms_lookup += b.ms_lookup; a.ms_scan += b.ms_scan; a.ms_ungapped += b.ms_ungapped; a.ms_dedup += b.ms_dedup;
    a.ms_prelim_dp += b.ms_prelim_dp; a.ms_host_2a += b.ms_host_2a; a.ms_traceback += b.ms_traceback;
    a.ms_host_2b += b.ms_host_2b;
    a.gpu_ms_scan += b.gpu_ms_scan; a.gpu_ms_ungapped += b.gpu_ms_ungapped; a.gpu_ms_dedup += b.gpu_ms_dedup;
    a.gpu_ms_prelim += b.gpu_ms_prelim; a.gpu_ms_traceback += b.gpu_ms_traceback; a.gpu_ms_lookup += b.gpu_ms_lookup;
    a.launches += b.launches;
    a.gpu_ms_prelim_main += b.gpu_ms_prelim_main; a.so_cells_main += b.so_cells_main;
    a.gpu_ms_dust += b.gpu_ms_dust;
    a.gpu_ms_sched += b.gpu_ms_sched;
}

// The search of a set of single-chunk queries.  ucut_override: per-query ungapped cutoffs (the
// chunks of a long query take their parent's).  collect: stop after Phase 2a and hand over the
// prelims of every pair instead of aligning them.
void run_core(rmb_ctx& C, rmb_queries& QH, std::vector<std::vector<Hit>>& out_hits, rmb_counters& ctr, Taps* taps,
              const std::vector<int32_t>* ucut_override, std::vector<PairPrelims>* collect) {
    const rmb_params& P = C.p;
    const uint32_t ns = (uint32_t)C.ids.size();
    const uint32_t nq = QH.n;
    const uint32_t* qlen = QH.len.data();
    out_hits.assign(nq, {});
    std::vector<int32_t> ucut(nq), lw_all(nq);
    for (uint32_t i = 0; i < nq; ++i) {
        if (qlen[i] >= 1999800u) throw Fail(RMB_ELIMIT, "queries of 1,999,800 bp or more take the chunked path");
        const uint64_t avg = ns ? C.total_letters / ns : 0;
        ucut[i] = ucut_override ? (*ucut_override)[i]
                  : P.ungapped_cutoff >= 0 ? P.ungapped_cutoff
                                          : ungapped_cutoff_for(C.matrix_name, P.gap_open, P.gap_extend,
                                                                P.min_raw_gapped_score, qlen[i], avg);
        lw_all[i] = choose_lut_width(P.word_size, 2ull * qlen[i]);
    }
    cudaStream_t st = C.st;
    upload(C.lw, lw_all, st);
    if (P.dust && !QH.dusted && nq) mask_queries(C, QH, false, ctr);
    const uint8_t* qmask = P.dust ? QH.d_qm.as<uint8_t>() : QH.d_q.as<uint8_t>();
    const uint8_t* qmask_rc = P.dust ? QH.d_qmrc.as<uint8_t>() : QH.d_qrc.as<uint8_t>();
    // Sub-batches of queries sharing one ungapped cutoff, bounded by lookup-table size; with two
    // lanes, cut further so each lane gets about two.
    const int lanes = (P.pipeline == 0 && !taps && !collect && !C.sched_log && C.tune.lanes > 1 && nq > 1) ? 2 : 1;
    const uint32_t piece = lanes > 1 ? std::max<uint32_t>(1, (nq + 2 * lanes - 1) / (2 * lanes)) : nq;
    std::vector<std::pair<uint32_t, uint32_t>> subs;
    for (uint32_t qb = 0; qb < nq;) {
        uint64_t cells_b = 0, pos_b = 0;
        uint32_t qe = qb;
        while (qe < nq) {
            const uint64_t c = (1ull << (2 * lw_all[qe])) + 1, p2 = 2ull * qlen[qe] + 1;
            if (qe > qb && (ucut[qe] != ucut[qb] || cells_b + c > (1ull << 30) || pos_b + p2 > (1ull << 30) ||
                            qe - qb >= piece))
                break;
            cells_b += c;
            pos_b += p2;
            ++qe;
        }
        subs.emplace_back(qb, qe);
        qb = qe;
    }
    CK(cudaStreamSynchronize(st));  // the lanes start after the query set's own work (upload, DUST)
    // With `tail`, the sub-batch's last host steps (the pending Phase 2b, masklevel and the hit
    // order) run on a thread of their own, *tail holding them (their host ms and hits), so the
    // next sub-batch's kernels start at once.
    using Tail = std::future<rmb_counters>;
    auto sub_batch = [&](Work& W, uint32_t qb, uint32_t qe, rmb_counters& ctr, Tail* tail) {
        cudaStream_t st = W.st;
        const uint32_t nb = qe - qb;
        auto t0 = std::chrono::steady_clock::now();
        // ---- lookup tables of the sub-batch, built on the device
        std::vector<uint64_t> hpvoff(nb), hcsoff(nb), hposoff(nb), hzero(nb, 0);
        std::vector<uint32_t> hqlen(qlen + qb, qlen + qe);
        std::vector<int32_t> hlw(lw_all.begin() + qb, lw_all.begin() + qe);
        // the batched pipeline's traceback and host Phase 2b of the last range, running while the
        // next one's kernels do (it writes out_hits; its counters come back with it)
        std::future<rmb_counters> pending;
        uint64_t npv = 0, ncs = 0, npos = 0;
        for (uint32_t i = 0; i < nb; ++i) {
            hpvoff[i] = npv;
            hcsoff[i] = ncs;
            hposoff[i] = npos;
            npv += std::max<uint64_t>((1ull << (2 * hlw[i])) / 32, 1);
            ncs += (1ull << (2 * hlw[i])) + 1;
            npos += 2ull * hqlen[i] + 1;
        }
        upload(W.pv_off, hpvoff, st);
        upload(W.cs_off, hcsoff, st);
        upload(W.cq_off, hzero, st);
        upload(W.pos_off, hposoff, st);
        W.pv.ensure(npv * 4);
        W.cs.ensure((ncs + 1) * 4);
        W.lut_counts.ensure((ncs + 1) * 4);
        W.cq.ensure(npos * 4);
        W.lut_keys.ensure(npos * 4);
        W.lut_vals.ensure(npos * 4);
        W.lut_keys2.ensure(npos * 4);
        W.lut_vals2.ensure(npos * 4);
        DevQueries Q{QH.d_q.as<uint8_t>(),       QH.d_qrc.as<uint8_t>(),  qmask, qmask_rc,
                     QH.d_off.as<uint64_t>() + qb, QH.d_len.as<uint32_t>() + qb, W.pv.as<uint32_t>(),
                     W.pv_off.as<uint64_t>(),    W.cs.as<uint32_t>(),     W.cs_off.as<uint64_t>(),
                     W.cq.as<uint32_t>(),        W.cq_off.as<uint64_t>(), C.lw.as<int32_t>() + qb, nb};
        EvTimer ev;
        ev.start(st);
        {
            size_t tb = W.temp.cap;
            uint64_t nvalid = 0;
            cudaError_t e = launch_lut_build(Q, P.word_size, nb, W.pos_off.as<uint64_t>(), npos, ncs, npv,
                                             W.lut_keys.as<uint32_t>(), W.lut_vals.as<uint32_t>(),
                                             W.lut_keys2.as<uint32_t>(), W.lut_vals2.as<uint32_t>(),
                                             W.lut_counts.as<uint32_t>(), W.cs.as<uint32_t>(), W.cq.as<uint32_t>(),
                                             W.pv.as<uint32_t>(), W.temp.p, tb, nvalid, st);
            if (e == cudaErrorNotReady) {
                W.temp.ensure(tb);
                tb = W.temp.cap;
                e = launch_lut_build(Q, P.word_size, nb, W.pos_off.as<uint64_t>(), npos, ncs, npv,
                                     W.lut_keys.as<uint32_t>(), W.lut_vals.as<uint32_t>(), W.lut_keys2.as<uint32_t>(),
                                     W.lut_vals2.as<uint32_t>(), W.lut_counts.as<uint32_t>(), W.cs.as<uint32_t>(),
                                     W.cq.as<uint32_t>(), W.pv.as<uint32_t>(), W.temp.p, tb, nvalid, st);
            }
            CK(e);
        }
        ev.stop(st);
        CK(cudaStreamSynchronize(st));
        ctr.gpu_ms_lookup += ev.ms();
        ctr.launches += 3;  // codes, place, pv
        if (taps && taps->lookup) {
            std::vector<uint32_t> hcs(ncs + 1), hcq(npos), hpv(npv);
            CK(cudaMemcpy(hcs.data(), W.cs.p, (ncs + 1) * 4, cudaMemcpyDeviceToHost));
            CK(cudaMemcpy(hcq.data(), W.cq.p, npos * 4, cudaMemcpyDeviceToHost));
            CK(cudaMemcpy(hpv.data(), W.pv.p, npv * 4, cudaMemcpyDeviceToHost));
            for (uint32_t i = 0; i < nb; ++i) {
                const uint64_t cells = 1ull << (2 * hlw[i]);
                for (uint64_t c = 0; c < cells; ++c) {
                    const uint32_t b = hcs[hcsoff[i] + c], e = hcs[hcsoff[i] + c + 1];
                    const bool present = (hpv[hpvoff[i] + (c >> 5)] >> (c & 31)) & 1u;
                    if (present != (e > b)) taps->lookup->insert(taps->lookup->end(), {qb + i, (uint32_t)c, 0xffffffffu});
                    for (uint32_t j = b; j < e; ++j) taps->lookup->insert(taps->lookup->end(), {qb + i, (uint32_t)c, hcq[j]});
                }
            }
            return;
        }
        ctr.ms_lookup += ms_since(t0);
        // by value: a deferred Phase 2b may call it after this sub-batch's body has returned
        auto qhost = [&QH, qb](uint32_t local) { return QH.host.data() + QH.off[qb + local]; };

        // ---- scan: one pass that counts and stages the hits per warp, offsets, then the hits in
        // pair order (pair ids are local to the sub-batch)
        t0 = std::chrono::steady_clock::now();
        const uint64_t npairs = (uint64_t)nb * ns;
        W.counts.ensure((npairs + 1) * 4);
        W.offs.ensure((npairs + 1) * 8);
        W.stage_start.ensure(npairs * 4);
        W.stage.ensure(scan_stage_entries(npairs, C.sms) * sizeof(SeedHit));
        W.stage_over.ensure(16);  // the overflow flag and the scan's pair queue
        // The batched pipeline feeds the scan's warps pairs from a queue where the sub-batch's
        // query lengths vary (over 2x): a pair's cost then follows its query too, and fixed
        // strides left warps idle (1,000 chunks of 1-200 kb: 54 -> 38 ms a step).  Over queries
        // of one length the strides balance and keep a block's warps on one query's tables in L1
        // (1,000 queries of 60 kb: 75 ms with strides, 109 with the queue).
        const uint32_t qlo = *std::min_element(hqlen.begin(), hqlen.end());
        const uint32_t qhi = *std::max_element(hqlen.begin(), hqlen.end());
        const bool scan_queue = P.pipeline != 1 && (uint64_t)qhi > 2ull * qlo;
        CK(cudaMemsetAsync(W.counts.p, 0, (npairs + 1) * 4, st));
        CK(cudaMemsetAsync(W.stage_over.p, 0, 16, st));
        ev.start(st);
        CK(launch_scan_stage(C.L, Q, P.word_size, npairs, W.counts.as<uint32_t>(), W.stage_start.as<uint32_t>(),
                             W.stage.as<SeedHit>(), W.stage_over.as<unsigned int>(), C.sms, st, scan_queue));
        size_t tb = 0;
        CK(launch_offsets(W.counts.as<uint32_t>(), npairs + 1, W.offs.as<uint64_t>(), nullptr, tb, st));
        W.temp.ensure(tb);
        CK(launch_offsets(W.counts.as<uint32_t>(), npairs + 1, W.offs.as<uint64_t>(), W.temp.p, tb, st));
        ev.stop(st);
        uint64_t nh = 0;
        unsigned int stage_over = 0;
        CK(cudaMemcpyAsync(&nh, W.offs.as<uint64_t>() + npairs, 8, cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(&stage_over, W.stage_over.p, 4, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        ctr.gpu_ms_scan += ev.ms();
        ctr.word_hits += nh;
        // Pair ranges whose word hits fit the stage buffers: one range unless the batch is huge
        // (an all-against-all search at word 7 makes tens of billions).  Every stage from the
        // write pass on works per pair, so ranges run one after another; masklevel and the hit
        // order run once over all of them.
        std::vector<uint64_t> ranges{0, npairs};
        std::vector<uint64_t> hoffs;
        if (nh > MAX_RANGE_HITS) {
            if (taps) throw Fail(RMB_ELIMIT, "stage taps take batches of at most 2^29 word hits");
            hoffs.resize(npairs + 1);
            CK(cudaMemcpy(hoffs.data(), W.offs.p, (npairs + 1) * 8, cudaMemcpyDeviceToHost));
            ranges.assign(1, 0);
            for (uint64_t pr = 0; pr < npairs; ++pr)
                if (hoffs[pr + 1] - hoffs[ranges.back()] > MAX_RANGE_HITS && pr > ranges.back()) ranges.push_back(pr);
            ranges.push_back(npairs);
        }
        bool tapped = false;
        const uint64_t nh_all = nh;
        for (size_t ri = 0; ri + 1 < ranges.size() && !tapped; ++ri) {
            const uint64_t pair0 = ranges[ri];
            const uint64_t npairs = ranges[ri + 1] - pair0;  // the pairs of this range
            const uint64_t nh = ranges.size() > 2 ? hoffs[pair0 + npairs] - hoffs[pair0] : nh_all;
            if (nh >= 0xffffffffull) throw Fail(RMB_ELIMIT, "more than 2^32 word hits in one pair range");
            if (ranges.size() > 2) {  // offsets local to the range
                tb = 0;
                CK(launch_offsets(W.counts.as<uint32_t>() + pair0, npairs + 1, W.offs.as<uint64_t>(), nullptr, tb,
                                  st));
                W.temp.ensure(tb);
                CK(launch_offsets(W.counts.as<uint32_t>() + pair0, npairs + 1, W.offs.as<uint64_t>(), W.temp.p, tb,
                                  st));
            }
            W.hits.ensure(nh * sizeof(SeedHit));
            W.hit_pair.ensure(nh * 4);
            ev.start(st);
            if (!stage_over)
                CK(launch_scan_gather(pair0, npairs, W.counts.as<uint32_t>(), W.offs.as<uint64_t>(),
                                      W.stage_start.as<uint32_t>(), W.stage.as<SeedHit>(), W.hits.as<SeedHit>(),
                                      W.hit_pair.as<uint32_t>(), C.sms, st));
            else  // a warp's stretch of the stage ran out: scan this range again, writing in place
                CK(launch_scan(true, C.L, Q, P.word_size, pair0, npairs, nullptr, W.offs.as<uint64_t>(),
                               W.hits.as<SeedHit>(), W.hit_pair.as<uint32_t>(), C.sms, st));
            ev.stop(st);
            CK(cudaStreamSynchronize(st));
            ctr.gpu_ms_scan += ev.ms();
            ctr.launches += 2;
            ctr.ms_scan += ms_since(t0);

            W.ub.ensure(std::max<uint64_t>(nh, 1) * sizeof(UngBox));
            std::vector<SurvivorRec> sv;
            if (C.tune.graph && P.pipeline != 1 && C.prelim_stream && !taps && !C.sched_log && P.schedule != 2) {
                // ---- the dedup through the prelim survivors as one graph, no host round trip
                t0 = std::chrono::steady_clock::now();
                uint32_t qmax = 0;
                for (uint32_t i = 0; i < nb; ++i) qmax = std::max(qmax, hqlen[i]);
                chain_graph(C, W, Q, ucut[qb], pair0, npairs, nh, qmax, sv, ctr);
                ctr.ms_prelim_dp += ms_since(t0);
            } else {
            // ---- ungapped extension of every hit, then the per-pair dedup; or, for hit-dense
            // pairs (most hits dropped by the hash), the dedup extending only what it admits
            t0 = std::chrono::steady_clock::now();
            const int32_t dx = C.tune.dedup_extend_hits_per_pair;
            const bool fused = P.pipeline != 1 && dx >= 0 && nh >= (uint64_t)dx * npairs;
            if (fused) {
                W.flags.ensure(nh + 1);
                W.dd_cells.ensure(std::max<uint64_t>(nh, 1) * diag_cell_bytes());
                W.ung_queue.ensure(16);
                W.dd_units.ensure(dedup_units_bytes(npairs, nh, C.sms));
                ev.start(st);
                CK(launch_dedup_extend(C.L, Q, C.d_params.as<DevParams>(), ucut[qb], pair0, npairs, nh,
                                       W.offs.as<uint64_t>(), W.hits.as<SeedHit>(), W.ub.as<UngBox>(),
                                       W.flags.as<uint8_t>(), W.dd_cells.p, W.ung_queue.as<unsigned long long>(),
                                       W.dd_units.p, C.sms, st));
                ev.stop(st);
                ctr.launches += 2;
            } else {
                ev.start(st);
                W.ung_queue.ensure(16);
                CK(launch_ungapped(C.L, Q, C.d_params.as<DevParams>(), ucut[qb], nh, W.hits.as<SeedHit>(),
                                   W.hit_pair.as<uint32_t>(), W.ub.as<UngBox>(), C.sms, st,
                                   P.pipeline == 1 ? nullptr : W.ung_queue.as<unsigned long long>(),
                                   C.tune.ungapped_blocks_per_sm));
                ev.stop(st);
                CK(cudaStreamSynchronize(st));
                ctr.gpu_ms_ungapped += ev.ms();
                ctr.launches += nh ? 1 : 0;
                ctr.ms_ungapped += ms_since(t0);
                t0 = std::chrono::steady_clock::now();
                W.flags.ensure(nh + 1);
                W.dd_scratch.ensure(dedup_threads(C.sms) * 1024 * 4);
                W.dd_cells.ensure(std::max<uint64_t>(nh, 1) * diag_cell_bytes());
                ev.start(st);
                CK(launch_dedup(C.L, Q, P.word_size, ucut[qb], pair0, npairs, W.offs.as<uint64_t>(), W.hits.as<SeedHit>(),
                                W.ub.as<UngBox>(), W.flags.as<uint8_t>(), W.dd_scratch.as<uint32_t>(), W.dd_cells.p, C.sms, st));
                ev.stop(st);
                ctr.launches += 1;
            }
            W.ung_idx.ensure(std::max<uint64_t>(nh, 1) * 4);
            W.n_sel.ensure(16);
            tb = 0;
            CK(launch_select_eq(W.flags.as<uint8_t>(), nh, 3, W.ung_idx.as<uint32_t>(), W.n_sel.as<uint32_t>(), nullptr, tb,
                                st));
            W.temp.ensure(tb);
            CK(launch_select_eq(W.flags.as<uint8_t>(), nh, 3, W.ung_idx.as<uint32_t>(), W.n_sel.as<uint32_t>(), W.temp.p,
                                tb, st));
            uint32_t nu = 0;
            CK(cudaMemcpyAsync(&nu, W.n_sel.p, 4, cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            ctr.gpu_ms_dedup += ev.ms();
            ctr.ms_dedup += ms_since(t0);
            ctr.ungapped += nu;
            if (taps && (taps->seeds || taps->ungapped)) {
                std::vector<SeedHit> hh(nh);
                std::vector<uint32_t> hp(nh);
                std::vector<uint8_t> fl(nh);
                std::vector<UngBox> uu(nh);
                if (nh) {
                    CK(cudaMemcpy(hh.data(), W.hits.p, nh * sizeof(SeedHit), cudaMemcpyDeviceToHost));
                    CK(cudaMemcpy(hp.data(), W.hit_pair.p, nh * 4, cudaMemcpyDeviceToHost));
                    CK(cudaMemcpy(fl.data(), W.flags.p, nh, cudaMemcpyDeviceToHost));
                    CK(cudaMemcpy(uu.data(), W.ub.p, nh * sizeof(UngBox), cudaMemcpyDeviceToHost));
                }
                for (uint64_t i = 0; i < nh; ++i) {
                    if (!fl[i]) continue;
                    const uint32_t qi = hp[i] / ns, si = hp[i] % ns;
                    const uint32_t s_len = C.slen[si];
                    const bool minus = hh[i].qs >> 31;
                    const uint32_t qo = hh[i].qs & 0x7fffffffu, so = hh[i].s;
                    if (taps->seeds) {
                        if (!minus) taps->seeds->insert(taps->seeds->end(), {0u, qo, so});
                        else {
                            const uint32_t en = (uint32_t)(P.word_size - hlw[qi]);
                            const uint32_t sl = so + (uint32_t)hlw[qi];
                            taps->seeds->insert(taps->seeds->end(), {1u, qo >= en ? qo - en : 0, s_len >= sl ? s_len - sl : 0});
                        }
                    }
                }
                if (taps->ungapped) {
                    // per pair, in the reference's sort order (engine.rs:1280-1309)
                    std::vector<std::vector<UngSurvivor>> per(npairs);
                    for (uint64_t i = 0; i < nh; ++i) {
                        if (fl[i] != 3) continue;
                        UngSurvivor r{};
                        r.q_seed = hh[i].qs & 0x7fffffffu;
                        r.s_seed = hh[i].s;
                        r.q_start = uu[i].q_start;
                        r.q_end = uu[i].q_end;
                        r.s_start = uu[i].s_start;
                        r.s_end = uu[i].s_end;
                        r.score = uu[i].score;
                        r.strand = (uint8_t)(hh[i].qs >> 31);
                        per[hp[i]].push_back(r);
                    }
                    for (uint64_t pr = 0; pr < npairs; ++pr) {
                        auto& v = per[pr];
                        if (v.empty()) continue;
                        const uint32_t qa = hqlen[pr / ns], sa = C.slen[pr % ns];
                        // sort exactly as phase2a_filter does, with every record kept
                        for (auto& r : v) { r.p_score = INT32_MIN; }
                        std::vector<UngSurvivor> w = v;
                        auto ss = [&](const UngSurvivor& r) { return r.strand == 0 ? r.s_start : sa - r.s_end; };
                        auto qk = [&](const UngSurvivor& r) -> uint64_t {
                            return r.strand == 0 ? r.q_start : ((uint64_t)qa + 1) + ((uint64_t)qa >= r.q_end ? qa - r.q_end : 0);
                        };
                        auto sk = [&](const UngSurvivor& r) { return r.strand == 0 ? r.s_seed : sa - r.s_seed; };
                        std::sort(w.begin(), w.end(), [&](const UngSurvivor& a, const UngSurvivor& b) {
                            if (a.score != b.score) return a.score > b.score;
                            if (ss(a) != ss(b)) return ss(a) < ss(b);
                            const uint32_t la = a.s_end - a.s_start, lb = b.s_end - b.s_start;
                            if (la != lb) return la > lb;
                            if (qk(a) != qk(b)) return qk(a) < qk(b);
                            return sk(a) < sk(b);
                        });
                        for (auto& r : w) {
                            const uint32_t s0 = r.strand == 0 ? r.s_start : sa - r.s_end;
                            const uint32_t s1 = r.strand == 0 ? r.s_end : sa - r.s_start;
                            taps->ungapped->insert(taps->ungapped->end(),
                                                   {(uint32_t)r.strand, r.q_start, r.q_end, s0, s1, (uint32_t)r.score});
                        }
                    }
                }
                if (!taps->prelims) { tapped = true; continue; }
            }

            // ---- preliminary gapped DP of every ungapped record
            t0 = std::chrono::steady_clock::now();
            W.po.ensure(std::max<uint64_t>(nu, 1) * sizeof(PrelimOut));
            W.wide.ensure(std::max<uint64_t>(nu, 1) * 4);
            W.n_wide.ensure(16);
            W.cells.ensure(16);
            W.fails.ensure(16);
            CK(cudaMemsetAsync(W.n_wide.p, 0, 16, st));
            CK(cudaMemsetAsync(W.cells.p, 0, 16, st));
            CK(cudaMemsetAsync(W.fails.p, 0, 16, st));
            ev.start(st);
            EvTimer ev_main, es;  // es: the learned order's kernels
            bool es_used = false;
            if (C.prelim_stream) {
                W.geo.ensure(std::max<uint64_t>(nu, 1) * prelim_geo_bytes());
                CK(launch_prelim_prep(C.L, Q, C.d_params.as<DevParams>(), nu, W.ung_idx.as<uint32_t>(),
                                      W.hits.as<SeedHit>(), W.hit_pair.as<uint32_t>(), W.ub.as<UngBox>(), W.geo.p, C.sms,
                                      st));
                ctr.launches += nu ? 1 : 0;
                const uint32_t* order = nullptr;
                uint32_t* cells_out = nullptr;
                if (C.sched_log && nu) {
                    // training pairs: each record's features, and its cells from the DP below
                    W.sched_feat.ensure(nu * SCHED_NF_HOST * 4);
                    W.sched_cells.ensure(nu * 4);
                    CK(launch_sched_features(C.L, Q, C.d_params.as<DevParams>(), nu, W.ung_idx.as<uint32_t>(),
                                             W.hits.as<SeedHit>(), W.hit_pair.as<uint32_t>(), W.ub.as<UngBox>(),
                                             W.counts.as<uint32_t>(), W.sched_feat.as<float>(), C.sms, st));
                    cells_out = W.sched_cells.as<uint32_t>();
                    ctr.launches += 1;
                } else if (C.p.schedule >= 1 && nu) {
                    // the records front-loaded by predicted cost (1), or all in descending cost (2)
                    W.sched_pred.ensure(nu * 4);
                    W.sched_order.ensure(nu * 4);
                    W.sched_scratch.ensure(sched_order_scratch_bytes());
                    size_t tb = C.p.schedule == 1 ? sched_front_temp_bytes(nu) : 0;
                    if (tb) W.temp.ensure(tb);
                    es.start(st);
                    es_used = true;
                    CK(launch_sched_order(C.L, Q, C.d_params.as<DevParams>(), nu, W.ung_idx.as<uint32_t>(),
                                          W.hits.as<SeedHit>(), W.hit_pair.as<uint32_t>(), W.ub.as<UngBox>(),
                                          W.counts.as<uint32_t>(), C.sched_params.as<float>(),
                                          W.sched_pred.as<float>(), W.sched_scratch.p, W.sched_order.as<uint32_t>(),
                                          C.sms, st, C.p.schedule, W.temp.p, tb));
                    es.stop(st);
                    order = W.sched_order.as<uint32_t>();
                    ctr.launches += 3;
                }
                ev_main.start(st);
                // the plain pipeline keeps the hand-swept shape; the batched one takes the tuned knobs
                const rmb_tune tn = P.pipeline == 1 ? default_tune() : C.tune;
                StreamLaunch cfg;
                cfg.group = tn.prelim_group;
                cfg.blocks_per_sm = tn.prelim_blocks_per_sm;
                cfg.window = tn.prelim_window;
                cfg.budget_div = tn.prelim_budget_div;
                CK(launch_prelim_stream(C.d_params.as<DevParams>(), nu, W.geo.p, W.po.as<PrelimOut>(),
                                        W.wide.as<uint32_t>(), W.n_wide.as<unsigned int>(),
                                        W.cells.as<unsigned long long>(), C.sms, st, order, cells_out,
                                        P.pipeline == 1, cfg,
                                        C.p.schedule == 1 && order
                                            ? StreamDevCounts{nullptr, sched_front_count(W.sched_scratch.p), nu}
                                            : StreamDevCounts{}));
                ev_main.stop(st);
                if (cells_out) {
                    std::vector<float> f(nu * SCHED_NF_HOST);
                    std::vector<uint32_t> c(nu);
                    CK(cudaMemcpyAsync(f.data(), W.sched_feat.p, f.size() * 4, cudaMemcpyDeviceToHost, st));
                    CK(cudaMemcpyAsync(c.data(), W.sched_cells.p, c.size() * 4, cudaMemcpyDeviceToHost, st));
                    CK(cudaStreamSynchronize(st));
                    for (uint64_t r = 0; r < nu; ++r) {
                        if (c[r] == 0xFFFFFFFFu) continue;  // passed on to the warp kernel
                        C.sched_log->feats.insert(C.sched_log->feats.end(), f.begin() + r * SCHED_NF_HOST,
                                                  f.begin() + (r + 1) * SCHED_NF_HOST);
                        C.sched_log->cells.push_back(c[r]);
                    }
                }
            }
            else
                CK(launch_prelim(C.L, Q, C.d_params.as<DevParams>(), nu, nullptr, W.ung_idx.as<uint32_t>(),
                                 W.hits.as<SeedHit>(), W.hit_pair.as<uint32_t>(), W.ub.as<UngBox>(), W.po.as<PrelimOut>(),
                                 W.wide.as<uint32_t>(), W.n_wide.as<unsigned int>(), W.cells.as<unsigned long long>(),
                                 C.sms, st));
            ev.stop(st);
            ctr.launches += nu ? 1 : 0;
            uint32_t nw = 0;
            unsigned long long main_cells = 0;
            CK(cudaMemcpyAsync(&nw, W.n_wide.p, 4, cudaMemcpyDeviceToHost, st));
            CK(cudaMemcpyAsync(&main_cells, W.cells.p, 8, cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            ctr.gpu_ms_prelim += ev.ms();
            if (C.prelim_stream) {
                ctr.gpu_ms_prelim_main += ev_main.ms();
                ctr.so_cells_main += main_cells;
            }
            if (es_used) ctr.gpu_ms_sched += es.ms();
            DBuf* wide_list = &W.wide;
            if (nw && C.prelim_stream) {
                // records whose band window outgrew the thread ring: the warp kernel's 256-cell rings
                W.wide2.ensure((uint64_t)nw * 4);
                W.dres.ensure((uint64_t)nw * 2 * sizeof(int4));
                CK(cudaMemsetAsync(W.n_wide.p, 0, 4, st));
                EvTimer e2;
                e2.start(st);
                CK(launch_prelim_split(C.L, Q, C.d_params.as<DevParams>(), nw, W.wide.as<uint32_t>(),
                                       W.ung_idx.as<uint32_t>(), W.hits.as<SeedHit>(), W.hit_pair.as<uint32_t>(),
                                       W.ub.as<UngBox>(), W.dres.as<int4>(), W.po.as<PrelimOut>(), W.wide2.as<uint32_t>(),
                                       W.n_wide.as<unsigned int>(), W.cells.as<unsigned long long>(), C.sms, st));
                e2.stop(st);
                ctr.launches += 2;
                CK(cudaMemcpyAsync(&nw, W.n_wide.p, 4, cudaMemcpyDeviceToHost, st));
                CK(cudaStreamSynchronize(st));
                ctr.gpu_ms_prelim += e2.ms();
                wide_list = &W.wide2;
            }
            if (nw) {
                uint32_t qmax = 0;
                for (uint32_t i = 0; i < nb; ++i) qmax = std::max(qmax, hqlen[i]);
                const uint64_t cap = (uint64_t)std::max(qmax, C.max_slen) + 2;
                const uint32_t threads = std::min<uint32_t>(nw, (uint32_t)std::max<uint64_t>(128, (1ull << 31) / (cap * 8)));
                W.band.ensure((uint64_t)((threads + 127) / 128 * 128) * cap * 8);
                EvTimer ew;
                ew.start(st);
                ctr.launches += 1;
                CK(launch_prelim_wide(C.L, Q, C.d_params.as<DevParams>(), nw, wide_list->as<uint32_t>(), W.ung_idx.as<uint32_t>(),
                                      W.hits.as<SeedHit>(), W.hit_pair.as<uint32_t>(), W.ub.as<UngBox>(),
                                      W.po.as<PrelimOut>(), W.band.as<int2>(), cap, threads,
                                      W.cells.as<unsigned long long>(), W.fails.as<unsigned int>(), st));
                ew.stop(st);
                ctr.gpu_ms_prelim += ew.ms();
            }
            unsigned long long cells = 0;
            unsigned int fails = 0;
            CK(cudaMemcpyAsync(&cells, W.cells.p, 8, cudaMemcpyDeviceToHost, st));
            CK(cudaMemcpyAsync(&fails, W.fails.p, 4, cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            if (fails) throw Fail(RMB_ECUDA, "prelim DP band exceeded its storage");
            ctr.so_cells += cells;
            ctr.prelim_dp += nu;
            // survivors (score >= gapped cutoff) to the host
            W.sel.ensure(std::max<uint64_t>(nu, 1) * 4);
            tb = 0;
            CK(launch_select_prelim(W.po.as<PrelimOut>(), nu, W.sel.as<uint32_t>(), W.n_sel.as<uint32_t>(), nullptr, tb, st));
            W.temp.ensure(tb);
            CK(launch_select_prelim(W.po.as<PrelimOut>(), nu, W.sel.as<uint32_t>(), W.n_sel.as<uint32_t>(), W.temp.p, tb, st));
            uint32_t nsv = 0;
            CK(cudaMemcpyAsync(&nsv, W.n_sel.p, 4, cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            W.surv.ensure(std::max<uint64_t>(nsv, 1) * sizeof(SurvivorRec));
            ctr.launches += nsv ? 1 : 0;
            CK(launch_gather_survivors(nsv, W.sel.as<uint32_t>(), W.ung_idx.as<uint32_t>(), W.hits.as<SeedHit>(),
                                       W.hit_pair.as<uint32_t>(), W.ub.as<UngBox>(), W.po.as<PrelimOut>(),
                                       W.surv.as<SurvivorRec>(), st));
            sv.resize(nsv);
            if (nsv) CK(cudaMemcpyAsync(sv.data(), W.surv.p, nsv * sizeof(SurvivorRec), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            ctr.ms_prelim_dp += ms_since(t0);
            }

            // ---- host Phase 2a filter per pair
            t0 = std::chrono::steady_clock::now();
            std::vector<uint32_t> pair_ids;
            std::vector<std::vector<UngSurvivor>> per_pair;
            for (const SurvivorRec& r : sv) {
                if (pair_ids.empty() || pair_ids.back() != r.pair) {
                    pair_ids.push_back(r.pair);
                    per_pair.emplace_back();
                }
                UngSurvivor u{};
                u.q_seed = r.hit.qs & 0x7fffffffu;
                u.s_seed = r.hit.s;
                u.q_start = r.ub.q_start;
                u.q_end = r.ub.q_end;
                u.s_start = r.ub.s_start;
                u.s_end = r.ub.s_end;
                u.score = r.ub.score;
                u.strand = (uint8_t)(r.hit.qs >> 31);
                u.p_score = r.po.score;
                u.p_qs = r.po.q_start;
                u.p_qe = r.po.q_end;
                u.p_ss = r.po.s_start;
                u.p_se = r.po.s_end;
                u.tb_q = r.po.tb_q;
                u.tb_s = r.po.tb_s;
                per_pair.back().push_back(u);
            }
            const size_t np = pair_ids.size();
            std::vector<std::vector<Prelim>> prelims(np);
            parallel_for(np, [&](size_t k) {
                const uint32_t qa = hqlen[pair_ids[k] / ns], sa = C.slen[pair_ids[k] % ns];
                prelims[k] = phase2a_filter(per_pair[k], qa, sa);
                if (!collect) sort_prelims_for_traceback(prelims[k], qa, sa);
            });
            per_pair.clear();
            uint64_t n_pre = 0;
            for (auto& v : prelims) n_pre += v.size();
            ctr.prelims += n_pre;
            if (taps && taps->prelims) {
                // in pipeline (purge) order: re-run the purge order is not kept after the traceback
                // sort, so report them in traceback order per pair
                for (size_t k = 0; k < np; ++k)
                    for (const Prelim& p : prelims[k])
                        taps->prelims->insert(taps->prelims->end(), {(uint32_t)p.strand, p.q_start, p.q_end, p.s_start,
                                                                     p.s_end, (uint32_t)p.score, p.q_seed, p.s_seed});
                tapped = true;
                continue;
            }
            ctr.ms_host_2a += ms_since(t0);
            if (collect) {
                for (size_t k = 0; k < np; ++k)
                    collect->push_back(PairPrelims{qb + pair_ids[k] / ns, pair_ids[k] % ns, std::move(prelims[k])});
                continue;  // next range
            }

            // ---- traceback DP and host Phase 2b of every prelim
            if (pending.valid()) add_counters(ctr, pending.get());
            if (traceback_2b(C, W, Q, hqlen.data(), nb, qhost, pair_ids, prelims, out_hits.data() + qb, ctr, taps,
                             P.pipeline != 1 && !taps ? &pending : nullptr)) {
                tapped = true;
                continue;
            }
        }
        if (tail && !tapped && !collect) {
            *tail = std::async(std::launch::async, [&C, &out_hits, qb, nb, hqlen, pending = std::move(pending)]() mutable {
                rmb_counters c{};
                if (pending.valid()) c = pending.get();
                const auto t3 = std::chrono::steady_clock::now();
                parallel_for(nb, [&](size_t i) { finish_query(C, out_hits[qb + i], hqlen[i]); });
                for (uint32_t i = 0; i < nb; ++i) c.finals += out_hits[qb + i].size();
                c.ms_host_2b += ms_since(t3);
                return c;
            });
            return;
        }
        if (pending.valid()) add_counters(ctr, pending.get());
        if (tapped || collect) return;
        t0 = std::chrono::steady_clock::now();
        parallel_for(nb, [&](size_t i) { finish_query(C, out_hits[qb + i], hqlen[i]); });
        for (uint32_t i = 0; i < nb; ++i) ctr.finals += out_hits[qb + i].size();
        ctr.ms_host_2b += ms_since(t0);
    };
    if (lanes == 1) {
        // the batched pipeline: each sub-batch's host tail beside the next one's kernels
        const bool overlap = P.pipeline != 1 && !taps && !collect;
        Tail last;
        auto join = [&]() {
            if (last.valid()) add_counters(ctr, last.get());
        };
        for (auto& sb : subs) {
            Tail next;
            sub_batch(C.work[0], sb.first, sb.second, ctr, overlap ? &next : nullptr);
            join();
            last = std::move(next);
        }
        join();
        return;
    }
    // lane k takes sub-batches k, k + 2, ... in order; lane 1 on a host thread of its own
    rmb_counters c1{};
    std::exception_ptr err1;
    std::thread t1([&]() {
        try {
            CK(cudaSetDevice(C.p.device));
            for (size_t i = 1; i < subs.size(); i += 2) sub_batch(C.work[1], subs[i].first, subs[i].second, c1, nullptr);
        } catch (...) {
            err1 = std::current_exception();
        }
    });
    std::exception_ptr err0;
    try {
        for (size_t i = 0; i < subs.size(); i += 2) sub_batch(C.work[0], subs[i].first, subs[i].second, ctr, nullptr);
    } catch (...) {
        err0 = std::current_exception();
    }
    t1.join();
    if (err0) std::rethrow_exception(err0);
    if (err1) std::rethrow_exception(err1);
    add_counters(ctr, c1);
}

// Traceback DP on the device and the host Phase 2b (engine.rs:1438-1762) of the prelims of
// (query, subject) pairs; pair = local query * n_subjects + subject over the queries of Q, whose
// lengths are hqlen and host copies qhost(local).  Hits go to out[local query].  Returns true
// when the traceback stage tap took the results instead.  With `defer` (no taps), the whole step,
// the traceback kernels on the lane's second stream and the host Phase 2b, runs on a thread of
// its own and *defer holds it (its counters): the caller waits for it before the next call (the
// traceback buffers and the hits of the same queries) and before it reads the hits.
bool traceback_2b(rmb_ctx& C, Work& W, const DevQueries& Q, const uint32_t* hqlen_in, uint32_t nb,
                  const std::function<const uint8_t*(uint32_t)>& qhost_in, const std::vector<uint32_t>& pair_ids_in,
                  std::vector<std::vector<Prelim>>& prelims_in, std::vector<Hit>* out, rmb_counters& ctr_in,
                  Taps* taps, std::future<rmb_counters>* defer) {
    // everything the job reads is owned by it or outlives the caller's sub-batch
    auto job = [&C, &W, Q, nb, out, taps, hq = std::vector<uint32_t>(hqlen_in, hqlen_in + nb), qhost = qhost_in,
                pair_ids = pair_ids_in, prelims = std::move(prelims_in)](rmb_counters& ctr,
                                                                          cudaStream_t st) mutable -> bool {
        const uint32_t* hqlen = hq.data();
        const uint32_t ns = (uint32_t)C.ids.size();
        const size_t np = pair_ids.size();
        unsigned long long cells = 0;
        std::unique_lock<std::mutex> tb_lock(W.tb_mu);  // the lane's traceback buffers, until the results are back
        auto t0 = std::chrono::steady_clock::now();
        {
            // ---- traceback DP of every prelim (GPU), with retries for scratch overflow
            uint64_t n_pre = 0;
            for (auto& v : prelims) n_pre += v.size();
            std::vector<TbIn> tin;
            tin.reserve(n_pre);
            std::vector<uint64_t> pre_off(np + 1, 0);
            for (size_t k = 0; k < np; ++k) {
                pre_off[k + 1] = pre_off[k] + prelims[k].size();
                for (const Prelim& p : prelims[k])
                    tin.push_back(TbIn{pair_ids[k], p.strand, p.q_seed, p.s_seed, p.q_start, p.q_end, p.s_start, p.s_end});
            }
            std::vector<TbResult> tres(tin.size());
            // each finished item's script stays packed in its round's ops until Phase 2b unpacks it
            // (in parallel, per pair): round, offset and count per item
            std::vector<std::vector<uint32_t>> rounds_ops;
            std::vector<uint32_t> raw_round(tin.size(), 0), raw_n(tin.size(), 0);
            std::vector<uint64_t> raw_off(tin.size(), 0);
            if (!tin.empty()) {
                uint32_t qmax = 0;
                for (uint32_t i = 0; i < nb; ++i) qmax = std::max(qmax, hqlen[i]);
                // batched: largest prelim boxes first (warps take items round-robin, so the long
                // alignments start in the first wave instead of stretching the end of the launch);
                // plain: in arrival order
                std::vector<uint32_t> todo(tin.size());
                for (uint32_t i = 0; i < todo.size(); ++i) todo[i] = i;
                auto box = [&](uint32_t i) {
                    return (uint64_t)(tin[i].q_end - tin[i].q_start) + (uint64_t)(tin[i].s_end - tin[i].s_start);
                };
                if (C.p.pipeline != 1)
                    std::stable_sort(todo.begin(), todo.end(), [&](uint32_t x, uint32_t y) { return box(x) > box(y); });
                uint64_t trace_cap = 1ull << 20;
                uint32_t ops_cap = 1024;
                int rounds = 0;
                while (!todo.empty()) {
                    if (++rounds > 12) throw Fail(RMB_ENOMEM, "traceback scratch kept overflowing");
                    std::vector<TbIn> chunk_in(todo.size());
                    for (size_t i = 0; i < todo.size(); ++i) chunk_in[i] = tin[todo[i]];
                    const uint64_t band_cells = (uint64_t)C.max_slen + 2;
                    const uint32_t rows_cap = qmax + 2;
                    const uint64_t per_thread = ((band_cells * 8 + (uint64_t)rows_cap * 8 + trace_cap) + 255) & ~255ull;
                    const uint64_t budget = 8ull << 30;
                    // one warp per scratch slot (two items, the left and the right extension, per
                    // prelim), blocks of 8 warps
                    // (the plain pipeline: one prelim per warp, its two extensions in turn)
                    const bool whole = C.p.pipeline == 1;
                    uint32_t threads = (uint32_t)std::min<uint64_t>((whole ? 1 : 2) * todo.size(),
                                                                    std::max<uint64_t>(8, budget / per_thread));
                    threads = (threads + 7) / 8 * 8;
                    upload(W.tb_in, chunk_in, st);
                    W.tb_out.ensure(todo.size() * sizeof(TbOut));
                    W.tb_half.ensure(2 * todo.size() * sizeof(TbHalf));
                    W.tb_ops.ensure(2 * todo.size() * (uint64_t)ops_cap * 4);
                    W.tb_scratch.ensure((uint64_t)threads * per_thread);
                    W.tb_cells.ensure(8);
                    CK(cudaMemsetAsync(W.tb_cells.p, 0, 8, st));
                    EvTimer et;
                    et.start(st);
                    ctr.launches += 2;
                    CK(launch_traceback(C.L, Q, C.d_params.as<DevParams>(), (uint32_t)todo.size(), W.tb_in.as<TbIn>(),
                                        W.tb_out.as<TbOut>(), W.tb_half.as<TbHalf>(), W.tb_ops.as<uint32_t>(), ops_cap,
                                        W.tb_scratch.as<uint8_t>(),
                                        per_thread, band_cells, rows_cap, threads, W.tb_cells.as<unsigned long long>(),
                                        whole, st));
                    et.stop(st);
                    std::vector<TbOut> to(todo.size());
                    CK(cudaMemcpyAsync(to.data(), W.tb_out.p, to.size() * sizeof(TbOut), cudaMemcpyDeviceToHost, st));
                    CK(cudaMemcpyAsync(&cells, W.tb_cells.p, 8, cudaMemcpyDeviceToHost, st));
                    CK(cudaStreamSynchronize(st));
                    ctr.gpu_ms_traceback += et.ms();
                    // only the ops of the finished items come back, packed
                    std::vector<uint64_t> ooff(todo.size() + 1, 0);
                    for (size_t i = 0; i < todo.size(); ++i)
                        ooff[i + 1] = ooff[i] + (to[i].status == 2 ? 0 : to[i].n_ops);
                    std::vector<uint32_t> ops(ooff.back());
                    if (!ops.empty()) {
                        upload(W.tb_ooff, ooff, st);
                        W.tb_ops2.ensure(ops.size() * 4);
                        // the merged script of prelim i sits in ops slot 2 i
                        CK(launch_gather_ops((uint32_t)todo.size(), W.tb_ops.as<uint32_t>(), 2 * ops_cap, W.tb_out.as<TbOut>(),
                                             W.tb_ooff.as<uint64_t>(), W.tb_ops2.as<uint32_t>(), C.sms, st));
                        CK(cudaMemcpyAsync(ops.data(), W.tb_ops2.p, ops.size() * 4, cudaMemcpyDeviceToHost, st));
                        CK(cudaStreamSynchronize(st));
                        ctr.launches += 1;
                    }
                    std::vector<uint32_t> again;
                    const uint32_t round_id = (uint32_t)rounds_ops.size();
                    for (size_t i = 0; i < todo.size(); ++i) {
                        const TbOut& o = to[i];
                        if (o.status == 2) { again.push_back(todo[i]); continue; }
                        if (o.status == 3) throw Fail(RMB_ECUDA, "traceback walk did not reach the origin");
                        TbResult& r = tres[todo[i]];
                        r.status = o.status;
                        r.score = o.score;
                        r.q0 = o.q0;
                        r.q1 = o.q1;
                        r.s0 = o.s0;
                        r.s1 = o.s1;
                        raw_round[todo[i]] = round_id;
                        raw_off[todo[i]] = ooff[i];
                        raw_n[todo[i]] = o.n_ops;
                    }
                    rounds_ops.push_back(std::move(ops));
                    if (again.size() == todo.size()) {  // nothing finished: grow the caps
                        trace_cap *= 4;
                        ops_cap *= 4;
                    } else if (!again.empty()) {
                        trace_cap *= 4;
                        ops_cap *= 4;
                    }
                    ctr.tb_cells += cells;
                    todo.swap(again);
                }
            }
            ctr.tb_dp += tin.size();
            tb_lock.unlock();  // the results are on the host
            ctr.ms_traceback += ms_since(t0);
            // item k's script from its round's packed ops (op << 30 | count)
            auto unpack = [](const std::vector<std::vector<uint32_t>>& rops, uint32_t rd, uint64_t off, uint32_t n,
                             Script& out) {
                out.clear();
                if (!n) return;
                const uint32_t* v = rops[rd].data() + off;
                for (uint32_t j = 0; j < n; ++j) out.push_back(RunOp{(uint8_t)(v[j] >> 30), v[j] & 0x3fffffffu});
            };
            if (taps && taps->tracebacks) {
                for (size_t k = 0; k < tin.size(); ++k) unpack(rounds_ops, raw_round[k], raw_off[k], raw_n[k], tres[k].script);
                for (size_t k = 0; k < tin.size(); ++k) {
                    const TbResult& r = tres[k];
                    uint32_t h = 2166136261u;  // FNV-1a over the run-length ops
                    for (const RunOp& o : r.script) {
                        const uint32_t v = ((uint32_t)o.op << 30) | o.n;
                        for (int b = 0; b < 4; ++b) h = (h ^ ((v >> (8 * b)) & 0xffu)) * 16777619u;
                    }
                    const bool ok = r.status == 0;
                    taps->tracebacks->insert(taps->tracebacks->end(),
                                             {tin[k].strand, ok ? 0u : 1u, ok ? (uint32_t)r.score : 0u, ok ? r.q0 : 0u,
                                              ok ? r.q1 : 0u, ok ? r.s0 : 0u, ok ? r.s1 : 0u,
                                              ok ? (uint32_t)r.script.size() : 0u, ok ? h : 2166136261u});
                }
                return true;
            }

            // ---- host Phase 2b per pair, then per query
            // everything it reads is owned by it or outlives the caller's sub-batch (it may still run
            // after the sub-batch body has returned, held by the sub-batch's host tail)
            auto phase2b = [&C, ns, np, out, hqlen = std::vector<uint32_t>(hqlen, hqlen + nb), qhost, pair_ids,
                            prelims = std::move(prelims),
                            tres = std::move(tres), pre_off = std::move(pre_off), rounds_ops = std::move(rounds_ops),
                            raw_round = std::move(raw_round), raw_off = std::move(raw_off), raw_n = std::move(raw_n),
                            unpack]() mutable {
                const auto t2 = std::chrono::steady_clock::now();
                std::vector<std::vector<Hit>> pair_hits(np);
                // the reverse complement of each query with prelims, once
                std::vector<uint32_t> uq;
                for (size_t k = 0; k < np; ++k) uq.push_back(pair_ids[k] / ns);
                std::sort(uq.begin(), uq.end());
                uq.erase(std::unique(uq.begin(), uq.end()), uq.end());
                std::vector<std::vector<uint8_t>> qrcs(uq.size());
                parallel_for(uq.size(), [&](size_t j) { qrcs[j] = revcomp_full(qhost(uq[j]), hqlen[uq[j]] + 2); });
                parallel_for(np, [&](size_t k) {
                    const uint32_t qi = pair_ids[k] / ns, si = pair_ids[k] % ns;
                    const uint8_t* qs = qhost(qi);
                    const std::vector<uint8_t>& qrc = qrcs[std::lower_bound(uq.begin(), uq.end(), qi) - uq.begin()];
                    SubjectView v;
                    v.align = C.h_align.data() + C.plus_off[si];
                    v.align_rc = C.h_align_rc.data() + C.plus_off[si];
                    v.n_mask = C.mask_off[si] >= 0 ? C.h_mask.data() + C.mask_off[si] : nullptr;
                    v.n_mask_rc = C.mask_off[si] >= 0 ? C.h_mask_rc.data() + C.mask_off[si] : nullptr;
                    v.len = C.slen[si];
                    std::vector<TbResult> tr(tres.begin() + pre_off[k], tres.begin() + pre_off[k + 1]);
                    for (uint64_t j = pre_off[k]; j < pre_off[k + 1]; ++j)
                        unpack(rounds_ops, raw_round[j], raw_off[j], raw_n[j], tr[j - pre_off[k]].script);
                    pair_hits[k] = phase2b_filter(prelims[k], tr, qs, qrc.data(), hqlen[qi], v, si, C.gp);
                });
                for (size_t k = 0; k < np; ++k) {
                    const uint32_t qi = pair_ids[k] / ns;
                    auto& dst = out[qi];
                    for (auto& h : pair_hits[k]) {
                        h.q_len = hqlen[qi];
                        dst.push_back(std::move(h));
                    }
                }
                return ms_since(t2);
            };
            ctr.ms_host_2b += phase2b();
        }
        return false;
    };
    if (defer) {
        const int dev = C.p.device;
        cudaStream_t st2 = W.st2;
        *defer = std::async(std::launch::async, [job = std::move(job), dev, st2]() mutable {
            CK(cudaSetDevice(dev));
            rmb_counters c{};
            job(c, st2);
            return c;
        });
        return false;
    }
    return job(ctr_in, W.st);
}

int fail_out(const std::exception& e, char* err, size_t errlen, int code) {
    if (err && errlen) {
        strncpy(err, e.what(), errlen - 1);
        err[errlen - 1] = 0;
    }
    return code;
}

}  // namespace

extern "C" {

const char* rmb_version(void) { return "rmblast-b200 0.1 (sm_100a)"; }

int rmb_ctx_create(const rmb_params* params, const int32_t scores[256], const double freqs[16], double lambda,
                   const char* matrix_name, rmb_ctx** out, char* err, size_t errlen) {
    rmb_ctx* C = nullptr;
    try {
        if (!params || !scores || !freqs || !out) throw Fail(RMB_EINVAL, "null argument");
        const rmb_params& p = *params;
        if (p.word_size < 4) throw Fail(RMB_EINVAL, "word_size must be at least 4");
        if (p.gap_open < 0 || p.gap_extend < 1) throw Fail(RMB_EINVAL, "gap costs out of range");
        if (p.xdrop_ungap < 0 || p.xdrop_gap < 0 || p.xdrop_gap_final < 0 || p.min_raw_gapped_score < 0)
            throw Fail(RMB_EINVAL, "negative X-drop or cutoff");
        if (p.schedule < 0 || p.schedule > 2)
            throw Fail(RMB_EINVAL, "schedule must be 0 (FIFO), 1 (learned, front-loaded) or 2 (learned, full order)");
        if (p.kernels != 0 && p.kernels != 1) throw Fail(RMB_EINVAL, "kernels must be 0 (automatic) or 1 (warp prelim)");
        if (p.pipeline != 0 && p.pipeline != 1) throw Fail(RMB_EINVAL, "pipeline must be 0 (batched) or 1 (plain)");
        if (p.pipeline == 1 && p.schedule != 0)
            throw Fail(RMB_EINVAL, "the learned order feeds the batched pipeline's record queue (pipeline 0)");
        C = new rmb_ctx();
        C->p = p;
        C->matrix_name = matrix_name ? matrix_name : "";
        C->gp.gap_open = p.gap_open;
        C->gp.gap_extend = p.gap_extend;
        C->gp.gapped_cutoff = p.min_raw_gapped_score > 1 ? p.min_raw_gapped_score : 1;
        C->gp.complexity_adjust = p.complexity_adjust != 0;
        for (int i = 0; i < 16; ++i)
            for (int j = 0; j < 16; ++j) C->gp.matrix[i][j] = scores[i * 16 + j];
        for (int i = 0; i < 16; ++i) C->gp.freqs[i] = freqs[i];
        C->gp.lambda = lambda;
        int ndev = 0;
        CK(cudaGetDeviceCount(&ndev));
        if (p.device < 0 || p.device >= ndev) throw Fail(RMB_EINVAL, "no such CUDA device");
        CK(cudaSetDevice(p.device));
        cudaDeviceProp prop;
        CK(cudaGetDeviceProperties(&prop, p.device));
        if (prop.major < 10) throw Fail(RMB_EINVAL, "this library is built for sm_100a (B200)");
        C->sms = prop.multiProcessorCount;
        CK(cudaStreamCreateWithFlags(&C->st, cudaStreamNonBlocking));
        for (Work& w : C->work) {
            CK(cudaStreamCreateWithFlags(&w.st, cudaStreamNonBlocking));
            CK(cudaStreamCreateWithFlags(&w.st2, cudaStreamNonBlocking));
        }
        DevParams dp{};
        dp.gap_open = p.gap_open;
        dp.gap_extend = p.gap_extend;
        dp.word_size = p.word_size;
        dp.xdrop_ungap = p.xdrop_ungap;
        dp.xdrop_gap = p.xdrop_gap;
        dp.xdrop_gap_final = p.xdrop_gap_final;
        dp.gapped_cutoff = C->gp.gapped_cutoff;
        for (int i = 0; i < 256; ++i) dp.matrix[i] = scores[i];
        C->prelim_stream = p.kernels == 0 && prelim_stream_eligible(dp.matrix, p.gap_open, p.gap_extend, p.xdrop_gap);
        if (p.ka_lambda > 0.0) {
            if (!(p.ka_k > 0.0) || !(p.ka_h > 0.0) || !(p.ka_alpha > 0.0))
                throw Fail(RMB_EINVAL, "statistics need K, H and alpha > 0 with lambda > 0");
            C->ka.lambda = p.ka_lambda;
            C->ka.k = p.ka_k;
            C->ka.log_k = std::log(p.ka_k);
            C->ka.h = p.ka_h;
            C->ka.alpha = p.ka_alpha;
            C->ka.beta = p.ka_beta;
        }
        if (p.evalue < 0.0) throw Fail(RMB_EINVAL, "evalue must be >= 0");
        C->d_params.ensure(sizeof(DevParams));
        CK(cudaMemcpy(C->d_params.p, &dp, sizeof dp, cudaMemcpyHostToDevice));
        *out = C;
        return RMB_OK;
    } catch (const Fail& e) {
        delete C;
        return fail_out(e, err, errlen, e.code);
    } catch (const std::exception& e) {
        delete C;
        return fail_out(e, err, errlen, RMB_EINVAL);
    }
}

int rmb_db_load(rmb_ctx* C, uint32_t n, const uint8_t* const* plus, const uint32_t* len, const uint8_t* const* n_mask,
                const char* const* ids, char* err, size_t errlen) {
    try {
        if (!C || !plus || !len || !ids) throw Fail(RMB_EINVAL, "null argument");
        if (n == 0) throw Fail(RMB_EINVAL, "the database contains no sequences");
        CK(cudaSetDevice(C->p.device));
        C->ids.assign(ids, ids + n);
        C->slen.assign(len, len + n);
        C->plus_off.resize(n);
        C->packed_off.resize(n);
        C->mask_off.assign(n, -1);
        C->h_align.clear();
        C->h_align_rc.clear();
        C->h_mask.clear();
        C->h_mask_rc.clear();
        std::vector<uint8_t> hplus, hrc, packed;
        C->total_letters = 0;
        C->max_slen = 0;
        for (uint32_t i = 0; i < n; ++i) {
            const uint32_t L = len[i];
            if (plus[i][0] != 15 || plus[i][L + 1] != 15) throw Fail(RMB_EINVAL, "subject is not sentinel-wrapped");
            C->total_letters += L;
            C->max_slen = std::max(C->max_slen, L);
            C->plus_off[i] = hplus.size();
            hplus.insert(hplus.end(), plus[i], plus[i] + L + 2);
            auto rc = revcomp_full(plus[i], L + 2);
            hrc.insert(hrc.end(), rc.begin(), rc.end());
            std::vector<uint8_t> al(plus[i], plus[i] + L + 2);
            if (n_mask && n_mask[i]) {
                C->mask_off[i] = (int64_t)C->h_mask.size();
                C->h_mask.insert(C->h_mask.end(), n_mask[i], n_mask[i] + L);
                for (uint32_t k = 0; k < L; ++k) {
                    const uint8_t c = n_mask[i][L - 1 - k];
                    C->h_mask_rc.push_back(c ? COMPL[c & 15] : 0);
                    if (n_mask[i][k]) al[k + 1] = n_mask[i][k];
                }
            }
            C->h_align.insert(C->h_align.end(), al.begin(), al.end());
            auto arc = revcomp_full(al.data(), al.size());
            C->h_align_rc.insert(C->h_align_rc.end(), arc.begin(), arc.end());
            // blast/util.rs:85-115: 3 pad bytes, 4 bases per byte (first base in bits 7:6), 3 pad bytes.
            // The plus strand is CRandom-resolved, so every base is 0..3.
            packed.insert(packed.end(), 3, 0);
            C->packed_off[i] = packed.size();
            for (uint32_t j = 0; j < L; j += 4) {
                uint8_t byte = 0;
                for (uint32_t k = 0; k < 4; ++k) {
                    const uint8_t b = j + k < L ? plus[i][1 + j + k] : 0;
                    if (j + k < L && b > 3) throw Fail(RMB_EINVAL, "subject bases must be CRandom-resolved (0..3)");
                    byte = (uint8_t)((byte << 2) | (b & 3));
                }
                packed.push_back(byte);
            }
            packed.insert(packed.end(), 3, 0);
        }
        packed.insert(packed.end(), 4, 0);
        cudaStream_t st = C->st;
        upload(C->d_plus, hplus, st);
        upload(C->d_rc, hrc, st);
        upload(C->d_align, C->h_align, st);
        upload(C->d_align_rc, C->h_align_rc, st);
        upload(C->d_packed, packed, st);
        upload(C->d_plus_off, C->plus_off, st);
        upload(C->d_packed_off, C->packed_off, st);
        upload(C->d_len, C->slen, st);
        CK(cudaStreamSynchronize(st));
        C->L = DevLib{C->d_plus.as<uint8_t>(),      C->d_rc.as<uint8_t>(),         C->d_align.as<uint8_t>(),
                      C->d_align_rc.as<uint8_t>(),  C->d_packed.as<uint8_t>(),     C->d_plus_off.as<uint64_t>(),
                      C->d_packed_off.as<uint64_t>(), C->d_len.as<uint32_t>(), n};
        C->loaded = true;
        return RMB_OK;
    } catch (const Fail& e) {
        return fail_out(e, err, errlen, e.code);
    } catch (const std::bad_alloc& e) {
        return fail_out(e, err, errlen, RMB_ENOMEM);
    } catch (const std::exception& e) {
        return fail_out(e, err, errlen, RMB_EINVAL);
    }
}

static void check_queries(uint32_t nq, const uint8_t* const* query, const uint32_t* qlen) {
    if (nq && (!query || !qlen)) throw Fail(RMB_EINVAL, "null argument");
    for (uint32_t i = 0; i < nq; ++i)
        if (!query[i] || query[i][0] != 15 || query[i][qlen[i] + 1] != 15)
            throw Fail(RMB_EINVAL, "query is not sentinel-wrapped BLASTNA");
}

// The queries on the device (and a pinned host copy), in a new object or, for `into`, in one whose
// buffers are reused (rmb_search_batch keeps one per context).
static rmb_queries* make_queries(rmb_ctx* C, uint32_t nq, const uint8_t* const* query, const uint32_t* qlen,
                                 rmb_queries* into = nullptr) {
    check_queries(nq, query, qlen);
    rmb_queries* H = into ? into : new rmb_queries();
    try {
        H->dusted = false;
        H->n = nq;
        H->device = C->p.device;
        H->len.assign(qlen, qlen + nq);
        H->off.resize(nq);
        uint64_t tot = 0;
        for (uint32_t i = 0; i < nq; ++i) {
            H->off[i] = tot;
            tot += (uint64_t)qlen[i] + 2;
        }
        H->host.resize(std::max<uint64_t>(tot, 1));
        for (uint32_t i = 0; i < nq; ++i) memcpy(H->host.data() + H->off[i], query[i], (size_t)qlen[i] + 2);
        cudaStream_t st = C->st;
        H->d_q.ensure(H->host.size());
        H->d_qrc.ensure(H->host.size());
        CK(cudaMemcpyAsync(H->d_q.p, H->host.data(), tot, cudaMemcpyHostToDevice, st));
        upload(H->d_off, H->off, st);
        upload(H->d_len, H->len, st);
        CK(launch_revcomp(H->d_q.as<uint8_t>(), H->d_off.as<uint64_t>(), H->d_len.as<uint32_t>(), nq,
                          H->d_qrc.as<uint8_t>(), st));
        CK(cudaStreamSynchronize(st));
        return H;
    } catch (...) {
        if (!into) {
            H->release();
            delete H;
        }
        throw;
    }
}

}  // extern "C"

namespace {

struct QueriesDeleter {
    void operator()(rmb_queries* H) const {
        if (!H) return;
        H->release();
        delete H;
    }
};
using QueriesPtr = std::unique_ptr<rmb_queries, QueriesDeleter>;

// main.rs:1236-1251 (NCBI SplitQuery_CalculateNumChunks + x_ComputeChunkRanges): the chunks
// [start, end) of a query; one chunk below 1,999,800 bp.
std::vector<std::pair<uint32_t, uint32_t>> query_chunks(uint64_t qlen, int word_size) {
    const uint64_t CHUNK = 1000000, OVERLAP = 100;
    const uint64_t n = qlen / (CHUNK - OVERLAP);
    std::vector<std::pair<uint32_t, uint32_t>> out;
    if (n <= 1) {
        out.push_back({0, (uint32_t)qlen});
        return out;
    }
    uint64_t cs = (qlen + (n - 1) * OVERLAP) / n;
    if (n < (cs > OVERLAP ? cs - OVERLAP : 0)) ++cs;
    const uint64_t step = cs > OVERLAP ? cs - OVERLAP : 0;
    for (uint64_t k = 0; k < n; ++k) {
        const uint64_t b = k * step;
        if (b >= qlen) break;
        const uint64_t e = std::min(b + cs, qlen);
        if (e - b < (uint64_t)word_size) break;
        out.push_back({(uint32_t)b, (uint32_t)e});
    }
    return out;
}

// main.rs:1018-1085 merge_chunk_prelims (NCBI Blast_HSPListsMerge): a chunk's prelims, in full-
// query coordinates, into the ones accumulated so far for the same subject; plus strand only.
// Each accumulated candidate, best first, absorbs every close new one whose start or end lies in
// its box, growing as it does; the merged score is the density of the two over the merged length
// (f64, as the reference) or the better score.
void merge_chunk_prelims(std::vector<Prelim>& acc, std::vector<Prelim>& add, uint32_t split) {
    const uint32_t OVERLAP = 100;
    const int64_t DIAG_CLOSE = 10;
    auto order = [](const Prelim& a, const Prelim& b) {  // ScoreCompareHSPs for plus-strand HSPs
        if (a.score != b.score) return a.score > b.score;
        if (a.s_start != b.s_start) return a.s_start < b.s_start;
        if (a.s_end != b.s_end) return a.s_end > b.s_end;
        if (a.q_start != b.q_start) return a.q_start < b.q_start;
        return a.q_end > b.q_end;
    };
    std::vector<uint8_t> absorbed(add.size(), 0);
    std::vector<size_t> ac, nc;
    for (size_t i = 0; i < acc.size(); ++i)
        if (acc[i].strand == 0 && acc[i].q_end > split) ac.push_back(i);
    std::stable_sort(ac.begin(), ac.end(), [&](size_t a, size_t b) { return order(acc[a], acc[b]); });
    for (size_t j = 0; j < add.size(); ++j)
        if (add[j].strand == 0 && add[j].q_start < split + OVERLAP) nc.push_back(j);
    std::stable_sort(nc.begin(), nc.end(), [&](size_t a, size_t b) { return order(add[a], add[b]); });
    for (size_t i : ac) {
        Prelim& h1 = acc[i];
        for (size_t j : nc) {
            if (absorbed[j]) continue;
            const Prelim& h2 = add[j];
            const int64_t dd = ((int64_t)h1.q_end - (int64_t)h1.s_end) - ((int64_t)h2.q_start - (int64_t)h2.s_start);
            if ((dd < 0 ? -dd : dd) >= DIAG_CLOSE) continue;
            const bool start_in = h2.q_start >= h1.q_start && h2.q_start <= h1.q_end && h2.s_start >= h1.s_start &&
                                  h2.s_start <= h1.s_end;
            const bool end_in = h2.q_end >= h1.q_start && h2.q_end <= h1.q_end && h2.s_end >= h1.s_start &&
                                h2.s_end <= h1.s_end;
            if (!start_in && !end_in) continue;
            const double density =
                (double)(h1.score + h2.score) / (double)((h1.q_end - h1.q_start) + (h2.q_end - h2.q_start));
            h1.q_start = std::min(h1.q_start, h2.q_start);
            h1.s_start = std::min(h1.s_start, h2.s_start);
            h1.q_end = std::max(h1.q_end, h2.q_end);
            h1.s_end = std::max(h1.s_end, h2.s_end);
            if (h2.score > h1.score) {
                h1.q_seed = h2.q_seed;
                h1.s_seed = h2.s_seed;
                h1.score = h2.score;
            }
            h1.score = std::max(h1.score, (int32_t)(density * (double)(h1.q_end - h1.q_start)));
            absorbed[j] = 1;
        }
    }
    for (size_t j = 0; j < add.size(); ++j)
        if (!absorbed[j]) acc.push_back(add[j]);
}

// One result record back to the host hit the formatters take.
void hit_from_record(const rmb_results* R, uint64_t k, Hit& h) {
    const rmb_hsp& x = R->hsps[k];
    h.score = x.score;
    h.q_start = x.q_start; h.q_end = x.q_end; h.q_len = x.q_len;
    h.s_start = x.s_start; h.s_end = x.s_end; h.s_len = x.s_len;
    h.oid = x.subject_oid;
    h.strand = (uint8_t)x.strand;
    h.stats.matches = x.matches; h.stats.mismatches = x.mismatches;
    h.stats.query_gaps = x.query_gaps; h.stats.subject_gaps = x.subject_gaps;
    h.stats.transitions = x.transitions; h.stats.transversions = x.transversions;
    h.stats.cpg_sites = x.cpg_sites;
    h.stats.perc_sub = x.perc_sub; h.stats.perc_query_gap = x.perc_query_gap;
    h.stats.perc_db_gap = x.perc_db_gap;
    h.stats.kdiv = x.kdiv; h.stats.cpg_kdiv = x.cpg_kdiv;
    h.evalue = x.evalue; h.bitscore = x.bitscore;
    h.q_seq.assign(R->q_seq + x.seq_off, R->q_seq + x.seq_off + x.aln_len);
    h.s_seq.assign(R->s_seq + x.seq_off, R->s_seq + x.seq_off + x.aln_len);
}

QueriesPtr subset_queries(rmb_ctx& C, const std::vector<const uint8_t*>& ptr, const std::vector<uint32_t>& len) {
    return QueriesPtr(make_queries(&C, (uint32_t)ptr.size(), ptr.data(), len.data()));
}

// One search: single-chunk queries through run_core; queries of 1,999,800 bp or more through the
// reference's multi-chunk pipeline (main.rs:1236-1400): DUST on the whole query with the chunked
// off-by-one, Phase 1 + 2a per chunk (engine.rs:1775-1848), the cross-chunk merge per subject in
// chunk order, then Phase 2b against the full query (engine.rs:1418-1431).
void run_search(rmb_ctx& C, rmb_queries& QH, std::vector<std::vector<Hit>>& out_hits, rmb_counters& ctr,
                Taps* taps) {
    const rmb_params& P = C.p;
    const uint32_t nq = QH.n, ns = (uint32_t)C.ids.size();
    std::vector<uint32_t> longq, shortq;
    for (uint32_t i = 0; i < nq; ++i) (query_chunks(QH.len[i], P.word_size).size() > 1 ? longq : shortq).push_back(i);
    if (longq.empty()) {
        run_core(C, QH, out_hits, ctr, taps, nullptr, nullptr);
        return;
    }
    if (taps) throw Fail(RMB_EINVAL, "stage taps take single-chunk queries (under 1,999,800 bp) only");
    for (uint32_t i : longq)
        if (QH.len[i] > 0x7fffffffu) throw Fail(RMB_ELIMIT, "queries of 2^31 bp or more are not supported");
    out_hits.assign(nq, {});
    auto hostq = [&](uint32_t i) { return (const uint8_t*)QH.host.data() + QH.off[i]; };
    if (!shortq.empty()) {
        std::vector<const uint8_t*> ptr;
        std::vector<uint32_t> len;
        for (uint32_t i : shortq) { ptr.push_back(hostq(i)); len.push_back(QH.len[i]); }
        QueriesPtr QS = subset_queries(C, ptr, len);
        std::vector<std::vector<Hit>> hs;
        run_core(C, *QS, hs, ctr, nullptr, nullptr, nullptr);
        for (size_t k = 0; k < shortq.size(); ++k) out_hits[shortq[k]] = std::move(hs[k]);
    }
    // the long queries in full, DUST-masked as one piece
    std::vector<const uint8_t*> lptr;
    std::vector<uint32_t> llen;
    for (uint32_t i : longq) { lptr.push_back(hostq(i)); llen.push_back(QH.len[i]); }
    QueriesPtr QL = subset_queries(C, lptr, llen);
    const uint32_t nl = QL->n;
    std::vector<uint8_t> lmask(QL->host.begin(), QL->host.end());
    if (P.dust) {
        mask_queries(C, *QL, true, ctr);
        CK(cudaMemcpy(lmask.data(), QL->d_qm.p, lmask.size(), cudaMemcpyDeviceToHost));
    }
    // their chunks as queries of their own: unmasked bytes for the extensions, masked bytes for the
    // tables and the exact word extension; the ungapped cutoff of the whole query
    const uint64_t avg = ns ? C.total_letters / ns : 0;
    std::vector<std::vector<uint8_t>> cbytes, cmask;
    std::vector<uint32_t> cparent, cstart, clen;
    std::vector<int32_t> cucut;
    for (uint32_t j = 0; j < nl; ++j) {
        const uint8_t* q = QL->host.data() + QL->off[j];
        const uint8_t* qm = lmask.data() + QL->off[j];
        const uint32_t qa = QL->len[j];
        const int32_t uc = P.ungapped_cutoff >= 0 ? P.ungapped_cutoff
                                                  : ungapped_cutoff_for(C.matrix_name, P.gap_open, P.gap_extend,
                                                                        P.min_raw_gapped_score, qa, avg);
        for (auto [b, e] : query_chunks(qa, P.word_size)) {
            std::vector<uint8_t> c, m;
            c.push_back(q[0]);
            c.insert(c.end(), q + 1 + b, q + 1 + e);
            c.push_back(q[qa + 1]);
            m.push_back(qm[0]);
            m.insert(m.end(), qm + 1 + b, qm + 1 + e);
            m.push_back(qm[qa + 1]);
            cbytes.push_back(std::move(c));
            cmask.push_back(std::move(m));
            cparent.push_back(j);
            cstart.push_back(b);
            clen.push_back(e - b);
            cucut.push_back(uc);
        }
    }
    std::vector<const uint8_t*> cptr;
    for (auto& c : cbytes) cptr.push_back(c.data());
    QueriesPtr CH = subset_queries(C, cptr, clen);
    if (P.dust) {
        std::vector<uint8_t> hm(CH->host.size());
        for (size_t k = 0; k < cmask.size(); ++k) memcpy(hm.data() + CH->off[k], cmask[k].data(), cmask[k].size());
        CH->d_qm.ensure(hm.size());
        CH->d_qmrc.ensure(hm.size());
        CK(cudaMemcpy(CH->d_qm.p, hm.data(), hm.size(), cudaMemcpyHostToDevice));
        CK(launch_revcomp(CH->d_qm.as<uint8_t>(), CH->d_off.as<uint64_t>(), CH->d_len.as<uint32_t>(), CH->n,
                          CH->d_qmrc.as<uint8_t>(), C.st));
        CK(cudaStreamSynchronize(C.st));
        ctr.launches += 1;
        CH->dusted = true;
    }
    std::vector<PairPrelims> col;
    std::vector<std::vector<Hit>> unused;
    run_core(C, *CH, unused, ctr, nullptr, &cucut, &col);
    // the merge, per (query, subject) in chunk order; prelims to full-query coordinates
    auto t0 = std::chrono::steady_clock::now();
    std::vector<std::vector<size_t>> by_pair((size_t)nl * ns);
    for (size_t k = 0; k < col.size(); ++k) by_pair[(size_t)cparent[col[k].q] * ns + col[k].s].push_back(k);
    std::vector<uint32_t> pair_ids;
    std::vector<std::vector<Prelim>> prelims;
    for (size_t pr = 0; pr < by_pair.size(); ++pr) {
        auto& ks = by_pair[pr];
        if (ks.empty()) continue;
        std::stable_sort(ks.begin(), ks.end(), [&](size_t a, size_t b) { return col[a].q < col[b].q; });
        std::vector<Prelim> acc;
        bool first = true;
        for (size_t k : ks) {
            const uint32_t b = cstart[col[k].q];
            for (Prelim& h : col[k].p) {
                h.q_start += b;
                h.q_end += b;
                h.q_seed += b;
            }
            // a chunk with no prelims for this pair leaves the accumulated list as it is
            if (first && b == 0) acc = std::move(col[k].p);
            else merge_chunk_prelims(acc, col[k].p, b);
            first = false;
        }
        if (acc.empty()) continue;
        const uint32_t qa = QL->len[pr / ns], sa = C.slen[pr % ns];
        sort_prelims_for_traceback(acc, qa, sa);
        pair_ids.push_back((uint32_t)pr);
        prelims.push_back(std::move(acc));
    }
    ctr.ms_host_2a += ms_since(t0);
    // Phase 2b on the full queries
    DevQueries Q{QL->d_q.as<uint8_t>(), QL->d_qrc.as<uint8_t>(), QL->d_q.as<uint8_t>(), QL->d_qrc.as<uint8_t>(),
                 QL->d_off.as<uint64_t>(), QL->d_len.as<uint32_t>(), nullptr, nullptr, nullptr, nullptr, nullptr,
                 nullptr, nullptr, nl};
    std::vector<std::vector<Hit>> lh(nl);
    auto qhost = [&](uint32_t j) { return (const uint8_t*)QL->host.data() + QL->off[j]; };
    traceback_2b(C, C.work[0], Q, QL->len.data(), nl, qhost, pair_ids, prelims, lh.data(), ctr, nullptr);
    t0 = std::chrono::steady_clock::now();
    for (uint32_t j = 0; j < nl; ++j) {
        finish_query(C, lh[j], QL->len[j]);
        ctr.finals += lh[j].size();
        out_hits[longq[j]] = std::move(lh[j]);
    }
    ctr.ms_host_2b += ms_since(t0);
}

}  // namespace

extern "C" {

static rmb_results* pack_results(const std::vector<std::vector<Hit>>& hits, const rmb_counters& ctr) {
    const uint32_t nq = (uint32_t)hits.size();
    uint64_t nh = 0, nops = 0, nseq = 0;
    for (auto& v : hits)
        for (auto& h : v) {
            ++nh;
            nops += h.script.size();
            nseq += h.q_seq.size();
        }
    rmb_results* R = (rmb_results*)calloc(1, sizeof(rmb_results));
    if (!R) throw std::bad_alloc();
    R->n_queries = nq;
    R->query_off = (uint64_t*)malloc((nq + 1) * sizeof(uint64_t));
    R->hsps = (rmb_hsp*)malloc(std::max<uint64_t>(nh, 1) * sizeof(rmb_hsp));
    R->ops = (uint32_t*)malloc(std::max<uint64_t>(nops, 1) * 4);
    R->q_seq = (uint8_t*)malloc(std::max<uint64_t>(nseq, 1));
    R->s_seq = (uint8_t*)malloc(std::max<uint64_t>(nseq, 1));
    if (!R->query_off || !R->hsps || !R->ops || !R->q_seq || !R->s_seq) {
        rmb_results_free(R);
        throw std::bad_alloc();
    }
    R->n_hsps = nh;
    uint64_t k = 0, o = 0, s = 0;
    for (uint32_t qi = 0; qi < nq; ++qi) {
        R->query_off[qi] = k;
        for (auto& h : hits[qi]) {
            rmb_hsp& x = R->hsps[k++];
            x.score = h.score;
            x.q_start = h.q_start; x.q_end = h.q_end; x.q_len = h.q_len;
            x.s_start = h.s_start; x.s_end = h.s_end; x.s_len = h.s_len;
            x.subject_oid = h.oid;
            x.strand = h.strand;
            x.matches = h.stats.matches; x.mismatches = h.stats.mismatches;
            x.query_gaps = h.stats.query_gaps; x.subject_gaps = h.stats.subject_gaps;
            x.transitions = h.stats.transitions; x.transversions = h.stats.transversions;
            x.cpg_sites = h.stats.cpg_sites;
            x.perc_sub = h.stats.perc_sub; x.perc_query_gap = h.stats.perc_query_gap;
            x.perc_db_gap = h.stats.perc_db_gap;
            x.kdiv = h.stats.kdiv; x.cpg_kdiv = h.stats.cpg_kdiv;
            x.evalue = h.evalue; x.bitscore = h.bitscore;
            x.ops_off = o;
            x.ops_len = (uint32_t)h.script.size();
            for (auto& r : h.script) R->ops[o++] = ((uint32_t)r.op << 30) | r.n;
            x.seq_off = s;
            x.aln_len = (uint32_t)h.q_seq.size();
            memcpy(R->q_seq + s, h.q_seq.data(), h.q_seq.size());
            memcpy(R->s_seq + s, h.s_seq.data(), h.s_seq.size());
            s += h.q_seq.size();
        }
    }
    R->query_off[nq] = k;
    R->counters = ctr;
    return R;
}

int rmb_queries_upload(rmb_ctx* C, uint32_t nq, const uint8_t* const* query, const uint32_t* qlen,
                       rmb_queries** out, char* err, size_t errlen) {
    try {
        if (!C || !out) throw Fail(RMB_EINVAL, "null argument");
        CK(cudaSetDevice(C->p.device));
        *out = make_queries(C, nq, query, qlen);
        return RMB_OK;
    } catch (const Fail& e) {
        return fail_out(e, err, errlen, e.code);
    } catch (const std::bad_alloc& e) {
        return fail_out(e, err, errlen, RMB_ENOMEM);
    } catch (const std::exception& e) {
        return fail_out(e, err, errlen, RMB_EINVAL);
    }
}

int rmb_search_resident(rmb_ctx* C, rmb_queries* H, rmb_results** out, char* err, size_t errlen) {
    try {
        if (!C || !H || !out) throw Fail(RMB_EINVAL, "null argument");
        if (!C->loaded) throw Fail(RMB_ESTATE, "rmb_db_load must come before the search");
        if (H->device != C->p.device) throw Fail(RMB_EINVAL, "queries were uploaded to another device");
        if (C->p.schedule >= 1 && !C->sched_ready)
            throw Fail(RMB_ESTATE, "schedule 1 needs the network: call rmb_sched_set_model first");
        CK(cudaSetDevice(C->p.device));
        std::vector<std::vector<Hit>> hits;
        rmb_counters ctr{};
        run_search(*C, *H, hits, ctr, nullptr);
        *out = pack_results(hits, ctr);
        return RMB_OK;
    } catch (const Fail& e) {
        return fail_out(e, err, errlen, e.code);
    } catch (const std::bad_alloc& e) {
        return fail_out(e, err, errlen, RMB_ENOMEM);
    } catch (const std::exception& e) {
        return fail_out(e, err, errlen, RMB_EINVAL);
    }
}

void rmb_queries_free(rmb_queries* H) {
    if (!H) return;
    cudaSetDevice(H->device);
    H->release();
    delete H;
}

int rmb_search_batch(rmb_ctx* C, uint32_t nq, const uint8_t* const* query, const uint32_t* qlen, rmb_results** out,
                     char* err, size_t errlen) {
    // the context's own query set: device and pinned host buffers kept from call to call
    try {
        if (!C || !out) throw Fail(RMB_EINVAL, "null argument");
        CK(cudaSetDevice(C->p.device));
        if (!C->batch) C->batch = new rmb_queries();
        make_queries(C, nq, query, qlen, C->batch);
    } catch (const Fail& e) {
        return fail_out(e, err, errlen, e.code);
    } catch (const std::bad_alloc& e) {
        return fail_out(e, err, errlen, RMB_ENOMEM);
    } catch (const std::exception& e) {
        return fail_out(e, err, errlen, RMB_EINVAL);
    }
    return rmb_search_resident(C, C->batch, out, err, errlen);
}

static void check_tune(const rmb_tune& t) {
    if (t.prelim_group != 4 && t.prelim_group != 8 && t.prelim_group != 16)
        throw Fail(RMB_EINVAL, "prelim_group must be 4, 8 or 16");
    if (t.prelim_blocks_per_sm < 1 || t.prelim_blocks_per_sm > 6) throw Fail(RMB_EINVAL, "prelim_blocks_per_sm: 1..6");
    if (t.prelim_window < 16 || t.prelim_window > 60) throw Fail(RMB_EINVAL, "prelim_window: 16..60");
    if (t.prelim_budget_div < 16 || t.prelim_budget_div > 4096) throw Fail(RMB_EINVAL, "prelim_budget_div: 16..4096");
    if (t.ungapped_blocks_per_sm < 1 || t.ungapped_blocks_per_sm > 8)
        throw Fail(RMB_EINVAL, "ungapped_blocks_per_sm: 1..8");
    if (t.lanes < 1 || t.lanes > 2) throw Fail(RMB_EINVAL, "lanes: 1 or 2");
    if (t.graph < 0 || t.graph > 2) throw Fail(RMB_EINVAL, "graph: 0, 1 or 2");
}

int rmb_tune_get(const rmb_ctx* C, rmb_tune* out) {
    if (!C || !out) return RMB_EINVAL;
    *out = C->tune;
    return RMB_OK;
}

int rmb_tune_set(rmb_ctx* C, const rmb_tune* t, char* err, size_t errlen) {
    try {
        if (!C || !t) throw Fail(RMB_EINVAL, "null argument");
        check_tune(*t);
        C->tune = *t;
        return RMB_OK;
    } catch (const Fail& e) {
        return fail_out(e, err, errlen, e.code);
    }
}

// Coordinate descent over the knobs: the defaults, then each knob's alternatives with the others
// at the best so far.  Each candidate runs the sample search twice; its time is the faster run's
// device time in the stages the knobs shape (ungapped extension, dedup, prelim DP).
int rmb_autotune(rmb_ctx* C, uint32_t nq, const uint8_t* const* query, const uint32_t* qlen, rmb_tune* best,
                 double* best_ms, double* default_ms, char* err, size_t errlen) {
    try {
        if (!C || !best) throw Fail(RMB_EINVAL, "null argument");
        if (!C->loaded) throw Fail(RMB_ESTATE, "rmb_db_load must come before rmb_autotune");
        if (C->p.pipeline == 1) throw Fail(RMB_EINVAL, "the plain pipeline has no tuned knobs");
        if (C->p.schedule >= 1 && !C->sched_ready)
            throw Fail(RMB_ESTATE, "schedule 1 needs the network: call rmb_sched_set_model first");
        CK(cudaSetDevice(C->p.device));
        QueriesPtr H(make_queries(C, nq, query, qlen));
        const rmb_tune keep = C->tune;
        // candidates run on one lane: two lanes' kernels overlap and blur each kernel's time
        auto time_of = [&](const rmb_tune& t) {
            C->tune = t;
            C->tune.lanes = 1;
            double ms = 1e300;
            for (int rep = 0; rep < 2; ++rep) {
                std::vector<std::vector<Hit>> hits;
                rmb_counters ctr{};
                run_search(*C, *H, hits, ctr, nullptr);
                ms = std::min(ms, ctr.gpu_ms_ungapped + ctr.gpu_ms_dedup + ctr.gpu_ms_prelim);
            }
            return ms;
        };
        try {
            rmb_tune cur = default_tune();
            {  // grow the device buffers before anything is timed
                std::vector<std::vector<Hit>> hits;
                rmb_counters ctr{};
                C->tune = cur;
                run_search(*C, *H, hits, ctr, nullptr);
            }
            const double d_ms = time_of(cur);
            double cur_ms = d_ms;
            auto knob = [&](int32_t rmb_tune::*field, std::initializer_list<int32_t> alts) {
                for (int32_t v : alts) {
                    if (cur.*field == v) continue;
                    rmb_tune t = cur;
                    t.*field = v;
                    const double ms = time_of(t);
                    if (ms < cur_ms) {
                        cur_ms = ms;
                        cur = t;
                    }
                }
            };
            knob(&rmb_tune::prelim_group, {4, 16});
            knob(&rmb_tune::prelim_blocks_per_sm, {4, 5});
            knob(&rmb_tune::prelim_window, {32, 48});
            knob(&rmb_tune::prelim_budget_div, {32, 512});
            knob(&rmb_tune::ungapped_blocks_per_sm, {4, 6});
            knob(&rmb_tune::dedup_extend_hits_per_pair, {0, -1});
            C->tune = cur;
            *best = cur;
            if (best_ms) *best_ms = cur_ms;
            if (default_ms) *default_ms = d_ms;
        } catch (...) {
            C->tune = keep;
            throw;
        }
        return RMB_OK;
    } catch (const Fail& e) {
        return fail_out(e, err, errlen, e.code);
    } catch (const std::bad_alloc& e) {
        return fail_out(e, err, errlen, RMB_ENOMEM);
    } catch (const std::exception& e) {
        return fail_out(e, err, errlen, RMB_EINVAL);
    }
}

int rmb_sched_set_model(rmb_ctx* C, const float* params, uint32_t n_params, char* err, size_t errlen) {
    try {
        if (!C || !params) throw Fail(RMB_EINVAL, "null argument");
        if (n_params != RMB_SCHED_NPARAM)
            throw Fail(RMB_EINVAL, "the schedule network takes " + std::to_string(RMB_SCHED_NPARAM) + " parameters");
        for (uint32_t i = 0; i < n_params; ++i)
            if (!std::isfinite(params[i])) throw Fail(RMB_EINVAL, "schedule network parameters must be finite");
        CK(cudaSetDevice(C->p.device));
        C->sched_params.ensure(n_params * 4);
        CK(cudaMemcpy(C->sched_params.p, params, n_params * 4, cudaMemcpyHostToDevice));
        C->sched_ready = true;
        return RMB_OK;
    } catch (const Fail& e) {
        return fail_out(e, err, errlen, e.code);
    } catch (const std::exception& e) {
        return fail_out(e, err, errlen, RMB_EINVAL);
    }
}

int rmb_sched_log(rmb_ctx* C, uint32_t nq, const uint8_t* const* query, const uint32_t* qlen, float** features,
                  uint32_t** cells, uint64_t* n_records, char* err, size_t errlen) {
    rmb_ctx::SchedLog log;
    try {
        if (!C || !features || !cells || !n_records) throw Fail(RMB_EINVAL, "null argument");
        if (!C->loaded) throw Fail(RMB_ESTATE, "rmb_db_load must come before rmb_sched_log");
        if (!C->prelim_stream) throw Fail(RMB_EINVAL, "cell logging needs the thread-per-extension prelim kernel");
        CK(cudaSetDevice(C->p.device));
        std::unique_ptr<rmb_queries, void (*)(rmb_queries*)> H(make_queries(C, nq, query, qlen), rmb_queries_free);
        std::vector<std::vector<Hit>> hits;
        rmb_counters ctr{};
        C->sched_log = &log;
        run_search(*C, *H, hits, ctr, nullptr);
        C->sched_log = nullptr;
        const uint64_t n = log.cells.size();
        float* f = (float*)malloc(std::max<uint64_t>(n, 1) * SCHED_NF_HOST * 4);
        uint32_t* c = (uint32_t*)malloc(std::max<uint64_t>(n, 1) * 4);
        if (!f || !c) {
            free(f);
            free(c);
            throw std::bad_alloc();
        }
        if (n) {
            memcpy(f, log.feats.data(), n * SCHED_NF_HOST * 4);
            memcpy(c, log.cells.data(), n * 4);
        }
        *features = f;
        *cells = c;
        *n_records = n;
        return RMB_OK;
    } catch (const Fail& e) {
        if (C) C->sched_log = nullptr;
        return fail_out(e, err, errlen, e.code);
    } catch (const std::bad_alloc& e) {
        if (C) C->sched_log = nullptr;
        return fail_out(e, err, errlen, RMB_ENOMEM);
    } catch (const std::exception& e) {
        if (C) C->sched_log = nullptr;
        return fail_out(e, err, errlen, RMB_EINVAL);
    }
}

int rmb_debug_stage(rmb_ctx* C, uint32_t nq, const uint8_t* const* query, const uint32_t* qlen, int32_t stage,
                    uint32_t** records, uint64_t* n_records, char* err, size_t errlen) {
    try {
        if (!C || !records || !n_records) throw Fail(RMB_EINVAL, "null argument");
        if (!C->loaded) throw Fail(RMB_ESTATE, "rmb_db_load must come before rmb_debug_stage");
        if (stage < 0 || stage > 4) throw Fail(RMB_EINVAL, "stage must be 0..4");
        CK(cudaSetDevice(C->p.device));
        std::unique_ptr<rmb_queries, void (*)(rmb_queries*)> H(make_queries(C, nq, query, qlen), rmb_queries_free);
        std::vector<uint32_t> v;
        Taps t;
        if (stage == 0) t.seeds = &v;
        else if (stage == 1) t.ungapped = &v;
        else if (stage == 2) t.prelims = &v;
        else if (stage == 3) t.lookup = &v;
        else t.tracebacks = &v;
        std::vector<std::vector<Hit>> hits;
        rmb_counters ctr{};
        run_search(*C, *H, hits, ctr, &t);
        const uint64_t width = stage == 0 ? 3 : stage == 1 ? 6 : stage == 2 ? 8 : stage == 3 ? 3 : 9;
        uint32_t* r = (uint32_t*)malloc(std::max<size_t>(v.size(), 1) * 4);
        if (!r) throw std::bad_alloc();
        if (!v.empty()) memcpy(r, v.data(), v.size() * 4);
        *records = r;
        *n_records = v.size() / width;
        return RMB_OK;
    } catch (const Fail& e) {
        return fail_out(e, err, errlen, e.code);
    } catch (const std::bad_alloc& e) {
        return fail_out(e, err, errlen, RMB_ENOMEM);
    } catch (const std::exception& e) {
        return fail_out(e, err, errlen, RMB_EINVAL);
    }
}

int rmb_format_pairwise(rmb_ctx* C, const rmb_results* R, const uint8_t* const* query, const uint32_t* qlen,
                        const char* const* query_deflines, const char* const* subject_deflines,
                        const char* db_name, int64_t db_mtime, int32_t parts, char** text, size_t* text_len, char* err,
                        size_t errlen) {
    try {
        if (!C || !R || !text || !db_name) throw Fail(RMB_EINVAL, "null argument");
        if (R->n_queries && (!query_deflines || !qlen)) throw Fail(RMB_EINVAL, "query deflines and lengths are needed");
        CK(cudaSetDevice(C->p.device));
        // the query's DUST intervals print in lower case (main.rs:948-956): the device masker's
        // interval bitmap over the plain (single-chunk) intervals
        std::vector<uint32_t> bits;
        std::vector<uint64_t> bits_off(R->n_queries + 1, 0);
        if (C->p.dust && R->n_queries) {
            if (!query) throw Fail(RMB_EINVAL, "with dust on, the query sequences are needed");
            QueriesPtr QH(make_queries(C, R->n_queries, query, qlen));
            for (uint32_t i = 0; i < R->n_queries; ++i) bits_off[i + 1] = bits_off[i] + (qlen[i] + 31) / 32;
            DBuf d_bits, d_off;
            d_bits.ensure(std::max<uint64_t>(bits_off.back(), 1) * 4);
            upload(d_off, bits_off, C->st);
            CK(cudaMemsetAsync(d_bits.p, 0, std::max<uint64_t>(bits_off.back(), 1) * 4, C->st));
            const uint32_t nt = dust_threads(R->n_queries, C->sms);
            C->dust_scratch.ensure(dust_scratch_bytes(nt));
            C->fails.ensure(16);
            CK(cudaMemsetAsync(C->fails.p, 0, 4, C->st));
            CK(launch_dust(QH->d_q.as<uint8_t>(), QH->d_off.as<uint64_t>(), QH->d_len.as<uint32_t>(), R->n_queries,
                           nullptr, C->dust_scratch.p, nt, C->fails.as<unsigned int>(), false, C->st,
                           d_bits.as<uint32_t>(), d_off.as<uint64_t>()));
            bits.resize(std::max<uint64_t>(bits_off.back(), 1));
            unsigned int over = 0;
            CK(cudaMemcpyAsync(bits.data(), d_bits.p, bits.size() * 4, cudaMemcpyDeviceToHost, C->st));
            CK(cudaMemcpyAsync(&over, C->fails.p, 4, cudaMemcpyDeviceToHost, C->st));
            CK(cudaStreamSynchronize(C->st));
            d_bits.release();
            d_off.release();
            if (over) throw Fail(RMB_ELIMIT, "DUST interval list outgrew its fixed capacity");
        }
        std::string out;
        if (parts & 1) out += pairwise_header(db_name, C->ids.size(), C->total_letters);
        std::vector<Hit> hits;
        for (uint32_t qi = 0; qi < R->n_queries; ++qi) {
            hits.clear();
            for (uint64_t k = R->query_off[qi]; k < R->query_off[qi + 1]; ++k) {
                hits.emplace_back();
                hit_from_record(R, k, hits.back());
            }
            pairwise_query(out, hits, query_deflines[qi], qlen[qi], C->ids, subject_deflines,
                           bits.empty() ? nullptr : bits.data() + bits_off[qi]);
        }
        if (parts & 2)
            out += pairwise_footer(db_name, C->ids.size(), C->total_letters, db_mtime, C->p.gap_open, C->p.gap_extend);
        char* o = (char*)malloc(out.size() + 1);
        if (!o) throw std::bad_alloc();
        memcpy(o, out.data(), out.size());
        o[out.size()] = 0;
        *text = o;
        if (text_len) *text_len = out.size();
        return RMB_OK;
    } catch (const Fail& e) {
        return fail_out(e, err, errlen, e.code);
    } catch (const std::bad_alloc& e) {
        return fail_out(e, err, errlen, RMB_ENOMEM);
    } catch (const std::exception& e) {
        return fail_out(e, err, errlen, RMB_EINVAL);
    }
}

int rmb_format_tabular(const rmb_ctx* C, const rmb_results* R, const char* const* query_ids, const char* outfmt,
                       char** text, size_t* text_len, char* err, size_t errlen) {
    try {
        if (!C || !R || !outfmt || !text) throw Fail(RMB_EINVAL, "null argument");
        std::istringstream is(outfmt);
        std::string t;
        std::vector<std::string> fields;
        is >> t;
        if (t != "6") throw Fail(RMB_EINVAL, "output format '" + t + "' is not supported; use 6 <fields>");
        while (is >> t) fields.push_back(t);
        if (fields.empty()) throw Fail(RMB_EINVAL, "-outfmt 6 needs a field list");
        // queries formatted in parallel, each into its own string, then joined in query order
        for (uint32_t qi = 0; qi < R->n_queries; ++qi)
            for (uint64_t k = R->query_off[qi]; k < R->query_off[qi + 1]; ++k)
                if (R->hsps[k].subject_oid >= C->ids.size()) throw Fail(RMB_EINVAL, "HSP subject out of range");
        std::vector<std::string> parts(R->n_queries);
        std::atomic<bool> unknown{false};
        parallel_for(R->n_queries, [&](size_t qi) {
            const std::string qid = query_ids ? query_ids[qi] : ("query" + std::to_string(qi));
            std::string& o = parts[qi];
            Hit h;
            for (uint64_t k = R->query_off[qi]; k < R->query_off[qi + 1] && !unknown; ++k) {
                hit_from_record(R, k, h);
                if (!format_line(o, h, qid, C->ids[R->hsps[k].subject_oid], fields)) unknown = true;
                o.push_back('\n');
            }
        });
        if (unknown) throw Fail(RMB_EINVAL, "unknown -outfmt field");
        size_t total = 0;
        for (const auto& x : parts) total += x.size();
        std::string out;
        out.reserve(total);
        for (const auto& x : parts) out += x;
        char* o = (char*)malloc(out.size() + 1);
        if (!o) throw std::bad_alloc();
        memcpy(o, out.data(), out.size());
        o[out.size()] = 0;
        *text = o;
        if (text_len) *text_len = out.size();
        return RMB_OK;
    } catch (const Fail& e) {
        return fail_out(e, err, errlen, e.code);
    } catch (const std::exception& e) {
        return fail_out(e, err, errlen, RMB_EINVAL);
    }
}

void rmb_results_free(rmb_results* R) {
    if (!R) return;
    free(R->query_off);
    free(R->hsps);
    free(R->ops);
    free(R->q_seq);
    free(R->s_seq);
    free(R);
}

void rmb_text_free(void* p) { free(p); }

void rmb_ctx_destroy(rmb_ctx* C) {
    if (!C) return;
    cudaSetDevice(C->p.device);
    DBuf* all[] = {&C->d_plus, &C->d_rc, &C->d_align, &C->d_align_rc, &C->d_packed, &C->d_plus_off, &C->d_packed_off,
                   &C->d_len, &C->d_params, &C->lw, &C->dust_scratch, &C->fails, &C->sched_params};
    for (DBuf* b : all) b->release();
    for (Work& w : C->work) w.release();
    if (C->batch) {
        C->batch->release();
        delete C->batch;
    }
    if (C->st) cudaStreamDestroy(C->st);
    delete C;
}

}  // extern "C"
