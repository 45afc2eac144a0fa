// sw_batch.cu -- batched search: many queries against the resident DB in one
// pass over the device, captured as a CUDA graph.
//
// The reference has no batched mode: WorkerPool searches one query per run
// and balances DB chunks across worker threads on the host
// (src/WorkerPool.cpp:10-82, src/DataPool.cpp:171-286).  Here a batch is:
//   * queries shorter than the stack height packed (first fit, longest first)
//     into "stacks": one virtual query whose R-row blocks belong to different
//     queries, so short queries fill the rows a single one would leave as
//     padding and share every column step; longer queries form stacks of their
//     own, bucketed by the kernel shape the tuning table picks for them;
//   * per bucket, one persistent launch of sw_batch<T,R> over its stacks
//     (blocks walk the stacks in order, groups claim record pairs from one
//     device counter per stack), plus, when a cut-over is set, a concurrent
//     launch of single-group blocks for the pairs longer than the cut-over, so
//     their inherently serial column steps overlap the bulk;
//   * one 32-bit re-score launch for every flagged (query, record) and one
//     top-k round sequence with a grid row per query.
// The whole sequence (query upload, launches, result download) is captured
// once per batch signature and replayed.
#include <algorithm>
#include <array>
#include <chrono>
#include <cstring>
#include <map>
#include <numeric>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/swb200.h"
#include "sw_aux.h"
#include "sw_device.cuh"
#include "sw_engine.h"
#include "sw_qpair.cuh"
#include "sw_registry.h"

using namespace swb;

struct BatchLaunch {
    const QpKernel* qk = nullptr;   // set: a paired-query launch over double stacks
    const WfKernel* k;
    int grid, threads;
    size_t smem;
    int sbegin, scount;        // stacks of this launch
    int pair_begin, pair_count;
    int counter_base;          // first counter of this launch
    bool long_part;            // runs on the side stream
    size_t bnd_group;
    int long_units = 0;        // paired: units of the long phase (QpArgs::long_units)
};

// Host image of a batch's stacks (uploaded as one block, see enqueue_batch).
struct StackPlan {
    std::vector<uint8_t> codes;           // stack rows (and the paired lanes' rows)
    std::vector<uint32_t> off, rows, rb_off;
    std::vector<int32_t> rb_map;
    // double stacks of the paired-query kernel: per double stack the two lanes'
    // codes offset and rows, and per (pass, thread) the (low, high) block map
    std::vector<uint32_t> qp_off_lo, qp_rows_lo, qp_off_hi, qp_rows_hi, qp_rb_off, qp_flags;
    std::vector<uint32_t> qp_slot;        // boundary region of each segmented entry
    std::vector<int32_t> qp_rb_map;       // pairs of entries
};

const QpKernel* swb::find_qp(int T, int R) {
    int n = 0;
    const QpKernel* q = qp_kernels(&n);
    for (int i = 0; i < n; ++i)
        if (q[i].T == T && q[i].R == R) return &q[i];
    return nullptr;
}

struct BatchGraph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint32_t launches = 0;
};

struct sw_batch_state {
    sw_batch_options opt{0, 32, 16, 1, 16, 64, 4096, 2048, 16, 64, 1, 0};
    // device
    uint8_t* d_queries = nullptr;
    size_t queries_cap = 0;
    uint8_t* d_meta = nullptr;       // qoff[nq] qlen[nq] | stack codes, off, rows, rb_off, rb_map
    size_t meta_cap = 0;
    int* d_counters = nullptr;       // 2 per query + 1 overflow count
    size_t counters_cap = 0;
    int* d_scores = nullptr;         // [query][sorted position]
    int* d_scores_rec = nullptr;     // [query][record]
    size_t scores_cap = 0;           // queries
    int* d_ovf = nullptr;
    size_t ovf_cap = 0;
    unsigned long long* d_keys[2] = {nullptr, nullptr};
    size_t keys_cap = 0;
    uint2* d_bnd = nullptr;
    size_t bnd_cap = 0;
    // boundary regions of tall paired double stacks whose segments share a
    // launch (one per stack of a wave; 1 = the context's own rows, d_segbnd unused)
    uint2* d_segbnd = nullptr;
    int seg_regions = 1;
    size_t seg_stride = 0;         // entries per region
    // pinned host staging
    uint8_t* h_stage = nullptr;      // queries, then meta
    size_t stage_cap = 0;
    unsigned long long* h_keys = nullptr;
    size_t hkeys_cap = 0;
    std::map<std::vector<uint64_t>, BatchGraph> graphs;
};

namespace swb {

void free_batch(sw_ctx* ctx) {
    sw_batch_state* b = ctx->batch;
    if (!b) return;
    for (auto& kv : b->graphs) {
        if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
        if (kv.second.graph) cudaGraphDestroy(kv.second.graph);
    }
    dev_free(b->d_queries);
    dev_free(b->d_meta);
    dev_free(b->d_counters);
    dev_free(b->d_scores);
    dev_free(b->d_scores_rec);
    dev_free(b->d_ovf);
    dev_free(b->d_keys[0]);
    dev_free(b->d_keys[1]);
    dev_free(b->d_bnd);
    dev_free(b->d_segbnd);
    if (b->h_stage) cudaFreeHost(b->h_stage);
    if (b->h_keys) cudaFreeHost(b->h_keys);
    delete b;
    ctx->batch = nullptr;
}

}  // namespace swb

namespace {

template <typename T>
sw_status grow(sw_ctx* ctx, T** p, size_t& cap, size_t need, const char* what) {
    if (need <= cap) return SW_OK;
    dev_free(*p);
    cap = 0;
    if (dev_alloc(p, need) != cudaSuccess) SW_SET(ctx, SW_ERR_NOMEM, "device allocation failed: %s", what);
    cap = need;
    return SW_OK;
}

double wall_ms() {
    return std::chrono::duration<double, std::milli>(
               std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

// Boundary regions for `want` tall double stacks whose segments share
// launches: at most `want`, as many as fit in a quarter of the free device memory
// (each is a copy of the context's per-record boundary rows, 8 bytes per
// column of every record); 1 means the context's own rows.  Grows (never
// shrinks) the batch state's region buffer; called before any capture.
int seg_regions_for(sw_ctx* ctx, sw_batch_state* b, int want) {
    const size_t stride = (size_t)ctx->db_units * 16;
    if (b->d_segbnd && b->seg_stride != stride) {   // sized for another DB
        for (auto& kv : b->graphs) {
            if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
            if (kv.second.graph) cudaGraphDestroy(kv.second.graph);
        }
        b->graphs.clear();
        dev_free(b->d_segbnd);
        b->d_segbnd = nullptr;
        b->seg_regions = 1;
        b->seg_stride = 0;
    }
    want = std::max(1, want);
    if (want <= 1 || stride == 0) return 1;
    if (b->seg_regions >= want && b->seg_stride == stride) return want;
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
        cudaGetLastError();
        return b->seg_stride == stride ? b->seg_regions : 1;
    }
    const size_t held = b->seg_stride == stride && b->d_segbnd ? (size_t)b->seg_regions : 0;
    const size_t fit = (free_b / 4 + held * stride * sizeof(uint2)) / (stride * sizeof(uint2));
    const int n = (int)std::min<size_t>((size_t)want, fit);
    if (n <= 1) return b->seg_stride == stride && b->d_segbnd ? b->seg_regions : 1;
    for (auto& kv : b->graphs) {      // graphs hold the old pointer
        if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
        if (kv.second.graph) cudaGraphDestroy(kv.second.graph);
    }
    b->graphs.clear();
    dev_free(b->d_segbnd);
    b->seg_regions = 1;
    b->seg_stride = 0;
    if (dev_alloc(&b->d_segbnd, (size_t)n * stride) != cudaSuccess) {
        cudaGetLastError();
        b->d_segbnd = nullptr;
        return 1;
    }
    b->seg_regions = n;
    b->seg_stride = stride;
    return n;
}

// Enqueues one batch on ctx->stream (and the side stream).  Buffers are sized.
// Device layout of d_meta (and of the staging area it is copied from):
//   qoff[nq], qlen[nq]                          uint32
//   stack_off[ns], stack_rows[ns], rb_off[ns]   uint32
//   rb_map[...]                                 int32
//   stack codes                                 uint8
//   qp_off_lo, qp_rows_lo, qp_off_hi, qp_rows_hi, qp_rb_off, qp_flags, qp_slot [nqp]  uint32
//   qp_rb_map[...] (16-byte aligned)            int2
struct MetaLayout {
    size_t qoff, qlen, soff, srows, rboff, rbmap, qp_off_lo, qp_rows_lo, qp_off_hi, qp_rows_hi,
        qp_rboff, qp_flags, qp_slot, qp_rbmap, codes, total;
    int nst, nqp;
};

MetaLayout meta_layout(uint32_t nq, const StackPlan& sp) {
    MetaLayout m;
    const size_t ns = sp.off.size(), nqp = sp.qp_off_lo.size();
    m.nst = (int)ns;
    m.nqp = (int)nqp;
    m.qoff = 0;
    m.qlen = m.qoff + 4 * (size_t)nq;
    m.soff = m.qlen + 4 * (size_t)nq;
    m.srows = m.soff + 4 * ns;
    m.rboff = m.srows + 4 * ns;
    m.rbmap = m.rboff + 4 * ns;
    m.qp_off_lo = m.rbmap + 4 * sp.rb_map.size();
    m.qp_rows_lo = m.qp_off_lo + 4 * nqp;
    m.qp_off_hi = m.qp_rows_lo + 4 * nqp;
    m.qp_rows_hi = m.qp_off_hi + 4 * nqp;
    m.qp_rboff = m.qp_rows_hi + 4 * nqp;
    m.qp_flags = m.qp_rboff + 4 * nqp;
    m.qp_slot = m.qp_flags + 4 * nqp;
    m.qp_rbmap = (m.qp_slot + 4 * nqp + 15) / 16 * 16;
    m.codes = m.qp_rbmap + 4 * sp.qp_rb_map.size();
    m.total = (m.codes + sp.codes.size() + 15) / 16 * 16;
    return m;
}

sw_status enqueue_batch(sw_ctx* ctx, sw_batch_state* b, uint32_t nq, size_t qbytes,
                        const MetaLayout& ml, const std::vector<BatchLaunch>& launches,
                        bool want_scores, uint32_t* n_launch) {
    cudaStream_t st = ctx->stream;
    const int n_rec = (int)ctx->n_records;
    const int k = ctx->params.top_k;
    *n_launch = 0;
    SW_CUDA(ctx, cudaMemcpyAsync(b->d_queries, b->h_stage, qbytes ? qbytes : 1,
                                 cudaMemcpyHostToDevice, st));
    const size_t meta_at = (b->stage_cap - ml.total) & ~(size_t)15;
    SW_CUDA(ctx, cudaMemcpyAsync(b->d_meta, b->h_stage + meta_at, ml.total,
                                 cudaMemcpyHostToDevice, st));
    const int nst = ml.nst;
    SW_CUDA(ctx, cudaMemsetAsync(b->d_counters, 0, (2 * (size_t)nst + 1 + ml.nqp) * sizeof(int),
                                 st));
    SW_CUDA(ctx, cudaMemsetAsync(b->d_scores, 0, (size_t)nq * n_rec * sizeof(int), st));
    const uint32_t* d_qoff = reinterpret_cast<const uint32_t*>(b->d_meta + ml.qoff);
    const uint32_t* d_qlen = reinterpret_cast<const uint32_t*>(b->d_meta + ml.qlen);
    const uint32_t* d_soff = reinterpret_cast<const uint32_t*>(b->d_meta + ml.soff);
    const uint32_t* d_srows = reinterpret_cast<const uint32_t*>(b->d_meta + ml.srows);
    const uint32_t* d_rboff = reinterpret_cast<const uint32_t*>(b->d_meta + ml.rboff);
    const int* d_rbmap = reinterpret_cast<const int*>(b->d_meta + ml.rbmap);
    const uint8_t* d_codes = b->d_meta + ml.codes;
    int* d_ovf_count = b->d_counters + 2 * nst;
    const int ovf_thresh = 32767 - std::max(ctx->max_score, 1) + 1;
    bool forked = false;
    for (const BatchLaunch& L : launches) {
        if (L.qk) {      // paired queries: main stream, the bulk half of the boundary rows
            QpArgs q;
            q.db = ctx->d_db;
            q.pairs = ctx->d_pairs;
            q.pair_begin = 0;
            q.pair_count = (int)ctx->n_pairs;
            q.codes = d_codes;
            q.off_lo = reinterpret_cast<const uint32_t*>(b->d_meta + ml.qp_off_lo) + L.sbegin;
            q.rows_lo = reinterpret_cast<const uint32_t*>(b->d_meta + ml.qp_rows_lo) + L.sbegin;
            q.off_hi = reinterpret_cast<const uint32_t*>(b->d_meta + ml.qp_off_hi) + L.sbegin;
            q.rows_hi = reinterpret_cast<const uint32_t*>(b->d_meta + ml.qp_rows_hi) + L.sbegin;
            q.rb_map = reinterpret_cast<const int2*>(b->d_meta + ml.qp_rbmap);
            q.rb_off = reinterpret_cast<const uint32_t*>(b->d_meta + ml.qp_rboff) + L.sbegin;
            q.nstacks = L.scount;
            q.counters = b->d_counters + L.counter_base;
            q.mat = ctx->d_mat;
            q.bias2 = (uint32_t)(ctx->params.gap_open + ctx->params.gap_extend);
            q.bias2 |= q.bias2 << 16;
            q.neg_e = (uint32_t)(uint16_t)(int16_t)(-ctx->params.gap_extend);
            q.neg_e |= q.neg_e << 16;
            q.bnd = b->d_bnd + b->bnd_cap / 2;
            q.bnd_group = L.bnd_group;
            q.scores = b->d_scores;
            q.n_records = n_rec;
            q.ovf_list = b->d_ovf;
            q.ovf_count = d_ovf_count;
            q.ovf_thresh = ovf_thresh;
            q.ovf_cap = (int)std::min<size_t>(b->ovf_cap, (size_t)INT32_MAX);
            q.pair_ids = nullptr;
            q.seg_flags = reinterpret_cast<const uint32_t*>(b->d_meta + ml.qp_flags) + L.sbegin;
            q.seg_bnd = b->d_segbnd ? b->d_segbnd : ctx->d_bnd;
            q.seg_slot = reinterpret_cast<const uint32_t*>(b->d_meta + ml.qp_slot) + L.sbegin;
            q.seg_stride = b->seg_stride;
            q.long_units = L.long_units;
            void* args[] = {&q};
            SW_CUDA(ctx, cudaLaunchKernel(L.qk->fn, dim3((unsigned)L.grid), dim3(L.threads), args,
                                          L.smem, st));
            ++*n_launch;
            continue;
        }
        BatchArgs a;
        a.db = ctx->d_db;
        a.pairs = ctx->d_pairs;
        a.pair_begin = L.pair_begin;
        a.pair_count = L.pair_count;
        a.codes = d_codes;
        a.stack_off = d_soff + L.sbegin;
        a.stack_rows = d_srows + L.sbegin;
        a.rb_map = d_rbmap;
        a.rb_off = d_rboff + L.sbegin;
        a.nstacks = L.scount;
        a.counters = b->d_counters + L.counter_base;
        a.mat = ctx->d_mat;
        a.bias2 = (uint32_t)(ctx->params.gap_open + ctx->params.gap_extend);
        a.bias2 |= a.bias2 << 16;
        a.neg_e = (uint32_t)(uint16_t)(int16_t)(-ctx->params.gap_extend);
        a.neg_e |= a.neg_e << 16;
        a.bnd = L.long_part ? b->d_bnd : b->d_bnd + b->bnd_cap / 2;
        a.bnd_group = L.bnd_group;
        a.scores = b->d_scores;
        a.n_records = n_rec;
        a.ovf_list = b->d_ovf;
        a.ovf_count = d_ovf_count;
        a.ovf_thresh = ovf_thresh;
        a.ovf_cap = (int)std::min<size_t>(b->ovf_cap, (size_t)INT32_MAX);
        a.pair_ids = nullptr;
        void* args[] = {&a};
        cudaStream_t ls = st;
        if (L.long_part) {
            if (!forked) {
                SW_CUDA(ctx, cudaEventRecord(ctx->fork_ev, st));
                SW_CUDA(ctx, cudaStreamWaitEvent(ctx->side_stream, ctx->fork_ev, 0));
                forked = true;
            }
            ls = ctx->side_stream;
        }
        SW_CUDA(ctx, cudaLaunchKernel(L.k->batch_fn, dim3((unsigned)L.grid), dim3(L.threads), args,
                                      L.smem, ls));
        ++*n_launch;
    }
    if (forked) {
        SW_CUDA(ctx, cudaEventRecord(ctx->join_ev, ctx->side_stream));
        SW_CUDA(ctx, cudaStreamWaitEvent(st, ctx->join_ev, 0));
    }
    {
        RescoreArgs r;
        r.db = ctx->d_db;
        r.pairs = ctx->d_pairs;
        r.query = nullptr;
        r.qlen = 0;
        r.queries = b->d_queries;
        r.qoff = d_qoff;
        r.qlens = d_qlen;
        r.n_records = n_rec;
        r.mat = ctx->d_mat;
        r.gap_oe = ctx->params.gap_open + ctx->params.gap_extend;
        r.gap_e = ctx->params.gap_extend;
        r.ovf_list = b->d_ovf;
        r.ovf_count = d_ovf_count;
        r.ovf_cap = (int)std::min<size_t>(b->ovf_cap, (size_t)INT32_MAX);
        r.scratch = ctx->d_rs_scratch;
        r.max_cols = ctx->max_cols;
        r.scores = b->d_scores;
        void* args[] = {&r};
        SW_CUDA(ctx, cudaLaunchKernel((const void*)sw_rescore32, dim3(kRescoreBlocks), dim3(64),
                                      args, 0, st));
        ++*n_launch;
    }
    const long long nblk0 = std::max<long long>(1, ((long long)n_rec + kTopkKeys - 1) / kTopkKeys);
    long long n = n_rec;
    int buf = 0;
    const unsigned long long* keys_in = nullptr;
    bool first = true;
    long long in_stride = n_rec;
    while (true) {
        const long long blocks = std::max<long long>(1, (n + kTopkKeys - 1) / kTopkKeys);
        TopkArgs t;
        t.scores = b->d_scores;
        t.perm = ctx->d_perm;
        t.keys_in = first ? nullptr : keys_in;
        t.n = n;
        t.k = k;
        t.cap = (ctx->params.flags & SW_FLAG_REFERENCE_CAP) ? 1 : 0;
        t.scores_by_record = (first && want_scores) ? b->d_scores_rec : nullptr;
        t.keys_out = b->d_keys[buf];
        t.in_stride = in_stride;
        t.rec_stride = n_rec;
        t.out_stride = nblk0 * kMaxTopK;
        t.rows = nullptr;
        void* args[] = {&t};
        SW_CUDA(ctx, cudaLaunchKernel((const void*)sw_topk_round, dim3((unsigned)blocks, nq),
                                      dim3(kTopkThreads), args, 0, st));
        ++*n_launch;
        keys_in = b->d_keys[buf];
        in_stride = nblk0 * kMaxTopK;
        buf ^= 1;
        first = false;
        if (blocks == 1) break;
        n = blocks * (long long)k;
    }
    // final keys: row y of the last buffer holds query y's k keys first
    SW_CUDA(ctx, cudaMemcpy2DAsync(b->h_keys, (size_t)k * sizeof(unsigned long long), keys_in,
                                   (size_t)(nblk0 * kMaxTopK) * sizeof(unsigned long long),
                                   (size_t)k * sizeof(unsigned long long), nq,
                                   cudaMemcpyDeviceToHost, st));
    return SW_OK;
}

}  // namespace

extern "C" sw_status sw_set_batch_options(sw_ctx* ctx, const sw_batch_options* opt) {
    if (!ctx) return SW_ERR_INVALID;
    if (!ctx->batch) ctx->batch = new sw_batch_state();
    if (opt) {
        if (opt->cutover < 0 || !find_kernel(opt->long_group_width, opt->long_rows_per_thread) ||
            !find_kernel(opt->group_width, opt->rows_per_thread) || opt->stack_rows < 0 ||
            opt->pair_rows < 0 || opt->pair_regions < 0 ||
            (opt->pair_rows > 0 && !find_qp(opt->pair_group_width, opt->pair_rows_per_thread)))
            SW_SET(ctx, SW_ERR_INVALID, "bad batch options");
        ctx->batch->opt = *opt;
    } else {
        ctx->batch->opt = sw_batch_options{0, 32, 16, 1, 16, 64, 4096, 2048, 16, 64, 1, 0};
    }
    for (auto& kv : ctx->batch->graphs) {
        if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
        if (kv.second.graph) cudaGraphDestroy(kv.second.graph);
    }
    ctx->batch->graphs.clear();
    return SW_OK;
}

extern "C" sw_status sw_search_batch(sw_ctx* ctx, uint32_t nq, const uint8_t* queries,
                                     const uint64_t* qoffsets, sw_hit* hits, uint32_t* n_hits,
                                     int32_t* scores) {
    if (!ctx) return SW_ERR_INVALID;
    if (ctx->serve) return SW_ERR_BUSY;   // the serving loop owns the stream
    if (!ctx->db_loaded) SW_SET(ctx, SW_ERR_STATE, "no DB loaded (call sw_db_load first)");
    if (nq == 0) return SW_OK;
    if (!qoffsets || !hits || !n_hits) SW_SET(ctx, SW_ERR_INVALID, "null argument");
    const double t0 = wall_ms();
    const int k = ctx->params.top_k;
    const int n_rec = (int)ctx->n_records;
    if ((uint64_t)nq * (uint64_t)std::max(n_rec, 1) >= (1ull << 31))
        SW_SET(ctx, SW_ERR_UNSUPPORTED, "batch too large: %u queries x %d records", nq, n_rec);
    for (uint32_t i = 0; i < nq; ++i) {
        if (qoffsets[i + 1] < qoffsets[i]) SW_SET(ctx, SW_ERR_INVALID, "query offsets not monotone");
        if (qoffsets[i + 1] - qoffsets[i] > kMaxQueryResidues)
            SW_SET(ctx, SW_ERR_UNSUPPORTED, "query %u: %llu residues (at most %u)", i,
                   (unsigned long long)(qoffsets[i + 1] - qoffsets[i]), kMaxQueryResidues);
    }
    const uint64_t qbytes = qoffsets[nq] - qoffsets[0];
    if (qbytes && !queries) SW_SET(ctx, SW_ERR_INVALID, "null queries");
    for (uint64_t i = 0; i < qbytes; ++i)
        if (queries[qoffsets[0] + i] > 24)
            SW_SET(ctx, SW_ERR_INVALID, "query code %d", queries[qoffsets[0] + i]);
    for (uint32_t i = 0; i < nq * (uint32_t)k; ++i) hits[i] = sw_hit{0, 0, 0};
    for (uint32_t i = 0; i < nq; ++i) n_hits[i] = 0;
    ctx->stats = sw_run_stats{};
    if (n_rec == 0) return SW_OK;
    SW_CUDA(ctx, cudaSetDevice(ctx->device));
    if (!ctx->batch) ctx->batch = new sw_batch_state();
    sw_batch_state* b = ctx->batch;

    // ---- plan: stacks of queries, buckets by kernel shape ----
    std::vector<uint32_t> qlen(nq), order(nq);
    for (uint32_t i = 0; i < nq; ++i) qlen[i] = (uint32_t)(qoffsets[i + 1] - qoffsets[i]);
    std::iota(order.begin(), order.end(), 0u);
    std::stable_sort(order.begin(), order.end(),
                     [&](uint32_t x, uint32_t y) { return qlen[x] > qlen[y]; });
    uint32_t nz = 0;       // queries with residues
    while (nz < nq && qlen[order[nz]] > 0) ++nz;
    const int cut = b->opt.cutover;
    int64_t n_long = 0;
    if (cut > 0)
        while (n_long < ctx->n_pairs && (int)ctx->pair_ncols[n_long] > cut) ++n_long;
    if (n_long == ctx->n_pairs) n_long = 0;     // all long: no split

    // A bucket = one kernel shape and the stacks it runs.  Queries of at least
    // stack_rows residues: one stack each, shape from the tuning table.  The
    // shorter ones: packed (first fit, longest first) into stacks of at most
    // stack_rows rows, each query padded to whole R-row blocks.
    struct Stack {
        std::vector<uint32_t> q;        // queries, in row order
        uint32_t rows = 0;
    };
    struct Bucket {
        int T, R;
        std::vector<Stack> stacks;
    };
    std::vector<Bucket> buckets;
    const int sT = b->opt.group_width, sR = b->opt.rows_per_thread;
    const uint32_t cap_rows = (uint32_t)std::max(b->opt.stack_rows, 0);
    // paired queries (sw_qpbatch, below): with pair_long every query, else the
    // queries of at most pair_rows residues
    const QpKernel* qk = b->opt.pair_rows > 0
                             ? find_qp(b->opt.pair_group_width, b->opt.pair_rows_per_thread)
                             : nullptr;
    const bool pair_all = qk && b->opt.pair_long;
    uint32_t i0 = 0;
    while (!pair_all && i0 < nz && qlen[order[i0]] >= cap_rows) {
        const sw_kernel_config c = choose_config(ctx, (int)qlen[order[i0]]);
        if (buckets.empty() || buckets.back().T != c.short_group_width ||
            buckets.back().R != c.short_rows_per_thread || buckets.back().stacks.size() >= 1024)
            buckets.push_back(Bucket{c.short_group_width, c.short_rows_per_thread, {}});
        Stack st1;
        st1.q.push_back(order[i0]);
        st1.rows = qlen[order[i0]];
        buckets.back().stacks.push_back(st1);
        ++i0;
    }
    uint32_t ip = nz;
    if (pair_all)
        ip = 0;
    else if (qk)
        while (ip > i0 && qlen[order[ip - 1]] <= (uint32_t)b->opt.pair_rows) --ip;
    if (i0 < ip) {
        Bucket bk{sT, sR, {}};
        for (uint32_t i = i0; i < ip; ++i) {
            const uint32_t q = order[i];
            const uint32_t need = (qlen[q] + sR - 1) / sR * sR;
            bool placed = false;
            for (Stack& stk : bk.stacks)
                if (stk.rows + need <= cap_rows) {
                    stk.q.push_back(q);
                    stk.rows += need;
                    placed = true;
                    break;
                }
            if (!placed) {
                Stack stk;
                stk.q.push_back(q);
                stk.rows = need;
                bk.stacks.push_back(stk);
            }
        }
        buckets.push_back(bk);
    }
    // host image of every stack: row codes and the (pass, thread) -> query map
    StackPlan sp;
    std::vector<BatchLaunch> launches;
    size_t bnd_long = 0, bnd_bulk = 0;
    int nst_total = 0;
    for (const Bucket& bk : buckets) nst_total += (int)bk.stacks.size();
    int sidx = 0;
    for (const Bucket& bk : buckets) {
        const WfKernel* kb = find_kernel(bk.T, bk.R);
        if (!kb) SW_SET(ctx, SW_ERR_INVALID, "no kernel for shape %dx%d", bk.T, bk.R);
        uint32_t max_rows = 0;
        const int s0 = sidx;
        for (const Stack& stk : bk.stacks) {
            const uint32_t rows = stk.q.size() == 1 ? qlen[stk.q[0]] : stk.rows;
            max_rows = std::max(max_rows, rows);
            sp.off.push_back((uint32_t)sp.codes.size());
            sp.rows.push_back(rows);
            sp.rb_off.push_back((uint32_t)sp.rb_map.size());
            std::vector<int32_t> block_q;           // per R-row block: query | first bit
            for (const uint32_t q : stk.q) {
                const uint8_t* src = queries + qoffsets[q];
                const uint32_t L = qlen[q];
                const uint32_t padded = stk.q.size() == 1 ? L : (L + bk.R - 1) / bk.R * bk.R;
                sp.codes.insert(sp.codes.end(), src, src + L);
                sp.codes.insert(sp.codes.end(), padded - L, (uint8_t)kZeroCode);
                const uint32_t nblk = (padded + bk.R - 1) / bk.R;
                for (uint32_t j = 0; j < nblk; ++j)
                    block_q.push_back((int32_t)q | (j == 0 ? kFirstBit : 0));
            }
            const uint32_t P = (rows + bk.T * bk.R - 1) / (bk.T * bk.R);
            for (uint32_t j = 0; j < P * (uint32_t)bk.T; ++j)
                sp.rb_map.push_back(j < block_q.size() ? block_q[j] : -1);
            ++sidx;
        }
        const int occ = shape_occupancy(ctx, *kb, (int)max_rows);
        if (occ == 0)
            SW_SET(ctx, SW_ERR_UNSUPPORTED, "stack of %u rows does not fit shape %dx%d", max_rows,
                   kb->T, kb->R);
        {   // bulk: pairs [n_long, n_pairs), groups with private boundary rows
            BatchLaunch L;
            L.k = kb;
            L.threads = kb->block;
            L.grid = occ * ctx->num_sms;
            L.smem = kb->smem((int)max_rows);
            L.sbegin = s0;
            L.scount = sidx - s0;
            L.pair_begin = (int)n_long;
            L.pair_count = (int)(ctx->n_pairs - n_long);
            L.counter_base = s0;
            L.long_part = false;
            const int cols = n_long > 0 ? ((int)ctx->pair_ncols[n_long] + 7) / 8 * 8 : ctx->max_cols;
            L.bnd_group = 2 * (size_t)cols;
            bnd_bulk = std::max(bnd_bulk, (size_t)L.grid * (L.threads / kb->T) * L.bnd_group);
            launches.push_back(L);
        }
        if (n_long > 0) {
            // long pairs: single-group blocks of the same shape (the stacks'
            // row maps are laid out for it)
            const int occl = shape_occupancy(ctx, *kb, (int)max_rows);
            BatchLaunch L;
            L.k = kb;
            L.threads = kb->T;
            L.grid = (int)std::min<int64_t>((int64_t)std::max(occl, 1) * 2 * ctx->num_sms, n_long);
            L.smem = kb->smem((int)max_rows);
            L.sbegin = s0;
            L.scount = sidx - s0;
            L.pair_begin = 0;
            L.pair_count = (int)n_long;
            L.counter_base = nst_total + s0;
            L.long_part = true;
            L.bnd_group = 2 * (size_t)ctx->max_cols;
            bnd_long = std::max(bnd_long, (size_t)L.grid * L.bnd_group);
            launches.push_back(L);
        }
    }
    // paired queries: lanes of at most `seg` rows (first fit, longest first,
    // each query padded to whole R-row blocks; a longer query gets a lane of
    // its own), consecutive lanes paired into double stacks.  A double stack
    // taller than `seg` rows is cut into segments of `seg` rows, scored by
    // consecutive launches; segment s takes its upper boundary row from
    // segment s-1 through the per-record boundary buffer.
    if (qk && ip < nz) {
        const uint32_t qR = (uint32_t)qk->R, qT = (uint32_t)qk->T, pass_rows = qT * qR;
        const uint32_t seg = std::max(pass_rows, (uint32_t)b->opt.pair_rows / pass_rows * pass_rows);
        struct Lane {
            std::vector<uint32_t> q;
            uint32_t rows = 0;
        };
        std::vector<uint32_t> need_rows;
        for (uint32_t i = ip; i < nz; ++i) need_rows.push_back((qlen[order[i]] + qR - 1) / qR * qR);
        std::vector<Lane> lanes;
        for (const PairLane& pl : plan_pair_lanes(need_rows, seg, pass_rows)) {
            Lane ln;
            for (const uint32_t it : pl.items) ln.q.push_back(order[ip + it]);
            ln.rows = pl.rows;
            lanes.push_back(ln);
        }
        struct Double {
            uint32_t off[2], rows[2], nseg;
            std::vector<int32_t> blocks[2];
        };
        std::vector<Double> dbl(lanes.size() / 2);
        for (size_t d = 0; d < dbl.size(); ++d) {
            Double& D = dbl[d];
            for (int h = 0; h < 2; ++h) {
                const Lane& ln = lanes[2 * d + h];
                D.off[h] = (uint32_t)sp.codes.size();
                D.rows[h] = ln.rows;
                for (const uint32_t q : ln.q) {
                    const uint8_t* src = queries + qoffsets[q];
                    const uint32_t L = qlen[q];
                    const uint32_t padded = (L + qR - 1) / qR * qR;
                    sp.codes.insert(sp.codes.end(), src, src + L);
                    sp.codes.insert(sp.codes.end(), padded - L, (uint8_t)kZeroCode);
                    for (uint32_t j = 0; j < padded / qR; ++j)
                        D.blocks[h].push_back((int32_t)q | (j == 0 ? kFirstBit : 0));
                }
            }
            D.nseg = std::max<uint32_t>(1, (std::max(D.rows[0], D.rows[1]) + seg - 1) / seg);
        }
        // launches: every single-segment double stack in one launch; then the
        // taller double stacks in waves of as many as there are boundary
        // regions (each stack of a wave hands its segments' last rows on
        // through a region of its own): per wave, one launch per segment
        // level with every stack of the wave that has that segment, the levels
        // one after another
        std::vector<size_t> tall;
        for (size_t d = 0; d < dbl.size(); ++d)
            if (dbl[d].nseg > 1) tall.push_back(d);
        const int regions = seg_regions_for(
            ctx, b, std::min((int)tall.size(), b->opt.pair_regions > 0 ? b->opt.pair_regions : 16));
        // (double stack, segment, region)
        std::vector<std::vector<std::array<uint32_t, 3>>> groups(1);
        for (size_t d = 0; d < dbl.size(); ++d)
            if (dbl[d].nseg == 1) groups[0].push_back({(uint32_t)d, 0u, 0u});
        for (size_t w0 = 0; w0 < tall.size(); w0 += (size_t)regions) {
            const size_t w1 = std::min(tall.size(), w0 + (size_t)regions);
            uint32_t levels = 0;
            for (size_t i = w0; i < w1; ++i) levels = std::max(levels, dbl[tall[i]].nseg);
            for (uint32_t lv = 0; lv < levels; ++lv) {
                groups.emplace_back();
                for (size_t i = w0; i < w1; ++i)
                    if (lv < dbl[tall[i]].nseg)
                        groups.back().push_back({(uint32_t)tall[i], lv, (uint32_t)(i - w0)});
            }
        }
        for (const auto& grp : groups) {
            if (grp.empty()) continue;
            const int first = (int)sp.qp_off_lo.size();
            uint32_t max_rows = 0;
            for (const auto& e : grp) {
                const Double& D = dbl[e[0]];
                const uint32_t lv = e[1];
                sp.qp_slot.push_back(e[2]);
                uint32_t rs[2];
                for (int h = 0; h < 2; ++h) {
                    rs[h] = D.rows[h] > lv * seg ? std::min(seg, D.rows[h] - lv * seg) : 0u;
                    (h ? sp.qp_off_hi : sp.qp_off_lo).push_back(D.off[h] + lv * seg);
                    (h ? sp.qp_rows_hi : sp.qp_rows_lo).push_back(rs[h]);
                }
                const uint32_t rows = std::max(rs[0], rs[1]);
                max_rows = std::max(max_rows, rows);
                const uint32_t P = std::max<uint32_t>(1, (rows + pass_rows - 1) / pass_rows);
                sp.qp_rb_off.push_back((uint32_t)(sp.qp_rb_map.size() / 2));
                sp.qp_flags.push_back((lv > 0 ? 1u : 0u) | (lv + 1 < D.nseg ? 2u : 0u));
                const size_t b0 = (size_t)lv * seg / qR;
                for (uint32_t j = 0; j < P * qT; ++j)
                    for (int h = 0; h < 2; ++h)
                        sp.qp_rb_map.push_back(b0 + j < D.blocks[h].size() ? D.blocks[h][b0 + j] : -1);
            }
            const size_t smem = qk->smem((int)std::max<uint32_t>(max_rows, 1));
            int occ = 0;
            if (smem <= (size_t)ctx->max_smem &&
                cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, qk->fn, qk->block, smem) !=
                    cudaSuccess) {
                cudaGetLastError();
                occ = 0;
            }
            if (occ == 0)
                SW_SET(ctx, SW_ERR_UNSUPPORTED, "paired segments of %u rows do not fit shape %dx%d",
                       max_rows, qk->T, qk->R);
            BatchLaunch L;
            L.qk = qk;
            L.k = nullptr;
            L.threads = qk->block;
            L.grid = occ * ctx->num_sms;
            L.smem = smem;
            L.sbegin = first;
            L.scount = (int)sp.qp_off_lo.size() - first;
            L.pair_begin = 0;
            L.pair_count = (int)ctx->n_pairs;
            L.counter_base = 2 * nst_total + 1 + first;
            L.long_part = false;
            L.bnd_group = 2 * (size_t)ctx->max_cols;
            L.long_units = qp_long_units(
                [&](int p) { return (uint64_t)ctx->pair_ncols[(size_t)p]; },
                (int)ctx->n_pairs, ctx->pair_cols_total,
                (long long)L.grid * (L.threads / qk->T));
            bnd_bulk = std::max(bnd_bulk, (size_t)L.grid * (L.threads / qk->T) * L.bnd_group);
            launches.push_back(L);
        }
    }
    // counters: bulk of stack i at [i], long at [nst_total + i], overflow count
    // at [2 nst_total], paired double stack j at [2 nst_total + 1 + j]
    const MetaLayout ml = meta_layout(nq, sp);

    // ---- buffers (before any capture) ----
    const long long nblk0 = std::max<long long>(1, ((long long)n_rec + kTopkKeys - 1) / kTopkKeys);
    sw_status s;
    auto drop_graphs = [&]() {
        for (auto& kv : b->graphs) {      // graphs hold the old pointers
            if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
            if (kv.second.graph) cudaGraphDestroy(kv.second.graph);
        }
        b->graphs.clear();
    };
    const size_t counters_need = 2 * (size_t)nst_total + 1 + ml.nqp;
    if (std::max<uint64_t>(qbytes, 1) > b->queries_cap || ml.total > b->meta_cap ||
        counters_need > b->counters_cap)
        drop_graphs();
    if ((s = grow(ctx, &b->d_queries, b->queries_cap, std::max<uint64_t>(qbytes, 1), "queries")) != SW_OK) return s;
    if ((s = grow(ctx, &b->d_meta, b->meta_cap, ml.total, "stack table")) != SW_OK) return s;
    if ((s = grow(ctx, &b->d_counters, b->counters_cap, counters_need, "counters")) != SW_OK) return s;
    if (nq > b->scores_cap) {
        drop_graphs();
        dev_free(b->d_scores);
        dev_free(b->d_scores_rec);
        b->scores_cap = 0;
        if (dev_alloc(&b->d_scores, (size_t)nq * n_rec) != cudaSuccess ||
            dev_alloc(&b->d_scores_rec, (size_t)nq * n_rec) != cudaSuccess)
            SW_SET(ctx, SW_ERR_NOMEM, "device allocation failed: batch scores");
        b->scores_cap = nq;
    }
    // a (query, record) is flagged once per pass its query spans; flags are
    // rare (scores near 32,767), so twice the records per query is ample and
    // the kernels drop what would not fit (reported below)
    const size_t ovf_need = 2 * (size_t)nq * n_rec + 1;
    if (ovf_need > b->ovf_cap) drop_graphs();
    if ((s = grow(ctx, &b->d_ovf, b->ovf_cap, ovf_need, "overflow list")) != SW_OK) return s;
    const size_t keys_need = (size_t)nq * nblk0 * kMaxTopK;
    if (keys_need > b->keys_cap) {
        drop_graphs();
        dev_free(b->d_keys[0]);
        dev_free(b->d_keys[1]);
        b->keys_cap = 0;
        if (dev_alloc(&b->d_keys[0], keys_need) != cudaSuccess ||
            dev_alloc(&b->d_keys[1], keys_need) != cudaSuccess)
            SW_SET(ctx, SW_ERR_NOMEM, "device allocation failed: keys");
        b->keys_cap = keys_need;
    }
    // boundary rows: long launches in the first half, bulk launches in the second
    const size_t bnd_need = 2 * std::max(bnd_long, bnd_bulk) + 2;
    if (bnd_need > b->bnd_cap) {
        drop_graphs();
        if ((s = grow(ctx, &b->d_bnd, b->bnd_cap, bnd_need, "boundary rows")) != SW_OK) return s;
    }
    const size_t stage_need = qbytes + ml.total + 64;
    if (stage_need > b->stage_cap) {
        drop_graphs();
        if (b->h_stage) cudaFreeHost(b->h_stage);
        b->h_stage = nullptr;
        b->stage_cap = 0;
        const size_t capb = std::max<size_t>(stage_need * 2, 1 << 16);
        if (cudaMallocHost((void**)&b->h_stage, capb) != cudaSuccess)
            SW_SET(ctx, SW_ERR_NOMEM, "pinned staging buffer");
        b->stage_cap = capb;
    }
    if ((size_t)nq * k > b->hkeys_cap) {
        drop_graphs();
        if (b->h_keys) cudaFreeHost(b->h_keys);
        b->h_keys = nullptr;
        b->hkeys_cap = 0;
        if (cudaMallocHost((void**)&b->h_keys, (size_t)nq * k * sizeof(unsigned long long)) != cudaSuccess)
            SW_SET(ctx, SW_ERR_NOMEM, "pinned key buffer");
        b->hkeys_cap = (size_t)nq * k;
    }

    // ---- stage the inputs: queries at the front, the table at the back ----
    if (qbytes) memcpy(b->h_stage, queries + qoffsets[0], qbytes);
    {
        uint8_t* m = b->h_stage + ((b->stage_cap - ml.total) & ~(size_t)15);
        uint32_t* qo = reinterpret_cast<uint32_t*>(m + ml.qoff);
        uint32_t* ql = reinterpret_cast<uint32_t*>(m + ml.qlen);
        for (uint32_t i = 0; i < nq; ++i) {
            qo[i] = (uint32_t)(qoffsets[i] - qoffsets[0]);
            ql[i] = qlen[i];
        }
        const size_t ns = sp.off.size();
        memcpy(m + ml.soff, sp.off.data(), 4 * ns);
        memcpy(m + ml.srows, sp.rows.data(), 4 * ns);
        memcpy(m + ml.rboff, sp.rb_off.data(), 4 * ns);
        memcpy(m + ml.rbmap, sp.rb_map.data(), 4 * sp.rb_map.size());
        const size_t nqp = sp.qp_off_lo.size();
        memcpy(m + ml.qp_off_lo, sp.qp_off_lo.data(), 4 * nqp);
        memcpy(m + ml.qp_rows_lo, sp.qp_rows_lo.data(), 4 * nqp);
        memcpy(m + ml.qp_off_hi, sp.qp_off_hi.data(), 4 * nqp);
        memcpy(m + ml.qp_rows_hi, sp.qp_rows_hi.data(), 4 * nqp);
        memcpy(m + ml.qp_rboff, sp.qp_rb_off.data(), 4 * nqp);
        memcpy(m + ml.qp_flags, sp.qp_flags.data(), 4 * nqp);
        memcpy(m + ml.qp_slot, sp.qp_slot.data(), 4 * nqp);
        memcpy(m + ml.qp_rbmap, sp.qp_rb_map.data(), 4 * sp.qp_rb_map.size());
        memcpy(m + ml.codes, sp.codes.data(), sp.codes.size());
    }

    // ---- run: replay the captured graph for this signature, or capture it ----
    std::vector<uint64_t> sig;
    sig.reserve(nq + 8);
    sig.push_back(nq);
    sig.push_back(scores ? 1 : 0);
    sig.push_back((uint64_t)b->opt.cutover);
    sig.push_back((uint64_t)b->opt.group_width << 32 | (uint32_t)b->opt.rows_per_thread);
    sig.push_back((uint64_t)b->opt.stack_rows);
    sig.push_back((uint64_t)b->opt.pair_rows << 32 |
                  (uint64_t)(b->opt.pair_group_width * 256 + b->opt.pair_rows_per_thread) << 1 |
                  (uint64_t)(b->opt.pair_long != 0));
    sig.push_back((uint64_t)b->opt.pair_regions);
    for (uint32_t i = 0; i < nq; ++i) sig.push_back(qlen[i]);
    uint32_t n_launch = 0;
    SW_CUDA(ctx, cudaEventRecord(ctx->ev[0], ctx->stream));
    if (b->opt.use_graph) {
        auto it = b->graphs.find(sig);
        if (it == b->graphs.end()) {
            BatchGraph g;
            SW_CUDA(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
            sw_status es =
                enqueue_batch(ctx, b, nq, qbytes, ml, launches, scores != nullptr, &g.launches);
            cudaGraph_t graph = nullptr;
            const cudaError_t ce = cudaStreamEndCapture(ctx->stream, &graph);
            if (es != SW_OK) {
                if (graph) cudaGraphDestroy(graph);
                return es;
            }
            SW_CUDA(ctx, ce);
            g.graph = graph;
            SW_CUDA(ctx, cudaGraphInstantiate(&g.exec, graph, 0));
            if (b->graphs.size() >= 8) {
                auto old = b->graphs.begin();
                cudaGraphExecDestroy(old->second.exec);
                cudaGraphDestroy(old->second.graph);
                b->graphs.erase(old);
            }
            it = b->graphs.emplace(sig, g).first;
        }
        SW_CUDA(ctx, cudaGraphLaunch(it->second.exec, ctx->stream));
        n_launch = it->second.launches;
    } else {
        s = enqueue_batch(ctx, b, nq, qbytes, ml, launches, scores != nullptr, &n_launch);
        if (s != SW_OK) return s;
    }
    SW_CUDA(ctx, cudaEventRecord(ctx->ev[1], ctx->stream));
    if (scores)
        SW_CUDA(ctx, cudaMemcpyAsync(scores, b->d_scores_rec, (size_t)nq * n_rec * sizeof(int32_t),
                                     cudaMemcpyDeviceToHost, ctx->stream));
    SW_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    SW_CUDA(ctx, cudaGetLastError());
    {
        int flagged = 0;
        SW_CUDA(ctx, cudaMemcpy(&flagged, b->d_counters + 2 * sp.off.size(), sizeof(int),
                                cudaMemcpyDeviceToHost));
        if ((size_t)flagged > b->ovf_cap)
            SW_SET(ctx, SW_ERR_UNSUPPORTED, "%d overflow entries exceed the list (%zu)", flagged,
                   b->ovf_cap);
        ctx->stats.rescored = (uint64_t)flagged;
    }
    for (uint32_t q = 0; q < nq; ++q) {
        uint32_t m = 0;
        for (int i = 0; i < k; ++i) {
            const unsigned long long key = b->h_keys[(size_t)q * k + i];
            if (key == 0ull || qlen[q] == 0) break;
            hits[(size_t)q * k + m].score = (int32_t)(key >> 32);
            hits[(size_t)q * k + m].reserved = 0;
            hits[(size_t)q * k + m].index = 0xffffffffull - (key & 0xffffffffull);
            ++m;
        }
        n_hits[q] = m;
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[1]);
    uint64_t cells = 0;
    for (uint32_t q = 0; q < nq; ++q) cells += (uint64_t)qlen[q] * ctx->n_residues;
    ctx->stats.kernel_ms = ms;
    ctx->stats.cells = cells;
    ctx->stats.launches = n_launch;
    ctx->stats.queries = nq;
    ctx->stats.total_ms = wall_ms() - t0;
    ctx->totals.search_ms += ms;
    ctx->totals.launches += n_launch;
    ctx->totals.cells += cells;
    ctx->totals.queries += nq;
    return SW_OK;
}
