// sw_batch.cu -- batched search: many queries against the resident DB in one
// pass over the device, captured as a CUDA graph.
//
// The reference has no batched mode: WorkerPool searches one query per run
// and balances DB chunks across worker threads on the host
// (src/WorkerPool.cpp:10-82, src/DataPool.cpp:171-286).  Here a batch is:
//   * the queries sorted by length and cut into length buckets, one bucket per
//     kernel shape the tuning table picks for those lengths;
//   * per bucket, one persistent launch of sw_batch<T,R> over the bucket's
//     queries (blocks walk the queries in order, groups claim record pairs from
//     one device counter per query), plus, when a cut-over is set, a concurrent
//     launch of single-group blocks for the pairs longer than the cut-over, so
//     their inherently serial column steps overlap the bulk;
//   * one 32-bit re-score launch for every flagged (query, record) and one
//     top-k round sequence with a grid row per query.
// The whole sequence (query upload, launches, result download) is captured
// once per batch signature and replayed.
#include <algorithm>
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
#include "sw_registry.h"

using namespace swb;

struct BatchLaunch {
    const WfKernel* k;
    int grid, threads;
    size_t smem;
    int qbegin, qcount;        // entries of the qlist
    int pair_begin, pair_count;
    int counter_base;          // first counter of this launch
    bool long_part;            // runs on the side stream
    size_t bnd_group;
};

struct BatchGraph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint32_t launches = 0;
};

struct sw_batch_state {
    sw_batch_options opt{8192, 32, 16, 1};
    // device
    uint8_t* d_queries = nullptr;
    size_t queries_cap = 0;
    uint32_t* d_meta = nullptr;      // qoff[nq] | qlen[nq] | qlist[nq] (as uint32)
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

// Enqueues one batch on ctx->stream (and the side stream).  Buffers are sized.
sw_status enqueue_batch(sw_ctx* ctx, sw_batch_state* b, uint32_t nq, size_t qbytes,
                        const std::vector<BatchLaunch>& launches, bool want_scores,
                        uint32_t* n_launch) {
    cudaStream_t st = ctx->stream;
    const int n_rec = (int)ctx->n_records;
    const int k = ctx->params.top_k;
    *n_launch = 0;
    const size_t meta_bytes = (size_t)3 * nq * sizeof(uint32_t);
    SW_CUDA(ctx, cudaMemcpyAsync(b->d_queries, b->h_stage, qbytes ? qbytes : 1,
                                 cudaMemcpyHostToDevice, st));
    SW_CUDA(ctx, cudaMemcpyAsync(b->d_meta, b->h_stage + b->stage_cap - meta_bytes, meta_bytes,
                                 cudaMemcpyHostToDevice, st));
    SW_CUDA(ctx, cudaMemsetAsync(b->d_counters, 0, (2 * (size_t)nq + 1) * sizeof(int), st));
    SW_CUDA(ctx, cudaMemsetAsync(b->d_scores, 0, (size_t)nq * n_rec * sizeof(int), st));
    const uint32_t* d_qoff = b->d_meta;
    const uint32_t* d_qlen = b->d_meta + nq;
    const int* d_qlist = reinterpret_cast<const int*>(b->d_meta + 2 * nq);
    int* d_ovf_count = b->d_counters + 2 * nq;
    const int ovf_thresh = 32767 - std::max(ctx->max_score, 1) + 1;
    bool forked = false;
    for (const BatchLaunch& L : launches) {
        BatchArgs a;
        a.db = ctx->d_db;
        a.pairs = ctx->d_pairs;
        a.pair_begin = L.pair_begin;
        a.pair_count = L.pair_count;
        a.queries = b->d_queries;
        a.qoff = d_qoff;
        a.qlen = d_qlen;
        a.qlist = d_qlist + L.qbegin;
        a.nq = L.qcount;
        a.counters = b->d_counters + L.counter_base;
        a.mat = ctx->d_mat;
        a.bias2 = (uint32_t)(ctx->params.gap_open + ctx->params.gap_extend);
        a.bias2 |= a.bias2 << 16;
        a.neg_e = (uint32_t)(uint16_t)(int16_t)(-ctx->params.gap_extend);
        a.neg_e |= a.neg_e << 16;
        a.one = 1u;
        a.bnd = L.long_part ? b->d_bnd : b->d_bnd + b->bnd_cap / 2;
        a.bnd_group = L.bnd_group;
        a.scores = b->d_scores;
        a.n_records = n_rec;
        a.ovf_list = b->d_ovf;
        a.ovf_count = d_ovf_count;
        a.ovf_thresh = ovf_thresh;
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
        if (opt->cutover < 0 || !find_kernel(opt->long_group_width, opt->long_rows_per_thread))
            SW_SET(ctx, SW_ERR_INVALID, "bad batch options");
        ctx->batch->opt = *opt;
    } else {
        ctx->batch->opt = sw_batch_options{8192, 32, 16, 1};
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
    if (!ctx->db_loaded) SW_SET(ctx, SW_ERR_STATE, "no DB loaded (call sw_db_load first)");
    if (nq == 0) return SW_OK;
    if (!qoffsets || !hits || !n_hits) SW_SET(ctx, SW_ERR_INVALID, "null argument");
    const double t0 = wall_ms();
    const int k = ctx->params.top_k;
    const int n_rec = (int)ctx->n_records;
    if ((uint64_t)nq * (uint64_t)std::max(n_rec, 1) >= (1ull << 31))
        SW_SET(ctx, SW_ERR_UNSUPPORTED, "batch too large: %u queries x %d records", nq, n_rec);
    for (uint32_t i = 0; i < nq; ++i)
        if (qoffsets[i + 1] < qoffsets[i]) SW_SET(ctx, SW_ERR_INVALID, "query offsets not monotone");
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

    // ---- plan: queries sorted by length, buckets by tuned shape ----
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
    std::vector<BatchLaunch> launches;
    int counter_base = 0;
    size_t bnd_long = 0, bnd_bulk = 0;
    uint32_t i0 = 0;
    while (i0 < nz) {
        const sw_kernel_config c0 = choose_config(ctx, (int)qlen[order[i0]]);
        uint32_t i1 = i0 + 1;
        while (i1 < nz) {
            const sw_kernel_config c1 = choose_config(ctx, (int)qlen[order[i1]]);
            if (c1.short_group_width != c0.short_group_width ||
                c1.short_rows_per_thread != c0.short_rows_per_thread)
                break;
            ++i1;
        }
        const int maxq = (int)qlen[order[i0]];
        const WfKernel* kb = find_kernel(c0.short_group_width, c0.short_rows_per_thread);
        if (!kb) SW_SET(ctx, SW_ERR_INVALID, "no kernel for the tuned shape");
        const int occ = shape_occupancy(ctx, *kb, maxq);
        if (occ == 0)
            SW_SET(ctx, SW_ERR_UNSUPPORTED, "query of %d residues does not fit shape %dx%d", maxq,
                   kb->T, kb->R);
        // bulk: pairs [n_long, n_pairs), groups with private boundary rows
        {
            BatchLaunch L;
            L.k = kb;
            L.threads = kb->block;
            L.grid = occ * ctx->num_sms;
            L.smem = kb->smem(maxq);
            L.qbegin = (int)i0;
            L.qcount = (int)(i1 - i0);
            L.pair_begin = (int)n_long;
            L.pair_count = (int)(ctx->n_pairs - n_long);
            L.counter_base = counter_base;
            L.long_part = false;
            const int cols = n_long > 0 ? ((int)ctx->pair_ncols[n_long] + 7) / 8 * 8 : ctx->max_cols;
            L.bnd_group = 2 * (size_t)cols;
            bnd_bulk = std::max(bnd_bulk, (size_t)L.grid * (L.threads / kb->T) * L.bnd_group);
            launches.push_back(L);
        }
        if (n_long > 0) {
            const WfKernel* kl = find_kernel(b->opt.long_group_width, b->opt.long_rows_per_thread);
            const int occl = shape_occupancy(ctx, *kl, maxq);
            if (occl == 0)
                SW_SET(ctx, SW_ERR_UNSUPPORTED, "query of %d residues does not fit the long shape",
                       maxq);
            BatchLaunch L;
            L.k = kl;
            L.threads = kl->T;
            L.grid = (int)std::min<int64_t>((int64_t)2 * ctx->num_sms, n_long);
            L.smem = kl->smem(maxq);
            L.qbegin = (int)i0;
            L.qcount = (int)(i1 - i0);
            L.pair_begin = 0;
            L.pair_count = (int)n_long;
            L.counter_base = counter_base + (int)nq;
            L.long_part = true;
            L.bnd_group = 2 * (size_t)ctx->max_cols;
            bnd_long = std::max(bnd_long, (size_t)L.grid * L.bnd_group);
            launches.push_back(L);
        }
        counter_base += (int)(i1 - i0);
        i0 = i1;
    }
    // counters: bulk i at [i], long i at [nq + i] (i = position in the qlist)

    // ---- buffers (before any capture) ----
    const long long nblk0 = std::max<long long>(1, ((long long)n_rec + kTopkKeys - 1) / kTopkKeys);
    sw_status s;
    if ((s = grow(ctx, &b->d_queries, b->queries_cap, std::max<uint64_t>(qbytes, 1), "queries")) != SW_OK) return s;
    if ((s = grow(ctx, &b->d_meta, b->meta_cap, (size_t)3 * nq, "query table")) != SW_OK) return s;
    if ((s = grow(ctx, &b->d_counters, b->counters_cap, 2 * (size_t)nq + 1, "counters")) != SW_OK) return s;
    if (nq > b->scores_cap) {
        dev_free(b->d_scores);
        dev_free(b->d_scores_rec);
        b->scores_cap = 0;
        if (dev_alloc(&b->d_scores, (size_t)nq * n_rec) != cudaSuccess ||
            dev_alloc(&b->d_scores_rec, (size_t)nq * n_rec) != cudaSuccess)
            SW_SET(ctx, SW_ERR_NOMEM, "device allocation failed: batch scores");
        b->scores_cap = nq;
    }
    if ((s = grow(ctx, &b->d_ovf, b->ovf_cap, (size_t)nq * n_rec + 1, "overflow list")) != SW_OK) return s;
    const size_t keys_need = (size_t)nq * nblk0 * kMaxTopK;
    if (keys_need > b->keys_cap) {
        dev_free(b->d_keys[0]);
        dev_free(b->d_keys[1]);
        b->keys_cap = 0;
        if (dev_alloc(&b->d_keys[0], keys_need) != cudaSuccess ||
            dev_alloc(&b->d_keys[1], keys_need) != cudaSuccess)
            SW_SET(ctx, SW_ERR_NOMEM, "device allocation failed: keys");
        b->keys_cap = keys_need;
    }
    // boundary rows: long launch in the first half, bulk launches in the second
    const size_t bnd_need = 2 * std::max(bnd_long, bnd_bulk) + 2;
    if (bnd_need > b->bnd_cap) {
        for (auto& kv : b->graphs) {      // graphs hold the old pointer
            if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
            if (kv.second.graph) cudaGraphDestroy(kv.second.graph);
        }
        b->graphs.clear();
        if ((s = grow(ctx, &b->d_bnd, b->bnd_cap, bnd_need, "boundary rows")) != SW_OK) return s;
    }
    const size_t meta_bytes = (size_t)3 * nq * sizeof(uint32_t);
    const size_t stage_need = qbytes + meta_bytes + 64;
    if (stage_need > b->stage_cap) {
        for (auto& kv : b->graphs) {
            if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
            if (kv.second.graph) cudaGraphDestroy(kv.second.graph);
        }
        b->graphs.clear();
        if (b->h_stage) cudaFreeHost(b->h_stage);
        b->h_stage = nullptr;
        b->stage_cap = 0;
        const size_t cap = std::max<size_t>(stage_need * 2, 1 << 16);
        if (cudaMallocHost((void**)&b->h_stage, cap) != cudaSuccess)
            SW_SET(ctx, SW_ERR_NOMEM, "pinned staging buffer");
        b->stage_cap = cap;
    }
    if ((size_t)nq * k > b->hkeys_cap) {
        for (auto& kv : b->graphs) {
            if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
            if (kv.second.graph) cudaGraphDestroy(kv.second.graph);
        }
        b->graphs.clear();
        if (b->h_keys) cudaFreeHost(b->h_keys);
        b->h_keys = nullptr;
        b->hkeys_cap = 0;
        if (cudaMallocHost((void**)&b->h_keys, (size_t)nq * k * sizeof(unsigned long long)) != cudaSuccess)
            SW_SET(ctx, SW_ERR_NOMEM, "pinned key buffer");
        b->hkeys_cap = (size_t)nq * k;
    }

    // ---- stage the inputs: queries, then [qoff | qlen | qlist] at the end ----
    if (qbytes) memcpy(b->h_stage, queries + qoffsets[0], qbytes);
    uint32_t* meta = reinterpret_cast<uint32_t*>(b->h_stage + b->stage_cap - meta_bytes);
    for (uint32_t i = 0; i < nq; ++i) {
        meta[i] = (uint32_t)(qoffsets[i] - qoffsets[0]);
        meta[nq + i] = qlen[i];
        meta[2 * nq + i] = order[i];
    }

    // ---- run: replay the captured graph for this signature, or capture it ----
    std::vector<uint64_t> sig;
    sig.reserve(nq + 8);
    sig.push_back(nq);
    sig.push_back(scores ? 1 : 0);
    sig.push_back((uint64_t)b->opt.cutover);
    for (uint32_t i = 0; i < nq; ++i) sig.push_back(qlen[i]);
    uint32_t n_launch = 0;
    SW_CUDA(ctx, cudaEventRecord(ctx->ev[0], ctx->stream));
    if (b->opt.use_graph) {
        auto it = b->graphs.find(sig);
        if (it == b->graphs.end()) {
            BatchGraph g;
            SW_CUDA(ctx, cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal));
            sw_status es = enqueue_batch(ctx, b, nq, qbytes, launches, scores != nullptr, &g.launches);
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
        s = enqueue_batch(ctx, b, nq, qbytes, launches, scores != nullptr, &n_launch);
        if (s != SW_OK) return s;
    }
    SW_CUDA(ctx, cudaEventRecord(ctx->ev[1], ctx->stream));
    if (scores)
        SW_CUDA(ctx, cudaMemcpyAsync(scores, b->d_scores_rec, (size_t)nq * n_rec * sizeof(int32_t),
                                     cudaMemcpyDeviceToHost, ctx->stream));
    SW_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    SW_CUDA(ctx, cudaGetLastError());
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
