// sw_serve.cu -- serving: a request loop with continuous batching on the
// device.
//
// The reference has no serving mode (one query per process run,
// src/main.cpp).  Here a scheduler thread owns the context between
// sw_serve_start and sw_serve_stop:
//   * the DB's record pairs are dealt round-robin (longest first) into
//     `chunks` chunks with the same length mix, and the chunks form a ring;
//   * a device round scores the next chunk of the ring for every request in
//     flight: short requests (up to pair_rows residues) two per register in
//     paired lanes (one launch of sw_qpbatch, packed profile, as in
//     sw_search_batch), the others in one persistent launch of the stacked
//     kernel (sw_batch: short ones share R-row blocks of a stack, long ones
//     get stacks of their own), one 32-bit re-score launch for the round's
//     flagged (request, record) entries and, for the requests that have now
//     seen every chunk, one top-k round sequence and the download of their
//     keys;
//   * rounds are pipelined: round r+1 is enqueued before the host waits for
//     round r (double-buffered host tables, keys and overflow count), so the
//     device does not idle while the host reads results and plans;
//   * a request joins the ring at whatever chunk is next and completes after
//     `chunks` rounds, so a request that arrives while a round runs waits at
//     most that round before its work shares the device with everything
//     already in flight (iteration-level batching);
//   * admission happens at every round boundary into free slots.  A slot is
//     the device memory of one request in flight (its score row); the slot
//     count is bounded by max_active and by a device-memory budget, and the
//     waiting queue by max_pending (SW_ERR_BUSY beyond it);
//   * a request longer than one stack of the serving shape can hold (its
//     query profile would not fit one block's shared memory) is scored alone
//     at a round boundary by the plain path, which splits its rows over
//     consecutive launches; it does not share launches with the batch.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/swb200.h"
#include "sw_aux.h"
#include "sw_device.cuh"
#include "sw_engine.h"
#include "sw_qpair.cuh"
#include "sw_registry.h"

using namespace swb;

namespace {

constexpr uint32_t kServeMaxQuery = 1u << 24;  // residues per request

double now_ms() {
    return std::chrono::duration<double, std::milli>(
               std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

struct Request {
    uint64_t id = 0;
    std::vector<uint8_t> query;
    double submit_ms = 0, start_ms = 0, done_ms = 0;
    sw_status status = SW_OK;
    std::vector<sw_hit> hits;
};

struct Slot {
    bool used = false;
    bool fresh = false;     // admitted at this round boundary: score row to clear
    int done_chunks = 0;    // chunks scored so far
    Request req;
};

}  // namespace

struct sw_serve_state {
    sw_serve_options opt{};
    const WfKernel* k = nullptr;
    const QpKernel* qk = nullptr;         // paired lanes for short requests (null = off)
    uint32_t pair_seg = 0;                // rows of a paired lane
    int n_slots = 0;
    int n_chunks = 1;
    uint32_t max_stack_rows = 0;          // longer requests run alone (plain path)
    int occ_max = 0;                      // most blocks per SM any stack height gives
    int occ_qp_max = 0;                   // ... and any paired lane height
    std::vector<int> chunk_begin;         // n_chunks + 1 entries into d_pairs
    std::vector<uint32_t> ring_ncols;     // column count of each entry of d_pairs
    std::vector<uint64_t> chunk_cols;     // sum of ring_ncols per chunk
    Pair2* d_pairs = nullptr;             // pair table, chunk after chunk
    uint32_t* d_pair_ids = nullptr;       // global pair index of each entry
    int* d_scores = nullptr;              // [slot][sorted position]
    uint8_t* d_meta = nullptr;            // per-round tables (layout in run_round)
    size_t meta_cap = 0;
    int* d_counters = nullptr;            // stacks, the overflow count, paired launch entries
    size_t counters_cap = 0;
    int* d_ovf = nullptr;
    size_t ovf_cap = 0;
    uint2* d_bnd = nullptr;
    size_t bnd_group = 0;
    uint2* d_segbnd = nullptr;            // boundary regions of tall paired double stacks
    int seg_regions = 1;                  // (1: the context's own rows, d_segbnd null)
    size_t seg_stride = 0;
    unsigned long long* d_keys[2] = {nullptr, nullptr};
    // per-round host buffers, two sets: round r+1 is enqueued before the host
    // waits for round r, so r's tables, keys and flagged count stay untouched
    uint8_t* h_stage[2] = {nullptr, nullptr};          // pinned: the round's tables
    size_t stage_cap[2] = {0, 0};
    unsigned long long* h_keys[2] = {nullptr, nullptr}; // pinned: n_slots * top_k
    int* h_flagged[2] = {nullptr, nullptr};            // pinned: the round's overflow count
    cudaEvent_t done_ev[2] = {nullptr, nullptr};       // the round's last operation
    cudaEvent_t start_ev[2] = {nullptr, nullptr};      // the round's first operation
    int cursor = 0;                       // next chunk of the ring
    std::vector<Slot> slots;
    std::deque<Request> pending, done;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    bool stopping = false;
    std::thread th;
    sw_serve_stats stats{};
};

namespace {

void serve_free(sw_serve_state* s) {
    dev_free(s->d_pairs);
    dev_free(s->d_pair_ids);
    dev_free(s->d_scores);
    dev_free(s->d_meta);
    dev_free(s->d_counters);
    dev_free(s->d_ovf);
    dev_free(s->d_bnd);
    dev_free(s->d_segbnd);
    dev_free(s->d_keys[0]);
    dev_free(s->d_keys[1]);
    for (int b = 0; b < 2; ++b) {
        if (s->h_stage[b]) cudaFreeHost(s->h_stage[b]);
        if (s->h_keys[b]) cudaFreeHost(s->h_keys[b]);
        if (s->h_flagged[b]) cudaFreeHost(s->h_flagged[b]);
        if (s->done_ev[b]) cudaEventDestroy(s->done_ev[b]);
        if (s->start_ev[b]) cudaEventDestroy(s->start_ev[b]);
        s->h_stage[b] = nullptr;
        s->h_keys[b] = nullptr;
        s->h_flagged[b] = nullptr;
        s->done_ev[b] = nullptr;
        s->start_ev[b] = nullptr;
        s->stage_cap[b] = 0;
    }
}

// Enqueues one device round on the context's stream: chunk `chunk` for every
// active slot, using host buffer set `buf`.  `finishing` gets the slots whose
// cycle ends with this round; their keys land in h_keys[buf] in that order,
// and the round's overflow count in h_flagged[buf], once done_ev[buf] has
// completed.  Runs on the scheduler thread only.
sw_status enqueue_round(sw_ctx* ctx, sw_serve_state* s, int chunk, int buf,
                        std::vector<int>& finishing, uint32_t* launches) {
    cudaStream_t st = ctx->stream;
    const int n_rec = (int)ctx->n_records;
    const int T = s->k->T, R = s->k->R;
    const uint32_t cap_rows = (uint32_t)std::max<int32_t>(s->opt.stack_rows, R);
    *launches = 0;
    std::vector<int> active;
    finishing.clear();
    for (int i = 0; i < s->n_slots; ++i)
        if (s->slots[i].used) {
            active.push_back(i);
            if (s->slots[i].done_chunks + 1 == s->n_chunks) finishing.push_back(i);
        }
    // stacks: first fit, longest first; requests of at least cap_rows rows
    // get a stack each
    std::stable_sort(active.begin(), active.end(), [&](int a, int b) {
        return s->slots[a].req.query.size() > s->slots[b].req.query.size();
    });
    // requests whose padded rows fit a paired lane: two per register against
    // one record (sw_qpbatch, packed profile); the others: stacks
    const QpKernel* qk = s->qk;
    const uint32_t qR = qk ? (uint32_t)qk->R : 1u, qT = qk ? (uint32_t)qk->T : 1u;
    // (with pair_long every request: one longer than a lane gets a lane of
    // its own, scored in lane-height segments by consecutive launches)
    std::vector<int> paired, stacked;
    for (int sl : active) {
        const uint32_t L = (uint32_t)s->slots[sl].req.query.size();
        const bool fits = (L + qR - 1) / qR * qR <= s->pair_seg;
        (qk && (fits || s->opt.pair_long) ? paired : stacked).push_back(sl);
    }
    struct Stack {
        std::vector<int> slots;
        uint32_t rows = 0;
    };
    std::vector<Stack> stacks;
    for (int sl : stacked) {
        const uint32_t L = (uint32_t)s->slots[sl].req.query.size();
        const uint32_t need = (L + R - 1) / R * R;
        bool placed = false;
        if (L < cap_rows)
            for (Stack& stk : stacks)
                if (stk.rows + need <= cap_rows) {
                    stk.slots.push_back(sl);
                    stk.rows += need;
                    placed = true;
                    break;
                }
        if (!placed) {
            Stack stk;
            stk.slots.push_back(sl);
            stk.rows = need;
            stacks.push_back(stk);
        }
    }
    // Device tables of this round, one upload:
    //   qoff[n_slots], qlen[n_slots]                uint32 (re-score: slot -> its codes)
    //   stack_off[ns], stack_rows[ns], rb_off[ns]   uint32
    //   rb_map[...]                                 int32
    //   rows[finishing]                             int32 (top-k score rows)
    //   codes, every stack's rows back to back      uint8
    const size_t ns = stacks.size();
    std::vector<uint32_t> qoff((size_t)s->n_slots, 0), qlen((size_t)s->n_slots, 0), soff, srows, rboff;
    std::vector<int32_t> rbmap;
    std::vector<uint8_t> codes;
    uint32_t max_rows = 0;
    for (const Stack& stk : stacks) {
        soff.push_back((uint32_t)codes.size());
        rboff.push_back((uint32_t)rbmap.size());
        std::vector<int32_t> block_q;          // per R-row block: slot | first bit
        for (int sl : stk.slots) {
            const std::vector<uint8_t>& q = s->slots[sl].req.query;
            const uint32_t L = (uint32_t)q.size();
            const uint32_t padded = (L + R - 1) / R * R;
            qoff[sl] = (uint32_t)codes.size();
            qlen[sl] = L;
            codes.insert(codes.end(), q.begin(), q.end());
            codes.insert(codes.end(), padded - L, (uint8_t)kZeroCode);
            for (uint32_t j = 0; j < padded / R; ++j)
                block_q.push_back((int32_t)sl | (j == 0 ? kFirstBit : 0));
        }
        srows.push_back(stk.rows);
        max_rows = std::max(max_rows, stk.rows);
        const uint32_t P = (stk.rows + T * R - 1) / (T * R);
        for (uint32_t j = 0; j < P * (uint32_t)T; ++j)
            rbmap.push_back(j < block_q.size() ? block_q[j] : -1);
    }
    // paired lanes (plan_pair_lanes, sw_qpair.cuh): a request longer than
    // pair_seg rows gets a lane of its own, the others fill the rows the
    // tall double stacks' last passes would leave as padding, then lanes of
    // at most pair_seg rows; each request padded to whole R-row blocks;
    // consecutive lanes form a double stack (low lane, high lane)
    struct Lane {
        std::vector<int> slots;
        uint32_t rows = 0;
    };
    std::vector<Lane> lanes;
    {
        std::vector<uint32_t> need_rows;
        for (int sl : paired)
            need_rows.push_back(((uint32_t)s->slots[sl].req.query.size() + qR - 1) / qR * qR);
        for (const PairLane& pl : plan_pair_lanes(need_rows, s->pair_seg, qT * qR)) {
            Lane ln;
            for (const uint32_t it : pl.items) ln.slots.push_back(paired[it]);
            ln.rows = pl.rows;
            lanes.push_back(ln);
        }
    }
    const size_t nd = lanes.size() / 2;
    // entries of the paired launches: one per (double stack, segment); every
    // single-segment double stack in the first launch, then each taller one's
    // segments in launches of their own, one after another (segment s reads
    // the rows above from segment s-1 through the per-record boundary rows)
    std::vector<uint32_t> qp_off[2], qp_rows[2], qp_rboff, qp_flags;
    std::vector<int32_t> qp_rbmap;           // (low, high) entries
    struct QpLaunch {
        size_t first = 0, count = 0;
        uint32_t max_rows = 0;
    };
    std::vector<QpLaunch> qp_launches;
    std::vector<uint32_t> d_off[2];
    std::vector<std::vector<int32_t>> d_blocks[2];
    std::vector<uint32_t> d_nseg;
    for (size_t d = 0; d < nd; ++d) {
        for (int h = 0; h < 2; ++h) {
            const Lane& ln = lanes[2 * d + h];
            d_off[h].push_back((uint32_t)codes.size());
            d_blocks[h].emplace_back();
            for (int sl : ln.slots) {
                const std::vector<uint8_t>& q = s->slots[sl].req.query;
                const uint32_t L = (uint32_t)q.size();
                const uint32_t padded = (L + qR - 1) / qR * qR;
                qoff[sl] = (uint32_t)codes.size();
                qlen[sl] = L;
                codes.insert(codes.end(), q.begin(), q.end());
                codes.insert(codes.end(), padded - L, (uint8_t)kZeroCode);
                for (uint32_t j = 0; j < padded / qR; ++j)
                    d_blocks[h].back().push_back((int32_t)sl | (j == 0 ? kFirstBit : 0));
            }
        }
        const uint32_t rows = std::max(lanes[2 * d].rows, lanes[2 * d + 1].rows);
        d_nseg.push_back(std::max<uint32_t>(1, (rows + s->pair_seg - 1) / s->pair_seg));
    }
    std::vector<uint32_t> qp_slot;           // boundary region of each entry
    auto add_entry = [&](size_t d, uint32_t lv, uint32_t region) {
        qp_slot.push_back(region);
        uint32_t rs[2];
        for (int h = 0; h < 2; ++h) {
            const uint32_t lr = lanes[2 * d + h].rows;
            rs[h] = lr > lv * s->pair_seg ? std::min(s->pair_seg, lr - lv * s->pair_seg) : 0u;
            qp_off[h].push_back(d_off[h][d] + lv * s->pair_seg);
            qp_rows[h].push_back(rs[h]);
        }
        const uint32_t rows = std::max(rs[0], rs[1]);
        const uint32_t P = std::max<uint32_t>(1, (rows + qT * qR - 1) / (qT * qR));
        qp_rboff.push_back((uint32_t)(qp_rbmap.size() / 2));
        qp_flags.push_back((lv > 0 ? 1u : 0u) | (lv + 1 < d_nseg[d] ? 2u : 0u));
        const size_t b0 = (size_t)lv * s->pair_seg / qR;
        for (uint32_t j = 0; j < P * qT; ++j)
            for (int h = 0; h < 2; ++h)
                qp_rbmap.push_back(b0 + j < d_blocks[h][d].size() ? d_blocks[h][d][b0 + j] : -1);
        return rows;
    };
    {
        QpLaunch L0;
        L0.first = qp_flags.size();
        for (size_t d = 0; d < nd; ++d)
            if (d_nseg[d] == 1) L0.max_rows = std::max(L0.max_rows, add_entry(d, 0, 0));
        L0.count = qp_flags.size() - L0.first;
        if (L0.count) qp_launches.push_back(L0);
        // taller double stacks in waves of as many as there are boundary
        // regions, one launch per segment level and wave
        std::vector<size_t> tall;
        for (size_t d = 0; d < nd; ++d)
            if (d_nseg[d] > 1) tall.push_back(d);
        const size_t R = (size_t)std::max(s->seg_regions, 1);
        for (size_t w0 = 0; w0 < tall.size(); w0 += R) {
            const size_t w1 = std::min(tall.size(), w0 + R);
            uint32_t levels = 0;
            for (size_t i = w0; i < w1; ++i) levels = std::max(levels, d_nseg[tall[i]]);
            for (uint32_t lv = 0; lv < levels; ++lv) {
                QpLaunch Ls;
                Ls.first = qp_flags.size();
                for (size_t i = w0; i < w1; ++i)
                    if (lv < d_nseg[tall[i]])
                        Ls.max_rows = std::max(Ls.max_rows, add_entry(tall[i], lv, (uint32_t)(i - w0)));
                Ls.count = qp_flags.size() - Ls.first;
                qp_launches.push_back(Ls);
            }
        }
    }
    const size_t ne = qp_flags.size();
    // table layout (one upload; the paired block map is read as int2)
    size_t total = 0;
    auto place = [&total](size_t bytes, size_t align) {
        const size_t o = (total + align - 1) / align * align;
        total = o + bytes;
        return o;
    };
    const size_t o_qoff = place(4 * (size_t)s->n_slots, 4), o_qlen = place(4 * (size_t)s->n_slots, 4);
    const size_t o_soff = place(4 * ns, 4), o_srows = place(4 * ns, 4), o_rboff = place(4 * ns, 4);
    const size_t o_rbmap = place(4 * rbmap.size(), 4);
    const size_t o_rows = place(4 * finishing.size(), 4);
    const size_t o_qpo0 = place(4 * ne, 4), o_qpr0 = place(4 * ne, 4);
    const size_t o_qpo1 = place(4 * ne, 4), o_qpr1 = place(4 * ne, 4), o_qprb = place(4 * ne, 4);
    const size_t o_qpfl = place(4 * ne, 4), o_qpsl = place(4 * ne, 4);
    const size_t o_qpmap = place(4 * qp_rbmap.size(), 8);
    const size_t o_codes = place(codes.size(), 16);
    total = (total + 15) / 16 * 16;
    if (total > s->meta_cap) {
        // the round in flight still reads the old tables
        SW_CUDA(ctx, cudaStreamSynchronize(st));
        dev_free(s->d_meta);
        s->meta_cap = 0;
        if (dev_alloc(&s->d_meta, total * 2) != cudaSuccess)
            SW_SET(ctx, SW_ERR_NOMEM, "device allocation failed: serving tables");
        s->meta_cap = total * 2;
    }
    if (total > s->stage_cap[buf]) {
        // the round that last used this set has completed (the caller waits
        // for it before reusing the set)
        if (s->h_stage[buf]) cudaFreeHost(s->h_stage[buf]);
        s->h_stage[buf] = nullptr;
        s->stage_cap[buf] = 0;
        if (cudaMallocHost((void**)&s->h_stage[buf], total * 2) != cudaSuccess)
            SW_SET(ctx, SW_ERR_NOMEM, "pinned allocation failed: serving tables");
        s->stage_cap[buf] = total * 2;
    }
    uint8_t* m = s->h_stage[buf];
    memcpy(m + o_qoff, qoff.data(), 4 * qoff.size());
    memcpy(m + o_qlen, qlen.data(), 4 * qlen.size());
    if (ns) {
        memcpy(m + o_soff, soff.data(), 4 * ns);
        memcpy(m + o_srows, srows.data(), 4 * ns);
        memcpy(m + o_rboff, rboff.data(), 4 * ns);
        memcpy(m + o_rbmap, rbmap.data(), 4 * rbmap.size());
    }
    if (!finishing.empty()) memcpy(m + o_rows, finishing.data(), 4 * finishing.size());
    if (ne) {
        memcpy(m + o_qpo0, qp_off[0].data(), 4 * ne);
        memcpy(m + o_qpr0, qp_rows[0].data(), 4 * ne);
        memcpy(m + o_qpo1, qp_off[1].data(), 4 * ne);
        memcpy(m + o_qpr1, qp_rows[1].data(), 4 * ne);
        memcpy(m + o_qprb, qp_rboff.data(), 4 * ne);
        memcpy(m + o_qpfl, qp_flags.data(), 4 * ne);
        memcpy(m + o_qpsl, qp_slot.data(), 4 * ne);
        memcpy(m + o_qpmap, qp_rbmap.data(), 4 * qp_rbmap.size());
    }
    if (!codes.empty()) memcpy(m + o_codes, codes.data(), codes.size());
    SW_CUDA(ctx, cudaEventRecord(s->start_ev[buf], st));
    SW_CUDA(ctx, cudaMemcpyAsync(s->d_meta, m, total, cudaMemcpyHostToDevice, st));
    // score rows of requests admitted at this boundary start at zero (atomicMax)
    for (int sl : active)
        if (s->slots[sl].fresh)
            SW_CUDA(ctx, cudaMemsetAsync(s->d_scores + (size_t)sl * n_rec, 0,
                                         (size_t)n_rec * sizeof(int), st));
    // counters: stack i at [i], the overflow count at [ns], paired entry j at
    // [ns + 1 + j]
    const size_t n_counters = ns + 1 + ne;
    if (n_counters > s->counters_cap)
        SW_SET(ctx, SW_ERR_UNSUPPORTED, "%zu paired launch entries exceed the counters (%zu)", ne,
               s->counters_cap);
    SW_CUDA(ctx, cudaMemsetAsync(s->d_counters, 0, n_counters * sizeof(int), st));
    const int occ = ns ? std::min(shape_occupancy(ctx, *s->k, (int)max_rows), s->occ_max) : 1;
    if (occ <= 0)
        SW_SET(ctx, SW_ERR_UNSUPPORTED, "a stack of %u rows does not fit shape %dx%d", max_rows,
               T, R);
    int* d_ovf_count = s->d_counters + ns;
    const int pair_count = s->chunk_begin[chunk + 1] - s->chunk_begin[chunk];
    for (const QpLaunch& L : pair_count > 0 ? qp_launches : std::vector<QpLaunch>()) {
        const size_t smem = qk->smem((int)std::max<uint32_t>(L.max_rows, 1));
        int occq = 0;
        if (smem > (size_t)ctx->max_smem ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occq, qk->fn, qk->block, smem) !=
                cudaSuccess) {
            cudaGetLastError();
            occq = 0;
        }
        occq = std::min(occq, s->occ_qp_max);
        if (occq <= 0)
            SW_SET(ctx, SW_ERR_UNSUPPORTED, "paired lanes of %u rows do not fit shape %dx%d",
                   L.max_rows, qk->T, qk->R);
        const uint32_t* base = reinterpret_cast<const uint32_t*>(s->d_meta);
        QpArgs q;
        q.db = ctx->d_db;
        q.pairs = s->d_pairs;
        q.pair_begin = s->chunk_begin[chunk];
        q.pair_count = pair_count;
        q.codes = s->d_meta + o_codes;
        q.off_lo = base + o_qpo0 / 4 + L.first;
        q.rows_lo = base + o_qpr0 / 4 + L.first;
        q.off_hi = base + o_qpo1 / 4 + L.first;
        q.rows_hi = base + o_qpr1 / 4 + L.first;
        q.rb_map = reinterpret_cast<const int2*>(s->d_meta + o_qpmap);
        q.rb_off = base + o_qprb / 4 + L.first;
        q.nstacks = (int)L.count;
        q.counters = s->d_counters + ns + 1 + L.first;
        q.mat = ctx->d_mat;
        q.bias2 = (uint32_t)(ctx->params.gap_open + ctx->params.gap_extend);
        q.bias2 |= q.bias2 << 16;
        q.neg_e = (uint32_t)(uint16_t)(int16_t)(-ctx->params.gap_extend);
        q.neg_e |= q.neg_e << 16;
        q.bnd = s->d_bnd;
        q.bnd_group = s->bnd_group;
        q.scores = s->d_scores;
        q.n_records = n_rec;
        q.ovf_list = s->d_ovf;
        q.ovf_count = d_ovf_count;
        q.ovf_thresh = 32767 - std::max(ctx->max_score, 1) + 1;
        q.ovf_cap = (int)std::min<size_t>(s->ovf_cap, (size_t)INT32_MAX);
        q.pair_ids = s->d_pair_ids;
        q.seg_flags = base + o_qpfl / 4 + L.first;
        // a segment's last row for the next segment: per-record boundary rows,
        // one region per double stack of a wave (the serving regions, or the
        // context's own rows when there is one region: the plain search does
        // not run while a round is on the stream)
        q.seg_bnd = s->d_segbnd ? s->d_segbnd : ctx->d_bnd;
        q.seg_slot = base + o_qpsl / 4 + L.first;
        q.seg_stride = s->seg_stride;
        const int cb = s->chunk_begin[chunk];
        q.long_units = qp_long_units([&](int p) { return (uint64_t)s->ring_ncols[(size_t)(cb + p)]; },
                                     pair_count, s->chunk_cols[(size_t)chunk],
                                     (long long)occq * ctx->num_sms * (qk->block / qk->T));
        void* qargs[] = {&q};
        SW_CUDA(ctx, cudaLaunchKernel(qk->fn, dim3((unsigned)(occq * ctx->num_sms)),
                                      dim3(qk->block), qargs, smem, st));
        ++*launches;
    }
    {
        BatchArgs a;
        a.db = ctx->d_db;
        a.pairs = s->d_pairs;
        a.pair_begin = s->chunk_begin[chunk];
        a.pair_count = s->chunk_begin[chunk + 1] - s->chunk_begin[chunk];
        a.codes = s->d_meta + o_codes;
        a.stack_off = reinterpret_cast<const uint32_t*>(s->d_meta + o_soff);
        a.stack_rows = reinterpret_cast<const uint32_t*>(s->d_meta + o_srows);
        a.rb_map = reinterpret_cast<const int*>(s->d_meta + o_rbmap);
        a.rb_off = reinterpret_cast<const uint32_t*>(s->d_meta + o_rboff);
        a.nstacks = (int)ns;
        a.counters = s->d_counters;
        a.mat = ctx->d_mat;
        a.bias2 = (uint32_t)(ctx->params.gap_open + ctx->params.gap_extend);
        a.bias2 |= a.bias2 << 16;
        a.neg_e = (uint32_t)(uint16_t)(int16_t)(-ctx->params.gap_extend);
        a.neg_e |= a.neg_e << 16;
        a.bnd = s->d_bnd;
        a.bnd_group = s->bnd_group;
        a.scores = s->d_scores;
        a.n_records = n_rec;
        a.ovf_list = s->d_ovf;
        a.ovf_count = d_ovf_count;
        a.ovf_thresh = 32767 - std::max(ctx->max_score, 1) + 1;
        a.ovf_cap = (int)std::min<size_t>(s->ovf_cap, (size_t)INT32_MAX);
        a.pair_ids = s->d_pair_ids;
        void* args[] = {&a};
        if (a.pair_count > 0 && ns > 0) {
            SW_CUDA(ctx, cudaLaunchKernel(s->k->batch_fn, dim3((unsigned)(occ * ctx->num_sms)),
                                          dim3(s->k->block), args, s->k->smem((int)max_rows), st));
            ++*launches;
        }
    }
    {
        RescoreArgs r;
        r.db = ctx->d_db;
        r.pairs = ctx->d_pairs;
        r.query = nullptr;
        r.qlen = 0;
        r.queries = s->d_meta + o_codes;
        r.qoff = reinterpret_cast<const uint32_t*>(s->d_meta + o_qoff);
        r.qlens = reinterpret_cast<const uint32_t*>(s->d_meta + o_qlen);
        r.n_records = n_rec;
        r.mat = ctx->d_mat;
        r.gap_oe = ctx->params.gap_open + ctx->params.gap_extend;
        r.gap_e = ctx->params.gap_extend;
        r.ovf_list = s->d_ovf;
        r.ovf_count = d_ovf_count;
        r.ovf_cap = (int)std::min<size_t>(s->ovf_cap, (size_t)INT32_MAX);
        r.scratch = ctx->d_rs_scratch;
        r.max_cols = ctx->max_cols;
        r.scores = s->d_scores;
        void* args[] = {&r};
        SW_CUDA(ctx, cudaLaunchKernel((const void*)sw_rescore32, dim3(kRescoreBlocks), dim3(64),
                                      args, 0, st));
        ++*launches;
    }
    if (!finishing.empty()) {
        const int k = ctx->params.top_k;
        const long long nblk0 = std::max<long long>(1, ((long long)n_rec + kTopkKeys - 1) / kTopkKeys);
        long long n = n_rec, in_stride = n_rec;
        int kb = 0;                // ping-pong between the two device key buffers
        const unsigned long long* keys_in = nullptr;
        bool first = true;
        while (true) {
            const long long blocks = std::max<long long>(1, (n + kTopkKeys - 1) / kTopkKeys);
            TopkArgs t;
            t.scores = s->d_scores;
            t.perm = ctx->d_perm;
            t.keys_in = first ? nullptr : keys_in;
            t.n = n;
            t.k = k;
            t.cap = (ctx->params.flags & SW_FLAG_REFERENCE_CAP) ? 1 : 0;
            t.scores_by_record = nullptr;
            t.keys_out = s->d_keys[kb];
            t.in_stride = in_stride;
            t.rec_stride = 0;
            t.out_stride = nblk0 * kMaxTopK;
            t.rows = reinterpret_cast<const int*>(s->d_meta + o_rows);
            void* args[] = {&t};
            SW_CUDA(ctx, cudaLaunchKernel((const void*)sw_topk_round,
                                          dim3((unsigned)blocks, (unsigned)finishing.size()),
                                          dim3(kTopkThreads), args, 0, st));
            ++*launches;
            keys_in = s->d_keys[kb];
            in_stride = nblk0 * kMaxTopK;
            kb ^= 1;
            first = false;
            if (blocks == 1) break;
            n = blocks * (long long)k;
        }
        SW_CUDA(ctx, cudaMemcpy2DAsync(s->h_keys[buf], (size_t)k * sizeof(unsigned long long), keys_in,
                                       (size_t)(nblk0 * kMaxTopK) * sizeof(unsigned long long),
                                       (size_t)k * sizeof(unsigned long long), finishing.size(),
                                       cudaMemcpyDeviceToHost, st));
    }
    SW_CUDA(ctx, cudaMemcpyAsync(s->h_flagged[buf], d_ovf_count, sizeof(int),
                                 cudaMemcpyDeviceToHost, st));
    SW_CUDA(ctx, cudaEventRecord(s->done_ev[buf], st));
    SW_CUDA(ctx, cudaGetLastError());
    return SW_OK;
}

// Waits for the round enqueued with buffer set `buf` and checks it; returns
// its overflow count in *rescored and its device time in *device_ms (from its
// table upload to its last copy: the stream reaches the round's first
// operation only when the round before has ended, so rounds do not overlap).
sw_status wait_round(sw_ctx* ctx, sw_serve_state* s, int buf, uint64_t* rescored,
                     double* device_ms) {
    SW_CUDA(ctx, cudaEventSynchronize(s->done_ev[buf]));
    SW_CUDA(ctx, cudaGetLastError());
    float ms = 0.f;
    SW_CUDA(ctx, cudaEventElapsedTime(&ms, s->start_ev[buf], s->done_ev[buf]));
    *device_ms = ms;
    const int flagged = *s->h_flagged[buf];
    if ((size_t)flagged > s->ovf_cap)
        SW_SET(ctx, SW_ERR_UNSUPPORTED, "%d overflow entries exceed the list (%zu)", flagged,
               s->ovf_cap);
    *rescored = (uint64_t)flagged;
    return SW_OK;
}

// Requests longer than a stack: one plain search each (its rows split over
// consecutive launches), at a round boundary, on the scheduler thread.
void run_solo(sw_ctx* ctx, sw_serve_state* s, std::vector<Request>& reqs) {
    const int k = ctx->params.top_k;
    std::vector<sw_hit> hits((size_t)std::max(k, 1));
    for (Request& r : reqs) {
        const double t0 = now_ms();
        uint32_t nh = 0;
        const sw_status st = search_host(ctx, r.query.data(), (uint32_t)r.query.size(),
                                         hits.data(), &nh, nullptr);
        const double t1 = now_ms();
        std::lock_guard<std::mutex> lock(s->mu);
        r.start_ms = t0;
        r.done_ms = t1;
        r.status = st;
        ++s->stats.admitted;
        ++s->stats.rounds;
        s->stats.launches += ctx->stats.launches;
        s->stats.rescored += ctx->stats.rescored;
        s->stats.busy_ms += t1 - t0;
        s->stats.device_ms += ctx->stats.kernel_ms;
        if (st == SW_OK) {
            r.hits.assign(hits.begin(), hits.begin() + nh);
            s->stats.cells += (uint64_t)r.query.size() * ctx->n_residues;
            ++s->stats.completed;
        } else {
            ++s->stats.failed;
        }
        s->done.push_back(std::move(r));
        s->cv_done.notify_all();
    }
}

// A round on the device whose results the host has not read yet.
struct InFlight {
    bool valid = false;
    int buf = 0;                      // its host buffer set
    std::vector<Request> leaving;     // requests whose cycle ends with it, in key order
    double t_enq = 0;
};

// Hands out the requests of a completed (or failed) round.  Caller holds mu.
void hand_out(sw_ctx* ctx, sw_serve_state* s, InFlight& r, sw_status st, double t1) {
    const int k = ctx->params.top_k;
    for (size_t f = 0; f < r.leaving.size(); ++f) {
        Request& q = r.leaving[f];
        q.done_ms = t1;
        q.status = st;
        if (st == SW_OK) {
            for (int j = 0; j < k; ++j) {
                const unsigned long long key = s->h_keys[r.buf][f * (size_t)k + j];
                if (key == 0ull) break;
                sw_hit h;
                h.score = (int32_t)(key >> 32);
                h.reserved = 0;
                h.index = 0xffffffffull - (key & 0xffffffffull);
                q.hits.push_back(h);
            }
            s->stats.cells += (uint64_t)q.query.size() * ctx->n_residues;
            ++s->stats.completed;
        } else {
            q.hits.clear();
            ++s->stats.failed;
        }
        s->done.push_back(std::move(q));
    }
    r.leaving.clear();
    r.valid = false;
}

// Fails every request still holding a slot.  Caller holds mu.
void fail_slots(sw_serve_state* s, sw_status st, double t1) {
    for (Slot& x : s->slots) {
        if (!x.used) continue;
        x.req.done_ms = t1;
        x.req.status = st;
        x.req.hits.clear();
        ++s->stats.failed;
        s->done.push_back(std::move(x.req));
        x.req = Request();
        x.used = false;
    }
}

// The scheduler thread.  Rounds are pipelined: round r+1 is enqueued (from the
// slots' state after r, which is known when r is enqueued) before the host
// waits for round r, so the device never idles while the host reads results
// and builds the next round's tables.  A slot whose cycle ends with round r
// is freed when r is enqueued: a request admitted into it clears its score
// row on the stream after r's top-k has read it.
void scheduler(sw_ctx* ctx) {
    sw_serve_state* s = ctx->serve;
    cudaSetDevice(ctx->device);
    std::vector<int> finishing;
    std::vector<Request> solo;
    InFlight prev;
    int next_buf = 0;
    double last_done = 0;
    // waits for a round and hands its requests out; on failure every request
    // in flight fails (the slots' score rows are no longer trustworthy)
    auto complete = [&](InFlight& r) {
        uint64_t rescored = 0;
        double device_ms = 0;
        const sw_status st = wait_round(ctx, s, r.buf, &rescored, &device_ms);
        const double t1 = now_ms();
        {
            std::lock_guard<std::mutex> lock(s->mu);
            s->stats.rescored += rescored;
            s->stats.device_ms += device_ms;
            s->stats.busy_ms += t1 - std::max(r.t_enq, last_done);
            last_done = t1;
            hand_out(ctx, s, r, st, t1);
            if (st != SW_OK) fail_slots(s, st, t1);
        }
        s->cv_done.notify_all();
        return st;
    };
    while (true) {
        {
            std::unique_lock<std::mutex> lock(s->mu);
            bool any = false;
            for (const Slot& x : s->slots) any |= x.used;
            if (!any && !prev.valid)
                s->cv_work.wait(lock, [&] { return s->stopping || !s->pending.empty(); });
            // requests too long for a stack leave the queue for the plain path
            for (auto it = s->pending.begin(); it != s->pending.end();) {
                if (it->query.size() > s->max_stack_rows) {
                    solo.push_back(std::move(*it));
                    it = s->pending.erase(it);
                } else {
                    ++it;
                }
            }
        }
        if (!solo.empty()) {
            if (prev.valid) complete(prev);
            run_solo(ctx, s, solo);
            solo.clear();
            continue;
        }
        bool any = false, stopping = false;
        {
            std::unique_lock<std::mutex> lock(s->mu);
            // admission: free slots take waiting requests, oldest first
            const double t_adm = now_ms();
            for (int i = 0; i < s->n_slots && !s->pending.empty(); ++i) {
                Slot& x = s->slots[i];
                if (x.used) continue;
                x.used = true;
                x.fresh = true;
                x.done_chunks = 0;
                x.req = std::move(s->pending.front());
                s->pending.pop_front();
                x.req.start_ms = t_adm;
                ++s->stats.admitted;
            }
            for (const Slot& x : s->slots) any |= x.used;
            stopping = s->stopping;
        }
        if (!any) {
            if (prev.valid) {
                complete(prev);
                continue;
            }
            if (stopping) break;
            continue;
        }
        InFlight cur;
        cur.valid = true;
        cur.buf = next_buf;
        cur.t_enq = now_ms();
        uint32_t launches = 0;
        const sw_status est = enqueue_round(ctx, s, s->cursor, cur.buf, finishing, &launches);
        {
            std::lock_guard<std::mutex> lock(s->mu);
            if (est == SW_OK) {
                ++s->stats.rounds;
                s->stats.launches += launches;
                for (int f : finishing) {
                    Slot& x = s->slots[(size_t)f];
                    cur.leaving.push_back(std::move(x.req));
                    x.req = Request();
                    x.used = false;
                }
                for (Slot& x : s->slots)
                    if (x.used) {
                        x.fresh = false;
                        ++x.done_chunks;
                    }
                s->cursor = (s->cursor + 1) % s->n_chunks;
            }
        }
        if (est != SW_OK) {
            cudaStreamSynchronize(ctx->stream);
            cudaGetLastError();
            const double t1 = now_ms();
            {
                std::lock_guard<std::mutex> lock(s->mu);
                if (prev.valid) hand_out(ctx, s, prev, est, t1);
                fail_slots(s, est, t1);
            }
            s->cv_done.notify_all();
            continue;
        }
        next_buf ^= 1;
        if (prev.valid && complete(prev) != SW_OK) {
            // the round just enqueued ran on failed state: drop it too
            cudaEventSynchronize(s->done_ev[cur.buf]);
            cudaGetLastError();
            {
                std::lock_guard<std::mutex> lock(s->mu);
                hand_out(ctx, s, cur, SW_ERR_CUDA, now_ms());
            }
            s->cv_done.notify_all();
            continue;
        }
        prev = std::move(cur);
    }
}

}  // namespace

namespace swb {

void serve_teardown(sw_ctx* ctx) {
    sw_serve_state* s = ctx->serve;
    if (!s) return;
    {
        std::lock_guard<std::mutex> lock(s->mu);
        s->stopping = true;
        // waiting requests are dropped; requests in flight finish their cycle
        s->pending.clear();
    }
    s->cv_work.notify_all();
    if (s->th.joinable()) s->th.join();
    serve_free(s);
    delete s;
    ctx->serve = nullptr;
}

}  // namespace swb

extern "C" void sw_serve_options_default(sw_serve_options* o) {
    if (!o) return;
    o->max_active = 128;
    o->chunks = 4;
    o->max_pending = 0;
    o->memory_budget = 0;
    o->group_width = 16;
    o->rows_per_thread = 64;
    o->stack_rows = 4096;
    o->pair_rows = 2048;
    o->pair_group_width = 16;
    o->pair_rows_per_thread = 64;
    o->pair_long = 1;
    o->pair_regions = 0;
}

extern "C" sw_status sw_serve_start(sw_ctx* ctx, const sw_serve_options* opt) {
    if (!ctx) return SW_ERR_INVALID;
    if (ctx->serve) SW_SET(ctx, SW_ERR_STATE, "already serving");
    if (!ctx->db_loaded) SW_SET(ctx, SW_ERR_STATE, "no DB loaded (call sw_db_load first)");
    SW_CUDA(ctx, cudaSetDevice(ctx->device));
    sw_serve_options o;
    sw_serve_options_default(&o);
    if (opt) o = *opt;
    const WfKernel* k = find_kernel(o.group_width, o.rows_per_thread);
    const QpKernel* qk = o.pair_rows > 0 ? find_qp(o.pair_group_width, o.pair_rows_per_thread)
                                         : nullptr;
    if (!k || o.max_active == 0 || o.chunks == 0 || o.stack_rows < 0 || o.pair_rows < 0 ||
        o.pair_regions < 0 ||
        (o.pair_rows > 0 && !qk))
        SW_SET(ctx, SW_ERR_INVALID, "bad serving options");
    // the tallest stack the shape holds (whole passes whose profile fits one
    // block); it must hold the configured stack height
    const int max_stack_rows = launch_rows(ctx, *k, 1 << 30);
    if (max_stack_rows < std::max(o.stack_rows, k->R))
        SW_SET(ctx, SW_ERR_UNSUPPORTED, "shape %dx%d cannot hold a stack of %d rows",
               o.group_width, o.rows_per_thread, std::max(o.stack_rows, k->R));
    const int n_rec = (int)ctx->n_records;
    if ((uint64_t)o.max_active * (uint64_t)std::max(n_rec, 1) >= (1ull << 31))
        SW_SET(ctx, SW_ERR_UNSUPPORTED, "max_active x records reaches 2^31");
    // slots: at most max_active, and as many as the memory budget holds at one
    // score row plus its share of the key buffers each
    const long long nblk0 = std::max<long long>(1, ((long long)n_rec + kTopkKeys - 1) / kTopkKeys);
    const size_t per_slot = (size_t)std::max(n_rec, 1) * 4 + 2 * (size_t)nblk0 * kMaxTopK * 8 +
                            (size_t)ctx->params.top_k * 8;
    size_t free_b = 0, total_b = 0;
    SW_CUDA(ctx, cudaMemGetInfo(&free_b, &total_b));
    const size_t budget = o.memory_budget ? (size_t)o.memory_budget : free_b / 2;
    if (budget / per_slot == 0)
        SW_SET(ctx, SW_ERR_NOMEM, "the memory budget (%zu bytes) holds no request (%zu bytes each)",
               budget, per_slot);
    sw_serve_state* s = new sw_serve_state();
    s->opt = o;
    s->k = k;
    s->n_slots = (int)std::min<size_t>(o.max_active, budget / per_slot);
    s->max_stack_rows = (uint32_t)max_stack_rows;
    s->occ_max = shape_occupancy(ctx, *k, k->R);
    if (qk) {
        const uint32_t pass_rows = (uint32_t)(qk->T * qk->R);
        s->pair_seg = std::max(pass_rows, (uint32_t)o.pair_rows / pass_rows * pass_rows);
        int occq = 0;
        const size_t smem_seg = qk->smem((int)s->pair_seg);
        if (smem_seg > (size_t)ctx->max_smem ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occq, qk->fn, qk->block, smem_seg) !=
                cudaSuccess ||
            occq <= 0) {
            cudaGetLastError();
            const unsigned seg = s->pair_seg;
            delete s;
            SW_SET(ctx, SW_ERR_UNSUPPORTED, "paired shape %dx%d cannot hold a lane of %u rows",
                   qk->T, qk->R, seg);
        }
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&s->occ_qp_max, qk->fn, qk->block,
                                                      qk->smem(qk->T * qk->R));
        s->qk = qk;
    }
    const int64_t npairs = ctx->n_pairs;
    s->n_chunks = (int)std::max<int64_t>(1, std::min<int64_t>(o.chunks, std::max<int64_t>(npairs, 1)));
    auto fail = [&](const char* what) {
        serve_free(s);
        delete s;
        ctx->err = std::string("device allocation failed: serving ") + what;
        return SW_ERR_NOMEM;
    };
    // the ring: pairs dealt round-robin (every n_chunks-th pair of the
    // length-sorted order) and stored chunk after chunk
    std::vector<Pair2> host_pairs((size_t)npairs);
    if (npairs && cudaMemcpy(host_pairs.data(), ctx->d_pairs, (size_t)npairs * sizeof(Pair2),
                             cudaMemcpyDeviceToHost) != cudaSuccess)
        return fail("pair ring");
    std::vector<Pair2> ring;
    std::vector<uint32_t> ids;
    ring.reserve((size_t)npairs);
    ids.reserve((size_t)npairs);
    s->chunk_begin.assign(1, 0);
    for (int c = 0; c < s->n_chunks; ++c) {
        uint64_t cols = 0;
        for (int64_t p = c; p < npairs; p += s->n_chunks) {
            ring.push_back(host_pairs[(size_t)p]);
            ids.push_back((uint32_t)p);
            s->ring_ncols.push_back(host_pairs[(size_t)p].ncols);
            cols += host_pairs[(size_t)p].ncols;
        }
        s->chunk_begin.push_back((int)ring.size());
        s->chunk_cols.push_back(cols);
    }
    if (dev_alloc(&s->d_pairs, ring.size()) != cudaSuccess ||
        dev_alloc(&s->d_pair_ids, ids.size()) != cudaSuccess)
        return fail("pair ring");
    if (!ring.empty() &&
        (cudaMemcpy(s->d_pairs, ring.data(), ring.size() * sizeof(Pair2), cudaMemcpyHostToDevice) !=
             cudaSuccess ||
         cudaMemcpy(s->d_pair_ids, ids.data(), ids.size() * 4, cudaMemcpyHostToDevice) != cudaSuccess))
        return fail("pair ring");
    if (dev_alloc(&s->d_scores, (size_t)s->n_slots * std::max(n_rec, 1)) != cudaSuccess ||
        dev_alloc(&s->d_counters, 6 * (size_t)s->n_slots + 16) != cudaSuccess)
        return fail("slots");
    // overflow entries: one per (request, record) at worst, bounded
    s->ovf_cap = std::min<size_t>((size_t)s->n_slots * std::max(n_rec, 1),
                                  std::max<size_t>((size_t)4 * std::max(n_rec, 1), (size_t)1 << 22));
    if (dev_alloc(&s->d_ovf, s->ovf_cap) != cudaSuccess) return fail("overflow list");
    if (dev_alloc(&s->d_keys[0], (size_t)s->n_slots * nblk0 * kMaxTopK) != cudaSuccess ||
        dev_alloc(&s->d_keys[1], (size_t)s->n_slots * nblk0 * kMaxTopK) != cudaSuccess)
        return fail("key buffers");
    s->bnd_group = 2 * (size_t)std::max(ctx->max_cols, 8);
    size_t groups = (size_t)std::max(s->occ_max, 1) * ctx->num_sms * (k->block / k->T);
    if (qk)
        groups = std::max(groups, (size_t)std::max(s->occ_qp_max, 1) * ctx->num_sms *
                                      (qk->block / qk->T));
    if (dev_alloc(&s->d_bnd, groups * s->bnd_group) != cudaSuccess) return fail("boundary rows");
    if (qk && o.pair_long) {
        // boundary regions (copies of the per-record rows, 8 bytes per column
        // of every record) so that tall double stacks' segments share
        // launches: pair_regions of them (0: up to 16), as many as fit in an
        // eighth of the free memory.  Few regions split the tall stacks into
        // waves of short launches, and each launch ends in a tail where the
        // last long records finish on a few SMs.
        const size_t stride = (size_t)ctx->db_units * 16;
        size_t fb = 0, tb = 0;
        if (cudaMemGetInfo(&fb, &tb) != cudaSuccess) cudaGetLastError();
        const size_t fit = stride ? fb / 8 / (stride * sizeof(uint2)) : 0;
        const int n = (int)std::min<size_t>(o.pair_regions > 0 ? (size_t)o.pair_regions : 16, fit);
        if (n > 1 && dev_alloc(&s->d_segbnd, (size_t)n * stride) == cudaSuccess) {
            s->seg_regions = n;
            s->seg_stride = stride;
        } else {
            cudaGetLastError();
            s->d_segbnd = nullptr;
        }
    }
    for (int b = 0; b < 2; ++b) {
        if (cudaMallocHost((void**)&s->h_keys[b],
                           (size_t)s->n_slots * ctx->params.top_k * sizeof(unsigned long long)) !=
                cudaSuccess ||
            cudaMallocHost((void**)&s->h_flagged[b], sizeof(int)) != cudaSuccess)
            return fail("pinned keys");
        if (cudaEventCreate(&s->done_ev[b]) != cudaSuccess ||
            cudaEventCreate(&s->start_ev[b]) != cudaSuccess)
            return fail("round events");
    }
    // stacks (at most one per slot), the overflow count, and paired entries
    // (a lane of at most max_stack_rows rows has at most that / pair_seg
    // segments; two lanes per double stack)
    s->counters_cap = 6 * (size_t)s->n_slots + 16;
    s->slots.assign((size_t)s->n_slots, Slot());
    s->stats.slots = (uint32_t)s->n_slots;
    s->stats.chunks = (uint32_t)s->n_chunks;
    ctx->serve = s;
    s->th = std::thread(scheduler, ctx);
    return SW_OK;
}

extern "C" sw_status sw_serve_submit(sw_ctx* ctx, uint64_t request_id, const uint8_t* query,
                                     uint32_t qlen) {
    if (!ctx || (qlen && !query)) return SW_ERR_INVALID;
    sw_serve_state* s = ctx->serve;
    if (!s) return SW_ERR_STATE;
    if (qlen == 0 || qlen > kServeMaxQuery) return SW_ERR_UNSUPPORTED;
    for (uint32_t i = 0; i < qlen; ++i)
        if (query[i] > 24) return SW_ERR_INVALID;
    Request r;
    r.id = request_id;
    r.query.assign(query, query + qlen);
    r.submit_ms = now_ms();
    {
        std::lock_guard<std::mutex> lock(s->mu);
        if (s->stopping) return SW_ERR_STATE;
        if (s->opt.max_pending && s->pending.size() >= s->opt.max_pending) return SW_ERR_BUSY;
        s->pending.push_back(std::move(r));
        ++s->stats.submitted;
    }
    s->cv_work.notify_one();
    return SW_OK;
}

extern "C" sw_status sw_serve_poll(sw_ctx* ctx, uint32_t max_results, sw_serve_result* results,
                                   sw_hit* hits, uint32_t* n_results, int32_t timeout_ms) {
    if (!ctx || !n_results || (max_results && (!results || !hits))) return SW_ERR_INVALID;
    *n_results = 0;
    sw_serve_state* s = ctx->serve;
    if (!s) return SW_ERR_STATE;
    std::unique_lock<std::mutex> lock(s->mu);
    if (s->done.empty() && timeout_ms != 0) {
        auto ready = [&] { return !s->done.empty(); };
        if (timeout_ms < 0)
            s->cv_done.wait(lock, ready);
        else
            s->cv_done.wait_for(lock, std::chrono::milliseconds(timeout_ms), ready);
    }
    const int k = ctx->params.top_k;
    uint32_t n = 0;
    while (n < max_results && !s->done.empty()) {
        Request& r = s->done.front();
        results[n].request_id = r.id;
        results[n].status = (int32_t)r.status;
        results[n].n_hits = (uint32_t)r.hits.size();
        results[n].submit_ms = r.submit_ms;
        results[n].start_ms = r.start_ms;
        results[n].done_ms = r.done_ms;
        for (int j = 0; j < k; ++j)
            hits[(size_t)n * k + j] = j < (int)r.hits.size() ? r.hits[(size_t)j] : sw_hit{0, 0, 0};
        s->done.pop_front();
        ++n;
    }
    *n_results = n;
    return SW_OK;
}

extern "C" sw_status sw_serve_get_stats(sw_ctx* ctx, sw_serve_stats* out) {
    if (!ctx || !out) return SW_ERR_INVALID;
    sw_serve_state* s = ctx->serve;
    if (!s) return SW_ERR_STATE;
    std::lock_guard<std::mutex> lock(s->mu);
    *out = s->stats;
    out->pending = (uint32_t)s->pending.size();
    uint32_t active = 0;
    for (const Slot& x : s->slots) active += x.used ? 1u : 0u;
    out->active = active;
    return SW_OK;
}

extern "C" double sw_serve_clock_ms(void) { return now_ms(); }

extern "C" sw_status sw_serve_stop(sw_ctx* ctx) {
    if (!ctx) return SW_ERR_INVALID;
    if (!ctx->serve) return SW_ERR_STATE;
    serve_teardown(ctx);
    return SW_OK;
}
