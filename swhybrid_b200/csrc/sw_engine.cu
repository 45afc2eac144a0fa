// sw_engine.cu -- host side of libswb200: context, resident DB layout, kernel
// shape selection and the plain search sequence behind the C ABI (swb200.h).
//
// Reference flow this replaces (SWhybrid, CUDA build): per query and per
// 256 MB chunk, DataPool::fillChunk reads batches from disk, CUDAWorker::packDB
// re-packs them on the host, asyncCopy ships the whole chunk over PCIe,
// kernelLaunch runs, and a synchronous cudaMemcpy brings the scores back
// (src/Worker.cpp:175-200, src/CUDAWorker.cu:144-246); overflowed records are
// re-scored on the host afterwards (src/RecalcWorker.cpp:99-268) and top-k is
// merged by list insertion (src/ResultList.h:37-79).
//
// Here the DB is laid out once (sorted by length, paired, column-interleaved)
// and stays in HBM; a search is: query H2D (a few KB), first-pass kernel(s),
// 32-bit re-score of the flagged records, device top-k, D2H of k hits.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <iterator>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/swb200.h"
#include "sw_aux.h"
#include "sw_device.cuh"
#include "sw_engine.h"
#include "sw_long.h"
#include "sw_tuned_default.h"
#include "sw_registry.h"

namespace swb {
extern const WfKernel wf_table_t4[];
extern const int wf_table_t4_n;
extern const WfKernel wf_table_t8[];
extern const int wf_table_t8_n;
extern const WfKernel wf_table_t16[];
extern const int wf_table_t16_n;
extern const WfKernel wf_table_t32[];
extern const int wf_table_t32_n;

const WfKernel* wf_kernels(int* n) {
    static std::vector<WfKernel> all;
    static std::once_flag once;
    std::call_once(once, [] {
        auto add = [](const WfKernel* t, int m) { all.insert(all.end(), t, t + m); };
        add(wf_table_t4, wf_table_t4_n);
        add(wf_table_t8, wf_table_t8_n);
        add(wf_table_t16, wf_table_t16_n);
        add(wf_table_t32, wf_table_t32_n);
    });
    *n = (int)all.size();
    return all.data();
}

const WfKernel* find_kernel(int T, int R) {
    int n = 0;
    const WfKernel* k = wf_kernels(&n);
    for (int i = 0; i < n; ++i)
        if (k[i].T == T && k[i].R == R) return &k[i];
    return nullptr;
}

}  // namespace swb

using namespace swb;

namespace {

double now_ms() {
    return std::chrono::duration<double, std::milli>(
               std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

}  // namespace

// ---------------------------------------------------------------------------
// parameters and encoding
// ---------------------------------------------------------------------------

// BLOSUM62 in the reference's code order (A B C D E F G H I K L M N P Q R S T
// V W X Y Z), the table of src/Param.h:8-51.  Rows/columns 23..31 are zero.
static const int8_t kBlosum62[23][23] = {
    {4, -2, 0, -2, -1, -2, 0, -2, -1, -1, -1, -1, -2, -1, -1, -1, 1, 0, 0, -3, 0, -2, -1},
    {-2, 4, -3, 4, 1, -3, -1, 0, -3, 0, -4, -3, 3, -2, 0, -1, 0, -1, -3, -4, -1, -3, 1},
    {0, -3, 9, -3, -4, -2, -3, -3, -1, -3, -1, -1, -3, -3, -3, -3, -1, -1, -1, -2, -2, -2, -3},
    {-2, 4, -3, 6, 2, -3, -1, -1, -3, -1, -4, -3, 1, -1, 0, -2, 0, -1, -3, -4, -1, -3, 1},
    {-1, 1, -4, 2, 5, -3, -2, 0, -3, 1, -3, -2, 0, -1, 2, 0, 0, -1, -2, -3, -1, -2, 4},
    {-2, -3, -2, -3, -3, 6, -3, -1, 0, -3, 0, 0, -3, -4, -3, -3, -2, -2, -1, 1, -1, 3, -3},
    {0, -1, -3, -1, -2, -3, 6, -2, -4, -2, -4, -3, 0, -2, -2, -2, 0, -2, -3, -2, -1, -3, -2},
    {-2, 0, -3, -1, 0, -1, -2, 8, -3, -1, -3, -2, 1, -2, 0, 0, -1, -2, -3, -2, -1, 2, 0},
    {-1, -3, -1, -3, -3, 0, -4, -3, 4, -3, 2, 1, -3, -3, -3, -3, -2, -1, 3, -3, -1, -1, -3},
    {-1, 0, -3, -1, 1, -3, -2, -1, -3, 5, -2, -1, 0, -1, 1, 2, 0, -1, -2, -3, -1, -2, 1},
    {-1, -4, -1, -4, -3, 0, -4, -3, 2, -2, 4, 2, -3, -3, -2, -2, -2, -1, 1, -2, -1, -1, -3},
    {-1, -3, -1, -3, -2, 0, -3, -2, 1, -1, 2, 5, -2, -2, 0, -1, -1, -1, 1, -1, -1, -1, -1},
    {-2, 3, -3, 1, 0, -3, 0, 1, -3, 0, -3, -2, 6, -2, 0, 0, 1, 0, -3, -4, -1, -2, 0},
    {-1, -2, -3, -1, -1, -4, -2, -2, -3, -1, -3, -2, -2, 7, -1, -2, -1, -1, -2, -4, -2, -3, -1},
    {-1, 0, -3, 0, 2, -3, -2, 0, -3, 1, -2, 0, 0, -1, 5, 1, 0, -1, -2, -2, -1, -1, 3},
    {-1, -1, -3, -2, 0, -3, -2, 0, -3, 2, -2, -1, 0, -2, 1, 5, -1, -1, -3, -3, -1, -2, 0},
    {1, 0, -1, 0, 0, -2, 0, -1, -2, 0, -2, -1, 1, -1, 0, -1, 4, 1, -2, -3, 0, -2, 0},
    {0, -1, -1, -1, -1, -2, -2, -2, -1, -1, -1, -1, 0, -1, -1, -1, 1, 5, 0, -2, 0, -2, -1},
    {0, -3, -1, -3, -2, -1, -3, -3, 3, -2, 1, 1, -3, -2, -2, -3, -2, 0, 4, -3, -1, -1, -2},
    {-3, -4, -2, -4, -3, 1, -2, -2, -3, -3, -2, -1, -4, -4, -2, -3, -3, -2, -3, 11, -2, 2, -3},
    {0, -1, -2, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -2, -1, -1, 0, 0, -1, -2, -1, -1, -1},
    {-2, -3, -2, -3, -2, 3, -3, 2, -1, -2, -1, -1, -2, -3, -1, -2, -2, -2, -1, 2, -1, 7, -2},
    {-1, 1, -3, 1, 4, -3, -2, 0, -3, 1, -3, -1, 0, -1, 3, 0, 0, -1, -2, -3, -1, -2, 4},
};

extern "C" void sw_params_default(sw_params* p) {
    if (!p) return;
    memset(p, 0, sizeof(*p));
    for (int i = 0; i < 23; ++i)
        for (int j = 0; j < 23; ++j) p->matrix[i * 32 + j] = kBlosum62[i][j];
    p->gap_open = 10;
    p->gap_extend = 2;
    p->top_k = 10;
    p->flags = SW_FLAG_REFERENCE_CAP;
}

extern "C" sw_status sw_encode(const char* letters, uint64_t n, uint8_t* codes) {
    if ((!letters || !codes) && n) return SW_ERR_INVALID;
    static const char* alpha = "ABCDEFGHIKLMNPQRSTVWXYZ";
    uint8_t tab[256];
    memset(tab, kZeroCode, sizeof(tab));
    for (int i = 0; alpha[i]; ++i) {
        tab[(uint8_t)alpha[i]] = (uint8_t)i;
        tab[(uint8_t)(alpha[i] - 'A' + 'a')] = (uint8_t)i;
    }
    tab[(uint8_t)'@'] = 23;
    for (uint64_t i = 0; i < n; ++i) codes[i] = tab[(uint8_t)letters[i]];
    return SW_OK;
}

// ---------------------------------------------------------------------------
// context
// ---------------------------------------------------------------------------

extern "C" const char* sw_last_error(const sw_ctx* ctx) {
    return ctx ? ctx->err.c_str() : swb::thread_error();
}

static sw_status validate_params(sw_ctx* ctx, const sw_params* p) {
    if (p->gap_open < 0 || p->gap_extend < 0 || p->gap_open + p->gap_extend > 1000)
        SW_SET(ctx, SW_ERR_INVALID, "gap costs out of range (open %d, extend %d)", p->gap_open,
               p->gap_extend);
    if (p->top_k < 1 || p->top_k > kMaxTopK)
        SW_SET(ctx, SW_ERR_INVALID, "top_k %d outside 1..%d", p->top_k, kMaxTopK);
    for (int i = 0; i < 1024; ++i)
        if (p->matrix[i] < -127 || p->matrix[i] > 127)
            SW_SET(ctx, SW_ERR_INVALID, "matrix entry %d = %d outside -127..127", i,
                   p->matrix[i]);
    return SW_OK;
}

extern "C" sw_status sw_ctx_create(int device, const sw_params* params, sw_ctx** out) {
    if (!out) return SW_ERR_INVALID;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return SW_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= ndev) return SW_ERR_INVALID;
    sw_ctx* ctx = new sw_ctx();
    ctx->device = device;
    if (params) ctx->params = *params;
    else sw_params_default(&ctx->params);
    sw_status st = validate_params(ctx, &ctx->params);
    if (st != SW_OK) {
        delete ctx;
        return st;
    }
    auto fail = [&](sw_status s) {
        cudaGetLastError();     // a refused call must not surface in the caller's next one
        sw_ctx_destroy(ctx);
        return s;
    };
    if (cudaSetDevice(device) != cudaSuccess) return fail(SW_ERR_CUDA);
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return fail(SW_ERR_CUDA);
    ctx->num_sms = prop.multiProcessorCount;
    ctx->max_smem = (int)prop.sharedMemPerBlockOptin;
    ctx->regs_per_sm = prop.regsPerMultiprocessor;
    if (cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking) != cudaSuccess)
        return fail(SW_ERR_CUDA);
    ctx->stream = ctx->own_stream;
    ctx->tuning.assign(std::begin(kDefaultTuning), std::end(kDefaultTuning));
    if (cudaStreamCreateWithFlags(&ctx->side_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&ctx->fork_ev, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&ctx->join_ev, cudaEventDisableTiming) != cudaSuccess)
        return fail(SW_ERR_CUDA);
    for (auto& e : ctx->ev)
        if (cudaEventCreate(&e) != cudaSuccess) return fail(SW_ERR_CUDA);
    // matrix: int8 copy; codes >= 24 (zero code, pads) score 0
    int8_t mat8[1024];
    int hi = 0;
    for (int i = 0; i < 32; ++i)
        for (int j = 0; j < 32; ++j) {
            int v = (i >= kZeroCode || j >= kZeroCode) ? 0 : ctx->params.matrix[i * 32 + j];
            mat8[i * 32 + j] = (int8_t)v;
            hi = std::max(hi, v);
        }
    ctx->max_score = hi;
    if (dev_alloc(&ctx->d_mat, 1024) != cudaSuccess) return fail(SW_ERR_NOMEM);
    if (cudaMemcpy(ctx->d_mat, mat8, 1024, cudaMemcpyHostToDevice) != cudaSuccess)
        return fail(SW_ERR_CUDA);
    if (dev_alloc(&ctx->d_counters, 16) != cudaSuccess) return fail(SW_ERR_NOMEM);
    // every first-pass kernel may use the opt-in shared-memory maximum, less
    // what it holds statically (the long-pair kernels hold a few words)
    auto allow_smem = [&](const void* fn) {
        cudaFuncAttributes fa;
        return cudaFuncGetAttributes(&fa, fn) == cudaSuccess &&
               cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    ctx->max_smem - (int)fa.sharedSizeBytes) == cudaSuccess;
    };
    int nk = 0;
    const WfKernel* ks = wf_kernels(&nk);
    for (int i = 0; i < nk; ++i)
        if (!allow_smem(ks[i].fn) || !allow_smem(ks[i].batch_fn)) return fail(SW_ERR_CUDA);
    const QpKernel* qks = qp_kernels(&nk);
    for (int i = 0; i < nk; ++i)
        if (!allow_smem(qks[i].fn)) return fail(SW_ERR_CUDA);
    const LongKernel* lks = long_kernels(&nk);
    for (int i = 0; i < nk; ++i)
        if (!allow_smem(lks[i].fn)) return fail(SW_ERR_CUDA);
    *out = ctx;
    return SW_OK;
}

static void free_db(sw_ctx* ctx) {
    swb::free_batch(ctx);
    swb::free_traceback(ctx);
    swb::free_image(ctx);
    ctx->rec_pos.clear();
    ctx->rec_len.clear();
    dev_free(ctx->d_rs_scratch);
    dev_free(ctx->d_db);
    dev_free(ctx->d_pairs);
    dev_free(ctx->d_perm);
    dev_free(ctx->d_bnd);
    dev_free(ctx->d_scores);
    dev_free(ctx->d_scores_rec);
    dev_free(ctx->d_ovf);
    dev_free(ctx->d_keys[0]);
    dev_free(ctx->d_keys[1]);
    ctx->n_records = 0;
    ctx->n_pairs = 0;
    ctx->pair_ncols.clear();
    ctx->pair_prefix.clear();
    ctx->db_loaded = false;
}

extern "C" sw_status sw_ctx_destroy(sw_ctx* ctx) {
    if (!ctx) return SW_ERR_INVALID;
    cudaSetDevice(ctx->device);
    serve_teardown(ctx);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    if (ctx->own_stream) cudaStreamSynchronize(ctx->own_stream);
    if (ctx->side_stream) cudaStreamSynchronize(ctx->side_stream);
    free_db(ctx);
    dev_free(ctx->d_mat);
    dev_free(ctx->d_counters);
    dev_free(ctx->d_query);
    if (ctx->h_query) cudaFreeHost(ctx->h_query);
    if (ctx->h_keys) cudaFreeHost(ctx->h_keys);
    for (auto& e : ctx->ev)
        if (e) cudaEventDestroy(e);
    for (auto* v : {&ctx->pending, &ctx->spare})
        for (auto& m : *v)
            for (auto& e : m.e) cudaEventDestroy(e);
    if (ctx->fork_ev) cudaEventDestroy(ctx->fork_ev);
    if (ctx->join_ev) cudaEventDestroy(ctx->join_ev);
    if (ctx->side_stream) cudaStreamDestroy(ctx->side_stream);
    if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
    delete ctx;
    return SW_OK;
}

// ---------------------------------------------------------------------------
// database layout
// ---------------------------------------------------------------------------

extern "C" sw_status sw_db_load(sw_ctx* ctx, const uint8_t* residues, const uint64_t* offsets,
                                uint64_t n) {
    return swb::db_load(ctx, residues, offsets, n, nullptr);
}

// The layout build behind sw_db_load and sw_db_load_image.  `given_order`
// (optional) is the length order stored in a DB image: used after checking
// that it is the stable longest-first permutation.
sw_status swb::db_load(sw_ctx* ctx, const uint8_t* residues, const uint64_t* offsets, uint64_t n,
                       const uint32_t* given_order) {
    if (!ctx) return SW_ERR_INVALID;
    if (ctx->serve) return SW_ERR_BUSY;   // the serving loop owns the stream and the DB
    if (!offsets || (n && !residues && offsets[n] != offsets[0]))
        SW_SET(ctx, SW_ERR_INVALID, "null residues/offsets");
    if (n >= (1ull << 31)) SW_SET(ctx, SW_ERR_UNSUPPORTED, "too many records (%llu)",
                                  (unsigned long long)n);
    SW_CUDA(ctx, cudaSetDevice(ctx->device));
    SW_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    free_db(ctx);
    std::vector<uint32_t> len(n);
    uint64_t total = 0, maxlen = 0;
    for (uint64_t i = 0; i < n; ++i) {
        if (offsets[i + 1] < offsets[i]) SW_SET(ctx, SW_ERR_INVALID, "offsets not monotone at %llu",
                                                (unsigned long long)i);
        const uint64_t l = offsets[i + 1] - offsets[i];
        if (l >= (1ull << 30)) SW_SET(ctx, SW_ERR_UNSUPPORTED, "record %llu too long",
                                      (unsigned long long)i);
        len[i] = (uint32_t)l;
        total += l;
        maxlen = std::max<uint64_t>(maxlen, l);
    }
    const uint8_t* base = residues ? residues + offsets[0] : nullptr;
    for (uint64_t i = 0; i < total; ++i)
        if (base[i] > 24) SW_SET(ctx, SW_ERR_INVALID, "residue code %d at %llu (codes are 0..24)",
                                 base[i], (unsigned long long)i);
    // sort by length (longest first), stable in record order
    std::vector<uint32_t> order(n);
    if (given_order) {
        std::vector<bool> seen(n, false);
        for (uint64_t k = 0; k < n; ++k) {
            const uint32_t r = given_order[k];
            bool ok = r < n && !seen[r];
            if (ok && k > 0) {
                const uint32_t p = given_order[k - 1];
                ok = len[p] > len[r] || (len[p] == len[r] && p < r);
            }
            if (!ok) SW_SET(ctx, SW_ERR_FORMAT, "stored length order is not the stable "
                                               "longest-first permutation (entry %llu)",
                            (unsigned long long)k);
            seen[r] = true;
            order[k] = r;
        }
    } else {
        std::iota(order.begin(), order.end(), 0u);
        std::stable_sort(order.begin(), order.end(),
                         [&](uint32_t a, uint32_t b) { return len[a] > len[b]; });
    }
    const uint64_t npairs_all = (n + 1) / 2;
    std::vector<Pair2> pairs(npairs_all);
    uint64_t units = 0, nonempty = 0;
    for (uint64_t p = 0; p < npairs_all; ++p) {
        const uint32_t nc = len[order[2 * p]];
        pairs[p].off16 = (uint32_t)units;
        pairs[p].ncols = nc;
        units += (nc + 7) / 8;
        if (nc > 0) nonempty = p + 1;
        if (units >= (1ull << 32)) SW_SET(ctx, SW_ERR_UNSUPPORTED, "DB too large for 32-bit unit offsets");
    }
    int max_cols = 8;
    for (uint64_t p = 0; p < npairs_all; ++p)
        max_cols = std::max(max_cols, (int)((pairs[p].ncols + 7) / 8 * 8));
    std::vector<uint8_t> stream((size_t)units * 16, (uint8_t)kZeroCode);
    for (uint64_t p = 0; p < npairs_all; ++p) {
        uint8_t* dst = stream.data() + (size_t)pairs[p].off16 * 16;
        for (int lane = 0; lane < 2; ++lane) {
            const uint64_t k = 2 * p + lane;
            if (k >= n) break;
            const uint32_t r = order[k];
            const uint8_t* src = base + (offsets[r] - offsets[0]);
            for (uint32_t c = 0; c < len[r]; ++c) dst[2 * (size_t)c + lane] = src[c];
        }
    }
    std::vector<uint32_t> perm(n);
    for (uint64_t k = 0; k < n; ++k) perm[k] = order[k];
    ctx->rec_pos.assign(n, 0u);
    for (uint64_t k = 0; k < n; ++k) ctx->rec_pos[order[k]] = (uint32_t)k;
    ctx->rec_len = len;

    ctx->n_records = (int64_t)n;
    ctx->n_pairs = (int64_t)nonempty;
    ctx->n_residues = total;
    ctx->max_len = maxlen;
    ctx->units = units;
    ctx->pair_ncols.resize(nonempty);
    ctx->pair_prefix.assign(nonempty + 1, 0u);
    ctx->pair_cols_total = 0;
    for (uint64_t p = 0; p < nonempty; ++p) {
        ctx->pair_ncols[p] = pairs[p].ncols;
        ctx->pair_cols_total += pairs[p].ncols;
        ctx->pair_prefix[p + 1] = ctx->pair_cols_total;
    }
    auto nomem = [&](const char* what) {
        free_db(ctx);
        ctx->err = std::string("device allocation failed: ") + what;
        return SW_ERR_NOMEM;
    };
    if (dev_alloc(&ctx->d_db, units) != cudaSuccess) return nomem("db");
    if (dev_alloc(&ctx->d_pairs, npairs_all) != cudaSuccess) return nomem("pairs");
    if (dev_alloc(&ctx->d_perm, n) != cudaSuccess) return nomem("perm");
    if (dev_alloc(&ctx->d_bnd, units * 16) != cudaSuccess) return nomem("boundary rows");
    ctx->db_units = (uint64_t)units;
    if (dev_alloc(&ctx->d_scores, n + 1) != cudaSuccess) return nomem("scores");
    if (dev_alloc(&ctx->d_scores_rec, n + 1) != cudaSuccess) return nomem("scores");
    if (dev_alloc(&ctx->d_ovf, n + 1) != cudaSuccess) return nomem("overflow list");
    ctx->max_cols = max_cols;
    if (dev_alloc(&ctx->d_rs_scratch, (size_t)kRescoreWarps * max_cols) != cudaSuccess)
        return nomem("re-score rows");
    const size_t nblk = (n + kTopkKeys - 1) / kTopkKeys + 1;
    if (dev_alloc(&ctx->d_keys[0], nblk * kMaxTopK) != cudaSuccess) return nomem("keys");
    if (dev_alloc(&ctx->d_keys[1], nblk * kMaxTopK) != cudaSuccess) return nomem("keys");
    if (!stream.empty())
        SW_CUDA(ctx, cudaMemcpy(ctx->d_db, stream.data(), stream.size(), cudaMemcpyHostToDevice));
    if (npairs_all)
        SW_CUDA(ctx, cudaMemcpy(ctx->d_pairs, pairs.data(), npairs_all * sizeof(Pair2),
                                cudaMemcpyHostToDevice));
    if (n) SW_CUDA(ctx, cudaMemcpy(ctx->d_perm, perm.data(), n * sizeof(uint32_t),
                                   cudaMemcpyHostToDevice));
    ctx->db_bytes = units * 16 + npairs_all * sizeof(Pair2) + n * 4 + units * 16 * 8;
    ctx->db_loaded = true;
    return SW_OK;
}

extern "C" sw_status sw_db_stats_get(const sw_ctx* ctx, sw_db_stats* out) {
    if (!ctx || !out) return SW_ERR_INVALID;
    out->n_records = (uint64_t)ctx->n_records;
    out->n_residues = ctx->n_residues;
    out->n_pairs = (uint64_t)ctx->n_pairs;
    out->max_length = ctx->max_len;
    out->device_bytes = ctx->db_bytes;
    return SW_OK;
}

// ---------------------------------------------------------------------------
// kernel shape selection
// ---------------------------------------------------------------------------

namespace swb {

// Blocks per SM for a shape at a query length (0 = does not fit).
int shape_occupancy(sw_ctx* ctx, const WfKernel& k, int qlen) {
    const size_t smem = k.smem(qlen);
    if (smem > (size_t)ctx->max_smem) return 0;
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k.fn, k.block, smem) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return nb;
}

// Query rows one launch of a shape scores: the whole query when its profile
// fits one block, else the most whole passes whose profile does (a longer
// query is scored in row segments by consecutive launches that hand the
// boundary row on); 0 when not even one pass fits.
int launch_rows(sw_ctx* ctx, const WfKernel& k, int qlen) {
    if (shape_occupancy(ctx, k, qlen) > 0) return qlen;
    const int rows_pass = k.T * k.R;
    int p = 0;
    while ((int64_t)(p + 1) * rows_pass < qlen && shape_occupancy(ctx, k, (p + 1) * rows_pass) > 0)
        ++p;
    return p * rows_pass;
}

// Sum over the pairs [b, e) of max(ncols, m): the column steps of one pass
// whose segments last at least m steps.  Pairs are sorted by ncols
// descending, so the pairs below m are a suffix of the range.
double cols_at_least(const sw_ctx* ctx, int64_t b, int64_t e, uint32_t m) {
    const auto first = ctx->pair_ncols.begin();
    const int64_t i = std::partition_point(first + b, first + e,
                                           [m](uint32_t n) { return n >= m; }) - first;
    return (double)(ctx->pair_prefix[i] - ctx->pair_prefix[b]) + (double)m * (double)(e - i);
}

// Modelled cost of running pairs [b, e) with a shape, for contexts without a
// shape table entry that fits: thread steps x (R + 12.9) plus 25 per pass
// column and group, over an efficiency by group width (several groups in a
// warp diverge at their pair switches) and by resident warps.  The constants
// were fitted to the sweep of every compiled shape at 20 query lengths on a
// B200 (570,200 records); the model's pick is within 0.93 of the best shape
// on average there.  Columns per pass are counted as the streaming loop runs
// them: at least 2T + 2 steps for a pass a later pass depends on, 3 otherwise.
double shape_cost(sw_ctx* ctx, const WfKernel& k, int qlen, int64_t b, int64_t e) {
    const int rows = launch_rows(ctx, k, qlen);
    const int occ = rows > 0 ? shape_occupancy(ctx, k, rows) : 0;
    if (occ == 0 || e <= b) return occ == 0 ? 1e300 : 0.0;
    const double P = (qlen + k.T * k.R - 1) / (k.T * k.R);
    const double cols = (P - 1) * cols_at_least(ctx, b, e, 2 * k.T + 2) + cols_at_least(ctx, b, e, 3);
    const double work = cols * (k.T * (k.R + 12.9) + 25.1);
    const double g_width = k.T >= 32 ? 1.0 : k.T >= 16 ? 0.854 : k.T >= 8 ? 0.687 : 0.663;
    const double warps = (double)occ * k.block / 32.0;
    const double g_warps = warps < 12 ? 0.912 : warps < 20 ? 1.0 : 1.09;
    return work / (g_width * g_warps);
}

// The shape-table entry for a query length whose shapes fit it, or null (no
// table, no entry, a shape override, or the entry's shapes do not fit).
const sw_tuning_entry* find_entry(sw_ctx* ctx, int qlen) {
    if (ctx->has_override) return nullptr;
    for (const sw_tuning_entry& e : ctx->tuning) {
        if ((uint32_t)qlen > e.max_qlen) continue;
        const WfKernel* kl = find_kernel(e.cfg.long_group_width, e.cfg.long_rows_per_thread);
        const WfKernel* ks = find_kernel(e.cfg.short_group_width, e.cfg.short_rows_per_thread);
        if (kl && ks && shape_occupancy(ctx, *kl, qlen) > 0 && shape_occupancy(ctx, *ks, qlen) > 0)
            return &e;
        return nullptr;   // the tuned shape does not fit this length: the model chooses
    }
    return nullptr;
}

sw_kernel_config choose_config(sw_ctx* ctx, int qlen) {
    if (ctx->has_override) return ctx->override_cfg;
    if (const sw_tuning_entry* e = find_entry(ctx, qlen)) return e->cfg;
    int n = 0;
    const WfKernel* ks = wf_kernels(&n);
    const int64_t np = ctx->n_pairs;
    double best = 1e301;
    sw_kernel_config cfg{32, 32, 32, 32, 0};
    for (int i = 0; i < n; ++i) {
        const double c = shape_cost(ctx, ks[i], qlen, 0, np);
        if (c < best) {
            best = c;
            cfg = sw_kernel_config{ks[i].T, ks[i].R, ks[i].T, ks[i].R, 0};
        }
    }
    return cfg;
}

}  // namespace swb

extern "C" sw_status sw_set_kernel_config(sw_ctx* ctx, const sw_kernel_config* cfg) {
    if (!ctx) return SW_ERR_INVALID;
    if (!cfg) {
        ctx->has_override = false;
        return SW_OK;
    }
    if (!find_kernel(cfg->long_group_width, cfg->long_rows_per_thread) ||
        !find_kernel(cfg->short_group_width, cfg->short_rows_per_thread) || cfg->cutover < 0)
        SW_SET(ctx, SW_ERR_INVALID, "no compiled kernel for shape %dx%d / %dx%d",
               cfg->long_group_width, cfg->long_rows_per_thread, cfg->short_group_width,
               cfg->short_rows_per_thread);
    ctx->override_cfg = *cfg;
    ctx->has_override = true;
    return SW_OK;
}

extern "C" sw_status sw_set_tuning(sw_ctx* ctx, const sw_tuning_entry* entries, uint32_t n) {
    if (!ctx || (n && !entries)) return SW_ERR_INVALID;
    std::vector<sw_tuning_entry> tab(entries, entries + n);
    for (const sw_tuning_entry& e : tab) {
        if (!find_kernel(e.cfg.long_group_width, e.cfg.long_rows_per_thread) ||
            !find_kernel(e.cfg.short_group_width, e.cfg.short_rows_per_thread) || e.cfg.cutover < 0)
            SW_SET(ctx, SW_ERR_INVALID, "tuning entry names an uncompiled shape");
        for (const sw_plan_step& s : e.plan) {
            if (s.group_width == 0) break;
            if (!find_kernel(s.group_width, s.rows_per_thread) || s.passes < 0 ||
                s.passes > (1 << 20))
                SW_SET(ctx, SW_ERR_INVALID, "plan step %dx%d x %d passes: no such shape",
                       s.group_width, s.rows_per_thread, s.passes);
        }
    }
    for (size_t i = 1; i < tab.size(); ++i)
        if (tab[i].max_qlen < tab[i - 1].max_qlen)
            SW_SET(ctx, SW_ERR_INVALID, "tuning entries not sorted by max_qlen");
    ctx->tuning = std::move(tab);
    return SW_OK;
}

extern "C" sw_status sw_get_kernel_config(sw_ctx* ctx, uint32_t qlen, sw_kernel_config* cfg) {
    if (!ctx || !cfg) return SW_ERR_INVALID;
    if (!ctx->db_loaded) SW_SET(ctx, SW_ERR_STATE, "no DB loaded");
    *cfg = choose_config(ctx, (int)std::max<uint32_t>(qlen, 1));
    return SW_OK;
}

namespace swb {
sw_status describe_plan(sw_ctx* ctx, int qlen, sw_plan_step* steps, uint32_t capacity,
                        uint32_t* n_steps);
}

extern "C" sw_status sw_get_plan(sw_ctx* ctx, uint32_t qlen, sw_plan_step* steps,
                                 uint32_t capacity, uint32_t* n_steps) {
    if (!ctx || !n_steps || (capacity && !steps)) return SW_ERR_INVALID;
    if (!ctx->db_loaded) SW_SET(ctx, SW_ERR_STATE, "no DB loaded");
    if (qlen > kMaxQueryResidues)
        SW_SET(ctx, SW_ERR_UNSUPPORTED, "query of %u residues (at most %u)", qlen, kMaxQueryResidues);
    return describe_plan(ctx, (int)std::max<uint32_t>(qlen, 1), steps, capacity, n_steps);
}

extern "C" sw_status sw_get_shapes(int32_t* group_width, int32_t* rows_per_thread,
                                   int32_t* threads_per_block, uint32_t capacity,
                                   uint32_t* n_shapes) {
    if (!n_shapes) return SW_ERR_INVALID;
    int n = 0;
    const WfKernel* k = wf_kernels(&n);
    *n_shapes = (uint32_t)n;
    for (uint32_t i = 0; i < capacity && i < (uint32_t)n; ++i) {
        if (group_width) group_width[i] = k[i].T;
        if (rows_per_thread) rows_per_thread[i] = k[i].R;
        if (threads_per_block) threads_per_block[i] = k[i].block;
    }
    return SW_OK;
}

extern "C" sw_status sw_get_run_stats(const sw_ctx* ctx, sw_run_stats* out) {
    if (!ctx || !out) return SW_ERR_INVALID;
    *out = ctx->stats;
    return SW_OK;
}

// ---------------------------------------------------------------------------
// search
// ---------------------------------------------------------------------------

namespace swb {

// Enqueues the whole device sequence of one plain search on ctx->stream:
// first pass (one or two shapes), 32-bit re-score, top-k rounds.  The query
// must already be in d_query.  Returns the buffer holding the final k keys.
sw_status take_marks(sw_ctx* ctx, sw_ctx::Marks* m) {
    if (!ctx->spare.empty()) {
        *m = ctx->spare.back();
        ctx->spare.pop_back();
        return SW_OK;
    }
    for (auto& e : m->e) SW_CUDA(ctx, cudaEventCreate(&e));
    return SW_OK;
}

// A row segment of a plain search: the next `rows` query rows with shape k
// (consecutive launches of whole passes when the profile of all of them does
// not fit one block).
struct RowSeg {
    const WfKernel* k;
    int rows;
};
constexpr int kMaxRowSegs = SW_PLAN_STEPS + 1;

// Columns of one pass over the DB that an evenly loaded group of shape k gets.
double group_share(sw_ctx* ctx, const WfKernel& k, int qlen) {
    const int occ = std::max(1, shape_occupancy(ctx, k, qlen));
    const double groups = (double)occ * ctx->num_sms * (k.block / k.T);
    return (double)ctx->pair_cols_total / groups;
}

// Cut-over for a configuration without one: a DB whose longest pair needs more
// column steps than an evenly loaded bulk group gets (the bulk launch would end
// on a few serial chains: groups claim pairs longest first, so below that the
// long pairs finish inside the share) sends the pairs above a quarter of the
// share to the long-pair kernel; otherwise no split.
int auto_cutover(sw_ctx* ctx, const sw_kernel_config& cfg, int qlen) {
    if (ctx->n_pairs == 0) return 0;
    const WfKernel* k = find_kernel(cfg.short_group_width, cfg.short_rows_per_thread);
    if (!k) return 0;
    const double share = group_share(ctx, *k, qlen);
    if ((double)ctx->pair_ncols[0] <= share) return 0;
    return std::max(1024, (int)(share / 4));
}

// The row segments a plain search runs on the pairs [bulk_begin, n_pairs):
// the table entry's plan when it applies, else the whole query with the bulk
// shape ks (which also takes the rest of a plan without a rest step).  The
// plan is dropped (one segment) when a step names an uncompiled shape, when
// its fixed steps need more rows than the query has, when a segment's profile
// does not fit one pass in shared memory, or when a segment's shape is narrow
// enough that one group's even share of the columns is below the longest
// pair's (its launch would end on that pair's serial column steps: narrow
// shapes only pay with the long-pair split).
int build_plan(sw_ctx* ctx, int qlen, const WfKernel* ks, int64_t bulk_begin, RowSeg* out) {
    out[0] = RowSeg{ks, qlen};
    const sw_tuning_entry* e = find_entry(ctx, qlen);
    if (!e || e->plan[0].group_width == 0 || !ks || bulk_begin >= ctx->n_pairs) return 1;
    RowSeg segs[kMaxRowSegs];
    int n = 0, left = qlen;
    for (int i = 0; i < SW_PLAN_STEPS && left > 0; ++i) {
        const sw_plan_step& s = e->plan[i];
        if (s.group_width == 0) break;
        const WfKernel* k = find_kernel(s.group_width, s.rows_per_thread);
        if (!k || s.passes < 0) return 1;
        if (s.passes == 0) {
            segs[n++] = RowSeg{k, left};
            left = 0;
            break;
        }
        const int64_t rows = (int64_t)s.passes * k->T * k->R;
        if (rows > left) return 1;
        segs[n++] = RowSeg{k, (int)rows};
        left -= (int)rows;
    }
    if (left > 0) segs[n++] = RowSeg{ks, left};
    const double longest = (double)ctx->pair_ncols[bulk_begin];
    for (int i = 0; i < n; ++i)
        if (launch_rows(ctx, *segs[i].k, segs[i].rows) == 0 ||
            longest > group_share(ctx, *segs[i].k, segs[i].rows))
            return 1;
    std::copy(segs, segs + n, out);
    return n;
}

// The long-pair kernel for a query: the configured long shape when the
// configuration names one apart from the bulk shape (a shape table names one
// shape for both) and it is a compiled sw_long row count (group width 32)
// whose passes fit one pipeline, else the smallest row count that needs at most 3 passes (measured on B200:
// 2-3 passes per pair balance pipeline parallelism against per-step
// overhead), else at most kLongMaxPasses.  A block takes a whole SM:
// *pipelines is how many pipelines of *passes warps fit its registers and
// shared memory.  Returns null when nothing fits.
const LongKernel* choose_long(sw_ctx* ctx, const sw_kernel_config& cfg, int qlen, int* passes,
                              int* pipelines, size_t* smem_bytes) {
    int n = 0;
    const LongKernel* lk = long_kernels(&n);
    auto fits = [&](const LongKernel& k) {
        const int P = (qlen + 32 * k.R - 1) / (32 * k.R);
        if (P > kLongMaxPasses) return false;
        cudaFuncAttributes fa;
        if (cudaFuncGetAttributes(&fa, k.fn) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        const size_t dyn = (size_t)ctx->max_smem - fa.sharedSizeBytes;
        const int warp_regs = (fa.numRegs + 7) / 8 * 8 * 32;
        int G = std::min(k.max_threads / 32, ctx->regs_per_sm / std::max(warp_regs, 1)) / P;
        while (G > 0 && k.smem(P, G) > dyn) --G;
        while (G > 0) {
            int nb = 0;
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k.fn, G * P * 32, dyn) ==
                    cudaSuccess && nb >= 1)
                break;
            cudaGetLastError();
            --G;
        }
        if (G == 0) return false;
        *passes = P;
        *pipelines = G;
        *smem_bytes = dyn;
        return true;
    };
    const bool named = cfg.long_group_width != cfg.short_group_width ||
                       cfg.long_rows_per_thread != cfg.short_rows_per_thread;
    if (named && cfg.long_group_width == 32)
        for (int i = 0; i < n; ++i)
            if (lk[i].R == cfg.long_rows_per_thread && fits(lk[i])) return &lk[i];
    for (int i = 0; i < n; ++i)
        if ((qlen + 32 * lk[i].R - 1) / (32 * lk[i].R) <= 3 && fits(lk[i])) return &lk[i];
    for (int i = 0; i < n; ++i)
        if (fits(lk[i])) return &lk[i];
    return nullptr;
}

// How a plain search of qlen divides the DB's pairs.  With a cut-over (the
// configured one, else auto_cutover's), the long-pair kernel takes the pairs
// above it, [0, n_long), when some but not all pairs are, and a pipelined
// shape fits the length; the bulk launches take the rest with the short shape.
// Otherwise one shape takes every pair: the long one when no pair is above
// the cut-over or all are, the short one when no pipelined shape fits.
struct SearchLayout {
    sw_kernel_config cfg;
    int cutover = 0;
    bool split = false;
    int64_t n_long = 0;                // pairs of the long-pair kernel (split only)
    const LongKernel* lk = nullptr;
    int lpasses = 0, lpipes = 0;
    size_t lsmem = 0;
    int bulk_T = 0, bulk_R = 0;        // the bulk launches' shape ...
    int64_t bulk_b = 0, bulk_e = 0;    // ... pairs ...
    int bulk_counter = 0;              // ... and claim counter
};

void layout_search(sw_ctx* ctx, int qlen, SearchLayout* L) {
    const sw_kernel_config& cfg = L->cfg = choose_config(ctx, qlen);
    L->cutover = cfg.cutover > 0 ? cfg.cutover : auto_cutover(ctx, cfg, qlen);
    int64_t n_long = ctx->n_pairs;
    if (L->cutover > 0) {
        n_long = 0;
        while (n_long < ctx->n_pairs && (int)ctx->pair_ncols[n_long] > L->cutover) ++n_long;
    }
    L->split = L->cutover > 0 && n_long > 0 && n_long < ctx->n_pairs;
    if (L->split) {
        L->lk = choose_long(ctx, cfg, qlen, &L->lpasses, &L->lpipes, &L->lsmem);
        if (!L->lk) L->split = false;      // no pipelined shape for this length
    }
    if (L->split || (n_long < ctx->n_pairs && L->cutover > 0)) {
        // the short shape: beside the long-pair kernel, or alone for every
        // pair when no pair is above the cut-over or no pipelined shape fits
        L->bulk_T = cfg.short_group_width;
        L->bulk_R = cfg.short_rows_per_thread;
        L->bulk_b = L->split ? n_long : 0;
        L->bulk_counter = 1;
    } else {
        L->bulk_T = cfg.long_group_width;
        L->bulk_R = cfg.long_rows_per_thread;
        L->bulk_b = 0;
        L->bulk_counter = 0;
    }
    L->bulk_e = ctx->n_pairs;
    L->n_long = L->split ? n_long : 0;
}

// sw_get_plan: the row segments enqueue_search would run.
sw_status describe_plan(sw_ctx* ctx, int qlen, sw_plan_step* steps, uint32_t capacity,
                        uint32_t* n_steps) {
    SearchLayout L;
    layout_search(ctx, qlen, &L);
    const WfKernel* k = find_kernel(L.bulk_T, L.bulk_R);
    if (!k) SW_SET(ctx, SW_ERR_INVALID, "no kernel %dx%d", L.bulk_T, L.bulk_R);
    RowSeg plan[kMaxRowSegs];
    const int n = build_plan(ctx, qlen, k, L.bulk_b, plan);
    *n_steps = (uint32_t)n;
    for (int i = 0; i < n && (uint32_t)i < capacity; ++i) {
        const int rp = plan[i].k->T * plan[i].k->R;
        steps[i] = sw_plan_step{plan[i].k->T, plan[i].k->R, (plan[i].rows + rp - 1) / rp};
    }
    return SW_OK;
}

sw_status enqueue_search(sw_ctx* ctx, const uint8_t* d_query, int qlen, int32_t* d_scores_rec,
                         unsigned long long** keys_final, uint32_t* launches) {
    cudaStream_t st = ctx->stream;
    SearchLayout L;
    layout_search(ctx, qlen, &L);
    ctx->stats.used = L.cfg;
    ctx->stats.used.cutover = L.cutover;
    *launches = 0;
    const bool split = L.split;
    const int64_t n_long = L.n_long;
    const LongKernel* lk = L.lk;
    const int lpasses = L.lpasses;
    int lpipes = L.lpipes;
    if (split) {
        ctx->stats.used.long_group_width = 32;
        ctx->stats.used.long_rows_per_thread = lk->R;
    }
    const int ovf_thresh = 32767 - std::max(ctx->max_score, 1) + 1;
    // With a cut-over, the long pairs run concurrently on the side stream in
    // sw_long blocks (one warp per query pass, the passes of a pair pipelined
    // across warps, several pipelines per block, one block per SM) on SMs the
    // bulk grid leaves free, as many SMs as the long pairs' share of the
    // columns.  The bulk launches take the other pairs in the row segments of
    // the length's plan.
    RowSeg plan[kMaxRowSegs];
    int nplan = 0;
    // every shape is checked before anything is launched: a search refused
    // half-way would leave a launch in flight that writes into the next one
    if (L.bulk_e > L.bulk_b) {
        const WfKernel* k = find_kernel(L.bulk_T, L.bulk_R);
        if (!k) SW_SET(ctx, SW_ERR_INVALID, "no kernel %dx%d", L.bulk_T, L.bulk_R);
        if (launch_rows(ctx, *k, qlen) == 0)
            SW_SET(ctx, SW_ERR_UNSUPPORTED,
                   "one pass of shape %dx%d does not fit shared memory (profile %zu bytes)",
                   L.bulk_T, L.bulk_R, k->smem(L.bulk_T * L.bulk_R));
        nplan = build_plan(ctx, qlen, k, L.bulk_b, plan);
        if (nplan > 1) {
            ctx->stats.used.short_group_width = plan[0].k->T;
            ctx->stats.used.short_rows_per_thread = plan[0].k->R;
        }
    }
    // the search's timing events, taken after every check (a refused search
    // holds none), then its buffers cleared
    sw_ctx::Marks mk{};
    sw_status ms = take_marks(ctx, &mk);
    if (ms != SW_OK) return ms;
    mk.fp_launches = 0;
    mk.cells = (uint64_t)qlen * ctx->n_residues;
    SW_CUDA(ctx, cudaEventRecord(mk.e[0], st));
    SW_CUDA(ctx, cudaMemsetAsync(ctx->d_counters, 0, 16 * sizeof(int), st));
    SW_CUDA(ctx, cudaMemsetAsync(ctx->d_scores, 0, (size_t)(ctx->n_records + 1) * sizeof(int), st));
    SW_CUDA(ctx, cudaEventRecord(mk.e[1], st));
    int reserved_sms = 0;
    if (split) {
        uint64_t long_cols = 0;
        for (int64_t p = 0; p < n_long; ++p) long_cols += ctx->pair_ncols[p];
        const double share = (double)long_cols / (double)std::max<uint64_t>(ctx->pair_cols_total, 1);
        // SMs for the long launch: their share of the columns, or, when there
        // are few long pairs, enough SMs that each warp scheduler runs about
        // one of their warps (a pair's column steps are serial, so a crowded
        // SM would make the longest pair the critical path), at most half
        reserved_sms = (int)std::lround(share * ctx->num_sms);
        const int64_t spread = (n_long * lpasses + 3) / 4;
        reserved_sms = (int)std::max<int64_t>(reserved_sms,
                                              std::min<int64_t>(spread, ctx->num_sms / 2));
        reserved_sms = std::max(1, std::min(reserved_sms, ctx->num_sms - 1));
        reserved_sms = (int)std::min<int64_t>(reserved_sms, (n_long + lpipes - 1) / lpipes);
        // pipelines per block: the long pairs spread evenly over those SMs
        lpipes = (int)std::min<int64_t>(lpipes, (n_long + reserved_sms - 1) / reserved_sms);
        SW_CUDA(ctx, cudaEventRecord(ctx->fork_ev, st));
        SW_CUDA(ctx, cudaStreamWaitEvent(ctx->side_stream, ctx->fork_ev, 0));
        LongArgs la;
        la.db = ctx->d_db;
        la.pairs = ctx->d_pairs;
        la.pair_begin = 0;
        la.pair_count = (int)n_long;
        la.counter = ctx->d_counters;      // counter 0: the long pairs' claims
        la.query = d_query;
        la.qlen = qlen;
        la.passes = lpasses;
        la.mat = ctx->d_mat;
        la.bias2 = (uint32_t)(ctx->params.gap_open + ctx->params.gap_extend);
        la.bias2 |= la.bias2 << 16;
        la.neg_e = (uint32_t)(uint16_t)(int16_t)(-ctx->params.gap_extend);
        la.neg_e |= la.neg_e << 16;
        la.scores = ctx->d_scores;
        la.n_records = (int)ctx->n_records;
        la.ovf_list = ctx->d_ovf;
        la.ovf_count = ctx->d_counters + 2;
        la.ovf_thresh = ovf_thresh;
        la.ovf_cap = (int)ctx->n_records + 1;
        void* args[] = {&la};
        SW_CUDA(ctx, cudaEventRecord(mk.e[4], ctx->side_stream));
        SW_CUDA(ctx, cudaLaunchKernel(lk->fn, dim3((unsigned)reserved_sms),
                                      dim3(lpasses * lpipes * 32), args, L.lsmem, ctx->side_stream));
        SW_CUDA(ctx, cudaEventRecord(mk.e[5], ctx->side_stream));
        ++*launches;
        ++mk.fp_launches;
        SW_CUDA(ctx, cudaEventRecord(mk.e[6], st));
    }
    mk.split = split;
    // Row segments of the plan (one for most lengths), each in launches of
    // whole passes up to what one block's profile holds: every launch but the
    // first reads the boundary row the one before wrote (pass0 counts the
    // query's passes before it, whatever their shapes: the row holds one
    // 8-byte (H, F) entry per column and parity of the pass index, so its
    // layout does not depend on the shape), and scores merge by maximum.
    int r0 = 0, passes_before = 0;
    for (int pi = 0; pi < nplan; ++pi) {
        const WfKernel* k = plan[pi].k;
        const int seg_rows = launch_rows(ctx, *k, plan[pi].rows);
        for (int s0 = 0; s0 < plan[pi].rows; s0 += seg_rows) {
            const int rows = std::min(seg_rows, plan[pi].rows - s0);
            const int occ = shape_occupancy(ctx, *k, rows);
            if (r0 > 0)   // the previous launch has claimed every pair
                SW_CUDA(ctx, cudaMemsetAsync(ctx->d_counters + L.bulk_counter, 0, sizeof(int), st));
            WfArgs a;
            a.db = ctx->d_db;
            a.pairs = ctx->d_pairs;
            a.pair_begin = (int)L.bulk_b;
            a.pair_count = (int)(L.bulk_e - L.bulk_b);
            a.query = d_query + r0;
            a.qlen = rows;
            a.pass0 = passes_before;
            a.more = r0 + rows < qlen ? 1 : 0;
            a.mat = ctx->d_mat;
            a.bias2 = (uint32_t)(ctx->params.gap_open + ctx->params.gap_extend);
            a.bias2 |= a.bias2 << 16;
            a.neg_e = (uint32_t)(uint16_t)(int16_t)(-ctx->params.gap_extend);
            a.neg_e |= a.neg_e << 16;
            a.counter = ctx->d_counters + L.bulk_counter;
            a.bnd = ctx->d_bnd;
            a.scores = ctx->d_scores;
            a.n_records = (int)ctx->n_records;
            a.ovf_list = ctx->d_ovf;
            a.ovf_count = ctx->d_counters + 2;
            a.ovf_thresh = ovf_thresh;
            void* args[] = {&a};
            int64_t grid = (int64_t)occ * (ctx->num_sms - reserved_sms);
            const int64_t groups_per_block = k->block / k->T;
            grid = std::min<int64_t>(grid, ((L.bulk_e - L.bulk_b) + groups_per_block - 1) / groups_per_block);
            grid = std::max<int64_t>(grid, 1);
            SW_CUDA(ctx, cudaLaunchKernel(k->fn, dim3((unsigned)grid), dim3(k->block), args,
                                          k->smem(rows), st));
            ++*launches;
            ++mk.fp_launches;
            r0 += rows;
            passes_before += (rows + k->T * k->R - 1) / (k->T * k->R);
        }
    }
    if (split) {
        SW_CUDA(ctx, cudaEventRecord(mk.e[7], st));
        SW_CUDA(ctx, cudaEventRecord(ctx->join_ev, ctx->side_stream));
        SW_CUDA(ctx, cudaStreamWaitEvent(st, ctx->join_ev, 0));
    }
    SW_CUDA(ctx, cudaEventRecord(mk.e[2], st));
    {
        RescoreArgs r;
        r.db = ctx->d_db;
        r.pairs = ctx->d_pairs;
        r.query = d_query;
        r.qlen = qlen;
        r.mat = ctx->d_mat;
        r.gap_oe = ctx->params.gap_open + ctx->params.gap_extend;
        r.gap_e = ctx->params.gap_extend;
        r.queries = nullptr;
        r.qoff = nullptr;
        r.qlens = nullptr;
        r.n_records = (int)ctx->n_records;
        r.ovf_list = ctx->d_ovf;
        r.ovf_count = ctx->d_counters + 2;
        r.ovf_cap = (int)ctx->n_records + 1;
        r.scratch = ctx->d_rs_scratch;
        r.max_cols = ctx->max_cols;
        r.scores = ctx->d_scores;
        void* args[] = {&r};
        SW_CUDA(ctx, cudaLaunchKernel((const void*)sw_rescore32, dim3(kRescoreBlocks), dim3(64),
                                      args, 0, st));
        ++*launches;
    }
    // top-k rounds: n -> ceil(n/4096)*k -> ... -> k
    const int k = ctx->params.top_k;
    long long n = ctx->n_records;
    int buf = 0;
    const unsigned long long* keys_in = nullptr;
    bool first = true;
    while (true) {
        const long long blocks = std::max<long long>(1, (n + kTopkKeys - 1) / kTopkKeys);
        TopkArgs t;
        t.scores = ctx->d_scores;
        t.perm = ctx->d_perm;
        t.keys_in = first ? nullptr : keys_in;
        t.n = n;
        t.k = k;
        t.cap = (ctx->params.flags & SW_FLAG_REFERENCE_CAP) ? 1 : 0;
        t.scores_by_record = first ? d_scores_rec : nullptr;
        t.keys_out = ctx->d_keys[buf];
        t.in_stride = 0;
        t.rec_stride = 0;
        t.out_stride = 0;
        t.rows = nullptr;
        void* args[] = {&t};
        SW_CUDA(ctx, cudaLaunchKernel((const void*)sw_topk_round, dim3((unsigned)blocks),
                                      dim3(kTopkThreads), args, 0, st));
        ++*launches;
        keys_in = ctx->d_keys[buf];
        buf ^= 1;
        first = false;
        if (blocks == 1) break;
        n = blocks * (long long)k;
    }
    *keys_final = const_cast<unsigned long long*>(keys_in);
    SW_CUDA(ctx, cudaEventRecord(mk.e[3], st));
    mk.launches = *launches;
    ctx->pending.push_back(mk);
    return SW_OK;
}

// Waits for the stream and folds the pending searches' event timings into
// the totals; returns the last search's (whole, first pass) device times.
sw_status drain(sw_ctx* ctx, float* last_ms, float* last_fp_ms) {
    SW_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    for (auto& m : ctx->pending) {
        float whole = 0.f, fp = 0.f, lms = 0.f, bms = 0.f;
        SW_CUDA(ctx, cudaEventElapsedTime(&whole, m.e[0], m.e[3]));
        SW_CUDA(ctx, cudaEventElapsedTime(&fp, m.e[1], m.e[2]));
        if (m.split) {
            SW_CUDA(ctx, cudaEventElapsedTime(&lms, m.e[4], m.e[5]));
            SW_CUDA(ctx, cudaEventElapsedTime(&bms, m.e[6], m.e[7]));
        }
        ctx->stats.long_ms = lms;
        ctx->stats.bulk_ms = bms;
        ctx->totals.search_ms += whole;
        ctx->totals.first_pass_ms += fp;
        ctx->totals.first_pass_launches += m.fp_launches;
        ctx->totals.launches += m.launches;
        ctx->totals.cells += m.cells;
        ctx->totals.queries += 1;
        if (last_ms) *last_ms = whole;
        if (last_fp_ms) *last_fp_ms = fp;
        ctx->spare.push_back(m);
    }
    ctx->pending.clear();
    return SW_OK;
}

sw_status ensure_query_buffers(sw_ctx* ctx, size_t qlen) {
    if (qlen <= ctx->query_cap) return SW_OK;
    size_t cap = std::max<size_t>(qlen, 4096);
    dev_free(ctx->d_query);
    if (ctx->h_query) cudaFreeHost(ctx->h_query);
    ctx->h_query = nullptr;
    ctx->query_cap = 0;
    if (dev_alloc(&ctx->d_query, cap) != cudaSuccess) SW_SET(ctx, SW_ERR_NOMEM, "query buffer");
    if (cudaMallocHost((void**)&ctx->h_query, cap) != cudaSuccess)
        SW_SET(ctx, SW_ERR_NOMEM, "pinned query buffer");
    if (!ctx->h_keys && cudaMallocHost((void**)&ctx->h_keys, kMaxTopK * sizeof(unsigned long long)) !=
                            cudaSuccess)
        SW_SET(ctx, SW_ERR_NOMEM, "pinned key buffer");
    ctx->query_cap = cap;
    return SW_OK;
}

}  // namespace swb

extern "C" sw_status sw_search(sw_ctx* ctx, const uint8_t* query, uint32_t qlen, sw_hit* hits,
                               uint32_t* n_hits, int32_t* scores) {
    if (!ctx) return SW_ERR_INVALID;
    if (ctx->serve) return SW_ERR_BUSY;   // the serving loop owns the stream and the DB
    return swb::search_host(ctx, query, qlen, hits, n_hits, scores);
}

namespace swb {

sw_status search_host(sw_ctx* ctx, const uint8_t* query, uint32_t qlen, sw_hit* hits,
                      uint32_t* n_hits, int32_t* scores) {
    if (!ctx->db_loaded) SW_SET(ctx, SW_ERR_STATE, "no DB loaded (call sw_db_load first)");
    if ((qlen && !query) || (!hits && ctx->params.top_k > 0) || !n_hits)
        SW_SET(ctx, SW_ERR_INVALID, "null argument");
    if (qlen > kMaxQueryResidues)
        SW_SET(ctx, SW_ERR_UNSUPPORTED, "query of %u residues (at most %u)", qlen, kMaxQueryResidues);
    const double t0 = now_ms();
    const int k = ctx->params.top_k;
    for (int i = 0; i < k; ++i) hits[i] = sw_hit{0, 0, 0};
    *n_hits = 0;
    ctx->stats = sw_run_stats{};
    if (qlen == 0 || ctx->n_records == 0) {
        if (scores) memset(scores, 0, (size_t)ctx->n_records * sizeof(int32_t));
        ctx->stats.total_ms = now_ms() - t0;
        return SW_OK;
    }
    for (uint32_t i = 0; i < qlen; ++i)
        if (query[i] > 24) SW_SET(ctx, SW_ERR_INVALID, "query code %d at %u", query[i], i);
    SW_CUDA(ctx, cudaSetDevice(ctx->device));
    sw_status st = ensure_query_buffers(ctx, qlen);
    if (st != SW_OK) return st;
    memcpy(ctx->h_query, query, qlen);
    SW_CUDA(ctx, cudaMemcpyAsync(ctx->d_query, ctx->h_query, qlen, cudaMemcpyHostToDevice,
                                 ctx->stream));
    unsigned long long* keys = nullptr;
    uint32_t launches = 0;
    st = enqueue_search(ctx, ctx->d_query, (int)qlen, scores ? ctx->d_scores_rec : nullptr, &keys,
                        &launches);
    if (st != SW_OK) return st;
    SW_CUDA(ctx, cudaMemcpyAsync(ctx->h_keys, keys, (size_t)k * sizeof(unsigned long long),
                                 cudaMemcpyDeviceToHost, ctx->stream));
    if (scores)
        SW_CUDA(ctx, cudaMemcpyAsync(scores, ctx->d_scores_rec,
                                     (size_t)ctx->n_records * sizeof(int32_t),
                                     cudaMemcpyDeviceToHost, ctx->stream));
    float kms = 0.f, fpms = 0.f;
    st = drain(ctx, &kms, &fpms);
    if (st != SW_OK) return st;
    SW_CUDA(ctx, cudaGetLastError());
    uint32_t m = 0;
    for (int i = 0; i < k; ++i) {
        const unsigned long long key = ctx->h_keys[i];
        if (key == 0ull) break;
        hits[m].score = (int32_t)(key >> 32);
        hits[m].reserved = 0;
        hits[m].index = 0xffffffffull - (key & 0xffffffffull);
        ++m;
    }
    *n_hits = m;
    int rescored = 0;
    cudaMemcpy(&rescored, ctx->d_counters + 2, sizeof(int), cudaMemcpyDeviceToHost);
    ctx->stats.kernel_ms = kms;
    ctx->stats.first_pass_ms = fpms;
    ctx->stats.cells = (uint64_t)qlen * ctx->n_residues;
    ctx->stats.rescored = (uint64_t)rescored;
    ctx->stats.launches = launches;
    ctx->stats.queries = 1;
    ctx->stats.total_ms = now_ms() - t0;
    return SW_OK;
}

}  // namespace swb

extern "C" sw_status sw_search_device(sw_ctx* ctx, const uint8_t* d_query, uint32_t qlen,
                                      int32_t* d_scores) {
    if (!ctx) return SW_ERR_INVALID;
    if (ctx->serve) return SW_ERR_BUSY;   // the serving loop owns the stream and the DB
    if (!ctx->db_loaded) SW_SET(ctx, SW_ERR_STATE, "no DB loaded (call sw_db_load first)");
    if (!d_query || qlen == 0) SW_SET(ctx, SW_ERR_INVALID, "empty query");
    if (qlen > kMaxQueryResidues)
        SW_SET(ctx, SW_ERR_UNSUPPORTED, "query of %u residues (at most %u)", qlen, kMaxQueryResidues);
    SW_CUDA(ctx, cudaSetDevice(ctx->device));
    ctx->stats = sw_run_stats{};
    unsigned long long* keys = nullptr;
    uint32_t launches = 0;
    sw_status st = enqueue_search(ctx, d_query, (int)qlen, d_scores, &keys, &launches);
    if (st != SW_OK) return st;
    ctx->stats.cells = (uint64_t)qlen * ctx->n_residues;
    ctx->stats.launches = launches;
    ctx->stats.queries = 1;
    return SW_OK;
}

extern "C" sw_status sw_set_stream(sw_ctx* ctx, void* cuda_stream) {
    if (!ctx) return SW_ERR_INVALID;
    if (ctx->serve) return SW_ERR_BUSY;   // the serving loop owns the stream and the DB
    SW_CUDA(ctx, cudaSetDevice(ctx->device));
    sw_status st = drain(ctx, nullptr, nullptr);
    if (st != SW_OK) return st;
    ctx->stream = cuda_stream ? (cudaStream_t)cuda_stream : ctx->own_stream;
    return SW_OK;
}

extern "C" sw_status sw_sync(sw_ctx* ctx) {
    if (!ctx) return SW_ERR_INVALID;
    SW_CUDA(ctx, cudaSetDevice(ctx->device));
    sw_status st = drain(ctx, nullptr, nullptr);
    if (st != SW_OK) return st;
    SW_CUDA(ctx, cudaGetLastError());
    return SW_OK;
}

extern "C" sw_status sw_reset_totals(sw_ctx* ctx) {
    if (!ctx) return SW_ERR_INVALID;
    sw_status st = sw_sync(ctx);
    ctx->totals = sw_totals{};
    return st;
}

extern "C" sw_status sw_get_totals(const sw_ctx* ctx, sw_totals* out) {
    if (!ctx || !out) return SW_ERR_INVALID;
    *out = ctx->totals;
    return SW_OK;
}
