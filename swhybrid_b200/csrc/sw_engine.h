// sw_engine.h -- the context behind the C ABI's opaque sw_ctx.
#pragma once
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/swb200.h"
#include "sw_device.cuh"

#define SW_SET(ctx, code, ...)                                              \
    do {                                                                    \
        char _b[512];                                                       \
        snprintf(_b, sizeof(_b), __VA_ARGS__);                              \
        if (ctx) (ctx)->err = _b;                                           \
        return code;                                                        \
    } while (0)

#define SW_CUDA(ctx, call)                                                  \
    do {                                                                    \
        cudaError_t _e = (call);                                            \
        if (_e != cudaSuccess)                                              \
            SW_SET(ctx, SW_ERR_CUDA, "%s failed: %s (%s:%d)", #call,        \
                   cudaGetErrorString(_e), __FILE__, __LINE__);             \
    } while (0)

// Longest query any search entry point takes, in residues (16.7 M, far above
// any protein; keeps row counts and offsets in 32-bit ints).
constexpr uint32_t kMaxQueryResidues = 1u << 24;

template <typename T>
inline cudaError_t dev_alloc(T** p, size_t count) {
    *p = nullptr;
    if (count == 0) count = 1;
    return cudaMalloc((void**)p, count * sizeof(T));
}

template <typename T>
inline void dev_free(T*& p) {
    if (p) cudaFree((void*)p);
    p = nullptr;
}

struct sw_batch_state;   // batched search buffers and captured graphs (sw_batch.cu)
struct sw_serve_state;   // serving loop: slots, ring of DB chunks, scheduler (sw_serve.cu)
struct sw_tb_state;      // traceback scratch (sw_traceback.cu)

struct sw_ctx {
    int device = 0;
    int num_sms = 0;
    int max_smem = 0;
    int regs_per_sm = 0;
    cudaStream_t stream = nullptr;       // stream in use
    cudaStream_t own_stream = nullptr;   // the context's own stream
    cudaStream_t side_stream = nullptr;  // concurrent launch of the long-record pairs
    cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    // timing events of enqueued searches: begin, first pass begin/end, end
    // (and, with a cut-over, long launch begin/end on the side stream, bulk
    // launch begin/end on the main stream)
    struct Marks {
        cudaEvent_t e[8];
        bool split;
        uint32_t fp_launches;
        uint32_t launches;
        uint64_t cells;
    };
    std::vector<Marks> pending;
    std::vector<Marks> spare;
    sw_totals totals{};
    sw_params params{};
    int max_score = 0;
    int8_t* d_mat = nullptr;           // 32x32 int8, codes >= 24 zeroed
    int* d_counters = nullptr;         // [0],[1] pair counters, [2] overflow count

    // resident DB
    bool db_loaded = false;
    int64_t n_records = 0;
    int64_t n_pairs = 0;               // pairs with at least one column
    uint64_t n_residues = 0;
    uint64_t max_len = 0;
    uint64_t units = 0;                // 16-byte units of the column stream
    uint64_t db_bytes = 0;
    std::vector<uint32_t> pair_ncols;  // host copy, for shape selection
    uint64_t pair_cols_total = 0;      // sum of pair_ncols
    std::vector<uint64_t> pair_prefix; // pair_prefix[p] = sum of pair_ncols[0, p)
    std::vector<uint32_t> rec_pos;     // record -> sorted position (host)
    std::vector<uint32_t> rec_len;     // record -> length (host)
    uint4* d_db = nullptr;
    swb::Pair2* d_pairs = nullptr;
    uint32_t* d_perm = nullptr;        // sorted position -> record
    uint2* d_bnd = nullptr;            // boundary rows between query passes
    uint64_t db_units = 0;             // 16-byte units of the column streams (d_bnd: 16 each)
    int* d_scores = nullptr;           // per sorted position
    int* d_scores_rec = nullptr;       // per record
    int* d_ovf = nullptr;              // overflow list
    unsigned long long* d_keys[2] = {nullptr, nullptr};
    uint2* d_rs_scratch = nullptr;     // 32-bit re-score: one boundary row per warp
    int max_cols = 0;                  // longest pair, padded to 8 columns
    sw_batch_state* batch = nullptr;
    sw_serve_state* serve = nullptr;   // non-null between sw_serve_start and sw_serve_stop
    sw_tb_state* tb = nullptr;
    // DB image the resident DB came from (read-only mapping; titles are read from it)
    const uint8_t* image = nullptr;
    size_t image_bytes = 0;

    // per-query buffers
    size_t query_cap = 0;
    uint8_t* d_query = nullptr;
    uint8_t* h_query = nullptr;        // pinned
    unsigned long long* h_keys = nullptr;  // pinned

    std::vector<sw_tuning_entry> tuning;
    bool has_override = false;
    sw_kernel_config override_cfg{};
    sw_run_stats stats{};
    std::string err;
};

namespace swb {
struct WfKernel;
const WfKernel* find_kernel(int T, int R);
int shape_occupancy(sw_ctx* ctx, const WfKernel& k, int qlen);
int launch_rows(sw_ctx* ctx, const WfKernel& k, int qlen);
// sw_search without the serving check: one plain search with host buffers
// (the serving scheduler runs requests too long for a stack through it)
sw_status search_host(sw_ctx* ctx, const uint8_t* query, uint32_t qlen, sw_hit* hits,
                      uint32_t* n_hits, int32_t* scores);
sw_kernel_config choose_config(sw_ctx* ctx, int qlen);
sw_status take_marks(sw_ctx* ctx, sw_ctx::Marks* m);
sw_status drain(sw_ctx* ctx, float* last_ms, float* last_fp_ms);
void free_batch(sw_ctx* ctx);
void serve_teardown(sw_ctx* ctx);
void free_traceback(sw_ctx* ctx);
void free_image(sw_ctx* ctx);
sw_status db_load(sw_ctx* ctx, const uint8_t* residues, const uint64_t* offsets, uint64_t n,
                  const uint32_t* given_order);
const char* thread_error();   // message of this thread's last context-free call
sw_status thread_fail(sw_status st, const char* fmt, ...) __attribute__((format(printf, 2, 3)));
sw_status ensure_query_buffers(sw_ctx* ctx, size_t qlen);
}  // namespace swb
