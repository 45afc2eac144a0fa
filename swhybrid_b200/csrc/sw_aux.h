// sw_aux.h -- argument blocks of the re-score and top-k kernels.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "sw_device.cuh"

namespace swb {

constexpr int kTopkThreads = 1024;
constexpr int kTopkKeys = 4096;     // keys sorted per block and round
constexpr int kMaxTopK = 1024;      // so that every round shrinks the key set

constexpr int kRescoreBlocks = 148;   // x 64 threads: 296 warps
constexpr int kRescoreWarps = kRescoreBlocks * 2;

struct RescoreArgs {
    const uint4* db;
    const Pair2* pairs;
    const uint8_t* query;       // plain search: the query
    int qlen;
    const uint8_t* queries;     // batched search (qoff != null): all queries
    const uint32_t* qoff;
    const uint32_t* qlens;
    int n_records;              // batched: entry = query * n_records + position
    const int8_t* mat;
    int gap_oe;
    int gap_e;
    const int* ovf_list;
    const int* ovf_count;
    int ovf_cap;
    uint2* scratch;             // kRescoreWarps rows of max_cols entries
    int max_cols;
    int* scores;                // indexed by the overflow entry
};

struct TopkArgs {
    const int* scores;                    // round 0: per sorted position
    const uint32_t* perm;                 // round 0: sorted position -> record
    const unsigned long long* keys_in;    // later rounds (null in round 0)
    long long n;                          // inputs of this round (per query)
    int k;
    int cap;                              // clamp scores to 65535 (round 0)
    int* scores_by_record;                // round 0, optional
    unsigned long long* keys_out;         // gridDim.x * k keys per query
    long long in_stride;                  // per query (blockIdx.y): scores / keys_in
    long long rec_stride;                 // per query: scores_by_record
    long long out_stride;                 // per query: keys_out
    const int* rows;                      // optional: round 0 reads score row rows[y]
};

__global__ void sw_rescore32(const RescoreArgs a);
__global__ void sw_topk_round(const TopkArgs a);

}  // namespace swb
