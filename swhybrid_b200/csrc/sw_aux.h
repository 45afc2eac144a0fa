// sw_aux.h -- argument blocks of the re-score and top-k kernels.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "sw_device.cuh"

namespace swb {

constexpr int kTopkThreads = 1024;
constexpr int kTopkKeys = 4096;     // keys sorted per block and round
constexpr int kMaxTopK = 1024;      // so that every round shrinks the key set

struct RescoreArgs {
    const uint4* db;
    const Pair2* pairs;
    const uint8_t* query;
    int qlen;
    const int8_t* mat;
    int gap_oe;
    int gap_e;
    const int* ovf_list;
    const int* ovf_count;
    uint2* bnd;
    int* scores;
};

struct TopkArgs {
    const int* scores;                    // round 0: per sorted position
    const uint32_t* perm;                 // round 0: sorted position -> record
    const unsigned long long* keys_in;    // later rounds (null in round 0)
    long long n;                          // inputs of this round
    int k;
    int cap;                              // clamp scores to 65535 (round 0)
    int* scores_by_record;                // round 0, optional
    unsigned long long* keys_out;         // gridDim.x * k keys
};

__global__ void sw_rescore32(const RescoreArgs a);
__global__ void sw_topk_round(const TopkArgs a);

}  // namespace swb
