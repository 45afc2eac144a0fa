// sw_long.h -- the long-pair first pass (sw_long.cu): arguments and the table
// of compiled row counts.
#pragma once
#include <cstddef>
#include <cstdint>

#include "sw_device.cuh"

namespace swb {

constexpr int kLongMaxPasses = 8;        // query passes of 32 x R rows = warps per pipeline
constexpr int kLongMaxWarps = 32;        // pipelines x passes per block

struct LongArgs {
    const uint4* db;            // pair column streams
    const Pair2* pairs;         // pair table, ncols descending
    int pair_begin;             // pairs [pair_begin, pair_begin + pair_count)
    int pair_count;
    int* counter;               // pairs claimed so far (one pipeline per pair)
    const uint8_t* query;
    int qlen;                   // at most kLongMaxPasses * 32 * R rows
    int passes;                 // ceil(qlen / (32 R)); blockDim.x = 32 * passes * pipelines
    const int8_t* mat;
    uint32_t bias2, neg_e;      // (open+extend) x2, (-extend) x2
    int* scores;                // by sorted position
    int n_records;
    int* ovf_list;              // positions whose 16-bit lanes may have wrapped
    int* ovf_count;
    int ovf_thresh;
    int ovf_cap;
};

struct LongKernel {
    int R;                                      // query rows per thread; 32 threads per pass
    const void* fn;                             // __global__ sw_long<R>
    size_t (*smem)(int passes, int pipelines);  // dynamic shared memory of one block
    int max_threads;                            // the kernel's launch bound
};

const LongKernel* long_kernels(int* n);

}  // namespace swb
