// sw_device.cuh -- device-side constants and packed-integer helpers.
//
// All score arithmetic is integer.  The first pass keeps two 16-bit lanes per
// 32-bit register (two DB records side by side) and uses the sm_100 DPX
// instructions (fused add+max, 3-way max, max with ReLU), which wrap on
// overflow; the host-visible threshold below turns any lane that could have
// wrapped into an exact 32-bit re-score.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace swb {

// Device residue codes: 0..23 as the reference encodes them (src/DataPool.cpp:
// 33-47, 23 = '@'), 24 = zero-score code used for letters the reference maps
// to -1 and for every tail pad added by the DB layout and the query padding.
constexpr int kZeroCode = 24;
constexpr int kCodes = 25;          // rows of the shared-memory query profile
constexpr uint32_t kPadPair = (kZeroCode << 8) | kZeroCode;

// A 16-bit lane that reaches this value may have wrapped: re-score in int32.
// (H grows by at most max(matrix) per cell, so a lane can only wrap after
// holding a value above 32767 - max(matrix); the host passes that bound.)

struct Pair2 {          // per DB record pair, 8 bytes
    uint32_t off16;     // start of the pair's column stream, in 16-byte units
    uint32_t ncols;     // columns (length of the longer record)
};

// Arguments of the first-pass kernel (sw_wavefront.cuh).
struct WfArgs {
    const uint4* db;            // pair column streams
    const Pair2* pairs;         // pair table, ncols descending
    int pair_begin;             // first pair handled by this launch
    int pair_count;             // pairs handled by this launch
    const uint8_t* query;       // device query codes of this launch's rows, qlen entries (< 25)
    int qlen;
    int pass0;                  // query passes scored by earlier launches (row segments)
    int more;                   // != 0: a later launch scores the next row segment
    const int8_t* mat;          // 32x32, [query code][db code]; codes >= 24 score 0
    uint32_t bias2;             // dup16(open+extend): the biased zero of a lane
    uint32_t neg_e;             // dup16(-extend)
    int* counter;               // pairs claimed (zero before the launch)
    uint2* bnd;                 // boundary rows: 16 entries per 16-byte stream unit
    int* scores;                // per sorted record position
    int n_records;
    int* ovf_list;              // sorted positions for the 32-bit pass
    int* ovf_count;
    int ovf_thresh;             // biased lane value >= this may have wrapped
};

// Row-block map entry of a stacked batch: the query starts at this block.
constexpr int kFirstBit = 1 << 30;

// Arguments of the batched first-pass kernel (sw_wavefront.cuh, sw_batch).
struct BatchArgs {
    const uint4* db;
    const Pair2* pairs;
    int pair_begin;             // pairs [pair_begin, pair_begin + pair_count) of every stack
    int pair_count;
    const uint8_t* codes;       // the stacks' row codes back to back (24 = padding row)
    const uint32_t* stack_off;  // per stack: offset into codes
    const uint32_t* stack_rows; // per stack: rows
    const int* rb_map;          // per stack, per pass and thread: query | first bit, or -1
    const uint32_t* rb_off;     // per stack: offset into rb_map
    int nstacks;
    int* counters;              // one pair counter per stack (zero before)
    const int8_t* mat;
    uint32_t bias2;
    uint32_t neg_e;
    uint2* bnd;                 // per-group boundary rows
    size_t bnd_group;           // entries per group (2 per column of the longest pair)
    int* scores;                // [query][sorted position], zero before (atomicMax)
    int n_records;
    int* ovf_list;              // query * n_records + position
    int* ovf_count;
    int ovf_thresh;
    int ovf_cap;                // entries the overflow list holds
    const uint32_t* pair_ids;   // optional: global pair of each entry of pairs
};

__device__ __forceinline__ uint32_t prmt(uint32_t a, uint32_t b, uint32_t sel) {
    uint32_t r;
    asm("prmt.b32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(sel));
    return r;
}

// Sign-extending byte gather: low half <- int8 byte i of a, high half <- int8
// byte i of b (PRMT selector nibbles 8..15 replicate the selected byte's sign).
template <int I>
__device__ __forceinline__ uint32_t pack_s8x2(uint32_t a, uint32_t b) {
    constexpr uint32_t sel = (uint32_t)I | ((uint32_t)(I | 8) << 4) |
                             ((uint32_t)(4 + I) << 8) | ((uint32_t)((4 + I) | 8) << 12);
    return prmt(a, b, sel);
}

__device__ __forceinline__ uint32_t dup16(int v) {
    uint32_t u = (uint16_t)(int16_t)v;
    return u | (u << 16);
}

__device__ __forceinline__ int lo16(uint32_t v) { return (int)(int16_t)(v & 0xffffu); }
__device__ __forceinline__ int hi16(uint32_t v) { return (int)(int16_t)(v >> 16); }

}  // namespace swb
