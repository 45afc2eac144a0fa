// sw_wavefront.cuh -- first-pass Smith-Waterman kernel (packed int16x2, DPX).
//
// Replaces the reference GPU kernel Compute/computeScalarQP
// (src/CUDAKernel.cu:63-192), which scores one DB record per thread in int32
// with a texture profile and a per-thread local-memory strip buffer.
//
// Work unit: a PAIR of DB records of similar length (the DB layout sorts by
// length and pairs neighbours), stored as one column stream of 2-byte columns
// (low byte = record 2p, high byte = record 2p+1).  Both records are scored
// at once: every H/E/F/S register holds two signed 16-bit lanes and every
// cell update is a handful of DPX instructions.
//
// A group of T threads (T = 1..32, a power of two, inside one warp) owns one
// pair at a time.  Thread t holds R consecutive query rows in registers as two
// half-columns: the top R/2 rows work on column c while the bottom R/2 rows
// work on column c-1, so every step runs two independent F chains side by side
// (twice the instruction-level parallelism of one R-row chain).  Thread t's
// top half trails thread t-1's bottom half by one step (anti-diagonal
// wavefront): through warp shuffles it receives the H/F of the row above;
// each thread loads its own column's residue pair one step ahead (2-byte
// loads that the group's threads make from one 64-byte span).  A query
// longer than T*R rows is done in passes; between passes the last row's H/F
// per column goes through a double-buffered boundary row
// in global memory (written by thread T-1, read back two columns ahead by
// thread 0).  T = 1 is the inter-sequence form (one pair per thread); T > 1
// is the warp-cooperative intra-sequence form.
//
// Recurrence per cell (same order as the reference's ONE_CELL_UPDATE,
// src/AVXKernel.cpp:196-218, with the floor at 0 made explicit):
//   h  = max(diag + P, E, F, 0);  S = max(S, h)
//   hq = h - (open+extend);  E = max(E - extend, hq);  F = max(F - extend, hq)
// Lanes hold value + (open+extend) (see CellK), so every lane stays in
// [0, 32767] and the subtraction of open+extend cannot borrow across halves; a
// lane can only wrap upward after exceeding 32767 - max(matrix), which is the
// overflow threshold handed to the 32-bit re-score pass.  The residue chunk
// and the boundary row are prefetched so that no step waits on global memory.
//
// The query profile lives in shared memory as signed bytes, laid out so that
// each thread's 8-row chunk for a residue code is one 8-byte word and the 16
// lanes of a half-warp always read 16 distinct bank pairs, whatever residues
// the lanes look up (groups narrower than 16 get replicated slots).
#pragma once
#include "sw_device.cuh"

namespace swb {


template <int T>
struct GroupShape {
    static_assert(T == 1 || T == 2 || T == 4 || T == 8 || T == 16 || T == 32, "T");
    static constexpr int SLOTS = T >= 16 ? T : 16;
};

// Shared-memory bytes of the query profile for a query of qlen rows.
template <int T, int R>
__host__ __device__ constexpr size_t wf_smem_bytes(int qlen) {
    return (size_t)((qlen + T * R - 1) / (T * R)) * ((R + 7) / 8) * kCodes *
           GroupShape<T>::SLOTS * sizeof(uint2);
}


// Packed profile word of row I of a chunk: sign-extended int8 scores of the
// two records' residues (low half record 2p, high half record 2p+1).
__device__ __forceinline__ uint32_t pack_row(int i, const uint2& A, const uint2& B) {
    const uint32_t a = i < 4 ? A.x : A.y, b = i < 4 ? B.x : B.y;
    switch (i & 3) {
        case 0: return pack_s8x2<0>(a, b);
        case 1: return pack_s8x2<1>(a, b);
        case 2: return pack_s8x2<2>(a, b);
        default: return pack_s8x2<3>(a, b);
    }
}

// Constants of the cell recurrence.  Every H/E/F/S lane holds value + B with
// B = open+extend (so "score 0" is B): h' >= B keeps h' - (open+extend) >= 0
// in both halves, which makes the packed subtraction an ordinary 32-bit add.
struct CellK {
    uint32_t bias2;     // (B, B)
    uint32_t neg_q2;    // -(B << 16 | B) mod 2^32, i.e. subtract open+extend per half
    uint32_t neg_e2;    // (-extend, -extend)
};

// Row k's profile word from a chunk pair (A: record 2p's residue, B: record
// 2p+1's residue), sign-extended into the two 16-bit halves.
__device__ __forceinline__ uint32_t pack_k(int k, const uint2& A, const uint2& B) {
    return pack_row(k & 7, A, B);
}

// Reverse sweep of one half: H[k] <- max(H[k-1] + P_k, E_k) for k = HI-1 down
// to LO, with H[LO-1] replaced by diag.  p0/p1 point at the residues' chunk 0.
template <int R, int LO, int HI>
__device__ __forceinline__ void reverse_sweep(uint32_t (&H)[R], const uint32_t (&E)[R],
                                              const uint2* p0, const uint2* p1, int jstride,
                                              uint32_t diag) {
    constexpr int JLO = LO / 8, JHI = (HI - 1) / 8;
    uint2 A = p0[JHI * jstride];
    uint2 B = p1[JHI * jstride];
#pragma unroll
    for (int j = JHI; j >= JLO; --j) {
        uint2 An = A, Bn = B;
        if (j > JLO) {
            An = p0[(j - 1) * jstride];
            Bn = p1[(j - 1) * jstride];
        }
#pragma unroll
        for (int i = 7; i >= 0; --i) {
            const int k = j * 8 + i;
            if (k >= LO && k < HI) {
                const uint32_t up = (k > LO) ? H[k > LO ? k - 1 : LO] : diag;
                H[k] = __viaddmax_s16x2(up, pack_k(k, A, B), E[k]);
            }
        }
        A = An;
        B = Bn;
    }
}

// One forward cell: h = max(t, F, B); hq = h - (open+extend);
// E = max(E - extend, hq); F = max(F - extend, hq).
__device__ __forceinline__ void forward_cell(uint32_t& Hk, uint32_t& Ek, uint32_t& f,
                                             const CellK& K) {
    const uint32_t h = __vimax3_s16x2(Hk, f, K.bias2);
    Hk = h;
    const uint32_t hq = h + K.neg_q2;
    Ek = __viaddmax_s16x2(Ek, K.neg_e2, hq);
    f = __viaddmax_s16x2(f, K.neg_e2, hq);
}

// One column step of a thread's two halves: the top half (rows [0, R/2)) on
// column c with profile words t0/t1, the bottom half (rows [R/2, R)) on column
// c - 1 with b0/b1.  prev_h / f_in: H and F of the row above the top half
// (handed down by the thread above, or the boundary row); mid_h / mid_f carry
// the top half's last row from one column to the bottom half's next; out_h /
// out_f receive the bottom half's last row (what the thread below takes).
template <int R, int JSTRIDE>
__device__ __forceinline__ void column_step(uint32_t (&H)[R], uint32_t (&E)[R],
                                            const uint2* t0, const uint2* t1,
                                            const uint2* b0, const uint2* b1,
                                            uint32_t prev_h, uint32_t f_in,
                                            uint32_t& mid_h, uint32_t& mid_f,
                                            uint32_t& out_h, uint32_t& out_f,
                                            uint32_t& S_top, uint32_t& S_bot,
                                            const CellK& K) {
    constexpr int HALF = R / 2;
    const uint32_t Z = K.bias2;
    const uint32_t bot_diag = mid_h;
    uint32_t f_top = f_in, f_bot = mid_f;
    mid_h = H[HALF - 1];     // the top's last row one column back
    reverse_sweep<R, 0, HALF>(H, E, t0, t1, JSTRIDE, prev_h);
    reverse_sweep<R, HALF, R>(H, E, b0, b1, JSTRIDE, bot_diag);
#pragma unroll
    for (int i = 0; i < HALF; ++i) {
        forward_cell(H[i], E[i], f_top, K);
        forward_cell(H[HALF + i], E[HALF + i], f_bot, K);
        if (i & 1) S_top = __vimax3_s16x2(S_top, H[i - 1], H[i]);
        if (i & 1) S_bot = __vimax3_s16x2(S_bot, H[HALF + i - 1], H[HALF + i]);
        if (!(i & 1) && i == HALF - 1) {
            S_top = __vimax3_s16x2(S_top, H[i], Z);
            S_bot = __vimax3_s16x2(S_bot, H[HALF + i], Z);
        }
    }
    mid_f = f_top;
    out_h = H[R - 1];
    out_f = f_bot;
}

// Chunks of 8 profile rows that rows [LO, HI) of a thread span.
template <int LO, int HI>
struct HalfChunks {
    static constexpr int JLO = LO / 8, JHI = (HI - 1) / 8, N = JHI - JLO + 1;
};

// The profile words rows [LO, HI) read for one column: chunk j of record
// 2p's residue in A[j - JLO], of record 2p+1's in B[j - JLO].
template <int LO, int HI>
__device__ __forceinline__ void load_words(uint2 (&A)[HalfChunks<LO, HI>::N],
                                           uint2 (&B)[HalfChunks<LO, HI>::N],
                                           const uint2* p0, const uint2* p1, int jstride) {
#pragma unroll
    for (int j = 0; j < HalfChunks<LO, HI>::N; ++j) {
        A[j] = p0[(HalfChunks<LO, HI>::JLO + j) * jstride];
        B[j] = p1[(HalfChunks<LO, HI>::JLO + j) * jstride];
    }
}

// reverse_sweep with the profile words already in registers.
template <int R, int LO, int HI>
__device__ __forceinline__ void reverse_sweep_w(uint32_t (&H)[R], const uint32_t (&E)[R],
                                                const uint2 (&A)[HalfChunks<LO, HI>::N],
                                                const uint2 (&B)[HalfChunks<LO, HI>::N],
                                                uint32_t diag) {
    constexpr int JLO = HalfChunks<LO, HI>::JLO, JHI = HalfChunks<LO, HI>::JHI;
#pragma unroll
    for (int j = JHI; j >= JLO; --j) {
#pragma unroll
        for (int i = 7; i >= 0; --i) {
            const int k = j * 8 + i;
            if (k >= LO && k < HI) {
                const uint32_t up = (k > LO) ? H[k > LO ? k - 1 : LO] : diag;
                H[k] = __viaddmax_s16x2(up, pack_k(k, A[j - JLO], B[j - JLO]), E[k]);
            }
        }
    }
}

// column_step with both halves' profile words already in registers.
template <int R>
__device__ __forceinline__ void column_step_w(
    uint32_t (&H)[R], uint32_t (&E)[R], const uint2 (&tA)[HalfChunks<0, R / 2>::N],
    const uint2 (&tB)[HalfChunks<0, R / 2>::N], const uint2 (&bA)[HalfChunks<R / 2, R>::N],
    const uint2 (&bB)[HalfChunks<R / 2, R>::N], uint32_t prev_h, uint32_t f_in, uint32_t& mid_h,
    uint32_t& mid_f, uint32_t& out_h, uint32_t& out_f, uint32_t& S_top, uint32_t& S_bot,
    const CellK& K) {
    constexpr int HALF = R / 2;
    const uint32_t Z = K.bias2;
    const uint32_t bot_diag = mid_h;
    uint32_t f_top = f_in, f_bot = mid_f;
    mid_h = H[HALF - 1];
    reverse_sweep_w<R, 0, HALF>(H, E, tA, tB, prev_h);
    reverse_sweep_w<R, HALF, R>(H, E, bA, bB, bot_diag);
#pragma unroll
    for (int i = 0; i < HALF; ++i) {
        forward_cell(H[i], E[i], f_top, K);
        forward_cell(H[HALF + i], E[HALF + i], f_bot, K);
        if (i & 1) S_top = __vimax3_s16x2(S_top, H[i - 1], H[i]);
        if (i & 1) S_bot = __vimax3_s16x2(S_bot, H[HALF + i - 1], H[HALF + i]);
        if (!(i & 1) && i == HALF - 1) {
            S_top = __vimax3_s16x2(S_top, H[i], Z);
            S_bot = __vimax3_s16x2(S_bot, H[HALF + i], Z);
        }
    }
    mid_f = f_top;
    out_h = H[R - 1];
    out_f = f_bot;
}

// Query profile of one query -> shared memory (whole block; the caller
// synchronises).  Layout [pass][chunk][code][slot] of 8-byte words holding the
// signed scores of 8 consecutive rows of the slot's thread.
template <int T, int R>
__device__ __forceinline__ void build_profile(uint2* prof, const uint8_t* query, int qlen,
                                              const int8_t* mat, int P) {
    constexpr int NJ = (R + 7) / 8;
    constexpr int SLOTS = GroupShape<T>::SLOTS;
    constexpr int JSTRIDE = kCodes * SLOTS;
    const int rows_per_pass = T * R;
    const int total = P * NJ * JSTRIDE;
    for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
        const int slot = idx % SLOTS;
        int rest = idx / SLOTS;
        const int d = rest % kCodes;
        rest /= kCodes;
        const int j = rest % NJ;
        const int p = rest / NJ;
        const int row0 = p * rows_per_pass + (slot % T) * R + j * 8;
        uint32_t w0 = 0u, w1 = 0u;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int row = row0 + i;
            int v = 0;
            if (row < qlen) v = mat[(query[row] & 31) * 32 + d];
            const uint32_t b = (uint32_t)(uint8_t)(int8_t)v << (8 * (i & 3));
            if (i < 4) w0 |= b; else w1 |= b;
        }
        prof[idx] = make_uint2(w0, w1);
    }
}

// What one call of run_stream works on.
struct RunArgs {
    const uint4* db;            // pair column streams
    const Pair2* pairs;         // pair table, ncols descending
    int pair_begin;             // pairs [pair_begin, pair_begin + pair_count)
    int pair_count;
    int* counter;               // pairs of the range claimed so far
    int P;                      // query passes of T*R rows
    // A query too long for one launch's profile is scored in row segments by
    // consecutive launches (plain search only): pass0 = passes of the query
    // before this launch's first one (that pass reads the boundary row the
    // previous launch's last pass wrote), more != 0 = a later launch
    // continues from this launch's last pass (which then writes the boundary
    // row).  0, 0 for a query that fits one launch.
    int pass0;
    int more;
    uint32_t bias2, neg_e;      // see CellK
    uint2* bnd;                 // boundary rows between passes
    size_t bnd_group;           // 0: per-pair rows at bnd + 16*off16; else this many
                                // entries per group at bnd + group * bnd_group
    int* scores;                // scores of this query, by sorted position
    int n_records;
    int* ovf_list;              // (ovf_base + position) of lanes for the 32-bit pass
    int* ovf_count;
    int ovf_base;
    int ovf_thresh;             // biased lane value >= this may have wrapped
    int ovf_cap;                // entries the overflow list holds
    const uint32_t* pair_ids;   // optional: global pair of table entry i (a
                                // permuted table); null = identity
    // stacked queries (batched search): several queries share the rows of one
    // "stack"; entry pass*T + t holds the query of thread t's rows in that pass
    // (-1: padding) with bit 30 set when the query starts at the thread's first
    // row.  Scores then go to scores[query * n_records + position] by atomicMax.
    const int* rb_map;
};



// A record whose first-pass lane may have wrapped, while its query is scored
// in row segments by several launches: listed once for the 32-bit pass, which
// overwrites this value with the exact score.
constexpr int kListed = 0x7fffffff;

// Plain search: a record's first-pass score (biased lane value s) at its
// sorted position.  A lane that may have wrapped lists the record for the
// 32-bit pass.  With the query in row segments (pass0 / more) the score is
// the maximum over the segments, and a listed record keeps kListed so that a
// later segment does not list it again.
__device__ __forceinline__ void put_score(const RunArgs& a, int pos, int s, int bias) {
    if (a.pass0 == 0 && !a.more) {
        a.scores[pos] = s - bias;
        if (s >= a.ovf_thresh) {
            const int j = atomicAdd(a.ovf_count, 1);
            if (j < a.ovf_cap) a.ovf_list[j] = a.ovf_base + pos;
        }
        return;
    }
    const int prev = a.scores[pos];
    if (prev == kListed) return;
    if (s >= a.ovf_thresh) {
        a.scores[pos] = kListed;
        const int j = atomicAdd(a.ovf_count, 1);
        if (j < a.ovf_cap) a.ovf_list[j] = a.ovf_base + pos;
    } else {
        a.scores[pos] = max(prev, s - bias);
    }
}

// The group loop: every group of T threads claims pairs from the range and
// scores them against the query (or query stack) whose profile is in prof;
// returns when the range is exhausted (warp-wide).
//
// The groups stream: each thread moves on to the group's next segment (the
// next pass of the pair, or the next pair) as soon as its own columns of the
// current one are done, so the wavefront fills once per range instead of
// draining for 2T-1 steps at the end of every pass (9 % of the steps at
// T = 16 on a DB of ~350-residue records, 18 % at T = 32).  Thread t's top
// half is on column c of a segment at group step G + c + 2t and its bottom
// half one column behind, so for one step after a switch the two halves work
// on different segments: the bottom keeps the profile base and boundary-row
// view the top had a step earlier.
//   * The pair descriptor (index, stream offset, columns) goes from thread t-1
//     to thread t by shuffle at t's switch, 2 steps after t-1's.
//   * A thread's maximum over a finished pair (plain) or pass (stacked) is
//     complete one step after its top leaves it; it travels down the group in
//     a third shuffle, each thread adding its own.  Plain: thread T-1 writes
//     the pair's scores.  Stacked (several queries share the rows of a pass,
//     aligned to threads): the chain restarts at a thread whose rows begin a
//     query, and the last thread of each query's rows adds the query's
//     maximum with atomicMax (a query longer than a pass is merged over its
//     passes the same way).
//   * Thread 0 of pass p+1 reads boundary column j at step G' + j - 2 while
//     thread T-1 of pass p wrote it at step G + 2T - 1 + j, so a segment that
//     a later pass depends on lasts at least 2T + 2 steps (padding columns of
//     zero-score residues, which cannot raise a score); every other segment
//     lasts at least 3 steps, which keeps the descriptor and maximum hand-offs
//     one segment apart.
template <int T, int R, bool STACKED>
__device__ __forceinline__ void run_stream(const RunArgs& a, const uint2* prof) {
    static_assert(R % 2 == 0 && R >= 4, "R");
    constexpr int NJ = (R + 7) / 8;    // 8-row profile chunks per thread (last one partial)
    constexpr int HALF = R / 2;
    constexpr int SLOTS = GroupShape<T>::SLOTS;
    constexpr int JSTRIDE = kCodes * SLOTS;
    constexpr int PSTRIDE = NJ * JSTRIDE;     // profile words per pass
    constexpr unsigned FULL = 0xffffffffu;
    const int P = a.P;
    const int lane = threadIdx.x & 31;
    const int t = lane & (T - 1);
    const int slot = lane & (SLOTS - 1);
    const unsigned gmask = (T == 32) ? FULL : (((1u << T) - 1u) << (lane & ~(T - 1)));
    CellK K;
    K.bias2 = a.bias2;
    K.neg_q2 = 0u - a.bias2;
    K.neg_e2 = a.neg_e;
    const uint32_t Z = a.bias2;        // biased zero of both lanes
    const int bias = (int)(a.bias2 & 0xffffu);
    const int pair_count = a.pair_count;
    const int dep_steps = 2 * T + 2;
    uint2* const grp_bnd =
        a.bnd + (size_t)((blockIdx.x * blockDim.x + threadIdx.x) / T) * a.bnd_group;

    // rows [0, HALF): top half, on column c; rows [HALF, R): bottom half, on
    // column c - 1 (c = the top's column in its segment)
    uint32_t H[R], E[R];
#pragma unroll
    for (int k = 0; k < R; ++k) {
        H[k] = Z;
        E[k] = Z;
    }
    uint32_t S_top = Z, S_bot = Z, S_pend = Z, acc_out = Z;
    uint32_t out_h = Z, out_f = Z, prev_h = Z, mid_h = Z, mid_f = Z;
    uint32_t d_bot = kPadPair, d_cur = kPadPair;
    // the top half's profile offsets of the last column it computed: the
    // bottom half takes them one step later (its profile base is then the one
    // the top used, see below)
    int po0 = kZeroCode * SLOTS, po1 = kZeroCode * SLOTS;
    // the top half's segment
    int pair = 0, pass = 0, ncols = 0, nst = 0, c = 0;
    uint32_t off16 = 0u;
    const unsigned short* col = reinterpret_cast<const unsigned short*>(a.db);
    const uint2* prof_t = prof + slot;
    uint2* wrow = a.bnd;       // boundary row this pass writes (thread T-1) ...
    int wlim = 0;              // ... for columns below this (0: last pass)
    // stacked: this thread's query in the top's pass (-1: padding), whether the
    // query starts at its first row, whether its last row ends the query's rows
    int my_q = 0;
    bool my_first = false, my_last = false;
    // the bottom half's view: the top's of the previous step (the profile base
    // and boundary row change only when the bottom reaches a segment's column 0)
    const uint2* prof_b = prof_t;
    uint2* b_wrow = wrow;
    int b_wlim = 0, b_col = -1;
    // a segment whose maximum is being finished
    int fpair = 0, f_q = 0;
    bool fpend = false, f_first = false, f_last = false, fin = false;
    // thread 0: the next pair (claimed one pair ahead) and the boundary row
    // read by passes after the first (two columns prefetched)
    int next = 0, nload = -1;   // nload: the step of the first pass that loads its entry
    Pair2 ninfo{0u, 0u};
    uint2 bq0 = make_uint2(Z, Z), bq1 = bq0;
    const uint2* rrow = a.bnd;

    // the boundary rows are double-buffered by the parity of the pass's index
    // in the whole query; a launch's last pass writes one only when a later
    // launch reads it (that launch starts after this one has finished, so the
    // 2T + 2 minimum only applies to passes read inside the launch)
#define SWS_SET_SEG()                                                          \
    {                                                                          \
        const int lo = (pass + 1 < P) ? dep_steps : 3;                         \
        nst = ncols > lo ? ncols : lo;                                         \
        col = reinterpret_cast<const unsigned short*>(a.db) + (size_t)off16 * 8; \
        uint2* const pb = a.bnd_group ? grp_bnd : a.bnd + (size_t)off16 * 16;  \
        wrow = pb + ((a.pass0 + pass) & 1);                                    \
        wlim = (pass + 1 < P || a.more) ? ncols : 0;                           \
        rrow = pb + ((a.pass0 + pass - 1) & 1);                                \
        prof_t = prof + pass * PSTRIDE + slot;                                 \
        nload = (pass == 0) ? (nst < 9 ? nst - 1 : 8) : -1;                    \
        if (STACKED) {                                                         \
            const int rb = a.rb_map[pass * T + t];                             \
            const int rn = (t + 1 < T) ? a.rb_map[pass * T + t + 1] : -1;      \
            my_first = (rb & kFirstBit) != 0;                                  \
            my_q = (rb < 0) ? -1 : (rb & (kFirstBit - 1));                     \
            my_last = rn < 0 || (rn & kFirstBit) != 0;                         \
        }                                                                      \
    }

    {
        int v = 0;
        if (t == 0) v = atomicAdd(a.counter, 1);
        v = __shfl_sync(gmask, v, 0, T);
        pair = v;
        if (v < pair_count) {
            const Pair2 pr = a.pairs[a.pair_begin + v];
            off16 = pr.off16;
            ncols = (int)pr.ncols;
            if (t == 0) next = atomicAdd(a.counter, 1);
        } else {
            fin = true;
        }
        SWS_SET_SEG()
        prof_b = prof_t;
        b_wrow = wrow;
        b_wlim = wlim;
        c = -2 * t;
        d_cur = (t == 0 && ncols > 0) ? (uint32_t)__ldg(col) : kPadPair;
        if (t == 0 && a.pass0 > 0) {
            if (ncols > 0) bq0 = rrow[0];
            if (ncols > 1) bq1 = rrow[2];
        }
    }

    while (!__all_sync(FULL, fin)) {
        if (P > 1) __syncwarp();      // orders the boundary row's stores and loads
        // thread t-1's bottom half handed down the last-row H and F of the
        // column it processed in the previous step
        uint32_t h_in = __shfl_up_sync(FULL, out_h, 1, T);
        uint32_t f_in = __shfl_up_sync(FULL, out_f, 1, T);
        const uint32_t acc_in = __shfl_up_sync(FULL, acc_out, 1, T);
        const uint32_t d_in = d_cur;
        {
            const int c1 = c + 1;     // this thread's top column next step
            d_cur = (c1 >= 0 && c1 < ncols) ? (uint32_t)__ldg(col + c1) : kPadPair;
        }
        if (t == 0) {
            h_in = Z;
            f_in = Z;
            if (a.pass0 + pass > 0 && c < ncols) {
                h_in = bq0.x;
                f_in = bq0.y;
                bq0 = bq1;
                if (c + 2 < ncols) bq1 = rrow[2 * (c + 2)];
            }
            // the next pair's table entry, once its claim has returned
            if (c == nload && next < pair_count) ninfo = a.pairs[a.pair_begin + next];
        }
        if (STACKED && my_first) {   // a query starts here: nothing flows in from above
            h_in = Z;
            f_in = Z;
        }
        if (!fin && c >= 0) {
            // a column past the segment's end runs on zero-score residues:
            // like a trailing padding column it cannot raise any score
            const int o0 = (int)(d_in & 0xffu) * SLOTS, o1 = (int)((d_in >> 8) & 0xffu) * SLOTS;
            column_step<R, JSTRIDE>(H, E, prof_t + o0, prof_t + o1,
                                    prof_b + (int)(d_bot & 0xffu) * SLOTS,
                                    prof_b + (int)((d_bot >> 8) & 0xffu) * SLOTS, prev_h, f_in,
                                    mid_h, mid_f, out_h, out_f, S_top, S_bot, K);
            po0 = o0;
            po1 = o1;
            if (t == T - 1 && b_col >= 0 && b_col < b_wlim)
                b_wrow[2 * b_col] = make_uint2(out_h, out_f);
        }
        prev_h = h_in;
        d_bot = d_in;
        b_col = c;
        // segment events, one warp vote per step: a finished maximum, the
        // bottom entering a segment, the top leaving one
        const bool ev = fpend || c == 0 || (!fin && c == nst - 1);
        if (__any_sync(FULL, ev)) {
            if (fpend) {
                // the bottom has just done the finished segment's last column:
                // this thread's maximum joins the chain down the group
                fpend = false;
                uint32_t m = __vimax3_s16x2(S_pend, S_bot, Z);
                if (STACKED) {
                    if (t > 0 && !f_first) m = __vimax3_s16x2(m, acc_in, Z);
                    acc_out = m;
                    if (f_q >= 0 && f_last) {
                        const int gp = a.pair_ids ? (int)a.pair_ids[a.pair_begin + fpair]
                                                  : a.pair_begin + fpair;
                        const int pos = 2 * gp;
                        const int s0 = lo16(m), s1 = hi16(m);
                        const int qb = f_q * a.n_records;
                        atomicMax(a.scores + qb + pos, s0 - bias);
                        if (s0 >= a.ovf_thresh) {
                            const int j = atomicAdd(a.ovf_count, 1);
                            if (j < a.ovf_cap) a.ovf_list[j] = qb + pos;
                        }
                        if (pos + 1 < a.n_records) {
                            atomicMax(a.scores + qb + pos + 1, s1 - bias);
                            if (s1 >= a.ovf_thresh) {
                                const int j = atomicAdd(a.ovf_count, 1);
                                if (j < a.ovf_cap) a.ovf_list[j] = qb + pos + 1;
                            }
                        }
                    }
                } else {
                    if (t > 0) m = __vimax3_s16x2(m, acc_in, Z);
                    acc_out = m;
                    if (t == T - 1) {
                        const int pos = 2 * (a.pair_begin + fpair);
                        put_score(a, pos, lo16(m), bias);
                        if (pos + 1 < a.n_records) put_score(a, pos + 1, hi16(m), bias);
                    }
                }
                S_bot = Z;
                if (pair >= pair_count) fin = true;
            }
            if (c == 0) {   // the bottom starts this segment's column 0 next step
#pragma unroll
                for (int k = HALF; k < R; ++k) {
                    H[k] = Z;
                    E[k] = Z;
                }
                prof_b = prof_t;
                b_wrow = wrow;
                b_wlim = wlim;
            }
            // the top leaves its segment: set up the next one
            const bool adv = !fin && c == nst - 1;
            const int up_pair = __shfl_up_sync(FULL, pair, 1, T);
            const uint32_t up_off = __shfl_up_sync(FULL, off16, 1, T);
            const int up_ncols = __shfl_up_sync(FULL, ncols, 1, T);
            if (adv) {
                const bool last_pass = pass + 1 >= P;
                if (STACKED || last_pass) {   // the maximum being finished
                    S_pend = S_top;
                    S_top = Z;
                    fpair = pair;
                    f_q = my_q;
                    f_first = my_first;
                    f_last = my_last;
                    fpend = true;
                }
                if (!last_pass) {
                    ++pass;
                } else {
                    pass = 0;
                    if (t == 0) {
                        pair = next;
                        off16 = ninfo.off16;
                        ncols = (int)ninfo.ncols;
                        if (pair < pair_count) next = atomicAdd(a.counter, 1);
                    } else {
                        pair = up_pair;
                        off16 = up_off;
                        ncols = up_ncols;
                    }
                    if (pair >= pair_count) ncols = 0;
                }
                SWS_SET_SEG()
                c = -1;
#pragma unroll
                for (int k = 0; k < HALF; ++k) {
                    H[k] = Z;
                    E[k] = Z;
                }
                prev_h = Z;
                if (t == 0 && a.pass0 + pass > 0) {
                    if (ncols > 0) bq0 = rrow[0];
                    if (ncols > 1) bq1 = rrow[2];
                }
                d_cur = (ncols > 0) ? (uint32_t)__ldg(col) : kPadPair;
            }
        }
        ++c;

        // Plain steps: as many steps as every lane of the warp can take with
        // no segment event (c stays in [1, nst - 2]: no maximum to finish, no
        // bottom reset, no segment switch), no bounds guard (the residue of
        // column c + 1 and thread 0's boundary column c + 2 lie inside the
        // pair) and no pending table-entry load.  In them the bottom half's
        // profile base and boundary row equal the top's, so the bottom takes
        // the top's profile offsets of the step before, and the warp runs
        // without votes or per-step checks.
        {
            int k = 0;
            if (!fin && c >= 1 && !(t == 0 && c <= nload)) {
                const int last = min(nst - 2, ncols - 3);
                k = max(last - c + 1, 0);
            }
            k = (int)__reduce_min_sync(FULL, (unsigned)k);
            const bool rd0 = t == 0 && a.pass0 + pass > 0;            // boundary row in
            const bool zin = (t == 0 && a.pass0 + pass == 0) || (STACKED && my_first);
            const bool wr = t == T - 1 && wlim > 0;                   // boundary row out
            if constexpr (R >= 40 && !(R == 64 && (T == 8 || T == 16))) {
                // With 40 rows or more per thread there are registers to hold the
                // next step's profile words: they are loaded at the start of a step
                // from residues already in registers, so no step waits for its
                // profile (+1.4..2.6 % at 16x48 and 8x40, +0.6 % at 16x56; at 32x24
                // it measured 1.2..1.6 % slower, so fewer rows keep the loads in the
                // step, and so do 16x64 and 8x64, 2.3 % and 0.6 % faster without it
                // at 249 registers, while 4x64 and 32x64 keep it: 0.7 % and 0.2 %).
                if (k > 0) {
                    constexpr int NT = HalfChunks<0, HALF>::N, NB = HalfChunks<HALF, R>::N;
                    // this step's words (top: the residues of column c; bottom: the
                    // top's of the step before) and the next step's top residues
                    uint2 tA[NT], tB[NT], bA[NB], bB[NB];
                    load_words<0, HALF>(tA, tB, prof_t + (int)(d_cur & 0xffu) * SLOTS,
                                        prof_t + (int)((d_cur >> 8) & 0xffu) * SLOTS, JSTRIDE);
                    load_words<HALF, R>(bA, bB, prof_t + po0, prof_t + po1, JSTRIDE);
                    uint32_t d_nx = (uint32_t)__ldg(col + c + 1);
#pragma unroll 2
                    for (; k > 0; --k) {
                        if (P > 1) __syncwarp();
                        uint32_t h_in = __shfl_up_sync(FULL, out_h, 1, T);
                        uint32_t f_in = __shfl_up_sync(FULL, out_f, 1, T);
                        const uint32_t d_in = d_cur;
                        d_cur = d_nx;
                        // column c + 2 lies inside the pair in a plain step
                        d_nx = (uint32_t)__ldg(col + c + 2);
                        if (rd0) {
                            h_in = bq0.x;
                            f_in = bq0.y;
                            bq0 = bq1;
                            bq1 = rrow[2 * (c + 2)];
                        }
                        if (zin) {
                            h_in = Z;
                            f_in = Z;
                        }
                        const int o0 = (int)(d_in & 0xffu) * SLOTS, o1 = (int)((d_in >> 8) & 0xffu) * SLOTS;
                        // the next step's words: its top takes column c + 1, its
                        // bottom this step's top column
                        uint2 nA[NT], nB[NT], mA[NB], mB[NB];
                        load_words<0, HALF>(nA, nB, prof_t + (int)(d_cur & 0xffu) * SLOTS,
                                            prof_t + (int)((d_cur >> 8) & 0xffu) * SLOTS, JSTRIDE);
                        load_words<HALF, R>(mA, mB, prof_t + o0, prof_t + o1, JSTRIDE);
                        column_step_w<R>(H, E, tA, tB, bA, bB, prev_h, f_in, mid_h, mid_f, out_h,
                                         out_f, S_top, S_bot, K);
                        if (wr) wrow[2 * (c - 1)] = make_uint2(out_h, out_f);
#pragma unroll
                        for (int j = 0; j < NT; ++j) {
                            tA[j] = nA[j];
                            tB[j] = nB[j];
                        }
#pragma unroll
                        for (int j = 0; j < NB; ++j) {
                            bA[j] = mA[j];
                            bB[j] = mB[j];
                        }
                        po0 = o0;
                        po1 = o1;
                        prev_h = h_in;
                        d_bot = d_in;
                        b_col = c;
                        ++c;
                    }
                }
            } else {
                // two steps per iteration (+0.9 % over the sweep, measured)
#pragma unroll 2
                for (; k > 0; --k) {
                    if (P > 1) __syncwarp();
                    uint32_t h_in = __shfl_up_sync(FULL, out_h, 1, T);
                    uint32_t f_in = __shfl_up_sync(FULL, out_f, 1, T);
                    const uint32_t d_in = d_cur;
                    d_cur = (uint32_t)__ldg(col + c + 1);
                    if (rd0) {
                        h_in = bq0.x;
                        f_in = bq0.y;
                        bq0 = bq1;
                        bq1 = rrow[2 * (c + 2)];
                    }
                    if (zin) {
                        h_in = Z;
                        f_in = Z;
                    }
                    const int o0 = (int)(d_in & 0xffu) * SLOTS, o1 = (int)((d_in >> 8) & 0xffu) * SLOTS;
                    column_step<R, JSTRIDE>(H, E, prof_t + o0, prof_t + o1, prof_t + po0, prof_t + po1,
                                            prev_h, f_in, mid_h, mid_f, out_h, out_f, S_top, S_bot, K);
                    if (wr) wrow[2 * (c - 1)] = make_uint2(out_h, out_f);
                    po0 = o0;
                    po1 = o1;
                    prev_h = h_in;
                    d_bot = d_in;
                    b_col = c;
                    ++c;
                }
            }
        }
    }
#undef SWS_SET_SEG
}

// Plain search: one query, the pairs of one range.
template <int T, int R, int BLOCK>
__global__ void __launch_bounds__(BLOCK, 1) sw_wavefront(const WfArgs a) {
    extern __shared__ uint2 prof[];
    const int P = (a.qlen + T * R - 1) / (T * R);
    build_profile<T, R>(prof, a.query, a.qlen, a.mat, P);
    __syncthreads();
    RunArgs r;
    r.db = a.db;
    r.pairs = a.pairs;
    r.pair_begin = a.pair_begin;
    r.pair_count = a.pair_count;
    r.counter = a.counter;
    r.P = P;
    r.pass0 = a.pass0;
    r.more = a.more;
    r.bias2 = a.bias2;
    r.neg_e = a.neg_e;
    r.bnd = a.bnd;
    r.bnd_group = 0;
    r.scores = a.scores;
    r.n_records = a.n_records;
    r.ovf_list = a.ovf_list;
    r.ovf_count = a.ovf_count;
    r.ovf_base = 0;
    r.ovf_thresh = a.ovf_thresh;
    r.ovf_cap = a.n_records + 1;
    r.pair_ids = nullptr;
    r.rb_map = nullptr;
    run_stream<T, R, false>(r, prof);
}

// Batched search: one persistent launch over a list of query stacks (each
// stack holds one long query or several short ones, aligned to R-row
// blocks).  Every block walks the stacks in order; for each it rebuilds the
// profile in shared memory and its groups claim record pairs from that
// stack's counter (the device work queue), so the whole grid moves through the
// batch without a launch per query, and a block only waits for its own groups
// at a stack switch.
template <int T, int R, int BLOCK>
__global__ void __launch_bounds__(BLOCK, 1) sw_batch(const BatchArgs a) {
    extern __shared__ uint2 prof[];
    for (int i = 0; i < a.nstacks; ++i) {
        const int rows = (int)a.stack_rows[i];
        const int P = (rows + T * R - 1) / (T * R);
        __syncthreads();        // every group is done with the previous profile
        build_profile<T, R>(prof, a.codes + a.stack_off[i], rows, a.mat, P);
        __syncthreads();
        RunArgs r;
        r.db = a.db;
        r.pairs = a.pairs;
        r.pair_begin = a.pair_begin;
        r.pair_count = a.pair_count;
        r.counter = a.counters + i;
        r.P = P;
        r.pass0 = 0;
        r.more = 0;
        r.bias2 = a.bias2;
        r.neg_e = a.neg_e;
        r.bnd = a.bnd;
        r.bnd_group = a.bnd_group;
        r.scores = a.scores;
        r.n_records = a.n_records;
        r.ovf_list = a.ovf_list;
        r.ovf_count = a.ovf_count;
        r.ovf_base = 0;
        r.ovf_thresh = a.ovf_thresh;
        r.ovf_cap = a.ovf_cap;
        r.pair_ids = a.pair_ids;
        r.rb_map = a.rb_map + a.rb_off[i];
        run_stream<T, R, true>(r, prof);
    }
}

}  // namespace swb
