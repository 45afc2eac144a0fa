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
// A group of T threads (T = 1..32, a power of two, inside one warp) is a
// systolic pipeline.  Thread t holds R consecutive query rows in registers as
// two half-columns: the top R/2 rows work on column c while the bottom R/2
// rows work on column c-1, so every step runs two independent F chains side
// by side (twice the instruction-level parallelism of one R-row chain).
// Each thread receives through warp shuffles the H/F of the row above (thread
// t-1's bottom half, one step earlier), the residue pair and the column's
// tags, and passes its bottom half's column on to thread t+1.  Thread 0 feeds the pipeline with a
// continuous stream of "segments" -- (pair, pass) column runs, one pass per
// T*R query rows -- so the pipeline never drains between passes or pairs;
// each thread resets its rows when the first column of a new segment reaches
// it.  Between passes of a pair the last row's H/F per column goes through a
// double-buffered boundary row in global memory (written by thread T-1, read
// back two columns ahead by thread 0 of a later segment).  T = 1 is the
// inter-sequence form (one pair per thread); T > 1 is the warp-cooperative
// intra-sequence form.
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
    return (size_t)((qlen + T * R - 1) / (T * R)) * (R / 8) * kCodes *
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

// 32-bit integer multiply-add (kept as IMAD: the multiplier is a run-time 1),
// used for the packed subtraction h - (open+extend) on lanes that are biased so
// that no half can borrow from the other.
__device__ __forceinline__ uint32_t mad_u32(uint32_t a, uint32_t b, uint32_t c) {
    uint32_t r;
    asm("mad.lo.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(c));
    return r;
}

// Constants of the cell recurrence.  Every H/E/F/S lane holds value + B with
// B = open+extend (so "score 0" is B): h' >= B keeps h' - (open+extend) >= 0
// in both halves, which makes the packed subtraction an ordinary 32-bit add.
struct CellK {
    uint32_t bias2;     // (B, B)
    uint32_t neg_q2;    // -(B << 16 | B) mod 2^32, i.e. subtract open+extend per half
    uint32_t neg_e2;    // (-extend, -extend)
    uint32_t one;       // 1, from a kernel argument
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
    const uint32_t hq = mad_u32(h, K.one, K.neg_q2);
    Ek = __viaddmax_s16x2(Ek, K.neg_e2, hq);
    f = __viaddmax_s16x2(f, K.neg_e2, hq);
}

// Tags carried with each column word down the pipeline (low 16 bits: the
// residue pair; bits 22..31: the pass of the column's segment).
constexpr uint32_t kValid = 1u << 16;      // a real column
constexpr uint32_t kFirst = 1u << 17;      // first column of a segment
constexpr uint32_t kLast = 1u << 18;       // last column of a segment
constexpr uint32_t kLastPass = 1u << 19;   // segment is the pair's last pass
constexpr uint32_t kFirstPass = 1u << 20;  // segment is the pair's first pass
constexpr uint32_t kDone = 1u << 21;       // the feeder has no more work
constexpr int kPassShift = 22;

template <int T, int R, int BLOCK>
__global__ void __launch_bounds__(BLOCK, 1) sw_wavefront(const WfArgs a) {
    static_assert(R % 8 == 0 && R >= 8, "R");
    constexpr int NJ = R / 8;
    constexpr int HALF = R / 2;
    constexpr int SLOTS = GroupShape<T>::SLOTS;
    constexpr int JSTRIDE = kCodes * SLOTS;
    extern __shared__ uint2 prof[];

    const int rows_per_pass = T * R;
    const int P = (a.qlen + rows_per_pass - 1) / rows_per_pass;

    // ---- query profile -> shared memory (once per block) ----
    {
        const int total = P * NJ * JSTRIDE;
        for (int idx = threadIdx.x; idx < total; idx += BLOCK) {
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
                if (row < a.qlen) v = a.mat[(a.query[row] & 31) * 32 + d];
                const uint32_t b = (uint32_t)(uint8_t)(int8_t)v << (8 * (i & 3));
                if (i < 4) w0 |= b; else w1 |= b;
            }
            prof[idx] = make_uint2(w0, w1);
        }
    }
    __syncthreads();

    constexpr unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int t = lane & (T - 1);
    const int slot = lane & (SLOTS - 1);
    CellK K;
    K.bias2 = a.bias2;
    K.neg_q2 = 0u - a.bias2;
    K.neg_e2 = a.neg_e;
    K.one = a.one;
    const uint32_t Z = a.bias2;        // biased zero of both lanes
    const int bias = (int)(a.bias2 & 0xffffu);
    const int pair_count = a.pair_count;

    // ---- pipeline state (every thread) ----
    // rows [0, HALF): top half, on the column of d_top; rows [HALF, R): bottom
    // half, one column behind, on the column of d_bot.
    uint32_t H[R], E[R];
#pragma unroll
    for (int k = 0; k < R; ++k) {
        H[k] = Z;
        E[k] = Z;
    }
    uint32_t S_top = Z, S_bot = Z, S_topfin = Z;
    uint32_t out_h = Z, out_f = Z, out_s = Z, prev_h = Z;
    uint32_t mid_h = Z, mid_f = Z;     // top's last row: H one column back, F out
    uint32_t d_bot = 0u, o_bot = 0u, p_bot = 0u;   // the bottom half's next column
    uint32_t d_out = 0u, o_out = 0u, p_out = 0u;   // the column it just processed
    int col_bot = 0;
    bool finished = false;

    // ---- feeder state (meaningful in thread 0 of each group) ----
    int f_pair = 0, f_next = 0, f_pass = 0, f_col = 0, f_ncols = 0, f_start = -(1 << 20);
    uint32_t f_off = 0u;
    bool f_done = false, f_open = false;
    Pair2 f_ninfo{0u, 0u};
    uint4 dcur = make_uint4(0u, 0u, 0u, 0u), dnext = dcur;
    uint2 bq0 = make_uint2(Z, Z), bq1 = bq0;
    if (t == 0) {
        f_pair = atomicAdd(a.counter, 1);
        if (f_pair >= pair_count) {
            f_done = true;
        } else {
            const Pair2 pr = a.pairs[a.pair_begin + f_pair];
            f_off = pr.off16;
            f_ncols = (int)pr.ncols;
        }
    }

    for (int step = 0; !__all_sync(FULL, finished); ++step) {
        // what the thread above handed down: the column its bottom half
        // processed in the previous step, with that column's outputs
        uint32_t d_in = __shfl_up_sync(FULL, d_out, 1, T);
        uint32_t h_in = __shfl_up_sync(FULL, out_h, 1, T);
        uint32_t f_in = __shfl_up_sync(FULL, out_f, 1, T);
        uint32_t s_in = __shfl_up_sync(FULL, out_s, 1, T);
        uint32_t o_in = __shfl_up_sync(FULL, o_out, 1, T);
        uint32_t p_in = __shfl_up_sync(FULL, p_out, 1, T);

        if (t == 0) {
            // ---- feeder: emit one column of the current segment ----
            d_in = 0u;
            h_in = Z;
            f_in = Z;
            s_in = Z;
            if (f_done) {
                d_in = kDone;
            } else {
                bool emit = true;
                if (!f_open) {
                    // open a new segment; a later pass of the same pair waits
                    // until thread T-1 has written the boundary row ahead of it
                    if (f_pass > 0 && step - f_start < 2 * T + 2) {
                        emit = false;
                    } else {
                        f_open = true;
                        f_col = 0;
                        f_start = step;
                        dcur = __ldg(a.db + f_off);
                        if (f_ncols > 8) dnext = __ldg(a.db + f_off + 1);
                        if (f_pass > 0) {
                            const uint2* pb = a.bnd + (size_t)f_off * 16 + ((f_pass - 1) & 1);
                            bq0 = pb[0];
                            if (f_ncols > 1) bq1 = pb[2];
                        }
                        if (f_pass == 0) f_next = atomicAdd(a.counter, 1);
                    }
                }
                if (emit) {
                    if (f_col > 0 && (f_col & 7) == 0) {
                        dcur = dnext;
                        if (f_col + 8 < f_ncols) dnext = __ldg(a.db + f_off + (f_col >> 3) + 1);
                    }
                    uint32_t w = (dcur.x & 0xffffu) | kValid | ((uint32_t)f_pass << kPassShift);
                    dcur.x = __funnelshift_r(dcur.x, dcur.y, 16);
                    dcur.y = __funnelshift_r(dcur.y, dcur.z, 16);
                    dcur.z = __funnelshift_r(dcur.z, dcur.w, 16);
                    dcur.w >>= 16;
                    if (f_col == 0) w |= kFirst;
                    if (f_pass == 0) w |= kFirstPass;
                    if (f_pass + 1 == P) w |= kLastPass;
                    if (f_pass > 0) {
                        h_in = bq0.x;
                        f_in = bq0.y;
                        bq0 = bq1;
                        if (f_col + 2 < f_ncols)
                            bq1 = a.bnd[(size_t)f_off * 16 + 2 * (f_col + 2) + ((f_pass - 1) & 1)];
                    }
                    o_in = f_off;
                    p_in = (uint32_t)f_pair;
                    // the next pair's table entry, once its claim has returned
                    if (f_pass == 0 && f_col == (f_ncols < 9 ? f_ncols - 1 : 8) &&
                        f_next < pair_count)
                        f_ninfo = a.pairs[a.pair_begin + f_next];
                    ++f_col;
                    if (f_col == f_ncols) {
                        w |= kLast;
                        f_open = false;
                        if (f_pass + 1 < P) {
                            ++f_pass;
                        } else if (f_next >= pair_count) {
                            f_done = true;
                        } else {
                            f_pair = f_next;
                            f_off = f_ninfo.off16;
                            f_ncols = (int)f_ninfo.ncols;
                            f_pass = 0;
                        }
                    }
                    d_in = w;
                }
            }
        }

        const uint32_t d_top = d_in;
        const bool top_valid = (d_top & kValid) != 0, bot_valid = (d_bot & kValid) != 0;
        const bool top_first = (d_top & kFirst) != 0, bot_first = (d_bot & kFirst) != 0;
        // resets at a segment's first column (warp-uniform branch, rare)
        if (__any_sync(FULL, top_first || bot_first)) {
#pragma unroll
            for (int k = 0; k < HALF; ++k) {
                H[k] = top_first ? Z : H[k];
                E[k] = top_first ? Z : E[k];
            }
#pragma unroll
            for (int k = HALF; k < R; ++k) {
                H[k] = bot_first ? Z : H[k];
                E[k] = bot_first ? Z : E[k];
            }
            if (top_first) prev_h = Z;
            if (bot_first) {
                mid_h = Z;
                col_bot = 0;
            }
            if (top_first && (d_top & kFirstPass)) S_top = Z;
            if (bot_first && (d_bot & kFirstPass)) S_bot = Z;
        }
        const uint32_t bot_diag = mid_h, bot_f_in = mid_f, topfin = S_topfin;
        uint32_t f_top = f_in, f_bot = bot_f_in;
        if (top_valid | bot_valid) {
            // a half without a real column runs on zero-score residues: like a
            // trailing padding column it cannot raise any score, and its rows
            // are reset before they are used again
            const uint32_t wt = top_valid ? d_top : kPadPair;
            const uint32_t wb = bot_valid ? d_bot : kPadPair;
            const int pt = (int)(wt >> kPassShift), pb = (int)(wb >> kPassShift);
            const uint2* t0 = prof + ((pt * NJ) * kCodes + (int)(wt & 0xffu)) * SLOTS + slot;
            const uint2* t1 = prof + ((pt * NJ) * kCodes + (int)((wt >> 8) & 0xffu)) * SLOTS + slot;
            const uint2* b0 = prof + ((pb * NJ) * kCodes + (int)(wb & 0xffu)) * SLOTS + slot;
            const uint2* b1 = prof + ((pb * NJ) * kCodes + (int)((wb >> 8) & 0xffu)) * SLOTS + slot;
            // the top's last row before this column: the bottom's diagonal next step
            mid_h = H[HALF - 1];
            reverse_sweep<R, 0, HALF>(H, E, t0, t1, JSTRIDE, prev_h);
            reverse_sweep<R, HALF, R>(H, E, b0, b1, JSTRIDE, bot_diag);
#pragma unroll
            for (int i = 0; i < HALF; ++i) {
                forward_cell(H[i], E[i], f_top, K);
                forward_cell(H[HALF + i], E[HALF + i], f_bot, K);
                if (i & 1) {
                    S_top = __vimax3_s16x2(S_top, H[i - 1], H[i]);
                    S_bot = __vimax3_s16x2(S_bot, H[HALF + i - 1], H[HALF + i]);
                } else if (i == HALF - 1) {
                    S_top = __vimax3_s16x2(S_top, H[i], Z);
                    S_bot = __vimax3_s16x2(S_bot, H[HALF + i], Z);
                }
            }
        }
        mid_f = f_top;
        if (top_valid && (d_top & kLast) && (d_top & kLastPass))
            S_topfin = __vimax3_s16x2(S_top, s_in, Z);
        if (bot_valid) {
            out_h = H[R - 1];
            out_f = f_bot;
            const int pb = (int)(d_bot >> kPassShift);
            if (t == T - 1 && !(d_bot & kLastPass))
                a.bnd[(size_t)o_bot * 16 + 2 * col_bot + (pb & 1)] = make_uint2(out_h, out_f);
            if ((d_bot & kLast) && (d_bot & kLastPass)) {
                out_s = __vimax3_s16x2(S_bot, topfin, Z);
                if (t == T - 1) {
                    const int pos = 2 * (a.pair_begin + (int)p_bot);
                    const int s0 = lo16(out_s), s1 = hi16(out_s);
                    a.scores[pos] = s0 - bias;
                    if (s0 >= a.ovf_thresh) a.ovf_list[atomicAdd(a.ovf_count, 1)] = pos;
                    if (pos + 1 < a.n_records) {
                        a.scores[pos + 1] = s1 - bias;
                        if (s1 >= a.ovf_thresh) a.ovf_list[atomicAdd(a.ovf_count, 1)] = pos + 1;
                    }
                }
            }
            ++col_bot;
        }
        if (d_bot & kDone) finished = true;
        prev_h = h_in;
        d_out = d_bot;
        o_out = o_bot;
        p_out = p_bot;
        d_bot = d_top;
        o_bot = o_in;
        p_bot = p_in;
        __syncwarp();   // orders thread T-1's boundary stores before later feeder loads
    }
}

}  // namespace swb
