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
// pair.  Thread t holds R consecutive query rows in registers and walks the
// DB columns one step behind thread t-1 (anti-diagonal wavefront): at step s
// it updates column s - t, receiving the H/F of the row above (the last row
// of thread t-1, one step old) and the residue pair through warp shuffles.
// A query longer than T*R rows is done in passes; between passes the last
// row's H/F per column goes through a double-buffered boundary row in global
// memory.  T = 1 is the inter-sequence form (one pair per thread, boundary
// row every R query rows); T > 1 is the warp-cooperative intra-sequence form.
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

template <int I>
__device__ __forceinline__ uint32_t pick_pack(const uint2& A, const uint2& B) {
    return pack_s8x2<I & 3>(I < 4 ? A.x : A.y, I < 4 ? B.x : B.y);
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

// One 8-row chunk of the cell recurrence (rows j*8 .. j*8+7 of this thread):
//   t  = max(diag + P, E)            (DPX add+max)
//   h  = max(t, F, B)                (DPX 3-way max; B = biased zero)
//   hq = h - (open+extend)           (IMAD, both halves at once)
//   E  = max(E - extend, hq), F = max(F - extend, hq)   (DPX add+max)
//   S  = max(S, h, h_next)           (DPX 3-way max, every second row)
template <int R, int J>
__device__ __forceinline__ void rows8(uint32_t (&H)[R], uint32_t (&E)[R], const uint2 A,
                                      const uint2 B, uint32_t& diag, uint32_t& f,
                                      uint32_t& S, const CellK& K) {
#define SWB_CELL(I)                                                          \
    {                                                                        \
        constexpr int k = J * 8 + I;                                         \
        const uint32_t sc = pick_pack<I>(A, B);                              \
        uint32_t h = __viaddmax_s16x2(diag, sc, E[k]);                       \
        h = __vimax3_s16x2(h, f, K.bias2);                                   \
        diag = H[k];                                                         \
        H[k] = h;                                                            \
        const uint32_t hq = mad_u32(h, K.one, K.neg_q2);                     \
        E[k] = __viaddmax_s16x2(E[k], K.neg_e2, hq);                         \
        f = __viaddmax_s16x2(f, K.neg_e2, hq);                               \
    }
    SWB_CELL(0)
    SWB_CELL(1)
    S = __vimax3_s16x2(S, H[J * 8 + 0], H[J * 8 + 1]);
    SWB_CELL(2)
    SWB_CELL(3)
    S = __vimax3_s16x2(S, H[J * 8 + 2], H[J * 8 + 3]);
    SWB_CELL(4)
    SWB_CELL(5)
    S = __vimax3_s16x2(S, H[J * 8 + 4], H[J * 8 + 5]);
    SWB_CELL(6)
    SWB_CELL(7)
    S = __vimax3_s16x2(S, H[J * 8 + 6], H[J * 8 + 7]);
#undef SWB_CELL
}

// Chunks J..NJ-1 of one column step; the profile words of chunk J+1 are
// loaded before chunk J is computed so the shared-memory latency overlaps.
template <int R, int J, int NJ>
struct RowChunks {
    static __device__ __forceinline__ void run(uint32_t (&H)[R], uint32_t (&E)[R],
                                               const uint2* p0, const uint2* p1, int jstride,
                                               uint2 A, uint2 B, uint32_t& diag, uint32_t& f,
                                               uint32_t& S, const CellK& K) {
        uint2 An = A, Bn = B;
        if constexpr (J + 1 < NJ) {
            An = p0[(J + 1) * jstride];
            Bn = p1[(J + 1) * jstride];
        }
        rows8<R, J>(H, E, A, B, diag, f, S, K);
        if constexpr (J + 1 < NJ)
            RowChunks<R, J + 1, NJ>::run(H, E, p0, p1, jstride, An, Bn, diag, f, S, K);
    }
};

template <int T, int R, int BLOCK>
__global__ void __launch_bounds__(BLOCK, 1) sw_wavefront(const WfArgs a) {
    static_assert(R % 8 == 0 && R >= 8, "R");
    constexpr int NJ = R / 8;
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
    const unsigned gmask = (T == 32) ? FULL : (((1u << T) - 1u) << (lane & ~(T - 1)));
    CellK K;
    K.bias2 = a.bias2;
    K.neg_q2 = 0u - a.bias2;
    K.neg_e2 = a.neg_e;
    K.one = a.one;
    const uint32_t Z = a.bias2;        // biased zero of both lanes
    const int bias = (int)(a.bias2 & 0xffffu);

    uint32_t H[R], E[R];
    uint32_t S = Z;
    int pair = 0, pass = 0, s = 0, nsteps = 0, ncols = 0, ncols_pad = 0;
    bool done = false;
    uint32_t off16 = 0;
    uint32_t out_h = Z, out_f = Z, prev_h = Z, myd = kPadPair;
    // thread 0 of a group: residue chunks (current, next) and the boundary row
    // entries of the next two columns, loaded ahead so no step waits on memory
    uint4 dcur = make_uint4(0u, 0u, 0u, 0u), dnext = dcur;
    uint2 bq0 = make_uint2(Z, Z), bq1 = bq0;
    uint2* pbnd = a.bnd;

#define SWB_START_PASS()                                                  \
    {                                                                     \
        s = 0;                                                            \
        nsteps = ncols + T - 1;                                           \
        _Pragma("unroll") for (int k = 0; k < R; ++k) {                   \
            H[k] = Z;                                                     \
            E[k] = Z;                                                     \
        }                                                                 \
        out_h = Z;                                                        \
        out_f = Z;                                                        \
        prev_h = Z;                                                       \
        myd = kPadPair;                                                   \
        if (t == 0) {                                                     \
            dcur = __ldg(a.db + off16);                                   \
            if (ncols > 8) dnext = __ldg(a.db + off16 + 1);               \
            if (pass > 0) {                                               \
                const uint2* pb = pbnd + ((pass - 1) & 1) * ncols_pad;    \
                bq0 = pb[0];                                              \
                if (ncols > 1) bq1 = pb[1];                               \
            }                                                             \
        }                                                                 \
    }
#define SWB_CLAIM()                                                      \
    {                                                                    \
        int v = 0;                                                       \
        if (t == 0) v = atomicAdd(a.counter, 1);                         \
        v = __shfl_sync(gmask, v, 0, T);                                 \
        if (v >= a.pair_count) {                                         \
            done = true;                                                 \
            ncols = 0;                                                   \
            nsteps = 0;                                                  \
        } else {                                                         \
            pair = v;                                                    \
            const Pair2 pr = a.pairs[a.pair_begin + v];                  \
            off16 = pr.off16;                                            \
            ncols = (int)pr.ncols;                                       \
            ncols_pad = (ncols + 7) & ~7;                                \
            pbnd = a.bnd + (size_t)off16 * 16;                           \
            pass = 0;                                                    \
            S = Z;                                                       \
            SWB_START_PASS()                                             \
        }                                                                \
    }

    SWB_CLAIM()

    while (!__all_sync(FULL, done)) {
        // ---- one wavefront step: receive from the thread above ----
        uint32_t d_in = __shfl_up_sync(FULL, myd, 1, T);
        uint32_t h_in = __shfl_up_sync(FULL, out_h, 1, T);
        uint32_t f_in = __shfl_up_sync(FULL, out_f, 1, T);
        if (t == 0) {
            d_in = kPadPair;
            h_in = Z;
            f_in = Z;
            if (s < ncols) {
                if ((s & 7) == 0 && s > 0) {
                    dcur = dnext;
                    if (s + 8 < ncols) dnext = __ldg(a.db + off16 + (s >> 3) + 1);
                }
                d_in = dcur.x & 0xffffu;
                dcur.x = __funnelshift_r(dcur.x, dcur.y, 16);
                dcur.y = __funnelshift_r(dcur.y, dcur.z, 16);
                dcur.z = __funnelshift_r(dcur.z, dcur.w, 16);
                dcur.w >>= 16;
                if (pass > 0) {
                    h_in = bq0.x;
                    f_in = bq0.y;
                    bq0 = bq1;
                    if (s + 2 < ncols) bq1 = pbnd[((pass - 1) & 1) * ncols_pad + s + 2];
                }
            }
        }
        const int c = s - t;
        if (!done && c >= 0 && c < ncols) {
            const int d0 = (int)(d_in & 0xffu), d1 = (int)((d_in >> 8) & 0xffu);
            const uint2* p0 = prof + ((pass * NJ) * kCodes + d0) * SLOTS + slot;
            const uint2* p1 = prof + ((pass * NJ) * kCodes + d1) * SLOTS + slot;
            uint32_t diag = prev_h, f = f_in;
            RowChunks<R, 0, NJ>::run(H, E, p0, p1, JSTRIDE, p0[0], p1[0], diag, f, S, K);
            out_h = H[R - 1];
            out_f = f;
            if (t == T - 1 && pass + 1 < P) pbnd[(pass & 1) * ncols_pad + c] = make_uint2(out_h, out_f);
        }
        prev_h = h_in;
        myd = d_in;
        ++s;
        if (!done && s == nsteps) {  // uniform within the group
            __syncwarp(gmask);
            if (pass + 1 < P) {
                ++pass;
                SWB_START_PASS()
            } else {
#pragma unroll
                for (int o = T / 2; o > 0; o >>= 1)
                    S = __vimax3_s16x2(S, __shfl_xor_sync(gmask, S, o, T), Z);
                if (t == 0) {
                    const int pos = 2 * (a.pair_begin + pair);
                    const int s0 = lo16(S), s1 = hi16(S);
                    a.scores[pos] = s0 - bias;
                    if (s0 >= a.ovf_thresh) a.ovf_list[atomicAdd(a.ovf_count, 1)] = pos;
                    if (pos + 1 < a.n_records) {
                        a.scores[pos + 1] = s1 - bias;
                        if (s1 >= a.ovf_thresh) a.ovf_list[atomicAdd(a.ovf_count, 1)] = pos + 1;
                    }
                }
                SWB_CLAIM()
            }
        }
    }
#undef SWB_CLAIM
#undef SWB_START_PASS
}

}  // namespace swb
