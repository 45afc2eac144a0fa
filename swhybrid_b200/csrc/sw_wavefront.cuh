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
// E, F stay >= -(open+extend) because h >= 0, so no lane underflows; a lane
// can only wrap upward after exceeding 32767 - max(matrix), which is the
// overflow threshold handed to the 32-bit re-score pass.
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

// One 8-row chunk of the cell recurrence (rows j*8 .. j*8+7 of this thread).
template <int R, int J>
__device__ __forceinline__ void rows8(uint32_t (&H)[R], uint32_t (&E)[R], const uint2 A,
                                      const uint2 B, uint32_t& diag, uint32_t& f,
                                      uint32_t& S, const uint32_t NEG_OE,
                                      const uint32_t NEG_E) {
    const uint32_t MIN16 = 0x80008000u;
#define SWB_CELL(I)                                                          \
    {                                                                        \
        constexpr int k = J * 8 + I;                                         \
        const uint32_t sc = pick_pack<I>(A, B);                              \
        uint32_t h = __viaddmax_s16x2_relu(diag, sc, E[k]);                  \
        h = __vimax_s16x2_relu(h, f);                                        \
        diag = H[k];                                                         \
        H[k] = h;                                                            \
        const uint32_t hq = __viaddmax_s16x2(h, NEG_OE, MIN16);              \
        E[k] = __viaddmax_s16x2(E[k], NEG_E, hq);                            \
        f = __viaddmax_s16x2(f, NEG_E, hq);                                  \
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
                                               uint32_t& S, uint32_t NEG_OE, uint32_t NEG_E) {
        uint2 An = A, Bn = B;
        if constexpr (J + 1 < NJ) {
            An = p0[(J + 1) * jstride];
            Bn = p1[(J + 1) * jstride];
        }
        rows8<R, J>(H, E, A, B, diag, f, S, NEG_OE, NEG_E);
        if constexpr (J + 1 < NJ)
            RowChunks<R, J + 1, NJ>::run(H, E, p0, p1, jstride, An, Bn, diag, f, S, NEG_OE, NEG_E);
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
    const uint32_t NEG_OE = a.neg_oe, NEG_E = a.neg_e;

    uint32_t H[R], E[R];
    uint32_t S = 0;
    int pair = 0, pass = 0, s = 0, nsteps = 0, ncols = 0, ncols_pad = 0;
    bool done = false;
    uint32_t off16 = 0;
    uint32_t out_h = 0, out_f = 0, prev_h = 0, myd = kPadPair;
    uint4 dbuf = make_uint4(0u, 0u, 0u, 0u);
    uint2* pbnd = a.bnd;

#define SWB_START_PASS()                                \
    {                                                   \
        s = 0;                                          \
        nsteps = ncols + T - 1;                         \
        _Pragma("unroll") for (int k = 0; k < R; ++k) { \
            H[k] = 0u;                                  \
            E[k] = 0u;                                  \
        }                                               \
        out_h = 0u;                                     \
        out_f = 0u;                                     \
        prev_h = 0u;                                    \
        myd = kPadPair;                                 \
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
            S = 0u;                                                      \
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
            h_in = 0u;
            f_in = 0u;
            if (s < ncols) {
                if ((s & 7) == 0) dbuf = __ldg(a.db + off16 + (s >> 3));
                d_in = dbuf.x & 0xffffu;
                dbuf.x = __funnelshift_r(dbuf.x, dbuf.y, 16);
                dbuf.y = __funnelshift_r(dbuf.y, dbuf.z, 16);
                dbuf.z = __funnelshift_r(dbuf.z, dbuf.w, 16);
                dbuf.w >>= 16;
                if (pass > 0) {
                    const uint2 b = pbnd[((pass - 1) & 1) * ncols_pad + s];
                    h_in = b.x;
                    f_in = b.y;
                }
            }
        }
        const int c = s - t;
        if (!done && c >= 0 && c < ncols) {
            const int d0 = (int)(d_in & 0xffu), d1 = (int)((d_in >> 8) & 0xffu);
            const uint2* p0 = prof + ((pass * NJ) * kCodes + d0) * SLOTS + slot;
            const uint2* p1 = prof + ((pass * NJ) * kCodes + d1) * SLOTS + slot;
            uint32_t diag = prev_h, f = f_in;
            RowChunks<R, 0, NJ>::run(H, E, p0, p1, JSTRIDE, p0[0], p1[0], diag, f, S, NEG_OE,
                                     NEG_E);
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
                    S = __vimax_s16x2_relu(S, __shfl_xor_sync(gmask, S, o, T));
                if (t == 0) {
                    const int pos = 2 * (a.pair_begin + pair);
                    const int s0 = lo16(S), s1 = hi16(S);
                    a.scores[pos] = s0;
                    if (s0 >= a.ovf_thresh) a.ovf_list[atomicAdd(a.ovf_count, 1)] = pos;
                    if (pos + 1 < a.n_records) {
                        a.scores[pos + 1] = s1;
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
