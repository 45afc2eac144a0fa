// sw_long.cu -- first pass for long record pairs: the query passes of one
// pair run concurrently in the warps of one block.
//
// The reference splits its GPU work into an "inter-sequence" kernel (one
// record per thread, src/CUDAKernel.cu:63-192) and sends records of 6,144
// residues or more to its CPU re-calculation instead
// (src/CUDAWorker.cu:144-201).  On B200 a long pair in the bulk kernel is a
// long serial chain of column steps in one group, so a DB whose residues sit
// in few long records leaves most of the GPU idle at the end.  Here a pair
// longer than the cut-over is scored by a pipeline of P warps, one warp per
// query pass of 32 x R rows: warp w runs the same anti-diagonal wavefront as
// the bulk kernel (sw_wavefront.cuh) on pass w, D = K + 64 column steps behind
// warp w-1, and takes the H/F of its first row's upper neighbour from a
// shared-memory ring that warp w-1's last thread fills.  The warps stay in
// step through one block barrier every K column steps (no flag waits):
//   * warp w-1's last thread writes column c at pipeline step (w-1)D + c + 63
//     and warp w's first thread reads it at pipeline step wD + c, K + 1 steps
//     later, so a barrier always separates the write from the read;
//   * the ring holds RING >= 2K + 1 columns, so the entry is overwritten
//     (column c + RING) at least K steps after it was read, again across a
//     barrier.
// The per-pair cost of the pipeline is (P-1)D + 63 steps of fill and drain
// against ncols >= cut-over steps of work.  A block holds G such pipelines
// (G x P warps) that share the query profile and claim pairs independently;
// a pipeline's pair starts and ends at a barrier.  Each block takes a whole
// SM (it requests the SM's shared memory), so the long pairs run on the SMs
// the concurrent bulk launch leaves free.
#include <cstdint>

#include <cuda_runtime.h>

#include "sw_device.cuh"
#include "sw_long.h"
#include "sw_wavefront.cuh"

namespace swb {

namespace {

constexpr int kLT = 32;                  // threads per pass (one warp)
constexpr int kLK = 64;                  // column steps between block barriers
constexpr int kLD = kLK + 64;            // step lag of warp w behind warp w-1
constexpr int kLRing = 256;              // ring columns per link (>= 2K + 1, power of 2)

// Threads per block the compiler plans registers for: as many warps as the
// register file holds at the row count's register need, without spills.
template <int R>
struct LongBlock {
    static constexpr int value = R <= 8 ? 768 : R <= 16 ? 512 : R <= 32 ? 384 : 256;
};

// One column step of a warp's two half-columns (top on column c with profile
// words t0/t1, bottom on column c - 1 with b0/b1); f_bot receives the bottom
// half's last-row F.  Both halves' maxima go into S.
template <int R>
__device__ __forceinline__ void long_step(uint32_t (&H)[R], uint32_t (&E)[R], const uint2* t0,
                                          const uint2* t1, const uint2* b0, const uint2* b1,
                                          uint32_t prev_h, uint32_t f_in, uint32_t& mid_h,
                                          uint32_t& mid_f, uint32_t& f_bot_out, uint32_t& S,
                                          const CellK& K) {
    constexpr int HALF = R / 2;
    constexpr int JSTRIDE = kCodes * GroupShape<kLT>::SLOTS;
    const uint32_t bot_diag = mid_h;
    uint32_t f_top = f_in, f_bot = mid_f;
    mid_h = H[HALF - 1];
    reverse_sweep<R, 0, HALF>(H, E, t0, t1, JSTRIDE, prev_h);
    reverse_sweep<R, HALF, R>(H, E, b0, b1, JSTRIDE, bot_diag);
#pragma unroll
    for (int i = 0; i < HALF; ++i) {
        forward_cell(H[i], E[i], f_top, K);
        forward_cell(H[HALF + i], E[HALF + i], f_bot, K);
        if (i & 1) S = __vimax3_s16x2(S, H[i - 1], H[i]);
        if (i & 1) S = __vimax3_s16x2(S, H[HALF + i - 1], H[HALF + i]);
        if (!(i & 1) && i == HALF - 1) S = __vimax3_s16x2(S, H[i], H[HALF + i]);
    }
    mid_f = f_top;
    f_bot_out = f_bot;
}

template <int R>
__global__ void __launch_bounds__(LongBlock<R>::value, 1) sw_long(const LongArgs a) {
    constexpr int T = kLT;
    constexpr int NJ = (R + 7) / 8;
    constexpr int HALF = R / 2;
    constexpr int SLOTS = GroupShape<T>::SLOTS;
    constexpr int JSTRIDE = kCodes * SLOTS;
    constexpr unsigned FULL = 0xffffffffu;
    extern __shared__ uint2 smem[];
    __shared__ int s_next[kLongMaxWarps];                 // per pipeline: its next pair
    __shared__ uint32_t s_max[kLongMaxWarps];             // per warp: its pass's max
    const int P = a.passes;                               // warps per pipeline
    uint2* const prof = smem;
    uint2* const ring = smem + (size_t)P * NJ * JSTRIDE;  // G pipelines x (P-1) links
    build_profile<T, R>(prof, a.query, a.qlen, a.mat, P);
    const int warp = (int)(threadIdx.x >> 5);
    const int g = warp / P;                               // this warp's pipeline
    const int w = warp - g * P;                           // ... and its pass in it
    const int t = (int)(threadIdx.x & 31);
    const bool leader = (w == 0 && t == 0);
    CellK K;
    K.bias2 = a.bias2;
    K.neg_q2 = 0u - a.bias2;
    K.neg_e2 = a.neg_e;
    const uint32_t Z = a.bias2;
    const int bias = (int)(a.bias2 & 0xffffu);
    const uint2* const prof_p = prof + (w * NJ) * JSTRIDE + t;
    uint2* const links = ring + (size_t)g * (P > 1 ? P - 1 : 0) * kLRing;
    uint2* const ring_out = links + (size_t)(w + 1 < P ? w : 0) * kLRing;       // link w -> w+1
    const uint2* const ring_in = links + (size_t)(w > 0 ? w - 1 : 0) * kLRing;  // link w-1 -> w
    uint32_t H[R], E[R];
    uint32_t S = Z, out_h = Z, out_f = Z, prev_h = Z, mid_h = Z, mid_f = Z;
    uint32_t d_bot = kPadPair, d_cur = kPadPair;
    const unsigned short* col = reinterpret_cast<const unsigned short*>(a.db);
    int pair = 0, ncols = 0, span = 0, total = 0, start = 0;
    uint32_t off16 = 0u;
    bool active = false;
    // a pipeline's pair starts at a barrier (block step `start`, a multiple of
    // K) and lasts `total` steps, also a multiple of K
#define SWL_BEGIN_PAIR(v, at)                                              \
    {                                                                      \
        pair = (v);                                                        \
        active = pair < a.pair_count;                                      \
        if (active) {                                                      \
            const Pair2 pr = a.pairs[a.pair_begin + pair];                 \
            ncols = (int)pr.ncols;                                         \
            off16 = pr.off16;                                              \
            span = ncols + 2 * T - 1;                                      \
            total = ((P - 1) * kLD + span + kLK - 1) / kLK * kLK;          \
            start = (at);                                                  \
            _Pragma("unroll") for (int k = 0; k < R; ++k) {                \
                H[k] = Z;                                                  \
                E[k] = Z;                                                  \
            }                                                              \
            S = Z;                                                         \
            out_h = Z;                                                     \
            out_f = Z;                                                     \
            prev_h = Z;                                                    \
            mid_h = Z;                                                     \
            mid_f = Z;                                                     \
            d_bot = kPadPair;                                              \
            col = reinterpret_cast<const unsigned short*>(a.db) + (size_t)off16 * 8; \
            d_cur = (t == 0 && ncols > 0) ? (uint32_t)__ldg(col) : kPadPair; \
        }                                                                  \
    }
    if (leader) s_next[g] = atomicAdd(a.counter, 1);
    __syncthreads();                                       // profile built, first claims made
    SWL_BEGIN_PAIR(s_next[g], 0)
    int gs = 0;                                            // block step
    while (true) {
        for (int j = 0; j < kLK;) {
            const int s = gs - start - w * kLD;            // this warp's step (warp-uniform)
            if (!active || s < 0 || s >= span) {
                ++j;
                ++gs;
                continue;
            }
            // Plain steps: every lane's two half-columns and its next residue
            // lie inside the pair (column s - 2t - 1 >= 0 for t = 31, column
            // s + 1 < ncols for t = 0), so the warp runs them with no bounds
            // guards, up to the next barrier.
            if (s >= 2 * T - 1 && s <= ncols - 2) {
                int n = ncols - 1 - s;
                if (n > kLK - j) n = kLK - j;
                const int ct0 = s - 2 * t;
                const bool ring_rd = t == 0 && w > 0;
                const bool ring_wr = t == T - 1 && w + 1 < P;
#pragma unroll 2
                for (int i = 0; i < n; ++i) {
                    uint32_t h_in = __shfl_up_sync(FULL, out_h, 1);
                    uint32_t f_in = __shfl_up_sync(FULL, out_f, 1);
                    const uint32_t d_in = d_cur;
                    const int ct = ct0 + i;
                    d_cur = (uint32_t)__ldg(col + ct + 1);
                    if (t == 0) {
                        h_in = Z;
                        f_in = Z;
                    }
                    if (ring_rd) {
                        const uint2 b = ring_in[(s + i) & (kLRing - 1)];
                        h_in = b.x;
                        f_in = b.y;
                    }
                    long_step<R>(H, E, prof_p + (int)(d_in & 0xffu) * SLOTS,
                                 prof_p + (int)((d_in >> 8) & 0xffu) * SLOTS,
                                 prof_p + (int)(d_bot & 0xffu) * SLOTS,
                                 prof_p + (int)((d_bot >> 8) & 0xffu) * SLOTS, prev_h, f_in,
                                 mid_h, mid_f, out_f, S, K);
                    out_h = H[R - 1];
                    if (ring_wr) ring_out[(ct - 1) & (kLRing - 1)] = make_uint2(out_h, out_f);
                    prev_h = h_in;
                    d_bot = d_in;
                }
                j += n;
                gs += n;
                continue;
            }
            // a general step: lanes at the pair's first or last columns
            uint32_t h_in = __shfl_up_sync(FULL, out_h, 1);
            uint32_t f_in = __shfl_up_sync(FULL, out_f, 1);
            const uint32_t d_in = d_cur;       // this thread's top column, loaded a step ahead
            {
                const int c1 = s + 1 - 2 * t;
                d_cur = (c1 >= 0 && c1 < ncols) ? (uint32_t)__ldg(col + c1) : kPadPair;
            }
            if (t == 0) {
                h_in = Z;
                f_in = Z;
                if (s < ncols) {
                    if (w > 0) {
                        const uint2 b = ring_in[s & (kLRing - 1)];
                        h_in = b.x;
                        f_in = b.y;
                    }
                }
            }
            const int ct = s - 2 * t;
            const bool top_valid = ct >= 0 && ct < ncols;
            const bool bot_valid = ct >= 1 && ct <= ncols;
            if (ct >= 0 && ct <= ncols) {
                const uint32_t wt = top_valid ? d_in : kPadPair;
                const uint32_t wb = bot_valid ? d_bot : kPadPair;
                uint32_t f_bot = Z;
                long_step<R>(H, E, prof_p + (int)(wt & 0xffu) * SLOTS,
                             prof_p + (int)((wt >> 8) & 0xffu) * SLOTS,
                             prof_p + (int)(wb & 0xffu) * SLOTS,
                             prof_p + (int)((wb >> 8) & 0xffu) * SLOTS, prev_h, f_in, mid_h,
                             mid_f, f_bot, S, K);
                if (bot_valid) {
                    out_h = H[R - 1];
                    out_f = f_bot;
                    if (t == T - 1 && w + 1 < P)
                        ring_out[(ct - 1) & (kLRing - 1)] = make_uint2(out_h, out_f);
                }
            }
            prev_h = h_in;
            d_bot = d_in;
            ++j;
            ++gs;
        }
        // barrier: pipelines whose pair ends here publish their passes' maxima
        // and (leader) claim the next pair; the OR says whether any pipeline
        // still has work after this barrier
        const bool ending = active && gs - start >= total;
        bool alive = active && !ending;
        if (ending) {
#pragma unroll
            for (int o = 16; o > 0; o >>= 1)
                S = __vimax3_s16x2(S, __shfl_xor_sync(FULL, S, o), Z);
            if (t == 0) s_max[warp] = S;
            if (leader) {
                const int v = atomicAdd(a.counter, 1);
                s_next[g] = v;
                alive = v < a.pair_count;
            }
        }
        const int any = __syncthreads_or(alive ? 1 : 0);
        if (ending) {
            if (leader) {
                for (int i = 1; i < P; ++i) S = __vimax3_s16x2(S, s_max[warp + i], Z);
                const int pos = 2 * (a.pair_begin + pair);
                const int s0 = lo16(S), s1 = hi16(S);
                a.scores[pos] = s0 - bias;
                if (s0 >= a.ovf_thresh) {
                    const int j = atomicAdd(a.ovf_count, 1);
                    if (j < a.ovf_cap) a.ovf_list[j] = pos;
                }
                if (pos + 1 < a.n_records) {
                    a.scores[pos + 1] = s1 - bias;
                    if (s1 >= a.ovf_thresh) {
                        const int j = atomicAdd(a.ovf_count, 1);
                        if (j < a.ovf_cap) a.ovf_list[j] = pos + 1;
                    }
                }
            }
            SWL_BEGIN_PAIR(s_next[g], gs)
        }
        if (!any) break;
    }
#undef SWL_BEGIN_PAIR
}

template <int R>
size_t long_smem(int passes, int pipelines) {
    constexpr int NJ = (R + 7) / 8;
    return (size_t)passes * NJ * kCodes * GroupShape<kLT>::SLOTS * sizeof(uint2) +
           (size_t)pipelines * (passes > 1 ? passes - 1 : 0) * kLRing * sizeof(uint2);
}

template <int R>
constexpr LongKernel linst() {
    return LongKernel{R, (const void*)&sw_long<R>, &long_smem<R>, LongBlock<R>::value};
}

// (48 rows would leave only 8 warps of 231 registers per SM, which measured
// slower than either neighbour, so it is not built.)
const LongKernel kLongTable[] = {
    linst<8>(), linst<16>(), linst<24>(), linst<32>(), linst<64>(),
};

}  // namespace

const LongKernel* long_kernels(int* n) {
    *n = (int)(sizeof(kLongTable) / sizeof(kLongTable[0]));
    return kLongTable;
}

}  // namespace swb
