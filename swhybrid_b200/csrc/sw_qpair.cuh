// sw_qpair.cuh -- batched first pass with two queries per register.
//
// In the plain and stacked kernels (sw_wavefront.cuh) a 32-bit register
// holds one query row against two DB records, so every row of every column
// step must assemble its two profile scores (one per record residue) with a
// PRMT: 1 of the 5.5 ALU-pipe instructions per row.  When a batch has many
// queries, the two 16-bit lanes can instead hold two QUERIES against one
// record: both lanes then look up the same residue, and the profile can be
// stored already packed -- word (code, row) = score of query A's row against
// the code in the low half, query B's in the high half -- so the per-row
// work is 4.5 ALU instructions (no PRMT) for the same two cells.
//
// Here a "double stack" is two stacks of short queries (the low lane's and
// the high lane's, each packed first-fit into R-row blocks as in sw_batch)
// scored together.  A group of T threads claims a unit = one record (a half
// of a DB record pair; the pair's column stream is shared, the unit uses
// its byte) and runs the same two-half-column anti-diagonal wavefront as the
// other kernels.  Each lane has its own row-block map (query and
// "starts here"), so the input reset at query starts and the per-pass
// segmented maxima are done per lane.  The profile is 4 bytes per row and
// code (a pair of int16 scores), 4 rows per 16-byte word, so a double stack
// holds at most ~2,200 rows in shared memory.
#pragma once
#include "sw_device.cuh"
#include "sw_wavefront.cuh"

namespace swb {

// Arguments of the paired-query batched kernel.
struct QpArgs {
    const uint4* db;
    const Pair2* pairs;
    int pair_begin;             // pairs [pair_begin, pair_begin + pair_count)
    int pair_count;             // units = 2 * pair_count (both records of each pair)
    const uint8_t* codes;       // stack row codes back to back
    const uint32_t* off_lo;     // per double stack: low lane's codes offset, rows
    const uint32_t* rows_lo;
    const uint32_t* off_hi;     // ... and the high lane's
    const uint32_t* rows_hi;
    const int2* rb_map;         // per double stack, pass and thread: (low, high) query | first bit, or -1
    const uint32_t* rb_off;     // per double stack: offset into rb_map
    int nstacks;
    int* counters;              // one unit counter per double stack (zero before)
    const int8_t* mat;
    uint32_t bias2, neg_e;
    uint2* bnd;                 // per-group boundary rows
    size_t bnd_group;
    int* scores;                // [query][sorted position], zero before (atomicMax)
    int n_records;
    int* ovf_list;              // query * n_records + position
    int* ovf_count;
    int ovf_thresh;
    int ovf_cap;
    const uint32_t* pair_ids;   // optional: global pair of each entry of pairs
    // segments: a double stack taller than one launch's limit is cut into row
    // segments scored by consecutive launches; per stack, bit 0 = read the
    // rows above from seg_bnd at pass 0, bit 1 = write the last row to it
    const uint32_t* seg_flags;
    uint2* seg_bnd;             // per record and column: (H, F) of a segment's last row,
                                // at 16 entries per 16-byte stream unit (2 per column)
};

// Shared-memory bytes of a double stack's profile (rows = the taller lane).
template <int T, int R>
__host__ __device__ constexpr size_t qp_smem_bytes(int rows) {
    return (size_t)((rows + T * R - 1) / (T * R)) * (R / 4) * kCodes * GroupShape<T>::SLOTS *
           sizeof(uint4);
}

// Paired profile -> shared memory (whole block; the caller synchronises).
// Layout [pass][chunk of 4 rows][code][slot] of 16-byte words; component i of
// a word is row 4*chunk + i of the slot's thread: low half the low lane's
// score, high half the high lane's.
template <int T, int R>
__device__ __forceinline__ void build_profile_qp(uint4* prof, const uint8_t* lo, int rows_lo,
                                                 const uint8_t* hi, int rows_hi,
                                                 const int8_t* mat, int P) {
    constexpr int NJ = R / 4;
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
        const int row0 = p * rows_per_pass + (slot % T) * R + j * 4;
        uint32_t w[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int row = row0 + i;
            const int a = row < rows_lo ? mat[(lo[row] & 31) * 32 + d] : 0;
            const int b = row < rows_hi ? mat[(hi[row] & 31) * 32 + d] : 0;
            w[i] = (uint32_t)(uint16_t)(int16_t)a | ((uint32_t)(uint16_t)(int16_t)b << 16);
        }
        prof[idx] = make_uint4(w[0], w[1], w[2], w[3]);
    }
}

__device__ __forceinline__ uint32_t qp_word(const uint4& v, int i) {
    return i == 0 ? v.x : i == 1 ? v.y : i == 2 ? v.z : v.w;
}

// Reverse sweep of one half with pre-packed profile words: H[k] <- max(H[k-1]
// + P_k, E_k) for k = HI-1 down to LO, H[LO-1] replaced by diag.
template <int R, int LO, int HI>
__device__ __forceinline__ void reverse_sweep_qp(uint32_t (&H)[R], const uint32_t (&E)[R],
                                                 const uint4* p, int jstride, uint32_t diag) {
    constexpr int JLO = LO / 4, JHI = (HI - 1) / 4;
    uint4 A = p[JHI * jstride];
#pragma unroll
    for (int j = JHI; j >= JLO; --j) {
        uint4 An = A;
        if (j > JLO) An = p[(j - 1) * jstride];
#pragma unroll
        for (int i = 3; i >= 0; --i) {
            const int k = j * 4 + i;
            if (k >= LO && k < HI) {
                const uint32_t up = (k > LO) ? H[k > LO ? k - 1 : LO] : diag;
                H[k] = __viaddmax_s16x2(up, qp_word(A, i), E[k]);
            }
        }
        A = An;
    }
}

// One double stack: every group claims units (records) and scores them
// against both lanes' stacks.  Returns when the units are exhausted.
template <int T, int R>
__device__ __forceinline__ void run_qpairs(const QpArgs& a, const uint4* prof, int P, int* counter,
                                           const int2* rb_map, uint32_t seg) {
    static_assert(R % 8 == 0, "R");
    constexpr int NJ = R / 4;
    constexpr int HALF = R / 2;
    constexpr int SLOTS = GroupShape<T>::SLOTS;
    constexpr int JSTRIDE = kCodes * SLOTS;
    constexpr unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int t = lane & (T - 1);
    const int slot = lane & (SLOTS - 1);
    const unsigned gmask = (T == 32) ? FULL : (((1u << T) - 1u) << (lane & ~(T - 1)));
    CellK K;
    K.bias2 = a.bias2;
    K.neg_q2 = 0u - a.bias2;
    K.neg_e2 = a.neg_e;
    const uint32_t Z = a.bias2;
    const int bias = (int)(a.bias2 & 0xffffu);
    const int units = 2 * a.pair_count;
    uint2* const pbnd = a.bnd + (size_t)((blockIdx.x * blockDim.x + threadIdx.x) / T) * a.bnd_group;

    uint32_t H[R], E[R];
    uint32_t S = Z, out_h = Z, out_f = Z, prev_h = Z, mid_h = Z, mid_f = Z;
    uint32_t d_bot = kZeroCode, d_cur = kZeroCode;
    const unsigned short* col = reinterpret_cast<const unsigned short*>(a.db);
    int unit = 0, next = 0, pass = 0, s = 0, nsteps = 0, ncols = 0, half = 0;
    uint32_t off16 = 0u;
    bool done = false;
    uint2 bq0 = make_uint2(Z, Z), bq1 = bq0;
    Pair2 ninfo{0u, 0u};
    int q_lo = -1, q_hi = -1;
    uint32_t reset = 0u;     // lanes whose query starts at this thread's first row
    bool has_in = false;     // the pass takes its rows above from a boundary row
    const uint2* in_b = pbnd;

#define SWQ_START_PASS()                                                   \
    {                                                                      \
        s = 0;                                                             \
        const int2 rb = rb_map[pass * T + t];                              \
        q_lo = rb.x < 0 ? -1 : (rb.x & (kFirstBit - 1));                   \
        q_hi = rb.y < 0 ? -1 : (rb.y & (kFirstBit - 1));                   \
        reset = ((rb.x >= 0 && (rb.x & kFirstBit)) ? 0x0000ffffu : 0u) |   \
                ((rb.y >= 0 && (rb.y & kFirstBit)) ? 0xffff0000u : 0u);    \
        S = Z;                                                             \
        nsteps = ncols + 2 * T - 1;                                        \
        _Pragma("unroll") for (int k = 0; k < R; ++k) {                    \
            H[k] = Z;                                                      \
            E[k] = Z;                                                      \
        }                                                                  \
        out_h = Z;                                                         \
        out_f = Z;                                                         \
        prev_h = Z;                                                        \
        mid_h = Z;                                                         \
        mid_f = Z;                                                         \
        d_bot = kZeroCode;                                                 \
        col = reinterpret_cast<const unsigned short*>(a.db) + (size_t)off16 * 8; \
        d_cur = (t == 0 && ncols > 0) ? (((uint32_t)__ldg(col) >> (8 * half)) & 0xffu) \
                                      : (uint32_t)kZeroCode;               \
        has_in = pass > 0 || (seg & 1u);                                   \
        in_b = pass > 0 ? pbnd + ((pass - 1) & 1)                          \
                        : a.seg_bnd + (size_t)off16 * 16 + half;           \
        if (t == 0) {                                                      \
            if (has_in) {                                                  \
                bq0 = in_b[0];                                             \
                if (ncols > 1) bq1 = in_b[2];                              \
            }                                                              \
        }                                                                  \
    }
#define SWQ_TAKE_UNIT(v)                                                   \
    {                                                                      \
        if ((v) >= units) {                                                \
            done = true;                                                   \
            ncols = 0;                                                     \
            nsteps = 0;                                                    \
        } else {                                                           \
            unit = (v);                                                    \
            half = unit & 1;                                               \
            pass = 0;                                                      \
            if (t == 0) next = atomicAdd(counter, 1);                      \
            SWQ_START_PASS()                                               \
        }                                                                  \
    }

    {
        int v = 0;
        if (t == 0) v = atomicAdd(counter, 1);
        v = __shfl_sync(gmask, v, 0, T);
        if (v < units) {
            const Pair2 pr = a.pairs[a.pair_begin + (v >> 1)];
            off16 = pr.off16;
            ncols = (int)pr.ncols;
        }
        SWQ_TAKE_UNIT(v)
    }

    while (!__all_sync(FULL, done)) {
        uint32_t h_in = __shfl_up_sync(FULL, out_h, 1, T);
        uint32_t f_in = __shfl_up_sync(FULL, out_f, 1, T);
        const uint32_t d_in = d_cur;           // this thread's top column, loaded a step ahead
        {
            const int c1 = s + 1 - 2 * t;
            d_cur = (c1 >= 0 && c1 < ncols) ? (((uint32_t)__ldg(col + c1) >> (8 * half)) & 0xffu)
                                             : (uint32_t)kZeroCode;
        }
        if (t == 0) {
            h_in = Z;
            f_in = Z;
            if (s < ncols) {
                if (has_in) {
                    h_in = bq0.x;
                    f_in = bq0.y;
                    bq0 = bq1;
                    if (s + 2 < ncols) bq1 = in_b[2 * (s + 2)];
                }
                // the next unit's pair entry, once its claim has returned
                if (pass == 0 && s == (ncols < 9 ? ncols - 1 : 8) && next < units)
                    ninfo = a.pairs[a.pair_begin + (next >> 1)];
            }
        }
        // a lane whose query starts here takes nothing from above
        h_in = (h_in & ~reset) | (Z & reset);
        f_in = (f_in & ~reset) | (Z & reset);
        const int ct = s - 2 * t;
        const bool top_valid = ct >= 0 && ct < ncols;
        const bool bot_valid = ct >= 1 && ct <= ncols;
        if (!done && (ct >= 0 && ct <= ncols)) {
            const uint32_t wt = top_valid ? d_in : kZeroCode;
            const uint32_t wb = bot_valid ? d_bot : kZeroCode;
            const uint4* prof_p = prof + (pass * NJ) * JSTRIDE + slot;
            const uint4* pt = prof_p + (int)wt * SLOTS;
            const uint4* pb = prof_p + (int)wb * SLOTS;
            const uint32_t bot_diag = mid_h;
            uint32_t f_top = f_in, f_bot = mid_f;
            mid_h = H[HALF - 1];
            reverse_sweep_qp<R, 0, HALF>(H, E, pt, JSTRIDE, prev_h);
            reverse_sweep_qp<R, HALF, R>(H, E, pb, JSTRIDE, bot_diag);
#pragma unroll
            for (int i = 0; i < HALF; ++i) {
                forward_cell(H[i], E[i], f_top, K);
                forward_cell(H[HALF + i], E[HALF + i], f_bot, K);
                if (i & 1) S = __vimax3_s16x2(S, H[i - 1], H[i]);
                if (i & 1) S = __vimax3_s16x2(S, H[HALF + i - 1], H[HALF + i]);
                if (!(i & 1) && i == HALF - 1) S = __vimax3_s16x2(S, H[i], H[HALF + i]);
            }
            mid_f = f_top;
            if (bot_valid) {
                out_h = H[R - 1];
                out_f = f_bot;
                if (t == T - 1) {
                    if (pass + 1 < P)
                        pbnd[2 * (ct - 1) + (pass & 1)] = make_uint2(out_h, out_f);
                    else if (seg & 2u)
                        a.seg_bnd[(size_t)off16 * 16 + 2 * (ct - 1) + half] =
                            make_uint2(out_h, out_f);
                }
            }
        }
        prev_h = h_in;
        d_bot = d_in;
        ++s;
        if (!done && s == nsteps) {   // uniform within the group
            __syncwarp(gmask);
            // per lane: segmented max over the threads of each query of this
            // pass; the segment's first thread adds it to the query's score
#pragma unroll
            for (int o = 1; o < T; o <<= 1) {
                const uint32_t v = __shfl_down_sync(gmask, S, o, T);
                const int vlo = __shfl_down_sync(gmask, q_lo, o, T);
                const int vhi = __shfl_down_sync(gmask, q_hi, o, T);
                uint32_t m = 0u;
                if (t + o < T) m = (vlo == q_lo ? 0x0000ffffu : 0u) | (vhi == q_hi ? 0xffff0000u : 0u);
                S = __vimax3_s16x2(S, (v & m) | (Z & ~m), Z);
            }
            const int gp = a.pair_ids ? (int)a.pair_ids[a.pair_begin + (unit >> 1)]
                                      : a.pair_begin + (unit >> 1);
            const int pos = 2 * gp + half;
            if (pos < a.n_records) {
                if (q_lo >= 0 && ((reset & 0xffffu) || t == 0)) {
                    const int s0 = lo16(S);
                    const int qb = q_lo * a.n_records;
                    atomicMax(a.scores + qb + pos, s0 - bias);
                    if (s0 >= a.ovf_thresh) {
                        const int j = atomicAdd(a.ovf_count, 1);
                        if (j < a.ovf_cap) a.ovf_list[j] = qb + pos;
                    }
                }
                if (q_hi >= 0 && ((reset >> 16) || t == 0)) {
                    const int s1 = hi16(S);
                    const int qb = q_hi * a.n_records;
                    atomicMax(a.scores + qb + pos, s1 - bias);
                    if (s1 >= a.ovf_thresh) {
                        const int j = atomicAdd(a.ovf_count, 1);
                        if (j < a.ovf_cap) a.ovf_list[j] = qb + pos;
                    }
                }
            }
            if (pass + 1 < P) {
                ++pass;
                SWQ_START_PASS()
            } else {
                const int v = __shfl_sync(gmask, next, 0, T);
                off16 = __shfl_sync(gmask, ninfo.off16, 0, T);
                ncols = (int)__shfl_sync(gmask, ninfo.ncols, 0, T);
                SWQ_TAKE_UNIT(v)
            }
        }
    }
#undef SWQ_TAKE_UNIT
#undef SWQ_START_PASS
}

// The paired-query batched kernel: blocks walk the double stacks in order.
template <int T, int R, int BLOCK>
__global__ void __launch_bounds__(BLOCK, 1) sw_qpbatch(const QpArgs a) {
    extern __shared__ uint4 prof4[];
    for (int i = 0; i < a.nstacks; ++i) {
        const int rows = (int)max(a.rows_lo[i], a.rows_hi[i]);
        const int P = (rows + T * R - 1) / (T * R);
        __syncthreads();        // every group is done with the previous profile
        build_profile_qp<T, R>(prof4, a.codes + a.off_lo[i], (int)a.rows_lo[i],
                               a.codes + a.off_hi[i], (int)a.rows_hi[i], a.mat, P);
        __syncthreads();
        run_qpairs<T, R>(a, prof4, P, a.counters + i, a.rb_map + a.rb_off[i],
                         a.seg_flags ? a.seg_flags[i] : 0u);
    }
}

}  // namespace swb
