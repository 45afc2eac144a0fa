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
#include <algorithm>
#include <vector>
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
    // several tall double stacks' segments in one launch: stack i uses the
    // boundary region seg_bnd + seg_slot[i] * seg_stride (null: region 0)
    const uint32_t* seg_slot;
    size_t seg_stride;
    // units [0, long_units) are the launch's long records (longest first):
    // they are scored before the rest, in items of one unit per group of a
    // block, all from one double stack, so that no block holds its groups at
    // a stack's end for one long unit
    int long_units;
};

// Host planning of paired lanes (batched search and serving).  Items (queries)
// come longest first with their rows padded to whole R-row blocks (`need`).
// An item taller than `seg` gets a lane of its own; those lanes are paired
// first (with an empty partner when their number is odd), and since a double
// stack computes whole passes of `pass_rows` rows, each of its lanes is then
// filled up to that height with the short items (first fit, longest first),
// rows that would otherwise be padding.  The remaining short items fill lanes
// of at most `seg` rows.  Consecutive lanes of the result form the double
// stacks (an even number of lanes).
struct PairLane {
    std::vector<uint32_t> items;
    uint32_t rows = 0;
};

inline std::vector<PairLane> plan_pair_lanes(const std::vector<uint32_t>& need, uint32_t seg,
                                             uint32_t pass_rows) {
    std::vector<PairLane> tall, shortl;
    std::vector<uint32_t> rest;
    for (uint32_t i = 0; i < (uint32_t)need.size(); ++i) {
        if (need[i] > seg) {
            PairLane ln;
            ln.items.push_back(i);
            ln.rows = need[i];
            tall.push_back(ln);
        } else {
            rest.push_back(i);
        }
    }
    if (tall.size() % 2) tall.push_back(PairLane{});
    std::vector<uint32_t> cap(tall.size());
    for (size_t d = 0; d + 1 < tall.size(); d += 2) {
        const uint32_t h = std::max(tall[d].rows, tall[d + 1].rows);
        cap[d] = cap[d + 1] = (h + pass_rows - 1) / pass_rows * pass_rows;
    }
    for (const uint32_t i : rest) {
        bool placed = false;
        for (size_t l = 0; l < tall.size() && !placed; ++l)
            if (tall[l].rows + need[i] <= cap[l]) {
                tall[l].items.push_back(i);
                tall[l].rows += need[i];
                placed = true;
            }
        for (size_t l = 0; l < shortl.size() && !placed; ++l)
            if (shortl[l].rows + need[i] <= seg) {
                shortl[l].items.push_back(i);
                shortl[l].rows += need[i];
                placed = true;
            }
        if (!placed) {
            PairLane ln;
            ln.items.push_back(i);
            ln.rows = need[i];
            shortl.push_back(ln);
        }
    }
    if (shortl.size() % 2) shortl.push_back(PairLane{});
    tall.insert(tall.end(), shortl.begin(), shortl.end());
    return tall;
}

// QpArgs::long_units of a launch over `count` pairs, longest first, whose
// column counts are ncols(p) and sum to cols_total, run by `groups` groups:
// both units of every leading pair longer than half of one group's share of
// a double stack (2 cols_total / groups).  A shorter unit, claimed at a
// stack's start, ends before the stack's other units run out.
template <class NCols>
inline int qp_long_units(NCols ncols, int count, uint64_t cols_total, long long groups) {
    if (count <= 0 || groups <= 0) return 0;
    const uint64_t thr = cols_total / (uint64_t)groups;
    int lo = 0, hi = count;            // the first pair with ncols <= thr
    while (lo < hi) {
        const int mid = lo + (hi - lo) / 2;
        if ((uint64_t)ncols(mid) > thr)
            lo = mid + 1;
        else
            hi = mid;
    }
    return 2 * lo;
}

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

// One column step of a thread's two halves with packed profile words: the
// top half (rows [0, R/2)) on column c at pt, the bottom half on column c - 1
// at pb (see column_step in sw_wavefront.cuh for the carried values).
template <int R, int JSTRIDE>
__device__ __forceinline__ void column_step_qp(uint32_t (&H)[R], uint32_t (&E)[R],
                                               const uint4* pt, const uint4* pb,
                                               uint32_t prev_h, uint32_t f_in,
                                               uint32_t& mid_h, uint32_t& mid_f,
                                               uint32_t& out_h, uint32_t& out_f,
                                               uint32_t& S_top, uint32_t& S_bot,
                                               const CellK& K) {
    constexpr int HALF = R / 2;
    const uint32_t bot_diag = mid_h;
    uint32_t f_top = f_in, f_bot = mid_f;
    mid_h = H[HALF - 1];
    reverse_sweep_qp<R, 0, HALF>(H, E, pt, JSTRIDE, prev_h);
    reverse_sweep_qp<R, HALF, R>(H, E, pb, JSTRIDE, bot_diag);
#pragma unroll
    for (int i = 0; i < HALF; ++i) {
        forward_cell(H[i], E[i], f_top, K);
        forward_cell(H[HALF + i], E[HALF + i], f_bot, K);
        if (i & 1) S_top = __vimax3_s16x2(S_top, H[i - 1], H[i]);
        if (i & 1) S_bot = __vimax3_s16x2(S_bot, H[HALF + i - 1], H[HALF + i]);
    }
    mid_f = f_top;
    out_h = H[R - 1];
    out_f = f_bot;
}

// One double stack: every group claims units (records) and scores them
// against both lanes' stacks.  Returns when the units are exhausted.  The
// groups stream from pass to pass and unit to unit without draining, as in
// run_stream (sw_wavefront.cuh), with the maximum chain and the last-thread
// atomicMax done per lane (each lane has its own query map).  Rows above pass
// 0 come from seg_bnd when the stack continues an earlier segment (bit 0 of
// seg), and the last pass writes its last row there for the next segment
// (bit 1): a column is read (pass 0, thread 0) 2T + 1 steps before the last
// pass's thread T-1 writes it, so one buffer serves both.
//
// Units come from `counter` (unit_first + claims, up to units_end) or, with a
// null counter, the group scores the one unit `single` (none when single >=
// units_end).
template <int T, int R>
__device__ __forceinline__ void run_qpairs(const QpArgs& a, const uint4* prof, int P, int* counter,
                                           const int2* rb_map, uint32_t seg, size_t seg_base,
                                           int unit_first, int units_end, int single) {
    static_assert(R % 8 == 0, "R");
    constexpr int NJ = R / 4;
    constexpr int HALF = R / 2;
    constexpr int SLOTS = GroupShape<T>::SLOTS;
    constexpr int JSTRIDE = kCodes * SLOTS;
    constexpr int PSTRIDE = NJ * JSTRIDE;
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
    const int units = units_end;
    const int dep_steps = 2 * T + 2;
    // thread 0 claims the group's units
    auto claim = [&]() -> int {
        if (counter) return unit_first + atomicAdd(counter, 1);
        const int v = single;
        single = units;
        return v;
    };
    uint2* const pbnd = a.bnd + (size_t)((blockIdx.x * blockDim.x + threadIdx.x) / T) * a.bnd_group;

    uint32_t H[R], E[R];
#pragma unroll
    for (int k = 0; k < R; ++k) {
        H[k] = Z;
        E[k] = Z;
    }
    uint32_t S_top = Z, S_bot = Z, S_pend = Z, acc_out = Z;
    uint32_t out_h = Z, out_f = Z, prev_h = Z, mid_h = Z, mid_f = Z;
    uint32_t d_bot = kZeroCode, d_cur = kZeroCode;
    // the top half's segment
    int unit = 0, half = 0, pass = 0, ncols = 0, nst = 0, c = 0;
    uint32_t off16 = 0u;
    const unsigned short* col = reinterpret_cast<const unsigned short*>(a.db);
    const uint4* prof_t = prof + slot;
    uint2* wrow = pbnd;        // where thread T-1 writes the last row ...
    int wlim = 0;              // ... for columns below this (0: nowhere)
    int q_lo = -1, q_hi = -1;
    uint32_t reset = 0u;       // lanes whose query starts at this thread's first row
    uint32_t last = 0u;        // lanes whose query's rows end at this thread's last row
    // the bottom half's view: the top's of the previous step
    const uint4* prof_b = prof_t;
    uint2* b_wrow = wrow;
    int b_wlim = 0, b_col = -1;
    // a segment whose maxima are being finished
    int f_unit = 0, fq_lo = -1, fq_hi = -1;
    uint32_t f_reset = 0u, f_last = 0u;
    bool fpend = false, fin = false;
    // thread 0: the next unit (claimed one unit ahead) and the rows above
    int next = 0;
    Pair2 ninfo{0u, 0u};
    uint2 bq0 = make_uint2(Z, Z), bq1 = bq0;
    bool has_in = false;
    const uint2* rrow = pbnd;

#define SWQ_SET_SEG()                                                          \
    {                                                                          \
        const int lo = (pass + 1 < P) ? dep_steps : 3;                         \
        nst = ncols > lo ? ncols : lo;                                         \
        col = reinterpret_cast<const unsigned short*>(a.db) + (size_t)off16 * 8; \
        uint2* const sb = a.seg_bnd + seg_base + (size_t)off16 * 16 + half;    \
        wrow = (pass + 1 < P) ? pbnd + (pass & 1) : sb;                        \
        wlim = (pass + 1 < P || (seg & 2u)) ? ncols : 0;                       \
        has_in = pass > 0 || (seg & 1u);                                       \
        rrow = pass > 0 ? pbnd + ((pass - 1) & 1) : sb;                        \
        prof_t = prof + pass * PSTRIDE + slot;                                 \
        const int2 rb = rb_map[pass * T + t];                                  \
        const int2 rn = (t + 1 < T) ? rb_map[pass * T + t + 1] : make_int2(-1, -1); \
        q_lo = rb.x < 0 ? -1 : (rb.x & (kFirstBit - 1));                       \
        q_hi = rb.y < 0 ? -1 : (rb.y & (kFirstBit - 1));                       \
        reset = ((rb.x >= 0 && (rb.x & kFirstBit)) ? 0x0000ffffu : 0u) |       \
                ((rb.y >= 0 && (rb.y & kFirstBit)) ? 0xffff0000u : 0u);        \
        last = ((rn.x < 0 || (rn.x & kFirstBit)) ? 0x0000ffffu : 0u) |         \
               ((rn.y < 0 || (rn.y & kFirstBit)) ? 0xffff0000u : 0u);          \
    }

    {
        int v = 0;
        if (t == 0) v = claim();
        v = __shfl_sync(gmask, v, 0, T);
        unit = v;
        if (v < units) {
            const Pair2 pr = a.pairs[a.pair_begin + (v >> 1)];
            off16 = pr.off16;
            ncols = (int)pr.ncols;
            half = v & 1;
            if (t == 0) next = claim();
        } else {
            fin = true;
        }
        SWQ_SET_SEG()
        c = -2 * t;
        d_cur = (t == 0 && ncols > 0) ? (((uint32_t)__ldg(col) >> (8 * half)) & 0xffu)
                                      : (uint32_t)kZeroCode;
        if (t == 0 && has_in) {
            if (ncols > 0) bq0 = rrow[0];
            if (ncols > 1) bq1 = rrow[2];
        }
    }

    while (!__all_sync(FULL, fin)) {
        __syncwarp();                 // orders the boundary rows' stores and loads
        uint32_t h_in = __shfl_up_sync(FULL, out_h, 1, T);
        uint32_t f_in = __shfl_up_sync(FULL, out_f, 1, T);
        const uint32_t acc_in = __shfl_up_sync(FULL, acc_out, 1, T);
        const uint32_t d_in = d_cur;
        {
            const int c1 = c + 1;
            d_cur = (c1 >= 0 && c1 < ncols) ? (((uint32_t)__ldg(col + c1) >> (8 * half)) & 0xffu)
                                             : (uint32_t)kZeroCode;
        }
        if (t == 0) {
            h_in = Z;
            f_in = Z;
            if (has_in && c < ncols) {
                h_in = bq0.x;
                f_in = bq0.y;
                bq0 = bq1;
                if (c + 2 < ncols) bq1 = rrow[2 * (c + 2)];
            }
            // the next unit's pair entry, once its claim has returned
            if (pass == 0 && c == (nst < 9 ? nst - 1 : 8) && next < units)
                ninfo = a.pairs[a.pair_begin + (next >> 1)];
        }
        // a lane whose query starts here takes nothing from above
        h_in = (h_in & ~reset) | (Z & reset);
        f_in = (f_in & ~reset) | (Z & reset);
        if (!fin && c >= 0) {
            column_step_qp<R, JSTRIDE>(H, E, prof_t + (int)d_in * SLOTS,
                                       prof_b + (int)d_bot * SLOTS, prev_h, f_in, mid_h, mid_f,
                                       out_h, out_f, S_top, S_bot, K);
            if (t == T - 1 && b_col >= 0 && b_col < b_wlim)
                b_wrow[2 * b_col] = make_uint2(out_h, out_f);
        }
        prev_h = h_in;
        d_bot = d_in;
        prof_b = prof_t;
        b_wrow = wrow;
        b_wlim = wlim;
        b_col = c;
        if (fpend) {
            // the bottom has just done the finished segment's last column:
            // per lane, this thread's maximum joins its query's chain
            fpend = false;
            uint32_t m = __vimax3_s16x2(S_pend, S_bot, Z);
            const uint32_t cont = (t > 0) ? ~f_reset : 0u;
            m = __vimax3_s16x2(m, (acc_in & cont) | (Z & ~cont), Z);
            acc_out = m;
            const int gp = a.pair_ids ? (int)a.pair_ids[a.pair_begin + (f_unit >> 1)]
                                      : a.pair_begin + (f_unit >> 1);
            const int pos = 2 * gp + (f_unit & 1);
            if (pos < a.n_records) {
                if (fq_lo >= 0 && (f_last & 0xffffu)) {
                    const int s0 = lo16(m);
                    const int qb = fq_lo * a.n_records;
                    atomicMax(a.scores + qb + pos, s0 - bias);
                    if (s0 >= a.ovf_thresh) {
                        const int j = atomicAdd(a.ovf_count, 1);
                        if (j < a.ovf_cap) a.ovf_list[j] = qb + pos;
                    }
                }
                if (fq_hi >= 0 && (f_last >> 16)) {
                    const int s1 = hi16(m);
                    const int qb = fq_hi * a.n_records;
                    atomicMax(a.scores + qb + pos, s1 - bias);
                    if (s1 >= a.ovf_thresh) {
                        const int j = atomicAdd(a.ovf_count, 1);
                        if (j < a.ovf_cap) a.ovf_list[j] = qb + pos;
                    }
                }
            }
            S_bot = Z;
            if (unit >= units) fin = true;
        }
        if (c == 0) {   // the bottom starts this segment's column 0 next step
#pragma unroll
            for (int k = HALF; k < R; ++k) {
                H[k] = Z;
                E[k] = Z;
            }
        }
        const bool adv = !fin && c == nst - 1;
        if (__any_sync(FULL, adv)) {
            const int up_unit = __shfl_up_sync(FULL, unit, 1, T);
            const uint32_t up_off = __shfl_up_sync(FULL, off16, 1, T);
            const int up_ncols = __shfl_up_sync(FULL, ncols, 1, T);
            if (adv) {
                S_pend = S_top;
                S_top = Z;
                f_unit = unit;
                fq_lo = q_lo;
                fq_hi = q_hi;
                f_reset = reset;
                f_last = last;
                fpend = true;
                if (pass + 1 < P) {
                    ++pass;
                } else {
                    pass = 0;
                    if (t == 0) {
                        unit = next;
                        off16 = ninfo.off16;
                        ncols = (int)ninfo.ncols;
                        if (unit < units) next = claim();
                    } else {
                        unit = up_unit;
                        off16 = up_off;
                        ncols = up_ncols;
                    }
                    if (unit >= units) ncols = 0;
                    half = unit & 1;
                }
                SWQ_SET_SEG()
                c = -1;
#pragma unroll
                for (int k = 0; k < HALF; ++k) {
                    H[k] = Z;
                    E[k] = Z;
                }
                prev_h = Z;
                if (t == 0 && has_in) {
                    if (ncols > 0) bq0 = rrow[0];
                    if (ncols > 1) bq1 = rrow[2];
                }
                d_cur = (ncols > 0) ? (((uint32_t)__ldg(col) >> (8 * half)) & 0xffu)
                                    : (uint32_t)kZeroCode;
            }
        }
        ++c;

        // Plain steps, as in run_stream: as many as every lane of the warp can
        // take with no segment event and no bounds guard.  The bottom half's
        // profile base is then the top's, so it takes the top's residue of
        // the step before; the residue is loaded as the unit's own byte.
        {
            int k = 0;
            if (!fin && c >= 1 && !(t == 0 && pass == 0 && c <= (nst < 9 ? nst - 1 : 8))) {
                const int lastc = min(nst - 2, ncols - 3);
                k = max(lastc - c + 1, 0);
            }
            k = (int)__reduce_min_sync(FULL, (unsigned)k);
            const bool rd0 = t == 0 && has_in;
            const bool z0 = t == 0 && !has_in;
            const bool wr = t == T - 1 && wlim > 0;
            const uint32_t keep = ~reset, zr = Z & reset;
            const uint8_t* colb = reinterpret_cast<const uint8_t*>(col) + half;
            for (; k > 0; --k) {
                __syncwarp();
                uint32_t h_in = __shfl_up_sync(FULL, out_h, 1, T);
                uint32_t f_in = __shfl_up_sync(FULL, out_f, 1, T);
                const uint32_t d_in = d_cur;
                d_cur = (uint32_t)__ldg(colb + 2 * (c + 1));
                if (rd0) {
                    h_in = bq0.x;
                    f_in = bq0.y;
                    bq0 = bq1;
                    bq1 = rrow[2 * (c + 2)];
                }
                if (z0) {
                    h_in = Z;
                    f_in = Z;
                }
                h_in = (h_in & keep) | zr;
                f_in = (f_in & keep) | zr;
                column_step_qp<R, JSTRIDE>(H, E, prof_t + (int)d_in * SLOTS,
                                           prof_t + (int)d_bot * SLOTS, prev_h, f_in, mid_h,
                                           mid_f, out_h, out_f, S_top, S_bot, K);
                if (wr) wrow[2 * (c - 1)] = make_uint2(out_h, out_f);
                prev_h = h_in;
                d_bot = d_in;
                b_col = c;
                ++c;
            }
        }
    }
#undef SWQ_SET_SEG
}

// The paired-query batched kernel.  First the long units: items of G = BLOCK
// / T consecutive long units of one double stack (similar lengths, the pair
// table being longest first), one per group, dealt to the blocks round-robin
// (block b takes items b, b + gridDim.x, ...; a block left with less long
// work starts the rest earlier); then the blocks walk the double stacks in
// order, claiming the other units.  The kernel holds no static shared memory
// (the host gives the dynamic profile the whole opt-in maximum).
template <int T, int R, int BLOCK>
__global__ void __launch_bounds__(BLOCK, 1) sw_qpbatch(const QpArgs a) {
    extern __shared__ uint4 prof4[];
    constexpr int G = BLOCK / T;
    const int units = 2 * a.pair_count;
    const int n_long = min(a.long_units, units);
    int cur = -1;               // the double stack whose profile is in shared memory
    auto stage = [&](int i) {   // caller: every group is done with the previous profile
        const int rows = (int)max(a.rows_lo[i], a.rows_hi[i]);
        const int P = (rows + T * R - 1) / (T * R);
        if (i != cur) {
            build_profile_qp<T, R>(prof4, a.codes + a.off_lo[i], (int)a.rows_lo[i],
                                   a.codes + a.off_hi[i], (int)a.rows_hi[i], a.mat, P);
            cur = i;
        }
        __syncthreads();
        return P;
    };
    if (n_long > 0) {
        const int per = (n_long + G - 1) / G;
        const int items = per * a.nstacks;
        for (int it = (int)blockIdx.x; it < items; it += (int)gridDim.x) {
            __syncthreads();    // every group is done with the previous item
            const int i = it / per;
            const int u = (it - i * per) * G + (int)threadIdx.x / T;
            const int P = stage(i);
            run_qpairs<T, R>(a, prof4, P, nullptr, a.rb_map + a.rb_off[i],
                             a.seg_flags ? a.seg_flags[i] : 0u,
                             a.seg_slot ? (size_t)a.seg_slot[i] * a.seg_stride : (size_t)0, 0,
                             n_long, u);
        }
    }
    for (int i = 0; i < a.nstacks; ++i) {
        __syncthreads();        // every group is done with the previous profile
        const int P = stage(i);
        run_qpairs<T, R>(a, prof4, P, a.counters + i, a.rb_map + a.rb_off[i],
                         a.seg_flags ? a.seg_flags[i] : 0u,
                         a.seg_slot ? (size_t)a.seg_slot[i] * a.seg_stride : (size_t)0, n_long,
                         units, 0);
    }
}

}  // namespace swb
