// sw_aux.cu -- exact 32-bit re-score of overflowed records, score finalisation
// and top-k selection.
//
// The reference re-scores int8-overflowed records on the host after all
// workers have finished (RecalcWorker::recalc_launch, src/RecalcWorker.cpp:
// 99-268, 16 int16 lanes, saturating at 65535).  Here the first pass is
// already 16-bit, and the few records whose 16-bit lane may have wrapped are
// re-scored on the device in plain int32, from the compacted list the first
// pass appended to.  With SW_FLAG_REFERENCE_CAP the result is then clamped to
// 65535, which is exactly what the reference reports.
#include <cstdint>
#include "sw_aux.h"
#include "sw_device.cuh"

namespace swb {

constexpr int kRsRows = 16;        // query rows per lane in the 32-bit pass

// One warp per overflowed record: the same anti-diagonal wavefront as the
// first pass (32 lanes x 16 rows per pass), int32 arithmetic, profile taken
// from a shared copy of the matrix.  The boundary row between query passes is
// the warp's own scratch row, so any two records (of the same or of
// different queries) can be re-scored concurrently.
__global__ void __launch_bounds__(64) sw_rescore32(const RescoreArgs a) {
    __shared__ int smat[32 * 32];
    for (int i = threadIdx.x; i < 1024; i += blockDim.x) smat[i] = a.mat[i];
    __syncthreads();
    constexpr unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    uint2* pb = a.scratch + (size_t)warp * a.max_cols;
    const int count = min(*a.ovf_count, a.ovf_cap);
    for (int it = warp; it < count; it += nwarps) {
        const int entry = a.ovf_list[it];
        int pos = entry;
        const uint8_t* query = a.query;
        int qlen = a.qlen;
        if (a.qoff) {
            const int q = entry / a.n_records;
            pos = entry - q * a.n_records;
            query = a.queries + a.qoff[q];
            qlen = (int)a.qlens[q];
        }
        const Pair2 pr = a.pairs[pos >> 1];
        const int sel = pos & 1;
        const uint8_t* seq = reinterpret_cast<const uint8_t*>(a.db + pr.off16);
        const int ncols = (int)pr.ncols;
        const int rows_per_pass = 32 * kRsRows;
        const int P = (qlen + rows_per_pass - 1) / rows_per_pass;
        int S = 0;
        for (int pass = 0; pass < P; ++pass) {
            int qc[kRsRows], H[kRsRows], E[kRsRows];
#pragma unroll
            for (int k = 0; k < kRsRows; ++k) {
                const int row = pass * rows_per_pass + lane * kRsRows + k;
                qc[k] = (row < qlen) ? (int)(query[row] & 31) * 32 : kZeroCode * 32;
                H[k] = 0;
                E[k] = 0;
            }
            int out_h = 0, out_f = 0, prev_h = 0, myd = kZeroCode;
            for (int s = 0; s < ncols + 31; ++s) {
                int d_in = __shfl_up_sync(FULL, myd, 1);
                int h_in = __shfl_up_sync(FULL, out_h, 1);
                int f_in = __shfl_up_sync(FULL, out_f, 1);
                if (lane == 0) {
                    d_in = kZeroCode;
                    h_in = 0;
                    f_in = 0;
                    if (s < ncols) {
                        d_in = seq[2 * s + sel] & 31;
                        if (pass > 0) {
                            const uint2 b = pb[s];
                            h_in = (int)b.x;
                            f_in = (int)b.y;
                        }
                    }
                }
                __syncwarp();
                const int c = s - lane;
                if (c >= 0 && c < ncols) {
                    int diag = prev_h, f = f_in;
#pragma unroll
                    for (int k = 0; k < kRsRows; ++k) {
                        int h = max(diag + smat[qc[k] + d_in], E[k]);
                        h = max(max(h, f), 0);
                        diag = H[k];
                        H[k] = h;
                        S = max(S, h);
                        const int hq = h - a.gap_oe;
                        E[k] = max(E[k] - a.gap_e, hq);
                        f = max(f - a.gap_e, hq);
                    }
                    out_h = H[kRsRows - 1];
                    out_f = f;
                    if (lane == 31 && pass + 1 < P) pb[c] = make_uint2((uint32_t)out_h, (uint32_t)out_f);
                }
                prev_h = h_in;
                myd = d_in;
                __syncwarp();
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) S = max(S, __shfl_xor_sync(FULL, S, o));
        if (lane == 0) a.scores[entry] = S;
        __syncwarp();
    }
}

// Top-k, one block: sort 4096 64-bit keys in shared memory (bitonic,
// descending) and keep the first k.  Key = score << 32 | ~record_index, so the
// order is score descending, then record index ascending.  In the first round
// the keys are made from the per-position scores (clamped when asked) and the
// position -> record permutation, and the record-order score array is filled.
__global__ void __launch_bounds__(kTopkThreads) sw_topk_round(const TopkArgs a) {
    __shared__ unsigned long long sk[kTopkKeys];
    const long long base = (long long)blockIdx.x * kTopkKeys;
    const long long y = blockIdx.y;                 // query of a batch
    const long long ys = (a.rows && !a.keys_in) ? a.rows[y] : y;   // its score row
    for (int i = threadIdx.x; i < kTopkKeys; i += kTopkThreads) {
        const long long g = base + i;
        unsigned long long key = 0ull;
        if (g < a.n) {
            if (a.keys_in) {
                key = a.keys_in[y * a.in_stride + g];
            } else {
                int s = a.scores[ys * a.in_stride + g];
                if (a.cap && s > 65535) s = 65535;
                const uint32_t rec = a.perm[g];
                if (a.scores_by_record) a.scores_by_record[ys * a.rec_stride + rec] = s;
                if (s > 0) key = ((unsigned long long)(uint32_t)s << 32) | (0xffffffffu - rec);
            }
        }
        sk[i] = key;
    }
    __syncthreads();
    for (int size = 2; size <= kTopkKeys; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int i = threadIdx.x; i < kTopkKeys / 2; i += kTopkThreads) {
                const int lo = 2 * i - (i & (stride - 1));
                const int hi = lo + stride;
                const bool desc = (lo & size) == 0;
                const unsigned long long x = sk[lo], y = sk[hi];
                if (desc ? (x < y) : (x > y)) {
                    sk[lo] = y;
                    sk[hi] = x;
                }
            }
            __syncthreads();
        }
    }
    for (int i = threadIdx.x; i < a.k; i += kTopkThreads)
        a.keys_out[y * a.out_stride + (long long)blockIdx.x * a.k + i] = sk[i];
}

}  // namespace swb
