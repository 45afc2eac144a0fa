// sw_traceback.cu -- alignments (coordinates and CIGAR) of chosen DB records.
//
// The reference reports scores and record titles only (WorkerPool::showResult,
// src/WorkerPool.cpp:130-155); it has no traceback.  sw_traceback gives the
// caller the best local alignment of the query against each record it names
// (typically the top-k hits of a search):
//   * one warp per record runs the exact int32 Gotoh recurrence as an
//     anti-diagonal wavefront (32 lanes x 16 query rows per pass, the last
//     row of a pass handed to the next through a boundary row in global
//     memory, as in the 32-bit re-score) and stores 4 direction bits per
//     cell: where H came from (zero / diagonal / E / F) and whether the next
//     E and the next F were opened at this cell;
//   * the end cell is the first cell with the maximal H in column-major order
//     (record position, then query position);
//   * lane 0 then walks the bits back from the end cell: in H it stops at
//     H = 0 and otherwise prefers the diagonal, then E, then F; inside a gap it
//     prefers "opened here" over "extended" on ties.
// The direction bits take qlen x record length / 2 bytes per record, in a
// scratch buffer the context keeps (grown on demand, bounded per call).
#include <algorithm>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/swb200.h"
#include "sw_device.cuh"
#include "sw_engine.h"

using namespace swb;

namespace {

constexpr int kTbRows = 16;                    // query rows per lane and pass
constexpr int kTbPassRows = 32 * kTbRows;      // rows per pass
constexpr int kTbNeg = -(1 << 28);             // below any reachable E/F
constexpr size_t kTbMaxScratch = (size_t)8 << 30;   // direction bits + boundary rows per call

struct TbJob {
    uint32_t pos;          // sorted position of the record (pair = pos / 2, half = pos % 2)
    uint32_t dlen;         // record length
    uint64_t dir;          // first direction word (uint2 units)
    uint64_t bnd;          // first boundary entry (int2 units)
    uint64_t ops;          // first op byte
};

struct TbOut {
    int32_t score;
    uint32_t q_begin, q_end, d_begin, d_end;
    uint32_t n_ops, matches, pad;
};

struct TbArgs {
    const uint8_t* db;     // the resident column streams, as bytes
    const Pair2* pairs;
    const uint8_t* query;
    int qlen;
    const int8_t* mat;
    int gap_oe, gap_e;
    int n;
    const TbJob* jobs;
    uint2* dir;
    int2* bnd;
    uint8_t* ops;          // per job: qlen + dlen bytes, written last op first
    TbOut* out;
};

__device__ __forceinline__ uint32_t tb_bits(const uint2* dir, int dlen, int i, int j) {
    const int pass = i / kTbPassRows;
    const int lane = (i % kTbPassRows) / kTbRows;
    const int k = i % kTbRows;
    const uint2 w = dir[((size_t)pass * 32 + lane) * dlen + j];
    const uint32_t half = k < 8 ? w.x : w.y;
    return (half >> (4 * (k & 7))) & 15u;
}

__global__ void __launch_bounds__(128) sw_traceback_kernel(const TbArgs a) {
    __shared__ int smat[1024];
    for (int i = threadIdx.x; i < 1024; i += blockDim.x) smat[i] = a.mat[i];
    __syncthreads();
    constexpr unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (wid >= a.n) return;                                  // warp-uniform
    const TbJob job = a.jobs[wid];
    const int dlen = (int)job.dlen;
    const int qlen = a.qlen;
    const uint8_t* rec = a.db + (size_t)a.pairs[job.pos >> 1].off16 * 16 + (job.pos & 1);
    uint2* dir = a.dir + job.dir;
    int2* bnd = a.bnd + job.bnd;
    const int P = (qlen + kTbPassRows - 1) / kTbPassRows;
    int best = 0, bcol = 0x7fffffff, brow = 0x7fffffff;
    for (int pass = 0; pass < P; ++pass) {
        const int r0 = pass * kTbPassRows + lane * kTbRows;
        int qc[kTbRows], H[kTbRows], E[kTbRows];
#pragma unroll
        for (int k = 0; k < kTbRows; ++k) {
            qc[k] = (r0 + k < qlen) ? (int)(a.query[r0 + k] & 31) * 32 : 24 * 32;
            H[k] = 0;
            E[k] = kTbNeg;
        }
        int out_h = 0, out_f = kTbNeg, prev_h = 0;
        for (int s = 0; s < dlen + 31; ++s) {
            int h_in = __shfl_up_sync(FULL, out_h, 1);
            int f_in = __shfl_up_sync(FULL, out_f, 1);
            if (lane == 0) {
                h_in = 0;
                f_in = kTbNeg;
                if (pass > 0 && s < dlen) {
                    const int2 b = bnd[s];
                    h_in = b.x;
                    f_in = b.y;
                }
            }
            const int c = s - lane;
            if (c >= 0 && c < dlen) {
                const int dres = rec[2 * (size_t)c] & 31;
                int diag = prev_h, f = f_in;
                uint32_t w0 = 0u, w1 = 0u;
#pragma unroll
                for (int k = 0; k < kTbRows; ++k) {
                    const int hd = diag + smat[qc[k] + dres];
                    const int h = max(max(hd, E[k]), max(f, 0));
                    const uint32_t src = h == 0 ? 0u : h == hd ? 1u : h == E[k] ? 2u : 3u;
                    const int eo = h - a.gap_oe, ee = E[k] - a.gap_e;
                    const int fo = h - a.gap_oe, fe = f - a.gap_e;
                    const uint32_t nib = src | (eo >= ee ? 4u : 0u) | (fo >= fe ? 8u : 0u);
                    E[k] = max(eo, ee);
                    f = max(fo, fe);
                    diag = H[k];
                    H[k] = h;
                    if (k < 8) w0 |= nib << (4 * k); else w1 |= nib << (4 * (k - 8));
                    if (r0 + k < qlen && h > best) {
                        best = h;
                        bcol = c;
                        brow = r0 + k;
                    }
                }
                out_h = H[kTbRows - 1];
                out_f = f;
                dir[((size_t)pass * 32 + lane) * dlen + c] = make_uint2(w0, w1);
                if (lane == 31 && pass + 1 < P) bnd[c] = make_int2(out_h, out_f);
            }
            prev_h = h_in;
            __syncwarp();
        }
    }
    // end cell: maximal score, then smallest record position, then smallest row
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const int b2 = __shfl_xor_sync(FULL, best, o);
        const int c2 = __shfl_xor_sync(FULL, bcol, o);
        const int r2 = __shfl_xor_sync(FULL, brow, o);
        if (b2 > best || (b2 == best && (c2 < bcol || (c2 == bcol && r2 < brow)))) {
            best = b2;
            bcol = c2;
            brow = r2;
        }
    }
    __syncwarp();            // every lane's direction words are visible to lane 0
    if (lane != 0) return;
    TbOut o{};
    o.score = best;
    if (best > 0) {
        uint8_t* ops = a.ops + job.ops;
        const uint32_t cap = (uint32_t)qlen + job.dlen;
        int i = brow, j = bcol, si = brow, sj = bcol, state = 0;    // 0 H, 1 E, 2 F
        uint32_t n = 0, matches = 0;
        while (n < cap) {
            if (state == 0) {
                if (i < 0 || j < 0) break;
                const uint32_t src = tb_bits(dir, dlen, i, j) & 3u;
                if (src == 0u) break;
                if (src == 1u) {
                    ops[n++] = 0;
                    matches += ((a.query[i] & 31) == (rec[2 * (size_t)j] & 31)) ? 1u : 0u;
                    si = i;
                    sj = j;
                    --i;
                    --j;
                } else {
                    state = src == 2u ? 1 : 2;
                }
            } else if (state == 1) {
                ops[n++] = 2;
                const uint32_t opened = (tb_bits(dir, dlen, i, j - 1) >> 2) & 1u;
                --j;
                state = opened ? 0 : 1;
            } else {
                ops[n++] = 1;
                const uint32_t opened = (tb_bits(dir, dlen, i - 1, j) >> 3) & 1u;
                --i;
                state = opened ? 0 : 2;
            }
        }
        o.q_begin = (uint32_t)si;
        o.q_end = (uint32_t)brow + 1;
        o.d_begin = (uint32_t)sj;
        o.d_end = (uint32_t)bcol + 1;
        o.n_ops = n;
        o.matches = matches;
    }
    a.out[wid] = o;
}

template <typename T>
cudaError_t grow(T** p, size_t& cap, size_t need) {
    if (need <= cap) return cudaSuccess;
    dev_free(*p);
    cap = 0;
    cudaError_t e = dev_alloc(p, need);
    if (e == cudaSuccess) cap = need;
    return e;
}

}  // namespace

struct sw_tb_state {
    uint2* d_dir = nullptr;
    size_t dir_cap = 0;
    int2* d_bnd = nullptr;
    size_t bnd_cap = 0;
    uint8_t* d_ops = nullptr;
    size_t ops_cap = 0;
    TbJob* d_jobs = nullptr;
    size_t jobs_cap = 0;
    TbOut* d_out = nullptr;
    size_t out_cap = 0;
};

namespace swb {
void free_traceback(sw_ctx* ctx) {
    sw_tb_state* t = ctx->tb;
    if (!t) return;
    dev_free(t->d_dir);
    dev_free(t->d_bnd);
    dev_free(t->d_ops);
    dev_free(t->d_jobs);
    dev_free(t->d_out);
    delete t;
    ctx->tb = nullptr;
}
}  // namespace swb

extern "C" sw_status sw_traceback(sw_ctx* ctx, const uint8_t* query, uint32_t qlen,
                                  const uint64_t* records, uint32_t n, sw_alignment* out,
                                  uint32_t* ops, uint64_t ops_cap, uint64_t* ops_used) {
    if (!ctx) return SW_ERR_INVALID;
    if (ctx->serve) return SW_ERR_BUSY;   // the serving loop owns the stream
    if (!ctx->db_loaded) SW_SET(ctx, SW_ERR_STATE, "no DB loaded (call sw_db_load first)");
    if (!ops_used || (n && (!records || !out)) || (qlen && !query))
        SW_SET(ctx, SW_ERR_INVALID, "null argument");
    *ops_used = 0;
    if (n == 0) return SW_OK;
    for (uint32_t i = 0; i < qlen; ++i)
        if (query[i] > 24) SW_SET(ctx, SW_ERR_INVALID, "query code %d at %u", query[i], i);
    for (uint32_t h = 0; h < n; ++h) {
        if (records[h] >= (uint64_t)ctx->n_records)
            SW_SET(ctx, SW_ERR_INVALID, "record %llu out of range",
                   (unsigned long long)records[h]);
        out[h] = sw_alignment{};
        out[h].index = records[h];
    }
    if (qlen == 0) return SW_OK;
    SW_CUDA(ctx, cudaSetDevice(ctx->device));
    if (!ctx->tb) ctx->tb = new sw_tb_state();
    sw_tb_state* tb = ctx->tb;
    const uint64_t P = (qlen + kTbPassRows - 1) / kTbPassRows;
    // jobs in rounds whose scratch fits the per-call bound
    std::vector<TbJob> jobs(n);
    std::vector<TbOut> res(n);
    uint64_t ops_total = 0;
    for (uint32_t h = 0; h < n; ++h) {
        const uint64_t dlen = ctx->rec_len[records[h]];
        const size_t need = (size_t)(P * 32 * dlen) * sizeof(uint2) + dlen * sizeof(int2);
        if (need > kTbMaxScratch)
            SW_SET(ctx, SW_ERR_UNSUPPORTED,
                   "traceback of a %u x %llu matrix needs %zu bytes of direction bits (limit %zu)",
                   qlen, (unsigned long long)dlen, need, kTbMaxScratch);
        jobs[h].pos = ctx->rec_pos[records[h]];
        jobs[h].dlen = (uint32_t)dlen;
    }
    std::vector<uint8_t> hops;
    uint32_t h0 = 0;
    while (h0 < n) {
        uint64_t dir = 0, bnd = 0, opsb = 0;
        uint32_t h1 = h0;
        while (h1 < n) {
            const uint64_t dlen = jobs[h1].dlen;
            const uint64_t ndir = P * 32 * dlen, nbnd = dlen;
            if (h1 > h0 && (dir + ndir) * sizeof(uint2) + (bnd + nbnd) * sizeof(int2) > kTbMaxScratch)
                break;
            jobs[h1].dir = dir;
            jobs[h1].bnd = bnd;
            jobs[h1].ops = opsb;
            dir += ndir;
            bnd += nbnd;
            opsb += qlen + dlen;
            ++h1;
        }
        const uint32_t m = h1 - h0;
        cudaStream_t st = ctx->stream;
        sw_status s = ensure_query_buffers(ctx, qlen);
        if (s != SW_OK) return s;
        memcpy(ctx->h_query, query, qlen);
        if (grow(&tb->d_dir, tb->dir_cap, std::max<uint64_t>(dir, 1)) != cudaSuccess ||
            grow(&tb->d_bnd, tb->bnd_cap, std::max<uint64_t>(bnd, 1)) != cudaSuccess ||
            grow(&tb->d_ops, tb->ops_cap, std::max<uint64_t>(opsb, 1)) != cudaSuccess ||
            grow(&tb->d_jobs, tb->jobs_cap, m) != cudaSuccess ||
            grow(&tb->d_out, tb->out_cap, m) != cudaSuccess)
            SW_SET(ctx, SW_ERR_NOMEM, "device allocation failed: traceback scratch");
        SW_CUDA(ctx, cudaMemcpyAsync(ctx->d_query, ctx->h_query, qlen, cudaMemcpyHostToDevice, st));
        SW_CUDA(ctx, cudaMemcpyAsync(tb->d_jobs, jobs.data() + h0, m * sizeof(TbJob),
                                     cudaMemcpyHostToDevice, st));
        TbArgs a;
        a.db = reinterpret_cast<const uint8_t*>(ctx->d_db);
        a.pairs = ctx->d_pairs;
        a.query = ctx->d_query;
        a.qlen = (int)qlen;
        a.mat = ctx->d_mat;
        a.gap_oe = ctx->params.gap_open + ctx->params.gap_extend;
        a.gap_e = ctx->params.gap_extend;
        a.n = (int)m;
        a.jobs = tb->d_jobs;
        a.dir = tb->d_dir;
        a.bnd = tb->d_bnd;
        a.ops = tb->d_ops;
        a.out = tb->d_out;
        void* args[] = {&a};
        SW_CUDA(ctx, cudaLaunchKernel((const void*)sw_traceback_kernel, dim3((m + 3) / 4),
                                      dim3(128), args, 0, st));
        SW_CUDA(ctx, cudaMemcpyAsync(res.data() + h0, tb->d_out, m * sizeof(TbOut),
                                     cudaMemcpyDeviceToHost, st));
        hops.resize(opsb);
        SW_CUDA(ctx, cudaMemcpyAsync(hops.data(), tb->d_ops, opsb, cudaMemcpyDeviceToHost, st));
        SW_CUDA(ctx, cudaStreamSynchronize(st));
        SW_CUDA(ctx, cudaGetLastError());
        // ops were written last first: run-length encode them in alignment order
        for (uint32_t h = h0; h < h1; ++h) {
            const TbOut& r = res[h];
            sw_alignment& al = out[h];
            al.score = r.score;
            al.q_begin = r.q_begin;
            al.q_end = r.q_end;
            al.d_begin = r.d_begin;
            al.d_end = r.d_end;
            al.matches = r.matches;
            al.ops_offset = ops_total;
            const uint8_t* o = hops.data() + jobs[h].ops;
            uint32_t runs = 0;
            for (int64_t x = (int64_t)r.n_ops - 1; x >= 0;) {
                const uint8_t op = o[x];
                uint32_t len = 0;
                while (x >= 0 && o[x] == op) {
                    ++len;
                    --x;
                }
                if (ops && ops_total < ops_cap) ops[ops_total] = (len << 4) | op;
                ++ops_total;
                ++runs;
            }
            al.n_ops = runs;
        }
        h0 = h1;
    }
    *ops_used = ops_total;
    if (ops_total > ops_cap)
        SW_SET(ctx, SW_ERR_UNSUPPORTED, "ops buffer too small: %llu entries needed",
               (unsigned long long)ops_total);
    return SW_OK;
}
