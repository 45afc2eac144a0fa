// sw_noalloc.cu -- scoring entry point that allocates no memory.
//
// Some callers cannot call cudaMalloc where they score: a request path that
// must never allocate once it has started (an allocation can block on the
// driver and stall every request queued behind it), or a plug-in living in a
// host process whose device memory is all reserved by that process's own
// allocator.  sw_score_noalloc serves them: the caller passes device inputs
// and a device output, and every byte of scratch the kernel needs comes from
// one file-scope __device__ array that is part of the loaded library image.
// That array (256 warps x 8192 columns x 8 bytes plus a 256-byte header,
// about 16 MiB) is held by every GPU that loads the library until the
// process exits.
//
// The kernel is a variant of the exact 32-bit re-score pass (sw_rescore32,
// sw_aux.cu): one warp per record, anti-diagonal wavefront over 32 lanes x 16
// query rows per pass, int32 arithmetic; the boundary row between query
// passes lives in the warp's slice of the static array instead of the DB's
// boundary buffer.  Records are claimed through a counter that also lives in
// the static array.
#include <climits>
#include <cstdint>
#include <cstring>
#include <mutex>

#include <cuda_runtime.h>

#include "../../include/swb200.h"

namespace {

constexpr int kNaWarps = 256;          // warps of one launch (64 blocks x 4 warps)
constexpr int kNaMaxLen = 8192;        // longest DB record accepted, in residues
constexpr int kNaRows = 16;            // query rows per lane and pass
constexpr int kNaHeader = 32;          // uint2 words before the boundary rows (256 B)
constexpr size_t kScratchWords = (size_t)kNaHeader + (size_t)kNaWarps * kNaMaxLen;

// Word 0: .x = record counter, .y = error flag (a record longer than
// kNaMaxLen was skipped).  Words kNaHeader.. : one boundary row of kNaMaxLen
// (H, F) entries per warp.  Host code must not use this name as an address.
static __device__ __align__(256) uint2 g_noalloc_scratch[kScratchWords];

struct NaArgs {
    const uint8_t* query;
    int qlen;
    const uint8_t* residues;
    const uint64_t* offsets;
    int n;
    int gap_oe;
    int gap_e;
    int cap;
    uint2* scratch;          // device address of g_noalloc_scratch
    int32_t* scores;
    int8_t mat[1024];
};

__global__ void __launch_bounds__(128) sw_score_noalloc_kernel(const NaArgs a) {
    __shared__ int smat[1024];
    for (int i = threadIdx.x; i < 1024; i += blockDim.x) smat[i] = a.mat[i];
    __syncthreads();
    constexpr unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    unsigned int* counter = reinterpret_cast<unsigned int*>(&a.scratch[0].x);
    unsigned int* error = reinterpret_cast<unsigned int*>(&a.scratch[0].y);
    uint2* pb = a.scratch + kNaHeader + (size_t)warp * kNaMaxLen;
    const int rows_per_pass = 32 * kNaRows;
    const int P = (a.qlen + rows_per_pass - 1) / rows_per_pass;
    while (true) {
        int rec = 0;
        if (lane == 0) rec = (int)atomicAdd(counter, 1u);
        rec = __shfl_sync(FULL, rec, 0);
        if (rec >= a.n) break;
        const uint64_t b = a.offsets[rec];
        const uint64_t e = a.offsets[rec + 1];
        const int len = (e <= b) ? 0 : (e - b > (uint64_t)kNaMaxLen) ? kNaMaxLen + 1 : (int)(e - b);
        if (len > kNaMaxLen) {
            if (lane == 0) {
                atomicExch(error, 1u);
                a.scores[rec] = 0;
            }
            continue;
        }
        const uint8_t* seq = a.residues + b;
        int S = 0;
        for (int pass = 0; pass < P; ++pass) {
            int qc[kNaRows], H[kNaRows], E[kNaRows];
#pragma unroll
            for (int k = 0; k < kNaRows; ++k) {
                const int row = pass * rows_per_pass + lane * kNaRows + k;
                qc[k] = (row < a.qlen) ? (int)(a.query[row] & 31) * 32 : 24 * 32;
                H[k] = 0;
                E[k] = 0;
            }
            int out_h = 0, out_f = 0, prev_h = 0, myd = 24;
            for (int s = 0; s < len + 31; ++s) {
                int d_in = __shfl_up_sync(FULL, myd, 1);
                int h_in = __shfl_up_sync(FULL, out_h, 1);
                int f_in = __shfl_up_sync(FULL, out_f, 1);
                if (lane == 0) {
                    d_in = 24;
                    h_in = 0;
                    f_in = 0;
                    if (s < len) {
                        d_in = seq[s] & 31;
                        if (pass > 0) {
                            const uint2 v = pb[s];
                            h_in = (int)v.x;
                            f_in = (int)v.y;
                        }
                    }
                }
                __syncwarp();
                const int c = s - lane;
                if (c >= 0 && c < len) {
                    int diag = prev_h, f = f_in;
#pragma unroll
                    for (int k = 0; k < kNaRows; ++k) {
                        int h = max(diag + smat[qc[k] + d_in], E[k]);
                        h = max(max(h, f), 0);
                        diag = H[k];
                        H[k] = h;
                        S = max(S, h);
                        const int hq = h - a.gap_oe;
                        E[k] = max(E[k] - a.gap_e, hq);
                        f = max(f - a.gap_e, hq);
                    }
                    out_h = H[kNaRows - 1];
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
        if (lane == 0) a.scores[rec] = (a.cap && S > 65535) ? 65535 : S;
        __syncwarp();
    }
}

// Device address of the static scratch, looked up once per device.
std::mutex g_na_mutex;
void* g_na_addr[64] = {nullptr};

}  // namespace

extern "C" sw_status sw_score_noalloc(int device, const sw_params* params, const uint8_t* d_query,
                                      uint32_t qlen, const uint8_t* d_residues,
                                      const uint64_t* d_offsets, uint32_t n_records,
                                      int32_t* d_scores, void* cuda_stream) {
    if (!params || (n_records && (!d_offsets || !d_scores)) || (qlen && !d_query) || device < 0 ||
        device >= 64)
        return SW_ERR_INVALID;
    if (params->gap_open < 0 || params->gap_extend < 0 ||
        params->gap_open + params->gap_extend > 1000)
        return SW_ERR_INVALID;
    for (int i = 0; i < 1024; ++i)
        if (params->matrix[i] < -127 || params->matrix[i] > 127) return SW_ERR_INVALID;
    if (qlen > (1u << 24) || n_records > (uint32_t)INT32_MAX) return SW_ERR_UNSUPPORTED;
    int prev = 0;
    if (cudaGetDevice(&prev) != cudaSuccess) return SW_ERR_CUDA;
    if (cudaSetDevice(device) != cudaSuccess) return SW_ERR_NO_DEVICE;
    cudaStream_t st = (cudaStream_t)cuda_stream;
    sw_status rc = SW_OK;
    do {
        void* addr = nullptr;
        {
            std::lock_guard<std::mutex> lock(g_na_mutex);
            if (!g_na_addr[device]) {
                if (cudaGetSymbolAddress(&g_na_addr[device], g_noalloc_scratch) != cudaSuccess) {
                    g_na_addr[device] = nullptr;
                    rc = SW_ERR_CUDA;
                    break;
                }
            }
            addr = g_na_addr[device];
        }
        if (n_records == 0) break;
        if (qlen == 0) {
            if (cudaMemsetAsync(d_scores, 0, (size_t)n_records * sizeof(int32_t), st) != cudaSuccess)
                rc = SW_ERR_CUDA;
            else if (cudaStreamSynchronize(st) != cudaSuccess)
                rc = SW_ERR_CUDA;
            break;
        }
        NaArgs a;
        a.query = d_query;
        a.qlen = (int)qlen;
        a.residues = d_residues;
        a.offsets = d_offsets;
        a.n = (int)n_records;
        a.gap_oe = params->gap_open + params->gap_extend;
        a.gap_e = params->gap_extend;
        a.cap = (params->flags & SW_FLAG_REFERENCE_CAP) ? 1 : 0;
        a.scratch = (uint2*)addr;
        a.scores = d_scores;
        for (int i = 0; i < 1024; ++i)
            a.mat[i] = (int8_t)(((i >> 5) >= 24 || (i & 31) >= 24) ? 0 : params->matrix[i]);
        // the counter and the error flag must start at zero on every call
        if (cudaMemsetAsync(addr, 0, sizeof(uint2), st) != cudaSuccess) {
            rc = SW_ERR_CUDA;
            break;
        }
        sw_score_noalloc_kernel<<<kNaWarps / 4, 128, 0, st>>>(a);
        if (cudaGetLastError() != cudaSuccess) {
            rc = SW_ERR_CUDA;
            break;
        }
        uint32_t err = 0;
        if (cudaMemcpyAsync(&err, (const char*)addr + sizeof(uint32_t), sizeof(err),
                            cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess) {
            rc = SW_ERR_CUDA;
            break;
        }
        if (err) rc = SW_ERR_UNSUPPORTED;
    } while (0);
    cudaSetDevice(prev);
    return rc;
}
