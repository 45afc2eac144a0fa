// sw_probe.cu -- measures the packed-integer issue rates that bound the
// Smith-Waterman first pass on the present GPU (the roofline denominator).
//
// Each kernel runs only register arithmetic (no memory traffic inside the
// timed loop), at full occupancy, with several independent dependency chains
// per thread:
//   op 0  __viaddmax_s16x2          (fused add + max, 2 x int16)
//   op 1  __vimax3_s16x2            (3-way max, 2 x int16)
//   op 2  prmt.b32                  (byte permute)
//   op 3  a per-row cell recurrence of 5 DPX + 1 PRMT per row and 1
//         three-way max per two rows (earlier form of the first pass)
//   op 4  mad.lo.u32 with a run-time multiplier (IMAD)
//   op 5  __viaddmax_s16x2 and IMAD interleaved 1:1 (do they co-issue?)
//   op 6  three-input integer add (IADD3)
//   op 7  three-input logic op (LOP3)
//   op 8  the first pass's per-row cell recurrence as sw_wavefront.cuh runs
//         it (4 DPX + 1 32-bit add + 1 PRMT per row, 1 three-way max per two rows),
//         without its shared-memory loads and shuffles
//   op 9  __hmax2 (half2 max), op 10 __hadd2, op 11 __hmax2 and
//         __viaddmax_s16x2 interleaved 1:1 (does half2 max use another pipe?)
//   op 12 an 8-bit first pass, four records per register, with CUDA's
//         byte-SIMD functions (__vaddus4, __vsubus4, __vmaxu4): the unsigned
//         saturating cell of the reference's int8 pass (bias added to the
//         profile and subtracted after the diagonal add), 10 byte operations
//         per row and register
//   op 13 the same 8-bit cell built by hand: 7-bit lanes under a guard bit,
//         a byte-wise maximum as a 32-bit subtract (IADD3), a sign-byte
//         broadcast (PRMT) and a select (LOP3), adds as plain 32-bit adds
//   op 14 the paired-query cell of the batched kernel (sw_qpair.cuh): the
//         first pass's mix without the PRMT (profile words arrive packed)
// Rates are returned in lane-operations per second (ops 0-2, 4-7; a 16x2
// operation counts as two) and in cell updates per second (ops 3, 8, 14: two
// cells per row and register; ops 12, 13: four).
#include <cstdint>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

namespace {

__device__ __forceinline__ uint32_t prmt(uint32_t a, uint32_t b, uint32_t sel) {
    uint32_t r;
    asm volatile("prmt.b32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(sel));
    return r;
}

__device__ __forceinline__ uint32_t mad(uint32_t a, uint32_t b, uint32_t c) {
    uint32_t r;
    asm volatile("mad.lo.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(c));
    return r;
}

template <int OP>
__global__ void __launch_bounds__(512) rate_kernel(uint32_t* sink, int iters, uint32_t seed) {
    uint32_t a[8];
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
#pragma unroll
    for (int j = 0; j < 8; ++j) a[j] = (tid * 2654435761u) ^ (seed + 97u * j);
    uint32_t b = seed | 0x00010001u, c = seed ^ 0x80008000u;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            if (OP == 0) a[j] = __viaddmax_s16x2(a[j], b, a[j ^ 1]);
            if (OP == 1) a[j] = __vimax3_s16x2(a[j], b, a[j ^ 1]);
            if (OP == 2) a[j] = prmt(a[j], a[j ^ 1], 0xC480u + (uint32_t)j);
            if (OP == 4) a[j] = mad(a[j], c, a[j ^ 1]);
            if (OP == 5) a[j] = (j & 1) ? mad(a[j], c, a[j ^ 1]) : __viaddmax_s16x2(a[j], b, a[j ^ 1]);
            if (OP == 6) {
                uint32_t r;
                asm volatile("add.u32 %0, %1, %2;\n\tadd.u32 %0, %0, %3;" : "=r"(r) : "r"(a[j]), "r"(a[j ^ 1]), "r"(b));
                a[j] = r;
            }
            if (OP == 7) a[j] = (a[j] & a[j ^ 1]) ^ b;
            if (OP == 9 || OP == 10 || (OP == 11 && (j & 1))) {
                __half2 x = *reinterpret_cast<__half2*>(&a[j]);
                __half2 y = *reinterpret_cast<__half2*>(&a[j ^ 1]);
                __half2 r = (OP == 10) ? __hadd2(x, y) : __hmax2(x, y);
                a[j] = *reinterpret_cast<uint32_t*>(&r);
            }
            if (OP == 11 && !(j & 1)) a[j] = __viaddmax_s16x2(a[j], b, a[j ^ 1]);
        }
        b += c;
    }
    uint32_t r = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) r ^= a[j];
    if (r == 0x9e3779b9u) sink[0] = r;
}

// 16 rows of the first-pass recurrence per iteration, profile words taken
// from registers.
__global__ void __launch_bounds__(512) cell_kernel(uint32_t* sink, int iters, uint32_t seed) {
    constexpr int R = 16;
    uint32_t H[R], E[R];
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
#pragma unroll
    for (int k = 0; k < R; ++k) {
        H[k] = (tid + k) & 0x000f000fu;
        E[k] = 0u;
    }
    uint32_t S = 0, f = 0, diag = 0;
    uint32_t A0 = seed ^ tid, A1 = seed * 3u, B0 = seed + tid, B1 = ~seed;
    const uint32_t NOE = 0xfff4fff4u, NE = 0xfffefffeu, MIN16 = 0x80008000u;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < R; ++k) {
            const uint32_t wa = (k & 4) ? A1 : A0, wb = (k & 4) ? B1 : B0;
            const uint32_t sel = (uint32_t)(k & 3) | ((uint32_t)((k & 3) | 8) << 4) |
                                 ((uint32_t)(4 + (k & 3)) << 8) |
                                 ((uint32_t)((4 + (k & 3)) | 8) << 12);
            const uint32_t sc = prmt(wa, wb, sel);
            uint32_t h = __viaddmax_s16x2_relu(diag, sc, E[k]);
            h = __vimax_s16x2_relu(h, f);
            diag = H[k];
            H[k] = h;
            const uint32_t hq = __viaddmax_s16x2(h, NOE, MIN16);
            E[k] = __viaddmax_s16x2(E[k], NE, hq);
            f = __viaddmax_s16x2(f, NE, hq);
            if (k & 1) S = __vimax3_s16x2(S, H[k - 1], H[k]);
        }
        A0 = A0 * 1664525u + 1013904223u;
        B0 ^= A0;
        f = 0;
        diag = S & 0x00ff00ffu;
    }
    uint32_t r = S;
#pragma unroll
    for (int k = 0; k < R; ++k) r ^= H[k] ^ E[k];
    if (r == 0x9e3779b9u) sink[0] = r;
}

// The first pass's cell recurrence with biased lanes (sw_wavefront.cuh rows8).
__global__ void __launch_bounds__(512) cell2_kernel(uint32_t* sink, int iters, uint32_t seed) {
    constexpr int R = 16;
    uint32_t H[R], E[R];
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t Z = 0x000c000cu, NQ = 0u - Z, NE = 0xfffefffeu;
#pragma unroll
    for (int k = 0; k < R; ++k) {
        H[k] = Z + ((tid + k) & 0x000f000fu);
        E[k] = Z;
    }
    uint32_t S = Z, f = Z, diag = Z;
    uint32_t A0 = seed ^ tid, A1 = seed * 3u, B0 = seed + tid, B1 = ~seed;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < R; ++k) {
            const uint32_t wa = (k & 4) ? A1 : A0, wb = (k & 4) ? B1 : B0;
            const uint32_t sel = (uint32_t)(k & 3) | ((uint32_t)((k & 3) | 8) << 4) |
                                 ((uint32_t)(4 + (k & 3)) << 8) |
                                 ((uint32_t)((4 + (k & 3)) | 8) << 12);
            const uint32_t sc = prmt(wa, wb, sel);
            uint32_t h = __viaddmax_s16x2(diag, sc, E[k]);
            h = __vimax3_s16x2(h, f, Z);
            diag = H[k];
            H[k] = h;
            const uint32_t hq = h + NQ;
            E[k] = __viaddmax_s16x2(E[k], NE, hq);
            f = __viaddmax_s16x2(f, NE, hq);
            if (k & 1) S = __vimax3_s16x2(S, H[k - 1], H[k]);
        }
        A0 = A0 * 1664525u + 1013904223u;
        B0 ^= A0;
        f = Z;
        diag = (S & 0x00ff00ffu) | Z;
    }
    uint32_t r = S;
#pragma unroll
    for (int k = 0; k < R; ++k) r ^= H[k] ^ E[k];
    if (r == 0x9e3779b9u) sink[0] = r;
}

// 8-bit first pass from CUDA's byte-SIMD functions: unsigned saturating
// lanes, score 0 = byte 0, profile bytes biased by +4 (so a negative score
// is an unsigned add of a small value followed by a saturating subtract).
__global__ void __launch_bounds__(512) cell8_intrin_kernel(uint32_t* sink, int iters,
                                                           uint32_t seed) {
    constexpr int R = 16;
    uint32_t H[R], E[R];
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t BIAS = 0x04040404u, Q = 0x0c0c0c0cu, EXT = 0x02020202u;
#pragma unroll
    for (int k = 0; k < R; ++k) {
        H[k] = (tid + k) & 0x0f0f0f0fu;
        E[k] = 0u;
    }
    uint32_t S = 0, f = 0, diag = 0;
    uint32_t A0 = seed ^ tid, A1 = seed * 3u, B0 = seed + tid, B1 = ~seed;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < R; ++k) {
            const uint32_t wa = (k & 4) ? A1 : A0, wb = (k & 4) ? B1 : B0;
            const uint32_t sc = prmt(wa, wb, 0x5140u + (uint32_t)(k & 3) * 0x1111u) & 0x0f0f0f0fu;
            uint32_t h = __vsubus4(__vaddus4(diag, sc), BIAS);
            h = __vmaxu4(__vmaxu4(h, E[k]), f);
            diag = H[k];
            H[k] = h;
            S = __vmaxu4(S, h);
            const uint32_t hq = __vsubus4(h, Q);
            E[k] = __vmaxu4(__vsubus4(E[k], EXT), hq);
            f = __vmaxu4(__vsubus4(f, EXT), hq);
        }
        A0 = A0 * 1664525u + 1013904223u;
        B0 ^= A0;
        f = 0;
        diag = S & 0x07070707u;
    }
    uint32_t r = S;
#pragma unroll
    for (int k = 0; k < R; ++k) r ^= H[k] ^ E[k];
    if (r == 0x9e3779b9u) sink[0] = r;
}

// Byte-wise maximum of 7-bit lanes (bit 7 of every byte clear): a + 128 - b
// per byte cannot borrow across bytes, its bit 7 says a >= b, PRMT's
// sign-replicating selector turns that bit into a byte mask, LOP3 selects.
__device__ __forceinline__ uint32_t max7x4(uint32_t a, uint32_t b) {
    const uint32_t d = a + 0x80808080u - b;
    const uint32_t m = prmt(d, d, 0xBA98u);
    return (a & m) | (b & ~m);
}

// 8-bit first pass built by hand: lanes hold value + 12 in 7 bits (exact
// while a score stays below 128 - 12 - max(matrix), flagged above, as the
// reference flags at 128 - max(matrix)); adds and the open/extend
// subtractions are plain 32-bit adds of biased lanes.
__global__ void __launch_bounds__(512) cell8_swar_kernel(uint32_t* sink, int iters,
                                                         uint32_t seed) {
    constexpr int R = 16;
    uint32_t H[R], E[R];
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t Z = 0x0c0c0c0cu, NQ = 0u - Z, NE = 0u - 0x02020202u;
#pragma unroll
    for (int k = 0; k < R; ++k) {
        H[k] = Z + ((tid + k) & 0x0f0f0f0fu);
        E[k] = Z;
    }
    uint32_t S = Z, f = Z, diag = Z;
    uint32_t A0 = seed ^ tid, A1 = seed * 3u, B0 = seed + tid, B1 = ~seed;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < R; ++k) {
            const uint32_t wa = (k & 4) ? A1 : A0, wb = (k & 4) ? B1 : B0;
            const uint32_t sc = prmt(wa, wb, 0x5140u + (uint32_t)(k & 3) * 0x1111u) & 0x07070707u;
            uint32_t h = max7x4(diag + sc, E[k]);
            h = max7x4(max7x4(h, f), Z);
            diag = H[k];
            H[k] = h;
            const uint32_t hq = h + NQ;
            E[k] = max7x4(E[k] + NE, hq) & 0x7f7f7f7fu;
            f = max7x4(f + NE, hq) & 0x7f7f7f7fu;
            if (k & 1) S = max7x4(S, max7x4(H[k - 1], H[k]));
        }
        A0 = A0 * 1664525u + 1013904223u;
        B0 ^= A0;
        f = Z;
        diag = (S & 0x03030303u) | Z;
    }
    uint32_t r = S;
#pragma unroll
    for (int k = 0; k < R; ++k) r ^= H[k] ^ E[k];
    if (r == 0x9e3779b9u) sink[0] = r;
}

// The paired-query cell (two queries against one record, profile words
// already packed): cell2_kernel's mix without the PRMT.
__global__ void __launch_bounds__(512) cell_pair_kernel(uint32_t* sink, int iters, uint32_t seed) {
    constexpr int R = 16;
    uint32_t H[R], E[R];
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t Z = 0x000c000cu, NQ = 0u - Z, NE = 0xfffefffeu;
#pragma unroll
    for (int k = 0; k < R; ++k) {
        H[k] = Z + ((tid + k) & 0x000f000fu);
        E[k] = Z;
    }
    uint32_t S = Z, f = Z, diag = Z;
    uint32_t W[4] = {(seed ^ tid) & 0x00070007u, (seed * 3u) & 0x00070007u,
                     (seed + tid) & 0x00070007u, (~seed) & 0x00070007u};
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < R; ++k) {
            uint32_t h = __viaddmax_s16x2(diag, W[k & 3], E[k]);
            h = __vimax3_s16x2(h, f, Z);
            diag = H[k];
            H[k] = h;
            const uint32_t hq = h + NQ;
            E[k] = __viaddmax_s16x2(E[k], NE, hq);
            f = __viaddmax_s16x2(f, NE, hq);
            if (k & 1) S = __vimax3_s16x2(S, H[k - 1], H[k]);
        }
        W[i & 3] = (W[i & 3] * 1664525u + 1013904223u) & 0x00070007u;
        f = Z;
        diag = (S & 0x00ff00ffu) | Z;
    }
    uint32_t r = S;
#pragma unroll
    for (int k = 0; k < R; ++k) r ^= H[k] ^ E[k];
    if (r == 0x9e3779b9u) sink[0] = r;
}

template <typename K>
double time_kernel(K kern, int sms, int iters, uint32_t* sink, double work_per_thread) {
    const int blocks = sms * 4, threads = 512;
    kern<<<blocks, threads>>>(sink, iters / 8, 12345u);  // warm-up
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0);
    kern<<<blocks, threads>>>(sink, iters, 777u);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (cudaGetLastError() != cudaSuccess || ms <= 0.f) return -1.0;
    return (double)blocks * threads * work_per_thread * iters / (ms * 1e-3);
}

}  // namespace

// out[0..8] = rates of ops 0..8 (see the file comment); out[9] = SM count;
// out[10] = SM clock in MHz reported by the device attribute; out[11..13] =
// rates of ops 9..11; out[14..16] = rates of ops 12..14 (out holds at least
// 17 entries).  Returns 0 on success.
extern "C" int swprobe_rates(int device, double* out, int iters) {
    if (cudaSetDevice(device) != cudaSuccess) return 1;
    int sms = 0, clk = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    cudaDeviceGetAttribute(&clk, cudaDevAttrClockRate, device);
    uint32_t* sink = nullptr;
    if (cudaMalloc(&sink, 64) != cudaSuccess) return 2;
    if (iters <= 0) iters = 4096;
    out[0] = time_kernel(rate_kernel<0>, sms, iters, sink, 8.0 * 2);
    out[1] = time_kernel(rate_kernel<1>, sms, iters, sink, 8.0 * 2);
    out[2] = time_kernel(rate_kernel<2>, sms, iters, sink, 8.0);
    out[3] = time_kernel(cell_kernel, sms, iters / 4, sink, 16.0 * 2);
    out[4] = time_kernel(rate_kernel<4>, sms, iters, sink, 8.0);
    out[5] = time_kernel(rate_kernel<5>, sms, iters, sink, 8.0);
    out[6] = time_kernel(rate_kernel<6>, sms, iters, sink, 16.0);
    out[7] = time_kernel(rate_kernel<7>, sms, iters, sink, 8.0);
    out[8] = time_kernel(cell2_kernel, sms, iters / 4, sink, 16.0 * 2);
    out[9] = sms;
    out[10] = clk / 1000.0;
    out[11] = time_kernel(rate_kernel<9>, sms, iters, sink, 16.0);
    out[12] = time_kernel(rate_kernel<10>, sms, iters, sink, 16.0);
    out[13] = time_kernel(rate_kernel<11>, sms, iters, sink, 16.0);
    out[14] = time_kernel(cell8_intrin_kernel, sms, iters / 4, sink, 16.0 * 4);
    out[15] = time_kernel(cell8_swar_kernel, sms, iters / 4, sink, 16.0 * 4);
    out[16] = time_kernel(cell_pair_kernel, sms, iters / 4, sink, 16.0 * 2);
    cudaFree(sink);
    return cudaGetLastError() == cudaSuccess ? 0 : 3;
}
