// oracle/ref_harness.cpp -- drives SWhybrid's own AVX2 kernels on a flat DB.
//
// TEST INFRASTRUCTURE ONLY (the checker and the timed CPU baseline).  Linked
// by oracle/Makefile with the reference's src/AVXKernel.cpp, compiled from
// the read-only reference tree into oracle/_ref/libswref.so.  Nothing in the
// product path loads it.
//
// The reference's packer (AVXWorker::packDB, src/AVXWorker.cpp:67-302) has a
// broken 32x32 byte transpose and its DB maker corrupts mixed-length batches
// (src/FastaFile.cpp:272-351), so this harness feeds the reference kernels
// from its own packer instead.  Everything downstream of the packer follows
// the reference's call sequence:
//   * batches of 32 equal-length lanes, [column][lane] bytes, tail-padded
//     with code 23 to a multiple of 4 columns (Worker.cpp:108-171 layout with
//     batchSize 32 / packSize 1, AVXWorker.cpp:40);
//   * per-thread profile / qtable set-up as AVXWorker::alloc
//     (AVXWorker.cpp:330-340) and the dup matrix from makeDupMatrix;
//   * avxCompute under `omp parallel` (AVXWorker.cpp:397-419) with
//     gapOE = open+extend, gapE = extend, SCORE_LIMIT_7 = 128 - max(matrix);
//   * flagged lanes de-interleaved as AVXWorker::handleOverflow
//     (AVXWorker.cpp:429-459) and appended as RecalcWorker::pushOverflowSeq
//     does (RecalcWorker.cpp:270-343: codes > 23 -> 23, 4 x 23 appended when
//     the record does not end in 23);
//   * avxCompute16 over contiguous, residue-balanced ranges, one per thread
//     (RecalcWorker.cpp:99-268); the range split is this harness's own
//     (the reference's split is not needed for the scores, which do not
//     depend on how the records are distributed over threads).
#include <stdint.h>
#include <string.h>
#include <stdlib.h>
#include <pthread.h>
#include <omp.h>
#include <mm_malloc.h>
#include <chrono>
#include <vector>
#include <algorithm>
#include <numeric>

#include "AVXKernel.h"

namespace {

struct Packed {
    std::vector<int64_t> order;     // batch lane -> input record
    char *buf = nullptr;            // [batch][column][32 lanes]
    std::vector<int> map;           // [pos, len] per batch
    size_t batches = 0;
    ~Packed() { if (buf) _mm_free(buf); }
};

void pack32(const uint8_t *res, const uint64_t *off, int64_t n, Packed &pk)
{
    pk.order.resize(n);
    std::iota(pk.order.begin(), pk.order.end(), 0);
    std::stable_sort(pk.order.begin(), pk.order.end(), [&](int64_t a, int64_t b) {
        return (off[a + 1] - off[a]) > (off[b + 1] - off[b]);
    });
    pk.batches = (size_t)((n + 31) / 32);
    std::vector<int64_t> blen(pk.batches);
    size_t total = 0;
    for (size_t b = 0; b < pk.batches; ++b) {
        int64_t mx = 0;
        for (int l = 0; l < 32; ++l) {
            int64_t k = (int64_t)b * 32 + l;
            if (k < n) mx = std::max<int64_t>(mx, off[pk.order[k] + 1] - off[pk.order[k]]);
        }
        if (mx == 0) mx = 4;
        blen[b] = (mx + 3) / 4 * 4;
        total += (size_t)blen[b] * 32;
    }
    pk.buf = (char *)_mm_malloc(total + 64, 32);
    memset(pk.buf, 23, total + 64);
    pk.map.resize(pk.batches * 2);
    size_t pos = 0;
    for (size_t b = 0; b < pk.batches; ++b) {
        pk.map[2 * b] = (int)pos;
        pk.map[2 * b + 1] = (int)blen[b];
        for (int l = 0; l < 32; ++l) {
            int64_t k = (int64_t)b * 32 + l;
            if (k >= n) continue;
            const uint8_t *s = res + off[pk.order[k]];
            int64_t len = off[pk.order[k] + 1] - off[pk.order[k]];
            for (int64_t c = 0; c < len; ++c) {
                uint8_t v = s[c];
                pk.buf[pos + (size_t)c * 32 + l] = (char)(v > 23 ? 23 : v);
            }
        }
        pos += (size_t)blen[b] * 32;
    }
}

}  // namespace

extern "C" {

// A DB packed once into the reference kernels' 32-lane batch layout.
struct SwRefDb {
    Packed pk;
    int64_t n = 0;
};

void *swref_db_pack(const uint8_t *res, const uint64_t *off, int64_t n)
{
    SwRefDb *db = new SwRefDb();
    db->n = n;
    if (n > 0) pack32(res, off, n, db->pk);
    return db;
}

void swref_db_free(void *h) { delete (SwRefDb *)h; }

// Scores every record (input order) the way the reference reports them.
// Returns 0 on success.  kernel_seconds receives the wall time of the two
// kernel phases only (packing excluded, as the DB is resident on the GPU side).
int swref_db_search(void *h, const uint8_t *query, int64_t qlen_in,
                    const int32_t *matrix1024, int32_t gap_open,
                    int32_t gap_extend, int32_t threads, int32_t *scores_out,
                    double *kernel_seconds, int64_t *n_overflow)
{
    SwRefDb *db = (SwRefDb *)h;
    const int64_t n = db->n;
    Packed &pk = db->pk;
    if (n <= 0 || qlen_in <= 0) {
        for (int64_t i = 0; i < n; ++i) scores_out[i] = 0;
        if (kernel_seconds) *kernel_seconds = 0.0;
        if (n_overflow) *n_overflow = 0;
        return 0;
    }
    if (threads <= 0) threads = omp_get_max_threads();
    // query padded to a multiple of 8 with 23 (DataPool.cpp:17,330-337)
    int qlen = (int)((qlen_in + 7) / 8 * 8);
    std::vector<char> q(qlen, 23);
    for (int64_t i = 0; i < qlen_in; ++i) q[i] = (char)query[i];
    int plain[1024];
    int hi = 0;
    for (int i = 0; i < 1024; ++i) {
        plain[i] = matrix1024[i];
        hi = std::max(hi, plain[i]);
    }
    const int limit7 = 128 - hi;
    char *dup8 = (char *)_mm_malloc(32 * 64, 32);
    short *dup16 = (short *)_mm_malloc(32 * 64 * sizeof(short), 32);
    makeDupMatrix(dup16, dup8, plain);

    char **g_qtable = (char **)_mm_malloc(sizeof(char *) * (size_t)threads * qlen, 32);
    char *g_profile = (char *)_mm_malloc((size_t)threads * 4096, 32);
    for (int t = 0; t < threads; ++t)
        for (int i = 0; i < qlen; ++i)
            g_qtable[(size_t)t * qlen + i] = g_profile + (size_t)t * 4096 + 4 * 32 * q[i];
    char *externHF = (char *)_mm_malloc(64, 32);

    std::vector<int> result(pk.batches * 32, 0);
    std::vector<int> ovf(pk.batches * 32, 0);
    volatile int overflow_cnt = 0;
    volatile int globalCounter = -1;
    pthread_mutex_t idxMutex, cntMutex;
    pthread_mutex_init(&idxMutex, nullptr);
    pthread_mutex_init(&cntMutex, nullptr);

    auto t0 = std::chrono::steady_clock::now();
#pragma omp parallel num_threads(threads)
    avxCompute(q.data(), qlen, gap_open + gap_extend, gap_extend, dup8, pk.buf,
               pk.map.data(), pk.batches, result.data(), ovf.data(), overflow_cnt,
               globalCounter, idxMutex, cntMutex, limit7, g_profile, g_qtable,
               externHF);

    // --- overflow hand-off (AVXWorker::handleOverflow + pushOverflowSeq) ---
    const int novf = overflow_cnt;
    std::vector<int> lanes(ovf.begin(), ovf.begin() + novf);
    std::sort(lanes.begin(), lanes.end());
    std::vector<char> recalc;
    std::vector<int> vec_pos;
    for (int idx : lanes) {
        int b = idx / 32, ch = idx % 32;
        int pos = pk.map[2 * b], len = pk.map[2 * b + 1];
        vec_pos.push_back((int)recalc.size());
        const char *seq = pk.buf + pos + ch;
        for (int j = 0; j < len; ++j) {
            char v = seq[(size_t)j * 32];
            recalc.push_back(v > 23 ? 23 : v);
        }
        if (recalc.back() != 23)
            for (int j = 0; j < 4; ++j) recalc.push_back(23);
    }
    // slack so that 4-residue reads past a record's terminator stay in bounds
    for (int j = 0; j < 64; ++j) recalc.push_back(23);
    std::vector<int> recalc_result(novf, 0);
    if (novf > 0) {
        short score16[1024];
        for (int i = 0; i < 1024; ++i) score16[i] = (short)plain[i];
        int nt = std::min<int>(threads, (novf + 15) / 16);
        // contiguous ranges holding about the same number of residues
        std::vector<int> start(nt + 1, novf);
        size_t total = recalc.size() - 64;
        start[0] = 0;
        int cur = 1;
        for (int i = 1; i < novf && cur < nt; ++i)
            if ((size_t)vec_pos[i] >= total * cur / nt) start[cur++] = i;
        for (int k = cur; k <= nt; ++k) start[k] = novf;
#pragma omp parallel for num_threads(nt) schedule(static, 1)
        for (int t = 0; t < nt; ++t) {
            int cnt = start[t + 1] - start[t];
            if (cnt > 0)
                avxCompute16(score16, recalc.data(), vec_pos.data(), cnt,
                             recalc_result.data(), start[t], q.data(), (size_t)qlen);
        }
    }
    auto t1 = std::chrono::steady_clock::now();
    if (kernel_seconds) *kernel_seconds = std::chrono::duration<double>(t1 - t0).count();
    if (n_overflow) *n_overflow = novf;

    for (size_t b = 0; b < pk.batches; ++b)
        for (int l = 0; l < 32; ++l) {
            int64_t k = (int64_t)b * 32 + l;
            if (k < n) scores_out[pk.order[k]] = result[b * 32 + l];
        }
    for (int i = 0; i < novf; ++i) {
        int idx = lanes[i];
        int64_t k = idx;  // batch*32 + lane == sorted position
        if (k < n) scores_out[pk.order[k]] = recalc_result[i];
    }

    pthread_mutex_destroy(&idxMutex);
    pthread_mutex_destroy(&cntMutex);
    _mm_free(dup8);
    _mm_free(dup16);
    _mm_free(g_qtable);
    _mm_free(g_profile);
    _mm_free(externHF);
    return 0;
}

int swref_search(const uint8_t *query, int64_t qlen, const uint8_t *res,
                 const uint64_t *off, int64_t n, const int32_t *matrix1024,
                 int32_t gap_open, int32_t gap_extend, int32_t threads,
                 int32_t *scores_out, double *kernel_seconds,
                 int64_t *n_overflow)
{
    void *h = swref_db_pack(res, off, n);
    int rc = swref_db_search(h, query, qlen, matrix1024, gap_open, gap_extend,
                             threads, scores_out, kernel_seconds, n_overflow);
    swref_db_free(h);
    return rc;
}

int swref_max_threads(void) { return omp_get_max_threads(); }

}  // extern "C"
