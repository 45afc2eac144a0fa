/*
 * B200Worker.cpp -- see B200Worker.h.  Built against the reference's headers
 * (Worker.h, DataPool.h, Param.h, RecalcWorker.h, ResultList.h, Defs.h) and
 * linked with libswb200.so.
 */
#include "B200Worker.h"

#include <cstdio>
#include <cstring>
#include <sys/timeb.h>

#include "swb200.h"

namespace {
double now_ms() {
    timeb t;
    ftime(&t);
    return t.time * 1000.0 + t.millitm;
}
}  // namespace

B200Worker::B200Worker(DataPool* loader, Param* params, RecalcWorker* recalcWorker, int deviceId)
    : Worker(loader, params, recalcWorker, /*packSize*/ 1, /*batchSize*/ 1, /*typeSize*/ 1),
      deviceId(deviceId), ctx(NULL), chunks(0), records(0), kernelMs(0.0) {
    /* chunk size asked of DataPool::fillChunk; the read buffer the base
     * class allocates holds maxReaderBufferSize bytes (src/Defs.h:14) */
    bufferSize = maxReaderBufferSize;
}

B200Worker::~B200Worker() {
    if (ctx) sw_ctx_destroy(ctx);
}

void B200Worker::fail(const char* where, int status) {
    static char msg[512];
    snprintf(msg, sizeof msg, "B200Worker(%d): %s failed (status %d): %s\n", deviceId, where,
             status, ctx ? sw_last_error(ctx) : sw_last_error(NULL));
    throw (const char*)msg;   /* caught and printed by Worker::threadControl */
}

/* CUDAWorker::alloc (src/CUDAWorker.cu:53-82): device context and the two
 * entries of the double buffer. */
void B200Worker::alloc() {
    if (!ctx) {
        sw_params p;
        sw_params_default(&p);
        for (int i = 0; i < 32 * 32; ++i) p.matrix[i] = params->plain_matrix[i];
        p.gap_open = params->gapOpen;
        p.gap_extend = params->gapExtend;
        p.top_k = params->topNum;
        p.flags = SW_FLAG_REFERENCE_CAP;
        int st = sw_ctx_create(deviceId, &p, &ctx);
        if (st != SW_OK) {
            ctx = NULL;
            fail("sw_ctx_create", st);
        }
    }
    for (int i = 0; i < 2; ++i) {
        entry[i].setEntry(NULL, NULL, NULL);
        entry[i].setResultSize(0);
        entry[i].setBatchNum(0);
        entry[i].setBaseIdx(0);
    }
    compEntry = entry + 1;
    auxEntry = entry;
}

void B200Worker::free() {
    if (ctx) sw_ctx_destroy(ctx);
    ctx = NULL;
}

/* CUDAWorker::asyncCopy uploads the packed chunk; here search() does. */
void B200Worker::asyncCopy() {}

/* Worker::packDB (src/Worker.cpp:108-171) / CUDAWorker::packDB: the chunk's
 * records leave the shared read buffer for this entry's storage. */
void B200Worker::packDB() {
    Entry* pEntry = entry + !bufFlag;
    Chunk& ch = chunk[pEntry - entry];
    ch.residues.clear();
    ch.offsets.assign(1, 0);
    const char* p = dbSeqBuf;
    for (size_t b = 0; b < infoSize; ++b) {
        const unsigned num = info[b].numSeqs, len = info[b].seqLen;
        for (unsigned i = 0; i < num; ++i) {
            for (unsigned j = 0; j < len; ++j) {
                const int c = (signed char)p[j];
                /* the reference's -1 (unknown letter) and anything above the
                 * pad code score 0: code 24 */
                ch.residues.push_back((uint8_t)((c < 0 || c > 24) ? 24 : c));
            }
            p += len;
            ch.offsets.push_back(ch.residues.size());
        }
    }
    const size_t n = ch.offsets.size() - 1;
    ch.scores.assign(n ? n : 1, 0);
    TotalAminoAcidResidue += ch.residues.size();
    pEntry->setEntry((char*)(ch.residues.empty() ? NULL : &ch.residues[0]), NULL, &ch.scores[0]);
    pEntry->setBatchNum((int)infoSize);
    pEntry->setBaseIdx(fillBaseIndex);
    pEntry->setResultSize((int)n);
}

/* CUDAWorker::search (src/CUDAWorker.cu:224-246): every record of the
 * computed entry's chunk scored into its score array. */
void B200Worker::search() {
    Chunk& ch = chunk[compEntry - entry];
    const size_t n = ch.offsets.size() - 1;
    if (n == 0 || compEntry->getResultSize() == 0) return;
    const double t0 = now_ms();
    int st = sw_db_load(ctx, ch.residues.empty() ? NULL : &ch.residues[0], &ch.offsets[0], n);
    if (st != SW_OK) fail("sw_db_load", st);
    std::vector<sw_hit> hits(params->topNum > 0 ? params->topNum : 1);
    uint32_t nh = 0;
    st = sw_search(ctx, queryCodes.empty() ? NULL : &queryCodes[0], (uint32_t)queryCodes.size(),
                   &hits[0], &nh, &ch.scores[0]);
    if (st != SW_OK) fail("sw_search", st);
    kernelMs += now_ms() - t0;
    ++chunks;
    records += n;
}

/* CUDAWorker::setQuery (src/CUDAWorker.cu:106-113): the codes DataPool::
 * getQuery made (padded with code 23 to a multiple of 8, which scores 0). */
void B200Worker::setQuery(const char* query, const size_t qlen) {
    queryCodes.resize(qlen);
    for (size_t i = 0; i < qlen; ++i) {
        const int c = (signed char)query[i];
        queryCodes[i] = (uint8_t)((c < 0 || c > 24) ? 24 : c);
    }
    this->queryLen = (int)qlen;
}

void B200Worker::showPerformance() {
    const double s = kernelMs * 1e-3;
    printf("B200 %d: %zu chunks, %zu records, %zu residues, %.3f s, GCUPS %.1f\n", deviceId,
           chunks, records, (size_t)TotalAminoAcidResidue, s,
           s > 0 ? (double)queryCodes.size() * (double)TotalAminoAcidResidue / s / 1e9 : 0.0);
}

void B200Worker::who() { printf("B200\n"); }
