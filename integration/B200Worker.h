/*
 * B200Worker.h -- the reference-side binding of libswb200: a Worker
 * (src/Worker.h:82-249) that scores SWhybrid's DB chunks on a B200 through
 * the C ABI of include/swb200.h.  It compiles against the reference's own
 * headers unchanged and runs under the reference's own driver loop,
 * Worker::launch (src/Worker.cpp:175-200): fill -> packDB -> search ->
 * auxWork, with WorkerPool-style construction and merging
 * (src/WorkerPool.cpp:10-105).  It takes the place of CUDAWorker
 * (src/CUDAWorker.cu:24-246).
 *
 * Per chunk handed out by DataPool::fillChunk (src/DataPool.cpp:171-286):
 *   packDB()  copies the chunk's records (whole 128-wide batches, sequence
 *             major, codes 0..23 with pad code 23 at the tails) out of the
 *             shared read buffer into this entry's own storage, since the
 *             next fill() overwrites that buffer while search() runs;
 *   search()  makes the chunk resident (sw_db_load) and scores every record
 *             (sw_search with all scores) into the entry's score array, so
 *             the base auxWork() pushes them into resultList with the
 *             chunk's base index, as it does for CUDAWorker's scores.
 * Scores are exact and final (SW_FLAG_REFERENCE_CAP: min(score, 65535), as
 * the reference's RecalcWorker reports), so nothing is pushed to
 * RecalcWorker::pushOverflowSeq and its queue stays empty.
 */
#ifndef B200WORKER_H_
#define B200WORKER_H_

#include <vector>
#include <stdint.h>

#include "Worker.h"

struct sw_ctx;

class B200Worker : public Worker {
public:
    /* Same arguments as CUDAWorker::CUDAWorker (src/CUDAWorker.cu:24-45). */
    B200Worker(DataPool* loader, Param* params, RecalcWorker* recalcWorker, int deviceId);
    virtual ~B200Worker();

    virtual void alloc();
    virtual void free();
    virtual void asyncCopy();
    virtual void search();
    virtual void showPerformance();
    virtual void setQuery(const char* query, const size_t qlen);

    /* Chunks scored and records scored by this worker so far. */
    size_t chunksScored() const { return chunks; }
    size_t recordsScored() const { return records; }

protected:
    virtual void packDB();
    virtual void who();

private:
    struct Chunk {
        std::vector<uint8_t> residues;   /* records back to back, codes 0..24 */
        std::vector<uint64_t> offsets;   /* n + 1 */
        std::vector<int> scores;         /* n, pushed by Worker::auxWork */
    };
    void fail(const char* where, int status);

    int deviceId;
    sw_ctx* ctx;
    std::vector<uint8_t> queryCodes;
    Chunk chunk[2];                      /* one per Entry (Worker::entry[2]) */
    size_t chunks, records;
    double kernelMs;
};

#endif /* B200WORKER_H_ */
