// swb200_worker.hpp -- the reference's plugin surface, B200 edition.
//
// C++ host classes with the names, members and semantics of SWhybrid's
// Param (src/Param.h:57-167), Result / ResultList (src/ResultList.h:8-93),
// Worker (src/Worker.h:82-249) and WorkerPool (src/WorkerPool.h:41-58),
// written for this library: the GPU worker, B200Worker, replaces CUDAWorker
// (src/CUDAWorker.h:10-77) and talks to libswb200.so through the C ABI in
// include/swb200.h.  Header-only; link with -lswb200 -lpthread.
#pragma once

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <list>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>
#include <chrono>

#include "../../include/swb200.h"

namespace swb200 {

// ---------------------------------------------------------------------------
// Param: search parameters (src/Param.h:59-117).  Switches: -o gap open,
// -e gap extend, -t top-k, -g GPU count, -q query path, -db DB path.
// ---------------------------------------------------------------------------
class Param {
public:
    Param(int argc, char** argv) {
        sw_params p;
        sw_params_default(&p);
        for (int i = 0; i < 32; ++i)
            for (int j = 0; j < 32; ++j) {
                matrix[i][j] = p.matrix[i * 32 + j];
                plain_matrix[i * 32 + j] = p.matrix[i * 32 + j];
            }
        for (int i = 1; i + 1 < argc; ++i) {
            if (argv[i][0] != '-') continue;
            switch (argv[i][1]) {
                case 'o': gapOpen = std::atoi(argv[++i]); break;
                case 'e': gapExtend = std::atoi(argv[++i]); break;
                case 't': topNum = std::atoi(argv[++i]); break;
                case 'g': cudaNum = std::atoi(argv[++i]); break;
                case 'q': queryPath = argv[++i]; break;
                case 'm': {   // scoring matrix: "blosum62" or a matrix file
                    if (sw_params_load_matrix(&p, argv[++i]) != SW_OK)
                        throw std::invalid_argument(std::string("-m: ") + sw_last_error(nullptr));
                    for (int r = 0; r < 32; ++r)
                        for (int c = 0; c < 32; ++c) {
                            matrix[r][c] = p.matrix[r * 32 + c];
                            plain_matrix[r * 32 + c] = p.matrix[r * 32 + c];
                        }
                    break;
                }
                case 'd':
                    if (argv[i][2] == 'b') dbPath = argv[++i];
                    break;
                default: throw std::invalid_argument(std::string("unknown switch ") + argv[i]);
            }
        }
        gapOE = gapOpen + gapExtend;
    }
    sw_params to_sw() const {
        sw_params p;
        sw_params_default(&p);
        std::memcpy(p.matrix, plain_matrix, sizeof(plain_matrix));
        p.gap_open = gapOpen;
        p.gap_extend = gapExtend;
        p.top_k = topNum;
        return p;
    }
    int gapOpen = 10, gapExtend = 2, gapOE = 12, topNum = 10, cudaNum = 1;
    std::string queryPath, dbPath;
    int matrix[32][32];
    int plain_matrix[32 * 32];
};

// ---------------------------------------------------------------------------
// Result / ResultList (src/ResultList.h): a top-k list pre-filled with (0, 0);
// push rejects score <= bottom and inserts before the first strictly smaller
// entry, so among equal scores the earlier push ranks first.
// ---------------------------------------------------------------------------
template <class T>
struct Result {
    Result() : score(0), idx(0) {}
    Result(T s, size_t i) : score(s), idx(i) {}
    T score;
    size_t idx;
};

template <class T>
class ResultList {
public:
    explicit ResultList(size_t n) : _size(n), _bottom(0), _results(n) {}
    std::list<Result<T> >& getResult() { return _results; }
    void push(T* in, size_t sz, size_t base) {
        for (size_t i = 0; i < sz; ++i)
            if (in[i] > _bottom) push(in[i], base + i);
    }
    void mergeList(ResultList<T>& other) {
        for (const Result<T>& r : other.getResult()) push(r.score, r.idx);
    }
    void push(T score, size_t idx) {
        if (score <= _bottom) return;
        if (_results.empty()) {
            _results.push_back(Result<T>(score, idx));
            return;
        }
        for (auto it = _results.begin(); it != _results.end(); ++it)
            if (it->score < score) {
                _results.insert(it, Result<T>(score, idx));
                break;
            }
        _results.pop_back();
        _bottom = _results.back().score;
    }
    void print() const {
        for (const Result<T>& r : _results) std::printf("score %d id %zu\n", (int)r.score, r.idx);
    }

private:
    size_t _size;
    T _bottom;
    std::list<Result<T> > _results;
};

// ---------------------------------------------------------------------------
// DataPool: the records and the query, as residue codes.  Replaces the
// reference's .seq/.map/.title reader (src/DataPool.cpp): records are held in
// input (FASTA) order; getTitle(idx) is the record's header line.
// ---------------------------------------------------------------------------
class DataPool {
public:
    static DataPool from_fasta(const std::string& dbPath, const std::string& queryPath) {
        DataPool d;
        d.read_fasta(dbPath, &d.titles, &d.residues, &d.offsets);
        std::vector<std::string> qt;
        std::vector<uint8_t> q;
        std::vector<uint64_t> qo;
        d.read_fasta(queryPath, &qt, &q, &qo);
        if (qo.size() < 2) throw std::runtime_error("no query record in " + queryPath);
        d.query.assign(q.begin() + qo[0], q.begin() + qo[1]);
        return d;
    }
    // The records and titles of a DB image (sw_fasta_to_image), the query from FASTA.
    static DataPool from_image(const std::string& imagePath, const std::string& queryPath) {
        DataPool d;
        sw_image_view v;
        if (sw_image_open(imagePath.c_str(), 1, &v) != SW_OK)
            throw std::runtime_error(std::string("DB image: ") + sw_last_error(nullptr));
        d.residues.assign(v.residues, v.residues + v.n_residues);
        d.offsets.assign(v.offsets, v.offsets + v.n_records + 1);
        d.titles.reserve(v.n_records);
        for (uint64_t i = 0; i < v.n_records; ++i)
            d.titles.emplace_back(v.titles + v.title_offsets[i],
                                  v.title_offsets[i + 1] - v.title_offsets[i]);
        sw_image_close(&v);
        std::vector<std::string> qt;
        std::vector<uint8_t> q;
        std::vector<uint64_t> qo;
        d.read_fasta(queryPath, &qt, &q, &qo);
        if (qo.size() < 2) throw std::runtime_error("no query record in " + queryPath);
        d.query.assign(q.begin() + qo[0], q.begin() + qo[1]);
        return d;
    }
    // An image when the file is one, else FASTA.
    static DataPool open(const std::string& dbPath, const std::string& queryPath) {
        sw_image_info info;
        if (sw_image_get_info(dbPath.c_str(), 0, &info) == SW_OK) return from_image(dbPath, queryPath);
        return from_fasta(dbPath, queryPath);
    }
    const uint8_t* getQuery() const { return query.data(); }
    size_t getQueryLen() const { return query.size(); }
    size_t getTotalResidue() const { return residues.size(); }
    const char* getTitle(size_t idx) const { return idx < titles.size() ? titles[idx].c_str() : ""; }

    std::vector<uint8_t> residues;     // codes 0..24, records back to back
    std::vector<uint64_t> offsets;     // n + 1
    std::vector<std::string> titles;
    std::vector<uint8_t> query;

private:
    static void read_fasta(const std::string& path, std::vector<std::string>* titles,
                           std::vector<uint8_t>* res, std::vector<uint64_t>* off) {
        FILE* f = std::fopen(path.c_str(), "r");
        if (!f) throw std::runtime_error("cannot open " + path);
        off->clear();
        char line[1 << 16];
        std::string seq;
        auto flush = [&]() {
            if (titles->size() > off->size()) {
                off->push_back(res->size());
                const size_t at = res->size();
                res->resize(at + seq.size());
                sw_encode(seq.data(), seq.size(), res->data() + at);
                seq.clear();
            }
        };
        while (std::fgets(line, sizeof(line), f)) {
            size_t n = std::strlen(line);
            while (n && (line[n - 1] == '\n' || line[n - 1] == '\r')) line[--n] = 0;
            if (line[0] == '>') {
                flush();
                titles->push_back(std::string(line));
            } else {
                seq.append(line, n);
            }
        }
        flush();
        off->push_back(res->size());
        std::fclose(f);
    }
};

// ---------------------------------------------------------------------------
// Worker (src/Worker.h:82-249): the abstract back end.  launch() drives
// alloc -> search -> free and times the computation.
// ---------------------------------------------------------------------------
class Worker {
public:
    Worker(DataPool* loader, Param* params) : loader(loader), params(params),
                                              resultList(params->topNum) {}
    virtual ~Worker() {}
    void launch() {
        alloc();
        setQuery(loader->getQuery(), loader->getQueryLen());
        start = std::chrono::steady_clock::now();
        search();
        stop = std::chrono::steady_clock::now();
        showPerformance();
        free();
    }
    virtual void alloc() {}
    virtual void free() {}
    virtual void asyncCopy() {}
    virtual void search() = 0;
    virtual void setQuery(const uint8_t* q, size_t qlen) { query.assign(q, q + qlen); }
    virtual void showPerformance() {}
    virtual void who() {}
    ResultList<int>& getResult() { return resultList; }
    double getStartTime() const { return std::chrono::duration<double>(start.time_since_epoch()).count(); }
    double getStopTime() const { return std::chrono::duration<double>(stop.time_since_epoch()).count(); }
    size_t getResidueCount() const { return loader->getTotalResidue(); }

protected:
    DataPool* loader;
    Param* params;
    ResultList<int> resultList;
    std::vector<uint8_t> query;
    std::chrono::steady_clock::time_point start, stop;
};

// ---------------------------------------------------------------------------
// B200Worker: replaces CUDAWorker.  alloc() creates the context and makes
// the DB resident (once), search() scores every record and pushes the top-k
// into the ResultList; overflowed records are already exact (no RecalcWorker).
// ---------------------------------------------------------------------------
class B200Worker : public Worker {
public:
    B200Worker(DataPool* loader, Param* params, int deviceId)
        : Worker(loader, params), dev(deviceId) {}
    ~B200Worker() override {
        if (ctx) sw_ctx_destroy(ctx);
    }
    void alloc() override {
        if (ctx) return;
        const sw_params p = params->to_sw();
        check(sw_ctx_create(dev, &p, &ctx), "sw_ctx_create");
        check(sw_db_load(ctx, loader->residues.data(), loader->offsets.data(),
                         loader->offsets.size() - 1), "sw_db_load");
    }
    void search() override {
        std::vector<sw_hit> hits(params->topNum);
        uint32_t n = 0;
        check(sw_search(ctx, query.data(), (uint32_t)query.size(), hits.data(), &n, nullptr),
              "sw_search");
        for (uint32_t i = 0; i < n; ++i) resultList.push(hits[i].score, (size_t)hits[i].index);
    }
    void showPerformance() override {
        sw_run_stats st;
        sw_get_run_stats(ctx, &st);
        std::printf("B200 %d: %.3f ms device, %.1f GCUPS\n", dev, st.kernel_ms,
                    st.kernel_ms > 0 ? st.cells / (st.kernel_ms * 1e6) : 0.0);
    }
    void who() override { std::printf("B200\n"); }

private:
    void check(sw_status s, const char* what) {
        if (s != SW_OK)
            throw std::runtime_error(std::string(what) + ": " + (ctx ? sw_last_error(ctx) : "") +
                                     " (status " + std::to_string((int)s) + ")");
    }
    int dev;
    sw_ctx* ctx = nullptr;
};

// ---------------------------------------------------------------------------
// Residue-balanced split of one DB over n devices: contiguous record ranges
// [cut[g], cut[g+1]) with about the same number of residues each.  Cut g is
// the first record whose start offset reaches g/n of the residues (the rule
// of shard_bounds in swhybrid_b200/shard.py), never before the previous cut.
// ---------------------------------------------------------------------------
inline std::vector<size_t> shard_bounds(const std::vector<uint64_t>& offsets, int n) {
    const size_t nrec = offsets.empty() ? 0 : offsets.size() - 1;
    std::vector<size_t> cuts(1, 0);
    if (n < 1) n = 1;
    const uint64_t base = nrec ? offsets[0] : 0, total = nrec ? offsets[nrec] - base : 0;
    for (int g = 1; g < n; ++g) {
        const uint64_t target = base + (uint64_t)((unsigned __int128)total * g / n);
        size_t c = (size_t)(std::lower_bound(offsets.begin(), offsets.end(), target) -
                            offsets.begin());
        c = std::min(std::max(c, cuts.back()), nrec);
        cuts.push_back(c);
    }
    cuts.push_back(nrec);
    return cuts;
}

// ---------------------------------------------------------------------------
// WorkerPool (src/WorkerPool.cpp:10-155): one B200Worker per GPU, each on its
// own thread, over a residue-balanced slice of the records; results merged
// into one list.
// ---------------------------------------------------------------------------
class WorkerPool {
public:
    WorkerPool(DataPool* loader, Param* params) : loader(loader), params(params),
                                                  resultList(params->topNum) {
        const int n = std::max(1, params->cudaNum);
        const std::vector<size_t> cuts = shard_bounds(loader->offsets, n);
        for (int g = 0; g < n; ++g) {
            // records [b, e) of the input order go to GPU g
            const size_t b = cuts[g], e = cuts[g + 1];
            DataPool* part = new DataPool();
            part->query = loader->query;
            part->offsets.assign(1, 0);
            for (size_t i = b; i < e; ++i) {
                part->residues.insert(part->residues.end(),
                                      loader->residues.begin() + loader->offsets[i],
                                      loader->residues.begin() + loader->offsets[i + 1]);
                part->offsets.push_back(part->residues.size());
            }
            parts.push_back(part);
            bases.push_back(b);
            workers.push_back(new B200Worker(part, params, g));
        }
    }
    ~WorkerPool() {
        for (Worker* w : workers) delete w;
        for (DataPool* p : parts) delete p;
    }
    // Runs every worker on its own thread, then merges the lists in worker
    // order (WorkerPool::getResult, src/WorkerPool.cpp:99-105).
    ResultList<int>& run() {
        std::vector<std::thread> th;
        std::vector<std::string> errors(workers.size());
        for (size_t i = 0; i < workers.size(); ++i)
            th.emplace_back([this, i, &errors]() {
                try {
                    workers[i]->launch();
                } catch (const std::exception& e) {
                    errors[i] = e.what();
                }
            });
        for (std::thread& t : th) t.join();
        for (size_t i = 0; i < workers.size(); ++i) {
            if (!errors[i].empty()) throw std::runtime_error(errors[i]);
            for (const Result<int>& r : workers[i]->getResult().getResult())
                if (r.score > 0) resultList.push(r.score, bases[i] + r.idx);
        }
        return resultList;
    }
    void showResult() {
        std::printf("----------------top %d scores---------------\n", params->topNum);
        for (const Result<int>& r : resultList.getResult())
            std::printf("score %d -- %s\n", r.score, loader->getTitle(r.idx));
        std::printf("--------------------------------------------\n");
    }

private:
    DataPool* loader;
    Param* params;
    ResultList<int> resultList;
    std::vector<Worker*> workers;
    std::vector<DataPool*> parts;
    std::vector<size_t> bases;
};

}  // namespace swb200
