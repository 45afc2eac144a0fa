// Test driver for the C++ plugin surface (swhybrid_b200/cpp/swb200_worker.hpp):
// parses the reference's switches, reads a FASTA DB or a DB image and a FASTA
// query, runs a WorkerPool of B200Workers and prints "score index" lines of
// the merged top-k (then the titled list as WorkerPool::showResult prints it).
#include <cstdio>
#include <exception>

#include "../../swhybrid_b200/cpp/swb200_worker.hpp"

int main(int argc, char** argv) {
    try {
        swb200::Param params(argc, argv);
        swb200::DataPool pool = swb200::DataPool::open(params.dbPath, params.queryPath);
        swb200::WorkerPool wp(&pool, &params);
        swb200::ResultList<int>& res = wp.run();
        for (const auto& r : res.getResult())
            if (r.score > 0) std::printf("HIT %d %zu\n", r.score, r.idx);
        wp.showResult();
    } catch (const std::exception& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        return 1;
    }
    return 0;
}
