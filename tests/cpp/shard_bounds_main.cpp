// Reads record offsets (n+1 integers) from stdin and prints the record cuts
// of swb200::shard_bounds for the device count in argv[1]: the CPU check of
// the C++ WorkerPool's residue-balanced split.
#include <cstdio>
#include <cstdlib>

#include "../../swhybrid_b200/cpp/swb200_worker.hpp"

int main(int argc, char** argv) {
    const int n = argc > 1 ? std::atoi(argv[1]) : 1;
    std::vector<uint64_t> off;
    unsigned long long v;
    while (std::scanf("%llu", &v) == 1) off.push_back(v);
    for (size_t c : swb200::shard_bounds(off, n)) std::printf("%zu\n", c);
    return 0;
}
