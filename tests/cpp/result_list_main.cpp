// Feeds "score" lines from stdin into swb200::ResultList<int> (k from argv[1])
// in order and prints the list as "score idx" lines: the CPU check of the
// mirror of the reference's ResultList semantics.
#include <cstdio>
#include <cstdlib>

#include "../../swhybrid_b200/cpp/swb200_worker.hpp"

int main(int argc, char** argv) {
    const int k = argc > 1 ? std::atoi(argv[1]) : 10;
    swb200::ResultList<int> list(k);
    int s;
    size_t i = 0;
    while (std::scanf("%d", &s) == 1) list.push(s, i++);
    for (const auto& r : list.getResult()) std::printf("%d %zu\n", r.score, r.idx);
    return 0;
}
