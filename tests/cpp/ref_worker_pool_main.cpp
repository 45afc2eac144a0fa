// Test driver: the reference's own search program (src/main.cpp) with
// WorkerPool's sequence (src/WorkerPool.cpp:10-105) spelled out for B200
// workers only -- Param from argv, DataPool over a DBmaker-made DB,
// RecalcWorker, one B200Worker per device started as a pthread running
// Worker::threadControl -> setQuery -> Worker::launch, join, the recalc pass,
// then the merge of every worker's ResultList followed by RecalcWorker's.
// Prints one line per hit: "hit <score> <layout index> <title>", and exits 1
// when a worker scored nothing.
//
// Usage: ref_worker_pool -q query.fa -db dbprefix -t 10 -g <devices>
#include <cstdio>
#include <string>
#include <vector>

#include "B200Worker.h"
#include "DataPool.h"
#include "Param.h"
#include "RecalcWorker.h"
#include "ResultList.h"

int main(int argc, char* argv[]) {
    Param* param = new Param(argc, argv);   // never deleted, as in src/main.cpp
    DataPool loader(param->topNum, param->queryPath, param->dbPath);
    RecalcWorker* recalc = new RecalcWorker(param);
    recalc->setQuery(loader.getQuery(), loader.getQueryLen());
    const int devices = param->cudaNum > 0 ? param->cudaNum : 1;
    std::vector<B200Worker*> workers;
    for (int i = 0; i < devices; ++i) workers.push_back(new B200Worker(&loader, param, recalc, i));
    for (size_t i = 0; i < workers.size(); ++i) workers[i]->startThread();
    for (size_t i = 0; i < workers.size(); ++i) workers[i]->waitForThread();
    recalc->launch();

    ResultList<int> merged(param->topNum);
    size_t scored = 0;
    for (size_t i = 0; i < workers.size(); ++i) {
        merged.mergeList(workers[i]->getResult());
        scored += workers[i]->recordsScored();
    }
    merged.mergeList(recalc->getResult());
    std::list<Result<int> >& res = merged.getResult();
    for (std::list<Result<int> >::iterator it = res.begin(); it != res.end(); ++it) {
        std::string title;
        if (it->score > 0) loader.getTitle(it->idx, title);
        printf("hit %d %zu %s\n", it->score, it->idx, title.c_str());
    }
    printf("records %zu recalc %zu\n", scored, recalc->getNum());
    for (size_t i = 0; i < workers.size(); ++i) delete workers[i];
    delete recalc;
    return scored > 0 ? 0 : 1;
}
