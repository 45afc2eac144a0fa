"""Sharded search on two ranks (gloo, CPU): the residue-balanced split, the
local-to-global index mapping and the k-hit all-gather merge must give the
whole-DB top-k, ties across the shard boundary included.  The oracle stands
in for each rank's device search (no GPU here)."""
import os
import socket

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import oracle
from swhybrid_b200 import param, shard, synth

K = 10


def make_case():
    rng = np.random.default_rng(91)
    db = synth.small_db(92, 900)
    q = synth.residues(rng, 120)
    recs = [db.record(i) for i in range(db.n)]
    # the same homolog at both ends of the DB: equal scores on both shards
    h = synth.mutate(rng, q, 0.15, 0.0)
    for i in (3, 7, db.n - 5, db.n - 2):
        recs[i] = h
    lens = np.array([len(r) for r in recs], dtype=np.int64)
    off = np.zeros(db.n + 1, dtype=np.uint64)
    off[1:] = np.cumsum(lens)
    return np.concatenate(recs).astype(np.uint8), off, q


def worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        res, off, q = make_case()
        b, e = shard.shard_bounds(off, world)[rank]
        lres, loff = shard.local_records(res, off, b, e)
        scores = oracle.search(q, lres, loff, param.blosum62(), 12, 2)
        sc, idx = oracle.topk(scores, K)
        merged = shard.gather_topk(list(zip(sc.tolist(), idx.tolist())), b, K)
        out[rank] = merged
    finally:
        dist.destroy_process_group()


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_rank_merge_equals_whole_db():
    world = 2
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.spawn(worker, args=(world, free_port(), out), nprocs=world, join=True)
        got = dict(out)
    res, off, q = make_case()
    sc, idx = oracle.topk(oracle.search(q, res, off, param.blosum62(), 12, 2), K)
    want = list(zip(sc.tolist(), idx.tolist()))
    assert got[0] == want and got[1] == want
    assert want[0][0] == want[3][0]            # the planted ties made it into the list


def test_shard_bounds_balance_and_cover():
    rng = np.random.default_rng(3)
    lens = rng.integers(0, 2000, size=1000)
    off = np.zeros(1001, dtype=np.int64)
    off[1:] = np.cumsum(lens)
    for world in (1, 2, 3, 8):
        b = shard.shard_bounds(off, world)
        assert b[0][0] == 0 and b[-1][1] == 1000
        assert all(b[i][1] == b[i + 1][0] for i in range(world - 1))
        sizes = [int(off[e] - off[s]) for s, e in b]
        assert max(sizes) - min(sizes) <= 2 * int(lens.max())
    assert shard.shard_bounds(np.zeros(1, dtype=np.int64), 4) == [(0, 0)] * 4


def test_cpp_worker_pool_split_equals_shard_bounds():
    """The C++ WorkerPool (swhybrid_b200/cpp/swb200_worker.hpp) splits by
    residues with the same rule: on a DB sorted longest first, a split by
    record count would give the first device most of the residues."""
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    exe = os.path.join(root, "swhybrid_b200", "cpp", "shard_bounds_test")
    rng = np.random.default_rng(8)
    lens = np.sort(rng.lognormal(5.6, 0.7, size=5000).astype(np.int64) + 1)[::-1]
    cases = [lens, rng.integers(0, 3000, size=777), np.zeros(5, dtype=np.int64),
             np.array([100000] + [1] * 50, dtype=np.int64)]
    for L in cases:
        off = np.zeros(len(L) + 1, dtype=np.int64)
        off[1:] = np.cumsum(L)
        for world in (1, 2, 3, 4, 8):
            out = subprocess.run([exe, str(world)], input=" ".join(map(str, off)),
                                 capture_output=True, text=True, check=True).stdout.split()
            cuts = [int(x) for x in out]
            want = shard.shard_bounds(off, world)
            assert [(cuts[i], cuts[i + 1]) for i in range(world)] == want
    off = np.zeros(len(lens) + 1, dtype=np.int64)
    off[1:] = np.cumsum(lens)
    (b0, e0), (b1, e1) = shard.shard_bounds(off, 2)
    assert abs(int(off[e0] - off[b0]) - int(off[e1] - off[b1])) <= int(lens.max())
    assert e0 < len(lens) // 2          # the long records sit in the first half


class _OracleCtx:
    """Stands in for a device context in the CPU test of bench.py --shard:
    the oracle scores the rank's shard."""

    class _P:
        top_k = K

    params = _P()

    def load_db(self, res, off):
        self.res, self.off = np.asarray(res), np.asarray(off)

    def search(self, q):
        sc, idx = oracle.topk(oracle.search(q, self.res, self.off, param.blosum62(), 12, 2), K)
        return list(zip(sc.tolist(), idx.tolist())), None


def shard_bench_worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        res, off, q = make_case()

        class _DB:
            residues, offsets = res, off
            n = len(off) - 1
            total = int(off[-1])

        args = bench.parse(["--shard", "--steps", "2", "--warmup", "1", "--workload", "small"])
        line, merged = bench.run_shard(args, rank, world, 0, make_ctx=_OracleCtx,
                                       workload=(_DB, [q, q[:50]]))
        out[rank] = (line, merged)
    finally:
        dist.destroy_process_group()


def test_bench_shard_mode_two_ranks_equals_whole_db():
    """bench.py --shard on two gloo ranks: each rank searches its residue-
    balanced slice, one all-gather per query merges the k best hits; the
    merged lists equal the whole-DB top-k and rank 0 reports the line."""
    world = 2
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.spawn(shard_bench_worker, args=(world, free_port(), out), nprocs=world, join=True)
        got = dict(out)
    res, off, q = make_case()
    for qq, i in ((q, 0), (q[:50], 1)):
        sc, idx = oracle.topk(oracle.search(qq, res, off, param.blosum62(), 12, 2), K)
        want = list(zip(sc.tolist(), idx.tolist()))
        assert got[0][1][i] == want and got[1][1][i] == want
    line = got[0][0]
    assert got[1][0] is None
    assert line["scaling"] == "strong" and line["n_gpus"] == 2 and line["value"] > 0
    assert line["config"]["rank0_records"][0] == 0


def bench_main_worker(rank, world, port, out):
    """One rank of bench.py's default (weak-scaling) mode, with run_ours
    stood in for by one max-over-ranks reduction: only rank 0 returns a line."""
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import bench

    def fake_run_ours(args, rank, world, local_rank):
        t = torch.tensor([float(rank)])
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return ({"value": float(t.item())} if rank == 0 else None), None, None, None

    bench.run_ours = fake_run_ours
    out[rank] = bench.main(["--no-cpu-baseline"])


def test_bench_ranks_meet_at_the_end():
    """Every rank of a multi-GPU bench run takes the same collective steps:
    the ranks without a line still join rank 0's final barrier, so no rank
    waits on a peer that has exited (gloo on CPU, two ranks)."""
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        port = free_port()
        procs = [ctx.Process(target=bench_main_worker, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
        hung = [p.is_alive() for p in procs]
        for p in procs:
            if p.is_alive():
                p.kill()
        assert not any(hung)
        assert dict(out) == {0: 0, 1: 0}
