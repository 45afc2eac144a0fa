"""Serving (sw_serve_*): every served request's hits must equal the plain
per-query search of the same query, whether it ran alone, in a mix admitted
together, or joined the ring while other requests were in flight; and the
golden vectors' top-k (including the saturating records that take the
32-bit re-score) must come out of the served path unchanged."""
import os
import time

import numpy as np
import pytest

import oracle
from swhybrid_b200 import capi, synth

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


def load(name):
    z = np.load(os.path.join(GOLD, name + ".npz"))
    qo = z["qoffsets"].astype(np.int64)
    queries = [z["queries"][qo[i]:qo[i + 1]] for i in range(len(qo) - 1)]
    return z["residues"], z["offsets"], queries, z["scores"]


def drain(ctx, n, timeout_s=120.0):
    out = {}
    t_end = time.time() + timeout_s
    while len(out) < n and time.time() < t_end:
        for r in ctx.serve_poll(64, timeout_ms=200):
            out[r["id"]] = r
    assert len(out) == n, f"{len(out)} of {n} requests completed"
    return out


@pytest.fixture(scope="module")
def mixed():
    rng = np.random.default_rng(77)
    db = synth.small_db(21, 4000)
    qs = [synth.residues(rng, int(L)) for L in
          (7, 30, 64, 144, 375, 511, 700, 1200, 2048, 3000, 4100, 6000, 8192)]
    db, _ = synth.plant_homologs(rng, db, qs[6], 0.01)
    db, _ = synth.plant_homologs(rng, db, qs[2], 0.01)
    return db, qs


@pytest.mark.parametrize("opts", [{}, {"pair_long": False}, {"pair_rows": 0}])
def test_served_alone_and_mixed_equal_plain(mixed, opts):
    """Default options pair every request two per register (requests longer
    than a 2,048-row lane in segments by consecutive launches); pair_long off
    pairs only the short ones and stacks the rest; pair_rows=0 stacks all."""
    db, qs = mixed
    with capi.Context(0, capi.default_params(top_k=10)) as c:
        c.load_db(db.residues, db.offsets)
        want = [c.search(q)[0] for q in qs]
        c.serve_start(max_active=64, chunks=3, **opts)
        try:
            # alone: one request at a time
            for i in (0, 6, 12):
                assert c.serve_submit(1000 + i, qs[i]) == 0
                r = drain(c, 1)[1000 + i]
                assert r["status"] == 0
                assert r["hits"] == want[i], f"alone, query {i} len {len(qs[i])}"
                assert r["submit_ms"] <= r["start_ms"] <= r["done_ms"]
            # mixed: all at once, admitted in one round, stacked together
            for i, q in enumerate(qs):
                assert c.serve_submit(i, q) == 0
            got = drain(c, len(qs))
            for i in range(len(qs)):
                assert got[i]["status"] == 0
                assert got[i]["hits"] == want[i], f"mixed, query {i} len {len(qs[i])}"
            st = c.serve_stats()
            assert st.completed == 3 + len(qs) and st.failed == 0
            assert st.chunks == 3 and st.active == 0 and st.pending == 0
        finally:
            c.serve_stop()


def test_joining_mid_ring_and_slot_limit(mixed):
    """Two slots, five chunks: requests wait for a slot, join the ring at
    whatever chunk is next, and still see every record once."""
    db, qs = mixed
    with capi.Context(0, capi.default_params(top_k=7)) as c:
        c.load_db(db.residues, db.offsets)
        want = [c.search(q)[0] for q in qs]
        c.serve_start(max_active=2, chunks=5)
        try:
            order = [3, 6, 0, 9, 2, 11, 5]
            for n, i in enumerate(order):
                assert c.serve_submit(i, qs[i]) == 0
                if n % 2:
                    time.sleep(0.002)
            got = drain(c, len(order))
            for i in order:
                assert got[i]["status"] == 0
                assert got[i]["hits"] == want[i], f"query {i} len {len(qs[i])}"
            st = c.serve_stats()
            assert st.slots == 2
            assert st.rounds >= 5 * (len(order) // 2)
        finally:
            c.serve_stop()


def test_served_golden_and_saturation():
    for name, k in (("edge", 10), ("saturation", 5)):
        res, off, queries, gold = load(name)
        with capi.Context(0, capi.default_params(top_k=k)) as c:
            c.load_db(res, off)
            c.serve_start(max_active=8, chunks=2)
            try:
                sent = 0
                for i, q in enumerate(queries):
                    if len(q) == 0:
                        continue
                    assert c.serve_submit(i, q) == 0
                    sent += 1
                got = drain(c, sent)
            finally:
                c.serve_stop()
        for i, r in got.items():
            sc, idx = oracle.topk(gold[i], k)
            assert r["hits"] == list(zip(sc.tolist(), idx.tolist())), f"{name} query {i}"


def test_admission_queue_bound_and_errors(mixed):
    db, qs = mixed
    with capi.Context(0, capi.default_params(top_k=5)) as c:
        c.load_db(db.residues, db.offsets)
        want = c.search(qs[8])[0]
        c.serve_start(max_active=1, chunks=4, max_pending=1)
        try:
            with pytest.raises(capi.SwError):
                c.serve_start()                                   # already serving
            with pytest.raises(capi.SwError):
                c.search(qs[0])                                   # the loop owns the context
            with pytest.raises(capi.SwError):
                c.serve_submit(1, np.zeros(0, dtype=np.uint8))    # empty
            with pytest.raises(capi.SwError):
                c.serve_submit(1, np.zeros((1 << 24) + 1, dtype=np.uint8))  # beyond 2^24
            with pytest.raises(capi.SwError):
                c.serve_submit(1, np.full(10, 25, dtype=np.uint8))  # bad code
            accepted, busy = [], 0
            for i in range(40):
                st = c.serve_submit(i, qs[8])
                if st == 0:
                    accepted.append(i)
                else:
                    busy += 1
            got = drain(c, len(accepted))
            assert sorted(got) == accepted
            for r in got.values():
                assert r["status"] == 0 and r["hits"] == want
            st = c.serve_stats()
            assert st.submitted == len(accepted) and st.completed == len(accepted)
            assert busy == 40 - len(accepted)
        finally:
            c.serve_stop()
        with pytest.raises(capi.SwError):
            c.serve_submit(1, qs[0])                              # not serving any more
        assert c.search(qs[8])[0] == want                             # context usable again


def test_memory_budget_bounds_slots(mixed):
    db, qs = mixed
    with capi.Context(0, capi.default_params(top_k=5)) as c:
        c.load_db(db.residues, db.offsets)
        per_slot = 4 * c.n_records + 2 * 1024 * 8 + 5 * 8
        c.serve_start(max_active=64, chunks=2, memory_budget=3 * per_slot)
        try:
            assert c.serve_stats().slots == 3
        finally:
            c.serve_stop()
