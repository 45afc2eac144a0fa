"""Queries of any length.  A query whose profile does not fit one block's
shared memory is scored in row segments of whole passes by consecutive
launches: each launch's last pass writes the boundary row (H and F of its
last query row per column) that the next launch's first pass reads, and a
record's score is the maximum over the segments; a record whose 16-bit lane
may have wrapped in any segment is listed once for the exact 32-bit pass.
The reference takes any query length (src/DataPool.cpp:312-344; avxCompute
walks the whole query).  Checked here against the oracle on the plain path
(several shapes, so the segment lengths differ), through the batched path,
and through serving, where a request longer than one stack runs alone at a
round boundary and must equal the plain search."""
import time

import numpy as np
import pytest

import oracle
from swhybrid_b200 import capi, param, synth

pytestmark = pytest.mark.gpu
M = param.blosum62()


@pytest.fixture(scope="module")
def case():
    rng = np.random.default_rng(404)
    q = synth.residues(rng, 12_000)
    db = synth.small_db(405, 500)
    # homologs of the query's two ends and of a stretch across the first
    # segment boundaries (rows 8,192 and 8,960 for the shapes below)
    db, _ = synth.plant_homologs(rng, db, q[:900], 0.01)
    db, _ = synth.plant_homologs(rng, db, q[7800:9400], 0.01)
    db, _ = synth.plant_homologs(rng, db, q[-700:], 0.01)
    want = oracle.search(q, db.residues, db.offsets, M, 12, 2, mode=1)
    return db, q, want


@pytest.mark.parametrize("shape", [None, (32, 64), (16, 64), (16, 16), (8, 40)])
def test_plain_long_query_equals_oracle(case, shape):
    db, q, want = case
    with capi.Context(0, capi.default_params(top_k=10)) as c:
        c.load_db(db.residues, db.offsets)
        if shape:
            c.set_kernel_config((shape[0], shape[1], shape[0], shape[1], 0))
        hits, scores = c.search(q, want_scores=True)
        launches = c.run_stats().launches
    np.testing.assert_array_equal(scores, want, err_msg=f"shape {shape}")
    ws, wi = oracle.topk(want, 10)
    assert hits == list(zip(ws.tolist(), wi.tolist()))
    assert want.max() >= 117          # the homologs overflow the reference's int8 pass
    if shape:
        assert launches >= 4          # at least two first-pass launches + re-score + top-k


def test_long_query_saturation_across_segments():
    """A W run: 11 per cell along the diagonal, the 16-bit lanes wrap in a
    later segment, the exact 32-bit pass (and the reference's 65535 cap)
    decide the score."""
    W = param.encode("W" * 10_000)
    rec = param.encode("A" * 50 + "W" * 9_000 + "A" * 50)
    short = synth.residues(np.random.default_rng(3), 300)
    off = np.array([0, len(rec), len(rec) + len(short)], dtype=np.uint64)
    res = np.concatenate([rec, short]).astype(np.uint8)
    exact = oracle.gotoh(W, rec, M)
    assert exact == 99_000
    for cap, top in ((True, 65535), (False, exact)):
        with capi.Context(0, capi.default_params(top_k=2, reference_cap=cap)) as c:
            c.load_db(res, off)
            c.set_kernel_config((32, 64, 32, 64, 0))
            hits, scores = c.search(W, want_scores=True)
        assert scores[0] == top, f"cap={cap}"
        assert scores[1] == oracle.gotoh(W, short, M)


def test_batched_long_query_equals_plain(case):
    db, q, want = case
    rng = np.random.default_rng(9)
    qs = [synth.residues(rng, 200), q, synth.residues(rng, 3000), q[:9000]]
    with capi.Context(0, capi.default_params(top_k=10)) as c:
        c.load_db(db.residues, db.offsets)
        hits, scores = c.search_batch(qs, want_scores=True)
        for i, qq in enumerate(qs):
            ph, ps = c.search(qq, want_scores=True)
            np.testing.assert_array_equal(scores[i], ps, err_msg=f"query {i}")
            assert hits[i] == ph
    np.testing.assert_array_equal(scores[1], want)


def test_served_long_request_equals_plain(case):
    db, q, want = case
    rng = np.random.default_rng(10)
    others = [synth.residues(rng, int(L)) for L in (40, 700, 2500)]
    with capi.Context(0, capi.default_params(top_k=10)) as c:
        c.load_db(db.residues, db.offsets)
        plain = {i: c.search(x)[0] for i, x in enumerate([q] + others)}
        c.serve_start(max_active=8, chunks=3)
        try:
            for i, x in enumerate([q] + others):
                assert c.serve_submit(500 + i, x) == 0
            got = {}
            t_end = time.time() + 120
            while len(got) < 4 and time.time() < t_end:
                for r in c.serve_poll(16, timeout_ms=200):
                    got[r["id"]] = r
            assert len(got) == 4
            for i in range(4):
                assert got[500 + i]["status"] == 0
                assert got[500 + i]["hits"] == plain[i], f"request {i}"
        finally:
            c.serve_stop()
    ws, wi = oracle.topk(want, 10)
    assert plain[0] == list(zip(ws.tolist(), wi.tolist()))
