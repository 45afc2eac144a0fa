"""Batched search (sw_search_batch): every query's scores and top-k must equal
what the plain per-query search returns (which is itself pinned to the
reference's golden vectors), for every bucket/cut-over arrangement, with the
captured CUDA graph replayed."""
import os

import numpy as np
import pytest

import oracle
from swhybrid_b200 import capi, param, synth

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
M = param.blosum62()


def load(name):
    z = np.load(os.path.join(GOLD, name + ".npz"))
    qo = z["qoffsets"].astype(np.int64)
    queries = [z["queries"][qo[i]:qo[i + 1]] for i in range(len(qo) - 1)]
    return z["residues"], z["offsets"], queries, z["scores"]


@pytest.fixture(scope="module")
def ctx():
    c = capi.Context(0, capi.default_params(top_k=10))
    yield c
    c.close()


def test_batch_equals_golden(ctx):
    res, off, queries, gold = load("edge")
    ctx.load_db(res, off)
    hits, scores = ctx.search_batch(queries, want_scores=True)
    for qi in range(len(queries)):
        np.testing.assert_array_equal(scores[qi], gold[qi], err_msg=f"query {qi}")
        sc, idx = oracle.topk(gold[qi], 10)
        assert hits[qi] == list(zip(sc.tolist(), idx.tolist()))


@pytest.mark.parametrize("cutover", [0, 300, 1000, 4096])
def test_batch_equals_plain_with_split(ctx, cutover):
    rng = np.random.default_rng(41)
    db = synth.small_db(12, 3000)
    qs = [synth.residues(rng, int(L)) for L in (5, 31, 144, 375, 700, 1500, 2600, 60, 0)]
    db, _ = synth.plant_homologs(rng, db, qs[4], 0.01)
    ctx.load_db(db.residues, db.offsets)
    ctx.set_batch_options(cutover=cutover)
    try:
        for rep in range(2):                # capture, then replay
            hits, scores = ctx.search_batch(qs, want_scores=True)
            for qi, q in enumerate(qs):
                h1, s1 = ctx.search(q, want_scores=True)
                np.testing.assert_array_equal(scores[qi], s1, err_msg=f"q{qi} len {len(q)}")
                assert hits[qi] == h1
    finally:
        ctx.set_batch_options()


def test_batch_saturation_and_cap():
    res, off, queries, gold = load("saturation")
    with capi.Context(0, capi.default_params(top_k=5)) as c:
        c.load_db(res, off)
        hits, scores = c.search_batch(queries, want_scores=True)
        np.testing.assert_array_equal(scores, gold)


def test_batch_without_graph_and_empty(ctx):
    db = synth.small_db(13, 500)
    ctx.load_db(db.residues, db.offsets)
    ctx.set_batch_options(use_graph=False)
    try:
        qs = [synth.query(1, 100), np.zeros(0, dtype=np.uint8), synth.query(2, 333)]
        hits, scores = ctx.search_batch(qs, want_scores=True)
        assert hits[1] == [] and not scores[1].any()
        for qi in (0, 2):
            want = oracle.search(qs[qi], db.residues, db.offsets, M, 12, 2)
            np.testing.assert_array_equal(scores[qi], want)
    finally:
        ctx.set_batch_options()


def test_many_short_queries_share_stacks(ctx):
    """Dozens of short queries packed into shared stacks (several per 16x32
    row block layout), plus planted homologs so some records overflow int16."""
    rng = np.random.default_rng(43)
    qs = [synth.residues(rng, int(L)) for L in rng.integers(1, 120, size=40)]
    db = synth.small_db(14, 2500)
    db, _ = synth.plant_homologs(rng, db, qs[0], 0.01)
    ctx.load_db(db.residues, db.offsets)
    for opts in ({}, {"stack_shape": (16, 8), "stack_rows": 256, "pair_rows": 0},
                 {"stack_shape": (32, 4), "stack_rows": 4096, "cutover": 200, "pair_rows": 0},
                 {"stack_shape": (16, 32), "stack_rows": 1024, "cutover": 1000, "pair_rows": 0}):
        ctx.set_batch_options(**opts)
        try:
            hits, scores = ctx.search_batch(qs, want_scores=True)
        finally:
            ctx.set_batch_options()
        for qi, q in enumerate(qs):
            want = oracle.search(q, db.residues, db.offsets, M, 12, 2)
            np.testing.assert_array_equal(scores[qi], want, err_msg=f"{opts} q{qi} len {len(q)}")
            sc, idx = oracle.topk(want, 10)
            assert hits[qi] == list(zip(sc.tolist(), idx.tolist()))


@pytest.mark.parametrize("pair_shape,pair_rows,pair_long", [
    ((16, 64), 2048, True), ((16, 64), 2048, False), ((16, 32), 2048, True),
    ((32, 32), 1024, True), ((8, 64), 512, True), ((16, 48), 1500, False),
    ((16, 64), 1024, True)])
def test_paired_queries_every_shape(ctx, pair_shape, pair_rows, pair_long):
    """Queries paired two per register (one per 16-bit lane, a pre-packed
    profile): every paired shape, lanes spanning several passes, an odd lane
    count, and queries longer than the pair limit -- paired too, in segments
    scored by consecutive launches (pair_long), or left to the stacked
    kernel."""
    rng = np.random.default_rng(47)
    lens = list(rng.integers(1, 400, size=23)) + [pair_rows, pair_rows + 1, 2600, 777, 5000, 4097]
    qs = [synth.residues(rng, int(L)) for L in lens]
    db = synth.small_db(15, 2000)
    db, _ = synth.plant_homologs(rng, db, qs[-1], 0.01)
    ctx.load_db(db.residues, db.offsets)
    ctx.set_batch_options(pair_rows=pair_rows, pair_shape=pair_shape, pair_long=pair_long)
    try:
        for rep in range(2):                           # capture, then replay
            hits, scores = ctx.search_batch(qs, want_scores=True)
            for qi, q in enumerate(qs):
                want = oracle.search(q, db.residues, db.offsets, M, 12, 2)
                np.testing.assert_array_equal(scores[qi], want,
                                              err_msg=f"{pair_shape} q{qi} len {len(q)}")
                sc, idx = oracle.topk(want, 10)
                assert hits[qi] == list(zip(sc.tolist(), idx.tolist()))
    finally:
        ctx.set_batch_options()


def test_paired_queries_saturate():
    """Paired lanes whose scores leave the 16-bit window (a matrix scoring
    W-W at 127, runs of W): the flagged (query, record) entries go through
    the 32-bit re-score and come out exact."""
    m = param.blosum62().copy()
    w = param.ALPHABET.index("W")
    m[w, w] = 127
    rng = np.random.default_rng(49)
    lens = [100, 257, 258, 300, 600]
    recs = [np.full(L, w, dtype=np.uint8) for L in lens] + \
           [synth.residues(rng, int(L)) for L in rng.integers(5, 500, size=60)]
    off = np.zeros(len(recs) + 1, dtype=np.uint64)
    off[1:] = np.cumsum([len(r) for r in recs])
    res = np.concatenate(recs)
    qs = [np.full(L, w, dtype=np.uint8) for L in (256, 258, 400)] + \
         [synth.residues(rng, 300), np.full(1000, w, dtype=np.uint8)]
    with capi.Context(0, capi.default_params(top_k=5, matrix=m, reference_cap=False)) as c:
        c.load_db(res, off)
        hits, scores = c.search_batch(qs, want_scores=True)
        for qi, q in enumerate(qs):
            want = oracle.search(q, res, off, m, 12, 2, mode=0)
            np.testing.assert_array_equal(scores[qi], want, err_msg=f"q{qi}")
        assert c.run_stats().rescored > 0
        assert scores[4].max() == 127 * 600
