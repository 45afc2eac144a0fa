"""Row-segment plans: a plain search whose shape-table entry names a plan runs
the query's rows as consecutive launches of different shapes (whole passes
of each, the last segment taking the rest), so that only the last pass
carries padding rows.  Each launch reads the boundary row the launch before
wrote and the scores merge by maximum, exactly as when one shape splits a
query too long for its profile.  The scores must equal the oracle's (the
restatement of the reference's avxCompute + avxCompute16,
src/AVXKernel.cpp:408-554, 866-1016) and the single-shape search's,
including a 16-bit lane that wraps in a later segment than the one it
started in."""
import numpy as np
import pytest

import oracle
from swhybrid_b200 import capi, param, synth

pytestmark = pytest.mark.gpu
M = param.blosum62()
PLAN = ((16, 48, 1), (32, 20, 1), (16, 56, 0))        # 768 + 640 rows, then the rest


def uniform_db(seed: int, n: int, lo: int, hi: int) -> synth.DB:
    rng = np.random.default_rng(seed)
    return synth.db_from_lengths(rng, rng.integers(lo, hi + 1, size=n))


def table(plan, cfg=(16, 48, 16, 48, 0)):
    return [(1 << 30, cfg, plan)]


@pytest.fixture(scope="module")
def case():
    """8,000 records of 60..100 residues (every shape of the plan gets more
    columns per group than the longest pair, so the plan runs) with homologs
    of the query's stretches around the segment boundaries (rows 768 and
    1,408)."""
    rng = np.random.default_rng(77)
    q = synth.residues(rng, 2400)
    db = uniform_db(78, 8000, 60, 100)
    db, _ = synth.plant_homologs(rng, db, q[700:800], 0.004)
    db, _ = synth.plant_homologs(rng, db, q[1360:1460], 0.004)
    db, _ = synth.plant_homologs(rng, db, q[2300:2400], 0.004)
    return db, q


@pytest.mark.parametrize("qlen,want_plan", [
    (1409, [(16, 48, 1), (32, 20, 1), (16, 56, 1)]),      # the rest is one row
    (1500, [(16, 48, 1), (32, 20, 1), (16, 56, 1)]),
    (2304, [(16, 48, 1), (32, 20, 1), (16, 56, 1)]),      # the rest fills its pass
    (2400, [(16, 48, 1), (32, 20, 1), (16, 56, 2)]),
    (1408, [(16, 48, 1), (32, 20, 1)]),                   # the fixed steps take it all
    (700, [(16, 48, 1)]),                                 # shorter than the first step
])
def test_plan_equals_oracle_and_single_shape(case, qlen, want_plan):
    db, q = case
    qq = q[:qlen]
    want = oracle.search(qq, db.residues, db.offsets, M, 12, 2, mode=1)
    with capi.Context(0, capi.default_params(top_k=10)) as c:
        c.load_db(db.residues, db.offsets)
        c.set_tuning(table(PLAN))
        assert c.plan(qlen) == want_plan
        hits, scores = c.search(qq, want_scores=True)
        st = c.run_stats()
        c.set_tuning(table(()))
        assert c.plan(qlen) == [(16, 48, -(-qlen // 768))]
        hits1, scores1 = c.search(qq, want_scores=True)
    np.testing.assert_array_equal(scores, want)
    np.testing.assert_array_equal(scores1, want)
    ws, wi = oracle.topk(want, 10)
    assert hits == list(zip(ws.tolist(), wi.tolist())) == hits1
    assert (st.used.short_group_width, st.used.short_rows_per_thread) == want_plan[0][:2]
    if qlen >= 800:                  # homologs of rows 700..799 beyond the int8 range
        assert want.max() > 117


def test_plan_dropped_when_one_pair_would_hold_a_launch(case):
    """The entry's own shape (32x56: 8 groups per SM) gets about 280 columns
    per group of this DB, the plan's shapes (16 groups per SM) about 140.  A
    record of 220 residues is below the first share, so no long-pair split is
    made, and above the second: the plan's launches would each end on that
    pair, so the search runs the entry's shape (same scores)."""
    db, q = case
    rng = np.random.default_rng(5)
    extra = synth.residues(rng, 220)
    res = np.concatenate([db.residues, extra]).astype(np.uint8)
    off = np.concatenate([db.offsets, [db.offsets[-1] + 220]]).astype(np.uint64)
    qq = q[:1500]
    with capi.Context(0, capi.default_params(top_k=10)) as c:
        c.load_db(res, off)
        c.set_tuning(table(PLAN, cfg=(32, 56, 32, 56, 0)))
        assert c.plan(1500) == [(32, 56, 1)]
        assert c.kernel_config(1500) == (32, 56, 32, 56, 0)
        _, scores = c.search(qq, want_scores=True)
        assert c.run_stats().used.cutover == 0          # no long-pair split
        c.load_db(db.residues, db.offsets)              # without the record: planned
        c.set_tuning(table(PLAN, cfg=(32, 56, 32, 56, 0)))
        assert c.plan(1500) == [(16, 48, 1), (32, 20, 1), (16, 56, 1)]
    np.testing.assert_array_equal(scores, oracle.search(qq, res, off, M, 12, 2, mode=1))


def test_plan_with_long_pair_split(case):
    """Five records of 3,000 residues make the entry's shape split its long
    pairs off to the long-pair kernel (which scores them against the whole
    query, concurrently); the plan then runs on the other pairs, whose
    longest is below every step's share.  Scores equal the oracle's."""
    db, q = case
    rng = np.random.default_rng(6)
    longs = [synth.residues(rng, 3000) for _ in range(4)] + [q[200:3000].copy()]
    res = np.concatenate([db.residues] + longs).astype(np.uint8)
    lens = np.concatenate([db.lengths(), [len(x) for x in longs]])
    off = np.zeros(len(lens) + 1, dtype=np.uint64)
    off[1:] = np.cumsum(lens)
    qq = q[:2400]
    with capi.Context(0, capi.default_params(top_k=10)) as c:
        c.load_db(res, off)
        c.set_tuning(table(PLAN))
        assert c.plan(2400) == [(16, 48, 1), (32, 20, 1), (16, 56, 2)]
        hits, scores = c.search(qq, want_scores=True)
        used = c.run_stats().used
    assert used.cutover > 0 and used.long_group_width == 32      # the split ran
    want = oracle.search(qq, res, off, M, 12, 2, mode=1)
    np.testing.assert_array_equal(scores, want)
    ws, wi = oracle.topk(want, 10)
    assert hits == list(zip(ws.tolist(), wi.tolist()))
    assert hits[0][1] == len(lens) - 1      # the record copied from the query


def test_plan_steps_refused_when_not_compiled():
    with capi.Context(0) as c:
        with pytest.raises(capi.SwError) as e:
            c.set_tuning(table(((16, 50, 1), (16, 48, 0))))
        assert e.value.status == 1


def test_plan_saturation_across_segments():
    """A run of W in query and record: 11 per cell along the diagonal.  The
    record's 16-bit lane passes the overflow threshold only in the plan's
    last segment (rows 1,920..3,299), after two launches of other shapes
    handed it on through the boundary row; the exact 32-bit pass gives the
    oracle's score (33,000 along the run, a few more from the query's random
    head).  The DB is large enough (48,000 records of 200..500 residues)
    that every shape of the plan gets more columns per group than the W
    record's 3,000."""
    plan = ((16, 64, 1), (16, 56, 1), (16, 48, 0))
    rng = np.random.default_rng(31)
    q = np.concatenate([synth.residues(rng, 300), param.encode("W" * 3000)]).astype(np.uint8)
    db = uniform_db(32, 48_000, 200, 500)
    wrec = param.encode("A" * 10 + "W" * 3000)
    mid = param.encode("W" * 1500)          # 16,500: no overflow
    res = np.concatenate([db.residues, wrec, mid]).astype(np.uint8)
    lens = np.concatenate([db.lengths(), [len(wrec), len(mid)]])
    off = np.zeros(len(lens) + 1, dtype=np.uint64)
    off[1:] = np.cumsum(lens)
    n = len(lens)
    with capi.Context(0, capi.default_params(top_k=10)) as c:
        c.load_db(res, off)
        c.set_tuning(table(plan))
        assert c.plan(len(q)) == [(16, 64, 1), (16, 56, 1), (16, 48, 2)]
        hits, scores = c.search(q, want_scores=True)
        rescored = c.run_stats().rescored
        c.set_kernel_config((16, 48, 16, 48, 0))
        hits1, scores1 = c.search(q, want_scores=True)
    top = oracle.gotoh(q, wrec, M)
    assert top >= 33_000 and scores[n - 2] == top
    assert scores[n - 1] == oracle.gotoh(q, mid, M) == 16_500
    assert rescored >= 1
    np.testing.assert_array_equal(scores, scores1)
    assert hits == hits1 and hits[0] == (top, n - 2)
    sample = np.random.default_rng(33).choice(n - 2, size=200, replace=False)
    sub = synth.DB(res, off).subset(sample)
    np.testing.assert_array_equal(scores[sample],
                                  oracle.search(q, sub.residues, sub.offsets, M, 12, 2, mode=1))
