"""Overflow / long-record stress at full size: 100,000 records (lengths
lognormal(5.6, 0.6) clipped to 20..5,000) plus 1 % long records uniform on
10,000..40,000, with 0.5 % of the records replaced by homologs of the eight
queries (substitution rate uniform on 10..30 %, indels 2 %), queries of
500..4,000 residues.  Every planted homolog overflows the reference's int8
pass and goes through its int16 re-score; the long records take the
concurrent long-pair launch.

The oracle cannot score the whole DB in test time, so exactness is checked on
a sample that holds every planted homolog, a slice of the long records and
random others (the oracle scores the sample as its own DB, and record scores
do not depend on the rest of the DB), and the top-10 is checked where it is
decidable: every GPU top-10 record lies in the sample, and every record
outside it scores below the 10th hit."""
import numpy as np
import pytest

import oracle
from swhybrid_b200 import capi, param, synth

pytestmark = pytest.mark.gpu
M = param.blosum62()


def stress_case(seed=4):
    rng = np.random.default_rng(seed + 1)
    db, queries, picks, owner = synth.stress_workload(seed)
    lens = np.diff(db.offsets.astype(np.int64))
    long_ids = np.flatnonzero(lens >= 10_000)
    rest = np.setdiff1d(np.arange(db.n), np.concatenate([picks, long_ids]))
    sample = np.unique(np.concatenate([
        picks, rng.choice(long_ids, size=24, replace=False),
        rng.choice(rest, size=400, replace=False)]))
    return db, queries, sample, owner


def sub_db(db, ids):
    recs = [db.record(int(i)) for i in ids]
    lens = np.array([len(r) for r in recs], dtype=np.int64)
    off = np.zeros(len(ids) + 1, dtype=np.uint64)
    off[1:] = np.cumsum(lens)
    return np.concatenate(recs).astype(np.uint8), off


def test_stress_full_size_sampled_exact_and_top10():
    db, queries, sample, owner = stress_case()
    res_s, off_s = sub_db(db, sample)
    with capi.Context(0, capi.default_params(top_k=10)) as c:
        c.load_db(db.residues, db.offsets)
        for qi, q in enumerate(queries):
            hits, scores = c.search(q, want_scores=True)
            want = oracle.search(q, res_s, off_s, M, 12, 2)
            np.testing.assert_array_equal(scores[sample], want, err_msg=f"query {qi}")
            # the top-10 is decidable from the sample
            assert len(hits) == 10
            top_idx = [i for (_, i) in hits]
            assert np.isin(top_idx, sample).all()
            outside = np.ones(db.n, dtype=bool)
            outside[sample] = False
            assert scores[outside].max() < hits[-1][0]
            sc, pos = oracle.topk(want, 10)
            assert hits == list(zip(sc.tolist(), sample[pos].tolist())), f"query {qi}"
            # the hits are this query's planted homologs, far above int8's range
            assert all(owner.get(i) == qi for i in top_idx)
            assert hits[-1][0] >= 117
