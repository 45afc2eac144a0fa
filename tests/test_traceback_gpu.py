"""Alignments of chosen records (sw_traceback): the coordinates and CIGAR of
every alignment must equal the oracle's traceback under the same rules (the
first maximal cell in record-then-query order; ties prefer the diagonal,
then a gap in the query, then a gap in the record, and an opened gap over an
extended one), and the alignment's score must be the record's search
score."""
import re

import numpy as np
import pytest

import oracle
from swhybrid_b200 import capi, param, synth

pytestmark = pytest.mark.gpu
M = param.blosum62()


def cigar_score(q, d, al, oe, e):
    """Score of the alignment the CIGAR describes, and its identities."""
    i, j, s, same = al["q_begin"], al["d_begin"], 0, 0
    for n, op in re.findall(r"(\d+)([MID])", al["cigar"]):
        n = int(n)
        if op == "M":
            for _ in range(n):
                s += int(M[q[i], d[j]])
                same += int(q[i] == d[j])
                i += 1
                j += 1
        elif op == "I":
            s -= oe + e * (n - 1)
            i += n
        else:
            s -= oe + e * (n - 1)
            j += n
    assert (i, j) == (al["q_end"], al["d_end"])
    return s, same


@pytest.fixture(scope="module")
def case():
    rng = np.random.default_rng(61)
    db = synth.small_db(62, 1500)
    q = synth.residues(rng, 1300)               # 3 passes of 512 rows
    db, planted = synth.plant_homologs(rng, db, q, 0.01)
    return db, q, planted


def check(db, q, recs, got, oe=12, e=2):
    for r, al in zip(recs, got):
        d = db.record(int(r))
        want = oracle.traceback(q, d, M, oe, e)
        assert al["index"] == int(r)
        for key in ("score", "q_begin", "q_end", "d_begin", "d_end", "cigar"):
            assert al[key] == want[key], f"record {r} ({len(d)} residues): {key} {al[key]} != {want[key]}"
        if al["score"] > 0:
            s, same = cigar_score(q, d, al, oe, e)
            assert s == al["score"]
            assert same == al["matches"]


def test_top_hits_and_random_records(case):
    db, q, planted = case
    with capi.Context(0, capi.default_params(top_k=10, reference_cap=False)) as c:
        c.load_db(db.residues, db.offsets)
        hits, scores = c.search(q, want_scores=True)
        recs = [i for (_, i) in hits] + list(np.random.default_rng(1).choice(db.n, 20, replace=False))
        got = c.traceback(q, recs)
        check(db, q, recs, got)
        for al in got:
            assert al["score"] == scores[al["index"]]
        assert all(int(i) in set(planted.tolist()) for (_, i) in hits)


def test_long_records_and_other_gaps():
    rng = np.random.default_rng(63)
    q = synth.residues(rng, 700)
    lens = np.concatenate([rng.integers(3000, 6000, size=4), rng.integers(1, 50, size=6), [0]])
    db = synth.db_from_lengths(rng, lens)
    db, _ = synth.plant_homologs(rng, db, q, 0.3)
    for go, ge in [(10, 2), (5, 1), (11, 3)]:
        with capi.Context(0, capi.default_params(gap_open=go, gap_extend=ge,
                                                 reference_cap=False)) as c:
            c.load_db(db.residues, db.offsets)
            recs = list(range(db.n))
            check(db, q, recs, c.traceback(q, recs), go + ge, ge)


def test_two_calls_in_a_row_and_edges(case):
    db, q, _ = case
    with capi.Context(0) as c:
        c.load_db(db.residues, db.offsets)
        a = c.traceback(q[:40], [0, 5, 9])
        b = c.traceback(q[:40], [0, 5, 9])
        assert a == b
        check(db, q[:40], [0, 5, 9], a)
        empty = c.traceback(np.zeros(0, dtype=np.uint8), [3])
        assert empty[0]["score"] == 0 and empty[0]["cigar"] == ""
        assert c.traceback(q, []) == []
        with pytest.raises(capi.SwError):
            c.traceback(q, [db.n])
