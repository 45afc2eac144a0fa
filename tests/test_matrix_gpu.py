"""Other scoring matrices and gap costs end to end: a random symmetric matrix
read through the -m text path, with several gap costs, must give the exact
Gotoh scores of the oracle in the plain, batched and traceback paths."""
import numpy as np
import pytest

import oracle
from swhybrid_b200 import capi, param, synth

pytestmark = pytest.mark.gpu
ALPHA = param.ALPHABET


def random_matrix(seed, lo=-12, hi=19):
    rng = np.random.default_rng(seed)
    r = rng.integers(lo, hi, size=(23, 23))
    r = np.triu(r) + np.triu(r, 1).T
    r[np.arange(23), np.arange(23)] = np.abs(r.diagonal()) + 4     # positive self scores
    lines = ["   " + " ".join(ALPHA)]
    lines += [ALPHA[i] + " " + " ".join(str(int(v)) for v in r[i]) for i in range(23)]
    return capi.parse_matrix("\n".join(lines) + "\n")


@pytest.mark.parametrize("seed,go,ge", [(1, 10, 2), (2, 6, 1), (3, 15, 4)])
def test_random_matrix_plain_batch_traceback(seed, go, ge):
    m = random_matrix(seed)
    rng = np.random.default_rng(100 + seed)
    db = synth.small_db(110 + seed, 1500)
    qs = [synth.residues(rng, L) for L in (90, 400, 1300)]
    db, _ = synth.plant_homologs(rng, db, qs[1], 0.01)
    want = [oracle.search(q, db.residues, db.offsets, m, go + ge, ge, mode=0) for q in qs]
    params = capi.default_params(gap_open=go, gap_extend=ge, matrix=m, reference_cap=False)
    with capi.Context(0, params) as c:
        c.load_db(db.residues, db.offsets)
        for q, w in zip(qs, want):
            hits, scores = c.search(q, want_scores=True)
            np.testing.assert_array_equal(scores, w)
            sc, idx = oracle.topk(w, 10)
            assert hits == list(zip(sc.tolist(), idx.tolist()))
        bh, bscores = c.search_batch(qs, want_scores=True)
        for qi, w in enumerate(want):
            np.testing.assert_array_equal(bscores[qi], w)
        recs = [i for (_, i) in c.search(qs[1])[0]][:5]
        for al in c.traceback(qs[1], recs):
            t = oracle.traceback(qs[1], db.record(al["index"]), m, go + ge, ge)
            assert (al["score"], al["cigar"], al["q_begin"], al["d_begin"]) == \
                (t["score"], t["cigar"], t["q_begin"], t["d_begin"])
