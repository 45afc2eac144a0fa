"""CPU tests of the oracle (test infrastructure): the C restatement against the
reference's own kernels' golden vectors, against a pure-Python Gotoh, and the
top-k tie order against a model of the reference's ResultList."""
import hashlib
import os

import numpy as np
import pytest

import oracle
from swhybrid_b200 import param, synth

GOLD = os.path.join(os.path.dirname(__file__), "golden")
M = param.blosum62()


def load(name):
    z = np.load(os.path.join(GOLD, name + ".npz"))
    qo = z["qoffsets"].astype(np.int64)
    queries = [z["queries"][qo[i]:qo[i + 1]] for i in range(len(qo) - 1)]
    return z["residues"], z["offsets"], queries, z["scores"]


def py_gotoh(q, d, oe=12, e=2):
    """Independent pure-Python Gotoh (rows = query, columns = DB record)."""
    best = 0
    H = [0] * (len(q) + 1)
    Ecol = [0] * (len(q) + 1)
    for j in range(len(d)):
        diag, f = 0, 0
        for i in range(len(q)):
            h = max(0, diag + int(M[q[i], d[j]]), Ecol[i + 1], f)
            best = max(best, h)
            diag = H[i + 1]
            H[i + 1] = h
            Ecol[i + 1] = max(Ecol[i + 1] - e, h - oe)
            f = max(f - e, h - oe)
    return best


@pytest.mark.parametrize("name", ["edge", "homolog", "saturation"])
def test_restatement_matches_reference_golden(name):
    res, off, queries, gold = load(name)
    for qi, q in enumerate(queries):
        got = oracle.search(q, res, off, M, 12, 2, mode=1)
        np.testing.assert_array_equal(got, gold[qi], err_msg=f"{name} query {qi}")


def test_restatement_small20k_golden():
    db = synth.small_db(1, 20_000)
    q = synth.query(375, 375)
    z = np.load(os.path.join(GOLD, "small20k_q375.npz"))
    h = hashlib.sha256()
    for a in (db.residues, db.offsets, q):
        h.update(np.ascontiguousarray(a).tobytes())
    assert h.hexdigest() == str(z["input_digest"]), "synthetic generator changed"
    got = oracle.search(q, db.residues, db.offsets, M, 12, 2, mode=1)
    np.testing.assert_array_equal(got, z["scores"])


def test_c_gotoh_matches_python():
    rng = np.random.default_rng(5)
    for _ in range(25):
        q = synth.residues(rng, int(rng.integers(1, 40)))
        d = synth.residues(rng, int(rng.integers(1, 40)))
        if rng.random() < 0.3:
            d = synth.mutate(rng, q, 0.1, 0.05)
            if len(d) == 0:
                continue
        assert oracle.gotoh(q, d, M) == py_gotoh(q, d)


def test_reference_cap_and_int16_window():
    W = param.encode("W" * 6000)
    off = np.array([0, 6000], dtype=np.uint64)
    assert oracle.gotoh(W, W, M) == 66000
    assert oracle.search(W, W, off, M, mode=1)[0] == 65535
    assert oracle.search(W, W, off, M, mode=0)[0] == 66000


@pytest.mark.skipif(not oracle.ref_available(), reason="reference kernels not built")
def test_reference_kernels_reproduce_golden():
    res, off, queries, gold = load("homolog")
    for qi, q in enumerate(queries):
        got, _, novf = oracle.ref_search(q, res, off, M, 10, 2, threads=4)
        np.testing.assert_array_equal(got, gold[qi])
        assert novf > 0     # the int16 recalc path ran


def _result_list_model(scores, k):
    """The reference ResultList<int> (src/ResultList.h:20-79), pushed in record
    order: pre-filled with (0, 0); push rejects score <= bottom and inserts
    before the first strictly smaller entry."""
    lst = [(0, 0)] * k
    bottom = 0
    for i, s in enumerate(scores):
        if s <= bottom:
            continue
        for p, (sc, _) in enumerate(lst):
            if sc < s:
                lst.insert(p, (int(s), i))
                break
        lst.pop()
        bottom = lst[-1][0]
    return [x for x in lst if x[0] > 0]


def test_topk_tie_order_matches_result_list():
    rng = np.random.default_rng(9)
    for k in (1, 3, 10, 25):
        s = rng.integers(0, 12, size=400).astype(np.int32)
        sc, idx = oracle.topk(s, k)
        assert list(zip(sc.tolist(), idx.tolist())) == _result_list_model(s, k)


def test_blosum62_is_the_reference_table():
    p = os.path.join(oracle.reference_root(), "src", "Param.h")
    if not os.path.exists(p):
        pytest.skip("reference tree not present")
    import re
    src = open(p).read()
    i = src.index("blosum62[32][32] =")
    j = src.index("};", i)
    nums = [int(x) for x in re.findall(r"-?\d+", src[i + len("blosum62[32][32] ="):j])]
    np.testing.assert_array_equal(np.array(nums).reshape(32, 32), M)


def test_oracle_traceback_is_consistent():
    """The oracle's traceback reaches the Gotoh score along the path its CIGAR
    describes, for homologs and random pairs under several gap costs."""
    import re
    rng = np.random.default_rng(71)
    M = param.blosum62()
    for trial in range(40):
        q = synth.residues(rng, int(rng.integers(1, 120)))
        d = synth.residues(rng, int(rng.integers(1, 160)))
        if trial % 2:
            d = np.concatenate([d[:20], synth.mutate(rng, q, 0.25, 0.08), d[20:]])
        oe, e = [(12, 2), (6, 1), (14, 3)][trial % 3]
        al = oracle.traceback(q, d, M, oe, e)
        assert al["score"] == oracle.gotoh(q, d, M, oe, e)
        i, j, s = al["q_begin"], al["d_begin"], 0
        for n, op in re.findall(r"(\d+)([MID])", al["cigar"]):
            n = int(n)
            if op == "M":
                s += sum(int(M[q[i + k], d[j + k]]) for k in range(n))
                i += n
                j += n
            else:
                s -= oe + e * (n - 1)
                i, j = (i + n, j) if op == "I" else (i, j + n)
        assert (i, j) == (al["q_end"], al["d_end"])
        assert s == al["score"]
