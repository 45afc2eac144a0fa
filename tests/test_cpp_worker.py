"""The C++ mirror of the reference's plugin surface (swhybrid_b200/cpp):
ResultList semantics on the CPU, and a WorkerPool of B200Workers end to end
on the GPU (FASTA in, merged top-k out), checked against the oracle."""
import os
import subprocess

import numpy as np
import pytest

import oracle
from swhybrid_b200 import capi, param, synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
RL = os.path.join(ROOT, "swhybrid_b200", "cpp", "result_list_test")
WP = os.path.join(ROOT, "swhybrid_b200", "worker_pool_test")


def _result_list_model(scores, k):
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
    return lst


def test_cpp_result_list_semantics():
    rng = np.random.default_rng(3)
    for k in (1, 5, 10):
        s = rng.integers(0, 9, size=300)
        out = subprocess.run([RL, str(k)], input=" ".join(map(str, s)), capture_output=True,
                             text=True, check=True).stdout.split()
        got = [(int(out[i]), int(out[i + 1])) for i in range(0, len(out), 2)]
        assert got == _result_list_model(s, k)


def write_fasta(path, records, prefix):
    with open(path, "w") as f:
        for i, r in enumerate(records):
            f.write(f">{prefix}{i} synthetic\n")
            seq = param.decode(r)
            for j in range(0, len(seq), 60):
                f.write(seq[j:j + 60] + "\n")


@pytest.mark.gpu
def test_worker_pool_end_to_end(tmp_path):
    rng = np.random.default_rng(17)
    db = synth.small_db(21, 1500)
    q = synth.residues(rng, 420)
    db, _ = synth.plant_homologs(rng, db, q, 0.01)
    dbf, qf = tmp_path / "db.fa", tmp_path / "q.fa"
    write_fasta(dbf, [db.record(i) for i in range(db.n)], "rec")
    write_fasta(qf, [q], "query")
    out = subprocess.run([WP, "-q", str(qf), "-db", str(dbf), "-t", "10", "-g", "1"],
                         capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    hits = [tuple(map(int, ln.split()[1:3])) for ln in out.stdout.splitlines()
            if ln.startswith("HIT ")]
    want = oracle.search(q, db.residues, db.offsets, param.blosum62(), 12, 2)
    sc, idx = oracle.topk(want, 10)
    assert hits == list(zip(sc.tolist(), idx.tolist()))
    assert f"score {sc[0]} -- >rec{idx[0]} synthetic" in out.stdout


@pytest.mark.gpu
def test_worker_pool_from_db_image(tmp_path):
    """The same pool fed from a DB image made by the FASTA converter: same
    hits, titles from the image's title index (the header without '>')."""
    rng = np.random.default_rng(18)
    db = synth.small_db(22, 1200)
    q = synth.residues(rng, 300)
    db, _ = synth.plant_homologs(rng, db, q, 0.01)
    dbf, qf, img = tmp_path / "db.fa", tmp_path / "q.fa", tmp_path / "db.swdb"
    write_fasta(dbf, [db.record(i) for i in range(db.n)], "rec")
    write_fasta(qf, [q], "query")
    capi.fasta_to_image(str(dbf), str(img))
    out = subprocess.run([WP, "-q", str(qf), "-db", str(img), "-t", "10", "-g", "1"],
                         capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    hits = [tuple(map(int, ln.split()[1:3])) for ln in out.stdout.splitlines()
            if ln.startswith("HIT ")]
    want = oracle.search(q, db.residues, db.offsets, param.blosum62(), 12, 2)
    sc, idx = oracle.topk(want, 10)
    assert hits == list(zip(sc.tolist(), idx.tolist()))
    assert f"score {sc[0]} -- rec{idx[0]} synthetic" in out.stdout
