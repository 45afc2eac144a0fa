"""The reference-side binding under the reference's own driver loop.

integration/_ref/ref_worker_pool links the reference's Worker, DataPool,
Param and RecalcWorker (compiled unchanged from its sources by
integration/Makefile) with integration/B200Worker.cpp, a Worker subclass over
libswb200; integration/_ref/dbmaker is the reference's DBmaker.  The test
writes a FASTA file, turns it into the reference's .seq/.map/.title DB with
that DBmaker, and runs one search: Worker::launch pulls chunks through
DataPool::fillChunk, B200Worker scores each chunk on the GPU, the base
Worker::auxWork pushes the scores into the worker's ResultList, and the
driver merges lists as WorkerPool does.  The DB is larger than DataPool's
32 MiB chunk, so the double-buffered chunk loop runs more than once.

Every length bucket holds whole 128-record batches: DBmaker corrupts records
of mixed-length batches (it inserts padding at offsets counted from the start
of the accumulated batch string), so only full batches keep the records
intact.  Hits are compared with the oracle by title (the FASTA position), as
the reference's hit index is a position in its own length-bucketed file."""
import os
import subprocess

import numpy as np
import pytest

import oracle
from swhybrid_b200 import param, synth

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "integration", "_ref")
ALPHA = "ABCDEFGHIKLMNPQRSTVWXYZ"


def _text(codes):
    return "".join(ALPHA[c] for c in codes)


def _make_db(rng, q, n_buckets):
    recs = []
    lens = np.clip(np.rint(rng.lognormal(5.6, 0.6, size=n_buckets)), 24, 3000).astype(int) // 4 * 4
    for L in lens:
        recs += [synth.residues(rng, int(L) - int(rng.integers(0, 4))) for _ in range(128)]
    # one bucket at the query's padded length holds 40 homologs of the query
    # (substitutions only, so their lengths stay in the bucket)
    Lq = (len(q) + 3) // 4 * 4
    for i in range(128):
        if i < 40:
            recs.append(synth.mutate(rng, q, 0.1 + 0.005 * i, 0.0))
        else:
            recs.append(synth.residues(rng, Lq - int(rng.integers(0, 4))))
    order = rng.permutation(len(recs))
    return [recs[i] for i in order]


@pytest.mark.skipif(not os.path.exists(os.path.join(BIN, "ref_worker_pool")),
                    reason="integration/_ref not built (needs the reference sources at build time)")
def test_b200_worker_under_reference_worker_launch(tmp_path):
    rng = np.random.default_rng(77)
    q = synth.residues(rng, 301)
    recs = _make_db(rng, q, 900)
    fa = tmp_path / "db.fa"
    with open(fa, "w") as f:
        for i, r in enumerate(recs):
            f.write(f">r{i}\n{_text(r)}\n")
    qf = tmp_path / "q.fa"
    qf.write_text(">query\n" + _text(q) + "\n")
    total = sum(len(r) for r in recs)
    assert total > 33 * 2**20          # more than one of DataPool's chunks

    out = subprocess.run([os.path.join(BIN, "dbmaker"), str(fa), str(tmp_path / "db")],
                         capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    out = subprocess.run([os.path.join(BIN, "ref_worker_pool"), "-q", str(qf), "-db",
                          str(tmp_path / "db"), "-t", "10", "-g", "1"],
                         capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout[-3000:] + out.stderr[-3000:]
    lines = out.stdout.splitlines()
    hits = [ln.split() for ln in lines if ln.startswith("hit ")]
    summary = [ln for ln in lines if ln.startswith("records ")][0].split()
    assert int(summary[1]) == len(recs)          # every record scored once
    assert int(summary[3]) == 0                  # nothing left for RecalcWorker

    off = np.zeros(len(recs) + 1, dtype=np.uint64)
    off[1:] = np.cumsum([len(r) for r in recs])
    want = oracle.search(q, np.concatenate(recs).astype(np.uint8), off, param.blosum62(), 12, 2)
    top = np.sort(want)[::-1][:10]
    assert [int(h[1]) for h in hits] == top.tolist()
    for h in hits:                   # DataPool::getTitle gives the header line, '>' included
        title = h[3].lstrip(">")
        assert title.startswith("r"), h
        assert want[int(title[1:])] == int(h[1]), h
    assert top[-1] >= 117      # the hits overflow the reference's int8 pass
