"""Generates the golden score vectors under tests/golden/ with the reference's
own kernels (SWhybrid src/AVXKernel.cpp: avxCompute int8 pass + avxCompute16
int16 recalc), compiled from the reference sources into oracle/_ref by
oracle/Makefile and driven by oracle/ref_harness.cpp.

Run in a checkout where oracle/_ref/libswref.so has been built:
    python tests/golden/make_golden.py
Inputs are seeded synthetic records (swhybrid_b200.synth); the small ones are
stored with their scores, the 20,000-record set is stored as a digest of its
inputs plus its scores.
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from swhybrid_b200 import param, synth  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
EDGE_LENGTHS = [1, 2, 3, 4, 5, 7, 8, 9, 15, 16, 17, 31, 32, 33, 63, 64, 65, 127, 128,
                129, 255, 256, 300, 511, 512, 513, 1000, 1023, 1024, 1025, 2047, 2048,
                2049, 4096, 6000]
EDGE_QUERIES = [1, 3, 4, 8, 31, 32, 33, 144, 375, 513, 1025, 2100]


def digest(*arrays) -> str:
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def all_codes_record(rng, n):
    """Records over all 23 alphabet codes (incl. B, X, Z), no '@'."""
    return rng.integers(0, 23, size=n).astype(np.uint8)


def edge_set():
    rng = np.random.default_rng(11)
    lens = list(EDGE_LENGTHS) + list(rng.integers(1, 700, size=60))
    recs = [synth.residues(rng, int(L)) for L in lens]
    recs += [all_codes_record(rng, int(L)) for L in (17, 250, 999)]
    recs.append(np.zeros(0, dtype=np.uint8))          # empty record
    lens = np.array([len(r) for r in recs], dtype=np.int64)
    off = np.zeros(len(recs) + 1, dtype=np.uint64)
    off[1:] = np.cumsum(lens)
    res = np.concatenate(recs).astype(np.uint8)
    queries = [synth.residues(rng, L) for L in EDGE_QUERIES]
    queries.append(all_codes_record(rng, 200))
    return res, off, queries


def homolog_set():
    rng = np.random.default_rng(12)
    q375 = synth.residues(rng, 375)
    q1000 = synth.residues(rng, 1000)
    base = synth.db_from_lengths(rng, synth.lognormal_lengths(rng, 1500, 5.6, 0.6, 20, 5000))
    db, p1 = synth.plant_homologs(rng, base, q375, 0.01)
    db, p2 = synth.plant_homologs(rng, db, q1000, 0.01)
    return db.residues, db.offsets, [q375, q1000]


def saturation_set():
    W = param.encode("W")[0]
    recs = [np.full(n, W, dtype=np.uint8) for n in (100, 2000, 2977, 2978, 2979, 2980, 4000, 6000)]
    lens = np.array([len(r) for r in recs], dtype=np.int64)
    off = np.zeros(len(recs) + 1, dtype=np.uint64)
    off[1:] = np.cumsum(lens)
    res = np.concatenate(recs)
    queries = [np.full(n, W, dtype=np.uint8) for n in (2977, 2978, 2979, 2980, 4000, 6000)]
    return res, off, queries


def run(res, off, queries):
    m = param.blosum62()
    out = []
    for q in queries:
        s, _, _ = oracle.ref_search(q, res, off, m, 10, 2)
        out.append(s)
    return out


def write_set(name, res, off, queries):
    scores = run(res, off, queries)
    qoff = np.zeros(len(queries) + 1, dtype=np.uint64)
    qoff[1:] = np.cumsum([len(q) for q in queries])
    np.savez_compressed(os.path.join(OUT, f"{name}.npz"), residues=res, offsets=off,
                        queries=np.concatenate(queries).astype(np.uint8), qoffsets=qoff,
                        scores=np.stack(scores).astype(np.int32))
    print(name, len(off) - 1, "records,", len(queries), "queries")


def main():
    if not oracle.ref_available():
        oracle.build()
    write_set("edge", *edge_set())
    write_set("homolog", *homolog_set())
    write_set("saturation", *saturation_set())
    db = synth.small_db(1, 20_000)
    q = synth.query(375, 375)
    s, _, _ = oracle.ref_search(q, db.residues, db.offsets, param.blosum62(), 10, 2)
    np.savez_compressed(os.path.join(OUT, "small20k_q375.npz"),
                        input_digest=np.array(digest(db.residues, db.offsets, q)),
                        scores=s.astype(np.int32))
    print("small20k_q375", db.n, "records, residues", db.total)


if __name__ == "__main__":
    main()
