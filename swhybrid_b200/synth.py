"""Seeded synthetic protein databases and queries for the benchmark workloads.

No public benchmark data is used.  Residues are drawn i.i.d. over the 20
standard amino acids from the background frequencies of Robinson & Robinson
(1991, PNAS 88:8880), the table BLAST uses for composition.  DB lengths are
lognormal and clipped; optional planted long records and planted homologs of a
query (substitutions at a uniform rate, indels at a fixed rate) stress the
overflow cascade.  Every generator takes an explicit seed and uses numpy's
PCG64 stream, so the same call gives the same bytes on every machine with the
same numpy.

Workloads (sizes as the benchmark definitions give them):
  small      20,000 records, lognormal(5.6, 0.6) clipped 20..5,000, query 375
  full       570,000 records, lognormal(5.6, 0.7) clipped 10..35,000, plus 200
             planted records uniform on 10,000..35,000 (~205 M residues);
             20 query lengths log-spaced 144..5,478
  batched    64 queries, lengths log-uniform on 50..5,000, over the full DB
  stress     100,000 records lognormal(5.6, 0.6) clipped 20..5,000, plus 1 %
             long records uniform 10,000..40,000, 0.5 % planted homologs of a
             query (substitution rate U(10 %, 30 %), indel rate 2 %); 8 queries
             of lengths 500..4,000
  serving    request lengths log-uniform on 30..8,000, Poisson arrivals
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .param import ALPHABET

# Robinson & Robinson (1991) background frequencies, one-letter code -> freq.
_RR91 = {
    "A": 0.07805, "R": 0.05129, "N": 0.04487, "D": 0.05364, "C": 0.01925,
    "Q": 0.04264, "E": 0.06295, "G": 0.07377, "H": 0.02199, "I": 0.05142,
    "L": 0.09019, "K": 0.05744, "M": 0.02243, "F": 0.03856, "P": 0.05203,
    "S": 0.07120, "T": 0.05841, "W": 0.01330, "Y": 0.03216, "V": 0.06441,
}
STANDARD = "ACDEFGHIKLMNPQRSTVWY"


def _lut16() -> np.ndarray:
    """65,536-entry table mapping a uniform uint16 to a residue code."""
    codes = np.array([ALPHABET.index(a) for a in STANDARD], dtype=np.uint8)
    p = np.array([_RR91[a] for a in STANDARD], dtype=np.float64)
    p /= p.sum()
    edges = np.round(np.cumsum(p) * 65536).astype(np.int64)
    edges[-1] = 65536
    lut = np.empty(65536, dtype=np.uint8)
    start = 0
    for c, e in zip(codes, edges):
        lut[start:e] = c
        start = e
    return lut


_LUT = _lut16()


def residues(rng: np.random.Generator, n: int) -> np.ndarray:
    out = np.empty(n, dtype=np.uint8)
    step = 1 << 26
    for s in range(0, n, step):
        e = min(n, s + step)
        out[s:e] = _LUT[rng.integers(0, 65536, size=e - s, dtype=np.uint16)]
    return out


def lognormal_lengths(rng, n, mu, sigma, lo, hi) -> np.ndarray:
    ln = np.rint(rng.lognormal(mu, sigma, size=n))
    return np.clip(ln, lo, hi).astype(np.int64)


@dataclass
class DB:
    residues: np.ndarray     # uint8 codes, all records back to back
    offsets: np.ndarray      # uint64, n+1 entries

    @property
    def n(self) -> int:
        return len(self.offsets) - 1

    @property
    def total(self) -> int:
        return int(self.offsets[-1])

    def lengths(self) -> np.ndarray:
        return np.diff(self.offsets.astype(np.int64))

    def record(self, i: int) -> np.ndarray:
        return self.residues[self.offsets[i]:self.offsets[i + 1]]

    def subset(self, idx) -> "DB":
        idx = np.asarray(idx, dtype=np.int64)
        lens = self.lengths()[idx]
        off = np.zeros(len(idx) + 1, dtype=np.uint64)
        off[1:] = np.cumsum(lens)
        res = np.concatenate([self.record(int(i)) for i in idx]) if len(idx) else np.zeros(0, np.uint8)
        return DB(res.astype(np.uint8), off)


def db_from_lengths(rng, lengths: np.ndarray) -> DB:
    lengths = np.asarray(lengths, dtype=np.int64)
    off = np.zeros(len(lengths) + 1, dtype=np.uint64)
    off[1:] = np.cumsum(lengths)
    return DB(residues(rng, int(off[-1])), off)


def mutate(rng, seq: np.ndarray, sub_rate: float, indel_rate: float) -> np.ndarray:
    """Homolog of ``seq``: substitutions at ``sub_rate``, then insertions and
    deletions, each at ``indel_rate / 2`` per position."""
    s = seq.copy()
    sub = rng.random(len(s)) < sub_rate
    s[sub] = residues(rng, int(sub.sum()))
    out = []
    for c in s:
        r = rng.random()
        if r < indel_rate / 2:
            continue                      # deletion
        out.append(c)
        if r > 1.0 - indel_rate / 2:
            out.append(residues(rng, 1)[0])  # insertion
    return np.array(out, dtype=np.uint8)


def plant_homologs(rng, db: DB, query: np.ndarray, rate: float,
                   indel_rate: float = 0.02, sub_lo: float = 0.10,
                   sub_hi: float = 0.30):
    """Replace a ``rate`` fraction of records with homologs of ``query``.
    Returns the new DB and the sorted indices of the planted records."""
    n = db.n
    k = max(1, int(round(rate * n)))
    picks = np.sort(rng.choice(n, size=k, replace=False))
    recs = [db.record(i) for i in range(n)]
    for i in picks:
        recs[i] = mutate(rng, query, rng.uniform(sub_lo, sub_hi), indel_rate)
    lens = np.array([len(r) for r in recs], dtype=np.int64)
    off = np.zeros(n + 1, dtype=np.uint64)
    off[1:] = np.cumsum(lens)
    return DB(np.concatenate(recs).astype(np.uint8), off), picks


def small_db(seed: int = 1, n: int = 20_000) -> DB:
    rng = np.random.default_rng(seed)
    return db_from_lengths(rng, lognormal_lengths(rng, n, 5.6, 0.6, 20, 5000))


def full_db(seed: int = 2, n: int = 570_000, n_long: int = 200) -> DB:
    rng = np.random.default_rng(seed)
    lens = lognormal_lengths(rng, n, 5.6, 0.7, 10, 35_000)
    long = rng.integers(10_000, 35_001, size=n_long)
    lens = np.concatenate([lens, long])
    lens = lens[rng.permutation(len(lens))]
    return db_from_lengths(rng, lens)


def stress_db(seed: int = 4, n: int = 100_000, query: np.ndarray | None = None):
    rng = np.random.default_rng(seed)
    lens = lognormal_lengths(rng, n, 5.6, 0.6, 20, 5000)
    n_long = n // 100
    long = rng.integers(10_000, 40_001, size=n_long)
    lens = np.concatenate([lens, long])
    lens = lens[rng.permutation(len(lens))]
    db = db_from_lengths(rng, lens)
    planted = np.zeros(0, dtype=np.int64)
    if query is not None:
        db, planted = plant_homologs(rng, db, query, 0.005)
    return db, planted


def query(seed: int, length: int) -> np.ndarray:
    return residues(np.random.default_rng(seed), int(length))


def sweep_lengths(n: int = 20, lo: int = 144, hi: int = 5478) -> np.ndarray:
    return np.unique(np.rint(np.geomspace(lo, hi, n)).astype(np.int64))


def loguniform_lengths(rng, n: int, lo: int, hi: int) -> np.ndarray:
    return np.rint(np.exp(rng.uniform(np.log(lo), np.log(hi), size=n))).astype(np.int64)


def batched_queries(seed: int = 3, n: int = 64, lo: int = 50, hi: int = 5000):
    rng = np.random.default_rng(seed)
    lens = loguniform_lengths(rng, n, lo, hi)
    return [residues(rng, int(L)) for L in lens]


def poisson_arrivals(rng, n: int, rate_per_s: float) -> np.ndarray:
    return np.cumsum(rng.exponential(1.0 / rate_per_s, size=n))


STRESS_QLENS = (500, 700, 1000, 1400, 1900, 2500, 3200, 4000)


def stress_workload(seed: int = 4, n: int = 100_000, homolog_rate: float = 0.005):
    """Overflow / long-record stress: ``stress_db`` records, eight queries of
    500..4,000 residues, and ``homolog_rate`` of the records replaced by
    homologs of the queries (an equal share each; substitutions uniform on
    10..30 %, indels 2 %).  Returns (db, queries, planted record ids, owner
    query of each planted id)."""
    rng = np.random.default_rng(seed)
    queries = [residues(rng, L) for L in STRESS_QLENS]
    db, _ = stress_db(seed, n)
    per_q = max(1, int(round(homolog_rate * db.n / len(queries))))
    picks = rng.choice(db.n, size=per_q * len(queries), replace=False)
    recs = [db.record(i) for i in range(db.n)]
    owner = {}
    for j, i in enumerate(picks):
        q = j // per_q
        recs[i] = mutate(rng, queries[q], rng.uniform(0.10, 0.30), 0.02)
        owner[int(i)] = q
    lens = np.array([len(r) for r in recs], dtype=np.int64)
    off = np.zeros(db.n + 1, dtype=np.uint64)
    off[1:] = np.cumsum(lens)
    return DB(np.concatenate(recs).astype(np.uint8), off), queries, np.sort(picks), owner
