"""Search parameters and residue encoding (mirror of SWhybrid's ``Param``).

Reference: ``src/Param.h:8-51`` (the BLOSUM62 table in the 23-letter alphabet
``ABCDEFGHIKLMNPQRSTVWXYZ`` plus code 23 for ``@``, rows/columns 23..31 zero),
``src/Param.h:59-117`` (defaults gapOpen 10, gapExtend 2, topNum 10,
``gapOE = gapOpen + gapExtend``) and ``src/DataPool.cpp:33-47`` (letter to
code translation; letters outside the alphabet map to -1 there).

Codes on this side: 0..22 for the alphabet, 23 for ``@``, and 24 for every
letter the reference maps to -1 (J, O, U, ``*`` ...).  Code 24 scores 0
against everything, which is what the reference's int8 kernel does for -1
(its byte shuffle returns 0 for an index with the high bit set).
"""
from __future__ import annotations

import numpy as np

ALPHABET = "ABCDEFGHIKLMNPQRSTVWXYZ"
PAD_CODE = 23          # '@', padding code of the reference (scores 0 in BLOSUM62)
UNKNOWN_CODE = 24      # letters the reference maps to -1

# BLOSUM62 (Henikoff & Henikoff 1992), classic table with the X row as shipped
# by the reference, in the reference's alphabet order.  A substitution matrix
# is data that must be identical to be the same search; tests compare it with
# the reference's table.
_B62_ROWS = """
A  4 -2  0 -2 -1 -2  0 -2 -1 -1 -1 -1 -2 -1 -1 -1  1  0  0 -3  0 -2 -1
B -2  4 -3  4  1 -3 -1  0 -3  0 -4 -3  3 -2  0 -1  0 -1 -3 -4 -1 -3  1
C  0 -3  9 -3 -4 -2 -3 -3 -1 -3 -1 -1 -3 -3 -3 -3 -1 -1 -1 -2 -2 -2 -3
D -2  4 -3  6  2 -3 -1 -1 -3 -1 -4 -3  1 -1  0 -2  0 -1 -3 -4 -1 -3  1
E -1  1 -4  2  5 -3 -2  0 -3  1 -3 -2  0 -1  2  0  0 -1 -2 -3 -1 -2  4
F -2 -3 -2 -3 -3  6 -3 -1  0 -3  0  0 -3 -4 -3 -3 -2 -2 -1  1 -1  3 -3
G  0 -1 -3 -1 -2 -3  6 -2 -4 -2 -4 -3  0 -2 -2 -2  0 -2 -3 -2 -1 -3 -2
H -2  0 -3 -1  0 -1 -2  8 -3 -1 -3 -2  1 -2  0  0 -1 -2 -3 -2 -1  2  0
I -1 -3 -1 -3 -3  0 -4 -3  4 -3  2  1 -3 -3 -3 -3 -2 -1  3 -3 -1 -1 -3
K -1  0 -3 -1  1 -3 -2 -1 -3  5 -2 -1  0 -1  1  2  0 -1 -2 -3 -1 -2  1
L -1 -4 -1 -4 -3  0 -4 -3  2 -2  4  2 -3 -3 -2 -2 -2 -1  1 -2 -1 -1 -3
M -1 -3 -1 -3 -2  0 -3 -2  1 -1  2  5 -2 -2  0 -1 -1 -1  1 -1 -1 -1 -1
N -2  3 -3  1  0 -3  0  1 -3  0 -3 -2  6 -2  0  0  1  0 -3 -4 -1 -2  0
P -1 -2 -3 -1 -1 -4 -2 -2 -3 -1 -3 -2 -2  7 -1 -2 -1 -1 -2 -4 -2 -3 -1
Q -1  0 -3  0  2 -3 -2  0 -3  1 -2  0  0 -1  5  1  0 -1 -2 -2 -1 -1  3
R -1 -1 -3 -2  0 -3 -2  0 -3  2 -2 -1  0 -2  1  5 -1 -1 -3 -3 -1 -2  0
S  1  0 -1  0  0 -2  0 -1 -2  0 -2 -1  1 -1  0 -1  4  1 -2 -3  0 -2  0
T  0 -1 -1 -1 -1 -2 -2 -2 -1 -1 -1 -1  0 -1 -1 -1  1  5  0 -2  0 -2 -1
V  0 -3 -1 -3 -2 -1 -3 -3  3 -2  1  1 -3 -2 -2 -3 -2  0  4 -3 -1 -1 -2
W -3 -4 -2 -4 -3  1 -2 -2 -3 -3 -2 -1 -4 -4 -2 -3 -3 -2 -3 11 -2  2 -3
X  0 -1 -2 -1 -1 -1 -1 -1 -1 -1 -1 -1 -1 -2 -1 -1  0  0 -1 -2 -1 -1 -1
Y -2 -3 -2 -3 -2  3 -3  2 -1 -2 -1 -1 -2 -3 -1 -2 -2 -2 -1  2 -1  7 -2
Z -1  1 -3  1  4 -3 -2  0 -3  1 -3 -1  0 -1  3  0  0 -1 -2 -3 -1 -2  4
"""


def blosum62() -> np.ndarray:
    """The 32x32 int32 BLOSUM62 matrix in reference code order."""
    m = np.zeros((32, 32), dtype=np.int32)
    rows = [ln.split() for ln in _B62_ROWS.strip().splitlines()]
    for i, r in enumerate(rows):
        assert r[0] == ALPHABET[i]
        m[i, :23] = [int(x) for x in r[1:]]
    return m


def _make_trans() -> np.ndarray:
    t = np.full(256, UNKNOWN_CODE, dtype=np.uint8)
    for i, ch in enumerate(ALPHABET):
        t[ord(ch)] = i
        t[ord(ch.lower())] = i
    t[ord("@")] = PAD_CODE
    return t


TRANS = _make_trans()


def encode(seq: str | bytes) -> np.ndarray:
    """Letters to residue codes (``DataPool.cpp:33-47``; unknown -> 24)."""
    if isinstance(seq, str):
        seq = seq.encode("ascii")
    return TRANS[np.frombuffer(seq, dtype=np.uint8)]


def decode(codes: np.ndarray) -> str:
    out = []
    for c in np.asarray(codes, dtype=np.int64):
        out.append(ALPHABET[c] if c < 23 else ("@" if c == PAD_CODE else "?"))
    return "".join(out)


class Param:
    """Search parameters, same names and defaults as the reference's ``Param``.

    ``Param(argv)`` accepts the reference's switches ``-o`` (gap open),
    ``-e`` (gap extend), ``-t`` (top-k), ``-q`` (query path), ``-db`` (DB path)
    and ``-g`` (GPU count); ``gapOE`` is ``gapOpen + gapExtend``.
    """

    def __init__(self, argv: list[str] | None = None, *, gapOpen: int = 10,
                 gapExtend: int = 2, topNum: int = 10):
        self.gapOpen = gapOpen
        self.gapExtend = gapExtend
        self.topNum = topNum
        self.queryPath = None
        self.dbPath = None
        self.cudaNum = -1
        argv = list(argv or [])
        i = 1 if argv and not argv[0].startswith("-") else 0
        while i < len(argv):
            a = argv[i]
            if a.startswith("-") and len(a) >= 2:
                val = argv[i + 1] if i + 1 < len(argv) else None
                if val is None:
                    raise ValueError(f"switch {a} needs a value")
                key = a[1]
                if key == "o":
                    self.gapOpen = int(val)
                elif key == "e":
                    self.gapExtend = int(val)
                elif key == "t":
                    self.topNum = int(val)
                elif key == "g":
                    self.cudaNum = int(val)
                elif key == "q":
                    self.queryPath = val
                elif key == "d" and a[2:3] == "b":
                    self.dbPath = val
                elif key in ("c", "p"):
                    pass  # CPU / coprocessor counts have no meaning here
                else:
                    raise ValueError(f"unknown switch {a}")
                i += 2
            else:
                i += 1
        self.matrix = blosum62()

    @property
    def gapOE(self) -> int:
        return self.gapOpen + self.gapExtend

    @property
    def plain_matrix(self) -> np.ndarray:
        return self.matrix.reshape(-1).astype(np.int32)
