"""Oracle loader -- TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
import this package.  It wraps:

* ``liboracle.so``: the C restatement of the reference scoring path
  (``oracle/gotoh.c``; scalar int64 Gotoh and the reference's int8 + int16
  cascade semantics);
* ``_ref/libswref.so``: the reference's own ``src/AVXKernel.cpp`` kernels
  (``avxCompute`` + ``avxCompute16``) compiled from the reference sources by
  ``oracle/Makefile`` and driven by ``oracle/ref_harness.cpp``.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(HERE, "liboracle.so")
_REF = os.path.join(HERE, "_ref", "libswref.so")

_c_i64 = ctypes.c_int64
_c_i32 = ctypes.c_int32
_ptr = ctypes.c_void_p


def reference_root() -> str:
    """The read-only reference source tree: the SWHYBRID_REF environment
    variable, by default the checkout this container mounts."""
    return os.environ.get("SWHYBRID_REF", "/root/reference")


def build(quiet: bool = True) -> None:
    """Compile the C restatement and, when the reference tree is present,
    the reference kernels."""
    out = subprocess.run(["make", "-C", HERE, f"SWHYBRID_REF={reference_root()}"],
                         capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    if not quiet:
        print(out.stdout)


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        _lib = ctypes.CDLL(_LIB)
        _lib.oracle_gotoh.restype = _c_i64
        _lib.oracle_gotoh.argtypes = [_ptr, _c_i64, _ptr, _c_i64, _ptr, _c_i32, _c_i32]
        _lib.oracle_reference_score.restype = _c_i64
        _lib.oracle_reference_score.argtypes = [_ptr, _c_i64, _ptr, _c_i64, _ptr, _c_i32, _c_i32]
        _lib.oracle_search.restype = None
        _lib.oracle_search.argtypes = [_ptr, _c_i64, _ptr, _ptr, _c_i64, _ptr, _c_i32,
                                       _c_i32, _c_i32, _c_i32, _ptr]
        _lib.oracle_topk.restype = _c_i32
        _lib.oracle_topk.argtypes = [_ptr, _c_i64, _c_i32, _ptr, _ptr]
        _lib.oracle_traceback.restype = _c_i64
        _lib.oracle_traceback.argtypes = [_ptr, _c_i64, _ptr, _c_i64, _ptr, _c_i32, _c_i32,
                                          _ptr, _ptr, _c_i64]
    return _lib


def ref_available() -> bool:
    return os.path.exists(_REF)


def ref():
    global _ref
    if _ref is None:
        if not os.path.exists(_REF):
            raise FileNotFoundError(
                "oracle/_ref/libswref.so is missing (built from the reference "
                "sources by `make -C oracle`)")
        _ref = ctypes.CDLL(_REF)
        _ref.swref_search.restype = ctypes.c_int
        _ref.swref_search.argtypes = [_ptr, _c_i64, _ptr, _ptr, _c_i64, _ptr, _c_i32,
                                      _c_i32, _c_i32, _ptr, ctypes.POINTER(ctypes.c_double),
                                      ctypes.POINTER(ctypes.c_int64)]
        _ref.swref_max_threads.restype = ctypes.c_int
        _ref.swref_db_pack.restype = ctypes.c_void_p
        _ref.swref_db_pack.argtypes = [_ptr, _ptr, _c_i64]
        _ref.swref_db_free.restype = None
        _ref.swref_db_free.argtypes = [ctypes.c_void_p]
        _ref.swref_db_search.restype = ctypes.c_int
        _ref.swref_db_search.argtypes = [ctypes.c_void_p, _ptr, _c_i64, _ptr, _c_i32, _c_i32,
                                         _c_i32, _ptr, ctypes.POINTER(ctypes.c_double),
                                         ctypes.POINTER(ctypes.c_int64)]
    return _ref


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def _mat(matrix) -> np.ndarray:
    m = np.ascontiguousarray(np.asarray(matrix, dtype=np.int32).reshape(32, 32))
    return m


def gotoh(q, d, matrix, gap_oe=12, gap_e=2) -> int:
    q = np.ascontiguousarray(q, dtype=np.uint8)
    d = np.ascontiguousarray(d, dtype=np.uint8)
    m = _mat(matrix)
    return int(lib().oracle_gotoh(_p(q), len(q), _p(d), len(d), _p(m), gap_oe, gap_e))


def search(query, residues, offsets, matrix, gap_oe=12, gap_e=2, mode=1,
           threads=0) -> np.ndarray:
    """Scores of every record (input order).  mode 1 = the reference's
    reported scores (int8 pass + int16 recalc), mode 0 = exact Gotoh."""
    q = np.ascontiguousarray(query, dtype=np.uint8)
    r = np.ascontiguousarray(residues, dtype=np.uint8)
    o = np.ascontiguousarray(offsets, dtype=np.uint64)
    m = _mat(matrix)
    n = len(o) - 1
    out = np.zeros(max(n, 1), dtype=np.int32)
    lib().oracle_search(_p(q), len(q), _p(r), _p(o), n, _p(m), gap_oe, gap_e,
                        mode, threads, _p(out))
    return out[:n]


OPS = "MID"


def traceback(q, d, matrix, gap_oe=12, gap_e=2):
    """Best local alignment of q against d under the library's traceback
    rules: dict(score, q_begin, q_end, d_begin, d_end, cigar)."""
    q = np.ascontiguousarray(q, dtype=np.uint8)
    d = np.ascontiguousarray(d, dtype=np.uint8)
    m = _mat(matrix)
    out = np.zeros(5, dtype=np.int64)
    cap = len(q) + len(d) + 1
    ops = np.zeros(cap, dtype=np.uint8)
    n = lib().oracle_traceback(_p(q), len(q), _p(d), len(d), _p(m), gap_oe, gap_e, _p(out),
                               _p(ops), cap)
    assert n >= 0
    return dict(score=int(out[0]), q_begin=int(out[1]), q_end=int(out[2]),
                d_begin=int(out[3]), d_end=int(out[4]), cigar=cigar(ops[:n]))


def cigar(ops) -> str:
    """Run-length CIGAR text of a per-column op sequence (0 M, 1 I, 2 D)."""
    out, prev, run = [], None, 0
    for o in list(ops) + [None]:
        if o == prev:
            run += 1
            continue
        if prev is not None:
            out.append(f"{run}{OPS[prev]}")
        prev, run = o, 1
    return "".join(out)


def topk(scores, k):
    s = np.ascontiguousarray(scores, dtype=np.int32)
    os_ = np.zeros(max(k, 1), dtype=np.int32)
    oi = np.zeros(max(k, 1), dtype=np.int64)
    m = lib().oracle_topk(_p(s), len(s), k, _p(os_), _p(oi))
    return os_[:m], oi[:m]


def ref_search(query, residues, offsets, matrix, gap_open=10, gap_extend=2,
               threads=0):
    """The reference's own kernels on this DB.  Returns (scores, kernel
    seconds, number of records re-scored in int16)."""
    q = np.ascontiguousarray(query, dtype=np.uint8)
    r = np.ascontiguousarray(residues, dtype=np.uint8)
    o = np.ascontiguousarray(offsets, dtype=np.uint64)
    m = _mat(matrix)
    n = len(o) - 1
    out = np.zeros(max(n, 1), dtype=np.int32)
    secs = ctypes.c_double(0.0)
    novf = ctypes.c_int64(0)
    rc = ref().swref_search(_p(q), len(q), _p(r), _p(o), n, _p(m), gap_open,
                            gap_extend, threads, _p(out), ctypes.byref(secs),
                            ctypes.byref(novf))
    if rc != 0:
        raise RuntimeError(f"swref_search failed: {rc}")
    return out[:n], secs.value, novf.value


class RefDB:
    """A DB packed once for the reference kernels; search() per query."""

    def __init__(self, residues, offsets):
        self._r = np.ascontiguousarray(residues, dtype=np.uint8)
        self._o = np.ascontiguousarray(offsets, dtype=np.uint64)
        self.n = len(self._o) - 1
        self.h = ref().swref_db_pack(_p(self._r), _p(self._o), self.n)

    def search(self, query, matrix, gap_open=10, gap_extend=2, threads=0):
        q = np.ascontiguousarray(query, dtype=np.uint8)
        m = _mat(matrix)
        out = np.zeros(max(self.n, 1), dtype=np.int32)
        secs = ctypes.c_double(0.0)
        novf = ctypes.c_int64(0)
        rc = ref().swref_db_search(self.h, _p(q), len(q), _p(m), gap_open, gap_extend,
                                   threads, _p(out), ctypes.byref(secs), ctypes.byref(novf))
        if rc != 0:
            raise RuntimeError(f"swref_db_search failed: {rc}")
        return out[:self.n], secs.value, novf.value

    def close(self):
        if self.h:
            ref().swref_db_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def ref_threads() -> int:
    return int(ref().swref_max_threads())
