"""ctypes binding of libswb200.so (declarations in include/swb200.h).

The library is built in place (``swhybrid_b200/libswb200.so``) by
``swhybrid_b200.build``.  There is no CPU fallback: when the library or a CUDA
device is missing, the calls raise.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libswb200.so")

SW_OK = 0
SW_ERR_UNSUPPORTED = 6
STATUS = {
    0: "SW_OK", 1: "SW_ERR_INVALID", 2: "SW_ERR_CUDA", 3: "SW_ERR_NOMEM",
    4: "SW_ERR_STATE", 5: "SW_ERR_FORMAT", 6: "SW_ERR_UNSUPPORTED",
    7: "SW_ERR_BUSY", 8: "SW_ERR_TIMEOUT", 9: "SW_ERR_NO_DEVICE",
}
SW_FLAG_REFERENCE_CAP = 1

# Every entry point include/swb200.h declares (checked by the CPU tests).
EXPORTS = [
    "sw_params_default", "sw_encode", "sw_ctx_create", "sw_ctx_destroy",
    "sw_last_error", "sw_db_load", "sw_db_stats_get", "sw_search",
    "sw_search_device", "sw_set_kernel_config", "sw_get_kernel_config", "sw_get_plan",
    "sw_get_run_stats", "sw_set_stream", "sw_sync", "sw_reset_totals", "sw_get_totals",
    "sw_set_tuning", "sw_score_noalloc", "sw_get_shapes", "sw_set_batch_options",
    "sw_search_batch", "sw_serve_options_default", "sw_serve_start", "sw_serve_submit",
    "sw_serve_poll", "sw_serve_get_stats", "sw_serve_clock_ms", "sw_serve_stop",
    "sw_traceback", "sw_db_write_image", "sw_fasta_to_image", "sw_image_get_info",
    "sw_db_load_image", "sw_db_title", "sw_params_parse_matrix", "sw_params_load_matrix",
    "sw_image_open", "sw_image_close",
]


class SwError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


class sw_params(ctypes.Structure):
    _fields_ = [("matrix", ctypes.c_int32 * 1024), ("gap_open", ctypes.c_int32),
                ("gap_extend", ctypes.c_int32), ("top_k", ctypes.c_int32),
                ("flags", ctypes.c_uint32)]


class sw_hit(ctypes.Structure):
    _fields_ = [("score", ctypes.c_int32), ("reserved", ctypes.c_uint32),
                ("index", ctypes.c_uint64)]


class sw_kernel_config(ctypes.Structure):
    _fields_ = [("long_group_width", ctypes.c_int32), ("long_rows_per_thread", ctypes.c_int32),
                ("short_group_width", ctypes.c_int32), ("short_rows_per_thread", ctypes.c_int32),
                ("cutover", ctypes.c_int32)]

    def as_tuple(self):
        return (self.long_group_width, self.long_rows_per_thread, self.short_group_width,
                self.short_rows_per_thread, self.cutover)


class sw_batch_options(ctypes.Structure):
    _fields_ = [("cutover", ctypes.c_int32), ("long_group_width", ctypes.c_int32),
                ("long_rows_per_thread", ctypes.c_int32), ("use_graph", ctypes.c_int32),
                ("group_width", ctypes.c_int32), ("rows_per_thread", ctypes.c_int32),
                ("stack_rows", ctypes.c_int32), ("pair_rows", ctypes.c_int32),
                ("pair_group_width", ctypes.c_int32), ("pair_rows_per_thread", ctypes.c_int32),
                ("pair_long", ctypes.c_int32), ("pair_regions", ctypes.c_int32)]


class sw_image_info(ctypes.Structure):
    _fields_ = [("n_records", ctypes.c_uint64), ("n_residues", ctypes.c_uint64),
                ("file_bytes", ctypes.c_uint64), ("titles_bytes", ctypes.c_uint64),
                ("checksum", ctypes.c_uint64), ("version", ctypes.c_uint32),
                ("reserved", ctypes.c_uint32)]


class sw_alignment(ctypes.Structure):
    _fields_ = [("index", ctypes.c_uint64), ("score", ctypes.c_int32),
                ("q_begin", ctypes.c_uint32), ("q_end", ctypes.c_uint32),
                ("d_begin", ctypes.c_uint32), ("d_end", ctypes.c_uint32),
                ("matches", ctypes.c_uint32), ("n_ops", ctypes.c_uint32),
                ("reserved", ctypes.c_uint32), ("ops_offset", ctypes.c_uint64)]


class sw_serve_options(ctypes.Structure):
    _fields_ = [("max_active", ctypes.c_uint32), ("chunks", ctypes.c_uint32),
                ("max_pending", ctypes.c_uint32), ("memory_budget", ctypes.c_uint64),
                ("group_width", ctypes.c_int32), ("rows_per_thread", ctypes.c_int32),
                ("stack_rows", ctypes.c_int32), ("pair_rows", ctypes.c_int32),
                ("pair_group_width", ctypes.c_int32), ("pair_rows_per_thread", ctypes.c_int32),
                ("pair_long", ctypes.c_int32), ("pair_regions", ctypes.c_int32)]


class sw_serve_result(ctypes.Structure):
    _fields_ = [("request_id", ctypes.c_uint64), ("status", ctypes.c_int32),
                ("n_hits", ctypes.c_uint32), ("submit_ms", ctypes.c_double),
                ("start_ms", ctypes.c_double), ("done_ms", ctypes.c_double)]


class sw_serve_stats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_uint64), ("admitted", ctypes.c_uint64),
                ("completed", ctypes.c_uint64), ("failed", ctypes.c_uint64),
                ("rounds", ctypes.c_uint64), ("launches", ctypes.c_uint64),
                ("rescored", ctypes.c_uint64), ("cells", ctypes.c_uint64),
                ("busy_ms", ctypes.c_double), ("slots", ctypes.c_uint32),
                ("chunks", ctypes.c_uint32), ("active", ctypes.c_uint32),
                ("pending", ctypes.c_uint32), ("device_ms", ctypes.c_double)]


class sw_plan_step(ctypes.Structure):
    _fields_ = [("group_width", ctypes.c_int32), ("rows_per_thread", ctypes.c_int32),
                ("passes", ctypes.c_int32)]


PLAN_STEPS = 4     # SW_PLAN_STEPS


class sw_tuning_entry(ctypes.Structure):
    _fields_ = [("max_qlen", ctypes.c_uint32), ("cfg", sw_kernel_config),
                ("plan", sw_plan_step * PLAN_STEPS)]


class sw_db_stats(ctypes.Structure):
    _fields_ = [("n_records", ctypes.c_uint64), ("n_residues", ctypes.c_uint64),
                ("n_pairs", ctypes.c_uint64), ("max_length", ctypes.c_uint64),
                ("device_bytes", ctypes.c_uint64)]


class sw_totals(ctypes.Structure):
    _fields_ = [("first_pass_ms", ctypes.c_double), ("search_ms", ctypes.c_double),
                ("first_pass_launches", ctypes.c_uint64), ("launches", ctypes.c_uint64),
                ("cells", ctypes.c_uint64), ("queries", ctypes.c_uint64)]


class sw_run_stats(ctypes.Structure):
    _fields_ = [("kernel_ms", ctypes.c_double), ("first_pass_ms", ctypes.c_double),
                ("total_ms", ctypes.c_double),
                ("cells", ctypes.c_uint64), ("rescored", ctypes.c_uint64),
                ("launches", ctypes.c_uint32), ("queries", ctypes.c_uint32),
                ("used", sw_kernel_config), ("long_ms", ctypes.c_double),
                ("bulk_ms", ctypes.c_double)]


_lib = None


def load(path: str | None = None):
    """Load libswb200.so and declare every C-ABI signature.  The library
    built in this package is used unless SWB200_LIBRARY names another build
    of it (for comparing builds)."""
    global _lib
    if _lib is not None:
        return _lib
    if path is None:
        path = os.environ.get("SWB200_LIBRARY") or LIB_PATH
    if not os.path.exists(path):
        raise FileNotFoundError(
            f"{path} is missing: build it with `python -c 'import swhybrid_b200.build as b; b.build()'`")
    L = ctypes.CDLL(path)
    P = ctypes.c_void_p
    u8p = ctypes.POINTER(ctypes.c_uint8)
    L.sw_params_default.restype = None
    L.sw_params_default.argtypes = [ctypes.POINTER(sw_params)]
    L.sw_encode.restype = ctypes.c_int
    L.sw_encode.argtypes = [ctypes.c_char_p, ctypes.c_uint64, u8p]
    L.sw_ctx_create.restype = ctypes.c_int
    L.sw_ctx_create.argtypes = [ctypes.c_int, ctypes.POINTER(sw_params), ctypes.POINTER(P)]
    L.sw_ctx_destroy.restype = ctypes.c_int
    L.sw_ctx_destroy.argtypes = [P]
    L.sw_last_error.restype = ctypes.c_char_p
    L.sw_last_error.argtypes = [P]
    L.sw_db_load.restype = ctypes.c_int
    L.sw_db_load.argtypes = [P, P, P, ctypes.c_uint64]
    L.sw_db_stats_get.restype = ctypes.c_int
    L.sw_db_stats_get.argtypes = [P, ctypes.POINTER(sw_db_stats)]
    L.sw_search.restype = ctypes.c_int
    L.sw_search.argtypes = [P, P, ctypes.c_uint32, ctypes.POINTER(sw_hit),
                            ctypes.POINTER(ctypes.c_uint32), P]
    L.sw_search_device.restype = ctypes.c_int
    L.sw_search_device.argtypes = [P, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_void_p]
    L.sw_set_kernel_config.restype = ctypes.c_int
    L.sw_set_kernel_config.argtypes = [P, ctypes.POINTER(sw_kernel_config)]
    L.sw_get_kernel_config.restype = ctypes.c_int
    L.sw_get_kernel_config.argtypes = [P, ctypes.c_uint32, ctypes.POINTER(sw_kernel_config)]
    L.sw_get_run_stats.restype = ctypes.c_int
    L.sw_get_run_stats.argtypes = [P, ctypes.POINTER(sw_run_stats)]
    L.sw_set_stream.restype = ctypes.c_int
    L.sw_set_stream.argtypes = [P, ctypes.c_void_p]
    L.sw_sync.restype = ctypes.c_int
    L.sw_sync.argtypes = [P]
    L.sw_reset_totals.restype = ctypes.c_int
    L.sw_reset_totals.argtypes = [P]
    L.sw_get_totals.restype = ctypes.c_int
    L.sw_get_totals.argtypes = [P, ctypes.POINTER(sw_totals)]
    L.sw_set_tuning.restype = ctypes.c_int
    L.sw_set_tuning.argtypes = [P, ctypes.POINTER(sw_tuning_entry), ctypes.c_uint32]
    L.sw_set_batch_options.restype = ctypes.c_int
    L.sw_set_batch_options.argtypes = [P, ctypes.POINTER(sw_batch_options)]
    L.sw_search_batch.restype = ctypes.c_int
    L.sw_search_batch.argtypes = [P, ctypes.c_uint32, P, P, ctypes.POINTER(sw_hit),
                                  ctypes.POINTER(ctypes.c_uint32), P]
    L.sw_get_shapes.restype = ctypes.c_int
    L.sw_get_shapes.argtypes = [ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32),
                                ctypes.POINTER(ctypes.c_int32), ctypes.c_uint32,
                                ctypes.POINTER(ctypes.c_uint32)]
    L.sw_get_plan.restype = ctypes.c_int
    L.sw_get_plan.argtypes = [P, ctypes.c_uint32, ctypes.POINTER(sw_plan_step), ctypes.c_uint32,
                              ctypes.POINTER(ctypes.c_uint32)]
    L.sw_score_noalloc.restype = ctypes.c_int
    L.sw_score_noalloc.argtypes = [ctypes.c_int, ctypes.POINTER(sw_params), ctypes.c_void_p,
                                   ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p,
                                   ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p]
    L.sw_params_parse_matrix.restype = ctypes.c_int
    L.sw_params_parse_matrix.argtypes = [ctypes.POINTER(sw_params), ctypes.c_char_p]
    L.sw_params_load_matrix.restype = ctypes.c_int
    L.sw_params_load_matrix.argtypes = [ctypes.POINTER(sw_params), ctypes.c_char_p]
    L.sw_db_write_image.restype = ctypes.c_int
    L.sw_db_write_image.argtypes = [ctypes.c_char_p, P, P, ctypes.c_uint64, P, P]
    L.sw_fasta_to_image.restype = ctypes.c_int
    L.sw_fasta_to_image.argtypes = [ctypes.c_char_p, ctypes.c_char_p,
                                    ctypes.POINTER(sw_image_info)]
    L.sw_image_get_info.restype = ctypes.c_int
    L.sw_image_get_info.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(sw_image_info)]
    L.sw_db_load_image.restype = ctypes.c_int
    L.sw_db_load_image.argtypes = [P, ctypes.c_char_p, ctypes.c_int]
    L.sw_db_title.restype = ctypes.c_int
    L.sw_db_title.argtypes = [P, ctypes.c_uint64, ctypes.POINTER(ctypes.c_void_p),
                              ctypes.POINTER(ctypes.c_uint64)]
    L.sw_traceback.restype = ctypes.c_int
    L.sw_traceback.argtypes = [P, P, ctypes.c_uint32, P, ctypes.c_uint32,
                               ctypes.POINTER(sw_alignment), P, ctypes.c_uint64,
                               ctypes.POINTER(ctypes.c_uint64)]
    L.sw_serve_options_default.restype = None
    L.sw_serve_options_default.argtypes = [ctypes.POINTER(sw_serve_options)]
    L.sw_serve_start.restype = ctypes.c_int
    L.sw_serve_start.argtypes = [P, ctypes.POINTER(sw_serve_options)]
    L.sw_serve_submit.restype = ctypes.c_int
    L.sw_serve_submit.argtypes = [P, ctypes.c_uint64, P, ctypes.c_uint32]
    L.sw_serve_poll.restype = ctypes.c_int
    L.sw_serve_poll.argtypes = [P, ctypes.c_uint32, ctypes.POINTER(sw_serve_result),
                                ctypes.POINTER(sw_hit), ctypes.POINTER(ctypes.c_uint32),
                                ctypes.c_int32]
    L.sw_serve_get_stats.restype = ctypes.c_int
    L.sw_serve_get_stats.argtypes = [P, ctypes.POINTER(sw_serve_stats)]
    L.sw_serve_clock_ms.restype = ctypes.c_double
    L.sw_serve_clock_ms.argtypes = []
    L.sw_serve_stop.restype = ctypes.c_int
    L.sw_serve_stop.argtypes = [P]
    _lib = L
    return L


def parse_matrix(text: str) -> np.ndarray:
    """32x32 scoring matrix (search codes) from substitution-matrix text."""
    p = sw_params()
    load().sw_params_default(ctypes.byref(p))
    _image_call(load().sw_params_parse_matrix(ctypes.byref(p), text.encode()),
                "sw_params_parse_matrix")
    return np.array(p.matrix[:], dtype=np.int32).reshape(32, 32)


def load_matrix(name_or_path: str) -> np.ndarray:
    """'blosum62' or a matrix file, as a 32x32 array (search codes)."""
    p = sw_params()
    load().sw_params_default(ctypes.byref(p))
    _image_call(load().sw_params_load_matrix(ctypes.byref(p), name_or_path.encode()),
                "sw_params_load_matrix")
    return np.array(p.matrix[:], dtype=np.int32).reshape(32, 32)


def _image_call(st: int, what: str):
    if st != SW_OK:
        raise SwError(st, f"{what}: {load().sw_last_error(None).decode()}")


def _info(i: sw_image_info) -> dict:
    return dict(n_records=i.n_records, n_residues=i.n_residues, file_bytes=i.file_bytes,
                titles_bytes=i.titles_bytes, checksum=i.checksum, version=i.version)


def write_image(path: str, residues: np.ndarray, offsets: np.ndarray, titles=None):
    """DB image of records held in memory; titles: list of str or None."""
    r = np.ascontiguousarray(residues, dtype=np.uint8)
    o = np.ascontiguousarray(offsets, dtype=np.uint64)
    t = to = None
    if titles is not None:
        enc = [x.encode() for x in titles]
        t = np.frombuffer(b"".join(enc) or b"\0", dtype=np.uint8).copy()
        to = np.zeros(len(enc) + 1, dtype=np.uint64)
        to[1:] = np.cumsum([len(x) for x in enc])
    _image_call(load().sw_db_write_image(path.encode(), _ptr(r) if r.size else None, _ptr(o),
                                         len(o) - 1, _ptr(t) if t is not None else None,
                                         _ptr(to) if to is not None else None),
                "sw_db_write_image")


def fasta_to_image(fasta_path: str, image_path: str) -> dict:
    i = sw_image_info()
    _image_call(load().sw_fasta_to_image(fasta_path.encode(), image_path.encode(),
                                         ctypes.byref(i)), "sw_fasta_to_image")
    return _info(i)


def image_info(path: str, verify: bool = True) -> dict:
    i = sw_image_info()
    _image_call(load().sw_image_get_info(path.encode(), 1 if verify else 0, ctypes.byref(i)),
                "sw_image_get_info")
    return _info(i)


def serve_clock_ms() -> float:
    """The clock of served requests' timestamps (steady, milliseconds)."""
    return load().sw_serve_clock_ms()


def default_params(gap_open=10, gap_extend=2, top_k=10, matrix=None,
                   reference_cap=True) -> sw_params:
    p = sw_params()
    load().sw_params_default(ctypes.byref(p))
    p.gap_open = gap_open
    p.gap_extend = gap_extend
    p.top_k = top_k
    p.flags = SW_FLAG_REFERENCE_CAP if reference_cap else 0
    if matrix is not None:
        m = np.asarray(matrix, dtype=np.int32).reshape(-1)
        for i in range(1024):
            p.matrix[i] = int(m[i])
    return p


def shapes() -> list:
    """Compiled (group width, rows per thread) shapes."""
    L = load()
    n = ctypes.c_uint32(0)
    L.sw_get_shapes(None, None, None, 0, ctypes.byref(n))
    T = (ctypes.c_int32 * n.value)()
    R = (ctypes.c_int32 * n.value)()
    L.sw_get_shapes(T, R, None, n.value, ctypes.byref(n))
    return [(T[i], R[i]) for i in range(n.value)]


def shape_blocks() -> dict:
    """Threads per block of every compiled shape: {(group width, rows): threads}."""
    L = load()
    n = ctypes.c_uint32(0)
    L.sw_get_shapes(None, None, None, 0, ctypes.byref(n))
    T = (ctypes.c_int32 * n.value)()
    R = (ctypes.c_int32 * n.value)()
    B = (ctypes.c_int32 * n.value)()
    L.sw_get_shapes(T, R, B, n.value, ctypes.byref(n))
    return {(T[i], R[i]): B[i] for i in range(n.value)}


def score_noalloc(device: int, params: sw_params, d_query: int, qlen: int, d_residues: int,
                  d_offsets: int, n_records: int, d_scores: int, stream: int | None = None) -> int:
    """sw_score_noalloc on device pointers (ints); returns the sw_status."""
    return load().sw_score_noalloc(device, ctypes.byref(params), ctypes.c_void_p(d_query), qlen,
                                   ctypes.c_void_p(d_residues), ctypes.c_void_p(d_offsets),
                                   n_records, ctypes.c_void_p(d_scores),
                                   ctypes.c_void_p(stream) if stream else None)


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


class Context:
    """One device context with a resident DB (see include/swb200.h)."""

    def __init__(self, device: int = 0, params: sw_params | None = None):
        self.L = load()
        self.params = params if params is not None else default_params()
        h = ctypes.c_void_p()
        st = self.L.sw_ctx_create(device, ctypes.byref(self.params), ctypes.byref(h))
        if st != SW_OK:
            raise SwError(st, "sw_ctx_create")
        self.h = h
        self.n_records = 0

    def _check(self, st: int, what: str):
        if st != SW_OK:
            raise SwError(st, f"{what}: {self.L.sw_last_error(self.h).decode()}")

    def close(self):
        if getattr(self, "h", None):
            self.L.sw_ctx_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def load_db(self, residues: np.ndarray, offsets: np.ndarray):
        r = np.ascontiguousarray(residues, dtype=np.uint8)
        o = np.ascontiguousarray(offsets, dtype=np.uint64)
        self._check(self.L.sw_db_load(self.h, _ptr(r), _ptr(o), len(o) - 1), "sw_db_load")
        self.n_records = len(o) - 1

    def load_image(self, path: str, verify: bool = True):
        self._check(self.L.sw_db_load_image(self.h, path.encode(), 1 if verify else 0),
                    "sw_db_load_image")
        self.n_records = int(self.db_stats().n_records)

    def title(self, record: int) -> str:
        p = ctypes.c_void_p()
        n = ctypes.c_uint64(0)
        self._check(self.L.sw_db_title(self.h, record, ctypes.byref(p), ctypes.byref(n)),
                    "sw_db_title")
        return ctypes.string_at(p.value, n.value).decode(errors="replace") if n.value else ""

    def db_stats(self) -> sw_db_stats:
        s = sw_db_stats()
        self._check(self.L.sw_db_stats_get(self.h, ctypes.byref(s)), "sw_db_stats_get")
        return s

    def search(self, query: np.ndarray, want_scores: bool = False):
        """Returns (hits as list of (score, index), scores or None)."""
        q = np.ascontiguousarray(query, dtype=np.uint8)
        k = self.params.top_k
        hits = (sw_hit * k)()
        nh = ctypes.c_uint32(0)
        scores = np.zeros(max(self.n_records, 1), dtype=np.int32) if want_scores else None
        self._check(self.L.sw_search(self.h, _ptr(q), len(q), hits, ctypes.byref(nh),
                                     _ptr(scores) if want_scores else None), "sw_search")
        out = [(hits[i].score, hits[i].index) for i in range(nh.value)]
        return out, (scores[:self.n_records] if want_scores else None)

    def search_device(self, d_query_ptr: int, qlen: int, d_scores_ptr: int | None = None):
        self._check(self.L.sw_search_device(self.h, ctypes.c_void_p(d_query_ptr), qlen,
                                            ctypes.c_void_p(d_scores_ptr) if d_scores_ptr else None),
                    "sw_search_device")

    def set_kernel_config(self, cfg: tuple | None):
        if cfg is None:
            self._check(self.L.sw_set_kernel_config(self.h, None), "sw_set_kernel_config")
            return
        c = sw_kernel_config(*cfg)
        self._check(self.L.sw_set_kernel_config(self.h, ctypes.byref(c)), "sw_set_kernel_config")

    def set_batch_options(self, cutover=0, long_shape=(32, 16), use_graph=True,
                          stack_shape=(16, 64), stack_rows=4096, pair_rows=2048,
                          pair_shape=(16, 64), pair_long=True, pair_regions=0):
        o = sw_batch_options(cutover, long_shape[0], long_shape[1], 1 if use_graph else 0,
                             stack_shape[0], stack_shape[1], stack_rows, pair_rows,
                             pair_shape[0], pair_shape[1], 1 if pair_long else 0, pair_regions)
        self._check(self.L.sw_set_batch_options(self.h, ctypes.byref(o)), "sw_set_batch_options")

    def search_batch(self, queries, want_scores: bool = False):
        """queries: list of code arrays.  Returns (list of hit lists, scores
        [n_queries, n_records] or None)."""
        nq = len(queries)
        off = np.zeros(nq + 1, dtype=np.uint64)
        off[1:] = np.cumsum([len(q) for q in queries])
        flat = (np.concatenate([np.asarray(q, dtype=np.uint8) for q in queries])
                if nq and off[-1] else np.zeros(1, dtype=np.uint8))
        k = self.params.top_k
        hits = (sw_hit * max(nq * k, 1))()
        nh = (ctypes.c_uint32 * max(nq, 1))()
        scores = np.zeros((nq, max(self.n_records, 1)), dtype=np.int32) if want_scores else None
        self._check(self.L.sw_search_batch(self.h, nq, _ptr(flat), _ptr(off), hits, nh,
                                           _ptr(scores) if want_scores else None),
                    "sw_search_batch")
        out = [[(hits[q * k + i].score, hits[q * k + i].index) for i in range(nh[q])]
               for q in range(nq)]
        return out, (scores[:, :self.n_records] if want_scores else None)

    def set_tuning(self, table):
        """table: [(max_qlen, (T, R, T, R, cutover)[, plan]), ...] sorted by
        max_qlen; plan: up to PLAN_STEPS (T, R, passes) row-segment steps
        (passes 0: the rest of the query)."""
        arr = (sw_tuning_entry * max(len(table), 1))()
        for i, row in enumerate(table):
            hi, cfg = row[0], row[1]
            plan = row[2] if len(row) > 2 else ()
            if len(plan) > PLAN_STEPS:
                raise ValueError(f"plan of {len(plan)} steps (at most {PLAN_STEPS})")
            arr[i].max_qlen = int(hi)
            arr[i].cfg = sw_kernel_config(*cfg)
            for j, (T, R, passes) in enumerate(plan):
                arr[i].plan[j] = sw_plan_step(int(T), int(R), int(passes))
        self._check(self.L.sw_set_tuning(self.h, arr, len(table)), "sw_set_tuning")

    def plan(self, qlen: int) -> list:
        """Row segments a plain search of qlen runs: [(T, R, passes), ...]."""
        steps = (sw_plan_step * (PLAN_STEPS + 1))()
        n = ctypes.c_uint32(0)
        self._check(self.L.sw_get_plan(self.h, qlen, steps, PLAN_STEPS + 1, ctypes.byref(n)),
                    "sw_get_plan")
        return [(steps[i].group_width, steps[i].rows_per_thread, steps[i].passes)
                for i in range(n.value)]

    def kernel_config(self, qlen: int) -> tuple:
        c = sw_kernel_config()
        self._check(self.L.sw_get_kernel_config(self.h, qlen, ctypes.byref(c)),
                    "sw_get_kernel_config")
        return c.as_tuple()

    def set_stream(self, stream_handle: int | None):
        self._check(self.L.sw_set_stream(self.h, ctypes.c_void_p(stream_handle or None)),
                    "sw_set_stream")

    def sync(self):
        self._check(self.L.sw_sync(self.h), "sw_sync")

    def reset_totals(self):
        self._check(self.L.sw_reset_totals(self.h), "sw_reset_totals")

    def totals(self) -> sw_totals:
        t = sw_totals()
        self._check(self.L.sw_get_totals(self.h, ctypes.byref(t)), "sw_get_totals")
        return t

    def traceback(self, query: np.ndarray, records) -> list:
        """Best local alignment of the query against each record (DB order
        indices): dicts with index, score, q_begin, q_end, d_begin, d_end,
        matches, cigar (text, M/I/D)."""
        q = np.ascontiguousarray(query, dtype=np.uint8)
        recs = np.ascontiguousarray(records, dtype=np.uint64)
        n = len(recs)
        out = (sw_alignment * max(n, 1))()
        cap = 64 * max(n, 1)
        while True:
            ops = np.zeros(cap, dtype=np.uint32)
            used = ctypes.c_uint64(0)
            st = self.L.sw_traceback(self.h, _ptr(q) if q.size else None, q.size,
                                     _ptr(recs) if n else None, n, out, _ptr(ops), cap,
                                     ctypes.byref(used))
            if st == 6 and used.value > cap:     # ops buffer too small: size it and repeat
                cap = int(used.value)
                continue
            self._check(st, "sw_traceback")
            break
        res = []
        for i in range(n):
            a = out[i]
            cig = "".join(f"{int(o) >> 4}{'MID'[int(o) & 15]}"
                          for o in ops[a.ops_offset:a.ops_offset + a.n_ops])
            res.append(dict(index=int(a.index), score=a.score, q_begin=a.q_begin,
                            q_end=a.q_end, d_begin=a.d_begin, d_end=a.d_end,
                            matches=a.matches, cigar=cig))
        return res

    # ---- serving ----------------------------------------------------------
    def serve_start(self, max_active=None, chunks=None, max_pending=None, memory_budget=None,
                    shape=None, stack_rows=None, pair_rows=None, pair_shape=None,
                    pair_long=None, pair_regions=None):
        o = sw_serve_options()
        self.L.sw_serve_options_default(ctypes.byref(o))
        if max_active is not None:
            o.max_active = max_active
        if chunks is not None:
            o.chunks = chunks
        if max_pending is not None:
            o.max_pending = max_pending
        if memory_budget is not None:
            o.memory_budget = memory_budget
        if shape is not None:
            o.group_width, o.rows_per_thread = shape
        if stack_rows is not None:
            o.stack_rows = stack_rows
        if pair_rows is not None:
            o.pair_rows = pair_rows
        if pair_shape is not None:
            o.pair_group_width, o.pair_rows_per_thread = pair_shape
        if pair_long is not None:
            o.pair_long = 1 if pair_long else 0
        if pair_regions is not None:
            o.pair_regions = pair_regions
        self._check(self.L.sw_serve_start(self.h, ctypes.byref(o)), "sw_serve_start")

    def serve_submit(self, request_id: int, query: np.ndarray) -> int:
        """Queues a request; returns SW_OK (0) or SW_ERR_BUSY (7) when the
        waiting queue is full; raises on any other status."""
        q = np.ascontiguousarray(query, dtype=np.uint8)
        st = self.L.sw_serve_submit(self.h, request_id, _ptr(q) if q.size else None, q.size)
        if st not in (0, 7):
            raise SwError(st, f"sw_serve_submit: {STATUS.get(st, st)}")
        return st

    def serve_poll(self, max_results: int = 64, timeout_ms: int = 0) -> list:
        """Completed requests: dicts with id, status, hits [(score, index)],
        submit_ms, start_ms, done_ms."""
        k = self.params.top_k
        res = (sw_serve_result * max(max_results, 1))()
        hits = (sw_hit * max(max_results * k, 1))()
        n = ctypes.c_uint32(0)
        self._check(self.L.sw_serve_poll(self.h, max_results, res, hits, ctypes.byref(n),
                                         timeout_ms), "sw_serve_poll")
        out = []
        for i in range(n.value):
            r = res[i]
            out.append(dict(id=r.request_id, status=r.status,
                            hits=[(hits[i * k + j].score, hits[i * k + j].index)
                                  for j in range(r.n_hits)],
                            submit_ms=r.submit_ms, start_ms=r.start_ms, done_ms=r.done_ms))
        return out

    def serve_stats(self) -> sw_serve_stats:
        s = sw_serve_stats()
        self._check(self.L.sw_serve_get_stats(self.h, ctypes.byref(s)), "sw_serve_get_stats")
        return s

    def serve_stop(self):
        self._check(self.L.sw_serve_stop(self.h), "sw_serve_stop")

    def run_stats(self) -> sw_run_stats:
        s = sw_run_stats()
        self._check(self.L.sw_get_run_stats(self.h, ctypes.byref(s)), "sw_get_run_stats")
        return s
