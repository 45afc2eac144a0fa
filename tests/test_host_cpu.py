"""CPU tests of the host side: parameters/encoding mirror, the workload
generators, and that libswb200.so loads and exports every C-ABI symbol of
include/swb200.h (no compute calls without a GPU)."""
import ctypes
import os
import re

import numpy as np
import pytest

from swhybrid_b200 import capi, param, synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    src = open(os.path.join(ROOT, "include", "swb200.h")).read()
    decl = r"^(?:const\s+)?(?:struct\s+)?[a-z_0-9]+\s*\**\s*(sw_[a-z0-9_]+)\s*\("
    return sorted(set(re.findall(decl, src, flags=re.M)))


def test_header_and_binding_agree():
    assert header_symbols() == sorted(capi.EXPORTS)


def test_library_exports_every_symbol():
    lib = ctypes.CDLL(capi.LIB_PATH)
    for name in header_symbols():
        assert hasattr(lib, name), name


def test_params_default_is_reference_param():
    L = capi.load()
    p = capi.sw_params()
    L.sw_params_default(ctypes.byref(p))
    assert (p.gap_open, p.gap_extend, p.top_k) == (10, 2, 10)
    np.testing.assert_array_equal(np.array(p.matrix[:]).reshape(32, 32), param.blosum62())
    ref = param.Param(["swhybrid", "-o", "11", "-e", "1", "-t", "5"])
    assert (ref.gapOpen, ref.gapExtend, ref.topNum, ref.gapOE) == (11, 1, 5, 12)


def test_encode_matches_python_table():
    L = capi.load()
    letters = b"ACDEFGHIKLMNPQRSTVWYBXZ@JOU*acdwxyz-"
    out = (ctypes.c_uint8 * len(letters))()
    assert L.sw_encode(letters, len(letters), out) == 0
    np.testing.assert_array_equal(np.frombuffer(bytes(out), dtype=np.uint8),
                                  param.encode(letters))
    assert param.encode("ABZ@J").tolist() == [0, 1, 22, 23, 24]


def test_no_device_is_reported_not_faked():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("GPU present")
    except Exception:
        pass
    with pytest.raises(capi.SwError) as e:
        capi.Context(0)
    assert e.value.status in (9, 2)


def test_generators_are_seeded_and_shaped():
    a = synth.small_db(1, 2000)
    b = synth.small_db(1, 2000)
    assert np.array_equal(a.residues, b.residues)
    L = a.lengths()
    assert L.min() >= 20 and L.max() <= 5000
    assert abs(np.median(L) - np.exp(5.6)) < 30
    # background composition close to the table
    counts = np.bincount(a.residues, minlength=23) / a.total
    assert abs(counts[param.ALPHABET.index("L")] - 0.09019) < 0.01
    assert counts[param.ALPHABET.index("B")] == 0
    sweep = synth.sweep_lengths()
    assert sweep[0] == 144 and sweep[-1] == 5478 and len(sweep) == 20


def test_tuning_table_accounts_for_pass_padding():
    """The shape table derived from a sweep predicts each shape from its rate on
    the rows it computes, so a shape whose last pass would be mostly padding
    loses to one that fits the length, and measured lengths reproduce."""
    from swhybrid_b200 import autotune
    rate = {"16x64": 4000.0, "32x56": 4100.0}          # GCUPS on computed rows
    res = {}
    for L in (1000, 1500, 2000, 3000):
        row = {s: rate[s] * L / autotune.rows_used(*map(int, s.split("x")), L) for s in rate}
        res[L] = {"best": max(row, key=row.get), "cutover": 0, "all": row}
    for L in res:
        for s in rate:
            assert abs(autotune.predict_gcups(res, s, L) - res[L]["all"][s]) < 1e-6
    tab = autotune.table_from_sweep(res)
    pick = lambda q: next(cfg for hi, cfg, _ in tab if q <= hi)[:2]
    assert pick(1792) == (32, 56)       # one full 1,792-row pass
    assert pick(1900) == (16, 64)       # 2 x 1,024 rows, not 2 x 1,792
    assert pick(3584) == (32, 56)
    assert [row[0] for row in tab] == sorted(row[0] for row in tab)
    committed = autotune.load_table()
    assert committed and [row[0] for row in committed] == sorted(row[0] for row in committed)
    # every shape whose profile fits one block was measured at every length
    # (a shape that does not fit still runs, in row segments over several
    # launches, and the table never picks it where it does not fit)
    import json
    sweep = json.load(open(autotune.DEFAULT_TABLE))["sweep"]
    for L, v in sweep.items():
        for T in autotune.GROUP_WIDTHS:
            for R in autotune.ROWS:
                if autotune.profile_fits(T, R, int(L)):
                    assert f"{T}x{R}" in v["all"], (L, T, R)
    for hi, c, _ in committed:
        if hi < (1 << 30):
            assert autotune.profile_fits(c[2], c[3], hi), (hi, c)
    # the library's built-in table is the committed one
    from swhybrid_b200 import build
    assert open(build.DEFAULT_HEADER).read() == build.default_header_text()
    shapes = set(capi.shapes())
    assert all((c[0], c[1]) in shapes and (c[2], c[3]) in shapes for _, c, _ in committed)


def test_tuning_table_row_segment_plans():
    """Row-segment plans: with two shapes of known rates on the rows they
    compute, a length that is one pass of each runs as those two segments
    instead of padding either shape's last pass.  In the committed table every
    plan has 2..4 steps of shapes with at most 16 groups per block, fixed
    steps of whole passes that leave rows for the rest at every length of the
    entry's range, and the rest last."""
    from swhybrid_b200 import autotune
    rate = {"16x64": 4000.0, "32x20": 3800.0}
    res = {}
    for L in (600, 1000, 1500, 2000, 3000):
        row = {s: rate[s] * L / autotune.rows_used(*map(int, s.split("x")), L) for s in rate}
        res[L] = {"best": max(row, key=row.get), "cutover": 0, "all": row}
    blocks = {(16, 64): 256, (32, 20): 512}
    tab = autotune.table_from_sweep(res, blocks=blocks)
    plan = next(p for hi, _, p in tab if 1664 <= hi)
    assert sorted(plan) == sorted([(16, 64, 1), (32, 20, 0)]) or \
        sorted(plan) == sorted([(32, 20, 1), (16, 64, 0)])
    assert next(p for hi, _, p in tab if 1024 <= hi) == ()      # one whole pass
    # a shape with more than 16 groups per block is never a plan step
    assert not any(p for _, _, p in autotune.table_from_sweep(res, blocks={(16, 64): 384,
                                                                           (32, 20): 640}))
    committed = autotune.load_table()
    lib_blocks = capi.shape_blocks()
    prev, n_plans = 0, 0
    for hi, cfg, plan in committed:
        if plan:
            n_plans += 1
            assert 2 <= len(plan) <= capi.PLAN_STEPS
            assert all(P > 0 for _, _, P in plan[:-1]) and plan[-1][2] == 0
            assert sum(P * T * R for T, R, P in plan[:-1]) <= prev
            assert all(lib_blocks[(T, R)] // T <= 16 for T, R, _ in plan)
        prev = hi
    assert n_plans > 0


def test_ctypes_structs_match_the_c_header(tmp_path):
    """The ctypes mirrors in capi.py have the sizes and field offsets the C
    compiler gives the structs of include/swb200.h (gcc on a generated
    program), so the Python binding passes what the library reads."""
    import subprocess
    structs = [getattr(capi, n) for n in dir(capi)
               if n.startswith("sw_") and isinstance(getattr(capi, n), type)
               and issubclass(getattr(capi, n), ctypes.Structure)]
    assert len(structs) >= 10
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "swb200.h"', "int main(void) {"]
    for s in structs:
        lines.append(f'printf("{s.__name__} size %zu\\n", sizeof({s.__name__}));')
        for f in s._fields_:
            lines.append(f'printf("{s.__name__} {f[0]} %zu\\n", offsetof({s.__name__}, {f[0]}));')
    lines += ["return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    inc = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")
    subprocess.run(["gcc", "-std=c11", "-I", inc, str(src), "-o", str(exe)], check=True)
    got = {}
    for line in subprocess.run([str(exe)], check=True, capture_output=True,
                               text=True).stdout.splitlines():
        name, field, value = line.split()
        got[(name, field)] = int(value)
    for s in structs:
        assert got[(s.__name__, "size")] == ctypes.sizeof(s), s.__name__
        for f in s._fields_:
            assert got[(s.__name__, f[0])] == getattr(s, f[0]).offset, (s.__name__, f[0])
