"""In-tree build of libswb200.so for sm_100a (nvcc cross-compiles without a GPU).

Before compiling, the shape table measured by the autotuner
(``tuned/b200.json``) is written into ``csrc/sw_tuned_default.h``: every new
context starts with it, so the C ABI and the C++ worker are tuned without a
call to ``sw_set_tuning``."""
from __future__ import annotations

import json
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
TABLE = os.path.join(HERE, "tuned", "b200.json")
DEFAULT_HEADER = os.path.join(HERE, "csrc", "sw_tuned_default.h")


def default_header_text(table_path: str = TABLE) -> str:
    """C++ text of the built-in shape table for the table in table_path."""
    with open(table_path) as f:
        doc = json.load(f)
    meta = doc.get("meta", {})
    lines = [
        "// sw_tuned_default.h -- the shape table every new context starts with",
        "// (sw_set_tuning replaces it; n = 0 leaves the cost model).  Written by",
        "// swhybrid_b200/build.py from swhybrid_b200/tuned/b200.json, the autotuner's",
        f"// sweep of every compiled shape on {meta.get('gpu', 'B200')} ({meta.get('records', '?')} records,",
        f"// {meta.get('residues', '?')} residues).  Do not edit; re-run the autotuner.",
        "#pragma once",
        '#include "../../include/swb200.h"',
        "",
        "namespace swb {",
        "",
        "// {max_qlen, {long T, long R, short T, short R, cut-over}[, row-segment plan:",
        "//  {{T, R, passes}, ...}, passes 0 = the rest of the query]}",
        "constexpr sw_tuning_entry kDefaultTuning[] = {",
    ]
    for row in doc["table"]:
        hi, cfg = row[0], row[1]
        text = "    {%du, {%d, %d, %d, %d, %d}" % (int(hi), *(int(x) for x in cfg))
        if len(row) > 2 and row[2]:
            text += ", {" + ", ".join("{%d, %d, %d}" % tuple(int(x) for x in st)
                                      for st in row[2]) + "}"
        lines.append(text + "},")
    lines += ["};", "", "}  // namespace swb", ""]
    return "\n".join(lines)


def write_default_header(table_path: str = TABLE, out: str = DEFAULT_HEADER) -> bool:
    """Writes the header when its text changes (so make rebuilds only then)."""
    text = default_header_text(table_path)
    if os.path.exists(out) and open(out).read() == text:
        return False
    with open(out, "w") as f:
        f.write(text)
    return True


def build(jobs: int = 8, verbose: bool = False) -> str:
    write_default_header()
    cmd = ["make", "-C", os.path.join(HERE, "csrc"), f"-j{jobs}"]
    out = subprocess.run(cmd, capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("libswb200 build failed:\n" + out.stdout[-4000:] + out.stderr[-4000:])
    if verbose:
        print(out.stdout)
    return os.path.join(HERE, "libswb200.so")


if __name__ == "__main__":
    print(build(verbose=True))
