"""Autotuner for the first-pass kernel shape (group width x rows per thread,
and the long/short cut-over).

For a DB and a list of query lengths it times every compiled shape on the
present GPU (device time of the first-pass launches, CUDA events inside the
library), keeps the fastest per length, and writes a JSON table that
``apply()`` hands to the library (``sw_set_tuning``).  Shapes whose profile
does not fit in shared memory for a length are skipped (the library refuses
them with SW_ERR_UNSUPPORTED).

    python -m swhybrid_b200.autotune --out swhybrid_b200/tuned/b200.json
"""
from __future__ import annotations

import argparse
import bisect
import json
import os
import time

import numpy as np

from . import capi, synth

GROUP_WIDTHS = (4, 8, 16, 32)
ROWS = (4, 6, 8, 10, 12, 16, 20, 24, 28, 32, 40, 48, 56, 64)
DEFAULT_TABLE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuned", "b200.json")


def time_shape(ctx: capi.Context, dq, qlen: int, cfg: tuple, reps: int = 2) -> float | None:
    """GCUPS of the first pass for one shape, or None if it does not fit."""
    ctx.set_kernel_config(cfg)
    try:
        ctx.search_device(dq.data_ptr(), qlen)          # warm-up
        ctx.sync()
    except capi.SwError as e:
        if e.status == 6:
            return None
        raise
    ctx.reset_totals()
    for _ in range(reps):
        ctx.search_device(dq.data_ptr(), qlen)
    ctx.sync()
    t = ctx.totals()
    return t.cells / (t.first_pass_ms * 1e-3) / 1e9


def reps_for(L: int, reps: int) -> int:
    """Searches timed per shape at query length L: at least `reps`, and
    enough that short queries (a few milliseconds per search on the full DB)
    are timed over about as many cells as a 4,000-residue one.  With one
    search per shape, two sweeps on the same DB picked shapes up to 22 %
    apart in speed for the queries of 144..310 residues."""
    return max(reps, -(-4000 // max(int(L), 1)))


def sweep(ctx: capi.Context, lengths, shapes=None, reps: int = 2, log=print,
          cutovers=(1024, 2048, 4096, 8192, 16384), warmup_s: float = 5.0):
    import torch
    shapes = shapes or [(T, R) for T in GROUP_WIDTHS for R in ROWS]
    results = {}
    # Bring the GPU to its working clock before the first timing: a sweep that
    # started cold measured its first (shortest) lengths up to 30 % low.
    warm = torch.from_numpy(synth.query(8999, 2000)).cuda()
    ctx.set_kernel_config(None)
    t_end = time.time() + warmup_s
    while time.time() < t_end:
        ctx.search_device(warm.data_ptr(), 2000)
        ctx.sync()
    for L in lengths:
        q = synth.query(9000 + int(L), int(L))
        dq = torch.from_numpy(q).cuda()
        row = {}
        n = reps_for(int(L), reps)
        for T, R in shapes:
            g = time_shape(ctx, dq, int(L), (T, R, T, R, 0), n)
            if g is not None:
                row[f"{T}x{R}"] = round(g, 1)
        best = max(row, key=row.get)
        T, R = (int(x) for x in best.split("x"))
        cut = {}
        for c in cutovers:
            g = time_shape(ctx, dq, int(L), (T, R, T, R, c), n)
            if g is not None:
                cut[c] = round(g, 1)
        best_cut = max(cut, key=cut.get) if cut else 0
        if cut and cut[best_cut] <= row[best]:
            best_cut = 0
        results[int(L)] = {"best": best, "cutover": int(best_cut),
                           "gcups": max(row[best], cut.get(best_cut, 0.0)),
                           "all": row, "cutovers": {str(k): v for k, v in cut.items()}}
        log(f"qlen {L}: best {best} cut-over {best_cut} {results[int(L)]['gcups']:.0f} GCUPS")
    ctx.set_kernel_config(None)
    return results


def rows_used(T: int, R: int, qlen: int) -> int:
    """Query rows a shape computes for a query: whole passes of T*R rows."""
    return -(-qlen // (T * R)) * T * R


SMEM_OPTIN = 232_448      # B200 shared memory a block may opt in to (bytes)
CODES = 25                # profile rows per pass chunk (residue codes incl. the zero code)


def profile_fits(T: int, R: int, qlen: int) -> bool:
    """Whether the query profile of a shape fits a block's shared memory (the
    library's wf_smem_bytes: passes x 8-row chunks x codes x slots x 8 B)."""
    passes = -(-qlen // (T * R))
    return passes * ((R + 7) // 8) * CODES * max(T, 16) * 8 <= SMEM_OPTIN


def predict_gcups(results, shape: str, qlen: int) -> float | None:
    """GCUPS of a shape at any query length from the sweep: a shape's rate on
    the rows it computes (measured GCUPS x rows computed / qlen) changes slowly
    with the length, while the share of those rows that are padding changes
    at every pass boundary.  The rate is interpolated (in log length) between
    the two measured lengths around qlen; None if the shape was not measured
    at both (its profile did not fit) or qlen is far past the last one."""
    T, R = (int(x) for x in shape.split("x"))
    if not profile_fits(T, R, qlen):
        return None
    Ls = sorted(results)

    def rate(L):
        g = results[L]["all"].get(shape)
        return None if g is None else g * rows_used(T, R, L) / L

    if qlen <= Ls[0]:
        r = rate(Ls[0])
    elif qlen >= Ls[-1]:
        r = rate(Ls[-1]) if qlen <= 1.5 * Ls[-1] else None
    else:
        i = bisect.bisect_left(Ls, qlen)        # Ls[i - 1] < qlen <= Ls[i]
        r0, r1 = rate(Ls[i - 1]), rate(Ls[i])
        if r0 is None or r1 is None:
            return None
        w = (np.log(qlen) - np.log(Ls[i - 1])) / (np.log(Ls[i]) - np.log(Ls[i - 1]))
        r = r0 * (1 - w) + r1 * w
    return None if r is None else r * qlen / rows_used(T, R, qlen)


def plan_shapes(results, blocks: dict) -> list:
    """Shapes a row-segment plan may use: at most 16 groups (record pairs in
    flight) per block.  On the 205 M-residue DB an evenly loaded group of
    such a shape gets more columns than the longest record pair (35,000), so
    its launch does not end on one pair's serial column steps; a narrower
    shape only pays with the long-pair split, which a plan does not use.  The
    library checks the same rule against the DB at hand and runs the single
    shape instead when a plan breaks it."""
    shapes = sorted({s for L in results for s in results[L]["all"]})
    out = []
    for s in shapes:
        T, R = (int(x) for x in s.split("x"))
        b = blocks.get((T, R))
        if b is not None and b // T <= 16:
            out.append(s)
    return out


def best_plans(results, shapes, step: int = 8, top: int = 8192, max_steps: int = 4) -> dict:
    """{q: (predicted time, [(T, R, passes), ...])} for q on the grid: the
    fastest predicted row-segment plan of at most max_steps steps from
    `shapes`, each step whole passes but the last (passes 0: the rest of the
    query, its last pass padded).  Time is in rows / GCUPS units: a step of
    P whole passes costs P*T*R / predict_gcups(shape, P*T*R), the rest
    L / predict_gcups(shape, L).  Whole passes are multiples of 8 rows
    (T >= 4, R even), so every remainder is again a grid point."""
    memo = {}

    def g(s, rows):
        key = (s, rows)
        if key not in memo:
            memo[key] = predict_gcups(results, s, rows)
        return memo[key]

    best = {}
    for q in range(step, top + step, step):
        bt, bp = float("inf"), None
        for s in shapes:
            v = g(s, q)
            if v and q / v < bt:
                T, R = (int(x) for x in s.split("x"))
                bt, bp = q / v, [(T, R, 0)]
        for s in shapes:
            T, R = (int(x) for x in s.split("x"))
            for P in range(1, (q - 1) // (T * R) + 1):
                rows = P * T * R
                v = g(s, rows)
                rest = best.get(q - rows)
                if not v or rest is None or rest[1] is None or len(rest[1]) >= max_steps:
                    continue
                t = rows / v + rest[0]
                if t < bt:
                    bt, bp = t, [(T, R, P)] + rest[1]
        best[q] = (bt, bp)
    return best


def table_from_sweep(results, step: int = 8, top: int = 8192, blocks: dict | None = None,
                     plan_margin: float = 0.02) -> list:
    """[(max_qlen, (T, R, T, R, cutover), plan), ...]: the shape with the best
    predicted GCUPS (predict_gcups) on a grid of query lengths, runs of equal
    choices merged.  The cut-over is the one measured with that shape at the
    nearest measured length when the shape was the best there, else 0 (the
    library's automatic rule).  plan: the fastest predicted row-segment plan
    (best_plans over plan_shapes) when it beats that shape by more than
    plan_margin and has at least two steps (whole passes of one shape, then
    the rest with another, so only the last pass holds padding rows), else
    ().  blocks: threads per block by shape (default: the library's)."""
    Ls = sorted(results)
    shapes = sorted({s for L in Ls for s in results[L]["all"]})
    if blocks is None:
        blocks = capi.shape_blocks()
    plans = best_plans(results, plan_shapes(results, blocks), step, top)
    out = []
    for q in range(step, top + step, step):
        best, bg = None, -1.0
        for s in shapes:
            g = predict_gcups(results, s, q)
            if g is not None and g > bg:
                best, bg = s, g
        if best is None:
            continue
        near = min(Ls, key=lambda L: abs(np.log(L) - np.log(q)))
        cut = int(results[near].get("cutover", 0)) if results[near]["best"] == best else 0
        T, R = (int(x) for x in best.split("x"))
        cfg = (T, R, T, R, cut)
        plan = ()
        pt, pp = plans.get(q, (float("inf"), None))
        if pp is not None and len(pp) >= 2 and pt * (1.0 + plan_margin) < q / bg:
            plan = tuple(pp)
        if out and out[-1][1] == cfg and out[-1][2] == plan:
            out[-1] = (q, cfg, plan)
        else:
            out.append((q, cfg, plan))
    if out:
        T, R = (int(x) for x in results[Ls[-1]]["best"].split("x"))
        out.append((1 << 30, (T, R, T, R, int(results[Ls[-1]].get("cutover", 0))), ()))
    return out


def save(results, path: str = DEFAULT_TABLE, meta=None):
    os.makedirs(os.path.dirname(path), exist_ok=True)
    doc = {"meta": meta or {}, "sweep": {str(k): v for k, v in results.items()},
           "table": [[hi, list(cfg)] + ([[list(st) for st in plan]] if plan else [])
                     for hi, cfg, plan in table_from_sweep(results)]}
    with open(path, "w") as f:
        json.dump(doc, f, indent=1)


def load_table(path: str = DEFAULT_TABLE):
    if not os.path.exists(path):
        return None
    with open(path) as f:
        doc = json.load(f)
    return [(int(row[0]), tuple(int(x) for x in row[1]),
             tuple(tuple(int(x) for x in st) for st in row[2]) if len(row) > 2 else ())
            for row in doc["table"]]


def apply(ctx: capi.Context, path: str = DEFAULT_TABLE) -> bool:
    tab = load_table(path)
    if not tab:
        return False
    ctx.set_tuning(tab)
    return True


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=DEFAULT_TABLE)
    ap.add_argument("--records", type=int, default=570_000)
    ap.add_argument("--long", type=int, default=200)
    ap.add_argument("--reps", type=int, default=1)
    ap.add_argument("--widths", type=str, default="4,8,16,32",
                    help="group widths to try (comma separated)")
    args = ap.parse_args()
    widths = [int(x) for x in args.widths.split(",")]
    db = synth.full_db(7, args.records, args.long)
    ctx = capi.Context(0)
    ctx.load_db(db.residues, db.offsets)
    t0 = time.time()
    res = sweep(ctx, synth.sweep_lengths(), shapes=[(T, R) for T in widths for R in ROWS],
                reps=args.reps)
    import torch
    save(res, args.out, meta={"gpu": torch.cuda.get_device_name(0), "records": db.n,
                              "residues": db.total, "seconds": round(time.time() - t0, 1)})
    print("wrote", args.out)


if __name__ == "__main__":
    main()
