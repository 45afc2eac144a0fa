#!/usr/bin/env python3
"""Benchmark: Smith-Waterman protein DB search on B200 (GCUPS).

Workload (default, "full"): a 570,000-record synthetic DB (lognormal(5.6,
0.7) lengths clipped 10..35,000, plus 200 planted records of 10,000..35,000,
~205 M residues) resident in HBM, and a 20-point query-length sweep
log-spaced 144..5,478; one step = the whole sweep, one query per search call
(the plain method).  BLOSUM62, gap open 10 / extend 2, top-10, int8/int16
reference semantics (scores bit-exact to the reference).

value : GCUPS of the resident path (sw_search_device, query already on the
        device), device time by CUDA events on the library's stream, K steps,
        max over ranks; algorithmic cells = qlen x sum of real record lengths.
e2e   : GCUPS through the public C-ABI call sw_search with host buffers
        (query H2D and top-k D2H inside the timed region), host wall clock.
roofline: the first-pass kernel against the packed-int16 DPX roofline
        measured live on this GPU by libswprobe.so (the per-row instruction
        mix of the kernel run from registers at full occupancy).
cpu_baseline: the reference's own AVX2 kernels (avxCompute + avxCompute16,
        compiled from the reference sources into oracle/_ref) on a bounded
        sample of the same workload, all host threads.

--impl reference runs only the reference's CPU kernels (rank 0), one step =
the whole sweep against the full DB, and prints the same metric.

Multi-GPU (torchrun): every rank holds its own 205 M-residue DB shard (a
different seed) and runs the same sweep; the work is independent per rank
(weak scaling), and only the timing is reduced (max over ranks).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "GCUPS on 1 B200, plain vs batched/served; p50/p99 query latency (bit-exact)"
WORKLOADS = {
    "full": "plain method, full size: 570,000+200 records (~205M residues), "
            "20 query lengths log-spaced 144..5,478, one query per call",
    "small": "plain method, small: 20,000 records (~6.5M residues), query 375",
    "profile": "profiling case: the full-size DB (~205M residues) and one query of 1,434",
    "stress": "overflow/long-record stress: 100,000 records + 1% of 10,000..40,000 (~58M residues), "
              "0.5% planted homologs, 8 queries 500..4,000, one query per call",
    "batched": "profiling case: the full-size DB and the 64-query batch (lengths log-uniform "
               "50..5,000), one sw_search_batch call per step",
    "traceback": "profiling case: the full-size DB, one query of 1,434 and the alignments of its "
                 "top-10 hits (sw_traceback) per step",
    "probe": "the roofline probe alone: register-only cell mixes and issue rates (libswprobe.so)",
    "serve": "profiling case: the full-size DB and --serve-requests requests (lengths log-uniform "
             "30..8,000) queued at once on sw_serve_* (the serving leg's saturated phase)",
}


# ---------------------------------------------------------------------------
def parse(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=list(WORKLOADS), default="full")
    ap.add_argument("--cpu-seconds", type=float, default=30.0,
                    help="target CPU time of the bounded reference sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--config", type=str, default=None,
                    help="force a kernel shape 'T,R,T,R,cutover'")
    ap.add_argument("--no-batched", action="store_true",
                    help="skip the batched (64-query) measurement")
    ap.add_argument("--serve-requests", type=int, default=96,
                    help="requests per offered load in the serving leg (0 = skip it)")
    ap.add_argument("--serve-levels", type=str, default="0.25,0.5,0.75,1.0",
                    help="offered loads of the serving leg, as fractions of the saturating rate")
    ap.add_argument("--serve-half-requests", type=int, default=1000,
                    help="requests at the 50%% offered load (p99 at half load)")
    ap.add_argument("--serve-chunks", type=int, default=None,
                    help="serving: DB chunks of the ring (default: the library's)")
    ap.add_argument("--serve-slots", type=int, default=None,
                    help="serving: requests in flight (default: the library's)")
    ap.add_argument("--serve-pair-long", type=int, choices=[0, 1], default=None,
                    help="serving: pair long requests too (default: the library's)")
    ap.add_argument("--serve-regions", type=int, default=None,
                    help="serving: boundary regions of tall paired lanes (default: the library's)")
    ap.add_argument("--no-stress", action="store_true",
                    help="skip the overflow / long-record stress measurement")
    ap.add_argument("--kernel-only", action="store_true",
                    help="time the resident path only (no e2e, probe or CPU baseline)")
    ap.add_argument("--no-pairs", action="store_true",
                    help="batched profiling case: no paired-query lanes (stacks only)")
    ap.add_argument("--shard", action="store_true",
                    help="one DB split over the ranks (residue-balanced shards, all-gather "
                         "of k hits per query): strong scaling of the sharded search")
    return ap.parse_args(argv)


def make_workload(name: str, rank: int):
    from swhybrid_b200 import synth
    if name == "small":
        db = synth.small_db(1, 20_000)
        queries = [synth.query(375, 375)]
    elif name == "profile":
        db = synth.full_db(2 + 1000 * rank)
        queries = [synth.query(112, 1434)]
    elif name == "stress":
        db, queries, _, _ = synth.stress_workload(4 + 1000 * rank)
    else:
        db = synth.full_db(2 + 1000 * rank)
        queries = [synth.query(100 + i, int(L)) for i, L in enumerate(synth.sweep_lengths())]
    return db, queries


# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi samples of SM clock / throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def probe_rates(device: int):
    """Packed-integer issue rates of this GPU (libswprobe.so)."""
    path = os.path.join(ROOT, "swhybrid_b200", "libswprobe.so")
    L = ctypes.CDLL(path)
    L.swprobe_rates.restype = ctypes.c_int
    L.swprobe_rates.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_double), ctypes.c_int]
    out = (ctypes.c_double * 20)()
    rc = L.swprobe_rates(device, out, 4096)
    if rc != 0:
        raise RuntimeError(f"swprobe_rates failed: {rc}")
    sms, mhz = out[9], out[10]
    per = lambda v, lanes: v / lanes / 32 / (sms * mhz * 1e6)  # warp-instr / clk / SM
    return {
        "viaddmax_s16x2_instr_per_clk_sm": per(out[0], 2),
        "vimax3_s16x2_instr_per_clk_sm": per(out[1], 2),
        "prmt_instr_per_clk_sm": per(out[2], 1),
        "imad_instr_per_clk_sm": per(out[4], 1),
        "dpx_imad_mix_instr_per_clk_sm": per(out[5], 1),
        "iadd_instr_per_clk_sm": per(out[6], 1),
        "lop3_instr_per_clk_sm": per(out[7], 1),
        "cell_mix_v1_gcups": out[3] / 1e9,
        "cell_mix_gcups": out[8] / 1e9,
        "hmax2_instr_per_clk_sm": per(out[11], 2),
        "hadd2_instr_per_clk_sm": per(out[12], 2),
        "hmax2_dpx_mix_instr_per_clk_sm": per(out[13], 2),
        # 8-bit first pass (four records per register): CUDA's byte-SIMD
        # functions, and the same cell built by hand from 32-bit operations
        "cell8_intrinsics_gcups": out[14] / 1e9,
        "cell8_swar_gcups": out[15] / 1e9,
        # the batched kernel's paired-query cell (no per-row byte unpacking)
        "cell_pair_mix_gcups": out[16] / 1e9,
        "sms": int(sms), "attr_clock_mhz": mhz,
    }


# ---------------------------------------------------------------------------
def _parity_entry(n_checked, n_records, mismatches, top_equal):
    return {"queries": n_checked, "records": n_records, "mismatches": mismatches,
            "top10_equal": top_equal}


def cpu_baseline(db, queries, target_s: float, gpu=None):
    """The reference's own AVX2 kernels on a bounded sample of the sweep.

    gpu: optional {"sweep": [(hits, scores) per query], "batched": [(query,
    hits, scores)]} from the GPU run on the same DB; every record score the
    reference kernels produce here is compared with it (full-size parity)."""
    import oracle
    from swhybrid_b200 import param
    m = param.blosum62()
    threads = oracle.ref_threads()
    rdb = oracle.RefDB(db.residues, db.offsets)
    cells, secs, used = 0, 0.0, []
    bad, top_ok, checked = 0, True, 0
    order = list(range(0, len(queries), 4)) + [i for i in range(len(queries)) if i % 4]
    for i in order:
        q = queries[i]
        want, s, _ = rdb.search(q, m, 10, 2, threads=threads)
        cells += len(q) * db.total
        secs += s
        used.append(len(q))
        if gpu is not None and gpu.get("sweep"):
            hits, sc = gpu["sweep"][i]
            bad += int(np.count_nonzero(sc != want))
            top_ok &= _top_equal(hits, want)
            checked += 1
        if secs >= target_s:
            break
    parity = None
    if gpu is not None:
        parity = {"sweep": _parity_entry(checked, int(db.n), bad, bool(top_ok))}
        bb, bt = 0, True
        for q, hits, sc in gpu.get("batched", []):
            want, _, _ = rdb.search(q, m, 10, 2, threads=threads)
            bb += int(np.count_nonzero(sc != want))
            bt &= _top_equal(hits, want)
        if gpu.get("batched"):
            parity["batched"] = _parity_entry(len(gpu["batched"]), int(db.n), bb, bool(bt))
            parity["batched"]["query_lengths"] = [len(q) for q, _, _ in gpu["batched"]]
        parity["reference"] = "avxCompute + avxCompute16 (oracle/_ref), every record of the DB"
    rdb.close()
    return {"value": cells / secs / 1e9, "unit": "GCUPS", "cores": threads,
            "kind": "reference",
            "sample": f"reference avxCompute+avxCompute16 on the full {db.n}-record DB, "
                      f"query lengths {used} ({secs:.1f} s of kernel time)"}, secs, parity


def _top_equal(hits, want_scores, k=10) -> bool:
    """The GPU hit list equals the top-k of the reference scores under the
    stated order (score descending, then index ascending)."""
    import oracle
    ws, wi = oracle.topk(want_scores, k)
    return [h[0] for h in hits] == ws.tolist() and [h[1] for h in hits] == wi.tolist()


# ---------------------------------------------------------------------------
def run_reference(args, rank, world):
    """--impl reference: the reference CPU kernels only, rank 0."""
    if rank != 0:
        return
    import oracle
    from swhybrid_b200 import param
    db, queries = make_workload(args.workload, 0)
    m = param.blosum62()
    threads = oracle.ref_threads()
    rdb = oracle.RefDB(db.residues, db.offsets)
    # one step = the whole sweep, as in the GPU arm; warm-up = the shortest query
    sample = queries
    cells_step = sum(len(q) for q in sample) * db.total
    for _ in range(args.warmup):
        rdb.search(min(sample, key=len), m, 10, 2, threads=threads)
    secs = 0.0
    for _ in range(args.steps):
        for q in sample:
            secs += rdb.search(q, m, 10, 2, threads=threads)[1]
    rdb.close()
    value = cells_step * args.steps / secs / 1e9
    line = {
        "impl": "reference", "metric": METRIC, "value": round(value, 3), "unit": "GCUPS",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(secs / args.steps * 1e3, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int8/int16", "data": "synthetic",
        "config": {"workload": WORKLOADS[args.workload],
                   "sample_query_lengths": [len(q) for q in sample],
                   "l2": "DB (205 MB) larger than L2"},
        "cpu_baseline": {"value": round(value, 3), "unit": "GCUPS", "cores": threads,
                         "kind": "reference",
                         "sample": f"the whole {len(sample)}-query sweep against the full DB "
                                   f"per step, {args.steps} steps"},
        "e2e": {"value": round(value, 3), "unit": "GCUPS", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
def serve_options(args) -> dict:
    """The serving options given on the command line (others: the library's)."""
    return {k: v for k, v in (("chunks", args.serve_chunks), ("max_active", args.serve_slots),
                              ("pair_long", args.serve_pair_long),
                              ("pair_regions", args.serve_regions)) if v is not None}


def serve_leg(ctx, db, n_req: int, seed: int = 5, loads=(0.25, 0.5, 0.75, 1.0), opts=None,
              n_half: int = 0):
    """Serving: requests of lengths log-uniform 30..8,000 (seeded) against the
    resident DB through sw_serve_*.  First the saturating rate (3x the slot
    count submitted at once), then Poisson arrivals at 25/50/75/100% of it,
    n_req requests each (n_half at 50%, when larger: the first n_req of them
    are the other levels' requests); a seeded subset of every level's top-10
    lists is checked against the plain path."""
    from swhybrid_b200 import capi, synth as _synth
    rng = np.random.default_rng(seed)

    def requests(n):
        return [_synth.residues(rng, int(L)) for L in _synth.loguniform_lengths(rng, n, 30, 8000)]

    def collect(n, t_limit_s):
        got = {}
        t_end = time.time() + t_limit_s
        while len(got) < n and time.time() < t_end:
            for r in ctx.serve_poll(256, timeout_ms=100):
                got[r["id"]] = r
        return got

    ctx.serve_start(**(opts or {}))
    try:
        slots = int(ctx.serve_stats().slots)
        # saturating rate: a full queue, throughput from first submit to last completion
        sat_q = requests(3 * slots)
        st_a = ctx.serve_stats()
        t0 = capi.serve_clock_ms()
        for i, q in enumerate(sat_q):
            ctx.serve_submit(i, q)
        got = collect(len(sat_q), 600)
        t1 = max(r["done_ms"] for r in got.values())
        st_b = ctx.serve_stats()
        sat_cells = sum(len(q) for q in sat_q) * db.total
        sat_rate = len(sat_q) / ((t1 - t0) * 1e-3)
        levels = []
        check_ids = []
        base = 1_000_000
        level_qs = requests(max(n_req, n_half))   # the same requests at every offered load
        for frac in loads:
            n_l = max(n_req, n_half) if frac == 0.5 else n_req
            qs = level_qs[:n_l]
            arr = _synth.poisson_arrivals(rng, n_l, frac * sat_rate)
            st0 = ctx.serve_stats()
            t_start = time.perf_counter()
            for i, (q, ta) in enumerate(zip(qs, arr)):
                delay = ta - (time.perf_counter() - t_start)
                if delay > 0:
                    time.sleep(delay)
                ctx.serve_submit(base + i, q)
            got_l = collect(n_l, 600)
            st1 = ctx.serve_stats()
            lat = np.array([r["done_ms"] - r["submit_ms"] for r in got_l.values()])
            wait = np.array([r["start_ms"] - r["submit_ms"] for r in got_l.values()])
            first = min(r["submit_ms"] for r in got_l.values())
            last = max(r["done_ms"] for r in got_l.values())
            cells = sum(len(q) for q in qs) * db.total
            levels.append({
                "offered_fraction": frac,
                "offered_rate_per_s": round(frac * sat_rate, 3),
                "requests": n_l, "completed": len(got_l),
                "ok": int(sum(1 for r in got_l.values() if r["status"] == 0)),
                "latency_ms_p50": round(float(np.percentile(lat, 50)), 1),
                "latency_ms_p99": round(float(np.percentile(lat, 99)), 1),
                "latency_ms_p999": round(float(np.percentile(lat, 99.9)), 1),
                "queue_wait_ms_p50": round(float(np.percentile(wait, 50)), 1),
                "gcups": round(cells / ((last - first) * 1e-3) / 1e9, 1),
                "device_ms": round(st1.device_ms - st0.device_ms, 1),
                "rounds": int(st1.rounds - st0.rounds),
                "launches": int(st1.launches - st0.launches),
            })
            sel = rng.choice(n_l, size=min(8, n_l), replace=False)
            check_ids += [(qs[i], got_l.get(base + i)) for i in sel]
            base += 1_000_000
        st = ctx.serve_stats()
    finally:
        ctx.serve_stop()
    exact = all(r is not None and r["status"] == 0 and r["hits"] == ctx.search(q)[0]
                for q, r in check_ids)
    return {
        "workload": "requests of lengths log-uniform 30..8,000 (seeded) against the full-size DB; "
                    "saturating rate from %d requests queued at once, then Poisson arrivals at "
                    "%s%% of it, the same %d requests at every level%s" % (
                        3 * slots, "/".join(f"{100 * f:g}" for f in loads), n_req,
                        " (%d at 50%%, the first %d of them the same)" % (n_half, n_req)
                        if n_half > n_req and 0.5 in loads else ""),
        "slots": slots, "chunks": int(st.chunks),
        "saturated": {"requests": len(sat_q), "rate_per_s": round(sat_rate, 3),
                      "gcups": round(sat_cells / ((t1 - t0) * 1e-3) / 1e9, 1),
                      "wall_ms": round(t1 - t0, 1),
                      "device_ms": round(st_b.device_ms - st_a.device_ms, 1),
                      "device_gcups": round(sat_cells / max(st_b.device_ms - st_a.device_ms,
                                                            1e-9) * 1e-6, 1),
                      "rounds": int(st_b.rounds - st_a.rounds),
                      "launches": int(st_b.launches - st_a.launches)},
        "levels": levels,
        "top10_equal_plain": {"checked": len(check_ids), "all_equal": bool(exact)},
        "rescored": int(st.rescored),
    }


def stress_leg(local_rank: int, steps: int):
    """Overflow / long-record stress: 100,000 records + 1 % long (10,000..40,000)
    with 0.5 % planted homologs of eight queries of 500..4,000 residues; GCUPS
    of the resident path, and how many records the reference's int8 pass
    would hand to its int16 re-score (score >= 117) on the same inputs."""
    import torch
    from swhybrid_b200 import capi, synth as _synth
    db, queries, picks, _ = _synth.stress_workload()
    ctx = capi.Context(local_rank, capi.default_params(top_k=10))
    try:
        ctx.load_db(db.residues, db.offsets)
        from swhybrid_b200 import autotune
        autotune.apply(ctx)
        over8 = 0
        for q in queries:
            _, sc = ctx.search(q, want_scores=True)
            over8 += int((sc >= 117).sum())
        stream = torch.cuda.Stream(device=local_rank)
        ctx.set_stream(stream.cuda_stream)
        dq = [torch.from_numpy(q.copy()).to(f"cuda:{local_rank}") for q in queries]
        for q in dq:
            ctx.search_device(q.data_ptr(), q.numel())
        ctx.sync()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(steps):
            for q in dq:
                ctx.search_device(q.data_ptr(), q.numel())
        ev1.record(stream)
        ctx.sync()
        torch.cuda.synchronize()
        ms = ev0.elapsed_time(ev1)
        cells = sum(len(q) for q in queries) * int(db.offsets[-1]) * steps
        return {
            "workload": "100,000 records lognormal(5.6,0.6) 20..5,000 + 1% uniform 10,000..40,000, "
                        "0.5% homologs of the queries (sub 10..30%, indels 2%), 8 queries 500..4,000",
            "n_residues": int(db.offsets[-1]), "planted": int(len(picks)),
            "value": round(cells / (ms * 1e-3) / 1e9, 1), "unit": "GCUPS",
            "ms_per_pass_of_8": round(ms / steps, 2),
            "records_over_int8_range": over8,
        }
    finally:
        ctx.close()


def run_ours(args, rank, world, local_rank):
    import torch
    from swhybrid_b200 import capi
    dist = None
    if world > 1:
        import torch.distributed as dist

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        if dist is None:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=f"cuda:{local_rank}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    torch.cuda.set_device(local_rank)
    t0 = time.time()
    db, queries = make_workload(args.workload, rank)
    gen_s = time.time() - t0
    ctx = capi.Context(local_rank, capi.default_params(top_k=10))
    t0 = time.time()
    ctx.load_db(db.residues, db.offsets)
    load_s = time.time() - t0
    from swhybrid_b200 import autotune
    tuned = autotune.apply(ctx)
    if args.config:
        ctx.set_kernel_config(tuple(int(x) for x in args.config.split(",")))
    stream = torch.cuda.Stream(device=local_rank)
    ctx.set_stream(stream.cuda_stream)
    dq = [torch.from_numpy(q.copy()).to(f"cuda:{local_rank}") for q in queries]
    torch.cuda.synchronize()
    cells_step = sum(len(q) for q in queries) * db.total

    # ---- warm-up ----
    for _ in range(args.warmup):
        for q in dq:
            ctx.search_device(q.data_ptr(), q.numel())
    ctx.sync()

    # ---- timed: resident path ----
    ctx.reset_totals()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            for q in dq:
                ctx.search_device(q.data_ptr(), q.numel())
        ev1.record(stream)
        ctx.sync()
        torch.cuda.synchronize()
    clocks = clk.summary()
    barrier()
    dev_ms = ev0.elapsed_time(ev1)
    tot = ctx.totals()
    dev_ms_max = max_over_ranks(dev_ms)
    value = cells_step * args.steps * world / (dev_ms_max * 1e-3) / 1e9

    if args.kernel_only:
        if rank == 0:
            print(json.dumps({"kernel_only": True, "value": round(value, 3), "unit": "GCUPS",
                              "ms": round(dev_ms_max, 3),
                              "first_pass_launches": int(tot.first_pass_launches),
                              "config": list(ctx.kernel_config(len(queries[0])))}), flush=True)
        ctx.close()
        return None, db, queries, None

    # ---- timed: end to end through sw_search (host buffers) ----
    ctx.set_stream(None)
    hq = [np.ascontiguousarray(q) for q in queries]
    for q in hq[:2]:
        ctx.search(q)
    per_query = []
    barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        for q in hq:
            ctx.search(q)
            st = ctx.run_stats()
            per_query.append((len(q), st.total_ms, st.kernel_ms))
    e2e_s = time.perf_counter() - t0
    barrier()
    e2e_s_max = max_over_ranks(e2e_s)
    e2e_value = cells_step * args.steps * world / e2e_s_max / 1e9

    # every record's score for the sweep, checked against the reference's own
    # kernels by the CPU-baseline leg (untimed)
    gpu_scores = None
    if rank == 0 and world == 1 and args.workload == "full" and not args.no_cpu_baseline:
        gpu_scores = {"sweep": [ctx.search(q, want_scores=True) for q in hq], "batched": []}

    # ---- batched: 64 queries, lengths log-uniform 50..5,000, one call ----
    batched = None
    if args.workload == "full" and not args.no_batched:
        from swhybrid_b200 import synth as _synth
        bq = _synth.batched_queries(3, 64, 50, 5000)
        bcells = sum(len(q) for q in bq) * db.total
        ctx.search_batch(bq)                       # capture the graph
        ctx.search_batch(bq)
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        bdev = 0.0
        b_launches = 0
        for _ in range(args.steps):
            ctx.search_batch(bq)
            st_b = ctx.run_stats()
            bdev += st_b.kernel_ms
            b_launches = int(st_b.launches)
        b_wall = time.perf_counter() - t0
        barrier()
        bdev_max = max_over_ranks(bdev)
        b_wall_max = max_over_ranks(b_wall)
        # the same 64 queries through the plain one-query-per-call path
        ctx.set_stream(stream.cuda_stream)
        dbq = [torch.from_numpy(q.copy()).to(f"cuda:{local_rank}") for q in bq]
        pev0 = torch.cuda.Event(enable_timing=True)
        pev1 = torch.cuda.Event(enable_timing=True)
        pev0.record(stream)
        for q in dbq:
            ctx.search_device(q.data_ptr(), q.numel())
        pev1.record(stream)
        ctx.sync()
        torch.cuda.synchronize()
        plain_ms = max_over_ranks(pev0.elapsed_time(pev1))
        ctx.set_stream(None)
        if gpu_scores is not None:
            # the shortest, the longest and two middle queries of the batch
            bh, bs = ctx.search_batch(bq, want_scores=True)
            order = np.argsort([len(q) for q in bq], kind="stable")
            picks = sorted({int(order[0]), int(order[len(bq) // 3]),
                            int(order[2 * len(bq) // 3]), int(order[-1])})
            gpu_scores["batched"] = [(bq[i], bh[i], bs[i].copy()) for i in picks]
            del bs
        batched = {
            "workload": "64 queries, lengths log-uniform 50..5,000 (seeded), full-size DB, "
                        "one sw_search_batch call (CUDA graph replay)",
            "value": round(bcells * args.steps * world / (bdev_max * 1e-3) / 1e9, 3),
            "e2e_value": round(bcells * args.steps * world / b_wall_max / 1e9, 3),
            "unit": "GCUPS",
            "ms_per_batch": round(bdev_max / args.steps, 3),
            "plain_same_queries_gcups": round(bcells * world / (plain_ms * 1e-3) / 1e9, 3),
            "speedup_vs_plain": round((bcells / (bdev_max / args.steps)) / (bcells / plain_ms), 3),
            "launches_per_batch": b_launches,
        }

    # ---- serving: continuous batching under Poisson arrivals (one GPU: the
    # serving and stress legs are single-GPU measurements, so a multi-GPU run
    # holds its GPUs only for the sharded sweep and the batched leg) ----
    served = None
    if args.workload == "full" and args.serve_requests > 0 and world == 1:
        ctx.set_stream(None)
        served = serve_leg(ctx, db, args.serve_requests,
                           loads=tuple(float(x) for x in args.serve_levels.split(",") if x),
                           opts=serve_options(args), n_half=args.serve_half_requests)

    # ---- overflow / long-record stress (its own DB and context) ----
    stress = None
    if args.workload == "full" and not args.no_stress and world == 1:
        stress = stress_leg(local_rank, args.steps)

    # ---- correctness spot check on the resident DB (rank 0, cheap) ----
    spot = None
    if rank == 0 and args.workload == "small":
        import oracle
        from swhybrid_b200 import param
        _, sc = ctx.search(queries[0], want_scores=True)
        want = oracle.search(queries[0], db.residues, db.offsets, param.blosum62(), 12, 2)
        spot = bool(np.array_equal(sc, want))

    line = None
    if rank == 0:
        peaks, peak_kind = measured_peaks()
        rates = probe_rates(local_rank)
        fp_gcups = tot.cells / (tot.first_pass_ms * 1e-3) / 1e9 if tot.first_pass_ms else None
        st = ctx.db_stats()
        lens = [L for (L, _, _) in per_query]
        lat = np.array([t for (_, t, _) in per_query])
        kernel_lat = np.array([k for (_, _, k) in per_query])
        gcups_by_len = {}
        for (L, tms, kms) in per_query:
            gcups_by_len.setdefault(int(L), []).append(L * db.total / (kms * 1e-3) / 1e9)
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": "GCUPS",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(dev_ms_max / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int16x2 (int32 re-score)",
            "data": "synthetic (seeded; Robinson & Robinson 1991 residue frequencies)",
            "config": {"workload": WORKLOADS[args.workload], "n_records": int(db.n),
                       "n_residues": int(db.total), "query_lengths": [len(q) for q in queries],
                       "top_k": 10, "gaps": "open 10 / extend 2", "matrix": "BLOSUM62",
                       "l2": "inputs larger than L2 (DB column streams ~%d MB)" %
                             (st.device_bytes // 9 // 2**20),
                       "tuning_table": "swhybrid_b200/tuned/b200.json" if tuned else "cost model",
                       "kernel_config_q144": list(ctx.kernel_config(144)),
                       "kernel_config_q5478": list(ctx.kernel_config(5478)),
                       "row_segment_plans": {str(L): [list(st) for st in p] for L, p in
                                             ((L, ctx.plan(L)) for L in sorted({len(q) for q in queries}))
                                             if len(p) > 1},
                       "db_generate_s": round(gen_s, 2), "db_load_s": round(load_s, 2)},
            "gpu_launches": int(tot.launches),
            "clocks": clocks,
            "e2e": {"value": round(e2e_value, 3), "unit": "GCUPS",
                    "h2d_bytes_per_step": int(sum(len(q) for q in queries)),
                    "d2h_bytes_per_step": int(len(queries) * 10 * 8),
                    "latency_ms_p50": round(float(np.percentile(lat, 50)), 3),
                    "latency_ms_p99": round(float(np.percentile(lat, 99)), 3)},
            "per_query_gcups": {str(k): round(float(np.median(v)), 1)
                                for k, v in sorted(gcups_by_len.items())},
            "roofline": {
                "bound": "int_alu (packed int16x2 DPX)",
                "achieved": round(fp_gcups, 1) if fp_gcups else None,
                "peak": round(rates["cell_mix_gcups"], 1),
                "unit": "GCUPS",
                "frac": round(fp_gcups / rates["cell_mix_gcups"], 4) if fp_gcups else None,
                # DRAM bytes (read + write) of one bulk first-pass launch, from the ncu
                # capture of sw_wavefront<16,48,256> on this DB with the 1,434-residue
                # query (dram__bytes_read.sum 1.87 GB + dram__bytes_write.sum 1.61 GB):
                # the 194 MB column stream once per pass plus the pass-boundary rows
                # (16 B per column written by pass 0, read by pass 1).  At 3.5 TCUPS
                # that is ~43 GB/s, far below HBM: the kernel is ALU-bound.
                "traffic": 3.48e9,
                "traffic_unit": "bytes per launch (query 1,434, 2 passes)",
                "algorithmic_bytes_per_launch": 194_000_000,   # the DB column stream, read once
                "peak_source": "measured live: libswprobe cell-mix kernel (first-pass "
                               "instruction mix from registers, full occupancy)",
                "first_pass_launches": int(tot.first_pass_launches),
                "first_pass_ms": round(tot.first_pass_ms, 3),
                "probe": {k: (round(v, 3) if isinstance(v, float) else v)
                          for k, v in rates.items()},
                "hbm_peak_gbs": peaks.get("hbm_gbs"), "hbm_peak_kind": peak_kind,
            },
        }
        if spot is not None:
            line["parity_spot_check"] = spot
        if batched is not None:
            # most of the batch runs two queries per register (no per-row byte
            # unpacking): its roofline is that cell's measured mix
            pm = rates.get("cell_pair_mix_gcups")
            batched["roofline"] = {
                "bound": "int_alu (packed int16x2 DPX, paired queries)",
                "achieved": batched["value"], "peak": round(pm, 1) if pm else None,
                "unit": "GCUPS", "frac": round(batched["value"] / pm, 4) if pm else None,
                "peak_source": "measured live: libswprobe paired-query cell mix"}
            line["batched"] = batched
        if served is not None:
            # the rounds run the same paired kernel: rate over the rounds'
            # device time against the same measured mix
            pm = rates.get("cell_pair_mix_gcups")
            dg = served["saturated"].get("device_gcups")
            served["roofline"] = {
                "bound": "int_alu (packed int16x2 DPX, paired queries)",
                "achieved": dg, "peak": round(pm, 1) if pm else None, "unit": "GCUPS",
                "frac": round(dg / pm, 4) if pm and dg else None,
                "peak_source": "measured live: libswprobe paired-query cell mix; achieved = "
                               "saturated cells / the rounds' device time (CUDA events)"}
            line["served"] = served
        if stress is not None:
            line["stress"] = stress
    ctx.close()
    return line, db, queries, gpu_scores


def run_shard(args, rank, world, local_rank, make_ctx=None, workload=None):
    """--shard: ONE DB (rank 0's seed on every rank) split into contiguous,
    residue-balanced record ranges, one per rank (swhybrid_b200/shard.py);
    every query is searched by all ranks on their shards and the k best hits
    are merged by one all-gather per query (WorkerPool's split of one DB over
    its workers, src/WorkerPool.cpp:10-105).  value = cells of the whole DB x
    the queries / the max-over-ranks time of the steps (strong scaling).

    make_ctx / workload stand in for the device context and the workload in
    the CPU test of this path (gloo ranks, the oracle as each rank's search).
    Returns (line or None, the merged hit lists of the last step)."""
    import torch
    import torch.distributed as dist
    from swhybrid_b200 import shard as _shard
    db, queries = workload if workload is not None else make_workload(args.workload, 0)
    on_gpu = make_ctx is None
    if on_gpu:
        from swhybrid_b200 import autotune, capi
        torch.cuda.set_device(local_rank)
        ctx = capi.Context(local_rank, capi.default_params(top_k=10))
    else:
        ctx = make_ctx()
    try:
        searcher = _shard.ShardedSearch(ctx, db.residues, db.offsets, rank, world)
        if on_gpu:
            autotune.apply(ctx)
        for _ in range(args.warmup):
            searcher.search(queries[0])
        dist.barrier()
        if on_gpu:
            torch.cuda.synchronize()
            ev0 = torch.cuda.Event(enable_timing=True)
            ev1 = torch.cuda.Event(enable_timing=True)
            ev0.record()
        t0 = time.perf_counter()
        merged = []
        for _ in range(args.steps):
            merged = [searcher.search(q) for q in queries]
        if on_gpu:
            ev1.record()
            torch.cuda.synchronize()
            ms = ev0.elapsed_time(ev1)
        else:
            ms = (time.perf_counter() - t0) * 1e3
        t = torch.tensor([ms], dtype=torch.float64,
                         device=f"cuda:{local_rank}" if on_gpu else "cpu")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_max = float(t.item())
        local_res = int(db.offsets[searcher.end] - db.offsets[searcher.begin])
        cells = sum(len(q) for q in queries) * db.total * args.steps
        line = None
        if rank == 0:
            line = {
                "metric": METRIC, "value": round(cells / (ms_max * 1e-3) / 1e9, 3),
                "unit": "GCUPS", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": round(ms_max / args.steps, 3), "higher_is_better": True,
                "scaling": "strong", "vs_baseline": None, "dtype": "int16x2 (int32 re-score)",
                "data": "synthetic (seeded; Robinson & Robinson 1991 residue frequencies)",
                "config": {"workload": WORKLOADS[args.workload] + "; the DB split over the ranks",
                           "n_records": int(db.n), "n_residues": int(db.total),
                           "rank0_records": [searcher.begin, searcher.end],
                           "rank0_residues": local_res, "merge": "all_gather of k hits per query"},
            }
        return line, merged
    finally:
        if on_gpu:
            ctx.close()


def run_case(args, local_rank):
    """Profiling cases (--workload batched | traceback | serve): one call of
    the batched search or of the traceback of a query's hits per step, or the
    serving leg's saturated phase once.  Batched: device time by CUDA events
    inside the library; traceback: host wall time (sw_traceback keeps no
    device timings); serve: the rounds' device time (sw_serve_stats) and wall
    time.  Prints one JSON line."""
    import torch
    from swhybrid_b200 import autotune, capi, synth
    torch.cuda.set_device(local_rank)
    db = synth.full_db(2)
    ctx = capi.Context(local_rank, capi.default_params(top_k=10))
    try:
        ctx.load_db(db.residues, db.offsets)
        autotune.apply(ctx)
        if args.workload == "serve":
            rng = np.random.default_rng(5)
            qs = [synth.residues(rng, int(L))
                  for L in synth.loguniform_lengths(rng, args.serve_requests, 30, 8000)]
            ctx.serve_start(**serve_options(args))
            try:
                t0 = capi.serve_clock_ms()
                for i, q in enumerate(qs):
                    ctx.serve_submit(i, q)
                got = {}
                while len(got) < len(qs):
                    for r in ctx.serve_poll(256, timeout_ms=200):
                        got[r["id"]] = r
                t1 = max(r["done_ms"] for r in got.values())
                st = ctx.serve_stats()
            finally:
                ctx.serve_stop()
            cells = sum(len(q) for q in qs) * db.total
            print(json.dumps({"workload": WORKLOADS[args.workload], "requests": len(qs),
                              "slots": int(st.slots), "chunks": int(st.chunks),
                              "ok": sum(1 for r in got.values() if r["status"] == 0),
                              "wall_ms": round(t1 - t0, 1), "device_ms": round(st.device_ms, 1),
                              "gcups": round(cells / ((t1 - t0) * 1e-3) / 1e9, 1),
                              "rounds": int(st.rounds), "launches": int(st.launches)}),
                  flush=True)
            return
        batched = args.workload == "batched"
        if batched:
            if args.no_pairs:        # every query in stacks (the stacked kernel alone)
                ctx.set_batch_options(pair_rows=0, pair_long=False)
            qs = synth.batched_queries(3, 64, 50, 5000)
            cells = sum(len(q) for q in qs) * db.total
            step = lambda: ctx.search_batch(qs)
        else:
            q = synth.query(112, 1434)
            hits, _ = ctx.search(q)
            recs = [i for (_, i) in hits]
            cells = sum(len(q) * len(db.record(int(i))) for i in recs)
            step = lambda: ctx.traceback(q, recs)
        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        dev = 0.0
        for _ in range(args.steps):
            step()
            if batched:
                dev += ctx.run_stats().kernel_ms
        wall = time.perf_counter() - t0
        if not batched:
            dev = wall * 1e3
        print(json.dumps({"workload": WORKLOADS[args.workload], "steps": args.steps,
                          "ms_per_step_device": round(dev / args.steps, 3),
                          "ms_per_step_wall": round(wall * 1e3 / args.steps, 3),
                          "gcups_device": round(cells * args.steps / (dev * 1e-3) / 1e9, 1)
                          if dev > 0 else None}), flush=True)
    finally:
        ctx.close()


def main(argv=None):
    args = parse(argv)
    if args.workload in ("batched", "traceback", "serve"):
        run_case(args, int(os.environ.get("LOCAL_RANK", "0")))
        return 0
    if args.workload == "probe":
        print(json.dumps(probe_rates(int(os.environ.get("LOCAL_RANK", "0")))), flush=True)
        return 0
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return 0
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        # NCCL on GPUs; gloo only where there is no GPU (the CPU test of this
        # control flow, with run_ours stood in for)
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local_rank)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    if args.shard:
        if world == 1:
            import torch.distributed as dist
            dist.init_process_group("nccl", init_method="tcp://127.0.0.1:29533", rank=0,
                                    world_size=1)
        line, _ = run_shard(args, rank, world, local_rank)
        if rank == 0:
            print(json.dumps(line), flush=True)
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
        return 0
    # every rank takes the same collective steps: only rank 0 has a line, and
    # all ranks meet at the final barrier (with or without one)
    line, db, queries, gpu_scores = run_ours(args, rank, world, local_rank)
    if line is not None and rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb, _, parity = cpu_baseline(db, queries, args.cpu_seconds, gpu_scores)
        if parity is not None:
            line["parity"] = parity
        line["cpu_baseline"] = {k: (round(v, 3) if isinstance(v, float) else v)
                                for k, v in cb.items()}
    if rank == 0 and line is not None:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
