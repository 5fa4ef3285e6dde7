"""Benchmark of the OLAP-core star-join on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = one star-join query (4-dimension probe, group-by SUM(m1) and
SUM(m1*m2) in int64) over the whole device-resident fact table of this rank:
600,000,000 rows x (4 int32 FKs + 2 int32 measures) = 14.4 GB per GPU,
dimensions of 3,000,000 / 200,000 / 1,400,000 / 2,556 rows (selectivity
0.5/0.2/0.1/1.0, 8 groups each: 4096 groups, joint selectivity 0.01).  Inputs
are larger than L2 (126 MB), so no flush is needed between steps.

Under torchrun each rank holds its own 600M-row shard (weak scaling) and the
step ends with the one real exchange of a distributed star-join: an NCCL
all-reduce of the int64 group vector.  Time is measured with CUDA events on
the launching stream and reduced as the max over ranks.

``--impl reference`` times the reference's own CPU OLAPcore (compiled from
its sources into oracle/_ref) on this host's cores instead.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "star-join fact rows/sec & HBM GB/s vs peak; queries/sec with p50/p99 latency"
WORKLOAD = ("OLAP-core star-join at scale: 600M fact rows/GPU, 4 int32 FK + 2 int32 measures "
            "(14.4 GB), dims 3,000,000/200,000/1,400,000/2,556, uniform FKs, per-dim selectivity "
            "0.5/0.2/0.1/1.0 (joint 0.01), 8x8x8x8 = 4096 groups, int64 SUM(m1) and SUM(m1*m2)")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--rows", type=int, default=600_000_000)
    ap.add_argument("--sele", type=float, nargs=4, default=[0.5, 0.2, 0.1, 1.0])
    ap.add_argument("--groups", type=int, nargs=4, default=[8, 8, 8, 8])
    ap.add_argument("--fk-dist", default="uniform", choices=["uniform", "zipf"])
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--e2e-mode", default="inplace", choices=["inplace", "copy"],
                    help="host call reads pinned columns in place (OLAP_TUNE_HOST_INPLACE) or copies them")
    ap.add_argument("--e2e-rows", type=int, default=0,
                    help="rows per rank of the e2e leg (0: the whole table at N=1, 150M per rank at N>1)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--tune", type=str, default="", help="knob=value,... (olap_ctx_set_tuning)")
    ap.add_argument("--suite", default="starjoin",
                    choices=["starjoin", "batched", "serving", "operators", "hostscan"],
                    help="starjoin: the headline line; batched: 64-query batches vs one launch per query; "
                         "serving: Poisson arrivals of the 70/30 star-join/Q5 mix, batched vs plain; "
                         "operators: select/gather/hash join/hash group-by at 2^28 rows; "
                         "hostscan: pinned host table read in place vs copied, over six pass-rate sets")
    ap.add_argument("--op-rows", type=int, default=1 << 28)
    ap.add_argument("--rates", type=float, nargs="+", default=[50, 200, 500, 1000, 2000])
    ap.add_argument("--serve-seconds", type=float, default=2.0)
    ap.add_argument("--queries", type=int, default=64)
    ap.add_argument("--batch-shape", type=str, default="",
                    help="block,slots of the batched scan (skips its autotuner), e.g. 1024,16384")
    ap.add_argument("--no-secondary", action="store_true",
                    help="headline line only (no batched / serving / operators / sweep sub-objects)")
    return ap.parse_args()


DIM_SIZES = (3_000_000, 200_000, 1_400_000, 2_556)


# ---------------------------------------------------------------------------
# clocks
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.rows: list[list[str]] = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self) -> dict:
        mhz, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in self.rows:
            try:
                mhz.append(float(r[1]))
                mx = float(r[2])
                for name, v in zip(names, r[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(name)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(mhz) if mhz else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(mhz)}


def measured_peak_gbs() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    try:
        return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ---------------------------------------------------------------------------
# CPU: the reference's own OLAPcore on this host
# ---------------------------------------------------------------------------
REF_FANOUTS = ("OLAPcore_rowwise", "OLAPcore_vwm_dv", "OLAPcore_vwm_sv")


def bench_config(a, world: int) -> dict:
    """The workload both arms run (identical dicts, so the lines compare)."""
    return {"workload": WORKLOAD, "rows_per_gpu": a.rows, "dim_sizes": list(DIM_SIZES), "sele": list(a.sele),
            "groups": list(a.groups), "fk_dist": a.fk_dist, "group_nums": int(_prod(a.groups)),
            "l2": "inputs 14.4 GB/GPU > 126 MB L2; no flush", "parallelism": f"row shards x{world}"}


def _prod(xs) -> int:
    p = 1
    for x in xs:
        p *= int(x) if int(x) else 1
    return p


def host_tables(a):
    """The benchmark's table in host memory, from the oracle's copy of the
    library's generators (bit-identical to the HBM table of rank 0)."""
    import oracle
    return oracle.star_schema(a.rows, DIM_SIZES, a.sele, a.groups, fk_dist=a.fk_dist, seed=42)


def reference_cpu(h, steps: int, warmup: int) -> dict:
    """Time the reference's own OLAPcore_rowwise, OLAPcore_vwm_dv and
    OLAPcore_vwm_sv (test_multi_compute_operator.cpp:973,1052,1258, compiled
    from its sources) on the host table ``h`` with every host thread; the
    fastest is the baseline.  Their int returns are SUM(M1+M2) modulo 2^32
    (rowwise's only when the measures are constant: it reads M1[i] with the
    thread-local index, :360).  Without the compiled reference, the oracle's
    restatement is timed instead (kind "port")."""
    import numpy as np
    import oracle
    cores = os.cpu_count() or 1
    n, nd, G = h.n_rows, h.dimvec_nums, h.group_nums
    if oracle.ref_available():
        ref, flags = oracle.ref_lib_for_host()
        o = np.array(h.orders + [0] * (4 - nd), np.int32)
        f = np.array(h.factor + [0] * (4 - nd), np.int32)
        dva, fka = oracle._ptr_array(h.dimvec), oracle._ptr_array(h.fk)
        variants = {}
        for name in REF_FANOUTS:
            fn = getattr(ref, "ref_" + name)

            def run():
                return fn(dva, fka, oracle._p(o), nd, oracle._p(f), n, G, oracle._p(h.m1), oracle._p(h.m2), cores)
            r = 0
            for _ in range(warmup):
                r = run()
            t0 = time.perf_counter()
            for _ in range(steps):
                r = run()
            dt = (time.perf_counter() - t0) / steps
            variants[name] = {"ms": dt * 1e3, "rows_per_s": n / dt, "int_return_mod_2^32": int(r) & 0xFFFFFFFF}
        best = min(variants, key=lambda k: variants[k]["ms"])
        return {"kind": "reference", "cores": cores, "ms": variants[best]["ms"], "value": n / (variants[best]["ms"] / 1e3),
                "best": best, "variants": variants, "build": flags,
                "sum_m1_plus_m2_mod_2^32": variants["OLAPcore_vwm_sv"]["int_return_mod_2^32"],
                "sample": f"all {n:,} rows of the workload; fastest of {', '.join(REF_FANOUTS)} "
                          f"(reference source, {flags}, {cores} threads), {steps} timed runs after {warmup} warm-up"}
    dims, fks = h.probe_dims, h.probe_fks
    out = None
    for _ in range(warmup):
        out = oracle.starjoin(dims, fks, h.factor, h.m1, h.m2, G, want_groups=False, nthreads=cores)
    t0 = time.perf_counter()
    for _ in range(steps):
        out = oracle.starjoin(dims, fks, h.factor, h.m1, h.m2, G, want_groups=False, nthreads=cores)
    dt = (time.perf_counter() - t0) / steps
    return {"kind": "port", "cores": cores, "ms": dt * 1e3, "value": n / dt, "best": "oracle restatement",
            "sum_m1_plus_m2_mod_2^32": int(out[1][0]) & 0xFFFFFFFF,
            "sample": f"all {n:,} rows of the workload; the oracle's restatement of OLAPcore_vwm_sv "
                      f"({cores} threads), {steps} timed runs after {warmup} warm-up"}


def run_reference_arm(a) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    world = int(os.environ.get("WORLD_SIZE", str(a.gpus)))
    h = host_tables(a)
    cb = reference_cpu(h, max(1, a.steps), max(1, a.warmup))
    line = {
        "impl": "reference", "metric": METRIC, "value": cb["value"], "unit": "rows/s",
        "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup, "ms_per_step": cb["ms"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
        "data": "synthetic (seeded counter-based generator, the oracle's host copy of the library's)",
        "config": bench_config(a, world),
        "aggregate": "SUM(M1+M2) per group in uint32 counters (the reference's only aggregate)",
        "rows_timed_per_step": h.n_rows,
        "reference_variants": cb.get("variants"),
        "check": {"sum_m1_plus_m2_mod_2^32": cb["sum_m1_plus_m2_mod_2^32"]},
        "cpu_baseline": {"value": cb["value"], "unit": "rows/s", "cores": cb["cores"], "kind": cb["kind"],
                         "sample": cb["sample"]},
        "e2e": {"value": cb["value"], "unit": "rows/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def run_batched(a) -> None:
    print(json.dumps(batched_result(a)), flush=True)


def batched_result(a) -> dict:
    """Batched configuration: Q star-join queries (own predicates, 1-3 group
    tables, 5-100% fact ranges) over the shared 600M-row table, one persistent
    launch per batch replayed as a CUDA graph, against one launch per query."""
    import numpy as np
    import torch
    from memory_database_b200 import batch, olapcore, workloads
    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx = olapcore.Context(0, scratch_bytes=512 << 20, stream=stream)
    groups = (25, 25, 40, 7)
    s = workloads.make_star_schema(ctx, a.rows, DIM_SIZES, (1, 1, 1, 1), (1, 1, 1, 1), seed=42)
    dims = batch.make_dim_tables(ctx, DIM_SIZES, groups, seed=7)
    rng = np.random.default_rng(2025)
    eng = batch.BatchEngine(ctx, dims, max_queries=a.queries)
    batches = [batch.random_queries(rng, a.queries, a.rows, groups) for _ in range(max(1, a.steps))]
    offs_max = max(sum(q.group_nums for q in qs) for qs in batches)
    out = torch.empty(offs_max, dtype=torch.int64, device="cuda")
    tot = torch.empty(a.queries, dtype=torch.int64, device="cuda")
    # launch shape (block size, shared accumulators) by the engine's autotuner, untimed
    if a.batch_shape:
        tuned_block, tuned_slots = (int(x) for x in a.batch_shape.split(","))
        eng.tune(tuned_block, tuned_slots)
    else:
        tuned_block, tuned_slots, _ = eng.autotune(batches[0], s.fk, s.m1, s.m2)
    for qs in batches[: max(1, a.warmup)]:
        eng.run(qs, s.fk, s.m1, s.m2, out=out, totals=tot)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(0) as clk:
        e0.record()
        for qs in batches:
            eng.run(qs, s.fk, s.m1, s.m2, out=out, totals=tot)
        e1.record()
        torch.cuda.synchronize()
    b_ms = e0.elapsed_time(e1) / len(batches)
    # one launch per query (dimension vectors + plain star-join), same queries
    vec_bufs = [torch.empty(n, dtype=torch.int8, device="cuda") for n in DIM_SIZES]
    gmax = max(q.group_nums for qs in batches for q in qs)
    pg = torch.empty((1, gmax), dtype=torch.int64, device="cuda")
    pt = torch.empty(1, dtype=torch.int64, device="cuda")
    qs0 = batches[0]
    for q in qs0[:3]:
        batch.run_plain(ctx, dims, q, s.fk, s.m1, s.m2, vec_buffers=vec_bufs, out=pg[:, : q.group_nums], totals_out=pt)
    torch.cuda.synchronize()
    e0.record()
    for q in qs0:
        batch.run_plain(ctx, dims, q, s.fk, s.m1, s.m2, vec_buffers=vec_bufs, out=pg[:, : q.group_nums], totals_out=pt)
    e1.record()
    torch.cuda.synchronize()
    p_ms = e0.elapsed_time(e1)
    # check (untimed): every query of the first batch equals the query run alone
    bo, bt, offs = eng.run(qs0, s.fk, s.m1, s.m2, out=out, totals=tot)
    checked = True
    for i, q in enumerate(qs0):
        batch.run_plain(ctx, dims, q, s.fk, s.m1, s.m2, vec_buffers=vec_bufs, out=pg[:, : q.group_nums],
                        totals_out=pt)
        checked &= bool(torch.equal(pg[0, : q.group_nums], bo[offs[i]: offs[i] + q.group_nums])
                        and torch.equal(pt[0], bt[i]))
    rows_scanned = sum(q.row_end - q.row_begin for q in qs0)
    line = {"metric": "batched star-join queries/sec", "value": a.queries / (b_ms / 1e3), "unit": "queries/s",
            "n_gpus": 1, "steps": len(batches), "warmup": a.warmup, "ms_per_batch": b_ms,
            "plain_ms_per_batch": p_ms, "plain_queries_per_s": a.queries / (p_ms / 1e3),
            "speedup_vs_one_launch_per_query": p_ms / b_ms, "higher_is_better": True, "clocks": clk.summary(),
            "checked": checked,
            "config": {"workload": f"{a.queries} star-join queries per batch over the shared {a.rows:,}-row table "
                                   "(joint selectivity log-uniform [1e-4, 0.3], 1-3 group tables of 25/25/40/7, "
                                   "fact range 5-100%), one persistent launch per batch replayed as a CUDA graph",
                       "fact_rows_covered_per_batch": rows_scanned,
                       "launch_shape": {"block_threads": tuned_block, "shared_accumulator_slots": tuned_slots,
                                        "parallel_probe": eng.tuning()[2],
                                        "chosen_by": "--batch-shape" if a.batch_shape
                                        else "olap_batch_autotune on a 64Mi-row sample"}},
            "data": "synthetic (seeded counter-based generator, generated in HBM)"}
    eng.close()
    ctx.close()
    return line


def run_serving(a) -> None:
    print(json.dumps(serving_result(a)), flush=True)


def serving_result(a) -> dict:
    """Serving configuration: Poisson arrivals at each rate of --rates, 70%
    star-joins of the batched configuration over the 600M-row table and 30%
    Q5 chains over SF~10-sized tables, served with continuous batching and
    with one launch per query; latency from arrival to the result on the
    host."""
    import numpy as np
    import torch
    from memory_database_b200 import batch, olapcore, q5 as Q5, serving as S, workloads
    torch.cuda.set_device(0)
    ctx = olapcore.Context(0)
    groups = (25, 25, 40, 7)
    s = workloads.make_star_schema(ctx, a.rows, DIM_SIZES, (1, 1, 1, 1), (1, 1, 1, 1), seed=42)
    dims = batch.make_dim_tables(ctx, DIM_SIZES, groups, seed=7)
    q5d = Q5.make_q5_data(ctx)
    ctx.synchronize()
    rng = np.random.default_rng(77)
    star = batch.random_queries(rng, 2000, a.rows, groups)
    q5q = Q5.random_q5_queries(rng, 500)
    batched, plain = S.gpu_servers(dims, s.fk, s.m1, s.m2, q5d, tune_queries=star[:64])
    warm = S.poisson_requests(rng, 1000.0, 64, star, q5q)
    batched.serve(S.reset(warm))
    plain.serve(S.reset(warm))
    # device time of one Q5 chain and of a 64-query Q5 batch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    qb = torch.empty((64, 25), dtype=torch.int64, device="cuda")
    qo = torch.empty(25, dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    e0.record()
    for q in q5q[:64]:
        Q5.q5(ctx, q5d, *q, out=qo)
    e1.record()
    torch.cuda.synchronize()
    q5_plain_ms = e0.elapsed_time(e1) / 64
    Q5.q5_batch(ctx, q5d, q5q[:64], out=qb)
    torch.cuda.synchronize()
    e0.record()
    for _ in range(5):
        Q5.q5_batch(ctx, q5d, q5q[:64], out=qb)
    e1.record()
    torch.cuda.synchronize()
    q5_batch_ms = e0.elapsed_time(e1) / 5
    per_rate = []
    checked = True
    for rate in a.rates:
        n = max(50, int(rate * a.serve_seconds))
        reqs = S.poisson_requests(np.random.default_rng(int(rate)), rate, n, star, q5q)
        with ClockSampler(0) as clk:
            rb = batched.serve(S.reset(reqs))
            nb = batched.batches
            rp = plain.serve(S.reset(reqs))
        sb, sp = S.summarize(rb, nb), S.summarize(rp)
        byid = {r.rid: r for r in rp}
        same = all(r.status == "ok" and byid[r.rid].status == "ok" and _same_result(r.result, byid[r.rid].result)
                   for r in rb)
        checked = checked and same
        per_rate.append({"offered_qps": rate, "requests": n,
                         "batched": {"qps": sb.qps, "p50_ms": sb.p50_ms, "p99_ms": sb.p99_ms,
                                     "mean_batch": sb.mean_batch, "by_kind": sb.by_kind},
                         "plain": {"qps": sp.qps, "p50_ms": sp.p50_ms, "p99_ms": sp.p99_ms, "by_kind": sp.by_kind},
                         "clocks": clk.summary()})
        batched.batches = 0
    top = per_rate[-1]
    line = {"metric": "serving queries/sec with p50/p99 latency", "value": top["batched"]["qps"],
            "checked": checked,
            "unit": "queries/s", "n_gpus": 1, "higher_is_better": True,
            "p50_ms": top["batched"]["p50_ms"], "p99_ms": top["batched"]["p99_ms"],
            "plain_qps": top["plain"]["qps"], "plain_p50_ms": top["plain"]["p50_ms"],
            "plain_p99_ms": top["plain"]["p99_ms"], "per_rate": per_rate,
            "q5_chain_ms": q5_plain_ms, "q5_batch64_ms": q5_batch_ms,
            "graph_captures": batched.engine.graph_captures(),
            "config": {"workload": f"Poisson arrivals at {a.rates} queries/s, {a.serve_seconds:g} s each: 70% "
                                   f"star-joins (batched configuration, {a.rows:,}-row table), 30% Q5 chains "
                                   "(5/25/100,000/1,500,000/15,000,000/60,000,000 rows, one-year date filter); "
                                   "continuous batching (<=64 per launch, 2 in flight per lane) vs one launch "
                                   "per query; latency = arrival to result on the host"},
            "data": "synthetic (seeded counter-based generator, generated in HBM)"}
    batched.engine.close()
    for c in batched.contexts:
        c.close()
    ctx.close()
    return line


def _same_result(x, y) -> bool:
    import numpy as np
    if isinstance(x, (tuple, list)):
        return len(x) == len(y) and all(_same_result(u, v) for u, v in zip(x, y))
    return bool(np.array_equal(np.asarray(x), np.asarray(y)))


def run_operators(a) -> None:
    print(json.dumps(operators_result(a)), flush=True)


def operators_result(a) -> dict:
    """Operator configuration at --op-rows int32 rows: select (col < t) to row
    ids at four selectivities, gather of 4 columns by those ids, hash join
    (2^24 unique build keys; probe keys uniform or Zipf(1.0) over them, half
    replaced by keys that match nothing), hash group-by SUM/COUNT at four
    cardinalities.  Device time per call (CUDA events, inputs resident, each
    input larger than L2); every result is checked on the device against a
    torch restatement."""
    import ctypes as C
    import torch
    from memory_database_b200 import _lib, olapcore
    from memory_database_b200.olapcore import _ptr
    L = _lib.lib
    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ctx = olapcore.Context(0, stream=stream)
    for kv in filter(None, a.tune.split(",")):
        k, v = kv.split("=")
        ctx.set_tuning(int(k), int(v))
    h = ctx.handle
    n = a.op_rows
    peak, peak_src = measured_peak_gbs()

    def gen(m, st, lo, hi):
        x = torch.empty(m, dtype=torch.int32, device="cuda")
        _lib.check(L.olap_gen_uniform_i32_dev(h, _ptr(x), m, 99, st, lo, hi), h)
        return x

    def timed(fn, reps=5, warm=2):
        for _ in range(warm):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    def entry(name, ms, alg_bytes, ok, **kw):
        gbs = alg_bytes / ms / 1e6
        d = {"op": name, "ms": ms, "rows_per_s": n / (ms / 1e3), "alg_GBs": gbs, "frac_of_peak": gbs / peak,
             "checked": bool(ok)}
        d.update(kw)
        return d

    res = []
    clk = ClockSampler(0).__enter__()  # sampled over every operator's timing
    col = gen(n, 100, 0, (1 << 20) - 1)
    cols4 = [gen(n, 101 + c, -1000, 1000) for c in range(4)]
    ids = torch.empty(n, dtype=torch.int32, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    outs = [torch.empty(n, dtype=torch.int32, device="cuda") for _ in range(4)]
    cp = (C.c_void_p * 4)(*[_ptr(x) for x in cols4])
    op = (C.c_void_p * 4)(*[_ptr(x) for x in outs])
    for sel in (0.001, 0.01, 0.1, 0.5):
        t = int(sel * (1 << 20))

        def sel_fn():
            _lib.check(L.olap_select_rowids(h, _ptr(col), n, t, _lib.CMP_LT, None, 0, _ptr(ids), _ptr(cnt)), h)
        ms = timed(sel_fn)
        k = int(cnt.item())
        got = ids[:k]
        ok = k == int((col < t).sum()) and bool((col[got.long()] < t).all()) and bool((got[1:] > got[:-1]).all())
        res.append(entry("select col<t -> row ids", ms, 4 * n + 4 * k, ok, selectivity=sel, matches=k))

        def gat_fn():
            _lib.check(L.olap_gather_i32(h, _ptr(ids), k, 4, cp, n, op), h)
        ms = timed(gat_fn)
        gl = got.long()
        ok = all(torch.equal(outs[c][:k], cols4[c][gl]) for c in range(4))
        res.append(entry("gather 4 int32 columns by row ids", ms, 36 * k, ok, selectivity=sel, k=k))
    del outs, ids, cols4
    torch.cuda.empty_cache()
    # hash join: build keys = a bijection of [0, 2^24) onto [1, 2^24] (odd multiplier mod 2^24)
    nb = 1 << 24
    bkeys = ((torch.arange(nb, device="cuda", dtype=torch.int64) * 2654435761) % nb + 1).to(torch.int32)
    bpay = gen(nb, 110, -1000, 1000)
    cap = int(L.olap_hashtable_capacity(nb))
    table = torch.empty(cap, dtype=torch.int64, device="cuda")
    words = int(L.olap_hashjoin_filter_words(nb))
    bloom = torch.empty(words, dtype=torch.int64, device="cuda")

    def build_fn():
        _lib.check(L.olap_hashjoin_build_filtered(h, _ptr(bkeys), _ptr(bpay), nb, _ptr(table), cap, _ptr(bloom),
                                                  words), h)
    ms = timed(build_fn, reps=3)
    res.append(entry("hash join build (2^24 unique keys; table + Bloom filter)", ms, 16 * nb, True, build_rows=nb,
                     capacity=cap, filter_bytes=8 * words))
    dense = torch.zeros(nb + 1, dtype=torch.int64, device="cuda")
    dense[bkeys.long()] = bpay.long()
    s_ = torch.zeros(1, dtype=torch.int64, device="cuda")
    m_ = torch.zeros(1, dtype=torch.int64, device="cuda")
    miss = gen(n, 112, 0, 1) == 0
    for dist in ("uniform", "zipf1.0"):
        idx = torch.empty(n, dtype=torch.int32, device="cuda")
        if dist == "uniform":
            _lib.check(L.olap_gen_uniform_i32_dev(h, _ptr(idx), n, 99, 111, 0, nb - 1), h)
        else:
            _lib.check(L.olap_gen_zipf_i32_dev(h, _ptr(idx), n, 99, 113, nb, 1.0), h)
        pk = bkeys[idx.long()]
        pk = torch.where(miss, pk + nb + 7, pk).contiguous()   # half match nothing
        del idx

        def probe_fn():
            _lib.check(L.olap_hashjoin_probe_filtered(h, _ptr(table), cap, _ptr(bloom), words, _ptr(pk), n, _ptr(s_),
                                                      _ptr(m_), None, None), h)
        ms = timed(probe_fn)
        inr = pk <= nb
        exp_s = int(dense[torch.where(inr, pk, 0).long()].sum())
        ok = int(s_.item()) == exp_s and int(m_.item()) == int(inr.sum())
        res.append(entry("hash join probe (SUM payload, 50% match)", ms, 12 * n, ok, keys=dist,
                         matches=int(m_.item())))
        del pk, inr
    del table, bloom, dense, bkeys, bpay, miss
    torch.cuda.empty_cache()
    vals = gen(n, 120, 1, 10000)
    for G, dist in ((16, "uniform"), (1 << 12, "uniform"), (1 << 20, "uniform"), (1 << 22, "uniform"),
                    (1 << 20, "zipf1.0")):
        if dist == "uniform":
            keys = gen(n, 121, 0, G - 1)
        else:
            keys = torch.empty(n, dtype=torch.int32, device="cuda")
            _lib.check(L.olap_gen_zipf_i32_dev(h, _ptr(keys), n, 99, 122, G, 1.0), h)
        gcap = int(L.olap_group_hash_capacity(G))
        ok_, os_, oc_ = (torch.empty(gcap, dtype=t, device="cuda") for t in (torch.int32, torch.int64, torch.int64))
        g_ = torch.zeros(1, dtype=torch.int64, device="cuda")

        def grp_fn():
            _lib.check(L.olap_group_hash(h, n, _ptr(keys), 0, _ptr(vals), None, gcap, _ptr(ok_), _ptr(os_),
                                         _ptr(oc_), _ptr(g_)), h)
        ms = timed(grp_fn, reps=3)
        k = int(g_.item())
        es = torch.zeros(G, dtype=torch.int64, device="cuda").index_add_(0, keys.long(), vals.long())
        ec = torch.bincount(keys.long(), minlength=G)
        gs = torch.zeros(G, dtype=torch.int64, device="cuda")
        gc = torch.zeros(G, dtype=torch.int64, device="cuda")
        gs[ok_[:k].long()] = os_[:k]
        gc[ok_[:k].long()] = oc_[:k]
        ok = k == int((ec > 0).sum()) and torch.equal(gs, es) and torch.equal(gc, ec)
        res.append(entry("hash group-by SUM/COUNT", ms, 8 * n, ok, groups=G, keys=dist))
        del keys, ok_, os_, oc_
    clk.__exit__(None, None, None)
    line = {"metric": "operator rows/sec and HBM GB/s vs peak", "value": min(r["frac_of_peak"] for r in res),
            "unit": "min fraction of peak over the operators", "n_gpus": 1, "rows": n, "operators": res,
            "peak_GBs": peak, "peak_source": peak_src, "all_checked": all(r["checked"] for r in res),
            "clocks": clk.summary(),
            "config": {"workload": f"operator set at {n:,} int32 rows (select at 0.001/0.01/0.1/0.5, gather of 4 "
                                   "columns, hash join 2^24 build / uniform and Zipf(1.0) probes at 50% match, "
                                   "hash group-by at 16/4096/2^20/2^22 uniform groups and 2^20 Zipf(1.0) groups)"},
            "data": "synthetic (seeded counter-based generator, generated in HBM)"}
    ctx.close()
    return line


def run_hostscan(a) -> None:
    """Host-resident star-join through olap_starjoin_groupsum_host, the fact
    table (--rows rows, the headline's columns) in pinned host memory: the
    in-place scan (OLAP_TUNE_HOST_INPLACE) against the chunked copies, over
    six sets of per-dimension pass rates.  Wall clock around the synchronous
    call (3 calls after one warm-up each); bytes moved as the library counts
    them; both paths' sums compared."""
    import numpy as np
    import torch
    from memory_database_b200 import _lib, olapcore, workloads
    torch.cuda.set_device(0)
    n = a.rows
    ctx = olapcore.Context(0, scratch_bytes=1 << 30)
    s = workloads.make_star_schema(ctx, n, DIM_SIZES, a.sele, a.groups, fk_dist=a.fk_dist, seed=42)
    pin = [torch.empty(n, dtype=torch.int32, pin_memory=True) for _ in range(6)]
    for t, col in enumerate(list(s.fk) + [s.m1, s.m2]):
        pin[t].copy_(col)
    del s
    torch.cuda.empty_cache()
    rng = np.random.default_rng(1)
    factor = [512, 64, 8, 1]
    aggs = (olapcore.AGG_M1, olapcore.AGG_M1_TIMES_M2)
    sweep = []
    with ClockSampler(0) as clk:
        for sele in [(1, 1, 1, 1), (0.5, 0.2, 0.1, 1.0), (0.3, 0.3, 0.3, 0.3), (0.1, 1, 1, 1), (0.01, 1, 1, 1),
                     (0.001, 1, 1, 1)]:
            dims = []
            for t in range(4):
                c = rng.integers(0, 8, DIM_SIZES[t]).astype(np.int8)
                c[rng.random(DIM_SIZES[t]) >= sele[t]] = 127
                dims.append(c)
            row = {"pass_rates": list(sele)}
            outs = []
            for mode, knob in (("inplace", 3), ("copy", 2)):  # each path forced
                ctx.set_tuning(_lib.TUNE_HOST_INPLACE, knob)

                def call():
                    return olapcore.starjoin_groupsum(dims, pin[:4], factor, pin[4], pin[5], 4096, aggs=aggs, ctx=ctx)
                outs.append(call())
                ctx.take_host_bytes()
                t0 = time.perf_counter()
                for _ in range(3):
                    call()
                dt = (time.perf_counter() - t0) / 3
                moved = ctx.take_host_bytes() / 3
                row[mode] = {"ms": dt * 1e3, "rows_per_s": n / dt, "host_bytes_per_row": moved / n,
                             "link_GBs": moved / dt / 1e9}
            row["same_sums"] = bool(np.array_equal(outs[0][0], outs[1][0]) and np.array_equal(outs[0][1], outs[1][1]))
            sweep.append(row)
    head = sweep[1]
    line = {"metric": "host-resident star-join rows/s (fact table in pinned host memory)",
            "value": head["inplace"]["rows_per_s"], "unit": "rows/s", "n_gpus": 1, "higher_is_better": True,
            "copy_path_rows_per_s": head["copy"]["rows_per_s"], "sweep": sweep,
            "all_checked": all(r["same_sums"] for r in sweep), "clocks": clk.summary(),
            "config": {"workload": f"star-join over {n:,} pinned host rows (4 int32 keys + 2 int32 measures), "
                                   "dimensions 3,000,000/200,000/1,400,000/2,556, 8 groups each, "
                                   "SUM(m1) and SUM(m1*m2); six sets of pass rates"},
            "data": "synthetic (seeded counter-based generator for the fact table, numpy for the dimensions)"}
    print(json.dumps(line), flush=True)


def main() -> None:
    a = parse()
    if a.impl == "reference":
        run_reference_arm(a)
        return
    if a.suite == "batched":
        run_batched(a)
        return
    if a.suite == "serving":
        run_serving(a)
        return
    if a.suite == "operators":
        run_operators(a)
        return
    if a.suite == "hostscan":
        run_hostscan(a)
        return
    import torch
    import torch.distributed as dist
    from memory_database_b200 import _lib, olapcore, workloads
    from memory_database_b200.distributed import reduce_group_sums

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)  # kernels and timing events share this stream
    ctx = olapcore.Context(local, scratch_bytes=512 << 20, stream=stream)
    for kv in filter(None, a.tune.split(",")):
        k, v = kv.split("=")
        ctx.set_tuning(int(k), int(v))

    # dimension vectors replicated on every rank, fact rows a shard per rank
    s = workloads.make_star_schema(ctx, a.rows, DIM_SIZES, a.sele, a.groups, fk_dist=a.fk_dist,
                                   seed=42, fact_seed=42 + 1000 * rank)
    aggs = (olapcore.AGG_M1, olapcore.AGG_M1_TIMES_M2)
    G = s.group_nums
    gs = torch.empty((2, G), dtype=torch.int64, device="cuda")
    tot = torch.empty((2,), dtype=torch.int64, device="cuda")

    # Plan choice for this query shape: the library's autotuner times its
    # candidate plans on a 64Mi-row sample of this rank's table (untimed).
    if a.tune:
        knobs = [0] * 17
        for kv in filter(None, a.tune.split(",")):
            k, v = kv.split("=")
            knobs[int(k)] = int(v)
    else:
        knobs, _ = olapcore.autotune(s.probe_dims, s.probe_fks, s.factor, s.m1, s.m2, G, aggs=aggs,
                                     dimvec_lens=s.probe_lens, ctx=ctx)
        knobs = list(knobs) + [0] * (17 - len(knobs))  # the star-join knobs; join_build is not one
    plan = {name: knobs[k] for k, name in enumerate(
        ["block_threads", "blocks_per_sm", "smem_dim_bytes", "smem_acc_bytes", "host_chunk_rows",
         "rows_per_thread_mode", "probe_bits", "smem_bits_bytes", "group_combine", "group_plan", "async_loads", "compact",
         "smem_nib_bytes", "host_inplace", "merge_probes", "probe_order", "join_build"]) if knobs[k]}

    # kernels per query with this plan (the star-join and its staging prepasses)
    per_query = olapcore.launch_count(s.probe_dims, s.probe_fks, s.factor, s.m1, s.m2, G, aggs=aggs,
                                      dimvec_lens=s.probe_lens, ctx=ctx)

    def step():
        olapcore.starjoin_groupsum(s.probe_dims, s.probe_fks, s.factor, s.m1, s.m2, G, aggs=aggs,
                                   dimvec_lens=s.probe_lens, ctx=ctx, out=gs, totals_out=tot)
        if world > 1:
            reduce_group_sums(gs)

    for _ in range(max(3, a.warmup)):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(a.steps)]
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record()
        for k in range(a.steps):
            ev[k][0].record()
            olapcore.starjoin_groupsum(s.probe_dims, s.probe_fks, s.factor, s.m1, s.m2, G,
                                       aggs=aggs, dimvec_lens=s.probe_lens, ctx=ctx, out=gs,
                                       totals_out=tot)
            ev[k][1].record()
            if world > 1:
                reduce_group_sums(gs)
        t1.record()
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
    elapsed_ms = t0.elapsed_time(t1)
    kernel_ms = statistics.mean(e0.elapsed_time(e1) for e0, e1 in ev)
    if world > 1:
        t = torch.tensor([elapsed_ms, kernel_ms], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        elapsed_ms, kernel_ms = t.tolist()
    ms_per_step = elapsed_ms / a.steps
    rows_all = a.rows * world * a.steps
    value = rows_all / (elapsed_ms / 1e3)

    algo_bytes = a.rows * s.bytes_per_row(2)
    peak, peak_src = measured_peak_gbs()
    achieved = algo_bytes / (kernel_ms / 1e3) / 1e9
    traffic = None
    prof = ROOT / "profiles" / "starjoin_traffic.json"
    if prof.exists():
        try:
            tr = json.loads(prof.read_text())
            traffic = tr["bytes_per_row"] * a.rows if tr.get("workload") == WORKLOAD else None
        except Exception:
            traffic = None

    # The timed query's result, and SUM(M1+M2) on the same table, the
    # reference's own aggregate (its int return is that modulo 2^32): both
    # untimed, for the parity check of the CPU-baseline leg.
    gs_h = tot_h = None
    if world == 1:
        gs_h, tot_h = gs.cpu().numpy(), tot.cpu().numpy()
    _, tot_pm = olapcore.starjoin_groupsum(s.probe_dims, s.probe_fks, s.factor, s.m1, s.m2, G,
                                           aggs=(olapcore.AGG_M1_PLUS_M2,), dimvec_lens=s.probe_lens,
                                           want_groups=False, ctx=ctx)
    sum_pm = int(tot_pm.cpu()[0])
    range_errors = ctx.take_range_errors()

    line = {
        "metric": METRIC, "value": value, "unit": "rows/s", "n_gpus": world, "steps": a.steps,
        "warmup": max(3, a.warmup), "ms_per_step": ms_per_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int64",
        "data": "synthetic (seeded counter-based generator, generated in HBM)",
        "config": bench_config(a, world),
        "aggregate": "SUM(m1) and SUM(m1*m2) per group, int64",
        "plan": plan or "automatic",
        "exchange": "NCCL all-reduce of the int64 group vector" if world > 1 else None,
        "check": {"sum_m1_plus_m2_mod_2^32": sum_pm & 0xFFFFFFFF, "range_errors": range_errors},
        "hbm_gbs": achieved,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "peak_source": f"{peak_src} MEASURED_PEAKS.json hbm_gbs" if peak_src == "measured" else "fallback 6650 GB/s",
                     "algorithmic_bytes_per_launch": algo_bytes, "kernel_ms": kernel_ms},
        "gpu_launches": a.steps * per_query,
        "clocks": clk.summary(),
    }

    # e2e: the same query through the host-memory C-ABI entry point, with the
    # fact table in pinned host memory; H2D copies and the D2H of the group
    # sums are inside the timed region.
    if not a.no_e2e:
        line["e2e"] = e2e_host(a, s, ctx, aggs, world, knobs)
        line["gpu_launches"] = a.steps * per_query + line["e2e"].pop("_launches") * (
            1 if a.e2e_mode == "inplace" else per_query)
    if rank == 0 and world == 1 and not a.no_cpu:
        line["cpu_baseline"], line["parity"] = cpu_leg(a, gs_h, tot_h, sum_pm)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0 and world == 1 and not a.no_secondary:
        del s, gs, tot
        torch.cuda.empty_cache()
        line["secondary"] = secondary_results(a, ctx)
    if rank == 0:
        print(json.dumps(line), flush=True)
    ctx.close()


def secondary_results(a, ctx) -> dict:
    """Compact, time-bounded lines of the other configurations, measured in
    the same run on the same GPU (each with its own clock record): the
    batched launch (64 queries) against one launch per query, serving at one
    offered rate, the operator set at 2^28 rows, and three points of the
    star-join sweep.  Each sub-run checks its results (batched and serving
    against the same queries run alone or one launch each, operators against
    a torch restatement on the device)."""
    import copy
    import torch
    out = {}
    main_stream = torch.cuda.current_stream()  # the sub-runs make their own streams current
    b = copy.copy(a)
    b.steps = min(a.steps, 10)
    b.warmup = min(a.warmup, 3)
    try:
        r = batched_result(b)
        out["batched"] = {k: r[k] for k in ("value", "unit", "ms_per_batch", "plain_ms_per_batch",
                                            "plain_queries_per_s", "speedup_vs_one_launch_per_query",
                                            "steps", "clocks", "checked")}
        out["batched"]["queries_per_batch"] = a.queries
        out["batched"]["launch_shape"] = r["config"]["launch_shape"]
    except Exception as e:
        out["batched"] = {"error": str(e)[:300]}
    torch.cuda.set_stream(main_stream)
    torch.cuda.empty_cache()
    try:
        b.rates = [2000.0]
        b.serve_seconds = 2.0
        r = serving_result(b)
        pr = r["per_rate"][0]
        out["serving"] = {"offered_qps": pr["offered_qps"], "requests": pr["requests"],
                          "qps": pr["batched"]["qps"], "p50_ms": pr["batched"]["p50_ms"],
                          "p99_ms": pr["batched"]["p99_ms"], "mean_batch": pr["batched"]["mean_batch"],
                          "plain_qps": pr["plain"]["qps"], "plain_p50_ms": pr["plain"]["p50_ms"],
                          "plain_p99_ms": pr["plain"]["p99_ms"], "clocks": pr["clocks"],
                          "checked": r.get("checked"), "mix": "70% star-joins, 30% Q5 chains"}
    except Exception as e:
        out["serving"] = {"error": str(e)[:300]}
    torch.cuda.set_stream(main_stream)
    torch.cuda.empty_cache()
    try:
        r = operators_result(b)
        out["operators"] = {"rows": r["rows"], "all_checked": r["all_checked"], "peak_GBs": r["peak_GBs"],
                            "clocks": r["clocks"],
                            "ops": [{k: v for k, v in o.items() if k in ("op", "ms", "alg_GBs", "frac_of_peak",
                                                                         "selectivity", "keys", "groups", "checked")}
                                    for o in r["operators"]]}
    except Exception as e:
        out["operators"] = {"error": str(e)[:300]}
    torch.cuda.set_stream(main_stream)
    torch.cuda.empty_cache()
    out["sweep"] = []
    for name, sele, groups, dist in (("zipf0.8", a.sele, a.groups, "zipf"),
                                     ("joint_sel_0.52", [0.85] * 4, a.groups, "uniform"),
                                     ("groups_2^20", a.sele, [32] * 4, "uniform")):
        try:
            out["sweep"].append(sweep_point(a, ctx, name, sele, groups, dist))
        except Exception as e:
            out["sweep"].append({"point": name, "error": str(e)[:300]})
        torch.cuda.empty_cache()
    return out


def sweep_point(a, ctx, name, sele, groups, fk_dist) -> dict:
    """One star-join point of the sweep over the full 600M-row table: the
    autotuned plan, 10 timed launches (CUDA events on the context stream)."""
    import torch
    from memory_database_b200 import olapcore, workloads
    s = workloads.make_star_schema(ctx, a.rows, DIM_SIZES, sele, groups, fk_dist=fk_dist, seed=42)
    aggs = (olapcore.AGG_M1, olapcore.AGG_M1_TIMES_M2)
    G = s.group_nums
    for k in range(16):
        ctx.set_tuning(k, 0)
    knobs, _ = olapcore.autotune(s.probe_dims, s.probe_fks, s.factor, s.m1, s.m2, G, aggs=aggs,
                                 dimvec_lens=s.probe_lens, ctx=ctx)
    gs = torch.empty((2, G), dtype=torch.int64, device="cuda")
    tot = torch.empty((2,), dtype=torch.int64, device="cuda")

    def step():
        olapcore.starjoin_groupsum(s.probe_dims, s.probe_fks, s.factor, s.m1, s.m2, G, aggs=aggs,
                                   dimvec_lens=s.probe_lens, ctx=ctx, out=gs, totals_out=tot)
    for _ in range(3):
        step()
    torch.cuda.synchronize()
    steps = 10
    # the events go on the stream the context launches on
    ctx_stream = torch.cuda.ExternalStream(ctx.stream_handle) if ctx.stream_handle else torch.cuda.default_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(0) as clk:
        e0.record(ctx_stream)
        for _ in range(steps):
            step()
        e1.record(ctx_stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    peak, _ = measured_peak_gbs()
    gbs = a.rows * s.bytes_per_row(2) / (ms / 1e3) / 1e9
    joint = 1.0
    for x in sele:
        joint *= x
    for k in range(16):
        ctx.set_tuning(k, 0)
    return {"point": name, "fk_dist": fk_dist, "sele": list(sele), "joint_selectivity": joint,
            "group_nums": G, "ms": ms, "rows_per_s": a.rows / (ms / 1e3), "alg_GBs": gbs,
            "frac_of_peak": gbs / peak, "range_errors": ctx.take_range_errors(),
            "plan": {str(k): v for k, v in enumerate(knobs) if v}, "clocks": clk.summary()}


def cpu_leg(a, gs_h, tot_h, sum_pm):
    """The CPU baseline (the reference's own fan-outs on the same table in
    host memory, every host thread) and, as the checker, the oracle's
    per-group sums of that table against the timed query's result."""
    import numpy as np
    import oracle
    from memory_database_b200 import olapcore
    try:
        h = host_tables(a)
        cb = reference_cpu(h, 3, 1)
        o_gs, o_tot, o_err = oracle.starjoin(h.probe_dims, h.probe_fks, h.factor, h.m1, h.m2, h.group_nums,
                                             aggs=(olapcore.AGG_M1, olapcore.AGG_M1_TIMES_M2), nthreads=cb["cores"])
        parity = {"rows": h.n_rows, "oracle": "oracle_starjoin (restated OLAPcore_vwm_sv, int64)",
                  "groups_equal": bool(np.array_equal(gs_h, o_gs)), "totals_equal": bool(np.array_equal(tot_h, o_tot)),
                  "oracle_range_errors": int(o_err),
                  "sum_m1_plus_m2_equal_to_reference_mod_2^32": (sum_pm & 0xFFFFFFFF) == cb["sum_m1_plus_m2_mod_2^32"],
                  "reference_check_from": cb["best"] if cb["kind"] == "port" else "OLAPcore_vwm_sv"}
        base = {"value": cb["value"], "unit": "rows/s", "cores": cb["cores"], "kind": cb["kind"],
                "sample": cb["sample"], "variants": cb.get("variants")}
        return base, parity
    except Exception as e:  # the baseline is reported, never the target
        return {"value": None, "error": str(e)[:200]}, {"error": str(e)[:200]}


def e2e_host(a, s, ctx, aggs, world, knobs) -> dict:
    import torch
    from memory_database_b200 import _lib, olapcore
    # rows of this rank's table in pinned host memory: all of them on one GPU;
    # with several ranks a 150M-row prefix each (the host's pinned memory is
    # shared by all ranks), the rate scaled by rows
    n = a.e2e_rows or (a.rows if world == 1 else min(a.rows, 150_000_000))
    n = min(n, a.rows)
    pin = [torch.empty(n, dtype=torch.int32, pin_memory=True) for _ in range(4)]
    pm1 = torch.empty(n, dtype=torch.int32, pin_memory=True)
    pm2 = torch.empty(n, dtype=torch.int32, pin_memory=True)
    for t in range(4):
        pin[t].copy_(s.fk[t][:n])
    pm1.copy_(s.m1[:n])
    pm2.copy_(s.m2[:n])
    dims_host = [d.cpu().numpy() for d in s.dimvec]
    G = s.group_nums
    hctx = olapcore.Context(ctx.device, scratch_bytes=1 << 30)
    for k, v in enumerate(knobs):
        if v and k != _lib.TUNE_HOST_CHUNK_ROWS:
            hctx.set_tuning(k, v)
    ref = None

    def run():
        # the public call with host (pinned) buffers: olap_starjoin_groupsum_host
        return olapcore.starjoin_groupsum([dims_host[t] for t in s.orders], [pin[t] for t in s.orders],
                                          s.factor, pm1, pm2, G, aggs=aggs,
                                          dimvec_lens=[DIM_SIZES[t] for t in s.orders], ctx=hctx)

    def measure(mode):
        nonlocal ref
        hctx.set_tuning(_lib.TUNE_HOST_INPLACE, 0 if mode == "inplace" else 2)  # 0: the default call
        out = run()
        if ref is None:
            ref = out
        else:  # both host paths give the same sums
            assert all(np_equal(x, y) for x, y in zip(out, ref)), "host paths disagree"
        steps = max(1, a.e2e_steps)
        torch.cuda.synchronize()
        hctx.take_host_bytes()
        t0 = time.perf_counter()
        for _ in range(steps):
            run()
        dt = (time.perf_counter() - t0) / steps
        h2d = hctx.take_host_bytes() // steps
        if world > 1:
            import torch.distributed as dist
            t = torch.tensor([dt], dtype=torch.float64, device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            dt = t.item()
        return dt, h2d, steps

    other = "copy" if a.e2e_mode == "inplace" else "inplace"
    dt, h2d, steps = measure(a.e2e_mode)
    dt_o, h2d_o, _ = measure(other)
    hctx.close()
    chunk = 1 << 22
    launches = {"inplace": 1 + s.dimvec_nums, "copy": (n + chunk - 1) // chunk}
    paths = {"inplace": "olap_starjoin_groupsum_host, default plan for pinned columns: one kernel reads the pinned "
                        "host columns in place over PCIe, the most selective dimension's keys whole and every "
                        "later column only for rows still alive (32-byte sectors counted on the device)",
             "copy": "olap_starjoin_groupsum_host with OLAP_TUNE_HOST_INPLACE=2: pinned host columns, chunked H2D "
                     "copies overlapped with the scan"}
    return {"value": n * world / dt, "unit": "rows/s", "h2d_bytes_per_step": h2d,
            # group sums, totals, the dropped-row count (+ the dimensions' pass counts in place)
            "d2h_bytes_per_step": 8 * 2 * G + 16 + 8 + (32 if a.e2e_mode == "inplace" else 0),
            "ms_per_step": dt * 1e3, "steps": steps, "rows_per_rank": n,
            "path": paths[a.e2e_mode],
            "other_path": {"path": paths[other], "value": n * world / dt_o, "unit": "rows/s",
                           "h2d_bytes_per_step": h2d_o, "ms_per_step": dt_o * 1e3},
            "_launches": steps * launches[a.e2e_mode]}


def np_equal(x, y) -> bool:
    import numpy as np
    return (x is None and y is None) or np.array_equal(x, y)


if __name__ == "__main__":
    main()
