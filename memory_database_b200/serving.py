"""Serving loop: mixed star-join and Q5 requests over device-resident tables.

Requests arrive as a Poisson process.  Each has a device-memory footprint
(the bytes of its result); a request is admitted to a batch only when its
footprint fits in the result pool, so the server never allocates on the
device while it runs.  Admitted requests are batched continuously: a lane
launches the next batch of waiting requests as soon as it has a free slot
(two batches in flight per lane by default), so a batch holds whatever
arrived while the previous ones ran.  Star-joins go to the batched
persistent star-join engine (one launch per batch, replayed as a CUDA
graph), Q5 chains to the batched Q5 kernels; each lane has its own context
and stream.  The same loop with one request per launch (the plain lanes)
is the one-launch-per-query baseline.

Every piece that decides anything (arrivals, the pool allocator, admission,
batching, completion bookkeeping, latency statistics) is host logic that
runs unchanged against fake lanes and a simulated clock, so it is tested on
the CPU; the GPU lanes only enqueue work and copy results back.
"""
from __future__ import annotations

import math
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

# ---------------------------------------------------------------------------
# requests


@dataclass
class Request:
    rid: int
    kind: str                  # "star" or "q5"
    arrival: float             # seconds after the start of the schedule
    query: object              # batch.Query, or (region, date1, date2)
    footprint: int             # device bytes of the result
    deadline: float | None = None   # give up if not launched by then (seconds)
    status: str = "pending"    # ok | rejected | late
    launched: float = math.nan
    done: float = math.nan
    batch_size: int = 0
    result: np.ndarray | None = None

    @property
    def latency(self) -> float:
        return self.done - self.arrival


def star_footprint(q) -> int:
    """Groups plus the total, int64 each."""
    return 8 * (int(q.group_nums) + 1)


def q5_footprint(n_nation: int = 25) -> int:
    return 8 * n_nation


def poisson_requests(rng: np.random.Generator, rate_qps: float, n: int, star_queries, q5_queries,
                     star_share: float = 0.7, n_nation: int = 25, deadline_s: float | None = None,
                     footprint=None) -> list[Request]:
    """n requests with exponential inter-arrival times of mean 1/rate; each is a
    star-join with probability star_share (drawn in order from star_queries,
    cycling), else a Q5 chain (from q5_queries).  footprint(kind, query)
    overrides the result sizes."""
    gaps = rng.exponential(1.0 / rate_qps, n)
    t = np.cumsum(gaps) - gaps[0]
    kinds = rng.random(n) < star_share
    out, si, qi = [], 0, 0
    for i in range(n):
        if kinds[i]:
            q = star_queries[si % len(star_queries)]
            si += 1
            out.append(Request(i, "star", float(t[i]), q, footprint("star", q) if footprint else star_footprint(q)))
        else:
            q = q5_queries[qi % len(q5_queries)]
            qi += 1
            out.append(Request(i, "q5", float(t[i]), q, footprint("q5", q) if footprint else q5_footprint(n_nation)))
        if deadline_s is not None:
            out[-1].deadline = out[-1].arrival + deadline_s
    return out


# ---------------------------------------------------------------------------
# result pool


class PoolAllocator:
    """First-fit allocator of byte ranges of one preallocated device buffer
    (host bookkeeping only).  Blocks are `align`-byte aligned; freeing
    coalesces with free neighbours.  `fail` (tests) makes an allocation fail
    on demand, as a device allocator out of memory would."""

    def __init__(self, capacity: int, align: int = 256, fail=None):
        self.capacity = capacity - capacity % align
        self.align = align
        self.free_list = [(0, self.capacity)] if self.capacity > 0 else []  # sorted (offset, size)
        self.used: dict[int, int] = {}
        self.fail = fail

    def _round(self, n: int) -> int:
        return max(self.align, -(-n // self.align) * self.align)

    def largest_free(self) -> int:
        return max((s for _, s in self.free_list), default=0)

    def in_use(self) -> int:
        return sum(self.used.values())

    def fits(self, nbytes: int) -> bool:
        return self._round(nbytes) <= self.largest_free()

    def alloc(self, nbytes: int) -> int | None:
        n = self._round(nbytes)
        if self.fail is not None and self.fail(n):
            return None
        for i, (off, size) in enumerate(self.free_list):
            if size >= n:
                if size == n:
                    self.free_list.pop(i)
                else:
                    self.free_list[i] = (off + n, size - n)
                self.used[off] = n
                return off
        return None

    def free(self, off: int) -> None:
        n = self.used.pop(off)
        fl = self.free_list
        i = 0
        while i < len(fl) and fl[i][0] < off:
            i += 1
        fl.insert(i, (off, n))
        if i + 1 < len(fl) and fl[i][0] + fl[i][1] == fl[i + 1][0]:   # merge right
            fl[i] = (fl[i][0], fl[i][1] + fl[i + 1][1])
            fl.pop(i + 1)
        if i > 0 and fl[i - 1][0] + fl[i - 1][1] == fl[i][0]:         # merge left
            fl[i - 1] = (fl[i - 1][0], fl[i - 1][1] + fl[i][1])
            fl.pop(i)


# ---------------------------------------------------------------------------
# the loop


@dataclass
class _Batch:
    reqs: list
    offset: int
    handle: object


@dataclass
class ServeStats:
    n: int
    ok: int
    rejected: int
    late: int
    batches: int
    mean_batch: float
    p50_ms: float
    p99_ms: float
    qps: float
    by_kind: dict = field(default_factory=dict)

    def as_dict(self) -> dict:
        return dict(self.__dict__)


def _pct(x, p):
    return float(np.percentile(x, p)) if len(x) else math.nan


def summarize(reqs: list[Request], batches: int = 0) -> ServeStats:
    ok = [r for r in reqs if r.status == "ok"]
    lat = np.array([r.latency for r in ok]) * 1e3
    span = (max(r.done for r in ok) - min(r.arrival for r in reqs)) if ok else math.nan
    by = {}
    for k in sorted({r.kind for r in reqs}):
        lk = np.array([r.latency for r in ok if r.kind == k]) * 1e3
        by[k] = {"n": int(len(lk)), "p50_ms": _pct(lk, 50), "p99_ms": _pct(lk, 99)}
    return ServeStats(len(reqs), len(ok), sum(r.status == "rejected" for r in reqs),
                      sum(r.status == "late" for r in reqs), batches,
                      float(np.mean([r.batch_size for r in ok])) if ok else 0.0,
                      _pct(lat, 50), _pct(lat, 99), len(ok) / span if ok and span > 0 else math.nan, by)


class Server:
    """Continuous batching over lanes that share one result pool.

    A lane has ``max_batch`` and ``depth`` (batches in flight) and three
    methods: ``launch(reqs, offset) -> handle`` enqueues the batch with its
    results at byte `offset` of the pool, ``poll(handle) -> bool`` says
    whether it finished, ``finish(handle) -> list`` returns one host result
    per request.  ``clock()`` gives seconds; ``sleep(s)`` waits."""

    def __init__(self, lanes: dict, pool: PoolAllocator, clock=time.perf_counter, sleep=None,
                 idle_wait_s: float = 50e-6):
        self.lanes = lanes
        self.pool = pool
        self.clock = clock
        self.sleep = sleep or (lambda s: time.sleep(s) if s > 0 else None)
        self.idle_wait_s = idle_wait_s
        self.batches = 0

    def serve(self, reqs: list[Request]) -> list[Request]:
        reqs = sorted(reqs, key=lambda r: r.arrival)
        waiting = {k: deque() for k in self.lanes}
        inflight = {k: deque() for k in self.lanes}
        t0 = self.clock()
        i = 0
        while i < len(reqs) or any(waiting.values()) or any(inflight.values()):
            now = self.clock() - t0
            progressed = False
            # arrivals
            while i < len(reqs) and reqs[i].arrival <= now:
                r = reqs[i]
                i += 1
                if r.kind not in self.lanes or r.footprint > self.pool.capacity:
                    r.status = "rejected"   # can never fit (or nobody serves it)
                else:
                    waiting[r.kind].append(r)
                progressed = True
            # completions, oldest first per lane (a lane's stream finishes in order)
            for k, lane in self.lanes.items():
                q = inflight[k]
                while q and lane.poll(q[0].handle):
                    b = q.popleft()
                    results = lane.finish(b.handle)
                    t = self.clock() - t0
                    for r, res in zip(b.reqs, results):
                        r.result, r.done, r.status = res, t, "ok"
                    self.pool.free(b.offset)
                    progressed = True
            # launches: FIFO per lane, as many requests as fit in one block
            for k, lane in self.lanes.items():
                w = waiting[k]
                while w and len(inflight[k]) < lane.depth:
                    batch, nbytes = [], 0
                    while w and len(batch) < lane.max_batch:
                        r = w[0]
                        if r.deadline is not None and now > r.deadline:
                            w.popleft()
                            r.status = "late"
                            progressed = True
                            continue
                        if not self.pool.fits(nbytes + r.footprint):
                            break
                        batch.append(w.popleft())
                        nbytes += r.footprint
                    if not batch:
                        break
                    off = self.pool.alloc(nbytes)
                    if off is None:             # allocation refused: retry later
                        w.extendleft(reversed(batch))
                        break
                    t = self.clock() - t0
                    for r in batch:
                        r.launched, r.batch_size = t, len(batch)
                    inflight[k].append(_Batch(batch, off, lane.launch(batch, off)))
                    self.batches += 1
                    progressed = True
            if not progressed:
                nxt = reqs[i].arrival - (self.clock() - t0) if i < len(reqs) else self.idle_wait_s
                busy = any(inflight.values())
                self.sleep(min(nxt, self.idle_wait_s) if busy else max(min(nxt, 1e-3), 0.0))
        return reqs


# ---------------------------------------------------------------------------
# GPU lanes


class _GpuLane:
    """Shared parts: a context with its own stream, views into the device
    result pool and its pinned host mirror, one event per batch."""

    def __init__(self, ctx, pool_dev, pool_host, max_batch: int, depth: int):
        import torch
        self.ctx = ctx
        self.stream = torch.cuda.Stream()
        self.pool_dev = pool_dev      # int64 CUDA tensor, capacity / 8 elements
        self.pool_host = pool_host    # pinned int64 tensor of the same size
        self.max_batch = max_batch
        self.depth = depth

    def _enqueue(self, fn, off_el: int, n_el: int):
        import torch
        with torch.cuda.stream(self.stream):
            fn()
            self.pool_host[off_el: off_el + n_el].copy_(self.pool_dev[off_el: off_el + n_el], non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(self.stream)
        return ev

    def poll(self, handle) -> bool:
        return handle[0].query()


class StarBatchLane(_GpuLane):
    """Star-joins through the batched persistent engine (graph replay).  A
    batch of at most `plain_below` requests runs the plain way instead (their
    dimension vectors, then one plain launch each): on the 600M-row table one
    to three plain launches take less time than one shared scan (measured
    1.8 / 2.9 / 3.7 ms against 4.2 / 5.4 / 4.9 ms; 8.3 against 7.1 ms at
    four).  The results are the same bit for bit."""

    def __init__(self, engine, fk, m1, m2, agg, pool_dev, pool_host, max_batch=64, depth=2, use_graph=True,
                 plain_below: int = 3):
        super().__init__(engine.ctx, pool_dev, pool_host, min(max_batch, engine.max_queries), depth)
        self.engine, self.fk, self.m1, self.m2, self.agg, self.use_graph = engine, fk, m1, m2, agg, use_graph
        self.plain_below = plain_below
        self.plain_batches = 0

    def launch(self, reqs, offset):
        from . import batch as B
        o = offset // 8
        n = len(reqs)
        gsum = sum(int(r.query.group_nums) for r in reqs)
        tot, out = self.pool_dev[o: o + n], self.pool_dev[o + n: o + n + gsum]

        def fn():
            if n <= self.plain_below:
                self.plain_batches += 1
                g = 0
                for j, r in enumerate(reqs):
                    gn = int(r.query.group_nums)
                    B.run_plain(self.ctx, self.engine.dims, r.query, self.fk, self.m1, self.m2, agg=self.agg,
                                out=out[g: g + gn].view(1, gn), totals_out=tot[j: j + 1])
                    g += gn
            else:
                self.engine.run([r.query for r in reqs], self.fk, self.m1, self.m2, agg=self.agg,
                                use_graph=self.use_graph, out=out, totals=tot)
        return (self._enqueue(fn, o, n + gsum), o, reqs)

    def finish(self, handle):
        _, o, reqs = handle
        n = len(reqs)
        host = self.pool_host.numpy()
        res, g = [], o + n
        for j, r in enumerate(reqs):
            gn = int(r.query.group_nums)
            res.append(np.concatenate([host[g: g + gn], host[o + j: o + j + 1]]))  # groups, then the total
            g += gn
        return res


class StarPlainLane(_GpuLane):
    """One star-join per launch: its dimension vectors, then the plain kernel."""

    def __init__(self, ctx, dims, fk, m1, m2, agg, pool_dev, pool_host, depth=4):
        super().__init__(ctx, pool_dev, pool_host, 1, depth)
        self.dims, self.fk, self.m1, self.m2, self.agg = dims, fk, m1, m2, agg

    def launch(self, reqs, offset):
        from . import batch as B
        (r,) = reqs
        o = offset // 8
        gn = int(r.query.group_nums)

        def fn():
            B.run_plain(self.ctx, self.dims, r.query, self.fk, self.m1, self.m2, agg=self.agg,
                        out=self.pool_dev[o: o + gn].view(1, gn), totals_out=self.pool_dev[o + gn: o + gn + 1])
        return (self._enqueue(fn, o, gn + 1), o, gn)

    def finish(self, handle):
        _, o, gn = handle
        return [self.pool_host.numpy()[o: o + gn + 1].copy()]


class Q5BatchLane(_GpuLane):
    """Q5 chains, up to 64 per pass over orders and lineitem."""

    def __init__(self, ctx, data, pool_dev, pool_host, max_batch=64, depth=2):
        super().__init__(ctx, pool_dev, pool_host, max_batch, depth)
        self.data = data
        self.n_nation = data.cols["n_regionkey"].numel()

    def launch(self, reqs, offset):
        from . import q5 as Q5
        o = offset // 8
        nn = self.n_nation * len(reqs)

        def fn():
            Q5.q5_batch(self.ctx, self.data, [r.query for r in reqs],
                        out=self.pool_dev[o: o + nn].view(len(reqs), self.n_nation))
        return (self._enqueue(fn, o, nn), o, len(reqs))

    def finish(self, handle):
        _, o, n = handle
        h = self.pool_host.numpy()
        return [h[o + j * self.n_nation: o + (j + 1) * self.n_nation].copy() for j in range(n)]


class Q5PlainLane(Q5BatchLane):
    """One Q5 chain per launch (olap_q5_chain)."""

    def __init__(self, ctx, data, pool_dev, pool_host, depth=4):
        super().__init__(ctx, data, pool_dev, pool_host, 1, depth)

    def launch(self, reqs, offset):
        from . import q5 as Q5
        (r,) = reqs
        o = offset // 8

        def fn():
            Q5.q5(self.ctx, self.data, *r.query, out=self.pool_dev[o: o + self.n_nation])
        return (self._enqueue(fn, o, self.n_nation), o, 1)


def make_pool(capacity_bytes: int):
    """Device result pool and its pinned host mirror (int64 views)."""
    import torch
    n = capacity_bytes // 8
    return (torch.zeros(n, dtype=torch.int64, device="cuda"),
            torch.zeros(n, dtype=torch.int64, pin_memory=True))


def gpu_servers(dims, fk, m1, m2, q5data, pool_bytes: int = 256 << 20, agg: int | None = None,
                max_batch: int = 64, depth: int = 2, plain_depth: int = 4, plain_below: int = 3,
                tune_queries=None):
    """(batched, plain) servers over the same tables and one result pool;
    with tune_queries, the batched engine's launch shape is autotuned first.

    Four contexts (own streams and scratch): the batched star lane, the
    batched Q5 lane, and the two plain lanes.  The two servers share the
    pool buffers, so run them one after the other."""
    from .batch import BatchEngine
    from .olapcore import AGG_M1_PLUS_M2, Context
    agg = AGG_M1_PLUS_M2 if agg is None else agg
    pool_dev, pool_host = make_pool(pool_bytes)
    ctxs = [Context() for _ in range(4)]
    eng = BatchEngine(ctxs[0], dims, max_queries=max_batch)
    if tune_queries:  # launch shape of the batched scan, timed on these queries
        eng.autotune(list(tune_queries)[:max_batch], fk, m1, m2, agg=agg)
    batched = Server({"star": StarBatchLane(eng, fk, m1, m2, agg, pool_dev, pool_host, max_batch, depth,
                                            plain_below=plain_below),
                      "q5": Q5BatchLane(ctxs[1], q5data, pool_dev, pool_host, max_batch, depth)},
                     PoolAllocator(pool_bytes))
    plain = Server({"star": StarPlainLane(ctxs[2], dims, fk, m1, m2, agg, pool_dev, pool_host, plain_depth),
                    "q5": Q5PlainLane(ctxs[3], q5data, pool_dev, pool_host, plain_depth)},
                   PoolAllocator(pool_bytes))
    batched.contexts = plain.contexts = ctxs
    batched.engine = eng
    return batched, plain


def reset(reqs: list[Request]) -> list[Request]:
    """Fresh copies of requests (same ids, arrivals, queries, footprints)."""
    return [Request(r.rid, r.kind, r.arrival, r.query, r.footprint, r.deadline) for r in reqs]
