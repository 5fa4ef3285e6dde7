"""CPU tests of the serving loop's host logic: Poisson arrivals, the result
pool allocator, footprint admission, continuous batching, deadlines and
injected allocation failures, run against fake lanes on a simulated clock
(no GPU; failures are made on the host)."""
import math

import numpy as np
import pytest

from memory_database_b200 import serving as S


class SimClock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        return self.t

    def sleep(self, s):
        self.t += max(s, 1e-6)


class FakeLane:
    """Runs batches one after another (like one stream) with a cost of
    fixed + per_query * n seconds; the result of a query is a pure function
    of it.  Checks that in-flight batches never share pool bytes."""

    def __init__(self, clock, pool, max_batch, depth, fixed=2e-3, per_query=1e-4):
        self.clock, self.pool = clock, pool
        self.max_batch, self.depth = max_batch, depth
        self.fixed, self.per_query = fixed, per_query
        self.busy_until = 0.0
        self.live = {}
        self.peak_bytes = 0
        self.launch_order = []

    def launch(self, reqs, off):
        nbytes = sum(r.footprint for r in reqs)
        for o, n in self.live.items():
            assert off + nbytes <= o or o + n <= off, "in-flight batches overlap in the pool"
        assert off + nbytes <= self.pool.capacity
        self.live[off] = nbytes
        self.peak_bytes = max(self.peak_bytes, sum(self.live.values()))
        self.launch_order += [r.rid for r in reqs]
        start = max(self.clock(), self.busy_until)
        self.busy_until = start + self.fixed + self.per_query * len(reqs)
        return (self.busy_until, reqs, off)

    def poll(self, h):
        return self.clock() >= h[0]

    def finish(self, h):
        del self.live[h[2]]
        return [compute(r.query) for r in h[1]]


def compute(q):
    return np.array([hash(q) % 1000003, len(str(q))], np.int64)


def _requests(n, rate, seed=0, deadline=None):
    rng = np.random.default_rng(seed)
    star = [("star", i) for i in range(50)]
    q5 = [("q5", i) for i in range(20)]
    # footprints of up to a few KB, like small group vectors
    return S.poisson_requests(rng, rate, n, star, q5, deadline_s=deadline,
                              footprint=lambda k, q: 8 * (1 + (hash(q) % 500)))


def _server(pool, clock, max_batch=64, depth=2, **kw):
    lanes = {"star": FakeLane(clock, pool, max_batch, depth, **kw),
             "q5": FakeLane(clock, pool, max_batch, depth, **kw)}
    return S.Server(lanes, pool, clock=clock, sleep=clock.sleep), lanes


def test_poisson_arrivals_rate_and_mix():
    rng = np.random.default_rng(1)
    reqs = S.poisson_requests(rng, 500.0, 20_000, [1], [2], footprint=lambda k, q: 8)
    t = np.array([r.arrival for r in reqs])
    assert t[0] == 0 and np.all(np.diff(t) >= 0)
    assert abs(len(t) / t[-1] - 500) < 25
    share = np.mean([r.kind == "star" for r in reqs])
    assert abs(share - 0.7) < 0.02
    gaps = np.diff(t)
    assert abs(gaps.std() / gaps.mean() - 1.0) < 0.05  # exponential: cv = 1


def test_pool_allocator_against_a_byte_model():
    rng = np.random.default_rng(2)
    pool = S.PoolAllocator(1 << 16, align=256)
    owner = np.zeros(pool.capacity, bool)
    live = {}
    for _ in range(3000):
        if live and rng.random() < 0.45:
            off = list(live)[rng.integers(len(live))]
            n = live.pop(off)
            assert owner[off: off + n].all()
            owner[off: off + n] = False
            pool.free(off)
        else:
            want = int(rng.integers(1, 5000))
            off = pool.alloc(want)
            n = pool._round(want)
            if off is None:
                # no free run of n aligned bytes exists
                free = ~owner.reshape(-1, 256).any(axis=1)
                runs = np.diff(np.flatnonzero(np.diff(np.concatenate([[0], free.astype(int), [0]]))))[::2]
                assert runs.max(initial=0) * 256 < n
                continue
            assert off % 256 == 0 and not owner[off: off + n].any()
            owner[off: off + n] = True
            live[off] = n
        assert pool.in_use() == owner.sum()
    for off in list(live):
        pool.free(off)
    assert pool.free_list == [(0, pool.capacity)]


def test_every_request_gets_its_own_result_and_batches_form_under_load():
    clock = SimClock()
    pool = S.PoolAllocator(1 << 20)
    srv, lanes = _server(pool, clock)
    reqs = srv.serve(_requests(3000, 2000.0))
    assert all(r.status == "ok" for r in reqs)
    for r in reqs:
        assert np.array_equal(r.result, compute(r.query))
        assert r.arrival <= r.launched <= r.done
    st = S.summarize(reqs, srv.batches)
    assert st.mean_batch > 1.5 and st.ok == 3000 and st.p99_ms >= st.p50_ms > 0
    # FIFO within each lane
    for k, lane in lanes.items():
        ids = [r.rid for r in reqs if r.kind == k]
        assert lane.launch_order == ids
    assert pool.in_use() == 0


def test_light_load_runs_requests_alone_with_low_latency():
    clock = SimClock()
    srv, _ = _server(S.PoolAllocator(1 << 20), clock)
    reqs = srv.serve(_requests(200, 20.0, seed=3))
    st = S.summarize(reqs)
    assert st.mean_batch < 1.2 and st.p99_ms < 5.0


def test_admission_by_footprint_bounds_device_bytes():
    clock = SimClock()
    pool = S.PoolAllocator(16 * 1024)
    srv, lanes = _server(pool, clock)
    reqs = _requests(800, 3000.0, seed=4)
    reqs[10].footprint = 1 << 20       # can never fit: rejected, the rest still served
    reqs = srv.serve(reqs)
    assert reqs[10].status == "rejected"
    assert all(r.status == "ok" for r in reqs if r.rid != 10)
    assert max(l.peak_bytes for l in lanes.values()) <= pool.capacity
    for r in reqs:
        if r.status == "ok":
            assert np.array_equal(r.result, compute(r.query))


def test_injected_allocation_failures_are_retried():
    clock = SimClock()
    calls = {"n": 0}

    def fail(_n):
        calls["n"] += 1
        return calls["n"] % 3 == 0

    pool = S.PoolAllocator(1 << 20, fail=fail)
    srv, _ = _server(pool, clock)
    reqs = srv.serve(_requests(500, 1000.0, seed=5))
    assert calls["n"] > 10 and all(r.status == "ok" for r in reqs)
    assert all(np.array_equal(r.result, compute(r.query)) for r in reqs)


def test_late_requests_are_dropped_before_launch():
    clock = SimClock()
    srv, _ = _server(S.PoolAllocator(1 << 20), clock, max_batch=1, depth=1, fixed=5e-3)
    reqs = srv.serve(_requests(400, 1000.0, seed=6, deadline=0.02))
    late = [r for r in reqs if r.status == "late"]
    ok = [r for r in reqs if r.status == "ok"]
    assert late and ok
    assert all(r.launched <= r.deadline for r in ok)
    assert all(math.isnan(r.launched) for r in late)


def test_batching_beats_one_request_per_launch_under_load():
    reqs_a, reqs_b = _requests(2000, 1500.0, seed=7), _requests(2000, 1500.0, seed=7)
    ca, cb = SimClock(), SimClock()
    batched, _ = _server(S.PoolAllocator(1 << 20), ca)
    plain, _ = _server(S.PoolAllocator(1 << 20), cb, max_batch=1, depth=4)
    sa = S.summarize(batched.serve(reqs_a))
    sb = S.summarize(plain.serve(reqs_b))
    assert sa.p99_ms < sb.p99_ms and sa.qps > sb.qps
    for a, b in zip(reqs_a, reqs_b):
        assert np.array_equal(a.result, b.result)


@pytest.mark.parametrize("cap", [0, 100])
def test_tiny_pool_rejects_everything(cap):
    clock = SimClock()
    srv, _ = _server(S.PoolAllocator(cap), clock)
    reqs = srv.serve(_requests(50, 100.0))
    assert all(r.status == "rejected" for r in reqs)
