"""Batched star-join queries over one device-resident fact table.

Dimension tables carry attributes (an int32 filter attribute and an int32
group attribute per row).  A query filters each table it uses with a range
[lo, hi) on the filter attribute, groups by the group attributes of 1-3
tables and scans a contiguous fact range.  ``BatchEngine.run`` executes up to
64 such queries in one persistent launch (optionally replayed as a CUDA
graph); ``run_plain`` executes one query the plain way — build its int8
dimension vectors with ``olap_build_dimvec``, then one
``olap_starjoin_groupsum`` launch — and gives bit-identical results.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import BatchQuery, check, lib
from .olapcore import AGG_M1_PLUS_M2, Context, _ptr, starjoin_groupsum

FILTER_DOMAIN = 1 << 20  # filter attributes are uniform in [0, 2^20)


@dataclass
class DimTables:
    """Attributes of the four dimension tables (customer, supplier, part, date)."""
    sizes: tuple
    groups: tuple                    # cardinality of each table's group attribute
    filt: list = field(default_factory=list)
    grp: list = field(default_factory=list)


def make_dim_tables(ctx: Context, sizes, groups, seed: int = 7) -> DimTables:
    import torch
    L = lib
    d = DimTables(tuple(sizes), tuple(groups))
    for t, (n, g) in enumerate(zip(sizes, groups)):
        f = torch.empty(n, dtype=torch.int32, device="cuda")
        gr = torch.empty(n, dtype=torch.int32, device="cuda")
        check(L.olap_gen_uniform_i32_dev(ctx.handle, f.data_ptr(), n, seed, 40 + t, 0, FILTER_DOMAIN - 1), ctx.handle)
        check(L.olap_gen_uniform_i32_dev(ctx.handle, gr.data_ptr(), n, seed, 50 + t, 0, g - 1), ctx.handle)
        d.filt.append(f)
        d.grp.append(gr)
    ctx.synchronize()
    return d


@dataclass
class Query:
    row_begin: int
    row_end: int
    lo: list            # per table
    hi: list
    grouped: list       # tables contributing their group attribute (in factor order)
    uses: list          # tables with a predicate
    factor: list        # per table
    group_nums: int
    selectivity: float = 0.0

    def to_c(self) -> BatchQuery:
        q = BatchQuery()
        q.row_begin, q.row_end = int(self.row_begin), int(self.row_end)
        for t in range(4):
            q.lo[t], q.hi[t], q.factor[t] = int(self.lo[t]), int(self.hi[t]), int(self.factor[t])
        q.uses = sum(1 << t for t in self.uses)
        q.grouped = sum(1 << t for t in self.grouped)
        q.group_nums = int(self.group_nums)
        return q


def random_queries(rng: np.random.Generator, n: int, n_rows: int, groups, sel_range=(1e-4, 0.3),
                   frac_range=(0.05, 1.0)) -> list[Query]:
    """Queries of the batched configuration: joint selectivity log-uniform in
    sel_range spread evenly over the four tables, 1-3 random group tables,
    a random contiguous fact range of frac_range of the rows."""
    out = []
    for _ in range(n):
        s = math.exp(rng.uniform(math.log(sel_range[0]), math.log(sel_range[1])))
        per = s ** 0.25
        width = max(1, int(round(per * FILTER_DOMAIN)))
        lo, hi = [], []
        for _t in range(4):
            a = int(rng.integers(0, FILTER_DOMAIN - width + 1))
            lo.append(a)
            hi.append(a + width)
        k = int(rng.integers(1, 4))
        grouped = sorted(rng.choice(4, size=k, replace=False).tolist())
        factor = [0, 0, 0, 0]
        mul = 1
        for t in reversed(grouped):
            factor[t] = mul
            mul *= groups[t]
        frac = rng.uniform(*frac_range)
        length = max(1, int(frac * n_rows))
        b = int(rng.integers(0, n_rows - length + 1))
        out.append(Query(b, b + length, lo, hi, grouped, [0, 1, 2, 3], factor, mul, s))
    return out


class BatchEngine:
    """``olap_batch``: packed dimension attributes + up to max_queries per launch."""

    def __init__(self, ctx: Context, dims: DimTables, max_queries: int = 64):
        self.ctx = ctx
        self.dims = dims
        self.max_queries = max_queries
        h = C.c_void_p()
        check(lib.olap_batch_create(ctx.handle, int(max_queries), C.byref(h)), ctx.handle)
        self._h = h
        for t in range(4):
            check(lib.olap_batch_set_dimension(h, t, _ptr(dims.filt[t]), _ptr(dims.grp[t]), len(dims.filt[t])),
                  ctx.handle)

    def close(self):
        if self._h is not None:
            lib.olap_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def graph_captures(self) -> int:
        n = C.c_int64()
        check(lib.olap_batch_graph_captures(self._h, C.byref(n)), self.ctx.handle)
        return n.value

    def tune(self, block: int, smem_slots: int, parallel_probe: int | None = None) -> None:
        """Launch shape of the scan (threads per block, shared accumulators,
        optionally the probe order: 1 reads every table's mask in one round
        trip)."""
        check(lib.olap_batch_tune(self._h, int(block), int(smem_slots)), self.ctx.handle)
        if parallel_probe is not None:
            check(lib.olap_batch_set_probe(self._h, int(parallel_probe)), self.ctx.handle)

    def tuning(self) -> tuple[int, int, int]:
        """(block, smem_slots, parallel_probe) in force."""
        b, s, p = C.c_int(), C.c_int(), C.c_int()
        check(lib.olap_batch_get_tuning(self._h, C.byref(b), C.byref(s), C.byref(p)), self.ctx.handle)
        return b.value, s.value, p.value

    def autotune(self, queries: list[Query], fk, m1, m2, agg: int = AGG_M1_PLUS_M2, sample_rows: int = 0):
        """Times the candidate launch shapes on a sample of the fact table with
        these queries and keeps the fastest; returns (block, smem_slots, ms)."""
        import torch
        self.ctx.follow_torch_stream()
        qs = (BatchQuery * len(queries))(*[q.to_c() for q in queries])
        slots = max(1, sum(int(q.group_nums) for q in queries))
        out = torch.empty(slots, dtype=torch.int64, device="cuda")
        tot = torch.empty(len(queries), dtype=torch.int64, device="cuda")
        fka = (C.c_void_p * 4)(*[_ptr(f) for f in fk])
        bb, bs, ms = C.c_int(), C.c_int(), C.c_double()
        check(lib.olap_batch_autotune(self._h, qs, len(queries), fka, _ptr(m1), _ptr(m2), int(fk[0].numel()),
                                      int(agg), _ptr(out), slots, _ptr(tot), int(sample_rows), C.byref(bb),
                                      C.byref(bs), C.byref(ms)), self.ctx.handle)
        return bb.value, bs.value, ms.value

    def run(self, queries: list[Query], fk, m1, m2, agg: int = AGG_M1_PLUS_M2, use_graph: bool = True,
            out=None, totals=None):
        """Returns (out int64[sum group_nums], totals int64[n], offsets list)."""
        import torch
        self.ctx.follow_torch_stream()
        qs = (BatchQuery * len(queries))(*[q.to_c() for q in queries])
        offs, o = [], 0
        for q in queries:
            offs.append(o)
            o += q.group_nums
        if out is None:
            out = torch.empty(max(o, 1), dtype=torch.int64, device="cuda")
        if totals is None:
            totals = torch.empty(len(queries), dtype=torch.int64, device="cuda")
        fka = (C.c_void_p * 4)(*[_ptr(f) for f in fk])
        check(lib.olap_batch_run(self._h, qs, len(queries), fka, _ptr(m1), _ptr(m2), int(fk[0].numel()), int(agg),
                                 _ptr(out), int(out.numel()), _ptr(totals), 1 if use_graph else 0), self.ctx.handle)
        return out, totals, offs


def build_dimvecs(ctx: Context, dims: DimTables, q: Query, out=None):
    """The query's int8 dimension vectors (olap_build_dimvec), one per used table."""
    import torch
    ctx.follow_torch_stream()
    vecs = []
    for j, t in enumerate(q.uses):
        v = out[j] if out is not None else torch.empty(dims.sizes[t], dtype=torch.int8, device="cuda")
        check(lib.olap_build_dimvec(ctx.handle, _ptr(dims.filt[t]), _ptr(dims.grp[t]), dims.sizes[t], int(q.lo[t]),
                                    int(q.hi[t]), 1 if t in q.grouped else 0, _ptr(v)), ctx.handle)
        vecs.append(v)
    return vecs


def run_plain(ctx: Context, dims: DimTables, q: Query, fk, m1, m2, agg: int = AGG_M1_PLUS_M2, vec_buffers=None,
              out=None, totals_out=None):
    """One query, one launch: dimension vectors, then the plain star-join."""
    vecs = build_dimvecs(ctx, dims, q, vec_buffers)
    return starjoin_groupsum(vecs, [fk[t] for t in q.uses], [q.factor[t] for t in q.uses], m1, m2, q.group_nums,
                             aggs=(agg,), row_range=(q.row_begin, q.row_end),
                             dimvec_lens=[dims.sizes[t] for t in q.uses], ctx=ctx, out=out, totals_out=totals_out)
