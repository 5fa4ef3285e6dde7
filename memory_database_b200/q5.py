"""TPC-H Q5-shaped join chain on the B200 (``olap_q5_chain``).

Synthetic tables with the configuration's shapes (no TPC-H data is used):
5 regions, 25 nations (5 per region), suppliers and customers with a uniform
nation, orders with a uniform customer and an order date uniform over seven
years of days (a one-year filter keeps ~1/7), and lines with a uniform order
row, a uniform supplier, a price uniform in [90000, 10500000] cents and a
discount uniform in [0, 10] percent.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

from ._lib import Q5_MAX_BATCH, Q5Query, Q5Tables, check, lib
from .olapcore import Context, _ptr

DAYS = 7 * 365


@dataclass
class Q5Data:
    cols: dict   # name -> int32 CUDA tensor

    def c_struct(self) -> Q5Tables:
        c = self.cols
        t = Q5Tables()
        t.r_regionkey, t.n_region = _ptr(c["r_regionkey"]), c["r_regionkey"].numel()
        t.n_regionkey, t.n_nation = _ptr(c["n_regionkey"]), c["n_regionkey"].numel()
        t.s_nationkey, t.n_supp = _ptr(c["s_nationkey"]), c["s_nationkey"].numel()
        t.c_nationkey, t.n_cust = _ptr(c["c_nationkey"]), c["c_nationkey"].numel()
        t.o_custkey, t.o_orderdate, t.n_orders = _ptr(c["o_custkey"]), _ptr(c["o_orderdate"]), c["o_custkey"].numel()
        t.l_orderkey, t.l_suppkey = _ptr(c["l_orderkey"]), _ptr(c["l_suppkey"])
        t.l_price, t.l_discount, t.n_lines = _ptr(c["l_price"]), _ptr(c["l_discount"]), c["l_orderkey"].numel()
        return t


def make_q5_data(ctx: Context, n_supp: int = 100_000, n_cust: int = 1_500_000, n_orders: int = 15_000_000,
                 n_lines: int = 60_000_000, seed: int = 11) -> Q5Data:
    import torch
    h = ctx.handle

    def uni(n, stream, lo, hi):
        x = torch.empty(n, dtype=torch.int32, device="cuda")
        check(lib.olap_gen_uniform_i32_dev(h, x.data_ptr(), n, seed, stream, lo, hi), h)
        return x

    cols = {
        "r_regionkey": torch.arange(5, dtype=torch.int32, device="cuda"),
        "n_regionkey": (torch.arange(25, dtype=torch.int32, device="cuda") % 5).contiguous(),
        "s_nationkey": uni(n_supp, 80, 0, 24),
        "c_nationkey": uni(n_cust, 81, 0, 24),
        "o_custkey": uni(n_orders, 82, 1, n_cust),
        "o_orderdate": uni(n_orders, 83, 0, DAYS - 1),
        "l_orderkey": uni(n_lines, 84, 0, n_orders - 1),
        "l_suppkey": uni(n_lines, 85, 1, n_supp),
        "l_price": uni(n_lines, 86, 90_000, 10_500_000),
        "l_discount": uni(n_lines, 87, 0, 10),
    }
    ctx.synchronize()
    return Q5Data(cols)


def q5(ctx: Context, data: Q5Data, region: int, date1: int, date2: int, out=None):
    """Per-nation int64 revenue (cents x percent) of the Q5 chain; asynchronous."""
    import torch
    ctx.follow_torch_stream()
    sums = out if out is not None else torch.empty(data.cols["n_regionkey"].numel(), dtype=torch.int64,
                                                   device="cuda")
    t = data.c_struct()
    check(lib.olap_q5_chain(ctx.handle, C.byref(t), int(region), int(date1), int(date2), _ptr(sums)), ctx.handle)
    return sums


def q5_batch(ctx: Context, data: Q5Data, queries, out=None):
    """Up to 64 (region, date1, date2) queries in one pass; int64 [n, n_nation]."""
    import torch
    if not 1 <= len(queries) <= Q5_MAX_BATCH:
        raise ValueError("1..64 queries per Q5 batch")
    ctx.follow_torch_stream()
    n_nation = data.cols["n_regionkey"].numel()
    sums = out if out is not None else torch.empty((len(queries), n_nation), dtype=torch.int64, device="cuda")
    qs = (Q5Query * len(queries))(*[Q5Query(int(r), int(a), int(b)) for r, a, b in queries])
    t = data.c_struct()
    check(lib.olap_q5_batch(ctx.handle, C.byref(t), qs, len(queries), _ptr(sums)), ctx.handle)
    return sums


def random_q5_queries(rng, n: int):
    """(region, date1, date2): a uniform region and a one-year range starting
    on a uniform day of the first six years (~1/7 of the orders)."""
    out = []
    for _ in range(n):
        d1 = int(rng.integers(0, DAYS - 365))
        out.append((int(rng.integers(0, 5)), d1, d1 + 365))
    return out
