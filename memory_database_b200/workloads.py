"""Seeded synthetic star schemas of the benchmark configurations.

The reference builds its inputs with ``gen_data`` (include/gendata_util.hpp
:449-542): per-dimension int8 vectors holding a group code with probability
``sele`` and DIM_NULL otherwise, uniform foreign keys, and measures.  The
schemas here have the same layout and distributions, generated in place in
HBM by the library's counter-based generators (value i of each column is a
pure function of (seed, stream, i), so the host can regenerate any slice).

Streams: fk of table t -> 10 + t, M1 -> 20, M2 -> 21, dimvec of table t -> 30 + t.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from .olapcore import Context, plan_olapcore

TABLES = ("customer", "supplier", "part", "date")

#: Star-join at scale: 600M fact rows, 4 int32 FKs + 2 int32 measures
#: (14.4 GB resident) over dimensions of 3,000,000 / 200,000 / 1,400,000 /
#: 2,556 rows; the headline point of the selectivity and group sweeps.
SCALE = dict(n_rows=600_000_000, dim_sizes=(3_000_000, 200_000, 1_400_000, 2_556),
             sele=(0.5, 0.2, 0.1, 1.0), groups=(8, 8, 8, 8), bitmap=(1, 1, 1, 1),
             m_range=(1, 10_000), fk_dist="uniform", zipf_s=0.8)

#: Small star-join: 6M rows, dims 30,000 / 2,000 / 200,000 / 2,556,
#: selectivity 0.2 per dimension, groups 5/25/40/7.
SMALL = dict(n_rows=6_000_000, dim_sizes=(30_000, 2_000, 200_000, 2_556),
             sele=(0.2, 0.2, 0.2, 0.2), groups=(5, 25, 40, 7), bitmap=(1, 1, 1, 1),
             m_range=(1, 10_000), fk_dist="uniform", zipf_s=0.8)


@dataclass
class StarSchema:
    n_rows: int
    dim_sizes: tuple
    sele: tuple
    groups: tuple
    bitmap: tuple
    dimvec: list = field(default_factory=list)   # per table, int8 (device tensors)
    fk: list = field(default_factory=list)       # per table, int32
    m1: object = None
    m2: object = None
    orders: list = field(default_factory=list)
    factor: list = field(default_factory=list)
    dimvec_nums: int = 0
    group_nums: int = 1

    @property
    def probe_dims(self):
        return [self.dimvec[t] for t in self.orders]

    @property
    def probe_fks(self):
        return [self.fk[t] for t in self.orders]

    @property
    def probe_lens(self):
        return [self.dim_sizes[t] for t in self.orders]

    def bytes_per_row(self, n_measures: int = 2) -> int:
        return 4 * self.dimvec_nums + 4 * n_measures


def make_star_schema(ctx: Context, n_rows: int, dim_sizes, sele, groups, bitmap=(1, 1, 1, 1),
                     m_range=(1, 10_000), fk_dist="uniform", zipf_s=0.8, seed: int = 42,
                     device: str = "cuda", fact_seed: int | None = None) -> StarSchema:
    """Generate the star schema on ``device`` (torch tensors, HBM-resident).
    ``fact_seed`` (default ``seed``) seeds the fact columns alone, so that the
    shards of several ranks share the dimension vectors."""
    import torch
    L = _lib.lib
    h = ctx.handle
    s = StarSchema(n_rows, tuple(dim_sizes), tuple(sele), tuple(groups), tuple(bitmap))
    fseed = seed if fact_seed is None else fact_seed
    for t in range(4):
        d = torch.empty(dim_sizes[t], dtype=torch.int8, device=device)
        g = max(1, int(groups[t])) if bitmap[t] else 1
        _lib.check(L.olap_gen_dimvec_dev(h, d.data_ptr(), dim_sizes[t], seed, 30 + t,
                                         float(sele[t]), g), h)
        s.dimvec.append(d)
        f = torch.empty(n_rows, dtype=torch.int32, device=device)
        if fk_dist == "zipf":
            _lib.check(L.olap_gen_zipf_i32_dev(h, f.data_ptr(), n_rows, fseed, 10 + t,
                                               dim_sizes[t], float(zipf_s)), h)
        else:
            _lib.check(L.olap_gen_uniform_i32_dev(h, f.data_ptr(), n_rows, fseed, 10 + t, 0,
                                                  dim_sizes[t] - 1), h)
        s.fk.append(f)
    s.m1 = torch.empty(n_rows, dtype=torch.int32, device=device)
    s.m2 = torch.empty(n_rows, dtype=torch.int32, device=device)
    _lib.check(L.olap_gen_uniform_i32_dev(h, s.m1.data_ptr(), n_rows, fseed, 20, m_range[0], m_range[1]), h)
    _lib.check(L.olap_gen_uniform_i32_dev(h, s.m2.data_ptr(), n_rows, fseed, 21, m_range[0], m_range[1]), h)
    ctx.synchronize()
    s.orders, s.factor, s.dimvec_nums, s.group_nums = plan_olapcore(sele, bitmap, groups)
    return s


def host_star_schema(n_rows: int, dim_sizes, sele, groups, bitmap=(1, 1, 1, 1),
                     m_range=(1, 10_000), fk_dist="uniform", zipf_s=0.8, seed: int = 42,
                     nthreads: int = 0) -> StarSchema:
    """The same schema generated in host memory (numpy), bit-identical to
    :func:`make_star_schema` for the same arguments."""
    L = _lib.lib
    s = StarSchema(n_rows, tuple(dim_sizes), tuple(sele), tuple(groups), tuple(bitmap))
    for t in range(4):
        d = np.empty(dim_sizes[t], np.int8)
        g = max(1, int(groups[t])) if bitmap[t] else 1
        _lib.check(L.olap_gen_dimvec(d.ctypes.data, dim_sizes[t], seed, 30 + t, float(sele[t]), g,
                                     nthreads))
        s.dimvec.append(d)
        f = np.empty(n_rows, np.int32)
        if fk_dist == "zipf":
            _lib.check(L.olap_gen_zipf_i32(f.ctypes.data, n_rows, seed, 10 + t, dim_sizes[t],
                                           float(zipf_s), nthreads))
        else:
            _lib.check(L.olap_gen_uniform_i32(f.ctypes.data, n_rows, seed, 10 + t, 0,
                                              dim_sizes[t] - 1, nthreads))
        s.fk.append(f)
    s.m1 = np.empty(n_rows, np.int32)
    s.m2 = np.empty(n_rows, np.int32)
    _lib.check(L.olap_gen_uniform_i32(s.m1.ctypes.data, n_rows, seed, 20, m_range[0], m_range[1], nthreads))
    _lib.check(L.olap_gen_uniform_i32(s.m2.ctypes.data, n_rows, seed, 21, m_range[0], m_range[1], nthreads))
    s.orders, s.factor, s.dimvec_nums, s.group_nums = plan_olapcore(sele, bitmap, groups)
    return s
