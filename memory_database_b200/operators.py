"""The reference's building-block operators on the B200, by their names.

Each function keeps the name and argument meaning of the reference function it
replaces (panjd123/memory_database, ``code/select``, ``code/project``,
``code/join``, ``code/group``, ``code/aggregation``, ``code/starjoin``) and runs
on device-resident torch CUDA tensors through ``libolapcore_b200.so``.  Sums
are exact int64 (the reference's ``int`` results equal them modulo 2^32).
Functions that return a count or a sum synchronise; the others are
asynchronous on torch's current stream.
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

from . import _lib
from ._lib import CMP_LE, CMP_LT, check, lib
from .olapcore import Context, default_context, _ptr, _nelem

__all__ = [
    "CMP_LE", "CMP_LT",
    "select_rowids", "select_bitmap", "sel_lt_T_fsel_independent_val_branching", "selalgo_rowwise",
    "proalgo_rowwise", "proalgo_rowwise_rows", "gather",
    "HashTable", "vecjoin_build", "vecjoin_probe",
    "vector_group", "hashtable_group", "group_hash",
    "aggalgo_fixed", "aggalgo_f64",
    "starjoinalgo_rowwise", "starjoinalgo_cwm_sv", "starjoinalgo_cwm_dv",
]


def _torch():
    import torch
    return torch


def _ctx(ctx: Context | None) -> Context:
    c = ctx or default_context()
    c.follow_torch_stream()
    return c


def _i64(dev):
    return _torch().zeros(1, dtype=_torch().int64, device=dev)


# ---- select ------------------------------------------------------------------

def select_rowids(col, val: int, cmp: int = CMP_LE, in_rowids=None, ctx: Context | None = None):
    """Row ids r with cmp(col[r], val), ascending (or the passing entries of the
    selection vector ``in_rowids``).  Returns an int32 CUDA tensor."""
    torch = _torch()
    c = _ctx(ctx)
    n_in = _nelem(in_rowids) if in_rowids is not None else 0
    cap = n_in if in_rowids is not None else _nelem(col)
    out = torch.empty(max(cap, 1), dtype=torch.int32, device=col.device)
    cnt = _i64(col.device)
    check(lib.olap_select_rowids(c.handle, _ptr(col), _nelem(col), int(val), int(cmp), _ptr(in_rowids),
                                 n_in, _ptr(out), _ptr(cnt)), c.handle)
    return out[: int(cnt.item())]


def select_bitmap(col, val: int, cmp: int = CMP_LE, ctx: Context | None = None):
    """Bitmap of cmp(col[r], val): int32 tensor of (n + 31) // 32 words, bit r%32 of word r//32."""
    torch = _torch()
    c = _ctx(ctx)
    n = _nelem(col)
    bits = torch.empty(max((n + 31) // 32, 1), dtype=torch.int32, device=col.device)
    check(lib.olap_select_bitmap(c.handle, _ptr(col), n, int(val), int(cmp), _ptr(bits)), c.handle)
    return bits[: (n + 31) // 32]


def sel_lt_T_fsel_independent_val_branching(n: int, res, col1, val2: int, if_sv=None,
                                            ctx: Context | None = None) -> int:
    """select/test_select_option.cpp:391-423: writes the passing row ids
    (``col1[r] <= val2``; of ``if_sv`` when given) into ``res`` and returns
    their count."""
    c = _ctx(ctx)
    cnt = _i64(col1.device)
    col_len = _nelem(col1) if if_sv is not None else int(n)
    check(lib.olap_select_rowids(c.handle, _ptr(col1), col_len, int(val2), CMP_LE, _ptr(if_sv),
                                 int(n) if if_sv is not None else 0, _ptr(res), _ptr(cnt)), c.handle)
    return int(cnt.item())


def selalgo_rowwise(condition: int, size_R: int, Ra, Rb, Rc, Rd, ctx: Context | None = None) -> int:
    """select/test_select_option.cpp:450-467: SUM(Rd) where Ra, Rb, Rc <= condition."""
    c = _ctx(ctx)
    s = _i64(Ra.device)
    check(lib.olap_selalgo(c.handle, int(condition), int(size_R), _ptr(Ra), _ptr(Rb), _ptr(Rc), _ptr(Rd),
                           _ptr(s), None), c.handle)
    return int(s.item())


# ---- project -----------------------------------------------------------------

def proalgo_rowwise(condition: int, size_R: int, Ra, Rc, ctx: Context | None = None):
    """project/test_project_option.cpp:34-49: the pairs (Ra, Rc) of the rows
    with Ra <= condition and Rc <= condition, in row order; returns
    ``(count, out_a, out_c)``."""
    torch = _torch()
    c = _ctx(ctx)
    n = int(size_R)
    oa = torch.empty(max(n, 1), dtype=torch.int32, device=Ra.device)
    oc = torch.empty(max(n, 1), dtype=torch.int32, device=Ra.device)
    cnt = _i64(Ra.device)
    check(lib.olap_project_pairs(c.handle, int(condition), n, _ptr(Ra), _ptr(Rc), _ptr(oa), _ptr(oc),
                                 _ptr(cnt)), c.handle)
    k = int(cnt.item())
    return k, oa[:k], oc[:k]


def proalgo_rowwise_rows(condition: int, size_R: int, rows, row_bytes: int, off_a: int = 0,
                         off_c: int | None = None, ctx: Context | None = None):
    """project/test_project_option.cpp:34-147 over a row store: ``rows`` is a
    CUDA tensor holding size_R rows of ``row_bytes`` bytes (the reference's
    row_store_min is 60 bytes with Ra at 0 and Rc at 56, row_store_max 72
    bytes with Rc at 68); returns ``(count, out_a, out_c)`` for the rows with
    Ra <= condition and Rc <= condition, in row order."""
    torch = _torch()
    c = _ctx(ctx)
    n = int(size_R)
    oc_off = int(row_bytes) - 4 if off_c is None else int(off_c)
    oa = torch.empty(max(n, 1), dtype=torch.int32, device=rows.device)
    oc = torch.empty(max(n, 1), dtype=torch.int32, device=rows.device)
    cnt = _i64(rows.device)
    check(lib.olap_project_pairs_rows(c.handle, int(condition), n, _ptr(rows), int(row_bytes), int(off_a), oc_off,
                                      _ptr(oa), _ptr(oc), _ptr(cnt)), c.handle)
    k = int(cnt.item())
    return k, oa[:k], oc[:k]


def gather(rowids, cols: Sequence, ctx: Context | None = None):
    """Late materialisation: ``[col[rowids] for col in cols]`` (1..8 int32 columns)."""
    torch = _torch()
    c = _ctx(ctx)
    k = _nelem(rowids)
    outs = [torch.empty(max(k, 1), dtype=torch.int32, device=rowids.device) for _ in cols]
    cp = (C.c_void_p * len(cols))(*[_ptr(x) for x in cols])
    op = (C.c_void_p * len(cols))(*[_ptr(x) for x in outs])
    check(lib.olap_gather_i32(c.handle, _ptr(rowids), k, len(cols), cp, _nelem(cols[0]), op), c.handle)
    return [o[:k] for o in outs]


# ---- join ----------------------------------------------------------------------

class HashTable:
    """Open-addressing build table of ``build(relation_t*, unordered_map&)``
    (join/test_join_option.cpp:44-50); ``probe`` mirrors ``probe`` (:90-96).
    With ``bloom`` (the default) a blocked Bloom filter of the build keys is
    kept beside the table and probes go through it (same results; probe keys
    that cannot match skip the table)."""

    def __init__(self, n_build: int, device="cuda", ctx: Context | None = None, bloom: bool = True):
        torch = _torch()
        self.capacity = int(lib.olap_hashtable_capacity(int(n_build)))
        self.table = torch.empty(self.capacity, dtype=torch.int64, device=device)
        self.words = int(lib.olap_hashjoin_filter_words(int(n_build))) if bloom else 0
        self.filter = torch.empty(self.words, dtype=torch.int64, device=device) if bloom else None
        self.ctx = ctx

    def build(self, keys, payload) -> "HashTable":
        c = _ctx(self.ctx)
        if self.filter is None:
            check(lib.olap_hashjoin_build(c.handle, _ptr(keys), _ptr(payload), _nelem(keys), _ptr(self.table),
                                          self.capacity), c.handle)
        else:  # table and filter in one call
            check(lib.olap_hashjoin_build_filtered(c.handle, _ptr(keys), _ptr(payload), _nelem(keys),
                                                   _ptr(self.table), self.capacity, _ptr(self.filter), self.words),
                  c.handle)
        return self

    def probe(self, keys) -> tuple[int, int]:
        """``(SUM of matched payloads, matches)``."""
        c = _ctx(self.ctx)
        s, m = _i64(keys.device), _i64(keys.device)
        check(lib.olap_hashjoin_probe_filtered(c.handle, _ptr(self.table), self.capacity, _ptr(self.filter),
                                               self.words, _ptr(keys), _nelem(keys), _ptr(s), _ptr(m), None, None),
              c.handle)
        return int(s.item()), int(m.item())

    def probe_pairs(self, keys):
        """Matches ``(probe row ids, payloads)`` in probe-row order."""
        torch = _torch()
        c = _ctx(self.ctx)
        n = _nelem(keys)
        rows = torch.empty(max(n, 1), dtype=torch.int32, device=keys.device)
        pay = torch.empty(max(n, 1), dtype=torch.int32, device=keys.device)
        m = _i64(keys.device)
        check(lib.olap_hashjoin_probe_filtered(c.handle, _ptr(self.table), self.capacity, _ptr(self.filter),
                                               self.words, _ptr(keys), n, None, _ptr(m), _ptr(rows), _ptr(pay)),
              c.handle)
        k = int(m.item())
        return rows[:k], pay[:k]


def vecjoin_build(keys, payload, vector, ctx: Context | None = None) -> None:
    """``build(relation_t*, int* vector)`` (join/test_join_option.cpp:30-36)."""
    c = _ctx(ctx)
    check(lib.olap_vecjoin_build(c.handle, _ptr(keys), _ptr(payload), _nelem(keys), _ptr(vector),
                                 _nelem(vector)), c.handle)


def vecjoin_probe(keys, vector, ctx: Context | None = None) -> int:
    """``probe(relation_t*, int* vector)`` (join:58-64): SUM vector[key]."""
    c = _ctx(ctx)
    s = _i64(keys.device)
    check(lib.olap_vecjoin_probe(c.handle, _ptr(keys), _nelem(keys), _ptr(vector), _nelem(vector), _ptr(s)),
          c.handle)
    return int(s.item())


# ---- group-by and aggregation --------------------------------------------------

def vector_group(size_R: int, vecInx, m1, m2, group_vector, group_num: int, counts=None,
                 ctx: Context | None = None) -> int:
    """group/test_group_option.cpp:44-60 (int64 group_vector); returns the total."""
    c = _ctx(ctx)
    t = _i64(vecInx.device)
    check(lib.olap_group_vector(c.handle, int(size_R), _ptr(vecInx), _ptr(m1), _ptr(m2), int(group_num),
                                _ptr(group_vector), _ptr(counts), _ptr(t)), c.handle)
    return int(t.item())


def group_hash(keys, vals, vals2=None, key_offset: int = 0, max_groups: int | None = None,
               ctx: Context | None = None):
    """Hash group-by: ``(keys, sums, counts)`` of the groups (unordered)."""
    torch = _torch()
    c = _ctx(ctx)
    n = _nelem(keys)
    cap = int(lib.olap_group_hash_capacity(int(max_groups if max_groups is not None else max(n, 1))))
    ok = torch.empty(cap, dtype=torch.int32, device=keys.device)
    os_ = torch.empty(cap, dtype=torch.int64, device=keys.device)
    oc = torch.empty(cap, dtype=torch.int64, device=keys.device)
    g = _i64(keys.device)
    check(lib.olap_group_hash(c.handle, n, _ptr(keys), int(key_offset), _ptr(vals), _ptr(vals2), cap, _ptr(ok),
                              _ptr(os_), _ptr(oc), _ptr(g)), c.handle)
    k = int(g.item())
    return ok[:k], os_[:k], oc[:k]


def hashtable_group(size_R: int, vecInx, m1, m2, max_groups: int | None = None,
                    ctx: Context | None = None) -> int:
    """group/test_group_option.cpp:71-88: groups of vecInx - 1 with SUM(m1 + m2);
    returns the total over the groups."""
    _, sums, _ = group_hash(vecInx[:size_R], m1, m2, key_offset=-1, max_groups=max_groups, ctx=ctx)
    return int(sums.sum().item())


def aggalgo_fixed(price, qty, tax_pct, ctx: Context | None = None) -> int:
    """aggalgo_* (aggregation/test_aggregation_option.cpp:28-107) in int64
    fixed point: SUM price*qty*(100 + tax_pct) = 100 x the decimal result."""
    c = _ctx(ctx)
    s = _i64(price.device)
    check(lib.olap_agg_fixed(c.handle, _nelem(price), _ptr(price), _ptr(qty), _ptr(tax_pct), _ptr(s)), c.handle)
    return int(s.item())


def aggalgo_f64(size_R: int, l_tax, l_quantity, l_extendedprice, ctx: Context | None = None) -> float:
    """aggalgo_rowwise (aggregation:28-37) in double, reduced in a fixed order."""
    torch = _torch()
    c = _ctx(ctx)
    s = torch.zeros(1, dtype=torch.float64, device=l_tax.device)
    check(lib.olap_agg_f64(c.handle, int(size_R), _ptr(l_tax), _ptr(l_quantity), _ptr(l_extendedprice), _ptr(s)),
          c.handle)
    return float(s.item())


# ---- star-join operator (code/starjoin) ----------------------------------------

def _four(dimvecs, fks, lens):
    dv = (C.c_void_p * 4)(*[_ptr(x) for x in dimvecs])
    fk = (C.c_void_p * 4)(*[_ptr(x) for x in fks])
    ln = (C.c_int64 * 4)(*[(_nelem(d) if lens is None else int(lens[j])) for j, d in enumerate(dimvecs)])
    return dv, fk, ln


def starjoinalgo_rowwise(size_lineorder: int, dimvec_c, dimvec_s, dimvec_p, dimvec_d, fk_c, fk_s, fk_p, fk_d,
                         dimvec_len=None, ctx: Context | None = None) -> int:
    """starjoin/test_starjoin_option.cpp:37-50: rows surviving the four probes."""
    c = _ctx(ctx)
    dv, fk, ln = _four([dimvec_c, dimvec_s, dimvec_p, dimvec_d], [fk_c, fk_s, fk_p, fk_d], dimvec_len)
    cnt = _i64(fk_c.device)
    check(lib.olap_starjoin_count(c.handle, int(size_lineorder), dv, ln, fk, _ptr(cnt)), c.handle)
    return int(cnt.item())


def starjoinalgo_cwm_sv(size_lineorder: int, dimvec_c, dimvec_s, dimvec_p, dimvec_d, fk_c, fk_s, fk_p, fk_d,
                        result, dimvec_len=None, ctx: Context | None = None) -> int:
    """starjoin:66-121: packed 4-bit group ids into ``result``; returns the count."""
    c = _ctx(ctx)
    dv, fk, ln = _four([dimvec_c, dimvec_s, dimvec_p, dimvec_d], [fk_c, fk_s, fk_p, fk_d], dimvec_len)
    cnt = _i64(fk_c.device)
    check(lib.olap_starjoin_cwm_sv(c.handle, int(size_lineorder), dv, ln, fk, _ptr(result), _ptr(cnt)), c.handle)
    return int(cnt.item())


def starjoinalgo_cwm_dv(size_lineorder: int, dimvec_c, dimvec_s, dimvec_p, dimvec_d, fk_c, fk_s, fk_p, fk_d,
                        dimvec_len=None, ctx: Context | None = None):
    """starjoin:137-189: ``(count, positions, packed groups)`` of the survivors."""
    torch = _torch()
    c = _ctx(ctx)
    n = int(size_lineorder)
    dv, fk, ln = _four([dimvec_c, dimvec_s, dimvec_p, dimvec_d], [fk_c, fk_s, fk_p, fk_d], dimvec_len)
    pos = torch.empty(max(n, 1), dtype=torch.int32, device=fk_c.device)
    grp = torch.empty(max(n, 1), dtype=torch.int32, device=fk_c.device)
    cnt = _i64(fk_c.device)
    check(lib.olap_starjoin_cwm_dv(c.handle, n, dv, ln, fk, _ptr(pos), _ptr(grp), _ptr(cnt)), c.handle)
    k = int(cnt.item())
    return k, pos[:k], grp[:k]
