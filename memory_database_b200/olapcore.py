"""Host-side mirror of the reference's OLAP-core interface over the C-ABI.

The reference (panjd123/memory_database, ``code/OLAPcore/
test_multi_compute_operator.cpp``) exposes the star-join as C++ functions

    int OLAPcore_rowwise(int8_t** dimvec_array, int32_t** fk_array, int* orders,
                         int& dimvec_nums, int* factor, int& size_lineorder,
                         int& group_nums, int32_t* M1, int32_t* M2, int nthreads)

(``:973``; ``OLAPcore_vwm_dv`` ``:1052`` and ``OLAPcore_vwm_sv`` ``:1258`` have
the same signature and result).  The functions below keep those names,
argument order and meaning, run on the B200 through ``libolapcore_b200.so``
and return the grand total as an exact int64 (the reference's ``int`` return
equals it modulo 2^32).  ``nthreads`` is accepted and ignored.

Arrays may be torch CUDA tensors (device-resident, the fast path) or numpy
arrays / host buffers (streamed through the GPU by the library).
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

import numpy as np

from . import _lib
from ._lib import (AGG_COUNT, AGG_M1, AGG_M1_PLUS_M2, AGG_M1_TIMES_M2, AGG_M2, DIM_NULL,
                   GROUP_NULL, MAX_DIMS, OlapError, StarjoinQuery, check, lib)

__all__ = [
    "Context", "default_context", "starjoin_groupsum", "autotune", "plan_olapcore",
    "OLAPcore_rowwise", "OLAPcore_vwm_dv", "OLAPcore_vwm_sv",
    "AGG_M1_PLUS_M2", "AGG_M1", "AGG_M2", "AGG_M1_TIMES_M2", "AGG_COUNT",
    "DIM_NULL", "GROUP_NULL", "OlapError",
]


def _torch():
    import torch  # plumbing only: device memory and streams
    return torch


def _is_cuda(x) -> bool:
    return hasattr(x, "is_cuda") and bool(x.is_cuda)


def _ptr(x) -> int | None:
    """Raw pointer of a torch tensor, numpy array or integer address."""
    if x is None:
        return None
    if isinstance(x, int):
        return x
    if hasattr(x, "data_ptr"):
        return int(x.data_ptr())
    if isinstance(x, np.ndarray):
        if not x.flags["C_CONTIGUOUS"]:
            raise ValueError("numpy arrays must be C-contiguous")
        return int(x.ctypes.data)
    raise TypeError(f"unsupported array type {type(x)!r}")


def _nelem(x) -> int:
    if hasattr(x, "numel"):
        return int(x.numel())
    return int(np.asarray(x).size)


class Context:
    """An ``olap_ctx``: one device, one stream, a scratch arena."""

    def __init__(self, device: int = 0, scratch_bytes: int = 0, stream=None):
        h = C.c_void_p()
        check(lib.olap_ctx_create(int(device), int(scratch_bytes), C.byref(h)))
        self._h = h
        self.device = int(device)
        self._fixed_stream = stream is not None
        self._cur_stream = None
        if stream is not None:
            self.set_stream(stream)

    @property
    def handle(self) -> C.c_void_p:
        if self._h is None:
            raise OlapError(_lib.OLAP_ERR_INVALID, "context is closed")
        return self._h

    def set_stream(self, stream) -> None:
        """Run on a CUDA stream (torch.cuda.Stream or raw handle; 0 / None is
        the legacy default stream) from now on, instead of following torch's
        current stream."""
        raw = getattr(stream, "cuda_stream", stream) or 0
        check(lib.olap_ctx_set_stream(self.handle, C.c_void_p(raw) if raw else None), self.handle)
        self._fixed_stream = True
        self._cur_stream = raw

    def follow_torch_stream(self) -> None:
        """Unless a stream was fixed, run on torch's current stream of this
        device, so that calls are ordered with the caller's torch work."""
        if self._fixed_stream:
            return
        torch = _torch()
        raw = torch.cuda.current_stream(self.device).cuda_stream
        if raw != self._cur_stream:
            check(lib.olap_ctx_set_stream(self.handle, C.c_void_p(raw) if raw else None), self.handle)
            self._cur_stream = raw

    @property
    def stream_handle(self) -> int:
        return int(lib.olap_ctx_get_stream(self.handle) or 0)

    def set_tuning(self, knob: int, value: int) -> None:
        check(lib.olap_ctx_set_tuning(self.handle, int(knob), int(value)), self.handle)

    def synchronize(self) -> None:
        check(lib.olap_ctx_synchronize(self.handle), self.handle)

    def take_range_errors(self) -> int:
        v = C.c_int64()
        check(lib.olap_ctx_take_range_errors(self.handle, C.byref(v)), self.handle)
        return int(v.value)

    def take_host_bytes(self) -> int:
        """Bytes the host-memory calls moved to the device since the last take
        (copies, plus the 32-byte sectors read in place)."""
        v = C.c_int64()
        check(lib.olap_ctx_take_host_bytes(self.handle, C.byref(v)), self.handle)
        return int(v.value)

    def close(self) -> None:
        if self._h is not None:
            lib.olap_ctx_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_DEFAULT: dict[int, Context] = {}


def default_context(device: int | None = None) -> Context:
    """Process-wide context per device (device 0, or torch's current device)."""
    if device is None:
        try:
            torch = _torch()
            device = torch.cuda.current_device() if torch.cuda.is_available() else 0
        except Exception:
            device = 0
    if device not in _DEFAULT:
        _DEFAULT[device] = Context(device)
    return _DEFAULT[device]


def _build_query(dimvecs, fks, factors, m1, m2, group_nums, aggs, row_begin, row_end,
                 dimvec_lens) -> StarjoinQuery:
    nd = len(dimvecs)
    if nd != len(fks) or nd != len(factors) or nd > MAX_DIMS:
        raise ValueError("dimvecs, fks and factors must have the same length (<= 4)")
    if not 1 <= len(aggs) <= 2:
        raise ValueError("one or two aggregates")
    q = StarjoinQuery()
    q.dimvec_nums = nd
    q.n_aggs = len(aggs)
    for a, ag in enumerate(aggs):
        q.agg[a] = int(ag)
    for j in range(nd):
        q.dimvec[j] = _ptr(dimvecs[j])
        q.fk[j] = _ptr(fks[j])
        q.factor[j] = int(factors[j])
        if dimvec_lens is not None and dimvec_lens[j] is not None:
            q.dimvec_len[j] = int(dimvec_lens[j])
        else:
            q.dimvec_len[j] = _nelem(dimvecs[j])
    q.m1 = _ptr(m1)
    q.m2 = _ptr(m2)
    q.row_begin = int(row_begin)
    q.row_end = int(row_end)
    q.group_nums = int(group_nums)
    return q


def starjoin_groupsum(dimvecs: Sequence, fks: Sequence, factors: Sequence[int], m1, m2,
                      group_nums: int, aggs: Sequence[int] = (AGG_M1_PLUS_M2,),
                      row_range: tuple[int, int] | None = None, dimvec_lens=None,
                      want_groups: bool = True, ctx: Context | None = None,
                      out=None, totals_out=None):
    """Star-join + group-by SUM over the dimensions in probe order.

    Device tensors: runs asynchronously on the context stream and returns
    ``(group_sums[n_aggs, group_nums], totals[n_aggs])`` as int64 CUDA tensors
    (``group_sums`` is None when ``want_groups`` is False).  Host arrays:
    synchronous, returns numpy arrays.
    """
    ctx = ctx or default_context()
    first = fks[0] if len(fks) else (m1 if m1 is not None else m2)
    n_rows = _nelem(first) if first is not None else 0
    rb, re = row_range if row_range is not None else (0, n_rows)
    q = _build_query(dimvecs, fks, factors, m1, m2, group_nums, aggs, rb, re, dimvec_lens)
    n_aggs = len(aggs)
    if first is not None and _is_cuda(first):
        torch = _torch()
        dev = first.device
        ctx.follow_torch_stream()
        gs = None
        if want_groups:
            gs = out if out is not None else torch.empty((n_aggs, group_nums), dtype=torch.int64, device=dev)
        tot = totals_out if totals_out is not None else torch.empty((n_aggs,), dtype=torch.int64, device=dev)
        check(lib.olap_starjoin_groupsum(ctx.handle, C.byref(q), _ptr(gs), _ptr(tot)), ctx.handle)
        return gs, tot
    gs = np.zeros((n_aggs, group_nums), dtype=np.int64) if want_groups else None
    tot = np.zeros((n_aggs,), dtype=np.int64)
    if dimvec_lens is None:
        for j in range(len(dimvecs)):
            q.dimvec_len[j] = _nelem(dimvecs[j])
    st = lib.olap_starjoin_groupsum_host(ctx.handle, C.byref(q), _ptr(gs), _ptr(tot))
    check(st, ctx.handle)
    return gs, tot


def launch_count(dimvecs: Sequence, fks: Sequence, factors: Sequence[int], m1, m2, group_nums: int,
                 aggs: Sequence[int] = (AGG_M1_PLUS_M2,), dimvec_lens=None, ctx: Context | None = None) -> int:
    """Kernels one device-side star-join call of this query launches."""
    ctx = ctx or default_context()
    first = fks[0] if len(fks) else (m1 if m1 is not None else m2)
    n_rows = _nelem(first) if first is not None else 0
    q = _build_query(dimvecs, fks, factors, m1, m2, group_nums, aggs, 0, n_rows, dimvec_lens)
    k = C.c_int()
    check(lib.olap_starjoin_launch_count(ctx.handle, C.byref(q), 1, C.byref(k)), ctx.handle)
    return k.value


def autotune(dimvecs: Sequence, fks: Sequence, factors: Sequence[int], m1, m2, group_nums: int,
             aggs: Sequence[int] = (AGG_M1_PLUS_M2,), dimvec_lens=None, sample_rows: int = 0,
             ctx: Context | None = None):
    """Pick the launch plan of this query shape on a sample of its own data.

    Leaves the chosen ``TUNE_*`` knobs set on ``ctx`` and returns
    ``(knobs[16], best_ms_per_sample)``."""
    ctx = ctx or default_context()
    first = fks[0] if len(fks) else (m1 if m1 is not None else m2)
    n_rows = _nelem(first) if first is not None else 0
    q = _build_query(dimvecs, fks, factors, m1, m2, group_nums, aggs, 0, n_rows, dimvec_lens)
    ctx.follow_torch_stream()
    knobs = (C.c_int64 * 16)()
    ms = C.c_double()
    check(lib.olap_starjoin_autotune(ctx.handle, C.byref(q), int(sample_rows), knobs, C.byref(ms)),
          ctx.handle)
    return list(knobs), ms.value


def plan_olapcore(sele: Sequence[float], bitmap: Sequence[int], groups: Sequence[int]):
    """The reference main's plan (orders, factor, dimvec_nums, group_nums)."""
    s = (C.c_double * 4)(*[float(x) for x in sele])
    b = (C.c_int * 4)(*[int(x) for x in bitmap])
    g = (C.c_int * 4)(*[int(x) for x in groups])
    orders = (C.c_int * 4)()
    factor = (C.c_int * 4)()
    nd = C.c_int()
    gn = C.c_int64()
    check(lib.olap_plan_olapcore(s, b, g, orders, factor, C.byref(nd), C.byref(gn)))
    return list(orders)[: nd.value], list(factor)[: nd.value], nd.value, gn.value


def _olapcore(dimvec_array, fk_array, orders, dimvec_nums, factor, size_lineorder, group_nums,
              M1, M2, nthreads=None, *, dimvec_len=None, ctx=None, group_vector=None) -> int:
    """Shared body of the three reference entry points (same result)."""
    del nthreads  # the GPU decides its own parallelism
    ctx = ctx or default_context()
    dimvec_nums = int(dimvec_nums)
    dims = [dimvec_array[orders[j]] for j in range(dimvec_nums)]
    fks = [fk_array[orders[j]] for j in range(dimvec_nums)]
    facs = [int(factor[j]) for j in range(dimvec_nums)]
    lens = None
    if dimvec_len is not None:
        lens = [dimvec_len[orders[j]] for j in range(dimvec_nums)]
    gs, tot = starjoin_groupsum(dims, fks, facs, M1, M2, int(group_nums),
                                aggs=(AGG_M1_PLUS_M2,), row_range=(0, int(size_lineorder)),
                                dimvec_lens=lens, want_groups=group_vector is not None, ctx=ctx,
                                out=None)
    if group_vector is not None and gs is not None:
        if _is_cuda(group_vector):
            group_vector.copy_(gs[0])
        else:
            np.copyto(group_vector, gs[0] if isinstance(gs, np.ndarray) else gs[0].cpu().numpy())
    if _is_cuda(tot):
        return int(tot[0].item())
    return int(tot[0])


def OLAPcore_rowwise(dimvec_array, fk_array, orders, dimvec_nums, factor, size_lineorder,
                     group_nums, M1, M2, nthreads=None, **kw) -> int:
    """``OLAPcore_rowwise`` (test_multi_compute_operator.cpp:973) on the B200."""
    return _olapcore(dimvec_array, fk_array, orders, dimvec_nums, factor, size_lineorder,
                     group_nums, M1, M2, nthreads, **kw)


def OLAPcore_vwm_dv(dimvec_array, fk_array, orders, dimvec_nums, factor, size_lineorder,
                    group_nums, M1, M2, nthreads=None, **kw) -> int:
    """``OLAPcore_vwm_dv`` (test_multi_compute_operator.cpp:1052) on the B200."""
    return _olapcore(dimvec_array, fk_array, orders, dimvec_nums, factor, size_lineorder,
                     group_nums, M1, M2, nthreads, **kw)


def OLAPcore_vwm_sv(dimvec_array, fk_array, orders, dimvec_nums, factor, size_lineorder,
                    group_nums, M1, M2, nthreads=None, **kw) -> int:
    """``OLAPcore_vwm_sv`` (test_multi_compute_operator.cpp:1258) on the B200."""
    return _olapcore(dimvec_array, fk_array, orders, dimvec_nums, factor, size_lineorder,
                     group_nums, M1, M2, nthreads, **kw)


# ---- column-wise model (device tensors, reference argument layout) -----------

def _tables(dimvec_array, fk_array, dimvec_len):
    dv = (C.c_void_p * 4)(*[_ptr(x) for x in list(dimvec_array) + [None] * (4 - len(dimvec_array))])
    fk = (C.c_void_p * 4)(*[_ptr(x) for x in list(fk_array) + [None] * (4 - len(fk_array))])
    lens = [(_nelem(d) if d is not None else 0) for d in dimvec_array] if dimvec_len is None else list(dimvec_len)
    ln = (C.c_int64 * 4)(*(lens + [0] * (4 - len(lens))))
    return dv, fk, ln


def join_cwm_sv(dimvec_array, fk_array, orders, dimvec_nums, groupID, factor, size_lineorder,
                nthreads=None, *, dimvec_len=None, ctx: Context | None = None) -> None:
    """``join_cwm_sv`` (test_multi_compute_operator.cpp:908): fills the int16
    static vector ``groupID`` (GROUP_NULL for dropped rows)."""
    ctx = ctx or default_context()
    ctx.follow_torch_stream()
    dv, fk, ln = _tables(dimvec_array, fk_array, dimvec_len)
    o = (C.c_int * 4)(*list(orders)[:4])
    f = (C.c_int * 4)(*list(factor)[:4])
    check(lib.olap_join_cwm_sv(ctx.handle, dv, ln, fk, o, int(dimvec_nums), _ptr(groupID), f, int(size_lineorder)),
          ctx.handle)


def agg_cwm_sv(groupID, size_lineorder, M1, M2, group_nums, nthreads=None, *, group_vector=None,
               ctx: Context | None = None) -> int:
    """``agg_cwm_sv`` (:764): SUM(M1+M2) by groupID; returns the total."""
    torch = _torch()
    ctx = ctx or default_context()
    ctx.follow_torch_stream()
    gv = group_vector if group_vector is not None else torch.empty(int(group_nums), dtype=torch.int64,
                                                                   device=groupID.device)
    cnt = torch.zeros(1, dtype=torch.int64, device=groupID.device)
    check(lib.olap_agg_cwm_sv(ctx.handle, _ptr(groupID), int(size_lineorder), _ptr(M1), _ptr(M2), int(group_nums),
                              _ptr(gv), _ptr(cnt)), ctx.handle)
    return int(cnt.item())


def join_cwm_dv(dimvec_array, fk_array, orders, dimvec_nums, OID, groupID, factor, size_lineorder,
                nthreads=None, *, dimvec_len=None, ctx: Context | None = None) -> int:
    """``join_cwm_dv`` (:840): surviving rows as (OID, groupID) in row order;
    returns their number (the reference's ``index``)."""
    torch = _torch()
    ctx = ctx or default_context()
    ctx.follow_torch_stream()
    dv, fk, ln = _tables(dimvec_array, fk_array, dimvec_len)
    o = (C.c_int * 4)(*list(orders)[:4])
    f = (C.c_int * 4)(*list(factor)[:4])
    idx = torch.zeros(1, dtype=torch.int64, device=OID.device)
    check(lib.olap_join_cwm_dv(ctx.handle, dv, ln, fk, o, int(dimvec_nums), _ptr(OID), _ptr(groupID), f, _ptr(idx),
                               int(size_lineorder)), ctx.handle)
    return int(idx.item())


def agg_cwm_dv(OID, groupID, index, M1, M2, size_lineorder, group_nums, nthreads=None, *, group_vector=None,
               ctx: Context | None = None) -> int:
    """``agg_cwm_dv`` (:685): SUM(M1[OID]+M2[OID]) by groupID; returns the total."""
    torch = _torch()
    ctx = ctx or default_context()
    ctx.follow_torch_stream()
    gv = group_vector if group_vector is not None else torch.empty(int(group_nums), dtype=torch.int64,
                                                                   device=OID.device)
    cnt = torch.zeros(1, dtype=torch.int64, device=OID.device)
    check(lib.olap_agg_cwm_dv(ctx.handle, _ptr(OID), _ptr(groupID), int(index), _ptr(M1), _ptr(M2),
                              int(size_lineorder), int(group_nums), _ptr(gv), _ptr(cnt)), ctx.handle)
    return int(cnt.item())
