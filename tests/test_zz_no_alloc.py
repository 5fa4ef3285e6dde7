"""GPU test of olap_starjoin_groupsum_noalloc, the star-join entry point for
callers that may not allocate device memory (a fixed device-memory budget
owned by someone else, a framework whose allocator must see every byte, a
request path where an allocation may not block or fail late).  It is called
through the C-ABI with plain device pointers and no context, twice in a row
(its static scratch keeps the previous call's contents), and must give the
same results, bit for bit, as the context-based olap_starjoin_groupsum; a
query too large for its fixed scratch must be refused.  This file is
collected last so that a run stopping at its first failure has already run
every other test; it also passes on its own in a fresh process."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from memory_database_b200 import _lib, olapcore

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

# the limit as the C header states it, so that the boundary cases below
# follow the header if it changes
_HEADER = (Path(__file__).resolve().parents[1] / "include" / "olap_capi.h").read_text()
OLAP_NOALLOC_MAX_DIM_ENTRIES = int(re.search(r"#define OLAP_NOALLOC_MAX_DIM_ENTRIES (\d+)", _HEADER).group(1))


def _fn():
    fn = _lib.lib.olap_starjoin_groupsum_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.POINTER(_lib.StarjoinQuery), C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    return fn


def _star(seed, n, sizes, sele, groups):
    rng = np.random.default_rng(seed)
    dv = []
    for s, p, g in zip(sizes, sele, groups):
        c = rng.integers(0, g, s).astype(np.int8)
        c[rng.random(s) >= p] = 127
        dv.append(torch.from_numpy(c).cuda())
    # a few keys out of range, so the dropped-row count is not trivially 0
    fk = [torch.from_numpy(rng.integers(0, s + 2, n).astype(np.int32)).cuda() for s in sizes]
    m1 = torch.from_numpy(rng.integers(1, 10001, n).astype(np.int32)).cuda()
    m2 = torch.from_numpy(rng.integers(1, 10001, n).astype(np.int32)).cuda()
    return dv, fk, m1, m2


def test_noalloc_matches_context_entry_point_twice_in_a_row():
    sizes, groups, sele = [300_000, 20_000, 140_000, 2_556], [8, 8, 8, 8], [0.5, 0.2, 0.1, 1.0]
    orders, factor, nd, G = olapcore.plan_olapcore(sele, [1] * 4, groups)
    dv, fk, m1, m2 = _star(5, 3_000_001, sizes, sele, groups)
    dims, fks = [dv[t] for t in orders], [fk[t] for t in orders]
    aggs = (olapcore.AGG_M1, olapcore.AGG_M1_TIMES_M2)
    with olapcore.Context(0) as ctx:
        ref_gs, ref_tot = olapcore.starjoin_groupsum(dims, fks, factor, m1, m2, G, aggs=aggs, ctx=ctx)
        torch.cuda.synchronize()
        ref_err = ctx.take_range_errors()
    assert ref_err > 0
    q = olapcore._build_query(dims, fks, factor, m1, m2, G, aggs, 0, m1.numel(), None)
    fn = _fn()
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):
        gs = torch.full((2, G), -1, dtype=torch.int64, device="cuda")
        tot = torch.full((2,), -1, dtype=torch.int64, device="cuda")
        err = torch.full((1,), -1, dtype=torch.int64, device="cuda")
        st = fn(C.byref(q), gs.data_ptr(), tot.data_ptr(), err.data_ptr(),
                C.c_void_p(stream) if stream else None)
        assert st == _lib.OLAP_OK
        torch.cuda.synchronize()
        assert torch.equal(gs, ref_gs) and torch.equal(tot, ref_tot)
        assert int(err.item()) == ref_err


def test_noalloc_accepts_exactly_its_maximum():
    """Dimension vectors of exactly OLAP_NOALLOC_MAX_DIM_ENTRIES entries in
    total: their pass bitmaps, alignment padding and counters must fit the
    static scratch, and the sums equal the context entry point's."""
    per = OLAP_NOALLOC_MAX_DIM_ENTRIES // 4
    sizes = [per, per, per, OLAP_NOALLOC_MAX_DIM_ENTRIES - 3 * per]
    groups, sele = [8, 8, 8, 8], [0.5, 0.3, 0.2, 0.9]
    orders, factor, nd, G = olapcore.plan_olapcore(sele, [1] * 4, groups)
    dv, fk, m1, m2 = _star(9, 1_000_003, sizes, sele, groups)
    dims, fks = [dv[t] for t in orders], [fk[t] for t in orders]
    aggs = (olapcore.AGG_M1_PLUS_M2,)
    with olapcore.Context(0) as ctx:
        ref_gs, ref_tot = olapcore.starjoin_groupsum(dims, fks, factor, m1, m2, G, aggs=aggs, ctx=ctx)
        torch.cuda.synchronize()
        ref_err = ctx.take_range_errors()
    q = olapcore._build_query(dims, fks, factor, m1, m2, G, aggs, 0, m1.numel(), None)
    assert sum(q.dimvec_len[j] for j in range(4)) == OLAP_NOALLOC_MAX_DIM_ENTRIES
    gs = torch.full((1, G), -1, dtype=torch.int64, device="cuda")
    tot = torch.full((1,), -1, dtype=torch.int64, device="cuda")
    err = torch.full((1,), -1, dtype=torch.int64, device="cuda")
    assert _fn()(C.byref(q), gs.data_ptr(), tot.data_ptr(), err.data_ptr(), None) == _lib.OLAP_OK
    torch.cuda.synchronize()
    assert torch.equal(gs, ref_gs) and torch.equal(tot, ref_tot) and int(err.item()) == ref_err


def test_noalloc_rejects_queries_beyond_its_scratch():
    big = torch.zeros(OLAP_NOALLOC_MAX_DIM_ENTRIES + 1, dtype=torch.int8, device="cuda")
    fk = torch.zeros(16, dtype=torch.int32, device="cuda")
    q = olapcore._build_query([big], [fk], [1], fk, fk, 1, (olapcore.AGG_M1_PLUS_M2,), 0, 16, None)
    out = torch.zeros(2, dtype=torch.int64, device="cuda")
    assert _fn()(C.byref(q), out.data_ptr(), out.data_ptr(), None, None) == _lib.OLAP_ERR_CAPACITY
