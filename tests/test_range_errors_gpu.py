"""GPU tests of the one dropped-row rule every star-join entry point shares.

A row with a key outside its dimension vector is never accumulated; it is
counted as a range error when none of its in-range keys meets DIM_NULL (a
row that a filter drops anyway is not an error), and a surviving row whose
group id falls outside [0, group_nums) is counted too.  The count does not
depend on the order the dimensions are probed in, so the device entry point,
the reference-layout entry point and the host entry point (in place or
through copies, pinned or pageable) drop the same rows and report the same
count as the oracle; the host entry point reports them with OLAP_ERR_RANGE
whichever path it takes."""
import ctypes as C
import re

import numpy as np
import pytest

import oracle
from memory_database_b200 import _lib, olapcore
from memory_database_b200.olapcore import AGG_M1, AGG_M1_PLUS_M2, AGG_M1_TIMES_M2

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

DIM_NULL = 127
SIZES, GROUPS, SELE = [30000, 2000, 200000, 2556], [5, 25, 4, 7], [0.5, 0.2, 0.1, 0.9]


def star(seed, n, key_lo, key_hi_extra, groups=GROUPS):
    rng = np.random.default_rng(seed)
    dv = []
    for s, p, g in zip(SIZES, SELE, groups):
        c = rng.integers(0, g, s).astype(np.int8)
        c[rng.random(s) >= p] = DIM_NULL
        dv.append(c)
    fk = [rng.integers(key_lo, s + key_hi_extra, n).astype(np.int32) for s in SIZES]
    m1 = rng.integers(-10000, 10001, n).astype(np.int32)
    m2 = rng.integers(1, 10001, n).astype(np.int32)
    return dv, fk, m1, m2


def host_call(ctx, dv, fks, factor, m1, m2, G, aggs):
    q = olapcore._build_query(dv, fks, factor, m1, m2, G, aggs, 0, len(m1), [len(d) for d in dv])
    gs = np.zeros((len(aggs), G), np.int64)
    tot = np.zeros(len(aggs), np.int64)
    st = _lib.lib.olap_starjoin_groupsum_host(ctx.handle, C.byref(q), gs.ctypes.data, tot.ctypes.data)
    dropped = 0
    if st == _lib.OLAP_ERR_RANGE:
        dropped = int(re.match(r"(\d+) rows dropped", _lib.lib.olap_ctx_last_error(ctx.handle).decode()).group(1))
    else:
        assert st == 0, _lib.lib.olap_ctx_last_error(ctx.handle).decode()
    return st, dropped, gs, tot


@pytest.mark.parametrize("groups_g", [None, 97])
@pytest.mark.parametrize("n", [1, 4099, 500_003])
def test_every_entry_point_drops_and_counts_the_same_rows(ctx, n, groups_g):
    dv, fk, m1, m2 = star(n + (groups_g or 0), n, -3, 4)
    factor = [int(np.prod(GROUPS[j + 1:])) for j in range(4)]
    G = groups_g or int(np.prod(GROUPS))
    aggs = (AGG_M1_PLUS_M2, AGG_M1_TIMES_M2)
    o_gs, o_tot, o_err = oracle.starjoin(dv, fk, factor, m1, m2, G, aggs=aggs)
    if n > 1000:
        assert o_err > 0
    want_status = _lib.OLAP_ERR_RANGE if o_err else 0
    # device pointers
    dd = [torch.from_numpy(x).cuda() for x in dv]
    df = [torch.from_numpy(x).cuda() for x in fk]
    dm1, dm2 = torch.from_numpy(m1).cuda(), torch.from_numpy(m2).cuda()
    gs, tot = olapcore.starjoin_groupsum(dd, df, factor, dm1, dm2, G, aggs=aggs, ctx=ctx)
    torch.cuda.synchronize()
    assert ctx.take_range_errors() == o_err
    assert np.array_equal(gs.cpu().numpy(), o_gs) and np.array_equal(tot.cpu().numpy(), o_tot)
    # the reference-layout entry point (tables in order 0..3, plain factors)
    dva = (C.c_void_p * 4)(*[x.data_ptr() for x in dd])
    fka = (C.c_void_p * 4)(*[x.data_ptr() for x in df])
    lens = (C.c_int64 * 4)(*SIZES)
    orders = (C.c_int * 4)(0, 1, 2, 3)
    fac = (C.c_int * 4)(*factor)
    gv = torch.zeros(G, dtype=torch.int64, device="cuda")
    cnt = C.c_int64()
    _lib.check(_lib.lib.olap_OLAPcore(ctx.handle, dva, lens, fka, orders, 4, fac, n, G, dm1.data_ptr(),
                                      dm2.data_ptr(), gv.data_ptr(), C.byref(cnt)), ctx.handle)
    assert ctx.take_range_errors() == o_err
    p_gs, p_tot, _ = oracle.starjoin(dv, fk, factor, m1, m2, G, aggs=(AGG_M1_PLUS_M2,))
    assert cnt.value == int(p_tot[0]) and np.array_equal(gv.cpu().numpy(), p_gs[0])
    # the host entry point: default, in place, copies (pinned), copies (pageable)
    pinned = [torch.from_numpy(x).pin_memory() for x in fk + [m1, m2]]
    ph = [t.numpy() for t in pinned]
    for knob, cols in ((0, ph), (3, ph), (2, ph), (0, list(fk) + [m1, m2])):
        ctx.set_tuning(_lib.TUNE_HOST_INPLACE, knob)
        try:
            st, dropped, hgs, htot = host_call(ctx, dv, cols[:4], factor, cols[4], cols[5], G, aggs)
        finally:
            ctx.set_tuning(_lib.TUNE_HOST_INPLACE, 0)
        assert (st, dropped) == (want_status, o_err), knob
        assert np.array_equal(hgs, o_gs) and np.array_equal(htot, o_tot), knob
    ctx.take_host_bytes()


def test_filtered_rows_are_not_range_errors(ctx):
    """A row with a key out of range and another key that meets DIM_NULL is
    dropped silently, in whichever order the two dimensions are met."""
    dv = [np.array([0, 1, 127, 2], np.int8), np.array([127, 3, 4], np.int8)]
    # rows: (oob, NULL), (NULL, oob), (oob, ok), (ok, oob), (oob, oob), (ok, ok), (ok, NULL)
    fk = [np.array([9, 2, -1, 1, 7, 3, 0], np.int32), np.array([0, 5, 1, -4, 8, 2, 0], np.int32)]
    m1 = np.arange(1, 8, dtype=np.int32)
    factor = [5, 1]
    _, tot, err = oracle.starjoin(dv, fk, factor, m1, m1, 15, aggs=(AGG_M1,))
    assert err == 3 and int(tot[0]) == 6
    for order in ((0, 1), (1, 0)):
        dd = [torch.from_numpy(dv[j]).cuda() for j in order]
        df = [torch.from_numpy(fk[j]).cuda() for j in order]
        f = [factor[j] for j in order]
        dm = torch.from_numpy(m1).cuda()
        _, t = olapcore.starjoin_groupsum(dd, df, f, dm, dm, 15, aggs=(AGG_M1,), ctx=ctx)
        torch.cuda.synchronize()
        assert int(t[0]) == 6 and ctx.take_range_errors() == 3
        pin = [torch.from_numpy(fk[j]).pin_memory() for j in order] + [torch.from_numpy(m1).pin_memory()]
        for knob in (3, 2):
            ctx.set_tuning(_lib.TUNE_HOST_INPLACE, knob)
            try:
                st, dropped, _, ht = host_call(ctx, [dv[j] for j in order], [p.numpy() for p in pin[:2]], f,
                                               pin[2].numpy(), pin[2].numpy(), 15, (AGG_M1,))
            finally:
                ctx.set_tuning(_lib.TUNE_HOST_INPLACE, 0)
            assert (st, dropped, int(ht[0])) == (_lib.OLAP_ERR_RANGE, 3, 6), (order, knob)
    ctx.take_host_bytes()


def test_reference_layout_without_lengths_never_reads_past_the_allocation(ctx):
    """olap_OLAPcore with dimvec_len NULL (the reference's signature has no
    lengths): keys past the device allocation that holds a vector are
    dropped and counted, never read; in-range keys give the oracle's sums."""
    n = 300_001
    dv, fk, m1, m2 = star(31, n, 0, 0)
    rng = np.random.default_rng(5)
    far = rng.random((4, n)) < 0.01
    for t in range(4):
        fk[t][far[t]] = (1 << 30) + rng.integers(0, 1 << 20, int(far[t].sum()))
    factor = [int(np.prod(GROUPS[j + 1:])) for j in range(4)]
    G = int(np.prod(GROUPS))
    lens_far = [len(d) for d in dv]
    o_gs, o_tot, o_err = oracle.starjoin(dv, fk, factor, m1, m2, G, aggs=(AGG_M1_PLUS_M2,), dim_lens=lens_far)
    assert o_err > 0
    dd = [torch.from_numpy(x).cuda() for x in dv]
    df = [torch.from_numpy(x).cuda() for x in fk]
    dm1, dm2 = torch.from_numpy(m1).cuda(), torch.from_numpy(m2).cuda()
    dva = (C.c_void_p * 4)(*[x.data_ptr() for x in dd])
    fka = (C.c_void_p * 4)(*[x.data_ptr() for x in df])
    orders = (C.c_int * 4)(0, 1, 2, 3)
    fac = (C.c_int * 4)(*factor)
    gv = torch.zeros(G, dtype=torch.int64, device="cuda")
    cnt = C.c_int64()
    _lib.check(_lib.lib.olap_OLAPcore(ctx.handle, dva, None, fka, orders, 4, fac, n, G, dm1.data_ptr(),
                                      dm2.data_ptr(), gv.data_ptr(), C.byref(cnt)), ctx.handle)
    assert ctx.take_range_errors() == o_err
    assert cnt.value == int(o_tot[0]) and np.array_equal(gv.cpu().numpy(), o_gs[0])
    # a vector that is not device memory is refused, nothing launched
    host_vec = np.zeros(16, np.int8)
    dva2 = (C.c_void_p * 4)(host_vec.ctypes.data, *[x.data_ptr() for x in dd[1:]])
    st = _lib.lib.olap_OLAPcore(ctx.handle, dva2, None, fka, orders, 4, fac, n, G, dm1.data_ptr(), dm2.data_ptr(),
                                gv.data_ptr(), C.byref(cnt))
    assert st == _lib.OLAP_ERR_INVALID
