"""GPU parity tests of the in-place host scan (the default of
olap_starjoin_groupsum_host for pinned columns when it reads fewer bytes;
OLAP_TUNE_HOST_INPLACE = 3 forces it):
the host call reading pinned host columns where they are, the most
selective dimension first.  Sums, totals and the dropped-row count must
equal the oracle's bit for bit; pageable or differently aligned columns
must fall back to the chunked copies."""
import ctypes as C
import re

import numpy as np
import pytest

import oracle
from memory_database_b200 import _lib, olapcore
from memory_database_b200.olapcore import AGG_M1, AGG_M1_PLUS_M2, AGG_M1_TIMES_M2, AGG_M2

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

DIM_NULL = 127


def random_star(seed, n, sizes, sele, groups, key_lo=0, key_hi_extra=0):
    rng = np.random.default_rng(seed)
    dv = []
    for s, p, g in zip(sizes, sele, groups):
        c = rng.integers(0, g, s).astype(np.int8)
        c[rng.random(s) >= p] = DIM_NULL
        dv.append(c)
    fk = [rng.integers(key_lo, s + key_hi_extra, n).astype(np.int32) for s in sizes]
    m1 = rng.integers(-10000, 10001, n).astype(np.int32)
    m2 = rng.integers(1, 10001, n).astype(np.int32)
    return dv, fk, m1, m2


def pinned(a):
    t = torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    return t, t.numpy()


def run_host(ctx, dvs, fks, factors, m1, m2, G, aggs, row_range):
    """olap_starjoin_groupsum_host; returns (status, dropped, sums, totals)."""
    q = olapcore._build_query(dvs, fks, factors, m1, m2, G, aggs, row_range[0], row_range[1],
                              [len(d) for d in dvs])
    gs = np.zeros((len(aggs), G), np.int64)
    tot = np.zeros(len(aggs), np.int64)
    st = _lib.lib.olap_starjoin_groupsum_host(ctx.handle, C.byref(q), gs.ctypes.data, tot.ctypes.data)
    dropped = 0
    if st == _lib.OLAP_ERR_RANGE:
        msg = _lib.lib.olap_ctx_last_error(ctx.handle).decode()
        dropped = int(re.match(r"(\d+) rows dropped", msg).group(1))
    else:
        assert st == 0, _lib.lib.olap_ctx_last_error(ctx.handle).decode()
    return st, dropped, gs, tot


@pytest.fixture
def inplace(ctx):
    ctx.set_tuning(_lib.TUNE_HOST_INPLACE, 3)  # in place whatever the filters
    ctx.take_host_bytes()
    yield ctx
    ctx.set_tuning(_lib.TUNE_HOST_INPLACE, 0)


SIZES, GROUPS, SELE = [30000, 2000, 200000, 2556], [5, 25, 4, 7], [0.5, 0.2, 0.1, 1.0]


@pytest.mark.parametrize("n,row_range", [
    (1, None), (3, None), (4, None), (5, None), (4097, None), (1_000_003, None),
    (1_000_003, (1, 999_998)), (1_000_003, (3, 1_000_003)), (100_000, (50_000, 50_001)),
])
@pytest.mark.parametrize("aggs", [(AGG_M1_PLUS_M2,), (AGG_M1, AGG_M1_TIMES_M2), (AGG_M2,)])
def test_inplace_matches_oracle(inplace, n, row_range, aggs):
    ctx = inplace
    orders, factor, nd, G = olapcore.plan_olapcore(SELE, [1] * 4, GROUPS)
    dv, fk, m1, m2 = random_star(n + 7, n, SIZES, SELE, GROUPS)
    dvs, fks = [dv[t] for t in orders], [fk[t] for t in orders]
    hold = [pinned(f) for f in fks] + [pinned(m1), pinned(m2)]
    pf = [h[1] for h in hold[:nd]]
    pm1, pm2 = hold[nd][1], hold[nd + 1][1]
    rr = row_range or (0, n)
    st, dropped, gs, tot = run_host(ctx, dvs, pf, factor, pm1, pm2, G, aggs, rr)
    o_gs, o_tot, o_err = oracle.starjoin(dvs, fks, factor, m1, m2, G, aggs=aggs, row_range=rr)
    assert st == 0 and dropped == 0 == o_err
    assert np.array_equal(tot, o_tot)
    assert np.array_equal(gs, o_gs)
    rows = rr[1] - rr[0]
    ncol = nd + (2 if aggs != (AGG_M2,) and aggs != (AGG_M1,) else 1)
    hb = ctx.take_host_bytes() - sum(len(d) for d in dvs)
    assert hb > 0
    if rows >= 100_000:
        # the selective dimension (0.1) is read whole, the rest sparsely
        assert hb < 0.6 * rows * 4 * ncol


@pytest.mark.parametrize("nd", [0, 1, 2, 3])
def test_inplace_fewer_dimensions(inplace, nd):
    ctx = inplace
    n = 300_001
    dv, fk, m1, m2 = random_star(3, n, SIZES[:nd], SELE[:nd], GROUPS[:nd])
    factor = [int(np.prod(GROUPS[j + 1:nd])) for j in range(nd)]
    G = int(np.prod(GROUPS[:nd])) if nd else 1
    hold = [pinned(f) for f in fk] + [pinned(m1), pinned(m2)]
    st, dropped, gs, tot = run_host(ctx, dv, [h[1] for h in hold[:nd]], factor, hold[nd][1],
                                    hold[nd + 1][1], G, (AGG_M1, AGG_M1_TIMES_M2), (0, n))
    o_gs, o_tot, _ = oracle.starjoin(dv, fk, factor, m1, m2, G, aggs=(AGG_M1, AGG_M1_TIMES_M2))
    assert st == 0 and np.array_equal(gs, o_gs) and np.array_equal(tot, o_tot)


@pytest.mark.parametrize("groups_g", [None, 20])
def test_inplace_dropped_rows_equal_the_oracle(inplace, groups_g):
    """Out-of-range keys (negative and past the end) and group ids: the sums
    and the dropped-row count equal the oracle's, although the scan reads a
    later key only while its row is alive."""
    ctx = inplace
    n = 500_003
    dv, fk, m1, m2 = random_star(11, n, SIZES, SELE, GROUPS, key_lo=-3, key_hi_extra=4)
    factor = [int(np.prod(GROUPS[j + 1:])) for j in range(4)]
    G = groups_g or int(np.prod(GROUPS))
    hold = [pinned(f) for f in fk] + [pinned(m1), pinned(m2)]
    st, dropped, gs, tot = run_host(ctx, dv, [h[1] for h in hold[:4]], factor, hold[4][1], hold[5][1], G,
                                    (AGG_M1_PLUS_M2, AGG_M1_TIMES_M2), (0, n))
    o_gs, o_tot, o_err = oracle.starjoin(dv, fk, factor, m1, m2, G, aggs=(AGG_M1_PLUS_M2, AGG_M1_TIMES_M2))
    assert st == _lib.OLAP_ERR_RANGE
    assert np.array_equal(gs, o_gs) and np.array_equal(tot, o_tot)
    assert dropped == o_err > 0


def test_inplace_falls_back_to_copies(inplace):
    """Pageable columns, and pinned columns at different 16-byte phases, take
    the chunked copy path: the oracle's exact dropped-row count, and the
    copied bytes counted in full."""
    ctx = inplace
    n = 200_000
    dv, fk, m1, m2 = random_star(5, n + 1, SIZES, SELE, GROUPS, key_hi_extra=2)
    factor = [int(np.prod(GROUPS[j + 1:])) for j in range(4)]
    G = int(np.prod(GROUPS))
    aggs = (AGG_M1_PLUS_M2,)
    o_gs, o_tot, o_err = oracle.starjoin(dv, [f[1:] for f in fk], factor, m1[1:], m2[1:], G, aggs=aggs)
    # pageable
    st, dropped, gs, tot = run_host(ctx, dv, [np.ascontiguousarray(f[1:]) for f in fk], factor,
                                    np.ascontiguousarray(m1[1:]), np.ascontiguousarray(m2[1:]), G, aggs, (0, n))
    assert dropped == o_err > 0 and np.array_equal(gs, o_gs) and np.array_equal(tot, o_tot)
    assert ctx.take_host_bytes() == n * 4 * 6 + sum(len(d) for d in dv)
    # pinned, one column shifted by one row against the others
    hold = [pinned(f) for f in fk] + [pinned(m1), pinned(m2)]
    cols = [h[1][1:] for h in hold]
    cols[0] = pinned(fk[0][1:])[1]
    hold.append(cols[0])
    st, dropped, gs, tot = run_host(ctx, dv, cols[:4], factor, cols[4], cols[5], G, aggs, (0, n))
    assert dropped == o_err and np.array_equal(gs, o_gs) and np.array_equal(tot, o_tot)
    assert ctx.take_host_bytes() == n * 4 * 6 + sum(len(d) for d in dv)


def test_copies_forced_for_pinned_columns(ctx):
    """OLAP_TUNE_HOST_INPLACE = 2: pinned columns take the chunked copies,
    with the oracle's exact dropped-row count and every byte copied."""
    n = 300_001
    dv, fk, m1, m2 = random_star(17, n, SIZES, SELE, GROUPS, key_lo=-2, key_hi_extra=3)
    factor = [int(np.prod(GROUPS[j + 1:])) for j in range(4)]
    G = int(np.prod(GROUPS))
    aggs = (AGG_M1, AGG_M1_TIMES_M2)
    hold = [pinned(f) for f in fk] + [pinned(m1), pinned(m2)]
    o_gs, o_tot, o_err = oracle.starjoin(dv, fk, factor, m1, m2, G, aggs=aggs)
    ctx.set_tuning(_lib.TUNE_HOST_INPLACE, 2)
    ctx.take_host_bytes()
    try:
        st, dropped, gs, tot = run_host(ctx, dv, [h[1] for h in hold[:4]], factor, hold[4][1], hold[5][1], G,
                                        aggs, (0, n))
        moved = ctx.take_host_bytes()
    finally:
        ctx.set_tuning(_lib.TUNE_HOST_INPLACE, 0)
    assert st == _lib.OLAP_ERR_RANGE and dropped == o_err > 0
    assert np.array_equal(gs, o_gs) and np.array_equal(tot, o_tot)
    assert moved == n * 4 * 6 + sum(len(d) for d in dv)


def test_default_takes_copies_when_nothing_is_filtered(ctx):
    """The default reads in place only when the filters save bytes: with
    every dimension entry passing, the call copies the columns (every byte
    moved once), and with the headline's filters it reads a third of them."""
    n = 400_003
    sele = [1.0, 1.0, 1.0, 1.0]
    dv, fk, m1, m2 = random_star(23, n, SIZES, sele, GROUPS)
    factor = [int(np.prod(GROUPS[j + 1:])) for j in range(4)]
    G = int(np.prod(GROUPS))
    hold = [pinned(f) for f in fk] + [pinned(m1), pinned(m2)]
    cols = [h[1] for h in hold]
    o_gs, o_tot, _ = oracle.starjoin(dv, fk, factor, m1, m2, G)
    ctx.take_host_bytes()
    st, dropped, gs, tot = run_host(ctx, dv, cols[:4], factor, cols[4], cols[5], G, (AGG_M1_PLUS_M2,), (0, n))
    assert st == 0 and np.array_equal(gs, o_gs) and np.array_equal(tot, o_tot)
    assert ctx.take_host_bytes() == n * 4 * 6 + sum(len(d) for d in dv)
    dv2, _, _, _ = random_star(23, 1, SIZES, SELE, GROUPS)
    o_gs, o_tot, _ = oracle.starjoin(dv2, fk, factor, m1, m2, G)
    st, dropped, gs, tot = run_host(ctx, dv2, cols[:4], factor, cols[4], cols[5], G, (AGG_M1_PLUS_M2,), (0, n))
    assert st == 0 and np.array_equal(gs, o_gs) and np.array_equal(tot, o_tot)
    assert ctx.take_host_bytes() < 0.5 * n * 4 * 6


def test_declined_inplace_scan_gives_back_its_scratch():
    """A query whose filters keep every row makes the default call decline
    the in-place scan and copy instead.  The scratch the in-place attempt
    took must be returned first: with group sums of 40 MB (2,500,000 groups,
    two aggregates) in the default 64 MiB arena, taking them twice would
    leave no room and fail the call."""
    n = 200_003
    groups = [50, 50, 40, 25]
    dv, fk, m1, m2 = random_star(29, n, SIZES, [1.0] * 4, groups)
    factor = [int(np.prod(groups[j + 1:])) for j in range(4)]
    G = int(np.prod(groups))
    aggs = (AGG_M1, AGG_M1_TIMES_M2)
    hold = [pinned(f) for f in fk] + [pinned(m1), pinned(m2)]
    cols = [h[1] for h in hold]
    o_gs, o_tot, o_err = oracle.starjoin(dv, fk, factor, m1, m2, G, aggs=aggs)
    with olapcore.Context(0) as c:  # default arena
        st, dropped, gs, tot = run_host(c, dv, cols[:4], factor, cols[4], cols[5], G, aggs, (0, n))
        moved = c.take_host_bytes()
    assert st == 0 and o_err == 0
    assert np.array_equal(gs, o_gs) and np.array_equal(tot, o_tot)
    assert moved == n * 4 * 6 + sum(len(d) for d in dv)  # the copies ran
