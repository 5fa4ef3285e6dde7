"""GPU parity tests of the building-block operators (select, project, gather,
hash and vector join, group-by, aggregation, the column-wise OLAP core and
the star-join operator) against the CPU oracle: bit-exact for every integer
result, 1e-12 relative for the double aggregation."""
import numpy as np
import pytest

import oracle
from memory_database_b200 import _lib, olapcore, operators as ops

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def host(t):
    return t.cpu().numpy()


@pytest.mark.parametrize("n", [0, 1, 3, 4, 5, 4095, 4096, 4097, 1_000_003])
@pytest.mark.parametrize("cmp", [ops.CMP_LE, ops.CMP_LT])
def test_select_rowids_and_bitmap(ctx, n, cmp):
    rng = np.random.default_rng(n + cmp)
    col = rng.integers(1, 1001, max(n, 1)).astype(np.int32)[:n]
    for val in (0, 1, 10, 500, 1000):
        ids = ops.select_rowids(dev(col), val, cmp, ctx=ctx)
        exp, _ = oracle.select_rowids(col, val, cmp)
        assert np.array_equal(host(ids), exp)
        bm = ops.select_bitmap(dev(col), val, cmp, ctx=ctx)
        assert np.array_equal(host(bm).view(np.uint32), oracle.select_bitmap(col, val, cmp))


def test_select_chained_selection_vector(ctx):
    rng = np.random.default_rng(7)
    n = 777_777
    a = rng.integers(1, 1001, n).astype(np.int32)
    b = rng.integers(1, 1001, n).astype(np.int32)
    ids = ops.select_rowids(dev(a), 300, ctx=ctx)
    ids2 = ops.select_rowids(dev(b), 700, in_rowids=ids, ctx=ctx)
    e1, _ = oracle.select_rowids(a, 300)
    e2, _ = oracle.select_rowids(b, 700, in_rowids=e1)
    assert np.array_equal(host(ids2), e2)
    # the reference-named primitive with an input selection vector
    res = torch.empty(len(e1), dtype=torch.int32, device="cuda")
    k = ops.sel_lt_T_fsel_independent_val_branching(len(e1), res, dev(b), 700, if_sv=ids, ctx=ctx)
    assert k == len(e2) and np.array_equal(host(res[:k]), e2)
    # out-of-range entries of an input selection vector are dropped and counted
    bad = dev(np.array([0, 5, -1, n, n + 7, 3], np.int32))
    got = ops.select_rowids(dev(b), 1000, in_rowids=bad, ctx=ctx)
    assert host(got).tolist() == [0, 5, 3] and ctx.take_range_errors() == 3


@pytest.mark.parametrize("sel", [0.001, 0.01, 0.1, 0.5])
def test_select_config2_selectivities(ctx, sel):
    """col < t at the config's selectivities (values uniform in [0, 2^20))."""
    n = 1 << 24
    L = _lib.lib
    col = torch.empty(n, dtype=torch.int32, device="cuda")
    _lib.check(L.olap_gen_uniform_i32_dev(ctx.handle, col.data_ptr(), n, 42, 50, 0, (1 << 20) - 1), ctx.handle)
    t = int(sel * (1 << 20))
    ids = ops.select_rowids(col, t, ops.CMP_LT, ctx=ctx)
    exp, _ = oracle.select_rowids(host(col), t, ops.CMP_LT)
    assert np.array_equal(host(ids), exp)
    # project gather of 4 columns by those row ids
    cols = [torch.roll(col, k) for k in range(4)]
    outs = ops.gather(ids, cols, ctx=ctx)
    eo, _ = oracle.gather(exp, [host(c) for c in cols])
    for o, e in zip(outs, eo):
        assert np.array_equal(host(o), e)


def test_selalgo_and_project(ctx):
    rng = np.random.default_rng(8)
    n = 2_000_003
    cols = [rng.integers(1, 1001, n).astype(np.int32) for _ in range(4)]
    d = [dev(c) for c in cols]
    for cond in (1, 215, 464, 1000):
        assert ops.selalgo_rowwise(cond, n, *d, ctx=ctx) == oracle.selalgo(cond, *cols)[0]
        k, oa, oc = ops.proalgo_rowwise(cond, n, d[0], d[2], ctx=ctx)
        ea, ec = oracle.project_pairs(cond, cols[0], cols[2])
        assert k == len(ea) and np.array_equal(host(oa), ea) and np.array_equal(host(oc), ec)
    # unaligned columns take the scalar paths
    assert ops.selalgo_rowwise(500, n - 1, d[0][1:], d[1][1:], d[2][1:], d[3][1:], ctx=ctx) == \
        oracle.selalgo(500, cols[0][1:], cols[1][1:], cols[2][1:], cols[3][1:])[0]
    k, oa, oc = ops.proalgo_rowwise(500, n - 1, d[0][1:], d[2][1:], ctx=ctx)
    ea, ec = oracle.project_pairs(500, cols[0][1:], cols[2][1:])
    assert np.array_equal(host(oa), ea) and np.array_equal(host(oc), ec)


@pytest.mark.parametrize("row_bytes,rb_bytes", [(60, 52), (72, 64)])
@pytest.mark.parametrize("n", [0, 1, 5, 4097, 1_000_003])
def test_project_row_store(ctx, row_bytes, rb_bytes, n):
    """proalgo_rowwise over the reference's row stores (row_store_min: Ra,
    char Rb[52], Rc; row_store_max: Rb[64]): the pairs equal the oracle's."""
    rng = np.random.default_rng(n + row_bytes)
    dt = np.dtype([("Ra", "<i4"), ("Rb", f"V{rb_bytes}"), ("Rc", "<i4")])
    assert dt.itemsize == row_bytes
    rows = np.zeros(n, dt)
    rows["Ra"] = rng.integers(1, 1001, n)
    rows["Rc"] = rng.integers(1, 1001, n)
    rows["Rb"] = rng.integers(0, 256, (n, rb_bytes), dtype=np.uint8).view(f"V{rb_bytes}").reshape(n)
    d = torch.from_numpy(rows.view(np.uint8).reshape(-1).copy()).cuda()
    for cond in (0, 1, 300, 1000):
        k, oa, oc = ops.proalgo_rowwise_rows(cond, n, d, row_bytes, ctx=ctx)
        ea, ec = oracle.project_pairs(cond, rows["Ra"].copy(), rows["Rc"].copy())
        assert k == len(ea) and np.array_equal(host(oa), ea) and np.array_equal(host(oc), ec)


def test_gather_out_of_range(ctx):
    col = np.arange(100, dtype=np.int32) * 3
    ids = np.array([0, 99, 100, -1, 50, 7, 7], np.int32)
    out = ops.gather(dev(ids), [dev(col)], ctx=ctx)
    assert host(out[0]).tolist() == [0, 297, 0, 0, 150, 21, 21]
    assert ctx.take_range_errors() == 2


@pytest.mark.parametrize("dist", ["uniform", "zipf"])
@pytest.mark.parametrize("bloom", [True, False])
def test_hash_join_config2_shape(ctx, dist, bloom):
    """2^20-row build side of unique shuffled keys, 2^24 probe keys over the
    build keys (uniform or Zipf(1.0)), half of them made non-matching; with
    and without the Bloom filter, and on unaligned probe keys (scalar path)."""
    rng = np.random.default_rng(9)
    R, S = 1 << 20, 1 << 24
    rk = rng.permutation(np.arange(1, R + 1)).astype(np.int32)
    rp = rng.integers(-1000, 1000, R).astype(np.int32)
    L = _lib.lib
    pos = torch.empty(S, dtype=torch.int32, device="cuda")
    if dist == "zipf":
        _lib.check(L.olap_gen_zipf_i32_dev(ctx.handle, pos.data_ptr(), S, 42, 60, R, 1.0), ctx.handle)
    else:
        _lib.check(L.olap_gen_uniform_i32_dev(ctx.handle, pos.data_ptr(), S, 42, 60, 0, R - 1), ctx.handle)
    ctx.synchronize()
    sk = rk[host(pos)]
    sk = np.where(rng.random(S) < 0.5, sk, sk + 4 * R).astype(np.int32)
    ht = ops.HashTable(R, ctx=ctx, bloom=bloom).build(dev(rk), dev(rp))
    s, m = ht.probe(dev(sk))
    es, em = oracle.hashjoin(rk, rp, sk)
    assert (s, m) == (es, em)
    rows, pay = ht.probe_pairs(dev(sk[:500_000]))
    es2, em2, erows, epay = oracle.hashjoin(rk, rp, sk[:500_000], want_pairs=True)
    assert np.array_equal(host(rows), erows) and np.array_equal(host(pay), epay)
    # unaligned probe keys
    assert ht.probe(dev(sk[:1_000_001])[1:]) == oracle.hashjoin(rk, rp, sk[1:1_000_001])


@pytest.mark.parametrize("bloom", [True, False])
def test_hash_join_duplicates_and_edge_keys(ctx, bloom):
    rng = np.random.default_rng(10)
    rk = rng.integers(-5000, 5000, 100_000).astype(np.int32)  # many duplicates, negatives
    rk[:3] = [np.iinfo(np.int32).min, np.iinfo(np.int32).max, 0]
    rp = np.arange(len(rk), dtype=np.int32)  # payload = row: "last row wins" visible
    sk = rng.integers(-6000, 6000, 300_001).astype(np.int32)
    sk[:2] = [np.iinfo(np.int32).min, np.iinfo(np.int32).max]
    ht = ops.HashTable(len(rk), ctx=ctx, bloom=bloom).build(dev(rk), dev(rp))
    assert ctx.take_range_errors() == 1  # the INT32_MIN build key
    assert ht.probe(dev(sk)) == oracle.hashjoin(rk, rp, sk)
    rows, pay = ht.probe_pairs(dev(sk))
    _, _, erows, epay = oracle.hashjoin(rk, rp, sk, want_pairs=True)
    assert np.array_equal(host(rows), erows) and np.array_equal(host(pay), epay)
    empty = ops.HashTable(0, ctx=ctx, bloom=bloom).build(dev(rk[:0]), dev(rp[:0]))
    assert empty.probe(dev(sk)) == (0, 0)


def test_vector_join(ctx):
    rng = np.random.default_rng(11)
    R = 1 << 20
    rk = rng.permutation(np.arange(1, R + 1)).astype(np.int32)
    rk = np.concatenate([rk, rk[:1000], np.array([-1, R + 5], np.int32)])  # duplicates, out of range
    rp = rng.integers(-100, 100, len(rk)).astype(np.int32)
    sk = rng.integers(0, R + 3, 3_000_000).astype(np.int32)
    vec = torch.zeros(R + 1, dtype=torch.int32, device="cuda")
    ops.vecjoin_build(dev(rk), dev(rp), vec, ctx=ctx)
    s = ops.vecjoin_probe(dev(sk), vec, ctx=ctx)
    es, evec, eerr = oracle.vecjoin(rk, rp, sk, R + 1)
    assert np.array_equal(host(vec), evec) and s == es and ctx.take_range_errors() == eerr


@pytest.mark.parametrize("G", [16, 1 << 12, 1 << 20, 1 << 22])
def test_group_by_config2_cardinalities(ctx, G):
    n = 1 << 24
    L = _lib.lib
    idx = torch.empty(n, dtype=torch.int32, device="cuda")
    m1 = torch.empty(n, dtype=torch.int32, device="cuda")
    m2 = torch.empty(n, dtype=torch.int32, device="cuda")
    _lib.check(L.olap_gen_uniform_i32_dev(ctx.handle, idx.data_ptr(), n, 42, 70, 1, G), ctx.handle)
    _lib.check(L.olap_gen_uniform_i32_dev(ctx.handle, m1.data_ptr(), n, 42, 71, 1, 10000), ctx.handle)
    _lib.check(L.olap_gen_uniform_i32_dev(ctx.handle, m2.data_ptr(), n, 42, 72, -5000, 5000), ctx.handle)
    gv = torch.empty(G, dtype=torch.int64, device="cuda")
    cnt = torch.empty(G, dtype=torch.int64, device="cuda")
    tot = ops.vector_group(n, idx, m1, m2, gv, G, counts=cnt, ctx=ctx)
    etot, egv, ecnt, _ = oracle.vector_group(host(idx), host(m1), host(m2), G)
    assert tot == etot and np.array_equal(host(gv), egv) and np.array_equal(host(cnt), ecnt)
    # hash group-by on the same keys (0-based as the reference's hashtable_group)
    keys, sums, counts = ops.group_hash(idx, m1, m2, key_offset=-1, max_groups=G, ctx=ctx)
    order = np.argsort(host(keys))
    k = host(keys)[order]
    present = np.nonzero(ecnt)[0]
    assert np.array_equal(k, present.astype(np.int32))
    assert np.array_equal(host(sums)[order], egv[present]) and np.array_equal(host(counts)[order], ecnt[present])
    assert ops.hashtable_group(n, idx, m1, m2, max_groups=G, ctx=ctx) == etot


def test_group_edge_cases(ctx):
    idx = np.array([1, 2, 0, 5, 3, 2, -7], np.int32)
    m = np.array([10, 20, 30, 40, 50, 60, 70], np.int32)
    gv = torch.empty(4, dtype=torch.int64, device="cuda")
    tot = ops.vector_group(len(idx), dev(idx), dev(m), dev(m), gv, 4, ctx=ctx)
    etot, egv, _, eerr = oracle.vector_group(idx, m, m, 4)
    assert tot == etot and np.array_equal(host(gv), egv) and ctx.take_range_errors() == eerr == 3
    keys, sums, counts = ops.group_hash(dev(idx), dev(m), ctx=ctx)
    got = sorted(zip(host(keys).tolist(), host(sums).tolist(), host(counts).tolist()))
    exp = {}
    for k, v in zip(idx.tolist(), m.tolist()):
        s, c = exp.get(k, (0, 0))
        exp[k] = (s + v, c + 1)
    assert got == sorted((k, s, c) for k, (s, c) in exp.items())


def test_aggregation(ctx):
    rng = np.random.default_rng(12)
    n = (1 << 24) + 3
    tax = rng.integers(1, 21, n).astype(np.int32)
    qty = rng.integers(1, 11, n).astype(np.int32)
    price = rng.integers(5, 21, n).astype(np.int32)
    assert ops.aggalgo_fixed(dev(price), dev(qty), dev(tax), ctx=ctx) == oracle.agg_fixed(price, qty, tax)
    td, qd, pd = tax.astype(np.float64) / 100, qty.astype(np.float64), price.astype(np.float64)
    got = ops.aggalgo_f64(n, dev(td), dev(qd), dev(pd), ctx=ctx)
    exp = oracle.agg_f64(td, qd, pd)
    assert abs(got - exp) <= 1e-12 * abs(exp)
    assert got == ops.aggalgo_f64(n, dev(td), dev(qd), dev(pd), ctx=ctx)  # deterministic


def test_column_wise_olapcore(ctx, golden_queries):
    """join_cwm_sv/agg_cwm_sv and join_cwm_dv/agg_cwm_dv on the reference's
    queries whose groups fit int16: same static vector as the oracle, same
    (OID, groupID) lists as the row order of the survivors, same totals."""
    for q in golden_queries:
        if q["group_nums"] > 32766:
            continue
        dv, fk, m1, m2 = oracle.gen_olapcore_compat(1.0, q["sele"], q["bitmap"], q["groups"])
        n, G = len(m1), q["group_nums"]
        ddv, dfk = [dev(d) for d in dv], [dev(f) for f in fk]
        gid = torch.empty(n, dtype=torch.int16, device="cuda")
        olapcore.join_cwm_sv(ddv, dfk, q["orders"], q["dimvec_nums"], gid, q["factor"], n, ctx=ctx)
        egid, _ = oracle.join_cwm_sv([dv[t] for t in q["orders"]], [len(dv[t]) for t in q["orders"]],
                                     [fk[t] for t in q["orders"]], q["factor"], n)
        assert np.array_equal(host(gid), egid)
        gv = torch.empty(G, dtype=torch.int64, device="cuda")
        tot = olapcore.agg_cwm_sv(gid, n, dev(m1), dev(m2), G, group_vector=gv, ctx=ctx)
        assert tot == q["total_sf1_reference"]
        oid = torch.empty(n, dtype=torch.int64, device="cuda")
        gid2 = torch.empty(n, dtype=torch.int16, device="cuda")
        k = olapcore.join_cwm_dv(ddv, dfk, q["orders"], q["dimvec_nums"], oid, gid2, q["factor"], n, ctx=ctx)
        live = np.nonzero(egid != 32767)[0]
        assert k == len(live) and np.array_equal(host(oid[:k]), live)
        assert np.array_equal(host(gid2[:k]), egid[live])
        gv2 = torch.empty(G, dtype=torch.int64, device="cuda")
        assert olapcore.agg_cwm_dv(oid, gid2, k, dev(m1), dev(m2), n, G, group_vector=gv2, ctx=ctx) == tot
        assert torch.equal(gv, gv2)


def test_starjoin_operator(ctx):
    rng = np.random.default_rng(13)
    sizes = [30000, 2000, 200000, 2555]
    n = 3_000_001
    dv = []
    for s in sizes:
        c = rng.integers(0, 16, s + 1).astype(np.int8)
        c[rng.random(s + 1) < 0.4] = 127
        c[s] = 0
        dv.append(c)
    fk = [rng.integers(0, s + 1, n).astype(np.int32) for s in sizes]
    lens = [s + 1 for s in sizes]
    ddv, dfk = [dev(d) for d in dv], [dev(f) for f in fk]
    _, tot, _ = oracle.starjoin(dv, fk, [0, 0, 0, 0], None, None, 1, aggs=(4,))
    assert ops.starjoinalgo_rowwise(n, *ddv, *dfk, ctx=ctx) == int(tot[0])
    res = torch.empty(n, dtype=torch.int32, device="cuda")
    c = ops.starjoinalgo_cwm_sv(n, *ddv, *dfk, res, ctx=ctx)
    ec, eres = oracle.starjoin_cwm_sv(dv, lens, fk, n)
    assert c == ec and np.array_equal(host(res), eres)
    k, pos, grp = ops.starjoinalgo_cwm_dv(n, *ddv, *dfk, ctx=ctx)
    assert k == int(tot[0])
    live = np.nonzero(eres != 32767)[0]
    assert np.array_equal(np.intersect1d(host(pos), live), live)
    assert np.array_equal(host(grp)[np.isin(host(pos), live)], eres[live])


def _group_expect(keys, vals, vals2):
    return oracle.hash_group(keys, vals, vals2)


@pytest.mark.parametrize("dist,G,n,two", [
    ("zipf", 300, 2_000_001, True),        # shared-table plan, skewed
    ("uniform", 1, (1 << 24) + 5, True),   # one key: its per-block count crosses the flush threshold
    ("uniform", 3, (1 << 24) + 7, False),
    ("uniform", 5000, 1_000_003, True),    # partitioned plan, few groups per partition
    ("zipf", 1 << 16, 3_000_001, False),   # partitioned plan, skewed
    ("wide", 1 << 18, 2_000_003, True),    # partitioned plan, keys over the whole int32 range
])
def test_group_hash_plans(ctx, dist, G, n, two):
    rng = np.random.default_rng(G + n)
    if dist == "uniform":
        keys = rng.integers(0, G, n).astype(np.int32)
    elif dist == "zipf":
        keys = (rng.zipf(1.2, n) % G).astype(np.int32)
    else:
        pool = rng.integers(-2**31 + 1, 2**31, G, dtype=np.int64).astype(np.int32)
        pool[:3] = [2**31 - 1, -2**31 + 1, 0]
        keys = pool[rng.integers(0, G, n)]
    vals = rng.integers(-2**31, 2**31, n, dtype=np.int64).astype(np.int32)  # extremes of the value split
    vals2 = rng.integers(-2**31, 2**31, n, dtype=np.int64).astype(np.int32) if two else None
    ek, es, ec = _group_expect(keys, vals, vals2)
    # combining off (default) / on; forced partitioned plan; 16-byte shared tables
    for combine, plan in ((2, 0), (1, 0), (2, 2), (2, 3)):
        ctx.set_tuning(_lib.TUNE_GROUP_COMBINE, combine)
        ctx.set_tuning(_lib.TUNE_GROUP_PLAN, plan)
        k, s, c = ops.group_hash(dev(keys), dev(vals), dev(vals2) if two else None, max_groups=G, ctx=ctx)
        order = np.argsort(host(k))
        assert np.array_equal(host(k)[order], ek)
        assert np.array_equal(host(s)[order], es) and np.array_equal(host(c)[order], ec)
    ctx.set_tuning(_lib.TUNE_GROUP_COMBINE, 0)
    ctx.set_tuning(_lib.TUNE_GROUP_PLAN, 0)
    # a key equal to the empty marker after the offset is dropped and counted
    off = ((-2**31 - int(keys[0])) + 2**31) % 2**32 - 2**31  # wraps keys[0] onto INT32_MIN
    ops.group_hash(dev(keys[:1000]), dev(vals[:1000]), key_offset=off, max_groups=G, ctx=ctx)
    assert ctx.take_range_errors() == int((keys[:1000] == keys[0]).sum())


@pytest.mark.parametrize("two", [False, True])
def test_group_hash_hot_partition(ctx, two):
    """Partitioned plan with one key in 90 % of the rows: its partition is
    split over several blocks whose partial tables are merged; every group's
    sum and count equal the oracle's, with and without a second value
    column, and the combining path agrees."""
    rng = np.random.default_rng(77)
    n, G = 2_000_003, 1 << 16
    keys = rng.integers(0, G, n).astype(np.int32)
    keys[rng.random(n) < 0.9] = 7
    vals = rng.integers(-2**31, 2**31, n, dtype=np.int64).astype(np.int32)
    vals2 = rng.integers(-2**31, 2**31, n, dtype=np.int64).astype(np.int32) if two else None
    ek, es, ec = oracle.hash_group(keys, vals, vals2)
    try:
        for combine in (2, 1):
            ctx.set_tuning(_lib.TUNE_GROUP_PLAN, 2)
            ctx.set_tuning(_lib.TUNE_GROUP_COMBINE, combine)
            k, sm, c = ops.group_hash(dev(keys), dev(vals), dev(vals2) if two else None, max_groups=G, ctx=ctx)
            order = np.argsort(host(k))
            assert np.array_equal(host(k)[order], ek)
            assert np.array_equal(host(sm)[order], es) and np.array_equal(host(c)[order], ec)
    finally:
        ctx.set_tuning(_lib.TUNE_GROUP_PLAN, 0)
        ctx.set_tuning(_lib.TUNE_GROUP_COMBINE, 0)


@pytest.mark.parametrize("max_groups,distinct", [(100, 5000), (5000, 40000)])
def test_group_hash_more_keys_than_capacity_fails(ctx, max_groups, distinct):
    keys = np.arange(distinct, dtype=np.int32)
    vals = np.ones(distinct, np.int32)
    with pytest.raises(_lib.OlapError):
        ops.group_hash(dev(keys), dev(vals), max_groups=max_groups, ctx=ctx)


def test_bounded_device_wait_reports_timeout_and_context_survives(ctx):
    # a look-back waiting for a tile status that nothing publishes gives up
    st = _lib.lib.olap_debug_wait_timeout(ctx.handle, 1 << 14)
    assert st == _lib.OLAP_ERR_TIMEOUT
    col = np.arange(100_000, dtype=np.int32)
    assert np.array_equal(host(ops.select_rowids(dev(col), 99, ctx=ctx)), np.arange(100, dtype=np.int32))


@pytest.mark.parametrize("cap,n", [(8, 7), (64, 63), (1000, 999), (200_008, 150_000)])
def test_hash_join_any_capacity(ctx, cap, n):
    """Tables of any capacity that is a multiple of 8 above the build rows:
    nearly full ones (probe runs that wrap past the last slot) and a 3/4-full
    one; sums, matches and pairs equal the oracle's.  Capacities that are
    not multiples of 8, or not above n, are rejected."""
    rng = np.random.default_rng(cap)
    rk = rng.permutation(np.arange(n) - n // 2).astype(np.int32)  # n distinct keys, negatives too
    rp = rng.integers(-1000, 1000, n).astype(np.int32)
    sk = rng.integers(-n, n, 4 * n + 3).astype(np.int32)
    L, h = _lib.lib, ctx.handle
    table = torch.empty(cap, dtype=torch.int64, device="cuda")
    drk, drp = dev(rk), dev(rp)  # kept alive across the calls
    _lib.check(L.olap_hashjoin_build(h, drk.data_ptr(), drp.data_ptr(), n, table.data_ptr(), cap), h)
    s_, m_ = torch.zeros(1, dtype=torch.int64, device="cuda"), torch.zeros(1, dtype=torch.int64, device="cuda")
    dk = dev(sk)
    _lib.check(L.olap_hashjoin_probe_filtered(h, table.data_ptr(), cap, None, 0, dk.data_ptr(), len(sk),
                                              s_.data_ptr(), m_.data_ptr(), None, None), h)
    es, em = oracle.hashjoin(rk, rp, sk)
    assert (int(s_.item()), int(m_.item())) == (es, em)
    rows = torch.empty(len(sk), dtype=torch.int32, device="cuda")
    pay = torch.empty(len(sk), dtype=torch.int32, device="cuda")
    _lib.check(L.olap_hashjoin_probe_filtered(h, table.data_ptr(), cap, None, 0, dk.data_ptr(), len(sk), None,
                                              m_.data_ptr(), rows.data_ptr(), pay.data_ptr()), h)
    k = int(m_.item())
    _, _, erows, epay = oracle.hashjoin(rk, rp, sk, want_pairs=True)
    assert np.array_equal(host(rows[:k]), erows) and np.array_equal(host(pay[:k]), epay)
    for bad in (cap + 4, n):
        with pytest.raises(_lib.OlapError):
            _lib.check(L.olap_hashjoin_build(h, drk.data_ptr(), drp.data_ptr(), n, table.data_ptr(), bad), h)


@pytest.mark.parametrize("bloom", [True, False])
def test_hash_join_probe_large_table(ctx, bloom):
    """2^22 + 5 build rows (a table of about 8.4M slots, 67 MB: above one L2-sized
    region) probed by 2^22 + 1001 keys, with and without the Bloom filter,
    aligned and unaligned, a ragged count and edge keys: the same (sum,
    matches) as the oracle."""
    rng = np.random.default_rng(37)
    n = (1 << 22) + 5
    rk = rng.integers(-(1 << 23), 1 << 23, n).astype(np.int32)  # duplicates and negatives
    rp = rng.integers(-1000, 1000, n).astype(np.int32)
    sk = rng.integers(-(1 << 23), 1 << 23, (1 << 22) + 1001).astype(np.int32)
    sk[:7] = [np.iinfo(np.int32).min, np.iinfo(np.int32).max, 0, -1, 1, rk[0], rk[-1]]
    ht = ops.HashTable(n, ctx=ctx, bloom=bloom).build(dev(rk), dev(rp))
    assert ht.capacity > 1 << 22  # above one 32 MB region
    d = dev(sk)
    assert ht.probe(d) == oracle.hashjoin(rk, rp, sk)
    assert ht.probe(d[1:]) == oracle.hashjoin(rk, rp, sk[1:])


_M32 = 0xFFFFFFFF


def _hash32(x):
    x &= _M32
    x ^= x >> 16
    x = (x * 0x85EBCA6B) & _M32
    x ^= x >> 13
    x = (x * 0xC2B2AE35) & _M32
    return x ^ (x >> 16)


def _key_of_hash(h):
    """The key whose 32-bit murmur finaliser is h (the finaliser is a bijection)."""
    h ^= h >> 16
    h = (h * pow(0xC2B2AE35, -1, 1 << 32)) & _M32
    h ^= (h >> 13) ^ (h >> 26)
    h = (h * pow(0x85EBCA6B, -1, 1 << 32)) & _M32
    return h ^ (h >> 16)


@pytest.mark.parametrize("mode", [0, 3])
def test_hash_join_region_overflow_wraps(ctx, mode):
    """30,000 distinct keys whose home slots all lie in the last 16,384-slot
    region of a 2^23-slot table (plus 100,000 random keys and duplicates):
    the region overflows, so its rows' probe runs cross the table's end and
    wrap into the first region.  The shared-memory region build sets those
    rows aside and inserts them where linear probing over the whole table
    puts them; probes equal the oracle's, as with the L2 region build."""
    rng = np.random.default_rng(41)
    cap = 1 << 23
    lo = ((cap - 16384) << 32) // cap + 1  # hashes whose home slot is in the last region
    hs = rng.choice(np.arange(lo, 1 << 32, 97, dtype=np.int64), 30_000, replace=False)
    hot = np.array([_key_of_hash(int(h)) for h in hs], dtype=np.uint32).view(np.int32)
    assert all(((_hash32(int(k) & _M32) * cap) >> 32) >= cap - 16384 for k in hot[:100].view(np.uint32))
    rk = np.concatenate([hot, rng.integers(-2**31 + 1, 2**31, 100_000).astype(np.int32), hot[:5000]])
    rk = rk[rk != np.iinfo(np.int32).min]
    rp = np.arange(len(rk), dtype=np.int32) * 3 - 7
    sk = np.concatenate([rk[::3], rng.integers(-2**31 + 1, 2**31, 50_000).astype(np.int32)])
    L, h = _lib.lib, ctx.handle
    table = torch.empty(cap, dtype=torch.int64, device="cuda")
    drk, drp, dsk = dev(rk), dev(rp), dev(sk)
    ctx.set_tuning(_lib.TUNE_JOIN_BUILD, mode)
    try:
        _lib.check(L.olap_hashjoin_build(h, drk.data_ptr(), drp.data_ptr(), len(rk), table.data_ptr(), cap), h)
    finally:
        ctx.set_tuning(_lib.TUNE_JOIN_BUILD, 0)
    s_, m_ = torch.zeros(1, dtype=torch.int64, device="cuda"), torch.zeros(1, dtype=torch.int64, device="cuda")
    _lib.check(L.olap_hashjoin_probe_filtered(h, table.data_ptr(), cap, None, 0, dsk.data_ptr(), len(sk),
                                              s_.data_ptr(), m_.data_ptr(), None, None), h)
    assert (int(s_.item()), int(m_.item())) == oracle.hashjoin(rk, rp, sk)


@pytest.mark.parametrize("mode", [0, 2, 3])
def test_hash_join_region_build(ctx, mode):
    """A build side whose table is larger than one 32 MB region (2^22 rows:
    about 8.4M slots, 67 MB) is built by default 128 KB region by 128 KB
    region in shared memory (mode 0), directly (OLAP_TUNE_JOIN_BUILD = 2) or
    32 MB region by 32 MB region in L2 (3): duplicate keys keep their last
    row, the reserved key is counted, and probes equal the oracle's."""
    rng = np.random.default_rng(31)
    n = 1 << 22
    rk = rng.integers(-(1 << 23), 1 << 23, n).astype(np.int32)  # about 1/4 duplicates, negatives
    rk[::100_003] = np.iinfo(np.int32).min
    rp = np.arange(n, dtype=np.int32) ^ 0x5A5A5A5A
    sk = rng.integers(-(1 << 23), 1 << 23, 1 << 23).astype(np.int32)
    ctx.set_tuning(_lib.TUNE_JOIN_BUILD, mode)
    try:
        ht = ops.HashTable(n, ctx=ctx).build(dev(rk), dev(rp))
    finally:
        ctx.set_tuning(_lib.TUNE_JOIN_BUILD, 0)
    assert ht.capacity > 1 << 22  # above one 32 MB region
    assert ctx.take_range_errors() == int((rk == np.iinfo(np.int32).min).sum())
    assert ht.probe(dev(sk)) == oracle.hashjoin(rk, rp, sk)
    rows, pay = ht.probe_pairs(dev(sk[:300_000]))
    _, _, erows, epay = oracle.hashjoin(rk, rp, sk[:300_000], want_pairs=True)
    assert np.array_equal(host(rows), erows) and np.array_equal(host(pay), epay)


@pytest.mark.gpu
def test_hash_join_region_build_heavy_duplicates(ctx):
    """Half of 2^21 + 1,000 build rows share one key, so one 16,384-slot region of
    the shared-memory build holds a million rows (its block works through
    them in many rounds and then settles the duplicate's payload), and the
    rest are 1,000 keys repeated about a thousand times each: every key
    keeps the payload of its last row, through the filter or not."""
    rng = np.random.default_rng(53)
    n = (1 << 21) + 1000  # a table just above 2^22 slots: the shared-memory build
    rk = rng.integers(-500, 500, n).astype(np.int32)
    rk[rng.permutation(n)[: n // 2]] = 123_456_789
    rp = rng.integers(-(1 << 31), 1 << 31, n).astype(np.int32)
    sk = np.concatenate([np.arange(-600, 600, dtype=np.int32), np.full(1000, 123_456_789, np.int32),
                         rng.integers(-700, 700, 1 << 20).astype(np.int32)])
    for bloom in (True, False):
        ht = ops.HashTable(n, ctx=ctx, bloom=bloom).build(dev(rk), dev(rp))
        assert ht.capacity > 1 << 22
        assert ht.probe(dev(sk)) == oracle.hashjoin(rk, rp, sk)
        rows, pay = ht.probe_pairs(dev(sk[:5000]))
        _, _, erows, epay = oracle.hashjoin(rk, rp, sk[:5000], want_pairs=True)
        assert np.array_equal(host(rows), erows) and np.array_equal(host(pay), epay)


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [0, 2, 3])
@pytest.mark.parametrize("words", ["default", "one", "wide"])
def test_hash_join_build_filtered_matches_two_calls(ctx, mode, words):
    """olap_hashjoin_build_filtered gives the filter words, bit for bit, and
    the full slots that olap_hashjoin_build followed by
    olap_hashjoin_build_filter give: on the shared-memory region build (mode
    0, where the region blocks set the filter bits; with one filter word, and
    with a filter too wide for a region's run of words, which falls back to
    the separate pass), directly (2) and by L2 regions (3).  A table of a
    capacity that is not a power of two, duplicates, the reserved key."""
    L, h = _lib.lib, ctx.handle
    rng = np.random.default_rng(47)
    n = (1 << 21) + 12_345
    rk = rng.integers(-(1 << 22), 1 << 22, n).astype(np.int32)
    rk[::70_001] = np.iinfo(np.int32).min
    rp = rng.integers(-(1 << 31), 1 << 31, n).astype(np.int32)
    cap = int(L.olap_hashtable_capacity(n))
    assert cap > 1 << 22 and cap & (cap - 1)
    w = {"default": int(L.olap_hashjoin_filter_words(n)), "one": 1, "wide": 1 << 20}[words]
    drk, drp = dev(rk), dev(rp)
    ta = torch.empty(cap, dtype=torch.int64, device="cuda")
    tb = torch.empty(cap, dtype=torch.int64, device="cuda")
    fa = torch.empty(w, dtype=torch.int64, device="cuda")
    fb = torch.empty(w, dtype=torch.int64, device="cuda")
    ctx.set_tuning(_lib.TUNE_JOIN_BUILD, mode)
    try:
        _lib.check(L.olap_hashjoin_build_filtered(h, drk.data_ptr(), drp.data_ptr(), n, ta.data_ptr(), cap,
                                                  fa.data_ptr(), w), h)
        _lib.check(L.olap_hashjoin_build(h, drk.data_ptr(), drp.data_ptr(), n, tb.data_ptr(), cap), h)
        _lib.check(L.olap_hashjoin_build_filter(h, drk.data_ptr(), n, fb.data_ptr(), w), h)
        torch.cuda.synchronize()
    finally:
        ctx.set_tuning(_lib.TUNE_JOIN_BUILD, 0)
    assert ctx.take_range_errors() == 2 * int((rk == np.iinfo(np.int32).min).sum())
    assert torch.equal(fa, fb)
    empty = np.int64(np.uint64(0x80000000FFFFFFFF).astype(np.int64))
    sa, sb = host(ta), host(tb)
    assert np.array_equal(np.sort(sa[sa != empty]), np.sort(sb[sb != empty]))
    sk = rng.integers(-(1 << 22), 1 << 22, 1 << 22).astype(np.int32)
    s_, m_ = torch.zeros(1, dtype=torch.int64, device="cuda"), torch.zeros(1, dtype=torch.int64, device="cuda")
    dsk = dev(sk)
    _lib.check(L.olap_hashjoin_probe_filtered(h, ta.data_ptr(), cap, fa.data_ptr(), w, dsk.data_ptr(), len(sk),
                                              s_.data_ptr(), m_.data_ptr(), None, None), h)
    assert (int(s_.item()), int(m_.item())) == oracle.hashjoin(rk, rp, sk)
