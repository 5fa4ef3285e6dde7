"""CPU tests: the oracle's operator restatements against the reference's own
operator modules (select, join, group, aggregation, starjoin, project), compiled from
their sources into oracle/_ref.  Inputs follow the reference's generators
(values in [1, 1000], keys 1..R shuffled, 1-based group ids)."""
import numpy as np
import pytest

import oracle


def _need(name):
    try:
        return oracle.ref_module(name)
    except FileNotFoundError:
        pytest.skip("reference not built here")


def test_select_matches_reference():
    ref = _need("select")
    rng = np.random.default_rng(1)
    n = 100_003
    cols = [rng.integers(1, 1001, n).astype(np.int32) for _ in range(4)]
    for cond in (1, 100, 464, 1000):
        s, _ = oracle.selalgo(cond, *cols)
        assert s == ref.ref_selalgo_rowwise(cond, n, *[oracle._p(c) for c in cols])
        ids, err = oracle.select_rowids(cols[0], cond)
        out = np.zeros(n, np.int32)
        k = ref.ref_sel_fsel_branching(n, oracle._p(out), oracle._p(cols[0]), cond, None)
        assert err == 0 and np.array_equal(ids, out[:k])
        out2 = np.zeros(n, np.int32)
        k2 = ref.ref_sel_fsel_non_branching(n, oracle._p(out2), oracle._p(cols[0]), cond, None)
        assert k2 == k and np.array_equal(out2[:k2], out[:k])
        # chained selection through the first vector (if_sv)
        ids2, _ = oracle.select_rowids(cols[1], cond, in_rowids=ids)
        out3 = np.zeros(max(k, 1), np.int32)
        k3 = ref.ref_sel_fsel_branching(k, oracle._p(out3), oracle._p(cols[1]), cond, oracle._p(ids))
        assert np.array_equal(ids2, out3[:k3])
        bm = oracle.select_bitmap(cols[2], cond)
        bytes_ = np.zeros(n, np.uint8)
        ref.ref_sel_bmp(n, oracle._p(bytes_), oracle._p(cols[2]), cond)
        unpacked = np.unpackbits(bm.view(np.uint8), bitorder="little")[:n]
        assert np.array_equal(unpacked, bytes_)


def test_join_matches_reference():
    ref = _need("join")
    rng = np.random.default_rng(2)
    R = 1 << 14
    rk = rng.permutation(np.arange(1, R + 1)).astype(np.int32)
    rp = rng.integers(-50, 50, R).astype(np.int32)
    sk = rng.integers(1, R + 1, 200_000).astype(np.int32)
    vec = np.zeros(R + 1, np.int32)
    s_ref = ref.ref_vecjoin(oracle._p(rk), oracle._p(rp), R, oracle._p(sk), len(sk), oracle._p(vec))
    s, _, err = oracle.vecjoin(rk, rp, sk, R + 1)
    assert err == 0 and s == s_ref
    # hash join, half of the probe keys missing, duplicates in the build side
    rk2 = np.concatenate([rk, rk[:100]])
    rp2 = np.concatenate([rp, rng.integers(-50, 50, 100).astype(np.int32)])
    sk2 = np.where(rng.random(len(sk)) < 0.5, sk, sk + 2 * R).astype(np.int32)
    s_ref = ref.ref_hashjoin(oracle._p(rk2), oracle._p(rp2), len(rk2), oracle._p(sk2), len(sk2))
    s, m = oracle.hashjoin(rk2, rp2, sk2)
    assert s == s_ref


def test_group_matches_reference():
    ref = _need("group")
    rng = np.random.default_rng(3)
    n = 300_001
    for G in (32, 4096):
        idx = rng.integers(1, G + 1, n).astype(np.int32)
        m1 = rng.integers(1, 100, n).astype(np.int32)
        m2 = rng.integers(1, 100, n).astype(np.int32)
        gv_ref = np.zeros(G, np.int32)
        t_ref = ref.ref_vector_group(n, oracle._p(idx), oracle._p(m1), oracle._p(m2), oracle._p(gv_ref), G)
        tot, gv, cnt, err = oracle.vector_group(idx, m1, m2, G)
        assert err == 0 and tot == t_ref and np.array_equal(gv.astype(np.int32), gv_ref)
        assert cnt.sum() == n
        assert ref.ref_hashtable_group(n, oracle._p(idx), oracle._p(m1), oracle._p(m2)) == tot
        # the per-key hash group-by restatement: keys vecInx - 1, int32 map values
        uk, sums, cnts = oracle.hash_group(idx - 1, m1, m2)
        assert np.array_equal(uk, np.arange(G)) and sums.sum() == t_ref and cnts.sum() == n
        assert np.array_equal(sums.astype(np.int32), gv_ref)


def test_aggregation_matches_reference():
    ref = _need("aggregation")
    rng = np.random.default_rng(4)
    n = 1 << 16
    tax_pct = rng.integers(1, 21, n).astype(np.int32)
    qty = rng.integers(1, 11, n).astype(np.int32)
    price = rng.integers(5, 21, n).astype(np.int32)
    tax = tax_pct.astype(np.float64) / 100
    qty_d, price_d = qty.astype(np.float64), price.astype(np.float64)  # kept alive for the call
    r = ref.ref_aggalgo_rowwise(n, oracle._p(tax), oracle._p(qty_d), oracle._p(price_d))
    assert oracle.agg_f64(tax, qty_d, price_d) == r
    fixed = oracle.agg_fixed(price, qty, tax_pct)
    assert abs(fixed / 100.0 - r) <= 1e-9 * abs(r)


def test_starjoin_operator_matches_reference():
    ref = _need("starjoin")
    rng = np.random.default_rng(5)
    sizes = [3000, 200, 20000, 2555]
    n = 200_000
    dv = []
    for s in sizes:
        c = rng.integers(0, 16, s + 1).astype(np.int8)
        c[rng.random(s + 1) < 0.5] = 127
        c[s] = 0
        dv.append(c)
    fk = [rng.integers(0, s + 1, n).astype(np.int32) for s in sizes]
    args = [oracle._p(x) for x in dv + fk]
    cnt_ref = ref.ref_starjoin_rowwise(n, *args)
    res_ref = np.zeros(n, np.int32)
    c_ref = ref.ref_starjoin_cwm_sv(n, *args, oracle._p(res_ref))
    c, res = oracle.starjoin_cwm_sv(dv, [s + 1 for s in sizes], fk, n)
    assert c == c_ref and np.array_equal(res, res_ref)
    # the row-wise count is every survivor; the cwm count (the reference's
    # final loop) also skips survivors whose packed id happens to be 32767
    gs, tot, err = oracle.starjoin(dv, fk, [0, 0, 0, 0], None, None, 1, aggs=(4,))
    assert int(tot[0]) == cnt_ref and c <= cnt_ref


def test_join_cwm_sv_matches_reference_static_vector():
    """The reference's join_cwm_sv (via its fan-out with one thread) fills the
    same int16 static vector as the oracle restatement."""
    if not oracle.ref_available():
        pytest.skip("reference not built here")
    ref = oracle.ref_lib()
    q = {"sele": [0.2, 0.2, 0.0, 0.857], "bitmap": [1, 1, 0, 1], "groups": [5, 5, 0, 6]}
    dv, fk, m1, m2 = oracle.gen_olapcore_compat(1.0, q["sele"], q["bitmap"], q["groups"])
    orders, factor, nd, G = oracle.plan(q["sele"], q["bitmap"], q["groups"])
    n = len(m1)
    gid_ref = np.zeros(n, np.int16)
    o = np.array(orders + [0] * (4 - nd), np.int32)
    f = np.array(factor + [0] * (4 - nd), np.int32)
    tot_ref = ref.ref_OLAPcore_cwm_sv(oracle._ptr_array(dv), oracle._ptr_array(fk), oracle._p(o), nd,
                                      oracle._p(f), n, G, oracle._p(m1), oracle._p(m2), oracle._p(gid_ref), 1)
    gid, errs = oracle.join_cwm_sv([dv[t] for t in orders], [len(dv[t]) for t in orders],
                                   [fk[t] for t in orders], factor, n)
    assert errs == 0 and np.array_equal(gid, gid_ref)
    gs, tot, _ = oracle.starjoin([dv[t] for t in orders], [fk[t] for t in orders], factor, m1, m2, G)
    assert int(tot[0]) == tot_ref


@pytest.mark.parametrize("cond", [0, 1, 300, 999, 1000])
def test_project_matches_reference(cond):
    """oracle_project_pairs equals the reference's project module, compiled
    from its sources: proalgo_rowwise over both of its row stores
    (project/test_project_option.cpp:62-147, rows of row_store_min and
    row_store_max) and proalgo_cwm_lm_ifv (:527-595).  The reference's
    proalgo_cwm_em (:190-232) keeps the right rows and Rc values, but its
    second pass reads value 1 back at the row id instead of the list
    position (result.value2[cur_pos + pre_size]), so its Ra values are wrong
    unless every row passes; the library follows the other variants."""
    lib = _need("project")
    rng = np.random.default_rng(cond + 11)
    n = 1_000_003
    ra = rng.integers(1, 1001, n).astype(np.int32)
    rc = rng.integers(1, 1001, n).astype(np.int32)
    ea, ec = oracle.project_pairs(cond, ra, rc)
    p = oracle._p

    def run(fn, *head):
        oa, oc = np.zeros(n, np.int32), np.zeros(n, np.int32)
        k = fn(*head, cond, n, p(ra), p(rc), p(oa), p(oc))
        return k, oa[:k], oc[:k]
    for which in (0, 1):
        k, oa, oc = run(lib.ref_proalgo_rowwise, which)
        assert k == len(ea) and np.array_equal(oa, ea) and np.array_equal(oc, ec), which
    k, oa, oc = run(lib.ref_proalgo_cwm_lm_ifv)
    assert k == len(ea) and np.array_equal(oa, ea) and np.array_equal(oc, ec)
    k, oa, oc = run(lib.ref_proalgo_cwm_em)
    assert k == len(ea) and np.array_equal(oc, ec)
    assert np.array_equal(oa, ea) == (len(ea) in (0, n))
