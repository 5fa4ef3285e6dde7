"""CPU tests of the oracle: pinned against the reference's own outputs.

The oracle (oracle/olap_oracle.c) is the checker of every GPU parity test, so
it is itself checked here against (a) the golden fixtures produced by the
reference (tests/golden), (b) the reference's own functions compiled from its
sources (oracle/_ref), and (c) the reference's published SF=100 totals (slow).
"""
import numpy as np
import pytest

import oracle


def test_plan_matches_reference_main(golden_queries):
    for q in golden_queries:
        orders, factor, nd, gn = oracle.plan(q["sele"], q["bitmap"], q["groups"])
        assert (orders, factor, nd, gn) == (q["orders"], q["factor"], q["dimvec_nums"], q["group_nums"])


def test_sort_by_rate_quirk_kept():
    # q2.1: tables s, p, d participate; sort_by_rate compares sele by position
    # (sele[1]=0.2 > sele[2]=0.04) and swaps orders[1], orders[2].
    orders, factor, nd, gn = oracle.plan([0, 0.2, 0.04, 1], [0, 0, 1, 1], [0, 1, 40, 7])
    assert orders == [1, 3, 2] and factor == [1, 40, 1] and gn == 280


@pytest.mark.parametrize("idx", [0, 3, 7])
def test_compat_generator_matches_reference(golden_queries, idx):
    if not oracle.ref_available():
        pytest.skip("reference not built here")
    q = golden_queries[idx]
    a = oracle.gen_olapcore_compat(1.0, q["sele"], q["bitmap"], q["groups"])
    b = oracle.gen_olapcore_compat(1.0, q["sele"], q["bitmap"], q["groups"], use_reference=True)
    for x, y in zip(a[0] + a[1] + [a[2], a[3]], b[0] + b[1] + [b[2], b[3]]):
        assert np.array_equal(x, y)


def _compat_run(q, sf=1.0):
    dv, fk, m1, m2 = oracle.gen_olapcore_compat(sf, q["sele"], q["bitmap"], q["groups"])
    orders, factor, nd = q["orders"], q["factor"], q["dimvec_nums"]
    return oracle.starjoin([dv[t] for t in orders], [fk[t] for t in orders], factor, m1, m2,
                           q["group_nums"])


def test_oracle_sf1_totals_match_reference(golden_queries):
    for q in golden_queries:
        gs, tot, err = _compat_run(q)
        assert err == 0
        assert int(tot[0]) == q["total_sf1_reference"], q["sqlnum"]
        assert int(gs[0].sum()) == int(tot[0])


def test_oracle_sf1_groups_match_reference(golden_queries, golden_sf1_groups):
    for q in golden_queries:
        key = str(q["sqlnum"])
        if key not in golden_sf1_groups:
            continue
        gs, tot, err = _compat_run(q)
        assert gs[0].tolist() == golden_sf1_groups[key], q["sqlnum"]


def _random_star(seed, n, sizes, sele, groups, mlo=1, mhi=10000):
    rng = np.random.default_rng(seed)
    dv = []
    for s, p, g in zip(sizes, sele, groups):
        codes = rng.integers(0, g, s).astype(np.int8)
        codes[rng.random(s) >= p] = oracle_dim_null()
        dv.append(codes)
    fk = [rng.integers(0, s, n).astype(np.int32) for s in sizes]
    m1 = rng.integers(mlo, mhi + 1, n).astype(np.int32)
    m2 = rng.integers(mlo, mhi + 1, n).astype(np.int32)
    return dv, fk, m1, m2


def oracle_dim_null():
    return 127


def test_oracle_matches_reference_thread_bodies_random():
    if not oracle.ref_available():
        pytest.skip("reference not built here")
    ref = oracle.ref_lib()
    sizes, sele, groups = [3000, 200, 20000, 256], [0.5, 0.7, 0.6, 0.9], [5, 4, 10, 7]
    orders, factor, nd, gn = oracle.plan(sele, [1, 1, 1, 1], groups)
    n = 200_003
    dv, fk, m1, m2 = _random_star(7, n, sizes, sele, groups)
    gs, tot, err = oracle.starjoin([dv[t] for t in orders], [fk[t] for t in orders], factor, m1, m2, gn)
    assert err == 0
    o = np.array(orders, np.int32)
    f = np.array(factor, np.int32)
    dva, fka = oracle._ptr_array(dv), oracle._ptr_array(fk)
    for body in ("vwm", "row"):
        gv = np.zeros(gn, np.uint32)
        if body == "vwm":
            ref.ref_vwm_sv_groups(dva, fka, oracle._p(o), nd, oracle._p(f), 0, n, oracle._p(m1),
                                  oracle._p(m2), oracle._p(gv))
        else:
            ref.ref_row_groups(dva, fka, oracle._p(o), nd, oracle._p(f), n, oracle._p(m1),
                               oracle._p(m2), oracle._p(gv))
        assert np.array_equal(gs[0].astype(np.uint32), gv), body
    # the reference's int return is the total modulo 2^32
    r = ref.ref_OLAPcore_vwm_sv(dva, fka, oracle._p(o), nd, oracle._p(f), n, gn, oracle._p(m1),
                                oracle._p(m2), 3)
    assert (int(tot[0]) - r) % (1 << 32) == 0


def test_oracle_range_errors_and_aggregates():
    dv = [np.array([0, 1, 127, 2], np.int8)]
    fk = [np.array([0, 1, 2, 3, 4, -1, 3], np.int32)]
    m1 = np.array([1, 2, 3, 4, 5, 6, 7], np.int32)
    m2 = np.array([10, 20, 30, 40, 50, 60, 70], np.int32)
    gs, tot, err = oracle.starjoin(dv, fk, [1], m1, m2, 3, aggs=(0, 3, ))
    assert err == 2  # keys 4 and -1
    assert gs[0].tolist() == [11, 22, 44 + 77]
    assert gs[1].tolist() == [10, 40, 160 + 490]
    # group id outside [0, group_nums) is a range error too
    gs, tot, err = oracle.starjoin(dv, fk[:1], [1], m1, m2, 2, aggs=(4,))
    assert err == 2 + 2 and gs[0].tolist() == [1, 1]


@pytest.mark.slow
def test_oracle_sf100_published_totals(golden_queries):
    """The reference's published SF=100 totals (GPU/plot/old.py), re-derived."""
    for q in golden_queries[:1]:
        gs, tot, err = _compat_run(q, sf=100.0)
        assert int(tot[0]) == q["total_sf100_published"]
