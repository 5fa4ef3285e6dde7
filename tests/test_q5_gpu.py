"""GPU parity of the TPC-H Q5-shaped join chain (olap_q5_chain) against the
oracle restatement of Q5.cpp:913-978 (int64 fixed point), on synthetic tables
of the serving configuration's shapes, every region and several date ranges,
plus invalid references."""
import numpy as np
import pytest

import oracle
from memory_database_b200 import q5 as Q5

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _host(data):
    return {k: v.cpu().numpy() for k, v in data.cols.items()}


def test_q5_matches_oracle(ctx):
    data = Q5.make_q5_data(ctx, n_supp=10_000, n_cust=150_000, n_orders=1_500_000, n_lines=6_000_000)
    h = _host(data)
    for region in range(5):
        for d1, d2 in ((0, 365), (730, 1095), (0, Q5.DAYS), (500, 500)):
            got = Q5.q5(ctx, data, region, d1, d2).cpu().numpy()
            exp, errs = oracle.q5(h, region, d1, d2)
            assert errs == 0 and np.array_equal(got, exp), (region, d1, d2)
            assert (got[[n for n in range(25) if n % 5 != region]] == 0).all()
    assert ctx.take_range_errors() == 0


def test_q5_config_sizes_and_invalid_references(ctx):
    data = Q5.make_q5_data(ctx)  # 100K suppliers, 1.5M customers, 15M orders, 60M lines
    h = _host(data)
    got = Q5.q5(ctx, data, 2, 365, 730).cpu().numpy()
    exp, _ = oracle.q5(h, 2, 365, 730)
    assert np.array_equal(got, exp) and got.sum() > 0
    data.cols["l_suppkey"][::1000] = 0          # not a supplier
    data.cols["l_orderkey"][7::999] = 15_000_000  # past the orders
    data.cols["o_custkey"][3::500] = 1_500_001    # past the customers
    h = _host(data)
    got = Q5.q5(ctx, data, 2, 365, 730).cpu().numpy()
    exp, errs = oracle.q5(h, 2, 365, 730)
    assert np.array_equal(got, exp) and ctx.take_range_errors() == errs > 0


def test_q5_batch_equals_queries_alone(ctx):
    data = Q5.make_q5_data(ctx, n_supp=20_000, n_cust=150_000, n_orders=2_000_000, n_lines=8_000_003)
    rng = np.random.default_rng(4)
    qs = Q5.random_q5_queries(rng, 64)
    qs[0] = (1, 100, 100)            # empty date range
    qs[1] = (7, 0, 365)              # no such region
    qs[2] = (3, -5, Q5.DAYS + 5)     # every order
    for n in (1, 2, 17, 64):
        got = Q5.q5_batch(ctx, data, qs[:n]).cpu().numpy()
        for q in range(n):
            alone = Q5.q5(ctx, data, *qs[q]).cpu().numpy()
            assert np.array_equal(got[q], alone), (n, q, qs[q])
    h = _host(data)
    exp, _ = oracle.q5(h, *qs[5])
    assert np.array_equal(got[5], exp)
    # a span wider than the date table: the per-query loop path
    wide = [(r, 0, 20_000) for r in range(5)] + [(2, 365, 730)]
    got = Q5.q5_batch(ctx, data, wide).cpu().numpy()
    for q, w in enumerate(wide):
        assert np.array_equal(got[q], Q5.q5(ctx, data, *w).cpu().numpy())
    assert ctx.take_range_errors() == 0


def test_q5_batch_counts_invalid_references_once(ctx):
    data = Q5.make_q5_data(ctx, n_supp=5_000, n_cust=50_000, n_orders=500_000, n_lines=2_000_000)
    data.cols["l_suppkey"][::997] = 5_001
    data.cols["o_custkey"][::101] = 0
    qs = [(r, 0, Q5.DAYS) for r in range(5)]
    got = Q5.q5_batch(ctx, data, qs).cpu().numpy()
    errs_batch = ctx.take_range_errors()
    for q, w in enumerate(qs):
        assert np.array_equal(got[q], Q5.q5(ctx, data, *w).cpu().numpy())
        ctx.synchronize()
        assert ctx.take_range_errors() == errs_batch  # every order in range: same count alone
