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
