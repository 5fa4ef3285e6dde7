"""GPU tests of the serving loop: every request's result, served in the
70/30 star-join / Q5 mix through continuous batching (and through the
one-launch-per-query lanes), equals the result of running that query alone."""
import numpy as np
import pytest

from memory_database_b200 import _lib, batch, olapcore, serving as S
from memory_database_b200 import q5 as Q5

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

SIZES = (30_000, 2_000, 200_000, 2_556)
GROUPS = (25, 25, 40, 7)


@pytest.fixture(scope="module")
def tables(ctx):
    dims = batch.make_dim_tables(ctx, SIZES, GROUPS, seed=5)
    n = 3_000_001
    L = _lib.lib
    fk = []
    for t, s in enumerate(SIZES):
        f = torch.empty(n, dtype=torch.int32, device="cuda")
        _lib.check(L.olap_gen_uniform_i32_dev(ctx.handle, f.data_ptr(), n, 12, 10 + t, 0, s - 1), ctx.handle)
        fk.append(f)
    m1 = torch.empty(n, dtype=torch.int32, device="cuda")
    m2 = torch.empty(n, dtype=torch.int32, device="cuda")
    _lib.check(L.olap_gen_uniform_i32_dev(ctx.handle, m1.data_ptr(), n, 12, 20, 1, 10000), ctx.handle)
    _lib.check(L.olap_gen_uniform_i32_dev(ctx.handle, m2.data_ptr(), n, 12, 21, -100, 100), ctx.handle)
    q5d = Q5.make_q5_data(ctx, n_supp=10_000, n_cust=100_000, n_orders=1_000_000, n_lines=4_000_000)
    ctx.synchronize()
    return dims, fk, m1, m2, n, q5d


def _alone(ctx, tables, r):
    dims, fk, m1, m2, n, q5d = tables
    if r.kind == "star":
        gs, tot = batch.run_plain(ctx, dims, r.query, fk, m1, m2)
        return np.concatenate([gs[0].cpu().numpy(), tot.cpu().numpy()])
    return Q5.q5(ctx, q5d, *r.query).cpu().numpy()


@pytest.mark.parametrize("rate,pool_bytes,plain_below", [(3000.0, 64 << 20, 3), (800.0, 512 << 10, 0)])
def test_mixed_requests_equal_queries_alone(ctx, tables, rate, pool_bytes, plain_below):
    dims, fk, m1, m2, n, q5d = tables
    rng = np.random.default_rng(int(rate))
    star = batch.random_queries(rng, 120, n, GROUPS)
    q5q = Q5.random_q5_queries(rng, 50)
    reqs = S.poisson_requests(rng, rate, 240, star, q5q)
    batched, plain = S.gpu_servers(dims, fk, m1, m2, q5d, pool_bytes=pool_bytes, plain_below=plain_below)
    a = batched.serve(S.reset(reqs))
    b = plain.serve(S.reset(reqs))
    torch.cuda.synchronize()
    assert all(r.status == "ok" for r in a) and all(r.status == "ok" for r in b)
    st = S.summarize(a, batched.batches)
    if rate >= 3000:
        assert st.mean_batch > 1.0   # requests shared launches
    for ra, rb in zip(a, b):
        exp = _alone(ctx, tables, ra)
        assert np.array_equal(ra.result, exp), (ra.rid, ra.kind, ra.batch_size)
        assert np.array_equal(rb.result, exp), (rb.rid, rb.kind)
    # the batched star lane replays its graphs instead of recording new ones
    assert batched.engine.graph_captures() <= 2
    for c in batched.contexts:
        assert c.take_range_errors() == 0
