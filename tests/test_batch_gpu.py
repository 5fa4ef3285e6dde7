"""GPU tests of the dimension-vector builder and the batched multi-query
star-join: every query of a batch gives, bit for bit, the result of running it
alone (its dimension vectors built by olap_build_dimvec, then one plain
star-join launch), with and without CUDA-graph replay, and the plain result
itself equals the CPU oracle."""
import numpy as np
import pytest

import oracle
from memory_database_b200 import _lib, batch, olapcore

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

SIZES = (30_000, 2_000, 200_000, 2_556)
GROUPS = (25, 25, 40, 7)


@pytest.fixture(scope="module")
def setup(ctx):
    dims = batch.make_dim_tables(ctx, SIZES, GROUPS, seed=3)
    n = 4_000_003
    L = _lib.lib
    fk = []
    for t, s in enumerate(SIZES):
        f = torch.empty(n, dtype=torch.int32, device="cuda")
        _lib.check(L.olap_gen_uniform_i32_dev(ctx.handle, f.data_ptr(), n, 9, 10 + t, 0, s - 1), ctx.handle)
        fk.append(f)
    m1 = torch.empty(n, dtype=torch.int32, device="cuda")
    m2 = torch.empty(n, dtype=torch.int32, device="cuda")
    _lib.check(L.olap_gen_uniform_i32_dev(ctx.handle, m1.data_ptr(), n, 9, 20, 1, 10000), ctx.handle)
    _lib.check(L.olap_gen_uniform_i32_dev(ctx.handle, m2.data_ptr(), n, 9, 21, -100, 100), ctx.handle)
    ctx.synchronize()
    return dims, fk, m1, m2, n


def test_build_dimvec_matches_definition(ctx, setup):
    dims = setup[0]
    for t in range(4):
        f, g = dims.filt[t].cpu().numpy(), dims.grp[t].cpu().numpy()
        for lo, hi, use in ((0, 1 << 20, 1), (1000, 300_000, 1), (5, 5, 0), (500_000, 900_000, 0)):
            q = batch.Query(0, 1, [lo] * 4, [hi] * 4, [t] if use else [], [t], [1] * 4, 1)
            v = batch.build_dimvecs(ctx, dims, q)[0].cpu().numpy()
            exp = np.where((f >= lo) & (f < hi), g if use else 0, 127).astype(np.int8)
            assert np.array_equal(v, exp)


def _check_batch(ctx, setup, queries, agg, use_graph, eng=None):
    dims, fk, m1, m2, n = setup
    eng = eng or batch.BatchEngine(ctx, dims, max_queries=max(64, len(queries)))
    out, tot, offs = eng.run(queries, fk, m1, m2, agg=agg, use_graph=use_graph)
    torch.cuda.synchronize()
    b_err = ctx.take_range_errors()
    p_err = 0
    for i, (q, off) in enumerate(zip(queries, offs)):
        gs, pt = batch.run_plain(ctx, dims, q, fk, m1, m2, agg=agg)
        torch.cuda.synchronize()
        p_err += ctx.take_range_errors()
        assert torch.equal(out[off: off + q.group_nums], gs[0]), q
        assert int(tot[i].item()) == int(pt[0].item())
    assert b_err == p_err
    return eng


@pytest.mark.parametrize("agg", [olapcore.AGG_M1_PLUS_M2, olapcore.AGG_M1_TIMES_M2, olapcore.AGG_COUNT])
def test_batch_equals_queries_alone(ctx, setup, agg):
    rng = np.random.default_rng(agg)
    qs = batch.random_queries(rng, 40, setup[4], GROUPS)
    # edge ranges: empty, one row at the end, the ragged tail, everything
    n = setup[4]
    qs[0].row_begin, qs[0].row_end = 100, 100
    qs[1].row_begin, qs[1].row_end = n - 1, n
    qs[2].row_begin, qs[2].row_end = n - 7, n
    qs[3].row_begin, qs[3].row_end = 0, n
    qs[4].lo, qs[4].hi = [0] * 4, [1 << 20] * 4  # no filtering at all
    _check_batch(ctx, setup, qs, agg, use_graph=False)


def test_batch_graph_replay_with_new_queries(ctx, setup):
    rng = np.random.default_rng(99)
    eng = None
    for rep, nq in enumerate((64, 64, 17, 40, 1, 64)):
        # recorded once per staging slot, then replayed for any query count
        qs = batch.random_queries(rng, nq, setup[4], GROUPS)
        eng = _check_batch(ctx, setup, qs, olapcore.AGG_M1_PLUS_M2, use_graph=True, eng=eng)
    assert eng.graph_captures() == 2


def test_batch_plain_path_matches_oracle(ctx, setup):
    dims, fk, m1, m2, n = setup
    rng = np.random.default_rng(5)
    q = batch.random_queries(rng, 1, n, GROUPS, sel_range=(0.05, 0.3))[0]
    vecs = [v.cpu().numpy() for v in batch.build_dimvecs(ctx, dims, q)]
    gs, tot = batch.run_plain(ctx, dims, q, fk, m1, m2)
    ogs, otot, _ = oracle.starjoin(vecs, [fk[t].cpu().numpy() for t in q.uses], [q.factor[t] for t in q.uses],
                                   m1.cpu().numpy(), m2.cpu().numpy(), q.group_nums,
                                   row_range=(q.row_begin, q.row_end))
    assert np.array_equal(gs.cpu().numpy(), ogs) and np.array_equal(tot.cpu().numpy(), otot)


@pytest.mark.parametrize("probe", [0, 1])
def test_batch_counts_out_of_range_keys_like_the_plain_path(ctx, setup, probe):
    dims, fk, m1, m2, n = setup
    bad = [f.clone() for f in fk]
    bad[1][::1000] = SIZES[1] + 3   # keys past the supplier table
    bad[3][5::777] = -1
    rng = np.random.default_rng(6)
    qs = batch.random_queries(rng, 16, n, GROUPS)
    eng = batch.BatchEngine(ctx, dims, max_queries=64)
    eng.tune(512, 4096, probe)
    _check_batch(ctx, (dims, bad, m1, m2, n), qs, olapcore.AGG_M1_PLUS_M2, use_graph=True, eng=eng)


@pytest.mark.parametrize("probe", [0, 1])
@pytest.mark.parametrize("block,slots", [(256, 0), (1024, 16384), (128, 2048), (768, 24576), (512, 4096)])
def test_launch_shapes_do_not_change_results(ctx, setup, block, slots, probe):
    """Every launch shape and both probe orders (all tables' masks in one
    round trip runs for blocks of at most 512 threads) give the results of
    the queries run alone."""
    rng = np.random.default_rng(block + slots)
    eng = batch.BatchEngine(ctx, setup[0], max_queries=64)
    eng.tune(block, slots, probe)
    assert eng.tuning() == (block, slots, probe if block <= 512 else 0)
    for nq in (64, 5):
        qs = batch.random_queries(rng, nq, setup[4], GROUPS)
        _check_batch(ctx, setup, qs, olapcore.AGG_M1_PLUS_M2, use_graph=True, eng=eng)
    with pytest.raises(_lib.OlapError):
        eng.tune(100, 0)
    with pytest.raises(_lib.OlapError):
        eng.tune(512, 1 << 20)


def test_autotuned_batch_shape(ctx, setup):
    rng = np.random.default_rng(17)
    eng = batch.BatchEngine(ctx, setup[0], max_queries=64)
    qs = batch.random_queries(rng, 64, setup[4], GROUPS)
    block, slots, ms = eng.autotune(qs, *setup[1:4], sample_rows=1 << 20)
    assert block in (256, 512, 1024) and slots in (0, 2048, 4096, 8192, 16384) and ms > 0
    assert ctx.take_range_errors() == 0
    _check_batch(ctx, setup, qs, olapcore.AGG_M1_PLUS_M2, use_graph=True, eng=eng)
