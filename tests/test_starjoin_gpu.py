"""GPU parity tests of the fused star-join (olap_starjoin_groupsum and the
reference-layout olap_OLAPcore) against the CPU oracle: bit-exact int64 per
group, on the reference's own queries and data stream, on the seeded
synthetic configurations, and on the edge cases the reference's contract
admits (empty and ragged ranges, unaligned columns, dropped rows)."""
import numpy as np
import pytest

import oracle
from memory_database_b200 import _lib, olapcore
from memory_database_b200.olapcore import (AGG_COUNT, AGG_M1, AGG_M1_PLUS_M2, AGG_M1_TIMES_M2,
                                           AGG_M2)

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def run_gpu(ctx, dvs, fks, factors, m1, m2, G, aggs=(AGG_M1_PLUS_M2,), row_range=None, lens=None):
    gs, tot = olapcore.starjoin_groupsum([dev(d) for d in dvs], [dev(f) for f in fks], factors,
                                         None if m1 is None else dev(m1),
                                         None if m2 is None else dev(m2), G, aggs=aggs,
                                         row_range=row_range, dimvec_lens=lens, ctx=ctx)
    torch.cuda.synchronize()
    return gs.cpu().numpy(), tot.cpu().numpy(), ctx.take_range_errors()


def check_same(ctx, dvs, fks, factors, m1, m2, G, aggs=(AGG_M1_PLUS_M2,), row_range=None, lens=None):
    g_gs, g_tot, g_err = run_gpu(ctx, dvs, fks, factors, m1, m2, G, aggs, row_range, lens)
    o_gs, o_tot, o_err = oracle.starjoin(dvs, fks, factors, m1, m2, G, aggs=aggs,
                                         row_range=row_range, dim_lens=lens)
    assert g_err == o_err
    assert np.array_equal(g_tot, o_tot)
    assert np.array_equal(g_gs, o_gs)
    return g_gs, g_tot


def random_star(seed, n, sizes, sele, groups, mlo=1, mhi=10000):
    rng = np.random.default_rng(seed)
    dv = []
    for s, p, g in zip(sizes, sele, groups):
        c = rng.integers(0, g, s).astype(np.int8)
        c[rng.random(s) >= p] = 127
        dv.append(c)
    fk = [rng.integers(0, s, n).astype(np.int32) for s in sizes]
    m1 = rng.integers(mlo, mhi + 1, n).astype(np.int32)
    m2 = rng.integers(mlo, mhi + 1, n).astype(np.int32)
    return dv, fk, m1, m2


def test_reference_queries_sf1_golden(ctx, golden_queries, golden_sf1_groups):
    """The reference's ten OLAPcore.sh queries on its own data stream (SF=1):
    grand totals equal the reference's, groups equal the reference's thread
    body, through the reference-layout entry point."""
    for q in golden_queries:
        dv, fk, m1, m2 = oracle.gen_olapcore_compat(1.0, q["sele"], q["bitmap"], q["groups"])
        ddv = [dev(d) for d in dv]
        dfk = [dev(f) for f in fk]
        G = q["group_nums"]
        gv = torch.zeros(G, dtype=torch.int64, device="cuda")
        for fn in (olapcore.OLAPcore_rowwise, olapcore.OLAPcore_vwm_dv, olapcore.OLAPcore_vwm_sv):
            total = fn(ddv, dfk, q["orders"], q["dimvec_nums"], q["factor"], len(m1), G,
                       dev(m1), dev(m2), 48, dimvec_len=[len(d) for d in dv], ctx=ctx,
                       group_vector=gv)
            assert total == q["total_sf1_reference"], (q["sqlnum"], fn.__name__)
            key = str(q["sqlnum"])
            if key in golden_sf1_groups:
                assert gv.cpu().tolist() == golden_sf1_groups[key]
        assert ctx.take_range_errors() == 0


def test_config1_small_star_join(ctx):
    """6M rows, 4 dims of 30000/2000/200000/2556 rows, selectivity 0.2,
    groups 5/25/40/7 (35,000 groups), measure uniform in [1, 10000]."""
    sizes, groups = [30000, 2000, 200000, 2556], [5, 25, 40, 7]
    orders, factor, nd, G = olapcore.plan_olapcore([0.2] * 4, [1] * 4, groups)
    dv, fk, m1, m2 = random_star(42, 6_000_000, sizes, [0.2] * 4, groups)
    for aggs in [(AGG_M1,), (AGG_M1_PLUS_M2,), (AGG_M1, AGG_M1_TIMES_M2), (AGG_COUNT, AGG_M2)]:
        check_same(ctx, [dv[t] for t in orders], [fk[t] for t in orders], factor, m1, m2, G, aggs)


@pytest.mark.parametrize("groups", [[1, 1, 1, 1], [2, 3, 1, 4], [5, 25, 40, 7], [16, 16, 64, 64]])
def test_group_cardinalities(ctx, groups):
    """From one group (contention) to 2^20 groups (global accumulators)."""
    sizes = [30000, 2000, 200000, 2556]
    sele = [0.9, 0.8, 0.7, 0.95]
    orders, factor, nd, G = olapcore.plan_olapcore(sele, [1] * 4, groups)
    dv, fk, m1, m2 = random_star(5, 1_000_003, sizes, sele, groups)
    check_same(ctx, [dv[t] for t in orders], [fk[t] for t in orders], factor, m1, m2, G,
               (AGG_M1, AGG_M1_TIMES_M2))


@pytest.mark.parametrize("nd", [0, 1, 2, 3])
def test_fewer_dimensions(ctx, nd):
    sizes, groups, sele = [3000, 20, 70000, 2556], [3, 4, 5, 6], [0.5, 0.9, 0.3, 1.0]
    dv, fk, m1, m2 = random_star(11, 300_001, sizes, sele, groups)
    fac = [int(np.prod(groups[j + 1:nd])) for j in range(nd)]
    G = int(np.prod(groups[:nd])) if nd else 1
    check_same(ctx, dv[:nd], fk[:nd], fac, m1, m2, G, (AGG_M1_PLUS_M2, AGG_COUNT))


@pytest.mark.parametrize("n", [0, 1, 2, 3, 4, 5, 7, 8, 9, 1023, 1024, 1025, 4097])
def test_ragged_sizes(ctx, n):
    _ragged(ctx, n)


@pytest.mark.parametrize("n", [0, 1, 3, 4, 5, 127, 128, 129, 131, 4095, 4097, 1_000_003])
def test_ragged_sizes_with_bulk_copy_prefetch(ctx, n):
    ctx.set_tuning(_lib.TUNE_ASYNC_LOADS, 2)
    try:
        _ragged(ctx, n)
        ctx.synchronize()  # raises if a prefetch wait gave up
    finally:
        ctx.set_tuning(_lib.TUNE_ASYNC_LOADS, 0)


@pytest.mark.parametrize("n", [1, 5, 129, 4097, 1_000_003])
def test_ragged_sizes_with_survivor_compaction(ctx, n):
    ctx.set_tuning(_lib.TUNE_COMPACT, 2)
    try:
        _ragged(ctx, n)
    finally:
        ctx.set_tuning(_lib.TUNE_COMPACT, 0)


def _ragged(ctx, n):
    sizes, groups, sele = [300, 20, 700, 25], [3, 4, 5, 6], [0.7, 0.9, 0.8, 1.0]
    dv, fk, m1, m2 = random_star(n + 1, max(n, 1), sizes, sele, groups)
    fk = [f[:n] for f in fk]
    check_same(ctx, dv, fk, [120, 30, 6, 1], m1[:n], m2[:n], 360)


@pytest.mark.parametrize("rb,re", [(0, 100000), (1, 100000), (3, 99997), (5, 6), (77777, 77777), (4, 64)])
def test_fact_ranges(ctx, rb, re):
    sizes, groups, sele = [300, 20, 700, 25], [3, 4, 5, 6], [0.7, 0.9, 0.8, 1.0]
    dv, fk, m1, m2 = random_star(3, 100000, sizes, sele, groups)
    check_same(ctx, dv, fk, [120, 30, 6, 1], m1, m2, 360, row_range=(rb, re))


def test_unaligned_columns_use_scalar_path(ctx):
    sizes, groups, sele = [300, 20, 700, 25], [3, 4, 5, 6], [0.7, 0.9, 0.8, 1.0]
    dv, fk, m1, m2 = random_star(9, 50001, sizes, sele, groups)
    dfk = [dev(f) for f in fk]
    dm1, dm2 = dev(m1), dev(m2)
    # views starting one element in: pointers are 4-byte but not 16-byte aligned
    gs, tot = olapcore.starjoin_groupsum([dev(d) for d in dv], [f[1:] for f in dfk], [120, 30, 6, 1],
                                         dm1[1:], dm2[1:], 360, ctx=ctx)
    o_gs, o_tot, _ = oracle.starjoin(dv, [f[1:] for f in fk], [120, 30, 6, 1], m1[1:], m2[1:], 360)
    assert np.array_equal(gs.cpu().numpy(), o_gs) and np.array_equal(tot.cpu().numpy(), o_tot)


def test_out_of_range_keys_and_groups_are_dropped_and_counted(ctx):
    rng = np.random.default_rng(1)
    n = 100_000
    dv = [rng.integers(-3, 6, 500).astype(np.int8), rng.integers(0, 4, 40).astype(np.int8)]
    dv[0][rng.random(500) < 0.2] = 127
    fk = [rng.integers(-2, 503, n).astype(np.int32), rng.integers(0, 41, n).astype(np.int32)]
    m1 = rng.integers(-1000, 1000, n).astype(np.int32)
    m2 = rng.integers(-(2 ** 31), 2 ** 31 - 1, n).astype(np.int32)
    g_gs, g_tot = check_same(ctx, dv, fk, [4, 1], m1, m2, 20, (AGG_M1_PLUS_M2, AGG_M1_TIMES_M2))
    assert g_gs.sum() != 0


def test_dimvec_len_pads_like_reference(ctx):
    """fk == size reads the extra (zero) byte, as the reference's inputs do."""
    dv = [np.array([127, 1, 127, 0], np.int8)]  # 3 entries + pad byte 0
    fk = [np.array([0, 1, 2, 3, 3, 1], np.int32)]
    m = np.arange(1, 7, dtype=np.int32)
    g, t = check_same(ctx, dv, fk, [1], m, m, 2)
    assert g[0].tolist() == [2 * (4 + 5), 2 * (2 + 6)]


@pytest.mark.parametrize("knobs", [
    {_lib.TUNE_SMEM_DIM_BYTES: 1},                       # nothing staged in smem
    {_lib.TUNE_SMEM_DIM_BYTES: 200 * 1024},              # everything small staged
    {_lib.TUNE_SMEM_ACC_BYTES: 1},                       # global accumulators
    {_lib.TUNE_UNROLL: 2},
    {_lib.TUNE_UNROLL: 3},
    {_lib.TUNE_BLOCK_THREADS: 128, _lib.TUNE_BLOCKS_PER_SM: 3},
    {_lib.TUNE_BLOCK_THREADS: 1024},
    {_lib.TUNE_PROBE_BITS: 1},                            # global pass bitmaps (L1)
    {_lib.TUNE_PROBE_BITS: 1, _lib.TUNE_SMEM_ACC_BYTES: 1},
    {_lib.TUNE_SMEM_BITS_BYTES: 200 * 1024},              # bitmaps staged in smem
    {_lib.TUNE_SMEM_BITS_BYTES: 8 * 1024, _lib.TUNE_PROBE_BITS: 1, _lib.TUNE_BLOCK_THREADS: 1024},
    {_lib.TUNE_SMEM_BITS_BYTES: 200 * 1024, _lib.TUNE_SMEM_DIM_BYTES: 1, _lib.TUNE_UNROLL: 2},
    {_lib.TUNE_BLOCK_THREADS: 768},
    {_lib.TUNE_ASYNC_LOADS: 2},                           # bulk-copy prefetch of the fact columns
    {_lib.TUNE_ASYNC_LOADS: 2, _lib.TUNE_UNROLL: 2},
    {_lib.TUNE_ASYNC_LOADS: 2, _lib.TUNE_SMEM_BITS_BYTES: 64 * 1024, _lib.TUNE_BLOCK_THREADS: 1024},
    {_lib.TUNE_ASYNC_LOADS: 2, _lib.TUNE_BLOCK_THREADS: 128, _lib.TUNE_BLOCKS_PER_SM: 3},
    {_lib.TUNE_ASYNC_LOADS: 2, _lib.TUNE_SMEM_ACC_BYTES: 1, _lib.TUNE_PROBE_BITS: 1},
    {_lib.TUNE_MERGE_PROBES: 1},                          # consecutive L2 probes issued together
    {_lib.TUNE_MERGE_PROBES: 1, _lib.TUNE_SMEM_DIM_BYTES: 1, _lib.TUNE_SMEM_ACC_BYTES: 1},
    {_lib.TUNE_MERGE_PROBES: 1, _lib.TUNE_SMEM_NIB_BYTES: 16 * 1024, _lib.TUNE_UNROLL: 2},
    {_lib.TUNE_PROBE_ORDER: 1},                           # int8-staged dimensions probed last
    {_lib.TUNE_PROBE_ORDER: 1, _lib.TUNE_MERGE_PROBES: 1, _lib.TUNE_SMEM_NIB_BYTES: 200 * 1024},
    {_lib.TUNE_PROBE_ORDER: 1, _lib.TUNE_COMPACT: 2, _lib.TUNE_SMEM_BITS_BYTES: 64 * 1024},
    {_lib.TUNE_PROBE_ORDER: 1, _lib.TUNE_ASYNC_LOADS: 2, _lib.TUNE_SMEM_NIB_BYTES: 16 * 1024},
    {_lib.TUNE_SMEM_NIB_BYTES: 200 * 1024},               # 4-bit codes staged in smem
    {_lib.TUNE_SMEM_NIB_BYTES: 16 * 1024, _lib.TUNE_SMEM_BITS_BYTES: 64 * 1024, _lib.TUNE_BLOCK_THREADS: 1024},
    {_lib.TUNE_SMEM_NIB_BYTES: 200 * 1024, _lib.TUNE_SMEM_DIM_BYTES: 1, _lib.TUNE_UNROLL: 2},
    {_lib.TUNE_SMEM_NIB_BYTES: 200 * 1024, _lib.TUNE_COMPACT: 2},
    {_lib.TUNE_COMPACT: 2},                               # per-warp survivor compaction
    {_lib.TUNE_COMPACT: 2, _lib.TUNE_SMEM_BITS_BYTES: 64 * 1024, _lib.TUNE_BLOCK_THREADS: 1024},
    {_lib.TUNE_COMPACT: 2, _lib.TUNE_PROBE_BITS: 1, _lib.TUNE_SMEM_ACC_BYTES: 1},
    {_lib.TUNE_COMPACT: 2, _lib.TUNE_SMEM_DIM_BYTES: 1, _lib.TUNE_BLOCK_THREADS: 128, _lib.TUNE_BLOCKS_PER_SM: 3},
])
def test_tuning_knobs_do_not_change_results(ctx, knobs):
    sizes, groups, sele = [30000, 2000, 20000, 2556], [5, 25, 4, 7], [0.3, 0.5, 0.7, 0.9]
    orders, factor, nd, G = olapcore.plan_olapcore(sele, [1] * 4, groups)
    dv, fk, m1, m2 = random_star(21, 777_777, sizes, sele, groups)
    try:
        for k, v in knobs.items():
            ctx.set_tuning(k, v)
        check_same(ctx, [dv[t] for t in orders], [fk[t] for t in orders], factor, m1, m2, G,
                   (AGG_M1, AGG_M1_TIMES_M2))
    finally:
        for k in knobs:
            ctx.set_tuning(k, 0)


def test_host_entry_point_matches_device(ctx):
    sizes, groups, sele = [30000, 2000, 200000, 2556], [5, 25, 40, 7], [0.2] * 4
    orders, factor, nd, G = olapcore.plan_olapcore(sele, [1] * 4, groups)
    dv, fk, m1, m2 = random_star(4, 2_000_001, sizes, sele, groups)
    dvs, fks = [dv[t] for t in orders], [fk[t] for t in orders]
    o_gs, o_tot, _ = oracle.starjoin(dvs, fks, factor, m1, m2, G, aggs=(AGG_M1, AGG_M1_TIMES_M2))
    ctx.set_tuning(_lib.TUNE_HOST_CHUNK_ROWS, 300_000)  # several chunks, ragged last one
    try:
        h_gs, h_tot = olapcore.starjoin_groupsum(dvs, fks, factor, m1, m2, G,
                                                 aggs=(AGG_M1, AGG_M1_TIMES_M2), ctx=ctx)
    finally:
        ctx.set_tuning(_lib.TUNE_HOST_CHUNK_ROWS, 0)
    assert np.array_equal(h_gs, o_gs) and np.array_equal(h_tot, o_tot)
    # pinned host buffers are read in place (the default for pinned columns)
    pin = [torch.from_numpy(f).pin_memory() for f in fks]
    pm1, pm2 = torch.from_numpy(m1).pin_memory(), torch.from_numpy(m2).pin_memory()
    h_gs2, h_tot2 = olapcore.starjoin_groupsum(dvs, [p.numpy() for p in pin], factor, pm1.numpy(),
                                               pm2.numpy(), G, aggs=(AGG_M1, AGG_M1_TIMES_M2), ctx=ctx)
    assert np.array_equal(h_gs2, o_gs) and np.array_equal(h_tot2, o_tot)


def test_host_entry_point_unknown_dim_lengths(ctx):
    """dimvec_len 0: the library copies dimvec[0 .. max fk], as the reference reads."""
    q = {"sele": [0.2, 0.2, 0.0, 0.857], "bitmap": [1, 1, 0, 1], "groups": [5, 5, 0, 6]}
    dv, fk, m1, m2 = oracle.gen_olapcore_compat(1.0, q["sele"], q["bitmap"], q["groups"])
    orders, factor, nd, G = olapcore.plan_olapcore(q["sele"], q["bitmap"], q["groups"])
    o_gs, o_tot, _ = oracle.starjoin([dv[t] for t in orders], [fk[t] for t in orders], factor, m1, m2, G)
    h_gs, h_tot = olapcore.starjoin_groupsum([dv[t] for t in orders], [fk[t] for t in orders], factor,
                                             m1, m2, G, dimvec_lens=[0] * nd, ctx=ctx)
    assert np.array_equal(h_gs, o_gs)


def test_device_generators_match_host(ctx):
    L = _lib.lib
    n = 3_000_017
    for fn_dev, fn_host, args, dt in [
        (L.olap_gen_uniform_i32_dev, L.olap_gen_uniform_i32, (42, 7, -100, 10000), torch.int32),
        (L.olap_gen_zipf_i32_dev, L.olap_gen_zipf_i32, (42, 8, 1_400_000, 0.8), torch.int32),
        (L.olap_gen_dimvec_dev, L.olap_gen_dimvec, (42, 9, 0.3, 40), torch.int8),
    ]:
        d = torch.empty(n, dtype=dt, device="cuda")
        _lib.check(fn_dev(ctx.handle, d.data_ptr(), n, *args), ctx.handle)
        ctx.synchronize()
        h = np.empty(n, dtype=np.int32 if dt == torch.int32 else np.int8)
        _lib.check(fn_host(h.ctypes.data, n, *args, 0))
        assert np.array_equal(d.cpu().numpy(), h)


def test_invalid_queries_rejected(ctx):
    d = dev(np.zeros(10, np.int8))
    f = dev(np.zeros(10, np.int32))
    with pytest.raises(_lib.OlapError):
        olapcore.starjoin_groupsum([d], [f], [1], f, f, 0, ctx=ctx)  # no groups
    with pytest.raises(_lib.OlapError):
        olapcore.starjoin_groupsum([d], [f], [1], None, f, 5, aggs=(AGG_M1,), ctx=ctx)  # M1 missing
    with pytest.raises(_lib.OlapError):
        olapcore.starjoin_groupsum([d], [f], [1], f, f, 5, aggs=(9,), ctx=ctx)


def test_bitmap_plans_with_nonzero_codes_and_drops(ctx):
    """Pass bitmaps (shared memory and global) must still fetch group codes
    for surviving rows, honour negative codes and count range errors."""
    rng = np.random.default_rng(12)
    n = 400_003
    sizes = [70_000, 9_000, 300_000]
    dv = [rng.integers(-2, 9, s).astype(np.int8) for s in sizes]
    for d in dv:
        d[rng.random(len(d)) < 0.4] = 127
    dv[1][:] = np.where(dv[1] == 127, 127, 0)  # a dimension whose live codes are all 0
    fk = [rng.integers(-1, s + 1, n).astype(np.int32) for s in sizes]
    m1 = rng.integers(1, 10000, n).astype(np.int32)
    m2 = rng.integers(1, 10000, n).astype(np.int32)
    for knobs in ({}, {_lib.TUNE_PROBE_BITS: 1}, {_lib.TUNE_SMEM_BITS_BYTES: 220 * 1024},
                  {_lib.TUNE_SMEM_BITS_BYTES: 2 * 1024, _lib.TUNE_PROBE_BITS: 1},
                  {_lib.TUNE_COMPACT: 2, _lib.TUNE_SMEM_BITS_BYTES: 2 * 1024},
                  {_lib.TUNE_COMPACT: 2, _lib.TUNE_PROBE_BITS: 1},
                  {_lib.TUNE_SMEM_NIB_BYTES: 200 * 1024}):  # negative codes: the int8 fallback
        try:
            for k, v in knobs.items():
                ctx.set_tuning(k, v)
            check_same(ctx, dv, fk, [100, 10, 1], m1, m2, 1000, (AGG_M1, AGG_M1_TIMES_M2))
        finally:
            for k in knobs:
                ctx.set_tuning(k, 0)


def test_autotuned_plan_gives_same_results(ctx):
    sizes, groups, sele = [300_000, 20_000, 140_000, 2556], [8, 8, 8, 8], [0.5, 0.2, 0.1, 1.0]
    orders, factor, nd, G = olapcore.plan_olapcore(sele, [1] * 4, groups)
    dv, fk, m1, m2 = random_star(31, 3_000_001, sizes, sele, groups)
    dvs, fks = [dv[t] for t in orders], [fk[t] for t in orders]
    try:
        knobs, ms = olapcore.autotune([dev(d) for d in dvs], [dev(f) for f in fks], factor, dev(m1),
                                      dev(m2), G, aggs=(AGG_M1, AGG_M1_TIMES_M2),
                                      sample_rows=1_000_000, ctx=ctx)
        assert ms > 0 and len(knobs) == 16
        check_same(ctx, dvs, fks, factor, m1, m2, G, (AGG_M1, AGG_M1_TIMES_M2))
    finally:
        for k in range(16):
            ctx.set_tuning(k, 0)


@pytest.mark.parametrize("hi", [14, 15, 40])
def test_four_bit_staging_and_its_fallback(ctx, hi):
    """Codes 0..14 use the staged 4-bit vectors; a code of 15 or more makes
    the kernel fall back to the int8 vector: same results either way."""
    rng = np.random.default_rng(hi)
    n = 300_001
    sizes = [5_000, 70_000, 2_000]
    dv = [rng.integers(0, hi + 1, s_).astype(np.int8) for s_ in sizes]
    for d in dv:
        d[rng.random(len(d)) < 0.3] = 127
    fk = [rng.integers(0, s_, n).astype(np.int32) for s_ in sizes]
    m1 = rng.integers(1, 10000, n).astype(np.int32)
    m2 = rng.integers(-50, 50, n).astype(np.int32)
    G = (hi + 1) ** 3
    for knobs in ({_lib.TUNE_SMEM_NIB_BYTES: 200 * 1024, _lib.TUNE_SMEM_DIM_BYTES: 1},
                  {_lib.TUNE_SMEM_NIB_BYTES: 4 * 1024, _lib.TUNE_SMEM_BITS_BYTES: 16 * 1024}):
        try:
            for k, v in knobs.items():
                ctx.set_tuning(k, v)
            check_same(ctx, dv, fk, [(hi + 1) ** 2, hi + 1, 1], m1, m2, G, (AGG_M1, AGG_M1_TIMES_M2))
        finally:
            for k in knobs:
                ctx.set_tuning(k, 0)


def test_launch_count_follows_the_plan(ctx):
    sizes, groups, sele = [30000, 2000, 20000, 2556], [5, 5, 4, 7], [0.3, 0.5, 0.7, 0.9]
    orders, factor, nd, G = olapcore.plan_olapcore(sele, [1] * 4, groups)
    dv, fk, m1, m2 = random_star(8, 100_000, sizes, sele, groups)
    dvs, fks = [dev(dv[t]) for t in orders], [dev(fk[t]) for t in orders]
    args = (dvs, fks, factor, dev(m1), dev(m2), G)
    try:
        # the star-join and its range pass (aligned columns: the 16-byte kernel)
        ctx.set_tuning(_lib.TUNE_SMEM_DIM_BYTES, 1)   # nothing staged as int8
        assert olapcore.launch_count(*args, ctx=ctx) == 2
        ctx.set_tuning(_lib.TUNE_SMEM_NIB_BYTES, 200 * 1024)  # every dimension as 4-bit codes
        assert olapcore.launch_count(*args, ctx=ctx) == 2 + nd
    finally:
        ctx.set_tuning(_lib.TUNE_SMEM_DIM_BYTES, 0)
        ctx.set_tuning(_lib.TUNE_SMEM_NIB_BYTES, 0)
