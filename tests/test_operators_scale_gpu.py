"""GPU parity of the building-block operators at the benchmark's operator
sizes: select and a 4-column gather over 2^28 int32 rows at the four
selectivities, a hash join with a 2^24-key build side and a 2^28-key probe
side (uniform and Zipf(1.0) over the build keys, half of them matching
nothing), and a hash group-by over 2^28 rows at 16, 2^12, 2^20 and 2^22
groups (and Zipf(1.0) keys over 2^20).  Every result is compared with the
oracle on the same columns, bit for bit."""
import os

import numpy as np
import pytest

import oracle
from memory_database_b200 import _lib, operators as ops
from memory_database_b200.olapcore import _ptr

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

N = 1 << 28
NB = 1 << 24
NT = os.cpu_count() or 1


def gen_dev(ctx, n, stream, lo, hi, seed=99):
    x = torch.empty(n, dtype=torch.int32, device="cuda")
    _lib.check(_lib.lib.olap_gen_uniform_i32_dev(ctx.handle, _ptr(x), n, seed, stream, lo, hi), ctx.handle)
    return x


@pytest.fixture(scope="module")
def select_cols(ctx):
    col = gen_dev(ctx, N, 100, 0, (1 << 20) - 1)
    cols4 = [gen_dev(ctx, N, 101 + c, -1000, 1000) for c in range(4)]
    torch.cuda.synchronize()
    yield col, cols4, col.cpu().numpy(), [c.cpu().numpy() for c in cols4]
    del col, cols4
    torch.cuda.empty_cache()


@pytest.mark.parametrize("sel", [0.001, 0.01, 0.1, 0.5])
def test_select_and_gather_2p28(ctx, select_cols, sel):
    col, cols4, hcol, hcols4 = select_cols
    t = int(sel * (1 << 20))
    ids = ops.select_rowids(col, t, ops.CMP_LT, ctx=ctx)
    exp, err = oracle.select_rowids(hcol, t, 1)  # CMP_LT
    assert err == 0
    assert np.array_equal(ids.cpu().numpy(), exp)
    outs = ops.gather(ids, cols4, ctx=ctx)
    want, errs = oracle.gather(exp, hcols4)
    assert errs == 0
    for o, w in zip(outs, want):
        assert np.array_equal(o.cpu().numpy(), w)


@pytest.fixture(scope="module")
def build_side(ctx):
    # build keys: a bijection of [0, 2^24) onto [1, 2^24] (odd multiplier mod 2^24)
    bkeys = ((torch.arange(NB, device="cuda", dtype=torch.int64) * 2654435761) % NB + 1).to(torch.int32)
    bpay = gen_dev(ctx, NB, 110, -1000, 1000)
    ht = ops.HashTable(NB, ctx=ctx).build(bkeys, bpay)
    torch.cuda.synchronize()
    yield bkeys, bpay, ht, bkeys.cpu().numpy(), bpay.cpu().numpy()
    del ht
    torch.cuda.empty_cache()


@pytest.mark.parametrize("dist", ["uniform", "zipf1.0"])
def test_hash_join_2p24_build_2p28_probe(ctx, build_side, dist):
    bkeys, bpay, ht, hk, hp = build_side
    idx = torch.empty(N, dtype=torch.int32, device="cuda")
    if dist == "uniform":
        _lib.check(_lib.lib.olap_gen_uniform_i32_dev(ctx.handle, _ptr(idx), N, 99, 111, 0, NB - 1), ctx.handle)
    else:
        _lib.check(_lib.lib.olap_gen_zipf_i32_dev(ctx.handle, _ptr(idx), N, 99, 113, NB, 1.0), ctx.handle)
    miss = gen_dev(ctx, N, 112, 0, 1) == 0
    pk = bkeys[idx.long()]
    pk = torch.where(miss, pk + NB + 7, pk).contiguous()  # half match nothing
    del idx, miss
    s, m = ht.probe(pk)
    es, em = oracle.hashjoin_sum(hk, hp, pk.cpu().numpy(), nthreads=NT)
    assert (s, m) == (es, em)
    assert abs(m - N // 2) < N // 100
    del pk
    torch.cuda.empty_cache()


@pytest.mark.parametrize("G,dist", [(16, "uniform"), (1 << 12, "uniform"), (1 << 20, "uniform"),
                                    (1 << 22, "uniform"), (1 << 20, "zipf1.0")])
def test_hash_group_by_2p28(ctx, G, dist):
    vals = gen_dev(ctx, N, 120, 1, 10000)
    if dist == "uniform":
        keys = gen_dev(ctx, N, 121, 0, G - 1)
    else:
        keys = torch.empty(N, dtype=torch.int32, device="cuda")
        _lib.check(_lib.lib.olap_gen_zipf_i32_dev(ctx.handle, _ptr(keys), N, 99, 122, G, 1.0), ctx.handle)
    ok, os_, oc = ops.group_hash(keys, vals, max_groups=G, ctx=ctx)
    hk, hv = keys.cpu().numpy(), vals.cpu().numpy()
    del keys, vals
    tot, gv, cnt, err = oracle.vector_group(hk + 1, hv, np.zeros_like(hv), G)
    assert err == 0
    k = ok.cpu().numpy().astype(np.int64)
    present = np.flatnonzero(cnt)
    assert len(k) == len(present)
    assert np.array_equal(np.sort(k), present)  # every group once
    assert np.array_equal(os_.cpu().numpy(), gv[k])
    assert np.array_equal(oc.cpu().numpy(), cnt[k])
    del ok, os_, oc
    torch.cuda.empty_cache()
