"""CPU tests of the C-ABI library: it loads, exports every declared symbol,
and its host-only functions (plan, generators) behave.  No GPU compute here."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

import oracle
from memory_database_b200 import _lib
from memory_database_b200 import olapcore

ROOT = Path(__file__).resolve().parents[1]


def declared_functions() -> list[str]:
    names = []
    for h in sorted((ROOT / "include").glob("*.h")):
        text = re.sub(r"/\*.*?\*/", "", h.read_text(), flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?[\w\s\*]+?\b(olap_\w+)\s*\(", text, flags=re.M)
    return sorted(set(names))


def test_library_exports_every_declared_symbol():
    names = declared_functions()
    assert len(names) >= 15
    lib = C.CDLL(str(_lib.LIB_PATH))
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_library_is_sm100a_build():
    assert "sm_100a" in _lib.build_info()


def test_status_strings():
    for st in range(0, -9, -1):
        assert _lib.lib.olap_status_string(st)


def test_no_device_fails_loudly():
    if _lib.device_count() > 0:
        pytest.skip("a device is present")
    with pytest.raises(_lib.OlapError) as e:
        olapcore.Context(0)
    assert e.value.status == _lib.OLAP_ERR_NO_DEVICE


def test_plan_matches_oracle(golden_queries):
    for q in golden_queries:
        assert olapcore.plan_olapcore(q["sele"], q["bitmap"], q["groups"]) == \
            oracle.plan(q["sele"], q["bitmap"], q["groups"])
    rng = np.random.default_rng(3)
    for _ in range(200):
        sele = rng.choice([0.0, 0.01, 0.2, 0.5, 1.0], 4).tolist()
        bitmap = rng.integers(0, 2, 4).tolist()
        groups = rng.integers(0, 9, 4).tolist()
        assert olapcore.plan_olapcore(sele, bitmap, groups) == oracle.plan(sele, bitmap, groups)


def _gen(fn, *args, n, dtype):
    out = np.empty(n, dtype)
    _lib.check(fn(out.ctypes.data, n, *args))
    return out


def test_uniform_generator_is_deterministic_and_in_range():
    L = _lib.lib
    a = _gen(L.olap_gen_uniform_i32, 42, 3, 1, 10000, 0, n=1_000_003, dtype=np.int32)
    b = _gen(L.olap_gen_uniform_i32, 42, 3, 1, 10000, 1, n=1_000_003, dtype=np.int32)
    assert np.array_equal(a, b)  # thread count does not change the values
    assert a.min() == 1 and a.max() == 10000
    assert abs(a.mean() - 5000.5) < 20
    c = _gen(L.olap_gen_uniform_i32, 42, 4, 1, 10000, 0, n=1000, dtype=np.int32)
    assert not np.array_equal(a[:1000], c)
    # a slice regenerates identically: value i depends only on (seed, stream, i)
    full = _gen(L.olap_gen_uniform_i32, 9, 1, -5, 5, 0, n=5000, dtype=np.int32)
    assert full.min() == -5 and full.max() == 5


def test_dimvec_generator_selectivity():
    L = _lib.lib
    d = _gen(L.olap_gen_dimvec, 42, 30, 0.2, 5, 0, n=400_000, dtype=np.int8)
    live = d != 127
    assert abs(live.mean() - 0.2) < 0.005
    assert set(np.unique(d[live]).tolist()) == {0, 1, 2, 3, 4}
    allnull = _gen(L.olap_gen_dimvec, 42, 30, 0.0, 5, 0, n=1000, dtype=np.int8)
    assert (allnull == 127).all()
    alllive = _gen(L.olap_gen_dimvec, 42, 30, 1.0, 3, 0, n=1000, dtype=np.int8)
    assert (alllive != 127).all()


def test_zipf_generator_skew():
    L = _lib.lib
    z = _gen(L.olap_gen_zipf_i32, 42, 5, 1000, 1.0, 0, n=500_000, dtype=np.int32)
    assert z.min() >= 0 and z.max() < 1000
    cnt = np.bincount(z, minlength=1000)
    h = (1.0 / np.arange(1, 1001)).sum()
    assert abs(cnt[0] / len(z) - 1.0 / h) < 0.01
    assert cnt[0] > cnt[1] > cnt[10] > cnt[500]
    u = _gen(L.olap_gen_zipf_i32, 42, 5, 1000, 0.0, 0, n=200_000, dtype=np.int32)
    assert abs(np.bincount(u, minlength=1000).std() / 200 - 0.07) < 0.05


def test_invalid_arguments_are_rejected():
    L = _lib.lib
    out = np.empty(4, np.int32)
    assert L.olap_gen_uniform_i32(out.ctypes.data, 4, 1, 1, 5, 4, 0) == _lib.OLAP_ERR_INVALID
    assert L.olap_gen_dimvec(out.ctypes.data, 4, 1, 1, 0.5, 200, 0) == _lib.OLAP_ERR_INVALID
    orders = (C.c_int * 4)()
    assert L.olap_plan_olapcore(None, None, None, orders, orders, None, None) == _lib.OLAP_ERR_INVALID
