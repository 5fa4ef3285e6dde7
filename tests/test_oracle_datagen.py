"""CPU tests: the oracle's host copy of the benchmark generators equals the
GPU library's own host generators bit for bit (so the CPU baseline can build
the benchmark's tables without loading the GPU library), and the oracle's
restatement of glibc's rand() equals the C library's."""
import ctypes
import ctypes.util

import numpy as np
import pytest

import oracle
from memory_database_b200 import _lib, workloads


@pytest.mark.parametrize("seed,stream,lo,hi", [(42, 10, 0, 2_999_999), (43, 21, 1, 10_000),
                                               (7, 3, -2**31, 2**31 - 1), (0, 0, 5, 5)])
def test_uniform_matches_library(seed, stream, lo, hi):
    n = 300_007
    want = np.empty(n, np.int32)
    _lib.check(_lib.lib.olap_gen_uniform_i32(want.ctypes.data, n, seed, stream, lo, hi, 3))
    assert np.array_equal(oracle.gen_uniform_i32(n, seed, stream, lo, hi, nthreads=5), want)


@pytest.mark.parametrize("sele,groups", [(0.5, 8), (0.0, 3), (1.0, 127), (0.013, 1)])
def test_dimvec_matches_library(sele, groups):
    n = 200_003
    want = np.empty(n, np.int8)
    _lib.check(_lib.lib.olap_gen_dimvec(want.ctypes.data, n, 42, 31, sele, groups, 2))
    assert np.array_equal(oracle.gen_dimvec(n, 42, 31, sele, groups, nthreads=3), want)


@pytest.mark.parametrize("n_keys,s", [(3_000_000, 0.8), (1 << 16, 1.0), (1, 0.5)])
def test_zipf_matches_library(n_keys, s):
    n = 100_003
    want = np.empty(n, np.int32)
    _lib.check(_lib.lib.olap_gen_zipf_i32(want.ctypes.data, n, 9, 12, n_keys, s, 4))
    assert np.array_equal(oracle.gen_zipf_i32(n, 9, 12, n_keys, s, nthreads=2), want)


def test_star_schema_matches_library():
    args = (100_001, (30_000, 2_000, 200_000, 2_556), (0.5, 0.2, 0.1, 1.0), (8, 8, 8, 8))
    a = oracle.star_schema(*args, seed=42)
    b = workloads.host_star_schema(*args, seed=42)
    assert (a.orders, a.factor, a.dimvec_nums, a.group_nums) == (b.orders, b.factor, b.dimvec_nums, b.group_nums)
    for x, y in zip(a.dimvec + a.fk + [a.m1, a.m2], b.dimvec + b.fk + [b.m1, b.m2]):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("seed", [1, 2, 12345, 0])
def test_glibc_rand_restatement_matches_c_library(seed):
    libc = ctypes.CDLL(ctypes.util.find_library("c"))
    if not hasattr(libc, "gnu_get_libc_version"):
        pytest.skip("the C library here is not glibc")
    libc.srand(seed)
    want = np.array([libc.rand() for _ in range(100_000)], np.int32)
    assert np.array_equal(oracle.glibc_rand_stream(seed, 100_000), want)
