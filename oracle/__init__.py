"""ctypes loader of the CPU oracle (test infrastructure only).

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg import this package, and only as the checker.  ``liboracle.so`` is the
plain-C restatement (``olap_oracle.c``); ``_ref/libref_olapcore.so`` is the
reference's own OLAPcore source compiled in place (``Makefile``), present
only where it was built.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "liboracle.so"
REF_OLAPCORE_SO = HERE / "_ref" / "libref_olapcore.so"
# where the reference tree is read from when it is present (OLAP_REFERENCE_TREE)
REFERENCE_TREE = Path(os.environ.get("OLAP_REFERENCE_TREE", "/root/reference"))

_vp, _i64, _i32 = C.c_void_p, C.c_int64, C.c_int32


def build(with_reference: bool | None = None) -> None:
    """Compile the oracle (and the reference bridge when the tree exists)."""
    targets = ["oracle"]
    if with_reference is None:
        with_reference = REFERENCE_TREE.exists()
    if with_reference:
        targets.append("ref")
    subprocess.run(["make", "-s", "-C", str(HERE), f"OLAP_REFERENCE_TREE={REFERENCE_TREE}", *targets], check=True)


def _load_oracle() -> C.CDLL:
    if not ORACLE_SO.exists():
        build(with_reference=False)
    lib = C.CDLL(str(ORACLE_SO))
    lib.oracle_plan.argtypes = [_vp, _vp, _vp, _vp, _vp, C.POINTER(C.c_int), C.POINTER(_i64)]
    lib.oracle_starjoin.argtypes = [C.c_int, _vp, _vp, _vp, _vp, _i64, _i64, _vp, _vp, C.c_int,
                                    _vp, _i64, _vp, _vp, C.POINTER(_i64)]
    lib.oracle_starjoin_mt.argtypes = [C.c_int, C.c_int, _vp, _vp, _vp, _vp, _i64, _i64, _vp, _vp, C.c_int,
                                       _vp, _i64, _vp, _vp, C.POINTER(_i64)]
    lib.oracle_starjoin_mt.restype = C.c_int
    lib.oracle_hashjoin_sum_mt.argtypes = [C.c_int, _vp, _vp, _i64, _vp, _i64, C.POINTER(_i64)]
    lib.oracle_hashjoin_sum_mt.restype = _i64
    lib.oracle_gen_uniform_i32.argtypes = [_vp, _i64, C.c_uint64, C.c_uint64, _i32, _i32, C.c_int]
    lib.oracle_gen_uniform_i32.restype = C.c_int
    lib.oracle_gen_dimvec.argtypes = [_vp, _i64, C.c_uint64, C.c_uint64, C.c_double, _i32, C.c_int]
    lib.oracle_gen_dimvec.restype = C.c_int
    lib.oracle_gen_zipf_i32.argtypes = [_vp, _i64, C.c_uint64, C.c_uint64, _i64, C.c_double, C.c_int]
    lib.oracle_gen_zipf_i32.restype = C.c_int
    lib.oracle_size_of_table.argtypes = [C.c_int, C.c_double]
    lib.oracle_size_of_table.restype = C.c_int
    lib.oracle_gen_olapcore_compat.argtypes = [C.c_double, _vp, _vp, _vp, _vp, _vp, _vp, _vp]
    lib.oracle_gen_olapcore_compat.restype = C.c_int
    lib.oracle_glibc_rand_stream.argtypes = [C.c_uint32, _i64, _vp]
    lib.oracle_glibc_rand_stream.restype = C.c_int
    lib.oracle_select_rowids.argtypes = [_vp, _i64, _i32, C.c_int, _vp, _i64, _vp, C.POINTER(_i64)]
    lib.oracle_select_rowids.restype = _i64
    lib.oracle_select_bitmap.argtypes = [_vp, _i64, _i32, C.c_int, _vp]
    lib.oracle_selalgo.argtypes = [_i32, _i64, _vp, _vp, _vp, _vp, C.POINTER(_i64)]
    lib.oracle_selalgo.restype = _i64
    lib.oracle_project_pairs.argtypes = [_i32, _i64, _vp, _vp, _vp, _vp]
    lib.oracle_project_pairs.restype = _i64
    lib.oracle_gather.argtypes = [_vp, _i64, C.c_int, _vp, _i64, _vp]
    lib.oracle_gather.restype = _i64
    lib.oracle_vecjoin.argtypes = [_vp, _vp, _i64, _vp, _i64, _vp, _i64, C.POINTER(_i64)]
    lib.oracle_vecjoin.restype = _i64
    lib.oracle_hashjoin.argtypes = [_vp, _vp, _i64, _vp, _i64, C.POINTER(_i64), _vp, _vp]
    lib.oracle_hashjoin.restype = _i64
    lib.oracle_vector_group.argtypes = [_i64, _vp, _vp, _vp, _i64, _vp, _vp, C.POINTER(_i64)]
    lib.oracle_vector_group.restype = _i64
    lib.oracle_agg_fixed.argtypes = [_i64, _vp, _vp, _vp]
    lib.oracle_agg_fixed.restype = _i64
    lib.oracle_agg_f64.argtypes = [_i64, _vp, _vp, _vp]
    lib.oracle_agg_f64.restype = C.c_double
    lib.oracle_join_cwm_sv.argtypes = [C.c_int, _vp, _vp, _vp, _vp, _i64, _vp]
    lib.oracle_join_cwm_sv.restype = _i64
    lib.oracle_starjoin_cwm_sv.argtypes = [_vp, _vp, _vp, _i64, _vp]
    lib.oracle_starjoin_cwm_sv.restype = _i64
    lib.oracle_q5.argtypes = [_vp, _i64, _vp, _i64, _vp, _i64, _vp, _i64, _vp, _vp, _i64, _vp, _vp, _vp, _vp, _i64,
                              _i32, _i32, _i32, _vp]
    lib.oracle_q5.restype = _i64
    return lib


_ORACLE: C.CDLL | None = None
_REF: C.CDLL | None = None


def oracle_lib() -> C.CDLL:
    global _ORACLE
    if _ORACLE is None:
        _ORACLE = _load_oracle()
    return _ORACLE


def ref_available() -> bool:
    return REF_OLAPCORE_SO.exists()


def host_has_x86_64_v4() -> bool:
    """Whether this host's CPU has the AVX-512 features of x86-64-v4."""
    try:
        flags = set()
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("flags"):
                flags = set(line.split(":", 1)[1].split())
                break
        return {"avx512f", "avx512bw", "avx512cd", "avx512dq", "avx512vl"} <= flags
    except OSError:
        return False


_REF_V4: C.CDLL | None = None


def ref_lib_for_host() -> tuple[C.CDLL, str]:
    """The reference's OLAPcore built for this host's CPU: the x86-64-v4
    (AVX-512) build where the CPU has it, else the x86-64-v3 one.  Returns
    (library, build flags)."""
    global _REF_V4
    v4 = HERE / "_ref" / "libref_olapcore_v4.so"
    if host_has_x86_64_v4() and v4.exists():
        if _REF_V4 is None:
            _REF_V4 = _bind_ref_olapcore(C.CDLL(str(v4)))
        return _REF_V4, "-O3 -march=x86-64-v4"
    return ref_lib(), "-O3 -march=x86-64-v3"


def ref_lib() -> C.CDLL:
    """The reference's own OLAPcore functions (built from its sources)."""
    global _REF
    if _REF is None:
        if not REF_OLAPCORE_SO.exists():
            raise FileNotFoundError(f"{REF_OLAPCORE_SO} not built (needs the reference tree)")
        _REF = _bind_ref_olapcore(C.CDLL(str(REF_OLAPCORE_SO)))
    return _REF


def _bind_ref_olapcore(lib: C.CDLL) -> C.CDLL:
    fan = [_vp, _vp, _vp, C.c_int, _vp, C.c_int, C.c_int, _vp, _vp, C.c_int]
    for name in ("ref_OLAPcore_rowwise", "ref_OLAPcore_vwm_dv", "ref_OLAPcore_vwm_sv",
                 "ref_OLAPcore_cwm_dv"):
        getattr(lib, name).argtypes = fan
        getattr(lib, name).restype = C.c_int
    lib.ref_OLAPcore_cwm_sv.argtypes = fan[:-1] + [_vp, C.c_int]
    lib.ref_OLAPcore_cwm_sv.restype = C.c_int
    lib.ref_vwm_sv_groups.argtypes = [_vp, _vp, _vp, C.c_int, _vp, _i64, _i64, _vp, _vp, _vp]
    lib.ref_row_groups.argtypes = [_vp, _vp, _vp, C.c_int, _vp, _i64, _vp, _vp, _vp]
    lib.ref_gen_data_olapcore.argtypes = [C.c_double, _vp, _vp, _vp, _vp, _vp, _vp, _vp]
    return lib


def _p(a: np.ndarray) -> int:
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data


def _ptr_array(arrs) -> C.Array:
    return (C.c_void_p * 4)(*[(_p(a) if a is not None else None) for a in list(arrs) + [None] * (4 - len(arrs))])


def plan(sele, bitmap, groups):
    """The reference main's plan, restated (orders, factor, dimvec_nums, group_nums)."""
    lib = oracle_lib()
    s = np.ascontiguousarray(sele, dtype=np.float64)
    b = np.ascontiguousarray(bitmap, dtype=np.int32)
    g = np.ascontiguousarray(groups, dtype=np.int32)
    orders = np.zeros(4, np.int32)
    factor = np.zeros(4, np.int32)
    nd = C.c_int()
    gn = _i64()
    lib.oracle_plan(_p(s), _p(b), _p(g), _p(orders), _p(factor), C.byref(nd), C.byref(gn))
    return orders[: nd.value].tolist(), factor[: nd.value].tolist(), nd.value, gn.value


def starjoin(dimvecs, fks, factors, m1, m2, group_nums, aggs=(0,), row_range=None,
             dim_lens=None, want_groups=True, nthreads=1):
    """Oracle star-join over dimensions in probe order (row ranges over
    ``nthreads`` host threads when it is above 1; same result).

    Returns (group_sums[n_aggs, group_nums] int64 or None, totals[n_aggs], range_errors)."""
    lib = oracle_lib()
    nd = len(dimvecs)
    dv = [np.ascontiguousarray(d, dtype=np.int8) for d in dimvecs]
    fk = [np.ascontiguousarray(f, dtype=np.int32) for f in fks]
    lens = np.array([len(d) if dim_lens is None else dim_lens[j] for j, d in enumerate(dv)] + [0] * (4 - nd), np.int64)
    fac = np.array(list(factors) + [0] * (4 - nd), np.int32)
    m1a = None if m1 is None else np.ascontiguousarray(m1, dtype=np.int32)
    m2a = None if m2 is None else np.ascontiguousarray(m2, dtype=np.int32)
    n = len(fk[0]) if nd else (len(m1a) if m1a is not None else len(m2a))
    rb, re = row_range if row_range is not None else (0, n)
    ag = np.array(list(aggs), np.int32)
    gs = np.zeros((len(aggs), group_nums), np.int64) if want_groups else None
    tot = np.zeros(len(aggs), np.int64)
    err = _i64()
    args = (nd, _ptr_array(dv), _p(lens), _ptr_array(fk), _p(fac), rb, re,
            None if m1a is None else _p(m1a), None if m2a is None else _p(m2a),
            len(aggs), _p(ag), group_nums, None if gs is None else _p(gs), _p(tot), C.byref(err))
    if nthreads > 1:
        assert lib.oracle_starjoin_mt(int(nthreads), *args) == 0
    else:
        lib.oracle_starjoin(*args)
    return gs, tot, err.value


# ---- the benchmark's seeded tables (host copies of the library's generators) ----

def gen_uniform_i32(n, seed, stream, lo, hi, nthreads=0):
    out = np.empty(max(n, 1), np.int32)
    assert oracle_lib().oracle_gen_uniform_i32(_p(out), n, seed, stream, lo, hi, _threads(nthreads)) == 0
    return out[:n]


def gen_dimvec(n, seed, stream, sele, groups, nthreads=0):
    out = np.empty(max(n, 1), np.int8)
    assert oracle_lib().oracle_gen_dimvec(_p(out), n, seed, stream, float(sele), int(groups),
                                          _threads(nthreads)) == 0
    return out[:n]


def gen_zipf_i32(n, seed, stream, n_keys, s, nthreads=0):
    out = np.empty(max(n, 1), np.int32)
    assert oracle_lib().oracle_gen_zipf_i32(_p(out), n, seed, stream, n_keys, float(s), _threads(nthreads)) == 0
    return out[:n]


def _threads(n):
    import os
    return int(n) if n and n > 0 else (os.cpu_count() or 1)


class StarTables:
    """A star schema in host memory (numpy), with the reference main's plan."""

    def __init__(self, **kw):
        self.__dict__.update(kw)

    @property
    def probe_dims(self):
        return [self.dimvec[t] for t in self.orders]

    @property
    def probe_fks(self):
        return [self.fk[t] for t in self.orders]


def star_schema(n_rows, dim_sizes, sele, groups, bitmap=(1, 1, 1, 1), m_range=(1, 10_000), fk_dist="uniform",
                zipf_s=0.8, seed=42, fact_seed=None, nthreads=0):
    """The benchmark's star schema, bit-identical to the tables the GPU
    library generates for the same arguments (streams: foreign keys of table
    t -> 10 + t, M1 -> 20, M2 -> 21, dimension vector of table t -> 30 + t;
    ``fact_seed``, default ``seed``, seeds the fact columns)."""
    fseed = seed if fact_seed is None else fact_seed
    dimvec, fk = [], []
    for t in range(4):
        g = max(1, int(groups[t])) if bitmap[t] else 1
        dimvec.append(gen_dimvec(dim_sizes[t], seed, 30 + t, sele[t], g, nthreads))
        if fk_dist == "zipf":
            fk.append(gen_zipf_i32(n_rows, fseed, 10 + t, dim_sizes[t], zipf_s, nthreads))
        else:
            fk.append(gen_uniform_i32(n_rows, fseed, 10 + t, 0, dim_sizes[t] - 1, nthreads))
    m1 = gen_uniform_i32(n_rows, fseed, 20, m_range[0], m_range[1], nthreads)
    m2 = gen_uniform_i32(n_rows, fseed, 21, m_range[0], m_range[1], nthreads)
    orders, factor, nd, gn = plan(sele, bitmap, groups)
    return StarTables(n_rows=n_rows, dim_sizes=tuple(dim_sizes), dimvec=dimvec, fk=fk, m1=m1, m2=m2,
                      orders=orders, factor=factor, dimvec_nums=nd, group_nums=gn)


def size_of_table(table: int, sf: float) -> int:
    return int(oracle_lib().oracle_size_of_table(table, sf))


def glibc_rand_stream(seed: int, n: int) -> np.ndarray:
    """The first n values of glibc's rand() after srand(seed), restated."""
    out = np.zeros(max(n, 1), np.int32)
    assert oracle_lib().oracle_glibc_rand_stream(int(seed), int(n), _p(out)) == 0
    return out[:n]


def gen_olapcore_compat(sf, sele, bitmap, groups, use_reference=False, measures=True, fk_out=None):
    """The reference's OLAPcore dataset (glibc rand() from its default seed).

    Returns (dimvecs[4] with size+1 bytes each, fks[4], m1, m2); m1 and m2
    (constant 5) are None when ``measures`` is false.  ``fk_out``: four
    int32 arrays of the table's row count to fill instead of new ones."""
    sizes = [size_of_table(t, sf) for t in range(4)]
    n = size_of_table(4, sf)
    dv = [np.zeros(s + 1, np.int8) for s in sizes]
    if fk_out is not None:
        assert len(fk_out) == 4 and all(f.dtype == np.int32 and len(f) == n and f.flags["C_CONTIGUOUS"]
                                        for f in fk_out)
        fk = list(fk_out)
    else:
        fk = [np.empty(n, np.int32) for _ in range(4)]
    m1 = np.zeros(n, np.int32) if measures or use_reference else None
    m2 = np.zeros(n, np.int32) if measures or use_reference else None
    s = np.ascontiguousarray(sele, dtype=np.float64)
    b = np.ascontiguousarray(bitmap, dtype=np.int32)
    g = np.ascontiguousarray(groups, dtype=np.int32)
    if use_reference:
        ref_lib().ref_gen_data_olapcore(float(sf), _p(s), _p(b), _p(g), _ptr_array(dv),
                                        _ptr_array(fk), _p(m1), _p(m2))
    else:
        rc = oracle_lib().oracle_gen_olapcore_compat(float(sf), _p(s), _p(b), _p(g), _ptr_array(dv),
                                                     _ptr_array(fk), None if m1 is None else _p(m1),
                                                     None if m2 is None else _p(m2))
        assert rc == 0
    return dv, fk, m1, m2


# ---- operators -----------------------------------------------------------------

def _c32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def select_rowids(col, val, cmp=0, in_rowids=None):
    """(row ids, range_errors) of sel_lt_T_fsel_independent_val_branching."""
    col = _c32(col)
    n_in = 0 if in_rowids is None else len(in_rowids)
    ir = None if in_rowids is None else _c32(in_rowids)
    out = np.zeros(max(len(col) if ir is None else n_in, 1), np.int32)
    err = _i64()
    k = oracle_lib().oracle_select_rowids(_p(col), len(col), int(val), int(cmp), None if ir is None else _p(ir),
                                          n_in, _p(out), C.byref(err))
    return out[:k], err.value


def select_bitmap(col, val, cmp=0):
    col = _c32(col)
    bits = np.zeros(max((len(col) + 31) // 32, 1), np.uint32)
    oracle_lib().oracle_select_bitmap(_p(col), len(col), int(val), int(cmp), _p(bits))
    return bits[: (len(col) + 31) // 32]


def selalgo(cond, ra, rb, rc, rd):
    a, b, c, d = map(_c32, (ra, rb, rc, rd))
    cnt = _i64()
    s = oracle_lib().oracle_selalgo(int(cond), len(a), _p(a), _p(b), _p(c), _p(d), C.byref(cnt))
    return s, cnt.value


def project_pairs(cond, ra, rc):
    a, c = _c32(ra), _c32(rc)
    oa = np.zeros(max(len(a), 1), np.int32)
    oc = np.zeros(max(len(a), 1), np.int32)
    k = oracle_lib().oracle_project_pairs(int(cond), len(a), _p(a), _p(c), _p(oa), _p(oc))
    return oa[:k], oc[:k]


def gather(rowids, cols):
    r = _c32(rowids)
    cs = [_c32(c) for c in cols]
    outs = [np.zeros(max(len(r), 1), np.int32) for _ in cs]
    errs = oracle_lib().oracle_gather(_p(r), len(r), len(cs), (C.c_void_p * len(cs))(*[_p(c) for c in cs]),
                                      len(cs[0]), (C.c_void_p * len(cs))(*[_p(o) for o in outs]))
    return [o[: len(r)] for o in outs], errs


def vecjoin(rk, rp, sk, vector_len, initial=None):
    rk, rp, sk = _c32(rk), _c32(rp), _c32(sk)
    vec = np.zeros(vector_len, np.int32) if initial is None else _c32(initial).copy()
    err = _i64()
    s = oracle_lib().oracle_vecjoin(_p(rk), _p(rp), len(rk), _p(sk), len(sk), _p(vec), vector_len, C.byref(err))
    return s, vec, err.value


def hashjoin(rk, rp, sk, want_pairs=False):
    rk, rp, sk = _c32(rk), _c32(rp), _c32(sk)
    m = _i64()
    rows = np.zeros(max(len(sk), 1), np.int32) if want_pairs else None
    pay = np.zeros(max(len(sk), 1), np.int32) if want_pairs else None
    s = oracle_lib().oracle_hashjoin(_p(rk), _p(rp), len(rk), _p(sk), len(sk), C.byref(m),
                                     None if rows is None else _p(rows), None if pay is None else _p(pay))
    if want_pairs:
        return s, m.value, rows[: m.value], pay[: m.value]
    return s, m.value


def hashjoin_sum(rk, rp, sk, nthreads=1):
    """(SUM of matched payloads, matches) of the hash join, the probe side
    over ``nthreads`` host threads."""
    rk, rp, sk = _c32(rk), _c32(rp), _c32(sk)
    m = _i64()
    s = oracle_lib().oracle_hashjoin_sum_mt(int(nthreads), _p(rk), _p(rp), len(rk), _p(sk), len(sk), C.byref(m))
    assert m.value >= 0
    return s, m.value


def vector_group(idx, m1, m2, G, want_counts=True):
    idx, m1, m2 = _c32(idx), _c32(m1), _c32(m2)
    gv = np.zeros(G, np.int64)
    cnt = np.zeros(G, np.int64) if want_counts else None
    err = _i64()
    tot = oracle_lib().oracle_vector_group(len(idx), _p(idx), _p(m1), _p(m2), G, _p(gv),
                                           None if cnt is None else _p(cnt), C.byref(err))
    return tot, gv, cnt, err.value


def hash_group(keys, vals, vals2=None):
    """Per-key (keys ascending, int64 SUM of vals + vals2, COUNT) of a hash
    group-by: ``hashtable_group`` (code/group/test_group_option.cpp:71-88)
    adds m1[i] + m2[i] into ``group_hashtable[vecInx[i] - 1]``; this keeps
    every key's exact int64 sum and its row count, which the reference's
    32-bit map values and its returned total over keys 0..size-1 are checked
    against (tests/test_oracle_ops.py)."""
    keys = np.ascontiguousarray(keys, np.int32)
    v = np.asarray(vals, np.int64) + (np.asarray(vals2, np.int64) if vals2 is not None else 0)
    uk, inv = np.unique(keys, return_inverse=True)
    sums = np.zeros(len(uk), np.int64)
    np.add.at(sums, inv, v)
    return uk, sums, np.bincount(inv, minlength=len(uk)).astype(np.int64)


def agg_fixed(price, qty, tax):
    p, q, t = _c32(price), _c32(qty), _c32(tax)
    return oracle_lib().oracle_agg_fixed(len(p), _p(p), _p(q), _p(t))


def agg_f64(tax, qty, price):
    t, q, p = (np.ascontiguousarray(x, dtype=np.float64) for x in (tax, qty, price))
    return oracle_lib().oracle_agg_f64(len(t), _p(t), _p(q), _p(p))


def join_cwm_sv(dimvecs, lens, fks, factors, n):
    nd = len(dimvecs)
    dv = [np.ascontiguousarray(d, dtype=np.int8) for d in dimvecs]
    fk = [_c32(f) for f in fks]
    ln = np.array(list(lens) + [0] * (4 - nd), np.int64)
    fac = np.array(list(factors) + [0] * (4 - nd), np.int32)
    gid = np.zeros(max(n, 1), np.int16)
    errs = oracle_lib().oracle_join_cwm_sv(nd, _ptr_array(dv), _p(ln), _ptr_array(fk), _p(fac), n, _p(gid))
    return gid[:n], errs


def starjoin_cwm_sv(dimvecs, lens, fks, n):
    dv = [np.ascontiguousarray(d, dtype=np.int8) for d in dimvecs]
    fk = [_c32(f) for f in fks]
    ln = np.array(list(lens), np.int64)
    res = np.zeros(max(n, 1), np.int32)
    c = oracle_lib().oracle_starjoin_cwm_sv(_ptr_array(dv), _p(ln), _ptr_array(fk), n, _p(res))
    return c, res[:n]


def ref_module(name: str) -> C.CDLL:
    """The reference's own operator module (select, join, group, aggregation,
    starjoin, project) compiled from its sources into oracle/_ref."""
    path = HERE / "_ref" / f"libref_{name}.so"
    if not path.exists():
        raise FileNotFoundError(f"{path} not built (needs the reference tree)")
    lib = C.CDLL(str(path))
    if name == "select":
        lib.ref_selalgo_rowwise.argtypes = [C.c_int, C.c_int, _vp, _vp, _vp, _vp]
        lib.ref_sel_fsel_branching.argtypes = [C.c_int, _vp, _vp, C.c_int, _vp]
        lib.ref_sel_fsel_non_branching.argtypes = [C.c_int, _vp, _vp, C.c_int, _vp]
        lib.ref_sel_bmp.argtypes = [C.c_int, _vp, _vp, C.c_int]
    elif name == "join":
        lib.ref_vecjoin.argtypes = [_vp, _vp, C.c_uint64, _vp, C.c_uint64, _vp]
        lib.ref_hashjoin.argtypes = [_vp, _vp, C.c_uint64, _vp, C.c_uint64]
    elif name == "group":
        lib.ref_vector_group.argtypes = [C.c_uint64, _vp, _vp, _vp, _vp, C.c_int]
        lib.ref_vector_group.restype = _i64
        lib.ref_hashtable_group.argtypes = [C.c_uint64, _vp, _vp, _vp]
        lib.ref_hashtable_group.restype = _i64
    elif name == "aggregation":
        lib.ref_aggalgo_rowwise.argtypes = [C.c_int, _vp, _vp, _vp]
        lib.ref_aggalgo_rowwise.restype = C.c_double
    elif name == "project":
        for fn in ("ref_proalgo_cwm_lm_ifv", "ref_proalgo_cwm_em"):
            getattr(lib, fn).argtypes = [C.c_int, C.c_int, _vp, _vp, _vp, _vp]
            getattr(lib, fn).restype = C.c_int
        lib.ref_proalgo_rowwise.argtypes = [C.c_int, C.c_int, C.c_int, _vp, _vp, _vp, _vp]
        lib.ref_proalgo_rowwise.restype = C.c_int
    elif name == "starjoin":
        lib.ref_starjoin_rowwise.argtypes = [C.c_int] + [_vp] * 8
        lib.ref_starjoin_cwm_sv.argtypes = [C.c_int] + [_vp] * 9
    return lib


def q5(tables: dict, region: int, date1: int, date2: int):
    """(nation_sums, range_errors) of the Q5 chain; tables: name -> numpy array."""
    t = {k: _c32(v) for k, v in tables.items()}
    sums = np.zeros(len(t["n_regionkey"]), np.int64)
    errs = oracle_lib().oracle_q5(_p(t["r_regionkey"]), len(t["r_regionkey"]), _p(t["n_regionkey"]),
                                  len(t["n_regionkey"]), _p(t["s_nationkey"]), len(t["s_nationkey"]),
                                  _p(t["c_nationkey"]), len(t["c_nationkey"]), _p(t["o_custkey"]),
                                  _p(t["o_orderdate"]), len(t["o_custkey"]), _p(t["l_orderkey"]), _p(t["l_suppkey"]),
                                  _p(t["l_price"]), _p(t["l_discount"]), len(t["l_orderkey"]), int(region),
                                  int(date1), int(date2), _p(sums))
    return sums, errs
