// olap_reference_api.hpp — the reference's OLAP-core and operator C++
// signatures over the B200 C-ABI (header-only; link with libolapcore_b200.so).
//
// The reference (panjd123/memory_database) defines its OLAP core and its
// building-block operators as free C++ functions over host arrays, in
// code/OLAPcore/test_multi_compute_operator.cpp and code/{join,select,
// project,group,aggregation,starjoin}/test_*_option.cpp.  This header
// re-exposes them with the same names, parameter lists (int& sizes,
// nthreads, relation_t*, std::unordered_map&, fixed_arrays&) and return
// values, so a caller written against the reference builds unchanged against
// the B200 library.  The OLAP core's fused entry points:
//
//   int OLAPcore_rowwise(int8_t** dimvec_array, int32_t** fk_array, int* orders,
//                        int& dimvec_nums, int* factor, int& size_lineorder,
//                        int& group_nums, int32_t* M1, int32_t* M2, int nthreads)
//       (test_multi_compute_operator.cpp:973-976; OLAPcore_vwm_dv :1052 and
//        OLAPcore_vwm_sv :1258 have the same signature and result)
//
// All pointers are host pointers, as in the reference.  The fact columns are
// streamed through the GPU; each dimension vector is copied up to the largest
// key its fk column holds (the bytes the reference itself reads, including the
// one past the end that its generator's keys reach).  The return value is the
// grand total truncated to int exactly as the reference's uint32 group vector
// summed into an int; olap_last_total() returns the exact int64 total.
// nthreads is accepted and ignored.  Errors are reported by olap_last_status()
// (the reference exits the process instead).
//
// The operators (each function below cites the one it replaces) take the same
// host arrays: the header copies them to device buffers it keeps between
// calls, runs the library's device entry point and copies the results back
// into the caller's arrays or containers.  Arrays the reference indexes by a
// key without passing their length (dimension vectors, join vectors, the
// column behind a selection vector) are copied up to the largest key on the
// device, which is what the reference itself would read.  Integer results
// are the library's exact int64 sums, returned in the reference's type (an
// int is the sum modulo 2^32, as the reference's int and uint32 counters
// give it).
//
// Define OLAP_B200_DROP_IN before including this header to get the functions
// in the global namespace under the reference's names; otherwise they live in
// namespace olap_b200.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <unordered_map>
#include <utility>
#include <vector>

#include "olap_capi.h"

namespace olap_b200 {

namespace detail {

struct Table {  // a device hash table and its Bloom filter, built by build(R, hashtable)
  void* dev = nullptr;
  int64_t capacity = 0;
  void* filter = nullptr;
  int64_t words = 0;
};

struct State {
  std::mutex mu;
  olap_ctx* ctx = nullptr;
  int status = OLAP_OK;
  int64_t total = 0;
  std::vector<std::pair<void*, size_t>> bufs;  // grow-only device buffers by slot
  std::unordered_map<const void*, Table> tables;  // keyed by the caller's map
};

inline State& state() {
  static State s;
  return s;
}

// One context per process on device 0, created on first use.
inline olap_ctx* context() {
  State& s = state();
  if (!s.ctx) {
    s.status = olap_ctx_create(0, 0, &s.ctx);
    if (s.status != OLAP_OK) s.ctx = nullptr;
  }
  return s.ctx;
}

// Device buffer of slot i holding at least `bytes` (kept between calls).
inline void* buf(size_t i, size_t bytes) {
  State& s = state();
  if (s.bufs.size() <= i) s.bufs.resize(i + 1, {nullptr, 0});
  auto& b = s.bufs[i];
  if (b.second < bytes || !b.first) {
    if (b.first) olap_buffer_free(s.ctx, b.first);
    b = {nullptr, 0};
    const size_t want = bytes ? bytes : 16;
    if (olap_buffer_alloc(s.ctx, want, &b.first) != OLAP_OK) {
      s.status = OLAP_ERR_NOMEM;
      b.first = nullptr;
      return nullptr;
    }
    b.second = want;
  }
  return b.first;
}

// Copies `count` host values into slot i and returns the device copy.
template <class V>
inline V* put(size_t i, const V* host, size_t count) {
  void* d = buf(i, count * sizeof(V));
  if (!d) return nullptr;
  if (count && olap_copy_h2d(state().ctx, d, host, count * sizeof(V)) != OLAP_OK) {
    state().status = OLAP_ERR_CUDA;
    return nullptr;
  }
  return static_cast<V*>(d);
}

template <class V>
inline bool get(V* host, const void* dev, size_t count) {
  if (count && olap_copy_d2h(state().ctx, host, dev, count * sizeof(V)) != OLAP_OK) {
    state().status = OLAP_ERR_CUDA;
    return false;
  }
  return true;
}

inline int64_t get_i64(const void* dev) {
  int64_t v = 0;
  get(&v, dev, 1);
  return v;
}

// Entries of an array indexed by the keys of a device column: largest key + 1
// (0 when there is no non-negative key).
inline int64_t key_span(const int32_t* dkeys, int64_t n) {
  int32_t m = INT32_MIN;
  if (olap_max_i32(state().ctx, dkeys, n, &m) != OLAP_OK) {
    state().status = OLAP_ERR_CUDA;
    return 0;
  }
  return m < 0 ? 0 : static_cast<int64_t>(m) + 1;
}

// Reference int results: the exact sum modulo 2^32.
inline int as_ref_int(int64_t v) { return static_cast<int>(static_cast<uint32_t>(static_cast<uint64_t>(v))); }

// Status of a device entry point; dropped rows (a key out of range) become
// OLAP_ERR_RANGE, the results of the other rows are still returned.
inline bool ok(int st) {
  State& s = state();
  if (st != OLAP_OK) {
    s.status = st;
    return false;
  }
  int64_t dropped = 0;
  if (olap_ctx_take_range_errors(s.ctx, &dropped) != OLAP_OK) s.status = OLAP_ERR_CUDA;
  else if (dropped) s.status = OLAP_ERR_RANGE;
  return true;
}

// Starts a call: context, status cleared.  Returns null without a device.
inline olap_ctx* begin() {
  State& s = state();
  s.status = OLAP_OK;
  return context();
}

inline int run(int8_t** dimvec_array, int32_t** fk_array, const int* orders, int dimvec_nums,
               const int* factor, int size_lineorder, int group_nums, const int32_t* M1,
               const int32_t* M2) {
  State& s = state();
  std::lock_guard<std::mutex> lk(s.mu);
  olap_ctx* ctx = context();
  s.total = 0;
  if (!ctx) return 0;
  olap_starjoin_query q;
  std::memset(&q, 0, sizeof(q));
  q.dimvec_nums = dimvec_nums;
  q.n_aggs = 1;
  q.agg[0] = OLAP_AGG_M1_PLUS_M2;
  for (int j = 0; j < dimvec_nums && j < OLAP_MAX_DIMS; ++j) {
    q.dimvec[j] = dimvec_array[orders[j]];
    q.fk[j] = fk_array[orders[j]];
    q.dimvec_len[j] = 0;  // unknown: copy up to the largest key, as the reference reads
    q.factor[j] = factor[j];
  }
  q.m1 = M1;
  q.m2 = M2;
  q.row_begin = 0;
  q.row_end = size_lineorder;
  q.group_nums = group_nums;
  int64_t total = 0;
  s.status = olap_starjoin_groupsum_host(ctx, &q, nullptr, &total);
  s.total = total;
  // The reference sums uint32 group counters into an int.
  return static_cast<int>(static_cast<uint32_t>(static_cast<uint64_t>(total)));
}

}  // namespace detail

/// Status of the last call (OLAP_OK or an OLAP_ERR_* code).
inline int olap_last_status() { return detail::state().status; }
/// Exact int64 grand total of the last call.
inline int64_t olap_last_total() { return detail::state().total; }

/// OLAPcore_rowwise (test_multi_compute_operator.cpp:973) on the B200.
inline int OLAPcore_rowwise(int8_t** dimvec_array, int32_t** fk_array, int* orders, int& dimvec_nums,
                            int* factor, int& size_lineorder, int& group_nums, int32_t* M1,
                            int32_t* M2, int nthreads) {
  (void)nthreads;
  return detail::run(dimvec_array, fk_array, orders, dimvec_nums, factor, size_lineorder,
                     group_nums, M1, M2);
}

/// OLAPcore_vwm_dv (test_multi_compute_operator.cpp:1052) on the B200.
inline int OLAPcore_vwm_dv(int8_t** dimvec_array, int32_t** fk_array, int* orders, int& dimvec_nums,
                           int* factor, int& size_lineorder, int& group_nums, int32_t* M1,
                           int32_t* M2, int nthreads) {
  (void)nthreads;
  return detail::run(dimvec_array, fk_array, orders, dimvec_nums, factor, size_lineorder,
                     group_nums, M1, M2);
}

/// OLAPcore_vwm_sv (test_multi_compute_operator.cpp:1258) on the B200.
inline int OLAPcore_vwm_sv(int8_t** dimvec_array, int32_t** fk_array, int* orders, int& dimvec_nums,
                           int* factor, int& size_lineorder, int& group_nums, int32_t* M1,
                           int32_t* M2, int nthreads) {
  (void)nthreads;
  return detail::run(dimvec_array, fk_array, orders, dimvec_nums, factor, size_lineorder,
                     group_nums, M1, M2);
}

// ---- OLAP core, column-wise model (test_multi_compute_operator.cpp) --------

namespace detail {

// The tables in `orders` on the device: keys, and each dimension vector up to
// its column's largest key.  Slots from `slot` on.
struct DeviceTables {
  int8_t* dv[OLAP_MAX_DIMS] = {};
  int32_t* fk[OLAP_MAX_DIMS] = {};
  int64_t len[OLAP_MAX_DIMS] = {};
};

inline bool put_tables(int8_t** dimvec_array, int32_t** fk_array, const int* orders, int dimvec_nums, int n,
                       size_t slot, DeviceTables* t) {
  for (int j = 0; j < dimvec_nums && j < OLAP_MAX_DIMS; ++j) {
    const int tb = orders[j];
    if (tb < 0 || tb >= OLAP_MAX_DIMS) {
      state().status = OLAP_ERR_INVALID;
      return false;
    }
    if (t->fk[tb]) continue;
    t->fk[tb] = put(slot + 2 * tb, fk_array[tb], static_cast<size_t>(n));
    if (!t->fk[tb]) return false;
    t->len[tb] = key_span(t->fk[tb], n);
    t->dv[tb] = put(slot + 2 * tb + 1, dimvec_array[tb], static_cast<size_t>(t->len[tb] ? t->len[tb] : 1));
    if (!t->dv[tb]) return false;
    if (!t->len[tb]) t->len[tb] = 1;
  }
  return true;
}

}  // namespace detail

/// join_cwm_sv (test_multi_compute_operator.cpp:908): groupID[r] = the sum of
/// code * factor over the dimensions in orders, or GROUP_NULL.
inline void join_cwm_sv(int8_t** dimvec_array, int32_t** fk_array, int* orders, int& dimvec_nums,
                        int16_t* groupID, int* factor, int& size_lineorder, int nthreads) {
  (void)nthreads;
  std::lock_guard<std::mutex> lk(detail::state().mu);
  olap_ctx* ctx = detail::begin();
  if (!ctx) return;
  const int n = size_lineorder;
  detail::DeviceTables t;
  if (!detail::put_tables(dimvec_array, fk_array, orders, dimvec_nums, n, 0, &t)) return;
  int16_t* dg = static_cast<int16_t*>(detail::buf(8, sizeof(int16_t) * static_cast<size_t>(n)));
  if (!dg) return;
  if (detail::ok(olap_join_cwm_sv(ctx, t.dv, t.len, t.fk, orders, dimvec_nums, dg, factor, n)))
    detail::get(groupID, dg, static_cast<size_t>(n));
}

/// agg_cwm_sv (test_multi_compute_operator.cpp:764): SUM(M1 + M2) per group
/// id of the static vector; returns the total as the reference's int.
inline int agg_cwm_sv(int16_t* groupID, int& size_lineorder, int32_t* M1, int32_t* M2, int group_nums,
                      int nthreads) {
  (void)nthreads;
  std::lock_guard<std::mutex> lk(detail::state().mu);
  olap_ctx* ctx = detail::begin();
  if (!ctx) return 0;
  const size_t n = static_cast<size_t>(size_lineorder);
  int16_t* dg = detail::put(0, groupID, n);
  int32_t* d1 = detail::put(1, M1, n);
  int32_t* d2 = detail::put(2, M2, n);
  int64_t* gv = static_cast<int64_t*>(detail::buf(3, sizeof(int64_t) * static_cast<size_t>(group_nums)));
  int64_t* cnt = static_cast<int64_t*>(detail::buf(4, sizeof(int64_t)));
  if (!dg || !d1 || !d2 || !gv || !cnt) return 0;
  if (!detail::ok(olap_agg_cwm_sv(ctx, dg, size_lineorder, d1, d2, group_nums, gv, cnt))) return 0;
  detail::state().total = detail::get_i64(cnt);
  return detail::as_ref_int(detail::state().total);
}

/// join_cwm_dv (test_multi_compute_operator.cpp:840): the surviving rows of
/// each of the nthreads row ranges the reference's fan-out cuts (thread j:
/// rows [j*(n/nthreads), ...), the last thread the rest) as OID[j] (global
/// row) and groupID[j] lists in row order, index[j] their number.
inline void join_cwm_dv(int8_t** dimvec_array, int32_t** fk_array, int* orders, int& dimvec_nums, int64_t** OID,
                        int16_t** groupID, int* factor, int* index, int& size_lineorder, int nthreads) {
  std::lock_guard<std::mutex> lk(detail::state().mu);
  olap_ctx* ctx = detail::begin();
  if (!ctx || nthreads < 1) return;
  const int n = size_lineorder;
  detail::DeviceTables t;
  if (!detail::put_tables(dimvec_array, fk_array, orders, dimvec_nums, n, 0, &t)) return;
  int64_t* doid = static_cast<int64_t*>(detail::buf(8, sizeof(int64_t) * static_cast<size_t>(n)));
  int16_t* dg = static_cast<int16_t*>(detail::buf(9, sizeof(int16_t) * static_cast<size_t>(n)));
  int64_t* dk = static_cast<int64_t*>(detail::buf(10, sizeof(int64_t)));
  if (!doid || !dg || !dk) return;
  if (!detail::ok(olap_join_cwm_dv(ctx, t.dv, t.len, t.fk, orders, dimvec_nums, doid, dg, factor, dk, n))) return;
  const int64_t k = detail::get_i64(dk);
  std::vector<int64_t> oid(static_cast<size_t>(k));
  std::vector<int16_t> gid(static_cast<size_t>(k));
  if (!detail::get(oid.data(), doid, oid.size()) || !detail::get(gid.data(), dg, gid.size())) return;
  // split the row-ordered lists at the thread ranges' first rows
  const int64_t per = n / nthreads;
  size_t at = 0;
  for (int j = 0; j < nthreads; ++j) {
    const int64_t end = j == nthreads - 1 ? n : per * (j + 1);
    size_t e = at;
    while (e < oid.size() && oid[e] < end) ++e;
    const size_t cnt = e - at;
    if (cnt) {
      std::memcpy(OID[j], oid.data() + at, cnt * sizeof(int64_t));
      std::memcpy(groupID[j], gid.data() + at, cnt * sizeof(int16_t));
    }
    index[j] = static_cast<int>(cnt);
    at = e;
  }
}

/// agg_cwm_dv (test_multi_compute_operator.cpp:685): SUM(M1[OID] + M2[OID])
/// per group over the nthreads lists; returns the total as the reference's int.
inline int agg_cwm_dv(int64_t** OID, int16_t** groupID, int* index, int& size_lineorder, int32_t* M1, int32_t* M2,
                      int group_nums, int nthreads) {
  std::lock_guard<std::mutex> lk(detail::state().mu);
  olap_ctx* ctx = detail::begin();
  if (!ctx || nthreads < 1) return 0;
  std::vector<int64_t> oid;
  std::vector<int16_t> gid;
  for (int j = 0; j < nthreads; ++j) {
    oid.insert(oid.end(), OID[j], OID[j] + index[j]);
    gid.insert(gid.end(), groupID[j], groupID[j] + index[j]);
  }
  const size_t n = static_cast<size_t>(size_lineorder);
  int64_t* doid = detail::put(0, oid.data(), oid.size());
  int16_t* dg = detail::put(1, gid.data(), gid.size());
  int32_t* d1 = detail::put(2, M1, n);
  int32_t* d2 = detail::put(3, M2, n);
  int64_t* gv = static_cast<int64_t*>(detail::buf(4, sizeof(int64_t) * static_cast<size_t>(group_nums)));
  int64_t* cnt = static_cast<int64_t*>(detail::buf(5, sizeof(int64_t)));
  if (!doid || !dg || !d1 || !d2 || !gv || !cnt) return 0;
  if (!detail::ok(olap_agg_cwm_dv(ctx, doid, dg, static_cast<int64_t>(oid.size()), d1, d2, size_lineorder,
                                  group_nums, gv, cnt)))
    return 0;
  detail::state().total = detail::get_i64(cnt);
  return detail::as_ref_int(detail::state().total);
}

// ---- star-join operator (code/starjoin/test_starjoin_option.cpp) -----------

/// starjoinalgo_rowwise (test_starjoin_option.cpp:37): fact rows whose four
/// dimension probes are not DIM_NULL.
inline int starjoinalgo_rowwise(const int& size_lineorder, const int8_t* dimvec_c, const int8_t* dimvec_s,
                                const int8_t* dimvec_p, const int8_t* dimvec_d, const int32_t* fk_c,
                                const int32_t* fk_s, const int32_t* fk_p, const int32_t* fk_d) {
  std::lock_guard<std::mutex> lk(detail::state().mu);
  olap_ctx* ctx = detail::begin();
  if (!ctx) return 0;
  int8_t* dv[4] = {const_cast<int8_t*>(dimvec_c), const_cast<int8_t*>(dimvec_s), const_cast<int8_t*>(dimvec_p),
                   const_cast<int8_t*>(dimvec_d)};
  int32_t* fk[4] = {const_cast<int32_t*>(fk_c), const_cast<int32_t*>(fk_s), const_cast<int32_t*>(fk_p),
                    const_cast<int32_t*>(fk_d)};
  const int orders[4] = {0, 1, 2, 3};
  detail::DeviceTables t;
  if (!detail::put_tables(dv, fk, orders, 4, size_lineorder, 0, &t)) return 0;
  int64_t* cnt = static_cast<int64_t*>(detail::buf(8, sizeof(int64_t)));
  if (!cnt || !detail::ok(olap_starjoin_count(ctx, size_lineorder, t.dv, t.len, t.fk, cnt))) return 0;
  detail::state().total = detail::get_i64(cnt);
  return detail::as_ref_int(detail::state().total);
}

// ---- join (code/join/test_join_option.cpp) -----------------------------------

/// The reference's relation (include/metadata.h:263-270), for callers that do
/// not include its header; the join functions take any struct with its
/// key / payload / num_tuples members.
struct relation_t {
  int32_t* key;
  int32_t* payload;
  uint64_t num_tuples;
  double payload_rate;
  int table_size;
};

/// build(relation_t*, int* vector) (test_join_option.cpp:30): vector[key] =
/// payload, the last row winning.  The vector is read and written up to the
/// largest key.
template <class Rel>
inline void build(Rel* R, int* vector) {
  std::lock_guard<std::mutex> lk(detail::state().mu);
  olap_ctx* ctx = detail::begin();
  if (!ctx) return;
  const size_t n = static_cast<size_t>(R->num_tuples);
  int32_t* dk = detail::put(0, R->key, n);
  int32_t* dp = detail::put(1, R->payload, n);
  if (!dk || !dp) return;
  const int64_t len = detail::key_span(dk, static_cast<int64_t>(n));
  int32_t* dv = detail::put(2, vector, static_cast<size_t>(len));
  if (!dv) return;
  if (detail::ok(olap_vecjoin_build(ctx, dk, dp, static_cast<int64_t>(n), dv, len)))
    detail::get(vector, dv, static_cast<size_t>(len));
}

/// probe(relation_t*, int* vector) (test_join_option.cpp:58): SUM vector[key]
/// over the probe rows, as the reference's int.
template <class Rel>
inline int probe(Rel* S, int* vector) {
  std::lock_guard<std::mutex> lk(detail::state().mu);
  olap_ctx* ctx = detail::begin();
  if (!ctx) return 0;
  const size_t n = static_cast<size_t>(S->num_tuples);
  int32_t* dk = detail::put(0, S->key, n);
  if (!dk) return 0;
  const int64_t len = detail::key_span(dk, static_cast<int64_t>(n));
  int32_t* dv = detail::put(1, vector, static_cast<size_t>(len));
  int64_t* sum = static_cast<int64_t*>(detail::buf(2, sizeof(int64_t)));
  if (!dv || !sum || !detail::ok(olap_vecjoin_probe(ctx, dk, static_cast<int64_t>(n), dv, len, sum))) return 0;
  detail::state().total = detail::get_i64(sum);
  return detail::as_ref_int(detail::state().total);
}

/// probe_prefetch(relation_t*, int* vector) (test_join_option.cpp:72): the
/// same sum (the prefetch is a CPU detail).
template <class Rel>
inline int probe_prefetch(Rel* S, int* vector) {
  return probe(S, vector);
}

/// build(relation_t*, std::unordered_map<int,int>&) (test_join_option.cpp:44):
/// the build side goes into a hash table in device memory (with the Bloom
/// filter of its keys, through which probes go), which this header keeps
/// under the address of the caller's map (the map object itself is neither
/// read nor written; release() frees the table).  A duplicate key keeps the
/// payload of its last row, as the reference's map does.
template <class Rel>
inline void build(Rel* R, std::unordered_map<int, int>& hashtable) {
  std::lock_guard<std::mutex> lk(detail::state().mu);
  olap_ctx* ctx = detail::begin();
  if (!ctx) return;
  detail::State& s = detail::state();
  const size_t n = static_cast<size_t>(R->num_tuples);
  detail::Table& tb = s.tables[&hashtable];
  const int64_t cap = olap_hashtable_capacity(static_cast<int64_t>(n));
  const int64_t words = olap_hashjoin_filter_words(static_cast<int64_t>(n));
  if (tb.capacity != cap || tb.words != words) {
    if (tb.dev) olap_buffer_free(ctx, tb.dev);
    if (tb.filter) olap_buffer_free(ctx, tb.filter);
    tb = detail::Table();
    if (olap_buffer_alloc(ctx, static_cast<size_t>(cap) * sizeof(uint64_t), &tb.dev) != OLAP_OK ||
        olap_buffer_alloc(ctx, static_cast<size_t>(words) * sizeof(uint64_t), &tb.filter) != OLAP_OK) {
      if (tb.dev) olap_buffer_free(ctx, tb.dev);
      s.tables.erase(&hashtable);
      s.status = OLAP_ERR_NOMEM;
      return;
    }
    tb.capacity = cap;
    tb.words = words;
  }
  int32_t* dk = detail::put(0, R->key, n);
  int32_t* dp = detail::put(1, R->payload, n);
  if (!dk || !dp) return;
  detail::ok(olap_hashjoin_build_filtered(ctx, dk, dp, static_cast<int64_t>(n), static_cast<uint64_t*>(tb.dev), cap,
                                          static_cast<uint64_t*>(tb.filter), words));
}

/// probe(relation_t*, std::unordered_map<int,int>&) (test_join_option.cpp:90):
/// SUM of the payloads of the matching build rows (a key with no match adds
/// 0, as operator[] does) as the reference's int.  Probes the device table
/// build() made for this map; a map filled by the caller instead is built
/// from its entries first.  Unlike operator[], missing keys are not inserted.
template <class Rel>
inline int probe(Rel* S, std::unordered_map<int, int>& hashtable) {
  std::unique_lock<std::mutex> lk(detail::state().mu);
  olap_ctx* ctx = detail::begin();
  if (!ctx) return 0;
  detail::State& s = detail::state();
  if (!s.tables.count(&hashtable)) {
    std::vector<int32_t> k, p;
    k.reserve(hashtable.size());
    p.reserve(hashtable.size());
    for (const auto& kv : hashtable) {
      k.push_back(kv.first);
      p.push_back(kv.second);
    }
    relation_t R{k.data(), p.data(), static_cast<uint64_t>(k.size()), 0.0, 0};
    lk.unlock();
    build(&R, hashtable);
    lk.lock();
    if (!s.tables.count(&hashtable)) return 0;
    s.status = OLAP_OK;
  }
  const detail::Table& tb = s.tables[&hashtable];
  const size_t n = static_cast<size_t>(S->num_tuples);
  int32_t* dk = detail::put(0, S->key, n);
  int64_t* sum = static_cast<int64_t*>(detail::buf(1, sizeof(int64_t)));
  if (!dk || !sum) return 0;
  if (!detail::ok(olap_hashjoin_probe_filtered(ctx, static_cast<const uint64_t*>(tb.dev), tb.capacity,
                                               static_cast<const uint64_t*>(tb.filter), tb.words, dk,
                                               static_cast<int64_t>(n), sum, nullptr, nullptr, nullptr)))
    return 0;
  s.total = detail::get_i64(sum);
  return detail::as_ref_int(s.total);
}

/// Frees the device table build() keeps for this map.
inline void release(std::unordered_map<int, int>& hashtable) {
  std::lock_guard<std::mutex> lk(detail::state().mu);
  detail::State& s = detail::state();
  auto it = s.tables.find(&hashtable);
  if (it == s.tables.end()) return;
  if (it->second.dev && s.ctx) olap_buffer_free(s.ctx, it->second.dev);
  if (it->second.filter && s.ctx) olap_buffer_free(s.ctx, it->second.filter);
  s.tables.erase(it);
}

// ---- select (code/select/test_select_option.cpp) -----------------------------

/// sel_lt_T_fsel_independent_val_branching (test_select_option.cpp:391): the
/// row ids i < n with col1[i] <= *val2 (or the entries of if_sv that pass),
/// ascending, into res; returns their count.
inline int sel_lt_T_fsel_independent_val_branching(int n, int* res, const int* col1, int* val2, int* if_sv) {
  std::lock_guard<std::mutex> lk(detail::state().mu);
  olap_ctx* ctx = detail::begin();
  if (!ctx) return 0;
  const size_t m = static_cast<size_t>(n);
  int32_t* dsv = nullptr;
  int64_t col_len = n;
  if (if_sv) {
    dsv = detail::put(0, if_sv, m);
    if (!dsv) return 0;
    col_len = detail::key_span(dsv, n);
  }
  int32_t* dc = detail::put(1, col1, static_cast<size_t>(col_len));
  int32_t* dr = static_cast<int32_t*>(detail::buf(2, sizeof(int32_t) * (m ? m : 1)));
  int64_t* cnt = static_cast<int64_t*>(detail::buf(3, sizeof(int64_t)));
  if (!dc || !dr || !cnt) return 0;
  if (!detail::ok(olap_select_rowids(ctx, dc, col_len, *val2, OLAP_CMP_LE, dsv, if_sv ? n : 0, dr, cnt))) return 0;
  const int64_t k = detail::get_i64(cnt);
  detail::get(res, dr, static_cast<size_t>(k));
  return static_cast<int>(k);
}

/// sel_lt_T_fsel_independent_val_non_branching (test_select_option.cpp:172):
/// the same row ids (branching is a CPU detail).
inline int sel_lt_T_fsel_independent_val_non_branching(int n, int* res, const int* col1, int* val2, int* if_sv) {
  return sel_lt_T_fsel_independent_val_branching(n, res, col1, val2, if_sv);
}

/// selalgo_rowwise (test_select_option.cpp:450): SUM(Rd) over the rows with
/// Ra, Rb and Rc all <= condition, as the reference's int.
inline int selalgo_rowwise(int condition, const int& size_R, const int* Ra, const int* Rb, const int* Rc,
                           const int* Rd) {
  std::lock_guard<std::mutex> lk(detail::state().mu);
  olap_ctx* ctx = detail::begin();
  if (!ctx) return 0;
  const size_t n = static_cast<size_t>(size_R);
  int32_t* a = detail::put(0, Ra, n);
  int32_t* b = detail::put(1, Rb, n);
  int32_t* c = detail::put(2, Rc, n);
  int32_t* d = detail::put(3, Rd, n);
  int64_t* sum = static_cast<int64_t*>(detail::buf(4, sizeof(int64_t)));
  if (!a || !b || !c || !d || !sum) return 0;
  if (!detail::ok(olap_selalgo(ctx, condition, size_R, a, b, c, d, sum, nullptr))) return 0;
  detail::state().total = detail::get_i64(sum);
  return detail::as_ref_int(detail::state().total);
}

// ---- project (code/project/test_project_option.cpp) -------------------------

namespace detail {

// Pairs (Ra, Rc) of the rows with both <= condition, from a device
// projection, copied to the host.
inline bool pairs_to_host(int64_t k, const int32_t* da, const int32_t* dc, std::vector<int32_t>* a,
                          std::vector<int32_t>* c) {
  a->resize(static_cast<size_t>(k));
  c->resize(static_cast<size_t>(k));
  return get(a->data(), da, a->size()) && get(c->data(), dc, c->size());
}

template <class Row>
inline int64_t project_rows(int condition, int size_R, const Row* rows, std::vector<int32_t>* a,
                            std::vector<int32_t>* c) {
  olap_ctx* ctx = begin();
  if (!ctx) return -1;
  const size_t n = static_cast<size_t>(size_R);
  void* dr = buf(0, sizeof(Row) * (n ? n : 1));
  int32_t* da = static_cast<int32_t*>(buf(1, sizeof(int32_t) * (n ? n : 1)));
  int32_t* dc = static_cast<int32_t*>(buf(2, sizeof(int32_t) * (n ? n : 1)));
  int64_t* cnt = static_cast<int64_t*>(buf(3, sizeof(int64_t)));
  if (!dr || !da || !dc || !cnt) return -1;
  if (n && olap_copy_h2d(ctx, dr, rows, sizeof(Row) * n) != OLAP_OK) return -1;
  if (!ok(olap_project_pairs_rows(ctx, condition, size_R, dr, sizeof(Row), offsetof(Row, Ra), offsetof(Row, Rc),
                                  da, dc, cnt)))
    return -1;
  const int64_t k = get_i64(cnt);
  return pairs_to_host(k, da, dc, a, c) ? k : -1;
}

inline int64_t project_cols(int condition, int size_R, const int* Ra, const int* Rc, std::vector<int32_t>* a,
                            std::vector<int32_t>* c) {
  olap_ctx* ctx = begin();
  if (!ctx) return -1;
  const size_t n = static_cast<size_t>(size_R);
  int32_t* ra = put(0, Ra, n);
  int32_t* rc = put(1, Rc, n);
  int32_t* da = static_cast<int32_t*>(buf(2, sizeof(int32_t) * (n ? n : 1)));
  int32_t* dc = static_cast<int32_t*>(buf(3, sizeof(int32_t) * (n ? n : 1)));
  int64_t* cnt = static_cast<int64_t*>(buf(4, sizeof(int64_t)));
  if (!ra || !rc || !da || !dc || !cnt) return -1;
  if (!ok(olap_project_pairs(ctx, condition, size_R, ra, rc, da, dc, cnt))) return -1;
  const int64_t k = get_i64(cnt);
  return pairs_to_host(k, da, dc, a, c) ? k : -1;
}

}  // namespace detail

/// proalgo_rowwise over a row store (test_project_option.cpp:34 and :92;
/// rows of struct row_store_min / row_store_max, include/metadata.h:251-262,
/// or any standard-layout row with int fields Ra and Rc): the pairs (Ra, Rc)
/// of the rows with both <= condition, appended to result; returns their count.
template <class Row>
inline int proalgo_rowwise(int condition, const int& size_R, Row* rows, std::vector<std::pair<int, int>>& result) {
  std::lock_guard<std::mutex> lk(detail::state().mu);
  std::vector<int32_t> a, c;
  const int64_t k = detail::project_rows(condition, size_R, rows, &a, &c);
  if (k < 0) return 0;
  for (int64_t i = 0; i < k; ++i) result.emplace_back(a[static_cast<size_t>(i)], c[static_cast<size_t>(i)]);
  return static_cast<int>(k);
}

/// proalgo_rowwise over a row store into fixed arrays (test_project_option.cpp
/// :62 and :120): result.pos_value1[i] = Ra, result.value2[i] = Rc.
template <class Row, class Fixed>
inline int proalgo_rowwise(int condition, const int& size_R, Row* rows, Fixed& result) {
  std::lock_guard<std::mutex> lk(detail::state().mu);
  std::vector<int32_t> a, c;
  const int64_t k = detail::project_rows(condition, size_R, rows, &a, &c);
  if (k < 0) return 0;
  if (k) {
    std::memcpy(result.pos_value1, a.data(), a.size() * sizeof(int32_t));
    std::memcpy(result.value2, c.data(), c.size() * sizeof(int32_t));
  }
  return static_cast<int>(k);
}

/// proalgo_cwm_lm_ifv (test_project_option.cpp:460, late materialisation over
/// the column store): the same pairs, appended to result; pos1 and pos2
/// (the reference's position scratch) are not used.
inline int proalgo_cwm_lm_ifv(int condition, const int& size_R, const int* Ra, const int* Rc, int* pos1, int* pos2,
                              std::vector<std::pair<int, int>>& result) {
  (void)pos1;
  (void)pos2;
  std::lock_guard<std::mutex> lk(detail::state().mu);
  std::vector<int32_t> a, c;
  const int64_t k = detail::project_cols(condition, size_R, Ra, Rc, &a, &c);
  if (k < 0) return 0;
  for (int64_t i = 0; i < k; ++i) result.emplace_back(a[static_cast<size_t>(i)], c[static_cast<size_t>(i)]);
  return static_cast<int>(result.size());
}

/// proalgo_cwm_lm_ifv into fixed arrays (test_project_option.cpp:527): the
/// pairs written from position pre_size on; returns their count.
template <class Fixed>
inline int proalgo_cwm_lm_ifv(int condition, const int& size_R, const int* Ra, const int* Rc, int* pos1, int* pos2,
                              Fixed& result, int pre_size) {
  (void)pos1;
  (void)pos2;
  std::lock_guard<std::mutex> lk(detail::state().mu);
  std::vector<int32_t> a, c;
  const int64_t k = detail::project_cols(condition, size_R, Ra, Rc, &a, &c);
  if (k < 0) return 0;
  if (k) {
    std::memcpy(result.pos_value1 + pre_size, a.data(), a.size() * sizeof(int32_t));
    std::memcpy(result.value2 + pre_size, c.data(), c.size() * sizeof(int32_t));
  }
  return static_cast<int>(k);
}

// ---- group-by (code/group/test_group_option.cpp) -----------------------------

/// vector_group (test_group_option.cpp:44): group_vector[vecInx[i] - 1] +=
/// m1[i] + m2[i] into the caller's int vector (its entries wrap as ints, as
/// the reference's do); returns the sum of the group_num entries afterwards.
inline int64_t vector_group(const size_t& size_R, const int* vecInx, const int* m1, const int* m2, int* group_vector,
                            const int& group_num) {
  std::lock_guard<std::mutex> lk(detail::state().mu);
  olap_ctx* ctx = detail::begin();
  if (!ctx) return 0;
  const size_t g = static_cast<size_t>(group_num);
  int32_t* di = detail::put(0, vecInx, size_R);
  int32_t* d1 = detail::put(1, m1, size_R);
  int32_t* d2 = detail::put(2, m2, size_R);
  int64_t* dg = static_cast<int64_t*>(detail::buf(3, sizeof(int64_t) * (g ? g : 1)));
  int64_t* tot = static_cast<int64_t*>(detail::buf(4, sizeof(int64_t)));
  if (!di || !d1 || !d2 || !dg || !tot) return 0;
  if (!detail::ok(olap_group_vector(ctx, static_cast<int64_t>(size_R), di, d1, d2, group_num, dg, nullptr, tot)))
    return 0;
  std::vector<int64_t> sums(g);
  if (!detail::get(sums.data(), dg, g)) return 0;
  int64_t result = 0;
  for (size_t i = 0; i < g; ++i) {
    group_vector[i] = static_cast<int>(static_cast<uint32_t>(group_vector[i]) + static_cast<uint32_t>(sums[i]));
    result += group_vector[i];
  }
  detail::state().total = result;
  return result;
}

/// hashtable_group (test_group_option.cpp:71): group_hashtable[vecInx[i] - 1]
/// += m1[i] + m2[i] (the groups found on the device, added into the caller's
/// map); returns, as the reference does, the sum of group_hashtable[i] for i
/// in [0, size()).
inline int64_t hashtable_group(const size_t& size_R, const int* vecInx, const int* m1, const int* m2,
                               std::unordered_map<int, int>& group_hashtable) {
  std::lock_guard<std::mutex> lk(detail::state().mu);
  olap_ctx* ctx = detail::begin();
  if (!ctx) return 0;
  int32_t* di = detail::put(0, vecInx, size_R);
  int32_t* d1 = detail::put(1, m1, size_R);
  int32_t* d2 = detail::put(2, m2, size_R);
  if (!di || !d1 || !d2) return 0;
  int64_t cap = olap_group_hash_capacity(static_cast<int64_t>(size_R ? size_R : 1));
  if (cap > (int64_t(1) << 27)) cap = int64_t(1) << 27;
  int32_t* ok = static_cast<int32_t*>(detail::buf(3, sizeof(int32_t) * static_cast<size_t>(cap)));
  int64_t* os = static_cast<int64_t*>(detail::buf(4, sizeof(int64_t) * static_cast<size_t>(cap)));
  int64_t* ng = static_cast<int64_t*>(detail::buf(5, sizeof(int64_t)));
  if (!ok || !os || !ng) return 0;
  if (!detail::ok(olap_group_hash(ctx, static_cast<int64_t>(size_R), di, -1, d1, d2, cap, ok, os, nullptr, ng)))
    return 0;
  const int64_t k = detail::get_i64(ng);
  std::vector<int32_t> keys(static_cast<size_t>(k));
  std::vector<int64_t> sums(static_cast<size_t>(k));
  if (!detail::get(keys.data(), ok, keys.size()) || !detail::get(sums.data(), os, sums.size())) return 0;
  for (size_t i = 0; i < keys.size(); ++i) {
    int& v = group_hashtable[keys[i]];
    v = static_cast<int>(static_cast<uint32_t>(v) + static_cast<uint32_t>(sums[i]));
  }
  int64_t result = 0;
  for (size_t i = 0; i != group_hashtable.size(); ++i) result += group_hashtable[static_cast<int>(i)];
  detail::state().total = result;
  return result;
}

// ---- aggregation (code/aggregation/test_aggregation_option.cpp) -------------

/// aggalgo_rowwise (test_aggregation_option.cpp:28): SUM(price * qty * tax +
/// price * qty) in double, reduced on the device in a fixed order (equal to
/// the reference's sequential sum up to rounding).
inline double aggalgo_rowwise(const int& size_R, const double* l_tax, const double* l_quantity,
                              const double* l_extendedprice) {
  std::lock_guard<std::mutex> lk(detail::state().mu);
  olap_ctx* ctx = detail::begin();
  if (!ctx) return 0.0;
  const size_t n = static_cast<size_t>(size_R);
  double* t = detail::put(0, l_tax, n);
  double* q = detail::put(1, l_quantity, n);
  double* p = detail::put(2, l_extendedprice, n);
  double* sum = static_cast<double*>(detail::buf(3, sizeof(double)));
  if (!t || !q || !p || !sum || !detail::ok(olap_agg_f64(ctx, size_R, t, q, p, sum))) return 0.0;
  double v = 0.0;
  detail::get(&v, sum, 1);
  return v;
}

}  // namespace olap_b200

#ifdef OLAP_B200_DROP_IN
using olap_b200::OLAPcore_rowwise;
using olap_b200::OLAPcore_vwm_dv;
using olap_b200::OLAPcore_vwm_sv;
using olap_b200::join_cwm_sv;
using olap_b200::agg_cwm_sv;
using olap_b200::join_cwm_dv;
using olap_b200::agg_cwm_dv;
using olap_b200::starjoinalgo_rowwise;
using olap_b200::build;
using olap_b200::probe;
using olap_b200::probe_prefetch;
using olap_b200::sel_lt_T_fsel_independent_val_branching;
using olap_b200::sel_lt_T_fsel_independent_val_non_branching;
using olap_b200::selalgo_rowwise;
using olap_b200::proalgo_rowwise;
using olap_b200::proalgo_cwm_lm_ifv;
using olap_b200::vector_group;
using olap_b200::hashtable_group;
using olap_b200::aggalgo_rowwise;
#endif
