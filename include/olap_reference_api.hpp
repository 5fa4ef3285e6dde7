// olap_reference_api.hpp — the reference's OLAP-core C++ signatures over the
// B200 C-ABI (header-only; link with libolapcore_b200.so).
//
// The reference (panjd123/memory_database) defines its OLAP core as free C++
// functions in code/OLAPcore/test_multi_compute_operator.cpp.  This header
// re-exposes the ones that form the hot path with the same names, parameter
// lists (int& sizes, nthreads) and return values, so a caller written against
// the reference builds unchanged against the B200 library:
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
// Define OLAP_B200_DROP_IN before including this header to get the functions
// in the global namespace under the reference's names; otherwise they live in
// namespace olap_b200.
#pragma once

#include <cstdint>
#include <cstring>
#include <mutex>

#include "olap_capi.h"

namespace olap_b200 {

namespace detail {

struct State {
  std::mutex mu;
  olap_ctx* ctx = nullptr;
  int status = OLAP_OK;
  int64_t total = 0;
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

}  // namespace olap_b200

#ifdef OLAP_B200_DROP_IN
using olap_b200::OLAPcore_rowwise;
using olap_b200::OLAPcore_vwm_dv;
using olap_b200::OLAPcore_vwm_sv;
#endif
