// Internal definitions shared by the sm_100a kernels and the C-ABI layer.
//
// Everything here is B200-specific: cache-policy hinted loads (streaming fact
// columns are marked evict-first in L2 and are not allocated in L1, while the
// small, randomly probed dimension vectors are marked evict-last), persistent
// grids sized by the SM count, and a per-context scratch arena so that no
// query allocates device memory on its hot path.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>

#include <mutex>
#include <string>

#include "olap_capi.h"

namespace olap {

// Per-context device scratch words.  Lives in the context's arena, zeroed at
// creation; kernels add to the counters, host calls read-and-clear them.
struct DeviceCounters {
  unsigned long long range_errors;  // rows dropped: fk or group id out of range
  unsigned long long wait_timeouts;  // bounded device waits that gave up
  unsigned long long host_sectors;   // 32-byte host-memory sectors read in place
  unsigned long long oob_seen;       // star-join: nonzero once a key out of range was met (see range pass)
  unsigned long long pad[12];
};

}  // namespace olap

// The opaque context handle of the C-ABI.
struct olap_ctx {
  int device = 0;
  int sm_count = 0;
  int smem_optin = 0;          // max dynamic shared memory per block (bytes)
  int64_t l2_bytes = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;

  // Scratch arena: one cudaMalloc at creation, bump-allocated per call and
  // reset at the start of each call (calls on one context are stream-ordered).
  char* arena = nullptr;
  size_t arena_bytes = 0;
  olap::DeviceCounters* counters = nullptr;  // first bytes of the arena

  // Grow-only device buffer for the large temporaries of synchronous calls
  // (hash group-by tables and partitions); kept between calls.
  char* big = nullptr;
  size_t big_bytes = 0;

  // Pinned host staging used by the host-memory entry points.
  void* pinned = nullptr;
  size_t pinned_bytes = 0;

  // Bytes the host-memory entry points copied to the device (host side;
  // the in-place sectors are counted on the device).
  int64_t host_bytes = 0;

  // Tuning knobs (0 = automatic); set by olap_ctx_set_tuning.
  int64_t tune[OLAP_TUNE_KNOBS] = {0};

  std::mutex mu;               // serialises calls that share this context
  std::string last_error;
};

namespace olap {

// Tuning knob indices (public values in olap_capi.h).
enum {
  TUNE_BLOCK = OLAP_TUNE_BLOCK_THREADS,
  TUNE_BLOCKS_PER_SM = OLAP_TUNE_BLOCKS_PER_SM,
  TUNE_SMEM_DIM_BYTES = OLAP_TUNE_SMEM_DIM_BYTES,
  TUNE_SMEM_ACC_BYTES = OLAP_TUNE_SMEM_ACC_BYTES,
  TUNE_CHUNK_ROWS = OLAP_TUNE_HOST_CHUNK_ROWS,
  TUNE_UNROLL = OLAP_TUNE_UNROLL,
  TUNE_PROBE_BITS = OLAP_TUNE_PROBE_BITS,
  TUNE_SMEM_BITS_BYTES = OLAP_TUNE_SMEM_BITS_BYTES,
  TUNE_GROUP_COMBINE = OLAP_TUNE_GROUP_COMBINE,
  TUNE_GROUP_PLAN = OLAP_TUNE_GROUP_PLAN,
  TUNE_ASYNC_LOADS = OLAP_TUNE_ASYNC_LOADS,
  TUNE_COMPACT = OLAP_TUNE_COMPACT,
  TUNE_SMEM_NIB_BYTES = OLAP_TUNE_SMEM_NIB_BYTES,
  TUNE_HOST_INPLACE = OLAP_TUNE_HOST_INPLACE,
  TUNE_MERGE_PROBES = OLAP_TUNE_MERGE_PROBES,
  TUNE_PROBE_ORDER = OLAP_TUNE_PROBE_ORDER,
  TUNE_JOIN_BUILD = OLAP_TUNE_JOIN_BUILD,
};

int set_error(olap_ctx* ctx, int status, const std::string& msg);
int check_cuda(olap_ctx* ctx, cudaError_t e, const char* what);

#define OLAP_CUDA_TRY(ctx, expr)                         \
  do {                                                   \
    cudaError_t _e = (expr);                             \
    if (_e != cudaSuccess) return olap::check_cuda((ctx), _e, #expr); \
  } while (0)

#define OLAP_REQUIRE(ctx, cond, msg)                     \
  do {                                                   \
    if (!(cond)) return olap::set_error((ctx), OLAP_ERR_INVALID, (msg)); \
  } while (0)


// Bump allocator over the context arena.  Returns nullptr when the arena is
// exhausted (the caller reports OLAP_ERR_CAPACITY).
struct Arena {
  char* base;
  size_t cap;
  size_t off;
  explicit Arena(olap_ctx* c)
      : base(c->arena), cap(c->arena_bytes), off(sizeof(DeviceCounters)) {}
  template <class T>
  T* take(size_t n) {
    size_t a = (off + 255) & ~size_t(255);
    size_t bytes = n * sizeof(T);
    if (a + bytes > cap) return nullptr;
    off = a + bytes;
    return reinterpret_cast<T*>(base + a);
  }
};

// Star-join on device pointers (starjoin.cu): plans, zeroes the outputs unless
// `accumulate`, builds pass bitmaps and launches on `stream`; scratch from `ar`.
int starjoin_device(olap_ctx* ctx, const olap_starjoin_query* q, int64_t* group_sums,
                    int64_t* totals, bool accumulate, cudaStream_t stream, Arena& ar);

// Host-memory star-join helpers (starjoin.cu, hostscan.cu).  stage_host_dims
// copies the query's host dimension vectors into `ar` (a dimvec_len of 0 is
// resolved from the largest key) and points dq at the copies.
int stage_host_dims(olap_ctx* ctx, const olap_starjoin_query* q, Arena& ar, olap_starjoin_query* dq);
// The context's grow-only device buffer, at least `bytes` long (the context's
// stream is synchronised before a smaller buffer is replaced); null when the
// allocation fails.  Used by calls whose scratch grows with their rows.
char* big_scratch(olap_ctx* ctx, size_t bytes);
// In-place scan of pinned host columns (dq: the query with its dimension
// vectors staged in `ar`); *handled is false (and nothing ran) when a column
// is not device-mapped, the columns' 16-byte phases differ, or the
// dimensions' pass fractions promise too little saving over the copies.
int starjoin_host_inplace(olap_ctx* ctx, const olap_starjoin_query* q, const olap_starjoin_query& dq, Arena& ar,
                          int64_t* group_sums, int64_t* totals, bool* handled);

inline int64_t tune_or(const olap_ctx* c, int knob, int64_t dflt) {
  return c->tune[knob] > 0 ? c->tune[knob] : dflt;
}

// ---------------------------------------------------------------------------
// Device helpers
// ---------------------------------------------------------------------------

// L2 cache policies.  Fact columns are read once per query: evict-first keeps
// them from displacing the dimension vectors and group tables, which are
// re-read at random and marked evict-last.
__device__ __forceinline__ uint64_t policy_evict_first() {
  uint64_t p;
  asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint64_t policy_evict_last() {
  uint64_t p;
  asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}

// 128-bit streaming load: read-only path, no L1 allocation, L2 evict-first.
// Asks L2 to fetch the 16-byte aligned part of [p, p + bytes) ahead of the
// loads that will read it (a bulk prefetch has no destination registers).
__device__ __forceinline__ void prefetch_l2_range(const void* p, uint64_t bytes) {
  const uint64_t a = (reinterpret_cast<uint64_t>(p) + 15) & ~uint64_t(15);
  const uint64_t z = (reinterpret_cast<uint64_t>(p) + bytes) & ~uint64_t(15);
  if (z > a) asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a), "r"(static_cast<uint32_t>(z - a)) : "memory");
}

__device__ __forceinline__ int4 ld_stream_v4(const int32_t* p, uint64_t pol) {
  int4 v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.s32 {%0,%1,%2,%3}, [%4], %5;"
      : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
      : "l"(p), "l"(pol));
  return v;
}
// The same load kept in program order with other issue-ordered loads, so a
// batch of them is in flight before the first result is used.
__device__ __forceinline__ int4 ld_stream_v4_ordered(const int32_t* p, uint64_t pol) {
  int4 v;
  asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.s32 {%0,%1,%2,%3}, [%4], %5;"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ int32_t ld_stream_s32(const int32_t* p, uint64_t pol) {
  int32_t v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.s32 %0, [%1], %2;"
      : "=r"(v)
      : "l"(p), "l"(pol));
  return v;
}
// Random probe of a byte vector kept hot in L1/L2 (sign-extended like the
// reference's `int idx_flag = dimvec[...]`).
__device__ __forceinline__ int32_t ld_probe_s8(const int8_t* p, uint64_t pol) {
  int32_t v;
  asm("ld.global.nc.L2::cache_hint.s8 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ int2 ld_probe_i2(const int2* p, uint64_t pol) {
  int2 v;
  asm("ld.global.nc.L2::cache_hint.v2.s32 {%0,%1}, [%2], %3;" : "=r"(v.x), "=r"(v.y) : "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ int32_t ld_probe_s32(const int32_t* p, uint64_t pol) {
  int32_t v;
  asm("ld.global.nc.L2::cache_hint.s32 %0, [%1], %2;" : "=r"(v) : "l"(p), "l"(pol));
  return v;
}

// The loads above are asm statements without `volatile`: the compiler treats
// them as free of side effects and may execute one where its C++ guard does
// not hold (hoisted out of a branch or a conditional expression).  So every
// address given to them must be valid whether or not the guard holds.  Where
// a guard protects an address that may be invalid (a null column, a key out
// of range, a row past the end), the `_if` forms below apply the guard as a
// predicate inside the asm statement: however the statement is moved, the
// load touches memory only when `pred` holds, and returns `dflt` (zeros for
// the vector form) otherwise.
__device__ __forceinline__ int4 ld_stream_v4_if(bool pred, const int32_t* p, uint64_t pol) {
  int4 v;
  asm("{\n\t.reg .pred q;\n\tsetp.ne.u32 q, %4, 0;\n\t"
      "@q ld.global.nc.L1::no_allocate.L2::cache_hint.v4.s32 {%0,%1,%2,%3}, [%5], %6;\n\t"
      "@!q mov.b32 %0, 0;\n\t@!q mov.b32 %1, 0;\n\t@!q mov.b32 %2, 0;\n\t@!q mov.b32 %3, 0;\n\t}"
      : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
      : "r"(static_cast<uint32_t>(pred)), "l"(p), "l"(pol));
  return v;
}
__device__ __forceinline__ int32_t ld_stream_s32_if(bool pred, const int32_t* p, uint64_t pol, int32_t dflt) {
  int32_t v;
  asm("{\n\t.reg .pred q;\n\tsetp.ne.u32 q, %1, 0;\n\t"
      "@q ld.global.nc.L1::no_allocate.L2::cache_hint.s32 %0, [%2], %3;\n\t@!q mov.b32 %0, %4;\n\t}"
      : "=r"(v)
      : "r"(static_cast<uint32_t>(pred)), "l"(p), "l"(pol), "r"(dflt));
  return v;
}
__device__ __forceinline__ int32_t ld_probe_s8_if(bool pred, const int8_t* p, uint64_t pol, int32_t dflt) {
  int32_t v;
  asm("{\n\t.reg .pred q;\n\tsetp.ne.u32 q, %1, 0;\n\t"
      "@q ld.global.nc.L2::cache_hint.s8 %0, [%2], %3;\n\t@!q mov.b32 %0, %4;\n\t}"
      : "=r"(v)
      : "r"(static_cast<uint32_t>(pred)), "l"(p), "l"(pol), "r"(dflt));
  return v;
}

// Exact 64-bit accumulation into shared memory with 32-bit atomics: the low
// word is added atomically and its carry-out is forwarded to the high word.
// Addition mod 2^64 is commutative, so the final pair is exact whatever the
// interleaving.  Non-negative addends below 2^32 (the common case: measures,
// counts) cost a single 32-bit atomic.
__device__ __forceinline__ void smem_add_u64(unsigned long long* slot, uint64_t v) {
  uint32_t* w = reinterpret_cast<uint32_t*>(slot);
  uint32_t lo = static_cast<uint32_t>(v);
  uint32_t hi = static_cast<uint32_t>(v >> 32);
  uint32_t old = atomicAdd(w, lo);
  hi += (old + lo) < old ? 1u : 0u;
  if (hi) atomicAdd(w + 1, hi);
}


// The same accumulation with the words in two arrays: slot i's low word at
// lo[i] and its high word at lo[n + i].  Consecutive slots' low words then
// sit in consecutive banks, so the random low-word atomics of a warp spread
// over all 32 banks instead of the 16 even ones of an array of 64-bit slots.
__device__ __forceinline__ void smem_add_split(uint32_t* lo, int64_t n, int64_t i, uint64_t v) {
  const uint32_t l = static_cast<uint32_t>(v);
  uint32_t h = static_cast<uint32_t>(v >> 32);
  const uint32_t old = atomicAdd(lo + i, l);
  h += (old + l) < old ? 1u : 0u;
  if (h) atomicAdd(lo + n + i, h);
}
__device__ __forceinline__ uint64_t smem_split_get(const uint32_t* lo, int64_t n, int64_t i) {
  return (static_cast<uint64_t>(lo[n + i]) << 32) | lo[i];
}

// ---- bulk asynchronous copies (TMA, untiled) and mbarriers ----------------
// cp.async.bulk global -> shared: both addresses and the size 16-byte
// aligned; completion is counted in bytes on an mbarrier of this CTA.  No
// multicast form is used anywhere in this library.
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(unsigned long long* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}
// Non-blocking test of the phase with parity `parity`.
__device__ __forceinline__ bool mbar_test(unsigned long long* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Generic-proxy accesses of shared memory before later async-proxy ones.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, unsigned long long* bar,
                                              uint64_t pol) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], [%1], %2, [%3], %4;"
      ::"r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(smem_addr(bar)), "l"(pol)
      : "memory");
}

// Value of aggregate OLAP_AGG_* `a` for a row with measures x, y.
__device__ __forceinline__ int64_t agg_value(int a, int32_t x, int32_t y) {
  switch (a) {
    case OLAP_AGG_M1_PLUS_M2: return static_cast<int64_t>(x) + y;
    case OLAP_AGG_M1: return x;
    case OLAP_AGG_M2: return y;
    case OLAP_AGG_M1_TIMES_M2: return static_cast<int64_t>(x) * y;
    default: return 1;
  }
}

__device__ __forceinline__ int64_t warp_sum_i64(int64_t v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

}  // namespace olap
