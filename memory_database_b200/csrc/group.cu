// Group-by and aggregation operators for sm_100a.
//
// Reference: code/group/test_group_option.cpp — vector_group (:44-60) adds
// m1[i] + m2[i] into group_vector[vecInx[i] - 1] (1-based group ids, int
// counters) and returns the int64 sum of the groups; hashtable_group (:71-88)
// does the same through std::unordered_map<int, int> keyed by vecInx[i] - 1.  Here
// sums and counts are int64.  code/aggregation/test_aggregation_option.cpp — aggalgo_*
// (:28-107) sums price*qty*tax + price*qty in double; here the same expression
// in int64 fixed point (tax in hundredths: sum of price*qty*(100 + tax),
// exactly 100x the decimal value) and, for parity with the double code, a
// deterministic double variant.
//
// Dense group-by accumulates per block in shared memory when the group vector
// fits (exact 64-bit sums from 32-bit shared atomics), else in L2 with 64-bit
// atomics.  Hash group-by aggregates in shared-memory tables: per block when
// every distinct key fits one table, else per partition of the key hash
// (see the plans below).
#include <algorithm>
#include <vector>
#include <cstring>

#include "compact.cuh"

namespace olap {

constexpr int kGroupThreads = 512;
constexpr int32_t kEmptyKey = INT32_MIN;

__host__ __device__ __forceinline__ uint32_t mix32(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}

// Dense: group_vector[vecInx[i] - 1] += m1[i] + m2[i]; counts optional.
template <bool SMEM>
__global__ void __launch_bounds__(kGroupThreads) group_vector_kernel(
    int64_t n, const int32_t* __restrict__ idx, const int32_t* __restrict__ m1, const int32_t* __restrict__ m2,
    int64_t G, unsigned long long* __restrict__ sums, unsigned long long* __restrict__ counts,
    unsigned long long* total, unsigned long long* range_err) {
  extern __shared__ unsigned long long sacc[];  // [G] sums, then [G] counts
  const int tid = threadIdx.x;
  const bool want_counts = counts != nullptr;
  if (SMEM) {
    for (int64_t i = tid; i < G * (want_counts ? 2 : 1); i += blockDim.x) sacc[i] = 0;
    __syncthreads();
  }
  const uint64_t pol = policy_evict_first();
  int64_t tot = 0;
  unsigned int bad = 0;
  auto add = [&](int32_t gi, int32_t a, int32_t b) {
    const int64_t g = static_cast<int64_t>(gi) - 1;
    if (g < 0 || g >= G) {
      ++bad;
      return;
    }
    const int64_t v = static_cast<int64_t>(a) + b;
    tot += v;
    if (SMEM) {
      smem_add_u64(&sacc[g], static_cast<uint64_t>(v));
      if (want_counts) atomicAdd(reinterpret_cast<unsigned int*>(&sacc[G + g]), 1u);
    } else {
      atomicAdd(&sums[g], static_cast<unsigned long long>(v));
      if (want_counts) atomicAdd(&counts[g], 1ull);
    }
  };
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  const int64_t t0 = static_cast<int64_t>(blockIdx.x) * blockDim.x + tid;
  const bool vec = ((reinterpret_cast<uintptr_t>(idx) | reinterpret_cast<uintptr_t>(m1) |
                     reinterpret_cast<uintptr_t>(m2)) & 15) == 0;
  const int64_t n4 = vec ? n >> 2 : 0;
  for (int64_t i = t0; i < n4; i += stride) {
    const int4 g = ld_stream_v4(idx + 4 * i, pol), a = ld_stream_v4(m1 + 4 * i, pol), b = ld_stream_v4(m2 + 4 * i, pol);
    add(g.x, a.x, b.x);
    add(g.y, a.y, b.y);
    add(g.z, a.z, b.z);
    add(g.w, a.w, b.w);
  }
  for (int64_t r = 4 * n4 + t0; r < n; r += stride) add(idx[r], m1[r], m2[r]);
  tot = warp_sum_i64(tot);
  const unsigned int wbad = __reduce_add_sync(0xffffffffu, bad);
  if ((tid & 31) == 0) {
    if (tot) atomicAdd(total, static_cast<unsigned long long>(tot));
    if (wbad) atomicAdd(range_err, static_cast<unsigned long long>(wbad));
  }
  if (SMEM) {
    __syncthreads();
    for (int64_t i = tid; i < G; i += blockDim.x) {
      if (sacc[i]) atomicAdd(&sums[i], sacc[i]);
      if (want_counts) {
        const unsigned int c = static_cast<unsigned int>(sacc[G + i]);
        if (c) atomicAdd(&counts[i], static_cast<unsigned long long>(c));
      }
    }
  }
}

// Global hash table of the hash group-by: keys[cap] (kEmptyKey = free),
// sums[cap], counts[cap].
struct HashAgg {
  int32_t* keys;
  unsigned long long* sums;
  unsigned long long* counts;
  uint64_t mask;
  unsigned long long* overflow;
};

__device__ __forceinline__ void global_add(const HashAgg& t, int32_t k, uint64_t s, uint64_t c) {
  uint64_t h = mix32(static_cast<uint32_t>(k)) & t.mask;
  for (uint64_t step = 0; step <= t.mask; ++step) {
    const int32_t prev = atomicCAS(t.keys + h, kEmptyKey, k);
    if (prev == kEmptyKey || prev == k) {
      if (s) atomicAdd(t.sums + h, static_cast<unsigned long long>(s));
      atomicAdd(t.counts + h, static_cast<unsigned long long>(c));
      return;
    }
    h = (h + 1) & t.mask;
  }
  atomicAdd(t.overflow, 1ull);
}

// ---- hash group-by --------------------------------------------------------
//
// Two plans, chosen by the capacity (a power of two >= 2 x the distinct keys):
//  * capacity <= kAggSlots: every block keeps a shared-memory table of at
//    least `capacity` slots, so each distinct key stays in shared memory; blocks
//    flush their tables into the global table once, and the occupied slots
//    are compacted into the outputs.  One read of the columns.
//  * larger: the rows are partitioned by high bits of the key hash into P
//    partitions of at most capacity / (2P) <= kAggSlots / 2 distinct keys (a
//    histogram pass, a scan of the partition offsets, a scatter pass), then
//    one block per partition aggregates it in a kAggSlots-slot shared table
//    and writes its groups straight to the outputs.
// Optionally (OLAP_TUNE_GROUP_COMBINE) a warp first combines its rows that
// share a key (match_any plus two 32-bit reductions of the split values), so
// each distinct key of a warp costs one shared-table update.

constexpr int kAggThreads = 1024;
constexpr int kAggSlots = 8192;  // 16 B per slot: 128 KB of shared memory

struct SmemAgg {
  int32_t* key;
  unsigned int* cnt;
  uint32_t* lo;     // low words of the 64-bit sums; the high words follow at lo + slots
  uint32_t slots;   // a multiple of 4
  uint32_t nb;      // buckets of 4 slots (any count, so a table can fill the shared memory)

  // Home bucket of key k: the low 16 hash bits scaled to [0, nb) (plan 2's
  // partitions take the high bits); probing wraps after the last bucket.
  __device__ __forceinline__ uint32_t home(int32_t k) const {
    return ((mix32(static_cast<uint32_t>(k)) & 0xFFFFu) * nb) >> 16;
  }
  __device__ __forceinline__ uint32_t next(uint32_t b) const { return b + 1 == nb ? 0u : b + 1; }
  __device__ __forceinline__ uint64_t sum(uint32_t i) const { return smem_split_get(lo, slots, i); }
};

__device__ __forceinline__ SmemAgg smem_agg(unsigned char* base, uint32_t slots) {
  SmemAgg t;
  t.lo = reinterpret_cast<uint32_t*>(base);
  t.key = reinterpret_cast<int32_t*>(t.lo + 2 * slots);
  t.cnt = reinterpret_cast<unsigned int*>(t.key + slots);
  t.slots = slots;
  t.nb = slots >> 2;
  return t;
}

__device__ __forceinline__ void smem_agg_clear(const SmemAgg& t) {
  for (uint32_t i = threadIdx.x; i < t.slots; i += blockDim.x) {
    t.key[i] = kEmptyKey;
    t.cnt[i] = 0;
    t.lo[i] = 0;
    t.lo[t.slots + i] = 0;
  }
}

__device__ __forceinline__ int4 lds_volatile_v4(const int32_t* p) {
  int4 v;
  const unsigned a = static_cast<unsigned>(__cvta_generic_to_shared(p));
  asm volatile("ld.volatile.shared.v4.s32 {%0,%1,%2,%3}, [%4];" : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "r"(a));
  return v;
}

// Adds (s, c) to key k's slot; false when the table has no room for k.
// Buckets of 4 slots, probed linearly: one 16-byte read finds k or the first
// free slot of a bucket, which keeps the probe loops of a warp short at low
// load.  Keys are never removed, so a key lives in the first bucket that had
// a free slot when it was inserted, and a thread that loses a slot's CAS to
// the same key uses that slot.  Returns k's slot from the bucket run starting
// at b, inserting k when absent (volatile reads: other threads insert
// concurrently); -1 when the table has no room for k.
__device__ __forceinline__ int smem_find_insert(const SmemAgg& t, int32_t k, uint32_t b) {
  for (uint32_t step = 0; step < t.nb; ++step) {
    const int4 q = lds_volatile_v4(t.key + 4 * b);
    int slot = q.x == k ? 0 : q.y == k ? 1 : q.z == k ? 2 : q.w == k ? 3 : -1;
    if (slot < 0 && (q.x == kEmptyKey || q.y == kEmptyKey || q.z == kEmptyKey || q.w == kEmptyKey)) {
      // k is new to this bucket and it has room: claim the first free slot
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int32_t cur = j == 0 ? q.x : j == 1 ? q.y : j == 2 ? q.z : q.w;
        if (slot < 0 && cur == kEmptyKey) {
          const int32_t prev = atomicCAS(t.key + 4 * b + j, kEmptyKey, k);
          if (prev == kEmptyKey || prev == k) slot = j;
        }
      }
    }
    if (slot >= 0) return static_cast<int>(4 * b) + slot;
    b = t.next(b);
  }
  return -1;
}

// Adds (s, c) to key k's slot; false when the table has no room for k.
__device__ __forceinline__ bool smem_agg_add(const SmemAgg& t, int32_t k, uint64_t s, uint32_t c) {
  const int i = smem_find_insert(t, k, t.home(k));
  if (i < 0) return false;
  smem_add_split(t.lo, t.slots, i, s);
  atomicAdd(t.cnt + i, c);
  return true;
}

// Warp combine of the rows that share a key: returns true on the lane that
// carries its key's (sum, count) for this warp step.  v lies in [-2^32, 2^32):
// v + 2^32 splits into 24 low and 9 high bits, whose 32-bit sums over at most
// 32 lanes cannot overflow.
__device__ __forceinline__ bool warp_combine(bool valid, int32_t k, int64_t v, int64_t* gs, uint32_t* gc) {
  const int lane = threadIdx.x & 31;
  const unsigned long long tag = valid ? static_cast<unsigned long long>(static_cast<uint32_t>(k))
                                       : (0x100000000ull | static_cast<unsigned long long>(lane));
  const unsigned int m = __match_any_sync(0xffffffffu, tag);
  if (__all_sync(0xffffffffu, (m & (m - 1)) == 0)) {  // no key repeats in this warp step
    *gs = v;
    *gc = 1;
    return valid;
  }
  if (!valid) return false;
  const uint64_t u = static_cast<uint64_t>(v + (int64_t(1) << 32));
  const uint32_t lo = __reduce_add_sync(m, static_cast<uint32_t>(u & 0xffffffu));
  const uint32_t hi = __reduce_add_sync(m, static_cast<uint32_t>(u >> 24));
  const uint32_t c = __popc(m);
  *gs = (static_cast<int64_t>(hi) << 24) + static_cast<int64_t>(lo) - (static_cast<int64_t>(c) << 32);
  *gc = c;
  return lane == __ffs(m) - 1;
}

__device__ __forceinline__ int32_t agg_key(int32_t key, int32_t key_offset) {
  return static_cast<int32_t>(static_cast<uint32_t>(key) + static_cast<uint32_t>(key_offset));
}

// Rows [b, e) of the columns, 4 per thread per step (16-byte loads when
// aligned), handed to f(valid, row, key, value) by every lane of the warp.
template <class F>
__device__ __forceinline__ void agg_rows(int64_t b, int64_t e, int64_t t0, int64_t stride, const int32_t* keys,
                                         const int32_t* vals, const int32_t* vals2, bool vec, F&& f) {
  const uint64_t pol = policy_evict_first();
  const int32_t* v2 = vals2 ? vals2 : vals;  // a valid address even where the guarded load is hoisted
  const int64_t b4 = vec ? (b + 3) & ~int64_t(3) : e;  // first aligned row
  const int64_t head = b4 < e ? b4 : e;
  // head rows one by one (at most 3), then groups of 4, then the tail
  for (int64_t base = b; base < head; base += stride) {
    const int64_t r = base + t0;
    const bool ok = r < head;
    f(ok, ok ? keys[r] : 0, ok ? static_cast<int64_t>(vals[r]) + (vals2 ? vals2[r] : 0) : 0);
  }
  const int64_t n4 = (e - head) >> 2;
  for (int64_t base = 0; base < n4; base += 2 * stride) {
    // two groups of 4 rows per thread in flight before either is used
    int4 k[2], v[2], w[2];
    bool ok[2];
#pragma unroll
    for (int g = 0; g < 2; ++g) {
      const int64_t i = base + g * stride + t0;
      ok[g] = i < n4;
      k[g] = make_int4(0, 0, 0, 0);
      v[g] = k[g];
      w[g] = k[g];
      if (ok[g]) {
        k[g] = ld_stream_v4(keys + head + 4 * i, pol);
        v[g] = ld_stream_v4(vals + head + 4 * i, pol);
        if (vals2) w[g] = ld_stream_v4(v2 + head + 4 * i, pol);
      }
    }
#pragma unroll
    for (int g = 0; g < 2; ++g) {
      f(ok[g], k[g].x, static_cast<int64_t>(v[g].x) + w[g].x);
      f(ok[g], k[g].y, static_cast<int64_t>(v[g].y) + w[g].y);
      f(ok[g], k[g].z, static_cast<int64_t>(v[g].z) + w[g].z);
      f(ok[g], k[g].w, static_cast<int64_t>(v[g].w) + w[g].w);
    }
  }
  for (int64_t base = head + 4 * n4; base < e; base += stride) {
    const int64_t r = base + t0;
    const bool ok = r < e;
    f(ok, ok ? keys[r] : 0, ok ? static_cast<int64_t>(vals[r]) + (vals2 ? vals2[r] : 0) : 0);
  }
}

// Plan 1: shared tables of `slots` = capacity slots per block, flushed into
// the global table.
__global__ void __launch_bounds__(kAggThreads) group_hash_smem_kernel(int64_t n, const int32_t* __restrict__ keys,
                                                                      int32_t key_offset,
                                                                      const int32_t* __restrict__ vals,
                                                                      const int32_t* __restrict__ vals2,
                                                                      uint32_t slots, int combine, HashAgg t,
                                                                      unsigned long long* range_err) {
  extern __shared__ __align__(16) unsigned char agg_smem[];
  const SmemAgg st = smem_agg(agg_smem, slots);
  smem_agg_clear(st);
  __syncthreads();
  const bool vec = ((reinterpret_cast<uintptr_t>(keys) | reinterpret_cast<uintptr_t>(vals) |
                     reinterpret_cast<uintptr_t>(vals2)) & 15) == 0;
  // each block takes a contiguous share of the rows
  const int64_t per = ((n + gridDim.x - 1) / gridDim.x + 3) & ~int64_t(3);
  const int64_t b = static_cast<int64_t>(blockIdx.x) * per;
  const int64_t e = b + per < n ? b + per : n;
  unsigned int bad = 0;
  if (b < e)
    agg_rows(b, e, threadIdx.x, blockDim.x, keys, vals, vals2, vec, [&](bool ok, int32_t key, int64_t v) {
      const int32_t k = agg_key(key, key_offset);
      if (ok && k == kEmptyKey) {  // reserved as the empty marker
        ++bad;
        ok = false;
      }
      int64_t gs = v;
      uint32_t gc = 1;
      if (combine ? warp_combine(ok, k, v, &gs, &gc) : ok)
        if (!smem_agg_add(st, k, static_cast<uint64_t>(gs), gc)) global_add(t, k, static_cast<uint64_t>(gs), gc);
    });
  const unsigned int wbad = __reduce_add_sync(0xffffffffu, bad);
  if ((threadIdx.x & 31) == 0 && wbad) atomicAdd(range_err, static_cast<unsigned long long>(wbad));
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < slots; i += blockDim.x)
    if (st.key[i] != kEmptyKey) global_add(t, st.key[i], st.sum(i), st.cnt[i]);
}

// ---- batched shared-table updates -------------------------------------------
// R rows (count 1 each) into the shared table, with every step of the R rows
// issued together: the R home buckets are read first (plain loads: a stale
// read can only miss a key, since keys are never removed, and a miss takes
// the volatile insert path), then the R low-word adds whose old values give
// the carries, the R count adds, and the high words where a carry or a
// negative value needs one.  Only 32-bit shared atomics: on B200 a 64-bit
// shared atomicAdd runs several times slower than a 32-bit one.  `sync`: the
// lanes of the warp that call together (0 when the callers are not
// warp-uniform); they are brought back together after the insert path, whose
// probe loop ends at a different step on each lane (left diverged, the warp
// would run all later steps once per lane group).  Returns the mask of the
// rows that found no room (the caller adds them elsewhere).
template <int R>
__device__ __forceinline__ uint32_t smem_agg_rows(const SmemAgg& t, const int32_t (&k)[R], const int64_t (&v)[R],
                                                  uint32_t valid, uint32_t sync) {
  uint32_t b[R];
  int4 q[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    b[r] = t.home(k[r]);
    q[r] = ((valid >> r) & 1u) ? *reinterpret_cast<const int4*>(t.key + 4 * b[r]) : make_int4(0, 0, 0, 0);
  }
  int s[R];
  uint32_t lost = 0;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int j = q[r].x == k[r] ? 0 : q[r].y == k[r] ? 1 : q[r].z == k[r] ? 2 : q[r].w == k[r] ? 3 : -1;
    s[r] = ((valid >> r) & 1u) && j >= 0 ? static_cast<int>(4 * b[r]) + j : -1;
  }
#pragma unroll
  for (int r = 0; r < R; ++r) {
    if (((valid >> r) & 1u) && s[r] < 0) {
      s[r] = smem_find_insert(t, k[r], b[r]);
      if (s[r] < 0) lost |= 1u << r;
    }
  }
  if (sync) __syncwarp(sync);
  uint32_t old[R];
#pragma unroll
  for (int r = 0; r < R; ++r)
    old[r] = s[r] >= 0 ? atomicAdd(t.lo + s[r], static_cast<uint32_t>(v[r])) : 0u;
#pragma unroll
  for (int r = 0; r < R; ++r)
    if (s[r] >= 0) atomicAdd(t.cnt + s[r], 1u);
#pragma unroll
  for (int r = 0; r < R; ++r) {
    if (s[r] < 0) continue;
    const uint32_t lo = static_cast<uint32_t>(v[r]);
    const uint32_t hi = static_cast<uint32_t>(static_cast<uint64_t>(v[r]) >> 32) + ((old[r] + lo) < old[r] ? 1u : 0u);
    if (hi) atomicAdd(t.lo + t.slots + s[r], hi);
  }
  return lost;
}

constexpr int kRowsThreads = 1024;

// Plan 1 with batched updates: each block aggregates a contiguous share of
// the rows in a `slots`-slot shared table, 4 rows per thread step with the
// next step's columns already loading (software pipelined), then adds its
// slots to the global table; a row whose key finds no room goes to the
// global table directly.
template <bool HAS2>
__global__ void __launch_bounds__(kRowsThreads) group_hash_rows_kernel(int64_t n, const int32_t* __restrict__ keys,
                                                                       int32_t key_offset,
                                                                       const int32_t* __restrict__ vals,
                                                                       const int32_t* __restrict__ vals2,
                                                                       uint32_t slots, HashAgg g,
                                                                       unsigned long long* range_err) {
  extern __shared__ __align__(16) unsigned char agg_smem[];
  const SmemAgg t = smem_agg(agg_smem, slots);
  smem_agg_clear(t);
  __syncthreads();
  const bool vec = ((reinterpret_cast<uintptr_t>(keys) | reinterpret_cast<uintptr_t>(vals) |
                     (HAS2 ? reinterpret_cast<uintptr_t>(vals2) : 0)) & 15) == 0;
  const int64_t per = ((n + gridDim.x - 1) / gridDim.x + 3) & ~int64_t(3);
  const int64_t b = static_cast<int64_t>(blockIdx.x) * per;
  const int64_t e = b + per < n ? b + per : n;
  const uint64_t pol = policy_evict_first();
  unsigned int bad = 0;
  auto rows = [&](const int4 kk, const int4 a, const int4 c, uint32_t valid, uint32_t sync) {
    const int32_t kr[4] = {kk.x, kk.y, kk.z, kk.w}, ar[4] = {a.x, a.y, a.z, a.w}, cr[4] = {c.x, c.y, c.z, c.w};
    int32_t k[4];
    int64_t v[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      k[u] = agg_key(kr[u], key_offset);
      v[u] = static_cast<int64_t>(ar[u]) + (HAS2 ? cr[u] : 0);
      if (((valid >> u) & 1u) && k[u] == kEmptyKey) {  // reserved as the empty marker
        ++bad;
        valid &= ~(1u << u);
      }
    }
    const uint32_t lost = smem_agg_rows<4>(t, k, v, valid, sync);
    if (lost) {  // rare: keys that found no room in the table
#pragma unroll
      for (int u = 0; u < 4; ++u)
        if ((lost >> u) & 1u) global_add(g, k[u], static_cast<uint64_t>(v[u]), 1);
    }
  };
  auto one = [&](int64_t r) {
    rows(make_int4(keys[r], 0, 0, 0), make_int4(vals[r], 0, 0, 0), make_int4(HAS2 ? vals2[r] : 0, 0, 0, 0), 1u, 0u);
  };
  if (b < e) {
    const int64_t b4 = (b + 3) & ~int64_t(3);
    const int64_t head = vec ? (b4 < e ? b4 : e) : e;
    const int64_t n4 = (e - head) >> 2;
    // rows before the first aligned one, and all rows when unaligned: one at a time
    for (int64_t r = b + threadIdx.x; r < head; r += blockDim.x) one(r);
    const int32_t* kp = keys + head;
    const int32_t* ap = vals + head;
    const int32_t* cp = HAS2 ? vals2 + head : vals + head;
    // Every lane of a warp runs the same steps (a lane past the end has no
    // rows in its last one), so the table updates can bring the warp back
    // together.
    const int64_t lane = threadIdx.x & 31;
    const int64_t w0 = static_cast<int64_t>(threadIdx.x) - lane;
    int4 kk = make_int4(0, 0, 0, 0), a = kk, c = kk;
    if (w0 + lane < n4) {
      kk = ld_stream_v4(kp + 4 * (w0 + lane), pol);
      a = ld_stream_v4(ap + 4 * (w0 + lane), pol);
      if (HAS2) c = ld_stream_v4(cp + 4 * (w0 + lane), pol);
    }
    for (int64_t i0 = w0; i0 < n4; i0 += blockDim.x) {
      // the next step's columns load while this step's rows update the table
      const int64_t i = i0 + lane, nx = i + blockDim.x;
      int4 kn = make_int4(0, 0, 0, 0), an = kn, cn = kn;
      if (nx < n4) {
        kn = ld_stream_v4(kp + 4 * nx, pol);
        an = ld_stream_v4(ap + 4 * nx, pol);
        if (HAS2) cn = ld_stream_v4(cp + 4 * nx, pol);
      }
      rows(kk, a, c, i < n4 ? 0xFu : 0u, 0xffffffffu);
      kk = kn;
      a = an;
      c = cn;
    }
    for (int64_t r = head + 4 * n4 + threadIdx.x; r < e; r += blockDim.x) one(r);
  }
  const unsigned int wbad = __reduce_add_sync(0xffffffffu, bad);
  if ((threadIdx.x & 31) == 0 && wbad) atomicAdd(range_err, static_cast<unsigned long long>(wbad));
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < slots; i += blockDim.x)
    if (t.key[i] != kEmptyKey && t.cnt[i]) global_add(g, t.key[i], t.sum(i), t.cnt[i]);
}

// Plan 2.  Partition of a key: the top bits of its hash (the shared tables
// index with the low bits).
__device__ __forceinline__ uint32_t agg_part(int32_t k, int part_shift) {
  return part_shift >= 32 ? 0u : mix32(static_cast<uint32_t>(k)) >> part_shift;
}

struct PartPlan {
  int64_t n;
  int64_t per;        // rows per block of the histogram and scatter passes (multiple of 4)
  int32_t n_blocks;   // blocks of those passes
  int32_t n_parts;    // P (power of two)
  int32_t part_shift; // 32 - log2(P)
  int32_t key_offset;
};

// Per block and partition: rows of the block's share in the partition,
// hist[b * P + p]; the partition totals are summed into ptot[p].
__global__ void __launch_bounds__(1024) group_part_hist_kernel(PartPlan pp, const int32_t* __restrict__ keys,
                                                               unsigned int* __restrict__ hist,
                                                               unsigned long long* __restrict__ ptot,
                                                               unsigned long long* range_err) {
  extern __shared__ unsigned int s_hist[];
  for (int p = threadIdx.x; p < pp.n_parts; p += blockDim.x) s_hist[p] = 0;
  __syncthreads();
  const int64_t b = static_cast<int64_t>(blockIdx.x) * pp.per;
  const int64_t e = b + pp.per < pp.n ? b + pp.per : pp.n;
  const uint64_t pol = policy_evict_first();
  const bool vec = (reinterpret_cast<uintptr_t>(keys) & 15) == 0;
  unsigned int bad = 0;
  auto one = [&](int32_t key) {
    const int32_t k = agg_key(key, pp.key_offset);
    if (k == kEmptyKey) {
      ++bad;
      return;
    }
    atomicAdd(&s_hist[agg_part(k, pp.part_shift)], 1u);
  };
  if (vec) {
    for (int64_t r = b + 4 * threadIdx.x; r < e; r += 4 * blockDim.x) {
      if (r + 4 <= e) {
        const int4 k = ld_stream_v4(keys + r, pol);
        one(k.x); one(k.y); one(k.z); one(k.w);
      } else {
        for (int64_t q = r; q < e; ++q) one(keys[q]);
      }
    }
  } else {
    for (int64_t r = b + threadIdx.x; r < e; r += blockDim.x) one(keys[r]);
  }
  const unsigned int wbad = __reduce_add_sync(0xffffffffu, bad);
  if ((threadIdx.x & 31) == 0 && wbad) atomicAdd(range_err, static_cast<unsigned long long>(wbad));
  __syncthreads();
  for (int p = threadIdx.x; p < pp.n_parts; p += blockDim.x) {
    const unsigned int c = s_hist[p];
    hist[static_cast<int64_t>(blockIdx.x) * pp.n_parts + p] = c;
    if (c) atomicAdd(&ptot[p], static_cast<unsigned long long>(c));
  }
}

// Partition starts: part_begin[p] = rows of the partitions before p
// (part_begin[P] = all rows); cursor[p] starts at part_begin[p].  One block.
__global__ void __launch_bounds__(1024) group_part_scan_kernel(PartPlan pp, const unsigned long long* __restrict__ ptot,
                                                               long long* __restrict__ part_begin,
                                                               unsigned long long* __restrict__ cursor) {
  __shared__ long long s_run[1024];
  const int per = (pp.n_parts + blockDim.x - 1) / blockDim.x;
  const int b = threadIdx.x * per;
  const int e = b + per < pp.n_parts ? b + per : pp.n_parts;
  long long s = 0;
  for (int i = b; i < e; ++i) s += static_cast<long long>(ptot[i]);
  s_run[threadIdx.x] = s;
  __syncthreads();
  for (int o = 1; o < 1024; o <<= 1) {
    const long long y = threadIdx.x >= o ? s_run[threadIdx.x - o] : 0;
    __syncthreads();
    s_run[threadIdx.x] += y;
    __syncthreads();
  }
  long long run = s_run[threadIdx.x] - s;
  for (int i = b; i < e; ++i) {
    part_begin[i] = run;
    cursor[i] = static_cast<unsigned long long>(run);
    run += static_cast<long long>(ptot[i]);
  }
  if (threadIdx.x == blockDim.x - 1) part_begin[pp.n_parts] = s_run[threadIdx.x];
}

// A partitioned row: {key, value} (8 bytes) or, with a second value
// column, {key, pad, value as int64} (16 bytes): one store per row.
template <bool HAS2>
struct PartRow;
template <>
struct PartRow<false> {
  using T = int2;
  __device__ static T make(int32_t k, int32_t a, int32_t) { return make_int2(k, a); }
  __device__ static int32_t key(const T& r) { return r.x; }
  __device__ static int64_t val(const T& r) { return r.y; }
};
template <>
struct PartRow<true> {
  using T = longlong2;
  __device__ static T make(int32_t k, int32_t a, int32_t c) {
    return make_longlong2(static_cast<long long>(static_cast<uint32_t>(k)), static_cast<long long>(a) + c);
  }
  __device__ static int32_t key(const T& r) { return static_cast<int32_t>(static_cast<uint32_t>(r.x)); }
  __device__ static int64_t val(const T& r) { return r.y; }
};

template <bool HAS2>
__global__ void __launch_bounds__(1024) group_part_scatter_kernel(PartPlan pp, const int32_t* __restrict__ keys,
                                                                  const int32_t* __restrict__ vals,
                                                                  const int32_t* __restrict__ vals2,
                                                                  const unsigned int* __restrict__ hist,
                                                                  unsigned long long* __restrict__ cursor,
                                                                  typename PartRow<HAS2>::T* __restrict__ rows) {
  extern __shared__ unsigned int s_cur[];
  // this block's run in each partition (order inside a partition is free)
  for (int p = threadIdx.x; p < pp.n_parts; p += blockDim.x) {
    const unsigned int c = hist[static_cast<int64_t>(blockIdx.x) * pp.n_parts + p];
    s_cur[p] = c ? static_cast<unsigned int>(atomicAdd(&cursor[p], static_cast<unsigned long long>(c))) : 0u;
  }
  __syncthreads();
  const int64_t b = static_cast<int64_t>(blockIdx.x) * pp.per;
  const int64_t e = b + pp.per < pp.n ? b + pp.per : pp.n;
  const uint64_t pol = policy_evict_first();
  const bool vec = ((reinterpret_cast<uintptr_t>(keys) | reinterpret_cast<uintptr_t>(vals) |
                     reinterpret_cast<uintptr_t>(vals2)) & 15) == 0;
  auto one = [&](int32_t key, int32_t a, int32_t c) {
    const int32_t k = agg_key(key, pp.key_offset);
    if (k == kEmptyKey) return;
    const unsigned int pos = atomicAdd(&s_cur[agg_part(k, pp.part_shift)], 1u);
    rows[pos] = PartRow<HAS2>::make(k, a, c);
  };
  if (vec) {
    for (int64_t r = b + 4 * threadIdx.x; r < e; r += 4 * blockDim.x) {
      if (r + 4 <= e) {
        const int4 kk = ld_stream_v4(keys + r, pol), a = ld_stream_v4(vals + r, pol);
        const int4 c = HAS2 ? ld_stream_v4(vals2 + r, pol) : make_int4(0, 0, 0, 0);
        // the four cursor updates are independent: issue them together
        const int32_t k[4] = {agg_key(kk.x, pp.key_offset), agg_key(kk.y, pp.key_offset),
                              agg_key(kk.z, pp.key_offset), agg_key(kk.w, pp.key_offset)};
        unsigned int pos[4];
#pragma unroll
        for (int u = 0; u < 4; ++u)
          pos[u] = k[u] != kEmptyKey ? atomicAdd(&s_cur[agg_part(k[u], pp.part_shift)], 1u) : 0u;
        const int32_t av[4] = {a.x, a.y, a.z, a.w}, cv[4] = {c.x, c.y, c.z, c.w};
#pragma unroll
        for (int u = 0; u < 4; ++u)
          if (k[u] != kEmptyKey) rows[pos[u]] = PartRow<HAS2>::make(k[u], av[u], cv[u]);
      } else {
        for (int64_t q = r; q < e; ++q) one(keys[q], vals[q], HAS2 ? vals2[q] : 0);
      }
    }
  } else {
    for (int64_t r = b + threadIdx.x; r < e; r += blockDim.x) one(keys[r], vals[r], HAS2 ? vals2[r] : 0);
  }
}

// The same scatter with coalesced writes (P <= kTiledParts): each tile of
// kScatterTile rows (8 per thread) is counting-sorted by partition in shared
// memory, then written out so that consecutive threads write consecutive
// rows of a partition's run.  A row's partition is hashed once and kept
// beside it in the sorted tile, and each partition's destination base is
// worked out once per tile, so the write-out looks up one word per row.
// Shared memory: the sorted rows and their partitions, then per partition
// the tile count, the tile offset, the block's cursor and the destination
// base.  The next tile's columns are prefetched into L2 while the current
// one is sorted and written.  (4,096-row tiles of 4 rows per thread with the
// partition hashed three times took 4.2 warp-instructions per row; now 2.8.)
constexpr int kScatterTile = 8192;
constexpr int kMaxPartials = 256;  // partial tables of split partitions (128 KB each)
constexpr int kTiledParts = 4096;

template <bool HAS2>
__global__ void __launch_bounds__(1024, 1) group_part_scatter_tiled_kernel(
    PartPlan pp, const int32_t* __restrict__ keys, const int32_t* __restrict__ vals,
    const int32_t* __restrict__ vals2, const unsigned int* __restrict__ hist, unsigned long long* __restrict__ cursor,
    typename PartRow<HAS2>::T* __restrict__ rows) {
  using Row = typename PartRow<HAS2>::T;
  extern __shared__ __align__(16) unsigned char sc_smem[];
  Row* s_rows = reinterpret_cast<Row*>(sc_smem);
  uint16_t* s_part = reinterpret_cast<uint16_t*>(s_rows + kScatterTile);
  unsigned int* s_cnt = reinterpret_cast<unsigned int*>(s_part + kScatterTile);
  unsigned int* s_off = s_cnt + pp.n_parts;
  unsigned int* s_cur = s_off + pp.n_parts;
  unsigned int* s_dst = s_cur + pp.n_parts;
  __shared__ unsigned int s_warp[32];
  const int P = pp.n_parts;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int p = tid; p < P; p += blockDim.x) {
    const unsigned int c = hist[static_cast<int64_t>(blockIdx.x) * P + p];
    s_cur[p] = c ? static_cast<unsigned int>(atomicAdd(&cursor[p], static_cast<unsigned long long>(c))) : 0u;
    s_cnt[p] = 0;
  }
  const int64_t b = static_cast<int64_t>(blockIdx.x) * pp.per;
  const int64_t e = b + pp.per < pp.n ? b + pp.per : pp.n;
  const uint64_t pol = policy_evict_first();
  const bool vec = ((reinterpret_cast<uintptr_t>(keys) | reinterpret_cast<uintptr_t>(vals) |
                     reinterpret_cast<uintptr_t>(vals2)) & 15) == 0;
  const int per_thread = (P + blockDim.x - 1) / blockDim.x;  // partitions per thread in the scan
  auto prefetch_tile = [&](int64_t t0) {  // the tile's columns into L2, ahead of its loads
    if (tid != 0 || t0 >= e) return;
    const int64_t m = e - t0 < kScatterTile ? e - t0 : kScatterTile;
    prefetch_l2_range(keys + t0, 4 * m);
    prefetch_l2_range(vals + t0, 4 * m);
    if (HAS2) prefetch_l2_range(vals2 + t0, 4 * m);
  };
  prefetch_tile(b);
  __syncthreads();
  for (int64_t t0 = b; t0 < e; t0 += kScatterTile) {
    prefetch_tile(t0 + kScatterTile);
    // 1. this thread's 8 rows (4 at t0 + 4 tid, 4 at t0 + 4 (tid + 1024)):
    //    key, partition and rank inside the tile
    int32_t k[8], a[8], c[8];
    uint32_t slot[8];  // partition << 13 | rank, or ~0u for no row
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int64_t r0 = t0 + 4 * (tid + h * static_cast<int64_t>(blockDim.x));
      if (vec && r0 + 4 <= e) {
        const int4 kk = ld_stream_v4(keys + r0, pol), av = ld_stream_v4(vals + r0, pol);
        const int4 cv = HAS2 ? ld_stream_v4(vals2 + r0, pol) : make_int4(0, 0, 0, 0);
        k[4 * h] = kk.x; k[4 * h + 1] = kk.y; k[4 * h + 2] = kk.z; k[4 * h + 3] = kk.w;
        a[4 * h] = av.x; a[4 * h + 1] = av.y; a[4 * h + 2] = av.z; a[4 * h + 3] = av.w;
        c[4 * h] = cv.x; c[4 * h + 1] = cv.y; c[4 * h + 2] = cv.z; c[4 * h + 3] = cv.w;
      } else {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const bool ok = r0 + u < e;
          k[4 * h + u] = ok ? keys[r0 + u] : kEmptyKey;
          a[4 * h + u] = ok ? vals[r0 + u] : 0;
          c[4 * h + u] = ok && HAS2 ? vals2[r0 + u] : 0;
        }
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int q = 4 * h + u;
        slot[q] = ~0u;
        if (r0 + u < e) {
          k[q] = agg_key(k[q], pp.key_offset);
          if (k[q] != kEmptyKey) {
            const uint32_t part = agg_part(k[q], pp.part_shift);
            slot[q] = (part << 13) | atomicAdd(&s_cnt[part], 1u);
          }
        }
      }
    }
    __syncthreads();
    // 2. exclusive scan of the tile counts (each thread a run of partitions);
    //    destination bases, and the block's cursors moved past the tile
    unsigned int run = 0;
    for (int j = 0; j < per_thread; ++j) {
      const int p = tid * per_thread + j;
      if (p < P) run += s_cnt[p];
    }
    unsigned int inc = run;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned int y = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += y;
    }
    if (lane == 31) s_warp[warp] = inc;
    __syncthreads();
    if (warp == 0) {
      unsigned int w = lane < static_cast<int>(blockDim.x >> 5) ? s_warp[lane] : 0u;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned int y = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += y;
      }
      s_warp[lane] = w;  // inclusive over warps
    }
    __syncthreads();
    unsigned int off = (warp > 0 ? s_warp[warp - 1] : 0u) + inc - run;
    const unsigned int n_valid = s_warp[(blockDim.x >> 5) - 1];
    for (int j = 0; j < per_thread; ++j) {
      const int p = tid * per_thread + j;
      if (p < P) {
        const unsigned int cnt = s_cnt[p];
        s_off[p] = off;
        s_dst[p] = s_cur[p] - off;
        s_cur[p] += cnt;
        s_cnt[p] = 0;
        off += cnt;
      }
    }
    __syncthreads();
    // 3. rows into their sorted places
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      if (slot[q] == ~0u) continue;
      const unsigned int at = s_off[slot[q] >> 13] + (slot[q] & 8191u);
      s_rows[at] = PartRow<HAS2>::make(k[q], a[q], c[q]);
      s_part[at] = static_cast<uint16_t>(slot[q] >> 13);
    }
    __syncthreads();
    // 4. coalesced writes: sorted row i goes to its partition's run
    for (unsigned int i = tid; i < n_valid; i += blockDim.x) rows[s_dst[s_part[i]] + i] = s_rows[i];
    __syncthreads();
  }
}

// Appends the occupied slots of a block's shared table to the outputs
// (positions from one global counter per block).  Every thread of the block
// calls it (it synchronises the block).
__device__ __forceinline__ void append_groups(const SmemAgg& st, int64_t capacity, int32_t* __restrict__ out_keys,
                                              int64_t* __restrict__ out_sums, int64_t* __restrict__ out_counts,
                                              unsigned long long* d_groups, unsigned long long* overflow) {
  __shared__ unsigned int s_n;
  __shared__ unsigned long long s_base;
  if (threadIdx.x == 0) s_n = 0;
  __syncthreads();
  constexpr int kPer = kAggSlots / kAggThreads;
  unsigned int pos[kPer];
#pragma unroll
  for (int j = 0; j < kPer; ++j) {
    const int i = j * kAggThreads + threadIdx.x;
    pos[j] = st.key[i] != kEmptyKey ? atomicAdd(&s_n, 1u) : ~0u;
  }
  __syncthreads();
  if (threadIdx.x == 0) s_base = s_n ? atomicAdd(d_groups, static_cast<unsigned long long>(s_n)) : 0ull;
  __syncthreads();
#pragma unroll
  for (int j = 0; j < kPer; ++j) {
    if (pos[j] == ~0u) continue;
    const int i = j * kAggThreads + threadIdx.x;
    const unsigned long long o = s_base + pos[j];
    if (o >= static_cast<unsigned long long>(capacity)) {  // more groups than the outputs hold
      atomicAdd(overflow, 1ull);
      continue;
    }
    out_keys[o] = st.key[i];
    out_sums[o] = static_cast<int64_t>(st.sum(i));
    if (out_counts) out_counts[o] = static_cast<int64_t>(st.cnt[i]);
  }
}

// A block's share of the partitioned rows: a whole partition (partial < 0:
// its groups go straight to the outputs), or a slice of a partition too
// large for one block (its table is written whole to partial table
// `partial`, and group_part_merge_kernel adds the slices' tables up).
struct AggUnit {
  long long begin, end;
  int32_t partial;
  int32_t pad;
};

// One block per unit (or, with units null, per partition): aggregate the
// rows in a shared table, then append the groups or write the partial table.
template <bool HAS2>
__global__ void __launch_bounds__(kAggThreads) group_part_agg_kernel(
    const long long* __restrict__ part_begin, const AggUnit* __restrict__ units,
    const typename PartRow<HAS2>::T* __restrict__ rows, int combine, int64_t capacity,
    int32_t* __restrict__ out_keys, int64_t* __restrict__ out_sums, int64_t* __restrict__ out_counts,
    unsigned long long* d_groups, unsigned long long* overflow, int4* __restrict__ partials) {
  extern __shared__ __align__(16) unsigned char agg_smem[];
  const SmemAgg st = smem_agg(agg_smem, kAggSlots);
  smem_agg_clear(st);
  __syncthreads();
  int64_t b, e;
  int partial = -1;
  if (units) {
    const AggUnit u = units[blockIdx.x];
    b = u.begin;
    e = u.end;
    partial = u.partial;
  } else {
    b = part_begin[blockIdx.x];
    e = part_begin[blockIdx.x + 1];
  }
  unsigned int lost = 0;
  // rows of the partition, 8 per thread in flight
  for (int64_t base = b; base < e; base += 8 * static_cast<int64_t>(blockDim.x)) {
    if (!combine) {  // two batches of 4 rows
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        int32_t k[4];
        int64_t v[4];
        uint32_t valid = 0;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int64_t i = base + (4 * h + u) * static_cast<int64_t>(blockDim.x) + threadIdx.x;
          const bool ok = i < e;
          typename PartRow<HAS2>::T x{};
          if (ok) x = rows[i];
          k[u] = ok ? PartRow<HAS2>::key(x) : 0;
          v[u] = ok ? PartRow<HAS2>::val(x) : 0;
          valid |= static_cast<uint32_t>(ok) << u;
        }
        lost += __popc(smem_agg_rows<4>(st, k, v, valid, 0xffffffffu));  // the loop is block-uniform
      }
      continue;
    }
    typename PartRow<HAS2>::T r[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int64_t i = base + u * static_cast<int64_t>(blockDim.x) + threadIdx.x;
      if (i < e) r[u] = rows[i];
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int64_t i = base + u * static_cast<int64_t>(blockDim.x) + threadIdx.x;
      const bool ok = i < e;
      const int32_t k = ok ? PartRow<HAS2>::key(r[u]) : 0;
      int64_t gs = ok ? PartRow<HAS2>::val(r[u]) : 0;
      uint32_t gc = 1;
      if (warp_combine(ok, k, gs, &gs, &gc))
        if (!smem_agg_add(st, k, static_cast<uint64_t>(gs), gc)) ++lost;
    }
  }
  if (lost) atomicAdd(overflow, static_cast<unsigned long long>(lost));
  __syncthreads();
  if (partial >= 0) {  // the whole table, as laid out in shared memory (16 bytes per slot)
    const int4* src = reinterpret_cast<const int4*>(agg_smem);
    int4* dst = partials + static_cast<int64_t>(partial) * kAggSlots;
    for (int i = threadIdx.x; i < kAggSlots; i += blockDim.x) dst[i] = src[i];
    return;
  }
  append_groups(st, capacity, out_keys, out_sums, out_counts, d_groups, overflow);
}

// One block per partition split over several units: adds up the partial
// tables of its units (merge[b] = (first partial, count)) in a shared table
// and appends the groups.
__global__ void __launch_bounds__(kAggThreads) group_part_merge_kernel(
    const int2* __restrict__ merge, const int4* __restrict__ partials, int64_t capacity,
    int32_t* __restrict__ out_keys, int64_t* __restrict__ out_sums, int64_t* __restrict__ out_counts,
    unsigned long long* d_groups, unsigned long long* overflow) {
  extern __shared__ __align__(16) unsigned char agg_smem[];
  const SmemAgg st = smem_agg(agg_smem, kAggSlots);
  smem_agg_clear(st);
  __syncthreads();
  const int2 m = merge[blockIdx.x];
  unsigned int lost = 0;
  for (int q = 0; q < m.y; ++q) {
    const SmemAgg pt = smem_agg(reinterpret_cast<unsigned char*>(const_cast<int4*>(partials) +
                                                                 static_cast<int64_t>(m.x + q) * kAggSlots),
                                kAggSlots);
    for (int i = threadIdx.x; i < kAggSlots; i += blockDim.x) {
      const int32_t k = pt.key[i];
      if (k != kEmptyKey && !smem_agg_add(st, k, pt.sum(i), pt.cnt[i])) ++lost;
    }
  }
  if (lost) atomicAdd(overflow, static_cast<unsigned long long>(lost));
  __syncthreads();
  append_groups(st, capacity, out_keys, out_sums, out_counts, d_groups, overflow);
}

// Compaction of the occupied slots into (key, sum, count) arrays.
struct SlotOp {
  static constexpr int kGroups = kCompactGroups;
  const int32_t* keys;
  const unsigned long long* sums;
  const unsigned long long* counts;
  int32_t* out_keys;
  int64_t* out_sums;
  int64_t* out_counts;
  int4 k4[kCompactGroups];

  __device__ __forceinline__ bool vec_ok() const { return true; }
  __device__ __forceinline__ void prefetch(int, int64_t) {}
  template <bool kFull>
  __device__ __forceinline__ uint32_t flags(int u, int64_t first, int nv) {
    int32_t k[4] = {kEmptyKey, kEmptyKey, kEmptyKey, kEmptyKey};
    for (int j = 0; j < nv; ++j) k[j] = keys[first + j];
    k4[u] = make_int4(k[0], k[1], k[2], k[3]);
    uint32_t m = 0;
#pragma unroll
    for (int j = 0; j < 4; ++j) m |= static_cast<uint32_t>(k[j] != kEmptyKey) << j;
    return m;
  }
  __device__ __forceinline__ void emit(int u, int j, int64_t item, int64_t pos) {
    out_keys[pos] = j == 0 ? k4[u].x : j == 1 ? k4[u].y : j == 2 ? k4[u].z : k4[u].w;
    out_sums[pos] = static_cast<int64_t>(sums[item]);
    if (out_counts) out_counts[pos] = static_cast<int64_t>(counts[item]);
  }
};

__global__ void fill_i32_kernel(int32_t* p, int64_t n, int32_t v) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) p[i] = v;
}

// SUM(price * qty * (100 + tax)) in int64 (exact modulo 2^64).
__global__ void __launch_bounds__(512) agg_fixed_kernel(int64_t n, const int32_t* __restrict__ price,
                                                        const int32_t* __restrict__ qty,
                                                        const int32_t* __restrict__ tax,
                                                        unsigned long long* sum) {
  __shared__ long long s_red[16];
  const uint64_t pol = policy_evict_first();
  uint64_t s = 0;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  const int64_t t0 = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  auto term = [](int32_t p, int32_t q, int32_t t) {
    return static_cast<uint64_t>(static_cast<int64_t>(p) * q) * static_cast<uint64_t>(static_cast<int64_t>(100) + t);
  };
  const bool vec = ((reinterpret_cast<uintptr_t>(price) | reinterpret_cast<uintptr_t>(qty) |
                     reinterpret_cast<uintptr_t>(tax)) & 15) == 0;
  const int64_t n4 = vec ? n >> 2 : 0;
  for (int64_t i = t0; i < n4; i += stride) {
    const int4 p = ld_stream_v4(price + 4 * i, pol), q = ld_stream_v4(qty + 4 * i, pol), t = ld_stream_v4(tax + 4 * i, pol);
    s += term(p.x, q.x, t.x) + term(p.y, q.y, t.y) + term(p.z, q.z, t.z) + term(p.w, q.w, t.w);
  }
  for (int64_t r = 4 * n4 + t0; r < n; r += stride) s += term(price[r], qty[r], tax[r]);
  int64_t v = warp_sum_i64(static_cast<int64_t>(s));
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) s_red[warp] = v;
  __syncthreads();
  if (warp == 0) {
    long long x = lane < static_cast<int>(blockDim.x >> 5) ? s_red[lane] : 0;
    x = warp_sum_i64(x);
    if (lane == 0) atomicAdd(sum, static_cast<unsigned long long>(x));
  }
}

// Double variant, deterministic: fixed per-block partial sums (each block a
// fixed contiguous range, reduced in a fixed tree order), then one block sums
// the partials in block order.
constexpr int kAggF64Blocks = 1024;
__global__ void __launch_bounds__(256) agg_f64_partial_kernel(int64_t n, const double* __restrict__ tax,
                                                              const double* __restrict__ qty,
                                                              const double* __restrict__ price,
                                                              double* __restrict__ partial) {
  __shared__ double s[256];
  const int64_t per = (n + gridDim.x - 1) / gridDim.x;
  const int64_t b = static_cast<int64_t>(blockIdx.x) * per;
  const int64_t e = b + per < n ? b + per : n;
  double acc = 0.0;
  for (int64_t r = b + threadIdx.x; r < e; r += blockDim.x) {
    const double netto = price[r] * qty[r];
    acc += netto * tax[r] + netto;
  }
  s[threadIdx.x] = acc;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (threadIdx.x < o) s[threadIdx.x] += s[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = s[0];
}

__global__ void agg_f64_final_kernel(const double* __restrict__ partial, int nb, double* out) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    double a = 0.0;
    for (int i = 0; i < nb; ++i) a += partial[i];
    *out = a;
  }
}

// The context's grow-only buffer (declared in olap_internal.cuh).
char* big_scratch(olap_ctx* ctx, size_t bytes) {
  if (bytes <= ctx->big_bytes) return ctx->big;
  if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) return nullptr;
  if (ctx->big) cudaFree(ctx->big);
  ctx->big = nullptr;
  ctx->big_bytes = 0;
  const size_t want = bytes + bytes / 4;
  if (cudaMalloc(reinterpret_cast<void**>(&ctx->big), want) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  ctx->big_bytes = want;
  return ctx->big;
}

static unsigned grid_of(const olap_ctx* ctx, int64_t items, int threads, int per_sm) {
  int64_t g = (items + threads - 1) / threads;
  const int64_t cap = static_cast<int64_t>(ctx->sm_count) * per_sm;
  if (g > cap) g = cap;
  return static_cast<unsigned>(g < 1 ? 1 : g);
}

}  // namespace olap

extern "C" {

int olap_group_vector(olap_ctx* ctx, int64_t n, const int32_t* vecInx, const int32_t* m1,
                      const int32_t* m2, int64_t group_num, int64_t* group_vector, int64_t* counts,
                      int64_t* d_total) {
  if (!ctx) return OLAP_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  OLAP_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  OLAP_REQUIRE(ctx, n >= 0 && group_num >= 1 && group_vector && d_total, "bad arguments");
  OLAP_REQUIRE(ctx, n == 0 || (vecInx && m1 && m2), "null column");
  OLAP_CUDA_TRY(ctx, cudaMemsetAsync(group_vector, 0, sizeof(int64_t) * group_num, ctx->stream));
  if (counts) OLAP_CUDA_TRY(ctx, cudaMemsetAsync(counts, 0, sizeof(int64_t) * group_num, ctx->stream));
  OLAP_CUDA_TRY(ctx, cudaMemsetAsync(d_total, 0, sizeof(int64_t), ctx->stream));
  if (n == 0) return OLAP_OK;
  const int64_t smem = group_num * 8 * (counts ? 2 : 1);
  const bool use_smem = smem <= 96 * 1024;
  auto sums = reinterpret_cast<unsigned long long*>(group_vector);
  auto cnts = reinterpret_cast<unsigned long long*>(counts);
  auto tot = reinterpret_cast<unsigned long long*>(d_total);
  if (use_smem) {
    OLAP_CUDA_TRY(ctx, cudaFuncSetAttribute(olap::group_vector_kernel<true>,
                                            cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024));
    const int per_sm = smem > 48 * 1024 ? 2 : 4;
    olap::group_vector_kernel<true><<<olap::grid_of(ctx, (n + 3) / 4, olap::kGroupThreads, per_sm),
                                      olap::kGroupThreads, static_cast<size_t>(smem), ctx->stream>>>(
        n, vecInx, m1, m2, group_num, sums, cnts, tot, &ctx->counters->range_errors);
  } else {
    olap::group_vector_kernel<false><<<olap::grid_of(ctx, (n + 3) / 4, olap::kGroupThreads, 4),
                                       olap::kGroupThreads, 0, ctx->stream>>>(
        n, vecInx, m1, m2, group_num, sums, cnts, tot, &ctx->counters->range_errors);
  }
  OLAP_CUDA_TRY(ctx, cudaGetLastError());
  return OLAP_OK;
}

int64_t olap_group_hash_capacity(int64_t max_groups) {
  int64_t cap = 1024;
  while (cap < 2 * max_groups) cap <<= 1;
  return cap;
}

int olap_group_hash(olap_ctx* ctx, int64_t n, const int32_t* keys, int32_t key_offset,
                    const int32_t* vals, const int32_t* vals2, int64_t capacity, int32_t* out_keys,
                    int64_t* out_sums, int64_t* out_counts, int64_t* d_groups) {
  if (!ctx) return OLAP_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  OLAP_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  OLAP_REQUIRE(ctx, n >= 0 && capacity >= 1024 && (capacity & (capacity - 1)) == 0,
               "capacity must be a power of two >= 1024 (see olap_group_hash_capacity)");
  OLAP_REQUIRE(ctx, n < (int64_t(1) << 32), "at most 2^32 - 1 rows per call");
  OLAP_REQUIRE(ctx, out_keys && out_sums && d_groups, "null output");
  OLAP_REQUIRE(ctx, n == 0 || (keys && vals), "null column");
  olap::Arena ar(ctx);
  unsigned long long* overflow = ar.take<unsigned long long>(1);
  if (!overflow) return olap::set_error(ctx, OLAP_ERR_CAPACITY, "scratch arena exhausted");
  OLAP_CUDA_TRY(ctx, cudaMemsetAsync(overflow, 0, sizeof(unsigned long long), ctx->stream));
  int st = OLAP_OK;
  char* mem = nullptr;
  cudaError_t e = cudaSuccess;
  // Warp combining of equal keys (match_any + reductions) costs more than the
  // same-address shared atomics it saves on uniform and mildly skewed keys
  // (measured on B200), so it is off unless the tuning knob asks for it.
  const int combine = ctx->tune[olap::TUNE_GROUP_COMBINE] == 1 ? 1 : 0;
  const int64_t plan_knob = ctx->tune[olap::TUNE_GROUP_PLAN];
  // Knob: 1 plan 1 where it fits (batched table updates), 2 plan 2 always,
  // 3 plan 1 with one row's table update after another; 0 the default (1).
  const bool plan1 = plan_knob == 2 ? false : capacity <= olap::kAggSlots;
  const bool batched = plan_knob != 3 && combine == 0;
  if (plan1) {
    // Plan 1: per-block shared tables of `capacity` slots, then the global
    // table (in the context's grow-only buffer) and its compaction.
    const size_t bytes = static_cast<size_t>(capacity) * (4 + 8 + 8);
    mem = olap::big_scratch(ctx, bytes);
    if (!mem) return olap::set_error(ctx, OLAP_ERR_NOMEM, "device memory for the group table");
    olap::HashAgg t;
    t.sums = reinterpret_cast<unsigned long long*>(mem);
    t.counts = t.sums + capacity;
    t.keys = reinterpret_cast<int32_t*>(t.counts + capacity);
    t.mask = static_cast<uint64_t>(capacity - 1);
    t.overflow = overflow;
    e = cudaMemsetAsync(mem, 0, static_cast<size_t>(capacity) * 16, ctx->stream);
    olap::fill_i32_kernel<<<olap::grid_of(ctx, capacity, 256, 8), 256, 0, ctx->stream>>>(t.keys, capacity,
                                                                                       olap::kEmptyKey);
    const uint32_t slots = static_cast<uint32_t>(capacity);  // per-block table
    if (n && e == cudaSuccess && batched) {
      // The block tables fill the shared memory once the keys are many: at
      // lower load fewer keys overflow their home bucket, and the lanes of a
      // warp take the insert path less often.
      uint32_t tslots = slots;
      if (capacity >= 2048)
        tslots = std::max<uint32_t>(slots, static_cast<uint32_t>(ctx->smem_optin / 16) & ~3u);
      const size_t smem = static_cast<size_t>(tslots) * 16;
      auto launch = [&](auto kern) {
        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        int bps = 1;
        if (e == cudaSuccess)
          e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kern, olap::kRowsThreads, smem);
        int64_t grid = static_cast<int64_t>(ctx->sm_count) * (bps < 1 ? 1 : bps);
        grid = std::min<int64_t>(grid, (n + 4 * olap::kRowsThreads - 1) / (4 * olap::kRowsThreads));
        if (e == cudaSuccess)
          kern<<<static_cast<unsigned>(grid < 1 ? 1 : grid), olap::kRowsThreads, smem, ctx->stream>>>(
              n, keys, key_offset, vals, vals2, tslots, t, &ctx->counters->range_errors);
      };
      if (vals2)
        launch(olap::group_hash_rows_kernel<true>);
      else
        launch(olap::group_hash_rows_kernel<false>);
    } else if (n && e == cudaSuccess) {
      const size_t smem = static_cast<size_t>(slots) * 16;
      e = cudaFuncSetAttribute(olap::group_hash_smem_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               static_cast<int>(smem));
      int bps = 1;
      if (e == cudaSuccess)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, olap::group_hash_smem_kernel, olap::kAggThreads,
                                                          smem);
      int64_t grid = static_cast<int64_t>(ctx->sm_count) * (bps < 1 ? 1 : bps);
      grid = std::min<int64_t>(grid, (n + 4 * olap::kAggThreads - 1) / (4 * olap::kAggThreads));
      if (e == cudaSuccess)
        olap::group_hash_smem_kernel<<<static_cast<unsigned>(grid < 1 ? 1 : grid), olap::kAggThreads, smem,
                                       ctx->stream>>>(n, keys, key_offset, vals, vals2,
                                                      slots, combine, t,
                                                      &ctx->counters->range_errors);
    }
    olap::SlotOp op;
    std::memset(&op, 0, sizeof(op));
    op.keys = t.keys;
    op.sums = t.sums;
    op.counts = t.counts;
    op.out_keys = out_keys;
    op.out_sums = out_sums;
    op.out_counts = out_counts;
    olap::ScanTiles sc;
    if (e == cudaSuccess)
      st = olap::make_scan_tiles(ctx, ar, capacity, reinterpret_cast<unsigned long long*>(d_groups), ctx->stream,
                                 &sc, olap::compact_tile_items<olap::SlotOp>());
    if (e == cudaSuccess && st == OLAP_OK)
      olap::compact_kernel<olap::SlotOp><<<olap::compact_grid(ctx, sc.n_tiles), olap::kCompactThreads, 0,
                                          ctx->stream>>>(op, capacity, sc);
  } else {
    // Plan 2: partition, then one block per partition.
    olap::PartPlan pp;
    pp.n = n;
    pp.key_offset = key_offset;
    int64_t parts = std::max<int64_t>(512, capacity / olap::kAggSlots);
    int lg = 0;
    while ((int64_t(1) << lg) < parts) ++lg;
    if (lg > 15) return olap::set_error(ctx, OLAP_ERR_UNSUPPORTED, "hash group-by capacity above 2^27 slots");
    pp.n_parts = 1 << lg;
    pp.part_shift = 32 - lg;
    pp.n_blocks = ctx->sm_count * 2;
    pp.per = ((n + pp.n_blocks - 1) / pp.n_blocks + 3) & ~int64_t(3);
    if (pp.per < 4) pp.per = 4;
    const size_t hist_bytes = sizeof(unsigned int) * static_cast<size_t>(pp.n_parts) * pp.n_blocks;
    // part_begin[P + 1], then ptot[P] and cursor[P] (zeroed together)
    const size_t begin_bytes = sizeof(long long) * (3 * static_cast<size_t>(pp.n_parts) + 1);
    const size_t row_bytes = vals2 ? 16 : 8;
    // after the rows: the work units, the merge list and the partial tables
    // of partitions too large for one block (at most kMaxPartials of them)
    const size_t rows_off = (begin_bytes + hist_bytes + 255) & ~size_t(255);
    const size_t units_off = (rows_off + static_cast<size_t>(n > 0 ? n : 1) * row_bytes + 255) & ~size_t(255);
    const size_t max_units = static_cast<size_t>(pp.n_parts) + olap::kMaxPartials;
    const size_t merge_off = (units_off + sizeof(olap::AggUnit) * max_units + 255) & ~size_t(255);
    const size_t part_off = (merge_off + sizeof(int2) * static_cast<size_t>(pp.n_parts) + 255) & ~size_t(255);
    const size_t bytes = part_off + static_cast<size_t>(olap::kMaxPartials) * olap::kAggSlots * 16;
    mem = olap::big_scratch(ctx, bytes);
    if (!mem) return olap::set_error(ctx, OLAP_ERR_NOMEM, "device memory for the group partitions");
    long long* part_begin = reinterpret_cast<long long*>(mem);
    auto* ptot = reinterpret_cast<unsigned long long*>(part_begin + pp.n_parts + 1);
    auto* cursor = ptot + pp.n_parts;
    unsigned int* hist = reinterpret_cast<unsigned int*>(mem + begin_bytes);
    char* rowbuf = mem + rows_off;
    auto* d_units = reinterpret_cast<olap::AggUnit*>(mem + units_off);
    auto* d_merge = reinterpret_cast<int2*>(mem + merge_off);
    auto* d_partials = reinterpret_cast<int4*>(mem + part_off);
    e = cudaMemsetAsync(d_groups, 0, sizeof(int64_t), ctx->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(ptot, 0, sizeof(unsigned long long) * pp.n_parts, ctx->stream);
    const size_t psmem = sizeof(unsigned int) * pp.n_parts;
    if (e == cudaSuccess && psmem > 48 * 1024) {
      e = cudaFuncSetAttribute(olap::group_part_hist_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               static_cast<int>(psmem));
      if (e == cudaSuccess)
        e = cudaFuncSetAttribute(olap::group_part_scatter_kernel<true>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(psmem));
      if (e == cudaSuccess)
        e = cudaFuncSetAttribute(olap::group_part_scatter_kernel<false>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(psmem));
    }
    const size_t asmem = static_cast<size_t>(olap::kAggSlots) * 16;
    if (pp.n_parts <= olap::kTiledParts) {
      const int tsm = static_cast<int>((vals2 ? 18 : 10) * olap::kScatterTile + 4 * psmem);
      if (e == cudaSuccess)
        e = cudaFuncSetAttribute(olap::group_part_scatter_tiled_kernel<true>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, tsm);
      if (e == cudaSuccess)
        e = cudaFuncSetAttribute(olap::group_part_scatter_tiled_kernel<false>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, tsm);
    }
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(olap::group_part_agg_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               static_cast<int>(asmem));
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(olap::group_part_agg_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               static_cast<int>(asmem));
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(olap::group_part_merge_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               static_cast<int>(asmem));
    if (e == cudaSuccess) {
      olap::group_part_hist_kernel<<<pp.n_blocks, 1024, psmem, ctx->stream>>>(pp, keys, hist, ptot,
                                                                              &ctx->counters->range_errors);
      olap::group_part_scan_kernel<<<1, 1024, 0, ctx->stream>>>(pp, ptot, part_begin, cursor);
      auto* d_groups_u = reinterpret_cast<unsigned long long*>(d_groups);
      // Partition sizes decide the blocks: a partition far above the average
      // (skewed keys) is split into slices of at most `limit` rows whose
      // partial tables are merged afterwards, so no single block gets it all.
      std::vector<long long> pb(static_cast<size_t>(pp.n_parts) + 1);
      e = cudaMemcpyAsync(pb.data(), part_begin, sizeof(long long) * pb.size(), cudaMemcpyDeviceToHost, ctx->stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
      std::vector<olap::AggUnit> units;
      std::vector<int2> merges;
      if (e == cudaSuccess) {
        const int64_t avg = (n + pp.n_parts - 1) / pp.n_parts;
        int64_t limit = std::max<int64_t>(2 * avg, int64_t(1) << 16);
        auto slices = [&](int64_t lim) {
          int64_t t = 0;
          for (int p = 0; p < pp.n_parts; ++p) {
            const int64_t sz = pb[p + 1] - pb[p];
            if (sz > lim) t += (sz + lim - 1) / lim;
          }
          return t;
        };
        while (slices(limit) > olap::kMaxPartials) limit *= 2;
        int32_t np = 0;
        for (int p = 0; p < pp.n_parts; ++p) {
          const int64_t sz = pb[p + 1] - pb[p];
          if (sz <= limit) continue;
          const int64_t k = (sz + limit - 1) / limit;
          merges.push_back(make_int2(np, static_cast<int>(k)));
          for (int64_t q = 0; q < k; ++q) {
            const long long lo = pb[p] + q * limit, hi = std::min<long long>(pb[p + 1], lo + limit);
            units.push_back(olap::AggUnit{lo, hi, np++, 0});
          }
        }
        if (!merges.empty()) {
          for (int p = 0; p < pp.n_parts; ++p)
            if (pb[p + 1] - pb[p] <= limit) units.push_back(olap::AggUnit{pb[p], pb[p + 1], -1, 0});
          e = cudaMemcpyAsync(d_units, units.data(), sizeof(olap::AggUnit) * units.size(), cudaMemcpyHostToDevice,
                              ctx->stream);
          if (e == cudaSuccess)
            e = cudaMemcpyAsync(d_merge, merges.data(), sizeof(int2) * merges.size(), cudaMemcpyHostToDevice,
                                ctx->stream);
        }
      }
      const olap::AggUnit* unit_arg = merges.empty() ? nullptr : d_units;
      const unsigned agg_grid = merges.empty() ? static_cast<unsigned>(pp.n_parts)
                                               : static_cast<unsigned>(units.size());
      const bool tiled = pp.n_parts <= olap::kTiledParts;
      const size_t tsmem = (vals2 ? 18 : 10) * static_cast<size_t>(olap::kScatterTile) + 4 * psmem;
      if (vals2) {
        auto* rows = reinterpret_cast<longlong2*>(rowbuf);
        if (tiled)
          olap::group_part_scatter_tiled_kernel<true><<<pp.n_blocks, 1024, tsmem, ctx->stream>>>(
              pp, keys, vals, vals2, hist, cursor, rows);
        else
          olap::group_part_scatter_kernel<true><<<pp.n_blocks, 1024, psmem, ctx->stream>>>(pp, keys, vals, vals2,
                                                                                          hist, cursor, rows);
        if (e == cudaSuccess)
          olap::group_part_agg_kernel<true><<<agg_grid, olap::kAggThreads, asmem, ctx->stream>>>(
              part_begin, unit_arg, rows, combine, capacity, out_keys, out_sums, out_counts, d_groups_u, overflow,
              d_partials);
      } else {
        auto* rows = reinterpret_cast<int2*>(rowbuf);
        if (tiled)
          olap::group_part_scatter_tiled_kernel<false><<<pp.n_blocks, 1024, tsmem, ctx->stream>>>(
              pp, keys, vals, nullptr, hist, cursor, rows);
        else
          olap::group_part_scatter_kernel<false><<<pp.n_blocks, 1024, psmem, ctx->stream>>>(pp, keys, vals,
                                                                                           nullptr, hist, cursor,
                                                                                           rows);
        if (e == cudaSuccess)
          olap::group_part_agg_kernel<false><<<agg_grid, olap::kAggThreads, asmem, ctx->stream>>>(
              part_begin, unit_arg, rows, combine, capacity, out_keys, out_sums, out_counts, d_groups_u, overflow,
              d_partials);
      }
      if (e == cudaSuccess && !merges.empty())
        olap::group_part_merge_kernel<<<static_cast<unsigned>(merges.size()), olap::kAggThreads, asmem,
                                        ctx->stream>>>(d_merge, d_partials, capacity, out_keys, out_sums,
                                                       out_counts, d_groups_u, overflow);
      if (e == cudaSuccess) e = cudaGetLastError();
    }
  }
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess && st == OLAP_OK) st = olap::check_cuda(ctx, e, "group_hash");
  unsigned long long ov = 0;
  if (st == OLAP_OK) cudaMemcpyAsync(&ov, overflow, sizeof(ov), cudaMemcpyDeviceToHost, ctx->stream);
  OLAP_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  if (st == OLAP_OK && ov) return olap::set_error(ctx, OLAP_ERR_CAPACITY, "group hash table full");
  if (st == OLAP_OK) st = olap::check_timeouts(ctx, ctx->stream);
  return st;
}

int olap_agg_fixed(olap_ctx* ctx, int64_t n, const int32_t* price, const int32_t* qty,
                   const int32_t* tax_pct, int64_t* d_sum) {
  if (!ctx) return OLAP_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  OLAP_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  OLAP_REQUIRE(ctx, n >= 0 && d_sum, "bad arguments");
  OLAP_REQUIRE(ctx, n == 0 || (price && qty && tax_pct), "null column");
  OLAP_CUDA_TRY(ctx, cudaMemsetAsync(d_sum, 0, sizeof(int64_t), ctx->stream));
  if (n == 0) return OLAP_OK;
  olap::agg_fixed_kernel<<<olap::grid_of(ctx, (n + 3) / 4, 512, 4), 512, 0, ctx->stream>>>(
      n, price, qty, tax_pct, reinterpret_cast<unsigned long long*>(d_sum));
  OLAP_CUDA_TRY(ctx, cudaGetLastError());
  return OLAP_OK;
}

int olap_agg_f64(olap_ctx* ctx, int64_t n, const double* tax, const double* qty, const double* price,
                 double* d_sum) {
  if (!ctx) return OLAP_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  OLAP_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  OLAP_REQUIRE(ctx, n >= 0 && d_sum, "bad arguments");
  OLAP_REQUIRE(ctx, n == 0 || (tax && qty && price), "null column");
  olap::Arena ar(ctx);
  double* partial = ar.take<double>(olap::kAggF64Blocks);
  if (!partial) return olap::set_error(ctx, OLAP_ERR_CAPACITY, "scratch arena exhausted");
  olap::agg_f64_partial_kernel<<<olap::kAggF64Blocks, 256, 0, ctx->stream>>>(n, tax, qty, price, partial);
  olap::agg_f64_final_kernel<<<1, 32, 0, ctx->stream>>>(partial, olap::kAggF64Blocks, d_sum);
  OLAP_CUDA_TRY(ctx, cudaGetLastError());
  return OLAP_OK;
}

}  // extern "C"
