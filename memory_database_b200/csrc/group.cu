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
// atomics.  Hash group-by keeps a 4096-slot shared-memory table per block
// (keys inserted with shared CAS) in front of a global open-addressing table;
// rows that do not fit the block table go to the global table directly.
#include <cstring>

#include "compact.cuh"

namespace olap {

constexpr int kGroupThreads = 512;
constexpr int kSmemSlots = 2048;  // block hash table slots (32 KiB of shared memory)
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

__global__ void __launch_bounds__(kGroupThreads) group_hash_kernel(int64_t n, const int32_t* __restrict__ keys,
                                                                   int32_t key_offset,
                                                                   const int32_t* __restrict__ vals,
                                                                   const int32_t* __restrict__ vals2, HashAgg t,
                                                                   unsigned long long* range_err) {
  __shared__ int32_t skey[kSmemSlots];
  __shared__ unsigned long long ssum[kSmemSlots];
  __shared__ unsigned int scnt[kSmemSlots];
  const int tid = threadIdx.x;
  for (int i = tid; i < kSmemSlots; i += blockDim.x) {
    skey[i] = kEmptyKey;
    ssum[i] = 0;
    scnt[i] = 0;
  }
  __syncthreads();
  unsigned int bad = 0;
  auto add = [&](int32_t key, int64_t v) {
    const int32_t k = static_cast<int32_t>(static_cast<uint32_t>(key) + static_cast<uint32_t>(key_offset));
    if (k == kEmptyKey) {  // reserved as the empty marker
      ++bad;
      return;
    }
    uint32_t h = mix32(static_cast<uint32_t>(k)) & (kSmemSlots - 1);
#pragma unroll 1
    for (int step = 0; step < 8; ++step) {
      const int32_t prev = atomicCAS(skey + h, kEmptyKey, k);
      if (prev == kEmptyKey || prev == k) {
        smem_add_u64(ssum + h, static_cast<uint64_t>(static_cast<int64_t>(v)));
        atomicAdd(scnt + h, 1u);
        return;
      }
      h = (h + 1) & (kSmemSlots - 1);
    }
    global_add(t, k, static_cast<uint64_t>(static_cast<int64_t>(v)), 1);  // block table crowded
  };
  const uint64_t pol = policy_evict_first();
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  const int64_t t0 = static_cast<int64_t>(blockIdx.x) * blockDim.x + tid;
  const bool vec = ((reinterpret_cast<uintptr_t>(keys) | reinterpret_cast<uintptr_t>(vals) |
                     reinterpret_cast<uintptr_t>(vals2)) & 15) == 0;
  const int64_t n4 = vec ? n >> 2 : 0;
  for (int64_t i = t0; i < n4; i += stride) {
    const int4 k = ld_stream_v4(keys + 4 * i, pol), v = ld_stream_v4(vals + 4 * i, pol);
    const int4 w = vals2 ? ld_stream_v4(vals2 + 4 * i, pol) : make_int4(0, 0, 0, 0);
    add(k.x, static_cast<int64_t>(v.x) + w.x);
    add(k.y, static_cast<int64_t>(v.y) + w.y);
    add(k.z, static_cast<int64_t>(v.z) + w.z);
    add(k.w, static_cast<int64_t>(v.w) + w.w);
  }
  for (int64_t r = 4 * n4 + t0; r < n; r += stride)
    add(keys[r], static_cast<int64_t>(vals[r]) + (vals2 ? vals2[r] : 0));
  const unsigned int wbad = __reduce_add_sync(0xffffffffu, bad);
  if ((tid & 31) == 0 && wbad) atomicAdd(range_err, static_cast<unsigned long long>(wbad));
  __syncthreads();
  for (int i = tid; i < kSmemSlots; i += blockDim.x)
    if (skey[i] != kEmptyKey) global_add(t, skey[i], ssum[i], scnt[i]);
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
  OLAP_REQUIRE(ctx, out_keys && out_sums && d_groups, "null output");
  OLAP_REQUIRE(ctx, n == 0 || (keys && vals), "null column");
  // Table from the stream-ordered pool: keys, sums, counts.
  char* mem = nullptr;
  const size_t bytes = static_cast<size_t>(capacity) * (4 + 8 + 8);
  OLAP_CUDA_TRY(ctx, cudaMallocAsync(reinterpret_cast<void**>(&mem), bytes, ctx->stream));
  olap::HashAgg t;
  t.sums = reinterpret_cast<unsigned long long*>(mem);
  t.counts = t.sums + capacity;
  t.keys = reinterpret_cast<int32_t*>(t.counts + capacity);
  t.mask = static_cast<uint64_t>(capacity - 1);
  olap::Arena ar(ctx);
  t.overflow = ar.take<unsigned long long>(1);
  int st = OLAP_OK;
  if (!t.overflow) st = olap::set_error(ctx, OLAP_ERR_CAPACITY, "scratch arena exhausted");
  if (st == OLAP_OK) {
    cudaMemsetAsync(t.overflow, 0, sizeof(unsigned long long), ctx->stream);
    cudaMemsetAsync(mem, 0, static_cast<size_t>(capacity) * 16, ctx->stream);
    olap::fill_i32_kernel<<<olap::grid_of(ctx, capacity, 256, 8), 256, 0, ctx->stream>>>(t.keys, capacity,
                                                                                       olap::kEmptyKey);
    if (n)
      olap::group_hash_kernel<<<olap::grid_of(ctx, (n + 3) / 4, olap::kGroupThreads, 2), olap::kGroupThreads,
                                0, ctx->stream>>>(n, keys, key_offset, vals, vals2, t,
                                                  &ctx->counters->range_errors);
    olap::SlotOp op;
    std::memset(&op, 0, sizeof(op));
    op.keys = t.keys;
    op.sums = t.sums;
    op.counts = t.counts;
    op.out_keys = out_keys;
    op.out_sums = out_sums;
    op.out_counts = out_counts;
    olap::ScanTiles sc;
    st = olap::make_scan_tiles(ctx, ar, capacity, reinterpret_cast<unsigned long long*>(d_groups), ctx->stream,
                               &sc, olap::compact_tile_items<olap::SlotOp>());
    if (st == OLAP_OK)
      olap::compact_kernel<olap::SlotOp><<<olap::compact_grid(ctx, sc.n_tiles), olap::kCompactThreads, 0,
                                          ctx->stream>>>(op, capacity, sc);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess && st == OLAP_OK) st = olap::check_cuda(ctx, e, "group_hash");
  }
  unsigned long long ov = 0;
  if (st == OLAP_OK && t.overflow)
    cudaMemcpyAsync(&ov, t.overflow, sizeof(ov), cudaMemcpyDeviceToHost, ctx->stream);
  cudaFreeAsync(mem, ctx->stream);
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
