// The TPC-H Q5-shaped join chain for sm_100a.
//
// Reference: code/TPCH_Q5/Q5.cpp.  set_bitmap (:913-920) marks the regions
// equal to REGION; DimVec_S (:921-931) maps each supplier to its nation when
// the nation lies in a marked region (else -1); DimVec_o (:932-944) maps each
// order to its customer's nation when that nation lies in a marked region and
// DATE1 <= o_orderdate < DATE2 (else -1); Tri_table_join (:945-978) keeps the
// line rows whose supplier nation is not -1 and equals their order's nation,
// and adds l_extendedprice * (1 - l_discount) to that nation's sum (double).
// Here the sum is int64 fixed point: SUM price_cents * (100 - discount_pct),
// exactly 100 x 100 x the decimal revenue.
//
// Three passes: suppliers -> int8 nation vector and its 4-bit codes (staged
// in shared memory by the line pass), orders -> int8 nation vector (one byte per order,
// L2-resident for the line pass), lines -> per-nation int64 sums in shared
// memory, flushed once per block.  Customer and supplier keys are 1-based as
// in the reference; orders are addressed by row (l_orderkey_new).
#include <algorithm>
#include <cstring>

#include "olap_internal.cuh"

namespace olap {

constexpr int kQ5MaxNations = 64;

// Nations whose region passes, as a bit mask (n_regionkey[n] == region).
__device__ __forceinline__ bool nation_ok(uint64_t mask, int32_t n) {
  return static_cast<uint32_t>(n) < kQ5MaxNations && ((mask >> n) & 1ull);
}

// set_bitmap + nation -> region: bit n set when nation n's region has key `region`.
__global__ void q5_nation_mask_kernel(const int32_t* __restrict__ r_regionkey, int64_t n_region,
                                      const int32_t* __restrict__ n_regionkey, int64_t n_nation, int32_t region,
                                      unsigned long long* __restrict__ mask) {
  const int n = threadIdx.x;
  const bool ok = n < n_nation && n_regionkey[n] >= 0 && n_regionkey[n] < n_region &&
                  r_regionkey[n_regionkey[n]] == region;
  __shared__ unsigned long long s[2];
  const unsigned int b = __ballot_sync(0xffffffffu, ok);
  if ((n & 31) == 0) s[n >> 5] = b;
  __syncthreads();
  if (n == 0) *mask = s[0] | (s[1] << 32);
}

__global__ void q5_supplier_kernel(const int32_t* __restrict__ s_nationkey, int64_t n_supp,
                                   const unsigned long long* __restrict__ d_mask, int8_t* __restrict__ dim_s) {
  const uint64_t nmask = *d_mask;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n_supp; i += stride) {
    const int32_t n = s_nationkey[i];
    dim_s[i] = nation_ok(nmask, n) ? static_cast<int8_t>(n) : static_cast<int8_t>(-1);
  }
}

// 4-bit codes of the supplier nations for the line pass: code c < 15 is the
// c-th nation of the region's mask, 15 none.  Exact when the region has at
// most 15 nations; the line pass checks that before it uses them.
__global__ void q5_supplier_nib_kernel(const int8_t* __restrict__ dim_s, int64_t n_supp,
                                       const unsigned long long* __restrict__ d_mask, uint8_t* __restrict__ nib) {
  const uint64_t nmask = *d_mask;
  auto code = [&](int32_t n) -> uint32_t {
    if (n < 0) return 15u;
    const uint32_t c = static_cast<uint32_t>(__popcll(nmask & ((1ull << n) - 1ull)));
    return c < 15u ? c : 15u;
  };
  const int64_t nbytes = (n_supp + 1) >> 1;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < nbytes; i += stride) {
    const uint32_t lo = code(dim_s[2 * i]);
    const uint32_t hi = 2 * i + 1 < n_supp ? code(dim_s[2 * i + 1]) : 15u;
    nib[i] = static_cast<uint8_t>(lo | (hi << 4));
  }
}

__global__ void q5_orders_kernel(const int32_t* __restrict__ o_custkey, const int32_t* __restrict__ o_orderdate,
                                 int64_t n_orders, const int32_t* __restrict__ c_nationkey, int64_t n_cust,
                                 const unsigned long long* __restrict__ d_mask, int32_t date1, int32_t date2,
                                 int8_t* __restrict__ dim_o, unsigned long long* range_err) {
  const uint64_t nmask = *d_mask;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  const int64_t t0 = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const uint64_t pol = policy_evict_first();
  unsigned int bad = 0;
  auto one = [&](int64_t i, int32_t d, int32_t c) {
    int8_t v = -1;
    if (d >= date1 && d < date2) {
      if (c < 1 || c > n_cust) {
        ++bad;
      } else {
        const int32_t n = __ldg(c_nationkey + (c - 1));
        if (nation_ok(nmask, n)) v = static_cast<int8_t>(n);
      }
    }
    dim_o[i] = v;
  };
  // 4 orders per thread (16-byte loads; their customer gathers together)
  const bool vec = ((reinterpret_cast<uintptr_t>(o_custkey) | reinterpret_cast<uintptr_t>(o_orderdate) |
                     reinterpret_cast<uintptr_t>(dim_o)) & 15) == 0;
  const int64_t n4 = vec ? n_orders >> 2 : 0;
  for (int64_t i = t0; i < n4; i += stride) {
    const int4 dv = ld_stream_v4(o_orderdate + 4 * i, pol), cv = ld_stream_v4(o_custkey + 4 * i, pol);
    const int32_t d[4] = {dv.x, dv.y, dv.z, dv.w}, c[4] = {cv.x, cv.y, cv.z, cv.w};
    int32_t n[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const bool want = d[e] >= date1 && d[e] < date2;
      const bool okc = c[e] >= 1 && c[e] <= n_cust;
      bad += want && !okc;
      n[e] = (want && okc) ? __ldg(c_nationkey + (c[e] - 1)) : -1;
    }
    uint32_t packed = 0;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int8_t v = (n[e] >= 0 && nation_ok(nmask, n[e])) ? static_cast<int8_t>(n[e]) : static_cast<int8_t>(-1);
      packed |= static_cast<uint32_t>(static_cast<uint8_t>(v)) << (8 * e);
    }
    reinterpret_cast<uint32_t*>(dim_o)[i] = packed;
  }
  for (int64_t i = 4 * n4 + t0; i < n_orders; i += stride) one(i, o_orderdate[i], o_custkey[i]);
  if (bad) atomicAdd(range_err, static_cast<unsigned long long>(bad));
}

// stage_s: 0 probes the int8 supplier vector through L1/L2; 2 stages the
// 4-bit codes in shared memory (half the bytes of the int8 vector, so more
// blocks fit an SM), and falls back to 0 when the region has more than 15
// nations.
__global__ void __launch_bounds__(512, 3) q5_lines_kernel(const int32_t* __restrict__ l_suppkey,
                                                       const int32_t* __restrict__ l_order,
                                                       const int32_t* __restrict__ price,
                                                       const int32_t* __restrict__ disc, int64_t n_lines,
                                                       const int8_t* __restrict__ dim_s, int64_t n_supp,
                                                       const uint8_t* __restrict__ nib_s,
                                                       const unsigned long long* __restrict__ d_mask,
                                                       const int8_t* __restrict__ dim_o, int64_t n_orders,
                                                       unsigned long long* __restrict__ sums,
                                                       unsigned long long* range_err, int stage_s) {
  extern __shared__ int8_t s_dim[];  // staged supplier nations or their 4-bit codes (stage_s)
  __shared__ unsigned long long s_sum[kQ5MaxNations];
  __shared__ int8_t s_nat[16];       // 4-bit code -> nation
  const int tid = threadIdx.x;
  const uint64_t nmask = stage_s == 2 ? *d_mask : 0ull;
  const int mode = stage_s == 2 && __popcll(nmask) > 15 ? 0 : stage_s;
  for (int i = tid; i < kQ5MaxNations; i += blockDim.x) s_sum[i] = 0;
  if (mode == 2 && tid < 16) {
    // the tid-th set bit of the mask
    uint64_t m = nmask;
    for (int k = 0; k < tid && m; ++k) m &= m - 1;
    s_nat[tid] = m ? static_cast<int8_t>(__ffsll(static_cast<long long>(m)) - 1) : static_cast<int8_t>(-1);
  }
  if (mode == 2)
    for (int64_t i = tid; i < ((n_supp + 1) >> 1); i += blockDim.x) s_dim[i] = static_cast<int8_t>(nib_s[i]);
  __syncthreads();
  // nation of supplier row s (0-based), -1 when it is not in the region
  auto snation = [&](int32_t s) -> int32_t {
    if (mode == 2) {
      const uint32_t c = (static_cast<uint8_t>(s_dim[s >> 1]) >> ((s & 1) << 2)) & 15u;
      return c == 15u ? -1 : s_nat[c];
    }
    return dim_s[s];
  };
  const uint64_t pol = policy_evict_first();
  const uint64_t keep = policy_evict_last();
  unsigned int bad = 0;
  auto one = [&](int32_t sk, int32_t ok, int32_t p, int32_t dc) {
    const bool in = sk >= 1 && sk <= n_supp && ok >= 0 && ok < n_orders;
    if (!in) {
      ++bad;
      return;
    }
    const int32_t ns = snation(sk - 1);
    if (ns < 0) return;
    const int32_t no = static_cast<int8_t>(ld_probe_s8_if(in, dim_o + ok, keep, -2));
    if (no != ns) return;
    smem_add_u64(&s_sum[ns], static_cast<uint64_t>(static_cast<int64_t>(p) * (100 - dc)));
  };
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  const int64_t t0 = static_cast<int64_t>(blockIdx.x) * blockDim.x + tid;
  const bool vec = ((reinterpret_cast<uintptr_t>(l_suppkey) | reinterpret_cast<uintptr_t>(l_order) |
                     reinterpret_cast<uintptr_t>(price) | reinterpret_cast<uintptr_t>(disc)) & 15) == 0;
  const int64_t n4 = vec ? n_lines >> 2 : 0;
  for (int64_t i = t0; i < n4; i += stride) {
    const int4 a = ld_stream_v4(l_suppkey + 4 * i, pol), b = ld_stream_v4(l_order + 4 * i, pol);
    const int4 c = ld_stream_v4(price + 4 * i, pol), d = ld_stream_v4(disc + 4 * i, pol);
    // The four lines in stages, so that their order-vector gathers are in
    // flight together: supplier nation, then order nation, then the sums.
    const int32_t sk[4] = {a.x, a.y, a.z, a.w}, ok[4] = {b.x, b.y, b.z, b.w};
    const int32_t pr[4] = {c.x, c.y, c.z, c.w}, dc[4] = {d.x, d.y, d.z, d.w};
    int32_t ns[4], no[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      ns[e] = -1;
      if (sk[e] < 1 || sk[e] > n_supp || ok[e] < 0 || ok[e] >= n_orders) ++bad;
      else ns[e] = snation(sk[e] - 1);
    }
#pragma unroll
    for (int e = 0; e < 4; ++e) no[e] = static_cast<int8_t>(ld_probe_s8_if(ns[e] >= 0, dim_o + ok[e], keep, -2));
#pragma unroll
    for (int e = 0; e < 4; ++e)
      if (ns[e] >= 0 && no[e] == ns[e])
        smem_add_u64(&s_sum[ns[e]], static_cast<uint64_t>(static_cast<int64_t>(pr[e]) * (100 - dc[e])));
  }
  for (int64_t r = 4 * n4 + t0; r < n_lines; r += stride) one(l_suppkey[r], l_order[r], price[r], disc[r]);
  const unsigned int wbad = __reduce_add_sync(0xffffffffu, bad);
  if ((tid & 31) == 0 && wbad) atomicAdd(range_err, static_cast<unsigned long long>(wbad));
  __syncthreads();
  for (int i = tid; i < kQ5MaxNations; i += blockDim.x)
    if (s_sum[i]) atomicAdd(&sums[i], s_sum[i]);
}

// ---- batched: one pass over orders and lineitem for up to 64 queries ------
//
// A line counts for query q exactly when its supplier's nation equals its
// order's customer nation n, n's region has key region_q, and the order date
// lies in [date1_q, date2_q).  So the batch keeps, per nation, the mask of
// queries whose region holds it (nat_q) and, per date of the queries' span,
// the mask of queries whose range holds it (date_q).  The supplier vector
// keeps nations some query wants, the order vector keeps the customer nation
// of orders some query wants (nat_q & date_q != 0), and a line whose two
// nations agree adds its value to sums[q][n] for every q in nat_q[n] &
// date_q[date].  Each query's result is the single-query chain's bit for bit.

constexpr int kQ5DateTable = 8192;  // dates per mask table (64 KB)

struct Q5BatchDesc {
  int32_t region[kQ5MaxNations], d1[kQ5MaxNations], d2[kQ5MaxNations];
  int32_t n_q;
  int32_t dlo, span;  // date table covers [dlo, dlo + span); span 0: no table
};

__device__ __forceinline__ uint64_t q5_date_mask(const Q5BatchDesc& D, const unsigned long long* tab, int32_t d) {
  if (D.span > 0) {
    const uint32_t k = static_cast<uint32_t>(d - D.dlo);
    return k < static_cast<uint32_t>(D.span) ? tab[k] : 0ull;
  }
  uint64_t m = 0;
  for (int q = 0; q < D.n_q; ++q) m |= static_cast<uint64_t>(d >= D.d1[q] && d < D.d2[q]) << q;
  return m;
}

// nat_q[n] for every nation and the date table, in global scratch.
__global__ void q5b_prep_kernel(const int32_t* __restrict__ r_regionkey, int64_t n_region,
                                const int32_t* __restrict__ n_regionkey, int64_t n_nation, Q5BatchDesc D,
                                unsigned long long* __restrict__ nat_q, unsigned long long* __restrict__ date_q) {
  const int64_t tid = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (tid < kQ5MaxNations) {
    uint64_t m = 0;
    const int n = static_cast<int>(tid);
    if (n < n_nation && n_regionkey[n] >= 0 && n_regionkey[n] < n_region) {
      const int32_t key = r_regionkey[n_regionkey[n]];
      for (int q = 0; q < D.n_q; ++q) m |= static_cast<uint64_t>(key == D.region[q]) << q;
    }
    nat_q[n] = m;
  }
  for (int64_t k = tid; k < D.span; k += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int32_t d = D.dlo + static_cast<int32_t>(k);
    uint64_t m = 0;
    for (int q = 0; q < D.n_q; ++q) m |= static_cast<uint64_t>(d >= D.d1[q] && d < D.d2[q]) << q;
    date_q[k] = m;
  }
}

__global__ void q5b_supplier_kernel(const int32_t* __restrict__ s_nationkey, int64_t n_supp,
                                    const unsigned long long* __restrict__ nat_q, int8_t* __restrict__ dim_s) {
  __shared__ unsigned long long s_nat[kQ5MaxNations];
  if (threadIdx.x < kQ5MaxNations) s_nat[threadIdx.x] = nat_q[threadIdx.x];
  __syncthreads();
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n_supp; i += stride) {
    const int32_t n = s_nationkey[i];
    const bool ok = static_cast<uint32_t>(n) < kQ5MaxNations && s_nat[n] != 0;
    dim_s[i] = ok ? static_cast<int8_t>(n) : static_cast<int8_t>(-1);
  }
}

__global__ void q5b_orders_kernel(const int32_t* __restrict__ o_custkey, const int32_t* __restrict__ o_orderdate,
                                  int64_t n_orders, const int32_t* __restrict__ c_nationkey, int64_t n_cust,
                                  const unsigned long long* __restrict__ nat_q,
                                  const unsigned long long* __restrict__ date_q, Q5BatchDesc D,
                                  int8_t* __restrict__ dim_o, unsigned long long* range_err) {
  extern __shared__ unsigned long long s_date[];
  __shared__ unsigned long long s_nat[kQ5MaxNations];
  if (threadIdx.x < kQ5MaxNations) s_nat[threadIdx.x] = nat_q[threadIdx.x];
  for (int k = threadIdx.x; k < D.span; k += blockDim.x) s_date[k] = date_q[k];
  __syncthreads();
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  const uint64_t pol = policy_evict_first();
  unsigned int bad = 0;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n_orders; i += stride) {
    const int32_t d = ld_stream_s32(o_orderdate + i, pol);
    const int32_t c = ld_stream_s32(o_custkey + i, pol);
    int8_t v = -1;
    const uint64_t dm = q5_date_mask(D, s_date, d);
    if (dm) {
      if (c < 1 || c > n_cust) {
        ++bad;
      } else {
        const int32_t n = __ldg(c_nationkey + (c - 1));
        if (static_cast<uint32_t>(n) < kQ5MaxNations && (s_nat[n] & dm)) v = static_cast<int8_t>(n);
      }
    }
    dim_o[i] = v;
  }
  if (bad) atomicAdd(range_err, static_cast<unsigned long long>(bad));
}

// Shared memory: [date table: span x 8][sums: n_q x n_nation x 8][supplier nations].
__global__ void __launch_bounds__(1024, 1) q5b_lines_kernel(
    const int32_t* __restrict__ l_suppkey, const int32_t* __restrict__ l_order, const int32_t* __restrict__ price,
    const int32_t* __restrict__ disc, int64_t n_lines, const int8_t* __restrict__ dim_s, int64_t n_supp,
    const int8_t* __restrict__ dim_o, const int32_t* __restrict__ o_orderdate, int64_t n_orders,
    const unsigned long long* __restrict__ nat_q, const unsigned long long* __restrict__ date_q, Q5BatchDesc D,
    int n_nation, unsigned long long* __restrict__ sums, unsigned long long* range_err, int stage_s) {
  extern __shared__ __align__(16) unsigned char q5b_smem[];
  unsigned long long* s_date = reinterpret_cast<unsigned long long*>(q5b_smem);
  unsigned long long* s_sum = s_date + D.span;
  int8_t* s_dim = reinterpret_cast<int8_t*>(s_sum + D.n_q * n_nation);
  __shared__ unsigned long long s_nat[kQ5MaxNations];
  const int tid = threadIdx.x;
  if (tid < kQ5MaxNations) s_nat[tid] = nat_q[tid];
  for (int k = tid; k < D.span; k += blockDim.x) s_date[k] = date_q[k];
  for (int k = tid; k < D.n_q * n_nation; k += blockDim.x) s_sum[k] = 0;
  if (stage_s)
    for (int64_t i = tid; i < n_supp; i += blockDim.x) s_dim[i] = dim_s[i];
  __syncthreads();
  const uint64_t pol = policy_evict_first();
  const uint64_t keep = policy_evict_last();
  unsigned int bad = 0;
  auto one = [&](int32_t sk, int32_t ok, int32_t p, int32_t dc) {
    const bool in = sk >= 1 && sk <= n_supp && ok >= 0 && ok < n_orders;
    if (!in) {
      ++bad;
      return;
    }
    const int32_t ns = stage_s ? s_dim[sk - 1] : dim_s[sk - 1];
    if (ns < 0) return;
    const int32_t no = static_cast<int8_t>(ld_probe_s8_if(in, dim_o + ok, keep, -2));
    if (no != ns) return;
    uint64_t m = s_nat[ns] & q5_date_mask(D, s_date, __ldg(o_orderdate + ok));
    const uint64_t v = static_cast<uint64_t>(static_cast<int64_t>(p) * (100 - dc));
    while (m) {
      const int q = __ffsll(static_cast<long long>(m)) - 1;
      m &= m - 1;
      smem_add_u64(&s_sum[q * n_nation + ns], v);
    }
  };
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  const int64_t t0 = static_cast<int64_t>(blockIdx.x) * blockDim.x + tid;
  const bool vec = ((reinterpret_cast<uintptr_t>(l_suppkey) | reinterpret_cast<uintptr_t>(l_order) |
                     reinterpret_cast<uintptr_t>(price) | reinterpret_cast<uintptr_t>(disc)) & 15) == 0;
  const int64_t n4 = vec ? n_lines >> 2 : 0;
  for (int64_t i = t0; i < n4; i += stride) {
    const int4 a = ld_stream_v4(l_suppkey + 4 * i, pol), b = ld_stream_v4(l_order + 4 * i, pol);
    const int4 c = ld_stream_v4(price + 4 * i, pol), d = ld_stream_v4(disc + 4 * i, pol);
    // Stages over the four lines (gathers of a stage in flight together):
    // supplier nation, order nation, order date of the matches, the sums.
    const int32_t sk[4] = {a.x, a.y, a.z, a.w}, ok[4] = {b.x, b.y, b.z, b.w};
    const int32_t pr[4] = {c.x, c.y, c.z, c.w}, dc[4] = {d.x, d.y, d.z, d.w};
    int32_t ns[4], no[4], dt[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      ns[e] = -1;
      if (sk[e] < 1 || sk[e] > n_supp || ok[e] < 0 || ok[e] >= n_orders) ++bad;
      else ns[e] = stage_s ? s_dim[sk[e] - 1] : dim_s[sk[e] - 1];
    }
#pragma unroll
    for (int e = 0; e < 4; ++e) no[e] = static_cast<int8_t>(ld_probe_s8_if(ns[e] >= 0, dim_o + ok[e], keep, -2));
#pragma unroll
    for (int e = 0; e < 4; ++e) dt[e] = (ns[e] >= 0 && no[e] == ns[e]) ? __ldg(o_orderdate + ok[e]) : 0;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      if (ns[e] < 0 || no[e] != ns[e]) continue;
      uint64_t m = s_nat[ns[e]] & q5_date_mask(D, s_date, dt[e]);
      const uint64_t v = static_cast<uint64_t>(static_cast<int64_t>(pr[e]) * (100 - dc[e]));
      while (m) {
        const int q = __ffsll(static_cast<long long>(m)) - 1;
        m &= m - 1;
        smem_add_u64(&s_sum[q * n_nation + ns[e]], v);
      }
    }
  }
  for (int64_t r = 4 * n4 + t0; r < n_lines; r += stride) one(l_suppkey[r], l_order[r], price[r], disc[r]);
  const unsigned int wbad = __reduce_add_sync(0xffffffffu, bad);
  if ((tid & 31) == 0 && wbad) atomicAdd(range_err, static_cast<unsigned long long>(wbad));
  __syncthreads();
  for (int k = tid; k < D.n_q * n_nation; k += blockDim.x)
    if (s_sum[k]) atomicAdd(&sums[k], s_sum[k]);
}

static unsigned grid_q5(const olap_ctx* ctx, int64_t n, int threads) {
  int64_t g = (n + threads - 1) / threads;
  const int64_t cap = static_cast<int64_t>(ctx->sm_count) * (2048 / threads);
  if (g > cap) g = cap;
  return static_cast<unsigned>(g < 1 ? 1 : g);
}

}  // namespace olap

extern "C" {

int olap_q5_chain(olap_ctx* ctx, const olap_q5_tables* t, int32_t region, int32_t date1, int32_t date2,
                  int64_t* nation_sums) {
  if (!ctx || !t) return OLAP_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  OLAP_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  OLAP_REQUIRE(ctx, nation_sums, "null output");
  OLAP_REQUIRE(ctx, t->n_region >= 1 && t->n_nation >= 1 && t->n_nation <= olap::kQ5MaxNations,
               "1..64 nations");
  OLAP_REQUIRE(ctx, t->n_supp >= 0 && t->n_cust >= 0 && t->n_orders >= 0 && t->n_lines >= 0, "bad sizes");
  OLAP_REQUIRE(ctx, t->r_regionkey && t->n_regionkey, "null region or nation table");
  OLAP_REQUIRE(ctx, t->n_supp == 0 || t->s_nationkey, "null s_nationkey");
  OLAP_REQUIRE(ctx, t->n_cust == 0 || t->c_nationkey, "null c_nationkey");
  OLAP_REQUIRE(ctx, t->n_orders == 0 || (t->o_custkey && t->o_orderdate), "null orders column");
  OLAP_REQUIRE(ctx, t->n_lines == 0 || (t->l_suppkey && t->l_orderkey && t->l_price && t->l_discount),
               "null lineitem column");
  olap::Arena ar(ctx);
  int8_t* dim_s = ar.take<int8_t>(static_cast<size_t>(t->n_supp > 0 ? t->n_supp : 1));
  uint8_t* nib_s = ar.take<uint8_t>(static_cast<size_t>(t->n_supp > 0 ? (t->n_supp + 1) / 2 : 1));
  int8_t* dim_o = ar.take<int8_t>(static_cast<size_t>(t->n_orders > 0 ? t->n_orders : 1));
  unsigned long long* nmask = ar.take<unsigned long long>(1);
  if (!dim_s || !nib_s || !dim_o || !nmask)
    return olap::set_error(ctx, OLAP_ERR_CAPACITY, "scratch arena too small for Q5 vectors");
  olap::q5_nation_mask_kernel<<<1, 64, 0, ctx->stream>>>(t->r_regionkey, t->n_region, t->n_regionkey, t->n_nation,
                                                        region, nmask);
  OLAP_CUDA_TRY(ctx, cudaMemsetAsync(nation_sums, 0, sizeof(int64_t) * t->n_nation, ctx->stream));
  if (t->n_supp)
    olap::q5_supplier_kernel<<<olap::grid_q5(ctx, t->n_supp, 256), 256, 0, ctx->stream>>>(t->s_nationkey, t->n_supp,
                                                                                         nmask, dim_s);
  if (t->n_orders)
    olap::q5_orders_kernel<<<olap::grid_q5(ctx, t->n_orders, 256), 256, 0, ctx->stream>>>(
        t->o_custkey, t->o_orderdate, t->n_orders, t->c_nationkey, t->n_cust, nmask, date1, date2, dim_o,
        &ctx->counters->range_errors);
  // Supplier nations in shared memory as 4-bit codes when they fit (160 KB).
  const int stage = t->n_lines && t->n_supp > 0 && (t->n_supp + 1) / 2 <= 160 * 1024 ? 2 : 0;
  if (stage == 2)
    olap::q5_supplier_nib_kernel<<<olap::grid_q5(ctx, (t->n_supp + 1) / 2, 256), 256, 0, ctx->stream>>>(
        dim_s, t->n_supp, nmask, nib_s);
  if (t->n_lines) {
    const size_t smem = stage == 2 ? static_cast<size_t>(((t->n_supp + 1) / 2 + 15) & ~int64_t(15)) : 0;
    if (smem > 48 * 1024)
      OLAP_CUDA_TRY(ctx, cudaFuncSetAttribute(olap::q5_lines_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              static_cast<int>(smem)));
    int bps = 1;
    OLAP_CUDA_TRY(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, olap::q5_lines_kernel, 512, smem));
    int64_t grid = static_cast<int64_t>(ctx->sm_count) * (bps < 1 ? 1 : bps);
    grid = std::min<int64_t>(grid, (t->n_lines / 4 + 511) / 512 + 1);
    olap::q5_lines_kernel<<<static_cast<unsigned>(grid), 512, smem, ctx->stream>>>(
        t->l_suppkey, t->l_orderkey, t->l_price, t->l_discount, t->n_lines, dim_s, t->n_supp, nib_s, nmask, dim_o,
        t->n_orders, reinterpret_cast<unsigned long long*>(nation_sums), &ctx->counters->range_errors, stage);
  }
  OLAP_CUDA_TRY(ctx, cudaGetLastError());
  return OLAP_OK;
}

int olap_q5_batch(olap_ctx* ctx, const olap_q5_tables* t, const olap_q5_query* queries, int n_queries,
                  int64_t* nation_sums) {
  if (!ctx || !t) return OLAP_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  OLAP_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  OLAP_REQUIRE(ctx, nation_sums && queries, "null output or query list");
  OLAP_REQUIRE(ctx, n_queries >= 1 && n_queries <= OLAP_Q5_MAX_BATCH, "1..64 queries per batch");
  OLAP_REQUIRE(ctx, t->n_region >= 1 && t->n_nation >= 1 && t->n_nation <= olap::kQ5MaxNations,
               "1..64 nations");
  OLAP_REQUIRE(ctx, t->n_supp >= 0 && t->n_cust >= 0 && t->n_orders >= 0 && t->n_lines >= 0, "bad sizes");
  OLAP_REQUIRE(ctx, t->r_regionkey && t->n_regionkey, "null region or nation table");
  OLAP_REQUIRE(ctx, t->n_supp == 0 || t->s_nationkey, "null s_nationkey");
  OLAP_REQUIRE(ctx, t->n_cust == 0 || t->c_nationkey, "null c_nationkey");
  OLAP_REQUIRE(ctx, t->n_orders == 0 || (t->o_custkey && t->o_orderdate), "null orders column");
  OLAP_REQUIRE(ctx, t->n_lines == 0 || (t->l_suppkey && t->l_orderkey && t->l_price && t->l_discount),
               "null lineitem column");
  olap::Q5BatchDesc D;
  std::memset(&D, 0, sizeof(D));
  D.n_q = n_queries;
  int64_t lo = INT64_MAX, hi = INT64_MIN;
  for (int q = 0; q < n_queries; ++q) {
    D.region[q] = queries[q].region;
    D.d1[q] = queries[q].date1;
    D.d2[q] = queries[q].date2;
    if (queries[q].date1 < queries[q].date2) {
      lo = std::min<int64_t>(lo, queries[q].date1);
      hi = std::max<int64_t>(hi, queries[q].date2);
    }
  }
  // every date range empty: span 1 at an arbitrary date, its mask 0
  if (lo > hi) lo = hi = 0;
  D.dlo = static_cast<int32_t>(lo);
  D.span = hi - lo <= olap::kQ5DateTable ? static_cast<int32_t>(hi - lo > 0 ? hi - lo : 1) : 0;
  olap::Arena ar(ctx);
  int8_t* dim_s = ar.take<int8_t>(static_cast<size_t>(t->n_supp > 0 ? t->n_supp : 1));
  int8_t* dim_o = ar.take<int8_t>(static_cast<size_t>(t->n_orders > 0 ? t->n_orders : 1));
  unsigned long long* nat_q = ar.take<unsigned long long>(olap::kQ5MaxNations);
  unsigned long long* date_q = ar.take<unsigned long long>(olap::kQ5DateTable);
  if (!dim_s || !dim_o || !nat_q || !date_q)
    return olap::set_error(ctx, OLAP_ERR_CAPACITY, "scratch arena too small for Q5 vectors");
  const size_t out_bytes = sizeof(int64_t) * static_cast<size_t>(n_queries) * t->n_nation;
  OLAP_CUDA_TRY(ctx, cudaMemsetAsync(nation_sums, 0, out_bytes, ctx->stream));
  olap::q5b_prep_kernel<<<8, 256, 0, ctx->stream>>>(t->r_regionkey, t->n_region, t->n_regionkey, t->n_nation, D,
                                                    nat_q, date_q);
  if (t->n_supp)
    olap::q5b_supplier_kernel<<<olap::grid_q5(ctx, t->n_supp, 256), 256, 0, ctx->stream>>>(t->s_nationkey,
                                                                                          t->n_supp, nat_q, dim_s);
  const size_t date_bytes = sizeof(unsigned long long) * static_cast<size_t>(D.span);
  if (t->n_orders) {
    if (date_bytes > 48 * 1024)
      OLAP_CUDA_TRY(ctx, cudaFuncSetAttribute(olap::q5b_orders_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              static_cast<int>(date_bytes)));
    olap::q5b_orders_kernel<<<olap::grid_q5(ctx, t->n_orders, 256), 256, date_bytes, ctx->stream>>>(
        t->o_custkey, t->o_orderdate, t->n_orders, t->c_nationkey, t->n_cust, nat_q, date_q, D, dim_o,
        &ctx->counters->range_errors);
  }
  if (t->n_lines) {
    const size_t fixed = date_bytes + out_bytes;
    const size_t stage_bytes = static_cast<size_t>((t->n_supp + 15) & ~int64_t(15));
    const size_t budget = static_cast<size_t>(ctx->smem_optin) - 2048;  // static shared + headroom
    const bool stage = fixed + stage_bytes <= budget;
    const size_t smem = fixed + (stage ? stage_bytes : 0);
    if (smem > 48 * 1024)
      OLAP_CUDA_TRY(ctx, cudaFuncSetAttribute(olap::q5b_lines_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              static_cast<int>(smem)));
    int bps = 1;
    OLAP_CUDA_TRY(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, olap::q5b_lines_kernel, 1024, smem));
    int64_t grid = static_cast<int64_t>(ctx->sm_count) * (bps < 1 ? 1 : bps);
    grid = std::min<int64_t>(grid, (t->n_lines / 4 + 1023) / 1024 + 1);
    olap::q5b_lines_kernel<<<static_cast<unsigned>(grid), 1024, smem, ctx->stream>>>(
        t->l_suppkey, t->l_orderkey, t->l_price, t->l_discount, t->n_lines, dim_s, t->n_supp, dim_o, t->o_orderdate,
        t->n_orders, nat_q, date_q, D, static_cast<int>(t->n_nation),
        reinterpret_cast<unsigned long long*>(nation_sums), &ctx->counters->range_errors, stage ? 1 : 0);
  }
  OLAP_CUDA_TRY(ctx, cudaGetLastError());
  return OLAP_OK;
}

}  // extern "C"
