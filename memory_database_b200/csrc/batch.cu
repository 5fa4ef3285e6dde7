// Dimension-vector builder and the batched multi-query star-join.
//
// The reference bakes each query's dimension vectors in its generator
// (include/gendata_util.hpp:449-542): entry k of table t is a group code when
// the dimension row passes the query's filter, else DIM_NULL.  Here dimension
// tables keep their attributes instead — an int32 filter attribute and an
// int32 group attribute per dimension row — and a query's predicate on a
// table is a range [lo, hi) on the filter attribute; its group code is the
// group attribute (or 0 when the table is not a group dimension).
//
// olap_build_dimvec materialises one query's int8 dimension vector from those
// attributes (the input of the plain star-join).
//
// The batched path runs up to 64 such queries in one persistent pass over
// the shared fact table, in two kernels:
//  * per dimension row, a 64-bit mask of the queries whose predicate the row
//    passes (a query that does not use the table passes every row), next to
//    the row's group attribute: a 16-byte record, 74 MB for the four
//    headline tables, kept hot in L2;
//  * over the fact rows: each row's record is probed once per table (only
//    while some live query still uses the table), the masks are ANDed with
//    the mask of the queries whose fact range covers the row, and only the
//    queries left in the mask do per-query work (group id, one int64 atomic).
// Per query the result is bit-identical to the plain star-join over the
// dimension vectors that olap_build_dimvec builds for it.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "olap_internal.cuh"

namespace olap {

// Packed dimension attribute record: filter attribute (low word) and group
// attribute (high word).
__global__ void pack_dim_attrs_kernel(const int32_t* __restrict__ filt, const int32_t* __restrict__ grp,
                                      int64_t n, int2* __restrict__ out) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
    out[i] = make_int2(filt[i], grp ? grp[i] : 0);
}

__global__ void build_dimvec_kernel(const int32_t* __restrict__ filt, const int32_t* __restrict__ grp, int64_t n,
                                    int32_t lo, int32_t hi, int use_group, int8_t* __restrict__ out,
                                    unsigned long long* range_err) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  unsigned int bad = 0;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
    const int32_t f = filt[i];
    int8_t v = static_cast<int8_t>(OLAP_DIM_NULL);
    if (f >= lo && f < hi) {
      const int32_t g = use_group ? grp[i] : 0;
      if (g < 0 || g >= OLAP_DIM_NULL) ++bad;  // not representable as a code
      else v = static_cast<int8_t>(g);
    }
    out[i] = v;
  }
  if (bad) atomicAdd(range_err, static_cast<unsigned long long>(bad));
}

// Device-side query descriptor of the batched kernel (one per query).
struct BatchQuery {
  int64_t row_begin, row_end;
  int32_t lo[OLAP_MAX_DIMS];      // filter range [lo, hi) per table
  int32_t hi[OLAP_MAX_DIMS];
  int32_t factor[OLAP_MAX_DIMS];  // group weight per table (0: not a group dimension)
  int32_t uses;                   // bit t: table t participates
  int32_t grouped;                // bit t: table t contributes its group attribute
  int64_t group_nums;
  int64_t out_offset;             // first slot of this query in the shared output
  int32_t smem_off;               // first slot of its per-block accumulators, or -1
  int32_t pad;
};

constexpr int kMaxBatchQueries = 64;
constexpr int kBatchSmemSlots = 4096;  // default per-block int64 accumulators (32 KiB); tunable
constexpr int kMaxSegments = 2 * kMaxBatchQueries + 2;

// Everything a batch uploads (one pinned staging copy per slot).
struct BatchDesc {
  BatchQuery q[kMaxBatchQueries];
  int64_t seg_begin[kMaxSegments];             // sorted; segment s = [seg_begin[s], seg_begin[s+1])
  unsigned long long seg_mask[kMaxSegments];   // queries whose fact range covers segment s
  unsigned long long uses_mask[OLAP_MAX_DIMS]; // queries using table t
  unsigned long long* out;                     // concatenated group vectors
  unsigned long long* totals;                  // [n_queries]
  int64_t out_total;                           // slots of out in use
  int32_t n_queries;
  int32_t n_seg;
};

struct DimRecord {
  unsigned long long mask;  // bit q: the row passes query q's predicate on this table
  int32_t grp;              // group attribute
  int32_t pad;
};

struct BatchParams {
  const int2* attrs[OLAP_MAX_DIMS];   // packed attribute records per table
  DimRecord* rec[OLAP_MAX_DIMS];      // per-batch query masks per table
  uint32_t dim_len[OLAP_MAX_DIMS];
  const int32_t* fk[OLAP_MAX_DIMS];
  const int32_t* m1;
  const int32_t* m2;
  int64_t n_rows;
  const BatchDesc* desc;
  int32_t tables_used;                // union of the queries' `uses`
  int32_t probe_order;                // 4 x 2-bit table ids, smallest table first
  int32_t agg;                        // OLAP_AGG_* of every query (one aggregate)
  int32_t smem_slots;                 // per-block shared accumulators (dynamic shared memory)
  int32_t block;                      // threads per block of the scan (part of a recorded graph)
  unsigned long long* range_err;
};

constexpr int kBatchThreads = 512;     // default block size; tunable (128..1024)
constexpr int kBatchMaxThreads = 1024;
constexpr int kBatchMaxSmemSlots = 24576;  // 192 KiB

__device__ __forceinline__ int64_t batch_value(int agg, int32_t x, int32_t y) {
  switch (agg) {
    case OLAP_AGG_M1_PLUS_M2: return static_cast<int64_t>(x) + y;
    case OLAP_AGG_M1: return x;
    case OLAP_AGG_M2: return y;
    case OLAP_AGG_M1_TIMES_M2: return static_cast<int64_t>(x) * y;
    default: return 1;
  }
}

// Query masks of the rows of table t.
__global__ void __launch_bounds__(256) batch_records_kernel(const BatchParams p, int t) {
  __shared__ int32_t slo[kMaxBatchQueries], shi[kMaxBatchQueries];
  __shared__ unsigned long long s_uses, s_grouped;
  const BatchDesc& D = *p.desc;
  const int nq = D.n_queries;
  if (threadIdx.x == 0) {
    unsigned long long u = 0, g = 0;
    for (int q = 0; q < nq; ++q) {
      if ((D.q[q].uses >> t) & 1) u |= 1ull << q;
      if ((D.q[q].grouped >> t) & 1) g |= 1ull << q;
    }
    s_uses = u;
    s_grouped = g;
  }
  for (int q = threadIdx.x; q < nq; q += blockDim.x) {
    slo[q] = D.q[q].lo[t];
    shi[q] = D.q[q].hi[t];
  }
  __syncthreads();
  const unsigned long long uses = s_uses, grouped = s_grouped;
  const unsigned long long all = nq == 64 ? ~0ull : ((1ull << nq) - 1);
  const int64_t n = p.dim_len[t];
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t k = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; k < n; k += stride) {
    const int2 a = p.attrs[t][k];
    // a group value that is not an int8 code is DIM_NULL in the dimension
    // vector the plain path builds
    const bool code_ok = static_cast<uint32_t>(a.y) < static_cast<uint32_t>(OLAP_DIM_NULL);
    unsigned long long m = all & ~uses;
    for (int q = 0; q < nq; ++q) {
      const bool pass = a.x >= slo[q] && a.x < shi[q] && (code_ok || !((grouped >> q) & 1));
      m |= static_cast<unsigned long long>(pass && ((uses >> q) & 1)) << q;
    }
    DimRecord r;
    r.mask = m;
    r.grp = a.y;
    r.pad = 0;
    reinterpret_cast<ulonglong2*>(p.rec[t])[k] = make_ulonglong2(r.mask, static_cast<uint32_t>(r.grp));
  }
}

// Record loads.  They are asm without `volatile`, which the compiler may
// execute where their guard does not hold, so the callers pass the record of
// key 0 (every table has at least one) in place of a key out of range.
__device__ __forceinline__ ulonglong2 ld_record(const DimRecord* r, uint64_t pol) {
  ulonglong2 v;
  asm("ld.global.nc.L2::cache_hint.v2.u64 {%0,%1}, [%2], %3;" : "=l"(v.x), "=l"(v.y) : "l"(r), "l"(pol));
  return v;
}
__device__ __forceinline__ unsigned long long ld_record_mask(const DimRecord* r, uint64_t pol) {
  unsigned long long v;
  asm("ld.global.nc.L2::cache_hint.u64 %0, [%1], %2;" : "=l"(v) : "l"(r), "l"(pol));
  return v;
}
__device__ __forceinline__ int32_t ld_record_grp(const DimRecord* r, uint64_t pol) {
  int32_t v;
  asm("ld.global.nc.L2::cache_hint.s32 %0, [%1], %2;" : "=r"(v) : "l"(&r->grp), "l"(pol));
  return v;
}

// The fact pass: persistent, 4 rows per thread per step (128-bit loads).
// PAR = false: the tables are probed one after another, smallest first, each
// only for the rows that still have a live query using it (up to four
// dependent L2 round trips per step, 16-byte records).  PAR = true: every
// used table's query mask is read in one round trip (the union of a batch's
// predicates passes nearly every row, so the skipped probes save little),
// then the group attributes only of the tables that a surviving query groups
// by; more registers, so at most 512 threads per block.
template <bool PAR>
__global__ void __launch_bounds__(PAR ? 512 : kBatchMaxThreads, 1) batch_scan_kernel(const BatchParams p) {
  __shared__ BatchQuery sq[kMaxBatchQueries];
  __shared__ int64_t sseg[kMaxSegments];
  __shared__ unsigned long long smask[kMaxSegments];
  extern __shared__ unsigned long long sacc[];  // p.smem_slots per-block accumulators
  __shared__ int4 s_qf[kMaxBatchQueries];  // per query: group factor at each probe position (0: not grouped)
  __shared__ int4 s_qi[kMaxBatchQueries];  // per query: {group_nums, smem_off, out_offset lo, hi}
  __shared__ unsigned int s_bad;
  const BatchDesc& D = *p.desc;
  unsigned long long* const out = D.out;
  const int tid = threadIdx.x;
  const int nq = D.n_queries, nseg = D.n_seg;
  // The used tables in probe order (smallest first).
  int tab[OLAP_MAX_DIMS] = {0, 0, 0, 0};
  uint32_t tlen[OLAP_MAX_DIMS] = {0, 0, 0, 0};
  unsigned long long tuses[OLAP_MAX_DIMS] = {0, 0, 0, 0};
  int ntab = 0;
#pragma unroll
  for (int o = 0; o < OLAP_MAX_DIMS; ++o) {
    const int t = (p.probe_order >> (2 * o)) & 3;
    if ((p.tables_used >> t) & 1) {
#pragma unroll
      for (int w = 0; w < OLAP_MAX_DIMS; ++w)
        if (w == ntab) {
          tab[w] = t;
          tlen[w] = p.dim_len[t];
          tuses[w] = D.uses_mask[t];
        }
      ++ntab;
    }
  }
  for (int i = tid; i < nq; i += blockDim.x) {
    const BatchQuery& Q = D.q[i];
    sq[i] = Q;
    int32_t f[OLAP_MAX_DIMS] = {0, 0, 0, 0};
#pragma unroll
    for (int o = 0; o < OLAP_MAX_DIMS; ++o)
      if (o < ntab && ((Q.grouped >> tab[o]) & 1)) f[o] = Q.factor[tab[o]];
    s_qf[i] = make_int4(f[0], f[1], f[2], f[3]);
    s_qi[i] = make_int4(static_cast<int32_t>(Q.group_nums), Q.smem_off, static_cast<int32_t>(Q.out_offset),
                        static_cast<int32_t>(Q.out_offset >> 32));
  }
  for (int i = tid; i < p.smem_slots; i += blockDim.x) sacc[i] = 0ull;
  for (int i = tid; i < nseg; i += blockDim.x) {
    sseg[i] = D.seg_begin[i];
    smask[i] = D.seg_mask[i];
  }
  if (tid == 0) s_bad = 0;
  __syncthreads();
  // queries grouping by the table at each probe position (their factor there is not 0)
  unsigned long long tgrp[OLAP_MAX_DIMS] = {0ull, 0ull, 0ull, 0ull};
  if (PAR) {
    for (int q = 0; q < nq; ++q) {
      const int4 f = s_qf[q];
      tgrp[0] |= static_cast<unsigned long long>(f.x != 0) << q;
      tgrp[1] |= static_cast<unsigned long long>(f.y != 0) << q;
      tgrp[2] |= static_cast<unsigned long long>(f.z != 0) << q;
      tgrp[3] |= static_cast<unsigned long long>(f.w != 0) << q;
    }
  }
  const uint64_t pol_stream = policy_evict_first();
  const uint64_t pol_keep = policy_evict_last();
  const int agg = p.agg;
  const bool need_m1 = agg == OLAP_AGG_M1_PLUS_M2 || agg == OLAP_AGG_M1 || agg == OLAP_AGG_M1_TIMES_M2;
  const bool need_m2 = agg == OLAP_AGG_M1_PLUS_M2 || agg == OLAP_AGG_M2 || agg == OLAP_AGG_M1_TIMES_M2;
  unsigned int bad = 0;
  const int64_t n4 = (p.n_rows + 3) >> 2;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + tid; i < n4; i += stride) {
    const int64_t r0 = 4 * i;
    const int nv = r0 + 4 <= p.n_rows ? 4 : static_cast<int>(p.n_rows - r0);
    const bool full = nv == 4;
    // Arrays are indexed by probe position o (table t = tab[o]), so that
    // every index is a compile-time constant.
    int32_t key[OLAP_MAX_DIMS][4];
    int32_t x[4] = {0, 0, 0, 0}, y[4] = {0, 0, 0, 0};
#pragma unroll
    for (int o = 0; o < OLAP_MAX_DIMS; ++o) {
      if (o >= ntab) continue;
      const int32_t* f = p.fk[tab[o]];
      if (full) {
        const int4 v = ld_stream_v4(f + r0, pol_stream);
        key[o][0] = v.x; key[o][1] = v.y; key[o][2] = v.z; key[o][3] = v.w;
      } else {
        for (int k = 0; k < 4; ++k) key[o][k] = k < nv ? f[r0 + k] : 0;
      }
    }
    if (need_m1) {
      if (full) {
        const int4 v = ld_stream_v4(p.m1 + r0, pol_stream);
        x[0] = v.x; x[1] = v.y; x[2] = v.z; x[3] = v.w;
      } else {
        for (int k = 0; k < nv; ++k) x[k] = p.m1[r0 + k];
      }
    }
    if (need_m2) {
      if (full) {
        const int4 v = ld_stream_v4(p.m2 + r0, pol_stream);
        y[0] = v.x; y[1] = v.y; y[2] = v.z; y[3] = v.w;
      } else {
        for (int k = 0; k < nv; ++k) y[k] = p.m2[r0 + k];
      }
    }
    // Queries whose fact range covers each row: segment of r0 by binary
    // search, later rows step forward.
    int lo = 0, hi = nseg - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (sseg[mid] <= r0) lo = mid; else hi = mid - 1;
    }
    unsigned long long m[4];
    int s = lo;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      while (s + 1 < nseg && sseg[s + 1] <= r0 + k) ++s;
      m[k] = k < nv ? smask[s] : 0ull;
    }
    // A key out of range drops the row for the queries that use the table;
    // the table is not probed for it, and the row counts once per such query
    // when every other table the query uses passes it (as the plain path
    // counts: no in-range key of the query meets its filter's null).
    uint32_t inr = 0;  // bit 4*o + k: key[o][k] in range
#pragma unroll
    for (int k = 0; k < 4; ++k) {
#pragma unroll
      for (int o = 0; o < OLAP_MAX_DIMS; ++o) {
        if (o >= ntab) continue;
        if (static_cast<uint32_t>(key[o][k]) < tlen[o]) inr |= 1u << (4 * o + k);
      }
    }
    // queries that use a table whose key of row k is out of range
    auto oob_queries = [&](int k) -> unsigned long long {
      unsigned long long q = 0;
#pragma unroll
      for (int o = 0; o < OLAP_MAX_DIMS; ++o)
        if (o < ntab && !((inr >> (4 * o + k)) & 1u)) q |= tuses[o];
      return q;
    };
    int32_t gr[OLAP_MAX_DIMS][4] = {};
    if (PAR) {
      // every used table's query mask of the 4 rows in one round trip
      unsigned long long tm[OLAP_MAX_DIMS][4];
#pragma unroll
      for (int o = 0; o < OLAP_MAX_DIMS; ++o) {
        if (o >= ntab) continue;
        const unsigned long long ut = tuses[o];
        const DimRecord* rt = p.rec[tab[o]];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const bool in = (inr >> (4 * o + k)) & 1u;
          tm[o][k] = ((m[k] & ut) && in) ? ld_record_mask(rt + (in ? key[o][k] : 0), pol_keep) : ~0ull;
        }
      }
#pragma unroll
      for (int o = 0; o < OLAP_MAX_DIMS; ++o) {
        if (o >= ntab) continue;
#pragma unroll
        for (int k = 0; k < 4; ++k) m[k] &= tm[o][k];
      }
      // group attributes where a surviving query groups by the table (and
      // its key is in range)
#pragma unroll
      for (int o = 0; o < OLAP_MAX_DIMS; ++o) {
        if (o >= ntab) continue;
        const unsigned long long ug = tgrp[o];
        const DimRecord* rt = p.rec[tab[o]];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const bool in = (inr >> (4 * o + k)) & 1u;
          gr[o][k] = ((m[k] & ug) != 0ull && in) ? ld_record_grp(rt + (in ? key[o][k] : 0), pol_keep) : 0;
        }
      }
    } else {
      // Probe the tables, smallest first, breadth-first across the 4 rows; a
      // table is probed for a row only while a live query of the row uses it.
#pragma unroll
      for (int o = 0; o < OLAP_MAX_DIMS; ++o) {
        if (o >= ntab) continue;
        const unsigned long long ut = tuses[o];
        const DimRecord* rt = p.rec[tab[o]];
        ulonglong2 rec[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const bool in = (inr >> (4 * o + k)) & 1u;
          rec[k] = ((m[k] & ut) && in) ? ld_record(rt + (in ? key[o][k] : 0), pol_keep)
                                       : make_ulonglong2(~0ull, 0ull);
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          m[k] &= rec[k].x;
          gr[o][k] = static_cast<int32_t>(static_cast<uint32_t>(rec[k].y));
        }
      }
    }
    if (inr != (1u << (4 * ntab)) - 1u) {  // rare: some key out of range
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const unsigned long long oq = k < nv ? oob_queries(k) : 0ull;
        bad += __popcll(m[k] & oq);
        m[k] &= ~oq;
      }
    }
    // Per-query work only for the queries left in each row's mask.
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      unsigned long long mk = m[k];
      if (!mk) continue;
      const int64_t v = batch_value(agg, x[k], y[k]);
      while (mk) {
        const int q = __ffsll(static_cast<long long>(mk)) - 1;
        mk &= mk - 1;
        // two 16-byte shared reads per emission: the query's factors by probe
        // position (0 for tables it does not group by) and its placement
        const int4 f = s_qf[q];
        const int4 qi = s_qi[q];
        const int32_t g = gr[0][k] * f.x + gr[1][k] * f.y + gr[2][k] * f.z + gr[3][k] * f.w;
        if (static_cast<uint32_t>(g) >= static_cast<uint32_t>(qi.x)) {
          ++bad;
          continue;
        }
        if (qi.y >= 0) {
          smem_add_split(reinterpret_cast<uint32_t*>(sacc), p.smem_slots, qi.y + g, static_cast<uint64_t>(v));
        } else {
          const int64_t base = (static_cast<int64_t>(qi.w) << 32) | static_cast<uint32_t>(qi.z);
          atomicAdd(&out[base + g], static_cast<unsigned long long>(v));
        }
      }
    }
  }
  const unsigned int wbad = __reduce_add_sync(0xffffffffu, bad);
  if ((tid & 31) == 0 && wbad) atomicAdd(&s_bad, wbad);
  __syncthreads();
  for (int q = 0; q < nq; ++q) {
    const BatchQuery& Q = sq[q];
    if (Q.smem_off < 0) continue;
    for (int64_t g = tid; g < Q.group_nums; g += blockDim.x) {
      const unsigned long long v = smem_split_get(reinterpret_cast<const uint32_t*>(sacc), p.smem_slots,
                                                  Q.smem_off + g);
      if (v) atomicAdd(&out[Q.out_offset + g], v);
    }
  }
  if (tid == 0 && s_bad) atomicAdd(p.range_err, static_cast<unsigned long long>(s_bad));
}

// Zero the batch's outputs (their location and size come with the descriptor,
// so a recorded graph serves any output buffer and query count).
__global__ void batch_zero_kernel(const BatchParams p) {
  const BatchDesc& D = *p.desc;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  const int64_t t0 = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  for (int64_t i = t0; i < D.out_total; i += stride) D.out[i] = 0ull;
  for (int64_t i = t0; i < D.n_queries; i += stride) D.totals[i] = 0ull;
}

// totals[q] = sum of query q's group vector (one block per query).  Launched
// with max_queries blocks; blocks past the batch's count return.
__global__ void batch_totals_kernel(const BatchParams p) {
  __shared__ long long red[32];
  const BatchDesc& D = *p.desc;
  if (static_cast<int>(blockIdx.x) >= D.n_queries) return;
  const BatchQuery& Q = D.q[blockIdx.x];
  int64_t s = 0;
  for (int64_t g = threadIdx.x; g < Q.group_nums; g += blockDim.x) s += static_cast<int64_t>(D.out[Q.out_offset + g]);
  s = warp_sum_i64(s);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    long long v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0;
    v = warp_sum_i64(v);
    if (threadIdx.x == 0) D.totals[blockIdx.x] = static_cast<unsigned long long>(v);
  }
}

static unsigned grid_n(const olap_ctx* ctx, int64_t n, int threads) {
  int64_t g = (n + threads - 1) / threads;
  const int64_t cap = static_cast<int64_t>(ctx->sm_count) * (2048 / threads);
  if (g > cap) g = cap;
  return static_cast<unsigned>(g < 1 ? 1 : g);
}

}  // namespace olap

// Batch handle: two staging slots (pinned host and device descriptors, one
// recorded graph each) so that one batch can be prepared while the previous
// one runs; packed attribute records and query-mask records per table.
struct olap_batch {
  olap_ctx* ctx = nullptr;
  int max_queries = 0;
  olap::BatchDesc* d_desc[2] = {};      // device
  olap::BatchDesc* h_desc[2] = {};      // pinned host staging
  cudaEvent_t done[2] = {};             // recorded after each slot's batch
  bool pending[2] = {false, false};
  cudaGraph_t graph[2] = {};
  cudaGraphExec_t exec[2] = {};
  olap::BatchParams params[2];
  bool have_params[2] = {false, false};
  int64_t runs = 0;
  int64_t captures = 0;                 // graphs recorded so far
  int2* attrs[OLAP_MAX_DIMS] = {};
  olap::DimRecord* rec[OLAP_MAX_DIMS] = {};
  int64_t attr_len[OLAP_MAX_DIMS] = {};
  int block = olap::kBatchThreads;        // scan kernel block size (olap_batch_tune / _autotune)
  int smem_slots = olap::kBatchSmemSlots; // per-block shared accumulators
  int parallel_probe = 0;                 // 1: every table's mask in one round trip (block <= 512)
};

extern "C" {

int olap_build_dimvec(olap_ctx* ctx, const int32_t* filter_attr, const int32_t* group_attr, int64_t n,
                      int32_t lo, int32_t hi, int use_group, int8_t* dimvec) {
  if (!ctx) return OLAP_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  OLAP_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  OLAP_REQUIRE(ctx, n >= 0, "n must be >= 0");
  OLAP_REQUIRE(ctx, n == 0 || (filter_attr && dimvec && (!use_group || group_attr)), "null argument");
  if (n == 0) return OLAP_OK;
  olap::build_dimvec_kernel<<<olap::grid_n(ctx, n, 256), 256, 0, ctx->stream>>>(
      filter_attr, group_attr, n, lo, hi, use_group, dimvec, &ctx->counters->range_errors);
  OLAP_CUDA_TRY(ctx, cudaGetLastError());
  return OLAP_OK;
}

int olap_batch_create(olap_ctx* ctx, int max_queries, olap_batch** out) {
  if (!ctx || !out || max_queries < 1 || max_queries > olap::kMaxBatchQueries) return OLAP_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  OLAP_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  olap_batch* b = new (std::nothrow) olap_batch();
  if (!b) return OLAP_ERR_NOMEM;
  b->ctx = ctx;
  b->max_queries = max_queries;
  bool ok = true;
  for (int s = 0; s < 2 && ok; ++s) {
    ok &= cudaMalloc(&b->d_desc[s], sizeof(olap::BatchDesc)) == cudaSuccess;
    ok &= cudaMallocHost(&b->h_desc[s], sizeof(olap::BatchDesc)) == cudaSuccess;
    ok &= cudaEventCreateWithFlags(&b->done[s], cudaEventDisableTiming) == cudaSuccess;
  }
  if (!ok) {
    cudaGetLastError();
    for (int s = 0; s < 2; ++s) {
      if (b->d_desc[s]) cudaFree(b->d_desc[s]);
      if (b->h_desc[s]) cudaFreeHost(b->h_desc[s]);
      if (b->done[s]) cudaEventDestroy(b->done[s]);
    }
    delete b;
    return OLAP_ERR_NOMEM;
  }
  *out = b;
  return OLAP_OK;
}

int olap_batch_destroy(olap_batch* b) {
  if (!b) return OLAP_ERR_INVALID;
  cudaSetDevice(b->ctx->device);
  for (int s = 0; s < 2; ++s) {
    if (b->pending[s]) cudaEventSynchronize(b->done[s]);
    if (b->exec[s]) cudaGraphExecDestroy(b->exec[s]);
    if (b->graph[s]) cudaGraphDestroy(b->graph[s]);
    cudaFree(b->d_desc[s]);
    cudaFreeHost(b->h_desc[s]);
    cudaEventDestroy(b->done[s]);
  }
  for (int t = 0; t < OLAP_MAX_DIMS; ++t) {
    if (b->attrs[t]) cudaFree(b->attrs[t]);
    if (b->rec[t]) cudaFree(b->rec[t]);
  }
  delete b;
  return OLAP_OK;
}

int olap_batch_set_dimension(olap_batch* b, int table, const int32_t* filter_attr, const int32_t* group_attr,
                             int64_t n) {
  if (!b || table < 0 || table >= OLAP_MAX_DIMS || n < 1 || n > INT32_MAX || !filter_attr)
    return OLAP_ERR_INVALID;
  olap_ctx* ctx = b->ctx;
  std::lock_guard<std::mutex> lk(ctx->mu);
  OLAP_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  if (b->attr_len[table] != n) {
    for (int s = 0; s < 2; ++s)
      if (b->pending[s]) cudaEventSynchronize(b->done[s]);
    cudaStreamSynchronize(ctx->stream);
    if (b->attrs[table]) cudaFree(b->attrs[table]);
    if (b->rec[table]) cudaFree(b->rec[table]);
    b->attrs[table] = nullptr;
    b->rec[table] = nullptr;
    b->attr_len[table] = 0;
    OLAP_CUDA_TRY(ctx, cudaMalloc(&b->attrs[table], sizeof(int2) * n));
    OLAP_CUDA_TRY(ctx, cudaMalloc(&b->rec[table], sizeof(olap::DimRecord) * n));
    b->attr_len[table] = n;
  }
  olap::pack_dim_attrs_kernel<<<olap::grid_n(ctx, n, 256), 256, 0, ctx->stream>>>(filter_attr, group_attr, n,
                                                                                 b->attrs[table]);
  OLAP_CUDA_TRY(ctx, cudaGetLastError());
  b->have_params[0] = b->have_params[1] = false;  // recorded graphs refer to the old buffers
  return OLAP_OK;
}

int olap_batch_graph_captures(olap_batch* b, int64_t* captures) {
  if (!b || !captures) return OLAP_ERR_INVALID;
  std::lock_guard<std::mutex> lk(b->ctx->mu);
  *captures = b->captures;
  return OLAP_OK;
}

int olap_batch_run(olap_batch* b, const olap_batch_query* queries, int n_queries, const int32_t* const* fk,
                   const int32_t* m1, const int32_t* m2, int64_t n_rows, int agg, int64_t* out,
                   int64_t out_slots, int64_t* totals, int use_graph) {
  if (!b) return OLAP_ERR_INVALID;
  olap_ctx* ctx = b->ctx;
  std::lock_guard<std::mutex> lk(ctx->mu);
  OLAP_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  OLAP_REQUIRE(ctx, n_queries >= 1 && n_queries <= b->max_queries && queries, "1..max_queries queries");
  OLAP_REQUIRE(ctx, n_rows >= 0 && out && totals && fk, "bad arguments");
  OLAP_REQUIRE(ctx, agg >= OLAP_AGG_M1_PLUS_M2 && agg <= OLAP_AGG_COUNT, "unknown aggregate");
  // The staging slot of this run; its previous batch must have finished
  // reading the pinned descriptors before they are overwritten.
  const int slot = static_cast<int>(b->runs & 1);
  if (b->pending[slot]) {
    OLAP_CUDA_TRY(ctx, cudaEventSynchronize(b->done[slot]));
    b->pending[slot] = false;
  }
  olap::BatchDesc& D = *b->h_desc[slot];
  std::memset(&D, 0, sizeof(D));
  int tables = 0;
  int64_t off = 0;
  std::vector<int64_t> cuts = {0, n_rows};
  for (int q = 0; q < n_queries; ++q) {
    const olap_batch_query& in = queries[q];
    olap::BatchQuery& d = D.q[q];
    OLAP_REQUIRE(ctx, in.row_begin >= 0 && in.row_end >= in.row_begin && in.row_end <= n_rows,
                 "query fact range outside the table");
    OLAP_REQUIRE(ctx, in.group_nums >= 1 && in.group_nums <= INT32_MAX, "group_nums must be in [1, 2^31)");
    d.row_begin = in.row_begin;
    d.row_end = in.row_end;
    d.group_nums = in.group_nums;
    d.out_offset = off;
    int64_t gbound = 0;
    for (int t = 0; t < OLAP_MAX_DIMS; ++t) {
      d.lo[t] = in.lo[t];
      d.hi[t] = in.hi[t];
      d.factor[t] = in.factor[t];
      if (in.uses & (1 << t)) {
        OLAP_REQUIRE(ctx, b->attrs[t] && fk[t], "query uses a table without attributes or fk column");
        d.uses |= 1 << t;
        D.uses_mask[t] |= 1ull << q;
        if (in.grouped & (1 << t)) {
          d.grouped |= 1 << t;
          gbound += 128 * std::llabs(static_cast<long long>(in.factor[t]));
        }
      }
    }
    OLAP_REQUIRE(ctx, gbound <= INT32_MAX, "group factors too large");
    tables |= d.uses;
    off += in.group_nums;
    cuts.push_back(in.row_begin);
    cuts.push_back(in.row_end);
  }
  OLAP_REQUIRE(ctx, off <= out_slots, "out holds fewer slots than the queries' groups");
  // Per-block shared accumulators for the queries with the fewest groups
  // (they see the most same-address atomics), as long as they fit.
  {
    std::vector<int> byg(n_queries);
    for (int q = 0; q < n_queries; ++q) byg[q] = q;
    std::stable_sort(byg.begin(), byg.end(), [&](int x, int y) { return D.q[x].group_nums < D.q[y].group_nums; });
    int64_t used = 0;
    for (int q : byg) {
      D.q[q].smem_off = -1;
      if (used + D.q[q].group_nums <= b->smem_slots) {
        D.q[q].smem_off = static_cast<int32_t>(used);
        used += D.q[q].group_nums;
      }
    }
  }
  // Fact-range segments: between consecutive cut points the set of queries
  // whose range covers a row is constant.
  std::sort(cuts.begin(), cuts.end());
  cuts.erase(std::unique(cuts.begin(), cuts.end()), cuts.end());
  int nseg = 0;
  for (size_t c = 0; c + 1 < cuts.size(); ++c) {
    unsigned long long m = 0;
    for (int q = 0; q < n_queries; ++q)
      if (D.q[q].row_begin <= cuts[c] && cuts[c + 1] <= D.q[q].row_end) m |= 1ull << q;
    D.seg_begin[nseg] = cuts[c];
    D.seg_mask[nseg] = m;
    ++nseg;
  }
  if (nseg == 0) {  // empty table
    D.seg_begin[0] = 0;
    D.seg_mask[0] = 0;
    nseg = 1;
  }
  D.n_queries = n_queries;
  D.n_seg = nseg;
  D.out = reinterpret_cast<unsigned long long*>(out);
  D.totals = reinterpret_cast<unsigned long long*>(totals);
  D.out_total = off;
  olap::BatchParams p;
  std::memset(&p, 0, sizeof(p));
  int order[OLAP_MAX_DIMS] = {0, 1, 2, 3};
  std::stable_sort(order, order + OLAP_MAX_DIMS, [&](int x, int y) { return b->attr_len[x] < b->attr_len[y]; });
  for (int o = 0; o < OLAP_MAX_DIMS; ++o) p.probe_order |= order[o] << (2 * o);
  for (int t = 0; t < OLAP_MAX_DIMS; ++t) {
    p.attrs[t] = b->attrs[t];
    p.rec[t] = b->rec[t];
    p.dim_len[t] = static_cast<uint32_t>(b->attr_len[t]);
    p.fk[t] = fk[t];
  }
  p.m1 = m1;
  p.m2 = m2;
  p.n_rows = n_rows;
  p.desc = b->d_desc[slot];
  p.tables_used = tables;
  p.agg = agg;
  p.smem_slots = b->smem_slots;
  p.block = b->block;
  p.range_err = &ctx->counters->range_errors;
  const bool need_m1 = agg == OLAP_AGG_M1_PLUS_M2 || agg == OLAP_AGG_M1 || agg == OLAP_AGG_M1_TIMES_M2;
  const bool need_m2 = agg == OLAP_AGG_M1_PLUS_M2 || agg == OLAP_AGG_M2 || agg == OLAP_AGG_M1_TIMES_M2;
  OLAP_REQUIRE(ctx, n_rows == 0 || ((!need_m1 || m1) && (!need_m2 || m2)), "measure columns required");
  const size_t scan_smem = sizeof(unsigned long long) * static_cast<size_t>(b->smem_slots);
  const bool par = b->parallel_probe != 0 && b->block <= 512;
  void (*scan)(const olap::BatchParams) = par ? olap::batch_scan_kernel<true> : olap::batch_scan_kernel<false>;
  if (scan_smem > 48 * 1024)
    OLAP_CUDA_TRY(ctx, cudaFuncSetAttribute(scan, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            static_cast<int>(scan_smem)));
  int bps = 1;
  OLAP_CUDA_TRY(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, scan, b->block, scan_smem));
  const unsigned grid = static_cast<unsigned>(ctx->sm_count) * static_cast<unsigned>(bps < 1 ? 1 : bps);
  // The work of one batch: descriptors H2D, zero outputs, query masks of the
  // used tables, one persistent pass over the fact table.
  auto enqueue = [&](cudaStream_t st) -> cudaError_t {
    cudaError_t e = cudaMemcpyAsync(b->d_desc[slot], b->h_desc[slot], sizeof(olap::BatchDesc),
                                    cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
      olap::batch_zero_kernel<<<static_cast<unsigned>(ctx->sm_count) * 2, 512, 0, st>>>(p);
      e = cudaGetLastError();
    }
    for (int t = 0; t < OLAP_MAX_DIMS && e == cudaSuccess; ++t) {
      if (!((tables >> t) & 1)) continue;
      olap::batch_records_kernel<<<olap::grid_n(ctx, b->attr_len[t], 256), 256, 0, st>>>(p, t);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess && n_rows > 0) {
      scan<<<grid, b->block, scan_smem, st>>>(p);
      e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
      olap::batch_totals_kernel<<<b->max_queries, 256, 0, st>>>(p);
      e = cudaGetLastError();
    }
    return e;
  };
  if (!use_graph) {
    OLAP_CUDA_TRY(ctx, enqueue(ctx->stream));
  } else {
    // Graph of this slot: re-captured when the launch parameters (tables,
    // fact columns, aggregate) change, replayed otherwise.  Queries, output
    // buffers and their sizes travel in the descriptor its copy node reads
    // from the slot's pinned staging.
    const bool same = b->have_params[slot] && b->exec[slot] && std::memcmp(&b->params[slot], &p, sizeof(p)) == 0;
    if (!same) {
      if (b->exec[slot]) cudaGraphExecDestroy(b->exec[slot]);
      if (b->graph[slot]) cudaGraphDestroy(b->graph[slot]);
      b->exec[slot] = nullptr;
      b->graph[slot] = nullptr;
      b->have_params[slot] = false;
      cudaStream_t cs;
      OLAP_CUDA_TRY(ctx, cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
      cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
      if (e == cudaSuccess) {
        cudaError_t e2 = enqueue(cs);
        e = cudaStreamEndCapture(cs, &b->graph[slot]);
        if (e == cudaSuccess) e = e2;
      }
      if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec[slot], b->graph[slot], 0);
      cudaStreamDestroy(cs);
      if (e != cudaSuccess) return olap::check_cuda(ctx, e, "batch graph capture");
      b->params[slot] = p;
      b->have_params[slot] = true;
      ++b->captures;
    }
    OLAP_CUDA_TRY(ctx, cudaGraphLaunch(b->exec[slot], ctx->stream));
  }
  OLAP_CUDA_TRY(ctx, cudaEventRecord(b->done[slot], ctx->stream));
  b->pending[slot] = true;
  ++b->runs;
  return OLAP_OK;
}

int olap_batch_tune(olap_batch* b, int block, int smem_slots) {
  if (!b) return OLAP_ERR_INVALID;
  olap_ctx* ctx = b->ctx;
  std::lock_guard<std::mutex> lk(ctx->mu);
  OLAP_REQUIRE(ctx, block >= 128 && block <= olap::kBatchMaxThreads && block % 32 == 0,
               "block must be a multiple of 32 in [128, 1024]");
  OLAP_REQUIRE(ctx, smem_slots >= 0 && smem_slots <= olap::kBatchMaxSmemSlots,
               "smem_slots must be in [0, 24576]");
  b->block = block;
  b->smem_slots = smem_slots;
  return OLAP_OK;
}

int olap_batch_set_probe(olap_batch* b, int parallel_probe) {
  if (!b || (parallel_probe != 0 && parallel_probe != 1)) return OLAP_ERR_INVALID;
  std::lock_guard<std::mutex> lk(b->ctx->mu);
  b->parallel_probe = parallel_probe;
  return OLAP_OK;
}

int olap_batch_get_tuning(olap_batch* b, int* block, int* smem_slots, int* parallel_probe) {
  if (!b) return OLAP_ERR_INVALID;
  std::lock_guard<std::mutex> lk(b->ctx->mu);
  if (block) *block = b->block;
  if (smem_slots) *smem_slots = b->smem_slots;
  if (parallel_probe) *parallel_probe = (b->parallel_probe && b->block <= 512) ? 1 : 0;
  return OLAP_OK;
}

int olap_batch_autotune(olap_batch* b, const olap_batch_query* queries, int n_queries,
                        const int32_t* const* fk, const int32_t* m1, const int32_t* m2, int64_t n_rows,
                        int agg, int64_t* out, int64_t out_slots, int64_t* totals, int64_t sample_rows,
                        int* best_block, int* best_slots, double* best_ms) {
  if (!b || !queries || n_queries < 1 || n_queries > b->max_queries) return OLAP_ERR_INVALID;
  olap_ctx* ctx = b->ctx;
  if (sample_rows <= 0) sample_rows = int64_t(64) << 20;
  const int64_t rows = std::min(n_rows, sample_rows);
  // The queries' fact ranges scaled onto the sample's rows [0, rows), so the
  // sample sees the same mix of live queries per row as the whole table (a
  // prefix cut would drop the queries whose ranges start past it, and the
  // shape that wins on fewer queries is not the one that wins on all).
  std::vector<olap_batch_query> qs(queries, queries + n_queries);
  const double scale = n_rows > rows ? static_cast<double>(rows) / static_cast<double>(n_rows) : 1.0;
  for (auto& q : qs) {
    const int64_t lo = std::min<int64_t>(rows, static_cast<int64_t>(static_cast<double>(q.row_begin) * scale));
    const int64_t hi = std::min<int64_t>(rows, static_cast<int64_t>(static_cast<double>(q.row_end) * scale));
    q.row_begin = std::max<int64_t>(0, lo);
    q.row_end = std::max<int64_t>(q.row_begin, hi);
  }
  cudaEvent_t e0, e1;
  {
    std::lock_guard<std::mutex> lk(ctx->mu);
    OLAP_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
    OLAP_CUDA_TRY(ctx, cudaEventCreate(&e0));
    OLAP_CUDA_TRY(ctx, cudaEventCreate(&e1));
  }
  unsigned long long errs_before = 0;
  cudaMemcpyAsync(&errs_before, &ctx->counters->range_errors, sizeof(errs_before), cudaMemcpyDeviceToHost,
                  ctx->stream);
  cudaStreamSynchronize(ctx->stream);
  const int saved_block = b->block, saved_slots = b->smem_slots, saved_probe = b->parallel_probe;
  double best = 1e30;
  int bb = saved_block, bs = saved_slots, bp = saved_probe;
  for (int probe : {0, 1})
  for (int block : {256, 512, 1024}) {
    if (probe && block > 512) continue;
    for (int slots : {0, 2048, 4096, 8192, 16384}) {
      b->block = block;
      b->smem_slots = slots;
      b->parallel_probe = probe;
      float ms = 0.f, best_c = 1e30f;
      bool ok = true;
      for (int rep = 0; rep < 3 && ok; ++rep) {
        cudaEventRecord(e0, ctx->stream);
        const int st = olap_batch_run(b, qs.data(), n_queries, fk, m1, m2, rows, agg, out, out_slots, totals, 0);
        cudaEventRecord(e1, ctx->stream);
        if (st != OLAP_OK || cudaEventSynchronize(e1) != cudaSuccess) {
          cudaGetLastError();
          ok = false;
          break;
        }
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0) best_c = std::min(best_c, ms);  // the first run warms caches
      }
      if (ok && best_c < best) {
        best = best_c;
        bb = block;
        bs = slots;
        bp = probe;
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  // Rows the timed runs dropped were counted; restore the earlier count.
  cudaMemcpyAsync(&ctx->counters->range_errors, &errs_before, sizeof(errs_before), cudaMemcpyHostToDevice,
                  ctx->stream);
  cudaStreamSynchronize(ctx->stream);
  if (best >= 1e29) {
    b->block = saved_block;
    b->smem_slots = saved_slots;
    b->parallel_probe = saved_probe;
    return olap::set_error(ctx, OLAP_ERR_CUDA, "no batch autotune candidate ran");
  }
  b->block = bb;
  b->smem_slots = bs;
  b->parallel_probe = bp;
  if (best_block) *best_block = bb;
  if (best_slots) *best_slots = bs;
  if (best_ms) *best_ms = best;
  return OLAP_OK;
}

}  // extern "C"
