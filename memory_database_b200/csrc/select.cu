// Select, project and gather operators for sm_100a.
//
// Reference: code/select/test_select_option.cpp (predicate `col <= val` in
// every sel_lt_T_* primitive, :28-440; the 3-predicate driver selalgo_rowwise
// :450-467) and code/project/test_project_option.cpp (pairs (Ra, Rc) of the
// rows where Ra <= c and Rc <= c, :34-864).  Selection vectors are int32 row
// ids in ascending order, produced in one pass by the order-preserving
// compaction of compact.cuh; bitmaps hold bit i of row i at byte i/8, bit
// i%8 (the storage order of a little-endian std::vector<bool>).
#include <cstring>

#include "compact.cuh"

namespace olap {

__device__ __forceinline__ bool cmp_pass(int32_t v, int32_t val, int cmp) {
  return cmp == OLAP_CMP_LT ? v < val : v <= val;
}

__device__ __forceinline__ int32_t lane4(const int4& v, int k) {
  return k == 0 ? v.x : k == 1 ? v.y : k == 2 ? v.z : v.w;
}

// Items are rows (kRid false) or positions of an input selection vector.
// The plain column case caches nothing between flags() and emit(), so it
// takes 16 groups per thread and 4 rounds per tile (256 KB tiles); with row
// ids, 8 groups and one round.
template <bool kRid>
struct SelectOp {
  static constexpr int kGroups = kRid ? 8 : 16;
  static constexpr int kRounds = kRid ? 1 : 4;  // emit() of a plain column needs nothing cached
  const int32_t* col;
  const int32_t* in_rowids;  // optional input selection vector
  int32_t* out;
  unsigned long long* range_err;
  int64_t col_len;
  int32_t val;
  int32_t cmp;
  int32_t vec;               // col (or in_rowids) 16-byte aligned
  int4 rid[kGroups];  // values (or row ids) of each group, loaded by prefetch()

  __device__ __forceinline__ bool vec_ok() const { return vec != 0; }
  __device__ __forceinline__ void prefetch(int u, int64_t first) {
    rid[u] = ld_stream_v4_ordered((kRid ? in_rowids : col) + first, policy_evict_first());
  }
  template <bool kFull>
  __device__ __forceinline__ uint32_t flags(int u, int64_t first, int nv) {
    const uint64_t pol = policy_evict_first();
    uint32_t m = 0;
    if constexpr (!kRid) {
      if (kFull) {
        const int4 v = rid[u];
#pragma unroll
        for (int k = 0; k < 4; ++k) m |= static_cast<uint32_t>(cmp_pass(lane4(v, k), val, cmp)) << k;
      } else if (vec && nv == 4) {
        const int4 v = ld_stream_v4(col + first, pol);
#pragma unroll
        for (int k = 0; k < 4; ++k) m |= static_cast<uint32_t>(cmp_pass(lane4(v, k), val, cmp)) << k;
      } else {
        for (int k = 0; k < nv; ++k) m |= static_cast<uint32_t>(cmp_pass(col[first + k], val, cmp)) << k;
      }
    } else {
      int4 r = make_int4(0, 0, 0, 0);
      if (kFull) {
        r = rid[u];
      } else if (vec && nv == 4) {
        r = ld_stream_v4(in_rowids + first, pol);
      } else {
        int32_t t[4] = {0, 0, 0, 0};
        for (int k = 0; k < nv; ++k) t[k] = in_rowids[first + k];
        r = make_int4(t[0], t[1], t[2], t[3]);
      }
      rid[u] = r;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        if (k >= nv) continue;
        const int32_t row = lane4(r, k);
        if (row < 0 || row >= col_len) {  // not a row of col: dropped and counted
          atomicAdd(range_err, 1ull);
          continue;
        }
        m |= static_cast<uint32_t>(cmp_pass(__ldg(col + row), val, cmp)) << k;
      }
    }
    return m;
  }
  __device__ __forceinline__ void emit(int u, int k, int64_t item, int64_t pos) {
    if constexpr (kRid) out[pos] = lane4(rid[u], k);
    else out[pos] = static_cast<int32_t>(item);
  }
};

// Rows where Ra <= c and Rc <= c; writes the pair (Ra, Rc).
struct ProjectOp {
  static constexpr int kGroups = kCompactGroups;
  const int32_t* ra;
  const int32_t* rc;
  int32_t* out_a;
  int32_t* out_c;
  int32_t cond;
  int32_t vec;
  int4 a[kCompactGroups], c[kCompactGroups];

  __device__ __forceinline__ bool vec_ok() const { return vec != 0; }
  __device__ __forceinline__ void prefetch(int u, int64_t first) {
    a[u] = ld_stream_v4(ra + first, policy_evict_first());
    c[u] = ld_stream_v4(rc + first, policy_evict_first());
  }
  template <bool kFull>
  __device__ __forceinline__ uint32_t flags(int u, int64_t first, int nv) {
    const uint64_t pol = policy_evict_first();
    if (kFull) {
      // a[u], c[u] loaded by prefetch()
    } else if (vec && nv == 4) {
      a[u] = ld_stream_v4(ra + first, pol);
      c[u] = ld_stream_v4(rc + first, pol);
    } else {
      int32_t x[4] = {0, 0, 0, 0}, y[4] = {0, 0, 0, 0};
      for (int k = 0; k < nv; ++k) {
        x[k] = ra[first + k];
        y[k] = rc[first + k];
      }
      a[u] = make_int4(x[0], x[1], x[2], x[3]);
      c[u] = make_int4(y[0], y[1], y[2], y[3]);
    }
    uint32_t m = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k)
      if (k < nv) m |= static_cast<uint32_t>(lane4(a[u], k) <= cond && lane4(c[u], k) <= cond) << k;
    return m;
  }
  __device__ __forceinline__ void emit(int u, int k, int64_t, int64_t pos) {
    out_a[pos] = lane4(a[u], k);
    out_c[pos] = lane4(c[u], k);
  }
};

// Rows of a row store (an array of structs, row_bytes apart): the pair (Ra,
// Rc) read as int32 at byte offsets off_a and off_c of each row, for the rows
// where both are <= c (proalgo_rowwise over row_store_min / row_store_max,
// project/test_project_option.cpp:34-147).  Rows are not 16-byte vectors, so
// every group takes the per-row loads.
struct ProjectRowsOp {
  static constexpr int kGroups = kCompactGroups;
  const unsigned char* rows;
  int64_t row_bytes;
  int32_t off_a, off_c;
  int32_t* out_a;
  int32_t* out_c;
  int32_t cond;
  int4 a[kCompactGroups], c[kCompactGroups];

  __device__ __forceinline__ bool vec_ok() const { return false; }
  __device__ __forceinline__ void prefetch(int, int64_t) {}
  template <bool kFull>
  __device__ __forceinline__ uint32_t flags(int u, int64_t first, int nv) {
    int32_t x[4] = {0, 0, 0, 0}, y[4] = {0, 0, 0, 0};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (k >= nv) continue;
      const unsigned char* r = rows + (first + k) * row_bytes;
      x[k] = __ldg(reinterpret_cast<const int32_t*>(r + off_a));
      y[k] = __ldg(reinterpret_cast<const int32_t*>(r + off_c));
    }
    a[u] = make_int4(x[0], x[1], x[2], x[3]);
    c[u] = make_int4(y[0], y[1], y[2], y[3]);
    uint32_t m = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k)
      if (k < nv) m |= static_cast<uint32_t>(x[k] <= cond && y[k] <= cond) << k;
    return m;
  }
  __device__ __forceinline__ void emit(int u, int k, int64_t, int64_t pos) {
    out_a[pos] = lane4(a[u], k);
    out_c[pos] = lane4(c[u], k);
  }
};

// One 32-bit word of the bitmap per warp step: lane l tests row 32w + l.
__global__ void select_bitmap_kernel(const int32_t* __restrict__ col, int64_t n, int32_t val, int cmp,
                                     uint32_t* __restrict__ bits) {
  const int64_t nwords = (n + 31) >> 5;
  const int64_t warp = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
  const int lane = threadIdx.x & 31;
  const uint64_t pol = policy_evict_first();
  for (int64_t w = warp; w < nwords; w += nwarps) {
    const int64_t r = (w << 5) + lane;
    const bool pass = r < n && cmp_pass(ld_stream_s32_if(r < n, col + r, pol, 0), val, cmp);
    const uint32_t word = __ballot_sync(0xffffffffu, pass);
    if (lane == 0) bits[w] = word;
  }
}

// SUM(Rd) and COUNT over rows with Ra, Rb, Rc all <= condition.
__global__ void __launch_bounds__(512) selalgo_kernel(int32_t cond, int64_t n, const int32_t* __restrict__ ra,
                                                      const int32_t* __restrict__ rb, const int32_t* __restrict__ rc,
                                                      const int32_t* __restrict__ rd, int vec,
                                                      unsigned long long* sum, unsigned long long* count) {
  __shared__ long long s_red[16][2];
  const uint64_t pol = policy_evict_first();
  int64_t s = 0, c = 0;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  const int64_t tid = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t n4 = vec ? n >> 2 : 0;
  for (int64_t i = tid; i < n4; i += stride) {
    const int4 a = ld_stream_v4(ra + 4 * i, pol), b = ld_stream_v4(rb + 4 * i, pol);
    const int4 cc = ld_stream_v4(rc + 4 * i, pol), d = ld_stream_v4(rd + 4 * i, pol);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const bool p = lane4(a, k) <= cond && lane4(b, k) <= cond && lane4(cc, k) <= cond;
      s += p ? lane4(d, k) : 0;
      c += p;
    }
  }
  for (int64_t r = 4 * n4 + tid; r < n; r += stride) {
    const bool p = ra[r] <= cond && rb[r] <= cond && rc[r] <= cond;
    s += p ? rd[r] : 0;
    c += p;
  }
  s = warp_sum_i64(s);
  c = warp_sum_i64(c);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    s_red[warp][0] = s;
    s_red[warp][1] = c;
  }
  __syncthreads();
  if (warp == 0) {
    long long x = lane < static_cast<int>(blockDim.x >> 5) ? s_red[lane][0] : 0;
    long long y = lane < static_cast<int>(blockDim.x >> 5) ? s_red[lane][1] : 0;
    x = warp_sum_i64(x);
    y = warp_sum_i64(y);
    if (lane == 0) {
      if (x) atomicAdd(sum, static_cast<unsigned long long>(x));
      if (y) atomicAdd(count, static_cast<unsigned long long>(y));
    }
  }
}

constexpr int kMaxGatherCols = 8;
struct GatherParams {
  const int32_t* cols[kMaxGatherCols];
  int32_t* outs[kMaxGatherCols];
  unsigned long long* range_err;
  int64_t col_len;
  int ncols;
};

// One gathered value.  kSparse: the load asks L2 for a 64-byte fetch on a
// miss; when the row ids are far apart (more than 16 rows, 64 bytes, between
// neighbours on average) the rest of a larger fetch is never used.  volatile
// keeps each load inside its guard, as __ldg's own asm does.
template <bool kSparse>
__device__ __forceinline__ int32_t ld_gather(const int32_t* p) {
  if (!kSparse) return __ldg(p);
  int32_t v;
  asm volatile("ld.global.nc.L2::64B.s32 %0, [%1];" : "=r"(v) : "l"(p));
  return v;
}

// outs[c][i] = cols[c][rowids[i]]: row ids read with 128-bit loads, values
// gathered through L1/L2 and written with 128-bit stores.  A row id outside
// [0, col_len) yields 0 and is counted.
template <bool kSparse>
__global__ void gather_kernel(const int32_t* __restrict__ rowids, int64_t k, const GatherParams gp, int vec) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  const int64_t tid = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const uint64_t pol = policy_evict_first();
  const int64_t k4 = vec ? k >> 2 : 0;
  unsigned int bad = 0;
  auto ok = [&](int32_t r) { return r >= 0 && r < gp.col_len; };
  for (int64_t i = tid; i < k4; i += stride) {
    const int4 r = ld_stream_v4(rowids + 4 * i, pol);
    const bool ox = ok(r.x), oy = ok(r.y), oz = ok(r.z), ow = ok(r.w);
    bad += !ox + !oy + !oz + !ow;
    for (int c = 0; c < gp.ncols; ++c) {
      const int32_t* col = gp.cols[c];
      int4 v;
      v.x = ox ? ld_gather<kSparse>(col + r.x) : 0;
      v.y = oy ? ld_gather<kSparse>(col + r.y) : 0;
      v.z = oz ? ld_gather<kSparse>(col + r.z) : 0;
      v.w = ow ? ld_gather<kSparse>(col + r.w) : 0;
      reinterpret_cast<int4*>(gp.outs[c])[i] = v;
    }
  }
  for (int64_t j = 4 * k4 + tid; j < k; j += stride) {
    const int32_t r = rowids[j];
    const bool o = ok(r);
    bad += !o;
    for (int c = 0; c < gp.ncols; ++c) gp.outs[c][j] = o ? ld_gather<kSparse>(gp.cols[c] + r) : 0;
  }
  if (bad) atomicAdd(gp.range_err, static_cast<unsigned long long>(bad));
}

static bool al16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

template <class Op>
static int run_compaction(olap_ctx* ctx, const Op& op, int64_t n_items, int64_t* d_count) {
  Arena ar(ctx);
  ScanTiles st;
  unsigned long long* total = d_count ? reinterpret_cast<unsigned long long*>(d_count)
                                      : ar.take<unsigned long long>(1);
  if (!total) return set_error(ctx, OLAP_ERR_CAPACITY, "scratch arena exhausted");
  int rc = make_scan_tiles(ctx, ar, n_items, total, ctx->stream, &st, compact_tile_items<Op>());
  if (rc != OLAP_OK) return rc;
  compact_kernel<Op><<<compact_grid(ctx, st.n_tiles), kCompactThreads, 0, ctx->stream>>>(op, n_items, st);
  OLAP_CUDA_TRY(ctx, cudaGetLastError());
  return OLAP_OK;
}

// Look-back of tile 1 while tile 0's status is never published: the wait
// runs out after spin_limit polls (the failure path of every compaction).
__global__ void lookback_timeout_kernel(ScanTiles st, uint32_t spin_limit, long long* out) {
  const int64_t b = lookback(st, 1, 1, spin_limit);
  if (threadIdx.x == 0) *out = b;
}

static unsigned stream_grid(const olap_ctx* ctx, int64_t items, int threads) {
  int64_t g = (items + threads - 1) / threads;
  const int64_t cap = static_cast<int64_t>(ctx->sm_count) * (2048 / threads);
  if (g > cap) g = cap;
  return static_cast<unsigned>(g < 1 ? 1 : g);
}

}  // namespace olap

extern "C" {

int olap_select_rowids(olap_ctx* ctx, const int32_t* col, int64_t col_len, int32_t val, int cmp,
                       const int32_t* in_rowids, int64_t n_in, int32_t* out_rowids, int64_t* d_count) {
  if (!ctx) return OLAP_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  OLAP_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  const int64_t n = in_rowids ? n_in : col_len;
  OLAP_REQUIRE(ctx, col_len >= 0 && col_len <= INT32_MAX && n >= 0 && n <= INT32_MAX,
               "lengths must be in [0, 2^31)");
  OLAP_REQUIRE(ctx, cmp == OLAP_CMP_LE || cmp == OLAP_CMP_LT, "cmp must be OLAP_CMP_LE or OLAP_CMP_LT");
  OLAP_REQUIRE(ctx, n == 0 || (col && out_rowids), "null column or output");
  auto fill = [&](auto& op) {
    std::memset(&op, 0, sizeof(op));
    op.col = col;
    op.in_rowids = in_rowids;
    op.out = out_rowids;
    op.range_err = &ctx->counters->range_errors;
    op.col_len = col_len;
    op.val = val;
    op.cmp = cmp;
    op.vec = in_rowids ? olap::al16(in_rowids) : olap::al16(col);
  };
  if (in_rowids) {
    olap::SelectOp<true> op;
    fill(op);
    return olap::run_compaction(ctx, op, n, d_count);
  }
  olap::SelectOp<false> op;
  fill(op);
  return olap::run_compaction(ctx, op, n, d_count);
}

int olap_debug_wait_timeout(olap_ctx* ctx, uint32_t spin_limit) {
  if (!ctx || spin_limit < 1) return OLAP_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  OLAP_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  olap::Arena ar(ctx);
  olap::ScanTiles st;
  unsigned long long* total = ar.take<unsigned long long>(1);
  long long* out = ar.take<long long>(1);
  if (!total || !out) return olap::set_error(ctx, OLAP_ERR_CAPACITY, "scratch arena exhausted");
  int rc = olap::make_scan_tiles(ctx, ar, 2, total, ctx->stream, &st, 1);  // two one-item tiles
  if (rc != OLAP_OK) return rc;
  olap::lookback_timeout_kernel<<<1, 32, 0, ctx->stream>>>(st, spin_limit, out);
  OLAP_CUDA_TRY(ctx, cudaGetLastError());
  return olap::check_timeouts(ctx, ctx->stream);
}

int olap_select_bitmap(olap_ctx* ctx, const int32_t* col, int64_t n, int32_t val, int cmp,
                       uint32_t* bitmap) {
  if (!ctx) return OLAP_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  OLAP_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  OLAP_REQUIRE(ctx, n >= 0, "n must be >= 0");
  OLAP_REQUIRE(ctx, cmp == OLAP_CMP_LE || cmp == OLAP_CMP_LT, "cmp must be OLAP_CMP_LE or OLAP_CMP_LT");
  if (n == 0) return OLAP_OK;
  OLAP_REQUIRE(ctx, col && bitmap, "null column or bitmap");
  olap::select_bitmap_kernel<<<olap::stream_grid(ctx, n, 256), 256, 0, ctx->stream>>>(col, n, val, cmp, bitmap);
  OLAP_CUDA_TRY(ctx, cudaGetLastError());
  return OLAP_OK;
}

int olap_selalgo(olap_ctx* ctx, int32_t condition, int64_t n, const int32_t* Ra, const int32_t* Rb,
                 const int32_t* Rc, const int32_t* Rd, int64_t* d_sum, int64_t* d_count) {
  if (!ctx) return OLAP_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  OLAP_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  OLAP_REQUIRE(ctx, n >= 0 && d_sum, "n must be >= 0 and d_sum given");
  OLAP_REQUIRE(ctx, n == 0 || (Ra && Rb && Rc && Rd), "null column");
  olap::Arena ar(ctx);
  int64_t* cnt = d_count ? d_count : ar.take<int64_t>(1);
  if (!cnt) return olap::set_error(ctx, OLAP_ERR_CAPACITY, "scratch arena exhausted");
  OLAP_CUDA_TRY(ctx, cudaMemsetAsync(d_sum, 0, sizeof(int64_t), ctx->stream));
  OLAP_CUDA_TRY(ctx, cudaMemsetAsync(cnt, 0, sizeof(int64_t), ctx->stream));
  if (n == 0) return OLAP_OK;
  const int vec = olap::al16(Ra) && olap::al16(Rb) && olap::al16(Rc) && olap::al16(Rd);
  olap::selalgo_kernel<<<olap::stream_grid(ctx, (n + 3) / 4, 512), 512, 0, ctx->stream>>>(
      condition, n, Ra, Rb, Rc, Rd, vec, reinterpret_cast<unsigned long long*>(d_sum),
      reinterpret_cast<unsigned long long*>(cnt));
  OLAP_CUDA_TRY(ctx, cudaGetLastError());
  return OLAP_OK;
}

int olap_project_pairs(olap_ctx* ctx, int32_t condition, int64_t n, const int32_t* Ra,
                       const int32_t* Rc, int32_t* out_a, int32_t* out_c, int64_t* d_count) {
  if (!ctx) return OLAP_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  OLAP_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  OLAP_REQUIRE(ctx, n >= 0 && n <= INT32_MAX, "n must be in [0, 2^31)");
  OLAP_REQUIRE(ctx, n == 0 || (Ra && Rc && out_a && out_c), "null column or output");
  olap::ProjectOp op;
  std::memset(&op, 0, sizeof(op));
  op.ra = Ra;
  op.rc = Rc;
  op.out_a = out_a;
  op.out_c = out_c;
  op.cond = condition;
  op.vec = olap::al16(Ra) && olap::al16(Rc);
  return olap::run_compaction(ctx, op, n, d_count);
}

int olap_project_pairs_rows(olap_ctx* ctx, int32_t condition, int64_t n, const void* rows, int64_t row_bytes,
                            int64_t off_a, int64_t off_c, int32_t* out_a, int32_t* out_c, int64_t* d_count) {
  if (!ctx) return OLAP_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  OLAP_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  OLAP_REQUIRE(ctx, n >= 0 && n <= INT32_MAX, "n must be in [0, 2^31)");
  OLAP_REQUIRE(ctx, n == 0 || (rows && out_a && out_c), "null rows or output");
  OLAP_REQUIRE(ctx, row_bytes >= 4 && row_bytes % 4 == 0, "row_bytes must be a positive multiple of 4");
  OLAP_REQUIRE(ctx, off_a >= 0 && off_c >= 0 && off_a % 4 == 0 && off_c % 4 == 0 && off_a + 4 <= row_bytes &&
                        off_c + 4 <= row_bytes,
               "field offsets must be 4-byte aligned and inside the row");
  OLAP_REQUIRE(ctx, (reinterpret_cast<uintptr_t>(rows) & 3) == 0, "rows must be 4-byte aligned");
  olap::ProjectRowsOp op;
  std::memset(&op, 0, sizeof(op));
  op.rows = static_cast<const unsigned char*>(rows);
  op.row_bytes = row_bytes;
  op.off_a = static_cast<int32_t>(off_a);
  op.off_c = static_cast<int32_t>(off_c);
  op.out_a = out_a;
  op.out_c = out_c;
  op.cond = condition;
  return olap::run_compaction(ctx, op, n, d_count);
}

int olap_gather_i32(olap_ctx* ctx, const int32_t* rowids, int64_t k, int ncols,
                    const int32_t* const* cols, int64_t col_len, int32_t* const* outs) {
  if (!ctx) return OLAP_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  OLAP_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  OLAP_REQUIRE(ctx, k >= 0 && ncols >= 1 && ncols <= olap::kMaxGatherCols, "1..8 columns");
  if (k == 0) return OLAP_OK;
  OLAP_REQUIRE(ctx, rowids && cols && outs, "null argument");
  olap::GatherParams gp;
  std::memset(&gp, 0, sizeof(gp));
  gp.ncols = ncols;
  gp.col_len = col_len;
  gp.range_err = &ctx->counters->range_errors;
  bool vec = olap::al16(rowids);
  for (int c = 0; c < ncols; ++c) {
    OLAP_REQUIRE(ctx, cols[c] && outs[c], "null column or output");
    gp.cols[c] = cols[c];
    gp.outs[c] = outs[c];
    vec &= olap::al16(outs[c]);
  }
  // row ids more than 16 rows apart on average: 64-byte fetches
  const unsigned grid = olap::stream_grid(ctx, (k + 3) / 4, 256);
  if (col_len > 16 * k)
    olap::gather_kernel<true><<<grid, 256, 0, ctx->stream>>>(rowids, k, gp, vec);
  else
    olap::gather_kernel<false><<<grid, 256, 0, ctx->stream>>>(rowids, k, gp, vec);
  OLAP_CUDA_TRY(ctx, cudaGetLastError());
  return OLAP_OK;
}

}  // extern "C"
