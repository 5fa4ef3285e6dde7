// Column-wise OLAP core and the star-join operator for sm_100a.
//
// Column-wise model (code/OLAPcore/test_multi_compute_operator.cpp):
//  * join_cwm_sv (:908-958, thread body :290-322) builds the static vector
//    int16 groupID[N] (GROUP_NULL when a dimension misses) one dimension per
//    pass; here all dimensions in one pass, same vector;
//  * agg_cwm_sv (:764-827, :662-673) sums M1+M2 by groupID;
//  * join_cwm_dv (:840-894, :240-283) keeps the surviving rows as (OID,
//    groupID) lists in row order; here one order-preserving compaction;
//  * agg_cwm_dv (:685-752, :645-655) sums M1[OID]+M2[OID] by groupID.
// Group ids are int16 there, so these entry points accept group_nums up to
// 32766 (GROUP_NULL is 32767).
//
// Star-join operator (code/starjoin/test_starjoin_option.cpp): the count of
// rows surviving four dimension probes (starjoinalgo_rowwise :37-50), the
// static vector of 4-bit packed group ids (starjoinalgo_cwm_sv :66-121:
// c<<12 + s<<8 + p<<4 + d, GROUP_NULL otherwise, count of entries that are
// not GROUP_NULL) and the compacted (position, group) pairs
// (starjoinalgo_cwm_dv :137-189).
#include <cstring>

#include "compact.cuh"

namespace olap {

struct DimSet {
  const int8_t* vec[OLAP_MAX_DIMS];
  const int32_t* fk[OLAP_MAX_DIMS];
  uint32_t len[OLAP_MAX_DIMS];
  int32_t mul[OLAP_MAX_DIMS];  // factor, or 1 << shift for the packed ids
  int32_t nd;
};

// Probe row r: -1 range error, 0 dropped (a DIM_NULL), 1 survived (*g set).
__device__ __forceinline__ int probe_row(const DimSet& d, int64_t r, int32_t* g) {
  uint32_t k[OLAP_MAX_DIMS];
  bool ok = true;
#pragma unroll
  for (int j = 0; j < OLAP_MAX_DIMS; ++j) {
    if (j < d.nd) {
      k[j] = static_cast<uint32_t>(d.fk[j][r]);
      ok &= k[j] < d.len[j];
    }
  }
  if (!ok) return -1;
  int32_t acc = 0;
#pragma unroll
  for (int j = 0; j < OLAP_MAX_DIMS; ++j) {
    if (j < d.nd) {
      const int32_t c = __ldg(d.vec[j] + k[j]);
      if (c == OLAP_DIM_NULL) return 0;
      acc += c * d.mul[j];
    }
  }
  *g = acc;
  return 1;
}

// join_cwm_sv: groupID[r] = sum code*factor (int16) or GROUP_NULL.
__global__ void join_cwm_sv_kernel(DimSet d, int64_t n, int16_t* __restrict__ gid, unsigned long long* range_err) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  unsigned int bad = 0;
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < n; r += stride) {
    int32_t g = 0;
    const int st = probe_row(d, r, &g);
    bad += st < 0;
    gid[r] = st > 0 ? static_cast<int16_t>(g) : static_cast<int16_t>(OLAP_GROUP_NULL);
  }
  if (bad) atomicAdd(range_err, static_cast<unsigned long long>(bad));
}

// agg_cwm_sv / agg_cwm_dv: group_vector[g] += M1[row] + M2[row].
__global__ void agg_cwm_kernel(const int16_t* __restrict__ gid, const int64_t* __restrict__ oid, int64_t n,
                               const int32_t* __restrict__ m1, const int32_t* __restrict__ m2, int64_t rows,
                               int64_t G, unsigned long long* __restrict__ gv, unsigned long long* total,
                               unsigned long long* range_err) {
  extern __shared__ unsigned long long sacc[];
  const bool smem = G * 8 <= 64 * 1024;
  for (int64_t i = threadIdx.x; smem && i < G; i += blockDim.x) sacc[i] = 0;
  __syncthreads();
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  int64_t tot = 0;
  unsigned int bad = 0;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
    const int32_t g = gid[i];
    if (g == OLAP_GROUP_NULL) continue;
    const int64_t row = oid ? oid[i] : i;
    if (g < 0 || g >= G || row < 0 || row >= rows) {
      ++bad;
      continue;
    }
    const int64_t v = static_cast<int64_t>(m1[row]) + m2[row];
    tot += v;
    if (smem) smem_add_u64(&sacc[g], static_cast<uint64_t>(v));
    else atomicAdd(&gv[g], static_cast<unsigned long long>(v));
  }
  tot = warp_sum_i64(tot);
  const unsigned int wbad = __reduce_add_sync(0xffffffffu, bad);
  if ((threadIdx.x & 31) == 0) {
    if (tot) atomicAdd(total, static_cast<unsigned long long>(tot));
    if (wbad) atomicAdd(range_err, static_cast<unsigned long long>(wbad));
  }
  __syncthreads();
  for (int64_t i = threadIdx.x; smem && i < G; i += blockDim.x)
    if (sacc[i]) atomicAdd(&gv[i], sacc[i]);
}

// join_cwm_dv and starjoinalgo_cwm_dv: surviving rows in row order.
struct SurvivorOp {
  static constexpr int kGroups = kCompactGroups;
  DimSet d;
  int64_t* oid64;        // join_cwm_dv: OID (int64)
  int16_t* gid16;        //              groupID (int16)
  int32_t* pos32;        // starjoin cwm_dv: position
  int32_t* grp32;        //                  group
  unsigned long long* range_err;
  int4 g[kCompactGroups];

  __device__ __forceinline__ bool vec_ok() const { return true; }
  __device__ __forceinline__ void prefetch(int, int64_t) {}
  template <bool kFull>
  __device__ __forceinline__ uint32_t flags(int u, int64_t first, int nv) {
    int32_t gg[4] = {0, 0, 0, 0};
    uint32_t m = 0;
    for (int k = 0; k < nv; ++k) {
      const int st = probe_row(d, first + k, &gg[k]);
      if (st < 0) atomicAdd(range_err, 1ull);
      if (st > 0) m |= 1u << k;
    }
    g[u] = make_int4(gg[0], gg[1], gg[2], gg[3]);
    return m;
  }
  __device__ __forceinline__ void emit(int u, int k, int64_t item, int64_t pos) {
    const int32_t v = k == 0 ? g[u].x : k == 1 ? g[u].y : k == 2 ? g[u].z : g[u].w;
    if (oid64) oid64[pos] = item;
    if (gid16) gid16[pos] = static_cast<int16_t>(v);
    if (pos32) pos32[pos] = static_cast<int32_t>(item);
    if (grp32) grp32[pos] = v;
  }
};

// starjoinalgo_cwm_sv: packed ids; counts entries that are not GROUP_NULL.
__global__ void starjoin_cwm_sv_kernel(DimSet d, int64_t n, int32_t* __restrict__ result,
                                       unsigned long long* count, unsigned long long* range_err) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  int64_t c = 0;
  unsigned int bad = 0;
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < n; r += stride) {
    int32_t g = 0;
    const int st = probe_row(d, r, &g);
    bad += st < 0;
    const int32_t v = st > 0 ? g : OLAP_GROUP_NULL;
    result[r] = v;
    c += v != OLAP_GROUP_NULL;
  }
  c = warp_sum_i64(c);
  const unsigned int wbad = __reduce_add_sync(0xffffffffu, bad);
  if ((threadIdx.x & 31) == 0) {
    if (c) atomicAdd(count, static_cast<unsigned long long>(c));
    if (wbad) atomicAdd(range_err, static_cast<unsigned long long>(wbad));
  }
}

static unsigned grid_n(const olap_ctx* ctx, int64_t n, int threads) {
  int64_t g = (n + threads - 1) / threads;
  const int64_t cap = static_cast<int64_t>(ctx->sm_count) * (2048 / threads);
  if (g > cap) g = cap;
  return static_cast<unsigned>(g < 1 ? 1 : g);
}

// Dimensions in probe order from the reference's table-indexed arrays.
static int make_dims(olap_ctx* ctx, int8_t* const* dimvec_array, const int64_t* dimvec_len,
                     int32_t* const* fk_array, const int* orders, int dimvec_nums, const int* factor,
                     bool empty, DimSet* d) {
  std::memset(d, 0, sizeof(*d));
  OLAP_REQUIRE(ctx, dimvec_nums >= 0 && dimvec_nums <= OLAP_MAX_DIMS, "dimvec_nums must be in [0, 4]");
  OLAP_REQUIRE(ctx, dimvec_nums == 0 || (dimvec_array && fk_array && orders && factor && dimvec_len),
               "null plan arrays");
  d->nd = dimvec_nums;
  for (int j = 0; j < dimvec_nums; ++j) {
    const int t = orders[j];
    OLAP_REQUIRE(ctx, t >= 0 && t < OLAP_MAX_DIMS, "orders[] entry must name table 0..3");
    OLAP_REQUIRE(ctx, dimvec_array[t] && (empty || fk_array[t]), "null dimension vector or fk column");
    OLAP_REQUIRE(ctx, dimvec_len[t] >= 1 && dimvec_len[t] <= INT32_MAX, "dimvec_len must be in [1, 2^31)");
    d->vec[j] = dimvec_array[t];
    d->fk[j] = fk_array[t];
    d->len[j] = static_cast<uint32_t>(dimvec_len[t]);
    d->mul[j] = factor[j];
  }
  return OLAP_OK;
}

}  // namespace olap

extern "C" {

int olap_join_cwm_sv(olap_ctx* ctx, int8_t* const* dimvec_array, const int64_t* dimvec_len,
                     int32_t* const* fk_array, const int* orders, int dimvec_nums, int16_t* groupID,
                     const int* factor, int64_t size_lineorder) {
  if (!ctx) return OLAP_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  OLAP_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  OLAP_REQUIRE(ctx, size_lineorder >= 0 && (size_lineorder == 0 || groupID), "bad output");
  olap::DimSet d;
  int st = olap::make_dims(ctx, dimvec_array, dimvec_len, fk_array, orders, dimvec_nums, factor,
                           size_lineorder == 0, &d);
  if (st != OLAP_OK || size_lineorder == 0) return st;
  olap::join_cwm_sv_kernel<<<olap::grid_n(ctx, size_lineorder, 256), 256, 0, ctx->stream>>>(
      d, size_lineorder, groupID, &ctx->counters->range_errors);
  OLAP_CUDA_TRY(ctx, cudaGetLastError());
  return OLAP_OK;
}

int olap_agg_cwm_sv(olap_ctx* ctx, const int16_t* groupID, int64_t size_lineorder, const int32_t* M1,
                    const int32_t* M2, int64_t group_nums, int64_t* group_vector, int64_t* d_count) {
  if (!ctx) return OLAP_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  OLAP_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  OLAP_REQUIRE(ctx, group_nums >= 1 && group_nums <= 32766, "group_nums must be in [1, 32766] (int16 ids)");
  OLAP_REQUIRE(ctx, size_lineorder >= 0 && group_vector && d_count, "bad arguments");
  OLAP_REQUIRE(ctx, size_lineorder == 0 || (groupID && M1 && M2), "null column");
  OLAP_CUDA_TRY(ctx, cudaMemsetAsync(group_vector, 0, sizeof(int64_t) * group_nums, ctx->stream));
  OLAP_CUDA_TRY(ctx, cudaMemsetAsync(d_count, 0, sizeof(int64_t), ctx->stream));
  if (size_lineorder == 0) return OLAP_OK;
  const size_t smem = group_nums * 8 <= 64 * 1024 ? static_cast<size_t>(group_nums * 8) : 0;
  OLAP_CUDA_TRY(ctx, cudaFuncSetAttribute(olap::agg_cwm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          64 * 1024));
  olap::agg_cwm_kernel<<<olap::grid_n(ctx, size_lineorder, 512), 512, smem, ctx->stream>>>(
      groupID, nullptr, size_lineorder, M1, M2, size_lineorder, group_nums,
      reinterpret_cast<unsigned long long*>(group_vector), reinterpret_cast<unsigned long long*>(d_count),
      &ctx->counters->range_errors);
  OLAP_CUDA_TRY(ctx, cudaGetLastError());
  return OLAP_OK;
}

int olap_join_cwm_dv(olap_ctx* ctx, int8_t* const* dimvec_array, const int64_t* dimvec_len,
                     int32_t* const* fk_array, const int* orders, int dimvec_nums, int64_t* OID,
                     int16_t* groupID, const int* factor, int64_t* d_index, int64_t size_lineorder) {
  if (!ctx) return OLAP_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  OLAP_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  OLAP_REQUIRE(ctx, size_lineorder >= 0 && d_index && (size_lineorder == 0 || (OID && groupID)), "bad output");
  olap::SurvivorOp op;
  std::memset(&op, 0, sizeof(op));
  int st = olap::make_dims(ctx, dimvec_array, dimvec_len, fk_array, orders, dimvec_nums, factor,
                           size_lineorder == 0, &op.d);
  if (st != OLAP_OK) return st;
  op.oid64 = OID;
  op.gid16 = groupID;
  op.range_err = &ctx->counters->range_errors;
  olap::Arena ar(ctx);
  olap::ScanTiles sc;
  st = olap::make_scan_tiles(ctx, ar, size_lineorder, reinterpret_cast<unsigned long long*>(d_index),
                             ctx->stream, &sc, olap::compact_tile_items<olap::SurvivorOp>());
  if (st != OLAP_OK) return st;
  olap::compact_kernel<olap::SurvivorOp><<<olap::compact_grid(ctx, sc.n_tiles), olap::kCompactThreads, 0,
                                          ctx->stream>>>(op, size_lineorder, sc);
  OLAP_CUDA_TRY(ctx, cudaGetLastError());
  return OLAP_OK;
}

int olap_agg_cwm_dv(olap_ctx* ctx, const int64_t* OID, const int16_t* groupID, int64_t index,
                    const int32_t* M1, const int32_t* M2, int64_t size_lineorder, int64_t group_nums,
                    int64_t* group_vector, int64_t* d_count) {
  if (!ctx) return OLAP_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  OLAP_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  OLAP_REQUIRE(ctx, group_nums >= 1 && group_nums <= 32766, "group_nums must be in [1, 32766] (int16 ids)");
  OLAP_REQUIRE(ctx, index >= 0 && group_vector && d_count, "bad arguments");
  OLAP_REQUIRE(ctx, index == 0 || (OID && groupID && M1 && M2), "null column");
  OLAP_CUDA_TRY(ctx, cudaMemsetAsync(group_vector, 0, sizeof(int64_t) * group_nums, ctx->stream));
  OLAP_CUDA_TRY(ctx, cudaMemsetAsync(d_count, 0, sizeof(int64_t), ctx->stream));
  if (index == 0) return OLAP_OK;
  const size_t smem = group_nums * 8 <= 64 * 1024 ? static_cast<size_t>(group_nums * 8) : 0;
  OLAP_CUDA_TRY(ctx, cudaFuncSetAttribute(olap::agg_cwm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          64 * 1024));
  olap::agg_cwm_kernel<<<olap::grid_n(ctx, index, 512), 512, smem, ctx->stream>>>(
      groupID, OID, index, M1, M2, size_lineorder, group_nums,
      reinterpret_cast<unsigned long long*>(group_vector), reinterpret_cast<unsigned long long*>(d_count),
      &ctx->counters->range_errors);
  OLAP_CUDA_TRY(ctx, cudaGetLastError());
  return OLAP_OK;
}

int olap_starjoin_count(olap_ctx* ctx, int64_t size_lineorder, int8_t* const* dimvec, const int64_t* dimvec_len,
                        int32_t* const* fk, int64_t* d_count) {
  if (!ctx) return OLAP_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  OLAP_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  OLAP_REQUIRE(ctx, dimvec && dimvec_len && fk && d_count, "null argument");
  olap_starjoin_query q;
  std::memset(&q, 0, sizeof(q));
  q.dimvec_nums = OLAP_MAX_DIMS;
  q.n_aggs = 1;
  q.agg[0] = OLAP_AGG_COUNT;
  for (int j = 0; j < OLAP_MAX_DIMS; ++j) {
    q.dimvec[j] = dimvec[j];
    q.dimvec_len[j] = dimvec_len[j];
    q.fk[j] = fk[j];
    q.factor[j] = 0;
  }
  q.row_begin = 0;
  q.row_end = size_lineorder;
  q.group_nums = 1;
  olap::Arena ar(ctx);
  return olap::starjoin_device(ctx, &q, nullptr, d_count, false, ctx->stream, ar);
}

int olap_starjoin_cwm_sv(olap_ctx* ctx, int64_t size_lineorder, int8_t* const* dimvec,
                         const int64_t* dimvec_len, int32_t* const* fk, int32_t* result, int64_t* d_count) {
  if (!ctx) return OLAP_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  OLAP_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  OLAP_REQUIRE(ctx, dimvec && dimvec_len && fk && d_count && size_lineorder >= 0, "null argument");
  OLAP_REQUIRE(ctx, size_lineorder == 0 || result, "null result");
  const int orders[4] = {0, 1, 2, 3};
  const int shifts[4] = {1 << 12, 1 << 8, 1 << 4, 1};  // GROUP_BITS_TABLE = 4 (metadata.h:76)
  olap::DimSet d;
  int st = olap::make_dims(ctx, dimvec, dimvec_len, fk, orders, 4, shifts, size_lineorder == 0, &d);
  if (st != OLAP_OK) return st;
  OLAP_CUDA_TRY(ctx, cudaMemsetAsync(d_count, 0, sizeof(int64_t), ctx->stream));
  if (size_lineorder == 0) return OLAP_OK;
  olap::starjoin_cwm_sv_kernel<<<olap::grid_n(ctx, size_lineorder, 256), 256, 0, ctx->stream>>>(
      d, size_lineorder, result, reinterpret_cast<unsigned long long*>(d_count), &ctx->counters->range_errors);
  OLAP_CUDA_TRY(ctx, cudaGetLastError());
  return OLAP_OK;
}

int olap_starjoin_cwm_dv(olap_ctx* ctx, int64_t size_lineorder, int8_t* const* dimvec,
                         const int64_t* dimvec_len, int32_t* const* fk, int32_t* out_pos,
                         int32_t* out_group, int64_t* d_count) {
  if (!ctx) return OLAP_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  OLAP_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  OLAP_REQUIRE(ctx, dimvec && dimvec_len && fk && d_count && size_lineorder >= 0 && size_lineorder <= INT32_MAX,
               "bad argument");
  OLAP_REQUIRE(ctx, size_lineorder == 0 || (out_pos && out_group), "null output");
  const int orders[4] = {0, 1, 2, 3};
  const int shifts[4] = {1 << 12, 1 << 8, 1 << 4, 1};
  olap::SurvivorOp op;
  std::memset(&op, 0, sizeof(op));
  int st = olap::make_dims(ctx, dimvec, dimvec_len, fk, orders, 4, shifts, size_lineorder == 0, &op.d);
  if (st != OLAP_OK) return st;
  op.pos32 = out_pos;
  op.grp32 = out_group;
  op.range_err = &ctx->counters->range_errors;
  olap::Arena ar(ctx);
  olap::ScanTiles sc;
  st = olap::make_scan_tiles(ctx, ar, size_lineorder, reinterpret_cast<unsigned long long*>(d_count),
                             ctx->stream, &sc, olap::compact_tile_items<olap::SurvivorOp>());
  if (st != OLAP_OK) return st;
  olap::compact_kernel<olap::SurvivorOp><<<olap::compact_grid(ctx, sc.n_tiles), olap::kCompactThreads, 0,
                                          ctx->stream>>>(op, size_lineorder, sc);
  OLAP_CUDA_TRY(ctx, cudaGetLastError());
  return OLAP_OK;
}

}  // extern "C"
