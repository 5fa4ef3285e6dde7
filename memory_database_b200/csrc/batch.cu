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
// The batched kernel runs Q such queries in one persistent launch over the
// shared fact table.  Each fact row is read once and each dimension it
// references is probed once (one 8-byte attribute record per key, kept hot in
// L2): the per-query work is then register arithmetic — the range tests, the
// group id and the fact-range test — followed by an int64 atomic into the
// query's own group vector for the rows that pass.  Per query the result is
// bit-identical to the plain star-join over the dimension vectors that
// olap_build_dimvec builds for it.
#include <cstdlib>
#include <cstring>

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
  int32_t lo[OLAP_MAX_DIMS];      // filter range [lo, hi) per table; lo > hi: table unused
  int32_t hi[OLAP_MAX_DIMS];
  int32_t factor[OLAP_MAX_DIMS];  // group weight per table (0: not a group dimension)
  int32_t uses;                   // bit t: table t participates
  int32_t grouped;                // bit t: table t contributes its group attribute
  int64_t group_nums;
  int64_t out_offset;             // first slot of this query in the shared output
};

struct BatchParams {
  const int2* attrs[OLAP_MAX_DIMS];   // packed attribute records per table
  uint32_t dim_len[OLAP_MAX_DIMS];
  const int32_t* fk[OLAP_MAX_DIMS];
  const int32_t* m1;
  const int32_t* m2;
  int64_t n_rows;
  const BatchQuery* queries;
  int32_t n_queries;
  int32_t tables_used;                // union of the queries' `uses`
  int32_t agg;                        // OLAP_AGG_* of every query (one aggregate)
  unsigned long long* out;            // concatenated group vectors
  unsigned long long* totals;         // [n_queries]
  unsigned long long* range_err;
};

constexpr int kBatchThreads = 512;
constexpr int kMaxBatchQueries = 256;

__device__ __forceinline__ int64_t batch_value(int agg, int32_t x, int32_t y) {
  switch (agg) {
    case OLAP_AGG_M1_PLUS_M2: return static_cast<int64_t>(x) + y;
    case OLAP_AGG_M1: return x;
    case OLAP_AGG_M2: return y;
    case OLAP_AGG_M1_TIMES_M2: return static_cast<int64_t>(x) * y;
    default: return 1;
  }
}

// Persistent: SMs x blocks, each thread 4 rows per step (128-bit loads), the
// query descriptors in shared memory, queries evaluated in a uniform loop.
__global__ void __launch_bounds__(kBatchThreads) batch_starjoin_kernel(const BatchParams p) {
  __shared__ BatchQuery sq[kMaxBatchQueries];
  __shared__ unsigned long long stot[kMaxBatchQueries];
  __shared__ unsigned int s_bad;
  const int tid = threadIdx.x;
  const int nq = p.n_queries;
  for (int i = tid; i < nq; i += blockDim.x) {
    sq[i] = p.queries[i];
    stot[i] = 0;
  }
  if (tid == 0) s_bad = 0;
  __syncthreads();
  const uint64_t pol_stream = policy_evict_first();
  const uint64_t pol_keep = policy_evict_last();
  const int agg = p.agg;
  const bool need_m1 = agg == OLAP_AGG_M1_PLUS_M2 || agg == OLAP_AGG_M1 || agg == OLAP_AGG_M1_TIMES_M2;
  const bool need_m2 = agg == OLAP_AGG_M1_PLUS_M2 || agg == OLAP_AGG_M2 || agg == OLAP_AGG_M1_TIMES_M2;
  unsigned int bad = 0;
  const int64_t n4 = p.n_rows >> 2;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  // Rows 4i..4i+3 (the tail of n_rows % 4 rows is taken by i == n4).
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + tid; i <= n4; i += stride) {
    const int64_t r0 = 4 * i;
    const int nv = r0 + 4 <= p.n_rows ? 4 : static_cast<int>(p.n_rows - r0);
    if (nv <= 0) continue;
    int32_t key[OLAP_MAX_DIMS][4];
    int32_t x[4] = {0, 0, 0, 0}, y[4] = {0, 0, 0, 0};
    const bool full = nv == 4;
#pragma unroll
    for (int t = 0; t < OLAP_MAX_DIMS; ++t) {
      if (!((p.tables_used >> t) & 1)) continue;
      if (full) {
        const int4 v = ld_stream_v4(p.fk[t] + r0, pol_stream);
        key[t][0] = v.x; key[t][1] = v.y; key[t][2] = v.z; key[t][3] = v.w;
      } else {
        for (int k = 0; k < 4; ++k) key[t][k] = k < nv ? p.fk[t][r0 + k] : 0;
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
    // One attribute probe per (row, table), shared by every query.
    int2 at[OLAP_MAX_DIMS][4];
    uint32_t valid = nv == 4 ? 0xFu : ((1u << nv) - 1u);
    uint32_t inb[OLAP_MAX_DIMS];
#pragma unroll
    for (int t = 0; t < OLAP_MAX_DIMS; ++t) {
      inb[t] = 0;
      if (!((p.tables_used >> t) & 1)) continue;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const bool ok = ((valid >> k) & 1) && static_cast<uint32_t>(key[t][k]) < p.dim_len[t];
        inb[t] |= static_cast<uint32_t>(ok) << k;
        at[t][k] = ok ? ld_probe_i2(p.attrs[t] + key[t][k], pol_keep) : make_int2(0, 0);
      }
    }
    for (int q = 0; q < nq; ++q) {
      const BatchQuery& Q = sq[q];
      uint32_t live = valid;
      // fact range
#pragma unroll
      for (int k = 0; k < 4; ++k)
        if (r0 + k < Q.row_begin || r0 + k >= Q.row_end) live &= ~(1u << k);
      if (!live) continue;
      // Every key the query uses is range-checked first (as in the plain
      // star-join), then the predicates and the group id.
      uint32_t oob = 0;
#pragma unroll
      for (int t = 0; t < OLAP_MAX_DIMS; ++t)
        if ((Q.uses >> t) & 1) oob |= live & ~inb[t];
      bad += __popc(oob);
      live &= ~oob;
      if (!live) continue;
      int32_t g[4] = {0, 0, 0, 0};
#pragma unroll
      for (int t = 0; t < OLAP_MAX_DIMS; ++t) {
        if (!((Q.uses >> t) & 1)) continue;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          bool pass = at[t][k].x >= Q.lo[t] && at[t][k].x < Q.hi[t];
          if ((Q.grouped >> t) & 1) {
            // a group value that is not an int8 code is DIM_NULL in the
            // dimension vector the plain path would build
            pass &= static_cast<uint32_t>(at[t][k].y) < static_cast<uint32_t>(OLAP_DIM_NULL);
            g[k] += at[t][k].y * Q.factor[t];
          }
          if (!pass) live &= ~(1u << k);
        }
      }
      if (!live) continue;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        if (!((live >> k) & 1)) continue;
        if (static_cast<uint64_t>(static_cast<int64_t>(g[k])) >= static_cast<uint64_t>(Q.group_nums)) {
          ++bad;
          continue;
        }
        const int64_t v = batch_value(agg, x[k], y[k]);
        atomicAdd(&p.out[Q.out_offset + g[k]], static_cast<unsigned long long>(v));
        atomicAdd(&stot[q], static_cast<unsigned long long>(v));
      }
    }
  }
  const unsigned int wbad = __reduce_add_sync(0xffffffffu, bad);
  if ((tid & 31) == 0 && wbad) atomicAdd(&s_bad, wbad);
  __syncthreads();
  for (int i = tid; i < nq; i += blockDim.x)
    if (stot[i]) atomicAdd(&p.totals[i], stot[i]);
  if (tid == 0 && s_bad) atomicAdd(p.range_err, static_cast<unsigned long long>(s_bad));
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
// one runs; packed attribute records per table.
struct olap_batch {
  olap_ctx* ctx = nullptr;
  int max_queries = 0;
  olap::BatchQuery* d_queries[2] = {};  // device
  olap::BatchQuery* h_queries[2] = {};  // pinned host staging
  cudaEvent_t done[2] = {};             // recorded after each slot's batch
  bool pending[2] = {false, false};
  cudaGraph_t graph[2] = {};
  cudaGraphExec_t exec[2] = {};
  olap::BatchParams params[2];
  int64_t out_slots[2] = {0, 0};
  bool have_params[2] = {false, false};
  int64_t runs = 0;
  int2* attrs[OLAP_MAX_DIMS] = {};
  int64_t attr_len[OLAP_MAX_DIMS] = {};
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
    ok &= cudaMalloc(&b->d_queries[s], sizeof(olap::BatchQuery) * max_queries) == cudaSuccess;
    ok &= cudaMallocHost(&b->h_queries[s], sizeof(olap::BatchQuery) * max_queries) == cudaSuccess;
    ok &= cudaEventCreateWithFlags(&b->done[s], cudaEventDisableTiming) == cudaSuccess;
  }
  if (!ok) {
    cudaGetLastError();
    for (int s = 0; s < 2; ++s) {
      if (b->d_queries[s]) cudaFree(b->d_queries[s]);
      if (b->h_queries[s]) cudaFreeHost(b->h_queries[s]);
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
    cudaFree(b->d_queries[s]);
    cudaFreeHost(b->h_queries[s]);
    cudaEventDestroy(b->done[s]);
  }
  for (int t = 0; t < OLAP_MAX_DIMS; ++t)
    if (b->attrs[t]) cudaFree(b->attrs[t]);
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
    if (b->attrs[table]) {
      for (int s = 0; s < 2; ++s)
        if (b->pending[s]) cudaEventSynchronize(b->done[s]);
      cudaStreamSynchronize(ctx->stream);
      cudaFree(b->attrs[table]);
      b->attrs[table] = nullptr;
    }
    OLAP_CUDA_TRY(ctx, cudaMalloc(&b->attrs[table], sizeof(int2) * n));
    b->attr_len[table] = n;
  }
  olap::pack_dim_attrs_kernel<<<olap::grid_n(ctx, n, 256), 256, 0, ctx->stream>>>(filter_attr, group_attr, n,
                                                                                 b->attrs[table]);
  OLAP_CUDA_TRY(ctx, cudaGetLastError());
  b->have_params[0] = b->have_params[1] = false;  // recorded graphs refer to the old records
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
  int tables = 0;
  int64_t off = 0;
  for (int q = 0; q < n_queries; ++q) {
    const olap_batch_query& in = queries[q];
    olap::BatchQuery& d = b->h_queries[slot][q];
    std::memset(&d, 0, sizeof(d));
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
        if (in.grouped & (1 << t)) {
          d.grouped |= 1 << t;
          gbound += 128 * std::llabs(static_cast<long long>(in.factor[t]));
        }
      }
    }
    OLAP_REQUIRE(ctx, gbound <= INT32_MAX, "group factors too large");
    tables |= d.uses;
    off += in.group_nums;
  }
  OLAP_REQUIRE(ctx, off <= out_slots, "out holds fewer slots than the queries' groups");
  olap::BatchParams p;
  std::memset(&p, 0, sizeof(p));
  for (int t = 0; t < OLAP_MAX_DIMS; ++t) {
    p.attrs[t] = b->attrs[t];
    p.dim_len[t] = static_cast<uint32_t>(b->attr_len[t]);
    p.fk[t] = fk[t];
  }
  p.m1 = m1;
  p.m2 = m2;
  p.n_rows = n_rows;
  p.queries = b->d_queries[slot];
  p.n_queries = n_queries;
  p.tables_used = tables;
  p.agg = agg;
  p.out = reinterpret_cast<unsigned long long*>(out);
  p.totals = reinterpret_cast<unsigned long long*>(totals);
  p.range_err = &ctx->counters->range_errors;
  const bool need_m = agg != OLAP_AGG_COUNT;
  OLAP_REQUIRE(ctx, !need_m || n_rows == 0 || (m1 || m2), "measure columns required");
  int bps = 1;
  OLAP_CUDA_TRY(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, olap::batch_starjoin_kernel,
                                                                   olap::kBatchThreads, 0));
  const unsigned grid = static_cast<unsigned>(ctx->sm_count) * static_cast<unsigned>(bps < 1 ? 1 : bps);
  // The work of one batch: descriptors H2D, zero outputs, one persistent launch.
  auto enqueue = [&](cudaStream_t s) -> cudaError_t {
    cudaError_t e = cudaMemcpyAsync(b->d_queries[slot], b->h_queries[slot],
                                    sizeof(olap::BatchQuery) * n_queries, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(out, 0, sizeof(int64_t) * off, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(totals, 0, sizeof(int64_t) * n_queries, s);
    if (e == cudaSuccess && n_rows > 0) {
      olap::batch_starjoin_kernel<<<grid, olap::kBatchThreads, 0, s>>>(p);
      e = cudaGetLastError();
    }
    return e;
  };
  if (!use_graph) {
    OLAP_CUDA_TRY(ctx, enqueue(ctx->stream));
  } else {
    // Graph of this slot: re-captured when the launch parameters change,
    // replayed otherwise (its copy node reads the slot's pinned staging).
    const bool same = b->have_params[slot] && b->exec[slot] &&
                      std::memcmp(&b->params[slot], &p, sizeof(p)) == 0 && b->out_slots[slot] == off;
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
      b->out_slots[slot] = off;
      b->have_params[slot] = true;
    }
    OLAP_CUDA_TRY(ctx, cudaGraphLaunch(b->exec[slot], ctx->stream));
  }
  OLAP_CUDA_TRY(ctx, cudaEventRecord(b->done[slot], ctx->stream));
  b->pending[slot] = true;
  ++b->runs;
  return OLAP_OK;
}

}  // extern "C"
