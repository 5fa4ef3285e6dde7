// In-place star-join over pinned host columns: late materialisation over PCIe.
//
// The host-memory entry point of the OLAP core (the reference's
// OLAPcore_vwm_sv, code/OLAPcore/test_multi_compute_operator.cpp:1258-1327,
// whose per-row contract is OLAPcore_vwm_sv_thread, :509-568) otherwise
// streams every fact column through the GPU, 24 bytes per row for four keys
// and two measures, so it runs at the speed of the PCIe link.  When the
// columns sit in pinned, device-mapped host memory this kernel reads them
// where they are, and only as far as the rows need them:
//  * dimensions are probed in ascending order of the fraction of their
//    entries that pass (counted on the device per call), so the one foreign-
//    key column read whole is the most selective one;
//  * every later column, foreign keys first and the measures last, is loaded
//    by a thread (16 bytes, its four rows) only while one of its rows is
//    alive, so a 32-byte host sector crosses the link only when one of its
//    eight rows still needs it;
//  * the dimension vectors are copied to the device once per call and probed
//    through L2; group sums accumulate in shared memory (flushed once per
//    block) or with L2 atomics.
// The sums and the dropped-row count equal the streaming path's: a row with a
// key out of range is never accumulated, and it keeps reading its later keys
// (it is rare) so that it counts as a range error exactly when none of its
// in-range keys meets DIM_NULL, the rule every star-join path shares.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>

#include "olap_internal.cuh"

namespace olap {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kHostScanThreads = 512;
// In place only when it reads at most this share of the columns' sectors:
// dense in-place reads run at about 93 % of the copy engines' rate.
constexpr double kInplaceMaxShare = 0.85;

struct HostDim {
  const int8_t* vec;   // device copy of the dimension vector
  const int32_t* fk;   // device address of the pinned host column
  uint32_t len;
  int32_t factor;
};

struct HostScanParams {
  HostDim dim[OLAP_MAX_DIMS];  // in probe order
  const int32_t* m1;           // device addresses of the host measures (null: unused)
  const int32_t* m2;
  int64_t row_begin, row_end;
  int64_t vec_begin;           // first row read with 16-byte loads
  uint32_t nvec;               // 16-byte vectors (4 rows) from vec_begin
  int64_t n_groups;
  unsigned long long* out;     // [n_aggs][n_groups]
  unsigned long long* totals;  // [n_aggs]
  unsigned long long* range_err;
  unsigned long long* sectors;
  int32_t n_aggs, agg0, agg1;
};

// 16-byte load from host memory.  volatile keeps it inside its branch: a
// thread whose rows are all dead must not touch the link.
__device__ __forceinline__ int4 ld_host_v4(const int32_t* p) {
  int4 v;
  asm volatile("ld.global.nc.L1::no_allocate.v4.s32 {%0,%1,%2,%3}, [%4];"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "l"(p));
  return v;
}

// Distinct 32-byte sectors among a warp's 16-byte loads, lane l reading p
// (addresses rising by 16 bytes per lane) when `need`.
__device__ __forceinline__ uint32_t warp_sectors(const void* p, bool need, int lane) {
  const uint32_t m = __ballot_sync(kFull, need);
  const uint32_t s = static_cast<uint32_t>(reinterpret_cast<uintptr_t>(p) >> 5);
  const uint32_t sp = __shfl_up_sync(kFull, s, 1);
  const bool first = need && (lane == 0 || !((m >> (lane - 1)) & 1u) || sp != s);
  return __popc(__ballot_sync(kFull, first));
}

__global__ void count_live_kernel(const int8_t* __restrict__ vec, uint32_t len, unsigned long long* cnt) {
  uint32_t c = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < len; i += gridDim.x * blockDim.x)
    c += vec[i] != OLAP_DIM_NULL ? 1u : 0u;
  c = __reduce_add_sync(kFull, c);
  if ((threadIdx.x & 31) == 0 && c) atomicAdd(cnt, static_cast<unsigned long long>(c));
}

template <int ND, bool SACC>
__global__ void __launch_bounds__(kHostScanThreads) starjoin_hostscan_kernel(const HostScanParams p) {
  extern __shared__ __align__(16) unsigned long long sacc[];
  __shared__ long long red[kHostScanThreads / 32][2];
  __shared__ unsigned int red_bad, red_sec;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t nacc = p.n_groups * p.n_aggs;
  if (tid == 0) {
    red_bad = 0;
    red_sec = 0;
  }
  if (SACC)
    for (int64_t i = tid; i < nacc; i += blockDim.x) sacc[i] = 0ull;
  __syncthreads();
  const uint64_t pol_keep = policy_evict_last();
  const uint64_t n_groups = static_cast<uint64_t>(p.n_groups);
  int64_t tot0 = 0, tot1 = 0;
  uint32_t bad = 0, sec = 0;

  auto add_row = [&](int64_t g, int32_t x, int32_t y) {
    if (static_cast<uint64_t>(g) >= n_groups) {
      ++bad;
      return;
    }
    const int64_t v0 = agg_value(p.agg0, x, y);
    tot0 += v0;
    if (SACC) smem_add_split(reinterpret_cast<uint32_t*>(sacc), nacc, g, static_cast<uint64_t>(v0));
    else atomicAdd(&p.out[g], static_cast<unsigned long long>(v0));
    if (p.n_aggs > 1) {
      const int64_t v1 = agg_value(p.agg1, x, y);
      tot1 += v1;
      if (SACC) smem_add_split(reinterpret_cast<uint32_t*>(sacc), nacc, n_groups + g, static_cast<uint64_t>(v1));
      else atomicAdd(&p.out[n_groups + g], static_cast<unsigned long long>(v1));
    }
  };

  // Loop bound and every ballot are warp-uniform (w0 is the warp's first vector).
  const uint32_t gstride = gridDim.x * blockDim.x;
  for (uint32_t w0 = blockIdx.x * blockDim.x + (tid & ~31u); w0 < p.nvec; w0 += gstride) {
    const bool in = w0 + lane < p.nvec;
    const uint32_t i = in ? w0 + lane : p.nvec - 1;  // lanes past the end keep a valid address
    const int64_t at = p.vec_begin + 4ll * i;
    uint32_t alive = in ? 0xFu : 0u;
    uint32_t oob = 0;  // rows with a key out of range: read on, never accumulated
    int64_t g[4] = {0, 0, 0, 0};
#pragma unroll
    for (int j = 0; j < ND; ++j) {
      if (!__any_sync(kFull, alive != 0)) break;
      const HostDim& d = p.dim[j];
      const int32_t* src = d.fk + at;
      const bool need = alive != 0;
      int4 k = make_int4(0, 0, 0, 0);
      if (need) k = ld_host_v4(src);
      const uint32_t ns = warp_sectors(src, need, lane);
      if (lane == 0) sec += ns;
      const uint32_t kk[4] = {static_cast<uint32_t>(k.x), static_cast<uint32_t>(k.y),
                              static_cast<uint32_t>(k.z), static_cast<uint32_t>(k.w)};
      int32_t c[4];
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const bool live = (alive >> r) & 1u;
        const bool inr = kk[r] < d.len;
        if (live && !inr) oob |= 1u << r;
        const bool a = live && inr;
        const uint32_t kp = a ? kk[r] : 0u;  // in bounds whether or not the load is predicated
        c[r] = a ? ld_probe_s8(d.vec + kp, pol_keep) : (live ? 0 : OLAP_DIM_NULL);
      }
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        if (c[r] == OLAP_DIM_NULL) alive &= ~(1u << r);
        else g[r] += static_cast<int64_t>(c[r]) * d.factor;
      }
    }
    bad += __popc(alive & oob);
    alive &= ~oob;
    if (!__any_sync(kFull, alive != 0)) continue;
    const bool need = alive != 0;
    int4 x = make_int4(0, 0, 0, 0), y = make_int4(0, 0, 0, 0);
    if (p.m1) {
      const int32_t* src = p.m1 + at;
      if (need) x = ld_host_v4(src);
      const uint32_t ns = warp_sectors(src, need, lane);
      if (lane == 0) sec += ns;
    }
    if (p.m2) {
      const int32_t* src = p.m2 + at;
      if (need) y = ld_host_v4(src);
      const uint32_t ns = warp_sectors(src, need, lane);
      if (lane == 0) sec += ns;
    }
    const int32_t xs[4] = {x.x, x.y, x.z, x.w}, ys[4] = {y.x, y.y, y.z, y.w};
#pragma unroll
    for (int r = 0; r < 4; ++r)
      if ((alive >> r) & 1u) add_row(g[r], xs[r], ys[r]);
  }

  // Rows before the first 16-byte boundary and after the last vector (block 0;
  // each 4-byte read counted as one sector).
  if (blockIdx.x == 0) {
    auto one = [&](int64_t r) {
      int64_t gg = 0;
      bool oob1 = false;
#pragma unroll
      for (int j = 0; j < ND; ++j) {
        const uint32_t k = static_cast<uint32_t>(p.dim[j].fk[r]);
        ++sec;
        if (k >= p.dim[j].len) {
          oob1 = true;
          continue;
        }
        const int32_t c = p.dim[j].vec[k];
        if (c == OLAP_DIM_NULL) return;
        gg += static_cast<int64_t>(c) * p.dim[j].factor;
      }
      if (oob1) {
        ++bad;
        return;
      }
      const int32_t x = p.m1 ? p.m1[r] : 0, y = p.m2 ? p.m2[r] : 0;
      sec += (p.m1 ? 1u : 0u) + (p.m2 ? 1u : 0u);
      add_row(gg, x, y);
    };
    for (int64_t r = p.row_begin + tid; r < p.vec_begin; r += blockDim.x) one(r);
    for (int64_t r = p.vec_begin + 4ll * p.nvec + tid; r < p.row_end; r += blockDim.x) one(r);
  }

  tot0 = warp_sum_i64(tot0);
  tot1 = warp_sum_i64(tot1);
  const unsigned int wbad = __reduce_add_sync(kFull, bad);
  const unsigned int wsec = __reduce_add_sync(kFull, sec);
  if (lane == 0) {
    red[warp][0] = tot0;
    red[warp][1] = tot1;
    if (wbad) atomicAdd(&red_bad, wbad);
    if (wsec) atomicAdd(&red_sec, wsec);
  }
  __syncthreads();
  if (warp == 0) {
    const int nw = blockDim.x >> 5;
    long long s0 = lane < nw ? red[lane][0] : 0;
    long long s1 = lane < nw ? red[lane][1] : 0;
    s0 = warp_sum_i64(s0);
    s1 = warp_sum_i64(s1);
    if (lane == 0) {
      if (s0) atomicAdd(&p.totals[0], static_cast<unsigned long long>(s0));
      if (p.n_aggs > 1 && s1) atomicAdd(&p.totals[1], static_cast<unsigned long long>(s1));
      if (red_bad) atomicAdd(p.range_err, static_cast<unsigned long long>(red_bad));
      if (red_sec) atomicAdd(p.sectors, static_cast<unsigned long long>(red_sec));
    }
  }
  if (SACC) {
    for (int64_t i = tid; i < nacc; i += blockDim.x) {
      const unsigned long long v = smem_split_get(reinterpret_cast<const uint32_t*>(sacc), nacc, i);
      if (v) atomicAdd(&p.out[i], v);
    }
  }
}

using HostScanKernel = void (*)(const HostScanParams);

template <bool SACC>
HostScanKernel pick_hostscan(int nd) {
  switch (nd) {
    case 0: return starjoin_hostscan_kernel<0, SACC>;
    case 1: return starjoin_hostscan_kernel<1, SACC>;
    case 2: return starjoin_hostscan_kernel<2, SACC>;
    case 3: return starjoin_hostscan_kernel<3, SACC>;
    default: return starjoin_hostscan_kernel<4, SACC>;
  }
}

// Device address of a pinned host pointer, or null (pageable or device memory).
const int32_t* mapped_host(const int32_t* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  if (a.type != cudaMemoryTypeHost || a.devicePointer == nullptr) return nullptr;
  return static_cast<const int32_t*>(a.devicePointer);
}

}  // namespace

int starjoin_host_inplace(olap_ctx* ctx, const olap_starjoin_query* q, const olap_starjoin_query& dq, Arena& ar,
                          int64_t* group_sums, int64_t* totals, bool* handled) {
  *handled = false;
  const int nd = q->dimvec_nums;
  bool need_m1 = false, need_m2 = false;
  for (int a = 0; a < q->n_aggs; ++a) {
    const int ag = q->agg[a];
    need_m1 |= (ag == OLAP_AGG_M1_PLUS_M2 || ag == OLAP_AGG_M1 || ag == OLAP_AGG_M1_TIMES_M2);
    need_m2 |= (ag == OLAP_AGG_M1_PLUS_M2 || ag == OLAP_AGG_M2 || ag == OLAP_AGG_M1_TIMES_M2);
  }
  // Every column device-mapped, all at one 16-byte phase at row_begin.
  const int32_t* dfk[OLAP_MAX_DIMS] = {};
  const int32_t* dm1 = nullptr;
  const int32_t* dm2 = nullptr;
  int phase = -1;
  auto map = [&](const int32_t* h, const int32_t** out) -> bool {
    if (!h) return false;
    const int32_t* d = mapped_host(h);
    if (!d) return false;
    const int ph = static_cast<int>(reinterpret_cast<uintptr_t>(d + q->row_begin) & 15);
    if (phase >= 0 && ph != phase) return false;
    phase = ph;
    *out = d;
    return true;
  };
  for (int j = 0; j < nd; ++j)
    if (!map(q->fk[j], &dfk[j])) return OLAP_OK;
  if (need_m1 && !map(q->m1, &dm1)) return OLAP_OK;
  if (need_m2 && !map(q->m2, &dm2)) return OLAP_OK;
  if (phase < 0 || (phase & 3)) return OLAP_OK;
  const int64_t rows = q->row_end - q->row_begin;
  const int64_t head = std::min<int64_t>(rows, ((16 - phase) & 15) / 4);
  const int64_t vec_begin = q->row_begin + head;
  const int64_t nvec = (q->row_end - vec_begin) / 4;
  if (nvec > (int64_t(1) << 31)) return OLAP_OK;
  *handled = true;
  for (int j = 0; j < nd; ++j)
    OLAP_REQUIRE(ctx, dq.dimvec_len[j] >= 1 && dq.dimvec_len[j] <= INT32_MAX, "dimvec_len must be in [1, 2^31)");

  // Probe order: ascending fraction of passing dimension entries.  Scratch
  // taken before the decision below is given back when the call declines, so
  // the copy path that then runs finds the arena as it was.
  const size_t arena_mark = ar.off;
  unsigned long long* cnt = ar.take<unsigned long long>(OLAP_MAX_DIMS);
  if (!cnt) return set_error(ctx, OLAP_ERR_CAPACITY, "scratch arena too small for the in-place scan");
  OLAP_CUDA_TRY(ctx, cudaMemsetAsync(cnt, 0, sizeof(unsigned long long) * OLAP_MAX_DIMS, ctx->stream));
  for (int j = 0; j < nd; ++j) {
    const uint32_t len = static_cast<uint32_t>(dq.dimvec_len[j]);
    const int grid = static_cast<int>(std::min<int64_t>(int64_t(ctx->sm_count) * 4, (len + 255) / 256));
    count_live_kernel<<<grid, 256, 0, ctx->stream>>>(dq.dimvec[j], len, cnt + j);
  }
  OLAP_CUDA_TRY(ctx, cudaGetLastError());
  unsigned long long live[OLAP_MAX_DIMS] = {0, 0, 0, 0};
  OLAP_CUDA_TRY(ctx, cudaMemcpyAsync(live, cnt, sizeof(live), cudaMemcpyDeviceToHost, ctx->stream));
  OLAP_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  int order[OLAP_MAX_DIMS] = {0, 1, 2, 3};
  std::stable_sort(order, order + nd, [&](int a, int b) {
    return static_cast<double>(live[a]) / static_cast<double>(dq.dimvec_len[a]) <
           static_cast<double>(live[b]) / static_cast<double>(dq.dimvec_len[b]);
  });
  // Expected share of the columns' 32-byte sectors read in place (eight rows
  // per sector, keys taken as uniform over the dimension entries).  Dense
  // reads over PCIe are slower than the copy engines, so a query whose
  // filters keep nearly every row takes the copies.
  {
    double alive = 1.0, sectors = 0.0;
    for (int t = 0; t < nd; ++t) {
      sectors += 1.0 - std::pow(1.0 - alive, 8.0);
      alive *= static_cast<double>(live[order[t]]) / static_cast<double>(dq.dimvec_len[order[t]]);
    }
    const int nm = (dm1 ? 1 : 0) + (dm2 ? 1 : 0);
    sectors += nm * (1.0 - std::pow(1.0 - alive, 8.0));
    if (tune_or(ctx, TUNE_HOST_INPLACE, 1) != 3 && sectors > kInplaceMaxShare * (nd + nm)) {
      ar.off = arena_mark;
      *handled = false;
      return OLAP_OK;
    }
  }
  const int64_t nacc = q->group_nums * q->n_aggs;
  int64_t* dsum = ar.take<int64_t>(static_cast<size_t>(nacc));
  int64_t* dtot = ar.take<int64_t>(2);
  if (!dsum || !dtot) return set_error(ctx, OLAP_ERR_CAPACITY, "scratch arena too small for the in-place scan");
  OLAP_CUDA_TRY(ctx, cudaMemsetAsync(dsum, 0, sizeof(int64_t) * nacc, ctx->stream));
  OLAP_CUDA_TRY(ctx, cudaMemsetAsync(dtot, 0, sizeof(int64_t) * 2, ctx->stream));

  HostScanParams hp;
  std::memset(&hp, 0, sizeof(hp));
  for (int t = 0; t < nd; ++t) {
    const int j = order[t];
    hp.dim[t].vec = dq.dimvec[j];
    hp.dim[t].fk = dfk[j];
    hp.dim[t].len = static_cast<uint32_t>(dq.dimvec_len[j]);
    hp.dim[t].factor = q->factor[j];
  }
  hp.m1 = dm1;
  hp.m2 = dm2;
  hp.row_begin = q->row_begin;
  hp.row_end = q->row_end;
  hp.vec_begin = vec_begin;
  hp.nvec = static_cast<uint32_t>(nvec);
  hp.n_groups = q->group_nums;
  hp.out = reinterpret_cast<unsigned long long*>(dsum);
  hp.totals = reinterpret_cast<unsigned long long*>(dtot);
  hp.range_err = &ctx->counters->range_errors;
  hp.sectors = &ctx->counters->host_sectors;
  hp.n_aggs = q->n_aggs;
  hp.agg0 = q->agg[0];
  hp.agg1 = q->n_aggs > 1 ? q->agg[1] : 0;

  const int64_t acc_budget =
      std::min<int64_t>(tune_or(ctx, TUNE_SMEM_ACC_BYTES, 64 * 1024), ctx->smem_optin - 4096);
  const bool sacc = nacc * 8 <= acc_budget;
  const HostScanKernel k = sacc ? pick_hostscan<true>(nd) : pick_hostscan<false>(nd);
  const size_t smem = sacc ? static_cast<size_t>(nacc) * 8 : 0;
  OLAP_CUDA_TRY(ctx, cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)));
  int per_sm = 0;
  OLAP_CUDA_TRY(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kHostScanThreads, smem));
  const int grid = ctx->sm_count * std::max(1, per_sm);
  k<<<grid, kHostScanThreads, smem, ctx->stream>>>(hp);
  OLAP_CUDA_TRY(ctx, cudaGetLastError());

  if (group_sums)
    OLAP_CUDA_TRY(ctx, cudaMemcpyAsync(group_sums, dsum, sizeof(int64_t) * nacc, cudaMemcpyDeviceToHost,
                                       ctx->stream));
  int64_t htot[2] = {0, 0};
  OLAP_CUDA_TRY(ctx, cudaMemcpyAsync(htot, dtot, sizeof(htot), cudaMemcpyDeviceToHost, ctx->stream));
  unsigned long long bad = 0;
  OLAP_CUDA_TRY(ctx, cudaMemcpyAsync(&bad, &ctx->counters->range_errors, sizeof(bad), cudaMemcpyDeviceToHost,
                                     ctx->stream));
  OLAP_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  if (totals)
    for (int a = 0; a < q->n_aggs; ++a) totals[a] = htot[a];
  if (bad) {
    OLAP_CUDA_TRY(ctx, cudaMemset(&ctx->counters->range_errors, 0, sizeof(bad)));
    return set_error(ctx, OLAP_ERR_RANGE, std::to_string(bad) + " rows dropped: fk or group id out of range");
  }
  return OLAP_OK;
}

}  // namespace olap
