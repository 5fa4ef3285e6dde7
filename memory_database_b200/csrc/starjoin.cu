// Fused star-join + multidimensional group-by SUM for sm_100a.
//
// Replaces the OLAP core of the reference (code/OLAPcore/
// test_multi_compute_operator.cpp): OLAPcore_rowwise (973-1037),
// OLAPcore_vwm_dv (1052-1126) and OLAPcore_vwm_sv (1258-1327), whose per-row
// contract is OLAPcore_vwm_sv_thread (509-568):
//
//   for each fact row r:  g = sum_j dimvec_j[fk_j[r]] * factor_j
//                         (row dropped when any probe returns DIM_NULL)
//                         group_vector[g] += M1[r] + M2[r]
//
// One pass over the fact table, HBM-bandwidth bound:
//  * every thread streams 4 consecutive rows of each needed column with one
//    128-bit load (ld.global.nc, no L1 allocation, L2 evict-first), two such
//    groups in flight per thread;
//  * dimension vectors are probed through L1/L2 with an evict-last policy, or
//    from shared memory when they are small enough to stage per block; probes
//    stop at the first DIM_NULL, so later dimensions are read only for the
//    rows that survive the earlier ones;
//  * group accumulators are int64: in shared memory when the group vector
//    fits (exact 64-bit sums built from 32-bit shared atomics), otherwise
//    L2-resident global atomics; totals are reduced in registers;
//  * the grid is persistent: SM count x resident blocks per SM.
#include <algorithm>
#include <cstring>
#include <thread>
#include <type_traits>
#include <vector>

#include "olap_internal.cuh"

namespace olap {

// One dimension in probe order.
struct Probe {
  const int8_t* vec;      // int8 group code or DIM_NULL
  const uint32_t* bits;   // pass bitmap (bit k: vec[k] != DIM_NULL) or null
  const int32_t* fk;      // foreign-key column
  uint32_t len;           // readable entries of vec
  int32_t factor;
  int32_t soff;           // byte offset of a staged int8 copy in shared memory, or -1
  int32_t boff;           // byte offset of a staged pass bitmap in shared memory, or -1
  int32_t code_flag;      // index into StarParams::code_nonzero (bitmap dims)
};

struct StarParams {
  Probe dim[OLAP_MAX_DIMS];
  const int32_t* m1;
  const int32_t* m2;
  int64_t row_begin, row_end;  // rows to process
  int64_t vec_begin, vec_end;  // sub-range read with 128-bit loads (VEC)
  int64_t n_groups;
  unsigned long long* out;     // [n_aggs][n_groups]
  unsigned long long* totals;  // [n_aggs] or null
  unsigned long long* range_err;
  const int32_t* code_nonzero; // per bitmap dim: 1 when some live code != 0
  int32_t n_aggs, agg0, agg1;
  int32_t smem_dim_bytes;      // staged dimension bytes and bitmaps (multiple of 16)
  int32_t need_m1, need_m2;
};

enum { ACC_NONE = 0, ACC_SMEM = 1, ACC_GLOBAL = 2 };
// Streaming modes of the 128-bit path: plain (64 registers, 2 x 512-thread
// blocks per SM), or software-pipelined (the next 4-row group's loads are in
// flight while the current group is probed) with 512 or 256-thread blocks.
enum { MODE_PLAIN = 0, MODE_PIPE_512 = 1, MODE_PIPE_256 = 2, MODE_SCALAR = 3 };

__device__ __forceinline__ int64_t agg_value(int a, int32_t x, int32_t y) {
  switch (a) {
    case OLAP_AGG_M1_PLUS_M2: return static_cast<int64_t>(x) + y;
    case OLAP_AGG_M1: return x;
    case OLAP_AGG_M2: return y;
    case OLAP_AGG_M1_TIMES_M2: return static_cast<int64_t>(x) * y;
    default: return 1;
  }
}

// Pass bitmap of one dimension vector: bit k of word k/32 is set when
// vec[k] != DIM_NULL; *nonzero becomes 1 when a live code is not 0 (then the
// code must be fetched for surviving rows).  One warp ballot per word.
__global__ void build_pass_bits(const int8_t* __restrict__ vec, uint32_t len,
                                uint32_t* __restrict__ bits, int32_t* __restrict__ nonzero) {
  const uint64_t nwords = (static_cast<uint64_t>(len) + 31) >> 5;
  const uint64_t total = nwords << 5;
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  bool any = false;
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < total; i += stride) {
    const int32_t c = i < len ? static_cast<int32_t>(vec[i]) : OLAP_DIM_NULL;
    const bool live = c != OLAP_DIM_NULL;
    any |= live && c != 0;
    const uint32_t w = __ballot_sync(0xffffffffu, live);
    if ((threadIdx.x & 31) == 0) bits[i >> 5] = w;
  }
  if (__any_sync(0xffffffffu, any) && (threadIdx.x & 31) == 0) atomicOr(nonzero, 1);
}

template <int ND>
struct Group4 {
  int4 f[ND > 0 ? ND : 1];
  int4 a, b;
};

template <int ND, int ACC, bool VEC, int MODE>
__global__ void __launch_bounds__(MODE == MODE_PIPE_256 ? 256 : MODE == MODE_PIPE_512 ? 512 : 1024,
                                  MODE == MODE_PIPE_256 ? 3 : 1)
starjoin_kernel(const StarParams p) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ long long red[32][2];
  __shared__ unsigned int red_bad;
  __shared__ int32_t s_code_nz[OLAP_MAX_DIMS];
  unsigned char* sdim = smem;
  unsigned long long* sacc = reinterpret_cast<unsigned long long*>(smem + p.smem_dim_bytes);
  const int tid = threadIdx.x;
  const int64_t nacc = p.n_groups * p.n_aggs;

  if (tid == 0) red_bad = 0;
  if (tid < OLAP_MAX_DIMS)
    s_code_nz[tid] = (tid < ND && p.dim[tid].code_flag >= 0) ? p.code_nonzero[p.dim[tid].code_flag] : 0;
  // Stage small dimension vectors into shared memory.
#pragma unroll
  for (int j = 0; j < ND; ++j) {
    if (p.dim[j].soff >= 0) {
      const int8_t* src = p.dim[j].vec;
      unsigned char* dst = sdim + p.dim[j].soff;
      const uint32_t n = p.dim[j].len;
      if ((reinterpret_cast<uintptr_t>(src) & 15) == 0) {
        const uint32_t n16 = n >> 4;
        for (uint32_t i = tid; i < n16; i += blockDim.x)
          reinterpret_cast<int4*>(dst)[i] = __ldg(reinterpret_cast<const int4*>(src) + i);
        for (uint32_t i = (n16 << 4) + tid; i < n; i += blockDim.x) dst[i] = src[i];
      } else {
        for (uint32_t i = tid; i < n; i += blockDim.x) dst[i] = src[i];
      }
    }
    if (p.dim[j].boff >= 0) {
      // Pass bitmap (built on the same stream before this kernel; the arena
      // allocation is 256-byte aligned, so 16-byte copies are safe).
      const uint32_t nw = (p.dim[j].len + 31) >> 5;
      const uint32_t n4 = nw >> 2;
      const int4* src = reinterpret_cast<const int4*>(p.dim[j].bits);
      int4* dst = reinterpret_cast<int4*>(sdim + p.dim[j].boff);
      for (uint32_t i = tid; i < n4; i += blockDim.x) dst[i] = __ldg(src + i);
      uint32_t* dw = reinterpret_cast<uint32_t*>(sdim + p.dim[j].boff);
      for (uint32_t i = (n4 << 2) + tid; i < nw; i += blockDim.x) dw[i] = __ldg(p.dim[j].bits + i);
    }
  }
  if (ACC == ACC_SMEM)
    for (int64_t i = tid; i < nacc; i += blockDim.x) sacc[i] = 0ull;
  __syncthreads();
  bool need_code[OLAP_MAX_DIMS];
#pragma unroll
  for (int j = 0; j < OLAP_MAX_DIMS; ++j) need_code[j] = s_code_nz[j] != 0;

  const uint64_t pol_stream = policy_evict_first();
  const uint64_t pol_keep = policy_evict_last();
  const int n_aggs = p.n_aggs;
  const int agg0 = p.agg0, agg1 = p.agg1;
  int64_t tot0 = 0, tot1 = 0;
  unsigned int bad = 0;

  // Accumulate one surviving row.
  auto emit = [&](int64_t g, int32_t x, int32_t y) {
    if (static_cast<uint64_t>(g) >= static_cast<uint64_t>(p.n_groups)) {
      ++bad;
      return;
    }
    const int64_t v0 = agg_value(agg0, x, y);
    tot0 += v0;
    if (ACC == ACC_SMEM) smem_add_u64(&sacc[g], static_cast<uint64_t>(v0));
    if (ACC == ACC_GLOBAL) atomicAdd(&p.out[g], static_cast<unsigned long long>(v0));
    if (n_aggs > 1) {
      const int64_t v1 = agg_value(agg1, x, y);
      tot1 += v1;
      if (ACC == ACC_SMEM) smem_add_u64(&sacc[p.n_groups + g], static_cast<uint64_t>(v1));
      if (ACC == ACC_GLOBAL)
        atomicAdd(&p.out[p.n_groups + g], static_cast<unsigned long long>(v1));
    }
  };

  // Probe R rows breadth-first: for each dimension, the R independent probes
  // are issued together before any of them is consumed.  Every key is
  // range-checked first (registers only), so the range-error count does not
  // depend on the probe order.
  auto probe_rows = [&](auto& key, const int32_t* x, const int32_t* y, auto rows_tag) {
    constexpr int R = decltype(rows_tag)::value;
    unsigned alive = (1u << R) - 1u;
#pragma unroll
    for (int r = 0; r < R; ++r) {
      bool inb = true;
#pragma unroll
      for (int j = 0; j < ND; ++j) inb &= static_cast<uint32_t>(key[r][j]) < p.dim[j].len;
      if (!inb) {
        alive &= ~(1u << r);
        ++bad;
      }
    }
    int64_t g[R];
#pragma unroll
    for (int r = 0; r < R; ++r) g[r] = 0;
#pragma unroll
    for (int j = 0; j < ND; ++j) {
      if (alive == 0) break;
      const Probe& d = p.dim[j];
      if (d.soff >= 0) {
#pragma unroll
        for (int r = 0; r < R; ++r) {
          if (alive & (1u << r)) {
            const int32_t c = static_cast<int8_t>(sdim[d.soff + static_cast<uint32_t>(key[r][j])]);
            if (c == OLAP_DIM_NULL) alive &= ~(1u << r);
            else g[r] += static_cast<int64_t>(c) * d.factor;
          }
        }
      } else if (d.boff >= 0) {
        const uint32_t* sw = reinterpret_cast<const uint32_t*>(sdim + d.boff);
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const uint32_t k = static_cast<uint32_t>(key[r][j]);
          if ((alive & (1u << r)) && !((sw[k >> 5] >> (k & 31)) & 1u)) alive &= ~(1u << r);
        }
      } else if (d.bits) {
        uint32_t w[R];
#pragma unroll
        for (int r = 0; r < R; ++r)
          w[r] = (alive & (1u << r)) ? __ldg(d.bits + (static_cast<uint32_t>(key[r][j]) >> 5)) : 0u;
#pragma unroll
        for (int r = 0; r < R; ++r)
          if (!((w[r] >> (static_cast<uint32_t>(key[r][j]) & 31)) & 1u)) alive &= ~(1u << r);
      } else {
        int32_t c[R];
#pragma unroll
        for (int r = 0; r < R; ++r)
          c[r] = (alive & (1u << r)) ? ld_probe_s8(d.vec + static_cast<uint32_t>(key[r][j]), pol_keep)
                                     : OLAP_DIM_NULL;
#pragma unroll
        for (int r = 0; r < R; ++r) {
          if (c[r] == OLAP_DIM_NULL) alive &= ~(1u << r);
          else g[r] += static_cast<int64_t>(c[r]) * d.factor;
        }
      }
    }
    if (alive == 0) return;
    // Group codes of bitmap-filtered dimensions, for surviving rows only.
#pragma unroll
    for (int j = 0; j < ND; ++j) {
      const Probe& d = p.dim[j];
      if (d.soff < 0 && d.bits && need_code[j]) {
        int32_t c[R];
#pragma unroll
        for (int r = 0; r < R; ++r)
          c[r] = (alive & (1u << r)) ? ld_probe_s8(d.vec + static_cast<uint32_t>(key[r][j]), pol_keep) : 0;
#pragma unroll
        for (int r = 0; r < R; ++r) g[r] += static_cast<int64_t>(c[r]) * d.factor;
      }
    }
#pragma unroll
    for (int r = 0; r < R; ++r)
      if (alive & (1u << r)) emit(g[r], x[r], y[r]);
  };

  auto scalar_rows = [&](int64_t b, int64_t e, int64_t first, int64_t step) {
    for (int64_t r = b + first; r < e; r += step) {
      int32_t key[1][ND > 0 ? ND : 1];
#pragma unroll
      for (int j = 0; j < ND; ++j) key[0][j] = ld_stream_s32(p.dim[j].fk + r, pol_stream);
      const int32_t x = p.need_m1 ? ld_stream_s32(p.m1 + r, pol_stream) : 0;
      const int32_t y = p.need_m2 ? ld_stream_s32(p.m2 + r, pol_stream) : 0;
      probe_rows(key, &x, &y, std::integral_constant<int, 1>{});
    }
  };

  auto load4 = [&](Group4<ND>& G, int64_t r) {
#pragma unroll
    for (int j = 0; j < ND; ++j) G.f[j] = ld_stream_v4(p.dim[j].fk + r, pol_stream);
    G.a = p.need_m1 ? ld_stream_v4(p.m1 + r, pol_stream) : make_int4(0, 0, 0, 0);
    G.b = p.need_m2 ? ld_stream_v4(p.m2 + r, pol_stream) : make_int4(0, 0, 0, 0);
  };
  auto process4 = [&](const Group4<ND>& G) {
    int32_t key[4][ND > 0 ? ND : 1];
#pragma unroll
    for (int j = 0; j < ND; ++j) {
      key[0][j] = G.f[j].x;
      key[1][j] = G.f[j].y;
      key[2][j] = G.f[j].z;
      key[3][j] = G.f[j].w;
    }
    const int32_t x[4] = {G.a.x, G.a.y, G.a.z, G.a.w};
    const int32_t y[4] = {G.b.x, G.b.y, G.b.z, G.b.w};
    probe_rows(key, x, y, std::integral_constant<int, 4>{});
  };

  const int64_t gtid = static_cast<int64_t>(blockIdx.x) * blockDim.x + tid;
  const int64_t gstride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  if (VEC) {
    // Head and tail rows outside the 16-byte aligned range.
    if (blockIdx.x == 0) {
      scalar_rows(p.row_begin, p.vec_begin, tid, blockDim.x);
      scalar_rows(p.vec_end, p.row_end, tid, blockDim.x);
    }
    const int64_t nvec = (p.vec_end - p.vec_begin) >> 2;
    const int64_t base = p.vec_begin;
    int64_t i = gtid;
    if (MODE == MODE_PIPE_512 || MODE == MODE_PIPE_256) {
      Group4<ND> cur;
      if (i < nvec) load4(cur, base + 4 * i);
      for (; i < nvec; i += gstride) {
        Group4<ND> nxt;
        const int64_t in = i + gstride;
        if (in < nvec) load4(nxt, base + 4 * in);
        process4(cur);
        cur = nxt;
      }
    } else {
      for (; i < nvec; i += gstride) {
        Group4<ND> cur;
        load4(cur, base + 4 * i);
        process4(cur);
      }
    }
  } else {
    scalar_rows(p.row_begin, p.row_end, gtid, gstride);
  }

  // Block reduction of totals and of the range-error count.
  const int lane = tid & 31, warp = tid >> 5;
  tot0 = warp_sum_i64(tot0);
  tot1 = warp_sum_i64(tot1);
  unsigned int wbad = __reduce_add_sync(0xffffffffu, bad);
  if (lane == 0) {
    red[warp][0] = tot0;
    red[warp][1] = tot1;
    if (wbad) atomicAdd(&red_bad, wbad);
  }
  __syncthreads();
  if (warp == 0) {
    const int nw = blockDim.x >> 5;
    long long s0 = lane < nw ? red[lane][0] : 0;
    long long s1 = lane < nw ? red[lane][1] : 0;
    s0 = warp_sum_i64(s0);
    s1 = warp_sum_i64(s1);
    if (lane == 0) {
      if (p.totals) {
        if (s0) atomicAdd(&p.totals[0], static_cast<unsigned long long>(s0));
        if (n_aggs > 1 && s1) atomicAdd(&p.totals[1], static_cast<unsigned long long>(s1));
      }
      if (red_bad) atomicAdd(p.range_err, static_cast<unsigned long long>(red_bad));
    }
  }
  if (ACC == ACC_SMEM) {
    for (int64_t i = tid; i < nacc; i += blockDim.x) {
      const unsigned long long v = sacc[i];
      if (v) atomicAdd(&p.out[i], v);
    }
  }
}

using StarKernel = void (*)(const StarParams);

template <int ND, int ACC>
static StarKernel pick_mode(bool vec, int mode) {
  if (!vec) return starjoin_kernel<ND, ACC, false, MODE_SCALAR>;
  switch (mode) {
    case MODE_PIPE_512: return starjoin_kernel<ND, ACC, true, MODE_PIPE_512>;
    case MODE_PIPE_256: return starjoin_kernel<ND, ACC, true, MODE_PIPE_256>;
    default: return starjoin_kernel<ND, ACC, true, MODE_PLAIN>;
  }
}

template <int ND>
static StarKernel pick_kernel(int acc, bool vec, int mode) {
  switch (acc) {
    case ACC_NONE: return pick_mode<ND, ACC_NONE>(vec, mode);
    case ACC_SMEM: return pick_mode<ND, ACC_SMEM>(vec, mode);
    default: return pick_mode<ND, ACC_GLOBAL>(vec, mode);
  }
}

static StarKernel select_kernel(int nd, int acc, bool vec, int mode) {
  switch (nd) {
    case 0: return pick_kernel<0>(acc, vec, mode);
    case 1: return pick_kernel<1>(acc, vec, mode);
    case 2: return pick_kernel<2>(acc, vec, mode);
    case 3: return pick_kernel<3>(acc, vec, mode);
    default: return pick_kernel<4>(acc, vec, mode);
  }
}

static bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

// A planned launch: parameters, kernel choice and the bitmap builds it needs.
struct StarPlan {
  StarParams sp;
  int nd = 0;
  int acc = ACC_NONE;
  bool vec = false;
  int mode = MODE_PLAIN;
  int block = 512;
  size_t smem = 0;
  int nbits = 0;                       // dims whose pass bitmap must be built
  int bits_dim[OLAP_MAX_DIMS] = {};    // probe index of each
  uint32_t* bits_buf[OLAP_MAX_DIMS] = {};
  int32_t* code_nz = nullptr;          // [OLAP_MAX_DIMS] in the arena
};

static bool agg_needs(int ag, bool* m1, bool* m2) {
  if (ag < OLAP_AGG_M1_PLUS_M2 || ag > OLAP_AGG_COUNT) return false;
  *m1 |= (ag == OLAP_AGG_M1_PLUS_M2 || ag == OLAP_AGG_M1 || ag == OLAP_AGG_M1_TIMES_M2);
  *m2 |= (ag == OLAP_AGG_M1_PLUS_M2 || ag == OLAP_AGG_M2 || ag == OLAP_AGG_M1_TIMES_M2);
  return true;
}

// Validates a query and plans its launch.  Scratch (bitmaps, flags) comes
// from `ar`, which the caller keeps alive until the launch has completed.
int plan_starjoin(olap_ctx* ctx, const olap_starjoin_query* q, int64_t* group_sums,
                  int64_t* totals, Arena& ar, StarPlan* pl) {
  OLAP_REQUIRE(ctx, q != nullptr, "null query");
  OLAP_REQUIRE(ctx, q->dimvec_nums >= 0 && q->dimvec_nums <= OLAP_MAX_DIMS,
               "dimvec_nums must be in [0, 4]");
  OLAP_REQUIRE(ctx, q->n_aggs >= 1 && q->n_aggs <= 2, "n_aggs must be 1 or 2");
  OLAP_REQUIRE(ctx, q->group_nums >= 1 && q->group_nums <= INT32_MAX,
               "group_nums must be in [1, 2^31)");
  OLAP_REQUIRE(ctx, q->row_begin >= 0 && q->row_end >= q->row_begin, "bad fact row range");
  bool need_m1 = false, need_m2 = false;
  for (int a = 0; a < q->n_aggs; ++a)
    OLAP_REQUIRE(ctx, agg_needs(q->agg[a], &need_m1, &need_m2), "unknown aggregate");
  const bool empty = q->row_end == q->row_begin;
  OLAP_REQUIRE(ctx, empty || !need_m1 || q->m1, "M1 column required by the aggregate");
  OLAP_REQUIRE(ctx, empty || !need_m2 || q->m2, "M2 column required by the aggregate");

  StarParams* sp = &pl->sp;
  std::memset(sp, 0, sizeof(*sp));
  const int nd = q->dimvec_nums;
  pl->nd = nd;
  const int64_t smem_cap = ctx->smem_optin - 2048;
  // Staging policy (all knobs from the context; the autotuner sets them):
  //  * int8 vectors up to TUNE_SMEM_DIM_BYTES in total are copied to shared
  //    memory whole (filter and group code in one shared-memory probe);
  //  * pass bitmaps of the next dimensions, in the caller's order, are staged
  //    up to TUNE_SMEM_BITS_BYTES (filter in shared memory, group code read
  //    from L2 for surviving rows only);
  //  * remaining dimensions use a global pass bitmap through L1
  //    (TUNE_PROBE_BITS = 1) or direct int8 probes.
  const int64_t smem_dim_budget =
      std::min<int64_t>(tune_or(ctx, TUNE_SMEM_DIM_BYTES, 48 * 1024), smem_cap);
  const int64_t smem_bits_budget = tune_or(ctx, TUNE_SMEM_BITS_BYTES, 0);
  const int64_t bits_knob = tune_or(ctx, TUNE_PROBE_BITS, 2);
  int idx[OLAP_MAX_DIMS];
  for (int j = 0; j < nd; ++j) idx[j] = j;
  std::stable_sort(idx, idx + nd, [&](int a, int b) { return q->dimvec_len[a] < q->dimvec_len[b]; });
  int kind[OLAP_MAX_DIMS] = {0, 0, 0, 0};  // 1 int8 staged, 2 bitmap staged, 3 global bitmap
  int64_t used = 0;
  for (int t = 0; t < nd; ++t) {
    const int j = idx[t];
    const int64_t bytes = (q->dimvec_len[j] + 15) & ~int64_t(15);
    if (used + bytes <= smem_dim_budget) {
      kind[j] = 1;
      used += bytes;
    }
  }
  int64_t bits_used = 0;
  for (int j = 0; j < nd; ++j) {
    if (kind[j] || empty) continue;
    const int64_t bbytes = ((q->dimvec_len[j] + 31) / 32 * 4 + 15) & ~int64_t(15);
    if (bits_used + bbytes <= smem_bits_budget && used + bits_used + bbytes <= smem_cap) {
      kind[j] = 2;
      bits_used += bbytes;
    } else if (bits_knob == 1) {
      kind[j] = 3;
    }
  }
  pl->nbits = 0;
  pl->code_nz = nullptr;
  int out = 0;
  int64_t soff = 0;
  // Probe order: shared-memory int8, then shared-memory bitmaps, then the rest.
  for (int pass = 1; pass <= 3; ++pass) {
    for (int j = 0; j < nd; ++j) {
      const int kj = kind[j] == 3 ? 0 : kind[j];
      if (pass == 3 ? kj != 0 : kj != pass) continue;
      OLAP_REQUIRE(ctx, q->dimvec[j] && (empty || q->fk[j]), "null dimension vector or fk column");
      OLAP_REQUIRE(ctx, q->dimvec_len[j] >= 1 && q->dimvec_len[j] <= INT32_MAX,
                   "dimvec_len must be in [1, 2^31)");
      const int k = out++;
      Probe& pr = sp->dim[k];
      pr.vec = q->dimvec[j];
      pr.fk = q->fk[j];
      pr.len = static_cast<uint32_t>(q->dimvec_len[j]);
      pr.factor = q->factor[j];
      pr.soff = -1;
      pr.boff = -1;
      pr.bits = nullptr;
      pr.code_flag = -1;
      if (kind[j] == 1) {
        pr.soff = static_cast<int32_t>(soff);
        soff += (q->dimvec_len[j] + 15) & ~int64_t(15);
      }
      if (kind[j] == 2 || kind[j] == 3) {
        if (!pl->code_nz) {
          pl->code_nz = ar.take<int32_t>(OLAP_MAX_DIMS);
          if (!pl->code_nz) return set_error(ctx, OLAP_ERR_CAPACITY, "scratch arena exhausted");
        }
        uint32_t* b = ar.take<uint32_t>((q->dimvec_len[j] + 31) / 32);
        if (!b) return set_error(ctx, OLAP_ERR_CAPACITY, "scratch arena too small for pass bitmaps");
        pr.bits = b;
        pr.code_flag = pl->nbits;
        pl->bits_dim[pl->nbits] = k;
        pl->bits_buf[pl->nbits] = b;
        ++pl->nbits;
        if (kind[j] == 2) {
          pr.boff = static_cast<int32_t>(soff);
          soff += ((q->dimvec_len[j] + 31) / 32 * 4 + 15) & ~int64_t(15);
        }
      }
    }
  }
  sp->code_nonzero = pl->code_nz;
  sp->smem_dim_bytes = static_cast<int32_t>(soff);
  sp->m1 = q->m1;
  sp->m2 = q->m2;
  sp->need_m1 = need_m1;
  sp->need_m2 = need_m2;
  sp->row_begin = q->row_begin;
  sp->row_end = q->row_end;
  sp->n_groups = q->group_nums;
  sp->n_aggs = q->n_aggs;
  sp->agg0 = q->agg[0];
  sp->agg1 = q->n_aggs > 1 ? q->agg[1] : q->agg[0];
  sp->out = reinterpret_cast<unsigned long long*>(group_sums);
  sp->totals = reinterpret_cast<unsigned long long*>(totals);
  sp->range_err = &ctx->counters->range_errors;

  // 128-bit path when every streamed column is 16-byte aligned.
  bool vec = true;
  for (int j = 0; j < nd; ++j) vec &= aligned16(sp->dim[j].fk);
  if (need_m1) vec &= aligned16(q->m1);
  if (need_m2) vec &= aligned16(q->m2);
  pl->vec = vec;
  if (vec) {
    int64_t vb = (q->row_begin + 3) & ~int64_t(3);
    if (vb > q->row_end) vb = q->row_end;
    const int64_t ve = vb + ((q->row_end - vb) & ~int64_t(3));
    sp->vec_begin = vb;
    sp->vec_end = ve;
  }
  pl->mode = static_cast<int>(tune_or(ctx, TUNE_UNROLL, 1)) - 1;  // knob 1..3 -> mode 0..2
  if (pl->mode < MODE_PLAIN || pl->mode > MODE_PIPE_256) pl->mode = MODE_PLAIN;
  const int max_block = pl->mode == MODE_PIPE_256 ? 256 : pl->mode == MODE_PIPE_512 ? 512 : 1024;
  // One 1024-thread block per SM when large bitmaps are staged (the staging
  // copy is paid once per SM), else 512-thread blocks.
  const int dflt_block = std::min(max_block, bits_used > 64 * 1024 ? 1024 : 512);
  pl->block = static_cast<int>(std::min<int64_t>(tune_or(ctx, TUNE_BLOCK, dflt_block), max_block));
  OLAP_REQUIRE(ctx, pl->block >= 64 && pl->block % 32 == 0, "block size must be a multiple of 32, >= 64");

  const int64_t acc_bytes = q->group_nums * q->n_aggs * 8;
  const int64_t smem_acc_budget = tune_or(ctx, TUNE_SMEM_ACC_BYTES, 96 * 1024);
  int acc = ACC_GLOBAL;
  if (!group_sums) acc = ACC_NONE;
  else if (acc_bytes <= smem_acc_budget && soff + acc_bytes <= smem_cap) acc = ACC_SMEM;
  pl->acc = acc;
  pl->smem = static_cast<size_t>(soff + (acc == ACC_SMEM ? acc_bytes : 0));
  return OLAP_OK;
}

int launch_starjoin(olap_ctx* ctx, StarPlan& pl, cudaStream_t stream) {
  // Pass bitmaps (and their code flags) first, on the same stream.
  if (pl.nbits) {
    OLAP_CUDA_TRY(ctx, cudaMemsetAsync(pl.code_nz, 0, sizeof(int32_t) * OLAP_MAX_DIMS, stream));
    for (int b = 0; b < pl.nbits; ++b) {
      const Probe& d = pl.sp.dim[pl.bits_dim[b]];
      const uint64_t threads = ((static_cast<uint64_t>(d.len) + 31) / 32) * 32;
      const unsigned grid = static_cast<unsigned>(std::min<uint64_t>((threads + 255) / 256,
                                                                     static_cast<uint64_t>(ctx->sm_count) * 8));
      build_pass_bits<<<grid, 256, 0, stream>>>(d.vec, d.len, pl.bits_buf[b], pl.code_nz + b);
      OLAP_CUDA_TRY(ctx, cudaGetLastError());
    }
  }
  StarKernel k = select_kernel(pl.nd, pl.acc, pl.vec, pl.mode);
  if (pl.smem > 48 * 1024)
    OLAP_CUDA_TRY(ctx, cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            static_cast<int>(pl.smem)));
  int bps = static_cast<int>(tune_or(ctx, TUNE_BLOCKS_PER_SM, 0));
  if (bps == 0) {
    OLAP_CUDA_TRY(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k, pl.block, pl.smem));
    if (bps < 1) return set_error(ctx, OLAP_ERR_CAPACITY, "star-join kernel does not fit an SM");
  }
  const StarParams& sp = pl.sp;
  const int64_t rows = sp.row_end - sp.row_begin;
  const int64_t work_items = pl.vec ? std::max<int64_t>((rows + 3) / 4, 1) : std::max<int64_t>(rows, 1);
  int64_t grid = static_cast<int64_t>(ctx->sm_count) * bps;
  grid = std::min<int64_t>(grid, (work_items + pl.block - 1) / pl.block);
  grid = std::max<int64_t>(grid, 1);
  k<<<static_cast<unsigned>(grid), pl.block, pl.smem, stream>>>(sp);
  OLAP_CUDA_TRY(ctx, cudaGetLastError());
  return OLAP_OK;
}

int starjoin_device(olap_ctx* ctx, const olap_starjoin_query* q, int64_t* group_sums,
                    int64_t* totals, bool accumulate, cudaStream_t stream, Arena& ar) {
  StarPlan pl;
  int st = plan_starjoin(ctx, q, group_sums, totals, ar, &pl);
  if (st != OLAP_OK) return st;
  if (!accumulate) {
    if (group_sums)
      OLAP_CUDA_TRY(ctx, cudaMemsetAsync(group_sums, 0,
                                         sizeof(int64_t) * q->group_nums * q->n_aggs, stream));
    if (totals) OLAP_CUDA_TRY(ctx, cudaMemsetAsync(totals, 0, sizeof(int64_t) * q->n_aggs, stream));
  }
  if (q->row_end == q->row_begin) return OLAP_OK;
  return launch_starjoin(ctx, pl, stream);
}

// Multi-threaded host maximum of an int32 column (used to size a dimension
// vector whose length the caller did not give).
static int32_t host_max_i32(const int32_t* v, int64_t n) {
  const int nt = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  std::vector<int32_t> part(nt, INT32_MIN);
  std::vector<std::thread> th;
  for (int t = 0; t < nt; ++t)
    th.emplace_back([&, t] {
      const int64_t b = n * t / nt, e = n * (t + 1) / nt;
      int32_t m = INT32_MIN;
      for (int64_t i = b; i < e; ++i) m = v[i] > m ? v[i] : m;
      part[t] = m;
    });
  for (auto& x : th) x.join();
  int32_t m = INT32_MIN;
  for (int32_t x : part) m = x > m ? x : m;
  return m;
}

static bool is_pinned(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

// Host-memory star-join: dimension vectors are copied once; the fact columns
// stream through two device buffers in chunks, H2D copies of chunk c+1
// overlapping the scan of chunk c.
int starjoin_host(olap_ctx* ctx, const olap_starjoin_query* q, int64_t* group_sums,
                  int64_t* totals) {
  const int nd = q->dimvec_nums;
  OLAP_REQUIRE(ctx, nd >= 0 && nd <= OLAP_MAX_DIMS, "dimvec_nums must be in [0, 4]");
  OLAP_REQUIRE(ctx, q->row_begin >= 0 && q->row_end >= q->row_begin, "bad fact row range");
  OLAP_REQUIRE(ctx, q->n_aggs >= 1 && q->n_aggs <= 2, "n_aggs must be 1 or 2");
  OLAP_REQUIRE(ctx, q->group_nums >= 1 && q->group_nums <= INT32_MAX,
               "group_nums must be in [1, 2^31)");
  bool need_m1 = false, need_m2 = false;
  for (int a = 0; a < q->n_aggs; ++a) {
    const int ag = q->agg[a];
    need_m1 |= (ag == OLAP_AGG_M1_PLUS_M2 || ag == OLAP_AGG_M1 || ag == OLAP_AGG_M1_TIMES_M2);
    need_m2 |= (ag == OLAP_AGG_M1_PLUS_M2 || ag == OLAP_AGG_M2 || ag == OLAP_AGG_M1_TIMES_M2);
  }
  const int64_t rows = q->row_end - q->row_begin;
  OLAP_REQUIRE(ctx, rows == 0 || !need_m1 || q->m1, "M1 column required by the aggregate");
  OLAP_REQUIRE(ctx, rows == 0 || !need_m2 || q->m2, "M2 column required by the aggregate");

  Arena ar(ctx);
  olap_starjoin_query dq = *q;
  // Dimension vectors.
  for (int j = 0; j < nd; ++j) {
    OLAP_REQUIRE(ctx, q->dimvec[j] && (rows == 0 || q->fk[j]), "null dimension vector or fk column");
    int64_t len = q->dimvec_len[j];
    if (len <= 0) {
      const int32_t m = rows ? host_max_i32(q->fk[j] + q->row_begin, rows) : 0;
      len = static_cast<int64_t>(m < 0 ? 0 : m) + 1;
    }
    int8_t* d = ar.take<int8_t>(static_cast<size_t>(len));
    if (!d) return set_error(ctx, OLAP_ERR_CAPACITY, "scratch arena too small for dimension vectors");
    OLAP_CUDA_TRY(ctx, cudaMemcpyAsync(d, q->dimvec[j], static_cast<size_t>(len),
                                       cudaMemcpyHostToDevice, ctx->stream));
    dq.dimvec[j] = d;
    dq.dimvec_len[j] = len;
  }
  const int64_t nacc = q->group_nums * q->n_aggs;
  int64_t* dsum = group_sums ? ar.take<int64_t>(static_cast<size_t>(nacc)) : nullptr;
  int64_t* dtot = ar.take<int64_t>(2);
  if ((group_sums && !dsum) || !dtot)
    return set_error(ctx, OLAP_ERR_CAPACITY, "scratch arena too small for group sums");
  if (dsum) OLAP_CUDA_TRY(ctx, cudaMemsetAsync(dsum, 0, sizeof(int64_t) * nacc, ctx->stream));
  OLAP_CUDA_TRY(ctx, cudaMemsetAsync(dtot, 0, sizeof(int64_t) * 2, ctx->stream));

  // Column list streamed per chunk.
  std::vector<const int32_t*> cols;
  for (int j = 0; j < nd; ++j) cols.push_back(q->fk[j]);
  const int i_m1 = need_m1 ? static_cast<int>(cols.size()) : -1;
  if (need_m1) cols.push_back(q->m1);
  const int i_m2 = need_m2 ? static_cast<int>(cols.size()) : -1;
  if (need_m2) cols.push_back(q->m2);
  const int ncol = static_cast<int>(cols.size());

  int64_t chunk = tune_or(ctx, TUNE_CHUNK_ROWS, int64_t(1) << 22);
  chunk = (chunk + 3) & ~int64_t(3);
  // Fit two chunk buffers into the remaining arena.
  const size_t left = ar.cap > ar.off ? ar.cap - ar.off : 0;
  while (chunk > 1024 && static_cast<size_t>(2 * ncol * chunk * 4 + 4096 * ncol) > left) chunk /= 2;
  int32_t* dbuf[2][6] = {};
  for (int b = 0; b < 2; ++b)
    for (int c = 0; c < ncol; ++c) {
      dbuf[b][c] = ar.take<int32_t>(static_cast<size_t>(chunk));
      if (!dbuf[b][c]) return set_error(ctx, OLAP_ERR_CAPACITY, "scratch arena too small for chunks");
    }
  bool pinned = true;
  for (auto* c : cols) pinned &= is_pinned(c);
  // Pageable input: bounce through the context's pinned staging buffer.
  const size_t stage_bytes = static_cast<size_t>(2 * ncol * chunk * 4);
  if (!pinned && ctx->pinned_bytes < stage_bytes) {
    if (ctx->pinned) cudaFreeHost(ctx->pinned);
    ctx->pinned = nullptr;
    ctx->pinned_bytes = 0;
    OLAP_CUDA_TRY(ctx, cudaMallocHost(&ctx->pinned, stage_bytes));
    ctx->pinned_bytes = stage_bytes;
  }
  cudaStream_t cs;
  OLAP_CUDA_TRY(ctx, cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
  cudaEvent_t copied[2], scanned[2];
  for (int b = 0; b < 2; ++b) {
    cudaEventCreateWithFlags(&copied[b], cudaEventDisableTiming);
    cudaEventCreateWithFlags(&scanned[b], cudaEventDisableTiming);
  }
  int st = OLAP_OK;
  // The dimension copies and memsets above are ordered on ctx->stream; the
  // copy stream starts after them.
  cudaEvent_t ready;
  cudaEventCreateWithFlags(&ready, cudaEventDisableTiming);
  cudaEventRecord(ready, ctx->stream);
  cudaStreamWaitEvent(cs, ready, 0);
  int64_t nchunks = (rows + chunk - 1) / chunk;
  for (int64_t c = 0; c < nchunks && st == OLAP_OK; ++c) {
    const int b = static_cast<int>(c & 1);
    const int64_t r0 = q->row_begin + c * chunk;
    const int64_t n = std::min(chunk, q->row_end - r0);
    cudaStreamWaitEvent(cs, scanned[b], 0);
    for (int k = 0; k < ncol; ++k) {
      const int32_t* src = cols[k] + r0;
      if (!pinned) {
        // The staging half b is free once its previous copy has completed.
        if (c >= 2) cudaEventSynchronize(copied[b]);
        int32_t* stg = static_cast<int32_t*>(ctx->pinned) + (static_cast<size_t>(b) * ncol + k) * chunk;
        std::memcpy(stg, src, static_cast<size_t>(n) * 4);
        src = stg;
      }
      cudaError_t e = cudaMemcpyAsync(dbuf[b][k], src, static_cast<size_t>(n) * 4,
                                      cudaMemcpyHostToDevice, cs);
      if (e != cudaSuccess) { st = check_cuda(ctx, e, "cudaMemcpyAsync(H2D chunk)"); break; }
    }
    cudaEventRecord(copied[b], cs);
    cudaStreamWaitEvent(ctx->stream, copied[b], 0);
    olap_starjoin_query cq = dq;
    for (int j = 0; j < nd; ++j) cq.fk[j] = dbuf[b][j];
    cq.m1 = i_m1 >= 0 ? dbuf[b][i_m1] : nullptr;
    cq.m2 = i_m2 >= 0 ? dbuf[b][i_m2] : nullptr;
    cq.row_begin = 0;
    cq.row_end = n;
    if (st == OLAP_OK) {
      // Per-chunk scratch (bitmaps) after the pipeline's buffers; chunks on
      // one stream reuse it in order.
      Arena car = ar;
      st = starjoin_device(ctx, &cq, dsum, dtot, true, ctx->stream, car);
    }
    cudaEventRecord(scanned[b], ctx->stream);
  }
  if (st == OLAP_OK && group_sums)
    st = cudaMemcpyAsync(group_sums, dsum, sizeof(int64_t) * nacc, cudaMemcpyDeviceToHost,
                         ctx->stream) == cudaSuccess ? OLAP_OK : set_error(ctx, OLAP_ERR_CUDA, "D2H group sums");
  int64_t htot[2] = {0, 0};
  if (st == OLAP_OK)
    st = cudaMemcpyAsync(htot, dtot, sizeof(htot), cudaMemcpyDeviceToHost, ctx->stream) == cudaSuccess
             ? OLAP_OK : set_error(ctx, OLAP_ERR_CUDA, "D2H totals");
  cudaError_t se = cudaStreamSynchronize(ctx->stream);
  cudaStreamSynchronize(cs);
  for (int b = 0; b < 2; ++b) {
    cudaEventDestroy(copied[b]);
    cudaEventDestroy(scanned[b]);
  }
  cudaEventDestroy(ready);
  cudaStreamDestroy(cs);
  if (st != OLAP_OK) return st;
  if (se != cudaSuccess) return check_cuda(ctx, se, "cudaStreamSynchronize");
  if (totals)
    for (int a = 0; a < q->n_aggs; ++a) totals[a] = htot[a];
  unsigned long long bad = 0;
  OLAP_CUDA_TRY(ctx, cudaMemcpy(&bad, &ctx->counters->range_errors, sizeof(bad), cudaMemcpyDeviceToHost));
  if (bad) {
    OLAP_CUDA_TRY(ctx, cudaMemset(&ctx->counters->range_errors, 0, sizeof(bad)));
    return set_error(ctx, OLAP_ERR_RANGE, std::to_string(bad) + " rows dropped: fk or group id out of range");
  }
  return OLAP_OK;
}

}  // namespace olap

extern "C" {

int olap_starjoin_groupsum(olap_ctx* ctx, const olap_starjoin_query* q, int64_t* group_sums,
                           int64_t* totals) {
  if (!ctx) return OLAP_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  OLAP_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  olap::Arena ar(ctx);
  return olap::starjoin_device(ctx, q, group_sums, totals, false, ctx->stream, ar);
}

int olap_starjoin_groupsum_host(olap_ctx* ctx, const olap_starjoin_query* q, int64_t* group_sums,
                                int64_t* totals) {
  if (!ctx || !q) return OLAP_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  OLAP_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  return olap::starjoin_host(ctx, q, group_sums, totals);
}

int olap_OLAPcore(olap_ctx* ctx, int8_t* const* dimvec_array, const int64_t* dimvec_len,
                  int32_t* const* fk_array, const int* orders, int dimvec_nums,
                  const int* factor, int64_t size_lineorder, int64_t group_nums,
                  const int32_t* M1, const int32_t* M2, int64_t* group_vector, int64_t* count) {
  if (!ctx) return OLAP_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  OLAP_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  OLAP_REQUIRE(ctx, dimvec_nums >= 0 && dimvec_nums <= OLAP_MAX_DIMS, "dimvec_nums must be in [0, 4]");
  OLAP_REQUIRE(ctx, count != nullptr, "count must not be null");
  OLAP_REQUIRE(ctx, dimvec_nums == 0 || (dimvec_array && fk_array && orders && factor),
               "null plan arrays");
  olap_starjoin_query q;
  std::memset(&q, 0, sizeof(q));
  q.dimvec_nums = dimvec_nums;
  q.n_aggs = 1;
  q.agg[0] = OLAP_AGG_M1_PLUS_M2;
  for (int j = 0; j < dimvec_nums; ++j) {
    const int t = orders[j];
    OLAP_REQUIRE(ctx, t >= 0 && t < OLAP_MAX_DIMS, "orders[] entry must name table 0..3");
    q.dimvec[j] = dimvec_array[t];
    q.fk[j] = fk_array[t];
    q.dimvec_len[j] = dimvec_len ? dimvec_len[t] : INT32_MAX;
    q.factor[j] = factor[j];
  }
  q.m1 = M1;
  q.m2 = M2;
  q.row_begin = 0;
  q.row_end = size_lineorder;
  q.group_nums = group_nums;
  olap::Arena ar(ctx);
  int64_t* dtot = ar.take<int64_t>(1);
  if (!dtot) return olap::set_error(ctx, OLAP_ERR_CAPACITY, "scratch arena exhausted");
  int st = olap::starjoin_device(ctx, &q, group_vector, dtot, false, ctx->stream, ar);
  if (st != OLAP_OK) return st;
  OLAP_CUDA_TRY(ctx, cudaMemcpyAsync(count, dtot, sizeof(int64_t), cudaMemcpyDeviceToHost, ctx->stream));
  OLAP_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return OLAP_OK;
}

}  // extern "C"
