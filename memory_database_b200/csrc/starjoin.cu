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
#include <cstdlib>
#include <cstring>
#include <thread>
#include <type_traits>
#include <vector>

#include <cuda.h>

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
  const uint8_t* nib;     // 4-bit codes, two entries per byte (15 = DIM_NULL), or null
  int32_t noff;           // byte offset of the staged 4-bit codes in shared memory, or -1
  int32_t nib_flag;       // index into code_nonzero[OLAP_MAX_DIMS + ...]: 1 when a code needs > 4 bits
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
  const int32_t* code_nonzero; // [0, 4): per bitmap dim, 1 when some live code != 0;
                               // [4, 8): per 4-bit dim, 1 when some code is outside [0, 14]
  int32_t n_aggs, agg0, agg1;
  int32_t smem_dim_bytes;      // staged dimension bytes and bitmaps (multiple of 16)
  int32_t need_m1, need_m2;
  int32_t pf_off, bar_off;     // ASYNC: per-warp prefetch buffers and mbarriers (shared-memory offsets)
  int32_t cmp_off;             // CMP: per-warp survivor buffers (shared-memory offset)
  int32_t merge_global;        // probe consecutive global int8 dimensions together
  unsigned long long* wait_timeouts;
  unsigned long long* oob_seen;  // vec kernel: set when a key is out of range (the range pass counts them)
};

enum { ACC_NONE = 0, ACC_SMEM = 1, ACC_GLOBAL = 2 };

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

// 4-bit codes of one dimension vector, two entries per byte (low nibble
// first): DIM_NULL becomes 15, codes 0..14 stay; any other code sets *bad
// (the kernel then probes the int8 vector instead).
__global__ void build_nibbles(const int8_t* __restrict__ vec, uint32_t len, uint8_t* __restrict__ nib,
                              int32_t* __restrict__ bad) {
  const uint32_t nbytes = (len + 1) >> 1;
  const uint32_t stride = gridDim.x * blockDim.x;
  bool any = false;
  auto enc = [&](int32_t c) -> uint32_t {
    if (c == OLAP_DIM_NULL) return 15u;
    if (c < 0 || c > 14) {
      any = true;
      return 15u;
    }
    return static_cast<uint32_t>(c);
  };
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nbytes; i += stride) {
    const uint32_t k = 2 * i;
    const uint32_t lo = enc(vec[k]);
    const uint32_t hi = k + 1 < len ? enc(vec[k + 1]) : 15u;
    nib[i] = static_cast<uint8_t>(lo | (hi << 4));
  }
  if (any) atomicOr(bad, 1);
}

// Aggregate sets fixed at compile time for the 128-bit path.
enum {
  AGGK_GENERIC = 0,   // n_aggs / agg0 / agg1 read at run time
  AGGK_M1PM2 = 1,     // SUM(M1 + M2): the reference's aggregate
  AGGK_M1_M1M2 = 2,   // SUM(M1), SUM(M1 * M2)
};

// Block prologue shared by both kernels: stage int8 vectors and pass
// bitmaps into shared memory, zero the shared accumulators.
template <int ND, int ACC>
__device__ __forceinline__ void stage_block(const StarParams& p, unsigned char* sdim,
                                            unsigned long long* sacc, int64_t nacc) {
  const int tid = threadIdx.x;
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
    if (p.dim[j].noff >= 0) {
      // 4-bit codes (built on the same stream before this kernel; 256-byte
      // aligned arena buffer).
      const uint32_t nb = (p.dim[j].len + 1) >> 1;
      const uint32_t n16 = nb >> 4;
      const int4* src = reinterpret_cast<const int4*>(p.dim[j].nib);
      int4* dst = reinterpret_cast<int4*>(sdim + p.dim[j].noff);
      for (uint32_t i = tid; i < n16; i += blockDim.x) dst[i] = __ldg(src + i);
      for (uint32_t i = (n16 << 4) + tid; i < nb; i += blockDim.x) sdim[p.dim[j].noff + i] = p.dim[j].nib[i];
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
}

// Block epilogue shared by both kernels: reduce totals and the range-error
// count, flush shared accumulators to the global group vector.
template <int ACC>
__device__ __forceinline__ void finish_block(const StarParams& p, int64_t tot0, int64_t tot1,
                                             unsigned int bad, unsigned long long* sacc,
                                             int64_t nacc, long long (*red)[2],
                                             unsigned int* red_bad) {
  const int tid = threadIdx.x;
  const int lane = tid & 31, warp = tid >> 5;
  tot0 = warp_sum_i64(tot0);
  tot1 = warp_sum_i64(tot1);
  const unsigned int wbad = __reduce_add_sync(0xffffffffu, bad);
  if (lane == 0) {
    red[warp][0] = tot0;
    red[warp][1] = tot1;
    if (wbad) atomicAdd(red_bad, wbad);
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
        if (p.n_aggs > 1 && s1) atomicAdd(&p.totals[1], static_cast<unsigned long long>(s1));
      }
      if (*red_bad) atomicAdd(p.range_err, static_cast<unsigned long long>(*red_bad));
    }
  }
  if (ACC == ACC_SMEM) {
    const uint32_t* w = reinterpret_cast<const uint32_t*>(sacc);
    for (int64_t i = tid; i < nacc; i += blockDim.x) {
      const unsigned long long v = smem_split_get(w, nacc, i);
      if (v) atomicAdd(&p.out[i], v);
    }
  }
}

// 128-bit path.  Each thread takes V rows per iteration (V/4 int4 groups,
// grid-strided so that every load instruction is fully coalesced), checks all
// keys, probes the dimensions breadth-first across its V rows, fetches group
// codes of bitmap-filtered dimensions for survivors, and accumulates.  Group
// ids are int32: the host selects this kernel only when sum_j 128*|factor_j|
// fits in int32, so every intermediate is exact.
// ASYNC: each warp's next 32 x 16-byte vectors of every streamed column are
// brought into shared memory by bulk asynchronous copies (one lane issues
// them, an mbarrier counts the bytes) while the warp probes the current
// ones, so the DRAM latency overlaps the dependent dimension probes instead
// of adding to them; registers hold only the current vectors.
constexpr uint32_t kAsyncWaitLimit = 1u << 24;  // polls of a prefetch barrier before giving up

// CMP: after the shared-memory dimensions, each warp packs its surviving
// rows (keys, partial group id, measures) densely into a shared buffer and
// runs the global probes, group-code fetches and accumulation over them with
// every lane busy, instead of once per row slot with most lanes idle.
template <int ND, int ACC, int AGGK, int V, bool ASYNC, bool CMP>
__global__ void __launch_bounds__(V == 8 ? 512 : 1024, 1) starjoin_vec_kernel(const StarParams p) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ long long red[32][2];
  __shared__ unsigned int red_bad;
  __shared__ int32_t s_code_nz[OLAP_MAX_DIMS];
  __shared__ int32_t s_nib_ok[OLAP_MAX_DIMS];
  constexpr int NG = V / 4;
  unsigned char* sdim = smem;
  unsigned long long* sacc = reinterpret_cast<unsigned long long*>(smem + p.smem_dim_bytes);
  uint32_t* sw = reinterpret_cast<uint32_t*>(sacc);  // accumulator words: low words, then high words
  const int tid = threadIdx.x;
  const int64_t nacc = p.n_groups * p.n_aggs;
  if (tid == 0) red_bad = 0;
  if (tid < OLAP_MAX_DIMS)
    s_code_nz[tid] = (tid < ND && p.dim[tid].code_flag >= 0) ? p.code_nonzero[p.dim[tid].code_flag] : 0;
  if (tid < OLAP_MAX_DIMS)
    s_nib_ok[tid] = (tid < ND && p.dim[tid].noff >= 0)
                        ? (p.code_nonzero[OLAP_MAX_DIMS + p.dim[tid].nib_flag] == 0 ? 1 : 0)
                        : 0;
  stage_block<ND, ACC>(p, sdim, sacc, nacc);
  const int lane = tid & 31;
  constexpr int NCOL = (ND > 0 ? ND : 1) + 2;
  int4* pf = nullptr;
  unsigned long long* bar = nullptr;
  if (ASYNC) {
    pf = reinterpret_cast<int4*>(smem + p.pf_off) + (tid >> 5) * (NG * NCOL * 32);
    bar = reinterpret_cast<unsigned long long*>(smem + p.bar_off) + (tid >> 5);
    if (lane == 0) {
      mbar_init(bar, 1);
      fence_mbar_init();
    }
  }
  __syncthreads();
  bool need_code[OLAP_MAX_DIMS], nib_ok[OLAP_MAX_DIMS];
#pragma unroll
  for (int j = 0; j < OLAP_MAX_DIMS; ++j) {
    need_code[j] = s_code_nz[j] != 0;
    nib_ok[j] = s_nib_ok[j] != 0;
  }

  const uint64_t pol_stream = policy_evict_first();
  const uint64_t pol_keep = policy_evict_last();
  const uint32_t n_groups = static_cast<uint32_t>(p.n_groups);
  int64_t tot0 = 0, tot1 = 0;
  unsigned int bad = 0;

  const int32_t* fkb[ND > 0 ? ND : 1];
#pragma unroll
  for (int j = 0; j < ND; ++j) fkb[j] = p.dim[j].fk + p.vec_begin;
  const int32_t* m1b = p.m1 + p.vec_begin;
  const int32_t* m2b = p.m2 + p.vec_begin;
  const bool need_m1 = AGGK == AGGK_GENERIC ? p.need_m1 != 0 : true;
  const bool need_m2 = AGGK == AGGK_GENERIC ? p.need_m2 != 0 : true;

  const uint32_t nvec = static_cast<uint32_t>((p.vec_end - p.vec_begin) >> 2);
  const uint32_t gstride = gridDim.x * blockDim.x;
  const uint32_t wstride = NG * gstride;
  // ASYNC (lane 0): bulk copies of the warp's vectors w0 .. w0+31 (+ u*gstride)
  // of every streamed column into its prefetch buffer.
  auto issue = [&](uint32_t w0) {
    uint32_t cnt[NG];
    uint32_t bytes = 0;
    const uint32_t ncols = ND + (need_m1 ? 1 : 0) + (need_m2 ? 1 : 0);
#pragma unroll
    for (int u = 0; u < NG; ++u) {
      const uint32_t b = w0 + u * gstride;
      cnt[u] = b < nvec ? min(32u, nvec - b) : 0u;
      bytes += cnt[u] * 16u * ncols;
    }
    if (bytes == 0) return;
    mbar_arrive_expect_tx(bar, bytes);
#pragma unroll
    for (int u = 0; u < NG; ++u) {
      if (cnt[u] == 0) continue;
      const uint32_t b = w0 + u * gstride;
#pragma unroll
      for (int j = 0; j < ND; ++j) bulk_copy_g2s(pf + (u * NCOL + j) * 32, fkb[j] + 4ull * b, cnt[u] * 16u, bar, pol_stream);
      if (need_m1) bulk_copy_g2s(pf + (u * NCOL + ND) * 32, m1b + 4ull * b, cnt[u] * 16u, bar, pol_stream);
      if (need_m2) bulk_copy_g2s(pf + (u * NCOL + ND + 1) * 32, m2b + 4ull * b, cnt[u] * 16u, bar, pol_stream);
    }
  };
  uint32_t w0 = blockIdx.x * blockDim.x + (tid & ~31u);  // the warp's first vector of this step
  uint32_t phase = 0;
  if (ASYNC && lane == 0 && w0 < nvec) issue(w0);
  // ASYNC and CMP use warp-wide operations in the loop, so a warp runs its
  // steps together while any of its lanes has rows (w0 is warp-uniform).
  for (uint32_t i = blockIdx.x * blockDim.x + tid; (ASYNC || CMP) ? w0 < nvec : i < nvec;
       i += wstride, w0 += wstride) {
    int4 kf[NG][ND > 0 ? ND : 1];
    int4 ka[NG], kb[NG];
    uint32_t alive = 0;
    if (ASYNC) {
      // this step's vectors (issued one step earlier); bounded wait
      bool ok = false;
      for (uint32_t t = 0; t < kAsyncWaitLimit; ++t) {
        if (mbar_test(bar, phase)) {
          ok = true;
          break;
        }
        __nanosleep(32);
      }
      if (!__all_sync(0xffffffffu, ok)) {
        if (lane == 0) atomicAdd(p.wait_timeouts, 1ull);
        break;
      }
      phase ^= 1u;
#pragma unroll
      for (int u = 0; u < NG; ++u) {
        const uint32_t gi = i + u * gstride;
        if (gi < nvec) {
          alive |= 0xFu << (4 * u);
#pragma unroll
          for (int j = 0; j < ND; ++j) kf[u][j] = pf[(u * NCOL + j) * 32 + lane];
          ka[u] = need_m1 ? pf[(u * NCOL + ND) * 32 + lane] : make_int4(0, 0, 0, 0);
          kb[u] = need_m2 ? pf[(u * NCOL + ND + 1) * 32 + lane] : make_int4(0, 0, 0, 0);
        } else {
#pragma unroll
          for (int j = 0; j < ND; ++j) kf[u][j] = make_int4(0, 0, 0, 0);
          ka[u] = kb[u] = make_int4(0, 0, 0, 0);
        }
      }
      __syncwarp();
      if (lane == 0) {
        fence_proxy_async_smem();  // the reads above before the buffer is refilled
        if (w0 + wstride < nvec) issue(w0 + wstride);
      }
    } else {
#pragma unroll
      for (int u = 0; u < NG; ++u) {
        const uint32_t gi = i + u * gstride;
        if ((u == 0 && !CMP) || gi < nvec) {
          alive |= 0xFu << (4 * u);
#pragma unroll
          for (int j = 0; j < ND; ++j) kf[u][j] = ld_stream_v4(fkb[j] + 4ull * gi, pol_stream);
          ka[u] = ld_stream_v4_if(need_m1, m1b + 4ull * gi, pol_stream);
          kb[u] = ld_stream_v4_if(need_m2, m2b + 4ull * gi, pol_stream);
        } else {
#pragma unroll
          for (int j = 0; j < ND; ++j) kf[u][j] = make_int4(0, 0, 0, 0);
          ka[u] = kb[u] = make_int4(0, 0, 0, 0);
        }
      }
    }
    auto key = [&](int r, int j) -> uint32_t {
      const int4& v = kf[r >> 2][j];
      const int c = r & 3;
      return static_cast<uint32_t>(c == 0 ? v.x : c == 1 ? v.y : c == 2 ? v.z : v.w);
    };
    auto mx = [&](const int4* m, int r) -> int32_t {
      const int4& v = m[r >> 2];
      const int c = r & 3;
      return c == 0 ? v.x : c == 1 ? v.y : c == 2 ? v.z : v.w;
    };
    // Range check of every key (registers only).  A row with a key out of
    // range is dropped here and only flagged: whether it is a range error
    // (none of its in-range keys meets DIM_NULL) is decided by the range pass
    // that runs after this kernel when the flag is set, so the rare case adds
    // nothing to this loop's registers.
    uint32_t oob = 0;
#pragma unroll
    for (int r = 0; r < V; ++r) {
      bool ok = true;
#pragma unroll
      for (int j = 0; j < ND; ++j) ok &= key(r, j) < p.dim[j].len;
      if (!ok) oob |= 1u << r;
    }
    oob &= alive;
    if (oob) {
      *reinterpret_cast<volatile unsigned long long*>(p.oob_seen) = 1ull;
      alive &= ~oob;
      // keys of dropped rows to 0: every key left in registers addresses
      // its vector, so no probe below can leave it, predicated or not
#pragma unroll
      for (int u = 0; u < NG; ++u) {
        const uint32_t ob = (oob >> (4 * u)) & 0xFu;
        if (!ob) continue;
#pragma unroll
        for (int j = 0; j < ND; ++j) {
          int4& v = kf[u][j];
          if (ob & 1u) v.x = 0;
          if (ob & 2u) v.y = 0;
          if (ob & 4u) v.z = 0;
          if (ob & 8u) v.w = 0;
        }
      }
    }
    int32_t g[V];
#pragma unroll
    for (int r = 0; r < V; ++r) g[r] = 0;
    bool skip = false;  // this dimension was probed with the previous one
#pragma unroll
    for (int j = 0; j < ND; ++j) {
      if (alive == 0) break;
      if (skip) {
        skip = false;
        continue;
      }
      const Probe& d = p.dim[j];
      if (CMP && d.soff < 0 && d.boff < 0) continue;  // global dimensions: after the compaction
      if (d.noff >= 0 && nib_ok[j]) {
        // 4-bit codes in shared memory: filter and group code in one probe
        const uint8_t* sn = reinterpret_cast<const uint8_t*>(sdim + d.noff);
#pragma unroll
        for (int r = 0; r < V; ++r) {
          if (alive & (1u << r)) {
            const uint32_t k = key(r, j);
            const int32_t c = (sn[k >> 1] >> ((k & 1u) << 2)) & 15;
            if (c == 15) alive &= ~(1u << r);
            g[r] += c * d.factor;
          }
        }
      } else if (d.soff >= 0) {
        const int8_t* sv = reinterpret_cast<const int8_t*>(sdim + d.soff);
#pragma unroll
        for (int r = 0; r < V; ++r) {
          if (alive & (1u << r)) {
            const int32_t c = sv[key(r, j)];
            if (c == OLAP_DIM_NULL) alive &= ~(1u << r);
            g[r] += c * d.factor;
          }
        }
      } else if (d.boff >= 0) {
        const uint32_t* sw = reinterpret_cast<const uint32_t*>(sdim + d.boff);
#pragma unroll
        for (int r = 0; r < V; ++r) {
          const uint32_t k = key(r, j);
          if ((alive & (1u << r)) && !((sw[k >> 5] >> (k & 31)) & 1u)) alive &= ~(1u << r);
        }
      } else if (d.bits) {
        uint32_t w[V];
#pragma unroll
        for (int r = 0; r < V; ++r) w[r] = (alive & (1u << r)) ? __ldg(d.bits + (key(r, j) >> 5)) : 0u;
#pragma unroll
        for (int r = 0; r < V; ++r)
          if (!((w[r] >> (key(r, j) & 31)) & 1u)) alive &= ~(1u << r);
      } else {
        // int8 probe through L2; with merge_global, the next dimension's too
        // when it is also one (both in flight: one round trip instead of two)
        const int j1 = j + 1 < ND ? j + 1 : j;
        const Probe& d1 = p.dim[j1];
        const bool two = !CMP && p.merge_global && j + 1 < ND && d1.soff < 0 && d1.boff < 0 && !d1.bits &&
                         !(d1.noff >= 0 && nib_ok[j1]);
        int32_t c[V], c1[V];
#pragma unroll
        for (int r = 0; r < V; ++r)
          c[r] = (alive & (1u << r)) ? ld_probe_s8(d.vec + key(r, j), pol_keep) : OLAP_DIM_NULL;
        if (two) {
#pragma unroll
          for (int r = 0; r < V; ++r)
            c1[r] = (alive & (1u << r)) ? ld_probe_s8(d1.vec + key(r, j1), pol_keep) : OLAP_DIM_NULL;
        }
#pragma unroll
        for (int r = 0; r < V; ++r) {
          if (c[r] == OLAP_DIM_NULL) alive &= ~(1u << r);
          g[r] += c[r] * d.factor;
        }
        if (two) {
#pragma unroll
          for (int r = 0; r < V; ++r) {
            if (c1[r] == OLAP_DIM_NULL) alive &= ~(1u << r);
            g[r] += c1[r] * d1.factor;
          }
          skip = true;
        }
      }
    }
    // One surviving row: group id check, aggregates, accumulate.
    auto add_row = [&](uint32_t gg, int32_t x, int32_t y) {
      if (gg >= n_groups) {
        ++bad;
        return;
      }
      int64_t v0, v1 = 0;
      if (AGGK == AGGK_M1PM2) {
        v0 = static_cast<int64_t>(x) + y;
      } else if (AGGK == AGGK_M1_M1M2) {
        v0 = x;
        v1 = static_cast<int64_t>(x) * y;
      } else {
        v0 = agg_value(p.agg0, x, y);
        v1 = p.n_aggs > 1 ? agg_value(p.agg1, x, y) : 0;
      }
      tot0 += v0;
      if (ACC == ACC_SMEM) smem_add_split(sw, nacc, gg, static_cast<uint64_t>(v0));
      if (ACC == ACC_GLOBAL) atomicAdd(&p.out[gg], static_cast<unsigned long long>(v0));
      if (AGGK == AGGK_M1_M1M2 || (AGGK == AGGK_GENERIC && p.n_aggs > 1)) {
        tot1 += v1;
        if (ACC == ACC_SMEM) smem_add_split(sw, nacc, n_groups + gg, static_cast<uint64_t>(v1));
        if (ACC == ACC_GLOBAL) atomicAdd(&p.out[n_groups + gg], static_cast<unsigned long long>(v1));
      }
    };
    if (CMP) {
      // pack the warp's survivors: row (slot r, lane l) goes to position
      // (survivors of slots < r) + (survivors of slot r in lanes < l)
      constexpr int ROWS = 32 * V;  // rows of a warp step
      uint32_t* sb = reinterpret_cast<uint32_t*>(smem + p.cmp_off) + (tid >> 5) * ((ND + 3) * ROWS);
      const uint32_t lt = (1u << lane) - 1u;
      uint32_t tot = 0;
#pragma unroll
      for (int r = 0; r < V; ++r) {
        const uint32_t b = __ballot_sync(0xffffffffu, (alive >> r) & 1u);
        if ((alive >> r) & 1u) {
          const uint32_t at = tot + __popc(b & lt);
#pragma unroll
          for (int j = 0; j < ND; ++j) sb[j * ROWS + at] = key(r, j);
          sb[ND * ROWS + at] = static_cast<uint32_t>(g[r]);
          sb[(ND + 1) * ROWS + at] = static_cast<uint32_t>(mx(ka, r));
          sb[(ND + 2) * ROWS + at] = static_cast<uint32_t>(mx(kb, r));
        }
        tot += __popc(b);
      }
      if (tot == 0) continue;
      __syncwarp();
      for (uint32_t base = 0; base < tot; base += 32) {
        const uint32_t at = base + lane;
        bool live = at < tot;
        uint32_t k[ND > 0 ? ND : 1];
        int32_t gg = 0, x = 0, y = 0;
        if (live) {
#pragma unroll
          for (int j = 0; j < ND; ++j) k[j] = sb[j * ROWS + at];
          gg = static_cast<int32_t>(sb[ND * ROWS + at]);
          x = static_cast<int32_t>(sb[(ND + 1) * ROWS + at]);
          y = static_cast<int32_t>(sb[(ND + 2) * ROWS + at]);
        } else {
#pragma unroll
          for (int j = 0; j < ND; ++j) k[j] = 0;
        }
#pragma unroll
        for (int j = 0; j < ND; ++j) {
          const Probe& d = p.dim[j];
          if (d.soff >= 0 || d.boff >= 0) continue;
          if (d.bits) {
            const uint32_t w = live ? __ldg(d.bits + (k[j] >> 5)) : 0u;
            if (!((w >> (k[j] & 31)) & 1u)) live = false;
          } else {
            const int32_t c = live ? ld_probe_s8(d.vec + k[j], pol_keep) : OLAP_DIM_NULL;
            if (c == OLAP_DIM_NULL) live = false;
            gg += c * d.factor;
          }
        }
#pragma unroll
        for (int j = 0; j < ND; ++j) {
          const Probe& d = p.dim[j];
          if (d.soff < 0 && d.bits && need_code[j]) {
            const int32_t c = live ? ld_probe_s8(d.vec + k[j], pol_keep) : 0;
            gg += c * d.factor;
          }
        }
        if (live) add_row(static_cast<uint32_t>(gg), x, y);
      }
      __syncwarp();  // the buffer is rewritten in the next step
      continue;
    }
    if (alive == 0) continue;
#pragma unroll
    for (int j = 0; j < ND; ++j) {
      const Probe& d = p.dim[j];
      if (d.soff < 0 && d.bits && need_code[j]) {
        int32_t c[V];
#pragma unroll
        for (int r = 0; r < V; ++r)
          c[r] = (alive & (1u << r)) ? ld_probe_s8(d.vec + key(r, j), pol_keep) : 0;
#pragma unroll
        for (int r = 0; r < V; ++r) g[r] += c[r] * d.factor;
      }
    }
#pragma unroll
    for (int r = 0; r < V; ++r)
      if (alive & (1u << r)) add_row(static_cast<uint32_t>(g[r]), mx(ka, r), mx(kb, r));
  }
  // Head and tail rows outside the 16-byte aligned range (block 0).
  if (blockIdx.x == 0) {
    auto one = [&](int64_t r) {
      uint32_t k[ND > 0 ? ND : 1];
      bool ok = true;
#pragma unroll
      for (int j = 0; j < ND; ++j) {
        k[j] = static_cast<uint32_t>(p.dim[j].fk[r]);
        ok &= k[j] < p.dim[j].len;
      }
      if (!ok) {  // dropped and flagged; the range pass decides whether it is a range error
        *reinterpret_cast<volatile unsigned long long*>(p.oob_seen) = 1ull;
        return;
      }
      int64_t g = 0;
#pragma unroll
      for (int j = 0; j < ND; ++j) {
        const int32_t c = p.dim[j].soff >= 0 ? static_cast<int8_t>(sdim[p.dim[j].soff + k[j]]) : p.dim[j].vec[k[j]];
        if (c == OLAP_DIM_NULL) return;
        g += static_cast<int64_t>(c) * p.dim[j].factor;
      }
      if (static_cast<uint64_t>(g) >= static_cast<uint64_t>(p.n_groups)) {
        ++bad;
        return;
      }
      const int32_t x = p.need_m1 ? p.m1[r] : 0, y = p.need_m2 ? p.m2[r] : 0;
      const int64_t v0 = agg_value(p.agg0, x, y);
      tot0 += v0;
      if (ACC == ACC_SMEM) smem_add_split(sw, nacc, g, static_cast<uint64_t>(v0));
      if (ACC == ACC_GLOBAL) atomicAdd(&p.out[g], static_cast<unsigned long long>(v0));
      if (p.n_aggs > 1) {
        const int64_t v1 = agg_value(p.agg1, x, y);
        tot1 += v1;
        if (ACC == ACC_SMEM) smem_add_split(sw, nacc, p.n_groups + g, static_cast<uint64_t>(v1));
        if (ACC == ACC_GLOBAL) atomicAdd(&p.out[p.n_groups + g], static_cast<unsigned long long>(v1));
      }
    };
    for (int64_t r = p.row_begin + tid; r < p.vec_begin; r += blockDim.x) one(r);
    for (int64_t r = p.vec_end + tid; r < p.row_end; r += blockDim.x) one(r);
  }
  finish_block<ACC>(p, tot0, tot1, bad, sacc, nacc, red, &red_bad);
}

// Generic path: one row per thread step, 32-bit loads, int64 group ids.  Used
// for columns that are not 16-byte aligned and for plans whose group-id
// arithmetic could leave int32.
template <int ND, int ACC>
__global__ void __launch_bounds__(1024, 1) starjoin_scalar_kernel(const StarParams p) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ long long red[32][2];
  __shared__ unsigned int red_bad;
  __shared__ int32_t s_code_nz[OLAP_MAX_DIMS];
  unsigned char* sdim = smem;
  unsigned long long* sacc = reinterpret_cast<unsigned long long*>(smem + p.smem_dim_bytes);
  uint32_t* sw = reinterpret_cast<uint32_t*>(sacc);  // accumulator words: low words, then high words
  const int tid = threadIdx.x;
  const int64_t nacc = p.n_groups * p.n_aggs;
  if (tid == 0) red_bad = 0;
  if (tid < OLAP_MAX_DIMS)
    s_code_nz[tid] = (tid < ND && p.dim[tid].code_flag >= 0) ? p.code_nonzero[p.dim[tid].code_flag] : 0;
  stage_block<ND, ACC>(p, sdim, sacc, nacc);
  __syncthreads();
  const uint64_t pol_stream = policy_evict_first();
  const uint64_t pol_keep = policy_evict_last();
  int64_t tot0 = 0, tot1 = 0;
  unsigned int bad = 0;
  const int64_t gstride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t r = p.row_begin + static_cast<int64_t>(blockIdx.x) * blockDim.x + tid; r < p.row_end;
       r += gstride) {
    uint32_t k[ND > 0 ? ND : 1];
    bool ok = true;
#pragma unroll
    for (int j = 0; j < ND; ++j) {
      k[j] = static_cast<uint32_t>(ld_stream_s32(p.dim[j].fk + r, pol_stream));
      ok &= k[j] < p.dim[j].len;
    }
    const int32_t x = ld_stream_s32_if(p.need_m1, p.m1 + r, pol_stream, 0);
    const int32_t y = ld_stream_s32_if(p.need_m2, p.m2 + r, pol_stream, 0);
    if (!ok) {  // a range error unless an in-range key meets DIM_NULL
      bool filtered = false;
#pragma unroll
      for (int j = 0; j < ND; ++j)
        if (k[j] < p.dim[j].len && p.dim[j].vec[k[j]] == OLAP_DIM_NULL) filtered = true;
      bad += filtered ? 0u : 1u;
      continue;
    }
    int64_t g = 0;
    bool live = true;
#pragma unroll
    for (int j = 0; j < ND; ++j) {
      if (!live) break;
      const Probe& d = p.dim[j];
      int32_t c;
      if (d.soff >= 0) {
        c = static_cast<int8_t>(sdim[d.soff + k[j]]);
      } else {
        if (d.boff >= 0) {
          const uint32_t* sw = reinterpret_cast<const uint32_t*>(sdim + d.boff);
          if (!((sw[k[j] >> 5] >> (k[j] & 31)) & 1u)) { live = false; break; }
        } else if (d.bits) {
          if (!((__ldg(d.bits + (k[j] >> 5)) >> (k[j] & 31)) & 1u)) { live = false; break; }
        }
        c = ld_probe_s8_if(ok, d.vec + k[j], pol_keep, OLAP_DIM_NULL);  // ok: all keys in range here
      }
      if (c == OLAP_DIM_NULL) live = false;
      else g += static_cast<int64_t>(c) * d.factor;
    }
    if (!live) continue;
    if (static_cast<uint64_t>(g) >= static_cast<uint64_t>(p.n_groups)) {
      ++bad;
      continue;
    }
    const int64_t v0 = agg_value(p.agg0, x, y);
    tot0 += v0;
    if (ACC == ACC_SMEM) smem_add_split(sw, nacc, g, static_cast<uint64_t>(v0));
    if (ACC == ACC_GLOBAL) atomicAdd(&p.out[g], static_cast<unsigned long long>(v0));
    if (p.n_aggs > 1) {
      const int64_t v1 = agg_value(p.agg1, x, y);
      tot1 += v1;
      if (ACC == ACC_SMEM) smem_add_split(sw, nacc, p.n_groups + g, static_cast<uint64_t>(v1));
      if (ACC == ACC_GLOBAL) atomicAdd(&p.out[p.n_groups + g], static_cast<unsigned long long>(v1));
    }
  }
  finish_block<ACC>(p, tot0, tot1, bad, sacc, nacc, red, &red_bad);
}

using StarKernel = void (*)(const StarParams);

// Range pass of the 128-bit kernel.  That kernel drops a row with a key out
// of range and only sets p.oob_seen; when the flag is set, this pass counts
// the rows of [row_begin, row_end) with a key out of range and no in-range
// key meeting DIM_NULL (the rows the plain path counts as range errors).
// With the flag clear (the normal case) every block returns at once.
template <int ND>
__global__ void __launch_bounds__(256) starjoin_range_pass_kernel(const StarParams p) {
  if (*reinterpret_cast<const volatile unsigned long long*>(p.oob_seen) == 0ull) return;
  unsigned int bad = 0;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t r = p.row_begin + static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < p.row_end;
       r += stride) {
    uint32_t k[ND > 0 ? ND : 1];
    bool ok = true;
#pragma unroll
    for (int j = 0; j < ND; ++j) {
      k[j] = static_cast<uint32_t>(p.dim[j].fk[r]);
      ok &= k[j] < p.dim[j].len;
    }
    if (ok) continue;
    bool filtered = false;
#pragma unroll
    for (int j = 0; j < ND; ++j)
      if (k[j] < p.dim[j].len && p.dim[j].vec[k[j]] == OLAP_DIM_NULL) filtered = true;
    bad += filtered ? 0u : 1u;
  }
  const unsigned int wbad = __reduce_add_sync(0xffffffffu, bad);
  if ((threadIdx.x & 31) == 0 && wbad) atomicAdd(p.range_err, static_cast<unsigned long long>(wbad));
}

static StarKernel pick_range_pass(int nd) {
  switch (nd) {
    case 1: return starjoin_range_pass_kernel<1>;
    case 2: return starjoin_range_pass_kernel<2>;
    case 3: return starjoin_range_pass_kernel<3>;
    default: return starjoin_range_pass_kernel<4>;
  }
}

template <int ND, int ACC, bool ASYNC>
static StarKernel pick_vec_a(int aggk, int v) {
  if (v >= 8) {
    switch (aggk) {
      case AGGK_M1PM2: return starjoin_vec_kernel<ND, ACC, AGGK_M1PM2, 8, ASYNC, false>;
      case AGGK_M1_M1M2: return starjoin_vec_kernel<ND, ACC, AGGK_M1_M1M2, 8, ASYNC, false>;
      default: return starjoin_vec_kernel<ND, ACC, AGGK_GENERIC, 8, ASYNC, false>;
    }
  }
  switch (aggk) {
    case AGGK_M1PM2: return starjoin_vec_kernel<ND, ACC, AGGK_M1PM2, 4, ASYNC, false>;
    case AGGK_M1_M1M2: return starjoin_vec_kernel<ND, ACC, AGGK_M1_M1M2, 4, ASYNC, false>;
    default: return starjoin_vec_kernel<ND, ACC, AGGK_GENERIC, 4, ASYNC, false>;
  }
}

// Compaction: 4 rows per thread, loads straight to registers.
template <int ND, int ACC>
static StarKernel pick_vec_cmp(int aggk) {
  switch (aggk) {
    case AGGK_M1PM2: return starjoin_vec_kernel<ND, ACC, AGGK_M1PM2, 4, false, true>;
    case AGGK_M1_M1M2: return starjoin_vec_kernel<ND, ACC, AGGK_M1_M1M2, 4, false, true>;
    default: return starjoin_vec_kernel<ND, ACC, AGGK_GENERIC, 4, false, true>;
  }
}

template <int ND, int ACC>
static StarKernel pick_vec(int aggk, int v, bool async, bool cmp) {
  if (cmp && ND >= 1) return pick_vec_cmp<ND, ACC>(aggk);
  return async ? pick_vec_a<ND, ACC, true>(aggk, v) : pick_vec_a<ND, ACC, false>(aggk, v);
}

template <int ND>
static StarKernel pick_kernel(int acc, bool vec, int aggk, int v, bool async, bool cmp) {
  switch (acc) {
    case ACC_NONE: return vec ? pick_vec<ND, ACC_NONE>(aggk, v, async, cmp) : starjoin_scalar_kernel<ND, ACC_NONE>;
    case ACC_SMEM: return vec ? pick_vec<ND, ACC_SMEM>(aggk, v, async, cmp) : starjoin_scalar_kernel<ND, ACC_SMEM>;
    default: return vec ? pick_vec<ND, ACC_GLOBAL>(aggk, v, async, cmp) : starjoin_scalar_kernel<ND, ACC_GLOBAL>;
  }
}

static StarKernel select_kernel(int nd, int acc, bool vec, int aggk, int v, bool async, bool cmp) {
  switch (nd) {
    case 0: return pick_kernel<0>(acc, vec, aggk, v, async, cmp);
    case 1: return pick_kernel<1>(acc, vec, aggk, v, async, cmp);
    case 2: return pick_kernel<2>(acc, vec, aggk, v, async, cmp);
    case 3: return pick_kernel<3>(acc, vec, aggk, v, async, cmp);
    default: return pick_kernel<4>(acc, vec, aggk, v, async, cmp);
  }
}

static bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

// A planned launch: parameters, kernel choice and the bitmap builds it needs.
struct StarPlan {
  StarParams sp;
  int nd = 0;
  int acc = ACC_NONE;
  bool vec = false;
  int aggk = 0;    // AGGK_* of the 128-bit path
  int rows_v = 4;  // rows per thread per iteration (4 or 8)
  bool async = false;  // bulk-copy prefetch of the streamed columns (TUNE_ASYNC_LOADS)
  bool cmp = false;    // warp compaction of the survivors of the shared-memory probes (TUNE_COMPACT)
  int block = 512;
  size_t smem = 0;
  int nbits = 0;                       // dims whose pass bitmap must be built
  int bits_dim[OLAP_MAX_DIMS] = {};    // probe index of each
  uint32_t* bits_buf[OLAP_MAX_DIMS] = {};
  int32_t* code_nz = nullptr;          // [2 * OLAP_MAX_DIMS] in the arena
  int nnib = 0;                        // dims whose 4-bit codes must be built
  int nib_dim[OLAP_MAX_DIMS] = {};
  uint8_t* nib_buf[OLAP_MAX_DIMS] = {};
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
  int kind[OLAP_MAX_DIMS] = {0, 0, 0, 0};  // 1 int8 staged, 2 bitmap staged, 3 global bitmap, 4 nibbles staged
  int64_t used = 0;
  for (int t = 0; t < nd; ++t) {
    const int j = idx[t];
    const int64_t bytes = (q->dimvec_len[j] + 15) & ~int64_t(15);
    if (used + bytes <= smem_dim_budget) {
      kind[j] = 1;
      used += bytes;
    }
  }
  // 4-bit codes (filter and group code in one shared-memory probe) up to
  // TUNE_SMEM_NIB_BYTES, in the caller's order.
  const int64_t smem_nib_budget = tune_or(ctx, TUNE_SMEM_NIB_BYTES, 0);
  int64_t nib_used = 0;
  for (int j = 0; j < nd; ++j) {
    if (kind[j] || empty) continue;
    const int64_t nbytes = ((q->dimvec_len[j] + 1) / 2 + 15) & ~int64_t(15);
    if (nib_used + nbytes <= smem_nib_budget && used + nib_used + nbytes <= smem_cap) {
      kind[j] = 4;
      nib_used += nbytes;
    }
  }
  used += nib_used;
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
  pl->nnib = 0;
  pl->code_nz = nullptr;
  int out = 0;
  int64_t soff = 0;
  // Probe order: shared-memory int8, shared-memory 4-bit codes, shared-memory
  // bitmaps, then the rest; with TUNE_PROBE_ORDER = 1 the shared-memory int8
  // dimensions go last (a dimension that filters nothing, such as the
  // headline's date, is then looked up only for the rows that survive).
  const bool int8_last = tune_or(ctx, TUNE_PROBE_ORDER, 2) == 1;
  const int pass_kind[4] = {int8_last ? 4 : 1, int8_last ? 2 : 4, int8_last ? 0 : 2, int8_last ? 1 : 0};
  for (int pass = 0; pass < 4; ++pass) {
    for (int j = 0; j < nd; ++j) {
      const int kj = kind[j] == 3 ? 0 : kind[j];
      if (kj != pass_kind[pass]) continue;
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
      pr.nib = nullptr;
      pr.noff = -1;
      pr.nib_flag = -1;
      if ((kind[j] >= 2) && !pl->code_nz) {
        pl->code_nz = ar.take<int32_t>(2 * OLAP_MAX_DIMS);
        if (!pl->code_nz) return set_error(ctx, OLAP_ERR_CAPACITY, "scratch arena exhausted");
      }
      if (kind[j] == 4) {
        const size_t nbytes = static_cast<size_t>((q->dimvec_len[j] + 1) / 2);
        uint8_t* nb = ar.take<uint8_t>(nbytes);
        if (!nb) return set_error(ctx, OLAP_ERR_CAPACITY, "scratch arena too small for 4-bit codes");
        pr.nib = nb;
        pr.noff = static_cast<int32_t>(soff);
        soff += (static_cast<int64_t>(nbytes) + 15) & ~int64_t(15);
        pr.nib_flag = pl->nnib;
        pl->nib_dim[pl->nnib] = k;
        pl->nib_buf[pl->nnib] = nb;
        ++pl->nnib;
      }
      if (kind[j] == 1) {
        pr.soff = static_cast<int32_t>(soff);
        soff += (q->dimvec_len[j] + 15) & ~int64_t(15);
      }
      if (kind[j] == 2 || kind[j] == 3) {
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
  if (vec) {
    int64_t vb = (q->row_begin + 3) & ~int64_t(3);
    if (vb > q->row_end) vb = q->row_end;
    const int64_t ve = vb + ((q->row_end - vb) & ~int64_t(3));
    sp->vec_begin = vb;
    sp->vec_end = ve;
  }
  // int32 group ids are exact when every partial sum of code*factor fits.
  int64_t gbound = 0;
  for (int j = 0; j < nd; ++j) gbound += 128 * std::llabs(static_cast<long long>(q->factor[j]));
  if (gbound > INT32_MAX) vec = false;
  if (vec && ((q->row_end - q->row_begin) >> 33) != 0) vec = false;
  pl->vec = vec;
  pl->aggk = AGGK_GENERIC;
  if (q->n_aggs == 1 && q->agg[0] == OLAP_AGG_M1_PLUS_M2) pl->aggk = AGGK_M1PM2;
  if (q->n_aggs == 2 && q->agg[0] == OLAP_AGG_M1 && q->agg[1] == OLAP_AGG_M1_TIMES_M2) pl->aggk = AGGK_M1_M1M2;
  pl->rows_v = tune_or(ctx, TUNE_UNROLL, 1) >= 2 ? 8 : 4;
  // One 1024-thread block per SM when large bitmaps are staged (the staging
  // copy is paid once per SM), else 512-thread blocks.
  const int dflt_block = bits_used > 64 * 1024 ? 1024 : 512;
  const int max_block = (vec && pl->rows_v == 8) ? 512 : 1024;
  pl->block = static_cast<int>(std::min<int64_t>(tune_or(ctx, TUNE_BLOCK, dflt_block), max_block));
  OLAP_REQUIRE(ctx, pl->block >= 64 && pl->block % 32 == 0, "block size must be a multiple of 32, >= 64");

  const int64_t acc_bytes = q->group_nums * q->n_aggs * 8;
  const int64_t smem_acc_budget = tune_or(ctx, TUNE_SMEM_ACC_BYTES, 96 * 1024);
  int acc = ACC_GLOBAL;
  if (!group_sums) acc = ACC_NONE;
  else if (acc_bytes <= smem_acc_budget && soff + acc_bytes <= smem_cap) acc = ACC_SMEM;
  pl->acc = acc;
  pl->smem = static_cast<size_t>(soff + (acc == ACC_SMEM ? acc_bytes : 0));
  // Bulk-copy prefetch: per warp, 32 vectors of each streamed column for each
  // group of 4 rows per thread, and one mbarrier; only when it fits.
  sp->wait_timeouts = &ctx->counters->wait_timeouts;
  sp->oob_seen = &ctx->counters->oob_seen;
  sp->merge_global = tune_or(ctx, TUNE_MERGE_PROBES, 2) == 1 ? 1 : 0;
  pl->async = false;
  if (vec && tune_or(ctx, TUNE_ASYNC_LOADS, 1) == 2 && nd + (need_m1 ? 1 : 0) + (need_m2 ? 1 : 0) > 0) {
    const int64_t warps = pl->block / 32;
    const int64_t pf_bytes = warps * (pl->rows_v / 4) * (std::max(nd, 1) + 2) * 32 * 16;
    const int64_t pf_off = (static_cast<int64_t>(pl->smem) + 127) & ~int64_t(127);
    const int64_t bar_off = pf_off + pf_bytes;
    const int64_t end = bar_off + warps * 8;
    if (end <= smem_cap) {
      pl->async = true;
      sp->pf_off = static_cast<int32_t>(pf_off);
      sp->bar_off = static_cast<int32_t>(bar_off);
      pl->smem = static_cast<size_t>(end);
    }
  }
  // Survivor compaction (4 rows per thread): per warp (ND + 3) x 128 words.
  pl->cmp = false;
  if (vec && !pl->async && pl->rows_v == 4 && nd >= 1 && tune_or(ctx, TUNE_COMPACT, 1) == 2) {
    const int64_t cmp_off = (static_cast<int64_t>(pl->smem) + 127) & ~int64_t(127);
    const int64_t end = cmp_off + (pl->block / 32) * (nd + 3) * 128 * 4;
    if (end <= smem_cap) {
      pl->cmp = true;
      sp->cmp_off = static_cast<int32_t>(cmp_off);
      pl->smem = static_cast<size_t>(end);
    }
  }
  return OLAP_OK;
}

int launch_starjoin(olap_ctx* ctx, StarPlan& pl, cudaStream_t stream) {
  // Pass bitmaps (and their code flags) first, on the same stream.
  if (pl.nbits || pl.nnib) OLAP_CUDA_TRY(ctx, cudaMemsetAsync(pl.code_nz, 0, sizeof(int32_t) * 2 * OLAP_MAX_DIMS, stream));
  for (int b = 0; b < pl.nnib; ++b) {
    const Probe& d = pl.sp.dim[pl.nib_dim[b]];
    const uint64_t nbytes = (static_cast<uint64_t>(d.len) + 1) / 2;
    const unsigned grid = static_cast<unsigned>(std::min<uint64_t>((nbytes + 255) / 256,
                                                                   static_cast<uint64_t>(ctx->sm_count) * 8));
    build_nibbles<<<grid, 256, 0, stream>>>(d.vec, d.len, pl.nib_buf[b], pl.code_nz + OLAP_MAX_DIMS + b);
    OLAP_CUDA_TRY(ctx, cudaGetLastError());
  }
  if (pl.nbits) {
    for (int b = 0; b < pl.nbits; ++b) {
      const Probe& d = pl.sp.dim[pl.bits_dim[b]];
      const uint64_t threads = ((static_cast<uint64_t>(d.len) + 31) / 32) * 32;
      const unsigned grid = static_cast<unsigned>(std::min<uint64_t>((threads + 255) / 256,
                                                                     static_cast<uint64_t>(ctx->sm_count) * 8));
      build_pass_bits<<<grid, 256, 0, stream>>>(d.vec, d.len, pl.bits_buf[b], pl.code_nz + b);
      OLAP_CUDA_TRY(ctx, cudaGetLastError());
    }
  }
  StarKernel k = select_kernel(pl.nd, pl.acc, pl.vec, pl.aggk, pl.rows_v, pl.async, pl.cmp);
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
  const bool range_pass = pl.vec && pl.nd >= 1;
  if (range_pass) OLAP_CUDA_TRY(ctx, cudaMemsetAsync(sp.oob_seen, 0, sizeof(unsigned long long), stream));
  k<<<static_cast<unsigned>(grid), pl.block, pl.smem, stream>>>(sp);
  OLAP_CUDA_TRY(ctx, cudaGetLastError());
  if (range_pass) {
    pick_range_pass(pl.nd)<<<static_cast<unsigned>(ctx->sm_count) * 2, 256, 0, stream>>>(sp);
    OLAP_CUDA_TRY(ctx, cudaGetLastError());
  }
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

int stage_host_dims(olap_ctx* ctx, const olap_starjoin_query* q, Arena& ar, olap_starjoin_query* dq) {
  const int64_t rows = q->row_end - q->row_begin;
  for (int j = 0; j < q->dimvec_nums; ++j) {
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
    ctx->host_bytes += len;
    dq->dimvec[j] = d;
    dq->dimvec_len[j] = len;
  }
  return OLAP_OK;
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
  const int sd = stage_host_dims(ctx, q, ar, &dq);
  if (sd != OLAP_OK) return sd;
  // Pinned columns are read in place (1: when that reads fewer bytes, the
  // default; 3: always) unless TUNE_HOST_INPLACE = 2 asks for the chunked
  // copies (the same sums and dropped-row count either way).
  const int64_t inplace = tune_or(ctx, TUNE_HOST_INPLACE, 1);
  if ((inplace == 1 || inplace == 3) && rows > 0) {
    bool handled = false;
    const int s = starjoin_host_inplace(ctx, q, dq, ar, group_sums, totals, &handled);
    if (handled) return s;
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
      ctx->host_bytes += n * 4;
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

// Bytes from device pointer p to the end of the device allocation holding it
// (the driver's cuMemGetAddressRange, reached through the runtime's entry
// point table so the library needs no link to libcuda).  False when p is not
// in a device allocation of the current context.
static bool device_bytes_from(const void* p, int64_t* bytes) {
  using AddressRange = CUresult (*)(CUdeviceptr*, size_t*, CUdeviceptr);
  static AddressRange fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult qr;
    if (cudaGetDriverEntryPoint("cuMemGetAddressRange", &f, cudaEnableDefault, &qr) == cudaSuccess &&
        qr == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<AddressRange>(f);
    else
      cudaGetLastError();
  });
  if (!fn || !p) return false;
  CUdeviceptr base = 0;
  size_t size = 0;
  const CUdeviceptr at = reinterpret_cast<CUdeviceptr>(p);
  if (fn(&base, &size, at) != CUDA_SUCCESS || at < base || at >= base + size) return false;
  *bytes = static_cast<int64_t>(base + size - at);
  return true;
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

int olap_starjoin_launch_count(olap_ctx* ctx, const olap_starjoin_query* q, int want_groups, int* kernels) {
  if (!ctx || !q || !kernels) return OLAP_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  OLAP_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  olap::Arena ar(ctx);
  olap::StarPlan pl;
  int64_t probe = 0;  // only its address: the plan records the output pointers
  const int st = olap::plan_starjoin(ctx, q, want_groups ? &probe : nullptr, &probe, ar, &pl);
  if (st != OLAP_OK) return st;
  // the star-join, its prepasses, and the range pass after the 128-bit kernel
  *kernels = q->row_end > q->row_begin ? 1 + pl.nbits + pl.nnib + (pl.vec && pl.nd >= 1 ? 1 : 0) : 0;
  return OLAP_OK;
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
    if (dimvec_len) {
      q.dimvec_len[j] = dimvec_len[t];
    } else {
      // No lengths (the reference's signature has none): a vector reaches to
      // the end of the device allocation that holds it, so a key past that
      // is dropped and counted, never read.
      int64_t avail = 0;
      OLAP_REQUIRE(ctx, olap::device_bytes_from(dimvec_array[t], &avail),
                   "dimvec_len is NULL and a dimension vector is not in a device allocation");
      q.dimvec_len[j] = std::min<int64_t>(avail, INT32_MAX);
    }
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
