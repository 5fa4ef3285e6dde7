// Single-pass, order-preserving stream compaction for sm_100a.
//
// Selection vectors in the reference are row ids in ascending order
// (select/test_select_option.cpp:391-423), and the column-wise OLAP core keeps
// its OID lists in row order (OLAPcore/test_multi_compute_operator.cpp
// :240-283).  The compaction here produces exactly that order in one pass
// over the input: each block claims tiles in increasing order through an
// atomic counter, ranks its selected items with warp ballots and a scan of
// the warp counts, and finds
// the tile's output offset with a decoupled look-back over the status words
// of the preceding tiles (a warp inspects 32 predecessors at a time).
//
// Every tile a block waits for was claimed earlier by a block that is already
// running, so the waits end; they are bounded anyway: after kSpinLimit polls a
// block records a timeout in the context's counters and stops, and the host
// call reports OLAP_ERR_TIMEOUT.
#pragma once

#include <type_traits>

#include "olap_internal.cuh"

namespace olap {

constexpr int kCompactThreads = 256;
constexpr int kCompactGroups = 4;  // default int4 loads per thread and tile (ops set Op::kGroups)
constexpr uint32_t kSpinLimit = 1u << 22;

// Status word of a tile: flag in bits 62-63 (0 none, 1 aggregate, 2
// inclusive prefix), value in bits 0-61.
constexpr uint64_t kFlagAgg = 1ull << 62;
constexpr uint64_t kFlagInc = 2ull << 62;
constexpr uint64_t kValMask = (1ull << 62) - 1;

struct ScanTiles {
  unsigned long long* status;   // [n_tiles], zeroed before the launch
  unsigned int* next_tile;      // claim counter, zeroed before the launch
  unsigned long long* timeouts; // context counter
  unsigned long long* total;    // selected items in all tiles (written by the last tile)
  int64_t n_tiles;
};

__device__ __forceinline__ uint64_t ld_relaxed_u64(const unsigned long long* p) {
  uint64_t v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed_u64(unsigned long long* p, uint64_t v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Claims the next tile for this block (all threads get the same id).
__device__ __forceinline__ int64_t claim_tile(const ScanTiles& st, unsigned int* s_tile) {
  if (threadIdx.x == 0) *s_tile = atomicAdd(st.next_tile, 1u);
  __syncthreads();
  const int64_t t = *s_tile;
  __syncthreads();
  return t;
}

// Exclusive prefix of this tile's count over all earlier tiles; run by one
// full warp (warp 0).  Returns -1 on timeout.
__device__ __forceinline__ int64_t lookback(const ScanTiles& st, int64_t tile, uint64_t count,
                                           uint32_t spin_limit = kSpinLimit) {
  const int lane = threadIdx.x & 31;
  if (tile == 0) {
    if (lane == 0) st_relaxed_u64(&st.status[0], kFlagInc | count);
    return 0;
  }
  if (lane == 0) st_relaxed_u64(&st.status[tile], kFlagAgg | count);
  uint64_t excl = 0;
  int64_t t = tile - 1;
  uint32_t spins = 0;
  while (true) {
    const int64_t idx = t - lane;
    uint64_t w = idx >= 0 ? ld_relaxed_u64(&st.status[idx]) : kFlagInc;
    while (__any_sync(0xffffffffu, (w >> 62) == 0)) {
      if (++spins > spin_limit) {
        if (lane == 0) atomicAdd(st.timeouts, 1ull);
        return -1;
      }
      __nanosleep(64);
      if ((w >> 62) == 0) w = ld_relaxed_u64(&st.status[idx]);
    }
    const uint32_t inc = __ballot_sync(0xffffffffu, (w >> 62) == 2);
    uint64_t v = w & kValMask;
    if (inc) {
      const int k = __ffs(inc) - 1;  // closest predecessor with an inclusive prefix
      if (lane > k) v = 0;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      excl += v;
      break;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    excl += v;
    t -= 32;
  }
  if (lane == 0) st_relaxed_u64(&st.status[tile], kFlagInc | (excl + count));
  return static_cast<int64_t>(excl);
}

// Compaction kernel.  Items are numbered 0 .. n_items-1.  A tile holds
// kCompactThreads x 4 x G items (G = Op::kGroups); in group u, lane l of
// warp w owns the 4 consecutive items tile_first + u*1024 + w*128 + 4l + k,
// so each group is one coalesced 16-byte load per thread and row order is
// (u, w, l, k).  A thread ranks its selected items inside its warp with four
// ballots, the block ranks the (u, w) warp counts with one warp scan, and the
// tile's output base comes from the look-back.  The Op is called per group
// and per selected item:
//   template <bool kFull> uint32_t op.flags(int u, int64_t first, int nv)
//       -> 4-bit mask of the selected items among first .. first+3 (only the
//       first nv exist); kFull: nv == 4 and op.vec_ok() (16-byte loads are
//       allowed), and op.prefetch(u, first) ran for every group first; the
//       op may cache what it loaded for group u;
//   void op.emit(int u, int k, int64_t item, int64_t pos)  -> write selected
//       item `item` (= first + k of group u) at output position `pos`.
// A larger G keeps more bytes in flight per block for ops that cache little.
// Rounds per tile: an op whose emit() needs nothing cached from flags()
// (Op::kRounds > 1) takes that many consecutive sub-tiles of kGroups loads
// per thread into one tile, keeping only their 4-bit masks, so that one
// look-back covers R times the bytes.
template <class Op, class = void>
struct OpRounds {
  static constexpr int value = 1;
};
template <class Op>
struct OpRounds<Op, std::void_t<decltype(Op::kRounds)>> {
  static constexpr int value = Op::kRounds;
};

template <class Op>
constexpr int64_t compact_sub_items() {
  return static_cast<int64_t>(kCompactThreads) * 4 * Op::kGroups;
}
template <class Op>
constexpr int64_t compact_tile_items() {
  return compact_sub_items<Op>() * OpRounds<Op>::value;
}

template <class Op>
__global__ void __launch_bounds__(kCompactThreads) compact_kernel(const Op op_in, int64_t n_items, ScanTiles st) {
  constexpr int G = Op::kGroups;
  constexpr int R = OpRounds<Op>::value;
  constexpr int W = kCompactThreads / 32;
  constexpr int E = R * G * W;  // warp counts per tile
  static_assert(G <= 16 && E % 32 == 0, "groups per thread: a multiple of 4, at most 16");
  constexpr int PER = E / 32;
  constexpr int64_t SUB = compact_sub_items<Op>();
  Op op = op_in;  // per-thread copy: ops cache the loaded items between flags() and emit()
  __shared__ unsigned int s_tile;
  __shared__ uint32_t s_cnt[E];  // warp counts of (r, u, w), then their exclusive prefixes in the tile
  __shared__ long long s_base;
  // masks of the rounds before the last (one round in flight at a time keeps
  // the registers of a single round)
  __shared__ uint64_t s_mask[R > 1 ? R - 1 : 1][kCompactThreads];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t lt = (1u << lane) - 1u;
  for (;;) {
    const int64_t tile = claim_tile(st, &s_tile);
    if (tile >= st.n_tiles) return;
    const int64_t tile_first = tile * compact_tile_items<Op>();
    const bool full = op.vec_ok() && tile_first + compact_tile_items<Op>() <= n_items;
    uint64_t last = 0;  // 4 bits per group of the last round
#pragma unroll 1
    for (int r = 0; r < R; ++r) {
      const int64_t sub_first = tile_first + r * SUB;
      uint64_t mk = 0;
      if (full) {
        // full tile, aligned columns: every group's loads are issued before
        // the first is used, so G x 16 bytes per thread are in flight
#pragma unroll
        for (int u = 0; u < G; ++u)
          op.prefetch(u, sub_first + static_cast<int64_t>(u) * kCompactThreads * 4 + 4 * threadIdx.x);
#pragma unroll
        for (int u = 0; u < G; ++u) {
          const int64_t first = sub_first + static_cast<int64_t>(u) * kCompactThreads * 4 + 4 * threadIdx.x;
          mk |= static_cast<uint64_t>(op.template flags<true>(u, first, 4)) << (4 * u);
        }
      } else {
#pragma unroll
        for (int u = 0; u < G; ++u) {
          const int64_t first = sub_first + static_cast<int64_t>(u) * kCompactThreads * 4 + 4 * threadIdx.x;
          const int64_t left = n_items - first;
          const int nv = left >= 4 ? 4 : (left > 0 ? static_cast<int>(left) : 0);
          const uint32_t m = nv > 0 ? op.template flags<false>(u, first, nv) : 0u;
          mk |= static_cast<uint64_t>(m) << (4 * u);
        }
      }
      if (r + 1 < R) s_mask[r][threadIdx.x] = mk;
      else last = mk;
#pragma unroll
      for (int u = 0; u < G; ++u) {
        const uint32_t c = __reduce_add_sync(0xffffffffu, __popc(static_cast<uint32_t>(mk >> (4 * u)) & 15u));
        if (lane == 0) s_cnt[(r * G + u) * W + warp] = c;
      }
    }
    __syncthreads();
    if (warp == 0) {
      uint32_t v[PER];
      uint32_t sum = 0;
#pragma unroll
      for (int i = 0; i < PER; ++i) {
        v[i] = s_cnt[lane * PER + i];
        sum += v[i];
      }
      uint32_t inc = sum;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
      }
      uint32_t run = inc - sum;
#pragma unroll
      for (int i = 0; i < PER; ++i) {
        s_cnt[lane * PER + i] = run;
        run += v[i];
      }
      const uint64_t tile_count = __shfl_sync(0xffffffffu, inc, 31);
      const int64_t b = lookback(st, tile, tile_count);
      if (lane == 0) {
        s_base = b;
        if (tile == st.n_tiles - 1 && b >= 0) *st.total = static_cast<unsigned long long>(b) + tile_count;
      }
    }
    __syncthreads();
    const long long base = s_base;
    if (base < 0) return;  // timed out: the host reports it
#pragma unroll 1
    for (int r = 0; r < R; ++r) {
      const uint64_t mk = r + 1 < R ? s_mask[r][threadIdx.x] : last;
#pragma unroll
      for (int u = 0; u < G; ++u) {
        const uint32_t m = static_cast<uint32_t>(mk >> (4 * u)) & 15u;
        uint32_t before = 0;
#pragma unroll
        for (int k = 0; k < 4; ++k) before += __popc(__ballot_sync(0xffffffffu, (m >> k) & 1u) & lt);
        if (!m) continue;
        int64_t pos = base + s_cnt[(r * G + u) * W + warp] + before;
        const int64_t first = tile_first + r * SUB + static_cast<int64_t>(u) * kCompactThreads * 4 + 4 * threadIdx.x;
#pragma unroll
        for (int k = 0; k < 4; ++k)
          if ((m >> k) & 1u) op.emit(u, k, first + k, pos++);
      }
    }
  }
}

// Host helper: scan-tile state for n_items in tiles of tile_items
// (compact_tile_items<Op>()) from the arena; zeroes it on the stream.
inline int make_scan_tiles(olap_ctx* ctx, Arena& ar, int64_t n_items, unsigned long long* total,
                           cudaStream_t stream, ScanTiles* st, int64_t tile_items) {
  st->n_tiles = (n_items + tile_items - 1) / tile_items;
  if (st->n_tiles < 1) st->n_tiles = 1;
  st->status = ar.take<unsigned long long>(static_cast<size_t>(st->n_tiles));
  st->next_tile = ar.take<unsigned int>(1);
  st->timeouts = &ctx->counters->wait_timeouts;
  st->total = total;
  if (!st->status || !st->next_tile)
    return set_error(ctx, OLAP_ERR_CAPACITY, "scratch arena too small for the compaction state");
  OLAP_CUDA_TRY(ctx, cudaMemsetAsync(st->status, 0, sizeof(unsigned long long) * st->n_tiles, stream));
  OLAP_CUDA_TRY(ctx, cudaMemsetAsync(st->next_tile, 0, sizeof(unsigned int), stream));
  if (total) OLAP_CUDA_TRY(ctx, cudaMemsetAsync(total, 0, sizeof(unsigned long long), stream));
  return OLAP_OK;
}

inline unsigned compact_grid(const olap_ctx* ctx, int64_t n_tiles) {
  int64_t g = static_cast<int64_t>(ctx->sm_count) * 8;  // 8 x 256 threads per SM
  if (g > n_tiles) g = n_tiles;
  return static_cast<unsigned>(g < 1 ? 1 : g);
}

// Checks the wait-timeout counter after a synchronising call.
inline int check_timeouts(olap_ctx* ctx, cudaStream_t stream) {
  unsigned long long t = 0;
  OLAP_CUDA_TRY(ctx, cudaMemcpyAsync(&t, &ctx->counters->wait_timeouts, sizeof(t),
                                     cudaMemcpyDeviceToHost, stream));
  OLAP_CUDA_TRY(ctx, cudaStreamSynchronize(stream));
  if (t) {
    OLAP_CUDA_TRY(ctx, cudaMemsetAsync(&ctx->counters->wait_timeouts, 0, sizeof(t), stream));
    return set_error(ctx, OLAP_ERR_TIMEOUT, "a bounded device wait expired in a compaction");
  }
  return OLAP_OK;
}

}  // namespace olap
