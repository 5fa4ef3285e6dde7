// Equi-join build and probe for sm_100a.
//
// Reference: code/join/test_join_option.cpp.  build(R, int* vector) stores
// vector[key] = payload (:30-36) and probe(S, vector) sums vector[key] over
// the probe keys (:58-64); the hash variants do the same through
// std::unordered_map (:44-50, :90-96), where operator[] makes a missing key
// contribute 0.  With duplicate build keys the sequential build keeps the last
// row's payload; both builds here keep exactly that row.
//
// Hash table (a format of this library): 2^k 64-bit slots, open addressing
// with linear probing over 32-byte buckets of 4 slots (one DRAM sector per
// probe step).  During the build a slot holds (key << 32 | row) so that a
// duplicate key keeps the largest row with one 64-bit atomicMax; a finishing
// pass replaces the row by that row's payload, so a probe reads key and
// payload in one load.  The key INT32_MIN marks an empty slot and cannot be
// built (such build rows are counted as range errors).
#include <cstring>

#include "compact.cuh"

namespace olap {

constexpr uint64_t kEmptySlot = 0x80000000FFFFFFFFull;  // key INT32_MIN, row 0xffffffff

__host__ __device__ __forceinline__ uint32_t hash32(uint32_t x) {  // murmur3 finaliser
  x ^= x >> 16;
  x *= 0x85ebca6bu;
  x ^= x >> 13;
  x *= 0xc2b2ae35u;
  x ^= x >> 16;
  return x;
}

// Home slot of key k in a table of `cap` slots: the hash scaled onto
// [0, cap) by a multiply and shift, so the capacity need not be a power of
// two (a caller sizes the table to its build side, any multiple of 8).
// Linear probing moves forward and wraps at the end.
__host__ __device__ __forceinline__ uint64_t home_slot(uint32_t k, uint64_t cap) {
  return (static_cast<uint64_t>(hash32(k)) * cap) >> 32;
}
__host__ __device__ __forceinline__ uint64_t next_slot(uint64_t h, uint64_t cap) { return h + 1 == cap ? 0 : h + 1; }

// Blocked Bloom filter of the build keys (a format of this library, built
// beside the table): 2^w 64-bit words, about 8 bits per build key; a key sets
// four bits of one word (the word from the top bits of hash32, the bits from
// a second hash).  A probe key whose four bits are not all set cannot match,
// so it skips the table: one L2-resident 8-byte read instead of a DRAM
// sector of the table.  About 2-4 % of absent keys pass anyway.
__host__ __device__ __forceinline__ uint32_t hash32b(uint32_t x) {
  x *= 0x9E3779B1u;
  x ^= x >> 15;
  x *= 0x85EBCA77u;
  x ^= x >> 13;
  x *= 0xC2B2AE3Du;
  x ^= x >> 16;
  return x;
}
__device__ __forceinline__ uint64_t bloom_bits(uint32_t k) {
  const uint32_t g = hash32b(k);
  return (1ull << (g & 63)) | (1ull << ((g >> 6) & 63)) | (1ull << ((g >> 12) & 63)) | (1ull << ((g >> 18) & 63));
}
// Word of key k for a filter of 2^(32 - shift) words.
__device__ __forceinline__ uint32_t bloom_word(uint32_t k, int shift) {
  return shift >= 32 ? 0u : hash32(k) >> shift;
}

struct Bloom {
  const uint64_t* words;  // null: no filter
  int shift;
};

__device__ __forceinline__ uint64_t ld_keep_u64(const uint64_t* p, uint64_t pol) {
  uint64_t v;
  asm("ld.global.nc.L2::cache_hint.u64 %0, [%1], %2;" : "=l"(v) : "l"(p), "l"(pol));
  return v;
}

// Keys of k4 that may be in the table: all four unless there is a filter.
// The kernels are instantiated with and without a filter, so the unfiltered
// ones form no filter address at all (the word loads below are asm without
// `volatile`; a null filter behind a runtime test could still be read).
template <bool kFilter>
__device__ __forceinline__ uint32_t bloom_pass4(const Bloom& f, const int4 k4, uint64_t pol) {
  if (!kFilter) return 0xFu;
  const uint32_t k[4] = {static_cast<uint32_t>(k4.x), static_cast<uint32_t>(k4.y), static_cast<uint32_t>(k4.z),
                         static_cast<uint32_t>(k4.w)};
  uint64_t w[4];
#pragma unroll
  for (int j = 0; j < 4; ++j) w[j] = ld_keep_u64(f.words + bloom_word(k[j], f.shift), pol);
  uint32_t m = 0;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const uint64_t b = bloom_bits(k[j]);
    m |= static_cast<uint32_t>((w[j] & b) == b) << j;
  }
  return m;
}

template <bool kFilter>
__device__ __forceinline__ bool bloom_pass(const Bloom& f, int32_t k) {
  if (!kFilter) return true;
  const uint64_t b = bloom_bits(static_cast<uint32_t>(k));
  return (__ldg(f.words + bloom_word(static_cast<uint32_t>(k), f.shift)) & b) == b;
}

__global__ void bloom_build_kernel(const int32_t* __restrict__ keys, int64_t n, uint64_t* __restrict__ words,
                                   int shift) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < n; r += stride) {
    const int32_t k = keys[r];
    if (k == INT32_MIN) continue;  // never in the table
    atomicOr(reinterpret_cast<unsigned long long*>(words + bloom_word(static_cast<uint32_t>(k), shift)),
             static_cast<unsigned long long>(bloom_bits(static_cast<uint32_t>(k))));
  }
}

__global__ void fill_u64_kernel(uint64_t* p, int64_t n, uint64_t v) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) p[i] = v;
}

__global__ void hash_build_kernel(const int32_t* __restrict__ keys, int64_t n, uint64_t* __restrict__ slots,
                                  uint64_t cap, unsigned long long* range_err, unsigned long long* overflow) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < n; r += stride) {
    const int32_t k = keys[r];
    if (k == INT32_MIN) {
      atomicAdd(range_err, 1ull);
      continue;
    }
    const uint64_t mine = (static_cast<uint64_t>(static_cast<uint32_t>(k)) << 32) | static_cast<uint32_t>(r);
    uint64_t h = home_slot(static_cast<uint32_t>(k), cap);
    bool done = false;
    for (uint64_t step = 0; step < cap && !done; ++step) {
      unsigned long long* s = reinterpret_cast<unsigned long long*>(slots + h);
      const unsigned long long prev = atomicCAS(s, kEmptySlot, mine);
      if (prev == kEmptySlot) {
        done = true;
      } else if ((prev >> 32) == static_cast<uint32_t>(k)) {
        atomicMax(s, mine);  // same key in the high word: keeps the largest row
        done = true;
      } else {
        h = next_slot(h, cap);
      }
    }
    if (!done) atomicAdd(overflow, 1ull);
  }
}

// Slots [0, cap): (key, row) becomes (key, payload[row]).  The payload reads
// are random over the whole payload column; marked evict-last in L2, the
// column (4 bytes per build row) stays there while the table streams past,
// so each payload sector comes from DRAM about once.
__global__ void hash_finish_kernel(uint64_t* __restrict__ slots, int64_t cap, const int32_t* __restrict__ payload) {
  const uint64_t keep = policy_evict_last();
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < cap; i += stride) {
    const uint64_t v = slots[i];
    const bool full = v != kEmptySlot;
    const uint32_t row = full ? static_cast<uint32_t>(v) : 0u;  // a valid row whether or not the slot is full
    const int32_t pay = ld_probe_s32(payload + row, keep);
    if (full) slots[i] = (v & 0xffffffff00000000ull) | static_cast<uint32_t>(pay);
  }
}

// ---- partitioned build in L2 -------------------------------------------------
// (Tables above 2^27 slots, which the shared-memory build below does not
// take, or any table above 32 MB with OLAP_TUNE_JOIN_BUILD = 3.)
// A table larger than L2 takes one random DRAM sector per CAS.  For such
// tables the build rows are first scattered by the region of the table their
// home slot falls in (regions of kBuildRegionSlots slots, 32 MB, which L2
// holds), then inserted one region at a time, so the CAS traffic of a region
// stays in L2 and each sector of the table crosses DRAM about once each way.
// Linear probing may run past a region's end; that only costs locality.  The
// finishing pass (row -> payload) runs once over the whole table afterwards.
constexpr int64_t kBuildRegionSlots = int64_t(1) << 22;
constexpr int kBuildPartThreads = 512;

struct BuildPlan {
  int64_t n;
  int64_t per;         // rows per block of the histogram and scatter passes
  int32_t n_blocks;
  int32_t n_regions;   // P = ceil(capacity / kBuildRegionSlots)
  int32_t region_shift;
  uint64_t cap;        // table slots
};

__device__ __forceinline__ uint32_t build_region(int32_t k, const BuildPlan& bp) {
  return static_cast<uint32_t>(home_slot(static_cast<uint32_t>(k), bp.cap) >> bp.region_shift);
}

// The histogram and scatter passes run warp-uniform loops, 4 rows per lane
// (16-byte loads when the keys are aligned), and aggregate a warp's rows per
// region (match_any): one shared atomic per region present in the warp
// instead of one per row (a table has few regions, so most rows of a warp
// share theirs).
__device__ __forceinline__ void build_keys4(const int32_t* __restrict__ keys, int64_t r, int64_t e, bool vec,
                                            int32_t (&k)[4]) {
  if (vec && r + 4 <= e) {
    const int4 v = ld_stream_v4(keys + r, policy_evict_first());
    k[0] = v.x; k[1] = v.y; k[2] = v.z; k[3] = v.w;
  } else {
#pragma unroll
    for (int u = 0; u < 4; ++u) k[u] = r + u < e ? keys[r + u] : INT32_MIN;
  }
}

__global__ void __launch_bounds__(kBuildPartThreads) build_hist_kernel(BuildPlan bp, const int32_t* __restrict__ keys,
                                                                      int vec, unsigned int* __restrict__ hist,
                                                                      unsigned long long* range_err) {
  extern __shared__ unsigned int s_cnt[];
  for (int p = threadIdx.x; p < bp.n_regions; p += blockDim.x) s_cnt[p] = 0;
  __syncthreads();
  const int64_t b = static_cast<int64_t>(blockIdx.x) * bp.per;
  const int64_t e = b + bp.per < bp.n ? b + bp.per : bp.n;
  const int lane = threadIdx.x & 31;
  const int64_t step = 4 * static_cast<int64_t>(blockDim.x);
  unsigned int bad = 0;
  for (int64_t r0 = b + 4 * static_cast<int64_t>(threadIdx.x - lane); r0 < e; r0 += step) {
    const int64_t r = r0 + 4 * lane;
    int32_t k[4];
    build_keys4(keys, r, e, vec, k);
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const bool live = k[u] != INT32_MIN;
      if (r + u < e && !live) ++bad;
      const uint32_t reg = live ? build_region(k[u], bp) : 0xFFFFFFFFu;
      const unsigned int m = __match_any_sync(0xffffffffu, reg);
      if (live && lane == __ffs(m) - 1) atomicAdd(&s_cnt[reg], static_cast<unsigned int>(__popc(m)));
    }
  }
  if (bad) atomicAdd(range_err, static_cast<unsigned long long>(bad));
  __syncthreads();
  for (int p = threadIdx.x; p < bp.n_regions; p += blockDim.x)
    hist[static_cast<int64_t>(blockIdx.x) * bp.n_regions + p] = s_cnt[p];
}

// Region-major offsets: offs[b * P + p] = start of block b's run in region p;
// region_begin[p] (and [P] = all rows).  One block.
__global__ void __launch_bounds__(1024) build_scan_kernel(BuildPlan bp, const unsigned int* __restrict__ hist,
                                                          unsigned long long* __restrict__ offs,
                                                          long long* __restrict__ region_begin) {
  __shared__ long long s_tot[2048];
  __shared__ long long s_run[1024];
  const int P = bp.n_regions, B = bp.n_blocks;
  for (int p = threadIdx.x; p < P; p += blockDim.x) {
    long long t = 0;
    for (int b = 0; b < B; ++b) t += hist[static_cast<int64_t>(b) * P + p];
    s_tot[p] = t;
  }
  __syncthreads();
  // exclusive scan of the region totals (each thread a run of regions)
  const int per = (P + blockDim.x - 1) / blockDim.x;
  const int lo = threadIdx.x * per, hi = lo + per < P ? lo + per : P;
  long long mine = 0;
  for (int p = lo; p < hi; ++p) mine += s_tot[p];
  s_run[threadIdx.x] = mine;
  __syncthreads();
  for (int o = 1; o < 1024; o <<= 1) {
    const long long y = threadIdx.x >= o ? s_run[threadIdx.x - o] : 0;
    __syncthreads();
    s_run[threadIdx.x] += y;
    __syncthreads();
  }
  long long run = s_run[threadIdx.x] - mine;
  for (int p = lo; p < hi; ++p) {
    region_begin[p] = run;
    long long c = run;
    for (int b = 0; b < B; ++b) {
      offs[static_cast<int64_t>(b) * P + p] = static_cast<unsigned long long>(c);
      c += hist[static_cast<int64_t>(b) * P + p];
    }
    run += s_tot[p];
  }
  if (threadIdx.x == blockDim.x - 1) region_begin[P] = s_run[threadIdx.x];
}

// Shared memory: the block's run starts (P x u64), then its positions taken
// so far in each run (P x u32).
__global__ void __launch_bounds__(kBuildPartThreads) build_scatter_kernel(BuildPlan bp,
                                                                         const int32_t* __restrict__ keys, int vec,
                                                                         const unsigned long long* __restrict__ offs,
                                                                         uint64_t* __restrict__ tuples) {
  extern __shared__ unsigned long long s_start[];
  unsigned int* s_taken = reinterpret_cast<unsigned int*>(s_start + bp.n_regions);
  for (int p = threadIdx.x; p < bp.n_regions; p += blockDim.x) {
    s_start[p] = offs[static_cast<int64_t>(blockIdx.x) * bp.n_regions + p];
    s_taken[p] = 0;
  }
  __syncthreads();
  const int64_t b = static_cast<int64_t>(blockIdx.x) * bp.per;
  const int64_t e = b + bp.per < bp.n ? b + bp.per : bp.n;
  const int lane = threadIdx.x & 31;
  const int64_t step = 4 * static_cast<int64_t>(blockDim.x);
  for (int64_t r0 = b + 4 * static_cast<int64_t>(threadIdx.x - lane); r0 < e; r0 += step) {
    const int64_t r = r0 + 4 * lane;
    int32_t k[4];
    build_keys4(keys, r, e, vec, k);
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const bool live = k[u] != INT32_MIN;
      const uint32_t reg = live ? build_region(k[u], bp) : 0xFFFFFFFFu;
      const unsigned int m = __match_any_sync(0xffffffffu, reg);
      if (live) {
        const int leader = __ffs(m) - 1;
        unsigned int at = 0;
        if (lane == leader) at = atomicAdd(&s_taken[reg], static_cast<unsigned int>(__popc(m)));
        at = __shfl_sync(m, at, leader) + __popc(m & ((1u << lane) - 1u));
        tuples[s_start[reg] + at] = (static_cast<uint64_t>(static_cast<uint32_t>(k[u])) << 32) |
                                    static_cast<uint32_t>(r + u);
      }
    }
  }
}

// Inserts `mine` = (key << 32 | row) into the table from slot h on (linear
// probing); a key already present keeps its largest row.  False when the
// table has no free slot.
__device__ __forceinline__ bool insert_from(uint64_t* __restrict__ slots, uint64_t cap, uint64_t h,
                                            uint64_t mine) {
  const uint32_t k = static_cast<uint32_t>(mine >> 32);
  for (uint64_t step = 0; step < cap; ++step) {
    unsigned long long* s = reinterpret_cast<unsigned long long*>(slots + h);
    const unsigned long long prev = atomicCAS(s, kEmptySlot, mine);
    if (prev == kEmptySlot) return true;
    if ((prev >> 32) == k) {
      atomicMax(s, mine);  // same key in the high word: keeps the largest row
      return true;
    }
    h = next_slot(h, cap);
  }
  return false;
}

// Inserts region p's rows (tuples [region_begin[p], region_begin[p+1])): the
// region's 32 MB of slots are read from DRAM once, and every later CAS on
// them is an L2 round trip.
__global__ void build_insert_kernel(const uint64_t* __restrict__ tuples, const long long* __restrict__ region_begin,
                                    int p, uint64_t* __restrict__ slots, uint64_t cap,
                                    unsigned long long* overflow) {
  const int64_t b = region_begin[p], e = region_begin[p + 1];
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = b + static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < e; i += stride) {
    const uint64_t mine = tuples[i];
    if (!insert_from(slots, cap, home_slot(static_cast<uint32_t>(mine >> 32), cap), mine)) atomicAdd(overflow, 1ull);
  }
}

// ---- region build in shared memory ------------------------------------------
// For tables up to 2^27 slots the rows are grouped by the 16,384-slot region
// (128 KB of table) of their home slot, each tuple with its payload beside
// it, and one block builds each region in shared memory: it inserts the
// region's rows with shared-memory atomics, then writes the whole region
// (empty slots too) with the payloads already in place, so the table needs no
// separate fill or finish pass, every slot crosses DRAM once and no payload
// is read at random.  A row whose probe run would leave its region (every
// slot from its home to the region's end taken) is set aside and inserted
// afterwards into the finished table from the next region's first slot on,
// where linear probing over the whole table finds it.
constexpr int kSmemRegionSlots = 16384;
constexpr int kSmemRegionShift = 14;
constexpr int64_t kSmemRegionMaxRegions = 8192;
constexpr int kSmemRegionThreads = 1024;

// Home slot for a table of at most 2^32 - 1 slots (every table this build
// path makes): the same value as home_slot, one 32-bit multiply-high.
__device__ __forceinline__ uint32_t home32(uint32_t k, uint32_t cap32) { return __umulhi(hash32(k), cap32); }

// Row offsets of a thread's 8 rows within a tile of kSmemTileRows rows:
// 4 * tid + {0..3} and 4 * (tid + kSmemRegionThreads) + {0..3}, so the 16-byte
// loads of a warp are coalesced.  The kernels below run kSmemRegionThreads
// threads per block.
constexpr int kSmemTileRows = 8 * kSmemRegionThreads;

__device__ __forceinline__ int tile_off(int u) {
  return 4 * static_cast<int>(threadIdx.x) + (u >> 2) * 4 * kSmemRegionThreads + (u & 3);
}

// A thread's 8 values of a tile starting at row r0; rows at or past e come
// back as INT32_MIN.
__device__ __forceinline__ void tile_load8(const int32_t* __restrict__ col, int64_t r0, int64_t e, bool vec,
                                           int32_t (&x)[8]) {
  int32_t a[4], b[4];
  build_keys4(col, r0 + tile_off(0), e, vec, a);
  build_keys4(col, r0 + tile_off(4), e, vec, b);
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    x[u] = a[u];
    x[u + 4] = b[u];
  }
}

// Region counts: per block in shared memory, then one global add per region.
__global__ void __launch_bounds__(kSmemRegionThreads) smem_region_count_kernel(
    const int32_t* __restrict__ keys, int64_t n, int64_t per, uint32_t cap32, int n_regions, int vec,
    unsigned int* __restrict__ counts, unsigned long long* range_err) {
  extern __shared__ unsigned int s_rc[];
  for (int p = threadIdx.x; p < n_regions; p += blockDim.x) s_rc[p] = 0;
  __syncthreads();
  const int64_t b = static_cast<int64_t>(blockIdx.x) * per;
  const int64_t e = b + per < n ? b + per : n;
  unsigned int bad = 0;
  for (int64_t r0 = b; r0 < e; r0 += kSmemTileRows) {
    const int lim = e - r0 < kSmemTileRows ? static_cast<int>(e - r0) : kSmemTileRows;
    int32_t k[8];
    tile_load8(keys, r0, e, vec, k);
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      if (tile_off(u) >= lim) continue;
      if (k[u] == INT32_MIN) {
        ++bad;
        continue;
      }
      atomicAdd(&s_rc[home32(static_cast<uint32_t>(k[u]), cap32) >> kSmemRegionShift], 1u);
    }
  }
  if (bad) atomicAdd(range_err, static_cast<unsigned long long>(bad));
  __syncthreads();
  for (int p = threadIdx.x; p < n_regions; p += blockDim.x)
    if (s_rc[p]) atomicAdd(&counts[p], s_rc[p]);
}

// Exclusive scan of the region counts (one block): begin[p], begin[P] = all
// rows, and cursor[p] = begin[p] for the scatter.
__global__ void __launch_bounds__(1024) smem_region_scan_kernel(const unsigned int* __restrict__ counts, int n_regions,
                                                                 long long* __restrict__ begin,
                                                                 unsigned long long* __restrict__ cursor) {
  __shared__ long long s_run[1024];
  const int per = (n_regions + blockDim.x - 1) / blockDim.x;
  const int lo = threadIdx.x * per, hi = lo + per < n_regions ? lo + per : n_regions;
  long long mine = 0;
  for (int p = lo; p < hi; ++p) mine += counts[p];
  s_run[threadIdx.x] = mine;
  __syncthreads();
  for (int o = 1; o < 1024; o <<= 1) {
    const long long y = threadIdx.x >= o ? s_run[threadIdx.x - o] : 0;
    __syncthreads();
    s_run[threadIdx.x] += y;
    __syncthreads();
  }
  long long run = s_run[threadIdx.x] - mine;
  for (int p = lo; p < hi; ++p) {
    begin[p] = run;
    cursor[p] = static_cast<unsigned long long>(run);
    run += counts[p];
  }
  if (threadIdx.x == blockDim.x - 1) begin[n_regions] = s_run[threadIdx.x];
}

// Scatter of the (key << 32 | row) tuples and their payloads by region (rows
// with the key INT32_MIN are range errors and dropped).  A block takes its
// rows a tile of 8,192 at a time: counting-sorts the tile by region in shared
// memory, claims one piece of each region's output per tile from the global
// cursors, and writes each region's rows as one contiguous piece.  Because
// every tile claims afresh, a region's output fills from its start in the
// order the tiles finish, so the piece that completes a partly written
// 32-byte sector follows within microseconds and L2 merges the two: DRAM
// sees whole sectors although a tile holds only about four rows per region.
// (One claim per block and region made at the start, filled tile by tile,
// left each sector partly written for the whole pass, and DRAM took twice
// the bytes as read-modify-writes; two passes, into 256 groups of regions
// and then into regions, wrote long pieces but cost a second pass; blocks of
// 512 threads, two per SM, waited longer on their claims.)  The next tile is
// prefetched into L2 while the current one is sorted and written.
__global__ void __launch_bounds__(kSmemRegionThreads, 1) smem_region_scatter_kernel(
    const int32_t* __restrict__ keys, const int32_t* __restrict__ payload, int64_t n, uint32_t cap32, int n_regions,
    int vec_k, int vec_p, unsigned long long* __restrict__ cursor, uint64_t* __restrict__ out_tup,
    int32_t* __restrict__ out_pay) {
  constexpr int kTile = kSmemTileRows;
  // the sorted tile (tuples, payloads, regions), then per region its tile
  // offset, its destination base and its tile count
  extern __shared__ unsigned long long s_stage[];
  int32_t* s_pay = reinterpret_cast<int32_t*>(s_stage + kTile);
  uint16_t* s_reg = reinterpret_cast<uint16_t*>(s_pay + kTile);
  unsigned int* s_off = reinterpret_cast<unsigned int*>(s_reg + kTile);
  unsigned int* s_dst = s_off + n_regions;
  unsigned int* s_cnt = s_dst + n_regions;
  __shared__ unsigned int s_wsum[33];
  const int64_t per = ((n + gridDim.x - 1) / gridDim.x + 3) & ~int64_t(3);
  const int64_t b = static_cast<int64_t>(blockIdx.x) * per;
  const int64_t e = b + per < n ? b + per : n;
  for (int p = threadIdx.x; p < n_regions; p += kSmemRegionThreads) s_cnt[p] = 0;
  const int cpt = (n_regions + kSmemRegionThreads - 1) / kSmemRegionThreads;  // regions per thread, at most 8
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  auto prefetch_tile = [&](int64_t r0) {
    if (threadIdx.x != 0 || r0 >= e) return;
    const int64_t m = e - r0 < kTile ? e - r0 : kTile;
    prefetch_l2_range(keys + r0, 4 * m);
    prefetch_l2_range(payload + r0, 4 * m);
  };
  prefetch_tile(b);
  __syncthreads();
  for (int64_t r0 = b; r0 < e; r0 += kTile) {
    const int lim = e - r0 < kTile ? static_cast<int>(e - r0) : kTile;
    int32_t k[8], v[8];
    tile_load8(keys, r0, e, vec_k, k);
    tile_load8(payload, r0, e, vec_p, v);
    prefetch_tile(r0 + kTile);
    uint32_t slot[8];  // region << 14 | rank in the tile, or ~0u for no row
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      slot[u] = ~0u;
      if (tile_off(u) < lim && k[u] != INT32_MIN) {
        const uint32_t reg = home32(static_cast<uint32_t>(k[u]), cap32) >> kSmemRegionShift;
        slot[u] = (reg << 14) | atomicAdd(&s_cnt[reg], 1u);
      }
    }
    __syncthreads();
    // exclusive scan of the tile counts over the regions, one claim per
    // non-empty region (its result is first needed after the rows are
    // placed, so the atomics' round trip overlaps the placing), and the
    // counts cleared for the next tile
    const int lo = threadIdx.x * cpt;
    unsigned int sum = 0;
    for (int j = 0; j < cpt && lo + j < n_regions; ++j) sum += s_cnt[lo + j];
    unsigned int x = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) s_wsum[warp] = x;
    __syncthreads();
    if (warp == 0) {
      const unsigned int w = s_wsum[lane];
      unsigned int z = w;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned int y = __shfl_up_sync(0xffffffffu, z, o);
        if (lane >= o) z += y;
      }
      s_wsum[lane] = z - w;
      if (lane == 31) s_wsum[32] = z;
    }
    __syncthreads();
    unsigned int run = s_wsum[warp] + x - sum;
    unsigned int claim[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int p = lo + j;
      claim[j] = 0;
      if (j < cpt && p < n_regions) {
        const unsigned int c = s_cnt[p];
        if (c) claim[j] = static_cast<unsigned int>(atomicAdd(&cursor[p], static_cast<unsigned long long>(c)));
        s_off[p] = run;
        s_cnt[p] = 0;
        run += c;
      }
    }
    __syncthreads();
    const uint32_t row0 = static_cast<uint32_t>(r0);
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      if (slot[u] == ~0u) continue;
      const unsigned int at = s_off[slot[u] >> 14] + (slot[u] & 16383u);
      s_stage[at] = (static_cast<uint64_t>(static_cast<uint32_t>(k[u])) << 32) |
                    (row0 + static_cast<uint32_t>(tile_off(u)));
      s_pay[at] = v[u];
      s_reg[at] = static_cast<uint16_t>(slot[u] >> 14);
    }
#pragma unroll
    for (int j = 0; j < 8; ++j)
      if (j < cpt && lo + j < n_regions) s_dst[lo + j] = claim[j] - s_off[lo + j];
    __syncthreads();
    const unsigned int total = s_wsum[32];
    for (unsigned int i = threadIdx.x; i < total; i += kSmemRegionThreads) {
      const unsigned int d = s_dst[s_reg[i]] + i;
      out_tup[d] = s_stage[i];
      out_pay[d] = s_pay[i];
    }
    __syncthreads();
  }
}

// One block per region: insert its rows into a shared-memory copy of the
// region (32-bit CAS on the key, 32-bit atomicMax on the row, so the last
// duplicate row wins as in the sequential build; the payload rides with the
// row), set aside the rows whose run would leave the region, then write the
// region with (key, payload) in every taken slot and the empty marker
// elsewhere.  Payloads of duplicate keys are settled by a second pass over
// the region's rows, run only when the region met a duplicate.
//
// With a filter (filter != null), the block also sets the Bloom bits of its
// rows (set-aside rows included): the filter word of a key is the top bits
// of the same hash that places it in the table, so a region's keys fall in
// one run of at most kSmemFilterWords words, kept in shared memory (low and
// high halves apart, for 32-bit atomics) and stored whole; the run's first
// and last words may be shared with the neighbouring regions and are ORed
// into the (zeroed) filter instead.
constexpr uint32_t kEmptyKey = 0x80000000u;  // INT32_MIN, the reserved empty key
constexpr int kSmemFilterWords = 2064;  // a region's run with olap_hashjoin_filter_words is at most 2050

__global__ void __launch_bounds__(kSmemRegionThreads, 1) smem_region_build_kernel(
    const uint64_t* __restrict__ tuples, const int32_t* __restrict__ pays, const long long* __restrict__ begin,
    uint64_t* __restrict__ slots, uint32_t cap32, uint64_t* __restrict__ spill, unsigned long long* __restrict__ n_spill,
    uint64_t* __restrict__ filter, int fshift) {
  extern __shared__ uint32_t s_key[];
  uint32_t* s_row = s_key + kSmemRegionSlots;
  int32_t* s_val = reinterpret_cast<int32_t*>(s_row + kSmemRegionSlots);
  uint32_t* s_flo = reinterpret_cast<uint32_t*>(s_val + kSmemRegionSlots);
  uint32_t* s_fhi = s_flo + kSmemFilterWords;
  __shared__ int s_dup;
  const uint32_t base = blockIdx.x << kSmemRegionShift;
  const uint32_t len = cap32 - base < kSmemRegionSlots ? cap32 - base : kSmemRegionSlots;
  // hashes whose home slot lies in this region: [h_lo, h_hi)
  const uint64_t h_lo = ((static_cast<uint64_t>(blockIdx.x) << (32 + kSmemRegionShift)) + cap32 - 1) / cap32;
  const uint64_t h_hi = (((static_cast<uint64_t>(blockIdx.x) + 1) << (32 + kSmemRegionShift)) + cap32 - 1) / cap32;
  const uint32_t w_lo = fshift >= 32 ? 0u : static_cast<uint32_t>(h_lo >> fshift);
  const uint32_t w_hi = fshift >= 32 ? 0u : static_cast<uint32_t>(((h_hi < (uint64_t(1) << 32) ? h_hi : (uint64_t(1) << 32)) - 1) >> fshift);
  const uint32_t n_words = filter ? w_hi - w_lo + 1 : 0;
  for (uint32_t i = threadIdx.x; i < len; i += blockDim.x) {
    s_key[i] = kEmptyKey;
    s_row[i] = 0;
  }
  for (uint32_t i = threadIdx.x; i < n_words; i += blockDim.x) {
    s_flo[i] = 0;
    s_fhi[i] = 0;
  }
  if (threadIdx.x == 0) s_dup = 0;
  const int64_t b = begin[blockIdx.x], e = begin[blockIdx.x + 1];
  __syncthreads();
  const int64_t chunk = 8 * static_cast<int64_t>(blockDim.x);
  for (int64_t t0 = b; t0 < e; t0 += chunk) {
    uint64_t tu[8];
    int32_t pv[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int64_t t = t0 + threadIdx.x + u * static_cast<int64_t>(blockDim.x);
      tu[u] = t < e ? tuples[t] : 0ull;
      pv[u] = t < e ? pays[t] : 0;
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      if (t0 + threadIdx.x + u * static_cast<int64_t>(blockDim.x) >= e) continue;
      const uint32_t k = static_cast<uint32_t>(tu[u] >> 32), row = static_cast<uint32_t>(tu[u]);
      const uint32_t h = hash32(k);
      if (filter) {
        const uint32_t w = (fshift >= 32 ? 0u : h >> fshift) - w_lo;
        const uint64_t bits = bloom_bits(k);
        if (static_cast<uint32_t>(bits)) atomicOr(&s_flo[w], static_cast<uint32_t>(bits));
        if (bits >> 32) atomicOr(&s_fhi[w], static_cast<uint32_t>(bits >> 32));
      }
      bool done = false;
      for (uint32_t j = __umulhi(h, cap32) - base; j < len; ++j) {
        const uint32_t prev = atomicCAS(&s_key[j], kEmptyKey, k);
        if (prev == kEmptyKey) {
          atomicMax(&s_row[j], row);
          s_val[j] = pv[u];
          done = true;
          break;
        }
        if (prev == k) {
          atomicMax(&s_row[j], row);
          s_dup = 1;
          done = true;
          break;
        }
      }
      if (!done) spill[atomicAdd(n_spill, 1ull)] = tu[u];  // the run reached the region's end
    }
  }
  __syncthreads();
  if (s_dup) {  // a key met twice: the payload of its largest row
    for (int64_t t = b + threadIdx.x; t < e; t += blockDim.x) {
      const uint64_t mine = tuples[t];
      const uint32_t k = static_cast<uint32_t>(mine >> 32), row = static_cast<uint32_t>(mine);
      for (uint32_t j = home32(k, cap32) - base; j < len; ++j) {
        if (s_key[j] != k) continue;
        if (s_row[j] == row) s_val[j] = pays[t];
        break;
      }
    }
    __syncthreads();
  }
  for (uint32_t i = threadIdx.x; i < len; i += blockDim.x) {
    const uint32_t k = s_key[i];
    slots[base + i] = k != kEmptyKey ? (static_cast<uint64_t>(k) << 32) | static_cast<uint32_t>(s_val[i]) : kEmptySlot;
  }
  for (uint32_t i = threadIdx.x; i < n_words; i += blockDim.x) {
    const uint64_t v = (static_cast<uint64_t>(s_fhi[i]) << 32) | s_flo[i];
    if (i == 0 || i == n_words - 1) {
      if (v) atomicOr(reinterpret_cast<unsigned long long*>(filter + w_lo + i), static_cast<unsigned long long>(v));
    } else {
      filter[w_lo + i] = v;
    }
  }
}

// The set-aside rows, into the finished table from the first slot after
// their region on (linear probing across regions, wrapping at the end); the
// slots they take are listed for the payload pass.  A key already there (an
// earlier set-aside copy) keeps its largest row.  One warp per row: the warp
// reads 32 consecutive slots at a time, takes the first that is empty or
// holds its key (ballot) with one CAS, and on a lost race reads on from
// there, so a row costs one or two round trips instead of one CAS per slot.
__global__ void smem_region_spill_kernel(const uint64_t* __restrict__ spill, const unsigned long long* n_spill,
                                         uint64_t* __restrict__ slots, uint64_t cap, uint64_t* __restrict__ taken,
                                         unsigned long long* __restrict__ n_taken, unsigned long long* overflow) {
  const int64_t n = static_cast<int64_t>(*n_spill);
  const int lane = threadIdx.x & 31;
  const int64_t n_warps = static_cast<int64_t>(gridDim.x) * (blockDim.x >> 5);
  for (int64_t i = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5; i < n; i += n_warps) {
    const unsigned long long mine = spill[i];
    const uint32_t k = static_cast<uint32_t>(mine >> 32);
    const uint64_t next = ((home_slot(k, cap) >> kSmemRegionShift) + 1) << kSmemRegionShift;
    uint64_t h = next >= cap ? 0 : next;  // first slot of the window
    uint64_t seen = 0;
    bool done = false;
    while (!done && seen < cap) {
      uint64_t at = h + lane;
      if (at >= cap) at -= cap;
      const uint64_t v = *reinterpret_cast<volatile const uint64_t*>(slots + at);
      const uint32_t vk = static_cast<uint32_t>(v >> 32);
      const unsigned int m = __ballot_sync(0xffffffffu, vk == kEmptyKey || vk == k);
      if (m == 0) {
        h = h + 32 >= cap ? h + 32 - cap : h + 32;
        seen += 32;
        continue;
      }
      const int f = __ffs(m) - 1;
      int ok = 0;
      if (lane == f) {
        unsigned long long* sl = reinterpret_cast<unsigned long long*>(slots + at);
        const unsigned long long prev = atomicCAS(sl, kEmptySlot, mine);
        if (prev == kEmptySlot) {
          taken[atomicAdd(n_taken, 1ull)] = at;
          ok = 1;
        } else if ((prev >> 32) == k) {
          atomicMax(sl, mine);
          ok = 1;
        }
      }
      ok = __shfl_sync(0xffffffffu, ok, f);
      if (ok) {
        done = true;
      } else {  // another key took the slot first: read on after it
        const uint64_t after = h + f + 1;
        h = after >= cap ? after - cap : after;
        seen += f + 1;
      }
    }
    if (!done && lane == 0) atomicAdd(overflow, 1ull);
  }
}

// Payloads into the slots the set-aside rows took.
__global__ void smem_region_taken_kernel(const uint64_t* __restrict__ taken, const unsigned long long* n_taken,
                                         uint64_t* __restrict__ slots, const int32_t* __restrict__ payload) {
  const int64_t n = static_cast<int64_t>(*n_taken);
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
    const uint64_t s = taken[i];
    const uint64_t v = slots[s];
    slots[s] = (v & 0xffffffff00000000ull) | static_cast<uint32_t>(payload[static_cast<uint32_t>(v)]);
  }
}

// Half a bucket (two slots) of the hash table, marked evict-last in L2: every
// probe re-reads the table at random while the probe keys stream past it once,
// so the part of the table that L2 holds should stay there.  The 64-byte
// prefetch size asks L2 to fetch only the 64 bytes around the bucket on a
// miss: 36 instead of 57 bytes of DRAM per probe (2^24 probes, 256 MB
// table), for about 5 % more time per probe.  The address is always inside
// the table (the callers' guards may be moved past this load).
__device__ __forceinline__ ulonglong2 ld_bucket_half(const uint64_t* p) {
  ulonglong2 v;
  asm("ld.global.nc.L2::cache_hint.L2::64B.v2.u64 {%0,%1}, [%2], %3;"
      : "=l"(v.x), "=l"(v.y)
      : "l"(p), "l"(policy_evict_last()));
  return v;
}

// Probe: SUM of matched payloads and the match count; optionally the matches
// (probe row, payload) compacted in probe-row order by the caller's second
// pass (see ProbeOp).
__device__ __forceinline__ bool hash_lookup_from(const uint64_t* __restrict__ slots, uint64_t cap, uint64_t h,
                                                 uint32_t uk, int32_t* payload) {
  for (uint64_t step = 0; step < cap; step += 4) {
    // the 4-slot bucket holding h (one 32-byte sector), starting at h
    const uint64_t b = h & ~3ull;
    const ulonglong2 lo = ld_bucket_half(slots + b);
    const ulonglong2 hi = ld_bucket_half(slots + b + 2);
    const uint64_t s[4] = {lo.x, lo.y, hi.x, hi.y};
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      if (j < static_cast<int>(h & 3)) continue;  // linear probing starts at h
      if (s[j] == kEmptySlot) return false;
      if ((s[j] >> 32) == uk) {
        *payload = static_cast<int32_t>(static_cast<uint32_t>(s[j]));
        return true;
      }
    }
    h = b + 4 == cap ? 0 : b + 4;
  }
  return false;
}

__device__ __forceinline__ bool hash_lookup(const uint64_t* __restrict__ slots, uint64_t cap, int32_t k,
                                            int32_t* payload) {
  return hash_lookup_from(slots, cap, home_slot(static_cast<uint32_t>(k), cap), static_cast<uint32_t>(k), payload);
}

// Four lookups with their first buckets read together (8 x 16-byte loads in
// flight) before any is resolved; a key whose run continues past its first
// bucket (rare at load <= 1/2) falls back to hash_lookup from the next one.
// Returns the 4-bit mask of matches; pay[j] holds the matched payloads.
// Only the keys in `want` are looked up (the others count as absent).
__device__ __forceinline__ uint32_t hash_lookup4(const uint64_t* __restrict__ slots, uint64_t cap, const int4 k4,
                                                 int32_t pay[4], uint32_t want = 0xFu) {
  const int32_t k[4] = {k4.x, k4.y, k4.z, k4.w};
  uint64_t h[4];
  ulonglong2 lo[4], hi[4];
  const ulonglong2 none = make_ulonglong2(kEmptySlot, kEmptySlot);
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    h[j] = home_slot(static_cast<uint32_t>(k[j]), cap);
    const uint64_t b = h[j] & ~3ull;
    const bool w = (want >> j) & 1u;
    lo[j] = w ? ld_bucket_half(slots + b) : none;
    hi[j] = w ? ld_bucket_half(slots + b + 2) : none;
  }
  uint32_t found = 0;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const uint64_t s[4] = {lo[j].x, lo[j].y, hi[j].x, hi[j].y};
    const uint32_t uk = static_cast<uint32_t>(k[j]);
    int state = ((want >> j) & 1u) ? 0 : 2;  // 0 go on, 1 found, 2 absent
    pay[j] = 0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      if (state != 0 || q < static_cast<int>(h[j] & 3)) continue;
      if (s[q] == kEmptySlot) {
        state = 2;
      } else if ((s[q] >> 32) == uk) {
        pay[j] = static_cast<int32_t>(static_cast<uint32_t>(s[q]));
        state = 1;
      }
    }
    if (state == 0) {
      int32_t p = 0;
      const uint64_t b4 = (h[j] & ~3ull) + 4;
      const uint64_t next = b4 == cap ? 0 : b4;
      // continue the run from the next bucket: a key whose home slot is
      // `next` has the same probe sequence from there on
      if (hash_lookup_from(slots, cap, next, uk, &p)) {
        pay[j] = p;
        state = 1;
      }
    }
    if (state == 1) found |= 1u << j;
  }
  return found;
}

template <bool kFilter>
__global__ void __launch_bounds__(512, 2) hash_probe_sum_kernel(const int32_t* __restrict__ keys, int64_t n,
                                                                const uint64_t* __restrict__ slots, uint64_t cap,
                                                                Bloom filter, int vec, unsigned long long* sum,
                                                                unsigned long long* matches) {
  __shared__ long long s_red[16][2];
  const uint64_t pol = policy_evict_first();
  const uint64_t keep = policy_evict_last();
  int64_t s = 0, c = 0;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  const int64_t tid = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t n4 = vec ? n >> 2 : 0;
  for (int64_t i = tid; i < n4; i += stride) {
    const int4 k = ld_stream_v4(keys + 4 * i, pol);
    int32_t p[4];
    const uint32_t f = hash_lookup4(slots, cap, k, p, bloom_pass4<kFilter>(filter, k, keep));
    s += static_cast<int64_t>(p[0]) + p[1] + static_cast<int64_t>(p[2]) + p[3];  // 0 where absent
    c += __popc(f);
  }
  for (int64_t r = 4 * n4 + tid; r < n; r += stride) {
    int32_t p = 0;
    if (bloom_pass<kFilter>(filter, keys[r]) && hash_lookup(slots, cap, keys[r], &p)) {
      s += p;
      ++c;
    }
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
      if (y) atomicAdd(matches, static_cast<unsigned long long>(y));
    }
  }
}

// Matches (probe row, payload) in probe-row order.
template <bool kFilter>
struct ProbeOp {
  static constexpr int kGroups = kCompactGroups;
  const int32_t* keys;
  const uint64_t* slots;
  uint64_t cap;
  Bloom filter;
  int32_t* out_rows;
  int32_t* out_payload;
  int32_t vec;
  int4 pay[kCompactGroups];

  __device__ __forceinline__ bool vec_ok() const { return vec != 0; }
  __device__ __forceinline__ void prefetch(int u, int64_t first) {
    pay[u] = ld_stream_v4_ordered(keys + first, policy_evict_first());  // the keys, until flags() replaces them
  }
  template <bool kFull>
  __device__ __forceinline__ uint32_t flags(int u, int64_t first, int nv) {
    int32_t k[4] = {0, 0, 0, 0};
    if (kFull) {
      k[0] = pay[u].x; k[1] = pay[u].y; k[2] = pay[u].z; k[3] = pay[u].w;
    } else if (vec && nv == 4) {
      const int4 v = ld_stream_v4(keys + first, policy_evict_first());
      k[0] = v.x; k[1] = v.y; k[2] = v.z; k[3] = v.w;
    } else {
      for (int j = 0; j < nv; ++j) k[j] = keys[first + j];
    }
    int32_t p[4] = {0, 0, 0, 0};
    uint32_t m = 0;
    if (nv == 4) {
      const int4 k4 = make_int4(k[0], k[1], k[2], k[3]);
      m = hash_lookup4(slots, cap, k4, p, bloom_pass4<kFilter>(filter, k4, policy_evict_last()));
    } else {
#pragma unroll
      for (int j = 0; j < 4; ++j)
        if (j < nv && bloom_pass<kFilter>(filter, k[j]) && hash_lookup(slots, cap, k[j], &p[j])) m |= 1u << j;
    }
    pay[u] = make_int4(p[0], p[1], p[2], p[3]);
    return m;
  }
  __device__ __forceinline__ void emit(int u, int k, int64_t item, int64_t pos) {
    out_rows[pos] = static_cast<int32_t>(item);
    out_payload[pos] = k == 0 ? pay[u].x : k == 1 ? pay[u].y : k == 2 ? pay[u].z : pay[u].w;
  }
};

// Direct-address join: build keeps the largest row per key through a 64-bit
// staging vector, then the int32 payload vector is written.
__global__ void vec_build_stage_kernel(const int32_t* __restrict__ keys, int64_t n, unsigned long long* stage,
                                       int64_t len, unsigned long long* range_err) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; r < n; r += stride) {
    const int32_t k = keys[r];
    if (k < 0 || k >= len) {
      atomicAdd(range_err, 1ull);
      continue;
    }
    atomicMax(stage + k, static_cast<unsigned long long>(r) + 1);
  }
}

__global__ void vec_build_write_kernel(const unsigned long long* __restrict__ stage, int64_t len,
                                       const int32_t* __restrict__ payload, int32_t* __restrict__ vector) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < len; i += stride) {
    const unsigned long long r = stage[i];
    if (r) vector[i] = payload[r - 1];
  }
}

__global__ void __launch_bounds__(512) vec_probe_kernel(const int32_t* __restrict__ keys, int64_t n,
                                                        const int32_t* __restrict__ vector, int64_t len,
                                                        int vec, unsigned long long* sum,
                                                        unsigned long long* range_err) {
  __shared__ long long s_red[16];
  const uint64_t pol = policy_evict_first();
  int64_t s = 0;
  unsigned int bad = 0;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  const int64_t tid = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t n4 = vec ? n >> 2 : 0;
  auto one = [&](int32_t k) {
    if (k < 0 || k >= len) {
      ++bad;
      return;
    }
    s += __ldg(vector + k);
  };
  for (int64_t i = tid; i < n4; i += stride) {
    const int4 k = ld_stream_v4(keys + 4 * i, pol);
    one(k.x);
    one(k.y);
    one(k.z);
    one(k.w);
  }
  for (int64_t r = 4 * n4 + tid; r < n; r += stride) one(keys[r]);
  s = warp_sum_i64(s);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) s_red[warp] = s;
  if (bad) atomicAdd(range_err, static_cast<unsigned long long>(bad));
  __syncthreads();
  if (warp == 0) {
    long long x = lane < static_cast<int>(blockDim.x >> 5) ? s_red[lane] : 0;
    x = warp_sum_i64(x);
    if (lane == 0 && x) atomicAdd(sum, static_cast<unsigned long long>(x));
  }
}

static bool al16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

// Matched pairs of n probe keys through the order-preserving compaction.
template <bool kFilter>
int probe_pairs(olap_ctx* ctx, Arena& ar, const uint64_t* table, uint64_t cap, const Bloom& bloom,
                const int32_t* keys, int64_t n, unsigned long long* total, int32_t* out_rows,
                int32_t* out_payload) {
  ProbeOp<kFilter> op;
  std::memset(&op, 0, sizeof(op));
  op.keys = keys;
  op.slots = table;
  op.cap = cap;
  op.filter = bloom;
  op.out_rows = out_rows;
  op.out_payload = out_payload;
  op.vec = al16(keys);
  ScanTiles st;
  const int rc = make_scan_tiles(ctx, ar, n, total, ctx->stream, &st, compact_tile_items<ProbeOp<kFilter>>());
  if (rc != OLAP_OK) return rc;
  compact_kernel<ProbeOp<kFilter>><<<compact_grid(ctx, st.n_tiles), kCompactThreads, 0, ctx->stream>>>(op, n, st);
  OLAP_CUDA_TRY(ctx, cudaGetLastError());
  return OLAP_OK;
}

static unsigned grid_for(const olap_ctx* ctx, int64_t items, int threads) {
  int64_t g = (items + threads - 1) / threads;
  const int64_t cap = static_cast<int64_t>(ctx->sm_count) * (2048 / threads);
  if (g > cap) g = cap;
  return static_cast<unsigned>(g < 1 ? 1 : g);
}

// Plan of the region passes over a table of `capacity` slots for n rows.
static BuildPlan region_plan(const olap_ctx* ctx, int64_t n, int64_t capacity, int64_t align) {
  BuildPlan bp;
  bp.n = n;
  bp.cap = static_cast<uint64_t>(capacity);
  bp.n_regions = static_cast<int32_t>((capacity + kBuildRegionSlots - 1) / kBuildRegionSlots);
  int lg_r = 0;
  while ((int64_t(1) << lg_r) < kBuildRegionSlots) ++lg_r;
  bp.region_shift = lg_r;
  bp.n_blocks = ctx->sm_count * 2;
  bp.per = ((n + bp.n_blocks - 1) / bp.n_blocks + align - 1) / align * align;
  return bp;
}

}  // namespace olap

extern "C" {

int64_t olap_hashtable_capacity(int64_t n_build) {
  if (n_build < 0) n_build = 0;
  // load <= 1/2: at 3/4 (a 179 MB table for 2^24 keys instead of 256 MB)
  // more of the table stayed in L2, but the longer probe runs cost more
  // dependent round trips (probe 5.9 ms instead of 3.3 ms over 2^28 keys)
  const int64_t cap = (2 * n_build + 7) & ~int64_t(7);
  return cap < 8 ? 8 : cap;
}

}  // extern "C"

namespace olap {
namespace {

// The table build, and with `filter` the Bloom filter of the same keys; the
// caller holds the context lock.
int hashjoin_build_locked(olap_ctx* ctx, const int32_t* keys, const int32_t* payload, int64_t n, uint64_t* table,
                          int64_t capacity, uint64_t* filter, int64_t words) {
  OLAP_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  OLAP_REQUIRE(ctx, n >= 0 && n <= UINT32_MAX - 1, "n must be in [0, 2^32-1)");
  OLAP_REQUIRE(ctx, capacity >= 8 && capacity % 8 == 0 && capacity <= (int64_t(1) << 32) && capacity > n,
               "capacity must be a multiple of 8 in (n, 2^32] (see olap_hashtable_capacity)");
  OLAP_REQUIRE(ctx, table && (olap::al16(table)), "table must be 16-byte aligned");
  OLAP_REQUIRE(ctx, n == 0 || (keys && payload), "null keys or payload");
  int fshift = 32;
  if (filter) {
    OLAP_REQUIRE(ctx, words >= 1 && words <= (int64_t(1) << 31) && (words & (words - 1)) == 0 &&
                          (reinterpret_cast<uintptr_t>(filter) & 7) == 0,
                 "filter must hold a power of two of words (see olap_hashjoin_filter_words)");
    int lg = 0;
    while ((int64_t(1) << lg) < words) ++lg;
    fshift = 32 - lg;
    OLAP_CUDA_TRY(ctx, cudaMemsetAsync(filter, 0, sizeof(uint64_t) * words, ctx->stream));
  }
  olap::Arena ar(ctx);
  unsigned long long* overflow = ar.take<unsigned long long>(1);
  if (!overflow) return olap::set_error(ctx, OLAP_ERR_CAPACITY, "scratch arena exhausted");
  OLAP_CUDA_TRY(ctx, cudaMemsetAsync(overflow, 0, sizeof(*overflow), ctx->stream));
  // Tables above 32 MB: built 128 KB region by 128 KB region in shared
  // memory (up to 2^27 slots), or 32 MB region by 32 MB region in L2
  // (OLAP_TUNE_JOIN_BUILD = 3, and above 2^27 slots); OLAP_TUNE_JOIN_BUILD = 2
  // asks for the direct build.
  const int64_t build_knob = ctx->tune[olap::TUNE_JOIN_BUILD];
  const bool big = capacity > olap::kBuildRegionSlots && n >= (int64_t(1) << 16) && build_knob != 2;
  const bool smem_regions = big && build_knob != 3 &&
                            capacity <= olap::kSmemRegionMaxRegions * olap::kSmemRegionSlots;
  const bool partitioned = big && !smem_regions;
  // the region blocks set the filter bits too when a region's keys fall in
  // at most kSmemFilterWords filter words
  const uint64_t region_hashes = ((uint64_t(1) << (32 + olap::kSmemRegionShift)) + capacity - 1) / capacity;
  const bool fused_filter = filter && smem_regions && (region_hashes >> fshift) + 2 <= olap::kSmemFilterWords;
  if (n && smem_regions) {
    const int P = static_cast<int>((capacity + olap::kSmemRegionSlots - 1) / olap::kSmemRegionSlots);
    const int nb = ctx->sm_count;
    const int64_t per = ((n + nb - 1) / nb + 3) & ~int64_t(3);
    const int vec_k = olap::al16(keys), vec_p = olap::al16(payload);
    const uint64_t cap = static_cast<uint64_t>(capacity);
    const uint32_t cap32 = static_cast<uint32_t>(capacity);  // at most 2^27 here
    // counts[P] | n_spill | n_taken (zeroed together), begin[P+1], cursor[P], region-ordered tuples[n] (then
    // the taken slots) and payloads[n], set-aside rows[n]
    auto up = [](size_t x) { return (x + 255) & ~size_t(255); };
    const size_t nn = static_cast<size_t>(n);
    const size_t cnt_bytes = up(sizeof(unsigned int) * P + 2 * sizeof(unsigned long long));
    const size_t begin_off = cnt_bytes;
    const size_t cur_off = up(begin_off + sizeof(long long) * (P + 1));
    const size_t tup_off = up(cur_off + sizeof(unsigned long long) * P);
    const size_t pay_off = up(tup_off + sizeof(uint64_t) * nn);
    const size_t spill_off = up(pay_off + sizeof(int32_t) * nn);
    char* mem = olap::big_scratch(ctx, spill_off + sizeof(uint64_t) * nn);
    if (!mem) return olap::set_error(ctx, OLAP_ERR_NOMEM, "device memory for the build regions");
    auto* counts = reinterpret_cast<unsigned int*>(mem);
    auto* n_spill = reinterpret_cast<unsigned long long*>(mem + ((sizeof(unsigned int) * P + 7) & ~size_t(7)));
    auto* n_taken = n_spill + 1;
    auto* begin = reinterpret_cast<long long*>(mem + begin_off);
    auto* cursor = reinterpret_cast<unsigned long long*>(mem + cur_off);
    auto* tuples = reinterpret_cast<uint64_t*>(mem + tup_off);
    auto* pays = reinterpret_cast<int32_t*>(mem + pay_off);
    auto* spill = reinterpret_cast<uint64_t*>(mem + spill_off);
    uint64_t* taken = tuples;  // free once the region build has read it
    const int rsm = static_cast<int>(3 * sizeof(uint32_t) * olap::kSmemRegionSlots +
                                     2 * sizeof(uint32_t) * olap::kSmemFilterWords);
    // sorted tile (tuple, payload, region: 14 B a row), then 12 B a region
    const int ssm = static_cast<int>(14 * olap::kSmemTileRows + 12 * P);
    OLAP_CUDA_TRY(ctx, cudaMemsetAsync(mem, 0, cnt_bytes, ctx->stream));
    OLAP_CUDA_TRY(ctx, cudaFuncSetAttribute(olap::smem_region_build_kernel,
                                            cudaFuncAttributeMaxDynamicSharedMemorySize, rsm));
    OLAP_CUDA_TRY(ctx, cudaFuncSetAttribute(olap::smem_region_scatter_kernel,
                                            cudaFuncAttributeMaxDynamicSharedMemorySize, ssm));
    olap::smem_region_count_kernel<<<nb, olap::kSmemRegionThreads, sizeof(unsigned int) * P, ctx->stream>>>(
        keys, n, per, cap32, P, vec_k, counts, &ctx->counters->range_errors);
    olap::smem_region_scan_kernel<<<1, 1024, 0, ctx->stream>>>(counts, P, begin, cursor);
    olap::smem_region_scatter_kernel<<<nb, olap::kSmemRegionThreads, ssm, ctx->stream>>>(
        keys, payload, n, cap32, P, vec_k, vec_p, cursor, tuples, pays);
    olap::smem_region_build_kernel<<<P, olap::kSmemRegionThreads, rsm, ctx->stream>>>(
        tuples, pays, begin, table, cap32, spill, n_spill, fused_filter ? filter : nullptr, fshift);
    const unsigned sg = static_cast<unsigned>(ctx->sm_count) * 4;
    olap::smem_region_spill_kernel<<<sg, 256, 0, ctx->stream>>>(spill, n_spill, table, cap, taken, n_taken,
                                                                overflow);
    olap::smem_region_taken_kernel<<<sg, 256, 0, ctx->stream>>>(taken, n_taken, table, payload);
  } else if (n && partitioned) {
    olap::fill_u64_kernel<<<olap::grid_for(ctx, capacity, 256), 256, 0, ctx->stream>>>(table, capacity,
                                                                                       olap::kEmptySlot);
    const olap::BuildPlan bp = olap::region_plan(ctx, n, capacity, 4);
    const int vec = olap::al16(keys);
    OLAP_REQUIRE(ctx, bp.n_regions <= 2048, "hash table capacity above 2^33 slots");  // never: cap <= 2^32
    const size_t hist_bytes = sizeof(unsigned int) * static_cast<size_t>(bp.n_blocks) * bp.n_regions;
    const size_t offs_bytes = sizeof(unsigned long long) * static_cast<size_t>(bp.n_blocks) * bp.n_regions;
    const size_t begin_bytes = sizeof(long long) * (bp.n_regions + 1);
    const size_t tup_off = (hist_bytes + 8 + offs_bytes + begin_bytes + 255) & ~size_t(255);
    char* mem = olap::big_scratch(ctx, tup_off + sizeof(uint64_t) * static_cast<size_t>(n));
    if (!mem) return olap::set_error(ctx, OLAP_ERR_NOMEM, "device memory for the build partitions");
    auto* hist = reinterpret_cast<unsigned int*>(mem);
    auto* offs = reinterpret_cast<unsigned long long*>(mem + ((hist_bytes + 7) & ~size_t(7)));
    auto* rbegin = reinterpret_cast<long long*>(reinterpret_cast<char*>(offs) + offs_bytes);
    auto* tuples = reinterpret_cast<uint64_t*>(mem + tup_off);
    const size_t hsm = sizeof(unsigned int) * bp.n_regions;
    const size_t csm = (sizeof(unsigned long long) + sizeof(unsigned int)) * bp.n_regions;
    olap::build_hist_kernel<<<bp.n_blocks, olap::kBuildPartThreads, hsm, ctx->stream>>>(
        bp, keys, vec, hist, &ctx->counters->range_errors);
    olap::build_scan_kernel<<<1, 1024, 0, ctx->stream>>>(bp, hist, offs, rbegin);
    olap::build_scatter_kernel<<<bp.n_blocks, olap::kBuildPartThreads, csm, ctx->stream>>>(bp, keys, vec, offs,
                                                                                          tuples);
    const unsigned ig = static_cast<unsigned>(ctx->sm_count) * 8;
    for (int p = 0; p < bp.n_regions; ++p)
      olap::build_insert_kernel<<<ig, 256, 0, ctx->stream>>>(tuples, rbegin, p, table, bp.cap, overflow);
    olap::hash_finish_kernel<<<olap::grid_for(ctx, capacity, 256), 256, 0, ctx->stream>>>(table, capacity, payload);
  } else {
    olap::fill_u64_kernel<<<olap::grid_for(ctx, capacity, 256), 256, 0, ctx->stream>>>(table, capacity,
                                                                                       olap::kEmptySlot);
  }
  if (n && !smem_regions && !partitioned) {
    olap::hash_build_kernel<<<olap::grid_for(ctx, n, 256), 256, 0, ctx->stream>>>(
        keys, n, table, static_cast<uint64_t>(capacity), &ctx->counters->range_errors, overflow);
    olap::hash_finish_kernel<<<olap::grid_for(ctx, capacity, 256), 256, 0, ctx->stream>>>(table, capacity, payload);
  }
  if (filter && !fused_filter && n)
    olap::bloom_build_kernel<<<olap::grid_for(ctx, n, 256), 256, 0, ctx->stream>>>(keys, n, filter, fshift);
  OLAP_CUDA_TRY(ctx, cudaGetLastError());
  unsigned long long ov = 0;
  OLAP_CUDA_TRY(ctx, cudaMemcpyAsync(&ov, overflow, sizeof(ov), cudaMemcpyDeviceToHost, ctx->stream));
  OLAP_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  if (ov) return olap::set_error(ctx, OLAP_ERR_CAPACITY, "hash table full");
  return OLAP_OK;
}

}  // namespace
}  // namespace olap

extern "C" {

int olap_hashjoin_build(olap_ctx* ctx, const int32_t* keys, const int32_t* payload, int64_t n,
                        uint64_t* table, int64_t capacity) {
  if (!ctx) return OLAP_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  return olap::hashjoin_build_locked(ctx, keys, payload, n, table, capacity, nullptr, 0);
}

int olap_hashjoin_build_filtered(olap_ctx* ctx, const int32_t* keys, const int32_t* payload, int64_t n,
                                 uint64_t* table, int64_t capacity, uint64_t* filter, int64_t words) {
  if (!ctx) return OLAP_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  OLAP_REQUIRE(ctx, filter, "null filter (olap_hashjoin_build builds the table alone)");
  return olap::hashjoin_build_locked(ctx, keys, payload, n, table, capacity, filter, words);
}

int64_t olap_hashjoin_filter_words(int64_t n_build) {
  int64_t w = 1;
  while (w < n_build / 8 && w < (int64_t(1) << 31)) w <<= 1;
  return w;
}

int olap_hashjoin_build_filter(olap_ctx* ctx, const int32_t* keys, int64_t n, uint64_t* filter, int64_t words) {
  if (!ctx) return OLAP_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  OLAP_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  OLAP_REQUIRE(ctx, n >= 0 && (n == 0 || keys), "null keys");
  OLAP_REQUIRE(ctx, filter && words >= 1 && words <= (int64_t(1) << 31) && (words & (words - 1)) == 0,
               "filter must hold a power of two of words (see olap_hashjoin_filter_words)");
  int lg = 0;
  while ((int64_t(1) << lg) < words) ++lg;
  OLAP_CUDA_TRY(ctx, cudaMemsetAsync(filter, 0, sizeof(uint64_t) * words, ctx->stream));
  if (n)
    olap::bloom_build_kernel<<<olap::grid_for(ctx, n, 256), 256, 0, ctx->stream>>>(keys, n, filter, 32 - lg);
  OLAP_CUDA_TRY(ctx, cudaGetLastError());
  return OLAP_OK;
}

int olap_hashjoin_probe(olap_ctx* ctx, const uint64_t* table, int64_t capacity, const int32_t* keys,
                        int64_t n, int64_t* d_sum, int64_t* d_matches, int32_t* out_rows,
                        int32_t* out_payload) {
  return olap_hashjoin_probe_filtered(ctx, table, capacity, nullptr, 0, keys, n, d_sum, d_matches, out_rows,
                                      out_payload);
}

int olap_hashjoin_probe_filtered(olap_ctx* ctx, const uint64_t* table, int64_t capacity, const uint64_t* filter,
                                 int64_t words, const int32_t* keys, int64_t n, int64_t* d_sum,
                                 int64_t* d_matches, int32_t* out_rows, int32_t* out_payload) {
  if (!ctx) return OLAP_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  OLAP_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  OLAP_REQUIRE(ctx, n >= 0 && n <= INT32_MAX, "n must be in [0, 2^31)");
  OLAP_REQUIRE(ctx, capacity >= 8 && capacity % 8 == 0 && capacity <= (int64_t(1) << 32) && table, "bad table");
  OLAP_REQUIRE(ctx, n == 0 || keys, "null keys");
  OLAP_REQUIRE(ctx, d_sum || (out_rows && out_payload), "nothing to compute");
  OLAP_REQUIRE(ctx, !filter || (words >= 1 && words <= (int64_t(1) << 31) && (words & (words - 1)) == 0),
               "filter must hold a power of two of words");
  olap::Bloom bloom;
  bloom.words = filter;
  bloom.shift = 32;
  if (filter) {
    int lg = 0;
    while ((int64_t(1) << lg) < words) ++lg;
    bloom.shift = 32 - lg;
  }
  olap::Arena ar(ctx);
  const uint64_t cap = static_cast<uint64_t>(capacity);
  if (d_sum) {
    unsigned long long* m = d_matches ? reinterpret_cast<unsigned long long*>(d_matches)
                                      : ar.take<unsigned long long>(1);
    if (!m) return olap::set_error(ctx, OLAP_ERR_CAPACITY, "scratch arena exhausted");
    OLAP_CUDA_TRY(ctx, cudaMemsetAsync(d_sum, 0, sizeof(int64_t), ctx->stream));
    OLAP_CUDA_TRY(ctx, cudaMemsetAsync(m, 0, sizeof(int64_t), ctx->stream));
    auto* ds = reinterpret_cast<unsigned long long*>(d_sum);
    if (n) {
      const dim3 grid(olap::grid_for(ctx, (n + 3) / 4, 512));
      if (filter)
        olap::hash_probe_sum_kernel<true><<<grid, 512, 0, ctx->stream>>>(keys, n, table, cap, bloom,
                                                                        olap::al16(keys), ds, m);
      else
        olap::hash_probe_sum_kernel<false><<<grid, 512, 0, ctx->stream>>>(keys, n, table, cap, bloom,
                                                                         olap::al16(keys), ds, m);
    }
    OLAP_CUDA_TRY(ctx, cudaGetLastError());
  }
  if (out_rows && out_payload) {
    unsigned long long* total = (!d_sum && d_matches) ? reinterpret_cast<unsigned long long*>(d_matches)
                                                      : ar.take<unsigned long long>(1);
    if (!total) return olap::set_error(ctx, OLAP_ERR_CAPACITY, "scratch arena exhausted");
    const int rc = filter ? olap::probe_pairs<true>(ctx, ar, table, cap, bloom, keys, n, total, out_rows, out_payload)
                          : olap::probe_pairs<false>(ctx, ar, table, cap, bloom, keys, n, total, out_rows,
                                                     out_payload);
    if (rc != OLAP_OK) return rc;
  }
  return OLAP_OK;
}

int olap_vecjoin_build(olap_ctx* ctx, const int32_t* keys, const int32_t* payload, int64_t n,
                       int32_t* vector, int64_t vector_len) {
  if (!ctx) return OLAP_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  OLAP_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  OLAP_REQUIRE(ctx, n >= 0 && vector_len >= 1 && vector, "bad sizes or null vector");
  OLAP_REQUIRE(ctx, n == 0 || (keys && payload), "null keys or payload");
  if (n == 0) return OLAP_OK;
  // 64-bit staging (row + 1 per key) from the stream-ordered pool.
  unsigned long long* stage = nullptr;
  OLAP_CUDA_TRY(ctx, cudaMallocAsync(reinterpret_cast<void**>(&stage), sizeof(unsigned long long) * vector_len,
                                     ctx->stream));
  OLAP_CUDA_TRY(ctx, cudaMemsetAsync(stage, 0, sizeof(unsigned long long) * vector_len, ctx->stream));
  olap::vec_build_stage_kernel<<<olap::grid_for(ctx, n, 256), 256, 0, ctx->stream>>>(
      keys, n, stage, vector_len, &ctx->counters->range_errors);
  olap::vec_build_write_kernel<<<olap::grid_for(ctx, vector_len, 256), 256, 0, ctx->stream>>>(
      stage, vector_len, payload, vector);
  cudaError_t e = cudaGetLastError();
  cudaFreeAsync(stage, ctx->stream);
  if (e != cudaSuccess) return olap::check_cuda(ctx, e, "vecjoin build");
  return OLAP_OK;
}

int olap_vecjoin_probe(olap_ctx* ctx, const int32_t* keys, int64_t n, const int32_t* vector,
                       int64_t vector_len, int64_t* d_sum) {
  if (!ctx) return OLAP_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  OLAP_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  OLAP_REQUIRE(ctx, n >= 0 && vector_len >= 1 && vector && d_sum, "bad arguments");
  OLAP_REQUIRE(ctx, n == 0 || keys, "null keys");
  OLAP_CUDA_TRY(ctx, cudaMemsetAsync(d_sum, 0, sizeof(int64_t), ctx->stream));
  if (n == 0) return OLAP_OK;
  olap::vec_probe_kernel<<<olap::grid_for(ctx, (n + 3) / 4, 512), 512, 0, ctx->stream>>>(
      keys, n, vector, vector_len, olap::al16(keys), reinterpret_cast<unsigned long long*>(d_sum),
      &ctx->counters->range_errors);
  OLAP_CUDA_TRY(ctx, cudaGetLastError());
  return OLAP_OK;
}

}  // extern "C"
