/*
 * olap_capi.h — C-ABI of the B200 (sm_100a) OLAP-core library
 * (libolapcore_b200.so).
 *
 * The reference (panjd123/memory_database) exposes its operators as free C++
 * functions with raw column pointers, C++ linkage and overloaded names.  This
 * header exposes the same computations with distinct C names, plain pointers
 * and sizes, and an int status instead of exit().  Each entry point names the
 * reference function it replaces (path:line inside the reference project).
 *
 * Conventions
 *  - Every call takes an olap_ctx (device, stream, scratch arena).  Calls with
 *    device pointers are stream-ordered on the context's stream and return
 *    once the work is enqueued, unless documented as synchronous.
 *  - Entry points whose name ends in _host take host pointers and are
 *    synchronous; they stream the columns through the GPU themselves.
 *  - Sums are int64 (the reference accumulates uint32 and returns int; the
 *    int64 result equals the reference's modulo 2^32).
 *  - Status: OLAP_OK (0) or a negative OLAP_ERR_* code; olap_ctx_last_error()
 *    returns the message of the last failure on a context.
 *  - There is no CPU fallback: without a usable CUDA device every compute call
 *    fails with OLAP_ERR_NO_DEVICE.
 */
#ifndef OLAP_CAPI_H
#define OLAP_CAPI_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define OLAP_API __attribute__((visibility("default")))
#else
#define OLAP_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* Sentinels and sizes shared with the reference (include/metadata.h). */
#define OLAP_DIM_NULL 127      /* metadata.h:69  DIM_NULL = INT8_MAX            */
#define OLAP_GROUP_NULL 32767  /* metadata.h:70  GROUP_NULL = INT16_MAX         */
#define OLAP_VECTOR_SIZE 1024  /* metadata.h:68  size_v (vector-wise chunk)     */
#define OLAP_MAX_DIMS 4        /* customer, supplier, part, date (metadata.h:288) */

/* Status codes. */
#define OLAP_OK 0
#define OLAP_ERR_INVALID (-1)     /* bad argument                                  */
#define OLAP_ERR_CUDA (-2)        /* CUDA runtime error                            */
#define OLAP_ERR_NO_DEVICE (-3)   /* no usable CUDA device                         */
#define OLAP_ERR_NOMEM (-4)       /* device or pinned allocation failed            */
#define OLAP_ERR_RANGE (-5)       /* rows dropped: fk or group id out of range     */
#define OLAP_ERR_CAPACITY (-6)    /* scratch arena or table capacity exceeded      */
#define OLAP_ERR_TIMEOUT (-7)     /* a bounded device wait expired                 */
#define OLAP_ERR_UNSUPPORTED (-8) /* shape not supported by this library           */

/* Aggregate expressions of the star-join (per surviving fact row). */
#define OLAP_AGG_M1_PLUS_M2 0  /* M1 + M2: the reference's SUM (cpp:360, :428) */
#define OLAP_AGG_M1 1
#define OLAP_AGG_M2 2
#define OLAP_AGG_M1_TIMES_M2 3 /* 64-bit product                               */
#define OLAP_AGG_COUNT 4

/* Tuning knobs (olap_ctx_set_tuning); 0 restores the automatic choice. */
#define OLAP_TUNE_BLOCK_THREADS 0   /* threads per block of the scan kernels     */
#define OLAP_TUNE_BLOCKS_PER_SM 1   /* resident blocks per SM (persistent grid)  */
#define OLAP_TUNE_SMEM_DIM_BYTES 2  /* bytes of dimension vectors staged in smem */
#define OLAP_TUNE_SMEM_ACC_BYTES 3  /* bytes of group accumulators kept in smem  */
#define OLAP_TUNE_HOST_CHUNK_ROWS 4 /* rows per H2D chunk of the _host calls     */
#define OLAP_TUNE_UNROLL 5          /* scan mode: 1 plain, 2 pipelined x512, 3 pipelined x256 */
#define OLAP_TUNE_PROBE_BITS 6      /* global pass bitmaps for unstaged dims: 1 on, 2 off (default) */
#define OLAP_TUNE_SMEM_BITS_BYTES 7 /* bytes of pass bitmaps staged in smem (default 0)          */
#define OLAP_TUNE_GROUP_COMBINE 8   /* hash group-by warp combining of equal keys: 1 on, 2 off (default) */
#define OLAP_TUNE_GROUP_PLAN 9      /* hash group-by: 1 per-block tables (capacity <= 8192), rows'
                                       updates batched, 2 partitioned, 3 per-block tables, one row's
                                       update after another */
#define OLAP_TUNE_ASYNC_LOADS 10    /* star-join: 2 prefetches fact columns by bulk async copies (TMA), 1 off */
#define OLAP_TUNE_COMPACT 11        /* star-join: 2 compacts survivors per warp before global probes, 1 off */
#define OLAP_TUNE_SMEM_NIB_BYTES 12 /* bytes of 4-bit code vectors staged in smem (default 0)        */
#define OLAP_TUNE_HOST_INPLACE 13   /* _host star-join over pinned columns: 1 reads them in place
                                       (late materialisation over PCIe) when the filters promise to
                                       read at most 85 % of the bytes (default), 2 chunked copies,
                                       3 in place always */
#define OLAP_TUNE_MERGE_PROBES 14   /* star-join: 1 probes consecutive L2 int8 dimensions together, 2 off */
#define OLAP_TUNE_PROBE_ORDER 15    /* star-join: 1 probes the dimensions staged as int8 last, 2 first */
#define OLAP_TUNE_JOIN_BUILD 16     /* hash join build of tables above 32 MB: 1 (default) 128 KB regions
                                       built in shared memory up to 2^27 slots, 32 MB regions in L2
                                       above; 2 direct (one random DRAM sector per insert); 3 32 MB
                                       regions in L2 at every size */
#define OLAP_TUNE_KNOBS 17          /* knobs olap_ctx_set_tuning accepts (the autotuner sets 0..15) */

typedef struct olap_ctx olap_ctx;

/* ---- context ---------------------------------------------------------------
 * A context binds one device, one stream (its own unless set), a device
 * scratch arena (scratch_bytes, 0 = 64 MiB) and a pinned host staging buffer
 * for the _host entry points.  Calls on one context are serialised by a
 * mutex; use one context per host thread for concurrent submission. */
OLAP_API int olap_ctx_create(int device, size_t scratch_bytes, olap_ctx** out);
OLAP_API int olap_ctx_destroy(olap_ctx* ctx);
/* Run later calls on cuda_stream (a cudaStream_t); NULL is CUDA's legacy
 * default stream.  The context's own stream is released on the first call. */
OLAP_API int olap_ctx_set_stream(olap_ctx* ctx, void* cuda_stream);
OLAP_API void* olap_ctx_get_stream(olap_ctx* ctx);
/* Waits for the context stream; OLAP_ERR_TIMEOUT when a bounded device wait
 * of an earlier call gave up (olap_ctx_take_range_errors reports it too). */
OLAP_API int olap_ctx_synchronize(olap_ctx* ctx);
OLAP_API int olap_ctx_set_tuning(olap_ctx* ctx, int knob, int64_t value);
/* Synchronises, returns and clears the count of rows that kernels dropped
 * because an fk or a group id was out of range. */
OLAP_API int olap_ctx_take_range_errors(olap_ctx* ctx, int64_t* count);
/* Synchronises, returns and clears the bytes that _host calls moved from
 * host memory to the device since the last take: the copied chunks and
 * dimension vectors, and for in-place reads (OLAP_TUNE_HOST_INPLACE) every
 * 32-byte sector of host memory that a kernel requested. */
OLAP_API int olap_ctx_take_host_bytes(olap_ctx* ctx, int64_t* bytes);
OLAP_API const char* olap_ctx_last_error(const olap_ctx* ctx);
OLAP_API const char* olap_status_string(int status);
/* Number of CUDA devices (0 when none; never fails). */
OLAP_API int olap_device_count(void);
/* Library build identification ("sm_100a ..."). */
OLAP_API const char* olap_build_info(void);

/* ---- star-join with multidimensional group-by SUM (the hot path) ---------
 *
 * Replaces the fused row-wise / vector-wise OLAP core:
 *   OLAPcore_rowwise  code/OLAPcore/test_multi_compute_operator.cpp:973-1037
 *   OLAPcore_vwm_dv   code/OLAPcore/test_multi_compute_operator.cpp:1052-1126
 *   OLAPcore_vwm_sv   code/OLAPcore/test_multi_compute_operator.cpp:1258-1327
 * All three compute, for every fact row r in [row_begin, row_end):
 *   g = sum_j dimvec[j][fk[j][r]] * factor[j]   (dropped if any code is DIM_NULL)
 *   group_sums[a][g] += agg_a(M1[r], M2[r])
 * with j over the dimensions in probe order (dimvec[j] is the reference's
 * dimvec_array[orders[j]]).  Semantics follow OLAPcore_vwm_sv_thread
 * (cpp:509-568): measures are read at the row's own position.  Where the
 * reference reads out of bounds, the library drops the row instead: a row
 * with an fk outside [0, dimvec_len[j]) is never accumulated, and it counts
 * as a range error unless one of its in-range keys meets DIM_NULL (a row
 * that a filter drops anyway is not an error); a surviving row whose g is
 * outside [0, group_nums) is dropped and counted too.  The count does not
 * depend on the order the dimensions are probed in, so every entry point
 * below (device, host in place or copied, reference layout, no-allocation)
 * reports the same count for the same rows. */
typedef struct olap_starjoin_query {
  int32_t dimvec_nums;                    /* participating dimensions, 0..4   */
  int32_t n_aggs;                         /* aggregates per group, 1..2       */
  int32_t agg[2];                         /* OLAP_AGG_*                       */
  const int8_t* dimvec[OLAP_MAX_DIMS];    /* int8 group code or DIM_NULL      */
  int64_t dimvec_len[OLAP_MAX_DIMS];      /* readable entries of dimvec[j]    */
  const int32_t* fk[OLAP_MAX_DIMS];       /* foreign-key column of dim j      */
  int32_t factor[OLAP_MAX_DIMS];          /* group-id weight of dim j         */
  const int32_t* m1;                      /* measure columns (unused: NULL)   */
  const int32_t* m2;
  int64_t row_begin;                      /* fact range [row_begin, row_end)  */
  int64_t row_end;
  int64_t group_nums;                     /* groups: ids in [0, group_nums)   */
} olap_starjoin_query;

/* Device pointers; asynchronous on the context stream.  group_sums
 * ([n_aggs][group_nums], row-major) and totals ([n_aggs]) are overwritten;
 * either may be NULL when not wanted. */
OLAP_API int olap_starjoin_groupsum(olap_ctx* ctx, const olap_starjoin_query* q,
                           int64_t* group_sums, int64_t* totals);
/* Kernels one olap_starjoin_groupsum call of this query launches with the
 * context's current knobs (the star-join, one prepass per dimension staged
 * as a pass bitmap or as 4-bit codes, and after the 16-byte-aligned kernel
 * its range pass, which counts the rows with keys out of range when that
 * kernel met one and returns at once otherwise); nothing is launched. */
OLAP_API int olap_starjoin_launch_count(olap_ctx* ctx, const olap_starjoin_query* q, int want_groups,
                                        int* kernels);

/* Host pointers; synchronous.  The fact columns are streamed through the GPU
 * in pinned chunks with copies overlapped with the scan.  When every column
 * is in pinned (device-mapped) host memory at one 16-byte phase and the
 * dimensions' pass fractions promise to read at most 85 % of the columns'
 * bytes, one kernel reads the columns in place instead (OLAP_TUNE_HOST_INPLACE
 * 2 forces the copies, 3 the in-place read): the foreign keys of the
 * dimension that drops the most rows first, each later column only for the
 * rows still alive (late materialisation over PCIe); sums and dropped-row
 * count are the same either way.  A dimvec_len[j] of
 * 0 means "unknown": the library then copies dimvec[j][0 .. max fk] (the
 * bytes the reference itself would read).  Returns OLAP_ERR_RANGE (results
 * still written) when rows were dropped. */
OLAP_API int olap_starjoin_groupsum_host(olap_ctx* ctx, const olap_starjoin_query* q,
                                int64_t* group_sums, int64_t* totals);

/* Autotuner of the launch plan (no counterpart in the reference, whose
 * thread counts are fixed by the caller): times candidate plans on rows
 * [row_begin, row_begin + sample_rows) of q (device pointers; 0 = 64Mi rows),
 * sets the fastest candidate's OLAP_TUNE_* knobs on the context and returns
 * them in knobs_out[16] (may be NULL) and its time in *best_ms (may be NULL).
 * Synchronous; the query's outputs are not written. */
OLAP_API int olap_starjoin_autotune(olap_ctx* ctx, const olap_starjoin_query* q,
                                    int64_t sample_rows, int64_t* knobs_out, double* best_ms);

/* ---- star-join without any allocation --------------------------------------
 * No counterpart in the reference (whose CPU functions allocate per-thread
 * group vectors with new/malloc on every call).  For callers that may not
 * allocate device memory at all (a fixed device-memory budget owned by
 * someone else, a framework whose allocator must see every byte, a request
 * path where an allocation may not block or fail late): no olap_ctx is
 * needed, and no cudaMalloc, cudaFree or other device or pinned allocation is
 * made.  Scratch is a static device array of OLAP_NOALLOC_SCRATCH_BYTES that
 * every GPU loading the library holds until the process exits.
 *  - Same query, outputs and results as olap_starjoin_groupsum; device
 *    pointers; asynchronous on cuda_stream (NULL: the legacy default stream)
 *    on the current device.  range_errors (device int64, may be NULL)
 *    receives the number of rows this call dropped.
 *  - Dimension vectors totalling more than OLAP_NOALLOC_MAX_DIM_ENTRIES
 *    entries are rejected with OLAP_ERR_CAPACITY (their pass bitmaps would
 *    not fit the scratch).
 *  - All calls share the scratch, which keeps the last call's contents; each
 *    call clears what must start at zero.  Calls that overlap on the GPU race
 *    on it: order them on one stream.
 *  - The first call on a device looks up the scratch's device address and
 *    keeps it for the life of the process; make it before any stream
 *    capture.  The device must not be reset (cudaDeviceReset, or a teardown
 *    of its primary context) between calls: the kept address would then
 *    point into a context that no longer exists. */
#define OLAP_NOALLOC_SCRATCH_BYTES (1 << 20)
#define OLAP_NOALLOC_MAX_DIM_ENTRIES 8000000
OLAP_API int olap_starjoin_groupsum_noalloc(const olap_starjoin_query* q, int64_t* group_sums,
                                            int64_t* totals, int64_t* range_errors,
                                            void* cuda_stream);

/* Reference-layout entry point, device pointers, synchronous.
 * dimvec_array / fk_array are host arrays of 4 device pointers indexed by
 * table (0 customer, 1 supplier, 2 part, 3 date); orders[0..dimvec_nums)
 * names the tables in probe order and factor[j] belongs to orders[j], exactly
 * as the reference's main builds them (cpp:1964-1987).  dimvec_len may be
 * NULL, as the reference's signature has no lengths: each dimension vector
 * is then taken to reach to the end of the device allocation that holds it
 * (a key past that is dropped and counted, never read; a key inside the
 * allocation but past the caller's vector reads the bytes that follow it, as
 * the reference would), and a vector outside any device allocation is
 * refused with OLAP_ERR_INVALID.  *count receives the grand total of M1+M2
 * over all groups (the reference's return value); group_vector (device,
 * [group_nums]) may be NULL.  Dropped rows are left in the context's count
 * (olap_ctx_take_range_errors). */
OLAP_API int olap_OLAPcore(olap_ctx* ctx, int8_t* const* dimvec_array, const int64_t* dimvec_len,
                  int32_t* const* fk_array, const int* orders, int dimvec_nums,
                  const int* factor, int64_t size_lineorder, int64_t group_nums,
                  const int32_t* M1, const int32_t* M2, int64_t* group_vector,
                  int64_t* count);

/* ---- column-wise OLAP core (device pointers, reference argument layout) ----
 * dimvec_array / fk_array / dimvec_len indexed by table as in olap_OLAPcore;
 * group ids are int16 as in the reference, so group_nums <= 32766. */
/* join_cwm_sv (cpp:908-958): groupID[r] = sum of code*factor over the
 * dimensions in orders, or GROUP_NULL (all dimensions fused in one pass). */
OLAP_API int olap_join_cwm_sv(olap_ctx* ctx, int8_t* const* dimvec_array, const int64_t* dimvec_len,
                              int32_t* const* fk_array, const int* orders, int dimvec_nums,
                              int16_t* groupID, const int* factor, int64_t size_lineorder);
/* agg_cwm_sv (cpp:764-827): group_vector[groupID[r]] += M1[r] + M2[r] for
 * groupID[r] != GROUP_NULL; *d_count = the total (the reference's return). */
OLAP_API int olap_agg_cwm_sv(olap_ctx* ctx, const int16_t* groupID, int64_t size_lineorder,
                             const int32_t* M1, const int32_t* M2, int64_t group_nums,
                             int64_t* group_vector, int64_t* d_count);
/* join_cwm_dv (cpp:840-894): the surviving rows as OID (int64 row) and
 * groupID lists in row order (the reference's per-thread lists concatenated);
 * *d_index = their number. */
OLAP_API int olap_join_cwm_dv(olap_ctx* ctx, int8_t* const* dimvec_array, const int64_t* dimvec_len,
                              int32_t* const* fk_array, const int* orders, int dimvec_nums,
                              int64_t* OID, int16_t* groupID, const int* factor, int64_t* d_index,
                              int64_t size_lineorder);
/* agg_cwm_dv (cpp:685-752): group_vector[groupID[k]] += M1[OID[k]] +
 * M2[OID[k]] for k < index (OID outside [0, size_lineorder) is a range
 * error); *d_count = the total. */
OLAP_API int olap_agg_cwm_dv(olap_ctx* ctx, const int64_t* OID, const int16_t* groupID, int64_t index,
                             const int32_t* M1, const int32_t* M2, int64_t size_lineorder,
                             int64_t group_nums, int64_t* group_vector, int64_t* d_count);

/* ---- star-join operator (code/starjoin/test_starjoin_option.cpp) -----------
 * dimvec / fk / dimvec_len for the four tables customer, supplier, part,
 * date (dimvec_len as in olap_starjoin_query). */
/* starjoinalgo_rowwise (:37-50): rows whose four probes are not DIM_NULL. */
OLAP_API int olap_starjoin_count(olap_ctx* ctx, int64_t size_lineorder, int8_t* const* dimvec,
                                 const int64_t* dimvec_len, int32_t* const* fk, int64_t* d_count);
/* starjoinalgo_cwm_sv (:66-121): result[r] = c<<12 + s<<8 + p<<4 + d
 * (GROUP_BITS_TABLE = 4, metadata.h:76) or GROUP_NULL; *d_count = entries
 * that are not GROUP_NULL (the reference's count, which also skips a packed
 * id equal to 32767). */
OLAP_API int olap_starjoin_cwm_sv(olap_ctx* ctx, int64_t size_lineorder, int8_t* const* dimvec,
                                  const int64_t* dimvec_len, int32_t* const* fk, int32_t* result,
                                  int64_t* d_count);
/* starjoinalgo_cwm_dv (:137-189): (position, packed group) of the surviving
 * rows in row order; *d_count = their number. */
OLAP_API int olap_starjoin_cwm_dv(olap_ctx* ctx, int64_t size_lineorder, int8_t* const* dimvec,
                                  const int64_t* dimvec_len, int32_t* const* fk, int32_t* out_pos,
                                  int32_t* out_group, int64_t* d_count);

/* Plan of the reference's main (cpp:1937-1987): dimensions with groups > 0
 * participate; orders is sorted by sort_by_rate (cpp:223-233, including its
 * comparison of sele[i] with sele[j] by position); group_nums = prod groups;
 * factor[j] = prod_{k>j} groups[orders[k]] when bitmap[orders[j]] != 0, else 1.
 * Host-only, no device needed. */
OLAP_API int olap_plan_olapcore(const double sele[4], const int bitmap[4], const int groups[4],
                       int orders[4], int factor[4], int* dimvec_nums, int64_t* group_nums);

/* ---- select, project, gather (code/select, code/project) -------------------
 * Selection vectors are int32 row ids in ascending order; bitmaps hold bit i
 * of row i at byte i/8, bit i%8 (little-endian 32-bit words), the storage
 * order of a std::vector<bool> on little-endian machines.  Counts are written
 * to device int64s (asynchronous); read them after synchronising. */
#define OLAP_CMP_LE 0 /* col <= val: every sel_lt_T_* primitive of the reference */
#define OLAP_CMP_LT 1 /* col <  val */

/* Row ids r of col (r in [0, col_len)) with cmp(col[r], val), or, when
 * in_rowids is given, the entries r = in_rowids[i] (i < n_in) that pass:
 * sel_lt_T_fsel_independent_val_{branching,non_branching}
 * (select/test_select_option.cpp:172-205, 391-423; if_sv is in_rowids).
 * out_rowids holds up to (in_rowids ? n_in : col_len) entries; *d_count
 * receives the count.  in_rowids entries outside [0, col_len) are dropped and
 * counted as range errors. */
OLAP_API int olap_select_rowids(olap_ctx* ctx, const int32_t* col, int64_t col_len, int32_t val,
                                int cmp, const int32_t* in_rowids, int64_t n_in,
                                int32_t* out_rowids, int64_t* d_count);
/* Failure path of the bounded device waits (no counterpart in the
 * reference): one look-back that waits for a tile status nothing publishes
 * gives up after spin_limit polls and the call returns OLAP_ERR_TIMEOUT; the
 * context stays usable.  For tests of the error handling. */
OLAP_API int olap_debug_wait_timeout(olap_ctx* ctx, uint32_t spin_limit);
/* Bitmap of cmp(col[r], val): sel_lt_T_bmp_independent_val_{branching,
 * non_branching} (select:206-228, 424-440); (n + 31) / 32 words written. */
OLAP_API int olap_select_bitmap(olap_ctx* ctx, const int32_t* col, int64_t n, int32_t val, int cmp,
                                uint32_t* bitmap);
/* selalgo_rowwise (select:450-467): SUM(Rd) (*d_sum) and the row count
 * (*d_count, may be NULL) over rows with Ra, Rb and Rc all <= condition.  The
 * column-wise and vector-wise drivers (select:479-901) return the same sum. */
OLAP_API int olap_selalgo(olap_ctx* ctx, int32_t condition, int64_t n, const int32_t* Ra,
                          const int32_t* Rb, const int32_t* Rc, const int32_t* Rd, int64_t* d_sum,
                          int64_t* d_count);
/* Projection of the pairs (Ra[r], Rc[r]) of the rows with Ra[r] <= condition
 * and Rc[r] <= condition, in row order: proalgo_rowwise / proalgo_cwm_em /
 * proalgo_cwm_lm_* (project/test_project_option.cpp:34-864). */
OLAP_API int olap_project_pairs(olap_ctx* ctx, int32_t condition, int64_t n, const int32_t* Ra,
                                const int32_t* Rc, int32_t* out_a, int32_t* out_c, int64_t* d_count);
/* proalgo_rowwise over a row store (project/test_project_option.cpp:34-147,
 * rows of struct row_store_min / row_store_max, include/metadata.h:251-262):
 * the pairs (Ra, Rc) of the rows r < n with Ra <= condition and Rc <=
 * condition, in row order, where Ra and Rc are the int32 fields at byte
 * offsets off_a and off_c of each row_bytes-long row (rows, row_bytes and
 * both offsets 4-byte aligned).  Device pointers; *d_count gets the count. */
OLAP_API int olap_project_pairs_rows(olap_ctx* ctx, int32_t condition, int64_t n, const void* rows,
                                     int64_t row_bytes, int64_t off_a, int64_t off_c, int32_t* out_a,
                                     int32_t* out_c, int64_t* d_count);
/* Late materialisation: outs[c][i] = cols[c][rowids[i]] for 1..8 int32
 * columns of col_len rows (a row id outside [0, col_len) gives 0 and is
 * counted as a range error). */
OLAP_API int olap_gather_i32(olap_ctx* ctx, const int32_t* rowids, int64_t k, int ncols,
                             const int32_t* const* cols, int64_t col_len, int32_t* const* outs);

/* ---- joins (code/join) -------------------------------------------------------
 * Hash table: capacity 64-bit slots (a multiple of 8 in (n, 2^32]; use
 * olap_hashtable_capacity(n), about 2n slots: load <= 1/2), 16-byte
 * aligned, caller-allocated.  A key's home slot is its hash scaled onto the
 * capacity (linear probing from there).  A duplicate build key keeps the payload of its last
 * row, as the reference's sequential build does.  Key INT32_MIN marks empty
 * slots and cannot be built (counted as a range error). */
OLAP_API int64_t olap_hashtable_capacity(int64_t n_build);
/* build(relation_t*, std::unordered_map&) (join/test_join_option.cpp:44-50);
 * synchronous; OLAP_ERR_CAPACITY if the table fills.  A table above 32 MB is
 * built region by region: up to 2^27 slots the rows are grouped by the
 * 16,384-slot (128 KB) region of their home slot (one scatter pass, each
 * tuple carrying its payload) and each region is built in shared memory and
 * written once,
 * payloads in place (a row whose probe run leaves its region is inserted
 * afterwards from the next region on, where linear probing over the whole
 * table puts it); above, by 32 MB regions inserted one at a time in L2.
 * Scratch: 20 (8 above 2^27 slots) bytes per build row from the context's
 * grow-only buffer.  OLAP_TUNE_JOIN_BUILD chooses the way (see its
 * values). */
OLAP_API int olap_hashjoin_build(olap_ctx* ctx, const int32_t* keys, const int32_t* payload,
                                 int64_t n, uint64_t* table, int64_t capacity);
/* probe(relation_t*, std::unordered_map&) (join:90-96): *d_sum = SUM of the
 * matched payloads (a missing key adds 0, as operator[] inserts 0) and
 * *d_matches the match count (may be NULL).  With out_rows/out_payload the
 * matches (probe row, payload) are also written in probe-row order (then
 * *d_matches, or the count of a NULL d_sum call, is their number). */
OLAP_API int olap_hashjoin_probe(olap_ctx* ctx, const uint64_t* table, int64_t capacity,
                                 const int32_t* keys, int64_t n, int64_t* d_sum, int64_t* d_matches,
                                 int32_t* out_rows, int32_t* out_payload);
/* Blocked Bloom filter of the build keys, kept beside the table (no
 * counterpart in the reference): `words` 64-bit words, a power of two
 * (olap_hashjoin_filter_words(n_build) gives about 8 bits per key: 16 MB for
 * 2^24 keys, which stays in L2).  A probe through the filter skips the table
 * for the keys that cannot match (all but about 2-4 % of them), so a probe
 * side whose keys often miss reads far less of the table.  Asynchronous. */
OLAP_API int64_t olap_hashjoin_filter_words(int64_t n_build);
OLAP_API int olap_hashjoin_build_filter(olap_ctx* ctx, const int32_t* keys, int64_t n, uint64_t* filter,
                                        int64_t words);
/* olap_hashjoin_build and olap_hashjoin_build_filter of the same keys in one
 * call, with the same table and filter as the two calls give.  The filter
 * word of a key is the top bits of the hash that places it in the table, so
 * on the shared-memory region build each region's block sets the filter
 * bits of its own keys and stores its run of words whole (no separate pass
 * over the keys, no global atomic per key).  Synchronous, like
 * olap_hashjoin_build. */
OLAP_API int olap_hashjoin_build_filtered(olap_ctx* ctx, const int32_t* keys, const int32_t* payload, int64_t n,
                                          uint64_t* table, int64_t capacity, uint64_t* filter, int64_t words);
/* olap_hashjoin_probe through the filter built from the same build keys
 * (filter NULL: no filter); the same results. */
OLAP_API int olap_hashjoin_probe_filtered(olap_ctx* ctx, const uint64_t* table, int64_t capacity,
                                          const uint64_t* filter, int64_t words, const int32_t* keys, int64_t n,
                                          int64_t* d_sum, int64_t* d_matches, int32_t* out_rows,
                                          int32_t* out_payload);
/* build(relation_t*, int* vector) (join:30-36): vector[key] = payload (last
 * row wins); keys outside [0, vector_len) are counted as range errors.
 * Entries not built are left as they are. */
OLAP_API int olap_vecjoin_build(olap_ctx* ctx, const int32_t* keys, const int32_t* payload, int64_t n,
                                int32_t* vector, int64_t vector_len);
/* probe(relation_t*, int* vector) (join:58-64): *d_sum = SUM vector[key]. */
OLAP_API int olap_vecjoin_probe(olap_ctx* ctx, const int32_t* keys, int64_t n, const int32_t* vector,
                                int64_t vector_len, int64_t* d_sum);

/* ---- group-by and aggregation (code/group, code/aggregation) ---------------- */
/* vector_group (group/test_group_option.cpp:44-60): group_vector[vecInx[i]-1]
 * += m1[i] + m2[i] over group_num groups (1-based ids; others are range
 * errors); optional per-group counts; *d_total = the sum of all groups (the
 * reference's return value). */
OLAP_API int olap_group_vector(olap_ctx* ctx, int64_t n, const int32_t* vecInx, const int32_t* m1,
                               const int32_t* m2, int64_t group_num, int64_t* group_vector,
                               int64_t* counts, int64_t* d_total);
OLAP_API int64_t olap_group_hash_capacity(int64_t max_groups);
/* hashtable_group (group:71-88) for any int32 keys: groups of key[i] +
 * key_offset with SUM(vals[i] + vals2[i]) (vals2 may be NULL) and COUNT,
 * written unordered to out_keys/out_sums/out_counts (out_counts may be NULL),
 * *d_groups their number.  capacity (a power of two, see
 * olap_group_hash_capacity; at most 2^27) bounds the number of distinct keys
 * (more give OLAP_ERR_CAPACITY).  Up to capacity 8192 each block aggregates
 * in a shared-memory table; above, the rows are first partitioned by key
 * hash (the context keeps a grow-only device buffer of about 8-16 bytes per
 * row, plus up to 32 MB of partial tables, for that), and a partition far
 * above the average size (skewed keys) is split over several blocks whose
 * tables are merged.  Synchronous. */
OLAP_API int olap_group_hash(olap_ctx* ctx, int64_t n, const int32_t* keys, int32_t key_offset,
                             const int32_t* vals, const int32_t* vals2, int64_t capacity,
                             int32_t* out_keys, int64_t* out_sums, int64_t* out_counts,
                             int64_t* d_groups);
/* aggalgo_* (aggregation/test_aggregation_option.cpp:28-107) in int64 fixed
 * point: *d_sum = SUM price*qty*(100 + tax_pct), i.e. 100 x SUM(price*qty*tax
 * + price*qty) with tax = tax_pct/100 (exact modulo 2^64). */
OLAP_API int olap_agg_fixed(olap_ctx* ctx, int64_t n, const int32_t* price, const int32_t* qty,
                            const int32_t* tax_pct, int64_t* d_sum);
/* The same expression in double, reduced in a fixed order (deterministic;
 * differs from a sequential CPU sum only by rounding). */
OLAP_API int olap_agg_f64(olap_ctx* ctx, int64_t n, const double* tax, const double* qty,
                          const double* price, double* d_sum);

/* ---- device buffers for host-memory callers ---------------------------------
 * No counterpart in the reference, whose operators take host arrays: the C++
 * drop-in header (olap_reference_api.hpp) moves a host caller's arrays
 * through these (allocate, copy in, run the device entry point, copy out).
 * Copies are synchronous on the context's stream. */
OLAP_API int olap_buffer_alloc(olap_ctx* ctx, size_t bytes, void** dev);
OLAP_API int olap_buffer_free(olap_ctx* ctx, void* dev);
OLAP_API int olap_copy_h2d(olap_ctx* ctx, void* dev, const void* host, size_t bytes);
OLAP_API int olap_copy_d2h(olap_ctx* ctx, void* host, const void* dev, size_t bytes);
/* Largest value of a device int32 column into *h_max (INT32_MIN when n is
 * 0); synchronous.  Sizes the arrays the reference indexes by key without
 * passing their length (dimension vectors, join vectors). */
OLAP_API int olap_max_i32(olap_ctx* ctx, const int32_t* col, int64_t n, int32_t* h_max);

/* ---- dimension-vector builder and batched multi-query star-join -------------
 * Dimension tables as attributes: per dimension row an int32 filter attribute
 * and an int32 group attribute.  A query's predicate on a table is the range
 * [lo, hi) on the filter attribute; its group code is the group attribute
 * (grouped tables) or 0.  This is how the reference's generator bakes a
 * query's dimension vector (include/gendata_util.hpp:449-542). */
/* One query's int8 dimension vector: dimvec[k] = (lo <= filter[k] < hi) ?
 * (use_group ? group[k] : 0) : DIM_NULL (a group value outside [0, 127) is a
 * range error and gives DIM_NULL). */
OLAP_API int olap_build_dimvec(olap_ctx* ctx, const int32_t* filter_attr, const int32_t* group_attr,
                               int64_t n, int32_t lo, int32_t hi, int use_group, int8_t* dimvec);

typedef struct olap_batch olap_batch;
/* One query of a batch (tables 0 customer, 1 supplier, 2 part, 3 date). */
typedef struct olap_batch_query {
  int64_t row_begin;               /* fact range [row_begin, row_end)          */
  int64_t row_end;
  int32_t lo[OLAP_MAX_DIMS];       /* filter range [lo, hi) per table          */
  int32_t hi[OLAP_MAX_DIMS];
  int32_t factor[OLAP_MAX_DIMS];   /* group weight per grouped table           */
  int32_t uses;                    /* bit t: table t participates              */
  int32_t grouped;                 /* bit t: table t contributes its group     */
  int64_t group_nums;              /* groups of this query                     */
} olap_batch_query;

/* A batch engine for up to max_queries (<= 64) queries per launch; holds the
 * packed attribute records of the dimensions and two staging slots (so one
 * batch can be prepared while the previous one runs). */
OLAP_API int olap_batch_create(olap_ctx* ctx, int max_queries, olap_batch** out);
OLAP_API int olap_batch_destroy(olap_batch* b);
/* Attributes of table `table` (n rows; group_attr may be NULL = all 0). */
OLAP_API int olap_batch_set_dimension(olap_batch* b, int table, const int32_t* filter_attr,
                                      const int32_t* group_attr, int64_t n);
/* Runs n_queries star-joins in one persistent launch over the shared fact
 * table (fk[4], m1, m2 of n_rows rows), aggregate `agg` (OLAP_AGG_*) per
 * query.  Query q's groups land in out[off_q .. off_q + group_nums_q), off_q
 * the sum of the earlier queries' group_nums; totals[q] its total.  Per query
 * the result equals olap_starjoin_groupsum over the dimension vectors of
 * olap_build_dimvec.  use_graph: record the launch as a CUDA graph and replay
 * it while the tables, fact columns and aggregate stay the same (queries,
 * their count and the output buffers may change between replays).
 * Asynchronous on the context stream. */
OLAP_API int olap_batch_run(olap_batch* b, const olap_batch_query* queries, int n_queries,
                            const int32_t* const* fk, const int32_t* m1, const int32_t* m2,
                            int64_t n_rows, int agg, int64_t* out, int64_t out_slots, int64_t* totals,
                            int use_graph);
/* Number of graphs recorded by olap_batch_run so far. */
OLAP_API int olap_batch_graph_captures(olap_batch* b, int64_t* captures);
/* Launch shape of the batched scan: threads per block (multiple of 32 in
 * [128, 1024]) and per-block shared int64 accumulators (0..24576 slots; the
 * queries with the fewest groups accumulate there, the rest in L2).  A change
 * re-records the graphs on the next run. */
OLAP_API int olap_batch_tune(olap_batch* b, int block, int smem_slots);
/* Probe order of the batched scan: 0 (the default) probes the tables one
 * after another, each only for rows that still have a live query using it;
 * 1 reads every table's query mask in one round trip, then the group
 * attributes of the tables a surviving query groups by (needs blocks of at
 * most 512 threads; with larger ones the first order runs).  The autotuner
 * tries both.  olap_batch_get_tuning reports the shape in force. */
OLAP_API int olap_batch_set_probe(olap_batch* b, int parallel_probe);
OLAP_API int olap_batch_get_tuning(olap_batch* b, int* block, int* smem_slots, int* parallel_probe);
/* Times the block sizes {256, 512, 1024} x accumulator slots {0, 2048, 4096,
 * 8192, 16384} x both probe orders on the first sample_rows rows (0 = 64 Mi)
 * of the fact table with these queries (their fact ranges scaled onto the
 * sample, so it sees the whole table's mix of live queries), keeps the
 * fastest on the handle and returns it (pointers may be NULL).
 * out/out_slots/totals as for olap_batch_run; their contents afterwards are
 * unspecified.  Synchronous. */
OLAP_API int olap_batch_autotune(olap_batch* b, const olap_batch_query* queries, int n_queries,
                                 const int32_t* const* fk, const int32_t* m1, const int32_t* m2,
                                 int64_t n_rows, int agg, int64_t* out, int64_t out_slots,
                                 int64_t* totals, int64_t sample_rows, int* best_block,
                                 int* best_slots, double* best_ms);

/* ---- TPC-H Q5-shaped join chain (code/TPCH_Q5/Q5.cpp) ---------------------
 * Tables by column (device pointers).  Supplier and customer keys are 1-based
 * row numbers; l_orderkey is the order's row (the reference's
 * l_orderkey_new); n_regionkey[n] is the region row of nation n; nation keys
 * are < 64. */
typedef struct olap_q5_tables {
  const int32_t* r_regionkey;  int64_t n_region;
  const int32_t* n_regionkey;  int64_t n_nation;
  const int32_t* s_nationkey;  int64_t n_supp;
  const int32_t* c_nationkey;  int64_t n_cust;
  const int32_t* o_custkey;
  const int32_t* o_orderdate;  int64_t n_orders;
  const int32_t* l_orderkey;
  const int32_t* l_suppkey;
  const int32_t* l_price;      /* extended price in cents     */
  const int32_t* l_discount;   /* discount in percent [0,100] */
  int64_t n_lines;
} olap_q5_tables;
/* set_bitmap + DimVec_S + DimVec_o + Tri_table_join (Q5.cpp:913-978):
 * nation_sums[n] (device, n_nation entries) = SUM l_price * (100 -
 * l_discount) over the lines whose supplier's nation is n, lies in a region
 * with key `region`, and equals the nation of the line's order's customer,
 * the order dated in [date1, date2).  int64 fixed point (the reference sums
 * price * (1 - discount) in double).  Out-of-range customer, supplier or
 * order references are dropped and counted as range errors. */
OLAP_API int olap_q5_chain(olap_ctx* ctx, const olap_q5_tables* t, int32_t region, int32_t date1,
                           int32_t date2, int64_t* nation_sums);

/* Up to OLAP_Q5_MAX_BATCH Q5 queries, each with its own region and date
 * range, in one pass over orders and one over lineitem (no counterpart in the
 * reference, which runs one query per process).  nation_sums is device
 * memory of n_queries x n_nation int64: row q equals, bit for bit, what
 * olap_q5_chain gives for query q alone.  Each out-of-range reference is
 * counted once per call (a customer reference only when the order's date
 * lies in some query's range). */
#define OLAP_Q5_MAX_BATCH 64
typedef struct olap_q5_query {
  int32_t region, date1, date2;
} olap_q5_query;
OLAP_API int olap_q5_batch(olap_ctx* ctx, const olap_q5_tables* t, const olap_q5_query* queries, int n_queries,
                           int64_t* nation_sums);

/* ---- seeded synthetic data (counter-based; identical on host and device) --
 * Value i of stream s under seed k is a pure function of (k, s, i), so any
 * slice can be generated anywhere.  _dev variants write device memory on the
 * context stream; the plain variants write host memory with nthreads threads
 * (0 = all cores). */
OLAP_API int olap_gen_uniform_i32_dev(olap_ctx* ctx, int32_t* out, int64_t n, uint64_t seed,
                             uint64_t stream, int32_t lo, int32_t hi);
OLAP_API int olap_gen_uniform_i32(int32_t* out, int64_t n, uint64_t seed, uint64_t stream,
                         int32_t lo, int32_t hi, int nthreads);
/* Zipf(s) keys in [0, n_keys): P(k) proportional to 1/(k+1)^s. */
OLAP_API int olap_gen_zipf_i32_dev(olap_ctx* ctx, int32_t* out, int64_t n, uint64_t seed,
                          uint64_t stream, int64_t n_keys, double s);
OLAP_API int olap_gen_zipf_i32(int32_t* out, int64_t n, uint64_t seed, uint64_t stream,
                      int64_t n_keys, double s, int nthreads);
/* Dimension vector: entry i is DIM_NULL with probability 1 - sele, else a
 * group code uniform in [0, groups). */
OLAP_API int olap_gen_dimvec_dev(olap_ctx* ctx, int8_t* out, int64_t n, uint64_t seed,
                        uint64_t stream, double sele, int32_t groups);
OLAP_API int olap_gen_dimvec(int8_t* out, int64_t n, uint64_t seed, uint64_t stream,
                    double sele, int32_t groups, int nthreads);

#ifdef __cplusplus
}
#endif

#endif /* OLAP_CAPI_H */
