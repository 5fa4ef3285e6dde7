// Empirical autotuner of the star-join launch plan.
//
// The best plan depends on the data, not only on the shape: how many rows
// survive each probe decides whether random L2 probes or shared-memory
// capacity bound the scan.  The tuner therefore times a handful of candidate
// plans (staging of int8 vectors and pass bitmaps in shared memory, global
// bitmaps through L1, accumulator placement, block size) on a sample of the
// query's own fact range, with CUDA events on the context stream, and leaves
// the fastest candidate's knobs set on the context.
#include <algorithm>
#include <cstring>
#include <vector>

#include "olap_internal.cuh"

namespace olap {

namespace {

struct Candidate {
  int64_t knob[16];  // indexed by OLAP_TUNE_*; 0 = automatic
};

std::vector<Candidate> candidates(const olap_ctx* ctx, const olap_starjoin_query* q) {
  const int64_t cap = ctx->smem_optin - 2048;
  int64_t bits_all = 0;
  for (int j = 0; j < q->dimvec_nums; ++j) bits_all += ((q->dimvec_len[j] + 31) / 32 * 4 + 15) & ~int64_t(15);
  std::vector<Candidate> c;
  auto add = [&](std::initializer_list<std::pair<int, int64_t>> kv) {
    Candidate x;
    std::memset(&x, 0, sizeof(x));
    for (auto& p : kv) x.knob[p.first] = p.second;
    c.push_back(x);
  };
  // int8 probes, small vectors staged, accumulators in smem when they fit.
  add({{OLAP_TUNE_PROBE_BITS, 2}});
  add({{OLAP_TUNE_PROBE_BITS, 2}, {OLAP_TUNE_BLOCK_THREADS, 1024}});
  // Global pass bitmaps through L1, accumulators in L2 (max L1 capacity).
  add({{OLAP_TUNE_PROBE_BITS, 1}, {OLAP_TUNE_SMEM_ACC_BYTES, 1}});
  // Pass bitmaps staged in shared memory: as many as fit, then half of that.
  for (int64_t budget : {std::min(cap, bits_all), std::min(cap, bits_all) / 2, int64_t(64) << 10}) {
    if (budget < 4096) continue;
    add({{OLAP_TUNE_PROBE_BITS, 2}, {OLAP_TUNE_SMEM_BITS_BYTES, budget}});
    add({{OLAP_TUNE_PROBE_BITS, 2}, {OLAP_TUNE_SMEM_BITS_BYTES, budget}, {OLAP_TUNE_BLOCK_THREADS, 1024}});
    add({{OLAP_TUNE_PROBE_BITS, 1}, {OLAP_TUNE_SMEM_BITS_BYTES, budget}, {OLAP_TUNE_SMEM_ACC_BYTES, 1},
         {OLAP_TUNE_BLOCK_THREADS, 1024}});
  }
  // 4-bit codes of the dimensions that fit, with and without pass bitmaps for
  // the rest (filter and group code of a dimension in one shared probe).
  add({{OLAP_TUNE_PROBE_BITS, 2}, {OLAP_TUNE_SMEM_NIB_BYTES, cap}, {OLAP_TUNE_BLOCK_THREADS, 1024}});
  add({{OLAP_TUNE_PROBE_BITS, 2}, {OLAP_TUNE_SMEM_NIB_BYTES, cap}, {OLAP_TUNE_SMEM_BITS_BYTES, int64_t(64) << 10},
       {OLAP_TUNE_BLOCK_THREADS, 1024}});
  add({{OLAP_TUNE_PROBE_BITS, 2}, {OLAP_TUNE_SMEM_NIB_BYTES, int64_t(112) << 10}, {OLAP_TUNE_BLOCK_THREADS, 1024}});
  // ... and with the accumulators in L2, which leaves L1 more room
  add({{OLAP_TUNE_PROBE_BITS, 2}, {OLAP_TUNE_SMEM_NIB_BYTES, cap}, {OLAP_TUNE_SMEM_ACC_BYTES, 1},
       {OLAP_TUNE_BLOCK_THREADS, 1024}});
  add({{OLAP_TUNE_PROBE_BITS, 2}, {OLAP_TUNE_SMEM_NIB_BYTES, int64_t(112) << 10}, {OLAP_TUNE_SMEM_ACC_BYTES, 1},
       {OLAP_TUNE_BLOCK_THREADS, 1024}});
  // Every plan also with the survivors of the shared-memory probes compacted
  // per warp, with the fact columns prefetched by bulk copies, with 8 rows
  // per thread (512-thread blocks) and with merged L2 probes.
  const size_t n4 = c.size();
  for (size_t i = 0; i < n4; ++i) {
    Candidate x = c[i];
    x.knob[OLAP_TUNE_COMPACT] = 2;
    c.push_back(x);
    x.knob[OLAP_TUNE_COMPACT] = 0;
    x.knob[OLAP_TUNE_ASYNC_LOADS] = 2;  // bulk-copy prefetch of the fact columns
    c.push_back(x);
  }
  for (size_t i = 0; i < n4; ++i) {
    Candidate x = c[i];
    x.knob[OLAP_TUNE_UNROLL] = 2;
    x.knob[OLAP_TUNE_BLOCK_THREADS] = 512;
    c.push_back(x);
  }
  // ... and with consecutive L2 probes issued together (one round trip),
  // also with the int8-staged dimensions probed last.
  for (size_t i = 0; i < n4; ++i) {
    Candidate x = c[i];
    x.knob[OLAP_TUNE_MERGE_PROBES] = 1;
    c.push_back(x);
    x.knob[OLAP_TUNE_PROBE_ORDER] = 1;
    c.push_back(x);
  }
  return c;
}

}  // namespace

}  // namespace olap

extern "C" {

// Times the candidate plans on rows [row_begin, row_begin + sample_rows) of
// the query (device pointers), sets the fastest candidate's knobs on the
// context and returns them in knobs_out[0..15] (may be NULL) with its time
// per sample in *best_ms (may be NULL).  Results of the timed runs are
// discarded; the query's own outputs are not touched.
int olap_starjoin_autotune(olap_ctx* ctx, const olap_starjoin_query* q, int64_t sample_rows,
                           int64_t* knobs_out, double* best_ms) {
  if (!ctx || !q) return OLAP_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  OLAP_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  OLAP_REQUIRE(ctx, q->n_aggs >= 1 && q->n_aggs <= 2 && q->group_nums >= 1 &&
                        q->group_nums <= INT32_MAX && q->row_end >= q->row_begin,
               "invalid query");
  unsigned long long errs_before = 0;
  OLAP_CUDA_TRY(ctx, cudaMemcpyAsync(&errs_before, &ctx->counters->range_errors, sizeof(errs_before),
                                     cudaMemcpyDeviceToHost, ctx->stream));
  OLAP_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  olap_starjoin_query sq = *q;
  if (sample_rows <= 0) sample_rows = int64_t(64) << 20;
  sq.row_end = std::min(q->row_end, q->row_begin + sample_rows);
  olap::Arena ar(ctx);
  int64_t* gs = ar.take<int64_t>(static_cast<size_t>(q->group_nums * q->n_aggs));
  int64_t* tot = ar.take<int64_t>(2);
  if (!gs || !tot) return olap::set_error(ctx, OLAP_ERR_CAPACITY, "scratch arena too small to autotune");
  const olap::Arena base = ar;
  // Candidates are evaluated from the automatic plan (the plan knobs of any
  // earlier tuning are cleared); knobs outside the plan are kept.
  int64_t saved[16];
  std::memcpy(saved, ctx->tune, sizeof(saved));
  for (int k : {OLAP_TUNE_BLOCK_THREADS, OLAP_TUNE_BLOCKS_PER_SM, OLAP_TUNE_SMEM_DIM_BYTES,
                OLAP_TUNE_SMEM_ACC_BYTES, OLAP_TUNE_UNROLL, OLAP_TUNE_PROBE_BITS,
                OLAP_TUNE_SMEM_BITS_BYTES, OLAP_TUNE_ASYNC_LOADS, OLAP_TUNE_COMPACT,
                OLAP_TUNE_SMEM_NIB_BYTES, OLAP_TUNE_MERGE_PROBES, OLAP_TUNE_PROBE_ORDER})
    saved[k] = 0;
  cudaEvent_t e0, e1;
  OLAP_CUDA_TRY(ctx, cudaEventCreate(&e0));
  OLAP_CUDA_TRY(ctx, cudaEventCreate(&e1));
  double best = 1e30;
  int64_t best_knob[16] = {0};
  int st = OLAP_OK;
  for (const auto& cand : olap::candidates(ctx, q)) {
    std::memcpy(ctx->tune, saved, sizeof(saved));
    for (int k = 0; k < 16; ++k) if (cand.knob[k]) ctx->tune[k] = cand.knob[k];
    float ms = 0.f, tot_ms = 1e30f;
    bool ok = true;
    for (int rep = 0; rep < 4 && ok; ++rep) {
      olap::Arena car = base;
      cudaEventRecord(e0, ctx->stream);
      int s2 = olap::starjoin_device(ctx, &sq, gs, tot, false, ctx->stream, car);
      cudaEventRecord(e1, ctx->stream);
      if (s2 != OLAP_OK || cudaEventSynchronize(e1) != cudaSuccess) {
        ok = false;
        cudaGetLastError();
        break;
      }
      cudaEventElapsedTime(&ms, e0, e1);
      if (rep > 0) tot_ms = std::min(tot_ms, ms);  // first run warms caches
    }
    if (ok && tot_ms < best) {
      best = tot_ms;
      std::memcpy(best_knob, cand.knob, sizeof(best_knob));
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  std::memcpy(ctx->tune, saved, sizeof(saved));
  if (best >= 1e29) return olap::set_error(ctx, OLAP_ERR_CUDA, "no autotune candidate ran");
  for (int k = 0; k < 16; ++k)
    if (best_knob[k]) ctx->tune[k] = best_knob[k];
  // Rows dropped in the timed runs were counted; the caller's query will
  // count them again, so restore the count from before the tuner ran.
  OLAP_CUDA_TRY(ctx, cudaMemcpyAsync(&ctx->counters->range_errors, &errs_before, sizeof(errs_before),
                                     cudaMemcpyHostToDevice, ctx->stream));
  OLAP_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  if (knobs_out) std::memcpy(knobs_out, best_knob, sizeof(best_knob));
  if (best_ms) *best_ms = best;
  return st;
}

}  // extern "C"
