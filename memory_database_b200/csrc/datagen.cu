// Seeded synthetic column generators (host and device, bit-identical).
//
// The reference generates its inputs with glibc rand() in one thread
// (include/gendata_util.hpp:449-542), which takes minutes at 600M rows and
// cannot be split.  These generators are counter-based instead: value i of
// stream s under seed k is mix(k, s, i) (a splitmix64 finaliser applied to a
// Weyl sequence), so the device fills 14 GB of fact columns in milliseconds
// and the host can regenerate any slice for the oracle.  All arithmetic that
// decides a value is integer (thresholds and CDF tables are computed once on
// the host and shared), so host and device outputs are identical.
#include <cmath>
#include <thread>
#include <vector>

#include "olap_internal.cuh"

namespace olap {

__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__host__ __device__ __forceinline__ uint64_t stream_key(uint64_t seed, uint64_t stream) {
  return mix64(seed ^ mix64(stream + 0x632BE59BD9B4E019ull));
}

__host__ __device__ __forceinline__ uint64_t draw(uint64_t key, uint64_t i) {
  return mix64(key + (i + 1) * 0x9E3779B97F4A7C15ull);
}

// Uniform integer in [lo, hi] from the high 32 bits (multiply-shift).
__host__ __device__ __forceinline__ int32_t uniform_i32(uint64_t r, int32_t lo, uint64_t span) {
  return static_cast<int32_t>(static_cast<int64_t>(lo) +
                              static_cast<int64_t>(((r >> 32) * span) >> 32));
}

__host__ __device__ __forceinline__ int8_t dimvec_code(uint64_t r, uint64_t thresh, uint32_t groups) {
  if ((r >> 32) >= thresh) return static_cast<int8_t>(OLAP_DIM_NULL);
  return static_cast<int8_t>(((r & 0xffffffffull) * groups) >> 32);
}

// Smallest k with u < cdf[k] (cdf strictly increasing to 2^53).
__host__ __device__ __forceinline__ int32_t zipf_pick(const uint64_t* cdf, int64_t n, uint64_t u) {
  int64_t lo = 0, hi = n - 1;
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (u < cdf[mid]) hi = mid; else lo = mid + 1;
  }
  return static_cast<int32_t>(lo);
}

__global__ void gen_uniform_kernel(int32_t* out, int64_t n, uint64_t key, int32_t lo, uint64_t span) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
    out[i] = uniform_i32(draw(key, i), lo, span);
}

__global__ void gen_dimvec_kernel(int8_t* out, int64_t n, uint64_t key, uint64_t thresh, uint32_t groups) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
    out[i] = dimvec_code(draw(key, i), thresh, groups);
}

__global__ void gen_zipf_kernel(int32_t* out, int64_t n, uint64_t key, const uint64_t* cdf, int64_t nk) {
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
    out[i] = zipf_pick(cdf, nk, draw(key, i) >> 11);
}

static uint64_t sele_threshold(double sele) {
  if (!(sele > 0.0)) return 0;
  if (sele >= 1.0) return uint64_t(1) << 32;
  return static_cast<uint64_t>(std::ldexp(sele, 32));
}

// CDF of Zipf(s) over n keys, scaled to 2^53; strictly increasing, last = 2^53.
static std::vector<uint64_t> zipf_cdf(int64_t n, double s) {
  std::vector<long double> w(static_cast<size_t>(n));
  long double tot = 0;
  for (int64_t k = 0; k < n; ++k) {
    w[k] = std::pow(static_cast<long double>(k + 1), -static_cast<long double>(s));
    tot += w[k];
  }
  std::vector<uint64_t> cdf(static_cast<size_t>(n));
  const long double scale = std::ldexp(1.0L, 53);
  long double acc = 0;
  uint64_t prev = 0;
  for (int64_t k = 0; k < n; ++k) {
    acc += w[k];
    uint64_t c = static_cast<uint64_t>(acc / tot * scale);
    if (c <= prev) c = prev + 1;
    cdf[k] = c;
    prev = c;
  }
  cdf[n - 1] = uint64_t(1) << 53;
  if (n > 1 && cdf[n - 2] >= cdf[n - 1]) cdf[n - 2] = cdf[n - 1] - 1;
  return cdf;
}

template <class F>
static void host_parallel(int64_t n, int nthreads, F f) {
  int nt = nthreads > 0 ? nthreads : static_cast<int>(std::thread::hardware_concurrency());
  if (nt < 1) nt = 1;
  if (n < (int64_t(1) << 16)) nt = 1;
  std::vector<std::thread> th;
  for (int t = 0; t < nt; ++t)
    th.emplace_back([=] { f(n * t / nt, n * (t + 1) / nt); });
  for (auto& x : th) x.join();
}

static unsigned gen_grid(olap_ctx* ctx, int64_t n) {
  int64_t g = (n + 255) / 256;
  const int64_t cap = static_cast<int64_t>(ctx->sm_count) * 8;
  if (g > cap) g = cap;
  return static_cast<unsigned>(g < 1 ? 1 : g);
}

}  // namespace olap

extern "C" {

int olap_gen_uniform_i32_dev(olap_ctx* ctx, int32_t* out, int64_t n, uint64_t seed, uint64_t stream,
                             int32_t lo, int32_t hi) {
  if (!ctx || n < 0 || (n > 0 && !out) || hi < lo) return OLAP_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  OLAP_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  if (n == 0) return OLAP_OK;
  const uint64_t span = static_cast<uint64_t>(static_cast<int64_t>(hi) - lo + 1);
  olap::gen_uniform_kernel<<<olap::gen_grid(ctx, n), 256, 0, ctx->stream>>>(
      out, n, olap::stream_key(seed, stream), lo, span);
  OLAP_CUDA_TRY(ctx, cudaGetLastError());
  return OLAP_OK;
}

int olap_gen_uniform_i32(int32_t* out, int64_t n, uint64_t seed, uint64_t stream, int32_t lo,
                         int32_t hi, int nthreads) {
  if (n < 0 || (n > 0 && !out) || hi < lo) return OLAP_ERR_INVALID;
  const uint64_t span = static_cast<uint64_t>(static_cast<int64_t>(hi) - lo + 1);
  const uint64_t key = olap::stream_key(seed, stream);
  olap::host_parallel(n, nthreads, [=](int64_t b, int64_t e) {
    for (int64_t i = b; i < e; ++i) out[i] = olap::uniform_i32(olap::draw(key, i), lo, span);
  });
  return OLAP_OK;
}

int olap_gen_dimvec_dev(olap_ctx* ctx, int8_t* out, int64_t n, uint64_t seed, uint64_t stream,
                        double sele, int32_t groups) {
  if (!ctx || n < 0 || (n > 0 && !out) || groups < 1 || groups > 127) return OLAP_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  OLAP_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  if (n == 0) return OLAP_OK;
  olap::gen_dimvec_kernel<<<olap::gen_grid(ctx, n), 256, 0, ctx->stream>>>(
      out, n, olap::stream_key(seed, stream), olap::sele_threshold(sele), static_cast<uint32_t>(groups));
  OLAP_CUDA_TRY(ctx, cudaGetLastError());
  return OLAP_OK;
}

int olap_gen_dimvec(int8_t* out, int64_t n, uint64_t seed, uint64_t stream, double sele,
                    int32_t groups, int nthreads) {
  if (n < 0 || (n > 0 && !out) || groups < 1 || groups > 127) return OLAP_ERR_INVALID;
  const uint64_t key = olap::stream_key(seed, stream);
  const uint64_t th = olap::sele_threshold(sele);
  olap::host_parallel(n, nthreads, [=](int64_t b, int64_t e) {
    for (int64_t i = b; i < e; ++i)
      out[i] = olap::dimvec_code(olap::draw(key, i), th, static_cast<uint32_t>(groups));
  });
  return OLAP_OK;
}

int olap_gen_zipf_i32_dev(olap_ctx* ctx, int32_t* out, int64_t n, uint64_t seed, uint64_t stream,
                          int64_t n_keys, double s) {
  if (!ctx || n < 0 || (n > 0 && !out) || n_keys < 1 || n_keys > INT32_MAX || !(s >= 0.0))
    return OLAP_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  OLAP_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  if (n == 0) return OLAP_OK;
  std::vector<uint64_t> cdf = olap::zipf_cdf(n_keys, s);
  uint64_t* dcdf = nullptr;
  OLAP_CUDA_TRY(ctx, cudaMallocAsync(reinterpret_cast<void**>(&dcdf), sizeof(uint64_t) * n_keys, ctx->stream));
  OLAP_CUDA_TRY(ctx, cudaMemcpyAsync(dcdf, cdf.data(), sizeof(uint64_t) * n_keys,
                                     cudaMemcpyHostToDevice, ctx->stream));
  olap::gen_zipf_kernel<<<olap::gen_grid(ctx, n), 256, 0, ctx->stream>>>(
      out, n, olap::stream_key(seed, stream), dcdf, n_keys);
  cudaError_t e = cudaGetLastError();
  cudaFreeAsync(dcdf, ctx->stream);
  // The host table must outlive the asynchronous copy.
  cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return olap::check_cuda(ctx, e, "gen_zipf_kernel");
  return OLAP_OK;
}

int olap_gen_zipf_i32(int32_t* out, int64_t n, uint64_t seed, uint64_t stream, int64_t n_keys,
                      double s, int nthreads) {
  if (n < 0 || (n > 0 && !out) || n_keys < 1 || n_keys > INT32_MAX || !(s >= 0.0))
    return OLAP_ERR_INVALID;
  if (n == 0) return OLAP_OK;
  std::vector<uint64_t> cdf = olap::zipf_cdf(n_keys, s);
  const uint64_t key = olap::stream_key(seed, stream);
  const uint64_t* c = cdf.data();
  olap::host_parallel(n, nthreads, [=](int64_t b, int64_t e) {
    for (int64_t i = b; i < e; ++i) out[i] = olap::zipf_pick(c, n_keys, olap::draw(key, i) >> 11);
  });
  return OLAP_OK;
}

}  // extern "C"
