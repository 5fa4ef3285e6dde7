// Context, status and plan helpers of the C-ABI (olap_capi.h).
#include <cstdio>
#include <cstring>
#include <new>

#include "compact.cuh"

namespace olap {

int set_error(olap_ctx* ctx, int status, const std::string& msg) {
  if (ctx) ctx->last_error = msg;
  return status;
}

int check_cuda(olap_ctx* ctx, cudaError_t e, const char* what) {
  std::string m = std::string(what) + ": " + cudaGetErrorString(e);
  int st = OLAP_ERR_CUDA;
  if (e == cudaErrorMemoryAllocation) st = OLAP_ERR_NOMEM;
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) st = OLAP_ERR_NO_DEVICE;
  return set_error(ctx, st, m);
}

// Largest value of a column: per-warp maxima, one atomicMax per warp.
__global__ void max_i32_kernel(const int32_t* __restrict__ col, int64_t n, int* out) {
  int m = INT32_MIN;
  const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
    m = max(m, __ldg(col + i));
  m = __reduce_max_sync(0xffffffffu, m);
  if ((threadIdx.x & 31) == 0 && m != INT32_MIN) atomicMax(out, m);
}

}  // namespace olap

extern "C" {

int olap_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

#define OLAP_STR2(x) #x
#define OLAP_STR(x) OLAP_STR2(x)
const char* olap_build_info(void) {
  return "libolapcore_b200: sm_100a kernels, CUDA runtime " OLAP_STR(CUDART_VERSION);
}

const char* olap_status_string(int status) {
  switch (status) {
    case OLAP_OK: return "ok";
    case OLAP_ERR_INVALID: return "invalid argument";
    case OLAP_ERR_CUDA: return "CUDA error";
    case OLAP_ERR_NO_DEVICE: return "no usable CUDA device";
    case OLAP_ERR_NOMEM: return "out of memory";
    case OLAP_ERR_RANGE: return "rows dropped: key or group id out of range";
    case OLAP_ERR_CAPACITY: return "capacity exceeded";
    case OLAP_ERR_TIMEOUT: return "bounded device wait expired";
    case OLAP_ERR_UNSUPPORTED: return "unsupported";
    default: return "unknown status";
  }
}

int olap_ctx_create(int device, size_t scratch_bytes, olap_ctx** out) {
  if (!out) return OLAP_ERR_INVALID;
  *out = nullptr;
  int n = olap_device_count();
  if (n <= 0) return OLAP_ERR_NO_DEVICE;
  if (device < 0 || device >= n) return OLAP_ERR_INVALID;
  olap_ctx* c = new (std::nothrow) olap_ctx();
  if (!c) return OLAP_ERR_NOMEM;
  c->device = device;
  auto fail = [&](int st) {
    if (c->arena) cudaFree(c->arena);
    if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return st;
  };
  if (cudaSetDevice(device) != cudaSuccess) return fail(OLAP_ERR_NO_DEVICE);
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return fail(OLAP_ERR_CUDA);
  c->sm_count = prop.multiProcessorCount;
  c->smem_optin = static_cast<int>(prop.sharedMemPerBlockOptin);
  c->l2_bytes = prop.l2CacheSize;
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess)
    return fail(OLAP_ERR_CUDA);
  c->own_stream = true;
  c->arena_bytes = scratch_bytes ? scratch_bytes : (size_t(64) << 20);
  if (c->arena_bytes < (size_t(1) << 20)) c->arena_bytes = size_t(1) << 20;
  if (cudaMalloc(&c->arena, c->arena_bytes) != cudaSuccess) {
    cudaGetLastError();
    c->arena = nullptr;
    return fail(OLAP_ERR_NOMEM);
  }
  c->counters = reinterpret_cast<olap::DeviceCounters*>(c->arena);
  if (cudaMemset(c->arena, 0, sizeof(olap::DeviceCounters)) != cudaSuccess)
    return fail(OLAP_ERR_CUDA);
  *out = c;
  return OLAP_OK;
}

int olap_ctx_destroy(olap_ctx* ctx) {
  if (!ctx) return OLAP_ERR_INVALID;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->arena) cudaFree(ctx->arena);
  if (ctx->big) cudaFree(ctx->big);
  if (ctx->pinned) cudaFreeHost(ctx->pinned);
  if (ctx->own_stream && ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return OLAP_OK;
}

int olap_ctx_set_stream(olap_ctx* ctx, void* cuda_stream) {
  if (!ctx) return OLAP_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);
  if (!ctx->own_stream && s == ctx->stream) return OLAP_OK;
  OLAP_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  if (ctx->own_stream && ctx->stream) {
    cudaStreamSynchronize(ctx->stream);
    cudaStreamDestroy(ctx->stream);
  }
  ctx->stream = s;
  ctx->own_stream = false;
  return OLAP_OK;
}

void* olap_ctx_get_stream(olap_ctx* ctx) { return ctx ? static_cast<void*>(ctx->stream) : nullptr; }

int olap_ctx_synchronize(olap_ctx* ctx) {
  if (!ctx) return OLAP_ERR_INVALID;
  cudaSetDevice(ctx->device);
  OLAP_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return olap::check_timeouts(ctx, ctx->stream);
}

int olap_ctx_set_tuning(olap_ctx* ctx, int knob, int64_t value) {
  if (!ctx || knob < 0 || knob >= OLAP_TUNE_KNOBS || value < 0) return OLAP_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  ctx->tune[knob] = value;
  return OLAP_OK;
}

int olap_ctx_take_range_errors(olap_ctx* ctx, int64_t* count) {
  if (!ctx || !count) return OLAP_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  unsigned long long v = 0;
  OLAP_CUDA_TRY(ctx, cudaMemcpyAsync(&v, &ctx->counters->range_errors, sizeof(v),
                                     cudaMemcpyDeviceToHost, ctx->stream));
  OLAP_CUDA_TRY(ctx, cudaMemsetAsync(&ctx->counters->range_errors, 0, sizeof(v), ctx->stream));
  OLAP_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  *count = static_cast<int64_t>(v);
  // A bounded device wait that gave up (asynchronous calls record it here).
  return olap::check_timeouts(ctx, ctx->stream);
}

int olap_ctx_take_host_bytes(olap_ctx* ctx, int64_t* bytes) {
  if (!ctx || !bytes) return OLAP_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  cudaSetDevice(ctx->device);
  unsigned long long sectors = 0;
  OLAP_CUDA_TRY(ctx, cudaMemcpyAsync(&sectors, &ctx->counters->host_sectors, sizeof(sectors),
                                     cudaMemcpyDeviceToHost, ctx->stream));
  OLAP_CUDA_TRY(ctx, cudaMemsetAsync(&ctx->counters->host_sectors, 0, sizeof(sectors), ctx->stream));
  OLAP_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  *bytes = ctx->host_bytes + static_cast<int64_t>(sectors) * 32;
  ctx->host_bytes = 0;
  return OLAP_OK;
}

const char* olap_ctx_last_error(const olap_ctx* ctx) {
  return ctx ? ctx->last_error.c_str() : "null context";
}

// Plan of the reference's main: code/OLAPcore/test_multi_compute_operator.cpp
// lines 1964-1987 (dimension selection, sort_by_rate at 223-233, group_nums
// and the factor rule).  The ordering step deliberately keeps the reference's
// comparison of sele[i] with sele[j] by position (not sele[orders[i]]), so
// that group ids come out exactly as the reference numbers them.
int olap_plan_olapcore(const double sele[4], const int bitmap[4], const int groups[4],
                       int orders[4], int factor[4], int* dimvec_nums, int64_t* group_nums) {
  if (!sele || !bitmap || !groups || !orders || !factor || !dimvec_nums || !group_nums)
    return OLAP_ERR_INVALID;
  int nd = 0;
  for (int t = 0; t < 4; ++t) {
    if (groups[t] < 0) return OLAP_ERR_INVALID;
    factor[t] = 1;
    orders[t] = -1;
    if (groups[t] != 0) orders[nd++] = t;
  }
  for (int i = 0; i < nd; ++i)
    for (int j = i + 1; j < nd; ++j)
      if (sele[i] > sele[j]) {
        int tmp = orders[i];
        orders[i] = orders[j];
        orders[j] = tmp;
      }
  int64_t g = 1;
  for (int i = 0; i < nd; ++i) {
    g *= groups[orders[i]];
    if (bitmap[orders[i]] == 0) continue;
    int64_t f = 1;
    for (int j = i + 1; j < nd; ++j) f *= groups[orders[j]];
    if (f > INT32_MAX) return OLAP_ERR_INVALID;
    factor[i] = static_cast<int>(f);
  }
  *dimvec_nums = nd;
  *group_nums = g;
  return OLAP_OK;
}

int olap_buffer_alloc(olap_ctx* ctx, size_t bytes, void** dev) {
  if (!ctx || !dev) return OLAP_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  *dev = nullptr;
  OLAP_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  OLAP_CUDA_TRY(ctx, cudaMalloc(dev, bytes ? bytes : 1));
  return OLAP_OK;
}

int olap_buffer_free(olap_ctx* ctx, void* dev) {
  if (!ctx) return OLAP_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (!dev) return OLAP_OK;
  OLAP_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  OLAP_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  OLAP_CUDA_TRY(ctx, cudaFree(dev));
  return OLAP_OK;
}

int olap_copy_h2d(olap_ctx* ctx, void* dev, const void* host, size_t bytes) {
  if (!ctx || (bytes && (!dev || !host))) return OLAP_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (!bytes) return OLAP_OK;
  OLAP_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  OLAP_CUDA_TRY(ctx, cudaMemcpyAsync(dev, host, bytes, cudaMemcpyHostToDevice, ctx->stream));
  OLAP_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return OLAP_OK;
}

int olap_copy_d2h(olap_ctx* ctx, void* host, const void* dev, size_t bytes) {
  if (!ctx || (bytes && (!dev || !host))) return OLAP_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  if (!bytes) return OLAP_OK;
  OLAP_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  OLAP_CUDA_TRY(ctx, cudaMemcpyAsync(host, dev, bytes, cudaMemcpyDeviceToHost, ctx->stream));
  OLAP_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  return OLAP_OK;
}

int olap_max_i32(olap_ctx* ctx, const int32_t* col, int64_t n, int32_t* h_max) {
  if (!ctx || !h_max || n < 0 || (n > 0 && !col)) return OLAP_ERR_INVALID;
  std::lock_guard<std::mutex> lk(ctx->mu);
  *h_max = INT32_MIN;
  if (n == 0) return OLAP_OK;
  OLAP_CUDA_TRY(ctx, cudaSetDevice(ctx->device));
  olap::Arena ar(ctx);
  int* d = ar.take<int>(1);
  if (!d) return olap::set_error(ctx, OLAP_ERR_CAPACITY, "scratch arena exhausted");
  const int init = INT32_MIN;
  OLAP_CUDA_TRY(ctx, cudaMemcpyAsync(d, &init, sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
  const int64_t blocks = std::min<int64_t>(int64_t(ctx->sm_count) * 4, (n + 255) / 256);
  olap::max_i32_kernel<<<static_cast<unsigned>(blocks), 256, 0, ctx->stream>>>(col, n, d);
  OLAP_CUDA_TRY(ctx, cudaGetLastError());
  int v = INT32_MIN;
  OLAP_CUDA_TRY(ctx, cudaMemcpyAsync(&v, d, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  OLAP_CUDA_TRY(ctx, cudaStreamSynchronize(ctx->stream));
  *h_max = v;
  return OLAP_OK;
}

}  // extern "C"
