// Star-join entry point for callers that cannot allocate device memory.
//
// Some host programs are not allowed to call cudaMalloc at all: a process
// that runs under a fixed device-memory budget set by someone else, code that
// runs inside another framework's allocator (which must see every byte), or a
// caller in a context where allocation could block or fail late, such as a
// real-time request path.  The normal entry points take their scratch from an
// olap_ctx, and creating one allocates.  This file gives those callers one
// entry point that needs no context: its scratch (the error counter, the
// "group code is not 0" flags and the pass bitmaps of the plan) lives in a
// fixed static device array, which the CUDA runtime reserves on every GPU
// that loads this library and keeps until the process exits.
//
// Limits and behaviour:
//  * Scratch is OLAP_NOALLOC_SCRATCH_BYTES (1 MiB).  A query whose pass
//    bitmaps would not fit (the dimension vectors together hold more than
//    OLAP_NOALLOC_MAX_DIM_ENTRIES entries) is rejected with
//    OLAP_ERR_CAPACITY before anything is launched.
//  * Every call uses the same array and it keeps the previous call's
//    contents; what must start at zero is cleared by each call on its stream.
//    Calls whose work overlaps on the GPU (different streams, or different
//    host threads without ordering) race on the array and must be avoided.
//  * The first call on each device looks up the array's device address with
//    cudaGetSymbolAddress (with that device current) and caches it for the
//    life of the process; make that first call before any stream capture.
//    The device must not be reset between calls (cudaDeviceReset, or a
//    teardown of its primary context): the cached address would then belong
//    to a context that no longer exists.
//  * No cudaMalloc, cudaFree or other allocation of device or pinned memory is
//    made; inputs and outputs are the caller's device pointers.
#include <cstring>
#include <mutex>

#include "olap_internal.cuh"

namespace {

constexpr size_t kNoallocScratchBytes = OLAP_NOALLOC_SCRATCH_BYTES;

// The scratch: counters first (the kernels address them through the
// context's `counters` pointer), then the arena's bump allocations.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
void* g_scratch_addr[kMaxDevices] = {};

// Device address of the scratch on `device` (current), looked up once.
cudaError_t scratch_address(int device, void** out) {
  std::lock_guard<std::mutex> lk(g_setup_mu);
  if (!g_scratch_addr[device]) {
    void* ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess) return e;
    g_scratch_addr[device] = ptr;
  }
  *out = g_scratch_addr[device];
  return cudaSuccess;
}

}  // namespace

extern "C" {

int olap_starjoin_groupsum_noalloc(const olap_starjoin_query* q, int64_t* group_sums,
                                   int64_t* totals, int64_t* range_errors, void* cuda_stream) {
  if (!q || q->dimvec_nums < 0 || q->dimvec_nums > OLAP_MAX_DIMS) return OLAP_ERR_INVALID;
  int64_t entries = 0;
  for (int j = 0; j < q->dimvec_nums; ++j) {
    if (q->dimvec_len[j] < 0) return OLAP_ERR_INVALID;
    entries += q->dimvec_len[j];
  }
  if (entries > OLAP_NOALLOC_MAX_DIM_ENTRIES) return OLAP_ERR_CAPACITY;
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess) {
    cudaGetLastError();
    return OLAP_ERR_NO_DEVICE;
  }
  if (device < 0 || device >= kMaxDevices) return OLAP_ERR_UNSUPPORTED;
  void* scratch = nullptr;
  if (scratch_address(device, &scratch) != cudaSuccess) {
    cudaGetLastError();
    return OLAP_ERR_CUDA;
  }
  // A context on the stack over the static scratch: the planner and the
  // kernels are the same as for olap_starjoin_groupsum.
  olap_ctx c;
  c.device = device;
  c.stream = static_cast<cudaStream_t>(cuda_stream);
  c.own_stream = false;
  if (cudaDeviceGetAttribute(&c.sm_count, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
      cudaDeviceGetAttribute(&c.smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device) !=
          cudaSuccess) {
    cudaGetLastError();
    return OLAP_ERR_CUDA;
  }
  c.arena = static_cast<char*>(scratch);
  c.arena_bytes = kNoallocScratchBytes;
  c.counters = reinterpret_cast<olap::DeviceCounters*>(scratch);
  // Plan: pass bitmaps for every dimension not staged whole in shared memory
  // (so the scratch holds them), up to 64 KiB of them staged in shared memory,
  // 1024-thread blocks.
  c.tune[OLAP_TUNE_PROBE_BITS] = 1;
  c.tune[OLAP_TUNE_SMEM_BITS_BYTES] = 64 * 1024;
  c.tune[OLAP_TUNE_BLOCK_THREADS] = 1024;
  // The error counter must start at zero for this call.
  if (cudaMemsetAsync(c.counters, 0, sizeof(olap::DeviceCounters), c.stream) != cudaSuccess) {
    cudaGetLastError();
    return OLAP_ERR_CUDA;
  }
  olap::Arena ar(&c);
  const int st = olap::starjoin_device(&c, q, group_sums, totals, false, c.stream, ar);
  if (st != OLAP_OK) return st;
  if (range_errors &&
      cudaMemcpyAsync(range_errors, &c.counters->range_errors, sizeof(int64_t),
                      cudaMemcpyDeviceToDevice, c.stream) != cudaSuccess) {
    cudaGetLastError();
    return OLAP_ERR_CUDA;
  }
  return OLAP_OK;
}

}  // extern "C"
