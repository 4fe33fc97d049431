// Allocation-free variant of the batched persistent launch.
//
// Some hosts of this library cannot let it allocate device memory at render
// time: an application that owns a fixed device-memory budget and hands every
// byte to its own allocator, a plugin living inside such a host, or a
// latency-critical serving loop where a cudaMalloc (which may synchronise the
// device) is not acceptable.  mtc_trace_batch needs a caller-provided scratch
// block for its job table and work-queue counter; this entry point instead
// keeps that scratch in one fixed-size array in the library's device image, so
// the caller passes only the jobs (their scene buffers and accumulation
// outputs) and nothing is allocated on the device by this call.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>

#include "batch_table.cuh"

using namespace mt;

namespace {

// The scratch: a job table (header, then MTC_BATCH_NOALLOC_MAX_JOBS entries)
// followed by the 256-byte work-queue block.
constexpr size_t kTableBytes =
    (kBatchTableOffset + size_t(MTC_BATCH_NOALLOC_MAX_JOBS) * sizeof(JobData) + 255) / 256 * 256;
constexpr size_t kScratchBytes = kTableBytes + 256;

// The shared scratch: every call on a device reuses it, so two calls whose
// work overlaps on that device would race on the table and the counter.
static __device__ __align__(256) unsigned char g_noallocScratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setupMutex;
struct ScratchAddress {
  void *ptr;
  unsigned long long context;  // id of the context the address belongs to
};
ScratchAddress g_scratchAddress[kMaxDevices] = {};

// Id of the calling thread's current context (cuCtxGetId through the
// runtime's driver entry point, so the library need not link libcuda);
// 0 when the driver does not provide it.
unsigned long long currentContextId() {
  using GetCurrent = CUresult (*)(CUcontext *);
  using GetId = CUresult (*)(CUcontext, unsigned long long *);
  static GetCurrent getCurrent = nullptr;
  static GetId getId = nullptr;
  static bool looked = false;
  if (!looked) {
    void *a = nullptr, *b = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &a, cudaEnableDefault) == cudaSuccess &&
        cudaGetDriverEntryPoint("cuCtxGetId", &b, cudaEnableDefault) == cudaSuccess) {
      getCurrent = reinterpret_cast<GetCurrent>(a);
      getId = reinterpret_cast<GetId>(b);
    }
    cudaGetLastError();
    looked = true;
  }
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if (getCurrent && getId && getCurrent(&ctx) == CUDA_SUCCESS && ctx && getId(ctx, &id) == CUDA_SUCCESS) return id;
  return 0;
}

// Device address of g_noallocScratch for the current device; resolved once
// per device and context (host code must not use the symbol itself as a
// pointer).  A device whose primary context was reset since the last call
// gets a new context id, and its address is looked up again.
cudaError_t scratchAddress(void **out) {
  int device = 0;
  cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess) return e;
  if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
  e = cudaSetDevice(device);  // initialises the device's primary context and makes it current
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> g(g_setupMutex);
  const unsigned long long context = currentContextId();
  ScratchAddress &slot = g_scratchAddress[device];
  if (!slot.ptr || slot.context != context) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noallocScratch);
    if (e != cudaSuccess) return e;
    slot.ptr = p;
    slot.context = context;
  }
  *out = slot.ptr;
  return cudaSuccess;
}

// The persistent batched kernel of batch_table.cuh over the fixed scratch.
template <bool kGpuLayout>
__global__ void __launch_bounds__(128, MT_BATCH_MIN_BLOCKS)
    k_batch_noalloc(const BatchHeader *__restrict__ header, uint32_t *queue, uint32_t grain, uint32_t *status,
                    mtc_counters *counters) {
  Counters cnt;
  uint32_t paths = 0;
  batchWorkLoop<kGpuLayout>(header, queue, grain, status, cnt, paths);
  if (counters) {
    unsigned mask = __activemask();
    uint32_t e = __reduce_add_sync(mask, cnt.ext), s = __reduce_add_sync(mask, cnt.shadow);
    uint32_t p = __reduce_add_sync(mask, paths);
    if ((threadIdx.x & 31) == uint32_t(__ffs(mask) - 1)) {
      atomicAdd(&counters->extension_rays, (unsigned long long)e);
      atomicAdd(&counters->shadow_rays, (unsigned long long)s);
      atomicAdd(&counters->path_samples, (unsigned long long)p);
    }
  }
}

}  // namespace

// Jobs and launch shape are validated by the same rules as mtc_trace_batch
// (validScene, validUniform, batchShape in batch_table.cuh), and every field
// of mtc_batch_config is applied as there.
extern "C" mt_status mtc_trace_batch_noalloc(const mtc_job_desc *jobs, uint32_t job_count,
                                             const mtc_batch_config *config, uint32_t *status_out,
                                             mtc_counters *counters, void *stream) {
  if (!jobs && job_count) return MT_ERROR_INVALID_ARGUMENT;
  if (job_count > MTC_BATCH_NOALLOC_MAX_JOBS) return MT_ERROR_INVALID_ARGUMENT;  // beyond the fixed scratch
  BatchShape shape;
  if (!batchShape(config, shape)) return MT_ERROR_INVALID_ARGUMENT;
  if (job_count == 0) return MT_OK;
  // The table is assembled in host stack memory: no allocation on either side.
  alignas(16) unsigned char table[kBatchTableOffset + size_t(MTC_BATCH_NOALLOC_MAX_JOBS) * sizeof(JobData)];
  mt_status st = writeBatchTable(jobs, job_count, shape, table, nullptr);
  if (st != MT_OK) return st;
  void *scratch = nullptr;
  cudaError_t e = scratchAddress(&scratch);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver ? MT_ERROR_UNAVAILABLE : MT_ERROR;
  }
  cudaStream_t cs = (cudaStream_t)stream;
  uint32_t *queue = (uint32_t *)((char *)scratch + kTableBytes);
  // The table is overwritten and the queue counter cleared on every call.
  e = cudaMemcpyAsync(scratch, table, kBatchTableOffset + size_t(job_count) * sizeof(JobData),
                      cudaMemcpyHostToDevice, cs);
  if (e == cudaSuccess) e = cudaMemsetAsync(queue, 0, 256, cs);
  if (e == cudaSuccess && status_out) e = cudaMemsetAsync(status_out, 0, sizeof(uint32_t), cs);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return MT_ERROR;
  }
  int device = 0, sms = 148;
  cudaGetDevice(&device);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  const uint32_t grid = uint32_t(sms) * shape.ctasPerSm;
  const uint32_t flagsUnion = reinterpret_cast<const BatchHeader *>(table)->flagsUnion;
  const BatchHeader *header = (const BatchHeader *)scratch;
  if (flagsUnion & MTC_SCENE_BLAS_GPU_LAYOUT)
    k_batch_noalloc<true><<<grid, shape.blockThreads, 0, cs>>>(header, queue, shape.grain, status_out, counters);
  else
    k_batch_noalloc<false><<<grid, shape.blockThreads, 0, cs>>>(header, queue, shape.grain, status_out, counters);
  e = cudaGetLastError();
  return e == cudaSuccess ? MT_OK : MT_ERROR;
}
