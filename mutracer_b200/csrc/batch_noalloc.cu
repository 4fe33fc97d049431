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
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "dev_shade.cuh"

using namespace mt;

namespace {

constexpr int kWarpTileW = 8, kWarpTileH = 4;  // same warp tile as k_batch
constexpr size_t kTableBytes = (size_t(MTC_BATCH_NOALLOC_MAX_JOBS) * sizeof(JobData) + 255) / 256 * 256;
constexpr size_t kScratchBytes = kTableBytes + 256;  // job table, then the queue counter

// The shared scratch: every call on a device reuses it, so two calls whose
// work overlaps on that device would race on the table and the counter.
static __device__ __align__(256) unsigned char g_noallocScratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setupMutex;
void *g_scratchAddress[kMaxDevices] = {};

// Device address of g_noallocScratch for the current device; resolved once
// per device (host code must not use the symbol itself as a pointer).
cudaError_t scratchAddress(void **out) {
  int device = 0;
  cudaError_t e = cudaGetDevice(&device);
  if (e != cudaSuccess) return e;
  if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> g(g_setupMutex);
  if (!g_scratchAddress[device]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noallocScratch);
    if (e != cudaSuccess) return e;
    g_scratchAddress[device] = p;
  }
  *out = g_scratchAddress[device];
  return cudaSuccess;
}

template <bool kGpuLayout>
__global__ void __launch_bounds__(128)
    k_batch_noalloc(const JobData *__restrict__ jobs, uint32_t job_count, uint32_t total_items, uint32_t *queue,
                    mtc_counters *counters) {
  const uint32_t lane = threadIdx.x & 31u;
  Counters cnt;
  uint32_t paths = 0;
  for (uint32_t guard = 0; guard < total_items + 1u; guard++) {
    uint32_t item = 0;
    if (lane == 0) item = atomicAdd(queue, 1u);
    item = __shfl_sync(0xffffffffu, item, 0);
    if (item >= total_items) break;
    uint32_t j = 0;
    while (j + 1 < job_count && jobs[j + 1].firstItem <= item) j++;
    const JobData &J = jobs[j];
    uint32_t local = item - J.firstItem;
    uint32_t tx = local % J.tilesX, ty = local / J.tilesX;
    uint32_t x = tx * kWarpTileW + (lane % kWarpTileW), y = ty * kWarpTileH + (lane / kWarpTileW);
    if (x < J.width && y < J.height) {
      tracePixelSamples<kGpuLayout>(J, x, y, J.samples, cnt);
      paths += J.samples;
    }
  }
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

bool fillJob(const mtc_job_desc &d, JobData &J) {
  const mtc_scene_view *v = &d.scene;
  if (v->struct_size != sizeof(mtc_scene_view) || !v->bvh || !v->instances || !v->attributes || !v->materials ||
      v->material_count == 0 || !v->energy_lut || !v->light_sampling || v->vertex_layout.stride < 4 ||
      (v->vertex_layout.uv_offset && (v->vertex_layout.uv_offset < 3 || v->vertex_layout.uv_offset + 2 > v->vertex_layout.stride)) ||
      (v->vertex_layout.uv1_offset && (v->vertex_layout.uv1_offset < 3 || v->vertex_layout.uv1_offset + 2 > v->vertex_layout.stride)) ||
      (v->vertex_layout.color_offset &&
       (v->vertex_layout.color_offset < 3 ||
        v->vertex_layout.color_offset + (v->vertex_layout.color_float ? 3u : 1u) > v->vertex_layout.stride)))
    return false;
  float w = d.uniform.output_size[0], h = d.uniform.output_size[1];
  if (!(w >= 1.0f && h >= 1.0f && w <= 65536.0f && h <= 65536.0f) || d.uniform.loop_unroll_guard != 4u) return false;
  if (!d.out.color || !d.out.normal || !d.out.albedo || !d.out.shadow_catcher) return false;
  std::memset(&J, 0, sizeof(J));
  J.s.bvh = (const float4 *)v->bvh;
  J.s.ins = (const float4 *)v->instances;
  J.s.attr = (const uint32_t *)v->attributes;
  J.s.mats = (const float4 *)v->materials;
  J.s.env = (const float4 *)v->env_map;
  J.s.envDist = (const float2 *)v->env_distribution;
  J.s.lightData = (const float4 *)v->light_sampling;
  J.s.lut = (const float *)v->energy_lut;
  J.s.lights = (const float4 *)v->analytic_lights;
  J.s.envW = v->env_width;
  J.s.envH = v->env_height;
  J.s.vstride = v->vertex_layout.stride;
  J.s.vnormalOff = v->vertex_layout.normal_offset;
  J.s.vnormalFloat = v->vertex_layout.normal_float;
  J.s.flags = v->flags;
  J.s.insCount = v->instance_count;
  J.s.matCount = v->material_count;
  J.s.maps = (const float4 *)v->maps;
  J.s.mapTexels = (const float4 *)v->map_texels;
  J.s.mapCount = v->maps && v->map_texels ? v->map_count : 0;
  J.s.mapTexelCount = v->map_texel_count;
  J.s.vuvOff = v->vertex_layout.uv_offset;
  J.s.vcolorOff = v->vertex_layout.color_offset;
  J.s.vuv1Off = v->vertex_layout.uv1_offset;
  J.s.triMats = v->triangle_materials;
  J.s.vcolorFloat = v->vertex_layout.color_float;
  J.u = d.uniform;
  J.cam = d.camera;
  J.outColor = (float4 *)d.out.color;
  J.outNormal = (float4 *)d.out.normal;
  J.outAlbedo = (float4 *)d.out.albedo;
  J.outCatcher = (float4 *)d.out.shadow_catcher;
  J.samples = d.samples;
  J.width = uint32_t(w);
  J.height = uint32_t(h);
  J.tilesX = (J.width + kWarpTileW - 1) / kWarpTileW;
  J.tilesY = (J.height + kWarpTileH - 1) / kWarpTileH;
  J.items = d.samples ? J.tilesX * J.tilesY : 0;
  return true;
}

}  // namespace

extern "C" mt_status mtc_trace_batch_noalloc(const mtc_job_desc *jobs, uint32_t job_count,
                                             const mtc_batch_config *config, uint32_t *status_out,
                                             mtc_counters *counters, void *stream) {
  if (!jobs && job_count) return MT_ERROR_INVALID_ARGUMENT;
  if (job_count > MTC_BATCH_NOALLOC_MAX_JOBS) return MT_ERROR_INVALID_ARGUMENT;  // beyond the fixed scratch
  if (config && config->struct_size != sizeof(mtc_batch_config)) return MT_ERROR_INVALID_ARGUMENT;
  if (job_count == 0) return MT_OK;
  // The table is assembled in host stack memory: no allocation on either side.
  JobData table[MTC_BATCH_NOALLOC_MAX_JOBS];
  uint64_t total = 0;
  for (uint32_t j = 0; j < job_count; j++) {
    if (!fillJob(jobs[j], table[j])) return MT_ERROR_INVALID_ARGUMENT;
    table[j].firstItem = uint32_t(total);
    total += table[j].items;
  }
  if (total >= 0xffffffffull) return MT_ERROR_INVALID_ARGUMENT;
  void *scratch = nullptr;
  cudaError_t e = scratchAddress(&scratch);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver ? MT_ERROR_UNAVAILABLE : MT_ERROR;
  }
  cudaStream_t st = (cudaStream_t)stream;
  uint32_t *queue = (uint32_t *)((char *)scratch + kTableBytes);
  // The table is overwritten and the queue counter cleared on every call.
  e = cudaMemcpyAsync(scratch, table, size_t(job_count) * sizeof(JobData), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(queue, 0, 256, st);
  if (e == cudaSuccess && status_out) e = cudaMemsetAsync(status_out, 0, sizeof(uint32_t), st);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return MT_ERROR;
  }
  int device = 0, sms = 148;
  cudaGetDevice(&device);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  uint32_t ctasPerSm = config && config->ctas_per_sm ? config->ctas_per_sm : 4u;
  uint32_t flagsUnion = 0;
  for (uint32_t j = 0; j < job_count; j++) flagsUnion |= jobs[j].scene.flags;
  const uint32_t grid = uint32_t(sms) * ctasPerSm;
  if (flagsUnion & MTC_SCENE_BLAS_GPU_LAYOUT)
    k_batch_noalloc<true><<<grid, 128, 0, st>>>((const JobData *)scratch, job_count, uint32_t(total), queue, counters);
  else
    k_batch_noalloc<false><<<grid, 128, 0, st>>>((const JobData *)scratch, job_count, uint32_t(total), queue, counters);
  e = cudaGetLastError();
  return e == cudaSuccess ? MT_OK : MT_ERROR;
}
