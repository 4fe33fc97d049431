// Job validation, job-table layout and the persistent work loop shared by the
// batched entry points (mtc_batch_prepare / mtc_batch_launch / mtc_trace_batch
// in megakernel.cu and mtc_trace_batch_noalloc in batch_noalloc.cu), so that
// every entry point accepts exactly the same jobs and launch shapes.
#pragma once
#include <cuda_runtime.h>

#include <cstring>

#include "dev_shade.cuh"

namespace mt {

// Header of a batched job table (host table and device copy alike); the
// JobData entries follow at kBatchTableOffset.  The kernels read the job
// count, item total and tile width from it, so a captured launch can be
// replayed after the host table is rewritten with other jobs.
struct BatchHeader {
  uint32_t jobCount, totalItems, tileW, flagsUnion, _pad[60];
};
static_assert(sizeof(BatchHeader) == 256, "batch header size");
constexpr size_t kBatchTableOffset = sizeof(BatchHeader);
// Work items of one table stay below this, so a queue counter that every
// warp advances once past the total cannot wrap.
constexpr uint64_t kBatchMaxItems = 0x7fffffffull;

// Bit set in a batched launch's status word when a warp's work loop ran out
// of iterations before the queue counter passed the item total (cannot
// happen while the counter only grows; reported instead of spinning).
constexpr uint32_t kBatchStatusGuardExhausted = MTC_BATCH_STATUS_GUARD_EXHAUSTED;

// A scene view the kernels can read: every mandatory binding present and
// every vertex-layout field inside the vertex record.
inline bool validScene(const mtc_scene_view *s) {
  return s && s->struct_size == sizeof(mtc_scene_view) && s->bvh && s->instances && s->attributes && s->materials &&
         s->material_count > 0 && s->energy_lut && s->light_sampling &&
         s->vertex_layout.stride >= 4 && s->vertex_layout.normal_offset + (s->vertex_layout.normal_float ? 3u : 1u) <=
                                             s->vertex_layout.stride &&
         (s->vertex_layout.uv_offset == 0 || (s->vertex_layout.uv_offset >= 3 &&
                                              s->vertex_layout.uv_offset + 2 <= s->vertex_layout.stride)) &&
         (s->vertex_layout.uv1_offset == 0 || (s->vertex_layout.uv1_offset >= 3 &&
                                               s->vertex_layout.uv1_offset + 2 <= s->vertex_layout.stride)) &&
         (s->vertex_layout.color_offset == 0 ||
          (s->vertex_layout.color_offset >= 3 &&
           s->vertex_layout.color_offset + (s->vertex_layout.color_float ? 3u : 1u) <= s->vertex_layout.stride));
}

inline bool validUniform(const mtc_trace_uniform *u) {
  if (!u) return false;
  float w = u->output_size[0], h = u->output_size[1];
  return w >= 1.0f && h >= 1.0f && w <= 65536.0f && h <= 65536.0f && u->loop_unroll_guard == 4u;
}

inline bool validOutputs(const mtc_outputs *o) {
  return o && o->color && o->normal && o->albedo && o->shadow_catcher;
}

inline DevScene toDev(const mtc_scene_view *v) {
  DevScene s;
  s.bvh = (const float4 *)v->bvh;
  s.ins = (const float4 *)v->instances;
  s.attr = (const uint32_t *)v->attributes;
  s.mats = (const float4 *)v->materials;
  s.env = (const float4 *)v->env_map;
  s.envDist = (const float2 *)v->env_distribution;
  s.lightData = (const float4 *)v->light_sampling;
  s.lut = (const float *)v->energy_lut;
  s.lights = (const float4 *)v->analytic_lights;
  s.envW = v->env_width;
  s.envH = v->env_height;
  s.vstride = v->vertex_layout.stride;
  s.vnormalOff = v->vertex_layout.normal_offset;
  s.vnormalFloat = v->vertex_layout.normal_float;
  s.flags = v->flags;
  s.insCount = v->instance_count;
  s.matCount = v->material_count;
  s.maps = (const float4 *)v->maps;
  s.mapTexels = (const float4 *)v->map_texels;
  s.mapCount = v->maps && v->map_texels ? v->map_count : 0;
  s.mapTexelCount = v->map_texel_count;
  s.vuvOff = v->vertex_layout.uv_offset;
  s.vcolorOff = v->vertex_layout.color_offset;
  s.vuv1Off = v->vertex_layout.uv1_offset;
  s.triMats = v->triangle_materials;
  s.vcolorFloat = v->vertex_layout.color_float;
  return s;
}

// One job's table entry for warp tiles of tileW x (32 / tileW) pixels.
inline JobData makeJob(const mtc_scene_view *scene, const mtc_camera_uniform *camera,
                       const mtc_trace_uniform *uniform, const mtc_outputs *out, uint32_t samples,
                       uint32_t tileW = 8u) {
  JobData J;
  std::memset(&J, 0, sizeof(J));
  J.s = toDev(scene);
  J.u = *uniform;
  J.cam = *camera;
  J.outColor = (float4 *)out->color;
  J.outNormal = (float4 *)out->normal;
  J.outAlbedo = (float4 *)out->albedo;
  J.outCatcher = (float4 *)out->shadow_catcher;
  J.samples = samples;
  J.width = uint32_t(uniform->output_size[0]);
  J.height = uint32_t(uniform->output_size[1]);
  const uint32_t tileH = 32u / tileW;
  J.tilesX = (J.width + tileW - 1) / tileW;
  J.tilesY = (J.height + tileH - 1) / tileH;
  J.items = samples ? J.tilesX * J.tilesY : 0u;
  return J;
}

// Resident CTAs of 128 threads per SM the persistent batched kernels are
// compiled for (32 registers; the default grid fills them): like the plain
// kernel, latency-bound, so more warps beat fewer spills.
#ifndef MT_BATCH_MIN_BLOCKS
#define MT_BATCH_MIN_BLOCKS 16
#endif

struct BatchShape {
  uint32_t blockThreads, tileW, tileH, ctasPerSm, grain;
};
// Resolves a (possibly NULL) mtc_batch_config to launch parameters; false for
// out-of-range values.
inline bool batchShape(const mtc_batch_config *c, BatchShape &out) {
  out = BatchShape{128u, 8u, 4u, uint32_t(MT_BATCH_MIN_BLOCKS), 1u};
  if (!c) return true;
  if (c->struct_size != sizeof(mtc_batch_config)) return false;
  if (c->block_threads) {
    if (c->block_threads > 128u || c->block_threads % 32u) return false;
    out.blockThreads = c->block_threads;
  }
  if (c->tile_width) {
    if (c->tile_width > 32u || (32u % c->tile_width)) return false;
    out.tileW = c->tile_width;
    out.tileH = 32u / c->tile_width;
  }
  if (c->ctas_per_sm) {
    if (c->ctas_per_sm > 32u) return false;
    out.ctasPerSm = c->ctas_per_sm;
  }
  if (c->items_per_fetch) {
    if (c->items_per_fetch > 16u) return false;
    out.grain = c->items_per_fetch;
  }
  return true;
}

// Writes the header and `job_count` entries of a job table to host memory
// `base` (kBatchTableOffset + job_count * sizeof(JobData) bytes).
inline mt_status writeBatchTable(const mtc_job_desc *jobs, uint32_t job_count, const BatchShape &shape, void *base,
                                 uint32_t *total_items) {
  char *out = static_cast<char *>(base);
  uint64_t total = 0;
  uint32_t flagsUnion = 0;
  for (uint32_t j = 0; j < job_count; j++) {
    const mtc_job_desc &d = jobs[j];
    if (!validScene(&d.scene) || !validUniform(&d.uniform) || !validOutputs(&d.out))
      return MT_ERROR_INVALID_ARGUMENT;
    JobData J = makeJob(&d.scene, &d.camera, &d.uniform, &d.out, d.samples, shape.tileW);
    J.firstItem = uint32_t(total);
    total += J.items;
    if (total >= kBatchMaxItems) return MT_ERROR_INVALID_ARGUMENT;
    flagsUnion |= d.scene.flags;
    std::memcpy(out + kBatchTableOffset + size_t(j) * sizeof(JobData), &J, sizeof(J));
  }
  BatchHeader h;
  std::memset(&h, 0, sizeof(h));
  h.jobCount = job_count;
  h.totalItems = uint32_t(total);
  h.tileW = shape.tileW;
  h.flagsUnion = flagsUnion;
  std::memcpy(out, &h, sizeof(h));
  if (total_items) *total_items = uint32_t(total);
  return MT_OK;
}

// The persistent work loop of the batched kernels.  queue[0] is the next
// work item; items are warp tiles (tileW x 32/tileW pixels) laid out job
// after job (JobData.firstItem / .items).  A warp takes `grain` consecutive
// items per atomic and runs every sample of each tile's pixels in order.
// The loop ends when the counter passes the item total, so every warp exits;
// its iteration bound only guards against a corrupted table, and running
// out of it sets kBatchStatusGuardExhausted in `status` (when given).
template <bool kGpuLayout>
__device__ __forceinline__ void batchWorkLoop(const BatchHeader *__restrict__ header, uint32_t *queue, uint32_t grain,
                                              uint32_t *status, Counters &cnt, uint32_t &paths) {
  const JobData *__restrict__ jobs =
      reinterpret_cast<const JobData *>(reinterpret_cast<const char *>(header) + kBatchTableOffset);
  const uint32_t job_count = header->jobCount, total_items = header->totalItems, tileW = header->tileW;
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t lx = lane % tileW, ly = lane / tileW, tileH = 32u / tileW;
  bool done = false;
  for (uint32_t guard = 0; guard < total_items + 1u; guard++) {
    uint32_t first = 0;
    if (lane == 0) first = atomicAdd(queue, grain);
    first = __shfl_sync(0xffffffffu, first, 0);
    if (first >= total_items) {
      done = true;
      break;
    }
    const uint32_t last = min(first + grain, total_items);
    uint32_t j = 0;
    for (uint32_t item = first; item < last; item++) {
      // Jobs are few; a forward scan of the prefix table finds the owner.
      while (j + 1 < job_count && jobs[j + 1].firstItem <= item) j++;
      const JobData &J = jobs[j];
      uint32_t local = item - J.firstItem;
      uint32_t tx = local % J.tilesX, ty = local / J.tilesX;
      uint32_t x = tx * tileW + lx, y = ty * tileH + ly;
      if (x < J.width && y < J.height) {
        tracePixelSamples<kGpuLayout>(J, x, y, J.samples, cnt);
        paths += J.samples;
      }
    }
  }
  if (!done && status && lane == 0) atomicOr(status, kBatchStatusGuardExhausted);
}

}  // namespace mt
