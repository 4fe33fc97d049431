// sm_100a kernels of the path tracer and their C-ABI entry points:
//  - k_trace:      plain megakernel, one thread per pixel, all requested
//                  samples of that pixel in order (the progressive pass of
//                  rayTrace.compute.ts:1157-1263 repeated `samples` times);
//  - k_batch:      persistent multi-job megakernel; each warp pulls
//                  (job, 32-pixel tile) work items from one global counter
//                  and runs every sample of its tile in order, so a job's
//                  image is bit-identical alone and in a batch;
//  - k_first_hit:  querySceneSoftware (intersect.wgsl.ts:660-684);
//  - k_sample_maps: raw material-map lookups (sampleMap) for parity checks;
//  - k_refit_*:    TLAS refit (bvhAccel.ts:579-740) on the device.
#include <cuda_runtime.h>
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <vector>

#include "batch_table.cuh"
#include "js_minmax.h"

using namespace mt;

namespace {

// 8x16 pixels per CTA, so a warp covers an 8x4 block (measured 0.5 % faster
// than 16x2 warps, 1 % faster than 32x1).
#ifndef MT_TRACE_TILE_W
#define MT_TRACE_TILE_W 8
#endif
constexpr int kTileW = MT_TRACE_TILE_W, kTileH = 128 / MT_TRACE_TILE_W;  // plain kernel CTA tile

__device__ __forceinline__ void flushCounters(const Counters &cnt, uint32_t paths, mtc_counters *out) {
  if (!out) return;
  if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) atomicAdd(&out->kernel_launches, 1ull);
  unsigned mask = __activemask();
  uint32_t e = __reduce_add_sync(mask, cnt.ext);
  uint32_t s = __reduce_add_sync(mask, cnt.shadow);
  uint32_t p = __reduce_add_sync(mask, paths);
  int leader = __ffs(mask) - 1;
  if ((threadIdx.x & 31) == leader) {
    atomicAdd(&out->extension_rays, (unsigned long long)e);
    atomicAdd(&out->shadow_rays, (unsigned long long)s);
    atomicAdd(&out->path_samples, (unsigned long long)p);
  }
}

// The plain kernel at 16 CTAs of 128 threads per SM (full occupancy, 32
// registers): it is bound by dependent-load latency, and the warps hide more
// of it than the spilled state costs (measured 11 % faster than 2 CTAs at
// 255 registers; 4, 8 and 12 CTAs in between).
#ifndef MT_TRACE_MIN_BLOCKS
#define MT_TRACE_MIN_BLOCKS 16
#endif
template <bool kGpuLayout>
__global__ void __launch_bounds__(kTileW *kTileH, MT_TRACE_MIN_BLOCKS)
    k_trace(const __grid_constant__ JobData J, uint32_t samples, mtc_counters *counters) {
  uint32_t lx = threadIdx.x % kTileW, ly = threadIdx.x / kTileW;
  uint32_t x = blockIdx.x * kTileW + lx, y = blockIdx.y * kTileH + ly;
  Counters cnt;
  uint32_t paths = 0;
  if (x < J.width && y < J.height) {
    tracePixelSamples<kGpuLayout>(J, x, y, samples, cnt);
    paths = samples;
  }
  flushCounters(cnt, paths, counters);
}

// Persistent batched kernel over a job table (batch_table.cuh).
template <bool kGpuLayout>
__global__ void __launch_bounds__(128, MT_BATCH_MIN_BLOCKS)
    k_batch(const BatchHeader *__restrict__ header, uint32_t *queue, mtc_counters *counters, uint32_t grain,
            uint32_t *status) {
  Counters cnt;
  uint32_t paths = 0;
  batchWorkLoop<kGpuLayout>(header, queue, grain, status, cnt, paths);
  flushCounters(cnt, paths, counters);
}

__global__ void k_sample_maps(const __grid_constant__ DevScene s, const int32_t *indices, const float2 *uvs,
                              uint32_t count, float4 *out) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const float2 uv = uvs[i];
  out[i] = sampleMap(s, indices[i], V2{uv.x, uv.y});
}

template <bool kGpuLayout>
__global__ void k_first_hit(const __grid_constant__ DevScene s, int32_t blasBase, int32_t isEmpty, const float4 *rays,
                            uint32_t count, mtc_hit *hits) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  float4 o4 = rays[size_t(i) * 2], d4 = rays[size_t(i) * 2 + 1];
  mtc_hit out;
  out.hit = 0; out.instance = -1; out.record = -1; out.t = RAY_MAX_DISTANCE;
  out.barycentric[0] = 0; out.barycentric[1] = 0; out.barycentric[2] = 0; out._pad = 0;
  if (!isEmpty) {
    TraversalHit h;
    h.tMax = RAY_MAX_DISTANCE;
    h.triangleIndex = -1;
    h.insIdx = -1;
    h.hitBary = v3(0.0f);
    traverse<false, kGpuLayout>(s, blasBase, xyz(o4), xyz(d4), 0, false, -1, -1, h);
    if (h.insIdx >= 0) {
      out.hit = 1; out.instance = h.insIdx; out.record = h.triangleIndex; out.t = h.tMax;
      out.barycentric[0] = h.hitBary.x; out.barycentric[1] = h.hitBary.y; out.barycentric[2] = h.hitBary.z;
    }
  }
  hits[i] = out;
}

// read_average (native/host/src/lib.rs:343-364): each f32 of an accumulation
// buffer divided by the completed sample count; any non-finite result raises
// the flag.  HBM-bound: 16 B read + 16 B written per pixel.
__global__ void k_average(const float4 *__restrict__ in, uint32_t pixels, float samples, float4 *__restrict__ out,
                          uint32_t *nonFinite) {
  bool bad = false;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < pixels; i += gridDim.x * blockDim.x) {
    float4 a = in[i];
    float4 r = make_float4(__fdiv_rn(a.x, samples), __fdiv_rn(a.y, samples), __fdiv_rn(a.z, samples),
                           __fdiv_rn(a.w, samples));
    bad |= !isfinite(r.x) || !isfinite(r.y) || !isfinite(r.z) || !isfinite(r.w);
    out[i] = r;
  }
  if (__any_sync(__activemask(), bad) && bad) atomicOr(nonFinite, 1u);
}

// ------------------------------------------------------------------ refit
// One thread per TLAS leaf entry: world bounds of the instance's BLAS box
// (computeBounds, scenePreparation.ts:19-47) and its instance record
// (writeInstanceRecord, bvhAccel.ts:330-353), both in float64 as the
// reference computes them and stored as f32.
__device__ void instanceBoundsD(const double *m, const float *local, float *out) {
  float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int corner = 0; corner < 8; corner++) {
    double x = (corner & 1) ? local[3] : local[0];
    double y = (corner & 2) ? local[4] : local[1];
    double z = (corner & 4) ? local[5] : local[2];
    double w = __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(m[3], x), __dmul_rn(m[7], y)), __dmul_rn(m[11], z)), m[15]);
    if (w == 0.0 || w != w) w = 1.0;
    float p[3];
    for (int k = 0; k < 3; k++) {
      double v = __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(m[k], x), __dmul_rn(m[4 + k], y)), __dmul_rn(m[8 + k], z)), m[12 + k]);
      p[k] = __double2float_rn(__ddiv_rn(v, w));
    }
    if (!isfinite(p[0]) || !isfinite(p[1]) || !isfinite(p[2])) continue;
    for (int k = 0; k < 3; k++) { mn[k] = jsMin(mn[k], p[k]); mx[k] = jsMax(mx[k], p[k]); }
  }
  for (int k = 0; k < 3; k++) { out[k] = mn[k]; out[3 + k] = mx[k]; }
}

#define DM(a, b) __dmul_rn(a, b)
#define DA(a, b) __dadd_rn(a, b)
#define DS(a, b) __dsub_rn(a, b)
__device__ bool invert4D(const double *a, double *o) {
  double a00 = a[0], a01 = a[1], a02 = a[2], a03 = a[3], a10 = a[4], a11 = a[5], a12 = a[6], a13 = a[7];
  double a20 = a[8], a21 = a[9], a22 = a[10], a23 = a[11], a30 = a[12], a31 = a[13], a32 = a[14], a33 = a[15];
  double b00 = DS(DM(a00, a11), DM(a01, a10)), b01 = DS(DM(a00, a12), DM(a02, a10)), b02 = DS(DM(a00, a13), DM(a03, a10));
  double b03 = DS(DM(a01, a12), DM(a02, a11)), b04 = DS(DM(a01, a13), DM(a03, a11)), b05 = DS(DM(a02, a13), DM(a03, a12));
  double b06 = DS(DM(a20, a31), DM(a21, a30)), b07 = DS(DM(a20, a32), DM(a22, a30)), b08 = DS(DM(a20, a33), DM(a23, a30));
  double b09 = DS(DM(a21, a32), DM(a22, a31)), b10 = DS(DM(a21, a33), DM(a23, a31)), b11 = DS(DM(a22, a33), DM(a23, a32));
  double det = DA(DS(DA(DA(DS(DM(b00, b11), DM(b01, b10)), DM(b02, b09)), DM(b03, b08)), DM(b04, b07)), DM(b05, b06));
  if (det == 0.0) return false;
  det = __ddiv_rn(1.0, det);
  o[0] = DM(DA(DS(DM(a11, b11), DM(a12, b10)), DM(a13, b09)), det);
  o[1] = DM(DS(DS(DM(a02, b10), DM(a01, b11)), DM(a03, b09)), det);
  o[2] = DM(DA(DS(DM(a31, b05), DM(a32, b04)), DM(a33, b03)), det);
  o[3] = DM(DS(DS(DM(a22, b04), DM(a21, b05)), DM(a23, b03)), det);
  o[4] = DM(DS(DS(DM(a12, b08), DM(a10, b11)), DM(a13, b07)), det);
  o[5] = DM(DA(DS(DM(a00, b11), DM(a02, b08)), DM(a03, b07)), det);
  o[6] = DM(DS(DS(DM(a32, b02), DM(a30, b05)), DM(a33, b01)), det);
  o[7] = DM(DA(DS(DM(a20, b05), DM(a22, b02)), DM(a23, b01)), det);
  o[8] = DM(DA(DS(DM(a10, b10), DM(a11, b08)), DM(a13, b06)), det);
  o[9] = DM(DS(DS(DM(a01, b08), DM(a00, b10)), DM(a03, b06)), det);
  o[10] = DM(DA(DS(DM(a30, b04), DM(a31, b02)), DM(a33, b00)), det);
  o[11] = DM(DS(DS(DM(a21, b02), DM(a20, b04)), DM(a23, b00)), det);
  o[12] = DM(DS(DS(DM(a11, b07), DM(a10, b09)), DM(a12, b06)), det);
  o[13] = DM(DA(DS(DM(a00, b09), DM(a01, b07)), DM(a02, b06)), det);
  o[14] = DM(DS(DS(DM(a31, b01), DM(a30, b03)), DM(a32, b00)), det);
  o[15] = DM(DA(DS(DM(a20, b03), DM(a21, b01)), DM(a22, b00)), det);
  return true;
}

// Refits leaves: writes each leaf node's union box and its instance records.
__global__ void k_refit_leaves(float4 *tlas, uint32_t nodeVec4, float *records, const double *transforms,
                               const float *localBounds, const int32_t *blasOffsets, const int32_t *blasLayouts,
                               const int32_t *vertexOffsets, const int32_t *materials, const float *colors,
                               const int32_t *leafNodes, uint32_t leafCount) {
  uint32_t l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= leafCount) return;
  int32_t node = leafNodes[l];
  if (node < 0 || uint32_t(node) + 1 >= nodeVec4) return;
  float4 n0 = tlas[node];
  int32_t count = -__float_as_int(n0.w);
  float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int32_t i = 0; i < count; i++) {
    float4 entry = tlas[node + 2 + i];
    int32_t target = __float_as_int(entry.x), source = __float_as_int(entry.z);
    const double *m = transforms + size_t(source) * 16;
    float b[6];
    instanceBoundsD(m, localBounds + size_t(source) * 6, b);
    for (int k = 0; k < 3; k++) { mn[k] = jsMin(mn[k], b[k]); mx[k] = jsMax(mx[k], b[3 + k]); }
    float *rec = records + size_t(target) * 40;
    uint32_t encoded = uint32_t(blasOffsets[source]) | (uint32_t(blasLayouts[source]) << 30);
    rec[0] = __int_as_float(int32_t(encoded));
    rec[1] = __int_as_float(vertexOffsets[source]);
    rec[2] = __int_as_float(materials[source]);
    rec[3] = 0.0f;
    rec[36] = colors[source * 3]; rec[37] = colors[source * 3 + 1]; rec[38] = colors[source * 3 + 2]; rec[39] = 0.0f;
    double inv[16];
    if (!invert4D(m, inv)) for (int k = 0; k < 16; k++) inv[k] = 0.0;
    for (int k = 0; k < 16; k++) {
      rec[4 + k] = __double2float_rn(inv[k]);
      rec[20 + k] = __double2float_rn(m[k]);
    }
  }
  tlas[node] = make_float4(mn[0], mn[1], mn[2], n0.w);
  float4 n1 = tlas[node + 1];
  tlas[node + 1] = make_float4(mx[0], mx[1], mx[2], n1.w);
}

// Interior nodes of one depth level: union of the two children.
__global__ void k_refit_level(float4 *tlas, const int32_t *nodes, uint32_t count) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  int32_t node = nodes[i];
  float4 a = tlas[node], b = tlas[node + 1];
  int32_t right = __float_as_int(a.w);
  float4 l0 = tlas[node + 2], l1 = tlas[node + 3], r0 = tlas[right], r1 = tlas[right + 1];
  tlas[node] = make_float4(jsMin(l0.x, r0.x), jsMin(l0.y, r0.y), jsMin(l0.z, r0.z), a.w);
  tlas[node + 1] = make_float4(jsMax(l1.x, r1.x), jsMax(l1.y, r1.y), jsMax(l1.z, r1.z), b.w);
}

// -------------------------------------------------------------- host glue
mt_status cudaStatus(cudaError_t e) {
  if (e == cudaSuccess) return MT_OK;
  if (e == cudaErrorInvalidValue || e == cudaErrorInvalidDevicePointer) return MT_ERROR_INVALID_ARGUMENT;
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return MT_ERROR_UNAVAILABLE;
  return MT_ERROR;
}

}  // namespace

extern "C" {

uint32_t mtc_abi_version(void) { return MTC_ABI_VERSION; }

mt_status mtc_trace_samples(const mtc_scene_view *scene, const mtc_camera_uniform *camera,
                            const mtc_trace_uniform *uniform, const mtc_outputs *out, uint32_t samples,
                            mtc_counters *counters, void *stream) {
  if (!validScene(scene) || !camera || !validUniform(uniform) || !validOutputs(out))
    return MT_ERROR_INVALID_ARGUMENT;
  if (samples == 0) return MT_OK;
  JobData J = makeJob(scene, camera, uniform, out, samples);
  dim3 grid((J.width + kTileW - 1) / kTileW, (J.height + kTileH - 1) / kTileH);
  if (scene->flags & MTC_SCENE_BLAS_GPU_LAYOUT)
    k_trace<true><<<grid, kTileW * kTileH, 0, (cudaStream_t)stream>>>(J, samples, counters);
  else
    k_trace<false><<<grid, kTileW * kTileH, 0, (cudaStream_t)stream>>>(J, samples, counters);
  return cudaStatus(cudaGetLastError());
}

mt_status mtc_query_first_hit(const mtc_scene_view *scene, const float *rays, uint32_t count, mtc_hit *hits,
                              void *stream) {
  if (!validScene(scene) || (!rays && count) || (!hits && count)) return MT_ERROR_INVALID_ARGUMENT;
  if (count == 0) return MT_OK;
  int32_t blasBase = scene->blas_offset;
  if (scene->flags & MTC_SCENE_BLAS_GPU_LAYOUT)
    k_first_hit<true><<<(count + 127) / 128, 128, 0, (cudaStream_t)stream>>>(
        toDev(scene), blasBase, scene->instance_count == 0, (const float4 *)rays, count, hits);
  else
    k_first_hit<false><<<(count + 127) / 128, 128, 0, (cudaStream_t)stream>>>(
        toDev(scene), blasBase, scene->instance_count == 0, (const float4 *)rays, count, hits);
  return cudaStatus(cudaGetLastError());
}

mt_status mtc_sample_maps(const mtc_scene_view *scene, const int32_t *indices, const float *uvs, uint32_t count,
                          float *texels, void *stream) {
  if (!validScene(scene) || (count && (!indices || !uvs || !texels))) return MT_ERROR_INVALID_ARGUMENT;
  if (count == 0) return MT_OK;
  k_sample_maps<<<(count + 127) / 128, 128, 0, (cudaStream_t)stream>>>(toDev(scene), indices, (const float2 *)uvs,
                                                                      count, (float4 *)texels);
  return cudaStatus(cudaGetLastError());
}

mt_status mtc_average_output(const void *accum, uint32_t pixels, uint32_t samples, void *out,
                             uint32_t *nonfinite_flag, void *stream) {
  if (!accum || !out || !nonfinite_flag || samples == 0) return MT_ERROR_INVALID_ARGUMENT;
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e = cudaMemsetAsync(nonfinite_flag, 0, sizeof(uint32_t), st);
  if (e != cudaSuccess) return cudaStatus(e);
  if (pixels == 0) return MT_OK;
  int device = 0, sms = 148;
  cudaGetDevice(&device);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  uint32_t grid = std::min<uint32_t>((pixels + 255) / 256, uint32_t(sms) * 8u);
  k_average<<<grid, 256, 0, st>>>((const float4 *)accum, pixels, float(samples), (float4 *)out, nonfinite_flag);
  return cudaStatus(cudaGetLastError());
}

size_t mtc_batch_table_bytes(uint32_t capacity) { return kBatchTableOffset + size_t(capacity) * sizeof(JobData); }

size_t mtc_batch_scratch_bytes(uint32_t capacity) {
  return (mtc_batch_table_bytes(capacity) + 255) / 256 * 256 + 256;
}

mt_status mtc_batch_prepare(const mtc_job_desc *jobs, uint32_t job_count, const mtc_batch_config *config,
                            void *table, uint32_t *total_items) {
  if ((!jobs && job_count) || !table) return MT_ERROR_INVALID_ARGUMENT;
  BatchShape shape;
  if (!batchShape(config, shape)) return MT_ERROR_INVALID_ARGUMENT;
  return writeBatchTable(jobs, job_count, shape, table, total_items);
}

}  // extern "C"

namespace {

// Copies the host table into `queue_state`, clears the work counter and
// launches k_batch; `status` (device, may be NULL) collects the kernel's
// status bits.
mt_status launchBatch(const void *table, uint32_t capacity, const BatchShape &shape, void *queue_state,
                      uint32_t *status, mtc_counters *counters, cudaStream_t st) {
  char *scratch = (char *)queue_state;
  size_t bytes = mtc_batch_table_bytes(capacity);
  uint32_t *queue = (uint32_t *)(scratch + (bytes + 255) / 256 * 256);
  cudaError_t e = cudaMemcpyAsync(scratch, table, bytes, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(queue, 0, 256, st);
  if (e != cudaSuccess) return cudaStatus(e);
  int device = 0, sms = 148;
  e = cudaGetDevice(&device);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  if (e != cudaSuccess) return cudaStatus(e);
  // A full persistent grid: the item total is only known on the device.
  uint32_t grid = uint32_t(sms) * shape.ctasPerSm;
  // The host copy of the header decides the BLAS-layout specialisation.
  uint32_t flagsUnion = static_cast<const BatchHeader *>(table)->flagsUnion;
  if (flagsUnion & MTC_SCENE_BLAS_GPU_LAYOUT)
    k_batch<true><<<grid, shape.blockThreads, 0, st>>>((const BatchHeader *)scratch, queue, counters, shape.grain,
                                                       status);
  else
    k_batch<false><<<grid, shape.blockThreads, 0, st>>>((const BatchHeader *)scratch, queue, counters, shape.grain,
                                                        status);
  return cudaStatus(cudaGetLastError());
}

}  // namespace

extern "C" {

mt_status mtc_batch_launch(const void *table, uint32_t capacity, const mtc_batch_config *config, void *queue_state,
                           mtc_counters *counters, void *stream) {
  if (!table || !queue_state) return MT_ERROR_INVALID_ARGUMENT;
  BatchShape shape;
  if (!batchShape(config, shape)) return MT_ERROR_INVALID_ARGUMENT;
  return launchBatch(table, capacity, shape, queue_state, nullptr, counters, (cudaStream_t)stream);
}

mt_status mtc_trace_batch(const mtc_job_desc *jobs, uint32_t job_count, const mtc_batch_config *config,
                          void *queue_state, uint32_t *status_out, mtc_counters *counters, void *stream) {
  if ((!jobs && job_count) || !queue_state) return MT_ERROR_INVALID_ARGUMENT;
  BatchShape shape;
  if (!batchShape(config, shape)) return MT_ERROR_INVALID_ARGUMENT;
  if (job_count == 0) return MT_OK;
  std::vector<char> table(mtc_batch_table_bytes(job_count));
  mt_status st = writeBatchTable(jobs, job_count, shape, table.data(), nullptr);
  if (st != MT_OK) return st;
  if (status_out) {
    cudaError_t e = cudaMemsetAsync(status_out, 0, sizeof(uint32_t), (cudaStream_t)stream);
    if (e != cudaSuccess) return cudaStatus(e);
  }
  // cudaMemcpyAsync from pageable memory has finished reading the table
  // when it returns, so the vector may go out of scope.
  return launchBatch(table.data(), job_count, shape, queue_state, status_out, counters, (cudaStream_t)stream);
}

mt_status mtc_refit_tlas(void *tlas, uint64_t tlas_vec4_count, void *instances, uint32_t instance_count,
                         const double *transforms, const float *local_bounds, const int32_t *blas_offsets,
                         const int32_t *blas_layouts, const int32_t *vertex_offsets, const int32_t *materials,
                         const float *colors, void *stream) {
  if (!tlas || !instances || !transforms || !local_bounds || !blas_offsets || !blas_layouts || !vertex_offsets ||
      !materials || !colors || tlas_vec4_count < 2)
    return MT_ERROR_INVALID_ARGUMENT;
  (void)instance_count;
  // Host walk of the (device-resident) topology: the node pointers never
  // change during a refit, so copy the w words once and order nodes by depth.
  cudaStream_t st = (cudaStream_t)stream;
  std::vector<float4> nodes(tlas_vec4_count);
  cudaError_t e = cudaMemcpyAsync(nodes.data(), tlas, tlas_vec4_count * sizeof(float4), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cudaStatus(e);
  std::vector<std::vector<int32_t>> levels;
  std::vector<int32_t> leaves;
  std::vector<std::pair<int32_t, int>> stack = {{0, 0}};
  while (!stack.empty()) {
    auto [node, depth] = stack.back();
    stack.pop_back();
    if (node < 0 || uint64_t(node) + 1 >= tlas_vec4_count) return MT_ERROR_INVALID_ARGUMENT;
    int32_t w;
    std::memcpy(&w, &nodes[node].w, 4);
    if (w >= 0) {
      if (int(levels.size()) <= depth) levels.resize(depth + 1);
      levels[depth].push_back(node);
      stack.push_back({node + 2, depth + 1});
      stack.push_back({w, depth + 1});
    } else {
      leaves.push_back(node);
    }
  }
  size_t bytes = (leaves.size() + 1) * 4;
  for (auto &l : levels) bytes += (l.size() + 1) * 4;
  int32_t *dIdx = nullptr;
  e = cudaMallocAsync((void **)&dIdx, bytes, st);
  if (e != cudaSuccess) return cudaStatus(e);
  std::vector<int32_t> flat(leaves);
  for (auto &l : levels) flat.insert(flat.end(), l.begin(), l.end());
  e = cudaMemcpyAsync(dIdx, flat.data(), flat.size() * 4, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && !leaves.empty())
    k_refit_leaves<<<(uint32_t(leaves.size()) + 127) / 128, 128, 0, st>>>(
        (float4 *)tlas, uint32_t(tlas_vec4_count), (float *)instances, transforms, local_bounds, blas_offsets,
        blas_layouts, vertex_offsets, materials, colors, dIdx, uint32_t(leaves.size()));
  size_t off = leaves.size();
  std::vector<size_t> levelOff(levels.size());
  for (size_t d = 0; d < levels.size(); d++) { levelOff[d] = off; off += levels[d].size(); }
  for (int d = int(levels.size()) - 1; d >= 0 && e == cudaSuccess; d--) {
    uint32_t n = uint32_t(levels[d].size());
    if (n) k_refit_level<<<(n + 127) / 128, 128, 0, st>>>((float4 *)tlas, dIdx + levelOff[d], n);
  }
  cudaFreeAsync(dIdx, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  return cudaStatus(e == cudaSuccess ? cudaGetLastError() : e);
}

}  // extern "C"
