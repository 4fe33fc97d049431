// BLAS refit on the device: refitBLAS (src/renderer/bvhAccel.ts:800-870,
// BVH2 layout, no displacement) after vertex deformation, topology kept.
//
// The reference caches, per BLAS buffer, its nodes in post order and each
// leaf's distinct vertices (getBlasRefitData, bvhAccel.ts:758-796), then
// rewrites every node box: a leaf's box is Math.min/max over its triangles'
// vertices whose three coordinates are finite (an index past the position
// array reads `undefined` and is skipped too), an interior box is the
// Math.min/max of its two children's boxes.  Here the cached data is a plan
// of node offsets grouped by depth, built once on the device by a top-down
// walk (mtc_blas_refit_prepare); a refit then runs one kernel per depth,
// deepest first, so every child box is final before its parent reads it.
// Min/max are exact and order independent (-0 below +0), so the boxes equal
// the reference's bit for bit.  The reference also sums the nodes' surface
// areas for its rebuild hint; the device sums the same per-node terms in a
// fixed tree order (deterministic, rounding may differ from the sequential
// post-order sum in the last bits).
#include <cuda_runtime.h>

#include <cstdint>
#include <cstring>

#include "../../include/mutracer_b200.h"
#include "js_minmax.h"

namespace {

constexpr int kThreads = 256;
constexpr uint32_t kMaxLevels = 1u << 16;

// Plan layout (device): header, level starts, node offsets by level, then
// one float64 surface-area term per node.
struct PlanHeader {
  uint32_t nodeCount, levels, capacity, error;
  uint32_t pad[12];
};

struct Plan {
  PlanHeader *h;
  uint32_t *levelStart;  // levels + 1 entries
  uint32_t *nodes;       // capacity entries
  double *area;          // capacity entries
};

size_t planBytes(uint64_t vec4, Plan *p, char *base) {
  uint64_t capacity = vec4 / 2 + 1;  // a node takes at least 2 vec4
  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t o = off;
    off = (off + bytes + 255) / 256 * 256;
    return base ? base + o : nullptr;
  };
  char *h = take(sizeof(PlanHeader));
  char *ls = take(sizeof(uint32_t) * (kMaxLevels + 1));
  char *nodes = take(sizeof(uint32_t) * capacity);
  char *area = take(sizeof(double) * capacity);
  if (p) {
    p->h = reinterpret_cast<PlanHeader *>(h);
    p->levelStart = reinterpret_cast<uint32_t *>(ls);
    p->nodes = reinterpret_cast<uint32_t *>(nodes);
    p->area = reinterpret_cast<double *>(area);
  }
  return off;
}

__global__ void k_plan_init(Plan p, uint32_t capacity) {
  p.h->nodeCount = 1;
  p.h->levels = 0;
  p.h->capacity = capacity;
  p.h->error = 0;
  p.levelStart[0] = 0;
  p.levelStart[1] = 1;
  p.nodes[0] = 0;
}

// Appends the children of one depth's interior nodes as the next depth.
__global__ void k_plan_level(Plan p, const int4 *bvh, uint64_t vec4, uint32_t level) {
  const uint32_t begin = p.levelStart[level], end = p.levelStart[level + 1];
  for (uint32_t i = begin + blockIdx.x * blockDim.x + threadIdx.x; i < end; i += gridDim.x * blockDim.x) {
    const uint32_t o = p.nodes[i];
    if (uint64_t(o) + 2 > vec4) {
      p.h->error = 1;
      continue;
    }
    const int32_t w = bvh[o].w;
    if (w < 0) {
      if (uint64_t(o) + 2 + uint64_t(-int64_t(w)) > vec4) p.h->error = 1;
      continue;
    }
    if (uint64_t(w) + 2 > vec4 || uint32_t(w) <= o + 2) {  // children lie after their parent in DFS order
      p.h->error = 1;
      continue;
    }
    uint32_t slot = atomicAdd(&p.h->nodeCount, 2u);
    if (slot + 2 > p.h->capacity) {
      p.h->error = 1;
      continue;
    }
    p.nodes[slot] = o + 2;
    p.nodes[slot + 1] = uint32_t(w);
  }
}

__global__ void k_plan_close_level(Plan p, uint32_t level) {
  p.levelStart[level + 2] = min(p.h->nodeCount, p.h->capacity);
  p.h->levels = level + 1;
}

// One depth of refitBLAS (bvhAccel.ts:832-868): leaves from their vertices,
// interior nodes from their (already refitted) children.
__global__ void __launch_bounds__(kThreads) k_refit_blas_level(Plan p, float4 *bvh, uint32_t level,
                                                               const float *pos, uint32_t vertexCount) {
  const uint32_t begin = p.levelStart[level], end = p.levelStart[level + 1];
  for (uint32_t i = begin + blockIdx.x * blockDim.x + threadIdx.x; i < end; i += gridDim.x * blockDim.x) {
    const uint32_t o = p.nodes[i];
    float4 a = bvh[o], b = bvh[o + 1];
    const int32_t w = __float_as_int(a.w);
    float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    if (w >= 0) {
      const float4 l0 = bvh[o + 2], l1 = bvh[o + 3], r0 = bvh[w], r1 = bvh[w + 1];
      mn[0] = jsMin(l0.x, r0.x); mn[1] = jsMin(l0.y, r0.y); mn[2] = jsMin(l0.z, r0.z);
      mx[0] = jsMax(l1.x, r1.x); mx[1] = jsMax(l1.y, r1.y); mx[2] = jsMax(l1.z, r1.z);
    } else {
      for (int32_t t = 0; t < -w; t++) {
        const int4 rec = reinterpret_cast<const int4 *>(bvh)[o + 2 + t];
        const uint32_t v[3] = {uint32_t(rec.x), uint32_t(rec.y), uint32_t(rec.z)};
        for (int c = 0; c < 3; c++) {
          if (v[c] >= vertexCount) continue;
          const float x = pos[size_t(v[c]) * 3], y = pos[size_t(v[c]) * 3 + 1], z = pos[size_t(v[c]) * 3 + 2];
          if (!isfinite(x) || !isfinite(y) || !isfinite(z)) continue;
          mn[0] = jsMin(mn[0], x); mn[1] = jsMin(mn[1], y); mn[2] = jsMin(mn[2], z);
          mx[0] = jsMax(mx[0], x); mx[1] = jsMax(mx[1], y); mx[2] = jsMax(mx[2], z);
        }
      }
    }
    bvh[o] = make_float4(mn[0], mn[1], mn[2], a.w);
    bvh[o + 1] = make_float4(mx[0], mx[1], mx[2], b.w);
    // 2 * (x * z + x * y + z * y) in float64 (bvhAccel.ts:863-864).
    const double x = __dadd_rn(double(mx[0]), -double(mn[0])), y = __dadd_rn(double(mx[1]), -double(mn[1]));
    const double z = __dadd_rn(double(mx[2]), -double(mn[2]));
    p.area[i] = __dmul_rn(2.0, __dadd_rn(__dadd_rn(__dmul_rn(x, z), __dmul_rn(x, y)), __dmul_rn(z, y)));
  }
}

// Deterministic sum of the per-node terms (fixed strided order, then a fixed
// tree), one CTA.
__global__ void __launch_bounds__(1024) k_area_sum(Plan p, double *out) {
  __shared__ double part[1024];
  const uint32_t n = p.h->nodeCount < p.h->capacity ? p.h->nodeCount : p.h->capacity;
  double s = 0.0;
  for (uint32_t i = threadIdx.x; i < n; i += 1024) s = __dadd_rn(s, p.area[i]);
  part[threadIdx.x] = s;
  __syncthreads();
  for (int w = 512; w; w >>= 1) {
    if (threadIdx.x < w) part[threadIdx.x] = __dadd_rn(part[threadIdx.x], part[threadIdx.x + w]);
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = part[0];
}

mt_status cudaStatus(cudaError_t e) {
  if (e == cudaSuccess) return MT_OK;
  if (e == cudaErrorInvalidValue || e == cudaErrorInvalidDevicePointer) return MT_ERROR_INVALID_ARGUMENT;
  return MT_ERROR;
}

int gridFor(uint32_t) {
  int device = 0, sms = 148;
  if (cudaGetDevice(&device) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  return sms * 4;
}

}  // namespace

extern "C" {

uint64_t mtc_blas_refit_plan_bytes(uint64_t bvh_vec4_count) {
  if (bvh_vec4_count < 2 || bvh_vec4_count > (1ull << 32)) return 0;
  return planBytes(bvh_vec4_count, nullptr, nullptr);
}

mt_status mtc_blas_refit_prepare(const void *bvh, uint64_t bvh_vec4_count, void *plan, uint64_t plan_bytes,
                                 mtc_blas_refit_plan_info *info, void *stream) {
  if (!bvh || !plan || !info || info->struct_size != sizeof(mtc_blas_refit_plan_info) || bvh_vec4_count < 2 ||
      bvh_vec4_count > (1ull << 32) || plan_bytes < planBytes(bvh_vec4_count, nullptr, nullptr) ||
      reinterpret_cast<uintptr_t>(plan) % 256 || reinterpret_cast<uintptr_t>(bvh) % 16)
    return MT_ERROR_INVALID_ARGUMENT;
  Plan p;
  planBytes(bvh_vec4_count, &p, static_cast<char *>(plan));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const uint32_t capacity = uint32_t(bvh_vec4_count / 2 + 1);
  k_plan_init<<<1, 1, 0, st>>>(p, capacity);
  const int grid = gridFor(0);
  PlanHeader h{};
  uint32_t level = 0, before = 1;
  for (;;) {
    k_plan_level<<<grid, kThreads, 0, st>>>(p, static_cast<const int4 *>(bvh), bvh_vec4_count, level);
    k_plan_close_level<<<1, 1, 0, st>>>(p, level);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(&h, p.h, sizeof(h), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cudaStatus(e);
    if (h.error) return MT_ERROR_INVALID_ARGUMENT;  // offsets outside the buffer or not in DFS order
    if (h.nodeCount == before) break;              // this level had no interior node: it is the deepest
    if (level + 3 >= kMaxLevels) return MT_ERROR_INVALID_ARGUMENT;
    before = h.nodeCount;
    level++;
  }
  info->node_count = h.nodeCount;
  info->levels = level + 1;
  return MT_OK;
}

mt_status mtc_refit_blas(void *bvh, uint64_t bvh_vec4_count, const void *plan, uint32_t levels,
                         const float *positions, uint32_t vertex_count, double *surface_area, void *stream) {
  if (!bvh || !plan || !levels || levels >= kMaxLevels || bvh_vec4_count < 2 || bvh_vec4_count > (1ull << 32) ||
      (vertex_count && !positions) || reinterpret_cast<uintptr_t>(plan) % 256 ||
      reinterpret_cast<uintptr_t>(bvh) % 16)
    return MT_ERROR_INVALID_ARGUMENT;
  Plan p;
  planBytes(bvh_vec4_count, &p, static_cast<char *>(const_cast<void *>(plan)));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const int grid = gridFor(0);
  for (uint32_t level = levels; level-- > 0;)
    k_refit_blas_level<<<grid, kThreads, 0, st>>>(p, static_cast<float4 *>(bvh), level, positions, vertex_count);
  if (surface_area) k_area_sum<<<1, 1024, 0, st>>>(p, surface_area);
  return cudaStatus(cudaGetLastError());
}

}  // extern "C"
