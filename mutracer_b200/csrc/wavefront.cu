// Wavefront form of the batched path tracer (mtc_stream_run).
//
// The megakernel keeps a whole path sample in one thread, so its traversal
// loops, latency-bound chains of dependent node loads, share one register
// budget with the shading code: either few warps or heavy spills, and lanes
// that drift between camera, traversal and shading code.  Here the integrator's
// event loop (rayTrace.compute.ts:891-946) is cut at its traversals into
// separate kernels that each see a queue of path slots:
//
//   k_wf_extend  closest hit of every queued extension ray (traverse<false>)
//   k_wf_shade   surface interaction, material, completeVertex, shadeVertex
//                (shadeStep, the same out-of-line code the megakernel calls);
//                queues the NEE shadow ray and either the continuation or the
//                finished sample
//   k_wf_shadow  the NEE visibility tests (traverse<true>)
//   k_wf_finish  accumulation of finished samples (endSample) and the start of
//                the pixel's next sample or of a new pixel (beginSample)
//
// A slot owns one pixel of one job until all of that pixel's samples are
// done, and starts sample k+1 only after sample k has been accumulated, so
// every pixel receives the same sums in the same order as in the megakernel:
// images are bit-identical to mtc_trace_samples.  Pixels (units) are handed
// out from one counter in the warp-tile order of the mtc_batch_prepare table,
// so neighbouring slots start on neighbouring pixels.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>

#include "dev_shade.cuh"

using namespace mt;

namespace {

struct Slot {
  PathSample ps;
  Sampler smp;
  ShadowQuery shadow;
  uint32_t job, x, y, left;  // pixel owned, samples still to start after the current one
};
static_assert(sizeof(Slot) % 16 == 0 && alignof(Slot) == 16, "slots keep their path sample 16-byte aligned");

// Queue state at the start of the stream state buffer (256 bytes).
struct StreamQueues {
  uint32_t unitNext;         // next unit (pixel) to hand out
  uint32_t rayCount[2];      // extension-ray queue sizes (double-buffered)
  uint32_t shadowCount;
  uint32_t finishCount;
  uint32_t extendNext;       // next extension ray to hand to a lane
  uint32_t shadowNext;       // next shadow ray to hand to a lane
  // Event-iteration state, advanced on the device by k_wf_continue: the
  // parity of the extension queue being traced, whether this iteration
  // regroups the shading queue, iterations completed, set when the
  // iteration limit stopped a run with rays still queued, and whether the
  // loop goes on (read by the host-driven loop).
  uint32_t cur;
  uint32_t regroup;
  uint32_t iterations;
  uint32_t limitHit;
  uint32_t more;
  uint32_t _pad[52];
};
static_assert(sizeof(StreamQueues) == 256, "queue header size");

// Same layout as the batched table header written by mtc_batch_prepare.
struct TableHeader {
  uint32_t jobCount, totalItems, tileW, flagsUnion, _pad[60];
};
static_assert(sizeof(TableHeader) == 256, "table header size");

struct StreamView {
  const TableHeader *header;
  const JobData *jobs;
  StreamQueues *q;
  Slot *slots;
  SpectralState *spectral;  // per slot, used by spectral jobs only
  TraversalHit *hits;
  uint32_t *rayQueue[2];
  uint32_t *shadowQueue, *finishQueue;
  uint32_t *keys, *sortedQueue;   // material-class key per slot; extension queue ordered by key
  uint32_t *classCount, *classCursor;  // kClasses each
  uint32_t *rayKeys, *sortedRays;  // (job, direction octant) key per slot; extension queue ordered by it
  uint32_t *rayKeyCount[2], *rayKeyCursor;  // kRayKeys each, counts per queue parity
  uint32_t sortRays;
  uint32_t slotCount;
  uint32_t refillLanes;  // idle lanes of a warp that trigger a ray refill
  uint32_t stepsPerCheck;  // traversal steps between refill checks
  mtc_counters *counters;
};

constexpr uint32_t kStreamThreads = 128;

__device__ __forceinline__ uint32_t laneId() { return threadIdx.x & 31u; }

// Copies a path sample between its slot (16-byte aligned: slots start on
// 256-byte boundaries and a Slot is a multiple of 16 bytes) and a 16-byte
// aligned register copy with 128-bit accesses, the tail in 32-bit words:
// a quarter of the load/store instructions of a field-by-field copy, whose
// 4-byte accesses each touch one sector per lane of this array of structs.
__device__ __forceinline__ void copyPathSample(PathSample &dst, const PathSample &src) {
  constexpr int kWide = int(sizeof(PathSample) / 16), kTail = int(sizeof(PathSample) % 16) / 4;
  static_assert(sizeof(PathSample) % 4 == 0, "path sample words");
  const uint4 *s = reinterpret_cast<const uint4 *>(&src);
  uint4 *d = reinterpret_cast<uint4 *>(&dst);
#pragma unroll
  for (int i = 0; i < kWide; i++) d[i] = s[i];
  const uint32_t *st = reinterpret_cast<const uint32_t *>(s + kWide);
  uint32_t *dt = reinterpret_cast<uint32_t *>(d + kWide);
#pragma unroll
  for (int i = 0; i < kTail; i++) dt[i] = st[i];
}

// Appends `value` to a queue with one atomic per converged group of lanes.
__device__ __forceinline__ void enqueue(uint32_t *queue, uint32_t *count, uint32_t value) {
  unsigned m = __activemask();
  int leader = __ffs(m) - 1;
  uint32_t rank = __popc(m & ((1u << laneId()) - 1u));
  uint32_t base = 0;
  if (int(laneId()) == leader) base = atomicAdd(count, uint32_t(__popc(m)));
  base = __shfl_sync(m, base, leader);
  queue[base + rank] = value;
}

__device__ __forceinline__ uint32_t takeUnit(uint32_t *counter) {
  unsigned m = __activemask();
  int leader = __ffs(m) - 1;
  uint32_t rank = __popc(m & ((1u << laneId()) - 1u));
  uint32_t base = 0;
  if (int(laneId()) == leader) base = atomicAdd(counter, uint32_t(__popc(m)));
  base = __shfl_sync(m, base, leader);
  return base + rank;
}

// Counts one launch of the calling kernel (block 0, thread 0).
__device__ __forceinline__ void countLaunch(const StreamView &v) {
  if (v.counters && blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&v.counters->kernel_launches, 1ull);
}

__device__ __forceinline__ void flush(const StreamView &v, uint32_t ext, uint32_t shadow, uint32_t paths) {
  if (!v.counters) return;
  countLaunch(v);
  unsigned m = __activemask();
  uint32_t e = __reduce_add_sync(m, ext), s = __reduce_add_sync(m, shadow), p = __reduce_add_sync(m, paths);
  if (int(laneId()) == __ffs(m) - 1) {
    if (e) atomicAdd(&v.counters->extension_rays, (unsigned long long)e);
    if (s) atomicAdd(&v.counters->shadow_rays, (unsigned long long)s);
    if (p) atomicAdd(&v.counters->path_samples, (unsigned long long)p);
  }
}

__device__ __forceinline__ BsdfContext bsdfContext(const JobData &J) {
  return BsdfContext{J.s.lut, (J.s.flags & MTC_SCENE_HAS_MEDIUM) != 0u, feature(J, MTC_FEATURE_HAS_THIN_FILM)};
}

// Material classes for regrouping the shading queue: 0 = miss, else 1 + a
// mask of the lobes the hit material switches on (metal, coat, transmission,
// fuzz/subsurface/thin film, non-default material type), read from the
// MaterialBuffer rows that getMaterial reads (materialLayoutSchema.ts:23-150).
constexpr uint32_t kClasses = 64;

__device__ __forceinline__ uint32_t materialClass(const JobData &J, const TraversalHit &h) {
  if (h.insIdx < 0) return 0u;
  const float4 *insv = J.s.ins + size_t(h.insIdx) * MTC_INSTANCE_VEC4_STRIDE;
  int32_t mi = asi(ld4(insv).z) >> 8;
  if (uint32_t(mi) >= J.s.matCount) mi = 0;
  const float4 *d = J.s.mats + size_t(mi) * MTC_MATERIAL_VEC4_ROWS;
  uint32_t k = 0;
  if (ld4(d + 2).x > 0.0f) k |= 1u;                                   // base_metalness
  if (ld4(d + 16).w > 0.0f) k |= 2u;                                  // coat_weight
  if (ld4(d + 4).y > 0.0f) k |= 4u;                                   // transmission_weight
  if (ld4(d + 11).w > 0.0f || ld4(d + 10).w > 0.0f || ld4(d + 18).x > 0.0f) k |= 8u;  // fuzz, subsurface, thin film
  if (int(ld4(d).w) != 0) k |= 16u;                                   // material type
  return 1u + k;
}

// Keys for ordering the extension queue: the job (mod 64) and the octant of
// the ray direction, so that a warp traverses rays of one scene heading the
// same way.
constexpr uint32_t kRayKeys = 512;

__device__ __forceinline__ uint32_t rayKey(uint32_t job, V3 d) {
  uint32_t oct = (d.x < 0.0f ? 1u : 0u) | (d.y < 0.0f ? 2u : 0u) | (d.z < 0.0f ? 4u : 0u);
  return (job & 63u) * 8u + oct;
}

// Appends slot `s` to the extension queue of parity `q` and, when the queue
// is ordered before traversal, counts it under its ray key.
__device__ __forceinline__ void enqueueRay(const StreamView &v, uint32_t q, uint32_t s) {
  enqueue(v.rayQueue[q], &v.q->rayCount[q], s);
  if (v.sortRays) {
    const Slot &sl = v.slots[s];
    uint32_t key = rayKey(sl.job, sl.ps.path.ray.d);
    v.rayKeys[s] = key;
    unsigned m = __match_any_sync(__activemask(), key);
    if (int(laneId()) == __ffs(m) - 1) atomicAdd(&v.rayKeyCount[q][key], uint32_t(__popc(m)));
  }
}

// Counts a finished extension ray in its material class (one atomic per
// class present in the converged group of lanes).
__device__ __forceinline__ void countClass(const StreamView &v, uint32_t s, uint32_t key) {
  v.keys[s] = key;
  unsigned m = __match_any_sync(__activemask(), key);
  if (int(laneId()) == __ffs(m) - 1) atomicAdd(&v.classCount[key], uint32_t(__popc(m)));
}

// Gives slot `s` the next pixel that has samples to add, and starts its first
// sample.  Returns false when the units are exhausted.
__device__ bool claimPixel(const StreamView &v, uint32_t s) {
  const uint32_t jobCount = v.header->jobCount;
  const uint32_t totalUnits = v.header->totalItems * 32u;
  const uint32_t tileW = v.header->tileW, tileH = 32u / tileW;
  // Units outside their image (ragged edge tiles) are skipped; the loop ends
  // at the first pixel with samples or when the units run out.
  for (uint32_t guard = 0; guard <= totalUnits; guard++) {
    uint32_t u = takeUnit(&v.q->unitNext);
    if (u >= totalUnits) return false;
    uint32_t item = u >> 5, lane = u & 31u;
    // Binary search of the job owning warp tile `item` (firstItem ascending).
    uint32_t lo = 0, hi = jobCount;
    while (hi - lo > 1u) {
      uint32_t mid = (lo + hi) >> 1;
      if (v.jobs[mid].firstItem <= item) lo = mid; else hi = mid;
    }
    const JobData &J = v.jobs[lo];
    uint32_t local = item - J.firstItem;
    uint32_t x = (local % J.tilesX) * tileW + lane % tileW;
    uint32_t y = (local / J.tilesX) * tileH + lane / tileW;
    if (x >= J.width || y >= J.height || J.samples == 0u) continue;
    Slot &sl = v.slots[s];
    sl.job = lo;
    sl.x = x;
    sl.y = y;
    sl.left = J.samples - 1u;
    Ctx c{J, Sampler(), bsdfContext(J), Counters(), ShadowQuery()};
    alignas(16) PathSample ps;
    beginSample(c, x, y, ps, v.spectral[s]);
    copyPathSample(sl.ps, ps);
    sl.smp = c.smp;
    sl.shadow.valid = false;
    return true;
  }
  return false;
}

__global__ void __launch_bounds__(kStreamThreads) k_wf_seed(StreamView v, uint32_t regroup0) {
  if (blockIdx.x == 0 && threadIdx.x == 0) v.q->regroup = regroup0;
  for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < v.slotCount; s += gridDim.x * blockDim.x) {
    if (claimPixel(v, s)) enqueueRay(v, 0u, s);
  }
  flush(v, 0, 0, 0);
}

// Closest hits of the queued extension rays.  Persistent: a lane whose ray
// has finished takes the next queued ray at once, so a warp is not held by
// its slowest ray (traversal lengths differ by an order of magnitude here).
// Resident CTAs per SM of the traversal kernels: the closest-hit kernel at
// 5 holds its traversal state in 95 registers without spilling, the shadow
// kernel at 6 in 80 (measured 2 % and 0.8 % faster than 8 CTAs at 64
// registers with spills; 4 is 3.5 % slower).
#ifndef MT_EXTEND_MIN_BLOCKS
#define MT_EXTEND_MIN_BLOCKS 5
#endif
#ifndef MT_SHADOW_MIN_BLOCKS
#define MT_SHADOW_MIN_BLOCKS 6
#endif
template <bool kGpuLayout>
__global__ void __launch_bounds__(kStreamThreads, MT_EXTEND_MIN_BLOCKS)
    k_wf_extend(StreamView v) {
  const uint32_t cur = v.q->cur;
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    v.q->rayCount[cur ^ 1u] = 0;
    v.q->shadowCount = 0;
    v.q->finishCount = 0;
  }
  const uint32_t n = v.q->rayCount[cur];
  const uint32_t *queue = v.sortRays ? v.sortedRays : v.rayQueue[cur];
  if (v.sortRays && blockIdx.x == 0) {
    // The ray-key counts of this queue were consumed by k_wf_sort_rays.
    for (uint32_t k = threadIdx.x; k < kRayKeys; k += blockDim.x) {
      v.rayKeyCount[cur][k] = 0;
      v.rayKeyCursor[k] = 0;
    }
  }
  int32_t stack[kTraversalStackEntries];
  RayTraversal<false, kGpuLayout> rt;
  rt.stack = stack;
  uint32_t s = 0, ext = 0;
  bool busy = false, exhausted = false;
  for (;;) {
    const unsigned idle = __ballot_sync(0xffffffffu, !busy && !exhausted);
    const unsigned live = __ballot_sync(0xffffffffu, busy);
    if (!idle && !live) break;
    // Refill once enough lanes wait (or none is left tracing).
    if (idle && (uint32_t(__popc(idle)) >= v.refillLanes || !live)) {
      if (busy || exhausted) continue;
      uint32_t t = takeUnit(&v.q->extendNext);
      if (t >= n) {
        exhausted = true;
      } else if ((s = queue[t]) >= v.slotCount) {
        // Not reachable with consistent queue counts; never index past the slots.
      } else {
        const Slot &sl = v.slots[s];
        const JobData &J = v.jobs[sl.job];
        // traceExtension: an empty scene is a miss without a traversal, and a
        // spectral wavelength path restarting at the shared primary vertex
        // traces nothing.
        if (J.u.is_empty > 0 || (isSpectral(J) && reusesPrimary(J, sl.ps, v.spectral[s].primaryReady)) ||
            (alphaSplit(J) && v.spectral[s].frontPending)) {
          TraversalHit none;
          none.tMax = RAY_MAX_DISTANCE;
          none.triangleIndex = -1;
          none.insIdx = -1;
          v.hits[s] = none;
        } else {
          ext++;
          if (rt.begin(J.s, J.u.blas_offset, sl.ps.path.ray.o, sl.ps.path.ray.d, sl.ps.depth, sl.ps.event != 0,
                       sl.ps.si.triangleIndex, sl.ps.si.instanceIndex, RAY_MAX_DISTANCE)) {
            busy = true;
          } else {
            v.hits[s] = rt.h;
          }
        }
      }
      continue;
    }
    // Several steps between refill checks: the votes cost as much as a node.
    bool finished = false;
    for (uint32_t k = 0; k < v.stepsPerCheck && busy && !finished; k++) finished = rt.step();
    if (finished) {
      v.hits[s] = rt.h;
      busy = false;
    }
  }
  flush(v, ext, 0, 0);
}

// Material class of every traced ray of this iteration (read from its hit),
// counted for k_wf_regroup; out of the traversal kernel, whose finishing
// lanes would otherwise make these dependent loads while the rest of their
// warp waits.
__global__ void __launch_bounds__(kStreamThreads) k_wf_classify(StreamView v) {
  countLaunch(v);
  if (!v.q->regroup) return;
  const uint32_t cur = v.q->cur;
  const uint32_t n = v.q->rayCount[cur];
  const uint32_t *queue = v.rayQueue[cur];
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const uint32_t s = queue[t];
    if (s >= v.slotCount) continue;
    countClass(v, s, materialClass(v.jobs[v.slots[s].job], v.hits[s]));
  }
}

// Orders the extension queue by ray key (counting sort, keys counted when
// the rays were queued).  Slot order never changes a result.
__global__ void __launch_bounds__(kStreamThreads) k_wf_sort_rays(StreamView v) {
  __shared__ uint32_t offset[kRayKeys];
  countLaunch(v);
  const uint32_t cur = v.q->cur;
  if (threadIdx.x == 0) {
    uint32_t acc = 0;
    for (uint32_t k = 0; k < kRayKeys; k++) {
      offset[k] = acc;
      acc += v.rayKeyCount[cur][k];
    }
  }
  __syncthreads();
  const uint32_t n = v.q->rayCount[cur];
  const uint32_t *queue = v.rayQueue[cur];
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    uint32_t s = queue[t];
    uint32_t key = v.rayKeys[s];
    unsigned m = __match_any_sync(__activemask(), key);
    int leader = __ffs(m) - 1;
    uint32_t base = 0;
    if (int(laneId()) == leader) base = atomicAdd(&v.rayKeyCursor[key], uint32_t(__popc(m)));
    base = __shfl_sync(m, base, leader);
    v.sortedRays[offset[key] + base + __popc(m & ((1u << laneId()) - 1u))] = s;
  }
}

// Orders the extension queue by material class (counting sort on the keys
// counted by k_wf_extend), so that the warps shading at any one time run the
// same BSDF code.  The order of slots inside a class is arbitrary; it cannot
// change any result, since slots never share state.
__global__ void __launch_bounds__(kStreamThreads) k_wf_regroup(StreamView v) {
  __shared__ uint32_t offset[kClasses];
  countLaunch(v);
  if (!v.q->regroup) return;
  const uint32_t cur = v.q->cur;
  if (threadIdx.x == 0) {
    uint32_t acc = 0;
    for (uint32_t k = 0; k < kClasses; k++) {
      offset[k] = acc;
      acc += v.classCount[k];
    }
  }
  __syncthreads();
  const uint32_t n = v.q->rayCount[cur];
  const uint32_t *queue = v.rayQueue[cur];
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    uint32_t s = queue[t];
    uint32_t key = v.keys[s];
    unsigned m = __match_any_sync(__activemask(), key);
    int leader = __ffs(m) - 1;
    uint32_t base = 0;
    if (int(laneId()) == leader) base = atomicAdd(&v.classCursor[key], uint32_t(__popc(m)));
    base = __shfl_sync(m, base, leader);
    v.sortedQueue[offset[key] + base + __popc(m & ((1u << laneId()) - 1u))] = s;
  }
}

// Shading at 8 CTAs per SM (64 registers, 32 warps): more spilled state, but
// twice the warps to hide its latency (measured: 4 CTAs at 128 registers
// 6 % slower on the headline, 10-16 CTAs 2-4 % slower).
#ifndef MT_SHADE_MIN_BLOCKS
#define MT_SHADE_MIN_BLOCKS 8
#endif
__global__ void __launch_bounds__(kStreamThreads, MT_SHADE_MIN_BLOCKS)
    k_wf_shade(StreamView v) {
  const uint32_t cur = v.q->cur, regroup = v.q->regroup;
  if (blockIdx.x == 0) {
    if (threadIdx.x == 0) v.q->extendNext = 0;
    // The class counts of this iteration have been consumed by k_wf_regroup.
    for (uint32_t k = threadIdx.x; k < kClasses && regroup; k += blockDim.x) {
      v.classCount[k] = 0;
      v.classCursor[k] = 0;
    }
  }
  const uint32_t n = v.q->rayCount[cur];
  const uint32_t *queue = regroup ? v.sortedQueue : v.rayQueue[cur];
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    uint32_t s = queue[t];
    if (s >= v.slotCount) continue;
    Slot &sl = v.slots[s];
    const JobData &J = v.jobs[sl.job];
    Ctx c{J, sl.smp, bsdfContext(J), Counters(), ShadowQuery()};
    c.shadow.valid = false;
    alignas(16) PathSample ps;
    copyPathSample(ps, sl.ps);
    TraversalHit h = v.hits[s];
    bool ended = isSpectral(J)   ? shadeStepSpectral(c, ps, v.spectral[s], h)
                 : alphaSplit(J) ? shadeStepAlpha(c, ps, v.spectral[s], h)
                                 : shadeStep(c, ps, v.spectral[s], h);
    copyPathSample(sl.ps, ps);
    sl.smp = c.smp;
    sl.shadow = c.shadow;
    if (c.shadow.valid) enqueue(v.shadowQueue, &v.q->shadowCount, s);
    if (ended) enqueue(v.finishQueue, &v.q->finishCount, s);
    else enqueueRay(v, cur ^ 1u, s);
  }
  flush(v, 0, 0, 0);
}

// NEE visibility of the queued shadow rays (intersectSceneShadow and
// resolveShadow), persistent like k_wf_extend.
template <bool kGpuLayout, bool kAlpha>
__global__ void __launch_bounds__(kStreamThreads, MT_SHADOW_MIN_BLOCKS) k_wf_shadow(StreamView v) {
  const uint32_t n = v.q->shadowCount;
  int32_t stack[kTraversalStackEntries];
  RayTraversal<true, kGpuLayout, kAlpha> rt;
  rt.stack = stack;
  uint32_t s = 0, shadowRays = 0;
  bool busy = false, exhausted = false;
  for (;;) {
    bool done = false;
    const unsigned idle = __ballot_sync(0xffffffffu, !busy && !exhausted);
    const unsigned live = __ballot_sync(0xffffffffu, busy);
    if (!idle && !live) break;
    const bool refill = idle && (uint32_t(__popc(idle)) >= v.refillLanes || !live);
    if (refill && !busy && !exhausted) {
      uint32_t t = takeUnit(&v.q->shadowNext);
      if (t >= n) {
        exhausted = true;
      } else {
        s = v.shadowQueue[t];
        const Slot &sl = v.slots[s];
        const JobData &J = v.jobs[sl.job];
        const ShadowQuery &q = sl.shadow;
        if (J.u.is_empty > 0) {
          rt.found = false;
          done = true;
        } else {
          shadowRays++;
          float tMax = fminf(fmaxf(q.maxDistance, 0.0f), RAY_MAX_DISTANCE);
          if (rt.begin(J.s, J.u.blas_offset, q.ray.o, q.ray.d, 1, true, q.triangleIndex, q.instanceIndex, tMax)) {
            busy = true;
            // Coverage draws advance the path's own sampler, in place.
            if (kAlpha && (J.s.flags & MTC_SCENE_HAS_ALPHA)) {
              rt.alphaScene = &J.s;
              rt.alphaSmp = &v.slots[s].smp;
            }
          } else {
            done = true;
          }
        }
      }
    }
    if (!refill && busy) {
      bool finished = false;
      for (uint32_t k = 0; k < v.stepsPerCheck && !finished; k++) finished = rt.step();
      if (finished) {
        busy = false;
        done = true;
      }
    }
    if (done) {
      Slot &sl = v.slots[s];
      if (!rt.found) {
        V3 li = sl.ps.path.li;
        li += sl.shadow.contribution;
        sl.ps.path.li = li;
      }
      sl.shadow.valid = false;
    }
  }
  flush(v, 0, shadowRays, 0);
}

__global__ void __launch_bounds__(kStreamThreads) k_wf_finish(StreamView v) {
  const uint32_t cur = v.q->cur;
  if (blockIdx.x == 0 && threadIdx.x == 0) v.q->shadowNext = 0;
  const uint32_t n = v.q->finishCount;
  uint32_t paths = 0;
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    uint32_t s = v.finishQueue[t];
    Slot &sl = v.slots[s];
    const JobData &J = v.jobs[sl.job];
    alignas(16) PathSample ps;
    if (isSpectral(J) || alphaSplit(J)) {
      copyPathSample(ps, sl.ps);
      if ((isSpectral(J) && !finishWavelength(J, ps, v.spectral[s])) ||
          (alphaSplit(J) && !finishAlphaSplit(J, ps, v.spectral[s]))) {
        // The next wavelength path, or the front path, of this sample starts
        // at event 0.
        copyPathSample(sl.ps, ps);
        enqueueRay(v, cur ^ 1u, s);
        continue;
      }
      endSample(J, sl.x + sl.y * J.width, ps);
    } else {
      // The accumulation reads a dozen words of the path sample: from the
      // slot itself rather than a copy of all of it.
      endSample(J, sl.x + sl.y * J.width, sl.ps);
    }
    paths++;
    bool again;
    if (sl.left > 0u) {
      sl.left--;
      Ctx c{J, Sampler(), bsdfContext(J), Counters(), ShadowQuery()};
      beginSample(c, sl.x, sl.y, ps, v.spectral[s]);
      copyPathSample(sl.ps, ps);
      sl.smp = c.smp;
      again = true;
    } else {
      again = claimPixel(v, s);
    }
    if (again) enqueueRay(v, cur ^ 1u, s);
  }
  flush(v, 0, 0, paths);
}

// The last node of the graph's loop body, one thread: ends event iteration
// `iterations` (flips the queue parity, decides whether the next iteration
// regroups the shading queue, as iteration % regroupInterval == 0) and keeps
// the loop running while rays are queued and fewer than maxIterations
// iterations have run.  An empty queue means every unit has been claimed and
// every path finished.
__global__ void k_wf_continue(StreamView v, cudaGraphConditionalHandle loop, uint32_t inGraph,
                              uint32_t regroupInterval, uint32_t maxIterations) {
  countLaunch(v);
  StreamQueues *q = v.q;
  const uint32_t it = q->iterations + 1u, cur = q->cur ^ 1u;
  q->iterations = it;
  q->cur = cur;
  q->regroup = regroupInterval && (it % regroupInterval) == 0u ? 1u : 0u;
  const bool pending = q->rayCount[cur] != 0u;
  const bool more = pending && it < maxIterations;
  if (pending && !more) q->limitHit = 1u;
  q->more = more ? 1u : 0u;
  if (inGraph) cudaGraphSetConditional(loop, more ? 1u : 0u);
}

size_t roundUp(size_t x) { return (x + 255) / 256 * 256; }

struct StreamLayout {
  size_t table, queues, slots, spectral, hits, rayQueues, shadowQueue, finishQueue, keys, sortedQueue, classes, rayKeys, sortedRays, rayKeyCounts, total;
};

StreamLayout layout(uint32_t capacity, uint32_t slots) {
  StreamLayout L;
  size_t off = 0;
  L.table = off;
  off += roundUp(sizeof(TableHeader) + size_t(capacity) * sizeof(JobData));
  L.queues = off;
  off += sizeof(StreamQueues);
  L.slots = off;
  off += roundUp(size_t(slots) * sizeof(Slot));
  L.spectral = off;
  off += roundUp(size_t(slots) * sizeof(SpectralState));
  L.hits = off;
  off += roundUp(size_t(slots) * sizeof(TraversalHit));
  L.rayQueues = off;
  off += 2 * roundUp(size_t(slots) * 4);
  L.shadowQueue = off;
  off += roundUp(size_t(slots) * 4);
  L.finishQueue = off;
  off += roundUp(size_t(slots) * 4);
  L.keys = off;
  off += roundUp(size_t(slots) * 4);
  L.sortedQueue = off;
  off += roundUp(size_t(slots) * 4);
  L.classes = off;
  off += roundUp(2 * kClasses * 4);
  L.rayKeys = off;
  off += roundUp(size_t(slots) * 4);
  L.sortedRays = off;
  off += roundUp(size_t(slots) * 4);
  L.rayKeyCounts = off;
  off += roundUp(3 * kRayKeys * 4);
  L.total = off;
  return L;
}

struct StreamShape {
  uint32_t slots, iterationsPerCheck, maxIterations, refillLanes, regroupInterval, sortRays, stepsPerCheck,
      traversalCtasPerSm;
};

bool streamShape(const mtc_stream_config *c, StreamShape &out) {
  out = StreamShape{1u << 21, 0u, 1u << 20, 4u, 1u, 0u, 8u, 0u};
  if (!c) return true;
  if (c->struct_size != sizeof(mtc_stream_config)) return false;
  if (c->slots) {
    if (c->slots < 1024u || c->slots > (1u << 25)) return false;
    out.slots = c->slots;
  }
  if (c->iterations_per_check) {
    if (c->iterations_per_check > 256u) return false;
    out.iterationsPerCheck = c->iterations_per_check;
  }
  if (c->max_iterations) out.maxIterations = c->max_iterations;
  if (c->regroup_interval == MTC_REGROUP_OFF) {
    out.regroupInterval = 0;
  } else if (c->regroup_interval) {
    if (c->regroup_interval > 1024u) return false;
    out.regroupInterval = c->regroup_interval;
  }
  if (c->sort_rays > 1u) return false;
  out.sortRays = c->sort_rays;
  if (c->steps_per_check) {
    if (c->steps_per_check > 64u) return false;
    out.stepsPerCheck = c->steps_per_check;
  }
  if (c->traversal_ctas_per_sm > 8u) return false;
  out.traversalCtasPerSm = c->traversal_ctas_per_sm;
  if (c->refill_lanes) {
    if (c->refill_lanes > 32u) return false;
    out.refillLanes = c->refill_lanes;
  }
  return true;
}

// Every wavefront kernel asks for the largest L1 that still holds the shared
// memory of as many blocks per SM as its registers allow: the spilled
// traversal and shading state and the node reads all go through L1 (measured
// +1 % on the 1080p instanced workload).  A smaller carve-out than the
// blocks need would cut the blocks per SM instead.
cudaError_t carveout(const void *kernel) {
  cudaFuncAttributes a;
  cudaError_t e = cudaFuncGetAttributes(&a, kernel);
  if (e != cudaSuccess) return e;
  if (a.sharedSizeBytes == 0) return cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, 0);
  int device = 0, perSm = 0, smemPerSm = 0, reserved = 0;
  if ((e = cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                int(cudaSharedmemCarveoutMaxShared))) != cudaSuccess ||
      (e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kernel, kStreamThreads, 0)) != cudaSuccess ||
      (e = cudaGetDevice(&device)) != cudaSuccess ||
      (e = cudaDeviceGetAttribute(&smemPerSm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, device)) != cudaSuccess ||
      (e = cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, device)) != cudaSuccess)
    return e;
  const size_t need = size_t(std::max(1, perSm)) * (a.sharedSizeBytes + size_t(reserved));
  const int percent = int(std::min<size_t>(100, (need * 100 + size_t(smemPerSm) - 1) / size_t(std::max(1, smemPerSm))));
  return cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, percent);
}

cudaError_t gridFor(const void *kernel, uint32_t &grid) {
  int device = 0, sms = 0, perSm = 0;
  cudaError_t e = carveout(kernel);
  if (e == cudaSuccess) e = cudaGetDevice(&device);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
  if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSm, kernel, kStreamThreads, 0);
  if (e != cudaSuccess) return e;
  grid = uint32_t(std::max(1, sms * std::max(1, perSm)));
  return cudaSuccess;
}

// Per device: a lock that serialises graph lookups and launches (and the
// host-driven loop, which polls its pinned words), the stream the loop
// bodies are captured on, and the instantiated loop graphs of recent launch
// shapes.
constexpr int kMaxDevices = 64;
constexpr int kCachedGraphs = 4;

// Everything a loop graph bakes in: the kernels' view of the state buffer,
// the grids, the kernel variants and the loop parameters.
struct GraphKey {
  StreamView v;
  uint32_t grids[6];  // extend, shade, shadow, finish, ray sort, regroup
  uint32_t gpuLayout, alpha, regroupInterval, maxIterations;
};

struct CachedGraph {
  bool valid = false;
  GraphKey key;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaEvent_t done = nullptr;  // recorded after each launch of `exec`
};

struct DeviceRunState {
  std::mutex m;
  cudaStream_t capture = nullptr;
  uint32_t *pinned = nullptr;  // loop-flag words of the host-driven loop
  CachedGraph graphs[kCachedGraphs];
  uint32_t nextSlot = 0;
};
DeviceRunState g_run[kMaxDevices];

// One event iteration's kernels on `s` (captured into the loop body, or
// launched directly by the host-driven loop), k_wf_continue last.
void launchIteration(const GraphKey &k, cudaStream_t s, cudaGraphConditionalHandle loop, bool inGraph) {
  const StreamView &v = k.v;
  const uint32_t gExtend = k.grids[0], gShade = k.grids[1], gShadow = k.grids[2], gFinish = k.grids[3],
                 gSort = k.grids[4], gRegroup = k.grids[5];
  if (v.sortRays) k_wf_sort_rays<<<gSort, kStreamThreads, 0, s>>>(v);
  if (k.gpuLayout) k_wf_extend<true><<<gExtend, kStreamThreads, 0, s>>>(v);
  else k_wf_extend<false><<<gExtend, kStreamThreads, 0, s>>>(v);
  if (k.regroupInterval) k_wf_classify<<<gRegroup, kStreamThreads, 0, s>>>(v);
  if (k.regroupInterval) k_wf_regroup<<<gRegroup, kStreamThreads, 0, s>>>(v);
  k_wf_shade<<<gShade, kStreamThreads, 0, s>>>(v);
  if (k.alpha) {
    if (k.gpuLayout) k_wf_shadow<true, true><<<gShadow, kStreamThreads, 0, s>>>(v);
    else k_wf_shadow<false, true><<<gShadow, kStreamThreads, 0, s>>>(v);
  } else {
    if (k.gpuLayout) k_wf_shadow<true, false><<<gShadow, kStreamThreads, 0, s>>>(v);
    else k_wf_shadow<false, false><<<gShadow, kStreamThreads, 0, s>>>(v);
  }
  k_wf_finish<<<gFinish, kStreamThreads, 0, s>>>(v);
  k_wf_continue<<<1, 1, 0, s>>>(v, loop, inGraph ? 1u : 0u, k.regroupInterval, k.maxIterations);
}

// The device-driven event loop: a graph whose one node is a WHILE
// conditional; its body is one event iteration (optional ray sort,
// extension, optional regroup, shading, shadow, finish) followed by
// k_wf_continue, which sets the loop condition.  The iteration's queue parity
// and regroup flag live in the queue header, so one body serves every
// iteration.
cudaError_t buildLoopGraph(DeviceRunState &d, const GraphKey &k, CachedGraph &out) {
  cudaGraph_t g = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaError_t e = cudaGraphCreate(&g, 0);
  if (e != cudaSuccess) return e;
  cudaGraphConditionalHandle loop;
  e = cudaGraphConditionalHandleCreate(&loop, g, 1u, cudaGraphCondAssignDefault);
  cudaGraphNodeParams p = {};
  p.type = cudaGraphNodeTypeConditional;
  p.conditional.handle = loop;
  p.conditional.type = cudaGraphCondTypeWhile;
  p.conditional.size = 1;
  cudaGraphNode_t node = nullptr;
  if (e == cudaSuccess) e = cudaGraphAddNode(&node, g, nullptr, 0, &p);
  if (e == cudaSuccess) {
    cudaGraph_t body = p.conditional.phGraph_out[0];
    cudaStream_t cs = d.capture;
    e = cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      launchIteration(k, cs, loop, true);
      cudaError_t launched = cudaGetLastError();
      e = cudaStreamEndCapture(cs, &body);
      if (e == cudaSuccess) e = launched;
    }
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, g, 0);
  if (e != cudaSuccess) {
    cudaGetLastError();
    if (g) cudaGraphDestroy(g);
    return e;
  }
  cudaEvent_t done = nullptr;
  if ((e = cudaEventCreateWithFlags(&done, cudaEventDisableTiming)) != cudaSuccess) {
    cudaGraphExecDestroy(exec);
    cudaGraphDestroy(g);
    return e;
  }
  out.valid = true;
  out.key = k;
  out.graph = g;
  out.exec = exec;
  out.done = done;
  return cudaSuccess;
}

// The cache entry of the loop graph for `k`, built on first use (the least
// recently built one replaced once its last launch has finished).  Called
// with d.m held.
cudaError_t loopGraph(DeviceRunState &d, const GraphKey &k, CachedGraph **entry) {
  for (CachedGraph &c : d.graphs) {
    if (c.valid && std::memcmp(&c.key, &k, sizeof(GraphKey)) == 0) {
      *entry = &c;
      return cudaSuccess;
    }
  }
  if (!d.capture) {
    cudaError_t e = cudaStreamCreateWithFlags(&d.capture, cudaStreamNonBlocking);
    if (e != cudaSuccess) return e;
  }
  CachedGraph &slot = d.graphs[d.nextSlot];
  d.nextSlot = (d.nextSlot + 1) % kCachedGraphs;
  if (slot.valid) {
    // The old graph's last launch (on whatever stream) finishes first.
    cudaEventSynchronize(slot.done);
    cudaEventDestroy(slot.done);
    cudaGraphExecDestroy(slot.exec);
    cudaGraphDestroy(slot.graph);
    slot = CachedGraph();
  }
  cudaError_t e = buildLoopGraph(d, k, slot);
  if (e != cudaSuccess) return e;
  *entry = &slot;
  return cudaSuccess;
}

mt_status toStatus(cudaError_t e) {
  if (e == cudaSuccess) return MT_OK;
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return MT_ERROR_UNAVAILABLE;
  return MT_ERROR;
}

}  // namespace

extern "C" {

size_t mtc_stream_state_bytes(uint32_t capacity, const mtc_stream_config *config) {
  StreamShape shape;
  if (!streamShape(config, shape)) return 0;
  return layout(capacity, shape.slots).total;
}

}  // extern "C"

namespace {

// The host-driven form of the event loop (iterations_per_check > 0): every
// kernel of every iteration is a separate launch on `st`; every
// `iterationsPerCheck` iterations the host reads the loop flag k_wf_continue
// wrote, one check behind so the device never waits for the host, and stops
// at max_iterations.  For tools that cannot look into conditional graphs.
cudaError_t hostLoop(DeviceRunState &d, const GraphKey &key, const StreamShape &shape, cudaStream_t st) {
  std::lock_guard<std::mutex> g(d.m);
  cudaError_t e = cudaSuccess;
  if (!d.pinned) {
    void *p = nullptr;
    if ((e = cudaHostAlloc(&p, 64, cudaHostAllocDefault)) != cudaSuccess) return e;
    std::memset(p, 0, 64);
    d.pinned = static_cast<uint32_t *>(p);
  }
  cudaEvent_t ev[2];
  if ((e = cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming)) != cudaSuccess) return e;
  if ((e = cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming)) != cudaSuccess) {
    cudaEventDestroy(ev[0]);
    return e;
  }
  uint32_t iterations = 0, chunk = 0;
  while (e == cudaSuccess && iterations < shape.maxIterations) {
    const uint32_t n = std::min(shape.iterationsPerCheck, shape.maxIterations - iterations);
    for (uint32_t k = 0; k < n; k++) launchIteration(key, st, 0, false);
    iterations += n;
    if ((e = cudaGetLastError()) != cudaSuccess) break;
    e = cudaMemcpyAsync(&d.pinned[chunk & 1u], &key.v.q->more, 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaEventRecord(ev[chunk & 1u], st);
    if (e != cudaSuccess) break;
    if (chunk > 0) {
      if ((e = cudaEventSynchronize(ev[(chunk - 1) & 1u])) != cudaSuccess) break;
      if (d.pinned[(chunk - 1) & 1u] == 0u) break;
    }
    chunk++;
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  cudaEventDestroy(ev[0]);
  cudaEventDestroy(ev[1]);
  return e;
}

// Enqueues one wavefront run on `st`: the job table upload, the queue and
// count resets, the seed kernel and one launch of the loop graph.  With
// `wait`, blocks until the run has finished and reports MT_ERROR_TIMEOUT
// when the iteration limit stopped it.
mt_status streamLaunch(const void *table, uint32_t capacity, const mtc_stream_config *config, void *state,
                       mtc_counters *counters, cudaStream_t st, bool wait) {
  if (!table || !state || capacity == 0) return MT_ERROR_INVALID_ARGUMENT;
  StreamShape shape;
  if (!streamShape(config, shape)) return MT_ERROR_INVALID_ARGUMENT;
  if (shape.iterationsPerCheck && !wait) return MT_ERROR_INVALID_ARGUMENT;  // the host loop blocks
  TableHeader hdr;
  std::memcpy(&hdr, table, sizeof(hdr));
  if (hdr.jobCount > capacity || hdr.tileW == 0 || hdr.tileW > 32 || 32 % hdr.tileW) return MT_ERROR_INVALID_ARGUMENT;
  StreamLayout L = layout(capacity, shape.slots);
  char *base = static_cast<char *>(state);
  GraphKey key;
  std::memset(&key, 0, sizeof(key));  // padding included: keys compare bytewise
  StreamView &v = key.v;
  v.header = reinterpret_cast<const TableHeader *>(base + L.table);
  v.jobs = reinterpret_cast<const JobData *>(base + L.table + sizeof(TableHeader));
  v.q = reinterpret_cast<StreamQueues *>(base + L.queues);
  v.slots = reinterpret_cast<Slot *>(base + L.slots);
  v.spectral = reinterpret_cast<SpectralState *>(base + L.spectral);
  v.hits = reinterpret_cast<TraversalHit *>(base + L.hits);
  v.rayQueue[0] = reinterpret_cast<uint32_t *>(base + L.rayQueues);
  v.rayQueue[1] = reinterpret_cast<uint32_t *>(base + L.rayQueues + roundUp(size_t(shape.slots) * 4));
  v.shadowQueue = reinterpret_cast<uint32_t *>(base + L.shadowQueue);
  v.finishQueue = reinterpret_cast<uint32_t *>(base + L.finishQueue);
  v.keys = reinterpret_cast<uint32_t *>(base + L.keys);
  v.sortedQueue = reinterpret_cast<uint32_t *>(base + L.sortedQueue);
  v.classCount = reinterpret_cast<uint32_t *>(base + L.classes);
  v.classCursor = v.classCount + kClasses;
  v.rayKeys = reinterpret_cast<uint32_t *>(base + L.rayKeys);
  v.sortedRays = reinterpret_cast<uint32_t *>(base + L.sortedRays);
  v.rayKeyCount[0] = reinterpret_cast<uint32_t *>(base + L.rayKeyCounts);
  v.rayKeyCount[1] = v.rayKeyCount[0] + kRayKeys;
  v.rayKeyCursor = v.rayKeyCount[1] + kRayKeys;
  v.sortRays = shape.sortRays;
  v.slotCount = shape.slots;
  v.refillLanes = shape.refillLanes;
  v.stepsPerCheck = shape.stepsPerCheck;
  v.counters = counters;

  cudaError_t e = cudaMemcpyAsync(base + L.table, table, sizeof(TableHeader) + size_t(capacity) * sizeof(JobData),
                                  cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(v.q, 0, sizeof(StreamQueues), st);
  if (e == cudaSuccess) e = cudaMemsetAsync(v.classCount, 0, 2 * kClasses * 4, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(v.rayKeyCount[0], 0, 3 * kRayKeys * 4, st);
  if (e != cudaSuccess) return toStatus(e);
  if (hdr.totalItems == 0 || hdr.jobCount == 0) return MT_OK;

  uint32_t gSeed, gExtend, gShade, gShadow, gFinish, gRegroup, gSort;
  if ((e = gridFor((const void *)k_wf_seed, gSeed)) != cudaSuccess ||
      (e = gridFor((const void *)k_wf_extend<false>, gExtend)) != cudaSuccess ||
      (e = gridFor((const void *)k_wf_shade, gShade)) != cudaSuccess ||
      (e = gridFor((const void *)k_wf_shadow<false, false>, gShadow)) != cudaSuccess ||
      (e = gridFor((const void *)k_wf_finish, gFinish)) != cudaSuccess ||
      (e = gridFor((const void *)k_wf_regroup, gRegroup)) != cudaSuccess ||
      (e = gridFor((const void *)k_wf_sort_rays, gSort)) != cudaSuccess ||
      (e = carveout((const void *)k_wf_extend<true>)) != cudaSuccess ||
      (e = carveout((const void *)k_wf_shadow<true, false>)) != cudaSuccess ||
      (e = carveout((const void *)k_wf_shadow<false, true>)) != cudaSuccess ||
      (e = carveout((const void *)k_wf_shadow<true, true>)) != cudaSuccess)
    return toStatus(e);
  int device = 0;
  if ((e = cudaGetDevice(&device)) != cudaSuccess) return toStatus(e);
  if (device < 0 || device >= kMaxDevices) return MT_ERROR_UNAVAILABLE;
  if (shape.traversalCtasPerSm) {
    // Fewer resident traversal warps: a smaller local-memory footprint per SM.
    int sms = 0;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device)) != cudaSuccess)
      return toStatus(e);
    gExtend = std::min(gExtend, uint32_t(sms) * shape.traversalCtasPerSm);
    gShadow = std::min(gShadow, uint32_t(sms) * shape.traversalCtasPerSm);
  }
  // The BLAS-layout specialisation (blasLayoutMask) of the traversal kernels,
  // and the coverage test of shadow rays in scenes with alpha.
  key.gpuLayout = (hdr.flagsUnion & MTC_SCENE_BLAS_GPU_LAYOUT) != 0u ? 1u : 0u;
  key.alpha = (hdr.flagsUnion & MTC_SCENE_HAS_ALPHA) != 0u ? 1u : 0u;
  key.grids[0] = gExtend;
  key.grids[1] = gShade;
  key.grids[2] = gShadow;
  key.grids[3] = gFinish;
  key.grids[4] = gSort;
  key.grids[5] = gRegroup;
  key.regroupInterval = shape.regroupInterval;
  key.maxIterations = shape.maxIterations;

  k_wf_seed<<<gSeed, kStreamThreads, 0, st>>>(v, shape.regroupInterval ? 1u : 0u);
  if ((e = cudaGetLastError()) != cudaSuccess) return toStatus(e);
  DeviceRunState &d = g_run[device];
  if (!shape.iterationsPerCheck) {
    std::lock_guard<std::mutex> g(d.m);
    CachedGraph *entry = nullptr;
    if ((e = loopGraph(d, key, &entry)) != cudaSuccess) return toStatus(e);
    if ((e = cudaGraphLaunch(entry->exec, st)) != cudaSuccess) return toStatus(e);
    if ((e = cudaEventRecord(entry->done, st)) != cudaSuccess) return toStatus(e);
  } else if ((e = hostLoop(d, key, shape, st)) != cudaSuccess) {
    return toStatus(e);
  }
  if (!wait) return MT_OK;
  uint32_t limitHit = 0;
  e = cudaMemcpyAsync(&limitHit, &v.q->limitHit, 4, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return toStatus(e);
  return limitHit ? MT_ERROR_TIMEOUT : MT_OK;
}

}  // namespace

extern "C" {

mt_status mtc_stream_run(const void *table, uint32_t capacity, const mtc_stream_config *config, void *state,
                         mtc_counters *counters, void *stream) {
  return streamLaunch(table, capacity, config, state, counters, (cudaStream_t)stream, true);
}

mt_status mtc_stream_launch(const void *table, uint32_t capacity, const mtc_stream_config *config, void *state,
                            mtc_counters *counters, void *stream) {
  return streamLaunch(table, capacity, config, state, counters, (cudaStream_t)stream, false);
}

mt_status mtc_stream_status(const void *state, uint32_t capacity, const mtc_stream_config *config, void *stream) {
  if (!state || capacity == 0) return MT_ERROR_INVALID_ARGUMENT;
  StreamShape shape;
  if (!streamShape(config, shape)) return MT_ERROR_INVALID_ARGUMENT;
  const StreamLayout L = layout(capacity, shape.slots);
  const StreamQueues *q = reinterpret_cast<const StreamQueues *>(static_cast<const char *>(state) + L.queues);
  cudaStream_t st = (cudaStream_t)stream;
  uint32_t limitHit = 0;
  cudaError_t e = cudaMemcpyAsync(&limitHit, &q->limitHit, 4, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return toStatus(e);
  return limitHit ? MT_ERROR_TIMEOUT : MT_OK;
}

}  // extern "C"
