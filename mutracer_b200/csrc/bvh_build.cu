// BLAS build on the device: buildBLAS (src/renderer/bvhAccel.ts:200-286,
// without displacement) with the binned-SAH builder of
// src/renderer/binnedSahBvh.ts:70-236 and the depth-first BVH2 layout of
// binnedSahBvh.ts:252-275, producing the same bytes as the host producer.
//
// The reference builds depth first on one CPU thread.  Every decision it makes
// for a node depends only on that node's primitives, so the same tree can be
// built breadth first:
//   * bins are reductions (counts, and JavaScript Math.min/max, which are
//     order independent: -0 sorts below +0), accumulated with shared- and
//     global-memory atomics on order-preserving integer keys of the f32
//     bounds;
//   * the split sweep, the leaf test and the child boxes run in float64 with
//     every operation rounded like the reference's (no contraction);
//   * the reference's in-place two-pointer partition is a fixed permutation of
//     the node's range given the side of each primitive.  With R_k the
//     position of the k-th right-side primitive from the left and L_k the k-th
//     left-side primitive from the right (L_0 = n):
//       left  primitive L_k moves to R_k when R_k < L_k, else stays;
//       right primitive R_k moves to L_{k-1} - 1 when R_k < L_{k-1}, else to
//       its position - 1,
//     so it is computed from per-element ranks (prefix counts) in parallel;
//   * node numbering differs from the reference's, but the emitted buffer
//     depends only on the tree (node boxes, child order, leaf primitive
//     order), not on node ids.
// Nodes with more than kSmallLimit primitives are split level by level across
// the whole GPU (one host read-back per level to learn the next level's node
// count); each remaining subtree is finished by one CTA in shared memory, one
// warp per node.  The layout pass then computes subtree sizes bottom up and
// DFS offsets top down, depth by depth, and writes the buffer.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/mutracer_b200.h"
#include "js_minmax.h"

namespace {

constexpr uint32_t kSmallLimit = 1024;  // subtree roots this small are finished by one CTA
constexpr uint32_t kChunk = 2048;       // primitives per CTA in the level-synchronous phase
constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kPerThread = kChunk / kThreads;
constexpr int kMaxBins = 64;
constexpr uint32_t kMaxTriangles = 400u << 20;  // keeps 5n vec4 offsets inside int32
constexpr double kFar = 1e30;                   // FAR of binnedSahBvh.ts
constexpr uint32_t kMinIdentity = 0xffffffffu;  // ordered-key identity of a min
constexpr uint32_t kMaxIdentity = 0u;

struct Globals {
  uint32_t nodeAlloc, activeNext, smallCount, maxDepth;
  uint32_t totalChunks, primCount, maxLeaf, error;  // error: a rank fell outside its node (never expected)
  double minDim[3];
  unsigned long long rootKey[6];
};

enum : uint32_t { kLeaf = 0, kSplit = 1, kPartitionLeaf = 2, kBinned = 3 };

// One node of the level-synchronous phase.
struct LargeNode {
  double nMin[3], scale[3];
  float childBounds[12];
  uint32_t node, first, count, depth;
  uint32_t chunkBegin, chunkCount, leftN, state;
  int32_t axis, pos;
};

struct Scratch {
  Globals *g;
  float *aabb, *center;
  uint32_t *tri, *prim, *tmp, *rank, *rf, *lb, *blockSum;
  float *nodeBounds;
  uint32_t *nodeFirst, *nodeCount, *nodeDepth, *nodeSize, *nodeOffset, *byDepth, *depthCursor;
  int32_t *nodeChild;
  uint32_t *activeA, *activeB, *smallQ, *chunkR, *bins;
  LargeNode *large;
  uint32_t maxActive, maxChunks, nodeCap, binWords;
};

template <class T>
T *take(char *base, size_t &off, size_t count) {
  size_t o = off;
  off = (off + count * sizeof(T) + 255) / 256 * 256;
  return base ? reinterpret_cast<T *>(base + o) : nullptr;
}

size_t carve(Scratch &s, char *base, uint32_t n, uint32_t bins) {
  size_t nn = std::max<size_t>(n, 1), off = 0;
  s.nodeCap = uint32_t(2 * nn - 1);
  s.maxActive = uint32_t(nn / (kSmallLimit + 1) + 1);
  s.maxChunks = uint32_t((nn + kChunk - 1) / kChunk + s.maxActive + 1);
  s.binWords = 21 * bins;  // 3 axes x bins: count, 3 min keys, 3 max keys
  size_t blocks = (nn + kChunk - 1) / kChunk;
  s.g = take<Globals>(base, off, 1);
  s.aabb = take<float>(base, off, nn * 6);
  s.center = take<float>(base, off, nn * 3);
  s.tri = take<uint32_t>(base, off, nn);
  s.prim = take<uint32_t>(base, off, nn);
  s.tmp = take<uint32_t>(base, off, nn);
  s.rank = take<uint32_t>(base, off, nn);
  s.rf = take<uint32_t>(base, off, nn);
  s.lb = take<uint32_t>(base, off, nn);
  s.blockSum = take<uint32_t>(base, off, blocks + 1);
  s.nodeBounds = take<float>(base, off, size_t(s.nodeCap) * 6);
  s.nodeFirst = take<uint32_t>(base, off, s.nodeCap);
  s.nodeCount = take<uint32_t>(base, off, s.nodeCap);
  s.nodeDepth = take<uint32_t>(base, off, s.nodeCap);
  s.nodeSize = take<uint32_t>(base, off, s.nodeCap);
  s.nodeOffset = take<uint32_t>(base, off, s.nodeCap);
  s.byDepth = take<uint32_t>(base, off, s.nodeCap);
  s.depthCursor = take<uint32_t>(base, off, size_t(s.nodeCap) + 2);
  s.nodeChild = take<int32_t>(base, off, s.nodeCap);
  s.activeA = take<uint32_t>(base, off, s.maxActive);
  s.activeB = take<uint32_t>(base, off, s.maxActive);
  s.smallQ = take<uint32_t>(base, off, s.nodeCap);
  s.chunkR = take<uint32_t>(base, off, s.maxChunks);
  s.bins = take<uint32_t>(base, off, size_t(s.maxActive) * s.binWords);
  s.large = take<LargeNode>(base, off, s.maxActive);
  return off;
}

// ------------------------------------------------------------ arithmetic
#define DA(a, b) __dadd_rn(a, b)
#define DM(a, b) __dmul_rn(a, b)

// Order-preserving u32 key of an f32 (-0 below +0; NaN never occurs: boxes
// are finite).
__device__ __forceinline__ uint32_t orderedKey(float f) {
  uint32_t b = __float_as_uint(f);
  return b ^ ((b >> 31) ? 0xffffffffu : 0x80000000u);
}
__device__ __forceinline__ float keyValue(uint32_t k) {
  return __uint_as_float((k & 0x80000000u) ? (k ^ 0x80000000u) : ~k);
}
// Key of the root-box reductions, whose `<` keeps the first of equal values:
// +0 and -0 share a key, ties go to the lowest position.
__device__ __forceinline__ uint32_t collapsedKey(float f) { return f == 0.0f ? 0x80000000u : orderedKey(f); }

// JavaScript `v | 0` (ToInt32).
__device__ __forceinline__ int32_t jsInt32(double v) {
  if (!(v == v) || isinf(v)) return 0;
  if (fabs(v) < 2147483648.0) return __double2int_rz(v);
  double m = fmod(trunc(v), 4294967296.0);
  if (m < 0) m += 4294967296.0;
  return int32_t(uint32_t(m));
}

// binOf of binnedSahBvh.ts:46-49.
__device__ __forceinline__ int binOf(float center, double nodeMin, double scale, int bins) {
  int32_t b = jsInt32(DM(DA(double(center), -nodeMin), scale));
  return b < 0 ? 0 : (b > bins - 1 ? bins - 1 : b);
}

__device__ __forceinline__ double areaOf(double x, double y, double z) { return DA(DA(DM(x, y), DM(y, z)), DM(z, x)); }

// triangleBounds of bvhAccel.ts:134-175 (no displacement).
__device__ bool triangleBox(const float *pos, const uint32_t *idx, uint32_t vertexCount, uint32_t t, float box[6]) {
  float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int c = 0; c < 3; c++) {
    uint32_t v = idx[size_t(t) * 3 + c];
    for (int k = 0; k < 3; k++) {
      float x = v < vertexCount ? pos[size_t(v) * 3 + k] : NAN;
      mn[k] = jsMin(mn[k], x);
      mx[k] = jsMax(mx[k], x);
    }
  }
  bool finite = true;
  for (int k = 0; k < 3; k++) {
    box[k] = mn[k];
    box[3 + k] = mx[k];
    finite = finite && isfinite(mn[k]) && isfinite(mx[k]);
  }
  return finite;
}

template <int NT>
__device__ uint32_t blockExclusiveSum(uint32_t v, uint32_t &total) {
  __shared__ uint32_t warpSums[NT / 32];
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint32_t x = v;
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warpSums[w] = x;
  __syncthreads();
  if (w == 0) {
    uint32_t s = lane < NT / 32 ? warpSums[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    if (lane < NT / 32) warpSums[lane] = s;
  }
  __syncthreads();
  uint32_t before = w ? warpSums[w - 1] : 0;
  total = warpSums[NT / 32 - 1];
  __syncthreads();
  return before + x - v;
}

// --------------------------------------------------- split decision (SAH)
struct Decision {
  uint32_t state, leftN;
  int32_t axis, pos;
  float childBounds[12];
};

// The bins of one node: counts[3B], min keys[3B*3], max keys[3B*3].
struct BinView {
  const uint32_t *w;
  int B;
  __device__ double mn(int bin, int k) const {
    return w[bin] ? jsMin(kFar, double(keyValue(w[3 * B + bin * 3 + k]))) : kFar;
  }
  __device__ double mx(int bin, int k) const {
    return w[bin] ? jsMax(-kFar, double(keyValue(w[12 * B + bin * 3 + k]))) : -kFar;
  }
};

// binnedSahBvh.ts:154-183 (sweep), :184-187 (leaf test) and :211-225 (child
// boxes).  Lanes 0-2 sweep one axis each (cost rows in `cost`, 6 * (B - 1)
// doubles of this warp); lane 0 combines them in axis order and returns the
// decision (valid on lane 0 only).
__device__ Decision decideSplit(const BinView &bins, const float nb[6], uint32_t count, const double minDim[3],
                                double *cost) {
  const int B = bins.B, lane = threadIdx.x & 31;
  double nMin[3], ext[3];
  for (int k = 0; k < 3; k++) {
    nMin[k] = nb[k];
    ext[k] = DA(double(nb[3 + k]), -nMin[k]);
  }
  double best = kFar;
  int bestPos = 0;
  if (lane < 3 && ext[lane] > minDim[lane]) {
    const int axis = lane;
    double *leftCost = cost + axis * 2 * (B - 1), *rightCost = leftCost + (B - 1);
    double lMin[3] = {kFar, kFar, kFar}, lMax[3] = {-kFar, -kFar, -kFar};
    double rMin[3] = {kFar, kFar, kFar}, rMax[3] = {-kFar, -kFar, -kFar};
    uint32_t leftN = 0, rightN = 0;
    for (int i = 0; i < B - 1; i++) {
      int l = axis * B + i, r = axis * B + B - 1 - i;
      for (int k = 0; k < 3; k++) {
        lMin[k] = jsMin(lMin[k], bins.mn(l, k));
        lMax[k] = jsMax(lMax[k], bins.mx(l, k));
        rMin[k] = jsMin(rMin[k], bins.mn(r, k));
        rMax[k] = jsMax(rMax[k], bins.mx(r, k));
      }
      leftN += bins.w[l];
      rightN += bins.w[r];
      double la = areaOf(DA(lMax[0], -lMin[0]), DA(lMax[1], -lMin[1]), DA(lMax[2], -lMin[2]));
      double ra = areaOf(DA(rMax[0], -rMin[0]), DA(rMax[1], -rMin[1]), DA(rMax[2], -rMin[2]));
      leftCost[i] = leftN == 0 ? kFar : DM(la, double(leftN));
      rightCost[B - 2 - i] = rightN == 0 ? kFar : DM(ra, double(rightN));
    }
    for (int i = 0; i < B - 1; i++) {
      double c = DA(leftCost[i], rightCost[i]);
      if (c < best) {
        best = c;
        bestPos = i;
      }
    }
  }
  double best1 = __shfl_sync(0xffffffffu, best, 1), best2 = __shfl_sync(0xffffffffu, best, 2);
  int pos1 = __shfl_sync(0xffffffffu, bestPos, 1), pos2 = __shfl_sync(0xffffffffu, bestPos, 2);
  Decision d;
  d.state = kLeaf;
  d.leftN = 0;
  d.axis = 0;
  d.pos = 0;
  if (lane != 0) return d;
  double split = kFar;
  if (best < split) { split = best; d.axis = 0; d.pos = bestPos; }
  if (best1 < split) { split = best1; d.axis = 1; d.pos = pos1; }
  if (best2 < split) { split = best2; d.axis = 2; d.pos = pos2; }
  double area = areaOf(ext[0], ext[1], ext[2]);
  split = DA(1.0, __ddiv_rn(split, area));  // C_TRAV + C_INT * cost / area
  if (!(split < double(count))) return d;
  uint32_t leftN = 0;
  for (int i = 0; i <= d.pos; i++) leftN += bins.w[d.axis * B + i];
  d.leftN = leftN;
  d.state = (leftN == 0 || leftN == count) ? kPartitionLeaf : kSplit;
  const float farF = float(kFar);
  for (int c = 0; c < 2; c++)
    for (int k = 0; k < 3; k++) {
      d.childBounds[c * 6 + k] = farF;
      d.childBounds[c * 6 + 3 + k] = -farF;
    }
  for (int i = 0; i < B; i++) {
    int bin = d.axis * B + i;
    float *base = d.childBounds + (i <= d.pos ? 0 : 6);
    for (int k = 0; k < 3; k++) {
      double lo = bins.mn(bin, k), hi = bins.mx(bin, k);
      if (lo < double(base[k])) base[k] = __double2float_rn(lo);
      if (hi > double(base[3 + k])) base[3 + k] = __double2float_rn(hi);
    }
  }
  return d;
}

__device__ __forceinline__ void addToBins(uint32_t *w, int B, const float *center, const float *box,
                                          const double nMin[3], const double scale[3]) {
  for (int axis = 0; axis < 3; axis++) {
    int bin = axis * B + binOf(center[axis], nMin[axis], scale[axis], B);
    atomicAdd(&w[bin], 1u);
    for (int k = 0; k < 3; k++) {
      atomicMin(&w[3 * B + bin * 3 + k], orderedKey(box[k]));
      atomicMax(&w[12 * B + bin * 3 + k], orderedKey(box[3 + k]));
    }
  }
}

__device__ __forceinline__ void initBins(uint32_t *w, int B, int tid, int stride) {
  for (int e = tid; e < 21 * B; e += stride) w[e] = e < 3 * B ? 0u : (e < 12 * B ? kMinIdentity : kMaxIdentity);
}

// Destination of relative position i in the node's permuted range (the
// two-pointer partition of binnedSahBvh.ts:193-204 in closed form).
// prefR = right-side primitives before i; rf[k] = position of the (k+1)-th
// right primitive from the left, lb[k] = of the (k+1)-th left primitive from
// the right.
__device__ __forceinline__ uint32_t partitionDest(uint32_t i, bool right, uint32_t prefR, uint32_t n, uint32_t nL,
                                                  const uint32_t *rf, const uint32_t *lb) {
  if (!right) {
    uint32_t k = nL - (i - prefR);  // 1-based rank among left primitives from the right
    if (k <= n - nL) {
      uint32_t q = rf[k - 1];
      if (q < i) return q;
    }
    return i;
  }
  uint32_t k = prefR + 1;  // 1-based rank among right primitives from the left
  uint32_t bound;
  if (k == 1) bound = n;
  else if (k - 1 <= nL) bound = lb[k - 2];
  else return i - 1;
  return i < bound ? bound - 1 : i - 1;
}

// ------------------------------------------------------- prepare kernels
__global__ void k_init(Globals *g) {
  g->nodeAlloc = 0;
  g->activeNext = 0;
  g->smallCount = 0;
  g->maxDepth = 0;
  g->totalChunks = 0;
  g->primCount = 0;
  g->maxLeaf = 0;
  g->error = 0;
  for (int k = 0; k < 3; k++) {
    g->rootKey[k] = ~0ull;
    g->rootKey[3 + k] = 0ull;
  }
}

__global__ void __launch_bounds__(kThreads) k_count_finite(Scratch s, const float *pos, const uint32_t *idx,
                                                           uint32_t vertexCount, uint32_t n) {
  uint32_t base = blockIdx.x * kChunk + threadIdx.x * kPerThread, cnt = 0;
  for (int j = 0; j < kPerThread; j++) {
    uint32_t t = base + j;
    float box[6];
    if (t < n && triangleBox(pos, idx, vertexCount, t, box)) cnt++;
  }
  uint32_t total;
  blockExclusiveSum<kThreads>(cnt, total);
  if (threadIdx.x == 0) s.blockSum[blockIdx.x] = total;
}

// In-place exclusive scan of v[0, *count) by one CTA of 1024 threads.
__global__ void __launch_bounds__(1024) k_scan(uint32_t *v, const uint32_t *countPtr, uint32_t count,
                                               uint32_t *total) {
  if (countPtr) count = *countPtr;
  uint32_t running = 0;
  for (uint32_t base = 0; base < count; base += 1024) {
    uint32_t i = base + threadIdx.x, x = i < count ? v[i] : 0, tot;
    uint32_t ex = blockExclusiveSum<1024>(x, tot);
    if (i < count) v[i] = running + ex;
    running += tot;
  }
  if (threadIdx.x == 0 && total) *total = running;
}

// Compacts the finite boxes in triangle order (bvhAccel.ts:219-236) with their
// centroids ((min + max) * 0.5 in float64, stored as f32: binnedSahBvh.ts:92-94).
__global__ void __launch_bounds__(kThreads) k_compact(Scratch s, const float *pos, const uint32_t *idx,
                                                      uint32_t vertexCount, uint32_t n) {
  uint32_t base = blockIdx.x * kChunk + threadIdx.x * kPerThread, cnt = 0, finiteMask = 0;
  for (int j = 0; j < kPerThread; j++) {
    uint32_t t = base + j;
    float box[6];
    if (t < n && triangleBox(pos, idx, vertexCount, t, box)) {
      finiteMask |= 1u << j;
      cnt++;
    }
  }
  uint32_t total;
  uint32_t out = s.blockSum[blockIdx.x] + blockExclusiveSum<kThreads>(cnt, total);
  for (int j = 0; j < kPerThread; j++) {
    if (!(finiteMask >> j & 1u)) continue;
    uint32_t t = base + j;
    float box[6];
    triangleBox(pos, idx, vertexCount, t, box);
    for (int k = 0; k < 6; k++) s.aabb[size_t(out) * 6 + k] = box[k];
    for (int k = 0; k < 3; k++)
      s.center[size_t(out) * 3 + k] = __double2float_rn(DM(DA(double(box[k]), double(box[3 + k])), 0.5));
    s.tri[out] = t;
    s.prim[out] = out;
    out++;
  }
}

// Root box (binnedSahBvh.ts:86-104): `if (v < rootMin) rootMin = v` from FAR
// keeps the first of equal values, so the keys carry the position.
__global__ void __launch_bounds__(kThreads) k_root_keys(Scratch s) {
  uint32_t count = s.g->primCount;
  unsigned long long key[6];
  for (int k = 0; k < 3; k++) {
    key[k] = ~0ull;
    key[3 + k] = 0ull;
  }
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    const float *b = s.aabb + size_t(i) * 6;
    for (int k = 0; k < 3; k++) {
      unsigned long long lo = (unsigned long long)collapsedKey(b[k]) << 32 | i;
      unsigned long long hi = (unsigned long long)collapsedKey(b[3 + k]) << 32 | (0xffffffffu - i);
      key[k] = lo < key[k] ? lo : key[k];
      key[3 + k] = hi > key[3 + k] ? hi : key[3 + k];
    }
  }
  for (int o = 16; o; o >>= 1)
    for (int k = 0; k < 3; k++) {
      unsigned long long lo = __shfl_xor_sync(0xffffffffu, key[k], o);
      unsigned long long hi = __shfl_xor_sync(0xffffffffu, key[3 + k], o);
      key[k] = lo < key[k] ? lo : key[k];
      key[3 + k] = hi > key[3 + k] ? hi : key[3 + k];
    }
  if ((threadIdx.x & 31) == 0)
    for (int k = 0; k < 3; k++) {
      atomicMin(&s.g->rootKey[k], key[k]);
      atomicMax(&s.g->rootKey[3 + k], key[3 + k]);
    }
}

__global__ void k_root_finalize(Scratch s) {
  Globals *g = s.g;
  uint32_t count = g->primCount;
  g->nodeAlloc = count ? 1 : 0;
  g->maxDepth = count ? 1 : 0;
  if (!count) return;
  double rMin[3], rMax[3];
  for (int k = 0; k < 3; k++) {
    uint32_t lo = uint32_t(g->rootKey[k]), hi = 0xffffffffu - uint32_t(g->rootKey[3 + k]);
    double vlo = s.aabb[size_t(lo) * 6 + k], vhi = s.aabb[size_t(hi) * 6 + 3 + k];
    rMin[k] = vlo < kFar ? vlo : kFar;
    rMax[k] = vhi > -kFar ? vhi : -kFar;
    s.nodeBounds[k] = __double2float_rn(rMin[k]);
    s.nodeBounds[3 + k] = __double2float_rn(rMax[k]);
    g->minDim[k] = DM(DA(rMax[k], -rMin[k]), 1e-20);
  }
  s.nodeFirst[0] = 0;
  s.nodeCount[0] = count;
  s.nodeDepth[0] = 1;
  s.nodeChild[0] = -1;
  if (count > kSmallLimit) {
    s.activeA[0] = 0;
    g->activeNext = 1;
  } else if (count >= 2) {
    s.smallQ[0] = 0;
    g->smallCount = 1;
  }
}

// ------------------------------------------- level-synchronous phase
__global__ void __launch_bounds__(1024) k_large_setup(Scratch s, const uint32_t *active, uint32_t activeCount,
                                                      int B) {
  uint32_t running = 0;
  for (uint32_t base = 0; base < activeCount; base += 1024) {
    uint32_t a = base + threadIdx.x, chunks = 0;
    if (a < activeCount) {
      LargeNode &L = s.large[a];
      uint32_t node = active[a];
      const float *nb = s.nodeBounds + size_t(node) * 6;
      double ext[3];
      for (int k = 0; k < 3; k++) {
        L.nMin[k] = nb[k];
        ext[k] = DA(double(nb[3 + k]), -L.nMin[k]);
        L.scale[k] = ext[k] > s.g->minDim[k] ? __ddiv_rn(double(B), ext[k]) : 0.0;
      }
      L.node = node;
      L.first = s.nodeFirst[node];
      L.count = s.nodeCount[node];
      L.depth = s.nodeDepth[node];
      if (areaOf(ext[0], ext[1], ext[2]) == 0.0) {
        L.state = kLeaf;
      } else {
        L.state = kBinned;
        chunks = (L.count + kChunk - 1) / kChunk;
      }
      initBins(s.bins + size_t(a) * s.binWords, B, 0, 1);
    }
    uint32_t total;
    uint32_t ex = blockExclusiveSum<1024>(chunks, total);
    if (a < activeCount) {
      s.large[a].chunkBegin = running + ex;
      s.large[a].chunkCount = chunks;
    }
    running += total;
  }
  if (threadIdx.x == 0) {
    s.g->totalChunks = running;
    s.g->activeNext = 0;
  }
}

// Node of chunk c: the last node whose first chunk is <= c (nodes without
// chunks share their chunkBegin with the next node).
__device__ uint32_t chunkNode(const Scratch &s, uint32_t activeCount, uint32_t c) {
  uint32_t lo = 0, hi = activeCount;
  while (hi - lo > 1) {
    uint32_t mid = (lo + hi) / 2;
    if (s.large[mid].chunkBegin <= c) lo = mid;
    else hi = mid;
  }
  return lo;
}

__global__ void __launch_bounds__(kThreads) k_large_bin(Scratch s, uint32_t activeCount, int B) {
  extern __shared__ uint32_t sBins[];
  uint32_t c = blockIdx.x;
  if (c >= s.g->totalChunks) return;
  const LargeNode &L = s.large[chunkNode(s, activeCount, c)];
  double nMin[3], scale[3];
  for (int k = 0; k < 3; k++) {
    nMin[k] = L.nMin[k];
    scale[k] = L.scale[k];
  }
  initBins(sBins, B, threadIdx.x, kThreads);
  __syncthreads();
  uint32_t begin = (c - L.chunkBegin) * kChunk, end = min(begin + kChunk, L.count);
  for (uint32_t i = begin + threadIdx.x; i < end; i += kThreads) {
    uint32_t p = s.prim[L.first + i];
    addToBins(sBins, B, s.center + size_t(p) * 3, s.aabb + size_t(p) * 6, nMin, scale);
  }
  __syncthreads();
  uint32_t *G = s.bins + size_t(&L - s.large) * s.binWords;
  for (int e = threadIdx.x; e < 21 * B; e += kThreads) {
    uint32_t v = sBins[e];
    if (e < 3 * B) {
      if (v) atomicAdd(&G[e], v);
    } else if (e < 12 * B) {
      if (v != kMinIdentity) atomicMin(&G[e], v);
    } else if (v != kMaxIdentity) {
      atomicMax(&G[e], v);
    }
  }
}

__global__ void __launch_bounds__(kThreads) k_large_sah(Scratch s, uint32_t activeCount, int B) {
  __shared__ double sCost[kWarps][6 * (kMaxBins - 1)];
  const int warp = threadIdx.x >> 5;
  uint32_t a = blockIdx.x * kWarps + warp;
  if (a >= activeCount) return;
  LargeNode &L = s.large[a];
  if (L.state != kBinned) return;
  BinView bins{s.bins + size_t(a) * s.binWords, B};
  double minDim[3] = {s.g->minDim[0], s.g->minDim[1], s.g->minDim[2]};
  Decision d = decideSplit(bins, s.nodeBounds + size_t(L.node) * 6, L.count, minDim, sCost[warp]);
  if ((threadIdx.x & 31) == 0) {
    L.state = d.state;
    L.axis = d.axis;
    L.pos = d.pos;
    L.leftN = d.leftN;
    for (int k = 0; k < 12; k++) L.childBounds[k] = d.childBounds[k];
  }
}

__device__ __forceinline__ bool partitions(uint32_t state) { return state == kSplit || state == kPartitionLeaf; }

__device__ __forceinline__ bool goesRight(const Scratch &s, const LargeNode &L, uint32_t i, int B) {
  uint32_t p = s.prim[L.first + i];
  return binOf(s.center[size_t(p) * 3 + L.axis], L.nMin[L.axis], L.scale[L.axis], B) > L.pos;
}

__global__ void __launch_bounds__(kThreads) k_large_classify(Scratch s, uint32_t activeCount, int B) {
  uint32_t c = blockIdx.x;
  if (c >= s.g->totalChunks) return;
  const LargeNode &L = s.large[chunkNode(s, activeCount, c)];
  uint32_t cnt = 0;
  if (partitions(L.state)) {
    uint32_t begin = (c - L.chunkBegin) * kChunk, end = min(begin + kChunk, L.count);
    for (uint32_t i = begin + threadIdx.x; i < end; i += kThreads) cnt += goesRight(s, L, i, B);
  }
  uint32_t total;
  blockExclusiveSum<kThreads>(cnt, total);
  if (threadIdx.x == 0) s.chunkR[c] = total;
}

// Per element: right-side count before it (rank), and the rf / lb tables.
__global__ void __launch_bounds__(kThreads) k_large_rank(Scratch s, uint32_t activeCount, int B) {
  uint32_t c = blockIdx.x;
  if (c >= s.g->totalChunks) return;
  const LargeNode &L = s.large[chunkNode(s, activeCount, c)];
  if (!partitions(L.state)) return;
  uint32_t begin = (c - L.chunkBegin) * kChunk, end = min(begin + kChunk, L.count);
  uint32_t i0 = begin + threadIdx.x * kPerThread, bits = 0, cnt = 0;
  for (int j = 0; j < kPerThread; j++) {
    uint32_t i = i0 + j;
    if (i < end && goesRight(s, L, i, B)) {
      bits |= 1u << j;
      cnt++;
    }
  }
  uint32_t total;
  uint32_t prefR = s.chunkR[c] - s.chunkR[L.chunkBegin] + blockExclusiveSum<kThreads>(cnt, total);
  for (int j = 0; j < kPerThread; j++) {
    uint32_t i = i0 + j;
    if (i >= end) break;
    bool right = bits >> j & 1u;
    s.rank[L.first + i] = prefR | (uint32_t(right) << 31);
    uint32_t slot = right ? prefR : L.leftN - (i - prefR) - 1;
    if (slot >= (right ? L.count - L.leftN : L.leftN)) {
      s.g->error = 1;
    } else if (right) {
      s.rf[L.first + slot] = i;
    } else {
      s.lb[L.first + slot] = i;
    }
    prefR += right;
  }
}

__global__ void __launch_bounds__(kThreads) k_large_scatter(Scratch s, uint32_t activeCount) {
  uint32_t c = blockIdx.x;
  if (c >= s.g->totalChunks) return;
  const LargeNode &L = s.large[chunkNode(s, activeCount, c)];
  if (!partitions(L.state)) return;
  uint32_t begin = (c - L.chunkBegin) * kChunk, end = min(begin + kChunk, L.count);
  for (uint32_t i = begin + threadIdx.x; i < end; i += kThreads) {
    uint32_t r = s.rank[L.first + i];
    uint32_t dest = partitionDest(i, r >> 31, r & 0x7fffffffu, L.count, L.leftN, s.rf + L.first, s.lb + L.first);
    if (dest < L.count) s.tmp[L.first + dest] = s.prim[L.first + i];
    else s.g->error = 1;
  }
}

__global__ void __launch_bounds__(kThreads) k_large_copy(Scratch s, uint32_t activeCount) {
  uint32_t c = blockIdx.x;
  if (c >= s.g->totalChunks) return;
  const LargeNode &L = s.large[chunkNode(s, activeCount, c)];
  if (!partitions(L.state)) return;
  uint32_t begin = (c - L.chunkBegin) * kChunk, end = min(begin + kChunk, L.count);
  for (uint32_t i = begin + threadIdx.x; i < end; i += kThreads) s.prim[L.first + i] = s.tmp[L.first + i];
}

__device__ void writeChild(const Scratch &s, uint32_t id, const float *bounds, uint32_t first, uint32_t count,
                           uint32_t depth) {
  for (int k = 0; k < 6; k++) s.nodeBounds[size_t(id) * 6 + k] = bounds[k];
  s.nodeFirst[id] = first;
  s.nodeCount[id] = count;
  s.nodeDepth[id] = depth;
  s.nodeChild[id] = -1;
}

__global__ void __launch_bounds__(kThreads) k_large_children(Scratch s, uint32_t activeCount, uint32_t *next) {
  uint32_t a = blockIdx.x * kThreads + threadIdx.x;
  if (a >= activeCount) return;
  const LargeNode &L = s.large[a];
  if (L.state != kSplit) return;
  uint32_t id = atomicAdd(&s.g->nodeAlloc, 2u);
  for (int c = 0; c < 2; c++) {
    uint32_t cnt = c ? L.count - L.leftN : L.leftN;
    writeChild(s, id + c, L.childBounds + 6 * c, L.first + (c ? L.leftN : 0), cnt, L.depth + 1);
    if (cnt > kSmallLimit) next[atomicAdd(&s.g->activeNext, 1u)] = id + c;
    else if (cnt >= 2) s.smallQ[atomicAdd(&s.g->smallCount, 1u)] = id + c;
  }
  s.nodeChild[L.node] = int32_t(id);
  atomicMax(&s.g->maxDepth, L.depth + 1);
}

// ------------------------------------------------ per-CTA subtree phase
struct SmallShared {
  float *aabb, *center;
  uint32_t *global, *perm, *tmp, *rf, *lb, *bins;
  uint4 *front[2];
  double *cost;
  Decision *dec;
  uint32_t *frontCount;
};

size_t smallSharedBytes(int B) {
  size_t bytes = size_t(kSmallLimit) * (6 + 3) * 4 + size_t(kSmallLimit) * 5 * 4;
  bytes += 2 * size_t(kSmallLimit / 2) * sizeof(uint4);
  bytes += size_t(kWarps) * 21 * B * 4;
  bytes = (bytes + 7) / 8 * 8;
  bytes += size_t(kWarps) * 6 * std::max(B - 1, 1) * sizeof(double);
  bytes += size_t(kWarps) * sizeof(Decision);
  bytes += 2 * sizeof(uint32_t);
  return bytes;
}

__device__ SmallShared carveShared(unsigned char *base, int B) {
  SmallShared S;
  size_t off = 0;
  auto grab = [&](size_t bytes) { unsigned char *p = base + off; off += bytes; return p; };
  S.aabb = (float *)grab(size_t(kSmallLimit) * 6 * 4);
  S.center = (float *)grab(size_t(kSmallLimit) * 3 * 4);
  S.global = (uint32_t *)grab(kSmallLimit * 4);
  S.perm = (uint32_t *)grab(kSmallLimit * 4);
  S.tmp = (uint32_t *)grab(kSmallLimit * 4);
  S.rf = (uint32_t *)grab(kSmallLimit * 4);
  S.lb = (uint32_t *)grab(kSmallLimit * 4);
  S.front[0] = (uint4 *)grab((kSmallLimit / 2) * sizeof(uint4));
  S.front[1] = (uint4 *)grab((kSmallLimit / 2) * sizeof(uint4));
  S.bins = (uint32_t *)grab(size_t(kWarps) * 21 * B * 4);
  off = (off + 7) / 8 * 8;
  S.cost = (double *)grab(size_t(kWarps) * 6 * (B > 1 ? B - 1 : 1) * sizeof(double));
  S.dec = (Decision *)grab(kWarps * sizeof(Decision));
  S.frontCount = (uint32_t *)grab(2 * sizeof(uint32_t));
  return S;
}

// One warp splits one node of a CTA-resident subtree (entry: node id, first
// in the CTA's range, count, depth) and appends its children to `next`.
__device__ void splitNodeWarp(const Scratch &s, const SmallShared &S, uint4 entry, uint32_t rootFirst, int B,
                              const double minDim[3], int nextSlot) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t id = entry.x, lf = entry.y, cnt = entry.z, depth = entry.w;
  float nb[6];
  for (int k = 0; k < 6; k++) nb[k] = s.nodeBounds[size_t(id) * 6 + k];
  double nMin[3], ext[3], scale[3];
  for (int k = 0; k < 3; k++) {
    nMin[k] = nb[k];
    ext[k] = DA(double(nb[3 + k]), -nMin[k]);
    scale[k] = ext[k] > minDim[k] ? __ddiv_rn(double(B), ext[k]) : 0.0;
  }
  if (areaOf(ext[0], ext[1], ext[2]) == 0.0 || cnt == 1) return;
  uint32_t *w = S.bins + size_t(warp) * 21 * B;
  initBins(w, B, lane, 32);
  __syncwarp();
  for (uint32_t i = lane; i < cnt; i += 32) {
    uint32_t li = S.perm[lf + i];
    addToBins(w, B, S.center + li * 3, S.aabb + li * 6, nMin, scale);
  }
  __syncwarp();
  Decision d = decideSplit(BinView{w, B}, nb, cnt, minDim, S.cost + size_t(warp) * 6 * (B > 1 ? B - 1 : 1));
  if (lane == 0) S.dec[warp] = d;
  __syncwarp();
  d = S.dec[warp];
  if (d.state == kLeaf) return;
  const int axis = d.axis;
  const uint32_t nL = d.leftN;
  // Pass 1: ranks and the rf / lb tables.
  uint32_t prefix = 0;
  for (uint32_t base = 0; base < cnt; base += 32) {
    uint32_t i = base + lane;
    bool right = i < cnt && binOf(S.center[S.perm[lf + i] * 3 + axis], nMin[axis], scale[axis], B) > d.pos;
    uint32_t ballot = __ballot_sync(0xffffffffu, right);
    uint32_t prefR = prefix + __popc(ballot & ((1u << lane) - 1));
    if (i < cnt) {
      uint32_t slot = right ? prefR : nL - (i - prefR) - 1;
      if (slot >= (right ? cnt - nL : nL)) s.g->error = 1;
      else if (right) S.rf[lf + slot] = i;
      else S.lb[lf + slot] = i;
    }
    prefix += __popc(ballot);
  }
  __syncwarp();
  // Pass 2: the permutation, into tmp.
  prefix = 0;
  for (uint32_t base = 0; base < cnt; base += 32) {
    uint32_t i = base + lane;
    bool right = i < cnt && binOf(S.center[S.perm[lf + i] * 3 + axis], nMin[axis], scale[axis], B) > d.pos;
    uint32_t ballot = __ballot_sync(0xffffffffu, right);
    uint32_t prefR = prefix + __popc(ballot & ((1u << lane) - 1));
    if (i < cnt) {
      uint32_t dest = partitionDest(i, right, prefR, cnt, nL, S.rf + lf, S.lb + lf);
      if (dest < cnt) S.tmp[lf + dest] = S.perm[lf + i];
      else s.g->error = 1;
    }
    prefix += __popc(ballot);
  }
  __syncwarp();
  for (uint32_t i = lane; i < cnt; i += 32) S.perm[lf + i] = S.tmp[lf + i];
  __syncwarp();
  if (d.state != kSplit || lane != 0) return;
  uint32_t child = atomicAdd(&s.g->nodeAlloc, 2u);
  for (int c = 0; c < 2; c++) {
    uint32_t ccnt = c ? cnt - nL : nL, clf = lf + (c ? nL : 0);
    writeChild(s, child + c, d.childBounds + 6 * c, rootFirst + clf, ccnt, depth + 1);
    if (ccnt >= 2) S.front[nextSlot][atomicAdd(&S.frontCount[nextSlot], 1u)] = make_uint4(child + c, clf, ccnt, depth + 1);
  }
  s.nodeChild[id] = int32_t(child);
  atomicMax(&s.g->maxDepth, depth + 1);
}

__global__ void __launch_bounds__(kThreads) k_small(Scratch s, int B) {
  extern __shared__ __align__(16) unsigned char smem[];
  SmallShared S = carveShared(smem, B);
  const uint32_t root = s.smallQ[blockIdx.x];
  const uint32_t rootFirst = s.nodeFirst[root], n = s.nodeCount[root];
  for (uint32_t i = threadIdx.x; i < n; i += kThreads) {
    uint32_t p = s.prim[rootFirst + i];
    S.global[i] = p;
    S.perm[i] = i;
    for (int k = 0; k < 6; k++) S.aabb[i * 6 + k] = s.aabb[size_t(p) * 6 + k];
    for (int k = 0; k < 3; k++) S.center[i * 3 + k] = s.center[size_t(p) * 3 + k];
  }
  double minDim[3] = {s.g->minDim[0], s.g->minDim[1], s.g->minDim[2]};
  if (threadIdx.x == 0) {
    S.front[0][0] = make_uint4(root, 0, n, s.nodeDepth[root]);
    S.frontCount[0] = 1;
  }
  __syncthreads();
  int cur = 0;
  uint32_t fcount = 1;
  while (fcount) {
    if (threadIdx.x == 0) S.frontCount[cur ^ 1] = 0;
    __syncthreads();
    for (uint32_t f = threadIdx.x >> 5; f < fcount; f += kWarps)
      splitNodeWarp(s, S, S.front[cur][f], rootFirst, B, minDim, cur ^ 1);
    __syncthreads();
    cur ^= 1;
    fcount = S.frontCount[cur];
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < n; i += kThreads) s.prim[rootFirst + i] = S.global[S.perm[i]];
}

// ------------------------------------------------------------ layout
__global__ void k_depth_hist(Scratch s, uint32_t nodeCount) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nodeCount) atomicAdd(&s.depthCursor[s.nodeDepth[i]], 1u);
}

__global__ void k_depth_scatter(Scratch s, uint32_t nodeCount) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nodeCount) s.byDepth[atomicAdd(&s.depthCursor[s.nodeDepth[i]], 1u)] = i;
}

// Subtree length in vec4 (2 per node plus one per leaf primitive), one depth.
__global__ void k_size_level(Scratch s, const uint32_t *nodes, uint32_t count) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  uint32_t node = nodes[i];
  int32_t child = s.nodeChild[node];
  if (child < 0) {
    s.nodeSize[node] = 2 + s.nodeCount[node];
    atomicMax(&s.g->maxLeaf, s.nodeCount[node]);
  } else {
    s.nodeSize[node] = 2 + s.nodeSize[child] + s.nodeSize[child + 1];
  }
}

// Writes one depth of the depth-first layout (binnedSahBvh.ts:252-275 and the
// packing of bvhAccel.ts:244-273) and places the children of its nodes.
__global__ void k_emit_level(Scratch s, const uint32_t *nodes, uint32_t count, float4 *out, const uint32_t *idx) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  uint32_t node = nodes[i], o = s.nodeOffset[node];
  const float *b = s.nodeBounds + size_t(node) * 6;
  int32_t child = s.nodeChild[node], w;
  if (child >= 0) {
    uint32_t right = o + 2 + s.nodeSize[child];
    s.nodeOffset[child] = o + 2;
    s.nodeOffset[child + 1] = right;
    w = int32_t(right);
  } else {
    uint32_t first = s.nodeFirst[node], prims = s.nodeCount[node];
    w = -int32_t(prims);
    for (uint32_t k = 0; k < prims; k++) {
      uint32_t t = s.tri[s.prim[first + k]];
      out[o + 2 + k] = make_float4(__uint_as_float(idx[size_t(t) * 3]), __uint_as_float(idx[size_t(t) * 3 + 1]),
                                   __uint_as_float(idx[size_t(t) * 3 + 2]), 0.0f);
    }
  }
  out[o] = make_float4(b[0], b[1], b[2], __int_as_float(w));
  out[o + 1] = make_float4(b[3], b[4], b[5], 0.0f);
}

// ------------------------------------------------------------ host glue
mt_status cudaStatus(cudaError_t e) {
  if (e == cudaSuccess) return MT_OK;
  if (e == cudaErrorInvalidValue || e == cudaErrorInvalidDevicePointer) return MT_ERROR_INVALID_ARGUMENT;
  return MT_ERROR;
}

struct HostSync {
  cudaStream_t stream;
  uint32_t syncs = 0;
  template <class T>
  cudaError_t read(T *dst, const T *src, size_t count = 1) {
    cudaError_t e = cudaMemcpyAsync(dst, src, sizeof(T) * count, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    syncs++;
    return e;
  }
};

#define MT_TRY(expr)                            \
  do {                                          \
    cudaError_t e_ = (expr);                    \
    if (e_ != cudaSuccess) return cudaStatus(e_); \
  } while (0)
#define MT_LAUNCHED() MT_TRY(cudaGetLastError())

}  // namespace

extern "C" {

uint64_t mtc_blas_build_scratch_bytes(uint32_t triangle_count, uint32_t bins) {
  if (bins < 1 || bins > uint32_t(kMaxBins) || triangle_count > kMaxTriangles) return 0;
  Scratch s;
  return carve(s, nullptr, triangle_count, bins);
}

uint64_t mtc_blas_build_max_vec4(uint32_t triangle_count) {
  return triangle_count ? 5ull * triangle_count - 2 : 0;
}

mt_status mtc_build_blas(const mtc_blas_build_input *input, void *scratch, uint64_t scratch_bytes, float *out_bvh,
                         uint64_t out_capacity_vec4, mtc_blas_build_result *result, void *stream) {
  if (!input || input->struct_size != sizeof(mtc_blas_build_input) || !result ||
      result->struct_size != sizeof(mtc_blas_build_result))
    return MT_ERROR_INVALID_ARGUMENT;
  const uint32_t n = input->triangle_count, B = input->bins;
  if (B < 1 || B > uint32_t(kMaxBins) || n > kMaxTriangles) return MT_ERROR_INVALID_ARGUMENT;
  if (n && (!input->indices || (input->vertex_count && !input->positions))) return MT_ERROR_INVALID_ARGUMENT;
  std::memset(reinterpret_cast<char *>(result) + sizeof(uint32_t), 0, sizeof(*result) - sizeof(uint32_t));
  for (int k = 0; k < 3; k++) {
    result->local_bounds[k] = INFINITY;
    result->local_bounds[3 + k] = -INFINITY;
  }
  if (!n) return MT_OK;
  Scratch s;
  if (!scratch || scratch_bytes < carve(s, nullptr, n, B) || reinterpret_cast<uintptr_t>(scratch) % 256 ||
      reinterpret_cast<uintptr_t>(out_bvh) % 16)
    return MT_ERROR_INVALID_ARGUMENT;
  carve(s, static_cast<char *>(scratch), n, B);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  HostSync hs{st};
  const float *pos = input->positions;
  const uint32_t *idx = input->indices, vc = input->vertex_count;
  const uint32_t blocks = (n + kChunk - 1) / kChunk;

  k_init<<<1, 1, 0, st>>>(s.g);
  k_count_finite<<<blocks, kThreads, 0, st>>>(s, pos, idx, vc, n);
  k_scan<<<1, 1024, 0, st>>>(s.blockSum, nullptr, blocks, &s.g->primCount);
  k_compact<<<blocks, kThreads, 0, st>>>(s, pos, idx, vc, n);
  k_root_keys<<<std::min<uint32_t>(blocks * 8, 148 * 8), kThreads, 0, st>>>(s);
  k_root_finalize<<<1, 1, 0, st>>>(s);
  MT_LAUNCHED();
  Globals g;
  MT_TRY(hs.read(&g, s.g));
  if (!g.primCount) {
    result->host_syncs = hs.syncs;
    return MT_OK;
  }

  // Level-synchronous top of the tree.
  const size_t binSmem = size_t(21) * B * 4;
  uint32_t active = g.activeNext, *cur = s.activeA, *next = s.activeB;
  while (active) {
    uint32_t grid = n / kChunk + 1 + active;
    k_large_setup<<<1, 1024, 0, st>>>(s, cur, active, int(B));
    k_large_bin<<<grid, kThreads, binSmem, st>>>(s, active, int(B));
    k_large_sah<<<(active + kWarps - 1) / kWarps, kThreads, 0, st>>>(s, active, int(B));
    k_large_classify<<<grid, kThreads, 0, st>>>(s, active, int(B));
    k_scan<<<1, 1024, 0, st>>>(s.chunkR, &s.g->totalChunks, 0, nullptr);
    k_large_rank<<<grid, kThreads, 0, st>>>(s, active, int(B));
    k_large_scatter<<<grid, kThreads, 0, st>>>(s, active);
    k_large_copy<<<grid, kThreads, 0, st>>>(s, active);
    k_large_children<<<(active + kThreads - 1) / kThreads, kThreads, 0, st>>>(s, active, next);
    MT_LAUNCHED();
    MT_TRY(hs.read(&g, s.g));
    active = g.activeNext;
    std::swap(cur, next);
  }

  // Subtrees of at most kSmallLimit primitives, one CTA each.
  if (g.smallCount) {
    size_t smem = smallSharedBytes(int(B));
    MT_TRY(cudaFuncSetAttribute(k_small, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    k_small<<<g.smallCount, kThreads, smem, st>>>(s, int(B));
    MT_LAUNCHED();
  }
  MT_TRY(hs.read(&g, s.g));
  if (g.error) {
    result->host_syncs = hs.syncs;
    return MT_ERROR;
  }
  const uint32_t nodes = g.nodeAlloc, maxDepth = g.maxDepth;

  // Nodes by depth, then sizes bottom up and offsets top down.
  MT_TRY(cudaMemsetAsync(s.depthCursor, 0, sizeof(uint32_t) * (maxDepth + 2), st));
  const uint32_t nodeBlocks = (nodes + 255) / 256;
  k_depth_hist<<<nodeBlocks, 256, 0, st>>>(s, nodes);
  MT_LAUNCHED();
  std::vector<uint32_t> hist(maxDepth + 2), base(maxDepth + 2);
  MT_TRY(hs.read(hist.data(), s.depthCursor, maxDepth + 2));
  uint32_t running = 0;
  for (uint32_t d = 0; d < maxDepth + 2; d++) {
    base[d] = running;
    running += hist[d];
  }
  MT_TRY(cudaMemcpyAsync(s.depthCursor, base.data(), sizeof(uint32_t) * (maxDepth + 2), cudaMemcpyHostToDevice, st));
  k_depth_scatter<<<nodeBlocks, 256, 0, st>>>(s, nodes);
  for (uint32_t d = maxDepth; d >= 1; d--)
    if (hist[d]) k_size_level<<<(hist[d] + 255) / 256, 256, 0, st>>>(s, s.byDepth + base[d], hist[d]);
  MT_LAUNCHED();
  uint32_t rootSize = 0;
  MT_TRY(hs.read(&rootSize, s.nodeSize));
  MT_TRY(hs.read(&g, s.g));
  float rootBox[6];
  MT_TRY(hs.read(rootBox, s.nodeBounds, 6));
  result->vec4_count = rootSize;
  result->max_depth = maxDepth;
  result->max_leaf_primitives = g.maxLeaf;
  result->node_count = nodes;
  result->primitive_count = g.primCount;
  for (int k = 0; k < 6; k++) result->local_bounds[k] = rootBox[k];
  if (!out_bvh || rootSize > out_capacity_vec4) {
    result->host_syncs = hs.syncs;
    return MT_ERROR_BUFFER_TOO_SMALL;
  }
  MT_TRY(cudaMemsetAsync(s.nodeOffset, 0, sizeof(uint32_t), st));
  for (uint32_t d = 1; d <= maxDepth; d++)
    if (hist[d])
      k_emit_level<<<(hist[d] + 255) / 256, 256, 0, st>>>(s, s.byDepth + base[d], hist[d],
                                                        reinterpret_cast<float4 *>(out_bvh), idx);
  MT_LAUNCHED();
  MT_TRY(cudaStreamSynchronize(st));
  result->host_syncs = hs.syncs + 1;
  return MT_OK;
}

}  // extern "C"
