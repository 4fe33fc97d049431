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

constexpr uint32_t kSmallLimit = 256;   // subtree roots this small are finished by one warp
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
  uint32_t holes, pad;                                 // node ids reserved by subtree warps and left unused
  double minDim[3];
  unsigned long long rootKey[6];
};

enum : uint32_t { kLeaf = 0, kSplit = 1, kPartitionLeaf = 2, kBinned = 3 };

// One node of the level-synchronous phase.
struct LargeNode {
  double nMin[3], scale[3];
  float childBounds[12];
  uint32_t node, first, count, depth;
  uint32_t leftN, state;
  int32_t axis, pos;
};

struct Scratch {
  Globals *g;
  float *aabb, *center;
  uint32_t *tri, *prim, *tmp, *rank, *rf, *lb, *blockSum;
  float *nodeBounds;
  uint32_t *nodeFirst, *nodeCount, *nodeDepth, *nodeSize, *nodeOffset, *byDepth, *depthCursor;
  int32_t *nodeChild;
  uint32_t *activeA, *activeB, *smallQ, *chunkR, *chunkStart, *bins;
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
  s.chunkStart = take<uint32_t>(base, off, size_t(s.maxActive) + 1);
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
  if (fabs(v) < 2147483648.0) return __double2int_rz(v);  // NaN fails the test
  if (!(v == v) || isinf(v)) return 0;
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
// Surface-area term of binnedSahBvh.ts:177-178 for bounds given as ordered
// keys: the reference's running bounds start at FAR / -FAR, hence the clamps.
// Math.min(FAR, v) / Math.max(-FAR, v) for a finite f32 v (never equal to FAR).
__device__ __forceinline__ double farMin(float v) { return double(v) < kFar ? double(v) : kFar; }
__device__ __forceinline__ double farMax(float v) { return double(v) > -kFar ? double(v) : -kFar; }
__device__ __forceinline__ double keyArea(uint32_t lo0, uint32_t lo1, uint32_t lo2, uint32_t hi0, uint32_t hi1,
                                          uint32_t hi2) {
  double x = DA(farMax(keyValue(hi0)), -farMin(keyValue(lo0)));
  double y = DA(farMax(keyValue(hi1)), -farMin(keyValue(lo1)));
  double z = DA(farMax(keyValue(hi2)), -farMin(keyValue(lo2)));
  return areaOf(x, y, z);
}

struct Decision {
  uint32_t state, leftN;
  int32_t axis, pos;
  float laneBound;  // lane j < 12: component j of the child boxes (left min xyz, max xyz, then right)
};

// The bins of one node: counts[3B], min keys[3B*3], max keys[3B*3].
struct BinView {
  const uint32_t *w;
  int B;
};

// binnedSahBvh.ts:154-183 (sweep), :184-187 (leaf test) and :211-225 (child
// boxes), one warp per node.  The reference sweeps each axis keeping running
// bounds; Math.min/max are exact, so each split candidate (axis, position) is
// evaluated on its own lane from its bins directly (the side bounds as min/max
// of ordered keys, then the same float64 operations on the same values), and
// the warp keeps the first candidate in the reference's (axis, position) order
// among the cheapest, as its strict `<` does.  The child boxes are 12 lanes, each folding its side's bins in bin
// order with the reference's strict comparison against the f32-stored box.
// Every lane returns the decision.
__device__ Decision decideSplit(const BinView &bins, const float nb[6], uint32_t count, const double minDim[3]) {
  const int B = bins.B, lane = threadIdx.x & 31, candidates = 3 * (B - 1);
  double ext[3];
  uint32_t splittable = 0;  // axes with extent > minDim (binnedSahBvh.ts:159)
  for (int k = 0; k < 3; k++) {
    ext[k] = DA(double(nb[3 + k]), -double(nb[k]));
    splittable |= uint32_t(ext[k] > minDim[k]) << k;
  }
  double bestCost = INFINITY;
  int bestKey = candidates;
  for (int c = lane; c < candidates; c += 32) {
    const int axis = c / (B - 1), pos = c - axis * (B - 1);
    if (!(splittable >> axis & 1u)) continue;
    // Bounds of each side as ordered keys (their min/max are Math.min/max
    // of the values); an empty side costs FAR whatever its bounds.
    uint32_t lLo0 = kMinIdentity, lLo1 = kMinIdentity, lLo2 = kMinIdentity;
    uint32_t lHi0 = kMaxIdentity, lHi1 = kMaxIdentity, lHi2 = kMaxIdentity;
    uint32_t rLo0 = kMinIdentity, rLo1 = kMinIdentity, rLo2 = kMinIdentity;
    uint32_t rHi0 = kMaxIdentity, rHi1 = kMaxIdentity, rHi2 = kMaxIdentity;
    uint32_t nLeft = 0, nRight = 0;
    for (int i = 0; i < B; i++) {
      const int bin = axis * B + i;
      const uint32_t *lo = bins.w + 3 * B + bin * 3, *hi = bins.w + 12 * B + bin * 3;
      if (i <= pos) {
        nLeft += bins.w[bin];
        lLo0 = min(lLo0, lo[0]); lLo1 = min(lLo1, lo[1]); lLo2 = min(lLo2, lo[2]);
        lHi0 = max(lHi0, hi[0]); lHi1 = max(lHi1, hi[1]); lHi2 = max(lHi2, hi[2]);
      } else {
        nRight += bins.w[bin];
        rLo0 = min(rLo0, lo[0]); rLo1 = min(rLo1, lo[1]); rLo2 = min(rLo2, lo[2]);
        rHi0 = max(rHi0, hi[0]); rHi1 = max(rHi1, hi[1]); rHi2 = max(rHi2, hi[2]);
      }
    }
    double sideCost[2] = {kFar, kFar};
    if (nLeft) sideCost[0] = DM(keyArea(lLo0, lLo1, lLo2, lHi0, lHi1, lHi2), double(nLeft));
    if (nRight) sideCost[1] = DM(keyArea(rLo0, rLo1, rLo2, rHi0, rHi1, rHi2), double(nRight));
    double cost = DA(sideCost[0], sideCost[1]);
    if (cost < bestCost) {  // candidates of a lane come in increasing order
      bestCost = cost;
      bestKey = c;
    }
  }
  for (int o = 16; o; o >>= 1) {
    double oc = __shfl_xor_sync(0xffffffffu, bestCost, o);
    int ok = __shfl_xor_sync(0xffffffffu, bestKey, o);
    if (oc < bestCost || (oc == bestCost && ok < bestKey)) {
      bestCost = oc;
      bestKey = ok;
    }
  }
  Decision d;
  d.state = kLeaf;
  d.leftN = 0;
  d.axis = 0;
  d.pos = 0;
  double split = kFar;
  if (bestCost < kFar) {
    split = bestCost;
    d.axis = bestKey / (B - 1);
    d.pos = bestKey - d.axis * (B - 1);
  }
  split = DA(1.0, __ddiv_rn(split, areaOf(ext[0], ext[1], ext[2])));  // C_TRAV + C_INT * cost / area
  if (!(split < double(count))) return d;
  uint32_t leftN = 0;
  for (int i = 0; i <= d.pos; i++) leftN += bins.w[d.axis * B + i];
  d.leftN = leftN;
  d.state = (leftN == 0 || leftN == count) ? kPartitionLeaf : kSplit;
  // Child boxes (binnedSahBvh.ts:215-224): the box starts at f32(FAR) and
  // takes a bin's bound when strictly smaller.  An empty bin's FAR, or a
  // bound at or beyond FAR, stores f32(FAR) again, so only the non-empty
  // bins' f32 values matter, clamped to f32(FAR); the first of equal values
  // stays.
  float v = 0.0f;
  if (lane < 12) {
    const int side = lane / 6, comp = lane % 6, k = comp % 3;
    const bool isMax = comp >= 3;
    const float far = float(kFar);
    v = isMax ? -far : far;
    const uint32_t *keys = bins.w + (isMax ? 12 * B : 3 * B) + k;
    for (int i = side ? d.pos + 1 : 0; i < (side ? B : d.pos + 1); i++) {
      const int bin = d.axis * B + i;
      if (!bins.w[bin]) continue;
      float x = keyValue(keys[bin * 3]);
      if (isMax) {
        x = x > -far ? x : -far;
        if (x > v) v = x;
      } else {
        x = x < far ? x : far;
        if (x < v) v = x;
      }
    }
  }
  d.laneBound = v;
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
  g->holes = 0;
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
// Per active node: split parameters, a fresh set of bins, and its chunk count
// (chunkStart, scanned into each node's first chunk afterwards).
__global__ void __launch_bounds__(kThreads) k_large_setup(Scratch s, const uint32_t *active, uint32_t activeCount,
                                                          int B) {
  uint32_t a = blockIdx.x * kThreads + threadIdx.x;
  if (a == 0) s.g->activeNext = 0;
  if (a >= activeCount) return;
  LargeNode &L = s.large[a];
  uint32_t node = active[a], chunks = 0;
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
  s.chunkStart[a] = chunks;
  initBins(s.bins + size_t(a) * s.binWords, B, 0, 1);
}

// Node of chunk c: the last node whose first chunk is <= c (nodes without
// chunks share their first chunk with the next node).
__device__ uint32_t chunkNode(const Scratch &s, uint32_t activeCount, uint32_t c) {
  uint32_t lo = 0, hi = activeCount;
  while (hi - lo > 1) {
    uint32_t mid = (lo + hi) / 2;
    if (s.chunkStart[mid] <= c) lo = mid;
    else hi = mid;
  }
  return lo;
}

__global__ void __launch_bounds__(kThreads) k_large_bin(Scratch s, uint32_t activeCount, int B) {
  extern __shared__ uint32_t sBins[];
  uint32_t c = blockIdx.x;
  if (c >= s.g->totalChunks) return;
  const uint32_t a = chunkNode(s, activeCount, c), cb = s.chunkStart[a];
  const LargeNode &L = s.large[a];
  double nMin[3], scale[3];
  for (int k = 0; k < 3; k++) {
    nMin[k] = L.nMin[k];
    scale[k] = L.scale[k];
  }
  initBins(sBins, B, threadIdx.x, kThreads);
  __syncthreads();
  uint32_t begin = (c - cb) * kChunk, end = min(begin + kChunk, L.count);
  for (uint32_t i = begin + threadIdx.x; i < end; i += kThreads) {
    uint32_t p = s.prim[L.first + i];
    addToBins(sBins, B, s.center + size_t(p) * 3, s.aabb + size_t(p) * 6, nMin, scale);
  }
  __syncthreads();
  uint32_t *G = s.bins + size_t(a) * s.binWords;
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
  const int warp = threadIdx.x >> 5;
  uint32_t a = blockIdx.x * kWarps + warp;
  if (a >= activeCount) return;
  LargeNode &L = s.large[a];
  if (L.state != kBinned) return;
  BinView bins{s.bins + size_t(a) * s.binWords, B};
  double minDim[3] = {s.g->minDim[0], s.g->minDim[1], s.g->minDim[2]};
  Decision d = decideSplit(bins, s.nodeBounds + size_t(L.node) * 6, L.count, minDim);
  if ((threadIdx.x & 31) < 12) L.childBounds[threadIdx.x & 31] = d.laneBound;
  if ((threadIdx.x & 31) == 0) {
    L.state = d.state;
    L.axis = d.axis;
    L.pos = d.pos;
    L.leftN = d.leftN;
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
  const uint32_t a = chunkNode(s, activeCount, c), cb = s.chunkStart[a];
  const LargeNode &L = s.large[a];
  uint32_t cnt = 0;
  if (partitions(L.state)) {
    uint32_t begin = (c - cb) * kChunk, end = min(begin + kChunk, L.count);
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
  const uint32_t a = chunkNode(s, activeCount, c), cb = s.chunkStart[a];
  const LargeNode &L = s.large[a];
  if (!partitions(L.state)) return;
  uint32_t begin = (c - cb) * kChunk, end = min(begin + kChunk, L.count);
  uint32_t i0 = begin + threadIdx.x * kPerThread, bits = 0, cnt = 0;
  for (int j = 0; j < kPerThread; j++) {
    uint32_t i = i0 + j;
    if (i < end && goesRight(s, L, i, B)) {
      bits |= 1u << j;
      cnt++;
    }
  }
  uint32_t total;
  uint32_t prefR = s.chunkR[c] - s.chunkR[cb] + blockExclusiveSum<kThreads>(cnt, total);
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
  const uint32_t a = chunkNode(s, activeCount, c), cb = s.chunkStart[a];
  const LargeNode &L = s.large[a];
  if (!partitions(L.state)) return;
  uint32_t begin = (c - cb) * kChunk, end = min(begin + kChunk, L.count);
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
  const uint32_t a = chunkNode(s, activeCount, c), cb = s.chunkStart[a];
  const LargeNode &L = s.large[a];
  if (!partitions(L.state)) return;
  uint32_t begin = (c - cb) * kChunk, end = min(begin + kChunk, L.count);
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

// ------------------------------------------------ per-warp subtree phase
constexpr int kSubtreeWarps = 4;  // warps (independent subtrees) per CTA

// Shared memory of one warp: centroids, the subtree's primitive ids, its
// working permutation, the partition scratch (tmp, and rf | lb side by side),
// the DFS stack and the bins.
struct WarpShared {
  float *center, *stackBounds;
  uint32_t *global, *perm, *tmp, *ranks, *bins;
  uint4 *stack;
};

// Pending nodes hold at least two primitives each, in disjoint ranges.
constexpr uint32_t kStackDepth = kSmallLimit / 2 + 1;

__host__ __device__ inline size_t warpSharedBytes(int B) {
  return (size_t(kStackDepth) * (sizeof(uint4) + 6 * 4) + size_t(kSmallLimit) * (3 * 4 + 4 * 4) + size_t(21) * B * 4 +
          15) / 16 * 16;
}

__device__ WarpShared carveWarp(unsigned char *base, int B) {
  WarpShared S;
  S.stack = reinterpret_cast<uint4 *>(base);
  S.stackBounds = reinterpret_cast<float *>(base + kStackDepth * sizeof(uint4));
  S.center = S.stackBounds + kStackDepth * 6;
  S.global = reinterpret_cast<uint32_t *>(S.center + kSmallLimit * 3);
  S.perm = S.global + kSmallLimit;
  S.tmp = S.perm + kSmallLimit;
  S.ranks = S.tmp + kSmallLimit;
  S.bins = S.ranks + kSmallLimit;
  return S;
}

// One warp builds the whole subtree under a node of at most kSmallLimit
// primitives, depth first (children are pushed right then left, so the stack
// holds at most one pending node per level).  Node ids come from a block of
// 2n - 2 reserved up front; ids left unused are marked depth 0 (holes the
// layout skips).
__global__ void __launch_bounds__(kSubtreeWarps * 32) k_subtree(Scratch s, uint32_t rootCount, int B) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t task = blockIdx.x * kSubtreeWarps + warp;
  if (task >= rootCount) return;
  WarpShared S = carveWarp(smem + size_t(warp) * warpSharedBytes(B), B);
  const uint32_t root = s.smallQ[task], rootFirst = s.nodeFirst[root], n = s.nodeCount[root];
  for (uint32_t i = lane; i < n; i += 32) {
    uint32_t p = s.prim[rootFirst + i];
    S.global[i] = p;
    S.perm[i] = i;
    for (int k = 0; k < 3; k++) S.center[i * 3 + k] = s.center[size_t(p) * 3 + k];
  }
  const double minDim[3] = {s.g->minDim[0], s.g->minDim[1], s.g->minDim[2]};
  uint32_t idBase = 0;
  if (lane == 0) idBase = atomicAdd(&s.g->nodeAlloc, 2 * n - 2);
  idBase = __shfl_sync(0xffffffffu, idBase, 0);
  uint32_t used = 0, top = 0, maxDepth = 0;
  if (lane == 0) S.stack[0] = make_uint4(root, 0, n, s.nodeDepth[root]);
  if (lane < 6) S.stackBounds[lane] = s.nodeBounds[size_t(root) * 6 + lane];
  top = 1;
  __syncwarp();
  while (top) {
    const uint4 e = S.stack[--top];
    float nb[6];
    for (int k = 0; k < 6; k++) nb[k] = S.stackBounds[top * 6 + k];
    __syncwarp();
    const uint32_t id = e.x, lf = e.y, cnt = e.z, depth = e.w;
    double nMin[3], ext[3], scale[3];
    for (int k = 0; k < 3; k++) {
      nMin[k] = nb[k];
      ext[k] = DA(double(nb[3 + k]), -nMin[k]);
      scale[k] = ext[k] > minDim[k] ? __ddiv_rn(double(B), ext[k]) : 0.0;
    }
    if (areaOf(ext[0], ext[1], ext[2]) == 0.0) continue;
    initBins(S.bins, B, lane, 32);
    __syncwarp();
    for (uint32_t i = lane; i < cnt; i += 32) {
      uint32_t li = S.perm[lf + i];
      addToBins(S.bins, B, S.center + li * 3, s.aabb + size_t(S.global[li]) * 6, nMin, scale);
    }
    __syncwarp();
    const Decision d = decideSplit(BinView{S.bins, B}, nb, cnt, minDim);
    if (d.state == kLeaf) continue;
    const int axis = d.axis;
    const double axisMin = axis == 0 ? nMin[0] : (axis == 1 ? nMin[1] : nMin[2]);
    const double axisScale = axis == 0 ? scale[0] : (axis == 1 ? scale[1] : scale[2]);
    const uint32_t nL = d.leftN, nR = cnt - nL;
    uint32_t *rf = S.ranks + lf, *lb = S.ranks + lf + nR;
    // Pass 1: sides (kept as ballots), ranks and the rf / lb tables.
    uint32_t ballots[kSmallLimit / 32];
    uint32_t prefix = 0;
#pragma unroll
    for (int j = 0; j < int(kSmallLimit / 32); j++) {
      const uint32_t i = j * 32 + lane;
      if (j * 32u >= cnt) break;
      bool right = i < cnt && binOf(S.center[S.perm[lf + i] * 3 + axis], axisMin, axisScale, B) > d.pos;
      ballots[j] = __ballot_sync(0xffffffffu, right);
      uint32_t prefR = prefix + __popc(ballots[j] & ((1u << lane) - 1));
      if (i < cnt) {
        uint32_t slot = right ? prefR : nL - (i - prefR) - 1;
        if (slot >= (right ? nR : nL)) s.g->error = 1;
        else if (right) rf[slot] = i;
        else lb[slot] = i;
      }
      prefix += __popc(ballots[j]);
    }
    __syncwarp();
    // Pass 2: the permutation, into tmp; then back.
    prefix = 0;
#pragma unroll
    for (int j = 0; j < int(kSmallLimit / 32); j++) {
      const uint32_t i = j * 32 + lane;
      if (j * 32u >= cnt) break;
      const bool right = ballots[j] >> lane & 1u;
      uint32_t prefR = prefix + __popc(ballots[j] & ((1u << lane) - 1));
      if (i < cnt) {
        uint32_t dest = partitionDest(i, right, prefR, cnt, nL, rf, lb);
        if (dest < cnt) S.tmp[lf + dest] = S.perm[lf + i];
        else s.g->error = 1;
      }
      prefix += __popc(ballots[j]);
    }
    __syncwarp();
    for (uint32_t i = lane; i < cnt; i += 32) S.perm[lf + i] = S.tmp[lf + i];
    __syncwarp();
    if (d.state != kSplit) continue;
    const uint32_t child = idBase + used;
    used += 2;
    if (lane < 12) s.nodeBounds[size_t(child) * 6 + lane] = d.laneBound;
    if (lane < 2) {
      const uint32_t c = child + lane;
      s.nodeFirst[c] = rootFirst + lf + (lane ? nL : 0);
      s.nodeCount[c] = lane ? nR : nL;
      s.nodeDepth[c] = depth + 1;
      s.nodeChild[c] = -1;
    }
    if (lane == 0) {
      s.nodeChild[id] = int32_t(child);
      if (nR >= 2) S.stack[top] = make_uint4(child + 1, lf + nL, nR, depth + 1);
      if (nL >= 2) S.stack[top + (nR >= 2)] = make_uint4(child, lf, nL, depth + 1);
    }
    if (lane < 6 && nL >= 2) S.stackBounds[(top + (nR >= 2)) * 6 + lane] = d.laneBound;
    if (lane >= 6 && lane < 12 && nR >= 2) S.stackBounds[top * 6 + lane - 6] = d.laneBound;
    top += (nR >= 2) + (nL >= 2);
    maxDepth = max(maxDepth, depth + 1);
    __syncwarp();
  }
  for (uint32_t i = lane; i < n; i += 32) s.prim[rootFirst + i] = S.global[S.perm[i]];
  for (uint32_t i = used + lane; i < 2 * n - 2; i += 32) s.nodeDepth[idBase + i] = 0;
  if (lane == 0) {
    if (maxDepth) atomicMax(&s.g->maxDepth, maxDepth);
    if (used < 2 * n - 2) atomicAdd(&s.g->holes, 2 * n - 2 - used);
  }
}

// ------------------------------------------------------------ layout
// Nodes by depth: per-CTA counts in shared memory (depths <= depthCount),
// then one global reservation per (CTA, depth).
constexpr uint32_t kDepthNodes = 2048;  // nodes per CTA
constexpr uint32_t kMaxSharedDepths = 8192;

__global__ void __launch_bounds__(kThreads) k_depth_hist(Scratch s, uint32_t nodeCount, uint32_t depthCount) {
  extern __shared__ uint32_t hist[];
  for (uint32_t d = threadIdx.x; d < depthCount; d += kThreads) hist[d] = 0;
  __syncthreads();
  uint32_t end = min(nodeCount, (blockIdx.x + 1) * kDepthNodes);
  for (uint32_t i = blockIdx.x * kDepthNodes + threadIdx.x; i < end; i += kThreads) atomicAdd(&hist[s.nodeDepth[i]], 1u);
  __syncthreads();
  for (uint32_t d = threadIdx.x; d < depthCount; d += kThreads)
    if (hist[d]) atomicAdd(&s.depthCursor[d], hist[d]);
}

__global__ void __launch_bounds__(kThreads) k_depth_scatter(Scratch s, uint32_t nodeCount, uint32_t depthCount) {
  extern __shared__ uint32_t hist[];
  for (uint32_t d = threadIdx.x; d < depthCount; d += kThreads) hist[d] = 0;
  __syncthreads();
  const uint32_t begin = blockIdx.x * kDepthNodes, end = min(nodeCount, begin + kDepthNodes);
  uint32_t rank[kDepthNodes / kThreads];
  for (int j = 0; j < int(kDepthNodes / kThreads); j++) {
    uint32_t i = begin + j * kThreads + threadIdx.x;
    if (i < end) rank[j] = atomicAdd(&hist[s.nodeDepth[i]], 1u);
  }
  __syncthreads();
  for (uint32_t d = threadIdx.x; d < depthCount; d += kThreads)
    if (hist[d]) hist[d] = atomicAdd(&s.depthCursor[d], hist[d]);
  __syncthreads();
  for (int j = 0; j < int(kDepthNodes / kThreads); j++) {
    uint32_t i = begin + j * kThreads + threadIdx.x;
    if (i < end) s.byDepth[hist[s.nodeDepth[i]] + rank[j]] = i;
  }
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
    k_large_setup<<<(active + kThreads - 1) / kThreads, kThreads, 0, st>>>(s, cur, active, int(B));
    k_scan<<<1, 1024, 0, st>>>(s.chunkStart, nullptr, active, &s.g->totalChunks);
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

  // Subtrees of at most kSmallLimit primitives, one warp each.
  if (g.smallCount) {
    size_t smem = warpSharedBytes(int(B)) * kSubtreeWarps;
    MT_TRY(cudaFuncSetAttribute(k_subtree, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    k_subtree<<<(g.smallCount + kSubtreeWarps - 1) / kSubtreeWarps, kSubtreeWarps * 32, smem, st>>>(s, g.smallCount,
                                                                                                  int(B));
    MT_LAUNCHED();
  }
  MT_TRY(hs.read(&g, s.g));
  if (g.error) {
    result->host_syncs = hs.syncs;
    return MT_ERROR;
  }
  const uint32_t nodes = g.nodeAlloc, maxDepth = g.maxDepth;

  // Nodes by depth, then sizes bottom up and offsets top down.
  const uint32_t depthCount = maxDepth + 2;
  if (depthCount > kMaxSharedDepths) return MT_ERROR_UNAVAILABLE;  // a BVH this deep has no traversal stack anyway
  MT_TRY(cudaMemsetAsync(s.depthCursor, 0, sizeof(uint32_t) * depthCount, st));
  const uint32_t nodeBlocks = (nodes + kDepthNodes - 1) / kDepthNodes;
  const size_t depthSmem = sizeof(uint32_t) * depthCount;
  MT_TRY(cudaFuncSetAttribute(k_depth_hist, cudaFuncAttributeMaxDynamicSharedMemorySize, int(depthSmem)));
  MT_TRY(cudaFuncSetAttribute(k_depth_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize, int(depthSmem)));
  k_depth_hist<<<nodeBlocks, kThreads, depthSmem, st>>>(s, nodes, depthCount);
  MT_LAUNCHED();
  std::vector<uint32_t> hist(maxDepth + 2), base(maxDepth + 2);
  MT_TRY(hs.read(hist.data(), s.depthCursor, maxDepth + 2));
  uint32_t running = 0;
  for (uint32_t d = 0; d < maxDepth + 2; d++) {
    base[d] = running;
    running += hist[d];
  }
  MT_TRY(cudaMemcpyAsync(s.depthCursor, base.data(), sizeof(uint32_t) * (maxDepth + 2), cudaMemcpyHostToDevice, st));
  k_depth_scatter<<<nodeBlocks, kThreads, depthSmem, st>>>(s, nodes, depthCount);
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
  result->node_count = nodes - g.holes;
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
