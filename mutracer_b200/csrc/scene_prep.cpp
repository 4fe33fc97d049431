// Host-side producers of the megakernel's input buffers; see scene_prep.h.
#include "scene_prep.h"
#include "js_minmax.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <limits>
#include <map>
#include <stdexcept>
#include <thread>
#include <unordered_map>

namespace mtp {

static inline float asFloat(int32_t i) { float f; std::memcpy(&f, &i, 4); return f; }
static inline float asFloatU(uint32_t i) { float f; std::memcpy(&f, &i, 4); return f; }
static inline int32_t asInt(float f) { int32_t i; std::memcpy(&i, &f, 4); return i; }

// JavaScript `value | 0` for a double in the binning range (NaN -> 0).
static inline int32_t toInt32(double v) {
  if (!(v == v) || std::isinf(v)) return 0;
  double t = std::trunc(v);
  double m = std::fmod(t, 4294967296.0);
  if (m < 0) m += 4294967296.0;
  uint32_t u = uint32_t(m);
  return int32_t(u);
}

// ------------------------------------------------------------ binned SAH
// Restates buildBinnedSahBvh of src/renderer/binnedSahBvh.ts:70-236 (float64
// arithmetic on f32-stored bounds and centroids).
BinnedBvh buildBinnedSahBvh(const float *aabbs, uint32_t count, int bins) {
  const int BINS = bins;
  const double FAR = 1e30;
  BinnedBvh r;
  uint32_t capacity = std::max<uint32_t>(1u, count * 2u - (count ? 1u : 0u));
  r.bounds.assign(size_t(capacity) * 6, 0.0f);
  r.leftFirst.assign(capacity, 0);
  r.primCount.assign(capacity, 0);
  r.primIndices.assign(count, 0);
  if (count == 0) { r.nodeCount = 0; return r; }
  std::vector<float> centers(size_t(count) * 3);
  double rMinX = FAR, rMinY = FAR, rMinZ = FAR, rMaxX = -FAR, rMaxY = -FAR, rMaxZ = -FAR;
  for (uint32_t i = 0; i < count; i++) {
    const float *b = aabbs + size_t(i) * 6;
    centers[i * 3] = float((double(b[0]) + double(b[3])) * 0.5);
    centers[i * 3 + 1] = float((double(b[1]) + double(b[4])) * 0.5);
    centers[i * 3 + 2] = float((double(b[2]) + double(b[5])) * 0.5);
    if (b[0] < rMinX) rMinX = b[0];
    if (b[1] < rMinY) rMinY = b[1];
    if (b[2] < rMinZ) rMinZ = b[2];
    if (b[3] > rMaxX) rMaxX = b[3];
    if (b[4] > rMaxY) rMaxY = b[4];
    if (b[5] > rMaxZ) rMaxZ = b[5];
    r.primIndices[i] = i;
  }
  r.bounds[0] = float(rMinX); r.bounds[1] = float(rMinY); r.bounds[2] = float(rMinZ);
  r.bounds[3] = float(rMaxX); r.bounds[4] = float(rMaxY); r.bounds[5] = float(rMaxZ);
  r.leftFirst[0] = 0;
  r.primCount[0] = count;
  const double minDim[3] = {(rMaxX - rMinX) * 1e-20, (rMaxY - rMinY) * 1e-20, (rMaxZ - rMinZ) * 1e-20};
  std::vector<double> binMin(size_t(3) * BINS * 3), binMax(size_t(3) * BINS * 3);
  std::vector<uint32_t> binCount(size_t(3) * BINS);
  std::vector<double> leftCost(BINS - 1), rightCost(BINS - 1);
  auto binOf = [&](double center, double nodeMin, double scale) {
    int32_t bin = toInt32((center - nodeMin) * scale);
    return bin < 0 ? 0 : (bin > BINS - 1 ? BINS - 1 : bin);
  };
  uint32_t newNode = 1;
  std::vector<uint32_t> tasks;
  uint32_t nodeIndex = 0;
  for (;;) {
    for (;;) {
      const size_t nb = size_t(nodeIndex) * 6;
      double nMin[3] = {r.bounds[nb], r.bounds[nb + 1], r.bounds[nb + 2]};
      double extent[3] = {double(r.bounds[nb + 3]) - nMin[0], double(r.bounds[nb + 4]) - nMin[1],
                          double(r.bounds[nb + 5]) - nMin[2]};
      double area = extent[0] * extent[1] + extent[1] * extent[2] + extent[2] * extent[0];
      if (area == 0) break;
      uint32_t first = r.leftFirst[nodeIndex];
      uint32_t nodePrims = r.primCount[nodeIndex];
      if (nodePrims == 1) break;
      double scale[3];
      for (int a = 0; a < 3; a++) scale[a] = extent[a] > minDim[a] ? double(BINS) / extent[a] : 0.0;
      std::fill(binMin.begin(), binMin.end(), FAR);
      std::fill(binMax.begin(), binMax.end(), -FAR);
      std::fill(binCount.begin(), binCount.end(), 0u);
      for (uint32_t i = first, end = first + nodePrims; i < end; i++) {
        uint32_t p = r.primIndices[i];
        const float *b = aabbs + size_t(p) * 6;
        int bx = binOf(centers[p * 3], nMin[0], scale[0]);
        int by = BINS + binOf(centers[p * 3 + 1], nMin[1], scale[1]);
        int bz = 2 * BINS + binOf(centers[p * 3 + 2], nMin[2], scale[2]);
        binCount[bx]++; binCount[by]++; binCount[bz]++;
        for (int bin : {bx, by, bz}) {
          size_t o = size_t(bin) * 3;
          binMin[o] = jsMin(binMin[o], double(b[0]));
          binMin[o + 1] = jsMin(binMin[o + 1], double(b[1]));
          binMin[o + 2] = jsMin(binMin[o + 2], double(b[2]));
          binMax[o] = jsMax(binMax[o], double(b[3]));
          binMax[o + 1] = jsMax(binMax[o + 1], double(b[4]));
          binMax[o + 2] = jsMax(binMax[o + 2], double(b[5]));
        }
      }
      double splitCost = FAR;
      int bestAxis = 0, bestPos = 0;
      for (int axis = 0; axis < 3; axis++) {
        if (!(extent[axis] > minDim[axis])) continue;
        double lMin[3] = {FAR, FAR, FAR}, lMax[3] = {-FAR, -FAR, -FAR};
        double rMin[3] = {FAR, FAR, FAR}, rMax[3] = {-FAR, -FAR, -FAR};
        uint32_t leftN = 0, rightN = 0;
        for (int i = 0; i < BINS - 1; i++) {
          size_t l = (size_t(axis) * BINS + i) * 3;
          size_t rr = (size_t(axis) * BINS + BINS - 1 - i) * 3;
          for (int k = 0; k < 3; k++) {
            lMin[k] = jsMin(lMin[k], binMin[l + k]);
            lMax[k] = jsMax(lMax[k], binMax[l + k]);
            rMin[k] = jsMin(rMin[k], binMin[rr + k]);
            rMax[k] = jsMax(rMax[k], binMax[rr + k]);
          }
          leftN += binCount[axis * BINS + i];
          rightN += binCount[axis * BINS + BINS - 1 - i];
          double lx = lMax[0] - lMin[0], ly = lMax[1] - lMin[1], lz = lMax[2] - lMin[2];
          double rx = rMax[0] - rMin[0], ry = rMax[1] - rMin[1], rz = rMax[2] - rMin[2];
          leftCost[i] = leftN == 0 ? FAR : (lx * ly + ly * lz + lz * lx) * double(leftN);
          rightCost[BINS - 2 - i] = rightN == 0 ? FAR : (rx * ry + ry * rz + rz * rx) * double(rightN);
        }
        for (int i = 0; i < BINS - 1; i++) {
          double cost = leftCost[i] + rightCost[i];
          if (cost < splitCost) { splitCost = cost; bestAxis = axis; bestPos = i; }
        }
      }
      splitCost = 1.0 + 1.0 * splitCost / area;
      if (!(splitCost < double(nodePrims) * 1.0)) break;
      double sc = scale[bestAxis], nm = nMin[bestAxis];
      uint32_t j = first + nodePrims, src = first;
      for (uint32_t i = 0; i < nodePrims; i++) {
        uint32_t p = r.primIndices[src];
        if (binOf(centers[p * 3 + bestAxis], nm, sc) <= bestPos) src++;
        else { r.primIndices[src] = r.primIndices[--j]; r.primIndices[j] = p; }
      }
      uint32_t leftPrims = src - first, rightPrims = nodePrims - leftPrims;
      if (leftPrims == 0 || rightPrims == 0) break;
      uint32_t n = newNode;
      newNode += 2;
      size_t lb = size_t(n) * 6, rb = lb + 6;
      double lbv[6] = {FAR, FAR, FAR, -FAR, -FAR, -FAR}, rbv[6] = {FAR, FAR, FAR, -FAR, -FAR, -FAR};
      for (int i = 0; i < BINS; i++) {
        size_t o = (size_t(bestAxis) * BINS + i) * 3;
        double *base = i <= bestPos ? lbv : rbv;
        for (int k = 0; k < 3; k++) {
          if (binMin[o + k] < base[k]) base[k] = binMin[o + k];
          if (binMax[o + k] > base[3 + k]) base[3 + k] = binMax[o + k];
        }
      }
      for (int k = 0; k < 6; k++) { r.bounds[lb + k] = float(lbv[k]); r.bounds[rb + k] = float(rbv[k]); }
      r.leftFirst[n] = first; r.primCount[n] = leftPrims;
      r.leftFirst[n + 1] = j; r.primCount[n + 1] = rightPrims;
      r.leftFirst[nodeIndex] = n; r.primCount[nodeIndex] = 0;
      tasks.push_back(n + 1);
      nodeIndex = n;
    }
    if (tasks.empty()) break;
    nodeIndex = tasks.back();
    tasks.pop_back();
  }
  r.nodeCount = newNode;
  return r;
}

// binnedSahBvh.ts:252-275 layoutBvh2 (depth-first: node, left, right)
Bvh2Layout layoutBvh2(const BinnedBvh &bvh) {
  Bvh2Layout L;
  L.order.assign(bvh.nodeCount, 0);
  L.offsets.assign(bvh.nodeCount, 0);
  if (!bvh.nodeCount) return L;
  std::vector<uint32_t> stack = {0, 1};
  uint32_t written = 0;
  while (!stack.empty()) {
    uint32_t depth = stack.back(); stack.pop_back();
    uint32_t node = stack.back(); stack.pop_back();
    L.order[written++] = node;
    L.offsets[node] = L.vec4Count;
    L.maxDepth = std::max(L.maxDepth, depth);
    uint32_t prims = bvh.primCount[node];
    L.vec4Count += 2 + prims;
    if (prims) L.maxLeafPrimitives = std::max(L.maxLeafPrimitives, prims);
    else {
      stack.push_back(bvh.leftFirst[node] + 1); stack.push_back(depth + 1);
      stack.push_back(bvh.leftFirst[node]); stack.push_back(depth + 1);
    }
  }
  return L;
}

// bvhAccel.ts:200-286 buildBLAS (no displacement)
Blas buildBlas(const std::vector<float> &positions, const std::vector<uint32_t> &indices, int bins) {
  Blas b;
  b.vertexCount = uint32_t(positions.size() / 3);
  uint32_t triCount = uint32_t(indices.size() / 3);
  std::vector<float> aabbs(size_t(triCount) * 6);
  std::vector<uint32_t> tris(triCount);
  uint32_t count = 0;
  for (uint32_t t = 0; t < triCount; t++) {
    // triangleBounds (bvhAccel.ts:134-175): Math.min/max over the corners; a
    // NaN coordinate, or an index past the vertex array (undefined in JS),
    // makes the box non-finite and the triangle is skipped.
    float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int c = 0; c < 3; c++) {
      uint32_t v = indices[t * 3 + c];
      for (int k = 0; k < 3; k++) {
        float x = v < b.vertexCount ? positions[size_t(v) * 3 + k] : NAN;
        mn[k] = jsMin(mn[k], x); mx[k] = jsMax(mx[k], x);
      }
    }
    bool finite = true;
    for (int k = 0; k < 3; k++) finite = finite && std::isfinite(mn[k]) && std::isfinite(mx[k]);
    if (!finite) continue;
    float *o = &aabbs[size_t(count) * 6];
    for (int k = 0; k < 3; k++) { o[k] = mn[k]; o[3 + k] = mx[k]; }
    tris[count++] = t;
  }
  const float noBounds[6] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY};
  std::memcpy(b.localBounds, noBounds, sizeof(noBounds));
  if (!count) return b;
  BinnedBvh bvh = buildBinnedSahBvh(aabbs.data(), count, bins);
  Bvh2Layout L = layoutBvh2(bvh);
  b.buffer.assign(size_t(L.vec4Count) * 4, 0.0f);
  float *f = b.buffer.data();
  for (uint32_t k = 0; k < L.order.size(); k++) {
    uint32_t node = L.order[k];
    size_t o = size_t(L.offsets[node]) * 4, bb = size_t(node) * 6;
    f[o] = bvh.bounds[bb]; f[o + 1] = bvh.bounds[bb + 1]; f[o + 2] = bvh.bounds[bb + 2];
    f[o + 4] = bvh.bounds[bb + 3]; f[o + 5] = bvh.bounds[bb + 4]; f[o + 6] = bvh.bounds[bb + 5];
    uint32_t prims = bvh.primCount[node];
    if (!prims) { f[o + 3] = asFloat(int32_t(L.offsets[bvh.leftFirst[node] + 1])); continue; }
    f[o + 3] = asFloat(-int32_t(prims));
    for (uint32_t i = 0; i < prims; i++) {
      uint32_t t = tris[bvh.primIndices[bvh.leftFirst[node] + i]];
      size_t e = o + 8 + size_t(i) * 4;
      f[e] = asFloat(int32_t(indices[t * 3]));
      f[e + 1] = asFloat(int32_t(indices[t * 3 + 1]));
      f[e + 2] = asFloat(int32_t(indices[t * 3 + 2]));
      f[e + 3] = asFloat(0);
    }
  }
  b.maxDepth = L.maxDepth;
  // getBvhBounds (geometryBvhBounds.ts:74-77): a bvh2 BLAS is bounded by its
  // root node's box.
  for (int k = 0; k < 3; k++) { b.localBounds[k] = f[k]; b.localBounds[3 + k] = f[4 + k]; }
  return b;
}

// bvhAccel.ts:800-870 refitBLAS (BVH2, no displacement): node boxes rewritten
// in post order (descendants first; in the depth-first layout that is
// descending offset order), leaves from their vertices with three finite
// coordinates (an index past the position array is skipped), interior nodes
// from their children, all with Math.min/max.  Returns the summed surface
// area 2(xz + xy + zy) in that order (the rebuild hint's numerator).
double refitBlasHost(float *f, size_t vec4, const float *positions, uint32_t vertexCount) {
  std::vector<uint32_t> preorder;
  std::vector<uint32_t> stack = {0};
  while (!stack.empty()) {
    uint32_t o = stack.back();
    stack.pop_back();
    if (size_t(o) + 2 > vec4) throw std::runtime_error("BLAS node offset outside the buffer");
    preorder.push_back(o);
    int32_t w = asInt(f[size_t(o) * 4 + 3]);
    if (w >= 0) {
      if (size_t(w) + 2 > vec4 || uint32_t(w) <= o + 2) throw std::runtime_error("BLAS child offset out of order");
      stack.push_back(uint32_t(w));
      stack.push_back(o + 2);
    } else if (size_t(o) + 2 + size_t(-int64_t(w)) > vec4) {
      throw std::runtime_error("BLAS leaf outside the buffer");
    }
  }
  double area = 0.0;
  for (size_t k = preorder.size(); k-- > 0;) {
    float *n = f + size_t(preorder[k]) * 4;
    int32_t w = asInt(n[3]);
    float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    if (w >= 0) {
      const float *l = n + 8, *r = f + size_t(w) * 4;
      for (int c = 0; c < 3; c++) { mn[c] = jsMin(l[c], r[c]); mx[c] = jsMax(l[4 + c], r[4 + c]); }
    } else {
      for (int32_t t = 0; t < -w; t++) {
        const float *rec = n + 8 + size_t(t) * 4;
        for (int c = 0; c < 3; c++) {
          uint32_t v = uint32_t(asInt(rec[c]));
          if (v >= vertexCount) continue;
          const float *p = positions + size_t(v) * 3;
          if (!std::isfinite(p[0]) || !std::isfinite(p[1]) || !std::isfinite(p[2])) continue;
          for (int k2 = 0; k2 < 3; k2++) { mn[k2] = jsMin(mn[k2], p[k2]); mx[k2] = jsMax(mx[k2], p[k2]); }
        }
      }
    }
    double x = double(mx[0]) - double(mn[0]), y = double(mx[1]) - double(mn[1]), z = double(mx[2]) - double(mn[2]);
    area += 2 * (x * z + x * y + z * y);
    for (int c = 0; c < 3; c++) { n[c] = mn[c]; n[4 + c] = mx[c]; }
  }
  return area;
}

std::vector<float> blasToGpuLayout(const std::vector<float> &f) {
  if (f.empty()) return {};
  auto ptr = [&](uint32_t off) { return asInt(f[size_t(off) * 4 + 3]); };
  // Depth-first preorder numbering of the BVH2 nodes (left before right).
  std::vector<uint32_t> order;
  std::vector<uint32_t> stack = {0};
  while (!stack.empty()) {
    uint32_t off = stack.back();
    stack.pop_back();
    order.push_back(off);
    int32_t p = ptr(off);
    if (p >= 0) {
      stack.push_back(uint32_t(p));
      stack.push_back(off + 2);
    }
  }
  std::vector<int64_t> index(f.size() / 4, -1);
  for (size_t k = 0; k < order.size(); k++) index[order[k]] = int64_t(k);
  size_t nodeVec4 = order.size() * 4, records = 0;
  for (uint32_t off : order)
    if (ptr(off) < 0) records += size_t(-ptr(off));
  std::vector<float> g((nodeVec4 + records) * 4, 0.0f);
  size_t next = nodeVec4;  // next primitive record, vec4 units
  for (size_t k = 0; k < order.size(); k++) {
    uint32_t off = order[k];
    float *n = &g[k * 16];
    int32_t p = ptr(off);
    if (p >= 0) {
      uint32_t left = off + 2, right = uint32_t(p);
      for (int c = 0; c < 3; c++) {
        n[c] = f[size_t(left) * 4 + c];           // left min
        n[4 + c] = f[size_t(left) * 4 + 4 + c];   // left max
        n[8 + c] = f[size_t(right) * 4 + c];      // right min
        n[12 + c] = f[size_t(right) * 4 + 4 + c]; // right max
      }
      n[3] = asFloat(int32_t(index[left]));
      n[7] = asFloat(int32_t(index[right]));
      n[11] = asFloat(int32_t(0));
      n[15] = asFloat(int32_t(0));
      continue;
    }
    uint32_t count = uint32_t(-p);
    n[11] = asFloat(int32_t(count));
    n[15] = asFloat(int32_t(next));
    std::memcpy(&g[next * 4], &f[(size_t(off) + 2) * 4], size_t(count) * 16);
    next += count;
  }
  return g;
}

void setBlasLayout(SceneHost &s, uint32_t layout) {
  if (layout != 0 && layout != 2) throw std::runtime_error("BLAS layout must be 0 or 2");
  std::vector<std::vector<float>> buffers(s.blases.size());
  for (size_t m = 0; m < s.blases.size(); m++)
    buffers[m] = layout == 2 ? blasToGpuLayout(s.blases[m].buffer) : s.blases[m].buffer;
  std::vector<uint32_t> offsets;
  uint32_t off = 0;
  for (auto &b : buffers) {
    offsets.push_back(off);
    off += uint32_t(b.size() / 4);
  }
  std::vector<float> bvh(s.bvh.begin(), s.bvh.begin() + size_t(s.tlasVec4) * 4);
  for (auto &b : buffers) bvh.insert(bvh.end(), b.begin(), b.end());
  // TLAS leaf records (instanceSlot, blasRoot, sourceIndex, box): walk the
  // TLAS and move each blasRoot to its BLAS's new start.
  std::vector<uint32_t> stack;
  if (s.tlasVec4) stack.push_back(0);
  while (!stack.empty()) {
    uint32_t node = stack.back();
    stack.pop_back();
    int32_t p = asInt(bvh[size_t(node) * 4 + 3]);
    if (p >= 0) {
      stack.push_back(node + 2);
      stack.push_back(uint32_t(p));
      continue;
    }
    for (int32_t i = 0; i < -p; i++) {
      float *rec = &bvh[(size_t(node) + 2 + i) * 4];
      int32_t source = asInt(rec[2]);
      uint32_t m = s.sourceInstances[size_t(source)].blasIndex;
      rec[1] = asFloat(int32_t(offsets[m]));
      float *ins = &s.instances[size_t(asInt(rec[0])) * 40];
      ins[0] = asFloat(int32_t(offsets[m] | (layout << 30)));  // as writeInstanceRecord
    }
  }
  s.bvh.swap(bvh);
  s.blasOffsets = offsets;
  s.blasLayout = layout;
  buildTrianglePlane(s);  // records moved
  if (layout == 2) s.flags |= MTC_SCENE_BLAS_GPU_LAYOUT;
  else s.flags &= ~uint32_t(MTC_SCENE_BLAS_GPU_LAYOUT);
}

void buildTrianglePlane(SceneHost &s) {
  s.triangleMaterials.clear();
  bool any = false;
  for (const auto &vm : s.sourceVertexMaterials) any |= !vm.empty();
  if (!any) return;
  s.triangleMaterials.assign(s.bvh.size() / 4, 0u);
  for (size_t m = 0; m < s.blasOffsets.size() && m < s.sourceVertexMaterials.size(); m++) {
    const std::vector<int32_t> &vm = s.sourceVertexMaterials[m];
    if (vm.empty()) continue;
    const size_t begin = size_t(s.tlasVec4) + s.blasOffsets[m];
    const size_t end = m + 1 < s.blasOffsets.size() ? size_t(s.tlasVec4) + s.blasOffsets[m + 1] : s.bvh.size() / 4;
    for (size_t r = begin; r < end; r++) {
      uint32_t vertex;
      std::memcpy(&vertex, &s.bvh[r * 4], 4);
      if (vertex < vm.size()) s.triangleMaterials[r] = uint32_t(vm[vertex]) + 1u;
    }
  }
}

// gl-matrix mat4 invert (cofactor expansion), float64, as called by
// writeInstanceRecord (bvhAccel.ts:330-353).
bool invert4(const double *a, double *out) {
  double a00 = a[0], a01 = a[1], a02 = a[2], a03 = a[3];
  double a10 = a[4], a11 = a[5], a12 = a[6], a13 = a[7];
  double a20 = a[8], a21 = a[9], a22 = a[10], a23 = a[11];
  double a30 = a[12], a31 = a[13], a32 = a[14], a33 = a[15];
  double b00 = a00 * a11 - a01 * a10, b01 = a00 * a12 - a02 * a10, b02 = a00 * a13 - a03 * a10;
  double b03 = a01 * a12 - a02 * a11, b04 = a01 * a13 - a03 * a11, b05 = a02 * a13 - a03 * a12;
  double b06 = a20 * a31 - a21 * a30, b07 = a20 * a32 - a22 * a30, b08 = a20 * a33 - a23 * a30;
  double b09 = a21 * a32 - a22 * a31, b10 = a21 * a33 - a23 * a31, b11 = a22 * a33 - a23 * a32;
  double det = b00 * b11 - b01 * b10 + b02 * b09 + b03 * b08 - b04 * b07 + b05 * b06;
  if (det == 0.0) return false;
  det = 1.0 / det;
  out[0] = (a11 * b11 - a12 * b10 + a13 * b09) * det;
  out[1] = (a02 * b10 - a01 * b11 - a03 * b09) * det;
  out[2] = (a31 * b05 - a32 * b04 + a33 * b03) * det;
  out[3] = (a22 * b04 - a21 * b05 - a23 * b03) * det;
  out[4] = (a12 * b08 - a10 * b11 - a13 * b07) * det;
  out[5] = (a00 * b11 - a02 * b08 + a03 * b07) * det;
  out[6] = (a32 * b02 - a30 * b05 - a33 * b01) * det;
  out[7] = (a20 * b05 - a22 * b02 + a23 * b01) * det;
  out[8] = (a10 * b10 - a11 * b08 + a13 * b06) * det;
  out[9] = (a01 * b08 - a00 * b10 - a03 * b06) * det;
  out[10] = (a30 * b04 - a31 * b02 + a33 * b00) * det;
  out[11] = (a21 * b02 - a20 * b04 - a23 * b00) * det;
  out[12] = (a11 * b07 - a10 * b09 - a12 * b06) * det;
  out[13] = (a00 * b09 - a01 * b07 + a02 * b06) * det;
  out[14] = (a31 * b01 - a30 * b03 - a32 * b00) * det;
  out[15] = (a20 * b03 - a21 * b01 + a22 * b00) * det;
  return true;
}

// scenePreparation.ts:19-47 computeBounds: eight BLAS corners through the
// float64 transform (vec3.transformMat4), each stored as f32.
void computeInstanceBounds(const Instance &ins, const float local[6], float out[6]) {
  float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
  const double *m = ins.transform;
  for (int corner = 0; corner < 8; corner++) {
    double x = (corner & 1) ? local[3] : local[0];
    double y = (corner & 2) ? local[4] : local[1];
    double z = (corner & 4) ? local[5] : local[2];
    double w = m[3] * x + m[7] * y + m[11] * z + m[15];
    if (w == 0.0 || w != w) w = 1.0;
    float p[3] = {float((m[0] * x + m[4] * y + m[8] * z + m[12]) / w),
                  float((m[1] * x + m[5] * y + m[9] * z + m[13]) / w),
                  float((m[2] * x + m[6] * y + m[10] * z + m[14]) / w)};
    if (!std::isfinite(p[0]) || !std::isfinite(p[1]) || !std::isfinite(p[2])) continue;
    for (int k = 0; k < 3; k++) { mn[k] = jsMin(mn[k], p[k]); mx[k] = jsMax(mx[k], p[k]); }
  }
  for (int k = 0; k < 3; k++) { out[k] = mn[k]; out[3 + k] = mx[k]; }
}

// bvhAccel.ts:330-353 writeInstanceRecord: blasOffset | layout << 30
void writeInstanceRecord(float *rec, const Instance &ins, uint32_t blasOffset, uint32_t vertexOffset,
                         uint32_t blasLayout) {
  if (blasOffset > 0x3fffffffu) throw std::runtime_error("BLAS offset exceeds the packed 30-bit range");
  rec[0] = asFloat(int32_t(blasOffset | (blasLayout << 30)));
  rec[1] = asFloat(int32_t(vertexOffset));
  rec[2] = asFloat(ins.material);
  rec[3] = 0.0f;
  rec[36] = ins.color[0]; rec[37] = ins.color[1]; rec[38] = ins.color[2]; rec[39] = 0.0f;
  double inv[16];
  if (!invert4(ins.transform, inv)) std::fill(inv, inv + 16, 0.0);
  for (int i = 0; i < 16; i++) {
    rec[4 + i] = float(inv[i]);
    rec[20 + i] = float(ins.transform[i]);
  }
}

// bvhAccel.ts:385-449 buildTLAS (native layout: perInstanceBounds = false)
Tlas buildTlas(const std::vector<Instance> &instances, const std::vector<Blas> &blases,
               const std::vector<uint32_t> &blasOffsets, const std::vector<uint32_t> &vertexOffsets, int bins) {
  Tlas t;
  uint32_t n = uint32_t(instances.size());
  if (!n) return t;
  std::vector<float> aabbs(size_t(n) * 6);
  for (uint32_t i = 0; i < n; i++) computeInstanceBounds(instances[i], blases[instances[i].blasIndex].localBounds, &aabbs[size_t(i) * 6]);
  BinnedBvh bvh = buildBinnedSahBvh(aabbs.data(), n, bins);
  Bvh2Layout L = layoutBvh2(bvh);
  t.buffer.assign(size_t(L.vec4Count) * 4, 0.0f);
  t.instances.assign(size_t(n) * 40, 0.0f);
  float *f = t.buffer.data();
  uint32_t target = 0;
  for (uint32_t k = 0; k < L.order.size(); k++) {
    uint32_t node = L.order[k];
    size_t o = size_t(L.offsets[node]) * 4, bb = size_t(node) * 6;
    f[o] = bvh.bounds[bb]; f[o + 1] = bvh.bounds[bb + 1]; f[o + 2] = bvh.bounds[bb + 2];
    f[o + 4] = bvh.bounds[bb + 3]; f[o + 5] = bvh.bounds[bb + 4]; f[o + 6] = bvh.bounds[bb + 5];
    uint32_t prims = bvh.primCount[node];
    if (!prims) { f[o + 3] = asFloat(int32_t(L.offsets[bvh.leftFirst[node] + 1])); continue; }
    f[o + 3] = asFloat(-int32_t(prims));
    for (uint32_t i = 0; i < prims; i++) {
      uint32_t source = bvh.primIndices[bvh.leftFirst[node] + i];
      const Instance &ins = instances[source];
      size_t e = o + 8 + size_t(i) * 4;
      f[e] = asFloat(int32_t(target));
      f[e + 1] = asFloat(int32_t(blasOffsets[ins.blasIndex]));
      f[e + 2] = asFloat(int32_t(source));
      f[e + 3] = asFloat(0);
      writeInstanceRecord(&t.instances[size_t(target) * 40], ins, blasOffsets[ins.blasIndex], vertexOffsets[ins.blasIndex]);
      target++;
    }
  }
  t.maxDepth = L.maxDepth;
  return t;
}

// bvhAccel.ts:579-740 refitTLAS with no dirty set (full refit, refitNode).
void refitTlasHost(float *tlas, float *records, const std::vector<Instance> &instances,
                   const std::vector<Blas> &blases, const std::vector<uint32_t> &blasOffsets,
                   const std::vector<uint32_t> &vertexOffsets, uint32_t blasLayout) {
  std::function<void(int32_t)> refitNode = [&](int32_t index) {
    size_t base = size_t(index) * 4;
    int32_t child = asInt(tlas[base + 3]);
    if (child >= 0) {
      refitNode(index + 2);
      refitNode(child);
      size_t left = base + 8, right = size_t(child) * 4;
      for (int k = 0; k < 3; k++) {
        tlas[base + k] = jsMin(tlas[left + k], tlas[right + k]);
        tlas[base + 4 + k] = jsMax(tlas[left + 4 + k], tlas[right + 4 + k]);
      }
      return;
    }
    float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int32_t i = 0; i < -child; i++) {
      size_t record = base + 8 + size_t(i) * 4;
      int32_t source = asInt(tlas[record + 2]);
      const Instance &ins = instances[source];
      float b[6];
      computeInstanceBounds(ins, blases[ins.blasIndex].localBounds, b);
      for (int k = 0; k < 3; k++) { mn[k] = jsMin(mn[k], b[k]); mx[k] = jsMax(mx[k], b[3 + k]); }
      int32_t target = asInt(tlas[record]);
      writeInstanceRecord(records + size_t(target) * 40, ins, blasOffsets[ins.blasIndex], vertexOffsets[ins.blasIndex],
                          blasLayout);
    }
    for (int k = 0; k < 3; k++) { tlas[base + k] = mn[k]; tlas[base + 4 + k] = mx[k]; }
  };
  refitNode(0);
}

// ------------------------------------------------------------- materials
// materialLayoutSchema.ts:23-150 row layout (26 rows x vec4).
void packMaterial(const MaterialDesc &m, float *r) {
  std::fill(r, r + MTC_MATERIAL_VEC4_ROWS * 4, 0.0f);
  auto row = [&](int i) { return r + i * 4; };
  auto set3 = [](float *d, const float *s) { d[0] = s[0]; d[1] = s[1]; d[2] = s[2]; };
  set3(row(0), m.baseColor); row(0)[3] = float(m.type);
  row(1)[0] = m.specularRoughness; row(1)[1] = float(m.maps[kMapNormal]);
  row(1)[2] = m.normalScale[0]; row(1)[3] = m.normalScale[1];
  row(2)[0] = m.baseMetalness; row(2)[1] = m.specularAnisotropy;
  row(2)[2] = float(m.maps[kMapBase]); row(2)[3] = float(m.maps[kMapMetallicRoughness]);
  set3(row(3), m.emission); row(3)[3] = float(m.maps[kMapEmissive]);
  row(4)[0] = m.specularIor; row(4)[1] = m.transmissionWeight; row(4)[2] = 0.0f; row(4)[3] = m.thin ? 1.0f : 0.0f;
  // finiteFilmThickness (thinFilmParameters.ts:9-11): negative thickness packs as 0
  row(5)[0] = 0.0f; row(5)[1] = m.dispersionScale; row(5)[2] = std::max(0.0f, m.thinFilmThickness);
  row(5)[3] = float(m.mapAlphaUsage);
  row(6)[0] = float(m.maps[kMapCoatWeight]); row(6)[1] = float(m.maps[kMapCoatRoughness]);
  row(6)[2] = float(m.maps[kMapCoatNormal]); row(6)[3] = float(m.maps[kMapFuzzColor]);
  row(7)[0] = float(m.uvProjection); row(7)[1] = float(m.maps[kMapDisplacement]); row(7)[2] = m.uvScale[0]; row(7)[3] = m.uvScale[1];
  row(9)[0] = m.opacity; row(9)[1] = float(m.maps[kMapThinFilm]); row(9)[2] = m.thinFilmIor;
  row(9)[3] = float(m.maps[kMapTransmission]);
  row(10)[0] = m.baseWeight; row(10)[1] = m.diffuseRoughness; row(10)[2] = m.specularWeight; row(10)[3] = m.subsurfaceWeight;
  set3(row(11), m.specularColor); row(11)[3] = m.fuzzWeight;
  set3(row(12), m.transmissionColor); row(12)[3] = 0.0f;
  set3(row(14), m.subsurfaceColor);
  set3(row(15), m.fuzzColor); row(15)[3] = m.fuzzRoughness;
  set3(row(16), m.coatColor); row(16)[3] = m.coatWeight;
  row(17)[0] = m.coatRoughness; row(17)[1] = 0.0f; row(17)[2] = m.coatIor; row(17)[3] = m.coatDarkening;
  row(18)[0] = m.thinFilmWeight; row(18)[1] = m.abbe; row(18)[2] = 0.0f; row(18)[3] = float(m.maps[kMapFuzzRoughness]);
  row(19)[3] = float(m.maps[kMapSpecularWeight]);
  set3(row(20), m.mediumExtinction); row(20)[3] = m.mediumAnisotropy;
  set3(row(21), m.mediumScattering); row(21)[3] = float(m.maps[kMapSpecularColor]);
  row(22)[0] = float(m.maps[kMapRoughness]); row(22)[1] = float(m.maps[kMapMetalness]);
  row(22)[2] = float(m.maps[kMapAlpha]); row(22)[3] = std::max(0.0f, m.alphaCutoff);
  row(23)[2] = m.doubleSided ? 1.0f : 0.0f; row(23)[3] = float(m.alphaMode);
  row(24)[0] = float(m.maps[kMapAnisotropy]); row(24)[1] = 0.0f; row(24)[2] = 1.0f; row(24)[3] = 1.0f;
  row(25)[2] = std::max(0.0f, m.thinFilmThicknessMinimum); row(25)[3] = float(m.thinFilmMapChannel);
}

// ---------------------------------------------------------- environment
static double luminanceD(double r, double g, double b) { return std::max(r * 0.2126 + g * 0.7152 + b * 0.0722, 0.0); }

// envMapDistribution.ts:57-134
void buildEnvDistribution(Environment &env) {
  const uint32_t W = env.width, H = env.height;
  const uint32_t dw = W + 2, dh = H + 1;
  env.distribution.assign(size_t(dw) * dh * 2, 0.0f);
  auto set = [&](uint32_t x, uint32_t y, int c, double v) { env.distribution[(size_t(y) * dw + x) * 2 + c] = float(v); };
  auto get = [&](uint32_t x, uint32_t y, int c) { return double(env.distribution[(size_t(y) * dw + x) * 2 + c]); };
  std::vector<float> lum(size_t(W) * H), horiz(size_t(W) * H);
  for (uint32_t i = 0; i < W * H; i++) {
    const float *p = &env.image[size_t(i) * 4];
    lum[i] = float(1.0 * (0.2126 * double(p[0]) + 0.7152 * double(p[1]) + 0.0722 * double(p[2])));
  }
  for (uint32_t y = 0; y < H; y++) {
    size_t row = size_t(y) * W;
    for (uint32_t x = 0; x < W; x++) {
      double v = std::max({0.0, double(lum[row + (x ? x - 1 : 0)]), double(lum[row + x]),
                           double(lum[row + std::min(W - 1, x + 1)])});
      horiz[row + x] = float(v);
    }
  }
  for (uint32_t y = 0; y < H; y++) {
    double sinTheta = std::sin(M_PI * (y + 0.5) / H);
    size_t above = size_t(y ? y - 1 : 0) * W, row = size_t(y) * W, below = size_t(std::min(H - 1, y + 1)) * W;
    for (uint32_t x = 0; x < W; x++) {
      double weight = std::max({double(horiz[above + x]), double(horiz[row + x]), double(horiz[below + x]), 1e-12}) * sinTheta;
      set(x + 2, y, 0, get(x + 1, y, 0) + weight / W);
      set(x + 1, y, 1, weight);
    }
    double rowIntegral = get(dw - 1, y, 0);
    for (uint32_t x = 1; x < dw; x++) {
      set(x, y, 0, get(x, y, 0) / rowIntegral);
      set(x, y, 1, get(x, y, 1) / rowIntegral);
    }
    set(0, y + 1, 0, get(0, y, 0) + rowIntegral / H);
    set(0, y, 1, rowIntegral);
  }
  double integral = get(0, dh - 1, 0);
  for (uint32_t y = 0; y < dh; y++) {
    set(0, y, 0, get(0, y, 0) / integral);
    set(0, y, 1, get(0, y, 1) / integral);
  }
  // lightSampling.ts:415-431 environmentPower
  double wl = 0.0;
  for (uint32_t y = 0; y < H; y++) {
    double s = std::sin(M_PI * (y + 0.5) / H);
    for (uint32_t x = 0; x < W; x++) {
      const float *p = &env.image[(size_t(y) * W + x) * 4];
      wl += luminanceD(p[0], p[1], p[2]) * s;
    }
  }
  env.power = wl * (2.0 * M_PI * M_PI) / (double(W) * H);
}

// PCG32 (O'Neill) for the seeded generators.
struct Pcg32 {
  uint64_t state, inc;
  explicit Pcg32(uint64_t seed, uint64_t stream = 54u) : state(0), inc((stream << 1u) | 1u) {
    next(); state += seed; next();
  }
  uint32_t next() {
    uint64_t old = state;
    state = old * 6364136223846793005ULL + inc;
    uint32_t xs = uint32_t(((old >> 18u) ^ old) >> 27u);
    uint32_t rot = uint32_t(old >> 59u);
    return (xs >> rot) | (xs << ((-rot) & 31));
  }
  double uniform() { return next() * (1.0 / 4294967296.0); }
  double range(double a, double b) { return a + (b - a) * uniform(); }
};

// Analytic sky of this build: zenith/horizon gradient, darker ground and a
// bright sun disk, stored as an equirect RGBA32F image in the layout
// sampleEnvmap expects (u: phi, v: theta from +y).
void makeAnalyticSky(Environment &env, uint32_t W, uint32_t H, uint64_t seed) {
  Pcg32 rng(seed, 7);
  env.width = W; env.height = H;
  env.image.assign(size_t(W) * H * 4, 0.0f);
  double sunPhi = rng.range(0.0, 2.0 * M_PI), sunElev = rng.range(0.35, 0.9);
  double sun[3] = {-std::cos(sunElev) * std::cos(sunPhi), std::sin(sunElev), -std::cos(sunElev) * std::sin(sunPhi)};
  const double sunCos = std::cos(1.5 * M_PI / 180.0);
  for (uint32_t y = 0; y < H; y++) {
    double theta = M_PI * (y + 0.5) / H;
    for (uint32_t x = 0; x < W; x++) {
      double phi = 2.0 * M_PI * (x + 0.5) / W;
      double d[3] = {-std::sin(theta) * std::cos(phi), std::cos(theta), -std::sin(theta) * std::sin(phi)};
      double c[3];
      if (d[1] >= 0.0) {
        double t = std::pow(d[1], 0.45);
        c[0] = 0.85 * (1 - t) + 0.18 * t;
        c[1] = 0.88 * (1 - t) + 0.32 * t;
        c[2] = 0.95 * (1 - t) + 0.78 * t;
      } else {
        double t = std::min(1.0, -d[1] * 4.0);
        c[0] = 0.85 * (1 - t) + 0.22 * t;
        c[1] = 0.88 * (1 - t) + 0.20 * t;
        c[2] = 0.95 * (1 - t) + 0.18 * t;
      }
      double cosSun = d[0] * sun[0] + d[1] * sun[1] + d[2] * sun[2];
      double glow = std::pow(std::max(0.0, cosSun), 64.0) * 2.0;
      for (int k = 0; k < 3; k++) c[k] += glow * (k == 2 ? 0.7 : 1.0);
      if (cosSun >= sunCos) { c[0] += 400.0; c[1] += 380.0; c[2] += 340.0; }
      float *p = &env.image[(size_t(y) * W + x) * 4];
      p[0] = float(c[0]); p[1] = float(c[1]); p[2] = float(c[2]); p[3] = 1.0f;
    }
  }
  buildEnvDistribution(env);
}

// ------------------------------------------------------------ energy LUT
// Adobe's OpenPBR energy-compensation tables (Apache License 2.0, Copyright
// 2026 Adobe; adobe/openpbr-bsdf), decoded from the reference's
// openPbrEnergyLut.ts by decodeOpenPbrEnergyLut.ts:35-83 into the 32 x 2177
// float32 rows the BSDF samples.  The build embeds the decoded table
// (csrc/openpbr_energy_lut.f32, written by csrc/gen_energy_lut.py) as
// little-endian float32 bit patterns.
extern "C" const uint32_t mtp_openpbr_energy_lut_bits[];
extern "C" const uint64_t mtp_openpbr_energy_lut_count;

void buildEnergyLut(std::vector<float> &lut) {
  const size_t n = size_t(MTC_ENERGY_LUT_WIDTH) * MTC_ENERGY_LUT_HEIGHT;
  if (mtp_openpbr_energy_lut_count != n) throw std::runtime_error("embedded energy LUT has the wrong size");
  lut.resize(n);
  std::memcpy(lut.data(), mtp_openpbr_energy_lut_bits, n * sizeof(float));
}

// ---------------------------------------------------------------- lights
double lightPower(const LightDesc &L) {
  double lum = luminanceD(L.color[0], L.color[1], L.color[2]) * L.intensity;
  if (!(lum > 0)) return 0.0;
  switch (L.type) {
    case MTC_LIGHT_RECT: return lum * M_PI * std::max(double(L.area), 0.0);
    case MTC_LIGHT_DISK: return lum * M_PI * double(L.area);
    case MTC_LIGHT_SPHERE:
      if (L.radius == 0.0f) return lum * 4.0 * M_PI;
      return lum * M_PI * std::max(4.0 * M_PI * double(L.radius) * L.radius, 0.0);
    default: return lum * 4.0 * M_PI;
  }
}


// lightSampling.ts:172-212 buildLightAliasTable
AliasTable buildAlias(const std::vector<int> &types, const std::vector<int> &indices, const std::vector<double> &weights) {
  AliasTable t;
  size_t count = weights.size();
  for (double w : weights) t.total += w;
  if (!count || !(t.total > 0)) { t.words.assign(4, 0); return t; }
  t.pmfs.resize(count);
  std::vector<double> scaled(count);
  std::vector<uint32_t> small(count), large(count);
  size_t sc = 0, lc = 0;
  for (size_t i = 0; i < count; i++) {
    t.pmfs[i] = float(weights[i] / t.total);
    scaled[i] = double(t.pmfs[i]) * double(count);
    if (scaled[i] < 1) small[sc++] = uint32_t(i); else large[lc++] = uint32_t(i);
  }
  std::vector<float> f(count * 4, 0.0f);
  std::vector<int32_t> &ii = *reinterpret_cast<std::vector<int32_t> *>(&f);
  (void)ii;
  auto seti = [&](size_t k, int32_t v) { f[k] = asFloat(v); };
  while (sc && lc) {
    uint32_t low = small[--sc], high = large[--lc];
    f[size_t(low) * 4] = float(scaled[low]);
    seti(size_t(low) * 4 + 1, int32_t(high));
    scaled[high] = scaled[high] + scaled[low] - 1;
    if (scaled[high] < 1) small[sc++] = high; else large[lc++] = high;
  }
  for (size_t i = 0; i < sc; i++) { f[size_t(small[i]) * 4] = 1.0f; seti(size_t(small[i]) * 4 + 1, int32_t(small[i])); }
  for (size_t i = 0; i < lc; i++) { f[size_t(large[i]) * 4] = 1.0f; seti(size_t(large[i]) * 4 + 1, int32_t(large[i])); }
  for (size_t i = 0; i < count; i++) { seti(i * 4 + 2, types[i]); seti(i * 4 + 3, indices[i]); }
  t.words.resize(count * 4);
  std::memcpy(t.words.data(), f.data(), count * 16);
  return t;
}

// -------------------------------------------------------------- assembly
static uint32_t octEncode(double x, double y, double z) {
  double len = std::fabs(x) + std::fabs(y) + std::fabs(z);
  if (!(len > 0)) return (1u << 15) | (1u << 31);
  x /= len; y /= len;
  if (z < 0) {
    double ox = x;
    x = (1 - std::fabs(y)) * (ox < 0 ? -1 : 1);
    y = (1 - std::fabs(ox)) * (y < 0 ? -1 : 1);
  }
  auto jsRound = [](double v) { return int32_t(std::floor(v + 0.5)); };
  uint32_t mask = 0xffffu;
  return (uint32_t(jsRound(x * 32767.0)) & mask) | ((uint32_t(jsRound(y * 32767.0)) & mask) << 16);
}

void setCamera(SceneHost &s, const CameraDesc &c) {
  // lookAt (view) and perspective projection, column-major, float64.
  double f[3] = {c.target[0] - c.eye[0], c.target[1] - c.eye[1], c.target[2] - c.eye[2]};
  double fl = std::sqrt(f[0] * f[0] + f[1] * f[1] + f[2] * f[2]);
  for (double &v : f) v /= fl;
  double sv[3] = {f[1] * c.up[2] - f[2] * c.up[1], f[2] * c.up[0] - f[0] * c.up[2], f[0] * c.up[1] - f[1] * c.up[0]};
  double sl = std::sqrt(sv[0] * sv[0] + sv[1] * sv[1] + sv[2] * sv[2]);
  for (double &v : sv) v /= sl;
  double u[3] = {sv[1] * f[2] - sv[2] * f[1], sv[2] * f[0] - sv[0] * f[2], sv[0] * f[1] - sv[1] * f[0]};
  double viewInv[16] = {sv[0], sv[1], sv[2], 0, u[0], u[1], u[2], 0, -f[0], -f[1], -f[2], 0,
                        c.eye[0], c.eye[1], c.eye[2], 1};
  double view[16];
  invert4(viewInv, view);
  double aspect = double(s.width) / double(s.height);
  double nearZ = 0.05, farZ = 1000.0;
  double t = 1.0 / std::tan(c.fovYDeg * M_PI / 360.0);
  double proj[16] = {t / aspect, 0, 0, 0, 0, t, 0, 0, 0, 0, (farZ + nearZ) / (nearZ - farZ), -1,
                     0, 0, 2 * farZ * nearZ / (nearZ - farZ), 0};
  double vp[16];
  for (int col = 0; col < 4; col++)
    for (int row = 0; row < 4; row++) {
      double acc = 0;
      for (int k = 0; k < 4; k++) acc += proj[k * 4 + row] * view[col * 4 + k];
      vp[col * 4 + row] = acc;
    }
  double vpInv[16];
  invert4(vp, vpInv);
  for (int i = 0; i < 16; i++) {
    s.camera.view_projection_inv[i] = float(vpInv[i]);
    s.camera.view_inv[i] = float(viewInv[i]);
  }
  s.camera.aperture_radius = float(c.aperture);
  s.camera.focus_distance = float(c.focus);
}

void defaultUniform(SceneHost &s, uint32_t bounces, uint32_t candidates, uint32_t seed, int pattern) {
  mtc_trace_uniform &u = s.uniform;
  u.output_size[0] = float(s.width);
  u.output_size[1] = float(s.height);
  u.scale_offset[0] = 1; u.scale_offset[1] = 1;
  u.transmissive_output_alpha_min = 1.0f;
  u.bevel = 1;
  u.dispersion_wavelengths = 3;
  u.bounces = int32_t(bounces);
  u.direct_light_candidates = int32_t(candidates);
  u.loop_unroll_guard = 4;
  u.sequence_seed = seed;
  u.zsobol_log_spp = 6;
  for (int i = 0; i < 4; i++) { u.environment_rotation[i * 5] = 1; u.background_map_rotation[i * 5] = 1; }
  u.background_map_transform[0] = 1; u.background_map_transform[2] = 1;
  s.flags = (s.flags & ~uint32_t(MTC_SCENE_PATTERN_MASK)) | (uint32_t(pattern) << MTC_SCENE_PATTERN_SHIFT);
}

void assembleScene(SceneHost &s, const std::vector<MeshData> &meshes, const std::vector<Instance> &instances,
                   const std::vector<MaterialDesc> &materials, const std::vector<LightDesc> &lights, int blasBins,
                   int tlasBins, bool normalFloat) {
  // BLASes in parallel.
  s.blases.assign(meshes.size(), Blas());
  {
    std::vector<std::thread> pool;
    unsigned nt = std::max(1u, std::min(8u, std::thread::hardware_concurrency()));
    for (unsigned t = 0; t < nt; t++)
      pool.emplace_back([&, t] {
        for (size_t m = t; m < meshes.size(); m += nt) s.blases[m] = buildBlas(meshes[m].positions, meshes[m].indices, blasBins);
      });
    for (auto &th : pool) th.join();
  }
  s.blasOffsets.clear(); s.vertexOffsets.clear();
  uint32_t blasOffset = 0, vertexOffset = 0;
  uint32_t blasDepth = 1;
  s.uniqueTriangleCount = 0;
  for (size_t m = 0; m < meshes.size(); m++) {
    s.blasOffsets.push_back(blasOffset);
    s.vertexOffsets.push_back(vertexOffset);
    blasOffset += uint32_t(s.blases[m].buffer.size() / 4);
    vertexOffset += s.blases[m].vertexCount;
    blasDepth = std::max(blasDepth, s.blases[m].maxDepth);
    s.uniqueTriangleCount += meshes[m].indices.size() / 3;
  }
  s.triangleCount = 0;
  for (const Instance &ins : instances) s.triangleCount += meshes[ins.blasIndex].indices.size() / 3;
  Tlas tlas = buildTlas(instances, s.blases, s.blasOffsets, s.vertexOffsets, tlasBins);
  s.sourceInstances = instances;
  s.sourcePositions.clear();
  s.sourceIndices.clear();
  s.sourceVertexMaterials.clear();
  for (const MeshData &md : meshes) {
    s.sourcePositions.push_back(md.positions);
    s.sourceIndices.push_back(md.indices);
    s.sourceVertexMaterials.push_back(md.vertexMaterials);
  }
  s.blasBins = uint32_t(blasBins);
  s.tlasVec4 = uint32_t(tlas.buffer.size() / 4);
  s.bvh = tlas.buffer;
  for (const Blas &b : s.blases) s.bvh.insert(s.bvh.end(), b.buffer.begin(), b.buffer.end());
  s.instances = tlas.instances;
  buildTrianglePlane(s);
  s.tlasStack = std::min(64u, std::max(1u, tlas.maxDepth));
  s.blasStack = std::min(64u, blasDepth);
  // Compact vertices (compactVertices.ts:7-27, 67-90): position f32x3 + oct
  // normal (or f32x3 normal), then an f32 UV pair when any mesh has UVs, then
  // the vertex color when any mesh has colors: RGBA8 in one word, or f32x3
  // when some component lies outside [0, 1].
  bool hasUv = false, hasUv1 = false, hasColor = false, colorFloat = false;
  for (const MeshData &md : meshes) {
    hasUv |= !md.uvs.empty() || !md.uv1s.empty();
    hasUv1 |= !md.uv1s.empty();
    hasColor |= !md.colors.empty();
    for (float c : md.colors)
      if (!(c >= 0.0f && c <= 1.0f)) colorFloat = true;
  }
  const uint32_t uvOffset = hasUv ? (normalFloat ? 6u : 4u) : 0u;
  uint32_t stride = (normalFloat ? 6 : 4) + (hasUv ? 2 : 0);
  const uint32_t uv1Offset = hasUv1 ? stride : 0u;  // UV1_OFF; absent: it aliases UV_OFF
  if (hasUv1) stride += 2;
  const uint32_t colorOffset = hasColor ? stride : 0u;
  if (hasColor) stride += colorFloat ? 3 : 1;
  s.layout = {stride, 3, normalFloat ? 1u : 0u, uvOffset, colorOffset, colorFloat ? 1u : 0u, uv1Offset, 0u};
  s.attributes.assign(size_t(vertexOffset) * stride, 0);
  for (size_t m = 0; m < meshes.size(); m++) {
    const MeshData &md = meshes[m];
    uint32_t vc = uint32_t(md.positions.size() / 3);
    for (uint32_t v = 0; v < vc; v++) {
      uint32_t *w = &s.attributes[size_t(s.vertexOffsets[m] + v) * stride];
      std::memcpy(w, &md.positions[size_t(v) * 3], 12);
      if (normalFloat) std::memcpy(w + 3, &md.normals[size_t(v) * 3], 12);
      else w[3] = octEncode(md.normals[v * 3], md.normals[v * 3 + 1], md.normals[v * 3 + 2]);
      if (uvOffset && !md.uvs.empty()) std::memcpy(w + uvOffset, &md.uvs[size_t(v) * 2], 8);
      // packCompactVertices: uv1 = geometry.uv1 ?? uv
      const std::vector<float> &second = md.uv1s.empty() ? md.uvs : md.uv1s;
      if (uv1Offset && !second.empty()) std::memcpy(w + uv1Offset, &second[size_t(v) * 2], 8);
      if (colorOffset) {
        const float *c = md.colors.empty() ? nullptr : &md.colors[size_t(v) * 3];
        const float r = c ? c[0] : 1.0f, g = c ? c[1] : 1.0f, b = c ? c[2] : 1.0f;
        if (colorFloat) {
          std::memcpy(w + colorOffset, &r, 4);
          std::memcpy(w + colorOffset + 1, &g, 4);
          std::memcpy(w + colorOffset + 2, &b, 4);
        } else {
          // Math.round(x * 255) (round half up) packed R | G << 8 | B << 16 | 0xff << 24
          auto q = [](float x) { return uint32_t(std::floor(double(x) * 255.0 + 0.5)); };
          w[colorOffset] = q(r) | q(g) << 8 | q(b) << 16 | 0xff000000u;
        }
      }
    }
  }
  // Materials.
  s.materials.assign(materials.size() * MTC_MATERIAL_VEC4_ROWS * 4, 0.0f);
  uint32_t features = 0;
  bool hasMedium = false, spectral = false;
  for (size_t i = 0; i < materials.size(); i++) {
    packMaterial(materials[i], &s.materials[i * MTC_MATERIAL_VEC4_ROWS * 4]);
    const MaterialDesc &m = materials[i];
    if (m.coatWeight > 0) features |= MTC_FEATURE_HAS_COAT;
    if (m.fuzzWeight > 0) features |= MTC_FEATURE_HAS_FUZZ;
    if (m.subsurfaceWeight > 0) features |= MTC_FEATURE_HAS_SUBSURFACE;
    if (m.thinFilmWeight > 0) features |= MTC_FEATURE_HAS_THIN_FILM;
    if (m.mediumExtinction[0] > 0 || m.mediumExtinction[1] > 0 || m.mediumExtinction[2] > 0) hasMedium = true;
    // SPECTRAL: some material disperses (wgpuMaterialConstants.ts:14-15).
    if (m.dispersionScale > 0) spectral = true;
  }
  if (!s.env.image.empty()) features |= MTC_FEATURE_USE_ENVMAP;
  if (hasMedium) s.flags |= MTC_SCENE_HAS_MEDIUM;
  if (spectral) s.flags |= MTC_SCENE_SPECTRAL;
  // HAS_ALPHA: some material resolves to mask or blend (wgpuMaterialConstants.ts:60-62).
  s.flags &= ~uint32_t(MTC_SCENE_HAS_ALPHA);
  for (const MaterialDesc &m : materials)
    if (m.alphaMode != 0) s.flags |= MTC_SCENE_HAS_ALPHA;
  // Light choices: environment, analytic lights (sceneAssembly.ts:42-82).
  std::vector<int> types, idx;
  std::vector<double> weights;
  auto push = [&](int type, int index, double w) {
    if (!(w > 0) || !std::isfinite(w)) return;
    types.push_back(type); idx.push_back(index); weights.push_back(w);
  };
  push(MTC_CHOICE_ENVIRONMENT, 0, s.env.image.empty() ? 0.0 : s.env.power);
  for (size_t i = 0; i < lights.size(); i++)
    push(MTC_CHOICE_ANALYTIC, int(i), lights[i].packed ? lights[i].power : lightPower(lights[i]));
  for (size_t i = 0; i < s.emissive.size(); i++)
    push(MTC_CHOICE_EMISSIVE_TRIANGLE, int(i), s.emissive[i].area * s.emissive[i].luminance);
  AliasTable alias = buildAlias(types, idx, weights);
  std::vector<float> analyticPmf(lights.size(), 0.0f), emissivePmf(s.emissive.size(), 0.0f);
  float envPmf = 0.0f;
  for (size_t i = 0; i < types.size(); i++) {
    if (types[i] == MTC_CHOICE_ENVIRONMENT) envPmf = alias.pmfs[i];
    else if (types[i] == MTC_CHOICE_ANALYTIC) analyticPmf[idx[i]] = alias.pmfs[i];
    else emissivePmf[idx[i]] = alias.pmfs[i];
  }
  // Texture: 6 texels per emissive triangle, then the choices (4096 texels
  // per side at most).
  const uint32_t emissiveTexels = uint32_t(s.emissive.size()) * 6;
  uint32_t choiceTexels = std::max<uint32_t>(uint32_t(types.size()), 1u);
  uint32_t totalTexels = std::max(emissiveTexels + choiceTexels, 1u);
  uint32_t width = std::min(4096u, std::max(16u, uint32_t(std::ceil(std::sqrt(double(totalTexels)) / 16.0) * 16)));
  uint32_t height = (totalTexels + width - 1) / width;
  if (height > 4096) throw std::runtime_error("Too many emissive triangles for the light sampling texture.");
  s.lightSampling.assign(size_t(width) * height * 4, 0.0f);
  for (size_t i = 0; i < s.emissive.size(); i++) {
    const EmissiveTriangle &t = s.emissive[i];
    float *d = &s.lightSampling[i * 24];
    d[0] = t.p[0]; d[1] = t.p[1]; d[2] = t.p[2]; d[3] = emissivePmf[i];
    d[4] = t.p[3]; d[5] = t.p[4]; d[6] = t.p[5]; d[7] = float(t.area);
    d[8] = t.p[6]; d[9] = t.p[7]; d[10] = t.p[8]; d[11] = float(t.material);
    for (int k = 0; k < 6; k++) {
      d[12 + k] = t.uv[k];
      d[18 + k] = t.uv1[k];
    }
  }
  std::memcpy(s.lightSampling.data() + size_t(emissiveTexels) * 4, alias.words.data(), alias.words.size() * 4);
  // Analytic light records (wgpuSceneUniform.ts:70-152).
  s.lights.assign(lights.size() * 24, 0.0f);
  for (size_t i = 0; i < lights.size(); i++) {
    const LightDesc &L = lights[i];
    float *d = &s.lights[i * 24];
    if (L.packed) {
      std::memcpy(d, L.rows, sizeof(L.rows));
      d[16] = analyticPmf[i];
      continue;
    }
    d[0] = L.position[0]; d[1] = L.position[1]; d[2] = L.position[2]; d[3] = float(L.type);
    d[4] = L.color[0] * L.intensity; d[5] = L.color[1] * L.intensity; d[6] = L.color[2] * L.intensity;
    d[15] = -1.0f;
    if (L.type == MTC_LIGHT_RECT) {
      d[7] = L.area;
      d[8] = L.u[0]; d[9] = L.u[1]; d[10] = L.u[2]; d[11] = L.spread;
      d[12] = L.v[0]; d[13] = L.v[1]; d[14] = L.v[2];
    } else if (L.type == MTC_LIGHT_SPHERE) {
      d[7] = float(4.0 * M_PI * double(L.radius) * L.radius);
      d[11] = L.radius;
    } else if (L.type == MTC_LIGHT_DISK) {
      d[7] = L.area;
      d[8] = L.u[0]; d[9] = L.u[1]; d[10] = L.u[2]; d[11] = L.radius;
      d[12] = L.v[0]; d[13] = L.v[1]; d[14] = L.v[2];
    } else if (L.type == MTC_LIGHT_DIRECTIONAL) {
      d[8] = L.u[0]; d[9] = L.u[1]; d[10] = L.u[2];
    }
    d[16] = analyticPmf[i];
    d[20] = L.frameX[0]; d[21] = L.frameX[1]; d[22] = L.frameX[2];
  }
  // Energy LUT (cached across scenes).
  static std::vector<float> lutCache;
  if (lutCache.empty()) buildEnergyLut(lutCache);
  s.lut = lutCache;
  // Uniform fields owned by the scene.
  mtc_trace_uniform &u = s.uniform;
  u.lights_count = int32_t(lights.size());
  u.blas_offset = int32_t(s.tlasVec4);
  u.is_empty = instances.empty() ? 1 : 0;
  u.env_light_pmf = envPmf;
  u.light_choice_count = int32_t(types.size());
  u.light_weight_total = float(alias.total);
  u.light_sampling_texture_width = int32_t(width);
  u.light_choice_texel_offset = int32_t(emissiveTexels);
  u.scene_feature_flags = features;
}

// ------------------------------------------------------------ generators
static double identity4[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};

static void trs(double *m, const double t[3], double rotY, double rotAxis[3], double angle, double scale) {
  // Rotation about an arbitrary unit axis (angle) composed with rotY about +y.
  double ax = rotAxis[0], ay = rotAxis[1], az = rotAxis[2];
  double c = std::cos(angle), s = std::sin(angle), C = 1 - c;
  double R1[9] = {c + ax * ax * C, ay * ax * C + az * s, az * ax * C - ay * s,
                  ax * ay * C - az * s, c + ay * ay * C, az * ay * C + ax * s,
                  ax * az * C + ay * s, ay * az * C - ax * s, c + az * az * C};
  double cy = std::cos(rotY), sy = std::sin(rotY);
  double R2[9] = {cy, 0, -sy, 0, 1, 0, sy, 0, cy};
  double R[9];
  for (int col = 0; col < 3; col++)
    for (int row = 0; row < 3; row++) {
      double acc = 0;
      for (int k = 0; k < 3; k++) acc += R2[k * 3 + row] * R1[col * 3 + k];
      R[col * 3 + row] = acc;
    }
  for (int col = 0; col < 3; col++) {
    for (int row = 0; row < 3; row++) m[col * 4 + row] = R[col * 3 + row] * scale;
    m[col * 4 + 3] = 0;
  }
  m[12] = t[0]; m[13] = t[1]; m[14] = t[2]; m[15] = 1;
}

static MeshData makeQuad() {
  MeshData m;
  // Unit quad in the xz plane facing +y.
  m.positions = {-0.5f, 0, -0.5f, 0.5f, 0, -0.5f, 0.5f, 0, 0.5f, -0.5f, 0, 0.5f};
  m.normals = {0, 1, 0, 0, 1, 0, 0, 1, 0, 0, 1, 0};
  m.indices = {0, 2, 1, 0, 3, 2};
  return m;
}
static MeshData makeBox() {
  MeshData m;
  const float n[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
  for (int f = 0; f < 6; f++) {
    float N[3] = {n[f][0], n[f][1], n[f][2]};
    float U[3] = {N[1], N[2], N[0]}, V[3];
    V[0] = N[1] * U[2] - N[2] * U[1]; V[1] = N[2] * U[0] - N[0] * U[2]; V[2] = N[0] * U[1] - N[1] * U[0];
    uint32_t base = uint32_t(m.positions.size() / 3);
    const float cs[4][2] = {{-1, -1}, {1, -1}, {1, 1}, {-1, 1}};
    for (auto &c : cs) {
      for (int k = 0; k < 3; k++) m.positions.push_back(0.5f * (N[k] + c[0] * U[k] + c[1] * V[k]));
      for (int k = 0; k < 3; k++) m.normals.push_back(N[k]);
    }
    m.indices.insert(m.indices.end(), {base, base + 1, base + 2, base, base + 2, base + 3});
  }
  return m;
}

// Value noise on an integer lattice, smoothstep-interpolated.
struct ValueNoise {
  std::vector<float> table;
  explicit ValueNoise(uint64_t seed) {
    Pcg32 r(seed, 11);
    table.resize(4096);
    for (float &v : table) v = float(r.uniform() * 2.0 - 1.0);
  }
  float lattice(int x, int y, int z) const {
    uint32_t h = uint32_t(x) * 73856093u ^ uint32_t(y) * 19349663u ^ uint32_t(z) * 83492791u;
    h ^= h >> 13; h *= 0x5bd1e995u; h ^= h >> 15;
    return table[h & 4095u];
  }
  float operator()(double x, double y, double z) const {
    int xi = int(std::floor(x)), yi = int(std::floor(y)), zi = int(std::floor(z));
    double fx = x - xi, fy = y - yi, fz = z - zi;
    auto sm = [](double t) { return t * t * (3 - 2 * t); };
    double u = sm(fx), v = sm(fy), w = sm(fz);
    double acc = 0;
    for (int c = 0; c < 8; c++) {
      int dx = c & 1, dy = (c >> 1) & 1, dz = (c >> 2) & 1;
      double wt = (dx ? u : 1 - u) * (dy ? v : 1 - v) * (dz ? w : 1 - w);
      acc += wt * lattice(xi + dx, yi + dy, zi + dz);
    }
    return float(acc);
  }
};

// Icosahedron with every face split at `frequency`, projected to the unit
// sphere and displaced along the normal by amplitude * value noise.
static MeshData makeIcosphere(uint32_t frequency, double amplitude, uint64_t seed) {
  const double t = (1.0 + std::sqrt(5.0)) / 2.0;
  double V[12][3] = {{-1, t, 0}, {1, t, 0}, {-1, -t, 0}, {1, -t, 0}, {0, -1, t}, {0, 1, t},
                     {0, -1, -t}, {0, 1, -t}, {t, 0, -1}, {t, 0, 1}, {-t, 0, -1}, {-t, 0, 1}};
  const int F[20][3] = {{0, 11, 5}, {0, 5, 1}, {0, 1, 7}, {0, 7, 10}, {0, 10, 11}, {1, 5, 9}, {5, 11, 4},
                        {11, 10, 2}, {10, 7, 6}, {7, 1, 8}, {3, 9, 4}, {3, 4, 2}, {3, 2, 6}, {3, 6, 8},
                        {3, 8, 9}, {4, 9, 5}, {2, 4, 11}, {6, 2, 10}, {8, 6, 7}, {9, 8, 1}};
  MeshData m;
  std::map<std::tuple<int64_t, int64_t, int64_t>, uint32_t> dedup;
  ValueNoise noise(seed);
  auto vertex = [&](double x, double y, double z) -> uint32_t {
    double l = std::sqrt(x * x + y * y + z * z);
    x /= l; y /= l; z /= l;
    auto key = std::make_tuple(int64_t(std::llround(x * 1e7)), int64_t(std::llround(y * 1e7)), int64_t(std::llround(z * 1e7)));
    auto it = dedup.find(key);
    if (it != dedup.end()) return it->second;
    double n = noise(x * 3.0 + 11.0, y * 3.0 + 7.0, z * 3.0 + 5.0) + 0.5 * noise(x * 7.0, y * 7.0, z * 7.0);
    double r = 1.0 + amplitude * n;
    uint32_t id = uint32_t(m.positions.size() / 3);
    m.positions.insert(m.positions.end(), {float(x * r), float(y * r), float(z * r)});
    dedup.emplace(key, id);
    return id;
  };
  for (auto &f : F) {
    const double *a = V[f[0]], *b = V[f[1]], *c = V[f[2]];
    std::vector<std::vector<uint32_t>> rows(frequency + 1);
    for (uint32_t i = 0; i <= frequency; i++)
      for (uint32_t j = 0; j <= frequency - i; j++) {
        double u = double(i) / frequency, v = double(j) / frequency, w = 1.0 - u - v;
        rows[i].push_back(vertex(a[0] * w + b[0] * u + c[0] * v, a[1] * w + b[1] * u + c[1] * v, a[2] * w + b[2] * u + c[2] * v));
      }
    for (uint32_t i = 0; i < frequency; i++)
      for (uint32_t j = 0; j < frequency - i; j++) {
        m.indices.insert(m.indices.end(), {rows[i][j], rows[i + 1][j], rows[i][j + 1]});
        if (j + 1 < frequency - i) m.indices.insert(m.indices.end(), {rows[i + 1][j], rows[i + 1][j + 1], rows[i][j + 1]});
      }
  }
  // Area-weighted vertex normals.
  m.normals.assign(m.positions.size(), 0.0f);
  std::vector<double> acc(m.positions.size(), 0.0);
  for (size_t k = 0; k < m.indices.size(); k += 3) {
    const float *p0 = &m.positions[m.indices[k] * 3], *p1 = &m.positions[m.indices[k + 1] * 3], *p2 = &m.positions[m.indices[k + 2] * 3];
    double e1[3] = {p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2]}, e2[3] = {p2[0] - p0[0], p2[1] - p0[1], p2[2] - p0[2]};
    double n[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
    for (int c = 0; c < 3; c++)
      for (int d = 0; d < 3; d++) acc[m.indices[k + c] * 3 + d] += n[d];
  }
  for (size_t v = 0; v < acc.size(); v += 3) {
    double l = std::sqrt(acc[v] * acc[v] + acc[v + 1] * acc[v + 1] + acc[v + 2] * acc[v + 2]);
    for (int d = 0; d < 3; d++) m.normals[v + d] = float(acc[v + d] / (l > 0 ? l : 1));
  }
  // Orient faces outward (normals point away from the center).
  for (size_t k = 0; k < m.indices.size(); k += 3) {
    const float *p0 = &m.positions[m.indices[k] * 3], *p1 = &m.positions[m.indices[k + 1] * 3], *p2 = &m.positions[m.indices[k + 2] * 3];
    double e1[3] = {p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2]}, e2[3] = {p2[0] - p0[0], p2[1] - p0[1], p2[2] - p0[2]};
    double n[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
    if (n[0] * p0[0] + n[1] * p0[1] + n[2] * p0[2] < 0) std::swap(m.indices[k + 1], m.indices[k + 2]);
  }
  return m;
}

static int32_t packMaterialIndex(int index) { return int32_t(255 + (index << 8)); }

// Procedural Cornell box: 5 wall quads, two boxes (one rotated 15 degrees)
// and a ceiling rect light; diffuse OpenPBR base colors from PCG32 seed 1.
void makeCornell(SceneHost &s, uint32_t width, uint32_t height, uint64_t seed) {
  s = SceneHost();
  s.name = "cornell";
  s.width = width; s.height = height;
  Pcg32 rng(seed, 1);
  std::vector<MeshData> meshes = {makeQuad(), makeBox()};
  std::vector<MaterialDesc> mats;
  auto diffuse = [&](float r, float g, float b) {
    MaterialDesc m;
    m.baseColor[0] = r; m.baseColor[1] = g; m.baseColor[2] = b;
    m.specularRoughness = 0.5f;
    mats.push_back(m);
    return int(mats.size() - 1);
  };
  auto rnd = [&]() { return float(rng.range(0.1, 0.8)); };
  int floorM = diffuse(rnd(), rnd(), rnd());
  int ceilM = diffuse(rnd(), rnd(), rnd());
  int backM = diffuse(rnd(), rnd(), rnd());
  int redM = diffuse(0.8f, 0.1f, 0.1f);
  int greenM = diffuse(0.1f, 0.8f, 0.1f);
  int tallM = diffuse(rnd(), rnd(), rnd());
  int shortM = diffuse(rnd(), rnd(), rnd());
  std::vector<Instance> ins;
  double ax[3] = {0, 1, 0}, xa[3] = {1, 0, 0}, za[3] = {0, 0, 1};
  auto quad = [&](const double t[3], double *axis, double angle, int mat) {
    Instance i;
    i.blasIndex = 0;
    trs(i.transform, t, 0.0, axis, angle, 2.0);
    i.material = packMaterialIndex(mat);
    ins.push_back(i);
  };
  double tf[3] = {0, 0, 0}, tc[3] = {0, 2, 0}, tb[3] = {0, 1, -1}, tl[3] = {-1, 1, 0}, tr_[3] = {1, 1, 0};
  quad(tf, ax, 0.0, floorM);
  quad(tc, xa, M_PI, ceilM);
  quad(tb, xa, M_PI / 2, backM);
  quad(tl, za, -M_PI / 2, redM);
  quad(tr_, za, M_PI / 2, greenM);
  auto box = [&](double x, double z, double sx, double sy, double sz, double rotY, int mat) {
    Instance i;
    i.blasIndex = 1;
    double R[16];
    double t[3] = {x, sy * 0.5, z};
    trs(R, t, rotY, ax, 0.0, 1.0);
    // non-uniform scale: M = T * R * S
    double S[3] = {sx, sy, sz};
    for (int col = 0; col < 3; col++)
      for (int row = 0; row < 3; row++) i.transform[col * 4 + row] = R[col * 4 + row] * S[col];
    for (int col = 0; col < 3; col++) i.transform[col * 4 + 3] = 0;
    i.transform[12] = t[0]; i.transform[13] = t[1]; i.transform[14] = t[2]; i.transform[15] = 1;
    i.material = packMaterialIndex(mat);
    ins.push_back(i);
  };
  box(-0.33, -0.25, 0.55, 1.2, 0.55, 15.0 * M_PI / 180.0, tallM);
  box(0.35, 0.3, 0.55, 0.6, 0.55, -18.0 * M_PI / 180.0, shortM);
  LightDesc L;
  L.type = MTC_LIGHT_RECT;
  L.position[0] = 0; L.position[1] = 1.98f; L.position[2] = 0;
  L.u[0] = 0.5f; L.u[1] = 0; L.u[2] = 0;
  L.v[0] = 0; L.v[1] = 0; L.v[2] = 0.4f;
  L.area = 0.5f * 0.4f;
  L.color[0] = 1.0f; L.color[1] = 0.85f; L.color[2] = 0.7f;
  L.intensity = 25.0f;
  L.spread = 1.0f;
  L.frameX[0] = 1; L.frameX[1] = 0; L.frameX[2] = 0;
  assembleScene(s, meshes, ins, mats, {L}, 16, 8, false);
  defaultUniform(s, 8, 2, 0, MT_SAMPLING_SOBOL);
  CameraDesc c{{0, 1, 3.4}, {0, 1, 0}, {0, 1, 0}, 40.0};
  setCamera(s, c);
  (void)identity4;
}

// 256 seeded affine instances of 16 displaced icospheres under an analytic
// sky with rect lights; 1/3 diffuse, 1/3 F82 metal, 1/3 coated.
void makeInstancedSpheres(SceneHost &s, uint32_t width, uint32_t height, uint64_t seed, uint32_t instances,
                          uint32_t baseMeshes, uint32_t frequency, uint32_t envWidth, uint32_t rectLights) {
  s = SceneHost();
  s.name = "instanced_spheres";
  s.width = width; s.height = height;
  Pcg32 rng(seed, 2);
  std::vector<MeshData> meshes(baseMeshes + 1);
  {
    std::vector<std::thread> pool;
    for (uint32_t t = 0; t < std::min(8u, baseMeshes); t++)
      pool.emplace_back([&, t] {
        for (uint32_t m = t; m < baseMeshes; m += std::min(8u, baseMeshes)) meshes[m] = makeIcosphere(frequency, 0.05, seed * 131 + m);
      });
    for (auto &th : pool) th.join();
  }
  meshes[baseMeshes] = makeQuad();
  std::vector<MaterialDesc> mats;
  std::vector<Instance> ins;
  double extent = 6.0 * std::cbrt(double(instances) / 256.0);
  for (uint32_t i = 0; i < instances; i++) {
    MaterialDesc m;
    int kind = int(i % 3);
    m.baseColor[0] = float(rng.range(0.1, 0.8)); m.baseColor[1] = float(rng.range(0.1, 0.8)); m.baseColor[2] = float(rng.range(0.1, 0.8));
    if (kind == 1) {
      m.baseMetalness = 1.0f;
      m.specularRoughness = float(rng.range(0.05, 0.6));
      m.specularColor[0] = float(rng.range(0.7, 1.0)); m.specularColor[1] = float(rng.range(0.7, 1.0)); m.specularColor[2] = float(rng.range(0.7, 1.0));
    } else if (kind == 2) {
      m.coatWeight = 1.0f;
      m.coatRoughness = float(rng.range(0.0, 0.2));
      m.specularRoughness = float(rng.range(0.2, 0.6));
    } else {
      m.specularRoughness = float(rng.range(0.3, 0.8));
    }
    mats.push_back(m);
    Instance inst;
    inst.blasIndex = uint32_t(rng.next() % baseMeshes);
    double axis[3] = {rng.range(-1, 1), rng.range(-1, 1), rng.range(-1, 1)};
    double al = std::sqrt(axis[0] * axis[0] + axis[1] * axis[1] + axis[2] * axis[2]);
    for (double &a : axis) a /= (al > 0 ? al : 1);
    double scale = rng.range(0.5, 2.0);
    double t[3] = {rng.range(-extent, extent), scale + rng.range(0.0, extent * 0.6), rng.range(-extent, extent)};
    trs(inst.transform, t, 0.0, axis, rng.range(0, 2 * M_PI), scale);
    inst.material = packMaterialIndex(int(i));
    ins.push_back(inst);
  }
  MaterialDesc ground;
  ground.baseColor[0] = 0.5f; ground.baseColor[1] = 0.5f; ground.baseColor[2] = 0.48f;
  ground.specularRoughness = 0.7f;
  mats.push_back(ground);
  Instance g;
  g.blasIndex = baseMeshes;
  double ax[3] = {0, 1, 0};
  double tg[3] = {0, 0, 0};
  trs(g.transform, tg, 0.0, ax, 0.0, extent * 4.0);
  g.material = packMaterialIndex(int(mats.size() - 1));
  ins.push_back(g);
  makeAnalyticSky(s.env, envWidth, envWidth / 2, seed);
  std::vector<LightDesc> lights;
  for (uint32_t l = 0; l < rectLights; l++) {
    LightDesc L;
    L.type = MTC_LIGHT_RECT;
    double ang = 2 * M_PI * (l + 0.5) / std::max(1u, rectLights);
    L.position[0] = float(std::cos(ang) * extent * 0.8); L.position[1] = float(extent * 1.4);
    L.position[2] = float(std::sin(ang) * extent * 0.8);
    L.u[0] = 2.0f; L.u[1] = 0; L.u[2] = 0;
    L.v[0] = 0; L.v[1] = 0; L.v[2] = 2.0f;
    L.area = 4.0f;
    L.color[0] = float(rng.range(0.7, 1.0)); L.color[1] = float(rng.range(0.7, 1.0)); L.color[2] = float(rng.range(0.7, 1.0));
    L.intensity = 8.0f;
    L.spread = 1.0f;
    lights.push_back(L);
  }
  assembleScene(s, meshes, ins, mats, lights, 8, 8, false);
  defaultUniform(s, 6, 2, 0, MT_SAMPLING_SOBOL);
  CameraDesc c{{extent * 1.9, extent * 1.1, extent * 1.9}, {0, extent * 0.3, 0}, {0, 1, 0}, 50.0};
  setCamera(s, c);
}

// Glass spheres (IOR 1.5, Abbe 40, dispersion scale 1) with homogeneous
// interiors over a diffuse ground, lit by one sphere light.
void makeGlassSpheres(SceneHost &s, uint32_t width, uint32_t height, uint64_t seed, uint32_t spheres) {
  s = SceneHost();
  s.name = "glass_spheres";
  s.width = width; s.height = height;
  Pcg32 rng(seed, 5);
  std::vector<MeshData> meshes = {makeIcosphere(12, 0.0, seed), makeQuad()};
  std::vector<MaterialDesc> mats;
  std::vector<Instance> ins;
  double ax[3] = {0, 1, 0};
  for (uint32_t i = 0; i < spheres; i++) {
    MaterialDesc m;
    m.transmissionWeight = 1.0f;
    m.specularRoughness = 0.02f;
    m.specularIor = 1.5f;
    m.dispersionScale = 1.0f;
    m.abbe = 40.0f;
    float sigmaS = float(rng.range(0.1, 2.0));
    for (int k = 0; k < 3; k++) {
      m.mediumScattering[k] = sigmaS;
      m.mediumExtinction[k] = sigmaS + float(rng.range(0.0, 0.3));
    }
    mats.push_back(m);
    Instance inst;
    inst.blasIndex = 0;
    double r = rng.range(0.25, 0.6);
    double t[3] = {rng.range(-3.0, 3.0), r, rng.range(-3.0, 3.0)};
    trs(inst.transform, t, 0.0, ax, 0.0, r);
    inst.material = packMaterialIndex(int(i));
    ins.push_back(inst);
  }
  MaterialDesc ground;
  ground.baseColor[0] = 0.6f; ground.baseColor[1] = 0.6f; ground.baseColor[2] = 0.6f;
  ground.specularRoughness = 0.8f;
  mats.push_back(ground);
  Instance g;
  g.blasIndex = 1;
  double tg[3] = {0, 0, 0};
  trs(g.transform, tg, 0.0, ax, 0.0, 20.0);
  g.material = packMaterialIndex(int(mats.size() - 1));
  ins.push_back(g);
  LightDesc L;
  L.type = MTC_LIGHT_SPHERE;
  L.position[0] = 2.0f; L.position[1] = 5.0f; L.position[2] = 1.0f;
  L.radius = 0.5f;
  L.intensity = 60.0f;
  assembleScene(s, meshes, ins, mats, {L}, 8, 8, false);
  defaultUniform(s, 32, 2, 0, MT_SAMPLING_SOBOL);
  CameraDesc c{{0, 2.5, 7.5}, {0, 0.4, 0}, {0, 1, 0}, 45.0};
  setCamera(s, c);
}

}  // namespace mtp
