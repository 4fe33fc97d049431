"""Test infrastructure only: pure-Python restatement of the reference's
binned-SAH BVH builder and depth-first BVH2 layout, used to check the C++
producer in mutracer_b200/csrc/scene_prep.cpp bit for bit on small inputs.

Follows src/renderer/binnedSahBvh.ts:70-236 (buildBinnedSahBvh) and :252-275
(layoutBvh2): float64 arithmetic on values stored as float32 (the JS
Float32Array bounds/centers and Float64Array bins), with JavaScript's
Math.min / Math.max (js_min / js_max) where the reference calls them.
"""
import math

import numpy as np

FAR = 1e30


def _f32(x):
    return float(np.float32(x))


def js_min(a, b):
    """JavaScript Math.min: NaN if either is NaN; -0 below +0."""
    if a != a or b != b:
        return float("nan")
    if a == b:
        return a if math.copysign(1.0, a) < 0 else b
    return b if b < a else a


def js_max(a, b):
    """JavaScript Math.max: NaN if either is NaN; +0 above -0."""
    if a != a or b != b:
        return float("nan")
    if a == b:
        return b if math.copysign(1.0, a) < 0 else a
    return b if b > a else a


def _to_int32(v):
    # JavaScript `v | 0` for the binning range.
    if v != v or v in (float("inf"), float("-inf")):
        return 0
    t = int(v)  # truncation toward zero
    t &= 0xFFFFFFFF
    return t - (1 << 32) if t >= 1 << 31 else t


def build_binned_sah(aabbs, bins=8):
    """aabbs: (n, 6) float32. Returns (node_count, bounds (m,6) f32,
    left_first, prim_count, prim_indices) as in BinnedSahBvh."""
    aabbs = np.asarray(aabbs, dtype=np.float32)
    count = aabbs.shape[0]
    capacity = max(1, count * 2 - 1)
    bounds = np.zeros((capacity, 6), np.float32)
    left_first = np.zeros(capacity, np.uint32)
    prim_count = np.zeros(capacity, np.uint32)
    prim = np.zeros(count, np.uint32)
    if count == 0:
        return 0, bounds, left_first, prim_count, prim
    a = aabbs.astype(np.float64)
    centers = np.zeros((count, 3), np.float32)
    root_min = [FAR] * 3
    root_max = [-FAR] * 3
    for i in range(count):
        for k in range(3):
            centers[i, k] = _f32((a[i, k] + a[i, 3 + k]) * 0.5)
            root_min[k] = float(a[i, k]) if a[i, k] < root_min[k] else root_min[k]
            root_max[k] = float(a[i, 3 + k]) if a[i, 3 + k] > root_max[k] else root_max[k]
        prim[i] = i
    bounds[0, :3] = root_min
    bounds[0, 3:] = root_max
    prim_count[0] = count
    min_dim = [(root_max[k] - root_min[k]) * 1e-20 for k in range(3)]

    def bin_of(center, nmin, scale):
        b = _to_int32((center - nmin) * scale)
        return 0 if b < 0 else (bins - 1 if b > bins - 1 else b)

    new_node = 1
    tasks = []
    node = 0
    while True:
        while True:
            nmin = [float(bounds[node, k]) for k in range(3)]
            extent = [float(bounds[node, 3 + k]) - nmin[k] for k in range(3)]
            area = extent[0] * extent[1] + extent[1] * extent[2] + extent[2] * extent[0]
            if area == 0:
                break
            first = int(left_first[node])
            nprims = int(prim_count[node])
            if nprims == 1:
                break
            scale = [bins / extent[k] if extent[k] > min_dim[k] else 0.0 for k in range(3)]
            bmin = [[FAR] * 3 for _ in range(3 * bins)]
            bmax = [[-FAR] * 3 for _ in range(3 * bins)]
            bcnt = [0] * (3 * bins)
            for i in range(first, first + nprims):
                p = int(prim[i])
                for axis in range(3):
                    b = axis * bins + bin_of(float(centers[p, axis]), nmin[axis], scale[axis])
                    bcnt[b] += 1
                    for k in range(3):
                        bmin[b][k] = js_min(bmin[b][k], float(a[p, k]))
                        bmax[b][k] = js_max(bmax[b][k], float(a[p, 3 + k]))
            split_cost, best_axis, best_pos = FAR, 0, 0
            for axis in range(3):
                if not extent[axis] > min_dim[axis]:
                    continue
                lmin, lmax, rmin, rmax = [FAR] * 3, [-FAR] * 3, [FAR] * 3, [-FAR] * 3
                ln = rn = 0
                lc = [0.0] * (bins - 1)
                rc = [0.0] * (bins - 1)
                for i in range(bins - 1):
                    l, r = axis * bins + i, axis * bins + bins - 1 - i
                    for k in range(3):
                        lmin[k] = js_min(lmin[k], bmin[l][k]); lmax[k] = js_max(lmax[k], bmax[l][k])
                        rmin[k] = js_min(rmin[k], bmin[r][k]); rmax[k] = js_max(rmax[k], bmax[r][k])
                    ln += bcnt[l]
                    rn += bcnt[r]
                    lx, ly, lz = lmax[0] - lmin[0], lmax[1] - lmin[1], lmax[2] - lmin[2]
                    rx, ry, rz = rmax[0] - rmin[0], rmax[1] - rmin[1], rmax[2] - rmin[2]
                    lc[i] = FAR if ln == 0 else (lx * ly + ly * lz + lz * lx) * ln
                    rc[bins - 2 - i] = FAR if rn == 0 else (rx * ry + ry * rz + rz * rx) * rn
                for i in range(bins - 1):
                    c = lc[i] + rc[i]
                    if c < split_cost:
                        split_cost, best_axis, best_pos = c, axis, i
            split_cost = 1 + 1 * split_cost / area
            if not split_cost < nprims * 1:
                break
            sc, nm = scale[best_axis], nmin[best_axis]
            j, src = first + nprims, first
            for _ in range(nprims):
                p = int(prim[src])
                if bin_of(float(centers[p, best_axis]), nm, sc) <= best_pos:
                    src += 1
                else:
                    j -= 1
                    prim[src] = prim[j]
                    prim[j] = p
            lp = src - first
            rp = nprims - lp
            if lp == 0 or rp == 0:
                break
            n = new_node
            new_node += 2
            lb = [FAR, FAR, FAR, -FAR, -FAR, -FAR]
            rb = [FAR, FAR, FAR, -FAR, -FAR, -FAR]
            for i in range(bins):
                o = best_axis * bins + i
                base = lb if i <= best_pos else rb
                for k in range(3):
                    if bmin[o][k] < base[k]:
                        base[k] = bmin[o][k]
                    if bmax[o][k] > base[3 + k]:
                        base[3 + k] = bmax[o][k]
            bounds[n] = lb
            bounds[n + 1] = rb
            left_first[n], prim_count[n] = first, lp
            left_first[n + 1], prim_count[n + 1] = j, rp
            left_first[node], prim_count[node] = n, 0
            tasks.append(n + 1)
            node = n
        if not tasks:
            break
        node = tasks.pop()
    return new_node, bounds, left_first, prim_count, prim


def layout_bvh2(node_count, left_first, prim_count):
    """binnedSahBvh.ts:252-275: (order, offsets, vec4_count, max_depth)."""
    order, offsets = [0] * node_count, [0] * node_count
    vec4, max_depth, written = 0, 0, 0
    if not node_count:
        return order, offsets, 0, 0
    stack = [0, 1]
    while stack:
        depth = stack.pop()
        node = stack.pop()
        order[written] = node
        written += 1
        offsets[node] = vec4
        max_depth = max(max_depth, depth)
        prims = int(prim_count[node])
        vec4 += 2 + prims
        if not prims:
            stack += [int(left_first[node]) + 1, depth + 1, int(left_first[node]), depth + 1]
    return order, offsets, vec4, max_depth


def refit_blas(buffer, positions):
    """bvhAccel.ts:800-870 refitBLAS (BVH2, no displacement) on a copy of a
    layout-0 BLAS buffer: post order (descendants before ancestors), leaves
    from the finite vertices of their triangles (indices past the position
    array skipped), interior nodes from their children, Math.min/max.
    Returns (buffer f32, summed surface area in post order)."""
    f = np.array(buffer, dtype=np.float32).reshape(-1, 4)
    ints = f.view(np.int32)
    pos = np.asarray(positions, dtype=np.float32).reshape(-1, 3)
    preorder, stack = [], [0]
    while stack:
        o = stack.pop()
        preorder.append(o)
        w = int(ints[o, 3])
        if w >= 0:
            stack += [w, o + 2]
    area = 0.0
    for o in reversed(preorder):
        w = int(ints[o, 3])
        mn, mx = [math.inf] * 3, [-math.inf] * 3
        if w >= 0:
            for c in range(3):
                mn[c] = js_min(float(f[o + 2, c]), float(f[w, c]))
                mx[c] = js_max(float(f[o + 3, c]), float(f[w + 1, c]))
        else:
            for t in range(-w):
                for c in range(3):
                    v = int(np.uint32(ints[o + 2 + t, c]))
                    if v >= len(pos):
                        continue
                    p = [float(x) for x in pos[v]]
                    if not all(math.isfinite(x) for x in p):
                        continue
                    for k in range(3):
                        mn[k] = js_min(mn[k], p[k])
                        mx[k] = js_max(mx[k], p[k])
        x, y, z = mx[0] - mn[0], mx[1] - mn[1], mx[2] - mn[2]
        area += 2 * (x * z + x * y + z * y)
        f[o, :3] = mn
        f[o + 1, :3] = mx
    return f.reshape(-1), area
