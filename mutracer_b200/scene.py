"""Seeded synthetic scenes in the reference's flattened buffer formats.

``SceneHost`` owns the host buffers produced by the C++ scene producers
(binned-SAH BVH2 TLAS/BLAS, instance records, compact vertices, 26-row
materials, analytic lights + alias table, environment CDF, energy LUT).
``DeviceScene`` uploads them into device memory and exposes the
``mtc_scene_view`` the kernels consume.
"""
import ctypes as C

import numpy as np

from . import abi

WORKLOADS = {
    # Plain method, small: Cornell box, 512^2, 64 spp, 8 bounces, 16 SAH bins.
    "cornell": dict(kind="cornell", width=512, height=512, spp=64, params=()),
    # Plain method, large: 256 instances of 16 displaced icospheres (frequency
    # 28, 15,680 triangles each), analytic sky 2048x1024 + 4 rect lights,
    # 1920x1080, 16 spp, 6 bounces.
    "instanced_spheres": dict(kind="instanced_spheres", width=1920, height=1080, spp=16,
                              params=(256, 16, 28, 2048, 4)),
    # Deep transport: 32 dispersive glass spheres with homogeneous media.
    "glass_spheres": dict(kind="glass_spheres", width=1280, height=720, spp=256, params=(32,)),
}


def _np(ptr, count, dtype):
    if not ptr or count == 0:
        return np.zeros(0, dtype=dtype)
    ctype = C.c_float if dtype == np.float32 else C.c_uint32
    buf = C.cast(ptr, C.POINTER(ctype))
    return np.ctypeslib.as_array(buf, shape=(int(count),)).view(dtype)


class SceneHost:
    """Host-memory scene produced by a seeded generator."""

    def __init__(self, kind, width, height, seed=1, params=()):
        L = abi.lib()
        arr = (C.c_uint32 * max(1, len(params)))(*params)
        self._handle = L.mtp_scene_make(kind.encode(), width, height, seed, arr, len(params))
        if not self._handle:
            raise abi.MtError(abi.MT_ERROR_INVALID_ARGUMENT, f"scene kind {kind!r}")
        self.kind = kind
        self.refresh()

    @classmethod
    def from_handle(cls, handle, kind="descriptor"):
        """Wraps a host scene made elsewhere (mtp_descriptor_decode)."""
        self = cls.__new__(cls)
        self._handle = handle
        self.kind = kind
        self.refresh()
        return self

    def refresh(self):
        L = abi.lib()
        self.bundle = abi.SceneBundle()
        abi.check(L.mtp_scene_bundle(self._handle, C.byref(self.bundle)))
        self.info = abi.SceneInfo()
        abi.check(L.mtp_scene_info(self._handle, C.byref(self.info)))
        b = self.bundle
        self.width, self.height = b.width, b.height
        self.bvh = _np(b.bvh, b.bvh_vec4_count * 4, np.float32)
        self.instances = _np(b.instances, b.instance_count * 40, np.float32)
        self.attributes = _np(b.attributes, b.attribute_words, np.uint32)
        self.materials = _np(b.materials, b.material_count * abi.MTC_MATERIAL_VEC4_ROWS * 4, np.float32)
        self.env_map = _np(b.env_map, b.env_width * b.env_height * 4, np.float32)
        self.env_distribution = _np(b.env_distribution, (b.env_width + 2) * (b.env_height + 1) * 2, np.float32) \
            if b.env_width else np.zeros(0, np.float32)
        self.light_sampling = _np(b.light_sampling, b.light_sampling_texels * 4, np.float32)
        self.energy_lut = _np(b.energy_lut, abi.MTC_ENERGY_LUT_WIDTH * abi.MTC_ENERGY_LUT_HEIGHT, np.float32)
        self.lights = _np(b.analytic_lights, b.lights_count * abi.MTC_LIGHT_VEC4_ROWS * 4, np.float32)
        self.maps = _np(b.maps, b.map_count * abi.MTC_MAP_VEC4_ROWS * 4, np.float32) if b.map_count \
            else np.zeros(0, np.float32)
        self.map_texels = _np(b.map_texels, b.map_texel_count * 4, np.float32) if b.map_texel_count \
            else np.zeros(0, np.float32)
        self.triangle_materials = _np(b.triangle_materials, b.bvh_vec4_count, np.uint32) \
            if b.triangle_materials else None

    @property
    def uniform(self):
        return self.bundle.uniform

    @property
    def camera(self):
        return self.bundle.camera

    @property
    def flags(self):
        return self.bundle.flags

    def set_uniform(self, uniform=None, camera=None, flags=None):
        abi.check(abi.lib().mtp_scene_set_uniform(
            self._handle, C.byref(uniform) if uniform is not None else None,
            C.byref(camera) if camera is not None else None, self.flags if flags is None else flags))
        self.refresh()

    def host_view(self):
        """mtc_scene_view over the host arrays (for the CPU oracle)."""
        b = self.bundle
        v = abi.SceneView()
        v.struct_size = C.sizeof(abi.SceneView)
        v.flags = b.flags
        v.bvh = C.cast(b.bvh, C.c_void_p)
        v.bvh_vec4_count = b.bvh_vec4_count
        v.instances = C.cast(b.instances, C.c_void_p)
        v.instance_count = b.instance_count
        v.material_count = b.material_count
        v.attributes = C.cast(b.attributes, C.c_void_p)
        v.attribute_words = b.attribute_words
        v.vertex_layout = b.vertex_layout
        v.materials = C.cast(b.materials, C.c_void_p)
        v.env_map = C.cast(b.env_map, C.c_void_p) if b.env_width else None
        v.env_distribution = C.cast(b.env_distribution, C.c_void_p) if b.env_width else None
        v.env_width, v.env_height = b.env_width, b.env_height
        v.light_sampling = C.cast(b.light_sampling, C.c_void_p)
        v.light_sampling_texels = b.light_sampling_texels
        v.blas_offset = b.uniform.blas_offset
        v.energy_lut = C.cast(b.energy_lut, C.c_void_p)
        v.analytic_lights = C.cast(b.analytic_lights, C.c_void_p) if b.lights_count else None
        v.tlas_stack_size, v.blas_stack_size = b.tlas_stack_size, b.blas_stack_size
        v.maps = C.cast(b.maps, C.c_void_p) if b.map_count else None
        v.map_texels = C.cast(b.map_texels, C.c_void_p) if b.map_texel_count else None
        v.map_count, v.map_texel_count = b.map_count, b.map_texel_count
        v.triangle_materials = C.cast(b.triangle_materials, C.c_void_p) if b.triangle_materials else None
        return v

    def refit_inputs(self):
        n = self.info.instances
        out = dict(transforms=np.zeros((n, 16), np.float64), local_bounds=np.zeros((n, 6), np.float32),
                   blas_offsets=np.zeros(n, np.int32), blas_layouts=np.zeros(n, np.int32),
                   vertex_offsets=np.zeros(n, np.int32), materials=np.zeros(n, np.int32),
                   colors=np.zeros((n, 3), np.float32))
        abi.check(abi.lib().mtp_scene_refit_inputs(self._handle, *[out[k].ctypes.data for k in
                  ("transforms", "local_bounds", "blas_offsets", "blas_layouts", "vertex_offsets", "materials",
                   "colors")]))
        return out

    def set_transforms(self, transforms):
        t = np.ascontiguousarray(transforms, dtype=np.float64)
        abi.check(abi.lib().mtp_scene_set_transforms(self._handle, t.ctypes.data, t.shape[0]))

    def set_blas_layout(self, layout):
        """Re-encodes every BLAS in layout code 0 (BVH2) or 2 (BVH_GPU: both
        child boxes in the parent node) and refreshes the host arrays."""
        abi.check(abi.lib().mtp_scene_set_blas_layout(self._handle, layout))
        self.refresh()

    def mesh(self, m):
        """Source mesh `m` (the input of BLAS m): (positions (V, 3) f32,
        indices (T, 3) u32, BLAS offset in bvh (vec4), BLAS length (vec4),
        SAH bins)."""
        L = abi.lib()
        u = [C.c_uint32() for _ in range(5)]
        abi.check(L.mtp_scene_mesh(self._handle, m, None, None, *[C.byref(x) for x in u]))
        pos = np.zeros((u[0].value, 3), np.float32)
        idx = np.zeros((u[1].value, 3), np.uint32)
        abi.check(L.mtp_scene_mesh(self._handle, m, pos.ctypes.data, idx.ctypes.data, *[C.byref(x) for x in u]))
        return pos, idx, u[2].value, u[3].value, u[4].value

    def refit_host(self):
        abi.check(abi.lib().mtp_scene_refit_host(self._handle))

    def close(self):
        if getattr(self, "_handle", None):
            abi.lib().mtp_scene_free(self._handle)
            self._handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def make_workload(name, seed=1, width=None, height=None, params=None):
    w = WORKLOADS[name]
    return SceneHost(w["kind"], width or w["width"], height or w["height"], seed,
                     tuple(params) if params is not None else w["params"])


class DeviceScene:
    """Device copy of a SceneHost (torch tensors own the memory)."""

    def __init__(self, host: SceneHost, device="cuda"):
        import torch
        self.host = host
        self.device = torch.device(device)

        def up(a):
            if a.size == 0:
                return None
            return torch.from_numpy(np.ascontiguousarray(a)).to(self.device)

        self.bvh = up(host.bvh)
        self.instances = up(host.instances)
        self.attributes = up(host.attributes.view(np.int32))
        self.materials = up(host.materials)
        self.env_map = up(host.env_map)
        self.env_distribution = up(host.env_distribution)
        self.light_sampling = up(host.light_sampling)
        self.energy_lut = up(host.energy_lut)
        self.lights = up(host.lights)
        self.maps = up(host.maps)
        self.map_texels = up(host.map_texels)
        self.triangle_materials = up(host.triangle_materials) if host.triangle_materials is not None else None
        b = host.bundle
        v = abi.SceneView()
        v.struct_size = C.sizeof(abi.SceneView)
        v.flags = b.flags

        def ptr(t):
            return t.data_ptr() if t is not None else None

        v.bvh = ptr(self.bvh)
        v.bvh_vec4_count = b.bvh_vec4_count
        v.instances = ptr(self.instances)
        v.instance_count = b.instance_count
        v.material_count = b.material_count
        v.attributes = ptr(self.attributes)
        v.attribute_words = b.attribute_words
        v.vertex_layout = b.vertex_layout
        v.materials = ptr(self.materials)
        v.env_map = ptr(self.env_map)
        v.env_distribution = ptr(self.env_distribution)
        v.env_width, v.env_height = b.env_width, b.env_height
        v.light_sampling = ptr(self.light_sampling)
        v.light_sampling_texels = b.light_sampling_texels
        v.blas_offset = b.uniform.blas_offset
        v.energy_lut = ptr(self.energy_lut)
        v.analytic_lights = ptr(self.lights)
        v.tlas_stack_size, v.blas_stack_size = b.tlas_stack_size, b.blas_stack_size
        v.maps, v.map_texels = ptr(self.maps), ptr(self.map_texels)
        v.map_count, v.map_texel_count = b.map_count, b.map_texel_count
        v.triangle_materials = ptr(self.triangle_materials)
        self.view = v
        self.uniform = abi.TraceUniform.from_buffer_copy(b.uniform)
        self.camera = abi.CameraUniform.from_buffer_copy(b.camera)
        self.width, self.height = b.width, b.height

    @property
    def device_bytes(self):
        return sum(t.numel() * t.element_size() for t in (self.bvh, self.instances, self.attributes,
                   self.materials, self.env_map, self.env_distribution, self.light_sampling, self.energy_lut,
                   self.lights, self.maps, self.map_texels, self.triangle_materials) if t is not None)
