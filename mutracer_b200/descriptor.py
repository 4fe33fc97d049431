"""Scene descriptor v8 writer: the byte buffer mt_context_commit takes
(native/docs/scene-format.md; records of native/include/mutracer-scene.h,
word offsets of native/include/mutracer-layout.h).  The record defaults are
those of mutracer-scene-builder.h (mt_material_v4_default,
mt_camera_v4_default, mt_texture_v4_default), and like that builder this
appends arrays first, then the record tables, and fills the header last.
"""
import ctypes as C
import math

import numpy as np

from . import abi

VERSION = 8
NO_TEXTURE = 0xFFFFFFFF
ORDINARY_MESH = 0xFFFFFFFF
LIGHT_RECT, LIGHT_SPHERE, LIGHT_DIRECTIONAL, LIGHT_SPOT, LIGHT_DISK, LIGHT_CYLINDER = range(6)
QUALITY_BEVEL, QUALITY_DISPERSION, QUALITY_HIDE_BACKGROUND = 1, 2, 4
IDENTITY = (1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1)


def look_at(eye, target):
    """mt_scene_look_at: camera-to-world matrix whose -Z axis points from eye
    to target, +Y up (f32 arithmetic)."""
    f = np.float32
    eye = np.asarray(eye, f)
    z = eye - np.asarray(target, f)
    z = (z / f(math.sqrt(float(np.dot(z, z))))).astype(f)
    x = np.array([z[2], 0, -z[0]], f)
    x = (x / f(math.sqrt(float(x[0] * x[0] + x[2] * x[2])))).astype(f)
    y = np.array([z[1] * x[2] - z[2] * x[1], z[2] * x[0] - z[0] * x[2], z[0] * x[1] - z[1] * x[0]], f)
    m = list(IDENTITY)
    for k in range(3):
        m[k], m[4 + k], m[8 + k], m[12 + k] = float(x[k]), float(y[k]), float(z[k]), float(eye[k])
    return m


def translate(t, scale=1.0):
    return [scale, 0, 0, 0, 0, scale, 0, 0, 0, 0, scale, 0, t[0], t[1], t[2], 1]


class Descriptor:
    def __init__(self, width, height, version=VERSION):
        self.width, self.height, self.version = width, height, version
        self.words = [0] * 32
        self.geometries, self.meshes, self.materials, self.lights, self.textures = [], [], [], [], []
        self.batches = None
        self.camera = self.camera_record()
        self.background = (0.0, 0.0, 0.0, 1.0)
        self.environment = 0
        self.quality = 0
        self.env_settings = None
        self.extra_header = {}

    # ------------------------------------------------------------- arrays
    def append(self, values, dtype=np.float32):
        """Appends an array of 32-bit words; returns its word offset."""
        arr = np.ascontiguousarray(values, dtype=dtype).reshape(-1)
        off = len(self.words)
        self.words.extend(arr.view(np.uint32).tolist())
        return off

    @staticmethod
    def _f(x):
        return int(np.array([x], np.float32).view(np.uint32)[0])

    # ------------------------------------------------------------ records
    def add_geometry(self, positions, indices, normals=None, material_indices=None, uvs=None, colors=None,
                     uv1s=None):
        pos = np.asarray(positions, np.float32).reshape(-1, 3)
        idx = np.asarray(indices, np.uint32).reshape(-1)
        rec = [len(pos), len(idx), self.append(pos), self.append(idx, np.uint32),
               self.append(normals) if normals is not None else 0,
               self.append(uvs) if uvs is not None else 0,
               self.append(uv1s) if uv1s is not None else 0,
               self.append(colors) if colors is not None else 0, 0,
               self.append(material_indices, np.uint32) if material_indices is not None else 0, 0, 0]
        self.geometries.append(rec)
        return len(self.geometries) - 1

    def add_material(self, base_color=(0.8, 0.8, 0.8), roughness=0.3, metalness=0.0, transmission=0.0, ior=1.5,
                     emission_color=(1, 1, 1), emission_luminance=0.0, coat_weight=0.0, coat_roughness=0.0,
                     opacity=1.0, thin_walled=False, textures=(NO_TEXTURE,) * 4, extensions=()):
        """textures: (map, normal map, metallic-roughness map, emissive map)
        texture indices or NO_TEXTURE.  extensions: (id, (x, y, z)) floats,
        or (id, int) for bool / enum / texture ids."""
        ext_off = 0
        if extensions:
            words = []
            for eid, value in extensions:
                if isinstance(value, (tuple, list)):
                    vals = [self._f(v) for v in value] + [0] * (3 - len(value))
                else:
                    vals = [int(value) & 0xFFFFFFFF, 0, 0]
                words += [eid] + vals
            ext_off = self.append(words, np.uint32)
        f = self._f
        rec = [f(c) for c in base_color] + [f(roughness), f(metalness), f(transmission), f(ior)] + \
              [f(c) for c in emission_color] + [f(emission_luminance), f(coat_weight), f(coat_roughness),
                                                f(opacity), int(thin_walled)] + list(textures) + \
              [len(extensions), ext_off, 0, 0, 0]
        self.materials.append(rec)
        return len(self.materials) - 1

    def add_mesh(self, geometry, material=0, transform=IDENTITY, hidden=False, material_table=None, batch=None):
        """batch: None (ordinary), or (transforms (n, 16), colors (n, 3) or None)."""
        table_off, table_n = 0, 0
        if material_table is not None:
            table_off, table_n = self.append(material_table, np.uint32), len(material_table)
        f = self._f
        rec = [geometry, material, table_off, table_n] + [f(v) for v in transform] + [int(hidden)]
        self.meshes.append(rec)
        if batch is not None and self.batches is None:
            self.batches = [[ORDINARY_MESH, 0, 0, 0] for _ in range(len(self.meshes) - 1)]
        if self.batches is not None:
            if batch is None:
                self.batches.append([ORDINARY_MESH, 0, 0, 0])
            else:
                transforms, colors = batch
                transforms = np.asarray(transforms, np.float32).reshape(-1, 16)
                self.batches.append([len(transforms), self.append(transforms) if len(transforms) else 0,
                                     self.append(colors) if colors is not None and len(transforms) else 0, 0])
        return len(self.meshes) - 1

    def add_light(self, kind, color=(1, 1, 1), intensity=1.0, size=1.0, height_or_inner=1.0, spread_or_outer=1.0,
                  transform=IDENTITY, radius=0.0, length=0.0, normalize=False):
        f = self._f
        rec = [kind] + [f(c) for c in color] + [f(intensity), f(size), f(height_or_inner), f(spread_or_outer),
                                                0, 0, 0, 0] + [f(v) for v in transform]
        if self.version >= 6:
            rec += [f(radius), f(length), int(normalize), 0]
        self.lights.append(rec)
        return len(self.lights) - 1

    def add_texture_rgba32f(self, width, height, pixels, **kw):
        return self.add_texture(width, height, np.asarray(pixels, np.float32), storage=1, **kw)

    def add_texture(self, width, height, pixels, storage=0, flip_y=False, uv_channel=0, uv_scale=(1, 1),
                    uv_offset=(0, 0), wrap_s=0, wrap_t=0, udim=0, pixels_offset=None):
        """storage 0: RGBA8, `pixels` (h, w, 4) uint8 packed one word per
        texel (R in the low byte); storage 1: RGBA32F floats.  `pixels_offset`
        reuses the pixel words of an earlier texture (shared source)."""
        if pixels_offset is not None:
            off = pixels_offset
        elif storage == 0:
            off = self.append(np.ascontiguousarray(pixels, np.uint8).reshape(-1).view(np.uint32), np.uint32)
        else:
            off = self.append(np.asarray(pixels, np.float32).reshape(-1))
        f = self._f
        rec = [width, height, storage, off, int(flip_y), uv_channel, f(uv_scale[0]), f(uv_scale[1]),
               f(uv_offset[0]), f(uv_offset[1]), wrap_s, wrap_t]
        if self.version >= 7:
            rec.append(udim)
        self.textures.append(rec)
        return len(self.textures) - 1

    def texture_pixels_offset(self, texture):
        return self.textures[texture][3]

    def camera_record(self, projection=0, fov=45.0, near=0.1, far=1000.0, left=-1.0, right=1.0, bottom=-1.0,
                      top=1.0, zoom=1.0, f_stop=0.0, focus_distance=10.0, sensor_height=24.0, meters_per_unit=1.0,
                      transform=IDENTITY):
        f = self._f
        return [projection] + [f(v) for v in (fov, near, far, left, right, bottom, top, zoom, f_stop, focus_distance,
                                              sensor_height, meters_per_unit)] + [0, 0, 0] + [f(v) for v in transform]

    def set_camera(self, **kw):
        self.camera = self.camera_record(**kw)

    def set_environment(self, texture, intensity=1.0, yaw=0.0, background_intensity=1.0, background_yaw=0.0):
        self.environment = texture + 1
        self.env_settings = (intensity, yaw, background_intensity, background_yaw)

    # -------------------------------------------------------------- bytes
    def to_bytes(self):
        w = list(self.words)
        header = [0] * 32
        header[0], header[2], header[3] = self.version, self.width, self.height
        header[4:9] = [len(self.geometries), len(self.meshes), len(self.materials), len(self.lights),
                       len(self.textures)]

        def table(records):
            off = len(w)
            for r in records:
                w.extend(r)
            return off
        header[9] = table(self.geometries)
        header[10] = table(self.meshes)
        header[11] = table(self.materials)
        header[12] = table(self.lights)
        header[13] = table(self.textures)
        header[14] = table([self.camera])
        header[16:20] = [self._f(c) for c in self.background]
        header[20] = self.environment
        header[22] = self.quality
        if self.batches is not None:
            header[23] = table(self.batches)
        if self.env_settings is not None:
            header[26] = len(w)
            w.extend(np.asarray(self.env_settings, np.float32).view(np.uint32).tolist())
        for k, v in self.extra_header.items():
            header[k] = v
        header[1] = len(w)
        w[:32] = header
        return np.array(w, np.uint32).tobytes()


def decode(data):
    """mtp_descriptor_decode: (status, message, SceneHost or None)."""
    from . import scene
    buf = np.frombuffer(bytes(data), np.uint8)
    status = C.c_int32()
    err = C.create_string_buffer(512)
    handle = abi.lib().mtp_descriptor_decode(buf.ctypes.data if buf.size else None, buf.size, C.byref(status), err,
                                             512)
    if not handle:
        return status.value, err.value.decode(), None
    return status.value, "", scene.SceneHost.from_handle(handle)
