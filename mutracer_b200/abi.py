"""ctypes mirror of include/mutracer_b200.h and the loader of the in-tree library.

The library is required: importing a compute entry point without
``_lib/libmutracer_b200.so`` raises, there is no Python or CPU fallback.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("MUTRACER_B200_LIB") or os.path.join(HERE, "_lib", "libmutracer_b200.so")

# Status codes (mutracer-status.h).
MT_OK = 0
MT_ERROR = 1
MT_ERROR_INVALID_ARGUMENT = 2
MT_ERROR_INVALID_HANDLE = 3
MT_ERROR_BUSY = 4
MT_ERROR_INVALID_STATE = 5
MT_ERROR_CANCELLED = 7
MT_ERROR_BUFFER_TOO_SMALL = 8
MT_ERROR_CONTEXT_FAILED = 9
MT_ERROR_UNAVAILABLE = 10
MT_ERROR_TIMEOUT = 11
MT_IMAGE_HDR, MT_IMAGE_NORMAL, MT_IMAGE_ALBEDO = 0, 1, 2
MT_JOB_QUEUED, MT_JOB_RUNNING, MT_JOB_COMPLETE, MT_JOB_CANCELLED, MT_JOB_FAILED, MT_JOB_CANCELLING = range(6)
MT_CONTEXT_EMPTY, MT_CONTEXT_COMMITTED, MT_CONTEXT_FAILED, MT_CONTEXT_JOB_ACTIVE = range(4)
MT_SAMPLING_SOBOL, MT_SAMPLING_ZSOBOL, MT_SAMPLING_RANDOM = 0, 1, 2
MTC_SCENE_HAS_MEDIUM = 1
MTC_SCENE_SPECTRAL = 2
MTC_SCENE_PATTERN_SHIFT = 4
MTC_SCENE_PATTERN_MASK = 0x30
MTC_SCENE_BLAS_GPU_LAYOUT = 0x100
MTC_SCENE_HAS_ALPHA = 0x200
MTC_SCENE_SPECTRAL_INDEPENDENT = 0x400
MTC_FEATURE_USE_ENVMAP = 1
MTC_INSTANCE_VEC4_STRIDE = 10
MTC_MATERIAL_VEC4_ROWS = 26
MTC_MAP_VEC4_ROWS = 3
MTC_LIGHT_VEC4_ROWS = 6
MTC_ENERGY_LUT_WIDTH = 32
MTC_ENERGY_LUT_HEIGHT = 2177
MTC_REGROUP_OFF = 0xFFFFFFFF
MTC_BATCH_NOALLOC_MAX_JOBS = 64
MTC_BATCH_STATUS_GUARD_EXHAUSTED = 1
MT_BACKEND_SOFTWARE = 0
MT_BACKEND_HWRT = 1


class MtError(RuntimeError):
    def __init__(self, status, message=""):
        super().__init__(f"mt_status {status}: {message}")
        self.status = status


class TraceUniform(C.Structure):
    _fields_ = [
        ("output_size", C.c_float * 2), ("sample_count", C.c_float), ("_pad0", C.c_float),
        ("scale_offset", C.c_float * 4), ("lights_count", C.c_int32),
        ("transmissive_output_alpha_min", C.c_float), ("jitter", C.c_float * 2),
        ("background_color", C.c_float * 4), ("grounded_background_params", C.c_float * 4),
        ("grounded_background_center", C.c_float * 2), ("blas_offset", C.c_int32), ("is_empty", C.c_int32),
        ("bevel", C.c_int32), ("dispersion_wavelengths", C.c_int32), ("env_light_pmf", C.c_float),
        ("light_choice_count", C.c_int32), ("light_weight_total", C.c_float),
        ("light_sampling_texture_width", C.c_int32), ("light_choice_texel_offset", C.c_int32),
        ("bounces", C.c_int32), ("variance_moments", C.c_int32), ("adaptive_sampling", C.c_int32),
        ("clamping", C.c_float), ("direct_light_candidates", C.c_int32), ("background_flags", C.c_int32),
        ("loop_unroll_guard", C.c_uint32), ("scene_feature_flags", C.c_uint32), ("sequence_seed", C.c_uint32),
        ("zsobol_log_spp", C.c_uint32), ("sample_sequence_offset", C.c_uint32),
        ("shadow_catcher_choice_offset", C.c_int32), ("shadow_catcher_choice_count", C.c_int32),
        ("environment_rotation", C.c_float * 16), ("background_map_transform", C.c_float * 4),
        ("background_map_rotation", C.c_float * 16),
    ]


class CameraUniform(C.Structure):
    _fields_ = [("view_projection_inv", C.c_float * 16), ("view_inv", C.c_float * 16),
                ("aperture_radius", C.c_float), ("focus_distance", C.c_float), ("_pad", C.c_float * 2)]


class VertexLayout(C.Structure):
    _fields_ = [("stride", C.c_uint32), ("normal_offset", C.c_uint32), ("normal_float", C.c_uint32),
                ("uv_offset", C.c_uint32), ("color_offset", C.c_uint32), ("color_float", C.c_uint32),
                ("uv1_offset", C.c_uint32), ("_pad", C.c_uint32)]


class SceneView(C.Structure):
    _fields_ = [
        ("struct_size", C.c_uint32), ("flags", C.c_uint32),
        ("bvh", C.c_void_p), ("bvh_vec4_count", C.c_uint64),
        ("instances", C.c_void_p), ("instance_count", C.c_uint32), ("material_count", C.c_uint32),
        ("attributes", C.c_void_p), ("attribute_words", C.c_uint64),
        ("vertex_layout", VertexLayout), ("materials", C.c_void_p),
        ("env_map", C.c_void_p), ("env_distribution", C.c_void_p), ("env_width", C.c_uint32),
        ("env_height", C.c_uint32), ("light_sampling", C.c_void_p), ("light_sampling_texels", C.c_uint32),
        ("blas_offset", C.c_int32), ("energy_lut", C.c_void_p), ("analytic_lights", C.c_void_p),
        ("tlas_stack_size", C.c_uint32), ("blas_stack_size", C.c_uint32),
        ("maps", C.c_void_p), ("map_texels", C.c_void_p), ("map_count", C.c_uint32), ("map_texel_count", C.c_uint32),
        ("triangle_materials", C.c_void_p),
    ]


class Outputs(C.Structure):
    _fields_ = [("color", C.c_void_p), ("normal", C.c_void_p), ("albedo", C.c_void_p),
                ("shadow_catcher", C.c_void_p)]


class Hit(C.Structure):
    _fields_ = [("hit", C.c_int32), ("instance", C.c_int32), ("record", C.c_int32), ("t", C.c_float),
                ("barycentric", C.c_float * 3), ("_pad", C.c_float)]


class Counters(C.Structure):
    _fields_ = [("path_samples", C.c_uint64), ("extension_rays", C.c_uint64), ("shadow_rays", C.c_uint64),
                ("kernel_launches", C.c_uint64)]


class JobDesc(C.Structure):
    _fields_ = [("scene", SceneView), ("camera", CameraUniform), ("uniform", TraceUniform),
                ("out", Outputs), ("samples", C.c_uint32), ("_pad", C.c_uint32 * 3)]


class BatchConfig(C.Structure):
    _fields_ = [("struct_size", C.c_uint32), ("block_threads", C.c_uint32), ("tile_width", C.c_uint32),
                ("ctas_per_sm", C.c_uint32), ("items_per_fetch", C.c_uint32), ("_pad", C.c_uint32 * 3)]

    @classmethod
    def make(cls, block_threads=0, tile_width=0, ctas_per_sm=0, items_per_fetch=0):
        c = cls()
        c.struct_size = C.sizeof(cls)
        c.block_threads, c.tile_width, c.ctas_per_sm, c.items_per_fetch = (block_threads, tile_width, ctas_per_sm,
                                                                          items_per_fetch)
        return c


class StreamConfig(C.Structure):
    _fields_ = [("struct_size", C.c_uint32), ("slots", C.c_uint32), ("iterations_per_check", C.c_uint32),
                ("max_iterations", C.c_uint32), ("refill_lanes", C.c_uint32), ("regroup_interval", C.c_uint32),
                ("sort_rays", C.c_uint32), ("steps_per_check", C.c_uint32),
                ("traversal_ctas_per_sm", C.c_uint32), ("_pad", C.c_uint32 * 3)]

    @classmethod
    def make(cls, slots=0, iterations_per_check=0, max_iterations=0, refill_lanes=0, regroup_interval=0,
             sort_rays=0, steps_per_check=0, traversal_ctas_per_sm=0):
        c = cls()
        c.struct_size = C.sizeof(cls)
        c.slots, c.iterations_per_check, c.max_iterations = slots, iterations_per_check, max_iterations
        c.refill_lanes, c.regroup_interval, c.sort_rays = refill_lanes, regroup_interval, sort_rays
        c.steps_per_check, c.traversal_ctas_per_sm = steps_per_check, traversal_ctas_per_sm
        return c


class BlasBuildInput(C.Structure):
    _fields_ = [("struct_size", C.c_uint32), ("bins", C.c_uint32), ("positions", C.c_void_p),
                ("indices", C.c_void_p), ("vertex_count", C.c_uint32), ("triangle_count", C.c_uint32)]


class BlasBuildResult(C.Structure):
    _fields_ = [("struct_size", C.c_uint32), ("vec4_count", C.c_uint32), ("max_depth", C.c_uint32),
                ("max_leaf_primitives", C.c_uint32), ("node_count", C.c_uint32), ("primitive_count", C.c_uint32),
                ("local_bounds", C.c_float * 6), ("host_syncs", C.c_uint32), ("_pad", C.c_uint32 * 3)]


class BlasRefitPlanInfo(C.Structure):
    _fields_ = [("struct_size", C.c_uint32), ("node_count", C.c_uint32), ("levels", C.c_uint32),
                ("_pad", C.c_uint32 * 5)]


class SceneBundle(C.Structure):
    _fields_ = [
        ("struct_size", C.c_uint32), ("width", C.c_uint32), ("height", C.c_uint32), ("flags", C.c_uint32),
        ("bvh", C.POINTER(C.c_float)), ("bvh_vec4_count", C.c_uint64),
        ("instances", C.POINTER(C.c_float)), ("instance_count", C.c_uint32), ("material_count", C.c_uint32),
        ("attributes", C.POINTER(C.c_uint32)), ("attribute_words", C.c_uint64),
        ("vertex_layout", VertexLayout), ("materials", C.POINTER(C.c_float)),
        ("env_map", C.POINTER(C.c_float)), ("env_width", C.c_uint32), ("env_height", C.c_uint32),
        ("env_distribution", C.POINTER(C.c_float)),
        ("light_sampling", C.POINTER(C.c_float)), ("light_sampling_texels", C.c_uint32),
        ("lights_count", C.c_uint32), ("energy_lut", C.POINTER(C.c_float)),
        ("analytic_lights", C.POINTER(C.c_float)),
        ("tlas_stack_size", C.c_uint32), ("blas_stack_size", C.c_uint32),
        ("camera", CameraUniform), ("uniform", TraceUniform),
        ("maps", C.POINTER(C.c_float)), ("map_count", C.c_uint32),
        ("map_texels", C.POINTER(C.c_float)), ("map_texel_count", C.c_uint64),
        ("triangle_materials", C.POINTER(C.c_uint32)),
    ]


class RenderSettings(C.Structure):
    _fields_ = [("struct_size", C.c_uint32), ("sampling_pattern", C.c_uint32), ("seed", C.c_uint32),
                ("max_samples", C.c_uint32), ("bounces", C.c_uint32), ("direct_light_candidates", C.c_uint32),
                ("bevel_samples", C.c_uint32), ("sample_sequence_offset", C.c_uint32),
                ("clamping", C.c_double), ("transmissive_output_alpha_min", C.c_double),
                ("caustic_flags", C.c_uint32), ("light_photons", C.c_uint32), ("photon_map_photons", C.c_uint32),
                ("photon_map_radius", C.c_float)]


class ContextSnapshot(C.Structure):
    _fields_ = [("struct_size", C.c_uint32), ("width", C.c_uint32), ("height", C.c_uint32),
                ("samples", C.c_uint32), ("state", C.c_uint32), ("last_commit", C.c_uint32)]


class JobSnapshot(C.Structure):
    _fields_ = [("struct_size", C.c_uint32), ("state", C.c_uint32), ("requested_samples", C.c_uint32),
                ("submitted_samples", C.c_uint32), ("completed_samples", C.c_uint32),
                ("base_samples", C.c_uint32)]


class SceneInfo(C.Structure):
    _fields_ = [("triangles", C.c_uint64), ("unique_triangles", C.c_uint64), ("instances", C.c_uint32),
                ("blases", C.c_uint32), ("tlas_vec4", C.c_uint32), ("_pad", C.c_uint32),
                ("bvh_vec4", C.c_uint64), ("vertices", C.c_uint64), ("world_bounds", C.c_float * 6),
                ("_pad2", C.c_float * 2)]


STRUCT_ORDER = [TraceUniform, CameraUniform, SceneView, Outputs, Hit, Counters, JobDesc, BatchConfig,
                SceneBundle, RenderSettings, ContextSnapshot, JobSnapshot, SceneInfo, StreamConfig, BlasBuildInput,
                BlasBuildResult, BlasRefitPlanInfo]

_lib = None


def _declare(lib):
    P = C.c_void_p
    sigs = {
        "mtc_abi_version": (C.c_uint32, []),
        "mtc_struct_sizes": (C.c_int, [C.POINTER(C.c_uint32), C.c_uint32]),
        "mtc_trace_samples": (C.c_int32, [C.POINTER(SceneView), C.POINTER(CameraUniform), C.POINTER(TraceUniform),
                                          C.POINTER(Outputs), C.c_uint32, P, P]),
        "mtc_query_first_hit": (C.c_int32, [C.POINTER(SceneView), P, C.c_uint32, P, P]),
        "mtc_sample_maps": (C.c_int32, [C.POINTER(SceneView), P, P, C.c_uint32, P, P]),
        "mtc_batch_scratch_bytes": (C.c_size_t, [C.c_uint32]),
        "mtc_trace_batch": (C.c_int32, [C.POINTER(JobDesc), C.c_uint32, C.POINTER(BatchConfig), P, P, P, P]),
        "mtc_batch_table_bytes": (C.c_size_t, [C.c_uint32]),
        "mtc_average_output": (C.c_int32, [P, C.c_uint32, C.c_uint32, P, P, P]),
        "mtc_stream_state_bytes": (C.c_size_t, [C.c_uint32, C.POINTER(StreamConfig)]),
        "mtc_stream_run": (C.c_int32, [P, C.c_uint32, C.POINTER(StreamConfig), P, P, P]),
        "mtc_stream_launch": (C.c_int32, [P, C.c_uint32, C.POINTER(StreamConfig), P, P, P]),
        "mtc_stream_status": (C.c_int32, [P, C.c_uint32, C.POINTER(StreamConfig), P]),
        "mtc_batch_prepare": (C.c_int32, [C.POINTER(JobDesc), C.c_uint32, C.POINTER(BatchConfig), P,
                                           C.POINTER(C.c_uint32)]),
        "mtc_batch_launch": (C.c_int32, [P, C.c_uint32, C.POINTER(BatchConfig), P, P, P]),
        "mtc_trace_batch_noalloc": (C.c_int32, [C.POINTER(JobDesc), C.c_uint32, C.POINTER(BatchConfig), P, P, P]),
        "mtc_refit_tlas": (C.c_int32, [P, C.c_uint64, P, C.c_uint32, P, P, P, P, P, P, P, P]),
        "mtc_blas_build_scratch_bytes": (C.c_uint64, [C.c_uint32, C.c_uint32]),
        "mtc_blas_build_max_vec4": (C.c_uint64, [C.c_uint32]),
        "mtc_build_blas": (C.c_int32, [C.POINTER(BlasBuildInput), P, C.c_uint64, P, C.c_uint64,
                                        C.POINTER(BlasBuildResult), P]),
        "mtp_scene_make": (P, [C.c_char_p, C.c_uint32, C.c_uint32, C.c_uint64, C.POINTER(C.c_uint32), C.c_uint32]),
        "mtp_scene_free": (None, [P]),
        "mtp_scene_bundle": (C.c_int, [P, C.POINTER(SceneBundle)]),
        "mtp_scene_info": (C.c_int, [P, C.POINTER(SceneInfo)]),
        "mtp_scene_set_uniform": (C.c_int, [P, C.POINTER(TraceUniform), C.POINTER(CameraUniform), C.c_uint32]),
        "mtp_scene_refit_inputs": (C.c_int, [P, P, P, P, P, P, P, P]),
        "mtp_scene_set_transforms": (C.c_int, [P, P, C.c_uint32]),
        "mtp_scene_refit_host": (C.c_int, [P]),
        "mtp_scene_set_blas_layout": (C.c_int, [P, C.c_uint32]),
        "mtp_scene_mesh": (C.c_int, [P, C.c_uint32, P, P, P, P, P, P, P]),
        "mtp_build_binned_sah": (C.c_int, [P, C.c_uint32, C.c_int, P, P, P, P, P]),
        "mtp_build_blas": (C.c_int, [P, C.c_uint32, P, C.c_uint32, C.c_int, P, C.c_uint64, P, P]),
        "mtp_energy_lut": (C.c_int, [P]),
        "mtp_light_alias_table": (C.c_int, [P, C.c_uint32, P, P, C.POINTER(C.c_double)]),
        "mtp_light_power": (C.c_double, [C.c_int, P, C.c_float, C.c_float, C.c_float]),
        "mtp_refit_blas": (C.c_int, [P, C.c_uint64, P, C.c_uint32, C.POINTER(C.c_double)]),
        "mtc_blas_refit_plan_bytes": (C.c_uint64, [C.c_uint64]),
        "mtc_blas_refit_prepare": (C.c_int32, [P, C.c_uint64, P, C.c_uint64, C.POINTER(BlasRefitPlanInfo), P]),
        "mtc_refit_blas": (C.c_int32, [P, C.c_uint64, P, C.c_uint32, P, C.c_uint32, P, P]),
        "mtp_camera_look_at": (C.c_int, [C.c_uint32, C.c_uint32, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                         C.POINTER(C.c_double), C.c_double, C.POINTER(CameraUniform)]),
        "mtp_env_distribution": (C.c_int, [P, C.c_uint32, C.c_uint32, P, P]),
        "mt_render_settings_default": (C.c_int32, [C.POINTER(RenderSettings)]),
        "mt_context_create": (C.c_int32, [C.POINTER(C.c_uint64), C.c_char_p, C.c_size_t]),
        "mt_context_create_with_backend": (C.c_int32, [C.c_uint32, C.POINTER(C.c_uint64), C.c_char_p, C.c_size_t]),
        "mt_context_backend": (C.c_int32, [C.c_uint64, C.POINTER(C.c_uint32), C.c_char_p, C.c_size_t, C.c_char_p,
                                           C.c_size_t]),
        "mt_context_cancel_commit": (C.c_int32, [C.c_uint64, C.c_char_p, C.c_size_t]),
        "mt_probe_render_scene": (C.c_int32, [P, C.c_size_t, C.c_char_p, C.c_uint32, C.c_char_p, C.c_size_t]),
        "mt_context_destroy": (C.c_int32, [C.c_uint64, C.c_char_p, C.c_size_t]),
        "mt_context_commit_bundle": (C.c_int32, [C.c_uint64, C.POINTER(SceneBundle), C.POINTER(RenderSettings),
                                                 C.c_char_p, C.c_size_t]),
        "mt_context_commit": (C.c_int32, [C.c_uint64, P, C.c_size_t, C.c_char_p, C.c_size_t]),
        "mt_context_commit_with_settings": (C.c_int32, [C.c_uint64, P, C.c_size_t, C.POINTER(RenderSettings),
                                                        C.c_char_p, C.c_size_t]),
        "mtp_descriptor_decode": (P, [P, C.c_size_t, C.POINTER(C.c_int32), C.c_char_p, C.c_size_t]),
        "mt_context_render": (C.c_int32, [C.c_uint64, C.c_uint32, C.c_char_p, C.c_size_t]),
        "mt_context_reset": (C.c_int32, [C.c_uint64, C.c_char_p, C.c_size_t]),
        "mt_context_wait": (C.c_int32, [C.c_uint64, C.c_uint32, C.c_char_p, C.c_size_t]),
        "mt_context_info": (C.c_int32, [C.c_uint64, C.POINTER(ContextSnapshot), C.c_char_p, C.c_size_t]),
        "mt_context_read_pixels": (C.c_int32, [C.c_uint64, C.c_uint32, P, C.c_size_t, C.POINTER(C.c_size_t),
                                               C.c_char_p, C.c_size_t]),
        "mt_context_submit": (C.c_int32, [C.c_uint64, C.c_uint32, C.POINTER(C.c_uint64), C.c_char_p, C.c_size_t]),
        "mt_job_poll": (C.c_int32, [C.c_uint64, C.c_uint32, C.c_char_p, C.c_size_t]),
        "mt_job_info": (C.c_int32, [C.c_uint64, C.POINTER(JobSnapshot), C.c_char_p, C.c_size_t]),
        "mt_job_cancel": (C.c_int32, [C.c_uint64, C.c_char_p, C.c_size_t]),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args


def lib():
    """The loaded libmutracer_b200.so; raises if it was not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: run `python -m mutracer_b200.build` (no fallback exists)")
        handle = C.CDLL(LIB_PATH)
        _declare(handle)
        sizes = (C.c_uint32 * 32)()
        n = handle.mtc_struct_sizes(sizes, 32)
        for i, cls in enumerate(STRUCT_ORDER[:n]):
            if C.sizeof(cls) != sizes[i]:
                raise RuntimeError(f"ABI mismatch for {cls.__name__}: {C.sizeof(cls)} != {sizes[i]}")
        _lib = handle
    return _lib


def check(status, err=None):
    if status != MT_OK:
        raise MtError(status, err.value.decode(errors="replace") if err is not None else "")
    return status
