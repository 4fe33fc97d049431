/*
 * mutracer_b200 — B200-native progressive path-tracing megakernel behind the
 * MuTracer buffer contract and C ABI.
 *
 * Two layers are exported, both plain C (no CUDA or torch types in any
 * signature; device memory is passed as plain pointers, streams as void*):
 *
 *  1. mtc_*  — kernel-level entry points on caller-owned DEVICE buffers.  They
 *     replace the reference's per-sample compute dispatch of the WGSL megakernel
 *     (native/host/src/lib.rs:1466-1600 `dispatch_target`,
 *     src/renderer/WGPURayTracePass.ts:1935-1939 `dispatchWorkgroups`) and read
 *     exactly the bind-group buffers declared in
 *     src/renderer/wgsl/chunks/rayTraceCore.wgsl.ts:320-338,383-386 and
 *     src/renderer/wgsl/rayTrace.compute.ts:294-299.
 *
 *  2. mt_context_* / mt_job_* — the persistent host API of
 *     native/include/mutracer-context.h:57-187 with the status codes of
 *     native/include/mutracer-status.h:15-45.  commit / commit_with_settings
 *     take the scene descriptor v8 (the features this build renders; others
 *     are refused by name); commit_bundle takes the flattened buffers.
 *
 * All entry points return an mt_status (0 = MT_OK).  Functions that take
 * `char *error, size_t capacity` write a truncated NUL-terminated message.
 */
#ifndef MUTRACER_B200_H
#define MUTRACER_B200_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ status */
/* Same values as native/include/mutracer-status.h:15-45. */
typedef int32_t mt_status;
enum {
  MT_OK = 0,
  MT_ERROR = 1,
  MT_ERROR_INVALID_ARGUMENT = 2,
  MT_ERROR_INVALID_HANDLE = 3,
  MT_ERROR_BUSY = 4,
  MT_ERROR_INVALID_STATE = 5,
  MT_ERROR_FULL_COMMIT_REQUIRED = 6,
  MT_ERROR_CANCELLED = 7,
  MT_ERROR_BUFFER_TOO_SMALL = 8,
  MT_ERROR_CONTEXT_FAILED = 9,
  MT_ERROR_UNAVAILABLE = 10,
  MT_ERROR_TIMEOUT = 11
};
/* mutracer-status.h mt_image_kind subset served by read_pixels. */
enum { MT_IMAGE_HDR = 0, MT_IMAGE_NORMAL = 1, MT_IMAGE_ALBEDO = 2 };
/* mutracer-status.h mt_context_state / mt_job_state / mt_sampling_pattern. */
enum { MT_CONTEXT_EMPTY = 0, MT_CONTEXT_COMMITTED = 1, MT_CONTEXT_FAILED = 2,
       MT_CONTEXT_JOB_ACTIVE = 3 };
enum { MT_COMMIT_NONE = 0, MT_COMMIT_FULL = 1, MT_COMMIT_INCREMENTAL = 2 };
enum { MT_JOB_QUEUED = 0, MT_JOB_RUNNING = 1, MT_JOB_COMPLETE = 2,
       MT_JOB_CANCELLED = 3, MT_JOB_FAILED = 4, MT_JOB_CANCELLING = 5 };
enum { MT_SAMPLING_SOBOL = 0, MT_SAMPLING_ZSOBOL = 1, MT_SAMPLING_RANDOM = 2 };

/* ------------------------------------------------------- buffer contract */
/* Light / choice / material constants: src/renderer/lightConstants.ts:1-15. */
enum { MTC_LIGHT_DIRECTIONAL = 1, MTC_LIGHT_SPHERE = 2, MTC_LIGHT_RECT = 3,
       MTC_LIGHT_SPOT = 4, MTC_LIGHT_DISK = 5, MTC_LIGHT_CYLINDER = 6 };
enum { MTC_CHOICE_ENVIRONMENT = 1, MTC_CHOICE_ANALYTIC = 2,
       MTC_CHOICE_EMISSIVE_TRIANGLE = 3 };
/* Scene feature bits of RayTraceUniform.sceneFeatureFlags
 * (src/renderer/WGPUSceneFeatures.ts:4-12). */
enum { MTC_FEATURE_USE_ENVMAP = 1u, MTC_FEATURE_HAS_THIN_FILM = 1u << 10,
       MTC_FEATURE_HAS_COAT = 1u << 11, MTC_FEATURE_HAS_FUZZ = 1u << 12,
       MTC_FEATURE_HAS_SUBSURFACE = 1u << 13,
       MTC_FEATURE_HAS_SHADOW_CATCHER = 1u << 14 };
/* backgroundFlags bits (rayTrace.compute.ts:1268-1276). */
enum { MTC_BACKGROUND_COLOR = 1, MTC_BACKGROUND_MAP = 2, MTC_BACKGROUND_GROUNDED = 4 };

#define MTC_INSTANCE_VEC4_STRIDE 10   /* bvhAccel.ts:16 */
#define MTC_MATERIAL_VEC4_ROWS 26     /* materialLayoutSchema.ts:23-150 */
#define MTC_LIGHT_VEC4_ROWS 6         /* wgpuSceneUniform.ts:11 PIXELS_PER_LIGHT */
#define MTC_ENERGY_LUT_WIDTH 32       /* decodeOpenPbrEnergyLut.ts:20-33 */
#define MTC_ENERGY_LUT_HEIGHT 2177
#define MTC_MAX_STACK 64              /* bvhAccel.ts:80 MAX_TRAVERSAL_STACK_SIZE */

/* RayTraceUniform, byte-identical to the WGSL struct of
 * rayTraceCore.wgsl.ts:281-318 as written by wgpuSceneUniform.ts:13-55
 * (320 bytes, offsets in comments). */
typedef struct mtc_trace_uniform {
  float output_size[2];                 /*   0 */
  float sample_count;                   /*   8 */
  float _pad0;                          /*  12 */
  float scale_offset[4];                /*  16 */
  int32_t lights_count;                 /*  32 */
  float transmissive_output_alpha_min;  /*  36 */
  float jitter[2];                      /*  40 */
  float background_color[4];            /*  48 */
  float grounded_background_params[4];  /*  64 */
  float grounded_background_center[2];  /*  80 */
  int32_t blas_offset;                  /*  88 */
  int32_t is_empty;                     /*  92 */
  int32_t bevel;                        /*  96 */
  int32_t dispersion_wavelengths;       /* 100 */
  float env_light_pmf;                  /* 104 */
  int32_t light_choice_count;           /* 108 */
  float light_weight_total;             /* 112 */
  int32_t light_sampling_texture_width; /* 116 */
  int32_t light_choice_texel_offset;    /* 120 */
  int32_t bounces;                      /* 124 */
  int32_t variance_moments;             /* 128 */
  int32_t adaptive_sampling;            /* 132 */
  float clamping;                       /* 136 */
  int32_t direct_light_candidates;      /* 140 */
  int32_t background_flags;             /* 144 */
  uint32_t loop_unroll_guard;           /* 148 */
  uint32_t scene_feature_flags;         /* 152 */
  uint32_t sequence_seed;               /* 156 */
  uint32_t zsobol_log_spp;              /* 160 */
  uint32_t sample_sequence_offset;      /* 164 */
  int32_t shadow_catcher_choice_offset; /* 168 */
  int32_t shadow_catcher_choice_count;  /* 172 */
  float environment_rotation[16];       /* 176 */
  float background_map_transform[4];    /* 240 */
  float background_map_rotation[16];    /* 256 */
} mtc_trace_uniform;                    /* 320 */

/* CameraUniform, rayTraceCore.wgsl.ts:274-279 (column-major mat4). */
typedef struct mtc_camera_uniform {
  float view_projection_inv[16];
  float view_inv[16];
  float aperture_radius;
  float focus_distance;
  float _pad[2];
} mtc_camera_uniform;

/* Compact vertex layout of attrBuffers (src/renderer/compactVertices.ts:7-28):
 * u32 words, position f32x3 at word 0, normal at normal_offset (oct-encoded
 * u32, or f32x3 when normal_float != 0), the primary UV set (f32x2) at
 * uv_offset when nonzero (UV_OFF; 0 = no UVs), the secondary UV set at
 * uv1_offset when nonzero (UV1_OFF; 0 = the primary set), the vertex color at
 * color_offset when nonzero (COLOR_OFF: RGBA8 in one word, or f32x3 when
 * color_float != 0; 0 = white).  Tangent words may be present in the stride
 * and are not read. */
typedef struct mtc_vertex_layout {
  uint32_t stride;
  uint32_t normal_offset;
  uint32_t normal_float;
  uint32_t uv_offset;
  uint32_t color_offset;
  uint32_t color_float;
  uint32_t uv1_offset;
  uint32_t _pad;
} mtc_vertex_layout;

/* Device-side view of the bind groups (all pointers are device pointers). */
typedef struct mtc_scene_view {
  uint32_t struct_size;
  uint32_t flags;                  /* MTC_SCENE_* below */
  /* G0 */
  const void *bvh;                 /* binding 0: vec4f[], TLAS at 0, BLASes after blas_offset */
  uint64_t bvh_vec4_count;
  const void *instances;           /* binding 1: vec4f[10 * instance_count] */
  uint32_t instance_count;
  uint32_t material_count;
  const void *attributes;          /* binding 2: u32 words */
  uint64_t attribute_words;
  mtc_vertex_layout vertex_layout;
  const void *materials;           /* binding 3: vec4f[26 * material_count] */
  /* G1 */
  const void *env_map;             /* binding 4: RGBA32F env_width x env_height */
  const void *env_distribution;    /* binding 5: RG32F (env_width+2) x (env_height+1) */
  uint32_t env_width, env_height;
  const void *light_sampling;      /* binding 8: RGBA32F, width in the uniform */
  uint32_t light_sampling_texels;
  int32_t blas_offset;             /* vec4 index of the first BLAS (RayTraceUniform.blasOffset) */
  const void *energy_lut;          /* binding 9: R32F 32 x 2177 */
  /* G2 */
  const void *analytic_lights;     /* binding 2: vec4f[6 * lights_count] */
  uint32_t tlas_stack_size;        /* TLAS_STACK_SIZE (1..64) */
  uint32_t blas_stack_size;        /* BLAS_STACK_SIZE (1..64) */
  /* Material maps (the map / mapInfo bindings of materialBuffer.wgsl.ts
   * :258-335 with independent textures): MTC_MAP_VEC4_ROWS vec4 per map
   * (see mtc_map_record below), texels as RGBA f32 vec4, row 0 at v = 0. */
  const void *maps;
  const void *map_texels;
  uint32_t map_count;
  uint32_t map_texel_count;        /* texels in map_texels (a map reaching past it samples zero) */
  /* Triangle material plane (triangleMaterial, vertexAttributes.wgsl.ts:51-56;
   * packTriangleMaterials, compactVertices.ts:93-102): one u32 per bvh vec4,
   * material index + 1 of the triangle whose record sits at that vec4, 0 for
   * the instance's material.  NULL: every triangle uses its instance's. */
  const uint32_t *triangle_materials;
} mtc_scene_view;
/* One material map, 3 vec4 (f32 words; integers as their bit patterns):
 *   [0] width (u32), height (u32), first texel (u32), 0
 *   [1] UV scale xy, UV offset xy (mapTransform)
 *   [2] UV set (0 / 1), color linear (1: data or float map, no sRGB decode),
 *       wrap S, wrap T (0 repeat, 1 clamp to edge, 2 mirrored repeat)
 * Texels are the decoded RGBA of the stored image (RGBA8 / 255, or the
 * float image rounded to f16 as the reference's RGBA16F storage keeps it),
 * rows flipped when the texture is. */
#define MTC_MAP_VEC4_ROWS 3
/* flags: shader specialisation constants that are not in the uniform
 * (HAS_MEDIUM, SPECTRAL, HAS_ALPHA and SAMPLING_PATTERN of
 * wgpuMaterialConstants.ts:40-70).  HAS_ALPHA (some material's resolved alpha
 * mode is mask or blend) turns on the shadow rays' alpha test
 * (intersectionAlpha.wgsl.ts) and the RGB integrator that splits a partly
 * covered primary hit into a back and a front path (rayTrace.compute.ts
 * :815-890); spectral scenes keep their integrator.
 * The sampling pattern (MT_SAMPLING_*) occupies bits 4..5.  BLAS_GPU_LAYOUT is
 * bit 2 (layout code 2) of the reference's blasLayoutMask: set it when any
 * instance record carries BLAS layout code 2 (BVH_GPU); without it such
 * instances are not traversed, as in a shader compiled without that layout.
 * BVH2 (layout code 0) is always traversed.
 * A SPECTRAL scene with three dispersion wavelengths shares each sample's
 * path prefix: the first wavelength path runs in RGB until it meets a
 * dispersive transmissive surface, where it forks into the three wavelength
 * paths (the reference's shareSpectralPrefix, spectralPrefix.wgsl.ts, its
 * default whenever dispersionWavelengths is 3: WGPURayTracePass.ts:2113,2122,
 * scene-core.ts:689).  SPECTRAL_INDEPENDENT selects the variant without
 * sharing, where every wavelength path is spectral from the camera (the
 * reference's shader compiled with shareSpectralPrefix off). */
enum { MTC_SCENE_HAS_MEDIUM = 1u, MTC_SCENE_SPECTRAL = 2u,
       MTC_SCENE_PATTERN_SHIFT = 4u, MTC_SCENE_PATTERN_MASK = 0x30u,
       MTC_SCENE_BLAS_GPU_LAYOUT = 0x100u, MTC_SCENE_HAS_ALPHA = 0x200u,
       MTC_SCENE_SPECTRAL_INDEPENDENT = 0x400u };

/* G3 accumulation outputs (rayTrace.compute.ts:294-299; never overwritten,
 * always accumulated).  shadow_catcher holds 3 vec4 per pixel
 * {mask, background, moments} (shadowCatcherAccumulation.wgsl.ts:9-15). */
typedef struct mtc_outputs {
  void *color;
  void *normal;
  void *albedo;
  void *shadow_catcher;
} mtc_outputs;

/* First-hit record of querySceneSoftware (intersect.wgsl.ts:660-684). */
typedef struct mtc_hit {
  int32_t hit;
  int32_t instance;
  int32_t record;
  float t;
  float barycentric[3];
  float _pad;
} mtc_hit;

/* Runtime counters (extension+shadow rays, path samples, kernel launches
 * that ran), for Mrays/s and launch counts. */
typedef struct mtc_counters {
  unsigned long long path_samples;
  unsigned long long extension_rays;
  unsigned long long shadow_rays;
  unsigned long long kernel_launches;
} mtc_counters;

/* Library ABI version of this header. */
#define MTC_ABI_VERSION 1u
uint32_t mtc_abi_version(void);

/* One progressive pass per sample over the whole image: for each of
 * `samples` passes, every pixel (x, y) with x < output_size.x and
 * y < output_size.y traces one path sample and adds to `out`.  The per-pixel
 * sample index is read from out->normal[idx].w + sample_sequence_offset,
 * exactly as rayTrace.compute.ts:1187-1193.  Replaces the per-sample dispatch
 * loop of native/host/src/lib.rs:1506-1560.  counters may be NULL. */
mt_status mtc_trace_samples(const mtc_scene_view *scene,
                            const mtc_camera_uniform *camera,
                            const mtc_trace_uniform *uniform,
                            const mtc_outputs *out, uint32_t samples,
                            mtc_counters *counters, void *stream);

/* Raw first-hit query over `count` rays (8 floats each: o.xyz, pad, d.xyz,
 * pad; device memory), writing `hits` (device memory).  The contract of
 * querySceneSoftware, intersect.wgsl.ts:660-684 (bounces 0, single-sided). */
mt_status mtc_query_first_hit(const mtc_scene_view *scene, const float *rays,
                              uint32_t count, mtc_hit *hits, void *stream);

/* Raw material-map lookups: texels[i] (RGBA, 4 floats) = the bilinear
 * sampleMap of map indices[i] at uvs[2i..2i+1] (materialBuffer.wgsl.ts:
 * 335-378: the map's UV transform and wrap modes applied, no color decoding);
 * zero for an index outside the scene's maps.  All arrays in device memory.
 * No reference counterpart: a diagnostic that exposes the shading code's
 * texture filter for bit-exact checks. */
mt_status mtc_sample_maps(const mtc_scene_view *scene, const int32_t *indices,
                          const float *uvs, uint32_t count, float *texels,
                          void *stream);

/* Full TLAS refit on the device: rewrites the instance records (inverse
 * transform, transform, BLAS placement) and every TLAS node box from the
 * per-source-instance transforms, following bvhAccel.ts:579-740 refitTLAS with
 * no dirty set.  transforms: f64[16 * n] column-major (device); local_bounds:
 * f32[6 * n] BLAS-local AABB per source instance (device); blas_offsets and
 * vertex_offsets: i32 per source instance; materials: packed i32 per source
 * instance; colors f32[3 * n].  tlas/instances are the device buffers to
 * update in place; tlas_vec4_count bounds the TLAS node range. */
mt_status mtc_refit_tlas(void *tlas, uint64_t tlas_vec4_count, void *instances,
                         uint32_t instance_count, const double *transforms,
                         const float *local_bounds, const int32_t *blas_offsets,
                         const int32_t *blas_layouts, const int32_t *vertex_offsets,
                         const int32_t *materials, const float *colors,
                         void *stream);

/* read_average of native/host/src/lib.rs:343-364 on the device: out[i] =
 * accum[i] / samples for the `pixels` float4 of an accumulation buffer
 * (outColor, outNormal or outAlbedo), ordered on `stream`.  *nonfinite_flag
 * (device) is cleared and then set to 1 if any result is not finite, which the
 * reference treats as a failed read ("Non-finite native output"). */
mt_status mtc_average_output(const void *accum, uint32_t pixels, uint32_t samples,
                             void *out, uint32_t *nonfinite_flag, void *stream);

/* ------------------------------------------------ BLAS build on the device */
/* buildBLAS (src/renderer/bvhAccel.ts:200-286, without displacement) on the
 * GPU: the per-triangle boxes of triangleBounds (bvhAccel.ts:134-175; a
 * triangle whose box is not finite, or that indexes past the vertex array, is
 * skipped), the binned-SAH build of src/renderer/binnedSahBvh.ts:70-236
 * (float64 binning and costs, JavaScript Math.min/max, the same in-place
 * partition order) and the depth-first BVH2 layout of binnedSahBvh.ts:252-275
 * (BLAS layout code 0), written to `out_bvh`.  The buffer is bit-identical to
 * the reference producer's for the same positions, indices and bins. */
typedef struct mtc_blas_build_input {
  uint32_t struct_size;
  uint32_t bins;                   /* SAH bins, 1..64 (buildBLAS uses 8) */
  const float *positions;          /* device: xyz f32 per vertex */
  const uint32_t *indices;         /* device: 3 u32 per triangle */
  uint32_t vertex_count;
  uint32_t triangle_count;
} mtc_blas_build_input;

typedef struct mtc_blas_build_result {
  uint32_t struct_size;
  uint32_t vec4_count;             /* length of the BVH2 buffer written */
  uint32_t max_depth;              /* layoutBvh2 maxDepth (traversal stack bound) */
  uint32_t max_leaf_primitives;
  uint32_t node_count;
  uint32_t primitive_count;        /* triangles with a finite box */
  float local_bounds[6];           /* root box, getBvhBounds (geometryBvhBounds.ts:74-77) */
  uint32_t host_syncs;             /* stream synchronisations the build made */
  uint32_t _pad[3];
} mtc_blas_build_result;

/* Device scratch bytes mtc_build_blas needs for `triangle_count` triangles. */
uint64_t mtc_blas_build_scratch_bytes(uint32_t triangle_count, uint32_t bins);
/* Upper bound of the BVH2 length (vec4 units) for `triangle_count` triangles:
 * 2 per node (at most 2n - 1 nodes) plus one per triangle. */
uint64_t mtc_blas_build_max_vec4(uint32_t triangle_count);
/* No reference counterpart as an entry point: it replaces the host-side
 * buildBLAS call above.  Runs on `stream` and returns once `out_bvh` is
 * complete (the top of the tree is built level by level, reading one counter
 * back per level).  result->struct_size must be set by the caller.
 * MT_ERROR_BUFFER_TOO_SMALL if the layout needs more than out_capacity_vec4
 * (result->vec4_count then holds the length needed). */
mt_status mtc_build_blas(const mtc_blas_build_input *input, void *scratch, uint64_t scratch_bytes,
                         float *out_bvh, uint64_t out_capacity_vec4, mtc_blas_build_result *result,
                         void *stream);

/* ------------------------------------------------ BLAS refit on the device */
/* refitBLAS (src/renderer/bvhAccel.ts:800-870, BVH2 layout, no displacement)
 * after vertex deformation: every node box of a layout-0 BLAS rewritten in
 * place, leaves from their finite vertices, interior nodes from their
 * children (Math.min/max), the boxes bit-identical to the reference's.
 * mtc_blas_refit_prepare walks the BLAS once and stores its nodes by depth
 * in `plan` (device memory of mtc_blas_refit_plan_bytes bytes, 256-byte
 * aligned), like the reference's cached getBlasRefitData (bvhAccel.ts:
 * 758-796); it synchronises `stream` once per depth and rejects a buffer
 * whose offsets leave it or do not follow the depth-first order.  A plan
 * stays valid while the BLAS topology does. */
typedef struct mtc_blas_refit_plan_info {
  uint32_t struct_size;
  uint32_t node_count;
  uint32_t levels;                 /* pass to mtc_refit_blas */
  uint32_t _pad[5];
} mtc_blas_refit_plan_info;
uint64_t mtc_blas_refit_plan_bytes(uint64_t bvh_vec4_count);
mt_status mtc_blas_refit_prepare(const void *bvh, uint64_t bvh_vec4_count, void *plan, uint64_t plan_bytes,
                                 mtc_blas_refit_plan_info *info, void *stream);
/* Asynchronous on `stream` (levels + 1 launches; capturable in a graph).
 * positions: xyz f32 per vertex (device).  surface_area (device, may be
 * NULL) receives the sum of 2(xz + xy + zy) over the refitted nodes, the
 * reference's rebuild hint, summed in a fixed tree order. */
mt_status mtc_refit_blas(void *bvh, uint64_t bvh_vec4_count, const void *plan, uint32_t levels,
                         const float *positions, uint32_t vertex_count, double *surface_area, void *stream);

/* ------------------------------------------------------ batched form */
/* One render job of a batched launch: its own scene view, camera, uniform
 * and outputs.  All jobs of a batch run in one persistent kernel that pulls
 * (job, pixel-tile, sample) work items from a global queue. */
typedef struct mtc_job_desc {
  mtc_scene_view scene;
  mtc_camera_uniform camera;
  mtc_trace_uniform uniform;
  mtc_outputs out;
  uint32_t samples;        /* samples to add in this launch */
  uint32_t _pad[3];
} mtc_job_desc;

/* Tuning knobs of the persistent batched kernel, chosen by the autotuner
 * (0 selects the built-in default).  None changes any job's result. */
typedef struct mtc_batch_config {
  uint32_t struct_size;
  uint32_t block_threads;    /* threads per CTA: 32, 64, 96 or 128 (default 128) */
  uint32_t tile_width;       /* warp tile width in pixels: 1, 2, 4, 8, 16 or 32;
                                height = 32 / width (default 8, an 8x4 tile) */
  uint32_t ctas_per_sm;      /* grid = SM count * ctas_per_sm (default 16) */
  uint32_t items_per_fetch;  /* warp tiles taken per queue atomic, 1..16 (default 1) */
  uint32_t _pad[3];
} mtc_batch_config;

/* Runs `job_count` jobs (descriptors in HOST memory; their buffers are device
 * pointers) to completion in one persistent launch.  `queue_state` is
 * caller-provided device scratch of mtc_batch_scratch_bytes(job_count) bytes
 * that receives the job table and the work-queue counter (reset by the call
 * on `stream`).  status_out (device, may be NULL) is cleared on `stream`; the
 * kernel then sets MTC_BATCH_STATUS_GUARD_EXHAUSTED in it if a warp's work
 * loop reached its iteration bound before the queue drained (a corrupted
 * table: the warp stops instead of spinning).  Work is
 * pulled with one atomic per warp tile (config->items_per_fetch tiles); every
 * sample of a tile runs in order on one warp, so each job's outputs are
 * bit-identical to running it alone through mtc_trace_samples. */
#define MTC_BATCH_STATUS_GUARD_EXHAUSTED 1u
size_t mtc_batch_scratch_bytes(uint32_t capacity);
mt_status mtc_trace_batch(const mtc_job_desc *jobs, uint32_t job_count,
                          const mtc_batch_config *config, void *queue_state,
                          uint32_t *status_out, mtc_counters *counters,
                          void *stream);

/* The two halves of mtc_trace_batch, for replay.  mtc_batch_prepare writes
 * the job table of `jobs` (a 256-byte header with the job count and work-item
 * total, then one entry per job) into caller HOST memory `table` of at least
 * mtc_batch_table_bytes(job_count) bytes and reports the item total (host
 * only, no CUDA call).  mtc_batch_launch copies mtc_batch_table_bytes(capacity)
 * bytes of `table` into `queue_state` (mtc_batch_scratch_bytes(capacity)
 * bytes of device memory), clears the work counter and launches the
 * persistent kernel, all ordered on `stream`.  The kernel reads the job count
 * and total from the copied header, so with `table` in pinned host memory the
 * three operations can be captured once in a CUDA graph and replayed after
 * mtc_batch_prepare has rewritten the table with up to `capacity` other jobs.
 * The tile shape is fixed by prepare's config; launch's config sets the
 * block size, CTAs per SM and fetch grain. */
size_t mtc_batch_table_bytes(uint32_t capacity);
mt_status mtc_batch_prepare(const mtc_job_desc *jobs, uint32_t job_count,
                            const mtc_batch_config *config, void *table,
                            uint32_t *total_items);
mt_status mtc_batch_launch(const void *table, uint32_t capacity,
                           const mtc_batch_config *config, void *queue_state,
                           mtc_counters *counters, void *stream);

/* Wavefront form of the batched launch.  The integrator's event loop is cut
 * at its traversals into kernels over queues of in-flight path slots
 * (closest-hit traversal, shading, NEE shadow traversal, accumulation and
 * restart), so the latency-bound traversals run at the occupancy of their own
 * small register budget instead of the shading code's.  A slot owns one
 * pixel until all of its samples are done, so outputs are bit-identical to
 * mtc_trace_samples and to mtc_trace_batch.  `table` is a HOST job table
 * written by mtc_batch_prepare for up to `capacity` jobs; `state` is device
 * memory of mtc_stream_state_bytes(capacity, config) bytes.  The event loop
 * runs on the device: one CUDA graph whose WHILE node repeats an event
 * iteration until the queues have drained or max_iterations iterations have
 * run, so a run needs no host round trip after it is enqueued (unless
 * iterations_per_check asks for the host-driven loop).
 * mtc_stream_run enqueues the run on `stream` and waits for it (returning
 * MT_ERROR_TIMEOUT when the iteration limit stopped it); mtc_stream_launch
 * only enqueues it, and mtc_stream_status reports the outcome of the last run
 * enqueued on `state` the same way (it waits on `stream`).  The table is
 * uploaded with cudaMemcpyAsync on `stream`: a table in pinned memory must
 * stay unchanged until the stream has passed the launch (pageable memory is
 * read before the call returns).  Neither call is for stream capture: a
 * run launches its own graph.  One `state` buffer serves one run at a time.
 * No counterpart in the reference. */
typedef struct mtc_stream_config {
  uint32_t struct_size;
  uint32_t slots;                 /* paths in flight, 1024..2^25 (default 2^21) */
  uint32_t iterations_per_check;  /* 0 (default): the device-driven loop (one graph
                                     launch, the queue checked on the device after
                                     every iteration); 1..256: a host-driven loop,
                                     every kernel a separate launch and the host
                                     checking the queue every N iterations (blocking
                                     mtc_stream_run only; for profilers that cannot
                                     look into conditional graphs) */
  uint32_t max_iterations;        /* MT_ERROR_TIMEOUT beyond this (default 2^20) */
  uint32_t refill_lanes;          /* idle lanes of a warp that trigger fetching new
                                     rays in the traversal kernels, 1..32 (default 4) */
  uint32_t regroup_interval;      /* order the shading queue by material class every
                                     N-th event iteration, 1..1024 (default 1);
                                     MTC_REGROUP_OFF never */
  uint32_t sort_rays;             /* 1: order each extension queue by (job, direction
                                     octant) before traversal (default 0) */
  uint32_t steps_per_check;       /* traversal steps between refill checks, 1..64
                                     (default 8) */
  uint32_t traversal_ctas_per_sm; /* caps the resident CTAs per SM of the persistent
                                     traversal kernels, 1..8 (default 0: as many as
                                     their registers allow, 5 for closest-hit and 6
                                     for shadow rays) */
  uint32_t _pad[3];
} mtc_stream_config;
#define MTC_REGROUP_OFF 0xffffffffu
size_t mtc_stream_state_bytes(uint32_t capacity, const mtc_stream_config *config);
mt_status mtc_stream_run(const void *table, uint32_t capacity,
                         const mtc_stream_config *config, void *state,
                         mtc_counters *counters, void *stream);
mt_status mtc_stream_launch(const void *table, uint32_t capacity,
                            const mtc_stream_config *config, void *state,
                            mtc_counters *counters, void *stream);
mt_status mtc_stream_status(const void *state, uint32_t capacity,
                            const mtc_stream_config *config, void *stream);

/* No counterpart in the reference.  For callers that cannot let the library
 * allocate device memory (a host that owns a fixed device budget and its own
 * allocator, a plugin inside such a host, a serving loop that cannot afford a
 * synchronising cudaMalloc): the same batched launch as mtc_trace_batch, but
 * its scratch (job table and work-queue counter) lives in one fixed array
 * inside the library's device image, sized for MTC_BATCH_NOALLOC_MAX_JOBS
 * jobs, so the call allocates nothing; a larger job_count returns
 * MT_ERROR_INVALID_ARGUMENT.  The caller still passes the jobs with their
 * scene buffers and accumulation outputs.  Jobs and `config` follow the rules
 * of mtc_trace_batch (same validation, every config field applied), and
 * status_out is used the same way.  The first call on a device (and the first
 * after its primary context was reset) looks up that array's device address
 * (cudaGetSymbolAddress) with the device current.  Each call assembles the
 * job table in host stack memory and uploads it with cudaMemcpyAsync on
 * `stream` (pageable memory: read before the call returns).  Every call on a
 * device shares the one array (each call rewrites the table and clears the
 * counter), so calls whose work overlaps on the same device race: serialise
 * them, for example on one stream.  The array stays resident on every device
 * that loads the library until the process exits. */
#define MTC_BATCH_NOALLOC_MAX_JOBS 64
mt_status mtc_trace_batch_noalloc(const mtc_job_desc *jobs, uint32_t job_count,
                                  const mtc_batch_config *config,
                                  uint32_t *status_out, mtc_counters *counters,
                                  void *stream);

/* ------------------------------------------------------- host context */
typedef uint64_t mt_context;
typedef uint64_t mt_render_job;

/* Flattened host buffer bundle: the same arrays as mtc_scene_view, in host
 * memory, plus camera and uniform defaults.  commit copies everything. */
typedef struct mt_scene_bundle {
  uint32_t struct_size;
  uint32_t width, height;
  uint32_t flags;                  /* MTC_SCENE_* */
  const float *bvh; uint64_t bvh_vec4_count;
  const float *instances; uint32_t instance_count;
  uint32_t material_count;
  const uint32_t *attributes; uint64_t attribute_words;
  mtc_vertex_layout vertex_layout;
  const float *materials;
  const float *env_map; uint32_t env_width, env_height;
  const float *env_distribution;
  const float *light_sampling; uint32_t light_sampling_texels;
  uint32_t lights_count;
  const float *energy_lut;
  const float *analytic_lights;
  uint32_t tlas_stack_size, blas_stack_size;
  mtc_camera_uniform camera;
  mtc_trace_uniform uniform;       /* settings fields are overwritten by mt_render_settings */
  const float *maps; uint32_t map_count;       /* MTC_MAP_VEC4_ROWS vec4 per map */
  const float *map_texels; uint64_t map_texel_count;
  const uint32_t *triangle_materials;  /* bvh_vec4_count words or NULL (mtc_scene_view) */
} mt_scene_bundle;

/* mutracer-context.h:86-100 */
typedef struct mt_render_settings {
  uint32_t struct_size, sampling_pattern, seed, max_samples;
  uint32_t bounces, direct_light_candidates, bevel_samples, sample_sequence_offset;
  double clamping, transmissive_output_alpha_min;
  uint32_t caustic_flags;
  uint32_t light_photons, photon_map_photons;
  float photon_map_radius;
} mt_render_settings;

/* mutracer-context.h:63-68 */
typedef struct mt_context_snapshot {
  uint32_t struct_size;
  uint32_t width, height, samples;
  uint32_t state;
  uint32_t last_commit;
} mt_context_snapshot;

/* mutracer-context.h:176-180 */
typedef struct mt_job_snapshot {
  uint32_t struct_size;
  uint32_t state;
  uint32_t requested_samples, submitted_samples, completed_samples, base_samples;
} mt_job_snapshot;

/* mutracer-status.h:68 */
typedef enum mt_backend { MT_BACKEND_SOFTWARE = 0, MT_BACKEND_HWRT = 1 } mt_backend;
/* mutracer-context.h:73 (native/host/src/context.rs:697-716).  backend is
 * MT_BACKEND_SOFTWARE or MT_BACKEND_HWRT (the mt_context_create default);
 * other values return MT_ERROR_INVALID_ARGUMENT, no CUDA device
 * MT_ERROR_UNAVAILABLE.  B200 has no ray-tracing cores: every context
 * traverses in software (the CUDA kernels), whichever backend is asked for. */
int32_t mt_context_create_with_backend(uint32_t backend, mt_context *output, char *error,
                                       size_t capacity);
/* mutracer-context.h:79 (context.rs:3516-3555).  After a commit: *active is
 * the backend used (always MT_BACKEND_SOFTWARE) and `reason` (caller storage,
 * reason_capacity >= 1, always NUL terminated) says why it differs from an
 * HWRT request, or is empty.  NULL outputs return MT_ERROR_INVALID_ARGUMENT;
 * no healthy committed scene MT_ERROR_INVALID_STATE. */
int32_t mt_context_backend(mt_context handle, uint32_t *active, char *reason, size_t reason_capacity,
                           char *error, size_t capacity);
/* mutracer-context.h:77 */
int32_t mt_context_create(mt_context *output, char *error, size_t capacity);
/* mutracer-context.h:81: also cancels a commit in preparation. */
int32_t mt_context_destroy(mt_context handle, char *error, size_t capacity);
/* mutracer-context.h:87 (context.rs:1409-1424).  Idempotent: a commit in
 * preparation on another thread returns MT_ERROR_CANCELLED after its current
 * preparation step (descriptor decode and buffer building, or the start of
 * publication) and keeps the previous scene; without one it has no effect.
 * A second commit while one is in preparation returns MT_ERROR_INVALID_STATE. */
int32_t mt_context_cancel_commit(mt_context handle, char *error, size_t capacity);
/* mutracer-context.h:101 */
int32_t mt_render_settings_default(mt_render_settings *output);
/* mutracer-context.h:91 (commit) and :102-103 (commit_with_settings): the
 * descriptor argument is the flattened bundle. settings may be NULL. */
int32_t mt_context_commit_bundle(mt_context handle, const mt_scene_bundle *bundle,
                                 const mt_render_settings *settings, char *error,
                                 size_t capacity);
/* mutracer-context.h:94 and :132-133: commit a scene descriptor v8 (the
 * byte layout of native/docs/scene-format.md).  A malformed descriptor returns
 * MT_ERROR_INVALID_ARGUMENT with a message naming the problem; a valid one
 * that uses a feature this build does not render (displacement, anisotropy
 * and coat-normal maps, UDIM sets, textures the atlas would downscale,
 * material graphs, IES profiles, rect-light textures, background maps,
 * bevel, shadow-catcher and unlit materials, alpha in a dispersive scene)
 * returns MT_ERROR_UNAVAILABLE naming the feature.  Either way the previously
 * committed scene stays.  commit uses mt_render_settings_default. */
int32_t mt_context_commit(mt_context handle, const uint8_t *input, size_t length, char *error,
                          size_t capacity);
int32_t mt_context_commit_with_settings(mt_context handle, const uint8_t *input, size_t length,
                                        const mt_render_settings *settings, char *error,
                                        size_t capacity);
/* mutracer-context.h:104 */
int32_t mt_context_render(mt_context handle, uint32_t additional_samples, char *error,
                          size_t capacity);
/* mutracer-context.h:105 */
int32_t mt_context_reset(mt_context handle, char *error, size_t capacity);
/* mutracer-context.h:112 */
#define MT_WAIT_INDEFINITELY UINT32_MAX
int32_t mt_context_wait(mt_context handle, uint32_t timeout_ms, char *error, size_t capacity);
/* mutracer-context.h:113 */
int32_t mt_context_info(mt_context handle, mt_context_snapshot *info, char *error,
                        size_t capacity);
/* mutracer-context.h:114-115: f32 RGBA, bottom row first, divided by the
 * per-pixel completed sample count. pixels=NULL,size=0 queries the size.
 * Checked in the reference's order: NULL written, unknown handle, no healthy
 * scene, an active job (MT_ERROR_INVALID_STATE), unknown kind, no completed
 * samples (MT_ERROR_INVALID_STATE), then the size query and destination. */
int32_t mt_context_read_pixels(mt_context handle, uint32_t kind, void *pixels, size_t size,
                               size_t *written, char *error, size_t capacity);
/* mutracer-debug.h:24-25 (debug and validation only, as in the reference):
 * commits the descriptor into a fresh context with the default settings
 * (Sobol, seed 12345, 6 bounces), renders `samples` (1..16384) samples and
 * writes render.rgba32f, normal.rgba32f, albedo.rgba32f (little-endian f32
 * RGBA, bottom row first), render.png (Reinhard + sRGB preview) and
 * result.json into output_directory.  A rejected descriptor returns the
 * commit's status; MT_ERROR_BUSY while another probe runs. */
int32_t mt_probe_render_scene(const uint8_t *input, size_t length, const char *output_directory,
                              uint32_t samples, char *error, size_t error_capacity);
/* mutracer-context.h:181-185 */
int32_t mt_context_submit(mt_context handle, uint32_t additional_samples, mt_render_job *job,
                          char *error, size_t capacity);
int32_t mt_job_poll(mt_render_job job, uint32_t max_new_samples, char *error, size_t capacity);
int32_t mt_job_info(mt_render_job job, mt_job_snapshot *info, char *error, size_t capacity);
int32_t mt_job_cancel(mt_render_job job, char *error, size_t capacity);

#ifdef __cplusplus
}
#endif
#endif
