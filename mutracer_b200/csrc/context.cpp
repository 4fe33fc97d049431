// Persistent host API of native/include/mutracer-context.h:57-187 on CUDA:
// contexts own device copies of a committed buffer bundle plus the four
// accumulation buffers; renders and job batches add samples through the
// wavefront engine (mtc_trace_samples when its state cannot be allocated);
// jobs are caller-polled with at most one batch in flight (a CUDA event), like
// native/host/src/context.rs:2002-2256 (submit/poll_job/advance_job).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <sys/stat.h>
#include <cerrno>

#include "../../include/mutracer_b200.h"
#include "mtp_api.h"
#include "scene_prep.h"

namespace {

void setError(char *error, size_t capacity, const std::string &msg) {
  if (!error || capacity == 0) return;
  size_t n = std::min(msg.size(), capacity - 1);
  std::memcpy(error, msg.data(), n);
  error[n] = '\0';
}

// Device allocation kept across commits: a commit of a scene that fits the
// previous capacity reuses it instead of freeing and reallocating.
struct DeviceBuffer {
  void *ptr = nullptr;
  size_t bytes = 0, capacity = 0;
  ~DeviceBuffer() { if (ptr) cudaFree(ptr); }
  cudaError_t reserve(size_t n) {
    bytes = n;
    if (n <= capacity) return cudaSuccess;
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    capacity = 0;
    cudaError_t e = cudaMalloc(&ptr, n);
    if (e != cudaSuccess) { ptr = nullptr; bytes = 0; return e; }
    capacity = n;
    return cudaSuccess;
  }
  // Copies `n` bytes of caller memory, ordered on `stream`; the caller's
  // memory is no longer needed when the call returns (pageable sources are
  // staged by the driver before cudaMemcpyAsync returns).
  cudaError_t upload(const void *host, size_t n, cudaStream_t stream) {
    if (!host || n == 0) { bytes = 0; return cudaSuccess; }
    cudaError_t e = reserve(n);
    if (e != cudaSuccess) return e;
    return cudaMemcpyAsync(ptr, host, n, cudaMemcpyHostToDevice, stream);
  }
  void *data() const { return bytes ? ptr : nullptr; }
};

struct SceneResources {
  DeviceBuffer bvh, ins, attr, mats, env, envDist, lightData, lut, lights, maps, mapTexels, triMats;
  DeviceBuffer color, normal, albedo, catcher;
  DeviceBuffer average, flag;  // read_pixels staging: averaged image, non-finite flag
  DeviceBuffer stream;         // wavefront state of blocking renders (mtc_stream_run)
  mtc_scene_view view{};
  uint32_t width = 0, height = 0;
};

struct Job {
  uint64_t handle = 0;
  uint32_t state = MT_JOB_QUEUED;
  uint32_t requested = 0, submitted = 0, completed = 0, base = 0;
  uint32_t inflight = 0;
  bool wavefront = false;  // the batch in flight runs in the wavefront engine
};

struct Context {
  std::mutex m;
  uint64_t handle = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t event = nullptr;
  std::unique_ptr<SceneResources> scene;
  mtc_camera_uniform camera{};
  mtc_trace_uniform uniform{};
  uint32_t samples = 0;  // completed samples
  bool failed = false;
  uint32_t lastCommit = MT_COMMIT_NONE;
  uint32_t backend = MT_BACKEND_SOFTWARE;  // requested at creation
  std::unique_ptr<Job> job;
  // A commit in preparation, and a cancellation request for it
  // (mt_context_cancel_commit); both are read without the context lock.
  std::atomic<bool> committing{false}, cancelCommit{false};
  ~Context() {
    if (stream) cudaStreamSynchronize(stream);
    scene.reset();
    if (event) cudaEventDestroy(event);
    if (stream) cudaStreamDestroy(stream);
  }
};

std::mutex gRegistry;
std::map<uint64_t, std::shared_ptr<Context>> gContexts;
std::map<uint64_t, uint64_t> gJobs;  // job handle -> context handle
uint64_t gNextHandle = 1;

std::shared_ptr<Context> findContext(uint64_t h) {
  std::lock_guard<std::mutex> g(gRegistry);
  auto it = gContexts.find(h);
  return it == gContexts.end() ? nullptr : it->second;
}

bool activeJob(const Context &c) {
  return c.job && (c.job->state == MT_JOB_QUEUED || c.job->state == MT_JOB_RUNNING || c.job->state == MT_JOB_CANCELLING);
}

void expireJob(Context &c) {
  if (!c.job) return;
  std::lock_guard<std::mutex> g(gRegistry);
  gJobs.erase(c.job->handle);
  c.job.reset();
}

int32_t failContext(Context &c, cudaError_t e, char *error, size_t capacity) {
  c.failed = true;
  setError(error, capacity, std::string("CUDA failure: ") + cudaGetErrorString(e));
  cudaGetLastError();
  return MT_ERROR_CONTEXT_FAILED;
}

// Marks a commit in preparation for its lifetime (mutracer-context.h:86-88,
// 114-119): a second commit meanwhile is refused, and a cancellation request
// made during it is seen at its next preparation step.
class CommitGuard {
 public:
  explicit CommitGuard(Context &c) : c_(c) {
    bool expected = false;
    owned_ = c.committing.compare_exchange_strong(expected, true);
    if (owned_) c.cancelCommit.store(false);
  }
  ~CommitGuard() {
    if (owned_) {
      c_.cancelCommit.store(false);
      c_.committing.store(false);
    }
  }
  bool owned() const { return owned_; }

 private:
  Context &c_;
  bool owned_ = false;
};

int32_t commitCancelled(Context &c, char *error, size_t capacity) {
  if (!c.cancelCommit.load()) return MT_OK;
  setError(error, capacity, "commit cancelled; the previous scene is kept");
  return MT_ERROR_CANCELLED;
}

uint32_t logSpp(uint32_t maxSamples) {
  // sceneAssembly.ts:34-37 traceSampling (ZSobol uses max_samples - 1).
  uint32_t n = std::max(1u, maxSamples);
  uint32_t l = 0;
  while ((1u << l) < n && l < 16) l++;
  return std::min(16u, l);
}

void applySettings(Context &c, const mt_render_settings &s) {
  c.uniform.sequence_seed = s.seed;
  c.uniform.bounces = int32_t(std::min(20u, std::max(1u, s.bounces)));
  c.uniform.direct_light_candidates = int32_t(std::min(16u, std::max(1u, s.direct_light_candidates)));
  c.uniform.sample_sequence_offset = s.sample_sequence_offset;
  c.uniform.clamping = float(s.clamping);
  c.uniform.transmissive_output_alpha_min = float(s.transmissive_output_alpha_min);
  c.uniform.zsobol_log_spp = logSpp(s.sampling_pattern == MT_SAMPLING_ZSOBOL ? std::max(1u, s.max_samples - 1) : s.max_samples);
}

mtc_stream_config streamConfig(size_t pixels) {
  mtc_stream_config cfg;
  std::memset(&cfg, 0, sizeof(cfg));
  cfg.struct_size = sizeof(cfg);
  cfg.slots = uint32_t(std::max<size_t>(1024, std::min<size_t>(pixels, size_t(1) << 21)));
  return cfg;
}

int32_t launch(Context &c, uint32_t samples) {
  mtc_outputs out{c.scene->color.ptr, c.scene->normal.ptr, c.scene->albedo.ptr, c.scene->catcher.ptr};
  return mtc_trace_samples(&c.scene->view, &c.camera, &c.uniform, &out, samples, nullptr, c.stream);
}

// Renders and job batches run their samples through the wavefront engine
// (queued traversal and material-regrouped shading, its event loop on the
// device), which writes the same bits as mtc_trace_samples at about twice the
// throughput: mtc_stream_run for blocking renders, mtc_stream_launch for job
// batches, which only enqueue.  Path slots scale with the image, up to 2^21;
// the state buffer is kept with the scene.  When it cannot be allocated the
// megakernel renders instead (*wavefront false).
int32_t renderSamples(Context &c, uint32_t samples, bool wait, bool *wavefront) {
  SceneResources &r = *c.scene;
  *wavefront = false;
  size_t px = size_t(r.width) * r.height;
  mtc_stream_config cfg = streamConfig(px);
  size_t bytes = mtc_stream_state_bytes(1, &cfg);
  if (bytes == 0 || r.stream.reserve(bytes) != cudaSuccess) {
    cudaGetLastError();
    return launch(c, samples);
  }
  mtc_job_desc job;
  std::memset(&job, 0, sizeof(job));
  job.scene = r.view;
  job.camera = c.camera;
  job.uniform = c.uniform;
  job.out = mtc_outputs{r.color.ptr, r.normal.ptr, r.albedo.ptr, r.catcher.ptr};
  job.samples = samples;
  std::vector<char> table(mtc_batch_table_bytes(1));
  int32_t st = mtc_batch_prepare(&job, 1, nullptr, table.data(), nullptr);
  if (st != MT_OK) return st;
  *wavefront = true;
  // The table is pageable host memory: the launch's upload has read it by
  // the time the call returns.
  return wait ? mtc_stream_run(table.data(), 1, &cfg, r.stream.ptr, nullptr, c.stream)
              : mtc_stream_launch(table.data(), 1, &cfg, r.stream.ptr, nullptr, c.stream);
}

// The publication step of every commit: validates the bundle, uploads it
// into the context's (reused) device buffers and restarts accumulation.  A
// cancellation requested before the first buffer is touched keeps the old
// scene; once uploads begin, the commit completes.
int32_t commitBundle(const std::shared_ptr<Context> &c, const mt_scene_bundle *b,
                     const mt_render_settings *settings, char *error, size_t capacity) {
  if (!b || b->struct_size != sizeof(mt_scene_bundle)) { setError(error, capacity, "bundle struct_size"); return MT_ERROR_INVALID_ARGUMENT; }
  if (settings && settings->struct_size != sizeof(mt_render_settings)) { setError(error, capacity, "settings struct_size"); return MT_ERROR_INVALID_ARGUMENT; }
  if (b->width == 0 || b->height == 0 || b->width > 16384 || b->height > 16384 || !b->bvh || !b->instances ||
      !b->attributes || !b->materials || !b->energy_lut || !b->light_sampling || b->vertex_layout.stride < 4 ||
      (b->env_map && !b->env_distribution) || (b->lights_count && !b->analytic_lights) ||
      (b->vertex_layout.uv_offset && (b->vertex_layout.uv_offset < 3 ||
                                      b->vertex_layout.uv_offset + 2 > b->vertex_layout.stride)) ||
      (b->vertex_layout.uv1_offset && (b->vertex_layout.uv1_offset < 3 ||
                                       b->vertex_layout.uv1_offset + 2 > b->vertex_layout.stride)) ||
      (b->vertex_layout.color_offset &&
       (b->vertex_layout.color_offset < 3 ||
        b->vertex_layout.color_offset + (b->vertex_layout.color_float ? 3u : 1u) > b->vertex_layout.stride)) ||
      (b->map_count && !b->maps) || (b->map_texel_count && !b->map_texels) || b->map_texel_count > UINT32_MAX) {
    setError(error, capacity, "invalid buffer bundle");
    return MT_ERROR_INVALID_ARGUMENT;
  }
  if (settings && (!std::isfinite(settings->clamping) || !std::isfinite(settings->transmissive_output_alpha_min) ||
                   settings->sampling_pattern > MT_SAMPLING_RANDOM)) {
    setError(error, capacity, "invalid settings");
    return MT_ERROR_INVALID_ARGUMENT;
  }
  std::unique_lock<std::mutex> l(c->m, std::try_to_lock);
  if (!l) { setError(error, capacity, "context busy"); return MT_ERROR_BUSY; }
  if (int32_t st = commitCancelled(*c, error, capacity)) return st;
  // The previous job expires and nothing may still read the buffers that the
  // new scene reuses.
  expireJob(*c);
  cudaError_t e = cudaStreamSynchronize(c->stream);
  std::unique_ptr<SceneResources> r = c->scene ? std::move(c->scene) : std::make_unique<SceneResources>();
  size_t px = size_t(b->width) * b->height;
  cudaStream_t st = c->stream;
  auto up = [&](DeviceBuffer &d, const void *h, size_t n) { if (e == cudaSuccess) e = d.upload(h, n, st); };
  up(r->bvh, b->bvh, b->bvh_vec4_count * 16);
  up(r->ins, b->instances, size_t(b->instance_count) * MTC_INSTANCE_VEC4_STRIDE * 16);
  up(r->attr, b->attributes, b->attribute_words * 4);
  up(r->mats, b->materials, size_t(b->material_count) * MTC_MATERIAL_VEC4_ROWS * 16);
  up(r->env, b->env_map, b->env_map ? size_t(b->env_width) * b->env_height * 16 : 0);
  up(r->envDist, b->env_distribution, b->env_map ? size_t(b->env_width + 2) * (b->env_height + 1) * 8 : 0);
  up(r->lightData, b->light_sampling, size_t(b->light_sampling_texels) * 16);
  up(r->lut, b->energy_lut, size_t(MTC_ENERGY_LUT_WIDTH) * MTC_ENERGY_LUT_HEIGHT * 4);
  up(r->lights, b->analytic_lights, b->lights_count ? size_t(b->lights_count) * MTC_LIGHT_VEC4_ROWS * 16 : 0);
  up(r->maps, b->maps, size_t(b->map_count) * MTC_MAP_VEC4_ROWS * 16);
  up(r->mapTexels, b->map_texels, size_t(b->map_texel_count) * 16);
  up(r->triMats, b->triangle_materials, b->triangle_materials ? size_t(b->bvh_vec4_count) * 4 : 0);
  for (DeviceBuffer *d : {&r->color, &r->normal, &r->albedo, &r->catcher}) {
    size_t bytes = px * 16 * (d == &r->catcher ? 3 : 1);
    if (e == cudaSuccess) e = d->reserve(bytes);
    if (e == cudaSuccess) e = cudaMemsetAsync(d->ptr, 0, bytes, st);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    cudaGetLastError();
    // Reused buffers may hold part of the new scene: the context is failed
    // until a later commit succeeds.
    c->scene = std::move(r);
    c->failed = true;
    c->samples = 0;
    setError(error, capacity, std::string("commit failed: ") + cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? MT_ERROR_UNAVAILABLE : MT_ERROR_CONTEXT_FAILED;
  }
  mtc_scene_view &v = r->view;
  v.struct_size = sizeof(mtc_scene_view);
  v.flags = b->flags;
  v.bvh = r->bvh.data(); v.bvh_vec4_count = b->bvh_vec4_count;
  v.instances = r->ins.data(); v.instance_count = b->instance_count; v.material_count = b->material_count;
  v.attributes = r->attr.data(); v.attribute_words = b->attribute_words; v.vertex_layout = b->vertex_layout;
  v.materials = r->mats.data();
  v.env_map = r->env.data(); v.env_distribution = r->envDist.data(); v.env_width = b->env_width; v.env_height = b->env_height;
  v.light_sampling = r->lightData.data(); v.light_sampling_texels = b->light_sampling_texels;
  v.blas_offset = b->uniform.blas_offset;
  v.energy_lut = r->lut.data();
  v.analytic_lights = r->lights.data();
  v.tlas_stack_size = b->tlas_stack_size; v.blas_stack_size = b->blas_stack_size;
  v.maps = b->map_count ? r->maps.data() : nullptr; v.map_count = b->map_count;
  v.map_texels = b->map_texel_count ? r->mapTexels.data() : nullptr;
  v.map_texel_count = uint32_t(b->map_texel_count);
  v.triangle_materials = b->triangle_materials ? static_cast<const uint32_t *>(r->triMats.data()) : nullptr;
  r->width = b->width; r->height = b->height;
  // Publish: accumulation restarts.
  c->scene = std::move(r);
  c->camera = b->camera;
  c->uniform = b->uniform;
  c->uniform.output_size[0] = float(b->width);
  c->uniform.output_size[1] = float(b->height);
  if (settings) {
    applySettings(*c, *settings);
    c->scene->view.flags = (c->scene->view.flags & ~uint32_t(MTC_SCENE_PATTERN_MASK)) |
                           (settings->sampling_pattern << MTC_SCENE_PATTERN_SHIFT);
  }
  c->samples = 0;
  c->failed = false;
  c->lastCommit = MT_COMMIT_FULL;
  return MT_OK;
}

// ---------------------------------------------------------------- probe
// Output files of mt_probe_render_scene (native/host/src/lib.rs:2227-2290):
// the linear images as little-endian f32 RGBA, bottom row first, a Reinhard +
// sRGB 8-bit preview PNG (top row first) and a small result.json.
bool makeDirectories(const std::string &path) {
  std::string part;
  for (size_t i = 0; i <= path.size(); i++) {
    if (i == path.size() || path[i] == '/') {
      if (!part.empty() && mkdir(part.c_str(), 0777) != 0 && errno != EEXIST) return false;
    }
    if (i < path.size()) part.push_back(path[i]);
  }
  return true;
}

bool writeFile(const std::string &path, const void *data, size_t n) {
  FILE *f = std::fopen(path.c_str(), "wb");
  if (!f) return false;
  bool ok = std::fwrite(data, 1, n, f) == n;
  return std::fclose(f) == 0 && ok;
}

uint32_t crc32(const uint8_t *p, size_t n, uint32_t crc = 0) {
  crc = ~crc;
  for (size_t i = 0; i < n; i++) {
    crc ^= p[i];
    for (int k = 0; k < 8; k++) crc = (crc >> 1) ^ (0xedb88320u & (0u - (crc & 1u)));
  }
  return ~crc;
}

// An RGB8 PNG whose zlib stream uses stored (uncompressed) deflate blocks.
std::vector<uint8_t> encodePng(const std::vector<uint8_t> &rgb, uint32_t width, uint32_t height) {
  std::vector<uint8_t> raw;
  raw.reserve(size_t(height) * (width * 3 + 1));
  for (uint32_t y = 0; y < height; y++) {
    raw.push_back(0);  // filter: none
    raw.insert(raw.end(), rgb.begin() + size_t(y) * width * 3, rgb.begin() + size_t(y + 1) * width * 3);
  }
  std::vector<uint8_t> z = {0x78, 0x01};
  uint32_t a = 1, b = 0;
  for (uint8_t v : raw) { a = (a + v) % 65521u; b = (b + a) % 65521u; }
  for (size_t at = 0; at < raw.size() || at == 0; at += 65535) {
    size_t n = std::min<size_t>(65535, raw.size() - at);
    z.push_back(at + n >= raw.size() ? 1 : 0);
    z.push_back(uint8_t(n)); z.push_back(uint8_t(n >> 8));
    z.push_back(uint8_t(~n)); z.push_back(uint8_t(~n >> 8));
    z.insert(z.end(), raw.begin() + at, raw.begin() + at + n);
    if (raw.empty()) break;
  }
  uint32_t adler = (b << 16) | a;
  for (int k = 3; k >= 0; k--) z.push_back(uint8_t(adler >> (8 * k)));
  std::vector<uint8_t> png = {0x89, 'P', 'N', 'G', 0x0d, 0x0a, 0x1a, 0x0a};
  auto chunk = [&](const char *type, const std::vector<uint8_t> &data) {
    uint32_t n = uint32_t(data.size());
    for (int k = 3; k >= 0; k--) png.push_back(uint8_t(n >> (8 * k)));
    std::vector<uint8_t> body(type, type + 4);
    body.insert(body.end(), data.begin(), data.end());
    png.insert(png.end(), body.begin(), body.end());
    uint32_t c = crc32(body.data(), body.size());
    for (int k = 3; k >= 0; k--) png.push_back(uint8_t(c >> (8 * k)));
  };
  std::vector<uint8_t> ihdr;
  for (uint32_t v : {width, height})
    for (int k = 3; k >= 0; k--) ihdr.push_back(uint8_t(v >> (8 * k)));
  ihdr.insert(ihdr.end(), {8, 2, 0, 0, 0});  // 8-bit RGB, deflate, no filter method, no interlace
  chunk("IHDR", ihdr);
  chunk("IDAT", z);
  chunk("IEND", {});
  return png;
}

std::mutex gProbe;

}  // namespace

extern "C" {

int32_t mt_render_settings_default(mt_render_settings *o) {
  if (!o) return MT_ERROR_INVALID_ARGUMENT;
  std::memset(o, 0, sizeof(*o));
  o->struct_size = sizeof(mt_render_settings);
  o->sampling_pattern = MT_SAMPLING_SOBOL;
  o->seed = 12345;
  o->max_samples = 64;
  o->bounces = 6;
  o->direct_light_candidates = 2;
  o->bevel_samples = 8;
  o->sample_sequence_offset = 0;
  o->clamping = 0.0;
  o->transmissive_output_alpha_min = 1.0;
  return MT_OK;
}

int32_t mt_context_create(mt_context *output, char *error, size_t capacity) {
  return mt_context_create_with_backend(MT_BACKEND_HWRT, output, error, capacity);
}

// mutracer-context.h:73 (context.rs:697-716, create_in :571-582): HWRT is
// the reference's default request.  B200 has no ray-tracing cores, so every
// context traverses in software (the CUDA kernels); mt_context_backend
// reports that, with the reason when HWRT was asked for.
int32_t mt_context_create_with_backend(uint32_t backend, mt_context *output, char *error, size_t capacity) {
  if (!output) { setError(error, capacity, "output is NULL"); return MT_ERROR_INVALID_ARGUMENT; }
  *output = 0;
  if (backend > MT_BACKEND_HWRT) { setError(error, capacity, "Unknown native intersection backend"); return MT_ERROR_INVALID_ARGUMENT; }
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    setError(error, capacity, "no CUDA device");
    return MT_ERROR_UNAVAILABLE;
  }
  auto c = std::make_shared<Context>();
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&c->event, cudaEventDisableTiming) != cudaSuccess) {
    cudaGetLastError();
    setError(error, capacity, "stream creation failed");
    return MT_ERROR_UNAVAILABLE;
  }
  c->backend = backend;
  std::lock_guard<std::mutex> g(gRegistry);
  c->handle = gNextHandle++;
  gContexts[c->handle] = c;
  *output = c->handle;
  return MT_OK;
}

// mutracer-context.h:79 mt_context_backend (context.rs:3516-3555): the
// backend actually used for the committed scene, and why it differs from the
// request.
int32_t mt_context_backend(mt_context handle, uint32_t *active, char *reason, size_t reason_capacity, char *error,
                           size_t capacity) {
  if (!active || !reason || reason_capacity == 0) {
    setError(error, capacity, "Invalid backend info output");
    return MT_ERROR_INVALID_ARGUMENT;
  }
  auto c = findContext(handle);
  if (!c) { setError(error, capacity, "unknown context"); return MT_ERROR_INVALID_HANDLE; }
  std::unique_lock<std::mutex> l(c->m, std::try_to_lock);
  if (!l) { setError(error, capacity, "context busy"); return MT_ERROR_BUSY; }
  if (!c->scene || c->failed) { setError(error, capacity, "no healthy committed scene"); return MT_ERROR_INVALID_STATE; }
  *active = MT_BACKEND_SOFTWARE;
  setError(reason, reason_capacity,
           c->backend == MT_BACKEND_HWRT ? "hardware ray tracing is unavailable on this device: software BVH traversal"
                                         : "");
  return MT_OK;
}

int32_t mt_context_destroy(mt_context handle, char *error, size_t capacity) {
  auto c = findContext(handle);
  if (!c) { setError(error, capacity, "unknown context"); return MT_ERROR_INVALID_HANDLE; }
  std::unique_lock<std::mutex> l(c->m, std::try_to_lock);
  if (!l) { setError(error, capacity, "context busy"); return MT_ERROR_BUSY; }
  if (activeJob(*c)) { setError(error, capacity, "active render job: cancel/poll it first"); return MT_ERROR_INVALID_STATE; }
  if (c->committing.load()) c->cancelCommit.store(true);
  expireJob(*c);
  std::lock_guard<std::mutex> g(gRegistry);
  gContexts.erase(handle);
  return MT_OK;
}

int32_t mt_context_commit_bundle(mt_context handle, const mt_scene_bundle *b, const mt_render_settings *settings,
                                 char *error, size_t capacity) {
  auto c = findContext(handle);
  if (!c) { setError(error, capacity, "unknown context"); return MT_ERROR_INVALID_HANDLE; }
  CommitGuard guard(*c);
  if (!guard.owned()) { setError(error, capacity, "another commit is in preparation"); return MT_ERROR_INVALID_STATE; }
  return commitBundle(c, b, settings, error, capacity);
}


// mutracer-context.h:94 / :132-133: the scene descriptor v8 decoded (and
// validated) on the host, then committed like a buffer bundle.  A rejected
// descriptor leaves the previous scene committed.
int32_t mt_context_commit_with_settings(mt_context handle, const uint8_t *input, size_t length,
                                        const mt_render_settings *settings, char *error, size_t capacity) {
  auto c = findContext(handle);
  if (!c) { setError(error, capacity, "unknown context"); return MT_ERROR_INVALID_HANDLE; }
  if (settings && settings->struct_size != sizeof(mt_render_settings)) {
    setError(error, capacity, "settings struct_size");
    return MT_ERROR_INVALID_ARGUMENT;
  }
  CommitGuard guard(*c);
  if (!guard.owned()) { setError(error, capacity, "another commit is in preparation"); return MT_ERROR_INVALID_STATE; }
  // Preparation on the calling thread: decode, validate and build the
  // flattened buffers (BVHs, light tables) without touching the context.
  mtp::SceneHost scene;
  std::string message;
  int32_t st = mtp::decodeSceneDescriptor(input, length, scene, message);
  if (st != MT_OK) {
    setError(error, capacity, message);
    return st;
  }
  if ((st = commitCancelled(*c, error, capacity)) != MT_OK) return st;
  mt_render_settings defaults;
  if (!settings) {
    mt_render_settings_default(&defaults);
    settings = &defaults;
  }
  mt_scene_bundle bundle;
  mtp_scene_bundle(&scene, &bundle);
  return commitBundle(c, &bundle, settings, error, capacity);
}

// mutracer-context.h:87 mt_context_cancel_commit (context.rs:1409-1424):
// idempotent; a commit in preparation returns MT_ERROR_CANCELLED at its next
// preparation step and the previous scene stays; no commit, no effect.
int32_t mt_context_cancel_commit(mt_context handle, char *error, size_t capacity) {
  auto c = findContext(handle);
  if (!c) { setError(error, capacity, "unknown context"); return MT_ERROR_INVALID_HANDLE; }
  if (c->committing.load()) c->cancelCommit.store(true);
  return MT_OK;
}

int32_t mt_context_commit(mt_context handle, const uint8_t *input, size_t length, char *error, size_t capacity) {
  return mt_context_commit_with_settings(handle, input, length, nullptr, error, capacity);
}

int32_t mt_context_render(mt_context handle, uint32_t additional, char *error, size_t capacity) {
  auto c = findContext(handle);
  if (!c) { setError(error, capacity, "unknown context"); return MT_ERROR_INVALID_HANDLE; }
  std::unique_lock<std::mutex> l(c->m, std::try_to_lock);
  if (!l) { setError(error, capacity, "context busy"); return MT_ERROR_BUSY; }
  if (!c->scene || c->failed) { setError(error, capacity, "no healthy committed scene"); return MT_ERROR_INVALID_STATE; }
  if (activeJob(*c)) { setError(error, capacity, "active render job"); return MT_ERROR_INVALID_STATE; }
  if (additional == 0 || uint64_t(c->samples) + additional > 16384u) {
    setError(error, capacity, "render total must stay within 1..16384 samples");
    return MT_ERROR_INVALID_ARGUMENT;
  }
  expireJob(*c);
  bool wavefront = false;
  int32_t st = renderSamples(*c, additional, true, &wavefront);
  if (st != MT_OK) { setError(error, capacity, "launch rejected"); return st; }
  cudaError_t e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return failContext(*c, e, error, capacity);
  c->samples += additional;
  return MT_OK;
}

int32_t mt_context_reset(mt_context handle, char *error, size_t capacity) {
  auto c = findContext(handle);
  if (!c) { setError(error, capacity, "unknown context"); return MT_ERROR_INVALID_HANDLE; }
  std::unique_lock<std::mutex> l(c->m, std::try_to_lock);
  if (!l) { setError(error, capacity, "context busy"); return MT_ERROR_BUSY; }
  if (!c->scene || c->failed) { setError(error, capacity, "no healthy committed scene"); return MT_ERROR_INVALID_STATE; }
  if (activeJob(*c)) { setError(error, capacity, "active render job"); return MT_ERROR_INVALID_STATE; }
  expireJob(*c);
  cudaError_t e = cudaSuccess;
  for (DeviceBuffer *d : {&c->scene->color, &c->scene->normal, &c->scene->albedo, &c->scene->catcher})
    if (e == cudaSuccess) e = cudaMemsetAsync(d->ptr, 0, d->bytes, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return failContext(*c, e, error, capacity);
  c->samples = 0;
  return MT_OK;
}

int32_t mt_context_wait(mt_context handle, uint32_t timeout_ms, char *error, size_t capacity) {
  auto c = findContext(handle);
  if (!c) { setError(error, capacity, "unknown context"); return MT_ERROR_INVALID_HANDLE; }
  std::unique_lock<std::mutex> l(c->m, std::try_to_lock);
  if (!l) { setError(error, capacity, "context busy"); return MT_ERROR_BUSY; }
  if (!c->scene || c->failed) { setError(error, capacity, "no healthy committed scene"); return MT_ERROR_INVALID_STATE; }
  if (activeJob(*c)) { setError(error, capacity, "active render job"); return MT_ERROR_INVALID_STATE; }
  auto start = std::chrono::steady_clock::now();
  for (;;) {
    cudaError_t e = cudaStreamQuery(c->stream);
    if (e == cudaSuccess) return MT_OK;
    if (e != cudaErrorNotReady) return failContext(*c, e, error, capacity);
    auto ms = std::chrono::duration_cast<std::chrono::milliseconds>(std::chrono::steady_clock::now() - start).count();
    if (timeout_ms != MT_WAIT_INDEFINITELY && uint64_t(ms) >= timeout_ms) {
      setError(error, capacity, "timeout");
      return MT_ERROR_TIMEOUT;
    }
    std::this_thread::sleep_for(std::chrono::microseconds(200));
  }
}

int32_t mt_context_info(mt_context handle, mt_context_snapshot *info, char *error, size_t capacity) {
  auto c = findContext(handle);
  if (!c) { setError(error, capacity, "unknown context"); return MT_ERROR_INVALID_HANDLE; }
  if (!info || info->struct_size != sizeof(mt_context_snapshot)) { setError(error, capacity, "struct_size"); return MT_ERROR_INVALID_ARGUMENT; }
  std::unique_lock<std::mutex> l(c->m, std::try_to_lock);
  if (!l) { setError(error, capacity, "context busy"); return MT_ERROR_BUSY; }
  info->width = c->scene ? c->scene->width : 0;
  info->height = c->scene ? c->scene->height : 0;
  info->samples = c->samples;
  info->state = !c->scene ? MT_CONTEXT_EMPTY : c->failed ? MT_CONTEXT_FAILED : activeJob(*c) ? MT_CONTEXT_JOB_ACTIVE : MT_CONTEXT_COMMITTED;
  info->last_commit = c->lastCommit;
  return MT_OK;
}

int32_t mt_context_read_pixels(mt_context handle, uint32_t kind, void *pixels, size_t size, size_t *written,
                               char *error, size_t capacity) {
  // Checks in the order of read_pixels_with (context.rs:1893-1960): the
  // output length, the scene, an active job, the image kind, completed
  // samples; then the size query and the destination.
  if (!written) { setError(error, capacity, "Null pixel length output"); return MT_ERROR_INVALID_ARGUMENT; }
  *written = 0;
  auto c = findContext(handle);
  if (!c) { setError(error, capacity, "unknown context"); return MT_ERROR_INVALID_HANDLE; }
  std::unique_lock<std::mutex> l(c->m, std::try_to_lock);
  if (!l) { setError(error, capacity, "context busy"); return MT_ERROR_BUSY; }
  if (!c->scene || c->failed) { setError(error, capacity, "no healthy committed scene"); return MT_ERROR_INVALID_STATE; }
  if (activeJob(*c)) { setError(error, capacity, "active render job"); return MT_ERROR_INVALID_STATE; }
  if (kind > MT_IMAGE_ALBEDO) { setError(error, capacity, "Unknown image kind"); return MT_ERROR_INVALID_ARGUMENT; }
  if (c->samples == 0) { setError(error, capacity, "no completed samples"); return MT_ERROR_INVALID_STATE; }
  size_t px = size_t(c->scene->width) * c->scene->height;
  size_t need = px * 16;
  *written = need;
  if (!pixels && size == 0) return MT_OK;
  if (!pixels) { setError(error, capacity, "Null pixel destination"); return MT_ERROR_INVALID_ARGUMENT; }
  if (size < need) { setError(error, capacity, "destination too small"); return MT_ERROR_BUFFER_TOO_SMALL; }
  // read_average (native/host/src/lib.rs:343-364): every value divided by the
  // completed sample count on the device, then one copy to the caller; a
  // non-finite value fails the read and marks the context failed.
  SceneResources &r = *c->scene;
  const void *buf = kind == MT_IMAGE_HDR ? r.color.ptr : kind == MT_IMAGE_NORMAL ? r.normal.ptr : r.albedo.ptr;
  cudaError_t e = r.average.reserve(need);
  if (e == cudaSuccess) e = r.flag.reserve(4);
  if (e != cudaSuccess) return failContext(*c, e, error, capacity);
  uint32_t nonFinite = 0;
  int32_t st = mtc_average_output(buf, uint32_t(px), c->samples, r.average.ptr, static_cast<uint32_t *>(r.flag.ptr),
                                  c->stream);
  if (st != MT_OK) { c->failed = true; setError(error, capacity, "average launch failed"); return MT_ERROR_CONTEXT_FAILED; }
  e = cudaMemcpyAsync(&nonFinite, r.flag.ptr, 4, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return failContext(*c, e, error, capacity);
  if (nonFinite) {
    c->failed = true;
    setError(error, capacity, "Non-finite native output");
    return MT_ERROR_CONTEXT_FAILED;
  }
  e = cudaMemcpyAsync(pixels, r.average.ptr, need, cudaMemcpyDeviceToHost, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return failContext(*c, e, error, capacity);
  return MT_OK;
}

int32_t mt_context_submit(mt_context handle, uint32_t additional, mt_render_job *job, char *error, size_t capacity) {
  auto c = findContext(handle);
  if (!c) { setError(error, capacity, "unknown context"); return MT_ERROR_INVALID_HANDLE; }
  if (!job) { setError(error, capacity, "job is NULL"); return MT_ERROR_INVALID_ARGUMENT; }
  std::unique_lock<std::mutex> l(c->m, std::try_to_lock);
  if (!l) { setError(error, capacity, "context busy"); return MT_ERROR_BUSY; }
  if (!c->scene || c->failed) { setError(error, capacity, "no healthy committed scene"); return MT_ERROR_INVALID_STATE; }
  if (activeJob(*c)) { setError(error, capacity, "active render job"); return MT_ERROR_INVALID_STATE; }
  if (additional == 0 || uint64_t(c->samples) + additional > 16384u) {
    setError(error, capacity, "render total must stay within 1..16384 samples");
    return MT_ERROR_INVALID_ARGUMENT;
  }
  expireJob(*c);
  auto j = std::make_unique<Job>();
  j->requested = additional;
  j->base = c->samples;
  {
    std::lock_guard<std::mutex> g(gRegistry);
    j->handle = gNextHandle++;
    gJobs[j->handle] = c->handle;
  }
  *job = j->handle;
  c->job = std::move(j);
  return MT_OK;
}

static std::shared_ptr<Context> contextOfJob(uint64_t job) {
  std::lock_guard<std::mutex> g(gRegistry);
  auto it = gJobs.find(job);
  if (it == gJobs.end()) return nullptr;
  auto c = gContexts.find(it->second);
  return c == gContexts.end() ? nullptr : c->second;
}

int32_t mt_job_poll(mt_render_job handle, uint32_t max_new_samples, char *error, size_t capacity) {
  auto c = contextOfJob(handle);
  if (!c) { setError(error, capacity, "unknown or expired job"); return MT_ERROR_INVALID_HANDLE; }
  if (max_new_samples > 64) { setError(error, capacity, "max_new_samples must be 0..64"); return MT_ERROR_INVALID_ARGUMENT; }
  std::unique_lock<std::mutex> l(c->m, std::try_to_lock);
  if (!l) { setError(error, capacity, "context busy"); return MT_ERROR_BUSY; }
  Job *j = c->job.get();
  if (!j || j->handle != handle) { setError(error, capacity, "unknown or expired job"); return MT_ERROR_INVALID_HANDLE; }
  if (j->inflight) {
    cudaError_t e = cudaEventQuery(c->event);
    if (e == cudaErrorNotReady) return MT_OK;
    if (e != cudaSuccess) {
      j->state = MT_JOB_FAILED;
      j->inflight = 0;
      return failContext(*c, e, error, capacity);
    }
    if (j->wavefront) {
      // The batch has finished; its run drained every queue unless the
      // iteration limit stopped it.
      mtc_stream_config cfg = streamConfig(size_t(c->scene->width) * c->scene->height);
      int32_t st = mtc_stream_status(c->scene->stream.ptr, 1, &cfg, c->stream);
      if (st != MT_OK) {
        j->state = MT_JOB_FAILED;
        j->inflight = 0;
        c->failed = true;
        setError(error, capacity, "render batch did not complete");
        return MT_ERROR_CONTEXT_FAILED;
      }
    }
    j->completed += j->inflight;
    c->samples += j->inflight;
    j->inflight = 0;
  }
  if (j->completed >= j->requested) { j->state = MT_JOB_COMPLETE; return MT_OK; }
  if (j->state == MT_JOB_CANCELLING || j->state == MT_JOB_CANCELLED) { j->state = MT_JOB_CANCELLED; return MT_OK; }
  if (max_new_samples == 0) return MT_OK;
  uint32_t n = std::min(max_new_samples, j->requested - j->submitted);
  int32_t st = renderSamples(*c, n, false, &j->wavefront);
  if (st != MT_OK) { j->state = MT_JOB_FAILED; setError(error, capacity, "launch rejected"); return st; }
  cudaError_t e = cudaEventRecord(c->event, c->stream);
  if (e != cudaSuccess) { j->state = MT_JOB_FAILED; return failContext(*c, e, error, capacity); }
  j->submitted += n;
  j->inflight = n;
  j->state = MT_JOB_RUNNING;
  return MT_OK;
}

int32_t mt_job_info(mt_render_job handle, mt_job_snapshot *info, char *error, size_t capacity) {
  auto c = contextOfJob(handle);
  if (!c) { setError(error, capacity, "unknown or expired job"); return MT_ERROR_INVALID_HANDLE; }
  if (!info || info->struct_size != sizeof(mt_job_snapshot)) { setError(error, capacity, "struct_size"); return MT_ERROR_INVALID_ARGUMENT; }
  std::unique_lock<std::mutex> l(c->m, std::try_to_lock);
  if (!l) { setError(error, capacity, "context busy"); return MT_ERROR_BUSY; }
  Job *j = c->job.get();
  if (!j || j->handle != handle) { setError(error, capacity, "unknown or expired job"); return MT_ERROR_INVALID_HANDLE; }
  info->state = j->state;
  info->requested_samples = j->requested;
  info->submitted_samples = j->submitted;
  info->completed_samples = j->completed;
  info->base_samples = j->base;
  return MT_OK;
}

int32_t mt_job_cancel(mt_render_job handle, char *error, size_t capacity) {
  auto c = contextOfJob(handle);
  if (!c) { setError(error, capacity, "unknown or expired job"); return MT_ERROR_INVALID_HANDLE; }
  std::unique_lock<std::mutex> l(c->m, std::try_to_lock);
  if (!l) { setError(error, capacity, "context busy"); return MT_ERROR_BUSY; }
  Job *j = c->job.get();
  if (!j || j->handle != handle) { setError(error, capacity, "unknown or expired job"); return MT_ERROR_INVALID_HANDLE; }
  if (j->state == MT_JOB_COMPLETE || j->state == MT_JOB_CANCELLED || j->state == MT_JOB_FAILED) return MT_OK;
  j->state = j->inflight ? MT_JOB_CANCELLING : MT_JOB_CANCELLED;
  return MT_OK;
}

// mutracer-debug.h:24-25 (native/host/src/scene.rs:2506-2547), debug and
// validation only: commits the descriptor into a fresh context with the
// default settings (Sobol, seed 12345, 6 bounces), renders `samples`
// samples, and writes render.rgba32f, normal.rgba32f, albedo.rgba32f,
// render.png and result.json into output_directory (created if missing).
int32_t mt_probe_render_scene(const uint8_t *input, size_t length, const char *output_directory, uint32_t samples,
                              char *error, size_t capacity) {
  if (!input || !output_directory) {
    setError(error, capacity, "Null scene input or oversized descriptor");
    return MT_ERROR_INVALID_ARGUMENT;
  }
  if (samples == 0 || samples > 16384) { setError(error, capacity, "Samples must be 1..16384"); return MT_ERROR_INVALID_ARGUMENT; }
  std::unique_lock<std::mutex> l(gProbe, std::try_to_lock);
  if (!l) { setError(error, capacity, "Native probe is already active"); return MT_ERROR_BUSY; }
  mt_context ctx = 0;
  int32_t st = mt_context_create_with_backend(MT_BACKEND_SOFTWARE, &ctx, error, capacity);
  if (st != MT_OK) return st;
  struct Destroy {
    mt_context h;
    ~Destroy() { mt_context_destroy(h, nullptr, 0); }
  } destroy{ctx};
  if ((st = mt_context_commit(ctx, input, length, error, capacity)) != MT_OK) return st;
  if ((st = mt_context_render(ctx, samples, error, capacity)) != MT_OK) return st;
  mt_context_snapshot info;
  info.struct_size = sizeof(info);
  if ((st = mt_context_info(ctx, &info, error, capacity)) != MT_OK) return st;
  const std::string dir(output_directory);
  if (!makeDirectories(dir)) { setError(error, capacity, "cannot create the output directory"); return MT_ERROR; }
  const size_t n = size_t(info.width) * info.height * 4;
  std::vector<float> image(n);
  const char *names[] = {"render", "normal", "albedo"};
  double lo = INFINITY, hi = -INFINITY, mean = 0.0;
  std::vector<uint8_t> rgb;
  for (uint32_t kind = MT_IMAGE_HDR; kind <= MT_IMAGE_ALBEDO; kind++) {
    size_t written = 0;
    if ((st = mt_context_read_pixels(ctx, kind, image.data(), n * 4, &written, error, capacity)) != MT_OK) return st;
    if (!writeFile(dir + "/" + names[kind] + ".rgba32f", image.data(), n * 4)) {
      setError(error, capacity, "cannot write the output files");
      return MT_ERROR;
    }
    if (kind != MT_IMAGE_HDR) continue;
    rgb.resize(size_t(info.width) * info.height * 3);
    for (size_t p = 0; p < size_t(info.width) * info.height; p++) {
      // Preview only: Reinhard plus sRGB, rows flipped to top-first.
      size_t y = p / info.width, x = p % info.width, out = ((info.height - 1 - y) * info.width + x) * 3;
      for (int ch = 0; ch < 3; ch++) {
        float v = image[p * 4 + ch];
        lo = std::min<double>(lo, v);
        hi = std::max<double>(hi, v);
        mean += v;
        float linear = std::max(v, 0.0f) / (1.0f + std::max(v, 0.0f));
        float srgb = linear <= 0.0031308f ? 12.92f * linear : 1.055f * std::pow(linear, 1.0f / 2.4f) - 0.055f;
        rgb[out + ch] = uint8_t(std::min(std::max(srgb, 0.0f), 1.0f) * 255.0f + 0.5f);
      }
    }
  }
  std::vector<uint8_t> png = encodePng(rgb, info.width, info.height);
  char json[1024];
  int len = std::snprintf(json, sizeof(json),
                          "{\n  \"width\": %u,\n  \"height\": %u,\n  \"samples\": %u,\n"
                          "  \"intersectionBackend\": \"software BVH\",\n  \"rgbMin\": %.9g,\n"
                          "  \"rgbMax\": %.9g,\n  \"rgbMean\": %.9g,\n"
                          "  \"hdrLayout\": \"little-endian f32 RGBA, bottom row first; linear sample average\"\n}\n",
                          info.width, info.height, samples, lo, hi,
                          mean / (double(info.width) * info.height * 3.0));
  if (!writeFile(dir + "/render.png", png.data(), png.size()) || !writeFile(dir + "/result.json", json, size_t(len))) {
    setError(error, capacity, "cannot write the output files");
    return MT_ERROR;
  }
  return MT_OK;
}

}  // extern "C"
