/* Node-API addon over libmutracer_b200's context API, so the reference's
 * TypeScript Engine / RenderLoop (Render.converge, src/Render.ts:827-900) can
 * drive the CUDA path.  The functions mirror native/include/mutracer-context.h
 * one to one; every failing call throws an Error whose `code` property is the
 * mt_status value and whose message is the library's error text.
 *
 *   const mt = require('./build/Release/mutracer_b200.node');
 *   const ctx = mt.create();                       // or mt.createWithBackend(0)
 *   mt.commit(ctx, descriptorBytes);               // Uint8Array, scene descriptor v8
 *   mt.render(ctx, 64);
 *   const hdr = mt.readPixels(ctx, mt.IMAGE_HDR);   // Float32Array, RGBA, bottom row first
 *   const job = mt.submit(ctx, 256);
 *   while (mt.jobInfo(job).state !== mt.JOB_COMPLETE) mt.jobPoll(job, 8);
 *   mt.destroy(ctx);
 *
 * Context and job handles are u64 values returned as BigInt.  Render settings
 * are a plain object whose keys are the mt_render_settings field names
 * (camelCase); missing keys keep mt_render_settings_default's values.
 *
 * Build: node-gyp configure build (binding.gyp beside this file), with
 * libmutracer_b200.so and include/mutracer_b200.h of this repository. */
#include <node_api.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "mutracer_b200.h"

#define ERROR_CAPACITY 1024

/* Throws an Error carrying the status in `code`; returns NULL for the
 * caller to return. */
static napi_value throw_status(napi_env env, int32_t status, const char *message) {
  char code[16];
  snprintf(code, sizeof code, "%d", (int)status);
  napi_throw_error(env, code, message && message[0] ? message : "mutracer_b200 call failed");
  return NULL;
}

#define CHECK_NAPI(call)                                            \
  do {                                                              \
    if ((call) != napi_ok) {                                        \
      napi_throw_error(env, NULL, "invalid arguments: " #call);     \
      return NULL;                                                  \
    }                                                               \
  } while (0)

static int get_args(napi_env env, napi_callback_info info, size_t expected, napi_value *argv) {
  size_t argc = expected;
  if (napi_get_cb_info(env, info, &argc, argv, NULL, NULL) != napi_ok || argc < expected) {
    napi_throw_type_error(env, NULL, "missing arguments");
    return 0;
  }
  return 1;
}

static int get_handle(napi_env env, napi_value value, uint64_t *out) {
  bool lossless = false;
  if (napi_get_value_bigint_uint64(env, value, out, &lossless) == napi_ok && lossless) return 1;
  napi_throw_type_error(env, NULL, "handle must be a BigInt returned by this addon");
  return 0;
}

static napi_value make_handle(napi_env env, uint64_t handle) {
  napi_value out;
  CHECK_NAPI(napi_create_bigint_uint64(env, handle, &out));
  return out;
}

static napi_value make_u32(napi_env env, uint32_t v) {
  napi_value out;
  CHECK_NAPI(napi_create_uint32(env, v, &out));
  return out;
}

static napi_value undefined_value(napi_env env) {
  napi_value out;
  CHECK_NAPI(napi_get_undefined(env, &out));
  return out;
}

/* create() / createWithBackend(backend) -> BigInt */
static napi_value Create(napi_env env, napi_callback_info info) {
  (void)info;
  char err[ERROR_CAPACITY] = {0};
  mt_context handle = 0;
  int32_t st = mt_context_create(&handle, err, sizeof err);
  if (st != MT_OK) return throw_status(env, st, err);
  return make_handle(env, handle);
}

static napi_value CreateWithBackend(napi_env env, napi_callback_info info) {
  napi_value argv[1];
  if (!get_args(env, info, 1, argv)) return NULL;
  uint32_t backend = 0;
  CHECK_NAPI(napi_get_value_uint32(env, argv[0], &backend));
  char err[ERROR_CAPACITY] = {0};
  mt_context handle = 0;
  int32_t st = mt_context_create_with_backend(backend, &handle, err, sizeof err);
  if (st != MT_OK) return throw_status(env, st, err);
  return make_handle(env, handle);
}

/* backend(ctx) -> {active, reason} */
static napi_value Backend(napi_env env, napi_callback_info info) {
  napi_value argv[1];
  if (!get_args(env, info, 1, argv)) return NULL;
  uint64_t handle;
  if (!get_handle(env, argv[0], &handle)) return NULL;
  char err[ERROR_CAPACITY] = {0}, reason[512] = {0};
  uint32_t active = 0;
  int32_t st = mt_context_backend(handle, &active, reason, sizeof reason, err, sizeof err);
  if (st != MT_OK) return throw_status(env, st, err);
  napi_value out, r;
  CHECK_NAPI(napi_create_object(env, &out));
  CHECK_NAPI(napi_set_named_property(env, out, "active", make_u32(env, active)));
  CHECK_NAPI(napi_create_string_utf8(env, reason, NAPI_AUTO_LENGTH, &r));
  CHECK_NAPI(napi_set_named_property(env, out, "reason", r));
  return out;
}

/* Calls taking only the context handle: destroy, reset, cancelCommit. */
typedef int32_t (*context_call)(mt_context, char *, size_t);
static napi_value call_context(napi_env env, napi_callback_info info, context_call fn) {
  napi_value argv[1];
  if (!get_args(env, info, 1, argv)) return NULL;
  uint64_t handle;
  if (!get_handle(env, argv[0], &handle)) return NULL;
  char err[ERROR_CAPACITY] = {0};
  int32_t st = fn(handle, err, sizeof err);
  if (st != MT_OK) return throw_status(env, st, err);
  return undefined_value(env);
}
static napi_value Destroy(napi_env env, napi_callback_info info) {
  return call_context(env, info, mt_context_destroy);
}
static napi_value Reset(napi_env env, napi_callback_info info) { return call_context(env, info, mt_context_reset); }
static napi_value CancelCommit(napi_env env, napi_callback_info info) {
  return call_context(env, info, mt_context_cancel_commit);
}

/* Reads optional numeric keys of a settings object into mt_render_settings. */
static int read_settings(napi_env env, napi_value object, mt_render_settings *s) {
  mt_render_settings_default(s);
  struct { const char *key; uint32_t *field; } u32s[] = {
      {"samplingPattern", &s->sampling_pattern}, {"seed", &s->seed}, {"maxSamples", &s->max_samples},
      {"bounces", &s->bounces}, {"directLightCandidates", &s->direct_light_candidates},
      {"bevelSamples", &s->bevel_samples}, {"sampleSequenceOffset", &s->sample_sequence_offset},
      {"causticFlags", &s->caustic_flags}, {"lightPhotons", &s->light_photons},
      {"photonMapPhotons", &s->photon_map_photons}};
  struct { const char *key; double *field; } f64s[] = {
      {"clamping", &s->clamping}, {"transmissiveOutputAlphaMin", &s->transmissive_output_alpha_min}};
  for (size_t i = 0; i < sizeof u32s / sizeof u32s[0]; i++) {
    bool has = false;
    napi_value v;
    if (napi_has_named_property(env, object, u32s[i].key, &has) != napi_ok) return 0;
    if (!has) continue;
    if (napi_get_named_property(env, object, u32s[i].key, &v) != napi_ok ||
        napi_get_value_uint32(env, v, u32s[i].field) != napi_ok)
      return 0;
  }
  for (size_t i = 0; i < sizeof f64s / sizeof f64s[0]; i++) {
    bool has = false;
    napi_value v;
    if (napi_has_named_property(env, object, f64s[i].key, &has) != napi_ok) return 0;
    if (!has) continue;
    if (napi_get_named_property(env, object, f64s[i].key, &v) != napi_ok ||
        napi_get_value_double(env, v, f64s[i].field) != napi_ok)
      return 0;
  }
  bool has = false;
  if (napi_has_named_property(env, object, "photonMapRadius", &has) == napi_ok && has) {
    napi_value v;
    double r = 0.0;
    if (napi_get_named_property(env, object, "photonMapRadius", &v) != napi_ok ||
        napi_get_value_double(env, v, &r) != napi_ok)
      return 0;
    s->photon_map_radius = (float)r;
  }
  return 1;
}

/* commit(ctx, Uint8Array[, settings]) */
static napi_value Commit(napi_env env, napi_callback_info info) {
  size_t argc = 3;
  napi_value argv[3];
  CHECK_NAPI(napi_get_cb_info(env, info, &argc, argv, NULL, NULL));
  if (argc < 2) return throw_status(env, MT_ERROR_INVALID_ARGUMENT, "commit(ctx, bytes[, settings])");
  uint64_t handle;
  if (!get_handle(env, argv[0], &handle)) return NULL;
  napi_typedarray_type type;
  size_t length = 0, offset = 0;
  void *data = NULL;
  napi_value buffer;
  CHECK_NAPI(napi_get_typedarray_info(env, argv[1], &type, &length, &data, &buffer, &offset));
  if (type != napi_uint8_array) return throw_status(env, MT_ERROR_INVALID_ARGUMENT, "descriptor must be a Uint8Array");
  char err[ERROR_CAPACITY] = {0};
  int32_t st;
  napi_valuetype t = napi_undefined;
  if (argc >= 3) CHECK_NAPI(napi_typeof(env, argv[2], &t));
  if (t == napi_object) {
    mt_render_settings settings;
    if (!read_settings(env, argv[2], &settings)) return throw_status(env, MT_ERROR_INVALID_ARGUMENT, "settings");
    st = mt_context_commit_with_settings(handle, (const uint8_t *)data, length, &settings, err, sizeof err);
  } else {
    st = mt_context_commit(handle, (const uint8_t *)data, length, err, sizeof err);
  }
  if (st != MT_OK) return throw_status(env, st, err);
  return undefined_value(env);
}

/* Calls taking the context handle and one u32: render, wait. */
typedef int32_t (*context_u32_call)(mt_context, uint32_t, char *, size_t);
static napi_value call_context_u32(napi_env env, napi_callback_info info, context_u32_call fn) {
  napi_value argv[2];
  if (!get_args(env, info, 2, argv)) return NULL;
  uint64_t handle;
  if (!get_handle(env, argv[0], &handle)) return NULL;
  uint32_t value = 0;
  CHECK_NAPI(napi_get_value_uint32(env, argv[1], &value));
  char err[ERROR_CAPACITY] = {0};
  int32_t st = fn(handle, value, err, sizeof err);
  if (st != MT_OK) return throw_status(env, st, err);
  return undefined_value(env);
}
static napi_value Render(napi_env env, napi_callback_info info) {
  return call_context_u32(env, info, mt_context_render);
}
static napi_value Wait(napi_env env, napi_callback_info info) { return call_context_u32(env, info, mt_context_wait); }

/* info(ctx) -> {width, height, samples, state, lastCommit} */
static napi_value Info(napi_env env, napi_callback_info info) {
  napi_value argv[1];
  if (!get_args(env, info, 1, argv)) return NULL;
  uint64_t handle;
  if (!get_handle(env, argv[0], &handle)) return NULL;
  mt_context_snapshot s;
  memset(&s, 0, sizeof s);
  s.struct_size = sizeof s;
  char err[ERROR_CAPACITY] = {0};
  int32_t st = mt_context_info(handle, &s, err, sizeof err);
  if (st != MT_OK) return throw_status(env, st, err);
  napi_value out;
  CHECK_NAPI(napi_create_object(env, &out));
  CHECK_NAPI(napi_set_named_property(env, out, "width", make_u32(env, s.width)));
  CHECK_NAPI(napi_set_named_property(env, out, "height", make_u32(env, s.height)));
  CHECK_NAPI(napi_set_named_property(env, out, "samples", make_u32(env, s.samples)));
  CHECK_NAPI(napi_set_named_property(env, out, "state", make_u32(env, s.state)));
  CHECK_NAPI(napi_set_named_property(env, out, "lastCommit", make_u32(env, s.last_commit)));
  return out;
}

/* readPixels(ctx, kind) -> Float32Array (RGBA, bottom row first) */
static napi_value ReadPixels(napi_env env, napi_callback_info info) {
  napi_value argv[2];
  if (!get_args(env, info, 2, argv)) return NULL;
  uint64_t handle;
  if (!get_handle(env, argv[0], &handle)) return NULL;
  uint32_t kind = 0;
  CHECK_NAPI(napi_get_value_uint32(env, argv[1], &kind));
  char err[ERROR_CAPACITY] = {0};
  size_t need = 0;
  int32_t st = mt_context_read_pixels(handle, kind, NULL, 0, &need, err, sizeof err);
  if (st != MT_OK) return throw_status(env, st, err);
  void *data = NULL;
  napi_value buffer, array;
  CHECK_NAPI(napi_create_arraybuffer(env, need, &data, &buffer));
  st = mt_context_read_pixels(handle, kind, data, need, &need, err, sizeof err);
  if (st != MT_OK) return throw_status(env, st, err);
  CHECK_NAPI(napi_create_typedarray(env, napi_float32_array, need / 4, buffer, 0, &array));
  return array;
}

/* submit(ctx, samples) -> BigInt job */
static napi_value Submit(napi_env env, napi_callback_info info) {
  napi_value argv[2];
  if (!get_args(env, info, 2, argv)) return NULL;
  uint64_t handle;
  if (!get_handle(env, argv[0], &handle)) return NULL;
  uint32_t samples = 0;
  CHECK_NAPI(napi_get_value_uint32(env, argv[1], &samples));
  char err[ERROR_CAPACITY] = {0};
  mt_render_job job = 0;
  int32_t st = mt_context_submit(handle, samples, &job, err, sizeof err);
  if (st != MT_OK) return throw_status(env, st, err);
  return make_handle(env, job);
}

/* jobPoll(job, maxNewSamples) */
static napi_value JobPoll(napi_env env, napi_callback_info info) {
  napi_value argv[2];
  if (!get_args(env, info, 2, argv)) return NULL;
  uint64_t job;
  if (!get_handle(env, argv[0], &job)) return NULL;
  uint32_t budget = 0;
  CHECK_NAPI(napi_get_value_uint32(env, argv[1], &budget));
  char err[ERROR_CAPACITY] = {0};
  int32_t st = mt_job_poll(job, budget, err, sizeof err);
  if (st != MT_OK) return throw_status(env, st, err);
  return undefined_value(env);
}

/* jobInfo(job) -> {state, requested, submitted, completed, base} */
static napi_value JobInfo(napi_env env, napi_callback_info info) {
  napi_value argv[1];
  if (!get_args(env, info, 1, argv)) return NULL;
  uint64_t job;
  if (!get_handle(env, argv[0], &job)) return NULL;
  mt_job_snapshot s;
  memset(&s, 0, sizeof s);
  s.struct_size = sizeof s;
  char err[ERROR_CAPACITY] = {0};
  int32_t st = mt_job_info(job, &s, err, sizeof err);
  if (st != MT_OK) return throw_status(env, st, err);
  napi_value out;
  CHECK_NAPI(napi_create_object(env, &out));
  CHECK_NAPI(napi_set_named_property(env, out, "state", make_u32(env, s.state)));
  CHECK_NAPI(napi_set_named_property(env, out, "requested", make_u32(env, s.requested_samples)));
  CHECK_NAPI(napi_set_named_property(env, out, "submitted", make_u32(env, s.submitted_samples)));
  CHECK_NAPI(napi_set_named_property(env, out, "completed", make_u32(env, s.completed_samples)));
  CHECK_NAPI(napi_set_named_property(env, out, "base", make_u32(env, s.base_samples)));
  return out;
}

/* jobCancel(job) */
static napi_value JobCancel(napi_env env, napi_callback_info info) {
  napi_value argv[1];
  if (!get_args(env, info, 1, argv)) return NULL;
  uint64_t job;
  if (!get_handle(env, argv[0], &job)) return NULL;
  char err[ERROR_CAPACITY] = {0};
  int32_t st = mt_job_cancel(job, err, sizeof err);
  if (st != MT_OK) return throw_status(env, st, err);
  return undefined_value(env);
}

static int export_function(napi_env env, napi_value exports, const char *name, napi_callback cb) {
  napi_value fn;
  return napi_create_function(env, name, NAPI_AUTO_LENGTH, cb, NULL, &fn) == napi_ok &&
         napi_set_named_property(env, exports, name, fn) == napi_ok;
}

static int export_constant(napi_env env, napi_value exports, const char *name, uint32_t value) {
  napi_value v;
  return napi_create_uint32(env, value, &v) == napi_ok && napi_set_named_property(env, exports, name, v) == napi_ok;
}

NAPI_MODULE_INIT() {
  struct { const char *name; napi_callback cb; } fns[] = {
      {"create", Create}, {"createWithBackend", CreateWithBackend}, {"backend", Backend}, {"destroy", Destroy},
      {"commit", Commit}, {"cancelCommit", CancelCommit}, {"render", Render}, {"reset", Reset}, {"wait", Wait},
      {"info", Info}, {"readPixels", ReadPixels}, {"submit", Submit}, {"jobPoll", JobPoll},
      {"jobInfo", JobInfo}, {"jobCancel", JobCancel}};
  struct { const char *name; uint32_t value; } constants[] = {
      {"IMAGE_HDR", MT_IMAGE_HDR}, {"IMAGE_NORMAL", MT_IMAGE_NORMAL}, {"IMAGE_ALBEDO", MT_IMAGE_ALBEDO},
      {"BACKEND_SOFTWARE", MT_BACKEND_SOFTWARE}, {"BACKEND_HWRT", MT_BACKEND_HWRT},
      {"JOB_QUEUED", MT_JOB_QUEUED}, {"JOB_RUNNING", MT_JOB_RUNNING}, {"JOB_COMPLETE", MT_JOB_COMPLETE},
      {"JOB_CANCELLED", MT_JOB_CANCELLED}, {"JOB_FAILED", MT_JOB_FAILED}, {"JOB_CANCELLING", MT_JOB_CANCELLING}};
  for (size_t i = 0; i < sizeof fns / sizeof fns[0]; i++)
    if (!export_function(env, exports, fns[i].name, fns[i].cb)) return NULL;
  for (size_t i = 0; i < sizeof constants / sizeof constants[0]; i++)
    if (!export_constant(env, exports, constants[i].name, constants[i].value)) return NULL;
  return exports;
}
