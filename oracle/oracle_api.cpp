// Test infrastructure only (the checker, never the product).
//
// C entry points of the CPU oracle, loaded by tests/ (ctypes) and by the
// cpu_baseline / reference arm of bench.py.  Host pointers everywhere; the
// scene is described by the same mtc_scene_view struct the CUDA path takes.
#include <atomic>
#include <thread>
#include <vector>
#include "oracle_bsdf.h"

using namespace oracle;

static Scene makeScene(const mtc_scene_view *sv, const mtc_trace_uniform *u, const mtc_camera_uniform *cam) {
  Scene s;
  s.bvh = (const V4 *)sv->bvh;
  s.ins = (const V4 *)sv->instances;
  s.attr = (const u32 *)sv->attributes;
  s.mats = (const V4 *)sv->materials;
  s.env = (const V4 *)sv->env_map;
  s.envDist = (const float *)sv->env_distribution;
  s.envW = sv->env_width;
  s.envH = sv->env_height;
  s.lightData = (const V4 *)sv->light_sampling;
  s.lut = (const float *)sv->energy_lut;
  s.lights = (const V4 *)sv->analytic_lights;
  s.vl = sv->vertex_layout;
  s.maps = (const V4 *)sv->maps;
  s.mapTexels = (const V4 *)sv->map_texels;
  s.mapCount = sv->maps && sv->map_texels ? sv->map_count : 0;
  s.mapTexelCount = sv->map_texel_count;
  s.triMats = sv->triangle_materials;
  s.matCount = sv->material_count;
  s.flags = sv->flags;
  s.tlasStack = sv->tlas_stack_size;
  s.blasStack = sv->blas_stack_size;
  s.u = u;
  s.cam = cam;
  return s;
}

template <class F>
static void parallelFor(uint32_t n, int threads, F f) {
  if (threads <= 1 || n < 2) {
    for (uint32_t i = 0; i < n; i++) f(i, 0);
    return;
  }
  std::atomic<uint32_t> next{0};
  std::vector<std::thread> pool;
  for (int t = 0; t < threads; t++) {
    pool.emplace_back([&, t] {
      for (;;) {
        uint32_t i = next.fetch_add(1);
        if (i >= n) break;
        f(i, t);
      }
    });
  }
  for (auto &th : pool) th.join();
}

extern "C" {

// querySceneSoftware over `count` rays of 8 floats (o.xyz, pad, d.xyz, pad).
int oracle_query_first_hit(const mtc_scene_view *sv, const mtc_trace_uniform *u, const float *rays,
                           uint32_t count, mtc_hit *hits, int threads) {
  Scene s = makeScene(sv, u, nullptr);
  const uint32_t chunk = 4096;
  uint32_t chunks = (count + chunk - 1) / chunk;
  parallelFor(chunks, threads, [&](uint32_t c, int) {
    uint32_t end = std::min(count, (c + 1) * chunk);
    for (uint32_t i = c * chunk; i < end; i++) {
      const float *r = rays + size_t(i) * 8;
      Ray ray{{r[0], r[1], r[2]}, {r[4], r[5], r[6]}};
      FirstHit h = querySceneSoftware(s, ray, nullptr);
      hits[i].hit = h.hit ? 1 : 0;
      hits[i].instance = h.instance;
      hits[i].record = h.record;
      hits[i].t = h.t;
      hits[i].barycentric[0] = h.bary.x;
      hits[i].barycentric[1] = h.bary.y;
      hits[i].barycentric[2] = h.bary.z;
      hits[i]._pad = 0.0f;
    }
  });
  return 0;
}

// `samples` progressive passes over rows [row_begin, row_end) (row_end = 0
// means the full image).  traffic_out (may be NULL) receives 8 u64 counters:
// box tests, primitive records, triangle tests, instance visits, material
// fetches, path samples, extension rays, shadow rays.
int oracle_trace_samples(const mtc_scene_view *sv, const mtc_camera_uniform *cam, const mtc_trace_uniform *u,
                         float *color, float *normal, float *albedo, float *catcher, uint32_t samples,
                         uint32_t row_begin, uint32_t row_end, int threads, uint64_t *traffic_out) {
  Scene s = makeScene(sv, u, cam);
  uint32_t W = uint32_t(u->output_size[0]), H = uint32_t(u->output_size[1]);
  if (row_end == 0 || row_end > H) row_end = H;
  if (row_begin >= row_end) return 0;
  int nt = std::max(threads, 1);
  std::vector<Traffic> traffic(static_cast<size_t>(nt));
  for (uint32_t sample = 0; sample < samples; sample++) {
    parallelFor(row_end - row_begin, nt, [&](uint32_t r, int t) {
      uint32_t y = row_begin + r;
      for (uint32_t x = 0; x < W; x++)
        tracePixel(s, x, y, (V4 *)color, (V4 *)normal, (V4 *)albedo, (V4 *)catcher, traffic_out ? &traffic[t] : nullptr);
    });
  }
  if (traffic_out) {
    Traffic total;
    for (auto &t : traffic) total.add(t);
    traffic_out[0] = total.box_tests; traffic_out[1] = total.prim_records; traffic_out[2] = total.tri_tests;
    traffic_out[3] = total.instance_visits; traffic_out[4] = total.material_fetches; traffic_out[5] = total.paths;
    traffic_out[6] = total.extension_rays; traffic_out[7] = total.shadow_rays;
  }
  return 0;
}

// Raw sampleMap lookups (materialBuffer.wgsl.ts:335-378) over a scene's maps:
// out[4i..4i+3] for map indices[i] at uvs[2i..2i+1].
void oracle_sample_maps(const mtc_scene_view *sv, const int32_t *indices, const float *uvs, uint32_t count,
                        float *out) {
  Scene s = makeScene(sv, nullptr, nullptr);
  for (uint32_t i = 0; i < count; i++) {
    V4 t = sampleMap(s, indices[i], {uvs[2 * i], uvs[2 * i + 1]});
    out[4 * i] = t.x; out[4 * i + 1] = t.y; out[4 * i + 2] = t.z; out[4 * i + 3] = t.w;
  }
}

// Sampler primitives for the golden tests (sobol.wgsl.ts).
uint32_t oracle_sample_hash(uint32_t x) { return sampleHash(x); }
uint32_t oracle_sample_seed(uint32_t a, uint32_t b) { return sampleSeed(a, b); }
uint32_t oracle_owen(uint32_t x, uint32_t seed) { return owen(x, seed); }
uint32_t oracle_sobol_d1(uint32_t v) { return sobolD1(v); }
uint32_t oracle_reverse_bits(uint32_t v) { return reverseBits(v); }
uint32_t oracle_zsobol_index(uint32_t morton, uint32_t dim, uint32_t log) { return zSobolIndex(morton, dim, log); }
uint32_t oracle_morton2(uint32_t x, uint32_t y) { return morton2(x, y); }
// Structured 2D sample for (pixel, sample index, dimension), in [EPS, 1-EPS].
void oracle_structured_sample(uint32_t px, uint32_t py, uint32_t width, uint32_t index, uint32_t dim, uint32_t seed,
                              int pattern, uint32_t logspp, float *out) {
  Sampler smp;
  smp.px = px; smp.py = py; smp.width = width; smp.index = index; smp.seed = seed; smp.pattern = pattern;
  smp.logspp = logspp;
  V2 v = smp.structured(dim);
  out[0] = v.x;
  out[1] = v.y;
}

}  // extern "C"
