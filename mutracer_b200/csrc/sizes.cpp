// Struct sizes of the public C ABI, so language bindings can verify their
// mirrors of include/mutracer_b200.h at load time.
#include "../../include/mutracer_b200.h"
#include "mtp_api.h"

static_assert(sizeof(mtc_trace_uniform) == 320, "RayTraceUniform is 320 bytes");
static_assert(sizeof(mt_render_settings) == 64, "mt_render_settings layout");

extern "C" int mtc_struct_sizes(uint32_t *out, uint32_t capacity) {
  const uint32_t sizes[] = {
      uint32_t(sizeof(mtc_trace_uniform)), uint32_t(sizeof(mtc_camera_uniform)), uint32_t(sizeof(mtc_scene_view)),
      uint32_t(sizeof(mtc_outputs)),       uint32_t(sizeof(mtc_hit)),            uint32_t(sizeof(mtc_counters)),
      uint32_t(sizeof(mtc_job_desc)),      uint32_t(sizeof(mtc_batch_config)),   uint32_t(sizeof(mt_scene_bundle)),
      uint32_t(sizeof(mt_render_settings)), uint32_t(sizeof(mt_context_snapshot)), uint32_t(sizeof(mt_job_snapshot)),
      uint32_t(sizeof(mtp_scene_info_t)), uint32_t(sizeof(mtc_stream_config)),
      uint32_t(sizeof(mtc_blas_build_input)), uint32_t(sizeof(mtc_blas_build_result)),
      uint32_t(sizeof(mtc_blas_refit_plan_info))};
  uint32_t n = sizeof(sizes) / sizeof(sizes[0]);
  for (uint32_t i = 0; i < n && i < capacity; i++) out[i] = sizes[i];
  return int(n);
}
