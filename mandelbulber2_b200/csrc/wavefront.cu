// wavefront.cu - placeholder until the persistent wavefront kernel lands.
#include "mbr_internal.h"

namespace mbr {
mbr_status render_wavefront(mbr_ctx *ctx, const DevScene &, const DevFrame &, const DevOutputs &, int, void *) {
  return set_err(ctx, MBR_EUNSUPPORTED, "wavefront engine not built yet");
}
}  // namespace mbr

extern "C" {
mbr_status mbr_batch_create(mbr_ctx *ctx, const mbr_scene *, int32_t, const mbr_job *, int32_t,
                            const mbr_render_params *, const mbr_outputs *, int, void *, mbr_batch **batch) {
  if (batch) *batch = nullptr;
  return mbr::set_err(ctx, MBR_EUNSUPPORTED, "batch not built yet");
}
mbr_status mbr_batch_launch(mbr_batch *, void *) { return MBR_EUNSUPPORTED; }
void mbr_batch_destroy(mbr_batch *) {}
mbr_status mbr_autotune(mbr_ctx *ctx, const mbr_camera *, const mbr_render_params *, const mbr_outputs *, int, void *,
                        mbr_tuning *) {
  return mbr::set_err(ctx, MBR_EUNSUPPORTED, "autotune not built yet");
}
mbr_status mbr_adjoint(mbr_ctx *ctx, const mbr_camera *, const mbr_render_params *, const double *, const uint8_t *,
                       const float *, const float *, double *, int, void *) {
  return mbr::set_err(ctx, MBR_EUNSUPPORTED, "adjoint not built yet");
}
}
