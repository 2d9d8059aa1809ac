// mbr_internal.h - host-side helpers shared by the library's translation units.
#pragma once
#include <string>

#include "../../include/mbr.h"
#include "mbr_device.h"

namespace mbr {

mbr_status set_err(mbr_ctx *ctx, mbr_status st, const char *fmt, ...);
mbr_status cuda_err(mbr_ctx *ctx, int code, const char *what);
mbr_status build_scene(mbr_ctx *ctx, const mbr_scene &sc, DevScene *out);
// The gamma table, when it changes, is copied on `stream`.
mbr_status build_frame(mbr_ctx *ctx, const mbr_camera &cam, const mbr_render_params &p, DevFrame *out, void *stream);
mbr_status validate_camera(mbr_ctx *ctx, const mbr_camera &cam);
void camera_matrix(const mbr_camera &cam, double mrot[9], bool *zero, double angles[3]);
DevOutputs dev_outputs(mbr_ctx *ctx, const mbr_outputs &o);
mbr_status build_frame_owned_gamma(const mbr_camera &cam, const mbr_render_params &p, uint16_t *gamma_dev,
                                   uint16_t *gamma_host, double *gamma_value, DevFrame *out, void *stream,
                                   std::string *err);
const DevScene *ctx_scene(mbr_ctx *ctx);
int ctx_device(mbr_ctx *ctx);
const mbr_scene *ctx_scene_src(mbr_ctx *ctx);
mbr_tuning &ctx_tuning(mbr_ctx *ctx);
int32_t *ctx_status(mbr_ctx *ctx);
mbr_status ctx_work(mbr_ctx *ctx, size_t words, unsigned long long **out);
// Device buffer of the adjoint's per-block partial sums, grown on demand.
mbr_status ctx_adjoint_partials(mbr_ctx *ctx, size_t bytes, double **out);

// wavefront.cu
mbr_status render_wavefront(mbr_ctx *ctx, const DevScene &sc, const DevFrame &fr, const DevOutputs &out, int engine,
                            void *stream);

}  // namespace mbr
