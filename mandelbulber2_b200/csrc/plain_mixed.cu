// plain_mixed.cu - one thread per pixel; FP32 formula iteration and march
// step, FP64 ray origin, accumulated t and hit refinement.
#include "plain_kernel.cuh"

namespace mbr {
int launch_plain_mixed(const DevScene &sc, const DevFrame &fr, const DevOutputs &out, void *stream) {
  return launch_plain_t<float, double, 2>(sc, fr, out, stream);
}
int launch_distance_fp32(const DevScene &sc, const double *pts, int64_t n, double detail, int normal_mode,
                         double *dist, int32_t *iters, void *stream) {
  return launch_distance_t<float, 2>(sc, pts, n, detail, normal_mode, dist, iters, stream);
}
}  // namespace mbr
