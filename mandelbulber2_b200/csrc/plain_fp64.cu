// plain_fp64.cu - plain FP64 kernel (one thread per pixel), FMA contraction on.
#include "plain_kernel.cuh"

namespace mbr {
int launch_plain_fp64(const DevScene &sc, const DevFrame &fr, const DevOutputs &out, void *stream) {
  return launch_plain_t<double, double, 0>(sc, fr, out, stream);
}
int launch_distance_fp64(const DevScene &sc, const double *pts, int64_t n, double detail, int normal_mode,
                         double *dist, int32_t *iters, void *stream) {
  return launch_distance_t<double, 0>(sc, pts, n, detail, normal_mode, dist, iters, stream);
}
}  // namespace mbr
