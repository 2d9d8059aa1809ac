// plain_fp64_strict.cu - the plain FP64 kernel compiled with --fmad=false:
// every double operation is a separately rounded IEEE operation, in the
// order the reference's CPU code performs them.
#include "plain_kernel.cuh"

namespace mbr {
int launch_plain_fp64_strict(const DevScene &sc, const DevFrame &fr, const DevOutputs &out, void *stream) {
  return launch_plain_t<double, double, 1>(sc, fr, out, stream);
}
int launch_distance_fp64_strict(const DevScene &sc, const double *pts, int64_t n, double detail, int normal_mode,
                                double *dist, int32_t *iters, void *stream) {
  return launch_distance_t<double, 1>(sc, pts, n, detail, normal_mode, dist, iters, stream);
}
}  // namespace mbr
