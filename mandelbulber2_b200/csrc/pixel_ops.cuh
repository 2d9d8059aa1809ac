// pixel_ops.cuh - per-ray operations shared by the kernels: random streams,
// camera rays, the march with its hit refinement, normals, shadow and AO
// marches, the GI path and the image conversion.
//
// The march state (ray origin, direction, accumulated scan t, thresholds)
// is FP64 everywhere; T is the precision of the distance estimate of the
// march steps, R the precision of the final hit refinement.
//
// Reference semantics (mandelbulber2 file:line):
//   pixel -> image point      src/render_worker.cpp:155-163, src/region.hpp:66-71
//   CalculateViewVector       src/projection_3d.cpp:77-89
//   CalcDistThresh / CalcDelta src/render_worker.cpp:653-690
//   RayMarching               src/render_worker.cpp:708-951
//   CalculateNormals          src/shader_calculate_normals.cpp:40-125
//   LightShading              src/shader_light_shading.cpp:40-122
//   AuxShadow (hard, soft)    src/shader_aux_shadow.cpp:39-323
//   AmbientOcclusion          src/shader_ambient_occlusion.cpp:41-120
//   FastAmbientOcclusion      src/shader_fast_ambient_occlusion.cpp:40-65
//   GlobalIlumination march   src/shader_global_illumination.cpp:75-125
//   MonteCarloDOF             src/render_worker.cpp:1832-1844
//   CalculatePixel + 8 bit    src/cimage.cpp:317-375, 460-469
#pragma once
#include "de_core.cuh"

namespace mbr {

struct D3 {
  double x, y, z;
};
__device__ __forceinline__ D3 d3add(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ D3 d3sub(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ D3 d3mul(D3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
__device__ __forceinline__ double d3dot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ double d3len(D3 a) { return sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
__device__ __forceinline__ D3 d3norm(D3 a) {  // CVector3::Normalize
  const double n = 1.0 / d3len(a);
  return {a.x * n, a.y * n, a.z * n};
}
// start + dir * scan, as `in.start + in.direction * scan`
__device__ __forceinline__ D3 d3ray(D3 s, D3 d, double t) { return {s.x + d.x * t, s.y + d.y * t, s.z + d.z * t}; }

// ---- random streams ------------------------------------------------------------
// Park-Miller without divisions (src/common_math.cpp:47-72), one state per ray.
struct ParkMiller {
  unsigned int s;
  __device__ __forceinline__ int next() {
    unsigned int lo = 16807u * (s & 0xFFFFu);
    unsigned int hi = 16807u * (s >> 16);
    lo += (hi & 0x7FFFu) << 16;
    hi >>= 15;
    lo += hi;
    if (lo > 2147483647u) lo -= 2147483647u;
    s = lo;
    return int(lo);
  }
  __device__ __forceinline__ int random(int max) { return next() % (max + 1); }
};
// Per-ray seed: multiplicative hash of (ray, seed) into [1, 2^31-2], then ten
// warm-up draws.
__device__ __forceinline__ ParkMiller pm_for_ray(unsigned long long ray, unsigned int seed) {
  unsigned long long h = (ray + 1ull) * 0x9E3779B97F4A7C15ull ^ ((unsigned long long)seed * 0xC2B2AE3D27D4EB4Full);
  h ^= h >> 29;
  ParkMiller pm;
  pm.s = (unsigned int)(h % 2147483646ull) + 1u;
  for (int i = 0; i < 10; i++) pm.next();
  return pm;
}

// PCG32 (O'Neill 2014): srandom(initstate, initseq) and XSH-RR output.
struct Pcg32 {
  unsigned long long state, inc;
  __device__ __forceinline__ unsigned int next() {
    const unsigned long long old = state;
    state = old * 6364136223846793005ull + inc;
    const unsigned int xorshifted = (unsigned int)(((old >> 18u) ^ old) >> 27u);
    const unsigned int rot = (unsigned int)(old >> 59u);
    return (xorshifted >> rot) | (xorshifted << ((0u - rot) & 31u));
  }
  __device__ __forceinline__ double uniform() { return double(next() >> 8) * (1.0 / 16777216.0); }
};
__device__ __forceinline__ Pcg32 pcg_init(unsigned long long initstate, unsigned long long initseq) {
  Pcg32 p;
  p.state = 0ull;
  p.inc = (initseq << 1u) | 1u;
  p.next();
  p.state += initstate;
  p.next();
  return p;
}

// Cosine-weighted direction about unit n (Malley's method) in the
// orthonormal basis of Duff et al., "Building an Orthonormal Basis,
// Revisited" (JCGT 6(1), 2017).
__device__ __forceinline__ D3 cosine_dir(D3 n, double u1, double u2) {
  const double r = sqrt(u1);
  const double phi = 2.0 * 3.14159265358979323846 * u2;
  double sp, cp;
  sincos(phi, &sp, &cp);
  const double lx = r * cp, ly = r * sp;
  const double lz = sqrt(fmax(0.0, 1.0 - u1));
  const double sign = n.z >= 0.0 ? 1.0 : -1.0;
  const double a = -1.0 / (sign + n.z);
  const double b = n.x * n.y * a;
  const D3 t{1.0 + sign * n.x * n.x * a, sign * b, -sign * n.x};
  const D3 bb{b, sign + n.y * n.y * a, -n.y};
  return {t.x * lx + bb.x * ly + n.x * lz, t.y * lx + bb.y * ly + n.y * lz, t.z * lx + bb.z * ly + n.z * lz};
}

// ---- frame helpers ---------------------------------------------------------------
__device__ __forceinline__ D3 rotate(const DevFrame &fr, D3 v) {  // CRotationMatrix::RotateVector
  if (fr.mrot_zero) return v;
  const double *m = fr.mrot;
  return {m[0] * v.x + m[1] * v.y + m[2] * v.z, m[3] * v.x + m[4] * v.y + m[5] * v.z,
          m[6] * v.x + m[7] * v.y + m[8] * v.z};
}
// cRegion::transpose from the screen to the image region (region.hpp:66-71):
// (-0.5, 0.5, 0.5, -0.5), or (-0.5, -0.5, 0.5, 0.5) in the legacy coordinate
// system (render_job.cpp:308-315)
__device__ __forceinline__ void image_point(const DevFrame &fr, double x, double y, double *ix, double *iy) {
  const double scaleX = 1.0 / double(fr.width);
  const double scaleY = (fr.legacy_y ? 1.0 : -1.0) / double(fr.height);
  *ix = (scaleX * x + -0.5) * fr.aspect;
  *iy = scaleY * y + (fr.legacy_y ? -0.5 : 0.5);
}
// CalculateViewVector (projection_3d.cpp:40-89) before the camera rotation:
// the view vector of image point (ix, iy) (aspect applied), with fov from
// CalcFOV.  Three-point: (x fov, 1, y fov); fish eye: at angle |v| fov from
// the axis; equirectangular: longitude x fov/2, latitude y fov/2.
__device__ __forceinline__ D3 projection_dir(int persp, double fov, double ix, double iy) {
  if (persp == MBR_PROJECTION_FISH_EYE || persp == MBR_PROJECTION_FISH_EYE_CUT) {
    const double r = sqrt(ix * ix + iy * iy);
    if (r == 0.0) return D3{0.0, 1.0, 0.0};
    return D3{ix / r * sin(r * fov), cos(r * fov), iy / r * sin(r * fov)};
  }
  if (persp == MBR_PROJECTION_EQUIRECTANGULAR) {
    const double vx = ix * 0.5, vy = iy * 0.5;
    return D3{sin(fov * vx) * cos(fov * vy), cos(fov * vx) * cos(fov * vy), sin(fov * vy)};
  }
  return D3{ix * fov, 1.0, iy * fov};
}
// Fish-eye cut: an image point more than 90 degrees off the axis is not
// traced (render_worker.cpp:165-170, 321); its pixel is black, with no hit.
__device__ __forceinline__ bool hemisphere_cut(int persp, double fov, double ix, double iy) {
  return persp == MBR_PROJECTION_FISH_EYE_CUT && sqrt(ix * ix + iy * iy) > 3.14159265358979323846 * 0.5 / fov;
}
__device__ __forceinline__ D3 view_vector(const DevFrame &fr, double ix, double iy) {
  return rotate(fr, d3norm(projection_dir(fr.persp, fr.fov, ix, iy)));
}
__device__ __forceinline__ D3 camera_of(const DevFrame &fr) { return {fr.camera[0], fr.camera[1], fr.camera[2]}; }
// The tail of CalcDistThresh (render_worker.cpp:669-677): an equirectangular
// view halves the threshold, then advanced quality clamps it to
// [detail_size_min, detail_size_max]; reduceDetail is 1 outside progressive
// previews (render_job.cpp:1177-1182).
__device__ __forceinline__ double thresh_tail(const DevFrame &fr, int persp, double distThresh) {
  if (persp == MBR_PROJECTION_EQUIRECTANGULAR) distThresh *= 0.5;
  if (fr.adv_quality) {
    if (distThresh > fr.detail_size_max) distThresh = fr.detail_size_max;
    if (distThresh < fr.detail_size_min) distThresh = fr.detail_size_min;
  }
  return distThresh;
}
__device__ __forceinline__ double dist_thresh(const DevScene &sc, const DevFrame &fr, D3 q) {
  const double l = d3len(d3sub(camera_of(fr), q));
  double t;
  if (sc.iter_thresh) t = l * fr.resolution * fr.fov;
  else if (fr.constant_de_threshold) t = fr.de_thresh;
  else t = l * fr.resolution * fr.fov / fr.detail_level;
  return thresh_tail(fr, fr.persp, t);
}
// CalcDelta (render_worker.cpp:684-690)
__device__ __forceinline__ double calc_delta(const DevFrame &fr, D3 q) {
  double delta = d3len(d3sub(camera_of(fr), q)) * fr.resolution * fr.fov;
  if (fr.persp == MBR_PROJECTION_EQUIRECTANGULAR) delta *= 0.5;
  return delta;
}
// The limits of one march step (render_worker.cpp:819-834): with advanced
// quality the absolute and threshold-relative bounds, else step <= 3.
__device__ __forceinline__ double step_limit(const DevFrame &fr, double step, double distThresh) {
  if (fr.adv_quality) {
    if (step > fr.abs_step_max) step = fr.abs_step_max;
    if (step < fr.abs_step_min) step = fr.abs_step_min;
    if (distThresh > fr.abs_step_min) {
      if (step > fr.rel_step_max * distThresh) step = fr.rel_step_max * distThresh;
    }
    if (step < fr.rel_step_min * distThresh) step = fr.rel_step_min * distThresh;
  } else if (step > 3.0) {
    step = 3.0;
  }
  return step;
}

// Per-thread counters: DE evaluations and summed iterations live in
// registers; phase totals go to block-shared counters at phase ends.
struct ThreadCount {
  unsigned int de, iters;
};
enum { K_DE = 0, K_ITERS, K_MARCH, K_BINARY, K_NORMAL, K_SHADOW, K_AO, K_GI, K_PIXELS, K_WATCHDOG, K_COUNT };

template <class T, int F, bool W>
__device__ __forceinline__ double de_eval(const DevScene &sc, D3 q, double detail, bool normal_mode, int *iters,
                                          ThreadCount &tc) {
  int it, total;
  const T d = calc_distance<T, F, W>(sc, T(q.x), T(q.y), T(q.z), T(detail), normal_mode, &it, &total);
  tc.de++;
  tc.iters += unsigned(total);
  *iters = it;
  return double(d);
}

struct MarchOut {
  bool found;
  double depth, dist, thr;
  D3 point;
  int iters;
};

// RayMarching (render_worker.cpp:708-951), minScan 0, no invert mode;
// refine = MBR_REFINE_ROOT replaces the windowed binary search by bisection
// of dist - thr to convergence, with R-precision DE evaluations.
template <class T, class R, int F, bool W>
__device__ MarchOut ray_marching(const DevScene &sc, const DevFrame &fr, D3 start, D3 dir, ParkMiller &pm,
                                 ThreadCount &tc, unsigned int *n_march, unsigned int *n_binary) {
  MarchOut o;
  D3 point{1e30, 1e30, 1e30};
  bool found = false, dead = false;
  double scan = 0.0, dist = 0.0, step = 0.0, distThresh = 0.0, prevScan = 0.0;
  const double search_limit = 1.0 - 0.001 * fr.detail_level;
  int iters = 0;
  const double dirLen = d3len(dir);
  unsigned int nm = 0, nb = 0;
  for (int i = 0; i < fr.max_steps; i++) {
    const D3 lastPoint = point;
    point = d3ray(start, dir, scan);
    if ((point.x == lastPoint.x && point.y == lastPoint.y && point.z == lastPoint.z) ||
        !(isfinite(point.x) && isfinite(point.y) && isfinite(point.z))) {
      found = true;
      dead = true;
      break;
    }
    distThresh = dist_thresh(sc, fr, point);
    dist = de_eval<T, F, W>(sc, point, distThresh, false, &iters, tc);
    nm++;
    if (dist < distThresh) {
      found = true;
      break;
    }
    const double jit = fr.jitter ? (1.0 - pm.random(1000) / 10000.0) : 1.0;
    if (sc.interior)
      step = (dist - 0.8 * distThresh) * fr.de_factor * jit;
    else
      step = (dist - 0.5 * distThresh) * fr.de_factor * jit;
    step = step_limit(fr, step, distThresh);
    prevScan = scan;
    scan += step / dirLen;
    if (scan > fr.view_distance_max) break;
  }
  point = d3ray(start, dir, scan);
  if (found && !dead) {
    if (fr.refine == MBR_REFINE_ROOT) {
      double lo = prevScan, hi = scan;
      if (hi > lo) {
        for (int i = 0; i < fr.binary_steps; i++) {
          const double mid = 0.5 * (lo + hi);
          if (mid <= lo || mid >= hi) break;
          const D3 q = d3ray(start, dir, mid);
          const double thr = dist_thresh(sc, fr, q);
          const double d = de_eval<R, F, W>(sc, q, thr, false, &iters, tc);
          nb++;
          if (d < thr) hi = mid;
          else lo = mid;
        }
        scan = hi;
        point = d3ray(start, dir, scan);
        distThresh = dist_thresh(sc, fr, point);
        dist = de_eval<R, F, W>(sc, point, distThresh, false, &iters, tc);
        nb++;
      }
    } else {
      step *= 0.5;
      for (int i = 0; i < fr.binary_steps; i++) {
        if (dist < distThresh && dist > distThresh * search_limit) break;
        if (dist > distThresh) {
          scan += step;
          point = d3ray(start, dir, scan);
        } else if (dist < distThresh * search_limit) {
          scan -= step;
          point = d3ray(start, dir, scan);
        }
        distThresh = dist_thresh(sc, fr, point);
        dist = de_eval<R, F, W>(sc, point, distThresh, false, &iters, tc);
        nb++;
        step *= 0.5;
      }
    }
  }
  if (sc.iter_thresh) {
    scan -= distThresh;
    point = d3ray(start, dir, scan);
    if (found) {
      dist = de_eval<R, F, W>(sc, point, distThresh, false, &iters, tc);
      nb++;
    }
  }
  o.found = found;
  o.dist = dist;
  o.depth = scan;
  o.thr = distThresh;
  o.point = point;
  o.iters = iters;
  *n_march += nm;
  *n_binary += nb;
  return o;
}

// CalculateNormals with slowShading (shader_calculate_normals.cpp:83-106):
// the orbit (Compute, no normal mode) at an 11 x 11 x 11 lattice of points
// q + (i, j, k) delta, i, j, k = -1, -0.8, ... accumulated in steps of 0.2
// as the reference's loops do, delta = CalcDelta(q) * smoothness; the normal
// is the sum of the lattice offsets weighted by 1 + N - iterations.  Every
// orbit counts as one distance evaluation.
template <class T, bool W>
__device__ __noinline__ D3 slow_normals(const DevScene &sc, const DevFrame &fr, D3 q, double thr, ThreadCount &tc) {
  double delta = calc_delta(fr, q) * fr.smoothness;
  if (sc.interior) delta = thr * 0.2 * fr.smoothness;
  D3 n{0.0, 0.0, 0.0};
  for (double px = -1.0; px <= 1.0; px += 0.2) {
    for (double py = -1.0; py <= 1.0; py += 0.2) {
      for (double pz = -1.0; pz <= 1.0; pz += 0.2) {
        const D3 p3{q.x + px * delta, q.y + py * delta, q.z + pz * delta};
        V4<T> z;
        T r, DE;
        bool mx;
        const int i = compute_orbit<T, F_EXT, W>(sc, T(p3.x), T(p3.y), T(p3.z), sc.formula_maxiter, z, r, DE, mx);
        const double pd = double(1 + sc.formula_maxiter - (i + 1));
        n.x = n.x + px * pd;
        n.y = n.y + py * pd;
        n.z = n.z + pz * pd;
        tc.de++;
        tc.iters += unsigned(i + 1);
      }
    }
  }
  return n;
}

template <class T, int F, bool W>
__device__ D3 normals(const DevScene &sc, const DevFrame &fr, D3 q, double thr, ThreadCount &tc) {
  if constexpr (F == F_EXT) {
    if (fr.slow_shading) {
      D3 n = slow_normals<T, W>(sc, fr, q, thr, tc);
      if (fabs(n.x) < 1e-50 && fabs(n.y) < 1e-50 && fabs(n.z) < 1e-50)
        n = D3{1.0, 0.0, 0.0};
      else
        n = d3norm(n);
      if (!(isfinite(n.x) && isfinite(n.y) && isfinite(n.z))) n = D3{1.0, 0.0, 0.0};
      return n;
    }
  }
  double delta = thr * fr.smoothness;
  if (sc.interior) delta = thr * 0.2 * fr.smoothness;
  int it;
  const double sx1 = de_eval<T, F, W>(sc, d3add(q, D3{delta, 0.0, 0.0}), thr, true, &it, tc);
  const double sx2 = de_eval<T, F, W>(sc, d3sub(q, D3{delta, 0.0, 0.0}), thr, true, &it, tc);
  const double sy1 = de_eval<T, F, W>(sc, d3add(q, D3{0.0, delta, 0.0}), thr, true, &it, tc);
  const double sy2 = de_eval<T, F, W>(sc, d3sub(q, D3{0.0, delta, 0.0}), thr, true, &it, tc);
  const double sz1 = de_eval<T, F, W>(sc, d3add(q, D3{0.0, 0.0, delta}), thr, true, &it, tc);
  const double sz2 = de_eval<T, F, W>(sc, d3sub(q, D3{0.0, 0.0, delta}), thr, true, &it, tc);
  D3 n{sx1 - sx2, sy1 - sy2, sz1 - sz2};
  if (fabs(n.x) < 1e-50 && fabs(n.y) < 1e-50 && fabs(n.z) < 1e-50)
    n = D3{1.0, 0.0, 0.0};
  else
    n = d3norm(n);
  if (!(isfinite(n.x) && isfinite(n.y) && isfinite(n.z))) n = D3{1.0, 0.0, 0.0};
  return n;
}

template <class T, int F, bool W>
__device__ double aux_shadow(const DevScene &sc, const DevFrame &fr, D3 q, double thr, D3 L, ThreadCount &tc) {
  // a penetrating directional light marches delta / resolution (light.cpp:277-290)
  const bool pen = fr.penetrating != 0;
  const double distance = pen ? calc_delta(fr, q) / fr.resolution : fr.view_distance_max;
  const bool soft = fr.soft_range > 0.0 && !sc.interior && !sc.iter_thresh;  // bSoft (:71-74)
  double start = thr;
  if (sc.interior) start = thr * fr.de_factor;
  double shadowTemp = 1.0;
  double maxSoft = 0.0;
  int count = 0;
  double step = thr;
  const float dist_thresh_f = float(thr);
  int it;
  for (double i = start; i < distance; i += step) {
    const D3 point2 = d3ray(q, L, i);
    const double dist = de_eval<T, F, W>(sc, point2, thr, false, &it, tc);
    // a soft shadow ignores samples outside the limit box (:130-147)
    const bool outside = F == F_EXT && sc.limits &&
                         (point2.x < sc.lim_min[0] || point2.x > sc.lim_max[0] || point2.y < sc.lim_min[1] ||
                          point2.y > sc.lim_max[1] || point2.z < sc.lim_min[2] || point2.z > sc.lim_max[2]);
    if (soft && !outside) {  // :142-151
      double angle = (dist - double(dist_thresh_f)) / i;
      if (angle < 0) angle = 0;
      if (dist < double(dist_thresh_f)) angle = 0;
      double softShadow = 1.0 - angle / fr.soft_range;
      if (pen) softShadow *= (distance - i) / distance;
      if (softShadow < 0) softShadow = 0;
      if (softShadow > maxSoft) maxSoft = softShadow;
    }
    if (dist < double(dist_thresh_f)) {  // :266-280
      if (pen) {
        shadowTemp -= (distance - i) / distance;
        if (shadowTemp < 0.0) shadowTemp = 0.0;
      } else {
        shadowTemp = 0.0;
      }
      break;
    }
    step = fmin(dist, 1000000.0) * fr.de_factor;
    step = fmax(step, 1e-15);
    count++;
    if (count > fr.max_steps) break;
  }
  return soft ? 1.0 - maxSoft : shadowTemp;
}

// AO march rule of the reference along cosine-hemisphere directions; each
// march is capped at max_steps evaluations (counted as a watchdog trip).
// Fast AO (fr.ao_fast) runs through the same loop, so that the kernel holds
// one inlined distance estimate for both: quality^2 - 1 samples at
// i^2 * distThresh along the normal, each clamped to twice the previous one,
// summed in float as 2^-i (scan - fast_tune * dist) / distThresh, giving
// ao = max(0, 1 - 0.2 sum).
template <class T, int F, bool W>
__device__ double ambient_occlusion(const DevScene &sc, const DevFrame &fr, D3 q, D3 n, double thr,
                                    unsigned long long pixel, ThreadCount &tc, unsigned int *trips) {
  const bool fast = fr.ao_fast != 0;
  const double start_dist = thr;
  const double end_dist = calc_delta(fr, q) / fr.resolution;
  const float dist_thresh_f = float(thr);
  const int rays = fast ? 1 : fr.ao_rays;
  const int samples = fr.ao_quality * fr.ao_quality;
  Pcg32 rng = pcg_init(fr.ao_seed, pixel);
  double sum = 0.0;
  int it;
  for (int k = 0; k < rays; k++) {
    D3 v = n;
    if (!fast) {
      const double u1 = rng.uniform(), u2 = rng.uniform();
      v = cosine_dir(n, u1, u2);
    }
    double dist = 0.0;
    double shadowTemp = fast ? 1e20 : 1.0;  // fast: the previous (clamped) sample
    int steps = 0;
    for (double r = start_dist; fast ? steps + 1 < samples : r < end_dist;) {
      if (steps >= fr.max_steps && !fast) {
        (*trips)++;
        break;
      }
      steps++;
      const D3 point2 = d3ray(q, v, r);
      dist = de_eval<T, F, W>(sc, point2, thr, false, &it, tc);
      if (fast) {  // sum holds the float sum
        if (dist > shadowTemp * 2) dist = shadowTemp * 2.0;
        shadowTemp = dist;
        sum = double(float(sum + ldexp(1.0, -steps) * (r - fr.ao_fast_tune * dist) / thr));
        r = double((steps + 1) * (steps + 1)) * thr;
        continue;
      }
      if (dist < double(dist_thresh_f)) {
        shadowTemp -= (end_dist - r) / end_dist;
        if (shadowTemp < 0.0) shadowTemp = 0.0;
        break;
      }
      r += dist * 2.0;
    }
    if (fast) {
      float ao = 1.0f - 0.2f * float(sum);
      if (ao < 0) ao = 0;
      return ao;
    }
    sum += shadowTemp;
  }
  return sum / fr.ao_rays;
}

// cImage::CalculatePixel + ConvertTo8bitChar for one colour.
__device__ __forceinline__ void to_rgb8(const DevFrame &fr, const float *rgb, uint8_t *o) {
  float c[3];
  for (int k = 0; k < 3; k++) {
    float v = rgb[k] * fr.brightness;
    v = (v - 0.5f) * fr.contrast + 0.5f;
    if (v < 0.0f) v = 0.0f;
    if (fr.hdr) v = tanhf(v);
    c[k] = v;
  }
  const float V = sqrtf(c[0] * c[0] * 0.299f + c[1] * c[1] * 0.587f + c[2] * c[2] * 0.114f);
  for (int k = 0; k < 3; k++) {
    float v = V + (c[k] - V) * fr.saturation;
    v = fminf(fmaxf(v, 0.0f), 1.0f);
    const unsigned short u16 = (unsigned short)(fr.gamma[(unsigned short)(v * 65535.0f)]);
    o[k] = (uint8_t)(u16 / 256);
  }
}

}  // namespace mbr
