// adjoint.cu - gradients of a per-pixel loss L(depth, shade) with respect to
// the formula parameters (Mandelbulb power; Mandelbox scale and min radius
// squared) and the camera (position at fixed view angles, yaw).
//
// Only the forward hit depth t per pixel is stored.  The backward pass
// recomputes, per hit pixel, the distance estimate at the hit point and at
// the six central-difference normal samples of CalculateNormals
// (src/shader_calculate_normals.cpp:44-79) in forward-mode dual numbers
// carrying six tangents (power, scale, mR2, x, y, z); the formula iteration
// follows Compute<calcModeNormal> (src/compute_fractal.cpp:175-321) and the
// formulas (fractal_mandelbulb.cpp:29-43, fractal_mandelbox.cpp:66-107) in the
// reference's order of operations.
//
// Depth: the hit t solves F(t) = dist(o + t d) - thr(t) = 0 with
// thr(t) = c0 * |o - p| = c0 * t |d| (CalcDistThresh, render_worker.cpp:653-679),
// so by the implicit function theorem
//   dt/dθ = -(∂dist/∂θ + ∇dist·∂p/∂θ|_t) / (∇dist·d - c0 |d|).
// Pixels whose stored depth is not a root of F (the refinement ended on a
// jump of the distance estimate) contribute nothing.
// Shade: the Lambert term s = N·L of the normal N = g/|g|, g_a = dist(p + δe_a)
// - dist(p - δe_a), δ = thr * smoothness, differentiated through p(θ) and δ(θ).
// A distance estimate whose orbit does not escape (a sample inside the set)
// is taken as constant: its value is ~0 and its exact derivative through
// dozens of chaotic iterations is noise.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "mbr_internal.h"
#include "pixel_ops.cuh"

namespace mbr {

enum { TN_POWER = 0, TN_SCALE = 1, TN_MR2 = 2, TN_X = 3, TN_Y = 4, TN_Z = 5, TN = 6 };

template <class T>
struct Dn {
  T v;
  T d[TN];
};

template <class T>
__device__ __forceinline__ Dn<T> dconst(T v) {
  Dn<T> r;
  r.v = v;
#pragma unroll
  for (int i = 0; i < TN; i++) r.d[i] = T(0);
  return r;
}
template <class T>
__device__ __forceinline__ Dn<T> dseed(T v, int k) {
  Dn<T> r = dconst<T>(v);
  r.d[k] = T(1);
  return r;
}
template <class T>
__device__ __forceinline__ Dn<T> operator+(const Dn<T> &a, const Dn<T> &b) {
  Dn<T> r;
  r.v = a.v + b.v;
#pragma unroll
  for (int i = 0; i < TN; i++) r.d[i] = a.d[i] + b.d[i];
  return r;
}
template <class T>
__device__ __forceinline__ Dn<T> operator-(const Dn<T> &a, const Dn<T> &b) {
  Dn<T> r;
  r.v = a.v - b.v;
#pragma unroll
  for (int i = 0; i < TN; i++) r.d[i] = a.d[i] - b.d[i];
  return r;
}
template <class T>
__device__ __forceinline__ Dn<T> operator*(const Dn<T> &a, const Dn<T> &b) {
  Dn<T> r;
  r.v = a.v * b.v;
#pragma unroll
  for (int i = 0; i < TN; i++) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
  return r;
}
template <class T>
__device__ __forceinline__ Dn<T> operator/(const Dn<T> &a, const Dn<T> &b) {
  Dn<T> r;
  r.v = a.v / b.v;
  const T ib2 = T(1) / (b.v * b.v);
#pragma unroll
  for (int i = 0; i < TN; i++) r.d[i] = (a.d[i] * b.v - a.v * b.d[i]) * ib2;
  return r;
}
template <class T>
__device__ __forceinline__ Dn<T> operator+(const Dn<T> &a, T b) {
  Dn<T> r = a;
  r.v = a.v + b;
  return r;
}
template <class T>
__device__ __forceinline__ Dn<T> operator-(const Dn<T> &a, T b) {
  Dn<T> r = a;
  r.v = a.v - b;
  return r;
}
template <class T>
__device__ __forceinline__ Dn<T> operator*(const Dn<T> &a, T b) {
  Dn<T> r;
  r.v = a.v * b;
#pragma unroll
  for (int i = 0; i < TN; i++) r.d[i] = a.d[i] * b;
  return r;
}
template <class T>
__device__ __forceinline__ Dn<T> neg(const Dn<T> &a) {
  return a * T(-1);
}
template <class T>
__device__ __forceinline__ Dn<T> chain(const Dn<T> &a, T fv, T dfa) {
  Dn<T> r;
  r.v = fv;
#pragma unroll
  for (int i = 0; i < TN; i++) r.d[i] = dfa * a.d[i];
  return r;
}
template <class T>
__device__ __forceinline__ Dn<T> dsqrt(const Dn<T> &a) {
  const T s = m_sqrt(a.v);
  return chain(a, s, s > T(0) ? T(0.5) / s : T(0));
}
template <class T>
__device__ __forceinline__ Dn<T> dabs(const Dn<T> &a) {
  return a.v < T(0) ? neg(a) : a;
}
template <class T>
__device__ __forceinline__ Dn<T> dlog(const Dn<T> &a) {
  return chain(a, m_log(a.v), T(1) / a.v);
}

template <class T>
__device__ __forceinline__ Dn<T> dlen3(const Dn<T> &x, const Dn<T> &y, const Dn<T> &z) {
  return dsqrt(x * x + y * y + z * z);
}

// The distance estimate of a non-hybrid Mandelbulb or Mandelbox scene in
// dual numbers: Compute<calcModeNormal> + CalculateDistanceSimple.
template <class T>
__device__ Dn<T> de_dual(const DevScene &sc, Dn<T> px, Dn<T> py, Dn<T> pz, T detail) {
  const DevSlot &s = sc.slot[0];
  const int maxN = sc.formula_maxiter;
  Dn<T> zx = px, zy = py, zz = pz;
  const Dn<T> cx = zx * T(sc.cmul[0]), cy = zy * T(sc.cmul[1]), cz = zz * T(sc.cmul[2]);
  Dn<T> r = dlen3(zx, zy, zz);
  Dn<T> DE = dconst<T>(T(1));
  const T bailout = T(s.d[P_BAILOUT]);
  const bool bulb = s.formula == MBR_FORMULA_MANDELBULB;
  // parameters with tangents
  const Dn<T> power = dseed<T>(T(s.d[P_POWER]), TN_POWER);
  const Dn<T> scale = dseed<T>(T(s.d[P_MB_SCALE]), TN_SCALE);
  const Dn<T> mR2 = dseed<T>(T(s.d[P_MB_MR2]), TN_MR2);
  const Dn<T> fR2 = dconst<T>(T(s.d[P_MB_FR2]));
  const Dn<T> factor1 = fR2 / mR2;
  const T limit = T(s.d[P_MB_LIMIT]), value = T(s.d[P_MB_VALUE]);
  int i;
  bool escaped = false;
  for (i = 0; i < maxN; i++) {
    if (bulb) {
      // th0 = asin(z/r) + beta; ph0 = atan2(y, x) + alpha
      const Dn<T> q = zz / r;
      Dn<T> th0 = chain(q, m_asin(q.v), T(1) / m_sqrt(T(1) - q.v * q.v)) + T(s.d[P_BETA]);
      Dn<T> ph0;
      {
        const T den = zx.v * zx.v + zy.v * zy.v;
        ph0.v = m_atan2(zy.v, zx.v);
#pragma unroll
        for (int k = 0; k < TN; k++) ph0.d[k] = (zx.v * zy.d[k] - zy.v * zx.d[k]) / den;
        ph0 = ph0 + T(s.d[P_ALPHA]);
      }
      // rp = r^(power-1): d = (p-1) r^(p-2) dr + r^(p-1) ln r dp
      const Dn<T> pm1 = power - T(1);
      Dn<T> rp;
      {
        const T v = m_pow(r.v, pm1.v);
        const T dr = pm1.v * m_pow(r.v, pm1.v - T(1));
        const T dp = r.v > T(0) ? v * m_log(r.v) : T(0);
        rp.v = v;
#pragma unroll
        for (int k = 0; k < TN; k++) rp.d[k] = dr * r.d[k] + dp * pm1.d[k];
      }
      const Dn<T> th = th0 * power, ph = ph0 * power;
      T sth, cth, sph, cph;
      m_sincos(th.v, &sth, &cth);
      m_sincos(ph.v, &sph, &cph);
      const Dn<T> Cth = chain(th, cth, -sth), Sth = chain(th, sth, cth);
      const Dn<T> Cph = chain(ph, cph, -sph), Sph = chain(ph, sph, cph);
      DE = (rp * DE) * power + T(1);
      rp = rp * r;
      zx = Cth * Cph * rp;
      zy = Cth * Sph * rp;
      zz = Sth * rp;
    } else {
      if (m_abs(zx.v) > limit) zx = dconst<T>(m_copysign(value, zx.v)) - zx;
      if (m_abs(zy.v) > limit) zy = dconst<T>(m_copysign(value, zy.v)) - zy;
      if (m_abs(zz.v) > limit) zz = dconst<T>(m_copysign(value, zz.v)) - zz;
      const Dn<T> r2 = zx * zx + zy * zy + zz * zz;
      const T offx = T(s.d[P_MB_OFF_X]), offy = T(s.d[P_MB_OFF_Y]), offz = T(s.d[P_MB_OFF_Z]);
      zx = zx + offx;
      zy = zy + offy;
      zz = zz + offz;
      if (r2.v < mR2.v) {
        zx = zx * factor1;
        zy = zy * factor1;
        zz = zz * factor1;
        DE = DE * factor1;
      } else if (r2.v < fR2.v) {
        const Dn<T> t = fR2 / r2;
        zx = zx * t;
        zy = zy * t;
        zz = zz * t;
        DE = DE * t;
      }
      zx = zx - offx;
      zy = zy - offy;
      zz = zz - offz;
      zx = zx * scale;
      zy = zy * scale;
      zz = zz * scale;
      DE = DE * dabs(scale) + T(1);
    }
    if (s.add_c) {
      zx = zx + cx;
      zy = zy + cy;
      zz = zz + cz;
    }
    r = dlen3(zx, zy, zz);
    if (!(isfinite(r.v))) break;
    if (s.check_bailout && r.v > bailout) {
      escaped = true;
      break;
    }
  }
  Dn<T> dist;
  if (DE.v > T(0)) {
    if (sc.de_analytic == 2) dist = (r.v > T(1)) ? (r * T(0.5)) * dlog(r) / DE : dconst<T>(T(0));
    else if (sc.de_analytic == 3) dist = (r - T(2)) / DE;
    else dist = r / DE;
  } else {
    dist = r;
  }
  const int iters = i + 1;
  if (iters < sc.min_n && dist.v < detail) dist = dconst<T>(detail);
  if (dist.v < T(0)) dist = dconst<T>(T(0));
  if (dist.v > T(10)) dist = dconst<T>(T(10));
  // a non-escaping orbit (a point inside the set): the estimate is ~0 and
  // constant to first order; its exact derivative is chaotic noise
  if (!escaped) dist = dconst<T>(dist.v);
  return dist;
}

struct AdjointFrame {
  double dM[9];  // d(mRot)/d(yaw)
};

template <class T>
__global__ void __launch_bounds__(128) adjoint_kernel(const __grid_constant__ DevScene sc,
                                                      const __grid_constant__ DevFrame fr,
                                                      const __grid_constant__ AdjointFrame af, const double *depth,
                                                      const uint8_t *hit, const float *dl_ddepth,
                                                      const float *dl_dshade, double *partials) {
  const long long n = (long long)fr.width * fr.height;
  double acc[MBR_GRAD_COUNT];
#pragma unroll
  for (int k = 0; k < MBR_GRAD_COUNT; k++) acc[k] = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    if (!hit[i]) continue;
    const double wt = dl_ddepth ? double(dl_ddepth[i]) : 0.0;
    const double ws = dl_dshade ? double(dl_dshade[i]) : 0.0;
    if (wt == 0.0 && ws == 0.0) continue;
    const int x = int(i % fr.width), y = int(i / fr.width);
    double ix, iy;
    image_point(fr, double(x), double(y), &ix, &iy);
    const D3 v0 = d3norm(D3{ix * fr.fov, 1.0, iy * fr.fov});
    const D3 w = rotate(fr, v0);
    const double wn = 1.0 / d3len(w);
    const D3 dir{w.x * wn, w.y * wn, w.z * wn};
    const double t = depth[i];
    const D3 cam = camera_of(fr);
    const D3 p = d3ray(cam, dir, t);
    const double thr = dist_thresh(sc, fr, p);
    const double c0 = fr.resolution * fr.fov / fr.detail_level * d3len(dir);
    // dist and its tangents at the hit point
    const Dn<T> dh = de_dual<T>(sc, dseed<T>(T(p.x), TN_X), dseed<T>(T(p.y), TN_Y), dseed<T>(T(p.z), TN_Z), T(thr));
    // implicit differentiation needs F(t) = dist - thr = 0 at the stored
    // depth; a refinement that ended on a jump of the distance estimate (an
    // orbit's bailout iteration changing along the ray) has no derivative
    if (fabs(double(dh.v) - thr) > (sizeof(T) == 8 ? 1e-6 : 1e-4) * thr) continue;
    const D3 g{double(dh.d[TN_X]), double(dh.d[TN_Y]), double(dh.d[TN_Z])};
    // ∂p/∂θ at fixed t
    D3 dp[MBR_GRAD_COUNT];
#pragma unroll
    for (int k = 0; k < MBR_GRAD_COUNT; k++) dp[k] = D3{0.0, 0.0, 0.0};
    dp[MBR_GRAD_CAMERA_X] = D3{1.0, 0.0, 0.0};
    dp[MBR_GRAD_CAMERA_Y] = D3{0.0, 1.0, 0.0};
    dp[MBR_GRAD_CAMERA_Z] = D3{0.0, 0.0, 1.0};
    {
      const double *m = af.dM;
      const D3 dw{m[0] * v0.x + m[1] * v0.y + m[2] * v0.z, m[3] * v0.x + m[4] * v0.y + m[5] * v0.z,
                  m[6] * v0.x + m[7] * v0.y + m[8] * v0.z};
      dp[MBR_GRAD_YAW] = d3mul(dw, t * wn);
    }
    double dd[MBR_GRAD_COUNT];
#pragma unroll
    for (int k = 0; k < MBR_GRAD_COUNT; k++) dd[k] = 0.0;
    dd[MBR_GRAD_BULB_POWER] = double(dh.d[TN_POWER]);
    dd[MBR_GRAD_MANDELBOX_SCALE] = double(dh.d[TN_SCALE]);
    dd[MBR_GRAD_MANDELBOX_MIN_R2] = double(dh.d[TN_MR2]);
    const double denom = d3dot(g, dir) - c0;
    double dt[MBR_GRAD_COUNT];
#pragma unroll
    for (int k = 0; k < MBR_GRAD_COUNT; k++) dt[k] = -(dd[k] + d3dot(g, dp[k])) / denom;
    // the Lambert term through the six normal samples
    double ds[MBR_GRAD_COUNT];
#pragma unroll
    for (int k = 0; k < MBR_GRAD_COUNT; k++) ds[k] = 0.0;
    if (ws != 0.0) {
      const double delta = thr * fr.smoothness;
      double gv[3];
      double gd[3][MBR_GRAD_COUNT];
      for (int a = 0; a < 3; a++) {
        const D3 e{a == 0 ? 1.0 : 0.0, a == 1 ? 1.0 : 0.0, a == 2 ? 1.0 : 0.0};
        const D3 pp = d3add(p, d3mul(e, delta)), pm = d3sub(p, d3mul(e, delta));
        const Dn<T> sp = de_dual<T>(sc, dseed<T>(T(pp.x), TN_X), dseed<T>(T(pp.y), TN_Y), dseed<T>(T(pp.z), TN_Z), T(thr));
        const Dn<T> sm = de_dual<T>(sc, dseed<T>(T(pm.x), TN_X), dseed<T>(T(pm.y), TN_Y), dseed<T>(T(pm.z), TN_Z), T(thr));
        gv[a] = double(sp.v) - double(sm.v);
        const D3 gp{double(sp.d[TN_X]), double(sp.d[TN_Y]), double(sp.d[TN_Z])};
        const D3 gm{double(sm.d[TN_X]), double(sm.d[TN_Y]), double(sm.d[TN_Z])};
#pragma unroll
        for (int k = 0; k < MBR_GRAD_COUNT; k++) {
          const D3 dpt = d3add(dp[k], d3mul(dir, dt[k]));
          const double ddelta = c0 * fr.smoothness * dt[k];
          double dplus = d3dot(gp, d3add(dpt, d3mul(e, ddelta)));
          double dminus = d3dot(gm, d3sub(dpt, d3mul(e, ddelta)));
          if (k <= MBR_GRAD_MANDELBOX_MIN_R2) {
            dplus += double(sp.d[k]);
            dminus += double(sm.d[k]);
          }
          gd[a][k] = dplus - dminus;
        }
      }
      const double gl = sqrt(gv[0] * gv[0] + gv[1] * gv[1] + gv[2] * gv[2]);
      const D3 N{gv[0] / gl, gv[1] / gl, gv[2] / gl};
      const D3 L{fr.light[0], fr.light[1], fr.light[2]};
      const double s = d3dot(N, L);
      if (s > 0.0) {
        const double scale = double(fr.material_shading) * double(fr.light_intensity);
#pragma unroll
        for (int k = 0; k < MBR_GRAD_COUNT; k++) {
          const D3 dg{gd[0][k], gd[1][k], gd[2][k]};
          const double ndg = d3dot(N, dg);
          const D3 dn = d3mul(d3sub(dg, d3mul(N, ndg)), 1.0 / gl);
          ds[k] = scale * d3dot(dn, L);
        }
      }
    }
#pragma unroll
    for (int k = 0; k < MBR_GRAD_COUNT; k++) acc[k] += wt * dt[k] + ws * ds[k];
  }
  // warp reduction, then the block's warps in order: one partial sum per
  // block and parameter, summed by adjoint_sum_kernel in block order, so the
  // gradient does not depend on the order in which blocks ran
  __shared__ double warp_sum[4][MBR_GRAD_COUNT];
#pragma unroll
  for (int k = 0; k < MBR_GRAD_COUNT; k++) {
    double v = acc[k];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) warp_sum[threadIdx.x >> 5][k] = v;
  }
  __syncthreads();
  if (threadIdx.x < MBR_GRAD_COUNT) {
    const int k = threadIdx.x;
    partials[(long long)blockIdx.x * MBR_GRAD_COUNT + k] =
        ((warp_sum[0][k] + warp_sum[1][k]) + warp_sum[2][k]) + warp_sum[3][k];
  }
}

// grad[k] += the blocks' partial sums of parameter k, in block order.
__global__ void adjoint_sum_kernel(const double *partials, int blocks, double *grad) {
  const int k = threadIdx.x;
  if (k >= MBR_GRAD_COUNT) return;
  double v = 0.0;
  for (int b = 0; b < blocks; b++) v += partials[(long long)b * MBR_GRAD_COUNT + k];
  grad[k] += v;
}

}  // namespace mbr

using namespace mbr;

extern "C" mbr_status mbr_adjoint(mbr_ctx *ctx, const mbr_camera *camera, const mbr_render_params *params,
                                  const double *depth, const uint8_t *hit, const float *dl_ddepth,
                                  const float *dl_dshade, double *grad, int engine, void *stream) {
  if (!ctx || !camera || !params || !depth || !hit || !grad) return set_err(ctx, MBR_EINVAL, "null argument");
  const DevScene *sc = ctx_scene(ctx);
  if (!sc) return set_err(ctx, MBR_EINVAL, "no scene set");
  if (!camera->use_angles)
    return set_err(ctx, MBR_EINVAL, "the adjoint differentiates a camera given by position and angles (use_angles = 1)");
  if (camera->perspective_type != MBR_PROJECTION_THREE_POINT)
    return set_err(ctx, MBR_EUNSUPPORTED, "the adjoint covers the three-point projection");
  if (params->slow_shading)
    return set_err(ctx, MBR_EUNSUPPORTED, "the adjoint differentiates the six-sample normals (no slow shading)");
  if (params->advanced_quality || params->constant_de_threshold)
    return set_err(ctx, MBR_EUNSUPPORTED, "the adjoint covers thresholds proportional to the distance (no advanced "
                                          "quality clamps, no constant threshold)");
  if (sc->mbrot.folds || sc->mbrot.main)
    return set_err(ctx, MBR_EUNSUPPORTED, "the adjoint covers the Mandelbox without rotations");
  if (sc->n_prims > 0 || sc->n_nodes > 0 || sc->limits || sc->gbox || sc->gsph)
    return set_err(ctx, MBR_EUNSUPPORTED,
                   "the adjoint covers scenes without primitives, objects tree, limit box or global folds");
  if (sc->delta_de || sc->de_final > DEF_IFS)
    return set_err(ctx, MBR_EUNSUPPORTED, "the adjoint covers the analytic linear and logarithmic DE functions");
  if (sc->is_hybrid || sc->has_w || sc->iter_thresh || sc->interior ||
      (sc->slot[0].formula != MBR_FORMULA_MANDELBULB && sc->slot[0].formula != MBR_FORMULA_MANDELBOX))
    return set_err(ctx, MBR_EUNSUPPORTED,
                   "the adjoint covers non-hybrid Mandelbulb and Mandelbox scenes without interior, iteration "
                   "threshold or 4-D modes");
  if (engine != MBR_ENGINE_PLAIN_FP64 && engine != MBR_ENGINE_PLAIN_MIXED)
    return set_err(ctx, MBR_EINVAL, "adjoint engine must be MBR_ENGINE_PLAIN_FP64 or MBR_ENGINE_PLAIN_MIXED");
  DevFrame fr;
  mbr_status st = build_frame(ctx, *camera, *params, &fr, stream);
  if (st != MBR_OK) return st;
  // d(mRot)/d(yaw) with mRot = Rz(yaw) Rx(pitch) Ry(roll) (PrepareMainVectors)
  AdjointFrame af;
  {
    const double yaw = camera->angles[0], pitch = camera->angles[1], roll = camera->angles[2];
    const double dz[9] = {-std::sin(yaw), -std::cos(yaw), 0, std::cos(yaw), -std::sin(yaw), 0, 0, 0, 0};
    const double cx = std::cos(pitch), sx = std::sin(pitch), cy = std::cos(roll), sy = std::sin(roll);
    const double rx[9] = {1, 0, 0, 0, cx, -sx, 0, sx, cx};
    const double ry[9] = {cy, 0, sy, 0, 1, 0, -sy, 0, cy};
    double t[9];
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) t[i * 3 + j] = dz[i * 3] * rx[j] + dz[i * 3 + 1] * rx[3 + j] + dz[i * 3 + 2] * rx[6 + j];
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++)
        af.dM[i * 3 + j] = t[i * 3] * ry[j] + t[i * 3 + 1] * ry[3 + j] + t[i * 3 + 2] * ry[6 + j];
  }
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const long long n = (long long)fr.width * fr.height;
  const int grid = int(std::max<long long>(1, std::min<long long>((n + 127) / 128, (long long)sms * 16)));
  double *partials = nullptr;
  st = ctx_adjoint_partials(ctx, size_t(grid) * MBR_GRAD_COUNT * sizeof(double), &partials);
  if (st != MBR_OK) return st;
  if (engine == MBR_ENGINE_PLAIN_FP64)
    adjoint_kernel<double><<<grid, 128, 0, s>>>(*sc, fr, af, depth, hit, dl_ddepth, dl_dshade, partials);
  else
    adjoint_kernel<float><<<grid, 128, 0, s>>>(*sc, fr, af, depth, hit, dl_ddepth, dl_dshade, partials);
  adjoint_sum_kernel<<<1, 32, 0, s>>>(partials, grid, grad);
  return cuda_err(ctx, int(cudaGetLastError()), "adjoint kernel launch");
}
