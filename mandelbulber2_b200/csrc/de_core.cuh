// de_core.cuh - distance estimation on the device: the formula iterations,
// the Compute<calcModeNormal> loop and CalculateDistanceSimple, templated on
// the scalar type T (double or float) and on the formula F (a fixed formula
// id for single-formula scenes, 0 for the generic per-iteration dispatch that
// hybrid sequences need).
//
// Reference semantics followed (file:line of mandelbulber2):
//   cFractalMandelbulb::FormulaCode   formula/definition/fractal_mandelbulb.cpp:29-43
//   cFractalMandelbox::FormulaCode    formula/definition/fractal_mandelbox.cpp:66-107
//   cFractalMengerSponge::FormulaCode formula/definition/fractal_menger_sponge.cpp:30-71
//   Compute<calcModeNormal>           src/compute_fractal.cpp:67-654
//   CalculateDistanceSimple           src/calculate_distance.cpp:533-606
// In FP64 every operation is written in the reference's order, so a build
// without FMA contraction performs the same IEEE operations as the CPU code.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

#include "formula_params.h"
#include "mbr_device.h"

namespace mbr {

template <class T>
__device__ __forceinline__ T P(const DevSlot &s, int i);
template <>
__device__ __forceinline__ double P<double>(const DevSlot &s, int i) {
  return s.d[i];
}
template <>
__device__ __forceinline__ float P<float>(const DevSlot &s, int i) {
  return s.f[i];
}

template <class T>
struct V4 {
  T x, y, z, w;
};

// Scalar helpers with one spelling for both precisions.
__device__ __forceinline__ double m_sqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float m_sqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ double m_abs(double x) { return fabs(x); }
__device__ __forceinline__ float m_abs(float x) { return fabsf(x); }
__device__ __forceinline__ double m_asin(double x) { return asin(x); }
__device__ __forceinline__ float m_asin(float x) { return asinf(x); }
__device__ __forceinline__ double m_acos(double x) { return acos(x); }
__device__ __forceinline__ float m_acos(float x) { return acosf(x); }
__device__ __forceinline__ double m_atan2(double y, double x) { return atan2(y, x); }
__device__ __forceinline__ float m_atan2(float y, float x) { return atan2f(y, x); }
__device__ __forceinline__ double m_pow(double a, double b) { return pow(a, b); }
__device__ __forceinline__ float m_pow(float a, float b) { return powf(a, b); }
__device__ __forceinline__ double m_log(double x) { return log(x); }
__device__ __forceinline__ float m_log(float x) { return logf(x); }
__device__ __forceinline__ void m_sincos(double x, double *s, double *c) { sincos(x, s, c); }
__device__ __forceinline__ void m_sincos(float x, float *s, float *c) { sincosf(x, s, c); }
__device__ __forceinline__ double m_copysign(double a, double b) { return copysign(a, b); }
__device__ __forceinline__ float m_copysign(float a, float b) { return copysignf(a, b); }
__device__ __forceinline__ bool m_finite(double x) { return isfinite(x); }
__device__ __forceinline__ bool m_finite(float x) { return isfinite(x); }

template <class T, bool W>
__device__ __forceinline__ T len4(const V4<T> &v) {  // CVector4::Length
  if (W) return m_sqrt(v.x * v.x + v.y * v.y + v.z * v.z + v.w * v.w);
  return m_sqrt(v.x * v.x + v.y * v.y + v.z * v.z);
}
template <class T, bool W>
__device__ __forceinline__ bool nan4(const V4<T> &v) {  // CVector4::IsNotANumber
  bool ok = m_finite(v.x) & m_finite(v.y) & m_finite(v.z);
  if (W) ok = ok & m_finite(v.w);
  return !ok;
}

// ---- formulas -----------------------------------------------------------------
template <class T>
__device__ __forceinline__ void f_mandelbulb(V4<T> &z, T r, T &DE, const DevSlot &s) {
  const T power = P<T>(s, P_POWER);
  const T th0 = m_asin(z.z / r) + P<T>(s, P_BETA);
  const T ph0 = m_atan2(z.y, z.x) + P<T>(s, P_ALPHA);
  T rp = m_pow(r, P<T>(s, P_POWER_M1));
  const T th = th0 * power;
  const T ph = ph0 * power;
  T sth, cth, sph, cph;
  m_sincos(th, &sth, &cth);
  m_sincos(ph, &sph, &cph);
  DE = (rp * DE) * power + T(1.0);
  rp = rp * r;
  z.x = cth * cph * rp;
  z.y = cth * sph * rp;
  z.z = sth * rp;
}

// CRotationMatrix::RotateVector on the xyz of a 4-vector (algebra.cpp:333-344,
// 168-175), or with the transpose (rotinv, fractal.cpp:670)
template <class T>
__device__ __forceinline__ V4<T> mb_turn(const double *m, bool transpose, const V4<T> &v) {
  V4<T> r = v;
  if (!transpose) {
    r.x = T(m[0]) * v.x + T(m[1]) * v.y + T(m[2]) * v.z;
    r.y = T(m[3]) * v.x + T(m[4]) * v.y + T(m[5]) * v.z;
    r.z = T(m[6]) * v.x + T(m[7]) * v.y + T(m[8]) * v.z;
  } else {
    r.x = T(m[0]) * v.x + T(m[3]) * v.y + T(m[6]) * v.z;
    r.y = T(m[1]) * v.x + T(m[4]) * v.y + T(m[7]) * v.z;
    r.z = T(m[2]) * v.x + T(m[5]) * v.y + T(m[8]) * v.z;
  }
  return r;
}

template <class T>
__device__ __forceinline__ T &v4_axis(V4<T> &v, int dim) {
  return dim == 0 ? v.x : (dim == 1 ? v.y : v.z);
}

// ROT: the rotation code is compiled in (rot: the scene's rotations; zero
// flags: none); kernels of scenes without rotations are built without it, so
// its registers do not lower their occupancy
template <class T, bool W, bool ROT = false>
__device__ __forceinline__ void f_mandelbox(V4<T> &z, T &DE, const DevSlot &s, const MbRot *rot = nullptr) {
  // box fold; the host requires folding_limit >= 0, so |z| > limit implies
  // z != 0 and copysign(value, z) equals sign(z) * value exactly
  const T limit = P<T>(s, P_MB_LIMIT), value = P<T>(s, P_MB_VALUE);
  if (ROT && rot->folds) {
    // each axis folded in the frame of rot[0][dim] above the limit, else of
    // rot[1][dim] below minus the limit, then turned back
    // (fractal_mandelbox.cpp:33-63)
    for (int dim = 0; dim < 3; dim++) {
      V4<T> zr = rot->zero[0][dim] ? z : mb_turn<T>(rot->m[0][dim], false, z);
      if (v4_axis(zr, dim) > limit) {
        v4_axis(zr, dim) = value - v4_axis(zr, dim);
        z = mb_turn<T>(rot->m[0][dim], true, zr);
      } else {
        zr = rot->zero[1][dim] ? z : mb_turn<T>(rot->m[1][dim], false, z);
        if (v4_axis(zr, dim) < -limit) {
          v4_axis(zr, dim) = -value - v4_axis(zr, dim);
          z = mb_turn<T>(rot->m[1][dim], true, zr);
        }
      }
    }
  } else {
    if (m_abs(z.x) > limit) z.x = m_copysign(value, z.x) - z.x;
    if (m_abs(z.y) > limit) z.y = m_copysign(value, z.y) - z.y;
    if (m_abs(z.z) > limit) z.z = m_copysign(value, z.z) - z.z;
  }
  T r2 = z.x * z.x + z.y * z.y + z.z * z.z;
  if (W) r2 = r2 + z.w * z.w;
  // FP64 always applies the offset, as the reference does; FP32 skips a zero
  // offset (adding and subtracting +0 changes nothing but the sign of a zero)
  const bool off = (sizeof(T) == 8) || s.has_offset != 0;
  if (off) {
    z.x = z.x + P<T>(s, P_MB_OFF_X);
    z.y = z.y + P<T>(s, P_MB_OFF_Y);
    z.z = z.z + P<T>(s, P_MB_OFF_Z);
  }
  if (r2 < P<T>(s, P_MB_MR2)) {
    const T f1 = P<T>(s, P_MB_FACTOR1);
    z.x = z.x * f1;
    z.y = z.y * f1;
    z.z = z.z * f1;
    if (W) z.w = z.w * f1;
    DE = DE * f1;
  } else if (r2 < P<T>(s, P_MB_FR2)) {
    const T t = P<T>(s, P_MB_FR2) / r2;
    z.x = z.x * t;
    z.y = z.y * t;
    z.z = z.z * t;
    if (W) z.w = z.w * t;
    DE = DE * t;
  }
  if (off) {
    z.x = z.x - P<T>(s, P_MB_OFF_X);
    z.y = z.y - P<T>(s, P_MB_OFF_Y);
    z.z = z.z - P<T>(s, P_MB_OFF_Z);
  }
  if (ROT && rot->main && !rot->main_zero) z = mb_turn<T>(rot->mm, false, z);  // :103
  const T scale = P<T>(s, P_MB_SCALE);
  z.x = z.x * scale;
  z.y = z.y * scale;
  z.z = z.z * scale;
  if (W) z.w = z.w * scale;
  DE = DE * P<T>(s, P_MB_ABS_SCALE) + T(1.0);
}

template <class T, bool W>
__device__ __forceinline__ void f_menger(V4<T> &z, T &DE, const DevSlot &s) {
  z.x = m_abs(z.x);
  z.y = m_abs(z.y);
  z.z = m_abs(z.z);
  if (W) z.w = m_abs(z.w);
  T tmp;
  if (z.x < z.y) { tmp = z.y; z.y = z.x; z.x = tmp; }
  if (z.x < z.z) { tmp = z.z; z.z = z.x; z.x = tmp; }
  if (z.y < z.z) { tmp = z.z; z.z = z.y; z.y = tmp; }
  const T s3 = P<T>(s, P_SCALE3);
  z.x = z.x * s3;
  z.y = z.y * s3;
  z.z = z.z * s3;
  if (W) z.w = z.w * s3;
  z.x = z.x - T(2.0);
  z.y = z.y - T(2.0);
  if (z.z > T(1.0)) z.z = z.z - T(2.0);
  DE = DE * s3;
}

// cFractalMandelbulbPower2::FormulaCode (fractal_mandelbulb_power2.cpp:30-45)
template <class T>
__device__ __forceinline__ void f_bulb_pow2(V4<T> &z, T r, T &DE) {
  DE = DE * T(2.0) * r;
  const T x2 = z.x * z.x;
  const T y2 = z.y * z.y;
  const T z2 = z.z * z.z;
  const T temp = T(1.0) - z2 / (x2 + y2);
  const T nx = (x2 - y2) * temp;
  const T ny = T(2.0) * z.x * z.y * temp;
  const T nz = T(-2.0) * z.z * m_sqrt(x2 + y2);
  z.x = nx;
  z.y = ny;
  z.z = nz;
}

// cFractalXenodreambuie::FormulaCode (fractal_xenodreambuie.cpp:30-49): the
// Mandelbulb's parameters, azimuth from atan2 + beta, polar angle from acos
// + alpha reflected into [-pi/2, pi/2]
template <class T>
__device__ __forceinline__ void f_xenodreambuie(V4<T> &z, T r, T &DE, const DevSlot &s) {
  const T power = P<T>(s, P_POWER);
  T rp = m_pow(r, P<T>(s, P_POWER_M1));
  DE = rp * DE * power + T(1.0);
  rp = rp * r;
  const T th = (m_atan2(z.y, z.x) + P<T>(s, P_BETA)) * power;
  T ph = m_acos(z.z / r) + P<T>(s, P_ALPHA);
  if (m_abs(ph) > T(0.5 * 3.14159265358979323846)) ph = m_copysign(T(3.14159265358979323846), ph) - ph;
  ph = ph * power;
  T sth, cth, sph, cph;
  m_sincos(th, &sth, &cth);
  m_sincos(ph, &sph, &cph);
  z.x = rp * cth * sph;
  z.y = rp * sth * sph;
  z.z = rp * cph;
}

// cFractalHypercomplex::FormulaCode (fractal_hypercomplex.cpp:30-45): the
// 4-D state is always carried (the host sets has_w for this formula)
template <class T>
__device__ __forceinline__ void f_hypercomplex(V4<T> &z, T r, T &DE) {
  DE = DE * T(2.0) * r;
  const T nx = z.x * z.x - z.y * z.y - z.z * z.z - z.w * z.w;
  const T ny = T(2.0) * z.x * z.y - T(2.0) * z.w * z.z;
  const T nz = T(2.0) * z.x * z.z - T(2.0) * z.y * z.w;
  const T nw = T(2.0) * z.x * z.w - T(2.0) * z.y * z.z;
  z.x = nx;
  z.y = ny;
  z.z = nz;
  z.w = nw;
}

// cFractalQuaternion::FormulaCode (fractal_quaternion.cpp:29-39)
template <class T>
__device__ __forceinline__ void f_quaternion(V4<T> &z, T r, T &DE) {
  DE = DE * T(2.0) * r;
  const T nx = z.x * z.x - z.y * z.y - z.z * z.z;
  const T ny = T(2.0) * z.x * z.y;
  const T nz = T(2.0) * z.x * z.z;
  z.x = nx;
  z.y = ny;
  z.z = nz;
}

// cFractalAexion::FormulaCode (fractal_aexion.cpp:29-59): at the orbit's
// first iteration the point is folded into the tetrahedral frame and becomes
// the orbit's c (aux.const_c, which the c-addition of other slots also reads);
// 4-D, so the host sets has_w
template <class T>
__device__ __forceinline__ void f_aexion(V4<T> &z, T r, T &DE, const DevSlot &s, int i, V4<T> &c) {
  V4<T> temp = z;
  if (i == 0) {
    const T cadd = T(s.d[P_AEX_CADD]);
    temp.x = z.x + z.y + z.z;
    temp.y = -z.x - z.y + z.z;
    temp.z = -z.x + z.y - z.z;
    temp.w = z.x - z.y - z.z;
    z = V4<T>{m_abs(temp.x) + cadd, m_abs(temp.y) + cadd, m_abs(temp.z) + cadd, m_abs(temp.w) + cadd};
    c = z;
  }
  T t = T(2.0) * z.w * z.z;
  temp.x = z.x * z.x - z.y * z.y;
  temp.y = t - temp.x;
  temp.x = temp.x + t;
  t = T(2.0) * z.x * z.y;
  temp.z = z.z * z.z - z.w * z.w;
  temp.w = t - temp.z;
  temp.z = temp.z + t;
  z = V4<T>{temp.x + c.x, temp.y + c.y, temp.z + c.z, temp.w + c.w};
  if (s.d[P_ADE_ON] != 0.0) {
    T de1 = T(1.1) * r;
    de1 = de1 + (len4<T, true>(z) / r - de1) * T(s.d[P_ADE_SCALE1]);
    DE = de1 * T(2.0) * DE + T(s.d[P_ADE_OFFSET1]);
  }
}

// std::max(a, b) of the reference: b when a < b, else a.
template <class T>
__device__ __forceinline__ T smax(T a, T b) {
  return (a < b) ? b : a;
}

// The orbit state of sExtendedAux that keyed formulas carry from one
// iteration to the next (compute_fractal.cpp:118-127): pk =
// aux.pseudoKleinianDE (initially 1), scale = aux.actualScale (initially the
// Mandelbox scale of the sequence's first slot), scaleA = aux.actualScaleA
// (initially 0).
template <class T>
struct AuxX {
  T pk, scale, scaleA;
  T pn;     // aux.pos_neg (initially 1)
  T dist;   // aux.dist, the custom DE (initially 1000)
  V4<T> c;  // aux.c (initially the point), which aboxMod11's alternate c-addition permutes
};

// (x, y, z) reordered as mandelbulbMulti.orderOfXYZ says (enumMulti_OrderOfXYZ,
// fractal.h:282-289): xyz, xzy, yxz, yzx, zxy, zyx; w kept
template <class T>
__device__ __forceinline__ V4<T> order_xyz(const V4<T> &v, int order) {
  switch (order) {
    case 1: return V4<T>{v.x, v.z, v.y, v.w};
    case 2: return V4<T>{v.y, v.x, v.z, v.w};
    case 3: return V4<T>{v.y, v.z, v.x, v.w};
    case 4: return V4<T>{v.z, v.x, v.y, v.w};
    case 5: return V4<T>{v.z, v.y, v.x, v.w};
    default: return v;
  }
}

// sign() of math_utilities.h:65-67: -1, 0 or 1
template <class T>
__device__ __forceinline__ T sgn_of(T v) {
  return (T(0.0) < v) ? T(1.0) : ((v < T(0.0)) ? T(-1.0) : T(0.0));
}

// cFractalPseudoKleinian::FormulaCode (fractal_pseudo_kleinian.cpp:30-202)
// from the slot's keyed block (PseudoKleinianX); the aux.color terms are not
// computed.  pk: aux.pseudoKleinianDE, which the pseudo-Kleinian DE function
// reads.
template <class T>
__device__ __noinline__ void f_pseudo_kleinian(V4<T> &z, T &DE, T &pk, const DevSlot &s, int i) {
  const double *x = s.x;
  if (x[PKX_SPH_INV] != 0.0 && i >= int(x[PKX_START_X]) && i < int(x[PKX_STOP_1])) {  // :33-44
    z.x = z.x + T(x[PKX_OFFSET000]);
    z.y = z.y + T(x[PKX_OFFSET000 + 1]);
    z.z = z.z + T(x[PKX_OFFSET000 + 2]);
    const T rr = z.x * z.x + z.y * z.y + z.z * z.z + z.w * z.w;
    const T q = T(x[PKX_MAXR2]) / rr;
    z.x = z.x * q;
    z.y = z.y * q;
    z.z = z.z * q;
    z.w = z.w * q;
    z.x = z.x + T(x[PKX_ADD_A000] - x[PKX_OFFSET000]);
    z.y = z.y + T(x[PKX_ADD_A000 + 1] - x[PKX_OFFSET000 + 1]);
    z.z = z.z + T(x[PKX_ADD_A000 + 2] - x[PKX_OFFSET000 + 2]);
    DE = DE * (T(x[PKX_MAXR2]) / rr) + T(x[PKX_DE_OFFSET0]);
  }
  if (x[PKX_PRISM] != 0.0 && i >= int(x[PKX_START_P]) && i < int(x[PKX_STOP_P1])) {  // prism shape :47-75
    z.y = m_abs(z.y);
    z.z = m_abs(z.z);
    const T dot1 = (z.x * T(-0.86602540378443864676372317075294) + z.y * T(0.5)) * T(x[PKX_SCALE]);
    T t = smax(T(0.0), dot1);
    z.x = z.x - t * T(-1.73205080756887729352744634150587);
    z.y = m_abs(T(z.y - t));
    if (z.y > z.z) {
      t = z.y;
      z.y = z.z;
      z.z = t;
    }
    z.x = z.x - T(x[PKX_CMUL000] * 0.86602540378443864676372317075294);
    z.y = z.y - T(x[PKX_CMUL000 + 1] * 1.5);
    z.z = z.z - T(x[PKX_CMUL000 + 2] * 1.5);
    if (z.z > z.x) {
      t = z.z;
      z.z = z.x;
      z.x = t;
    }
    if (z.x > T(0.0)) {
      z.y = smax(T(0.0), z.y);
      z.z = smax(T(0.0), z.z);
    }
  }
  if (x[PKX_ABS_BOX] != 0.0 && i >= int(x[PKX_START_E]) && i < int(x[PKX_STOP_E])) {  // abs box fold :78-91
    const T ax = T(x[PKX_ADD111]), ay = T(x[PKX_ADD111 + 1]), az = T(x[PKX_ADD111 + 2]);
    z.x = m_abs(T(z.x + ax)) - m_abs(T(z.x - ax)) - z.x;
    z.y = m_abs(T(z.y + ay)) - m_abs(T(z.y - ay)) - z.y;
    if (x[PKX_ABS_BOX_Z] != 0.0) z.z = m_abs(T(z.z + az)) - m_abs(T(z.z - az)) - z.z;
  }
  if (x[PKX_BOX] != 0.0 && i >= int(x[PKX_START_A]) && i < int(x[PKX_STOP_A])) {  // box fold :94-115
    const T limit = T(x[PKX_MB_LIMIT]), value = T(x[PKX_MB_VALUE]);
    if (m_abs(z.x) > limit) z.x = sgn_of(z.x) * value - z.x;
    if (m_abs(z.y) > limit) z.y = sgn_of(z.y) * value - z.y;
    const T zLimit = T(x[PKX_MB_LIMIT] * x[PKX_SCALE1]);
    const T zValue = T(x[PKX_MB_VALUE] * x[PKX_SCALE1]);
    if (m_abs(z.z) > zLimit) z.z = sgn_of(z.z) * zValue - z.z;
  }
  if (i >= int(x[PKX_START_C]) && i < int(x[PKX_STOP_C])) {  // the Kleinian fold :118-138
    const T cx = T(x[PKX_CSIZE]), cy = T(x[PKX_CSIZE + 1]), cz = T(x[PKX_CSIZE + 2]);
    V4<T> t = z;
    if (z.x > cx) t.x = cx;
    if (z.x < -cx) t.x = -cx;
    if (z.y > cy) t.y = cy;
    if (z.y < -cy) t.y = -cy;
    if (z.z > cz) t.z = cz;
    if (z.z < -cz) t.z = -cz;
    z.x = t.x * T(2.0) - z.x;
    z.y = t.y * T(2.0) - z.y;
    z.z = t.z * T(2.0) - z.z;
    z.w = t.w * T(2.0) - z.w;
    const T k = smax(T(T(x[PKX_MINR05]) / (z.x * z.x + z.y * z.y + z.z * z.z + z.w * z.w)), T(1.0));
    z.x = z.x * k;
    z.y = z.y * k;
    z.z = z.z * k;
    z.w = z.w * k;
    if (x[PKX_FLIP_Z] != 0.0) z.z = -z.z;
    if (x[PKX_FLIP_W] != 0.0) z.w = -z.w;
    DE = DE * (k + T(x[PKX_TWEAK005]));
    pk = T(x[PKX_DE_SCALE1]);
  }
  if (x[PKX_ROT_ON] != 0.0 && i >= int(x[PKX_START_R]) && i < int(x[PKX_STOP_R]) && x[PKX_ROT] == 0.0)
    z = mb_turn<T>(x + PKX_ROT + 1, false, z);  // :141-144 (the matrix's zero flag first)
  z.x = z.x + T(x[PKX_ADD000]);  // :147
  z.y = z.y + T(x[PKX_ADD000 + 1]);
  z.z = z.z + T(x[PKX_ADD000 + 2]);
}

// cFractalBoxFoldBulbPow2::FormulaCode (fractal_box_fold_bulb_pow2.cpp:27-76):
// a box fold, the fixed spherical fold (min radius^2 0.25, fixed 1), then the
// power-2 bulb with its z factor; a delta-DE formula (its analytic DE terms
// apply only under a forced analytic method)
template <class T>
__device__ __noinline__ void f_box_fold_bulb_pow2(V4<T> &z, T r, T &DE, const DevSlot &s) {
  const double *x = s.x;
  const double ff = x[BFX_FOLD];
  if (m_abs(z.x) > T(ff)) z.x = T(double(sgn_of(z.x)) * ff * 2.0) - z.x;
  if (m_abs(z.y) > T(ff)) z.y = T(double(sgn_of(z.y)) * ff * 2.0) - z.y;
  if (m_abs(z.z) > T(ff)) z.z = T(double(sgn_of(z.z)) * ff * 2.0) - z.z;
  const T r2 = z.x * z.x + z.y * z.y + z.z * z.z + z.w * z.w;
  if (r2 < T(0.25)) {
    z.x = z.x * T(4.0);
    z.y = z.y * T(4.0);
    z.z = z.z * T(4.0);
    z.w = z.w * T(4.0);
    DE = DE * T(4.0);
  } else if (r2 < T(1.0)) {
    const T f2 = T(1.0) / r2;
    z.x = z.x * f2;
    z.y = z.y * f2;
    z.z = z.z * f2;
    z.w = z.w * f2;
    DE = DE * f2;
  }
  z.x = z.x * T(2.0);
  z.y = z.y * T(2.0);
  z.z = z.z * T(2.0);
  z.w = z.w * T(2.0);
  const T x2 = z.x * z.x, y2 = z.y * z.y, z2 = z.z * z.z;
  const T temp = T(1.0) - z2 / (x2 + y2);
  const T nx = (x2 - y2) * temp;
  const T ny = T(2.0) * z.x * z.y * temp;
  const T nz = T(-2.0) * z.z * m_sqrt(T(x2 + y2));
  z.x = nx;
  z.y = ny;
  z.z = nz * T(x[BFX_ZFACTOR]);
  if (x[BFX_ADE_ON] != 0.0)  // :67-73
    DE = (DE + T(1.0)) * T(5.0) * r * T(x[BFX_ADE_SCALE1]) *
             T(sqrt(x[BFX_ZFACTOR] * x[BFX_ZFACTOR] + 2.0 + x[BFX_ADE_OFFSET2])) +
         T(x[BFX_ADE_OFFSET1]);
}

// cFractalBoxFoldBulbPow2V2::FormulaCode (fractal_box_fold_bulb_pow2_v2.cpp:
// 29-146), the aux.color terms left out: tglad fold, spherical fold, a scale
// that may vary from one iteration to the next (scaleA = aux.actualScaleA),
// the power-2 bulb with its z factor
template <class T>
__device__ __noinline__ void f_box_fold_bulb_pow2_v2(V4<T> &z, T &DE, T &scaleA, const DevSlot &s, int i) {
  const double *x = s.x;
  if (i >= int(x[B2X_START_B]) && i < int(x[B2X_STOP_B])) {  // tglad fold :35-45
    const T ax = T(x[B2X_ADD111]), ay = T(x[B2X_ADD111 + 1]), az = T(x[B2X_ADD111 + 2]);
    z.x = m_abs(T(z.x + ax)) - m_abs(T(z.x - ax)) - z.x;
    z.y = m_abs(T(z.y + ay)) - m_abs(T(z.y - ay)) - z.y;
    z.z = m_abs(T(z.z + az)) - m_abs(T(z.z - az)) - z.z;
  }
  if (i >= int(x[B2X_START_S]) && i < int(x[B2X_STOP_S])) {  // spherical fold :48-67
    const T rr = z.x * z.x + z.y * z.y + z.z * z.z + z.w * z.w;
    const T ox = T(x[B2X_MB_OFFSET]), oy = T(x[B2X_MB_OFFSET + 1]), oz = T(x[B2X_MB_OFFSET + 2]);
    z.x = z.x + ox;
    z.y = z.y + oy;
    z.z = z.z + oz;
    if (rr < T(x[B2X_MINR2])) {
      const T f1 = T(x[B2X_MAXR2] / x[B2X_MINR2]);
      z.x = z.x * f1;
      z.y = z.y * f1;
      z.z = z.z * f1;
      z.w = z.w * f1;
      DE = DE * f1;
    } else if (rr < T(x[B2X_MAXR2])) {
      const T f2 = T(x[B2X_MAXR2]) / rr;
      z.x = z.x * f2;
      z.y = z.y * f2;
      z.z = z.z * f2;
      z.w = z.w * f2;
      DE = DE * f2;
    }
    z.x = z.x - ox;
    z.y = z.y - oy;
    z.z = z.z - oz;
  }
  if (i >= int(x[B2X_START_C]) && i < int(x[B2X_STOP_C])) {  // scale :70-88
    const T useScale = scaleA + T(x[B2X_SCALE]);
    z.x = z.x * useScale;
    z.y = z.y * useScale;
    z.z = z.z * useScale;
    z.w = z.w * useScale;
    DE = DE * m_abs(useScale);
    if (i >= int(x[B2X_START_X]) && i < int(x[B2X_STOP_X])) {
      const T vary = T(x[B2X_SCALE_VARY]) * (m_abs(scaleA) - T(x[B2X_SCALE_B1]));
      scaleA = (x[B2X_VARY_M] != 0.0) ? T(-vary) : T(scaleA - vary);
    }
  }
  if (i >= int(x[B2X_START_A]) && i < int(x[B2X_STOP_A])) {  // :90-110
    const T r = len4<T, true>(z);
    DE = r * DE * T(16.0) * T(x[B2X_ADE_SCALE1]) *
             T(sqrt(x[B2X_ZFACTOR] * x[B2X_ZFACTOR] + 2.0 + x[B2X_ADE_OFFSET2])) /
             T(1.73205080756887729352744634150587) +
         T(x[B2X_ADE_OFFSET1]);
    z.x = z.x * T(2.0);
    z.y = z.y * T(2.0);
    z.z = z.z * T(2.0);
    z.w = z.w * T(2.0);
    const T x2 = z.x * z.x, y2 = z.y * z.y, z2 = z.z * z.z;
    const T temp = T(1.0) - z2 / (x2 + y2);
    const T nx = (x2 - y2) * temp;
    const T ny = T(2.0) * z.x * z.y * temp;
    const T nz = T(-2.0) * z.z * m_sqrt(T(x2 + y2));
    z.x = nx;
    z.y = ny;
    z.z = nz * T(x[B2X_ZFACTOR]);
  }
}

// cFractalAboxMod11::FormulaCode (fractal_abox_mod11.cpp:34-250), the
// aux.color terms left out: a scale that varies with |aux.actualScale|, tglad
// fold, the smooth fold, a swap, a spherical fold whose inner radius follows
// a curve over the iterations, scale, offset, c-addition (optionally of aux.c
// permuted every iteration), rotation and a tweak scale.  c: aux.const_c.
template <class T>
__device__ __noinline__ void f_abox_mod11(V4<T> &z, T &DE, AuxX<T> &ax, const V4<T> &c, const DevSlot &s, int i) {
  const double *x = s.x;
  ax.scale = T(x[ABX_MB_SCALE] + x[ABX_SCALE_VARY] * (fabs(double(ax.scale)) - 1.0));  // :36-37
  if (i >= int(x[ABX_START_B]) && i < int(x[ABX_STOP_B])) {  // tglad fold :41-55
    const T ax0 = T(x[ABX_ADD111]), ay = T(x[ABX_ADD111 + 1]), az = T(x[ABX_ADD111 + 2]);
    z.x = m_abs(T(z.x + ax0)) - m_abs(T(z.x - ax0)) - z.x;
    z.y = m_abs(T(z.y + ay)) - m_abs(T(z.y - ay)) - z.y;
    if (x[ABX_FOLD_Z] != 0.0) z.z = m_abs(T(z.z + az)) - m_abs(T(z.z - az)) - z.z;
  }
  if (x[ABX_FOLD_D] != 0.0 && i >= int(x[ABX_START_D]) && i < int(x[ABX_STOP_D1])) {  // :56-77
    T *zc[3] = {&z.x, &z.y, &z.z};
    T add[3];
    for (int a = 0; a < 3; a++) {
      const double lim = x[ABX_ADD111 + a], len = 2.0 * lim, tS = 1.0 / len;
      const T v = *zc[a], av = m_abs(v);
      add[a] = T(0.0);
      if (av < T(lim)) add[a] = v * v * T(tS);
      if (av > T(lim) && av < T(len)) add[a] = (T(len) - av) * (T(len) - av) * T(tS);
      add[a] = add[a] * T(x[ABX_SCALE3D + a]);
    }
    for (int a = 0; a < 3; a++) *zc[a] = *zc[a] - sgn_of(*zc[a]) * add[a];
  }
  if (x[ABX_SWAP] != 0.0) z = V4<T>{z.z, z.y, z.x, z.w};  // :79-82
  if (i >= int(x[ABX_START_S]) && i < int(x[ABX_STOP_S])) {  // spherical fold :85-174
    const double para = abox_mod11_para(x, i);
    const T rr = z.x * z.x + z.y * z.y + z.z * z.z + z.w * z.w;
    const T ox = T(x[ABX_MB_OFFSET]), oy = T(x[ABX_MB_OFFSET + 1]), oz = T(x[ABX_MB_OFFSET + 2]);
    z.x = z.x + ox;
    z.y = z.y + oy;
    z.z = z.z + oz;
    if (rr < T(para)) {
      const T f1 = T(x[ABX_MAXR2] / para);
      z.x = z.x * f1;
      z.y = z.y * f1;
      z.z = z.z * f1;
      z.w = z.w * f1;
      DE = DE * f1;
    } else if (rr < T(x[ABX_MAXR2])) {
      const T f2 = T(x[ABX_MAXR2]) / rr;
      z.x = z.x * f2;
      z.y = z.y * f2;
      z.z = z.z * f2;
      z.w = z.w * f2;
      DE = DE * f2;
    }
    z.x = z.x - ox;
    z.y = z.y - oy;
    z.z = z.z - oz;
  }
  if (i >= int(x[ABX_START_A]) && i < int(x[ABX_STOP_A])) {  // scale :177-186
    z.x = z.x * ax.scale;
    z.y = z.y * ax.scale;
    z.z = z.z * ax.scale;
    z.w = z.w * ax.scale;
    if (x[ABX_ADE_ON] == 0.0) DE = DE * m_abs(ax.scale) + T(1.0);
    else DE = DE * m_abs(ax.scale) * T(x[ABX_ADE_SCALE1]) + T(x[ABX_ADE_OFFSET1]);
  }
  z.x = z.x + T(x[ABX_ADD000]);  // :188
  z.y = z.y + T(x[ABX_ADD000 + 1]);
  z.z = z.z + T(x[ABX_ADD000 + 2]);
  if (x[ABX_ADDC] != 0.0 && i >= int(x[ABX_START_E]) && i < int(x[ABX_STOP_E])) {  // :191-225
    V4<T> t;
    if (x[ABX_ALTERNATE] != 0.0) {
      t = order_xyz(ax.c, int(x[ABX_ORDER]));
      ax.c = t;
    } else {
      t = order_xyz(c, int(x[ABX_ORDER]));
    }
    z.x = z.x + t.x * T(x[ABX_CM111]);
    z.y = z.y + t.y * T(x[ABX_CM111 + 1]);
    z.z = z.z + t.z * T(x[ABX_CM111 + 2]);
    z.w = z.w + t.w * T(1.0);
  }
  if (x[ABX_ROT_ON] != 0.0 && i >= int(x[ABX_START_R]) && i < int(x[ABX_STOP_R]) && x[ABX_ROT] == 0.0)
    z = mb_turn<T>(x + ABX_ROT + 1, false, z);  // :227-232
  if (i >= int(x[ABX_START_C]) && i < int(x[ABX_STOP_C1])) {  // tweak scale :234-239
    const T g = T(x[ABX_SCALE_G1]);
    z.x = z.x * g;
    z.y = z.y * g;
    z.z = z.z * g;
    z.w = z.w * g;
    DE = DE * T(fabs(x[ABX_SCALE_G1]));
  }
}

// cFractalPseudoKleinianMod4::FormulaCode (fractal_pseudo_kleinian_mod4.cpp:
// 29-145) without the aux.color terms; pk and pos_neg are
// aux.pseudoKleinianDE and aux.pos_neg
template <class T>
__device__ __noinline__ void f_pseudo_kleinian_mod4(V4<T> &z, T &DE, AuxX<T> &ax, const DevSlot &s, int i) {
  const double *x = s.x;
  if (x[P4X_SPH_INV] != 0.0 && i >= int(x[P4X_START_X]) && i < int(x[P4X_STOP_1])) {  // :37-47
    z.x = z.x + T(x[P4X_OFFSET000]);
    z.y = z.y + T(x[P4X_OFFSET000 + 1]);
    z.z = z.z + T(x[P4X_OFFSET000 + 2]);
    const T rr = z.x * z.x + z.y * z.y + z.z * z.z + z.w * z.w;
    const T q = T(x[P4X_SCALE_G1]) / rr;
    z.x = z.x * q;
    z.y = z.y * q;
    z.z = z.z * q;
    z.w = z.w * q;
    DE = DE * (T(x[P4X_SCALE_G1]) / rr);
    z.x = z.x + T(x[P4X_ADD_P000] - x[P4X_OFFSET000]);
    z.y = z.y + T(x[P4X_ADD_P000 + 1] - x[P4X_OFFSET000 + 1]);
    z.z = z.z + T(x[P4X_ADD_P000 + 2] - x[P4X_OFFSET000 + 2]);
    const T a1 = T(x[P4X_SCALE_A1]);
    z.x = z.x * a1;
    z.y = z.y * a1;
    z.z = z.z * a1;
    z.w = z.w * a1;
    DE = DE * a1;
  }
  if (i >= int(x[P4X_START_M]) && i < int(x[P4X_STOP_M])) {  // box offset :49-55
    z.x = z.x - T(x[P4X_CM000]) * sgn_of(z.x);
    z.y = z.y - T(x[P4X_CM000 + 1]) * sgn_of(z.y);
    z.z = z.z - T(x[P4X_CM000 + 2]) * sgn_of(z.z);
  }
  {  // the Kleinian fold :58-66
    const T cx = T(x[P4X_CSIZE]), cy = T(x[P4X_CSIZE + 1]), cz = T(x[P4X_CSIZE + 2]);
    z.x = m_abs(T(z.x + cx)) - m_abs(T(z.x - cx)) - z.x;
    z.y = m_abs(T(z.y + cy)) - m_abs(T(z.y - cy)) - z.y;
    z.z = m_abs(T(z.z + cz)) - m_abs(T(z.z - cz)) - z.z;
    z.w = m_abs(z.w) - m_abs(z.w) - z.w;
    const T k = smax(T(T(x[P4X_MINR05]) / (z.x * z.x + z.y * z.y + z.z * z.z + z.w * z.w)), T(1.0));
    z.x = z.x * k;
    z.y = z.y * k;
    z.z = z.z * k;
    z.w = z.w * k;
    DE = DE * (k + T(x[P4X_TWEAK005]));
    ax.pk = T(x[P4X_DE_SCALE1]);
  }
  z.x = z.x + T(x[P4X_ADD000]);
  z.y = z.y + T(x[P4X_ADD000 + 1]);
  z.z = z.z + T(x[P4X_ADD000 + 2]);
  if (x[P4X_G_ON] != 0.0 && i >= int(x[P4X_START_G]) && i < int(x[P4X_STOP_G])) {  // :70-78
    z.x = z.x + ax.pn * T(x[P4X_ADD_A000]);
    z.y = z.y + ax.pn * T(x[P4X_ADD_A000 + 1]);
    z.z = z.z + ax.pn * T(x[P4X_ADD_A000 + 2]);
    ax.pn = ax.pn * T(x[P4X_SCALE_NEG1]);
  }
  if (x[P4X_F_ON] != 0.0 && i >= int(x[P4X_START_F]) && i < int(x[P4X_STOP_F])) {  // :80-85
    const T ox = T(x[P4X_OFFSET_A000]), oy = T(x[P4X_OFFSET_A000 + 1]), oz = T(x[P4X_OFFSET_A000 + 2]);
    z.x = m_abs(T(z.x + ox)) - m_abs(T(z.x - ox)) - z.x;
    z.y = m_abs(T(z.y + oy)) - m_abs(T(z.y - oy)) - z.y;
    z.z = m_abs(T(z.z + oz)) - m_abs(T(z.z - oz)) - z.z;
    z.w = m_abs(z.w) - m_abs(z.w) - z.w;
  }
  if (x[P4X_N_ON] != 0.0 && i >= int(x[P4X_START_N]) && i < int(x[P4X_STOP_N])) {  // :87-127
    T t;
    z.x = m_abs(z.x);
    z.y = m_abs(z.y);
    if (x[P4X_SWAP_A] != 0.0) {
      t = z.x;
      z.x = z.y;
      z.y = t;
    }
    t = z.x;
    z.x = z.x + z.y - T(x[P4X_OFFSET0]);
    z.y = t - z.y - T(x[P4X_OFFSET_A0]);
    if (x[P4X_BX_F] != 0.0 && i >= int(x[P4X_START_O]) && i < int(x[P4X_STOP_O])) z.x = -m_abs(z.x);
    if (x[P4X_BX] != 0.0 && i >= int(x[P4X_START_P]) && i < int(x[P4X_STOP_P])) z.y = -m_abs(z.y);
    t = z.x;
    z.x = z.x + z.y;
    z.y = t - z.y;
    z.x = z.x * T(0.5);
    z.y = z.y * T(0.5);
    if (x[P4X_AX] != 0.0 && i >= int(x[P4X_START_R]) && i < int(x[P4X_STOP_R]))
      z.x = T(x[P4X_OFFSET1]) - m_abs(T(z.x + T(x[P4X_OFFSET1])));
    if (x[P4X_AX_F] != 0.0 && i >= int(x[P4X_START_RV]) && i < int(x[P4X_STOP_RV]))
      z.y = T(x[P4X_OFFSET_A1]) - m_abs(T(z.y + T(x[P4X_OFFSET_A1])));
  }
  if (x[P4X_FLIP_X] != 0.0) z.x = -z.x;
  if (x[P4X_FLIP_Y] != 0.0) z.y = -z.y;
  if (x[P4X_FLIP_Z] != 0.0) z.z = -z.z;
}

// the tetrahedral frame turn of Benesi's transforms (SQRT_1_3, SQRT_2_3,
// SQRT_1_2 of abstract_fractal.h:30-32): into the frame and back
template <class T>
__device__ __forceinline__ V4<T> benesi_in(const V4<T> &z) {
  const T t = z.x * T(0.81649658092772603273242802490196) - z.z * T(0.57735026918962576450914878050196);
  return V4<T>{(t - z.y) * T(0.70710678118654752440084436210485), (t + z.y) * T(0.70710678118654752440084436210485),
               z.x * T(0.57735026918962576450914878050196) + z.z * T(0.81649658092772603273242802490196), z.w};
}
template <class T>
__device__ __forceinline__ V4<T> benesi_out(const V4<T> &z) {
  const T t = (z.y + z.x) * T(0.70710678118654752440084436210485);
  return V4<T>{z.z * T(0.57735026918962576450914878050196) + t * T(0.81649658092772603273242802490196),
               (z.y - z.x) * T(0.70710678118654752440084436210485),
               z.z * T(0.81649658092772603273242802490196) - t * T(0.57735026918962576450914878050196), z.w};
}

// cFractalPseudoKleinianStdDE::FormulaCode (fractal_pseudo_kleinian_std_de.cpp:
// 29-215) without the aux.color terms: prism, rotation, Benesi's T1 and the
// T1 mod, an abs fold, a Menger fold, the Kleinian fold (two variants) and
// the custom distance aux.dist (ax.dist)
template <class T>
__device__ __noinline__ void f_pseudo_kleinian_std_de(V4<T> &z, T &DE, AuxX<T> &ax, const DevSlot &s, int i) {
  const double *x = s.x;
  if (x[PSX_P_ON] != 0.0 && i >= int(x[PSX_START_P]) && i < int(x[PSX_STOP_P1])) {  // prism :38-58
    z.y = m_abs(z.y);
    z.z = m_abs(z.z);
    const T dot1 = (z.x * T(-0.86602540378443864676372317075294) + z.y * T(0.5)) * T(x[PSX_SCALE]);
    T t = smax(T(0.0), dot1);
    z.x = z.x - t * T(-1.73205080756887729352744634150587);
    z.y = m_abs(T(z.y - t));
    if (z.y > z.z) {
      t = z.y;
      z.y = z.z;
      z.z = t;
    }
    z.x = z.x - T(x[PSX_CM000] * 0.86602540378443864676372317075294);
    z.y = z.y - T(x[PSX_CM000 + 1] * 1.5);
    z.z = z.z - T(x[PSX_CM000 + 2] * 1.5);
    if (z.z > z.x) {
      t = z.z;
      z.z = z.x;
      z.x = t;
    }
    if (z.x > T(0.0)) {
      z.y = smax(T(0.0), z.y);
      z.z = smax(T(0.0), z.z);
    }
  }
  if (x[PSX_R_ON] != 0.0 && i >= int(x[PSX_START_R]) && i < int(x[PSX_STOP_R]) && x[PSX_ROT] == 0.0)
    z = mb_turn<T>(x + PSX_ROT + 1, false, z);  // :60-63
  if (x[PSX_T1_ON] != 0.0 && i >= int(x[PSX_START]) && i < int(x[PSX_STOP_T1])) {  // benesi T1 :65-83
    z = benesi_in(z);
    const T tempL = len4<T, true>(z);
    z = V4<T>{m_abs(z.x) * T(x[PSX_S222]), m_abs(z.y) * T(x[PSX_S222 + 1]), m_abs(z.z) * T(x[PSX_S222 + 2]),
              m_abs(z.w)};
    const T avgScale = len4<T, true>(z) / tempL;
    DE = DE * avgScale + T(1.0);
    z = benesi_out(z);
    z.x = z.x - T(x[PSX_OFF200]);
    z.y = z.y - T(x[PSX_OFF200 + 1]);
    z.z = z.z - T(x[PSX_OFF200 + 2]);
  }
  if (x[PSX_TM_ON] != 0.0 && i >= int(x[PSX_START_D]) && i < int(x[PSX_STOP_TM1])) {  // benesi T1 mod :85-104
    z = benesi_in(z);
    const T tempL = len4<T, true>(z);
    z = V4<T>{m_abs(z.x) * T(x[PSX_S333]), m_abs(z.y) * T(x[PSX_S333 + 1]), m_abs(z.z) * T(x[PSX_S333 + 2]),
              m_abs(z.w)};
    const T avgScale = len4<T, true>(z) / tempL;
    DE = DE * avgScale + T(1.0);
    const T ax0 = T(x[PSX_ADD111]), ay = T(x[PSX_ADD111 + 1]), az = T(x[PSX_ADD111 + 2]);
    z.x = m_abs(T(z.x + ax0)) - m_abs(T(z.x - ax0)) - z.x;
    z.y = m_abs(T(z.y + ay)) - m_abs(T(z.y - ay)) - z.y;
    z.z = m_abs(T(z.z + az)) - m_abs(T(z.z - az)) - z.z;
    z.w = m_abs(z.w) - m_abs(z.w) - z.w;
    z = benesi_out(z);
  }
  if (x[PSX_F_ON] != 0.0 && i >= int(x[PSX_START_F]) && i < int(x[PSX_STOP_F])) {  // :106-127
    T ta = T(0.0), tb = T(0.0);
    if (x[PSX_F_AX] != 0.0) ta = m_abs(T(z.x + T(x[PSX_OFFF000])));
    if (x[PSX_F_X] != 0.0) tb = m_abs(T(z.x - T(x[PSX_OFF000])));
    z.x = ta - tb - (z.x * T(x[PSX_S111]));
    ta = T(0.0);
    tb = T(0.0);
    if (x[PSX_F_AY] != 0.0) ta = m_abs(T(z.y + T(x[PSX_OFFF000 + 1])));
    if (x[PSX_F_Y] != 0.0) tb = m_abs(T(z.y - T(x[PSX_OFF000 + 1])));
    z.y = ta - tb - (z.y * T(x[PSX_S111 + 1]));
    ta = T(0.0);
    tb = T(0.0);
    if (x[PSX_F_AZ] != 0.0) ta = m_abs(T(z.z + T(x[PSX_OFFF000 + 2])));
    if (x[PSX_F_Z] != 0.0) tb = m_abs(T(z.z - T(x[PSX_OFF000 + 2])));
    z.z = ta - tb - (z.z * T(x[PSX_S111 + 2]));
  }
  if (x[PSX_M_ON] != 0.0 && i >= int(x[PSX_START_M]) && i < int(x[PSX_STOP_M])) {  // Menger fold :129-142
    z = V4<T>{m_abs(z.x), m_abs(z.y), m_abs(z.z), m_abs(z.w)};
    T t;
    if (z.x - z.y < T(0.0)) {
      t = z.y;
      z.y = z.x;
      z.x = t;
    }
    if (z.x - z.z < T(0.0)) {
      t = z.z;
      z.z = z.x;
      z.x = t;
    }
    if (z.y - z.z < T(0.0)) {
      t = z.z;
      z.z = z.y;
      z.y = t;
    }
    const T s3 = T(x[PSX_SCALE3]);
    z.x = z.x * s3;
    z.y = z.y * s3;
    z.z = z.z * s3;
    z.w = z.w * s3;
    z.x = z.x - T(2.0 * x[PSX_CMA111]);
    z.y = z.y - T(2.0 * x[PSX_CMA111 + 1]);
    if (z.z > T(1.0)) z.z = z.z - T(2.0 * x[PSX_CMA111 + 2]);
    DE = DE * T(x[PSX_SCALE3] * x[PSX_SCALE_A1]);
    z.x = z.x + T(x[PSX_ADD_A000]);
    z.y = z.y + T(x[PSX_ADD_A000 + 1]);
    z.z = z.z + T(x[PSX_ADD_A000 + 2]);
  }
  if (x[PSX_FLIP_Z] != 0.0) z.z = -z.z;
  const T cx = T(x[PSX_CSIZE]), cy = T(x[PSX_CSIZE + 1]), cz = T(x[PSX_CSIZE + 2]);
  if (x[PSX_AW] != 0.0 && i >= int(x[PSX_START_C]) && i < int(x[PSX_STOP_C])) {  // :148-166
    V4<T> t = z;
    if (z.x > cx) t.x = cx;
    if (z.x < -cx) t.x = -cx;
    if (z.y > cy) t.y = cy;
    if (z.y < -cy) t.y = -cy;
    if (z.z > cz) t.z = cz;
    if (z.z < -cz) t.z = -cz;
    const T b1 = T(x[PSX_SCALE_B1]);
    z.x = z.x * b1;
    z.y = z.y * b1;
    z.z = z.z * b1;
    z.w = z.w * b1;
    DE = DE * T(fabs(x[PSX_SCALE_B1]));
    z.x = t.x * T(2.0) - z.x;
    z.y = t.y * T(2.0) - z.y;
    z.z = t.z * T(2.0) - z.z;
    z.w = t.w * T(2.0) - z.w;
    const T k = smax(T(T(x[PSX_MINR05]) / (z.x * z.x + z.y * z.y + z.z * z.z + z.w * z.w)), T(1.0));
    z.x = z.x * k;
    z.y = z.y * k;
    z.z = z.z * k;
    z.w = z.w * k;
    DE = DE * (k + T(x[PSX_TWEAK005]));
  }
  if (x[PSX_AYF] != 0.0 && i >= int(x[PSX_START_B]) && i < int(x[PSX_STOP_B])) {  // :167-181
    if (z.x > cx) z.x = T(x[PSX_CSIZE] * 2.0) - z.x;
    if (z.x < -cx) z.x = T(-x[PSX_CSIZE] * 2.0) - z.x;
    if (z.y > cy) z.y = T(x[PSX_CSIZE + 1] * 2.0) - z.y;
    if (z.y < -cy) z.y = T(-x[PSX_CSIZE + 1] * 2.0) - z.y;
    if (z.z > cz) z.z = T(x[PSX_CSIZE + 2] * 2.0) - z.z;
    if (z.z < -cz) z.z = T(-x[PSX_CSIZE + 2] * 2.0) - z.z;
    const T k = smax(T(T(x[PSX_MINR05]) / (z.x * z.x + z.y * z.y + z.z * z.z + z.w * z.w)), T(1.0));
    z.x = z.x * k;
    z.y = z.y * k;
    z.z = z.z * k;
    z.w = z.w * k;
    DE = DE * (k + T(x[PSX_TWEAK005]));
  }
  z.x = z.x + T(x[PSX_ADD000]);  // :182
  z.y = z.y + T(x[PSX_ADD000 + 1]);
  z.z = z.z + T(x[PSX_ADD000 + 2]);
  ax.dist = m_sqrt(T(z.x * z.x + z.y * z.y)) / DE;  // :183
}

// three-vector helpers of the generalized fold box (CVector3 Dot, Cross)
template <class T>
struct G3 {
  T x, y, z;
};
template <class T>
__device__ __forceinline__ T g3dot(const G3<T> &a, const G3<T> &b) {
  return a.x * b.x + a.y * b.y + a.z * b.z;
}

// cFractalGeneralizedFoldBox::FormulaCode (fractal_generalized_fold_box.cpp:
// 31-245), the aux.color terms left out: a fold in the planes of a
// polyhedron (mirror, rotation line or inversion point, above the melt
// layer), then the Mandelbox sphere fold, main rotation and scale
template <class T>
__device__ __noinline__ void f_generalized_fold_box(V4<T> &z, T &DE, const DevSlot &s) {
  const double *x = s.x;
  const int sides = int(x[GFX_SIDES]);
  const T solid = T(x[GFX_SOLID]), melt = T(x[GFX_MELT]);
  auto nv = [&](int i) { return G3<T>{T(x[GFX_NV + 3 * i]), T(x[GFX_NV + 3 * i + 1]), T(x[GFX_NV + 3 * i + 2])}; };
  G3<T> zz{z.x, z.y, z.z};
  G3<T> L = zz;
  T a = T(1.0);
  int side = -1;
  for (int i = 0; i < sides; i++) {  // the closest plane cutting the line origin..z
    const T b = solid, c = g3dot(L, nv(i));
    if ((c > T(0.0)) && ((a * c) > b)) {
      side = i;
      a = b / c;
    }
  }
  if (side != -1) {
    const int side_m = side;
    const G3<T> Nm = nv(side_m);
    const T dm = g3dot(zz, Nm) - solid;
    const G3<T> Xm{zz.x - Nm.x * dm, zz.y - Nm.y * dm, zz.z - Nm.z * dm};
    L = G3<T>{Xm.x - Nm.x, Xm.y - Nm.y, Xm.z - Nm.z};
    G3<T> Y = Nm;
    a = T(1.0);
    side = -1;
    for (int i = 0; i < sides; i++) {
      if (i != side_m) {
        const T b = solid - g3dot(Y, nv(i)), c = g3dot(L, nv(i));
        if ((c > T(0.0)) && ((a * c) > b)) {
          side = i;
          a = b / c;
        }
      }
    }
    G3<T> target;
    if (side != -1) {  // rotation check
      const G3<T> Xmr{Y.x + L.x * a, Y.y + L.y * a, Y.z + L.z * a};
      const int side_r = side;
      const G3<T> Nr = nv(side_r);
      G3<T> Lr{Nm.y * Nr.z - Nm.z * Nr.y, -Nm.x * Nr.z + Nm.z * Nr.x, Nm.x * Nr.y - Nm.y * Nr.x};
      T a_rmin = (g3dot(zz, Lr) - g3dot(Xmr, Lr)) / (g3dot(Lr, Lr));
      if (a_rmin < T(0.0)) {
        a_rmin = -a_rmin;
        Lr = G3<T>{Lr.x * T(-1.0), Lr.y * T(-1.0), Lr.z * T(-1.0)};
      }
      const G3<T> Xr{Xmr.x + Lr.x * a_rmin, Xmr.y + Lr.y * a_rmin, Xmr.z + Lr.z * a_rmin};
      L = G3<T>{Xr.x - Xmr.x, Xr.y - Xmr.y, Xr.z - Xmr.z};
      Y = Xmr;
      a = T(1.0);
      side = -1;
      for (int i = 0; i < sides; i++) {
        if ((i != side_m) && (i != side_r)) {
          const T b = solid - g3dot(Y, nv(i)), c = g3dot(L, nv(i));
          if ((c > T(0.0)) && ((a * c) > b)) {
            side = i;
            a = b / c;
          }
        }
      }
      target = (side != -1) ? G3<T>{Y.x + L.x * a, Y.y + L.y * a, Y.z + L.z * a} : Xr;
    } else {
      target = Xm;
    }
    const G3<T> z2X{target.x - zz.x, target.y - zz.y, target.z - zz.z};
    if (g3dot(z2X, z2X) > (melt * melt)) {  // above the melt layer
      const T mag = m_sqrt(g3dot(z2X, z2X));
      const T k = T(2.0) * (mag - melt) / (mag + T(.00000001));
      zz = G3<T>{zz.x + z2X.x * k, zz.y + z2X.y * k, zz.z + z2X.z * k};
    }
  }
  const T r2 = g3dot(zz, zz);
  z.x = zz.x + T(x[GFX_MB_OFFSET]);
  z.y = zz.y + T(x[GFX_MB_OFFSET + 1]);
  z.z = zz.z + T(x[GFX_MB_OFFSET + 2]);
  const double mR2 = x[GFX_MB_MINR] * x[GFX_MB_MINR], fR2 = x[GFX_MB_FIXEDR] * x[GFX_MB_FIXEDR];
  if (r2 < T(mR2)) {
    const T f1 = T(fR2 / mR2);
    z.x = z.x * f1;
    z.y = z.y * f1;
    z.z = z.z * f1;
    z.w = z.w * f1;
    DE = DE * f1;
  } else if (r2 < T(fR2)) {
    const T f2 = T(fR2) / r2;
    z.x = z.x * f2;
    z.y = z.y * f2;
    z.z = z.z * f2;
    z.w = z.w * f2;
    DE = DE * f2;
  }
  z.x = z.x - T(x[GFX_MB_OFFSET]);
  z.y = z.y - T(x[GFX_MB_OFFSET + 1]);
  z.z = z.z - T(x[GFX_MB_OFFSET + 2]);
  if (x[GFX_MAIN_ON] != 0.0 && x[GFX_MAIN_ROT] == 0.0) z = mb_turn<T>(x + GFX_MAIN_ROT + 1, false, z);
  const T sc = T(x[GFX_MB_SCALE]);
  z.x = z.x * sc;
  z.y = z.y * sc;
  z.z = z.z * sc;
  z.w = z.w * sc;
  DE = DE * T(fabs(x[GFX_MB_SCALE])) + T(1.0);
}

// cFractalMandelbulbPupuku::FormulaCode (fractal_mandelbulb_pupuku.cpp:29-144):
// a Mandelbulb with optional pre-folds, acos latitude, sin/cos swap, polar
// scalings and a y fold; dist is aux.dist (set when its own DE block is on)
template <class T>
__device__ __noinline__ void f_mandelbulb_pupuku(V4<T> &z, T r, T &DE, T &dist, const DevSlot &s, int i) {
  const double *x = s.x;
  if (x[PPX_P_ON] != 0.0 && i >= int(x[PPX_START_P]) && i < int(x[PPX_STOP_P])) {  // :34-45
    if (x[PPX_CX] != 0.0) z.x = m_abs(z.x);
    if (x[PPX_CY] != 0.0) z.y = m_abs(z.y);
    if (x[PPX_CZ] != 0.0) z.z = m_abs(z.z);
    z.x = z.x + T(x[PPX_OFFSET_A000]);
    z.y = z.y + T(x[PPX_OFFSET_A000 + 1]);
    z.z = z.z + T(x[PPX_OFFSET_A000 + 2]);
    if (x[PPX_T_ON] != 0.0) r = len4<T, true>(z);
  }
  T t = (x[PPX_SW] == 0.0) ? m_asin(T(z.z / r)) : m_acos(T(z.z / r));
  const T power = T(x[PPX_POWER]);
  const T th = (t + T(x[PPX_BETA])) * power * T(x[PPX_SCALE_A1]);
  T ph = (m_atan2(z.y, z.x) + T(x[PPX_ALPHA])) * power * T(x[PPX_SCALE_B1]);
  T rp = m_pow(r, T(x[PPX_POWER] - x[PPX_OFFSET1]));
  T sth, cth;
  m_sincos(th, &sth, &cth);
  if (x[PPX_X_ON] != 0.0 && i >= int(x[PPX_START_X]) && i < int(x[PPX_STOP_X])) {  // :53-57
    if (cth < T(0.0)) ph = ph + T(3.14159265358979323846);
  }
  DE = rp * DE * m_abs(power) + T(x[PPX_ADE_OFFSET1]);
  rp = rp * r;
  T zth;
  if (x[PPX_D_ON] == 0.0) {
    t = cth;
    zth = sth;
  } else {
    t = sth;
    zth = cth;
  }
  T sph, cph;
  m_sincos(ph, &sph, &cph);
  if (x[PPX_B_ON] != 0.0 && i >= int(x[PPX_START_B]) && i < int(x[PPX_STOP_B]))
    z.x = (T(1.0) + (t - T(1.0)) * T(x[PPX_SCALE_B0])) * cph;
  else
    z.x = t * cph;
  if (x[PPX_A_ON] != 0.0 && i >= int(x[PPX_START_A]) && i < int(x[PPX_STOP_A]))
    z.y = (T(1.0) + (t - T(1.0)) * T(x[PPX_SCALE_A0])) * sph;
  else
    z.y = t * sph;
  z.z = zth;
  z.x = z.x * rp;
  z.y = z.y * rp;
  z.z = z.z * rp;
  z.w = z.w * rp;
  if (x[PPX_BZ] != 0.0) {  // min(z.y, offset0 - z.y)
    const T o = T(x[PPX_OFFSET0]) - z.y;
    if (o < z.y) z.y = o;
  }
  z.x = z.x + T(x[PPX_OFFSET000]);
  z.y = z.y + T(x[PPX_OFFSET000 + 1]);
  z.z = z.z + T(x[PPX_OFFSET000 + 2]);
  if (i >= int(x[PPX_START_S]) && i < int(x[PPX_STOP_S])) {
    const T c1 = T(x[PPX_SCALE_C1]);
    z.x = z.x * c1;
    z.y = z.y * c1;
    z.z = z.z * c1;
    z.w = z.w * c1;
    DE = DE * T(fabs(x[PPX_SCALE_C1]));
  }
  if (x[PPX_ADE_ON] != 0.0) DE = DE * T(x[PPX_ADE_SCALE1]) + T(x[PPX_ADE_OFFSET0]);
  if (x[PPX_C_ON] != 0.0) {  // :120-143
    T de0 = len4<T, true>(z);
    de0 = (de0 > T(1.0)) ? T(T(0.5) * m_log(de0) * de0 / DE) : T(0.0);
    if (x[PPX_E_ON] == 0.0 || !(i >= int(x[PPX_START_E]) && i < int(x[PPX_STOP_E]))) {
      dist = de0;
    } else if (de0 < dist) {
      dist = de0;
    }
  }
}

// cFractalDIFSHextgrid2::FormulaCode (fractal_difs_hextgrid2.cpp:30-138), the
// aux.color terms left out: a hexagonal grid distance into aux.dist (a
// custom-DE formula) after sphere inversion, a tiling fold, a varying scale
// (scaleA = aux.actualScaleA), offset and rotation
template <class T>
__device__ __noinline__ void f_difs_hextgrid2(V4<T> &z, T &DE, AuxX<T> &ax, const DevSlot &s, int i) {
  const double *x = s.x;
  if (x[HGX_SPH_INV] != 0.0 && i >= int(x[HGX_START_X]) && i < int(x[HGX_STOP_1])) {  // :35-45
    z.x = z.x + T(x[HGX_OFFSET000]);
    z.y = z.y + T(x[HGX_OFFSET000 + 1]);
    z.z = z.z + T(x[HGX_OFFSET000 + 2]);
    const T rr = z.x * z.x + z.y * z.y + z.z * z.z + z.w * z.w;
    const T q = T(x[HGX_SCALE_G1]) / rr;
    z.x = z.x * q;
    z.y = z.y * q;
    z.z = z.z * q;
    z.w = z.w * q;
    DE = DE * (T(x[HGX_SCALE_G1]) / rr);
    z.x = z.x + T(x[HGX_ADD000] - x[HGX_OFFSET000]);
    z.y = z.y + T(x[HGX_ADD000 + 1] - x[HGX_OFFSET000 + 1]);
    z.z = z.z + T(x[HGX_ADD000 + 2] - x[HGX_OFFSET000 + 2]);
    const T a1 = T(x[HGX_SCALE_A1]);
    z.x = z.x * a1;
    z.y = z.y * a1;
    z.z = z.z * a1;
    z.w = z.w * a1;
    DE = DE * a1;
  }
  if (x[HGX_C_ON] != 0.0 && i >= int(x[HGX_START_C]) && i < int(x[HGX_STOP_C1])) {  // :46-54
    T tp = T(x[HGX_OFFSET2]);
    z.x = T(fmod(m_abs(z.x) + tp, T(T(2.0) * tp))) - tp;
    tp = T(x[HGX_OFFSETA2]);
    z.y = T(fmod(m_abs(z.y) + tp, T(T(2.0) * tp))) - tp;
  }
  if (i >= int(x[HGX_START_S]) && i < int(x[HGX_STOP_S])) {  // scale :56-71
    const T useScale = ax.scaleA + T(x[HGX_SCALE2]);
    z.x = z.x * useScale;
    z.y = z.y * useScale;
    z.z = z.z * useScale;
    z.w = z.w * useScale;
    DE = DE * m_abs(useScale);
    if (x[HGX_K_ON] != 0.0 && i >= int(x[HGX_START_K]) && i < int(x[HGX_STOP_K])) {
      const T vary = T(x[HGX_SCALE_VARY]) * (m_abs(ax.scaleA) - T(x[HGX_SCALE_C1]));
      ax.scaleA = ax.scaleA - vary;
    }
  }
  z.x = z.x + T(x[HGX_OFFSET001]);  // :73
  z.y = z.y + T(x[HGX_OFFSET001 + 1]);
  z.z = z.z + T(x[HGX_OFFSET001 + 2]);
  if (x[HGX_R_ON] != 0.0 && i >= int(x[HGX_START_R]) && i < int(x[HGX_STOP_R]) && x[HGX_ROT] == 0.0)
    z = mb_turn<T>(x + HGX_ROT + 1, false, z);  // :75-80
  if (i >= int(x[HGX_START]) && i < int(x[HGX_STOP])) {  // the grid :84-105
    const T size = T(x[HGX_SCALE1]), cosPi6 = T(x[HGX_COS6]);
    const T zx = z.x, zy = z.y, zz = z.z / T(x[HGX_SCALE_F1]);
    const T yFloor = m_abs(T(zy - size * T(floor(zy / size + T(0.5)))));
    const T xFloor =
        m_abs(T(zx - size * T(1.5) / cosPi6 * T(floor(zx / size / T(1.5) * cosPi6 + T(0.5)))));
    const T gridMax = smax(yFloor, T(xFloor * cosPi6 + yFloor * T(x[HGX_SIN6])));
    const T gm = gridMax - size * T(0.5);
    const T gridMin = (yFloor < gm) ? yFloor : gm;  // std::min
    T hexD = (x[HGX_J_ON] == 0.0) ? m_sqrt(T(gridMin * gridMin + zz * zz)) : smax(m_abs(gridMin), m_abs(zz));
    hexD = hexD - T(x[HGX_OFFSET0005]);
    const T d = hexD / (DE + T(1.0));
    if (d < ax.dist) ax.dist = d;
  }
}

// cFractalMengerMod1::FormulaCode (fractal_menger_mod1.cpp:29-103), the
// aux.color terms left out
template <class T>
__device__ __noinline__ void f_menger_mod1(V4<T> &z, T &DE, const DevSlot &s, int i) {
  const double *x = s.x;
  z = V4<T>{m_abs(z.x), m_abs(z.y), m_abs(z.z), m_abs(z.w)};
  T t;
  if (z.x < z.y) {
    t = z.y;
    z.y = z.x;
    z.x = t;
  }
  if (z.x < z.z) {
    t = z.z;
    z.z = z.x;
    z.x = t;
  }
  if (z.y < z.z) {
    t = z.z;
    z.z = z.y;
    z.y = t;
  }
  const T s3 = T(x[MMX_SCALE3]);
  z.x = z.x * s3;
  z.y = z.y * s3;
  z.z = z.z * s3;
  z.w = z.w * s3;
  z.x = z.x - T(2.0 * x[MMX_CM111]);
  z.y = z.y - T(2.0 * x[MMX_CM111 + 1]);
  if (z.z > T(1.0)) z.z = z.z - T(2.0 * x[MMX_CM111 + 2]);
  DE = DE * s3;
  if (x[MMX_ROT_ON] != 0.0 && i >= int(x[MMX_START]) && i < int(x[MMX_STOP])) {
    if (x[MMX_ROT] == 0.0) z = mb_turn<T>(x + MMX_ROT + 1, false, z);
    DE = DE * T(x[MMX_SCALED1]) + T(x[MMX_OFFSET1]);
  }
  z.x = z.x + T(x[MMX_ADD000]);
  z.y = z.y + T(x[MMX_ADD000 + 1]);
  z.z = z.z + T(x[MMX_ADD000 + 2]);
  if (x[MMX_BOX_OFF] != 0.0 && i >= int(x[MMX_START_A]) && i < int(x[MMX_STOP_A])) {  // box offset :74-89
    const V4<T> t0 = z;
    z.x = sgn_of(z.x) * T(x[MMX_ADD_A000]) + z.x;
    z.y = sgn_of(z.y) * T(x[MMX_ADD_A000 + 1]) + z.y;
    z.z = sgn_of(z.z) * T(x[MMX_ADD_A000 + 2]) + z.z;
    if (x[MMX_AVG_SCALE] != 0.0) {
      const T tempL = len4<T, true>(t0);
      const T avgScale = len4<T, true>(z) / tempL;
      DE = DE * avgScale + T(1.0);
    }
  }
  if (x[MMX_BLEND] != 0.0) {  // :91-102
    const bool a = i == int(x[MMX_INT_A]), b = i == int(x[MMX_INT_B]);
    const T sc1 = T(x[MMX_SCALE1]), oA = T(x[MMX_OFFSET]), oB = T(x[MMX_OFFSET0]);
    const V4<T> zA = a ? z : V4<T>{T(0.0), T(0.0), T(0.0), T(0.0)};
    const V4<T> zB = b ? z : V4<T>{T(0.0), T(0.0), T(0.0), T(0.0)};
    z.x = z.x * sc1 + zA.x * oA + zB.x * oB;
    z.y = z.y * sc1 + zA.y * oA + zB.y * oB;
    z.z = z.z * sc1 + zA.z * oA + zB.z * oB;
    z.w = z.w * sc1 + zA.w * oA + zB.w * oB;
    DE = DE * sc1;
  }
}

// cFractalKaleidoscopicIfs::FormulaCode (fractal_kaleidoscopic_ifs.cpp:30-85)
// over the enabled vectors of the scene's IFS block; the 4-vector terms with
// w keep the reference's operations (its direction and offset have w = 0)
template <class T>
__device__ __forceinline__ void f_ifs(V4<T> &z, T &DE, const IfsBlock &b) {
  if (b.abs_x) z.x = m_abs(z.x);
  if (b.abs_y) z.y = m_abs(z.y);
  if (b.abs_z) z.z = m_abs(z.z);
  for (int k = 0; k < b.n; k++) {
    if (!b.rot_zero[k]) z = mb_turn<T>(b.rot[k], false, z);
    const T dx = T(b.dir[k][0]), dy = T(b.dir[k][1]), dz = T(b.dir[k][2]);
    const T len = z.x * dx + z.y * dy + z.z * dz + z.w * T(0.0);
    if (len < T(b.dist[k])) {
      const T f = T(2.0) * (len - T(b.dist[k])) * T(b.inten[k]);
      z.x = z.x - dx * f;
      z.y = z.y - dy * f;
      z.z = z.z - dz * f;
      z.w = z.w - T(0.0) * f;
    }
  }
  const T ox = T(b.offset[0]), oy = T(b.offset[1]), oz = T(b.offset[2]);
  if (b.rot_on) {
    V4<T> t{z.x - ox, z.y - oy, z.z - oz, z.w - T(0.0)};
    if (!b.main_zero) t = mb_turn<T>(b.main, false, t);
    z = V4<T>{t.x + ox, t.y + oy, t.z + oz, t.w + T(0.0)};
  }
  if (b.edge_on) {
    if (b.edge[0] > 0.0) z.x = T(b.edge[0]) - m_abs(T(b.edge[0]) - z.x);
    if (b.edge[1] > 0.0) z.y = T(b.edge[1]) - m_abs(T(b.edge[1]) - z.y);
    if (b.edge[2] > 0.0) z.z = T(b.edge[2]) - m_abs(T(b.edge[2]) - z.z);
  }
  const T sc = T(b.scale);
  z.x = z.x * sc;
  z.y = z.y * sc;
  z.z = z.z * sc;
  z.w = z.w * sc;
  if (b.menger) {
    z.x = z.x - ox * (sc - T(1.0));
    z.y = z.y - oy * (sc - T(1.0));
    if (z.z > T(0.5) * oz * (sc - T(1.0))) z.z = z.z - oz * (sc - T(1.0));
  } else {
    z.x = z.x - ox * (sc - T(1.0));
    z.y = z.y - oy * (sc - T(1.0));
    z.z = z.z - oz * (sc - T(1.0));
    z.w = z.w - T(0.0) * (sc - T(1.0));
  }
  DE = DE * m_abs(sc);
}

// EXT: the formulas beyond the three specialised ones and the Mandelbox
// rotations are compiled in; kernels of scenes that use none of them (hybrids
// of the three included) are built without that code.
// i: the iteration (aux.i); c: the orbit's c (aux.const_c), which the Aexion
// replaces at its first iteration.
template <class T, bool W, bool EXT = false>
__device__ __forceinline__ void formula_dispatch(int formula, V4<T> &z, T r, T &DE, const DevSlot &s,
                                                 const MbRot *rot, const IfsBlock *ifs, int i, V4<T> &c,
                                                 AuxX<T> &ax) {
  if constexpr (EXT) {
    switch (formula) {
      case MBR_FORMULA_PSEUDO_KLEINIAN: f_pseudo_kleinian<T>(z, DE, ax.pk, s, i); break;
      case MBR_FORMULA_BOX_FOLD_BULB_POW2_V2: f_box_fold_bulb_pow2_v2<T>(z, DE, ax.scaleA, s, i); break;
      case MBR_FORMULA_ABOX_MOD11: f_abox_mod11<T>(z, DE, ax, c, s, i); break;
      case MBR_FORMULA_PSEUDO_KLEINIAN_MOD4: f_pseudo_kleinian_mod4<T>(z, DE, ax, s, i); break;
      case MBR_FORMULA_PSEUDO_KLEINIAN_STD_DE: f_pseudo_kleinian_std_de<T>(z, DE, ax, s, i); break;
      case MBR_FORMULA_GENERALIZED_FOLD_BOX: f_generalized_fold_box<T>(z, DE, s); break;
      case MBR_FORMULA_MANDELBULB_PUPUKU: f_mandelbulb_pupuku<T>(z, r, DE, ax.dist, s, i); break;
      case MBR_FORMULA_DIFS_HEXTGRID2: f_difs_hextgrid2<T>(z, DE, ax, s, i); break;
      case MBR_FORMULA_BOX_FOLD_BULB_POW2: f_box_fold_bulb_pow2<T>(z, r, DE, s); break;
      case MBR_FORMULA_MENGER_MOD1: f_menger_mod1<T>(z, DE, s, i); break;
      case MBR_FORMULA_QUATERNION: f_quaternion<T>(z, r, DE); break;
      case MBR_FORMULA_AEXION: f_aexion<T>(z, r, DE, s, i, c); break;
      case MBR_FORMULA_MANDELBULB: f_mandelbulb<T>(z, r, DE, s); break;
      case MBR_FORMULA_MANDELBOX: f_mandelbox<T, W, true>(z, DE, s, rot); break;
      case MBR_FORMULA_MANDELBULB_POWER2: f_bulb_pow2<T>(z, r, DE); break;
      case MBR_FORMULA_HYPERCOMPLEX: f_hypercomplex<T>(z, r, DE); break;
      case MBR_FORMULA_KALEIDOSCOPIC_IFS: f_ifs<T>(z, DE, *ifs); break;
      case MBR_FORMULA_XENODREAMBUIE: f_xenodreambuie<T>(z, r, DE, s); break;
      default: f_menger<T, W>(z, DE, s); break;
    }
  } else {
    switch (formula) {
      case MBR_FORMULA_MANDELBULB: f_mandelbulb<T>(z, r, DE, s); break;
      case MBR_FORMULA_MANDELBOX: f_mandelbox<T, W>(z, DE, s); break;
      default: f_menger<T, W>(z, DE, s); break;
    }
  }
}

// SmoothCVector (src/common_math.cpp:133-163)
template <class T, bool W>
__device__ __forceinline__ V4<T> smooth4(const V4<T> &v1, const V4<T> &v2, double k) {
  if (k <= 0.0) return v1;
  if (k >= 1.0) return v2;
  const T kk = T(k), nk = T(1.0 - k);
  const T l1 = len4<T, W>(v1), l2 = len4<T, W>(v2);
  const T lenInterp = l1 * nk + l2 * kk;
  V4<T> t{v1.x * nk + v2.x * kk, v1.y * nk + v2.y * kk, v1.z * nk + v2.z * kk, v1.w * nk + v2.w * kk};
  const T lt = len4<T, W>(t);
  if (lt > T(0.0)) return V4<T>{t.x / lt * lenInterp, t.y / lt * lenInterp, t.z / lt * lenInterp, t.w / lt * lenInterp};
  return v1;
}

template <class T>
__device__ __forceinline__ T cmul_of(const DevScene &sc, int k);
template <>
__device__ __forceinline__ double cmul_of<double>(const DevScene &sc, int k) {
  return sc.cmul[k];
}
template <>
__device__ __forceinline__ float cmul_of<float>(const DevScene &sc, int k) {
  return sc.fcmul[k];
}
template <class T>
__device__ __forceinline__ T juliac_of(const DevScene &sc, int k) {
  return T(sc.julia_c[k] * sc.cmul[k]);
}
// the same for a fractal node of an explicit tree
template <class T>
__device__ __forceinline__ T node_cmul(const DevNode &nd, int k) {
  if constexpr (sizeof(T) == 8) return T(nd.cmul[k]);
  else return T(nd.fcmul[k]);
}
template <class T>
__device__ __forceinline__ T node_juliac(const DevNode &nd, int k) {
  return T(nd.julia_c[k] * nd.cmul[k]);
}


// One component of CVector3::repeatMod (algebra.hpp:106-115): ((p - v/2) % v
// + v) % v - v/2, with % the fmod of a positive period.
template <class T>
__device__ __forceinline__ T repeat_mod(T p, T v) {
  T t = p - v * T(0.5);
  if (v > T(0.0)) t = fmod(t, v);
  t = t + v;
  if (v > T(0.0)) t = fmod(t, v);
  return t - v * T(0.5);
}

// Primitive distances (src/primitive.cpp) at a world point: the node's
// world-to-local transform and repeat (calculate_distance.cpp:268-282), the
// primitive's local distance, times the node's scale (:398-401).
template <class T>
__device__ __noinline__ T prim_distance(const DevPrim &q, T wx, T wy, T wz) {
  T x = T(q.m[0]) * wx + T(q.m[1]) * wy + T(q.m[2]) * wz + T(q.m[3]);
  T y = T(q.m[4]) * wx + T(q.m[5]) * wy + T(q.m[6]) * wz + T(q.m[7]);
  T z = T(q.m[8]) * wx + T(q.m[9]) * wy + T(q.m[10]) * wz + T(q.m[11]);
  if (q.has_repeat) {
    x = repeat_mod(x, T(q.repeat[0]));
    y = repeat_mod(y, T(q.repeat[1]));
    z = repeat_mod(z, T(q.repeat[2]));
  }
  T d;
  bool limits = q.limits != 0;
  switch (q.type) {
    case MBR_PRIMITIVE_PLANE:
      d = z;
      break;
    case MBR_PRIMITIVE_BOX:
      if (q.empty) {
        d = T(-1e10);
        d = smax(T(fabs(x) - T(q.size[0]) * T(0.5)), d);
        d = smax(T(fabs(y) - T(q.size[1]) * T(0.5)), d);
        d = smax(T(fabs(z) - T(q.size[2]) * T(0.5)), d);
        d = fabs(d);
      } else {
        const T bx = smax(T(fabs(x) - T(q.size[0]) * T(0.5)), T(0.0));
        const T by = smax(T(fabs(y) - T(q.size[1]) * T(0.5)), T(0.0));
        const T bz = smax(T(fabs(z) - T(q.size[2]) * T(0.5)), T(0.0));
        d = sqrt(bx * bx + by * by + bz * bz) - T(q.rounding);
      }
      break;
    case MBR_PRIMITIVE_SPHERE:
      d = sqrt(x * x + y * y + z * z) - T(q.radius);
      break;
    case MBR_PRIMITIVE_CYLINDER:
      d = sqrt(x * x + y * y) - T(q.radius);
      if (!q.caps) d = fabs(d);
      d = smax(T(fabs(z) - T(q.height) * T(0.5)), d);
      break;
    case MBR_PRIMITIVE_CIRCLE:
      d = smax(T(fabs(z)), T(sqrt(x * x + y * y) - T(q.radius)));
      break;
    case MBR_PRIMITIVE_RECTANGLE: {
      const T bx = smax(T(fabs(x) - T(q.width) * T(0.5)), T(0.0));
      const T by = smax(T(fabs(y) - T(q.height) * T(0.5)), T(0.0));
      const T bz = fabs(z);
      d = sqrt(bx * bx + by * by + bz * bz);
      break;
    }
    case MBR_PRIMITIVE_TORUS: {
      const T pr = T(q.pow_r), pt = T(q.pow_t);
      const T d1 = pow(pow(x, pr) + pow(y, pr), T(1.0) / pr) - T(q.radius);
      d = pow(pow(d1, pt) + pow(z, pt), T(1.0) / pt) - T(q.tube);
      break;
    }
    case MBR_PRIMITIVE_CONE: {  // primitive.cpp:547-564 (the shifted z also feeds the limits)
      z = z - T(q.height);
      const T r = sqrt(x * x + y * y);
      d = T(q.wn[0]) * r + T(q.wn[1]) * z;
      if (!q.caps) d = fabs(d);
      d = smax(T(-z - T(q.height)), d);
      break;
    }
    case MBR_PRIMITIVE_PRISM: {  // primitive.cpp:657-668
      const T ax = fabs(x), az = fabs(z), tri = T(q.tri);
      d = smax(T(az - T(q.height)), T(smax(T(ax * T(q.pn[1]) + y * T(q.pn[2])), T(-y + tri)) - tri));
      break;
    }
    case MBR_PRIMITIVE_ELLIPSOID: {  // primitive.cpp:670-686: k0 and k1 are floats there
      const T sx = T(q.size[0]), sy = T(q.size[1]), sz = T(q.size[2]);
      const T ux = x / sx, uy = y / sy, uz = z / sz;
      const T vx = x / (sx * sx), vy = y / (sy * sy), vz = z / (sz * sz);
      const float k0 = float(sqrt(ux * ux + uy * uy + uz * uz));
      const float k1 = float(sqrt(vx * vx + vy * vy + vz * vz));
      d = T(double(k0) * (double(k0) - 1.0) / double(k1));
      break;
    }
    default: {  // MBR_PRIMITIVE_WATER: sPrimitiveWater::PrimitiveDistanceWater (primitive.cpp:572-638)
      const T amplitude = T(q.amp), len = T(q.length);
      d = z;
      if (d < amplitude * T(10.0)) {
        const double phase = q.phase;
        const T k = T(0.23);
        T waveX = T(0.0), waveY = T(0.0);
        T p = T(1.0), p2 = T(0.05);
        x = x + T(q.xshift);
        for (int i = 1; i <= q.iterations; i++) {
          const float p3 = float(p * p2);
          const float shift = float(phase / (double(i) / 2.697 + 1.0));
          const T wxt = sin(T(i) + T(0.4) * waveX * T(p3) + sin(k * y / len * T(p3) + T(shift) * T(0.134) * T(p3)) +
                            x / len * T(p3) + T(shift * p3)) /
                        p;
          const T wyt = cos(T(i) + T(0.4) * waveY * T(p3) + sin(x / len * T(p3) + T(shift) * T(0.0179) * T(p3)) +
                            k * y / len * T(p3) + T(shift) * T(0.023) * T(p3)) /
                        p;
          waveX = waveX + wxt;
          waveY = waveY + wyt;
          p2 = p2 + (T(1.0) - p2 + T(0.5) * sin(T(shift) * T(0.0323))) * T(0.7);
          p = p * T(1.872);
        }
        d = d + (waveX + waveY) * amplitude;
      }
      break;
    }
  }
  if (q.type != MBR_PRIMITIVE_CIRCLE && q.type != MBR_PRIMITIVE_RECTANGLE) {
    if (q.empty && q.type != MBR_PRIMITIVE_BOX) d = fabs(d);
    d = smax(T(d - T(q.wall)), T(0.0));
  }
  if (limits) {
    const T lx = smax(T(x - T(q.lmax[0])), T(T(q.lmin[0]) - x));
    const T ly = smax(T(y - T(q.lmax[1])), T(T(q.lmin[1]) - y));
    const T lz = smax(T(z - T(q.lmax[2])), T(T(q.lmin[2]) - z));
    d = smax(d, smax(smax(lx, ly), lz));
  }
  return d * T(q.abs_scale);
}

// The limit box of CalculateDistance (calculate_distance.cpp:261-275): the
// largest of the per-axis distances outside [lim_min, lim_max].
template <class T>
__device__ __forceinline__ T limit_box_distance(const DevScene &sc, T px, T py, T pz) {
  const bool f = sizeof(T) == 4;
  const T bx0 = px - T(f ? sc.flim_max[0] : sc.lim_max[0]), bx1 = -(px - T(f ? sc.flim_min[0] : sc.lim_min[0]));
  const T by0 = py - T(f ? sc.flim_max[1] : sc.lim_max[1]), by1 = -(py - T(f ? sc.flim_min[1] : sc.lim_min[1]));
  const T bz0 = pz - T(f ? sc.flim_max[2] : sc.lim_max[2]), bz1 = -(pz - T(f ? sc.flim_min[2] : sc.lim_min[2]));
  const T bx = (bx0 < bx1) ? bx1 : bx0, by = (by0 < by1) ? by1 : by0, bz = (bz0 < bz1) ? bz1 : bz0;
  T m = bx;
  if (m < by) m = by;
  if (m < bz) m = bz;
  return m;
}

// The global folds before a formula iteration (compute_fractal.cpp:190-202):
// BoxFolding and SphericalFolding (legacy_fractal_transforrms.cpp:43-103),
// each followed by r = |z|.
template <class T, bool W>
__device__ __forceinline__ void global_folds(const DevScene &sc, V4<T> &z, T &r, T &DE) {
  const bool f = sizeof(T) == 4;
  if (sc.gbox) {
    const T lim = T(f ? sc.fgbox_limit : sc.gbox_limit), val = T(f ? sc.fgbox_value : sc.gbox_value);
    if (z.x > lim) z.x = val - z.x;
    else if (z.x < -lim) z.x = -val - z.x;
    if (z.y > lim) z.y = val - z.y;
    else if (z.y < -lim) z.y = -val - z.y;
    if (z.z > lim) z.z = val - z.z;
    else if (z.z < -lim) z.z = -val - z.z;
    r = len4<T, W>(z);
  }
  if (sc.gsph) {
    const T fR2 = T(f ? sc.fgsph_fr2 : sc.gsph_fr2), mR2 = T(f ? sc.fgsph_mr2 : sc.gsph_mr2);
    const T r2 = r * r;
    const T f1 = fR2 / mR2;
    if (r2 < mR2) {
      z.x = z.x * f1;
      z.y = z.y * f1;
      z.z = z.z * f1;
      if (W) z.w = z.w * f1;
      DE = DE * f1;
    } else if (r2 < fR2) {
      const T f2 = fR2 / r2;
      z.x = z.x * f2;
      z.y = z.y * f2;
      z.z = z.z * f2;
      if (W) z.w = z.w * f2;
      DE = DE * f2;
    }
    r = len4<T, W>(z);
  }
}

// The orbit of Compute<calcModeNormal> and Compute<calcModeDeltaDE1>
// (compute_fractal.cpp:170-492; the two modes iterate alike) from the point
// (px, py, pz), at most maxN iterations.  Returns the loop index at exit (the
// orbit's iteration count is one more) and leaves the final z, r = |z| (4-D),
// the derivative DE and the orbit's maxiter flag.
template <class T, int F, bool W, bool TREE = false>
__device__ __forceinline__ int compute_orbit(const DevScene &sc, T px, T py, T pz, int maxN, V4<T> &z, T &r, T &DE,
                                             bool &maxiter, const DevNode *nd = nullptr, T *pk_out = nullptr,
                                             T *dist_out = nullptr) {
  z = V4<T>{px, py, pz, W ? T(TREE ? nd->w0 : sc.w0) : T(0.0)};
  V4<T> c = z;  // aux.const_c
  r = len4<T, W>(z);
  DE = T(1.0);
  AuxX<T> ax{T(1.0), T(0.0), T(0.0), T(1.0), T(1000.0), z};
  if (F == F_EXT)  // aux.actualScale: the Mandelbox scale of the sequence's first slot (compute_fractal.cpp:97-98, 123)
    ax.scale = T(sc.slot[TREE ? nd->slot : int(sc.seq[0])].d[P_MB_SCALE]);
  V4<T> lastZ{T(0.0), T(0.0), T(0.0), T(0.0)}, lastLastZ = lastZ;
  maxiter = true;
  int i;
  for (i = 0; i < maxN; i++) {
    lastLastZ = lastZ;
    lastZ = z;
    const int k = TREE ? nd->slot : ((F > 0) ? 0 : ((i < sc.length) ? int(sc.seq[i]) : int(sc.seq[0])));
    const DevSlot &s = sc.slot[k];
    if (F == F_EXT) global_folds<T, W>(sc, z, r, DE);
    const V4<T> tempZ = z;
    const T tempDE = DE;
    if (F > 0) {
      if (F == MBR_FORMULA_MANDELBULB) f_mandelbulb<T>(z, r, DE, s);
      if (F == MBR_FORMULA_MANDELBOX) f_mandelbox<T, W>(z, DE, s);
      if (F == MBR_FORMULA_MENGER_SPONGE) f_menger<T, W>(z, DE, s);
    } else if (s.d[P_WEIGHT] > 0.0) {
      formula_dispatch<T, W, F == F_EXT>(s.formula, z, r, DE, s, &sc.mbrot, &sc.ifs, i, c, ax);
    }
    if (s.add_c) {
      if (TREE ? nd->julia : sc.julia) {
        z.x = z.x + (TREE ? node_juliac<T>(*nd, 0) : juliac_of<T>(sc, 0));
        z.y = z.y + (TREE ? node_juliac<T>(*nd, 1) : juliac_of<T>(sc, 1));
        z.z = z.z + (TREE ? node_juliac<T>(*nd, 2) : juliac_of<T>(sc, 2));
      } else {
        z.x = z.x + c.x * (TREE ? node_cmul<T>(*nd, 0) : cmul_of<T>(sc, 0));
        z.y = z.y + c.y * (TREE ? node_cmul<T>(*nd, 1) : cmul_of<T>(sc, 1));
        z.z = z.z + c.z * (TREE ? node_cmul<T>(*nd, 2) : cmul_of<T>(sc, 2));
        if (W) z.w = z.w + c.w;
      }
    }
    if (!TREE && F <= 0 && sc.is_hybrid) {
      const double kw = s.d[P_WEIGHT];
      if (kw < 1.0) {
        z = smooth4<T, W>(tempZ, z, kw);
        DE = DE * T(kw) + tempDE * T(1.0 - kw);
      }
    }
    r = len4<T, W>(z);
    if (nan4<T, W>(z)) {
      z = lastZ;
      r = len4<T, W>(z);
      maxiter = true;
      break;
    }
    if (s.check_bailout && r > P<T>(s, P_BAILOUT)) {
      maxiter = false;
      break;
    }
    // the convergence bailout of pseudo- and Jos-Kleinian formulas
    // (compute_fractal.cpp:323-336; hybrid_fractal_sequences.cpp:242-246)
    if (F == F_EXT && s.check_bailout && s.add_bail) {
      maxiter = false;
      const T lim = T(0.1 / s.d[P_BAILOUT]);
      if (len4<T, W>(V4<T>{z.x - lastZ.x, z.y - lastZ.y, z.z - lastZ.z, z.w - lastZ.w}) / r < lim) break;
      if (len4<T, W>(V4<T>{z.x - lastLastZ.x, z.y - lastLastZ.y, z.z - lastLastZ.z, z.w - lastLastZ.w}) / r < lim)
        break;
    }
  }
  if (pk_out) *pk_out = ax.pk;
  if (dist_out) *dist_out = ax.dist;
  return i;
}

// The final distance of an analytic orbit (compute_fractal.cpp:495-621).
// The specialised iterations carry linear, logarithmic and IFS; the extended
// one every DevDeFinal code.
template <class T, int F, bool W>
__device__ __forceinline__ T final_distance(const DevScene &sc, const V4<T> &z, T r, T DE, int de_final = -1,
                                            T pk = T(1.0), T dist = T(1000.0)) {
  if (!(DE > T(0.0))) return r;
  if (F == F_EXT) {
    switch (de_final >= 0 ? de_final : sc.de_final) {
      case DEF_LINEAR_OFFSET: return (r - (sizeof(T) == 8 ? T(sc.linear_de_offset) : T(sc.flinear_de_offset))) / DE;
      case DEF_LOG: return (r > T(1.0)) ? T(T(0.5) * r * m_log(r) / DE) : T(0.0);
      case DEF_LINEAR: return r / DE;
      case DEF_IFS: return (r - T(2.0)) / DE;
      case DEF_PSEUDO_KLEINIAN: {  // pk: aux.pseudoKleinianDE, 1 unless a pseudo-Kleinian formula set it
        const T rxy = m_sqrt(z.x * z.x + z.y * z.y);
        return smax(T(rxy - pk), T(m_abs(rxy * z.z) / r)) / DE;
      }
      case DEF_CUSTOM: return dist;  // aux.dist: 1000 unless a formula set it (:119)
      case DEF_MAX_AXIS: {
        const T rd = smax(m_abs(z.x), smax(m_abs(z.y), m_abs(z.z)));
        return rd / DE;
      }
      case DEF_NONE: return T(-1.0);
      default: return r;
    }
  }
  // 1 linear r/DE, 2 log, 3 IFS, 4 hybrid linear with offset
  const int fn = (F <= 0 && sc.is_hybrid) ? ((sc.de_function == 1) ? 4 : 2) : sc.de_analytic;
  if (fn == 4) return (r - (sizeof(T) == 8 ? T(sc.linear_de_offset) : T(sc.flinear_de_offset))) / DE;
  if (fn == 2) return (r > T(1.0)) ? T(T(0.5) * r * m_log(r) / DE) : T(0.0);
  if (fn == 1) return r / DE;
  if (fn == 3) return (r - T(2.0)) / DE;
  return r;
}

// CalculateDistanceSimple, delta-DE branch (calculate_distance.cpp:607-760):
// the orbit radius at the point and at three points offset by deltaDE along
// x, y and z, each capped at the first orbit's iteration count; the distance
// divides the radius by the gradient of |z| through the sequence's DE
// function.  FP64 only: the offsets are 1e-5 of the detail size.
template <class T, bool W, bool TREE = false>
__device__ __noinline__ T delta_distance(const DevScene &sc, T px, T py, T pz, T detail, bool normal_mode,
                                         int *iters_out, int *total_out, const DevNode *nd = nullptr) {
  const int maxN = TREE ? nd->maxN : sc.formula_maxiter;
  const int delta_fn = TREE ? nd->delta_fn : sc.delta_fn;
  const int mult = (normal_mode && sc.iter_thresh) ? 5 : 1;
  const T plen = m_sqrt(px * px + py * py + pz * pz);  // fractIn.point.Length()
  const T deltaDE = smax(T(plen * T(1e-14)), T(T(sc.delta_factor) * detail));
  V4<T> z;
  T r4, DE;
  bool mx;
  // Compute's delta-mode ending for the Jos Kleinian function
  // (compute_fractal.cpp:627-638): z.y = min(z.y, foldingValue - z.y) with
  // the default transf_spheres_enabled (true) and transf_folding_value (2)
  const bool jos = delta_fn == 4;
  const int i1 = compute_orbit<T, F_EXT, W, TREE>(sc, px, py, pz, maxN * mult, z, r4, DE, mx, nd);
  if (jos && T(2.0) - z.y < z.y) z.y = T(2.0) - z.y;
  const T r = m_sqrt(z.x * z.x + z.y * z.y + z.z * z.z);  // fractOut.z.Length(): the 3-D part
  const T zfx = z.x, zfy = z.y, zfz = z.z;
  const int iters1 = i1 + 1;
  int total = iters1;
  bool out_maxiter = mx;
  bool maxiter = mx;
  if (!sc.limits) {
    if (!sc.iter_thresh) maxiter = false;
  } else {
    if (normal_mode) maxiter = false;
  }
  T drv[3];
  int last_iters = iters1;
  for (int a = 0; a < 3; a++) {  // x, y, z offsets, each with forcedMaxiter = the first orbit's count
    const int i = compute_orbit<T, F_EXT, W, TREE>(sc, a == 0 ? T(px + deltaDE) : T(px + T(0.0)),
                                                   a == 1 ? T(py + deltaDE) : T(py + T(0.0)),
                                                   a == 2 ? T(pz + deltaDE) : T(pz + T(0.0)), iters1, z, r4, DE, mx,
                                                   nd);
    if (jos && T(2.0) - z.y < z.y) z.y = T(2.0) - z.y;
    const T r2 = m_sqrt(z.x * z.x + z.y * z.y + z.z * z.z);
    drv[a] = m_abs(T(r2 - r)) / deltaDE;
    last_iters = i + 1;
    total += last_iters;
  }
  const T dr = m_sqrt(drv[0] * drv[0] + drv[1] * drv[1] + drv[2] * drv[2]);
  T distance = T(0.0);
  if (dr > T(0.0)) {
    switch (delta_fn) {
      case 1: distance = T(0.5) * r / dr; break;
      case 2: distance = T(0.5) * r * m_log(r) / dr; break;
      case 3: {  // the last offset orbit's z (:686-690)
        const T rxy = m_sqrt(z.x * z.x + z.y * z.y);
        distance = smax(T(rxy - T(0.92784)), T(m_abs(rxy * z.z) / r)) / dr;
        break;
      }
      case 4: {
        const T rxy = m_sqrt(z.x * z.x + z.z * z.z);
        distance = (m_abs(rxy * z.y) / r) / dr;
        maxiter = false;
        break;
      }
      case 5: distance = r; break;
      case 6: {  // the first orbit's z; dMax (common_math.cpp:74-83)
        const T ax = m_abs(zfx), ay = m_abs(zfy), az = m_abs(zfz);
        const T d0 = m_abs(drv[0]), d1 = m_abs(drv[1]), d2 = m_abs(drv[2]);
        const T maxZ = (ax > ay) ? ((ax > az) ? ax : az) : ((ay > az) ? ay : az);
        const T maxDr = (d0 > d1) ? ((d0 > d2) ? d0 : d2) : ((d1 > d2) ? d1 : d2);
        distance = T(0.5) * maxZ / maxDr;
        break;
      }
      default: break;
    }
  } else {
    distance = r;
  }
  if (!sc.iter_thresh) out_maxiter = false;
  if (normal_mode) out_maxiter = false;
  if (out_maxiter) distance = T(0.0);
  if (last_iters < sc.min_n && distance < detail) distance = detail;  // fractOut of the last offset orbit
  if (sc.interior) {
    if (!normal_mode) {
      if (distance < T(0.5) * detail || maxiter) distance = detail;
    } else {
      if (distance < T(0.9) * detail) distance = detail - distance;
    }
  }
  if (sc.iter_thresh && !normal_mode && !maxiter) {
    if (distance < detail) distance = detail * T(1.01);
  }
  if (distance < T(0.0)) distance = T(0.0);
  if (distance > T(10.0)) distance = T(10.0);
  *iters_out = iters1;
  if (total_out) *total_out = total;
  return distance;
}

// CalculateDistanceSimple (calculate_distance.cpp:533-760): the delta
// branch (FP64) or the analytic branch, with its post-processing.  TREE: for
// the fractal node nd of an explicit tree (its slot, iteration limit, julia
// and constant factor, DE function).
template <class T, int F, bool W, bool TREE = false>
__device__ __forceinline__ T calc_distance_simple(const DevScene &sc, T px, T py, T pz, T detail, bool normal_mode,
                                                  int *iters_out, int *total_out, const DevNode *nd = nullptr) {
  if constexpr (F == F_EXT && sizeof(T) == 8) {
    if (TREE ? nd->delta_de : sc.delta_de)
      return delta_distance<T, W, TREE>(sc, px, py, pz, detail, normal_mode, iters_out, total_out, nd);
  }
  const int mult = (normal_mode && sc.iter_thresh) ? 5 : 1;
  V4<T> z;
  T r, DE, pk, cdist;
  bool maxiter;
  const int i = compute_orbit<T, F, W, TREE>(sc, px, py, pz, (TREE ? nd->maxN : sc.formula_maxiter) * mult, z, r,
                                             DE, maxiter, nd, &pk, &cdist);
  T distance = final_distance<T, F, W>(sc, z, r, DE, TREE ? nd->de_final : -1, pk, cdist);
  const int iters = i + 1;
  *iters_out = iters;
  if (total_out) *total_out = iters;
  // CalculateDistanceSimple post-processing (calculate_distance.cpp:561-605)
  bool mx = maxiter;
  if (!sc.iter_thresh) mx = false;
  if (normal_mode) mx = false;
  if (mx) distance = T(0.0);
  if (iters < sc.min_n && distance < detail) distance = detail;
  if (sc.interior) {
    if (!normal_mode) {
      if (distance < T(0.5) * detail || maxiter) distance = detail;
    } else {
      if (distance < T(0.9) * detail) distance = detail - distance;
    }
  }
  if (sc.iter_thresh && !normal_mode && !maxiter) {
    if (distance < detail) distance = detail * T(1.01);
  }
  if (distance < T(0.0)) distance = T(0.0);
  if (distance > T(10.0)) distance = T(10.0);
  return distance;
}

// mergeChildIntoParent (calculate_distance.cpp:103-204) on the distance and
// the smooth-combine settings: intersection takes the larger distance,
// subtraction pushes the first operand's surface 1.5 detail sizes out where a
// later operand is within one detail size, union takes the smaller or, for a
// child that asks for it, the smooth union (opSmoothUnion, math_utilities.h:99-103).
template <class T>
struct TreeFrame {
  T dist, detail, smooth_dist;
  int type;
  bool smooth;
};
template <class T>
__device__ __forceinline__ void tree_merge(T cd, bool csmooth, T csdist, TreeFrame<T> &p) {
  if (p.type == MBR_NODE_BOOLEAN_MUL) {
    if (cd > p.dist) p.dist = cd;
  } else if (p.type == MBR_NODE_BOOLEAN_SUB) {
    if (p.dist >= T(1e19)) {
      p.dist = cd;
    } else if (p.detail > T(0.0) && cd < p.detail) {
      const T limitDist = p.detail * T(1.5);
      if (cd < limitDist) {
        p.dist = limitDist;
      } else {
        const T adjusted = smax(T(limitDist - cd), p.dist);
        p.dist = (adjusted < T(0.0)) ? T(0.0) : adjusted;
      }
    }
  } else {
    if (csmooth && p.dist < T(1e19)) {
      const T k = csdist, d1 = cd, d2 = p.dist;
      const T t = T(0.5) + T(0.5) * (d2 - d1) / k;
      const T h = (t < T(0.0)) ? T(0.0) : ((t > T(1.0)) ? T(1.0) : t);
      p.dist = (d2 * (T(1.0) - h) + d1 * h) - k * h * (T(1.0) - h);
    } else if (cd < p.dist) {
      p.dist = cd;
    }
  }
}

// CalculateDistanceFromObjectsTree (calculate_distance.cpp:225-516) over the
// scene's explicit tree: each node's world-to-local transform, repeat in its
// own frame, detail size / (absScale * detail multiplier); boolean groups on
// a stack of at most 9 levels; the leaves' iterations summed.
template <class T, bool W>
__device__ __noinline__ T tree_distance(const DevScene &sc, T px, T py, T pz, T detail, bool normal_mode,
                                        int *iters_out, int *total_out) {
  TreeFrame<T> st[10];
  st[0] = TreeFrame<T>{T(1e20), detail, T(0.1), MBR_NODE_BOOLEAN_ADD, false};
  int sl = 0, total_iters = 0, total_all = 0;
  for (int n = 0; n < sc.n_nodes; n++) {
    const DevNode &nd = sc.node[n];
    const double *m = nd.w2l;
    T lx = T(m[0]) * px + T(m[1]) * py + T(m[2]) * pz + T(m[3]);
    T ly = T(m[4]) * px + T(m[5]) * py + T(m[6]) * pz + T(m[7]);
    T lz = T(m[8]) * px + T(m[9]) * py + T(m[10]) * pz + T(m[11]);
    if (nd.has_repeat) {
      lx = repeat_mod(lx, T(nd.repeat[0]));
      ly = repeat_mod(ly, T(nd.repeat[1]));
      lz = repeat_mod(lz, T(nd.repeat[2]));
    }
    T nodeDetail;
    if (nd.abs_scale > 0.0 && nd.detail_mult > 0.0) nodeDetail = detail / T(nd.abs_scale) / T(nd.detail_mult);
    else if (nd.abs_scale > 0.0) nodeDetail = detail / T(nd.abs_scale);
    else if (nd.detail_mult > 0.0) nodeDetail = detail / T(nd.detail_mult);
    else nodeDetail = detail;
    while (sl > nd.level) {
      const TreeFrame<T> child = st[sl];
      sl--;
      tree_merge<T>(child.dist, child.smooth, child.smooth_dist, st[sl]);
    }
    T distance;
    int leaf_iters = 0, leaf_total = 0;
    if (nd.type == MBR_NODE_FRACTAL) {
      distance = calc_distance_simple<T, F_EXT, W, true>(sc, lx, ly, lz, nodeDetail, normal_mode, &leaf_iters,
                                                         &leaf_total, &nd);
      distance = distance * T(nd.abs_scale);
    } else if (nd.type == MBR_NODE_PRIMITIVE) {
      distance = prim_distance<T>(sc.prim[nd.prim], px, py, pz);
    } else {
      sl++;
      st[sl] = TreeFrame<T>{nd.type == MBR_NODE_BOOLEAN_MUL ? T(-1e20) : T(1e20), nodeDetail, T(nd.smooth_dist),
                            nd.type, nd.smooth != 0};
      continue;
    }
    tree_merge<T>(distance, nd.smooth != 0, T(nd.smooth_dist), st[sl]);
    total_iters += leaf_iters;
    total_all += leaf_total;
  }
  while (sl > 0) {
    const TreeFrame<T> child = st[sl];
    sl--;
    tree_merge<T>(child.dist, child.smooth, child.smooth_dist, st[sl]);
  }
  *iters_out = total_iters;
  if (total_out) *total_out = total_all;
  return st[0].dist;
}

// CalculateDistance for one point: the limit box, then the objects tree -
// the scene's explicit tree (F_EXT), or the default one: CalculateDistanceSimple
// of the fractal or hybrid node and the union with the primitives.
// F: fixed formula id (non-hybrid scene), 0 (generic: the sequence table over
// the three specialised formulas) or F_EXT (generic with every formula and
// the Mandelbox rotations).  W: 4-D state.  *iters_out: the iteration count
// of the (first) orbit; *total_out, when given: the iterations of all orbits.
template <class T, int F, bool W>
__device__ __forceinline__ T calc_distance(const DevScene &sc, T px, T py, T pz, T detail, bool normal_mode,
                                           int *iters_out, int *total_out = nullptr) {
  if (F == F_EXT && sc.limits) {  // outside the limit box: its distance, no iteration
    const T lbd = limit_box_distance<T>(sc, px, py, pz);
    if (lbd > detail) {
      *iters_out = 0;
      if (total_out) *total_out = 0;
      return lbd;
    }
  }
  if constexpr (F == F_EXT) {
    if (sc.n_nodes > 0) return tree_distance<T, W>(sc, px, py, pz, detail, normal_mode, iters_out, total_out);
  }
  T distance = calc_distance_simple<T, F, W>(sc, px, py, pz, detail, normal_mode, iters_out, total_out);
  if (F == F_EXT) {  // the union with the primitives (booleanAdd, calculate_distance.cpp:166-201)
    for (int k = 0; k < sc.n_prims; k++) {
      const T pd = prim_distance<T>(sc.prim[k], px, py, pz);
      if (pd < distance) distance = pd;
    }
  }
  return distance;
}

}  // namespace mbr
