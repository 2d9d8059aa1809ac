// fast_formula.cuh - one formula iteration in FP32, written for the issue
// slots of the B200 SM: the FMA pipe takes a warp instruction every cycle,
// the ALU pipe every second cycle and the XU (MUFU) pipe every eighth, so
// clamps and compares are expressed as saturating FMAs where possible.
// Used by the wavefront kernels, whose lanes advance their distance
// estimates a few iterations at a time.
//
// Rewrites of the reference formulas (equal in real arithmetic; in FP32 they
// differ from a literal transcription by a few units in the last place):
//  * Mandelbox box fold (fractal_mandelbox.cpp:91-105): when folding_value ==
//    2*folding_limit (the reference default, 1 and 2), sign(z)*value - z for
//    |z| > limit and z otherwise equals 2*clamp(z, -L, L) - z
//    = 4L*sat(z/(2L) + 1/2) - 2L - z, with sat() the free [0,1] saturation.
//  * Mandelbox sphere fold (:109-126): the factor (fR2/mR2 if r2 < mR2,
//    fR2/r2 if r2 < fR2, else 1) equals clamp(fR2/r2, 1, fR2/mR2) whenever
//    mR2 <= fR2, i.e. 1 + (F-1)*sat((fR2/r2 - 1)/(F-1)) with F = fR2/mR2; the
//    scale and the c-addition fold into one FMA per axis.
//  * Menger sponge sort (fractal_menger_sponge.cpp:34-56): the three
//    conditional swaps are a sorting network, written with min/max.
//  * bailout |z| > b is tested as |z|^2 > b^2; |z| is taken once, for the DE.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

#include "mbr_device.h"

namespace mbr {

// FP32 parameters of a non-hybrid formula, as a lane holds them.
struct FastParams {
  int formula;     // MBR_FORMULA_*
  int maxN;        // formula_maxiter
  int de_fn;       // 1 linear, 2 log, 3 IFS
  int box_simple;  // mandelbox: folding_value == 2*limit, mR2 < fR2, no offset
  int add_c;       // slot adds the c constant
  int julia;       // c is the Julia constant instead of the point
  int min_n;       // minN
  int bulb_n;      // mandelbulb: the power when it is an integer 2..32 and both angle offsets are 0, else 0
  float bailout2;
  float cm_x, cm_y, cm_z;        // fractal_constant_factor
  float jc_x, jc_y, jc_z;        // julia_c * fractal_constant_factor
  float p0, p1, p2, p3, p4, p5;  // formula specific (see load_fast_params)
  float q0, q1, q2, q3, q4;      // derived constants of the simple Mandelbox path
  float off_x, off_y, off_z;     // mandelbox offset (0 when absent)
  // mandelbox rotations (MbRot in FP32; the simple path is off when any is on)
  int rot_folds;                 // box fold in rotated frames
  int rot_main;                  // main rotation (enabled and not the identity)
  int rot_zero[2][3];            // rot[fold][axis] is the identity
  float rot_m[2][3][9];          // rot[fold][axis], row-major; rotinv is the transpose
  float rot_mm[9];               // main rotation
};

// mandelbulb: p0 power, p1 power-1, p2 alpha, p3 beta
// mandelbox:  p0 scale, p1 |scale|, p2 limit, p3 value, p4 fR2, p5 factor1 (fR2/mR2)
//             simple path: q0 = 1/(2L), q1 = 4L, q2 = fR2/(F-1), q3 = F-1, q4 = -1/(F-1)
// menger:     p0 scale3
__host__ __device__ inline FastParams load_fast_params(const DevScene &sc) {
  FastParams f;
  const DevSlot &s = sc.slot[0];
  f.formula = s.formula;
  f.maxN = sc.formula_maxiter;
  f.de_fn = sc.de_analytic;
  f.bailout2 = s.f[P_BAILOUT] * s.f[P_BAILOUT];
  f.add_c = s.add_c;
  f.julia = sc.julia;
  f.min_n = sc.min_n;
  f.cm_x = sc.fcmul[0];
  f.cm_y = sc.fcmul[1];
  f.cm_z = sc.fcmul[2];
  f.jc_x = sc.fjulia_c[0];
  f.jc_y = sc.fjulia_c[1];
  f.jc_z = sc.fjulia_c[2];
  f.off_x = f.off_y = f.off_z = 0.0f;
  f.box_simple = 0;
  f.bulb_n = 0;
  f.rot_folds = sc.mbrot.folds;
  f.rot_main = (sc.mbrot.main && !sc.mbrot.main_zero) ? 1 : 0;
  for (int a = 0; a < 2; a++)
    for (int b = 0; b < 3; b++) {
      f.rot_zero[a][b] = sc.mbrot.zero[a][b];
      for (int k = 0; k < 9; k++) f.rot_m[a][b][k] = float(sc.mbrot.m[a][b][k]);
    }
  for (int k = 0; k < 9; k++) f.rot_mm[k] = float(sc.mbrot.mm[k]);
  f.p0 = f.p1 = f.p2 = f.p3 = f.p4 = f.p5 = 0.0f;
  f.q0 = f.q1 = f.q2 = f.q3 = f.q4 = 0.0f;
  if (s.formula == MBR_FORMULA_MANDELBULB) {
    f.p0 = s.f[P_POWER];
    f.p1 = s.f[P_POWER_M1];
    f.p2 = s.f[P_ALPHA];
    f.p3 = s.f[P_BETA];
    const double pw = s.d[P_POWER];
    if (s.d[P_ALPHA] == 0.0 && s.d[P_BETA] == 0.0 && pw >= 2.0 && pw <= 32.0 && pw == double(int(pw)))
      f.bulb_n = int(pw);
  } else if (s.formula == MBR_FORMULA_MANDELBOX) {
    f.p0 = s.f[P_MB_SCALE];
    f.p1 = s.f[P_MB_ABS_SCALE];
    f.p2 = s.f[P_MB_LIMIT];
    f.p3 = s.f[P_MB_VALUE];
    f.p4 = s.f[P_MB_FR2];
    f.p5 = s.f[P_MB_FACTOR1];
    const double L = s.d[P_MB_LIMIT], F = s.d[P_MB_FACTOR1];
    f.box_simple = (s.d[P_MB_VALUE] == 2.0 * L && L > 0.0 && F > 1.0 && !s.has_offset && !sc.mbrot.folds &&
                    !sc.mbrot.main) ? 1 : 0;
    if (f.box_simple) {
      f.q0 = float(1.0 / (2.0 * L));
      f.q1 = float(4.0 * L);
      f.q2 = float(s.d[P_MB_FR2] / (F - 1.0));
      f.q3 = float(F - 1.0);
      f.q4 = float(-1.0 / (F - 1.0));
    }
    if (s.has_offset) {
      f.off_x = s.f[P_MB_OFF_X];
      f.off_y = s.f[P_MB_OFF_Y];
      f.off_z = s.f[P_MB_OFF_Z];
    }
  } else {
    f.p0 = s.f[P_SCALE3];
  }
  return f;
}

struct Z3 {
  float x, y, z;
};

// a*b + c clamped to [0, 1] in one FFMA.SAT (a separate saturate of an fmaf
// result costs the ALU pipe another instruction)
__device__ __forceinline__ float fma_sat(float a, float b, float c) {
  float y;
  asm("fma.rn.sat.f32 %0, %1, %2, %3;" : "=f"(y) : "f"(a), "f"(b), "f"(c));
  return y;
}

// Blackwell's paired FP32 arithmetic (PTX fma.rn.f32x2): two lanes of an
// FMA in one instruction on a 64-bit register pair
__device__ __forceinline__ unsigned long long pack2(float lo, float hi) {
  unsigned long long v;
  asm("mov.b64 %0, {%1, %2};" : "=l"(v) : "f"(lo), "f"(hi));
  return v;
}
__device__ __forceinline__ void unpack2(unsigned long long v, float &lo, float &hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ unsigned long long ffma2(unsigned long long a, unsigned long long b, unsigned long long c) {
  unsigned long long d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}

// 1/x from the MUFU unit (max. 1 ulp; 0 -> +inf, flushes denormals)
__device__ __forceinline__ float rcp_approx(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// sqrt(x) from the MUFU unit (max. 2 ulp; flushes denormals)
__device__ __forceinline__ float sqrt_approx(float x) {
  float y;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// z turned by the row-major matrix m, or by its transpose
__device__ __forceinline__ Z3 turn3(const float *m, bool transpose, const Z3 &v) {
  if (!transpose)
    return Z3{fmaf(m[0], v.x, fmaf(m[1], v.y, m[2] * v.z)), fmaf(m[3], v.x, fmaf(m[4], v.y, m[5] * v.z)),
              fmaf(m[6], v.x, fmaf(m[7], v.y, m[8] * v.z))};
  return Z3{fmaf(m[0], v.x, fmaf(m[3], v.y, m[6] * v.z)), fmaf(m[1], v.x, fmaf(m[4], v.y, m[7] * v.z)),
            fmaf(m[2], v.x, fmaf(m[5], v.y, m[8] * v.z))};
}
__device__ __forceinline__ float &z3_axis(Z3 &v, int dim) { return dim == 0 ? v.x : (dim == 1 ? v.y : v.z); }

// One Mandelbox iteration + c-addition.  c holds the (pre-multiplied) constant.
template <bool SIMPLE>
__device__ __forceinline__ void it_mandelbox(Z3 &z, float &dr, const Z3 &c, const FastParams &f) {
  if (SIMPLE) {
    const float L2 = 0.5f * f.q1;  // 2L
    // x and y of the box fold in one f32x2 register pair: w = -z - 2L, then
    // 4L * sat(...) + w - two paired FMAs where the scalar form issues four
    const unsigned long long w = ffma2(pack2(z.x, z.y), pack2(-1.0f, -1.0f), pack2(-L2, -L2));
    unpack2(ffma2(pack2(f.q1, f.q1), pack2(fma_sat(z.x, f.q0, 0.5f), fma_sat(z.y, f.q0, 0.5f)), w), z.x, z.y);
    z.z = fmaf(f.q1, fma_sat(z.z, f.q0, 0.5f), -z.z) - L2;
    const float r2 = fmaf(z.x, z.x, fmaf(z.y, z.y, z.z * z.z));
    // factor = 1 + (F-1) * sat((fR2/r2 - 1) / (F-1)); r2 = 0 gives +inf -> factor F
    const float fs = fmaf(f.q3, fma_sat(f.q2, rcp_approx(r2), f.q4), 1.0f);
    const float s = fs * f.p0;
    dr = fmaf(dr, fs * f.p1, 1.0f);
    z.x = fmaf(z.x, s, c.x);
    z.y = fmaf(z.y, s, c.y);
    z.z = fmaf(z.z, s, c.z);
  } else {
    const float L = f.p2, V = f.p3;
    if (f.rot_folds) {  // fractal_mandelbox.cpp:33-63
      for (int dim = 0; dim < 3; dim++) {
        Z3 zr = f.rot_zero[0][dim] ? z : turn3(f.rot_m[0][dim], false, z);
        if (z3_axis(zr, dim) > L) {
          z3_axis(zr, dim) = V - z3_axis(zr, dim);
          z = turn3(f.rot_m[0][dim], true, zr);
        } else {
          zr = f.rot_zero[1][dim] ? z : turn3(f.rot_m[1][dim], false, z);
          if (z3_axis(zr, dim) < -L) {
            z3_axis(zr, dim) = -V - z3_axis(zr, dim);
            z = turn3(f.rot_m[1][dim], true, zr);
          }
        }
      }
    } else {
      if (fabsf(z.x) > L) z.x = copysignf(V, z.x) - z.x;
      if (fabsf(z.y) > L) z.y = copysignf(V, z.y) - z.y;
      if (fabsf(z.z) > L) z.z = copysignf(V, z.z) - z.z;
    }
    const float r2 = fmaf(z.x, z.x, fmaf(z.y, z.y, z.z * z.z));
    z.x += f.off_x;
    z.y += f.off_y;
    z.z += f.off_z;
    const float mR2 = f.p4 / f.p5;
    float fs = 1.0f;
    if (r2 < mR2) fs = f.p5;
    else if (r2 < f.p4) fs = __fdividef(f.p4, r2);
    z.x = z.x * fs - f.off_x;
    z.y = z.y * fs - f.off_y;
    z.z = z.z * fs - f.off_z;
    if (f.rot_main) z = turn3(f.rot_mm, false, z);  // :103
    dr = fmaf(dr * fs, f.p1, 1.0f);
    z.x = fmaf(z.x, f.p0, c.x);
    z.y = fmaf(z.y, f.p0, c.y);
    z.z = fmaf(z.z, f.p0, c.z);
  }
}

// (re + i im)^n for n >= 1 by binary exponentiation.
__device__ __forceinline__ void cpow_int(float &re, float &im, int n) {
  float ar = re, ai = im;  // the result so far (the lowest set bit of n taken first)
  while (!(n & 1)) {
    const float t = fmaf(ar, ar, -ai * ai);
    ai = 2.0f * ar * ai;
    ar = t;
    n >>= 1;
  }
  float br = ar, bi = ai;
  n >>= 1;
  while (n) {
    const float t = fmaf(br, br, -bi * bi);
    bi = 2.0f * br * bi;
    br = t;
    if (n & 1) {
      const float u = fmaf(ar, br, -ai * bi);
      ai = fmaf(ar, bi, ai * br);
      ar = u;
    }
    n >>= 1;
  }
  re = ar;
  im = ai;
}

// One Mandelbulb iteration (asin latitude form of fractal_mandelbulb.cpp:32-42) + c-addition.
// With an integer power n and no angle offsets the angle multiplication is
// De Moivre's: cos(n th) + i sin(n th) = (cos th + i sin th)^n with
// cos th = rho/r, sin th = z/r (th = asin(z/r) lies in [-pi/2, pi/2]) and
// cos ph = x/rho, sin ph = y/rho (ph = atan2(y, x)), rho = |(x, y)|; equal to
// the transcendental form in real arithmetic, with no asin, atan2, sincos or pow.
__device__ __forceinline__ void it_mandelbulb(Z3 &z, float &dr, const Z3 &c, const FastParams &f, float r) {
  if (f.bulb_n) {
    const int n = f.bulb_n;
    const float ir = rcp_approx(r);
    const float rho2 = fmaf(z.x, z.x, z.y * z.y);
    float ct = sqrt_approx(rho2) * ir, st = z.z * ir;
    float cp = 1.0f, sp = 0.0f;
    if (rho2 > 0.0f) {
      const float irho = rsqrtf(rho2);
      cp = z.x * irho;
      sp = z.y * irho;
    }
    cpow_int(ct, st, n);
    cpow_int(cp, sp, n);
    float rn = r;  // r^n
    {
      float b = r;
      int m = n - 1;
      while (m) {
        if (m & 1) rn *= b;
        b *= b;
        m >>= 1;
      }
    }
    dr = fmaf(rn * ir * dr, float(n), 1.0f);
    z.x = fmaf(ct * cp, rn, c.x);
    z.y = fmaf(ct * sp, rn, c.y);
    z.z = fmaf(st, rn, c.z);
    return;
  }
  const float th0 = asinf(z.z / r) + f.p3;
  const float ph0 = atan2f(z.y, z.x) + f.p2;
  float rp = __powf(r, f.p1);
  float sth, cth, sph, cph;
  sincosf(th0 * f.p0, &sth, &cth);
  sincosf(ph0 * f.p0, &sph, &cph);
  dr = fmaf(rp * dr, f.p0, 1.0f);
  rp *= r;
  z.x = fmaf(cth * cph, rp, c.x);
  z.y = fmaf(cth * sph, rp, c.y);
  z.z = fmaf(sth, rp, c.z);
}

// One Menger sponge iteration; c (zero unless the slot adds it) is added after.
__device__ __forceinline__ void it_menger(Z3 &z, float &dr, const Z3 &c, const FastParams &f) {
  const float ax = fabsf(z.x), ay = fabsf(z.y), az = fabsf(z.z);
  const float a = fmaxf(ax, ay), b = fminf(ax, ay);
  const float x = fmaxf(a, az), m = fminf(a, az);
  const float y = fmaxf(b, m), zz = fminf(b, m);
  const float s = f.p0;
  z.x = fmaf(x, s, -2.0f);
  z.y = fmaf(y, s, -2.0f);
  float t = zz * s;
  z.z = (t > 1.0f) ? t - 2.0f : t;
  dr *= s;
  if (f.add_c) {
    z.x += c.x;
    z.y += c.y;
    z.z += c.z;
  }
}

// Final distance of Compute + CalculateDistanceSimple clamps
// (compute_fractal.cpp:561-621, calculate_distance.cpp:569, 604-605).
__device__ __forceinline__ float final_de(const FastParams &f, float r2, float dr, int iters, float detail) {
  const float r = sqrt_approx(r2);
  float d;
  if (!(dr > 0.0f)) d = r;
  else if (f.de_fn == 2) d = (r > 1.0f) ? __fdividef(0.5f * r * __logf(r), dr) : 0.0f;
  else if (f.de_fn == 3) d = __fdividef(r - 2.0f, dr);
  else d = __fdividef(r, dr);
  if (iters < f.min_n && d < detail) d = detail;
  if (!(d == d)) d = 0.0f;  // a NaN orbit: treated as on the surface
  return fminf(fmaxf(d, 0.0f), 10.0f);
}

}  // namespace mbr
