// mbr_oracle.cpp - CPU restatement of mandelbulber2's distance-estimation
// raymarching path.  TEST INFRASTRUCTURE ONLY: the parity checker for the CUDA
// kernels and the timed CPU baseline.  The product never links or calls it.
//
// Every function follows the reference file:line it names.  Parity of the
// restatement is pinned against the reference itself: the formula iterations,
// the camera set-up and the Park-Miller generator are checked bit-for-bit
// against the reference's own sources compiled into oracle/_ref (golden
// vectors in tests/golden/, produced by tests/golden/make_golden.py).
//
// Built twice by oracle/Makefile: strict IEEE (-O2 -fno-fast-math
// -ffp-contract=off, the parity oracle) and as the reference ships
// (-O3 -ffast-math -fopenmp, qmake/common.pri:116-121, the timed baseline).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <type_traits>
#include <memory>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/mbr.h"
// the keyed formulas' parameter tables and defaults (the settings keys and
// values of InitFractalParams, a format both sides must read alike)
#include "../mandelbulber2_b200/csrc/formula_params.h"
#include "oracle_scalar.hpp"

namespace oracle {
using std::acos;
using std::asin;
using std::atan2;
using std::cos;
using std::fabs;
using std::isfinite;
using std::log;
using std::pow;
using std::sin;
using std::sqrt;

thread_local OpTally g_tally;

// ============================================================================
// Formula metadata: the constructors of the three formula classes
// (fractal_mandelbulb.cpp:16-27, fractal_mandelbox.cpp:18-29,
//  fractal_menger_sponge.cpp:17-28).  fractal_enums.h:47-88 numbering.
// ============================================================================
struct FormulaInfo {
  int de_function;      // enumDEFunctionType
  int cpixel;           // enumCPixelAddition: 0 enabled by default, 1 disabled by default, 2 already has
  double default_bailout;
  int analytic;         // enumDEAnalyticFunction
  int delta;            // DEType: 1 deltaDEType
};
static bool formula_info(int formula, FormulaInfo *fi) {
  switch (formula) {
    case MBR_FORMULA_MANDELBULB: *fi = {2, 0, 10.0, 2}; return true;
    case MBR_FORMULA_MANDELBULB_POWER2: *fi = {2, 0, 10.0, 2}; return true;  // fractal_mandelbulb_power2.cpp:17-28
    case MBR_FORMULA_HYPERCOMPLEX: *fi = {2, 0, 10.0, 2}; return true;      // fractal_hypercomplex.cpp:17-28
    case MBR_FORMULA_KALEIDOSCOPIC_IFS: *fi = {1, 1, 100.0, 3}; return true;  // fractal_kaleidoscopic_ifs.cpp:17-28
    case MBR_FORMULA_XENODREAMBUIE: *fi = {2, 0, 10.0, 2}; return true;       // fractal_xenodreambuie.cpp:17-28
    case MBR_FORMULA_QUATERNION: *fi = {2, 0, 10.0, 2}; return true;          // fractal_quaternion.cpp:16-27
    case MBR_FORMULA_AEXION: *fi = {2, 2, 10000.0, 2}; return true;           // fractal_aexion.cpp:16-27
    case MBR_FORMULA_MANDELBOX: *fi = {1, 0, 100.0, 1}; return true;
    case MBR_FORMULA_MENGER_SPONGE: *fi = {1, 1, 10.0, 3}; return true;
    case MBR_FORMULA_PSEUDO_KLEINIAN: *fi = {3, 1, 100.0, 4, 0}; return true;  // fractal_pseudo_kleinian.cpp:17-28
    case MBR_FORMULA_BOX_FOLD_BULB_POW2: *fi = {1, 0, 10000.0, 1, 1}; return true;  // fractal_box_fold_bulb_pow2.cpp:14-25
    case MBR_FORMULA_MENGER_MOD1: *fi = {1, 1, 10.0, 3, 0}; return true;  // fractal_menger_mod1.cpp:16-27
    case MBR_FORMULA_BOX_FOLD_BULB_POW2_V2: *fi = {2, 0, 100.0, 2, 0}; return true;  // fractal_box_fold_bulb_pow2_v2.cpp:16-27
    case MBR_FORMULA_ABOX_MOD11: *fi = {1, 0, 100.0, 1, 0}; return true;  // fractal_abox_mod11.cpp:21-32
    case MBR_FORMULA_PSEUDO_KLEINIAN_MOD4: *fi = {3, 1, 100.0, 4, 0}; return true;  // fractal_pseudo_kleinian_mod4.cpp:17-28
    case MBR_FORMULA_PSEUDO_KLEINIAN_STD_DE: *fi = {5, 1, 100.0, 6, 0}; return true;  // fractal_pseudo_kleinian_std_de.cpp:16-27
    case MBR_FORMULA_GENERALIZED_FOLD_BOX: *fi = {1, 0, 100.0, 1, 0}; return true;  // fractal_generalized_fold_box.cpp:17-29
    case MBR_FORMULA_MANDELBULB_PUPUKU: *fi = {2, 0, 10.0, 2, 0}; return true;  // fractal_mandelbulb_pupuku.cpp:16-27
    case MBR_FORMULA_DIFS_HEXTGRID2: *fi = {5, 1, 100.0, 6, 0}; return true;  // fractal_difs_hextgrid2.cpp:18-29
    default: return false;
  }
}

// ============================================================================
// Hybrid sequence: cHybridFractalSequences::CollectSequenceData +
// CreateSequence (hybrid_fractal_sequences.cpp:181-499) for one fractal or
// hybrid node of the default objects tree.
// ============================================================================
struct Slot {
  int formula = 0;
  bool add_c = false, check_bailout = true;
  bool add_bail = false;  // pseudo- / Jos-Kleinian DE function: the convergence bailout
  double weight = 1.0, bailout = 10.0;
  int iterations = 1, start = 0, stop = 250;
  double power = 9, alpha = 0, beta = 0;
  double mb_scale = 2, mb_limit = 1, mb_value = 2, mb_min = 0.5, mb_fixed = 1;
  double mb_offset[3] = {0, 0, 0};
  double scale3 = 3;
  bool mb_rot = false, mb_main = false;       // rotationsEnabled, mainRotationEnabled
  double mb_rot_deg[2][3][3] = {};            // rotation[fold][axis]: neg (fold 0), pos (fold 1), degrees
  double mb_main_deg[3] = {0, 0, 0};          // rotationMain, degrees
  mbr_fractal ifs = {};                       // the IFS_* parameters (fractal.cpp:96-115)
};
// A primitive of the union with its node transform (objects_tree.cpp:290-385).
struct OPrim {
  mbr_primitive q;
  double w2l[12];  // worldToLocalMatrix rows 1-3 (CMatrix44::InverseAffine, algebra.cpp:528-576)
  double abs_scale;
  double repeat[3];  // node repeat / absScale (calculate_distance.cpp:277-282)
};

struct OTree;  // an explicit objects tree (below)

struct Seq {
  std::vector<OPrim> prims;
  std::shared_ptr<OTree> tree;  // set when the scene lists nodes
  // limit box (fractparams.cpp:175-177) and global folds (:346-351)
  bool limits = false, gbox = false, gsph = false;
  double lim_min[3] = {-10, -10, -10}, lim_max[3] = {10, 10, 10};
  double gbox_limit = 1.0, gbox_value = 2.0, gsph_inner = 0.5, gsph_outer = 1.0;
  bool is_hybrid = false, julia = false;
  int length = 0, n = 0, formula_maxiter = 250, min_n = 1;
  int de_function = 1, de_analytic = 1;
  // delta DE (calculate_distance.cpp:607-760): on, and the offset factor
  // (1e-5, or deltade_relative_delta under advanced quality: set per render)
  bool delta_de = false;
  double delta_rel = 0.01, delta_factor = 1e-5;
  bool iter_thresh = false, interior = false;
  double julia_c[3] = {0, 0, 0}, cmul[3] = {1, 1, 1}, w0 = 0, linear_de_offset = 0;
  std::vector<int> seq;
  Slot slot[MBR_MAX_FRACTALS];
};

static bool build_prim(const mbr_primitive &q, OPrim *o);
static bool build_tree(const mbr_scene &sc, Seq *s);

// Returns false for scenes the restatement does not cover.
static bool build_sequence(const mbr_scene &sc, Seq *out) {
  Seq s;
  const bool hybrid = sc.hybrid_fractal_enable != 0;
  const int n = hybrid ? sc.n_fractals : 1;
  if (n < 1 || n > MBR_MAX_FRACTALS) return false;
  s.is_hybrid = hybrid;
  s.n = n;
  double maxBailout = 0.0;
  for (int i = 0; i < n; i++) {
    const mbr_fractal &f = sc.fractal[i];
    Slot &sl = s.slot[i];
    FormulaInfo fi;
    if (hybrid && f.formula == MBR_FORMULA_NONE) {  // skipped by the sequence generator
      sl.formula = MBR_FORMULA_NONE;
      continue;
    }
    if (!formula_info(f.formula, &fi)) return false;
    sl.formula = f.formula;
    sl.iterations = f.formula_iterations;
    sl.weight = f.formula_weight;
    sl.start = f.formula_start_iteration;
    sl.stop = f.formula_stop_iteration;
    sl.check_bailout = f.check_for_bailout != 0;
    if (!hybrid) sl.check_bailout = true;  // :201
    // c-constant rule :204-215
    bool addc = !(f.dont_add_c_constant != 0);
    if (fi.cpixel == 1) addc = !addc;
    if (fi.cpixel == 2) addc = false;  // cpixelAlreadyHas (hybrid_fractal_sequences.cpp:209-212)
    sl.add_c = addc;
    sl.add_bail = fi.de_function == 3 || fi.de_function == 4;  // hybrid_fractal_sequences.cpp:242-246
    if (sc.use_default_bailout) {  // :217-224
      if (hybrid) maxBailout = std::max(maxBailout, fi.default_bailout);
      else sl.bailout = fi.default_bailout;
    } else {
      sl.bailout = sc.bailout;
    }
    // sFractal::RecalculateFractalParams (fractal.cpp:673-678)
    sl.power = f.bulb_power;
    sl.alpha = f.bulb_alpha_angle_offset * 0.01745329251994329576923690768489;
    sl.beta = f.bulb_beta_angle_offset * 0.01745329251994329576923690768489;
    sl.mb_scale = f.mandelbox_scale;
    sl.mb_limit = f.mandelbox_folding_limit;
    sl.mb_value = f.mandelbox_folding_value;
    sl.mb_min = f.mandelbox_folding_min_radius;
    sl.mb_fixed = f.mandelbox_folding_fixed_radius;
    for (int k = 0; k < 3; k++) sl.mb_offset[k] = f.mandelbox_offset[k];
    sl.scale3 = f.transf_scale3;
    // fractal.cpp:67-80: rotation[0][i] = mandelbox_rotation_neg_i, rotation[1][i] = ..._pos_i
    sl.mb_rot = f.mandelbox_rotations_enabled != 0;
    sl.mb_main = f.mandelbox_main_rotation_enabled != 0;
    for (int a = 0; a < 3; a++)
      for (int k = 0; k < 3; k++) {
        sl.mb_rot_deg[0][a][k] = f.mandelbox_rotation_neg[a][k];
        sl.mb_rot_deg[1][a][k] = f.mandelbox_rotation_pos[a][k];
      }
    for (int k = 0; k < 3; k++) sl.mb_main_deg[k] = f.mandelbox_rotation_main[k];
    sl.ifs = f;
    double keyed[MBR_SLOT_X];
    if (mbr::pack_keyed(f, keyed) != -1) return false;  // a key the formula does not read
  }
  if (hybrid && sc.use_default_bailout)
    for (int i = 0; i < n; i++) s.slot[i].bailout = maxBailout;  // :253-259
  s.julia = sc.julia_mode != 0;
  for (int k = 0; k < 3; k++) {
    s.julia_c[k] = sc.julia_c[k];
    s.cmul[k] = sc.fractal_constant_factor[k];
  }
  s.w0 = sc.initial_waxis;
  s.formula_maxiter = sc.formula_maxiter;
  s.min_n = sc.min_n;
  s.iter_thresh = sc.iteration_threshold_mode != 0;
  s.interior = sc.interior_mode != 0;
  s.linear_de_offset = sc.linear_de_offset;

  // sequence generation :296-370
  const int maxN = 250;
  s.length = maxN * 5;
  s.seq.assign(s.length, 0);
  int repeatFromIndex = std::max(0, std::min(sc.repeat_from - 1, n - 1));
  int k = 0, counter = 0, last = 0;
  bool rapidEnd = false;
  for (int i = 0; i < s.length; i++) {
    counter++;
    int searchRepeatCount = 0;
    while ((s.slot[k].formula == MBR_FORMULA_NONE || i < s.slot[k].start || i > s.slot[k].stop) &&
           searchRepeatCount < n) {
      k++;
      if (k >= n) k = repeatFromIndex;
      searchRepeatCount++;
    }
    if (searchRepeatCount >= n) {
      rapidEnd = true;
      break;
    }
    s.seq[i] = k;
    last = i;
    if (counter >= s.slot[k].iterations) {
      counter = 0;
      k++;
      if (k >= n) k = repeatFromIndex;
    }
  }
  if (rapidEnd) s.length = last + 1;
  if (s.length <= 0) return false;

  // DE function choice :377-485 (analytic formulas only)
  if (hybrid) {
    if (sc.delta_de_function == MBR_DE_FUNCTION_PREFERRED) {
      int count[7] = {0, 0, 0, 0, 0, 0, 0};
      for (int i = 0; i < n; i++) {
        FormulaInfo fi;
        if (formula_info(s.slot[i].formula, &fi)) count[fi.de_function] += s.slot[i].iterations;
      }
      int maxCount = -1;
      for (int i = 1; i <= 6; i++)
        if (count[i] > maxCount) {
          maxCount = count[i];
          s.de_function = i;
        }
      if (count[5] > 0) s.de_function = 5;  // a custom-DE formula wins (:425-429)
    } else {
      s.de_function = sc.delta_de_function;
    }
  } else {
    FormulaInfo fi;
    formula_info(s.slot[0].formula, &fi);
    s.de_function = fi.de_function;
    s.de_analytic = fi.analytic;
    if (sc.delta_de_function != MBR_DE_FUNCTION_PREFERRED) {  // :477-500
      s.de_function = sc.delta_de_function;
      static const int fn_analytic[7] = {1, 1, 2, 4, 5, 6, 7};  // enumDEAnalyticFunction
      s.de_analytic = fn_analytic[s.de_function];
    }
  }
  // a delta-DE formula among the iterated slots, then the forcing switches
  // (:376-377, 412-421, 450-474)
  bool any_delta = false;
  for (int i = 0; i < n; i++) {
    FormulaInfo fi;
    if (s.slot[i].formula != MBR_FORMULA_NONE && formula_info(s.slot[i].formula, &fi) && fi.delta) any_delta = true;
  }
  s.delta_de = (any_delta || sc.delta_de_method == MBR_DE_METHOD_FORCE_DELTA) &&
               sc.delta_de_method != MBR_DE_METHOD_FORCE_ANALYTIC;
  s.delta_rel = sc.deltade_relative_delta;
  if (s.de_function < 1 || s.de_function > 6) return false;
  // the analytic Jos Kleinian function reads formula parameters not carried here
  if (!s.delta_de && (hybrid ? s.de_function == 4 : s.de_analytic == 5)) return false;
  if (sc.n_primitives < 0 || sc.n_primitives > MBR_MAX_PRIMITIVES) return false;
  for (int k = 0; k < sc.n_primitives; k++) {
    OPrim op;
    if (!build_prim(sc.primitive[k], &op)) return false;
    s.prims.push_back(op);
  }
  s.limits = sc.limits_enabled != 0;
  s.gbox = sc.box_folding != 0;
  s.gsph = sc.spherical_folding != 0;
  for (int i = 0; i < 3; i++) {
    s.lim_min[i] = sc.limit_min[i];
    s.lim_max[i] = sc.limit_max[i];
  }
  s.gbox_limit = sc.box_folding_limit;
  s.gbox_value = sc.box_folding_value;
  s.gsph_inner = sc.spherical_folding_inner;
  s.gsph_outer = sc.spherical_folding_outer;
  if (!build_tree(sc, &s)) return false;
  *out = s;
  return true;
}

// ============================================================================
// Formula iterations, templated on the scalar.
// ============================================================================
template <class S>
struct V4 {
  S x, y, z, w;
};
template <class S, class K>
inline V4<S> operator*(const V4<S> &v, const K &k) {  // CVector4 * double (algebra.hpp)
  return V4<S>{v.x * k, v.y * k, v.z * k, v.w * k};
}
template <class S>
inline S len4(const V4<S> &v) {  // CVector4::Length (algebra.hpp:401)
  return sqrt(v.x * v.x + v.y * v.y + v.z * v.z + v.w * v.w);
}
template <class S>
inline bool nan4(const V4<S> &v) {  // CVector4::IsNotANumber (algebra.hpp:444-451)
  return !(static_cast<int>(isfinite(v.x)) & static_cast<int>(isfinite(v.y)) &
           static_cast<int>(isfinite(v.z)) & static_cast<int>(isfinite(v.w)));
}
inline int sgn(double v) { return (0.0 < v) - (v < 0.0); }  // math_utilities.h:65-67

// CRotationMatrix::SetRotation2(angles * M_PI_180) (fractal.cpp:663, 669;
// algebra.cpp:296-302, 198-247): from the identity, RotateZ(z), RotateY(y),
// RotateX(x), each post-multiplying the matrix and skipped for a zero angle;
// `zero` stays set (RotateVector is the identity) when all three are zero.
// set3: SetRotation3 instead (algebra.cpp:304-310): RotateZ(x), RotateY(y), RotateX(z).
inline void mb_rotation(const double deg[3], double m[9], bool *zero, bool set3 = false,
                        double k = 0.01745329251994329576923690768489 /* M_PI_180, fractal.h:45-46 */) {
  for (int i = 0; i < 9; i++) m[i] = (i % 4 == 0) ? 1.0 : 0.0;
  *zero = true;
  const double ang[3] = {deg[set3 ? 0 : 2] * k, deg[1] * k, deg[set3 ? 2 : 0] * k};
  const int axis[3] = {2, 1, 0};
  for (int j = 0; j < 3; j++) {
    const double a = ang[j];
    if (a == 0.0) continue;
    double r[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    const double sn = sin(a), cs = cos(a);
    if (axis[j] == 0) { r[0] = 1.0; r[4] = cs; r[8] = cs; r[5] = -sn; r[7] = sn; }
    if (axis[j] == 1) { r[4] = 1.0; r[8] = cs; r[0] = cs; r[6] = -sn; r[2] = sn; }
    if (axis[j] == 2) { r[8] = 1.0; r[0] = cs; r[4] = cs; r[1] = -sn; r[3] = sn; }
    double t[9];
    for (int row = 0; row < 3; row++)
      for (int col = 0; col < 3; col++)
        t[row * 3 + col] = m[row * 3 + 0] * r[0 * 3 + col] + m[row * 3 + 1] * r[1 * 3 + col] + m[row * 3 + 2] * r[2 * 3 + col];
    std::memcpy(m, t, sizeof(t));
    *zero = false;
  }
}

// The legacy settings put every enabled primitive in a node under identity
// boolean groups (settings.cpp:2551-2940); the node's localToWorld is
// [R^T s | position] with R = SetRotation2(rotation * M_PI / 180), its world
// matrix identity * localToWorld (algebra.cpp:477-500), and the distance
// reads InverseAffine of that (objects_tree.cpp:290-385).
static bool build_prim(const mbr_primitive &q, OPrim *o) {
  if (q.type < MBR_PRIMITIVE_PLANE || q.type > MBR_PRIMITIVE_ELLIPSOID) return false;
  o->q = q;
  double R[9];
  bool zero;
  mb_rotation(q.rotation, R, &zero, false, M_PI / 180.0);
  const double s = q.scale;
  double L[4][4] = {{R[0] * s, R[3] * s, R[6] * s, q.position[0]},
                    {R[1] * s, R[4] * s, R[7] * s, q.position[1]},
                    {R[2] * s, R[5] * s, R[8] * s, q.position[2]},
                    {0.0, 0.0, 0.0, 1.0}};
  double W[4][4];
  for (int r = 0; r < 4; r++)
    for (int c = 0; c < 4; c++) {
      const double I[4] = {r == 0 ? 1.0 : 0.0, r == 1 ? 1.0 : 0.0, r == 2 ? 1.0 : 0.0, r == 3 ? 1.0 : 0.0};
      W[r][c] = I[0] * L[0][c] + I[1] * L[1][c] + I[2] * L[2][c] + I[3] * L[3][c];
    }
  const double ws = sqrt(W[0][0] * W[0][0] + W[0][1] * W[0][1] + W[0][2] * W[0][2]);
  const double sSq = ws * ws;
  double *m = o->w2l;
  for (int i = 0; i < 12; i++) m[i] = 0.0;
  if (ws > 1e-12) {
    for (int r = 0; r < 3; r++)
      for (int c = 0; c < 3; c++) m[r * 4 + c] = W[c][r] / sSq;
  }
  for (int r = 0; r < 3; r++) m[r * 4 + 3] = -(W[0][r] * W[0][3] + W[1][r] * W[1][3] + W[2][r] * W[2][3]) / sSq;
  o->abs_scale = fabs(ws);
  for (int i = 0; i < 3; i++) o->repeat[i] = q.repeat[i] / o->abs_scale;
  return true;
}

// std::max
static inline double dmax(double a, double b) { return (a < b) ? b : a; }

// One component of CVector3::repeatMod (algebra.hpp:106-115)
static inline double repeat_mod(double p, double v) {
  double t = p - v * 0.5;
  t = (v > 0.0) ? fmod(t, v) : t;
  t = t + v;
  t = (v > 0.0) ? fmod(t, v) : t;
  return t - v * 0.5;
}

// A node's local-to-world matrix composed with its parent's
// (objects_tree.cpp:285-330): W = P * [R s | t], R from SetRotation2 of the
// rotation in degrees
static void node_world(const double P[4][4], const double pos[3], const double rot[3], double scale,
                       double W[4][4]) {
  double R[9];
  bool zero;
  mb_rotation(rot, R, &zero, false, M_PI / 180.0);
  const double L[4][4] = {{R[0] * scale, R[3] * scale, R[6] * scale, pos[0]},
                          {R[1] * scale, R[4] * scale, R[7] * scale, pos[1]},
                          {R[2] * scale, R[5] * scale, R[8] * scale, pos[2]},
                          {0.0, 0.0, 0.0, 1.0}};
  for (int r = 0; r < 4; r++)
    for (int c = 0; c < 4; c++) W[r][c] = P[r][0] * L[0][c] + P[r][1] * L[1][c] + P[r][2] * L[2][c] + P[r][3] * L[3][c];
}

// CMatrix44::InverseAffine (algebra.cpp:528-576) into rows 1-3, and the
// world scale (the norm of the first row)
static void inverse_affine(const double W[4][4], double m[12], double *abs_scale) {
  const double ws = sqrt(W[0][0] * W[0][0] + W[0][1] * W[0][1] + W[0][2] * W[0][2]);
  const double sSq = ws * ws;
  for (int i = 0; i < 12; i++) m[i] = 0.0;
  if (ws > 1e-12) {
    for (int r = 0; r < 3; r++)
      for (int c = 0; c < 3; c++) m[r * 4 + c] = W[c][r] / sSq;
  }
  for (int r = 0; r < 3; r++) m[r * 4 + 3] = -(W[0][r] * W[0][3] + W[1][r] * W[1][3] + W[2][r] * W[2][3]) / sSq;
  *abs_scale = fabs(ws);
}

// Limits box of a primitive (primitive.cpp, e.g. :490-495)
static inline double limit_box(const mbr_primitive &q, double x, double y, double z, double dist) {
  if (!q.limits_enable) return dist;
  const double ax = dmax(x - q.limits_max[0], q.limits_min[0] - x);
  const double ay = dmax(y - q.limits_max[1], q.limits_min[1] - y);
  const double az = dmax(z - q.limits_max[2], q.limits_min[2] - z);
  return dmax(dist, dmax(dmax(ax, ay), az));
}

// The primitive's distance at a world point: node transform and repeat
// (calculate_distance.cpp:268-282), PrimitiveDistance (primitive.cpp:459-686;
// the water's distance from another object is the leaf's initial 1e20,
// :385-396, so its wave-from-objects terms vanish), times the node scale.
static double prim_distance(const OPrim &op, double wx, double wy, double wz) {
  const mbr_primitive &q = op.q;
  const double *m = op.w2l;
  double x = m[0] * wx + m[1] * wy + m[2] * wz + m[3];
  double y = m[4] * wx + m[5] * wy + m[6] * wz + m[7];
  double z = m[8] * wx + m[9] * wy + m[10] * wz + m[11];
  const double *v = op.repeat;
  if (sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) > 0.0) {  // CVector3::repeatMod (algebra.hpp:106-115)
    double *c[3] = {&x, &y, &z};
    for (int i = 0; i < 3; i++) {
      double t = *c[i] - v[i] * 0.5;
      t = (v[i] > 0.0) ? fmod(t, v[i]) : t;
      t = t + v[i];
      t = (v[i] > 0.0) ? fmod(t, v[i]) : t;
      *c[i] = t - v[i] * 0.5;
    }
  }
  double dist = 0.0;
  switch (q.type) {
    case MBR_PRIMITIVE_PLANE:  // :459-465
      dist = z;
      dist = q.empty ? fabs(dist) : dist;
      dist = dmax(dist - q.wall_thickness, 0.0);
      break;
    case MBR_PRIMITIVE_BOX: {  // :467-497
      double boxDist = -1e10;
      if (q.empty) {
        boxDist = dmax(fabs(x) - q.size[0] * 0.5, boxDist);
        boxDist = dmax(fabs(y) - q.size[1] * 0.5, boxDist);
        boxDist = dmax(fabs(z) - q.size[2] * 0.5, boxDist);
        boxDist = fabs(boxDist);
      } else {
        const double bx = dmax(fabs(x) - q.size[0] * 0.5, 0.0);
        const double by = dmax(fabs(y) - q.size[1] * 0.5, 0.0);
        const double bz = dmax(fabs(z) - q.size[2] * 0.5, 0.0);
        boxDist = sqrt(bx * bx + by * by + bz * bz) - q.rounding;
      }
      boxDist = dmax(boxDist - q.wall_thickness, 0.0);
      dist = limit_box(q, x, y, z, boxDist);
      break;
    }
    case MBR_PRIMITIVE_SPHERE:  // :499-511
      dist = sqrt(x * x + y * y + z * z) - q.radius;
      dist = q.empty ? fabs(dist) : dist;
      dist = dmax(dist - q.wall_thickness, 0.0);
      dist = limit_box(q, x, y, z, dist);
      break;
    case MBR_PRIMITIVE_RECTANGLE: {  // :513-520
      const double bx = dmax(fabs(x) - q.width * 0.5, 0.0);
      const double by = dmax(fabs(y) - q.height * 0.5, 0.0);
      const double bz = fabs(z);
      dist = sqrt(bx * bx + by * by + bz * bz);
      break;
    }
    case MBR_PRIMITIVE_CYLINDER:  // :522-537
      dist = sqrt(x * x + y * y) - q.radius;
      if (!q.caps) dist = fabs(dist);
      dist = dmax(fabs(z) - q.height * 0.5, dist);
      dist = q.empty ? fabs(dist) : dist;
      dist = dmax(dist - q.wall_thickness, 0.0);
      dist = limit_box(q, x, y, z, dist);
      break;
    case MBR_PRIMITIVE_CIRCLE:  // :539-545
      dist = dmax(fabs(z), sqrt(x * x + y * y) - q.radius);
      break;
    case MBR_PRIMITIVE_TORUS: {  // :640-655, CVector2::LengthPow (algebra.hpp:538)
      const double pr = pow(2, q.radius_lpow), pt = pow(2, q.tube_radius_lpow);
      const double d1 = pow(pow(x, pr) + pow(y, pr), 1.0 / pr) - q.radius;
      dist = pow(pow(d1, pt) + pow(z, pt), 1.0 / pt) - q.tube_radius;
      dist = q.empty ? fabs(dist) : dist;
      dist = dmax(dist - q.wall_thickness, 0.0);
      dist = limit_box(q, x, y, z, dist);
      break;
    }
    case MBR_PRIMITIVE_CONE: {  // :222-237 (wallNormal), :547-564
      double wx2 = 1.0, wy2 = q.radius / q.height;
      const double norm = 1.0 / sqrt(wx2 * wx2 + wy2 * wy2);
      wx2 = wx2 * norm;
      wy2 = wy2 * norm;
      z -= q.height;
      const double qq = sqrt(x * x + y * y);
      dist = wx2 * qq + wy2 * z;
      if (!q.caps) dist = fabs(dist);
      dist = dmax(-z - q.height, dist);
      dist = q.empty ? fabs(dist) : dist;
      dist = dmax(dist - q.wall_thickness, 0.0);
      dist = limit_box(q, x, y, z, dist);
      break;
    }
    case MBR_PRIMITIVE_PRISM: {  // :380-393, :657-668
      const double height = q.height / 2.0;
      const double prismAngle = q.prism_angle * M_PI / 180.0 / 2.0;
      const double triangleHeight = q.triangle_height * sin(prismAngle);
      const double ny = cos(prismAngle), nz = sin(prismAngle);
      dist = dmax(fabs(z) - height, dmax(fabs(x) * ny + y * nz, -y + triangleHeight) - triangleHeight);
      dist = q.empty ? fabs(dist) : dist;
      dist = dmax(dist - q.wall_thickness, 0.0);
      break;
    }
    case MBR_PRIMITIVE_ELLIPSOID: {  // :670-686
      const float k0 = sqrt((x / q.size[0]) * (x / q.size[0]) + (y / q.size[1]) * (y / q.size[1]) +
                            (z / q.size[2]) * (z / q.size[2]));
      const double s0 = q.size[0] * q.size[0], s1 = q.size[1] * q.size[1], s2 = q.size[2] * q.size[2];
      const float k1 = sqrt((x / s0) * (x / s0) + (y / s1) * (y / s1) + (z / s2) * (z / s2));
      dist = k0 * (k0 - 1.0) / k1;
      dist = q.empty ? fabs(dist) : dist;
      dist = dmax(dist - q.wall_thickness, 0.0);
      dist = limit_box(q, x, y, z, dist);
      break;
    }
    case MBR_PRIMITIVE_WATER: {  // :572-638
      const double length = q.length;
      const double amplitude = length * q.relative_amplitude;
      double planeDistance = z;
      if (planeDistance < amplitude * 10.0) {
        const double phase = -q.anim_speed * q.frame_no * 0.1;
        const double k = 0.23;
        double waveX = 0.0, waveY = -0.0, p = 1.0, p2 = 0.05;
        x += phase * 0.05 * (q.anim_progression_speed * 3.0 - 3.0);
        for (int i = 1; i <= q.iterations; i++) {
          const float p3 = p * p2;
          const float shift = phase / (i / 2.697 + 1.0);
          const double waveXTemp =
              sin(i + 0.4 * (waveX)*p3 + sin(k * y / length * p3 + shift * 0.134 * p3) + x / length * p3 + shift * p3) / p;
          const double waveYTemp =
              cos(i + 0.4 * (waveY)*p3 + sin(x / length * p3 + shift * 0.0179 * p3) + k * y / length * p3 +
                  shift * 0.023 * p3) /
              p;
          waveX += waveXTemp;
          waveY += waveYTemp;
          p2 = p2 + (1.0 - p2 + 0.5 * sin(shift * 0.0323)) * 0.7;
          p *= 1.872;
        }
        planeDistance += (waveX + waveY) * amplitude;
      }
      planeDistance = q.empty ? fabs(planeDistance) : planeDistance;
      planeDistance = dmax(planeDistance - q.wall_thickness, 0.0);
      dist = limit_box(q, x, y, z, planeDistance);
      break;
    }
  }
  return dist * op.abs_scale;
}

// Formula parameters in the scalar type, so tangents can be seeded.
template <class S>
struct SlotT {
  S power, alpha, beta;
  S mb_scale, mb_limit, mb_value, mb_mR2, mb_fR2, mb_factor1;
  S mb_off[3];
  S scale3;
  bool mb_rot, mb_main;
  double mb_rm[2][3][9];  // rot[fold][axis]; rotinv is its transpose (fractal.cpp:670)
  bool mb_rz[2][3];       // rot[fold][axis].zero
  double mb_mm[9];        // mainRot
  bool mb_mz;             // mainRot.zero
  // kaleidoscopic IFS (sFractalIFS after RecalculateFractalParams, fractal.cpp:655-661)
  bool ifs_abs[3], ifs_enabled[9], ifs_menger, ifs_rot_on, ifs_edge_on, ifs_main_zero, ifs_rot_zero[9];
  double ifs_scale, ifs_offset[3], ifs_edge[3], ifs_main[9], ifs_rot[9][9], ifs_dir[9][3], ifs_dist[9], ifs_int[9];
  double x[MBR_SLOT_X];   // a keyed formula's parameters (formula_params.h layout)
};
enum { TAN_POWER = 0, TAN_SCALE = 1, TAN_MR2 = 2, TAN_X = 3, TAN_Y = 4, TAN_Z = 5 };

template <class S>
S seeded(double v, int k, int want);
template <>
inline double seeded<double>(double v, int, int) { return v; }
template <>
inline OpCount seeded<OpCount>(double v, int, int) { return OpCount(v); }
template <class S>
S seeded(double v, int k, int want) {
  return want ? S::seed(v, k) : S(v);
}

template <class S>
SlotT<S> make_slot(const Slot &s, bool tangents) {
  SlotT<S> t;
  t.power = seeded<S>(s.power, TAN_POWER, tangents);
  t.alpha = S(s.alpha);
  t.beta = S(s.beta);
  t.mb_scale = seeded<S>(s.mb_scale, TAN_SCALE, tangents);
  t.mb_limit = S(s.mb_limit);
  t.mb_value = S(s.mb_value);
  // RecalculateFractalParams (fractal.cpp:673-675)
  t.mb_fR2 = S(s.mb_fixed * s.mb_fixed);
  t.mb_mR2 = seeded<S>(s.mb_min * s.mb_min, TAN_MR2, tangents);
  t.mb_factor1 = t.mb_fR2 / t.mb_mR2;
  for (int k = 0; k < 3; k++) t.mb_off[k] = S(s.mb_offset[k]);
  t.scale3 = S(s.scale3);
  t.mb_rot = s.mb_rot;
  t.mb_main = s.mb_main;
  for (int f = 0; f < 2; f++)
    for (int a = 0; a < 3; a++) mb_rotation(s.mb_rot_deg[f][a], t.mb_rm[f][a], &t.mb_rz[f][a]);
  mb_rotation(s.mb_main_deg, t.mb_mm, &t.mb_mz);
  const mbr_fractal &f = s.ifs;
  t.ifs_abs[0] = f.ifs_abs_x != 0;
  t.ifs_abs[1] = f.ifs_abs_y != 0;
  t.ifs_abs[2] = f.ifs_abs_z != 0;
  t.ifs_menger = f.ifs_menger_sponge_mode != 0;
  t.ifs_rot_on = f.ifs_rotation_enabled != 0;
  t.ifs_edge_on = f.ifs_edge_enabled != 0;
  t.ifs_scale = f.ifs_scale;
  for (int k = 0; k < 3; k++) {
    t.ifs_offset[k] = f.ifs_offset[k];
    t.ifs_edge[k] = f.ifs_edge[k];
  }
  mb_rotation(f.ifs_rotation, t.ifs_main, &t.ifs_main_zero, true);
  for (int i = 0; i < 9; i++) {
    t.ifs_enabled[i] = f.ifs_enabled[i] != 0;
    mb_rotation(f.ifs_rotations[i], t.ifs_rot[i], &t.ifs_rot_zero[i], true);
    // CVector4(direction, 0).Normalize() when read and again in RecalculateFractalParams
    double d[4] = {f.ifs_direction[i][0], f.ifs_direction[i][1], f.ifs_direction[i][2], 0.0};
    for (int rep = 0; rep < 2; rep++) {
      const double norm = 1.0 / sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2] + d[3] * d[3]);
      for (int c = 0; c < 4; c++) d[c] = d[c] * norm;
    }
    for (int c = 0; c < 3; c++) t.ifs_dir[i][c] = d[c];
    t.ifs_dist[i] = f.ifs_distance[i];
    t.ifs_int[i] = f.ifs_intensity[i];
  }
  mbr::pack_keyed(f, t.x);  // validated when the sequence was built
  return t;
}

// CRotationMatrix::RotateVector of a CVector4: xyz turned, w kept
// (algebra.cpp:333-344, 168-175); `transpose` applies the matrix's transpose
// (rotinv, whose zero flag Transpose() clears: algebra.cpp:398-411).
template <class S>
inline V4<S> mb_turn(const double *m, bool zero, bool transpose, const V4<S> &v) {
  if (zero && !transpose) return v;
  V4<S> r = v;
  if (!transpose) {
    r.x = S(m[0]) * v.x + S(m[1]) * v.y + S(m[2]) * v.z;
    r.y = S(m[3]) * v.x + S(m[4]) * v.y + S(m[5]) * v.z;
    r.z = S(m[6]) * v.x + S(m[7]) * v.y + S(m[8]) * v.z;
  } else {
    r.x = S(m[0]) * v.x + S(m[3]) * v.y + S(m[6]) * v.z;
    r.y = S(m[1]) * v.x + S(m[4]) * v.y + S(m[7]) * v.z;
    r.z = S(m[2]) * v.x + S(m[5]) * v.y + S(m[8]) * v.z;
  }
  return r;
}

// cFractalMandelbulb::FormulaCode (fractal_mandelbulb.cpp:29-43)
template <class S>
inline void formula_mandelbulb(V4<S> &z, const SlotT<S> &f, S &r, S &DE) {
  const S th0 = asin(z.z / r) + f.beta;
  const S ph0 = atan2(z.y, z.x) + f.alpha;
  S rp = pow(r, f.power - 1.0);
  const S th = th0 * f.power;
  const S ph = ph0 * f.power;
  const S cth = cos(th);
  DE = (rp * DE) * f.power + 1.0;
  rp = rp * r;
  z.x = cth * cos(ph) * rp;
  z.y = cth * sin(ph) * rp;
  z.z = sin(th) * rp;
}

// cFractalMandelbox::FormulaCode (fractal_mandelbox.cpp:31-107)
template <class S>
inline void formula_mandelbox(V4<S> &z, const SlotT<S> &f, S &DE) {
  if (f.mb_rot) {
    // each axis folded in the frame of rot[0][dim] (above the limit), else
    // of rot[1][dim] (below minus the limit), and turned back (:33-63)
    for (int dim = 0; dim < 3; dim++) {
      V4<S> zr = mb_turn(f.mb_rm[0][dim], f.mb_rz[0][dim], false, z);
      S &a = dim == 0 ? zr.x : (dim == 1 ? zr.y : zr.z);
      if (a > f.mb_limit) {
        a = f.mb_value - a;
        z = mb_turn(f.mb_rm[0][dim], false, true, zr);
      } else {
        zr = mb_turn(f.mb_rm[1][dim], f.mb_rz[1][dim], false, z);
        S &b = dim == 0 ? zr.x : (dim == 1 ? zr.y : zr.z);
        if (b < -f.mb_limit) {
          b = -f.mb_value - b;
          z = mb_turn(f.mb_rm[1][dim], false, true, zr);
        }
      }
    }
  } else {
    if (fabs(z.x) > f.mb_limit) z.x = S(double(sgn(val(z.x)))) * f.mb_value - z.x;
    if (fabs(z.y) > f.mb_limit) z.y = S(double(sgn(val(z.y)))) * f.mb_value - z.y;
    if (fabs(z.z) > f.mb_limit) z.z = S(double(sgn(val(z.z)))) * f.mb_value - z.z;
  }
  const S r2 = z.x * z.x + z.y * z.y + z.z * z.z + z.w * z.w;
  z.x = z.x + f.mb_off[0];
  z.y = z.y + f.mb_off[1];
  z.z = z.z + f.mb_off[2];
  z.w = z.w + 0.0;
  if (r2 < f.mb_mR2) {
    z.x = z.x * f.mb_factor1; z.y = z.y * f.mb_factor1; z.z = z.z * f.mb_factor1; z.w = z.w * f.mb_factor1;
    DE = DE * f.mb_factor1;
  } else if (r2 < f.mb_fR2) {
    const S tglad_factor2 = f.mb_fR2 / r2;
    z.x = z.x * tglad_factor2; z.y = z.y * tglad_factor2; z.z = z.z * tglad_factor2; z.w = z.w * tglad_factor2;
    DE = DE * tglad_factor2;
  }
  z.x = z.x - f.mb_off[0];
  z.y = z.y - f.mb_off[1];
  z.z = z.z - f.mb_off[2];
  z.w = z.w - 0.0;
  if (f.mb_main) z = mb_turn(f.mb_mm, f.mb_mz, false, z);  // :103
  z.x = z.x * f.mb_scale; z.y = z.y * f.mb_scale; z.z = z.z * f.mb_scale; z.w = z.w * f.mb_scale;
  DE = DE * fabs(f.mb_scale) + 1.0;
}

// cFractalMandelbulbPower2::FormulaCode (fractal_mandelbulb_power2.cpp:30-45)
template <class S>
inline void formula_bulb_pow2(V4<S> &z, const S &r, S &DE) {
  DE = DE * 2.0 * r;
  const S x2 = z.x * z.x;
  const S y2 = z.y * z.y;
  const S z2 = z.z * z.z;
  const S temp = 1.0 - z2 / (x2 + y2);
  const S nx = (x2 - y2) * temp;
  const S ny = 2.0 * z.x * z.y * temp;
  const S nz = -2.0 * z.z * sqrt(x2 + y2);
  z.x = nx;
  z.y = ny;
  z.z = nz;
}

// cFractalXenodreambuie::FormulaCode (fractal_xenodreambuie.cpp:30-49)
template <class S>
inline void formula_xenodreambuie(V4<S> &z, const SlotT<S> &f, const S &r, S &DE) {
  S rp = pow(r, f.power - 1.0);
  DE = rp * DE * f.power + 1.0;
  rp = rp * r;
  const S th = (atan2(z.y, z.x) + f.beta) * f.power;
  S ph = acos(z.z / r) + f.alpha;
  if (fabs(ph) > 0.5 * M_PI) ph = double(sgn(val(ph))) * M_PI - ph;  // sign(ph) * M_PI - ph
  ph = ph * f.power;
  const S sph = sin(ph);
  z.x = rp * cos(th) * sph;
  z.y = rp * sin(th) * sph;
  z.z = rp * cos(ph);
}

// cFractalPseudoKleinian::FormulaCode (fractal_pseudo_kleinian.cpp:30-202)
// without the aux.color terms; pk is aux.pseudoKleinianDE.
template <class S>
inline void formula_pseudo_kleinian(V4<S> &z, const SlotT<S> &f, S &DE, S &pk, int i) {
  using namespace mbr;
  const double *x = f.x;
  if (x[PKX_SPH_INV] != 0.0 && i >= int(x[PKX_START_X]) && i < int(x[PKX_STOP_1])) {  // :33-44
    z.x = z.x + x[PKX_OFFSET000];
    z.y = z.y + x[PKX_OFFSET000 + 1];
    z.z = z.z + x[PKX_OFFSET000 + 2];
    z.w = z.w + 0.0;
    const S rr = z.x * z.x + z.y * z.y + z.z * z.z + z.w * z.w;
    const S q = x[PKX_MAXR2] / rr;
    z.x = z.x * q;
    z.y = z.y * q;
    z.z = z.z * q;
    z.w = z.w * q;
    z.x = z.x + (x[PKX_ADD_A000] - x[PKX_OFFSET000]);
    z.y = z.y + (x[PKX_ADD_A000 + 1] - x[PKX_OFFSET000 + 1]);
    z.z = z.z + (x[PKX_ADD_A000 + 2] - x[PKX_OFFSET000 + 2]);
    z.w = z.w + (0.0 - 0.0);
    DE = DE * (x[PKX_MAXR2] / rr) + x[PKX_DE_OFFSET0];
  }
  if (x[PKX_PRISM] != 0.0 && i >= int(x[PKX_START_P]) && i < int(x[PKX_STOP_P1])) {  // :47-75
    const double kSqrt34 = 0.86602540378443864676372317075294, kSqrt3 = 1.73205080756887729352744634150587;
    z.y = fabs(z.y);
    z.z = fabs(z.z);
    const S dot1 = (z.x * -kSqrt34 + z.y * 0.5) * x[PKX_SCALE];
    S t = std::max(S(0.0), dot1);
    z.x = z.x - t * -kSqrt3;
    z.y = fabs(z.y - t);
    if (z.y > z.z) {
      t = z.y;
      z.y = z.z;
      z.z = t;
    }
    z.x = z.x - x[PKX_CMUL000] * kSqrt34;
    z.y = z.y - x[PKX_CMUL000 + 1] * 1.5;
    z.z = z.z - x[PKX_CMUL000 + 2] * 1.5;
    z.w = z.w - 1.0 * 0.0;
    if (z.z > z.x) {
      t = z.z;
      z.z = z.x;
      z.x = t;
    }
    if (z.x > 0.0) {
      z.y = std::max(S(0.0), z.y);
      z.z = std::max(S(0.0), z.z);
    }
  }
  if (x[PKX_ABS_BOX] != 0.0 && i >= int(x[PKX_START_E]) && i < int(x[PKX_STOP_E])) {  // :78-91
    z.x = fabs(z.x + x[PKX_ADD111]) - fabs(z.x - x[PKX_ADD111]) - z.x;
    z.y = fabs(z.y + x[PKX_ADD111 + 1]) - fabs(z.y - x[PKX_ADD111 + 1]) - z.y;
    if (x[PKX_ABS_BOX_Z] != 0.0) z.z = fabs(z.z + x[PKX_ADD111 + 2]) - fabs(z.z - x[PKX_ADD111 + 2]) - z.z;
  }
  if (x[PKX_BOX] != 0.0 && i >= int(x[PKX_START_A]) && i < int(x[PKX_STOP_A])) {  // :94-115
    if (fabs(z.x) > x[PKX_MB_LIMIT]) z.x = S(double(sgn(val(z.x)))) * x[PKX_MB_VALUE] - z.x;
    if (fabs(z.y) > x[PKX_MB_LIMIT]) z.y = S(double(sgn(val(z.y)))) * x[PKX_MB_VALUE] - z.y;
    const double zLimit = x[PKX_MB_LIMIT] * x[PKX_SCALE1];
    const double zValue = x[PKX_MB_VALUE] * x[PKX_SCALE1];
    if (fabs(z.z) > zLimit) z.z = S(double(sgn(val(z.z)))) * zValue - z.z;
  }
  if (i >= int(x[PKX_START_C]) && i < int(x[PKX_STOP_C])) {  // :118-138
    const double cx = x[PKX_CSIZE], cy = x[PKX_CSIZE + 1], cz = x[PKX_CSIZE + 2];
    V4<S> t = z;
    if (z.x > cx) t.x = cx;
    if (z.x < -cx) t.x = -cx;
    if (z.y > cy) t.y = cy;
    if (z.y < -cy) t.y = -cy;
    if (z.z > cz) t.z = cz;
    if (z.z < -cz) t.z = -cz;
    z.x = t.x * 2.0 - z.x;
    z.y = t.y * 2.0 - z.y;
    z.z = t.z * 2.0 - z.z;
    z.w = t.w * 2.0 - z.w;
    const S k = std::max(S(x[PKX_MINR05] / (z.x * z.x + z.y * z.y + z.z * z.z + z.w * z.w)), S(1.0));
    z.x = z.x * k;
    z.y = z.y * k;
    z.z = z.z * k;
    z.w = z.w * k;
    if (x[PKX_FLIP_Z] != 0.0) z.z = -z.z;
    if (x[PKX_FLIP_W] != 0.0) z.w = -z.w;
    DE = DE * (k + x[PKX_TWEAK005]);
    pk = x[PKX_DE_SCALE1];
  }
  if (x[PKX_ROT_ON] != 0.0 && i >= int(x[PKX_START_R]) && i < int(x[PKX_STOP_R]))  // :141-144
    z = mb_turn(x + PKX_ROT + 1, x[PKX_ROT] != 0.0, false, z);
  z.x = z.x + x[PKX_ADD000];  // :147
  z.y = z.y + x[PKX_ADD000 + 1];
  z.z = z.z + x[PKX_ADD000 + 2];
  z.w = z.w + 0.0;
}

// cFractalBoxFoldBulbPow2::FormulaCode (fractal_box_fold_bulb_pow2.cpp:27-76)
template <class S>
inline void formula_box_fold_bulb_pow2(V4<S> &z, const SlotT<S> &f, const S &r, S &DE) {
  using namespace mbr;
  const double *x = f.x;
  const double ff = x[BFX_FOLD];
  if (fabs(z.x) > ff) z.x = S(double(sgn(val(z.x))) * ff * 2.0) - z.x;
  if (fabs(z.y) > ff) z.y = S(double(sgn(val(z.y))) * ff * 2.0) - z.y;
  if (fabs(z.z) > ff) z.z = S(double(sgn(val(z.z))) * ff * 2.0) - z.z;
  const double fR2_2 = 1.0, mR2_2 = 0.25;
  const S r2_2 = z.x * z.x + z.y * z.y + z.z * z.z + z.w * z.w;
  const double tglad_factor1_2 = fR2_2 / mR2_2;
  if (r2_2 < mR2_2) {
    z = z * tglad_factor1_2;
    DE = DE * tglad_factor1_2;
  } else if (r2_2 < fR2_2) {
    const S tglad_factor2_2 = fR2_2 / r2_2;
    z = z * tglad_factor2_2;
    DE = DE * tglad_factor2_2;
  }
  z = z * 2.0;
  const S x2 = z.x * z.x, y2 = z.y * z.y, z2 = z.z * z.z;
  const S temp = 1.0 - z2 / (x2 + y2);
  V4<S> t;
  t.x = (x2 - y2) * temp;
  t.y = 2.0 * z.x * z.y * temp;
  t.z = -2.0 * z.z * sqrt(x2 + y2);
  t.w = z.w;
  z = t;
  z.z = z.z * x[BFX_ZFACTOR];
  if (x[BFX_ADE_ON] != 0.0)  // :67-73
    DE = (DE + 1.0) * 5.0 * r * x[BFX_ADE_SCALE1] *
             sqrt(x[BFX_ZFACTOR] * x[BFX_ZFACTOR] + 2.0 + x[BFX_ADE_OFFSET2]) +
         x[BFX_ADE_OFFSET1];
}

// cFractalBoxFoldBulbPow2V2::FormulaCode (fractal_box_fold_bulb_pow2_v2.cpp:
// 29-146) without the aux.color terms; scaleA is aux.actualScaleA
template <class S>
inline void formula_box_fold_bulb_pow2_v2(V4<S> &z, const SlotT<S> &f, S &DE, S &scaleA, int i) {
  using namespace mbr;
  const double *x = f.x;
  if (i >= int(x[B2X_START_B]) && i < int(x[B2X_STOP_B])) {  // :35-45
    z.x = fabs(z.x + x[B2X_ADD111]) - fabs(z.x - x[B2X_ADD111]) - z.x;
    z.y = fabs(z.y + x[B2X_ADD111 + 1]) - fabs(z.y - x[B2X_ADD111 + 1]) - z.y;
    z.z = fabs(z.z + x[B2X_ADD111 + 2]) - fabs(z.z - x[B2X_ADD111 + 2]) - z.z;
  }
  if (i >= int(x[B2X_START_S]) && i < int(x[B2X_STOP_S])) {  // :48-67
    const S rr = z.x * z.x + z.y * z.y + z.z * z.z + z.w * z.w;
    z.x = z.x + x[B2X_MB_OFFSET];
    z.y = z.y + x[B2X_MB_OFFSET + 1];
    z.z = z.z + x[B2X_MB_OFFSET + 2];
    z.w = z.w + 0.0;
    if (rr < x[B2X_MINR2]) {
      const double tglad_factor1 = x[B2X_MAXR2] / x[B2X_MINR2];
      z = z * tglad_factor1;
      DE = DE * tglad_factor1;
    } else if (rr < x[B2X_MAXR2]) {
      const S tglad_factor2 = x[B2X_MAXR2] / rr;
      z = z * tglad_factor2;
      DE = DE * tglad_factor2;
    }
    z.x = z.x - x[B2X_MB_OFFSET];
    z.y = z.y - x[B2X_MB_OFFSET + 1];
    z.z = z.z - x[B2X_MB_OFFSET + 2];
    z.w = z.w - 0.0;
  }
  if (i >= int(x[B2X_START_C]) && i < int(x[B2X_STOP_C])) {  // :70-88
    const S useScale = scaleA + x[B2X_SCALE];
    z = z * useScale;
    DE = DE * fabs(useScale);
    if (i >= int(x[B2X_START_X]) && i < int(x[B2X_STOP_X])) {
      const S vary = x[B2X_SCALE_VARY] * (fabs(scaleA) - x[B2X_SCALE_B1]);
      if (x[B2X_VARY_M] != 0.0) scaleA = -vary;
      else scaleA = scaleA - vary;
    }
  }
  if (i >= int(x[B2X_START_A]) && i < int(x[B2X_STOP_A])) {  // :90-110
    const S r = len4(z);
    DE = r * DE * 16.0 * x[B2X_ADE_SCALE1] * sqrt(x[B2X_ZFACTOR] * x[B2X_ZFACTOR] + 2.0 + x[B2X_ADE_OFFSET2]) /
             1.73205080756887729352744634150587 +
         x[B2X_ADE_OFFSET1];
    z = z * 2.0;
    const S x2 = z.x * z.x, y2 = z.y * z.y, z2 = z.z * z.z;
    const S temp = 1.0 - z2 / (x2 + y2);
    V4<S> t;
    t.x = (x2 - y2) * temp;
    t.y = 2.0 * z.x * z.y * temp;
    t.z = -2.0 * z.z * sqrt(x2 + y2);
    t.w = z.w;
    z = t;
    z.z = z.z * x[B2X_ZFACTOR];
  }
}

// cFractalPseudoKleinianMod4::FormulaCode (fractal_pseudo_kleinian_mod4.cpp:
// 29-145) without the aux.color terms
template <class S>
inline void formula_pseudo_kleinian_mod4(V4<S> &z, const SlotT<S> &f, S &DE, S &pk, S &posNeg, int i) {
  using namespace mbr;
  const double *x = f.x;
  if (x[P4X_SPH_INV] != 0.0 && i >= int(x[P4X_START_X]) && i < int(x[P4X_STOP_1])) {
    z.x = z.x + x[P4X_OFFSET000];
    z.y = z.y + x[P4X_OFFSET000 + 1];
    z.z = z.z + x[P4X_OFFSET000 + 2];
    z.w = z.w + 0.0;
    const S rr = z.x * z.x + z.y * z.y + z.z * z.z + z.w * z.w;
    z = z * S(x[P4X_SCALE_G1] / rr);
    DE = DE * (x[P4X_SCALE_G1] / rr);
    z.x = z.x + (x[P4X_ADD_P000] - x[P4X_OFFSET000]);
    z.y = z.y + (x[P4X_ADD_P000 + 1] - x[P4X_OFFSET000 + 1]);
    z.z = z.z + (x[P4X_ADD_P000 + 2] - x[P4X_OFFSET000 + 2]);
    z.w = z.w + (0.0 - 0.0);
    z = z * x[P4X_SCALE_A1];
    DE = DE * x[P4X_SCALE_A1];
  }
  if (i >= int(x[P4X_START_M]) && i < int(x[P4X_STOP_M])) {
    z.x = z.x - x[P4X_CM000] * S(double(sgn(val(z.x))));
    z.y = z.y - x[P4X_CM000 + 1] * S(double(sgn(val(z.y))));
    z.z = z.z - x[P4X_CM000 + 2] * S(double(sgn(val(z.z))));
  }
  z.x = fabs(z.x + x[P4X_CSIZE]) - fabs(z.x - x[P4X_CSIZE]) - z.x;
  z.y = fabs(z.y + x[P4X_CSIZE + 1]) - fabs(z.y - x[P4X_CSIZE + 1]) - z.y;
  z.z = fabs(z.z + x[P4X_CSIZE + 2]) - fabs(z.z - x[P4X_CSIZE + 2]) - z.z;
  z.w = fabs(z.w + 0.0) - fabs(z.w - 0.0) - z.w;
  const S k = std::max(S(x[P4X_MINR05] / (z.x * z.x + z.y * z.y + z.z * z.z + z.w * z.w)), S(1.0));
  z = z * k;
  DE = DE * (k + x[P4X_TWEAK005]);
  pk = x[P4X_DE_SCALE1];
  z.x = z.x + x[P4X_ADD000];
  z.y = z.y + x[P4X_ADD000 + 1];
  z.z = z.z + x[P4X_ADD000 + 2];
  z.w = z.w + 0.0;
  if (x[P4X_G_ON] != 0.0 && i >= int(x[P4X_START_G]) && i < int(x[P4X_STOP_G])) {
    z.x = z.x + posNeg * x[P4X_ADD_A000];
    z.y = z.y + posNeg * x[P4X_ADD_A000 + 1];
    z.z = z.z + posNeg * x[P4X_ADD_A000 + 2];
    posNeg = posNeg * x[P4X_SCALE_NEG1];
  }
  if (x[P4X_F_ON] != 0.0 && i >= int(x[P4X_START_F]) && i < int(x[P4X_STOP_F])) {
    z.x = fabs(z.x + x[P4X_OFFSET_A000]) - fabs(z.x - x[P4X_OFFSET_A000]) - z.x;
    z.y = fabs(z.y + x[P4X_OFFSET_A000 + 1]) - fabs(z.y - x[P4X_OFFSET_A000 + 1]) - z.y;
    z.z = fabs(z.z + x[P4X_OFFSET_A000 + 2]) - fabs(z.z - x[P4X_OFFSET_A000 + 2]) - z.z;
    z.w = fabs(z.w + 0.0) - fabs(z.w - 0.0) - z.w;
  }
  if (x[P4X_N_ON] != 0.0 && i >= int(x[P4X_START_N]) && i < int(x[P4X_STOP_N])) {
    S t;
    z.x = fabs(z.x);
    z.y = fabs(z.y);
    if (x[P4X_SWAP_A] != 0.0) {
      t = z.x;
      z.x = z.y;
      z.y = t;
    }
    t = z.x;
    z.x = z.x + z.y - x[P4X_OFFSET0];
    z.y = t - z.y - x[P4X_OFFSET_A0];
    if (x[P4X_BX_F] != 0.0 && i >= int(x[P4X_START_O]) && i < int(x[P4X_STOP_O])) z.x = -fabs(z.x);
    if (x[P4X_BX] != 0.0 && i >= int(x[P4X_START_P]) && i < int(x[P4X_STOP_P])) z.y = -fabs(z.y);
    t = z.x;
    z.x = z.x + z.y;
    z.y = t - z.y;
    z.x = z.x * 0.5;
    z.y = z.y * 0.5;
    if (x[P4X_AX] != 0.0 && i >= int(x[P4X_START_R]) && i < int(x[P4X_STOP_R]))
      z.x = x[P4X_OFFSET1] - fabs(z.x + x[P4X_OFFSET1]);
    if (x[P4X_AX_F] != 0.0 && i >= int(x[P4X_START_RV]) && i < int(x[P4X_STOP_RV]))
      z.y = x[P4X_OFFSET_A1] - fabs(z.y + x[P4X_OFFSET_A1]);
  }
  if (x[P4X_FLIP_X] != 0.0) z.x = -z.x;
  if (x[P4X_FLIP_Y] != 0.0) z.y = -z.y;
  if (x[P4X_FLIP_Z] != 0.0) z.z = -z.z;
}

// cFractalGeneralizedFoldBox::FormulaCode (fractal_generalized_fold_box.cpp:
// 31-245) without the aux.color terms
template <class S>
inline void formula_generalized_fold_box(V4<S> &z, const SlotT<S> &f, S &DE) {
  using namespace mbr;
  const double *x = f.x;
  struct V3 {
    S x, y, z;
  };
  auto dot = [](const V3 &a, const V3 &b) { return a.x * b.x + a.y * b.y + a.z * b.z; };
  auto nv = [&](int i) { return V3{S(x[GFX_NV + 3 * i]), S(x[GFX_NV + 3 * i + 1]), S(x[GFX_NV + 3 * i + 2])}; };
  const int sides = int(x[GFX_SIDES]);
  const double melt = x[GFX_MELT], solid = x[GFX_SOLID];
  V3 zXYZ{z.x, z.y, z.z};
  V3 L = zXYZ;
  S a = 1.0;
  int side = -1;
  for (int i = 0; i < sides; i++) {
    const S b = solid;
    const S c = dot(L, nv(i));
    if ((c > 0.0) && ((a * c) > b)) {
      side = i;
      a = b / c;
    }
  }
  if (side != -1) {
    const int side_m = side;
    const V3 Nm = nv(side_m);
    const S dm = dot(zXYZ, Nm) - solid;
    const V3 Xm{zXYZ.x - Nm.x * dm, zXYZ.y - Nm.y * dm, zXYZ.z - Nm.z * dm};
    L = V3{Xm.x - Nm.x, Xm.y - Nm.y, Xm.z - Nm.z};
    V3 Y = Nm;
    a = 1.0;
    side = -1;
    for (int i = 0; i < sides; i++) {
      if (i != side_m) {
        const S b = solid - dot(Y, nv(i));
        const S c = dot(L, nv(i));
        if ((c > 0.0) && ((a * c) > b)) {
          side = i;
          a = b / c;
        }
      }
    }
    V3 target;
    if (side != -1) {
      const V3 Xmr{Y.x + L.x * a, Y.y + L.y * a, Y.z + L.z * a};
      const int side_r = side;
      const V3 Nr = nv(side_r);
      V3 Lr{Nm.y * Nr.z - Nm.z * Nr.y, -Nm.x * Nr.z + Nm.z * Nr.x, Nm.x * Nr.y - Nm.y * Nr.x};
      S a_rmin = (dot(zXYZ, Lr) - dot(Xmr, Lr)) / (dot(Lr, Lr));
      if (a_rmin < 0.0) {
        a_rmin = -a_rmin;
        Lr = V3{Lr.x * -1.0, Lr.y * -1.0, Lr.z * -1.0};
      }
      const V3 Xr{Xmr.x + Lr.x * a_rmin, Xmr.y + Lr.y * a_rmin, Xmr.z + Lr.z * a_rmin};
      L = V3{Xr.x - Xmr.x, Xr.y - Xmr.y, Xr.z - Xmr.z};
      Y = Xmr;
      a = 1.0;
      side = -1;
      for (int i = 0; i < sides; i++) {
        if ((i != side_m) && (i != side_r)) {
          const S b = solid - dot(Y, nv(i));
          const S c = dot(L, nv(i));
          if ((c > 0.0) && ((a * c) > b)) {
            side = i;
            a = b / c;
          }
        }
      }
      target = (side != -1) ? V3{Y.x + L.x * a, Y.y + L.y * a, Y.z + L.z * a} : Xr;
    } else {
      target = Xm;
    }
    const V3 z2X{target.x - zXYZ.x, target.y - zXYZ.y, target.z - zXYZ.z};
    if (dot(z2X, z2X) > (melt * melt)) {
      const S mag = sqrt(dot(z2X, z2X));
      const S k = 2.0 * (mag - melt) / (mag + .00000001);
      zXYZ = V3{zXYZ.x + z2X.x * k, zXYZ.y + z2X.y * k, zXYZ.z + z2X.z * k};
    }
  }
  const S r2 = dot(zXYZ, zXYZ);
  z = V4<S>{zXYZ.x, zXYZ.y, zXYZ.z, z.w};
  z.x = z.x + x[GFX_MB_OFFSET];
  z.y = z.y + x[GFX_MB_OFFSET + 1];
  z.z = z.z + x[GFX_MB_OFFSET + 2];
  z.w = z.w + 0.0;
  const double mR2 = x[GFX_MB_MINR] * x[GFX_MB_MINR], fR2 = x[GFX_MB_FIXEDR] * x[GFX_MB_FIXEDR];
  const double factor1 = fR2 / mR2;
  if (r2 < mR2) {
    z = z * factor1;
    DE = DE * factor1;
  } else if (r2 < fR2) {
    const S f2 = fR2 / r2;
    z = z * f2;
    DE = DE * f2;
  }
  z.x = z.x - x[GFX_MB_OFFSET];
  z.y = z.y - x[GFX_MB_OFFSET + 1];
  z.z = z.z - x[GFX_MB_OFFSET + 2];
  z.w = z.w - 0.0;
  if (x[GFX_MAIN_ON] != 0.0) z = mb_turn(x + GFX_MAIN_ROT + 1, x[GFX_MAIN_ROT] != 0.0, false, z);
  z = z * x[GFX_MB_SCALE];
  DE = DE * fabs(x[GFX_MB_SCALE]) + 1.0;
}

// cFractalMandelbulbPupuku::FormulaCode (fractal_mandelbulb_pupuku.cpp:29-144);
// r is aux.r (the formula may replace it), dist is aux.dist
template <class S>
inline void formula_mandelbulb_pupuku(V4<S> &z, const SlotT<S> &f, S r, S &DE, S &dist, int i) {
  using namespace mbr;
  const double *x = f.x;
  S t;
  if (x[PPX_P_ON] != 0.0 && i >= int(x[PPX_START_P]) && i < int(x[PPX_STOP_P])) {
    if (x[PPX_CX] != 0.0) z.x = fabs(z.x);
    if (x[PPX_CY] != 0.0) z.y = fabs(z.y);
    if (x[PPX_CZ] != 0.0) z.z = fabs(z.z);
    z.x = z.x + x[PPX_OFFSET_A000];
    z.y = z.y + x[PPX_OFFSET_A000 + 1];
    z.z = z.z + x[PPX_OFFSET_A000 + 2];
    z.w = z.w + 0.0;
    if (x[PPX_T_ON] != 0.0) r = len4(z);
  }
  if (x[PPX_SW] == 0.0) t = asin(z.z / r);
  else t = acos(z.z / r);
  const S th = (t + x[PPX_BETA]) * x[PPX_POWER] * x[PPX_SCALE_A1];
  S ph = (atan2(z.y, z.x) + x[PPX_ALPHA]) * x[PPX_POWER] * x[PPX_SCALE_B1];
  S rp = pow(r, S(x[PPX_POWER] - x[PPX_OFFSET1]));
  if (x[PPX_X_ON] != 0.0 && i >= int(x[PPX_START_X]) && i < int(x[PPX_STOP_X])) {
    if (cos(th) < 0.0) ph = ph + M_PI;
  }
  DE = rp * DE * fabs(x[PPX_POWER]) + x[PPX_ADE_OFFSET1];
  rp = rp * r;
  S zth;
  if (x[PPX_D_ON] == 0.0) {
    t = cos(th);
    zth = sin(th);
  } else {
    t = sin(th);
    zth = cos(th);
  }
  if (x[PPX_B_ON] != 0.0 && i >= int(x[PPX_START_B]) && i < int(x[PPX_STOP_B]))
    z.x = (1.0 + (t - 1.0) * x[PPX_SCALE_B0]) * cos(ph);
  else
    z.x = t * cos(ph);
  if (x[PPX_A_ON] != 0.0 && i >= int(x[PPX_START_A]) && i < int(x[PPX_STOP_A]))
    z.y = (1.0 + (t - 1.0) * x[PPX_SCALE_A0]) * sin(ph);
  else
    z.y = t * sin(ph);
  z.z = zth;
  z = z * rp;
  if (x[PPX_BZ] != 0.0) z.y = std::min(z.y, S(x[PPX_OFFSET0] - z.y));
  z.x = z.x + x[PPX_OFFSET000];
  z.y = z.y + x[PPX_OFFSET000 + 1];
  z.z = z.z + x[PPX_OFFSET000 + 2];
  z.w = z.w + 0.0;
  if (i >= int(x[PPX_START_S]) && i < int(x[PPX_STOP_S])) {
    z = z * x[PPX_SCALE_C1];
    DE = DE * fabs(x[PPX_SCALE_C1]);
  }
  if (x[PPX_ADE_ON] != 0.0) DE = DE * x[PPX_ADE_SCALE1] + x[PPX_ADE_OFFSET0];
  if (x[PPX_C_ON] != 0.0) {
    S de0 = len4(z);
    if (de0 > 1.0) de0 = 0.5 * log(de0) * de0 / DE;
    else de0 = 0.0;
    if (x[PPX_E_ON] == 0.0) {
      dist = de0;
    } else {
      if (i >= int(x[PPX_START_E]) && i < int(x[PPX_STOP_E])) dist = std::min(dist, de0);
      else dist = de0;
    }
  }
}

// cFractalDIFSHextgrid2::FormulaCode (fractal_difs_hextgrid2.cpp:30-138)
// without the aux.color terms; scaleA and dist are aux.actualScaleA, aux.dist
template <class S>
inline void formula_difs_hextgrid2(V4<S> &z, const SlotT<S> &f, S &DE, S &scaleA, S &dist, int i) {
  using namespace mbr;
  const double *x = f.x;
  if (x[HGX_SPH_INV] != 0.0 && i >= int(x[HGX_START_X]) && i < int(x[HGX_STOP_1])) {
    z.x = z.x + x[HGX_OFFSET000];
    z.y = z.y + x[HGX_OFFSET000 + 1];
    z.z = z.z + x[HGX_OFFSET000 + 2];
    z.w = z.w + 0.0;
    const S rr = z.x * z.x + z.y * z.y + z.z * z.z + z.w * z.w;
    z = z * S(x[HGX_SCALE_G1] / rr);
    DE = DE * (x[HGX_SCALE_G1] / rr);
    z.x = z.x + (x[HGX_ADD000] - x[HGX_OFFSET000]);
    z.y = z.y + (x[HGX_ADD000 + 1] - x[HGX_OFFSET000 + 1]);
    z.z = z.z + (x[HGX_ADD000 + 2] - x[HGX_OFFSET000 + 2]);
    z.w = z.w + (0.0 - 0.0);
    z = z * x[HGX_SCALE_A1];
    DE = DE * x[HGX_SCALE_A1];
  }
  if (x[HGX_C_ON] != 0.0 && i >= int(x[HGX_START_C]) && i < int(x[HGX_STOP_C1])) {
    double Tp = x[HGX_OFFSET2];
    z.x = S(fmod(val(fabs(z.x) + Tp), 2.0 * Tp)) - Tp;
    Tp = x[HGX_OFFSETA2];
    z.y = S(fmod(val(fabs(z.y) + Tp), 2.0 * Tp)) - Tp;
  }
  if (i >= int(x[HGX_START_S]) && i < int(x[HGX_STOP_S])) {
    const S useScale = scaleA + x[HGX_SCALE2];
    z = z * useScale;
    DE = DE * fabs(useScale);
    if (x[HGX_K_ON] != 0.0 && i >= int(x[HGX_START_K]) && i < int(x[HGX_STOP_K])) {
      const S vary = x[HGX_SCALE_VARY] * (fabs(scaleA) - x[HGX_SCALE_C1]);
      scaleA = scaleA - vary;
    }
  }
  z.x = z.x + x[HGX_OFFSET001];
  z.y = z.y + x[HGX_OFFSET001 + 1];
  z.z = z.z + x[HGX_OFFSET001 + 2];
  z.w = z.w + 0.0;
  if (x[HGX_R_ON] != 0.0 && i >= int(x[HGX_START_R]) && i < int(x[HGX_STOP_R]))
    z = mb_turn(x + HGX_ROT + 1, x[HGX_ROT] != 0.0, false, z);
  if (i >= int(x[HGX_START]) && i < int(x[HGX_STOP])) {
    const double size = x[HGX_SCALE1], cosPi6 = x[HGX_COS6];
    V4<S> zc = z;
    zc.z = zc.z / x[HGX_SCALE_F1];
    const S yFloor = fabs(zc.y - size * S(floor(val(zc.y / size + 0.5))));
    const S xFloor = fabs(zc.x - size * 1.5 / cosPi6 * S(floor(val(zc.x / size / 1.5 * cosPi6 + 0.5))));
    const S gridMax = std::max(yFloor, S(xFloor * cosPi6 + yFloor * x[HGX_SIN6]));
    const S gridMin = std::min(S(gridMax - size * 0.5), yFloor);
    S hexD;
    if (x[HGX_J_ON] == 0.0) hexD = sqrt(gridMin * gridMin + zc.z * zc.z);
    else hexD = std::max(S(fabs(gridMin)), S(fabs(zc.z)));
    hexD = hexD - x[HGX_OFFSET0005];
    dist = std::min(dist, S(hexD / (DE + 1.0)));
  }
}

// Benesi's tetrahedral frame turns (abstract_fractal.h:30-32 constants)
template <class S>
inline V4<S> benesi_in(const V4<S> &z) {
  const double s13 = 0.57735026918962576450914878050196, s12 = 0.70710678118654752440084436210485,
               s23 = 0.81649658092772603273242802490196;
  const S t = z.x * s23 - z.z * s13;
  return V4<S>{(t - z.y) * s12, (t + z.y) * s12, z.x * s13 + z.z * s23, z.w};
}
template <class S>
inline V4<S> benesi_out(const V4<S> &z) {
  const double s13 = 0.57735026918962576450914878050196, s12 = 0.70710678118654752440084436210485,
               s23 = 0.81649658092772603273242802490196;
  const S t = (z.y + z.x) * s12;
  return V4<S>{z.z * s13 + t * s23, (z.y - z.x) * s12, z.z * s23 - t * s13, z.w};
}

// cFractalPseudoKleinianStdDE::FormulaCode (fractal_pseudo_kleinian_std_de.cpp:
// 29-215) without the aux.color terms; dist is aux.dist
template <class S>
inline void formula_pseudo_kleinian_std_de(V4<S> &z, const SlotT<S> &f, S &DE, S &dist, int i) {
  using namespace mbr;
  const double *x = f.x;
  if (x[PSX_P_ON] != 0.0 && i >= int(x[PSX_START_P]) && i < int(x[PSX_STOP_P1])) {
    const double kSqrt34 = 0.86602540378443864676372317075294, kSqrt3 = 1.73205080756887729352744634150587;
    z.y = fabs(z.y);
    z.z = fabs(z.z);
    const S dot1 = (z.x * -kSqrt34 + z.y * 0.5) * x[PSX_SCALE];
    S t = std::max(S(0.0), dot1);
    z.x = z.x - t * -kSqrt3;
    z.y = fabs(z.y - t);
    if (z.y > z.z) std::swap(z.y, z.z);
    z.x = z.x - x[PSX_CM000] * kSqrt34;
    z.y = z.y - x[PSX_CM000 + 1] * 1.5;
    z.z = z.z - x[PSX_CM000 + 2] * 1.5;
    z.w = z.w - 1.0 * 0.0;
    if (z.z > z.x) std::swap(z.z, z.x);
    if (z.x > 0.0) {
      z.y = std::max(S(0.0), z.y);
      z.z = std::max(S(0.0), z.z);
    }
  }
  if (x[PSX_R_ON] != 0.0 && i >= int(x[PSX_START_R]) && i < int(x[PSX_STOP_R]))
    z = mb_turn(x + PSX_ROT + 1, x[PSX_ROT] != 0.0, false, z);
  if (x[PSX_T1_ON] != 0.0 && i >= int(x[PSX_START]) && i < int(x[PSX_STOP_T1])) {
    z = benesi_in(z);
    const S tempL = len4(z);
    z = V4<S>{fabs(z.x) * x[PSX_S222], fabs(z.y) * x[PSX_S222 + 1], fabs(z.z) * x[PSX_S222 + 2], fabs(z.w) * 1.0};
    const S avgScale = len4(z) / tempL;
    DE = DE * avgScale + 1.0;
    z = benesi_out(z);
    z.x = z.x - x[PSX_OFF200];
    z.y = z.y - x[PSX_OFF200 + 1];
    z.z = z.z - x[PSX_OFF200 + 2];
    z.w = z.w - 0.0;
  }
  if (x[PSX_TM_ON] != 0.0 && i >= int(x[PSX_START_D]) && i < int(x[PSX_STOP_TM1])) {
    z = benesi_in(z);
    const S tempL = len4(z);
    z = V4<S>{fabs(z.x) * x[PSX_S333], fabs(z.y) * x[PSX_S333 + 1], fabs(z.z) * x[PSX_S333 + 2], fabs(z.w) * 1.0};
    const S avgScale = len4(z) / tempL;
    DE = DE * avgScale + 1.0;
    z.x = fabs(z.x + x[PSX_ADD111]) - fabs(z.x - x[PSX_ADD111]) - z.x;
    z.y = fabs(z.y + x[PSX_ADD111 + 1]) - fabs(z.y - x[PSX_ADD111 + 1]) - z.y;
    z.z = fabs(z.z + x[PSX_ADD111 + 2]) - fabs(z.z - x[PSX_ADD111 + 2]) - z.z;
    z.w = fabs(z.w + 0.0) - fabs(z.w - 0.0) - z.w;
    z = benesi_out(z);
  }
  if (x[PSX_F_ON] != 0.0 && i >= int(x[PSX_START_F]) && i < int(x[PSX_STOP_F])) {
    S ta = S(0.0), tb = S(0.0);
    if (x[PSX_F_AX] != 0.0) ta = fabs(z.x + x[PSX_OFFF000]);
    if (x[PSX_F_X] != 0.0) tb = fabs(z.x - x[PSX_OFF000]);
    z.x = ta - tb - (z.x * x[PSX_S111]);
    ta = S(0.0);
    tb = S(0.0);
    if (x[PSX_F_AY] != 0.0) ta = fabs(z.y + x[PSX_OFFF000 + 1]);
    if (x[PSX_F_Y] != 0.0) tb = fabs(z.y - x[PSX_OFF000 + 1]);
    z.y = ta - tb - (z.y * x[PSX_S111 + 1]);
    ta = S(0.0);
    tb = S(0.0);
    if (x[PSX_F_AZ] != 0.0) ta = fabs(z.z + x[PSX_OFFF000 + 2]);
    if (x[PSX_F_Z] != 0.0) tb = fabs(z.z - x[PSX_OFF000 + 2]);
    z.z = ta - tb - (z.z * x[PSX_S111 + 2]);
  }
  if (x[PSX_M_ON] != 0.0 && i >= int(x[PSX_START_M]) && i < int(x[PSX_STOP_M])) {
    z = V4<S>{fabs(z.x), fabs(z.y), fabs(z.z), fabs(z.w)};
    if (z.x - z.y < 0.0) std::swap(z.y, z.x);
    if (z.x - z.z < 0.0) std::swap(z.z, z.x);
    if (z.y - z.z < 0.0) std::swap(z.z, z.y);
    z = z * x[PSX_SCALE3];
    z.x = z.x - 2.0 * x[PSX_CMA111];
    z.y = z.y - 2.0 * x[PSX_CMA111 + 1];
    if (z.z > 1.0) z.z = z.z - 2.0 * x[PSX_CMA111 + 2];
    DE = DE * (x[PSX_SCALE3] * x[PSX_SCALE_A1]);
    z.x = z.x + x[PSX_ADD_A000];
    z.y = z.y + x[PSX_ADD_A000 + 1];
    z.z = z.z + x[PSX_ADD_A000 + 2];
    z.w = z.w + 0.0;
  }
  if (x[PSX_FLIP_Z] != 0.0) z.z = -z.z;
  const double cx = x[PSX_CSIZE], cy = x[PSX_CSIZE + 1], cz = x[PSX_CSIZE + 2];
  if (x[PSX_AW] != 0.0 && i >= int(x[PSX_START_C]) && i < int(x[PSX_STOP_C])) {
    V4<S> t = z;
    if (z.x > cx) t.x = cx;
    if (z.x < -cx) t.x = -cx;
    if (z.y > cy) t.y = cy;
    if (z.y < -cy) t.y = -cy;
    if (z.z > cz) t.z = cz;
    if (z.z < -cz) t.z = -cz;
    z = z * x[PSX_SCALE_B1];
    DE = DE * fabs(x[PSX_SCALE_B1]);
    z.x = t.x * 2.0 - z.x;
    z.y = t.y * 2.0 - z.y;
    z.z = t.z * 2.0 - z.z;
    z.w = t.w * 2.0 - z.w;
    const S k = std::max(S(x[PSX_MINR05] / (z.x * z.x + z.y * z.y + z.z * z.z + z.w * z.w)), S(1.0));
    z = z * k;
    DE = DE * (k + x[PSX_TWEAK005]);
  }
  if (x[PSX_AYF] != 0.0 && i >= int(x[PSX_START_B]) && i < int(x[PSX_STOP_B])) {
    if (z.x > cx) z.x = cx * 2.0 - z.x;
    if (z.x < -cx) z.x = -cx * 2.0 - z.x;
    if (z.y > cy) z.y = cy * 2.0 - z.y;
    if (z.y < -cy) z.y = -cy * 2.0 - z.y;
    if (z.z > cz) z.z = cz * 2.0 - z.z;
    if (z.z < -cz) z.z = -cz * 2.0 - z.z;
    const S k = std::max(S(x[PSX_MINR05] / (z.x * z.x + z.y * z.y + z.z * z.z + z.w * z.w)), S(1.0));
    z = z * k;
    DE = DE * (k + x[PSX_TWEAK005]);
  }
  z.x = z.x + x[PSX_ADD000];
  z.y = z.y + x[PSX_ADD000 + 1];
  z.z = z.z + x[PSX_ADD000 + 2];
  z.w = z.w + 0.0;
  dist = sqrt(z.x * z.x + z.y * z.y) / DE;
}

// (x, y, z) in the order of enumMulti_OrderOfXYZ (fractal.h:282-289)
template <class S>
inline V4<S> order_xyz(const V4<S> &v, int order) {
  switch (order) {
    case 1: return V4<S>{v.x, v.z, v.y, v.w};
    case 2: return V4<S>{v.y, v.x, v.z, v.w};
    case 3: return V4<S>{v.y, v.z, v.x, v.w};
    case 4: return V4<S>{v.z, v.x, v.y, v.w};
    case 5: return V4<S>{v.z, v.y, v.x, v.w};
    default: return v;
  }
}

// cFractalAboxMod11::FormulaCode (fractal_abox_mod11.cpp:34-250) without the
// aux.color terms; actualScale and auxC are aux.actualScale and aux.c, c is
// aux.const_c
template <class S>
inline void formula_abox_mod11(V4<S> &z, const SlotT<S> &f, S &DE, S &actualScale, V4<S> &auxC, const V4<S> &c,
                               int i) {
  using namespace mbr;
  const double *x = f.x;
  actualScale = x[ABX_MB_SCALE] + x[ABX_SCALE_VARY] * (fabs(actualScale) - 1.0);
  if (i >= int(x[ABX_START_B]) && i < int(x[ABX_STOP_B])) {
    z.x = fabs(z.x + x[ABX_ADD111]) - fabs(z.x - x[ABX_ADD111]) - z.x;
    z.y = fabs(z.y + x[ABX_ADD111 + 1]) - fabs(z.y - x[ABX_ADD111 + 1]) - z.y;
    if (x[ABX_FOLD_Z] != 0.0) z.z = fabs(z.z + x[ABX_ADD111 + 2]) - fabs(z.z - x[ABX_ADD111 + 2]) - z.z;
  }
  if (x[ABX_FOLD_D] != 0.0 && i >= int(x[ABX_START_D]) && i < int(x[ABX_STOP_D1])) {
    const double limit[3] = {x[ABX_ADD111], x[ABX_ADD111 + 1], x[ABX_ADD111 + 2]};
    S add[3] = {S(0.0), S(0.0), S(0.0)};
    const S zz[3] = {z.x, z.y, z.z};
    for (int a = 0; a < 3; a++) {
      const double length = 2.0 * limit[a];
      const double tgladS = 1.0 / length;
      if (fabs(zz[a]) < limit[a]) add[a] = zz[a] * zz[a] * tgladS;
      if (fabs(zz[a]) > limit[a] && fabs(zz[a]) < length) add[a] = (length - fabs(zz[a])) * (length - fabs(zz[a])) * tgladS;
    }
    for (int a = 0; a < 3; a++) add[a] = add[a] * x[ABX_SCALE3D + a];
    z.x = (z.x - (S(double(sgn(val(z.x)))) * (add[0])));
    z.y = (z.y - (S(double(sgn(val(z.y)))) * (add[1])));
    z.z = (z.z - (S(double(sgn(val(z.z)))) * (add[2])));
  }
  if (x[ABX_SWAP] != 0.0) z = V4<S>{z.z, z.y, z.x, z.w};
  if (i >= int(x[ABX_START_S]) && i < int(x[ABX_STOP_S])) {
    const double para = abox_mod11_para(x, i);
    const S rr = z.x * z.x + z.y * z.y + z.z * z.z + z.w * z.w;
    z.x = z.x + x[ABX_MB_OFFSET];
    z.y = z.y + x[ABX_MB_OFFSET + 1];
    z.z = z.z + x[ABX_MB_OFFSET + 2];
    z.w = z.w + 0.0;
    if (rr < para) {
      const double tglad_factor1 = x[ABX_MAXR2] / para;
      z = z * tglad_factor1;
      DE = DE * tglad_factor1;
    } else if (rr < x[ABX_MAXR2]) {
      const S tglad_factor2 = x[ABX_MAXR2] / rr;
      z = z * tglad_factor2;
      DE = DE * tglad_factor2;
    }
    z.x = z.x - x[ABX_MB_OFFSET];
    z.y = z.y - x[ABX_MB_OFFSET + 1];
    z.z = z.z - x[ABX_MB_OFFSET + 2];
    z.w = z.w - 0.0;
  }
  if (i >= int(x[ABX_START_A]) && i < int(x[ABX_STOP_A])) {
    z = z * actualScale;
    if (x[ABX_ADE_ON] == 0.0) DE = DE * fabs(actualScale) + 1.0;
    else DE = DE * fabs(actualScale) * x[ABX_ADE_SCALE1] + x[ABX_ADE_OFFSET1];
  }
  z.x = z.x + x[ABX_ADD000];
  z.y = z.y + x[ABX_ADD000 + 1];
  z.z = z.z + x[ABX_ADD000 + 2];
  z.w = z.w + 0.0;
  if (x[ABX_ADDC] != 0.0 && i >= int(x[ABX_START_E]) && i < int(x[ABX_STOP_E])) {
    V4<S> t;
    if (x[ABX_ALTERNATE] != 0.0) {
      t = order_xyz(auxC, int(x[ABX_ORDER]));
      auxC = t;
    } else {
      t = order_xyz(c, int(x[ABX_ORDER]));
    }
    z.x = z.x + t.x * x[ABX_CM111];
    z.y = z.y + t.y * x[ABX_CM111 + 1];
    z.z = z.z + t.z * x[ABX_CM111 + 2];
    z.w = z.w + t.w * 1.0;
  }
  if (x[ABX_ROT_ON] != 0.0 && i >= int(x[ABX_START_R]) && i < int(x[ABX_STOP_R]))
    z = mb_turn(x + ABX_ROT + 1, x[ABX_ROT] != 0.0, false, z);
  if (i >= int(x[ABX_START_C]) && i < int(x[ABX_STOP_C1])) {
    z = z * x[ABX_SCALE_G1];
    DE = DE * fabs(x[ABX_SCALE_G1]);
  }
}

// cFractalMengerMod1::FormulaCode (fractal_menger_mod1.cpp:29-103), the
// aux.color terms left out
template <class S>
inline void formula_menger_mod1(V4<S> &z, const SlotT<S> &f, S &DE, int i) {
  using namespace mbr;
  const double *x = f.x;
  z = V4<S>{fabs(z.x), fabs(z.y), fabs(z.z), fabs(z.w)};
  S temp;
  if (z.x < z.y) {
    temp = z.y;
    z.y = z.x;
    z.x = temp;
  }
  if (z.x < z.z) {
    temp = z.z;
    z.z = z.x;
    z.x = temp;
  }
  if (z.y < z.z) {
    temp = z.z;
    z.z = z.y;
    z.y = temp;
  }
  z = z * x[MMX_SCALE3];
  z.x = z.x - 2.0 * x[MMX_CM111];
  z.y = z.y - 2.0 * x[MMX_CM111 + 1];
  if (z.z > 1.0) z.z = z.z - 2.0 * x[MMX_CM111 + 2];
  DE = DE * x[MMX_SCALE3];
  if (x[MMX_ROT_ON] != 0.0 && i >= int(x[MMX_START]) && i < int(x[MMX_STOP])) {
    z = mb_turn(x + MMX_ROT + 1, x[MMX_ROT] != 0.0, false, z);
    DE = DE * x[MMX_SCALED1] + x[MMX_OFFSET1];
  }
  z.x = z.x + x[MMX_ADD000];
  z.y = z.y + x[MMX_ADD000 + 1];
  z.z = z.z + x[MMX_ADD000 + 2];
  z.w = z.w + 0.0;
  if (x[MMX_BOX_OFF] != 0.0 && i >= int(x[MMX_START_A]) && i < int(x[MMX_STOP_A])) {  // box offset :74-89
    const V4<S> t = z;
    z.x = S(double(sgn(val(z.x)))) * x[MMX_ADD_A000] + z.x;
    z.y = S(double(sgn(val(z.y)))) * x[MMX_ADD_A000 + 1] + z.y;
    z.z = S(double(sgn(val(z.z)))) * x[MMX_ADD_A000 + 2] + z.z;
    if (x[MMX_AVG_SCALE] != 0.0) {
      const S tempL = len4(t);
      const S avgScale = len4(z) / tempL;
      DE = DE * avgScale + 1.0;
    }
  }
  if (x[MMX_BLEND] != 0.0) {  // :91-102
    const bool a = i == int(x[MMX_INT_A]), b = i == int(x[MMX_INT_B]);
    const V4<S> zA = a ? z : V4<S>{S(0.0), S(0.0), S(0.0), S(0.0)};
    const V4<S> zB = b ? z : V4<S>{S(0.0), S(0.0), S(0.0), S(0.0)};
    z.x = z.x * x[MMX_SCALE1] + zA.x * x[MMX_OFFSET] + zB.x * x[MMX_OFFSET0];
    z.y = z.y * x[MMX_SCALE1] + zA.y * x[MMX_OFFSET] + zB.y * x[MMX_OFFSET0];
    z.z = z.z * x[MMX_SCALE1] + zA.z * x[MMX_OFFSET] + zB.z * x[MMX_OFFSET0];
    z.w = z.w * x[MMX_SCALE1] + zA.w * x[MMX_OFFSET] + zB.w * x[MMX_OFFSET0];
    DE = DE * x[MMX_SCALE1];
  }
}

// cFractalHypercomplex::FormulaCode (fractal_hypercomplex.cpp:30-45)
template <class S>
inline void formula_hypercomplex(V4<S> &z, const S &r, S &DE) {
  DE = DE * 2.0 * r;
  const S nx = z.x * z.x - z.y * z.y - z.z * z.z - z.w * z.w;
  const S ny = 2.0 * z.x * z.y - 2.0 * z.w * z.z;
  const S nz = 2.0 * z.x * z.z - 2.0 * z.y * z.w;
  const S nw = 2.0 * z.x * z.w - 2.0 * z.y * z.z;
  z.x = nx;
  z.y = ny;
  z.z = nz;
  z.w = nw;
}

// cFractalQuaternion::FormulaCode (fractal_quaternion.cpp:29-39)
template <class S>
inline void formula_quaternion(V4<S> &z, const S &r, S &DE) {
  DE = DE * 2.0 * r;
  const S nx = z.x * z.x - z.y * z.y - z.z * z.z;
  const S ny = 2.0 * z.x * z.y;
  const S nz = 2.0 * z.x * z.z;
  z.x = nx;
  z.y = ny;
  z.z = nz;
}

// cFractalAexion::FormulaCode (fractal_aexion.cpp:29-59); c is aux.const_c,
// replaced at the orbit's first iteration
template <class S>
inline void formula_aexion(V4<S> &z, const S &r, S &DE, const mbr_fractal &p, int i, V4<S> &c) {
  V4<S> temp = z;
  S t;
  if (i == 0) {
    t = p.aexion_cadd;
    temp.x = z.x + z.y + z.z;
    temp.y = -z.x - z.y + z.z;
    temp.z = -z.x + z.y - z.z;
    temp.w = z.x - z.y - z.z;
    z = V4<S>{fabs(temp.x) + t, fabs(temp.y) + t, fabs(temp.z) + t, fabs(temp.w) + t};
    c = z;
  }
  t = 2.0 * z.w * z.z;
  temp.x = z.x * z.x - z.y * z.y;
  temp.y = t - temp.x;
  temp.x = temp.x + t;
  t = 2.0 * z.x * z.y;
  temp.z = z.z * z.z - z.w * z.w;
  temp.w = t - temp.z;
  temp.z = temp.z + t;
  z = V4<S>{temp.x + c.x, temp.y + c.y, temp.z + c.z, temp.w + c.w};
  if (p.analytic_de_enabled) {
    S de1 = 1.1 * r;
    de1 = de1 + (len4(z) / r - de1) * p.analytic_de_scale1;
    DE = de1 * 2.0 * DE + p.analytic_de_offset1;
  }
}

// cFractalKaleidoscopicIfs::FormulaCode (fractal_kaleidoscopic_ifs.cpp:30-85)
template <class S>
inline void formula_ifs(V4<S> &z, const SlotT<S> &f, S &DE) {
  if (f.ifs_abs[0]) z.x = fabs(z.x);
  if (f.ifs_abs[1]) z.y = fabs(z.y);
  if (f.ifs_abs[2]) z.z = fabs(z.z);
  for (int i = 0; i < 9; i++) {
    if (!f.ifs_enabled[i]) continue;
    z = mb_turn(f.ifs_rot[i], f.ifs_rot_zero[i], false, z);
    const double *d = f.ifs_dir[i];
    const S length = z.x * d[0] + z.y * d[1] + z.z * d[2] + z.w * 0.0;  // CVector4::Dot, direction w = 0
    if (length < f.ifs_dist[i]) {
      const S k = 2.0 * (length - f.ifs_dist[i]) * f.ifs_int[i];
      z.x = z.x - d[0] * k;
      z.y = z.y - d[1] * k;
      z.z = z.z - d[2] * k;
      z.w = z.w - 0.0 * k;
    }
  }
  const double *o = f.ifs_offset;
  if (f.ifs_rot_on) {
    V4<S> t{z.x - o[0], z.y - o[1], z.z - o[2], z.w - 0.0};
    t = mb_turn(f.ifs_main, f.ifs_main_zero, false, t);
    z = V4<S>{t.x + o[0], t.y + o[1], t.z + o[2], t.w + 0.0};
  }
  if (f.ifs_edge_on) {
    if (f.ifs_edge[0] > 0.0) z.x = f.ifs_edge[0] - fabs(f.ifs_edge[0] - z.x);
    if (f.ifs_edge[1] > 0.0) z.y = f.ifs_edge[1] - fabs(f.ifs_edge[1] - z.y);
    if (f.ifs_edge[2] > 0.0) z.z = f.ifs_edge[2] - fabs(f.ifs_edge[2] - z.z);
  }
  const double sc = f.ifs_scale;
  z.x = z.x * sc;
  z.y = z.y * sc;
  z.z = z.z * sc;
  z.w = z.w * sc;
  if (f.ifs_menger) {
    z.x = z.x - o[0] * (sc - 1.0);
    z.y = z.y - o[1] * (sc - 1.0);
    if (z.z > 0.5 * o[2] * (sc - 1.0)) z.z = z.z - o[2] * (sc - 1.0);
  } else {
    z.x = z.x - o[0] * (sc - 1.0);
    z.y = z.y - o[1] * (sc - 1.0);
    z.z = z.z - o[2] * (sc - 1.0);
    z.w = z.w - 0.0 * (sc - 1.0);
  }
  DE = DE * fabs(sc);
}

// cFractalMengerSponge::FormulaCode (fractal_menger_sponge.cpp:30-71)
template <class S>
inline void formula_menger(V4<S> &z, const SlotT<S> &f, S &DE) {
  z.x = fabs(z.x); z.y = fabs(z.y); z.z = fabs(z.z); z.w = fabs(z.w);
  S temp;
  if (z.x < z.y) { temp = z.y; z.y = z.x; z.x = temp; }
  if (z.x < z.z) { temp = z.z; z.z = z.x; z.x = temp; }
  if (z.y < z.z) { temp = z.z; z.z = z.y; z.y = temp; }
  z.x = z.x * f.scale3; z.y = z.y * f.scale3; z.z = z.z * f.scale3; z.w = z.w * f.scale3;
  z.x = z.x - 2.0;
  z.y = z.y - 2.0;
  if (z.z > 1.0) z.z = z.z - 2.0;
  DE = DE * f.scale3;
}

// SmoothCVector (common_math.cpp:133-163)
template <class S>
inline V4<S> smooth4(const V4<S> &v1, const V4<S> &v2, double k) {
  if (k <= 0.0) return v1;
  if (k >= 1.0) return v2;
  const double nk = 1.0 - k;
  S l1 = len4(v1), l2 = len4(v2);
  S lenInterp = l1 * nk + l2 * k;
  V4<S> t{v1.x * nk + v2.x * k, v1.y * nk + v2.y * k, v1.z * nk + v2.z * k, v1.w * nk + v2.w * k};
  S lt = len4(t);
  if (lt > 0.0) return V4<S>{t.x / lt * lenInterp, t.y / lt * lenInterp, t.z / lt * lenInterp, t.w / lt * lenInterp};
  return v1;
}

template <class S>
struct FractalOut {
  S distance;
  int iters;
  bool maxiter;
  V4<S> z;  // the orbit's last z (fractOut.z)
};

// Compute<calcModeNormal> (compute_fractal.cpp:67-654), without global
// foldings (sCommonParams::foldings disabled) and colouring modes.
template <class S>
FractalOut<S> compute(const Seq &seq, const SlotT<S> *slots, S px, S py, S pz, int maxiterMultiplier,
                      int forcedMaxiter) {
  FractalOut<S> out;
  V4<S> z{px, py, pz, S(0.0)};
  z.w = S(seq.w0);
  out.maxiter = true;
  V4<S> const_c = z;  // aux.const_c (the Aexion replaces it)
  S r = len4(z);
  S DE = 1.0;
  S pk = 1.0;  // aux.pseudoKleinianDE (:120)
  S scaleA = 0.0;  // aux.actualScaleA (:124)
  // aux.actualScale: the Mandelbox scale of the first sequence slot (:97-98, 123)
  S actualScale = seq.length > 0 ? S(seq.slot[seq.seq[0]].mb_scale) : S(seq.slot[0].mb_scale);
  V4<S> auxC = z;  // aux.c (:107)
  S posNeg = 1.0;  // aux.pos_neg (:109)
  S auxDist = 1000.0;  // aux.dist (:119)
  V4<S> lastZ{S(0.0), S(0.0), S(0.0), S(0.0)}, lastGoodZ = lastZ, lastLastZ = lastZ;
  int maxN = seq.formula_maxiter * maxiterMultiplier;
  if (forcedMaxiter >= 0) maxN = forcedMaxiter;
  int i;
  for (i = 0; i < maxN; i++) {
    lastGoodZ = lastZ;
    lastLastZ = lastZ;
    lastZ = z;
    const int sequence = (i < seq.length) ? seq.seq[i] : seq.seq[0];  // GetSequence
    const Slot &sd = seq.slot[sequence];
    const SlotT<S> &f = slots[sequence];
    if (seq.gbox) {  // BoxFolding (legacy_fractal_transforrms.cpp:43-75), compute_fractal.cpp:192-196
      if (z.x > seq.gbox_limit) z.x = seq.gbox_value - z.x;
      else if (z.x < -seq.gbox_limit) z.x = -seq.gbox_value - z.x;
      if (z.y > seq.gbox_limit) z.y = seq.gbox_value - z.y;
      else if (z.y < -seq.gbox_limit) z.y = -seq.gbox_value - z.y;
      if (z.z > seq.gbox_limit) z.z = seq.gbox_value - z.z;
      else if (z.z < -seq.gbox_limit) z.z = -seq.gbox_value - z.z;
      r = len4(z);
    }
    if (seq.gsph) {  // SphericalFolding (:77-103), compute_fractal.cpp:198-202
      const double fR2_2 = seq.gsph_outer * seq.gsph_outer;
      const double mR2_2 = seq.gsph_inner * seq.gsph_inner;
      const S r2_2 = r * r;
      const double fold_factor1_2 = fR2_2 / mR2_2;
      if (r2_2 < mR2_2) {
        z = z * fold_factor1_2;
        DE = DE * fold_factor1_2;
      } else if (r2_2 < fR2_2) {
        const S fold_factor2_2 = fR2_2 / r2_2;
        z = z * fold_factor2_2;
        DE = DE * fold_factor2_2;
      }
      r = len4(z);
    }
    const V4<S> tempZ = z;
    const S tempAuxDE = DE;
    if (sd.weight > 0.0) {
      switch (sd.formula) {
        case MBR_FORMULA_MANDELBULB: formula_mandelbulb(z, f, r, DE); break;
        case MBR_FORMULA_MANDELBOX: formula_mandelbox(z, f, DE); break;
        case MBR_FORMULA_MENGER_SPONGE: formula_menger(z, f, DE); break;
        case MBR_FORMULA_MANDELBULB_POWER2: formula_bulb_pow2(z, r, DE); break;
        case MBR_FORMULA_HYPERCOMPLEX: formula_hypercomplex(z, r, DE); break;
        case MBR_FORMULA_KALEIDOSCOPIC_IFS: formula_ifs(z, f, DE); break;
        case MBR_FORMULA_XENODREAMBUIE: formula_xenodreambuie(z, f, r, DE); break;
        case MBR_FORMULA_QUATERNION: formula_quaternion(z, r, DE); break;
        case MBR_FORMULA_AEXION: formula_aexion(z, r, DE, sd.ifs, i, const_c); break;
        case MBR_FORMULA_PSEUDO_KLEINIAN: formula_pseudo_kleinian(z, f, DE, pk, i); break;
        case MBR_FORMULA_BOX_FOLD_BULB_POW2: formula_box_fold_bulb_pow2(z, f, r, DE); break;
        case MBR_FORMULA_MENGER_MOD1: formula_menger_mod1(z, f, DE, i); break;
        case MBR_FORMULA_BOX_FOLD_BULB_POW2_V2: formula_box_fold_bulb_pow2_v2(z, f, DE, scaleA, i); break;
        case MBR_FORMULA_ABOX_MOD11: formula_abox_mod11(z, f, DE, actualScale, auxC, const_c, i); break;
        case MBR_FORMULA_PSEUDO_KLEINIAN_MOD4: formula_pseudo_kleinian_mod4(z, f, DE, pk, posNeg, i); break;
        case MBR_FORMULA_PSEUDO_KLEINIAN_STD_DE: formula_pseudo_kleinian_std_de(z, f, DE, auxDist, i); break;
        case MBR_FORMULA_GENERALIZED_FOLD_BOX: formula_generalized_fold_box(z, f, DE); break;
        case MBR_FORMULA_MANDELBULB_PUPUKU: formula_mandelbulb_pupuku(z, f, r, DE, auxDist, i); break;
        case MBR_FORMULA_DIFS_HEXTGRID2: formula_difs_hextgrid2(z, f, DE, scaleA, auxDist, i); break;
        default: {  // :228-238
          out.distance = 10.0;
          out.iters = 1;
          out.maxiter = true;
          out.z = z;
          return out;
        }
      }
    }
    if (sd.add_c) {  // :246-281
      if (seq.julia) {
        z.x = z.x + seq.julia_c[0] * seq.cmul[0];
        z.y = z.y + seq.julia_c[1] * seq.cmul[1];
        z.z = z.z + seq.julia_c[2] * seq.cmul[2];
        z.w = z.w + 0.0;
      } else {
        z.x = z.x + const_c.x * seq.cmul[0];
        z.y = z.y + const_c.y * seq.cmul[1];
        z.z = z.z + const_c.z * seq.cmul[2];
        z.w = z.w + const_c.w;
      }
    }
    if (seq.is_hybrid) {  // :287-297
      const double k = sd.weight;
      if (k < 1.0) {
        z = smooth4(tempZ, z, k);
        const double kn = 1.0 - k;
        DE = DE * k + tempAuxDE * kn;
      }
    }
    r = len4(z);
    if (nan4(z)) {  // :303-309
      z = lastZ;
      r = len4(z);
      out.maxiter = true;
      break;
    }
    if (sd.check_bailout) {  // :312-321
      if (r > sd.bailout) {
        out.maxiter = false;
        break;
      }
      if (sd.add_bail) {  // :323-336
        out.maxiter = false;
        const V4<S> d1{z.x - lastZ.x, z.y - lastZ.y, z.z - lastZ.z, z.w - lastZ.w};
        if (len4(d1) / r < 0.1 / sd.bailout) break;
        const V4<S> d2{z.x - lastLastZ.x, z.y - lastLastZ.y, z.z - lastLastZ.z, z.w - lastLastZ.w};
        if (len4(d2) / r < 0.1 / sd.bailout) break;
      }
    }
    if (nan4(z)) {  // :487-491
      z = lastGoodZ;
      break;
    }
  }
  // final DE :495-621 (aux.dist = 1000 keeps its initial value :119 for
  // every formula restated here; aux.pseudoKleinianDE is pk)
  if (DE > 0.0) {
    if (seq.is_hybrid) {
      switch (seq.de_function) {
        case 1: out.distance = (r - seq.linear_de_offset) / DE; break;
        case 2: out.distance = (r > 1.0) ? S(0.5 * r * log(r) / DE) : S(0.0); break;
        case 3: {
          const S rxy = sqrt(z.x * z.x + z.y * z.y);
          out.distance = std::max(S(rxy - pk), S(fabs(rxy * z.z) / r)) / DE;
          break;
        }
        case 5: out.distance = auxDist; break;
        case 6: out.distance = std::max(fabs(z.x), std::max(fabs(z.y), fabs(z.z))) / DE; break;
        default: out.distance = 0.0; break;
      }
    } else {
      switch (seq.de_analytic) {
        case 2: out.distance = (r > 1.0) ? S(0.5 * r * log(r) / DE) : S(0.0); break;
        case 1: out.distance = r / DE; break;
        case 3: out.distance = (r - 2.0) / DE; break;
        case 4: {
          const S rxy = sqrt(z.x * z.x + z.y * z.y);
          out.distance = std::max(S(rxy - pk), S(fabs(rxy * z.z) / r)) / DE;
          break;
        }
        case 6: out.distance = auxDist; break;
        case 7: out.distance = std::max(fabs(z.x), std::max(fabs(z.y), fabs(z.z))) / DE; break;
        case 0: out.distance = -1.0; break;
        default: out.distance = r; break;
      }
    }
  } else {
    out.distance = r;
  }
  out.iters = i + 1;
  out.z = z;
  return out;
}

// The gradient model of a non-escaping orbit (a point inside the set): its
// distance estimate is ~0 and, to first order, constant - its exact
// derivative through 50+ chaotic iterations is noise.  No-op for plain values.
template <class S>
inline void zero_tangents(S &) {}
template <int N>
inline void zero_tangents(Dual<N> &d) {
  for (int i = 0; i < N; i++) d.d[i] = 0.0;
}

// CalculateDistanceSimple, delta-DE branch (calculate_distance.cpp:607-760):
// the orbit radius |z| (3-D) at the point and at three points offset by
// deltaDE along x, y and z, the offset orbits capped at the first orbit's
// iteration count (forcedMaxiter), the DE function of the sequence applied to
// the radius and the gradient of |z|.  *iters_out: the first orbit's count;
// *total_iters (when given): all four.
static double delta_distance(const Seq &seq, const SlotT<double> *slots, double px, double py, double pz,
                             double detailSize, bool normalMode, int mult, int *iters_out, int *total_iters = nullptr) {
  const double plen = sqrt(px * px + py * py + pz * pz);
  const double deltaDE = std::max(plen * 1e-14, seq.delta_factor * detailSize);
  // Compute's delta-mode ending for the Jos Kleinian function
  // (compute_fractal.cpp:627-638): z.y = min(z.y, foldingValue - z.y) with
  // the default transf_spheres_enabled (true) and transf_folding_value (2)
  auto jos_fold = [&](FractalOut<double> &f) {
    if (seq.de_function == 4) f.z.y = std::min(f.z.y, 2.0 - f.z.y);
  };
  FractalOut<double> fo = compute<double>(seq, slots, px, py, pz, mult, -1);
  jos_fold(fo);
  const V4<double> zFromIters = fo.z;
  const double r = sqrt(fo.z.x * fo.z.x + fo.z.y * fo.z.y + fo.z.z * fo.z.z);
  bool out_maxiter = fo.maxiter;
  bool maxiter = fo.maxiter;
  const int iters1 = fo.iters;
  int total = fo.iters;
  if (!seq.limits) {
    if (!seq.iter_thresh) maxiter = false;
  } else {
    if (normalMode) maxiter = false;
  }
  double drv[3];
  for (int a = 0; a < 3; a++) {
    fo = compute<double>(seq, slots, px + (a == 0 ? deltaDE : 0.0), py + (a == 1 ? deltaDE : 0.0),
                         pz + (a == 2 ? deltaDE : 0.0), mult, iters1);
    jos_fold(fo);
    const double r2 = sqrt(fo.z.x * fo.z.x + fo.z.y * fo.z.y + fo.z.z * fo.z.z);
    drv[a] = fabs(r2 - r) / deltaDE;
    total += fo.iters;
  }
  const double dr = sqrt(drv[0] * drv[0] + drv[1] * drv[1] + drv[2] * drv[2]);
  double distance = 0.0;
  if (dr > 0) {
    const V4<double> &z = fo.z;  // the last offset orbit (:686-698)
    switch (seq.de_function) {
      case 1: distance = 0.5 * r / dr; break;
      case 2: distance = 0.5 * r * log(r) / dr; break;
      case 3: {
        const double rxy = sqrt(z.x * z.x + z.y * z.y);
        distance = std::max(rxy - 0.92784, fabs(rxy * z.z) / r) / dr;
        break;
      }
      case 4: {
        const double rxy = sqrt(z.x * z.x + z.z * z.z);
        distance = (fabs(rxy * z.y) / r) / dr;
        maxiter = false;
        break;
      }
      case 5: distance = r; break;
      case 6: {  // dMax (common_math.cpp:74-83)
        auto dmax3 = [](double a, double b, double c) { return (a > b) ? ((a > c) ? a : c) : ((b > c) ? b : c); };
        const double maxZ = dmax3(fabs(zFromIters.x), fabs(zFromIters.y), fabs(zFromIters.z));
        const double maxDr = dmax3(fabs(drv[0]), fabs(drv[1]), fabs(drv[2]));
        distance = 0.5 * maxZ / maxDr;
        break;
      }
      default: break;
    }
  } else {
    distance = r;
  }
  if (!seq.iter_thresh) out_maxiter = false;
  if (normalMode) out_maxiter = false;
  if (out_maxiter) distance = 0.0;
  if (fo.iters < seq.min_n && distance < detailSize) distance = detailSize;  // the last offset orbit's count
  if (seq.interior && !normalMode) {
    if (distance < 0.5 * detailSize || maxiter) distance = detailSize;
  } else if (seq.interior && normalMode) {
    if (distance < 0.9 * detailSize) distance = detailSize - distance;
  }
  if (seq.iter_thresh && !normalMode && !maxiter) {
    if (distance < detailSize) distance = detailSize * 1.01;
  }
  if (distance < 0.0) distance = 0.0;
  if (distance > 10.0) distance = 10.0;
  if (iters_out) *iters_out = iters1;
  if (total_iters) *total_iters = total;
  return distance;
}

// CalculateDistanceSimple (calculate_distance.cpp:533-760): the delta branch
// (FP64) or the analytic branch, with its post-processing.
template <class S>
S calc_distance_simple(const Seq &seq, const SlotT<S> *slots, S px, S py, S pz, double detailSize, bool normalMode,
                       int *iters_out, int *total_out) {
  const int mult = (normalMode && seq.iter_thresh) ? 5 : 1;
  if constexpr (std::is_same<S, double>::value) {
    if (seq.delta_de) return delta_distance(seq, slots, px, py, pz, detailSize, normalMode, mult, iters_out, total_out);
  }
  FractalOut<S> fo = compute<S>(seq, slots, px, py, pz, mult, -1);
  S distance = fo.distance;
  if (fo.maxiter) zero_tangents(distance);
  bool maxiter = fo.maxiter;
  if (iters_out) *iters_out = fo.iters;
  if (total_out) *total_out = fo.iters;
  if (!seq.iter_thresh) maxiter = false;
  if (normalMode) maxiter = false;
  if (maxiter) distance = 0.0;
  if (fo.iters < seq.min_n && distance < detailSize) distance = detailSize;
  if (seq.interior && !normalMode) {
    if (distance < 0.5 * detailSize || fo.maxiter) distance = detailSize;
  } else if (seq.interior && normalMode) {
    if (distance < 0.9 * detailSize) distance = detailSize - distance;
  }
  if (seq.iter_thresh && !normalMode && !fo.maxiter) {
    if (distance < detailSize) distance = detailSize * 1.01;
  }
  if (distance < 0.0) distance = 0.0;
  if (distance > 10.0) distance = 10.0;
  return distance;
}

// One node of an explicit objects tree as the walk reads it
// (cObjectsTree::sNodeDataForRendering, objects_tree.h:50-80): the world-to-
// local matrix of its accumulated transform, its scale and repeat, and for a
// fractal node its own sequence (the scene's general settings with the
// node's slot, iteration limit, julia and constant factor).
struct ONode {
  int type = 0, level = 0;
  double w2l[12] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0};
  double abs_scale = 1.0, detail_mult = 1.0, smooth_dist = 0.1;
  double repeat[3] = {0, 0, 0};  // repeat / absScale
  bool smooth = false;
  OPrim prim;                    // PRIMITIVE: its world transform, repeat and scale
  std::shared_ptr<Seq> seq;      // FRACTAL
  std::vector<SlotT<double>> slots;
};
struct OTree {
  std::vector<ONode> nodes;
};

// cObjectsTree::GetNodeDataListForRendering (objects_tree.cpp:185-410) for
// the listed nodes: a disabled node drops its subtree, every node's world
// matrix is its parent's times its own, and a fractal node's sequence is
// built from the scene with that node's slot and settings.
static bool build_tree(const mbr_scene &sc, Seq *s) {
  if (sc.n_nodes <= 0) return true;
  if (sc.n_nodes > MBR_MAX_NODES || sc.hybrid_fractal_enable) return false;
  auto tree = std::make_shared<OTree>();
  double Wl[12][4][4];
  static const double I[4][4] = {{1, 0, 0, 0}, {0, 1, 0, 0}, {0, 0, 1, 0}, {0, 0, 0, 1}};
  int skip = -1, prev_level = -1, prev_type = 0;
  for (int i = 0; i < sc.n_nodes; i++) {
    const mbr_node &n = sc.node[i];
    const bool group = n.type == MBR_NODE_BOOLEAN_ADD || n.type == MBR_NODE_BOOLEAN_MUL || n.type == MBR_NODE_BOOLEAN_SUB;
    if (n.level < 0 || n.level > 8 || n.level > prev_level + 1) return false;
    if (n.level == prev_level + 1 && i > 0 && prev_type != 1) return false;  // only a group has children
    prev_level = n.level;
    prev_type = group ? 1 : 0;
    if (skip >= 0 && n.level > skip) continue;
    skip = -1;
    if (!n.enabled) {
      skip = n.level;
      continue;
    }
    ONode nd;
    nd.type = n.type;
    nd.level = n.level;
    nd.detail_mult = n.detail_level_multiplier;
    nd.smooth = n.smooth_combine != 0;
    nd.smooth_dist = n.smooth_combine_distance;
    const double(*P)[4] = (n.level == 0) ? I : Wl[n.level - 1];
    const mbr_primitive *q = nullptr;
    if (n.type == MBR_NODE_PRIMITIVE) {
      if (n.index < 0 || n.index >= sc.n_primitives) return false;
      q = &sc.primitive[n.index];
      node_world(P, q->position, q->rotation, q->scale, Wl[n.level]);
    } else {
      node_world(P, n.position, n.rotation, n.scale, Wl[n.level]);
    }
    inverse_affine(Wl[n.level], nd.w2l, &nd.abs_scale);
    const double *rep = q ? q->repeat : n.repeat;
    for (int k = 0; k < 3; k++) nd.repeat[k] = rep[k] / nd.abs_scale;
    if (n.type == MBR_NODE_FRACTAL) {
      if (n.index < 0 || n.index >= MBR_MAX_FRACTALS) return false;
      mbr_scene t = sc;
      t.n_nodes = 0;
      t.n_primitives = 0;
      t.hybrid_fractal_enable = 0;
      t.n_fractals = 1;
      t.fractal[0] = sc.fractal[n.index];
      t.formula_maxiter = n.formula_maxiter;
      t.julia_mode = n.julia_mode;
      for (int k = 0; k < 3; k++) {
        t.julia_c[k] = n.julia_c[k];
        t.fractal_constant_factor[k] = n.fractal_constant_factor[k];
      }
      t.initial_waxis = n.initial_waxis;
      auto seq = std::make_shared<Seq>();
      if (!build_sequence(t, seq.get())) return false;
      nd.seq = seq;
      nd.slots.push_back(make_slot<double>(seq->slot[0], false));
    } else if (n.type == MBR_NODE_PRIMITIVE) {
      nd.prim.q = *q;
      for (int k = 0; k < 12; k++) nd.prim.w2l[k] = nd.w2l[k];
      nd.prim.abs_scale = nd.abs_scale;
      for (int k = 0; k < 3; k++) nd.prim.repeat[k] = nd.repeat[k];
    } else if (!group) {
      return false;
    }
    tree->nodes.push_back(nd);
  }
  s->tree = tree;
  return true;
}

// mergeChildIntoParent (calculate_distance.cpp:103-204) on the distance and
// the smooth-combine settings (the closest-object bookkeeping is for shading)
struct OFrame {
  double dist = 1e20, detail = 0.0, smooth_dist = 0.1;
  int level = 0, type = MBR_NODE_BOOLEAN_ADD;
  bool smooth = false;
};
static void merge_child(const OFrame &child, OFrame *parent) {
  const double cd = child.dist;
  switch (parent->type) {
    case MBR_NODE_BOOLEAN_MUL:
      if (cd > parent->dist) parent->dist = cd;
      break;
    case MBR_NODE_BOOLEAN_SUB:
      if (parent->dist >= 1e19) {
        parent->dist = cd;
      } else if (parent->detail > 0 && cd < parent->detail) {
        const double limitDist = parent->detail * 1.5;
        if (cd < limitDist) {
          parent->dist = limitDist;
        } else {
          const double adjusted = std::max(limitDist - cd, parent->dist);
          parent->dist = (adjusted < 0) ? 0 : adjusted;
        }
      }
      break;
    default:
      if (child.smooth && parent->dist < 1e19) {  // opSmoothUnion (math_utilities.h:99-103)
        const double k = child.smooth_dist, d1 = cd, d2 = parent->dist;
        const double t = 0.5 + 0.5 * (d2 - d1) / k;
        const double h = (t < 0.0) ? 0.0 : ((t > 1.0) ? 1.0 : t);
        parent->dist = (d2 * (1.0 - h) + d1 * h) - k * h * (1.0 - h);
      } else if (cd < parent->dist) {
        parent->dist = cd;
      }
      break;
  }
}

// CalculateDistanceFromObjectsTree (calculate_distance.cpp:225-516) over an
// explicit tree: each enabled node's world-to-local transform, repeat in its
// own frame and detail size / (absScale * detail multiplier), boolean groups
// on a stack of at most 10 levels.  iters: the leaves' iterations summed.
static double tree_distance(const Seq &seq, double px, double py, double pz, double detailSize, bool normalMode,
                            int *iters_out, int *total_out) {
  OFrame st[10];
  st[0].dist = 1e20;
  st[0].level = 0;
  st[0].type = MBR_NODE_BOOLEAN_ADD;
  st[0].detail = detailSize;
  int sl = 0, total_iters = 0, total_all = 0;
  for (const ONode &nd : seq.tree->nodes) {
    const double *m = nd.w2l;
    double lx = m[0] * px + m[1] * py + m[2] * pz + m[3];
    double ly = m[4] * px + m[5] * py + m[6] * pz + m[7];
    double lz = m[8] * px + m[9] * py + m[10] * pz + m[11];
    if (sqrt(nd.repeat[0] * nd.repeat[0] + nd.repeat[1] * nd.repeat[1] + nd.repeat[2] * nd.repeat[2]) > 0.0) {
      lx = repeat_mod(lx, nd.repeat[0]);
      ly = repeat_mod(ly, nd.repeat[1]);
      lz = repeat_mod(lz, nd.repeat[2]);
    }
    double nodeDetail;
    if (nd.abs_scale > 0.0 && nd.detail_mult > 0.0) nodeDetail = detailSize / nd.abs_scale / nd.detail_mult;
    else if (nd.abs_scale > 0.0) nodeDetail = detailSize / nd.abs_scale;
    else if (nd.detail_mult > 0.0) nodeDetail = detailSize / nd.detail_mult;
    else nodeDetail = detailSize;
    if (nd.level < sl) {
      while (sl > nd.level) {
        const OFrame child = st[sl];
        sl--;
        merge_child(child, &st[sl]);
      }
    }
    double distance = 1e20;
    int leafIters = 0, leafTotal = 0;
    if (nd.type == MBR_NODE_FRACTAL) {
      distance = calc_distance_simple<double>(*nd.seq, nd.slots.data(), lx, ly, lz, nodeDetail, normalMode,
                                              &leafIters, &leafTotal);
      distance *= nd.abs_scale;
    } else if (nd.type == MBR_NODE_PRIMITIVE) {
      distance = prim_distance(nd.prim, px, py, pz);
    } else {
      sl++;
      st[sl].dist = (nd.type == MBR_NODE_BOOLEAN_MUL) ? -1e20 : 1e20;
      st[sl].level = nd.level;
      st[sl].type = nd.type;
      st[sl].detail = nodeDetail;
      st[sl].smooth = nd.smooth;
      st[sl].smooth_dist = nd.smooth_dist;
      continue;
    }
    OFrame leaf;
    leaf.dist = distance;
    leaf.detail = nodeDetail;
    leaf.smooth = nd.smooth;
    leaf.smooth_dist = nd.smooth_dist;
    merge_child(leaf, &st[sl]);
    total_iters += leafIters;
    total_all += leafTotal;
  }
  while (sl > 0) {
    const OFrame child = st[sl];
    sl--;
    merge_child(child, &st[sl]);
  }
  if (iters_out) *iters_out = total_iters;
  if (total_out) *total_out = total_all;
  return st[0].dist;
}

// CalculateDistance: the limit box early-out, then the objects tree - the
// explicit one, or the default (the fractal node, identity transform, and
// the primitives joined by union, calculate_distance.cpp:166-201).
template <class S>
S calc_distance(const Seq &seq, const SlotT<S> *slots, S px, S py, S pz, double detailSize, bool normalMode,
                int *iters_out, int *total_out = nullptr) {
  if (seq.limits) {  // the limit box early-out (calculate_distance.cpp:261-275)
    S bx = std::max(px - seq.lim_max[0], -(px - seq.lim_min[0]));
    S by = std::max(py - seq.lim_max[1], -(py - seq.lim_min[1]));
    S bz = std::max(pz - seq.lim_max[2], -(pz - seq.lim_min[2]));
    S limitBoxDist = std::max({bx, by, bz});
    if (limitBoxDist > detailSize) {
      if (iters_out) *iters_out = 0;  // the reference leaves out->iters unset here
      if (total_out) *total_out = 0;
      return limitBoxDist;
    }
  }
  if constexpr (std::is_same<S, double>::value) {
    if (seq.tree) return tree_distance(seq, px, py, pz, detailSize, normalMode, iters_out, total_out);
  }
  S distance = calc_distance_simple<S>(seq, slots, px, py, pz, detailSize, normalMode, iters_out, total_out);
  if constexpr (std::is_same<S, double>::value) {  // booleanAdd with the primitives (calculate_distance.cpp:166-201)
    for (const OPrim &op : seq.prims) {
      const double pd = prim_distance(op, px, py, pz);
      if (pd < distance) distance = pd;
    }
  }
  return distance;
}

// ============================================================================
// Camera: cCameraTarget::SetCameraTargetTop (camera_target.cpp:86-130) and
// cRenderWorker::PrepareMainVectors (render_worker.cpp:539-564).
// ============================================================================
struct D3 {
  double x, y, z;
};
static inline D3 add(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
static inline D3 sub(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
static inline D3 mul(D3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
static inline double dot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline double length(D3 a) { return sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
static inline D3 cross(D3 a, D3 v) {  // algebra.hpp:188-195
  return {a.y * v.z - a.z * v.y, -a.x * v.z + a.z * v.x, a.x * v.y - a.y * v.x};
}
static inline D3 normalize(D3 a) {  // algebra.hpp:204-211
  const double n = 1.0 / length(a);
  return {a.x * n, a.y * n, a.z * n};
}
static D3 rotate_around(D3 v, D3 axis, double angle) {  // algebra.cpp:70-76
  D3 r = mul(v, cos(angle));
  r = add(r, mul(cross(axis, v), sin(angle)));
  r = add(r, mul(mul(axis, dot(axis, v)), 1 - cos(angle)));
  return r;
}
static double correct_angle(double a) { return fmod(a + 3 * M_PI, 2 * M_PI) - M_PI; }  // camera_target.hpp:62

struct Mat3 {
  double m[9];  // row-major m11 m12 m13 / m21 ...
  bool zero;
};
static void mat_mul(const double *a, const double *b, double *r) {  // algebra.cpp:152-166
  double t[9];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++)
      t[i * 3 + j] = a[i * 3 + 0] * b[0 * 3 + j] + a[i * 3 + 1] * b[1 * 3 + j] + a[i * 3 + 2] * b[2 * 3 + j];
  std::memcpy(r, t, sizeof(t));
}
static void rot_axis(Mat3 &M, int axis, double angle) {  // algebra.cpp:198-247
  if (angle == 0.0) return;
  double r[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  const double s = sin(angle), c = cos(angle);
  if (axis == 0) { r[0] = 1.0; r[4] = c; r[8] = c; r[5] = -s; r[7] = s; }
  if (axis == 1) { r[4] = 1.0; r[8] = c; r[0] = c; r[6] = -s; r[2] = s; }
  if (axis == 2) { r[8] = 1.0; r[0] = c; r[4] = c; r[1] = -s; r[3] = s; }
  mat_mul(M.m, r, M.m);
  M.zero = false;
}
static D3 rotate(const Mat3 &M, D3 v) {  // algebra.cpp:320-331, :168-175
  if (M.zero) return v;
  const double *m = M.m;
  return {m[0] * v.x + m[1] * v.y + m[2] * v.z, m[3] * v.x + m[4] * v.y + m[5] * v.z,
          m[6] * v.x + m[7] * v.y + m[8] * v.z};
}

static void camera_setup(const mbr_camera &cam, Mat3 *M, double angles[3]) {
  double yaw, pitch, roll;
  if (cam.use_angles) {
    yaw = cam.angles[0];
    pitch = cam.angles[1];
    roll = cam.angles[2];
  } else {
    const D3 c{cam.camera[0], cam.camera[1], cam.camera[2]};
    const D3 t{cam.target[0], cam.target[1], cam.target[2]};
    D3 fwd = (c.x == t.x && c.y == t.y && c.z == t.z) ? D3{0.0, 1.0, 0.0} : sub(t, c);
    fwd = normalize(fwd);
    yaw = atan2(fwd.y, fwd.x) - 0.5 * M_PI;                       // GetAlpha
    pitch = atan2(fwd.z, sqrt(fwd.x * fwd.x + fwd.y * fwd.y));   // GetBeta
    D3 top = normalize(D3{cam.top[0], cam.top[1], cam.top[2]});
    top = rotate_around(top, D3{0.0, 0.0, 1.0}, -yaw);
    top = rotate_around(top, D3{1.0, 0.0, 0.0}, -pitch);
    roll = -atan2(top.z, top.x) + 0.5 * M_PI;
    yaw = correct_angle(yaw);
    pitch = correct_angle(pitch);
    roll = correct_angle(roll);
  }
  Mat3 m;
  for (int i = 0; i < 9; i++) m.m[i] = (i % 4 == 0) ? 1.0 : 0.0;
  m.zero = true;
  rot_axis(m, 2, yaw);
  rot_axis(m, 0, pitch);
  rot_axis(m, 1, roll);
  *M = m;
  angles[0] = yaw;
  angles[1] = pitch;
  angles[2] = roll;
}

// ============================================================================
// Random streams.
// ============================================================================
// Park-Miller without divisions (common_math.cpp:47-72), one state per ray.
struct ParkMiller {
  unsigned int s;
  int next() {
    unsigned int lo = 16807 * (s & 0xFFFF);
    unsigned int hi = 16807 * (s >> 16);
    lo += (hi & 0x7FFF) << 16;
    hi >>= 15;
    lo += hi;
    if (lo > 2147483647) lo -= 2147483647;
    return int(s = lo);
  }
  int random(int max) { return next() % (max + 1); }
};
// Per-ray seeding: a multiplicative hash of (ray, seed) into [1, 2^31-2],
// then ten warm-up draws (the OpenCL engine warms its per-pixel seed the same
// way, full_engine.cl:58-64).
static ParkMiller pm_for_ray(uint64_t ray, uint32_t seed) {
  uint64_t h = (ray + 1) * 0x9E3779B97F4A7C15ull ^ (uint64_t(seed) * 0xC2B2AE3D27D4EB4Full);
  h ^= h >> 29;
  ParkMiller pm;
  pm.s = uint32_t(h % 2147483646ull) + 1u;
  for (int i = 0; i < 10; i++) pm.next();
  return pm;
}

// PCG32 (O'Neill 2014, pcg32_srandom_r / pcg32_random_r; XSH-RR output).
struct Pcg32 {
  uint64_t state, inc;
  uint32_t next() {
    uint64_t old = state;
    state = old * 6364136223846793005ull + inc;
    uint32_t xorshifted = uint32_t(((old >> 18u) ^ old) >> 27u);
    uint32_t rot = uint32_t(old >> 59u);
    return (xorshifted >> rot) | (xorshifted << ((-rot) & 31));
  }
  double uniform() { return double(next() >> 8) * (1.0 / 16777216.0); }  // [0,1), 24 bits
};
static Pcg32 pcg_init(uint64_t initstate, uint64_t initseq) {
  Pcg32 p;
  p.state = 0u;
  p.inc = (initseq << 1u) | 1u;
  p.next();
  p.state += initstate;
  p.next();
  return p;
}

// Cosine-weighted direction about n (Malley's method), orthonormal basis by
// Duff et al., "Building an Orthonormal Basis, Revisited" (JCGT 2017).
static D3 cosine_dir(D3 n, double u1, double u2) {
  const double r = sqrt(u1);
  const double phi = 2.0 * M_PI * u2;
  const double lx = r * cos(phi), ly = r * sin(phi);
  const double lz = sqrt(std::max(0.0, 1.0 - u1));
  const double sign = n.z >= 0.0 ? 1.0 : -1.0;
  const double a = -1.0 / (sign + n.z);
  const double b = n.x * n.y * a;
  const D3 t{1.0 + sign * n.x * n.x * a, sign * b, -sign * n.x};
  const D3 bb{b, sign + n.y * n.y * a, -n.y};
  return {t.x * lx + bb.x * ly + n.x * lz, t.y * lx + bb.y * ly + n.y * lz, t.z * lx + bb.z * ly + n.z * lz};
}

// ============================================================================
// Render state shared by the pixel pipeline.
// ============================================================================
struct Counters {
  uint64_t de = 0, iters = 0, march = 0, binary = 0, normal = 0, shadow = 0, ao = 0, gi = 0, pixels = 0, watchdog = 0;
};

// CalcFOV (projection_3d.cpp:140-159)
inline double calc_fov(const mbr_camera &c) {
  if (c.perspective_type == MBR_PROJECTION_THREE_POINT) return 2.0 * tan(c.fov_deg / 360.0 * M_PI);
  return c.fov_deg / 180.0 * M_PI;
}

struct Renderer {
  Seq seq;
  std::vector<SlotT<double>> slots;
  mbr_render_params p;
  mbr_camera cam;
  Mat3 M;
  D3 camera;
  double fov, resolution, aspect;
  D3 light;
  std::vector<int> gamma;
  bool want_normal = false;

  double de(D3 q, double detail, bool normalMode, int *iters, Counters &c) const {
    int it = 0, total = 0;
    double d = calc_distance<double>(seq, slots.data(), q.x, q.y, q.z, detail, normalMode, &it, &total);
    c.de++;
    c.iters += total;
    if (iters) *iters = it;
    return d;
  }
  // CalcDistThresh (render_worker.cpp:653-679), reduceDetail = 1
  double dist_thresh(D3 q) const {
    double distThresh;
    if (seq.iter_thresh) {
      distThresh = length(sub(camera, q)) * resolution * fov;
    } else {
      if (p.constant_de_threshold)
        distThresh = p.de_thresh;
      else
        distThresh = length(sub(camera, q)) * resolution * fov / p.detail_level;
    }
    if (cam.perspective_type == MBR_PROJECTION_EQUIRECTANGULAR) distThresh *= 0.5;  // :669
    if (p.advanced_quality) {  // :671-675
      if (distThresh > p.detail_size_max) distThresh = p.detail_size_max;
      if (distThresh < p.detail_size_min) distThresh = p.detail_size_min;
    }
    return distThresh;
  }
  double calc_delta(D3 q) const {  // :684-690
    double delta = length(sub(camera, q)) * resolution * fov;
    if (cam.perspective_type == MBR_PROJECTION_EQUIRECTANGULAR) delta *= 0.5f;
    return delta;
  }

  struct March {
    bool found = false;
    double depth = 0, dist = 0, thr = 0;
    D3 point{0, 0, 0};
    int iters = 0;
    double prev_scan = 0;
  };

  // RayMarching (render_worker.cpp:708-951), minScan = 0, invertMode off.
  March ray_marching(D3 start, D3 dir, double maxScan, ParkMiller &pm, Counters &c) const {
    March o;
    D3 point{1e30, 1e30, 1e30};
    bool found = false, dead = false;
    double scan = 0.0, dist = 0.0, step = 0.0, distThresh = 0.0, prevScan = 0.0;
    const double search_accuracy = 0.001 * p.detail_level;
    const double search_limit = 1.0 - search_accuracy;
    int iters = 0;
    const double dirLen = length(dir);
    for (int i = 0; i < p.max_raymarching_steps; i++) {
      D3 lastPoint = point;
      point = add(start, mul(dir, scan));
      if ((point.x == lastPoint.x && point.y == lastPoint.y && point.z == lastPoint.z) ||
          !(isfinite(point.x) && isfinite(point.y) && isfinite(point.z))) {
        found = true;
        dead = true;
        break;
      }
      distThresh = dist_thresh(point);
      dist = de(point, distThresh, false, &iters, c);
      c.march++;
      if (dist < distThresh) {
        found = true;
        break;
      }
      const double jit = p.jitter ? (1.0 - pm.random(1000) / 10000.0) : 1.0;
      if (seq.interior)
        step = (dist - 0.8 * distThresh) * p.de_factor * jit;
      else
        step = (dist - 0.5 * distThresh) * p.de_factor * jit;
      if (p.advanced_quality) {  // :819-834
        if (step > p.abs_max_marching_step) step = p.abs_max_marching_step;
        if (step < p.abs_min_marching_step) step = p.abs_min_marching_step;
        if (distThresh > p.abs_min_marching_step) {
          if (step > p.rel_max_marching_step * distThresh) step = p.rel_max_marching_step * distThresh;
        }
        if (step < p.rel_min_marching_step * distThresh) step = p.rel_min_marching_step * distThresh;
      } else {
        if (step > 3.0) step = 3.0;
      }
      prevScan = scan;
      scan += step / dirLen;
      if (scan > maxScan) break;
    }
    point = add(start, mul(dir, scan));
    if (found && !dead) {
      if (p.refine == MBR_REFINE_ROOT) {
        // Bisection of F(t) = dist - thr on [previous scan, hit scan].
        double lo = prevScan, hi = scan;
        if (hi > lo) {
          for (int i = 0; i < p.binary_steps; i++) {
            const double mid = 0.5 * (lo + hi);
            if (mid <= lo || mid >= hi) break;
            const D3 q = add(start, mul(dir, mid));
            const double thr = dist_thresh(q);
            const double d = de(q, thr, false, &iters, c);
            c.binary++;
            if (d < thr) hi = mid; else lo = mid;
          }
          scan = hi;
          point = add(start, mul(dir, scan));
          distThresh = dist_thresh(point);
          dist = de(point, distThresh, false, &iters, c);
          c.binary++;
        }
      } else {
        step *= 0.5;
        for (int i = 0; i < p.binary_steps; i++) {
          if (dist < distThresh && dist > distThresh * search_limit) break;
          if (dist > distThresh) {
            scan += step;
            point = add(start, mul(dir, scan));
          } else if (dist < distThresh * search_limit) {
            scan -= step;
            point = add(start, mul(dir, scan));
          }
          distThresh = dist_thresh(point);
          dist = de(point, distThresh, false, &iters, c);
          c.binary++;
          step *= 0.5;
        }
      }
    }
    if (seq.iter_thresh) {  // :917-939
      scan -= distThresh;
      point = add(start, mul(dir, scan));
      if (found) {
        dist = de(point, distThresh, false, &iters, c);
        c.binary++;
      }
    }
    o.found = found;
    o.dist = dist;
    o.depth = scan;
    o.thr = distThresh;
    o.point = point;
    o.iters = iters;
    o.prev_scan = prevScan;
    return o;
  }

  // CalculateNormals fast path (shader_calculate_normals.cpp:40-125)
  D3 normals(D3 q, double thr, Counters &c, uint64_t *counter) const {
    if (p.slow_shading) {  // shader_calculate_normals.cpp:83-106
      double delta = calc_delta(q) * p.smoothness;
      if (seq.interior) delta = thr * 0.2 * p.smoothness;
      D3 n{0.0, 0.0, 0.0};
      for (double px = -1.0; px <= 1.0; px += 0.2)
        for (double py = -1.0; py <= 1.0; py += 0.2)
          for (double pz = -1.0; pz <= 1.0; pz += 0.2) {
            const D3 p3{q.x + px * delta, q.y + py * delta, q.z + pz * delta};
            const FractalOut<double> fo = compute<double>(seq, slots.data(), p3.x, p3.y, p3.z, 1, -1);
            const double pd = double(1 + seq.formula_maxiter - fo.iters);
            n.x = n.x + px * pd;
            n.y = n.y + py * pd;
            n.z = n.z + pz * pd;
            c.de++;
            c.iters += fo.iters;
            *counter += 1;
          }
      if (fabs(n.x) < 1e-50 && fabs(n.y) < 1e-50 && fabs(n.z) < 1e-50)
        n = D3{1.0, 0.0, 0.0};
      else
        n = normalize(n);
      if (!(isfinite(n.x) && isfinite(n.y) && isfinite(n.z))) n = D3{1.0, 0.0, 0.0};
      return n;
    }
    double delta = thr * p.smoothness;
    if (seq.interior) delta = thr * 0.2 * p.smoothness;
    const uint64_t before = c.de;
    const double sx1 = de(add(q, D3{delta, 0.0, 0.0}), thr, true, nullptr, c);
    const double sx2 = de(sub(q, D3{delta, 0.0, 0.0}), thr, true, nullptr, c);
    const double sy1 = de(add(q, D3{0.0, delta, 0.0}), thr, true, nullptr, c);
    const double sy2 = de(sub(q, D3{0.0, delta, 0.0}), thr, true, nullptr, c);
    const double sz1 = de(add(q, D3{0.0, 0.0, delta}), thr, true, nullptr, c);
    const double sz2 = de(sub(q, D3{0.0, 0.0, delta}), thr, true, nullptr, c);
    *counter += c.de - before;
    D3 n{sx1 - sx2, sy1 - sy2, sz1 - sz2};
    if (fabs(n.x) < 1e-50 && fabs(n.y) < 1e-50 && fabs(n.z) < 1e-50)
      n = D3{1.0, 0.0, 0.0};
    else
      n = normalize(n);
    if (!(isfinite(n.x) && isfinite(n.y) && isfinite(n.z))) n = D3{1.0, 0.0, 0.0};
    return n;
  }

  // AuxShadow, hard shadow of a non-penetrating directional light
  // (shader_aux_shadow.cpp:39-323 with softShadowCone = 0, no fog/clouds/SSS;
  //  distance = viewDistanceMax, light.cpp:281-291).
  double aux_shadow(D3 q, double thr, D3 L, Counters &c, uint64_t *counter) const {
    // directional light: a penetrating one marches delta / resolution (light.cpp:277-290)
    const bool pen = p.penetrating != 0;
    const double distance = pen ? calc_delta(q) / resolution : p.view_distance_max;
    // cLight::softShadowCone is a float (light.h:113, light.cpp:87), so the
    // tangent is the float one (shader_aux_shadow.cpp:64)
    const float cone = float(p.soft_shadow_cone / 180.0 * M_PI);
    const double softRange = std::tan(cone);
    const bool bSoft = !seq.iter_thresh && !seq.interior && softRange > 0.0;  // :71-74
    double start = thr;
    if (seq.interior) start = thr * p.de_factor;
    double shadowTemp = 1.0;
    double maxSoft = 0.0;
    int count = 0;
    double step = thr;
    const float dist_thresh = float(thr);
    const uint64_t before = c.de;
    for (double i = start; i < distance; i += step) {
      const D3 point2 = add(q, mul(L, i));
      const double dist = de(point2, thr, false, nullptr, c);
      bool limitsReached = false;  // :130-140
      if (seq.limits) {
        if (point2.x < seq.lim_min[0] || point2.x > seq.lim_max[0] || point2.y < seq.lim_min[1] ||
            point2.y > seq.lim_max[1] || point2.z < seq.lim_min[2] || point2.z > seq.lim_max[2])
          limitsReached = true;
      }
      if (bSoft && !limitsReached) {  // :142-151
        double angle = (dist - dist_thresh) / i;
        if (angle < 0) angle = 0;
        if (dist < dist_thresh) angle = 0;
        double softShadow = 1.0 - angle / softRange;
        if (pen) softShadow *= (distance - i) / distance;
        if (softShadow < 0) softShadow = 0;
        if (softShadow > maxSoft) maxSoft = softShadow;
      }
      shadowTemp = 1.0 - 0.0;
      if (dist < dist_thresh || shadowTemp < 0.0) {  // :266-280
        if (pen) {
          shadowTemp -= (distance - i) / distance;
          if (shadowTemp < 0.0) shadowTemp = 0.0;
        } else {
          shadowTemp = 0.0;
        }
        break;
      }
      step = std::min(dist, double(1e6f)) * p.de_factor;
      step = std::max(step, 1e-15);
      count++;
      if (count > p.max_raymarching_steps) break;
    }
    *counter += c.de - before;
    return bSoft ? 1.0 - maxSoft : shadowTemp;
  }

  // AmbientOcclusion march rule (shader_ambient_occlusion.cpp:41-120) along
  // ao_rays cosine-hemisphere directions from PCG32(state ao_seed, stream pixel).
  double ambient_occlusion(D3 q, D3 n, double thr, uint64_t pixel, Counters &c, uint64_t *counter) const {
    const double start_dist = thr;
    const double end_dist = calc_delta(q) / resolution;
    const float dist_thresh = float(thr);
    Pcg32 rng = pcg_init(p.ao_seed, pixel);
    double sum = 0.0;
    const uint64_t before = c.de;
    for (int k = 0; k < p.ao_rays; k++) {
      const double u1 = rng.uniform(), u2 = rng.uniform();
      const D3 v = cosine_dir(n, u1, u2);
      double dist = 0.0;
      double shadowTemp = 1.0;
      int steps = 0;  // cap: max_raymarching_steps evaluations per AO march
      for (double r = start_dist; r < end_dist; r += dist * 2.0) {
        if (steps >= p.max_raymarching_steps) {
          c.watchdog++;
          break;
        }
        steps++;
        const D3 point2 = add(q, mul(v, r));
        dist = de(point2, thr, false, nullptr, c);
        if (dist < dist_thresh || shadowTemp < 0.0) {
          shadowTemp -= (end_dist - r) / end_dist;
          if (shadowTemp < 0.0) shadowTemp = 0.0;
          break;
        }
      }
      sum += shadowTemp;
    }
    *counter += c.de - before;
    return sum / p.ao_rays;
  }

  // FastAmbientOcclusion (shader_fast_ambient_occlusion.cpp:40-65): quality^2 - 1
  // distance samples at i^2 * distThresh along the normal, each clamped to twice
  // the previous one; the float sum of 2^-i (scan - fastTune * dist) / distThresh
  // gives ao = max(0, 1 - 0.2 sum).
  double fast_ao(D3 q, D3 n, double thr, Counters &c, uint64_t *counter) const {
    const uint64_t before = c.de;
    float aoTemp = 0.0f;
    double lastDist = 1e20;
    const int samples = p.ao_quality * p.ao_quality;
    for (int i = 1; i < samples; i++) {
      const double scan = double(i * i) * thr;
      double dist = de(add(q, mul(n, scan)), thr, false, nullptr, c);
      if (dist > lastDist * 2) dist = lastDist * 2.0;
      lastDist = dist;
      aoTemp += std::ldexp(1.0, -i) * (scan - p.ao_fast_tune * dist) / thr;
    }
    *counter += c.de - before;
    float ao = 1.0f - 0.2f * aoTemp;
    if (ao < 0) ao = 0;
    return ao;
  }

  // Image point and view direction of pixel (x, y): doWork (render_worker.cpp:155-163,
  // 247, 326-327), region.hpp:66-71 with imageRegion (-0.5, 0.5, 0.5, -0.5),
  // CalculateViewVector three-point (projection_3d.cpp:77-84, 87).
  // legacy coordinate system: imageRegion (-0.5, -0.5, 0.5, 0.5) (render_job.cpp:308-315)
  void image_point(double x, double y, double *ix, double *iy) const {
    const bool legacy = cam.legacy_coordinate_system != 0;
    const double scaleX = 1.0 / double(cam.width);
    const double scaleY = (legacy ? 1.0 : -1.0) / double(cam.height);
    *ix = (scaleX * x + -0.5) * aspect;
    *iy = scaleY * y + (legacy ? -0.5 : 0.5);
  }
  // CalculateViewVector (projection_3d.cpp:40-89) for the camera's projection
  D3 view_vector(double ix, double iy) const {
    D3 v;
    if (cam.perspective_type == MBR_PROJECTION_FISH_EYE || cam.perspective_type == MBR_PROJECTION_FISH_EYE_CUT) {
      const double r = sqrt(ix * ix + iy * iy);
      if (r == 0.0) {
        v = D3{0.0, 1.0, 0.0};
      } else {
        v = D3{ix / r * sin(r * fov), cos(r * fov), iy / r * sin(r * fov)};
      }
    } else if (cam.perspective_type == MBR_PROJECTION_EQUIRECTANGULAR) {
      const double vx = ix * 0.5, vy = iy * 0.5;
      v = D3{sin(fov * vx) * cos(fov * vy), cos(fov * vx) * cos(fov * vy), sin(fov * vy)};
    } else {
      v = D3{ix * fov, 1.0, iy * fov};
    }
    v = normalize(v);
    return rotate(M, v);
  }
  // fish-eye cut: image points beyond 90 degrees are not traced (render_worker.cpp:165-170, 321)
  bool hemisphere_cut(double ix, double iy) const {
    return cam.perspective_type == MBR_PROJECTION_FISH_EYE_CUT && sqrt(ix * ix + iy * iy) > M_PI * 0.5 / fov;
  }

  struct PixelOut {
    bool hit;
    double depth;
    int iters;
    float normal[3];
    float shade, ao, rgb[3];
    float shadow;  // the AuxShadow factor (1: lit; 0 when the surface faces away)
  };

  void shade_pixel(const March &m, uint64_t pixel, Counters &c, PixelOut &po) const {
    po.normal[0] = po.normal[1] = po.normal[2] = 0.0f;
    po.shade = 0.0f;
    po.ao = 1.0f;
    po.shadow = 1.0f;
    if (!m.found) {
      for (int k = 0; k < 3; k++) po.rgb[k] = float(p.background[k]);
      return;
    }
    const bool fast = p.ao_fast && p.gi_samples == 0;
    const bool need_normal = p.shading_enable || p.ao_rays > 0 || fast || want_normal;
    D3 n{1.0, 0.0, 0.0};
    if (need_normal) {
      n = normals(m.point, m.thr, c, &c.normal);
      po.normal[0] = float(n.x);
      po.normal[1] = float(n.y);
      po.normal[2] = float(n.z);
    }
    float shade = 0.0f;
    if (p.shading_enable) {  // LightShading (shader_light_shading.cpp:40-122), directional
      const float intensity = float(p.light_intensity);
      float s = float(dot(n, light));
      if (s < 0) s = 0;
      const float mshade = float(p.material_shading);
      s = 1.0f - mshade + s * mshade;
      s = s * intensity;
      if (s > 500.0f) s = 500.0f;
      float aux = 1.0f;
      if (p.shadow_enable) {
        if (s > 0.001f)
          aux = float(aux_shadow(m.point, m.thr, light, c, &c.shadow));
        else
          aux = 0.0f;
      }
      shade = s * aux;
      po.shadow = aux;
    }
    float ao = 1.0f;
    if (fast) ao = float(fast_ao(m.point, n, m.thr, c, &c.ao));
    else if (p.ao_rays > 0) ao = float(ambient_occlusion(m.point, n, m.thr, pixel, c, &c.ao));
    po.shade = shade;
    po.ao = ao;
    const float col = float(p.albedo) * (shade + float(p.ambient_intensity) * ao);
    po.rgb[0] = po.rgb[1] = po.rgb[2] = col;
  }

  // One path of the Monte Carlo GI estimator: primary ray with MC pixel
  // jitter (render_worker.cpp:228-232) and thin-lens DOF (MonteCarloDOF,
  // :1832-1844), then diffuse bounces with the GI march rule
  // (shader_global_illumination.cpp:75-125): scan from distThresh, step
  // dist*DEFactor, a hit closer than 2*distThresh ends the path.
  double gi_path(int x, int y, uint64_t pixel, int sample, Counters &c, March *first) const {
    const uint64_t ray = pixel * uint64_t(p.gi_samples) + uint64_t(sample);
    Pcg32 rng = pcg_init(p.gi_seed, ray);
    const double ujx = rng.uniform(), ujy = rng.uniform(), ulr = rng.uniform(), ula = rng.uniform();
    double ix, iy;
    image_point(double(x), double(y), &ix, &iy);
    ix = ix + (ujx - 0.5) / double(cam.width) * aspect;
    iy = iy + (ujy - 0.5) / double(cam.height);
    D3 view = view_vector(ix, iy);
    D3 start = camera;
    if (p.dof_aperture > 0.0) {
      const double randR = p.dof_aperture * sqrt(ulr);
      const double randAngle = 2.0 * M_PI * ula;
      const D3 rv = rotate(M, D3{randR * sin(randAngle), 0.0, randR * cos(randAngle)});
      view = sub(view, mul(rv, 1.0 / p.dof_focus));
      start = add(camera, rv);
    }
    const D3 dir = normalize(view);
    ParkMiller pm = pm_for_ray(ray, p.seed);
    March m = ray_marching(start, dir, p.view_distance_max, pm, c);
    if (first) *first = m;
    // every DE evaluation after the primary march counts as a GI evaluation
    const uint64_t after_primary = c.de;
    uint64_t unused = 0;
    double radiance = 0.0, throughput = 1.0;
    if (!m.found) {
      radiance = p.gi_sky;
    } else {
      D3 q = m.point;
      double thr = m.thr;
      D3 n = normals(q, thr, c, &unused);
      for (int bounce = 0;; bounce++) {
        const double ndl = dot(n, light);
        if (ndl > 0.0) {
          const double sh = aux_shadow(q, thr, light, c, &unused);
          radiance += throughput * p.albedo * p.gi_sun * ndl * sh;
        }
        if (bounce >= p.gi_bounces) break;
        throughput *= p.albedo;
        const double u1 = rng.uniform(), u2 = rng.uniform();
        const D3 d = cosine_dir(n, u1, u2);
        bool found = false, ended = false;
        int steps = 0;
        double dist = 0.0;
        for (double scan = thr; scan < p.view_distance_max; scan += dist * p.de_factor) {
          if (steps >= p.max_raymarching_steps) break;
          const D3 point = add(q, mul(d, scan));
          const double t2 = dist_thresh(point);
          dist = de(point, t2, false, nullptr, c);
          if (dist < t2) {
            if (scan < t2 * 2.0) {
              ended = true;
              break;
            }
            q = point;
            thr = t2;
            n = normals(q, thr, c, &unused);
            found = true;
            break;
          }
          steps++;
        }
        if (ended) break;
        if (!found) {
          radiance += throughput * p.gi_sky;
          break;
        }
      }
    }
    c.gi += c.de - after_primary;
    return radiance;
  }
};

// cImage::CalculateGammaTable (cimage.cpp:366-375)
static std::vector<int> gamma_table(double gamma) {
  std::vector<int> t(65536);
  for (int i = 0; i < 65536; i++) t[i] = int(powf(i / 65536.0f, 1.0f / float(gamma)) * 65535.0f);
  return t;
}

// cImage::CalculatePixel (cimage.cpp:317-362) + ConvertTo8bitChar (:460-469)
static void to_rgb8(const float *rgb, const mbr_render_params &p, const std::vector<int> &gamma, uint8_t *o) {
  const float br = float(p.brightness), co = float(p.contrast), sat = float(p.saturation);
  float R = rgb[0] * br, G = rgb[1] * br, B = rgb[2] * br;
  R = (R - 0.5f) * co + 0.5f;
  G = (G - 0.5f) * co + 0.5f;
  B = (B - 0.5f) * co + 0.5f;
  if (R < 0.0f) R = 0.0f;
  if (G < 0.0f) G = 0.0f;
  if (B < 0.0f) B = 0.0f;
  if (p.hdr) {
    R = tanhf(R);
    G = tanhf(G);
    B = tanhf(B);
  }
  const float rF = 0.299f, gF = .587f, bF = .114f;
  const float V = sqrtf(R * R * rF + G * G * gF + B * B * bF);
  R = V + (R - V) * sat;
  G = V + (G - V) * sat;
  B = V + (B - V) * sat;
  R = std::min(std::max(R, 0.0f), 1.0f);
  G = std::min(std::max(G, 0.0f), 1.0f);
  B = std::min(std::max(B, 0.0f), 1.0f);
  const uint16_t r16 = uint16_t(gamma[uint16_t(R * 65535.0f)]);
  const uint16_t g16 = uint16_t(gamma[uint16_t(G * 65535.0f)]);
  const uint16_t b16 = uint16_t(gamma[uint16_t(B * 65535.0f)]);
  o[0] = uint8_t(r16 / 256);
  o[1] = uint8_t(g16 / 256);
  o[2] = uint8_t(b16 / 256);
}

static bool make_renderer(const mbr_scene *scene, const mbr_camera *cam, const mbr_render_params *params,
                          Renderer *R) {
  if (!build_sequence(*scene, &R->seq)) return false;
  // the delta DE's offset factor (calculate_distance.cpp:616-623)
  R->seq.delta_factor = params->advanced_quality ? R->seq.delta_rel : 1e-5;
  R->slots.clear();
  for (int i = 0; i < R->seq.n; i++) R->slots.push_back(make_slot<double>(R->seq.slot[i], false));
  R->p = *params;
  R->cam = *cam;
  double ang[3];
  camera_setup(*cam, &R->M, ang);
  R->camera = D3{cam->camera[0], cam->camera[1], cam->camera[2]};
  R->fov = calc_fov(*cam);
  R->resolution = 1.0 / cam->height;                // render_job.cpp:477
  R->aspect = double(cam->width) / cam->height;     // render_worker.cpp:98
  if (cam->perspective_type == MBR_PROJECTION_EQUIRECTANGULAR) R->aspect = 2.0;  // :100
  R->light = normalize(D3{params->light_direction[0], params->light_direction[1], params->light_direction[2]});
  R->gamma = gamma_table(params->gamma);
  return true;
}

}  // namespace oracle

using namespace oracle;

// ============================================================================
// C entry points (called through ctypes by tests/ and bench.py only).
// ============================================================================
extern "C" {

typedef struct oracle_outputs {  // host buffers, same meaning as mbr_outputs
  double *depth;
  int32_t *iters;
  uint8_t *hit;
  float *normal;
  float *shade;
  float *ao;
  float *rgb;
  uint8_t *rgb8;
  float *shadow;  // the main light's AuxShadow factor per pixel (may be NULL)
} oracle_outputs;

// The reference's defaults (src/initparameters.cpp) for the C-ABI structs,
// so that the CPU legs of the benchmark fill their parameters without the
// product library.  tests/test_oracle_defaults.py holds them equal to the
// library's mbr_*_defaults.
void oracle_fractal_defaults(mbr_fractal *f, int formula) {
  std::memset(f, 0, sizeof(*f));
  f->formula = formula;
  f->formula_iterations = 1;     // initparameters.cpp:2109-2125 (node defaults)
  f->formula_stop_iteration = 250;
  f->check_for_bailout = 1;
  f->formula_weight = 1.0;
  f->bulb_power = 9.0;           // :717
  f->mandelbox_scale = 2.0;      // :746-750
  f->mandelbox_folding_limit = 1.0;
  f->mandelbox_folding_value = 2.0;
  f->mandelbox_folding_min_radius = 0.5;
  f->mandelbox_folding_fixed_radius = 1.0;
  f->transf_scale3 = 3.0;        // :1010
  f->ifs_scale = 2.0;            // :724-743
  f->ifs_offset[0] = 1.0;
  for (int i = 0; i < 9; i++) {
    f->ifs_direction[i][0] = 1.0;
    f->ifs_intensity[i] = 1.0;
  }
  f->aexion_cadd = -1.3;        // initparameters.cpp:722
  f->analytic_de_enabled = 1;   // :904-909
  f->analytic_de_scale1 = 1.0;
  f->analytic_de_offset1 = 1.0;
}

void oracle_scene_defaults(mbr_scene *s) {
  std::memset(s, 0, sizeof(*s));
  s->n_fractals = 1;             // :128-157, node :2102-2125
  s->formula_maxiter = 250;
  s->repeat_from = 1;
  s->use_default_bailout = 1;
  s->min_n = 1;
  s->bailout = 100.0;
  for (int i = 0; i < 3; i++) s->fractal_constant_factor[i] = 1.0;
  oracle_fractal_defaults(&s->fractal[0], MBR_FORMULA_MANDELBULB);
  for (int i = 1; i < MBR_MAX_FRACTALS; i++) oracle_fractal_defaults(&s->fractal[i], MBR_FORMULA_NONE);
  for (int i = 0; i < 3; i++) {  // :143-145
    s->limit_min[i] = -10.0;
    s->limit_max[i] = 10.0;
  }
  s->box_folding_limit = 1.0;  // :199-204
  s->box_folding_value = 2.0;
  s->spherical_folding_inner = 0.5;
  s->spherical_folding_outer = 1.0;
  s->delta_de_method = MBR_DE_METHOD_PREFERRED;
  s->deltade_relative_delta = 0.01;  // initparameters.cpp:166
}

void oracle_camera_defaults(mbr_camera *c) {
  std::memset(c, 0, sizeof(*c));
  c->camera[0] = 3.0;            // :113-120
  c->camera[1] = -6.0;
  c->camera[2] = 2.0;
  c->top[0] = -0.1277753;
  c->top[1] = 0.2555506;
  c->top[2] = 0.958314;
  c->fov_deg = 53.13;
  c->width = 800;                // :173-174
  c->height = 600;
}

void oracle_render_params_defaults(mbr_render_params *p) {
  std::memset(p, 0, sizeof(*p));
  p->detail_level = 1.0;         // :133-167
  p->de_factor = 1.0;
  p->view_distance_max = 50.0;
  p->smoothness = 1.0;
  p->max_raymarching_steps = 10000;
  p->binary_steps = 30;          // render_worker.cpp:854
  p->refine = MBR_REFINE_REFERENCE;
  p->jitter = 1;
  p->de_thresh = 0.01;
  p->shading_enable = 1;
  p->shadow_enable = 1;
  p->light_direction[0] = 1.0;
  p->light_direction[1] = -1.0;
  p->light_direction[2] = 1.0;
  p->light_intensity = 1.0;
  p->material_shading = 1.0;
  p->albedo = 1.0;
  p->dof_focus = 3.0;
  p->gi_sky = 0.3;
  p->gi_sun = 3.0;
  p->brightness = 1.0;           // :208-212
  p->contrast = 1.0;
  p->gamma = 1.0;
  p->saturation = 1.0;
  p->soft_shadow_cone = 1.0;     // light 1, :1901, 1919
  p->penetrating = 1;
  p->ao_quality = 4;             // :214-216
  p->ao_fast_tune = 1.0;
  p->abs_max_marching_step = 3.0;  // :159-165
  p->abs_min_marching_step = 1e-15;
  p->rel_max_marching_step = 1e4;
  p->rel_min_marching_step = 1e-2;
  p->detail_size_max = 1.0;
  p->detail_size_min = 1e-12;
}

int oracle_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

// Renders rows [row0, row1) (all columns) of the frame.  Rows are handed to
// threads one at a time, dynamically (the cScheduler line model,
// scheduler.cpp:122-183).  Returns 0 on success.
//
// params->jitter == 2 (the oracle only): the march jitter draws from ONE
// Park-Miller state seeded with params->seed and consumed in pixel order
// (rows top to bottom, pixels left to right), as the reference's
// process-global Random() is consumed by one render thread without
// progressive passes (common_math.cpp:47-72; render_worker.cpp:126-134,
// 811-815).  It renders on one thread, so that golden frames of the
// reference's own render worker can be reproduced bit for bit.
int oracle_render(const mbr_scene *scene, const mbr_camera *cam, const mbr_render_params *params,
                  const oracle_outputs *out, int row0, int row1, int nthreads, mbr_stats *stats) {
  Renderer R;
  if (!make_renderer(scene, cam, params, &R)) return 1;
  R.want_normal = out->normal != nullptr;
  const int W = cam->width;
  std::atomic<uint64_t> tot[10];
  for (auto &t : tot) t = 0;
  const bool global_stream = params->jitter == 2;
  ParkMiller gpm;
  gpm.s = params->seed;
  if (global_stream) nthreads = 1;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel
#endif
  {
    Counters c;
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 1)
#endif
    for (int y = row0; y < row1; y++) {
      for (int x = 0; x < W; x++) {
        const uint64_t pixel = uint64_t(y) * W + x;
        Renderer::PixelOut po;
        Renderer::March m;
        double cx, cy;
        R.image_point(double(x), double(y), &cx, &cy);
        if (R.hemisphere_cut(cx, cy)) {  // black, depth 1e20, no hit
          po.hit = false;
          po.depth = 1e20;
          po.iters = 0;
          po.normal[0] = po.normal[1] = po.normal[2] = 0.0f;
          po.shade = 0.0f;
          po.ao = 1.0f;
          po.shadow = 1.0f;
          po.rgb[0] = po.rgb[1] = po.rgb[2] = 0.0f;
        } else if (params->gi_samples > 0) {
          double acc = 0.0;
          for (int s = 0; s < params->gi_samples; s++) {
            Renderer::March mm;
            acc += R.gi_path(x, y, pixel, s, c, s == 0 ? &m : &mm);
          }
          const float v = float(acc / params->gi_samples);
          po.hit = m.found;
          po.depth = m.found ? m.depth : 1e20;
          po.iters = m.iters;
          po.normal[0] = po.normal[1] = po.normal[2] = 0.0f;
          po.shade = 0.0f;
          po.ao = 1.0f;
          po.shadow = 1.0f;
          po.rgb[0] = po.rgb[1] = po.rgb[2] = v;
        } else {
          double ix, iy;
          R.image_point(double(x), double(y), &ix, &iy);
          D3 dir = R.view_vector(ix, iy);
          dir = normalize(dir);
          ParkMiller pm = global_stream ? gpm : pm_for_ray(pixel, params->seed);
          m = R.ray_marching(R.camera, dir, params->view_distance_max, pm, c);
          if (global_stream) gpm = pm;
          R.shade_pixel(m, pixel, c, po);
          po.hit = m.found;
          po.depth = m.found ? m.depth : 1e20;
          po.iters = m.iters;
        }
        c.pixels++;
        const size_t o = size_t(pixel - uint64_t(row0) * W);
        if (out->depth) out->depth[o] = po.depth;
        if (out->iters) out->iters[o] = po.iters;
        if (out->hit) out->hit[o] = po.hit ? 1 : 0;
        if (out->normal) for (int k = 0; k < 3; k++) out->normal[o * 3 + k] = po.normal[k];
        if (out->shade) out->shade[o] = po.shade;
        if (out->ao) out->ao[o] = po.ao;
        if (out->rgb) for (int k = 0; k < 3; k++) out->rgb[o * 3 + k] = po.rgb[k];
        if (out->rgb8) to_rgb8(po.rgb, *params, R.gamma, &out->rgb8[o * 3]);
        if (out->shadow) out->shadow[o] = po.shadow;
      }
    }
    tot[0] += c.de; tot[1] += c.iters; tot[2] += c.march; tot[3] += c.binary; tot[4] += c.normal;
    tot[5] += c.shadow; tot[6] += c.ao; tot[7] += c.gi; tot[8] += c.pixels; tot[9] += c.watchdog;
  }
  if (stats) {
    stats->de_evals += tot[0]; stats->formula_iterations += tot[1]; stats->march_steps += tot[2];
    stats->binary_steps += tot[3]; stats->normal_evals += tot[4]; stats->shadow_evals += tot[5];
    stats->ao_evals += tot[6]; stats->gi_evals += tot[7]; stats->pixels += tot[8];
    stats->watchdog_trips += tot[9];
  }
  return 0;
}

// CalculateDistance at n points (xyz interleaved).
int oracle_distance(const mbr_scene *scene, const double *pts, int64_t n, double detail, int normal_mode,
                    double *dist, int32_t *iters) {
  Seq seq;
  if (!build_sequence(*scene, &seq)) return 1;
  std::vector<SlotT<double>> slots;
  for (int i = 0; i < seq.n; i++) slots.push_back(make_slot<double>(seq.slot[i], false));
  for (int64_t i = 0; i < n; i++) {
    int it = 0;
    dist[i] = calc_distance<double>(seq, slots.data(), pts[3 * i], pts[3 * i + 1], pts[3 * i + 2], detail,
                                    normal_mode != 0, &it);
    if (iters) iters[i] = it;
  }
  return 0;
}

// Hybrid sequence of a scene (for cross-checking the library's host builder).
int oracle_sequence(const mbr_scene *scene, int32_t *seq_out, int32_t *length, int32_t *de_function,
                    double *bailout) {
  Seq seq;
  if (!build_sequence(*scene, &seq)) return 1;
  for (int i = 0; i < seq.length; i++) seq_out[i] = seq.seq[i];
  *length = seq.length;
  *de_function = seq.is_hybrid ? seq.de_function : seq.de_analytic;
  for (int i = 0; i < seq.n; i++) bailout[i] = seq.slot[i].bailout;
  return 0;
}

// One formula iteration of slot `slot` at z (4 doubles in/out) with running
// derivative *de and radius *r, exactly as Compute calls FormulaCode.
int oracle_formula_step(const mbr_scene *scene, int slot, double *z, double *r, double *de) {
  Seq seq;
  if (!build_sequence(*scene, &seq)) return 1;
  SlotT<double> f = make_slot<double>(seq.slot[slot], false);
  V4<double> v{z[0], z[1], z[2], z[3]};
  switch (seq.slot[slot].formula) {
    case MBR_FORMULA_MANDELBULB: formula_mandelbulb(v, f, *r, *de); break;
    case MBR_FORMULA_MANDELBOX: formula_mandelbox(v, f, *de); break;
    case MBR_FORMULA_MENGER_SPONGE: formula_menger(v, f, *de); break;
    case MBR_FORMULA_MANDELBULB_POWER2: formula_bulb_pow2(v, *r, *de); break;
    case MBR_FORMULA_HYPERCOMPLEX: formula_hypercomplex(v, *r, *de); break;
    case MBR_FORMULA_KALEIDOSCOPIC_IFS: formula_ifs(v, f, *de); break;
    case MBR_FORMULA_XENODREAMBUIE: formula_xenodreambuie(v, f, *r, *de); break;
    case MBR_FORMULA_QUATERNION: formula_quaternion(v, *r, *de); break;
    default: return 1;
  }
  z[0] = v.x; z[1] = v.y; z[2] = v.z; z[3] = v.w;
  return 0;
}

// Camera rotation (row-major mRot, zero flag in mrot[9]) and view angles.
int oracle_camera(const mbr_camera *cam, double *mrot10, double *angles) {
  Mat3 M;
  camera_setup(*cam, &M, angles);
  for (int i = 0; i < 9; i++) mrot10[i] = M.m[i];
  mrot10[9] = M.zero ? 1.0 : 0.0;
  return 0;
}

// View direction (after both normalisations) of pixel (x, y).
int oracle_view(const mbr_camera *cam, int x, int y, double *dir) {
  Renderer R;
  R.cam = *cam;
  double ang[3];
  camera_setup(*cam, &R.M, ang);
  R.fov = calc_fov(*cam);
  R.aspect = double(cam->width) / cam->height;
  if (cam->perspective_type == MBR_PROJECTION_EQUIRECTANGULAR) R.aspect = 2.0;  // render_worker.cpp:100
  double ix, iy;
  R.image_point(double(x), double(y), &ix, &iy);
  D3 d = normalize(R.view_vector(ix, iy));
  dir[0] = d.x; dir[1] = d.y; dir[2] = d.z;
  return 0;
}

// View direction (after both normalisations) of a normalised image point.
int oracle_view_ip(const mbr_camera *cam, double ix, double iy, double *dir) {
  Renderer R;
  R.cam = *cam;
  double ang[3];
  camera_setup(*cam, &R.M, ang);
  R.fov = calc_fov(*cam);
  D3 d = normalize(R.view_vector(ix, iy));
  dir[0] = d.x; dir[1] = d.y; dir[2] = d.z;
  return 0;
}

// Park-Miller draws: n values of Random(max) from the reference generator
// state `seed` (seed = 0 selects the per-ray stream of ray `ray`).
int oracle_park_miller(uint32_t seed, uint64_t ray, uint32_t ray_seed, int max, int n, int32_t *out) {
  ParkMiller pm;
  if (seed != 0) pm.s = seed; else pm = pm_for_ray(ray, ray_seed);
  for (int i = 0; i < n; i++) out[i] = (max < 0) ? pm.next() : pm.random(max);
  return 0;
}

int oracle_pcg32(uint64_t initstate, uint64_t initseq, int n, uint32_t *out) {
  Pcg32 p = pcg_init(initstate, initseq);
  for (int i = 0; i < n; i++) out[i] = p.next();
  return 0;
}

// Operation counts of one formula iteration of `slot` at z (for the
// roofline's algorithmic-work figure).  out: add, mul, div, sqrt, transc, cmp.
int oracle_opcount(const mbr_scene *scene, int slot, const double *z, uint64_t *out) {
  Seq seq;
  if (!build_sequence(*scene, &seq)) return 1;
  SlotT<OpCount> f = make_slot<OpCount>(seq.slot[slot], false);
  g_tally = OpTally();
  V4<OpCount> v{OpCount(z[0]), OpCount(z[1]), OpCount(z[2]), OpCount(z[3])};
  OpCount DE(1.0);
  OpCount r = len4(v);
  g_tally = OpTally();
  switch (seq.slot[slot].formula) {
    case MBR_FORMULA_MANDELBULB: formula_mandelbulb(v, f, r, DE); break;
    case MBR_FORMULA_MANDELBOX: formula_mandelbox(v, f, DE); break;
    case MBR_FORMULA_MENGER_SPONGE: formula_menger(v, f, DE); break;
    case MBR_FORMULA_MANDELBULB_POWER2: formula_bulb_pow2(v, r, DE); break;
    case MBR_FORMULA_HYPERCOMPLEX: formula_hypercomplex(v, r, DE); break;
    case MBR_FORMULA_KALEIDOSCOPIC_IFS: formula_ifs(v, f, DE); break;
    case MBR_FORMULA_XENODREAMBUIE: formula_xenodreambuie(v, f, r, DE); break;
    default: return 1;
  }
  // the per-iteration work of Compute around the formula: c-add and |z|
  if (seq.slot[slot].add_c) {
    v.x = v.x + OpCount(z[0]) * seq.cmul[0];
    v.y = v.y + OpCount(z[1]) * seq.cmul[1];
    v.z = v.z + OpCount(z[2]) * seq.cmul[2];
    v.w = v.w + OpCount(z[3]);
  }
  r = len4(v);
  (void)(r > 10.0);
  out[0] = g_tally.add; out[1] = g_tally.mul; out[2] = g_tally.div;
  out[3] = g_tally.sqrt; out[4] = g_tally.transc; out[5] = g_tally.cmp;
  return 0;
}

// Operation counts of whole CalculateDistance evaluations at n points
// (xyz interleaved): out = add, mul, div, sqrt, transc, cmp, sum of iters, n,
// essential add, essential mul.
// The per-iteration algorithmic work of the roofline is (add + mul) / iters.
int oracle_opcount_de(const mbr_scene *scene, const double *pts, int64_t n, double detail, uint64_t *out) {
  Seq seq;
  if (!build_sequence(*scene, &seq)) return 1;
  std::vector<SlotT<OpCount>> slots;
  for (int i = 0; i < seq.n; i++) slots.push_back(make_slot<OpCount>(seq.slot[i], false));
  g_tally = OpTally();
  uint64_t iters = 0;
  for (int64_t i = 0; i < n; i++) {
    int it = 0;
    calc_distance<OpCount>(seq, slots.data(), OpCount::computed(pts[3 * i]), OpCount::computed(pts[3 * i + 1]),
                           OpCount::computed(pts[3 * i + 2]),
                           detail, false, &it);
    iters += uint64_t(it);
  }
  out[0] = g_tally.add; out[1] = g_tally.mul; out[2] = g_tally.div;
  out[3] = g_tally.sqrt; out[4] = g_tally.transc; out[5] = g_tally.cmp;
  out[6] = iters; out[7] = uint64_t(n); out[8] = g_tally.e_add; out[9] = g_tally.e_mul;
  return 0;
}

// CalculateDistance and its forward-mode tangents (power, scale, mR2, x, y, z)
// at n points: out[7 i] = value, out[7 i + 1 + k] = tangent k.
int oracle_de_tangents(const mbr_scene *scene, const double *pts, int64_t n, double detail, int normal_mode,
                       double *out) {
  Seq seq;
  if (!build_sequence(*scene, &seq)) return 1;
  typedef Dual<6> DD;
  std::vector<SlotT<DD>> slots;
  for (int i = 0; i < seq.n; i++) slots.push_back(make_slot<DD>(seq.slot[i], true));
  for (int64_t i = 0; i < n; i++) {
    DD x = DD::seed(pts[3 * i], TAN_X), y = DD::seed(pts[3 * i + 1], TAN_Y), z = DD::seed(pts[3 * i + 2], TAN_Z);
    DD d = calc_distance<DD>(seq, slots.data(), x, y, z, detail, normal_mode != 0, nullptr);
    out[7 * i] = d.v;
    for (int k = 0; k < 6; k++) out[7 * i + 1 + k] = d.d[k];
  }
  return 0;
}

// Dual-number reference of the adjoint: for each pixel with hit[i] != 0, the
// depth derivative dt/dθ (by the implicit function of F(t) = dist - thr at the
// stored depth) and the derivative of the Lambert term max(N·L, 0) through the
// six central-difference DE evaluations.  Parameters θ in MBR_GRAD_* order.
// dt_dtheta / ds_dtheta: [n_pixels * MBR_GRAD_COUNT] (host).
int oracle_pixel_gradients(const mbr_scene *scene, const mbr_camera *cam, const mbr_render_params *params,
                           const double *depth, const uint8_t *hit, double *dt_dtheta, double *ds_dtheta,
                           double *shade_out) {
  Renderer R;
  if (!make_renderer(scene, cam, params, &R)) return 1;
  if (!cam->use_angles) return 2;
  typedef Dual<6> DD;  // tangents: power, scale, mR2, x, y, z
  const Seq &seq = R.seq;
  std::vector<SlotT<DD>> slots;
  for (int i = 0; i < seq.n; i++) slots.push_back(make_slot<DD>(seq.slot[i], true));
  const int W = cam->width, H = cam->height;
  const double c0 = R.resolution * R.fov / params->detail_level;  // thr = c0 * |cam - p|
  // d(mRot)/d(yaw): mRot = Rz(yaw) Rx(pitch) Ry(roll)
  const double yaw = cam->angles[0], pitch = cam->angles[1], roll = cam->angles[2];
  double Rz_d[9] = {-sin(yaw), -cos(yaw), 0, cos(yaw), -sin(yaw), 0, 0, 0, 0};
  Mat3 Rx, Ry;
  for (int i = 0; i < 9; i++) Rx.m[i] = Ry.m[i] = (i % 4 == 0) ? 1.0 : 0.0;
  Rx.zero = Ry.zero = true;
  rot_axis(Rx, 0, pitch);
  rot_axis(Ry, 1, roll);
  double dM[9];
  mat_mul(Rz_d, Rx.m, dM);
  mat_mul(dM, Ry.m, dM);
  auto eval = [&](D3 q, double thr, bool nm, double *g) -> double {
    DD x = DD::seed(q.x, TAN_X), y = DD::seed(q.y, TAN_Y), z = DD::seed(q.z, TAN_Z);
    DD d = calc_distance<DD>(seq, slots.data(), x, y, z, thr, nm, nullptr);
    for (int k = 0; k < 6; k++) g[k] = d.d[k];
    return d.v;
  };
  for (int py = 0; py < H; py++) {
    for (int px = 0; px < W; px++) {
      const size_t i = size_t(py) * W + px;
      double *dt = dt_dtheta + i * MBR_GRAD_COUNT;
      double *ds = ds_dtheta + i * MBR_GRAD_COUNT;
      for (int k = 0; k < MBR_GRAD_COUNT; k++) dt[k] = ds[k] = 0.0;
      if (shade_out) shade_out[i] = 0.0;
      if (!hit[i]) continue;
      double ix, iy;
      R.image_point(double(px), double(py), &ix, &iy);
      const D3 v0 = normalize(D3{ix * R.fov, 1.0, iy * R.fov});
      const D3 dir = normalize(rotate(R.M, v0));
      const double t = depth[i];
      const D3 p = add(R.camera, mul(dir, t));
      const double thr = R.dist_thresh(p);
      double g[6];
      const double dv = eval(p, thr, false, g);
      // implicit differentiation needs F(t) = dist - thr = 0; a bisection
      // that converged onto a jump of the distance estimate (an orbit's
      // bailout iteration changing along the ray) leaves |F| large
      if (std::fabs(dv - thr) > 1e-6 * thr) continue;
      const D3 grad{g[3], g[4], g[5]};
      // ∂p/∂θ at fixed t, for θ in MBR_GRAD order
      D3 dp[MBR_GRAD_COUNT];
      for (int k = 0; k < MBR_GRAD_COUNT; k++) dp[k] = D3{0, 0, 0};
      dp[MBR_GRAD_CAMERA_X] = D3{1, 0, 0};
      dp[MBR_GRAD_CAMERA_Y] = D3{0, 1, 0};
      dp[MBR_GRAD_CAMERA_Z] = D3{0, 0, 1};
      {  // d(dir)/d(yaw): dir = normalize(M v0); |M v0| = 1 for orthonormal M
        const D3 w{dM[0] * v0.x + dM[1] * v0.y + dM[2] * v0.z, dM[3] * v0.x + dM[4] * v0.y + dM[5] * v0.z,
                   dM[6] * v0.x + dM[7] * v0.y + dM[8] * v0.z};
        dp[MBR_GRAD_YAW] = mul(w, t);
      }
      double dd[MBR_GRAD_COUNT] = {0};
      dd[MBR_GRAD_BULB_POWER] = g[TAN_POWER];
      dd[MBR_GRAD_MANDELBOX_SCALE] = g[TAN_SCALE];
      dd[MBR_GRAD_MANDELBOX_MIN_R2] = g[TAN_MR2];
      const double denom = dot(grad, dir) - c0;
      for (int k = 0; k < MBR_GRAD_COUNT; k++) dt[k] = -(dd[k] + dot(grad, dp[k])) / denom;
      // Lambert term through CalculateNormals
      const double delta = thr * params->smoothness;
      const D3 e[3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
      double gval[3];
      double gder[3][MBR_GRAD_COUNT];
      for (int a = 0; a < 3; a++) {
        double gp[6], gm[6];
        const double dpv = eval(add(p, mul(e[a], delta)), thr, true, gp);
        const double dmv = eval(sub(p, mul(e[a], delta)), thr, true, gm);
        gval[a] = dpv - dmv;
        for (int k = 0; k < MBR_GRAD_COUNT; k++) {
          // total dp/dθ = ∂p/∂θ + dir dt/dθ ; dδ/dθ = c0 * smoothness * dt/dθ (thr = c0 t)
          const D3 dpt = add(dp[k], mul(dir, dt[k]));
          const double ddelta = c0 * params->smoothness * dt[k];
          double dplus = 0.0, dminus = 0.0;
          if (k <= MBR_GRAD_MANDELBOX_MIN_R2) {
            dplus += gp[k];
            dminus += gm[k];
          }
          const D3 gpv{gp[3], gp[4], gp[5]}, gmv{gm[3], gm[4], gm[5]};
          dplus += dot(gpv, add(dpt, mul(e[a], ddelta)));
          dminus += dot(gmv, sub(dpt, mul(e[a], ddelta)));
          gder[a][k] = dplus - dminus;
        }
      }
      const double gl = sqrt(gval[0] * gval[0] + gval[1] * gval[1] + gval[2] * gval[2]);
      const D3 N{gval[0] / gl, gval[1] / gl, gval[2] / gl};
      const double s = dot(N, R.light);
      if (shade_out) shade_out[i] = s > 0 ? s : 0.0;
      if (s > 0.0) {
        for (int k = 0; k < MBR_GRAD_COUNT; k++) {
          const D3 dg{gder[0][k], gder[1][k], gder[2][k]};
          // dN = (I - N N^T) dg / |g|
          const double ndg = dot(N, dg);
          const D3 dn = mul(sub(dg, mul(N, ndg)), 1.0 / gl);
          ds[k] = dot(dn, R.light);
        }
      }
    }
  }
  return 0;
}

}  // extern "C"
