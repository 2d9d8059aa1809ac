// ref_harness.cpp - C entry points around the REFERENCE's own compiled
// sources (formula/definition/fractal_{mandelbulb,mandelbox,menger_sponge}.cpp,
// src/camera_target.cpp, src/projection_3d.cpp, src/common_math.cpp,
// src/algebra.cpp), built by oracle/build_ref.sh into oracle/_ref/libref.so.
// Used only by tests/golden/make_golden.py and the CPU tests that pin the
// oracle against the reference.
#include <cstring>

#include "formula/definition/all_fractal_definitions.h"
#include "src/camera_target.hpp"
#include "src/common_math.h"
#include "src/fractal.h"
#include "src/projection_3d.hpp"

// cAbstractFractal's out-of-line members live in abstract_fractal.cpp, which
// needs Qt; the formulas need only construction and the vtable.
cAbstractFractal::cAbstractFractal() {}
cAbstractFractal::~cAbstractFractal() {}
std::string cAbstractFractal::getIconName() const { return std::string(); }
std::string cAbstractFractal::getUiFilename() const { return std::string(); }
std::string cAbstractFractal::getOpenCLFilename() const { return std::string(); }

static sFractal g_fractal;  // zero-initialised static storage; rotations disabled

extern "C" {

// One FormulaCode call.  params: formula-specific doubles
//   mandelbulb: power, alpha(rad), beta(rad)
//   mandelbox:  scale, limit, value, minR, fixedR, offset x, y, z
//   menger:     scale3
// z: 4 doubles in/out; aux_r, aux_de in/out.  Returns 0 on success.
int ref_formula_step(int formula, const double *params, double *z, double *aux_r, double *aux_de, int iter) {
  sFractal &f = g_fractal;
  sExtendedAux aux;
  std::memset(&aux, 0, sizeof(aux));
  aux.r = *aux_r;
  aux.DE = *aux_de;
  aux.i = iter;
  aux.color = 1.0;
  CVector4 v(z[0], z[1], z[2], z[3]);
  if (formula == 2) {
    f.bulb.power = params[0];
    f.bulb.alphaAngleOffset = params[1];
    f.bulb.betaAngleOffset = params[2];
    static cFractalMandelbulb fm;
    fm.FormulaCode(v, &f, aux);
  } else if (formula == 8) {
    f.mandelbox.scale = params[0];
    f.mandelbox.foldingLimit = params[1];
    f.mandelbox.foldingValue = params[2];
    f.mandelbox.foldingSphericalMin = params[3];
    f.mandelbox.foldingSphericalFixed = params[4];
    f.mandelbox.offset = CVector4(params[5], params[6], params[7], 0.0);
    f.mandelbox.rotationsEnabled = false;
    f.mandelbox.mainRotationEnabled = false;
    // sFractal::RecalculateFractalParams (fractal.cpp:673-675)
    f.mandelbox.fR2 = f.mandelbox.foldingSphericalFixed * f.mandelbox.foldingSphericalFixed;
    f.mandelbox.mR2 = f.mandelbox.foldingSphericalMin * f.mandelbox.foldingSphericalMin;
    f.mandelbox.mboxFactor1 = f.mandelbox.fR2 / f.mandelbox.mR2;
    static cFractalMandelbox fb;
    fb.FormulaCode(v, &f, aux);
  } else if (formula == 3) {
    static cFractalMandelbulbPower2 fp2;
    fp2.FormulaCode(v, &f, aux);
  } else if (formula == 4) {
    static cFractalHypercomplex fh;
    fh.FormulaCode(v, &f, aux);
  } else if (formula == 11) {
    f.bulb.power = params[0];
    f.bulb.alphaAngleOffset = params[1];
    f.bulb.betaAngleOffset = params[2];
    static cFractalXenodreambuie fx;
    fx.FormulaCode(v, &f, aux);
  } else if (formula == 7) {
    f.transformCommon.scale3 = params[0];
    f.foldColor.auxColorEnabledFalse = false;
    static cFractalMengerSponge fs;
    fs.FormulaCode(v, &f, aux);
  } else {
    return 1;
  }
  z[0] = v.x;
  z[1] = v.y;
  z[2] = v.z;
  z[3] = v.w;
  *aux_r = aux.r;
  *aux_de = aux.DE;
  return 0;
}

// One cFractalKaleidoscopicIfs::FormulaCode step.  params (97 values):
// scale, rotationEnabled, rotation (3, degrees), offset (3), edgeEnabled,
// edge (3), absX, absY, absZ, mengerSpongeMode, then for each of the nine
// vectors: enabled, direction (3), rotations (3, degrees), distance,
// intensity.  Directions and matrices are derived as sFractal's constructor
// and RecalculateFractalParams derive them (fractal.cpp:96-115, 655-661).
int ref_ifs_step(const double *params, double *z, double *aux_r, double *aux_de, int iter) {
  sFractal &f = g_fractal;
  sExtendedAux aux;
  std::memset(&aux, 0, sizeof(aux));
  aux.r = *aux_r;
  aux.DE = *aux_de;
  aux.i = iter;
  aux.color = 1.0;
  CVector4 v(z[0], z[1], z[2], z[3]);
  sFractalIFS &I = f.IFS;
  I.scale = params[0];
  I.rotationEnabled = params[1] != 0.0;
  I.rotation = CVector3(params[2], params[3], params[4]);
  I.offset = CVector4(CVector3(params[5], params[6], params[7]), 0.0);
  I.edgeEnabled = params[8] != 0.0;
  I.edge = CVector3(params[9], params[10], params[11]);
  I.absX = params[12] != 0.0;
  I.absY = params[13] != 0.0;
  I.absZ = params[14] != 0.0;
  I.mengerSpongeMode = params[15] != 0.0;
  for (int i = 0; i < IFS_VECTOR_COUNT; i++) {
    const double *q = params + 16 + 9 * i;
    I.enabled[i] = q[0] != 0.0;
    I.direction[i] = CVector4(CVector3(q[1], q[2], q[3]), 0.0);
    I.rotations[i] = CVector3(q[4], q[5], q[6]);
    I.distance[i] = q[7];
    I.intensity[i] = q[8];
    I.direction[i].Normalize();
  }
  I.mainRot.SetRotation3(I.rotation * M_PI_180);
  for (int i = 0; i < IFS_VECTOR_COUNT; i++) {
    I.rot[i].SetRotation3(I.rotations[i] * M_PI_180);
    I.direction[i].Normalize();
  }
  static cFractalKaleidoscopicIfs fk;
  fk.FormulaCode(v, &f, aux);
  z[0] = v.x;
  z[1] = v.y;
  z[2] = v.z;
  z[3] = v.w;
  *aux_r = aux.r;
  *aux_de = aux.DE;
  return 0;
}

// One cFractalMandelbox::FormulaCode step with rotations.  params: the eight
// Mandelbox parameters of ref_formula_step, then rotationsEnabled,
// mainRotationEnabled, rotation[0][0..2] (mandelbox_rotation_neg_1..3, 9
// degrees), rotation[1][0..2] (mandelbox_rotation_pos_1..3, 9 degrees) and
// rotationMain (3 degrees): 31 values.  The matrices are built as
// sFractal::RecalculateFractalParams builds them (fractal.cpp:663-671).
int ref_mandelbox_rot_step(const double *params, double *z, double *aux_r, double *aux_de, int iter) {
  sFractal &f = g_fractal;
  sExtendedAux aux;
  std::memset(&aux, 0, sizeof(aux));
  aux.r = *aux_r;
  aux.DE = *aux_de;
  aux.i = iter;
  aux.color = 1.0;
  CVector4 v(z[0], z[1], z[2], z[3]);
  f.mandelbox.scale = params[0];
  f.mandelbox.foldingLimit = params[1];
  f.mandelbox.foldingValue = params[2];
  f.mandelbox.foldingSphericalMin = params[3];
  f.mandelbox.foldingSphericalFixed = params[4];
  f.mandelbox.offset = CVector4(params[5], params[6], params[7], 0.0);
  f.mandelbox.rotationsEnabled = params[8] != 0.0;
  f.mandelbox.mainRotationEnabled = params[9] != 0.0;
  for (int fold = 0; fold < 2; fold++)
    for (int axis = 0; axis < 3; axis++) {
      const double *a = params + 10 + fold * 9 + axis * 3;
      f.mandelbox.rotation[fold][axis] = CVector3(a[0], a[1], a[2]);
    }
  f.mandelbox.rotationMain = CVector3(params[28], params[29], params[30]);
  f.mandelbox.mainRot.SetRotation2(f.mandelbox.rotationMain * M_PI_180);
  for (int fold = 0; fold < MANDELBOX_FOLDS; ++fold)
    for (int axis = 0; axis < 3; ++axis) {
      f.mandelbox.rot[fold][axis].SetRotation2(f.mandelbox.rotation[fold][axis] * M_PI_180);
      f.mandelbox.rotinv[fold][axis] = f.mandelbox.rot[fold][axis].Transpose();
    }
  f.mandelbox.fR2 = f.mandelbox.foldingSphericalFixed * f.mandelbox.foldingSphericalFixed;
  f.mandelbox.mR2 = f.mandelbox.foldingSphericalMin * f.mandelbox.foldingSphericalMin;
  f.mandelbox.mboxFactor1 = f.mandelbox.fR2 / f.mandelbox.mR2;
  static cFractalMandelbox fb;
  fb.FormulaCode(v, &f, aux);
  f.mandelbox.rotationsEnabled = false;
  f.mandelbox.mainRotationEnabled = false;
  z[0] = v.x;
  z[1] = v.y;
  z[2] = v.z;
  z[3] = v.w;
  *aux_r = aux.r;
  *aux_de = aux.DE;
  return 0;
}

// cCameraTarget(camera, target, top) + the mRot of PrepareMainVectors.
// out: yaw, pitch, roll, then mRot row-major (9).
int ref_camera(const double *cam, const double *target, const double *top, double *out) {
  cCameraTarget ct(CVector3(cam[0], cam[1], cam[2]), CVector3(target[0], target[1], target[2]),
                   CVector3(top[0], top[1], top[2]));
  CVector3 a = ct.GetRotation();
  CRotationMatrix m;
  m.RotateZ(a.x);
  m.RotateX(a.y);
  m.RotateY(a.z);
  out[0] = a.x;
  out[1] = a.y;
  out[2] = a.z;
  CVector3 e[3] = {CVector3(1, 0, 0), CVector3(0, 1, 0), CVector3(0, 0, 1)};
  for (int j = 0; j < 3; j++) {
    CVector3 c = m.RotateVector(e[j]);
    out[3 + 0 * 3 + j] = c.x;
    out[3 + 1 * 3 + j] = c.y;
    out[3 + 2 * 3 + j] = c.z;
  }
  return 0;
}

// View vector of normalised image point (x, y) through CalculateViewVector
// (three-point) with the camera's mRot, then normalised as in doWork.
int ref_view_vector(const double *cam, const double *target, const double *top, double fov_deg, double ix,
                    double iy, double *out) {
  cCameraTarget ct(CVector3(cam[0], cam[1], cam[2]), CVector3(target[0], target[1], target[2]),
                   CVector3(top[0], top[1], top[2]));
  CVector3 a = ct.GetRotation();
  CRotationMatrix m;
  m.RotateZ(a.x);
  m.RotateX(a.y);
  m.RotateY(a.z);
  double fov = CalcFOV(fov_deg, params::perspThreePoint);
  CVector3 v = CalculateViewVector(CVector2<double>(ix, iy), fov, params::perspThreePoint, m);
  v.Normalize();
  out[0] = v.x;
  out[1] = v.y;
  out[2] = v.z;
  return 0;
}

double ref_calc_fov(double fov_deg) { return CalcFOV(fov_deg, params::perspThreePoint); }

// The same for projection `persp` (params::enumPerspectiveType): CalcFOV and
// CalculateViewVector of that projection, then normalised as in doWork.
int ref_view_vector_p(const double *cam, const double *target, const double *top, double fov_deg, int persp,
                      double ix, double iy, double *out) {
  cCameraTarget ct(CVector3(cam[0], cam[1], cam[2]), CVector3(target[0], target[1], target[2]),
                   CVector3(top[0], top[1], top[2]));
  CVector3 a = ct.GetRotation();
  CRotationMatrix m;
  m.RotateZ(a.x);
  m.RotateX(a.y);
  m.RotateY(a.z);
  const params::enumPerspectiveType pt = params::enumPerspectiveType(persp);
  double fov = CalcFOV(fov_deg, pt);
  CVector3 v = CalculateViewVector(CVector2<double>(ix, iy), fov, pt, m);
  v.Normalize();
  out[0] = v.x;
  out[1] = v.y;
  out[2] = v.z;
  return 0;
}

double ref_calc_fov_p(double fov_deg, int persp) { return CalcFOV(fov_deg, params::enumPerspectiveType(persp)); }

// n draws of Random(max) from gRandomSeed = seed (max < 0: RandomInt()).
int ref_random(unsigned int seed, int max, int n, int *out) {
  gRandomSeed = seed;
  for (int i = 0; i < n; i++) out[i] = (max < 0) ? RandomInt() : Random(max);
  return 0;
}

}  // extern "C"
