// mbr_host.cpp - host side of the C-ABI (include/mbr.h): context, parameter
// validation, the hybrid-sequence builder, camera set-up and kernel dispatch.
//
// The host work restates what cRenderJob / sParamRender / cHybridFractalSequences
// / cRenderWorker::PrepareMainVectors do before the per-pixel loop:
//   sequence table      src/hybrid_fractal_sequences.cpp:181-499
//   derived parameters  src/fractal.cpp:653-678 (fR2, mR2, mboxFactor1, radians)
//   camera rotation     src/camera_target.cpp:86-130, src/render_worker.cpp:539-564
//   fov, resolution     src/projection_3d.cpp:140-159, src/render_job.cpp:477
//   gamma table         src/cimage.cpp:366-375
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../include/mbr.h"
#include "mbr_device.h"
#include "mbr_internal.h"

using namespace mbr;

namespace {

const double kPi = 3.14159265358979323846;

struct FormulaMeta {
  int de_function;   // enumDEFunctionType
  int cpixel;        // 0 enabled by default, 1 disabled by default
  double bailout;    // default bailout
  int analytic;      // enumDEAnalyticFunction
  int delta;         // DEType: 1 deltaDEType, 0 analyticDEType
};
// cAbstractFractal metadata of the formula classes (fractal_mandelbulb.cpp:16-27,
// fractal_mandelbulb_power2.cpp:17-28, fractal_hypercomplex.cpp:17-28,
// fractal_mandelbox.cpp:18-29, fractal_menger_sponge.cpp:17-28)
bool formula_meta(int formula, FormulaMeta *m) {
  switch (formula) {
    case MBR_FORMULA_MANDELBULB: *m = {2, 0, 10.0, 2}; return true;
    case MBR_FORMULA_MANDELBULB_POWER2: *m = {2, 0, 10.0, 2}; return true;
    case MBR_FORMULA_HYPERCOMPLEX: *m = {2, 0, 10.0, 2}; return true;
    case MBR_FORMULA_KALEIDOSCOPIC_IFS: *m = {1, 1, 100.0, 3}; return true;  // fractal_kaleidoscopic_ifs.cpp:17-28
    case MBR_FORMULA_XENODREAMBUIE: *m = {2, 0, 10.0, 2}; return true;       // fractal_xenodreambuie.cpp:17-28
    case MBR_FORMULA_QUATERNION: *m = {2, 0, 10.0, 2}; return true;          // fractal_quaternion.cpp:16-27
    case MBR_FORMULA_AEXION: *m = {2, 2, 10000.0, 2}; return true;           // fractal_aexion.cpp:16-27
    case MBR_FORMULA_MANDELBOX: *m = {1, 0, 100.0, 1}; return true;
    case MBR_FORMULA_MENGER_SPONGE: *m = {1, 1, 10.0, 3}; return true;
    case MBR_FORMULA_PSEUDO_KLEINIAN: *m = {3, 1, 100.0, 4}; return true;  // fractal_pseudo_kleinian.cpp:17-28
    case MBR_FORMULA_BOX_FOLD_BULB_POW2: *m = {1, 0, 10000.0, 1, 1}; return true;  // fractal_box_fold_bulb_pow2.cpp:14-25
    case MBR_FORMULA_MENGER_MOD1: *m = {1, 1, 10.0, 3}; return true;  // fractal_menger_mod1.cpp:16-27
    case MBR_FORMULA_BOX_FOLD_BULB_POW2_V2: *m = {2, 0, 100.0, 2}; return true;  // fractal_box_fold_bulb_pow2_v2.cpp:16-27
    case MBR_FORMULA_ABOX_MOD11: *m = {1, 0, 100.0, 1}; return true;  // fractal_abox_mod11.cpp:21-32
    case MBR_FORMULA_PSEUDO_KLEINIAN_MOD4: *m = {3, 1, 100.0, 4}; return true;  // fractal_pseudo_kleinian_mod4.cpp:17-28
    case MBR_FORMULA_PSEUDO_KLEINIAN_STD_DE: *m = {5, 1, 100.0, 6}; return true;  // fractal_pseudo_kleinian_std_de.cpp:16-27
    case MBR_FORMULA_GENERALIZED_FOLD_BOX: *m = {1, 0, 100.0, 1}; return true;  // fractal_generalized_fold_box.cpp:17-29
    case MBR_FORMULA_MANDELBULB_PUPUKU: *m = {2, 0, 10.0, 2}; return true;  // fractal_mandelbulb_pupuku.cpp:16-27
    case MBR_FORMULA_DIFS_HEXTGRID2: *m = {5, 1, 100.0, 6}; return true;  // fractal_difs_hextgrid2.cpp:18-29
    default: return false;
  }
}

bool finite3(const double *v) { return std::isfinite(v[0]) && std::isfinite(v[1]) && std::isfinite(v[2]); }

}  // namespace

struct mbr_ctx {
  int device = 0;
  std::string err;
  bool has_scene = false;
  DevScene scene;
  mbr_scene scene_src;
  uint16_t *d_gamma = nullptr;
  uint16_t *h_gamma = nullptr;      // pinned staging table of the gamma copies
  cudaEvent_t gamma_evt = nullptr;  // recorded after the last gamma copy
  double gamma_value = -1.0;
  int32_t *d_status = nullptr;
  mbr_tuning tuning{128, 12, 2, 0};  // fastest on the 1920x1080 Mandelbox of the autotuner grid
  // scratch of the wavefront kernel (work counter + per-lane queue cursor)
  unsigned long long *d_work = nullptr;
  size_t work_words = 0;
  void *adjoint_scratch = nullptr;  // the adjoint's per-block partial sums
  size_t adjoint_scratch_bytes = 0;
};

namespace mbr {

mbr_status set_err(mbr_ctx *ctx, mbr_status st, const char *fmt, ...) {
  if (ctx) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    ctx->err = buf;
  }
  return st;
}

mbr_status cuda_err(mbr_ctx *ctx, int code, const char *what) {
  if (code == 0) return MBR_OK;
  return set_err(ctx, MBR_ECUDA, "%s: %s", what, cudaGetErrorString(cudaError_t(code)));
}

// The matrix of CRotationMatrix::SetRotation2(angles_deg * M_PI_180)
// (fractal.cpp:663, 669; algebra.cpp:296-302, 198-247): from the identity,
// rotations about z, y and x by the vector's z, y and x angles, each
// multiplied onto the right and skipped for a zero angle; *zero is set when
// all three are zero (RotateVector then returns its argument unchanged).
// set3: CRotationMatrix::SetRotation3 instead (algebra.cpp:304-310):
// rotations about z, y and x by the vector's x, y and z angles.
static void mandelbox_rotation(const double deg[3], double m[9], bool *zero, bool set3 = false) {
  const double k = 0.01745329251994329576923690768489;  // M_PI_180 (fractal.h:45-46)
  for (int i = 0; i < 9; i++) m[i] = (i % 4 == 0) ? 1.0 : 0.0;
  *zero = true;
  for (int axis = 2; axis >= 0; axis--) {
    const double a = deg[set3 ? 2 - axis : axis] * k;
    if (a == 0.0) continue;
    const double sn = std::sin(a), cs = std::cos(a);
    double r[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    if (axis == 0) { r[0] = 1.0; r[4] = cs; r[8] = cs; r[5] = -sn; r[7] = sn; }
    if (axis == 1) { r[4] = 1.0; r[8] = cs; r[0] = cs; r[6] = -sn; r[2] = sn; }
    if (axis == 2) { r[8] = 1.0; r[0] = cs; r[4] = cs; r[1] = -sn; r[3] = sn; }
    double t[9];
    for (int row = 0; row < 3; row++)
      for (int col = 0; col < 3; col++)
        t[row * 3 + col] = m[row * 3 + 0] * r[col] + m[row * 3 + 1] * r[3 + col] + m[row * 3 + 2] * r[6 + col];
    std::memcpy(m, t, sizeof(t));
    *zero = false;
  }
}

static void rotate_axis(double *m, bool *zero, int axis, double angle);

static const double kIdentity44[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};

// A node's localToWorld under its parent's (objects_tree.cpp:285-330):
// W = P * [R^T s | t], R from SetRotation2(rotation * pi/180), row-major 4x4.
static void node_world(const double P[16], const double pos[3], const double rot[3], double scale, double W[16]) {
  double R[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  bool zero = true;
  const double k = kPi / 180.0;
  rotate_axis(R, &zero, 2, rot[2] * k);
  rotate_axis(R, &zero, 1, rot[1] * k);
  rotate_axis(R, &zero, 0, rot[0] * k);
  const double L[16] = {R[0] * scale, R[3] * scale, R[6] * scale, pos[0],  //
                        R[1] * scale, R[4] * scale, R[7] * scale, pos[1],  //
                        R[2] * scale, R[5] * scale, R[8] * scale, pos[2],  //
                        0.0,          0.0,          0.0,          1.0};
  for (int r = 0; r < 4; r++)
    for (int c = 0; c < 4; c++)
      W[r * 4 + c] = P[r * 4 + 0] * L[c] + P[r * 4 + 1] * L[4 + c] + P[r * 4 + 2] * L[8 + c] + P[r * 4 + 3] * L[12 + c];
}

// CMatrix44::InverseAffine (algebra.cpp:528-576) of W into rows 1-3 of m
// (m must hold zeros), and the world scale |first row of W|
static void world_to_local(const double W[16], double m[12], double *abs_scale) {
  const double ws = std::sqrt(W[0] * W[0] + W[1] * W[1] + W[2] * W[2]);
  const double s2 = ws * ws;
  if (ws > 1e-12) {
    m[0] = W[0] / s2;
    m[1] = W[4] / s2;
    m[2] = W[8] / s2;
    m[4] = W[1] / s2;
    m[5] = W[5] / s2;
    m[6] = W[9] / s2;
    m[8] = W[2] / s2;
    m[9] = W[6] / s2;
    m[10] = W[10] / s2;
  }
  const double tx = W[3], ty = W[7], tz = W[11];
  m[3] = -(W[0] * tx + W[4] * ty + W[8] * tz) / s2;
  m[7] = -(W[1] * tx + W[5] * ty + W[9] * tz) / s2;
  m[11] = -(W[2] * tx + W[6] * ty + W[10] * tz) / s2;
  *abs_scale = std::fabs(ws);
}

// A primitive's node as the distance reads it: localToWorld = [R^T s | t] with
// R from SetRotation2(rotation * pi/180), accumulated under the parent
// transform P (identity groups for the default objects tree), then
// InverseAffine (objects_tree.cpp:290-385, algebra.cpp:477-576).
static bool build_prim(const mbr_primitive &q, DevPrim *o, const double P[16] = kIdentity44) {
  std::memset(o, 0, sizeof(*o));
  const bool finite = finite3(q.position) && finite3(q.rotation) && finite3(q.repeat) && finite3(q.size) &&
                      finite3(q.limits_min) && finite3(q.limits_max) && std::isfinite(q.scale) &&
                      std::isfinite(q.radius) && std::isfinite(q.height) && std::isfinite(q.width) &&
                      std::isfinite(q.tube_radius) && std::isfinite(q.radius_lpow) &&
                      std::isfinite(q.tube_radius_lpow) && std::isfinite(q.rounding) &&
                      std::isfinite(q.wall_thickness) && std::isfinite(q.relative_amplitude) &&
                      std::isfinite(q.length) && std::isfinite(q.anim_speed) &&
                      std::isfinite(q.anim_progression_speed) && std::isfinite(q.prism_angle) &&
                      std::isfinite(q.triangle_height);
  if (!finite || !(std::fabs(q.scale) > 1e-12) || q.type < MBR_PRIMITIVE_PLANE || q.type > MBR_PRIMITIVE_ELLIPSOID ||
      q.iterations < 0 || q.iterations > 100)
    return false;
  if (q.type == MBR_PRIMITIVE_CONE && !(q.height != 0.0)) return false;
  if (q.type == MBR_PRIMITIVE_ELLIPSOID && !(q.size[0] != 0.0 && q.size[1] != 0.0 && q.size[2] != 0.0)) return false;
  if (q.type == MBR_PRIMITIVE_WATER && !(q.length != 0.0)) return false;
  double W[16];
  node_world(P, q.position, q.rotation, q.scale, W);
  world_to_local(W, o->m, &o->abs_scale);
  for (int i = 0; i < 3; i++) o->repeat[i] = q.repeat[i] / o->abs_scale;
  o->has_repeat = std::sqrt(o->repeat[0] * o->repeat[0] + o->repeat[1] * o->repeat[1] + o->repeat[2] * o->repeat[2]) > 0.0;
  o->type = q.type;
  o->empty = q.empty ? 1 : 0;
  // the plane, circle, rectangle and prism have no limits box (primitive.cpp:459-465, 513-520, 539-545, 657-668)
  o->limits = (q.limits_enable && q.type != MBR_PRIMITIVE_PLANE && q.type != MBR_PRIMITIVE_CIRCLE &&
               q.type != MBR_PRIMITIVE_RECTANGLE && q.type != MBR_PRIMITIVE_PRISM)
                  ? 1
                  : 0;
  o->caps = q.caps ? 1 : 0;
  o->iterations = q.iterations;
  for (int i = 0; i < 3; i++) {
    o->size[i] = q.size[i];
    o->lmin[i] = q.limits_min[i];
    o->lmax[i] = q.limits_max[i];
  }
  o->radius = q.radius;
  o->height = q.height;
  o->width = q.width;
  o->tube = q.tube_radius;
  o->pow_r = std::pow(2.0, q.radius_lpow);
  o->pow_t = std::pow(2.0, q.tube_radius_lpow);
  o->rounding = q.rounding;
  o->wall = q.wall_thickness;
  // water (primitive.cpp:172-191, 583-603)
  o->amp = q.length * q.relative_amplitude;
  o->length = q.length;
  o->phase = -q.anim_speed * double(q.frame_no) * 0.1;
  o->xshift = o->phase * 0.05 * (q.anim_progression_speed * 3.0 - 3.0);
  // cone: wallNormal = (1, radius / height), CVector2::Normalize (primitive.cpp:222-237, algebra.hpp:566-572)
  o->wn[0] = 1.0;
  o->wn[1] = q.type == MBR_PRIMITIVE_CONE ? q.radius / q.height : 0.0;
  {
    const double norm = 1.0 / std::sqrt(o->wn[0] * o->wn[0] + o->wn[1] * o->wn[1]);
    o->wn[0] = o->wn[0] * norm;
    o->wn[1] = o->wn[1] * norm;
  }
  // prism (primitive.cpp:380-393): half height, half angle, triangle height
  if (q.type == MBR_PRIMITIVE_PRISM) {
    o->height = q.height / 2.0;
    const double a = q.prism_angle * kPi / 180.0 / 2.0;
    o->tri = q.triangle_height * std::sin(a);
    o->pn[0] = std::sin(a);
    o->pn[1] = std::cos(a);
    o->pn[2] = std::sin(a);
  }
  return true;
}

// ---- explicit objects tree -----------------------------------------------------
// The node list's shape (cObjectsTree, objects_tree.cpp:185-245): levels
// start at 0 and go down by at most one per node, only a boolean group has
// children, a disabled node drops its subtree.  live[i]: node i is walked.
static mbr_status tree_shape(mbr_ctx *ctx, const mbr_scene &sc, bool live[MBR_MAX_NODES]) {
  int skip = -1, prev_level = -1;
  bool prev_group = false;
  for (int i = 0; i < sc.n_nodes; i++) {
    const mbr_node &q = sc.node[i];
    const bool group =
        q.type == MBR_NODE_BOOLEAN_ADD || q.type == MBR_NODE_BOOLEAN_MUL || q.type == MBR_NODE_BOOLEAN_SUB;
    if (!group && q.type != MBR_NODE_FRACTAL && q.type != MBR_NODE_PRIMITIVE)
      return set_err(ctx, MBR_EINVAL, "node %d: type must be FRACTAL, PRIMITIVE or a boolean group, got %d", i,
                     q.type);
    if (q.level < 0 || q.level > 8 || q.level > prev_level + 1)
      return set_err(ctx, MBR_EINVAL, "node %d: level must be in [0, 8] and at most one below the node before", i);
    if (q.level == prev_level + 1 && i > 0 && !prev_group)
      return set_err(ctx, MBR_EINVAL, "node %d: only a boolean group has children", i);
    prev_level = q.level;
    prev_group = group;
    if (skip >= 0 && q.level > skip) continue;
    skip = -1;
    if (!q.enabled) {
      skip = q.level;
      continue;
    }
    if (q.type == MBR_NODE_FRACTAL && (q.index < 0 || q.index >= sc.n_fractals))
      return set_err(ctx, MBR_EINVAL, "node %d: fractal index must be in [0, n_fractals)", i);
    if (q.type == MBR_NODE_PRIMITIVE && (q.index < 0 || q.index >= sc.n_primitives))
      return set_err(ctx, MBR_EINVAL, "node %d: primitive index must be in [0, n_primitives)", i);
    if (!finite3(q.position) || !finite3(q.rotation) || !finite3(q.repeat) || !std::isfinite(q.scale) ||
        !std::isfinite(q.detail_level_multiplier) || !std::isfinite(q.smooth_combine_distance) ||
        !finite3(q.julia_c) || !finite3(q.fractal_constant_factor) || !std::isfinite(q.initial_waxis))
      return set_err(ctx, MBR_EINVAL, "node %d: non-finite value", i);
    if (group || q.type == MBR_NODE_FRACTAL) {
      if (!(std::fabs(q.scale) > 1e-12)) return set_err(ctx, MBR_EINVAL, "node %d: |scale| must be > 1e-12", i);
    }
    if (q.smooth_combine && !(q.smooth_combine_distance != 0.0))
      return set_err(ctx, MBR_EINVAL, "node %d: smooth_combine_distance must be non-zero", i);
    if (q.type == MBR_NODE_FRACTAL && (q.formula_maxiter < 1 || q.formula_maxiter > 9999))
      return set_err(ctx, MBR_EINVAL, "node %d: formula_maxiter must be in [1, 9999]", i);
    live[i] = true;
  }
  return MBR_OK;
}

// cObjectsTree::GetNodeDataListForRendering (objects_tree.cpp:185-410) into
// the scene: per walked node its world matrix (the parent's times its own)
// inverted, |world scale|, repeat / |world scale|; a fractal node's slot with
// the sequence settings CreateSequence gives a non-hybrid node (iteration
// limit, julia, constant factor, w, DE selection, hybrid_fractal_sequences.cpp:
// 377-500); a primitive node's record in d->prim under the accumulated
// transform (one record per primitive node).
static mbr_status build_tree(mbr_ctx *ctx, const mbr_scene &sc, const bool live[MBR_MAX_NODES], DevScene *d) {
  double Wl[9][16];
  int nn = 0, np = 0;
  for (int i = 0; i < sc.n_nodes; i++) {
    if (!live[i]) continue;
    const mbr_node &q = sc.node[i];
    DevNode &o = d->node[nn];
    std::memset(&o, 0, sizeof(o));
    o.type = q.type;
    o.level = q.level;
    o.smooth = q.smooth_combine ? 1 : 0;
    o.smooth_dist = q.smooth_combine_distance;
    o.detail_mult = q.detail_level_multiplier;
    const double *P = (q.level == 0) ? kIdentity44 : Wl[q.level - 1];
    if (q.type == MBR_NODE_PRIMITIVE) {
      if (np >= MBR_MAX_PRIMITIVES)
        return set_err(ctx, MBR_EUNSUPPORTED, "an objects tree holds at most %d primitive nodes", MBR_MAX_PRIMITIVES);
      const mbr_primitive &pq = sc.primitive[q.index];
      if (!build_prim(pq, &d->prim[np], P))
        return set_err(ctx, MBR_EINVAL,
                       "primitive %d: type must be 1..8, every value finite, |scale| > 1e-12, iterations in "
                       "[0, 100] and a water length != 0",
                       q.index);
      node_world(P, pq.position, pq.rotation, pq.scale, Wl[q.level]);
      const DevPrim &pr = d->prim[np];
      for (int k = 0; k < 12; k++) o.w2l[k] = pr.m[k];
      o.abs_scale = pr.abs_scale;
      for (int k = 0; k < 3; k++) o.repeat[k] = pr.repeat[k];
      o.has_repeat = pr.has_repeat;
      o.prim = np++;
    } else {
      node_world(P, q.position, q.rotation, q.scale, Wl[q.level]);
      world_to_local(Wl[q.level], o.w2l, &o.abs_scale);
      for (int k = 0; k < 3; k++) o.repeat[k] = q.repeat[k] / o.abs_scale;
      o.has_repeat =
          std::sqrt(o.repeat[0] * o.repeat[0] + o.repeat[1] * o.repeat[1] + o.repeat[2] * o.repeat[2]) > 0.0;
    }
    if (q.type == MBR_NODE_FRACTAL) {
      const int slot = q.index;
      FormulaMeta m;
      formula_meta(d->slot[slot].formula, &m);  // validated with the slots
      o.slot = slot;
      o.maxN = q.formula_maxiter;
      o.julia = q.julia_mode ? 1 : 0;
      for (int k = 0; k < 3; k++) {
        o.julia_c[k] = q.julia_c[k];
        o.cmul[k] = q.fractal_constant_factor[k];
        o.fcmul[k] = float(q.fractal_constant_factor[k]);
      }
      o.w0 = q.initial_waxis;
      const int f = d->slot[slot].formula;
      o.has_w = (q.initial_waxis != 0.0 || f == MBR_FORMULA_HYPERCOMPLEX || f == MBR_FORMULA_AEXION) ? 1 : 0;
      if (o.has_w) d->has_w = 1;
      int de_function = m.de_function, de_analytic = m.analytic;
      if (sc.delta_de_function != MBR_DE_FUNCTION_PREFERRED) {
        static const int fn_analytic[7] = {1, 1, 2, 4, 5, 6, 7};  // enumDEAnalyticFunction
        de_function = sc.delta_de_function;
        de_analytic = fn_analytic[de_function];
      }
      static const int an_final[8] = {DEF_NONE, DEF_LINEAR, DEF_LOG, DEF_IFS, DEF_PSEUDO_KLEINIAN, 0, DEF_CUSTOM,
                                      DEF_MAX_AXIS};
      o.de_analytic = de_analytic;
      o.de_final = an_final[de_analytic];
      // DEType and the forcing switches (hybrid_fractal_sequences.cpp:466-474)
      o.delta_de = (m.delta || sc.delta_de_method == MBR_DE_METHOD_FORCE_DELTA) &&
                   sc.delta_de_method != MBR_DE_METHOD_FORCE_ANALYTIC;
      o.delta_fn = de_function;
      if (!o.delta_de && o.de_final == 0)
        return set_err(ctx, MBR_EUNSUPPORTED,
                       "node %d: the analytic Jos Kleinian DE function reads formula parameters this build does "
                       "not carry (the delta DE takes it)",
                       i);
    }
    nn++;
  }
  if (nn == 0) return set_err(ctx, MBR_EINVAL, "every node of the objects tree is disabled");
  d->n_nodes = nn;
  d->n_prims = np;
  d->generic = 1;  // the tree is walked by the reference-order iteration only
  return MBR_OK;
}

// ---- scene -------------------------------------------------------------------
// Validates `sc` and flattens it into a DevScene.  Restates CollectSequenceData
// and CreateSequence for the single fractal (or hybrid) node of the default
// objects tree.
mbr_status build_scene(mbr_ctx *ctx, const mbr_scene &sc, DevScene *out) {
  DevScene d;
  std::memset(&d, 0, sizeof(d));
  const bool hybrid = sc.hybrid_fractal_enable != 0;
  const int n = hybrid ? sc.n_fractals : 1;
  if (sc.n_fractals < 1 || sc.n_fractals > MBR_MAX_FRACTALS)
    return set_err(ctx, MBR_EINVAL, "n_fractals must be in [1, %d], got %d", MBR_MAX_FRACTALS, sc.n_fractals);
  if (sc.formula_maxiter < 1 || sc.formula_maxiter > 9999)
    return set_err(ctx, MBR_EINVAL, "formula_maxiter must be in [1, 9999], got %d", sc.formula_maxiter);
  if (sc.repeat_from < 1 || sc.repeat_from > MBR_MAX_FRACTALS)
    return set_err(ctx, MBR_EINVAL, "repeat_from must be in [1, 9], got %d", sc.repeat_from);
  if (sc.min_n < 0) return set_err(ctx, MBR_EINVAL, "min_n must be >= 0");
  if (!sc.use_default_bailout && !(sc.bailout > 0.0))
    return set_err(ctx, MBR_EINVAL, "bailout must be > 0");
  if (!finite3(sc.julia_c) || !finite3(sc.fractal_constant_factor) || !std::isfinite(sc.initial_waxis) ||
      !std::isfinite(sc.linear_de_offset))
    return set_err(ctx, MBR_EINVAL, "non-finite scene vector");
  if (sc.delta_de_function < MBR_DE_FUNCTION_PREFERRED || sc.delta_de_function > MBR_DE_FUNCTION_MAX_AXIS)
    return set_err(ctx, MBR_EINVAL, "delta_de_function must be in [0, 6], got %d", sc.delta_de_function);
  if (sc.delta_de_method < MBR_DE_METHOD_PREFERRED || sc.delta_de_method > MBR_DE_METHOD_FORCE_ANALYTIC)
    return set_err(ctx, MBR_EINVAL, "delta_de_method must be in [0, 2], got %d", sc.delta_de_method);
  if (!(sc.deltade_relative_delta > 0.0) || !std::isfinite(sc.deltade_relative_delta))
    return set_err(ctx, MBR_EINVAL, "deltade_relative_delta must be finite and > 0");
  // the slots the scene iterates: the fractal (or the hybrid sequence's
  // slots) of the default objects tree, or the slots that the enabled fractal
  // nodes of an explicit tree name
  if (sc.n_nodes < 0 || sc.n_nodes > MBR_MAX_NODES)
    return set_err(ctx, MBR_EINVAL, "n_nodes must be in [0, %d], got %d", MBR_MAX_NODES, sc.n_nodes);
  const bool tree = sc.n_nodes > 0;
  if (tree && hybrid)
    return set_err(ctx, MBR_EUNSUPPORTED, "an explicit objects tree takes non-hybrid fractal nodes");
  bool used[MBR_MAX_FRACTALS] = {};
  for (int i = 0; i < (hybrid ? n : 1); i++) used[i] = true;
  bool live[MBR_MAX_NODES] = {};
  if (tree) {
    mbr_status st = tree_shape(ctx, sc, live);
    if (st != MBR_OK) return st;
    for (int i = 0; i < sc.n_nodes; i++)
      if (live[i] && sc.node[i].type == MBR_NODE_FRACTAL) used[sc.node[i].index] = true;
  }
  // Mandelbox rotations and the kaleidoscopic IFS: the scene holds one block
  // of each, for its single Mandelbox slot and its single IFS slot
  int n_box = 0, n_ifs = 0;
  for (int i = 0; i < MBR_MAX_FRACTALS; i++) {
    if (!used[i]) continue;
    if (sc.fractal[i].formula == MBR_FORMULA_MANDELBOX) n_box++;
    if (sc.fractal[i].formula == MBR_FORMULA_KALEIDOSCOPIC_IFS) n_ifs++;
  }
  for (int i = 0; i < MBR_MAX_FRACTALS; i++) {
    if (!used[i]) continue;
    const mbr_fractal &f = sc.fractal[i];
    const bool rot = f.mandelbox_rotations_enabled || f.mandelbox_main_rotation_enabled;
    if (!rot || f.formula != MBR_FORMULA_MANDELBOX) continue;
    if (n_box > 1)
      return set_err(ctx, MBR_EUNSUPPORTED,
                     "Mandelbox rotations are supported when the scene iterates one Mandelbox slot");
    bool ok = finite3(f.mandelbox_rotation_main);
    for (int a = 0; a < 3; a++) ok = ok && finite3(f.mandelbox_rotation_neg[a]) && finite3(f.mandelbox_rotation_pos[a]);
    if (!ok) return set_err(ctx, MBR_EINVAL, "non-finite Mandelbox rotation angle");
    MbRot &r = d.mbrot;
    r.folds = f.mandelbox_rotations_enabled ? 1 : 0;
    r.main = f.mandelbox_main_rotation_enabled ? 1 : 0;
    bool zero;
    for (int a = 0; a < 3; a++) {
      mandelbox_rotation(f.mandelbox_rotation_neg[a], r.m[0][a], &zero);
      r.zero[0][a] = zero ? 1 : 0;
      mandelbox_rotation(f.mandelbox_rotation_pos[a], r.m[1][a], &zero);
      r.zero[1][a] = zero ? 1 : 0;
    }
    mandelbox_rotation(f.mandelbox_rotation_main, r.mm, &zero);
    r.main_zero = zero ? 1 : 0;
  }
  for (int i = 0; i < MBR_MAX_FRACTALS; i++) {
    if (!used[i]) continue;
    const mbr_fractal &f = sc.fractal[i];
    if (f.formula != MBR_FORMULA_KALEIDOSCOPIC_IFS) continue;
    if (n_ifs > 1)
      return set_err(ctx, MBR_EUNSUPPORTED, "the kaleidoscopic IFS is supported in one slot of a scene");
    IfsBlock &b = d.ifs;
    b.abs_x = f.ifs_abs_x ? 1 : 0;
    b.abs_y = f.ifs_abs_y ? 1 : 0;
    b.abs_z = f.ifs_abs_z ? 1 : 0;
    b.menger = f.ifs_menger_sponge_mode ? 1 : 0;
    b.rot_on = f.ifs_rotation_enabled ? 1 : 0;
    b.edge_on = f.ifs_edge_enabled ? 1 : 0;
    b.scale = f.ifs_scale;
    for (int k = 0; k < 3; k++) {
      b.offset[k] = f.ifs_offset[k];
      b.edge[k] = f.ifs_edge[k];
    }
    bool zero;
    mandelbox_rotation(f.ifs_rotation, b.main, &zero, true);
    b.main_zero = zero ? 1 : 0;
    b.n = 0;
    for (int v = 0; v < 9; v++) {
      if (!f.ifs_enabled[v]) continue;
      const int j = b.n++;
      mandelbox_rotation(f.ifs_rotations[v], b.rot[j], &zero, true);
      b.rot_zero[j] = zero ? 1 : 0;
      // CVector4(direction, 0), normalised when read and again when derived (fractal.cpp:110-115, 660)
      double x = f.ifs_direction[v][0], y = f.ifs_direction[v][1], z = f.ifs_direction[v][2];
      for (int rep = 0; rep < 2; rep++) {
        const double norm = 1.0 / std::sqrt(x * x + y * y + z * z + 0.0 * 0.0);
        x = x * norm;
        y = y * norm;
        z = z * norm;
      }
      b.dir[j][0] = x;
      b.dir[j][1] = y;
      b.dir[j][2] = z;
      b.dist[j] = f.ifs_distance[v];
      b.inten[j] = f.ifs_intensity[v];
    }
  }
  d.n = n;
  d.is_hybrid = hybrid ? 1 : 0;
  double maxBailout = 0.0;
  bool any = false;
  for (int i = 0; i < MBR_MAX_FRACTALS; i++) {
    if (!used[i]) continue;
    const mbr_fractal &f = sc.fractal[i];
    DevSlot &s = d.slot[i];
    s.formula = f.formula;
    if (f.formula == MBR_FORMULA_NONE && hybrid) {
      s.check_bailout = 1;
      continue;
    }
    FormulaMeta m;
    if (!formula_meta(f.formula, &m))
      return set_err(ctx, MBR_EUNSUPPORTED,
                     "slot %d: formula %d is not supported (2, 3, 4, 5, 7, 8, 10, 11, 16, 19, 37, 61, 101, 103, 119, 125, 217, 266, 608)", i, f.formula);
    any = true;
    if (f.formula_iterations < 1) return set_err(ctx, MBR_EINVAL, "slot %d: formula_iterations < 1", i);
    if (f.formula_start_iteration < 0 || f.formula_stop_iteration < 0)
      return set_err(ctx, MBR_EINVAL, "slot %d: negative start/stop iteration", i);
    if (!(f.formula_weight >= 0.0 && f.formula_weight <= 1.0))
      return set_err(ctx, MBR_EINVAL, "slot %d: formula_weight must be in [0, 1]", i);
    if (f.formula == MBR_FORMULA_MANDELBULB && !std::isfinite(f.bulb_power))
      return set_err(ctx, MBR_EINVAL, "slot %d: non-finite power", i);
    if (f.formula == MBR_FORMULA_MANDELBOX) {
      if (!(f.mandelbox_folding_limit >= 0.0))
        return set_err(ctx, MBR_EINVAL, "slot %d: mandelbox_folding_limit must be >= 0", i);
      if (!(f.mandelbox_folding_min_radius > 0.0) || !(f.mandelbox_folding_fixed_radius >= 0.0))
        return set_err(ctx, MBR_EINVAL, "slot %d: mandelbox radii must be min > 0, fixed >= 0", i);
      if (!std::isfinite(f.mandelbox_scale) || !std::isfinite(f.mandelbox_folding_value) || !finite3(f.mandelbox_offset))
        return set_err(ctx, MBR_EINVAL, "slot %d: non-finite mandelbox parameter", i);
    }
    if (f.formula == MBR_FORMULA_MENGER_SPONGE && !std::isfinite(f.transf_scale3))
      return set_err(ctx, MBR_EINVAL, "slot %d: non-finite scale3", i);
    // checkForBailout and the c-constant rule (hybrid_fractal_sequences.cpp:199-215)
    s.check_bailout = hybrid ? (f.check_for_bailout != 0) : 1;
    bool addc = f.dont_add_c_constant == 0;
    if (m.cpixel == 1) addc = !addc;
    if (m.cpixel == 2) addc = false;  // cpixelAlreadyHas: the formula adds c itself (:209-212)
    s.add_c = addc ? 1 : 0;
    s.add_bail = (m.de_function == 3 || m.de_function == 4) ? 1 : 0;  // hybrid_fractal_sequences.cpp:242-246
    double bailout;
    if (sc.use_default_bailout) {
      bailout = m.bailout;
      if (hybrid) maxBailout = std::max(maxBailout, m.bailout);
    } else {
      bailout = sc.bailout;
    }
    // sFractal::RecalculateFractalParams (fractal.cpp:673-678)
    const double deg = 0.01745329251994329576923690768489;
    double *p = s.d;
    p[P_POWER] = f.bulb_power;
    p[P_POWER_M1] = f.bulb_power - 1.0;
    p[P_ALPHA] = f.bulb_alpha_angle_offset * deg;
    p[P_BETA] = f.bulb_beta_angle_offset * deg;
    p[P_MB_SCALE] = f.mandelbox_scale;
    p[P_MB_ABS_SCALE] = std::fabs(f.mandelbox_scale);
    p[P_MB_LIMIT] = f.mandelbox_folding_limit;
    p[P_MB_VALUE] = f.mandelbox_folding_value;
    p[P_MB_FR2] = f.mandelbox_folding_fixed_radius * f.mandelbox_folding_fixed_radius;
    p[P_MB_MR2] = f.mandelbox_folding_min_radius * f.mandelbox_folding_min_radius;
    p[P_MB_FACTOR1] = p[P_MB_FR2] / p[P_MB_MR2];
    p[P_MB_OFF_X] = f.mandelbox_offset[0];
    p[P_MB_OFF_Y] = f.mandelbox_offset[1];
    p[P_MB_OFF_Z] = f.mandelbox_offset[2];
    p[P_SCALE3] = f.transf_scale3;
    p[P_BAILOUT] = bailout;
    p[P_WEIGHT] = f.formula_weight;
    p[P_AEX_CADD] = f.aexion_cadd;
    p[P_ADE_ON] = f.analytic_de_enabled ? 1.0 : 0.0;
    p[P_ADE_SCALE1] = f.analytic_de_scale1;
    p[P_ADE_OFFSET1] = f.analytic_de_offset1;
    s.has_offset = (f.mandelbox_offset[0] != 0.0 || f.mandelbox_offset[1] != 0.0 || f.mandelbox_offset[2] != 0.0);
    // the keyed parameters (formula_params.h); any other formula takes none
    const int bad = pack_keyed(f, s.x);
    if (bad == -2) return set_err(ctx, MBR_EINVAL, "slot %d: n_params must be in [0, %d]", i, MBR_MAX_FORMULA_PARAMS);
    if (bad >= 0)
      return set_err(ctx, MBR_EINVAL,
                     "slot %d: param[%d] (\"%.*s\") is not a parameter formula %d reads, or its value is not "
                     "finite (an int within 32 bits)",
                     i, bad, MBR_PARAM_KEY_LEN, f.param[bad].key, f.formula);
  }
  if (!any) return set_err(ctx, MBR_EINVAL, "scene has no formula");
  if (hybrid && sc.use_default_bailout)
    for (int i = 0; i < n; i++) d.slot[i].d[P_BAILOUT] = maxBailout;
  for (int i = 0; i < MBR_MAX_FRACTALS; i++)
    for (int k = 0; k < P_COUNT; k++) d.slot[i].f[k] = float(d.slot[i].d[k]);

  // the sequence (hybrid_fractal_sequences.cpp:296-370)
  int length = MBR_SEQUENCE_LENGTH;
  const int repeatFromIndex = std::max(0, std::min(sc.repeat_from - 1, n - 1));
  int k = 0, counter = 0, last = 0;
  bool rapidEnd = false;
  for (int i = 0; i < length; i++) {
    counter++;
    int search = 0;
    while ((d.slot[k].formula == MBR_FORMULA_NONE || i < sc.fractal[k].formula_start_iteration ||
            i > sc.fractal[k].formula_stop_iteration) &&
           search < n) {
      k++;
      if (k >= n) k = repeatFromIndex;
      search++;
    }
    if (search >= n) {
      rapidEnd = true;
      break;
    }
    d.seq[i] = uint8_t(k);
    last = i;
    const int iters = hybrid ? sc.fractal[k].formula_iterations : sc.fractal[0].formula_iterations;
    if (counter >= iters) {
      counter = 0;
      k++;
      if (k >= n) k = repeatFromIndex;
    }
  }
  if (rapidEnd) length = last + 1;
  d.length = length;

  // DE function (hybrid_fractal_sequences.cpp:377-485)
  if (hybrid) {
    if (sc.delta_de_function == MBR_DE_FUNCTION_PREFERRED) {
      int count[7] = {0, 0, 0, 0, 0, 0, 0};
      for (int i = 0; i < n; i++) {
        FormulaMeta m;
        if (formula_meta(d.slot[i].formula, &m)) count[m.de_function] += sc.fractal[i].formula_iterations;
      }
      int maxCount = -1;
      for (int i = 1; i <= 6; i++)
        if (count[i] > maxCount) {
          maxCount = count[i];
          d.de_function = i;
        }
      if (count[MBR_DE_FUNCTION_CUSTOM] > 0) d.de_function = MBR_DE_FUNCTION_CUSTOM;  // a custom-DE formula wins (:425-429)
    } else {
      d.de_function = sc.delta_de_function;
    }
    d.de_analytic = (d.de_function == 2) ? 2 : 1;
    d.uniform_formula = 0;
    // a delta-DE formula in any slot makes the sequence a delta-DE one, and
    // the forcing switches override (:450-464)
    bool any_delta = false;
    for (int i = 0; i < n; i++) {
      FormulaMeta m;
      if (formula_meta(d.slot[i].formula, &m) && m.delta) any_delta = true;
    }
    d.delta_de = (any_delta || sc.delta_de_method == MBR_DE_METHOD_FORCE_DELTA) &&
                 sc.delta_de_method != MBR_DE_METHOD_FORCE_ANALYTIC;
    static const int hyb_final[7] = {0, DEF_LINEAR_OFFSET, DEF_LOG, DEF_PSEUDO_KLEINIAN, 0, DEF_CUSTOM, DEF_MAX_AXIS};
    d.de_final = hyb_final[d.de_function];
  } else {
    FormulaMeta m;
    formula_meta(d.slot[0].formula, &m);
    d.de_function = m.de_function;
    d.de_analytic = m.analytic;
    if (sc.delta_de_function != MBR_DE_FUNCTION_PREFERRED) {  // :477-500
      d.de_function = sc.delta_de_function;
      static const int fn_analytic[7] = {1, 1, 2, 4, 5, 6, 7};  // enumDEAnalyticFunction
      d.de_analytic = fn_analytic[d.de_function];
    }
    // DEType and the forcing switches (:466-474)
    d.delta_de = (m.delta || sc.delta_de_method == MBR_DE_METHOD_FORCE_DELTA) &&
                 sc.delta_de_method != MBR_DE_METHOD_FORCE_ANALYTIC;
    // enumDEAnalyticFunction -> DevDeFinal (Jos Kleinian: 0, refused below)
    static const int an_final[8] = {DEF_NONE, DEF_LINEAR, DEF_LOG, DEF_IFS, DEF_PSEUDO_KLEINIAN, 0, DEF_CUSTOM,
                                    DEF_MAX_AXIS};
    d.de_final = an_final[d.de_analytic];
    d.uniform_formula = d.slot[0].formula;
  }
  if (!d.delta_de && d.de_final == 0)
    return set_err(ctx, MBR_EUNSUPPORTED,
                   "the analytic Jos Kleinian DE function reads formula parameters this build does not carry "
                   "(the delta DE takes it)");
  d.delta_fn = d.de_function;
  d.delta_rel = sc.deltade_relative_delta;
  d.delta_factor = 1e-5;
  d.formula_maxiter = sc.formula_maxiter;
  d.min_n = sc.min_n;
  d.iter_thresh = sc.iteration_threshold_mode ? 1 : 0;
  d.interior = sc.interior_mode ? 1 : 0;
  d.julia = sc.julia_mode ? 1 : 0;
  for (int i = 0; i < 3; i++) {
    d.julia_c[i] = sc.julia_c[i];
    d.cmul[i] = sc.fractal_constant_factor[i];
    d.fjulia_c[i] = float(sc.julia_c[i] * sc.fractal_constant_factor[i]);
    d.fcmul[i] = float(sc.fractal_constant_factor[i]);
  }
  d.w0 = sc.initial_waxis;
  d.has_w = sc.initial_waxis != 0.0;
  for (int i = 0; i < MBR_MAX_FRACTALS; i++) {
    if (!used[i]) continue;
    const int f = d.slot[i].formula;
    if (f == MBR_FORMULA_HYPERCOMPLEX || f == MBR_FORMULA_AEXION) d.has_w = 1;  // z.w evolves from w = 0
    if (f != MBR_FORMULA_NONE && f != MBR_FORMULA_MANDELBULB && f != MBR_FORMULA_MANDELBOX &&
        f != MBR_FORMULA_MENGER_SPONGE)
      d.generic = 1;
  }
  d.linear_de_offset = sc.linear_de_offset;
  d.flinear_de_offset = float(sc.linear_de_offset);
  if (sc.n_primitives < 0 || sc.n_primitives > MBR_MAX_PRIMITIVES)
    return set_err(ctx, MBR_EINVAL, "n_primitives must be in [0, %d], got %d", MBR_MAX_PRIMITIVES, sc.n_primitives);
  for (int k = 0; k < sc.n_primitives; k++)
    if (!build_prim(sc.primitive[k], &d.prim[k]))
      return set_err(ctx, MBR_EINVAL,
                     "primitive %d: type must be 1..8, every value finite, |scale| > 1e-12, iterations in "
                     "[0, 100] and a water length != 0",
                     k);
  d.n_prims = sc.n_primitives;
  if (d.n_prims > 0) d.generic = 1;  // the union is evaluated by the reference-order iteration only
  // limit box (fractparams.cpp:175-177) and global folds (fractparams.cpp:346-351)
  if (!finite3(sc.limit_min) || !finite3(sc.limit_max) || !std::isfinite(sc.box_folding_limit) ||
      !std::isfinite(sc.box_folding_value) || !std::isfinite(sc.spherical_folding_inner) ||
      !std::isfinite(sc.spherical_folding_outer))
    return set_err(ctx, MBR_EINVAL, "non-finite limit box or global fold parameter");
  if (sc.spherical_folding && !(sc.spherical_folding_inner != 0.0))
    return set_err(ctx, MBR_EINVAL, "spherical_folding_inner must be non-zero");
  d.limits = sc.limits_enabled ? 1 : 0;
  d.gbox = sc.box_folding ? 1 : 0;
  d.gsph = sc.spherical_folding ? 1 : 0;
  for (int i = 0; i < 3; i++) {
    d.lim_min[i] = sc.limit_min[i];
    d.lim_max[i] = sc.limit_max[i];
    d.flim_min[i] = float(sc.limit_min[i]);
    d.flim_max[i] = float(sc.limit_max[i]);
  }
  d.gbox_limit = sc.box_folding_limit;
  d.gbox_value = sc.box_folding_value;
  d.gsph_fr2 = sc.spherical_folding_outer * sc.spherical_folding_outer;
  d.gsph_mr2 = sc.spherical_folding_inner * sc.spherical_folding_inner;
  d.fgbox_limit = float(d.gbox_limit);
  d.fgbox_value = float(d.gbox_value);
  d.fgsph_fr2 = float(d.gsph_fr2);
  d.fgsph_mr2 = float(d.gsph_mr2);
  if (d.limits || d.gbox || d.gsph) d.generic = 1;  // the reference-order iteration carries them
  if (d.delta_de || d.de_final > DEF_LINEAR_OFFSET) d.generic = 1;  // so do the delta DE and the other DE functions
  if (tree) {
    mbr_status st = build_tree(ctx, sc, live, &d);
    if (st != MBR_OK) return st;
  }
  *out = d;
  return MBR_OK;
}

// cCameraTarget::SetCameraTargetTop + PrepareMainVectors (restated).
struct HV {
  double x, y, z;
};
static HV hadd(HV a, HV b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
static HV hmul(HV a, double s) { return {a.x * s, a.y * s, a.z * s}; }
static double hdot(HV a, HV b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static HV hcross(HV a, HV v) { return {a.y * v.z - a.z * v.y, -a.x * v.z + a.z * v.x, a.x * v.y - a.y * v.x}; }
static HV hnorm(HV a) {
  const double n = 1.0 / std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z);
  return {a.x * n, a.y * n, a.z * n};
}
static HV hrotate_around(HV v, HV axis, double angle) {  // CVector3::RotateAroundVectorByAngle
  HV r = hmul(v, std::cos(angle));
  r = hadd(r, hmul(hcross(axis, v), std::sin(angle)));
  r = hadd(r, hmul(hmul(axis, hdot(axis, v)), 1 - std::cos(angle)));
  return r;
}
static double correct_angle(double a) { return std::fmod(a + 3 * kPi, 2 * kPi) - kPi; }
static void mat3_mul(const double *a, const double *b, double *r) {
  double t[9];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) t[i * 3 + j] = a[i * 3 + 0] * b[j] + a[i * 3 + 1] * b[3 + j] + a[i * 3 + 2] * b[6 + j];
  std::memcpy(r, t, sizeof(t));
}
static void rotate_axis(double *m, bool *zero, int axis, double angle) {  // CRotationMatrix::RotateX/Y/Z
  if (angle == 0.0) return;
  double r[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  const double s = std::sin(angle), c = std::cos(angle);
  if (axis == 0) { r[0] = 1.0; r[4] = c; r[8] = c; r[5] = -s; r[7] = s; }
  if (axis == 1) { r[4] = 1.0; r[8] = c; r[0] = c; r[6] = -s; r[2] = s; }
  if (axis == 2) { r[8] = 1.0; r[0] = c; r[4] = c; r[1] = -s; r[3] = s; }
  mat3_mul(m, r, m);
  *zero = false;
}

void camera_matrix(const mbr_camera &cam, double mrot[9], bool *zero, double angles[3]) {
  double yaw, pitch, roll;
  if (cam.use_angles) {
    yaw = cam.angles[0];
    pitch = cam.angles[1];
    roll = cam.angles[2];
  } else {
    const HV c{cam.camera[0], cam.camera[1], cam.camera[2]};
    const HV t{cam.target[0], cam.target[1], cam.target[2]};
    HV fwd = (c.x == t.x && c.y == t.y && c.z == t.z) ? HV{0.0, 1.0, 0.0} : HV{t.x - c.x, t.y - c.y, t.z - c.z};
    fwd = hnorm(fwd);
    yaw = std::atan2(fwd.y, fwd.x) - 0.5 * kPi;
    pitch = std::atan2(fwd.z, std::sqrt(fwd.x * fwd.x + fwd.y * fwd.y));
    HV top = hnorm(HV{cam.top[0], cam.top[1], cam.top[2]});
    top = hrotate_around(top, HV{0.0, 0.0, 1.0}, -yaw);
    top = hrotate_around(top, HV{1.0, 0.0, 0.0}, -pitch);
    roll = -std::atan2(top.z, top.x) + 0.5 * kPi;
    yaw = correct_angle(yaw);
    pitch = correct_angle(pitch);
    roll = correct_angle(roll);
  }
  for (int i = 0; i < 9; i++) mrot[i] = (i % 4 == 0) ? 1.0 : 0.0;
  *zero = true;
  rotate_axis(mrot, zero, 2, yaw);
  rotate_axis(mrot, zero, 0, pitch);
  rotate_axis(mrot, zero, 1, roll);
  angles[0] = yaw;
  angles[1] = pitch;
  angles[2] = roll;
}

mbr_status validate_camera(mbr_ctx *ctx, const mbr_camera &cam) {
  if (cam.width < 1 || cam.height < 1 || cam.width > 65535 || cam.height > 65535)
    return set_err(ctx, MBR_EINVAL, "image size %dx%d out of range [1, 65535]", cam.width, cam.height);
  if (cam.perspective_type < MBR_PROJECTION_THREE_POINT || cam.perspective_type > MBR_PROJECTION_FISH_EYE_CUT)
    return set_err(ctx, MBR_EINVAL, "unknown perspective_type %d", cam.perspective_type);
  if (cam.perspective_type == MBR_PROJECTION_THREE_POINT && !(cam.fov_deg > 0.0 && cam.fov_deg < 180.0))
    return set_err(ctx, MBR_EINVAL, "fov_deg must be in (0, 180) for the three-point projection, got %g", cam.fov_deg);
  if (cam.perspective_type != MBR_PROJECTION_THREE_POINT && !(cam.fov_deg > 0.0 && cam.fov_deg <= 720.0))
    return set_err(ctx, MBR_EINVAL, "fov_deg must be in (0, 720], got %g", cam.fov_deg);
  if (!finite3(cam.camera) || !finite3(cam.target) || !finite3(cam.top) || !finite3(cam.angles))
    return set_err(ctx, MBR_EINVAL, "non-finite camera vector");
  if (!cam.use_angles && cam.top[0] == 0.0 && cam.top[1] == 0.0 && cam.top[2] == 0.0)
    return set_err(ctx, MBR_EINVAL, "top vector is zero");
  return MBR_OK;
}

mbr_status build_frame(mbr_ctx *ctx, const mbr_camera &cam, const mbr_render_params &p, DevFrame *out, void *stream) {
  mbr_status st = validate_camera(ctx, cam);
  if (st != MBR_OK) return st;
  if (!(p.detail_level > 0.0) || !(p.de_factor > 0.0) || !(p.view_distance_max > 0.0) || !(p.smoothness > 0.0))
    return set_err(ctx, MBR_EINVAL, "detail_level, de_factor, view_distance_max and smoothness must be > 0");
  if (p.max_raymarching_steps < 1 || p.max_raymarching_steps > 100000000)
    return set_err(ctx, MBR_EINVAL, "max_raymarching_steps must be in [1, 1e8]");
  if (p.binary_steps < 0 || p.binary_steps > 200) return set_err(ctx, MBR_EINVAL, "binary_steps must be in [0, 200]");
  if (p.refine != MBR_REFINE_REFERENCE && p.refine != MBR_REFINE_ROOT)
    return set_err(ctx, MBR_EINVAL, "unknown refine mode %d", p.refine);
  if (p.ao_rays < 0 || p.ao_rays > 4096) return set_err(ctx, MBR_EINVAL, "ao_rays must be in [0, 4096]");
  if (p.gi_samples < 0 || p.gi_samples > 65536 || p.gi_bounces < 0 || p.gi_bounces > 64)
    return set_err(ctx, MBR_EINVAL, "gi_samples in [0, 65536] and gi_bounces in [0, 64] required");
  if (p.gi_samples > 0 && p.dof_aperture > 0.0 && !(p.dof_focus > 0.0))
    return set_err(ctx, MBR_EINVAL, "dof_focus must be > 0 with an aperture");
  if (!(p.gamma > 0.0)) return set_err(ctx, MBR_EINVAL, "gamma must be > 0");
  if (p.constant_de_threshold && !(p.de_thresh > 0.0)) return set_err(ctx, MBR_EINVAL, "de_thresh must be > 0");
  const int row_end = p.row_end == 0 ? cam.height : p.row_end;
  if (p.row_begin < 0 || p.row_begin >= row_end || row_end > cam.height)
    return set_err(ctx, MBR_EINVAL, "row band [%d, %d) outside the %d rows of the frame", p.row_begin, p.row_end,
                   cam.height);
  if (p.ao_fast && (p.ao_quality < 1 || p.ao_quality > 10 || !std::isfinite(p.ao_fast_tune)))
    return set_err(ctx, MBR_EINVAL, "fast AO needs ao_quality in [1, 10] and a finite ao_fast_tune");
  if (p.advanced_quality &&
      !(std::isfinite(p.detail_size_min) && std::isfinite(p.detail_size_max) && p.abs_min_marching_step > 0.0 &&
        p.abs_max_marching_step > 0.0 && p.rel_min_marching_step > 0.0 && p.rel_max_marching_step > 0.0 &&
        std::isfinite(p.abs_min_marching_step) && std::isfinite(p.abs_max_marching_step) &&
        std::isfinite(p.rel_min_marching_step) && std::isfinite(p.rel_max_marching_step)))
    return set_err(ctx, MBR_EINVAL, "advanced quality needs finite detail sizes and finite marching step limits > 0");
  if (!(p.soft_shadow_cone >= 0.0 && p.soft_shadow_cone < 90.0))
    return set_err(ctx, MBR_EINVAL, "soft_shadow_cone must be in [0, 90) degrees, got %g", p.soft_shadow_cone);
  const double *L = p.light_direction;
  if (!finite3(L) || (L[0] == 0.0 && L[1] == 0.0 && L[2] == 0.0))
    return set_err(ctx, MBR_EINVAL, "light_direction must be finite and non-zero");
  DevFrame f;
  std::memset(&f, 0, sizeof(f));
  for (int i = 0; i < 3; i++) f.camera[i] = cam.camera[i];
  bool zero;
  double ang[3];
  camera_matrix(cam, f.mrot, &zero, ang);
  f.mrot_zero = zero ? 1 : 0;
  f.width = cam.width;
  f.height = cam.height;
  f.row0 = p.row_begin;
  f.row1 = row_end;
  f.max_steps = p.max_raymarching_steps;
  f.binary_steps = p.binary_steps;
  f.refine = p.refine;
  f.jitter = p.jitter ? 1 : 0;
  f.seed = p.seed;
  // CalcFOV (projection_3d.cpp:140-159)
  f.persp = cam.perspective_type;
  f.legacy_y = cam.legacy_coordinate_system ? 1 : 0;
  f.fov = cam.perspective_type == MBR_PROJECTION_THREE_POINT ? 2.0 * std::tan(cam.fov_deg / 360.0 * kPi)
                                                              : cam.fov_deg / 180.0 * kPi;
  f.resolution = 1.0 / cam.height;
  // the image plane of an equirectangular view spans 2:1 (render_worker.cpp:98-100)
  f.aspect = cam.perspective_type == MBR_PROJECTION_EQUIRECTANGULAR ? 2.0 : double(cam.width) / cam.height;
  f.detail_level = p.detail_level;
  f.de_factor = p.de_factor;
  f.view_distance_max = p.view_distance_max;
  f.smoothness = p.smoothness;
  f.constant_de_threshold = p.constant_de_threshold ? 1 : 0;
  f.de_thresh = p.de_thresh;
  f.shading_enable = p.shading_enable ? 1 : 0;
  f.shadow_enable = p.shadow_enable ? 1 : 0;
  // cLight::softShadowCone is a float (light.h:113, light.cpp:87): the
  // tangent of shader_aux_shadow.cpp:64 is the float one
  f.soft_range = double(std::tan(float(p.soft_shadow_cone / 180.0 * kPi)));
  f.penetrating = p.penetrating ? 1 : 0;
  f.ao_fast = (p.ao_fast && p.gi_samples == 0) ? 1 : 0;
  f.ao_quality = p.ao_quality;
  f.ao_fast_tune = p.ao_fast_tune;
  f.ao_rays = p.ao_rays;
  const HV l = hnorm(HV{L[0], L[1], L[2]});
  f.light[0] = l.x;
  f.light[1] = l.y;
  f.light[2] = l.z;
  f.light_intensity = float(p.light_intensity);
  f.material_shading = float(p.material_shading);
  f.albedo = float(p.albedo);
  f.ambient = float(p.ambient_intensity);
  for (int i = 0; i < 3; i++) f.background[i] = float(p.background[i]);
  f.ao_seed = p.ao_seed;
  f.gi_samples = p.gi_samples;
  f.gi_bounces = p.gi_bounces;
  f.gi_seed = p.gi_seed;
  f.gi_sky = p.gi_sky;
  f.gi_sun = p.gi_sun;
  f.dof_aperture = p.dof_aperture;
  f.dof_focus = p.dof_focus;
  f.brightness = float(p.brightness);
  f.contrast = float(p.contrast);
  f.saturation = float(p.saturation);
  f.hdr = p.hdr ? 1 : 0;
  f.adv_quality = p.advanced_quality ? 1 : 0;
  f.slow_shading = p.slow_shading ? 1 : 0;
  f.detail_size_min = p.detail_size_min;
  f.detail_size_max = p.detail_size_max;
  f.abs_step_min = p.abs_min_marching_step;
  f.abs_step_max = p.abs_max_marching_step;
  f.rel_step_min = p.rel_min_marching_step;
  f.rel_step_max = p.rel_max_marching_step;
  // gamma table (cImage::CalculateGammaTable), cached per context.  A new
  // table is copied on `stream`, so frames queued earlier on that stream
  // still read the table they were built with.  The staging buffer is
  // pinned; before it is refilled, the host waits for its previous copy.
  if (ctx->gamma_value != p.gamma || !ctx->d_gamma) {
    const size_t bytes = 65536 * sizeof(uint16_t);
    if (!ctx->d_gamma) {
      int e = int(cudaMalloc(&ctx->d_gamma, bytes));
      if (e) {
        ctx->d_gamma = nullptr;
        return set_err(ctx, MBR_ENOMEM, "cudaMalloc(gamma): %s", cudaGetErrorString(cudaError_t(e)));
      }
    }
    if (!ctx->h_gamma) {
      int e = int(cudaMallocHost(&ctx->h_gamma, bytes));
      if (!e) e = int(cudaEventCreateWithFlags(&ctx->gamma_evt, cudaEventDisableTiming));
      if (e) return set_err(ctx, MBR_ENOMEM, "gamma staging buffer: %s", cudaGetErrorString(cudaError_t(e)));
    } else if (ctx->gamma_evt) {
      const int e = int(cudaEventSynchronize(ctx->gamma_evt));
      if (e) return cuda_err(ctx, e, "cudaEventSynchronize(gamma)");
    }
    uint16_t *t = ctx->h_gamma;
    for (int i = 0; i < 65536; i++) t[i] = uint16_t(int(powf(i / 65536.0f, 1.0f / float(p.gamma)) * 65535.0f));
    int e = int(cudaMemcpyAsync(ctx->d_gamma, t, bytes, cudaMemcpyHostToDevice, static_cast<cudaStream_t>(stream)));
    if (!e && ctx->gamma_evt) e = int(cudaEventRecord(ctx->gamma_evt, static_cast<cudaStream_t>(stream)));
    if (e) return cuda_err(ctx, e, "cudaMemcpyAsync(gamma)");
    ctx->gamma_value = p.gamma;
  }
  f.gamma = ctx->d_gamma;
  *out = f;
  return MBR_OK;
}

// Builds a frame exactly as build_frame does, with the gamma table in device
// memory the caller already owns (`gamma_dev`, 65536 entries) and a host
// staging table the caller owns too (`gamma_host`, 65536 entries, pageable):
// the table is copied on `stream` when *gamma_value differs from
// params.gamma, and nothing is allocated.  A copy from pageable memory has
// read its source when cudaMemcpyAsync returns, so the staging table may be
// refilled by the next call.  The error text, if any, goes to *err.
mbr_status build_frame_owned_gamma(const mbr_camera &cam, const mbr_render_params &p, uint16_t *gamma_dev,
                                   uint16_t *gamma_host, double *gamma_value, DevFrame *out, void *stream,
                                   std::string *err) {
  mbr_ctx tmp;  // holds no memory of its own; nothing to release
  tmp.d_gamma = gamma_dev;
  tmp.h_gamma = gamma_host;
  tmp.gamma_value = *gamma_value;
  const mbr_status st = build_frame(&tmp, cam, p, out, stream);
  *gamma_value = tmp.gamma_value;
  tmp.d_gamma = nullptr;
  tmp.h_gamma = nullptr;
  if (err) *err = tmp.err;
  return st;
}

DevOutputs dev_outputs(mbr_ctx *ctx, const mbr_outputs &o) {
  DevOutputs d;
  d.depth = o.depth;
  d.iters = o.iters;
  d.hit = o.hit;
  d.normal = o.normal;
  d.shade = o.shade;
  d.ao = o.ao;
  d.rgb = o.rgb;
  d.rgb8 = o.rgb8;
  d.stats = o.stats;
  d.status = ctx->d_status;
  d.pixel_offset = 0;
  return d;
}

const DevScene *ctx_scene(mbr_ctx *ctx) { return ctx->has_scene ? &ctx->scene : nullptr; }
int ctx_device(mbr_ctx *ctx) { return ctx->device; }
const mbr_scene *ctx_scene_src(mbr_ctx *ctx) { return ctx->has_scene ? &ctx->scene_src : nullptr; }
mbr_tuning &ctx_tuning(mbr_ctx *ctx) { return ctx->tuning; }
int32_t *ctx_status(mbr_ctx *ctx) { return ctx->d_status; }

// Device scratch of the wavefront kernel, grown on demand (never shrunk).
mbr_status ctx_work(mbr_ctx *ctx, size_t words, unsigned long long **out) {
  if (ctx->work_words < words) {
    if (ctx->d_work) cudaFree(ctx->d_work);
    ctx->d_work = nullptr;
    ctx->work_words = 0;
    const int e = int(cudaMalloc(&ctx->d_work, words * sizeof(unsigned long long)));
    if (e) return set_err(ctx, MBR_ENOMEM, "cudaMalloc(work): %s", cudaGetErrorString(cudaError_t(e)));
    ctx->work_words = words;
  }
  *out = ctx->d_work;
  return MBR_OK;
}

mbr_status ctx_adjoint_partials(mbr_ctx *ctx, size_t bytes, double **out) {
  if (ctx->adjoint_scratch_bytes < bytes) {
    if (ctx->adjoint_scratch) cudaFree(ctx->adjoint_scratch);
    ctx->adjoint_scratch = nullptr;
    ctx->adjoint_scratch_bytes = 0;
    const int e = int(cudaMalloc(&ctx->adjoint_scratch, bytes));
    if (e) return set_err(ctx, MBR_ENOMEM, "cudaMalloc(adjoint partials): %s", cudaGetErrorString(cudaError_t(e)));
    ctx->adjoint_scratch_bytes = bytes;
  }
  *out = static_cast<double *>(ctx->adjoint_scratch);
  return MBR_OK;
}

}  // namespace mbr

// ============================================================================
// C-ABI
// ============================================================================
extern "C" {

const char *mbr_version(void) { return "mandelbulber2_b200 1.0 (sm_100a)"; }

mbr_status mbr_create(mbr_ctx **out, int device) {
  if (!out) return MBR_EINVAL;
  *out = nullptr;
  mbr_ctx *ctx = new (std::nothrow) mbr_ctx();
  if (!ctx) return MBR_ENOMEM;
  ctx->device = device;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || device < 0 || device >= n) {
    delete ctx;
    return MBR_ECUDA;
  }
  if (cudaSetDevice(device) != cudaSuccess) {
    delete ctx;
    return MBR_ECUDA;
  }
  if (cudaMalloc(&ctx->d_status, sizeof(int32_t)) != cudaSuccess) {
    delete ctx;
    return MBR_ENOMEM;
  }
  cudaMemset(ctx->d_status, 0, sizeof(int32_t));
  mbr_scene_defaults(&ctx->scene_src);
  *out = ctx;
  return MBR_OK;
}

void mbr_destroy(mbr_ctx *ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->d_gamma) cudaFree(ctx->d_gamma);
  if (ctx->gamma_evt) {
    cudaEventSynchronize(ctx->gamma_evt);
    cudaEventDestroy(ctx->gamma_evt);
  }
  if (ctx->h_gamma) cudaFreeHost(ctx->h_gamma);
  if (ctx->d_status) cudaFree(ctx->d_status);
  if (ctx->d_work) cudaFree(ctx->d_work);
  if (ctx->adjoint_scratch) cudaFree(ctx->adjoint_scratch);
  delete ctx;
}

const char *mbr_last_error_string(const mbr_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

void mbr_primitive_defaults(mbr_primitive *q, int type) {
  if (!q) return;
  std::memset(q, 0, sizeof(*q));
  // InitPrimitiveParams (src/initparameters.cpp:1313-1420) and the legacy
  // node transform defaults (src/settings.cpp:2217-2241)
  q->type = type;
  q->caps = 1;
  q->iterations = 5;
  q->scale = 1.0;
  for (int i = 0; i < 3; i++) {
    q->size[i] = 1.0;
    q->limits_min[i] = -0.7;
    q->limits_max[i] = 0.7;
  }
  q->radius = 1.0;
  q->height = 1.0;
  q->width = 1.0;
  q->tube_radius = 0.2;
  q->radius_lpow = 1.0;
  q->tube_radius_lpow = 1.0;
  q->rounding = 1e-15;
  q->relative_amplitude = 0.2;
  q->length = 0.1;
  q->anim_speed = 1.0;
  q->anim_progression_speed = 1.0;
  q->prism_angle = 60.0;
  q->triangle_height = 1.0;
  if (type == MBR_PRIMITIVE_ELLIPSOID) {
    q->size[1] = q->size[2] = 0.5;
    q->limits_min[0] = -1.4;
    q->limits_max[0] = 1.4;
  }
}

void mbr_fractal_defaults(mbr_fractal *f, int formula) {
  if (!f) return;
  std::memset(f, 0, sizeof(*f));
  // src/initparameters.cpp:701-750, 1010
  f->formula = formula;
  f->formula_iterations = 1;
  f->formula_start_iteration = 0;
  f->formula_stop_iteration = 250;
  f->dont_add_c_constant = 0;
  f->check_for_bailout = 1;
  f->formula_weight = 1.0;
  f->bulb_power = 9.0;
  f->mandelbox_scale = 2.0;
  f->mandelbox_folding_limit = 1.0;
  f->mandelbox_folding_value = 2.0;
  f->mandelbox_folding_min_radius = 0.5;
  f->mandelbox_folding_fixed_radius = 1.0;
  f->transf_scale3 = 3.0;
  // IFS (initparameters.cpp:724-743)
  f->ifs_scale = 2.0;
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

void mbr_scene_defaults(mbr_scene *s) {
  if (!s) return;
  std::memset(s, 0, sizeof(*s));
  // src/initparameters.cpp:128-157 and the default node (:2102-2125)
  s->n_fractals = 1;
  s->formula_maxiter = 250;
  s->repeat_from = 1;
  s->use_default_bailout = 1;
  s->delta_de_function = MBR_DE_FUNCTION_PREFERRED;
  s->min_n = 1;
  s->bailout = 100.0;
  for (int i = 0; i < 3; i++) s->fractal_constant_factor[i] = 1.0;
  mbr_fractal_defaults(&s->fractal[0], MBR_FORMULA_MANDELBULB);
  for (int i = 1; i < MBR_MAX_FRACTALS; i++) mbr_fractal_defaults(&s->fractal[i], MBR_FORMULA_NONE);
  // initparameters.cpp:143-145, 199-204
  for (int i = 0; i < 3; i++) {
    s->limit_min[i] = -10.0;
    s->limit_max[i] = 10.0;
  }
  s->box_folding_limit = 1.0;
  s->box_folding_value = 2.0;
  s->spherical_folding_inner = 0.5;
  s->spherical_folding_outer = 1.0;
  s->delta_de_method = MBR_DE_METHOD_PREFERRED;
  s->deltade_relative_delta = 0.01;  // :166
}

void mbr_camera_defaults(mbr_camera *c) {
  if (!c) return;
  std::memset(c, 0, sizeof(*c));
  // src/initparameters.cpp:113-120
  c->camera[0] = 3.0;
  c->camera[1] = -6.0;
  c->camera[2] = 2.0;
  c->top[0] = -0.1277753;
  c->top[1] = 0.2555506;
  c->top[2] = 0.958314;
  c->fov_deg = 53.13;
  c->width = 800;
  c->height = 600;
}

void mbr_render_params_defaults(mbr_render_params *p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->detail_level = 1.0;
  p->de_factor = 1.0;
  p->view_distance_max = 50.0;
  p->smoothness = 1.0;
  p->max_raymarching_steps = 10000;
  p->binary_steps = 30;
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
  p->ambient_intensity = 0.0;
  p->dof_focus = 3.0;
  p->gi_sky = 0.3;
  p->gi_sun = 3.0;
  p->brightness = 1.0;
  p->contrast = 1.0;
  p->gamma = 1.0;
  p->saturation = 1.0;
  // light 1 (initparameters.cpp:1901, 1919)
  p->soft_shadow_cone = 1.0;
  p->penetrating = 1;
  // initparameters.cpp:214-216
  p->ao_quality = 4;
  p->ao_fast_tune = 1.0;
  // initparameters.cpp:159-165
  p->advanced_quality = 0;
  p->abs_max_marching_step = 3.0;
  p->abs_min_marching_step = 1e-15;
  p->rel_max_marching_step = 1e4;
  p->rel_min_marching_step = 1e-2;
  p->detail_size_max = 1.0;
  p->detail_size_min = 1e-12;
}

mbr_status mbr_scene_set(mbr_ctx *ctx, const mbr_scene *scene) {
  if (!ctx || !scene) return set_err(ctx, MBR_EINVAL, "null argument");
  DevScene d;
  mbr_status st = build_scene(ctx, *scene, &d);
  if (st != MBR_OK) return st;
  ctx->scene = d;
  ctx->scene_src = *scene;
  ctx->has_scene = true;
  return MBR_OK;
}

mbr_status mbr_camera_rotation(const mbr_camera *camera, double mrot[9], double angles[3]) {
  if (!camera || !mrot || !angles) return MBR_EINVAL;
  bool zero;
  camera_matrix(*camera, mrot, &zero, angles);
  return MBR_OK;
}

mbr_status mbr_scene_sequence(const mbr_scene *scene, int32_t *seq_out, int32_t *length_out,
                              int32_t *de_function_out, double *bailout_out) {
  if (!scene) return MBR_EINVAL;
  DevScene d;
  mbr_status st = build_scene(nullptr, *scene, &d);
  if (st != MBR_OK) return st;
  if (seq_out)
    for (int i = 0; i < d.length; i++) seq_out[i] = d.seq[i];
  if (length_out) *length_out = d.length;
  if (de_function_out) *de_function_out = d.is_hybrid ? d.de_function : d.de_analytic;
  if (bailout_out)
    for (int i = 0; i < d.n; i++) bailout_out[i] = d.slot[i].d[P_BAILOUT];
  return MBR_OK;
}

mbr_status mbr_render(mbr_ctx *ctx, const mbr_camera *camera, const mbr_render_params *params,
                      const mbr_outputs *out, int engine, void *stream) {
  if (!ctx || !camera || !params || !out) return set_err(ctx, MBR_EINVAL, "null argument");
  if (!ctx->has_scene) return set_err(ctx, MBR_EINVAL, "no scene set (call mbr_scene_set first)");
  if (cudaSetDevice(ctx->device) != cudaSuccess) return set_err(ctx, MBR_ECUDA, "cudaSetDevice failed");
  DevFrame fr;
  mbr_status st = build_frame(ctx, *camera, *params, &fr, stream);
  if (st != MBR_OK) return st;
  fr.want_normal = out->normal != nullptr;
  const DevOutputs d = dev_outputs(ctx, *out);
  const bool fp32 = engine == MBR_ENGINE_PLAIN_MIXED || engine == MBR_ENGINE_WAVEFRONT_FP32;
  if (fp32 && ctx->scene.has_w)
    return set_err(ctx, MBR_EUNSUPPORTED, "FP32 engines need a 3-D state: initial_waxis == 0 and no hypercomplex "
                                          "formula");
  if (params->slow_shading && ctx->scene.n_prims > 0)
    return set_err(ctx, MBR_EUNSUPPORTED,
                   "slow shading takes its normals from the fractal's orbit; with primitives a hit may lie on one");
  if (engine == MBR_ENGINE_PLAIN_MIXED && ctx->scene.delta_de)
    return set_err(ctx, MBR_EUNSUPPORTED,
                   "the delta DE offsets points by 1e-5 of the detail size, which FP32 points do not resolve: use a "
                   "plain FP64 engine");
  // the delta DE's offset factor follows this render's advanced quality
  // (calculate_distance.cpp:616-623); the scene is a launch parameter
  DevScene scd;
  const DevScene *scp = &ctx->scene;
  if (ctx->scene.delta_de) {
    scd = ctx->scene;
    scd.delta_factor = params->advanced_quality ? scd.delta_rel : 1e-5;
    scp = &scd;
  }
  int e;
  switch (engine) {
    case MBR_ENGINE_PLAIN_FP64: e = launch_plain_fp64(*scp, fr, d, stream); break;
    case MBR_ENGINE_PLAIN_FP64_STRICT: e = launch_plain_fp64_strict(*scp, fr, d, stream); break;
    case MBR_ENGINE_PLAIN_MIXED: e = launch_plain_mixed(ctx->scene, fr, d, stream); break;
    case MBR_ENGINE_WAVEFRONT_FP32:
    case MBR_ENGINE_WAVEFRONT_FP64:
    case MBR_ENGINE_WAVEFRONT_AUTO:
      return render_wavefront(ctx, ctx->scene, fr, d, engine, stream);
    default: return set_err(ctx, MBR_EINVAL, "unknown engine %d", engine);
  }
  return cuda_err(ctx, e, "kernel launch");
}

mbr_status mbr_sync(mbr_ctx *ctx, void *stream) {
  if (!ctx) return MBR_EINVAL;
  int e = int(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
  if (e) return cuda_err(ctx, e, "cudaStreamSynchronize");
  int32_t status = 0;
  e = int(cudaMemcpy(&status, ctx->d_status, sizeof(status), cudaMemcpyDeviceToHost));
  if (e) return cuda_err(ctx, e, "cudaMemcpy(status)");
  if (status != 0) {
    e = int(cudaMemset(ctx->d_status, 0, sizeof(int32_t)));
    if (e) return cuda_err(ctx, e, "cudaMemset(status)");
    if (status & STATUS_AO_MARCH_CAP)
      return set_err(ctx, MBR_ETIMEOUT,
                     "device watchdog: an AO march reached max_raymarching_steps and was ended as unoccluded "
                     "(status %d; the frame is complete, stats.watchdog_trips counts the marches)",
                     status);
    return set_err(ctx, MBR_ETIMEOUT, "device watchdog tripped (status %d)", status);
  }
  return MBR_OK;
}

mbr_status mbr_distance(mbr_ctx *ctx, const double *points, int64_t n, double detail_size, int normal_mode,
                        double *dist, int32_t *iters, int engine, void *stream) {
  if (!ctx) return MBR_EINVAL;
  if (!ctx->has_scene) return set_err(ctx, MBR_EINVAL, "no scene set");
  if (n < 0 || (n > 0 && (!points || !dist))) return set_err(ctx, MBR_EINVAL, "bad point buffers");
  if (cudaSetDevice(ctx->device) != cudaSuccess) return set_err(ctx, MBR_ECUDA, "cudaSetDevice failed");
  int e;
  switch (engine) {
    case MBR_ENGINE_PLAIN_FP64:
    case MBR_ENGINE_WAVEFRONT_FP64:
    case MBR_ENGINE_WAVEFRONT_AUTO:
      e = launch_distance_fp64(ctx->scene, points, n, detail_size, normal_mode, dist, iters, stream);
      break;
    case MBR_ENGINE_PLAIN_FP64_STRICT:
      e = launch_distance_fp64_strict(ctx->scene, points, n, detail_size, normal_mode, dist, iters, stream);
      break;
    case MBR_ENGINE_PLAIN_MIXED:
    case MBR_ENGINE_WAVEFRONT_FP32:
      if (ctx->scene.has_w) return set_err(ctx, MBR_EUNSUPPORTED, "FP32 engines need initial_waxis == 0");
      if (ctx->scene.delta_de)
        return set_err(ctx, MBR_EUNSUPPORTED, "the delta DE needs FP64 points: use a plain FP64 engine");
      e = launch_distance_fp32(ctx->scene, points, n, detail_size, normal_mode, dist, iters, stream);
      break;
    default: return set_err(ctx, MBR_EINVAL, "unknown engine %d", engine);
  }
  return cuda_err(ctx, e, "distance kernel launch");
}

mbr_status mbr_set_tuning(mbr_ctx *ctx, const mbr_tuning *t) {
  if (!ctx || !t) return MBR_EINVAL;
  if (t->block_size < 32 || t->block_size > 256 || t->block_size % 32 || t->ctas_per_sm < 1 ||
      t->ctas_per_sm > 32 || t->refill_k < 0 || t->refill_k > 32 || t->queue_layout < 0 || t->queue_layout > 1)
    return set_err(ctx, MBR_EINVAL, "tuning out of range");
  ctx->tuning = *t;
  return MBR_OK;
}

mbr_status mbr_get_tuning(const mbr_ctx *ctx, mbr_tuning *t) {
  if (!ctx || !t) return MBR_EINVAL;
  *t = ctx->tuning;
  return MBR_OK;
}

}  // extern "C"
