// mbr_device.h - data the host prepares for the kernels (host and device).
//
// A scene is flattened into DevScene: the hybrid sequence table and the
// per-slot formula parameters in both FP64 and FP32, derived on the host once
// (sFractal::RecalculateFractalParams, src/fractal.cpp:653-678, and
// cHybridFractalSequences::CreateSequence, src/hybrid_fractal_sequences.cpp:289-499).
// It is passed to the kernels by value (__grid_constant__), so every lane
// reads it through the constant cache.
#pragma once
#include <stdint.h>

#include "../../include/mbr.h"
#include "formula_params.h"

namespace mbr {

// Indices into DevSlot::d / DevSlot::f.
enum SlotParam {
  P_POWER = 0,      // bulb power
  P_POWER_M1,       // power - 1
  P_ALPHA,          // radians
  P_BETA,
  P_MB_SCALE,
  P_MB_ABS_SCALE,
  P_MB_LIMIT,
  P_MB_VALUE,
  P_MB_MR2,
  P_MB_FR2,
  P_MB_FACTOR1,     // fR2 / mR2
  P_MB_OFF_X,
  P_MB_OFF_Y,
  P_MB_OFF_Z,
  P_SCALE3,
  P_BAILOUT,
  P_WEIGHT,
  P_AEX_CADD,       // aexion cadd
  P_ADE_ON,         // analyticDE enabled (0 or 1)
  P_ADE_SCALE1,     // analyticDE scale1
  P_ADE_OFFSET1,    // analyticDE offset1
  P_COUNT
};

struct DevSlot {
  int32_t formula;
  int32_t add_c;
  int32_t check_bailout;
  int32_t has_offset;
  int32_t add_bail;      // the formula's DE function is pseudo- or Jos-Kleinian: the convergence bailout
  int32_t pad_slot;
  double d[P_COUNT];
  float f[P_COUNT];
  double x[MBR_SLOT_X];  // a keyed formula's parameter block (formula_params.h)
};

// Mandelbox rotations of slot 0 of a single-fractal scene (sFractalMandelbox
// rot, rotinv, mainRot; fractal.cpp:663-671): row-major matrices built on the
// host from the angles.  rotinv is the transpose of rot and is applied as
// such; zero marks a matrix whose angles were all 0 (CRotationMatrix::zero:
// RotateVector returns its argument).
struct MbRot {
  int32_t folds;        // rotationsEnabled: the box fold in rotated frames
  int32_t main;         // mainRotationEnabled
  int32_t zero[2][3];   // rot[fold][axis].zero
  int32_t main_zero;    // mainRot.zero
  int32_t pad;
  double m[2][3][9];    // rot[fold][axis]: fold 0 from mandelbox_rotation_neg, 1 from _pos
  double mm[9];         // mainRot
};

// Kaleidoscopic IFS of slot 0 of a single-fractal scene (sFractalIFS,
// fractal.h:155-174): the enabled vectors in order, with their rotation
// matrices (SetRotation3), twice-normalised directions, distances and
// intensities, built on the host (fractal.cpp:96-115, 655-661).
struct IfsBlock {
  int32_t abs_x, abs_y, abs_z, menger;
  int32_t rot_on, edge_on, n, main_zero;
  int32_t rot_zero[9];
  int32_t pad;
  double scale;
  double offset[3];
  double edge[3];
  double main[9];       // mainRot, row-major
  double rot[9][9];     // rot of the k-th enabled vector
  double dir[9][3];
  double dist[9];
  double inten[9];
};

// The F template value of the generic iteration that carries every formula
// and the Mandelbox rotations (de_core.cuh calc_distance).
constexpr int F_EXT = -1;

// Whether a scene needs that iteration.
struct DevScene;
__host__ __device__ inline bool scene_extended(const DevScene &sc);

// One primitive of the union in the form its distance reads: the node's
// world-to-local matrix and scale (objects_tree.cpp:290-385,
// CMatrix44::InverseAffine) and the primitive's own fields (primitive.cpp),
// built on the host.
struct DevPrim {
  int32_t type, empty, limits, caps;
  int32_t iterations, has_repeat;
  double m[12];         // worldToLocalMatrix rows 1-3: m11 m12 m13 m14, m21 ...
  double abs_scale;     // |world scale|: a local distance times this is a world distance
  double repeat[3];     // repeat period / abs_scale
  double size[3];       // box
  double radius, height, width, tube;
  double pow_r, pow_t;  // torus: pow(2, radius_lpow), pow(2, tube_radius_lpow)
  double rounding, wall;
  double lmin[3], lmax[3];
  double amp, length, phase, xshift;  // water: length * relative amplitude, animation phase and drift
  double wn[2];         // cone: the unit wall normal (1, radius / height) normalised
  double pn[3], tri;    // prism: (sin a, cos a, sin a) of half its angle a, triangle height * sin a
};

// One node of an explicit objects tree as the walk reads it
// (cObjectsTree::sNodeDataForRendering, objects_tree.h:50-80), built on the
// host: the world-to-local matrix of its accumulated transform, its scale,
// repeat and detail multiplier, the smooth-union settings, and for a fractal
// node its own sequence settings (one slot iterated alone).
struct DevNode {
  int32_t type, level, smooth, has_repeat;
  double w2l[12];
  double abs_scale, detail_mult, smooth_dist;
  double repeat[3];     // repeat / absScale
  // FRACTAL
  int32_t slot, maxN, julia, has_w;
  int32_t de_final, de_analytic, delta_de, delta_fn;
  double julia_c[3];    // julia_c
  double cmul[3];       // fractal_constant_factor
  double w0;
  float fcmul[3], pad_f;
  // PRIMITIVE: its record in DevScene::prim
  int32_t prim, pad;
};

struct DevScene {
  int32_t n;
  int32_t is_hybrid;
  int32_t length;          // sequence length (entries of seq)
  int32_t formula_maxiter;
  int32_t min_n;
  int32_t iter_thresh;
  int32_t interior;
  int32_t julia;
  int32_t de_function;     // hybrid: enumDEFunctionType (1 linear, 2 log)
  int32_t de_analytic;     // non-hybrid: enumDEAnalyticFunction (1 linear, 2 log, 3 IFS)
  int32_t uniform_formula; // formula id when every iteration uses slot 0, else 0
  int32_t has_w;           // initial w != 0 or a 4-D formula (4-D state needed)
  int32_t generic;         // a slot's formula has no specialised FP32/FP64 form (reference-order iteration only)
  int32_t pad1;
  double julia_c[3];
  double cmul[3];
  double w0;
  double linear_de_offset;
  float fjulia_c[3];
  float fcmul[3];
  float flinear_de_offset;
  float pad0;
  DevSlot slot[MBR_MAX_FRACTALS];
  MbRot mbrot;             // zero (no rotations) unless slot 0 is a rotated Mandelbox
  IfsBlock ifs;            // slot 0 of a kaleidoscopic IFS scene
  int32_t n_prims;         // primitives joined by union (F_EXT iteration only)
  int32_t pad2;
  DevPrim prim[MBR_MAX_PRIMITIVES];
  // limit box and global folds (F_EXT iteration only)
  int32_t limits, gbox, gsph, pad4;
  double lim_min[3], lim_max[3];
  double gbox_limit, gbox_value, gsph_fr2, gsph_mr2;  // spherical: outer^2, inner^2
  float flim_min[3], flim_max[3];
  float fgbox_limit, fgbox_value, fgsph_fr2, fgsph_mr2;
  // the final distance of the orbit (DevDeFinal), and the delta DE
  // (calculate_distance.cpp:607-760): its DE function (enumDEFunctionType)
  // and offset factor (1e-5, or deltade_relative_delta under advanced
  // quality; set per render)
  int32_t de_final;
  int32_t delta_de;
  int32_t delta_fn;
  int32_t pad5;
  double delta_factor;
  double delta_rel;
  // an explicit objects tree (F_EXT iteration only)
  int32_t n_nodes;
  int32_t pad6;
  DevNode node[MBR_MAX_NODES];
  uint8_t seq[MBR_SEQUENCE_LENGTH];
};

// The final distance of an analytic orbit (compute_fractal.cpp:495-621):
// one code for the hybrid DEFunctionType and the non-hybrid
// DEAnalyticFunction.  The first four are the ones the specialised
// iterations carry; the others make a scene extended.
enum DevDeFinal {
  DEF_LINEAR = 1,         // r / DE
  DEF_LOG = 2,            // 0.5 r log r / DE (0 for r <= 1)
  DEF_IFS = 3,            // (r - 2) / DE
  DEF_LINEAR_OFFSET = 4,  // hybrid linear: (r - linearDEOffset) / DE
  DEF_PSEUDO_KLEINIAN = 5,// max(rxy - 1, |rxy z| / r) / DE (aux.pseudoKleinianDE stays 1)
  DEF_CUSTOM = 6,         // aux.dist: 1000 for every formula built here
  DEF_MAX_AXIS = 7,       // max |z_i| / DE
  DEF_NONE = 8            // analyticFunctionNone: -1
};

__host__ __device__ inline bool scene_extended(const DevScene &sc) {
  return sc.generic || sc.mbrot.folds || sc.mbrot.main || sc.n_prims > 0 || sc.limits || sc.gbox || sc.gsph ||
         sc.delta_de || sc.de_final > DEF_LINEAR_OFFSET || sc.n_nodes > 0;
}

// Everything about one frame that is not the scene: camera, march and
// shading parameters, derived on the host.
struct DevFrame {
  double camera[3];
  double mrot[9];      // PrepareMainVectors mRot, row-major
  int32_t mrot_zero;   // CRotationMatrix::zero: RotateVector is the identity
  int32_t width, height;
  int32_t row0, row1;  // rows rendered: [row0, row1)
  int32_t max_steps;
  int32_t binary_steps;
  int32_t refine;
  int32_t jitter;
  uint32_t seed;
  double fov;          // CalcFOV: 2 tan(FOV/2) three-point, FOV in radians otherwise
  double resolution;   // 1 / height
  double aspect;
  double detail_level;
  double de_factor;
  double view_distance_max;
  double smoothness;
  int32_t constant_de_threshold;
  int32_t shading_enable;
  int32_t shadow_enable;
  int32_t ao_rays;
  double de_thresh;
  double light[3];     // unit vector toward the light
  double soft_range;   // tan(soft shadow cone); 0: hard shadow
  int32_t penetrating; // shadow march to |camera - p| * fov, darkened by depth
  int32_t ao_fast;     // fast AO: quality^2 - 1 samples along the normal
  int32_t ao_quality;
  int32_t pad2;
  double ao_fast_tune;
  float light_intensity;
  float material_shading;
  float albedo;
  float ambient;
  float background[3];
  uint32_t ao_seed;
  int32_t gi_samples;
  int32_t gi_bounces;
  uint32_t gi_seed;
  int32_t want_normal;
  int32_t persp;       // mbr_projection
  int32_t legacy_y;    // legacy coordinate system: image y runs -0.5 (top) to +0.5
  double gi_sky;
  double gi_sun;
  double dof_aperture;
  double dof_focus;
  float brightness, contrast, saturation;
  int32_t hdr;
  const uint16_t *gamma;  // 65536-entry table (device)
  // advanced quality: threshold clamps and march step limits (render_worker.cpp:671-675, 819-834)
  int32_t adv_quality;
  int32_t slow_shading;  // normals from the iteration-count gradient (plain engines, F_EXT kernels)
  double detail_size_min, detail_size_max;
  double abs_step_min, abs_step_max, rel_step_min, rel_step_max;
};

// Bits of the device status word (DevOutputs::status), read and cleared by
// mbr_sync: a bounded loop ran out of its budget.  The frame is complete;
// the loops that ran out were ended as the watchdog rule says.
enum DevStatus {
  STATUS_AO_MARCH_CAP = 1,  // an AO march reached max_raymarching_steps (ended unoccluded)
};

struct DevOutputs {
  double *depth;
  int32_t *iters;
  uint8_t *hit;
  float *normal;
  float *shade;
  float *ao;
  float *rgb;
  uint8_t *rgb8;
  mbr_stats *stats;
  int32_t *status;        // watchdog status word (device, context-owned)
  int64_t pixel_offset;   // added to the pixel index when writing
};

// Counters a thread accumulates before one reduction per warp.
struct Counters {
  unsigned long long de, iters, march, binary, normal, shadow, ao, gi, pixels, watchdog;
};

// ---- launchers (one per translation unit) ---------------------------------
// Plain per-pixel kernels: rows [0, height) of the frame.
int launch_plain_fp64(const DevScene &sc, const DevFrame &fr, const DevOutputs &out, void *stream);
int launch_plain_fp64_strict(const DevScene &sc, const DevFrame &fr, const DevOutputs &out, void *stream);
int launch_plain_mixed(const DevScene &sc, const DevFrame &fr, const DevOutputs &out, void *stream);
int launch_distance_fp64(const DevScene &sc, const double *pts, int64_t n, double detail, int normal_mode,
                         double *dist, int32_t *iters, void *stream);
int launch_distance_fp64_strict(const DevScene &sc, const double *pts, int64_t n, double detail, int normal_mode,
                                double *dist, int32_t *iters, void *stream);
int launch_distance_fp32(const DevScene &sc, const double *pts, int64_t n, double detail, int normal_mode,
                         double *dist, int32_t *iters, void *stream);

}  // namespace mbr
