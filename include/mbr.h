/*
 * mbr.h - C-ABI of the B200-native distance-estimation raymarcher.
 *
 * This library replaces the per-pixel work of mandelbulber2's cRenderWorker
 * (src/render_worker.cpp:91-530) and everything beneath it on one GPU:
 *   Compute<calcModeNormal>        src/compute_fractal.cpp:67-654
 *   CalculateDistance(Simple)      src/calculate_distance.cpp:60-64, 225-516, 533-606
 *   cRenderWorker::RayMarching     src/render_worker.cpp:708-951
 *   CalculateNormals (fast path)   src/shader_calculate_normals.cpp:40-79
 *   LightShading + AuxShadow       src/shader_light_shading.cpp:40-122,
 *                                  src/shader_aux_shadow.cpp:39-323 (hard, soft, penetrating)
 *   AmbientOcclusion               src/shader_ambient_occlusion.cpp:41-120
 *   GlobalIlumination + MC DOF     src/shader_global_illumination.cpp:41-209,
 *                                  src/render_worker.cpp:1832-1862
 *   cImage::CalculatePixel + 8 bit src/cimage.cpp:317-375, 460-469
 *
 * Only plain C types cross this boundary.  All buffers in mbr_outputs are
 * caller-owned DEVICE pointers; streams are passed as `void*` (a cudaStream_t,
 * NULL = legacy default stream).  A context is not thread-safe: use one
 * context per host thread.  No call throws; every call returns an mbr_status
 * and, on failure, mbr_last_error_string() describes the cause.
 */
#ifndef MBR_H_
#define MBR_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MBR_ABI_VERSION 6

/* Number of formula slots of one hybrid sequence (the reference's nine
 * fractal tabs; "repeat_from" is limited to 1..9, src/initparameters.cpp:151). */
#define MBR_MAX_FRACTALS 9
/* Length of a hybrid sequence table: maxN * 5 with maxN = 250
 * (src/hybrid_fractal_sequences.cpp:296-298). */
#define MBR_SEQUENCE_LENGTH 1250
/* primitives joined to the fractal by union (at most this many) */
#define MBR_MAX_PRIMITIVES 8
/* nodes of an explicit objects tree */
#define MBR_MAX_NODES 16

typedef enum mbr_status {
  MBR_OK = 0,
  MBR_EINVAL = 1,        /* invalid argument (sizes, NULL pointers, ranges) */
  MBR_ECUDA = 2,         /* a CUDA runtime call failed */
  MBR_ETIMEOUT = 3,      /* a kernel watchdog budget ran out (status word set on device) */
  MBR_ENOMEM = 4,        /* device allocation failed */
  MBR_EUNSUPPORTED = 5   /* valid request that this build does not implement */
} mbr_status;

/* Formula ids, numerically equal to fractal::enumFractalFormula
 * (formula/definition/all_fractal_list_enums.hpp:40-52). */
typedef enum mbr_formula {
  MBR_FORMULA_NONE = 0,
  MBR_FORMULA_MANDELBULB = 2,   /* formula/definition/fractal_mandelbulb.cpp:29-43 */
  MBR_FORMULA_MANDELBULB_POWER2 = 3, /* formula/definition/fractal_mandelbulb_power2.cpp:30-45 */
  MBR_FORMULA_HYPERCOMPLEX = 4, /* formula/definition/fractal_hypercomplex.cpp:30-45; 4-D: plain FP64 engines */
  MBR_FORMULA_QUATERNION = 5,   /* formula/definition/fractal_quaternion.cpp:29-39 */
  MBR_FORMULA_AEXION = 19,      /* formula/definition/fractal_aexion.cpp:29-59; 4-D: plain FP64 engines */
  MBR_FORMULA_KALEIDOSCOPIC_IFS = 10, /* formula/definition/fractal_kaleidoscopic_ifs.cpp:30-85 */
  MBR_FORMULA_XENODREAMBUIE = 11, /* formula/definition/fractal_xenodreambuie.cpp:30-49; Mandelbulb parameters */
  MBR_FORMULA_MENGER_SPONGE = 7,/* formula/definition/fractal_menger_sponge.cpp:30-71 */
  MBR_FORMULA_MANDELBOX = 8,    /* formula/definition/fractal_mandelbox.cpp:31-107 */
  /* formulas whose parameters are passed by settings key (mbr_fractal.param) */
  MBR_FORMULA_BOX_FOLD_BULB_POW2 = 16, /* formula/definition/fractal_box_fold_bulb_pow2.cpp:27-76 (delta DE) */
  MBR_FORMULA_GENERALIZED_FOLD_BOX = 37, /* formula/definition/fractal_generalized_fold_box.cpp:31-245 */
  MBR_FORMULA_MENGER_MOD1 = 61,       /* formula/definition/fractal_menger_mod1.cpp:29-103 */
  MBR_FORMULA_BOX_FOLD_BULB_POW2_V2 = 125, /* formula/definition/fractal_box_fold_bulb_pow2_v2.cpp:29-146 */
  MBR_FORMULA_MANDELBULB_PUPUKU = 266, /* formula/definition/fractal_mandelbulb_pupuku.cpp:29-144 */
  MBR_FORMULA_DIFS_HEXTGRID2 = 608,   /* formula/definition/fractal_difs_hextgrid2.cpp:30-138 (custom DE) */
  MBR_FORMULA_PSEUDO_KLEINIAN_STD_DE = 101, /* formula/definition/fractal_pseudo_kleinian_std_de.cpp:29-215 (custom DE) */
  MBR_FORMULA_PSEUDO_KLEINIAN = 103,  /* formula/definition/fractal_pseudo_kleinian.cpp:30-202 */
  MBR_FORMULA_ABOX_MOD11 = 119,       /* formula/definition/fractal_abox_mod11.cpp:34-250 */
  MBR_FORMULA_PSEUDO_KLEINIAN_MOD4 = 217 /* formula/definition/fractal_pseudo_kleinian_mod4.cpp:29-145 */
} mbr_formula;

/* fractal::enumDEFunctionType (src/fractal_enums.h:47-60).  The Jos
 * Kleinian function is taken with the delta DE only: its analytic form reads
 * formula parameters that mbr_fractal does not carry. */
typedef enum mbr_de_function {
  MBR_DE_FUNCTION_PREFERRED = 0,
  MBR_DE_FUNCTION_LINEAR = 1,
  MBR_DE_FUNCTION_LOGARITHMIC = 2,
  MBR_DE_FUNCTION_PSEUDO_KLEINIAN = 3,
  MBR_DE_FUNCTION_JOS_KLEINIAN = 4,
  MBR_DE_FUNCTION_CUSTOM = 5,
  MBR_DE_FUNCTION_MAX_AXIS = 6
} mbr_de_function;

/* fractal::enumDEMethod (src/fractal_enums.h:40-45), "delta_DE_method". */
typedef enum mbr_de_method {
  MBR_DE_METHOD_PREFERRED = 0,     /* each formula's own (all formulas built here are analytic) */
  MBR_DE_METHOD_FORCE_DELTA = 1,   /* the delta DE of CalculateDistanceSimple */
  MBR_DE_METHOD_FORCE_ANALYTIC = 2
} mbr_de_method;

/* Which kernel renders a frame. */
typedef enum mbr_engine {
  /* One FP64 thread per pixel; FMA contraction allowed (the plain FP64 path). */
  MBR_ENGINE_PLAIN_FP64 = 0,
  /* Same kernel compiled without FMA contraction: every double operation is
   * the IEEE-rounded operation the CPU reference performs. */
  MBR_ENGINE_PLAIN_FP64_STRICT = 1,
  /* One thread per pixel; formula iteration and march step in FP32, ray
   * origin, accumulated t and the final hit bisection in FP64. */
  MBR_ENGINE_PLAIN_MIXED = 2,
  /* Persistent wavefront kernel: FP32 iteration, FP64 origin and t, per-lane
   * ray refill, re-convergence of finished lanes every k iterations. */
  MBR_ENGINE_WAVEFRONT_FP32 = 3,
  /* The wavefront kernels with the formula iteration in FP64, in the
   * reference's operation order, and the march arithmetic of the plain FP64
   * kernel: for views whose hit threshold FP32 points cannot resolve. */
  MBR_ENGINE_WAVEFRONT_FP64 = 4,
  /* The wavefront kernels, FP32 or FP64 iteration chosen per frame (per job
   * in a batch) on the device: FP64 when DE(camera) * (threshold per unit
   * distance), a lower bound of the view's hit thresholds, is below 256 FP32
   * units (2^-24) of the camera coordinates - deep zooms and cameras inside
   * the solid. */
  MBR_ENGINE_WAVEFRONT_AUTO = 5
} mbr_engine;

/* How the hit is refined after the march finds dist < threshold. */
typedef enum mbr_refine {
  /* Reference binary search: at most binary_steps halvings, stopped when
   * threshold*(1-0.001*detail) < dist < threshold (render_worker.cpp:854-912). */
  MBR_REFINE_REFERENCE = 0,
  /* Bisection of F(t) = dist(t) - threshold(t) to convergence (64 halvings);
   * makes depth a smooth function of the parameters (used by the adjoint). */
  MBR_REFINE_ROOT = 1
} mbr_refine;

/* One formula slot: the subset of sFractal (src/fractal.h:888-940) and of
 * cHybridFractalSequences::sFractalData (src/hybrid_fractal_sequences.h:33-54)
 * that the three supported formulas read.  Angles are in degrees, as in the
 * settings file; the library converts them like
 * sFractal::RecalculateFractalParams (src/fractal.cpp:653-678). */
/* One formula parameter by its settings key (see mbr_fractal.param).
 * Integers and booleans (0 / 1) use value[0]; vectors use value[0..2];
 * rotations are vectors of angles in degrees. */
#define MBR_MAX_FORMULA_PARAMS 48
#define MBR_PARAM_KEY_LEN 48
typedef struct mbr_formula_param {
  char key[MBR_PARAM_KEY_LEN];               /* NUL-terminated */
  double value[3];
} mbr_formula_param;

typedef struct mbr_fractal {
  int32_t formula;                 /* mbr_formula */
  int32_t formula_iterations;      /* "formula_iterations", default 1 */
  int32_t formula_start_iteration; /* default 0 */
  int32_t formula_stop_iteration;  /* default 250 */
  int32_t dont_add_c_constant;     /* default 0 */
  int32_t check_for_bailout;       /* default 1 */
  double formula_weight;           /* default 1.0 */
  /* Mandelbulb: sFractalMandelbulb (src/fractal.h:227-234) */
  double bulb_power;               /* "power", default 9 */
  double bulb_alpha_angle_offset;  /* degrees, default 0 */
  double bulb_beta_angle_offset;   /* degrees, default 0 */
  /* Mandelbox: sFractalMandelbox (src/fractal.h:185-219) */
  double mandelbox_scale;                 /* default 2 */
  double mandelbox_folding_limit;         /* default 1 */
  double mandelbox_folding_value;         /* default 2 */
  double mandelbox_folding_min_radius;    /* default 0.5 */
  double mandelbox_folding_fixed_radius;  /* default 1 */
  double mandelbox_offset[3];             /* default (0,0,0) */
  /* Menger sponge: sFractalTransformCommon::scale3 (default 3) */
  double transf_scale3;
  /* Mandelbox rotations (sFractalMandelbox rotationsEnabled, rotation[2][3],
   * mainRotationEnabled, rotationMain: src/fractal.h:185-219; matrices as in
   * src/fractal.cpp:663-671).  Angles in degrees; a vector (x, y, z) is the
   * rotation RotateZ(z) RotateY(y) RotateX(x).  With rotations on, axis k of
   * the box fold is folded in the frame of rotation_neg[k] (the side above
   * the limit) or rotation_pos[k] (the side below it)
   * (formula/definition/fractal_mandelbox.cpp:33-63); the main rotation turns
   * z after the sphere fold (:103).  Only in a scene that is not a hybrid. */
  int32_t mandelbox_rotations_enabled;      /* default 0 */
  int32_t mandelbox_main_rotation_enabled;  /* default 0 */
  double mandelbox_rotation_neg[3][3];      /* "mandelbox_rotation_neg_1..3" */
  double mandelbox_rotation_pos[3][3];      /* "mandelbox_rotation_pos_1..3" */
  double mandelbox_rotation_main[3];        /* "mandelbox_rotation_main" */
  /* Kaleidoscopic IFS (formula 10): sFractalIFS (src/fractal.h:155-174),
   * read as in src/fractal.cpp:96-115, 655-661.  Angles in degrees; a vector
   * (x, y, z) is the rotation RotateZ(x) RotateY(y) RotateX(z).  Only in a
   * scene that is not a hybrid. */
  int32_t ifs_abs_x, ifs_abs_y, ifs_abs_z;   /* "IFS_abs_x/y/z", default 0 */
  int32_t ifs_rotation_enabled;              /* default 0 */
  int32_t ifs_edge_enabled;                  /* default 0 */
  int32_t ifs_menger_sponge_mode;            /* default 0 */
  int32_t ifs_enabled[9];                    /* "IFS_enabled_0..8", default 0 */
  int32_t ifs_reserved;
  double ifs_scale;                          /* default 2 */
  double ifs_rotation[3];                    /* main rotation, default 0 */
  double ifs_offset[3];                      /* default (1, 0, 0) */
  double ifs_edge[3];                        /* default 0 */
  double ifs_direction[9][3];                /* "IFS_direction_0..8", default (1, 0, 0) */
  double ifs_rotations[9][3];                /* default 0 */
  double ifs_distance[9];                    /* default 0 */
  double ifs_intensity[9];                   /* default 1 */
  /* Aexion: "cadd" (sFractalAexion, fractal.cpp:118) */
  double aexion_cadd;                        /* default -1.3 */
  /* sFractalAnalyticDE (fractal.cpp:260-265) as the Aexion reads it */
  int32_t analytic_de_enabled;               /* "analyticDE_enabled", default 1 */
  int32_t reserved_ade;
  double analytic_de_scale1;                 /* "analyticDE_scale_1", default 1 */
  double analytic_de_offset1;                /* "analyticDE_offset_1", default 1 */
  /* Formula parameters by settings key, for the formulas listed after the
   * Mandelbox in mbr_formula: each entry names one parameter of the fractal
   * container (sFractal, src/fractal.cpp:47-720, e.g.
   * "transf_addition_constant_0777", "analyticDE_tweak_005") and its value;
   * a parameter not listed keeps the reference's default
   * (InitFractalParams, src/initparameters.cpp:700-1300).  A key the slot's
   * formula does not read makes mbr_scene_set fail with MBR_EINVAL. */
  int32_t n_params;                          /* 0..MBR_MAX_FORMULA_PARAMS */
  int32_t reserved_params;
  mbr_formula_param param[MBR_MAX_FORMULA_PARAMS];
} mbr_fractal;

/* Primitive kinds (fractal::enumObjectType primitives, src/primitive.cpp) */
typedef enum mbr_primitive_type {
  MBR_PRIMITIVE_PLANE = 1,     /* z = 0, solid below (sPrimitivePlane, :459-465) */
  MBR_PRIMITIVE_BOX = 2,       /* size, rounding (sPrimitiveBox, :467-497) */
  MBR_PRIMITIVE_SPHERE = 3,    /* radius (sPrimitiveSphere, :499-511) */
  MBR_PRIMITIVE_WATER = 4,     /* wavy plane (sPrimitiveWater, :572-638) */
  MBR_PRIMITIVE_TORUS = 5,     /* radius, tube radius, their L-powers (sPrimitiveTorus, :640-655) */
  MBR_PRIMITIVE_CYLINDER = 6,  /* radius, height, caps (sPrimitiveCylinder, :522-537) */
  MBR_PRIMITIVE_CIRCLE = 7,    /* flat disc of radius (sPrimitiveCircle, :539-545) */
  MBR_PRIMITIVE_RECTANGLE = 8, /* flat width x height (sPrimitiveRectangle, :513-520) */
  MBR_PRIMITIVE_CONE = 9,      /* radius, height, caps (sPrimitiveCone, :547-564) */
  MBR_PRIMITIVE_PRISM = 10,    /* prism angle, triangle height, height (sPrimitivePrism, :657-668) */
  MBR_PRIMITIVE_ELLIPSOID = 11 /* size (sPrimitiveEllipsoid, :670-686) */
} mbr_primitive_type;

/* One primitive (the legacy primitive_<type>_<n>_* parameters,
 * src/initparameters.cpp:1313-1420) and its node transform (position,
 * rotation in degrees as CRotationMatrix::SetRotation2, uniform scale,
 * repeat period; src/objects_tree.cpp:290-385). */
typedef struct mbr_primitive {
  int32_t type;               /* mbr_primitive_type */
  int32_t empty;              /* hollow: |distance| */
  int32_t limits_enable;      /* clip to the box [limits_min, limits_max] (local frame) */
  int32_t caps;               /* cylinder: closed ends, default 1 */
  int32_t iterations;         /* water: wave octaves, default 5 */
  int32_t frame_no;           /* water: animation frame ("frame_no"), default 0 */
  double position[3];
  double rotation[3];         /* degrees */
  double scale;               /* default 1 */
  double repeat[3];           /* tiling period, 0 = none */
  double size[3];             /* box: default (1,1,1); ellipsoid: default (1,0.5,0.5) */
  double radius;              /* sphere, torus, cylinder, circle, cone: default 1 */
  double height;              /* cylinder, rectangle, cone, prism: default 1 */
  double width;               /* rectangle: default 1 */
  double tube_radius;         /* torus: default 0.2 */
  double radius_lpow;         /* torus: L-power exponent log2, default 1 */
  double tube_radius_lpow;    /* torus: default 1 */
  double rounding;            /* box: default 1e-15 */
  double wall_thickness;      /* default 0 */
  double limits_min[3];       /* default (-0.7,-0.7,-0.7); ellipsoid (-1.4,-0.7,-0.7) */
  double limits_max[3];       /* default (0.7,0.7,0.7); ellipsoid (1.4,0.7,0.7) */
  double relative_amplitude;  /* water: default 0.2 */
  double length;              /* water: default 0.1 */
  double anim_speed;          /* water: default 1 */
  double anim_progression_speed; /* water: default 1 */
  double prism_angle;         /* prism: degrees, default 60 */
  double triangle_height;     /* prism ("trangle_height"): default 1 */
} mbr_primitive;

/* enumNodeType (src/object_node_type.h:11-19). */
typedef enum mbr_node_type {
  MBR_NODE_FRACTAL = 1,      /* one formula slot, iterated alone */
  MBR_NODE_PRIMITIVE = 2,    /* one primitive */
  MBR_NODE_BOOLEAN_ADD = 11, /* union of the children (smooth union where a child asks for it) */
  MBR_NODE_BOOLEAN_MUL = 12, /* intersection of the children */
  MBR_NODE_BOOLEAN_SUB = 13  /* the first child minus the others */
} mbr_node_type;

/* One node of an explicit objects tree (cObjectsTree::sNodeData,
 * src/objects_tree.h:24-48; the node_NNNN_* parameters of
 * src/initparameters.cpp:2102-2125).  Nodes are listed in the order
 * CalculateDistanceFromObjectsTree walks them (src/calculate_distance.cpp:
 * 225-516): preorder, a boolean node's children following it one level
 * deeper.  The node's transform (position, rotation in degrees, uniform
 * scale) composes with its ancestors' (objects_tree.cpp:285-330); a leaf
 * repeats in its own frame.  A PRIMITIVE node's local transform is the
 * mbr_primitive's own position, rotation, scale and repeat. */
typedef struct mbr_node {
  int32_t type;                 /* mbr_node_type */
  int32_t level;                /* 0 for the top nodes */
  int32_t index;                /* FRACTAL: the slot of mbr_scene.fractal; PRIMITIVE: of mbr_scene.primitive */
  int32_t enabled;              /* default 1; a disabled node takes its subtree with it */
  double position[3];
  double rotation[3];           /* degrees */
  double scale;                 /* default 1 */
  double repeat[3];             /* default 0: no tiling */
  double detail_level_multiplier; /* default 1 */
  double smooth_combine_distance; /* default 0.1 */
  int32_t smooth_combine;       /* smooth union with what precedes it in a union, default 0 */
  int32_t formula_maxiter;      /* FRACTAL: default 250 */
  int32_t julia_mode;           /* FRACTAL: default 0 */
  int32_t reserved;
  double julia_c[3];            /* FRACTAL */
  double fractal_constant_factor[3]; /* FRACTAL: default (1,1,1) */
  double initial_waxis;         /* FRACTAL: default 0 */
} mbr_node;

/* The fractal part of a scene: one fractal (or hybrid) object node with the
 * general fractal parameters of src/initparameters.cpp:128-157 and the node
 * parameters of :2102-2125.  The objects tree holds exactly this one node at
 * the origin with unit scale (the reference's default scene). */
typedef struct mbr_scene {
  int32_t n_fractals;          /* 1..MBR_MAX_FRACTALS slots in use */
  int32_t hybrid_fractal_enable;
  int32_t formula_maxiter;     /* node "formula_maxiter", default 250 */
  int32_t repeat_from;         /* 1-based, default 1 */
  int32_t julia_mode;          /* default 0 */
  int32_t use_default_bailout; /* default 1 */
  int32_t delta_de_function;   /* mbr_de_function, default PREFERRED */
  int32_t min_n;               /* "minN", default 1 */
  int32_t iteration_threshold_mode; /* default 0 */
  int32_t interior_mode;       /* default 0 */
  double bailout;              /* used when use_default_bailout == 0; default 100 */
  double julia_c[3];
  double fractal_constant_factor[3]; /* default (1,1,1) */
  double initial_waxis;        /* default 0 */
  double linear_de_offset;     /* default 0 */
  mbr_fractal fractal[MBR_MAX_FRACTALS];
  /* primitives joined to the fractal by union (boolean operator OR, the
   * default of a primitive): the distance is the smallest of the fractal's
   * and theirs (objects-tree walk, src/calculate_distance.cpp:225-516) */
  int32_t n_primitives;        /* 0..MBR_MAX_PRIMITIVES, default 0 */
  int32_t reserved_prim;
  mbr_primitive primitive[MBR_MAX_PRIMITIVES];
  /* "limits_enabled": outside the box [limit_min, limit_max] by more than the
   * detail size, CalculateDistance returns the distance to the box without
   * iterating (src/calculate_distance.cpp:261-275); a soft shadow ignores
   * samples outside it (src/shader_aux_shadow.cpp:130-147) */
  int32_t limits_enabled;      /* default 0 */
  /* the global folds applied before every formula iteration
   * (src/compute_fractal.cpp:190-202, formula/definition/
   * legacy_fractal_transforrms.cpp:43-103): "box_folding" with
   * box_folding_limit / _value, "spherical_folding" with
   * spherical_folding_inner / _outer */
  int32_t box_folding;         /* default 0 */
  int32_t spherical_folding;   /* default 0 */
  int32_t reserved_folds;
  double limit_min[3];         /* default (-10, -10, -10) */
  double limit_max[3];         /* default (10, 10, 10) */
  double box_folding_limit;    /* default 1 */
  double box_folding_value;    /* default 2 */
  double spherical_folding_inner; /* default 0.5 */
  double spherical_folding_outer; /* default 1 */
  /* "delta_DE_method" (mbr_de_method, default PREFERRED): with the delta DE,
   * CalculateDistanceSimple (src/calculate_distance.cpp:607-760) runs the
   * orbit at the point and at three points offset by deltaDE along x, y and
   * z, each capped at the first orbit's iteration count, and divides the
   * orbit radius by the gradient of |z|.  deltaDE = max(|p| 1e-14, f detail)
   * with f = "deltade_relative_delta" under advanced quality, else 1e-5.
   * Offsets of 1e-5 of the detail size need FP64 points: the plain FP64
   * engines take it; the others return MBR_EUNSUPPORTED.  mbr_distance uses
   * f = 1e-5 (a render without advanced quality). */
  int32_t delta_de_method;
  int32_t reserved_delta;
  double deltade_relative_delta; /* default 0.01 (src/initparameters.cpp:166) */
  /* An explicit objects tree: with n_nodes > 0 the nodes replace the default
   * tree (the fractal or hybrid node and the primitives joined by union).
   * FRACTAL nodes iterate their slot alone, with the node's iteration limit,
   * julia and constant-factor settings (hybrid_fractal_enable must be 0);
   * the general settings above (bailout, DE method and function, minN,
   * interior and iteration-threshold modes, limits, global folds) hold for
   * every node.  Explicit trees run on the plain engines. */
  int32_t n_nodes;              /* 0..MBR_MAX_NODES, default 0 */
  int32_t reserved_nodes;
  mbr_node node[MBR_MAX_NODES];
} mbr_scene;

/* params::enumPerspectiveType (src/projection_3d.hpp:44-50): the view
 * vector of CalculateViewVector (src/projection_3d.cpp:40-89). */
typedef enum mbr_projection {
  MBR_PROJECTION_THREE_POINT = 0,     /* normalize(x fov, 1, y fov), fov = 2 tan(FOV/2) */
  MBR_PROJECTION_FISH_EYE = 1,        /* angle from the axis = |image point| * FOV (radians) */
  MBR_PROJECTION_EQUIRECTANGULAR = 2, /* longitude x FOV/2, latitude y FOV/2 */
  /* fish eye whose pixels more than 90 degrees off the axis are not traced:
   * black, depth 1e20, no hit (render_worker.cpp:165-170, 321) */
  MBR_PROJECTION_FISH_EYE_CUT = 3
} mbr_projection;

/* Camera in the reference's terms: camera/target/top vectors
 * (cCameraTarget::SetCameraTargetTop, src/camera_target.cpp:86-130) or, when
 * use_angles != 0, explicit yaw/pitch/roll in radians (viewAngle, as used by
 * PrepareMainVectors, src/render_worker.cpp:539-564), and the projection. */
typedef struct mbr_camera {
  double camera[3];
  double target[3];
  double top[3];
  double fov_deg;        /* "fov", default 53.13; (0, 180) three-point, (0, 720] the others */
  int32_t width;
  int32_t height;
  int32_t use_angles;
  int32_t perspective_type; /* mbr_projection, default three-point */
  double angles[3];      /* yaw, pitch, roll (radians) when use_angles != 0 */
  /* "legacy_coordinate_system": the image region runs from y = -0.5 at the
   * top row to +0.5 at the bottom instead of +0.5 to -0.5
   * (cRenderJob::PrepareData, src/render_job.cpp:308-315); default 0 */
  int32_t legacy_coordinate_system;
  int32_t reserved1;
} mbr_camera;

typedef struct mbr_render_params {
  double detail_level;          /* default 1 */
  double de_factor;             /* default 1 */
  double view_distance_max;     /* default 50 */
  double smoothness;            /* default 1 */
  int32_t max_raymarching_steps;/* default 10000 */
  int32_t binary_steps;         /* reference: 30 */
  int32_t refine;               /* mbr_refine */
  int32_t jitter;               /* 1: step *= 1 - Random(1000)/10000 from a per-pixel
                                   Park-Miller stream (common_math.cpp:47-72); 0: off */
  uint32_t seed;                /* jitter stream seed */
  int32_t constant_de_threshold;/* default 0 */
  double de_thresh;             /* "DE_thresh", default 0.01 */
  /* shading of the level-0 ray */
  int32_t shading_enable;       /* normals + directional light + shadow */
  int32_t shadow_enable;        /* hard AuxShadow toward the light */
  double light_direction[3];    /* direction TOWARD the light, normalised by the library */
  double light_intensity;       /* default 1 */
  double material_shading;      /* material "shading", default 1 */
  double albedo;                /* constant surface colour, default 1 */
  double ambient_intensity;     /* multiplies AO (or 1 when AO is off); default 0 */
  int32_t ao_rays;              /* 0 = no AO; else cosine-hemisphere rays per hit */
  uint32_t ao_seed;             /* PCG32 state seed of the AO stream (stream = pixel) */
  double background[3];         /* colour of missed pixels */
  /* Monte Carlo GI (path tracer) - used by mbr_render when gi_samples > 0 */
  int32_t gi_samples;           /* samples per pixel */
  int32_t gi_bounces;           /* diffuse bounces after the primary hit */
  double gi_sky;                /* constant sky radiance */
  double gi_sun;                /* sun radiance scale (directional, light_direction) */
  double dof_aperture;          /* thin lens radius; 0 = pinhole */
  double dof_focus;             /* focus distance */
  uint32_t gi_seed;             /* PCG32 state seed (stream = pixel*spp + sample) */
  int32_t row_begin;            /* render rows [row_begin, row_end) only (a band of the frame, for
                                   sharding one frame over several GPUs); 0, 0 = the whole frame.
                                   Pixels outside the band keep their buffer contents. */
  /* image adjustments (sImageAdjustments, cimage.cpp:317-362) */
  double brightness;            /* default 1 */
  double contrast;              /* default 1 */
  double gamma;                 /* default 1 */
  double saturation;            /* default 1 */
  int32_t hdr;                  /* default 0 */
  int32_t row_end;              /* 0 = the last row */
  /* the main light's shadow (cLight, light.cpp:87; AuxShadow,
   * shader_aux_shadow.cpp:55-77, 142-151, 266-301): */
  double soft_shadow_cone;      /* "soft_shadow_cone", degrees; default 1; 0 = hard shadow */
  int32_t penetrating;          /* "penetrating": march only |camera - p| * fov and darken by depth; default 1 */
  /* fast ambient occlusion (ambient_occlusion_mode "fast": FastAmbientOcclusion,
   * src/shader_fast_ambient_occlusion.cpp:40-65): quality^2 - 1 distance
   * samples along the normal instead of the ao_rays marches */
  int32_t ao_fast;              /* default 0 */
  int32_t ao_quality;           /* "ambient_occlusion_quality", default 4, 1..10 */
  double ao_fast_tune;          /* "ambient_occlusion_fast_tune", default 1 */
  /* "advanced_quality" (sParamRender, src/fractparams.cpp:48-50, 112-113,
   * 214-215): CalcDistThresh clamps the threshold to [detail_size_min,
   * detail_size_max] (src/render_worker.cpp:671-675), and RayMarching limits
   * each step by the absolute and relative bounds below instead of step <= 3
   * (:819-834).  Defaults from src/initparameters.cpp:159-165. */
  int32_t advanced_quality;     /* default 0 */
  /* "slow_shading": normals from the gradient of the orbit's iteration count
   * over an 11 x 11 x 11 lattice of points CalcDelta apart, each weighted by
   * 1 + N - iterations (src/shader_calculate_normals.cpp:83-106); plain
   * engines, scenes without primitives.  Default 0 (the six-sample DE
   * gradient). */
  int32_t slow_shading;
  double detail_size_min;       /* default 1e-12 */
  double detail_size_max;       /* default 1 */
  double abs_min_marching_step; /* default 1e-15 */
  double abs_max_marching_step; /* default 3 */
  double rel_min_marching_step; /* default 1e-2 (times the threshold) */
  double rel_max_marching_step; /* default 1e4 (times the threshold) */
} mbr_render_params;

/* Per-launch counters (src/statistics.h:42-70 mirrored).  A DE evaluation
 * is one CalculateDistance call; formula_iterations sums its `iters`. */
typedef struct mbr_stats {
  unsigned long long de_evals;
  unsigned long long formula_iterations;
  unsigned long long march_steps;
  unsigned long long binary_steps;
  unsigned long long normal_evals;
  unsigned long long shadow_evals;
  unsigned long long ao_evals;
  unsigned long long gi_evals;
  unsigned long long pixels;
  unsigned long long watchdog_trips;
} mbr_stats;

/* Caller-owned device buffers, each width*height elements (x3 for vectors),
 * row-major, pixel (x,y) at y*width + x.  Any pointer may be NULL. */
typedef struct mbr_outputs {
  double *depth;      /* scan distance of the hit; 1e20 when nothing was hit */
  int32_t *iters;     /* iters of the last DE evaluation of the primary march */
  uint8_t *hit;       /* 1 when the primary ray found the surface */
  float *normal;      /* world-space unit normal (0,0,0 on miss) */
  float *shade;       /* Lambert term incl. shadow, before albedo/ambient */
  float *ao;          /* ambient occlusion in [0,1] (1 when off) */
  float *rgb;         /* linear colour */
  uint8_t *rgb8;      /* 8-bit colour after CalculatePixel + ConvertTo8bitChar */
  mbr_stats *stats;   /* device counters, ADDED to (caller zeroes them) */
} mbr_outputs;

typedef struct mbr_ctx mbr_ctx;
typedef struct mbr_batch mbr_batch;

/* ---- context ----------------------------------------------------------- */
/* Library version string. */
const char *mbr_version(void);
/* Creates a context on `device`.  Replaces the per-render set-up of
 * cRenderer::RenderImage (src/render_image.cpp:354-485). */
mbr_status mbr_create(mbr_ctx **out, int device);
void mbr_destroy(mbr_ctx *ctx);
const char *mbr_last_error_string(const mbr_ctx *ctx);

/* Fill structs with the reference defaults (src/initparameters.cpp). */
void mbr_scene_defaults(mbr_scene *scene);
void mbr_fractal_defaults(mbr_fractal *fractal, int formula);
void mbr_primitive_defaults(mbr_primitive *primitive, int type);
void mbr_camera_defaults(mbr_camera *camera);
void mbr_render_params_defaults(mbr_render_params *params);

/* Validates a scene and builds its hybrid sequence
 * (cHybridFractalSequences::CreateSequences, hybrid_fractal_sequences.cpp:27-499)
 * on the host, then uploads it.  Replaces cRenderJob's sequence set-up
 * (src/render_job.cpp:300-351). */
mbr_status mbr_scene_set(mbr_ctx *ctx, const mbr_scene *scene);

/* Host helper: the camera rotation matrix (row-major 3x3) and view angles
 * exactly as PrepareMainVectors builds mRot (render_worker.cpp:539-564). */
mbr_status mbr_camera_rotation(const mbr_camera *camera, double mrot[9], double angles[3]);

/* Host helper: the hybrid sequence table built for `scene` (length entries of
 * slot indices) - the product of CreateSequence, exposed for testing. */
mbr_status mbr_scene_sequence(const mbr_scene *scene, int32_t *seq_out, int32_t *length_out,
                              int32_t *de_function_out, double *bailout_out);

/* Renders one frame of the current scene: the body of cRenderWorker::doWork
 * for every pixel (render_worker.cpp:126-525) on `stream`.  Asynchronous:
 * returns after the launches are queued.  Call mbr_sync to wait and to read
 * the watchdog status. */
mbr_status mbr_render(mbr_ctx *ctx, const mbr_camera *camera, const mbr_render_params *params,
                      const mbr_outputs *out, int engine, void *stream);

/* Waits for `stream` and reads (and clears) the context's device status word:
 * MBR_ETIMEOUT when a kernel's bounded loop ran out of its budget since the
 * last mbr_sync - an AO march that reached max_raymarching_steps (the
 * reference's AO march has no cap; the march is ended as unoccluded and
 * counted in mbr_stats.watchdog_trips).  The frame itself is complete. */
mbr_status mbr_sync(mbr_ctx *ctx, void *stream);

/* Distance estimate at n points (device arrays, xyz interleaved): the
 * reference's CalculateDistance, also what distance_engine.cl:42 computes.
 * normal_mode selects sDistanceIn::normalCalculationMode. */
mbr_status mbr_distance(mbr_ctx *ctx, const double *points, int64_t n, double detail_size,
                        int normal_mode, double *dist, int32_t *iters, int engine, void *stream);

/* ---- batches of render jobs (one persistent, graph-captured launch) ---- */
typedef struct mbr_job {
  mbr_camera camera;
  int32_t scene_index;   /* into the scenes array of mbr_batch_create */
  int32_t reserved0;
  int64_t pixel_offset;  /* first pixel of this job in the batch outputs */
} mbr_job;

/* Builds the job table for n_jobs renders of uneven size and captures the
 * launch into a CUDA graph: one pipeline per formula kind and precision, each
 * over its jobs with one persistent launch per stage.  Outputs are indexed
 * pixel_offset + y*width + x.  engine must be a WAVEFRONT engine; with
 * MBR_ENGINE_WAVEFRONT_AUTO the precision is chosen per job here (a
 * synchronous device evaluation of DE at every camera). */
mbr_status mbr_batch_create(mbr_ctx *ctx, const mbr_scene *scenes, int32_t n_scenes,
                            const mbr_job *jobs, int32_t n_jobs,
                            const mbr_render_params *params, const mbr_outputs *out,
                            int engine, void *stream, mbr_batch **batch);
/* Replays the captured graph on `stream`. */
mbr_status mbr_batch_launch(mbr_batch *batch, void *stream);
void mbr_batch_destroy(mbr_batch *batch);
/* Number of pipelines in the batch's graph (one per formula kind and
 * precision) and, in *wide_jobs (may be NULL), how many jobs iterate in FP64;
 * -1 for a NULL batch. */
int32_t mbr_batch_groups(const mbr_batch *batch, int32_t *wide_jobs);

/* Host helper (no device call): the layout of the wavefront engines' scratch
 * for a launch over `pixels` work items with `tasks_per_hit` shadow/AO tasks
 * per hit.  offsets[0..2] receive the byte offsets of the hit records, the
 * FP32 start records and the shadow/AO direction records; *total_bytes the
 * size.  Both record regions start on a 16-byte boundary for every pixel
 * count.  No counterpart in the reference (exposed for testing). */
mbr_status mbr_wavefront_scratch_layout(int64_t pixels, int32_t tasks_per_hit, uint64_t offsets[3],
                                        uint64_t *total_bytes);

/* The precision MBR_ENGINE_WAVEFRONT_AUTO uses for the current scene seen
 * from `camera` with `params`: *fp64 = 1 for FP64 iteration, 0 for FP32.
 * Synchronous (one device evaluation of DE at the camera). */
mbr_status mbr_choose_precision(mbr_ctx *ctx, const mbr_camera *camera, const mbr_render_params *params,
                                int32_t *fp64);

/* Launch configuration of the wavefront kernel, chosen by the autotuner. */
typedef struct mbr_tuning {
  int32_t block_size;     /* threads per CTA */
  int32_t ctas_per_sm;    /* persistent CTAs per SM */
  int32_t refill_k;       /* re-converge finished lanes once <= k lanes still iterate */
  int32_t queue_layout;   /* 0 = row-linear pixel queue, 1 = 8x4 tiles */
} mbr_tuning;

/* Sets / reads the wavefront launch configuration of the context. */
mbr_status mbr_set_tuning(mbr_ctx *ctx, const mbr_tuning *tuning);
mbr_status mbr_get_tuning(const mbr_ctx *ctx, mbr_tuning *tuning);

/* Times the wavefront kernel over a grid of configurations on the given
 * camera (outputs are scratch the caller provides) and keeps the fastest. */
mbr_status mbr_autotune(mbr_ctx *ctx, const mbr_camera *camera, const mbr_render_params *params,
                        const mbr_outputs *out, int engine, void *stream, mbr_tuning *best);

/* ---- adjoint ------------------------------------------------------------ */
/* Parameters the adjoint differentiates, in this order. */
enum {
  MBR_GRAD_BULB_POWER = 0,
  MBR_GRAD_MANDELBOX_SCALE = 1,
  MBR_GRAD_MANDELBOX_MIN_R2 = 2,   /* w.r.t. min radius squared (mR2) */
  MBR_GRAD_CAMERA_X = 3,           /* camera position at fixed view angles */
  MBR_GRAD_CAMERA_Y = 4,
  MBR_GRAD_CAMERA_Z = 5,
  MBR_GRAD_YAW = 6,
  MBR_GRAD_COUNT = 8               /* array length (last entry unused) */
};

/* Gradient of a per-pixel loss L(depth, shade) with respect to the
 * MBR_GRAD_* parameters of slot 0 of the current (non-hybrid) scene and of
 * the camera (given with use_angles = 1), by implicit differentiation at the
 * hit: with F(t) = dist(o + t d) - threshold(t),
 *   dt/dθ = -(∂dist/∂θ + ∇dist·∂p/∂θ) / (∇dist·d - ∂threshold/∂t).
 * depth and hit are the forward outputs (rendered with MBR_REFINE_ROOT);
 * dl_ddepth / dl_dshade are dL/d(depth) and dL/d(shade) per pixel (device,
 * may be NULL = 0).  The shade term differentiates the central-difference
 * normal of CalculateNormals through its six DE evaluations; the formula
 * iteration is recomputed in forward-mode tangents.  grad (device, 8 doubles)
 * is ADDED to.  `engine` selects FP64 (PLAIN_FP64) or FP32 (PLAIN_MIXED)
 * recomputation. */
mbr_status mbr_adjoint(mbr_ctx *ctx, const mbr_camera *camera, const mbr_render_params *params,
                       const double *depth, const uint8_t *hit, const float *dl_ddepth,
                       const float *dl_dshade, double *grad, int engine, void *stream);

/* ---- allocation-free rendering ------------------------------------------------- */
/* Size of the device scratch array that mbr_render_noalloc works in. */
#define MBR_NOALLOC_SCRATCH_BYTES (64u * 1024u * 1024u)

/* Renders one frame with the FP32 wavefront engine, like mbr_render with
 * MBR_ENGINE_WAVEFRONT_FP32, without allocating any device memory and without
 * a context.  No counterpart in the reference: it is for callers that cannot
 * allocate device memory - applications whose device memory belongs to their
 * own allocator or pool, or processes under a hard memory cap where a
 * cudaMalloc during a frame could fail or synchronise the device.
 *
 * All scratch lives in one static device array of MBR_NOALLOC_SCRATCH_BYTES
 * (64 MiB) that every GPU loading this library holds until the process exits.
 * A frame needs 128 KiB + 512 B + pixels * (88 + 16 * (1 + tasks)) bytes, with
 * tasks = ao_rays + 1 when the shadow march runs and the 88-byte hit records
 * rounded up to a multiple of 256 bytes; larger frames are rejected with
 * MBR_EINVAL and the limit in `err` (178,130 pixels with a shadow and 16 AO
 * rays, 644,011 with neither).  The caller passes the scene, camera,
 * parameters and device output buffers as for mbr_render; `err` (may be NULL)
 * receives a message of at most err_len bytes on failure.
 *
 * The first call on a device looks up the array's device address on the
 * current device (cudaGetSymbolAddress); make that first call before any
 * stream capture.  Every call shares the one array and keeps the previous
 * call's contents; calls that overlap on the GPU (other streams, other
 * threads) race on it, so serialise them.  Asynchronous: returns after the
 * launches are queued on `stream`. */
mbr_status mbr_render_noalloc(const mbr_scene *scene, const mbr_camera *camera, const mbr_render_params *params,
                              const mbr_outputs *out, void *stream, char *err, size_t err_len);

/* ---- settings files ------------------------------------------------------------ */
/* Reads the text of a mandelbulber2 settings file (.fract, the flat form of
 * versions up to 2.34 that the reference's example scenes use: header lines,
 * [main_parameters], [fractal_N]) into a scene, a camera and render
 * parameters.  Replaces, for the DE path, cSettings::LoadFromString + Decode
 * (src/settings.cpp:513-527, 647-977) followed by the parameter structs the
 * path reads (sParamRender, src/fractparams.cpp:42-362; sFractal,
 * src/fractal.cpp:47-89).  Unlisted parameters keep the reference's defaults
 * (src/initparameters.cpp).
 *
 * MBR_OK: everything that changes the geometry is representable.
 * MBR_EUNSUPPORTED: the structs are filled, but the file uses geometry this
 * path does not build (another formula, boolean combinations, primitives
 * combined other than by union, more than 8 primitives, a transform of the
 * primitives group, formula and fractal transforms, the analytic Jos
 * Kleinian DE function, iteration-count normals, stereo images); each is
 * named in the report.  The eleven primitive kinds joined by union, advanced
 * quality, the limits box, the global folds and the DE method and function
 * (the delta DE included) are read into the structs.
 * MBR_EINVAL: not a settings file, or a malformed value of a
 * parameter read here.  The report (optional, NUL-terminated, truncated to
 * report_size) also lists the shading parameters outside the path that were
 * ignored, and how the main light and AO were mapped. */
mbr_status mbr_fract_parse(const char *text, mbr_scene *scene, mbr_camera *camera, mbr_render_params *params,
                           char *report, int32_t report_size);

/* ---- measurement ------------------------------------------------------------ */
/* FMA throughput of the current device (FLOP/s, an FMA counted as 2), FP32
 * (fp64 = 0) or FP64: the roofline denominator for the DE kernels, which are
 * bound by the FMA/SFU pipes.  Synchronous.  No counterpart in the reference. */
mbr_status mbr_fma_peak(int fp64, int iters, void *stream, double *flops_per_s);

#ifdef __cplusplus
}
#endif
#endif /* MBR_H_ */
