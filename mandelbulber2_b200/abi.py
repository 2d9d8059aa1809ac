"""ctypes mirror of ``include/mbr.h`` (the C-ABI of ``libmbr.so``).

The structures below are field-for-field copies of the C structs; their sizes
are checked against the C declarations by the CPU tests.  This module only
loads the library; it performs no GPU work.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmbr.so")

MBR_MAX_FRACTALS = 9
MBR_SEQUENCE_LENGTH = 1250
MBR_MAX_PRIMITIVES = 8
MBR_MAX_NODES = 16
# mbr_node_type
NODE_FRACTAL, NODE_PRIMITIVE, NODE_BOOLEAN_ADD, NODE_BOOLEAN_MUL, NODE_BOOLEAN_SUB = 1, 2, 11, 12, 13

# mbr_status
MBR_OK, MBR_EINVAL, MBR_ECUDA, MBR_ETIMEOUT, MBR_ENOMEM, MBR_EUNSUPPORTED = range(6)
STATUS_NAMES = {0: "MBR_OK", 1: "MBR_EINVAL", 2: "MBR_ECUDA", 3: "MBR_ETIMEOUT", 4: "MBR_ENOMEM",
                5: "MBR_EUNSUPPORTED"}

# mbr_formula (fractal::enumFractalFormula)
FORMULA_NONE, FORMULA_MANDELBULB, FORMULA_MENGER_SPONGE, FORMULA_MANDELBOX = 0, 2, 7, 8
FORMULA_MANDELBULB_POWER2, FORMULA_HYPERCOMPLEX, FORMULA_KALEIDOSCOPIC_IFS, FORMULA_XENODREAMBUIE = 3, 4, 10, 11
FORMULA_QUATERNION, FORMULA_AEXION = 5, 19
# formulas whose parameters are passed by settings key (Fractal.param)
FORMULA_BOX_FOLD_BULB_POW2, FORMULA_MENGER_MOD1, FORMULA_PSEUDO_KLEINIAN = 16, 61, 103
FORMULA_BOX_FOLD_BULB_POW2_V2, FORMULA_ABOX_MOD11, FORMULA_PSEUDO_KLEINIAN_MOD4 = 125, 119, 217
FORMULA_PSEUDO_KLEINIAN_STD_DE, FORMULA_GENERALIZED_FOLD_BOX, FORMULA_MANDELBULB_PUPUKU = 101, 37, 266
FORMULA_DIFS_HEXTGRID2 = 608
MBR_MAX_FORMULA_PARAMS = 48
MBR_PARAM_KEY_LEN = 48
PROJECTION_THREE_POINT, PROJECTION_FISH_EYE, PROJECTION_EQUIRECTANGULAR, PROJECTION_FISH_EYE_CUT = range(4)
# mbr_primitive_type
(PRIMITIVE_PLANE, PRIMITIVE_BOX, PRIMITIVE_SPHERE, PRIMITIVE_WATER, PRIMITIVE_TORUS, PRIMITIVE_CYLINDER,
 PRIMITIVE_CIRCLE, PRIMITIVE_RECTANGLE, PRIMITIVE_CONE, PRIMITIVE_PRISM, PRIMITIVE_ELLIPSOID) = range(1, 12)
# mbr_de_function
DE_PREFERRED, DE_LINEAR, DE_LOG, DE_PSEUDO_KLEINIAN, DE_JOS_KLEINIAN, DE_CUSTOM, DE_MAX_AXIS = range(7)
# mbr_de_method
DE_METHOD_PREFERRED, DE_METHOD_FORCE_DELTA, DE_METHOD_FORCE_ANALYTIC = range(3)
# mbr_engine
ENGINE_PLAIN_FP64, ENGINE_PLAIN_FP64_STRICT, ENGINE_PLAIN_MIXED, ENGINE_WAVEFRONT_FP32, ENGINE_WAVEFRONT_FP64, \
    ENGINE_WAVEFRONT_AUTO = range(6)
ENGINE_NAMES = {0: "plain_fp64", 1: "plain_fp64_strict", 2: "plain_mixed", 3: "wavefront_fp32", 4: "wavefront_fp64",
                5: "wavefront_auto"}
# mbr_refine
REFINE_REFERENCE, REFINE_ROOT = 0, 1
# gradient slots
GRAD_BULB_POWER, GRAD_MANDELBOX_SCALE, GRAD_MANDELBOX_MIN_R2 = 0, 1, 2
GRAD_CAMERA_X, GRAD_CAMERA_Y, GRAD_CAMERA_Z, GRAD_YAW, GRAD_COUNT = 3, 4, 5, 6, 8

D3 = C.c_double * 3


class FormulaParam(C.Structure):
    _fields_ = [("key", C.c_char * MBR_PARAM_KEY_LEN), ("value", D3)]


class Fractal(C.Structure):
    _fields_ = [
        ("formula", C.c_int32), ("formula_iterations", C.c_int32), ("formula_start_iteration", C.c_int32),
        ("formula_stop_iteration", C.c_int32), ("dont_add_c_constant", C.c_int32), ("check_for_bailout", C.c_int32),
        ("formula_weight", C.c_double),
        ("bulb_power", C.c_double), ("bulb_alpha_angle_offset", C.c_double), ("bulb_beta_angle_offset", C.c_double),
        ("mandelbox_scale", C.c_double), ("mandelbox_folding_limit", C.c_double),
        ("mandelbox_folding_value", C.c_double), ("mandelbox_folding_min_radius", C.c_double),
        ("mandelbox_folding_fixed_radius", C.c_double), ("mandelbox_offset", D3),
        ("transf_scale3", C.c_double),
        ("mandelbox_rotations_enabled", C.c_int32), ("mandelbox_main_rotation_enabled", C.c_int32),
        ("mandelbox_rotation_neg", D3 * 3), ("mandelbox_rotation_pos", D3 * 3), ("mandelbox_rotation_main", D3),
        ("ifs_abs_x", C.c_int32), ("ifs_abs_y", C.c_int32), ("ifs_abs_z", C.c_int32),
        ("ifs_rotation_enabled", C.c_int32), ("ifs_edge_enabled", C.c_int32), ("ifs_menger_sponge_mode", C.c_int32),
        ("ifs_enabled", C.c_int32 * 9), ("ifs_reserved", C.c_int32),
        ("ifs_scale", C.c_double), ("ifs_rotation", D3), ("ifs_offset", D3), ("ifs_edge", D3),
        ("ifs_direction", D3 * 9), ("ifs_rotations", D3 * 9), ("ifs_distance", C.c_double * 9),
        ("ifs_intensity", C.c_double * 9),
        ("aexion_cadd", C.c_double), ("analytic_de_enabled", C.c_int32), ("reserved_ade", C.c_int32),
        ("analytic_de_scale1", C.c_double), ("analytic_de_offset1", C.c_double),
        ("n_params", C.c_int32), ("reserved_params", C.c_int32),
        ("param", FormulaParam * MBR_MAX_FORMULA_PARAMS),
    ]

    def set_param(self, key: str, value) -> None:
        """Sets formula parameter `key` (the reference's settings name) to a
        number, a bool or a 3-vector, replacing an earlier value of the key."""
        v = list(value) if isinstance(value, (list, tuple)) else [float(value), 0.0, 0.0]
        k = key.encode()
        if len(k) >= MBR_PARAM_KEY_LEN:
            raise ValueError(f"parameter key longer than {MBR_PARAM_KEY_LEN - 1} bytes: {key}")
        for i in range(self.n_params):
            if self.param[i].key == k:
                self.param[i].value[:] = [float(x) for x in v]
                return
        if self.n_params >= MBR_MAX_FORMULA_PARAMS:
            raise ValueError("too many formula parameters")
        p = self.param[self.n_params]
        p.key = k
        p.value[:] = [float(x) for x in v]
        self.n_params += 1

    def params(self) -> dict:
        """The listed formula parameters, key -> (x, y, z)."""
        return {self.param[i].key.decode(): tuple(self.param[i].value) for i in range(self.n_params)}


class Primitive(C.Structure):
    _fields_ = [
        ("type", C.c_int32), ("empty", C.c_int32), ("limits_enable", C.c_int32), ("caps", C.c_int32),
        ("iterations", C.c_int32), ("frame_no", C.c_int32), ("position", D3), ("rotation", D3),
        ("scale", C.c_double), ("repeat", D3), ("size", D3), ("radius", C.c_double), ("height", C.c_double),
        ("width", C.c_double), ("tube_radius", C.c_double), ("radius_lpow", C.c_double),
        ("tube_radius_lpow", C.c_double), ("rounding", C.c_double), ("wall_thickness", C.c_double),
        ("limits_min", D3), ("limits_max", D3), ("relative_amplitude", C.c_double), ("length", C.c_double),
        ("anim_speed", C.c_double), ("anim_progression_speed", C.c_double), ("prism_angle", C.c_double),
        ("triangle_height", C.c_double),
    ]


class Node(C.Structure):
    _fields_ = [
        ("type", C.c_int32), ("level", C.c_int32), ("index", C.c_int32), ("enabled", C.c_int32),
        ("position", D3), ("rotation", D3), ("scale", C.c_double), ("repeat", D3),
        ("detail_level_multiplier", C.c_double), ("smooth_combine_distance", C.c_double),
        ("smooth_combine", C.c_int32), ("formula_maxiter", C.c_int32), ("julia_mode", C.c_int32),
        ("reserved", C.c_int32), ("julia_c", D3), ("fractal_constant_factor", D3), ("initial_waxis", C.c_double),
    ]


def node_defaults(node_type: int, index: int = 0, level: int = 0) -> Node:
    """A node with the reference's node defaults (initparameters.cpp:2102-2125)."""
    n = Node()
    n.type, n.index, n.level, n.enabled = node_type, index, level, 1
    n.scale = 1.0
    n.detail_level_multiplier = 1.0
    n.smooth_combine_distance = 0.1
    n.formula_maxiter = 250
    n.fractal_constant_factor[:] = [1.0, 1.0, 1.0]
    return n


class Scene(C.Structure):
    _fields_ = [
        ("n_fractals", C.c_int32), ("hybrid_fractal_enable", C.c_int32), ("formula_maxiter", C.c_int32),
        ("repeat_from", C.c_int32), ("julia_mode", C.c_int32), ("use_default_bailout", C.c_int32),
        ("delta_de_function", C.c_int32), ("min_n", C.c_int32), ("iteration_threshold_mode", C.c_int32),
        ("interior_mode", C.c_int32), ("bailout", C.c_double), ("julia_c", D3),
        ("fractal_constant_factor", D3), ("initial_waxis", C.c_double), ("linear_de_offset", C.c_double),
        ("fractal", Fractal * MBR_MAX_FRACTALS),
        ("n_primitives", C.c_int32), ("reserved_prim", C.c_int32), ("primitive", Primitive * MBR_MAX_PRIMITIVES),
        ("limits_enabled", C.c_int32), ("box_folding", C.c_int32), ("spherical_folding", C.c_int32),
        ("reserved_folds", C.c_int32), ("limit_min", D3), ("limit_max", D3), ("box_folding_limit", C.c_double),
        ("box_folding_value", C.c_double), ("spherical_folding_inner", C.c_double),
        ("spherical_folding_outer", C.c_double),
        ("delta_de_method", C.c_int32), ("reserved_delta", C.c_int32), ("deltade_relative_delta", C.c_double),
        ("n_nodes", C.c_int32), ("reserved_nodes", C.c_int32), ("node", Node * MBR_MAX_NODES),
    ]


class Camera(C.Structure):
    _fields_ = [
        ("camera", D3), ("target", D3), ("top", D3), ("fov_deg", C.c_double), ("width", C.c_int32),
        ("height", C.c_int32), ("use_angles", C.c_int32), ("perspective_type", C.c_int32), ("angles", D3),
        ("legacy_coordinate_system", C.c_int32), ("reserved1", C.c_int32),
    ]


class RenderParams(C.Structure):
    _fields_ = [
        ("detail_level", C.c_double), ("de_factor", C.c_double), ("view_distance_max", C.c_double),
        ("smoothness", C.c_double), ("max_raymarching_steps", C.c_int32), ("binary_steps", C.c_int32),
        ("refine", C.c_int32), ("jitter", C.c_int32), ("seed", C.c_uint32), ("constant_de_threshold", C.c_int32),
        ("de_thresh", C.c_double), ("shading_enable", C.c_int32), ("shadow_enable", C.c_int32),
        ("light_direction", D3), ("light_intensity", C.c_double), ("material_shading", C.c_double),
        ("albedo", C.c_double), ("ambient_intensity", C.c_double), ("ao_rays", C.c_int32),
        ("ao_seed", C.c_uint32), ("background", D3), ("gi_samples", C.c_int32), ("gi_bounces", C.c_int32),
        ("gi_sky", C.c_double), ("gi_sun", C.c_double), ("dof_aperture", C.c_double), ("dof_focus", C.c_double),
        ("gi_seed", C.c_uint32), ("row_begin", C.c_int32), ("brightness", C.c_double), ("contrast", C.c_double),
        ("gamma", C.c_double), ("saturation", C.c_double), ("hdr", C.c_int32), ("row_end", C.c_int32),
        ("soft_shadow_cone", C.c_double), ("penetrating", C.c_int32), ("ao_fast", C.c_int32),
        ("ao_quality", C.c_int32), ("ao_fast_tune", C.c_double),
        ("advanced_quality", C.c_int32), ("slow_shading", C.c_int32), ("detail_size_min", C.c_double),
        ("detail_size_max", C.c_double), ("abs_min_marching_step", C.c_double),
        ("abs_max_marching_step", C.c_double), ("rel_min_marching_step", C.c_double),
        ("rel_max_marching_step", C.c_double),
    ]


class Stats(C.Structure):
    _fields_ = [(n, C.c_ulonglong) for n in (
        "de_evals", "formula_iterations", "march_steps", "binary_steps", "normal_evals", "shadow_evals",
        "ao_evals", "gi_evals", "pixels", "watchdog_trips")]


class Outputs(C.Structure):
    _fields_ = [
        ("depth", C.c_void_p), ("iters", C.c_void_p), ("hit", C.c_void_p), ("normal", C.c_void_p),
        ("shade", C.c_void_p), ("ao", C.c_void_p), ("rgb", C.c_void_p), ("rgb8", C.c_void_p),
        ("stats", C.c_void_p),
    ]


class Job(C.Structure):
    _fields_ = [("camera", Camera), ("scene_index", C.c_int32), ("reserved0", C.c_int32),
                ("pixel_offset", C.c_int64)]


class Tuning(C.Structure):
    _fields_ = [("block_size", C.c_int32), ("ctas_per_sm", C.c_int32), ("refill_k", C.c_int32),
                ("queue_layout", C.c_int32)]


# Every function the header declares: name -> (restype, argtypes).
_P = C.c_void_p
PROTOTYPES = {
    "mbr_version": (C.c_char_p, []),
    "mbr_create": (C.c_int, [C.POINTER(_P), C.c_int]),
    "mbr_destroy": (None, [_P]),
    "mbr_last_error_string": (C.c_char_p, [_P]),
    "mbr_scene_defaults": (None, [C.POINTER(Scene)]),
    "mbr_fractal_defaults": (None, [C.POINTER(Fractal), C.c_int]),
    "mbr_primitive_defaults": (None, [C.POINTER(Primitive), C.c_int]),
    "mbr_camera_defaults": (None, [C.POINTER(Camera)]),
    "mbr_render_params_defaults": (None, [C.POINTER(RenderParams)]),
    "mbr_scene_set": (C.c_int, [_P, C.POINTER(Scene)]),
    "mbr_camera_rotation": (C.c_int, [C.POINTER(Camera), C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "mbr_scene_sequence": (C.c_int, [C.POINTER(Scene), C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                     C.POINTER(C.c_int32), C.POINTER(C.c_double)]),
    "mbr_render": (C.c_int, [_P, C.POINTER(Camera), C.POINTER(RenderParams), C.POINTER(Outputs), C.c_int, _P]),
    "mbr_sync": (C.c_int, [_P, _P]),
    "mbr_distance": (C.c_int, [_P, _P, C.c_int64, C.c_double, C.c_int, _P, _P, C.c_int, _P]),
    "mbr_batch_create": (C.c_int, [_P, C.POINTER(Scene), C.c_int32, C.POINTER(Job), C.c_int32,
                                   C.POINTER(RenderParams), C.POINTER(Outputs), C.c_int, _P, C.POINTER(_P)]),
    "mbr_batch_launch": (C.c_int, [_P, _P]),
    "mbr_batch_destroy": (None, [_P]),
    "mbr_batch_groups": (C.c_int32, [_P, _P]),
    "mbr_wavefront_scratch_layout": (C.c_int, [C.c_int64, C.c_int32, C.POINTER(C.c_uint64),
                                               C.POINTER(C.c_uint64)]),
    "mbr_choose_precision": (C.c_int, [_P, _P, _P, _P]),
    "mbr_set_tuning": (C.c_int, [_P, C.POINTER(Tuning)]),
    "mbr_get_tuning": (C.c_int, [_P, C.POINTER(Tuning)]),
    "mbr_autotune": (C.c_int, [_P, C.POINTER(Camera), C.POINTER(RenderParams), C.POINTER(Outputs), C.c_int, _P,
                               C.POINTER(Tuning)]),
    "mbr_adjoint": (C.c_int, [_P, C.POINTER(Camera), C.POINTER(RenderParams), _P, _P, _P, _P, _P, C.c_int, _P]),
    "mbr_fma_peak": (C.c_int, [C.c_int, C.c_int, _P, C.POINTER(C.c_double)]),
    "mbr_render_noalloc": (C.c_int, [C.POINTER(Scene), C.POINTER(Camera), C.POINTER(RenderParams),
                                     C.POINTER(Outputs), _P, C.c_char_p, C.c_size_t]),
    "mbr_fract_parse": (C.c_int, [C.c_char_p, C.POINTER(Scene), C.POINTER(Camera), C.POINTER(RenderParams),
                                  C.c_char_p, C.c_int32]),
}

_lib = None


def load(path: str | None = None) -> C.CDLL:
    """Loads libmbr.so (built in-tree) and declares its prototypes.

    Raises RuntimeError when the library is missing: there is no fallback.
    """
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(f"{p} is missing; build it with `python -m mandelbulber2_b200.build`")
    lib = C.CDLL(p)
    for name, (res, args) in PROTOTYPES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


# Where the struct defaults come from: this library's mbr_*_defaults, or
# another library exporting the same functions under another prefix (a CPU
# program that must not load libmbr.so, see use_defaults_from).
_defaults_src = None  # (library, prefix)


def use_defaults_from(lib: C.CDLL | None, prefix: str = "mbr_") -> None:
    """Takes the struct defaults from `lib`'s <prefix>scene_defaults,
    fractal_defaults, camera_defaults and render_params_defaults (same
    signatures as mbr_*); None restores libmbr.so."""
    global _defaults_src
    _defaults_src = None if lib is None else (lib, prefix)


def _defaults_fn(name: str):
    lib, prefix = _defaults_src if _defaults_src is not None else (load(), "mbr_")
    return getattr(lib, prefix + name)


def fractal_defaults(f: Fractal, formula: int) -> None:
    _defaults_fn("fractal_defaults")(C.byref(f), formula)


def scene_defaults(formula: int = FORMULA_MANDELBULB) -> Scene:
    s = Scene()
    _defaults_fn("scene_defaults")(C.byref(s))
    fractal_defaults(s.fractal[0], formula)
    return s


def primitive_defaults(kind: int) -> Primitive:
    q = Primitive()
    load().mbr_primitive_defaults(C.byref(q), kind)
    return q


def camera_defaults() -> Camera:
    c = Camera()
    _defaults_fn("camera_defaults")(C.byref(c))
    return c


def params_defaults() -> RenderParams:
    p = RenderParams()
    _defaults_fn("render_params_defaults")(C.byref(p))
    return p


def library_loaded() -> bool:
    """True once this process has loaded libmbr.so through load()."""
    return _lib is not None
