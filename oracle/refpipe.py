"""ctypes wrapper of oracle/_ref/librefpipe.so: the reference's own sources
for the distance-estimation path (parameter containers with the reference's
defaults, objects tree, sequences, Compute, CalculateDistance and the render
worker), compiled here by oracle/build_ref.sh.

TEST INFRASTRUCTURE ONLY: used by tests/golden/make_golden.py to write golden
vectors and by the CPU tests that pin the oracle against the reference.  It
needs the reference tree at build time, so it exists only where that tree
was; everything that runs elsewhere reads the committed fixtures instead.

`configure` writes a scene / camera / render-parameter triple of the C-ABI
structs into the reference's containers under the reference's own parameter
names (those of src/initparameters.cpp and the settings files).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "librefpipe.so")
_P = C.c_void_p

KIND_INT, KIND_DOUBLE, KIND_BOOL, KIND_VEC3 = 0, 1, 2, 3
NODE_FRACTAL, NODE_HYBRID = 1, 10  # enumNodeType (object_node_type.h:11-19)
NODE_FRACTAL_T, NODE_PRIMITIVE_T = 1, 2
# mbr_primitive_type -> the reference's primitive type names (primitives.cpp:60-100)
PRIMITIVE_NAMES = {1: "plane", 2: "box", 3: "sphere", 4: "water", 5: "torus", 6: "cylinder", 7: "circle",
                   8: "rectangle", 9: "cone", 10: "prism", 11: "ellipsoid"}


def available() -> bool:
    return os.path.exists(LIB)


class RefPipeline:
    """One set of reference containers (main + nine fractal slots)."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            L = C.CDLL(LIB)
            L.refp_new.restype = _P
            L.refp_free.argtypes = [_P]
            L.refp_set.argtypes = [_P, C.c_int, C.c_char_p, C.c_int, _P]
            L.refp_set_string.argtypes = [_P, C.c_int, C.c_char_p, C.c_char_p]
            L.refp_param_kind.argtypes = [_P, C.c_int, C.c_char_p]
            L.refp_add_node.argtypes = [_P, C.c_int]
            L.refp_add_primitive.argtypes = [_P, C.c_char_p, C.c_int]
            L.refp_prepare.argtypes = [_P]
            L.refp_distance.argtypes = [_P, _P, C.c_int, C.c_double, C.c_int, _P, _P]
            L.refp_compute.argtypes = [_P, _P, C.c_int, C.c_int, _P, _P, _P, _P]
            L.refp_sequence.argtypes = [_P, _P, C.c_int, _P, _P, _P, _P, _P, _P]
            L.refp_light_direction.argtypes = [_P, C.c_int, _P]
            L.refp_render.argtypes = [_P, C.c_uint, _P, _P, _P, _P]
            cls._lib = L
        return cls._lib

    def __init__(self):
        self.L = self.lib()
        self.h = self.L.refp_new()

    def close(self):
        if self.h:
            self.L.refp_free(self.h)
            self.h = None

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass

    def set(self, name: str, value, kind: int, fractal: int = -1) -> None:
        v = list(value) if kind == KIND_VEC3 else [float(value), 0.0, 0.0]
        arr = (C.c_double * 3)(*v)
        rc = self.L.refp_set(self.h, fractal, name.encode(), kind, arr)
        if rc:
            raise KeyError(f"reference parameter {name!r} (fractal {fractal}): {rc}")

    def set_string(self, name: str, value: str, fractal: int = -1) -> None:
        if self.L.refp_set_string(self.h, fractal, name.encode(), value.encode()):
            raise KeyError(name)

    def add_node(self, node_id: int) -> None:
        self.L.refp_add_node(self.h, node_id)

    def add_primitive(self, type_name: str, pid: int) -> None:
        self.L.refp_add_primitive(self.h, type_name.encode(), pid)

    def _primitive(self, q, pid: int, object_id: int) -> str:
        """primitive_<type>_<pid>: the mbr_primitive's shape parameters (its
        transform goes to its node)."""
        name = PRIMITIVE_NAMES[q.type]
        self.add_primitive(name, pid)
        pre = f"primitive_{name}_{pid}_"
        self.set(pre + "enabled", 1, KIND_BOOL)
        self.set(pre + "object_id", object_id, KIND_INT)
        for key, kind, val in (("empty", KIND_BOOL, q.empty), ("limits_enable", KIND_BOOL, q.limits_enable),
                               ("caps", KIND_BOOL, q.caps), ("iterations", KIND_INT, q.iterations),
                               ("size", KIND_VEC3, list(q.size)), ("radius", KIND_DOUBLE, q.radius),
                               ("height", KIND_DOUBLE, q.height), ("width", KIND_DOUBLE, q.width),
                               ("tube_radius", KIND_DOUBLE, q.tube_radius),
                               ("radius_lpow", KIND_DOUBLE, q.radius_lpow),
                               ("tube_radius_lpow", KIND_DOUBLE, q.tube_radius_lpow),
                               ("rounding", KIND_DOUBLE, q.rounding), ("wall_thickness", KIND_DOUBLE, q.wall_thickness),
                               ("limits_min", KIND_VEC3, list(q.limits_min)),
                               ("limits_max", KIND_VEC3, list(q.limits_max)),
                               ("relative_amplitude", KIND_DOUBLE, q.relative_amplitude),
                               ("length", KIND_DOUBLE, q.length), ("anim_speed", KIND_DOUBLE, q.anim_speed),
                               ("anim_progression_speed", KIND_DOUBLE, q.anim_progression_speed),
                               ("prism_angle", KIND_DOUBLE, q.prism_angle),
                               ("trangle_height", KIND_DOUBLE, q.triangle_height)):
            try:
                self.set(pre + key, val, kind)
            except KeyError:  # not a parameter of this kind of primitive
                pass
        return name

    def _tree(self, s) -> None:
        """The scene's explicit objects tree as node_NNNN_* parameters: node i
        (0-based) gets id i + 1 and display order i; its parent is the nearest
        preceding node one level up."""
        parents = []
        for i in range(s.n_nodes):
            nd = s.node[i]
            nid = i + 1
            if nid > 1:
                self.add_node(nid)
            while len(parents) > nd.level:
                parents.pop()
            parent = parents[-1] if parents else 0
            pre = f"node_{nid:04d}_"
            if nd.type == NODE_FRACTAL_T:
                name, oid = "fractal", nd.index + 1
            elif nd.type == NODE_PRIMITIVE_T:
                q = s.primitive[nd.index]
                oid = 200 + i
                name = self._primitive(q, nd.index + 1, oid)
                self.set(pre + "position", list(q.position), KIND_VEC3)
                self.set(pre + "rotation", list(q.rotation), KIND_VEC3)
                self.set(pre + "scale", q.scale, KIND_DOUBLE)
                self.set(pre + "repeat", list(q.repeat), KIND_VEC3)
            else:
                name, oid = "group", 100 + i
            self.set_string(pre + "definition", f"{name} {nid},{nid},{nd.type},{parent},{oid},{i}")
            if nd.type != NODE_PRIMITIVE_T:
                self.set(pre + "position", list(nd.position), KIND_VEC3)
                self.set(pre + "rotation", list(nd.rotation), KIND_VEC3)
                self.set(pre + "scale", nd.scale, KIND_DOUBLE)
                self.set(pre + "repeat", list(nd.repeat), KIND_VEC3)
            self.set(pre + "enabled", nd.enabled, KIND_BOOL)
            self.set(pre + "detail_level_multiplier", nd.detail_level_multiplier, KIND_DOUBLE)
            self.set(pre + "smooth_de_combine_enable", nd.smooth_combine, KIND_BOOL)
            self.set(pre + "smooth_de_combine_distance", nd.smooth_combine_distance, KIND_DOUBLE)
            self.set(pre + "formula_maxiter", nd.formula_maxiter, KIND_INT)
            self.set(pre + "julia_mode", nd.julia_mode, KIND_BOOL)
            self.set(pre + "julia_c", list(nd.julia_c), KIND_VEC3)
            self.set(pre + "fractal_constant_factor", list(nd.fractal_constant_factor), KIND_VEC3)
            self.set(pre + "initial_waxis", nd.initial_waxis, KIND_DOUBLE)
            if nd.type in (11, 12, 13):
                parents.append(nid)

    def prepare(self) -> None:
        if self.L.refp_prepare(self.h):
            raise RuntimeError("refp_prepare")

    def distance(self, pts: np.ndarray, detail: float, normal_mode: bool = False):
        pts = np.ascontiguousarray(pts, dtype=np.float64)
        n = len(pts)
        d = np.zeros(n)
        it = np.zeros(n, np.int32)
        if self.L.refp_distance(self.h, pts.ctypes.data, n, detail, int(normal_mode), d.ctypes.data,
                                it.ctypes.data):
            raise RuntimeError("refp_distance")
        return d, it

    def compute(self, pts: np.ndarray, normal_mode: bool = False):
        pts = np.ascontiguousarray(pts, dtype=np.float64)
        n = len(pts)
        z = np.zeros((n, 3))
        d = np.zeros(n)
        it = np.zeros(n, np.int32)
        mx = np.zeros(n, np.int32)
        if self.L.refp_compute(self.h, pts.ctypes.data, n, int(normal_mode), z.ctypes.data, d.ctypes.data,
                               it.ctypes.data, mx.ctypes.data):
            raise RuntimeError("refp_compute")
        return z, d, it, mx

    def sequence(self):
        seq = np.zeros(1250, np.int32)
        length, fn, tp, an, ns = (C.c_int() for _ in range(5))
        bail = np.zeros(9)
        if self.L.refp_sequence(self.h, seq.ctypes.data, 1250, C.byref(length), C.byref(fn), C.byref(tp), C.byref(an),
                                bail.ctypes.data, C.byref(ns)):
            raise RuntimeError("refp_sequence")
        return {"seq": seq[: length.value].tolist(), "length": length.value, "de_function": fn.value,
                "de_type": tp.value, "analytic": an.value, "bailout": bail[: ns.value].tolist()}

    def light_direction(self, index: int = 0):
        d = (C.c_double * 3)()
        if self.L.refp_light_direction(self.h, index, d):
            raise RuntimeError("refp_light_direction")
        return list(d)

    def render(self, width: int, height: int, seed: int = 1):
        """(zbuffer float32 [H*W], world normal float32 [H*W,3], shadows float32 [H*W,3], rgb8 [H*W,3])."""
        self.set("image_width", width, KIND_INT)
        self.set("image_height", height, KIND_INT)
        n = width * height
        z = np.zeros(n, np.float32)
        nw = np.zeros((n, 3), np.float32)
        sh = np.zeros((n, 3), np.float32)
        r8 = np.zeros((n, 3), np.uint8)
        if self.L.refp_render(self.h, seed, z.ctypes.data, nw.ctypes.data, sh.ctypes.data, r8.ctypes.data):
            raise RuntimeError("refp_render")
        return z, nw, sh, r8

    # ---- the C-ABI structs in the reference's parameter names -------------------
    def configure(self, scene, camera=None, params=None) -> None:
        """Writes an mbr_scene (and optionally an mbr_camera and
        mbr_render_params) into the containers.  A single fractal keeps the
        default node 1; a hybrid becomes a hybrid node 1 with one fractal
        child per slot (the objects tree the reference builds for a legacy
        hybrid, settings.cpp:2700-2800)."""
        s = scene
        hybrid = bool(s.hybrid_fractal_enable)
        n = s.n_fractals if (hybrid or s.n_nodes > 0) else 1
        for i in range(n):
            f = s.fractal[i]
            self.set("formula", f.formula, KIND_INT, i)
            self.set("formula_iterations", f.formula_iterations, KIND_INT, i)
            self.set("formula_weight", f.formula_weight, KIND_DOUBLE, i)
            self.set("formula_start_iteration", f.formula_start_iteration, KIND_INT, i)
            self.set("formula_stop_iteration", f.formula_stop_iteration, KIND_INT, i)
            self.set("dont_add_c_constant", f.dont_add_c_constant, KIND_BOOL, i)
            self.set("check_for_bailout", f.check_for_bailout, KIND_BOOL, i)
            self.set("power", f.bulb_power, KIND_DOUBLE, i)
            self.set("alpha_angle_offset", f.bulb_alpha_angle_offset, KIND_DOUBLE, i)
            self.set("beta_angle_offset", f.bulb_beta_angle_offset, KIND_DOUBLE, i)
            self.set("mandelbox_scale", f.mandelbox_scale, KIND_DOUBLE, i)
            self.set("mandelbox_folding_limit", f.mandelbox_folding_limit, KIND_DOUBLE, i)
            self.set("mandelbox_folding_value", f.mandelbox_folding_value, KIND_DOUBLE, i)
            self.set("mandelbox_folding_min_radius", f.mandelbox_folding_min_radius, KIND_DOUBLE, i)
            self.set("mandelbox_folding_fixed_radius", f.mandelbox_folding_fixed_radius, KIND_DOUBLE, i)
            self.set("mandelbox_offset", list(f.mandelbox_offset), KIND_VEC3, i)
            self.set("transf_scale_3", f.transf_scale3, KIND_DOUBLE, i)
            self.set("cadd", f.aexion_cadd, KIND_DOUBLE, i)
            self.set("analyticDE_enabled", f.analytic_de_enabled, KIND_BOOL, i)
            self.set("analyticDE_scale_1", f.analytic_de_scale1, KIND_DOUBLE, i)
            self.set("analyticDE_offset_1", f.analytic_de_offset1, KIND_DOUBLE, i)
            self.set("mandelbox_rotations_enabled", f.mandelbox_rotations_enabled, KIND_BOOL, i)
            self.set("mandelbox_main_rotation_enabled", f.mandelbox_main_rotation_enabled, KIND_BOOL, i)
            self.set("mandelbox_rotation_main", list(f.mandelbox_rotation_main), KIND_VEC3, i)
            for k in range(3):
                self.set(f"mandelbox_rotation_neg_{k + 1}", list(f.mandelbox_rotation_neg[k]), KIND_VEC3, i)
                self.set(f"mandelbox_rotation_pos_{k + 1}", list(f.mandelbox_rotation_pos[k]), KIND_VEC3, i)
            if f.formula == 10:  # kaleidoscopic IFS (initparameters.cpp:724-743)
                for nm, v in (("abs_x", f.ifs_abs_x), ("abs_y", f.ifs_abs_y), ("abs_z", f.ifs_abs_z),
                              ("rotation_enabled", f.ifs_rotation_enabled), ("edge_enabled", f.ifs_edge_enabled),
                              ("menger_sponge_mode", f.ifs_menger_sponge_mode)):
                    self.set("IFS_" + nm, v, KIND_BOOL, i)
                self.set("IFS_scale", f.ifs_scale, KIND_DOUBLE, i)
                for nm, v in (("rotation", f.ifs_rotation), ("offset", f.ifs_offset), ("edge", f.ifs_edge)):
                    self.set("IFS_" + nm, list(v), KIND_VEC3, i)
                for k in range(9):
                    self.set(f"IFS_enabled_{k}", f.ifs_enabled[k], KIND_BOOL, i)
                    self.set(f"IFS_direction_{k}", list(f.ifs_direction[k]), KIND_VEC3, i)
                    self.set(f"IFS_rotations_{k}", list(f.ifs_rotations[k]), KIND_VEC3, i)
                    self.set(f"IFS_distance_{k}", f.ifs_distance[k], KIND_DOUBLE, i)
                    self.set(f"IFS_intensity_{k}", f.ifs_intensity[k], KIND_DOUBLE, i)
            # the keyed formula parameters: ints, bools and doubles as their
            # container holds them (a rotation is a vector of degrees)
            for j in range(f.n_params):
                key = f.param[j].key.decode()
                kind = self.L.refp_param_kind(self.h, i, key.encode())
                if kind < 0:
                    raise KeyError(f"fractal {i}: no parameter {key}")
                self.set(key, list(f.param[j].value) if kind == KIND_VEC3 else f.param[j].value[0], kind, i)
        self.set("use_default_bailout", s.use_default_bailout, KIND_BOOL)
        self.set("bailout", s.bailout, KIND_DOUBLE)
        self.set("minN", s.min_n, KIND_INT)
        self.set("iteration_threshold_mode", s.iteration_threshold_mode, KIND_BOOL)
        self.set("interior_mode", s.interior_mode, KIND_BOOL)
        self.set("linear_DE_offset", s.linear_de_offset, KIND_DOUBLE)
        self.set("delta_DE_function", s.delta_de_function, KIND_INT)
        self.set("delta_DE_method", s.delta_de_method, KIND_INT)
        self.set("deltade_relative_delta", s.deltade_relative_delta, KIND_DOUBLE)
        self.set("N", s.formula_maxiter, KIND_INT)
        self.set("repeat_from", s.repeat_from, KIND_INT)
        self.set("limits_enabled", s.limits_enabled, KIND_BOOL)
        self.set("limit_min", list(s.limit_min), KIND_VEC3)
        self.set("limit_max", list(s.limit_max), KIND_VEC3)
        self.set("box_folding", s.box_folding, KIND_BOOL)
        self.set("box_folding_limit", s.box_folding_limit, KIND_DOUBLE)
        self.set("box_folding_value", s.box_folding_value, KIND_DOUBLE)
        self.set("spherical_folding", s.spherical_folding, KIND_BOOL)
        self.set("spherical_folding_inner", s.spherical_folding_inner, KIND_DOUBLE)
        self.set("spherical_folding_outer", s.spherical_folding_outer, KIND_DOUBLE)
        if s.n_nodes > 0:
            self._tree(s)
        else:
            if hybrid:
                self.set_string("node_0001_definition", f"hybrid 1,1,{NODE_HYBRID},0,-1")
                for i in range(n):
                    nid = i + 2
                    self.add_node(nid)
                    self.set_string(f"node_{nid:04d}_definition", f"fractal {i + 1},{nid},{NODE_FRACTAL},1,{i + 1}")
            node = "node_0001_"
            self.set(node + "formula_maxiter", s.formula_maxiter, KIND_INT)
            self.set(node + "julia_mode", s.julia_mode, KIND_BOOL)
            self.set(node + "julia_c", list(s.julia_c), KIND_VEC3)
            self.set(node + "fractal_constant_factor", list(s.fractal_constant_factor), KIND_VEC3)
            self.set(node + "initial_waxis", s.initial_waxis, KIND_DOUBLE)
        if camera is not None:
            c = camera
            self.set("camera", list(c.camera), KIND_VEC3)
            self.set("target", list(c.target), KIND_VEC3)
            self.set("camera_top", list(c.top), KIND_VEC3)
            self.set("fov", c.fov_deg, KIND_DOUBLE)
            self.set("image_width", c.width, KIND_INT)
            self.set("image_height", c.height, KIND_INT)
            self.set("perspective_type", c.perspective_type, KIND_INT)
            self.set("legacy_coordinate_system", c.legacy_coordinate_system, KIND_BOOL)
        if params is not None:
            p = params
            self.set("detail_level", p.detail_level, KIND_DOUBLE)
            self.set("DE_factor", p.de_factor, KIND_DOUBLE)
            self.set("view_distance_max", p.view_distance_max, KIND_DOUBLE)
            self.set("smoothness", p.smoothness, KIND_DOUBLE)
            self.set("max_raymarching_steps", p.max_raymarching_steps, KIND_INT)
            self.set("constant_DE_threshold", p.constant_de_threshold, KIND_BOOL)
            self.set("DE_thresh", p.de_thresh, KIND_DOUBLE)
            self.set("advanced_quality", p.advanced_quality, KIND_BOOL)
            self.set("slow_shading", p.slow_shading, KIND_BOOL)
            self.set("detail_size_min", p.detail_size_min, KIND_DOUBLE)
            self.set("detail_size_max", p.detail_size_max, KIND_DOUBLE)
            self.set("abs_min_marching_step", p.abs_min_marching_step, KIND_DOUBLE)
            self.set("abs_max_marching_step", p.abs_max_marching_step, KIND_DOUBLE)
            self.set("rel_min_marching_step", p.rel_min_marching_step, KIND_DOUBLE)
            self.set("rel_max_marching_step", p.rel_max_marching_step, KIND_DOUBLE)
            self.set("ambient_occlusion_enabled", 0, KIND_BOOL)
            # the restated path shades without specular highlights; the
            # reference's default metallic highlight would also draw from the
            # global Random() stream (shader_specular_highlight.cpp:63-66)
            self.set("mat1_metallic", 0, KIND_BOOL)
            self.set("light1_cast_shadows", p.shadow_enable, KIND_BOOL)
            self.set("light1_penetrating", p.penetrating, KIND_BOOL)
            self.set("light1_soft_shadow_cone", p.soft_shadow_cone, KIND_DOUBLE)
