"""ctypes wrapper of the CPU oracle (oracle/mbr_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() as
the checker, and by bench.py for the CPU-baseline leg.  The product never
imports this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
REF_LIB = os.path.join(HERE, "_ref", "libref.so")

_P = C.c_void_p


class OracleOutputs(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in ("depth", "iters", "hit", "normal", "shade", "ao", "rgb", "rgb8",
                                          "shadow")]


def build() -> None:
    """make -C oracle (both builds); cheap when up to date."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def _lib_path(kind: str) -> str:
    return os.path.join(BUILD, f"liboracle_{kind}.so")


class Oracle:
    """kind: 'strict' (IEEE, the parity oracle) or 'fast' (-O3 -ffast-math, the timed baseline)."""

    def __init__(self, kind: str = "strict"):
        path = _lib_path(kind)
        if not os.path.exists(path):
            build()
        self.lib = C.CDLL(path)
        from mandelbulber2_b200 import abi  # struct layouts shared with the C-ABI

        self.abi = abi
        L = self.lib
        L.oracle_render.argtypes = [C.POINTER(abi.Scene), C.POINTER(abi.Camera), C.POINTER(abi.RenderParams),
                                    C.POINTER(OracleOutputs), C.c_int, C.c_int, C.c_int, C.POINTER(abi.Stats)]
        L.oracle_distance.argtypes = [C.POINTER(abi.Scene), _P, C.c_int64, C.c_double, C.c_int, _P, _P]
        L.oracle_sequence.argtypes = [C.POINTER(abi.Scene), _P, _P, _P, _P]
        L.oracle_formula_step.argtypes = [C.POINTER(abi.Scene), C.c_int, _P, _P, _P]
        L.oracle_camera.argtypes = [C.POINTER(abi.Camera), _P, _P]
        L.oracle_view.argtypes = [C.POINTER(abi.Camera), C.c_int, C.c_int, _P]
        L.oracle_view_ip.argtypes = [C.POINTER(abi.Camera), C.c_double, C.c_double, _P]
        L.oracle_park_miller.argtypes = [C.c_uint32, C.c_uint64, C.c_uint32, C.c_int, C.c_int, _P]
        L.oracle_pcg32.argtypes = [C.c_uint64, C.c_uint64, C.c_int, _P]
        L.oracle_opcount.argtypes = [C.POINTER(abi.Scene), C.c_int, _P, _P]
        L.oracle_opcount_de.argtypes = [C.POINTER(abi.Scene), _P, C.c_int64, C.c_double, _P]
        L.oracle_de_tangents.argtypes = [C.POINTER(abi.Scene), _P, C.c_int64, C.c_double, C.c_int, _P]
        L.oracle_pixel_gradients.argtypes = [C.POINTER(abi.Scene), C.POINTER(abi.Camera),
                                             C.POINTER(abi.RenderParams), _P, _P, _P, _P, _P]
        L.oracle_threads.restype = C.c_int
        L.oracle_scene_defaults.argtypes = [C.POINTER(abi.Scene)]
        L.oracle_fractal_defaults.argtypes = [C.POINTER(abi.Fractal), C.c_int]
        L.oracle_camera_defaults.argtypes = [C.POINTER(abi.Camera)]
        L.oracle_render_params_defaults.argtypes = [C.POINTER(abi.RenderParams)]
        for f in ("oracle_scene_defaults", "oracle_fractal_defaults", "oracle_camera_defaults",
                  "oracle_render_params_defaults"):
            getattr(L, f).restype = None

    def threads(self) -> int:
        return self.lib.oracle_threads()

    def camera_rotation(self, cam):
        """(mRot row-major as a list of 9, [yaw, pitch, roll]) of PrepareMainVectors."""
        m = (C.c_double * 10)()
        ang = (C.c_double * 3)()
        self.lib.oracle_camera(C.byref(cam), m, ang)
        return list(m)[:9], list(ang)

    def render(self, scene, cam, params, rows=None, threads: int = 0,
               outputs=("depth", "iters", "hit", "normal", "shade", "ao", "rgb", "rgb8")):
        r0, r1 = rows if rows is not None else (0, cam.height)
        n = (r1 - r0) * cam.width
        spec = {"depth": (np.float64, 1), "iters": (np.int32, 1), "hit": (np.uint8, 1), "normal": (np.float32, 3),
                "shade": (np.float32, 1), "ao": (np.float32, 1), "rgb": (np.float32, 3), "rgb8": (np.uint8, 3),
                "shadow": (np.float32, 1)}
        bufs = {}
        o = OracleOutputs()
        for k in outputs:
            dt, ch = spec[k]
            bufs[k] = np.zeros((n,) if ch == 1 else (n, ch), dtype=dt)
            setattr(o, k, bufs[k].ctypes.data)
        st = self.abi.Stats()
        rc = self.lib.oracle_render(C.byref(scene), C.byref(cam), C.byref(params), C.byref(o), r0, r1, threads,
                                    C.byref(st))
        if rc != 0:
            raise RuntimeError(f"oracle_render failed ({rc})")
        stats = {f: int(getattr(st, f)) for f, _ in self.abi.Stats._fields_}
        return bufs, stats

    def distance(self, scene, pts: np.ndarray, detail: float, normal_mode: bool = False):
        pts = np.ascontiguousarray(pts, dtype=np.float64)
        n = pts.shape[0]
        d = np.zeros(n, dtype=np.float64)
        it = np.zeros(n, dtype=np.int32)
        rc = self.lib.oracle_distance(C.byref(scene), pts.ctypes.data, n, detail, int(normal_mode), d.ctypes.data,
                                      it.ctypes.data)
        if rc != 0:
            raise RuntimeError("oracle_distance failed")
        return d, it

    def sequence(self, scene):
        seq = np.zeros(1250, dtype=np.int32)
        length, fn = C.c_int32(), C.c_int32()
        bail = np.zeros(9, dtype=np.float64)
        rc = self.lib.oracle_sequence(C.byref(scene), seq.ctypes.data, C.addressof(length), C.addressof(fn),
                                      bail.ctypes.data)
        if rc != 0:
            raise RuntimeError("oracle_sequence failed")
        return seq[: length.value].tolist(), length.value, fn.value, bail.tolist()

    def formula_step(self, scene, slot: int, z, r: float, de: float):
        zz = np.array(z, dtype=np.float64)
        rr = C.c_double(r)
        dd = C.c_double(de)
        rc = self.lib.oracle_formula_step(C.byref(scene), slot, zz.ctypes.data, C.addressof(rr), C.addressof(dd))
        if rc != 0:
            raise RuntimeError("oracle_formula_step failed")
        return zz, rr.value, dd.value

    def camera(self, cam):
        m = np.zeros(10, dtype=np.float64)
        a = np.zeros(3, dtype=np.float64)
        self.lib.oracle_camera(C.byref(cam), m.ctypes.data, a.ctypes.data)
        return m[:9], bool(m[9]), a

    def view(self, cam, x: int, y: int):
        d = np.zeros(3, dtype=np.float64)
        self.lib.oracle_view(C.byref(cam), x, y, d.ctypes.data)
        return d

    def view_ip(self, cam, ix: float, iy: float):
        d = np.zeros(3, dtype=np.float64)
        self.lib.oracle_view_ip(C.byref(cam), ix, iy, d.ctypes.data)
        return d

    def park_miller(self, seed: int, n: int, max_: int = -1, ray: int = 0, ray_seed: int = 0):
        out = np.zeros(n, dtype=np.int32)
        self.lib.oracle_park_miller(seed, ray, ray_seed, max_, n, out.ctypes.data)
        return out

    def pcg32(self, initstate: int, initseq: int, n: int):
        out = np.zeros(n, dtype=np.uint32)
        self.lib.oracle_pcg32(initstate, initseq, n, out.ctypes.data)
        return out

    def opcount(self, scene, slot: int, z):
        zz = np.array(z, dtype=np.float64)
        out = np.zeros(6, dtype=np.uint64)
        self.lib.oracle_opcount(C.byref(scene), slot, zz.ctypes.data, out.ctypes.data)
        return dict(zip(("add", "mul", "div", "sqrt", "transc", "cmp"), out.tolist()))

    def opcount_de(self, scene, pts: np.ndarray, detail: float):
        pts = np.ascontiguousarray(pts, dtype=np.float64)
        out = np.zeros(10, dtype=np.uint64)
        rc = self.lib.oracle_opcount_de(C.byref(scene), pts.ctypes.data, pts.shape[0], detail, out.ctypes.data)
        if rc != 0:
            raise RuntimeError("oracle_opcount_de failed")
        return dict(zip(("add", "mul", "div", "sqrt", "transc", "cmp", "iters", "evals", "e_add", "e_mul"),
                        out.tolist()))

    def de_tangents(self, scene, pts: np.ndarray, detail: float, normal_mode: bool = False):
        """Distance and its tangents (power, scale, mR2, x, y, z) at points: (n, 7)."""
        pts = np.ascontiguousarray(pts, dtype=np.float64)
        out = np.zeros((pts.shape[0], 7), dtype=np.float64)
        rc = self.lib.oracle_de_tangents(C.byref(scene), pts.ctypes.data, pts.shape[0], detail, int(normal_mode),
                                         out.ctypes.data)
        if rc != 0:
            raise RuntimeError("oracle_de_tangents failed")
        return out

    def pixel_gradients(self, scene, cam, params, depth: np.ndarray, hit: np.ndarray):
        n = cam.width * cam.height
        depth = np.ascontiguousarray(depth, dtype=np.float64)
        hit = np.ascontiguousarray(hit, dtype=np.uint8)
        dt = np.zeros((n, 8), dtype=np.float64)
        ds = np.zeros((n, 8), dtype=np.float64)
        shade = np.zeros(n, dtype=np.float64)
        rc = self.lib.oracle_pixel_gradients(C.byref(scene), C.byref(cam), C.byref(params), depth.ctypes.data,
                                             hit.ctypes.data, dt.ctypes.data, ds.ctypes.data, shade.ctypes.data)
        if rc != 0:
            raise RuntimeError(f"oracle_pixel_gradients failed ({rc})")
        return dt, ds, shade


class Reference:
    """The reference's own formula, camera and RNG sources compiled into
    oracle/_ref/libref.so (oracle/build_ref.sh).  Needs the reference tree at
    build time; absent on machines without it."""

    def __init__(self):
        if not os.path.exists(REF_LIB):
            raise FileNotFoundError(REF_LIB)
        L = self.lib = C.CDLL(REF_LIB)
        L.ref_formula_step.argtypes = [C.c_int, _P, _P, _P, _P, C.c_int]
        L.ref_camera.argtypes = [_P, _P, _P, _P]
        L.ref_view_vector.argtypes = [_P, _P, _P, C.c_double, C.c_double, C.c_double, _P]
        L.ref_calc_fov.restype = C.c_double
        L.ref_calc_fov.argtypes = [C.c_double]
        L.ref_mandelbox_rot_step.argtypes = [_P, _P, _P, _P, C.c_int]
        L.ref_ifs_step.argtypes = [_P, _P, _P, _P, C.c_int]
        L.ref_view_vector_p.argtypes = [_P, _P, _P, C.c_double, C.c_int, C.c_double, C.c_double, _P]
        L.ref_calc_fov_p.restype = C.c_double
        L.ref_calc_fov_p.argtypes = [C.c_double, C.c_int]
        L.ref_random.argtypes = [C.c_uint, C.c_int, C.c_int, _P]

    @staticmethod
    def available() -> bool:
        return os.path.exists(REF_LIB)

    def formula_step(self, formula: int, params, z, r: float, de: float, i: int = 0):
        p = np.array(params, dtype=np.float64)
        zz = np.array(z, dtype=np.float64)
        rr, dd = C.c_double(r), C.c_double(de)
        rc = self.lib.ref_formula_step(formula, p.ctypes.data, zz.ctypes.data, C.addressof(rr), C.addressof(dd), i)
        if rc != 0:
            raise RuntimeError("ref_formula_step failed")
        return zz, rr.value, dd.value

    def mandelbox_rot_step(self, params, z, r: float, de: float, i: int = 0):
        p = np.array(params, dtype=np.float64)
        assert p.size == 31
        zz = np.array(z, dtype=np.float64)
        rr, dd = C.c_double(r), C.c_double(de)
        if self.lib.ref_mandelbox_rot_step(p.ctypes.data, zz.ctypes.data, C.addressof(rr), C.addressof(dd), i) != 0:
            raise RuntimeError("ref_mandelbox_rot_step failed")
        return zz, rr.value, dd.value

    def ifs_step(self, params, z, r: float, de: float, i: int = 0):
        p = np.array(params, dtype=np.float64)
        assert p.size == 97
        zz = np.array(z, dtype=np.float64)
        rr, dd = C.c_double(r), C.c_double(de)
        if self.lib.ref_ifs_step(p.ctypes.data, zz.ctypes.data, C.addressof(rr), C.addressof(dd), i) != 0:
            raise RuntimeError("ref_ifs_step failed")
        return zz, rr.value, dd.value

    def camera(self, cam, target, top):
        out = np.zeros(12, dtype=np.float64)
        a = [np.array(v, dtype=np.float64) for v in (cam, target, top)]
        self.lib.ref_camera(a[0].ctypes.data, a[1].ctypes.data, a[2].ctypes.data, out.ctypes.data)
        return out

    def view_vector(self, cam, target, top, fov_deg, ix, iy):
        out = np.zeros(3, dtype=np.float64)
        a = [np.array(v, dtype=np.float64) for v in (cam, target, top)]
        self.lib.ref_view_vector(a[0].ctypes.data, a[1].ctypes.data, a[2].ctypes.data, fov_deg, ix, iy,
                                 out.ctypes.data)
        return out

    def view_vector_p(self, cam, target, top, fov_deg, persp, ix, iy):
        out = np.zeros(3, dtype=np.float64)
        a = [np.array(v, dtype=np.float64) for v in (cam, target, top)]
        self.lib.ref_view_vector_p(a[0].ctypes.data, a[1].ctypes.data, a[2].ctypes.data, fov_deg, persp, ix, iy,
                                   out.ctypes.data)
        return out

    def random(self, seed: int, n: int, max_: int = -1):
        out = np.zeros(n, dtype=np.int32)
        self.lib.ref_random(seed, max_, n, out.ctypes.data)
        return out
