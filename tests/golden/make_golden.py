"""Generates the golden vectors of tests/golden/ from the REFERENCE's own
sources, compiled unchanged into oracle/_ref/libref.so by oracle/build_ref.sh:

  formula_kat.json  chains of cFractal*::FormulaCode calls (Mandelbulb,
                    Mandelbox with and without rotations, Menger sponge,
                    Mandelbulb power 2, hypercomplex, kaleidoscopic IFS,
                    xenodreambuie)
                    on seeded random points
  projection_kat.json  CalcFOV + CalculateViewVector of the fish-eye,
                    equirectangular and fish-eye-cut projections
  camera_kat.json   cCameraTarget + PrepareMainVectors rotations and
                    CalculateViewVector directions
  random_kat.json   Park-Miller Random()/RandomInt() sequences

and, from the reference's sources for the whole path compiled into
oracle/_ref/librefpipe.so (parameter containers with the reference's
defaults, objects tree, sequences, Compute, CalculateDistance, the render
worker with its shaders, cImage):

  pipeline_kat.json CalculateDistance and the hybrid sequence of the scene
                    variants of pipeline_cases.cases() at seeded points
  render_kat.json   small frames of pipeline_cases.render_cases() rendered by
                    cRenderWorker::doWork: z-buffer, world normals, shadows

Doubles are stored with float.hex() so the comparison is bit-exact.
Run: python tests/golden/make_golden.py  (needs the reference tree to build libref.so)
"""
from __future__ import annotations

import json
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.oracle import Reference  # noqa: E402
from tests.golden.pipeline_cases import cases, render_cases  # noqa: E402

FORMULAS = [
    # (name, formula id, params for ref_formula_step, scene fields)
    ("mandelbulb_p8", 2, [8.0, 0.0, 0.0], {"bulb_power": 8.0}),
    ("mandelbulb_p3_5", 2, [3.5, 0.0, 0.0], {"bulb_power": 3.5}),
    ("mandelbulb_p8_angles", 2, [8.0, 10.0 * math.pi / 180.0, -20.0 * math.pi / 180.0],
     {"bulb_power": 8.0, "bulb_alpha_angle_offset": 10.0, "bulb_beta_angle_offset": -20.0}),
    ("mandelbox_m1_5", 8, [-1.5, 1.0, 2.0, 0.5, 1.0, 0.0, 0.0, 0.0],
     {"mandelbox_scale": -1.5, "mandelbox_folding_min_radius": 0.5}),
    ("mandelbox_2_offset", 8, [2.0, 1.0, 2.0, 0.5, 1.0, 0.1, -0.2, 0.05],
     {"mandelbox_scale": 2.0, "mandelbox_offset": [0.1, -0.2, 0.05]}),
    ("mandelbox_m2_2_minr", 8, [-2.2, 0.9, 1.8, 0.35, 1.1, 0.0, 0.0, 0.0],
     {"mandelbox_scale": -2.2, "mandelbox_folding_limit": 0.9, "mandelbox_folding_value": 1.8,
      "mandelbox_folding_min_radius": 0.35, "mandelbox_folding_fixed_radius": 1.1}),
    ("menger_3", 7, [3.0], {"transf_scale3": 3.0}),
    ("mandelbulb_power2", 3, [], {}),
    ("hypercomplex", 4, [], {}),
    ("xenodreambuie_p5", 11, [5.0, 0.0, 0.0], {"bulb_power": 5.0}),
    ("xenodreambuie_p3_angles", 11, [3.0, 15.0 * math.pi / 180.0, -30.0 * math.pi / 180.0],
     {"bulb_power": 3.0, "bulb_alpha_angle_offset": 15.0, "bulb_beta_angle_offset": -30.0}),
]
# Mandelbox with rotations (fractal_mandelbox.cpp:33-63, 103): the eight
# parameters above, rotationsEnabled, mainRotationEnabled, the neg and pos
# rotation vectors of the three axes and the main rotation, in degrees.
_NEG = [[10.0, 0.0, -5.0], [0.0, 25.0, 0.0], [-15.0, 5.0, 30.0]]
_POS = [[0.0, -20.0, 0.0], [12.0, 0.0, 7.0], [0.0, 0.0, 0.0]]
_MAIN = [3.0, -17.0, 41.0]
ROT_FORMULAS = [
    ("mandelbox_m1_5_rotations", [-1.5, 1.0, 2.0, 0.5, 1.0, 0.0, 0.0, 0.0, 1.0, 0.0] + sum(_NEG, []) + sum(_POS, [])
     + [0.0, 0.0, 0.0],
     {"mandelbox_scale": -1.5, "mandelbox_rotations_enabled": 1, "mandelbox_rotation_neg": _NEG,
      "mandelbox_rotation_pos": _POS}),
    ("mandelbox_2_main_rotation", [2.0, 1.0, 2.0, 0.5, 1.0, 0.1, -0.2, 0.05, 0.0, 1.0] + [0.0] * 18 + _MAIN,
     {"mandelbox_scale": 2.0, "mandelbox_offset": [0.1, -0.2, 0.05], "mandelbox_main_rotation_enabled": 1,
      "mandelbox_rotation_main": _MAIN}),
    ("mandelbox_m2_both_rotations", [-2.0, 1.0, 2.0, 0.4, 1.0, 0.0, 0.0, 0.0, 1.0, 1.0] + sum(_NEG, [])
     + sum(_POS, []) + _MAIN,
     {"mandelbox_scale": -2.0, "mandelbox_folding_min_radius": 0.4, "mandelbox_rotations_enabled": 1,
      "mandelbox_main_rotation_enabled": 1, "mandelbox_rotation_neg": _NEG, "mandelbox_rotation_pos": _POS,
      "mandelbox_rotation_main": _MAIN}),
]
N_POINTS = 32
N_STEPS = 6


# Kaleidoscopic IFS: (name, ref_ifs_step parameters, scene fields)
def _ifs(scale, rot_on, rotation, offset, edge_on, edge, absxyz, menger, vectors):
    p = [scale, rot_on] + rotation + offset + [edge_on] + edge + absxyz + [menger]
    fields = {"ifs_scale": scale, "ifs_rotation_enabled": rot_on, "ifs_rotation": rotation, "ifs_offset": offset,
              "ifs_edge_enabled": edge_on, "ifs_edge": edge, "ifs_abs_x": absxyz[0], "ifs_abs_y": absxyz[1],
              "ifs_abs_z": absxyz[2], "ifs_menger_sponge_mode": menger, "ifs_enabled": [0] * 9,
              "ifs_direction": [[1.0, 0.0, 0.0] for _ in range(9)], "ifs_rotations": [[0.0] * 3 for _ in range(9)],
              "ifs_distance": [0.0] * 9, "ifs_intensity": [1.0] * 9}
    for i in range(9):
        en, d, r, dist, inten = vectors.get(i, (0, [1.0, 0.0, 0.0], [0.0, 0.0, 0.0], 0.0, 1.0))
        p += [en] + d + r + [dist, inten]
        fields["ifs_enabled"][i] = en
        fields["ifs_direction"][i] = d
        fields["ifs_rotations"][i] = r
        fields["ifs_distance"][i] = dist
        fields["ifs_intensity"][i] = inten
    return p, fields


IFS_FORMULAS = [
    ("ifs_menger_mode", *_ifs(3.0, 0, [0.0, 0.0, 0.0], [1.0, 1.0, 1.0], 0, [0.0] * 3, [1, 1, 1], 1,
                              {0: (1, [1.0, -1.0, 0.0], [0.0, 0.0, 0.0], 0.0, 1.0),
                               1: (1, [0.0, 1.0, -1.0], [0.0, 0.0, 0.0], 0.0, 1.0),
                               2: (1, [1.0, 0.0, -1.0], [0.0, 0.0, 0.0], 0.0, 1.0)})),
    ("ifs_rotated_edges", *_ifs(2.2, 1, [45.0, 0.0, 12.0], [1.0, 0.5, 0.3], 1, [0.8, 0.0, 0.6], [1, 0, 1], 0,
                                {3: (1, [0.0, 0.71, -0.71], [10.0, -5.0, 20.0], 0.1, 0.9),
                                 7: (1, [1.0, 1.0, 1.0], [0.0, 30.0, 0.0], -0.2, 1.0)})),
]


def hexs(a):
    return [float(x).hex() for x in np.asarray(a, dtype=np.float64).ravel()]


def formula_kats(ref: Reference) -> dict:
    rng = np.random.default_rng(20241203)
    out = {}
    entries = ([(n, f, p, fl, False) for n, f, p, fl in FORMULAS] + [(n, 8, p, fl, True) for n, p, fl in ROT_FORMULAS]
               + [(n, 10, p, fl, "ifs") for n, p, fl in IFS_FORMULAS])
    for name, fid, params, fields, rot in entries:
        cases = []
        for _ in range(N_POINTS):
            z = np.zeros(4)
            z[:3] = rng.uniform(-1.5, 1.5, size=3)
            r = math.sqrt(z[0] * z[0] + z[1] * z[1] + z[2] * z[2] + z[3] * z[3])
            de = 1.0
            steps = []
            for i in range(N_STEPS):
                zin, rin, dein = z.copy(), r, de
                if rot == "ifs":
                    z, _, de = ref.ifs_step(params, z, r, de, i)
                elif rot:
                    z, _, de = ref.mandelbox_rot_step(params, z, r, de, i)
                else:
                    z, _, de = ref.formula_step(fid, params, z, r, de, i)
                steps.append({"z_in": hexs(zin), "r_in": float(rin).hex(), "de_in": float(dein).hex(),
                              "z_out": hexs(z), "de_out": float(de).hex()})
                r = math.sqrt(z[0] * z[0] + z[1] * z[1] + z[2] * z[2] + z[3] * z[3])
                if not math.isfinite(r) or r > 1e6:
                    break
            cases.append(steps)
        out[name] = {"formula": fid, "fields": fields, "cases": cases}
    return out


CAMERAS = [
    ((0.0, -3.0, 0.0), (0.0, 0.0, 0.0), (0.0, 0.0, 1.0)),
    ((0.0, -6.0, 0.0), (0.0, 0.0, 0.0), (0.0, 0.0, 1.0)),
    ((3.0, -6.0, 2.0), (0.0, 0.0, 0.0), (0.0, 0.0, 1.0)),
    ((-2.1, 1.7, 0.9), (0.3, -0.2, 0.1), (0.0, 0.0, 1.0)),
    ((1.0, 2.0, 3.0), (0.0, 0.0, 0.0), (0.2, 0.1, 1.0)),
    ((0.5, -0.5, -3.5), (0.0, 0.0, 0.0), (0.0, 1.0, 0.0)),
]
VIEW_POINTS = [(0.0, 0.0), (0.25, -0.1), (-0.4, 0.3), (0.7, 0.45), (-0.888, -0.5)]


def camera_kats(ref: Reference) -> list:
    out = []
    for cam, tgt, top in CAMERAS:
        r = ref.camera(cam, tgt, top)
        views = []
        for ix, iy in VIEW_POINTS:
            views.append({"ix": float(ix).hex(), "iy": float(iy).hex(),
                          "dir": hexs(ref.view_vector(cam, tgt, top, 53.0, ix, iy))})
        out.append({"camera": cam, "target": tgt, "top": top, "angles": hexs(r[:3]), "mrot": hexs(r[3:]),
                    "fov53": float(ref.lib.ref_calc_fov(53.0)).hex(), "views": views})
    return out


# (projection, FOV degrees): fish eye below and beyond a hemisphere,
# equirectangular over the full sphere, fish-eye cut
PROJECTIONS = [(1, 120.0), (1, 200.0), (2, 360.0), (2, 90.0), (3, 180.0)]


def projection_kats(ref: Reference) -> list:
    out = []
    for cam, tgt, top in CAMERAS[:4]:
        for persp, fov in PROJECTIONS:
            views = []
            for ix, iy in VIEW_POINTS:
                views.append({"ix": float(ix).hex(), "iy": float(iy).hex(),
                              "dir": hexs(ref.view_vector_p(cam, tgt, top, fov, persp, ix, iy))})
            out.append({"camera": cam, "target": tgt, "top": top, "perspective_type": persp, "fov_deg": fov,
                        "fov": float(ref.lib.ref_calc_fov_p(fov, persp)).hex(), "views": views})
    return out


def random_kats(ref: Reference) -> list:
    out = []
    for seed in (1, 12345, 2147483646, 987654321):
        out.append({"seed": seed, "max": -1, "values": ref.random(seed, 64, -1).tolist()})
        out.append({"seed": seed, "max": 1000, "values": ref.random(seed, 64, 1000).tolist()})
    return out


def pipeline_kats() -> dict:
    """CalculateDistance (both normal modes, two detail sizes) at 48 seeded
    points per scene, and the scene's sequence."""
    from oracle.refpipe import RefPipeline

    rng = np.random.default_rng(20241)
    out = {}
    for name, sc in cases().items():
        r = RefPipeline()
        r.configure(sc)
        pts = rng.uniform(-2.0, 2.0, size=(48, 3))
        entry = {"points": [hexs(p) for p in pts], "runs": []}
        for nm in (0, 1):
            for det in (1e-3, 0.05):
                d, it = r.distance(pts, det, bool(nm))
                entry["runs"].append({"normal_mode": nm, "detail": det.hex(), "dist": hexs(d),
                                      "iters": [int(x) for x in it]})
        entry["sequence"] = r.sequence()
        out[name] = entry
        r.close()
    return out


def _pack(a: np.ndarray) -> str:
    import base64
    import zlib

    return base64.b64encode(zlib.compress(np.ascontiguousarray(a).astype("<f4").tobytes(), 9)).decode()


def render_kats() -> dict:
    from oracle.refpipe import RefPipeline

    out = {}
    for name, sc, cam, p in render_cases():
        r = RefPipeline()
        r.configure(sc, cam, p)
        r.prepare()
        light = r.light_direction(0)
        z, nw, sh, _ = r.render(cam.width, cam.height, seed=1)
        out[name] = {"width": cam.width, "height": cam.height, "seed": 1, "light": [float(v).hex() for v in light],
                     "zbuffer": _pack(z), "normal_world": _pack(nw), "shadow": _pack(sh[:, 0])}
        r.close()
    return out


def main() -> None:
    ref = Reference()
    with open(os.path.join(HERE, "formula_kat.json"), "w") as f:
        json.dump(formula_kats(ref), f, separators=(",", ":"))
    with open(os.path.join(HERE, "camera_kat.json"), "w") as f:
        json.dump(camera_kats(ref), f, indent=1)
    with open(os.path.join(HERE, "projection_kat.json"), "w") as f:
        json.dump(projection_kats(ref), f, indent=1)
    with open(os.path.join(HERE, "random_kat.json"), "w") as f:
        json.dump(random_kats(ref), f)
    from oracle.refpipe import available

    if available():
        with open(os.path.join(HERE, "pipeline_kat.json"), "w") as f:
            json.dump(pipeline_kats(), f, separators=(",", ":"))
        with open(os.path.join(HERE, "render_kat.json"), "w") as f:
            json.dump(render_kats(), f, indent=1)
    print("golden vectors written to", HERE)


if __name__ == "__main__":
    main()
