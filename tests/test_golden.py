"""The oracle pinned against the reference: golden vectors produced by the
reference's own sources (tests/golden/make_golden.py) must be reproduced
bit-for-bit by the oracle's restatement, and by the library's host code
where it restates the same function (camera set-up)."""
import ctypes as C
import json
import math
import os

import numpy as np
import pytest

from mandelbulber2_b200 import abi
from mandelbulber2_b200.render import camera_rotation

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def load(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


def fh(v):
    return [float.fromhex(x) for x in v] if isinstance(v, list) else float.fromhex(v)


def same(a, b):
    """Bit-level equality of double arrays (NaN equals NaN)."""
    return np.array_equal(np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64), equal_nan=True)


def scene_for(formula, fields):
    s = abi.scene_defaults(formula)
    f = s.fractal[0]
    for k, v in fields.items():
        if isinstance(v, list) and isinstance(v[0], list):
            for i, row in enumerate(v):
                getattr(f, k)[i][:] = row
        elif isinstance(v, list):
            getattr(f, k)[:] = v
        else:
            setattr(f, k, v)
    return s


@pytest.mark.parametrize("name", list(load("formula_kat.json").keys()))
def test_formula_kat_bit_exact(oracle, name):
    kat = load("formula_kat.json")[name]
    sc = scene_for(kat["formula"], kat["fields"])
    n = 0
    for case in kat["cases"]:
        for st in case:
            z, _, de = oracle.formula_step(sc, 0, fh(st["z_in"]), fh(st["r_in"]), fh(st["de_in"]))
            assert same(z, fh(st["z_out"])), (name, st)
            assert same([de], [fh(st["de_out"])]), (name, st)
            n += 1
    assert n >= 32


def _cam(c):
    cam = abi.camera_defaults()
    cam.camera[:] = c["camera"]
    cam.target[:] = c["target"]
    cam.top[:] = c["top"]
    cam.fov_deg = 53.0
    cam.width = cam.height = 64
    return cam


def test_camera_kat_oracle(oracle):
    for c in load("camera_kat.json"):
        cam = _cam(c)
        m, zero, ang = oracle.camera(cam)
        assert list(ang) == fh(c["angles"])
        ref_m = fh(c["mrot"])
        if zero:  # identity rotation: RotateVector returns the vector itself
            assert ref_m == [1.0, 0, 0, 0, 1.0, 0, 0, 0, 1.0]
        else:
            assert list(m) == ref_m
        for v in c["views"]:
            d = oracle.view_ip(cam, fh(v["ix"]), fh(v["iy"]))
            assert list(d) == fh(v["dir"])


def test_camera_kat_library_host():
    """The library's host-side camera set-up (mbr_camera_rotation) is bit-exact too."""
    for c in load("camera_kat.json"):
        cam = _cam(c)
        m, ang = camera_rotation(cam)
        assert ang == fh(c["angles"])
        assert m == fh(c["mrot"])


def test_projection_kat_oracle(oracle):
    """Fish-eye, equirectangular and fish-eye-cut view vectors of the oracle
    equal the reference's CalcFOV + CalculateViewVector bit for bit."""
    kats = load("projection_kat.json")
    assert {k["perspective_type"] for k in kats} == {1, 2, 3}
    for c in kats:
        cam = _cam(c)
        cam.fov_deg = c["fov_deg"]
        cam.perspective_type = c["perspective_type"]
        for v in c["views"]:
            d = oracle.view_ip(cam, fh(v["ix"]), fh(v["iy"]))
            assert list(d) == fh(v["dir"]), (c["perspective_type"], c["fov_deg"], v)


def test_fov_kat():
    for c in load("camera_kat.json"):
        assert 2.0 * math.tan(53.0 / 360.0 * math.pi) == fh(c["fov53"])


def test_park_miller_kat(oracle):
    for k in load("random_kat.json"):
        got = oracle.park_miller(k["seed"], len(k["values"]), k["max"])
        assert got.tolist() == k["values"]


# ---- live comparison against the compiled reference (only where it was built)
ref_available = pytest.mark.skipif(
    not __import__("oracle.oracle", fromlist=["Reference"]).Reference.available(),
    reason="oracle/_ref not built (needs the reference tree)")


@ref_available
@pytest.mark.parametrize("formula,params,fields", [
    (2, [8.0, 0.0, 0.0], {"bulb_power": 8.0}),
    (2, [11.3, 0.0, 0.0], {"bulb_power": 11.3}),
    (8, [-1.5, 1.0, 2.0, 0.5, 1.0, 0.0, 0.0, 0.0], {"mandelbox_scale": -1.5}),
    (8, [2.7, 1.0, 2.0, 0.6, 1.0, 0.0, 0.0, 0.0], {"mandelbox_scale": 2.7, "mandelbox_folding_min_radius": 0.6}),
    (7, [3.0], {"transf_scale3": 3.0}),
])
def test_formula_live_reference(oracle, formula, params, fields):
    from oracle.oracle import Reference

    ref = Reference()
    sc = scene_for(formula, fields)
    rng = np.random.default_rng(5)
    for _ in range(200):
        z = np.zeros(4)
        z[:3] = rng.uniform(-2, 2, 3)
        r = float(np.sqrt((z * z).sum()))
        a, _, da = ref.formula_step(formula, params, z, r, 1.7)
        b, _, db = oracle.formula_step(sc, 0, z, r, 1.7)
        assert same(a, b) and same([da], [db])
