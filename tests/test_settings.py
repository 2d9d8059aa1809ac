"""Settings files (.fract) read by mbr_fract_parse, on the CPU.

The fixtures under tests/golden/settings/ are scenes written for these tests
in the reference's flat settings format (header, [main_parameters],
[fractal_N], comma decimals).  The expected values restate the reference's
rules: defaults from initparameters.cpp, the renames of Compatibility for old
versions (settings.cpp:1283-1466), N as the iteration limit of the fractal
node (settings.cpp:2494-2501, 2775-2778), and the main light's direction from
cLight (light.cpp:90-190, rotation scaled by pi/180.8).  When the reference
tree is present, every example scene it ships is read as well.
"""
import glob
import math
import os

import numpy as np
import pytest

from mandelbulber2_b200 import abi, settings

HERE = os.path.dirname(os.path.abspath(__file__))
FIX = os.path.join(HERE, "golden", "settings")
# the reference's example scenes: read when MANDELBULBER2_SOURCE names the
# reference's mandelbulber2 directory (the tests are skipped otherwise)
_SRC = os.environ.get("MANDELBULBER2_SOURCE", "")
EXAMPLES = os.path.join(_SRC, "deploy", "share", "mandelbulber2", "examples") if _SRC else ""

HEADER = "# Mandelbulber settings file\n# version 2.33\n# only modified parameters\n"


def rot_about(v, a, ang):
    v, a = np.asarray(v, float), np.asarray(a, float)
    return v * math.cos(ang) + np.cross(a, v) * math.sin(ang) + a * np.dot(a, v) * (1 - math.cos(ang))


def camera_frame(cam, tgt, top):
    """cCameraTarget::SetCameraTargetTop (camera_target.cpp:88-126)."""
    f = np.asarray(tgt, float) - np.asarray(cam, float)
    f = f / np.linalg.norm(f)
    yaw = math.atan2(f[1], f[0]) - 0.5 * math.pi
    pitch = math.atan2(f[2], math.sqrt(f[0] ** 2 + f[1] ** 2))
    t = np.asarray(top, float) / np.linalg.norm(top)
    t = rot_about(t, [0, 0, 1], -yaw)
    t = rot_about(t, [1, 0, 0], -pitch)
    roll = -math.atan2(t[2], t[0]) + 0.5 * math.pi
    up = rot_about([0, 0, 1], [0, 1, 0], roll)
    up = rot_about(up, [1, 0, 0], pitch)
    up = rot_about(up, [0, 0, 1], yaw)
    return f, up, np.cross(f, up)


def relative_light(cam, tgt, top, rotation_deg):
    """Directional light 1 relative to the camera (light.cpp:90-160)."""
    r = np.asarray(rotation_deg, float) / 180.8 * math.pi * np.array([1.0, -1.0, 1.0])
    f, up, right = camera_frame(cam, tgt, top)
    d = -f
    d = rot_about(d, f, r[2])
    d = rot_about(d, right, r[1])
    d = rot_about(d, up, r[0])
    return d


def test_mandelbox_with_ao():
    s = settings.load_from_file(os.path.join(FIX, "box_ao.fract"))
    assert s.status == abi.MBR_OK, s.report
    sc, cam, p = s.scene, s.camera, s.params
    assert sc.n_fractals == 1 and not sc.hybrid_fractal_enable
    f = sc.fractal[0]
    assert f.formula == abi.FORMULA_MANDELBOX
    assert f.mandelbox_scale == -1.73 and f.mandelbox_folding_min_radius == 0.4
    assert f.mandelbox_folding_limit == 1.0 and f.mandelbox_folding_value == 2.0  # defaults
    assert sc.formula_maxiter == 40
    assert list(cam.camera) == [0.5, -5.5, 1.4] and list(cam.target) == [0.0, 0.0, 0.1]
    assert list(cam.top) == [0.05, 0.2, 0.97]
    assert (cam.width, cam.height) == (96, 54) and cam.fov_deg == 53.13
    assert p.detail_level == 1.5 and p.de_factor == 0.9 and p.view_distance_max == 25.0
    assert p.ao_rays == 16 and p.ambient_intensity == 0.8
    assert p.shading_enable == 1 and p.shadow_enable == 1
    want = relative_light(cam.camera, cam.target, cam.top, [30, -20, 0])
    np.testing.assert_allclose(list(p.light_direction), want, rtol=0, atol=1e-12)
    assert "volumetric_fog_enabled" in s.report and "mat1_specular" in s.report
    assert p.penetrating == 0 and p.soft_shadow_cone == 0.0  # light1_penetrating false, cone 0


def test_primitives():
    """Enabled primitives join the fractal by union; a water of a file before
    2.13 reads its amplitude as the relative amplitude (settings.cpp:1365-1372);
    a disabled primitive is skipped."""
    s = settings.load_from_file(os.path.join(FIX, "box_primitives.fract"))
    assert s.ok, s.report
    sc = s.scene
    assert sc.n_primitives == 3
    w, sp, bx = sc.primitive[0], sc.primitive[1], sc.primitive[2]
    assert w.type == abi.PRIMITIVE_WATER and list(w.position) == [0.0, 0.0, -2.2] and list(w.rotation) == [0, 0, 15]
    assert w.relative_amplitude == 0.25 and w.length == 0.4 and w.iterations == 4 and w.anim_speed == 1.0
    assert sp.type == abi.PRIMITIVE_SPHERE and sp.radius == 0.7 and list(sp.position) == [2.1, 0.6, -0.4]
    assert bx.type == abi.PRIMITIVE_BOX and list(bx.size) == [0.8, 1.2, 0.6] and bx.rounding == 0.05
    assert list(bx.rotation) == [10.0, 0.0, 35.0] and bx.scale == 1.0 and list(bx.repeat) == [0.0] * 3
    assert "primitive_water_1_material_id" in s.report  # ignored: a material


@pytest.mark.parametrize("lines,what", [
    ("primitive_blob_1_enabled true;\n", "unknown primitive"),
    ("primitive_sphere_1_enabled true;\nprimitive_sphere_1_boolean_operator 2;\n", "other than by union"),
    ("primitive_box_1_enabled true;\nprimitive_box_1_smooth_de_combine_enable true;\n", "smooth union"),
    ("primitive_box_1_enabled true;\nall_primitives_rotation 0 0 10;\n", "primitive group transform"),
])
def test_primitives_not_built_here(lines, what):
    s = settings.load_from_string(HEADER + "[main_parameters]\n" + lines)
    assert s.status == abi.MBR_EUNSUPPORTED and any(what in u for u in s.unsupported()), s.report


def test_nine_primitives_are_too_many():
    txt = HEADER + "[main_parameters]\n" + "".join(
        f"primitive_sphere_{i}_enabled true;\nprimitive_sphere_{i}_position {i} 0 0;\n" for i in range(1, 10))
    s = settings.load_from_string(txt)
    assert s.status == abi.MBR_EUNSUPPORTED and s.scene.n_primitives == 8
    assert any("more than 8 primitives" in u for u in s.unsupported())


def test_hybrid_sequence():
    s = settings.load_from_file(os.path.join(FIX, "hybrid_bulb_menger.fract"))
    assert s.status == abi.MBR_OK, s.report
    sc = s.scene
    assert sc.hybrid_fractal_enable == 1 and sc.n_fractals == 2
    assert sc.fractal[0].formula == abi.FORMULA_MANDELBULB and sc.fractal[0].formula_iterations == 3
    assert sc.fractal[0].bulb_power == 8.0
    assert sc.fractal[1].formula == abi.FORMULA_MENGER_SPONGE and sc.fractal[1].formula_iterations == 9
    assert sc.formula_maxiter == 12
    assert s.params.view_distance_max == 20.0  # quoted name and value
    # the default light: rotation (-45, 45, 0) relative to the camera
    want = relative_light(s.camera.camera, s.camera.target, s.camera.top, [-45, 45, 0])
    np.testing.assert_allclose(list(s.params.light_direction), want, rtol=0, atol=1e-12)
    # penetrating shadows with a 1 degree soft cone are the reference's defaults
    assert s.params.penetrating == 1 and s.params.soft_shadow_cone == 1.0
    # the sequence the library builds: 3 bulb passes, then 9 Menger passes
    lib = abi.load()
    import ctypes as C

    seq = (C.c_int32 * abi.MBR_SEQUENCE_LENGTH)()
    n, fn, bo = C.c_int32(), C.c_int32(), C.c_double()
    assert lib.mbr_scene_sequence(C.byref(sc), seq, C.byref(n), C.byref(fn), C.byref(bo)) == abi.MBR_OK
    assert list(seq[:12]) == [0, 0, 0] + [1] * 9


def test_legacy_renames():
    s = settings.load_from_file(os.path.join(FIX, "legacy_light.fract"))
    assert s.status == abi.MBR_OK, s.report
    sc, p = s.scene, s.params
    assert sc.fractal[0].formula == abi.FORMULA_MANDELBULB and sc.fractal[0].bulb_power == 6.0
    assert sc.delta_de_function == 2  # before 2.09 the values 0 and 2 were swapped
    assert list(sc.fractal_constant_factor) == [1.1, 1.1, 1.1]  # a scalar before 2.05
    assert p.shading_enable == 1 and p.shadow_enable == 0  # shadows_enabled -> light1_cast_shadows
    # main_light_alpha / beta -> light1 rotation (alpha, beta, 0) (settings.cpp:1420-1421, 1643-1649)
    want = relative_light(s.camera.camera, s.camera.target, s.camera.top, [10, -35, 0])
    np.testing.assert_allclose(list(p.light_direction), want, rtol=0, atol=1e-12)
    assert sc.formula_maxiter == 250  # N's default


def test_light_rotation_zero_points_back_along_the_view():
    txt = HEADER + "[main_parameters]\ncamera 1 -5 2;\ntarget 0 0 0;\ncamera_top 0 0 1;\nlight1_rotation 0 0 0;\n"
    s = settings.load_from_string(txt)
    assert s.ok, s.report
    f = np.array([-1.0, 5.0, -2.0]) / math.sqrt(30.0)
    np.testing.assert_allclose(list(s.params.light_direction), -f, atol=1e-15)


def test_absolute_light_rotation():
    txt = HEADER + ("[main_parameters]\nlight1_relative_position false;\nlight1_rotation 20 10 5;\n")
    s = settings.load_from_string(txt)
    assert s.ok, s.report
    a, b, c = np.array([20.0, -10.0, 5.0]) / 180.8 * math.pi
    rz = np.array([[math.cos(a), -math.sin(a), 0], [math.sin(a), math.cos(a), 0], [0, 0, 1]])
    rx = np.array([[1, 0, 0], [0, math.cos(b), -math.sin(b)], [0, math.sin(b), math.cos(b)]])
    ry = np.array([[math.cos(c), 0, math.sin(c)], [0, 1, 0], [-math.sin(c), 0, math.cos(c)]])
    want = rz @ rx @ ry @ np.array([0.0, -1.0, 0.0])
    np.testing.assert_allclose(list(s.params.light_direction), want, atol=1e-15)


def test_defaults_of_an_empty_file():
    s = settings.load_from_string(HEADER + "[main_parameters]\n")
    assert s.ok, s.report
    sc, cam, p = s.scene, s.camera, s.params
    assert sc.fractal[0].formula == abi.FORMULA_MANDELBULB and sc.fractal[0].bulb_power == 9.0
    assert sc.formula_maxiter == 250 and sc.bailout == 100.0 and sc.use_default_bailout == 1
    assert list(cam.camera) == [3.0, -6.0, 2.0] and list(cam.target) == [0.0, 0.0, 0.0]
    assert list(cam.top) == [-0.1277753, 0.2555506, 0.958314]
    assert (cam.width, cam.height) == (800, 600) and cam.fov_deg == 53.13
    assert p.detail_level == 1.0 and p.view_distance_max == 50.0 and p.max_raymarching_steps == 10000
    assert p.ao_rays == 0 and p.binary_steps == 30


@pytest.mark.parametrize("text,what", [
    ("[main_parameters]\nformula_1 8;\n", "no header"),
    ("# some other file\n# version 2.3\n# only modified parameters\n", "wrong header"),
    ("# Mandelbulber settings file\n# no number here\n# only modified parameters\n", "version"),
    ("# Mandelbulber settings file\n# version 2.33\n# something\n", "format"),
    (HEADER + "[main_parameters]\ncamera 1 2;\n", "malformed"),
    (HEADER + "[main_parameters]\ndetail_level fast;\n", "malformed"),
    (HEADER + "[main_parameters]\nformula_1 8\n", "malformed"),
])
def test_invalid_files(text, what):
    s = settings.load_from_string(text)
    assert s.status == abi.MBR_EINVAL, (what, s.report)
    assert "error" in s.report


def test_unsupported_geometry_is_named():
    txt = HEADER + ("[main_parameters]\nformula_1 104;\n")
    s = settings.load_from_string(txt)
    assert s.status == abi.MBR_EUNSUPPORTED
    assert any(u.startswith("formula_1 104") for u in s.unsupported()), s.report
    txt = HEADER + ("[main_parameters]\nformula_1 8;\nprimitive_prism_1_enabled true;\nprimitive_prism_1_boolean_operator 0;\n"
                    "boolean_operators true;\n"
                    "delta_DE_function 4;\nhybrid_fractal_enable true;\nformula_2 8;\n"
                    "[fractal_1]\nmandelbox_rotations_enabled true;\n")
    s = settings.load_from_string(txt)
    assert s.status == abi.MBR_EUNSUPPORTED
    u = " | ".join(s.unsupported())
    for key in ("primitive_prism_1_boolean_operator 0", "boolean_operators",
                "delta_DE_function 4", "Mandelbox rotations with more than one Mandelbox slot"):
        assert key in u, (key, s.report)
    # a slot that a single-fractal scene does not iterate may name any formula
    s = settings.load_from_string(HEADER + "[main_parameters]\nformula_1 8;\nformula_2 104;\n")
    assert s.ok, s.report


def test_mandelbox_rotations():
    txt = HEADER + ("[main_parameters]\nformula_1 8;\n[fractal_1]\nmandelbox_rotations_enabled true;\n"
                    "mandelbox_main_rotation_enabled true;\nmandelbox_rotation_neg_2 10 0 -5,5;\n"
                    "mandelbox_rotation_pos_3 0 20 0;\nmandelbox_rotation_main 3 -17 41;\n")
    s = settings.load_from_string(txt)
    assert s.ok, s.report
    f = s.scene.fractal[0]
    assert f.mandelbox_rotations_enabled == 1 and f.mandelbox_main_rotation_enabled == 1
    assert list(f.mandelbox_rotation_neg[1]) == [10.0, 0.0, -5.5] and list(f.mandelbox_rotation_neg[0]) == [0.0] * 3
    assert list(f.mandelbox_rotation_pos[2]) == [0.0, 20.0, 0.0]
    assert list(f.mandelbox_rotation_main) == [3.0, -17.0, 41.0]


def test_legacy_coordinate_system():
    s = settings.load_from_string(HEADER + "[main_parameters]\nlegacy_coordinate_system true;\n")
    assert s.ok, s.report
    assert s.camera.legacy_coordinate_system == 1


@pytest.mark.parametrize("quality,tune,want_q,want_t", [("3", "0,5", 3, 0.5), ("50", "0", 10, 1e-5),
                                                        (None, None, 4, 1.0)])
def test_fast_ambient_occlusion(quality, tune, want_q, want_t):
    """ambient_occlusion_mode fast maps onto the fast AO with the quality and
    fast tune clamped to the reference's ranges (initparameters.cpp:215-216)."""
    txt = HEADER + "[main_parameters]\nambient_occlusion_enabled true;\nambient_occlusion_mode fast;\n"
    txt += "ambient_occlusion 0,7;\n"
    if quality is not None:
        txt += f"ambient_occlusion_quality {quality};\nambient_occlusion_fast_tune {tune};\n"
    s = settings.load_from_string(txt)
    assert s.ok, s.report
    p = s.params
    assert p.ao_fast == 1 and p.ao_rays == 0 and p.ambient_intensity == 0.7
    assert p.ao_quality == want_q and p.ao_fast_tune == want_t
    assert "ambient_occlusion" not in s.report


def test_screen_space_ao_is_noted_and_off():
    txt = HEADER + "[main_parameters]\nambient_occlusion_enabled true;\nambient_occlusion_mode screen_space;\n"
    s = settings.load_from_string(txt)
    assert s.ok, s.report
    assert s.params.ao_fast == 0 and s.params.ao_rays == 0
    assert "screen space is not on this path" in s.report


@pytest.mark.parametrize("value,want", [("three_point", 0), ("fish_eye", 1), ("equirectangular", 2),
                                        ("fish_eye_cut", 3), ("2", 2)])
def test_projection(value, want):
    s = settings.load_from_string(HEADER + f"[main_parameters]\nperspective_type {value};\nfov 200;\n")
    assert s.ok, s.report
    assert s.camera.perspective_type == want and s.camera.fov_deg == 200.0


def test_report_is_truncated_safely():
    import ctypes as C

    lib = abi.load()
    sc, cam, p = abi.Scene(), abi.Camera(), abi.RenderParams()
    buf = C.create_string_buffer(8)
    txt = (HEADER + "[main_parameters]\nfog_color_1 1 2 3;\n").encode()
    assert lib.mbr_fract_parse(txt, C.byref(sc), C.byref(cam), C.byref(p), buf, 8) == abi.MBR_OK
    assert len(buf.value) == 7
    assert lib.mbr_fract_parse(txt, C.byref(sc), C.byref(cam), C.byref(p), None, 0) == abi.MBR_OK
    assert lib.mbr_fract_parse(None, C.byref(sc), C.byref(cam), C.byref(p), None, 0) == abi.MBR_EINVAL


@pytest.mark.skipif(not EXAMPLES or not os.path.isdir(EXAMPLES), reason="reference example scenes not present")
def test_reference_examples():
    """Every example scene the reference ships is read: none is malformed, and a
    scene is accepted exactly when the formulas it iterates are built here and
    none of the unsupported features appears.  A stereo image (a switch
    that changes the image plane and is not built) turns a scene away;
    iteration-count normals are read into the render parameters."""
    files = sorted(glob.glob(os.path.join(EXAMPLES, "**", "*.fract"), recursive=True))
    assert len(files) > 150
    ok = 0
    for path in files:
        s = settings.load_from_file(path)
        assert s.status in (abi.MBR_OK, abi.MBR_EUNSUPPORTED), (path, s.report)
        sc = s.scene
        used = range(sc.n_fractals) if sc.hybrid_fractal_enable else range(1)
        formulas = {sc.fractal[i].formula for i in used} - {0}
        text = open(path, errors="replace").read()
        if "\nstereo_enabled true;" in text:
            assert not s.ok and any(u.startswith("stereo_enabled true") for u in s.unsupported()), path
        if "\nslow_shading true;" in text:
            assert s.params.slow_shading == 1, path
        if s.ok:
            ok += 1
            assert formulas <= {2, 3, 4, 5, 7, 8, 10, 11, 19}, (path, formulas)
            assert sc.formula_maxiter >= 1 and s.camera.width >= 5 and s.camera.height >= 5
        elif not formulas <= {2, 3, 4, 5, 7, 8, 10, 11, 19}:
            assert any("formula not built here" in u for u in s.unsupported()), (path, s.report)
    assert ok >= 165, ok


@pytest.mark.skipif(not EXAMPLES or not os.path.isdir(EXAMPLES), reason="reference example scenes not present")
def test_reference_examples_render_on_the_oracle(oracle):
    """Three accepted example scenes (one per formula) rendered small by the
    oracle from the parsed structs: the fractal is in view."""
    names = {"mandelbox001.fract": 8, "iteration fog.fract": 7, "mandelbulb001.fract": 2}
    seen = 0
    for name, formula in names.items():
        path = os.path.join(EXAMPLES, name)
        if not os.path.exists(path):
            continue
        s = settings.load_from_file(path)
        if not s.ok or s.scene.fractal[0].formula != formula:
            continue
        cam = s.camera
        aspect = cam.width / cam.height
        cam.height = 18
        cam.width = max(8, int(round(18 * aspect)))
        p = s.params
        p.ao_rays = 0
        out, st = oracle.render(s.scene, cam, p)
        frac = float(np.mean(out["hit"]))
        assert 0.02 < frac <= 1.0, (name, frac)
        seen += 1
    assert seen >= 1


def test_malformed_text_never_crashes():
    """Random and truncated settings texts: the reader returns a status and a
    report for every one, and never reads past the text."""
    import random

    rng = random.Random(5)
    base = open(os.path.join(FIX, "box_ao.fract")).read()
    pieces = ["camera", "formula_1", "IFS_direction_3", "mandelbox_rotation_neg_2", "fov", ";", " ", ",", "[",
              "]", "fractal_9", "fractal_12", "\n", "\r\n", "true", "1e308", "-0", "nan", "\"", "'", "0,5 1 2"]
    statuses = set()
    for k in range(400):
        if k % 2:
            t = base[: rng.randrange(len(base))]
        else:
            t = HEADER + "".join(rng.choice(pieces) for _ in range(rng.randrange(1, 60)))
        s = settings.load_from_string(t)
        statuses.add(s.status)
        assert s.status in (abi.MBR_OK, abi.MBR_EINVAL, abi.MBR_EUNSUPPORTED)
        assert isinstance(s.report, str)
    assert abi.MBR_EINVAL in statuses


def test_delta_de_settings():
    """delta_DE_method, delta_DE_function and deltade_relative_delta are read
    into the scene (the delta DE renders on the plain FP64 engines); the Jos
    Kleinian function is taken with the delta DE only."""
    s = settings.load_from_string(HEADER + "[main_parameters]\nformula_1 8;\ndelta_DE_method 1;\n"
                                  "delta_DE_function 3;\ndeltade_relative_delta 0,02;\n")
    assert s.ok, s.report
    assert s.scene.delta_de_method == abi.DE_METHOD_FORCE_DELTA
    assert s.scene.delta_de_function == abi.DE_PSEUDO_KLEINIAN
    assert s.scene.deltade_relative_delta == 0.02
    assert "forced delta DE" in s.report
    s = settings.load_from_string(HEADER + "[main_parameters]\nformula_1 8;\ndelta_DE_method 1;\n"
                                  "delta_DE_function 4;\n")
    assert s.ok, s.report
    s = settings.load_from_string(HEADER + "[main_parameters]\nformula_1 8;\ndelta_DE_function 6;\n")
    assert s.ok and s.scene.delta_de_function == abi.DE_MAX_AXIS, s.report
    for bad in ("delta_DE_method 3;", "delta_DE_function 7;", "deltade_relative_delta 0;"):
        s = settings.load_from_string(HEADER + "[main_parameters]\nformula_1 8;\n" + bad + "\n")
        assert s.status == abi.MBR_EINVAL, (bad, s.report)
