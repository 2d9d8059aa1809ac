"""Mandelbulb power 2 (formula 3), hypercomplex (formula 4) and the
kaleidoscopic IFS (formula 10), the formulas beyond the Mandelbulb, Mandelbox
and Menger sponge.  They iterate in
the reference's operation order (de_core.cuh), on the plain engines and, for
the 3-D ones, on the FP32 wavefront through the reference-order policy.  The
oracle's steps equal the reference's FormulaCode bit for bit
(tests/golden/formula_kat.json); the formulas use only +, -, *, /, sqrt and
fabs (the IFS matrices are built on the host), so the strict FP64 kernel is
held to bit-exactness against the oracle.
"""
import numpy as np
import pytest

from mandelbulber2_b200 import abi, configs

from .parity import compare

pytestmark = pytest.mark.gpu
NAMES = ("depth", "iters", "hit", "normal", "ao", "rgb8")


def scene(formula):
    sc = abi.scene_defaults(formula)
    sc.formula_maxiter = 30
    cam = configs.camera((0.3, -1.8, 0.6), width=96, height=64)
    p = configs.base_params(5, 20.0)
    p.ao_rays = 4
    return sc, cam, p


def check(renderer, sc, cam, p, o, ost, engine, name):
    fr = renderer.render(cam, p, engine, outputs=NAMES)
    g = {k: v.cpu().numpy() for k, v in fr.buffers.items()}
    m = compare(g, o)
    print(name, abi.ENGINE_NAMES[engine], m)
    if engine == abi.ENGINE_PLAIN_FP64_STRICT:
        for k in NAMES:
            assert np.array_equal(g[k], o[k]), (name, k)
        assert fr.stats == ost
    elif engine == abi.ENGINE_PLAIN_FP64:
        assert m["hit_iters_match"] >= 0.999, m
        assert m["depth_rel_le_1e-9"] >= 0.999, m
    else:
        assert m["hit_mismatch"] <= 0.005, m
        assert m["depth_rel_median"] <= 1e-4, m


def test_mandelbulb_power2(renderer, oracle):
    sc, cam, p = scene(abi.FORMULA_MANDELBULB_POWER2)
    renderer.set_scene(sc)
    o, ost = oracle.render(sc, cam, p)
    assert 0.1 < float(np.mean(o["hit"])) < 0.95
    for engine in (abi.ENGINE_PLAIN_FP64_STRICT, abi.ENGINE_PLAIN_FP64, abi.ENGINE_PLAIN_MIXED,
                   abi.ENGINE_WAVEFRONT_FP32, abi.ENGINE_WAVEFRONT_AUTO):
        check(renderer, sc, cam, p, o, ost, engine, "power2")


def test_hypercomplex(renderer, oracle):
    from mandelbulber2_b200.render import MbrError

    sc, cam, p = scene(abi.FORMULA_HYPERCOMPLEX)
    renderer.set_scene(sc)
    o, ost = oracle.render(sc, cam, p)
    assert 0.1 < float(np.mean(o["hit"])) < 0.95
    for engine in (abi.ENGINE_PLAIN_FP64_STRICT, abi.ENGINE_PLAIN_FP64):
        check(renderer, sc, cam, p, o, ost, engine, "hypercomplex")
    # the 4-D state runs on the plain FP64 engines only
    for engine in (abi.ENGINE_PLAIN_MIXED, abi.ENGINE_WAVEFRONT_FP32):
        with pytest.raises(MbrError) as e:
            renderer.render(cam, p, engine, outputs=NAMES)
        assert e.value.status == abi.MBR_EUNSUPPORTED


def test_generic_formulas_refused_where_not_built(renderer):
    from mandelbulber2_b200.render import MbrError

    sc, cam, p = scene(abi.FORMULA_MANDELBULB_POWER2)
    renderer.set_scene(sc)
    with pytest.raises(MbrError) as e:
        renderer.render(cam, p, abi.ENGINE_WAVEFRONT_FP64, outputs=NAMES)
    assert e.value.status == abi.MBR_EUNSUPPORTED


def ifs_scene():
    sc = abi.scene_defaults(abi.FORMULA_KALEIDOSCOPIC_IFS)
    f = sc.fractal[0]
    f.ifs_scale = 3.0
    f.ifs_offset[:] = [1.0, 1.0, 1.0]
    f.ifs_menger_sponge_mode = 1
    f.ifs_abs_x = f.ifs_abs_y = f.ifs_abs_z = 1
    for i, d in ((5, [1.0, -1.0, 0.0]), (6, [1.0, 0.0, -1.0]), (7, [0.39, 1.0, -1.0])):
        f.ifs_enabled[i] = 1
        f.ifs_direction[i][:] = d
    f.ifs_rotation_enabled = 1
    f.ifs_rotation[:] = [20.0, 0.0, 10.0]
    sc.formula_maxiter = 20
    cam = configs.camera((1.2, -2.2, 1.5), width=96, height=64)
    p = configs.base_params(5, 20.0)
    p.ao_rays = 4
    return sc, cam, p


def test_kaleidoscopic_ifs(renderer, oracle):
    sc, cam, p = ifs_scene()
    renderer.set_scene(sc)
    o, ost = oracle.render(sc, cam, p)
    assert 0.1 < float(np.mean(o["hit"])) < 0.95
    for engine in (abi.ENGINE_PLAIN_FP64_STRICT, abi.ENGINE_PLAIN_FP64, abi.ENGINE_PLAIN_MIXED,
                   abi.ENGINE_WAVEFRONT_FP32, abi.ENGINE_WAVEFRONT_AUTO):
        check(renderer, sc, cam, p, o, ost, engine, "ifs")


def test_xenodreambuie(renderer, oracle):
    """Formula 11: transcendental, so FP64 is held to the FP64 bar (not
    bit-exactness) and FP32 to the FP32 bar."""
    sc = abi.scene_defaults(abi.FORMULA_XENODREAMBUIE)
    sc.fractal[0].bulb_power = 5.0
    sc.formula_maxiter = 30
    cam = configs.camera((0.5, -2.4, 0.9), width=96, height=64)
    p = configs.base_params(5, 20.0)
    p.ao_rays = 4
    renderer.set_scene(sc)
    o, _ = oracle.render(sc, cam, p)
    assert 0.1 < float(np.mean(o["hit"])) < 0.95
    for engine in (abi.ENGINE_PLAIN_FP64_STRICT, abi.ENGINE_PLAIN_FP64, abi.ENGINE_PLAIN_MIXED,
                   abi.ENGINE_WAVEFRONT_FP32, abi.ENGINE_WAVEFRONT_AUTO):
        fr = renderer.render(cam, p, engine, outputs=NAMES)
        g = {k: v.cpu().numpy() for k, v in fr.buffers.items()}
        m = compare(g, o)
        print("xenodreambuie", abi.ENGINE_NAMES[engine], m)
        if engine in (abi.ENGINE_PLAIN_FP64_STRICT, abi.ENGINE_PLAIN_FP64):
            assert m["hit_iters_match"] >= 0.999, m
            assert m["depth_rel_le_1e-9"] >= 0.999, m
        else:
            assert m["hit_mismatch"] <= 0.005, m
            assert m["depth_rel_median"] <= 1e-4, m


def test_quaternion(renderer, oracle):
    """Formula 5 (fractal_quaternion.cpp:29-39): +, -, * only, so the strict
    FP64 kernel is bit-exact; 3-D, so every engine that takes extended
    scenes renders it."""
    sc, cam, p = scene(abi.FORMULA_QUATERNION)
    cam.camera[:] = [0.3, -2.4, 0.8]
    renderer.set_scene(sc)
    o, ost = oracle.render(sc, cam, p)
    assert 0.05 < float(np.mean(o["hit"])) < 0.95
    for engine in (abi.ENGINE_PLAIN_FP64_STRICT, abi.ENGINE_PLAIN_FP64, abi.ENGINE_PLAIN_MIXED,
                   abi.ENGINE_WAVEFRONT_FP32, abi.ENGINE_WAVEFRONT_AUTO):
        check(renderer, sc, cam, p, o, ost, engine, "quaternion")


@pytest.mark.parametrize("case", ["aexion", "hybrid_aexion_quaternion"])
def test_aexion(renderer, oracle, case):
    """Formula 19 (fractal_aexion.cpp:29-59): 4-D, with the orbit's c replaced
    at its first iteration; the plain FP64 engines render it (strict
    bit-exact), the FP32 engines refuse its 4-D state."""
    from mandelbulber2_b200.render import MbrError
    from tests.golden.pipeline_cases import cases

    sc = cases()[case]
    _, cam, p = scene(abi.FORMULA_AEXION)
    cam.camera[:] = [0.5, -3.5, 1.2]
    renderer.set_scene(sc)
    o, ost = oracle.render(sc, cam, p)
    assert 0.05 < float(np.mean(o["hit"])) < 0.95, float(np.mean(o["hit"]))
    for engine in (abi.ENGINE_PLAIN_FP64_STRICT, abi.ENGINE_PLAIN_FP64):
        check(renderer, sc, cam, p, o, ost, engine, case)
    for engine in (abi.ENGINE_PLAIN_MIXED, abi.ENGINE_WAVEFRONT_FP32, abi.ENGINE_WAVEFRONT_AUTO):
        with pytest.raises(MbrError) as e:
            renderer.render(cam, p, engine)
        assert e.value.status == abi.MBR_EUNSUPPORTED


@pytest.mark.parametrize("case", ["hybrid_box_ifs_pow2", "hybrid_bulb_rotated_box"])
def test_ifs_and_rotated_mandelbox_in_hybrids(renderer, oracle, case):
    """A hybrid with its one kaleidoscopic IFS slot, and one with its one
    (rotated) Mandelbox slot: the scene's IFS and rotation blocks belong to
    that slot.  Strict FP64 is bit-exact where the sequence has no
    transcendental function; every engine that takes hybrids is held to its
    bar."""
    from tests.golden.pipeline_cases import cases

    sc = cases()[case]
    cam = configs.camera((0.4, -3.0, 0.9), width=96, height=64)
    p = configs.base_params(5, 20.0)
    p.ao_rays = 4
    renderer.set_scene(sc)
    o, ost = oracle.render(sc, cam, p)
    assert 0.05 < float(np.mean(o["hit"])) < 0.95, float(np.mean(o["hit"]))
    engines = [abi.ENGINE_PLAIN_FP64, abi.ENGINE_PLAIN_MIXED, abi.ENGINE_WAVEFRONT_FP32, abi.ENGINE_WAVEFRONT_AUTO]
    if "bulb_rotated" not in case:
        engines.insert(0, abi.ENGINE_PLAIN_FP64_STRICT)
    for engine in engines:
        check(renderer, sc, cam, p, o, ost, engine, case)


KEYED_CASES = ["pk_default", "pk_params", "pk_sphere_inversion", "pk_prism", "pk_box_folds",
               "pk_rotation_flip_scale", "hybrid_pk_box", "pk_delta", "bfbp2_default", "bfbp2_params",
               "bfbp2_forced_analytic", "menger_mod1_default", "menger_mod1_rotation",
               "menger_mod1_box_offset_blend", "hybrid_menger_mod1_bfbp2", "bfbp2v2_default", "bfbp2v2_vary",
               "bfbp2v2_vary_m", "abox_mod11_default", "abox_mod11_folds", "abox_mod11_curve_c",
               "hybrid_abox_mod11_bulb", "pkm4_default", "pkm4_sphere_box", "pkm4_fold_n", "pksd_default",
               "pksd_benesi", "pksd_folds", "hybrid_pksd_box"] + [f"gfb_type{k}" for k in range(8)] + ["gfb_rotated", "pupuku_default", "pupuku_options", "pupuku_custom_de",
                                                             "hextgrid2_default", "hextgrid2_options"]


# formulas whose orbits at random points are chaotic in every engine that
# rounds differently from the strict one (folds that branch on the sign or
# the order of coordinates, no escape): their FMA and FP32 distances there
# are reported, and their frames are held to the frame bars below
CHAOTIC = ("pksd_", "gfb_", "hextgrid2_")


@pytest.mark.parametrize("case", KEYED_CASES)
def test_keyed_formula_distances(renderer, oracle, case):
    """The formulas whose parameters come by settings key: the pseudo-Kleinian
    (103, fractal_pseudo_kleinian.cpp:30-202, with its DE state and the
    convergence bailout of compute_fractal.cpp:323-336), the box fold bulb
    pow 2 (16, a delta-DE formula), Menger mod 1 (61), box fold bulb pow 2 V2
    (125, with its varying scale) and Abox mod 11 (119, with aux.actualScale,
    the parameter curve and the permuted aux.c).  The oracle equals
    the reference's own CalculateDistance on these scenes
    (tests/golden/pipeline_kat.json).  The formulas use +, -, *, /, sqrt and
    fabs only (rotation matrices are built on the host), so the strict FP64
    engine equals the oracle bit for bit, iteration counts included, except
    where libm enters (a Mandelbulb slot, or the logarithmic DE function of
    the box fold bulb pow 2 V2): there CUDA's and the host's functions differ
    by an ulp here and there, and the strict engine is held to identical
    iteration counts and 1e-13 relative on >= 99 % of the points (the
    Mandelbulb Pupuku calls asin, atan2, pow and sincos every iteration, and
    its non-escaping orbits magnify an ulp: 99.6 % to 99.7 % are within
    1e-13).  The FMA
    and mixed engines are held to a median relative error of 1e-6 (FMA) and
    1e-3 (FP32): pseudo-Kleinian orbits never escape (the convergence bailout
    ends them) and an FMA's rounding can end one an iteration apart, so no
    tight per-point bar holds for them; for the std-DE pseudo-Kleinian and
    the generalized fold box not even the median holds (their orbits at
    random points branch chaotically), so those two are reported there and
    held to the frame bars instead.  FP32 engines refuse the delta DE."""
    from tests.golden.pipeline_cases import cases

    sc = cases()[case]
    renderer.set_scene(sc)
    pts = np.random.default_rng(31).uniform(-2.0, 2.0, size=(4096, 3))
    import torch
    for det in (1e-3, 0.05):
        for nm in (False, True):
            od, oit = oracle.distance(sc, pts, det, nm)
            d, it = renderer.distance(torch.from_numpy(pts), det, nm, abi.ENGINE_PLAIN_FP64_STRICT)
            d0, it0 = d.cpu().numpy(), it.cpu().numpy()
            if "bulb" not in case and "bfbp2v2" not in case and "pupuku" not in case:
                assert np.array_equal(d0, od) and np.array_equal(it0, oit), (case, det, nm)
            else:  # libm's log (the logarithmic DE function) or the Mandelbulb's functions: an ulp apart
                rel0 = np.abs(d0 - od) / np.maximum(np.abs(od), 1e-300)
                assert np.array_equal(it0, oit) and np.mean(rel0 <= 1e-13) >= 0.99, (case, det, nm)
            n = sc.n_fractals if sc.hybrid_fractal_enable else 1
            uses_delta_formula = any(sc.fractal[k].formula == abi.FORMULA_BOX_FOLD_BULB_POW2 for k in range(n))
            delta = (uses_delta_formula or sc.delta_de_method == abi.DE_METHOD_FORCE_DELTA) and \
                sc.delta_de_method != abi.DE_METHOD_FORCE_ANALYTIC
            engines = [abi.ENGINE_PLAIN_FP64] + ([] if delta else [abi.ENGINE_PLAIN_MIXED])
            for engine in engines:
                d, it = renderer.distance(torch.from_numpy(pts), det, nm, engine)
                d, it = d.cpu().numpy(), it.cpu().numpy()
                rel = np.abs(d - od) / np.maximum(np.abs(od), 1e-300)
                print(case, det, nm, abi.ENGINE_NAMES[engine], "rel median", np.median(rel), "p90",
                      np.percentile(rel, 90), "iters", np.mean(it == oit))
                if case.startswith(CHAOTIC):
                    continue  # reported only: see the docstring
                assert np.median(rel) <= (1e-6 if engine == abi.ENGINE_PLAIN_FP64 else 1e-3), (case, engine)


def test_pseudo_kleinian_frames(renderer, oracle):
    """An interior view of the pseudo-Kleinian (the settings of the
    reference's example 'pseudo kleinian 002', whose frame the oracle
    reproduces bit for bit, tests/golden/render_kat.json): strict FP64
    bit-exact, FP64 and mixed engines to their bars; the wavefront engines
    refuse the formula."""
    from mandelbulber2_b200.render import MbrError
    from tests.golden.pipeline_cases import render_cases

    _, sc, cam, _ = [c for c in render_cases() if c[0] == "pseudo_kleinian"][0]
    cam.width, cam.height = 96, 64
    p = configs.base_params(5, 20.0)
    p.ao_rays = 4
    renderer.set_scene(sc)
    o, ost = oracle.render(sc, cam, p)
    for engine in (abi.ENGINE_PLAIN_FP64_STRICT, abi.ENGINE_PLAIN_FP64, abi.ENGINE_PLAIN_MIXED):
        check(renderer, sc, cam, p, o, ost, engine, "pseudo_kleinian")
    for engine in (abi.ENGINE_WAVEFRONT_FP32, abi.ENGINE_WAVEFRONT_FP64, abi.ENGINE_WAVEFRONT_AUTO):
        with pytest.raises(MbrError) as e:
            renderer.render(cam, p, engine)
        assert e.value.status == abi.MBR_EUNSUPPORTED


@pytest.mark.parametrize("case,pos", [("gfb_type3", (0.5, -5.0, 1.5)), ("gfb_rotated", (0.0, -14.0, 2.0)),
                                      ("pksd_default", (2.12066528836305, -3.70836995527439, 1.90220668159675))])
def test_chaotic_keyed_formula_frames(renderer, oracle, case, pos):
    """Frames of the formulas whose random-point distances are chaotic on
    the rounding-different engines: strict FP64 bit-exact against the oracle;
    plain FP64 (FMA) hits and iterations >= 99 % identical; mixed FP32 hit
    mismatch <= 2 % and median depth error <= 1e-3 (a march ends where an
    orbit's branch flips, so a few pixels move)."""
    from tests.golden.pipeline_cases import cases

    sc = cases()[case]
    cam = configs.camera(pos, width=96, height=64)
    p = configs.base_params(5, 30.0)
    p.ao_rays = 4
    renderer.set_scene(sc)
    o, ost = oracle.render(sc, cam, p)
    assert 0.05 < float(np.mean(o["hit"])), float(np.mean(o["hit"]))
    for engine in (abi.ENGINE_PLAIN_FP64_STRICT, abi.ENGINE_PLAIN_FP64, abi.ENGINE_PLAIN_MIXED):
        fr = renderer.render(cam, p, engine, outputs=NAMES)
        g = {k: v.cpu().numpy() for k, v in fr.buffers.items()}
        m = compare(g, o)
        print(case, abi.ENGINE_NAMES[engine], m)
        if engine == abi.ENGINE_PLAIN_FP64_STRICT:
            for k in NAMES:
                assert np.array_equal(g[k], o[k]), (case, k)
            assert fr.stats == ost
        elif engine == abi.ENGINE_PLAIN_FP64:
            assert m["hit_iters_match"] >= 0.99, (case, m)
        else:
            assert m["hit_mismatch"] <= 0.02 and m["depth_rel_median"] <= 1e-3, (case, m)
