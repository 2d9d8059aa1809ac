"""The oracle's reading of CalcDistThresh's tail, CalcDelta and the march
step limits (render_worker.cpp:98-100, 653-690, 819-834), on the CPU."""
import ctypes as C

import numpy as np

from mandelbulber2_b200 import abi, configs


def view(oracle, cam, x, y):
    d = (C.c_double * 3)()
    oracle.lib.oracle_view(C.byref(cam), x, y, d)
    return list(d)


def view_ip(oracle, cam, ix, iy):
    d = (C.c_double * 3)()
    oracle.lib.oracle_view_ip(C.byref(cam), ix, iy, d)
    return list(d)


def test_equirectangular_image_plane_is_2_to_1(oracle):
    """aspectRatio = 2.0 for an equirectangular view whatever the frame's shape:
    pixel (0, 0) of a 96 x 72 frame is the image point (-1, 0.5)."""
    cam = configs.camera((0.1, -2.0, 0.3), fov=360.0, width=96, height=72)
    cam.perspective_type = abi.PROJECTION_EQUIRECTANGULAR
    assert view(oracle, cam, 0, 0) == view_ip(oracle, cam, -1.0, 0.5)
    cam.perspective_type = abi.PROJECTION_FISH_EYE  # the frame's own aspect otherwise
    assert view(oracle, cam, 0, 0) == view_ip(oracle, cam, -0.5 * 96 / 72, 0.5)


def test_equirectangular_halves_the_threshold(oracle):
    """With the threshold halved the surface is found closer to itself: the
    equirectangular frame needs more march and binary steps than the same
    rays marched with the full threshold would (here: detail_level 2 halves
    the threshold of a fish-eye view of the same rays instead)."""
    sc = configs.mandelbulb_scene(8.0, 20)
    p = configs.base_params(5, 20.0)
    p.shading_enable = 0
    p.jitter = 0
    cam = configs.camera((0.15, -1.4, 0.3), fov=360.0, width=48, height=24)
    cam.perspective_type = abi.PROJECTION_EQUIRECTANGULAR
    eq, _ = oracle.render(sc, cam, p)
    # the same view vectors, through detail_level 2 instead of the halving
    # (fish eye at 2:1 gives other vectors, so compare the threshold effect
    # by detail level on the equirectangular view itself)
    p2 = configs.base_params(5, 20.0)
    p2.shading_enable = 0
    p2.jitter = 0
    p2.detail_level = 0.5  # doubles the threshold back: the pre-halving frame
    full, _ = oracle.render(sc, cam, p2)
    both = (eq["hit"] > 0) & (full["hit"] > 0)
    assert both.mean() > 0.1
    # a smaller threshold stops the march later along the ray
    assert np.mean(eq["depth"][both] >= full["depth"][both]) > 0.9


def test_advanced_quality_with_the_default_limits(oracle):
    """With the reference's default limits (detail sizes 1e-12..1, steps
    1e-15..3, relative 0.01..1e4 thresholds) only the start of the march
    changes: at the camera the threshold is 0, clamped up to 1e-12, so the
    first step is limited to 1e4 x 1e-12 = 1e-8 and the next ones grow by
    about 1e4 / (distance per unit threshold) each.  The march takes a few
    more steps per pixel and finds the same surface."""
    sc, cam, p = configs.mandelbox_1080p("A", 64, 36, ao_rays=0)
    p.jitter = 0
    a, ast = oracle.render(sc, cam, p)
    p.advanced_quality = 1
    b, bst = oracle.render(sc, cam, p)
    extra = (bst["march_steps"] - ast["march_steps"]) / (64 * 36)
    assert 2.0 <= extra <= 6.0, extra
    assert np.mean(a["hit"] == b["hit"]) >= 0.99
    both = (a["hit"] > 0) & (b["hit"] > 0)
    assert np.median(np.abs(a["depth"][both] - b["depth"][both]) / a["depth"][both]) < 1e-2


def test_advanced_quality_limits_bind(oracle):
    sc, cam, p = configs.mandelbox_1080p("A", 64, 36, ao_rays=0)
    a, ast = oracle.render(sc, cam, p)
    p.advanced_quality = 1
    p.abs_max_marching_step = 0.25
    b, bst = oracle.render(sc, cam, p)
    assert bst["march_steps"] > 1.5 * ast["march_steps"]
    p.abs_max_marching_step = 3.0
    p.detail_size_max = 1e-3  # a smaller threshold everywhere: later, more precise hits
    c, cst = oracle.render(sc, cam, p)
    both = (a["hit"] > 0) & (c["hit"] > 0)
    assert np.mean(c["depth"][both] >= a["depth"][both]) > 0.95
