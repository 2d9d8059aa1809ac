"""The wavefront engines with FP64 iteration and the per-frame precision policy.

MBR_ENGINE_WAVEFRONT_FP64 runs the reference-order FP64 iteration inside the
wavefront stages and is held to the plain FP64 bar against the oracle: hit
masks and iteration counts identical on >= 99.9 % of pixels, depth within
1e-9 relative on >= 99.9 % of common hits.  AO directions are built in FP32
(as in the FP32 engine), so the AO term and the 8-bit image are held to a
looser bar.  MBR_ENGINE_WAVEFRONT_AUTO must give exactly the frame of the
engine its policy picks: FP32 for the wide view, FP64 for the deep zoom.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from mandelbulber2_b200 import abi, configs
from mandelbulber2_b200.render import STATS_FIELDS, alloc_outputs, outputs_struct, stats_dict

from .parity import compare

pytestmark = pytest.mark.gpu
WF32, WF64, AUTO = abi.ENGINE_WAVEFRONT_FP32, abi.ENGINE_WAVEFRONT_FP64, abi.ENGINE_WAVEFRONT_AUTO
NAMES = ("depth", "iters", "hit", "normal", "ao", "rgb8")


def frame(renderer, sc, cam, p, engine):
    renderer.set_scene(sc)
    fr = renderer.render(cam, p, engine, outputs=NAMES)
    return {k: v.cpu().numpy() for k, v in fr.buffers.items()}, fr.stats


def deep_zoom(renderer, width, height, ao_rays=4):
    """View B: the camera 1e-5 in front of the surface point of view A's centre ray."""
    sc, cam, p = configs.mandelbox_1080p("A", 192, 108, ao_rays=ao_rays)
    a, _ = frame(renderer, sc, cam, p, abi.ENGINE_PLAIN_FP64)
    cdepth = float(a["depth"][(cam.height // 2) * cam.width + cam.width // 2])
    assert cdepth < 1e19
    return configs.mandelbox_1080p("B", width, height, ao_rays=ao_rays, centre_depth=cdepth)


@pytest.mark.parametrize("name", ["mandelbox", "mandelbulb", "menger"])
def test_wavefront_fp64_vs_oracle(renderer, oracle, name):
    if name == "mandelbox":
        sc, cam, p = configs.mandelbox_1080p("A", 192, 108)
    elif name == "mandelbulb":
        sc, cam, p = configs.mandelbulb_512(128, 128)
    else:
        sc = configs.menger_scene()
        cam = configs.camera((0.0, -3.0, 0.5), width=96, height=96)
        p = configs.base_params(5, 20.0)
    g, gs = frame(renderer, sc, cam, p, WF64)
    o, os_ = oracle.render(sc, cam, p)
    m = compare(g, o)
    print(name, m, gs["de_evals"], os_["de_evals"])
    assert m["hit_mismatch"] <= 0.001, m
    assert m["hit_iters_match"] >= 0.999, m
    assert m["depth_rel_le_1e-9"] >= 0.999, m
    assert m["normal_deg_p99"] <= 1e-3, m
    both = g["hit"].astype(bool) & o["hit"].astype(bool)
    assert np.median(np.abs(g["ao"][both] - o["ao"][both])) <= 1e-6
    assert m["psnr"] >= 40.0, m
    assert gs["pixels"] == cam.width * cam.height
    parts = sum(gs[k] for k in ("march_steps", "binary_steps", "normal_evals", "shadow_evals", "ao_evals"))
    assert parts == gs["de_evals"]
    assert abs(gs["de_evals"] - os_["de_evals"]) <= 0.01 * os_["de_evals"]


def test_wavefront_fp64_deep_zoom_matches_plain_fp64(renderer):
    """Camera 1e-5 from the surface, FOV 0.5: the FP64 wavefront keeps the
    plain FP64 frame, normals included (FP32 points cannot resolve them)."""
    sc, cam, p = deep_zoom(renderer, 96, 54)
    w, _ = frame(renderer, sc, cam, p, WF64)
    f, _ = frame(renderer, sc, cam, p, abi.ENGINE_PLAIN_FP64)
    m = compare(w, f)
    print("deep zoom fp64 wavefront vs plain", m)
    assert m["hit_mismatch"] <= 0.001, m
    assert m["depth_rel_le_1e-9"] >= 0.999, m
    assert m["normal_deg_p99"] <= 1e-2, m


def test_auto_picks_fp32_for_the_wide_view_and_fp64_for_the_deep_zoom(renderer):
    sc, cam, p = configs.mandelbox_1080p("A", 160, 90, ao_rays=4)
    a, ast = frame(renderer, sc, cam, p, AUTO)
    f32, st32 = frame(renderer, sc, cam, p, WF32)
    for k in NAMES:
        assert np.array_equal(a[k], f32[k]), k
    assert ast == st32
    sc, cam, p = deep_zoom(renderer, 80, 45)
    a, ast = frame(renderer, sc, cam, p, AUTO)
    f64, st64 = frame(renderer, sc, cam, p, WF64)
    for k in NAMES:
        assert np.array_equal(a[k], f64[k]), k
    assert ast == st64


def test_wavefront_fp64_results_independent_of_tuning(renderer):
    sc, cam, p = configs.mandelbox_1080p("A", 128, 72, ao_rays=4)
    base = None
    for t in [(128, 12, 2, 0), (64, 8, 0, 1), (256, 2, 24, 1)]:
        renderer.set_tuning(*t)
        g, st = frame(renderer, sc, cam, p, WF64)
        if base is None:
            base, bst = g, st
            continue
        for k in base:
            assert np.array_equal(base[k], g[k]), (t, k)
        assert st == bst
    renderer.set_tuning(128, 12, 2, 0)


@pytest.mark.parametrize("engine", [WF64, AUTO])
def test_batch_matches_single_renders_fp64_and_auto(renderer, engine):
    """Jobs of two formulas, one with the camera inside a positive-scale
    Mandelbox (FP64 under the policy); the batch gives the single renders."""
    lib = abi.load()
    scenes = [configs.mandelbulb_scene(8.0, 100), configs.mandelbox_scene(-1.5, 0.5, 40),
              configs.mandelbox_scene(2.2, 0.4, 40), configs.mandelbulb_scene(5.5, 100),
              configs.mandelbox_scene(2.2, 0.4, 40)]
    cams = [configs.camera((0.0, -3.0, 0.5), width=64, height=64),
            configs.camera((0.5, -5.5, 1.0), width=100, height=30),
            configs.camera((2.0, 3.0, -1.0), width=32, height=96),
            configs.camera((-2.5, 0.5, 1.5), width=48, height=48),
            configs.camera((1.65, 1.65, 1.14), width=40, height=40)]  # inside the solid: DE 4e-18
    p = configs.base_params(5, 20.0)
    p.ao_rays = 4
    p.ao_seed = 9
    jobs = (abi.Job * len(cams))()
    off = 0
    offs = []
    for i, c in enumerate(cams):
        jobs[i].camera = c
        jobs[i].scene_index = i
        jobs[i].pixel_offset = off
        offs.append(off)
        off += c.width * c.height
    sc_arr = (abi.Scene * len(scenes))(*scenes)
    bufs = alloc_outputs(off, renderer.device, ("depth", "iters", "hit", "normal", "ao", "rgb8"))
    stats = torch.zeros(len(STATS_FIELDS), dtype=torch.int64, device=renderer.device)
    o = outputs_struct(bufs, stats)
    b = C.c_void_p()
    st = lib.mbr_batch_create(renderer.ctx, sc_arr, len(scenes), jobs, len(cams), C.byref(p), C.byref(o), engine,
                              None, C.byref(b))
    assert st == abi.MBR_OK, lib.mbr_last_error_string(renderer.ctx)
    try:
        wide = C.c_int32(0)
        groups = lib.mbr_batch_groups(b, C.byref(wide))
        if engine == WF64:
            assert wide.value == len(cams) and groups == 2
        else:
            assert wide.value == 1 and groups == 3  # only the camera inside the solid iterates in FP64
        s = torch.cuda.current_stream()
        stats.zero_()
        assert lib.mbr_batch_launch(b, C.c_void_p(s.cuda_stream)) == abi.MBR_OK
        renderer.sync()
        got = {k: v.cpu().numpy() for k, v in bufs.items()}
        assert stats_dict(stats)["pixels"] == off
        for i, (sc, cam) in enumerate(zip(scenes, cams)):
            single, _ = frame(renderer, sc, cam, p, engine)
            n = cam.width * cam.height
            for k in got:
                part = got[k][offs[i]: offs[i] + n]
                if k == "depth":
                    assert np.allclose(part, single[k], rtol=1e-6), (i, k)
                else:
                    assert np.mean(part == single[k]) >= 0.999, (i, k)
    finally:
        lib.mbr_batch_destroy(b)
