"""The persistent FP32 wavefront kernel and the multi-job batch launch.

Against the FP64 oracle the FP32 path is held to: hit mismatch <= 0.5 % at
these small sizes (<= 0.1 % at the 1920x1080 benchmark size, bench.py) and
median depth relative error <= 1e-4.  Per-pixel results do not depend on
scheduling, so every launch configuration gives bit-identical frames, and a
batch gives the frames of its jobs rendered one by one.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from mandelbulber2_b200 import abi, configs
from mandelbulber2_b200.render import STATS_FIELDS, alloc_outputs, outputs_struct, stats_dict

from .parity import compare

pytestmark = pytest.mark.gpu
WF = abi.ENGINE_WAVEFRONT_FP32


def frame(renderer, sc, cam, p, engine=WF):
    renderer.set_scene(sc)
    fr = renderer.render(cam, p, engine)
    return {k: v.cpu().numpy() for k, v in fr.buffers.items()}, fr.stats


@pytest.mark.parametrize("name", ["mandelbox", "mandelbulb", "menger"])
def test_wavefront_vs_oracle(renderer, oracle, name):
    if name == "mandelbox":
        sc, cam, p = configs.mandelbox_1080p("A", 192, 108)
    elif name == "mandelbulb":
        sc, cam, p = configs.mandelbulb_512(128, 128)
    else:
        sc = configs.menger_scene()
        cam = configs.camera((0.0, -3.0, 0.5), width=96, height=96)
        p = configs.base_params(5, 20.0)
    g, gs = frame(renderer, sc, cam, p)
    o, os_ = oracle.render(sc, cam, p)
    m = compare(g, o)
    print(name, m, gs["de_evals"], os_["de_evals"])
    assert m["hit_mismatch"] <= 0.005, m
    assert m["depth_rel_median"] <= 1e-4, m
    assert gs["pixels"] == cam.width * cam.height
    assert m["psnr"] >= 30.0, m
    # device counters are consistent: phases add up to all DE evaluations
    parts = sum(gs[k] for k in ("march_steps", "binary_steps", "normal_evals", "shadow_evals", "ao_evals"))
    assert parts == gs["de_evals"]
    assert abs(gs["de_evals"] - os_["de_evals"]) <= 0.05 * os_["de_evals"]


def test_wavefront_results_independent_of_tuning(renderer):
    sc, cam, p = configs.mandelbox_1080p("A", 160, 90)
    base = None
    for t in [(128, 12, 2, 0), (64, 8, 0, 1), (256, 2, 24, 1), (128, 16, 4, 0)]:
        renderer.set_tuning(*t)
        g, st = frame(renderer, sc, cam, p)
        if base is None:
            base, bst = g, st
            continue
        for k in base:
            assert np.array_equal(base[k], g[k]), (t, k)
        assert st == bst
    renderer.set_tuning(128, 12, 2, 0)


@pytest.mark.parametrize("lighting", ["hard_ao_rays", "penetrating_soft_fast_ao"])
def test_batch_matches_single_renders(renderer, lighting):
    """Every job of a batch renders its frame as a render of its own would;
    the second case uses the camera-dependent parts of the shading (the
    penetrating shadow's march length and the fast AO's samples)."""
    lib = abi.load()
    scenes = [configs.mandelbulb_scene(8.0, 100), configs.mandelbox_scene(-1.5, 0.5, 40),
              configs.mandelbox_scene(2.2, 0.4, 40), configs.mandelbulb_scene(5.5, 100)]
    cams = [configs.camera((0.0, -3.0, 0.5), width=64, height=64),
            configs.camera((0.5, -5.5, 1.0), width=100, height=30),
            configs.camera((2.0, 3.0, -1.0), width=32, height=96),
            configs.camera((-2.5, 0.5, 1.5), width=48, height=48)]
    p = configs.base_params(5, 20.0)
    p.ao_rays = 4
    p.ao_seed = 9
    if lighting == "penetrating_soft_fast_ao":
        p.penetrating = 1
        p.soft_shadow_cone = 1.0
        p.ao_rays = 0
        p.ao_fast = 1
        p.ao_quality = 4
        p.ambient_intensity = 0.5
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
    st = lib.mbr_batch_create(renderer.ctx, sc_arr, len(scenes), jobs, len(cams), C.byref(p), C.byref(o), WF,
                              None, C.byref(b))
    assert st == abi.MBR_OK, lib.mbr_last_error_string(renderer.ctx)
    try:
        s = torch.cuda.current_stream()
        for rep in range(2):
            stats.zero_()
            assert lib.mbr_batch_launch(b, C.c_void_p(s.cuda_stream)) == abi.MBR_OK
            renderer.sync()
            got = {k: v.cpu().numpy() for k, v in bufs.items()}
            assert stats_dict(stats)["pixels"] == off
            for i, (sc, cam) in enumerate(zip(scenes, cams)):
                single, _ = frame(renderer, sc, cam, p)
                n = cam.width * cam.height
                for k in got:
                    part = got[k][offs[i]: offs[i] + n]
                    if k == "depth":
                        assert np.allclose(part, single[k], rtol=1e-6), (i, k)
                    else:
                        assert np.mean(part == single[k]) >= 0.999, (i, k)
    finally:
        lib.mbr_batch_destroy(b)


def test_wavefront_rejects_unsupported(renderer):
    from mandelbulber2_b200.render import MbrError

    sc, cam, p = configs.mandelbox_1080p("A", 32, 18)
    p.refine = abi.REFINE_ROOT  # root refinement runs on the plain engines
    renderer.set_scene(sc)
    with pytest.raises(MbrError) as e:
        renderer.render(cam, p, WF)
    assert e.value.status == abi.MBR_EUNSUPPORTED


@pytest.mark.parametrize("engine", [abi.ENGINE_PLAIN_FP64, WF])
def test_row_bands_compose_into_the_frame(renderer, engine):
    """Two row bands rendered into one buffer give the whole frame (sharding a frame over GPUs)."""
    from mandelbulber2_b200.shard import band_params, row_band

    sc, cam, p = configs.mandelbox_1080p("A", 96, 54, ao_rays=4)
    renderer.set_scene(sc)
    whole = renderer.render(cam, p, engine, outputs=("depth", "iters", "hit", "normal", "rgb8"))
    bufs = alloc_outputs(cam.width * cam.height, renderer.device, ("depth", "iters", "hit", "normal", "rgb8"))
    total = 0
    for rank in range(2):
        r0, r1 = row_band(cam.height, 2, rank)
        stats = torch.zeros(len(STATS_FIELDS), dtype=torch.int64, device=renderer.device)
        renderer.render_into(cam, band_params(p, r0, r1), bufs, stats, engine)
        renderer.sync()
        total += stats_dict(stats)["de_evals"]
    for k in bufs:
        assert np.array_equal(bufs[k].cpu().numpy(), whole[k].cpu().numpy()), k
    assert total == whole.stats["de_evals"]
