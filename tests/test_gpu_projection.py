"""The fish-eye, equirectangular and fish-eye-cut projections
(CalculateViewVector, projection_3d.cpp:40-89; the cut, render_worker.cpp:
165-170, 321) on every engine, against the oracle whose view vectors equal the
reference's bit for bit (tests/golden/projection_kat.json).  Bars as for the
three-point frames: FP64 hits and iterations >= 99.9 % identical with depth
within 1e-9; FP32 and mixed hit mismatch <= 0.5 % with median depth error
<= 1e-4.  Cut pixels are black, with no hit and depth 1e20, on every engine.
"""
import numpy as np
import pytest

from mandelbulber2_b200 import abi, configs

from .parity import compare

pytestmark = pytest.mark.gpu
NAMES = ("depth", "iters", "hit", "normal", "ao", "rgb8")

CASES = [
    ("fish_eye_160", abi.PROJECTION_FISH_EYE, 160.0, 96, 64),
    ("equirectangular_360", abi.PROJECTION_EQUIRECTANGULAR, 360.0, 128, 64),
    ("fish_eye_cut_220", abi.PROJECTION_FISH_EYE_CUT, 220.0, 80, 80),
]


def cut_mask(cam):
    """Pixels of a fish-eye-cut frame beyond 90 degrees from the axis."""
    x = np.arange(cam.width, dtype=np.float64)
    y = np.arange(cam.height, dtype=np.float64)
    ix = (1.0 / cam.width * x[None, :] + -0.5) * (cam.width / cam.height)
    iy = -1.0 / cam.height * y[:, None] + 0.5
    fov = cam.fov_deg / 180.0 * np.pi
    return (np.sqrt(ix * ix + iy * iy) > np.pi * 0.5 / fov).reshape(-1)


@pytest.mark.parametrize("name,persp,fov,w,h", CASES)
def test_projection_vs_oracle(renderer, oracle, name, persp, fov, w, h):
    sc = configs.mandelbulb_scene(8.0, 20)
    cam = configs.camera((0.15, -1.4, 0.3), fov=fov, width=w, height=h)
    cam.perspective_type = persp
    p = configs.base_params(5, 20.0)
    p.ao_rays = 4
    renderer.set_scene(sc)
    o, _ = oracle.render(sc, cam, p)
    assert 0.05 < float(np.mean(o["hit"])) < 0.95, "the fractal is in view"
    cut = cut_mask(cam) if persp == abi.PROJECTION_FISH_EYE_CUT else np.zeros(w * h, bool)
    if persp == abi.PROJECTION_FISH_EYE_CUT:
        assert 0.05 < float(np.mean(cut)) < 0.6
        assert not o["hit"][cut].any() and (o["rgb8"].reshape(-1, 3)[cut] == 0).all()
    for engine in (abi.ENGINE_PLAIN_FP64, abi.ENGINE_PLAIN_MIXED, abi.ENGINE_WAVEFRONT_FP32,
                   abi.ENGINE_WAVEFRONT_AUTO):
        fr = renderer.render(cam, p, engine, outputs=NAMES)
        g = {k: v.cpu().numpy() for k, v in fr.buffers.items()}
        m = compare(g, o)
        print(name, abi.ENGINE_NAMES[engine], m)
        assert fr.stats["pixels"] == w * h
        if engine == abi.ENGINE_PLAIN_FP64:
            assert m["hit_iters_match"] >= 0.999, m
            assert m["depth_rel_le_1e-9"] >= 0.999, m
        else:
            assert m["hit_mismatch"] <= 0.005, m
            assert m["depth_rel_median"] <= 1e-4, m
        if cut.any():
            assert not g["hit"][cut].any()
            assert (g["depth"][cut] == 1e20).all()
            assert (g["rgb8"].reshape(-1, 3)[cut] == 0).all()


def test_fish_eye_cut_gi(renderer, oracle):
    """A GI frame through a fish-eye cut: cut pixels black on the GPU and in
    the oracle, the rest within the GI bar."""
    sc, _, p = configs.hybrid_gi_2160p(48, 48, spp=2)
    cam = configs.camera((0.0, -2.2, 0.3), fov=200.0, width=48, height=48)
    cam.perspective_type = abi.PROJECTION_FISH_EYE_CUT
    renderer.set_scene(sc)
    o, _ = oracle.render(sc, cam, p)
    cut = cut_mask(cam)
    for engine in (abi.ENGINE_PLAIN_MIXED, abi.ENGINE_WAVEFRONT_FP32):
        fr = renderer.render(cam, p, engine, outputs=("depth", "hit", "rgb", "rgb8"))
        g = {k: v.cpu().numpy() for k, v in fr.buffers.items()}
        assert not g["hit"][cut].any() and (g["rgb8"].reshape(-1, 3)[cut] == 0).all()
        diff = np.abs(g["rgb"] - o["rgb"]).reshape(-1, 3)[~cut]
        print(abi.ENGINE_NAMES[engine], float(np.mean(diff < 1e-3)), float(np.mean(diff)))
        assert np.mean(diff < 1e-3) >= 0.9
        assert float(np.mean(diff)) <= 0.01


def test_projection_arguments(renderer):
    from mandelbulber2_b200.render import MbrError

    sc = configs.mandelbulb_scene(8.0, 20)
    renderer.set_scene(sc)
    p = configs.base_params(5, 20.0)
    cam = configs.camera((0.4, -2.4, 0.6), fov=200.0, width=16, height=16)
    with pytest.raises(MbrError):  # beyond 180 degrees only for the other projections
        renderer.render(cam, p)
    cam.perspective_type = 7
    with pytest.raises(MbrError):
        renderer.render(cam, p)


def test_legacy_coordinate_system(renderer, oracle):
    """The legacy image region (y from -0.5 at the top to +0.5 at the bottom,
    render_job.cpp:308-315): every engine against the oracle, and the frame
    is the ordinary one upside down."""
    sc = configs.mandelbulb_scene(8.0, 20)
    cam = configs.camera((0.4, -2.2, 0.9), width=64, height=48)
    p = configs.base_params(5, 20.0)
    renderer.set_scene(sc)
    plain, _ = oracle.render(sc, cam, p)
    cam.legacy_coordinate_system = 1
    o, ost = oracle.render(sc, cam, p)
    hp = plain["hit"].reshape(48, 64)
    ho = o["hit"].reshape(48, 64)
    assert np.mean(ho[1:][::-1] == hp[1:]) >= 0.99 and not np.array_equal(ho, hp)
    for engine in (abi.ENGINE_PLAIN_FP64_STRICT, abi.ENGINE_PLAIN_MIXED, abi.ENGINE_WAVEFRONT_FP32,
                   abi.ENGINE_WAVEFRONT_FP64):
        fr = renderer.render(cam, p, engine, outputs=NAMES)
        g = {k: v.cpu().numpy() for k, v in fr.buffers.items()}
        m = compare(g, o)
        print("legacy", abi.ENGINE_NAMES[engine], m)
        if engine == abi.ENGINE_PLAIN_FP64_STRICT:
            assert m["hit_iters_match"] >= 0.999 and m["depth_rel_le_1e-9"] >= 0.999, m
        else:
            assert m["hit_mismatch"] <= 0.005 and m["depth_rel_median"] <= 1e-4, m
