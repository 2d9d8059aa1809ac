"""Hybrid sequences and Monte Carlo GI on the wavefront engines.

Hybrids iterate in FP32 in the reference's operation order (the plain mixed
kernel's formulas, one pass at a time), held to the FP32 bar against the
oracle.  A GI frame is one task per (pixel, sample) walking its path through
the same random streams as the plain kernel.  In FP64 the wavefront GI gives
the plain FP64 frame up to last-bit differences; in FP32 a path can branch
differently where an estimate falls on the other side of a threshold, so the
FP32 frame is compared with the oracle's pixel by pixel within a tolerance.
Radiance is summed in fixed point, so a GI frame does not depend on the
launch shape.
"""
import numpy as np
import pytest

from mandelbulber2_b200 import abi, configs

from .parity import compare

pytestmark = pytest.mark.gpu
WF32, WF64, AUTO = abi.ENGINE_WAVEFRONT_FP32, abi.ENGINE_WAVEFRONT_FP64, abi.ENGINE_WAVEFRONT_AUTO
NAMES = ("depth", "iters", "hit", "normal", "shade", "ao", "rgb", "rgb8")


def frame(renderer, sc, cam, p, engine):
    renderer.set_scene(sc)
    fr = renderer.render(cam, p, engine, outputs=NAMES)
    return {k: v.cpu().numpy() for k, v in fr.buffers.items()}, fr.stats


def test_hybrid_wavefront_vs_oracle(renderer, oracle):
    sc = configs.hybrid_scene()
    cam = configs.camera((0.0, -3.0, 0.5), width=96, height=72)
    p = configs.base_params(5, 20.0)
    p.ao_rays = 4
    p.ao_seed = 5
    for engine in (WF32, AUTO):
        g, gs = frame(renderer, sc, cam, p, engine)
        o, os_ = oracle.render(sc, cam, p)
        m = compare(g, o)
        print(abi.ENGINE_NAMES[engine], m, gs["de_evals"], os_["de_evals"])
        assert m["hit_mismatch"] <= 0.005, m
        assert m["depth_rel_median"] <= 1e-4, m
        assert m["psnr"] >= 30.0, m
        assert gs["pixels"] == cam.width * cam.height
        assert abs(gs["de_evals"] - os_["de_evals"]) <= 0.05 * os_["de_evals"]


def test_hybrid_fp64_wavefront_is_refused(renderer):
    from mandelbulber2_b200.render import MbrError

    sc = configs.hybrid_scene()
    cam = configs.camera((0.0, -3.0, 0.5), width=16, height=16)
    renderer.set_scene(sc)
    with pytest.raises(MbrError) as e:
        renderer.render(cam, configs.base_params(5, 20.0), WF64)
    assert e.value.status == abi.MBR_EUNSUPPORTED


def test_gi_wavefront_fp32_vs_oracle(renderer, oracle):
    sc, cam, p = configs.hybrid_gi_2160p(64, 36, spp=4)
    g, gs = frame(renderer, sc, cam, p, WF32)
    o, os_ = oracle.render(sc, cam, p)
    m = compare(g, o)
    diff = np.abs(g["rgb"] - o["rgb"])
    print("gi fp32", m, float(np.mean(diff)), gs, os_)
    assert m["hit_mismatch"] <= 0.005, m
    assert m["depth_rel_median"] <= 1e-4, m
    # per-pixel colour: most pixels agree closely; a pixel whose path took
    # another branch differs by one sample's share
    assert np.mean(diff < 1e-3) >= 0.9, float(np.mean(diff < 1e-3))
    assert float(np.mean(diff)) <= 0.01
    assert gs["gi_evals"] > 0 and gs["pixels"] == cam.width * cam.height
    assert abs(gs["de_evals"] - os_["de_evals"]) <= 0.05 * os_["de_evals"]


def test_gi_wavefront_fp64_matches_plain_fp64(renderer):
    """A non-hybrid GI frame: FP64 wavefront and plain FP64 walk the same paths."""
    _, cam, p = configs.hybrid_gi_2160p(64, 36, spp=3)
    sc = configs.mandelbulb_scene(8.0, 20)
    cam = configs.camera((0.0, -2.6, 0.4), width=64, height=36)
    w, ws = frame(renderer, sc, cam, p, WF64)
    f, fs = frame(renderer, sc, cam, p, abi.ENGINE_PLAIN_FP64)
    m = compare(w, f)
    diff = np.abs(w["rgb"] - f["rgb"])
    print("gi fp64", m, float(np.max(diff)), ws, fs)
    assert m["hit_mismatch"] <= 0.001, m
    assert m["depth_rel_le_1e-9"] >= 0.999, m
    assert np.mean(diff < 1e-6) >= 0.99, float(np.mean(diff < 1e-6))
    assert abs(ws["de_evals"] - fs["de_evals"]) <= 0.01 * fs["de_evals"]


def test_gi_wavefront_independent_of_tuning(renderer):
    sc, cam, p = configs.hybrid_gi_2160p(48, 27, spp=2)
    base = None
    for t in [(128, 12, 2, 0), (64, 8, 0, 1), (256, 2, 24, 0)]:
        renderer.set_tuning(*t)
        g, st = frame(renderer, sc, cam, p, WF32)
        if base is None:
            base, bst = g, st
            continue
        for k in base:
            assert np.array_equal(base[k], g[k]), (t, k)
        assert st == bst
    renderer.set_tuning(128, 12, 2, 0)
