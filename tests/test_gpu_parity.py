"""CUDA kernels (through the C-ABI) against the CPU oracle on the same inputs.

Plain FP64 bar: hit mask and iteration count identical on >= 99.9 % of pixels,
depth within 1e-9 relative on common hits, 8-bit image PSNR >= 50 dB.  The
strict-FP64 build (no FMA contraction) performs the oracle's IEEE operations:
for the Mandelbox and Menger sponge (no transcendental functions) it is
expected bit-exact.  Mixed precision: depth relative error <= 1e-4 (median and
99th percentile stated), hit mismatch <= 0.1 %.
"""
import numpy as np
import pytest
import torch

from mandelbulber2_b200 import abi, configs

from .parity import compare

pytestmark = pytest.mark.gpu


def gpu_frame(renderer, sc, cam, p, engine):
    renderer.set_scene(sc)
    fr = renderer.render(cam, p, engine)
    out = {k: v.cpu().numpy() for k, v in fr.buffers.items()}
    return out, fr.stats


FP64_ENGINES = [abi.ENGINE_PLAIN_FP64_STRICT, abi.ENGINE_PLAIN_FP64]


@pytest.mark.parametrize("engine", FP64_ENGINES)
def test_mandelbulb_fp64_parity(renderer, oracle, engine):
    sc, cam, p = configs.mandelbulb_512(128, 128)
    g, gs = gpu_frame(renderer, sc, cam, p, engine)
    o, os_ = oracle.render(sc, cam, p)
    m = compare(g, o)
    print(abi.ENGINE_NAMES[engine], m)
    assert m["hit_iters_match"] >= 0.999, m
    assert m["depth_rel_le_1e-9"] >= 0.999, m
    assert m["psnr"] >= 50.0, m
    assert gs["pixels"] == os_["pixels"] == 128 * 128


@pytest.mark.parametrize("engine", FP64_ENGINES)
def test_mandelbox_fp64_parity(renderer, oracle, engine):
    sc, cam, p = configs.mandelbox_1080p("A", 192, 108)
    g, gs = gpu_frame(renderer, sc, cam, p, engine)
    o, os_ = oracle.render(sc, cam, p)
    m = compare(g, o)
    print(abi.ENGINE_NAMES[engine], m, gs, os_)
    assert m["hit_iters_match"] >= 0.999, m
    assert m["depth_rel_le_1e-9"] >= 0.999, m
    assert m["psnr"] >= 50.0, m
    if engine == abi.ENGINE_PLAIN_FP64_STRICT:
        # only IEEE-rounded +,-,*,/,sqrt on this path: bit-exact, counters identical
        for k in ("depth", "iters", "hit", "normal", "ao", "rgb8"):
            assert np.array_equal(g[k], o[k]), k
        assert gs == os_


def test_menger_and_hybrid_fp64_strict(renderer, oracle):
    for sc in (configs.menger_scene(), configs.hybrid_scene()):
        cam = configs.camera((0.0, -3.0, 0.5), fov=53.0, width=96, height=96)
        p = configs.base_params(5, 20.0)
        g, _ = gpu_frame(renderer, sc, cam, p, abi.ENGINE_PLAIN_FP64_STRICT)
        o, _ = oracle.render(sc, cam, p)
        m = compare(g, o)
        print(m)
        assert m["hit_iters_match"] >= 0.999, m
        assert m["depth_rel_le_1e-9"] >= 0.999, m
        assert m["psnr"] >= 50.0, m


def test_reference_binary_search_30(renderer, oracle):
    """The reference's own refinement (30 halvings with the 0.1 % window)."""
    sc, cam, p = configs.mandelbulb_512(64, 64, binary_steps=30)
    g, _ = gpu_frame(renderer, sc, cam, p, abi.ENGINE_PLAIN_FP64_STRICT)
    o, _ = oracle.render(sc, cam, p)
    m = compare(g, o)
    assert m["hit_iters_match"] >= 0.999 and m["depth_rel_le_1e-9"] >= 0.999, m


def test_gi_fp64(renderer, oracle):
    sc, cam, p = configs.hybrid_gi_2160p(48, 27, spp=2)
    g, gs = gpu_frame(renderer, sc, cam, p, abi.ENGINE_PLAIN_FP64_STRICT)
    o, os_ = oracle.render(sc, cam, p)
    m = compare(g, o)
    print(m, gs, os_)
    assert m["hit_mismatch"] <= 0.01, m
    diff = np.abs(g["rgb"] - o["rgb"])
    assert np.mean(diff < 1e-3) >= 0.98, float(np.mean(diff < 1e-3))


def test_distance_strict_bit_exact_box_menger(renderer, oracle):
    rng = np.random.default_rng(11)
    pts = rng.uniform(-3, 3, size=(20000, 3))
    for sc in (configs.mandelbox_scene(), configs.menger_scene()):
        renderer.set_scene(sc)
        d, it = renderer.distance(torch.from_numpy(pts).cuda(), 1e-3, False, abi.ENGINE_PLAIN_FP64_STRICT)
        od, oit = oracle.distance(sc, pts, 1e-3, False)
        assert np.array_equal(it.cpu().numpy(), oit)
        assert np.array_equal(d.cpu().numpy(), od)


def test_distance_bulb_fp64(renderer, oracle):
    rng = np.random.default_rng(12)
    pts = rng.uniform(-1.5, 1.5, size=(20000, 3))
    sc = configs.mandelbulb_scene()
    renderer.set_scene(sc)
    d, it = renderer.distance(torch.from_numpy(pts).cuda(), 1e-3, False, abi.ENGINE_PLAIN_FP64_STRICT)
    od, oit = oracle.distance(sc, pts, 1e-3, False)
    assert np.mean(it.cpu().numpy() == oit) >= 0.999
    d = d.cpu().numpy()
    # escaping orbits only: a bounded (interior) orbit is chaotic over 250
    # iterations, so last-ulp differences of the transcendentals grow there
    ok = (oit == it.cpu().numpy()) & (oit <= sc.formula_maxiter)
    # near-surface points have tiny, cancellation-dominated estimates: an
    # absolute floor of 1e-12 (well below any threshold used) covers them
    close = np.abs(d[ok] - od[ok]) <= 1e-9 * np.abs(od[ok]) + 1e-12
    assert np.mean(close) >= 0.999


def test_mixed_precision_error_metrics(renderer, oracle):
    sc, cam, p = configs.mandelbox_1080p("A", 192, 108)
    g, _ = gpu_frame(renderer, sc, cam, p, abi.ENGINE_PLAIN_MIXED)
    o, _ = oracle.render(sc, cam, p)
    m = compare(g, o)
    print("mixed", m)
    assert m["hit_mismatch"] <= 0.001, m
    assert m["depth_rel_median"] <= 1e-4 and m["depth_rel_le_1e-4"] >= 0.99, m


def test_invalid_arguments_fail_loudly(renderer):
    from mandelbulber2_b200.render import MbrError

    sc, cam, p = configs.mandelbulb_512(16, 16)
    renderer.set_scene(sc)
    cam.width = 0
    with pytest.raises(MbrError):
        renderer.render(cam, p)
    cam.width = 16
    p.detail_level = 0.0
    with pytest.raises(MbrError):
        renderer.render(cam, p)
