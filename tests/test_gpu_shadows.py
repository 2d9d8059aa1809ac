"""The main light's soft and penetrating shadows (AuxShadow,
shader_aux_shadow.cpp:55-77, 142-151, 266-301; the penetrating march length,
light.cpp:277-290) - the reference's defaults are a 1 degree soft cone and a
penetrating light - on every engine against the oracle.  On the Mandelbox
(only IEEE operations; the cone's tangent is taken on the host) the strict
FP64 kernel is held to bit-exactness; on the Mandelbulb, where each mode
changes the shading of a sixth to a quarter of the hits, the engines are
held to the FP64 and FP32 bars with the 8-bit image within 35 dB.
"""
import numpy as np
import pytest

from mandelbulber2_b200 import abi, configs

from .parity import compare

pytestmark = pytest.mark.gpu
NAMES = ("depth", "iters", "hit", "normal", "shade", "rgb8")


@pytest.mark.parametrize("cone,pen", [(1.0, 1), (10.0, 0), (0.0, 1)])
def test_shadow_modes_vs_oracle(renderer, oracle, cone, pen):
    sc, cam, p = configs.mandelbulb_512(128, 128)
    hard = p.__class__.from_buffer_copy(p)
    p.soft_shadow_cone = cone
    p.penetrating = pen
    renderer.set_scene(sc)
    o, ost = oracle.render(sc, cam, p)
    oh, _ = oracle.render(sc, cam, hard)
    both = o["hit"].astype(bool)
    assert np.mean(np.abs(o["shade"][both] - oh["shade"][both]) > 1e-6) > 0.1, "the mode changes the shading"
    for engine in (abi.ENGINE_PLAIN_FP64_STRICT, abi.ENGINE_PLAIN_FP64, abi.ENGINE_WAVEFRONT_FP32,
                   abi.ENGINE_WAVEFRONT_FP64):
        fr = renderer.render(cam, p, engine, outputs=NAMES)
        g = {k: v.cpu().numpy() for k, v in fr.buffers.items()}
        m = compare(g, o)
        print(cone, pen, abi.ENGINE_NAMES[engine], m)
        if engine in (abi.ENGINE_PLAIN_FP64_STRICT, abi.ENGINE_PLAIN_FP64, abi.ENGINE_WAVEFRONT_FP64):
            assert m["hit_iters_match"] >= 0.999, m
        else:
            assert m["hit_mismatch"] <= 0.005, m
        assert m["psnr"] >= 35.0, m


def test_soft_penetrating_shadow_strict_bit_exact(renderer, oracle):
    sc, cam, p = configs.mandelbox_1080p("A", 160, 90, ao_rays=0)
    p.soft_shadow_cone = 20.0
    p.penetrating = 1
    renderer.set_scene(sc)
    o, ost = oracle.render(sc, cam, p)
    fr = renderer.render(cam, p, abi.ENGINE_PLAIN_FP64_STRICT, outputs=NAMES)
    g = {k: v.cpu().numpy() for k, v in fr.buffers.items()}
    for k in NAMES:
        assert np.array_equal(g[k], o[k]), k
    assert fr.stats == ost
