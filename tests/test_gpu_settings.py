"""Scenes read from settings files (.fract), rendered through the C-ABI and
held to the same bars as the hand-built scenes against the oracle: the plain
FP64 kernel to the FP64 bar, the FP32 and auto-precision wavefront engines to
the FP32 bar (hit mismatch <= 0.5 %, median depth error <= 1e-4)."""
import os

import numpy as np
import pytest

from mandelbulber2_b200 import abi, settings

from .parity import compare

pytestmark = pytest.mark.gpu
FIX = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "settings")
NAMES = ("depth", "iters", "hit", "normal", "ao", "rgb8")


@pytest.mark.parametrize("name", ["box_ao.fract", "hybrid_bulb_menger.fract", "legacy_light.fract",
                                  "box_primitives.fract"])
def test_settings_scene_vs_oracle(renderer, oracle, name):
    s = settings.load_from_file(os.path.join(FIX, name))
    assert s.ok, s.report
    sc, cam, p = s.scene, s.camera, s.params
    renderer.set_scene(sc)
    o, ost = oracle.render(sc, cam, p)
    for engine in (abi.ENGINE_PLAIN_FP64, abi.ENGINE_WAVEFRONT_FP32, abi.ENGINE_WAVEFRONT_AUTO):
        fr = renderer.render(cam, p, engine, outputs=NAMES)
        g = {k: v.cpu().numpy() for k, v in fr.buffers.items()}
        m = compare(g, o)
        print(name, abi.ENGINE_NAMES[engine], m)
        assert fr.stats["pixels"] == cam.width * cam.height
        assert 0.02 < float(np.mean(o["hit"])), "the scene's fractal is in view"
        if engine == abi.ENGINE_PLAIN_FP64:
            assert m["hit_iters_match"] >= 0.999, m
            assert m["depth_rel_le_1e-9"] >= 0.999, m
        else:
            assert m["hit_mismatch"] <= 0.005, m
            assert m["depth_rel_median"] <= 1e-4, m


@pytest.mark.parametrize("name", ["box_transform.fract", "pseudo_kleinian.fract"])
def test_settings_tree_and_keyed_formula_scenes(renderer, oracle, name):
    """A file whose fractal carries a formula and fractal transform (read as
    an explicit objects tree) and a pseudo-Kleinian file (parameters by
    settings key), on the plain engines: strict FP64 bit-exact against the
    oracle, FP64 and mixed to their bars; the wavefront refuses both."""
    from mandelbulber2_b200.render import MbrError

    s = settings.load_from_file(os.path.join(FIX, name))
    assert s.ok, s.report
    sc, cam, p = s.scene, s.camera, s.params
    renderer.set_scene(sc)
    o, ost = oracle.render(sc, cam, p)
    assert 0.02 < float(np.mean(o["hit"])), "the scene's fractal is in view"
    for engine in (abi.ENGINE_PLAIN_FP64_STRICT, abi.ENGINE_PLAIN_FP64, abi.ENGINE_PLAIN_MIXED):
        fr = renderer.render(cam, p, engine, outputs=NAMES)
        g = {k: v.cpu().numpy() for k, v in fr.buffers.items()}
        m = compare(g, o)
        print(name, abi.ENGINE_NAMES[engine], m)
        if engine == abi.ENGINE_PLAIN_FP64_STRICT:
            for k in NAMES:
                assert np.array_equal(g[k], o[k]), (name, k)
            assert fr.stats == ost
        elif engine == abi.ENGINE_PLAIN_FP64:
            assert m["hit_iters_match"] >= 0.999 and m["depth_rel_le_1e-9"] >= 0.999, m
        else:
            assert m["hit_mismatch"] <= 0.005 and m["depth_rel_median"] <= 1e-4, m
    with pytest.raises(MbrError) as e:
        renderer.render(cam, p, abi.ENGINE_WAVEFRONT_FP32)
    assert e.value.status == abi.MBR_EUNSUPPORTED
