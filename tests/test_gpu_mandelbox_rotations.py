"""The Mandelbox with rotations (fractal_mandelbox.cpp:33-63: the box fold in
rotated frames; :103: the main rotation) on every engine, against the oracle,
whose rotated Mandelbox step equals the reference's bit for bit
(tests/golden/formula_kat.json).  The strict FP64 kernel performs the
oracle's IEEE operations and is held to bit-exactness; the other engines to
the usual FP64 and FP32 bars.
"""
import numpy as np
import pytest
import torch

from mandelbulber2_b200 import abi, configs

from .parity import compare

pytestmark = pytest.mark.gpu
NAMES = ("depth", "iters", "hit", "normal", "ao", "rgb8")
NEG = [[10.0, 0.0, -5.0], [0.0, 25.0, 0.0], [-15.0, 5.0, 30.0]]
POS = [[0.0, -20.0, 0.0], [12.0, 0.0, 7.0], [0.0, 0.0, 0.0]]
MAIN = [3.0, -17.0, 41.0]


def rotated(mode, width=192, height=108):
    sc, cam, p = configs.mandelbox_1080p("A", width, height, ao_rays=4)
    f = sc.fractal[0]
    if mode in ("folds", "both"):
        f.mandelbox_rotations_enabled = 1
        for a in range(3):
            f.mandelbox_rotation_neg[a][:] = NEG[a]
            f.mandelbox_rotation_pos[a][:] = POS[a]
    if mode in ("main", "both"):
        f.mandelbox_main_rotation_enabled = 1
        f.mandelbox_rotation_main[:] = MAIN
    return sc, cam, p


@pytest.mark.parametrize("mode", ["folds", "main", "both"])
def test_rotated_mandelbox_vs_oracle(renderer, oracle, mode):
    sc, cam, p = rotated(mode)
    renderer.set_scene(sc)
    o, ost = oracle.render(sc, cam, p)
    assert 0.05 < float(np.mean(o["hit"])) < 0.99
    for engine in (abi.ENGINE_PLAIN_FP64_STRICT, abi.ENGINE_PLAIN_FP64, abi.ENGINE_PLAIN_MIXED,
                   abi.ENGINE_WAVEFRONT_FP32, abi.ENGINE_WAVEFRONT_FP64, abi.ENGINE_WAVEFRONT_AUTO):
        fr = renderer.render(cam, p, engine, outputs=NAMES)
        g = {k: v.cpu().numpy() for k, v in fr.buffers.items()}
        m = compare(g, o)
        print(mode, abi.ENGINE_NAMES[engine], m)
        if engine == abi.ENGINE_PLAIN_FP64_STRICT:
            for k in NAMES:
                assert np.array_equal(g[k], o[k]), (mode, k)
            assert fr.stats == ost
        elif engine in (abi.ENGINE_PLAIN_FP64, abi.ENGINE_WAVEFRONT_FP64):
            assert m["hit_iters_match"] >= 0.999, m
            assert m["depth_rel_le_1e-9"] >= 0.999, m
        else:
            assert m["hit_mismatch"] <= 0.005, m
            assert m["depth_rel_median"] <= 1e-4, m


def test_rotated_distance_strict_bit_exact(renderer, oracle):
    sc, _, _ = rotated("both")
    renderer.set_scene(sc)
    pts = np.random.default_rng(21).uniform(-3, 3, size=(20000, 3))
    d, it = renderer.distance(torch.from_numpy(pts).cuda(), 1e-3, False, abi.ENGINE_PLAIN_FP64_STRICT)
    od, oit = oracle.distance(sc, pts, 1e-3, False)
    assert np.array_equal(it.cpu().numpy(), oit)
    assert np.array_equal(d.cpu().numpy(), od)


def test_rotations_with_two_mandelbox_slots_are_refused(renderer):
    """The scene carries one Mandelbox rotation block: a hybrid whose one
    Mandelbox slot is rotated is accepted, one with two Mandelbox slots and
    rotations is refused."""
    from mandelbulber2_b200.render import MbrError

    sc = configs.hybrid_scene()
    sc.fractal[0] = configs.mandelbox_scene().fractal[0]
    sc.fractal[0].formula_iterations = 2
    sc.fractal[0].mandelbox_main_rotation_enabled = 1
    sc.fractal[0].mandelbox_rotation_main[:] = MAIN
    renderer.set_scene(sc)
    sc.fractal[1] = configs.mandelbox_scene().fractal[0]
    with pytest.raises(MbrError) as e:
        renderer.set_scene(sc)
    assert e.value.status == abi.MBR_EUNSUPPORTED
