"""Explicit objects trees on the plain engines through the C-ABI against the
oracle, whose tree walk equals the reference's own CalculateDistance and
render worker on these scenes (tests/golden/pipeline_kat.json,
render_kat.json): fractal nodes with their own transform, iteration limit,
julia and constant factor; primitive nodes under the accumulated transform;
union, smooth union, intersection and subtraction groups; repeat and detail
multiplier; a disabled subtree.

Trees of Mandelbox and IEEE-only primitives are bit-identical on the strict
FP64 engine (distances, iteration sums, every frame buffer and the counters).
Elsewhere (a Mandelbulb's asin, atan2 and pow from CUDA's libm against the
host's, a torus's pow, the FMA engine's contractions) distances are compared
at the points more than 10 detail sizes from every surface, where no orbit
in the fractals' interior (chaotic: an ulp decides the result on either
side) reaches the result: FP64 engines within 1e-8 relative on >= 99.9 % of
them with iteration sums equal on >= 99.9 %, the mixed engine median
relative error <= 1e-4 and iteration sums equal on >= 95 %.  Frames: FP64
engines hit/iteration agreement >= 99.9 % and depth within 1e-9 on >= 99.9 %
of common hits; the mixed engine hit mismatch <= 0.5 % and median depth
error <= 1e-4.  The
wavefront engines and the adjoint refuse trees.
"""
import numpy as np
import pytest
import torch

from mandelbulber2_b200 import abi, configs
from mandelbulber2_b200.render import MbrError
from tests.golden.pipeline_cases import _trees

from .parity import compare

pytestmark = pytest.mark.gpu
NAMES = ("depth", "iters", "hit", "normal", "ao", "rgb8")
EXACT = {"tree_intersection", "tree_disabled_branch"}
CAMERAS = {"tree_two_fractals": (0.0, -3.0, 0.3), "tree_intersection": (0.3, -3.5, 1.2),
           "tree_subtraction": (0.0, -3.0, 0.3), "tree_smooth_nested": (1.0, -10.0, 2.0),
           "tree_repeat_detail": (0.0, -4.0, 0.5), "tree_disabled_branch": (0.0, -8.0, 1.0)}
# half the edge of the cube the distance points are drawn from: the julia
# Mandelbox of the nested tree and the full-size Mandelbox reach further out
EXTENT = {"tree_smooth_nested": 8.0, "tree_disabled_branch": 6.0}


def _rel(a, b):
    return np.abs(a - b) / np.maximum(np.abs(b), 1e-300)


@pytest.mark.parametrize("case", sorted(CAMERAS))
def test_tree_distances(renderer, oracle, case):
    sc = _trees()[case]
    renderer.set_scene(sc)
    r = EXTENT.get(case, 2.5)
    pts = np.random.default_rng(21).uniform(-r, r, size=(8192, 3))
    for det in (1e-3, 0.05):
        for nm in (False, True):
            od, oit = oracle.distance(sc, pts, det, nm)
            for engine in (abi.ENGINE_PLAIN_FP64_STRICT, abi.ENGINE_PLAIN_FP64, abi.ENGINE_PLAIN_MIXED):
                d, it = renderer.distance(torch.from_numpy(pts), det, nm, engine)
                d, it = d.cpu().numpy(), it.cpu().numpy()
                rel = _rel(d, od)
                far = od > 10.0 * det  # no leaf within reach is an interior (chaotic) orbit
                print(case, det, nm, abi.ENGINE_NAMES[engine], "far", int(far.sum()), "rel<=1e-8 (far)",
                      np.mean(rel[far] <= 1e-8), "median", np.median(rel[far]), "iters (far)",
                      np.mean(it[far] == oit[far]), "all points rel<=1e-8", np.mean(rel <= 1e-8))
                if engine == abi.ENGINE_PLAIN_FP64_STRICT and case in EXACT:
                    assert np.array_equal(d, od) and np.array_equal(it, oit), (case, det, nm)
                    continue
                assert far.sum() >= 1000
                if engine != abi.ENGINE_PLAIN_MIXED:
                    assert np.mean(rel[far] <= 1e-8) >= 0.999, (case, det, nm, engine)
                    assert np.mean(it[far] == oit[far]) >= 0.999, (case, det, nm, engine)
                else:
                    assert np.median(rel[far]) <= 1e-4 and np.mean(it[far] == oit[far]) >= 0.95, (case, det, nm)


@pytest.mark.parametrize("case", sorted(CAMERAS))
def test_tree_frames(renderer, oracle, case):
    sc = _trees()[case]
    cam = configs.camera(CAMERAS[case], width=64, height=40)
    p = configs.base_params(5, 20.0)
    p.ao_rays = 4
    p.soft_shadow_cone = 15.0
    o, ost = oracle.render(sc, cam, p)
    assert 0.05 < float(np.mean(o["hit"])) < 0.98, float(np.mean(o["hit"]))
    renderer.set_scene(sc)
    for engine in (abi.ENGINE_PLAIN_FP64_STRICT, abi.ENGINE_PLAIN_FP64, abi.ENGINE_PLAIN_MIXED):
        fr = renderer.render(cam, p, engine, outputs=NAMES)
        g = {k: v.cpu().numpy() for k, v in fr.buffers.items()}
        m = compare(g, o)
        print(case, abi.ENGINE_NAMES[engine], m)
        if engine == abi.ENGINE_PLAIN_FP64_STRICT and case in EXACT:
            for k in NAMES:
                assert np.array_equal(g[k], o[k]), (case, k)
            assert fr.stats == ost
        elif engine != abi.ENGINE_PLAIN_MIXED:
            assert m["hit_iters_match"] >= 0.999 and m["depth_rel_le_1e-9"] >= 0.999, (case, engine, m)
        else:
            assert m["hit_mismatch"] <= 0.005 and m["depth_rel_median"] <= 1e-4, (case, m)
    for engine in (abi.ENGINE_WAVEFRONT_FP32, abi.ENGINE_WAVEFRONT_FP64, abi.ENGINE_WAVEFRONT_AUTO):
        with pytest.raises(MbrError) as e:
            renderer.render(cam, p, engine)
        assert e.value.status == abi.MBR_EUNSUPPORTED


def test_tree_node_transform_on_the_gpu(renderer):
    """A fractal node scaled by s at t: its distance at t + s p equals s times
    the plain fractal's at p with the detail size divided by s, iteration
    counts identical (strict FP64 engine, Mandelbox: IEEE operations only;
    s = 0.5 keeps every product exact)."""
    from tests.golden.pipeline_cases import _node

    sc = configs.mandelbox_scene(-1.5, 0.5, 30)
    pts = np.random.default_rng(22).uniform(-2.0, 2.0, size=(4096, 3))
    renderer.set_scene(sc)
    d0, i0 = renderer.distance(torch.from_numpy(pts), 2e-3, False, abi.ENGINE_PLAIN_FP64_STRICT)
    s, t = 0.5, np.array([0.25, -0.5, 1.0])
    tree = abi.Scene.from_buffer_copy(sc)
    tree.n_nodes = 1
    tree.node[0] = _node(abi.NODE_FRACTAL, 0, 0, pos=tuple(t), scale=s, formula_maxiter=30)
    renderer.set_scene(tree)
    d1, i1 = renderer.distance(torch.from_numpy(t + s * pts), 1e-3, False, abi.ENGINE_PLAIN_FP64_STRICT)
    assert torch.equal(i0, i1)
    np.testing.assert_allclose(d1.cpu().numpy(), s * d0.cpu().numpy(), rtol=1e-12, atol=1e-15)
