"""The oracle pinned against the reference's own sources for the whole path.

tests/golden/pipeline_kat.json and render_kat.json were produced by the
reference's compiled sources (oracle/_ref/librefpipe.so: parameter
containers with the reference's defaults, objects tree, hybrid sequences,
Compute, CalculateDistance, cRenderWorker::doWork with its shaders, cImage;
tests/golden/make_golden.py).  The oracle's restatement must reproduce them
bit for bit:

- CalculateDistance (distance and iteration count) of 22 scene variants at
  seeded points, both normal-calculation modes, two detail sizes, and each
  scene's hybrid sequence table;
- whole frames of the render worker: the z-buffer (the depth as float), the
  hit mask, the world normals and the main light's shadow factor, with the
  march jitter drawn from the reference's global Park-Miller stream (the
  oracle's jitter mode 2).

Where the reference was compiled here, the same comparisons also run live on
fresh random points.
"""
import base64
import json
import os
import zlib

import numpy as np
import pytest

from tests.golden.pipeline_cases import cases, render_cases

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def load(name):
    with open(os.path.join(GOLDEN, name)) as f:
        return json.load(f)


def fh(v):
    flat = [x for row in v for x in row] if v and isinstance(v[0], list) else v
    return np.array([float.fromhex(x) for x in flat])


def unpack(s):
    return np.frombuffer(zlib.decompress(base64.b64decode(s)), dtype="<f4")


CASES = cases()
PIPE = load("pipeline_kat.json")
RENDER = load("render_kat.json")


@pytest.mark.parametrize("name", sorted(PIPE))
def test_calculate_distance_equals_the_reference(oracle, name):
    kat = PIPE[name]
    sc = CASES[name]
    pts = fh(kat["points"]).reshape(-1, 3)
    for run in kat["runs"]:
        d, it = oracle.distance(sc, pts, float.fromhex(run["detail"]), bool(run["normal_mode"]))
        assert np.array_equal(d, fh(run["dist"]), equal_nan=True), (name, run["normal_mode"], run["detail"])
        assert it.tolist() == run["iters"], (name, run["normal_mode"])


@pytest.mark.parametrize("name", sorted(PIPE))
def test_sequence_equals_the_reference(oracle, name):
    ref = PIPE[name]["sequence"]
    seq, length, _, bail = oracle.sequence(CASES[name])
    assert length == ref["length"] and seq == ref["seq"], name
    assert bail[: len(ref["bailout"])] == ref["bailout"], name


RENDERS = {n: (sc, cam, p) for n, sc, cam, p in render_cases()}


@pytest.mark.parametrize("name", sorted(RENDER))
def test_render_equals_the_reference_render_worker(oracle, name):
    kat = RENDER[name]
    sc, cam, p = RENDERS[name]
    p.jitter = 2  # the reference's global Park-Miller stream, pixel order
    p.seed = kat["seed"]
    p.light_direction[:] = [float.fromhex(x) for x in kat["light"]]
    out, _ = oracle.render(sc, cam, p, outputs=("depth", "hit", "normal", "shade", "shadow"))
    z = unpack(kat["zbuffer"])
    hit = z < 1e19
    assert hit.mean() > 0.05
    assert np.array_equal(hit, out["hit"] > 0), name
    zo = np.where(out["hit"] > 0, out["depth"], 1e20).astype(np.float32)
    assert np.array_equal(z, zo), name
    nw = unpack(kat["normal_world"]).reshape(-1, 3)
    assert np.array_equal(nw[hit], out["normal"][hit]), name
    # the shadow factor where the surface faces the light (LightShading runs
    # AuxShadow there, shader_light_shading.cpp:90-98)
    lit = hit & (out["shade"] > 0.001)
    assert np.array_equal(unpack(kat["shadow"])[lit], out["shadow"][lit]), name


def _live():
    from oracle.refpipe import available

    return available()


@pytest.mark.skipif(not _live(), reason="the reference's sources were not compiled here (oracle/_ref)")
def test_live_random_points_equal_the_reference(oracle):
    from oracle.refpipe import RefPipeline

    rng = np.random.default_rng()
    for name, sc in CASES.items():
        r = RefPipeline()
        r.configure(sc)
        pts = rng.uniform(-2.5, 2.5, size=(200, 3))
        for nm in (False, True):
            d_ref, it_ref = r.distance(pts, 1e-3, nm)
            d, it = oracle.distance(sc, pts, 1e-3, nm)
            assert np.array_equal(d, d_ref, equal_nan=True), name
            assert np.array_equal(it, it_ref), name
        r.close()
