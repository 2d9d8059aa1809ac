"""Primitives joined to the fractal by union (the objects-tree walk,
calculate_distance.cpp:225-516; primitive.cpp) on every engine against the
oracle.  Plane, box, sphere (with a limits box), repeated cylinder, circle and
rectangle use only IEEE operations, and the node transforms are built on the
host, so the strict FP64 kernel is held to bit-exactness, counts included;
the water and the torus (sin, cos, pow) are held to the FP64 and FP32 bars.
"""
import numpy as np
import pytest
import torch

from mandelbulber2_b200 import abi, configs

from .parity import compare

pytestmark = pytest.mark.gpu
NAMES = ("depth", "iters", "hit", "normal", "ao", "rgb8")
ENGINES = (abi.ENGINE_PLAIN_FP64_STRICT, abi.ENGINE_PLAIN_FP64, abi.ENGINE_PLAIN_MIXED, abi.ENGINE_WAVEFRONT_FP32,
           abi.ENGINE_WAVEFRONT_AUTO)


def prim(kind, **kw):
    q = abi.primitive_defaults(kind)
    for k, v in kw.items():
        if isinstance(v, (list, tuple)):
            getattr(q, k)[:] = v
        else:
            setattr(q, k, v)
    return q


def scene_with(prims, width=160, height=90):
    sc, cam, p = configs.mandelbox_1080p("A", width, height, ao_rays=4)
    sc.n_primitives = len(prims)
    for i, q in enumerate(prims):
        sc.primitive[i] = q
    return sc, cam, p


def ieee_prims():
    return [prim(abi.PRIMITIVE_PLANE, position=[0, 0, -2.2], rotation=[6, -4, 0]),
            prim(abi.PRIMITIVE_BOX, position=[2.4, -1.0, 0.8], size=[0.8, 1.2, 0.6], rotation=[10, 0, 35],
                 rounding=0.05),
            prim(abi.PRIMITIVE_SPHERE, position=[-2.3, -0.8, 0.9], radius=0.7, limits_enable=1,
                 limits_min=[-1, -1, -0.3], limits_max=[1, 1, 1]),
            prim(abi.PRIMITIVE_CYLINDER, position=[0, -2.5, -1.6], radius=0.1, height=0.8, repeat=[1.8, 0, 0]),
            prim(abi.PRIMITIVE_CIRCLE, position=[-1.0, -2.2, 1.1], radius=0.35, rotation=[70, 0, 0]),
            prim(abi.PRIMITIVE_RECTANGLE, position=[1.2, -2.0, -1.1], width=0.6, height=0.4, rotation=[80, 0, 20])]


def check_engines(renderer, sc, cam, p, o, ost, strict_exact, name):
    for engine in ENGINES:
        fr = renderer.render(cam, p, engine, outputs=NAMES)
        g = {k: v.cpu().numpy() for k, v in fr.buffers.items()}
        m = compare(g, o)
        print(name, abi.ENGINE_NAMES[engine], m)
        if engine == abi.ENGINE_PLAIN_FP64_STRICT and strict_exact:
            for k in NAMES:
                assert np.array_equal(g[k], o[k]), k
            assert fr.stats == ost
        elif engine in (abi.ENGINE_PLAIN_FP64_STRICT, abi.ENGINE_PLAIN_FP64):
            assert m["hit_iters_match"] >= 0.999, m
            assert m["depth_rel_le_1e-9"] >= 0.999, m
        else:
            assert m["hit_mismatch"] <= 0.005, m
            assert m["depth_rel_median"] <= 1e-4, m


def test_ieee_primitives_vs_oracle(renderer, oracle):
    sc, cam, p = scene_with(ieee_prims())
    renderer.set_scene(sc)
    o, ost = oracle.render(sc, cam, p)
    base = abi.Scene.from_buffer_copy(sc)
    base.n_primitives = 0
    ob, _ = oracle.render(base, cam, p)
    assert float(np.mean(o["hit"])) > float(np.mean(ob["hit"])) + 0.1  # the plane and the objects are in view
    check_engines(renderer, sc, cam, p, o, ost, True, "ieee")


def test_cone_prism_ellipsoid_vs_oracle(renderer, oracle):
    """Cone and prism (host-built wall normals) and the ellipsoid (float
    k0, k1 as in the reference) use IEEE operations only: strict bit-exact."""
    sc, cam, p = scene_with([
        prim(abi.PRIMITIVE_PLANE, position=[0, 0, -2.2]),
        prim(abi.PRIMITIVE_CONE, position=[2.3, -1.2, -0.9], radius=0.5, height=1.0, rotation=[0, 10, 0]),
        prim(abi.PRIMITIVE_PRISM, position=[-2.3, -1.2, -0.6], prism_angle=70.0, triangle_height=0.8, height=0.6,
             rotation=[90, 0, 20]),
        prim(abi.PRIMITIVE_ELLIPSOID, position=[0.0, -2.4, 1.0], size=[0.6, 0.3, 0.3], rotation=[0, 0, 30])])
    renderer.set_scene(sc)
    o, ost = oracle.render(sc, cam, p)
    for k in range(1, 4):  # every object changes the frame
        s2 = abi.Scene.from_buffer_copy(sc)
        s2.primitive[k].position[:] = [0.0, 0.0, 100.0]  # moved out of view
        o2, _ = oracle.render(s2, cam, p)
        assert np.mean(np.abs(o2["depth"] - o["depth"]) > 1e-6) > 0.002, k
    check_engines(renderer, sc, cam, p, o, ost, True, "cone+prism+ellipsoid")


def test_water_and_torus_vs_oracle(renderer, oracle):
    sc, cam, p = scene_with([
        prim(abi.PRIMITIVE_WATER, position=[0, 0, -1.9], rotation=[0, 0, 15], length=0.4, relative_amplitude=0.25,
             iterations=4),
        prim(abi.PRIMITIVE_TORUS, position=[2.2, -1.2, 0.6], rotation=[70, 0, 0], radius=0.5, tube_radius=0.12)])
    renderer.set_scene(sc)
    o, ost = oracle.render(sc, cam, p)
    assert float(np.mean(o["hit"])) > 0.7
    check_engines(renderer, sc, cam, p, o, ost, False, "water+torus")


def test_primitive_distance_strict_bit_exact(renderer, oracle):
    sc, _, _ = scene_with(ieee_prims())
    renderer.set_scene(sc)
    pts = np.random.default_rng(5).uniform(-4, 4, size=(20000, 3))
    d, it = renderer.distance(torch.from_numpy(pts).cuda(), 1e-3, False, abi.ENGINE_PLAIN_FP64_STRICT)
    od, oit = oracle.distance(sc, pts, 1e-3, False)
    assert np.array_equal(it.cpu().numpy(), oit)
    assert np.array_equal(d.cpu().numpy(), od)
    assert np.mean(od < 9.999) > 0.5


def test_primitives_refused_where_not_built(renderer):
    from mandelbulber2_b200.render import MbrError

    sc, cam, p = scene_with(ieee_prims()[:1], 32, 18)
    renderer.set_scene(sc)
    with pytest.raises(MbrError) as e:
        renderer.render(cam, p, abi.ENGINE_WAVEFRONT_FP64, outputs=NAMES)
    assert e.value.status == abi.MBR_EUNSUPPORTED
    for field, kind, value in (("scale", abi.PRIMITIVE_PLANE, 0.0), ("height", abi.PRIMITIVE_CONE, 0.0)):
        bad = abi.Scene.from_buffer_copy(sc)
        bad.primitive[0] = prim(kind)
        setattr(bad.primitive[0], field, value)
        with pytest.raises(MbrError) as e:
            renderer.set_scene(bad)
        assert e.value.status == abi.MBR_EINVAL
