"""Primitives joined to the fractal by union, on the CPU: the oracle's
primitive distances (src/primitive.cpp) against closed forms, through the
node transform of the objects tree (position, rotation in degrees, scale,
repeat; src/objects_tree.cpp:290-385, calculate_distance.cpp:268-282)."""
import math

import numpy as np
import pytest

from mandelbulber2_b200 import abi


def far_bulb():
    """A Mandelbulb whose distance is 10 (the clamp) at the test points."""
    sc = abi.scene_defaults(abi.FORMULA_MANDELBULB)
    sc.formula_maxiter = 20
    return sc


def with_prims(*prims):
    sc = far_bulb()
    sc.n_primitives = len(prims)
    for i, q in enumerate(prims):
        sc.primitive[i] = q
    return sc


def prim(kind, **kw):
    q = abi.primitive_defaults(kind)
    for k, v in kw.items():
        if isinstance(v, (list, tuple)):
            getattr(q, k)[:] = v
        else:
            setattr(q, k, v)
    return q


def dist(oracle, sc, pts):
    d, _ = oracle.distance(sc, np.asarray(pts, dtype=np.float64), 1e-4, False)
    return d


def test_defaults():
    q = abi.primitive_defaults(abi.PRIMITIVE_BOX)
    assert list(q.size) == [1.0, 1.0, 1.0] and q.rounding == 1e-15 and q.scale == 1.0
    assert list(q.limits_max) == [0.7, 0.7, 0.7] and q.caps == 1
    w = abi.primitive_defaults(abi.PRIMITIVE_WATER)
    assert w.relative_amplitude == 0.2 and w.length == 0.1 and w.iterations == 5


def test_plane_sphere_box_closed_forms(oracle):
    sc = with_prims(prim(abi.PRIMITIVE_PLANE, position=[0, 0, -6]),
                    prim(abi.PRIMITIVE_SPHERE, position=[0, 0, 20], radius=2.0),
                    prim(abi.PRIMITIVE_BOX, position=[20, 0, 0], size=[2, 4, 6], rounding=0.0))
    pts = [[30, 30, -3], [0, 0, 25], [20, 0, 7], [25, 0, 0], [20, 3, 0]]
    want = [3.0, 3.0, 4.0, 4.0, 1.0]
    np.testing.assert_allclose(dist(oracle, sc, pts), want, rtol=0, atol=1e-12)
    # far from everything: the fractal's clamp
    assert dist(oracle, sc, [[0, 60, 10]])[0] == 10.0


def test_rotation_and_scale(oracle):
    # a box long in x, rotated 90 degrees about z: long in y
    sc = with_prims(prim(abi.PRIMITIVE_BOX, position=[0, 30, 0], size=[8, 1, 1], rotation=[0, 0, 90], rounding=0.0))
    d = dist(oracle, sc, [[0, 30 + 4 + 1.5, 0], [4 + 1.5, 30, 0]])
    np.testing.assert_allclose(d, [1.5, 5.0], rtol=0, atol=1e-12)
    # scale 2 doubles the sphere
    sc = with_prims(prim(abi.PRIMITIVE_SPHERE, position=[0, 0, 30], radius=1.0, scale=2.0))
    np.testing.assert_allclose(dist(oracle, sc, [[0, 0, 35]]), [3.0], rtol=0, atol=1e-12)


def test_repeat_tiles_the_primitive(oracle):
    sc = with_prims(prim(abi.PRIMITIVE_SPHERE, position=[0, 0, 30], radius=1.0, repeat=[10, 0, 0]))
    d = dist(oracle, sc, [[0, 0, 32], [10, 0, 32], [-40, 0, 32], [5, 0, 30]])
    np.testing.assert_allclose(d, [1.0, 1.0, 1.0, 4.0], rtol=0, atol=1e-12)


def test_empty_wall_and_limits(oracle):
    sc = with_prims(prim(abi.PRIMITIVE_SPHERE, position=[0, 0, 30], radius=4.0, empty=1, wall_thickness=0.5))
    d = dist(oracle, sc, [[0, 0, 30], [0, 0, 36]])
    np.testing.assert_allclose(d, [3.5, 1.5], rtol=0, atol=1e-12)
    sc = with_prims(prim(abi.PRIMITIVE_SPHERE, position=[0, 0, 30], radius=4.0, limits_enable=1,
                         limits_min=[-10, -10, 0], limits_max=[10, 10, 10]))
    d = dist(oracle, sc, [[0, 0, 24], [0, 0, 35]])  # below the limits box: its distance; above: the sphere's
    np.testing.assert_allclose(d, [6.0, 1.0], rtol=0, atol=1e-12)


def test_flat_and_round_shapes(oracle):
    sc = with_prims(prim(abi.PRIMITIVE_CYLINDER, position=[0, 0, 30], radius=1.0, height=4.0),
                    prim(abi.PRIMITIVE_CIRCLE, position=[30, 0, 0], radius=1.0),
                    prim(abi.PRIMITIVE_RECTANGLE, position=[-30, 0, 0], width=2.0, height=2.0),
                    prim(abi.PRIMITIVE_TORUS, position=[0, -30, 0], radius=2.0, tube_radius=0.5))
    d = dist(oracle, sc, [[3, 0, 30], [0, 0, 34], [30, 0, 2], [-30, 0, -3], [0, -30, 1.5], [2, -30, 0]])
    np.testing.assert_allclose(d, [2.0, 2.0, 2.0, 3.0, math.hypot(2.0, 1.5) - 0.5, 0.0], rtol=0, atol=1e-9)


def test_cone_prism_ellipsoid(oracle):
    sc = with_prims(prim(abi.PRIMITIVE_CONE, position=[0, 0, 30], radius=1.0, height=2.0),
                    prim(abi.PRIMITIVE_PRISM, position=[30, 0, 0], prism_angle=60.0, triangle_height=1.0, height=1.0),
                    prim(abi.PRIMITIVE_ELLIPSOID, position=[-30, 0, 0], size=[2, 1, 1]))
    d = dist(oracle, sc, [[0, 0, 35], [0, 0, 29], [30, 0, 3], [30, -2, 0], [-27, 0, 0]])
    # above the apex: the distance to the wall's plane; below: to the base
    np.testing.assert_allclose(d, [3 / math.sqrt(5), 1.0, 2.5, 2.0, 1.0], rtol=0, atol=1e-7)
    cone = prim(abi.PRIMITIVE_CONE)
    assert cone.radius == 1.0 and cone.height == 1.0 and cone.caps == 1
    e = abi.primitive_defaults(abi.PRIMITIVE_ELLIPSOID)
    assert list(e.size) == [1.0, 0.5, 0.5] and list(e.limits_max) == [1.4, 0.7, 0.7]
    p = abi.primitive_defaults(abi.PRIMITIVE_PRISM)
    assert p.prism_angle == 60.0 and p.triangle_height == 1.0


def test_water_is_a_wavy_plane(oracle):
    sc = with_prims(prim(abi.PRIMITIVE_WATER, position=[0, 0, -2], length=0.5, relative_amplitude=0.2))
    rng = np.random.default_rng(3)
    pts = np.c_[rng.uniform(40, 50, (200, 2)), np.full(200, -1.5)]  # far from the fractal
    d = dist(oracle, sc, pts)
    # 0.5 above the plane, moved by the waves (a few amplitudes of 0.1)
    assert np.all((d > 0.05) & (d < 0.95)) and np.std(d) > 0.01
    # above 10 amplitudes (1.0) the waves are not evaluated: the plane's distance
    assert dist(oracle, sc, [[45, 45, 5]])[0] == 7.0


def test_invalid_primitives_are_refused(oracle):
    with pytest.raises(RuntimeError):
        oracle.distance(with_prims(prim(99)), np.zeros((1, 3)), 1e-3, False)
