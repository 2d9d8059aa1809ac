"""Explicit objects trees (cObjectsTree, objects_tree.cpp:185-410; the walk
of CalculateDistanceFromObjectsTree, calculate_distance.cpp:225-516) on the
host: the library accepts every tree of the golden cases and refuses
malformed ones with the reference's shape rules, and the oracle's tree walk
reduces to the default objects tree where the two describe the same scene.
The oracle's tree distances and frames are pinned to the reference's own
compiled pipeline in tests/golden/pipeline_kat.json and render_kat.json.
"""
import numpy as np
import pytest

from mandelbulber2_b200 import abi, configs
from mandelbulber2_b200.render import MbrError, scene_sequence
from tests.golden.pipeline_cases import _node, _trees

F, P = abi.NODE_FRACTAL, abi.NODE_PRIMITIVE
ADD, MUL, SUB = abi.NODE_BOOLEAN_ADD, abi.NODE_BOOLEAN_MUL, abi.NODE_BOOLEAN_SUB


@pytest.mark.parametrize("name", sorted(_trees()))
def test_golden_trees_accepted(name):
    scene_sequence(_trees()[name])


def _with_nodes(nodes, base="tree_intersection"):
    s = abi.Scene.from_buffer_copy(_trees()[base])
    s.n_nodes = len(nodes)
    for i, n in enumerate(nodes):
        s.node[i] = n
    return s


def _bad_type():
    n = _node(F, 0, 0)
    n.type = 7
    return _with_nodes([n])


def _hybrid_tree():
    s = abi.Scene.from_buffer_copy(_trees()["tree_two_fractals"])
    s.hybrid_fractal_enable = 1
    return s


def _too_many():
    s = _with_nodes([_node(F, 0, 0)])
    s.n_nodes = abi.MBR_MAX_NODES + 1
    return s


@pytest.mark.parametrize("make,status", [
    (lambda: _with_nodes([_node(ADD), _node(F, 0, 2)]), abi.MBR_EINVAL),             # level jumps by two
    (lambda: _with_nodes([_node(F, 0, 1)]), abi.MBR_EINVAL),                         # first node below the top
    (lambda: _with_nodes([_node(F, 0, 0), _node(P, 0, 1)]), abi.MBR_EINVAL),         # a leaf with a child
    (lambda: _with_nodes([_node(F, 1, 0)]), abi.MBR_EINVAL),                         # fractal slot >= n_fractals
    (lambda: _with_nodes([_node(P, 1, 0)]), abi.MBR_EINVAL),                         # primitive >= n_primitives
    (_bad_type, abi.MBR_EINVAL),
    (lambda: _with_nodes([_node(MUL, enabled=0), _node(F, 0, 1)]), abi.MBR_EINVAL),  # nothing left to walk
    (lambda: _with_nodes([_node(F, 0, 0, formula_maxiter=0)]), abi.MBR_EINVAL),
    (lambda: _with_nodes([_node(ADD, scale=0.0), _node(F, 0, 1)]), abi.MBR_EINVAL),
    (lambda: _with_nodes([_node(F, 0, 0, pos=(float("nan"), 0.0, 0.0))]), abi.MBR_EINVAL),
    (lambda: _with_nodes([_node(F, 0, 0), _node(P, 0, 0, smooth_combine=1, smooth_combine_distance=0.0)]),
     abi.MBR_EINVAL),
    (_hybrid_tree, abi.MBR_EUNSUPPORTED),
    (_too_many, abi.MBR_EINVAL),
])
def test_malformed_trees_refused(make, status):
    with pytest.raises(MbrError) as e:
        scene_sequence(make())
    assert e.value.status == status


def test_disabled_subtree_is_skipped():
    """A disabled group drops its children: the tree equals the one without
    the subtree (objects_tree.cpp:185-245)."""
    scene_sequence(_with_nodes([_node(ADD), _node(F, 0, 1), _node(MUL, 0, 1, enabled=0), _node(F, 5, 2),
                                _node(P, 0, 1)]))


def test_oracle_tree_reduces_to_the_default_tree(oracle):
    """One fractal node at the identity, and that node beside a primitive in
    the root union, give the default objects tree's distances and iteration
    counts bit for bit (the default tree is the fractal node and the
    primitives joined by union, calculate_distance.cpp:166-201)."""
    pts = np.random.default_rng(3).uniform(-2.0, 2.0, size=(2000, 3))
    sc = configs.mandelbox_scene(-1.5, 0.5, 30)
    sc.n_primitives = 1
    sc.primitive[0] = abi.primitive_defaults(abi.PRIMITIVE_SPHERE)
    sc.primitive[0].radius = 0.7
    sc.primitive[0].position[:] = [1.0, 0.5, 0.0]
    for nodes in ([_node(F, 0, 0, formula_maxiter=30)],
                  [_node(F, 0, 0, formula_maxiter=30), _node(P, 0, 0)]):
        base = abi.Scene.from_buffer_copy(sc)
        base.n_primitives = len(nodes) - 1
        tree = abi.Scene.from_buffer_copy(base)
        tree.n_nodes = len(nodes)
        for i, n in enumerate(nodes):
            tree.node[i] = n
        for det, nm in ((1e-3, False), (0.05, True)):
            d0, i0 = oracle.distance(base, pts, det, nm)
            d1, i1 = oracle.distance(tree, pts, det, nm)
            assert np.array_equal(d0, d1) and np.array_equal(i0, i1), (len(nodes), det, nm)


def test_oracle_tree_transform_moves_the_object(oracle):
    """A node's position and scale move and scale its object: the distance of
    a fractal node scaled by s at t, at t + s p, is s times the plain
    fractal's distance at p with the detail size divided by s."""
    pts = np.random.default_rng(4).uniform(-2.0, 2.0, size=(1000, 3))
    sc = configs.mandelbox_scene(-1.5, 0.5, 30)
    s, t = 0.5, np.array([0.25, -0.5, 1.0])
    tree = abi.Scene.from_buffer_copy(sc)
    tree.n_nodes = 1
    tree.node[0] = _node(F, 0, 0, pos=tuple(t), scale=s, formula_maxiter=30)
    d0, i0 = oracle.distance(sc, pts, 2e-3, False)
    d1, i1 = oracle.distance(tree, t + s * pts, 1e-3, False)
    assert np.array_equal(i0, i1)
    np.testing.assert_allclose(d1, s * d0, rtol=1e-12, atol=1e-15)


def test_settings_transform_of_a_single_fractal_becomes_a_tree():
    """A legacy file's formula transform (formula_position_1, ..._rotation_1,
    ..._scale_1, ..._repeat_1; a non-default fractal_position / _rotation /
    repeat overrides them, settings.cpp:2372-2401) becomes the fractal node
    of an explicit tree, with the file's primitives beside it in the root
    union; a hybrid with a transform stays refused."""
    from mandelbulber2_b200 import settings

    head = "# Mandelbulber settings file\n# version 2.33\n# only modified parameters\n"
    txt = head + ("[main_parameters]\nformula_1 8;\nN 30;\nfractal_rotation 0 -90 0;\n"
                  "primitive_sphere_1_enabled true;\nprimitive_sphere_1_radius 0,5;\n"
                  "formula_position_1 0 0 1;\nformula_scale_1 0,5;\nformula_repeat_1 3 0 0;\n")
    s = settings.load_from_string(txt)
    assert s.ok, s.report
    sc = s.scene
    assert sc.n_nodes == 2 and sc.n_primitives == 1
    n = sc.node[0]
    assert n.type == abi.NODE_FRACTAL and n.level == 0 and n.formula_maxiter == 30
    assert list(n.position) == [0.0, 0.0, 1.0] and list(n.rotation) == [0.0, -90.0, 0.0]
    assert n.scale == 0.5 and list(n.repeat) == [3.0, 0.0, 0.0]
    assert sc.node[1].type == abi.NODE_PRIMITIVE and sc.node[1].index == 0
    scene_sequence(sc)
    s = settings.load_from_string(head + "[main_parameters]\nformula_1 8;\nformula_2 2;\nhybrid_fractal_enable true;\n"
                                  "fractal_position 1 0 0;\n")
    assert s.status == abi.MBR_EUNSUPPORTED


def test_settings_boolean_mode_becomes_a_tree():
    """The legacy boolean mode (boolean_operators): the slots with a formula
    combine left to right as nested groups (boolean_operator_K: 0
    intersection, 2 subtraction, else union; a missing operator takes
    boolean_operator_1's value), each fractal node with its own iteration
    limit (N before version 2.29) and julia settings; primitives join by
    union at the root."""
    from mandelbulber2_b200 import settings

    head = "# Mandelbulber settings file\n# version 2.26\n# only modified parameters\n"
    txt = head + ("[main_parameters]\nboolean_operators true;\nboolean_operator_1 2;\nN 20;\n"
                  "formula_1 8;\nformula_2 2;\nformula_3 7;\njulia_mode_2 true;\njulia_c_2 0,1 0,2 0,3;\n"
                  "formula_position_3 0 0 1;\nprimitive_plane_1_enabled true;\n")
    s = settings.load_from_string(txt)
    assert s.ok, s.report
    sc = s.scene
    kinds = [(sc.node[i].type, sc.node[i].level, sc.node[i].index) for i in range(sc.n_nodes)]
    SUB, ADD, F, P = abi.NODE_BOOLEAN_SUB, abi.NODE_BOOLEAN_ADD, abi.NODE_FRACTAL, abi.NODE_PRIMITIVE
    # root union with the plane; ((box - bulb) - menger): operators 1 and 2 both take operator 1's value
    assert kinds == [(ADD, 0, 0), (SUB, 1, 0), (SUB, 2, 0), (F, 3, 0), (F, 3, 1), (F, 2, 2), (P, 1, 0)], kinds
    assert all(sc.node[i].formula_maxiter == 20 for i in (3, 4, 5))
    assert sc.node[4].julia_mode == 1 and list(sc.node[4].julia_c) == [0.1, 0.2, 0.3]
    assert list(sc.node[5].position) == [0.0, 0.0, 1.0]
    scene_sequence(sc)
