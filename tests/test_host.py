"""Host-side logic of the library against the oracle: hybrid sequence
construction, DE-function vote, bailout rules, camera set-up and argument
validation.  CPU only."""
import ctypes as C
import math
import os

import numpy as np
import pytest

from mandelbulber2_b200 import abi, configs
from mandelbulber2_b200.render import MbrError, camera_rotation, scene_sequence


def hybrid(slots, maxiter=12, repeat_from=1, use_default_bailout=1, de_function=0):
    s = abi.scene_defaults(slots[0][0])
    s.hybrid_fractal_enable = 1
    s.n_fractals = len(slots)
    s.formula_maxiter = maxiter
    s.repeat_from = repeat_from
    s.use_default_bailout = use_default_bailout
    s.delta_de_function = de_function
    for i, sl in enumerate(slots):
        formula, iters = sl[0], sl[1]
        abi.load().mbr_fractal_defaults(s.fractal[i], formula)
        s.fractal[i].formula_iterations = iters
        if len(sl) > 2:
            s.fractal[i].formula_start_iteration = sl[2]
            s.fractal[i].formula_stop_iteration = sl[3]
    return s


SCENES = [
    ("bulb", configs.mandelbulb_scene()),
    ("box", configs.mandelbox_scene()),
    ("menger", configs.menger_scene()),
    ("hybrid_bulb_menger", configs.hybrid_scene()),
    ("hybrid_3", hybrid([(8, 2), (2, 1), (7, 4)])),
    ("hybrid_repeat", hybrid([(8, 2), (2, 3), (7, 1)], repeat_from=2)),
    ("hybrid_ranges", hybrid([(2, 1, 0, 4), (7, 2, 3, 100), (8, 1, 5, 7)])),
    ("hybrid_none_slot", hybrid([(2, 2), (0, 1), (8, 1)])),
    ("hybrid_common_bailout", hybrid([(2, 1), (8, 1)], use_default_bailout=0)),
    ("hybrid_log_forced", hybrid([(8, 5), (2, 1)], de_function=2)),
    ("hybrid_tie", hybrid([(2, 2), (8, 2)])),
]


@pytest.mark.parametrize("name,scene", SCENES)
def test_sequence_matches_oracle(oracle, name, scene):
    seq, length, fn, bail = scene_sequence(scene)
    oseq, olength, ofn, obail = oracle.sequence(scene)
    assert length == olength
    assert seq == oseq
    assert fn == ofn
    n = scene.n_fractals if scene.hybrid_fractal_enable else 1
    for i in range(n):
        if scene.fractal[i].formula != 0:
            assert bail[i] == obail[i]


def test_hybrid_c5_sequence_and_vote():
    seq, length, fn, bail = scene_sequence(configs.hybrid_scene())
    assert seq[:12] == [0, 0, 0] + [1] * 9
    assert fn == abi.DE_LINEAR  # linear (Menger, 9 iterations) outvotes log (bulb, 3)
    assert bail[0] == bail[1] == 10.0


def test_camera_rotation_matches_oracle(oracle):
    rng = np.random.default_rng(3)
    for _ in range(50):
        cam = configs.camera(tuple(rng.uniform(-4, 4, 3)), target=tuple(rng.uniform(-0.5, 0.5, 3)))
        m, ang = camera_rotation(cam)
        om, zero, oang = oracle.camera(cam)
        assert ang == list(oang)
        assert m == list(om)


@pytest.mark.parametrize("mutate,status", [
    (lambda s: setattr(s, "n_fractals", 0), abi.MBR_EINVAL),
    (lambda s: setattr(s, "formula_maxiter", 0), abi.MBR_EINVAL),
    (lambda s: setattr(s.fractal[0], "formula", 6), abi.MBR_EUNSUPPORTED),
    (lambda s: setattr(s.fractal[0], "formula_weight", 1.5), abi.MBR_EINVAL),
    (lambda s: setattr(s, "delta_de_function", 7), abi.MBR_EINVAL),
    (lambda s: setattr(s, "delta_de_function", abi.DE_JOS_KLEINIAN), abi.MBR_EUNSUPPORTED),  # analytic Jos Kleinian
    (lambda s: setattr(s, "delta_de_method", 3), abi.MBR_EINVAL),
    (lambda s: setattr(s, "deltade_relative_delta", 0.0), abi.MBR_EINVAL),
    (lambda s: (setattr(s.fractal[0], "formula", 8), setattr(s.fractal[0], "mandelbox_folding_min_radius", 0.0)),
     abi.MBR_EINVAL),
    (lambda s: (setattr(s.fractal[0], "formula", 8), setattr(s.fractal[0], "mandelbox_folding_limit", -1.0)),
     abi.MBR_EINVAL),
    (lambda s: setattr(s.fractal[0], "bulb_power", float("nan")), abi.MBR_EINVAL),
])
def test_scene_validation(mutate, status):
    s = abi.scene_defaults()
    mutate(s)
    with pytest.raises(MbrError) as e:
        scene_sequence(s)
    assert e.value.status == status


def test_opcount_mandelbox_and_bulb(oracle):
    box = oracle.opcount(configs.mandelbox_scene(), 0, [0.5, 0.4, 0.3, 0.0])  # 0.25 < r2 < 1: fixed-radius fold
    assert box["transc"] == 0 and box["sqrt"] == 1 and box["div"] == 1
    assert 25 <= box["add"] + box["mul"] <= 45
    bulb = oracle.opcount(configs.mandelbulb_scene(), 0, [0.3, 0.2, 0.1, 0.0])
    assert bulb["transc"] == 7 and bulb["div"] == 1


def test_oracle_render_deterministic_and_counts(oracle):
    sc, cam, p = configs.mandelbulb_512(24, 16)
    a, sa = oracle.render(sc, cam, p, threads=2)
    b, sb = oracle.render(sc, cam, p, threads=3)
    for k in a:
        assert np.array_equal(a[k], b[k]), k
    assert sa == sb
    assert sa["pixels"] == 24 * 16
    parts = sum(sa[k] for k in ("march_steps", "binary_steps", "normal_evals", "shadow_evals", "ao_evals", "gi_evals"))
    assert parts == sa["de_evals"]
    assert sa["normal_evals"] == 6 * int(a["hit"].sum())


def test_oracle_row_bands_compose(oracle):
    """Rendering two row bands separately equals the whole frame (row-band sharding)."""
    sc, cam, p = configs.mandelbox_1080p("A", 40, 24, ao_rays=4)
    whole, _ = oracle.render(sc, cam, p)
    top, _ = oracle.render(sc, cam, p, rows=(0, 10))
    bot, _ = oracle.render(sc, cam, p, rows=(10, 24))
    for k in whole:
        assert np.array_equal(whole[k], np.concatenate([top[k], bot[k]])), k


def test_fastdiv_exact(tmp_path):
    """The multiply-high division of csrc/fastdiv.h equals integer division
    for divisors 1..300, powers of two and their neighbours, 2^31-1, and
    numerators up to 2^63-1 (edge cases, exact multiples, random)."""
    import shutil
    import subprocess

    cxx = shutil.which("g++") or "/usr/bin/g++"
    here = os.path.dirname(os.path.abspath(__file__))
    csrc = os.path.join(os.path.dirname(here), "mandelbulber2_b200", "csrc")
    exe = str(tmp_path / "fastdiv_check")
    subprocess.run([cxx, "-O2", "-std=c++17", "-I", csrc, os.path.join(here, "fastdiv_check.cpp"), "-o", exe],
                   check=True)
    out = subprocess.run([exe], capture_output=True, text=True)
    bad, checked = map(int, out.stdout.split())
    assert checked > 1_000_000
    assert bad == 0 and out.returncode == 0
