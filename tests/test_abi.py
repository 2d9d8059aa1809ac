"""The C-ABI library: it loads, exports every function include/mbr.h
declares, and its structs have the C layout the ctypes mirror assumes.
No GPU work is done here."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import pytest

from mandelbulber2_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "mbr.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(mbr_[a-z0-9_]+)\s*\(", src)))


def test_library_loads_and_exports_every_declared_symbol():
    lib = abi.load()
    names = declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) == set(abi.PROTOTYPES), set(names) ^ set(abi.PROTOTYPES)


def test_struct_layout_matches_c(tmp_path):
    prog = tmp_path / "sizes.c"
    structs = {"mbr_fractal": abi.Fractal, "mbr_scene": abi.Scene, "mbr_camera": abi.Camera,
               "mbr_render_params": abi.RenderParams, "mbr_stats": abi.Stats, "mbr_outputs": abi.Outputs,
               "mbr_job": abi.Job, "mbr_tuning": abi.Tuning}
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void){"]
    for cname, py in structs.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for f, _ in py._fields_:
            lines.append(f'printf("{cname}.{f} %zu\\n", offsetof({cname}, {f}));')
    lines.append("return 0;}")
    prog.write_text("\n".join(lines))
    exe = tmp_path / "sizes"
    subprocess.run(["gcc", "-std=c99", str(prog), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    got = dict(l.split() for l in out if l.strip())
    for cname, py in structs.items():
        assert int(got[cname]) == C.sizeof(py), cname
        for f, _ in py._fields_:
            assert int(got[f"{cname}.{f}"]) == getattr(py, f).offset, (cname, f)


def test_defaults_are_the_reference_defaults():
    s = abi.scene_defaults()
    assert s.n_fractals == 1 and s.formula_maxiter == 250 and s.repeat_from == 1
    assert s.use_default_bailout == 1 and s.min_n == 1 and s.bailout == 100.0
    f = s.fractal[0]
    assert f.formula == abi.FORMULA_MANDELBULB and f.bulb_power == 9.0 and f.formula_stop_iteration == 250
    assert f.mandelbox_scale == 2.0 and f.mandelbox_folding_min_radius == 0.5 and f.transf_scale3 == 3.0
    p = abi.params_defaults()
    assert p.detail_level == 1.0 and p.de_factor == 1.0 and p.view_distance_max == 50.0
    assert p.max_raymarching_steps == 10000 and p.binary_steps == 30
    c = abi.camera_defaults()
    assert list(c.camera) == [3.0, -6.0, 2.0] and c.fov_deg == 53.13


def test_version_string():
    assert b"sm_100a" in abi.load().mbr_version()


def test_create_without_gpu_fails_loudly():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    ctx = C.c_void_p()
    assert abi.load().mbr_create(C.byref(ctx), 0) == abi.MBR_ECUDA
    from mandelbulber2_b200.render import Renderer

    with pytest.raises(RuntimeError):
        Renderer(0)
