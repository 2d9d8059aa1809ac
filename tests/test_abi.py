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
               "mbr_job": abi.Job, "mbr_tuning": abi.Tuning, "mbr_formula_param": abi.FormulaParam,
               "mbr_node": abi.Node, "mbr_primitive": abi.Primitive}
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


def _layout(pixels, per):
    off = (C.c_uint64 * 3)()
    total = C.c_uint64()
    assert abi.load().mbr_wavefront_scratch_layout(pixels, per, off, C.byref(total)) == abi.MBR_OK
    return list(off), total.value


@pytest.mark.parametrize("pixels", [0, 1, 2, 3, 7, 99 * 55, 99 * 99, 1001 * 751, 1920 * 1080, 178131, 3840 * 2160])
@pytest.mark.parametrize("per", [0, 1, 5, 17])
def test_wavefront_scratch_records_are_16_byte_aligned(pixels, per):
    """The float4 start and direction records follow the 88-byte hit records:
    both regions must start on a 16-byte boundary for odd pixel counts too."""
    off, total = _layout(pixels, per)
    assert off[0] == 256
    assert all(o % 16 == 0 for o in off), off
    assert off[1] >= off[0] + 88 * pixels and off[1] - (off[0] + 88 * pixels) < 256
    assert off[2] == off[1] + 16 * pixels
    assert total == off[2] + 16 * pixels * per


def test_noalloc_pixel_limits_match_the_header():
    """The largest frames the allocation-free entry point accepts (documented
    in mbr.h: 178,130 pixels with a shadow and 16 AO rays, 644,011 with
    neither), from the scratch layout and the static array's size."""
    have = 64 * 1024 * 1024 - (65536 * 2 + 256)
    for per, documented in ((17, 178130), (0, 644011)):
        assert _layout(documented, per)[1] <= have
        assert _layout(documented + 1, per)[1] > have
    assert b"178,130" in open(HEADER, "rb").read() and b"644,011" in open(HEADER, "rb").read()


def test_advanced_quality_defaults():
    p = abi.params_defaults()
    assert p.advanced_quality == 0
    assert (p.detail_size_min, p.detail_size_max) == (1e-12, 1.0)
    assert (p.abs_min_marching_step, p.abs_max_marching_step) == (1e-15, 3.0)
    assert (p.rel_min_marching_step, p.rel_max_marching_step) == (1e-2, 1e4)
