"""The oracle's restatement of the reference's struct defaults equals the
library's mbr_*_defaults byte for byte, so the CPU arm of the benchmark
(which must not load the product library) fills the same structs."""
import ctypes as C
import json
import os
import subprocess
import sys

from mandelbulber2_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def raw(s):
    return bytes(memoryview(s))


def test_defaults_equal_the_libraries(oracle):
    lib, ol = abi.load(), oracle.lib
    for name, cls in (("scene_defaults", abi.Scene), ("camera_defaults", abi.Camera),
                      ("render_params_defaults", abi.RenderParams)):
        a, b = cls(), cls()
        getattr(lib, "mbr_" + name)(C.byref(a))
        getattr(ol, "oracle_" + name)(C.byref(b))
        assert raw(a) == raw(b), name
    for formula in (0, 2, 3, 4, 7, 8, 10, 11):
        a, b = abi.Fractal(), abi.Fractal()
        lib.mbr_fractal_defaults(C.byref(a), formula)
        ol.oracle_fractal_defaults(C.byref(b), formula)
        assert raw(a) == raw(b), formula


def test_reference_arm_runs_without_the_product_library():
    """bench.py --impl reference on the 512 x 512 Mandelbulb: one full frame
    per step through the oracle, with libmbr.so never mapped."""
    env = dict(os.environ, OMP_NUM_THREADS=str(min(8, os.cpu_count() or 1)))
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                          "--warmup", "0", "--workload", "mandelbulb_512"], capture_output=True, text=True,
                         env=env, timeout=600, check=True).stdout
    line = json.loads(out.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["product_library_loaded"] is False
    assert line["cpu_baseline"]["sample"].startswith("the whole 512x512 frame")
    assert line["config"]["width"] == 512 and "parallelism" in line["config"] and "l2" in line["config"]
