"""The allocation-free entry point, mbr_render_noalloc, called through the C-ABI.

It exists for callers that cannot allocate device memory (an application
whose device memory belongs to its own allocator, or a process under a hard
memory cap).  It must give the frame that mbr_render gives with the FP32
wavefront engine, on two calls in a row (the scratch array keeps the previous
call's contents), reject frames larger than its static scratch with a clear
error, and leave the device's free memory unchanged.  This file is collected
last so that a run stopping at its first failure has run every other test.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from mandelbulber2_b200 import abi, configs
from mandelbulber2_b200.render import STATS_FIELDS, alloc_outputs, outputs_struct, stats_dict

pytestmark = pytest.mark.gpu
NAMES = ("depth", "iters", "hit", "normal", "shade", "ao", "rgb", "rgb8")


@pytest.mark.parametrize("size", [(160, 90), (99, 55)])  # 99 x 55: an odd pixel count
def test_noalloc_matches_mbr_render_on_two_calls(renderer, size):
    lib = abi.load()
    sc, cam, p = configs.mandelbox_1080p("A", *size)
    renderer.set_scene(sc)
    ref = renderer.render(cam, p, abi.ENGINE_WAVEFRONT_FP32, outputs=NAMES)
    want = {k: v.cpu().numpy() for k, v in ref.buffers.items()}
    err = C.create_string_buffer(512)
    for call in range(2):
        bufs = alloc_outputs(cam.width * cam.height, renderer.device, NAMES)
        for v in bufs.values():
            v.fill_(0)
        stats = torch.zeros(len(STATS_FIELDS), dtype=torch.int64, device=renderer.device)
        o = outputs_struct(bufs, stats)
        torch.cuda.synchronize()
        free_before = torch.cuda.mem_get_info()[0]
        s = torch.cuda.current_stream()
        st = lib.mbr_render_noalloc(C.byref(sc), C.byref(cam), C.byref(p), C.byref(o), C.c_void_p(s.cuda_stream),
                                    err, len(err))
        assert st == abi.MBR_OK, err.value
        torch.cuda.synchronize()
        if call == 1:  # the first call may load the library's device image; later calls allocate nothing
            assert torch.cuda.mem_get_info()[0] == free_before
        got = {k: v.cpu().numpy() for k, v in bufs.items()}
        assert np.allclose(got["depth"], want["depth"], rtol=1e-6), call
        for k in ("iters", "hit", "rgb8"):
            assert np.mean(got[k] == want[k]) >= 0.999, (call, k)
        for k in ("normal", "shade", "ao", "rgb"):
            assert np.allclose(got[k], want[k], rtol=1e-5, atol=1e-6), (call, k)
        assert stats_dict(stats) == ref.stats, call


def test_noalloc_rejects_frames_beyond_its_scratch():
    lib = abi.load()
    sc, cam, p = configs.mandelbox_1080p("A", 1920, 1080)  # 2.07M pixels with 17 shading tasks per hit
    o = abi.Outputs()
    err = C.create_string_buffer(512)
    st = lib.mbr_render_noalloc(C.byref(sc), C.byref(cam), C.byref(p), C.byref(o), None, err, len(err))
    assert st == abi.MBR_EINVAL
    assert b"at most 178130 pixels" in err.value, err.value


def test_noalloc_gamma_tables_stay_ordered_on_the_stream(renderer):
    """Two frames with different gamma values queued back to back on one
    non-blocking stream: each must be coloured with its own table."""
    lib = abi.load()
    sc, cam, p = configs.mandelbox_1080p("A", 96, 64)
    renderer.set_scene(sc)
    gammas = (0.6, 1.7)
    want = []
    for g in gammas:
        p.gamma = g
        want.append(renderer.render(cam, p, abi.ENGINE_WAVEFRONT_FP32, outputs=("rgb8",)).buffers["rgb8"].cpu().numpy())
    s = torch.cuda.Stream()
    err = C.create_string_buffer(512)
    bufs = []
    torch.cuda.synchronize()
    with torch.cuda.stream(s):
        for g in gammas:
            p.gamma = g
            b = alloc_outputs(cam.width * cam.height, renderer.device, ("rgb8",))
            o = outputs_struct(b, None)
            st = lib.mbr_render_noalloc(C.byref(sc), C.byref(cam), C.byref(p), C.byref(o), C.c_void_p(s.cuda_stream),
                                        err, len(err))
            assert st == abi.MBR_OK, err.value
            bufs.append(b)
    s.synchronize()
    for b, w in zip(bufs, want):
        assert np.mean(b["rgb8"].cpu().numpy() == w) >= 0.999
