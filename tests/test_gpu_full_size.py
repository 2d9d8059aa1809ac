"""Parity at the workloads' own sizes against the oracle (the CPU
restatement, run on the host's cores), with the bars the engines are
specified to: the plain FP64 engine - hit masks and iteration counts
identical on >= 99.9 % of pixels, depth within 1e-9 on >= 99.9 % of common
hits, 8-bit PSNR >= 50 dB; the FP32 forms - hit mismatch <= 0.1 %, depth
within 1e-4 on >= 99.9 % of common hits.

- the 512 x 512 Mandelbulb (plain FP64, FP32 wavefront, AUTO);
- the 1920 x 1080 Mandelbox, wide view (FP32 wavefront, 16 AO rays);
- the same Mandelbox at the deep zoom (AUTO: split precision), on bands of
  rows spread over the frame;
- jobs of the 2048-job batch (AUTO batch: FP32 jobs, and FP64 for the
  cameras whose hit thresholds FP32 cannot resolve), a sample of 24 jobs
  rendered by the oracle: hit mismatch <= 0.1 % per job, depth within 1e-4
  on >= 99.9 % of the sample's common hits together and >= 99.5 % of each
  job's (a Mandelbox that fills the view at grazing angles stays above
  99.8 %);
- the hybrid GI frame at 3840 x 2160 x 16 spp, on a band of rows (FP32
  hybrid iteration; GI colour within the FP32 GI bar).
"""
import ctypes as C

import numpy as np
import pytest
import torch

from mandelbulber2_b200 import abi, configs
from mandelbulber2_b200.render import STATS_FIELDS, alloc_outputs, outputs_struct
from mandelbulber2_b200.shard import band_params

from .parity import compare

pytestmark = pytest.mark.gpu
NAMES = ("depth", "iters", "hit", "normal", "ao", "rgb8")


def fp32_bar(m):
    assert m["hit_mismatch"] <= 0.001, m
    assert m["depth_rel_le_1e-4"] >= 0.999, m


def test_mandelbulb_512(renderer, oracle):
    sc, cam, p = configs.mandelbulb_512()
    o, _ = oracle.render(sc, cam, p, threads=oracle.threads())
    renderer.set_scene(sc)
    for engine in (abi.ENGINE_PLAIN_FP64, abi.ENGINE_WAVEFRONT_FP32, abi.ENGINE_WAVEFRONT_AUTO):
        fr = renderer.render(cam, p, engine, outputs=NAMES)
        m = compare({k: v.cpu().numpy() for k, v in fr.buffers.items()}, o)
        print("mandelbulb 512", abi.ENGINE_NAMES[engine], m)
        if engine == abi.ENGINE_PLAIN_FP64:
            assert m["hit_iters_match"] >= 0.999, m
            assert m["depth_rel_le_1e-9"] >= 0.999, m
            assert m["psnr"] >= 50.0, m
        else:
            fp32_bar(m)


def test_mandelbox_1080p_wide_view(renderer, oracle):
    sc, cam, p = configs.mandelbox_1080p("A")
    o, _ = oracle.render(sc, cam, p, threads=oracle.threads())
    renderer.set_scene(sc)
    fr = renderer.render(cam, p, abi.ENGINE_WAVEFRONT_FP32, outputs=NAMES)
    m = compare({k: v.cpu().numpy() for k, v in fr.buffers.items()}, o)
    print("mandelbox 1080p A fp32", m)
    fp32_bar(m)
    assert m["normal_deg_p99"] <= 0.1, m


def test_mandelbox_1080p_deep_zoom(renderer, oracle):
    sc, cam, p = configs.mandelbox_1080p("A")
    renderer.set_scene(sc)
    c = renderer.render(cam, band_params(p, 540, 541), abi.ENGINE_PLAIN_FP64, outputs=("depth",))
    cdepth = float(c.buffers["depth"].cpu().numpy()[540 * 1920 + 960])
    sc, cam, p = configs.mandelbox_1080p("B", centre_depth=cdepth)
    renderer.set_scene(sc)
    for r0 in (0, 270, 536, 810, 1072):
        pb = band_params(p, r0, r0 + 8)
        o, _ = oracle.render(sc, cam, pb, rows=(r0, r0 + 8), threads=oracle.threads())
        fr = renderer.render(cam, pb, abi.ENGINE_WAVEFRONT_AUTO, outputs=NAMES)
        lo, hi = r0 * cam.width, (r0 + 8) * cam.width
        m = compare({k: v.cpu().numpy()[lo:hi] for k, v in fr.buffers.items()}, o)
        print("mandelbox 1080p B auto rows", r0, m)
        fp32_bar(m)
        assert m["normal_deg_p99"] <= 0.05, m


def test_batch_jobs_against_the_oracle(renderer, oracle):
    scenes, cams, offs, total = configs.batch_jobs()
    p = configs.base_params(5, 20.0)
    p.shadow_enable = 0
    lib = abi.load()
    jobs = (abi.Job * len(cams))()
    for i, c in enumerate(cams):
        jobs[i].camera = c
        jobs[i].scene_index = i
        jobs[i].pixel_offset = offs[i]
    sc_arr = (abi.Scene * len(scenes))(*scenes)
    bufs = alloc_outputs(total, renderer.device, ("depth", "iters", "hit", "normal"))
    stats = torch.zeros(len(STATS_FIELDS), dtype=torch.int64, device=renderer.device)
    o = outputs_struct(bufs, stats)
    b = C.c_void_p()
    st = lib.mbr_batch_create(renderer.ctx, sc_arr, len(scenes), jobs, len(cams), C.byref(p), C.byref(o),
                              abi.ENGINE_WAVEFRONT_AUTO, None, C.byref(b))
    assert st == abi.MBR_OK, lib.mbr_last_error_string(renderer.ctx)
    try:
        s = torch.cuda.current_stream()
        assert lib.mbr_batch_launch(b, C.c_void_p(s.cuda_stream)) == abi.MBR_OK
        renderer.sync()
    finally:
        lib.mbr_batch_destroy(b)
    got = {k: v.cpu().numpy() for k, v in bufs.items()}
    rng = np.random.default_rng(3)
    picked = [i for i in rng.permutation(len(cams)) if cams[i].width <= 256][:24]
    worst, within, common = [], 0, 0
    for i in picked:
        c = cams[i]
        n = c.width * c.height
        ora, _ = oracle.render(scenes[i], c, p, threads=oracle.threads(), outputs=("depth", "iters", "hit", "normal"))
        if ora["hit"].mean() > 0.999:  # a camera inside the solid: every pixel at depth ~0
            continue
        g = {k: got[k][offs[i]: offs[i] + n] for k in got}
        m = compare(g, ora)
        worst.append(m["hit_mismatch"])
        print("job", i, c.width, m)
        assert m["hit_mismatch"] <= 0.001, (i, m)
        both = g["hit"].astype(bool) & ora["hit"].astype(bool)
        if both.any():
            rel = np.abs(g["depth"][both] - ora["depth"][both]) / np.abs(ora["depth"][both])
            within += int((rel <= 1e-4).sum())
            common += int(both.sum())
            assert m["depth_rel_le_1e-4"] >= 0.995, (i, m)
    assert len(worst) >= 12
    # over the sampled jobs' common hits together
    print("batch sample: depth within 1e-4 on", within / common, "of", common, "common hits")
    assert within / common >= 0.999


def test_hybrid_gi_2160p_band(renderer, oracle):
    sc, cam, p = configs.hybrid_gi_2160p()
    pb = band_params(p, 1076, 1084)
    o, _ = oracle.render(sc, cam, pb, rows=(1076, 1084), threads=oracle.threads(),
                         outputs=("depth", "iters", "hit", "rgb", "rgb8"))
    renderer.set_scene(sc)
    fr = renderer.render(cam, pb, abi.ENGINE_WAVEFRONT_FP32, outputs=("depth", "iters", "hit", "rgb", "rgb8"))
    lo, hi = 1076 * cam.width, 1084 * cam.width
    g = {k: v.cpu().numpy()[lo:hi] for k, v in fr.buffers.items()}
    m = compare(g, o)
    print("hybrid GI 2160p band", m)
    assert m["hit_mismatch"] <= 0.005, m
    assert m["depth_rel_median"] <= 1e-4, m
    d = np.abs(g["rgb"].astype(np.float64) - o["rgb"].astype(np.float64)).max(axis=1)
    assert np.mean(d <= 1e-3) >= 0.9 and float(np.mean(d)) <= 0.01, (np.mean(d <= 1e-3), float(np.mean(d)))
