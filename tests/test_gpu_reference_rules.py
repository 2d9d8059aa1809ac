"""Reference rules of the march that the engines must apply like the oracle,
and launch shapes that earlier tests did not reach, on the GPU through the
C-ABI:

- the equirectangular projection's halved threshold and CalcDelta and its 2:1
  image plane (render_worker.cpp:98-100, 669, 688), on a frame that is not 2:1;
- advanced quality: the threshold clamps (render_worker.cpp:671-675) and the
  march step limits (:819-834);
- odd pixel counts on the wavefront engines (a single frame, a batch with odd
  job sizes, row bands of odd height), where the scratch records follow the
  88-byte hit records;
- the watchdog status word: AO marches that reach max_raymarching_steps end
  as unoccluded (the reference's AO march has no cap), are counted, and
  mbr_sync reports MBR_ETIMEOUT;
- the autotuner's launch shape, and the gamma table ordered on the stream.

Bars: FP64 engines hit/iteration agreement >= 99.9 % and depth within 1e-9
on >= 99.9 % of common hits; FP32 engines hit mismatch <= 0.5 % and median
depth error <= 1e-4 (the FP32 wavefront's bar at these small sizes).
"""
import ctypes as C

import numpy as np
import pytest
import torch

from mandelbulber2_b200 import abi, configs
from mandelbulber2_b200.render import STATS_FIELDS, MbrError, alloc_outputs, outputs_struct, stats_dict

from .parity import compare

pytestmark = pytest.mark.gpu
NAMES = ("depth", "iters", "hit", "normal", "ao", "rgb8")
FP64_ENGINES = (abi.ENGINE_PLAIN_FP64_STRICT, abi.ENGINE_PLAIN_FP64, abi.ENGINE_WAVEFRONT_FP64)
FP32_ENGINES = (abi.ENGINE_PLAIN_MIXED, abi.ENGINE_WAVEFRONT_FP32, abi.ENGINE_WAVEFRONT_AUTO)


def check_engines(renderer, sc, cam, p, o, label, engines=FP64_ENGINES + FP32_ENGINES):
    renderer.set_scene(sc)
    for engine in engines:
        fr = renderer.render(cam, p, engine, outputs=NAMES)
        g = {k: v.cpu().numpy() for k, v in fr.buffers.items()}
        m = compare(g, o)
        print(label, abi.ENGINE_NAMES[engine], m)
        assert fr.stats["pixels"] == cam.width * cam.height
        if engine in FP64_ENGINES:
            assert m["hit_iters_match"] >= 0.999, (engine, m)
            assert m["depth_rel_le_1e-9"] >= 0.999, (engine, m)
        else:
            assert m["hit_mismatch"] <= 0.005, (engine, m)
            assert m["depth_rel_median"] <= 1e-4, (engine, m)


def test_equirectangular_on_a_4_to_3_frame(renderer, oracle):
    sc = configs.mandelbulb_scene(8.0, 20)
    cam = configs.camera((0.15, -1.4, 0.3), fov=360.0, width=96, height=72)
    cam.perspective_type = abi.PROJECTION_EQUIRECTANGULAR
    p = configs.base_params(5, 20.0)
    p.ao_rays = 4
    p.penetrating = 1  # the march length of a penetrating light is CalcDelta / resolution
    o, _ = oracle.render(sc, cam, p)
    assert 0.05 < float(np.mean(o["hit"])) < 0.95
    check_engines(renderer, sc, cam, p, o, "equirectangular 96x72")


def test_advanced_quality(renderer, oracle):
    sc, cam, p = configs.mandelbox_1080p("A", 160, 90, ao_rays=4)
    plain, pst = oracle.render(sc, cam, p)
    p.advanced_quality = 1
    p.detail_size_max = 0.01      # below the distance-proportional threshold of this view: clamps
    p.detail_size_min = 0.004
    p.abs_max_marching_step = 0.4  # below the step the march would take far from the surface
    p.rel_min_marching_step = 0.6
    o, ost = oracle.render(sc, cam, p)
    assert ost["march_steps"] > 1.2 * pst["march_steps"]  # the limits bind
    assert not np.array_equal(o["depth"], plain["depth"])
    check_engines(renderer, sc, cam, p, o, "advanced quality")


@pytest.mark.parametrize("engine", [abi.ENGINE_WAVEFRONT_FP32, abi.ENGINE_WAVEFRONT_FP64, abi.ENGINE_WAVEFRONT_AUTO])
def test_wavefront_odd_pixel_count(renderer, oracle, engine):
    sc, cam, p = configs.mandelbox_1080p("A", 99, 55, ao_rays=16)
    o, _ = oracle.render(sc, cam, p)
    engines = (engine,)
    check_engines(renderer, sc, cam, p, o, "99x55", engines)


def test_batch_with_odd_job_sizes(renderer):
    lib = abi.load()
    scenes = [configs.mandelbox_scene(-1.5, 0.5, 40), configs.mandelbulb_scene(8.0, 100),
              configs.mandelbox_scene(2.2, 0.4, 40)]
    cams = [configs.camera((0.5, -5.5, 1.0), width=33, height=17),
            configs.camera((0.0, -3.0, 0.5), width=45, height=21),
            configs.camera((2.0, 3.0, -1.0), width=99, height=55)]
    p = configs.base_params(5, 20.0)
    p.ao_rays = 4
    jobs = (abi.Job * len(cams))()
    off, offs = 0, []
    for i, c in enumerate(cams):
        jobs[i].camera = c
        jobs[i].scene_index = i
        jobs[i].pixel_offset = off
        offs.append(off)
        off += c.width * c.height
    sc_arr = (abi.Scene * len(scenes))(*scenes)
    names = ("depth", "iters", "hit", "normal", "ao", "rgb8")
    bufs = alloc_outputs(off, renderer.device, names)
    stats = torch.zeros(len(STATS_FIELDS), dtype=torch.int64, device=renderer.device)
    o = outputs_struct(bufs, stats)
    b = C.c_void_p()
    st = lib.mbr_batch_create(renderer.ctx, sc_arr, len(scenes), jobs, len(cams), C.byref(p), C.byref(o),
                              abi.ENGINE_WAVEFRONT_FP32, None, C.byref(b))
    assert st == abi.MBR_OK, lib.mbr_last_error_string(renderer.ctx)
    try:
        s = torch.cuda.current_stream()
        assert lib.mbr_batch_launch(b, C.c_void_p(s.cuda_stream)) == abi.MBR_OK
        renderer.sync()
        got = {k: v.cpu().numpy() for k, v in bufs.items()}
        assert stats_dict(stats)["pixels"] == off
        for i, (sc, cam) in enumerate(zip(scenes, cams)):
            renderer.set_scene(sc)
            single = renderer.render(cam, p, abi.ENGINE_WAVEFRONT_FP32, outputs=names)
            n = cam.width * cam.height
            for k in got:
                part = got[k][offs[i]: offs[i] + n]
                want = single.buffers[k].cpu().numpy()
                if k == "depth":
                    assert np.allclose(part, want, rtol=1e-6), (i, k)
                else:
                    assert np.mean(part == want) >= 0.999, (i, k)
    finally:
        lib.mbr_batch_destroy(b)


@pytest.mark.parametrize("engine", [abi.ENGINE_WAVEFRONT_FP32, abi.ENGINE_WAVEFRONT_FP64])
def test_odd_row_bands_compose_into_the_frame(renderer, engine):
    from mandelbulber2_b200.shard import band_params

    sc, cam, p = configs.mandelbox_1080p("A", 99, 55, ao_rays=4)
    renderer.set_scene(sc)
    names = ("depth", "iters", "hit", "normal", "rgb8")
    whole = renderer.render(cam, p, engine, outputs=names)
    bufs = alloc_outputs(cam.width * cam.height, renderer.device, names)
    for r0, r1 in ((0, 27), (27, 55)):  # 99 x 27 and 99 x 28 pixels: an odd and an even count
        stats = torch.zeros(len(STATS_FIELDS), dtype=torch.int64, device=renderer.device)
        renderer.render_into(cam, band_params(p, r0, r1), bufs, stats, engine)
        renderer.sync()
    for k in bufs:
        assert np.array_equal(bufs[k].cpu().numpy(), whole[k].cpu().numpy()), k


@pytest.mark.parametrize("engine", [abi.ENGINE_PLAIN_FP64_STRICT, abi.ENGINE_WAVEFRONT_FP64,
                                    abi.ENGINE_WAVEFRONT_FP32])
def test_ao_march_cap_sets_the_status_word(renderer, oracle, engine):
    """max_raymarching_steps = 6 cuts some AO marches short: every engine ends
    them as unoccluded, counts them as watchdog trips, and mbr_sync returns
    MBR_ETIMEOUT once (the status word is cleared by the read)."""
    sc, cam, p = configs.mandelbox_1080p("A", 64, 36, ao_rays=4)
    p.max_raymarching_steps = 6
    o, ost = oracle.render(sc, cam, p)
    assert ost["watchdog_trips"] > 0
    renderer.set_scene(sc)
    bufs = alloc_outputs(cam.width * cam.height, renderer.device, NAMES)
    stats = torch.zeros(len(STATS_FIELDS), dtype=torch.int64, device=renderer.device)
    renderer.render_into(cam, p, bufs, stats, engine)
    with pytest.raises(MbrError) as e:
        renderer.sync()
    assert e.value.status == abi.MBR_ETIMEOUT
    assert "AO march" in str(e.value)
    renderer.sync()  # cleared
    trips = stats_dict(stats)["watchdog_trips"]
    assert trips > 0
    g = {k: v.cpu().numpy() for k, v in bufs.items()}
    m = compare(g, o)
    if engine == abi.ENGINE_PLAIN_FP64_STRICT:
        assert trips == ost["watchdog_trips"]
        assert np.array_equal(g["ao"], o["ao"])
    else:
        assert abs(trips - ost["watchdog_trips"]) <= 0.1 * ost["watchdog_trips"] + 2
        assert m["hit_mismatch"] <= 0.005, m
    # a frame with the default budget trips nothing
    p.max_raymarching_steps = 10000
    renderer.render_into(cam, p, bufs, None, engine)
    renderer.sync()


def test_autotune_returns_a_legal_shape_with_the_same_frame(renderer):
    sc, cam, p = configs.mandelbox_1080p("A", 96, 54, ao_rays=4)
    renderer.set_scene(sc)
    renderer.set_tuning(128, 12, 2, 0)
    base = renderer.render(cam, p, abi.ENGINE_WAVEFRONT_FP32, outputs=NAMES)
    t = renderer.autotune(cam, p)
    try:
        assert t.block_size in (128, 256) and t.ctas_per_sm in (6, 8, 12)
        assert t.block_size * t.ctas_per_sm <= 2048
        assert t.refill_k in (0, 2, 4, 8, 16, 24) and t.queue_layout in (0, 1)
        got = renderer.get_tuning()
        assert (got.block_size, got.ctas_per_sm, got.refill_k, got.queue_layout) == \
            (t.block_size, t.ctas_per_sm, t.refill_k, t.queue_layout)
        tuned = renderer.render(cam, p, abi.ENGINE_WAVEFRONT_FP32, outputs=NAMES)
        for k in NAMES:
            assert np.array_equal(base[k].cpu().numpy(), tuned[k].cpu().numpy()), k
        assert base.stats == tuned.stats
    finally:
        renderer.set_tuning(128, 12, 2, 0)


@pytest.mark.parametrize("engine", [abi.ENGINE_PLAIN_FP64, abi.ENGINE_WAVEFRONT_FP32])
def test_gamma_tables_stay_ordered_on_the_stream(renderer, engine):
    """Frames with different gamma values queued back to back on one
    non-blocking stream each use their own gamma table."""
    sc, cam, p = configs.mandelbox_1080p("A", 96, 64, ao_rays=0)
    renderer.set_scene(sc)
    gammas = (0.6, 1.7, 0.6)
    want = {}
    for g in set(gammas):
        p.gamma = g
        want[g] = renderer.render(cam, p, engine, outputs=("rgb8",))["rgb8"].cpu().numpy()
    assert not np.array_equal(want[0.6], want[1.7])
    s = torch.cuda.Stream()
    torch.cuda.synchronize()
    got = []
    with torch.cuda.stream(s):
        for g in gammas:
            p.gamma = g
            b = alloc_outputs(cam.width * cam.height, renderer.device, ("rgb8",))
            renderer.render_into(cam, p, b, None, engine, stream=s)
            got.append(b)
    renderer.sync(s)
    for g, b in zip(gammas, got):
        assert np.array_equal(b["rgb8"].cpu().numpy(), want[g]), g


@pytest.mark.parametrize("case", ["box_limits", "bulb_global_box_fold", "bulb_global_spherical_fold",
                                  "hybrid_folds_limits"])
def test_limit_box_and_global_folds(renderer, oracle, case):
    """The limit box (calculate_distance.cpp:261-275; with a soft shadow,
    shader_aux_shadow.cpp:130-147) and the global box and spherical folds
    (compute_fractal.cpp:190-202): the oracle reproduces the reference's own
    CalculateDistance and render worker bit for bit (tests/golden/
    pipeline_kat.json, render_kat.json); every engine that takes these scenes
    is held to the oracle.  The FP64 wavefront, batches and the allocation-free
    path refuse them."""
    from tests.golden.pipeline_cases import cases

    sc = cases()[case]
    pos = {"box_limits": (0.0, -5.0, 0.5), "bulb_global_box_fold": (0.3, -6.0, 0.4)}.get(case, (0.3, -2.8, 0.4))
    cam = configs.camera(pos, width=64, height=40)
    p = configs.base_params(5, 20.0)
    p.ao_rays = 4
    p.soft_shadow_cone = 15.0
    o, _ = oracle.render(sc, cam, p)
    assert 0.05 < float(np.mean(o["hit"])) < 0.98
    check_engines(renderer, sc, cam, p, o, case,
                  engines=(abi.ENGINE_PLAIN_FP64_STRICT, abi.ENGINE_PLAIN_FP64) + FP32_ENGINES)
    with pytest.raises(MbrError) as e:
        renderer.render(cam, p, abi.ENGINE_WAVEFRONT_FP64)
    assert e.value.status == abi.MBR_EUNSUPPORTED


# Formulas without transcendental functions (the Mandelbox, the Menger
# sponge) run the same IEEE operations on the strict FP64 engine as in the
# oracle, so their distances are bit-identical; the Mandelbulb's asin, atan2,
# sincos and pow differ from the host's libm by an ulp here and there.
def _exact(case):
    return "bulb" not in case and "hybrid" not in case


def _rel(a, b):
    return np.abs(a - b) / np.maximum(np.abs(b), 1e-300)


@pytest.mark.parametrize("case", ["box_delta_preferred", "bulb_delta_pseudo_kleinian", "box_delta_jos_kleinian",
                                  "box_delta_max_axis", "hybrid_delta", "box_delta_iter_thresh_limits"])
def test_delta_de_distances(renderer, oracle, case):
    """The delta DE (calculate_distance.cpp:607-760) through mbr_distance
    against the oracle (which equals the reference's own CalculateDistance on
    these scenes, tests/golden/pipeline_kat.json).  The strict FP64 engine is
    bit-identical on the Mandelbox and Menger scenes.  The difference quotient
    over offsets of 1e-5 of the detail size magnifies an ulp of |z| about
    1e7-fold (the max-axis function, one derivative component, more), so the
    FMA engine and the Mandelbulb scenes are held, over the points whose
    orbit escapes within N iterations, to median relative error <= 1e-6 and
    95th percentile <= 1e-3, with iteration counts identical on >= 99.9 % of
    them.  Longer orbits (the set's interior, iterated up to 5 x N for the
    normals in iteration-threshold mode) are chaotic: there an ulp decides
    the result on either engine, so they are not compared.  FP32 engines
    refuse the delta DE."""
    from tests.golden.pipeline_cases import cases

    sc = cases()[case]
    renderer.set_scene(sc)
    rng = np.random.default_rng(11)
    pts = rng.uniform(-2.0, 2.0, size=(4096, 3))
    for det in (1e-3, 0.05):
        for nm in (False, True):
            od, oit = oracle.distance(sc, pts, det, nm)
            for engine in (abi.ENGINE_PLAIN_FP64_STRICT, abi.ENGINE_PLAIN_FP64):
                d, it = renderer.distance(torch.from_numpy(pts), det, nm, engine)
                d, it = d.cpu().numpy(), it.cpu().numpy()
                if engine == abi.ENGINE_PLAIN_FP64_STRICT and _exact(case):
                    assert np.array_equal(d, od) and np.array_equal(it, oit), (case, det, nm)
                    continue
                esc = oit <= sc.formula_maxiter
                rel = _rel(d[esc], od[esc])
                print(case, det, nm, abi.ENGINE_NAMES[engine], "escaping", int(esc.sum()), "rel median",
                      np.median(rel), "p95", np.percentile(rel, 95), "iters", np.mean(it[esc] == oit[esc]))
                assert esc.sum() >= 256
                assert np.median(rel) <= 1e-6 and np.percentile(rel, 95) <= 1e-3, (case, det, nm, engine)
                assert np.mean(it[esc] == oit[esc]) >= 0.999, (case, det, nm, engine)
    with pytest.raises(MbrError) as e:
        renderer.distance(torch.from_numpy(pts), 1e-3, False, abi.ENGINE_PLAIN_MIXED)
    assert e.value.status == abi.MBR_EUNSUPPORTED


@pytest.mark.parametrize("case", ["box_delta_de", "bulb_delta_de_advanced_quality"])
def test_delta_de_frames(renderer, oracle, case):
    """Frames with the delta DE on the plain FP64 engines against the oracle
    (whose render worker equals the reference's on these frames,
    tests/golden/render_kat.json): bit-identical on the strict engine for the
    Mandelbox; otherwise hits and iteration counts identical on >= 99.5 % of
    the pixels (the delta quotient's magnified rounding moves a few march
    steps) and depth within 1e-6 on >= 99 % of the common hits.  The other
    engines refuse delta-DE scenes."""
    from tests.golden.pipeline_cases import render_cases

    _, sc, cam, p = [c for c in render_cases() if c[0] == case][0]
    cam.width, cam.height = 96, 64
    p.ao_rays = 4
    o, ost = oracle.render(sc, cam, p)
    assert 0.05 < float(np.mean(o["hit"])) < 0.98
    renderer.set_scene(sc)
    for engine in (abi.ENGINE_PLAIN_FP64_STRICT, abi.ENGINE_PLAIN_FP64):
        fr = renderer.render(cam, p, engine, outputs=NAMES)
        g = {k: v.cpu().numpy() for k, v in fr.buffers.items()}
        if engine == abi.ENGINE_PLAIN_FP64_STRICT and _exact(case):
            for k in ("depth", "iters", "hit", "normal", "ao", "rgb8"):
                assert np.array_equal(g[k], o[k]), (case, k)
            for k in ("de_evals", "formula_iterations", "march_steps", "normal_evals", "ao_evals"):
                assert fr.stats[k] == ost[k], (case, k, fr.stats[k], ost[k])
            continue
        m = compare(g, o)
        print(case, abi.ENGINE_NAMES[engine], m)
        assert m["hit_iters_match"] >= 0.995, (engine, m)
        assert m["depth_rel_le_1e-4"] >= 0.99, (engine, m)
        both = g["hit"].astype(bool) & o["hit"].astype(bool)
        assert np.mean(_rel(g["depth"][both], o["depth"][both]) <= 1e-6) >= 0.99, engine
    for engine in (abi.ENGINE_PLAIN_MIXED, abi.ENGINE_WAVEFRONT_FP32, abi.ENGINE_WAVEFRONT_FP64,
                   abi.ENGINE_WAVEFRONT_AUTO):
        with pytest.raises(MbrError) as e:
            renderer.render(cam, p, engine)
        assert e.value.status == abi.MBR_EUNSUPPORTED, engine


@pytest.mark.parametrize("case", ["bulb_pseudo_kleinian", "box_max_axis", "hybrid_max_axis", "hybrid_pseudo_kleinian"])
def test_other_analytic_de_functions(renderer, oracle, case):
    """The pseudo-Kleinian and max-axis analytic DE functions
    (compute_fractal.cpp:495-621) on every engine that takes extended scenes;
    the strict FP64 engine equals the oracle bit for bit on Mandelbox
    distances; on the Mandelbulb ones (whose libm functions differ by an ulp
    here and there) it agrees within 1e-8 on >= 99.9 % of the points whose
    orbit escapes (interior orbits are chaotic)."""
    from tests.golden.pipeline_cases import cases

    sc = cases()[case]
    renderer.set_scene(sc)
    rng = np.random.default_rng(12)
    pts = rng.uniform(-2.0, 2.0, size=(4096, 3))
    od, oit = oracle.distance(sc, pts, 1e-3, False)
    d, it = renderer.distance(torch.from_numpy(pts), 1e-3, False, abi.ENGINE_PLAIN_FP64_STRICT)
    d, it = d.cpu().numpy(), it.cpu().numpy()
    if _exact(case):
        assert np.array_equal(d, od) and np.array_equal(it, oit), case
    else:
        esc = oit <= sc.formula_maxiter
        rel = _rel(d[esc], od[esc])
        print(case, "escaping", int(esc.sum()), "rel median", np.median(rel), "max", rel.max(),
              "iters", np.mean(it[esc] == oit[esc]))
        assert esc.sum() >= 256
        assert np.mean(rel <= 1e-8) >= 0.999 and np.mean(it[esc] == oit[esc]) >= 0.999, case
    cam = configs.camera((0.0, -3.0, 0.3) if "bulb" in case or "hybrid" in case else (0.0, -6.0, 0.0), width=64,
                         height=40)
    p = configs.base_params(5, 20.0)
    p.ao_rays = 4
    o, _ = oracle.render(sc, cam, p)
    assert 0.02 < float(np.mean(o["hit"])) < 0.98, float(np.mean(o["hit"]))
    check_engines(renderer, sc, cam, p, o, case,
                  engines=(abi.ENGINE_PLAIN_FP64_STRICT, abi.ENGINE_PLAIN_FP64) + FP32_ENGINES)


@pytest.mark.parametrize("case", ["bulb_slow_shading", "box_slow_shading"])
def test_slow_shading(renderer, oracle, case):
    """Iteration-count normals (shader_calculate_normals.cpp:83-106): the
    gradient of 1 + N - iterations over an 11^3 lattice of orbits around the
    hit.  The oracle equals the reference's render worker on these frames
    (tests/golden/render_kat.json); the strict FP64 engine equals the oracle
    bit for bit on the Mandelbox, the other plain engines are held to their
    bars, and the wavefront engines refuse slow shading."""
    from tests.golden.pipeline_cases import render_cases

    _, sc, cam, p = [c for c in render_cases() if c[0] == case][0]
    cam.width, cam.height = 64, 40
    o, ost = oracle.render(sc, cam, p)
    assert 0.05 < float(np.mean(o["hit"])) < 0.98
    renderer.set_scene(sc)
    for engine in (abi.ENGINE_PLAIN_FP64_STRICT, abi.ENGINE_PLAIN_FP64, abi.ENGINE_PLAIN_MIXED):
        fr = renderer.render(cam, p, engine, outputs=NAMES)
        g = {k: v.cpu().numpy() for k, v in fr.buffers.items()}
        m = compare(g, o)
        print(case, abi.ENGINE_NAMES[engine], m)
        if engine == abi.ENGINE_PLAIN_FP64_STRICT and _exact(case):
            for k in NAMES:
                assert np.array_equal(g[k], o[k]), (case, k)
            assert fr.stats["normal_evals"] == ost["normal_evals"]
        elif engine != abi.ENGINE_PLAIN_MIXED:
            assert m["hit_iters_match"] >= 0.999 and m["depth_rel_le_1e-9"] >= 0.999, m
            # the normal is the gradient of integer iteration counts: where an
            # FMA's rounding moves a lattice orbit across the bailout, a count
            # changes by one and the normal turns by a degree or two
            assert m["normal_deg_median"] <= 1e-3 and m["normal_deg_p99"] <= 5.0, m
        else:
            assert m["hit_mismatch"] <= 0.005 and m["depth_rel_median"] <= 1e-4, m
            # FP32 orbits near the bailout shift some lattice points' iteration counts
            assert m["normal_deg_median"] <= 1.0, m
    for engine in (abi.ENGINE_WAVEFRONT_FP32, abi.ENGINE_WAVEFRONT_FP64, abi.ENGINE_WAVEFRONT_AUTO):
        with pytest.raises(MbrError) as e:
            renderer.render(cam, p, engine)
        assert e.value.status == abi.MBR_EUNSUPPORTED
