"""Fast ambient occlusion (FastAmbientOcclusion,
shader_fast_ambient_occlusion.cpp:40-65: quality^2 - 1 distance samples along
the normal) on every engine against the oracle.  On the Mandelbox (IEEE
operations only) the strict FP64 kernel is held to bit-exactness, counts
included; the other engines to the FP64 and FP32 bars on the hits and to the
AO factor itself on 99 % of the common hits: FP64 within 1e-6 of the
oracle's, FP32 within 1e-4 (measured on a B200: 1.2e-7 and 2.6e-6).
"""
import numpy as np
import pytest

from mandelbulber2_b200 import abi, configs

from .parity import compare

pytestmark = pytest.mark.gpu
NAMES = ("depth", "iters", "hit", "normal", "ao", "rgb8")
ENGINES = (abi.ENGINE_PLAIN_FP64_STRICT, abi.ENGINE_PLAIN_FP64, abi.ENGINE_PLAIN_MIXED, abi.ENGINE_WAVEFRONT_FP32,
           abi.ENGINE_WAVEFRONT_FP64, abi.ENGINE_WAVEFRONT_AUTO)


def with_fast_ao(p, quality=4, tune=1.0):
    p.ao_rays = 0
    p.ao_fast = 1
    p.ao_quality = quality
    p.ao_fast_tune = tune
    p.ambient_intensity = 0.5
    return p


def ao_error(g, o):
    both = g["hit"].astype(bool) & o["hit"].astype(bool)
    return np.abs(g["ao"][both].astype(np.float64) - o["ao"][both].astype(np.float64))


@pytest.mark.parametrize("quality,tune", [(4, 1.0), (3, 0.6)])
def test_fast_ao_mandelbox(renderer, oracle, quality, tune):
    sc, cam, p = configs.mandelbox_1080p("A", 160, 90, ao_rays=0)
    with_fast_ao(p, quality, tune)
    renderer.set_scene(sc)
    o, ost = oracle.render(sc, cam, p)
    hits = o["hit"].astype(bool)
    assert ost["ao_evals"] == int(hits.sum()) * (quality * quality - 1)
    assert np.ptp(o["ao"][hits]) > 0.1
    for engine in ENGINES:
        fr = renderer.render(cam, p, engine, outputs=NAMES)
        g = {k: v.cpu().numpy() for k, v in fr.buffers.items()}
        m = compare(g, o)
        err = ao_error(g, o)
        print(quality, tune, abi.ENGINE_NAMES[engine], m, "ao err p99", np.quantile(err, 0.99))
        if engine == abi.ENGINE_PLAIN_FP64_STRICT:
            for k in NAMES:
                assert np.array_equal(g[k], o[k]), k
            assert fr.stats == ost
        elif engine in (abi.ENGINE_PLAIN_FP64, abi.ENGINE_WAVEFRONT_FP64):
            assert m["hit_iters_match"] >= 0.999, m
            assert np.quantile(err, 0.99) <= 1e-6
        else:
            assert m["hit_mismatch"] <= 0.005, m
            assert np.quantile(err, 0.99) <= 1e-4
        if engine != abi.ENGINE_PLAIN_FP64_STRICT:
            # every hit takes its quality^2 - 1 samples on every engine
            assert fr.stats["ao_evals"] == int(g["hit"].sum()) * (quality * quality - 1)


def test_fast_ao_mandelbulb(renderer, oracle):
    sc, cam, p = configs.mandelbulb_512(128, 128)
    with_fast_ao(p)
    renderer.set_scene(sc)
    o, _ = oracle.render(sc, cam, p)
    for engine in ENGINES:
        fr = renderer.render(cam, p, engine, outputs=NAMES)
        g = {k: v.cpu().numpy() for k, v in fr.buffers.items()}
        m = compare(g, o)
        err = ao_error(g, o)
        print("bulb", abi.ENGINE_NAMES[engine], m, "ao err p99", np.quantile(err, 0.99))
        if engine in (abi.ENGINE_PLAIN_FP64_STRICT, abi.ENGINE_PLAIN_FP64, abi.ENGINE_WAVEFRONT_FP64):
            assert m["hit_iters_match"] >= 0.999, m
            assert np.quantile(err, 0.99) <= 1e-6
        else:
            assert m["hit_mismatch"] <= 0.005, m
            assert np.quantile(err, 0.99) <= 1e-4
        assert m["psnr"] >= 35.0, m


def test_fast_ao_quality_out_of_range_is_refused(renderer):
    from mandelbulber2_b200.render import MbrError

    sc, cam, p = configs.mandelbox_1080p("A", 32, 18, ao_rays=0)
    with_fast_ao(p, quality=11)
    renderer.set_scene(sc)
    with pytest.raises(MbrError) as e:
        renderer.render(cam, p, abi.ENGINE_PLAIN_FP64)
    assert e.value.status == abi.MBR_EINVAL
