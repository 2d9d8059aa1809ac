"""The oracle's fast ambient occlusion (FastAmbientOcclusion,
shader_fast_ambient_occlusion.cpp:40-65), on the CPU: quality^2 - 1 distance
estimates per hit, an occlusion factor clamped at 0 (not at 1: a sample whose
distance exceeds its scan distance adds a negative term, as in the reference)
that is lower in creases than on open surfaces, and the quality and fast tune
changing it."""
import numpy as np

from mandelbulber2_b200 import configs


def small(quality=4, tune=1.0):
    sc, cam, p = configs.mandelbox_1080p("A", 48, 27, ao_rays=0)
    p.ao_fast = 1
    p.ao_quality = quality
    p.ao_fast_tune = tune
    p.ambient_intensity = 0.5
    return sc, cam, p


def test_fast_ao_counts_and_range(oracle):
    sc, cam, p = small()
    o, st = oracle.render(sc, cam, p)
    hits = o["hit"].astype(bool)
    assert 0.05 < hits.mean() < 0.99
    assert st["ao_evals"] == int(hits.sum()) * (4 * 4 - 1)
    ao = o["ao"][hits]
    assert np.all((ao >= 0.0) & (ao < 1.5))
    assert ao.max() - ao.min() > 0.1  # creases are darker than open surfaces
    assert np.all(o["ao"][~hits] == 1.0)


def test_fast_ao_quality_and_tune(oracle):
    o4, _ = oracle.render(*small(4, 1.0))
    o2, st2 = oracle.render(*small(2, 1.0))
    ot, _ = oracle.render(*small(4, 0.5))
    hits = o4["hit"].astype(bool)
    assert st2["ao_evals"] == int(hits.sum()) * 3
    assert np.mean(o4["ao"][hits] != o2["ao"][hits]) > 0.5
    # a smaller tune counts less of the measured distance: more occlusion
    assert np.all(ot["ao"][hits] <= o4["ao"][hits])
    assert np.mean(ot["ao"][hits] < o4["ao"][hits]) > 0.5


def test_quality_one_takes_no_samples(oracle):
    o, st = oracle.render(*small(1, 1.0))
    assert st["ao_evals"] == 0
    assert np.all(o["ao"] == 1.0)
