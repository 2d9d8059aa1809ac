"""Multi-GPU partition logic on CPU: world-size-2 gloo process groups render
their shares with the oracle and the gathered result equals the whole; the
bench's max-over-ranks timing reduction; job dealing."""
import os
import tempfile

import numpy as np
import pytest
import torch.multiprocessing as mp

from mandelbulber2_b200 import configs
from mandelbulber2_b200.shard import deal_jobs, job_cost, row_band


def test_row_bands_cover_the_frame():
    for h in (1, 7, 1080, 2160):
        for world in (1, 2, 3, 8):
            bands = [row_band(h, world, r) for r in range(world)]
            assert bands[0][0] == 0 and bands[-1][1] == h
            assert all(a[1] == b[0] for a, b in zip(bands, bands[1:]))
            sizes = [b - a for a, b in bands]
            assert max(sizes) - min(sizes) <= 1


def test_deal_jobs_balances_and_covers():
    rng = np.random.default_rng(7)
    costs = [job_cost(int(s), int(s), int(f)) for s, f in zip(rng.choice([64, 128, 256, 512, 1024], 2048),
                                                                 rng.choice([2, 8], 2048))]
    for world in (2, 4, 8):
        parts = deal_jobs(costs, world)
        assert sorted(j for p in parts for j in p) == list(range(len(costs)))
        loads = [sum(costs[j] for j in p) for p in parts]
        assert max(loads) <= (sum(costs) / world) * 4 / 3 + max(costs)


def _rank(rank, world, init, outdir):
    import torch
    import torch.distributed as dist

    from oracle.oracle import Oracle

    dist.init_process_group("gloo", init_method=init, rank=rank, world_size=world)
    sc, cam, p = configs.mandelbox_1080p("A", 48, 27, ao_rays=4)
    r0, r1 = row_band(cam.height, world, rank)
    bufs, st = Oracle("strict").render(sc, cam, p, rows=(r0, r1), threads=1)
    # gather the bands (the assembly step; nothing else crosses ranks)
    parts = [None] * world
    dist.all_gather_object(parts, {k: v for k, v in bufs.items()})
    # the bench's timing reduction: max over ranks
    t = torch.tensor([float(rank + 1)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    de = torch.tensor([float(st["de_evals"])], dtype=torch.float64)
    dist.all_reduce(de)
    if rank == 0:
        whole = {k: np.concatenate([pp[k] for pp in parts]) for k in parts[0]}
        np.savez(os.path.join(outdir, "gathered.npz"), **whole, tmax=t.numpy(), de=de.numpy())
    dist.barrier()
    dist.destroy_process_group()


def test_gloo_two_ranks_render_bands(oracle):
    with tempfile.TemporaryDirectory() as d:
        init = "file://" + os.path.join(d, "pg")
        mp.start_processes(_rank, args=(2, init, d), nprocs=2, join=True, start_method="spawn")
        g = np.load(os.path.join(d, "gathered.npz"))
        sc, cam, p = configs.mandelbox_1080p("A", 48, 27, ao_rays=4)
        whole, st = oracle.render(sc, cam, p, threads=1)
        for k in whole:
            assert np.array_equal(g[k], whole[k]), k
        assert g["tmax"][0] == 2.0
        assert g["de"][0] == st["de_evals"]
