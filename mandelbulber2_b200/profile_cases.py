"""Small named render cases for profiling one kernel at a time (ncu -k ...).

  python -m mandelbulber2_b200.profile_cases <case>

cases: plain_fp64, plain_strict, plain_mixed, wavefront, wavefront64
(Mandelbox s=-1.5, 960x540, camera A, 16 AO rays; two frames; wavefront64
iterates in FP64), gi and gi_wavefront (hybrid Mandelbulb/Menger 480x270,
2 spp, on the plain mixed kernel and on the wavefront), hybrid_wavefront (the
hybrid fractal, 480x270, Lambert + shadow + 4 AO rays), adjoint
(Mandelbulb 256x256 forward + FP64 adjoint), distance (CalculateDistance at
2^20 random points).
"""
from __future__ import annotations

import sys

import torch

from . import abi, configs
from .render import STATS_FIELDS, Renderer, alloc_outputs

FRAME_ENGINES = {"plain_fp64": abi.ENGINE_PLAIN_FP64, "plain_strict": abi.ENGINE_PLAIN_FP64_STRICT,
                 "plain_mixed": abi.ENGINE_PLAIN_MIXED, "wavefront": abi.ENGINE_WAVEFRONT_FP32,
                 "wavefront64": abi.ENGINE_WAVEFRONT_FP64}


def frame(r: Renderer, sc, cam, p, engine: int, reps: int = 2) -> dict:
    r.set_scene(sc)
    bufs = alloc_outputs(cam.width * cam.height, r.device, ("depth", "iters", "hit", "normal", "rgb8"))
    st = torch.zeros(len(STATS_FIELDS), dtype=torch.int64, device=r.device)
    for _ in range(reps):
        r.render_into(cam, p, bufs, st, engine)
    r.sync()
    return bufs


def run(case: str) -> None:
    r = Renderer(0)
    if case in FRAME_ENGINES:
        sc, cam, p = configs.mandelbox_1080p("A", 960, 540)
        frame(r, sc, cam, p, FRAME_ENGINES[case])
    elif case in ("gi", "gi_wavefront"):
        sc, cam, p = configs.hybrid_gi_2160p(480, 270, spp=2)
        frame(r, sc, cam, p, abi.ENGINE_PLAIN_MIXED if case == "gi" else abi.ENGINE_WAVEFRONT_FP32, reps=1)
    elif case == "hybrid_wavefront":
        sc = configs.hybrid_scene()
        cam = configs.camera((0.0, -3.0, 0.5), width=480, height=270)
        p = configs.base_params(5, 20.0)
        p.ao_rays = 4
        frame(r, sc, cam, p, abi.ENGINE_WAVEFRONT_FP32)
    elif case == "adjoint":
        sc, cam, p = configs.adjoint_256("mandelbulb", 256, 256)
        b = frame(r, sc, cam, p, abi.ENGINE_PLAIN_MIXED, reps=1)
        w = torch.ones(cam.width * cam.height, dtype=torch.float32, device=r.device)
        r.adjoint(cam, p, b["depth"], b["hit"], w, w, abi.ENGINE_PLAIN_FP64)
    elif case == "distance":
        r.set_scene(configs.mandelbox_scene())
        pts = torch.rand(1 << 20, 3, dtype=torch.float64, device=r.device) * 6 - 3
        r.distance(pts, 1e-3, False, abi.ENGINE_PLAIN_FP64)
    else:
        raise SystemExit(f"unknown case {case}")
    r.close()
    print("ok", case)


if __name__ == "__main__":
    run(sys.argv[1])
