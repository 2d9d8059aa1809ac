"""Writes profiles/opcount.json: algorithmic operations per formula iteration
of each benchmark formula, counted by the op-counting instantiation of the
oracle over whole CalculateDistance evaluations at near-surface points (the
hit points of a small render, jittered by up to 2 % of the depth).

flops_per_iteration = essential (adds + muls) / sum of iters, where the
essential count leaves out operations on a structural zero (the unused 4-D
component w when the initial w is 0, a zero Mandelbox offset);
flops_per_iteration_as_written counts every operation of the reference's
code as written.  Divisions, square roots
and transcendental calls are reported per iteration separately (SFU work, not
folded into flops).  Run: python oracle/make_opcount.py
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from mandelbulber2_b200 import configs  # noqa: E402
from oracle.oracle import Oracle  # noqa: E402

OUT = os.path.join(ROOT, "profiles", "opcount.json")


def near_surface_points(o: Oracle, sc, cam, p, n=4000, seed=0):
    b, _ = o.render(sc, cam, p, outputs=("depth", "hit"))
    hit = b["hit"] > 0
    ys, xs = np.divmod(np.nonzero(hit)[0], cam.width)
    pts = np.array([o.view(cam, int(x), int(y)) for x, y in zip(xs, ys)])
    depth = b["depth"][hit]
    pts = np.array(cam.camera[:]) + pts * depth[:, None]
    rng = np.random.default_rng(seed)
    idx = rng.integers(0, len(pts), size=n)
    return pts[idx] + rng.normal(scale=0.02 * depth[idx, None] / 3.0, size=(n, 3))


def table() -> dict:
    o = Oracle("strict")
    out = {}
    cases = {
        "mandelbox": configs.mandelbox_1080p("A", 64, 36, ao_rays=0),
        "mandelbulb": configs.mandelbulb_512(48, 48),
        "menger": (configs.menger_scene(),) + configs.mandelbulb_512(48, 48)[1:],
        "hybrid": (configs.hybrid_scene(),) + configs.mandelbulb_512(48, 48)[1:],
    }
    for name, (sc, cam, p) in cases.items():
        pts = near_surface_points(o, sc, cam, p)
        c = o.opcount_de(sc, pts, 1e-3)
        it = c["iters"]
        out[name] = {"flops_per_iteration": (c["e_add"] + c["e_mul"]) / it,
                     "flops_per_iteration_as_written": (c["add"] + c["mul"]) / it, "div_per_iteration": c["div"] / it,
                     "sqrt_per_iteration": c["sqrt"] / it, "transcendental_per_iteration": c["transc"] / it,
                     "iterations_per_de_eval": it / c["evals"], "points": c["evals"]}
    return out


if __name__ == "__main__":
    t = table()
    with open(OUT, "w") as f:
        json.dump(t, f, indent=1, sort_keys=True)
    print(json.dumps(t, indent=1))
