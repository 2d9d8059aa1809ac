"""Partition of render work over GPUs: one process per GPU, no collective on
the data path (the reference distributes image lines over threads,
src/scheduler.cpp:122-247, and frames or lines over machines, netrender_*.cpp).

  row_band(height, world, rank)      a contiguous band of one frame per rank
  deal_jobs(costs, world)            batch jobs per rank, longest cost first,
                                     each to the least loaded rank
  job_cost(width, height, formula)   the cost model used to deal jobs
  band_params(params, r0, r1)        render parameters restricted to a band

Only the assembly of a sharded frame (gather of the bands) and the timing
reduction (max over ranks) cross GPUs.
"""
from __future__ import annotations

import ctypes as C
import heapq

from . import abi

# relative cost per pixel of a formula, measured DE work of the benchmark scenes
FORMULA_COST = {abi.FORMULA_MANDELBULB: 1.0, abi.FORMULA_MANDELBOX: 1.6, abi.FORMULA_MENGER_SPONGE: 0.6}


def row_band(height: int, world: int, rank: int) -> tuple[int, int]:
    """Rows [r0, r1) of `rank`: bands differ in size by at most one row."""
    if not (0 <= rank < world) or world < 1:
        raise ValueError("rank outside the world")
    base, extra = divmod(height, world)
    r0 = rank * base + min(rank, extra)
    return r0, r0 + base + (1 if rank < extra else 0)


def job_cost(width: int, height: int, formula: int) -> float:
    return float(width * height) * FORMULA_COST.get(formula, 1.0)


def deal_jobs(costs, world: int) -> list[list[int]]:
    """Longest-processing-time dealing: jobs by decreasing cost, each to the
    rank with the least work so far (makespan <= 4/3 of the optimum)."""
    heap = [(0.0, r) for r in range(world)]
    heapq.heapify(heap)
    out = [[] for _ in range(world)]
    for j in sorted(range(len(costs)), key=lambda i: -costs[i]):
        load, r = heapq.heappop(heap)
        out[r].append(j)
        heapq.heappush(heap, (load + costs[j], r))
    for lst in out:
        lst.sort()
    return out


def band_params(params: abi.RenderParams, r0: int, r1: int) -> abi.RenderParams:
    p = abi.RenderParams()
    C.memmove(C.addressof(p), C.addressof(params), C.sizeof(p))
    p.row_begin, p.row_end = r0, r1
    return p
