"""Cell-parallel runs of many independent cells over the ranks of a process
group (one rank per GPU).

The cells share nothing, so no collective runs inside an SD step: each rank
steps its share of the cells together, one CUDA graph launch per SD step
(``api.GpuBatch``), and the only exchange is the gather of the energies at
the end.  Work is split by the longest-processing-time rule on a cost model
dominated by the transforms (n^3 log n per band), so uneven cells (grids
32^3 to 64^3, 4 to 32 bands) still give every rank about the same load.
"""
from __future__ import annotations

import math
from typing import Callable, List, Optional, Sequence

import numpy as np


def cell_cost(spec) -> float:
    """Relative cost of one SD step of a cell: its 3-D transforms."""
    n = spec.nfft
    return float(n ** 3 * math.log2(n) * (spec.ne[0] + (spec.ne[1] if spec.ispin == 2 else 0)))


def assign(specs: Sequence, world: int) -> List[List[int]]:
    """Cell indices per rank: cells by decreasing cost (ties by index) each
    go to the least-loaded rank so far (ties to the lower rank).  Every cell
    lands on exactly one rank; each rank's list is in increasing order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(specs)), key=lambda i: (-cell_cost(specs[i]), i))
    load = [0.0] * world
    out: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(i)
        load[r] += cell_cost(specs[i])
    return [sorted(x) for x in out]


def gpu_runner(specs: Sequence, calls: int, inner: int) -> np.ndarray:
    """E[0..9] of each cell after `calls` batched cpsd() calls of `inner`
    SD steps on this process's current GPU."""
    from . import api, inputs
    cells = []
    try:
        for spec in specs:
            inp = inputs.build_inputs(spec)
            c = api.GpuCell(inp)
            c.set_state(inp.c2, inp.r2)
            cells.append(c)
        if not cells:
            return np.zeros((0, 10))
        batch = api.GpuBatch(cells)
        try:
            for _ in range(calls):
                batch.run(inner)
            return batch.E.copy()
        finally:
            batch.close()
    finally:
        for c in cells:
            c.close()


def run_cells(specs: Sequence, calls: int, inner: int, rank: int = 0, world: int = 1, dist=None,
              runner: Optional[Callable] = None) -> np.ndarray:
    """E[cell][0..9] of all cells after `calls` calls of `inner` steps, each
    rank stepping its share (``assign``) with ``runner`` (``gpu_runner`` by
    default); with a process group ``dist`` (torch.distributed) the shares
    are gathered, and every rank returns the full array in cell order."""
    runner = runner or gpu_runner
    mine = assign(specs, world)[rank]
    if mine:
        local = np.asarray(runner([specs[i] for i in mine], calls, inner), dtype=np.float64).reshape(len(mine), -1)
    else:
        # more ranks than cells: this rank runs nothing but still joins the gather
        local = np.zeros((0, 10))
    if dist is None or world == 1:
        parts = [(mine, local)]
    else:
        parts = [None] * world
        dist.all_gather_object(parts, (mine, local))
    width = max((p[1].shape[1] for p in parts if len(p[0])), default=10)
    E = np.full((len(specs), width), np.nan)
    for idx, e in parts:
        for k, i in enumerate(idx):
            E[i] = e[k]
    if np.isnan(E).any():
        raise RuntimeError("a cell was not run by any rank")
    return E
