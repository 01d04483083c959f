"""Autotuner for the neighbour passes: picks the threads per block, the pair
lanes per particle, the grid cell size (h or h/2 with a 5x5x5 stencil) and
whether each pass is one persistent launch (resident blocks striding over all
tiles of slots) of a workload by timing each candidate on the GPU from the same
initial state, and caches the choice.

The candidates change the launch shape, the neighbour-list order and the FP32
summation order (pair lanes), never the neighbour sets (test_gpu_batch.py checks
the sets for cells of h/2); every candidate is bit-exact with the oracle run
with the same settings.
"""
from __future__ import annotations

import json
import math
import os
from typing import Optional, Sequence

CANDIDATES = [(cs, bs, ln, ps) for cs in (1.0, 0.5) for bs in (64, 128, 256) for ln in (1, 2, 4) for ps in (0, 1)]


def dims_for_scale(dims: Sequence[int], cell_scale: float) -> list:
    """Grid cells per axis covering the same extent with cells of h * cell_scale."""
    return [int(math.ceil(d / cell_scale - 1e-9)) for d in dims]


def signature(scenes, iterations: int) -> str:
    n = sum(s.n for s in scenes)
    return f"scenes={len(scenes)}:n={n}:h={float(scenes[0].para.h):.6g}:it={iterations}"


def ext_for(tuned: dict) -> dict:
    """Ext overrides of a tuning result (grid_dims excluded: they are per scene)."""
    return {"cell_scale": tuned["cell_scale"], "block_size": tuned["block_size"], "pair_lanes": tuned["pair_lanes"],
            "persistent": tuned.get("persistent", 0)}


def _time_candidate(scenes, iterations, cell_scale, block, lanes, persistent, substeps, warm):
    import torch

    from . import scenes as S
    from .solver import BatchSolver, Solver
    scs = list(scenes)
    if len(scs) == 1:
        sc = scs[0]
        dims = dims_for_scale(sc.ext_overrides["grid_dims"], cell_scale)
        s = Solver(sc.para, sc.grid_space, sc.boundary,
                   sc.ext(grid_dims=dims, cell_scale=cell_scale, block_size=block, pair_lanes=lanes,
                          persistent=persistent))
        s.upload(sc.pos, sc.vel)
    else:
        para, descs, ov, pos, vel = S.batch_inputs(scs, iterations=iterations)
        for d in descs:
            d["grid_dims"] = dims_for_scale(d["grid_dims"], cell_scale)
        ov.update(cell_scale=cell_scale, block_size=block, pair_lanes=lanes, persistent=persistent)
        s = BatchSolver(para, descs, S.default_ext(**ov))
        s.upload(pos, vel)
    st = torch.cuda.current_stream()
    s.step(warm, st)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(st)
    s.step(substeps, st)
    b.record(st)
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / substeps
    s.close()
    return ms


TIE = 0.01  # candidates within 1 % of the fastest are a tie (the timing's run-to-run spread)


def pick(table: list) -> dict:
    """The fastest row of a timing table, preferring one-block-per-tile launches
    (persistent 0) among the rows within TIE of the fastest: a persistent launch
    is chosen only when it is faster by more than the spread."""
    best = min(r["ms_per_substep"] for r in table)
    pool = [r for r in table if r["ms_per_substep"] <= best * (1.0 + TIE)]
    plain = [r for r in pool if not r.get("persistent", 0)]
    return min(plain or pool, key=lambda r: r["ms_per_substep"])


def tune(scenes, iterations: int = 4, substeps: int = 6, warm: int = 2, candidates=None,
         cache_path: Optional[str] = None) -> dict:
    """Times every (cell_scale, block_size, pair_lanes, persistent) candidate and
    returns the fastest: {"cell_scale", "block_size", "pair_lanes", "persistent",
    "ms_per_substep", "table"}."""
    key = signature(scenes, iterations)
    if cache_path and os.path.exists(cache_path):
        with open(cache_path) as f:
            cache = json.load(f)
        if key in cache:
            return cache[key]
    table = []
    for cand in candidates or CANDIDATES:
        cs, bs, ln = cand[:3]
        ps = cand[3] if len(cand) > 3 else 0
        table.append({"cell_scale": cs, "block_size": bs, "pair_lanes": ln, "persistent": ps,
                      "ms_per_substep": _time_candidate(scenes, iterations, cs, bs, ln, ps, substeps, warm)})
    out = dict(pick(table))
    out["table"] = table
    if cache_path:
        cache = {}
        if os.path.exists(cache_path):
            with open(cache_path) as f:
                cache = json.load(f)
        cache[key] = out
        os.makedirs(os.path.dirname(os.path.abspath(cache_path)), exist_ok=True)
        with open(cache_path, "w") as f:
            json.dump(cache, f, indent=1)
    return out
