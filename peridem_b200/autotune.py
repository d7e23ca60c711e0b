"""Autotuner of the step's launch parameters, by timing the scene itself.

Three knobs decide how a scene maps onto the GPU and have no single best
value across scenes:

  pd_lanes      threads per node in the bond loop (mixed form 1, 2, 4;
                FP64 form 4, 8, 32): few bonds per node favour one thread per
                node, many bonds favour a group sharing a node's row
  tile_nodes    nodes per bond-loop tile (the unit a persistent CTA claims and
                stages into shared memory): small tiles balance uneven
                particles, large tiles amortise the staging
  search_factor the contact search radius in contact radii (the skin): a
                larger skin rebuilds the candidate lists less often but makes
                every contact pass scan longer lists

The tuner runs coordinate descent: lanes x tile size on the scene's own skin,
then the skin with the best pair.  Each candidate is a fresh GpuDEMModel of
the scene (the launch geometry is fixed at set-up), stepped through its CUDA
graph for ``warmup`` steps and then timed over ``steps`` steps with CUDA
events on the model's stream; ``steps`` should span several rebuilds so that
the skin's trade-off is seen.  The returned choice is what a run passes to
GpuDEMModel (pd_lanes, tile_nodes) and to the scene (search_factor).
"""
from __future__ import annotations

import copy
import dataclasses
from typing import Dict, List, Optional, Sequence

LANES = {"mixed": (1, 2, 4), "fp64": (4, 8, 32)}
TILES = (128, 256, 512, 1024)
SKINS = (2.0, 3.0, 5.0)


@dataclasses.dataclass
class Choice:
    pd_lanes: int
    tile_nodes: int
    search_factor: float
    ms_per_step: float
    table: List[Dict]


def time_candidate(scene, precision: int, pd_lanes: int, tile_nodes: int, steps: int, warmup: int,
                   device: int = 0) -> float:
    """Milliseconds per step of ``scene`` with the given launch parameters
    (graph replay, one step per launch, CUDA events on the model's stream)."""
    import torch
    from .model import GpuDEMModel
    m = GpuDEMModel(scene, precision=precision, device=device, build_neighbors=True, compute_mx=True,
                    pd_lanes=pd_lanes, tile_nodes=tile_nodes)
    try:
        m.integrate_begin()
        stream = torch.cuda.ExternalStream(m.stream_handle(), device=device)
        for _ in range(warmup):
            m.integrate_step(1, graph_steps=1)
        m.sync()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(steps):
            m.integrate_step(1, graph_steps=1)
        b.record(stream)
        m.sync()
        b.synchronize()
        return a.elapsed_time(b) / steps
    finally:
        m.close()


def autotune(scene, precision: int, steps: int = 200, warmup: int = 20, lanes: Optional[Sequence[int]] = None,
             tiles: Sequence[int] = TILES, skins: Sequence[float] = SKINS, device: int = 0,
             log=None) -> Choice:
    """Choose (pd_lanes, tile_nodes, search_factor) for ``scene`` by timing."""
    from .model import PREC_MIXED
    lanes = lanes or LANES["mixed" if precision == PREC_MIXED else "fp64"]
    table = []

    def run(sc, ln, tn, sf):
        ms = time_candidate(sc, precision, ln, tn, steps, warmup, device)
        row = {"pd_lanes": ln, "tile_nodes": tn, "search_factor": sf, "ms_per_step": round(ms, 5)}
        table.append(row)
        if log:
            log(row)
        return ms

    sf0 = float(scene.search_factor)
    best = None
    for ln in lanes:
        for tn in tiles:
            ms = run(scene, ln, tn, sf0)
            if best is None or ms < best[3]:
                best = (ln, tn, sf0, ms)
    for sf in skins:
        if sf == sf0:
            continue
        sc = copy.copy(scene)
        sc.search_factor = float(sf)
        ms = run(sc, best[0], best[1], sf)
        if ms < best[3]:
            best = (best[0], best[1], float(sf), ms)
    return Choice(best[0], best[1], best[2], best[3], table)
