"""Autotuner of the step's launch parameters, by timing the scene itself.

Three knobs decide how a scene maps onto the GPU and have no single best
value across scenes:

  pd_lanes      threads per node in the bond loop (mixed form 1, 2, 4;
                FP64 form 4, 8, 32): few bonds per node favour one thread per
                node, many bonds favour a group sharing a node's row
  tile_nodes    nodes per bond-loop tile (the unit a persistent CTA claims and
                stages into shared memory): small tiles balance uneven
                particles, large tiles amortise the staging
  contact_lanes threads per node of the contact pass (1, 2, 4, 8): a loaded
                packing has few candidates per node, and the pass is bound
                by the latency of its gathers, so fewer lanes keep more nodes
                in flight
  search_factor the contact search radius in contact radii (the skin): a
                larger skin rebuilds the candidate lists less often but makes
                every contact pass scan longer lists

The tuner runs coordinate descent: bond-loop lanes x tile size on the
scene's own skin, then the contact lanes, then the skin.  Each candidate is
a fresh GpuDEMModel of the scene (the launch geometry is fixed at set-up),
started from the scene's initial state or, when a state snapshot is given
(pdgpu_save_state of a run of the same scene), from that state, stepped
through its CUDA graph for ``warmup`` steps and then timed over ``steps``
steps with CUDA events on the model's stream; ``steps`` should span several
rebuilds so that the skin's trade-off is seen.  The returned choice is what a
run passes to GpuDEMModel (pd_lanes, tile_nodes, contact_lanes) and to the
scene (search_factor).
"""
from __future__ import annotations

import copy
import dataclasses
from typing import Dict, List, Optional, Sequence

LANES = {"mixed": (1, 2, 4), "fp64": (4, 8, 32)}
TILES = (128, 256, 512, 1024)
CONTACT_LANES = (1, 2, 4, 8)
SKINS = (2.0, 3.0, 5.0)
DEFAULT_CONTACT_LANES = 1


@dataclasses.dataclass
class Choice:
    pd_lanes: int
    tile_nodes: int
    search_factor: float
    ms_per_step: float
    table: List[Dict]
    contact_lanes: int = DEFAULT_CONTACT_LANES


def time_candidate(scene, precision: int, pd_lanes: int, tile_nodes: int, steps: int, warmup: int,
                   device: int = 0, contact_lanes: int = 0, state: Optional[str] = None) -> float:
    """Milliseconds per step of ``scene`` with the given launch parameters
    (graph replay, one step per launch, CUDA events on the model's stream),
    from the scene's start or from the state snapshot ``state``."""
    import torch
    from . import api
    from .model import GpuDEMModel
    m = GpuDEMModel(scene, precision=precision, device=device, build_neighbors=True, compute_mx=True,
                    pd_lanes=pd_lanes, tile_nodes=tile_nodes)
    try:
        if contact_lanes:
            api.set_lanes(m, 0, contact_lanes)
        if state:
            m.load_state(state)
        else:
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
             log=None, contact_lanes: Sequence[int] = (), state: Optional[str] = None) -> Choice:
    """Choose (pd_lanes, tile_nodes, contact lanes, search_factor) for
    ``scene`` by timing, from its start or from the snapshot ``state``."""
    from .model import PREC_MIXED
    lanes = lanes or LANES["mixed" if precision == PREC_MIXED else "fp64"]
    table = []

    def run(sc, ln, tn, sf, cl):
        ms = time_candidate(sc, precision, ln, tn, steps, warmup, device, contact_lanes=cl, state=state)
        row = {"pd_lanes": ln, "tile_nodes": tn, "search_factor": sf, "contact_lanes": cl,
               "ms_per_step": round(ms, 5)}
        table.append(row)
        if log:
            log(row)
        return ms

    sf0 = float(scene.search_factor)
    cl0 = DEFAULT_CONTACT_LANES
    best = None
    for ln in lanes:
        for tn in tiles:
            ms = run(scene, ln, tn, sf0, cl0)
            if best is None or ms < best[3]:
                best = (ln, tn, sf0, ms, cl0)
    for cl in contact_lanes:
        if cl == cl0:
            continue
        ms = run(scene, best[0], best[1], sf0, cl)
        if ms < best[3]:
            best = (best[0], best[1], sf0, ms, cl)
    for sf in skins:
        if sf == sf0:
            continue
        sc = copy.copy(scene)
        sc.search_factor = float(sf)
        ms = run(sc, best[0], best[1], sf, best[4])
        if ms < best[3]:
            best = (best[0], best[1], float(sf), ms, best[4])
    return Choice(best[0], best[1], best[2], best[3], table, best[4])
