#!/usr/bin/env python
"""Benchmark: node-steps/s of the PeriDEM explicit step on B200.

Workload (default): the 2-D compressive test — 502 discs and hexagons
(50/50), radius U[1, 1.5] mm, random orientation, h = R/15 scaled per
particle, horizon 3h, RNPBond (E = 2 GPa, nu = 0.25, rho = 1200, Gc = 500),
fixed frame plus a top wall pressing at 0.1 m/s, seeded synthetic packing.

A step is one DEMModel::integrateStep over the whole scene (integrate,
displacement BC, peridynamic bond loop, contact-list control and rebuilds,
contact forces, particle damping, external forces, post-processing).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--precision mixed|fp64]
                  [--impl ours|reference]

Timing: W untimed steps, then K steps each timed with CUDA events on the
model's stream, with a 512 MiB buffer written and then read back between
steps to flush the 126 MB L2 (the read leaves it clean); max over ranks.
N > 1 runs N independent replicas (one scene per GPU, no collective), so
scaling is weak.
"""
import argparse
import glob
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "node-steps/s on 1 B200: mixed+surrogate vs plain FP64 at ≤1e-3 wall-force err"
UNIT = "node-steps/s"


def workload_spec(args):
    """The deck the reference's CPU run times: the scene itself, or for an
    ensemble its first scene (the reference runs one scene per process)."""
    from peridem_b200 import scene as scn
    if args.workload == "ensemble":
        return scn.ensemble_specs(n_scenes=args.scenes, seed=args.seed)[0]
    if args.workload == "column3d":
        # bounded CPU sample: 8 spheres of the same size distribution and mesh
        return scn.column_3d(n_spheres=8, median_r=2e-3, h_div=10, seed=args.seed)
    if args.workload == "surrogate":
        return scn.compressive_2d(n_particles=2000, r_range=(1e-3, 1.5e-3), h_div=15, width=80e-3,
                                  seed=args.seed, material="RNPBond", wall_speed=-0.1, nt=100000)
    # dt = 5e-8 s as configured; the contact spring softened to omega dt = 0.3
    # (scene.stable_kn), since the configured 10x-bulk stiffness blows up at
    # this step in the reference itself (tests/test_reference_stability.py)
    return scn.compressive_2d(n_particles=args.particles, r_range=(1e-3, 1.5e-3), h_div=15,
                              width=40e-3, seed=args.seed, material="RNPBond", wall_speed=-0.1,
                              dt=5e-8, nt=50000, packing="deposit")


def build_workload(args):
    from peridem_b200 import scene as scn
    if args.workload == "ensemble":
        return scn.merge_scenes(scn.build_scenes(scn.ensemble_specs(n_scenes=args.scenes, seed=args.seed)))
    if args.workload == "surrogate":
        return scn.build_scene(workload_spec(args))
    if args.workload == "column3d":
        # median radius 2 mm: at 1 mm and h = R/10 the smaller spheres' weighted
        # volume m_x falls under the reference's absolute 1e-18 guard
        # (materialUtil.cpp:57) and the reference rejects the scene; node and
        # bond counts per sphere do not depend on the scale
        return scn.build_scene(scn.column_3d(n_spheres=args.spheres, median_r=2e-3, h_div=10, seed=args.seed,
                                             footprint=(16, 16), wall_h=2e-4, wall_layers=2.0))
    return scn.build_scene(workload_spec(args))


def workload_config(args, sc):
    if args.workload == "ensemble":
        head = {"workload": "batched ensemble: %d independent 2-D compression scenes in one model, particles "
                            "U[20,200] per scene, discs/hexagons R~U[0.8,1.6] mm, h=R/U{8..16}, horizon 3h, "
                            "RNPBond, top-wall speed U[0.05,0.2] m/s per scene, shared dt" % args.scenes,
                "scenes": args.scenes,
                "particles": int(sc.n_particles) if sc is not None else None}
    elif args.workload == "surrogate":
        head = {"workload": "surrogate form of the 2-D compressive test scaled to 2000 particles: discs/hexagons "
                            "R~U[1,1.5] mm, h=R/15, horizon 3h, RNPBond, top wall 0.1 m/s; per shape rank-32 "
                            "modes, MLP 32-256-256-32 (BF16, FP32 accumulate), full bond-loop check every 50 "
                            "steps, stretch, error and contact-proximity gates",
                "particles": 2000}
    elif args.workload == "column3d":
        force = (int(sum(int(sc.p_end[p] - sc.p_start[p]) for p in range(sc.n_particles) if sc.p_compute_force[p]))
                 if sc is not None else None)
        head = {"workload": "3-D granular column: %d spheres, lognormal R (median 2 mm, sigma 0.2), h=R/10 "
                            "(~4200 nodes per sphere), horizon 3h, PDState E=5 GPa, 16x16 lattice footprint, "
                            "box and piston meshed at 0.2 mm, piston 0.05 m/s" % args.spheres,
                "spheres": args.spheres, "sphere_nodes": force}
    else:
        head = {"workload": "2-D compressive test, %d discs/hexagons R~U[1,1.5] mm, h=R/15, "
                            "horizon 3h, RNPBond, top wall 0.1 m/s, seeded ballistic deposition of the "
                            "particles' nodes; timed from the state after an untimed pre-run of the "
                            "compression: %d steps, then 10-step strides until the top wall touches the "
                            "packing" % (args.particles, args.prerun),
                "particles": args.particles, "prerun_steps": args.prerun}
    return head | {"nodes": int(sc.n_nodes) if sc is not None else None,
                   "dt": sc.dt if sc is not None else None,
                   "precision": args.precision, "l2": "flushed between timed steps (512 MiB write, then read back)",
                   "graph_steps_per_launch": args.graph_steps,
                   "pd_lanes": args.pd_lanes or "auto", "tile_nodes": args.tile_nodes or "auto",
                   "contact_lanes": getattr(args, "contact_lanes", 0) or "auto",
                   "search_factor": sc.search_factor if sc is not None else None}


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    """SM clock and throttle reasons polled every 5 ms through NVML while the
    timed region runs (read-only queries; the device is found by PCI bus id,
    so CUDA_VISIBLE_DEVICES remapping does not matter).  Falls back to
    `nvidia-smi -lms 100` when NVML cannot be used."""
    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"))
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.samples = []       # (sm_mhz, max_mhz, set of reasons)
        self.proc = None
        self.nvml = None
        self.stop = threading.Event()

    def __enter__(self):
        try:
            import pynvml
            import torch
            pynvml.nvmlInit()
            p = torch.cuda.get_device_properties(self.device)
            bus = "%08x:%02x:%02x.0" % (p.pci_domain_id, p.pci_bus_id, p.pci_device_id)
            self.h = pynvml.nvmlDeviceGetHandleByPciBusId(bus.encode())
            self.max = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
            self.nvml = pynvml
            self.t = threading.Thread(target=self._poll, daemon=True)
        except Exception:
            self.nvml = None
            try:
                self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device),
                                              "--query-gpu=" + self.Q,
                                              "--format=csv,noheader,nounits", "-lms", "100"],
                                             stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                                             text=True)
                self.t = threading.Thread(target=self._read, daemon=True)
            except OSError:
                self.proc = None
                return self
        self.t.start()
        return self

    def _poll(self):
        nv = self.nvml
        masks = [(n, getattr(nv, m)) for n, m in self.REASONS]
        while not self.stop.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                self.samples.append((float(sm), float(self.max), {n for n, m in masks if r & m}))
            except Exception:
                pass
            self.stop.wait(0.005)

    def _read(self):
        names = [n for n, _ in self.REASONS]
        for ln in self.proc.stdout:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                self.samples.append((float(f[1]), float(f[2]),
                                     {nm for k, nm in enumerate(names)
                                      if f[5 + k].lower().startswith("active")}))
            except ValueError:
                continue

    def __exit__(self, *a):
        self.stop.set()
        if self.nvml:
            self.t.join(timeout=2)
            try:
                self.nvml.nvmlShutdown()
            except Exception:
                pass
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm = sorted(s[0] for s in self.samples)
        reasons = set().union(*[s[2] for s in self.samples]) if self.samples else set()
        return {"sm_mhz": sm[len(sm) // 2] if sm else None,
                "sm_max_mhz": self.samples[-1][1] if self.samples else None,
                "reasons": sorted(reasons), "samples": len(sm),
                "source": "nvml 5 ms" if self.nvml else "nvidia-smi 100 ms"}


# ---------------------------------------------------------------------------
def measured_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def traffic_from_profiles(kernel):
    """DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum)
    that an ncu capture summary in profiles/ recorded for `kernel`, and the
    summary's file name; a recorded figure, not measured by this run."""
    for p in sorted(glob.glob(os.path.join(ROOT, "profiles", "*.md"))):
        with open(p) as fh:
            for line in fh:
                if line.startswith(f"traffic_bytes_per_launch[{kernel}]:"):
                    try:
                        return float(line.split(":", 1)[1].split()[0]), os.path.basename(p)
                    except ValueError:
                        pass
    return None, None


def algorithmic_bytes(kernel, sc, precision):
    """Bytes one launch must move at minimum, counted independently of the
    storage layout: per bond a 32-bit neighbour index and the broken bit; per
    active node its reference coordinates and displacement (FP64, or FP32 in
    the mixed form), volume, row offset and force (FP64) and damage (FP32);
    neighbour data are re-read from cache.  The mixed form's own layout moves
    less (16-bit neighbour columns where a tile's window allows them, FP32
    node records, FP64 displacement)."""
    import numpy as np
    dim = sc.dim
    active = np.zeros(sc.n_nodes, dtype=bool)
    for p in range(sc.n_particles):
        if sc.p_compute_force[p]:
            active[sc.p_start[p]:sc.p_end[p]] = True
    rp = np.asarray(sc.pd_rowptr, dtype=np.int64)
    bonds = int((rp[1:] - rp[:-1])[active].sum())
    nodes = int(active.sum())
    state = bool(np.any(np.asarray(sc.p_material) == 3))  # PDState: m_x and theta per node
    if kernel == "pd_force":
        per_bond, per_node = 4 + 1 / 8, 8 * dim * 3 + 8 + 8 + 4 + (16 if state else 0)
    elif kernel == "pd_force_mixed":
        per_bond, per_node = 4 + 1 / 8, 4 * dim + 4 * dim + 8 + 8 + 8 * dim + 4 + (16 if state else 0)
    else:
        return None, None
    return bonds * per_bond + nodes * per_node, {"bonds": bonds, "nodes": nodes,
                                                  "bytes_per_bond": per_bond,
                                                  "bytes_per_node": per_node}


# ---------------------------------------------------------------------------
def max_over_ranks(x: float, world: int, device: str) -> float:
    """The largest x over the ranks of the process group (x itself on one
    rank): a multi-GPU time is the slowest rank's."""
    if world <= 1:
        return float(x)
    import torch
    t = torch.tensor([float(x)], device=device, dtype=torch.float64)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def job_throughput(nodes: int, steps: int, world: int, max_ms: float) -> float:
    """Whole-job node-steps/s of N independent replicas: every rank advances
    its own scene of `nodes` nodes by `steps` steps; the job takes as long
    as its slowest rank."""
    return nodes * steps * world / (max_ms * 1e-3)


def mixed_error(a, b, steps, every):
    """Error of run a (FP32 bond loop) against run b (plain FP64) over the
    timed window: relative max-norm error of the compressive-test wall
    reaction (the reference's Σ_wall f·vol) and of the contact reaction on
    the wall, over the records of the window's test steps; the broken-bond
    fraction and the fraction of nodes with damage Z >= 1 at the window's
    end (absolute differences); relative max-norm error of u at the end."""
    import numpy as np
    ha, hb = a["hist"], b["hist"]
    rows = []
    for k in range(min(len(ha), len(hb))):
        if abs(ha[k, 0] - hb[k, 0]) > 1e-12 * max(abs(hb[k, 0]), 1e-30):
            raise RuntimeError("compressive-test records of the two runs are not aligned")
        rows.append(k)
    n0, n1 = steps
    dt_rows = [k for k in rows if hb[k, 0] > 0]
    # records are written every `every` steps; the window's are the last ones
    nwin = max(1, (n1 - n0 + 1) // max(every, 1))
    win = dt_rows[-nwin:]
    out = {"records": len(win)}
    for col, key in ((2, "wall_reaction"), (3, "contact_reaction")):
        ref = hb[win, col]
        den = float(np.max(np.abs(ref))) if len(win) else 0.0
        diff = float(np.max(np.abs(ha[win, col] - ref))) if len(win) else 0.0
        out[key + "_max_abs"] = den
        out[key + "_rel_err"] = diff / den if den > 0 else None
    B = max(len(b["bonds"]), 1)
    out["broken_fraction"] = float(b["bonds"].sum()) / B
    out["broken_fraction_abs_err"] = abs(float(a["bonds"].sum()) - float(b["bonds"].sum())) / B
    out["z_ge_1_fraction_abs_err"] = abs(float(np.mean(a["Z"] >= 1.0)) - float(np.mean(b["Z"] >= 1.0)))
    ub = np.abs(b["u"]).max()
    out["u_rel_err"] = float(np.abs(a["u"] - b["u"]).max() / ub) if ub > 0 else None
    return out


def run_ours(args, rank, world):
    import numpy as np
    import torch
    from peridem_b200 import scene as scn
    from peridem_b200.model import GpuDEMModel, PREC_FP64, PREC_MIXED

    dev = int(os.environ.get("LOCAL_RANK", 0))
    torch.cuda.set_device(dev)
    sc = build_workload(args)
    prec = PREC_MIXED if args.precision == "mixed" else PREC_FP64
    # untimed pre-run: the wall presses the packing; every arm starts from
    # the state it reaches (a state snapshot)
    snap, pre_s = None, 0.0
    if args.prerun > 0:
        snap, pre_s, pre_steps, pre_touch = prerun_state(sc, args, dev)
    tuned = None
    if args.autotune:
        from peridem_b200.autotune import autotune, CONTACT_LANES
        t0 = time.perf_counter()
        ch = autotune(sc, prec, steps=args.tune_steps, warmup=5, device=dev, contact_lanes=CONTACT_LANES,
                      state=snap)
        args.pd_lanes, args.tile_nodes, sc.search_factor = ch.pd_lanes, ch.tile_nodes, ch.search_factor
        args.contact_lanes = ch.contact_lanes
        tuned = {"seconds": round(time.perf_counter() - t0, 1), "candidates": ch.table}
    model = GpuDEMModel(sc, precision=prec, device=dev, build_neighbors=True, compute_mx=True,
                        pd_lanes=args.pd_lanes, tile_nodes=args.tile_nodes)
    if args.contact_lanes:
        from peridem_b200 import api
        api.set_lanes(model, 0, args.contact_lanes)
    rp, col = model.pd_neighbors()
    sc.pd_rowptr, sc.pd_col = rp, col
    sur = None
    if args.workload == "surrogate":
        # trained beforehand (not timed) on a 64-particle packing of the same
        # meshes, driven harder so that its trajectory deforms the particles
        # (0.5 m/s: the wall meets the packing after ~9 000 steps and presses
        # it for the rest of the 16 000 without breaking a bond; at 1 m/s the
        # impact breaks bonds, and the internal contact of broken bonds,
        # 18 K / (pi delta^5), is beyond this dt's stability limit: the
        # packing explodes, in the reference too)
        from peridem_b200 import surrogate as sg
        t0 = time.perf_counter()
        train = scn.build_scene(scn.compressive_2d(n_particles=64, r_range=(1e-3, 1.5e-3), h_div=15,
                                                   width=22e-3, seed=args.seed + 1, wall_speed=-0.5,
                                                   nt=20000))
        model_s = sg.build(train, steps=16000, every=40, iters=6000, samples_per_particle=400)
        t_train = time.perf_counter() - t0
        model_s.attach(model, check_interval=50)
        sur = {"train_seconds": round(t_train, 1),
               "shapes": [{"zone": S.zone, "nodes": S.n_nodes,
                           **{k: round(v, 5) for k, v in S.report.items()}} for S in model_s.shapes]}
    if snap:
        model.load_state(snap)
    else:
        model.integrate_begin()
    stream = torch.cuda.ExternalStream(model.stream_handle(), device=dev)
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def flush_l2(buf, k):
        # write 512 MiB (4x the 126 MB L2), then read it back: the read pass
        # writes the dirty lines back before the timed step starts, so the
        # step begins with a cold, clean L2 and pays no write-back of the flush
        buf.fill_(float(k))
        buf.sum()

    def timed_window(m, s):
        """W untimed steps, then K steps each timed with CUDA events on the
        model's stream, the L2 flushed before each; per-step ms."""
        def step():
            # one step per launch (the L2 flush sits between steps); graph
            # replay by default, the plain stream path with --graph-steps 0
            if args.graph_steps:
                m.integrate_step(args.graph_steps, graph_steps=args.graph_steps)
            else:
                m.integrate_step(1)
        with torch.cuda.stream(s):
            for _ in range(args.warmup):
                step()
            m.sync()
            if world > 1:
                torch.distributed.barrier()
            torch.cuda.synchronize()
            ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                  for _ in range(args.steps)]
            # hold the stream (untimed) while the host queues every timed
            # step, so that no event pair brackets host launch latency
            torch.cuda._sleep(int(min(2e6 * args.steps, 1e9)))
            for k in range(args.steps):
                flush_l2(flush, k)
                ev[k][0].record(s)
                step()
                ev[k][1].record(s)
            m.sync()
            torch.cuda.synchronize()
        return [a.elapsed_time(b) for a, b in ev]

    before = model.scalars()
    if args.profile_window:
        torch.cuda.profiler.start()  # cudaProfilerStart: a profiler started with it off sees the window only
    with ClockSampler(dev) as clk:
        step_ms = timed_window(model, stream)
    if args.profile_window:
        torch.cuda.profiler.stop()
    after = model.scalars()
    window = {"steps": [int(before["n"]) + args.warmup + 1, int(after["n"])],
              "contact_rebuilds": int(after["contact_updates"] - before["contact_updates"]),
              "contact_entries": int(after["contact_entries"]),
              "contact_reaction": after["contact_reaction"], "reaction": after["reaction"],
              "max_velocity": after["max_velocity"], "prerun_seconds": round(pre_s, 2)}
    if snap:
        window.update({"prerun_steps": pre_steps, "wall_in_contact_at_start": bool(pre_touch)})
    if sc.test_interval > 0 and args.workload == "compressive":
        # the compressive-test records of the timed steps: how many carry a
        # contact reaction on the wall, and its largest magnitude
        hist = model.history()
        nwin = max(1, args.steps // sc.test_interval)
        cr = hist[-nwin:, 3] if len(hist) else np.zeros(0)
        window.update({"test_records": int(len(cr)), "records_with_wall_contact": int(np.sum(cr != 0.0)),
                       "wall_contact_reaction_max_abs": float(np.max(np.abs(cr))) if len(cr) else 0.0})
    mixed_end = None
    if prec == PREC_MIXED and args.fp64_arm:
        mixed_end = {"hist": model.history(), "bonds": model.field("bonds"), "Z": model.field("Z"),
                     "u": model.field("u")}
    total_ms = max_over_ranks(float(sum(step_ms)), world, f"cuda:{dev}")
    nodes = sc.n_nodes
    value = job_throughput(nodes, args.steps, world, total_ms)

    # the plain FP64 form (the drop-in) on the same state and steps: its
    # throughput, and the FP32 form's error against it over the window
    fp64 = None
    if mixed_end is not None:
        m64 = GpuDEMModel(sc, precision=PREC_FP64, device=dev, build_neighbors=True, compute_mx=True)
        try:
            if args.contact_lanes:
                from peridem_b200 import api
                api.set_lanes(m64, 0, args.contact_lanes)
            if snap:
                m64.load_state(snap)
            else:
                m64.integrate_begin()
            s64 = torch.cuda.ExternalStream(m64.stream_handle(), device=dev)
            ms64 = max_over_ranks(float(sum(timed_window(m64, s64))), world, f"cuda:{dev}")
            fp64 = {"value": job_throughput(nodes, args.steps, world, ms64), "ms_per_step": ms64 / args.steps}
            fp64["speedup_of_mixed"] = value / fp64["value"]
            fp64["error_of_mixed"] = mixed_error(mixed_end, {"hist": m64.history(), "bonds": m64.field("bonds"),
                                                             "Z": m64.field("Z"), "u": m64.field("u")},
                                                 window["steps"], sc.test_interval)
        finally:
            m64.close()
    # the surrogate form against the same scene without it (mixed form):
    # what the learned part gains or costs, and its error against FP64
    if sur is not None:
        m2 = GpuDEMModel(sc, precision=PREC_MIXED, device=dev, build_neighbors=True, compute_mx=True,
                         pd_lanes=args.pd_lanes, tile_nodes=args.tile_nodes)
        try:
            m2.integrate_begin()
            s2 = torch.cuda.ExternalStream(m2.stream_handle(), device=dev)
            ms2 = max_over_ranks(float(sum(timed_window(m2, s2))), world, f"cuda:{dev}")
            sur["without_surrogate_value"] = job_throughput(nodes, args.steps, world, ms2)
            sur["speedup_of_surrogate"] = value / sur["without_surrogate_value"]
        finally:
            m2.close()

    # per-kernel device times over a second timed pass (same flush)
    model.enable_timing(True)
    with torch.cuda.stream(stream):
        for k in range(args.steps):
            flush_l2(flush, k)
            model.integrate_step(1)
        model.sync()
    ktimes = model.kernel_times()
    model.enable_timing(False)
    if sur is not None:
        on, tot, steps_on, steps_all = model.surrogate_stats()
        sur.update({"particles_on_now": on, "particles_covered": tot, "particle_steps_on": steps_on,
                    "particle_steps": steps_all, "fraction_on": round(steps_on / max(steps_all, 1), 4)})
    sc_vals = model.scalars()

    # phase clock of the contact-list rebuild (--rebuild-phases R): the next
    # R rebuilds after the window, one-step graphs, per-phase median (us)
    rebuild_phases = None
    if args.rebuild_phases > 0 and sc.multi_particle:
        names = ["clear", "count nodes per cell", "scan cell offsets", "scatter", "in-cell sort",
                 "count candidates", "scan row offsets", "scan compaction offsets", "compact",
                 "fill (first CTA's share)"]
        model.rebuild_phases(True)
        runs = []
        for _ in range(args.rebuild_phases):
            u0 = model.scalars()["contact_updates"]
            for _ in range(1000):
                model.integrate_step(1, graph_steps=1)
                model.sync()
                if model.scalars()["contact_updates"] != u0:
                    break
            t = model.rebuild_phases()
            if len(t) >= 2:
                runs.append(np.diff(np.asarray(t, dtype=np.float64)) / 1e3)
        model.rebuild_phases(False)
        if runs:
            n = min(len(r) for r in runs)
            med = np.median(np.stack([r[:n] for r in runs]), axis=0)
            rebuild_phases = {"rebuilds": len(runs), "first_cta_done_us": round(float(med.sum()), 1),
                              "phases_us": {nm: round(float(x), 1) for nm, x in zip(names, med)}}

    # end to end through the host-buffer call: H2D of u, v, x and D2H of
    # u, v, x, f every step (pinned buffers)
    N = sc.n_nodes
    bufs = [torch.empty((N, 3), dtype=torch.float64, pin_memory=True).numpy() for _ in range(4)]
    u_h, v_h, x_h, f_h = bufs
    u_h[:] = model.field("u")
    v_h[:] = model.field("v")
    x_h[:] = model.field("x")
    for _ in range(3):
        model.step_host(u_h, v_h, x_h, f_h, 1)
    e2e_steps = max(10, min(args.steps, 200))
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        model.step_host(u_h, v_h, x_h, f_h, 1)
    e2e_s = max_over_ranks(time.perf_counter() - t0, world, f"cuda:{dev}")
    e2e = {"value": nodes * e2e_steps * world / e2e_s, "unit": UNIT,
           "h2d_bytes_per_step": 3 * N * 3 * 8, "d2h_bytes_per_step": 4 * N * 3 * 8,
           "call": "pdgpu_step_host (host u,v,x in; u,v,x,f out; 1 step per call)"}

    # roofline of the dominant kernel among those with an algorithmic-byte
    # model (the contact pass runs beside the bond loop on its own stream, so
    # its event time mostly measures the bond loop it shares the SMs with)
    modeled = {k: v for k, v in ktimes.items() if k in ("pd_force", "pd_force_mixed")}
    dom = max(modeled.items(), key=lambda kv: kv[1][0]) if modeled else None
    roof = None
    gpu_launches = model.step_kernel_count() * args.steps
    if dom:
        name, (ms, launches) = dom
        bytes_, units = algorithmic_bytes(name, sc, args.precision)
        peak, kind = measured_peak()
        avg_s = ms / launches * 1e-3
        if bytes_:
            ach = bytes_ / avg_s / 1e9
            # the committed ncu capture covers the default workload only
            traffic, tsrc = traffic_from_profiles(name) if args.workload == "compressive" else (None, None)
            roof = {"kernel": name, "bound": "hbm", "achieved": round(ach, 1), "peak": peak,
                    "unit": "GB/s", "frac": round(ach / peak, 4), "peak_source": kind,
                    "traffic": traffic,
                    "traffic_source": (f"recorded by the ncu capture summarised in profiles/{tsrc} "
                                       "(not measured in this run)") if tsrc else None,
                    "avg_launch_us": round(avg_s * 1e6, 2),
                    "algorithmic_bytes_per_launch": int(bytes_), "units": units}
        else:
            roof = {"kernel": name, "bound": "hbm", "achieved": None, "peak": peak,
                    "unit": "GB/s", "frac": None, "avg_launch_us": round(avg_s * 1e6, 2)}
    kt = {k: {"ms_total": round(v[0], 4), "launches": v[1], "us_avg": round(1e3 * v[0] / max(v[1], 1), 2)}
          for k, v in sorted(ktimes.items(), key=lambda kv: -kv[1][0])}
    model.close()
    return {"value": value, "ms_per_step": total_ms / args.steps, "e2e": e2e, "roofline": roof,
            "kernels": kt, "clocks": clk.summary(), "gpu_launches": gpu_launches, "autotune": tuned,
            "surrogate": sur, "fp64": fp64, "window": window, "snapshot": snap,
            "rebuild_phases": rebuild_phases,
            "scalars": {k: sc_vals[k] for k in ("n", "contact_updates", "contact_entries",
                                                 "contact_update_interval", "broken_bonds",
                                                 "reaction", "contact_reaction")},
            "sc": sc}


def cpu_reference(args, steps, warmup, load=None):
    """The reference's own CPU step (oracle/_ref/peridem_ref, Taskflow on all
    host threads) on the same workload deck, from the state snapshot `load`
    when given (the portable part: x, u, v, broken bonds, step, contact
    control); returns the parsed JSON line."""
    from peridem_b200 import scene as scn
    ref = os.path.join(ROOT, "oracle", "_ref", "peridem_ref")
    if not os.path.exists(ref):
        return None
    spec = workload_spec(args)
    threads = os.cpu_count() or 1
    with tempfile.TemporaryDirectory(prefix="peridem_deck_") as d:
        scn.write_deck(spec, d)
        cmd = [ref, "-i", "deck.yaml", "-nThreads", str(threads), "-time", str(steps)]
        if load:
            cmd += ["-load", load]
        r = subprocess.run(cmd, cwd=d, capture_output=True, text=True, timeout=1800)
    for line in r.stdout.splitlines()[::-1]:
        if line.startswith("{"):
            out = json.loads(line)
            out["threads"] = threads
            return out
    raise RuntimeError("reference timing failed: " + r.stdout[-500:] + r.stderr[-500:])


def prerun_state(sc, args, device=0):
    """The untimed pre-run of the compression (mixed form, graph replay):
    args.prerun steps, then, for the compressive test, 10-step strides until
    the top wall is in contact with the packing (a non-zero contact reaction
    in the latest test record; at most args.prerun_contact_cap more steps),
    so that the timed window starts under the wall's load.  Saved as a state
    snapshot; returns (path, seconds, steps run, wall in contact)."""
    from peridem_b200.model import GpuDEMModel, PREC_MIXED
    t0 = time.perf_counter()
    m = GpuDEMModel(sc, precision=PREC_MIXED, device=device, build_neighbors=True, compute_mx=True)
    try:
        m.integrate_begin()
        m.integrate_step(args.prerun, graph_steps=min(args.prerun, 500))
        m.sync()
        steps, touching = args.prerun, False
        if args.workload == "compressive":
            while True:
                touching = m.scalars()["contact_reaction"] != 0.0
                if touching or steps - args.prerun >= args.prerun_contact_cap:
                    break
                m.integrate_step(10, graph_steps=10)
                m.sync()
                steps += 10
        path = os.path.join(tempfile.mkdtemp(prefix="pdgpu_bench_"), "prerun.pdsnap")
        m.save_state(path)
    finally:
        m.close()
    return path, time.perf_counter() - t0, steps, touching


def prerun_snapshot(args):
    """The state the timed window starts from, for the reference arm: the
    same untimed pre-run on the GPU (state preparation only; the reference's
    own code is what is timed), saved as a state snapshot.  Without a GPU,
    or without a pre-run, the reference starts from the deck's initial
    state; returns (path or None, description)."""
    if args.prerun <= 0:
        return None, "from the deck's initial state"
    try:
        import torch
        if not torch.cuda.is_available():
            return None, "from the deck's initial state (no GPU to run the pre-run)"
        path, _, steps, touching = prerun_state(build_workload(args), args)
        return path, ("from the state after the %d-step pre-run of the compression (made on the GPU, "
                      "loaded by peridem_ref -load; top wall %s)"
                      % (steps, "in contact" if touching else "not in contact"))
    except Exception as e:  # report, do not hide
        return None, f"from the deck's initial state (pre-run failed: {e})"


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--particles", type=int, default=502)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--graph-steps", type=int, default=1)
    ap.add_argument("--cpu-steps", type=int, default=40)
    ap.add_argument("--pd-lanes", type=int, default=0, help="lanes per node in the bond loop (0 = auto)")
    ap.add_argument("--tile-nodes", type=int, default=0, help="nodes per bond-loop tile (0 = auto)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", default="compressive", choices=["compressive", "ensemble", "column3d", "surrogate"],
                    help="compressive: one 502-particle scene; ensemble: --scenes independent scenes in "
                         "one model; column3d: --spheres spheres in a 3-D column; surrogate: the learned "
                         "surrogate on 2000 particles (its training, untimed, takes ~15 s at h = R/15)")
    ap.add_argument("--scenes", type=int, default=256)
    ap.add_argument("--spheres", type=int, default=4096)
    ap.add_argument("--autotune", action="store_true",
                    help="choose lanes, tile size and search skin by timing the scene first")
    ap.add_argument("--tune-steps", type=int, default=100)
    ap.add_argument("--prerun", type=int, default=20000,
                    help="untimed steps of the compression before the timed window (compressive "
                         "workload), continued until the top wall touches the packing; the state "
                         "they reach is what every arm times")
    ap.add_argument("--prerun-contact-cap", type=int, default=60000,
                    help="at most this many more pre-run steps waiting for the top wall's contact")
    ap.add_argument("--contact-lanes", type=int, default=0, help="lanes per node in the contact pass (0 = auto)")
    ap.add_argument("--rebuild-phases", type=int, default=0,
                    help="after the window, time this many contact-list rebuilds phase by phase "
                         "(GPU global timer at each grid-wide barrier) and report the medians")
    ap.add_argument("--profile-window", action="store_true",
                    help="bracket the timed window with cudaProfilerStart/Stop (for ncu --profile-from-start off)")
    ap.add_argument("--no-fp64", dest="fp64_arm", action="store_false",
                    help="skip the plain FP64 form on the same state (and the mixed form's error)")
    args = ap.parse_args()
    if args.workload != "compressive":
        args.prerun = 0

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference" and rank != 0:
        return  # the reference arm runs on rank 0 alone and needs no collective
    if world > 1 and args.impl != "reference":
        import torch
        import datetime
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))

    if args.impl == "reference":
        t0 = time.perf_counter()
        snap, how = prerun_snapshot(args)
        res = cpu_reference(args, args.steps, args.warmup, load=snap)
        if res is None:
            print(json.dumps({"impl": "reference", "unavailable": "reference binary oracle/_ref/peridem_ref not built"}))
            return
        if snap:
            import shutil
            shutil.rmtree(os.path.dirname(snap), ignore_errors=True)
        v = res["node_steps_per_s"]
        line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
                "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": 1e3 * res["seconds"] / res["steps"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": workload_config(args, None) | {"nodes": int(res["nodes"])},
                "cpu_baseline": {"value": v, "unit": UNIT, "cores": res["threads"], "kind": "reference",
                                 "sample": f"{res['steps']} steps of the full scene after one warm-up step "
                                           f"(init {res['init_seconds']:.1f} s excluded), {how}"},
                "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                "wall_s": time.perf_counter() - t0}
        print(json.dumps(line))
        return

    res = run_ours(args, rank, world)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            r = cpu_reference(args, args.cpu_steps, 1, load=res.get("snapshot"))
            if r is not None:
                if args.workload == "ensemble":
                    what = ("the ensemble's first scene (%d nodes; the reference runs one scene per process)"
                            % int(r["nodes"]))
                elif args.workload == "column3d":
                    what = ("an 8-sphere column of the same sphere mesh and material (%d nodes, most of "
                            "them box walls)" % int(r["nodes"]))
                elif res.get("snapshot"):
                    what = ("the same scene from the GPU's state after the %d-step pre-run (x, u, v, broken "
                            "bonds, step and contact control loaded by peridem_ref -load)"
                            % res["window"].get("prerun_steps", args.prerun))
                else:
                    what = "the same scene"
                cpu = {"value": r["node_steps_per_s"], "unit": UNIT, "cores": r["threads"],
                       "kind": "reference",
                       "sample": f"{r['steps']} steps of {what} after one warm-up step "
                                 f"(init {r['init_seconds']:.1f} s excluded)"}
        except Exception as e:  # report, do not hide
            cpu = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
                   "sample": f"failed: {e}"}
    if res.get("snapshot"):
        import shutil
        shutil.rmtree(os.path.dirname(res["snapshot"]), ignore_errors=True)
    if rank == 0:
        sc = res.pop("sc")
        line = {"metric": METRIC, "value": res["value"], "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": res["ms_per_step"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "f32-bond/f64" if args.precision == "mixed" else "f64",
                "data": "synthetic", "config": workload_config(args, sc),
                "e2e": res["e2e"], "roofline": res["roofline"], "cpu_baseline": cpu,
                "clocks": res["clocks"], "gpu_launches": res["gpu_launches"],
                "kernels": res["kernels"], "scalars": res["scalars"], "window": res["window"]}
        if res.get("fp64"):
            f64 = res["fp64"]
            line["fp64_value"] = f64["value"]
            line["fp64_ms_per_step"] = f64["ms_per_step"]
            line["speedup_vs_fp64"] = f64["speedup_of_mixed"]
            line["error_vs_fp64"] = f64["error_of_mixed"]
        if res.get("autotune"):
            line["autotune"] = res["autotune"]
        if res.get("rebuild_phases"):
            line["rebuild_phases"] = res["rebuild_phases"]
        if res.get("surrogate"):
            line["surrogate"] = res["surrogate"]
        print(json.dumps(line))
    if world > 1:
        import torch
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
