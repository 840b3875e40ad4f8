#!/usr/bin/env python
"""Benchmark: particle-steps/s of the plain path at N=1,048,576, theta=0.5.

Workload (the precision-study disk at theta 0.5): N = 1,048,576 equal-mass
bodies (m = 1e-9 Msun) around a 1 Msun star, Keplerian disk in XZ with r in
[0.3, 30] AU (Sigma ~ r^-1.5), Rayleigh e/i (sigma 0.01 / 0.005 rad),
softening 5e-4 AU, dt 0.002 T0, no collisions, drag or perturber, FP32 state
(the reference's ParticleData precision), FP32 forces.  Inputs are seeded
synthetic disks (seed = rank); there is no dataset.

A step is one pass of src/main.cu:101-139 through the engine (nbody_sim_step):
fused stream kernel, keys, radix sort, permute, tree, walk.  Each timed step
is bracketed by CUDA events on the engine's stream with an L2 flush (a 256 MB
write) before it, outside the events.  ``value`` is whole-job particle-steps/s
(sum over ranks / max time over ranks).  ``e2e`` is the same metric through
nbody_sim_step_host with pinned host buffers: copyToGPU of x..az + mass, one
step, copyToCPU of x..az, every step.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU (torchrun): every rank advances its own disk (independent replicas,
no collective in the data path; "scaling": "weak").
"""
from __future__ import annotations

import argparse
import importlib
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
METRIC = "particle-steps/s at N=1M theta=0.5"
UNIT = "particle-steps/s"
WORKLOAD = dict(n=1 << 20, r_min=0.3, r_max=30.0, m=1e-9, eps=5e-4, theta=0.5, dt=0.002)
# FLOP of the walk per accepted source-target interaction, as the kernel
# computes it: 3 sub (d = s - p), 3 FMA as 2 each (r^2 + eps^2), rsqrt as 1,
# 3 mul (inv^3 and m inv^3), 3 FMA as 2 each (the three accumulations) = 19
FLOP_PER_INTERACTION = 19


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=WORKLOAD["n"])
    ap.add_argument("--theta", type=float, default=WORKLOAD["theta"])
    ap.add_argument("--precision", choices=["f32", "f64"], default="f32")
    ap.add_argument("--leaf-max", type=int, default=0,
                    help="walk leaf size (nbody_sim_params.leaf_max); 0: the engine's default")
    ap.add_argument("--walk-mode", type=int, default=None, choices=[0, 1, 2],
                    help="force-walk variant (nbody_sim_params.walk_mode); default: the engine's")
    ap.add_argument("--group-span", type=int, default=None,
                    help="target groups from maximal nodes of <= span x 32 bodies "
                         "(nbody_sim_params.group_span)")
    ap.add_argument("--span-walk", type=int, default=None, choices=[0, 1, 2],
                    help="shared walk (nbody_sim_params.span_walk); default: the engine's")
    ap.add_argument("--targets-per-lane", type=int, default=None, choices=[1, 2],
                    help="walk targets per lane, groups of 32 or 64 "
                         "(nbody_sim_params.targets_per_lane); default: the engine's")
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-studies", action="store_true",
                    help="headline line without the force-error, reference-engine, ensemble "
                         "and adjoint sub-records")
    ap.add_argument("--adjoint-fd", type=int, default=48,
                    help="velocity components checked by central differences in the headline "
                         "line's adjoint record")
    ap.add_argument("--no-flush", action="store_true")
    ap.add_argument("--workload", choices=["disk1m", "ensemble", "precision", "adjoint", "c2run"],
                    default="disk1m",
                    help="disk1m: the headline single disk; ensemble: 64 disks (C4) against "
                         "the same disks run one by one; precision: force error vs FP64 "
                         "direct sum over theta, and energy / L_y drift per state precision")
    ap.add_argument("--targets", type=int, default=16384,
                    help="precision study: force-error targets (seeded random subset)")
    ap.add_argument("--drift-steps", type=int, default=200)
    ap.add_argument("--fd-components", type=int, default=1024,
                    help="adjoint study: velocity components checked by central differences")
    ap.add_argument("--disks", type=int, default=64)
    ap.add_argument("--solo-steps", type=int, default=10,
                    help="timed steps per disk of the one-by-one comparison")
    return ap.parse_args()


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=timedelta(seconds=300))
    return ws, rank, local


def allreduce_max(v: float, ws: int) -> float:
    if ws == 1:
        return v
    import torch
    import torch.distributed as dist
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def make_ic(nb, n, seed, dtype=np.float32):
    d = nb.make_disk(n, WORKLOAD["r_min"], WORKLOAD["r_max"], 0.01, 0.005, 1.0, seed)
    st = {k: v.astype(dtype) for k, v in d.items()}
    st["m"] = np.full(n, WORKLOAD["m"], np.float32)
    return st


def oracle_port():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    return oracle.Port()


def make_ic_oracle(n, seed):
    """The same disk as make_ic, from the oracle's restatement of the recipe
    (oracle/port.c orc_make_disk, bit-identical), so that the reference arm
    loads none of the product's libraries."""
    d = oracle_port().make_disk(n, WORKLOAD["r_min"], WORKLOAD["r_max"], 0.01, 0.005, 1.0, seed)
    st = {k: v.astype(np.float32) for k, v in d.items()}
    st["m"] = np.full(n, WORKLOAD["m"], np.float32)
    return st


class Clocks:
    """SM clock and clock-event reasons sampled during the timed region: NVML
    read every 5 ms from a thread (the region lasts ~0.1-1 s), else
    nvidia-smi at its 200 ms rate.  Reads only; nothing is set."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # NVML clocks-event reason bits
    REASONS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20,
               "hw_thermal_slowdown": 0x40}

    def __init__(self, index: int):
        self.p = None
        self.samples = []
        self.smax = None
        self.thread = None
        self.stop_ev = threading.Event()
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nvml = pynvml
            self.h = self._handle(pynvml, index)
            self.smax = float(pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM))
            # both reads the poll makes, once here: a failure falls back to nvidia-smi
            pynvml.nvmlDeviceGetClockInfo(self.h, pynvml.NVML_CLOCK_SM)
            pynvml.nvmlDeviceGetCurrentClocksEventReasons(self.h)
            self.thread = threading.Thread(target=self._poll, daemon=True)
            self.thread.start()
            return
        except Exception:
            self.thread = None
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-i", str(index), "-lms", "200"], stdout=subprocess.PIPE,
                stderr=subprocess.DEVNULL, text=True)
        except (OSError, ValueError):
            self.p = None

    @staticmethod
    def _handle(pynvml, index: int):
        """The NVML handle of CUDA device `index`, matched by PCI bus id (NVML
        numbers every GPU of the machine, CUDA only the visible ones)."""
        try:
            pr = torch.cuda.get_device_properties(index)
            bus = f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
            return pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            return pynvml.nvmlDeviceGetHandleByIndex(index)

    def _poll(self):
        nv = self.nvml
        while not self.stop_ev.is_set():
            try:
                sm = float(nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM))
                rs = int(nv.nvmlDeviceGetCurrentClocksEventReasons(self.h))
                self.samples.append((sm, rs))
            except Exception:
                return
            self.stop_ev.wait(0.005)

    def stop(self):
        if self.thread is not None:
            self.stop_ev.set()
            self.thread.join(timeout=5)
            if not self.samples:
                return None
            reasons = sorted({nm for _, rs in self.samples for nm, bit in self.REASONS.items()
                              if rs & bit})
            return {"sm_mhz": statistics.median(sm for sm, _ in self.samples),
                    "sm_max_mhz": self.smax, "reasons": reasons, "samples": len(self.samples),
                    "source": "NVML, 5 ms"}
        if self.p is None:
            return None
        time.sleep(0.25)
        self.p.terminate()
        try:
            out, _ = self.p.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
            out, _ = self.p.communicate()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if f[5 + k].lower() in ("active", "1", "yes"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm), "source": "nvidia-smi, 200 ms"}


def fp32_peak(smax_mhz: float | None):
    """FP32 SIMT peak from the SM count and the max SM clock (no measured
    FP32 figure exists for this pool): SMs x 128 lanes x 2 FLOP x clock."""
    import torch
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    mhz = smax_mhz or 1965.0
    peaks = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(peaks):
        with open(peaks) as f:
            mhz = float(json.load(f).get("sm_max_mhz", mhz))
    return sms * 128 * 2 * mhz * 1e6 / 1e12, f"derived: {sms} SM x 128 FP32 lanes x 2 x {mhz:.0f} MHz"


def walk_traffic():
    """Per-launch DRAM bytes of the walk from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "walk_n1m_traffic.txt")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        for line in f:
            if line.startswith("bytes_per_launch"):
                return float(line.split("=")[1])
    return None


def workload_name(n, theta, precision="f32"):
    return (f"Keplerian disk N={n} r=[0.3,30] AU theta={theta} eps=5e-4 dt=0.002, "
            f"{precision.upper()} state, no collisions/drag/perturber")


# what one timed CPU step of the reference algorithm does (oracle/port.c)
CPU_STEP = ("CAS octree build, the reference's 20 parallel summarize passes, DFS sort, walk, "
            "KDK")


def cpu_port_step(st, n, nthreads=0, steps=1):
    """The CPU restatement of the reference step (oracle/port.c), timed, with
    the reference's fixed 20 summarize passes (BHTree.cu:501-516) rather than
    the oracle's converged sweep (same values on these trees, the reference's
    amount of work)."""
    port = oracle_port()
    w = WORKLOAD
    sp = port.step_params(w["dt"], w["theta"], w["eps"], 1.0, r_coll=0.0, collisions=False)
    s = {k: np.array(st[k][:n], np.float32) for k in ("x", "y", "z", "vx", "vy", "vz", "m")}
    port.set_summarize_passes(20)
    try:
        port.run(s, sp, 0, nthreads=nthreads)  # initial forces (untimed)
        t0 = time.perf_counter()
        port.run(s, sp, steps, nthreads=nthreads, initial_forces=False)
        return time.perf_counter() - t0
    finally:
        port.set_summarize_passes(0)


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_study(nb, st, n, all_core_step_secs):
    """The reference's CPU path on the host cores beside the GPU: one step of
    the CPU restatement (oracle/port.c) on one core and on all cores at the
    C1 and C2 sizes and at N (one core: one step), and the reference's own
    detectAggregates (Aggregate.cpp, one core, O(N^2)) at C1 and C2 sizes with
    their collision radii as linking lengths, beside the engine's GPU FoF on
    the same bodies."""
    import torch
    cores = os.cpu_count() or 1
    out = {"cores": cores, "cpu": cpu_model(), "port_step_s": {}, "detect_aggregates_s": {},
           "gpu_fof_s": {}}
    for size in (4096, 131072):
        out["port_step_s"][str(size)] = {"1": cpu_port_step(st, size, 1, 1),
                                         "all": cpu_port_step(st, size, 0, 1)}
    out["port_step_s"][str(n)] = {"1": cpu_port_step(st, n, 1, 1), "all": all_core_step_secs}
    ref = os.path.join(ROOT, "oracle", "_ref", "libref_host.so")
    rh = None
    if os.path.exists(ref):
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
        rh = oracle.RefHost(ref)
    # C1: factor 1 at m = 1e-8; C2: factor 5 (the reference's collision radius)
    r1 = nb.particle_physical_radius(1e-8)
    for size, link in ((4096, r1), (131072, 5.0 * r1)):
        xs = [np.ascontiguousarray(st[k][:size], np.float32) for k in ("x", "y", "z")]
        key = str(size)
        if rh is not None:
            t0 = time.perf_counter()
            rh.detect_aggregates_count(*xs, float(link))
            out["detect_aggregates_s"][key] = time.perf_counter() - t0
        tree = nb.Octree(size)
        dev = [torch.from_numpy(a).cuda() for a in xs]
        tree.fof(*dev, float(link))  # warm-up
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        tree.fof(*dev, float(link))
        torch.cuda.synchronize()
        out["gpu_fof_s"][key] = time.perf_counter() - t0
        tree.close()
    out["sample"] = ("bodies 0..size-1 of the headline disk; one step (or one FoF call) each, "
                     "after one untimed forces pass; GPU FoF is the stand-alone nbody_fof, host "
                     "wall time of one call")
    return out


def run_reference(args, ws, rank):
    """The reference's CPU path (its host build of the force and integrator
    formulas, oracle/port.c) on all host cores; rank 0 only."""
    if rank != 0:
        return
    n = args.n
    st = make_ic_oracle(n, 0)
    cores = os.cpu_count() or 1
    for _ in range(args.warmup):
        cpu_port_step(st, n, 0, 1)
    secs = [cpu_port_step(st, n, 0, 1) for _ in range(args.steps)]
    total = sum(secs)
    value = n * args.steps / total
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": workload_name(n, args.theta), "n": n, "theta": args.theta,
                   "state": "f32", "parallelism": "cpu", "l2": "n/a (host)"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"{args.steps} full steps at N={n} ({CPU_STEP}), OpenMP "
                                   "over all host threads; initial conditions from the oracle's "
                                   "restatement of the disk recipe"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# Algorithmic HBM bytes per body of each step phase at FP32 state without
# collisions (the unique bytes a phase must move; its kernels' own layout):
#   stream  read x, v, a (36) + write x, v (24)
#   sort    keys: read x (12) + write key, index (8); four 8-bit passes of
#           key + index read and written (4 x 16)
#   permute read index (4) + gather x, v, mass, id (32); write x, v, mass, id
#           (32) + the walk's float4 body (16) + the FP64 moment prefix (32)
#   tree    keys (4) + binary topology (16) + moment prefix read (32) + node
#           COM and mass (32)
PHASE_BYTES_F32 = {"stream": 60, "sort": 84, "permute": 116, "tree": 84}


def hbm_peak():
    """Measured copy bandwidth of this pool's B200s (GB/s), else the
    earlier measurement used as the fallback."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        for k in ("hbm_gbs", "hbm_GBs", "hbm_copy_gbs"):
            if k in d:
                return float(d[k]), "measured (MEASURED_PEAKS.json)"
    return 6650.0, "fallback (6.65 TB/s)"


def phase_hbm(prof, n):
    peak, src = hbm_peak()
    out = {"peak_gbs": peak, "peak_source": src}
    for k, b in PHASE_BYTES_F32.items():
        ms = prof.get(k, 0.0)
        if ms > 0:
            gbs = b * n / (ms * 1e-3) / 1e9
            out[k] = {"bytes_per_body": b, "ms": ms, "gbs": gbs, "frac": gbs / peak}
    return out


def ref_engine_study(st, n, theta, steps=3):
    """The reference's own CUDA engine (src/physics/*.cu compiled unchanged for
    sm_100a, oracle/_ref/libref_engine.so) through the step loop of
    src/main.cu:101-139 on the same disk: the throughput that the plain
    path's 3x target is set against.  The CPU restatement first checks that
    the reference build keeps every body and summarizes the whole tree on
    this input."""
    path = os.path.join(ROOT, "oracle", "_ref", "libref_engine.so")
    if not os.path.exists(path):
        return {"unavailable": "oracle/_ref/libref_engine.so not built"}
    port = oracle_port()
    import oracle
    t = port.build_tree(st["x"], st["y"], st["z"], st["m"])
    info = port.tree_info(t)
    port.free_tree(t)
    if info.lost_bodies or info.unsummarized or info.height > 20:
        return {"unavailable": f"reference build unsafe on this input (lost {info.lost_bodies}, "
                               f"unsummarized {info.unsummarized}, height {info.height})"}
    w = WORKLOAD
    eng = oracle.RefEngine(n, path=path)
    try:
        eng.set_state(st)
        eng.build()
        eng.force(theta, w["eps"], 1.0)
        eng.steps(0, 1, w["dt"], theta, w["eps"], 1.0, 0.0, 0.0, 0.0)  # warm-up
        ms = eng.steps(1, steps, w["dt"], theta, w["eps"], 1.0, 0.0, 0.0, 0.0)
    finally:
        eng.close()
    return {"value": n * steps / (ms * 1e-3), "unit": UNIT, "ms_per_step": ms / steps,
            "steps": steps, "tree_height": info.height,
            "how": "src/main.cu:101-139 launcher sequence (each launcher synchronous), "
                   "wall time of the loop, after one warm-up step"}


def run_ours(args, ws, rank, local):
    import torch
    nb = importlib.import_module("nbody-sim_b200")
    torch.cuda.set_device(local)
    n = args.n
    w = WORKLOAD
    prec = nb.STATE_F64 if args.precision == "f64" else nb.STATE_F32
    st = make_ic(nb, n, rank, np.float64 if prec == nb.STATE_F64 else np.float32)
    prm = nb.sim_params(dt=w["dt"], theta=args.theta, softening=w["eps"], star_mass=1.0,
                        r_coll=0.0, restitution=0.0, gas_drag_rate=0.0, state_precision=prec,
                        leaf_max=args.leaf_max)
    if args.walk_mode is not None:
        prm.walk_mode = args.walk_mode
    if args.group_span is not None:
        prm.group_span = args.group_span
    if args.span_walk is not None:
        prm.span_walk = args.span_walk
    if args.targets_per_lane is not None:
        prm.targets_per_lane = args.targets_per_lane
    stream = torch.cuda.current_stream()
    sim = nb.Sim(prm, n)
    sim.set_stream(stream.cuda_stream)
    sim.set_state(st["x"], st["y"], st["z"], st["vx"], st["vy"], st["vz"], st["m"])
    # Steps are taken one call at a time, each left open (nbody_sim_step_open):
    # a step is then one CUDA-graph replay that starts with the previous
    # step's second kick and drag fused into its own first kick and drift, as
    # in any multi-step run.  The run's last second kick comes after the
    # timed region.
    for _ in range(args.warmup):
        sim.step_open(1)
    sim.sync()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps)]
    clocks = Clocks(torch.cuda.current_device()) if rank == 0 else None
    l0 = sim.stats().launches
    barrier(ws)
    torch.cuda.synchronize()
    for k in range(args.steps):  # each step: one CUDA-graph replay
        if not args.no_flush:
            flush.zero_()
        starts[k].record(stream)
        sim.step_open(1)
        ends[k].record(stream)
    torch.cuda.synchronize()
    barrier(ws)
    ck = clocks.stop() if clocks else None
    sim.sync()
    step_ms = [s.elapsed_time(e) for s, e in zip(starts, ends)]
    ms = sum(step_ms)
    launches = sim.stats().launches - l0
    ms_max = allreduce_max(ms, ws)
    value = n * ws * args.steps / (ms_max * 1e-3)
    # phase breakdown and the walk's own time: a separate profiled pass
    # (events between the phases, kernels launched one by one)
    sim.set_profiling(True)
    sim.profile(reset=True)
    per_step = []
    for _ in range(7):  # median over steps read one at a time
        if not args.no_flush:
            flush.zero_()
        sim.step_open(1)
        sim.sync()
        per_step.append(sim.profile(reset=True))
    sim.set_profiling(False)
    sim.close_steps()
    stats = sim.stats()
    prof = {k: statistics.median(p[k] / max(p["steps"], 1) for p in per_step)
            for k in nb.PHASE_NAMES}
    prof["steps"] = 1

    # e2e: the public host-buffer call, pinned memory, copies in the timed region
    e2e = None
    if args.e2e_steps > 0 and prec == nb.STATE_F32:
        pin = {k: torch.from_numpy(np.ascontiguousarray(st[k], np.float32)).pin_memory()
               for k in ("x", "y", "z", "vx", "vy", "vz", "m")}
        g = sim.get_state()
        for k in ("ax", "ay", "az"):
            pin[k] = torch.from_numpy(g[k]).pin_memory()
        for k in ("x", "y", "z", "vx", "vy", "vz"):
            pin[k].copy_(torch.from_numpy(g[k]))
        host = {k: v.numpy() for k, v in pin.items()}
        sim.set_profiling(False)
        sim.step_host(host, host["m"], 1)  # warm-up
        es = [torch.cuda.Event(enable_timing=True) for _ in range(args.e2e_steps)]
        ee = [torch.cuda.Event(enable_timing=True) for _ in range(args.e2e_steps)]
        barrier(ws)
        for k in range(args.e2e_steps):
            es[k].record(stream)
            sim.step_host(host, host["m"], 1)
            ee[k].record(stream)
        torch.cuda.synchronize()
        e_ms = allreduce_max(sum(a.elapsed_time(b) for a, b in zip(es, ee)), ws)
        e2e = {"value": n * ws * args.e2e_steps / (e_ms * 1e-3), "unit": UNIT,
               "h2d_bytes_per_step": 4 * n * 10, "d2h_bytes_per_step": 4 * n * 9,
               "ms_per_step": e_ms / args.e2e_steps}

    walk_ms = prof["walk"] / max(prof["steps"], 1)
    flops = FLOP_PER_INTERACTION * stats.interactions
    peak, peak_src = fp32_peak(ck["sm_max_mhz"] if ck else None)
    achieved = flops / (walk_ms * 1e-3) / 1e12
    traffic = walk_traffic()
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": workload_name(n, args.theta, args.precision), "n": n,
                   "theta": args.theta,
                   "state": args.precision, "leaf_max": stats.leaf_max,
                   "parallelism": f"replicas x{ws}",
                   "l2": "flushed (256 MB write) before every timed step"},
        "gpu_launches": int(launches),
        "graph_launches_per_step": 1,
        "ms_per_step_median": statistics.median(step_ms),
        "ms_per_step_best": min(step_ms),
        "phase_ms_per_step": {k: prof[k] / max(prof["steps"], 1)
                              for k in nb.PHASE_NAMES},
        "interactions_per_particle": stats.interactions / n,
        "roofline": {"bound": "fp32-simt", "kernel": "k_walk", "achieved": achieved,
                     "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                     "peak_source": peak_src, "traffic": traffic,
                     "algorithmic": f"{FLOP_PER_INTERACTION} FLOP x {stats.interactions} "
                                    "interactions per launch"},
        "e2e": e2e,
        "clocks": ck,
    }
    line["phase_hbm"] = phase_hbm(line["phase_ms_per_step"], n)
    if rank == 0 and ws == 1 and not args.no_studies and prec == nb.STATE_F32:
        sim.close()
        # each sub-record on its own: a study that fails leaves an "error"
        # entry, never the headline line unprinted
        def study(name, fn):
            try:
                line[name] = fn()
            except Exception as e:  # noqa: BLE001 -- recorded in the line
                line[name] = {"error": f"{type(e).__name__}: {e}"}

        def force_err():
            dg = importlib.import_module("nbody-sim_b200.diagnostics")
            targets = np.sort(np.random.default_rng(0).choice(n, min(args.targets, n),
                                                              replace=False))
            fe = dg.engine_force_errors(prm, st, targets)
            return {"targets": len(targets), "total": fe["total"], "self": fe["self"],
                    "vs": "FP64 direct sum (nbody_direct_f64) on the same FP32 positions; the "
                          "engine's own walk (the timed one)"}

        def ref_engine():
            ref = ref_engine_study(st, n, args.theta)
            if "value" in ref:
                ref["ours_over_reference"] = value / ref["value"]
            return ref

        def ensemble():
            ens = ensemble_study(args, ws, rank, local, args.steps)
            return {"value": ens["value"], "ms_per_step": ens["ms_per_step"],
                    "n_total": ens["config"]["n_total"], "disks": args.disks,
                    "one_by_one_value": ens["one_by_one"]["value"],
                    "one_by_one_ms_per_step": ens["one_by_one"]["ms_per_step"],
                    "ensemble_over_one_by_one": ens["one_by_one"]["speedup"],
                    "workload": ens["config"]["workload"]}

        def adjoint():
            adj = adjoint_study(args, args.adjoint_fd)
            fdc = {k: v for k, v in adj["fd_check"].items() if k != "misses_at_h1e-6"}
            # each miss at h = 1e-6 with its error at 1e-5 and 1e-4: how the
            # quotient's error moves with h says whether round-off limits it
            fdc["misses_at_h1e-6"] = adj["fd_check"]["misses_at_h1e-6"][:10]
            return {"gradient_over_plain_forward": adj["ms"]["gradient_over_plain_forward"],
                    "ms": adj["ms"], "memory_bytes": adj["memory_bytes"],
                    "checkpointed": adj["checkpointed"],
                    "direct_sum_reference": adj["direct_sum_reference"],
                    "fd_check": fdc, "perturber": adj["perturber"],
                    "workload": adj["config"]["workload"]}

        study("force_err", force_err)
        study("ref_engine", ref_engine)
        study("ensemble", ensemble)
        study("adjoint", adjoint)
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        cores = os.cpu_count() or 1
        secs = cpu_port_step(st, n, 0, 1)
        line["cpu_baseline"] = {"value": n / secs, "unit": UNIT, "cores": cores, "kind": "port",
                                "sample": f"1 full step at N={n} of the reference algorithm "
                                          f"(oracle/port.c: {CPU_STEP}), OpenMP"}
        if not args.no_studies and prec == nb.STATE_F32:
            try:
                line["cpu_study"] = cpu_study(nb, st, n, secs)
            except Exception as e:  # noqa: BLE001 -- recorded in the line
                line["cpu_study"] = {"error": f"{type(e).__name__}: {e}"}
    sim.close()
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_ensemble(args, ws, rank, local):
    line = ensemble_study(args, ws, rank, local, args.steps)
    if rank == 0:
        print(json.dumps(line), flush=True)


def ensemble_study(args, ws, rank, local, steps):
    """64 disks of uneven size (N log-uniform in [2048, 65536]) with their own
    perturbers, collisions and drag, FP64 state: the batched ensemble engine
    against the same disks stepped one by one through nbody_sim.  With several
    ranks each rank takes a share of the disks balanced by N log N (strong
    scaling, no collective in the data path)."""
    import torch
    nb = importlib.import_module("nbody-sim_b200")
    wl = importlib.import_module("nbody-sim_b200.workloads")
    torch.cuda.set_device(local)
    specs_all = wl.c4_disks(args.disks)
    mine = wl.partition_disks([d["n"] for d in specs_all], ws)[rank]
    specs = [specs_all[k] for k in mine]
    prm = wl.c4_params(nb)
    if args.group_span is not None:
        prm.group_span = args.group_span
    st, m = wl.ensemble_state(nb, specs)
    n = len(m)
    n_all = sum(d["n"] for d in specs_all)
    stream = torch.cuda.current_stream()
    ens = nb.Ensemble(prm, specs)
    ens.set_stream(stream.cuda_stream)
    ens.set_state(st["x"], st["y"], st["z"], st["vx"], st["vy"], st["vz"], m)
    tuned = ens.autotune()
    for _ in range(args.warmup):
        ens.step(1)
    ens.sync()
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    s0 = ens.stats()
    clocks = Clocks(torch.cuda.current_device()) if rank == 0 else None
    barrier(ws)
    torch.cuda.synchronize()
    for k in range(steps):
        if not args.no_flush:
            flush.zero_()
        starts[k].record(stream)
        ens.step(1)
        ends[k].record(stream)
    torch.cuda.synchronize()
    barrier(ws)
    ck = clocks.stop() if clocks else None
    ens.sync()
    s1 = ens.stats()
    ms = sum(a.elapsed_time(b) for a, b in zip(starts, ends))
    ms_max = allreduce_max(ms, ws)
    value = n_all * steps / (ms_max * 1e-3)

    # e2e: nbody_ensemble_step_host, state and accelerations in from pinned
    # host buffers and back out, every step
    g = ens.get_state(double=True, accel=True)
    host = {k: torch.from_numpy(np.ascontiguousarray(g[k])).pin_memory().numpy()
            for k in ("x", "y", "z", "vx", "vy", "vz", "ax", "ay", "az")}
    hm = torch.from_numpy(m).pin_memory().numpy()
    e_steps = max(args.e2e_steps, 1)
    ens.step_host(host, hm, 1)  # warm-up
    es = [torch.cuda.Event(enable_timing=True) for _ in range(e_steps)]
    ee = [torch.cuda.Event(enable_timing=True) for _ in range(e_steps)]
    barrier(ws)
    for k in range(e_steps):
        es[k].record(stream)
        ens.step_host(host, hm, 1)
        ee[k].record(stream)
    torch.cuda.synchronize()
    e_ms = allreduce_max(sum(a.elapsed_time(b) for a, b in zip(es, ee)), ws)

    # the same disks one by one through nbody_sim (each its own tree, walk, ...)
    solo_ms = 0.0
    for spec in specs:
        d, md = wl.disk_state(nb, spec)
        p = wl.c4_params(nb)
        p.perturber_enabled = spec["perturber_enabled"]
        p.perturber_mass_mjup = spec["perturber_mass_mjup"]
        p.perturber_radius_au = spec["perturber_radius_au"]
        p.perturber_phase0 = spec["perturber_phase0"]
        sim = nb.Sim(p, spec["n"])
        sim.set_stream(stream.cuda_stream)
        sim.set_state(d["x"], d["y"], d["z"], d["vx"], d["vy"], d["vz"], md)
        for _ in range(2):
            sim.step(1)
        sim.sync()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        if not args.no_flush:
            flush.zero_()
        a.record(stream)
        for _ in range(args.solo_steps):
            sim.step(1)
        b.record(stream)
        torch.cuda.synchronize()
        solo_ms += a.elapsed_time(b) / args.solo_steps
        sim.close()
    solo_ms = allreduce_max(solo_ms, ws)
    line = {
        "metric": f"ensemble particle-steps/s ({args.disks} disks)", "value": value, "unit": UNIT,
        "n_gpus": ws, "steps": steps, "warmup": args.warmup,
        "ms_per_step": ms_max / steps, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"{args.disks} Keplerian disks, N log-uniform [2048,65536] "
                               f"(total {n_all}), r=[0.5,5] AU, m=1e-8, perturber log-uniform "
                               "[0.3,10] MJ at U[5,30] AU, collisions (factor 5, e=0), drag "
                               "1e-3, theta 0.5, dt 0.005, FP64 state",
                   "n_total": n_all, "disks": args.disks, "parallelism": f"disks over {ws} ranks",
                   "l2": "flushed (256 MB write) before every timed step",
                   "autotune": [list(t) for t in tuned],
                   "targets_per_lane": s1.targets_per_lane, "leaf_max": s1.leaf_max,
                   "walk_mode": s1.walk_mode},
        "gpu_launches": int(s1.launches - s0.launches),
        "graph_launches": int(s1.graph_launches - s0.graph_launches),
        "one_by_one": {"ms_per_step": solo_ms,
                       "value": n_all / (solo_ms * 1e-3),
                       "speedup": solo_ms / (ms_max / steps),
                       "sample": f"each disk alone through nbody_sim, {args.solo_steps} steps "
                                 "after 2 warm-up, per-step times summed"},
        "e2e": {"value": n_all * e_steps / (e_ms * 1e-3), "unit": UNIT,
                "h2d_bytes_per_step": n * (6 * 8 + 3 * 4 + 4),
                "d2h_bytes_per_step": n * (6 * 8 + 3 * 4),
                "ms_per_step": e_ms / e_steps},
        "clocks": ck,
    }
    ens.close()
    return line


def run_precision(args, ws, rank, local):
    """Precision study on the headline disk (N = 2^20, r in [0.3, 30] AU,
    m = 1e-9, eps = 5e-4, dt = 0.002, gravity only, so E and L_y are
    conserved).  (1) Relative error of the walk's total and self-gravity
    accelerations against the FP64 direct sum on a seeded random subset of
    targets, theta in {0.3, 0.5, 0.7}.  (2) |dE/E| and |dL_y/L_y| after
    --drift-steps steps at theta 0.5 for FP32, FP64 and hi/lo float-pair
    state, with the softened pair energy summed directly in FP64."""
    import torch
    if rank != 0:
        return
    nb = importlib.import_module("nbody-sim_b200")
    dg = importlib.import_module("nbody-sim_b200.diagnostics")
    torch.cuda.set_device(local)
    n, w = args.n, WORKLOAD
    ic = make_ic(nb, n, 0, np.float64)
    targets = np.sort(np.random.default_rng(0).choice(n, min(args.targets, n), replace=False))
    st32 = {k: ic[k].astype(np.float32) for k in ("x", "y", "z")}
    st32["m"] = ic["m"]
    forces = {}
    for theta in (0.3, 0.5, 0.7):
        forces[f"{theta}"] = dg.force_errors(st32, theta, w["eps"], 1.0, targets)
    drift = {}
    stream = torch.cuda.current_stream()
    for name, prec in (("f32", nb.STATE_F32), ("f64", nb.STATE_F64),
                       ("f32x2", nb.STATE_F32X2)):
        prm = nb.sim_params(dt=w["dt"], theta=0.5, softening=w["eps"], star_mass=1.0,
                            r_coll=0.0, restitution=0.0, gas_drag_rate=0.0,
                            state_precision=prec, leaf_max=args.leaf_max)
        sim = nb.Sim(prm, n)
        sim.set_stream(stream.cuda_stream)
        dt_ = np.float32 if prec == nb.STATE_F32 else np.float64
        sim.set_state(*[ic[k].astype(dt_) for k in ("x", "y", "z", "vx", "vy", "vz")], ic["m"])
        c0 = dg.conserved(sim.get_state(double=True), ic["m"], w["eps"], 1.0)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        sim.step(args.drift_steps)
        b.record(stream)
        sim.sync()
        ms = a.elapsed_time(b) / args.drift_steps
        c1 = dg.conserved(sim.get_state(double=True), ic["m"], w["eps"], 1.0)
        sim.close()
        drift[name] = {"dE_over_E": abs(c1["E"] - c0["E"]) / abs(c0["E"]),
                       "dLy_over_Ly": abs(c1["L_y"] - c0["L_y"]) / abs(c0["L_y"]),
                       "ms_per_step": ms, "E0": c0, "E1": c1}
    line = {
        "study": "precision", "n": n, "targets": len(targets), "data": "synthetic",
        "config": {"workload": f"Keplerian disk N={n} r=[0.3,30] AU m=1e-9 eps=5e-4 dt=0.002, "
                               "gravity only", "drift_steps": args.drift_steps,
                   "drift_theta": 0.5,
                   "leaf_max": args.leaf_max or "engine default (12 from 2^19 bodies, else 8)"},
        "force_error_vs_fp64_direct": forces, "drift": drift,
    }
    print(json.dumps(line), flush=True)


def run_adjoint(args, ws, rank, local):
    if rank != 0:
        return
    import torch
    torch.cuda.set_device(local)
    print(json.dumps(adjoint_study(args, args.fd_components)), flush=True)


def adjoint_study(args, fd_components):
    """Gradient study: N = 65536 disk (r in [0.5, 5] AU, m = 1e-8, eps 1e-3),
    gas drag 1e-3, perturber 3 M_J at 10 AU, 200 steps of dt 0.005, FP64
    state.  Loss: mass-weighted mean e^2 of the bodies ending inside 2 AU.
    Gradients with respect to every initial velocity and the perturber's mass
    and radius through the adjoint engine; checked against FP64 central
    differences (h = 1e-6 relative) of the frozen-tree forward on a seeded
    set of velocity components and both perturber parameters.  Costs: the
    recording forward and the backward against the plain engine
    (nbody_sim, FP64 state, same physics) over the same steps."""
    import torch
    nb = importlib.import_module("nbody-sim_b200")
    n, steps, pm, pr = 65536, 200, 3.0, 10.0
    prm = nb.sim_params(dt=0.005, theta=0.5, softening=1e-3, star_mass=1.0, r_coll=0.0,
                        restitution=0.0, gas_drag_rate=1e-3, perturber_enabled=1,
                        perturber_mass_mjup=pm, perturber_radius_au=pr, perturber_phase0=0.0,
                        state_precision=nb.STATE_F64, leaf_max=args.leaf_max)
    d = nb.make_disk(n, 0.5, 5.0, 0.01, 0.005, 1.0, 0)
    x0 = torch.tensor(np.stack([d["x"], d["y"], d["z"]]), dtype=torch.float64, device="cuda")
    v0 = torch.tensor(np.stack([d["vx"], d["vy"], d["vz"]]), dtype=torch.float64, device="cuda")
    mass = torch.full((n,), 1e-8, dtype=torch.float32, device="cuda")
    stream = torch.cuda.current_stream()

    # plain forward: the engine, same physics and steps
    sim = nb.Sim(prm, n)
    sim.set_stream(stream.cuda_stream)
    m_np = np.full(n, 1e-8, np.float32)
    sim.set_state(d["x"], d["y"], d["z"], d["vx"], d["vy"], d["vz"], m_np)
    sim.step(5)
    sim.sync()
    sim.set_state(d["x"], d["y"], d["z"], d["vx"], d["vy"], d["vz"], m_np)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    sim.step(steps)
    b.record(stream)
    sim.sync()
    plain_ms = a.elapsed_time(b)
    sim.close()

    def gradient(eng):
        """Warm-up (sizes the tape pool, captures the forward and backward
        graphs), then the measured gradient through torch.autograd."""
        eng.set_stream(stream.cuda_stream)
        eng.forward(x0, v0, mass, pm, pr)
        eng.backward(torch.zeros_like(x0), torch.zeros_like(v0))
        x0r = x0.clone().requires_grad_(True)
        v0r = v0.clone().requires_grad_(True)
        pmt = torch.tensor(pm, dtype=torch.float64, device="cuda", requires_grad=True)
        prt = torch.tensor(pr, dtype=torch.float64, device="cuda", requires_grad=True)
        x, v = nb.disk_trajectory(eng, x0r, v0r, pmt, prt, mass)
        loss = nb.eccentricity_loss(x, v, mass)
        loss.backward()
        return (float(loss.item()), x0r.grad, v0r.grad, float(pmt.grad), float(prt.grad),
                eng.stats())

    eng = nb.Adjoint(prm, n, steps)
    loss, gx0, gv0, g_pm, g_pr, st = gradient(eng)

    def loss_diff(plus, minus):
        (xp, vp), (xm, vm) = plus, minus
        rp = torch.sqrt((xp * xp).sum(0))
        w = mass.to(torch.float64) * (rp < 2.0).to(torch.float64)
        dd = nb.eccentricity2(xp, vp) - nb.eccentricity2(xm, vm)
        return float(((w * dd).sum() / w.sum()).item())

    speed = torch.sqrt((v0 * v0).sum(0))
    rng = np.random.default_rng(0)
    picks = rng.choice(3 * n, min(fd_components, 3 * n), replace=False)
    def fd_v(c, k, hrel):
        h = hrel * float(speed[k])
        vp = v0.clone(); vp[c, k] += h
        vm = v0.clone(); vm[c, k] -= h
        return loss_diff(eng.replay(x0, vp, pm, pr, fp64=True),
                         eng.replay(x0, vm, pm, pr, fp64=True)) / (2 * h)

    # Central differences of the FP64 frozen-tree replay at h = 1e-6 of each
    # body's speed; a component that misses 1e-4 there is re-taken at 1e-5
    # and 1e-4.  The quotient's round-off falls as 1/h and its truncation
    # error grows as h^2, so a component whose error falls ~10x per 10x in h
    # is round-off-limited at the small step.
    rels, rels_best, abs_best, skipped, misses = [], [], [], 0, []
    gnorm = float(gv0.abs().max())
    t0 = time.perf_counter()
    for q in picks:
        c, k = int(q) // n, int(q) % n
        g_fd = fd_v(c, k, 1e-6)
        g_ad = float(gv0[c, k])
        scale = max(abs(g_ad), abs(g_fd))
        if scale < 1e-6 * gnorm:  # bodies that barely touch the loss: no signal to check
            skipped += 1
            continue
        r6 = abs(g_ad - g_fd) / scale
        rels.append(r6)
        best, err = r6, abs(g_ad - g_fd)
        if r6 > 1e-4:
            row = {"component": [c, k], "adjoint": g_ad, "rel_h1e-6": r6}
            for hrel in (1e-5, 1e-4):
                gh = fd_v(c, k, hrel)
                rh = abs(g_ad - gh) / max(abs(g_ad), abs(gh))
                row[f"rel_h{hrel:g}"] = rh
                best, err = min(best, rh), min(err, abs(g_ad - gh))
            misses.append(row)
        rels_best.append(best)
        abs_best.append(err)
    fd_secs = time.perf_counter() - t0
    par = {}
    for name, g_ad, base in (("perturber_mass_mjup", g_pm, pm),
                             ("perturber_radius_au", g_pr, pr)):
        row = {"adjoint": g_ad}
        for hrel in (1e-4, 1e-5, 1e-6):
            dpm = hrel * pm if name.startswith("perturber_mass") else 0.0
            dpr = hrel * pr if dpm == 0.0 else 0.0
            g_fd = loss_diff(eng.replay(x0, v0, pm + dpm, pr + dpr, fp64=True),
                             eng.replay(x0, v0, pm - dpm, pr - dpr, fp64=True)) / (2 * hrel * base)
            row[f"fd_h{hrel:g}"] = g_fd
            row[f"rel_h{hrel:g}"] = abs(g_ad - g_fd) / max(abs(g_ad), abs(g_fd), 1e-300)
        par[name] = row
    eng.close()
    rels = np.array(rels)
    rels_best = np.array(rels_best)

    # the checkpointed engine: FP64 states every 50 levels, the others rebuilt
    # backwards in time in the backward
    eng_c = nb.Adjoint(prm, n, steps, mode="checkpoint", checkpoint_every=50)
    _, gx_c, gv_c, gpm_c, gpr_c, st_c = gradient(eng_c)
    eng_c.close()
    # the reference gradient: the same loss with FP64 direct-sum self-gravity
    eng_d = nb.Adjoint(prm, n, steps, mode="direct")
    t1 = time.perf_counter()
    _, gx_d, gv_d, gpm_d, gpr_d, st_d = gradient(eng_d)
    direct_secs = time.perf_counter() - t1
    eng_d.close()

    def relmax(a, b):
        return float((a - b).abs().max() / b.abs().max())

    line = {
        "study": "adjoint", "n": n, "steps": steps, "data": "synthetic",
        "config": {"workload": "Keplerian disk N=65536 r=[0.5,5] AU m=1e-8 eps=1e-3, drag 1e-3, "
                               "perturber 3 MJ at 10 AU, dt 0.005, 200 steps, FP64 state, "
                               "theta 0.5", "loss": "mass-weighted mean e^2, final r < 2 AU"},
        "loss": loss,
        "ms": {"plain_forward": plain_ms, "recording_forward": st.ms_forward,
               "backward": st.ms_backward,
               "gradient_over_plain_forward": (st.ms_forward + st.ms_backward) / plain_ms,
               "backward_over_plain_forward": st.ms_backward / plain_ms},
        "memory_bytes": {"tape": st.tape_bytes, "states": st.state_bytes},
        "checkpointed": {"every": 50, "forward_ms": st_c.ms_forward,
                         "backward_ms": st_c.ms_backward,
                         "gradient_over_plain_forward":
                             (st_c.ms_forward + st_c.ms_backward) / plain_ms,
                         "memory_bytes": {"tape": st_c.tape_bytes, "states": st_c.state_bytes},
                         "vs_tape_max_abs_err_over_max_grad": {
                             "velocity": relmax(gv_c, gv0), "position": relmax(gx_c, gx0)},
                         "vs_tape_rel": {"perturber_mass": abs(gpm_c - g_pm) / abs(g_pm),
                                         "perturber_radius": abs(gpr_c - g_pr) / abs(g_pr)}},
        "direct_sum_reference": {
            "what": "the same loss and step with FP64 direct-sum self-gravity; its gradient",
            "seconds": direct_secs, "forward_ms": st_d.ms_forward,
            "backward_ms": st_d.ms_backward,
            "tree_vs_direct_rel_l2": {"velocity": float((gv0 - gv_d).norm() / gv_d.norm()),
                                      "position": float((gx0 - gx_d).norm() / gx_d.norm())},
            "tree_vs_direct_rel": {"perturber_mass": abs(g_pm - gpm_d) / abs(gpm_d),
                                   "perturber_radius": abs(g_pr - gpr_d) / abs(gpr_d)}},
        "fd_check": {"components": int(len(picks)), "checked": int(len(rels)),
                     "skipped_no_signal": skipped,
                     "max_rel": float(rels.max()) if len(rels) else None,
                     "median_rel": float(np.median(rels)) if len(rels) else None,
                     "p99_rel": float(np.percentile(rels, 99)) if len(rels) else None,
                     "within_1e-4": int((rels <= 1e-4).sum()),
                     "within_1e-4_best_h": int((rels_best <= 1e-4).sum()),
                     "max_rel_best_h": float(rels_best.max()) if len(rels_best) else None,
                     # the worst disagreement against the gradient's largest component: the
                     # quotient's round-off is about the same for every component, so this
                     # is the check that does not punish components with little signal
                     "max_abs_err_over_max_grad": float(max(abs_best) / gnorm) if abs_best else None,
                     "misses_at_h1e-6": misses[:40],
                     "seconds": fd_secs},
        "perturber": par,
    }
    return line


def run_c2(args, ws, rank, local):
    """The full-physics run end to end through the reference's loop
    (src/main.cu:85-190): N = 131072, r in [0.5, 5] AU, m = 1e-8, eps 1e-3,
    collisions (factor 5, e = 0), drag 1e-3, perturber 1 M_J at 5.2 AU,
    dt 0.005, 2000 steps, frame + aggregates every 50 steps (40 outputs)
    written to frames.bin / stats.csv, FP64 state.  Wall-clock particle-steps/s
    with the GPU output pipeline and with the reference's stop-copy-detect-write
    order (GPU FoF), and without outputs; the reference's own detectAggregates
    (one host thread, the O(N^2) loop) timed on one snapshot as the CPU
    baseline of the output step."""
    import shutil
    import tempfile
    import torch
    if rank != 0:
        return
    nb = importlib.import_module("nbody-sim_b200")
    run = importlib.import_module("nbody-sim_b200.run")
    torch.cuda.set_device(local)
    cfg = nb.default_config()
    cfg.n_particles = 131072
    cfg.disk_r_min, cfg.disk_r_max = 0.5, 5.0
    cfg.particle_mass_msun = 1e-8
    cfg.softening_AU = 1e-3
    cfg.theta = 0.5
    cfg.collision_radius_factor = 5.0
    cfg.restitution = 0.0
    cfg.gas_drag_rate = 1e-3
    cfg.dt = 0.005
    cfg.total_time = 10.0
    cfg.output_every_n_steps = 50
    cfg.perturber_enabled = 1
    cfg.perturber_mass_mjup = 1.0
    cfg.perturber_radius_AU = 5.2
    cfg.perturber_phase0 = 0.0
    n = cfg.n_particles
    total = int(np.float32(cfg.total_time) / np.float32(cfg.dt))
    res = {}
    tmp = tempfile.mkdtemp(prefix="nbody_c2_")
    try:
        # warm-up (library init, allocations)
        run.run_simulation(cfg, os.path.join(tmp, "warm"), precision=nb.STATE_F64,
                           total_steps=100)
        for name, pipelined in (("pipelined", True), ("synchronous", False)):
            d = os.path.join(tmp, name)
            r = run.run_simulation(cfg, d, precision=nb.STATE_F64, pipelined=pipelined)
            r["frames_bytes"] = os.path.getsize(os.path.join(d, "frames.bin"))
            res[name] = r
        same = all(open(os.path.join(tmp, "pipelined", f), "rb").read() ==
                   open(os.path.join(tmp, "synchronous", f), "rb").read()
                   for f in ("frames.bin", "stats.csv"))
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    # stepping alone
    prm = nb.sim_params(cfg)
    prm.state_precision = nb.STATE_F64
    dsk = nb.make_disk(n, 0.5, 5.0, 0.01, 0.005, 1.0, 0)
    sim = nb.Sim(prm, n)
    m = np.full(n, cfg.particle_mass_msun, np.float32)
    sim.set_state(dsk["x"], dsk["y"], dsk["z"], dsk["vx"], dsk["vy"], dsk["vz"], m)
    sim.step(10)
    sim.sync()
    t0 = time.perf_counter()
    sim.step(total)
    sim.sync()
    step_secs = time.perf_counter() - t0
    sim.close()
    line = {
        "study": "c2run", "data": "synthetic",
        "config": {"workload": "Keplerian disk N=131072 r=[0.5,5] AU m=1e-8 eps=1e-3, "
                               "collisions (factor 5), drag 1e-3, perturber 1 MJ at 5.2 AU, "
                               "dt 0.005, 2000 steps, output every 50, FP64 state"},
        "steps": total, "outputs": res["pipelined"]["frames"],
        "particle_steps_per_s": {k: v["particle_steps_per_s"] for k, v in res.items()},
        "seconds": {k: v["seconds"] for k, v in res.items()},
        "host_seconds": {k: v["host_seconds"] for k, v in res.items()},
        "stepping_only_seconds": step_secs,
        "output_overhead_seconds": {k: v["seconds"] - step_secs for k, v in res.items()},
        "frames_bytes": res["pipelined"]["frames_bytes"],
        "pipelined_equals_synchronous_bytes": same,
    }
    if not args.no_cpu_baseline:
        ref = os.path.join(ROOT, "oracle", "_ref", "libref_host.so")
        if os.path.exists(ref):
            sys.path.insert(0, os.path.join(ROOT, "oracle"))
            import oracle
            rh = oracle.RefHost(ref)
            xs = [dsk[k].astype(np.float32) for k in ("x", "y", "z")]
            t0 = time.perf_counter()
            rh.detect_aggregates_count(*xs, float(prm.r_coll))
            secs = time.perf_counter() - t0
            line["cpu_baseline"] = {
                "value": secs, "unit": "s per output (detectAggregates)", "cores": 1,
                "kind": "reference",
                "sample": "the reference's Aggregate.cpp detectAggregates on one N=131072 "
                          "snapshot (its O(N^2) pair loop), x40 outputs in a C2 run"}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    ws, rank, local = dist_setup()
    try:
        if args.impl == "reference":
            run_reference(args, ws, rank)
        elif args.workload == "ensemble":
            run_ensemble(args, ws, rank, local)
        elif args.workload == "precision":
            run_precision(args, ws, rank, local)
        elif args.workload == "adjoint":
            run_adjoint(args, ws, rank, local)
        elif args.workload == "c2run":
            run_c2(args, ws, rank, local)
        else:
            run_ours(args, ws, rank, local)
    finally:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
