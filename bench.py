#!/usr/bin/env python3
"""Benchmark: particle-steps/s of the Barnes-Hut evolution step on B200.

Workload (one GPU): cold collapse of a uniform unit disc, N = 2^20 equal
masses (total 1, G = 1), f32 state, eps = 0.005, theta = 0.5, bucket 1,
32-bit Morton codes, full tree rebuild every step, KDK leapfrog dt = 5e-4,
seed 7.  One "step" = kick/drift + bounds + Morton + stable radix sort +
topology + aggregates + theta-MAC traversal + final kick over all bodies.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]

Prints one JSON line (rank 0).  With N > 1 (launched by torchrun) every rank
advances its own replica of the workload (the path does not shard: replicas
only, weak scaling); time is the max over ranks.  ``--impl reference`` times
the reference's CPU flat-tree evolution (its C restatement, all host
threads) on the same workload.
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_BODIES = 1 << 20
THETA, EPS, G, BUCKET, DT, SEED = 0.5, 0.005, 1.0, 1, 5e-4, 7
METRIC = "particle-steps/s"
# DRAM bytes (ncu dram__bytes_read.sum + dram__bytes_write.sum) of integrate,
# Morton, 4 radix passes, count/scan, cells and aggregate for one step at
# N=2^20, from one capture of this bench's workload; re-measured whenever one
# of those kernels changes
BUILD_DRAM_BYTES_PER_STEP = 465.5e6
WORKLOAD = "cold-collapse uniform disc N=2^20, eps=0.005, theta=0.5, bucket=1, dt=5e-4, seed 7"

def algorithmic_bytes(c: float) -> dict:
    """Bytes per body-step each HBM-bound stage must move (reads + writes) in
    the reference's record layout (32 B state, 16 B accel, 8 B key+index,
    64 B cells); c = cells per body (measured).  Total 264 + 160c."""
    return {
        # fused leapfrog + bounds partials: read 32 B state + 16 B accel, write 32 B
        "integrate": 80.0,
        # Morton: read 32 B state, write 8 B key+index
        "morton": 40.0,
        # 4 stable 8-bit passes (4 + 4x16) plus positions and the sorted
        # gather (read 4 + 32, write 4 + 16), which the last pass performs
        "radix": 68.0 + 56.0,
        # topology: read 4 B codes, write 64 B per cell
        "topology": 4.0 + 64.0 * c,
        # aggregates: read 64 B per cell + 16 B sorted body, write 32 B per cell
        "aggregate": 16.0 + 96.0 * c,
    }


def load_peaks() -> dict:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return {"hbm_gbs": d["hbm_gbs"], "source": "measured", "sm_max_mhz": d.get("sm_max_mhz")}
    return {"hbm_gbs": 6650.0, "source": "fallback", "sm_max_mhz": 1965.0}


class ClockSampler:
    """nvidia-smi sampling of SM clock and throttle reasons during a region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100", "-i", str(self.index)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            time.sleep(0.3)
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.t.join(timeout=2)

    def summary(self) -> dict:
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx),
                "reasons": sorted(reasons), "samples": len(sm)}


class HostNumaBinding:
    """Binds this process to the host CPUs that NVML lists as local to the GPU.

    Used around the legs that copy host buffers: pinned pages are first touched
    and copies issued from the GPU's own NUMA node instead of across the socket
    link.  A process setting only (sched_setaffinity); the previous CPU set is
    restored on exit.  Nothing on the GPU changes."""

    def __init__(self, device: int):
        self.device = device
        self.saved = None
        self.cpus = None

    def local_cpus(self):
        try:
            import pynvml
            import torch
            pynvml.nvmlInit()
            try:
                p = torch.cuda.get_device_properties(self.device)
                bus = f"{p.pci_domain_id:08x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0"
                h = pynvml.nvmlDeviceGetHandleByPciBusId(bus)
                words = (os.cpu_count() + 63) // 64
                mask = pynvml.nvmlDeviceGetCpuAffinity(h, words)
            finally:
                pynvml.nvmlShutdown()
        except Exception:
            return None
        cpus = {w * 64 + b for w in range(len(mask)) for b in range(64) if (mask[w] >> b) & 1}
        cpus &= os.sched_getaffinity(0)
        return cpus or None

    def __enter__(self):
        self.cpus = self.local_cpus()
        if self.cpus:
            self.saved = os.sched_getaffinity(0)
            os.sched_setaffinity(0, self.cpus)
        return self

    def __exit__(self, *exc):
        if self.saved:
            os.sched_setaffinity(0, self.saved)

    def summary(self) -> dict:
        return {"bound": bool(self.cpus), "cpus": len(self.cpus) if self.cpus else None}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        backend = "gloo" if args.impl == "reference" else "nccl"
        if backend == "nccl":
            import torch
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
        pg = dist
    return world, rank, local, pg


def config_dict(world: int) -> dict:
    """The workload's config, identical in the engine and reference arms."""
    return {"workload": WORKLOAD, "n_bodies": N_BODIES, "theta": THETA, "eps": EPS,
            "bucket": BUCKET, "dt": DT, "parallelism": f"replicas x{world}",
            "l2": "working set > L2 (state 32 MiB + accel 16 MiB + sort keys 24 MiB + cells "
                  "~180 MiB touched per step)"}


def f32_workload():
    from galaxy_b200 import scenarios
    from galaxy_b200.nbody_gpu import bodies_to_state
    bodies = scenarios.cold_disc(N_BODIES, SEED)
    return bodies, bodies_to_state(bodies)


# ------------------------------------------------------------ reference --

def reference_kernels(s) -> dict | None:
    """The reference's own CUDA kernels (runtime/cuda/barnes_hut_flat.cu,
    compiled unmodified from its source into oracle/_ref): bh_traverse over
    the packed tree of the workload's initial state (its CPU tree,
    pack_flat_tree), bh_kick_drift and bh_final_kick over the same bodies, in
    128-thread groups as nbody_gpu.rs dispatches them.  Median device ms of
    single launches, each bracketed by its own events, with L2 warm and with
    L2 evicted before each launch (cold).  None when they were not built."""
    from galaxy_b200.nbody_gpu import state_to_bodies
    from oracle import oracle
    if oracle.ref_cuda() is None:
        return None
    b = np.ascontiguousarray(state_to_bodies(s))
    cfg = oracle.Config(theta=THETA, softening=EPS, g=G, bucket=BUCKET, max_depth=48)
    tree = oracle.build_flat_tree(b, cfg)
    packed = oracle.pack_flat_tree(b, tree, cfg)
    acc, _ = oracle.ref_cuda_traverse(packed, repeats=1)
    t = oracle.ref_cuda_single_times(packed, s.view(np.float32).reshape(-1, 8), acc, DT)
    out = {"tree": f"initial state of the workload (cold disc 2^20, seed 7), "
                   f"{len(packed.cells)} cells",
           "source": "runtime/cuda/barnes_hut_flat.cu (bh_traverse, bh_kick_drift, "
                     "bh_final_kick), 128-thread groups as nbody_gpu.rs dispatches them",
           "how": "median of single launches, device time (CUDA events); cold = L2 evicted "
                  "before each launch"}
    for k, (w, c) in t.items():
        out[k + "_ms"] = float(f"{w:.4g}")
        out[k + "_cold_ms"] = float(f"{c:.4g}")
    return out


def run_reference(args, world, rank, pg):
    """The reference's CPU flat-tree evolution (cpu_flat_evolve,
    galaxy-bh-evolve.rs:339-363) through its C restatement, all host threads,
    on the same workload: W untimed warm-up steps, then K timed steps, each
    one full KDK step at N = 2^20 (the timed steps stop early at a 150 s
    budget and the rate covers the steps that ran).  The line also carries
    the reference's own CUDA kernels timed on the workload's tree."""
    if rank != 0:
        if pg:
            pg.barrier()
            pg.destroy_process_group()
        return
    from galaxy_b200.nbody_gpu import state_to_bodies
    from oracle import oracle
    threads = os.cpu_count() or 1
    _, s = f32_workload()
    try:
        kernels = reference_kernels(s)
    except Exception as exc:  # the kernels are a side figure; the CPU arm stands alone
        kernels = {"unavailable": f"{type(exc).__name__}: {exc}"[:200]}
    b = np.ascontiguousarray(state_to_bodies(s))
    cfg = oracle.Config(theta=THETA, softening=EPS, g=G, bucket=BUCKET, max_depth=48)
    tree = oracle.build_flat_tree(b, cfg)
    acc, _ = oracle.flat_accelerations(b, tree, cfg, nthreads=threads)
    acc = np.ascontiguousarray(acc)
    warm = max(args.warmup, 0)
    for _ in range(warm):
        oracle.cpu_flat_steps(b, acc, 1, DT, cfg, threads)
    t0 = time.perf_counter()
    done = 0
    tb = tf = 0.0
    while done < args.steps:
        b1, f1 = oracle.cpu_flat_steps(b, acc, 1, DT, cfg, threads)
        tb += b1
        tf += f1
        done += 1
        if time.perf_counter() - t0 > 150.0:
            break
    secs = time.perf_counter() - t0
    value = N_BODIES * done / secs
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": METRIC,
        "n_gpus": args.gpus, "steps": done, "warmup": warm,
        "ms_per_step": 1e3 * secs / done, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded cold uniform disc)",
        "config": config_dict(world),
        "cpu_baseline": {"value": value, "unit": METRIC, "cores": threads, "kind": "port",
                         "sample": f"{done} KDK steps at N=2^20 (of {args.steps} requested; "
                                   f"150 s budget); tree build {tb:.2f} s single-threaded, "
                                   f"forces {tf:.2f} s on {threads} threads"},
        "e2e": {"value": value, "unit": METRIC, "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "reference_kernels": kernels,
    }
    print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()


# --------------------------------------------------------------- engine --

def cpu_baseline_sample() -> dict:
    """One single-threaded KDK step of the oracle at the full workload size
    (the reference CPU path is single-threaded)."""
    from galaxy_b200.nbody_gpu import state_to_bodies
    from oracle import oracle
    _, s = f32_workload()
    b = np.ascontiguousarray(state_to_bodies(s))
    cfg = oracle.Config(theta=THETA, softening=EPS, g=G, bucket=BUCKET, max_depth=48)
    tree = oracle.build_flat_tree(b, cfg)
    acc, _ = oracle.flat_accelerations(b, tree, cfg, nthreads=os.cpu_count() or 1)
    acc = np.ascontiguousarray(acc)
    t0 = time.perf_counter()
    tb, tf = oracle.cpu_flat_steps(b, acc, 1, DT, cfg, 1)
    secs = time.perf_counter() - t0
    return {"value": N_BODIES / secs, "unit": METRIC, "cores": 1, "kind": "port",
            "sample": f"1 KDK step at N=2^20, single thread (tree build {tb:.2f} s, "
                      f"forces {tf:.2f} s)"}


def cpu_config1_sample(steps: int = 100) -> dict:
    """The reference CPU path on config 1 (exponential disc, N = 16,384, eps
    0.01, theta 0.5, bucket 1, dt 1e-3, seed 42): `steps` single-threaded KDK
    steps of its C restatement (all 100 of the config by default, ~10 s)."""
    from galaxy_b200 import scenarios
    from galaxy_b200.nbody_gpu import bodies_to_state, state_to_bodies
    from oracle import oracle
    b = np.ascontiguousarray(state_to_bodies(bodies_to_state(scenarios.exponential_disc(
        16384, 42, eps=0.01))))
    cfg = oracle.Config(theta=0.5, softening=0.01, g=1.0, bucket=1, max_depth=48)
    tree = oracle.build_flat_tree(b, cfg)
    acc, _ = oracle.flat_accelerations(b, tree, cfg, nthreads=1)
    acc = np.ascontiguousarray(acc)
    t0 = time.perf_counter()
    oracle.cpu_flat_steps(b, acc, steps, 1e-3, cfg, 1)
    secs = time.perf_counter() - t0
    return {"value": 16384 * steps / secs, "unit": METRIC, "cores": 1, "kind": "port",
            "sample": (f"{steps} of the config's 100 KDK steps" if steps < 100 else
                       "the config's 100 KDK steps (boundary solve untimed)") + ", single thread"}


def run_config1_leg(gpu, rt) -> dict:
    """Config 1: rotating exponential disc, N = 16,384, total mass 1, G 1,
    eps 0.01, theta 0.5, bucket 1, 100 KDK steps at dt 1e-3 from seed 42;
    FP64 direct-sum error of the final forces at every body."""
    import numpy as np
    import torch

    from galaxy_b200 import scenarios
    from galaxy_b200.nbody_gpu import Config
    cfg = Config(theta=0.5, softening_kpc=0.01, g=1.0, bucket=1, max_depth=48)
    bodies = scenarios.exponential_disc(16384, 42, eps=0.01)
    stream = torch.cuda.ExternalStream(gpu.stream_ptr())
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    warm, _ = gpu.create_evolving_state(bodies)  # graphs and arena, untimed
    tw = rt.create_tree(gpu, warm, cfg)
    rt.rebuild(gpu, warm, tw, cfg)
    rt.force(gpu, warm, tw, cfg)
    rt.step(gpu, warm, tw, cfg, 1e-3, 5)
    tw.close()
    warm.close()
    ev, _ = gpu.create_evolving_state(bodies)
    tree = rt.create_tree(gpu, ev, cfg)
    torch.cuda.synchronize()
    e0.record(stream)
    rt.rebuild(gpu, ev, tree, cfg)  # the boundary solve is part of the run
    rt.force(gpu, ev, tree, cfg)
    rt.step(gpu, ev, tree, cfg, 1e-3, 100)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    err = gpu.probe_error(ev, cfg, np.arange(16384, dtype=np.uint32))
    tree.close()
    ev.close()
    return {"workload": "exponential disc N=16384, eps 0.01, theta 0.5, bucket 1, dt 1e-3, "
                        "seed 42, 100 KDK steps (boundary solve included)",
            "value": 16384 * 100 / (ms * 1e-3), "unit": METRIC, "ms_per_step": ms / 100,
            "force_error_all_bodies": err}


def r4(x):
    """Four significant digits (None passes through) for the compact summary."""
    return None if x is None else float(f"{x:.4g}")


def per_body_force_error(gpu, rt, ev, tree, cfg) -> dict:
    """Per-body relative error of the f32 forces of the plain and the
    compensated summation forms against the reference's own f64 flat
    traversal of the same tree (galaxy_bh_force_f64, flat.rs:270-371, the
    same cells, order and f64 arithmetic as the CPU reference), at every
    body; for the bodies above 1e-5, S/|a| (S = sum of the body's term
    magnitudes) says how far their terms cancel.  The opening decisions
    are compared through the two traversals' counters (cells visited,
    approximated, bodies summed directly): their differences count MAC flips
    in aggregate.  Leaves the plain forces (the step's own) in the state."""
    ref, s, f64_counts = rt.force_f64(gpu, ev, tree, cfg, abs_sum=True)
    mag = np.hypot(ref[:, 0], ref[:, 1])
    ratio = s / np.maximum(mag, 1e-300)
    out = {"against": "galaxy_bh_force_f64 (reference f64 flat traversal, same tree)",
           "bodies": int(len(ref)), "S_over_a_median": r4(float(np.median(ratio)))}
    rt.force(gpu, ev, tree, dataclasses.replace(cfg, compensated=False, force_stats=True))
    f32_counts = rt.force_stats(gpu, tree)
    out["decisions"] = {"f64": f64_counts, "f32": {k: f32_counts[k] for k in f64_counts},
                        "differences": {k: int(f32_counts[k] - v) for k, v in f64_counts.items()},
                        "identical": all(f32_counts[k] == v for k, v in f64_counts.items())}
    for name, comp in (("compensated", True), ("plain", False)):
        c = dataclasses.replace(cfg, compensated=comp, force_stats=False)
        rt.force(gpu, ev, tree, c)
        acc, _ = gpu.read_evolving_accelerations(ev)
        err = np.hypot(acc[:, 0] - ref[:, 0], acc[:, 1] - ref[:, 1])
        rel = err / np.maximum(mag, 1e-30)
        above = rel > 1e-5
        bound_ok = bool((err <= 1e-5 * mag + 2e-6 * s).all())
        d = {"above_1e-5": int(above.sum()), "fraction_above": r4(float(above.mean())),
             "median": r4(float(np.median(rel))), "p99": r4(float(np.quantile(rel, 0.99))),
             "max": r4(float(rel.max())), "within_1e-5_a_plus_2e-6_S": bound_ok}
        if above.any():
            d["S_over_a_of_above_min"] = r4(float(ratio[above].min()))
            d["S_over_a_of_above_median"] = r4(float(np.median(ratio[above])))
        out[name] = d
    return out


def same_tree_kernels(gpu, rt, s0, cfg, reps: int = 7) -> dict:
    """This engine's kernels on the tree of the workload's initial state,
    the tree the reference arm hands the reference's own CUDA kernels
    (runtime/cuda/barnes_hut_flat.cu): the BH #2B1 packed traversal of the
    same packed records (galaxy_bh_traverse_packed), the engine's own
    traversal of that tree (galaxy_bh_force), and the kick/drift (with the
    fused bounds reduction) and final kick.  Median device ms of `reps`
    single calls, each kernel bracketed by its own events, as the reference
    arm times the reference's kernels: "warm" right after the previous call,
    "cold" after a 256 MiB write that evicts L2 (the packed traversal
    uploads its tree first, so it has only the one figure)."""
    import torch
    ev, _ = gpu.create_evolving_state_records(s0)
    tree = rt.create_tree(gpu, ev, cfg)
    rt.rebuild(gpu, ev, tree, cfg)
    packed = rt.read_evidence(gpu, tree).packed(cfg)
    plain = dataclasses.replace(cfg, force_stats=False)
    stream = torch.cuda.ExternalStream(gpu.stream_ptr())
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def timed(call, cold):
        out = []
        for r in range(reps):
            if cold:
                with torch.cuda.stream(stream):
                    flush.fill_(r & 0xFF)
            out.append(call() * 1e3)
        return r4(float(np.median(out)))

    res = {"tree": "initial state of the workload (cold disc 2^20, seed 7), "
                   f"{len(packed.cells)} cells",
           "how": "median of single calls, device time of the kernel (CUDA events); cold = "
                  "L2 evicted before each call"}
    res["traverse_packed_ms"] = timed(lambda: gpu.traverse(packed).dispatch_seconds, False)
    for cold in (False, True):
        sfx = "_cold_ms" if cold else "_ms"
        res["traverse" + sfx] = timed(lambda: rt.force(gpu, ev, tree, plain).dispatch_seconds,
                                      cold)
        res["kick_drift" + sfx] = timed(lambda: gpu.kick_drift(ev, DT).dispatch_seconds, cold)
        res["final_kick" + sfx] = timed(lambda: gpu.final_kick(ev, DT).dispatch_seconds, cold)
        # the pass the fused step runs between steps: final kick + kick/drift
        # + bounds, against the reference's two launches per step
        res["final_kick_drift" + sfx] = timed(
            lambda: gpu.final_kick_drift(ev, DT).dispatch_seconds, cold)
    del flush
    tree.close()
    ev.close()
    return res


def run_engine(args, world, rank, local, pg):
    import torch

    from galaxy_b200 import _lib, shard
    from galaxy_b200.nbody_gpu import Config, NbodyGpu, ParallelTreeRuntime

    torch.cuda.set_device(local)
    gpu = NbodyGpu(str(local))
    rt = ParallelTreeRuntime(gpu)
    cfg = Config(theta=THETA, softening_kpc=EPS, g=G, bucket=BUCKET, max_depth=48)
    bodies, s0 = f32_workload()
    if args.only_batched:
        # the batched leg alone (for profilers; its timed steps sit in an
        # NVTX range "batched")
        batched = run_batched_leg(gpu, steps=min(args.steps, 20), warmup=args.warmup, pg=pg,
                                  rank=rank, world=world)
        if rank == 0:
            print(json.dumps({"batched": {k: batched[k] for k in
                                          ("bodies", "steps", "ms_per_step", "value",
                                           "speedup_vs_plain")},
                              "only_batched": True}), flush=True)
        if pg:
            pg.barrier()
            pg.destroy_process_group()
        return
    if args.only_same_tree:
        # the same-tree kernel timings alone (for profilers)
        kernels = same_tree_kernels(gpu, rt, s0, cfg)
        if rank == 0:
            print(json.dumps({"same_tree_kernels": kernels, "only_same_tree": True,
                              "config": config_dict(world)}), flush=True)
        if pg:
            pg.barrier()
            pg.destroy_process_group()
        return
    ev, _ = gpu.create_evolving_state_records(s0)
    tree = rt.create_tree(gpu, ev, cfg)
    rt.rebuild(gpu, ev, tree, cfg)
    rt.force(gpu, ev, tree, cfg)
    stream = torch.cuda.ExternalStream(gpu.stream_ptr(), device=torch.device("cuda", local))

    rt.step(gpu, ev, tree, cfg, DT, max(args.warmup, 3))
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clocks:
        torch.cuda.synchronize()
        if pg:
            pg.barrier()
        torch.cuda.nvtx.range_push("timed")  # ncu --nvtx --nvtx-include timed/
        e0.record(stream)
        rt.step(gpu, ev, tree, cfg, DT, args.steps)
        e1.record(stream)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
    ms = shard.max_over_ranks(pg, e0.elapsed_time(e1), "cuda")  # the slowest replica
    if pg:
        pg.barrier()
    value = world * N_BODIES * args.steps / (ms * 1e-3)
    if args.only_step:
        # the timed steps alone (for profilers: no other leg launches a kernel)
        tree.close()
        ev.close()
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": METRIC,
                              "n_gpus": world, "steps": args.steps,
                              "warmup": max(args.warmup, 3), "ms_per_step": ms / args.steps,
                              "only_step": True, "config": config_dict(world)}), flush=True)
        if pg:
            pg.barrier()
            pg.destroy_process_group()
        return

    # --- spread: the same steps as 10 shorter timed runs, p50/p99 per step
    rep_steps, rep_ms = 20, []
    for _ in range(10):
        e0.record(stream)
        rt.step(gpu, ev, tree, cfg, DT, rep_steps)
        e1.record(stream)
        torch.cuda.synchronize()
        rep_ms.append(shard.max_over_ranks(pg, e0.elapsed_time(e1), "cuda") / rep_steps)
    repeats = {"runs": len(rep_ms), "steps_each": rep_steps,
               "p50_ms_per_step": float(np.percentile(rep_ms, 50)),
               "p99_ms_per_step": float(np.percentile(rep_ms, 99)),
               "min_ms_per_step": float(min(rep_ms)), "max_ms_per_step": float(max(rep_ms))}

    # --- FP64 direct-sum error of the evolved state's forces, 4096 probes
    probes = np.random.default_rng(4096).choice(N_BODIES, 4096, replace=False)
    force_error = gpu.probe_error(ev, cfg, probes)
    force_error["theta"] = THETA

    # --- the same workload at the opening angle whose median FP64 error is
    # <= 1e-3 (theta = 0.12 on this workload; monopole cells at theta 0.5
    # give ~1.6e-2, inherent to the reference's MAC)
    acc_cfg = Config(theta=0.12, softening_kpc=EPS, g=G, bucket=BUCKET, max_depth=48)
    ev2, _ = gpu.create_evolving_state_records(s0)
    tree2 = rt.create_tree(gpu, ev2, acc_cfg)
    rt.rebuild(gpu, ev2, tree2, acc_cfg)
    rt.force(gpu, ev2, tree2, acc_cfg)
    rt.step(gpu, ev2, tree2, acc_cfg, DT, 2)
    acc_steps = max(3, min(args.steps // 10, 10))
    torch.cuda.synchronize()
    e0.record(stream)
    rt.step(gpu, ev2, tree2, acc_cfg, DT, acc_steps)
    e1.record(stream)
    torch.cuda.synchronize()
    acc_ms = e0.elapsed_time(e1) / acc_steps
    accurate = {"theta": 0.12, "value": world * N_BODIES / (acc_ms * 1e-3), "unit": METRIC,
                "ms_per_step": acc_ms, "steps": acc_steps,
                "force_error": gpu.probe_error(ev2, acc_cfg, probes)}
    tree2.close()
    ev2.close()

    # --- per-stage device times (instrumented rebuild + force, same state).
    # "integrate" is the step's own first kernel (kick/drift + bounds, the
    # 80 B/body leapfrog stage), timed on a scratch copy of the state;
    # "bounds" is the bounds-only pass a standalone rebuild runs instead.
    reps = 5
    stage = {"integrate": 0.0, "bounds": 0.0, "morton": 0.0, "radix": 0.0, "topology": 0.0,
             "aggregate": 0.0, "traverse": 0.0}
    cfg_plain = dataclasses.replace(cfg, force_stats=False)  # the kernel the step replays
    ev_scratch, _ = gpu.create_evolving_state_records(s0)
    for _ in range(reps):
        stage["integrate"] += gpu.kick_drift(ev_scratch, DT).dispatch_seconds / reps
        bt = rt.rebuild(gpu, ev, tree, cfg)
        ft = rt.force(gpu, ev, tree, cfg_plain)
        stage["bounds"] += bt.bounds_seconds / reps
        stage["morton"] += bt.morton_seconds / reps
        stage["radix"] += bt.radix_seconds / reps
        stage["topology"] += bt.topology_seconds / reps
        stage["aggregate"] += bt.aggregate_seconds / reps
        stage["traverse"] += ft.dispatch_seconds / reps
    ev_scratch.close()
    rt.force(gpu, ev, tree, cfg)
    fstats = rt.force_stats(gpu, tree)
    evid_meta_cells = tree_cells(gpu, rt, tree)
    # every body's f32 force (plain and compensated) against the reference's
    # f64 traversal of the same tree; restores the step's own forces
    per_body = per_body_force_error(gpu, rt, ev, tree, cfg)
    kernels = same_tree_kernels(gpu, rt, s0, cfg)
    c = evid_meta_cells / N_BODIES
    ab = algorithmic_bytes(c)
    peaks = load_peaks()
    # sort/build/leapfrog: every HBM-bound stage of the step
    hbm_bytes = N_BODIES * sum(ab.values())
    hbm_secs = stage["integrate"] + stage["morton"] + stage["radix"] + stage["topology"] + \
        stage["aggregate"]
    achieved = hbm_bytes / hbm_secs / 1e9
    interactions = fstats["approximated_cells"] + fstats["direct_terms"]
    flops = 20.0 * interactions
    clk = clocks.summary()
    sm_mhz = clk.get("sm_mhz") or peaks.get("sm_max_mhz") or 1965.0
    fp32_peak = 148 * 128 * 2 * sm_mhz * 1e6 / 1e12  # TFLOP/s at the sampled clock

    # --- end to end through the public API with host buffers
    e2e_steps = min(args.steps, 20)
    numa = HostNumaBinding(local)
    with numa:
        pinned = torch.empty(N_BODIES * 32, dtype=torch.uint8, pin_memory=True)
        host = pinned.numpy().view(_lib.EVOLVE_STATE_DTYPE)
        gpu_state, _ = gpu.read_evolving_state_records(ev)
        host[:] = gpu_state
        L = _lib.load()
        hp = host.ctypes.data
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e0.record(stream)
        for _ in range(e2e_steps):
            _lib.check(L.galaxy_bh_write_state(gpu.handle, ev.handle, hp, N_BODIES))
            rt.step(gpu, ev, tree, cfg, DT, 1)
            _lib.check(L.galaxy_bh_read_state(gpu.handle, ev.handle, hp, N_BODIES, None))
        e1.record(stream)
        torch.cuda.synchronize()
        e2e_wall = time.perf_counter() - t0
        del host, pinned
    e2e_ms = shard.max_over_ranks(pg, e0.elapsed_time(e1), "cuda")
    e2e_value = world * N_BODIES * e2e_steps / (e2e_ms * 1e-3)

    tree.close()
    ev.close()
    batched = None
    if not args.no_batched:
        batched = run_batched_leg(gpu, steps=min(args.steps, 20), warmup=args.warmup, pg=pg,
                                  rank=rank, world=world)
    served = None
    if not args.no_served:
        with HostNumaBinding(local):
            served = run_served_leg(gpu, capacity=(batched or {}).get("value", value), pg=pg,
                                    rank=rank, world=world)
    config1 = run_config1_leg(gpu, rt)
    roofline_large = run_large_roofline(gpu, rt, load_peaks()["hbm_gbs"])
    precision = None
    if not args.no_precision:
        precision = run_precision_leg(gpu, steps=args.precision_steps)
    if rank != 0:
        if pg:
            pg.barrier()
            pg.destroy_process_group()
        return
    cpu = None if args.no_cpu_baseline else cpu_baseline_sample()
    if cpu is not None:
        config1["cpu_baseline"] = cpu_config1_sample()
    stage_gbs = {k: round(N_BODIES * ab[m] / stage[k] / 1e9, 1) for k, m in
                 (("integrate", "integrate"), ("morton", "morton"), ("radix", "radix"),
                  ("topology", "topology"), ("aggregate", "aggregate")) if stage[k] > 0}
    traversal = {"bound": "fp32", "interactions_per_step": interactions,
                 "interactions_per_s": interactions / stage["traverse"],
                 "achieved_tflops": flops / stage["traverse"] / 1e12,
                 "peak_tflops": fp32_peak, "peak_source": "nominal FP32 at sampled clock",
                 "frac": flops / stage["traverse"] / 1e12 / fp32_peak,
                 "share_of_step": stage["traverse"] / (ms * 1e-3 / args.steps),
                 "cells_per_body": c, "exact_mac_fallbacks": fstats["exact_mac_fallbacks"],
                 "lane_visits": fstats["visited_nodes"],
                 "warp_iterations": fstats["warp_iterations"],
                 "union_over_lane": 32.0 * fstats["warp_iterations"] /
                 max(1, fstats["visited_nodes"])}
    summary = {
        "step_ms": r4(ms / args.steps),
        "roofline_frac": r4(achieved / peaks["hbm_gbs"]), "stage_gbs": stage_gbs,
        "roofline_n2p24_frac": r4(roofline_large["frac"]),
        "traversal_frac": r4(traversal["frac"]), "traversal_share": r4(traversal["share_of_step"]),
        "force_error_theta_0.5": {"median": r4(force_error["median"]),
                                  "p99": r4(force_error["p99"])},
        "at_1e-3_force_error": {"theta": accurate["theta"], "value": r4(accurate["value"]),
                                "median": r4(accurate["force_error"]["median"])},
        "per_body_above_1e-5": {k: {"count": per_body[k]["above_1e-5"],
                                    "fraction": per_body[k]["fraction_above"],
                                    "max": per_body[k]["max"]}
                                for k in ("plain", "compensated")},
        "mac_decision_counts_identical": per_body["decisions"]["identical"],
        "same_tree_kernels_ms": {k: v for k, v in kernels.items() if k.endswith("_ms")},
        "e2e": r4(e2e_value),
    }
    if batched:
        summary["batched"] = {"value": r4(batched["value"]),
                              "speedup_vs_plain": r4(batched["speedup_vs_plain"]),
                              "untuned": r4(batched["untuned"]["value"])}
    if served:
        lat, sat, spec = served["latency"], served["saturated"], served.get("specified")
        summary["served"] = {
            "rate_per_s": r4(lat["rate_per_s"]), "p50_s": r4(lat["p50_s"]),
            "p99_s": r4(lat["p99_s"]), "busy_frac": r4(lat.get("busy_frac")),
            "saturated": r4(sat["particle_steps_per_s"]),
            "speedup_vs_plain": r4(served["speedup_vs_plain"])}
        if spec:
            summary["served_at_200_per_s"] = {
                "requests": spec["requests"], "completed": spec["completed"],
                "p50_s": r4(spec["p50_s"]), "p99_s": r4(spec["p99_s"]),
                "value": r4(spec["particle_steps_per_s"]), "busy_frac": r4(spec.get("busy_frac")),
                "thread_seconds": spec.get("thread_seconds")}
    # long objects first, the contract keys and the compact summary last
    # (the end of the line is what a log tail keeps)
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world,
        "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded cold uniform disc)",
        "config": config_dict(world),
        "precision": precision,
        "config1": config1,
        "served": served,
        "batched": batched,
        "roofline_n2p24": roofline_large,
        "traversal": traversal,
        "repeats": repeats,
        "force_error": force_error,
        "at_1e-3_force_error": accurate,
        "per_body_force_error": per_body,
        "same_tree_kernels": kernels,
        "gpu": gpu.info().get("name"),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peaks["hbm_gbs"],
                     "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"],
                     "traffic": BUILD_DRAM_BYTES_PER_STEP,
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one "
                                       "step's sort, build and leapfrog kernels on this workload "
                                       "(one capture, per step)",
                     "kernels": "sort/build/leapfrog (integrate+bounds, morton, 4 radix "
                                "passes, count/scan, cells, aggregate)",
                     "peak_source": peaks["source"],
                     "algorithmic_bytes_per_body": {k: round(v, 1) for k, v in ab.items()},
                     "stage_ms": {k: round(v * 1e3, 4) for k, v in stage.items()},
                     "stage_gbs": stage_gbs},
        "e2e": {"value": e2e_value, "unit": METRIC, "h2d_bytes_per_step": 32 * N_BODIES,
                "d2h_bytes_per_step": 32 * N_BODIES, "steps": e2e_steps,
                "how": "per step: galaxy_bh_write_state from pinned host, one fused KDK step, "
                       "galaxy_bh_read_state to pinned host (C ABI)",
                "host_numa": numa.summary(), "wall_s": e2e_wall},
        "cpu_baseline": cpu,
        "clocks": clk,
        "gpu_launches": 10 * args.steps + 1,
        "summary": summary,
    }
    print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()


def run_precision_leg(gpu, steps: int = 500, n: int = 1 << 22, every: int = 10,
                      probes: int = 8192, thetas=(0.3, 0.5, 0.7)) -> dict:
    """Precision form: a binary disc encounter of two 2^21-body exponential
    discs (scale lengths 1.0 / 0.7, masses 1 : 0.5, 8 apart, relative speed
    0.3), f32 state with compensated two-sum force sums, eps 0.005, dt 5e-4.
    Per theta: FP64 energy / momentum / angular momentum every `every` steps
    (drifts relative to the initial values, momentum relative to the sum of
    m|v|), median / p99 force error against FP64 direct sums at `probes`
    probes at the start and the end, and the particle-steps/s of the steps
    themselves (log points excluded)."""
    import dataclasses as dc

    import numpy as np
    import torch

    from galaxy_b200 import scenarios
    from galaxy_b200.nbody_gpu import Config, ParallelTreeRuntime, bodies_to_state

    rt = ParallelTreeRuntime(gpu)
    s0 = bodies_to_state(scenarios.binary_encounter(n, seed=11, eps=0.005))
    probe_idx = np.linspace(0, n - 1, probes).astype(np.uint32)
    stream = torch.cuda.ExternalStream(gpu.stream_ptr())
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    out = {"workload": f"binary disc encounter N={n}, eps 0.005, dt 5e-4, compensated two-sum "
                       f"forces, {steps} steps, FP64 invariants every {every} steps",
           "thetas": {}}
    for theta in thetas:
        cfg = Config(theta=theta, softening_kpc=0.005, g=1.0, bucket=1, max_depth=48,
                     compensated=True)
        cfg_pot = dc.replace(cfg, potential=True)
        ev, _ = gpu.create_evolving_state_records(s0)
        tree = rt.create_tree(gpu, ev, cfg)
        rt.rebuild(gpu, ev, tree, cfg)
        rt.force(gpu, ev, tree, cfg_pot)  # boundary solve, with the potential for E0
        err0 = gpu.probe_error(ev, cfg, probe_idx)
        c0 = gpu.conservation(ev)
        drift = {"energy": 0.0, "momentum": 0.0, "lz": 0.0}
        step_ms = 0.0
        done = 0
        while done < steps:
            k = min(every, steps - done)
            torch.cuda.synchronize()
            e0.record(stream)
            rt.step(gpu, ev, tree, cfg, 5e-4, k)
            e1.record(stream)
            torch.cuda.synchronize()
            step_ms += e0.elapsed_time(e1)
            done += k
            # the same tree and positions: this force reproduces the boundary
            # accelerations bit for bit and adds the potential
            rt.force(gpu, ev, tree, cfg_pot)
            c = gpu.conservation(ev)
            drift["energy"] = max(drift["energy"],
                                  abs(c["energy"] - c0["energy"]) / abs(c0["energy"]))
            drift["momentum"] = max(drift["momentum"],
                                    float(np.hypot(c["px"] - c0["px"], c["py"] - c0["py"]))
                                    / c0["mass_speed_scale"])
            drift["lz"] = max(drift["lz"], abs(c["lz"] - c0["lz"]) / abs(c0["lz"]))
        err1 = gpu.probe_error(ev, cfg, probe_idx)
        out["thetas"][str(theta)] = {
            "value": n * steps / (step_ms * 1e-3), "unit": METRIC,
            "ms_per_step": step_ms / steps, "force_error_start": err0,
            "force_error_end": err1, "max_relative_drift": drift,
            "initial": {k: c0[k] for k in ("energy", "px", "py", "lz", "mass")}}
        tree.close()
        ev.close()
    return out


def run_batched_leg(gpu, steps: int, warmup: int, count: int = 512, plain_steps: int = 5,
                    plain_sims: int | None = None, pg=None, rank: int = 0, world: int = 1) -> dict:
    """Mixed workload: `count` independent simulations, N log-uniform in
    [2^10, 2^18], scenarios uniform over the three, per-simulation seeds,
    eps 0.01, theta 0.5, dt 1e-3.  Batched: one launch per stage for all of
    them.  Plain: each simulation alone through the plain path, one after
    another (the same engine, tree per simulation).  With several ranks the
    simulations are placed by estimated work (galaxy_b200.shard), each rank
    runs its share, and the rates use the slowest rank's time."""
    import torch

    from galaxy_b200 import autotune, scenarios, shard
    from galaxy_b200.batch import Batch
    from galaxy_b200.nbody_gpu import Config, ParallelTreeRuntime, bodies_to_state
    full_plan = scenarios.mixed_batch(count, 10, 18, seed=2024)
    shares = shard.plan_shards([n for _, n, _ in full_plan], world)
    plan = [full_plan[i] for i in shares[rank]]
    cfg = Config(theta=0.5, softening_kpc=0.01, g=1.0, bucket=1)
    states = []
    for name, n, seed in plan:
        states.append(gpu.create_evolving_state_records(
            bodies_to_state(scenarios.make(name, n, seed, eps=0.01)))[0])
    total = int(shard.sum_over_ranks(pg, sum(s.count for s in states)))
    stream = torch.cuda.ExternalStream(gpu.stream_ptr())
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    # autotuner (untimed, on copies of the states): leaf size per size class,
    # sort digit width, traversal warps per block
    tuning = autotune.tune_batch(gpu, states, [cfg] * len(states), dt=1e-3, steps=2,
                                 probes=128)
    tuned_cfgs = tuning.configs([s.count for s in states], [cfg] * len(states))

    def timed(cfgs, bits, warps, run_states, label):
        batch = Batch(gpu, run_states, cfgs)
        batch.tune(bits, warps)
        batch.solve()
        batch.step(1e-3, max(warmup, 3))
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_push(label)  # ncu --nvtx --nvtx-include <label>/
        e0.record(stream)
        batch.step(1e-3, steps)
        e1.record(stream)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
        ms = shard.max_over_ranks(pg, e0.elapsed_time(e1), "cuda")
        arena = batch.arena_bytes()
        batch.close()
        return ms, arena

    untuned_states = [gpu.create_evolving_state_records(gpu.read_evolving_state_records(s)[0])[0]
                      for s in states]
    u_ms, _ = timed([cfg] * len(states), 8, 4, untuned_states, "batched_untuned")
    for s in untuned_states:
        s.close()
    b_ms, arena = timed(tuned_cfgs, tuning.radix_bits, tuning.traverse_warps, states, "batched")
    # plain path, simulation after simulation (a prefix of the plan when
    # plain_sims is set; the rate is per body-step either way)
    rt = ParallelTreeRuntime(gpu)
    sims = states if plain_sims is None else states[:plain_sims]
    trees = []
    for s in sims:
        t = rt.create_tree(gpu, s, cfg)
        rt.rebuild(gpu, s, t, cfg)
        rt.force(gpu, s, t, cfg)
        rt.step(gpu, s, t, cfg, 1e-3, 1)
        trees.append(t)
    torch.cuda.synchronize()
    e0.record(stream)
    for s, t in zip(sims, trees):
        rt.step(gpu, s, t, cfg, 1e-3, plain_steps)
    e1.record(stream)
    torch.cuda.synchronize()
    p_ms = shard.max_over_ranks(pg, e0.elapsed_time(e1), "cuda")
    p_bodies = shard.sum_over_ranks(pg, sum(s.count for s in sims))
    for t in trees:
        t.close()
    for s in states:
        s.close()
    batched = total * steps / (b_ms * 1e-3)
    plain = p_bodies * plain_steps / (p_ms * 1e-3)
    return {"workload": f"{count} sims, N log-uniform [2^10, 2^18], mixed scenarios, "
                        "eps 0.01, theta 0.5, dt 1e-3, autotuned leaf size / sort digits / "
                        "traversal warps",
            "bodies": total, "steps": steps, "ms_per_step": b_ms / steps,
            "value": batched, "unit": METRIC, "arena_bytes": arena,
            "tuning": tuning.as_dict(), "tuning_force_error_median": tuning.errors,
            "untuned": {"value": total * steps / (u_ms * 1e-3), "ms_per_step": u_ms / steps,
                        "settings": "leaf size 1, 8-bit digits, 4 traversal warps (defaults)"},
            "ranks": world,
            "plain_serial": {"value": plain, "steps": plain_steps, "sims": len(sims) * world,
                             "ms_per_step": p_ms / plain_steps},
            "speedup_vs_plain": batched / plain}


def run_served_leg(gpu, capacity: float, duration: float = 20.0, budget_gb: float = 150.0,
                   deadline: float = 120.0, pg=None, rank: int = 0, world: int = 1,
                   burst_s: float = 0.5) -> dict:
    """Served workload: Poisson arrivals, N log-uniform [2^12, 2^22], steps
    log-uniform [10, 1000], scenario uniform, theta 0.5, eps 0.01, dt 1e-3,
    admitted against a 150 GB budget and continuously batched; each request
    brings its initial conditions (generated before the clock starts).

    Latency: arrivals at 60% of the measured batched capacity for
    `duration` s (the specified 200/s offers ~50x more work than one GPU
    serves; its load factor is reported) -> p50/p99 time-to-result.
    Throughput: the specified 200/s stream for `burst_s` s (a saturating
    burst of ~100 requests) served with continuous batching, against the same requests
    run one after another through the plain path (both include state upload,
    tree allocation, boundary solve and all steps).  With several ranks
    (`capacity` is then the whole job's) every rank draws the same request
    stream and serves the requests placed on it by estimated work
    (galaxy_b200.shard); latencies are pooled over ranks and rates use the
    slowest rank's wall time."""
    import torch

    from galaxy_b200 import scenarios, shard
    from galaxy_b200.nbody_gpu import Config, ParallelTreeRuntime, bodies_to_state
    from galaxy_b200.serve import NativeServer, poisson_requests
    mean_work = 605_000 * 215.0  # E[N] * E[steps] of the distributions above
    rate = max(0.2, 0.6 * capacity / mean_work)
    cfg = Config(theta=0.5, softening_kpc=0.01, g=1.0, bucket=1)

    def bodies(r):
        return scenarios.make(r.scenario, r.n, r.seed, eps=0.01)

    def with_inputs(reqs):
        for r in reqs:
            r.bodies = bodies(r)
        return reqs

    budget = int(budget_gb * 2 ** 30)

    def my_share(reqs):
        shares = shard.plan_shards([r.n for r in reqs], world, steps=[r.steps for r in reqs])
        return [reqs[i] for i in shares[rank]]

    def pooled(out, mine):
        if world == 1:
            return out
        lat = [x for part in shard.gather_to_all(pg, [r.latency for r in mine
                                                       if r.latency is not None]) for x in part]
        wall = shard.max_over_ranks(pg, out["wall_s"])
        steps_done = shard.sum_over_ranks(pg, out["particle_steps"])
        return dict(out, requests=int(shard.sum_over_ranks(pg, out["requests"])),
                    completed=len(lat), p50_s=float(np.percentile(lat, 50)) if lat else None,
                    p99_s=float(np.percentile(lat, 99)) if lat else None, wall_s=wall,
                    particle_steps=steps_done, particle_steps_per_s=steps_done / wall)

    def serve(reqs):
        """The native server (galaxy_bh_serve_*): a submitter thread releases
        each request at its arrival time, this thread polls for results;
        latency = finish - arrival."""
        import threading
        srv = NativeServer(gpu.info()["index"], budget_bytes=budget, round_steps=16)
        recs = [bodies_to_state(r.bodies) for r in reqs]
        ids = {}
        t0 = time.perf_counter()

        def submitter():
            for r, rec in zip(reqs, recs):
                delay = r.arrival - (time.perf_counter() - t0)
                if delay > 0:
                    time.sleep(delay)
                ids[srv.submit(rec, cfg, r.dt, r.steps)] = r

        th = threading.Thread(target=submitter)
        th.start()
        done, ps, first_submit, last_finish = 0, 0, None, 0.0

        def collect():
            nonlocal done, ps, first_submit, last_finish
            while done < len(reqs) and time.perf_counter() - t0 < deadline:
                got = srv.poll(timeout_s=1.0)
                if got is None:
                    continue
                info, _ = got
                done += 1
                while info["request_id"] not in ids:  # the submitter records ids after submit
                    time.sleep(1e-4)
                r = ids[info["request_id"]]
                r.finished = r.arrival + (info["finished_s"] - info["submitted_s"])
                ps += r.n * r.steps
                first_submit = info["submitted_s"] if first_submit is None else \
                    min(first_submit, info["submitted_s"])
                last_finish = max(last_finish, info["finished_s"])

        try:
            collect()
        finally:
            th.join()
            st = srv.stats()
            srv.stop()
        wall = (last_finish - first_submit) if first_submit is not None else 0.0
        lat = np.array([r.latency for r in reqs if r.latency is not None])
        return {"requests": len(reqs), "completed": int(len(lat)),
                "p50_s": float(np.percentile(lat, 50)) if len(lat) else None,
                "p99_s": float(np.percentile(lat, 99)) if len(lat) else None,
                "wall_s": wall, "busy_s": st["busy_seconds"], "rounds": st["rounds"],
                # share of the serving thread's working time (rounds, batch
                # re-formation, readback) spent in rounds; admission and
                # boundary solves run on the stager thread, overlapping them
                "busy_frac": st["busy_seconds"] / max(1e-9, sum(
                    st[k] for k in ("busy_seconds", "form_seconds", "readback_seconds"))),
                "thread_seconds": {k[:-8]: round(st[k], 3) for k in
                                   ("busy_seconds", "admit_seconds", "solve_seconds",
                                    "form_seconds", "readback_seconds", "elapsed_seconds")},
                "particle_steps": ps, "particle_steps_per_s": ps / wall if wall > 0 else 0.0,
                "server": "native (galaxy_bh_serve_*)"}

    reqs = with_inputs(my_share(poisson_requests(rate, duration, seed=11)))
    out = pooled(serve(reqs), reqs)
    for r in reqs:
        r.bodies = None
    # the specified rate: 200 requests/s, the first `burst_s` seconds of the
    # stream (its 60 s would offer ~25x what one GPU serves; p50/p99 here are
    # backlog-dominated), served to completion
    burst = with_inputs(my_share(poisson_requests(200.0, burst_s, seed=12)))
    sat = pooled(serve(burst), burst)
    torch.cuda.synchronize()
    rt = ParallelTreeRuntime(gpu)
    t0 = time.perf_counter()
    ps = 0
    for r in burst:
        ev, _ = gpu.create_evolving_state_records(bodies_to_state(r.bodies))
        tree = rt.create_tree(gpu, ev, cfg)
        rt.rebuild(gpu, ev, tree, cfg)
        rt.force(gpu, ev, tree, cfg)
        rt.step(gpu, ev, tree, cfg, r.dt, r.steps)
        tree.close()
        ev.close()
        ps += r.n * r.steps
    plain = shard.sum_over_ranks(pg, ps) / shard.max_over_ranks(pg, time.perf_counter() - t0)
    return {
        "workload": "Poisson arrivals, N log-uniform [2^12,2^22], steps log-uniform [10,1000], "
                    "mixed scenarios, theta 0.5, eps 0.01, dt 1e-3, 150 GB budget",
        "latency": dict(out, rate_per_s=rate, arrival_window_s=duration),
        "specified_rate_per_s": 200.0,
        "specified_load_factor": 200.0 * mean_work / capacity,
        "saturated": dict(sat, rate_per_s=200.0, arrival_window_s=burst_s),
        "specified": dict(sat, rate_per_s=200.0, arrival_window_s=burst_s,
                          note="the same run as saturated: arrivals at the specified rate"),
        "ranks": world,
        "plain_serial": {"particle_steps_per_s": plain, "requests": sat["requests"],
                         "includes": "state upload, tree allocation, boundary solve, steps"},
        "speedup_vs_plain": sat["particle_steps_per_s"] / plain if plain else None}


def run_large_roofline(gpu, rt, peak_gbs: float, n: int = 1 << 24, reps: int = 3) -> dict:
    """The sort/build/leapfrog stages of the same workload at N = 2^24 (cold
    uniform disc, seed 7): the kernels of the 2^20 headline with 16x the
    bodies, where fewer of their steps are latency-bound.  Device stage times
    from instrumented rebuilds (mean of `reps`) and the step's kick/drift +
    bounds kernel on the same state; algorithmic bytes as at 2^20."""
    from galaxy_b200 import scenarios
    from galaxy_b200.nbody_gpu import Config, bodies_to_state
    cfg = Config(theta=THETA, softening_kpc=EPS, g=G, bucket=BUCKET, max_depth=48)
    s0 = bodies_to_state(scenarios.cold_disc(n, SEED))
    ev, _ = gpu.create_evolving_state_records(s0)
    tree = rt.create_tree(gpu, ev, cfg)
    rt.rebuild(gpu, ev, tree, cfg)
    stage = {"integrate": 0.0, "morton": 0.0, "radix": 0.0, "topology": 0.0, "aggregate": 0.0}
    import torch
    torch.cuda.nvtx.range_push("n2p24")  # ncu --nvtx --nvtx-include n2p24/
    for _ in range(reps):
        stage["integrate"] += gpu.kick_drift(ev, DT).dispatch_seconds / reps
        bt = rt.rebuild(gpu, ev, tree, cfg)
        for k in ("morton", "radix", "topology", "aggregate"):
            stage[k] += getattr(bt, k + "_seconds") / reps
    torch.cuda.nvtx.range_pop()
    c = tree_cells(gpu, rt, tree) / n
    tree.close()
    ev.close()
    ab = algorithmic_bytes(c)
    secs = sum(stage.values())
    achieved = n * sum(ab.values()) / secs / 1e9
    return {"n_bodies": n, "achieved": achieved, "peak": peak_gbs, "unit": "GB/s",
            "frac": achieved / peak_gbs, "cells_per_body": c,
            "stage_ms": {k: round(v * 1e3, 4) for k, v in stage.items()},
            "stage_gbs": {k: round(n * ab[k] / v / 1e9, 1) for k, v in stage.items() if v > 0}}


def tree_cells(gpu, rt, tree) -> int:
    import ctypes as C

    from galaxy_b200 import _lib
    cnt = C.c_uint32()
    _lib.check(_lib.load().galaxy_bh_read_tree_evidence(gpu.handle, tree.handle, None, None,
                                                         None, 0, None, 0, C.byref(cnt)))
    return int(cnt.value)


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["engine", "reference"], default="engine")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true",
                    help="skip the mixed-size batched workload leg")
    ap.add_argument("--no-served", action="store_true", help="skip the served workload leg")
    ap.add_argument("--no-precision", action="store_true",
                    help="skip the precision-form leg (binary encounter, N=2^22)")
    ap.add_argument("--precision-steps", type=int, default=500)
    ap.add_argument("--only-step", action="store_true",
                    help="run the timed steps of the headline workload and nothing else "
                         "(a short line without the side legs; for profilers)")
    ap.add_argument("--only-batched", action="store_true",
                    help="run the mixed-size batched leg and nothing else (for profilers)")
    ap.add_argument("--only-same-tree", action="store_true",
                    help="time this engine's kernels on the workload's initial tree and "
                         "nothing else (for profilers)")
    args = ap.parse_args()
    world, rank, local, pg = dist_setup(args)
    if args.impl == "reference":
        run_reference(args, world, rank, pg)
    else:
        run_engine(args, world, rank, local, pg)


if __name__ == "__main__":
    main()
