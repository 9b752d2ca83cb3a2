"""Receipts of the BH #2D evolution run in the schema of the reference's
hardware sweep (`galaxy.barnes-hut-parallel-gpu-tree-receipt.v1`, produced by
runtime/src/bin/galaxy-bh-gpu-tree-parallel.rs:515-598 and checked by
scripts/bench-bh2d-hardware.py:1013-1389).

`run_receipt` repeats that binary's run on this engine: `steps` KDK steps as
separate kick/drift, rebuild, force and final-kick calls, tree evidence and
its checksum before and after, a same-state repeat rebuild, the FP64 direct
probe gate, and the same-state rebuild benchmark.  The evidence is hashed in
the sparse level-order slot layout the receipt declares (cells ordered by
depth, then start; children named by slot depth * N + start), the sort runs
at the declared 4-bit digit width (the permutation is the same at 8 bits),
and the initial conditions are the reference's presets (`presets.py`).

Two fields cannot take the reference's values and say so:
* `gpu.backend` is "CUDA" (the sweep script admits Vulkan, Metal and Dx12;
  accepting this engine's receipts means adding "CUDA" to that set);
* `parallel_tree_buffer_bytes` is this engine's tree buffer, whose formula
  is `galaxy_bh_tree_footprint` (the sweep script's frozen formula describes
  the reference's 17 N 64-byte sparse cells).
The CPU flat-tree, trajectory and serial-GPU oracle sections run only in the
reference's own binaries; receipts here therefore need particles above the
oracle limit and above the 4096-body cap of the serial GPU builder, where
those sections are skipped by the schema itself.

`validate_receipt` restates the sweep's checks with those two changes.
"""
from __future__ import annotations

import ctypes as C
import json
import math
import time

import numpy as np

from . import _lib, presets
from .nbody_gpu import Config, NbodyGpu, ParallelTreeRuntime

SCHEMA = "galaxy.barnes-hut-parallel-gpu-tree-receipt.v1"
BUILDER = "gpu-parallel-sparse-radix-v1"
ORDERING = "stable-lsd-radix-4bit-morton-code; resident body index retained for equal Morton keys"
LAYOUT = "sparse-level-order-slot=depth*N+group_start"
SAMPLE_SCOPE = ("complete rebuild call including host-side uniform/bind-group setup, "
                "command encoding, submit and synchronization")
SERIAL_CAP = 4096          # the reference's serial GPU builder runs up to this size
TREE_LEVELS = 17
BACKENDS = {"Vulkan", "Metal", "Dx12", "CUDA"}
_MASK = (1 << 64) - 1


def _mix(h: int, word: int) -> int:
    """One word of the FNV-offset / 0x100000001b3 / rotl-23 mix
    (galaxy-bh-gpu-tree-parallel.rs:150-154)."""
    h ^= word
    h = (h * 0x100000001B3) & _MASK
    return h ^ (((word << 23) | (word >> 41)) & _MASK)


def evidence_checksum(meta, entries, cells) -> int:
    """Checksum of tree evidence: metadata words, bound bits, every entry word,
    then per cell its f32 centre/half/mass and centre of mass bits, range,
    depth, valid flag and children (galaxy-bh-gpu-tree-parallel.rs:156-187)."""
    h = 0xCBF29CE484222325
    words = [np.asarray(meta["data"], np.uint32).ravel(),
             np.asarray(meta["bounds"], np.float32).view(np.uint32).ravel(),
             np.asarray(entries["data"], np.uint32).ravel()]
    cw = np.concatenate([cells["center_half_mass"].astype(np.float32).view(np.uint32),
                         cells["com"].astype(np.float32).view(np.uint32),
                         cells["range_depth"].astype(np.uint32),
                         cells["children"].astype(np.uint32)], axis=1)
    words.append(cw.ravel())
    for w in np.concatenate(words).tolist():
        h = _mix(h, w)
    return h


def level_order_cells(cells: np.ndarray, n: int) -> np.ndarray:
    """The engine's preorder cells (children as preorder indices) rearranged
    into the declared slot layout: ordered by slot = depth * n + start, the
    valid flag set, children named by their slots."""
    rd = cells["range_depth"]
    slot = rd[:, 2].astype(np.int64) * n + rd[:, 0].astype(np.int64)
    order = np.argsort(slot, kind="stable")
    out = cells[order].copy()
    ch = cells["children"][order]
    none = ch == _lib.NO_CHILD
    mapped = np.where(none, 0, slot[np.where(none, 0, ch).astype(np.int64)])
    out["children"] = np.where(none, _lib.NO_CHILD, mapped).astype(np.uint32)
    out["range_depth"][:, 3] = 1
    return out


def tree_footprint_bytes(particles: int, config: Config) -> int:
    v = C.c_uint64()
    _lib.check(_lib.load().galaxy_bh_tree_footprint(int(particles), C.byref(config.to_c()),
                                                      C.byref(v)))
    return int(v.value)


def _probe_indices(n: int, count: int) -> np.ndarray:
    """k * (n - 1) / (count - 1), as probe_error (nbody/src/lib.rs:370-395)."""
    count = max(1, min(count, n))
    den = max(count - 1, 1)
    return np.array([k * (n - 1) // den for k in range(count)], dtype=np.uint32)


def _gpu_info(gpu: NbodyGpu, ordinal: int) -> dict:
    import torch
    info = gpu.info()
    return {"index": ordinal, "adapter_count": torch.cuda.device_count(),
            "name": info.get("name", "CUDA device"), "backend": "CUDA",
            "device_type": info.get("device_type", "DiscreteGpu"),
            "driver": f"CUDA driver {info.get('cuda_driver', '')}".strip(),
            "driver_info": f"CUDA runtime {info.get('cuda_runtime', '')}, "
                           f"compute capability {info.get('compute_capability', '')}",
            "software": False}


def run_receipt(preset: str = "disc", particles: int = 8192, steps: int = 3, dt_myr: float = 0.01,
                seed: int = 303, theta: float = 0.5, softening_kpc: float = 0.05,
                direct_probes: int = 12, oracle_limit: int = 4096, benchmark_warmup: int = 2,
                benchmark_repeats: int = 7, ordinal: int = 0) -> dict:
    """The BH #2D run and receipt of galaxy-bh-gpu-tree-parallel.rs:282-598."""
    if not 2 <= particles <= 65536:
        raise ValueError("--particles must be in 2..=65536 for BH #2D")
    if particles <= max(oracle_limit, SERIAL_CAP):
        raise ValueError("receipts here need particles above the oracle limit and above 4096: "
                         "the CPU and serial-GPU oracle sections run in the reference binaries")
    if not 1 <= steps <= 256:
        raise ValueError("--steps must be in 1..=256")
    if not (math.isfinite(dt_myr) and 1e-6 <= dt_myr <= 1.0):
        raise ValueError("--dt-myr must be finite and in [1e-6, 1]")
    if not (math.isfinite(theta) and 0.0 <= theta <= 2.0):
        raise ValueError("--theta must be finite and in [0, 2]")
    if not (math.isfinite(softening_kpc) and 0.0 <= softening_kpc <= 100.0):
        raise ValueError("--softening-kpc must be finite and in [0, 100]")
    if not 1 <= direct_probes <= 64:
        raise ValueError("--direct-probes must be in 1..=64")
    if not 2 <= oracle_limit <= 4096:
        raise ValueError("--oracle-limit must be in 2..=4096")
    if benchmark_repeats == 0 or benchmark_repeats > 31 or benchmark_warmup > 10:
        raise ValueError("benchmark warmup/repeats must be warmup<=10 and repeats in 1..=31")
    initial = presets.make(preset, particles, seed)
    config = Config(theta=theta, softening_kpc=softening_kpc)
    gpu = NbodyGpu(str(ordinal))
    rt = ParallelTreeRuntime(gpu)
    wall = time.perf_counter()
    ev, create_t = gpu.create_evolving_state(initial)
    tree = rt.create_tree(gpu, ev, config)
    rt.tune(tree, radix_bits=4)  # the declared digit width
    build = {k: 0.0 for k in ("bounds", "morton", "radix", "positions", "topology", "aggregate")}
    stage = {k: 0.0 for k in ("force", "kick_drift", "final_kick")}

    def add_build(t):
        for k in build:
            build[k] += getattr(t, k + "_seconds")

    add_build(rt.rebuild(gpu, ev, tree, config))
    stage["force"] += rt.force(gpu, ev, tree, config).dispatch_seconds

    def evidence():
        e = rt.read_evidence(gpu, tree)
        codes = e.entries["data"][:, :2].astype(np.uint64)
        keys = (codes[:, 0] << np.uint64(32)) | codes[:, 1]
        if len(keys) > 1 and not np.all(keys[1:] > keys[:-1]):
            raise RuntimeError("BH #2D radix order is not strict by (Morton code, body index)")
        return e, evidence_checksum(e.meta, e.entries, level_order_cells(e.cells, particles))

    _, initial_sum = evidence()
    for _ in range(steps):
        stage["kick_drift"] += gpu.kick_drift(ev, dt_myr).dispatch_seconds
        add_build(rt.rebuild(gpu, ev, tree, config))
        stage["force"] += rt.force(gpu, ev, tree, config).dispatch_seconds
        stage["final_kick"] += gpu.final_kick(ev, dt_myr).dispatch_seconds
    _, state_t = gpu.read_evolving_state(ev)
    _, accel_t = gpu.read_evolving_accelerations(ev)
    final_ev, final_sum = evidence()
    rt.rebuild(gpu, ev, tree, config)
    _, repeat_sum = evidence()
    if repeat_sum != final_sum:
        raise RuntimeError("BH #2D unchanged-state repeat tree checksum changed")
    probe_count = min(direct_probes, particles)
    t0 = time.perf_counter()
    err = gpu.probe_error(ev, config, _probe_indices(particles, probe_count))
    direct_s = time.perf_counter() - t0
    if err["rms"] >= 0.04 or err["max"] >= 0.30:
        raise RuntimeError(f"BH #2D direct-force gate failed: rms={err['rms']} max={err['max']}")
    for _ in range(benchmark_warmup):
        rt.rebuild(gpu, ev, tree, config)
    samples = []
    for _ in range(benchmark_repeats):
        t0 = time.perf_counter()
        rt.rebuild(gpu, ev, tree, config)
        samples.append(time.perf_counter() - t0)
    median = sorted(samples)[len(samples) // 2]
    leaf_count = final_ev.leaf_count
    receipt = {
        "schema": SCHEMA, "status": "complete", "phase": "BH-2D", "builder": BUILDER,
        "engine": "galaxy_b200 (CUDA sm_100a): onesweep radix, chain-count preorder cells, "
                  "bottom-up f64 aggregates, lane-parallel group traversal",
        "measurement_class": "hardware", "hardware_performance_claim_allowed": True,
        "preset": preset, "particles": particles, "steps": steps, "dt_myr": dt_myr,
        "simulated_time_myr": dt_myr * steps, "seed": seed, "theta": theta,
        "softening_kpc": softening_kpc, "gpu": _gpu_info(gpu, ordinal),
        "host_tree_rebuilds": 0, "host_particle_readbacks_during_steps": 0,
        "force_solves": steps + 1, "evolution_tree_builds": steps + 1,
        "parallel_tree_buffer_bytes": rt.buffer_bytes(tree),
        "tree": {
            "initial_checksum_fnv_mix64": f"{initial_sum:016x}",
            "final_checksum_fnv_mix64": f"{final_sum:016x}",
            "repeat_checksum_fnv_mix64": f"{repeat_sum:016x}",
            "repeat_rebuild_matches": repeat_sum == final_sum,
            "active_cell_count": final_ev.active_cell_count, "leaf_count": leaf_count,
            "max_depth": final_ev.max_depth,
            "root_bounds_f32": [float(v) for v in final_ev.meta["bounds"]],
            "ordering": ORDERING, "layout": LAYOUT},
        "final_force": {
            "bh2a_flat_status": "skipped-particle-limit",
            "gpu_vs_bh2a_flat_rms_relative": None, "gpu_vs_bh2a_flat_max_relative": None,
            "direct_probe_count": probe_count, "direct_probe_rms_relative": err["rms"],
            "direct_probe_max_relative": err["max"]},
        "trajectory_vs_bh2a_flat_f64": {
            "status": "skipped-particle-limit", "limit": oracle_limit,
            "reason": "large BH #2D runs keep CPU trajectory evidence bounded"},
        "gpu_oracles": {
            "status": "skipped-particle-limit", "limit": oracle_limit,
            "reason": "BH #2C serialized GPU oracle is intentionally capped at 4096 bodies"},
        "tree_build_benchmark": {
            "sample_scope": SAMPLE_SCOPE, "stage_timings_are_diagnostics": True,
            "warmup": benchmark_warmup, "repeats": benchmark_repeats,
            "parallel_samples_seconds": samples, "parallel_median_seconds": median,
            "bh2c_serial": {"status": "skipped-bh2c-cap", "limit": SERIAL_CAP}},
        "timings_seconds": {
            "gpu_state_create_transfer": create_t.transfer_seconds,
            **{f"parallel_{k}_total": v for k, v in build.items()},
            "parallel_tree_build_total": sum(build.values()),
            "gpu_force_dispatch_total": stage["force"],
            "gpu_kick_drift_dispatch_total": stage["kick_drift"],
            "gpu_final_kick_dispatch_total": stage["final_kick"],
            "final_state_readback": state_t.readback_seconds,
            "final_acceleration_readback": accel_t.readback_seconds,
            "direct_probe_reference": direct_s,
            "total_wall": time.perf_counter() - wall},
        "scope": "BH #2D evolution on the galaxy_b200 CUDA engine: GPU bounds, stable 4-bit "
                 "LSD radix Morton ordering, parallel cell topology and f64 aggregates, "
                 "theta-MAC traversal; CPU and serial-GPU oracle sections belong to the "
                 "reference binaries and are skipped above their limits."}
    tree.close()
    ev.close()
    return receipt


# ---------------------------------------------------------------- checks --

class ReceiptError(ValueError):
    pass


def _req(cond: bool, msg: str) -> None:
    if not cond:
        raise ReceiptError(msg)


def _num(v, name, *, positive=False, nonnegative=False) -> float:
    _req(isinstance(v, (int, float)) and not isinstance(v, bool) and math.isfinite(v),
         f"{name} must be a finite number")
    if positive:
        _req(v > 0, f"{name} must be positive")
    if nonnegative:
        _req(v >= 0, f"{name} must be nonnegative")
    return float(v)


def _int(v, name, minimum=None) -> int:
    _req(isinstance(v, int) and not isinstance(v, bool), f"{name} must be an integer")
    if minimum is not None:
        _req(v >= minimum, f"{name} must be >= {minimum}")
    return v


def _checksum(v, name) -> str:
    _req(isinstance(v, str) and len(v) == 16 and all(c in "0123456789abcdef" for c in v),
         f"{name} must be a 16-digit lowercase hexadecimal checksum")
    return v


def validate_receipt(r: dict, *, particles: int, preset: str, steps: int, dt_myr: float,
                     seed: int, theta: float, softening_kpc: float, direct_probes: int,
                     oracle_limit: int, benchmark_warmup: int, benchmark_repeats: int,
                     bucket: int = 4) -> dict:
    """The checks of scripts/bench-bh2d-hardware.py:1013-1389, with "CUDA"
    admitted as a backend and this engine's tree-buffer formula."""
    _req(isinstance(r, dict), "receipt must be an object")
    for key, want in (("schema", SCHEMA), ("status", "complete"), ("phase", "BH-2D"),
                      ("builder", BUILDER), ("preset", preset), ("measurement_class", "hardware")):
        _req(r.get(key) == want, f"receipt.{key} must be {want!r}")
    _req(_int(r.get("particles"), "particles") == particles, "particle count mismatch")
    _req(_int(r.get("steps"), "steps") == steps, "step count mismatch")
    _req(_int(r.get("seed"), "seed") == seed, "seed mismatch")
    for key, want in (("dt_myr", dt_myr), ("theta", theta), ("softening_kpc", softening_kpc),
                      ("simulated_time_myr", dt_myr * steps)):
        _req(_num(r.get(key), key) == float(want), f"receipt.{key} mismatch")
    _req(r.get("hardware_performance_claim_allowed") is True, "no hardware performance claim")
    _req(_int(r.get("host_tree_rebuilds"), "host_tree_rebuilds", 0) == 0, "host tree rebuild")
    _req(_int(r.get("host_particle_readbacks_during_steps"), "readbacks", 0) == 0,
         "host readback inside the evolution loop")
    _req(_int(r.get("force_solves"), "force_solves", 0) == steps + 1, "force-solve count")
    _req(_int(r.get("evolution_tree_builds"), "tree builds", 0) == steps + 1, "tree-build count")
    gpu = r.get("gpu")
    _req(isinstance(gpu, dict), "receipt.gpu must be an object")
    idx = _int(gpu.get("index"), "gpu.index", 0)
    _req(idx < _int(gpu.get("adapter_count"), "gpu.adapter_count", 1), "gpu index out of range")
    name = gpu.get("name")
    _req(isinstance(name, str) and name.strip(), "gpu.name must be nonempty")
    dtype = gpu.get("device_type")
    _req(isinstance(dtype, str) and dtype.strip(), "gpu.device_type must be nonempty")
    _req(dtype.lower() != "cpu" and not any(m in name.lower() for m in
                                            ("llvmpipe", "lavapipe", "swiftshader", "software")),
         "gpu is a software adapter")
    _req(gpu.get("backend") in BACKENDS, "gpu.backend not admitted")
    _req(bool(str(gpu.get("driver", "")).strip() or str(gpu.get("driver_info", "")).strip()),
         "gpu needs driver provenance")
    _req(gpu.get("software") is False, "gpu.software must be false")
    t = r.get("tree")
    _req(isinstance(t, dict), "receipt.tree must be an object")
    _req(t.get("ordering") == ORDERING, "tree.ordering mismatch")
    _req(t.get("layout") == LAYOUT, "tree.layout mismatch")
    _req(t.get("repeat_rebuild_matches") is True, "repeat tree checksum changed")
    _checksum(t.get("initial_checksum_fnv_mix64"), "tree.initial_checksum_fnv_mix64")
    final = _checksum(t.get("final_checksum_fnv_mix64"), "tree.final_checksum_fnv_mix64")
    _req(final == _checksum(t.get("repeat_checksum_fnv_mix64"), "tree.repeat"),
         "repeat checksum differs from final checksum")
    active = _int(t.get("active_cell_count"), "active_cell_count", 1)
    leaves = _int(t.get("leaf_count"), "leaf_count", 1)
    depth = _int(t.get("max_depth"), "max_depth", 0)
    internal = active - leaves
    _req(active <= TREE_LEVELS * particles, "active cells exceed the sparse capacity")
    _req(leaves <= active and leaves <= particles, "leaf count too large")
    _req(leaves <= 3 * internal + 1, "leaf count exceeds quadtree fan-out")
    _req(depth <= TREE_LEVELS - 1, "max_depth exceeds the Morton depth")
    per_depth = particles // (bucket + 1)
    _req(active <= leaves + sum(min(4 ** d, per_depth) for d in range(depth)),
         "active cells exceed per-depth occupancy")
    _req(active >= depth + 1 and internal >= depth, "too few cells for the depth")
    _req(internal <= sum(min(4 ** d, leaves) for d in range(depth)),
         "too many internal cells for the leaf paths")
    if depth < TREE_LEVELS - 1:
        _req(leaves >= (particles + bucket - 1) // bucket, "too few leaves for the bucket size")
    if particles > bucket:
        _req(active > leaves and depth > 0, "an internal cell is required")
    f = r.get("final_force")
    _req(isinstance(f, dict), "receipt.final_force must be an object")
    probes = min(direct_probes, particles)
    _req(_int(f.get("direct_probe_count"), "direct_probe_count") == probes, "probe count")
    rms = _num(f.get("direct_probe_rms_relative"), "direct rms", nonnegative=True)
    mx = _num(f.get("direct_probe_max_relative"), "direct max", nonnegative=True)
    _req(rms <= mx <= rms * math.sqrt(probes), "direct rms/max inconsistent")
    _req(rms < 0.04 and mx < 0.30, "direct-force gate failed")
    status = "executed" if particles <= oracle_limit else "skipped-particle-limit"
    _req(f.get("bh2a_flat_status") == status, "flat-oracle status mismatch")
    for key in ("gpu_oracles", "trajectory_vs_bh2a_flat_f64"):
        sec = r.get(key)
        _req(isinstance(sec, dict) and sec.get("status") == status, f"{key} status mismatch")
        if status != "executed":
            _req(_int(sec.get("limit"), f"{key}.limit") == oracle_limit, f"{key} limit mismatch")
    b = r.get("tree_build_benchmark")
    _req(isinstance(b, dict), "receipt.tree_build_benchmark must be an object")
    _req(b.get("sample_scope") == SAMPLE_SCOPE, "benchmark sample scope mismatch")
    _req(b.get("stage_timings_are_diagnostics") is True, "stage timings must be diagnostics")
    _req(_int(b.get("warmup"), "warmup") == benchmark_warmup, "benchmark warmup mismatch")
    _req(_int(b.get("repeats"), "repeats") == benchmark_repeats, "benchmark repeats mismatch")
    samples = b.get("parallel_samples_seconds")
    _req(isinstance(samples, list) and len(samples) == benchmark_repeats, "sample count")
    vals = [_num(v, "sample", positive=True) for v in samples]
    median = sorted(vals)[len(vals) // 2]
    _req(_num(b.get("parallel_median_seconds"), "median", positive=True) == median,
         "benchmark median does not match its samples")
    serial = b.get("bh2c_serial")
    _req(isinstance(serial, dict), "bh2c_serial must be an object")
    if particles > SERIAL_CAP:
        _req(serial.get("status") == "skipped-bh2c-cap" and serial.get("limit") == SERIAL_CAP,
             "serial comparison must skip above 4096")
    else:
        _req(serial.get("status") == "executed", "serial comparison should execute")
    want_bytes = tree_footprint_bytes(particles, Config(theta=theta, softening_kpc=softening_kpc))
    _req(_int(r.get("parallel_tree_buffer_bytes"), "buffer bytes", 1) == want_bytes,
         "parallel_tree_buffer_bytes does not match galaxy_bh_tree_footprint")
    return {"particles": particles, "parallel_tree_buffer_bytes": want_bytes,
            "active_cell_count": active, "leaf_count": leaves, "max_depth": depth,
            "parallel_median_seconds": median, "direct_probe_rms_relative": rms,
            "direct_probe_max_relative": mx}


def main(argv=None) -> int:
    import argparse
    ap = argparse.ArgumentParser(description="BH #2D receipt on the galaxy_b200 engine "
                                             "(arguments of galaxy-bh-gpu-tree-parallel)")
    ap.add_argument("--preset", choices=("disc", "collision"), default="disc")
    ap.add_argument("--particles", type=int, default=8192)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--dt-myr", type=float, default=0.01)
    ap.add_argument("--seed", type=int, default=303)
    ap.add_argument("--theta", type=float, default=0.5)
    ap.add_argument("--softening-kpc", type=float, default=0.05)
    ap.add_argument("--direct-probes", type=int, default=12)
    ap.add_argument("--oracle-limit", type=int, default=4096)
    ap.add_argument("--benchmark-warmup", type=int, default=2)
    ap.add_argument("--benchmark-repeats", type=int, default=7)
    ap.add_argument("--adapter", type=int, default=0)
    ap.add_argument("--receipt", required=True)
    a = ap.parse_args(argv)
    r = run_receipt(a.preset, a.particles, a.steps, a.dt_myr, a.seed, a.theta, a.softening_kpc,
                    a.direct_probes, a.oracle_limit, a.benchmark_warmup, a.benchmark_repeats,
                    a.adapter)
    with open(a.receipt, "w") as fh:
        json.dump(r, fh, indent=2)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
