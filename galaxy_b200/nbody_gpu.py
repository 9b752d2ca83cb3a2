"""Host mirror of the reference's BH GPU API over the CUDA engine.

Same names, argument meaning and error behaviour as
``runtime/src/nbody_gpu.rs`` (``NbodyGpu``, ``EvolvingState``,
``pack_flat_tree``, ``PackedFlat``) and ``runtime/src/nbody_parallel.rs``
(``ParallelTreeRuntime``, ``ParallelGpuTree``), so a caller of the reference
reads the same program.  Bodies are float64 arrays of shape (n, 5) with
columns x, y, vx, vy, mass (``Body``, nbody/src/lib.rs:12-19); accelerations
are float64 (n, 2) (``Accel``).  Every numeric stage runs in the C ABI
(``include/galaxy_bh.h``); nothing here computes forces or trees.
"""
from __future__ import annotations

import ctypes as C
import json
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import (BH_FLAG_COMPENSATED, BH_FLAG_NO_STATS, BH_FLAG_POTENTIAL, BhBuildTiming,
                   BhConfig, BhForceStats, BhStageTiming, EngineError, EngineUnavailable, check,
                   ptr)

G_KPC3_PER_MSUN_MYR2 = 4.498502151575286e-12  # nbody/src/lib.rs:6
DEFAULT_THETA = 0.5
DEFAULT_SOFTENING_KPC = 0.05
DEFAULT_BUCKET = 4
DEFAULT_MAX_DEPTH = 48
MORTON_TREE_DEPTH = 16

__all__ = ["Config", "NbodyGpu", "EvolvingState", "ParallelTreeRuntime", "ParallelGpuTree",
           "PackedFlat", "pack_flat_tree", "StageTiming", "ParallelTreeBuildTiming",
           "ParallelGpuTreeEvidence", "TraversalResult", "EngineError", "EngineUnavailable",
           "bodies_to_state", "state_to_bodies", "G_KPC3_PER_MSUN_MYR2"]


@dataclass
class Config:
    """nbody/src/lib.rs:27-67, plus engine flags (compensated force sums,
    per-body potential)."""

    theta: float = DEFAULT_THETA
    softening_kpc: float = DEFAULT_SOFTENING_KPC
    g: float = G_KPC3_PER_MSUN_MYR2
    bucket: int = DEFAULT_BUCKET
    max_depth: int = DEFAULT_MAX_DEPTH
    compensated: bool = False
    potential: bool = False
    force_stats: bool = True  # ParallelTreeRuntime.force also counts visits/terms

    def validate(self) -> None:
        if not np.isfinite(self.theta) or self.theta < 0.0:
            raise ValueError("theta must be finite and >= 0")
        if not np.isfinite(self.softening_kpc) or self.softening_kpc < 0.0:
            raise ValueError("softening_kpc must be finite and >= 0")
        if not np.isfinite(self.g) or self.g <= 0.0:
            raise ValueError("g must be positive and finite")
        if not 1 <= self.bucket <= 1024:
            raise ValueError("bucket must be in 1..=1024")
        if not 1 <= self.max_depth <= 128:
            raise ValueError("max_depth must be in 1..=128")

    def to_c(self) -> BhConfig:
        self.validate()
        flags = (BH_FLAG_COMPENSATED if self.compensated else 0) | (
            BH_FLAG_POTENTIAL if self.potential else 0) | (
            0 if self.force_stats else BH_FLAG_NO_STATS)
        return BhConfig(float(self.theta), float(self.softening_kpc), float(self.g),
                        int(self.bucket), int(self.max_depth), flags, 0)


@dataclass
class StageTiming:
    """nbody_gpu.rs:125-130."""

    transfer_seconds: float = 0.0
    dispatch_seconds: float = 0.0
    readback_seconds: float = 0.0

    @classmethod
    def of(cls, t: BhStageTiming) -> "StageTiming":
        return cls(t.transfer_seconds, t.dispatch_seconds, t.readback_seconds)


@dataclass
class ParallelTreeBuildTiming:
    """nbody_parallel.rs:45-64 (device stage times from CUDA events)."""

    bounds_seconds: float = 0.0
    morton_seconds: float = 0.0
    radix_seconds: float = 0.0
    positions_seconds: float = 0.0
    topology_seconds: float = 0.0
    aggregate_seconds: float = 0.0

    def total_seconds(self) -> float:
        return (self.bounds_seconds + self.morton_seconds + self.radix_seconds
                + self.positions_seconds + self.topology_seconds + self.aggregate_seconds)


@dataclass
class TraversalResult:
    """nbody_gpu.rs:157-165."""

    accelerations: np.ndarray
    gpu_info: dict
    packed_bytes: int
    transfer_seconds: float
    dispatch_seconds: float
    readback_seconds: float


@dataclass
class PackedFlat:
    """nbody_gpu.rs:141-155 in the frozen record dtypes of ``_lib``."""

    settings: np.ndarray  # BH_SETTINGS_DTYPE, shape ()
    bodies: np.ndarray    # GPU_BODY_DTYPE (n,)
    entries: np.ndarray   # GPU_ENTRY_DTYPE (n,)
    cells: np.ndarray     # GPU_CELL_DTYPE (C,)

    def byte_len(self) -> int:
        return 32 + self.bodies.nbytes + self.entries.nbytes + self.cells.nbytes


def _checked_f32(values, name: str) -> np.ndarray:
    """nbody_gpu.rs:167-173: f64 -> f32, failing when not finite."""
    with np.errstate(over="ignore", invalid="ignore"):
        packed = np.asarray(values, dtype=np.float64).astype(np.float32)
    if not np.isfinite(packed).all():
        raise ValueError(f"{name} cannot be represented as finite f32")
    return packed


def bodies_to_state(bodies) -> np.ndarray:
    """f64 Body rows -> GpuEvolveState records with the checks of
    create_evolving_state (nbody_gpu.rs:786-825)."""
    b = np.asarray(bodies, dtype=np.float64)
    if b.ndim != 2 or b.shape[1] != 5:
        raise ValueError("bodies must have shape (n, 5): x, y, vx, vy, mass")
    if len(b) < 2 or len(b) > 2 ** 30:
        raise ValueError("GPU evolving state requires 2..=2^30 resident bodies")
    bad = ~np.isfinite(b).all(axis=1) | ~(b[:, 4] > 0.0)
    if bad.any():
        raise ValueError(f"body {int(np.argmax(bad))} contains invalid evolving state")
    s = np.zeros(len(b), _lib.EVOLVE_STATE_DTYPE)
    s["position_mass"][:, 0] = _checked_f32(b[:, 0], "body.x")
    s["position_mass"][:, 1] = _checked_f32(b[:, 1], "body.y")
    s["position_mass"][:, 2] = _checked_f32(b[:, 4], "body.mass")
    s["velocity"][:, 0] = _checked_f32(b[:, 2], "body.vx")
    s["velocity"][:, 1] = _checked_f32(b[:, 3], "body.vy")
    return s


def state_to_bodies(s: np.ndarray) -> np.ndarray:
    """GpuEvolveState records -> f64 Body rows (nbody_gpu.rs:1042-1061)."""
    out = np.empty((len(s), 5))
    out[:, 0] = s["position_mass"][:, 0]
    out[:, 1] = s["position_mass"][:, 1]
    out[:, 2] = s["velocity"][:, 0]
    out[:, 3] = s["velocity"][:, 1]
    out[:, 4] = s["position_mass"][:, 2]
    return out


def pack_flat_tree(bodies, tree, config: Config) -> PackedFlat:
    """nbody_gpu.rs:175-250.  ``tree`` is any object exposing ``entries``
    (fields code, body_index), ``position_by_body``, ``cells`` (fields cx,
    cy, half, mass, com_x, com_y, start, end, depth, children) and ``root``
    — the BH #2A flat tree of the host's CPU builder."""
    config.validate()
    b = np.asarray(bodies, dtype=np.float64)
    n = len(b)
    if n != len(tree.entries) or n != len(tree.position_by_body):
        raise ValueError("flat tree/body cardinality mismatch")
    if len(tree.cells) == 0 or tree.root >= len(tree.cells):
        raise ValueError("flat tree has invalid root")
    if n > 0xFFFFFFFF or len(tree.cells) > 0xFFFFFFFF:
        raise ValueError("GPU Barnes-Hut transfer requires u32-sized body/cell counts")
    settings = np.zeros((), _lib.BH_SETTINGS_DTYPE)
    settings["info"] = [n, len(tree.cells), tree.root, 0]
    settings["physics"] = [_checked_f32(config.theta, "theta"),
                           _checked_f32(config.softening_kpc, "softening_kpc"),
                           _checked_f32(config.g, "G"), 0.0]
    pb = np.zeros(n, _lib.GPU_BODY_DTYPE)
    pb["position_mass"][:, 0] = _checked_f32(b[:, 0], "body.x")
    pb["position_mass"][:, 1] = _checked_f32(b[:, 1], "body.y")
    pb["position_mass"][:, 2] = _checked_f32(b[:, 4], "body.mass")
    pb["meta"][:, 0] = tree.position_by_body
    pe = np.zeros(n, _lib.GPU_ENTRY_DTYPE)
    pe["data"][:, 0] = tree.entries["code"]
    pe["data"][:, 1] = tree.entries["body_index"]
    c = tree.cells
    pc = np.zeros(len(c), _lib.GPU_CELL_DTYPE)
    for k, name in enumerate(["cx", "cy", "half", "mass"]):
        pc["center_half_mass"][:, k] = _checked_f32(c[name], f"cell.{name}")
    pc["com"][:, 0] = _checked_f32(c["com_x"], "cell.com_x")
    pc["com"][:, 1] = _checked_f32(c["com_y"], "cell.com_y")
    pc["range_depth"][:, 0] = c["start"]
    pc["range_depth"][:, 1] = c["end"]
    pc["range_depth"][:, 2] = c["depth"]
    pc["children"] = c["children"]
    return PackedFlat(settings, pb, pe, pc)


class _Handle:
    """Owns one C handle and frees it with its destroy function."""

    def __init__(self, destroy_name: str):
        self.p = C.c_void_p()
        self._destroy = destroy_name

    def close(self):
        if self.p:
            try:
                getattr(_lib.load(), self._destroy)(self.p)
            finally:
                self.p = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class EvolvingState:
    """nbody_gpu.rs:132-138: persistent f32 state + acceleration buffers."""

    def __init__(self, gpu: "NbodyGpu", count: int):
        self.gpu = gpu
        self.count = count
        self._h = _Handle("galaxy_bh_state_destroy")

    @property
    def handle(self):
        return self._h.p

    def close(self):
        self._h.close()


class NbodyGpu:
    """nbody_gpu.rs:312-1433 on a CUDA device.

    ``name`` selects the device: an ordinal string ("0") or a substring of the
    device name, as the reference's adapter selection (nbody_gpu.rs:278-296);
    ``allow_software`` is accepted for signature parity (a CUDA device is
    always hardware)."""

    def __init__(self, name: str | None = None, allow_software: bool = False):
        L = _lib.load()
        ordinal = 0
        if name is not None and str(name).isdigit():
            ordinal = int(name)
        self._h = _Handle("galaxy_bh_device_close")
        check(L.galaxy_bh_device_open(ordinal, C.byref(self._h.p)))
        self._info = json.loads(self._info_raw())
        if name is not None and not str(name).isdigit() and \
                str(name).lower() not in self._info["name"].lower():
            self.close()
            raise EngineUnavailable("No matching hardware compute adapter.")
        self.allow_software = allow_software

    def _info_raw(self) -> str:
        buf = C.create_string_buffer(1024)
        check(_lib.load().galaxy_bh_device_info(self._h.p, buf, len(buf)))
        return buf.value.decode()

    @property
    def handle(self):
        return self._h.p

    def close(self):
        self._h.close()

    def info(self) -> dict:
        return dict(self._info)

    def stream_ptr(self) -> int:
        s = C.c_void_p()
        check(_lib.load().galaxy_bh_device_stream(self._h.p, C.byref(s)))
        return s.value or 0

    # -- BH #2B1 host-tree path ------------------------------------------
    def traverse(self, packed: PackedFlat) -> TraversalResult:
        """nbody_gpu.rs:640-780."""
        n = len(packed.bodies)
        out = np.zeros(n, _lib.GPU_ACCEL_DTYPE)
        t = BhStageTiming()
        s = np.ascontiguousarray(packed.settings)
        check(_lib.load().galaxy_bh_traverse_packed(
            self._h.p, ptr(s), ptr(np.ascontiguousarray(packed.bodies)), n,
            ptr(np.ascontiguousarray(packed.entries)), ptr(np.ascontiguousarray(packed.cells)),
            len(packed.cells), ptr(out), C.byref(t)))
        acc = out["value"][:, :2].astype(np.float64)
        return TraversalResult(acc, self.info(), packed.byte_len(), t.transfer_seconds,
                               t.dispatch_seconds, t.readback_seconds)

    def force_into(self, evolving: EvolvingState, packed: PackedFlat) -> StageTiming:
        """nbody_gpu.rs:854-938."""
        if len(packed.bodies) != evolving.count or len(packed.entries) != evolving.count:
            raise EngineError(_lib.BH_INVALID_ARG,
                              "Barnes-Hut force/tree count does not match evolving state")
        t = BhStageTiming()
        check(_lib.load().galaxy_bh_force_into(
            self._h.p, evolving.handle, ptr(np.ascontiguousarray(packed.settings)),
            ptr(np.ascontiguousarray(packed.bodies)), ptr(np.ascontiguousarray(packed.entries)),
            ptr(np.ascontiguousarray(packed.cells)), len(packed.cells), C.byref(t)))
        return StageTiming.of(t)

    # -- persistent evolving state ----------------------------------------
    def create_evolving_state(self, bodies) -> tuple[EvolvingState, StageTiming]:
        """nbody_gpu.rs:786-852."""
        s = bodies_to_state(bodies)
        return self.create_evolving_state_records(s)

    def create_evolving_state_records(self, s: np.ndarray) -> tuple[EvolvingState, StageTiming]:
        s = np.ascontiguousarray(s, dtype=_lib.EVOLVE_STATE_DTYPE)
        ev = EvolvingState(self, len(s))
        t = BhStageTiming()
        check(_lib.load().galaxy_bh_state_create(self._h.p, ptr(s), len(s), C.byref(ev._h.p),
                                                 C.byref(t)))
        return ev, StageTiming.of(t)

    def kick_drift(self, evolving: EvolvingState, dt_myr: float) -> StageTiming:
        t = BhStageTiming()
        check(_lib.load().galaxy_bh_kick_drift(self._h.p, evolving.handle, float(dt_myr),
                                               C.byref(t)))
        return StageTiming.of(t)

    def final_kick(self, evolving: EvolvingState, dt_myr: float) -> StageTiming:
        t = BhStageTiming()
        check(_lib.load().galaxy_bh_final_kick(self._h.p, evolving.handle, float(dt_myr),
                                               C.byref(t)))
        return StageTiming.of(t)

    def final_kick_drift(self, evolving: EvolvingState, dt_myr: float) -> StageTiming:
        """final_kick then kick_drift in one pass, bit-identical to the two
        calls (what the fused step runs between steps)."""
        t = BhStageTiming()
        check(_lib.load().galaxy_bh_final_kick_drift(self._h.p, evolving.handle, float(dt_myr),
                                                     C.byref(t)))
        return StageTiming.of(t)

    def read_evolving_state_records(self, evolving: EvolvingState):
        out = np.zeros(evolving.count, _lib.EVOLVE_STATE_DTYPE)
        t = BhStageTiming()
        check(_lib.load().galaxy_bh_read_state(self._h.p, evolving.handle, ptr(out),
                                               evolving.count, C.byref(t)))
        return out, StageTiming.of(t)

    def read_evolving_state(self, evolving: EvolvingState) -> tuple[np.ndarray, StageTiming]:
        """nbody_gpu.rs:1019-1069."""
        out, t = self.read_evolving_state_records(evolving)
        return state_to_bodies(out), t

    def write_evolving_state(self, evolving: EvolvingState, bodies) -> None:
        s = bodies_to_state(bodies)
        check(_lib.load().galaxy_bh_write_state(self._h.p, evolving.handle, ptr(s), len(s)))

    def read_evolving_accelerations_f32(self, evolving: EvolvingState):
        out = np.zeros(evolving.count, _lib.GPU_ACCEL_DTYPE)
        t = BhStageTiming()
        check(_lib.load().galaxy_bh_read_accel(self._h.p, evolving.handle, ptr(out),
                                               evolving.count, C.byref(t)))
        return out["value"], StageTiming.of(t)

    def read_evolving_accelerations(self, evolving: EvolvingState):
        """nbody_gpu.rs:1071-1114."""
        v, t = self.read_evolving_accelerations_f32(evolving)
        return v[:, :2].astype(np.float64), t

    def evolving_buffer_bytes(self, evolving: EvolvingState) -> int:
        v = C.c_uint64()
        check(_lib.load().galaxy_bh_state_bytes(evolving.handle, C.byref(v)))
        return int(v.value)

    def direct_probes(self, evolving: EvolvingState, config: Config, probes) -> np.ndarray:
        """FP64 direct accelerations (k, 2) of the probe bodies on the device
        (direct_acceleration_for, nbody/src/lib.rs:315-329)."""
        p = np.ascontiguousarray(probes, dtype=np.uint32)
        out = np.zeros((len(p), 2))
        c = config.to_c()
        check(_lib.load().galaxy_bh_direct_probes(self._h.p, evolving.handle, C.byref(c), ptr(p),
                                                  len(p), ptr(out)))
        return out

    def probe_error(self, evolving: EvolvingState, config: Config, probes) -> dict:
        """Median / p99 / max relative error of the resident accelerations
        against FP64 direct sums at the probe bodies (probe_error,
        nbody/src/lib.rs:370-395, with percentiles)."""
        p = np.ascontiguousarray(probes, dtype=np.uint32)
        exact = self.direct_probes(evolving, config, p)
        acc, _ = self.read_evolving_accelerations(evolving)
        a = acc[p]
        den = np.maximum(np.hypot(exact[:, 0], exact[:, 1]), 1e-30)
        rel = np.hypot(a[:, 0] - exact[:, 0], a[:, 1] - exact[:, 1]) / den
        return {"probes": int(len(p)), "median": float(np.median(rel)),
                "p99": float(np.quantile(rel, 0.99)), "max": float(rel.max()),
                "rms": float(np.sqrt(np.mean(rel ** 2)))}

    def conservation(self, evolving: EvolvingState) -> dict:
        """FP64 invariants of the resident state (galaxy-bh-evolve.rs:252-278
        plus kinetic, potential and total energy)."""
        out = (C.c_double * 10)()
        check(_lib.load().galaxy_bh_conservation(self._h.p, evolving.handle, out))
        keys = ["mass", "com_x", "com_y", "px", "py", "lz", "kinetic", "potential",
                "mass_speed_scale", "energy"]
        return dict(zip(keys, list(out)))


@dataclass
class ParallelGpuTree:
    """nbody_parallel.rs:66-81."""

    count: int
    config: Config
    _h: _Handle = field(repr=False, default=None)

    @property
    def handle(self):
        return self._h.p

    def close(self):
        self._h.close()


@dataclass
class ParallelGpuTreeEvidence:
    """nbody_parallel.rs:83-91 (cells in the reference preorder)."""

    meta: np.ndarray
    entries: np.ndarray
    bodies: np.ndarray
    cells: np.ndarray
    active_cell_count: int
    leaf_count: int
    max_depth: int

    def packed(self, config: Config) -> PackedFlat:
        """The BH #2B1 packed flat tree (nbody_gpu.rs:175-250) of this
        evidence: the same records pack_flat_tree writes for the
        reference's CPU tree of the same bodies (root cell 0)."""
        settings = np.zeros((), _lib.BH_SETTINGS_DTYPE)
        settings["info"] = [len(self.bodies), self.active_cell_count, 0, 0]
        settings["physics"] = [_checked_f32(config.theta, "theta"),
                               _checked_f32(config.softening_kpc, "softening_kpc"),
                               _checked_f32(config.g, "G"), 0.0]
        return PackedFlat(settings, self.bodies, self.entries, self.cells)


class ParallelTreeRuntime:
    """nbody_parallel.rs:93-993: GPU tree construction, force and evidence."""

    def __init__(self, gpu: NbodyGpu):
        self.gpu = gpu

    def create_tree(self, gpu: NbodyGpu, evolving: EvolvingState,
                    config: Config | None = None) -> ParallelGpuTree:
        config = config or Config()
        tree = ParallelGpuTree(evolving.count, config, _Handle("galaxy_bh_tree_destroy"))
        c = config.to_c()
        check(_lib.load().galaxy_bh_tree_create(gpu.handle, evolving.handle, C.byref(c),
                                                C.byref(tree._h.p)))
        tree._state = evolving
        tree._gpu = gpu
        return tree

    def rebuild(self, gpu: NbodyGpu, evolving: EvolvingState, tree: ParallelGpuTree,
                config: Config) -> ParallelTreeBuildTiming:
        if tree.count != evolving.count:
            raise EngineError(_lib.BH_INVALID_ARG,
                              "BH #2D tree count does not match evolving state")
        c = config.to_c()
        t = BhBuildTiming()
        check(_lib.load().galaxy_bh_tree_rebuild(gpu.handle, evolving.handle, tree.handle,
                                                 C.byref(c), C.byref(t)))
        tree.config = config
        return ParallelTreeBuildTiming(t.bounds_seconds, t.morton_seconds, t.radix_seconds,
                                       t.positions_seconds, t.topology_seconds,
                                       t.aggregate_seconds)

    def force(self, gpu: NbodyGpu, evolving: EvolvingState, tree: ParallelGpuTree,
              config: Config) -> StageTiming:
        if tree.count != evolving.count:
            raise EngineError(_lib.BH_INVALID_ARG,
                              "BH #2D force/tree count does not match evolving state")
        c = config.to_c()
        t = BhStageTiming()
        check(_lib.load().galaxy_bh_force(gpu.handle, evolving.handle, tree.handle, C.byref(c),
                                          C.byref(t)))
        return StageTiming.of(t)

    def force_stats(self, gpu: NbodyGpu, tree: ParallelGpuTree) -> dict:
        s = BhForceStats()
        check(_lib.load().galaxy_bh_force_stats(gpu.handle, tree.handle, C.byref(s)))
        return {"visited_nodes": s.visited_nodes, "approximated_cells": s.approximated_cells,
                "direct_terms": s.direct_terms, "exact_mac_fallbacks": s.exact_mac_fallbacks,
                "warp_iterations": s.warp_iterations}

    def force_f64(self, gpu: NbodyGpu, evolving: EvolvingState, tree: ParallelGpuTree,
                  config: Config, abs_sum: bool = False):
        """flat_accelerations_from_tree (nbody/src/flat.rs:270-371) in f64 on
        the device over the tree of the last rebuild: (n, 2) accelerations in
        resident order, the per-body sum of term magnitudes (or None) and the
        reference's force counters."""
        n = evolving.count
        acc = np.zeros((n, 2))
        s = np.zeros(n) if abs_sum else None
        st = BhForceStats()
        c = config.to_c()
        check(_lib.load().galaxy_bh_force_f64(gpu.handle, evolving.handle, tree.handle,
                                              C.byref(c), ptr(acc),
                                              ptr(s) if s is not None else None, C.byref(st)))
        return acc, s, {"visited_nodes": st.visited_nodes,
                        "approximated_cells": st.approximated_cells,
                        "direct_terms": st.direct_terms}

    def step(self, gpu: NbodyGpu, evolving: EvolvingState, tree: ParallelGpuTree,
             config: Config, dt_myr: float, steps: int) -> None:
        """``steps`` fused KDK steps (kick_drift, rebuild, force, final_kick
        each), replayed as CUDA graphs; rebuild + force must have run once."""
        c = config.to_c()
        check(_lib.load().galaxy_bh_step(gpu.handle, evolving.handle, tree.handle, C.byref(c),
                                         float(dt_myr), int(steps)))

    def read_evidence(self, gpu: NbodyGpu, tree: ParallelGpuTree) -> ParallelGpuTreeEvidence:
        n = tree.count
        meta = np.zeros((), _lib.TREE_META_DTYPE)
        cnt = C.c_uint32()
        L = _lib.load()
        check(L.galaxy_bh_read_tree_evidence(gpu.handle, tree.handle, ptr(meta), None, None, 0,
                                             None, 0, C.byref(cnt)))
        entries = np.zeros(n, _lib.GPU_ENTRY_DTYPE)
        bodies = np.zeros(n, _lib.GPU_BODY_DTYPE)
        cells = np.zeros(cnt.value, _lib.GPU_CELL_DTYPE)
        check(L.galaxy_bh_read_tree_evidence(gpu.handle, tree.handle, ptr(meta), ptr(entries),
                                             ptr(bodies), n, ptr(cells), len(cells),
                                             C.byref(cnt)))
        if len(cells) == 0:
            raise EngineError(_lib.BH_INVALID_ARG, "BH #2D tree evidence contains no active cells")
        leaf = (cells["children"] == _lib.NO_CHILD).all(axis=1)
        return ParallelGpuTreeEvidence(meta, entries, bodies, cells, len(cells),
                                       int(leaf.sum()), int(cells["range_depth"][:, 2].max()))

    def tune(self, tree: ParallelGpuTree, radix_bits: int = 8, traverse_warps: int = 4) -> None:
        """Launch-shape knobs of this tree's steps (no counterpart in the
        reference); results are bit-identical under every setting."""
        t = _lib.BhTuning(int(radix_bits), int(traverse_warps), (C.c_uint32 * 2)(0, 0))
        check(_lib.load().galaxy_bh_tree_tune(tree.handle, C.byref(t)))

    def buffer_bytes(self, tree: ParallelGpuTree) -> int:
        v = C.c_uint64()
        check(_lib.load().galaxy_bh_tree_buffer_bytes(tree.handle, C.byref(v)))
        return int(v.value)
