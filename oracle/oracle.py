"""CPU oracle for the Barnes-Hut evolution path — TEST INFRASTRUCTURE ONLY.

ctypes bindings over ``liboracle_bh.so`` (``bh_oracle.c``), the f64 C
restatement of the reference's CPU substrate (nbody/src/lib.rs,
nbody/src/flat.rs, runtime/src/nbody_gpu.rs:175-250,
runtime/src/bin/galaxy-bh-evolve.rs:252-363).  Only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline legs of ``bench.py`` import
this module: it is the checker, never part of the engine.

Bodies are numpy float64 arrays of shape (n, 5) with columns
(x, y, vx, vy, mass), the field order of ``Body`` (nbody/src/lib.rs:12-19).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle_bh.so")
REF_CUDA_PATH = os.path.join(HERE, "_ref", "libref_bh_cuda.so")

NO_CHILD = 0xFFFFFFFF
G_KPC3_PER_MSUN_MYR2 = 4.498502151575286e-12
DEFAULT_SOFTENING_KPC = 0.05


class OracleError(RuntimeError):
    pass


class Config(C.Structure):
    """nbody/src/lib.rs:27-46 (defaults theta 0.5, eps 0.05, G kpc units,
    bucket 4, max_depth 48)."""

    _fields_ = [
        ("theta", C.c_double),
        ("softening", C.c_double),
        ("g", C.c_double),
        ("bucket", C.c_uint64),
        ("max_depth", C.c_uint64),
    ]

    def __init__(self, theta=0.5, softening=DEFAULT_SOFTENING_KPC, g=G_KPC3_PER_MSUN_MYR2,
                 bucket=4, max_depth=48):
        super().__init__(theta, softening, g, bucket, max_depth)


class _TreeStats(C.Structure):
    _fields_ = [("node_count", C.c_uint64), ("leaf_count", C.c_uint64), ("max_depth", C.c_uint64)]


class _ForceStats(C.Structure):
    _fields_ = [("visited_nodes", C.c_uint64), ("approximated_cells", C.c_uint64),
                ("direct_terms", C.c_uint64)]


class _TreeInfo(C.Structure):
    _fields_ = [("body_count", C.c_uint32), ("cell_count", C.c_uint32), ("root", C.c_uint32),
                ("morton_axis_bits", C.c_uint32), ("stats", _TreeStats),
                ("root_cx", C.c_double), ("root_cy", C.c_double), ("root_half", C.c_double)]


ENTRY_DTYPE = np.dtype([("code", "<u4"), ("body_index", "<u4")])
CELL_DTYPE = np.dtype([
    ("cx", "<f8"), ("cy", "<f8"), ("half", "<f8"), ("mass", "<f8"),
    ("com_x", "<f8"), ("com_y", "<f8"),
    ("start", "<u4"), ("end", "<u4"), ("depth", "<u4"), ("children", "<u4", (4,)),
], align=True)
assert CELL_DTYPE.itemsize == 80  # sizeof(ob_cell), the FlatCell size (flat.rs:447)


def build_oracle() -> None:
    """Compile liboracle_bh.so (and the reference CUDA shim when the
    reference tree is present) with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
    ref = os.environ.get("GALAXY_REFERENCE_DIR", "/root/reference")
    if os.path.isdir(ref):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={ref}"], check=False)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build_oracle()
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        sz = C.c_size_t
        cfg = C.POINTER(Config)
        L.ob_last_error.restype = C.c_char_p
        L.ob_validate_config.argtypes = [cfg]
        L.ob_validate_bodies.argtypes = [P, sz]
        L.ob_root_bounds.argtypes = [P, sz, P]
        L.ob_root_bounds.restype = None
        L.ob_spread16.argtypes = [C.c_uint32]
        L.ob_spread16.restype = C.c_uint32
        L.ob_morton2.argtypes = [C.c_uint32, C.c_uint32]
        L.ob_morton2.restype = C.c_uint32
        L.ob_quantize_axis.argtypes = [C.c_double] * 3
        L.ob_quantize_axis.restype = C.c_uint32
        L.ob_morton_key_for_point.argtypes = [C.c_double] * 5
        L.ob_morton_key_for_point.restype = C.c_uint32
        L.ob_flat_tree_build.argtypes = [P, sz, cfg, C.POINTER(P)]
        L.ob_flat_tree_free.argtypes = [P]
        L.ob_flat_tree_free.restype = None
        L.ob_flat_tree_get_info.argtypes = [P, C.POINTER(_TreeInfo)]
        L.ob_flat_tree_get_info.restype = None
        L.ob_flat_tree_copy.argtypes = [P, P, P, P]
        L.ob_flat_tree_copy.restype = None
        L.ob_flat_topology_checksum.argtypes = [P]
        L.ob_flat_topology_checksum.restype = C.c_uint64
        L.ob_topology_checksum_arrays.argtypes = [C.c_uint32, P, C.c_uint32, C.c_uint32, P]
        L.ob_topology_checksum_arrays.restype = C.c_uint64
        L.ob_flat_accelerations.argtypes = [P, sz, P, cfg, P, sz, P, P, C.POINTER(_ForceStats),
                                            C.c_int]
        L.ob_direct_acceleration_for.argtypes = [sz, P, sz, cfg, P]
        L.ob_direct_accelerations.argtypes = [P, sz, cfg, P]
        L.ob_direct_accelerations_for.argtypes = [P, sz, cfg, P, sz, P, C.c_int]
        L.ob_probe_error.argtypes = [P, sz, P, cfg, sz, P]
        L.ob_bh1_accelerations.argtypes = [P, sz, cfg, P, C.POINTER(_TreeStats),
                                           C.POINTER(_ForceStats)]
        L.ob_bh1_leapfrog_step_from_acceleration.argtypes = [P, sz, C.c_double, cfg, P, sz, P]
        L.ob_make_disc.argtypes = [sz, C.c_uint64, C.c_double, C.c_double, P]
        L.ob_make_collision.argtypes = [sz, C.c_uint64, P]
        L.ob_state_checksum.argtypes = [P, sz]
        L.ob_state_checksum.restype = C.c_uint64
        L.ob_pack_flat_tree.argtypes = [P, sz, P, cfg, P, P, P, P]
        L.ob_cpu_flat_evolve.argtypes = [P, sz, sz, C.c_double, cfg, C.c_int]
        L.ob_cpu_flat_steps.argtypes = [P, sz, P, sz, C.c_double, cfg, C.c_int,
                                         C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.ob_invariants.argtypes = [P, sz, P]
        L.ob_invariants.restype = None
        L.ob_f32_kick_drift.argtypes = [P, P, sz, C.c_float]
        L.ob_f32_kick_drift.restype = None
        L.ob_f32_final_kick.argtypes = [P, P, sz, C.c_float]
        L.ob_f32_final_kick.restype = None
        L.ob_f32_traverse_packed.argtypes = [P, P, P, P, sz, P]
        _lib = L
    return _lib


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def _check(rc: int) -> None:
    if rc != 0:
        raise OracleError(lib().ob_last_error().decode())


def _bodies(b) -> np.ndarray:
    b = np.ascontiguousarray(b, dtype=np.float64)
    if b.ndim != 2 or b.shape[1] != 5:
        raise ValueError("bodies must have shape (n, 5): x, y, vx, vy, mass")
    return b


def nthreads_default() -> int:
    return max(1, os.cpu_count() or 1)


# -------------------------------------------------------------- primitives --

def spread16(v: int) -> int:
    return lib().ob_spread16(v)


def morton2(x: int, y: int) -> int:
    return lib().ob_morton2(x, y)


def quantize_axis(value: float, center: float, half: float) -> int:
    return lib().ob_quantize_axis(value, center, half)


def morton_key_for_point(x, y, cx, cy, half) -> int:
    return lib().ob_morton_key_for_point(x, y, cx, cy, half)


def root_bounds(bodies) -> tuple[float, float, float]:
    b = _bodies(bodies)
    out = np.zeros(3)
    lib().ob_root_bounds(_ptr(b), len(b), _ptr(out))
    return float(out[0]), float(out[1]), float(out[2])


def validate_config(cfg: Config) -> None:
    _check(lib().ob_validate_config(C.byref(cfg)))


# ---------------------------------------------------------------- flat tree --

@dataclass
class FlatTree:
    """nbody/src/flat.rs:49-58 plus the root bounds."""

    entries: np.ndarray           # ENTRY_DTYPE, sorted order
    position_by_body: np.ndarray  # u32
    cells: np.ndarray             # CELL_DTYPE, recursive preorder
    root: int
    node_count: int
    leaf_count: int
    max_depth: int
    root_bounds: tuple
    checksum: int
    _handle: object = None

    @property
    def codes(self) -> np.ndarray:
        return self.entries["code"]

    @property
    def order(self) -> np.ndarray:
        return self.entries["body_index"]


class _Handle:
    def __init__(self, p):
        self.p = p

    def __del__(self):
        if self.p:
            lib().ob_flat_tree_free(self.p)
            self.p = None


def build_flat_tree(bodies, cfg: Config) -> FlatTree:
    b = _bodies(bodies)
    h = C.c_void_p()
    _check(lib().ob_flat_tree_build(_ptr(b), len(b), C.byref(cfg), C.byref(h)))
    handle = _Handle(h)
    info = _TreeInfo()
    lib().ob_flat_tree_get_info(h, C.byref(info))
    entries = np.zeros(info.body_count, ENTRY_DTYPE)
    pos = np.zeros(info.body_count, np.uint32)
    cells = np.zeros(info.cell_count, CELL_DTYPE)
    lib().ob_flat_tree_copy(h, _ptr(entries), _ptr(pos), _ptr(cells))
    return FlatTree(entries, pos, cells, info.root, info.stats.node_count, info.stats.leaf_count,
                    info.stats.max_depth, (info.root_cx, info.root_cy, info.root_half),
                    int(lib().ob_flat_topology_checksum(h)), handle)


def topology_checksum_arrays(entry_words: np.ndarray, cells16: np.ndarray) -> int:
    """flat_topology_checksum (flat.rs:416-433) of a tree given as raw words:
    entry_words (n, k>=2) u32 with code, body_index first; cells16 (C, 16) u32
    GpuCell records."""
    e = np.ascontiguousarray(entry_words, dtype=np.uint32)
    c = np.ascontiguousarray(cells16, dtype=np.uint32).reshape(-1, 16)
    return int(lib().ob_topology_checksum_arrays(len(e), _ptr(e), e.shape[1], len(c), _ptr(c)))


def flat_accelerations(bodies, tree: FlatTree, cfg: Config, targets=None, abs_sum=False,
                       nthreads=None):
    """flat.rs:348-371; returns (acc (k,2), stats dict[, abs_sum (k,)])."""
    b = _bodies(bodies)
    nthreads = nthreads or nthreads_default()
    if targets is None:
        t_ptr, k = None, len(b)
    else:
        targets = np.ascontiguousarray(targets, dtype=np.uint32)
        t_ptr, k = _ptr(targets), len(targets)
    out = np.zeros((k, 2))
    s = np.zeros(k) if abs_sum else None
    st = _ForceStats()
    _check(lib().ob_flat_accelerations(_ptr(b), len(b), tree._handle.p, C.byref(cfg), t_ptr,
                                       k, _ptr(out), _ptr(s) if abs_sum else None,
                                       C.byref(st), nthreads))
    stats = {"visited_nodes": st.visited_nodes, "approximated_cells": st.approximated_cells,
             "direct_terms": st.direct_terms}
    return (out, stats, s) if abs_sum else (out, stats)


def flat_barnes_hut_accelerations(bodies, cfg: Config):
    tree = build_flat_tree(bodies, cfg)
    acc, stats = flat_accelerations(bodies, tree, cfg)
    return acc, tree, stats


# ------------------------------------------------------------------ direct --

def direct_accelerations(bodies, cfg: Config) -> np.ndarray:
    b = _bodies(bodies)
    out = np.zeros((len(b), 2))
    _check(lib().ob_direct_accelerations(_ptr(b), len(b), C.byref(cfg), _ptr(out)))
    return out


def direct_acceleration_for(index: int, bodies, cfg: Config) -> np.ndarray:
    b = _bodies(bodies)
    out = np.zeros(2)
    _check(lib().ob_direct_acceleration_for(index, _ptr(b), len(b), C.byref(cfg), _ptr(out)))
    return out


def direct_accelerations_for(bodies, cfg: Config, targets, nthreads=None) -> np.ndarray:
    b = _bodies(bodies)
    targets = np.ascontiguousarray(targets, dtype=np.uint32)
    out = np.zeros((len(targets), 2))
    _check(lib().ob_direct_accelerations_for(_ptr(b), len(b), C.byref(cfg), _ptr(targets),
                                             len(targets), _ptr(out),
                                             nthreads or nthreads_default()))
    return out


def probe_error(bodies, approx, cfg: Config, probes: int) -> tuple[float, float]:
    b = _bodies(bodies)
    a = np.ascontiguousarray(approx, dtype=np.float64).reshape(len(b), 2)
    out = np.zeros(2)
    _check(lib().ob_probe_error(_ptr(b), len(b), _ptr(a), C.byref(cfg), probes, _ptr(out)))
    return float(out[0]), float(out[1])


def relative_errors(approx, exact) -> np.ndarray:
    """|a - e| / max(|e|, 1e-30) per row (nbody/src/lib.rs:549-551)."""
    approx = np.asarray(approx, dtype=np.float64)[:, :2]
    exact = np.asarray(exact, dtype=np.float64)[:, :2]
    den = np.maximum(np.hypot(exact[:, 0], exact[:, 1]), 1e-30)
    return np.hypot(approx[:, 0] - exact[:, 0], approx[:, 1] - exact[:, 1]) / den


# ------------------------------------------------------------------- BH #1 --

def bh1_accelerations(bodies, cfg: Config):
    b = _bodies(bodies)
    out = np.zeros((len(b), 2))
    ts, fs = _TreeStats(), _ForceStats()
    _check(lib().ob_bh1_accelerations(_ptr(b), len(b), C.byref(cfg), _ptr(out), C.byref(ts),
                                      C.byref(fs)))
    return out, {"node_count": ts.node_count, "leaf_count": ts.leaf_count,
                 "max_depth": ts.max_depth}, {"visited_nodes": fs.visited_nodes,
                                              "approximated_cells": fs.approximated_cells,
                                              "direct_terms": fs.direct_terms}


def bh1_leapfrog_step_from_acceleration(bodies, dt, cfg: Config, first):
    """Returns (new_bodies, second_acc); raises on length mismatch."""
    b = _bodies(bodies).copy()
    f = np.ascontiguousarray(first, dtype=np.float64).reshape(-1, 2)
    second = np.zeros((len(b), 2))
    _check(lib().ob_bh1_leapfrog_step_from_acceleration(_ptr(b), len(b), dt, C.byref(cfg),
                                                        _ptr(f), len(f), _ptr(second)))
    return b, second


def bh1_leapfrog_step(bodies, dt, cfg: Config):
    first, _, _ = bh1_accelerations(bodies, cfg)
    return bh1_leapfrog_step_from_acceleration(bodies, dt, cfg, first)


# --------------------------------------------------------------------- ICs --

def make_disc(count, seed, total_mass=5.0e10, scale=3.0) -> np.ndarray:
    out = np.zeros((count, 5))
    _check(lib().ob_make_disc(count, seed, total_mass, scale, _ptr(out)))
    return out


def make_collision(count, seed) -> np.ndarray:
    out = np.zeros((count, 5))
    _check(lib().ob_make_collision(count, seed, _ptr(out)))
    return out


def state_checksum(bodies) -> int:
    b = _bodies(bodies)
    return int(lib().ob_state_checksum(_ptr(b), len(b)))


def invariants(bodies) -> np.ndarray:
    b = _bodies(bodies)
    out = np.zeros(7)
    lib().ob_invariants(_ptr(b), len(b), _ptr(out))
    return out


# ----------------------------------------------------------------- packing --

@dataclass
class Packed:
    """runtime/src/nbody_gpu.rs:141-146 as raw little-endian u32 words."""

    settings: np.ndarray  # (8,) u32
    bodies: np.ndarray    # (n, 8) u32
    entries: np.ndarray   # (n, 4) u32
    cells: np.ndarray     # (C, 16) u32

    def as_bytes(self) -> bytes:
        return (self.settings.tobytes() + self.bodies.tobytes() + self.entries.tobytes()
                + self.cells.tobytes())


def pack_flat_tree(bodies, tree: FlatTree, cfg: Config) -> Packed:
    b = _bodies(bodies)
    n, nc = len(b), len(tree.cells)
    s = np.zeros(8, np.uint32)
    pb = np.zeros((n, 8), np.uint32)
    pe = np.zeros((n, 4), np.uint32)
    pc = np.zeros((nc, 16), np.uint32)
    _check(lib().ob_pack_flat_tree(_ptr(b), n, tree._handle.p, C.byref(cfg), _ptr(s), _ptr(pb),
                                   _ptr(pe), _ptr(pc)))
    return Packed(s, pb, pe, pc)


# --------------------------------------------------------------- evolution --

def cpu_flat_evolve(bodies, steps: int, dt: float, cfg: Config, nthreads=1) -> np.ndarray:
    """runtime/src/bin/galaxy-bh-evolve.rs:339-363 (f64, rebuild every step)."""
    b = _bodies(bodies).copy()
    _check(lib().ob_cpu_flat_evolve(_ptr(b), len(b), steps, dt, C.byref(cfg), nthreads))
    return b


def cpu_flat_steps(bodies: np.ndarray, acc: np.ndarray, steps: int, dt: float, cfg: Config,
                   nthreads=1) -> tuple[float, float]:
    """In place: ``steps`` KDK steps of bodies (n,5) from boundary acc (n,2)
    (galaxy-bh-evolve.rs:348-361).  Returns (build_seconds, force_seconds)."""
    assert bodies.dtype == np.float64 and bodies.flags.c_contiguous
    assert acc.dtype == np.float64 and acc.flags.c_contiguous and acc.shape == (len(bodies), 2)
    tb, tf = C.c_double(0.0), C.c_double(0.0)
    _check(lib().ob_cpu_flat_steps(_ptr(bodies), len(bodies), _ptr(acc), steps, dt,
                                   C.byref(cfg), nthreads, C.byref(tb), C.byref(tf)))
    return tb.value, tf.value


def f32_kick_drift(states: np.ndarray, accel: np.ndarray, dt: float) -> np.ndarray:
    """nbody_evolve.wgsl:19-33 on (n, 8) float32 GpuEvolveState records."""
    s = np.ascontiguousarray(states, dtype=np.float32).copy()
    a = np.ascontiguousarray(accel, dtype=np.float32)
    lib().ob_f32_kick_drift(_ptr(s), _ptr(a), len(s), np.float32(dt))
    return s


def f32_final_kick(states: np.ndarray, accel: np.ndarray, dt: float) -> np.ndarray:
    s = np.ascontiguousarray(states, dtype=np.float32).copy()
    a = np.ascontiguousarray(accel, dtype=np.float32)
    lib().ob_f32_final_kick(_ptr(s), _ptr(a), len(s), np.float32(dt))
    return s


def f32_traverse_packed(p: Packed) -> np.ndarray:
    n = len(p.bodies)
    out = np.zeros((n, 4), np.float32)
    rc = lib().ob_f32_traverse_packed(_ptr(p.settings), _ptr(p.bodies), _ptr(p.entries),
                                      _ptr(p.cells), n, _ptr(out))
    if rc:
        raise OracleError("f32 traversal stack overflow")
    return out


# ------------------------------------------------ reference CUDA kernels --

_ref = None


def ref_cuda():
    """The reference's own barnes_hut_flat.cu kernels, built from source into
    _ref/ (None when they were not built)."""
    global _ref
    if _ref is None:
        if not os.path.exists(REF_CUDA_PATH):
            return None
        L = C.CDLL(REF_CUDA_PATH)
        P = C.c_void_p
        L.ref_bh_traverse.argtypes = [P, P, C.c_uint32, P, P, C.c_uint32, P,
                                      C.POINTER(C.c_float), C.c_int]
        L.ref_bh_kick_drift.argtypes = [P, P, C.c_uint32, C.c_float]
        L.ref_bh_final_kick.argtypes = [P, P, C.c_uint32, C.c_float]
        L.ref_bh_integrate_timed.argtypes = [C.c_int, P, P, C.c_uint32, C.c_float,
                                             C.POINTER(C.c_float), C.c_int]
        L.ref_bh_integrate_single.argtypes = [C.c_int, P, P, C.c_uint32, C.c_float,
                                              C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_int]
        L.ref_bh_traverse_single.argtypes = [P, P, C.c_uint32, P, P, C.c_uint32,
                                             C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_int]
        _ref = L
    return _ref


def ref_cuda_traverse(p: Packed, repeats=1):
    L = ref_cuda()
    n = len(p.bodies)
    out = np.zeros((n, 4), np.float32)
    ms = C.c_float(0.0)
    rc = L.ref_bh_traverse(_ptr(p.settings), _ptr(p.bodies), n, _ptr(p.entries), _ptr(p.cells),
                           len(p.cells), _ptr(out), C.byref(ms), repeats)
    if rc:
        raise OracleError(f"reference CUDA traversal failed: cudaError {rc}")
    return out, float(ms.value)


def ref_cuda_integrate_timed(states, accel, dt, final_kick=False, repeats=5):
    """The reference's bh_kick_drift / bh_final_kick over (states, accel):
    (states after one launch, mean device ms of `repeats` further launches)."""
    L = ref_cuda()
    s = np.ascontiguousarray(states, dtype=np.float32).copy()
    a = np.ascontiguousarray(accel, dtype=np.float32)
    ms = C.c_float(0.0)
    rc = L.ref_bh_integrate_timed(int(final_kick), _ptr(s), _ptr(a), len(s), np.float32(dt),
                                  C.byref(ms), repeats)
    if rc:
        raise OracleError(f"reference CUDA integrate failed: cudaError {rc}")
    return s, float(ms.value)


def ref_cuda_single_times(p: Packed, states, accel, dt, repeats=7) -> dict:
    """Median single-launch device ms of the reference's bh_traverse (over
    the packed tree p), bh_kick_drift and bh_final_kick (over states,
    accel), each with L2 warm and with L2 flushed before every launch."""
    L = ref_cuda()
    out = {}
    w, c = C.c_float(0.0), C.c_float(0.0)
    rc = L.ref_bh_traverse_single(_ptr(p.settings), _ptr(p.bodies), len(p.bodies),
                                  _ptr(p.entries), _ptr(p.cells), len(p.cells), C.byref(w),
                                  C.byref(c), repeats)
    if rc:
        raise OracleError(f"reference CUDA traversal failed: cudaError {rc}")
    out["traverse"] = (float(w.value), float(c.value))
    s = np.ascontiguousarray(states, dtype=np.float32)
    a = np.ascontiguousarray(accel, dtype=np.float32)
    for name, fk in (("kick_drift", 0), ("final_kick", 1)):
        rc = L.ref_bh_integrate_single(fk, _ptr(s), _ptr(a), len(s), np.float32(dt), C.byref(w),
                                       C.byref(c), repeats)
        if rc:
            raise OracleError(f"reference CUDA integrate failed: cudaError {rc}")
        out[name] = (float(w.value), float(c.value))
    return out


def ref_cuda_integrate(states, accel, dt, final_kick=False):
    L = ref_cuda()
    s = np.ascontiguousarray(states, dtype=np.float32).copy()
    a = np.ascontiguousarray(accel, dtype=np.float32)
    fn = L.ref_bh_final_kick if final_kick else L.ref_bh_kick_drift
    rc = fn(_ptr(s), _ptr(a), len(s), np.float32(dt))
    if rc:
        raise OracleError(f"reference CUDA integrate failed: cudaError {rc}")
    return s
