"""ctypes binding of the C ABI declared in include/galaxy_bh.h.

The engine is the in-tree ``libgalaxy_bh.so`` built by ``galaxy_b200.build``
(nvcc, sm_100a).  There is no fallback: when the library is missing every
call raises ``EngineUnavailable``.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# GALAXY_BH_LIB selects another build of the same library (e.g. a tuning variant).
LIB_PATH = os.environ.get("GALAXY_BH_LIB") or os.path.join(HERE, "libgalaxy_bh.so")

NO_CHILD = 0xFFFFFFFF

BH_OK = 0
BH_INVALID_ARG = 1
BH_CAPACITY_OVERFLOW = 2
BH_NONFINITE = 3
BH_OOM = 4
BH_TIMEOUT = 5
BH_CUDA_ERROR = 6
BH_NO_DEVICE = 7
STATUS_NAMES = {0: "OK", 1: "INVALID_ARG", 2: "CAPACITY_OVERFLOW", 3: "NONFINITE", 4: "OOM",
                5: "TIMEOUT", 6: "CUDA_ERROR", 7: "NO_DEVICE"}

BH_FLAG_COMPENSATED = 1
BH_FLAG_POTENTIAL = 2
BH_FLAG_NO_STATS = 4

# Frozen record dtypes (runtime/src/nbody_gpu.rs:22-83), all little-endian.
EVOLVE_STATE_DTYPE = np.dtype([("position_mass", "<f4", (4,)), ("velocity", "<f4", (4,))])
GPU_BODY_DTYPE = np.dtype([("position_mass", "<f4", (4,)), ("meta", "<u4", (4,))])
GPU_ENTRY_DTYPE = np.dtype([("data", "<u4", (4,))])
GPU_CELL_DTYPE = np.dtype([("center_half_mass", "<f4", (4,)), ("com", "<f4", (4,)),
                           ("range_depth", "<u4", (4,)), ("children", "<u4", (4,))])
GPU_ACCEL_DTYPE = np.dtype([("value", "<f4", (4,))])
BH_SETTINGS_DTYPE = np.dtype([("info", "<u4", (4,)), ("physics", "<f4", (4,))])
TREE_META_DTYPE = np.dtype([("data", "<u4", (4,)), ("bounds", "<f4", (4,))])
for _dt, _size in [(EVOLVE_STATE_DTYPE, 32), (GPU_BODY_DTYPE, 32), (GPU_ENTRY_DTYPE, 16),
                   (GPU_CELL_DTYPE, 64), (GPU_ACCEL_DTYPE, 16), (BH_SETTINGS_DTYPE, 32),
                   (TREE_META_DTYPE, 32)]:
    assert _dt.itemsize == _size


class EngineError(RuntimeError):
    """A C ABI call failed; ``status`` is the bh_status code."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{message} [{STATUS_NAMES.get(status, status)}]")
        self.status = status
        self.message = message


class EngineUnavailable(EngineError):
    def __init__(self, message: str):
        super().__init__(BH_NO_DEVICE, message)


class BhConfig(C.Structure):
    _fields_ = [("theta", C.c_double), ("softening", C.c_double), ("g", C.c_double),
                ("bucket", C.c_uint32), ("max_depth", C.c_uint32), ("flags", C.c_uint32),
                ("reserved", C.c_uint32)]


class BhStageTiming(C.Structure):
    _fields_ = [("transfer_seconds", C.c_double), ("dispatch_seconds", C.c_double),
                ("readback_seconds", C.c_double)]


class BhBuildTiming(C.Structure):
    _fields_ = [("bounds_seconds", C.c_double), ("morton_seconds", C.c_double),
                ("radix_seconds", C.c_double), ("positions_seconds", C.c_double),
                ("topology_seconds", C.c_double), ("aggregate_seconds", C.c_double)]


class BhTuning(C.Structure):
    _fields_ = [("radix_bits", C.c_uint32), ("traverse_warps", C.c_uint32),
                ("reserved", C.c_uint32 * 2)]


class BhServeConfig(C.Structure):
    _fields_ = [("budget_bytes", C.c_uint64), ("round_steps", C.c_uint32),
                ("max_members", C.c_uint32)]


class BhServeResult(C.Structure):
    _fields_ = [("request_id", C.c_uint64), ("n", C.c_uint32), ("status", C.c_uint32),
                ("steps", C.c_uint32), ("reserved", C.c_uint32), ("submitted_s", C.c_double),
                ("admitted_s", C.c_double), ("finished_s", C.c_double)]


class BhServeStats(C.Structure):
    _fields_ = [("rounds", C.c_uint64), ("particle_steps", C.c_uint64),
                ("completed", C.c_uint64), ("busy_seconds", C.c_double),
                ("elapsed_seconds", C.c_double), ("admit_seconds", C.c_double),
                ("solve_seconds", C.c_double), ("form_seconds", C.c_double),
                ("readback_seconds", C.c_double)]


class BhForceStats(C.Structure):
    _fields_ = [("visited_nodes", C.c_uint64), ("approximated_cells", C.c_uint64),
                ("direct_terms", C.c_uint64), ("exact_mac_fallbacks", C.c_uint64),
                ("warp_iterations", C.c_uint64)]


# name -> (restype, argtypes); every exported symbol of include/galaxy_bh.h.
_P = C.c_void_p
_PP = C.POINTER(C.c_void_p)
_U32 = C.c_uint32
SIGNATURES = {
    "galaxy_bh_last_error": (C.c_size_t, [C.c_char_p, C.c_size_t]),
    "galaxy_bh_abi_version": (_U32, []),
    "galaxy_bh_device_open": (C.c_int, [C.c_int, _PP]),
    "galaxy_bh_device_close": (C.c_int, [_P]),
    "galaxy_bh_device_info": (C.c_int, [_P, C.c_char_p, C.c_size_t]),
    "galaxy_bh_device_stream": (C.c_int, [_P, _PP]),
    "galaxy_bh_state_create": (C.c_int, [_P, _P, _U32, _PP, C.POINTER(BhStageTiming)]),
    "galaxy_bh_state_destroy": (C.c_int, [_P]),
    "galaxy_bh_state_count": (C.c_int, [_P, C.POINTER(_U32)]),
    "galaxy_bh_state_bytes": (C.c_int, [_P, C.POINTER(C.c_uint64)]),
    "galaxy_bh_kick_drift": (C.c_int, [_P, _P, C.c_double, C.POINTER(BhStageTiming)]),
    "galaxy_bh_final_kick": (C.c_int, [_P, _P, C.c_double, C.POINTER(BhStageTiming)]),
    "galaxy_bh_final_kick_drift": (C.c_int, [_P, _P, C.c_double, C.POINTER(BhStageTiming)]),
    "galaxy_bh_read_state": (C.c_int, [_P, _P, _P, _U32, C.POINTER(BhStageTiming)]),
    "galaxy_bh_read_accel": (C.c_int, [_P, _P, _P, _U32, C.POINTER(BhStageTiming)]),
    "galaxy_bh_write_state": (C.c_int, [_P, _P, _P, _U32]),
    "galaxy_bh_tree_create": (C.c_int, [_P, _P, C.POINTER(BhConfig), _PP]),
    "galaxy_bh_tree_destroy": (C.c_int, [_P]),
    "galaxy_bh_tree_rebuild": (C.c_int, [_P, _P, _P, C.POINTER(BhConfig),
                                         C.POINTER(BhBuildTiming)]),
    "galaxy_bh_force": (C.c_int, [_P, _P, _P, C.POINTER(BhConfig), C.POINTER(BhStageTiming)]),
    "galaxy_bh_force_stats": (C.c_int, [_P, _P, C.POINTER(BhForceStats)]),
    "galaxy_bh_force_f64": (C.c_int, [_P, _P, _P, C.POINTER(BhConfig), _P, _P,
                                      C.POINTER(BhForceStats)]),
    "galaxy_bh_wait_probe": (C.c_int, [_P, C.c_uint64]),
    "galaxy_bh_read_tree_evidence": (C.c_int, [_P, _P, _P, _P, _P, _U32, _P, _U32,
                                               C.POINTER(_U32)]),
    "galaxy_bh_tree_buffer_bytes": (C.c_int, [_P, C.POINTER(C.c_uint64)]),
    "galaxy_bh_traverse_packed": (C.c_int, [_P, _P, _P, _U32, _P, _P, _U32, _P,
                                            C.POINTER(BhStageTiming)]),
    "galaxy_bh_force_into": (C.c_int, [_P, _P, _P, _P, _P, _P, _U32, C.POINTER(BhStageTiming)]),
    "galaxy_bh_step": (C.c_int, [_P, _P, _P, C.POINTER(BhConfig), C.c_double, _U32]),
    "galaxy_bh_conservation": (C.c_int, [_P, _P, C.POINTER(C.c_double)]),
    "galaxy_bh_direct_probes": (C.c_int, [_P, _P, C.POINTER(BhConfig), _P, _U32, _P]),
    "galaxy_bh_conservation_noalloc": (C.c_int, [_P, _P, _U32, _P, _P]),
    "galaxy_bh_batch_create": (C.c_int, [_P, _P, C.POINTER(BhConfig), _U32, _PP]),
    "galaxy_bh_batch_destroy": (C.c_int, [_P]),
    "galaxy_bh_batch_solve": (C.c_int, [_P, _P]),
    "galaxy_bh_batch_step": (C.c_int, [_P, _P, C.POINTER(C.c_double), _U32]),
    "galaxy_bh_batch_bytes": (C.c_int, [_P, C.POINTER(C.c_uint64)]),
    "galaxy_bh_batch_tune": (C.c_int, [_P, _P]),
    "galaxy_bh_serve_start": (C.c_int, [C.c_int, _P, C.POINTER(C.c_void_p)]),
    "galaxy_bh_serve_submit": (C.c_int, [_P, _P, C.c_uint32, _P, C.c_double, C.c_uint32,
                                         C.POINTER(C.c_uint64)]),
    "galaxy_bh_serve_poll": (C.c_int, [_P, C.c_uint32, _P, _P, C.c_uint32]),
    "galaxy_bh_serve_stats": (C.c_int, [_P, _P]),
    "galaxy_bh_serve_stop": (C.c_int, [_P]),
    "galaxy_bh_tree_footprint": (C.c_int, [C.c_uint32, _P, C.POINTER(C.c_uint64)]),
    "galaxy_bh_tree_tune": (C.c_int, [_P, _P]),
    "galaxy_bh_batch_footprint": (C.c_int, [_P, C.POINTER(BhConfig), _U32,
                                            C.POINTER(C.c_uint64)]),
}

_lib = None


def load():
    """Loads libgalaxy_bh.so and declares every entry point."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise EngineUnavailable(
                f"CUDA extension {LIB_PATH} is missing: build it with "
                "`python -m galaxy_b200.build` (nvcc, sm_100a)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def last_error() -> str:
    buf = C.create_string_buffer(1024)
    load().galaxy_bh_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(rc: int) -> None:
    if rc != BH_OK:
        msg = last_error()
        if rc == BH_NO_DEVICE:
            raise EngineUnavailable(msg)
        raise EngineError(rc, msg)


def ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)
