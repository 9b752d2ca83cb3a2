"""Batched engine: many independent simulations of uneven size advanced
together, one launch per stage for all of them (galaxy_bh_batch_* of the C
ABI).  Each member keeps its own resident state; the batch owns one scratch
arena for the per-step tree of every member.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check
from .nbody_gpu import Config, EvolvingState, NbodyGpu, _Handle


class Batch:
    """A fixed set of evolving states, each with its own Config."""

    def __init__(self, gpu: NbodyGpu, states: list[EvolvingState], configs: list[Config]):
        if len(states) != len(configs) or not states:
            raise ValueError("batch needs one config per state and at least one state")
        self.gpu = gpu
        self.states = list(states)
        self.configs = list(configs)
        arr = (C.c_void_p * len(states))(*[s.handle.value for s in states])
        cfgs = (_lib.BhConfig * len(configs))(*[c.to_c() for c in configs])
        self._h = _Handle("galaxy_bh_batch_destroy")
        check(_lib.load().galaxy_bh_batch_create(gpu.handle, arr, cfgs, len(states),
                                                 C.byref(self._h.p)))
        self.solved = False

    @property
    def bodies(self) -> int:
        return sum(s.count for s in self.states)

    def solve(self) -> None:
        """Tree rebuild + force for every member (the boundary acceleration)."""
        check(_lib.load().galaxy_bh_batch_solve(self.gpu.handle, self._h.p))
        self.solved = True

    def step(self, dts, steps: int) -> None:
        """``steps`` fused KDK steps for every member (dt per member)."""
        d = np.ascontiguousarray(np.broadcast_to(np.asarray(dts, dtype=np.float64),
                                                 (len(self.states),)))
        check(_lib.load().galaxy_bh_batch_step(self.gpu.handle, self._h.p,
                                               d.ctypes.data_as(C.POINTER(C.c_double)),
                                               int(steps)))

    def tune(self, radix_bits: int = 8, traverse_warps: int = 4) -> None:
        """Launch-shape knobs (sort digit width, warps per traversal block);
        results are bit-identical under every setting."""
        t = _lib.BhTuning(int(radix_bits), int(traverse_warps), (C.c_uint32 * 2)(0, 0))
        check(_lib.load().galaxy_bh_batch_tune(self._h.p, C.byref(t)))

    def arena_bytes(self) -> int:
        v = C.c_uint64()
        check(_lib.load().galaxy_bh_batch_bytes(self._h.p, C.byref(v)))
        return int(v.value)

    def close(self) -> None:
        self._h.close()


def footprint_bytes(counts, configs: list[Config]) -> int:
    """Device bytes a batch of these sizes needs (states + arena): the
    admission figure of the serving loop."""
    n = np.ascontiguousarray(counts, dtype=np.uint32)
    cfgs = (_lib.BhConfig * len(configs))(*[c.to_c() for c in configs])
    v = C.c_uint64()
    check(_lib.load().galaxy_bh_batch_footprint(_lib.ptr(n), cfgs, len(n), C.byref(v)))
    return int(v.value)
