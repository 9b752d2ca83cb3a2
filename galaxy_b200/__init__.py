"""B200-native Barnes-Hut resident self-gravity engine (sm_100a).

Drop-in for the reference BH evolution path: ``NbodyGpu`` /
``ParallelTreeRuntime`` (host mirror in ``nbody_gpu``) over the C ABI of
``include/galaxy_bh.h``, implemented by the CUDA kernels in ``csrc/``.
"""
from .nbody_gpu import (Config, EngineError, EngineUnavailable, EvolvingState, NbodyGpu,
                        PackedFlat, ParallelGpuTree, ParallelTreeRuntime, StageTiming,
                        bodies_to_state, pack_flat_tree, state_to_bodies)

__all__ = ["Config", "EngineError", "EngineUnavailable", "EvolvingState", "NbodyGpu",
           "PackedFlat", "ParallelGpuTree", "ParallelTreeRuntime", "StageTiming",
           "bodies_to_state", "pack_flat_tree", "state_to_bodies"]
