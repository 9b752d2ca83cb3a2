"""Failure detection on the GPU without a fault.

Every device wait of the engine (the sort's and the scan's look-back) is
bounded.  galaxy_bh_wait_probe runs the sort's look-back against a
predecessor tile that never publishes: the wait must give up after its
limit, the host must see BH_TIMEOUT with the stalled-sort message, and the
same device handle must go on computing bit-identical results.
"""
import pytest

from galaxy_b200 import _lib, scenarios
from galaxy_b200.nbody_gpu import Config, NbodyGpu, ParallelTreeRuntime, bodies_to_state

pytestmark = pytest.mark.gpu


def _evolve(gpu, rt, rec, cfg):
    ev, _ = gpu.create_evolving_state_records(rec)
    tree = rt.create_tree(gpu, ev, cfg)
    rt.rebuild(gpu, ev, tree, cfg)
    rt.force(gpu, ev, tree, cfg)
    rt.step(gpu, ev, tree, cfg, 1e-3, 3)
    out = gpu.read_evolving_state_records(ev)[0]
    tree.close()
    ev.close()
    return out


def test_bounded_wait_times_out_and_the_device_stays_usable():
    gpu = NbodyGpu("0")
    rt = ParallelTreeRuntime(gpu)
    cfg = Config(theta=0.5, softening_kpc=0.01, g=1.0)
    rec = bodies_to_state(scenarios.make("cold_disc", 5000, 3, eps=0.01))
    before = _evolve(gpu, rt, rec, cfg)
    lib = _lib.load()
    # a limit of 2e6 cycles: about a millisecond of waiting on a flag that
    # nothing sets
    assert lib.galaxy_bh_wait_probe(gpu.handle, 2_000_000) == _lib.BH_TIMEOUT
    assert "timed out" in _lib.last_error()
    assert lib.galaxy_bh_wait_probe(gpu.handle, 5_000_000_000) == _lib.BH_INVALID_ARG
    after = _evolve(gpu, rt, rec, cfg)
    assert after.tobytes() == before.tobytes()
