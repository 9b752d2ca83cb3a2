"""Batched engine: a member's result is the same alone and in the mix.

Each simulation advanced inside a batch of uneven sizes, scenarios and
configs must end bit-identical (state and accelerations) to the same
simulation advanced alone through the plain path — per-simulation results
never depend on the batch composition.
"""
import numpy as np
import pytest

from galaxy_b200 import scenarios
from galaxy_b200.batch import Batch
from galaxy_b200.nbody_gpu import Config, NbodyGpu, ParallelTreeRuntime

pytestmark = pytest.mark.gpu

MEMBERS = [
    ("exponential_disc", 1500, 11, Config(theta=0.5, softening_kpc=0.01, g=1.0, bucket=1)),
    ("cold_disc", 40000, 12, Config(theta=0.5, softening_kpc=0.01, g=1.0, bucket=4)),
    # compensated two-sum beside plain members: each keeps its own summation form
    ("binary_encounter", 4097, 13, Config(theta=0.3, softening_kpc=0.005, g=1.0, bucket=1,
                                          compensated=True)),
    ("exponential_disc", 70001, 14, Config(theta=0.7, softening_kpc=0.01, g=1.0, bucket=8)),
    ("cold_disc", 33, 15, Config(theta=0.5, softening_kpc=0.01, g=1.0, bucket=16)),
]
DTS = [1e-3, 5e-4, 1e-3, 2e-3, 1e-3]
STEPS = 4


@pytest.fixture(scope="module")
def gpu():
    return NbodyGpu("0")


def _alone(gpu, bodies, cfg, dt):
    rt = ParallelTreeRuntime(gpu)
    ev, _ = gpu.create_evolving_state(bodies)
    tree = rt.create_tree(gpu, ev, cfg)
    rt.rebuild(gpu, ev, tree, cfg)
    rt.force(gpu, ev, tree, cfg)
    rt.step(gpu, ev, tree, cfg, dt, STEPS)
    return (gpu.read_evolving_state_records(ev)[0], gpu.read_evolving_accelerations_f32(ev)[0])


def test_batch_members_equal_alone(gpu):
    bodies = [scenarios.make(name, n, seed) for name, n, seed, _ in MEMBERS]
    states = [gpu.create_evolving_state(b)[0] for b in bodies]
    batch = Batch(gpu, states, [m[3] for m in MEMBERS])
    batch.solve()
    batch.step(DTS, STEPS)
    for k, (b, (_, _, _, cfg), dt) in enumerate(zip(bodies, MEMBERS, DTS)):
        want_state, want_acc = _alone(gpu, b, cfg, dt)
        got_state = gpu.read_evolving_state_records(states[k])[0]
        got_acc = gpu.read_evolving_accelerations_f32(states[k])[0]
        assert got_state.tobytes() == want_state.tobytes(), f"member {k} state"
        assert np.array_equal(got_acc, want_acc), f"member {k} accelerations"


def test_batch_solve_matches_plain_force(gpu):
    bodies = [scenarios.make(name, n, seed) for name, n, seed, _ in MEMBERS]
    states = [gpu.create_evolving_state(b)[0] for b in bodies]
    batch = Batch(gpu, states, [m[3] for m in MEMBERS])
    batch.solve()
    rt = ParallelTreeRuntime(gpu)
    for k, (b, (_, _, _, cfg)) in enumerate(zip(bodies, MEMBERS)):
        ev, _ = gpu.create_evolving_state(b)
        tree = rt.create_tree(gpu, ev, cfg)
        rt.rebuild(gpu, ev, tree, cfg)
        rt.force(gpu, ev, tree, cfg)
        assert np.array_equal(gpu.read_evolving_accelerations_f32(states[k])[0],
                              gpu.read_evolving_accelerations_f32(ev)[0])


def test_launch_tuning_changes_no_bit(gpu):
    """4-bit vs 8-bit sort digits and 4 vs 8 traversal warps per block give
    the same tree, accelerations and trajectory, bit for bit, on the plain
    path and in a batch."""
    rt = ParallelTreeRuntime(gpu)
    bodies = scenarios.binary_encounter(30000, seed=21)
    cfg = Config(theta=0.5, softening_kpc=0.005, g=1.0, bucket=1)
    results = []
    for bits, warps in ((8, 8), (4, 8), (8, 4), (4, 4), (8, 2)):
        ev, _ = gpu.create_evolving_state(bodies)
        tree = rt.create_tree(gpu, ev, cfg)
        rt.tune(tree, bits, warps)
        rt.rebuild(gpu, ev, tree, cfg)
        evid = rt.read_evidence(gpu, tree)
        rt.force(gpu, ev, tree, cfg)
        a0 = gpu.read_evolving_accelerations_f32(ev)[0]
        rt.step(gpu, ev, tree, cfg, 5e-4, 3)
        results.append((evid.entries.tobytes(), evid.cells.tobytes(), a0.tobytes(),
                        gpu.read_evolving_state_records(ev)[0].tobytes()))
        tree.close()
        ev.close()
    assert all(r == results[0] for r in results[1:])
    # batched: same members, both knob settings
    states = []
    for bits, warps in ((8, 8), (4, 4)):
        evs = [gpu.create_evolving_state(scenarios.make(n, c, s))[0] for n, c, s, _ in MEMBERS]
        b = Batch(gpu, evs, [m[3] for m in MEMBERS])
        b.tune(bits, warps)
        b.solve()
        b.step(DTS, STEPS)
        states.append([gpu.read_evolving_state_records(e)[0].tobytes() for e in evs])
        b.close()
    assert states[0] == states[1]


def test_autotune_batch_picks_admissible_settings(gpu):
    from galaxy_b200.autotune import LEAF_SIZES, size_class, tune_batch
    rng = np.random.default_rng(5)
    sizes = [int(2 ** rng.uniform(10, 15)) for _ in range(10)]
    evs = [gpu.create_evolving_state(scenarios.make("exponential_disc", n, 100 + i))[0]
           for i, n in enumerate(sizes)]
    cfgs = [Config(theta=0.5, softening_kpc=0.01, g=1.0, bucket=1)] * len(evs)
    before = [gpu.read_evolving_state_records(e)[0].tobytes() for e in evs]
    t = tune_batch(gpu, evs, cfgs, dt=1e-3, steps=2, probes=128)
    assert set(t.leaf_by_class) == {size_class(n) for n in sizes}
    assert all(v in LEAF_SIZES for v in t.leaf_by_class.values())
    assert t.radix_bits in (4, 8) and t.traverse_warps in (2, 4, 8)
    assert t.trials[-1][0] == "best" and t.trials[-1][2] > 0
    # tuning ran on copies: the caller's states are untouched
    assert before == [gpu.read_evolving_state_records(e)[0].tobytes() for e in evs]


def test_receipt_run_passes_the_sweep_checks(gpu):
    """A receipt of the reference sweep's workload (disc preset, 8192 bodies,
    3 steps) produced on this engine passes the restated sweep validator."""
    from galaxy_b200 import receipt
    work = dict(particles=8192, preset="disc", steps=3, dt_myr=0.01, seed=303, theta=0.5,
                softening_kpc=0.05, direct_probes=12, oracle_limit=4096, benchmark_warmup=2,
                benchmark_repeats=7)
    r = receipt.run_receipt(**work)
    out = receipt.validate_receipt(r, **work)
    assert out["leaf_count"] > 0 and r["tree"]["repeat_rebuild_matches"]
