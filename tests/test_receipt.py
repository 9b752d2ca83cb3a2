"""Receipt helpers on the host: slot-layout evidence, checksum mixing, and
the restated sweep validator on a synthetic receipt (accepts a consistent
one, rejects each inconsistency)."""
import copy

import numpy as np
import pytest

from galaxy_b200 import _lib, receipt
from galaxy_b200.nbody_gpu import Config

WORK = dict(particles=8192, preset="disc", steps=3, dt_myr=0.01, seed=303, theta=0.5,
            softening_kpc=0.05, direct_probes=12, oracle_limit=4096, benchmark_warmup=2,
            benchmark_repeats=7)


def test_mix_rotates_and_multiplies():
    h = receipt._mix(0xCBF29CE484222325, 1)
    assert h == (((0xCBF29CE484222325 ^ 1) * 0x100000001B3) & ((1 << 64) - 1)) ^ (1 << 23)


def test_level_order_cells(oracle):
    from galaxy_b200 import presets
    b = presets.make_disc(3000, 7)
    cfg = oracle.Config(theta=0.5, softening=0.05, g=4.498502151575286e-12, bucket=4,
                        max_depth=48)
    t = oracle.build_flat_tree(b, cfg)
    packed = oracle.pack_flat_tree(b, t, cfg)
    cells = np.frombuffer(packed.cells.tobytes(), dtype=_lib.GPU_CELL_DTYPE)
    lv = receipt.level_order_cells(cells, 3000)
    rd = lv["range_depth"]
    slots = rd[:, 2].astype(np.int64) * 3000 + rd[:, 0]
    assert np.all(np.diff(slots) > 0) and np.all(rd[:, 3] == 1)
    pos = {int(s): i for i, s in enumerate(slots)}
    for i in range(len(lv)):
        for c in lv["children"][i]:
            if c == _lib.NO_CHILD:
                continue
            j = pos[int(c)]
            assert rd[j, 2] == rd[i, 2] + 1 and rd[i, 0] <= rd[j, 0] < rd[j, 1] <= rd[i, 1]


def synthetic():
    samples = [0.003, 0.002, 0.004, 0.0025, 0.0031, 0.0029, 0.0027]
    return {
        "schema": receipt.SCHEMA, "status": "complete", "phase": "BH-2D",
        "builder": receipt.BUILDER, "measurement_class": "hardware",
        "hardware_performance_claim_allowed": True, "preset": "disc", "particles": 8192,
        "steps": 3, "dt_myr": 0.01, "simulated_time_myr": 0.01 * 3, "seed": 303, "theta": 0.5,
        "softening_kpc": 0.05,
        "gpu": {"index": 0, "adapter_count": 1, "name": "NVIDIA B200", "backend": "CUDA",
                "device_type": "DiscreteGpu", "driver": "CUDA driver 13000", "driver_info": "",
                "software": False},
        "host_tree_rebuilds": 0, "host_particle_readbacks_during_steps": 0, "force_solves": 4,
        "evolution_tree_builds": 4,
        "parallel_tree_buffer_bytes": receipt.tree_footprint_bytes(8192, Config()),
        "tree": {"initial_checksum_fnv_mix64": "0123456789abcdef",
                 "final_checksum_fnv_mix64": "fedcba9876543210",
                 "repeat_checksum_fnv_mix64": "fedcba9876543210", "repeat_rebuild_matches": True,
                 "active_cell_count": 3500, "leaf_count": 2300, "max_depth": 11,
                 "ordering": receipt.ORDERING, "layout": receipt.LAYOUT},
        "final_force": {"bh2a_flat_status": "skipped-particle-limit", "direct_probe_count": 12,
                        "direct_probe_rms_relative": 0.01, "direct_probe_max_relative": 0.02},
        "trajectory_vs_bh2a_flat_f64": {"status": "skipped-particle-limit", "limit": 4096},
        "gpu_oracles": {"status": "skipped-particle-limit", "limit": 4096},
        "tree_build_benchmark": {"sample_scope": receipt.SAMPLE_SCOPE,
                                 "stage_timings_are_diagnostics": True, "warmup": 2,
                                 "repeats": 7, "parallel_samples_seconds": samples,
                                 "parallel_median_seconds": sorted(samples)[3],
                                 "bh2c_serial": {"status": "skipped-bh2c-cap", "limit": 4096}},
    }


def test_validator_accepts_consistent_receipt():
    out = receipt.validate_receipt(synthetic(), **WORK)
    assert out["active_cell_count"] == 3500


@pytest.mark.parametrize("path,value", [
    (("gpu", "backend"), "OpenGL"),
    (("gpu", "software"), True),
    (("tree", "repeat_checksum_fnv_mix64"), "0000000000000000"),
    (("tree", "layout"), "preorder"),
    (("tree", "leaf_count"), 10000),
    (("tree_build_benchmark", "parallel_median_seconds"), 0.002),
    (("final_force", "direct_probe_rms_relative"), 0.05),
    (("force_solves",), 3),
    (("parallel_tree_buffer_bytes",), 12345),
])
def test_validator_rejects(path, value):
    r = copy.deepcopy(synthetic())
    d = r
    for k in path[:-1]:
        d = d[k]
    d[path[-1]] = value
    with pytest.raises(receipt.ReceiptError):
        receipt.validate_receipt(r, **WORK)


def _reference_sweep_module():
    """The reference's scripts/bench-bh2d-hardware.py, imported from the
    reference tree (present where fixtures are made, absent on GPU hosts)."""
    import importlib.util
    import os
    ref = os.environ.get("GALAXY_REFERENCE_DIR", "/root/reference")
    path = os.path.join(ref, "scripts", "bench-bh2d-hardware.py")
    if not os.path.exists(path):
        pytest.skip("reference tree absent")
    spec = importlib.util.spec_from_file_location("reference_bh2d_sweep", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_reference_sweep_validator_accepts_engine_receipts(monkeypatch):
    """Receipts this engine produced on a GPU (tests/golden/engine_receipts.json,
    made by tests/golden/make_engine_receipts.py) pass the reference's OWN
    validate_receipt (scripts/bench-bh2d-hardware.py:1013), with exactly two
    documented substitutions: the backend set admits "CUDA" (:993 admits
    Vulkan / Metal / Dx12), and the tree-buffer formula (:837-853, the
    reference's 17 N sparse 64-byte cells) is this engine's
    galaxy_bh_tree_footprint.  Every other check is the reference's code."""
    import json
    import os
    path = os.path.join(os.path.dirname(__file__), "golden", "engine_receipts.json")
    if not os.path.exists(path):
        pytest.skip("engine receipts not generated yet")
    mod = _reference_sweep_module()
    backend_msg = "receipt.gpu.backend is not enabled by the producer"
    real_require = mod.require
    seen = {"backend": 0}

    def require(condition, message):
        if message == backend_msg and not condition:
            seen["backend"] += 1
            return  # "CUDA": the one backend the reference set does not list
        real_require(condition, message)

    monkeypatch.setattr(mod, "require", require)
    monkeypatch.setattr(mod, "expected_parallel_tree_buffer_bytes",
                        lambda n: receipt.tree_footprint_bytes(n, Config()))
    cases = json.load(open(path))
    assert len(cases) >= 2
    for case in cases:
        assert case["receipt"]["gpu"]["backend"] == "CUDA"
        mod.validate_receipt(case["receipt"], **case["workload"])
    assert seen["backend"] == len(cases)
    # the unpatched validator rejects exactly on the backend
    monkeypatch.setattr(mod, "require", real_require)
    with pytest.raises(mod.SweepError, match="backend"):
        mod.validate_receipt(cases[0]["receipt"], **cases[0]["workload"])
