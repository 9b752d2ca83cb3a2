"""The CPU oracle pinned against the reference's own golden vectors and unit-test
gates (nbody/src/lib.rs:545-635, nbody/src/flat.rs:435-598,
runtime/src/nbody_gpu.rs:1435-1512, runtime/src/nbody_parallel.rs:995-1013)."""
import json
import os
import struct

import numpy as np
import pytest

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden",
                                     "reference_vectors.json")))


def cfg(o, **kw):
    return o.Config(**kw)


def test_morton_known_answers(oracle):
    # flat.rs:451-457
    for x, y, code in GOLDEN["morton_known_answers"]:
        assert oracle.morton2(x, y) == code
    assert oracle.morton2(65535, 0) < oracle.morton2(0, 65535)
    assert oracle.spread16(0xFFFF) == 0x55555555


def test_quantize_axis_clamps_and_floors(oracle):
    assert oracle.quantize_axis(-10.0, 0.0, 1.0) == 0
    assert oracle.quantize_axis(10.0, 0.0, 1.0) == 65535
    assert oracle.quantize_axis(0.0, 0.0, 1.0) == 32768
    assert oracle.quantize_axis(1.0, 0.0, 1.0) == 65535


def test_canonical_layout_fixture_hex(oracle):
    # nbody_gpu.rs:1453-1489 / check_barnes_hut_layout.py:22-36
    f = GOLDEN["canonical_fixture_fields"]
    raw = b"".join([
        struct.pack("<4I4f", *f["settings"]["info"], *f["settings"]["physics"]),
        struct.pack("<4f4I", *f["body"]["position_mass"], *f["body"]["meta"]),
        struct.pack("<4I", *f["entry"]["data"]),
        struct.pack("<8f8I", *f["cell"]["center_half_mass"], *f["cell"]["com"],
                    *f["cell"]["range_depth"], *f["cell"]["children"]),
    ])
    assert len(raw) == 144
    assert raw.hex() == GOLDEN["canonical_fixture_hex"]
    assert GOLDEN["reference_layout_checker_output"]["status"] == "pass"


def test_record_sizes_are_frozen():
    sizes = GOLDEN["gpu_record_bytes"]
    assert sizes == {"BhSettings": 32, "GpuBody": 32, "GpuEntry": 16, "GpuCell": 64,
                     "GpuAccel": 16, "EvolveSettings": 32, "GpuEvolveState": 32,
                     "TreeSettings": 32, "TreeMeta": 32}
    assert GOLDEN["flat_record_bytes"] == {"MortonEntry": 8, "FlatCell": 80}


def test_stable_equal_keys_preserve_resident_order(oracle):
    # flat.rs:483-506
    fx = GOLDEN["stable_order_fixture"]
    t = oracle.build_flat_tree(np.array(fx["bodies"]), cfg(oracle, **fx["config"]))
    assert list(t.order) == fx["expected_order"]
    assert t.max_depth == fx["expected_max_depth"]


def test_configured_max_depth_honored(oracle):
    # flat.rs:459-481
    fx = GOLDEN["max_depth_fixture"]
    t = oracle.build_flat_tree(np.array(fx["bodies"]), cfg(oracle, **fx["config"]))
    assert t.max_depth == fx["expected_max_depth"]
    assert (t.cells["depth"] <= 1).all()


def test_flat_tree_preserves_range_and_mass(oracle):
    # flat.rs:508-518
    b = oracle.make_disc(256, 303, 5.0e10, 3.0)
    t = oracle.build_flat_tree(b, cfg(oracle))
    root = t.cells[t.root]
    assert root["start"] == 0 and root["end"] == 256
    assert abs(root["mass"] - 5.0e10) < 1e-3
    assert t.node_count > t.leaf_count
    assert t.max_depth <= 16


def test_flat_theta_zero_matches_direct(oracle):
    # flat.rs:520-537
    b = oracle.make_disc(128, 303, 5.0e10, 3.0)
    c = cfg(oracle, theta=0.0)
    acc, _, _ = oracle.flat_barnes_hut_accelerations(b, c)
    direct = oracle.direct_accelerations(b, c)
    assert oracle.relative_errors(acc, direct).max() < GOLDEN["gates"]["theta0_vs_direct"]


def test_self_exclusion_uses_morton_range(oracle):
    # flat.rs:539-564
    fx = GOLDEN["self_exclusion_fixture"]
    b = np.array(fx["bodies"])
    c = cfg(oracle, **fx["config"])
    acc, _, _ = oracle.flat_barnes_hut_accelerations(b, c)
    direct = oracle.direct_accelerations(b, c)
    assert oracle.relative_errors(acc, direct).max() < fx["max_relative_vs_direct"]


def test_flat_theta_half_gate(oracle):
    # flat.rs:566-573
    b = oracle.make_disc(256, 303, 5.0e10, 3.0)
    c = cfg(oracle)
    acc, _, stats = oracle.flat_barnes_hut_accelerations(b, c)
    rel = oracle.relative_errors(acc, oracle.direct_accelerations(b, c))
    assert np.sqrt(np.mean(rel ** 2)) < 0.03
    assert rel.max() < 0.25
    assert stats["approximated_cells"] > 0


def test_flat_and_recursive_agree(oracle):
    # flat.rs:575-589
    b = oracle.make_disc(256, 303, 5.0e10, 3.0)
    c = cfg(oracle)
    rec, _, _ = oracle.bh1_accelerations(b, c)
    flat, _, _ = oracle.flat_barnes_hut_accelerations(b, c)
    assert oracle.relative_errors(flat, rec).max() < GOLDEN["gates"]["flat_vs_recursive"]


def test_topology_checksum_repeatable(oracle):
    # flat.rs:591-597
    b = oracle.make_disc(512, 919, 5.0e10, 3.0)
    a = oracle.build_flat_tree(b, cfg(oracle))
    bb = oracle.build_flat_tree(b, cfg(oracle))
    assert a.checksum == bb.checksum


def test_bh1_tree_preserves_count_and_mass(oracle):
    # lib.rs:553-561
    b = oracle.make_disc(256, 303, 5.0e10, 3.0)
    _, ts, _ = oracle.bh1_accelerations(b, cfg(oracle))
    assert ts["node_count"] > ts["leaf_count"] and ts["max_depth"] > 0


def test_bh1_theta_zero_matches_direct(oracle):
    # lib.rs:563-572
    b = oracle.make_disc(128, 303, 5.0e10, 3.0)
    c = cfg(oracle, theta=0.0)
    acc, _, _ = oracle.bh1_accelerations(b, c)
    assert oracle.relative_errors(acc, oracle.direct_accelerations(b, c)).max() < 2e-12


def test_bh1_duplicates_terminate_at_depth_bound(oracle):
    # lib.rs:583-592
    b = np.array([[0.0, 0.0, 0.0, 0.0, 1.0]] * 8)
    c = cfg(oracle, bucket=1, max_depth=12, softening=0.1)
    acc, ts, _ = oracle.bh1_accelerations(b, c)
    assert ts["max_depth"] <= 12
    assert np.isfinite(acc).all()


def test_leapfrog_moves_state_and_reuse_matches(oracle):
    # lib.rs:594-618
    c = cfg(oracle)
    b = oracle.make_disc(128, 77, 5.0e10, 3.0)
    moved, _ = oracle.bh1_leapfrog_step(b, 0.01, c)
    assert (moved[:, :2] != b[:, :2]).any() and np.isfinite(moved).all()
    conv = oracle.make_disc(128, 88, 5.0e10, 3.0)
    first, _, _ = oracle.bh1_accelerations(conv, c)
    a, acc_a = oracle.bh1_leapfrog_step(conv, 0.01, c)
    r, acc_r = oracle.bh1_leapfrog_step_from_acceleration(conv, 0.01, c, first)
    assert np.array_equal(a, r) and np.array_equal(acc_a, acc_r)


def test_leapfrog_rejects_wrong_length(oracle):
    # lib.rs:620-626
    b = oracle.make_disc(8, 89, 5.0e10, 3.0)
    with pytest.raises(oracle.OracleError, match="acceleration count"):
        oracle.bh1_leapfrog_step_from_acceleration(b, 0.01, cfg(oracle), np.zeros((0, 2)))


def test_seeded_state_and_checksum_repeatable(oracle):
    # lib.rs:628-634
    a = oracle.make_collision(256, 999)
    b = oracle.make_collision(256, 999)
    assert np.array_equal(a, b)
    assert oracle.state_checksum(a) == oracle.state_checksum(b)
    assert oracle.state_checksum(a) != oracle.state_checksum(oracle.make_collision(256, 998))


def test_config_validation_messages(oracle):
    # lib.rs:48-66
    for kw, msg in [({"theta": -1.0}, "theta"), ({"softening": float("nan")}, "softening"),
                    ({"g": 0.0}, "g must be"), ({"bucket": 0}, "bucket"),
                    ({"max_depth": 129}, "max_depth")]:
        with pytest.raises(oracle.OracleError, match=msg):
            oracle.validate_config(cfg(oracle, **kw))


def test_invalid_bodies_rejected(oracle):
    # lib.rs:122-135
    with pytest.raises(oracle.OracleError, match="at least two"):
        oracle.build_flat_tree(np.zeros((1, 5)) + [0, 0, 0, 0, 1], cfg(oracle))
    b = oracle.make_disc(16, 1)
    b[3, 4] = 0.0
    with pytest.raises(oracle.OracleError, match="mass"):
        oracle.build_flat_tree(b, cfg(oracle))
    b = oracle.make_disc(16, 1)
    b[5, 0] = np.inf
    with pytest.raises(oracle.OracleError, match="non-finite"):
        oracle.build_flat_tree(b, cfg(oracle))


def test_pack_preserves_ranges_children_positions(oracle):
    # nbody_gpu.rs:1491-1511
    b = oracle.make_disc(128, 303, 5.0e10, 3.0)
    c = cfg(oracle)
    t = oracle.build_flat_tree(b, c)
    p = oracle.pack_flat_tree(b, t, c)
    assert p.settings[0] == 128 and p.settings[1] == len(t.cells) and p.settings[2] == t.root
    assert np.array_equal(p.bodies[:, 4], t.position_by_body)
    assert np.array_equal(p.cells[:, 8], t.cells["start"])
    assert np.array_equal(p.cells[:, 9], t.cells["end"])
    assert np.array_equal(p.cells[:, 10], t.cells["depth"])
    assert np.array_equal(p.cells[:, 12:16], t.cells["children"])
    assert (p.cells[:, 12:16] != 0xFFFFFFFF).any()


def test_pack_rejects_unrepresentable_f32(oracle):
    # nbody_gpu.rs:167-173
    b = oracle.make_disc(16, 3)
    b[0, 4] = 1e300
    c = cfg(oracle)
    t = oracle.build_flat_tree(b, c)
    with pytest.raises(oracle.OracleError, match="finite f32"):
        oracle.pack_flat_tree(b, t, c)


def test_parallel_capacity_below_128mib():
    # nbody_parallel.rs:1006-1012
    p = GOLDEN["parallel_capacity"]
    assert p["max_bodies"] * p["levels"] * p["cell_bytes"] < p["limit_bytes"]


def test_preorder_equals_start_depth_order(oracle):
    """The engine numbers cells by ascending (start, depth); the oracle's
    recursive preorder (flat.rs:127-177) must be exactly that order."""
    for seed, bucket in [(3, 1), (4, 4), (5, 16)]:
        b = oracle.make_disc(3000, seed)
        t = oracle.build_flat_tree(b, cfg(oracle, bucket=bucket))
        key = t.cells["start"].astype(np.int64) * 64 + t.cells["depth"]
        assert (np.diff(key) > 0).all()


def test_f32_traversal_model_close_to_f64(oracle):
    """The f32 model of nbody.wgsl agrees with the f64 flat traversal within
    the reference GPU-vs-flat gate (galaxy-bh-gpu.rs:109)."""
    b = oracle.make_disc(1024, 303, 5.0e10, 3.0)
    c = cfg(oracle)
    t = oracle.build_flat_tree(b, c)
    p = oracle.pack_flat_tree(b, t, c)
    a32 = oracle.f32_traverse_packed(p)
    a64, _ = oracle.flat_accelerations(b, t, c)
    rel = oracle.relative_errors(a32.astype(np.float64), a64)
    assert np.sqrt(np.mean(rel ** 2)) < 0.01 and rel.max() < 0.10


def test_cpu_flat_evolve_matches_manual_kdk(oracle):
    """galaxy-bh-evolve.rs:339-363 restated: N steps equal a hand-written KDK
    over the oracle's own tree and forces."""
    b0 = oracle.make_disc(200, 5, 5.0e10, 3.0)
    c = cfg(oracle)
    out = oracle.cpu_flat_evolve(b0, 3, 0.01, c)
    b = b0.copy()
    acc, _, _ = oracle.flat_barnes_hut_accelerations(b, c)
    for _ in range(3):
        b[:, 2] += 0.5 * 0.01 * acc[:, 0]
        b[:, 3] += 0.5 * 0.01 * acc[:, 1]
        b[:, 0] += 0.01 * b[:, 2]
        b[:, 1] += 0.01 * b[:, 3]
        acc, _, _ = oracle.flat_barnes_hut_accelerations(b, c)
        b[:, 2] += 0.5 * 0.01 * acc[:, 0]
        b[:, 3] += 0.5 * 0.01 * acc[:, 1]
    assert np.array_equal(out, b)


def test_threaded_force_equals_single_thread(oracle):
    b = oracle.make_collision(4000, 12)
    c = cfg(oracle)
    t = oracle.build_flat_tree(b, c)
    a1, s1 = oracle.flat_accelerations(b, t, c, nthreads=1)
    a8, s8 = oracle.flat_accelerations(b, t, c, nthreads=8)
    assert np.array_equal(a1, a8) and s1 == s8
