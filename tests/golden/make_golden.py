"""Regenerates tests/golden/reference_vectors.json from the reference tree.

Reads the reference's own test sources as text (nothing is executed except
the reference's Python layout checker, which only packs a struct fixture):
  runtime/cuda/check_barnes_hut_layout.py:14-20   canonical 144-byte hex
  runtime/src/nbody_gpu.rs:1453-1489              the same fixture in Rust
  runtime/src/nbody_gpu.rs:1440-1451              frozen record sizes
  nbody/src/flat.rs:444-457                       entry/cell sizes, Morton KATs
  nbody/src/flat.rs:483-506                       stable-order fixture
  nbody/src/flat.rs:539-564                       self-exclusion fixture
  runtime/src/nbody_parallel.rs:999-1012           control records, capacity bound
The output is committed; the tests never read the reference tree.
"""
import json
import os
import re
import subprocess
import sys

REF = (sys.argv[1] if len(sys.argv) > 1 else
       os.environ.get("GALAXY_REFERENCE_DIR", "/root/reference"))
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_vectors.json")


def read(rel):
    with open(os.path.join(REF, rel)) as f:
        return f.read()


def main():
    py = read("runtime/cuda/check_barnes_hut_layout.py")
    hex_py = "".join(re.findall(r'"([0-9a-f]+)"', py.split("EXPECTED_HEX = (")[1].split(")")[0]))
    rs = read("runtime/src/nbody_gpu.rs")
    block = rs.split("assert_eq!(\n            hex,")[1].split(".replace")[0]
    hex_rs = "".join(re.findall(r"[0-9a-f]{8,}", block))
    assert hex_py == hex_rs, "reference Python and Rust fixtures disagree"
    sizes = {m[0]: int(m[1]) for m in re.findall(r"size_of::<(\w+)>\(\), (\d+)\)", rs)}
    flat = read("nbody/src/flat.rs")
    flat_sizes = {m[0]: int(m[1]) for m in re.findall(r"size_of::<(\w+)>\(\), (\d+)\)", flat)}
    kats = [[int(a), int(b), int(c)] for a, b, c in
            re.findall(r"assert_eq!\(morton2\((\d+), (\d+)\), (\d+)\);", flat)]
    par = read("runtime/src/nbody_parallel.rs")
    ctrl = {m[0]: int(m[1]) for m in re.findall(r"size_of::<(\w+)>\(\), (\d+)\)", par)}
    checker = subprocess.run([sys.executable, os.path.join(REF, "runtime/cuda/check_barnes_hut_layout.py")],
                             capture_output=True, text=True, check=True)
    checker_json = json.loads(checker.stdout)
    out = {
        "source": "QSOLKCB/GALAXY reference tests (see make_golden.py docstring)",
        "canonical_fixture_hex": hex_py,
        "canonical_fixture_fields": {
            "settings": {"info": [1, 2, 3, 4], "physics": [0.5, 0.25, 1.0, 0.0]},
            "body": {"position_mass": [1.0, -2.0, 3.0, 0.0], "meta": [4, 5, 6, 7]},
            "entry": {"data": [0x01234567, 8, 9, 10]},
            "cell": {"center_half_mass": [1.0, 2.0, 3.0, 4.0], "com": [5.0, 6.0, 0.0, 0.0],
                     "range_depth": [7, 8, 9, 0], "children": [10, 11, 12, 0xFFFFFFFF]},
        },
        "gpu_record_bytes": sizes,
        "flat_record_bytes": flat_sizes,
        "parallel_control_record_bytes": ctrl,
        "morton_known_answers": kats,
        "morton_order_known_answer": "morton2(65535, 0) < morton2(0, 65535)",
        "stable_order_fixture": {"bodies": [[0.0, 0.0, 0.0, 0.0, 1.0]] * 8,
                                 "config": {"bucket": 1, "max_depth": 48, "softening": 0.1},
                                 "expected_order": list(range(8)), "expected_max_depth": 16},
        "max_depth_fixture": {"bodies": [[0.0, 0.0, 0.0, 0.0, 1.0]] * 8,
                              "config": {"bucket": 1, "max_depth": 1, "softening": 0.1},
                              "expected_max_depth": 1},
        "self_exclusion_fixture": {
            "bodies": [[0.0, 0.0, 0.0, 0.0, 1.0], [2.220446049250313e-16, 0.0, 0.0, 0.0, 2.0],
                       [1.0, 1.0, 0.0, 0.0, 3.0], [-1.0, -1.0, 0.0, 0.0, 4.0]],
            "config": {"theta": 2.0, "bucket": 1, "max_depth": 16, "softening": 0.01},
            "max_relative_vs_direct": 0.5},
        "parallel_capacity": {"max_bodies": 65536, "levels": 17, "cell_bytes": 64,
                              "limit_bytes": 128 * 1024 * 1024},
        "gates": {
            "theta0_vs_direct": 2e-12, "flat_vs_recursive": 1e-9,
            "theta_half_rms": 0.03, "theta_half_max": 0.25,
            "gpu_vs_flat_rms": 0.01, "gpu_vs_flat_max": 0.10,
            "direct_rms": 0.04, "direct_max": 0.30,
            "trajectory_2b2_rms": 0.02, "trajectory_2b2_max": 0.20,
            "trajectory_2d_rms": 0.03, "trajectory_2d_max": 0.30},
        "reference_layout_checker_output": checker_json,
    }
    with open(OUT, "w") as f:
        json.dump(out, f, indent=1)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
