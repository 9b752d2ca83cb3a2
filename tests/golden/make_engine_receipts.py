"""Writes tests/golden/engine_receipts.json: receipts of the BH #2D run
(galaxy.barnes-hut-parallel-gpu-tree-receipt.v1) produced by this engine on a
GPU, for the reference sweep's own workloads (scripts/bench-bh2d-hardware.py
defaults: disc and collision presets, 3 steps, dt 0.01 Myr, seed 303, theta
0.5, softening 0.05 kpc, 12 direct probes, oracle limit 4096, 2 warm-up and
7 timed rebuilds).  Needs a CUDA device; run from the repository root:

    python tests/golden/make_engine_receipts.py

tests/test_receipt.py hands the committed receipts to the reference's own
validate_receipt (when the reference tree is present).
"""
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "engine_receipts.json")

WORKLOADS = [
    dict(particles=8192, preset="disc", steps=3, dt_myr=0.01, seed=303, theta=0.5,
         softening_kpc=0.05, direct_probes=12, oracle_limit=4096, benchmark_warmup=2,
         benchmark_repeats=7),
    dict(particles=65536, preset="disc", steps=3, dt_myr=0.01, seed=303, theta=0.5,
         softening_kpc=0.05, direct_probes=12, oracle_limit=4096, benchmark_warmup=2,
         benchmark_repeats=7),
    dict(particles=16384, preset="collision", steps=3, dt_myr=0.01, seed=303, theta=0.5,
         softening_kpc=0.05, direct_probes=12, oracle_limit=4096, benchmark_warmup=2,
         benchmark_repeats=7),
]


def main():
    from galaxy_b200 import receipt
    out = []
    for work in WORKLOADS:
        r = receipt.run_receipt(**work)
        receipt.validate_receipt(r, **work)  # the restated checks first
        out.append({"workload": work, "receipt": r})
    with open(OUT, "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print(f"wrote {len(out)} receipts to {OUT}")


if __name__ == "__main__":
    main()
