"""Autotuner decision logic on the host (no GPU): the coordinate search finds
the fastest admissible setting of a synthetic cost model and records every
trial."""
from galaxy_b200.autotune import (LEAF_SIZES, Tuning, coordinate_search, size_class)


def test_size_classes_are_two_octave_bins():
    assert size_class(1 << 10) == 10
    assert size_class((1 << 12) - 1) == 10
    assert size_class(1 << 12) == 12
    assert size_class(3 << 20) == 20
    assert size_class(1 << 22) == 22


def cost(t: Tuning) -> float:
    # separable model: class 10 prefers leaf 8, class 16 prefers leaf 4,
    # 4-bit digits are slower, 4 traversal warps are fastest
    ms = 10.0
    ms += {1: 3.0, 4: 2.0, 8: 1.0, 16: 1.5}[t.leaf_by_class.get(10, 1)]
    ms += {1: 5.0, 4: 1.0, 8: 2.0, 16: 4.0}[t.leaf_by_class.get(16, 1)]
    ms += 0.0 if t.radix_bits == 8 else 0.7
    ms += {4: 0.0, 8: 0.3, 2: 0.2}[t.traverse_warps]
    return ms


def test_coordinate_search_finds_separable_optimum():
    best = coordinate_search(Tuning({10: 1, 16: 1}), [10, 16], cost)
    assert best.leaf_by_class == {10: 8, 16: 4}
    assert best.radix_bits == 8 and best.traverse_warps == 4
    # baseline + 3 alternatives per class + the other launch-knob values + the result
    assert len(best.trials) == 1 + 2 * (len(LEAF_SIZES) - 1) + 1 + 2 + 1
    assert best.trials[-1][2] == cost(best)


def test_inadmissible_leaf_sizes_are_skipped():
    # forbid leaf 8 for class 10 (say, its force error is too high)
    best = coordinate_search(Tuning({10: 1, 16: 1}), [10, 16], cost,
                             admissible=lambda cls, leaf: not (cls == 10 and leaf == 8))
    assert best.leaf_by_class[10] == 16
    assert ("leaf 2^10", 8, None, False) in best.trials


def test_tuning_maps_sizes_to_leaf_sizes():
    from galaxy_b200.nbody_gpu import Config
    t = Tuning({10: 8, 20: 4})
    cfgs = t.configs([2000, 1 << 20, 1 << 16], [Config(bucket=1)] * 3)
    assert [c.bucket for c in cfgs] == [8, 4, 1]
    assert t.as_dict()["leaf_by_class"] == {"2^10": 8, "2^20": 4}
