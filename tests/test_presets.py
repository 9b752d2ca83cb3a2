"""The product's restatement of the reference ICs equals the oracle's (both
follow nbody/src/lib.rs:430-528) bit for bit."""
import numpy as np

from galaxy_b200 import presets


def test_disc_matches_oracle(oracle):
    for n, seed in ((2, 0), (1000, 42), (4097, 303)):
        got = presets.make_disc(n, seed)
        want = oracle.make_disc(n, seed)
        assert np.array_equal(got.view(np.uint64), np.ascontiguousarray(want).view(np.uint64))


def test_collision_matches_oracle(oracle):
    for n, seed in ((4, 1), (3001, 303)):
        got = presets.make_collision(n, seed)
        want = oracle.make_collision(n, seed)
        assert np.array_equal(got.view(np.uint64), np.ascontiguousarray(want).view(np.uint64))


def test_state_checksum_of_preset(oracle):
    b = presets.make("disc", 512, 303)
    assert oracle.state_checksum(b) == oracle.state_checksum(oracle.make_disc(512, 303))
