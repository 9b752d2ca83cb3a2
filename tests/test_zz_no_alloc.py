"""galaxy_bh_conservation_noalloc, the entry point for callers that cannot
allocate device memory (a serving loop with a fixed, pre-reserved budget, a
host whose allocator owns the device memory, code handed only device
buffers).  It is called here through the C ABI with device buffers the test
owns, twice in a row on different inputs, and each result is checked
against galaxy_bh_conservation on the same records.  Kept in a file pytest
collects last; it passes alone in a fresh process and after the others.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

REL = 1e-12  # f64 sums in a different association order


def _device_records(torch, records):
    return torch.from_numpy(records.view(np.uint8).copy()).cuda()


def _noalloc(torch, lib, records, potential=None):
    d_state = _device_records(torch, records)
    d_pot = None if potential is None else torch.from_numpy(potential).cuda()
    d_sums = torch.full((9,), float("nan"), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()
    from galaxy_b200 import _lib
    _lib.check(lib.galaxy_bh_conservation_noalloc(
        C.c_void_p(d_state.data_ptr()), None if d_pot is None else C.c_void_p(d_pot.data_ptr()),
        len(records), C.c_void_p(d_sums.data_ptr()), C.c_void_p(stream.cuda_stream)))
    stream.synchronize()
    return d_sums.cpu().numpy()


def _existing(gpu, records):
    ev, _ = gpu.create_evolving_state_records(records)
    c = gpu.conservation(ev)
    ev.close()
    return c


def _compare(sums, ref):
    scale = sums[8] + abs(sums[0])
    assert sums[0] == pytest.approx(ref["mass"], rel=REL)
    assert sums[1] / sums[0] == pytest.approx(ref["com_x"], rel=REL, abs=REL * 10)
    assert sums[2] / sums[0] == pytest.approx(ref["com_y"], rel=REL, abs=REL * 10)
    for k, name in [(3, "px"), (4, "py"), (5, "lz"), (6, "kinetic")]:
        assert sums[k] == pytest.approx(ref[name], rel=REL, abs=REL * scale), name
    assert sums[7] == 0.0
    assert sums[8] == pytest.approx(ref["mass_speed_scale"], rel=REL)


def test_noalloc_matches_existing_on_two_calls():
    import torch

    from galaxy_b200 import _lib, scenarios
    from galaxy_b200.nbody_gpu import NbodyGpu, bodies_to_state
    lib = _lib.load()
    gpu = NbodyGpu("0")
    first = bodies_to_state(scenarios.exponential_disc(300_000, 5))
    second = bodies_to_state(scenarios.binary_encounter(12_345, 6))
    s1 = _noalloc(torch, lib, first)
    s2 = _noalloc(torch, lib, second)
    _compare(s1, _existing(gpu, first))
    _compare(s2, _existing(gpu, second))


def test_noalloc_potential_and_limits():
    import torch

    from galaxy_b200 import _lib, scenarios
    from galaxy_b200.nbody_gpu import bodies_to_state
    lib = _lib.load()
    recs = bodies_to_state(scenarios.cold_disc(50_000, 3))
    phi = np.random.default_rng(0).uniform(-3.0, -1.0, len(recs)).astype(np.float32)
    sums = _noalloc(torch, lib, recs, phi)
    m = recs["position_mass"][:, 2].astype(np.float64)
    assert sums[7] == pytest.approx(0.5 * np.sum(m * phi.astype(np.float64)), rel=REL)
    # beyond the scratch limit: rejected before any device work
    d = torch.zeros(32, dtype=torch.uint8, device="cuda")
    out = torch.zeros(9, dtype=torch.float64, device="cuda")
    rc = lib.galaxy_bh_conservation_noalloc(C.c_void_p(d.data_ptr()), None, 4_194_305,
                                            C.c_void_p(out.data_ptr()), None)
    assert rc == _lib.BH_INVALID_ARG
    assert "4194304" in _lib.last_error()
    assert lib.galaxy_bh_conservation_noalloc(None, None, 10, None, None) == _lib.BH_INVALID_ARG


def test_noalloc_at_the_limit_allocates_nothing():
    """n = 4,194,304 fills every scratch row; the sums equal the existing
    entry point's, and a repeated call on buffers the caller already holds
    leaves the device's free memory unchanged."""
    import torch

    from galaxy_b200 import _lib, scenarios
    from galaxy_b200.nbody_gpu import NbodyGpu, bodies_to_state
    lib = _lib.load()
    n = 4_194_304
    recs = bodies_to_state(scenarios.binary_encounter(n, 13))
    d_state = _device_records(torch, recs)
    d_sums = torch.full((9,), float("nan"), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()

    def call():
        _lib.check(lib.galaxy_bh_conservation_noalloc(
            C.c_void_p(d_state.data_ptr()), None, n, C.c_void_p(d_sums.data_ptr()),
            C.c_void_p(stream.cuda_stream)))
        stream.synchronize()
        return d_sums.cpu().numpy()

    first = call()
    # on a stream of the caller's own, too
    side = torch.cuda.Stream()
    d_side = torch.full((9,), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()  # the side stream is not ordered after the fill
    _lib.check(lib.galaxy_bh_conservation_noalloc(
        C.c_void_p(d_state.data_ptr()), None, n, C.c_void_p(d_side.data_ptr()),
        C.c_void_p(side.cuda_stream)))
    side.synchronize()
    assert np.array_equal(d_side.cpu().numpy(), first)
    free_before, _ = torch.cuda.mem_get_info()
    second = call()
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after == free_before
    assert np.array_equal(first, second)
    _compare(second, _existing(NbodyGpu("0"), recs))
