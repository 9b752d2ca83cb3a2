"""Serving loop logic on the CPU with a fake engine (admission against the
memory budget, FIFO order, rounds, completion accounting), and on the GPU:
every served result equals the same request run alone through the plain
path, bit for bit, while other requests join and leave around it."""
import numpy as np
import pytest

from galaxy_b200.serve import EngineOps, Request, Server, poisson_requests


class FakeClock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        return self.t

    def sleep(self, dt):
        self.t += max(dt, 1e-4)


class FakeOps(EngineOps):
    """Each body costs 100 bytes; a step costs 1 ns per body."""

    def __init__(self, clock):
        self.clock = clock
        self.live = {}
        self.peak_bytes = 0
        self.admit_order = []
        self.steps_done = {}

    def footprint(self, counts):
        return 100 * sum(counts)

    def create(self, req):
        self.live[req.rid] = req.n
        self.admit_order.append(req.rid)
        self.peak_bytes = max(self.peak_bytes, self.footprint(list(self.live.values())))
        self.steps_done[req.rid] = 0
        return req.rid

    def make_batch(self, handles):
        return list(handles)

    def solve(self, batch):
        pass

    def step(self, batch, dts, steps):
        for h in batch:
            self.steps_done[h] += steps
        self.clock.t += 1e-9 * steps * sum(self.live[h] for h in batch)

    def result(self, handle):
        return self.steps_done[handle]

    def release(self, handle):
        del self.live[handle]

    def release_batch(self, batch):
        pass


def test_poisson_requests_distribution():
    reqs = poisson_requests(200.0, 5.0, seed=3)
    assert 800 < len(reqs) < 1200
    ns = np.array([r.n for r in reqs])
    steps = np.array([r.steps for r in reqs])
    assert ns.min() >= 2 ** 12 and ns.max() <= 2 ** 22
    assert steps.min() >= 10 and steps.max() <= 1000
    arr = np.array([r.arrival for r in reqs])
    assert (np.diff(arr) > 0).all() and arr[-1] < 5.0
    # log-uniform: median near the geometric mean
    assert 2 ** 16 < np.median(ns) < 2 ** 18


def test_server_admits_within_budget_and_completes_everything():
    clock = FakeClock()
    ops = FakeOps(clock)
    reqs = [Request(i, "cold_disc", n, i, s, arr) for i, (n, s, arr) in enumerate(
        [(1000, 30, 0.0), (5000, 10, 0.0), (3000, 25, 1e-6), (8000, 40, 2e-6), (500, 5, 5e-5)])]
    budget = 100 * 9500  # never all at once
    srv = Server(ops, budget, round_steps=8, keep_results=True, clock=clock, sleep=clock.sleep)
    out = srv.run(reqs)
    assert out["completed"] == len(reqs)
    assert ops.peak_bytes <= budget
    assert ops.admit_order == sorted(ops.admit_order)  # FIFO admission
    for r in reqs:
        assert r.result == r.steps  # every request got exactly its steps
        assert r.finished >= r.admitted >= r.arrival
    assert out["p99_s"] >= out["p50_s"] > 0
    assert out["particle_steps"] == sum(r.n * r.steps for r in reqs)


def test_server_rejects_request_larger_than_budget():
    clock = FakeClock()
    srv = Server(FakeOps(clock), 100 * 10, clock=clock, sleep=clock.sleep)
    with pytest.raises(ValueError, match="exceeds the budget"):
        srv.run([Request(0, "cold_disc", 100, 1, 10, 0.0)])


def test_server_deadline_stops_early():
    clock = FakeClock()
    ops = FakeOps(clock)
    reqs = [Request(i, "cold_disc", 10 ** 6, i, 1000, 0.0) for i in range(3)]
    srv = Server(ops, 10 ** 12, round_steps=10, clock=clock, sleep=clock.sleep)
    out = srv.run(reqs, deadline=0.05)
    assert out["completed"] < 3


@pytest.mark.gpu
def test_served_results_equal_alone():
    from galaxy_b200 import scenarios
    from galaxy_b200.nbody_gpu import Config, NbodyGpu, ParallelTreeRuntime
    from galaxy_b200.serve import GpuEngineOps

    gpu = NbodyGpu("0")
    cfg = Config(theta=0.5, softening_kpc=0.01, g=1.0, bucket=1)

    def bodies(r):
        return scenarios.make(r.scenario, r.n, r.seed, eps=0.01)

    ops = GpuEngineOps(gpu, cfg, bodies)
    clock = FakeClock()

    class Timed(GpuEngineOps):
        def step(self, batch, dts, steps):
            super().step(batch, dts, steps)
            clock.t += 1e-3 * steps

    ops = Timed(gpu, cfg, bodies)
    reqs = [Request(0, "exponential_disc", 20000, 3, 23, 0.0),
            Request(1, "cold_disc", 5000, 4, 7, 0.0),
            Request(2, "binary_encounter", 12000, 5, 15, 0.005),
            Request(3, "cold_disc", 3000, 6, 40, 0.012)]
    srv = Server(ops, 1 << 40, round_steps=4, keep_results=True, clock=clock, sleep=clock.sleep)
    out = srv.run(reqs)
    assert out["completed"] == 4 and srv.rounds > 4
    rt = ParallelTreeRuntime(gpu)
    for r in reqs:
        ev, _ = gpu.create_evolving_state(bodies(r))
        tree = rt.create_tree(gpu, ev, cfg)
        rt.rebuild(gpu, ev, tree, cfg)
        rt.force(gpu, ev, tree, cfg)
        rt.step(gpu, ev, tree, cfg, r.dt, r.steps)
        alone = gpu.read_evolving_state_records(ev)[0]
        assert alone.tobytes() == r.result.tobytes(), f"request {r.rid}"


def test_native_server_needs_a_device_and_a_config():
    import ctypes as C

    from galaxy_b200 import _lib, build
    build.build()
    lib = _lib.load()
    h = C.c_void_p()
    bad = _lib.BhServeConfig(0, 16, 8)
    assert lib.galaxy_bh_serve_start(0, C.byref(bad), C.byref(h)) != _lib.BH_OK
    if not _gpu_available():
        good = _lib.BhServeConfig(1 << 30, 16, 8)
        assert lib.galaxy_bh_serve_start(0, C.byref(good), C.byref(h)) == _lib.BH_NO_DEVICE


def _gpu_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.gpu
def test_native_server_results_equal_alone():
    """Requests of uneven size, configs and step counts, submitted while others
    run, finish bit-identical to the same simulations stepped alone; one that
    can never fit the budget fails on its own."""
    import time

    from galaxy_b200 import _lib, scenarios
    from galaxy_b200.batch import footprint_bytes
    from galaxy_b200.nbody_gpu import Config, NbodyGpu, ParallelTreeRuntime, bodies_to_state
    from galaxy_b200.serve import NativeServer

    plan = [("exponential_disc", 20000, 3, 23, Config(theta=0.5, softening_kpc=0.01, g=1.0)),
            ("cold_disc", 5000, 4, 7, Config(theta=0.7, softening_kpc=0.01, g=1.0, bucket=4)),
            ("binary_encounter", 12000, 5, 15, Config(theta=0.3, softening_kpc=0.005, g=1.0)),
            ("cold_disc", 3000, 6, 40, Config(theta=0.5, softening_kpc=0.01, g=1.0,
                                              compensated=True))]
    budget = footprint_bytes([20000, 5000, 12000], [p[4] for p in plan[:3]])
    srv = NativeServer(0, budget_bytes=budget, round_steps=4)
    try:
        ids = {}
        for k, (name, n, seed, steps, cfg) in enumerate(plan):
            rec = bodies_to_state(scenarios.make(name, n, seed, eps=0.01))
            ids[srv.submit(rec, cfg, 1e-3, steps)] = k
            time.sleep(0.01)
        too_big = srv.submit(bodies_to_state(scenarios.make("cold_disc", 400000, 9)),
                             plan[0][4], 1e-3, 2)
        results, failed = {}, {}
        while len(results) + len(failed) < len(plan) + 1:
            got = srv.poll(timeout_s=30.0)
            assert got is not None, "server stalled"
            info, rec = got
            if info["status"] == _lib.BH_OK:
                results[ids[info["request_id"]]] = rec
            else:
                failed[info["request_id"]] = info["status"]
        assert failed == {too_big: _lib.BH_CAPACITY_OVERFLOW}
        st = srv.stats()
        assert st["completed"] == len(plan) and st["rounds"] >= 10
    finally:
        srv.stop()
    gpu = NbodyGpu("0")
    rt = ParallelTreeRuntime(gpu)
    for k, (name, n, seed, steps, cfg) in enumerate(plan):
        ev, _ = gpu.create_evolving_state_records(bodies_to_state(scenarios.make(name, n, seed,
                                                                                 eps=0.01)))
        tree = rt.create_tree(gpu, ev, cfg)
        rt.rebuild(gpu, ev, tree, cfg)
        rt.force(gpu, ev, tree, cfg)
        rt.step(gpu, ev, tree, cfg, 1e-3, steps)
        alone, _ = gpu.read_evolving_state_records(ev)
        assert np.array_equal(alone.view(np.uint32), results[k].view(np.uint32)), name


@pytest.mark.gpu
def test_native_server_stop_releases_a_waiting_poll():
    """stop ends the loop while a request is still stepping and a poll is
    waiting in another thread: the poll returns "server stopped", stop
    returns, and nothing waits for the dropped request."""
    import threading
    import time

    from galaxy_b200 import _lib, scenarios
    from galaxy_b200._lib import EngineError
    from galaxy_b200.nbody_gpu import Config, bodies_to_state
    from galaxy_b200.serve import NativeServer

    srv = NativeServer(0, budget_bytes=8 << 30, round_steps=2)
    srv.submit(bodies_to_state(scenarios.make("cold_disc", 200000, 3)),
               Config(theta=0.5, softening_kpc=0.01, g=1.0), 1e-3, 100000)
    out = {}

    def waiter():
        try:
            out["result"] = srv.poll(timeout_s=60.0)
        except EngineError as e:
            out["error"] = e

    th = threading.Thread(target=waiter)
    th.start()
    time.sleep(0.5)
    t0 = time.perf_counter()
    srv.stop()
    th.join(timeout=20.0)
    assert not th.is_alive()
    assert time.perf_counter() - t0 < 20.0
    assert "error" in out, out
    assert out["error"].status == _lib.BH_INVALID_ARG and "stopped" in out["error"].message
