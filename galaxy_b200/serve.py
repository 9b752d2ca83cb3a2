"""Serving loop: continuous batching of simulation requests on one GPU.

Requests (a scenario, N, seed, step count) arrive over time.  The loop admits
waiting requests, in arrival order, as soon as the device-memory footprint of
the active set plus the newcomer fits the budget; keeps every admitted
simulation's particles resident; and advances all active simulations
together in rounds of fused KDK steps through one batch (one launch per
stage for all of them).  A round stops at the smallest remaining step count,
so finished simulations leave and waiting ones join between rounds; their
work overlaps on the device with the simulations already running.  A
simulation's result does not depend on who it shared rounds with: the
per-simulation arithmetic of a batch is that of the plain path.

The engine is injected (``EngineOps``) so that admission and scheduling can
be exercised without a GPU.
"""
from __future__ import annotations

import atexit
import time
from collections import deque
from dataclasses import dataclass, field
from typing import Callable, Optional

import numpy as np


@dataclass
class Request:
    rid: int
    scenario: str
    n: int
    seed: int
    steps: int
    arrival: float          # seconds after the start of the run
    dt: float = 1e-3
    bodies: object = field(default=None, repr=False)  # initial conditions, when supplied
    admitted: Optional[float] = None
    finished: Optional[float] = None
    result: object = None   # final GpuEvolveState records (when keep_results)
    remaining: int = field(default=0, repr=False)

    @property
    def latency(self) -> Optional[float]:
        return None if self.finished is None else self.finished - self.arrival


class EngineOps:
    """What the loop needs from the engine.  The GPU implementation is
    ``GpuEngineOps``; tests use a fake."""

    def footprint(self, counts: list[int]) -> int:
        raise NotImplementedError

    def create(self, req: Request):
        raise NotImplementedError

    def make_batch(self, handles: list):
        raise NotImplementedError

    def solve(self, batch) -> None:
        raise NotImplementedError

    def step(self, batch, dts: list[float], steps: int) -> None:
        raise NotImplementedError

    def result(self, handle):
        raise NotImplementedError

    def release(self, handle) -> None:
        raise NotImplementedError

    def release_batch(self, batch) -> None:
        raise NotImplementedError


def poisson_requests(rate: float, duration: float, seed: int = 5, n_lo: int = 12,
                     n_hi: int = 22, steps_lo: int = 10, steps_hi: int = 1000,
                     scenarios=("exponential_disc", "cold_disc", "binary_encounter"),
                     dt: float = 1e-3) -> list[Request]:
    """Poisson arrivals at `rate` per second over `duration` seconds; N
    log-uniform in [2^n_lo, 2^n_hi], steps log-uniform in [steps_lo,
    steps_hi], scenario uniform."""
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= duration:
            break
        n = int(np.exp(rng.uniform(n_lo * np.log(2), n_hi * np.log(2))))
        steps = int(round(np.exp(rng.uniform(np.log(steps_lo), np.log(steps_hi)))))
        out.append(Request(len(out), scenarios[int(rng.integers(0, len(scenarios)))],
                           max(n, 4), int(rng.integers(1, 2 ** 31 - 1)), steps, t, dt))
    return out


class Server:
    """Continuous-batching loop over an ``EngineOps``."""

    def __init__(self, ops: EngineOps, budget_bytes: int, round_steps: int = 16,
                 max_members: int = 4096, keep_results: bool = False,
                 clock: Callable[[], float] = time.perf_counter,
                 sleep: Callable[[float], None] = time.sleep):
        self.ops = ops
        self.budget = budget_bytes
        self.round_steps = round_steps
        self.max_members = max_members
        self.keep_results = keep_results
        self.clock = clock
        self.sleep = sleep
        self.rounds = 0
        self.particle_steps = 0

    def run(self, requests: list[Request], deadline: float = float("inf")) -> dict:
        pending = deque(sorted(requests, key=lambda r: r.arrival))
        waiting: deque[Request] = deque()
        active: list[tuple[Request, object]] = []
        batch = None
        t0 = self.clock()
        busy = 0.0
        while pending or waiting or active:
            now = self.clock() - t0
            if now > deadline:
                break
            while pending and pending[0].arrival <= now:
                waiting.append(pending.popleft())
            # admission in arrival order against the device-memory budget
            joined = []
            while waiting and len(active) + len(joined) < self.max_members:
                cand = waiting[0]
                counts = [r.n for r, _ in active] + [r.n for r, _ in joined] + [cand.n]
                if self.ops.footprint(counts) > self.budget:
                    if not active and not joined:
                        raise ValueError(f"request {cand.rid} (N={cand.n}) exceeds the budget")
                    break
                waiting.popleft()
                cand.admitted = self.clock() - t0
                cand.remaining = cand.steps
                joined.append((cand, self.ops.create(cand)))
            if joined:
                active.extend(joined)
                if batch is not None:
                    self.ops.release_batch(batch)
                batch = self.ops.make_batch([h for _, h in active])
                self.ops.solve(batch)
            if not active:
                if pending:
                    self.sleep(max(0.0, min(pending[0].arrival - (self.clock() - t0), 0.05)))
                continue
            r_steps = min(self.round_steps, min(r.remaining for r, _ in active))
            tb = self.clock()
            self.ops.step(batch, [r.dt for r, _ in active], r_steps)
            busy += self.clock() - tb
            self.rounds += 1
            self.particle_steps += r_steps * sum(r.n for r, _ in active)
            done_now = self.clock() - t0
            still = []
            for r, h in active:
                r.remaining -= r_steps
                if r.remaining == 0:
                    if self.keep_results:
                        r.result = self.ops.result(h)
                    r.finished = done_now
                    self.ops.release(h)
                else:
                    still.append((r, h))
            if len(still) != len(active):
                self.ops.release_batch(batch)
                batch = self.ops.make_batch([h for _, h in still]) if still else None
            active = still
        if batch is not None:
            self.ops.release_batch(batch)
        wall = self.clock() - t0
        lat = np.array([r.latency for r in requests if r.latency is not None])
        return {"requests": len(requests), "completed": int(len(lat)),
                "p50_s": float(np.percentile(lat, 50)) if len(lat) else None,
                "p99_s": float(np.percentile(lat, 99)) if len(lat) else None,
                "wall_s": wall, "busy_s": busy, "rounds": self.rounds,
                "particle_steps": self.particle_steps,
                "particle_steps_per_s": self.particle_steps / wall if wall > 0 else 0.0}


class GpuEngineOps(EngineOps):
    """EngineOps over the CUDA engine: states are resident EvolvingStates,
    a batch is a galaxy_b200.batch.Batch."""

    def __init__(self, gpu, config, make_bodies: Callable[[Request], np.ndarray]):
        from .batch import footprint_bytes
        self.gpu = gpu
        self.config = config
        self.make_bodies = make_bodies
        self._footprint = footprint_bytes

    def footprint(self, counts):
        return self._footprint(counts, [self.config] * len(counts))

    def create(self, req):
        from .nbody_gpu import bodies_to_state
        b = req.bodies if req.bodies is not None else self.make_bodies(req)
        st, _ = self.gpu.create_evolving_state_records(bodies_to_state(b))
        return st

    def make_batch(self, handles):
        from .batch import Batch
        return Batch(self.gpu, handles, [self.config] * len(handles))

    def solve(self, batch):
        batch.solve()

    def step(self, batch, dts, steps):
        batch.step(dts, steps)

    def result(self, handle):
        return self.gpu.read_evolving_state_records(handle)[0]

    def release(self, handle):
        handle.close()

    def release_batch(self, batch):
        batch.close()


class NativeServer:
    """The serving loop of the C ABI (galaxy_bh_serve_*): its own host
    thread and device handle; submit from here, poll for results."""

    def __init__(self, ordinal: int = 0, budget_bytes: int = 150 << 30, round_steps: int = 16,
                 max_members: int = 4096):
        import ctypes as C

        from . import _lib
        self._C, self._lib = C, _lib
        cfg = _lib.BhServeConfig(int(budget_bytes), int(round_steps), int(max_members))
        self._h = C.c_void_p()
        _lib.check(_lib.load().galaxy_bh_serve_start(int(ordinal), C.byref(cfg),
                                                     C.byref(self._h)))
        self._max_n = 0
        _LIVE_SERVERS.add(self)

    def submit(self, records: np.ndarray, config, dt: float, steps: int) -> int:
        """Queues a simulation (GpuEvolveState records); returns its id."""
        C, _lib = self._C, self._lib
        rec = np.ascontiguousarray(records, dtype=_lib.EVOLVE_STATE_DTYPE)
        self._max_n = max(self._max_n, len(rec))  # before the server can finish it
        rid = C.c_uint64()
        _lib.check(_lib.load().galaxy_bh_serve_submit(self._h, _lib.ptr(rec), len(rec),
                                                      C.byref(config.to_c()), float(dt),
                                                      int(steps), C.byref(rid)))
        return rid.value

    def poll(self, timeout_s: float = 0.0):
        """(result info dict, final records) of the next finished request, or
        None when none finishes within the timeout."""
        C, _lib = self._C, self._lib
        res = _lib.BhServeResult()
        cap = self._max_n
        out = np.empty(max(cap, 1), _lib.EVOLVE_STATE_DTYPE)
        rc = _lib.load().galaxy_bh_serve_poll(self._h, int(timeout_s * 1000), C.byref(res),
                                              _lib.ptr(out), cap)
        if rc == _lib.BH_TIMEOUT:
            return None
        if rc == _lib.BH_INVALID_ARG and res.n > cap:  # sized by another submitter
            cap = res.n
            out = np.empty(cap, _lib.EVOLVE_STATE_DTYPE)
            rc = _lib.load().galaxy_bh_serve_poll(self._h, 0, C.byref(res), _lib.ptr(out), cap)
        _lib.check(rc)
        info = {"request_id": res.request_id, "n": res.n, "status": res.status,
                "steps": res.steps, "submitted_s": res.submitted_s,
                "admitted_s": res.admitted_s, "finished_s": res.finished_s}
        return info, (out[:res.n].copy() if res.status == _lib.BH_OK else None)

    def stats(self) -> dict:
        C, _lib = self._C, self._lib
        st = _lib.BhServeStats()
        _lib.check(_lib.load().galaxy_bh_serve_stats(self._h, C.byref(st)))
        return {"rounds": st.rounds, "particle_steps": st.particle_steps,
                "completed": st.completed, "busy_seconds": st.busy_seconds,
                "elapsed_seconds": st.elapsed_seconds, "admit_seconds": st.admit_seconds,
                "solve_seconds": st.solve_seconds, "form_seconds": st.form_seconds,
                "readback_seconds": st.readback_seconds}

    def stop(self) -> None:
        """Ends the loop and joins its thread; always call it (or use the
        server as a context manager) before the process exits."""
        if self._h:
            self._lib.load().galaxy_bh_serve_stop(self._h)
            self._h = self._C.c_void_p()
        _LIVE_SERVERS.discard(self)

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.stop()

    def __del__(self):
        try:
            self.stop()
        except Exception:
            pass


_LIVE_SERVERS: set = set()


def _stop_live_servers():
    for srv in list(_LIVE_SERVERS):
        srv.stop()


atexit.register(_stop_live_servers)
