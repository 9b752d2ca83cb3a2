"""Autotuner of the batched and plain engines.

Picks, by timing short runs of the caller's own workload on the device:

* the leaf size (``Config.bucket``, one of 1, 4, 8, 16) per simulation size
  class, so the leaf size is a pure function of N once tuned;
* the sort digit width (8 or 4 bits) and the warps per traversal block
  (4, 8 or 2), launch shapes that change no result bit.

A leaf-size candidate is admitted only if its median force error against FP64
direct sums (probes of the class's largest simulation) is no worse than the
leaf-size-1 error by more than ``max_error_ratio``: larger leaves sum more
bodies directly, so they normally lower the error.  Tuning runs on copies of
the caller's states, which it leaves untouched.
"""
from __future__ import annotations

import dataclasses as dc
from dataclasses import dataclass, field
from typing import Callable, Sequence

import numpy as np

LEAF_SIZES = (1, 4, 8, 16)
RADIX_BITS = (8, 4)
TRAVERSE_WARPS = (4, 8, 2)


def size_class(n: int) -> int:
    """Size class of a simulation: floor(log2 n) rounded down to even (2^10,
    2^12, ... 2^22 bins of two octaves)."""
    return max(0, int(np.log2(max(int(n), 1))) // 2 * 2)


@dataclass
class Tuning:
    leaf_by_class: dict = field(default_factory=dict)  # size class -> bucket
    radix_bits: int = 8
    traverse_warps: int = 4
    trials: list = field(default_factory=list)  # (knob, value, ms per step, accepted)
    errors: dict = field(default_factory=dict)  # "2^class" -> {leaf: median force error}

    def bucket_for(self, n: int, default: int = 1) -> int:
        return int(self.leaf_by_class.get(size_class(n), default))

    def configs(self, counts: Sequence[int], configs) -> list:
        """The per-simulation configs with the tuned leaf sizes."""
        return [dc.replace(c, bucket=self.bucket_for(n, c.bucket)) for n, c in zip(counts, configs)]

    def as_dict(self) -> dict:
        return {"leaf_by_class": {f"2^{k}": v for k, v in sorted(self.leaf_by_class.items())},
                "radix_bits": self.radix_bits, "traverse_warps": self.traverse_warps}


def coordinate_search(start: Tuning, classes: Sequence[int],
                      measure: Callable[[Tuning], float],
                      admissible: Callable[[int, int], bool] = lambda cls, leaf: True) -> Tuning:
    """One pass of coordinate descent over the knobs, each candidate timed by
    ``measure`` (ms per step, lower is better): the leaf size of each size
    class (largest classes first: they carry most of the work), then the
    sort digit width, then the traversal warps.  Pure host logic, so it is
    testable without a GPU."""
    best = dc.replace(start, leaf_by_class=dict(start.leaf_by_class), trials=list(start.trials))
    best_ms = measure(best)
    best.trials.append(("baseline", None, best_ms, True))
    for cls in sorted(classes, reverse=True):
        for leaf in LEAF_SIZES:
            if leaf == best.leaf_by_class.get(cls, 1):
                continue
            ok = admissible(cls, leaf)
            if not ok:
                best.trials.append((f"leaf 2^{cls}", leaf, None, False))
                continue
            cand = dc.replace(best, leaf_by_class={**best.leaf_by_class, cls: leaf})
            ms = measure(cand)
            best.trials.append((f"leaf 2^{cls}", leaf, ms, ms < best_ms))
            if ms < best_ms:
                best, best_ms = dc.replace(cand, trials=best.trials), ms
    for knob, values in (("radix_bits", RADIX_BITS), ("traverse_warps", TRAVERSE_WARPS)):
        for v in values:
            if v == getattr(best, knob):
                continue
            cand = dc.replace(best, **{knob: v})
            ms = measure(cand)
            best.trials.append((knob, v, ms, ms < best_ms))
            if ms < best_ms:
                best, best_ms = dc.replace(cand, trials=best.trials), ms
    best.trials.append(("best", None, best_ms, True))
    return best


def _clone(gpu, states):
    out = []
    for st in states:
        rec, _ = gpu.read_evolving_state_records(st)
        ev, _ = gpu.create_evolving_state_records(rec)
        out.append(ev)
    return out


def tune_batch(gpu, states, configs, dt: float, steps: int = 3, probes: int = 256,
               max_error_ratio: float = 1.05) -> Tuning:
    """Tunes a batch of ``states`` (with their ``configs``) by timing
    ``steps`` fused steps per candidate on copies of the states."""
    import torch

    from .batch import Batch

    counts = [st.count for st in states]
    classes = sorted({size_class(n) for n in counts})
    stream = torch.cuda.ExternalStream(gpu.stream_ptr())
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)

    def measure(t: Tuning) -> float:
        copies = _clone(gpu, states)
        b = Batch(gpu, copies, t.configs(counts, configs))
        try:
            b.tune(t.radix_bits, t.traverse_warps)
            b.solve()
            b.step(dt, 1)
            torch.cuda.synchronize()
            e0.record(stream)
            b.step(dt, steps)
            e1.record(stream)
            torch.cuda.synchronize()
            return e0.elapsed_time(e1) / steps
        finally:
            b.close()
            for c in copies:
                c.close()

    errors: dict = {}

    def class_error(cls: int, leaf: int) -> float:
        if (cls, leaf) not in errors:
            from .nbody_gpu import ParallelTreeRuntime
            i = max((k for k, n in enumerate(counts) if size_class(n) == cls),
                    key=lambda k: counts[k])
            cfg = dc.replace(configs[i], bucket=leaf)
            (ev,) = _clone(gpu, [states[i]])
            rt = ParallelTreeRuntime(gpu)
            tree = rt.create_tree(gpu, ev, cfg)
            try:
                rt.rebuild(gpu, ev, tree, cfg)
                rt.force(gpu, ev, tree, cfg)
                p = np.linspace(0, counts[i] - 1, min(probes, counts[i])).astype(np.uint32)
                errors[(cls, leaf)] = gpu.probe_error(ev, cfg, p)["median"]
            finally:
                tree.close()
                ev.close()
        return errors[(cls, leaf)]

    def admissible(cls: int, leaf: int) -> bool:
        return class_error(cls, leaf) <= max_error_ratio * class_error(cls, 1)

    start = Tuning({c: 1 for c in classes})
    best = coordinate_search(start, classes, measure, admissible)
    for (cls, leaf), e in sorted(errors.items()):
        best.errors.setdefault(f"2^{cls}", {})[leaf] = e
    return best


def tune_tree(gpu, rt, state, tree, config, dt: float, steps: int = 5) -> Tuning:
    """Launch-shape tuning of a plain single-simulation tree (its leaf size is
    the caller's): times ``steps`` steps of a copy of ``state`` per setting
    and installs the fastest on ``tree``."""
    import torch

    stream = torch.cuda.ExternalStream(gpu.stream_ptr())
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)

    def measure(t: Tuning) -> float:
        (ev,) = _clone(gpu, [state])
        tr = rt.create_tree(gpu, ev, config)
        try:
            rt.tune(tr, t.radix_bits, t.traverse_warps)
            rt.rebuild(gpu, ev, tr, config)
            rt.force(gpu, ev, tr, config)
            rt.step(gpu, ev, tr, config, dt, 1)
            torch.cuda.synchronize()
            e0.record(stream)
            rt.step(gpu, ev, tr, config, dt, steps)
            e1.record(stream)
            torch.cuda.synchronize()
            return e0.elapsed_time(e1) / steps
        finally:
            tr.close()
            ev.close()

    best = coordinate_search(Tuning({}), [], measure)
    rt.tune(tree, best.radix_bits, best.traverse_warps)
    return best
