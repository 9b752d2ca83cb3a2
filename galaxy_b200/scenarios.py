"""Seeded synthetic initial conditions of the engine's benchmark workloads.

All bodies are float64 rows (x, y, vx, vy, mass), G = 1 units:

* ``exponential_disc``  rotating disc, surface density ~ exp(-r) (scale 1,
  truncated at 5), circular speed from the enclosed mass plus an isotropic
  Gaussian dispersion of 0.05 v_c per component;
* ``cold_disc``         uniform unit disc (r = sqrt(u)), zero velocity;
* ``binary_encounter``  two exponential discs (scale 1.0 and 0.7, masses
  1 : 0.5) 8 units apart, relative speed 0.3, approaching off-axis.

They stand in for the workloads' published shapes and distributions; no
external dataset is involved.
"""
from __future__ import annotations

import numpy as np

R_TRUNC = 5.0


def _enclosed_fraction(r: np.ndarray, scale: float) -> np.ndarray:
    """M(<r)/M of an exponential disc truncated at R_TRUNC * scale."""
    q = r / scale
    full = 1.0 - np.exp(-R_TRUNC) * (1.0 + R_TRUNC)
    return (1.0 - np.exp(-q) * (1.0 + q)) / full


def _exp_disc(rng: np.random.Generator, n: int, mass: float, scale: float, eps: float,
              g: float = 1.0) -> np.ndarray:
    # Sigma ~ exp(-r/h): radial mass density ~ r exp(-r/h) -> Gamma(2, h), truncated.
    r = np.empty(0)
    while len(r) < n:
        draw = rng.gamma(2.0, scale, size=2 * (n - len(r)) + 16)
        r = np.concatenate([r, draw[draw <= R_TRUNC * scale]])
    r = r[:n]
    phi = rng.uniform(0.0, 2.0 * np.pi, n)
    x, y = r * np.cos(phi), r * np.sin(phi)
    vc = np.sqrt(g * mass * _enclosed_fraction(r, scale) / np.sqrt(r * r + eps * eps))
    vx = -vc * np.sin(phi) + rng.normal(0.0, 1.0, n) * 0.05 * vc
    vy = vc * np.cos(phi) + rng.normal(0.0, 1.0, n) * 0.05 * vc
    return np.stack([x, y, vx, vy, np.full(n, mass / n)], axis=1)


def exponential_disc(n: int, seed: int = 42, eps: float = 0.01, total_mass: float = 1.0,
                     scale: float = 1.0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return _exp_disc(rng, n, total_mass, scale, eps)


def cold_disc(n: int, seed: int = 7, total_mass: float = 1.0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    r = np.sqrt(rng.uniform(0.0, 1.0, n))
    phi = rng.uniform(0.0, 2.0 * np.pi, n)
    b = np.zeros((n, 5))
    b[:, 0] = r * np.cos(phi)
    b[:, 1] = r * np.sin(phi)
    b[:, 4] = total_mass / n
    return b


def binary_encounter(n: int, seed: int = 11, eps: float = 0.005, separation: float = 8.0,
                     v_rel: float = 0.3, approach_deg: float = 30.0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    na = n // 2
    nb = n - na
    ma, mb = 1.0, 0.5
    a = _exp_disc(rng, na, ma, 1.0, eps)
    b = _exp_disc(rng, nb, mb, 0.7, eps)
    mt = ma + mb
    # centre of mass at rest at the origin; B approaches A off-axis
    ang = np.deg2rad(180.0 - approach_deg)
    rel_v = v_rel * np.array([np.cos(ang), np.sin(ang)])
    a[:, 0] -= separation * mb / mt
    b[:, 0] += separation * ma / mt
    a[:, 2:4] -= rel_v * mb / mt
    b[:, 2:4] += rel_v * ma / mt
    return np.concatenate([a, b], axis=0)


SCENARIOS = {"exponential_disc": exponential_disc, "cold_disc": cold_disc,
             "binary_encounter": binary_encounter}


def make(name: str, n: int, seed: int, eps: float = 0.01) -> np.ndarray:
    if name == "cold_disc":
        return cold_disc(n, seed)
    if name == "exponential_disc":
        return exponential_disc(n, seed, eps)
    if name == "binary_encounter":
        return binary_encounter(n, seed, eps)
    raise ValueError(f"unknown scenario {name!r}")


def mixed_batch(count: int = 512, lo_exp: int = 10, hi_exp: int = 18, seed: int = 2024,
                eps: float = 0.01) -> list[tuple[str, int, int]]:
    """(scenario, n, seed) for the batched workload: n log-uniform in
    [2^lo_exp, 2^hi_exp], scenario uniform over the three."""
    rng = np.random.default_rng(seed)
    names = list(SCENARIOS)
    ns = np.exp(rng.uniform(lo_exp * np.log(2), hi_exp * np.log(2), count)).astype(np.int64)
    picks = rng.integers(0, 3, count)
    seeds = rng.integers(1, 2 ** 31 - 1, count)
    return [(names[p], int(max(n, 4)), int(s)) for p, n, s in zip(picks, ns, seeds)]
