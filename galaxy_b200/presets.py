"""The reference's initial conditions for its BH binaries (`--preset disc` and
`--preset collision`): the seeded XorShift64 Gaussian-profile discs of
nbody/src/lib.rs:430-528, restated in IEEE double arithmetic (Python floats
and the platform libm, as the Rust code uses), so the bodies equal the
reference's bit for bit.  Used by the receipt producer (`receipt.py`).
"""
from __future__ import annotations

import math

import numpy as np

G_KPC3_PER_MSUN_MYR2 = 4.498502151575286e-12  # nbody/src/lib.rs:6
DEFAULT_SOFTENING_KPC = 0.05                  # nbody/src/lib.rs:8
_MASK64 = (1 << 64) - 1


class XorShift64:
    """nbody/src/lib.rs:435-451 (seed 0 becomes 1)."""

    def __init__(self, seed: int):
        self.state = (seed & _MASK64) or 1

    def next_u64(self) -> int:
        x = self.state
        x ^= (x << 13) & _MASK64
        x ^= x >> 7
        x ^= (x << 17) & _MASK64
        self.state = x
        return x

    def unit(self) -> float:
        return float(self.next_u64() >> 11) / float(1 << 53)


def _disc_body(rng: XorShift64, per_body_mass, total_mass, scale_kpc, cx, cy, cvx, cvy,
               direction, spin, softening_kpc):
    """nbody/src/lib.rs:454-483: r = h sqrt(-ln u), uniform angle, circular
    speed from the enclosed mass of that profile, softened."""
    u = max(1.0 - rng.unit(), 1e-15)
    r = scale_kpc * math.sqrt(-math.log(u))
    angle = math.tau * rng.unit()
    x = cx + r * math.cos(angle)
    y = cy + r * math.sin(angle)
    q = max(r / scale_kpc, 0.0)
    enclosed = min(max(1.0 - math.exp(-q) * (1.0 + q), 0.0), 1.0)
    softened_r = max(math.sqrt(r * r + softening_kpc * softening_kpc), 1e-9)
    circular = math.sqrt(G_KPC3_PER_MSUN_MYR2 * total_mass * enclosed / softened_r)
    vx = cvx - direction * spin * circular * math.sin(angle)
    vy = cvy + direction * spin * circular * math.cos(angle)
    return (x, y, vx, vy, per_body_mass)


def make_disc(count: int, seed: int, total_mass: float = 5.0e10, scale: float = 3.0) -> np.ndarray:
    """nbody/src/lib.rs:485-502; (count, 5) f64 rows x, y, vx, vy, mass."""
    if not 2 <= count <= 1_000_000:
        raise ValueError("particle count must be in 2..=1000000")
    if not (math.isfinite(total_mass) and total_mass > 0 and math.isfinite(scale) and scale > 0):
        raise ValueError("disc mass and scale must be positive and finite")
    rng = XorShift64(seed)
    per = total_mass / count
    return np.array([_disc_body(rng, per, total_mass, scale, 0.0, 0.0, 0.0, 0.0, 1.0, 0.88,
                                DEFAULT_SOFTENING_KPC) for _ in range(count)], dtype=np.float64)


def make_collision(count: int, seed: int) -> np.ndarray:
    """nbody/src/lib.rs:504-528: two counter-moving discs."""
    if not 4 <= count <= 1_000_000:
        raise ValueError("collision particle count must be in 4..=1000000")
    left = count // 2
    right = count - left
    half_mass = 5.0e10 * 0.5
    a = XorShift64(seed)
    b = XorShift64((seed + 1) & _MASK64)
    rows = [_disc_body(a, half_mass / left, half_mass, 3.0, -7.5, -1.2, 0.030, 0.010, 1.0, 0.86,
                       DEFAULT_SOFTENING_KPC) for _ in range(left)]
    rows += [_disc_body(b, half_mass / right, half_mass, 2.7, 7.5, 1.2, -0.030, -0.010, -1.0, 0.86,
                        DEFAULT_SOFTENING_KPC) for _ in range(right)]
    return np.array(rows, dtype=np.float64)


def make(preset: str, count: int, seed: int) -> np.ndarray:
    if preset == "disc":
        return make_disc(count, seed, 5.0e10, 3.0)
    if preset == "collision":
        return make_collision(count, seed)
    raise ValueError("--preset must be disc or collision")
