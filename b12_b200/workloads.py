"""Synthetic workload generators for the configured benchmarks (seeded, reproducible).

SplitMix64 (Steele, Lea, Flood, "Fast splittable pseudorandom number generators",
OOPSLA 2014; the 64-bit finaliser constants of Vigna's splitmix64) drives every draw:
u = (x >> 11) * 2^-53.
"""
from __future__ import annotations

import math

MASK = (1 << 64) - 1

LORENZ_CENTER = (0.0, 0.0, 27.0)
LORENZ_RADIUS = (30.0, 30.0, 40.0)
HENON_CENTER = (0.0, 0.0)
HENON_RADIUS = (1.5, 0.45)
FORCED_CENTER = (0.0, 0.0)
FORCED_RADIUS = (2.0, 2.0)


class SplitMix64:
    def __init__(self, seed: int):
        self.x = seed & MASK

    def next_u64(self) -> int:
        self.x = (self.x + 0x9E3779B97F4A7C15) & MASK
        z = self.x
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK
        return z ^ (z >> 31)

    def uniform(self) -> float:
        return (self.next_u64() >> 11) * (1.0 / (1 << 53))


def lorenz_scan(n: int = 512, seed: int = 0):
    """n instances: rho = 15 + 20 u, depth = 18 + floor(10 u'), drawn (rho0, depth0, rho1, ...)."""
    g = SplitMix64(seed)
    rho, depth = [], []
    for _ in range(n):
        rho.append(15.0 + 20.0 * g.uniform())
        depth.append(18 + int(math.floor(10.0 * g.uniform())))
    return rho, depth


def job_stream(n_jobs: int, rate: float, seed: int):
    """Served-stream jobs: Poisson arrivals (exponential gaps -ln(1-u)/rate) and one of
    three families chosen uniformly: Henon (a ~ U[1.0,1.4], b = 0.3, depth 14-22),
    Lorenz (rho ~ U[15,35], depth 18-27), forced Duffing (depth 16-22)."""
    g = SplitMix64(seed)
    t = 0.0
    jobs = []
    for j in range(n_jobs):
        t += -math.log(1.0 - g.uniform()) / rate
        fam = min(2, int(3.0 * g.uniform()))
        if fam == 0:
            a = 1.0 + 0.4 * g.uniform()
            d = 14 + min(8, int(9.0 * g.uniform()))
            jobs.append(dict(id=j, arrival=t, family="henon", params=(a, 0.3), depth=d))
        elif fam == 1:
            rho = 15.0 + 20.0 * g.uniform()
            d = 18 + min(9, int(10.0 * g.uniform()))
            jobs.append(dict(id=j, arrival=t, family="lorenz", params=(10.0, rho, 8.0 / 3.0), depth=d))
        else:
            d = 16 + min(6, int(7.0 * g.uniform()))
            jobs.append(dict(id=j, arrival=t, family="forced_duffing", params=(0.25, -1.0, 1.0, 0.3), depth=d))
    return jobs
