"""Seeded generators of dipolar Ising systems (no counterpart in the reference, which only
loads CSV/XYZ geometry, src/physics.cpp:77-149, or builds a uniform simple-cubic lattice,
src/physics.cpp:58-75).

All randomness comes from xoshiro256** streams seeded exactly like the reference's
Xoshiro256StarStar(seed, stream) (include/wl/rng.hpp), so a (generator, seed) pair names a
system independently of the numpy version.  Systems can be written in the reference's CSV
format (x,y,z,mx,my,mz) with round-trip-exact numbers, so the reference can load the very
same doubles.

* random_sphere_axes   -- unit axes uniform on the sphere (normalised Gaussian triples)
* simple_cubic_random  -- nx x ny x nz lattice with random axes (periodic, slab or open)
* diluted_cubic        -- the same lattice with a seeded fraction of sites removed
* random_sequential    -- random sequential addition in a periodic cube at a target
                          density with a minimum separation
"""
from __future__ import annotations

import math

import numpy as np

from .engine import Geometry

_MASK = (1 << 64) - 1


class Xoshiro:
    """xoshiro256** with splitmix64 seeding (include/wl/rng.hpp:10-56)."""

    def __init__(self, seed: int, stream: int = 0):
        x = (seed ^ ((0xD2B74407B1CE6E93 * (stream + 1)) & _MASK)) & _MASK
        s = []
        for _ in range(4):
            x = (x + 0x9E3779B97F4A7C15) & _MASK
            z = x
            z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _MASK
            z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _MASK
            s.append(z ^ (z >> 31))
        self.s = s

    def next(self) -> int:
        s = self.s
        r = (((((s[1] * 5) & _MASK) << 7) | (((s[1] * 5) & _MASK) >> 57)) & _MASK) * 9 & _MASK
        t = (s[1] << 17) & _MASK
        s[2] ^= s[0]
        s[3] ^= s[1]
        s[1] ^= s[2]
        s[0] ^= s[3]
        s[2] ^= t
        s[3] = ((s[3] << 45) | (s[3] >> 19)) & _MASK
        return r

    def uniform(self) -> float:
        return (self.next() >> 11) * (1.0 / 9007199254740992.0)

    def normal(self) -> float:
        """Box-Muller on two uniforms (the first mapped to (0, 1])."""
        u1 = 1.0 - self.uniform()
        u2 = self.uniform()
        return math.sqrt(-2.0 * math.log(u1)) * math.cos(2.0 * math.pi * u2)


def random_sphere_axes(n: int, seed: int) -> np.ndarray:
    """n unit vectors uniform on the sphere; site i uses stream i of `seed`."""
    out = np.empty((n, 3), dtype=np.float64)
    for i in range(n):
        rng = Xoshiro(seed, i)
        while True:
            g = (rng.normal(), rng.normal(), rng.normal())
            length = math.sqrt(g[0] * g[0] + g[1] * g[1] + g[2] * g[2])
            if length > 1e-12:
                break
        out[i] = (g[0] / length, g[1] / length, g[2] / length)
    return out


def simple_cubic_random(nx: int, ny: int, nz: int, seed: int, periodic: bool = True,
                        box=None, spacing: float = 1.0) -> Geometry:
    """Geometry::simple_cubic with random-sphere axes; box=(Lx, Ly, 0) gives a slab."""
    g = Geometry.simple_cubic(nx, ny, nz, spacing, (0.0, 0.0, 1.0), periodic)
    g.axes = random_sphere_axes(g.size(), seed)
    if box is not None:
        g.box = tuple(float(b) for b in box)
    g.validate()
    return g


def diluted_cubic(nx: int, ny: int, nz: int, fraction_removed: float, seed: int, periodic: bool = True,
                  box=None) -> Geometry:
    """A simple-cubic lattice with round(fraction*N) sites removed (seeded), random axes."""
    full = Geometry.simple_cubic(nx, ny, nz, 1.0, (0.0, 0.0, 1.0), periodic)
    n = full.size()
    remove = int(round(fraction_removed * n))
    rng = Xoshiro(seed, 1 << 32)
    order = list(range(n))
    for i in range(n - 1, 0, -1):  # Fisher-Yates with the reference's bounded() rejection
        bound = i + 1
        threshold = ((1 << 64) - bound) % bound
        while True:
            x = rng.next()
            if x >= threshold:
                break
        j = x % bound
        order[i], order[j] = order[j], order[i]
    keep = np.sort(np.array(order[remove:], dtype=np.int64))
    g = Geometry(full.positions[keep], np.zeros((len(keep), 3)), full.box if box is None else box, periodic)
    g.axes = random_sphere_axes(g.size(), seed)
    g.validate()
    return g


def random_sequential(n: int, density: float, min_separation: float, seed: int,
                      max_tries: int = 1_000_000) -> Geometry:
    """n sites added one by one at uniform random positions in a periodic cube of side
    (n/density)^(1/3), rejecting any closer than min_separation (minimum image)."""
    side = (n / density) ** (1.0 / 3.0)
    rng = Xoshiro(seed, 1 << 33)
    pts = np.empty((n, 3))
    count = 0
    tries = 0
    while count < n:
        tries += 1
        if tries > max_tries:
            raise RuntimeError("random sequential addition did not place every site")
        p = np.array([rng.uniform() * side, rng.uniform() * side, rng.uniform() * side])
        if count:
            d = pts[:count] - p
            d -= side * np.rint(d / side)
            if np.min(np.einsum("ij,ij->i", d, d)) < min_separation * min_separation:
                continue
        pts[count] = p
        count += 1
    g = Geometry(pts, random_sphere_axes(n, seed), (side, side, side), True)
    g.validate()
    return g
