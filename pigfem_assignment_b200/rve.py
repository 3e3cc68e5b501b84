"""RVE descriptions and seeded synthetic inclusion sets.

An RVE is what the reference's driver builds from an inclusion CSV
(PIGFEM4.6.1/Tests/Main.cpp read_csv/add_circle :565-806) plus the mesh
generator call and materials: a rectangular domain meshed with a structured
TRI3 grid, circular inclusions with their own linear elastic material, an
optional cohesive law on every inclusion interface, and the displacement-
driven uniaxial load of Main.cpp:444-450.

Synthetic inclusion sets use random sequential addition (RSA) driven by a
splitmix64 stream seeded per RVE, so every configuration is reproducible
from its seed alone.
"""
from __future__ import annotations

import dataclasses
import math
from typing import List, Sequence, Tuple

import numpy as np

# Cohesive laws (include/pigfem_b200.h)
COH_OP = 0
COH_BILINEAR = 1

MATRIX_E = 3000.0       # MPa (3.0 GPa)
MATRIX_NU = 0.35
INCLUSION_E = 70000.0   # MPa (70 GPa)
INCLUSION_NU = 0.2


@dataclasses.dataclass
class RVE:
    nx: int
    ny: int
    x0: float = 0.0
    x1: float = 1.0
    y0: float = 0.0
    y1: float = 1.0
    inclusions: List[Tuple[float, float, float, int]] = dataclasses.field(default_factory=list)  # cx, cy, r, mat
    materials: List[Tuple[float, float]] = dataclasses.field(
        default_factory=lambda: [(MATRIX_E, MATRIX_NU), (INCLUSION_E, INCLUSION_NU)])
    matrix_mat: int = 0
    cohesive: bool = False
    coh_law: int = COH_OP
    coh_params: Tuple[float, ...] = (0.0, 0.0, 0.0, 0.0, 0.0)
    strain: float = 0.01
    plane_strain: bool = True
    seed: int = -1

    @property
    def n_elements(self) -> int:
        return 2 * self.nx * self.ny


class SplitMix64:
    """splitmix64 (Steele, Lea, Flood 2014): x += 0x9E3779B97F4A7C15, then two
    xor-shift-multiply rounds."""

    MASK = (1 << 64) - 1

    def __init__(self, seed: int):
        self.state = seed & self.MASK

    def next_u64(self) -> int:
        self.state = (self.state + 0x9E3779B97F4A7C15) & self.MASK
        z = self.state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & self.MASK
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & self.MASK
        return z ^ (z >> 31)

    def uniform(self, lo: float = 0.0, hi: float = 1.0) -> float:
        return lo + (hi - lo) * ((self.next_u64() >> 11) * (1.0 / (1 << 53)))

    def randint(self, lo: int, hi: int) -> int:
        """uniform integer in [lo, hi]"""
        return lo + int(self.uniform() * (hi - lo + 1))


def rsa_circles(seed: int, n: int, rmin: float, rmax: float, gap: float, domain=(0.0, 1.0, 0.0, 1.0),
                margin: float | None = None, max_tries: int = 200000) -> List[Tuple[float, float, float]]:
    """Random sequential addition of ``n`` non-overlapping circles with radii
    uniform in [rmin, rmax] and pairwise surface gap >= ``gap``, strictly
    inside the domain (at least ``margin`` from every edge; default ``gap``)."""
    rng = SplitMix64(seed)
    x0, x1, y0, y1 = domain
    margin = gap if margin is None else margin
    out: List[Tuple[float, float, float]] = []
    # bucket grid for neighbour queries
    cell = 2 * rmax + gap
    grid: dict = {}
    tries = 0
    while len(out) < n:
        tries += 1
        if tries > max_tries:
            raise RuntimeError(f"RSA could not place {n} circles (placed {len(out)})")
        r = rng.uniform(rmin, rmax)
        cx = rng.uniform(x0 + r + margin, x1 - r - margin)
        cy = rng.uniform(y0 + r + margin, y1 - r - margin)
        gi, gj = int(cx // cell), int(cy // cell)
        ok = True
        for di in (-1, 0, 1):
            for dj in (-1, 0, 1):
                for (ox, oy, orr) in grid.get((gi + di, gj + dj), ()):
                    if math.hypot(cx - ox, cy - oy) < r + orr + gap:
                        ok = False
                        break
                if not ok:
                    break
            if not ok:
                break
        if ok:
            out.append((cx, cy, r))
            grid.setdefault((gi, gj), []).append((cx, cy, r))
    return out


# ---------------------------------------------------------------------------
# The benchmark configurations (seeded synthetic stand-ins)
# ---------------------------------------------------------------------------

def config0() -> RVE:
    """Unit square, one centred circle r=0.25, 64x64 background mesh (8,192
    TRI3), matrix 3.0 GPa/0.35, inclusion 70 GPa/0.2, perfect bonding, 1%
    uniaxial strain."""
    return RVE(nx=64, ny=64, inclusions=[(0.5, 0.5, 0.25, 1)], strain=0.01)


def config1(seed: int = 1) -> RVE:
    """512x512 mesh (524,288 TRI3), 100 seeded RSA circles, r ~ U[0.02,0.04],
    minimum gap 0.005, same materials and 1% strain."""
    circ = rsa_circles(seed, 100, 0.02, 0.04, 0.005)
    return RVE(nx=512, ny=512, inclusions=[(x, y, r, 1) for (x, y, r) in circ], strain=0.01, seed=seed)


# cohesive parameters: bilinear law sigma_c = 30 MPa, G_c = 10 J/m^2 = 0.01 N/mm,
# K_p = 1e6 MPa/mm
BILINEAR_PARAMS = (30.0, 0.01, 1.0e6, 1.0)


def config2(seed: int = 2, nx: int = 256, n_inc: int = 40) -> RVE:
    """256x256 mesh (131,072 TRI3), 40 seeded circles r ~ U[0.03,0.06],
    bilinear cohesive interfaces, 2% strain reached in 50 equal load steps."""
    circ = rsa_circles(seed, n_inc, 0.03, 0.06, 0.01)
    return RVE(nx=nx, ny=nx, inclusions=[(x, y, r, 1) for (x, y, r) in circ], cohesive=True,
               coh_law=COH_BILINEAR, coh_params=BILINEAR_PARAMS, strain=0.02, seed=seed)


def config3_rves(seed: int = 3, count: int = 512) -> List[RVE]:
    """Batched uneven workload: each RVE has a side in {64,96,128,192,256},
    1..64 circles r ~ U[0.02,0.08] by RSA, inclusion E ~ U[20,100] GPa."""
    rng = SplitMix64(seed)
    sides = (64, 96, 128, 192, 256)
    out = []
    for k in range(count):
        side = sides[rng.randint(0, 4)]
        n_inc = rng.randint(1, 64)
        E_inc = rng.uniform(20000.0, 100000.0)
        sub = rng.next_u64()
        h = 1.0 / side
        gap = max(0.005, 3.0 * h)
        try:
            circ = rsa_circles(sub, n_inc, 0.02, 0.08, gap, max_tries=20000)
        except RuntimeError:
            circ = rsa_circles(sub, max(1, n_inc // 2), 0.02, 0.08, gap, max_tries=200000)
        out.append(RVE(nx=side, ny=side, inclusions=[(x, y, r, 1) for (x, y, r) in circ],
                       materials=[(MATRIX_E, MATRIX_NU), (E_inc, INCLUSION_NU)], strain=0.01, seed=sub))
    return out


def config4(seed: int = 4) -> RVE:
    """1024x1024 mesh (~2.1M TRI3), 400 seeded circles r ~ U[0.01,0.02],
    bilinear cohesive interfaces, 1% strain in 20 load steps."""
    circ = rsa_circles(seed, 400, 0.01, 0.02, 0.005)
    return RVE(nx=1024, ny=1024, inclusions=[(x, y, r, 1) for (x, y, r) in circ], cohesive=True,
               coh_law=COH_BILINEAR, coh_params=BILINEAR_PARAMS, strain=0.01, seed=seed)


def scaled(rve: RVE, nx: int, ny: int | None = None) -> RVE:
    """Same inclusions and materials on a different background mesh."""
    r = dataclasses.replace(rve)
    r.nx = nx
    r.ny = nx if ny is None else ny
    return r
