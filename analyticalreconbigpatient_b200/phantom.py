"""Seeded synthetic phantoms (the data source for tests and benchmarks).

The reference ships no data (its GE ``.dat`` inputs are not distributed), so
projections are analytic line integrals through ellipsoid phantoms on the
reference's own helical curved-detector geometry. An object is one row of 17
doubles::

    [type, cx, cy, cz, a, b, c, R00, R01, R02, R10, R11, R12, R20, R21, R22, mu]

``R`` (row-major) has the body axes in world coordinates as its columns.
type 0 is an ellipsoid with semi-axes a, b, c; type 1 is an elliptic cylinder
with in-plane semi-axes a, b and z extent cz +- c. ``mu`` (1/mm) adds where
objects overlap.

Random numbers come from a project-written SplitMix64 generator so that a seed
gives the same phantom on every machine.
"""
from __future__ import annotations

import math

import numpy as np

from .geometry import MU_WATER, Scan

_MASK = (1 << 64) - 1


class SplitMix64:
    """SplitMix64 (Steele, Lea, Flood 2014): 64-bit state, additive Weyl step,
    two xor-shift-multiply mixing rounds."""

    def __init__(self, seed: int):
        self.state = seed & _MASK

    def next_u64(self) -> int:
        self.state = (self.state + 0x9E3779B97F4A7C15) & _MASK
        z = self.state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _MASK
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _MASK
        return z ^ (z >> 31)

    def uniform(self, lo: float = 0.0, hi: float = 1.0) -> float:
        return lo + (hi - lo) * ((self.next_u64() >> 11) * (1.0 / (1 << 53)))

    def rotation(self) -> np.ndarray:
        """Uniform random rotation (Shoemake's unit-quaternion construction)."""
        u1, u2, u3 = self.uniform(), self.uniform(), self.uniform()
        q = (math.sqrt(1 - u1) * math.sin(2 * math.pi * u2), math.sqrt(1 - u1) * math.cos(2 * math.pi * u2),
             math.sqrt(u1) * math.sin(2 * math.pi * u3), math.sqrt(u1) * math.cos(2 * math.pi * u3))
        x, y, z, w = q
        return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                         [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                         [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def _obj(type_, c, axes, R, mu) -> list:
    return [float(type_), *map(float, c), *map(float, axes), *map(float, np.asarray(R).reshape(9)), float(mu)]


def _rz(deg: float) -> np.ndarray:
    a = math.radians(deg)
    return np.array([[math.cos(a), -math.sin(a), 0.0], [math.sin(a), math.cos(a), 0.0], [0.0, 0.0, 1.0]])


# In-plane layout of the Shepp-Logan head (Shepp & Logan 1974): centre (x, y),
# semi-axes (a, b), tilt (deg), additive density in units of water. The z
# semi-axes and centres are this project's own choice for a 3D version.
_SHEPP_LOGAN_2D = [
    (0.0, 0.0, 0.69, 0.92, 0.0, 2.0),
    (0.0, -0.0184, 0.6624, 0.874, 0.0, -0.98),
    (0.22, 0.0, 0.11, 0.31, -18.0, -0.02),
    (-0.22, 0.0, 0.16, 0.41, 18.0, -0.02),
    (0.0, 0.35, 0.21, 0.25, 0.0, 0.01),
    (0.0, 0.1, 0.046, 0.046, 0.0, 0.01),
    (0.0, -0.1, 0.046, 0.046, 0.0, 0.01),
    (-0.08, -0.605, 0.046, 0.023, 0.0, 0.01),
    (0.0, -0.605, 0.023, 0.023, 0.0, 0.01),
    (0.06, -0.605, 0.023, 0.046, 0.0, 0.01),
]
_SHEPP_LOGAN_Z = [(0.0, 0.9), (0.0, 0.88), (0.0, 0.25), (0.0, 0.3), (0.02, 0.2), (0.0, 0.046), (-0.02, 0.046),
                  (0.01, 0.05), (0.0, 0.023), (-0.01, 0.05)]


def shepp_logan(fov: float = 400.0, z_centre: float = 0.0, contrast_scale: float = 1.0) -> np.ndarray:
    """3D Shepp-Logan-style head scaled so that [-1, 1] spans ``fov`` mm; 1.0 in
    the table's density units is water (0.0193/mm)."""
    s = fov / 2.0
    rows = []
    for i, ((x, y, a, b, tilt, rho), (zc, cz)) in enumerate(zip(_SHEPP_LOGAN_2D, _SHEPP_LOGAN_Z)):
        mu = rho * MU_WATER * (1.0 if i < 2 else contrast_scale)
        rows.append(_obj(0, (x * s, y * s, z_centre + zc * s), (a * s, b * s, cz * s), _rz(tilt), mu))
    return np.array(rows)


def water_cylinder(radius: float = 100.0, half_length: float = 2000.0, z_centre: float = 0.0,
                   mu: float = MU_WATER) -> np.ndarray:
    return np.array([_obj(1, (0.0, 0.0, z_centre), (radius, radius, half_length), np.eye(3), mu)])


def random_ellipsoids(seed: int, n: int, z_range: tuple[float, float], body=(180.0, 140.0),
                      semi_axes=(5.0, 120.0), mu_range=(0.010, 0.030), body_half_length: float | None = None,
                      fill: float = 0.85) -> np.ndarray:
    """``n`` seeded random ellipsoids inside an elliptic water cylinder.

    Each ellipsoid has semi-axes uniform in ``semi_axes``, a uniform random
    orientation and an absolute attenuation uniform in ``mu_range``; it is
    stored as the difference to water so that it replaces the cylinder's water
    where it lies. Centres are uniform inside the body ellipse scaled by
    ``fill`` and uniform in z over ``z_range``."""
    rng = SplitMix64(seed)
    zlo, zhi = z_range
    half = body_half_length if body_half_length is not None else 0.5 * (zhi - zlo) + 200.0
    rows = [_obj(1, (0.0, 0.0, 0.5 * (zlo + zhi)), (body[0], body[1], half), np.eye(3), MU_WATER)]
    for _ in range(n):
        while True:
            x, y = rng.uniform(-1, 1), rng.uniform(-1, 1)
            if x * x + y * y <= 1.0:
                break
        c = (x * body[0] * fill, y * body[1] * fill, rng.uniform(zlo, zhi))
        axes = (rng.uniform(*semi_axes), rng.uniform(*semi_axes), rng.uniform(*semi_axes))
        R = rng.rotation()
        mu = rng.uniform(*mu_range)
        rows.append(_obj(0, c, axes, R, mu - MU_WATER))
    return np.array(rows)


def phantom_for(scan: Scan, kind: str, seed: int = 0, n: int = 60) -> np.ndarray:
    """Default phantom of each workload."""
    zlo = scan.h * (scan.BetaS / (2 * math.pi))
    zhi = scan.h * ((scan.BetaS + scan.views * scan.dBeta) / (2 * math.pi))
    if kind == "shepp_logan":
        return shepp_logan(z_centre=scan.z_centre)
    if kind == "random":
        return random_ellipsoids(seed, n, (zlo, zhi))
    if kind == "water":
        return water_cylinder(half_length=abs(zhi - zlo) + 400.0, z_centre=0.5 * (zlo + zhi))
    raise KeyError(kind)


def projector_args(scan: Scan) -> dict:
    """Geometry of the analytic projector for a scan (fan data, post-flip channels)."""
    return dict(YL=scan.YL, ZL=scan.ZL, ViewN=scan.views, SO=scan.SO, SD=scan.SD, dYA=scan.dYA,
                YLC0=scan.YLC1 - 1.0, dZL=scan.row_height, ZLC0=scan.ZLC1 - 1.0, BetaS=scan.BetaS,
                dBeta=scan.dBeta, h=scan.h)
