"""Earth-ionosphere conductivity model sampled on (direction, altitude) grids.

Same parameters, defaults and ``sample()`` contract as the reference's
``EarthIonosphereMaterial`` and ``SphericalAnomaly`` (materials.py:22-113,
242-326), so checkpoints written by either implementation restore in the
other.  Any object with a compatible ``sample(directions, altitudes_m,
earth_radius_m) -> (sigma, epsilon_r)`` method may be used as a material.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
from numpy.typing import NDArray

from .constants import EPSILON_0

FloatArray = NDArray[np.float64]


@dataclass(frozen=True, slots=True)
class SphericalAnomaly:
    """Multiplicative conductivity anomaly in a spherical volume."""

    latitude_deg: float
    longitude_deg: float
    radius_m: float
    altitude_min_m: float
    altitude_max_m: float
    conductivity_factor: float
    relative_permittivity: float | None = None
    maximum_background_conductivity_s_m: float | None = None
    target_area_m2: float | None = None

    def __post_init__(self) -> None:
        finite = (self.latitude_deg, self.longitude_deg, self.radius_m, self.altitude_min_m, self.altitude_max_m, self.conductivity_factor)
        if not all(np.isfinite(v) for v in finite):
            raise ValueError("anomaly geometry and conductivity must be finite")
        if not -90.0 <= self.latitude_deg <= 90.0:
            raise ValueError("anomaly latitude must be in [-90, 90]")
        if self.radius_m <= 0.0:
            raise ValueError("anomaly radius_m must be positive")
        if self.altitude_min_m > self.altitude_max_m:
            raise ValueError("anomaly altitude bounds are reversed")
        if self.conductivity_factor <= 0.0:
            raise ValueError("conductivity_factor must be positive")
        if self.relative_permittivity is not None and (not np.isfinite(self.relative_permittivity) or self.relative_permittivity <= 0.0):
            raise ValueError("relative permittivity must be finite and positive")
        if self.maximum_background_conductivity_s_m is not None and (
            not np.isfinite(self.maximum_background_conductivity_s_m) or self.maximum_background_conductivity_s_m <= 0.0
        ):
            raise ValueError("maximum background conductivity must be finite and positive")
        if self.target_area_m2 is not None and (not np.isfinite(self.target_area_m2) or self.target_area_m2 <= 0.0):
            raise ValueError("target anomaly area must be finite and positive")

    @property
    def center(self) -> FloatArray:
        lat = np.deg2rad(self.latitude_deg)
        lon = np.deg2rad(self.longitude_deg)
        return np.asarray((np.cos(lat) * np.cos(lon), np.cos(lat) * np.sin(lon), np.sin(lat)), dtype=np.float64)


def apply_spherical_anomalies(sigma, epsilon_r, directions, altitudes_m, earth_radius_m, anomalies) -> None:
    """Point-support anomaly overrides in place (materials.py:89-112)."""

    for a in anomalies:
        horizontal = np.arccos(np.clip(directions @ a.center, -1.0, 1.0)) <= a.radius_m / earth_radius_m
        vertical = (altitudes_m >= a.altitude_min_m) & (altitudes_m <= a.altitude_max_m)
        inside = horizontal[:, None] & vertical[None, :]
        if a.maximum_background_conductivity_s_m is not None:
            inside &= sigma <= a.maximum_background_conductivity_s_m
        sigma[inside] *= a.conductivity_factor
        if a.relative_permittivity is not None:
            epsilon_r[inside] = a.relative_permittivity


@dataclass(frozen=True, slots=True)
class EarthIonosphereMaterial:
    """Homogeneous lithosphere below 0 m and an exponential ionosphere above:
    sigma(h) = prefactor * epsilon_0 * exp((h - H') / zeta)."""

    lithosphere_conductivity_s_m: float = 1.0e-3
    lithosphere_relative_permittivity: float = 10.0
    atmosphere_relative_permittivity: float = 1.0
    ionosphere_reference_height_m: float = 74_000.0
    ionosphere_scale_height_m: float = 6_000.0
    ionosphere_prefactor_hz: float = 2.5e5
    anomalies: tuple[SphericalAnomaly, ...] = field(default_factory=tuple)

    def __post_init__(self) -> None:
        values = (
            self.lithosphere_conductivity_s_m,
            self.lithosphere_relative_permittivity,
            self.atmosphere_relative_permittivity,
            self.ionosphere_reference_height_m,
            self.ionosphere_scale_height_m,
            self.ionosphere_prefactor_hz,
        )
        if not all(np.isfinite(v) for v in values):
            raise ValueError("material parameters must be finite")
        if self.lithosphere_conductivity_s_m < 0.0:
            raise ValueError("lithosphere conductivity cannot be negative")
        if self.lithosphere_relative_permittivity < 1.0:
            raise ValueError("lithosphere relative permittivity must be >= 1")
        if self.atmosphere_relative_permittivity < 1.0:
            raise ValueError("atmosphere relative permittivity must be >= 1")
        if self.ionosphere_scale_height_m <= 0.0:
            raise ValueError("ionosphere scale height must be positive")
        if self.ionosphere_prefactor_hz < 0.0:
            raise ValueError("ionosphere prefactor cannot be negative")

    def sample(self, directions: FloatArray, altitudes_m: FloatArray, earth_radius_m: float) -> tuple[FloatArray, FloatArray]:
        h = np.asarray(altitudes_m, dtype=np.float64)
        exponent = np.clip((h - self.ionosphere_reference_height_m) / self.ionosphere_scale_height_m, -80.0, 80.0)
        air = self.ionosphere_prefactor_hz * EPSILON_0 * np.exp(exponent)
        ground = h < 0.0
        sigma_profile = np.where(ground, self.lithosphere_conductivity_s_m, air)
        eps_profile = np.where(ground, self.lithosphere_relative_permittivity, self.atmosphere_relative_permittivity)
        n = len(directions)
        sigma = np.broadcast_to(sigma_profile, (n, len(h))).copy()
        eps = np.broadcast_to(eps_profile, (n, len(h))).copy()
        apply_spherical_anomalies(sigma, eps, np.asarray(directions, dtype=np.float64), h, earth_radius_m, self.anomalies)
        return sigma, eps
