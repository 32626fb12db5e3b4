"""The benchmark workloads built on the CPU oracle (test and CPU-baseline
infrastructure only).

These are the seeded synthetic inputs of the two plain-solver benchmark
configurations, restated on ``OracleFDTD`` with the oracle's own mesh builder,
so that the CPU legs of ``bench.py`` and the parity tests load nothing of the
CUDA product:

* ``config2``: icosahedral subdivision 7 x 40 radial cells over -100..100 km,
  a volume ground (sigma 1e-2 S/m, eps_r 10), air sigma 0 below 50 km and
  ``min(1e-7 exp((h - 60 km)/4 km), 1e-3)`` S/m above, a Drude electron plasma
  with ``n_e(h) = 1e6 exp((h - 85 km)/3 km)`` m^-3 and
  ``nu(h) = 1e7 exp(-(h - 70 km)/6 km)`` s^-1, and a 50 Hz Gaussian current at
  a seed-chosen vertex;
* ``config4``: subdivision 9 x 80 radial cells over 0..100 km with the same
  air and plasma, a surface-impedance lower boundary over a seeded smooth
  log-normal ground-conductivity map (median 1e-2 S/m) and a 20 Hz source.

Subdivision and radial cells can be lowered for bounded CPU samples.  The
reference has no such workload builder (its users assemble
``GeodesicFDTD`` from a configuration, material, source, surface and plasma
model, ``solver.py:184-198``); the pieces here follow the reference's material
sampling contract (``materials.py:242-326``: ``sample(directions, altitudes,
earth_radius) -> (sigma, eps_r)``).
"""

from __future__ import annotations

import numpy as np

from .fdtd import (EPSILON_0, EarthIonosphereParams, OracleFDTD, OraclePlasma, OracleSource, OracleSpecies, OracleSurface,
                   build_mesh)

ELEMENTARY_CHARGE_C = 1.602_176_634e-19
ELECTRON_MASS_KG = 9.109_383_713_9e-31


class ProfileMaterial:
    """Volume ground below 0 m; air sigma 0 below ``cutoff_m`` and
    ``min(prefactor exp((h - h0)/zeta), cap)`` above it."""

    def __init__(self, ground_sigma=1.0e-2, ground_eps=10.0, cutoff_m=50_000.0, prefactor=1.0e-7, h0_m=60_000.0,
                 zeta_m=4_000.0, cap=1.0e-3):
        self.ground_sigma, self.ground_eps = ground_sigma, ground_eps
        self.cutoff_m, self.prefactor, self.h0_m, self.zeta_m, self.cap = cutoff_m, prefactor, h0_m, zeta_m, cap

    def sample(self, directions, altitudes_m, earth_radius_m):
        h = np.asarray(altitudes_m, dtype=np.float64)
        air = np.minimum(self.prefactor * np.exp((h - self.h0_m) / self.zeta_m), self.cap)
        air = np.where(h < self.cutoff_m, 0.0, air)
        sigma = np.where(h < 0.0, self.ground_sigma, air)
        eps = np.where(h < 0.0, self.ground_eps, 1.0)
        n = len(directions)
        return np.broadcast_to(sigma, (n, len(h))), np.broadcast_to(eps, (n, len(h)))


def smooth_log_normal(directions, seed: int, median: float = 1.0e-2, spread: float = 0.5) -> np.ndarray:
    """Seeded smooth field on the sphere made log-normal around ``median``: the
    eleven monomials of degree <= 3 in (x, y, z), weighted by N(0, 1) draws and
    added one at a time in the order listed, standardised, then exponentiated."""

    d = np.asarray(directions, dtype=np.float64)
    rng = np.random.default_rng(seed)
    x, y, z = (np.ascontiguousarray(d[:, k]) for k in range(3))
    monomials = (
        lambda: x, lambda: y, lambda: z, lambda: x * y, lambda: y * z, lambda: z * x, lambda: x * x - y * y,
        lambda: 3 * z * z - 1, lambda: x * y * z, lambda: x**3 - 3 * x * y * y, lambda: z**3,
    )
    weights = rng.standard_normal(len(monomials))
    field = np.zeros(len(d))
    for w, term in zip(weights, monomials):
        field += w * term()
    field = (field - field.mean()) / max(field.std(), 1e-30)
    return median * np.exp(spread * field)


def drude_plasma(n_faces: int, midpoint_altitudes_m) -> OraclePlasma:
    """Electron plasma with the benchmark's altitude profiles and B = 0."""

    h = np.asarray(midpoint_altitudes_m, dtype=np.float64)
    shape = (n_faces, len(h))
    density = np.broadcast_to(1.0e6 * np.exp((h - 85_000.0) / 3_000.0), shape)
    collision = np.broadcast_to(1.0e7 * np.exp(-(h - 70_000.0) / 6_000.0), shape)
    return OraclePlasma(np.zeros((*shape, 3)), [OracleSpecies(-ELEMENTARY_CHARGE_C, ELECTRON_MASS_KG, density, collision)])


def vertex_lat_lon(vertices, index: int) -> tuple[float, float]:
    """Geographic latitude and longitude (degrees) of one mesh vertex."""

    v = np.asarray(vertices)[index]
    return float(np.degrees(np.arcsin(np.clip(v[2], -1.0, 1.0)))), float(np.degrees(np.arctan2(v[1], v[0])))


def _midpoint_altitudes(lo: float, hi: float, cells: int) -> np.ndarray:
    alt = np.linspace(lo, hi, cells + 1)
    return 0.5 * (alt[:-1] + alt[1:])


def config2(subdivision: int = 7, radial_cells: int = 40, seed: int = 20260805, dtype=np.float32, mesh=None) -> OracleFDTD:
    """The s7 / 40-cell plasma workload on the oracle (fields zero)."""

    mesh = build_mesh(subdivision) if mesh is None else mesh
    lo, hi = -100_000.0, 100_000.0
    lat, lon = vertex_lat_lon(mesh.vertices, int(np.random.default_rng(seed).integers(mesh.n_vertices)))
    return OracleFDTD(
        subdivision=subdivision, radial_cells=radial_cells, minimum_altitude_m=lo, maximum_altitude_m=hi,
        material=ProfileMaterial(), plasma=drude_plasma(mesh.n_faces, _midpoint_altitudes(lo, hi, radial_cells)),
        mesh=mesh, dtype=dtype,
        source=OracleSource(latitude_deg=lat, longitude_deg=lon, peak_current_a=1.0, carrier_frequency_hz=50.0),
    )


def config4(subdivision: int = 9, radial_cells: int = 80, seed: int = 20260814, dtype=np.float32, mesh=None,
            surface_map=None) -> OracleFDTD:
    """The s9 / 80-cell surface-impedance plasma workload on the oracle (fields
    zero); ``surface_map`` overrides the per-edge ground conductivity."""

    mesh = build_mesh(subdivision) if mesh is None else mesh
    lo, hi = 0.0, 100_000.0
    lat, lon = vertex_lat_lon(mesh.vertices, int(np.random.default_rng(seed).integers(mesh.n_vertices)))
    sigma = smooth_log_normal(mesh.edge_midpoints(), seed) if surface_map is None else surface_map
    return OracleFDTD(
        subdivision=subdivision, radial_cells=radial_cells, minimum_altitude_m=lo, maximum_altitude_m=hi,
        material=ProfileMaterial(), plasma=drude_plasma(mesh.n_faces, _midpoint_altitudes(lo, hi, radial_cells)),
        surface=OracleSurface(sigma), mesh=mesh, dtype=dtype,
        source=OracleSource(latitude_deg=lat, longitude_deg=lon, altitude_m=2_500.0, peak_current_a=1.0,
                            carrier_frequency_hz=20.0),
    )


def seed_fields(sim: OracleFDTD, seed: int = 20260814, amplitude: float = 1.0e-6) -> None:
    """Random initial fields (N(0, 1) x amplitude drawn in float64, rounded to
    the oracle's dtype), as the reference benchmark seeds them
    (``benchmarks/backend_matrix.py:179-183``)."""

    rng = np.random.default_rng(seed)
    for f in ("er", "et", "hr", "ht"):
        a = getattr(sim, f)
        a[:] = (amplitude * rng.standard_normal(a.shape)).astype(a.dtype)


def config3_draws(seed: int = 20260803, members: int = 64) -> list[dict]:
    """Seeded per-member parameters of the 64-member ensemble workload, drawn in
    this order per member: subdivision uniform in {5, 6, 7}, radial cells uniform
    in 24-60, sigma0 log-uniform in 1e-8-1e-6 S/m, h0 uniform in 55-70 km, zeta
    uniform in 3-6 km, ground sigma log-uniform in 1e-3-1e-1 S/m, carrier
    uniform in 10-60 Hz, then a source draw and a receiver seed."""

    rng = np.random.default_rng(seed)
    out = []
    for _ in range(members):
        d = {"subdivision": int(rng.integers(5, 8)), "radial_cells": int(rng.integers(24, 61))}
        d["sigma0"] = 10.0 ** rng.uniform(-8.0, -6.0)
        d["h0"] = rng.uniform(55_000.0, 70_000.0)
        d["zeta"] = rng.uniform(3_000.0, 6_000.0)
        d["ground"] = 10.0 ** rng.uniform(-3.0, -1.0)
        d["carrier"] = rng.uniform(10.0, 60.0)
        d["source_draw"] = int(rng.integers(1 << 31))
        d["receiver_seed"] = int(rng.integers(1 << 31))
        out.append(d)
    return out


def config3_member(draw: dict, mesh=None, dtype=np.float32) -> OracleFDTD:
    """One member of the ensemble workload on the oracle (fields zero): the
    exponential ionosphere (``sigma0`` at ``h0``, scale height ``zeta``) over
    a homogeneous ground of conductivity ``ground``, the default -100..100 km
    column, and a Gaussian current of the drawn carrier at vertex
    ``source_draw mod n_vertices``."""

    mesh = build_mesh(draw["subdivision"]) if mesh is None else mesh
    lat, lon = vertex_lat_lon(mesh.vertices, draw["source_draw"] % mesh.n_vertices)
    material = EarthIonosphereParams(
        lithosphere_conductivity_s_m=draw["ground"], ionosphere_reference_height_m=draw["h0"],
        ionosphere_scale_height_m=draw["zeta"], ionosphere_prefactor_hz=draw["sigma0"] / EPSILON_0,
    )
    return OracleFDTD(
        subdivision=draw["subdivision"], radial_cells=draw["radial_cells"], material=material, mesh=mesh, dtype=dtype,
        source=OracleSource(latitude_deg=lat, longitude_deg=lon, peak_current_a=1.0, carrier_frequency_hz=draw["carrier"]),
    )
